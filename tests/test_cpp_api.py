"""The C++ surfaces a reference app compiles against: main_template.h's INSERT_MAIN_FUNCTION with a
mining_graph on the device (include/khz_main_template.h), and a schedule built with the
Khuzdul::Schedule builder and registered from C++ (include/khz_khuzdul.hpp).  The programs are
compiled here with g++ against the in-tree library; the runs need a GPU."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden_graph
import orc

PKG = os.path.join(ROOT, "openkhuzdulgraph_b200")

MINING_APP = r"""
#include "khz_main_template.h"
KHZ_MINING_FUNCTION(KHZ_KAUTO_4CLIQUE)
INSERT_MAIN_FUNCTION(four_clique)
"""

SCHEDULE_APP = r"""
#include <cstdio>
#include "khz_khuzdul.hpp"
using namespace Khuzdul;
int main(int argc, char **argv) {
    // the non-induced 3-star: v1 in N(v0); v2 in N(v0) above v1; count N(v0) above v2
    Schedule star(4);
    star.Level(Term(SetExpr::N(0)))
        .Level(Term(SetExpr::N(0)).Above({1}))
        .Count(Term(SetExpr::N(0)).Above({2}));
    // the kautomine 3-motif, fused: triangles above v1 (guarded v0 < v1) and N(v0) \ N(v1)
    Schedule motif(3);
    motif.Level(Term(SetExpr::N(0)))
        .Count(Term(SetExpr::N(0).And(1)).Above({1}).Into(0).OnlyIf(0, 1))
        .Count(Term(SetExpr::N(0).Sub(1)).Except({1}).Into(1));
    try {
        const khz_app_id a = register_app({star}, {1});
        const khz_app_id b = register_app({motif}, {1, 2});
        if (argc < 2) { printf("registered %d %d\n", (int)a, (int)b); return 0; }
        DistributedApplication app(-1, argv[1], 4, a);
        Aggregator<EdgeId> *cnt = app.alloc_aggregator<EdgeId>();
        app.run();
        printf("star %lu ext %lu\n", (unsigned long)cnt->evaluate(), (unsigned long)app.num_extensions());
        DistributedApplication app2(-1, argv[1], 3, b);
        Aggregator<EdgeId> *t = app2.alloc_aggregator<EdgeId>();
        Aggregator<EdgeId> *w = app2.alloc_aggregator<EdgeId>();
        app2.run();
        printf("motif %lu %lu\n", (unsigned long)t->evaluate(), (unsigned long)(w->evaluate() / 2));
    } catch (const Error &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
"""


def _build(td, name, src):
    path = os.path.join(td, name + ".cpp")
    with open(path, "w") as f:
        f.write(src)
    exe = os.path.join(td, name)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
                    path, "-o", exe, "-L" + PKG, "-lkhz_b200", "-Wl,-rpath," + PKG], check=True,
                   capture_output=True, text=True)
    return exe


def test_programs_compile_and_register_without_gpu():
    with tempfile.TemporaryDirectory() as td:
        mining = _build(td, "mining", MINING_APP)
        out = subprocess.run([mining], capture_output=True, text=True)
        assert out.returncode != 0 and "usage: four_clique" in out.stdout
        sched = _build(td, "sched", SCHEDULE_APP)
        out = subprocess.run([sched], capture_output=True, text=True)  # registration needs no device
        assert out.returncode == 0 and re.match(r"registered 1[2-9]|registered [2-9]\d", out.stdout), out


@pytest.mark.gpu
def test_programs_count_on_the_device(golden):
    spec = golden["graphs"][0]
    _, n, sym, off, _ = golden_graph(spec)
    d = np.diff(off.astype(np.int64))
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "g.dgraph")
        orc.write_dgraph(path, n, sym)
        out = subprocess.run([_build(td, "mining", MINING_APP), path], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        assert ("four_clique result: %d" % spec["apps"]["kautomine_four_clique"]["counts"][0]) in out.stdout
        out = subprocess.run([_build(td, "sched", SCHEDULE_APP), path], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        star = int((d * (d - 1) * (d - 2) // 6).sum())
        ext = int(n + d.sum() + (d * (d - 1) // 2).sum())
        assert "star %d ext %d" % (star, ext) in out.stdout
        motif = spec["apps"]["kautomine_three_motif"]["counts"]
        assert "motif %d %d" % (motif[0], motif[1]) in out.stdout
