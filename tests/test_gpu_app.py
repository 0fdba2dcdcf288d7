"""The reference-style program (khz_app, C++ over the C ABI) prints the reference apps' lines
with the reference's values on the same .dgraph files."""
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT, golden_graph
import orc

APP = os.path.join(ROOT, "openkhuzdulgraph_b200", "khz_app")


def test_usage_without_gpu():
    out = subprocess.run([APP], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


@pytest.mark.gpu
def test_app_output_matches_reference(golden):
    with tempfile.TemporaryDirectory() as td:
        for spec in golden["graphs"][:5]:
            _, n, sym, _, _ = golden_graph(spec)
            path = os.path.join(td, "g.dgraph")
            orc.write_dgraph(path, n, sym)
            for app in orc.REF_APPS:
                ref = spec["apps"][app]
                out = subprocess.run([APP, app, path, "-1", "2", "true"], capture_output=True, text=True,
                                     timeout=300)
                assert out.returncode == 0, out.stderr
                counts = {}
                for pid, c in re.findall(r"Pattern count (\d+): (\d+)", out.stdout):
                    counts[int(pid)] = int(c)
                assert [counts[k] for k in sorted(counts)] == ref["counts"], (spec["name"], app)
                ext = float(re.findall(r"NumExtensions: ([0-9.]+)", out.stdout)[-1])
                assert int(ext) == ref["num_extensions"], (spec["name"], app)
                assert "Average runtime:" in out.stdout


@pytest.mark.gpu
def test_three_fsm_app_prints_the_reference_lines():
    """khz_app kautomine_three_fsm prints three_fsm's per-level lines with the reference's values."""
    import json
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_fsm_golden
    with open(os.path.join(ROOT, "tests", "golden", "fsm.json")) as f:
        case = json.load(f)["cases"][0]
    sym, n, labels = make_fsm_golden.graph_of(case["graph"])
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "fsm.dgraph")
        orc.write_dgraph(path, n, sym, labels)
        out = subprocess.run([APP, "kautomine_three_fsm", path, str(case["threshold"])], capture_output=True,
                             text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = re.findall(r"Number of frequent ([a-z-]+) patterns: (\d+), support sum(?: of them)?: (\d+)", out.stdout)
        assert [(int(a), int(b)) for _, a, b in got] == [(lv["num_frequent"], lv["support_sum"])
                                                           for lv in case["levels"]]
