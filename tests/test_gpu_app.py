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
