"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402  (the CPU oracle: test infrastructure)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


def golden_graph(spec):
    """Regenerate a golden graph: canonical pairs, vertex count, symmetric CSR."""
    if spec["kind"] == "er":
        canon, n = orc.er(spec["n"], spec["m"], spec["seed"])
    elif spec["kind"] == "rmat":
        canon, n = orc.rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    else:
        canon = np.array(spec["pairs"], dtype=np.uint32).reshape(-1, 2)
        n = int(canon.max()) + 1
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    return canon, n, sym, off, adj


@pytest.fixture(scope="session")
def oracle_lib():
    orc.lib()
    return orc


@pytest.fixture(scope="session")
def khz_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openkhuzdulgraph_b200 import khz
    ctx = khz.Context(0)
    yield ctx
    ctx.close()
