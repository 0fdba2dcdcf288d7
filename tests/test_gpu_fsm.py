"""3-FSM on the device against the reference's own three_fsm app (tests/golden/fsm.json, written by
tests/golden/make_fsm_golden.py from oracle/_ref/kautomine_three_fsm): per level, the number of
frequent patterns and the support sum must be the app's."""
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_fsm_golden  # noqa: E402  (the fixture's graph definitions)


def _cases():
    with open(os.path.join(ROOT, "tests", "golden", "fsm.json")) as f:
        return json.load(f)["cases"]


def test_fsm_matches_reference_app(khz_ctx):
    graphs = {}
    try:
        for case in _cases():
            spec = case["graph"]
            if spec["name"] not in graphs:
                sym, n, labels = make_fsm_golden.graph_of(spec)
                g = khz_ctx.graph_from_edges(sym, n)
                g.set_labels(labels)
                graphs[spec["name"]] = g
            levels, patterns, _ = khz_ctx.fsm(graphs[spec["name"]], case["threshold"])
            for lv, (got, exp) in enumerate(zip(levels, case["levels"])):
                assert got["num_frequent"] == exp["num_frequent"], (spec["name"], case["threshold"], lv)
                assert got["support_sum"] == exp["support_sum"], (spec["name"], case["threshold"], lv)
            assert len(patterns) == sum(lv["num_frequent"] for lv in levels)
            assert all(s >= case["threshold"] for _, _, s in patterns)
    finally:
        for g in graphs.values():
            g.free()


def test_fsm_needs_labels(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    import orc
    canon, n = orc.er(50, 100, seed=1)
    g = khz_ctx.graph_from_edges(orc.symmetrize(canon), n)
    with pytest.raises(khz.KhzError) as e:
        khz_ctx.fsm(g, 5)
    assert e.value.status == 1
    g.free()


def test_fsm_needs_symmetric_graph(khz_ctx):
    """The domains assume the undirected CSR: a graph stored one way round is refused."""
    from openkhuzdulgraph_b200 import khz
    import orc
    canon, n = orc.er(60, 150, seed=2)
    g = khz_ctx.graph_from_edges(canon, n)
    try:
        g.set_labels(np.arange(n, dtype=np.uint32) % 3)
        with pytest.raises(khz.KhzError) as e:
            khz_ctx.fsm(g, 5)
        assert e.value.status == 1
    finally:
        g.free()


def _skewed_labels(n, num_labels, mult=7919):
    """label l with weight l + 1, spread over the ids by a multiplier coprime to the weight sum"""
    r = (np.arange(n, dtype=np.uint64) * mult) % (num_labels * (num_labels + 1) // 2)
    return np.searchsorted(np.cumsum(np.arange(1, num_labels + 1)), r, side="right").astype(np.uint32)


# (scale, edge factor, labels, threshold divisor): thresholds n // divisor prune some candidates at
# every level; up to 4 272 four-chain candidates (12 labels).  Seed 12: the golden fixture holds the
# reference's own results for the same shapes on seed 11.
_ORACLE_CASES = [(14, 16, 2, 3), (14, 16, 3, 4), (14, 16, 5, 6), (14, 16, 8, 10), (14, 16, 8, 40),
                 (13, 16, 12, 60), (15, 8, 4, 5), (16, 8, 6, 12)]


def test_fsm_matches_oracle_on_larger_graphs(khz_ctx):
    """The device's levels (candidates, frequent patterns, support sums) against the oracle's
    restatement (orc_fsm) on labelled R-MAT graphs of 6 500 to 40 000 vertices with skewed labels."""
    import orc
    for scale, ef, num_labels, div in _ORACLE_CASES:
        canon, n = orc.rmat(scale, ef, seed=12)
        sym = orc.symmetrize(canon)
        off, adj = orc.csr(sym, n)
        labels = _skewed_labels(n, num_labels)
        threshold = max(1, n // div)
        want = orc.fsm(off, adj, labels, threshold)
        g = khz_ctx.graph_from_edges(sym, n)
        try:
            g.set_labels(labels)
            got, _, _ = khz_ctx.fsm(g, threshold)
        finally:
            g.free()
        assert [(x["num_candidates"], x["num_frequent"], x["support_sum"]) for x in got] == \
            [(x["num_candidates"], x["num_frequent"], x["support_sum"]) for x in want], (scale, ef, num_labels, div)
