"""The oracle's 3-FSM restatement (oracle/khz_oracle.c orc_fsm, following kautomine/three_fsm.cc)
against the reference's own three_fsm app (tests/golden/fsm.json, written by
tests/golden/make_fsm_golden.py from oracle/_ref/kautomine_three_fsm): per level, the number of
frequent patterns and the support sum.  CPU only."""
import json
import os
import sys

import numpy as np

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_fsm_golden  # noqa: E402
import orc  # noqa: E402


def _cases():
    with open(os.path.join(ROOT, "tests", "golden", "fsm.json")) as f:
        return json.load(f)["cases"]


def test_oracle_fsm_matches_reference_app():
    graphs = {}
    for case in _cases():
        spec = case["graph"]
        if spec["name"] not in graphs:
            sym, n, labels = make_fsm_golden.graph_of(spec)
            off, adj = orc.csr(sym, n)
            graphs[spec["name"]] = (off, adj, labels)
        off, adj, labels = graphs[spec["name"]]
        got = orc.fsm(off, adj, labels, case["threshold"])
        for lv, (g, exp) in enumerate(zip(got, case["levels"])):
            assert g["num_frequent"] == exp["num_frequent"], (spec["name"], case["threshold"], lv, g, exp)
            assert g["support_sum"] == exp["support_sum"], (spec["name"], case["threshold"], lv, g, exp)


def test_oracle_fsm_edge_cases():
    """A path 0 - 1 - 2 - 3 labelled (0, 1, 1, 0), worked out by hand from three_fsm.cc's rules."""
    pairs = np.array([[0, 1], [1, 0], [1, 2], [2, 1], [2, 3], [3, 2]], dtype=np.uint32)
    off, adj = orc.csr(pairs, 4)
    labels = np.array([0, 1, 1, 0], dtype=np.uint32)
    for threshold in (1, 2):
        lv = orc.fsm(off, adj, labels, threshold)
        # edges: candidates (0,0) (0,1) (1,1), the last two with 2 images per position;
        # wedges: candidates (0,1,1) (1,0,0) (1,0,1) (1,1,1), only (1,0,1) embeds (centres 1 and 2);
        # no triangle candidate; four-chain (1,1,0,0) = 0 - 1 - 2 - 3 both ways; no three-star candidate
        assert [(x["num_candidates"], x["num_frequent"], x["support_sum"]) for x in lv] == [
            (2, 2, 4), (3, 2, 4), (4, 1, 2), (0, 0, 0), (1, 1, 2), (0, 0, 0)]
    # a threshold above every support leaves the levels empty; level 0 still sums every label
    lv = orc.fsm(off, adj, labels, 5)
    assert [x["num_frequent"] for x in lv] == [0, 0, 0, 0, 0, 0]
    assert lv[0]["support_sum"] == 4
