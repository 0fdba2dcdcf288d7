"""The CPU oracle pinned against the reference's own outputs (tests/golden/golden.json,
produced by the reference's binaries) and against brute-force enumeration."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_graph
import orc

REF_CLIQUES = ["kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique",
               "kgraphpi_triangle", "kgraphpi_four_clique", "kgraphpi_five_clique"]


def _sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def test_golden_graphs_regenerate(golden):
    """The generator + symmetrisation + .dgraph writer reproduce the reference converter's bytes."""
    with tempfile.TemporaryDirectory() as td:
        for spec in golden["graphs"]:
            canon, n, sym, off, adj = golden_graph(spec)
            assert n == spec["n"] and canon.shape[0] == spec["m_undirected"]
            p = os.path.join(td, "g.dgraph")
            orc.write_dgraph(p, n, sym)
            assert _sha(p) == spec["sha256_dgraph"], spec["name"]


def test_orientation_matches_reference_converter(golden):
    with tempfile.TemporaryDirectory() as td:
        for spec in golden["graphs"]:
            if spec["sha256_oriented"] is None:
                continue
            _, n, _, off, adj = golden_graph(spec)
            ooff, oadj, _ = orc.orient(off, adj)
            src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(ooff).astype(np.int64))
            pairs = np.stack([src, oadj], axis=1)
            p = os.path.join(td, "o.dgraph")
            orc.write_dgraph(p, n, pairs)
            assert _sha(p) == spec["sha256_oriented"], spec["name"]


@pytest.mark.parametrize("app", orc.REF_APPS)
def test_oracle_matches_reference_apps(golden, app):
    for spec in golden["graphs"]:
        ref = spec["apps"].get(app)
        if ref is None:
            continue
        _, n, _, off, adj = golden_graph(spec)
        counts, ext, _ = orc.count(app, off, adj, threads=2)
        assert counts == ref["counts"], (spec["name"], app)
        assert ext == ref["num_extensions"], (spec["name"], app)


@pytest.mark.parametrize("app", REF_CLIQUES)
def test_oracle_matches_reference_on_oriented(golden, app):
    for spec in golden["graphs"]:
        ref = spec["apps_oriented"].get(app)
        if ref is None:
            continue
        _, n, _, off, adj = golden_graph(spec)
        ooff, oadj, _ = orc.orient(off, adj)
        counts, ext, _ = orc.count(app, ooff, oadj, threads=2)
        assert counts == ref["counts"], (spec["name"], app)
        assert ext == ref["num_extensions"], (spec["name"], app)


@pytest.mark.parametrize("app", orc.REF_APPS)
def test_oracle_matches_reference_sampled_driver(golden, app):
    mod, rem = golden["sample"]["mod"], golden["sample"]["rem"]
    for spec in golden["graphs"]:
        ref = spec["apps_sampled"].get(app)
        if ref is None:
            continue
        _, n, _, off, adj = golden_graph(spec)
        counts, ext, _ = orc.count(app, off, adj, v0_mod=mod, v0_rem=rem, threads=2)
        assert counts == ref["counts"], (spec["name"], app)
        assert ext == ref["num_extensions"], (spec["name"], app)


@pytest.mark.parametrize("app", orc.REF_APPS)
def test_labeled_oracle_matches_reference_sampled_driver(golden, app):
    """The label-restricted run (raw aggregator values) against the reference's own sampled driver,
    which runs the app with restrict_starting_vertex_label on labels v % mod."""
    mod, rem = golden["sample"]["mod"], golden["sample"]["rem"]
    aid = orc.APPS[app]
    for spec in golden["graphs"]:
        ref = spec["apps_sampled"].get(app)
        if ref is None:
            continue
        _, n, _, off, adj = golden_graph(spec)
        labels = (np.arange(n, dtype=np.uint64) % mod).astype(np.uint32)
        raw, ext, _ = orc.count_labeled(app, off, adj, labels, rem, threads=2)
        mult = [2 if (aid == 3 and p == 1) else 1 for p in range(len(raw))]
        assert [r // m for r, m in zip(raw, mult)] == ref["counts"], (spec["name"], app)
        assert ext == ref["num_extensions"], (spec["name"], app)


def test_label_slices_partition_the_whole_count():
    """Summed over all labels, the restricted runs give the unrestricted raw counts and NumExtensions."""
    canon, n = orc.er(300, 2500, seed=5)
    off, adj = orc.csr(orc.symmetrize(canon), n)
    labels = (np.arange(n, dtype=np.uint64) * 7919 % 5).astype(np.uint32)
    for app in orc.APPS:
        whole, ext, _ = orc.count(app, off, adj, threads=2)
        aid = orc.APPS[app]
        mult = {3: [1, 2], 11: [1, 2, 1, 8, 1, 1]}.get(aid, [1] * len(whole))
        tot, tot_ext = [0] * len(whole), 0
        for lab in range(5):
            raw, e, _ = orc.count_labeled(app, off, adj, labels, lab, threads=2)
            tot = [a + b for a, b in zip(tot, raw)]
            tot_ext += e
        assert [t // m for t, m in zip(tot, mult)] == whole, app
        assert tot_ext == ext, app


# brute-force pattern ids (khz_oracle.h) for each app's counts
BRUTE = {
    "kautomine_triangle": [0], "kautomine_four_clique": [1], "kautomine_five_clique": [2],
    "kautomine_three_motif": [0, 4], "kgraphpi_triangle": [0], "kgraphpi_four_clique": [1],
    "kgraphpi_five_clique": [2], "kgraphpi_three_motif": [0, 3], "kgraphpi_four_cycle": [5],
    "kgraphpi_house": [6], "kgraphpi_tailed_triangle": [7], "kautomine_four_motif": [10, 11, 12, 13, 14, 15],
}


@pytest.mark.parametrize("seed", [3, 4, 11])
def test_oracle_matches_brute_force(seed):
    canon, n = orc.er(30, 160, seed=seed)
    off, adj = orc.csr(orc.symmetrize(canon), n)
    for app, pats in BRUTE.items():
        counts, _, _ = orc.count(app, off, adj, threads=2)
        assert counts == [orc.brute(p, off, adj) for p in pats], app


def test_closed_form_identities():
    """sum C(d,2) = edge-induced wedges; vertex-induced = that - 3 * triangles; 3-stars = sum C(d,3)."""
    canon, n = orc.rmat(9, 8, seed=5)
    off, adj = orc.csr(orc.symmetrize(canon), n)
    d = np.diff(off).astype(np.int64)
    tri = orc.count("kautomine_triangle", off, adj)[0][0]
    kg = orc.count("kgraphpi_three_motif", off, adj)[0]
    ka = orc.count("kautomine_three_motif", off, adj)[0]
    assert kg == [tri, int((d * (d - 1) // 2).sum())]
    assert ka == [tri, kg[1] - 3 * tri]
    motif = orc.count("kautomine_four_motif", off, adj)[0]
    # non-induced 3-stars = induced 3-stars + paws + 2 diamonds + 4 4-cliques
    assert int((d * (d - 1) * (d - 2) // 6).sum()) == motif[0] + motif[2] + 2 * motif[4] + 4 * motif[5]


def _ref_setops(a, b, ub):
    A, B = list(a), set(b)
    return {
        "intersect": [x for x in A if x in B] if len(a) and len(b) else [],
        "subtract": [x for x in A if x not in B],
        "bounded_intersect": [x for x in A if x < ub and x in B] if len(a) and len(b) else [],
        "bounded_subtract": [x for x in A if x < ub and x not in B],
        "trim": sum(1 for x in A if x < ub),
        "trim_lower_bound": sum(1 for x in A if x <= ub),
    }


def test_oracle_set_ops_edge_cases():
    L = orc.lib()
    rng = np.random.default_rng(0)
    cases = [([], []), ([1, 2, 3], []), ([], [4, 5]), ([5], [5]), ([0, 2**32 - 1], [2**32 - 1])]
    for _ in range(50):
        a = np.unique(rng.integers(0, 200, rng.integers(0, 60)))
        b = np.unique(rng.integers(0, 200, rng.integers(0, 60)))
        cases.append((a.tolist(), b.tolist()))
    for a, b in cases:
        A = np.array(a + [0], dtype=np.uint32)
        B = np.array(b + [0], dtype=np.uint32)
        out = np.zeros(len(a) + 1, dtype=np.uint32)
        ub = 100
        exp = _ref_setops(a, b, ub)
        r = L.orc_intersect(A, len(a), B, len(b), out)
        assert out[:r].tolist() == exp["intersect"]
        assert L.orc_intersect_count(A, len(a), B, len(b)) == len(exp["intersect"])
        r = L.orc_subtract(A, len(a), B, len(b), out)
        assert out[:r].tolist() == exp["subtract"]
        r = L.orc_bounded_intersect(A, len(a), B, len(b), ub, out)
        assert out[:r].tolist() == exp["bounded_intersect"]
        r = L.orc_bounded_subtract(A, len(a), B, len(b), ub, out)
        assert out[:r].tolist() == exp["bounded_subtract"]
        assert L.orc_trim(A, len(a), ub) == exp["trim"]
        assert L.orc_trim_lower_bound(A, len(a), ub) == exp["trim_lower_bound"]


def test_rmat_generator_properties():
    canon, n = orc.rmat(10, 8, seed=9)
    assert (canon[:, 0] < canon[:, 1]).all()
    keys = canon[:, 0].astype(np.uint64) << np.uint64(32) | canon[:, 1].astype(np.uint64)
    assert (np.diff(keys.astype(np.int64)) > 0).all()
    present = np.zeros(n, dtype=bool)
    present[canon.ravel()] = True
    assert present.all() and canon.max() == n - 1
