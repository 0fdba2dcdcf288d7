"""Parity of the CUDA engine (through the C ABI) with the reference's outputs and the oracle.

Counts and NumExtensions are integers: every comparison is exact.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_graph
import orc

pytestmark = pytest.mark.gpu

ALL_APPS = list(orc.APPS)
CLIQUES = ["kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique",
           "kgraphpi_triangle", "kgraphpi_four_clique", "kgraphpi_five_clique"]


@pytest.fixture(scope="module")
def graphs(golden, khz_ctx):
    out = []
    for spec in golden["graphs"]:
        canon, n, sym, off, adj = golden_graph(spec)
        g = khz_ctx.graph_from_edges(sym, n)
        out.append((spec, n, sym, off, adj, g))
    return out


def test_csr_build_matches_oracle(graphs):
    for spec, n, sym, off, adj, g in graphs:
        goff, gadj = g.export_csr()
        assert np.array_equal(goff, off), spec["name"]
        assert np.array_equal(gadj, adj), spec["name"]
        assert g.info().max_degree == int(np.diff(off).max())


def test_orientation_matches_oracle(graphs, khz_ctx):
    for spec, n, sym, off, adj, g in graphs:
        og = g.orient()
        ooff, oadj, _ = orc.orient(off, adj)
        goff, gadj = og.export_csr()
        assert np.array_equal(goff, ooff), spec["name"]
        assert np.array_equal(gadj, oadj), spec["name"]
        og.free()


def test_write_dgraph_matches_reference_bytes(graphs, khz_ctx):
    import hashlib
    with tempfile.TemporaryDirectory() as td:
        for spec, n, sym, off, adj, g in graphs:
            p = os.path.join(td, "g.dgraph")
            g.write_dgraph(p)
            with open(p, "rb") as f:
                assert hashlib.sha256(f.read()).hexdigest() == spec["sha256_dgraph"], spec["name"]
            if spec["sha256_oriented"]:
                og = g.orient()
                og.write_dgraph(p)
                with open(p, "rb") as f:
                    assert hashlib.sha256(f.read()).hexdigest() == spec["sha256_oriented"], spec["name"]
                og.free()


def test_load_dgraph(graphs, khz_ctx):
    with tempfile.TemporaryDirectory() as td:
        spec, n, sym, off, adj, _ = graphs[2]
        p = os.path.join(td, "g.dgraph")
        orc.write_dgraph(p, n, sym, labels=np.arange(n, dtype=np.uint32) % 3)
        g = khz_ctx.load_dgraph(p)
        goff, gadj = g.export_csr()
        assert np.array_equal(goff, off) and np.array_equal(gadj, adj)
        g.free()


@pytest.mark.parametrize("engine", ["auto", "dfs"])
@pytest.mark.parametrize("app", ALL_APPS)
def test_counts_match_reference(graphs, golden, khz_ctx, app, engine):
    """Symmetric input: counts and NumExtensions equal the reference apps' (golden) or the oracle's."""
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_AUTO if engine == "auto" else khz.ENGINE_DFS, want_algo_bytes=0)
    for spec, n, sym, off, adj, g in graphs:
        counts, st = khz_ctx.count(g, app)
        ref = spec["apps"].get(app)
        if ref is not None:
            assert counts == ref["counts"], (spec["name"], app)
            assert st.num_extensions == ref["num_extensions"], (spec["name"], app)
        else:
            oc, oext, _ = orc.count(app, off, adj)
            assert counts == oc, (spec["name"], app)
            assert st.num_extensions == oext, (spec["name"], app)
    khz_ctx.set_config(engine=khz.ENGINE_AUTO)


@pytest.mark.parametrize("app", ALL_APPS)
def test_algorithmic_bytes_match_oracle(graphs, khz_ctx, app):
    """The instrumented DFS variant sums the same set-op sizes as the restated schedule."""
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_DFS, want_algo_bytes=1)
    try:
        for spec, n, sym, off, adj, g in graphs[:5]:
            counts, st = khz_ctx.count(g, app)
            oc, oext, obytes = orc.count(app, off, adj)
            assert counts == oc and st.num_extensions == oext
            assert st.algo_bytes == obytes, (spec["name"], app)
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, want_algo_bytes=0)


@pytest.mark.parametrize("engine", ["bitmap", "dfs"])
@pytest.mark.parametrize("app", CLIQUES)
def test_cliques_on_oriented_input(graphs, golden, khz_ctx, app, engine):
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_BITMAP if engine == "bitmap" else khz.ENGINE_DFS, want_algo_bytes=1)
    try:
        for spec, n, sym, off, adj, g in graphs:
            og = khz_ctx.graph_from_edges(sym, n, orient=True)
            counts, st = khz_ctx.count(og, app)
            ooff, oadj, _ = orc.orient(off, adj)
            oc, oext, obytes = orc.count(app, ooff, oadj)
            ref = spec["apps_oriented"].get(app)
            if ref is not None:
                assert oc == ref["counts"] and oext == ref["num_extensions"]
            assert counts == oc, (spec["name"], app, engine)
            assert st.num_extensions == oext, (spec["name"], app, engine)
            assert st.algo_bytes == obytes, (spec["name"], app, engine)
            og.free()
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, want_algo_bytes=0)


def test_rmat_generator_matches_oracle(khz_ctx):
    for scale, ef, seed in [(8, 4, 1), (10, 8, 3), (12, 16, 2)]:
        canon, n = orc.rmat(scale, ef, seed=seed)
        off, adj = orc.csr(orc.symmetrize(canon), n)
        g = khz_ctx.generate_rmat(scale, ef, seed=seed)
        goff, gadj = g.export_csr()
        assert np.array_equal(goff, off) and np.array_equal(gadj, adj), (scale, ef, seed)
        g.free()


def test_invalid_inputs_are_rejected(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    bad_sets = [
        np.array([[1, 0], [0, 1]], dtype=np.uint32),   # unsorted
        np.array([[0, 1], [0, 1]], dtype=np.uint32),   # duplicate
        np.array([[0, 0]], dtype=np.uint32),           # self-loop
        np.array([[0, 5]], dtype=np.uint32),           # id >= n
    ]
    for pairs in bad_sets:
        with pytest.raises(khz.KhzError) as e:
            khz_ctx.graph_from_edges(pairs, 3)
        assert e.value.status == 6
    g = khz_ctx.graph_from_edges(np.array([[0, 1], [1, 0]], dtype=np.uint32), 2)
    with pytest.raises(khz.KhzError) as e:
        khz_ctx.count(g, 77)
    assert e.value.status == 1
    g.free()
    with pytest.raises(khz.KhzError):
        khz_ctx.count(g, 0)
    # empty graph and isolated vertices
    e0 = khz_ctx.graph_from_edges(np.zeros((0, 2), dtype=np.uint32), 5)
    for app in ALL_APPS:
        counts, st = khz_ctx.count(e0, app)
        assert all(c == 0 for c in counts) and st.num_extensions == 5 * {7: 2, 11: 6}.get(orc.APPS[app], 1)
    e0.free()


def test_set_op_batch_matches_oracle(khz_ctx):
    import torch
    from openkhuzdulgraph_b200 import khz
    rng = np.random.default_rng(1)
    lists_a, lists_b = [[], [1, 2, 3], [], [5], [0, 2**32 - 1]], [[], [], [4, 5], [5], [2**32 - 1]]
    for _ in range(300):
        sa = int(rng.choice([0, 3, 40, 300, 2000]))
        sb = int(rng.choice([0, 5, 50, 700, 5000]))
        lists_a.append(np.unique(rng.integers(0, 6000, sa)).tolist())
        lists_b.append(np.unique(rng.integers(0, 6000, sb)).tolist())
    a_off = np.cumsum([0] + [len(x) for x in lists_a]).astype(np.int64)
    b_off = np.cumsum([0] + [len(x) for x in lists_b]).astype(np.int64)
    a = np.array(sum(lists_a, []) + [0], dtype=np.uint32)
    b = np.array(sum(lists_b, []) + [0], dtype=np.uint32)
    bounds = rng.integers(0, 6000, len(lists_a)).astype(np.uint32)
    dev = "cuda"
    ta_off, tb_off = torch.from_numpy(a_off).to(dev), torch.from_numpy(b_off).to(dev)
    ta, tb = torch.from_numpy(a.view(np.int32)).to(dev), torch.from_numpy(b.view(np.int32)).to(dev)
    tbound = torch.from_numpy(bounds.view(np.int32)).to(dev)
    L = orc.lib()
    for op in ["intersect", "subtract", "intersect_count", "bounded_intersect", "bounded_subtract", "trim",
               "trim_lower_bound"]:
        out = torch.zeros(max(len(a), 1), dtype=torch.int32, device=dev)
        out_len = torch.zeros(len(lists_a), dtype=torch.int32, device=dev)
        khz.set_op_batch(op, ta_off, ta, tb_off, tb, tbound, out, out_len)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        glen = out_len.cpu().numpy().view(np.uint32)
        for i, (la, lb) in enumerate(zip(lists_a, lists_b)):
            A = np.array(la + [0], dtype=np.uint32)
            B = np.array(lb + [0], dtype=np.uint32)
            buf = np.zeros(len(la) + 1, dtype=np.uint32)
            ub = int(bounds[i])
            if op == "intersect":
                r = L.orc_intersect(A, len(la), B, len(lb), buf)
            elif op == "subtract":
                r = L.orc_subtract(A, len(la), B, len(lb), buf)
            elif op == "intersect_count":
                r = L.orc_intersect_count(A, len(la), B, len(lb))
            elif op == "bounded_intersect":
                r = L.orc_bounded_intersect(A, len(la), B, len(lb), ub, buf)
            elif op == "bounded_subtract":
                r = L.orc_bounded_subtract(A, len(la), B, len(lb), ub, buf)
            elif op == "trim":
                r = L.orc_trim(A, len(la), ub)
            else:
                r = L.orc_trim_lower_bound(A, len(la), ub)
            assert glen[i] == r, (op, i)
            if op in ("intersect", "subtract", "bounded_intersect", "bounded_subtract"):
                s = int(a_off[i])
                assert got[s:s + r].tolist() == buf[:r].tolist(), (op, i)


BATCH_APPS = ["kautomine_triangle", "kautomine_four_clique", "kgraphpi_four_cycle", "kautomine_three_motif",
              "kgraphpi_five_clique", "kautomine_four_motif"]


def test_batch_matches_single(graphs, khz_ctx):
    """Uneven batch (8 graphs x 6 apps, clique jobs on the bitmap engine, the rest on the DFS
    engine, plus oriented inputs) in one launch sequence == one count per job."""
    jobs, extra = [], []
    for spec, n, sym, off, adj, g in graphs:
        for app in BATCH_APPS:
            jobs.append((g, app))
        og = khz_ctx.graph_from_edges(sym, n, orient=True)
        extra.append(og)
        jobs.append((og, "kautomine_four_clique"))
    counts, exts, st = khz_ctx.count_batch(jobs)
    for (g, app), c, e in zip(jobs, counts, exts):
        c1, st1 = khz_ctx.count(g, app)
        assert c == c1 and e == st1.num_extensions, app
    for og in extra:
        og.free()


def test_batch_cuda_graph_replay(graphs, khz_ctx):
    from openkhuzdulgraph_b200 import khz
    jobs = [(g, app) for spec, n, sym, off, adj, g in graphs[:5] for app in BATCH_APPS]
    expect = [khz_ctx.count(g, app) for g, app in jobs]
    for cuda_graph in (False, True):
        b = khz.Batch(khz_ctx, jobs, cuda_graph=cuda_graph)
        try:
            for _ in range(2):  # replays reuse the batch's scratch
                b.launch()
                counts, exts = b.wait()
                for (c, st), c2, e2 in zip(expect, counts, exts):
                    assert c == c2 and st.num_extensions == e2
        finally:
            b.close()


def test_deterministic_repeat(graphs, khz_ctx):
    g = graphs[3][5]
    a = [khz_ctx.count(g, app)[0] for app in ALL_APPS]
    b = [khz_ctx.count(g, app)[0] for app in ALL_APPS]
    assert a == b


def test_graph_shape_detection_and_as_stored_semantics(graphs, khz_ctx):
    """An oriented edge list is counted as stored (bitmap engine); a directed graph that is
    neither symmetric nor a DAG runs the schedule as stored, like the reference does."""
    spec, n, sym, off, adj, g = graphs[3]
    gi = g.info()
    assert gi.symmetric == 1 and gi.oriented == 0
    ooff, oadj, _ = orc.orient(off, adj)
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(ooff).astype(np.int64))
    og = khz_ctx.graph_from_edges(np.stack([src, oadj], axis=1), n)
    oi = og.info()
    assert oi.oriented == 1 and oi.symmetric == 0
    for app in CLIQUES:
        assert khz_ctx.count(og, app)[0] == orc.count(app, ooff, oadj)[0], app
    og.free()
    # a directed graph: keep (u, v) when (u + v) is even or u < v
    keep = ((sym[:, 0] + sym[:, 1]) % 2 == 0) | (sym[:, 0] < sym[:, 1])
    dpairs = np.ascontiguousarray(sym[keep])
    doff, dadj = orc.csr(dpairs, n)
    dg = khz_ctx.graph_from_edges(dpairs, n)
    di = dg.info()
    assert di.oriented == 0 and di.symmetric == 0
    from openkhuzdulgraph_b200 import khz
    for app in ALL_APPS:
        try:
            exp, ext, _ = orc.count(app, doff, dadj)
        except RuntimeError:
            # the raw count is not divisible by the multiplicity: the reference asserts here
            with pytest.raises(khz.KhzError) as e:
                khz_ctx.count(dg, app)
            assert e.value.status == 9, app
            continue
        got, st = khz_ctx.count(dg, app)
        assert got == exp and st.num_extensions == ext, app
    dg.free()


def test_bitmap_large_tier_matches_oracle(khz_ctx):
    """A dense graph whose oriented out-degrees reach the large block tier (> 256)."""
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.er(1500, 250000, seed=5)
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    ooff, oadj, _ = orc.orient(off, adj)
    assert int(np.diff(ooff).max()) > 256
    og = khz_ctx.graph_from_edges(sym, n, orient=True)
    try:
        for app in ["kautomine_triangle", "kautomine_four_clique"]:
            khz_ctx.set_config(engine=khz.ENGINE_BITMAP)
            got, st = khz_ctx.count(og, app)
            exp, ext, _ = orc.count(app, ooff, oadj)
            assert got == exp and st.num_extensions == ext, app
            assert st.phase_launches[2] == 1  # the large tier ran
        # a launch prepared later with less shared memory must not invalidate this graph's cached one
        canon2, n2 = orc.rmat(9, 16, seed=3)
        small = khz_ctx.graph_from_edges(orc.symmetrize(canon2), n2, orient=True)
        khz_ctx.count(small, "kautomine_four_clique")
        small.free()
        got, st = khz_ctx.count(og, "kautomine_four_clique")
        assert got == orc.count("kautomine_four_clique", ooff, oadj)[0]
        khz_ctx.set_config(engine=khz.ENGINE_BITMAP)
        b5, sb = khz_ctx.count(og, "kautomine_five_clique")
        khz_ctx.set_config(engine=khz.ENGINE_DFS)
        d5, sd = khz_ctx.count(og, "kautomine_five_clique")
        assert b5 == d5 and sb.num_extensions == sd.num_extensions
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        og.free()


@pytest.mark.timeout(900, method="thread")
def test_tensor_core_four_clique_matches(khz_ctx):
    """bitmap_tensor_cores = 1: the large tiers count 4-cliques as a masked 0/1 matrix product on the
    tensor cores.  Dense ER (out-degrees up to ~700, both large tiers, row blocks of 128 with ragged
    ends) against the oracle; an R-MAT s18 against the CUDA-core count; 5-clique and triangle jobs
    of the same launches stay on the CUDA cores and keep their counts."""
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.er(1500, 250000, seed=5)
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    ooff, oadj, _ = orc.orient(off, adj)
    og = khz_ctx.graph_from_edges(sym, n, orient=True)
    rm = khz_ctx.generate_rmat(18, 16, seed=1)
    rog = rm.orient()
    try:
        khz_ctx.set_config(engine=khz.ENGINE_BITMAP, bitmap_tensor_cores=1)
        got, st = khz_ctx.count(og, "kautomine_four_clique")
        exp, ext, _ = orc.count("kautomine_four_clique", ooff, oadj)
        assert got == exp and st.num_extensions == ext
        assert st.phase_launches[2] >= 1
        tc = {app: khz_ctx.count(rog, app) for app in ["kautomine_four_clique", "kgraphpi_four_clique",
                                                        "kautomine_five_clique", "kautomine_triangle"]}
        batch, exts, _ = khz_ctx.count_batch([(rog, "kautomine_five_clique"), (rog, "kautomine_four_clique"),
                                             (og, "kgraphpi_four_clique")])
        khz_ctx.set_config(engine=khz.ENGINE_BITMAP, bitmap_tensor_cores=0)
        for app, (c, s) in tc.items():
            c0, s0 = khz_ctx.count(rog, app)
            assert c == c0 and s.num_extensions == s0.num_extensions, app
        assert batch[1] == tc["kautomine_four_clique"][0] and batch[2] == exp
        assert batch[0] == tc["kautomine_five_clique"][0]
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, bitmap_tensor_cores=0)
        og.free()
        rog.free()
        rm.free()


@pytest.mark.parametrize("hub_rows", [64, 992, 1 << 30])
def test_hub_triangle_matches_oracle(graphs, khz_ctx, hub_rows):
    """Rows of hub vertices read from the hub adjacency triangle (here forced on small graphs, up
    to every vertex a hub) give the oracle's counts, NumExtensions and algorithmic bytes."""
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.er(1500, 250000, seed=5)
    dense = orc.symmetrize(canon)
    cases = [(spec["name"], n_, sym) for spec, n_, sym, _, _, _ in graphs] + [("er_n1500_dense", n, dense)]
    khz_ctx.set_config(engine=khz.ENGINE_BITMAP, want_algo_bytes=1, bitmap_hub_rows=hub_rows)
    try:
        for name, n_, sym in cases:
            off, adj = orc.csr(sym, n_)
            ooff, oadj, _ = orc.orient(off, adj)
            og = khz_ctx.graph_from_edges(sym, n_, orient=True)
            try:
                for app in ["kautomine_triangle", "kautomine_four_clique", "kgraphpi_five_clique"]:
                    got, st = khz_ctx.count(og, app)
                    exp, ext, byt = orc.count(app, ooff, oadj)
                    assert got == exp and st.num_extensions == ext and st.algo_bytes == byt, (name, app)
            finally:
                og.free()
        # 3-motif on symmetric input: triangles of the oriented view through the same path
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, want_algo_bytes=0, bitmap_hub_rows=hub_rows)
        g = khz_ctx.graph_from_edges(dense, n)
        try:
            off, adj = orc.csr(dense, n)
            for app in ["kautomine_three_motif", "kgraphpi_three_motif"]:
                got, st = khz_ctx.count(g, app)
                exp, ext, _ = orc.count(app, off, adj)
                assert got == exp and st.num_extensions == ext, app
        finally:
            g.free()
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, want_algo_bytes=0, bitmap_hub_rows=0)


def test_bitmap_overflow_tier_complete_graph(khz_ctx):
    """K_1250: out-degrees up to 1249 exceed the block tier, so the heaviest start vertices go to
    the DFS engine; counts and NumExtensions follow from binomial coefficients."""
    from math import comb
    from openkhuzdulgraph_b200 import khz
    n = 1250
    iu = np.triu_indices(n, 1)
    canon = np.stack([iu[0], iu[1]], axis=1).astype(np.uint32)
    g = khz_ctx.graph_from_edges(orc.symmetrize(canon), n)
    m = comb(n, 2)
    try:
        for engine in [khz.ENGINE_AUTO, khz.ENGINE_DFS]:
            khz_ctx.set_config(engine=engine)
            got, st = khz_ctx.count(g, "kautomine_triangle")
            assert got == [comb(n, 3)] and st.num_extensions == n + m
            got, st = khz_ctx.count(g, "kautomine_four_clique")
            assert got == [comb(n, 4)] and st.num_extensions == n + m + comb(n, 3)
            if engine == khz.ENGINE_AUTO:
                assert st.phase_launches[3] == 1  # overflow start vertices ran on the DFS engine
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        g.free()


def test_wedge_engine_matches_dfs_engine(khz_ctx):
    """4-cycle on a skewed R-MAT (hub start vertices reach the global-memory tier): the wedge
    engine and the DFS engine (the schedule as written) agree on counts and NumExtensions."""
    from openkhuzdulgraph_b200 import khz
    g = khz_ctx.generate_rmat(14, 16, seed=4)
    try:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        w, sw = khz_ctx.count(g, "kgraphpi_four_cycle")
        assert sw.engine == khz.ENGINE_WEDGE
        khz_ctx.set_config(engine=khz.ENGINE_DFS)
        d, sd = khz_ctx.count(g, "kgraphpi_four_cycle")
        assert w == d and sw.num_extensions == sd.num_extensions
        # and on a small graph against the oracle
        canon, n = orc.rmat(11, 16, seed=6)
        sym = orc.symmetrize(canon)
        off, adj = orc.csr(sym, n)
        g2 = khz_ctx.graph_from_edges(sym, n)
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        got, st = khz_ctx.count(g2, "kgraphpi_four_cycle")
        exp, ext, _ = orc.count("kgraphpi_four_cycle", off, adj)
        assert got == exp and st.num_extensions == ext
        g2.free()
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        g.free()


IDENTITY_APPS = ["kgraphpi_house", "kgraphpi_tailed_triangle", "kautomine_four_motif"]


@pytest.mark.timeout(900, method="thread")
def test_identity_engine_matches_dfs_engine(khz_ctx):
    """House, tailed triangle and 4-motif on a skewed R-MAT whose hub start vertices reach every
    wedge tier: the identity engine (per-edge triangles, weighted wedge walk) and the DFS engine
    (the schedules as written) agree on counts and NumExtensions; on a small graph both equal the
    oracle."""
    from openkhuzdulgraph_b200 import khz
    g = khz_ctx.generate_rmat(14, 16, seed=4)
    canon, n = orc.rmat(11, 16, seed=6)
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    g2 = khz_ctx.graph_from_edges(sym, n)
    try:
        for app in IDENTITY_APPS:
            khz_ctx.set_config(engine=khz.ENGINE_AUTO)
            a, sa = khz_ctx.count(g, app)
            assert sa.engine == khz.ENGINE_BITMAP, app  # the identity engine reports as the bitmap engine
            small, ss = khz_ctx.count(g2, app)
            khz_ctx.set_config(engine=khz.ENGINE_DFS)
            d, sd = khz_ctx.count(g, app)
            assert a == d and sa.num_extensions == sd.num_extensions, app
            exp, ext, _ = orc.count(app, off, adj)
            assert small == exp and ss.num_extensions == ext, app
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        g.free()
        g2.free()


def test_house_identity_wide_window(khz_ctx):
    """Two adjacent hubs joined to 70 000 common leaves: degrees above 65 535 put the heaviest start
    vertex on the 32-bit window counters.  Every 4-cycle is hub-leaf-hub-leaf and every triangle's
    apex over a cycle edge is the other hub, inside the cycle, so there are no houses while the
    4-cycle and diamond terms are C(L, 2) each; NumExtensions follow from the degrees."""
    from math import comb
    ctx = khz_ctx
    L = 70000
    leaves = np.arange(2, L + 2, dtype=np.uint32)
    canon = np.concatenate([np.array([[0, 1]], np.uint32), np.stack([np.zeros(L, np.uint32), leaves], 1),
                            np.stack([np.ones(L, np.uint32), leaves], 1)])
    n = L + 2
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    g = ctx.graph_from_edges(sym, n)
    try:
        h, sh = ctx.count(g, "kgraphpi_house")
        c4, _ = ctx.count(g, "kgraphpi_four_cycle")
        assert c4 == [comb(L, 2)]
        d = np.diff(off).astype(np.int64)
        below = np.array([np.searchsorted(adj[off[v]:off[v + 1]], v) for v in range(n)], dtype=np.int64)
        depth2 = int(((d - 1) * below).sum())
        assert h == [0]
        assert sh.num_extensions == n + (2 * L + 1) + depth2 + 4 * comb(L, 2)
    finally:
        g.free()


def test_autotuner_keeps_counts_and_installs_settings(graphs, khz_ctx):
    from openkhuzdulgraph_b200 import khz
    jobs = [(g, app) for spec, n, sym, off, adj, g in graphs[:4]
            for app in ["kautomine_four_clique", "kgraphpi_four_cycle", "kautomine_four_motif"]]
    expect = [khz_ctx.count(g, app)[0] for g, app in jobs]
    rep = khz_ctx.autotune(jobs, reps=1)
    try:
        assert rep["trials"] >= 5 and rep["best_ms"] <= rep["baseline_ms"]
        cfg = khz_ctx.config()
        assert cfg.engine == rep["engine"] and cfg.dfs_chunk == rep["dfs_chunk"]
        assert [khz_ctx.count(g, app)[0] for g, app in jobs] == expect
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO, dfs_warps_per_sm=0, dfs_chunk=0, bitmap_warp_max=64,
                           bitmap_hub_rows=0)  # 0: the defaults
