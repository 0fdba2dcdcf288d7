"""The configurations at full size, through the C ABI.

* ER n = 100 000, m = 1 000 000 (the CPU-runnable configuration): every app equals the oracle
  (counts and NumExtensions), which the golden tests pin to the reference's own binaries.
* R-MAT scale 20, edge factor 24 (motif configuration) and scale 22, edge factor 16 (clique
  configuration): too large for the CPU oracle in a test, so the fast engines are checked against
  the DFS engine (the schedules as written) and against closed forms that hold at any size.  The
  schedules whose work grows with the square of hub degrees (4-motif, 4-cycle as written, the DFS
  4-clique) are cross-checked on smaller graphs of the same generator.
"""
import numpy as np
import pytest

import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def er_graph(khz_ctx):
    canon, n = orc.er(100000, 1000000, seed=1)
    sym = orc.symmetrize(canon)
    off, adj = orc.csr(sym, n)
    g = khz_ctx.graph_from_edges(sym, n)
    yield g, off, adj
    g.free()


@pytest.mark.parametrize("app", list(orc.APPS))
def test_er_full_size_matches_oracle(er_graph, khz_ctx, app):
    g, off, adj = er_graph
    got, st = khz_ctx.count(g, app)
    exp, ext, _ = orc.count(app, off, adj)
    assert got == exp and st.num_extensions == ext


def _engine(khz_ctx, g, app, engine):
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=engine)
    try:
        return khz_ctx.count(g, app)
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)


@pytest.mark.timeout(600, method="thread")
def test_motif_config_scale20(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    g = khz_ctx.generate_rmat(20, 24, seed=1)
    try:
        off, _ = g.export_csr()
        d = np.diff(off).astype(np.int64)
        s2 = int((d * (d - 1) // 2).sum())
        tri, st_t = _engine(khz_ctx, g, "kautomine_triangle", khz.ENGINE_AUTO)
        tri_dfs, st_td = _engine(khz_ctx, g, "kautomine_triangle", khz.ENGINE_DFS)
        assert tri == tri_dfs and st_t.num_extensions == st_td.num_extensions
        T = tri[0]
        m3a, s3a = _engine(khz_ctx, g, "kautomine_three_motif", khz.ENGINE_AUTO)
        m3d, s3d = _engine(khz_ctx, g, "kautomine_three_motif", khz.ENGINE_DFS)
        assert m3a == m3d == [T, s2 - 3 * T] and s3a.num_extensions == s3d.num_extensions
        k3a, _ = _engine(khz_ctx, g, "kgraphpi_three_motif", khz.ENGINE_AUTO)
        assert k3a == [T, s2]
    finally:
        g.free()


@pytest.mark.timeout(600, method="thread")
def test_four_vertex_patterns_scale14(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    g = khz_ctx.generate_rmat(14, 24, seed=1)
    try:
        off, _ = g.export_csr()
        d = np.diff(off).astype(np.int64)
        a, sa = _engine(khz_ctx, g, "kgraphpi_four_cycle", khz.ENGINE_AUTO)
        dd, sd = _engine(khz_ctx, g, "kgraphpi_four_cycle", khz.ENGINE_DFS)
        assert a == dd and sa.num_extensions == sd.num_extensions
        m4, _ = khz_ctx.count(g, "kautomine_four_motif")
        # non-induced 3-stars = induced 3-stars + paws + 2 diamonds + 4 four-cliques
        assert int((d * (d - 1) * (d - 2) // 6).sum()) == m4[0] + m4[2] + 2 * m4[4] + 4 * m4[5]
        # non-induced 4-cycles = induced 4-cycles + diamonds + 3 four-cliques
        assert a[0] == m4[3] + m4[4] + 3 * m4[5]
        k4, _ = khz_ctx.count(g, "kautomine_four_clique")
        assert m4[5] == k4[0]
    finally:
        g.free()


@pytest.mark.timeout(600, method="thread")
def test_clique_engines_agree_scale18(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    sym = khz_ctx.generate_rmat(18, 16, seed=1)
    og = sym.orient()
    try:
        for app in ["kautomine_four_clique", "kgraphpi_five_clique"]:
            b, sb = _engine(khz_ctx, og, app, khz.ENGINE_BITMAP)
            dd, sd = _engine(khz_ctx, og, app, khz.ENGINE_DFS)
            assert b == dd and sb.num_extensions == sd.num_extensions, app
    finally:
        og.free()
        sym.free()


@pytest.mark.timeout(600, method="thread")
def test_clique_config_scale22(khz_ctx):
    """4-clique on the bench graph: the count the bench reports, symmetric input == oriented input."""
    from openkhuzdulgraph_b200 import khz
    sym = khz_ctx.generate_rmat(22, 16, seed=1)
    og = sym.orient()
    try:
        b, sb = _engine(khz_ctx, og, "kautomine_four_clique", khz.ENGINE_BITMAP)
        assert b == [123601255038]
        s, ss = _engine(khz_ctx, sym, "kgraphpi_four_clique", khz.ENGINE_AUTO)
        assert s == b and ss.num_extensions == sb.num_extensions
    finally:
        og.free()
        sym.free()
