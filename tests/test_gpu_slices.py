"""Counting restricted to the start vertices of one label (the reference's
run(disable_output, restrict_starting_vertex_label, label), distributed_application.h:54, with the
start vertices handed out by WorkloadDistributer::fetch_next_batch_local, engine.cc:1457-1496).

Pinned on the golden graphs to the reference's own sampled driver (tests/golden/golden.json,
`apps_sampled`: the reference app run with labels v % mod on the start vertices of label rem), and
for every app and engine to the oracle's label-restricted run.  Restricted counts are the raw
aggregator values; the reference apps divide them by their multiplicities after run()."""
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


def _mults(khz, app):
    aid = orc.APPS[app]
    return [khz.lib().khz_app_multiplicity(aid, p) for p in range(khz.num_counts(aid))]


@pytest.fixture(scope="module")
def labelled(golden, khz_ctx):
    """Golden graphs on the device with labels v % mod, as the sampled driver's files carry."""
    mod = golden["sample"]["mod"]
    out = []
    for spec in golden["graphs"]:
        _, n, sym, off, adj = golden_graph(spec)
        g = khz_ctx.graph_from_edges(sym, n)
        labels = (np.arange(n, dtype=np.uint64) % mod).astype(np.uint32)
        g.set_labels(labels)
        out.append((spec, g, off, adj, labels))
    yield out
    for _, g, _, _, _ in out:
        g.free()


@pytest.mark.parametrize("engine", ["auto", "dfs"])
def test_restricted_matches_reference_sampled_driver(golden, labelled, khz_ctx, engine):
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_DFS if engine == "dfs" else khz.ENGINE_AUTO)
    rem = golden["sample"]["rem"]
    try:
        for spec, g, _, _, _ in labelled:
            for app in orc.REF_APPS:
                ref = spec["apps_sampled"].get(app)
                if ref is None:
                    continue
                raw, st = khz_ctx.count_restricted(g, app, rem)
                got = [r // m for r, m in zip(raw, _mults(khz, app))]
                assert got == ref["counts"], (spec["name"], app, engine)
                assert st.num_extensions == ref["num_extensions"], (spec["name"], app, engine)
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)


@pytest.mark.parametrize("engine", ["auto", "dfs"])
def test_restricted_matches_oracle_every_app(golden, labelled, khz_ctx, engine):
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_DFS if engine == "dfs" else khz.ENGINE_AUTO)
    mod = golden["sample"]["mod"]
    try:
        for spec, g, off, adj, labels in labelled:
            for app in ALL_APPS:
                for lab in sorted({0, golden["sample"]["rem"], mod - 1}):
                    if lab >= g.info().num_labels:  # a graph of fewer vertices than the modulus
                        continue
                    exp, ext, _ = orc.count_labeled(app, off, adj, labels, lab, threads=4)
                    raw, st = khz_ctx.count_restricted(g, app, lab)
                    assert raw == exp, (spec["name"], app, lab, engine)
                    assert st.num_extensions == ext, (spec["name"], app, lab, engine)
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)


@pytest.mark.parametrize("engine", ["bitmap", "dfs"])
def test_restricted_cliques_on_oriented_input(golden, khz_ctx, engine):
    """On a graph stored oriented the bitmap engine serves restricted clique counts itself."""
    from openkhuzdulgraph_b200 import khz
    khz_ctx.set_config(engine=khz.ENGINE_BITMAP if engine == "bitmap" else khz.ENGINE_DFS)
    try:
        for spec in golden["graphs"]:
            _, n, sym, off, adj = golden_graph(spec)
            ooff, oadj, _ = orc.orient(off, adj)
            src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(ooff).astype(np.int64))
            g = khz_ctx.graph_from_edges(np.stack([src, oadj], axis=1), n)
            labels = (np.arange(n, dtype=np.uint64) * 2654435761 % 7).astype(np.uint32)
            if len(set(labels.tolist())) != 7:
                g.free()
                continue
            g.set_labels(labels)
            for app in CLIQUES:
                for lab in (0, 3, 6):
                    exp, ext, _ = orc.count_labeled(app, ooff, oadj, labels, lab, threads=4)
                    raw, st = khz_ctx.count_restricted(g, app, lab)
                    assert raw == exp and st.num_extensions == ext, (spec["name"], app, lab, engine)
            g.free()
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)


def test_label_slices_partition_the_whole_count(khz_ctx):
    """Summed over all labels, the restricted counts and NumExtensions are the unrestricted ones
    (every start vertex has exactly one label), on every engine the apps take."""
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.rmat(13, 8, seed=3)
    sym = orc.symmetrize(canon)
    g = khz_ctx.graph_from_edges(sym, n)
    og = g.orient()
    nl = 5
    # every app on the symmetric graph; the clique apps on the oriented one (the others count
    # patterns of an undirected graph, whose multiplicities a DAG does not honour)
    for gg, apps in ((g, ALL_APPS), (og, CLIQUES)):
        labels = (np.arange(n, dtype=np.uint64) * 40503 % nl).astype(np.uint32)
        gg.set_labels(labels)
        for app in apps:
            whole, st = khz_ctx.count(gg, app)
            mult = _mults(khz, app)
            tot, ext = [0] * len(whole), 0
            for lab in range(nl):
                raw, s2 = khz_ctx.count_restricted(gg, app, lab)
                tot = [a + b for a, b in zip(tot, raw)]
                ext += s2.num_extensions
            assert [t // m for t, m in zip(tot, mult)] == whole, app
            assert ext == st.num_extensions, app
    og.free()
    g.free()


def test_labels_are_validated_and_loaded(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.er(200, 900, seed=2)
    sym = orc.symmetrize(canon)
    g = khz_ctx.graph_from_edges(sym, n)
    with pytest.raises(khz.KhzError) as e:  # no labels yet
        khz_ctx.count_restricted(g, "kautomine_triangle", 0)
    assert e.value.status == 1
    gap = np.zeros(n, dtype=np.uint32)
    gap[:10] = 2  # label 1 unused: the reference's loader rejects such files
    with pytest.raises(khz.KhzError) as e:
        g.set_labels(gap)
    assert e.value.status == 6
    with pytest.raises(khz.KhzError) as e:
        g.set_labels(np.zeros(n - 1, dtype=np.uint32))
    assert e.value.status == 1
    labels = (np.arange(n, dtype=np.uint64) % 3).astype(np.uint32)
    g.set_labels(labels)
    assert g.info().num_labels == 3
    with pytest.raises(khz.KhzError) as e:  # label out of range
        khz_ctx.count_restricted(g, "kautomine_triangle", 3)
    assert e.value.status == 1
    off, adj = orc.csr(sym, n)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "lab.dgraph")
        orc.write_dgraph(path, n, sym, labels)
        g2 = khz_ctx.load_dgraph(path)
        assert g2.info().num_labels == 3
        raw, st = khz_ctx.count_restricted(g2, "kautomine_three_motif", 1)
        exp, ext, _ = orc.count_labeled("kautomine_three_motif", off, adj, labels, 1, threads=4)
        assert raw == exp and st.num_extensions == ext
        g3 = khz_ctx.load_dgraph(path, labels=False)
        assert g3.info().num_labels == 0
        g3.free()
        g2.free()
    g.free()
