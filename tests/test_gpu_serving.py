"""Serving: queries submitted while others run are admitted as slots and HBM budget free up;
every result equals the same query counted alone."""
import random

import numpy as np
import pytest

from conftest import golden_graph
import orc

pytestmark = pytest.mark.gpu

APPS = ["kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique", "kgraphpi_four_cycle",
        "kgraphpi_house", "kautomine_four_motif", "kautomine_three_motif", "kgraphpi_tailed_triangle"]


@pytest.fixture(scope="module")
def resident(golden, khz_ctx):
    graphs = []
    for spec in golden["graphs"][:5]:
        canon, n, sym, off, adj = golden_graph(spec)
        graphs.append(khz_ctx.graph_from_edges(sym, n))
    alone = {(i, app): khz_ctx.count(g, app) for i, g in enumerate(graphs) for app in APPS}
    yield graphs, alone
    for g in graphs:
        g.free()


@pytest.mark.parametrize("slots,max_batch,budget", [(4, 16, 0), (2, 1, 0), (3, 8, 1)])
def test_mixed_stream_matches_alone(khz_ctx, resident, slots, max_batch, budget):
    """A shuffled mix of 240 queries; budget 1 byte forces one query in flight at a time."""
    from openkhuzdulgraph_b200 import khz
    graphs, alone = resident
    rng = random.Random(slots * 7 + max_batch)
    queries = [(rng.randrange(len(graphs)), rng.choice(APPS)) for _ in range(240)]
    sv = khz.Server(khz_ctx, slots=slots, max_batch=max_batch, hbm_budget=budget)
    try:
        tickets = [(sv.submit(graphs[i], app), i, app) for i, app in queries]
        for t, i, app in tickets:
            counts, ext, lat = sv.wait(t, app)
            exp, st = alone[(i, app)]
            assert counts == exp and ext == st.num_extensions, (i, app)
            assert lat > 0
        s = sv.stats()
        assert s["completed"] == len(queries) and s["p99_ms"] >= s["p50_ms"] > 0
        if budget == 1:
            assert s["batches"] == len(queries)
    finally:
        sv.close()


def test_ticket_errors(khz_ctx, resident):
    from openkhuzdulgraph_b200 import khz
    graphs, _ = resident
    sv = khz.Server(khz_ctx, slots=1)
    try:
        with pytest.raises(khz.KhzError) as e:
            sv.wait(12345, "kautomine_triangle")
        assert e.value.status == 8
        t = sv.submit(graphs[0], "kautomine_triangle")
        sv.wait(t, "kautomine_triangle")
        with pytest.raises(khz.KhzError):  # consumed
            sv.wait(t, "kautomine_triangle")
        with pytest.raises(khz.KhzError) as e:
            sv.submit(graphs[0], 99)
        assert e.value.status == 1
    finally:
        sv.close()
