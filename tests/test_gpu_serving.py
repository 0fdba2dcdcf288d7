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


# ---- failures made on the host (no device fault is ever provoked) -------------------------------
@pytest.fixture(scope="module")
def heavy(khz_ctx):
    """A graph whose house count on the DFS engine takes milliseconds, so queued queries wait (the
    context runs the schedule on the DFS engine while the fixture is alive)."""
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.rmat(13, 16, seed=9)
    g = khz_ctx.graph_from_edges(orc.symmetrize(canon), n)
    khz_ctx.set_config(engine=khz.ENGINE_DFS)
    try:
        alone = khz_ctx.count(g, "kgraphpi_house")
        yield g, alone
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        g.free()


def test_allocation_failure_reaches_tickets_without_stalling(khz_ctx, resident):
    """With the context's device memory capped below what it already holds, every launch's scratch
    allocation fails on the host side of the scheduler: each ticket reports KHZ_ERR_OOM promptly and
    the server keeps serving once the cap is lifted."""
    from openkhuzdulgraph_b200 import khz
    graphs, alone = resident
    sv = khz.Server(khz_ctx, slots=2, max_batch=4)
    try:
        khz_ctx.set_config(device_mem_limit_mib=1)
        tickets = [(sv.submit(graphs[i % len(graphs)], app), i % len(graphs), app)
                   for i, app in enumerate(APPS * 3)]
        for t, _, app in tickets:
            with pytest.raises(khz.KhzError) as e:
                sv.wait(t, app, timeout_ms=20000.0)
            assert e.value.status == 2 and "memory limit" in str(e.value)
        khz_ctx.set_config(device_mem_limit_mib=0)
        for i, app in [(0, "kautomine_four_clique"), (3, "kgraphpi_house")]:
            counts, ext, _ = sv.wait(sv.submit(graphs[i], app), app, timeout_ms=20000.0)
            exp, st = alone[(i, app)]
            assert counts == exp and ext == st.num_extensions
    finally:
        khz_ctx.set_config(device_mem_limit_mib=0)
        sv.close()


def test_memory_limit_rejects_graphs_and_counts(khz_ctx):
    from openkhuzdulgraph_b200 import khz
    canon, n = orc.rmat(10, 8, seed=4)
    sym = orc.symmetrize(canon)
    g = khz_ctx.graph_from_edges(sym, n)
    try:
        khz_ctx.set_config(device_mem_limit_mib=1)
        with pytest.raises(khz.KhzError) as e:
            khz_ctx.graph_from_edges(sym, n)
        assert e.value.status == 2
        with pytest.raises(khz.KhzError) as e:
            khz_ctx.count(g, "kautomine_four_clique")
        assert e.value.status == 2
        khz_ctx.set_config(device_mem_limit_mib=0)
        off, adj = orc.csr(sym, n)
        assert khz_ctx.count(g, "kautomine_four_clique")[0] == orc.count("kautomine_four_clique", off, adj)[0]
    finally:
        khz_ctx.set_config(device_mem_limit_mib=0)
        g.free()


def test_timed_out_wait_then_success(khz_ctx, heavy):
    """A wait that runs out returns KHZ_ERR_TIMEOUT (KHZ_ERR_BUSY when only polling) and leaves the
    ticket valid: a later wait returns the result."""
    from openkhuzdulgraph_b200 import khz
    g, (exp, st) = heavy
    sv = khz.Server(khz_ctx, slots=1, max_batch=1)
    try:
        tickets = [sv.submit(g, "kgraphpi_house") for _ in range(24)]
        last = tickets[-1]
        with pytest.raises(khz.KhzError) as e:
            sv.wait(last, "kgraphpi_house", timeout_ms=0.0)
        assert e.value.status == 7
        with pytest.raises(khz.KhzError) as e:
            sv.wait(last, "kgraphpi_house", timeout_ms=0.5)
        assert e.value.status == 4
        for t in tickets:
            counts, ext, _ = sv.wait(t, "kgraphpi_house", timeout_ms=120000.0)
            assert counts == exp and ext == st.num_extensions
    finally:
        sv.close()


def test_cancel_withdraws_pending_queries(khz_ctx, heavy):
    from openkhuzdulgraph_b200 import khz
    g, (exp, st) = heavy
    sv = khz.Server(khz_ctx, slots=1, max_batch=1)
    try:
        tickets = [sv.submit(g, "kgraphpi_house") for _ in range(40)]
        cancelled = {t for t in tickets[20:] if sv.cancel(t)}
        assert cancelled  # the queue of 40 cannot have drained this fast
        for t in tickets:
            if t in cancelled:
                with pytest.raises(khz.KhzError) as e:
                    sv.wait(t, "kgraphpi_house", timeout_ms=1000.0)
                assert e.value.status == 10
            else:
                counts, ext, _ = sv.wait(t, "kgraphpi_house", timeout_ms=120000.0)
                assert counts == exp and ext == st.num_extensions
        with pytest.raises(khz.KhzError) as e:  # consumed
            sv.cancel(tickets[0])
        assert e.value.status == 8
        # one slot, one query per launch, admission in arrival order: once t2 is done, t is done too
        t = sv.submit(g, "kgraphpi_house")
        t2 = sv.submit(g, "kgraphpi_house")
        sv.wait(t2, "kgraphpi_house", timeout_ms=120000.0)
        assert sv.cancel(t) is False  # finished, not yet consumed: too late to cancel
        counts, _, _ = sv.wait(t, "kgraphpi_house", timeout_ms=120000.0)
        assert counts == exp
    finally:
        sv.close()
