"""Schedules registered by the app (khz_app_register) run on the device engine.

Pinned three ways: registered copies of built-in schedules give the built-in apps' counts and
NumExtensions; a schedule with a closed form (the non-induced 3-star, as toolkits/degree_analysis.cc
:40-51 computes it) gives sum C(d, 3); and hand-written schedules, including ones whose level sets
are re-read below their own bound, match a plain-Python interpreter of the schedule semantics."""
import numpy as np
import pytest

from conftest import golden_graph
import orc

pytestmark = pytest.mark.gpu


def _k():
    from openkhuzdulgraph_b200 import khz
    return khz


def builtin_copies():
    k = _k()
    N, S, AND, SUB, level, term, schedule = k.N, k.S, k.AND, k.SUB, k.level, k.term, k.schedule
    four_cycle = schedule(4, [level(term(N(0), gt=[0])), level(term(N(1), gt=[0], ne=[0, 1]))],
                          [term(AND(N(0), 2), gt=[1], ne=[0, 1, 2])])
    house = schedule(5, [level(term(N(0), gt=[0])), level(term(N(1), ne=[0, 1]), cached=AND(N(0), 1)),
                         level(term(AND(N(0), 2), ne=[0, 1, 2]))], [term(S(4), ne=[0, 1, 2, 3])])
    motif3 = schedule(3, [level(term(N(0)))], [term(AND(N(0), 1), gt=[1], counter=0, guard=(0, 1)),
                                               term(SUB(N(0), 1), ne=[1], counter=1)])
    kgpi5 = schedule(5, [level(term(N(0), gt=[0], ne=[0])), level(term(AND(N(0), 1), gt=[1], ne=[0, 1])),
                         level(term(AND(S(2), 2), gt=[0, 2], ne=[0, 1, 2]))],
                     [term(AND(S(3), 3), gt=[1, 3], ne=[0, 1, 2, 3])])
    return [("kgraphpi_four_cycle", [four_cycle], [1]), ("kgraphpi_house", [house], [1]),
            ("kautomine_three_motif", [motif3], [1, 2]), ("kgraphpi_five_clique", [kgpi5], [1])]


@pytest.mark.parametrize("engine", ["auto", "dfs"])
def test_registered_copies_match_builtin_apps(golden, khz_ctx, engine):
    khz = _k()
    ids = [(name, khz.register_app(runs, mult)) for name, runs, mult in builtin_copies()]
    khz_ctx.set_config(engine=khz.ENGINE_DFS if engine == "dfs" else khz.ENGINE_AUTO)
    try:
        for spec in golden["graphs"][:6]:
            _, n, sym, _, _ = golden_graph(spec)
            g = khz_ctx.graph_from_edges(sym, n)
            for name, app in ids:
                got, st = khz_ctx.count(g, app)
                exp, st2 = khz_ctx.count(g, name)
                assert got == exp and st.num_extensions == st2.num_extensions, (spec["name"], name)
            g.free()
    finally:
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)


def test_three_star_closed_form(golden, khz_ctx):
    khz = _k()
    N, level, term, schedule = khz.N, khz.level, khz.term, khz.schedule
    star = khz.register_app([schedule(4, [level(term(N(0))), level(term(N(0), gt=[1]))], [term(N(0), gt=[2])])],
                            [1])
    for spec in golden["graphs"]:
        _, n, sym, off, _ = golden_graph(spec)
        d = np.diff(off.astype(np.int64))
        g = khz_ctx.graph_from_edges(sym, n)
        got, st = khz_ctx.count(g, star)
        assert got == [int((d * (d - 1) * (d - 2) // 6).sum())], spec["name"]
        assert st.num_extensions == int(n + d.sum() + (d * (d - 1) // 2).sum()), spec["name"]
        g.free()


def interpret(sched, nbrs, n, runs_counts):
    """Plain-Python semantics of one schedule: each level's candidate set, its filters, cached sets,
    the counting terms; NumExtensions as the engine counts it (every start vertex, every candidate
    passing a non-finalized level's filters)."""
    k, levels, last = sched
    counts = [0] * 6
    ext = 0

    def ev(e, v, sets):
        base = set(nbrs[v[e[1]]]) if e[0] == 0 else set(sets[e[1]])
        for o, b in e[2]:
            base = base & set(nbrs[v[b]]) if o == 1 else base - set(nbrs[v[b]])
        return sorted(base)

    def ok(x, t, v):
        return all(x > v[a] for a in t[1]) and all(x != v[a] for a in t[2])

    def rec(L, v, sets):
        nonlocal ext
        if L == k - 1:
            for t in last:
                if t[4] and not v[t[4][0]] < v[t[4][1]]:
                    continue
                counts[t[3]] += sum(1 for x in ev(t[0], v, sets) if ok(x, t, v))
            return
        t, cached, fin = levels[L - 1]
        sets = dict(sets)
        if cached is not None:
            sets[4] = ev(cached, v, sets)
        cand = ev(t[0], v, sets)
        if t[0][2]:
            sets[L] = cand
        for x in cand:
            if ok(x, t, v):
                if not fin:
                    ext += 1
                rec(L + 1, v + [x], sets)

    for v0 in range(n):
        ext += 1
        rec(1, [v0], {})
    return counts[:runs_counts], ext


def hand_written():
    k = _k()
    N, S, AND, SUB, level, term, schedule = k.N, k.S, k.AND, k.SUB, k.level, k.term, k.schedule
    return [
        # level set 2 re-read below its own bound (x > v0 only): must be materialised whole
        schedule(4, [level(term(N(0), gt=[0])), level(term(AND(N(0), 1), gt=[1]))], [term(AND(S(2), 2), gt=[0])]),
        # a cached set built from a level set, a finalized level, a subtraction chain
        schedule(5, [level(term(N(0))), level(term(SUB(N(0), 1), gt=[1]), finalized=True),
                     level(term(AND(S(2), 2), ne=[0, 1]), cached=SUB(S(2), 2))],
                 [term(SUB(S(4), 3), gt=[2], ne=[0, 1, 3])]),
        # two guarded counting terms on a 4-vertex pattern
        schedule(4, [level(term(N(0), gt=[0])), level(term(N(1), ne=[0, 1]))],
                 [term(AND(N(0), 2), gt=[1], ne=[0, 1, 2], counter=0, guard=(1, 2)),
                  term(SUB(N(2), 0), ne=[0, 1], counter=1)]),
    ]


def test_hand_written_schedules_match_interpreter(khz_ctx):
    khz = _k()
    scheds = hand_written()
    ncounts = [1, 1, 2]
    ids = [khz.register_app([s], [1] * c) for s, c in zip(scheds, ncounts)]
    for seed in (1, 2):
        canon, n = orc.er(48, 260, seed=seed)
        sym = orc.symmetrize(canon)
        off, adj = orc.csr(sym, n)
        nbrs = [adj[off[v]:off[v + 1]].tolist() for v in range(n)]
        g = khz_ctx.graph_from_edges(sym, n)
        for s, c, app in zip(scheds, ncounts, ids):
            exp, ext = interpret(s, nbrs, n, c)
            for engine in (khz.ENGINE_AUTO, khz.ENGINE_DFS):
                khz_ctx.set_config(engine=engine)
                got, st = khz_ctx.count(g, app)
                assert got == exp and st.num_extensions == ext, (seed, app)
        khz_ctx.set_config(engine=khz.ENGINE_AUTO)
        g.free()


def test_registered_apps_in_batches_and_restricted_runs(khz_ctx):
    khz = _k()
    ids = [khz.register_app([s], [1] * c) for s, c in zip(hand_written(), [1, 1, 2])]
    canon, n = orc.rmat(9, 8, seed=2)
    sym = orc.symmetrize(canon)
    g = khz_ctx.graph_from_edges(sym, n)
    single = [khz_ctx.count(g, a) for a in ids]
    counts, exts, _ = khz_ctx.count_batch([(g, a) for a in ids])
    assert counts == [s[0] for s in single] and exts == [s[1].num_extensions for s in single]
    labels = (np.arange(n, dtype=np.uint64) % 3).astype(np.uint32)
    g.set_labels(labels)
    for a, (whole, st) in zip(ids, single):
        parts = [khz_ctx.count_restricted(g, a, lab) for lab in range(3)]
        assert [sum(p[0][i] for p in parts) for i in range(len(whole))] == whole
        assert sum(p[1].num_extensions for p in parts) == st.num_extensions
    g.free()
