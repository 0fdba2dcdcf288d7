"""The 3-FSM domain rules of fsm.cu, restated in Python, against brute-force enumeration (CPU only).

The reference's three_fsm app (kautomine/three_fsm.cc:53-262) inserts every embedding of each
template into its pattern domain; a (candidate, position) domain is the set of vertices some
embedding with that label tuple puts at that position.  The device does not enumerate wedges,
four-chains or three-stars: fsm_exist_kernel decides each (candidate, position, vertex) from
label counts lc(v, l) and a search for one witness (open_positions screens, then the per-template
searches, chain_pair and star_fits), and the triangle level lists each triangle once in
(degree, id) order and marks all six vertex orders (fsm_pair).  This test restates those rules
step for step and checks that they give exactly the enumerated domains on random small labelled
graphs, for every label tuple (not only the canonical ones the host generates), repeated labels
and one-label graphs included.  The device itself is checked against the reference's own app in
test_gpu_fsm.py."""
import itertools
import random

import pytest

# embedding constraints of the app's apply() levels (three_fsm.cc:53-262), symmetric simple graph


def enumerate_domains(adj, lab, k_template):
    dom = {}

    def put(tup, vs):
        d = dom.setdefault(tup, [set() for _ in vs])
        for p, v in enumerate(vs):
            d[p].add(v)

    n = len(adj)
    for v0 in range(n):
        for v1 in adj[v0]:
            if k_template == "edge":
                put((lab[v0], lab[v1]), (v0, v1))
                continue
            if k_template == "star":
                for v2 in adj[v1]:
                    if v2 == v0:
                        continue
                    for v3 in adj[v1]:
                        if v3 in (v0, v2):
                            continue
                        put((lab[v0], lab[v1], lab[v2], lab[v3]), (v0, v1, v2, v3))
                continue
            for v2 in adj[v0]:
                if v2 == v1:
                    continue
                if k_template == "wedge":
                    put((lab[v0], lab[v1], lab[v2]), (v0, v1, v2))
                elif k_template == "triangle":
                    if v2 in adj[v1]:
                        put((lab[v0], lab[v1], lab[v2]), (v0, v1, v2))
                else:  # chain
                    for v3 in adj[v1]:
                        if v3 in (v0, v2):
                            continue
                        put((lab[v0], lab[v1], lab[v2], lab[v3]), (v0, v1, v2, v3))
    return dom


class Counts:
    def __init__(self, adj, lab):
        self.adj, self.lab = adj, lab
        self.lc = [{} for _ in adj]
        for v, nb in enumerate(adj):
            for u in nb:
                self.lc[v][lab[u]] = self.lc[v].get(lab[u], 0) + 1

    def __call__(self, v, l):
        return self.lc[v].get(l, 0)


# ---- the device's rules ------------------------------------------------------------------------


def chain_pair(adj, lab, lc, v0, v1, c):
    c0, c1, c2, c3 = c
    A = lc(v0, c2) - (c1 == c2)
    B = lc(v1, c3) - (c0 == c3)
    if A == 0 or B == 0:
        return False
    if A >= 2 or B >= 2 or c2 != c3:
        return True
    a_end = next(u for u in sorted(adj[v0]) if u != v1 and lab[u] == c2)
    b_end = next(w for w in sorted(adj[v1]) if w != v0 and lab[w] == c3)
    return a_end != b_end


def star_fits(lc, y, need, lex):
    for l in need:
        if lc(y, l) - (l == lex) < need.count(l):
            return False
    return True


def device_domains(adj, lab, template, c):
    lc = Counts(adj, lab)
    k = len(c)
    dom = [set() for _ in range(k)]
    for x in range(len(adj)):
        lx = lab[x]
        # open_positions: the screen on x's own counts (centres decided outright)
        open_p = []
        if template == "wedge":
            c0, c1, c2 = c
            same = 1 if c1 == c2 else 0
            if c0 == lx and lc(x, c1) >= 1 and lc(x, c2) >= 1 + same:
                dom[0].add(x)
            if (c1 == lx or c2 == lx) and lc(x, c0) >= 1:
                open_p += [p for p in (1, 2) if c[p] == lx]
        elif template == "chain":
            c0, c1, c2, c3 = c
            if c0 == lx and lc(x, c1) >= 1 and lc(x, c2) >= 1 + (c1 == c2):
                open_p.append(0)
            if c1 == lx and lc(x, c0) >= 1 and lc(x, c3) >= 1 + (c0 == c3):
                open_p.append(1)
            if c2 == lx and lc(x, c0) >= 1:
                open_p.append(2)
            if c3 == lx and lc(x, c1) >= 1:
                open_p.append(3)
        else:  # star
            c0, c1, c2, c3 = c
            if c1 == lx and star_fits(lc, x, [c0, c2, c3], -1):
                dom[1].add(x)
            if (c0 == lx or c2 == lx or c3 == lx) and lc(x, c1) >= 1:
                open_p += [p for p in (0, 2, 3) if c[p] == lx]
        # the witness searches
        for p in open_p:
            found = False
            if template == "wedge":
                lend = c[2] if p == 1 else c[1]
                end_min = 1 + (c[1] == c[2])
                found = any(lab[y] == c[0] and lc(y, lend) >= end_min for y in adj[x])
            elif template == "star":
                need = [c[2] if p == 0 else c[0], c[2] if p == 3 else c[3]]
                found = any(lab[y] == c[1] and star_fits(lc, y, need, lx) for y in adj[x])
            elif p <= 1:
                want = c[1] if p == 0 else c[0]
                found = any(lab[y] == want and (chain_pair(adj, lab, lc, x, y, c) if p == 0 else
                                                chain_pair(adj, lab, lc, y, x, c)) for y in adj[x])
            else:
                c0, c1, c2, c3 = c
                lmid, lfar, lend = (c0, c1, c3) if p == 2 else (c1, c0, c2)
                far_min = 1 + (lx == lfar)
                for m in adj[x]:
                    if found:
                        break
                    if lab[m] != lmid or lc(m, lfar) < far_min:
                        continue
                    for f in adj[m]:
                        if f == x or lab[f] != lfar:
                            continue
                        kk = lc(f, lend) - (lmid == lend)
                        if kk >= 2 or (kk == 1 and (lx != lend or x not in adj[f])):
                            found = True
                            break
            if found:
                dom[p].add(x)
    return dom


def triangle_domains_listed_once(adj, lab, canon):
    """fsm_pair: each triangle from its lowest (degree, id) vertex, all six orders marked."""
    dom = {c: [set(), set(), set()] for c in canon}
    rk = [(len(adj[v]), v) for v in range(len(adj))]
    for v0 in range(len(adj)):
        for v1 in adj[v0]:
            if not rk[v0] < rk[v1]:
                continue
            for v2 in adj[v0]:
                if not rk[v1] < rk[v2] or v2 not in adj[v1]:
                    continue
                for o in itertools.permutations((v0, v1, v2)):
                    t = tuple(lab[v] for v in o)
                    if t in dom:
                        for p, v in enumerate(o):
                            dom[t][p].add(v)
    return dom


def random_graph(seed):
    rnd = random.Random(seed)
    n = rnd.randrange(4, 17)
    p = rnd.choice([0.15, 0.3, 0.5, 0.8])
    adj = [set() for _ in range(n)]
    for u in range(n):
        for v in range(u + 1, n):
            if rnd.random() < p:
                adj[u].add(v)
                adj[v].add(u)
    L = rnd.choice([1, 2, 3])
    lab = [rnd.randrange(L) for _ in range(n)]
    return adj, lab, L


@pytest.mark.parametrize("template,k", [("wedge", 3), ("chain", 4), ("star", 4)])
def test_witness_rules_equal_enumeration(template, k):
    for seed in range(60):
        adj, lab, L = random_graph(seed * 7 + k)
        enum = enumerate_domains(adj, lab, template)
        for c in itertools.product(range(L), repeat=k):
            want = enum.get(c, [set() for _ in range(k)])
            got = device_domains(adj, lab, template, c)
            assert got == want, (template, seed, c)


def test_triangles_listed_once_equal_enumeration():
    for seed in range(80):
        adj, lab, L = random_graph(seed * 11 + 5)
        canon = [c for c in itertools.product(range(L), repeat=3) if c[0] <= c[1] <= c[2]]
        enum = enumerate_domains(adj, lab, "triangle")
        got = triangle_domains_listed_once(adj, lab, canon)
        for c in canon:
            assert got[c] == enum.get(c, [set(), set(), set()]), (seed, c)
