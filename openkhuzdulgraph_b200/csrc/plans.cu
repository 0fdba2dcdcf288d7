// Schedule tables: each reference apply() restated as a declarative plan for the DFS
// engine (and flagged for the bitmap clique engine where it counts cliques).
//
// Level l produces v_l.  Notation in the comments: N(i) = N(v_i), P_l = the materialised
// candidate set of level l (the reference's prefix_{l-1} / cached object).
#include <stdio.h>

#include <deque>
#include <mutex>
#include <string>

#include "khz_internal.cuh"

namespace khz {

namespace {

constexpr uint8_t B(int a) { return (uint8_t)(1u << a); }

SetExpr N(int a) { return SetExpr{BASE_NBR, (int8_t)a, {OP_NONE, OP_NONE}, {0, 0}}; }
SetExpr S(int s) { return SetExpr{BASE_SLOT, (int8_t)s, {OP_NONE, OP_NONE}, {0, 0}}; }
SetExpr op(SetExpr e, int8_t o, int b) {
    const int k = e.op[0] == OP_NONE ? 0 : 1;
    e.op[k] = o;
    e.op_arg[k] = (int8_t)b;
    return e;
}
SetExpr AND(SetExpr e, int b) { return op(e, OP_AND, b); }
SetExpr SUB(SetExpr e, int b) { return op(e, OP_SUB, b); }

Term T(SetExpr s, uint8_t gt = 0, uint8_t ne = 0, int counter = 0, int glo = -1, int ghi = -1) {
    Term t{};
    t.set = s;
    t.gt_mask = gt;
    t.ne_mask = ne;
    t.guard_lo = (int8_t)glo;
    t.guard_hi = (int8_t)ghi;
    t.counter = (int8_t)counter;
    return t;
}
Level L(Term t, bool finalized = false) {
    Level l{};
    l.t = t;
    l.finalized = finalized ? 1 : 0;
    l.has_extra = 0;
    return l;
}
Level LX(Term t, SetExpr extra) {
    Level l = L(t);
    l.has_extra = 1;
    l.extra = extra;
    return l;
}

Plan plan3(Level l1, Term last0) {
    Plan p{};
    p.k = 3;
    p.bounded_sets = 1;
    p.num_terms = 1;
    p.lv[1] = l1;
    p.last[0] = last0;
    return p;
}
Plan plan4(Level l1, Level l2, Term last0) {
    Plan p{};
    p.k = 4;
    p.bounded_sets = 1;
    p.num_terms = 1;
    p.lv[1] = l1;
    p.lv[2] = l2;
    p.last[0] = last0;
    return p;
}
Plan plan5(Level l1, Level l2, Level l3, Term last0) {
    Plan p{};
    p.k = 5;
    p.bounded_sets = 1;
    p.num_terms = 1;
    p.lv[1] = l1;
    p.lv[2] = l2;
    p.lv[3] = l3;
    p.last[0] = last0;
    return p;
}

AppDef one(Plan p, int counts = 1) {
    AppDef a{};
    a.num_runs = 1;
    a.plans[0] = p;
    a.num_counts = counts;
    for (int i = 0; i < 6; ++i) a.mult[i] = 1;
    return a;
}

// kgraphpi triangle, kgraphpi/triangle.cc:53-122
Plan kgpi_triangle_plan() {
    return plan3(L(T(N(0), B(0), B(0))), T(AND(N(0), 1), B(1), B(0) | B(1), 0));
}

AppDef make(int app) {
    switch (app) {
        case KHZ_KAUTO_TRIANGLE: {  // kautomine/triangle.cc:58-121: v1 > v0; count N(0) n N(1) above v1
            AppDef a = one(plan3(L(T(N(0), B(0))), T(AND(N(0), 1), B(1))));
            a.clique = true;
            a.clique_k = 3;
            return a;
        }
        case KHZ_KAUTO_4CLIQUE: {  // kautomine/four_clique.cc:58-153
            AppDef a = one(plan4(L(T(N(0), B(0))), L(T(AND(N(0), 1), B(1))), T(AND(S(2), 2), B(2))));
            a.clique = true;
            a.clique_k = 4;
            return a;
        }
        case KHZ_KAUTO_5CLIQUE: {  // kautomine/five_clique.cc:58-186
            AppDef a = one(plan5(L(T(N(0), B(0))), L(T(AND(N(0), 1), B(1))), L(T(AND(S(2), 2), B(2))),
                                 T(AND(S(3), 3), B(3))));
            a.clique = true;
            a.clique_k = 5;
            return a;
        }
        case KHZ_KAUTO_3MOTIF: {  // kautomine/three_motif.cc:59-138, fused, multiplicities {1, 2}
            Plan p = plan3(L(T(N(0))), T(AND(N(0), 1), B(1), 0, 0, 0, 1));
            p.num_terms = 2;
            p.last[1] = T(SUB(N(0), 1), 0, B(1), 1);
            AppDef a = one(p, 2);
            a.mult[1] = 2;
            return a;
        }
        case KHZ_KGPI_TRIANGLE: {
            AppDef a = one(kgpi_triangle_plan());
            a.clique = true;
            a.clique_k = 3;
            return a;
        }
        case KHZ_KGPI_4CLIQUE: {  // kgraphpi/four_clique.cc:53-159
            AppDef a = one(plan4(L(T(N(0), B(0), B(0))), L(T(AND(N(0), 1), B(1), B(0) | B(1))),
                                 T(AND(S(2), 2), B(0) | B(2), B(0) | B(1) | B(2))));
            a.clique = true;
            a.clique_k = 4;
            return a;
        }
        case KHZ_KGPI_5CLIQUE: {  // kgraphpi/five_clique.cc:53-195
            AppDef a = one(plan5(L(T(N(0), B(0), B(0))), L(T(AND(N(0), 1), B(1), B(0) | B(1))),
                                 L(T(AND(S(2), 2), B(0) | B(2), B(0) | B(1) | B(2))),
                                 T(AND(S(3), 3), B(1) | B(3), B(0) | B(1) | B(2) | B(3))));
            a.clique = true;
            a.clique_k = 5;
            return a;
        }
        case KHZ_KGPI_3MOTIF: {  // kgraphpi/three_motif.cc:52-174: triangle, then the edge-induced wedge
            AppDef a{};
            a.num_runs = 2;
            a.plans[0] = kgpi_triangle_plan();
            a.plans[1] = plan3(L(T(N(0), 0, B(0)), true), T(N(0), B(1), B(0) | B(1), 1));
            a.num_counts = 2;
            for (int i = 0; i < 6; ++i) a.mult[i] = 1;
            return a;
        }
        case KHZ_KGPI_4CYCLE:  // v0-v1-v2-v3-v0 with v1 > v0, v2 > v0, v3 > v1
            return one(plan4(L(T(N(0), B(0))), L(T(N(1), B(0), B(0) | B(1))),
                             T(AND(N(0), 2), B(1), B(0) | B(1) | B(2))));
        case KHZ_KGPI_HOUSE:  // square v0-v1-v2-v3, roof v4 on v0 and v1; roof set N(0) n N(1) cached at size 2
            return one(plan5(L(T(N(0), B(0))), LX(T(N(1), 0, B(0) | B(1)), AND(N(0), 1)),
                             L(T(AND(N(0), 2), 0, B(0) | B(1) | B(2))), T(S(4), 0, B(0) | B(1) | B(2) | B(3))));
        case KHZ_KGPI_TAILED_TRIANGLE:  // triangle v0 v1 v2 (v2 > v1) plus tail on v0
            return one(plan4(L(T(N(0), 0, B(0))), L(T(AND(N(0), 1), B(1), B(0) | B(1))),
                             T(N(0), 0, B(0) | B(1) | B(2))));
        case KHZ_KAUTO_4MOTIF: {  // vertex-induced 4-motifs, one run per pattern
            AppDef a{};
            a.num_runs = 6;
            // 3-star: v1, v2 > v1 in N(0) \ N(1), v3 > v2 in P2 \ N(2)
            a.plans[0] = plan4(L(T(N(0))), L(T(SUB(N(0), 1), B(1))), T(SUB(S(2), 2), B(2), 0, 0));
            // 4-path v2-v0-v1-v3: v2 in N(0) \ N(1); v3 in (N(1) \ N(0)) \ N(2)
            a.plans[1] = plan4(L(T(N(0))), LX(T(SUB(N(0), 1), 0, B(1)), SUB(N(1), 0)), T(SUB(S(4), 2), 0, B(0), 1));
            // tailed triangle: v2 > v1 in N(0) n N(1); tail v3 in (N(0) \ N(1)) \ N(2)
            a.plans[2] = plan4(L(T(N(0))), LX(T(AND(N(0), 1), B(1)), SUB(N(0), 1)),
                               T(SUB(S(4), 2), 0, B(1) | B(2), 2));
            // 4-cycle v0-v1-v3-v2-v0: v2 in N(0) \ N(1); v3 in (N(1) n N(2)) \ N(0)
            a.plans[3] = plan4(L(T(N(0))), L(T(SUB(N(0), 1), 0, B(1))), T(SUB(AND(N(1), 2), 0), 0, B(0), 3));
            // diamond: v1 > v0; v2 in N(0) n N(1); v3 > v2 in P2 \ N(2)
            a.plans[4] = plan4(L(T(N(0), B(0))), L(T(AND(N(0), 1))), T(SUB(S(2), 2), B(2), 0, 4));
            // 4-clique
            a.plans[5] = plan4(L(T(N(0), B(0))), L(T(AND(N(0), 1), B(1))), T(AND(S(2), 2), B(2), 0, 5));
            a.num_counts = 6;
            for (int i = 0; i < 6; ++i) a.mult[i] = 1;
            a.mult[1] = 2;
            a.mult[3] = 8;
            return a;
        }
        default:
            return AppDef{};
    }
}

struct Table {
    AppDef apps[KHZ_NUM_APPS];
    Table() {
        for (int i = 0; i < KHZ_NUM_APPS; ++i) apps[i] = make(i);
    }
};

// Apps registered at run time (khz_app_register): ids KHZ_NUM_APPS, KHZ_NUM_APPS + 1, ...; a deque
// keeps references stable while it grows.
constexpr int kMaxRegistered = 4096;
std::mutex g_reg_mu;
std::deque<AppDef> g_registered;

// ---- validation of an app's schedule: everything the DFS engine indexes by must be in range ----
struct Checker {
    std::string err;
    bool fail(const char *fmt, int a = 0, int b = 0, int c = 0) {
        if (err.empty()) {
            char buf[256];
            snprintf(buf, sizeof(buf), fmt, a, b, c);
            err = buf;
        }
        return false;
    }
    // an expression evaluated when `nv` vertices are matched (v_0 .. v_{nv-1}); `slots` = the
    // materialised sets readable then (bit s: set s)
    bool expr(const khz_set_expr &e, int nv, unsigned slots, int run, int level, const char *what) {
        if (e.base_kind == KHZ_BASE_NBR) {
            if (e.base_arg < 0 || e.base_arg >= nv)
                return fail("run %d level %d: base N(v_i) names a vertex not yet matched", run, level);
        } else if (e.base_kind == KHZ_BASE_SET) {
            if (e.base_arg < 2 || e.base_arg > 4 || !(slots & (1u << e.base_arg)))
                return fail("run %d level %d: base set %d is not materialised before this use", run, level,
                            e.base_arg);
        } else {
            return fail("run %d level %d: base kind %d unknown", run, level, e.base_kind);
        }
        for (int o = 0; o < 2; ++o) {
            if (e.op[o] == KHZ_OP_NONE) {
                if (o == 0 && e.op[1] != KHZ_OP_NONE)
                    return fail("run %d level %d: second operation without a first", run, level);
                continue;
            }
            if (e.op[o] != KHZ_OP_AND && e.op[o] != KHZ_OP_SUB)
                return fail("run %d level %d: operation code %d unknown", run, level, e.op[o]);
            if (e.op_arg[o] < 0 || e.op_arg[o] >= nv)
                return fail("run %d level %d: operand N(v_b) names a vertex not yet matched", run, level);
        }
        (void)what;
        return true;
    }
    bool term(const khz_term &t, int nv, unsigned slots, int run, int level, int num_counts, bool last) {
        if (!expr(t.set, nv, slots, run, level, "term")) return false;
        const unsigned avail = (1u << nv) - 1u;
        if ((t.gt_mask & ~avail) || (t.ne_mask & ~avail))
            return fail("run %d level %d: a filter names a vertex not yet matched", run, level);
        if (__builtin_popcount(t.ne_mask) > 4) return fail("run %d level %d: more than 4 exclusions", run, level);
        if (last) {
            if (t.counter < 0 || t.counter >= num_counts)
                return fail("run %d: counting term adds to counter %d of %d", run, t.counter, num_counts);
            const bool g = t.guard_lo >= 0 || t.guard_hi >= 0;
            if (g && (t.guard_lo < 0 || t.guard_hi < 0 || t.guard_lo >= nv || t.guard_hi >= nv))
                return fail("run %d: guard names a vertex not yet matched", run);
        }
        return true;
    }
};

Term to_term(const khz_term &t) {
    Term r{};
    r.set = SetExpr{t.set.base_kind, t.set.base_arg, {t.set.op[0], t.set.op[1]}, {t.set.op_arg[0], t.set.op_arg[1]}};
    r.gt_mask = t.gt_mask;
    r.ne_mask = t.ne_mask;
    r.guard_lo = t.guard_lo >= 0 && t.guard_hi >= 0 ? t.guard_lo : -1;
    r.guard_hi = t.guard_lo >= 0 && t.guard_hi >= 0 ? t.guard_hi : -1;
    r.counter = t.counter;
    return r;
}

// A later use of level set s (materialised with the level's lower bound `gt_s` applied) sees all it
// needs when it keeps only members above v_s, or above every vertex gt_s does.
bool use_ok(uint8_t gt_use, int s, uint8_t gt_s) { return (gt_use & (1u << s)) || ((gt_use & gt_s) == gt_s); }

}  // namespace

const AppDef &app_def(int app) {
    static Table t;
    if (app >= 0 && app < KHZ_NUM_APPS) return t.apps[app];
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return g_registered[(size_t)(app - KHZ_NUM_APPS)];
}

bool app_known(int app) {
    if (app >= 0 && app < KHZ_NUM_APPS) return true;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return app >= KHZ_NUM_APPS && (size_t)(app - KHZ_NUM_APPS) < g_registered.size();
}

}  // namespace khz

using namespace khz;

extern "C" khz_status khz_app_register(const khz_app_desc *desc, int32_t *app_id) {
    if (!desc || !app_id) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    Checker ck;
    const khz_app_desc &d = *desc;
    if (d.num_runs < 1 || d.num_runs > 6) ck.fail("num_runs %d out of 1..6", d.num_runs);
    if (d.num_counts < 1 || d.num_counts > KHZ_MAX_COUNTS) ck.fail("num_counts %d out of 1..6", d.num_counts);
    for (int c = 0; c < d.num_counts && c < KHZ_MAX_COUNTS && ck.err.empty(); ++c)
        if (d.multiplicity[c] == 0) ck.fail("multiplicity of count %d is 0", c);
    AppDef a{};
    a.num_runs = d.num_runs;
    a.num_counts = d.num_counts;
    for (int c = 0; c < KHZ_MAX_COUNTS; ++c) a.mult[c] = c < d.num_counts ? d.multiplicity[c] : 1;
    for (int r = 0; r < d.num_runs && ck.err.empty(); ++r) {
        const khz_pattern_schedule &s = d.runs[r];
        Plan p{};
        if (s.k < 3 || s.k > kMaxK) {
            ck.fail("run %d: pattern size %d out of 3..5", r, s.k);
            break;
        }
        if (s.num_terms < 1 || s.num_terms > 2) {
            ck.fail("run %d: %d counting terms (1 or 2)", r, s.num_terms);
            break;
        }
        p.k = s.k;
        p.num_terms = s.num_terms;
        const khz_term &t1 = s.levels[1].term;
        if (t1.set.base_kind != KHZ_BASE_NBR || t1.set.base_arg != 0 || t1.set.op[0] != KHZ_OP_NONE ||
            s.levels[1].has_cached) {
            ck.fail("run %d: level 1 must enumerate N(v_0) itself, with no cached set", r);
            break;
        }
        unsigned slots = 0;  // materialised sets readable at the current level
        uint8_t gt_of[5] = {0, 0, 0, 0, 0};
        bool bounded = true;
        auto note_uses = [&](const khz_set_expr &e, uint8_t gt_use, bool unfiltered) {
            if (e.base_kind == KHZ_BASE_SET && (e.base_arg == 2 || e.base_arg == 3) &&
                (unfiltered || !use_ok(gt_use, e.base_arg, gt_of[e.base_arg])))
                bounded = false;
        };
        for (int l = 1; l <= s.k - 2 && ck.err.empty(); ++l) {
            const khz_level &lv = s.levels[l];
            Level out{};
            if (lv.has_cached) {
                if (lv.cached.base_kind == KHZ_BASE_SET && lv.cached.base_arg == 4) {
                    ck.fail("run %d level %d: the cached set cannot be computed from itself", r, l);
                    break;
                }
                if (!ck.expr(lv.cached, l, slots, r, l, "cached")) break;
                note_uses(lv.cached, 0, true);
                out.has_extra = 1;
                out.extra = to_term(khz_term{lv.cached, 0, 0, -1, -1, 0, {0, 0, 0}}).set;
                slots |= 1u << 4;
            }
            if (!ck.term(lv.term, l, slots, r, l, d.num_counts, false)) break;
            note_uses(lv.term.set, lv.term.gt_mask, false);
            out.t = to_term(lv.term);
            out.t.counter = 0;
            out.finalized = lv.finalized ? 1 : 0;
            p.lv[l] = out;
            if (lv.term.set.op[0] != KHZ_OP_NONE) {
                if (l < 2) {
                    ck.fail("run %d level %d: level 1 cannot materialise a set", r, l);
                    break;
                }
                slots |= 1u << l;
                gt_of[l] = lv.term.gt_mask;
            }
        }
        for (int ti = 0; ti < s.num_terms && ck.err.empty(); ++ti) {
            const khz_term &t = s.last[ti];
            if (!ck.term(t, s.k - 1, slots, r, s.k - 1, d.num_counts, true)) break;
            note_uses(t.set, t.gt_mask, false);
            p.last[ti] = to_term(t);
        }
        p.bounded_sets = bounded ? 1 : 0;
        a.plans[r] = p;
    }
    if (!ck.err.empty()) {
        set_error("invalid schedule: %s", ck.err.c_str());
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_reg_mu);
    if ((int)g_registered.size() >= kMaxRegistered) {
        set_error("at most %d registered apps per process", kMaxRegistered);
        return KHZ_ERR_ARG;
    }
    g_registered.push_back(a);
    *app_id = KHZ_NUM_APPS + (int32_t)g_registered.size() - 1;
    return KHZ_OK;
}
