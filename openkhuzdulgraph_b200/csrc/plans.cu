// Schedule tables: each reference apply() restated as a declarative plan for the DFS
// engine (and flagged for the bitmap clique engine where it counts cliques).
//
// Level l produces v_l.  Notation in the comments: N(i) = N(v_i), P_l = the materialised
// candidate set of level l (the reference's prefix_{l-1} / cached object).
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
    p.num_terms = 1;
    p.lv[1] = l1;
    p.last[0] = last0;
    return p;
}
Plan plan4(Level l1, Level l2, Term last0) {
    Plan p{};
    p.k = 4;
    p.num_terms = 1;
    p.lv[1] = l1;
    p.lv[2] = l2;
    p.last[0] = last0;
    return p;
}
Plan plan5(Level l1, Level l2, Level l3, Term last0) {
    Plan p{};
    p.k = 5;
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

}  // namespace

const AppDef &app_def(int app) {
    static Table t;
    return t.apps[app];
}

}  // namespace khz
