// khz_khuzdul.hpp — the reference's application API on top of the C ABI (header-only C++).
//
// Mirrors Khuzdul::DistributedApplication / Aggregator (distributed_application.h:12-60,
// engine.h:615-673) so that an app's main() keeps its shape: construct the application on a
// .dgraph, allocate aggregators, run(), evaluate().  The one difference: the app names its
// schedule (a khz_app_id) where the reference passes its apply() function, because apply() is
// host code and the schedules are held by the library as device plans.
#pragma once

#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <initializer_list>
#include <vector>

#include "khz.h"

namespace Khuzdul {

using VertexId = uint32_t;  // types.h:7-9
using EdgeId = uint64_t;
using LabelId = uint32_t;

class Error : public std::runtime_error {
  public:
    Error(khz_status s, const std::string &m) : std::runtime_error(m), status(s) {}
    khz_status status;
};

inline void check(khz_status s) {
    if (s != KHZ_OK) throw Error(s, khz_last_error_string());
}

// Aggregator<T> (engine.h:615-673): the device aggregates; evaluate() returns the value of the
// last run() for the pattern this aggregator was allocated for (in allocation order).
template <typename T>
class Aggregator {
  public:
    void clear() { value_ = 0; }
    T evaluate() const { return value_; }
    void set(T v) { value_ = v; }

  private:
    T value_ = 0;
};

// Builder for a schedule an app brings itself (khz_app_register): the apply() levels written as
// data.  Sets: N(i) = N(v_i), Set(2|3) = the set materialised by level 2 / 3, Cached() = the level's
// cached set; .And(b) / .Sub(b) = intersect_with / subtracted_by N(v_b) (vertex_set.cc:20-86).
struct SetExpr {
    khz_set_expr e;
    static SetExpr N(int i) { return SetExpr{{KHZ_BASE_NBR, (int8_t)i, {KHZ_OP_NONE, KHZ_OP_NONE}, {0, 0}}}; }
    static SetExpr Set(int s) { return SetExpr{{KHZ_BASE_SET, (int8_t)s, {KHZ_OP_NONE, KHZ_OP_NONE}, {0, 0}}}; }
    static SetExpr Cached() { return Set(4); }
    SetExpr And(int b) const { return with(KHZ_OP_AND, b); }
    SetExpr Sub(int b) const { return with(KHZ_OP_SUB, b); }

  private:
    SetExpr with(int op, int b) const {
        SetExpr r = *this;
        const int k = r.e.op[0] == KHZ_OP_NONE ? 0 : 1;
        r.e.op[k] = (int8_t)op;
        r.e.op_arg[k] = (int8_t)b;
        return r;
    }
};

// A candidate set with the generated code's filters: Above({a, ...}) keeps x > v_a for each a,
// Except({a, ...}) keeps x != v_a; for a counting term, Into(c) names its counter and
// OnlyIf(lo, hi) evaluates it only when v_lo < v_hi.
struct Term {
    khz_term t{};
    explicit Term(SetExpr s) {
        t.set = s.e;
        t.guard_lo = t.guard_hi = -1;
    }
    Term &Above(std::initializer_list<int> vs) {
        for (int a : vs) t.gt_mask |= (uint8_t)(1u << a);
        return *this;
    }
    Term &Except(std::initializer_list<int> vs) {
        for (int a : vs) t.ne_mask |= (uint8_t)(1u << a);
        return *this;
    }
    Term &Into(int counter) {
        t.counter = (int8_t)counter;
        return *this;
    }
    Term &OnlyIf(int lo, int hi) {
        t.guard_lo = (int8_t)lo;
        t.guard_hi = (int8_t)hi;
        return *this;
    }
};

class Schedule {
  public:
    explicit Schedule(int k) { s_.k = (int8_t)k; }
    // the next enumerating level (levels 1 .. k-2, in order); `cached` is computed on entry
    Schedule &Level(const Term &t, bool finalized = false) { return add(t, nullptr, finalized); }
    Schedule &Level(const Term &t, const SetExpr &cached, bool finalized = false) { return add(t, &cached, finalized); }
    Schedule &Count(const Term &t) {
        if (s_.num_terms < 2) s_.last[s_.num_terms++] = t.t;
        return *this;
    }
    const khz_pattern_schedule &get() const { return s_; }

  private:
    Schedule &add(const Term &t, const SetExpr *cached, bool finalized) {
        if (next_ < 5) {
            khz_level &l = s_.levels[next_++];
            l.term = t.t;
            l.finalized = finalized ? 1 : 0;
            if (cached) {
                l.has_cached = 1;
                l.cached = cached->e;
            }
        }
        return *this;
    }
    khz_pattern_schedule s_{};
    int next_ = 1;
};

// Registers an app of one or more schedules run one after another; returns its app id.
inline khz_app_id register_app(const std::vector<Schedule> &runs, const std::vector<uint32_t> &multiplicities) {
    khz_app_desc d{};
    d.num_runs = (int32_t)runs.size();
    d.num_counts = (int32_t)multiplicities.size();
    for (size_t i = 0; i < multiplicities.size() && i < KHZ_MAX_COUNTS; ++i) d.multiplicity[i] = multiplicities[i];
    for (size_t r = 0; r < runs.size() && r < 6; ++r) d.runs[r] = runs[r].get();
    int32_t id = 0;
    check(khz_app_register(&d, &id));
    return (khz_app_id)id;
}

class DistributedApplication {
  public:
    // (num_threads, graph_path, max_pattern_size, apply, load_vertex_labels, ...) of
    // distributed_application.h:38-43; `schedule` replaces `apply`.  Threads, memory sizes and
    // cache parameters of the CPU engine have no meaning on the device and are ignored.
    DistributedApplication(int num_threads, const std::string &graph_path, int max_pattern_size,
                           khz_app_id schedule, bool load_vertex_labels = false, int device = 0)
        : num_threads_(num_threads), max_pattern_size_(max_pattern_size), schedule_(schedule) {
        check(khz_ctx_create(device, &ctx_));
        // node labels are kept only when asked for, as the reference's loader does
        // (graph_loader.h:773-822)
        khz_status s = khz_graph_load_dgraph(ctx_, graph_path.c_str(), load_vertex_labels ? 0u : KHZ_SKIP_LABELS,
                                             &graph_);
        if (s != KHZ_OK) {
            khz_ctx_destroy(ctx_);
            check(s);
        }
    }
    ~DistributedApplication() { khz_ctx_destroy(ctx_); }
    DistributedApplication(const DistributedApplication &) = delete;
    DistributedApplication &operator=(const DistributedApplication &) = delete;

    template <typename T>
    Aggregator<T> *alloc_aggregator() {
        aggregators_.push_back(new Aggregator<EdgeId>());
        return reinterpret_cast<Aggregator<T> *>(aggregators_.back());
    }
    template <typename T>
    void dealloc_aggregator(Aggregator<T> *a) {
        for (auto &p : aggregators_)
            if ((void *)p == (void *)a) p = nullptr;
        delete a;
    }

    // run() (distributed_application.cc:259-356): one count of every pattern of the schedule.
    // Each aggregator receives its pattern's raw count (the app's own `evaluate() /
    // multiplicities[i]` stays as written).  With restrict_starting_vertex_label only the start
    // vertices of that label are extended (engine.cc:1457-1496); the graph must have been loaded
    // with load_vertex_labels.
    void run(bool disable_output = false, bool restrict_starting_vertex_label = false, LabelId label = 0) {
        (void)disable_output;
        uint64_t counts[KHZ_MAX_COUNTS];
        khz_stats st;
        const int nc = khz_app_num_counts(schedule_);
        if (restrict_starting_vertex_label) {
            check(khz_count_restricted(ctx_, graph_, schedule_, label, counts, &st, nullptr));  // raw counts
        } else {
            check(khz_count(ctx_, graph_, schedule_, counts, &st, nullptr));
            for (int i = 0; i < nc; ++i) counts[i] *= (uint64_t)khz_app_multiplicity(schedule_, i);
        }
        num_extensions_ += st.num_extensions;
        for (int i = 0; i < nc && i < (int)aggregators_.size(); ++i)
            if (aggregators_[i]) aggregators_[i]->set(counts[i]);
        last_counts_.assign(counts, counts + nc);
    }

    int get_num_threads() const { return num_threads_; }
    int get_max_pattern_size() const { return max_pattern_size_; }
    // the engine's NumExtensions summed over all run() calls (engine.cc:924, engine.h:1250-1254)
    EdgeId num_extensions() const { return num_extensions_; }
    const std::vector<uint64_t> &last_counts() const { return last_counts_; }
    khz_ctx *context() { return ctx_; }
    khz_graph graph() const { return graph_; }

  private:
    int num_threads_, max_pattern_size_;
    khz_app_id schedule_;
    khz_ctx *ctx_ = nullptr;
    khz_graph graph_ = 0;
    std::vector<Aggregator<EdgeId> *> aggregators_;
    std::vector<uint64_t> last_counts_;
    EdgeId num_extensions_ = 0;
};

}  // namespace Khuzdul
