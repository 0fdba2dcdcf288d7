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
