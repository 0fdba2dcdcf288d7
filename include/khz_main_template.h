// khz_main_template.h — the reference's legacy main_template.h entry point on the device engine.
//
// An app written against main_template.h (main_template.h:1-122) defines
//     EdgeId mining_graph(CSRGraph<Empty, Empty> &graph);
// and expands INSERT_MAIN_FUNCTION(APP_NAME) to get its main(): usage check, graph load, one
// warm-up call, one timed run, "<APP_NAME> result: <count>".  Here the graph is the device graph
// (Khuzdul::DeviceGraph, loaded from the same .dgraph file), and mining_graph counts with one of the
// device schedules: KHZ_MINING_FUNCTION(schedule) defines it for a built-in or registered app.
// The reference's INSERT_MINING_FUNCTION_INITIALIZATION / FINALIZATION macros set up CPU memory
// pools and per-thread vertex ranges for a hand-written CPU loop; a device schedule needs neither,
// so they are not provided.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "khz_khuzdul.hpp"

namespace Khuzdul {

// The device-resident stand-in for CSRGraph<Empty, Empty> (graph.h:54-141).
class DeviceGraph {
  public:
    explicit DeviceGraph(const std::string &path, int device = 0) {
        check(khz_ctx_create(device, &ctx_));
        khz_status s = khz_graph_load_dgraph(ctx_, path.c_str(), KHZ_SKIP_LABELS, &g_);
        if (s != KHZ_OK) {
            khz_ctx_destroy(ctx_);
            check(s);
        }
        check(khz_graph_info_get(ctx_, g_, &info_));
    }
    ~DeviceGraph() { khz_ctx_destroy(ctx_); }
    DeviceGraph(const DeviceGraph &) = delete;
    DeviceGraph &operator=(const DeviceGraph &) = delete;
    VertexId get_num_vertices() const { return info_.num_vertices; }
    EdgeId get_num_edges() const { return info_.num_entries; }
    VertexId get_max_degree() const { return info_.max_degree; }
    // the first pattern count of `app` (its only one for the single-pattern apps)
    EdgeId count(khz_app_id app) {
        uint64_t c[KHZ_MAX_COUNTS];
        check(khz_count(ctx_, g_, app, c, nullptr, nullptr));
        return c[0];
    }
    // every pattern count of `app`
    std::vector<EdgeId> count_all(khz_app_id app) {
        uint64_t c[KHZ_MAX_COUNTS];
        check(khz_count(ctx_, g_, app, c, nullptr, nullptr));
        return std::vector<EdgeId>(c, c + khz_app_num_counts(app));
    }
    khz_ctx *context() { return ctx_; }
    khz_graph handle() const { return g_; }

  private:
    khz_ctx *ctx_ = nullptr;
    khz_graph g_ = 0;
    khz_graph_info info_{};
};

inline double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace Khuzdul

// mining_graph for a device schedule (a khz_app_id: built-in, or returned by khz_app_register)
#define KHZ_MINING_FUNCTION(SCHEDULE) \
    Khuzdul::EdgeId mining_graph(Khuzdul::DeviceGraph &graph) { return graph.count((khz_app_id)(SCHEDULE)); }

// main() of a single-pattern app (main_template.h:1-27): one warm-up call, one timed run.
#define INSERT_MAIN_FUNCTION(APP_NAME)                                                   \
    int main(int argc, char **argv) {                                                    \
        if (argc != 2) {                                                                 \
            printf("usage: " #APP_NAME " [graph dataset (dgraph format)]\n");            \
            exit(-1);                                                                    \
        }                                                                                \
        try {                                                                            \
            Khuzdul::DeviceGraph graph(argv[1]);                                         \
            printf("warming up...\n");                                                   \
            Khuzdul::EdgeId count = mining_graph(graph);                                 \
            int runs = 1;                                                                \
            double mining = 0;                                                           \
            for (int run = 0; run < runs; ++run) {                                       \
                printf("run = %d\n", run);                                               \
                mining -= Khuzdul::wall_seconds();                                       \
                count = mining_graph(graph);                                             \
                mining += Khuzdul::wall_seconds();                                       \
                printf("\tcnt = %lu\n", (unsigned long)count);                           \
            }                                                                            \
            printf(#APP_NAME " result: %lu\n", (unsigned long)count);                    \
            printf("mining: %.3f (ms)\n", mining * 1000.0);                              \
        } catch (const Khuzdul::Error &e) {                                              \
            fprintf(stderr, #APP_NAME ": %s\n", e.what());                               \
            return 1;                                                                    \
        }                                                                                \
        return 0;                                                                        \
    }

// main() of a multi-pattern app (main_template.h:29-53): mining_graph prints its own counts.
#define INSERT_MAIN_FUNCTION_MULTI_PATTERNS(APP_NAME)                                    \
    int main(int argc, char **argv) {                                                    \
        if (argc != 2) {                                                                 \
            printf("usage: " #APP_NAME " [graph dataset (dgraph format)]\n");            \
            exit(-1);                                                                    \
        }                                                                                \
        try {                                                                            \
            Khuzdul::DeviceGraph graph(argv[1]);                                         \
            int runs = 1;                                                                \
            for (int run = 0; run < runs; ++run) {                                       \
                double runtime = -Khuzdul::wall_seconds();                               \
                mining_graph(graph);                                                     \
                runtime += Khuzdul::wall_seconds();                                      \
                printf("Runtime: %.3f (ms)\n", runtime * 1000.);                         \
            }                                                                            \
        } catch (const Khuzdul::Error &e) {                                              \
            fprintf(stderr, #APP_NAME ": %s\n", e.what());                               \
            return 1;                                                                    \
        }                                                                                \
        return 0;                                                                        \
    }
