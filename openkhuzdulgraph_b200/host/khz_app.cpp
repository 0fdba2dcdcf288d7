// khz_app — the reference's pattern-counting programs, one binary for all schedules.
//
//   khz_app <app> <graph_path (*.dgraph)> [num_threads (-1: all)] [num_runs, default 3] [need_warmup: false]
//
// <app> is a schedule name (kautomine_triangle, kautomine_four_clique, kautomine_five_clique,
// kautomine_three_motif, kgraphpi_triangle, kgraphpi_four_clique, kgraphpi_five_clique,
// kgraphpi_three_motif, kgraphpi_four_cycle, kgraphpi_house, kgraphpi_tailed_triangle,
// kautomine_four_motif).  The argument list and the output lines follow the reference apps'
// main() (kautomine/triangle.cc:124-259): "Pattern count <i>: <n>" per run, then
// "Average runtime: <ms> (ms)" (count time, graph load excluded), then the engine's NumExtensions.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "khz_khuzdul.hpp"

static const char *kNames[KHZ_NUM_APPS] = {
    "kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique", "kautomine_three_motif",
    "kgraphpi_triangle",  "kgraphpi_four_clique",  "kgraphpi_five_clique",  "kgraphpi_three_motif",
    "kgraphpi_four_cycle", "kgraphpi_house",       "kgraphpi_tailed_triangle", "kautomine_four_motif"};

// kautomine_three_fsm <graph_path (*.dgraph)> <support threshold> [num_threads]: the 3-FSM app's
// main() (kautomine/three_fsm.cc:744-800) with its per-level lines
static int three_fsm_main(int argc, char **argv) {
    if (argc != 4 && argc != 5) {
        fprintf(stderr, "usage: %s kautomine_three_fsm <graph_path (*.dgraph)> <support threshold> [num_threads, default: all]\n",
                argv[0]);
        return 2;
    }
    static const char *kLevel[6] = {"single-vertex", "single-edge", "wedge", "triangle", "four-chain", "three-star"};
    try {
        Khuzdul::DistributedApplication application(argc == 5 ? atoi(argv[4]) : -1, argv[2], 4, KHZ_KAUTO_3MOTIF,
                                                    true);
        khz_fsm_result r;
        uint32_t found = 0;
        Khuzdul::check(khz_fsm(application.context(), application.graph(), (uint32_t)strtoul(argv[3], nullptr, 10),
                               &r, nullptr, 0, &found));
        printf("\nrun = 0\n");
        for (int l = 0; l < 6; ++l)
            printf("Number of frequent %s patterns: %u, support sum%s: %lu\n", kLevel[l], r.level[l].num_frequent,
                   l == 0 ? "" : " of them", (unsigned long)r.level[l].support_sum);
        printf("\n************************************************\n");
        printf("Average runtime: %.3f (ms)\n", r.ms);
        printf("************************************************\n\n");
    } catch (const Khuzdul::Error &e) {
        fprintf(stderr, "khz_app: %s\n", e.what());
        return 1;
    }
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && strcmp(argv[1], "kautomine_three_fsm") == 0) return three_fsm_main(argc, argv);
    if (argc < 3 || argc > 6) {
        fprintf(stderr,
                "usage: %s <app> <graph_path (*.dgraph)> [num_threads (-1: all threads), default: all] "
                "[num_runs, default: 3] [need_warmup: false]\n",
                argv[0]);
        return 2;
    }
    int app = -1;
    for (int i = 0; i < KHZ_NUM_APPS; ++i)
        if (strcmp(argv[1], kNames[i]) == 0) app = i;
    if (app < 0) {
        fprintf(stderr, "unknown app %s\n", argv[1]);
        return 2;
    }
    const int num_threads = argc >= 4 ? atoi(argv[3]) : -1;
    const int runs = argc >= 5 ? atoi(argv[4]) : 3;
    bool warmup = false;
    if (argc >= 6) {
        if (strcmp(argv[5], "true") == 0) warmup = true;
        else if (strcmp(argv[5], "false") != 0) {
            fprintf(stderr, "Bad need_warmup argument: %s\n", argv[5]);
            return 2;
        }
    }
    try {
        const int npat = khz_app_num_counts((khz_app_id)app);
        Khuzdul::DistributedApplication application(num_threads, argv[2], 5, (khz_app_id)app);
        std::vector<Khuzdul::Aggregator<Khuzdul::EdgeId> *> counts;
        for (int p = 0; p < npat; ++p) counts.push_back(application.alloc_aggregator<Khuzdul::EdgeId>());
        if (warmup) {
            printf("****** Warming up... ******\n");
            application.run();
        }
        const Khuzdul::EdgeId ext_before = application.num_extensions();
        double total = 0;
        for (int run = 0; run < runs; ++run) {
            printf("\nrun = %d\n", run);
            for (auto *c : counts) c->clear();
            const auto t0 = std::chrono::steady_clock::now();
            application.run();
            total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            for (int p = 0; p < npat; ++p) {
                const Khuzdul::EdgeId raw = counts[p]->evaluate();
                const int mult = khz_app_multiplicity((khz_app_id)app, p);
                printf("    Pattern count %d: %lu\n", p, (unsigned long)(raw / (Khuzdul::EdgeId)mult));
            }
        }
        printf("\n************************************************\n");
        printf("Average runtime: %.3f (ms)\n", runs > 0 ? total * 1000.0 / runs : 0.0);
        printf("************************************************\n\n");
        printf("NumExtensions: %.3f\n",
               runs > 0 ? (double)(application.num_extensions() - ext_before) / runs : 0.0);
        for (auto *c : counts) application.dealloc_aggregator(c);
    } catch (const Khuzdul::Error &e) {
        fprintf(stderr, "khz_app: %s\n", e.what());
        return 1;
    }
    return 0;
}
