// Sampled driver for the reference's own pattern apps (CPU oracle / CPU baseline only).
//
// The app source named by KHZ_APP_SRC is compiled unmodified; only its main() is
// renamed out of the way.  This driver then runs the app's own apply(), aggregators
// and multiplicities through the reference's DistributedApplication, but with
// load_vertex_labels = true and run(disable_output, restrict_starting_vertex_label =
// true, label) (distributed_application.h:38-54, engine.cc:1457-1496), so that a run
// extends only the start vertices v_0 whose on-disk label equals `label`.  With a
// .dgraph whose node labels are v % S this processes one S-th slice of the start
// vertices: a bounded, reproducible sample of the full workload.
//
// usage: sample_<app> <labeled graph.dgraph> <num_threads|-1> <label> <runs> [warm-up runs]
// prints the reference's own lines: "Pattern count <i>: <n>" and "Average runtime: <ms> (ms)" (over
// the timed runs, which follow the untimed warm-up runs), plus "NumExtensionsTotal: <n>" (the
// engine's NumExtensions accumulated over all runs, warm-up runs included).
#define main khz_reference_app_main
#include KHZ_APP_SRC
#undef main

int main(int argc, char **argv) {
    if (argc != 5 && argc != 6) {
        fprintf(stderr, "usage: %s <labeled graph.dgraph> <num_threads|-1> <label> <runs> [warm-up runs]\n",
                argv[0]);
        return 2;
    }
    DistributedSys::init_distributed_sys();
    int num_threads = std::atoi(argv[2]);
    LabelId label = (LabelId)std::atoi(argv[3]);
    int runs = std::atoi(argv[4]);
    int warmup = argc == 6 ? std::atoi(argv[5]) : 0;
    Khuzdul::DistributedApplication *app = new Khuzdul::DistributedApplication(
        num_threads, std::string(argv[1]), MAX_COUNTING_PATTERN_SIZE, Khuzdul::apply, true);
#ifndef ENABLE_COMPUTE_FUSION
    Khuzdul::count = app->alloc_aggregator<EdgeId>();
#else
    for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) Khuzdul::counts[p] = app->alloc_aggregator<EdgeId>();
#endif
    Khuzdul::LocalPerformanceMetric::init_local_metrics();
    double average_runtime = 0;
    EdgeId cnt[NUM_COUNTING_PATTERNS];
    for (int run = -warmup; run < runs; ++run) {
        if (run == 0) average_runtime = 0;  // the warm-up runs are not timed
        average_runtime -= get_time();
#ifndef ENABLE_COMPUTE_FUSION
        for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) {
            Khuzdul::curr_pattern_id = p;
            Khuzdul::count->clear();
            app->run(true, true, label);
            cnt[p] = Khuzdul::count->evaluate();
#ifndef KHZ_NO_MULTIPLICITIES  // kgraphpi apps count each embedding once and define no multiplicities
            assert(cnt[p] % multiplicities[p] == 0);
            cnt[p] /= multiplicities[p];
#endif
        }
#else
        Khuzdul::curr_pattern_id = 0;
        for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) Khuzdul::counts[p]->clear();
        app->run(true, true, label);
        for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) {
            EdgeId raw = Khuzdul::counts[p]->evaluate();
            assert(raw % multiplicities[p] == 0);
            cnt[p] = raw / multiplicities[p];
        }
#endif
        average_runtime += get_time();
    }
    for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) printf("Pattern count %d: %lu\n", p, (unsigned long)cnt[p]);
    printf("Average runtime: %.3f (ms)\n", average_runtime * 1000 / (runs > 0 ? runs : 1));
    // The engine adds its NumExtensions to the global metric in its destructor (engine.cc:1272).
#ifndef ENABLE_COMPUTE_FUSION
    app->dealloc_aggregator(Khuzdul::count);
#else
    for (int p = 0; p < NUM_COUNTING_PATTERNS; ++p) app->dealloc_aggregator(Khuzdul::counts[p]);
#endif
    delete app;
    printf("NumExtensionsTotal: %.0f\n", Khuzdul::LocalPerformanceMetric::num_extensions);
    fflush(stdout);
    DistributedSys::finalize_distributed_sys();
    return 0;
}
