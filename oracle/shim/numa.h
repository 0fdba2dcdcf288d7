/*
 * One-node libnuma shim used only to compile the reference's own C++ sources
 * as a CPU oracle (test infrastructure; never linked into the product).
 * Allocations are zeroed heap blocks (the reference relies on
 * numa_alloc_onnode returning zeroed memory, engine.cc:15-85); placement and
 * interleave calls are no-ops on a single node.
 */
#ifndef KHZ_ORACLE_NUMA_SHIM_H
#define KHZ_ORACLE_NUMA_SHIM_H

#include <stdlib.h>
#include <string.h>
#include <unistd.h>

struct bitmask { unsigned long size; unsigned long *maskp; };

static inline int numa_available(void) { return 0; }
static inline int numa_num_configured_cpus(void) {
    const char *env = getenv("KHZ_ORACLE_CPUS");
    if (env && atoi(env) > 0) return atoi(env);
    return (int)sysconf(_SC_NPROCESSORS_ONLN);
}
static inline int numa_num_configured_nodes(void) { return 1; }
static inline int numa_run_on_node(int node) { (void)node; return 0; }
static inline void *numa_alloc_onnode(size_t size, int node) {
    (void)node;
    if (size == 0) size = 1;
    return calloc(1, size);
}
static inline void *numa_alloc_interleaved(size_t size) { return numa_alloc_onnode(size, 0); }
static inline void numa_free(void *p, size_t size) {
    (void)size;
    free(p);
}
static inline struct bitmask *numa_parse_nodestring(const char *s) {
    (void)s;
    static unsigned long bits = 1;
    static struct bitmask m = {1, &bits};
    return &m;
}
static inline void numa_set_interleave_mask(struct bitmask *m) { (void)m; }

#endif
