// khz_vertex_set.cuh — the reference's VertexSet (vertex_set.h:14-55) as a device type, for CUDA
// code that does its own set algebra on the engine's CSR (khz_graph_info gives its device pointers).
//
// A VertexSet is a non-owning view {vertices_list_, num_vertices_} of a sorted, strictly
// increasing uint32 list, exactly as in the reference; operations that produce a set write into a
// caller-provided VertexSet whose buffer holds at least as many entries as this set (the
// reference's contract, vertex_set.cc:30-48).  Every member function is WARP-COLLECTIVE: all 32
// lanes of a warp call it with the same arguments and get the same result; outputs stay sorted.
// Semantics follow vertex_set.cc:20-184 and utilities.h:64-86, including the early returns on
// empty inputs and the bounded variants, which only consider this set's members below
// `upper_bound`.
#pragma once
#include <stdint.h>

#include "khz_setops.cuh"

namespace Khuzdul {
namespace device {

struct VertexSet {
    uint32_t *vertices_list_;
    uint32_t num_vertices_;

    __device__ VertexSet() : vertices_list_(nullptr), num_vertices_(0) {}
    __device__ VertexSet(uint32_t *list, uint32_t n) : vertices_list_(list), num_vertices_(n) {}
    __device__ uint32_t get_num_vertices() const { return num_vertices_; }
    __device__ uint32_t get_vertex(uint32_t i) const { return vertices_list_[i]; }
    __device__ uint32_t *get_vertices_list() const { return vertices_list_; }

    // result = this n other (vertex_set.cc:20-49)
    __device__ void intersect_with(const VertexSet &other, VertexSet *result) const {
        result->num_vertices_ = intersect_into(num_vertices_, other, result->vertices_list_);
    }
    // result = this \ other (vertex_set.cc:51-86)
    __device__ void subtracted_by(const VertexSet &other, VertexSet *result) const {
        result->num_vertices_ = subtract_into(num_vertices_, other, result->vertices_list_);
    }
    // |this n other| without materialising it (vertex_set.cc:88-111)
    __device__ uint32_t intersect_and_count(const VertexSet &other) const {
        return intersect_into(num_vertices_, other, nullptr);
    }
    // the same over this set's members < upper_bound (vertex_set.cc:113-184)
    __device__ void bounded_intersect_with(const VertexSet &other, VertexSet *result, uint32_t upper_bound) const {
        result->num_vertices_ = intersect_into(prefix_below(upper_bound), other, result->vertices_list_);
    }
    __device__ void bounded_subtracted_by(const VertexSet &other, VertexSet *result, uint32_t upper_bound) const {
        result->num_vertices_ = subtract_into(prefix_below(upper_bound), other, result->vertices_list_);
    }

  private:
    __device__ uint32_t prefix_below(uint32_t ub) const { return khz::lower_bound_plain(vertices_list_, 0, num_vertices_, ub); }
    __device__ uint32_t intersect_into(uint32_t na, const VertexSet &o, uint32_t *out) const {
        const khz::Filter none = {0, 0, 0, {0, 0, 0, 0}};
        if (na == 0 || o.num_vertices_ == 0) return 0;
        // probe with the shorter list; the result is ordered either way
        return na <= o.num_vertices_ ? khz::warp_probe<false>(vertices_list_, na, o.vertices_list_, o.num_vertices_, out, none).full
                                     : khz::warp_probe<false>(o.vertices_list_, o.num_vertices_, vertices_list_, na, out, none).full;
    }
    __device__ uint32_t subtract_into(uint32_t na, const VertexSet &o, uint32_t *out) const {
        const khz::Filter none = {0, 0, 0, {0, 0, 0, 0}};
        if (na == 0) return 0;
        return khz::warp_probe<true>(vertices_list_, na, o.vertices_list_, o.num_vertices_, out, none).full;
    }
};

// trim_v_list (utilities.h:64-74): the number of members < upper_bound
__device__ inline uint32_t trim_v_list(const VertexSet &s, uint32_t upper_bound) {
    return khz::lower_bound_plain(s.vertices_list_, 0, s.num_vertices_, upper_bound);
}
// trim_v_list_lower_bound (utilities.h:76-86): the number of members <= lower_bound
__device__ inline uint32_t trim_v_list_lower_bound(const VertexSet &s, uint32_t lower_bound) {
    return khz::upper_bound_plain(s.vertices_list_, 0, s.num_vertices_, lower_bound);
}

}  // namespace device
}  // namespace Khuzdul
