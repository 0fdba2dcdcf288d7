"""include/khz_vertex_set.cuh: the reference's VertexSet as a warp-collective device type.  A small
CUDA library written against the header is compiled here with nvcc for sm_100a (no GPU needed);
on a GPU its results are compared with the oracle's restatement of vertex_set.cc."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
import orc

SRC = r"""
#include <cuda_runtime.h>
#include "khz_vertex_set.cuh"
using Khuzdul::device::VertexSet;

// one warp per pair: op 0 intersect_with, 1 subtracted_by, 2 intersect_and_count,
// 3 bounded_intersect_with, 4 bounded_subtracted_by, 5 trim_v_list, 6 trim_v_list_lower_bound
__global__ void vs_kernel(int op, const uint64_t *a_off, uint32_t *a, const uint64_t *b_off, uint32_t *b,
                          const uint32_t *bound, uint32_t *out, uint32_t *out_len, uint32_t n_pairs) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n_pairs) return;
    VertexSet A(a + a_off[w], (uint32_t)(a_off[w + 1] - a_off[w]));
    VertexSet B(b + b_off[w], (uint32_t)(b_off[w + 1] - b_off[w]));
    VertexSet R(out + a_off[w], 0);
    uint32_t r = 0;
    switch (op) {
        case 0: A.intersect_with(B, &R); r = R.get_num_vertices(); break;
        case 1: A.subtracted_by(B, &R); r = R.get_num_vertices(); break;
        case 2: r = A.intersect_and_count(B); break;
        case 3: A.bounded_intersect_with(B, &R, bound[w]); r = R.get_num_vertices(); break;
        case 4: A.bounded_subtracted_by(B, &R, bound[w]); r = R.get_num_vertices(); break;
        case 5: r = Khuzdul::device::trim_v_list(A, bound[w]); break;
        default: r = Khuzdul::device::trim_v_list_lower_bound(A, bound[w]); break;
    }
    if ((threadIdx.x & 31) == 0) out_len[w] = r;
}

extern "C" int vs_run(int op, const uint64_t *a_off, uint32_t *a, const uint64_t *b_off, uint32_t *b,
                      const uint32_t *bound, uint32_t *out, uint32_t *out_len, uint32_t n_pairs) {
    vs_kernel<<<(n_pairs + 7) / 8, 256>>>(op, a_off, a, b_off, b, bound, out, out_len, n_pairs);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}
"""


def _compile(td, shared):
    src = os.path.join(td, "vs.cu")
    with open(src, "w") as f:
        f.write(SRC)
    out = os.path.join(td, "libvs.so" if shared else "vs.o")
    cmd = ["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
           "-I" + os.path.join(ROOT, "include"), "-Xcompiler", "-fPIC", src, "-o", out]
    cmd += ["-shared"] if shared else ["-c"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def test_header_compiles_for_sm100a():
    with tempfile.TemporaryDirectory() as td:
        assert os.path.getsize(_compile(td, shared=False)) > 0


def _pairs(rng, n_pairs):
    a_lists, b_lists, bounds = [], [], []
    for i in range(n_pairs):
        na, nb = [(0, 5), (7, 0), (0, 0), (1, 1)][i] if i < 4 else (int(rng.integers(0, 300)), int(rng.integers(0, 300)))
        a_lists.append(np.unique(rng.integers(0, 600, na)).astype(np.uint32))
        b_lists.append(np.unique(rng.integers(0, 600, nb)).astype(np.uint32))
        bounds.append(int(rng.integers(0, 620)))
    return a_lists, b_lists, bounds


@pytest.mark.gpu
def test_device_vertex_set_matches_oracle():
    import torch
    rng = np.random.default_rng(5)
    a_lists, b_lists, bounds = _pairs(rng, 200)
    a_off = np.concatenate([[0], np.cumsum([len(x) for x in a_lists])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([len(x) for x in b_lists])]).astype(np.uint64)
    cat = lambda ls: np.concatenate(ls + [np.zeros(1, np.uint32)]).astype(np.uint32)  # noqa: E731
    dev = lambda x: torch.from_numpy(x.view(np.int64) if x.dtype == np.uint64 else x.view(np.int32)).cuda()  # noqa
    d_aoff, d_boff, d_a, d_b = dev(a_off), dev(b_off), dev(cat(a_lists)), dev(cat(b_lists))
    d_bound = dev(np.array(bounds, dtype=np.uint32))
    with tempfile.TemporaryDirectory() as td:
        L = ctypes.CDLL(_compile(td, shared=True))
        L.vs_run.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 7 + [ctypes.c_uint32]
        for op in range(7):
            d_out = torch.zeros(max(int(a_off[-1]), 1), dtype=torch.int32, device="cuda")
            d_len = torch.zeros(len(a_lists), dtype=torch.int32, device="cuda")
            assert L.vs_run(op, d_aoff.data_ptr(), d_a.data_ptr(), d_boff.data_ptr(), d_b.data_ptr(),
                            d_bound.data_ptr(), d_out.data_ptr(), d_len.data_ptr(), len(a_lists)) == 0
            out, lens = d_out.cpu().numpy().view(np.uint32), d_len.cpu().numpy().view(np.uint32)
            for i, (a, b, ub) in enumerate(zip(a_lists, b_lists, bounds)):
                buf = np.zeros(max(len(a), 1), dtype=np.uint32)
                if op == 0:
                    k = orc.lib().orc_intersect(a, len(a), b, len(b), buf)
                elif op == 1:
                    k = orc.lib().orc_subtract(a, len(a), b, len(b), buf)
                elif op == 2:
                    k = orc.lib().orc_intersect_count(a, len(a), b, len(b))
                elif op == 3:
                    k = orc.lib().orc_bounded_intersect(a, len(a), b, len(b), ub, buf)
                elif op == 4:
                    k = orc.lib().orc_bounded_subtract(a, len(a), b, len(b), ub, buf)
                elif op == 5:
                    k = orc.lib().orc_trim(a, len(a), ub)
                else:
                    k = orc.lib().orc_trim_lower_bound(a, len(a), ub)
                assert lens[i] == k, (op, i)
                if op in (0, 1, 3, 4):
                    s = int(a_off[i])
                    assert np.array_equal(out[s:s + k], buf[:k]), (op, i)
