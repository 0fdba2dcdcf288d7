"""The counting entry point that allocates no device memory.

It exists for callers that may not call cudaMalloc (a host framework that owns all device
memory through its own pool, a plugin in a process with a locked-down allocator).  Through
the C ABI it must give exactly the output of the regular entry point, call after call: its
scratch lives in one fixed device array that every call reuses, so a second call must not
see the first call's leftovers.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import orc

pytestmark = pytest.mark.gpu

APPS = list(orc.APPS)


def _graphs():
    out = []
    canon, n = orc.er(400, 4000, seed=7)
    out.append((orc.symmetrize(canon), n))
    canon, n = orc.rmat(10, 8, seed=1)
    out.append((orc.symmetrize(canon), n))
    return out


def test_no_alloc_matches_regular_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openkhuzdulgraph_b200 import khz
    with khz.Context(0) as ctx:
        ctx.set_config(engine=khz.ENGINE_DFS)
        d_out = torch.zeros(8, dtype=torch.int64, device="cuda")
        for sym, n in _graphs():
            g = ctx.graph_from_edges(sym, n)
            gi = g.info()
            for app in APPS:
                exp_counts, st = ctx.count(g, app)
                nc = khz.num_counts(app)
                for _ in range(2):  # two calls in a row on the shared scratch
                    d_out.fill_(-1)
                    khz.count_noalloc(gi.d_offsets, gi.d_adj, gi.num_vertices, gi.num_entries, app,
                                      d_out.data_ptr())
                    got = d_out.cpu().numpy().view(np.uint64)
                    assert [int(x) for x in got[:nc]] == exp_counts, app
                    assert int(got[6]) == st.num_extensions, app
                    assert int(got[7]) == 0
            g.free()


def test_no_alloc_at_its_degree_limit_allocates_nothing():
    """A graph whose largest degree is exactly the limit (a star of 1024 leaves, consecutive leaves
    joined into triangles with the centre, plus a few chords) fills every warp slot to capacity; the
    counts must still be the regular entry point's, and the device's free memory must not change
    across the calls (after the first, which may load the library's device code)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openkhuzdulgraph_b200 import khz
    leaves = 1024
    pairs = [(0, v) for v in range(1, leaves + 1)]
    pairs += [(v, v + 1) for v in range(1, leaves, 2)]
    pairs += [(v, v + 7) for v in range(2, leaves - 7, 37)]
    canon = np.array(sorted(set(pairs)), dtype=np.uint32)
    sym = orc.symmetrize(canon)
    with khz.Context(0) as ctx:
        ctx.set_config(engine=khz.ENGINE_DFS)
        g = ctx.graph_from_edges(sym, leaves + 1)
        gi = g.info()
        assert gi.max_degree == 1024
        d_out = torch.zeros(8, dtype=torch.int64, device="cuda")
        expected = {app: ctx.count(g, app) for app in APPS}
        khz.count_noalloc(gi.d_offsets, gi.d_adj, gi.num_vertices, gi.num_entries, 0, d_out.data_ptr())
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        for app in APPS:
            exp_counts, st = expected[app]
            nc = khz.num_counts(app)
            for _ in range(2):
                d_out.fill_(-1)
                khz.count_noalloc(gi.d_offsets, gi.d_adj, gi.num_vertices, gi.num_entries, app, d_out.data_ptr())
                got = d_out.cpu().numpy().view(np.uint64)
                assert [int(x) for x in got[:nc]] == exp_counts, app
                assert int(got[6]) == st.num_extensions, app
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
        g.free()


def test_no_alloc_rejects_degrees_beyond_its_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openkhuzdulgraph_b200 import khz
    leaves = 1100
    canon = np.stack([np.zeros(leaves, dtype=np.uint32), np.arange(1, leaves + 1, dtype=np.uint32)], axis=1)
    sym = orc.symmetrize(canon)
    with khz.Context(0) as ctx:
        g = ctx.graph_from_edges(sym, leaves + 1)
        gi = g.info()
        d_out = torch.zeros(8, dtype=torch.int64, device="cuda")
        with pytest.raises(khz.KhzError) as e:
            khz.count_noalloc(gi.d_offsets, gi.d_adj, gi.num_vertices, gi.num_entries, 0, d_out.data_ptr())
        assert e.value.status == 1
        g.free()
