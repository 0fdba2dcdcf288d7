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
