"""The bench's multi-rank plumbing (one process per GPU under torchrun) on CPU: two gloo ranks
rendezvous through the same helpers, agree on the maximum of their timings and meet at barriers."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "KHZ_BENCH_DIST_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    r, w, local = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank)
    bench.barrier(w, "cpu")
    m = bench.max_over_ranks(10.0 * (rank + 1) + 0.5, w, "cpu")
    bench.barrier(w, "cpu")
    out.put((rank, m))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 20.5), (1, 20.5)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25


def test_bench_reads_kernel_traffic_from_the_profile():
    sys.path.insert(0, ROOT)
    import bench
    from openkhuzdulgraph_b200 import khz
    got = {k: bench.profile_traffic(k) for k in khz.Stats.PHASES[:3]}
    assert all(isinstance(v, int) and v > 0 for v in got.values()), got
    assert bench.profile_traffic("no_such_kernel") is None


def test_clock_summary_reads_nvidia_smi_lines():
    """The clocks object of the bench line: the median SM clock under load, the highest max clock and
    the throttle reasons seen active (nvidia-smi csv, noheader, nounits)."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0)
    c.lines = ["1965, 1965, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "1950, 1965, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "1900, 1965, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "[N/A], 1965, garbage",
               ""]
    s = c.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    c.lines = ["1300, 1965, 0x0000000000000048, Active, Not Active, Active, Not Active"]
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    c.lines = []
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
