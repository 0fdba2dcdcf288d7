"""Benchmark: 4-clique counting on the degree-oriented R-MAT scale-22, edge-factor-16 graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one exact 4-clique count (kautomine/four_clique.cc schedule semantics) over the
whole graph.  The metric is embeddings/s = (NumExtensions + count) / time, NumExtensions
being the reference engine's own extension counter (engine.cc:924) for that schedule.

* value: device time (CUDA events around the counting launches, graph resident in HBM);
  the graph (256 MB of adjacency + 19 MB of offsets) is larger than the 126 MB L2, so no
  flush is needed between steps.
* e2e: the C-ABI path a user takes with host buffers: upload the oriented .dgraph edge list
  from pinned memory, device CSR build, count, copy the result back.
* roofline: the dominant kernel's DRAM bytes per launch (committed ncu capture, profiles/) / its
  CUDA-event time, against the measured HBM copy bandwidth; the kernel is instruction-issue bound,
  so the schedule's algorithmic bytes (instrumented run) / time are reported beside it, apart.
* --workload batch | serve | configs | app | fsm: the multi-graph batch, Poisson serving, every
  app of the full-size configurations, one app on one engine (profiling driver), and the 3-FSM.
* cpu_baseline: the reference's own kautomine four_clique app (oracle/_ref, compiled from the
  reference's sources) on a label-restricted slice of the start vertices, all host threads.
* --impl reference: the same reference binary as the timed arm, on the same slice.
* N > 1 (torchrun): replicas only; each rank counts the same graph on its own GPU.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, SEED = 22, 16, 1   # defaults; --scale / --edge-factor select a smaller case for profiling
RMAT_ABC = (0.57, 0.19, 0.19)
APP = "kautomine_four_clique"
KNOWN_COUNTS = {(22, 16): 123601255038, (21, 16): 46044614288}
SAMPLE_MOD = 32      # CPU sample: start vertices with v0 % 32 == 0 (one label class of 32)
METRIC = "embeddings/s (4-clique, exact uint64 count)"
def workload_name(scale=SCALE, edge_factor=EDGE_FACTOR):
    return ("4-clique count, R-MAT scale %d ef %d (a,b,c)=(0.57,0.19,0.19) seed 1, degree-oriented DAG"
            % (scale, edge_factor))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def profile_traffic(kernel):
    """DRAM bytes (read + write) per launch of a bench kernel, from the committed ncu summary of the
    bench workload (lines `traffic_bytes_per_launch <kernel> <bytes>`), or None."""
    path = os.path.join(ROOT, "profiles", "dram_clique4_rmat22.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                return int(parts[2])
    return None


def profile_counters(kernel):
    """Issue-active fraction, IPC and L2 hit rate of a bench kernel from the committed ncu capture of
    its small case (lines `ncu_counter <kernel> <name> <value>`), as a dict (empty if absent)."""
    out = {}
    path = os.path.join(ROOT, "profiles", "clique_block_kernel_rmat21.md")
    if not os.path.exists(path):
        return out
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 4 and parts[0] == "ncu_counter" and parts[1] == kernel:
                out[parts[2]] = float(parts[3])
    return out


def host_cpu():
    """CPU model, physical cores and logical CPUs of this host."""
    model, cores = "unknown", set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name":
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None and core is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None and core is not None:
            cores.add((phys, core))
    except OSError:
        pass
    logical = os.cpu_count() or 1
    return model, (len(cores) or logical), logical


def dist_setup(gpus):
    """One process per GPU (torchrun env).  The process group is NCCL; KHZ_BENCH_DIST_BACKEND=gloo
    selects gloo for CPU-only runs of the rank plumbing."""
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(os.environ.get("KHZ_BENCH_DIST_BACKEND", "nccl"),
                                timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def max_over_ranks(x, world, device):
    """The maximum of x over all ranks (device: the local CUDA device index, or "cpu")."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world, device):
    """All ranks meet, then the local device drains (device: CUDA index, or "cpu")."""
    import torch
    if world > 1:
        import torch.distributed as dist
        if isinstance(device, int):
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()
    if isinstance(device, int):
        torch.cuda.synchronize()


# ------------------------------------------------------------------------------ reference / CPU
def labelled_oriented_dgraph(g, tmpdir):
    """Writes the oriented graph as a labelled .dgraph (labels v % SAMPLE_MOD) for the sampled
    reference driver."""
    import numpy as np
    n = g.num_vertices
    path = os.path.join(tmpdir, "k_oriented_labeled.dgraph")
    g.write_dgraph(path, labels=(np.arange(n, dtype=np.uint64) % SAMPLE_MOD).astype(np.uint32))
    return path


def run_reference_sample(dgraph, runs, warmup=0):
    """The reference's own kautomine four_clique (apply + engine, compiled unmodified) over the
    start vertices of label class 0, `warmup` untimed runs first.  Returns a dict: per-run seconds,
    embeddings, count and NumExtensions per run, kind ("reference" or "port"), threads used."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    logical = os.cpu_count() or 1
    exe = os.path.join(orc.REF_DIR, "sample_" + APP)
    if os.path.exists(exe):
        counts, avg_ms, ext = orc.run_reference(APP, dgraph, threads=-1, runs=runs, label=0, timeout=3000,
                                                warmup=warmup)
        per_run_ext = ext // (runs + warmup)
        threads = max(1, logical - 2)  # the reference caps compute threads at CPUs - 2 (distributed_application.cc:80)
        return {"secs": avg_ms / 1000.0, "embeddings": per_run_ext + counts[0], "count": counts[0],
                "num_extensions": per_run_ext, "kind": "reference", "threads": threads}
    # the oracle port (C restatement) when the reference binaries are not present
    n, pairs, _ = orc.read_dgraph(dgraph)
    off, adj = orc.csr(pairs, n)
    for _ in range(warmup):
        orc.count(APP, off, adj, v0_mod=SAMPLE_MOD, v0_rem=0, threads=logical)
    t0 = time.time()
    for _ in range(runs):
        counts, ext, _ = orc.count(APP, off, adj, v0_mod=SAMPLE_MOD, v0_rem=0, threads=logical)
    dt = (time.time() - t0) / runs
    return {"secs": dt, "embeddings": ext + counts[0], "count": counts[0], "num_extensions": ext, "kind": "port",
            "threads": logical}


def reference_built_graph(scale, edge_factor, tmpdir):
    """The bench graph made without this repository's library: the oracle's generator (bit-identical
    to the device generator) writes the edge list, the reference's own converter and
    to_oriented_dataset_converter build the oriented .dgraph, and the node labels v % SAMPLE_MOD are
    inserted after its header.  Returns the labelled file's path (or None without oracle/_ref)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    conv = os.path.join(orc.REF_DIR, "converter")
    ori = os.path.join(orc.REF_DIR, "to_oriented_dataset_converter")
    if not (os.path.exists(conv) and os.path.exists(ori)):
        return None
    a, b, c = RMAT_ABC
    canon, n = orc.rmat(scale, edge_factor, a, b, c, seed=SEED)
    base = os.path.join(tmpdir, "k")
    canon.astype(np.uint32).tofile(base + ".biedgelist")
    del canon
    subprocess.run([conv, base, base, str(n), "0", "0", "0"], check=True, stdout=subprocess.DEVNULL)
    os.remove(base + ".biedgelist")
    subprocess.run([ori, base + ".dgraph", base + ".oriented"], check=True, stdout=subprocess.DEVNULL)
    os.remove(base + ".dgraph")
    raw = np.fromfile(base + ".oriented", dtype=np.uint8)
    os.remove(base + ".oriented")
    hdr = raw[:20].copy()
    hdr[12:16] = np.frombuffer(np.int32(1).tobytes(), dtype=np.uint8)  # has_node_label
    path = os.path.join(tmpdir, "k_oriented_labeled.dgraph")
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write((np.arange(n, dtype=np.uint64) % SAMPLE_MOD).astype(np.uint32).tobytes())
        f.write(raw[20:].tobytes())
    return path


# ------------------------------------------------------------------------------ main arms
def ours(args, rank, world, local):
    import numpy as np
    import torch
    from openkhuzdulgraph_b200 import khz

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = khz.Context(local)
    a, b, c = RMAT_ABC
    sym = ctx.generate_rmat(args.scale, args.edge_factor, a, b, c, SEED)
    g = sym.orient()
    gi = g.info()
    n, m = gi.num_vertices, gi.num_entries
    sym_info = sym.info()
    sym.free()

    # instrumented run (untimed): algorithmic bytes per phase, NumExtensions, count
    ctx.set_config(want_algo_bytes=1)
    ref_counts, st_stats = ctx.count(g, APP)
    ctx.set_config(want_algo_bytes=0)
    embeddings = st_stats.num_extensions + ref_counts[0]
    # 4-clique counts of these generated graphs, equal on the DFS engine (the schedule as written),
    # the bitmap engine and the symmetric input
    known = KNOWN_COUNTS.get((args.scale, args.edge_factor))
    assert known is None or ref_counts[0] == known, (ref_counts, known)

    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream
    for _ in range(args.warmup):
        counts, st = ctx.count(g, APP, stream=sptr)
        assert counts == ref_counts
    barrier(world, local)
    phase_ms = [0.0] * 4
    launches = 0
    step_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            counts, st = ctx.count(g, APP, stream=sptr)
            assert counts == ref_counts and st.num_extensions == st_stats.num_extensions
            step_ms.append(st.kernel_ms)
            launches += st.launches
            for p in range(4):
                phase_ms[p] += st.phase_ms[p]
    barrier(world, local)
    total_ms = max_over_ranks(sum(step_ms), world, local)
    ms_per_step = total_ms / args.steps
    value = embeddings * world / (ms_per_step / 1000.0)

    # dominant kernel and its roofline: DRAM bytes it moves per launch (committed ncu capture of this
    # workload) over its CUDA-event time, against the measured HBM copy bandwidth; the reference
    # schedule's algorithmic bytes over the same time are reported beside it (algo_gbs), since the
    # bitmap engine replaces list intersections by bit-matrix popcounts and never moves those bytes
    dom = max(range(4), key=lambda p: phase_ms[p])
    dom_ms = phase_ms[dom] / args.steps
    dom_bytes = st_stats.phase_bytes[dom]
    peak, peak_kind = peaks()
    algo_gbs = dom_bytes / (dom_ms / 1000.0) / 1e9 if dom_ms > 0 else 0.0
    traffic = None
    if (args.scale, args.edge_factor) == (SCALE, EDGE_FACTOR):
        traffic = profile_traffic(khz.Stats.PHASES[dom])
    dram_gbs = traffic / (dom_ms / 1000.0) / 1e9 if traffic and dom_ms > 0 else None
    counters = profile_counters(khz.Stats.PHASES[dom])

    # e2e: oriented .dgraph edge list in pinned host memory -> C ABI -> count -> host
    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "embeddings/s", "ms_per_step": ms_per_step,
                              "phase_ms_per_step": [x / args.steps for x in phase_ms],
                              "phase_algo_bytes": list(st_stats.phase_bytes), "count": ref_counts[0],
                              "scale": args.scale, "edge_factor": args.edge_factor}), flush=True)
        ctx.close()
        return
    off_h, adj_h = g.export_csr()
    src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off_h).astype(np.int64))
    pairs = torch.from_numpy(np.stack([src, adj_h], axis=1).reshape(-1).view(np.int32)).pin_memory()
    del src
    e2e_ms = []
    e2e_parts = [0.0, 0.0, 0.0]  # build (upload + validate + CSR), count (+ result copy), free
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = ctx.graph_from_edges(pairs, n, stream=sptr)
        ta = time.perf_counter()
        c2, st2 = ctx.count(g2, APP, stream=sptr)
        tb = time.perf_counter()
        g2.free()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        assert c2 == ref_counts
        if i >= args.warmup:
            e2e_ms.append((t1 - t0) * 1000.0)
            e2e_parts[0] += (ta - t0) * 1000.0 / args.steps
            e2e_parts[1] += (tb - ta) * 1000.0 / args.steps
            e2e_parts[2] += (t1 - tb) * 1000.0 / args.steps
    e2e_total = max_over_ranks(sum(e2e_ms), world, local)
    e2e_value = embeddings * world / (e2e_total / args.steps / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import numpy as np
        with tempfile.TemporaryDirectory() as td:
            path = labelled_oriented_dgraph(g, td)
            r = run_reference_sample(path, runs=1, warmup=1)
        # the same slice on the device (restrict_starting_vertex_label): the reference's count and
        # NumExtensions must be the device's
        g.set_labels((np.arange(n, dtype=np.uint64) % SAMPLE_MOD).astype(np.uint32))
        slice_counts, slice_st = ctx.count_restricted(g, APP, 0)
        assert slice_counts[0] == r["count"] and slice_st.num_extensions == r["num_extensions"], \
            (slice_counts, slice_st.num_extensions, r)
        model, cores, logical = host_cpu()
        cpu = {"value": r["embeddings"] / r["secs"], "unit": "embeddings/s", "cores": cores, "threads": r["threads"],
               "logical_cpus": logical, "cpu_model": model, "kind": r["kind"],
               "sample": "start vertices v0 %% %d == 0 of the same oriented graph (%d embeddings, %.1f s); "
                         "count %d and NumExtensions %d equal the device's restricted count of that slice"
                         % (SAMPLE_MOD, r["embeddings"], r["secs"], r["count"], r["num_extensions"])}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "embeddings/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32/u64 integer", "data": "synthetic (device R-MAT generator)",
            "config": {"workload": workload_name(args.scale, args.edge_factor), "vertices": n, "oriented_edges": m,
                       "undirected_edges": sym_info.num_entries // 2, "max_out_degree": gi.max_degree,
                       "count": ref_counts[0], "num_extensions": st_stats.num_extensions,
                       "embeddings_per_step": embeddings, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs (275 MB CSR) larger than L2; no flush"},
            "e2e": {"value": e2e_value, "unit": "embeddings/s", "h2d_bytes_per_step": int(pairs.numel() * 4),
                    "d2h_bytes_per_step": 8 * 8, "ms_per_step": e2e_total / args.steps,
                    "ms_build_count_free": e2e_parts},
            # the roofline is the HBM one (peak = measured copy bandwidth); what limits the kernel
            # below it is instruction issue (bitmap tiers) or latency (DFS engine)
            "roofline": {"bound": "hbm", "limiter": "issue" if dom < 3 else "latency", "achieved": dram_gbs,
                         "peak": peak,
                         "unit": "GB/s", "frac": dram_gbs / peak if dram_gbs is not None else None,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "basis": "DRAM bytes per launch (ncu, committed capture) / CUDA-event time",
                         "kernel": khz.Stats.PHASES[dom], "kernel_ms": dom_ms,
                         "algo_bytes_per_launch": dom_bytes, "algo_gbs": algo_gbs, "algo_frac": algo_gbs / peak,
                         "ncu_small_case": counters},
            "phase_ms_per_step": [x / args.steps for x in phase_ms],
            "phase_algo_bytes": list(st_stats.phase_bytes),
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


BATCH_APPS = ["kautomine_triangle", "kautomine_four_clique", "kgraphpi_four_cycle", "kautomine_three_motif"]


def batch_specs(n_graphs, seed=7):
    """The uneven batch: vertex counts log-uniform in [64, 200000], average degree uniform in
    [4, 40], one app each from BATCH_APPS.  A graph is R-MAT with scale = round(log2 n) and
    edge factor = round(degree / 2) (2 * edge factor is the pre-dedupe average degree)."""
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_graphs):
        n = math.exp(rng.uniform(math.log(64), math.log(200000)))
        deg = rng.uniform(4, 40)
        scale = max(6, int(round(math.log2(n))))
        ef = max(1, int(round(deg / 2)))
        specs.append((scale, ef, 1000003 * seed + i, BATCH_APPS[int(rng.integers(0, len(BATCH_APPS)))]))
    return specs


def batch_workload(args):
    """Plain (one khz_count per query, prepared launches cached) vs batched (all queries in one
    launch sequence captured in a CUDA graph) on the same uneven batch."""
    import torch
    from openkhuzdulgraph_b200 import khz
    torch.cuda.set_device(0)
    ctx = khz.Context(0)
    a, b, c = RMAT_ABC
    t0 = time.time()
    jobs, edges = [], 0
    for scale, ef, seed, app in batch_specs(args.graphs):
        g = ctx.generate_rmat(scale, ef, a, b, c, seed, orient=app in ("kautomine_triangle", "kautomine_four_clique"))
        edges += g.num_entries
        jobs.append((g, app))
    t_gen = time.time() - t0
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    steps = max(3, args.steps)
    # plain: one query at a time (first pass prepares and caches each launch, and builds the
    # per-graph views the engines use: one-time work, not a query's cost)
    ref, exts_ref, emb = [], [], 0
    for g, app in jobs:
        cnt, st = ctx.count(g, app, stream=sptr)
        ref.append(cnt)
        exts_ref.append(st.num_extensions)
        emb += st.num_extensions + sum(cnt)

    def plain_pass(sel):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for k in sel:
            g, app = jobs[k]
            cnt, _ = ctx.count(g, app, stream=sptr)
            assert cnt == ref[k]
        torch.cuda.synchronize()
        return (time.perf_counter() - t1) * 1000

    everything = list(range(len(jobs)))
    by_app = {app: [k for k, (_, a2) in enumerate(jobs) if a2 == app] for app in BATCH_APPS}
    batch = khz.Batch(ctx, jobs, cuda_graph=True, stream=sptr)
    batch.launch(sptr)
    counts, exts = batch.wait(sptr)
    assert counts == ref and exts == exts_ref

    def batch_pass(b):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        b.launch(sptr)
        cnts, _ = b.wait(sptr)
        ms = (time.perf_counter() - t1) * 1000
        return ms, cnts

    # served: every query of the batch submitted at once to the continuous-batching server
    sv = khz.Server(ctx, slots=args.slots, max_batch=args.max_batch)
    for k in range(0, len(jobs), 997):  # warm the scheduler's per-(graph, app) footprint cache
        sv.wait(sv.submit(*jobs[k]), jobs[k][1], timeout_ms=600000.0)

    def serve_pass():
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        tickets = [sv.submit(g, app) for g, app in jobs]
        for k, t in enumerate(tickets):
            cnt, ext, _ = sv.wait(t, jobs[k][1], timeout_ms=600000.0)
            assert cnt == ref[k] and ext == exts_ref[k]
        return (time.perf_counter() - t1) * 1000

    plain_ms, batch_ms, serve_ms = [], [], []
    with ClockSampler(0) as clk:
        for _ in range(steps):
            plain_ms.append(plain_pass(everything))
            ms, cnts = batch_pass(batch)
            assert cnts == ref
            batch_ms.append(ms)
            serve_ms.append(serve_pass())
    sv.close()
    batch.close()
    # per app: plain vs one batched launch sequence of that app's queries (median of `steps`)
    per_app = {}
    for app, sel in by_app.items():
        if not sel:
            continue
        b = khz.Batch(ctx, [jobs[k] for k in sel], cuda_graph=True, stream=sptr)
        b.launch(sptr)
        b.wait(sptr)
        pm = statistics.median(plain_pass(sel) for _ in range(steps))
        bm = statistics.median(batch_pass(b)[0] for _ in range(steps))
        b.close()
        per_app[app] = {"queries": len(sel), "ms_plain": pm, "ms_batched": bm, "batched_over_plain": pm / bm}
    p_ms, b_ms, s_ms = statistics.median(plain_ms), statistics.median(batch_ms), statistics.median(serve_ms)
    print(json.dumps({
        "metric": "embeddings/s (uneven batch of %d graphs)" % len(jobs), "unit": "embeddings/s",
        "value": emb / (b_ms / 1000), "plain_value": emb / (p_ms / 1000), "served_value": emb / (s_ms / 1000),
        "batched_over_plain": p_ms / b_ms, "served_over_plain": p_ms / s_ms,
        "ms_batched": b_ms, "ms_plain": p_ms, "ms_served": s_ms,
        "ms_steps": {"plain": plain_ms, "batched": batch_ms, "served": serve_ms}, "per_app": per_app,
        "embeddings": emb, "graphs": len(jobs), "csr_entries": edges, "generation_s": t_gen, "steps": steps,
        "slots": args.slots, "max_batch": args.max_batch, "clocks": clk.summary(), "higher_is_better": True,
        "data": "synthetic (device R-MAT)",
        "config": {"workload": "uneven batch: n log-uniform [64, 200000], degree U[4, 40], "
                               "apps %s" % BATCH_APPS,
                   "timing": "wall clock per pass (host calls included), median of %d" % steps}}), flush=True)
    ctx.close()


SERVE_APPS = ["kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique", "kgraphpi_four_cycle",
              "kgraphpi_house", "kautomine_four_motif"]


def serve_graph_specs(n_graphs=64, e_min=1e3, e_max=5e8):
    """R-MAT (scale, edge factor) whose raw edge count ef * 2^scale is log-spaced over [e_min, e_max]
    (the largest is scale 24, edge factor 32)."""
    import math
    specs = []
    for i in range(n_graphs):
        e = e_min * (e_max / e_min) ** (i / (n_graphs - 1))
        scale = min(24, max(6, int(round(math.log2(e / 16)))))
        ef = max(1, int(round(e / 2 ** scale)))
        specs.append((scale, ef, 5000 + i))
    return specs


def serve_workload(args):
    """Poisson arrivals of counting queries against 64 device-resident graphs; p50/p99 latency and
    throughput of the continuous-batching server, and its saturated throughput against plain
    one-query-at-a-time counting on the same query list."""
    import random
    import threading
    import torch
    from openkhuzdulgraph_b200 import khz
    torch.cuda.set_device(0)
    ctx = khz.Context(0)
    a, b, c = RMAT_ABC
    t0 = time.time()
    graphs = [ctx.generate_rmat(sc, ef, a, b, c, seed) for sc, ef, seed in serve_graph_specs()]
    sizes = [g.num_entries // 2 for g in graphs]
    t_gen = time.time() - t0
    # feasibility: per app, graphs in increasing size until one query alone exceeds the cap
    feasible, alone, first_excluded = [], {}, {}
    for app in SERVE_APPS:  # load every kernel once
        ctx.count(graphs[0], app)
    for app in SERVE_APPS:
        for gi, g in enumerate(graphs):
            ctx.count(g, app)  # one-time work (orientation, launch preparation) is not the query's cost
            t1 = time.perf_counter()
            cnt, st = ctx.count(g, app)
            dt = (time.perf_counter() - t1) * 1000
            alone[(gi, app)] = (cnt, st.num_extensions, dt)
            if dt > args.query_cap_ms:
                first_excluded[app] = {"graph": gi, "undirected_edges": int(sizes[gi]), "ms_alone": dt,
                                       "excluded_graphs": len(graphs) - gi}
                break
            feasible.append((gi, app))
    rng = random.Random(11)
    clk = ClockSampler(0)
    clk.__enter__()
    sv = khz.Server(ctx, slots=args.slots, max_batch=args.max_batch)
    # warm: every feasible query once through the server
    for gi, app in feasible:
        sv.wait(sv.submit(graphs[gi], app), app)
    # saturation: the same query list submitted at once vs plain sequential counting
    qs = [rng.choice(feasible) for _ in range(args.sat_queries)]
    sv.reset_stats()
    t1 = time.perf_counter()
    tk = [sv.submit(graphs[gi], app) for gi, app in qs]
    for (gi, app), t in zip(qs, tk):
        sv.wait(t, app, timeout_ms=600000.0)
    served_s = time.perf_counter() - t1
    capacity = len(qs) / served_s
    # Poisson arrivals at the given rates, or at fractions of the measured capacity; at most
    # --rate-queries queries per rate, so heavy mixes stay bounded in time
    rates = args.rates if args.rates else [round(f * capacity, 1) for f in (0.25, 0.5, 0.75, 0.9)]
    rates_out = []
    for rate in rates:
        sv.reset_stats()
        n_q = max(50, min(args.rate_queries, int(rate * args.duration)))
        qs_r = [rng.choice(feasible) for _ in range(n_q)]
        arrivals = []
        t = 0.0
        for _ in qs_r:
            t += rng.expovariate(rate)
            arrivals.append(t)
        tickets = [None] * n_q

        def submitter():
            start = time.perf_counter()
            for k, ((gi, app), ta) in enumerate(zip(qs_r, arrivals)):
                d = ta - (time.perf_counter() - start)
                if d > 0:
                    time.sleep(d)
                tickets[k] = sv.submit(graphs[gi], app)

        th = threading.Thread(target=submitter)
        ts = time.perf_counter()
        th.start()
        lat = []
        for k in range(n_q):
            while tickets[k] is None:
                time.sleep(0.0002)
            gi, app = qs_r[k]
            cnt, ext, l = sv.wait(tickets[k], app, timeout_ms=600000.0)
            assert cnt == alone[(gi, app)][0] and ext == alone[(gi, app)][1]
            lat.append(l)
        th.join()
        wall = time.perf_counter() - ts
        lat.sort()
        rates_out.append({"offered_qps": rate, "queries": n_q, "achieved_qps": n_q / wall,
                          "p50_ms": lat[len(lat) // 2], "p99_ms": lat[int(0.99 * (len(lat) - 1))],
                          "batches": sv.stats()["batches"]})
    sv.close()
    t1 = time.perf_counter()
    for gi, app in qs:
        ctx.count(graphs[gi], app)
    plain_s = time.perf_counter() - t1
    clk.__exit__(None, None, None)
    out = {"metric": "served queries/s and latency (continuous batching)", "unit": "queries/s",
           "clocks": clk.summary(), "excluded": first_excluded,
           "value": len(qs) / served_s, "plain_value": len(qs) / plain_s, "served_over_plain": plain_s / served_s,
           "rates": rates_out, "graphs": len(graphs), "undirected_edges_total": int(sum(sizes)),
           "largest_graph_edges": int(max(sizes)), "feasible_queries": len(feasible),
           "feasible_per_app": {app: sum(1 for _, a2 in feasible if a2 == app) for app in SERVE_APPS},
           "query_cap_ms": args.query_cap_ms, "slots": args.slots, "max_batch": args.max_batch,
           "generation_s": t_gen, "data": "synthetic (device R-MAT)", "higher_is_better": True,
           "config": {"workload": "serving: Poisson arrivals, 64 resident R-MAT graphs with 1e3..5e8 raw edges "
                                  "(log-spaced), apps %s; a (graph, app) pair is served when that query alone "
                                  "takes <= query_cap_ms" % SERVE_APPS}}
    print(json.dumps(out), flush=True)
    ctx.close()


CONFIG_RUNS = [
    # (label, scale, edge factor, oriented, apps): the triangle configuration is the ER graph
    ("K: R-MAT s22 ef16, degree-oriented", 22, 16, True, ["kautomine_four_clique", "kgraphpi_four_clique",
                                                       "kautomine_five_clique", "kgraphpi_five_clique"]),
    ("M: R-MAT s20 ef24, symmetric", 20, 24, False, ["kautomine_triangle", "kautomine_three_motif",
                                                    "kgraphpi_three_motif", "kgraphpi_four_cycle",
                                                    "kgraphpi_tailed_triangle", "kautomine_four_motif",
                                                    "kgraphpi_house"]),
]


def configs_workload(args):
    """Every app of the full-size configurations, device time per count (median of the steps), with
    the engine each app took."""
    import torch
    from openkhuzdulgraph_b200 import khz
    torch.cuda.set_device(0)
    ctx = khz.Context(0)
    a, b, c = RMAT_ABC
    steps = max(3, args.steps)
    out = []
    with ClockSampler(0) as clk:
        for label, scale, ef, oriented, apps in CONFIG_RUNS:
            sym = ctx.generate_rmat(scale, ef, a, b, c, SEED)
            g = sym.orient() if oriented else sym
            if oriented:
                sym.free()
            for app in apps:
                cnt, st = ctx.count(g, app)  # one-time work (views, prepared launch) first
                ms = []
                for _ in range(steps):
                    c2, st = ctx.count(g, app)
                    assert c2 == cnt
                    ms.append(st.kernel_ms)
                out.append({"config": label, "app": app, "counts": cnt, "num_extensions": st.num_extensions,
                            "ms": statistics.median(ms), "engine": ["auto", "dfs", "bitmap", "wedge"][st.engine],
                            "embeddings_per_s": (st.num_extensions + sum(cnt)) / (statistics.median(ms) / 1000)})
                print(json.dumps(out[-1]), flush=True)
            g.free()
    print(json.dumps({"metric": "device time per count, full-size configurations", "runs": out,
                      "clocks": clk.summary(), "steps": steps, "data": "synthetic (device R-MAT)"}), flush=True)
    ctx.close()


def app_workload(args):
    """One app on one R-MAT graph (symmetric; degree-oriented with --oriented) with one engine:
    device time per count (median of the steps).  The small-case driver for profiling one engine's
    kernels, e.g. the DFS engine on the 4-motif at scale 14."""
    import torch
    from openkhuzdulgraph_b200 import khz
    torch.cuda.set_device(0)
    ctx = khz.Context(0)
    engines = {"auto": khz.ENGINE_AUTO, "dfs": khz.ENGINE_DFS, "bitmap": khz.ENGINE_BITMAP,
               "wedge": khz.ENGINE_WEDGE}
    a, b, c = RMAT_ABC
    sym = ctx.generate_rmat(args.scale, args.edge_factor, a, b, c, SEED)
    g = sym.orient() if args.oriented else sym
    if args.oriented:
        sym.free()
    settings = {k: int(v) for k, v in (kv.split("=", 1) for kv in args.set)}
    ctx.set_config(engine=engines[args.engine], **settings)
    cnt, st = ctx.count(g, args.app)
    for _ in range(max(0, args.warmup - 1)):
        ctx.count(g, args.app)
    ms = []
    with ClockSampler(0) as clk:
        for _ in range(max(1, args.steps)):
            c2, st = ctx.count(g, args.app)
            assert c2 == cnt
            ms.append(st.kernel_ms)
    med = statistics.median(ms)
    print(json.dumps({"metric": "device time per count", "app": args.app, "counts": cnt,
                      "num_extensions": st.num_extensions, "ms": med, "ms_steps": ms,
                      "engine": ["auto", "dfs", "bitmap", "wedge"][st.engine],
                      "embeddings_per_s": (st.num_extensions + sum(cnt)) / (med / 1000), "clocks": clk.summary(),
                      "config": {"workload": "R-MAT scale %d edge factor %d%s" % (
                          args.scale, args.edge_factor, ", degree-oriented" if args.oriented else ""),
                          "engine": args.engine, "settings": settings}, "data": "synthetic (device R-MAT)"}),
          flush=True)
    g.free()
    ctx.close()


FSM_LEVELS = ["single-vertex", "single-edge", "wedge", "triangle", "four-chain", "three-star"]
FSM_LABELS, FSM_MULT = 5, 7919  # node label of v: (v * 7919) mod 5


def fsm_reference(scale, edge_factor, threshold):
    """The reference's own kautomine three_fsm (compiled unmodified into oracle/_ref) on the same
    labelled R-MAT graph: per level (frequent patterns, support sum) and its "Average runtime"."""
    import re
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    exe = os.path.join(orc.REF_DIR, "kautomine_three_fsm")
    if not os.path.exists(exe):
        return None
    canon, n = orc.rmat(scale, edge_factor, *RMAT_ABC, seed=SEED)
    labels = (np.arange(n, dtype=np.uint64) * FSM_MULT % FSM_LABELS).astype(np.uint32)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "fsm.dgraph")
        orc.write_dgraph(path, n, orc.symmetrize(canon), labels)
        out = subprocess.run([exe, path, str(threshold)], capture_output=True, text=True, timeout=3000)
    if out.returncode != 0:
        raise RuntimeError("reference three_fsm failed: " + out.stderr[-500:])
    lines = re.findall(r"Number of frequent ([a-z-]+) patterns: (\d+), support sum(?: of them)?: (\d+)", out.stdout)
    got = {k: (int(a), int(b)) for k, a, b in lines}
    ms = float(re.search(r"Average runtime: ([0-9.]+) \(ms\)", out.stdout).group(1))
    return {"levels": [got[k] for k in FSM_LEVELS], "ms": ms}


def fsm_workload(args):
    """3-FSM (kautomine/three_fsm.cc) on labelled R-MAT graphs (labels (v * 7919) mod 5, support
    threshold 300 per 8192 vertices): host wall time of the device mining run (median of the
    steps).  At scale 13 the reference's own three_fsm runs the same graph on the host cores: its
    per-level frequent patterns and support sums must be the device's."""
    import numpy as np
    import torch
    from openkhuzdulgraph_b200 import khz
    torch.cuda.set_device(0)
    ctx = khz.Context(0)
    runs = []
    with ClockSampler(0) as clk:
        for scale in args.fsm_scales:
            g = ctx.generate_rmat(scale, 16, *RMAT_ABC, SEED)
            n = g.num_vertices
            g.set_labels((np.arange(n, dtype=np.uint64) * FSM_MULT % FSM_LABELS).astype(np.uint32))
            thr = max(1, 300 * n // 8192)
            levels, pats, _ = ctx.fsm(g, thr)
            ms = []
            for _ in range(max(1, args.steps)):
                lv2, _, t = ctx.fsm(g, thr)
                assert lv2 == levels
                ms.append(t)
            runs.append({"graph": "R-MAT scale %d edge factor 16, %d vertices, %d labels" % (scale, n, FSM_LABELS),
                         "scale": scale,
                         "threshold": thr, "ms": statistics.median(ms), "ms_steps": ms,
                         "levels": [(lv["num_frequent"], lv["support_sum"]) for lv in levels],
                         "candidates": [lv["num_candidates"] for lv in levels]})
            print(json.dumps(runs[-1]), flush=True)
            g.free()
    ref = None
    if not args.no_cpu and 13 in args.fsm_scales:
        mine = runs[args.fsm_scales.index(13)]
        r = fsm_reference(13, 16, mine["threshold"])
        if r is not None:
            assert [tuple(x) for x in mine["levels"]] == r["levels"], (mine["levels"], r["levels"])
            model, cores, logical = host_cpu()
            ref = {"ms": r["ms"], "levels_equal": True, "threads": max(1, logical - 2), "cores": cores,
                   "cpu_model": model, "kind": "reference", "graph": "the scale-13 graph above",
                   "device_over_reference": r["ms"] / mine["ms"]}
    print(json.dumps({"metric": "3-FSM wall time per mining run", "runs": runs, "reference": ref,
                      "clocks": clk.summary(), "steps": args.steps, "data": "synthetic (device R-MAT)"}),
          flush=True)
    ctx.close()


def reference_arm(args, rank, world, local):
    """The reference's own CPU path only: the graph is built by the oracle generator and the
    reference's converters (reference_built_graph), and the reference's kautomine four_clique
    counts the label-0 slice of its start vertices; this repository's library is not loaded."""
    if rank != 0:
        return
    import numpy as np
    t0 = time.time()
    with tempfile.TemporaryDirectory() as td:
        path = reference_built_graph(args.scale, args.edge_factor, td)
        if path is None:  # no oracle/_ref: the oracle restatement of the same schedule
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import orc
            a, b, c = RMAT_ABC
            canon, n = orc.rmat(args.scale, args.edge_factor, a, b, c, seed=SEED)
            off, adj = orc.csr(orc.symmetrize(canon), n)
            ooff, oadj, _ = orc.orient(off, adj)
            src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(ooff).astype(np.int64))
            path = os.path.join(td, "k_oriented_labeled.dgraph")
            orc.write_dgraph(path, n, np.stack([src, oadj], axis=1),
                             (np.arange(n, dtype=np.uint64) % SAMPLE_MOD).astype(np.uint32))
        t_build = time.time() - t0
        r = run_reference_sample(path, runs=args.steps, warmup=args.warmup)
    value = r["embeddings"] / r["secs"]
    model, cores, logical = host_cpu()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "embeddings/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["secs"] * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64 integer", "data": "synthetic",
            "config": {"workload": workload_name(args.scale, args.edge_factor), "sample": "v0 %% %d == 0" % SAMPLE_MOD,
                       "same_config": False,
                       "graph_built_by": "oracle generator + reference converter + to_oriented_dataset_converter",
                       "graph_build_s": t_build},
            "cpu_baseline": {"value": value, "unit": "embeddings/s", "cores": cores, "threads": r["threads"],
                             "logical_cpus": logical, "cpu_model": model, "kind": r["kind"],
                             "sample": "start vertices v0 %% %d == 0 (%d embeddings per step; count %d, "
                                       "NumExtensions %d)" % (SAMPLE_MOD, r["embeddings"], r["count"],
                                                              r["num_extensions"])},
            "e2e": {"value": value, "unit": "embeddings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="device-resident steps only (profiling)")
    ap.add_argument("--workload", default="clique4",
                    choices=["clique4", "batch", "serve", "configs", "app", "fsm"],
                    help="clique4: the bench line; batch: the uneven multi-graph batch; serve: Poisson serving; "
                         "configs: every app of the full-size configurations; app: one app (--app, --engine); "
                         "fsm: 3-FSM on labelled R-MAT graphs (--fsm-scales)")
    ap.add_argument("--fsm-scales", type=int, nargs="+", default=[13, 16, 18])
    ap.add_argument("--app", default="kautomine_four_motif", help="app of the app workload")
    ap.add_argument("--engine", default="auto", choices=["auto", "dfs", "bitmap", "wedge"],
                    help="engine of the app workload")
    ap.add_argument("--oriented", action="store_true", help="app workload: degree-oriented graph")
    ap.add_argument("--set", nargs="*", default=[], metavar="KEY=VALUE",
                    help="app workload: khz_config fields, e.g. dfs_warps_per_sm=24")
    ap.add_argument("--rates", type=float, nargs="*", default=[],
                    help="serve: offered rates in queries/s (default: 0.25, 0.5, 0.75 and 0.9 of the measured capacity)")
    ap.add_argument("--rate-queries", type=int, default=400, help="serve: at most this many queries per rate")
    ap.add_argument("--duration", type=float, default=2.0, help="seconds of arrivals per rate (serve)")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--max-batch", type=int, default=64)
    ap.add_argument("--query-cap-ms", type=float, default=1000.0,
                    help="serve: a (graph, app) pair is served when that query alone takes at most this long")
    ap.add_argument("--sat-queries", type=int, default=500)
    ap.add_argument("--graphs", type=int, default=20000, help="graphs in the batch workload")
    ap.add_argument("--scale", type=int, default=SCALE, help="R-MAT scale (the bench workload is 22)")
    ap.add_argument("--edge-factor", type=int, default=EDGE_FACTOR, help="R-MAT edge factor (workload: 16)")
    args = ap.parse_args()
    if args.workload == "batch":
        batch_workload(args)
        return
    if args.workload == "serve":
        serve_workload(args)
        return
    if args.workload == "configs":
        configs_workload(args)
        return
    if args.workload == "app":
        app_workload(args)
        return
    if args.workload == "fsm":
        fsm_workload(args)
        return
    if args.impl == "reference":
        # the reference arm is a CPU run on rank 0; other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        reference_arm(args, rank, 1, int(os.environ.get("LOCAL_RANK", "0")))
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world, local)
        else:
            ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
