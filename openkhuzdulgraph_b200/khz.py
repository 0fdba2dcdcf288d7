"""Python view of libkhz_b200.so (the engine's C ABI, include/khz.h).

This is a thin ctypes binding for tests, the bench and Python callers; the engine and
its host logic are native.  There is no CPU fallback: if the library is missing the
import fails with an explicit error.

The names follow the reference's application API (AmadeusChan/OpenKhuzdulGraph):
apps are the kautomine / kgraphpi pattern programs, `count()` is the
`count->clear(); app->run(); count->evaluate()` sequence of their main()
(kautomine/triangle.cc:211-216), and graphs are the .dgraph CSR of graph_loader.h.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkhz_b200.so")

APPS = {
    "kautomine_triangle": 0, "kautomine_four_clique": 1, "kautomine_five_clique": 2,
    "kautomine_three_motif": 3, "kgraphpi_triangle": 4, "kgraphpi_four_clique": 5,
    "kgraphpi_five_clique": 6, "kgraphpi_three_motif": 7, "kgraphpi_four_cycle": 8,
    "kgraphpi_house": 9, "kgraphpi_tailed_triangle": 10, "kautomine_four_motif": 11,
}
APP_NAMES = {v: k for k, v in APPS.items()}
MAX_COUNTS = 6

EDGES_ON_DEVICE = 0x1
ORIENT = 0x2
UNCHECKED = 0x4
SKIP_LABELS = 0x8

ENGINE_AUTO, ENGINE_DFS, ENGINE_BITMAP, ENGINE_WEDGE = 0, 1, 2, 3

SETOP = {"intersect": 0, "subtract": 1, "intersect_count": 2, "bounded_intersect": 3,
         "bounded_subtract": 4, "trim": 5, "trim_lower_bound": 6}

STATUS = {0: "KHZ_OK", 1: "KHZ_ERR_ARG", 2: "KHZ_ERR_OOM", 3: "KHZ_ERR_OVERFLOW", 4: "KHZ_ERR_TIMEOUT",
          5: "KHZ_ERR_CUDA", 6: "KHZ_ERR_FORMAT", 7: "KHZ_ERR_BUSY", 8: "KHZ_ERR_NOT_FOUND",
          9: "KHZ_ERR_MULTIPLICITY", 10: "KHZ_ERR_CANCELLED"}

# every entry point include/khz.h declares
EXPORTS = ["khz_ctx_create", "khz_ctx_destroy", "khz_ctx_set_config", "khz_ctx_get_config",
           "khz_last_error_string", "khz_abi_version", "khz_graph_from_edges", "khz_graph_load_dgraph",
           "khz_graph_orient", "khz_graph_generate_rmat", "khz_graph_info_get", "khz_graph_export_csr",
           "khz_graph_write_dgraph", "khz_graph_set_labels", "khz_graph_free", "khz_count", "khz_count_async",
           "khz_count_restricted", "khz_app_num_counts",
           "khz_app_multiplicity", "khz_count_batch", "khz_set_op_batch", "khz_count_noalloc",
           "khz_batch_create", "khz_batch_launch", "khz_batch_wait", "khz_batch_destroy",
           "khz_server_create", "khz_server_submit", "khz_server_wait", "khz_server_stats_get",
           "khz_server_reset_stats", "khz_server_cancel", "khz_server_destroy", "khz_autotune",
           "khz_app_register", "khz_fsm"]


class KhzError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class GraphInfo(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_uint32), ("max_degree", ctypes.c_uint32),
                ("num_entries", ctypes.c_uint64), ("oriented", ctypes.c_int32), ("symmetric", ctypes.c_int32),
                ("d_offsets", ctypes.c_void_p), ("d_adj", ctypes.c_void_p), ("device_bytes", ctypes.c_uint64),
                ("num_labels", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("d_labels", ctypes.c_void_p)]


class Stats(ctypes.Structure):
    _fields_ = [("num_extensions", ctypes.c_uint64), ("algo_bytes", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("engine", ctypes.c_uint32), ("launches", ctypes.c_uint32),
                ("phase_ms", ctypes.c_double * 4), ("phase_bytes", ctypes.c_uint64 * 4),
                ("phase_launches", ctypes.c_uint32 * 4)]

    PHASES = ["bitmap_warp_tier", "bitmap_mid_block_tier", "bitmap_large_block_tier", "dfs"]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_[:5]}
        d["phase_ms"] = list(self.phase_ms)
        d["phase_bytes"] = list(self.phase_bytes)
        d["phase_launches"] = list(self.phase_launches)
        return d


class Config(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int32), ("want_algo_bytes", ctypes.c_int32),
                ("dfs_warps_per_sm", ctypes.c_int32), ("dfs_chunk", ctypes.c_int32),
                ("bitmap_warp_max", ctypes.c_int32), ("bitmap_block_warps", ctypes.c_int32),
                ("bitmap_hub_rows", ctypes.c_int32), ("device_mem_limit_mib", ctypes.c_int32),
                ("bitmap_tensor_cores", ctypes.c_int32), ("reserved", ctypes.c_int32 * 7)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("pending", ctypes.c_uint64),
                ("max_bytes_in_flight", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("queries_per_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneReport(ctypes.Structure):
    _fields_ = [("trials", ctypes.c_int32), ("reserved", ctypes.c_int32), ("baseline_ms", ctypes.c_double),
                ("best_ms", ctypes.c_double), ("best", Config)]


class Job(ctypes.Structure):
    _fields_ = [("graph", ctypes.c_uint32), ("app", ctypes.c_int32), ("reserved", ctypes.c_int32)]


# ---- schedules an app brings itself (khz_app_register; the apply() levels as data) -------------
class SetExpr(ctypes.Structure):
    _fields_ = [("base_kind", ctypes.c_int8), ("base_arg", ctypes.c_int8), ("op", ctypes.c_int8 * 2),
                ("op_arg", ctypes.c_int8 * 2)]


class Term(ctypes.Structure):
    _fields_ = [("set", SetExpr), ("gt_mask", ctypes.c_uint8), ("ne_mask", ctypes.c_uint8),
                ("guard_lo", ctypes.c_int8), ("guard_hi", ctypes.c_int8), ("counter", ctypes.c_int8),
                ("reserved", ctypes.c_int8 * 3)]


class Level(ctypes.Structure):
    _fields_ = [("term", Term), ("has_cached", ctypes.c_int8), ("finalized", ctypes.c_int8),
                ("reserved", ctypes.c_int8 * 2), ("cached", SetExpr)]


class PatternSchedule(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int8), ("num_terms", ctypes.c_int8), ("reserved", ctypes.c_int8 * 2),
                ("levels", Level * 5), ("last", Term * 2)]


class AppDesc(ctypes.Structure):
    _fields_ = [("num_runs", ctypes.c_int32), ("num_counts", ctypes.c_int32),
                ("multiplicity", ctypes.c_uint32 * 6), ("runs", PatternSchedule * 6)]


class FsmLevel(ctypes.Structure):
    _fields_ = [("num_candidates", ctypes.c_uint32), ("num_frequent", ctypes.c_uint32),
                ("support_sum", ctypes.c_uint64)]


class FsmResult(ctypes.Structure):
    _fields_ = [("level", FsmLevel * 6), ("ms", ctypes.c_double)]


class FsmPattern(ctypes.Structure):
    _fields_ = [("level", ctypes.c_uint32), ("size", ctypes.c_uint32), ("labels", ctypes.c_uint32 * 4),
                ("support", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


FSM_LEVELS = ["single-vertex", "single-edge", "wedge", "triangle", "four-chain", "three-star"]

BASE_NBR, BASE_SET = 0, 1
OP_NONE, OP_AND, OP_SUB = 0, 1, 2


def N(i):
    """N(v_i): the neighbour list of matched vertex i."""
    return (BASE_NBR, i, [])


def S(s):
    """A set materialised earlier: 2 or 3 = level 2 / 3's set, 4 = the cached set."""
    return (BASE_SET, s, [])


def AND(e, b):
    """e.intersect_with(N(v_b))"""
    return (e[0], e[1], e[2] + [(OP_AND, b)])


def SUB(e, b):
    """e.subtracted_by(N(v_b))"""
    return (e[0], e[1], e[2] + [(OP_SUB, b)])


def _mask(vs):
    m = 0
    for v in vs:
        m |= 1 << v
    return m


def _set_expr(dst, e):
    dst.base_kind, dst.base_arg = e[0], e[1]
    if len(e[2]) > 2:
        raise ValueError("at most two operations per set")
    for k, (o, b) in enumerate(e[2]):
        dst.op[k], dst.op_arg[k] = o, b


def _term(dst, t):
    e, gt, ne, counter, guard = t
    _set_expr(dst.set, e)
    dst.gt_mask, dst.ne_mask, dst.counter = _mask(gt), _mask(ne), counter
    dst.guard_lo, dst.guard_hi = guard if guard else (-1, -1)


def term(e, gt=(), ne=(), counter=0, guard=None):
    """A level's candidate set with its filters: keep x > v_a (a in gt) and x != v_a (a in ne);
    at the last level, adds to `counter`, only when v[guard[0]] < v[guard[1]] if a guard is given."""
    return (e, tuple(gt), tuple(ne), counter, guard)


def level(t, cached=None, finalized=False):
    return (t, cached, finalized)


def schedule(k, levels, last):
    """k: pattern size; levels: the enumerating levels 1 .. k-2; last: 1 or 2 counting terms."""
    return (k, list(levels), list(last))


def register_app(runs, multiplicities):
    """Registers an app made of `runs` (schedules run one after another) -> its app id."""
    d = AppDesc()
    d.num_runs, d.num_counts = len(runs), len(multiplicities)
    for c, m in enumerate(multiplicities):
        d.multiplicity[c] = m
    for r, (k, levels, last) in enumerate(runs):
        ps = d.runs[r]
        ps.k, ps.num_terms = k, len(last)
        for li, (t, cached, fin) in enumerate(levels, start=1):
            _term(ps.levels[li].term, t)
            ps.levels[li].finalized = 1 if fin else 0
            if cached is not None:
                ps.levels[li].has_cached = 1
                _set_expr(ps.levels[li].cached, cached)
        for ti, t in enumerate(last):
            _term(ps.last[ti], t)
    app = ctypes.c_int32(0)
    _check(lib().khz_app_register(ctypes.byref(d), ctypes.byref(app)))
    return app.value


_lib = None


def lib():
    """Load the engine.  Raises if the native library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libkhz_b200.so not found at %s; build it with "
                              "`python -m openkhuzdulgraph_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        P, u32, u64, i32, vp = ctypes.POINTER, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p
        sigs = {
            "khz_ctx_create": (i32, [i32, P(vp)]),
            "khz_ctx_destroy": (i32, [vp]),
            "khz_ctx_set_config": (i32, [vp, P(Config)]),
            "khz_ctx_get_config": (i32, [vp, P(Config)]),
            "khz_last_error_string": (ctypes.c_char_p, []),
            "khz_abi_version": (i32, []),
            "khz_graph_from_edges": (i32, [vp, vp, u64, u32, u32, P(u32), vp]),
            "khz_graph_load_dgraph": (i32, [vp, ctypes.c_char_p, u32, P(u32)]),
            "khz_graph_orient": (i32, [vp, u32, P(u32), vp]),
            "khz_graph_generate_rmat": (i32, [vp, i32, i32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              u64, u32, P(u32), vp]),
            "khz_graph_info_get": (i32, [vp, u32, P(GraphInfo)]),
            "khz_graph_export_csr": (i32, [vp, u32, vp, vp]),
            "khz_graph_write_dgraph": (i32, [vp, u32, ctypes.c_char_p, vp]),
            "khz_graph_set_labels": (i32, [vp, u32, vp, u32]),
            "khz_graph_free": (i32, [vp, u32]),
            "khz_count": (i32, [vp, u32, i32, P(u64), P(Stats), vp]),
            "khz_count_async": (i32, [vp, u32, i32, vp, vp]),
            "khz_count_restricted": (i32, [vp, u32, i32, u32, P(u64), P(Stats), vp]),
            "khz_app_num_counts": (i32, [i32]),
            "khz_app_multiplicity": (i32, [i32, i32]),
            "khz_count_batch": (i32, [vp, P(Job), i32, P(u64), P(u64), P(Stats), vp]),
            "khz_set_op_batch": (i32, [i32, vp, vp, vp, vp, vp, vp, vp, u32, vp]),
            "khz_count_noalloc": (i32, [vp, vp, u32, u64, i32, vp, vp]),
            "khz_batch_create": (i32, [vp, P(Job), i32, u32, P(vp), vp]),
            "khz_batch_launch": (i32, [vp, vp]),
            "khz_batch_wait": (i32, [vp, P(u64), P(u64), vp]),
            "khz_batch_destroy": (i32, [vp]),
            "khz_server_create": (i32, [vp, i32, i32, u64, P(vp)]),
            "khz_server_submit": (i32, [vp, u32, i32, P(u64)]),
            "khz_server_wait": (i32, [vp, u64, P(u64), P(u64), P(ctypes.c_double), ctypes.c_double]),
            "khz_server_stats_get": (i32, [vp, P(ServerStats)]),
            "khz_server_reset_stats": (i32, [vp]),
            "khz_server_cancel": (i32, [vp, u64]),
            "khz_server_destroy": (i32, [vp]),
            "khz_autotune": (i32, [vp, P(Job), i32, i32, P(TuneReport)]),
            "khz_app_register": (i32, [P(AppDesc), P(ctypes.c_int32)]),
            "khz_fsm": (i32, [vp, u32, u32, P(FsmResult), P(FsmPattern), u32, P(u32)]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise KhzError(status, lib().khz_last_error_string().decode(errors="replace"))


def _app_id(app):
    return APPS[app] if isinstance(app, str) else int(app)


def num_counts(app):
    return lib().khz_app_num_counts(_app_id(app))


class Graph:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.handle = handle

    def info(self):
        gi = GraphInfo()
        _check(lib().khz_graph_info_get(self.ctx.ptr, self.handle, ctypes.byref(gi)))
        return gi

    @property
    def num_vertices(self):
        return self.info().num_vertices

    @property
    def num_entries(self):
        return self.info().num_entries

    def export_csr(self):
        gi = self.info()
        off = np.empty(gi.num_vertices + 1, dtype=np.uint64)
        adj = np.empty(max(gi.num_entries, 1), dtype=np.uint32)
        _check(lib().khz_graph_export_csr(self.ctx.ptr, self.handle, off.ctypes.data, adj.ctypes.data))
        return off, adj[: gi.num_entries]

    def orient(self, stream=None):
        h = ctypes.c_uint32(0)
        _check(lib().khz_graph_orient(self.ctx.ptr, self.handle, ctypes.byref(h), stream))
        return Graph(self.ctx, h.value)

    def set_labels(self, labels):
        """Node labels (one uint32 per vertex, dense in [0, num_labels))."""
        labels = np.ascontiguousarray(labels, dtype=np.uint32)
        _check(lib().khz_graph_set_labels(self.ctx.ptr, self.handle, labels.ctypes.data, labels.shape[0]))

    def write_dgraph(self, path, labels=None):
        lab = None
        if labels is not None:
            labels = np.ascontiguousarray(labels, dtype=np.uint32)
            lab = labels.ctypes.data
        _check(lib().khz_graph_write_dgraph(self.ctx.ptr, self.handle, path.encode(), lab))

    def free(self):
        if self.handle:
            _check(lib().khz_graph_free(self.ctx.ptr, self.handle))
            self.handle = 0


class Context:
    """One engine context on one device: owns the graphs and all device scratch
    (the reference's DistributedApplication + engines, distributed_application.h:12-60)."""

    def __init__(self, device=0):
        p = ctypes.c_void_p()
        _check(lib().khz_ctx_create(device, ctypes.byref(p)))
        self.ptr = p

    def close(self):
        if self.ptr:
            lib().khz_ctx_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def config(self):
        c = Config()
        _check(lib().khz_ctx_get_config(self.ptr, ctypes.byref(c)))
        return c

    def set_config(self, **kw):
        c = self.config()
        for k, v in kw.items():
            setattr(c, k, v)
        _check(lib().khz_ctx_set_config(self.ptr, ctypes.byref(c)))

    def graph_from_edges(self, pairs, n, orient=False, validate=True, stream=None):
        """pairs: (m, 2) uint32 numpy array on the host, or a CUDA tensor (device pointer)."""
        flags = (ORIENT if orient else 0) | (0 if validate else UNCHECKED)
        if hasattr(pairs, "data_ptr"):  # torch tensor
            assert pairs.dtype.itemsize == 4 and pairs.is_contiguous()
            ptr, m = pairs.data_ptr(), pairs.numel() // 2
            if pairs.is_cuda:
                flags |= EDGES_ON_DEVICE
        else:
            pairs = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
            ptr, m = pairs.ctypes.data, pairs.shape[0]
        h = ctypes.c_uint32(0)
        _check(lib().khz_graph_from_edges(self.ptr, ptr, m, n, flags, ctypes.byref(h), stream))
        return Graph(self, h.value)

    def load_dgraph(self, path, orient=False, labels=True):
        """labels=False: ignore the file's node labels (load_vertex_labels = false)."""
        h = ctypes.c_uint32(0)
        flags = (ORIENT if orient else 0) | (0 if labels else SKIP_LABELS)
        _check(lib().khz_graph_load_dgraph(self.ptr, path.encode(), flags, ctypes.byref(h)))
        return Graph(self, h.value)

    def generate_rmat(self, scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=1, orient=False, stream=None):
        h = ctypes.c_uint32(0)
        _check(lib().khz_graph_generate_rmat(self.ptr, scale, edge_factor, a, b, c, seed,
                                             ORIENT if orient else 0, ctypes.byref(h), stream))
        return Graph(self, h.value)

    def count(self, graph, app, stream=None):
        """-> (counts list, Stats)"""
        aid = _app_id(app)
        counts = (ctypes.c_uint64 * MAX_COUNTS)()
        st = Stats()
        _check(lib().khz_count(self.ptr, graph.handle, aid, counts, ctypes.byref(st), stream))
        return [int(counts[i]) for i in range(num_counts(aid))], st

    def count_restricted(self, graph, app, label, stream=None):
        """run(..., restrict_starting_vertex_label=True, label): (raw counts list, Stats) over the
        start vertices whose label is `label`; counts are not divided by the multiplicities."""
        aid = _app_id(app)
        counts = (ctypes.c_uint64 * MAX_COUNTS)()
        st = Stats()
        _check(lib().khz_count_restricted(self.ptr, graph.handle, aid, label, counts, ctypes.byref(st), stream))
        return [int(counts[i]) for i in range(num_counts(aid))], st

    def fsm(self, graph, threshold, capacity=4096):
        """3-FSM (kautomine/three_fsm.cc) -> (per level {num_candidates, num_frequent, support_sum},
        list of frequent patterns (level, labels, support), ms)"""
        res = FsmResult()
        pats = (FsmPattern * max(capacity, 1))()
        num = ctypes.c_uint32(0)
        _check(lib().khz_fsm(self.ptr, graph.handle, threshold, ctypes.byref(res), pats, capacity,
                             ctypes.byref(num)))
        levels = [{"num_candidates": lv.num_candidates, "num_frequent": lv.num_frequent,
                   "support_sum": lv.support_sum} for lv in res.level]
        found = [(p.level, list(p.labels)[:p.size], p.support) for p in pats[:min(num.value, capacity)]]
        return levels, found, res.ms

    def count_async(self, graph, app, d_out_ptr, stream=None):
        _check(lib().khz_count_async(self.ptr, graph.handle, _app_id(app), d_out_ptr, stream))

    def autotune(self, jobs, reps=2):
        """jobs: list of (Graph, app); installs the fastest settings -> report dict"""
        arr = (Job * len(jobs))()
        for i, (g, app) in enumerate(jobs):
            arr[i].graph = g.handle
            arr[i].app = _app_id(app)
        rep = TuneReport()
        _check(lib().khz_autotune(self.ptr, arr, len(jobs), reps, ctypes.byref(rep)))
        b = rep.best
        return {"trials": rep.trials, "baseline_ms": rep.baseline_ms, "best_ms": rep.best_ms,
                "engine": b.engine, "dfs_warps_per_sm": b.dfs_warps_per_sm, "dfs_chunk": b.dfs_chunk,
                "bitmap_warp_max": b.bitmap_warp_max, "bitmap_hub_rows": b.bitmap_hub_rows}

    def count_batch(self, jobs, stream=None):
        """jobs: list of (Graph, app) -> (list of count lists, list of NumExtensions, Stats)"""
        arr = (Job * len(jobs))()
        for i, (g, app) in enumerate(jobs):
            arr[i].graph = g.handle
            arr[i].app = _app_id(app)
        counts = (ctypes.c_uint64 * (MAX_COUNTS * len(jobs)))()
        ext = (ctypes.c_uint64 * len(jobs))()
        st = Stats()
        _check(lib().khz_count_batch(self.ptr, arr, len(jobs), counts, ext, ctypes.byref(st), stream))
        out = []
        for i, (_, app) in enumerate(jobs):
            nc = num_counts(app)
            out.append([int(counts[i * MAX_COUNTS + c]) for c in range(nc)])
        return out, [int(x) for x in ext], st


class Batch:
    """A prepared batch of (graph, app) jobs: one launch sequence for all of them, optionally
    captured into a CUDA graph (cuda_graph=True) and replayed by launch()."""

    def __init__(self, ctx, jobs, cuda_graph=False, stream=None):
        self.jobs = list(jobs)
        arr = (Job * len(self.jobs))()
        for i, (g, app) in enumerate(self.jobs):
            arr[i].graph = g.handle
            arr[i].app = _app_id(app)
        p = ctypes.c_void_p()
        _check(lib().khz_batch_create(ctx.ptr, arr, len(self.jobs), 1 if cuda_graph else 0, ctypes.byref(p), stream))
        self.ptr = p

    def launch(self, stream=None):
        _check(lib().khz_batch_launch(self.ptr, stream))

    def wait(self, stream=None):
        n = len(self.jobs)
        counts = (ctypes.c_uint64 * (MAX_COUNTS * n))()
        ext = (ctypes.c_uint64 * n)()
        _check(lib().khz_batch_wait(self.ptr, counts, ext, stream))
        return ([[int(counts[i * MAX_COUNTS + c]) for c in range(num_counts(app))]
                 for i, (_, app) in enumerate(self.jobs)], [int(x) for x in ext])

    def close(self):
        if self.ptr:
            lib().khz_batch_destroy(self.ptr)
            self.ptr = None


class Server:
    """Continuous-batching counting server on device-resident graphs (native scheduler thread)."""

    def __init__(self, ctx, slots=4, max_batch=64, hbm_budget=0):
        p = ctypes.c_void_p()
        _check(lib().khz_server_create(ctx.ptr, slots, max_batch, hbm_budget, ctypes.byref(p)))
        self.ptr = p

    def submit(self, graph, app):
        t = ctypes.c_uint64(0)
        _check(lib().khz_server_submit(self.ptr, graph.handle, _app_id(app), ctypes.byref(t)))
        return t.value

    def wait(self, ticket, app, timeout_ms=60000.0):
        """-> (counts, NumExtensions, latency ms)"""
        counts = (ctypes.c_uint64 * MAX_COUNTS)()
        ext = ctypes.c_uint64(0)
        lat = ctypes.c_double(0)
        _check(lib().khz_server_wait(self.ptr, ticket, counts, ctypes.byref(ext), ctypes.byref(lat), timeout_ms))
        return [int(counts[i]) for i in range(num_counts(app))], ext.value, lat.value

    def stats(self):
        st = ServerStats()
        _check(lib().khz_server_stats_get(self.ptr, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        _check(lib().khz_server_reset_stats(self.ptr))

    def cancel(self, ticket):
        """Withdraws a query not yet admitted -> True; False if it already runs or has finished."""
        rc = lib().khz_server_cancel(self.ptr, ticket)
        if rc == 7:  # KHZ_ERR_BUSY
            return False
        _check(rc)
        return True

    def close(self):
        if self.ptr:
            lib().khz_server_destroy(self.ptr)
            self.ptr = None


def count_noalloc(d_offsets, d_adj, n, num_entries, app, d_out, stream=None):
    """Count through the entry point that allocates no device memory (for callers whose
    device memory is owned by a pool they may not bypass).  All pointers are device pointers
    (ints); d_out receives 8 uint64.  Degree limit 1024; overlapping calls race."""
    _check(lib().khz_count_noalloc(d_offsets, d_adj, n, num_entries, _app_id(app), d_out, stream))


def set_op_batch(op, a_off, a, b_off=None, b=None, bound=None, out=None, out_len=None, stream=None):
    """VertexSet ops over device tensors (torch CUDA tensors: a_off/b_off int64, the rest int32)."""
    def ptr(t):
        return None if t is None else t.data_ptr()
    n_pairs = a_off.numel() - 1
    _check(lib().khz_set_op_batch(SETOP[op] if isinstance(op, str) else op, ptr(a_off), ptr(a), ptr(b_off), ptr(b),
                                  ptr(bound), ptr(out), ptr(out_len), n_pairs, stream))
