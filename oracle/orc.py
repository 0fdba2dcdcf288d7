"""ctypes view of the CPU oracle (liborc.so) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module.  It wraps the plain-C restatement in khz_oracle.c (see that file for the
reference file:line each routine follows) and drives the reference's own apps
compiled under oracle/_ref.
"""
import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")

APPS = {
    "kautomine_triangle": 0, "kautomine_four_clique": 1, "kautomine_five_clique": 2,
    "kautomine_three_motif": 3, "kgraphpi_triangle": 4, "kgraphpi_four_clique": 5,
    "kgraphpi_five_clique": 6, "kgraphpi_three_motif": 7, "kgraphpi_four_cycle": 8,
    "kgraphpi_house": 9, "kgraphpi_tailed_triangle": 10, "kautomine_four_motif": 11,
}
# apps the reference ships (and oracle/_ref builds)
REF_APPS = [a for a in APPS if APPS[a] < 8]

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_lib = None


def build():
    """Compile liborc.so (and, when the reference tree is present, oracle/_ref)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liborc.so"])
    ref = reference_tree()
    if ref:
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", "REF=" + ref])


def reference_tree():
    """The reference source tree the recipe compiles oracle/_ref from: $KHZ_REF, else the
    default checkout location named in oracle/Makefile; None when absent (as on a machine
    that only runs the prebuilt files)."""
    path = os.environ.get("KHZ_REF")
    if not path:
        with open(os.path.join(HERE, "Makefile")) as f:
            for line in f:
                if line.startswith("KHZ_REF ?="):
                    path = line.split("?=", 1)[1].strip()
    return path if path and os.path.isdir(path) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_mix64.restype = ctypes.c_uint64
        L.orc_mix64.argtypes = [ctypes.c_uint64]
        L.orc_rmat.restype = ctypes.c_uint64
        L.orc_rmat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_uint64, _u32p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]
        L.orc_er.restype = ctypes.c_uint64
        L.orc_er.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u32p,
                             ctypes.POINTER(ctypes.c_uint32)]
        L.orc_symmetrize.restype = None
        L.orc_symmetrize.argtypes = [_u32p, ctypes.c_uint64, _u32p]
        L.orc_csr_from_edges.restype = ctypes.c_int
        L.orc_csr_from_edges.argtypes = [_u32p, ctypes.c_uint64, ctypes.c_uint32, _u64p, _u32p]
        L.orc_orient.restype = ctypes.c_int
        L.orc_orient.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u64p, _u32p, _u32p]
        for name in ("orc_intersect", "orc_subtract"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint32
            f.argtypes = [_u32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p]
        L.orc_intersect_count.restype = ctypes.c_uint32
        L.orc_intersect_count.argtypes = [_u32p, ctypes.c_uint32, _u32p, ctypes.c_uint32]
        for name in ("orc_bounded_intersect", "orc_bounded_subtract"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint32
            f.argtypes = [_u32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        for name in ("orc_trim", "orc_trim_lower_bound"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint32
            f.argtypes = [_u32p, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_num_counts.restype = ctypes.c_int
        L.orc_num_counts.argtypes = [ctypes.c_int]
        L.orc_count.restype = ctypes.c_int
        L.orc_count.argtypes = [ctypes.c_int, ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32, ctypes.c_uint32,
                                ctypes.c_int, _u64p, ctypes.POINTER(ctypes.c_uint64),
                                ctypes.POINTER(ctypes.c_uint64)]
        L.orc_count_labeled.restype = ctypes.c_int
        L.orc_count_labeled.argtypes = [ctypes.c_int, ctypes.c_uint32, _u64p, _u32p, _u32p, ctypes.c_uint32,
                                        ctypes.c_int, _u64p, ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_uint64)]
        L.orc_brute.restype = ctypes.c_uint64
        L.orc_brute.argtypes = [ctypes.c_int, ctypes.c_uint32, _u64p, _u32p]
        L.orc_fsm.restype = ctypes.c_int
        L.orc_fsm.argtypes = [ctypes.c_uint32, _u64p, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32,
                              ctypes.c_int, _u32p, _u32p, _u64p]
        _lib = L
    return _lib


def mix64(x):
    return lib().orc_mix64(x)


def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=1):
    """Sorted canonical unique pairs (m, 2) uint32 and the compacted vertex count."""
    cap = edge_factor << scale
    out = np.empty(2 * cap, dtype=np.uint32)
    n = ctypes.c_uint32(0)
    m = lib().orc_rmat(scale, edge_factor, a, b, c, seed, out, cap, ctypes.byref(n))
    return out[: 2 * m].reshape(-1, 2).copy(), n.value


def er(n, m, seed=1):
    out = np.empty(2 * m, dtype=np.uint32)
    nn = ctypes.c_uint32(0)
    lib().orc_er(n, m, seed, out, ctypes.byref(nn))
    return out.reshape(-1, 2), nn.value


def symmetrize(canon):
    canon = np.ascontiguousarray(canon, dtype=np.uint32)
    out = np.empty(4 * canon.shape[0], dtype=np.uint32)
    lib().orc_symmetrize(canon.reshape(-1), canon.shape[0], out)
    return out.reshape(-1, 2)


def csr(pairs, n):
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    m = pairs.shape[0]
    off = np.empty(n + 1, dtype=np.uint64)
    adj = np.empty(max(m, 1), dtype=np.uint32)
    rc = lib().orc_csr_from_edges(pairs.reshape(-1), m, n, off, adj)
    if rc != 0:
        raise ValueError("edge list is not sorted/unique or out of range (code %d)" % rc)
    return off, adj[:m]


def orient(off, adj):
    n = off.shape[0] - 1
    ooff = np.empty(n + 1, dtype=np.uint64)
    oadj = np.empty(max(adj.shape[0] // 2, 1), dtype=np.uint32)
    rank = np.empty(max(n, 1), dtype=np.uint32)
    lib().orc_orient(n, off, np.ascontiguousarray(adj, dtype=np.uint32), ooff, oadj, rank)
    return ooff, oadj[: int(ooff[-1])], rank[:n]


def count(app, off, adj, v0_mod=1, v0_rem=0, threads=0):
    """(counts list, num_extensions, algorithmic bytes) of the restated reference schedule."""
    aid = APPS[app] if isinstance(app, str) else int(app)
    nc = lib().orc_num_counts(aid)
    counts = np.zeros(6, dtype=np.uint64)
    ne = ctypes.c_uint64(0)
    nb = ctypes.c_uint64(0)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    if adj.shape[0] == 0:
        adj = np.zeros(1, dtype=np.uint32)
    rc = lib().orc_count(aid, off.shape[0] - 1, off, adj, v0_mod, v0_rem, threads, counts,
                         ctypes.byref(ne), ctypes.byref(nb))
    if rc != 0:
        raise RuntimeError("orc_count failed (%d)" % rc)
    return [int(x) for x in counts[:nc]], ne.value, nb.value


def count_labeled(app, off, adj, labels, label, threads=0):
    """(raw counts, num_extensions, algorithmic bytes) of the run restricted to the start vertices
    whose label is `label`; counts are not divided by the multiplicities."""
    aid = APPS[app] if isinstance(app, str) else int(app)
    nc = lib().orc_num_counts(aid)
    counts = np.zeros(6, dtype=np.uint64)
    ne = ctypes.c_uint64(0)
    nb = ctypes.c_uint64(0)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    if adj.shape[0] == 0:
        adj = np.zeros(1, dtype=np.uint32)
    labels = np.ascontiguousarray(labels, dtype=np.uint32)
    rc = lib().orc_count_labeled(aid, off.shape[0] - 1, off, adj, labels, label, threads, counts,
                                 ctypes.byref(ne), ctypes.byref(nb))
    if rc != 0:
        raise RuntimeError("orc_count_labeled failed (%d)" % rc)
    return [int(x) for x in counts[:nc]], ne.value, nb.value


def brute(pattern, off, adj):
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    if adj.shape[0] == 0:
        adj = np.zeros(1, dtype=np.uint32)
    return int(lib().orc_brute(pattern, off.shape[0] - 1, off, adj))


def write_dgraph(path, n, pairs, labels=None):
    """.dgraph writer (graph_loader.h:31-42): 20-byte packed header, labels, packed pairs."""
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    hdr = np.zeros(20, dtype=np.uint8)
    hdr[0:4] = np.frombuffer(np.uint32(n).tobytes(), dtype=np.uint8)
    hdr[4:12] = np.frombuffer(np.uint64(pairs.shape[0]).tobytes(), dtype=np.uint8)
    hdr[12:16] = np.frombuffer(np.int32(1 if labels is not None else 0).tobytes(), dtype=np.uint8)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        if labels is not None:
            f.write(np.ascontiguousarray(labels, dtype=np.uint32).tobytes())
        f.write(pairs.tobytes())


def read_dgraph(path):
    with open(path, "rb") as f:
        raw = f.read()
    n = int(np.frombuffer(raw[0:4], dtype=np.uint32)[0])
    m = int(np.frombuffer(raw[4:12], dtype=np.uint64)[0])
    hl = int(np.frombuffer(raw[12:16], dtype=np.int32)[0])
    pos = 20
    labels = None
    if hl:
        labels = np.frombuffer(raw[pos:pos + 4 * n], dtype=np.uint32).copy()
        pos += 4 * n
    pairs = np.frombuffer(raw[pos:pos + 8 * m], dtype=np.uint32).reshape(-1, 2).copy()
    return n, pairs, labels


_COUNT_RE = re.compile(r"Pattern count (\d+): (\d+)")
_RT_RE = re.compile(r"Average runtime: ([0-9.]+) \(ms\)")
_EXT_RE = re.compile(r"NumExtensionsTotal: ([0-9.]+)")


def run_reference(app, dgraph, threads=-1, runs=1, label=None, timeout=3600, warmup=0):
    """Run the reference's own app binary from oracle/_ref.  With label=None the stock
    app runs on the whole graph; with a label the sampled driver runs the v0 slice whose
    on-disk node label equals it, after `warmup` untimed runs.  Returns (counts, average runtime
    ms of the timed runs, num_extensions or None; the sampled driver's is the total over all runs,
    warm-up runs included)."""
    env = dict(os.environ)
    if label is None:
        exe = os.path.join(REF_DIR, app)
        args = [exe, dgraph, str(threads), str(runs), "false"]
    else:
        exe = os.path.join(REF_DIR, "sample_" + app)
        args = [exe, dgraph, str(threads), str(label), str(runs)] + ([str(warmup)] if warmup > 0 else [])
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout, env=env)
    if out.returncode != 0:
        raise RuntimeError("%s failed (%d): %s" % (exe, out.returncode, out.stderr[-2000:]))
    counts = {}
    for pid, c in _COUNT_RE.findall(out.stdout):
        counts[int(pid)] = int(c)          # the last run's values win
    rt = float(_RT_RE.findall(out.stdout)[-1])
    ext = None
    m = _EXT_RE.findall(out.stdout)
    if m:
        ext = int(float(m[-1]))
    else:
        for line in out.stdout.splitlines():
            if line.strip().startswith("NumExtensions"):
                ext = line
    return [counts[k] for k in sorted(counts)], rt, ext


def fsm(off, adj, labels, threshold, threads=0):
    """The 3-FSM levels (kautomine/three_fsm.cc) of a symmetric labelled graph: per level (single
    vertices, edges, wedges, triangles, four-chains, three-stars) a dict with num_candidates,
    num_frequent and support_sum."""
    labels = np.ascontiguousarray(labels, dtype=np.uint32)
    n = off.shape[0] - 1
    nl = int(labels.max()) + 1 if n else 1
    nc = np.zeros(6, dtype=np.uint32)
    nf = np.zeros(6, dtype=np.uint32)
    ss = np.zeros(6, dtype=np.uint64)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    if adj.shape[0] == 0:
        adj = np.zeros(1, dtype=np.uint32)
    rc = lib().orc_fsm(n, off, adj, labels if n else np.zeros(1, dtype=np.uint32), nl, threshold, threads,
                       nc, nf, ss)
    if rc != 0:
        raise ValueError("orc_fsm failed (%d)" % rc)
    return [{"num_candidates": int(nc[i]), "num_frequent": int(nf[i]), "support_sum": int(ss[i])}
            for i in range(6)]
