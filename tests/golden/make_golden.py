"""Generate tests/golden/golden.json from the reference's OWN binaries.

Runs only in a container that holds the reference tree (the binaries are built from
it by oracle/Makefile into oracle/_ref).  For each seeded graph it records:
  * the sha256 of the .dgraph the reference's toolkits/converter writes from the
    graph's .biedgelist (pins this project's .dgraph writer and symmetrisation),
  * the sha256 of the .dgraph the reference's toolkits/to_oriented_dataset_converter
    writes (pins degree orientation),
  * for every reference app: the counts and NumExtensions printed by the stock app on
    the symmetric graph (and, for cliques, on the oriented graph),
  * for every reference app: counts and NumExtensions of the sampled driver over the
    start vertices with v0 % 4 == 1 (node labels v % 4).
The graph generators are this project's (oracle/khz_oracle.c); the graph parameters
are stored so the tests regenerate each graph and check its hash first.

usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import orc  # noqa: E402

CLIQUES = ["kautomine_triangle", "kautomine_four_clique", "kautomine_five_clique",
           "kgraphpi_triangle", "kgraphpi_four_clique", "kgraphpi_five_clique"]

GRAPHS = [
    {"name": "er_n400_m4000_s7", "kind": "er", "n": 400, "m": 4000, "seed": 7},
    {"name": "er_n2000_m30000_s1", "kind": "er", "n": 2000, "m": 30000, "seed": 1},
    {"name": "rmat_s10_ef8_s1", "kind": "rmat", "scale": 10, "ef": 8, "seed": 1},
    {"name": "rmat_s12_ef16_s2", "kind": "rmat", "scale": 12, "ef": 16, "seed": 2},
    {"name": "rmat_s9_ef24_s3", "kind": "rmat", "scale": 9, "ef": 24, "seed": 3},
    {"name": "complete_k7", "kind": "explicit",
     "pairs": [[a, b] for a in range(7) for b in range(a + 1, 7)]},
    {"name": "star_and_path", "kind": "explicit",
     "pairs": [[0, 1], [0, 2], [0, 3], [0, 4], [0, 5], [5, 6], [6, 7], [7, 8]]},
    {"name": "single_edge", "kind": "explicit", "pairs": [[0, 1]]},
]


def make_graph(spec):
    """canonical sorted unique pairs (m, 2) and vertex count, from the graph spec"""
    if spec["kind"] == "er":
        return orc.er(spec["n"], spec["m"], spec["seed"])
    if spec["kind"] == "rmat":
        return orc.rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    pairs = np.array(spec["pairs"], dtype=np.uint32).reshape(-1, 2)
    return pairs, int(pairs.max()) + 1


def sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main():
    ref = orc.REF_DIR
    out = {"generator": "oracle/khz_oracle.c orc_er / orc_rmat (a,b,c)=(0.57,0.19,0.19)",
           "sample": {"mod": 4, "rem": 1}, "graphs": []}
    with tempfile.TemporaryDirectory() as td:
        for spec in GRAPHS:
            canon, n = make_graph(spec)
            base = os.path.join(td, spec["name"])
            canon.astype(np.uint32).tofile(base + ".biedgelist")
            subprocess.run([os.path.join(ref, "converter"), base, base, str(n), "0", "0", "0"],
                           check=True, capture_output=True)
            sym_path = base + ".dgraph"
            ori_path = base + "_oriented.dgraph"
            r = subprocess.run([os.path.join(ref, "to_oriented_dataset_converter"), sym_path, ori_path],
                               capture_output=True)
            oriented_ok = r.returncode == 0
            # labelled copy for the sampled driver (labels v % 4)
            _, sym_pairs, _ = orc.read_dgraph(sym_path)
            lab_path = base + "_labeled.dgraph"
            orc.write_dgraph(lab_path, n, sym_pairs, labels=np.arange(n, dtype=np.uint32) % 4)
            rec = {k: v for k, v in spec.items() if k != "pairs"}
            if spec["kind"] == "explicit":
                rec["pairs"] = spec["pairs"]
            rec.update({"n": n, "m_undirected": int(canon.shape[0]),
                        "sha256_dgraph": sha(sym_path),
                        "sha256_oriented": sha(ori_path) if oriented_ok else None,
                        "apps": {}, "apps_oriented": {}, "apps_sampled": {}})
            # The reference's tools and apps divide work by thread count and abort on some
            # tiny graphs (SIGFPE in to_oriented_dataset_converter on n < threads); those
            # entries are recorded as null and pinned by brute force in the tests instead.
            for app in orc.REF_APPS:
                rec["apps"][app] = _try(lambda: orc.run_reference(app, sym_path, threads=4, runs=1))
                if n >= 4:
                    rec["apps_sampled"][app] = _try(
                        lambda: orc.run_reference(app, lab_path, threads=4, runs=1, label=1))
            for app in CLIQUES:
                if oriented_ok:
                    rec["apps_oriented"][app] = _try(lambda: orc.run_reference(app, ori_path, threads=4, runs=1))
            out["graphs"].append(rec)
            print(spec["name"], n, canon.shape[0], rec["apps"]["kautomine_four_clique"], oriented_ok, flush=True)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


def _try(fn):
    try:
        c, _, ext = fn()
        return {"counts": c, "num_extensions": _ext_value(ext)}
    except Exception as e:  # reference crashed on this input
        print("   reference failed:", str(e)[:200], flush=True)
        return None


def _ext_value(ext):
    """the stock apps print 'NumExtensions,\\t<avg>,\\t<max>,\\t<min>,\\t' (engine.h:1250-1254)"""
    if isinstance(ext, int):
        return ext
    return int(float(ext.split(",")[1]))


if __name__ == "__main__":
    main()
