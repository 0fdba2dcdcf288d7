"""Writes tests/golden/fsm.json: the reference's own 3-FSM app (kautomine/three_fsm.cc, compiled
unmodified into oracle/_ref/kautomine_three_fsm by oracle/Makefile) on seeded labelled graphs.
For each (graph, threshold) it records the lines the app prints per level: the number of frequent
patterns and their support sum.

    python tests/golden/make_fsm_golden.py      # about 13 minutes on 8 cores
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import orc  # noqa: E402

# graph generator, parameters, label rule (labels = (v * mult) % num_labels), thresholds
GRAPHS = [
    {"name": "er_n400_m4000_s7_l4", "kind": "er", "n": 400, "m": 4000, "seed": 7, "labels": 4, "mult": 7919,
     "thresholds": [20, 60, 150]},
    {"name": "rmat_s10_ef8_s2_l5", "kind": "rmat", "scale": 10, "ef": 8, "seed": 2, "labels": 5, "mult": 40503,
     "thresholds": [10, 40]},
    {"name": "rmat_s12_ef6_s3_l7", "kind": "rmat", "scale": 12, "ef": 6, "seed": 3, "labels": 7, "mult": 1,
     "thresholds": [60]},
    {"name": "er_n3000_m20000_s5_l3", "kind": "er", "n": 3000, "m": 20000, "seed": 5, "labels": 3, "mult": 31,
     "thresholds": [300]},
    # two labels: patterns with equal labels on symmetric positions, hubs of degree ~300
    {"name": "rmat_s11_ef8_s4_l2", "kind": "rmat", "scale": 11, "ef": 8, "seed": 4, "labels": 2, "mult": 3,
     "thresholds": [100, 400]},
    # skewed labels (label l with weight l + 1): thresholds that prune candidates at every level,
    # up to 12 labels (4 608 four-chain candidates)
    {"name": "rmat_s14_ef16_s11_skew2", "kind": "rmat", "scale": 14, "ef": 16, "seed": 11, "labels": 2,
     "mult": 7919, "rule": "skew", "thresholds": [4181]},
    {"name": "rmat_s14_ef16_s11_skew3", "kind": "rmat", "scale": 14, "ef": 16, "seed": 11, "labels": 3,
     "mult": 7919, "rule": "skew", "thresholds": [3136]},
    {"name": "rmat_s14_ef16_s11_skew5", "kind": "rmat", "scale": 14, "ef": 16, "seed": 11, "labels": 5,
     "mult": 7919, "rule": "skew", "thresholds": [2090]},
    {"name": "rmat_s14_ef16_s11_skew8", "kind": "rmat", "scale": 14, "ef": 16, "seed": 11, "labels": 8,
     "mult": 7919, "rule": "skew", "thresholds": [1254, 313]},
    {"name": "rmat_s13_ef16_s11_skew12", "kind": "rmat", "scale": 13, "ef": 16, "seed": 11, "labels": 12,
     "mult": 7919, "rule": "skew", "thresholds": [108]},
    {"name": "rmat_s15_ef8_s11_skew4", "kind": "rmat", "scale": 15, "ef": 8, "seed": 11, "labels": 4,
     "mult": 7919, "rule": "skew", "thresholds": [4213]},
]

LEVELS = ["single-vertex", "single-edge", "wedge", "triangle", "four-chain", "three-star"]
_LINE = re.compile(r"Number of frequent ([a-z-]+) patterns: (\d+), support sum(?: of them)?: (\d+)")


def graph_of(spec):
    if spec["kind"] == "er":
        canon, n = orc.er(spec["n"], spec["m"], spec["seed"])
    else:
        canon, n = orc.rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    if spec.get("rule", "mod") == "skew":
        # label l with weight l + 1: the residue of v * mult modulo L(L+1)/2 picks the label
        nl = spec["labels"]
        r = np.arange(n, dtype=np.uint64) * spec["mult"] % (nl * (nl + 1) // 2)
        labels = np.searchsorted(np.cumsum(np.arange(1, nl + 1)), r, side="right").astype(np.uint32)
    else:
        labels = (np.arange(n, dtype=np.uint64) * spec["mult"] % spec["labels"]).astype(np.uint32)
    return orc.symmetrize(canon), n, labels


def run_reference(path, threshold):
    exe = os.path.join(orc.REF_DIR, "kautomine_three_fsm")
    out = subprocess.run([exe, path, str(threshold)], capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(out.stderr[-2000:])
    levels = {}
    for kind, num, ssum in _LINE.findall(out.stdout):
        levels[kind] = {"num_frequent": int(num), "support_sum": int(ssum)}
    return [levels[k] for k in LEVELS]


def main():
    out = {"generator": "oracle/_ref/kautomine_three_fsm <graph.dgraph> <threshold>", "levels": LEVELS, "cases": []}
    with tempfile.TemporaryDirectory() as td:
        for spec in GRAPHS:
            sym, n, labels = graph_of(spec)
            path = os.path.join(td, spec["name"] + ".dgraph")
            orc.write_dgraph(path, n, sym, labels)
            for th in spec["thresholds"]:
                res = run_reference(path, th)
                out["cases"].append({"graph": spec, "threshold": th, "levels": res})
                print(spec["name"], th, res, flush=True)
    with open(os.path.join(HERE, "fsm.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
