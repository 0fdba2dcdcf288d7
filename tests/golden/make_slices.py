"""Writes tests/golden/slices_m.json: the oracle's counts for the four schedules the reference does
not ship (kgraphpi 4-cycle, house, tailed triangle; kautomine 4-motif) on configuration M (R-MAT
scale 20, edge factor 24, symmetric), restricted to one label class of the start vertices.

The whole-graph counts of these schedules take the CPU oracle far too long (their work grows with
the square of hub degrees: ~1.8e14 list-element steps for the 4-cycle alone), so one class of
labels v % 4096 is counted: label 341, a class of median cost (label 0 would hold vertex 0, the
largest hub).  Counts are the raw aggregator values of the restricted run (no multiplicity
division) and NumExtensions is the engine's counter for that run.

    python tests/golden/make_slices.py        # about 4 minutes on 8 cores
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import orc  # noqa: E402

SCALE, EDGE_FACTOR, SEED = 20, 24, 1
MOD, LABEL = 4096, 341
APPS = ["kgraphpi_four_cycle", "kgraphpi_house", "kgraphpi_tailed_triangle", "kautomine_four_motif"]


def main():
    canon, n = orc.rmat(SCALE, EDGE_FACTOR, seed=SEED)
    off, adj = orc.csr(orc.symmetrize(canon), n)
    labels = (np.arange(n, dtype=np.uint64) % MOD).astype(np.uint32)
    cases = []
    for app in APPS:
        raw, ext, _ = orc.count_labeled(app, off, adj, labels, LABEL)
        cases.append({"app": app, "mod": MOD, "label": LABEL, "raw_counts": raw, "num_extensions": ext})
        print(app, raw, ext, flush=True)
    out = {"graph": {"kind": "rmat", "scale": SCALE, "edge_factor": EDGE_FACTOR, "seed": SEED,
                     "a": 0.57, "b": 0.19, "c": 0.19, "n": n, "undirected_edges": int(canon.shape[0])},
           "generator": "oracle/khz_oracle.c orc_rmat (bit-identical to khz_graph_generate_rmat)",
           "cases": cases}
    with open(os.path.join(HERE, "slices_m.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
