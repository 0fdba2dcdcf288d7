"""The full-size configurations pinned to the reference itself, through label-restricted slices.

Configuration K (4- and 5-clique on the degree-oriented R-MAT scale 22, edge factor 16 graph) and
configuration M (motifs on the symmetric R-MAT scale 20, edge factor 24 graph) are too large for the
reference's CPU path to count whole inside a test, so each is checked on one label class of its
start vertices: the graph is written as a labelled .dgraph (labels v % S), the reference's own app
(oracle/_ref/sample_<app>: the app's apply() and aggregators, compiled unmodified, run through
DistributedApplication with restrict_starting_vertex_label, distributed_application.h:54) counts
the start vertices of label 0, and the device counts the same slice of the same file through
khz_count_restricted.  Counts and NumExtensions must be equal.  The four schedules the reference
does not ship are checked against the oracle's slice, stored in tests/golden/slices_m.json by
tests/golden/make_slices.py.

The reference's own converter pipeline (converter, then to_oriented_dataset_converter) also builds
K from the oracle generator's edge list, and its oriented file must be byte-identical to the one the
device writes."""
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
import orc

pytestmark = pytest.mark.gpu

K_MOD = 256   # 1/256 of K's start vertices: about 20 s of reference 5-clique work on 14 threads
M_MOD = 32


def _have_ref(app):
    return os.path.exists(os.path.join(orc.REF_DIR, "sample_" + app))


def _sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def _divided(khz, app, raw):
    aid = orc.APPS[app]
    return [r // khz.lib().khz_app_multiplicity(aid, p) for p, r in enumerate(raw)]


@pytest.fixture(scope="module")
def k_file(khz_ctx):
    """K as a labelled oriented .dgraph written by the device, and its unlabelled twin."""
    with tempfile.TemporaryDirectory() as td:
        sym = khz_ctx.generate_rmat(22, 16, 0.57, 0.19, 0.19, 1)
        og = sym.orient()
        sym.free()
        n = og.num_vertices
        plain = os.path.join(td, "k_oriented.dgraph")
        og.write_dgraph(plain)
        path = os.path.join(td, "k_oriented_labelled.dgraph")
        og.write_dgraph(path, labels=(np.arange(n, dtype=np.uint64) % K_MOD).astype(np.uint32))
        og.free()
        yield path, plain, n


@pytest.mark.timeout(900, method="thread")
@pytest.mark.parametrize("app", ["kautomine_four_clique", "kautomine_five_clique", "kgraphpi_five_clique"])
def test_clique_config_slice_matches_reference(khz_ctx, k_file, app):
    from openkhuzdulgraph_b200 import khz
    if not _have_ref(app):
        pytest.skip("oracle/_ref not built")
    path, _, _ = k_file
    g = khz_ctx.load_dgraph(path)
    assert g.info().oriented == 1 and g.info().num_labels == K_MOD
    raw, st = khz_ctx.count_restricted(g, app, 0)
    assert st.engine == khz.ENGINE_BITMAP
    g.free()
    ref_counts, _, ref_ext = orc.run_reference(app, path, threads=-1, runs=1, label=0, timeout=900)
    assert _divided(khz, app, raw) == ref_counts, app
    assert st.num_extensions == ref_ext, app


@pytest.mark.timeout(900, method="thread")
def test_clique_config_orientation_matches_reference_converters(k_file):
    """orc.rmat (bit-identical to the device generator) -> the reference's converter ->
    to_oriented_dataset_converter: the same bytes as the device's oriented K."""
    conv = os.path.join(orc.REF_DIR, "converter")
    ori = os.path.join(orc.REF_DIR, "to_oriented_dataset_converter")
    if not (os.path.exists(conv) and os.path.exists(ori)):
        pytest.skip("oracle/_ref not built")
    _, plain, n = k_file
    with tempfile.TemporaryDirectory() as td:
        canon, n2 = orc.rmat(22, 16, seed=1)
        assert n2 == n
        base = os.path.join(td, "k")
        canon.astype(np.uint32).tofile(base + ".biedgelist")
        del canon
        subprocess.run([conv, base, base, str(n), "0", "0", "0"], check=True, stdout=subprocess.DEVNULL,
                       timeout=600)
        os.remove(base + ".biedgelist")
        subprocess.run([ori, base + ".dgraph", base + ".oriented.dgraph"], check=True, stdout=subprocess.DEVNULL,
                       timeout=600)
        assert _sha(base + ".oriented.dgraph") == _sha(plain)


@pytest.fixture(scope="module")
def m_graph(khz_ctx):
    with tempfile.TemporaryDirectory() as td:
        g = khz_ctx.generate_rmat(20, 24, 0.57, 0.19, 0.19, 1)
        n = g.num_vertices
        path = os.path.join(td, "m_labelled.dgraph")
        g.write_dgraph(path, labels=(np.arange(n, dtype=np.uint64) % M_MOD).astype(np.uint32))
        g.free()
        g = khz_ctx.load_dgraph(path)
        assert g.info().symmetric == 1 and g.info().num_labels == M_MOD
        yield g, path, n
        g.free()


@pytest.mark.timeout(900, method="thread")
@pytest.mark.parametrize("app", ["kautomine_three_motif", "kgraphpi_three_motif", "kautomine_triangle",
                                 "kgraphpi_triangle"])
def test_motif_config_slice_matches_reference(khz_ctx, m_graph, app):
    from openkhuzdulgraph_b200 import khz
    if not _have_ref(app):
        pytest.skip("oracle/_ref not built")
    g, path, _ = m_graph
    raw, st = khz_ctx.count_restricted(g, app, 0)
    ref_counts, _, ref_ext = orc.run_reference(app, path, threads=-1, runs=1, label=0, timeout=900)
    assert _divided(khz, app, raw) == ref_counts, app
    assert st.num_extensions == ref_ext, app


@pytest.mark.timeout(900, method="thread")
def test_motif_config_new_schedules_match_oracle_slices(khz_ctx):
    """4-cycle, house, tailed triangle and 4-motif on M: the device's slice against the oracle's
    (the fixture records the generator, the label modulus and the label)."""
    with open(os.path.join(ROOT, "tests", "golden", "slices_m.json")) as f:
        fx = json.load(f)
    gen = fx["graph"]
    g = khz_ctx.generate_rmat(gen["scale"], gen["edge_factor"], 0.57, 0.19, 0.19, gen["seed"])
    n = g.num_vertices
    assert n == gen["n"]
    for case in fx["cases"]:
        labels = (np.arange(n, dtype=np.uint64) % case["mod"]).astype(np.uint32)
        g.set_labels(labels)
        raw, st = khz_ctx.count_restricted(g, case["app"], case["label"])
        assert raw == case["raw_counts"], case
        assert st.num_extensions == case["num_extensions"], case
    g.free()
