"""The C-ABI library loads and exports every entry point include/khz.h declares (no GPU needed)."""
import os
import re

import pytest

from openkhuzdulgraph_b200 import khz

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        with open(os.path.join(ROOT, "include", hdr)) as f:
            text = f.read()
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(khz_[a-z_0-9]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_the_known_api():
    decl = declared_entry_points()
    assert set(khz.EXPORTS) <= set(decl)


def test_library_exports_every_declared_symbol():
    L = khz.lib()
    for name in declared_entry_points():
        assert hasattr(L, name), name


def test_metadata_without_gpu():
    L = khz.lib()
    assert L.khz_abi_version() == 2
    assert [khz.num_counts(a) for a in range(12)] == [1, 1, 1, 2, 1, 1, 1, 2, 1, 1, 1, 6]
    assert L.khz_app_multiplicity(3, 1) == 2
    assert [L.khz_app_multiplicity(11, p) for p in range(6)] == [1, 2, 1, 8, 1, 1]
    assert L.khz_app_num_counts(99) == 0


def test_errors_are_codes_not_aborts():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-device path")
    with pytest.raises(khz.KhzError) as e:
        khz.Context(0)
    assert e.value.status in (1, 5)
    L = khz.lib()
    assert L.khz_set_op_batch(42, None, None, None, None, None, None, None, 0, None) == 1
    assert L.khz_ctx_set_config(None, None) == 1


def test_config_layout_is_fixed():
    """khz_config keeps its size when fields are taken from the reserved words (64 bytes)."""
    import ctypes
    assert ctypes.sizeof(khz.Config) == 64
    assert khz.Config.bitmap_hub_rows.offset == 24 and khz.Config.device_mem_limit_mib.offset == 28
    assert khz.Config.bitmap_tensor_cores.offset == 32 and khz.Config.reserved.offset == 36


def test_graph_info_layout():
    """khz_graph_info (ABI version 2): the label fields follow device_bytes."""
    import ctypes
    assert ctypes.sizeof(khz.GraphInfo) == 64
    assert khz.GraphInfo.device_bytes.offset == 40 and khz.GraphInfo.num_labels.offset == 48
    assert khz.GraphInfo.d_labels.offset == 56
