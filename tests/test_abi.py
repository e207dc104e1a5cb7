"""CPU tests of the drop-in boundary: the C-ABI library loads and exports every
entry point that include/pepcg.h declares (no compute without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

import pepc_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if not name.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", name)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|const char\*|int64_t|long long)\s+\**(pepcg_\w+)\s*\(", txt):
            syms.add(m.group(1))
    return syms


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert {"pepcg_create", "pepcg_grow_tree", "pepcg_traverse_tree", "pepcg_timber_tree"} <= syms


def test_library_exports_every_declared_symbol():
    lib = pepc_b200.lib()
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_symbols() == set(pepc_b200.EXPORTS)


def test_params_layout_matches_header():
    # pepcg_params: theta2, eps2; 13 int32 + 4 bytes of padding; 12 lattice
    # doubles; device, overwrite_results; kelbg_invsqrttemp; group_size,
    # reserved0; 3 cutoff doubles; reserved[4] (see pepcg.h)
    p = pepc_b200.make_params()
    assert p.theta2 == 0.36 and p.eps2 == 0.0 and p.force_law == 3 and p.tile_size == 16
    assert list(p.spatial_interaction_cutoff) == [np.finfo(np.float64).max] * 3
    assert ctypes.sizeof(pepc_b200.Params) == 2 * 8 + 14 * 4 + 12 * 8 + 2 * 4 + 8 + 2 * 4 + 3 * 8 + 4 * 4


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(pepc_b200.PepcgError):
        pepc_b200.TreeCode()
