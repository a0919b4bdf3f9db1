"""CPU checks of the C ABI: the library loads and exports every declared symbol.

No compute call is made (there is no GPU here); these tests pin the boundary
between ``include/tsph.h``, the built library and the ctypes binding.
"""
import ctypes
import math
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(tsph_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def library():
    from tensorsph_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from tensorsph_b200.build import build
        build()
    return _lib.lib()


def test_header_declares_functions():
    assert len(declared_functions()) >= 20


def test_library_exports_every_declared_symbol(library):
    missing = [n for n in sorted(declared_functions()) if not hasattr(library, n)]
    assert not missing, missing


def test_ctypes_binding_covers_header():
    from tensorsph_b200 import _lib
    assert declared_functions() == set(_lib.EXPORTED)


def test_pure_host_entry_points(library):
    assert library.tsph_abi_version() == 2
    assert library.tsph_status_string(0) == b"ok"
    assert b"finite" in library.tsph_status_string(2)
    assert library.tsph_grid_plan_scratch_bytes() >= 64
    assert library.tsph_pairs_emit_workspace_bytes(100, 10) >= 400
    assert library.tsph_csr_workspace_bytes(100, 10) > 0


def test_engine_sizing_is_host_only(library):
    """Engine footprint and per-case cell counts need no GPU (admission control)."""
    import ctypes
    from tensorsph_b200 import _lib
    prm = _lib.EngineParams(max_fluid=1000, max_wall=500, max_obstacle=0, max_cells=4096,
                            max_cases=4, max_neighbors=64, diag_ring=8)
    small = library.tsph_engine_bytes(ctypes.byref(prm))
    prm.max_fluid = 2000
    assert library.tsph_engine_bytes(ctypes.byref(prm)) > small > 1000 * 64 * 4
    prm.max_cases = 0
    assert library.tsph_engine_bytes(ctypes.byref(prm)) == -1
    c = _lib.CaseParams(dim=2, n_fluid=10, n_wall=0, h=0.013, rho0=1000.0, sound_speed=20.0,
                        gamma=7.0, dt=1e-4, skin=0.0)
    c.grid_lo[0], c.grid_lo[1] = -0.1, -0.1
    c.grid_hi[0], c.grid_hi[1] = 0.9, 0.4
    cell = 2 * 0.013
    nx, ny = math.ceil(1.0 / cell) + 1, math.ceil(0.5 / cell) + 1
    assert library.tsph_engine_case_cells(ctypes.byref(c)) == nx * ny
    c.n_fluid = 0
    assert library.tsph_engine_case_cells(ctypes.byref(c)) == -1


def test_struct_sizes_match_header():
    """ctypes mirrors of the parameter structs have the C layout (all 8-byte fields)."""
    from tensorsph_b200 import _lib
    assert ctypes.sizeof(_lib.Grid) == 8 * (4 + 1 + 3 + 3 + 3 + 3 + 4)
    assert ctypes.sizeof(_lib.WcsphParams) == 8 * (6 + 14 + 5)
    assert ctypes.sizeof(_lib.WcsphIO) == 8 * 16
    assert ctypes.sizeof(_lib.ThreedParams) == 8 * (9 + 8 + 6)
    assert ctypes.sizeof(_lib.ShiftParams) == 8 * 9
    assert ctypes.sizeof(_lib.ClampParams) == 8 * (3 + 3 + 3 + 1 + 1 + 3 + 3 + 1)
    assert ctypes.sizeof(_lib.EngineParams) == 8 * 8
    assert ctypes.sizeof(_lib.CaseParams) == 8 * (6 + 11 + 3 + 1 + 3 + 3 + 1 + 4 + 3 + 3 + 2 + 4 + 1 + 3 + 2 + 5 + 6 + 2 + 2 + 3 + 2 + 7)
    assert ctypes.sizeof(_lib.Csf3Params) == 8 * (3 + 3 + 4 + 1)
    assert ctypes.sizeof(_lib.Csf3IO) == 8 * 11
    assert ctypes.sizeof(_lib.TvcParams) == 8 * (8 + 8)
    assert ctypes.sizeof(_lib.Csf2Params) == 8 * (8 + 7)
    assert ctypes.sizeof(_lib.Csf2IO) == 8 * 11
    assert ctypes.sizeof(_lib.TvcIO) == 8 * 13


def test_product_path_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from tensorsph_b200.neighbor_search import cell_linked_pairs
    with pytest.raises(RuntimeError, match="CUDA device"):
        cell_linked_pairs(torch.rand((10, 2)), 0.3)
