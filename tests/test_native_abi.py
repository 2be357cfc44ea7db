"""The C-ABI library loads here (no GPU) and exports every symbol include/pmb200.h declares."""
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "pmb200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long long|void\*)\s+(pm_\w+)\s*\(", text, re.M)))


def test_library_exports_header_symbols():
    from pbh_b200 import _lib
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(_lib.exported_symbols()) == syms


def test_cell_key_layout_host_helper():
    # [tile Morton | boundary mask | in-tile Morton] for N = 32, tile 8
    import ctypes as C
    from pbh_b200 import _lib
    lib = _lib.load()
    N, T = 32, 8
    ix, iy, iz = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    cells = ((ix * N + iy) * N + iz).astype(np.int32).ravel()
    keys = np.empty(cells.size, np.uint32)
    rc = lib.pm_cell_keys(cells.ctypes.data_as(C.c_void_p), cells.size, N, T, keys.ctypes.data_as(C.c_void_p))
    assert rc == 0
    assert len(np.unique(keys)) == cells.size             # a bijection of cells
    local = keys & np.uint32((1 << 9) - 1)
    mask = (keys >> np.uint32(9)) & np.uint32(7)
    tile = keys >> np.uint32(12)

    def spread(v):
        out = np.zeros_like(v)
        for b in range(10):
            out |= ((v >> b) & 1) << (3 * b)
        return out
    lx, ly, lz = ix.ravel() % T, iy.ravel() % T, iz.ravel() % T
    assert np.array_equal(local, (spread(lx) << 2) | (spread(ly) << 1) | spread(lz))
    m = (lx == T - 1) * 1 + (ly == T - 1) * 2 + (lz == T - 1) * 4
    assert np.array_equal(mask, m)
    tx, ty, tz = ix.ravel() // T, iy.ravel() // T, iz.ravel() // T
    assert np.array_equal(tile, (spread(tx) << 2) | (spread(ty) << 1) | spread(tz))
