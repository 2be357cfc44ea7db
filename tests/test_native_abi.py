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
    # Morton code of the CIC cell, z in the lowest bit of each triple (codes nest by super-tile)
    import ctypes as C
    from pbh_b200 import _lib
    lib = _lib.load()
    N = 32
    ix, iy, iz = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    cells = ((ix * N + iy) * N + iz).astype(np.int32).ravel()
    keys = np.empty(cells.size, np.uint32)
    rc = lib.pm_cell_keys(cells.ctypes.data_as(C.c_void_p), cells.size, N, 16, keys.ctypes.data_as(C.c_void_p))
    assert rc == 0
    assert len(np.unique(keys)) == cells.size             # a bijection of cells

    def spread(v):
        out = np.zeros_like(v)
        for b in range(10):
            out |= ((v >> b) & 1) << (3 * b)
        return out
    ref = (spread(ix.ravel()) << 2) | (spread(iy.ravel()) << 1) | spread(iz.ravel())
    assert np.array_equal(keys, ref.astype(np.uint32))
    # the top bits are the Morton code of the 16^3 super-tile
    st = (spread(ix.ravel() // 16) << 2) | (spread(iy.ravel() // 16) << 1) | spread(iz.ravel() // 16)
    assert np.array_equal(keys >> np.uint32(12), st.astype(np.uint32))


def test_invariant_divisor_magic_numbers():
    """The Green kernel splits a mode index m = row * (N/2 + 1) + kz with a multiply-high by a
    magic number (common.cuh pm_div_magic / pm_div_by); the same arithmetic, exactly, for every
    mesh size on samples that include every multiple of the divisor near the range ends."""
    import numpy as np
    rng = np.random.default_rng(0)
    for N in (8, 16, 32, 64, 128, 256, 512, 1024):
        d = N // 2 + 1
        l = 0
        while (1 << l) < d:
            l += 1
        magic = ((1 << 32) * ((1 << l) - d)) // d + 1
        top = N * N * d
        n = np.concatenate([np.arange(0, min(top, 200000)), np.arange(max(0, top - 200000), top),
                            rng.integers(0, top, 200000), (np.arange(1, 2000) * d)[:, None].ravel() - 1])
        n = n[(n >= 0) & (n < top)].astype(np.uint64)
        q = (((n * np.uint64(magic)) >> np.uint64(32)) + n) >> np.uint64(l)
        assert np.array_equal(q, n // np.uint64(d)), N


def test_native_fft_rejects_other_sizes_before_touching_the_device():
    """Only 64^3 to 512^3 have a native transform; other sizes are refused with the
    invalid-argument code for the size, before any pointer is used or any CUDA call is made."""
    from pbh_b200 import _lib
    lib = _lib.load()
    assert lib.pm_rfft3_native(32, 16, 16, 1, None) == -2000
    assert lib.pm_irfft3_native(1024, 16, 16, 16, 1, None) == -2000
    assert lib.pm_rfft3_native(300, 16, 16, 1, None) == -2000


def test_ctypes_structures_match_the_header_layout(tmp_path):
    """Every structure the bindings pass through the C ABI has the header's size and field
    offsets (a mismatch would silently corrupt the engine's configuration or results)."""
    import ctypes as C
    import shutil
    import subprocess

    import pytest
    from pbh_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"pm_peak_cfg": _lib.PeakCfg, "pm_clock_info": _lib.ClockInfo, "pm_stats_info": _lib.StatsInfo,
               "pm_ic_params": _lib.ICParams}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pmb200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, key, val = row.split()
        got[(cname, key)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_bindings_pass_as_many_arguments_as_the_header_declares():
    """The ctypes signatures of every entry point have the header prototype's parameter count and
    a return type of the same width."""
    import ctypes as C

    from pbh_b200 import _lib
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "pmb200.h").read_text(), flags=re.S)
    protos = re.findall(r"^\s*(int|long long|void\*)\s+(pm_\w+)\s*\(([^)]*)\)\s*;", text, re.M | re.S)
    assert sorted(name for _, name, _ in protos) == header_symbols()
    width = {"int": C.sizeof(C.c_int), "long long": C.sizeof(C.c_longlong), "void*": C.sizeof(C.c_void_p)}
    for ret, name, args in protos:
        restype, argtypes = _lib._SIGS[name]
        nargs = 0 if args.strip() in ("", "void") else len(args.split(","))
        assert len(argtypes) == nargs, name
        assert C.sizeof(restype) == width[ret], name


def test_no_kernel_spills_registers(tmp_path):
    """Every kernel compiles for sm_100a without register spills (the push and the deposit run
    at the register limit of their launch bounds, where a spill would add local-memory traffic
    to an HBM-bound loop).  Compiles each source to an object in a scratch folder."""
    import shutil
    import subprocess

    import pytest
    from pbh_b200 import build
    try:
        nvcc = build.nvcc()
    except RuntimeError:
        pytest.skip("nvcc not found")
    if not shutil.which(nvcc) and not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    for src in build.sources():
        res = subprocess.run([nvcc, *build.ARCH, "-O3", "-std=c++17", "-Xptxas", "-v", "-c", str(src),
                              "-o", str(tmp_path / (src.stem + ".o"))], capture_output=True, text=True)
        assert res.returncode == 0, res.stderr[-2000:]
        counts = re.findall(r"(\d+) bytes spill stores, (\d+) bytes spill loads", res.stderr)
        assert counts or "__global__" not in src.read_text(), src.name
        assert all(st == "0" and ld == "0" for st, ld in counts), (src.name, res.stderr[-2000:])
