"""The C-ABI library loads and exports every entry point include/*.h declares;
argument validation and the table / variant queries work without a GPU (no
compute call is made here)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# header -> shared library that must export everything it declares
LIBS = {"tk_ntt.h": "libtk.so", "tk_pqcrystals.h": "libtk_pqcrystals.so"}


def declared_functions(header=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if header and os.path.basename(h) != header:
            continue
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9 ]+[\s\*]+(\w+)\s*\(", src, flags=re.M):
            if m.group(1) not in ("if", "while", "defined", "sizeof"):
                names.add(m.group(1))
    return names


def test_every_header_has_a_library():
    headers = {os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h"))}
    assert headers <= set(LIBS), headers - set(LIBS)


def test_every_declared_symbol_is_exported(tk):
    assert {"tk_ntt", "tk_invntt", "tk_ntt_host", "tk_invntt_host"} <= declared_functions("tk_ntt.h")
    for header, so in LIBS.items():
        names = declared_functions(header)
        assert names, header
        lib = ctypes.CDLL(os.path.join(ROOT, "tensorkyber_b200", so))
        missing = [n for n in sorted(names) if not hasattr(lib, n)]
        assert not missing, (header, missing)


def test_abi_version_and_strings(tk):
    L = tk.lib()
    assert L.tk_abi_version() == 1
    for code in range(9):
        assert L.tk_status_string(code)
    assert L.tk_status_string(99) == b"unknown status"
    assert tk.variant_count() >= 1
    assert all(tk.variant_name(v) for v in range(tk.variant_count()))
    assert tk.variant_name(99) == ""


def test_argument_errors_before_any_device_work(tk):
    """These return before the library touches the GPU."""
    L = tk.lib()
    assert L.tk_ntt(None, 0, None) == 0                       # empty batch: no-op
    assert L.tk_ntt(None, 5, None) == 1                       # NULL
    assert L.tk_invntt_oop(None, None, 5, None) == 1
    buf = np.zeros(8 * 256 + 16, dtype=np.int16)
    base = (buf.ctypes.data + 15) & ~15
    assert L.tk_ntt(base + 2, 4, None) == 2                   # misaligned
    assert L.tk_ntt(base, (1 << 32) + 1, None) == 3           # too large
    assert L.tk_ntt_oop(base, base + 512, 4, None) == 1       # partial overlap
    assert L.tk_ntt_host(None, 3) == 1
    assert L.tk_ntt_host(None, 0) == 0
    assert b"aligned" in L.tk_last_error() or L.tk_last_error() == b""


def test_variant_selection(tk):
    L = tk.lib()
    assert L.tk_set_variant(tk.FORWARD, 99) == 1
    assert L.tk_set_variant(5, 0) == 1
    tk.set_variant(tk.FORWARD, 1)
    assert tk.get_variant(tk.FORWARD, 1000) == 1
    tk.set_variant(tk.FORWARD, -1)
    assert 0 <= tk.get_variant(tk.FORWARD, 1000) < tk.variant_count()
    assert L.tk_get_variant(7, 10) < 0
    assert tk.variant_count() == 5
    assert L.tk_set_variant(tk.FORWARD, 5) == 1
    for d in (tk.FORWARD, tk.INVERSE):                   # the tcgen05 variant
        assert L.tk_set_variant(d, 4) == 0
        assert tk.get_variant(d, 1000) == 4
        tk.set_variant(d, -1)
    assert "tcgen05" in tk.variant_name(4)


def test_untuned_defaults(tk):
    """Without forcing or tuning: the int32-tile mma.sync forward (3) at every
    size; the inverse on the 3-slot mma.sync kernel (0) below 2^18
    polynomials and on the tcgen05 kernel (4) from there, where it leads."""
    for d in (tk.FORWARD, tk.INVERSE):
        tk.set_variant(d, -1)
    for n in (1, 4096, (1 << 18) - 1, 1 << 18, 1 << 24):
        assert tk.get_variant(tk.FORWARD, n) == 3
        assert tk.get_variant(tk.INVERSE, n) == (4 if n >= (1 << 18) else 0)


def test_get_table_sizes(tk):
    L = tk.lib()
    assert L.tk_get_table(0, None, 0) == 16 * 16 * 2
    assert L.tk_get_table(1, None, 0) == 16 * 16 * 16 * 2
    assert L.tk_get_table(6, None, 0) == 128 * 4
    assert L.tk_get_table(7, None, 0) == L.tk_get_table(5, None, 0)
    assert L.tk_get_table(8, None, 0) == 68 * 1024            # the tcgen05 kernels' tiles
    assert L.tk_get_table(9, None, 0) < 0
    assert L.tk_get_table(-1, None, 0) < 0
    small = (ctypes.c_uint8 * 4)()
    assert L.tk_get_table(0, small, 4) == 512                 # truncating copy is allowed


def test_matvec_argument_errors_without_gpu(tk):
    L = tk.lib()
    buf = np.zeros(64 * 256 + 16, dtype=np.int16)
    base = (buf.ctypes.data + 15) & ~15
    B = tk.MatvecBatch
    assert L.tk_matvec(None, 0, None) == 0
    assert L.tk_matvec(None, 2, None) == 1
    for k, expect in ((1, 1), (5, 1)):
        arr = (B * 1)(B(k, 2, base, base + 8192, None, base + 16384))
        assert L.tk_matvec(arr, 1, None) == expect
    arr = (B * 1)(B(2, 2, None, base, None, base))
    assert L.tk_matvec(arr, 1, None) == 1
    arr = (B * 1)(B(2, 2, base + 2, base + 8192, None, base + 16384))
    assert L.tk_matvec(arr, 1, None) == 2
    arr = (B * 1)(B(2, 2, base, base + 8192, None, base + 512))      # out inside A
    assert L.tk_matvec(arr, 1, None) == 1
    arr = (B * 1)(B(2, 0, None, None, None, None))                  # empty batch: no-op
    assert L.tk_matvec(arr, 1, None) == 0


def test_server_argument_errors_without_gpu(tk):
    import ctypes
    L = tk.lib()
    h = ctypes.c_void_p()
    assert L.tk_server_create(0, None, None) == 1
    bad = tk.ServerConfig(100, 0, 0.0)                 # budget below 4 KiB
    assert L.tk_server_create(0, ctypes.byref(bad), ctypes.byref(h)) == 1
    t = ctypes.c_uint64()
    assert L.tk_server_submit(None, 2, 1, None, None, None, None, ctypes.byref(t)) == 1
    assert L.tk_server_wait(None, 1, 0.0) == 1
    assert L.tk_server_destroy(None, 0.0) == 1


def test_matvec_host_argument_errors_without_gpu(tk):
    L = tk.lib()
    B = tk.MatvecBatch
    assert L.tk_matvec_host(None, 0) == 0
    assert L.tk_matvec_host(None, 1) == 1
    buf = np.zeros(64 * 256, dtype=np.int16)
    p = buf.ctypes.data
    assert L.tk_matvec_host((B * 1)(B(5, 1, p, p, None, p)), 1) == 1
    assert L.tk_matvec_host((B * 1)(B(2, 1, None, p, None, p)), 1) == 1
    assert L.tk_matvec_host((B * 1)(B(2, 1 << 29, p, p, None, p)), 1) == 3
    assert L.tk_matvec_host((B * 1)(B(4, 1 << 27, p, p, p, p)), 1) == 3   # > 8 GiB staging


def test_input_form_errors_without_gpu(tk):
    L = tk.lib()
    buf = np.zeros(8 * 256 + 16, dtype=np.int16)
    base = (buf.ctypes.data + 15) & ~15
    assert L.tk_ntt_small(None, None, 0, None) == 0
    assert L.tk_ntt_small(None, base, 3, None) == 1
    assert L.tk_ntt_small(base + 2, base + 2, 3, None) == 2
    assert L.tk_ntt_small(base, base + 512, 2, None) == 1          # partial overlap
    assert L.tk_ntt_packed(base, 5, base, 1, None) == 1
    x = np.zeros((2, 256), dtype=np.int16)
    x[1, 9] = 2                                                  # outside [-2, 1]
    with pytest.raises(tk.TKError):
        tk.pack_small(x, 2)
    x[1, 9] = -2
    p = tk.pack_small(x, 2)
    assert p.shape == (2, 64) and p[1, 2] == (2 << 2)


def test_selftest_argument_errors(tk):
    L = tk.lib()
    assert L.tk_selftest_bounded_wait(0, 0.0) == 1
    assert L.tk_selftest_bounded_wait(0, 11.0) == 1
