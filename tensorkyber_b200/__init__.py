"""tensorkyber_b200 -- B200 batched ML-KEM NTT / iNTT engine.

Python face of the C ABI in ``include/tk_ntt.h`` (``libtk.so``).  The compute
path is the sm_100a CUDA library; there is no CPU implementation here, and the
module raises when the library cannot be loaded.

Conventions follow the pqcrystals reference ``ntt()`` / ``invntt()``
(TensorKyber ``ntt_bench/ref/ntt.c:80-126``): forward output is bit-reversed
and lands in [0, q); inverse output is multiplied by 2^16 and centred in
[-(q-1)/2, (q-1)/2].  Every coefficient is congruent mod q to the reference's.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

Q = 3329
N = 256
_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtk.so")
CSRC = os.path.join(_HERE, "csrc")

STATUS = {
    0: "TK_SUCCESS", 1: "TK_ERR_INVALID_VALUE", 2: "TK_ERR_MISALIGNED",
    3: "TK_ERR_TOO_LARGE", 4: "TK_ERR_NO_DEVICE", 5: "TK_ERR_CUDA",
    6: "TK_ERR_NOT_DEVICE_MEMORY", 7: "TK_ERR_KERNEL_TIMEOUT", 8: "TK_ERR_TIMEOUT",
}


class MatvecBatch(ctypes.Structure):
    """Mirror of tk_matvec_batch (include/tk_ntt.h)."""
    _fields_ = [("k", ctypes.c_int), ("njobs", ctypes.c_size_t), ("A", ctypes.c_void_p),
                ("s", ctypes.c_void_p), ("e", ctypes.c_void_p), ("out", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    """Mirror of tk_server_config (include/tk_ntt.h)."""
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight_requests", ctypes.c_int),
                ("idle_exit_seconds", ctypes.c_double), ("zero_copy", ctypes.c_int)]


class ServerCounters(ctypes.Structure):
    """Mirror of tk_server_counters (include/tk_ntt.h)."""
    _fields_ = [(n, ctypes.c_ulonglong) for n in (
        "requests_done", "jobs_done", "device_loop_launches", "direct_requests",
        "staged_requests", "direct_outputs", "queue_ns", "device_ns", "return_ns",
        "input_copies")]


class TKError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    """Compile libtk.so in-tree (nvcc, sm_100a)."""
    with _lock:
        if force or not os.path.exists(LIB_PATH) or _stale():
            subprocess.run(["make", "-s", "-C", CSRC], check=True)
    return LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(LIB_PATH)
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".cpp", ".c", ".h")) and os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(_HERE, "..", "include")
    if os.path.isdir(hdr):
        for f in os.listdir(hdr):
            if os.path.getmtime(os.path.join(hdr, f)) > t:
                return True
    return False


def lib() -> ctypes.CDLL:
    """Load libtk.so (building it first if it is missing or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) or _stale():
        build()
    L = ctypes.CDLL(LIB_PATH)
    p16 = ctypes.c_void_p
    for name in ("tk_ntt", "tk_invntt"):
        f = getattr(L, name)
        f.argtypes = [p16, ctypes.c_size_t, ctypes.c_void_p]
        f.restype = ctypes.c_int
    for name in ("tk_ntt_oop", "tk_invntt_oop"):
        f = getattr(L, name)
        f.argtypes = [p16, p16, ctypes.c_size_t, ctypes.c_void_p]
        f.restype = ctypes.c_int
    for name in ("tk_ntt_host", "tk_invntt_host"):
        f = getattr(L, name)
        f.argtypes = [p16, ctypes.c_size_t]
        f.restype = ctypes.c_int
    L.tk_init.argtypes = [ctypes.c_int]
    L.tk_init.restype = ctypes.c_int
    L.tk_device_status.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]
    L.tk_device_status.restype = ctypes.c_int
    L.tk_selftest_bounded_wait.argtypes = [ctypes.c_int, ctypes.c_double]
    L.tk_selftest_bounded_wait.restype = ctypes.c_int
    L.tk_status_string.argtypes = [ctypes.c_int]
    L.tk_status_string.restype = ctypes.c_char_p
    L.tk_last_error.argtypes = []
    L.tk_last_error.restype = ctypes.c_char_p
    L.tk_abi_version.restype = ctypes.c_int
    L.tk_get_table.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    L.tk_get_table.restype = ctypes.c_longlong
    L.tk_variant_count.restype = ctypes.c_int
    L.tk_variant_name.argtypes = [ctypes.c_int]
    L.tk_variant_name.restype = ctypes.c_char_p
    L.tk_set_variant.argtypes = [ctypes.c_int, ctypes.c_int]
    L.tk_set_variant.restype = ctypes.c_int
    L.tk_get_variant.argtypes = [ctypes.c_int, ctypes.c_size_t]
    L.tk_get_variant.restype = ctypes.c_int
    L.tk_autotune.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_char_p]
    L.tk_autotune.restype = ctypes.c_int
    L.tk_autotune_reset.restype = ctypes.c_int
    L.tk_ntt_small.argtypes = [p16, p16, ctypes.c_size_t, ctypes.c_void_p]
    L.tk_ntt_small.restype = ctypes.c_int
    L.tk_ntt_packed.argtypes = [ctypes.c_void_p, ctypes.c_int, p16, ctypes.c_size_t,
                                ctypes.c_void_p]
    L.tk_ntt_packed.restype = ctypes.c_int
    L.tk_pack_small.argtypes = [p16, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
    L.tk_pack_small.restype = ctypes.c_int
    L.tk_matvec.argtypes = [ctypes.POINTER(MatvecBatch), ctypes.c_int, ctypes.c_void_p]
    L.tk_matvec.restype = ctypes.c_int
    L.tk_matvec_host.argtypes = [ctypes.POINTER(MatvecBatch), ctypes.c_int]
    L.tk_matvec_host.restype = ctypes.c_int
    L.tk_matvec_host_noalloc.argtypes = [ctypes.POINTER(MatvecBatch), ctypes.c_int,
                                         ctypes.c_void_p]
    L.tk_matvec_host_noalloc.restype = ctypes.c_int
    vp, u64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)
    L.tk_server_create.argtypes = [ctypes.c_int, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.tk_server_submit.argtypes = [vp, ctypes.c_int, ctypes.c_size_t, vp, vp, vp, vp, u64p]
    L.tk_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double]
    L.tk_server_query.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double)]
    L.tk_server_release.argtypes = [vp, ctypes.c_uint64]
    L.tk_server_stats.argtypes = [vp, ctypes.POINTER(ServerCounters)]
    L.tk_server_destroy.argtypes = [vp, ctypes.c_double]
    for f in ("tk_server_create", "tk_server_submit", "tk_server_wait", "tk_server_query",
              "tk_server_release", "tk_server_stats", "tk_server_destroy"):
        getattr(L, f).restype = ctypes.c_int
    L.tk_set_option.argtypes = [ctypes.c_int, ctypes.c_longlong]
    L.tk_set_option.restype = ctypes.c_int
    L.tk_get_option.argtypes = [ctypes.c_int]
    L.tk_get_option.restype = ctypes.c_longlong
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise TKError(rc, lib().tk_last_error().decode(errors="replace"))


# ---------------------------------------------------------------- tables ----
_TABLE_SHAPES = {0: (16, 16), 1: (16, 16, 16), 2: (16, 16, 16), 3: (16, 16)}


def get_table(which: int) -> np.ndarray:
    """Host matrix builder output (no GPU needed): 0 M1, 1 M2, 2 MA, 3 Minv as
    int16 residues; 4 / 5 the forward / inverse fragment tables as raw uint32;
    6 the basemul pair constants as int32[128]; 7 the tiled matrix-vector
    kernel's inverse fragment tables (2^-16 * invntt) as raw uint32; 8 the
    tcgen05 kernels' 68 int8 B-operand tiles of 1 KiB, raw (view as uint8)."""
    L = lib()
    size = L.tk_get_table(which, None, 0)
    if size < 0:
        raise TKError(-size, f"table {which}")
    buf = np.zeros(size, dtype=np.uint8)
    L.tk_get_table(which, buf.ctypes.data, size)
    if which in _TABLE_SHAPES:
        return buf.view(np.int16).reshape(_TABLE_SHAPES[which])
    if which == 6:
        return buf.view(np.int32)
    return buf.view(np.uint32)


# ----------------------------------------------------------- transforms -----
def _stream_ptr(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(getattr(stream, "cuda_stream", stream))


def _check_tensor(t) -> int:
    import torch
    if not isinstance(t, torch.Tensor) or t.dtype != torch.int16 or not t.is_cuda:
        raise TypeError("expected a CUDA int16 tensor")
    if not t.is_contiguous() or t.numel() % N:
        raise ValueError("expected a contiguous tensor of whole int16[256] polynomials")
    return t.numel() // N


def ntt(polys, out=None, stream=None):
    """Batched forward NTT of a CUDA int16 tensor (..., 256).  In place when
    out is None or out is polys; returns the output tensor."""
    n = _check_tensor(polys)
    if out is None or out is polys:
        _check(lib().tk_ntt(polys.data_ptr(), n, _stream_ptr(stream)))
        return polys
    if _check_tensor(out) != n:
        raise ValueError("out has a different number of polynomials")
    _check(lib().tk_ntt_oop(polys.data_ptr(), out.data_ptr(), n, _stream_ptr(stream)))
    return out


def invntt(polys, out=None, stream=None):
    """Batched inverse NTT (with the 2^16 factor) of a CUDA int16 tensor."""
    n = _check_tensor(polys)
    if out is None or out is polys:
        _check(lib().tk_invntt(polys.data_ptr(), n, _stream_ptr(stream)))
        return polys
    if _check_tensor(out) != n:
        raise ValueError("out has a different number of polynomials")
    _check(lib().tk_invntt_oop(polys.data_ptr(), out.data_ptr(), n, _stream_ptr(stream)))
    return out


def _host_arr(a: np.ndarray) -> int:
    if not isinstance(a, np.ndarray) or a.dtype != np.int16 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous numpy int16 array")
    if a.size % N:
        raise ValueError("expected whole int16[256] polynomials")
    return a.size // N


def ntt_host(a: np.ndarray) -> np.ndarray:
    """Forward NTT of host polynomials in place (synchronous, through the GPU)."""
    _check(lib().tk_ntt_host(a.ctypes.data, _host_arr(a)))
    return a


def invntt_host(a: np.ndarray) -> np.ndarray:
    """Inverse NTT of host polynomials in place (synchronous, through the GPU)."""
    _check(lib().tk_invntt_host(a.ctypes.data, _host_arr(a)))
    return a


FLAG_FORWARD_TIMEOUT, FLAG_INVERSE_TIMEOUT, FLAG_SMALL_RANGE, FLAG_SELFTEST_TIMEOUT = 1, 2, 4, 8
FLAG_MATVEC_TIMEOUT = 16


def ntt_small(polys, out=None, stream=None):
    """Forward NTT of CUDA int16 polynomials with coefficients in [-128, 127]
    (single-limb stage 1).  Out-of-range inputs set FLAG_SMALL_RANGE."""
    n = _check_tensor(polys)
    if out is None:
        out = polys
    elif _check_tensor(out) != n:
        raise ValueError("out must hold as many polynomials as polys")
    _check(lib().tk_ntt_small(polys.data_ptr(), out.data_ptr(), n, _stream_ptr(stream)))
    return out


def ntt_packed(packed, bits, out=None, stream=None):
    """Forward NTT of packed small polynomials: packed is a CUDA uint8 tensor
    of (npoly, 256 * bits / 8 rounded to 64 or 128) bytes; returns int16
    (npoly, 256) NTT-domain polynomials in [0, q)."""
    import torch
    row = 64 if bits == 2 else 128
    if not isinstance(packed, torch.Tensor) or packed.dtype != torch.uint8 or not packed.is_cuda \
            or not packed.is_contiguous() or packed.numel() % row:
        raise TypeError(f"expected a contiguous CUDA uint8 tensor of {row}-byte rows")
    n = packed.numel() // row
    if out is None:
        out = torch.empty((n, N), dtype=torch.int16, device=packed.device)
    elif _check_tensor(out) != n:
        raise ValueError("out must hold one polynomial per packed row")
    _check(lib().tk_ntt_packed(packed.data_ptr(), bits, out.data_ptr(), n, _stream_ptr(stream)))
    return out


def pack_small(polys: np.ndarray, bits: int) -> np.ndarray:
    """Host packing of int16 polynomials into the tk_ntt_packed format."""
    n = _host_arr(polys)
    row = 64 if bits == 2 else 128
    out = np.zeros((n, row), dtype=np.uint8)
    _check(lib().tk_pack_small(polys.ctypes.data, n, bits, out.ctypes.data))
    return out


def matvec(batches, stream=None):
    """ML-KEM matrix-vector jobs on CUDA int16 tensors.

    batches: iterable of (k, A, s, e, out) with A of shape (njobs, k, k, 256),
    s / e / out of shape (njobs, k, 256); e may be None; out may be s.
    out_i = invntt(sum_j basemul(A_ij, ntt(s_j))) + e_i for every job."""
    items = []
    for k, A, s, e, out in batches:
        n = _check_tensor(s) // k
        if _check_tensor(A) != n * k * k or _check_tensor(out) != n * k or (
                e is not None and _check_tensor(e) != n * k):
            raise ValueError("inconsistent matvec batch shapes")
        items.append(MatvecBatch(k, n, A.data_ptr(), s.data_ptr(),
                                 e.data_ptr() if e is not None else None, out.data_ptr()))
    arr = (MatvecBatch * len(items))(*items)
    _check(lib().tk_matvec(arr, len(items), _stream_ptr(stream)))


NOALLOC_SCRATCH_BYTES = 4 << 20


def _host_batches(batches):
    items = []
    for k, A, s, e, out in batches:
        n = _host_arr(s) // k
        if _host_arr(A) != n * k * k or _host_arr(out) != n * k or (
                e is not None and _host_arr(e) != n * k):
            raise ValueError("inconsistent matvec batch shapes")
        items.append(MatvecBatch(k, n, A.ctypes.data, s.ctypes.data,
                                 e.ctypes.data if e is not None else None, out.ctypes.data))
    return (MatvecBatch * len(items))(*items), len(items)


def matvec_host_noalloc(batches, stream=0):
    """tk_matvec_host_noalloc: like matvec_host, staged in the library's static
    device scratch (NOALLOC_SCRATCH_BYTES); allocates nothing."""
    arr, n = _host_batches(batches)
    _check(lib().tk_matvec_host_noalloc(arr, n, int(getattr(stream, "cuda_stream", stream))))


def matvec_host(batches):
    """tk_matvec on numpy int16 host arrays (synchronous; same shapes as matvec)."""
    items = []
    for k, A, s, e, out in batches:
        n = _host_arr(s) // k
        if _host_arr(A) != n * k * k or _host_arr(out) != n * k or (
                e is not None and _host_arr(e) != n * k):
            raise ValueError("inconsistent matvec batch shapes")
        items.append(MatvecBatch(k, n, A.ctypes.data, s.ctypes.data,
                                 e.ctypes.data if e is not None else None, out.ctypes.data))
    arr = (MatvecBatch * len(items))(*items)
    _check(lib().tk_matvec_host(arr, len(items)))


class Server:
    """Continuous-batching server for matrix-vector requests (tk_server_*).

    Requests are numpy int16 arrays in host memory: A (njobs, k, k, 256),
    s / e (njobs, k, 256), out (njobs, k, 256); they must stay alive until the
    request completes (the object keeps references until release).  With
    zero_copy, arrays in page-locked memory (e.g. torch.empty(...,
    pin_memory=True).numpy()) are read and written in place by the device loop;
    everything else is staged through the server's HBM pool."""

    def __init__(self, hbm_budget_bytes=1 << 30, max_inflight_requests=1024,
                 idle_exit_seconds=0.02, device=0, zero_copy=False):
        cfg = ServerConfig(hbm_budget_bytes, max_inflight_requests, idle_exit_seconds,
                           int(zero_copy))
        h = ctypes.c_void_p()
        _check(lib().tk_server_create(device, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, k, A, s, e, out) -> int:
        n = _host_arr(s) // k
        if _host_arr(A) != n * k * k or _host_arr(out) != n * k or (
                e is not None and _host_arr(e) != n * k):
            raise ValueError("inconsistent request shapes")
        t = ctypes.c_uint64()
        _check(lib().tk_server_submit(self._h, k, n, A.ctypes.data, s.ctypes.data,
                                      e.ctypes.data if e is not None else None,
                                      out.ctypes.data, ctypes.byref(t)))
        self._keep[t.value] = (A, s, e, out)
        return t.value

    def wait(self, ticket: int, timeout: float = 30.0) -> None:
        _check(lib().tk_server_wait(self._h, ticket, timeout))

    def latency(self, ticket: int):
        done, lat = ctypes.c_int(), ctypes.c_double()
        _check(lib().tk_server_query(self._h, ticket, ctypes.byref(done), ctypes.byref(lat)))
        return lat.value if done.value else None

    def release(self, ticket: int) -> None:
        _check(lib().tk_server_release(self._h, ticket))
        self._keep.pop(ticket, None)

    def stats(self):
        c = ServerCounters()
        _check(lib().tk_server_stats(self._h, ctypes.byref(c)))
        return {n: getattr(c, n) for n, _ in ServerCounters._fields_}

    def close(self, timeout: float = 60.0) -> None:
        if self._h:
            rc = lib().tk_server_destroy(self._h, timeout)
            self._h = None
            self._keep.clear()
            _check(rc)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# Options (tk_set_option): the pipeline mode's chunk in vector polynomials,
# the host path's largest chunk in polynomials, and the matrix-vector mode:
# MATVEC_TILED (the default: one kernel, a CTA per tile of 8-16 jobs),
# MATVEC_PIPELINE (NTT, basemul-accumulate, iNTT + e as three kernels per
# chunk) or MATVEC_FUSED (one kernel, one warp per job).
OPT_MATVEC_CHUNK_POLYS = 1
OPT_HOST_CHUNK_POLYS = 3
OPT_MATVEC_MODE = 2
MATVEC_PIPELINE, MATVEC_FUSED, MATVEC_TILED = 0, 1, 2


def set_option(option: int, value: int) -> None:
    _check(lib().tk_set_option(option, value))


def get_option(option: int) -> int:
    return lib().tk_get_option(option)


FORWARD, INVERSE = 0, 1


def variant_count() -> int:
    return lib().tk_variant_count()


def variant_name(v: int) -> str:
    return lib().tk_variant_name(v).decode()


def set_variant(direction: int, variant: int) -> None:
    """Force a kernel variant for a direction (-1: automatic choice)."""
    _check(lib().tk_set_variant(direction, variant))


def get_variant(direction: int, npoly: int) -> int:
    return lib().tk_get_variant(direction, npoly)


def autotune(max_npoly: int = 1 << 20, device: int = 0, cache_path: str | None = None) -> None:
    """Pick the fastest kernel variant per direction and power-of-two size."""
    _check(lib().tk_autotune(device, max_npoly, cache_path.encode() if cache_path else None))


def autotune_reset() -> None:
    lib().tk_autotune_reset()


def init(device: int = 0) -> None:
    _check(lib().tk_init(device))


def device_status(device: int = 0) -> int:
    flags = ctypes.c_uint(0)
    rc = lib().tk_device_status(device, ctypes.byref(flags))
    if rc not in (0, 7):
        _check(rc)
    return int(flags.value)
