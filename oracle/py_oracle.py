"""ctypes access to the CPU parity checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
arm import this module.  The shipped library never does.

* ``Oracle``      -- liboracle.so, this repo's restatement of the pqcrystals
                     reference (oracle/tk_oracle.c, citing ntt_bench/ref/*.c).
* ``RefKyber``    -- oracle/_ref/libkyber_ref.so, the reference's own
                     ntt_bench/ref/{ntt,reduce}.c compiled unmodified.  Present
                     only where the reference sources were available at build
                     time (or the built file travelled with the checkout).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
Q = 3329
N = 256

_build_lock = threading.Lock()


def _ensure_built(path: str, target: str) -> None:
    src = os.path.join(HERE, "tk_oracle.c")
    stale = not os.path.exists(path) or (
        target == "liboracle.so" and os.path.getmtime(path) < os.path.getmtime(src))
    if stale:
        with _build_lock:
            subprocess.run(["make", "-s", "-C", HERE, target], check=True,
                           stdout=subprocess.DEVNULL)


def canon(a: np.ndarray) -> np.ndarray:
    """Canonical residue in [0, q) of any integer array, as int16."""
    return np.mod(np.asarray(a, dtype=np.int64), Q).astype(np.int16)


_I16P = ctypes.POINTER(ctypes.c_int16)
POLY_FN = ctypes.CFUNCTYPE(None, _I16P)


def _ptr(a: np.ndarray):
    assert a.dtype == np.int16 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_I16P)


class Oracle:
    """This repo's C restatement (oracle/tk_oracle.c)."""

    def __init__(self) -> None:
        path = os.path.join(HERE, "liboracle.so")
        _ensure_built(path, "liboracle.so")
        L = ctypes.CDLL(path)
        L.tko_init.restype = None
        L.tko_init()
        for name in ("tko_ntt", "tko_invntt"):
            getattr(L, name).argtypes = [_I16P]
            getattr(L, name).restype = None
        for name in ("tko_ntt_batch", "tko_invntt_batch"):
            getattr(L, name).argtypes = [_I16P, ctypes.c_size_t]
            getattr(L, name).restype = None
        L.tko_basemul.argtypes = [_I16P, _I16P, _I16P, ctypes.c_int16]
        L.tko_poly_basemul.argtypes = [_I16P, _I16P, _I16P]
        L.tko_matvec_job.argtypes = [ctypes.c_int, _I16P, _I16P, _I16P, _I16P]
        L.tko_pack_small.argtypes = [ctypes.c_int, _I16P, ctypes.c_void_p]
        L.tko_pack_small.restype = ctypes.c_size_t
        L.tko_unpack_small.argtypes = [ctypes.c_int, ctypes.c_void_p, _I16P]
        L.tko_montgomery_reduce.argtypes = [ctypes.c_int32]
        L.tko_montgomery_reduce.restype = ctypes.c_int16
        L.tko_barrett_reduce.argtypes = [ctypes.c_int16]
        L.tko_barrett_reduce.restype = ctypes.c_int16
        L.tko_time_roundtrip.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _I16P,
                                         ctypes.c_size_t, ctypes.c_int, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_uint64)]
        L.tko_time_roundtrip.restype = ctypes.c_double
        L.tko_split_roundtrip.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _I16P,
                                          ctypes.c_size_t, ctypes.c_int]
        L.tko_split_roundtrip.restype = ctypes.c_double
        self.lib = L
        self.zetas = np.ctypeslib.as_array(
            (ctypes.c_int16 * 128).in_dll(L, "tko_zetas")).copy()

    # batched transforms on copies -------------------------------------------
    def ntt(self, polys: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(polys, dtype=np.int16).copy()
        self.lib.tko_ntt_batch(_ptr(out), out.size // N)
        return out

    def invntt(self, polys: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(polys, dtype=np.int16).copy()
        self.lib.tko_invntt_batch(_ptr(out), out.size // N)
        return out

    def poly_basemul(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.int16)
        b = np.ascontiguousarray(b, dtype=np.int16)
        r = np.zeros(N, dtype=np.int16)
        self.lib.tko_poly_basemul(_ptr(r), _ptr(a), _ptr(b))
        return r

    def matvec_job(self, k: int, A: np.ndarray, s: np.ndarray, e: np.ndarray) -> np.ndarray:
        A = np.ascontiguousarray(A, dtype=np.int16).reshape(k * k, N)
        s = np.ascontiguousarray(s, dtype=np.int16).reshape(k, N)
        e = np.ascontiguousarray(e, dtype=np.int16).reshape(k, N)
        out = np.zeros((k, N), dtype=np.int16)
        self.lib.tko_matvec_job(k, _ptr(A), _ptr(s), _ptr(e), _ptr(out))
        return out

    def pack_small(self, bits: int, polys: np.ndarray) -> np.ndarray:
        """(npoly, 256) small int16 -> (npoly, 256*bits/8 rounded) packed bytes."""
        p = np.ascontiguousarray(polys, dtype=np.int16).reshape(-1, 256)
        per = 8 // bits
        out = np.zeros((p.shape[0], (256 + per - 1) // per), dtype=np.uint8)
        for i in range(p.shape[0]):
            self.lib.tko_pack_small(bits, _ptr(p[i]), out[i].ctypes.data)
        return out

    def unpack_small(self, bits: int, packed: np.ndarray) -> np.ndarray:
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        out = np.zeros((pk.shape[0], 256), dtype=np.int16)
        for i in range(pk.shape[0]):
            self.lib.tko_unpack_small(bits, pk[i].ctypes.data, _ptr(out[i]))
        return out

    def fn(self, name: str) -> int:
        return ctypes.cast(getattr(self.lib, name), ctypes.c_void_p).value

    def time_roundtrip(self, fwd_addr: int, inv_addr: int, src: np.ndarray,
                       threads: int, min_seconds: float):
        src = np.ascontiguousarray(src, dtype=np.int16)
        done = ctypes.c_uint64(0)
        rate = self.lib.tko_time_roundtrip(fwd_addr, inv_addr, _ptr(src), src.size // N,
                                           threads, min_seconds, ctypes.byref(done))
        return rate, int(done.value)

    def split_roundtrip(self, fwd_addr: int, inv_addr: int, polys: np.ndarray,
                        threads: int) -> float:
        assert polys.dtype == np.int16 and polys.flags["C_CONTIGUOUS"]
        return self.lib.tko_split_roundtrip(fwd_addr, inv_addr, _ptr(polys),
                                            polys.size // N, threads)


class RefKyber:
    """The reference's own C NTT (ntt_bench/ref), compiled unmodified."""

    PATH = os.path.join(HERE, "_ref", "libkyber_ref.so")

    @classmethod
    def available(cls) -> bool:
        if not os.path.exists(cls.PATH):
            try:
                _ensure_built(cls.PATH, "ref")
            except Exception:
                return False
        return os.path.exists(cls.PATH)

    def __init__(self, k: int = 3) -> None:
        self.lib = ctypes.CDLL(self.PATH)
        self.prefix = {2: "pqcrystals_kyber512_ref_", 3: "pqcrystals_kyber768_ref_",
                       4: "pqcrystals_kyber1024_ref_"}[k]
        for n in ("ntt", "invntt"):
            f = getattr(self.lib, self.prefix + n)
            f.argtypes = [_I16P]
            f.restype = None
        f = getattr(self.lib, self.prefix + "basemul")
        f.argtypes = [_I16P, _I16P, _I16P, ctypes.c_int16]
        f.restype = None
        for n, at, rt in (("montgomery_reduce", ctypes.c_int32, ctypes.c_int16),
                          ("barrett_reduce", ctypes.c_int16, ctypes.c_int16)):
            f = getattr(self.lib, self.prefix + n)
            f.argtypes = [at]
            f.restype = rt
        self.zetas = np.ctypeslib.as_array(
            (ctypes.c_int16 * 128).in_dll(self.lib, self.prefix + "zetas")).copy()

    def _each(self, name: str, polys: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(polys, dtype=np.int16).copy().reshape(-1, N)
        f = getattr(self.lib, self.prefix + name)
        for i in range(out.shape[0]):
            f(_ptr(out[i]))
        return out.reshape(np.shape(polys))

    def ntt(self, polys: np.ndarray) -> np.ndarray:
        return self._each("ntt", polys)

    def invntt(self, polys: np.ndarray) -> np.ndarray:
        return self._each("invntt", polys)

    def basemul(self, a: np.ndarray, b: np.ndarray, zeta: int) -> np.ndarray:
        r = np.zeros(2, dtype=np.int16)
        a = np.ascontiguousarray(a, dtype=np.int16)
        b = np.ascontiguousarray(b, dtype=np.int16)
        getattr(self.lib, self.prefix + "basemul")(_ptr(r), _ptr(a), _ptr(b), int(zeta))
        return r

    def fn(self, name: str) -> int:
        return ctypes.cast(getattr(self.lib, self.prefix + name), ctypes.c_void_p).value
