"""Pins the oracle (oracle/tk_oracle.c) before anything is checked against it.

* byte-for-byte against the committed fixtures made by the reference's own C
  (tests/golden/gen_golden.py runs ntt_bench/ref/{ntt,reduce}.c);
* byte-for-byte against that reference build itself when it is present
  (oracle/_ref, built from the reference sources);
* algebraic properties of the ring transform.
"""
import os

import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_vectors.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_zetas_match_reference_table(oracle, gold):
    assert (oracle.zetas == gold["zetas"]).all()
    assert oracle.zetas.min() >= -(Q // 2) and oracle.zetas.max() <= Q // 2


@pytest.mark.parametrize("name", ["uniform", "ternary", "edge"])
def test_golden_vectors_bit_exact(oracle, gold, name):
    x = gold[name + "_in"]
    assert (oracle.ntt(x) == gold[name + "_ntt"]).all()
    assert (oracle.invntt(x) == gold[name + "_invntt"]).all()
    assert (oracle.invntt(oracle.ntt(x)) == gold[name + "_roundtrip"]).all()


def test_golden_basemul(oracle, gold):
    import ctypes
    import py_oracle
    a, b, z, r = gold["basemul_a"], gold["basemul_b"], gold["basemul_zeta"], gold["basemul_r"]
    L = oracle.lib
    for i in range(len(a)):
        out = np.zeros(2, dtype=np.int16)
        ai = np.ascontiguousarray(a[i])
        bi = np.ascontiguousarray(b[i])
        L.tko_basemul(py_oracle._ptr(out), py_oracle._ptr(ai), py_oracle._ptr(bi),
                      ctypes.c_int16(int(z[i])))
        assert (out == r[i]).all(), i


def test_against_reference_build(oracle, ref_kyber):
    r = rng(1)
    for lo, hi in ((0, Q), (-3, 4), (-9471, 9472)):
        x = r.integers(lo, hi, size=(600, 256)).astype(np.int16)
        assert (oracle.ntt(x) == ref_kyber.ntt(x)).all()
    for lo, hi in ((0, Q), (-16384, 16384)):
        x = r.integers(lo, hi, size=(600, 256)).astype(np.int16)
        assert (oracle.invntt(x) == ref_kyber.invntt(x)).all()


def test_scalar_reductions_against_reference(oracle, ref_kyber):
    L, R, p = oracle.lib, ref_kyber.lib, ref_kyber.prefix
    r = rng(2)
    lim = Q * (1 << 15)
    vals = np.concatenate([r.integers(-lim, lim, 20000), [-lim, lim - 1, 0, 1, -1]])
    for v in vals:
        assert L.tko_montgomery_reduce(int(v)) == getattr(R, p + "montgomery_reduce")(int(v))
    for v in list(range(-32768, 32768, 7)) + [32767]:
        assert L.tko_barrett_reduce(v) == getattr(R, p + "barrett_reduce")(v)


def test_roundtrip_identity(oracle):
    """invntt(ntt(x)) == 2^16 * x (mod q): invntt carries the Montgomery factor."""
    x = rng(3).integers(-4000, 4000, size=(500, 256)).astype(np.int16)
    y = oracle.invntt(oracle.ntt(x))
    assert (canon(y) == canon(x.astype(np.int64) * 65536)).all()


def test_linearity(oracle):
    r = rng(4)
    a = r.integers(0, Q, size=(200, 256)).astype(np.int16)
    b = r.integers(0, Q, size=(200, 256)).astype(np.int16)
    s = canon(a.astype(np.int64) + b).astype(np.int16)
    assert (canon(oracle.ntt(s)) ==
            canon(oracle.ntt(a).astype(np.int64) + oracle.ntt(b))).all()


def negacyclic(a, b):
    out = np.zeros(256, dtype=np.int64)
    for i in range(256):
        for j in range(256):
            k = i + j
            if k < 256:
                out[k] += int(a[i]) * int(b[j])
            else:
                out[k - 256] -= int(a[i]) * int(b[j])
    return canon(out)


def test_basemul_is_negacyclic_product(oracle):
    """invntt(basemul(ntt(a), ntt(b))) == a*b in Z_q[x]/(x^256+1): the
    Montgomery factor 2^-16 of basemul cancels the 2^16 of invntt."""
    r = rng(5)
    for _ in range(3):
        a = r.integers(-3, 4, size=256).astype(np.int16)
        b = r.integers(0, Q, size=256).astype(np.int16)
        prod = oracle.poly_basemul(oracle.ntt(a[None])[0], oracle.ntt(b[None])[0])
        got = oracle.invntt(prod[None])[0]
        assert (canon(got) == negacyclic(a, b)).all()


def test_matvec_job_composition(oracle):
    """tko_matvec_job == its definition built from the single-poly pieces."""
    r = rng(6)
    for k in (2, 3, 4):
        A = r.integers(0, Q, size=(k * k, 256)).astype(np.int16)
        s = r.integers(-3, 4, size=(k, 256)).astype(np.int16)
        e = r.integers(-3, 4, size=(k, 256)).astype(np.int16)
        got = oracle.matvec_job(k, A, s, e)
        shat = oracle.ntt(s)
        for i in range(k):
            acc = np.zeros(256, dtype=np.int64)
            for j in range(k):
                acc += oracle.poly_basemul(A[i * k + j], shat[j])
            want = canon(oracle.invntt(canon(acc).astype(np.int16)[None])[0].astype(np.int64) + e[i])
            assert (canon(got[i]) == want).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_matvec_job_golden(oracle, gold, k):
    """tko_matvec_job, int16 for int16, against jobs that tests/golden/gen_golden.py
    composed from the reference's own ntt, basemul, barrett_reduce and invntt."""
    A, s, e, want = (gold[f"matvec{k}_{n}"] for n in ("A", "s", "e", "out"))
    for t in range(A.shape[0]):
        assert (oracle.matvec_job(k, A[t], s[t], e[t]) == want[t]).all(), t


def test_pack_small_format(oracle):
    """TC-PACK byte layout (ntt_bench/ntt_bench.cu:744-752): coefficient i in
    byte i/(8/bits), field at bit (i % (8/bits))*bits, two's complement."""
    x = np.zeros((1, 256), dtype=np.int16)
    x[0, :4] = [1, -1, 0, -2]
    p2 = oracle.pack_small(2, x)
    assert p2.shape == (1, 64) and p2[0, 0] == (1 | 3 << 2 | 0 << 4 | 2 << 6)
    x[0, :2] = [3, -4]
    p3 = oracle.pack_small(3, x)
    assert p3.shape == (1, 128) and p3[0, 0] == (3 | 4 << 3)


@pytest.mark.parametrize("bits,lo,hi", [(2, -2, 2), (3, -4, 4)])
def test_pack_unpack_roundtrip(oracle, bits, lo, hi):
    x = np.random.default_rng(bits).integers(lo, hi, size=(50, 256)).astype(np.int16)
    assert (oracle.unpack_small(bits, oracle.pack_small(bits, x)) == x).all()
