"""CPU model of the kernels' basemul-accumulate arithmetic (basemul_row in
tk_stages.cuh, used by the tiled matrix-vector kernel and the pipeline's
basemul kernel), checked against the oracle's composition of the reference's
basemul (ntt_bench/ref/ntt.c:139-146, applied pairwise as ML-KEM's
poly_basemul_montgomery).  Integer work, no GPU: every intermediate bound the
kernels rely on is asserted, on random and extreme inputs."""
import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

BAR_LAZY = 1290167            # floor(2^32 / q)
RINV = 169                    # 2^-16 mod q
SUM_BIAS = 3329 * 262144      # the raw sums' bias (>= their magnitude)


def brv7(x):
    return int(format(x, "07b")[::-1], 2)


def pair_constants():
    """z_t * 2^-16 mod q for pair t: z_t = 17^brv7(64 + t/2), negated for odd t."""
    zr = np.zeros(128, dtype=np.int64)
    for t in range(128):
        z = pow(17, brv7(64 + t // 2), Q)
        if t & 1:
            z = (-z) % Q
        zr[t] = z * RINV % Q
    return zr


def red_wide(x):
    assert x.min() >= 0 and x.max() < (1 << 31)
    return x - ((x * BAR_LAZY) >> 32) * Q


def basemul_row_model(a, b, zr):
    """a: (K, 256) int16 (row i of A), b: (K, 256) int16 in [0, q) (ntt(s)).
    Returns the kernel's output polynomial (values in [0, 3q))."""
    a = a.astype(np.int64).reshape(-1, 128, 2)
    b = b.astype(np.int64).reshape(-1, 128, 2)
    assert b.min() >= 0 and b.max() < Q
    a0, a1, b0, b1 = a[..., 0], a[..., 1], b[..., 0], b[..., 1]
    t00 = (a0 * b0).sum(0)
    t11 = (a1 * b1).sum(0)
    t1 = (a0 * b1 + a1 * b0).sum(0)
    for t in (t00, t11, t1):            # int32 accumulators, then the bias
        assert np.abs(t).max() <= SUM_BIAS
    r00, r11, r1 = (red_wide(t + SUM_BIAS) for t in (t00, t11, t1))
    assert max(r00.max(), r11.max(), r1.max()) < 3 * Q
    out0 = red_wide(r00 * RINV + r11 * zr)
    out1 = red_wide(r1 * RINV)
    out = np.stack([out0, out1], axis=1).reshape(256)
    assert out.min() >= 0 and out.max() < 3 * Q       # fits the int16 rows
    return out


def test_pair_constants_match_library(tk):
    """The table the matrix-vector kernels upload is the one modelled here."""
    assert (tk.get_table(6).astype(np.int64) == pair_constants()).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_basemul_row_model_matches_oracle(oracle, k):
    zr = pair_constants()
    r = rng(400 + k)
    for trial in range(20):
        A = r.integers(-32768, 32768, size=(k, k, 256)).astype(np.int16)
        b = r.integers(0, Q, size=(k, 256)).astype(np.int16)
        for i in range(k):
            ref = np.zeros(256, dtype=np.int64)
            for j in range(k):
                ref += oracle.poly_basemul(A[i, j], b[j]).astype(np.int64)
            assert (canon(basemul_row_model(A[i], b, zr)) == canon(ref)).all(), (trial, i)


@pytest.mark.parametrize("aval", [-32768, 32767, Q - 1, -(Q - 1)])
def test_basemul_row_model_extremes(oracle, aval):
    """k = 4 with every A coefficient at an extreme and ntt(s) at q - 1: the
    raw sums reach their largest magnitude (|sum| <= 8 * 32768 * (q-1), just
    under the bias)."""
    k = 4
    zr = pair_constants()
    A = np.full((k, k, 256), aval, dtype=np.int16)
    b = np.full((k, 256), Q - 1, dtype=np.int16)
    ref = np.zeros(256, dtype=np.int64)
    for j in range(k):
        ref += oracle.poly_basemul(A[0, j], b[j]).astype(np.int64)
    assert (canon(basemul_row_model(A[0], b, zr)) == canon(ref)).all()
