"""CPU model of the kernels' basemul-accumulate arithmetic, checked against
the oracle's composition of the reference's basemul (ntt_bench/ref/ntt.c:139-146,
applied pairwise as ML-KEM's poly_basemul_montgomery):

* basemul_row (tk_stages.cuh, the pipeline's basemul kernel): three raw sums
  per pair, the pair constant z_t * 2^-16 applied after the sum;
* basemul_row_z with pair_zb (the tiled matrix-vector kernel): z_t folded
  into ntt(s) once per polynomial, two raw sums per pair, and 2^-16 left to
  the inverse tables that kernel uses (table 7);
* fused_job's products (tk_matvec.cu, the fused kernel and the server's
  device loop): 2^-16 and z_t both folded into ntt(s), lazily reduced, with
  the accumulator bias kAccBias.

Integer work, no GPU: every intermediate bound the kernels rely on is
asserted, on random and extreme inputs."""
import numpy as np
import pytest

import kernel_model as KM
from conftest import rng
from py_oracle import Q, canon

BAR_LAZY = 1290167            # floor(2^32 / q)
RINV = 169                    # 2^-16 mod q
SUM_BIAS = 3329 * 262144      # the raw sums' bias (>= their magnitude)


def brv7(x):
    return int(format(x, "07b")[::-1], 2)


def pair_roots():
    """z_t = 17^brv7(64 + t/2), negated for odd t."""
    z = np.zeros(128, dtype=np.int64)
    for t in range(128):
        w = pow(17, brv7(64 + t // 2), Q)
        z[t] = (-w) % Q if t & 1 else w
    return z


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


def test_red_wide_bounds():
    """red_wide on any uint32: the residue is kept and the representative lies
    in [0, 1.41 q) ([0, 1.21 q) below 2^31), random and top-of-range values,
    including every q j - 1 near 2^32."""
    top = 1 << 32
    s = np.concatenate([rng(9).integers(0, top, 1 << 20, dtype=np.int64),
                        np.arange(top - (1 << 20), top, dtype=np.int64),
                        Q * np.arange(top // Q - 4096, top // Q + 1, dtype=np.int64) - 1])
    s = s[(s >= 0) & (s < top)]
    r = s - ((s * BAR_LAZY) >> 32) * Q
    assert (r % Q == s % Q).all() and r.min() >= 0 and r.max() < 1.41 * Q
    low = s < (1 << 31)
    assert r[low].max() < 1.21 * Q


def test_pair_constants_match_library(tk):
    """The table the matrix-vector kernels upload is the one modelled here."""
    assert (tk.get_table(6).astype(np.int64) == pair_constants()).all()


SUM_BIAS_Z = 3329 << 19


def pair_zb_model(b, z):
    """b: (K, 256) in [0, q); returns z_t * b1 per pair, (K, 128), lazily reduced."""
    b1 = b.astype(np.int64).reshape(-1, 128, 2)[..., 1]
    zb = red_wide(b1 * z)
    assert zb.max() < Q + 4
    return zb


def basemul_row_z_model(a, b, zb):
    """2^16 * sum_j basemul(A_ij, b_j) mod q, values in [0, 1.41 q)."""
    a = a.astype(np.int64).reshape(-1, 128, 2)
    b = b.astype(np.int64).reshape(-1, 128, 2)
    assert b.min() >= 0 and b.max() < Q
    t0 = (a[..., 0] * b[..., 0] + a[..., 1] * zb).sum(0)
    t1 = (a[..., 0] * b[..., 1] + a[..., 1] * b[..., 0]).sum(0)
    out = []
    for t in (t0, t1):
        assert np.abs(t).max() <= SUM_BIAS_Z
        s = t + SUM_BIAS_Z
        assert s.min() >= 0 and s.max() < (1 << 32)        # uint32 accumulator
        r = s - ((s * BAR_LAZY) >> 32) * Q
        assert r.min() >= 0 and r.max() < 4682                # [0, 1.41 q)
        out.append(r)
    return np.stack(out, axis=1).reshape(256)


def test_pair_roots_match_library(tk):
    assert (pair_roots() * RINV % Q == tk.get_table(6)).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_basemul_row_z_model_matches_oracle(oracle, k):
    z = pair_roots()
    r = rng(500 + k)
    for trial in range(20):
        A = r.integers(-32768, 32768, size=(k, k, 256)).astype(np.int16)
        b = r.integers(0, Q, size=(k, 256)).astype(np.int16)
        zb = pair_zb_model(b, z)
        for i in range(k):
            ref = np.zeros(256, dtype=np.int64)
            for j in range(k):
                ref += oracle.poly_basemul(A[i, j], b[j]).astype(np.int64)
            got = basemul_row_z_model(A[i], b, zb) * RINV
            assert (canon(got) == canon(ref)).all(), (trial, i)


@pytest.mark.parametrize("aval", [-32768, 32767])
@pytest.mark.parametrize("bval", [Q - 1, 0, 1])
def test_basemul_row_z_model_extremes(oracle, aval, bval):
    """k = 4, every A coefficient at an int16 extreme, ntt(s) constant: the
    raw sums reach their largest magnitude."""
    k = 4
    z = pair_roots()
    A = np.full((k, k, 256), aval, dtype=np.int16)
    A[:, :, 1::2] = -1 - aval if bval == 0 else aval        # a1 of the other sign too
    b = np.full((k, 256), bval, dtype=np.int16)
    b[:, 1::2] = Q - 1
    zb = pair_zb_model(b, z)
    ref = np.zeros(256, dtype=np.int64)
    for j in range(k):
        ref += oracle.poly_basemul(A[0, j], b[j]).astype(np.int64)
    assert (canon(basemul_row_z_model(A[0], b, zb) * RINV) == canon(ref)).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_tiled_job_model_matches_oracle(tk, oracle, k):
    """One job of the tiled kernel on the CPU: the forward model on the
    library's tables, basemul_row_z, the inverse model on table 7 (stage B
    scaled by 2^-16, bias folded into its init), then + e with int16
    wrap-around, against the oracle's job."""
    fw = KM.FwdModel(tk.get_table(4))
    iv = KM.InvModel(tk.get_table(7))
    z = pair_roots()
    r = rng(600 + k)
    for trial in range(4):
        A = r.integers(-32768, 32768, size=(k, k, 256)).astype(np.int16)
        s = r.integers(-3, 4, size=(k, 256)).astype(np.int16)
        e = r.integers(-3, 4, size=(k, 256)).astype(np.int16)
        b = fw(s)
        zb = pair_zb_model(b, z)
        acc = np.stack([basemul_row_z_model(A[i], b, zb) for i in range(k)]).astype(np.int16)
        v = iv(acc, fold=True)
        out = (v.astype(np.int64) + e).astype(np.int16)
        assert (canon(out) == canon(oracle.matvec_job(k, A, s, e))).all(), trial


ACC_BIAS = 1073742318          # q * ceil(2^30 / q)


def fused_job_basemul_model(a, b, zr):
    """fused_job step 4 for one output row: B0 = b0 * 2^-16, B1 = b1 * 2^-16,
    Bz = b1 * z_t 2^-16, each lazily reduced (mulmod_lazy); int32 accumulators
    biased by kAccBias, reduced once.  Equals the reference's basemul sum mod q."""
    b = b.astype(np.int64).reshape(-1, 128, 2)
    a = a.astype(np.int64).reshape(-1, 128, 2)
    assert b.min() >= 0 and b.max() < Q              # forward stage 2 output

    def lazy(x):                                        # red_lazy, x < 2^24
        assert x.min() >= 0 and x.max() < (1 << 24)
        r = x - ((x * BAR_LAZY) >> 32) * Q
        assert r.max() < Q + 8
        return r
    B0, B1, Bz = lazy(b[..., 0] * RINV), lazy(b[..., 1] * RINV), lazy(b[..., 1] * zr)
    acc0 = (a[..., 0] * B0 + a[..., 1] * Bz).sum(0)
    acc1 = (a[..., 0] * B1 + a[..., 1] * B0).sum(0)
    out = []
    for acc in (acc0, acc1):
        assert np.abs(acc).max() < (1 << 31) and np.abs(acc).max() <= ACC_BIAS
        s = acc + ACC_BIAS
        assert s.min() >= 0 and s.max() < (1 << 31)
        out.append(red_wide(s))
    r = np.stack(out, axis=1).reshape(256)
    assert r.max() < (1 << 15)                          # int16 row for the inverse
    return r


@pytest.mark.parametrize("k", [2, 3, 4])
def test_fused_job_basemul_model_matches_oracle(oracle, k):
    zr = pair_constants()
    r = rng(700 + k)
    for trial in range(10):
        A = r.integers(-32768, 32768, size=(k, k, 256)).astype(np.int16)
        b = r.integers(0, Q, size=(k, 256)).astype(np.int16)
        for i in range(k):
            ref = np.zeros(256, dtype=np.int64)
            for j in range(k):
                ref += oracle.poly_basemul(A[i, j], b[j]).astype(np.int64)
            assert (canon(fused_job_basemul_model(A[i], b, zr)) == canon(ref)).all(), (trial, i)


@pytest.mark.parametrize("aval", [-32768, 32767])
def test_fused_job_basemul_model_extremes(oracle, aval):
    """k = 4, A at an int16 extreme, ntt(s) chosen so every lazy product lands
    at the top of its range: the accumulators reach their largest magnitude."""
    k = 4
    zr = pair_constants()
    A = np.full((k, k, 256), aval, dtype=np.int16)
    v = np.arange(Q, dtype=np.int64)

    def lazy_argmax(c):                                  # the b maximising red_lazy(b * c)
        x = v * c
        return int(np.argmax(x - ((x * BAR_LAZY) >> 32) * Q))
    worst = np.zeros((k, 256), dtype=np.int16)
    worst[:, 0::2] = lazy_argmax(RINV)
    worst[:, 1::2] = [lazy_argmax(int(c)) for c in zr]
    ref = np.zeros(256, dtype=np.int64)
    for j in range(k):
        ref += oracle.poly_basemul(A[0, j], worst[j]).astype(np.int64)
    assert (canon(fused_job_basemul_model(A[0], worst, zr)) == canon(ref)).all()


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
