"""CPU checks of the host matrix builder and of the kernels' integer arithmetic.

The logical matrices must compose to the oracle's transforms mod q, and the
per-lane fragment tables, pushed through a bit-level model of the kernels'
byte-operand MMAs, recombination and Barrett steps (tests/kernel_model.py),
must reproduce the oracle on every coefficient, including the full int16 input
range and the stated representatives.  No GPU is involved.
"""
import numpy as np
import pytest

import kernel_model as KM
from conftest import rng
from py_oracle import Q, canon


@pytest.fixture(scope="module")
def mats(tk):
    return {i: tk.get_table(i).astype(np.int64) for i in range(4)}


def apply_fwd(m, x):
    x = canon(x).astype(np.int64).reshape(-1, 16, 16)          # [p][m][c]
    y = np.einsum("im,pmc->pic", m[0], x) % Q                   # stage 1
    z = np.einsum("bjc,pbc->pbj", m[1], y) % Q                  # stage 2, per block
    return z.reshape(-1, 256)


def apply_inv(m, x):
    x = canon(x).astype(np.int64).reshape(-1, 16, 16)
    y = np.einsum("bjc,pbc->pbj", m[2], x) % Q                  # stage A, per block
    z = np.einsum("im,pmc->pic", m[3], y) % Q                   # stage B
    return z.reshape(-1, 256)


def test_matrix_shapes_and_range(mats):
    for i, m in mats.items():
        assert m.min() >= 0 and m.max() < Q
    # layers 5-7 never mix even and odd positions of a block
    for key in (1, 2):
        m = mats[key]
        for cp in range(16):
            for c in range(16):
                if (cp ^ c) & 1:
                    assert (m[:, cp, c] == 0).all()


def test_logical_matrices_compose_to_oracle(mats, oracle):
    x = rng(1).integers(-5000, 5000, size=(300, 256)).astype(np.int16)
    assert (apply_fwd(mats, x) == canon(oracle.ntt(x))).all()
    assert (apply_inv(mats, x) == canon(oracle.invntt(x))).all()


@pytest.mark.parametrize("wide", [False, True], ids=["int16-mid", "int32-mid"])
@pytest.mark.parametrize("lo,hi", [(0, Q), (-3, 4), (-32768, 32768)])
def test_kernel_arithmetic_model(tk, oracle, lo, hi, wide):
    fw = KM.FwdModel(tk.get_table(4))
    iv = KM.InvModel(tk.get_table(5))
    x = rng(hi).integers(lo, hi, size=(200, 256)).astype(np.int16)
    ref_in = canon(x).astype(np.int16)        # the oracle overflows outside |x| < 9471
    f = fw(x, wide=wide)
    assert f.min() >= 0 and f.max() < Q
    assert (f == canon(oracle.ntt(ref_in))).all()
    v = iv(x, wide=wide, fold=True)
    assert v.min() >= -(Q // 2) and v.max() <= Q // 2
    assert (canon(v) == canon(oracle.invntt(ref_in))).all()
    v = iv(x, wide=wide)
    assert v.min() >= -(Q // 2) and v.max() <= Q // 2
    assert (canon(v) == canon(oracle.invntt(ref_in))).all()


@pytest.mark.parametrize("wide", [False, True], ids=["int16-mid", "int32-mid"])
def test_kernel_model_extreme_rows(tk, oracle, wide):
    fw = KM.FwdModel(tk.get_table(4))
    iv = KM.InvModel(tk.get_table(5))
    x = np.array([[-32768] * 256, [32767] * 256, [Q - 1] * 256, [0] * 256,
                  np.tile([32767, -32768], 128)], dtype=np.int16)
    ref_in = canon(x).astype(np.int16)
    assert (fw(x, wide=wide) == canon(oracle.ntt(ref_in))).all()
    assert (canon(iv(x, wide=wide)) == canon(oracle.invntt(ref_in))).all()
    assert (canon(iv(x, wide=wide, fold=True)) == canon(oracle.invntt(ref_in))).all()


@pytest.mark.parametrize("wide", [False, True], ids=["int16-mid", "int32-mid"])
@pytest.mark.parametrize("lo,hi", [(-128, 128), (-3, 4), (-1, 2)])
def test_single_limb_stage1_model(tk, oracle, lo, hi, wide):
    """The single-limb stage-1 fragments (inputs in [-128, 127]) give the same
    transform as the reference's ntt, extremes included."""
    fw = KM.FwdModel(tk.get_table(4))
    x = rng(7 + hi).integers(lo, hi, size=(200, 256)).astype(np.int16)
    x[0], x[1] = lo, hi - 1
    assert (fw(x, single_limb=True, wide=wide) == canon(oracle.ntt(x))).all()


def test_lazy_reduction_bound():
    """red_lazy (S - umulhi(S, floor(2^32 / q)) q) on its whole documented
    domain, checked on its extremes and a random sample: congruent to S, in
    [0, q + 11) for S < 2^25 (the top of the range reaches q + 10) and in
    [0, q + 6) for S < 2^24; the high byte is at most 13 either way."""
    M = (1 << 32) // Q
    r = rng(7)
    for top, bound in ((1 << 25, Q + 11), (1 << 24, Q + 6)):
        s = np.concatenate([np.arange(0, 1 << 18), np.arange(top - (1 << 20), top),
                            r.integers(0, top, size=1 << 20)]).astype(np.int64)
        v = s - ((s * M) >> 32) * Q
        assert v.min() >= 0 and v.max() < bound and ((v - s) % Q == 0).all()
        assert v.max() >> 8 <= 13
    # the error term: when the quotient is one short, S mod q < S e / 2^32
    # with e = 2^32 - q M
    e = (1 << 32) - Q * M
    assert (1 << 25) * e < 11 * (1 << 32) and (1 << 24) * e < 6 * (1 << 32)
