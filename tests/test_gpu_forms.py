"""GPU parity of the forward input forms: small int16 (single-limb stage 1,
tk_ntt_small) and packed 2/3-bit fields (tk_ntt_packed), against the oracle's
ntt and against tk_ntt on the same polynomials.  Integer work: bit-exact."""
import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

pytestmark = pytest.mark.gpu


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("npoly", [1, 7, 8, 33, 257, 4096, 100003])
def test_small_matches_oracle_and_tk_ntt(tk, cuda, oracle, npoly):
    x = rng(npoly).integers(-128, 128, size=(npoly, 256)).astype(np.int16)
    x[0, :2] = (-128, 127)
    d = dev(x)
    out = d.clone()
    tk.ntt_small(d, out)
    full = d.clone()
    tk.ntt(full)
    got = out.cpu().numpy()
    assert (got == full.cpu().numpy()).all()
    assert got.min() >= 0 and got.max() < Q
    k = min(npoly, 512)
    assert (got[:k] == canon(oracle.ntt(x[:k]))).all()
    tk.ntt_small(d)                                   # in place
    assert (d.cpu().numpy() == got).all()
    assert tk.device_status(0) == 0


def test_small_golden_ternary(tk, cuda, golden):
    d = dev(golden["ternary_in"])
    tk.ntt_small(d)
    assert (d.cpu().numpy() == canon(golden["ternary_ntt"])).all()


def test_small_range_flag(tk, cuda):
    for bad in (128, -129, 3328, -32768):
        x = np.zeros((40, 256), dtype=np.int16)
        x[37, 200] = bad
        tk.ntt_small(dev(x))
        assert tk.device_status(0) == tk.FLAG_SMALL_RANGE, bad
    tk.ntt_small(dev(np.full((40, 256), -128, dtype=np.int16)))
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("bits,lo,hi", [(2, -2, 2), (3, -4, 4)])
@pytest.mark.parametrize("npoly", [1, 9, 32, 1000, 65537])
def test_packed_matches_tk_ntt(tk, cuda, oracle, bits, lo, hi, npoly):
    x = rng(bits * npoly).integers(lo, hi, size=(npoly, 256)).astype(np.int16)
    pk = tk.pack_small(x, bits)
    k = min(npoly, 64)
    assert (pk[:k] == oracle.pack_small(bits, x[:k])).all()
    got = tk.ntt_packed(dev(pk), bits).cpu().numpy()
    full = dev(x)
    tk.ntt(full)
    assert (got == full.cpu().numpy()).all()
    assert (got[:k] == canon(oracle.ntt(x[:k]))).all()


def test_packed_golden_ternary(tk, cuda, golden, oracle):
    """The reference's packed-ternary input (seed 20240819 + 2*10) through the
    packed path equals the reference ntt's output mod q."""
    pk = oracle.pack_small(2, golden["ternary_in"])
    got = tk.ntt_packed(dev(pk), 2).cpu().numpy()
    assert (got == canon(golden["ternary_ntt"])).all()


def test_packed_errors(tk, cuda):
    import torch
    pk = torch.zeros((4, 64), dtype=torch.uint8, device="cuda")
    out = torch.empty((4, 256), dtype=torch.int16, device="cuda")
    L = tk.lib()
    assert L.tk_ntt_packed(pk.data_ptr(), 4, out.data_ptr(), 4, None) == 1
    assert L.tk_ntt_packed(pk.data_ptr() + 4, 2, out.data_ptr(), 4, None) == 2
    assert L.tk_ntt_packed(out.data_ptr(), 2, out.data_ptr(), 4, None) == 1   # overlap
