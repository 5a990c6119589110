"""tk_matvec_host_noalloc: tk_matvec_host staged in the library's static
device array instead of memory allocated per call, for callers that reserve
their device memory up front or cannot pay for cudaMalloc / cudaFree on a
latency-bound path.  Collected last, so it also runs after every other test
has used the library in the same process.

Outputs are compared with the oracle's composition of the reference's ntt,
basemul and invntt (tko_matvec_job), every coefficient, mod q."""
import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

# A batch list that needs exactly the 4 MiB static scratch: staging per job is
# A + s + e + out = (k*k + 3k) * 512 bytes with e, (k*k + 2k) * 512 without,
# so 37 jobs of k = 4 with e (14,336 B each), 791 jobs of k = 2 without e
# (4,096 B each) and 46 jobs of k = 3 with e (9,216 B each) add up to
# 512 * (1036 + 6328 + 828) = 4,194,304 bytes.  Every batch is a multiple of
# 256 bytes (no rounding), the k = 3 / 4 batches end in partial tiles of the
# tiled kernel (8 jobs per tile), the k = 2 one too (16 per tile), and the
# last batch ends at the scratch's last byte.
EXACT_FIT = ((4, 37, True), (2, 791, False), (3, 46, True))


def staging_bytes(spec):
    total = 0
    for k, n, with_e in spec:
        b = n * (k * k + (3 if with_e else 2) * k) * 512
        total += (b + 255) // 256 * 256
    return total


def jobs(seed, k, n, with_e=True):
    r = rng(seed)
    A = r.integers(0, Q, size=(n, k, k, 256)).astype(np.int16)
    s = r.integers(-32768, 32768, size=(n, k, 256)).astype(np.int16)
    # e is added to the inverse's output with int16 wrap-around (as the
    # reference's polynomial add): noise-sized, so neither side's sum wraps
    e = r.integers(-3, 4, size=(n, k, 256)).astype(np.int16) if with_e else None
    return A, s, e


def oracle_out(oracle, k, A, s, e):
    # the oracle's ntt overflows int16 outside |x| <= 9471: feed it canon(s)
    s_c = canon(s).astype(np.int16)
    return np.stack([oracle.matvec_job(k, A[t].reshape(k * k, 256), s_c[t],
                                       e[t] if e is not None else np.zeros_like(s[t]))
                     for t in range(A.shape[0])])


def make_list(seed, spec):
    items = []
    for i, (k, n, with_e) in enumerate(spec):
        A, s, e = jobs(seed + i, k, n, with_e)
        items.append((k, A, s, e, np.zeros_like(s)))
    return items


def test_exact_fit_spec_fills_the_scratch(tk):
    assert staging_bytes(EXACT_FIT) == tk.NOALLOC_SCRATCH_BYTES == 4 << 20


def test_rejects_lists_above_the_static_scratch(tk):
    """Checked before any device work (no GPU needed)."""
    k, n = 4, 300                       # 300 * 14 KiB > 4 MiB
    A, s, e = jobs(1, k, n)
    with pytest.raises(tk.TKError) as ex:
        tk.matvec_host_noalloc([(k, A, s, e, np.zeros_like(s))])
    assert ex.value.status == 3 and "static scratch" in str(ex.value)


def test_rejects_one_job_past_an_exact_fit(tk):
    """The exact-fit list plus one job of k = 2 (4 KiB more): refused before
    any device work, with the size in the message."""
    spec = list(EXACT_FIT)
    spec[1] = (2, 792, False)
    assert staging_bytes(spec) == (4 << 20) + 4096
    with pytest.raises(tk.TKError) as ex:
        tk.matvec_host_noalloc(make_list(5, spec))
    assert ex.value.status == 3 and str((4 << 20) + 4096) in str(ex.value)


def test_rejects_more_than_16_batches_before_device_work(tk):
    items = make_list(9, [(2, 1, False)] * 17)
    with pytest.raises(tk.TKError) as ex:
        tk.matvec_host_noalloc(items)
    assert ex.value.status == 1 and "16 batches" in str(ex.value)


@pytest.mark.gpu
def test_two_calls_in_a_row_match_the_oracle(tk, cuda, oracle):
    """Two calls back to back on one stream with different data (the second
    reuses the array the first left filled), small mixed lists with e."""
    import torch
    stream = torch.cuda.Stream()
    for call in range(2):
        items = make_list(100 * call, ((2, 17, True), (3, 40, True), (4, 64, True)))
        tk.matvec_host_noalloc(items, stream=stream)
        for k, A, s, e, out in items:
            assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all(), (call, k)
    assert tk.device_status(0) == 0


@pytest.mark.gpu
def test_exact_fit_list_twice_matches_the_oracle(tk, cuda, oracle):
    """The list that fills the 4 MiB scratch to its last byte (partial tiles,
    a batch without e), called twice in a row with different data: every
    output coefficient equals the oracle, and equals tk_matvec_host."""
    import torch
    stream = torch.cuda.Stream()
    for call in range(2):
        items = make_list(1000 + 10 * call, EXACT_FIT)
        ref = [(k, A, s, e, np.zeros_like(s)) for k, A, s, e, _ in items]
        tk.matvec_host_noalloc(items, stream=stream)
        tk.matvec_host(ref)
        for (k, A, s, e, out), r in zip(items, ref):
            assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all(), (call, k)
            assert (out == r[4]).all(), (call, k)
    assert tk.device_status(0) == 0
