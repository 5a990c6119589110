"""GPU parity of the batched NTT / iNTT against the oracle (every coefficient).

Bar: for every coefficient of every polynomial, canon(gpu) == canon(oracle),
with canon(v) = v mod q in [0, q); integer work, so no tolerance.  In addition
the GPU's own representatives are pinned: forward in [0, q), inverse centred
in [-(q-1)/2, (q-1)/2], byte-identical from run to run.
"""
import ctypes
import threading

import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

pytestmark = pytest.mark.gpu


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int16)).cuda()


def gpu_fwd(tk, torch, x):
    t = to_dev(torch, x)
    tk.ntt(t)
    torch.cuda.synchronize()
    return t.cpu().numpy()


def gpu_inv(tk, torch, x):
    t = to_dev(torch, x)
    tk.invntt(t)
    torch.cuda.synchronize()
    return t.cpu().numpy()


def check_fwd(out, ref):
    assert out.min() >= 0 and out.max() < Q
    bad = np.argwhere(out != canon(ref))
    assert bad.size == 0, f"{len(bad)} mismatches, first at {bad[:4].tolist()}"


def check_inv(out, ref):
    assert out.min() >= -(Q // 2) and out.max() <= Q // 2
    bad = np.argwhere(canon(out) != canon(ref))
    assert bad.size == 0, f"{len(bad)} mismatches, first at {bad[:4].tolist()}"


SIZES = [1, 2, 7, 8, 9, 31, 33, 64, 100, 257, 1000, 4096, 4097, 65541]


@pytest.mark.parametrize("n", SIZES)
def test_uniform_sizes(tk, cuda, oracle, n):
    x = rng(n).integers(0, Q, size=(n, 256)).astype(np.int16)
    check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
    check_inv(gpu_inv(tk, cuda, x), oracle.invntt(x))


NVARIANTS = 5
TC5 = 4          # the tcgen05 kernels


def force_variant(tk, variant):
    tk.set_variant(tk.FORWARD, variant)
    tk.set_variant(tk.INVERSE, variant)


@pytest.mark.parametrize("variant", range(NVARIANTS))
def test_every_variant(tk, cuda, oracle, variant):
    assert tk.variant_count() == NVARIANTS
    try:
        force_variant(tk, variant)
        for n in (1, 9, 63, 64, 65, 1000, 20001):
            x = rng(100 + n).integers(-4000, 4000, size=(n, 256)).astype(np.int16)
            check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
            check_inv(gpu_inv(tk, cuda, x), oracle.invntt(x))
    finally:
        tk.set_variant(tk.FORWARD, -1)
        tk.set_variant(tk.INVERSE, -1)


def test_roundtrip_matches_reference_chain(tk, cuda, oracle):
    """The reference harness runs iNTT on its own NTT output
    (ntt_bench/ntt_bench.cu:618-621, 949-955); do the same on the GPU."""
    x = rng(11).integers(0, Q, size=(3000, 256)).astype(np.int16)
    t = to_dev(cuda, x)
    tk.ntt(t)
    tk.invntt(t)
    cuda.cuda.synchronize()
    out = t.cpu().numpy()
    check_inv(out, oracle.invntt(oracle.ntt(x)))
    assert (canon(out) == canon(x.astype(np.int64) * 65536)).all()


def test_reference_seed_inputs(tk, cuda, oracle):
    """Inputs of the reference benchmark itself: glibc srand(20240816),
    rand() % q (ntt_bench/ntt_bench.cu:942-945)."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(20240816)
    n = 4096
    x = np.array([libc.rand() % Q for _ in range(n * 256)], dtype=np.int16).reshape(n, 256)
    check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
    check_inv(gpu_inv(tk, cuda, x), oracle.invntt(x))


def test_small_signed_inputs(tk, cuda, oracle):
    """ML-KEM calls ntt() on CBD secrets in [-3, 3]; the TC-PACK inputs of the
    reference are ternary (ntt_bench/ntt_bench.cu:782-785)."""
    r = rng(3)
    for lo, hi in ((-1, 2), (-2, 3), (-3, 4)):
        x = r.integers(lo, hi, size=(2048, 256)).astype(np.int16)
        check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
        check_inv(gpu_inv(tk, cuda, x), oracle.invntt(x))


def test_edge_inputs(tk, cuda, oracle):
    rows = [np.zeros(256), np.full(256, Q - 1), np.full(256, -(Q - 1)),
            np.full(256, 9471), np.full(256, -9471),
            np.tile([9471, -9471], 128), np.arange(256) * 37 % Q - 1664]
    rows += [np.eye(256)[j] for j in range(256)]          # unit vectors = matrix columns
    x = np.array(rows, dtype=np.int16)
    check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
    y = np.concatenate([x, np.full((1, 256), 16383), np.full((1, 256), -16384),
                        np.tile([16383, -16384], (1, 128))]).astype(np.int16)
    check_inv(gpu_inv(tk, cuda, y), oracle.invntt(y))


def test_zero_maps_to_zero(tk, cuda):
    x = np.zeros((17, 256), dtype=np.int16)
    assert (gpu_fwd(tk, cuda, x) == 0).all()
    assert (gpu_inv(tk, cuda, x) == 0).all()


def test_full_int16_domain(tk, cuda, oracle):
    """Both directions accept any int16: outputs stay exact mod q
    (the reference overflows there, so compare with its result on canon(x))."""
    r = rng(7)
    x = r.integers(-32768, 32768, size=(1024, 256)).astype(np.int16)
    check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(canon(x)))
    y = r.integers(-32768, 32768, size=(1024, 256)).astype(np.int16)
    check_inv(gpu_inv(tk, cuda, y), oracle.invntt(canon(y)))


def test_out_of_place_and_guards(tk, cuda, oracle):
    """Out-of-place equals in-place, and nothing outside [0, npoly) is touched."""
    n = 1003
    x = rng(5).integers(-3000, 3000, size=(n, 256)).astype(np.int16)
    guard = 8
    buf = cuda.full(((n + 2 * guard) * 256,), 0x5A5A, dtype=cuda.int16, device="cuda")
    out = cuda.full_like(buf, 0x3C3C)
    buf[guard * 256:(guard + n) * 256] = to_dev(cuda, x).flatten()
    src = buf[guard * 256:(guard + n) * 256]
    dst = out[guard * 256:(guard + n) * 256]
    tk.ntt(src, out=dst)
    cuda.cuda.synchronize()
    o = out.cpu().numpy()
    assert (o[:guard * 256] == 0x3C3C).all() and (o[(guard + n) * 256:] == 0x3C3C).all()
    check_fwd(o[guard * 256:(guard + n) * 256].reshape(n, 256), oracle.ntt(x))
    b = buf.cpu().numpy()
    assert (b[guard * 256:(guard + n) * 256].reshape(n, 256) == x).all(), "input modified"
    tk.invntt(src)
    cuda.cuda.synchronize()
    b = buf.cpu().numpy()
    assert (b[:guard * 256] == 0x5A5A).all() and (b[(guard + n) * 256:] == 0x5A5A).all()
    check_inv(b[guard * 256:(guard + n) * 256].reshape(n, 256), oracle.invntt(x))


def test_deterministic_bytes(tk, cuda):
    x = rng(9).integers(-5000, 5000, size=(20000, 256)).astype(np.int16)
    a = gpu_fwd(tk, cuda, x)
    b = gpu_fwd(tk, cuda, x)
    assert (a == b).all()
    a = gpu_inv(tk, cuda, x)
    b = gpu_inv(tk, cuda, x)
    assert (a == b).all()


def test_host_api_matches_device(tk, cuda, oracle):
    n = (1 << 15) * 2 + 77   # spans several host-path chunks, ragged tail
    x = rng(13).integers(0, Q, size=(n, 256)).astype(np.int16)
    h = x.copy()
    tk.ntt_host(h)
    assert (h == gpu_fwd(tk, cuda, x)).all()
    check_fwd(h[:5000], oracle.ntt(x[:5000]))
    tk.invntt_host(h)
    assert (canon(h) == canon(x.astype(np.int64) * 65536)).all()


@pytest.mark.parametrize("chunk", [0, 1000, 4096, 5000])
def test_host_api_chunk_schedules(tk, cuda, chunk):
    """The host path's chunk schedule (growing from 4096 polynomials to the
    chunk option and shrinking at the end) on sizes around its steps: equal
    to the device path byte for byte, both directions."""
    x = rng(57).integers(-32768, 32768, size=(70001, 256)).astype(np.int16)
    tk.set_option(tk.OPT_HOST_CHUNK_POLYS, chunk)
    try:
        for n in (1, 4095, 4097, 8193, 12289, 32769, 70001):
            h = x[:n].copy()
            tk.ntt_host(h)
            assert (h == gpu_fwd(tk, cuda, x[:n])).all(), (chunk, n)
            g = x[:n].copy()
            tk.invntt_host(g)
            assert (g == gpu_inv(tk, cuda, x[:n])).all(), (chunk, n)
    finally:
        tk.set_option(tk.OPT_HOST_CHUNK_POLYS, 0)


def test_non_default_stream_and_threads(tk, cuda, oracle):
    xs = [rng(20 + i).integers(0, Q, size=(777 + 100 * i, 256)).astype(np.int16) for i in range(4)]
    ts = [to_dev(cuda, x) for x in xs]
    cuda.cuda.synchronize()
    errs = []

    def work(i):
        try:
            s = cuda.cuda.Stream()
            with cuda.cuda.stream(s):
                tk.ntt(ts[i], stream=s)
            s.synchronize()
        except Exception as e:  # pragma: no cover - reported below
            errs.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(4)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert not errs
    for x, t in zip(xs, ts):
        check_fwd(t.cpu().numpy(), oracle.ntt(x))


def test_error_paths(tk, cuda):
    L = tk.lib()
    t = cuda.zeros(64 * 256 + 8, dtype=cuda.int16, device="cuda")
    s = cuda.cuda.current_stream().cuda_stream
    assert L.tk_ntt(t.data_ptr() + 2, 4, s) == 2          # misaligned
    assert L.tk_ntt(t.data_ptr(), 0, s) == 0              # empty batch
    assert L.tk_ntt(None, 4, s) == 1                      # NULL
    host = np.zeros(4 * 256, dtype=np.int16)
    assert L.tk_ntt(host.ctypes.data, 4, s) == 6          # host pointer to device API
    assert L.tk_ntt_oop(t.data_ptr(), t.data_ptr() + 512, 4, s) == 1   # overlap
    assert L.tk_ntt(t.data_ptr(), (1 << 32) + 1, s) == 3  # too large
    assert tk.device_status(0) == 0


def test_large_batch_every_coefficient(tk, cuda, oracle):
    """2^20 polynomials (512 MiB), every coefficient against the oracle."""
    n = 1 << 20
    x = rng(21).integers(0, Q, size=(n, 256), dtype=np.int16)
    t = to_dev(cuda, x)
    tk.ntt(t)
    cuda.cuda.synchronize()
    check_fwd(t.cpu().numpy(), oracle.ntt(x))
    tk.invntt(t)
    cuda.cuda.synchronize()
    out = t.cpu().numpy()
    assert (canon(out) == canon(x.astype(np.int64) * 65536)).all()
    assert tk.device_status(0) == 0


HEADLINE = 262144


def test_headline_configuration_every_coefficient(tk, cuda, oracle):
    """The configuration the headline metric is quoted on: 262,144
    polynomials, uniform in [0, q), forward and inverse as separate launches
    with the variants the library picks for that size.  Every coefficient of
    both directions is compared with the oracle (the inverse on the raw input,
    not only through the round trip)."""
    n = HEADLINE
    x = rng(262144).integers(0, Q, size=(n, 256), dtype=np.int16)
    t = to_dev(cuda, x)
    tk.ntt(t)
    cuda.cuda.synchronize()
    check_fwd(t.cpu().numpy(), oracle.ntt(x))
    t = to_dev(cuda, x)
    tk.invntt(t)
    cuda.cuda.synchronize()
    check_inv(t.cpu().numpy(), oracle.invntt(x))
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("variant", range(NVARIANTS))
def test_headline_size_every_inverse_variant(tk, cuda, oracle, variant):
    """Each inverse variant at the headline size, every coefficient against
    the oracle, inputs over the full int16 range."""
    n = HEADLINE
    x = rng(4000 + variant).integers(-32768, 32768, size=(n, 256), dtype=np.int16)
    try:
        tk.set_variant(tk.INVERSE, variant)
        out = gpu_inv(tk, cuda, x)
    finally:
        tk.set_variant(tk.INVERSE, -1)
    check_inv(out, oracle.invntt(canon(x).astype(np.int16)))
    assert tk.device_status(0) == 0


def test_reference_name_shims(tk, cuda, oracle):
    """libtk_pqcrystals.so exports the reference's own symbol names
    (ntt_bench/ref/ntt.h under KYBER_NAMESPACE) and matches the oracle mod q."""
    import os
    shim = ctypes.CDLL(os.path.join(os.path.dirname(tk.LIB_PATH), "libtk_pqcrystals.so"))
    x = rng(31).integers(-3000, 3000, size=(3, 256)).astype(np.int16)
    for k in ("512", "768", "1024"):
        f = getattr(shim, f"pqcrystals_kyber{k}_ref_ntt")
        g = getattr(shim, f"pqcrystals_kyber{k}_ref_invntt")
        for i in range(3):
            p = np.ascontiguousarray(x[i].copy())
            f(p.ctypes.data)
            assert shim.tk_pqcrystals_last_status() == 0
            assert (p == canon(oracle.ntt(x[i:i + 1])[0])).all()
            g(p.ctypes.data)
            assert (canon(p) == canon(x[i].astype(np.int64) * 65536)).all()


def test_autotune_small_range(tk, cuda, oracle, tmp_path):
    """The autotuner picks a valid variant per size, writes/loads its cache,
    and transforms stay exact afterwards."""
    cache = str(tmp_path / "tune.txt")
    try:
        tk.autotune(max_npoly=1 << 12, device=0, cache_path=cache)
        lines = open(cache).read().splitlines()
        assert lines[0] == "tk-autotune 1" and len(lines) == 1 + 2 * 13
        for n in (1, 100, 4096, 1 << 20):
            for d in (tk.FORWARD, tk.INVERSE):
                assert 0 <= tk.get_variant(d, n) < tk.variant_count()
        tk.autotune_reset()
        tk.autotune(max_npoly=1 << 12, device=0, cache_path=cache)   # loads the cache
        x = rng(77).integers(-3000, 3000, size=(3000, 256)).astype(np.int16)
        check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))
        check_inv(gpu_inv(tk, cuda, x), oracle.invntt(x))
    finally:
        tk.autotune_reset()


@pytest.mark.parametrize("variant", range(NVARIANTS))
def test_every_variant_many_tiles_per_cta(tk, cuda, oracle, variant):
    """300,000 polynomials: every CTA walks tens of tiles, so each slot of
    every variant's ring is refilled many times.  Outputs must equal the
    default variant's byte for byte and the oracle on a sample."""
    n = 300000
    x = rng(5150).integers(-32768, 32768, size=(n, 256)).astype(np.int16)
    base_f, base_i = gpu_fwd(tk, cuda, x), gpu_inv(tk, cuda, x)
    try:
        force_variant(tk, variant)
        f, i = gpu_fwd(tk, cuda, x), gpu_inv(tk, cuda, x)
    finally:
        tk.set_variant(tk.FORWARD, -1)
        tk.set_variant(tk.INVERSE, -1)
    assert (f == base_f).all() and (i == base_i).all()
    rows = rng(1).choice(n, 1500, replace=False)
    ref_in = canon(x[rows]).astype(np.int16)
    check_fwd(f[rows], oracle.ntt(ref_in))
    check_inv(i[rows], oracle.invntt(ref_in))


def test_bounded_wait_gives_up_and_context_survives(tk, cuda, oracle):
    """A wait on an mbarrier that nothing completes ends after its limit with
    the status flag set (the batch kernels' give-up path); the device keeps
    working afterwards."""
    import time
    t0 = time.perf_counter()
    assert tk.lib().tk_selftest_bounded_wait(0, 0.02) == 0
    assert time.perf_counter() - t0 < 5
    assert tk.device_status(0) == tk.FLAG_SELFTEST_TIMEOUT
    assert tk.device_status(0) == 0                         # read and cleared
    x = rng(3).integers(0, Q, size=(100, 256)).astype(np.int16)
    check_fwd(gpu_fwd(tk, cuda, x), oracle.ntt(x))


def test_sweep_maximum_size_properties(tk, cuda):
    """2^24 polynomials (8 GiB, the top of the batch-size sweep), checked on
    the device through size-independent properties: invntt(ntt(x)) == 2^16 x
    mod q for every coefficient, and linearity ntt(a + b) == ntt(a) + ntt(b)
    mod q (both are exact identities of the transform)."""
    torch = cuda
    n = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(424242)
    x = torch.randint(0, Q, (n, 256), dtype=torch.int16, device="cuda", generator=g)
    y = x.clone()
    tk.ntt(y)
    tk.invntt(y)
    step = 1 << 21
    for i in range(0, n, step):
        want = (x[i:i + step].to(torch.int64) * 65536) % Q
        got = y[i:i + step].to(torch.int64) % Q
        assert torch.equal(got, want), i
    del y
    a, b = x[:step], x[step:2 * step]
    s = ((a.to(torch.int32) + b.to(torch.int32)) % Q).to(torch.int16)
    fa, fb, fs = a.clone(), b.clone(), s
    tk.ntt(fa)
    tk.ntt(fb)
    tk.ntt(fs)
    assert torch.equal(fs.to(torch.int64) % Q,
                       (fa.to(torch.int64) + fb.to(torch.int64)) % Q)
    torch.cuda.synchronize()
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("inverse", [False, True], ids=["forward", "inverse"])
def test_tcgen05_tile_boundaries_and_guards(tk, cuda, oracle, inverse):
    """The tcgen05 kernels' 128-polynomial tiles: sizes on and around tile and
    grid boundaries (one tile per SM and more), out of place with guard
    polynomials around the output that must stay untouched, in place too,
    every coefficient against the oracle and byte-equal to the mma.sync
    kernels."""
    torch = cuda
    d = tk.INVERSE if inverse else tk.FORWARD
    run = gpu_inv if inverse else gpu_fwd
    ref = oracle.invntt if inverse else oracle.ntt
    check = check_inv if inverse else check_fwd
    fn = tk.invntt if inverse else tk.ntt
    try:
        for n in (1, 127, 128, 129, 255, 256, 148 * 128 - 1, 148 * 128 + 1, 3 * 148 * 128 + 77):
            x = rng(9000 + n).integers(-32768, 32768, size=(n, 256), dtype=np.int16)
            tk.set_variant(d, 0)
            base = run(tk, cuda, x)
            tk.set_variant(d, TC5)
            src = to_dev(torch, x)
            guard = 3
            out = torch.full(((n + 2 * guard), 256), 0x7E7E, dtype=torch.int16, device="cuda")
            fn(src, out=out[guard:guard + n])
            torch.cuda.synchronize()
            o = out.cpu().numpy()
            assert (o[:guard] == 0x7E7E).all() and (o[guard + n:] == 0x7E7E).all(), n
            assert (src.cpu().numpy() == x).all(), n            # input untouched
            got = o[guard:guard + n]
            assert (got == base).all(), n
            assert (run(tk, cuda, x) == base).all(), n          # in place
            pick = np.unique(np.r_[0:min(n, 300), max(0, n - 300):n])
            check(got[pick], ref(canon(x[pick]).astype(np.int16)))
    finally:
        tk.set_variant(d, -1)
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("variant", range(NVARIANTS))
def test_headline_size_every_forward_variant(tk, cuda, oracle, variant):
    """Each forward variant at the headline size, every coefficient against
    the oracle, inputs over the full int16 range."""
    n = HEADLINE
    x = rng(5000 + variant).integers(-32768, 32768, size=(n, 256), dtype=np.int16)
    try:
        tk.set_variant(tk.FORWARD, variant)
        out = gpu_fwd(tk, cuda, x)
    finally:
        tk.set_variant(tk.FORWARD, -1)
    check_fwd(out, oracle.ntt(canon(x).astype(np.int16)))
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("n", [(1 << 18) - 1, (1 << 18) + 1])
def test_default_inverse_across_the_kernel_switch(tk, cuda, oracle, n):
    """The untuned inverse runs the mma.sync kernel below 2^18 polynomials and
    the tcgen05 kernel from there: both sides of the switch, full-range
    inputs, every coefficient of a spread sample against the oracle and the
    two kernels byte-equal on the whole batch."""
    for d in (tk.FORWARD, tk.INVERSE):
        tk.set_variant(d, -1)
    assert tk.get_variant(tk.INVERSE, n) == (0 if n < (1 << 18) else TC5)
    x = rng(7000 + n % 7).integers(-32768, 32768, size=(n, 256), dtype=np.int16)
    out = gpu_inv(tk, cuda, x)
    pick = np.unique(np.r_[0:300, n // 2 - 150:n // 2 + 150, n - 300:n])
    check_inv(out[pick], oracle.invntt(canon(x[pick]).astype(np.int16)))
    try:
        tk.set_variant(tk.INVERSE, TC5 if n < (1 << 18) else 0)
        other = gpu_inv(tk, cuda, x)
    finally:
        tk.set_variant(tk.INVERSE, -1)
    assert (other == out).all()
    assert tk.device_status(0) == 0


def test_tcgen05_random_sizes_stress(tk, cuda):
    """120 launches of the tcgen05 kernels at random sizes (log-uniform, 1 ..
    2^19) and directions, in place and out of place, each byte-equal to the
    mma.sync kernels on the same input: many tile counts per CTA and ragged
    last tiles, under whatever timing the GPU gives each launch."""
    torch = cuda
    r = np.random.default_rng(31337)
    try:
        for it in range(120):
            n = int(np.exp(r.uniform(0, np.log(1 << 19))))
            inverse = bool(r.integers(2))
            d = tk.INVERSE if inverse else tk.FORWARD
            fn = tk.invntt if inverse else tk.ntt
            x = torch.from_numpy(r.integers(-32768, 32768, size=(n, 256), dtype=np.int16)).cuda()
            tk.set_variant(d, 0 if inverse else 3)
            ref = x.clone()
            fn(ref)
            tk.set_variant(d, TC5)
            if it % 2:
                got = torch.empty_like(x)
                fn(x, out=got)
            else:
                got = x.clone()
                fn(got)
            torch.cuda.synchronize()
            assert torch.equal(got, ref), (it, n, inverse)
    finally:
        for d in (tk.FORWARD, tk.INVERSE):
            tk.set_variant(d, -1)
    assert tk.device_status(0) == 0
