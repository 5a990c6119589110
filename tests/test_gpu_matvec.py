"""GPU parity of the ML-KEM matrix-vector jobs (tk_matvec) against the oracle's
composition of the reference's ntt / basemul / invntt (tko_matvec_job).
Integer work: every output coefficient must agree mod q."""
import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[0, 1, 2], ids=["pipeline", "fused", "tiled"])
def mode(request, tk):
    before = tk.get_option(tk.OPT_MATVEC_MODE)
    tk.set_option(tk.OPT_MATVEC_MODE, request.param)
    yield request.param
    tk.set_option(tk.OPT_MATVEC_MODE, before)


def make_jobs(seed, k, n, a_lo=0, a_hi=Q, small=3):
    r = rng(seed)
    A = r.integers(a_lo, a_hi, size=(n, k, k, 256)).astype(np.int16)
    s = r.integers(-small, small + 1, size=(n, k, 256)).astype(np.int16)
    e = r.integers(-small, small + 1, size=(n, k, 256)).astype(np.int16)
    return A, s, e


def oracle_out(oracle, k, A, s, e):
    return np.stack([oracle.matvec_job(k, A[t].reshape(k * k, 256), s[t],
                                       e[t] if e is not None else np.zeros_like(s[t]))
                     for t in range(A.shape[0])])


def run(tk, cuda, items, inplace=False):
    dev = []
    for k, A, s, e in items:
        tA, ts = cuda.from_numpy(A).cuda(), cuda.from_numpy(s).cuda()
        te = cuda.from_numpy(e).cuda() if e is not None else None
        out = ts if inplace else cuda.empty_like(ts)
        dev.append((k, tA, ts, te, out))
    tk.matvec(dev)
    cuda.cuda.synchronize()
    return [d[4].cpu().numpy() for d in dev]


@pytest.mark.parametrize("k", [2, 3, 4])
def test_matvec_each_k(tk, cuda, oracle, mode, k):
    A, s, e = make_jobs(k, k, 203)
    (out,) = run(tk, cuda, [(k, A, s, e)])
    assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()


def test_matvec_mixed_batches_one_call(tk, cuda, oracle, mode):
    items = [(k,) + make_jobs(10 + k, k, n) for k, n in ((3, 77), (2, 130), (4, 51))]
    outs = run(tk, cuda, items)
    for (k, A, s, e), out in zip(items, outs):
        assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()


def test_matvec_no_addend_in_place_and_wide_inputs(tk, cuda, oracle, mode):
    """e = NULL, out == s, A over (-q, q) and s over the full int16 range."""
    k = 3
    A, s, _ = make_jobs(21, k, 64, a_lo=-Q + 1, a_hi=Q)
    s_wide = rng(22).integers(-32768, 32768, size=s.shape).astype(np.int16)
    (out,) = run(tk, cuda, [(k, A, s_wide, None)], inplace=True)
    # the oracle's ntt overflows int16 outside |x| <= 9471: feed it canon(s)
    ref = oracle_out(oracle, k, A, canon(s_wide).astype(np.int16), None)
    assert (canon(out) == canon(ref)).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_matvec_golden_reference_jobs(tk, cuda, golden, mode, k):
    """The jobs that tests/golden/gen_golden.py composed from the reference's
    own C functions, straight from the fixture (no oracle in between)."""
    A = golden[f"matvec{k}_A"].reshape(-1, k, k, 256)
    s, e, want = golden[f"matvec{k}_s"], golden[f"matvec{k}_e"], golden[f"matvec{k}_out"]
    (out,) = run(tk, cuda, [(k, A, s, e)])
    assert (canon(out) == canon(want)).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_matvec_full_int16_A_and_extremes(tk, cuda, oracle, mode, k):
    """A over the full int16 range, plus jobs whose A is all -32768 or all
    32767, s over the full int16 range (the worst-case sums themselves are
    pinned by the CPU models of the basemul arithmetic).  The oracle's job
    adds its k basemul terms in int16, which can wrap for such A (a term
    reaches ~30,000 when ntt(s) nears its 8q bound), so the reference here is
    its primitives with the sum taken exactly: each basemul, on ntt(s) reduced
    to [0, q), stays in int16 for any int16 A."""
    A, _, e = make_jobs(40 + k, k, 40, a_lo=-32768, a_hi=32768)
    A[0], A[1] = -32768, 32767
    s = rng(50 + k).integers(-32768, 32768, size=e.shape).astype(np.int16)
    (out,) = run(tk, cuda, [(k, A, s, e)])
    n = A.shape[0]
    # the oracle's ntt overflows int16 outside |x| <= 9471: feed it canon(s)
    b = canon(oracle.ntt(canon(s).reshape(-1, 256))).reshape(n, k, 256)
    ref = np.zeros((n, k, 256), dtype=np.int64)
    for t in range(n):
        for i in range(k):
            acc = sum(oracle.poly_basemul(A[t, i, j], b[t, j]).astype(np.int64) for j in range(k))
            ref[t, i] = oracle.invntt(canon(acc)[None])[0].astype(np.int64) + e[t, i]
    assert (canon(out) == canon(ref)).all()


def test_matvec_spans_several_chunks(tk, cuda, oracle, mode):
    """k = 2 with more jobs than one chunk (chunk set to 32768 vector polys)."""
    k, n = 2, 40000
    A, s, e = make_jobs(31, k, n)
    tk.set_option(tk.OPT_MATVEC_CHUNK_POLYS, 32768)
    try:
        (out,) = run(tk, cuda, [(k, A, s, e)])
    finally:
        tk.set_option(tk.OPT_MATVEC_CHUNK_POLYS, 0)
    pick = np.r_[0:50, 16380:16390, n - 50:n]
    assert (canon(out[pick]) == canon(oracle_out(oracle, k, A[pick], s[pick], e[pick]))).all()
    assert tk.device_status(0) == 0


def test_matvec_five_batches_small_chunks(tk, cuda, oracle, mode):
    """Five batches (more than one launch's segments) with a chunk of 1000
    vector polynomials: chunks straddle batch boundaries, and one batch has a
    single job and no addend.  Equal to each batch run alone."""
    spec = [(3, 301, True), (2, 1, False), (4, 260, True), (2, 517, True), (3, 9, True)]
    items = []
    for i, (k, n, with_e) in enumerate(spec):
        A, s, e = make_jobs(40 + i, k, n)
        items.append((k, A, s, e if with_e else None))
    tk.set_option(tk.OPT_MATVEC_CHUNK_POLYS, 1000)
    try:
        outs = run(tk, cuda, items)
    finally:
        tk.set_option(tk.OPT_MATVEC_CHUNK_POLYS, 0)
    for (k, A, s, e), out in zip(items, outs):
        (alone,) = run(tk, cuda, [(k, A, s, e)])
        assert (out == alone).all()
        pick = np.unique(np.r_[0:5, A.shape[0] - 5:A.shape[0]].clip(0, A.shape[0] - 1))
        assert (canon(out[pick]) == canon(oracle_out(oracle, k, A[pick], s[pick],
                                                     None if e is None else e[pick]))).all()


def test_matvec_rejects_bad_batches(tk, cuda):
    import ctypes
    t = cuda.zeros((4, 2, 256), dtype=cuda.int16, device="cuda")
    A = cuda.zeros((4, 2, 2, 256), dtype=cuda.int16, device="cuda")
    L = tk.lib()
    bad_k = (tk.MatvecBatch * 1)(tk.MatvecBatch(5, 4, A.data_ptr(), t.data_ptr(), None, t.data_ptr()))
    assert L.tk_matvec(bad_k, 1, None) == 1
    overlap = (tk.MatvecBatch * 1)(tk.MatvecBatch(2, 4, A.data_ptr(), t.data_ptr(), None, A.data_ptr()))
    assert L.tk_matvec(overlap, 1, None) == 1
    mis = (tk.MatvecBatch * 1)(tk.MatvecBatch(2, 4, A.data_ptr() + 2, t.data_ptr(), None, t.data_ptr()))
    assert L.tk_matvec(mis, 1, None) == 2
    assert L.tk_matvec(None, 0, None) == 0
    assert L.tk_matvec(None, 1, None) == 1
    del ctypes


def test_matvec_host_matches_device(tk, cuda, oracle, mode):
    """The host-buffer form (staging + the same kernels) on a mixed list."""
    r = rng(77)
    items, expect = [], []
    for k, n in ((2, 3), (4, 2), (3, 5)):
        A = r.integers(0, 3329, size=(n, k, k, 256)).astype(np.int16)
        s = r.integers(-3, 4, size=(n, k, 256)).astype(np.int16)
        e = r.integers(-3, 4, size=(n, k, 256)).astype(np.int16)
        out = np.zeros_like(s)
        items.append((k, A, s, e, out))
        expect.append(np.stack([oracle.matvec_job(k, A[t].reshape(k * k, 256), s[t], e[t])
                                for t in range(n)]))
    tk.matvec_host(items)
    for (k, A, s, e, out), x in zip(items, expect):
        assert (canon(out) == canon(x)).all()
    k, A, s, e, out = items[1]                           # A, s, e back to back: one copy
    buf = np.concatenate([A.ravel(), s.ravel(), e.ravel()])
    pA = buf[:A.size].reshape(A.shape)
    ps = buf[A.size:A.size + s.size].reshape(s.shape)
    pe = buf[A.size + s.size:].reshape(e.shape)
    out2 = np.zeros_like(s)
    tk.matvec_host([(k, pA, ps, pe, out2)])
    assert (out2 == out).all()
    k, A, s, e, out = items[2]
    tk.matvec_host([(k, A, s, None, s)])                 # in place, no addend
    assert (canon(s) == canon(expect[2] - e)).all()


def test_matvec_full_mixed_workload_sample(tk, cuda, oracle, mode):
    """The full matrix-vector workload: 65,536 jobs, k ~ U{2,3,4}, A uniform in
    [0, q), s and e in [-3, 3], one call with three batches; 300 sampled jobs
    of every batch against the oracle's composition."""
    r = rng(65536)
    ks = r.integers(2, 5, size=65536)
    items = []
    for k in (2, 3, 4):
        n = int((ks == k).sum())
        items.append((k,) + make_jobs(900 + k, k, n))
    outs = run(tk, cuda, items)
    for (k, A, s, e), out in zip(items, outs):
        pick = rng(k).choice(A.shape[0], 300, replace=False)
        assert (canon(out[pick]) == canon(oracle_out(oracle, k, A[pick], s[pick], e[pick]))).all()
    assert tk.device_status(0) == 0


@pytest.mark.parametrize("variant", range(5))
def test_matvec_pipeline_every_variant(tk, cuda, oracle, variant):
    """The pipeline's forward and inverse-with-addend launches in each batch
    kernel variant (one batch, so the single-batch kernels run)."""
    A, s, e = make_jobs(40 + variant, 3, 150)
    before = tk.get_option(tk.OPT_MATVEC_MODE)
    tk.set_option(tk.OPT_MATVEC_MODE, tk.MATVEC_PIPELINE)
    try:
        tk.set_variant(tk.FORWARD, variant)
        tk.set_variant(tk.INVERSE, variant)
        (out,) = run(tk, cuda, [(3, A, s, e)])
    finally:
        tk.set_variant(tk.FORWARD, -1)
        tk.set_variant(tk.INVERSE, -1)
        tk.set_option(tk.OPT_MATVEC_MODE, before)
    assert (canon(out) == canon(oracle_out(oracle, 3, A, s, e))).all()


@pytest.mark.parametrize("k", [2, 3, 4])
def test_matvec_tile_boundaries(tk, cuda, oracle, mode, k):
    """Job counts on and around the tiled kernel's tile sizes (16 jobs for
    k = 2, 8 for k = 3, 4) and around a whole first wave of CTAs: every job
    equals the oracle, and the same jobs give the same bytes in every count."""
    per = 16 if k == 2 else 8
    A, s, e = make_jobs(90 + k, k, 8 * per + 1)
    ref = oracle_out(oracle, k, A, s, e)
    for n in (1, per - 1, per, per + 1, 8 * per + 1):
        (out,) = run(tk, cuda, [(k, A[:n], s[:n], e[:n])])
        assert (canon(out) == canon(ref[:n])).all(), n
    assert tk.device_status(0) == 0


def test_matvec_mixed_k_in_place_many_batches(tk, cuda, oracle, mode):
    """Six batches of alternating k in one call (two launches of the tiled
    kernel), in place, some without e: equal to the oracle."""
    spec = [(4, 37, True), (2, 5, False), (3, 100, True), (4, 1, True), (2, 64, True), (3, 17, False)]
    items = []
    for i, (k, n, with_e) in enumerate(spec):
        A, s, e = make_jobs(70 + i, k, n)
        items.append((k, A, s, e if with_e else None))
    outs = run(tk, cuda, items, inplace=True)
    for (k, A, s, e), out in zip(items, outs):
        assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()
    assert tk.device_status(0) == 0


def test_matvec_graph_replay_matches_oracle(tk, cuda, oracle, mode):
    """tk_matvec captured in a CUDA graph (three mixed-k batches, the form the
    matrix-vector benchmark replays), replayed twice with new inputs written
    into the captured buffers in between: each replay equals the oracle's
    composition of the reference's ntt / basemul / invntt."""
    torch = cuda
    tk.init(0)
    spec = ((2, 70), (3, 41), (4, 29))
    dev = []
    for k, n in spec:
        dev.append((k, torch.empty((n, k, k, 256), dtype=torch.int16, device="cuda"),
                    torch.empty((n, k, 256), dtype=torch.int16, device="cuda"),
                    torch.empty((n, k, 256), dtype=torch.int16, device="cuda"),
                    torch.empty((n, k, 256), dtype=torch.int16, device="cuda")))

    def fill(seed):
        host = []
        for i, ((k, n), (_, tA, ts, te, _o)) in enumerate(zip(spec, dev)):
            A, s, e = make_jobs(seed + i, k, n)
            tA.copy_(torch.from_numpy(A))
            ts.copy_(torch.from_numpy(s))
            te.copy_(torch.from_numpy(e))
            host.append((k, A, s, e))
        torch.cuda.synchronize()
        return host

    fill(500)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        tk.matvec(dev, stream=side)               # warm-up outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        tk.matvec(dev)
    for rep, seed in enumerate((600, 700)):
        host = fill(seed)
        for d in dev:
            d[4].fill_(0x2B2B)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        for (k, A, s, e), d in zip(host, dev):
            out = d[4].cpu().numpy()
            assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all(), (rep, k)
    del graph
    assert tk.device_status(0) == 0
