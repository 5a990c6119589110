"""Serving loop (tk_server_*): continuous batching of matrix-vector requests.

Every result must equal the oracle's composition mod q, and must be the same
byte for byte whether the request ran alone or mixed with others that were
admitted while it was on the GPU (integer work: no tolerance)."""
import threading
import time

import numpy as np
import pytest

from conftest import rng
from py_oracle import Q, canon

pytestmark = pytest.mark.gpu


def request(seed, k, n, uniform=False):
    """A uniform in [0, q); s, e in [-3, 3] (ML-KEM secrets) or, with uniform,
    in [0, q) like the serving workload."""
    r = rng(seed)
    lo, hi = (0, Q) if uniform else (-3, 4)
    A = r.integers(0, Q, size=(n, k, k, 256)).astype(np.int16)
    s = r.integers(lo, hi, size=(n, k, 256)).astype(np.int16)
    e = r.integers(lo, hi, size=(n, k, 256)).astype(np.int16)
    return A, s, e


def pinned_copy(a):
    """a copied into page-locked host memory (read in place by the server)."""
    import torch
    p = torch.empty(a.shape, dtype=torch.int16, pin_memory=True).numpy()
    p[...] = a
    return p


def packed(A, s, e):
    """A, s, e as views of one contiguous buffer (A then s then e)."""
    buf = np.empty(A.size + s.size + e.size, dtype=np.int16)
    pa, ps = buf[:A.size].reshape(A.shape), buf[A.size:A.size + s.size].reshape(s.shape)
    pe = buf[A.size + s.size:].reshape(e.shape)
    pa[...], ps[...], pe[...] = A, s, e
    return pa, ps, pe


@pytest.fixture(params=["pageable", "pageable-packed", "pinned", "pinned-zero-copy"])
def memkind(request):
    return request.param


def oracle_out(oracle, k, A, s, e):
    return np.stack([oracle.matvec_job(k, A[t].reshape(k * k, 256), s[t], e[t])
                     for t in range(A.shape[0])])


def test_single_request_matches_oracle(tk, cuda, oracle):
    with tk.Server(hbm_budget_bytes=64 << 20) as srv:
        for k in (2, 3, 4):
            A, s, e = request(k, k, 5)
            out = np.zeros_like(s)
            t = srv.submit(k, A, s, e, out)
            srv.wait(t)
            assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()
            assert srv.latency(t) > 0
            srv.release(t)


def test_alone_equals_in_the_mix(tk, cuda, oracle, memkind):
    """48 requests (k in {2,3,4}, 1..64 jobs) from 3 client threads; then the
    same requests one at a time.  Outputs must be identical.  Pageable buffers
    are staged through a small HBM budget, so admission has to wait for memory
    to free up; pinned buffers are read and written in place."""
    r = rng(99)
    reqs = [(int(r.integers(2, 5)), int(r.integers(1, 65))) for _ in range(48)]
    data = [request(1000 + i, k, n, uniform=True) for i, (k, n) in enumerate(reqs)]
    conv = pinned_copy if memkind.startswith("pinned") else (lambda a: a)
    zero_copy = memkind == "pinned-zero-copy"
    data = [tuple(conv(x) for x in d) for d in data]
    if memkind == "pageable-packed":
        data = [packed(*d) for d in data]
    mixed = [conv(np.zeros_like(d[1])) for d in data]
    with tk.Server(hbm_budget_bytes=4 << 20, max_inflight_requests=16,
                   zero_copy=zero_copy) as srv:
        errors = []

        def client(idx):
            try:
                mine = []
                for i in idx:
                    k = reqs[i][0]
                    A, s, e = data[i]
                    mine.append(srv.submit(k, A, s, e, mixed[i]))
                    time.sleep(0.0005)
                for t in mine:
                    srv.wait(t, timeout=60)
            except Exception as ex:  # pragma: no cover - reported below
                errors.append(ex)

        th = [threading.Thread(target=client, args=(list(range(j, 48, 3)),)) for j in range(3)]
        [t.start() for t in th]
        [t.join() for t in th]
        assert not errors
        stats = srv.stats()
        assert stats["jobs_done"] == sum(n for _, n in reqs)
        kind = "direct_requests" if zero_copy else "staged_requests"
        assert stats[kind] == len(reqs), stats
        assert stats["direct_outputs"] == (len(reqs) if memkind.startswith("pinned") else 0)
    alone = []
    with tk.Server(hbm_budget_bytes=64 << 20) as srv:
        for i, (k, n) in enumerate(reqs):
            A, s, e = data[i]
            out = np.zeros_like(s)
            srv.wait(srv.submit(k, A, s, e, out))
            alone.append(out)
    for i, (k, n) in enumerate(reqs):
        assert (mixed[i] == alone[i]).all(), i
    for i in (0, 7, 29, 47):
        k = reqs[i][0]
        A, s, e = data[i]
        assert (canon(mixed[i]) == canon(oracle_out(oracle, k, A, s, e))).all()


def test_server_idle_exit_and_relaunch(tk, cuda, oracle):
    """The device loop leaves after its idle limit and comes back for new work."""
    with tk.Server(hbm_budget_bytes=16 << 20, idle_exit_seconds=0.005) as srv:
        k = 3
        A, s, e = request(5, k, 3)
        out1, out2 = np.zeros_like(s), np.zeros_like(s)
        srv.wait(srv.submit(k, A, s, e, out1))
        time.sleep(0.1)
        srv.wait(srv.submit(k, A, s, e, out2))
        assert (out1 == out2).all()
        assert srv.stats()["device_loop_launches"] >= 2
    assert tk.device_status(0) == 0


def test_server_rejects_oversized_and_bad_requests(tk, cuda):
    import ctypes
    with tk.Server(hbm_budget_bytes=1 << 20) as srv:
        A, s, e = request(1, 4, 128)         # 1.75 MiB > 1 MiB budget
        out = np.zeros_like(s)
        with pytest.raises(tk.TKError):
            srv.submit(4, A, s, e, out)
        t = ctypes.c_uint64()
        L = tk.lib()
        assert L.tk_server_submit(srv._h, 5, 1, s.ctypes.data, s.ctypes.data, None,
                                  out.ctypes.data, ctypes.byref(t)) == 1
        assert L.tk_server_wait(srv._h, 12345, 0.01) == 1
        A, s, e = request(2, 2, 3)
        buf = np.zeros(A.size + s.size, dtype=np.int16)
        assert L.tk_server_submit(srv._h, 2, 3, buf.ctypes.data, s.ctypes.data, None,
                                  buf.ctypes.data + 512, ctypes.byref(t)) == 1   # out inside A


def test_pinned_buffers_rewritten_between_requests(tk, cuda, oracle):
    """The device loop keeps running while the host rewrites a pinned input
    buffer; the next request must see the new contents (no stale cache line)."""
    k, n = 3, 8
    with tk.Server(idle_exit_seconds=1.0, zero_copy=True) as srv:
        bufs = [pinned_copy(x) for x in request(31, k, n, uniform=True)]
        out = pinned_copy(np.zeros_like(bufs[1]))
        for rnd in range(4):
            A, s, e = request(40 + rnd, k, n, uniform=True)
            bufs[0][...], bufs[1][...], bufs[2][...] = A, s, e
            srv.wait(srv.submit(k, *bufs, out))
            assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all(), rnd
        st = srv.stats()
        assert st["direct_requests"] == 4 and st["device_loop_launches"] == 1, st


def test_pinned_is_staged_without_zero_copy(tk, cuda, oracle):
    k, n = 2, 5
    A, s, e = (pinned_copy(x) for x in request(8, k, n, uniform=True))
    out = pinned_copy(np.zeros_like(s))
    with tk.Server() as srv:
        srv.wait(srv.submit(k, A, s, e, out))
        st = srv.stats()
        assert st["staged_requests"] == 1 and st["direct_requests"] == 0
        assert st["direct_outputs"] == 1
        assert st["queue_ns"] + st["device_ns"] + st["return_ns"] > 0
    assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()


def test_back_to_back_requests_share_input_copies(tk, cuda, oracle):
    """200 requests whose A | s | e lie back to back in one page-locked arena
    (outputs page-locked too, written in place), submitted in one burst: once
    64 are active, admission takes the next ones 32 at a time, and inputs that
    continue each other in the arena and in the pool go in one copy.  Every
    result equals the oracle's, and fewer input copies were issued than
    requests staged."""
    import torch
    r = rng(4242)
    reqs = [(int(r.integers(2, 5)), int(r.integers(16, 65))) for _ in range(200)]
    sizes = [n * (k * k + 2 * k) * 256 for k, n in reqs]
    arena = torch.empty(sum(sizes), dtype=torch.int16, pin_memory=True).numpy()
    outs, views, off = [], [], 0
    for i, ((k, n), sz) in enumerate(zip(reqs, sizes)):
        A, s, e = request(5000 + i, k, n, uniform=True)
        m = arena[off:off + sz]
        pa = m[:A.size].reshape(A.shape)
        ps = m[A.size:A.size + s.size].reshape(s.shape)
        pe = m[A.size + s.size:].reshape(e.shape)
        pa[...], ps[...], pe[...] = A, s, e
        views.append((k, pa, ps, pe))
        outs.append(pinned_copy(np.zeros_like(s)))
        off += sz
    with tk.Server(hbm_budget_bytes=1 << 30, max_inflight_requests=256) as srv:
        st0 = srv.stats()
        tickets = [srv.submit(k, A, s, e, out) for (k, A, s, e), out in zip(views, outs)]
        for t in tickets:
            srv.wait(t, timeout=60)
            srv.release(t)
        st = srv.stats()
    staged = st["staged_requests"] - st0["staged_requests"]
    copies = st["input_copies"] - st0["input_copies"]
    assert staged == 200 and st["direct_outputs"] - st0["direct_outputs"] == 200
    assert 0 < copies < staged, (copies, staged)
    for (k, A, s, e), out in zip(views, outs):
        assert (canon(out) == canon(oracle_out(oracle, k, A, s, e))).all()
