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


def test_alone_equals_in_the_mix(tk, cuda, oracle):
    """48 requests (k in {2,3,4}, 1..64 jobs) from 3 client threads with a
    small HBM budget, so admission has to wait for memory to free up; then the
    same requests one at a time.  Outputs must be identical."""
    r = rng(99)
    reqs = [(int(r.integers(2, 5)), int(r.integers(1, 65))) for _ in range(48)]
    data = [request(1000 + i, k, n, uniform=True) for i, (k, n) in enumerate(reqs)]
    mixed = [np.zeros_like(d[1]) for d in data]
    with tk.Server(hbm_budget_bytes=4 << 20, max_inflight_requests=16) as srv:
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
