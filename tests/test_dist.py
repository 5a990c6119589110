"""Multi-process host logic on CPU: two gloo ranks shard a batch, each
transforms its contiguous range (the oracle stands in for the GPU here: this
test covers the partitioning, timing reduction and gathering, not the
kernels), and rank 0 reassembles the whole."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tensorkyber_b200 import dist as tkdist


def test_shard_tiles_the_range():
    for n in (0, 1, 7, 1000, 262144):
        for world in (1, 2, 3, 8):
            ranges = [tkdist.shard(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        tkdist.shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    from py_oracle import Oracle
    from tensorkyber_b200 import dist as tkd
    d = tkd.init("gloo", timeout_s=60)
    r, w, _ = tkd.env()
    assert (r, w) == (rank, world)
    x = np.random.default_rng(7).integers(0, 3329, size=(n, 256)).astype(np.int16)
    a, b = tkd.shard(n, r, w)
    local = Oracle().ntt(x[a:b])
    full = tkd.gather_shards(local, n, d)
    slowest = tkd.max_over_ranks(0.001 * (rank + 1), d)
    if rank == 0:
        np.save(out_path, full)
        with open(out_path + ".max", "w") as f:
            f.write(repr(slowest))
    d.barrier()
    d.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(tmp_path):
    n, world = 1001, 2
    out = str(tmp_path / "full.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    from py_oracle import Oracle
    x = np.random.default_rng(7).integers(0, 3329, size=(n, 256)).astype(np.int16)
    assert (np.load(out) == Oracle().ntt(x)).all()
    assert float(open(out + ".max").read()) == pytest.approx(0.002)
