"""CPU model of k_matvec_tiles' work split (tk_ntt_mma.cu): tiles numbered
across up to four batches (first_tile, launch_matvec_tile), dealt round robin
to G CTAs (tile c, c + G, ...), each tile's 8-row TMA boxes (issue_load), its
basemul jobs (basemul_phase) and its stores (inv_phase).  Every vector row of
every batch must be loaded and stored exactly once, every job computed exactly
once, and a job's accumulator rows must lie inside its tile."""
import itertools

import pytest

MAX_SEGS = 4
W = 4  # warps per CTA


def tile_units(k):
    return 3 if k == 3 else 4


def tile_jobs(k):
    return 8 * tile_units(k) // k


def simulate(batches, cap):
    """batches: [(k, njobs)]; cap: CTAs the device allows.  Returns per-batch
    counters of row loads, row stores and job computations."""
    first = [0]
    for k, n in batches:
        first.append(first[-1] + (n + tile_jobs(k) - 1) // tile_jobs(k))
    ntiles = first[-1]
    G = min(ntiles, cap)
    loads = [[0] * (n * k) for k, n in batches]
    stores = [[0] * (n * k) for k, n in batches]
    jobs = [[0] * n for k, n in batches]

    def batch_of(t):
        return sum(1 for j in range(1, MAX_SEGS) if j < len(batches) and t >= first[j])

    for c in range(G):
        nmine = (ntiles - 1 - c) // G + 1 if ntiles > c else 0
        for kk in range(nmine):
            t = c + kk * G
            b = batch_of(t)
            k, n = batches[b]
            nvec = n * k
            tl = t - first[b]
            row0 = tl * 8 * tile_units(k)
            for warp in range(W):
                row = row0 + 8 * warp
                if warp < tile_units(k) and row < nvec:          # issue_load
                    for r in range(row, min(row + 8, nvec)):     # box rows past the batch: OOB
                        loads[b][r] += 1
                if warp < tile_units(k) and row < nvec:          # inv_phase store
                    for r in range(row, min(row + 8, nvec)):
                        stores[b][r] += 1
                for jl in range(warp, tile_jobs(k), W):          # basemul_phase
                    job = tl * tile_jobs(k) + jl
                    if job >= n:
                        break
                    jobs[b][job] += 1
                    for i in range(k):                           # accumulator rows
                        assert jl * k + i < 8 * tile_units(k)
                        assert row0 + jl * k + i == job * k + i  # the job's own rows
    return loads, stores, jobs


CASES = [
    [(3, 77), (2, 130), (4, 51)],
    [(2, 1)],
    [(4, 1), (3, 1), (2, 1), (4, 2)],
    [(3, 8), (3, 9), (3, 7)],
    [(2, 16), (2, 17), (4, 8), (4, 9)],
    [(3, 1000)],
]


@pytest.mark.parametrize("batches", CASES)
@pytest.mark.parametrize("cap", [1, 3, 592])
def test_tiles_cover_rows_and_jobs_once(batches, cap):
    loads, stores, jobs = simulate(batches, cap)
    for lb, sb, jb in zip(loads, stores, jobs):
        assert all(v == 1 for v in lb)
        assert all(v == 1 for v in sb)
        assert all(v == 1 for v in jb)


def test_all_small_mixed_lists():
    """Every list of up to three batches with k in {2, 3, 4} and 1..17 jobs."""
    for nb in (1, 2, 3):
        for ks in itertools.product((2, 3, 4), repeat=nb):
            for ns in itertools.product((1, 5, 8, 16, 17), repeat=nb):
                loads, stores, jobs = simulate(list(zip(ks, ns)), 7)
                for lb, sb, jb in zip(loads, stores, jobs):
                    assert all(v == 1 for v in lb) and all(v == 1 for v in sb)
                    assert all(v == 1 for v in jb)
