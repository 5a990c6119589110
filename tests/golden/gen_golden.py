"""Generate the golden fixtures from the reference's own C code.

Runs ntt_bench/ref/{ntt,reduce}.c (compiled unmodified into
oracle/_ref/libkyber_ref.so by oracle/Makefile) on:
  * the reference benchmark's own inputs: glibc srand(20240816), rand() % q,
    first 64 polynomials (ntt_bench/ntt_bench.cu:942-956);
  * the reference's packed-ternary inputs: srand(20240819 + 2*10),
    rand() % 3 - 1 (ntt_bench/ntt_bench.cu:782-785), first 64 polynomials;
  * edge cases: zeros, +-(q-1), +-9471 (the largest |x| on which ntt() does
    not overflow int16), unit vectors;
  * basemul on seeded pairs (ntt_bench/ref/ntt.c:139-146);
  * matrix-vector jobs for k = 2, 3, 4 (A uniform in [0, q), s and e in
    [-3, 3], seeded), composed from the reference's ntt, basemul (pairwise,
    +-zetas[64 + t/2]), barrett_reduce and invntt the way ML-KEM composes them
    (int16 polynomial adds, one reduction of the k-term sum, then + e).
Writes tests/golden/ref_vectors.npz.  Needs the reference sources (to build
oracle/_ref) and glibc; run from the repository root:
    python tests/golden/gen_golden.py
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import py_oracle  # noqa: E402

Q = 3329


def glibc_rand(seed, count, f):
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    return np.array([f(libc.rand()) for _ in range(count)], dtype=np.int16)


def ref_matvec_job(ref, k, A, s, e):
    """out_i = invntt(reduce(sum_j basemul(A_ij, ntt(s_j)))) + e_i, through the
    reference's own C functions only."""
    barrett = getattr(ref.lib, ref.prefix + "barrett_reduce")
    shat = ref.ntt(s.reshape(k, 256))
    out = np.zeros((k, 256), dtype=np.int16)
    for i in range(k):
        acc = np.zeros(256, dtype=np.int16)
        for j in range(k):
            a = A[i * k + j]
            t = np.zeros(256, dtype=np.int16)
            for p in range(128):                      # pair p: +-zetas[64 + p/2]
                z = int(ref.zetas[64 + p // 2])
                t[2 * p:2 * p + 2] = ref.basemul(a[2 * p:2 * p + 2], shat[j, 2 * p:2 * p + 2],
                                                 -z if p & 1 else z)
            acc = (acc.astype(np.int32) + t).astype(np.int16)   # poly_add (int16)
        acc = np.array([barrett(int(v)) for v in acc], dtype=np.int16)
        out[i] = (ref.invntt(acc[None])[0].astype(np.int32) + e[i]).astype(np.int16)
    return out


def main():
    if not py_oracle.RefKyber.available():
        raise SystemExit("oracle/_ref/libkyber_ref.so not available (needs the reference sources)")
    ref = py_oracle.RefKyber(3)
    uni = glibc_rand(20240816, 64 * 256, lambda r: r % Q).reshape(64, 256)
    tern = glibc_rand(20240819 + 2 * 10, 64 * 256, lambda r: r % 3 - 1).reshape(64, 256)
    edge = [np.zeros(256), np.full(256, Q - 1), np.full(256, -(Q - 1)), np.full(256, 9471),
            np.full(256, -9471), np.tile([9471, -9471], 128)]
    edge += [np.eye(256)[j] for j in (0, 1, 2, 15, 16, 17, 128, 255)]
    edge = np.array(edge, dtype=np.int16)
    out = {}
    for name, x in (("uniform", uni), ("ternary", tern), ("edge", edge)):
        f = ref.ntt(x)
        out[name + "_in"] = x
        out[name + "_ntt"] = f
        out[name + "_invntt"] = ref.invntt(x)
        out[name + "_roundtrip"] = ref.invntt(f)
    g = np.random.default_rng(7)
    a = g.integers(-Q + 1, Q, size=(256, 2)).astype(np.int16)
    b = g.integers(-Q + 1, Q, size=(256, 2)).astype(np.int16)
    z = ref.zetas[64 + (np.arange(256) % 64)]
    r = np.array([ref.basemul(a[i], b[i], int(z[i])) for i in range(256)], dtype=np.int16)
    out.update(basemul_a=a, basemul_b=b, basemul_zeta=z.astype(np.int16), basemul_r=r,
               zetas=ref.zetas)
    g = np.random.default_rng(11)
    for k in (2, 3, 4):
        jobs = 3
        A = g.integers(0, Q, size=(jobs, k * k, 256)).astype(np.int16)
        sv = g.integers(-3, 4, size=(jobs, k, 256)).astype(np.int16)
        ev = g.integers(-3, 4, size=(jobs, k, 256)).astype(np.int16)
        mv = np.stack([ref_matvec_job(ref, k, A[t], sv[t], ev[t]) for t in range(jobs)])
        out.update({f"matvec{k}_A": A, f"matvec{k}_s": sv, f"matvec{k}_e": ev,
                    f"matvec{k}_out": mv})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_vectors.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
