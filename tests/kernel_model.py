"""Bit-level CPU model of the sm_100a kernels' integer arithmetic.

It rebuilds the logical int8 operand matrices from the per-lane fragment tables
that the library uploads (using the mma.sync register layouts of the PTX ISA),
feeds them the same unsigned data bytes the kernels feed the tensor cores, and
applies the same recombination and Barrett steps.  Agreement with the oracle
here pins the tables and the arithmetic on the CPU; the GPU parity tests then
only have to confirm the kernels' data movement.
"""
from __future__ import annotations

import numpy as np

Q = 3329
BAR_LAZY = 1290167        # floor(2^32 / q)
BAR_EXACT = 82570715      # ceil(2^38 / q)


def unpack_k32(frag: np.ndarray) -> np.ndarray:
    """frag[32 lanes][4 regs] uint32 -> A[16][32] int8 (m16n8k32 row-major A)."""
    A = np.zeros((16, 32), dtype=np.int64)
    for lane in range(32):
        for j in range(4):
            w = int(frag[lane][j])
            for e in range(4):
                row = lane // 4 + (8 if j & 1 else 0)
                col = 4 * (lane % 4) + e + (16 if j & 2 else 0)
                A[row, col] = np.int8(np.uint8((w >> (8 * e)) & 255))
    return A


def unpack_k16(frag: np.ndarray) -> np.ndarray:
    """frag[32 lanes][2 regs] uint32 -> A[16][16] int8 (m16n8k16 row-major A)."""
    A = np.zeros((16, 16), dtype=np.int64)
    for lane in range(32):
        for j in range(2):
            w = int(frag[lane][j])
            for e in range(4):
                A[lane // 4 + 8 * j, 4 * (lane % 4) + e] = np.int8(np.uint8((w >> (8 * e)) & 255))
    return A


def fwd_slot_e(slot: int) -> int:
    return (slot >> 1) + 4 * (slot & 1)


class FwdModel:
    def __init__(self, words: np.ndarray):
        w = np.asarray(words, dtype=np.uint32)
        s1 = w[:256].reshape(2, 32, 4)
        c1 = w[256:320].view(np.int32).reshape(32, 2)
        s2 = w[320:2368].reshape(16, 2, 32, 2)
        s1b = w[2368:2496].reshape(2, 32, 2)
        c1b = w[2496:2560].view(np.int32).reshape(32, 2)
        s2w = w[2560:6656].reshape(16, 2, 32, 4)
        # stage 2 from int32 intermediates: K = 4 * slot + byte
        self.A2w = [[unpack_k32(s2w[b][s]) for s in range(2)] for b in range(16)]
        # single-limb stage 1: A columns k' hold block m = pi(k')
        self.A1b = [unpack_k16(s1b[g]) for g in range(2)]
        self.corr_b = np.zeros(16, dtype=np.int64)
        for lane in range(32):
            self.corr_b[lane // 4] = c1b[lane][0]
            self.corr_b[lane // 4 + 8] = c1b[lane][1]
        self.pi = [(2 * (k >> 2) + (k & 3)) if (k & 3) < 2 else (8 + 2 * (k >> 2) + (k & 3) - 2)
                   for k in range(16)]
        self.A1 = [unpack_k32(s1[g]) for g in range(2)]
        corr = np.zeros(16, dtype=np.int64)
        for lane in range(32):
            corr[lane // 4] = c1[lane][0]
            corr[lane // 4 + 8] = c1[lane][1]
        self.corr = corr
        self.A2 = [[unpack_k16(s2[b][s]) for s in range(2)] for b in range(16)]

    def __call__(self, x: np.ndarray, single_limb: bool = False, wide: bool = False) -> np.ndarray:
        """single_limb: the stage-1 form for inputs in [-128, 127] (one data
        byte x + 128 per coefficient, K in the pi order of the fragments).
        wide: the stage-1 sums stay unreduced int32 and stage 2 reads their
        four bytes (the int32-intermediate kernels)."""
        x = np.asarray(x, dtype=np.int16).reshape(-1, 256)
        P = x.shape[0]
        if single_limb:
            assert x.min() >= -128 and x.max() <= 127
            u = (x.astype(np.int64) + 128).reshape(P, 16, 16)                # [p][m][c]
            X = u[:, self.pi, :]                                             # [p][k'][c]
            D0 = self.corr_b[None, :, None] + np.einsum("ik,pkc->pic", self.A1b[0], X)
            D1 = np.einsum("ik,pkc->pic", self.A1b[1], X)
        else:
            u = (x.view(np.uint16).astype(np.int64) ^ 0x8000).reshape(P, 16, 16)  # [p][m][c]
            X = np.stack([u & 255, u >> 8], axis=2).reshape(P, 32, 16)     # [p][k=2m+b][c]
            D0 = self.corr[None, :, None] + np.einsum("ik,pkc->pic", self.A1[0], X)
            D1 = np.einsum("ik,pkc->pic", self.A1[1], X)
        S = D0 + 128 * D1
        assert S.min() >= 0 and S.max() < (1 << 25), (S.min(), S.max())
        if wide:
            mid = S
        else:
            mid = S - ((S * BAR_LAZY) >> 32) * Q                             # [p][i][c]
            assert mid.min() >= 0 and mid.max() < Q + 11       # red_lazy below 2^25
        out = np.zeros((P, 256), dtype=np.int64)
        for b in range(16):
            for s in range(2):
                cols = [2 * fwd_slot_e(j) + s for j in range(8)]
                v = mid[:, b, cols]                                          # [p][slot]
                if wide:
                    B = np.stack([(v >> (8 * t)) & 255 for t in range(4)], axis=2).reshape(P, 32)
                    D = B @ self.A2w[b][s].T
                else:
                    B = np.stack([v & 255, v >> 8], axis=2).reshape(P, 16)   # [p][k]
                    D = B @ self.A2[b][s].T                                   # [p][row]
                S2 = D[:, :8] + 128 * D[:, 8:]
                assert S2.min() >= 0 and S2.max() < (1 << 26)
                r = S2 - ((S2 * BAR_EXACT) >> 38) * Q
                for a in range(8):
                    out[:, 16 * b + 2 * a + s] = r[:, a]
        assert out.min() >= 0 and out.max() < Q
        return out.astype(np.int16)


class InvModel:
    def __init__(self, words: np.ndarray):
        w = np.asarray(words, dtype=np.uint32)
        sa = w[:2048].reshape(16, 2, 32, 2)
        ca = w[2048:3072].view(np.int32).reshape(16, 2, 32)
        sb = w[3072:3328].reshape(2, 32, 4)
        cbz = w[3840:4096].view(np.int32).reshape(32, 2, 4)
        # stage-B init [i][c] when stage A runs without its bias correction
        self.binit = np.zeros((16, 16), dtype=np.int64)
        for lane in range(32):
            for t in range(2):
                c = 8 * t + 2 * (lane % 4)
                i = lane // 4
                self.binit[i, c], self.binit[i, c + 1] = cbz[lane][t][0], cbz[lane][t][1]
                self.binit[i + 8, c], self.binit[i + 8, c + 1] = cbz[lane][t][2], cbz[lane][t][3]
        sbw = w[3328:3840].reshape(2, 2, 32, 4)
        self.ABw = [[unpack_k32(sbw[g][j]) for j in range(2)] for g in range(2)]
        self.AA = [[unpack_k16(sa[b][s]) for s in range(2)] for b in range(16)]
        self.corr = np.zeros((16, 2, 8), dtype=np.int64)          # [block][parity][row a]
        for b in range(16):
            for s in range(2):
                for lane in range(32):
                    self.corr[b, s, lane // 4] = ca[b][s][lane]
        self.AB = [unpack_k32(sb[g]) for g in range(2)]

    def __call__(self, x: np.ndarray, wide: bool = False, fold: bool = False) -> np.ndarray:
        """wide: the stage-A sums stay unreduced int32 and stage B reads their
        four bytes in two K chunks of 8 blocks (the int32-intermediate kernels).
        fold: stage A without its bias correction, stage B initialised with
        the constant that cancels it (the batch kernels)."""
        x = np.asarray(x, dtype=np.int16).reshape(-1, 256)
        P = x.shape[0]
        u = x.view(np.uint16).astype(np.int64) ^ 0x8000                   # x + 32768
        mid = np.zeros((P, 256), dtype=np.int64)
        for b in range(16):
            for s in range(2):
                v = u[:, [16 * b + 2 * fwd_slot_e(j) + s for j in range(8)]]
                B = np.stack([v & 255, v >> 8], axis=2).reshape(P, 16)
                D = B @ self.AA[b][s].T
                S = D[:, :8] + (0 if fold else self.corr[b, s][None, :]) + 128 * D[:, 8:]
                assert S.min() >= 0 and S.max() < (1 << (24 if wide else 25))
                r = S if wide else S - ((S * BAR_LAZY) >> 32) * Q
                for a in range(8):
                    mid[:, 16 * b + 2 * a + s] = r[:, a]
        m = mid.reshape(P, 16, 16)                                        # [p][m][c]
        if wide:
            D0 = 0
            D1 = 0
            for j in range(2):
                X = np.stack([(m[:, 8 * j:8 * j + 8, :] >> (8 * t)) & 255 for t in range(4)],
                             axis=2).reshape(P, 32, 16)                  # [p][4 m' + byte][c]
                D0 = D0 + np.einsum("ik,pkc->pic", self.ABw[0][j], X)
                D1 = D1 + np.einsum("ik,pkc->pic", self.ABw[1][j], X)
        else:
            X = np.stack([m & 255, m >> 8], axis=2).reshape(P, 32, 16)
            D0 = np.einsum("ik,pkc->pic", self.AB[0], X)
            D1 = np.einsum("ik,pkc->pic", self.AB[1], X)
        S = D0 + 128 * D1 + (self.binit[None, :, :] if fold else 0)
        # centred reduction: floor((S + 1664) / q) from the exact multiplier
        assert S.min() >= 0 and S.max() + 1664 < (1 << 26)
        r = S - (((S + 1664) * BAR_EXACT) >> 38) * Q
        assert r.min() >= -1664 and r.max() <= 1664
        return r.reshape(P, 256).astype(np.int16)
