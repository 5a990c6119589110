"""CPU model of the tcgen05 kernels (tensorkyber_b200/csrc/tk_tc5.cu).

The library's own B-operand tiles (table 8) are decoded from the tcgen05
K-major layout and pushed through the kernel's integer steps with numpy: stage
A as a pair of MMAs per block (unsigned data against the low-byte constants,
signed data against the high-byte constants) into one int32 accumulator per
constant limb, the recombination S = D_lo + 128 D_hi, stage B over the four
bytes of each stage-A sum (bytes 0-2 unsigned, byte 3 signed) and the 40-bit
centred reduction.  Every coefficient must agree with the oracle mod q, the
intermediate bounds the kernel relies on must hold, and the shared-memory
addresses the kernel writes its output to must be the TMA 128-byte-swizzle
layout of the tile (the layout its loads and stores use).  No GPU needed."""
import numpy as np

from conftest import rng
from py_oracle import Q, canon

M40 = 330282857                      # ceil(2^40 / q)
ADD40 = (Q * 65536 + 1664) * M40
TILE_BYTES = 1024


def tile_offset(n, k):
    return (n >> 3) * 256 + (k >> 4) * 128 + (n & 7) * 16 + (k & 15)


NTILES = 102          # 0-35 the inverse's, 36-101 the forward's


def decode(raw: np.ndarray) -> np.ndarray:
    """The tiles of B[n][k] (n = out + 16 limb, k = K byte), each read back from
    the K-major core-matrix layout; even tiles as unsigned, odd as signed."""
    raw = raw.view(np.uint8)
    assert raw.size == NTILES * TILE_BYTES
    off = np.array([[tile_offset(n, k) for k in range(32)] for n in range(32)])
    assert sorted(off.ravel().tolist()) == list(range(TILE_BYTES))   # a bijection
    tiles = np.zeros((NTILES, 32, 32), dtype=np.int64)
    for t in range(NTILES):
        b = raw[t * TILE_BYTES:(t + 1) * TILE_BYTES][off]
        tiles[t] = b.view(np.int8) if t & 1 else b
    return tiles


def as_u8(a):
    return a.astype(np.uint8).astype(np.int64)


def as_s8(a):
    return a.astype(np.uint8).view(np.int8).astype(np.int64)


def model_inverse(tiles: np.ndarray, x: np.ndarray):
    """The kernel's arithmetic on int16 rows x[n][256]; returns (int16 rows,
    stage-A sums, stage-B sums)."""
    n = x.shape[0]
    raw = np.ascontiguousarray(x.astype(np.int16)).view(np.uint8).reshape(n, 16, 32)
    SA = np.zeros((n, 16, 16), dtype=np.int64)          # [poly][m][c]
    for m in range(16):
        d = as_u8(raw[:, m]) @ tiles[2 * m].T + as_s8(raw[:, m]) @ tiles[2 * m + 1].T
        assert np.abs(d).max() < 2 ** 31
        SA[:, m] = d[:, :16] + 128 * d[:, 16:]
    assert SA.min() >= -2 ** 31 and SA.max() < 2 ** 31
    sa32 = SA.astype(np.int32)
    SB = np.zeros((n, 16, 16), dtype=np.int64)          # [poly][i][c]
    for c in range(16):
        by = sa32[:, :, c].copy().view(np.uint8).reshape(n, 64)   # byte j of S[m] at 4m + j
        d = np.zeros((n, 32), dtype=np.int64)
        for h in range(2):
            kb = by[:, 32 * h:32 * h + 32]
            d += as_u8(kb) @ tiles[32 + 2 * h].T + as_s8(kb) @ tiles[33 + 2 * h].T
        assert np.abs(d).max() < 2 ** 31
        SB[:, :, c] = d[:, :16] + 128 * d[:, 16:]
    xx = SB * M40 + ADD40
    assert xx.min() >= 0 and xx.max() < 2 ** 63
    quot = xx >> 40
    r = (SB - quot * Q) & 0xFFFF
    out = np.where(r >= 32768, r - 65536, r).astype(np.int16)
    return out.reshape(n, 256), SA, SB


def inputs():
    r = rng(2026)
    x = r.integers(-32768, 32768, size=(200, 256))
    special = [np.full(256, -32768), np.full(256, 32767), np.tile([32767, -32768], 128),
               np.zeros(256), np.full(256, Q - 1), r.integers(0, Q, size=256),
               np.tile([-32768, 32767, 32767, -32768], 64)]
    return np.concatenate([x, np.array(special)]).astype(np.int16)


def test_tables_hold_the_stage_matrices(tk):
    """Decoded tiles: limbs of MA / 256 MA (stage A) and of Minv 256^j (stage
    B) on their K rows, zero on the rows the other MMA kind covers."""
    tiles = decode(tk.get_table(8))
    ma = tk.get_table(2).astype(np.int64)       # [m][out][in]
    minv = tk.get_table(3).astype(np.int64)     # [i][m]

    def limbs(v):
        return np.concatenate([v & 127, v >> 7])
    for m in range(16):
        assert (tiles[2 * m][:, 1::2] == 0).all() and (tiles[2 * m + 1][:, 0::2] == 0).all()
        assert (tiles[2 * m][:, 0::2] == limbs(ma[m])).all()
        assert (tiles[2 * m + 1][:, 1::2] == limbs(256 * ma[m] % Q)).all()
    for h in range(2):
        for mm in range(8):
            for j in range(4):
                col = minv[:, 8 * h + mm] * pow(256, j, Q) % Q
                u, s = tiles[32 + 2 * h][:, 4 * mm + j], tiles[33 + 2 * h][:, 4 * mm + j]
                assert (u == (limbs(col) if j < 3 else 0)).all()
                assert (s == (limbs(col) if j == 3 else 0)).all()


def test_model_matches_the_oracle_and_bounds_hold(tk, oracle):
    tiles = decode(tk.get_table(8))
    x = inputs()
    out, SA, SB = model_inverse(tiles, x)
    assert SA.min() >= -(2 ** 24) and SA.max() < 2 ** 25
    assert SB.min() >= -(2 ** 16) and SB.max() < 2 ** 26     # red_centred_wide's domain
    assert out.min() >= -(Q // 2) and out.max() <= Q // 2
    want = oracle.invntt(canon(x).astype(np.int16))
    assert (canon(out) == canon(want)).all()


def test_centred_reduction_exact_on_its_domain():
    s = np.concatenate([np.arange(-(2 ** 16), -(2 ** 16) + 100000),
                        rng(5).integers(-(2 ** 16), 2 ** 26, size=2_000_000),
                        np.arange(2 ** 26 - 100000, 2 ** 26)]).astype(np.int64)
    quot = (s * M40 + ADD40) >> 40
    r = (s - quot * Q) & 0xFFFF
    got = np.where(r >= 32768, r - 65536, r)
    t = s % Q
    assert (got == np.where(t > Q // 2, t - Q, t)).all()


def test_output_addresses_are_the_tma_swizzle_layout():
    """The kernel writes coefficients 16 i + c0 .. + 3 of row p (c0 = 0, 4, 8,
    12) as 8 bytes at quarter i / 4, 16-byte chunk (2 (i % 4) + c0 / 8) xor (p
    % 8), byte 8 ((c0 / 4) % 2); TMA's 128-byte swizzle places coefficient e of
    row p at quarter e / 64, row p * 128, chunk ((2 e % 128) / 16) xor (p % 8).
    The two must agree for every coefficient and cover the 64 KiB slot once."""
    seen = np.zeros(65536, dtype=np.int64)
    for p in range(128):
        for i in range(16):
            for c0 in (0, 4, 8, 12):
                chunk = 2 * (i & 3) + (c0 >> 3)
                addr = (i >> 2) * 16384 + p * 128 + ((chunk ^ (p & 7)) << 4) + 8 * ((c0 >> 2) & 1)
                for u in range(4):
                    e = 16 * i + c0 + u
                    w = 2 * (e % 64)
                    tma = (e // 64) * 16384 + p * 128 + (((w // 16) ^ (p % 8)) << 4) + w % 16
                    assert addr + 2 * u == tma
                    seen[tma:tma + 2] += 1
    assert (seen == 1).all()


def test_stage_a_operand_reads_stay_in_its_quarter():
    """Stage A's A descriptor for block m starts 32 (m % 4) bytes into input
    quarter m / 4 (1024-byte aligned, 128 rows of 128 bytes): the 32 K bytes of
    every row are that block's coefficients, read through the same swizzle."""
    for m in range(16):
        start = (m // 4) * 16384 + 32 * (m % 4)
        for r in range(128):
            for k in range(32):
                logical = 32 * (m % 4) + k            # byte of the quarter's row
                phys = (m // 4) * 16384 + r * 128 + (((logical >> 4) ^ (r & 7)) << 4) + (logical & 15)
                assert (m // 4) * 16384 <= phys < (m // 4 + 1) * 16384
                # coefficient of the natural row behind it
                assert (64 * (m // 4) * 2 + logical) // 2 == 16 * m + k // 2
        assert start % 16 == 0


def model_forward(tiles: np.ndarray, x: np.ndarray):
    """The forward kernel's arithmetic: stage 1 per coefficient c from the
    transposed operand (K byte 2m + b = byte b of X[m][c]), stage 2 per block
    i from the bytes of the int32 stage-1 sums, exact reduction to [0, q)."""
    n = x.shape[0]
    X = np.ascontiguousarray(x.astype(np.int16)).reshape(n, 16, 16)   # [p][m][c]
    S1 = np.zeros((n, 16, 16), dtype=np.int64)                          # [p][i][c]
    for c in range(16):
        col = np.ascontiguousarray(X[:, :, c]).view(np.uint8).reshape(n, 32)
        d = as_u8(col) @ tiles[36].T + as_s8(col) @ tiles[37].T
        assert np.abs(d).max() < 2 ** 31
        S1[:, :, c] = d[:, :16] + 128 * d[:, 16:]
    s32 = S1.astype(np.int32)
    S2 = np.zeros((n, 16, 16), dtype=np.int64)                          # [p][i][c']
    for i in range(16):
        by = s32[:, i, :].copy().view(np.uint8).reshape(n, 64)          # byte j of S[c] at 4c + j
        d = np.zeros((n, 32), dtype=np.int64)
        for h in range(2):
            kb = by[:, 32 * h:32 * h + 32]
            t = 38 + 4 * i + 2 * h
            d += as_u8(kb) @ tiles[t].T + as_s8(kb) @ tiles[t + 1].T
        assert np.abs(d).max() < 2 ** 31
        S2[:, i] = d[:, :16] + 128 * d[:, 16:]
    quot = (S2 * M40 + Q * 65536 * M40) >> 40
    r = (S2 - quot * Q) & 0xFFFF
    return r.astype(np.int16).reshape(n, 256), S1, S2


def test_forward_tables_hold_the_stage_matrices(tk):
    tiles = decode(tk.get_table(8))
    m1 = tk.get_table(0).astype(np.int64)       # [i][m]
    m2 = tk.get_table(1).astype(np.int64)       # [block][out][in]

    def limbs(v):
        return np.concatenate([v & 127, v >> 7])
    assert (tiles[36][:, 1::2] == 0).all() and (tiles[37][:, 0::2] == 0).all()
    assert (tiles[36][:, 0::2] == limbs(m1)).all()
    assert (tiles[37][:, 1::2] == limbs(256 * m1 % Q)).all()
    for i in range(16):
        for h in range(2):
            for cc in range(8):
                for j in range(4):
                    col = m2[i][:, 8 * h + cc] * pow(256, j, Q) % Q
                    u, s = tiles[38 + 4 * i + 2 * h][:, 4 * cc + j], tiles[39 + 4 * i + 2 * h][:, 4 * cc + j]
                    assert (u == (limbs(col) if j < 3 else 0)).all()
                    assert (s == (limbs(col) if j == 3 else 0)).all()


def test_forward_model_matches_the_oracle_and_bounds_hold(tk, oracle):
    tiles = decode(tk.get_table(8))
    x = inputs()
    out, S1, S2 = model_forward(tiles, x)
    assert S1.min() >= -(2 ** 24) and S1.max() < 2 ** 25
    assert S2.min() >= -(2 ** 16) and S2.max() < 2 ** 26
    assert out.min() >= 0 and out.max() < Q
    assert (out == canon(oracle.ntt(canon(x).astype(np.int16)))).all()


def test_forward_transposition_layout():
    """In-place transposition of a loaded tile: warp half h reads chunk 2m + h
    (coefficients 8h .. 8h+7 of block m) of its row from the swizzled slot and
    writes c-tile c = 8h + cc at 4096 c + (p / 8) 256 + (p % 8) 16 + 128 kc,
    K bytes 16 kc .. 16 kc + 15 = blocks 8 kc .. 8 kc + 7 of coefficient c.
    Checked: the reads cover the slot once, the writes cover it once, and a
    K-major no-swizzle descriptor (LBO 128, SBO 256) at 4096 c reads back
    X[m][c] for K byte 2m + b of row p."""
    reads = np.zeros(65536, dtype=np.int64)
    writes = np.zeros(65536, dtype=np.int64)
    for p in range(128):
        for h in range(2):
            for m in range(16):
                k = 2 * m + h
                a = (k >> 3) * 16384 + p * 128 + (((k & 7) ^ (p & 7)) << 4)
                reads[a:a + 16] += 1
            for cc in range(8):
                c = 8 * h + cc
                for kc in range(2):
                    a = 4096 * c + (p >> 3) * 256 + (p & 7) * 16 + 128 * kc
                    writes[a:a + 16] += 1
                    for kb in range(16):        # descriptor view of the same byte
                        kbyte = 16 * kc + kb
                        d = 4096 * c + (p // 8) * 256 + (kbyte // 16) * 128 + (p % 8) * 16 + kbyte % 16
                        assert d == a + kb
                        assert kbyte // 2 < 16                      # block m = kbyte / 2
    assert (reads == 1).all() and (writes == 1).all()


def test_forward_output_addresses_are_the_tma_swizzle_layout():
    """Block i of row p (coefficients 16 i .. 16 i + 15) goes to natural chunks
    2i and 2i + 1 through the swizzle: the two 16-byte stores per block cover
    the slot once and agree with TMA's placement of each coefficient."""
    seen = np.zeros(65536, dtype=np.int64)
    for p in range(128):
        for i in range(16):
            for half in range(2):
                k = 2 * i + half
                a = (k >> 3) * 16384 + p * 128 + (((k & 7) ^ (p & 7)) << 4)
                for u in range(8):
                    e = 16 * i + 8 * half + u
                    w = 2 * (e % 64)
                    assert a + 2 * u == (e // 64) * 16384 + p * 128 + (((w // 16) ^ (p % 8)) << 4) + w % 16
                seen[a:a + 16] += 1
    assert (seen == 1).all()
