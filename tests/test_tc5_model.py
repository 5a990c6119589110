"""CPU model of the tcgen05 kernels (tensorkyber_b200/csrc/tk_tc5.cu).

The library's own B-operand tiles (table 8) are decoded from the tcgen05
K-major layout and pushed through the kernels' integer steps with numpy: the
first stage as a pair of MMAs per block or coefficient (unsigned data against
the low-byte constants, signed data against the high-byte constants) into one
int32 accumulator per constant limb, the recombination S = D_lo + 128 D_hi
plus 2048 q (non-negative, below 2^25), the second stage as two unsigned MMAs
over the four bytes of those sums, and the exact (forward) or centred
(inverse) reduction.  Every coefficient must agree with the oracle mod q, the
intermediate bounds the kernels rely on must hold, and the shared-memory
addresses they read and write must be the TMA 128-byte-swizzle layout of the
tile (the layout its loads and stores use).  No GPU needed."""
import numpy as np

from conftest import rng
from py_oracle import Q, canon

TILE_BYTES = 1024
NTILES = 68           # 0-33 the inverse's, 34-67 the forward's
FIRST_BIAS = 2048 * Q
BAR_EXACT = 82570715  # ceil(2^38 / q)


def tile_offset(n, k):
    return (n >> 3) * 256 + (k >> 4) * 128 + (n & 7) * 16 + (k & 15)


def decode(raw: np.ndarray) -> np.ndarray:
    """The tiles of B[n][k] (n = out + 16 limb, k = K byte), each read back from
    the K-major core-matrix layout; the signed-data tiles (1, 3, .., 31 and
    35) as signed bytes, the others unsigned."""
    raw = raw.view(np.uint8)
    assert raw.size == NTILES * TILE_BYTES
    off = np.array([[tile_offset(n, k) for k in range(32)] for n in range(32)])
    assert sorted(off.ravel().tolist()) == list(range(TILE_BYTES))   # a bijection
    tiles = np.zeros((NTILES, 32, 32), dtype=np.int64)
    for t in range(NTILES):
        b = raw[t * TILE_BYTES:(t + 1) * TILE_BYTES][off]
        signed = (t < 32 and t & 1) or t == 35
        tiles[t] = b.view(np.int8) if signed else b
    return tiles


def as_u8(a):
    return a.astype(np.uint8).astype(np.int64)


def as_s8(a):
    return a.astype(np.uint8).view(np.int8).astype(np.int64)


def first_stage_sums(d):
    """[n][32] accumulators -> S + 2048 q [n][16], non-negative, below 2^25."""
    assert np.abs(d).max() < 2 ** 31
    s = d[:, :16] + 128 * d[:, 16:] + FIRST_BIAS
    assert s.min() >= 0 and s.max() < 2 ** 25
    return s


def second_stage(sums, tiles):
    """sums[n][16] (K byte 4 (v % 8) + j of step v / 8 = byte j of sum v)
    against two unsigned tiles -> S = D_lo + 128 D_hi [n][16], below 2^26."""
    by = sums.astype(np.int32).view(np.uint8).reshape(sums.shape[0], 64).astype(np.int64)
    d = by[:, :32] @ tiles[0].T + by[:, 32:] @ tiles[1].T
    s = d[:, :16] + 128 * d[:, 16:]
    assert s.min() >= 0 and s.max() < 2 ** 26
    return s


def model_inverse(tiles: np.ndarray, x: np.ndarray):
    n = x.shape[0]
    raw = np.ascontiguousarray(x.astype(np.int16)).view(np.uint8).reshape(n, 16, 32)
    Y = np.zeros((n, 16, 16), dtype=np.int64)           # [poly][m][c]
    for m in range(16):
        d = as_u8(raw[:, m]) @ tiles[2 * m].T + as_s8(raw[:, m]) @ tiles[2 * m + 1].T
        Y[:, m] = first_stage_sums(d)
    out = np.zeros((n, 16, 16), dtype=np.int64)         # [poly][i][c]
    for c in range(16):
        s = second_stage(np.ascontiguousarray(Y[:, :, c]), tiles[32:34])
        quot = ((s * BAR_EXACT + 1664 * BAR_EXACT) >> 38)   # red_centred
        out[:, :, c] = s - quot * Q
    assert out.min() >= -(Q // 2) and out.max() <= Q // 2
    return out.reshape(n, 256).astype(np.int16)


def model_forward(tiles: np.ndarray, x: np.ndarray):
    n = x.shape[0]
    X = np.ascontiguousarray(x.astype(np.int16)).reshape(n, 16, 16)   # [p][m][c]
    Y = np.zeros((n, 16, 16), dtype=np.int64)                         # [p][i][c]
    for c in range(16):
        col = np.ascontiguousarray(X[:, :, c]).view(np.uint8).reshape(n, 32)
        d = as_u8(col) @ tiles[34].T + as_s8(col) @ tiles[35].T
        Y[:, :, c] = first_stage_sums(d)
    out = np.zeros((n, 16, 16), dtype=np.int64)                       # [p][i][c']
    for i in range(16):
        s = second_stage(np.ascontiguousarray(Y[:, i, :]), tiles[36 + 2 * i:38 + 2 * i])
        out[:, i] = s - ((s * BAR_EXACT) >> 38) * Q                   # red_exact
    assert out.min() >= 0 and out.max() < Q
    return out.reshape(n, 256).astype(np.int16)


def inputs():
    r = rng(2026)
    x = r.integers(-32768, 32768, size=(200, 256))
    special = [np.full(256, -32768), np.full(256, 32767), np.tile([32767, -32768], 128),
               np.zeros(256), np.full(256, Q - 1), r.integers(0, Q, size=256),
               np.tile([-32768, 32767, 32767, -32768], 64)]
    return np.concatenate([x, np.array(special)]).astype(np.int16)


def limbs(v):
    return np.concatenate([v & 127, v >> 7])


def test_tables_hold_the_stage_matrices(tk):
    """Decoded tiles: limbs of the stage constants (times 256^j on byte j's K
    rows) and zeros on the rows the other MMA kind covers."""
    tiles = decode(tk.get_table(8))
    m1 = tk.get_table(0).astype(np.int64)       # [i][m]
    m2 = tk.get_table(1).astype(np.int64)       # [block][out][in]
    ma = tk.get_table(2).astype(np.int64)       # [m][out][in]
    minv = tk.get_table(3).astype(np.int64)     # [i][m]
    for m in range(16):
        assert (tiles[2 * m][:, 1::2] == 0).all() and (tiles[2 * m + 1][:, 0::2] == 0).all()
        assert (tiles[2 * m][:, 0::2] == limbs(ma[m])).all()
        assert (tiles[2 * m + 1][:, 1::2] == limbs(256 * ma[m] % Q)).all()
    assert (tiles[34][:, 1::2] == 0).all() and (tiles[35][:, 0::2] == 0).all()
    assert (tiles[34][:, 0::2] == limbs(m1)).all()
    assert (tiles[35][:, 1::2] == limbs(256 * m1 % Q)).all()
    for h in range(2):
        for v in range(8):
            for j in range(4):
                w = pow(256, j, Q)
                assert (tiles[32 + h][:, 4 * v + j] == limbs(minv[:, 8 * h + v] * w % Q)).all()
                for i in range(16):
                    assert (tiles[36 + 2 * i + h][:, 4 * v + j] ==
                            limbs(m2[i][:, 8 * h + v] * w % Q)).all()


def test_inverse_model_matches_the_oracle(tk, oracle):
    out = model_inverse(decode(tk.get_table(8)), inputs())
    assert (canon(out) == canon(oracle.invntt(canon(inputs()).astype(np.int16)))).all()


def test_forward_model_matches_the_oracle(tk, oracle):
    out = model_forward(decode(tk.get_table(8)), inputs())
    assert (out == canon(oracle.ntt(canon(inputs()).astype(np.int16)))).all()


def test_first_stage_bias_covers_the_sum_range():
    """The first stage's sums lie in [-16 * 128 (q-1), 16 * 382 (q-1)]
    (16 inputs of unsigned low and signed high bytes against constants below
    q); adding 2048 q makes them non-negative and keeps them below 2^25, so
    their four bytes are unsigned (the top one 0 or 1)."""
    lo, hi = -16 * 128 * (Q - 1), 16 * (255 + 127) * (Q - 1)
    assert lo + FIRST_BIAS >= 0 and hi + FIRST_BIAS < 2 ** 25
    assert (FIRST_BIAS % Q) == 0


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



def test_forward_transposition_layout():
    """In-place transposition of a loaded tile by the four warps of a lane
    quarter: group g (mh = g / 2, ch = g % 2) reads chunks 2 (8 mh + mm) + ch
    (coefficients 8 ch .. 8 ch + 7 of blocks 8 mh .. 8 mh + 7) of its row from
    the swizzled slot and writes c-tile c = 8 ch + cc at 4096 c + (p / 8) 256 +
    (p % 8) 16 + 128 mh, K bytes 16 mh .. 16 mh + 15 = blocks 8 mh .. 8 mh + 7
    of coefficient c.  Checked: the reads cover the slot once, the writes cover
    it once, a K-major no-swizzle descriptor (LBO 128, SBO 256) at 4096 c reads
    back X[m][c] for K byte 2m + b of row p, and the eight lanes of one
    shared-memory wavefront (rows p .. p + 7) touch eight distinct 16-byte
    bank groups on both sides."""
    reads = np.zeros(65536, dtype=np.int64)
    writes = np.zeros(65536, dtype=np.int64)
    for p in range(128):
        for g in range(4):
            mh, ch = g >> 1, g & 1
            for mm in range(8):
                m = 8 * mh + mm
                k = 2 * m + ch
                a = (k >> 3) * 16384 + p * 128 + (((k & 7) ^ (p & 7)) << 4)
                reads[a:a + 16] += 1
                # the 16 bytes are coefficients 8 ch .. 8 ch + 7 of block m
                assert (64 * (k >> 3) * 2 + 16 * (k & 7)) // 32 == m
            for cc in range(8):
                c = 8 * ch + cc
                a = 4096 * c + (p >> 3) * 256 + (p & 7) * 16 + 128 * mh
                writes[a:a + 16] += 1
                for kb in range(16):        # descriptor view of the same byte
                    kbyte = 16 * mh + kb
                    d = 4096 * c + (p // 8) * 256 + (kbyte // 16) * 128 + (p % 8) * 16 + kbyte % 16
                    assert d == a + kb
                    assert kbyte // 2 == 8 * mh + kb // 2          # block m = kbyte / 2
    assert (reads == 1).all() and (writes == 1).all()
    for p0 in range(0, 128, 8):
        for k in range(32):
            groups = {((((k & 7) ^ (p & 7)) << 4) % 128) // 16 for p in range(p0, p0 + 8)}
            assert len(groups) == 8
        assert len({((p & 7) * 16) // 16 for p in range(p0, p0 + 8)}) == 8


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


def test_first_half_of_the_sums_is_the_second_stage_step_zero():
    """The epilogue group g writes first-stage chunk a = g + 4 jj (results
    2a, 2a + 1) into tensor-memory columns 16 n + 2a + u of every output n;
    the second stage's K step h of output n reads the eight columns 16 n + 8 h
    .. + 7.  So the four groups' chunks jj = 0 (the y_half barrier) fill
    exactly the columns of step 0 for every n, and those of jj = 1 exactly
    step 1: step 0 may start after the first half, and the halves never
    share a column."""
    for n in range(16):
        written = {0: set(), 1: set()}
        for g in range(4):
            for jj in range(2):
                a = g + 4 * jj
                for u in range(2):
                    written[jj].add(16 * n + 2 * a + u)
        for h in range(2):
            assert written[h] == set(range(16 * n + 8 * h, 16 * n + 8 * h + 8))
