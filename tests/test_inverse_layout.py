"""Shared-memory layout of the inverse's intermediate in the mma.sync kernels
(tensorkyber_b200/csrc/tk_ntt_mma.cu: k_ntt_mma's inverse, k_matvec_tiles'
inverse).

Stage A (block-wise) writes, per warp-instruction, one 32-bit word per lane:
coefficients 2 g8, 2 g8 + 1 (g8 = lane / 4) of block m = blk0 + 2 p + h of
polynomial 2 q4 (or 2 q4 + 1), q4 = lane % 4, at byte 32 m + 4 (g8 xor 4 hbw)
of the polynomial's 528-byte row, hbw = bit 2 of the warp's first block
(every block of a warp shares it).  Stage B (over m) reads each polynomial
with one ldmatrix.x4.trans: lane l gives the row address 32 m + 16 (l / 16
xor bit 2 of m), m = l % 8 + 8 ((l / 8) % 2), for matrix j = l / 8, which must
hold coefficients 8 (j / 2) .. + 7 of blocks m.  Checked: the reader finds
every word where the writer put it, each 8-row ldmatrix phase touches eight
distinct 16-byte bank groups, and the writes stay conflict-free.  No GPU."""
ROW = 528           # kRowBytes
WARPS = (4, 8)


def written_word_offset(m, g8):
    """Byte offset in the polynomial row of block m's word g8 (coefficients
    2 g8, 2 g8 + 1), as stage A stores it."""
    return 32 * m + 4 * (g8 ^ (4 * ((m >> 2) & 1)))


def test_writer_offsets_follow_the_kernel_rule():
    for W in WARPS:
        per = 16 // W
        for w in range(W):
            blk0 = per * w
            hbw = (blk0 >> 2) & 1
            for b in range(blk0, blk0 + per):
                assert (b >> 2) & 1 == hbw          # uniform within the warp
            for p in range(per // 2):
                for h in range(2):
                    m = blk0 + 2 * p + h
                    for lane in range(32):
                        q4, g8 = lane & 3, lane >> 2
                        stc = ROW * (2 * q4) + 4 * (g8 ^ (4 * hbw))
                        assert stc + 32 * m == ROW * 2 * q4 + written_word_offset(m, g8)


def test_reader_finds_every_word():
    for lane in range(32):
        j = lane >> 3
        m = (lane & 7) + 8 * (j & 1)
        ldt = 32 * m + 16 * ((lane >> 4) ^ ((lane >> 2) & 1))
        # the 16 bytes at ldt are coefficients 8 (j >> 1) .. + 7 of block m
        for g in range(4):                       # words of the row
            c = 8 * (j >> 1) + 2 * g
            assert ldt + 4 * g == written_word_offset(m, c >> 1)


def test_reader_rows_conflict_free():
    for j in range(4):
        groups = set()
        for lane in range(8 * j, 8 * j + 8):
            m = (lane & 7) + 8 * (j & 1)
            ldt = 32 * m + 16 * ((lane >> 4) ^ ((lane >> 2) & 1))
            groups.add((ldt % 128) // 16)
        assert len(groups) == 8


def test_writer_instruction_conflict_free():
    for m in range(16):
        hbw = (m >> 2) & 1
        for r in range(2):                       # the 2 q4 and 2 q4 + 1 stores
            banks = set()
            for lane in range(32):
                q4, g8 = lane & 3, lane >> 2
                addr = ROW * (2 * q4 + r) + 32 * m + 4 * (g8 ^ (4 * hbw))
                banks.add((addr // 4) % 32)
            assert len(banks) == 32


def test_covers_each_block_once():
    seen = {}
    for m in range(16):
        for g8 in range(8):
            off = written_word_offset(m, g8)
            assert 32 * m <= off < 32 * m + 32
            seen[off] = seen.get(off, 0) + 1
    assert sorted(seen) == list(range(0, 512, 4)) and set(seen.values()) == {1}
