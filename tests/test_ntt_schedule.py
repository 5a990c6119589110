"""CPU model of the batch kernels' work split and TMA ring (k_ntt_mma in
tk_ntt_mma.cu): units of 8 polynomials split evenly over the CTAs
(u_begin / u_end), tiles of W units per CTA, an S-slot ring with a prologue of
S - 1 loads and a refill of tile k + S - 1 into the slot that held tile k - 1,
and mbarrier waits with parity floor(k / S) & 1.  Every unit must be loaded,
computed and stored exactly once; a refill must target a slot whose tile was
computed and stored; each wait must find the tile its iteration computes."""
import pytest


def simulate(nunits, G, W, S):
    done = [0] * nunits
    counts = []
    for b in range(G):
        u_begin = b * nunits // G
        u_end = (b + 1) * nunits // G
        counts.append(u_end - u_begin)
        nmine = (u_end - u_begin + W - 1) // W
        slot = [None] * S              # tile loaded into each slot, None when free

        def load(k, s):
            assert slot[s] is None, ("refill into a busy slot", b, k, s)
            slot[s] = k

        for t in range(S - 1):         # prologue
            if t < nmine:
                load(t, t)
        slot_i, phase = 0, 0
        for k in range(nmine):
            assert slot[slot_i] == k, ("wait finds another tile", b, k)
            assert phase == (k // S) & 1
            if k + S - 1 < nmine:      # refill: the slot that held tile k - 1
                load(k + S - 1, (slot_i + S - 1) % S)
            for w in range(W):
                unit = u_begin + k * W + w
                if unit < u_end:
                    done[unit] += 1
            slot[slot_i] = None        # computed, stored, store read out
            slot_i += 1
            if slot_i == S:
                slot_i, phase = 0, phase ^ 1
        assert all(s is None for s in slot)
    return done, counts


@pytest.mark.parametrize("W,S", [(4, 2), (4, 3), (8, 3), (8, 2)])
@pytest.mark.parametrize("npoly", [1, 7, 8, 9, 100, 4096, 262144, (1 << 20) + 3])
@pytest.mark.parametrize("cap", [1, 5, 444, 592])
def test_units_once_and_ring_protocol(W, S, npoly, cap):
    nunits = (npoly + 7) // 8
    # launch_variant: one CTA per 8 W polynomials, at most the resident cap
    G = max(1, min(cap, (npoly + 8 * W - 1) // (8 * W)))
    done, counts = simulate(nunits, G, W, S)
    assert all(d == 1 for d in done)
    assert max(counts) - min(counts) <= 1          # even split by units
