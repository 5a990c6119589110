"""CPU model of the tcgen05 kernels' synchronisation
(tensorkyber_b200/csrc/tk_tc5.cu, k_tc5): the producer thread (TMA loads and
stores over three slots), two MMA-issuing threads (groups j and j + 2 each),
and 16 epilogue warps in four groups, exchanging through mbarriers with the
kernel's parity waits.  Random interleavings and random completion delays of
the asynchronous work (TMA loads, store reads, MMAs) are run for several tile
counts and both directions.  Checked: every run completes; every wait sees
exactly the phase it means (the parity never laps); and each shared resource
is written only after its previous readers are done:
  * slot s: a tile's load only after the previous tile's store has been read
    out; its output written only after every first-stage MMA that reads it
    (or the forward's transposed copy of it) has completed;
  * accumulator buffer g: MMAs only after the group released its previous
    contents; the group reads only completed results;
  * the first stage's sums in tensor memory: written for tile k only after
    every second-stage MMA of tile k - 1 (both issuers) has completed; each
    second-stage K step (h = 0 reads the sums of first-stage chunks 0-3, h =
    1 those of chunks 4-7) only after all 16 warps wrote its half: h = 0 of
    a tile's first two second-stage chunks runs while the other half is
    still being written.
No GPU."""
import random

import pytest

SLOTS, GROUPS, EPI_WARPS, ISSUERS = 3, 4, 16, 2


class Bar:
    def __init__(self, count):
        self.count, self.pending, self.done = count, 0, 0

    def arrive(self):
        self.pending += 1
        assert self.pending <= self.count
        if self.pending == self.count:
            self.pending, self.done = 0, self.done + 1

    def ready(self, parity, phase):
        """mbarrier try_wait.parity: true once the phase with that parity has
        completed.  `phase` is the completion the waiter means: it must never
        be lapped (two completions ahead, or behind by one)."""
        assert parity == phase & 1
        r = (self.done & 1) != parity
        if r:
            assert self.done == phase + 1, (self.done, phase)
        else:
            assert self.done == phase, (self.done, phase)
        return r


class Sim:
    def __init__(self, ntiles, inverse, seed):
        self.rng = random.Random(seed)
        self.n, self.inv = ntiles, inverse
        self.in_full = [Bar(1) for _ in range(SLOTS)]
        self.out_ready = [Bar(EPI_WARPS) for _ in range(SLOTS)]
        self.d_full = [Bar(1) for _ in range(GROUPS)]
        self.d_empty = [Bar(4) for _ in range(GROUPS)]
        self.y_full, self.x_ready, self.x_read = Bar(EPI_WARPS), Bar(EPI_WARPS), Bar(EPI_WARPS)
        self.y_half = Bar(EPI_WARPS)
        self.y_free, self.drain = Bar(ISSUERS), Bar(ISSUERS)
        self.events = []                      # pending asynchronous completions
        self.mma_pending = [[] for _ in range(ISSUERS)]   # per issuer, in issue order
        # resource state
        self.slot_tile = [None] * SLOTS       # tile whose data the slot holds
        self.slot_store_reading = [False] * SLOTS
        self.slot_readers = [0] * SLOTS       # first-stage MMAs not yet completed
        self.buf_unread = [False] * GROUPS    # results written, not yet read out
        self.buf_writers = [0] * GROUPS       # MMAs in flight into the buffer
        self.y_writes = {}                    # tile -> warps that wrote its sums
        self.y_half_writes = {}               # tile -> warps that wrote the first half
        self.y_readers = {}                   # tile -> its second-stage MMAs in flight

    # asynchronous work ------------------------------------------------------
    def later(self, fn):
        self.events.append(fn)

    def mma(self, issuer, kind, g, slot, tile):
        """An MMA into buffer g; kind 'a' reads the slot, 'b0' / 'b1' read the
        first / second half of the sums of `tile` (second-stage K step h)."""
        assert not self.buf_unread[g], "MMA overwrites results the group has not read"
        self.buf_writers[g] += 1
        if kind == 'a':
            self.slot_readers[slot] += 1
        else:
            written = self.y_half_writes if kind == 'b0' else self.y_writes
            assert len(written.get(tile, ())) == EPI_WARPS, "second stage before its sums"
            self.y_readers[tile] = self.y_readers.get(tile, 0) + 1
        self.mma_pending[issuer].append((kind, g, slot, tile))

    def commit(self, issuer, bar, mark_buf=None):
        """The barrier arrives once every MMA this issuer issued before has
        completed (they complete in issue order, after random delays)."""
        upto = len(self.mma_pending[issuer])
        self.mma_pending[issuer].append(('commit', bar, mark_buf, upto))

    def step_mma(self):
        """Complete the oldest MMA (or commit) of a random issuer."""
        live = [i for i in range(ISSUERS) if self.mma_pending[i]]
        if not live:
            return False
        q = self.mma_pending[self.rng.choice(live)]
        op = q.pop(0)
        if op[0] == 'commit':
            _, bar, mark_buf, _ = op
            if mark_buf is not None:
                self.buf_unread[mark_buf] = True
            bar.arrive()
        else:
            kind, g, slot, tile = op
            self.buf_writers[g] -= 1
            if kind == 'a':
                self.slot_readers[slot] -= 1
            else:
                self.y_readers[tile] -= 1
        return True

    # agents (generators yielding a readiness predicate) ---------------------
    def producer(self):
        def load(k):
            s = k % SLOTS
            assert not self.slot_store_reading[s] and self.slot_readers[s] == 0
            self.slot_tile[s] = ('loading', k)

            def land():
                self.slot_tile[s] = ('in', k)
                self.in_full[s].arrive()
            self.later(land)
        for k in range(min(SLOTS, self.n)):
            load(k)
        for k in range(self.n):
            s = k % SLOTS
            yield lambda: self.out_ready[s].ready((k // SLOTS) & 1, k // SLOTS)
            assert self.slot_tile[s] == ('out', k)
            self.slot_store_reading[s] = True
            done = []

            def read_out():
                self.slot_store_reading[s] = False
                done.append(1)
            self.later(read_out)
            yield lambda: bool(done)          # bulk_wait_read
            if k + SLOTS < self.n:
                load(k + SLOTS)

    def issuer(self, j):
        for k in range(self.n):
            s = k % SLOTS
            if self.inv:
                yield lambda: self.in_full[s].ready((k // SLOTS) & 1, k // SLOTS)
                assert self.slot_tile[s] == ('in', k)
            else:
                yield lambda: self.x_ready.ready(k & 1, k)
                assert self.slot_tile[s] == ('transposed', k)
            def take(g, pos):
                if k > 0 or pos > 0:
                    ph = 4 * k + pos - 1
                    return lambda: self.d_empty[g].ready(ph & 1, ph)
                return lambda: True
            for c in range(4):                    # first stage
                g, jj = j + 2 * (c & 1), c >> 1
                yield take(g, jj)
                for _ in range(4):
                    self.mma(j, 'a', g, s, k)
                self.commit(j, self.d_full[g], mark_buf=g)
            # second stage: K step 0 of chunks c = 0, 1 once the first half
            # of the sums is written, the rest once all of them are
            yield lambda: self.y_half.ready(k & 1, k)
            for c in range(2):
                g = j + 2 * c
                yield take(g, 2)
                for _ in range(2):
                    self.mma(j, 'b0', g, s, k)
            yield lambda: self.y_full.ready(k & 1, k)
            for c in range(2):
                g = j + 2 * c
                for _ in range(2):
                    self.mma(j, 'b1', g, s, k)
                self.commit(j, self.d_full[g], mark_buf=g)
            for c in range(2):
                g = j + 2 * c
                yield take(g, 3)
                for _ in range(2):
                    self.mma(j, 'b0', g, s, k)
                for _ in range(2):
                    self.mma(j, 'b1', g, s, k)
                self.commit(j, self.d_full[g], mark_buf=g)
            self.commit(j, self.y_free)
        self.commit(j, self.drain)
        yield lambda: self.drain.ready(0, 0)

    def epi(self, w):
        g = w >> 2
        use = [0]

        def take():
            ph = use[0]
            use[0] += 1
            return lambda: self.d_full[g].ready(ph & 1, ph)

        def read_out():
            assert self.buf_unread[g] and self.buf_writers[g] == 0, "read before completion"

        def give_back(last_of_group):
            # the group's buffer is free once all four warps read it
            self.reads[g] += 1
            if self.reads[g] == 4:
                self.reads[g] = 0
                self.buf_unread[g] = False
            self.d_empty[g].arrive()

        def transpose(t):
            s = t % SLOTS
            yield lambda: self.in_full[s].ready((t // SLOTS) & 1, t // SLOTS)
            assert self.slot_tile[s] in (('in', t), ('reading', t))
            self.slot_tile[s] = ('reading', t)
            self.xr[t] = self.xr.get(t, 0) + 1        # this warp's rows read
            self.x_read.arrive()
            yield lambda: self.x_read.ready(t & 1, t)
            # in place: no c-tile row is written before every warp has read
            assert self.xr[t] == EPI_WARPS, "transposition writes before all reads"
            assert self.slot_readers[s] == 0
            self.xt[t] = self.xt.get(t, 0) + 1
            if self.xt[t] == EPI_WARPS:
                self.slot_tile[s] = ('transposed', t)
            self.x_ready.arrive()

        for k in range(self.n):
            s = k % SLOTS
            if not self.inv and k == 0:
                yield from transpose(0)
            for jj in range(2):
                yield take()
                read_out()
                give_back(jj == 1)
                if jj == 0 and k > 0:
                    yield lambda: self.y_free.ready((k - 1) & 1, k - 1)
                # sums of tile k over those of tile k - 1: its second stage is done
                assert self.y_readers.get(k - 1, 0) == 0, "sums overwritten in use"
                if jj == 0:                      # the first half of the sums written
                    self.y_half_writes.setdefault(k, set()).add(w)
                    self.y_half.arrive()
            self.y_writes.setdefault(k, set()).add(w)
            self.y_full.arrive()
            if not self.inv and k + 1 < self.n:
                yield from transpose(k + 1)
            for jj in range(2):
                yield take()
                read_out()
                give_back(jj == 1)
                # output over the slot: every first-stage MMA reading it is done
                assert self.slot_readers[s] == 0
            self.outs[k] = self.outs.get(k, 0) + 1
            if self.outs[k] == EPI_WARPS:
                self.slot_tile[s] = ('out', k)
            self.out_ready[s].arrive()

    def run(self):
        self.reads = [0] * GROUPS
        self.xt, self.xr, self.outs = {}, {}, {}
        agents = [self.producer()] + [self.issuer(j) for j in range(ISSUERS)] + \
            [self.epi(w) for w in range(EPI_WARPS)]
        waiting = [None] * len(agents)
        alive = set(range(len(agents)))
        for i in list(alive):
            try:
                waiting[i] = next(agents[i])
            except StopIteration:
                alive.discard(i)
        steps = 0
        while alive or self.events or any(self.mma_pending):
            steps += 1
            assert steps < 2_000_000, "no progress"
            ready = [i for i in alive if waiting[i]()]
            choices = len(ready) + len(self.events) + (1 if any(self.mma_pending) else 0)
            assert choices > 0, "deadlock"
            pick = self.rng.randrange(choices)
            if pick < len(ready):
                i = ready[pick]
                try:
                    waiting[i] = next(agents[i])
                except StopIteration:
                    alive.discard(i)
            elif pick < len(ready) + len(self.events):
                self.events.pop(pick - len(ready))()
            else:
                self.step_mma()
        assert all(st == ('out', None) or st is None or st[0] == 'out'
                   for st in self.slot_tile)


@pytest.mark.parametrize("inverse", [True, False], ids=["inverse", "forward"])
@pytest.mark.parametrize("ntiles", [1, 2, 3, 4, 7, 14])
def test_protocol_random_interleavings(inverse, ntiles):
    for seed in range(6):
        Sim(ntiles, inverse, 1000 * ntiles + seed).run()


def test_a_lapped_wait_is_detected():
    """The checker itself: a wait for a phase two completions back fails."""
    b = Bar(1)
    b.arrive()
    b.arrive()
    with pytest.raises(AssertionError):
        b.ready(0, 0)
