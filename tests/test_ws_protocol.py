"""CPU: the named-barrier protocol of the warp-specialised sigma kernel
(pyscf-forge_b200/csrc/sigma_ws.cu), restated as the sequence of barrier
operations each warp role executes, run under random schedules: no schedule
deadlocks, no barrier generation mixes two tiles, and no arrival is left
over at the end.  Barrier ids and counts are those of the kernel: 9 = row
setup (all warps), 1+s / 4+s = "D of stage s gathered" / "V of stage s
written" (all warps; one role arrives, the other waits), 7 = movers, 8 = MMA
warps.

The register-split kernel (pyscf-forge_b200/csrc/sigma_wsr.cu) runs the same
sequence on 12 MMA warps and 4 movers; four of its MMA warps (the "tail")
also pass partial sums of the two K halves through a shared buffer indexed
by the parity of the tile count: the second half writes before barrier 8 of
the tile, the first half reads after it.  Its model checks that every read
sees the partial of its own tile."""
import random

import pytest


def _job_lookups(rows):
    """A job-table launch (batch=True) looks up each unit's job first
    (ws_batch_job: two barrier-9 syncs); a gated unit (None) stops there.
    Yields None before each lookup and the tile count of each row."""
    for r in rows:
        yield None
        if r is not None:
            yield from (r if isinstance(r, tuple) else (r,))


def _mma_warp(rows, tail=None, batch=False):
    """tail: None for an MMA warp without partial sums, else (n-tile, K
    half) of a tail warp of the register-split kernel."""
    t = 0  # tiles so far (its parity indexes the partial-sum buffer)
    seq = _job_lookups(rows) if batch else rows
    for r, nch in enumerate(seq):
        if nch is None:
            yield ("sync", 9, None)
            yield ("sync", 9, None)
            continue
        for _ in range(4):  # ws_row_setup (3) + after the fold (1)
            yield ("sync", 9, None)
        for c in range(nch):
            s = c % 3
            yield ("sync", 1 + s, ("D", c))
            if tail is not None and tail[1] == 1:
                yield ("write", (t & 1, tail[0]), (r, c))
            yield ("sync", 8, None)
            if tail is not None and tail[1] == 0:
                yield ("read", (t & 1, tail[0]), (r, c))
            yield ("arrive", 4 + s, ("V", c))
            t += 1


def _mover_warp(rows, batch=False):
    for nch in (_job_lookups(rows) if batch else rows):
        if nch is None:
            yield ("sync", 9, None)
            yield ("sync", 9, None)
            continue
        for _ in range(4):
            yield ("sync", 9, None)
        for c in range(nch + 2):
            yield ("sync", 7, None)
            if 1 <= c <= nch:
                yield ("sync", 7, None)
                yield ("arrive", 1 + (c - 1) % 3, ("D", c - 1))
            if c >= 2:
                yield ("sync", 4 + (c - 2) % 3, ("V", c - 2))


def _run(rows, nwm, nmov, seed, tails=(), batch=False):
    rng = random.Random(seed)
    counts = {9: nwm + nmov, 7: nmov, 8: nwm}
    for s in range(3):
        counts[1 + s] = counts[4 + s] = nwm + nmov
    warps = ([_mma_warp(rows, batch=batch) for _ in range(nwm - len(tails))]
             + [_mma_warp(rows, t, batch) for t in tails] + [_mover_warp(rows, batch) for _ in range(nmov)])
    slots = {}
    cur = [next(w) for w in warps]
    blocked, gen = {}, {b: 0 for b in counts}
    arrived = {b: [] for b in counts}
    done = [False] * len(warps)

    def advance(i):
        try:
            cur[i] = next(warps[i])
        except StopIteration:
            done[i] = True

    while not all(done):
        ready = [i for i in range(len(warps)) if not done[i] and i not in blocked]
        assert ready, "deadlock"
        i = rng.choice(ready)
        op, bid, tag = cur[i]
        if op == "write":
            slots[bid] = tag
            advance(i)
            continue
        if op == "read":
            assert slots.get(bid) == tag, ("partial sum of another tile", bid, slots.get(bid), tag)
            advance(i)
            continue
        arrived[bid].append(tag)
        if op == "sync":
            blocked[i] = (bid, gen[bid])
        else:
            advance(i)
        if len(arrived[bid]) == counts[bid]:
            tags = {t for t in arrived[bid] if t is not None}
            assert len(tags) <= 1, ("a barrier generation mixes tiles", bid, tags)
            for j, (b2, g2) in list(blocked.items()):
                if b2 == bid and g2 == gen[bid]:
                    del blocked[j]
                    advance(j)
            arrived[bid] = []
            gen[bid] += 1
    assert all(not a for a in arrived.values()), "arrivals left over"


@pytest.mark.parametrize("nwm,nmov", [(17, 3), (16, 4), (15, 5), (12, 4), (3, 2)])
def test_ws_barrier_protocol(nwm, nmov):
    for rows in ([1], [2], [3], [1, 4, 2, 7, 3], [5, 1, 1, 6], [10, 9, 8], [0, 3, 0, 0, 2], [0]):
        for seed in range(25):
            _run(rows, nwm, nmov, seed)


def test_wsr_tail_partial_sums():
    """12 MMA warps of which 4 are tail warps ((n-tile, K half) = (0,0),
    (1,0), (0,1), (1,1)) and 4 movers: the shapes of the register-split
    kernel at 16 orbitals."""
    tails = [(0, 0), (1, 0), (0, 1), (1, 1)]
    for rows in ([1], [2], [3], [1, 4, 2, 7, 3], [5, 1, 1, 6], [10, 9, 8]):
        for seed in range(40):
            _run(rows, 12, 4, seed, tails)


@pytest.mark.parametrize("nwm,nmov", [(5, 3), (8, 4), (7, 5), (9, 3), (12, 4)])
def test_ws_job_table_protocol(nwm, nmov):
    """The job-table form at 8..12 orbitals (MMA warps, movers as the kernel
    lays them out): units of live jobs with one row or a spin-symmetric pair
    of rows (a tuple), and gated units (None) that only look up their job."""
    units = ([None], [3, None, 2], [(2, 5), None, None, 4], [None, (1, 0), 6, None, (3, 3)],
             [0, None, (0, 2), 1], [4, 4, None, 4, (7, 1)])
    for rows in units:
        for seed in range(25):
            _run(rows, nwm, nmov, seed, batch=True)
