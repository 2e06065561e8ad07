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


def _mma_warp(rows, tail=None):
    """tail: None for an MMA warp without partial sums, else (n-tile, K
    half) of a tail warp of the register-split kernel."""
    t = 0  # tiles so far (its parity indexes the partial-sum buffer)
    for r, nch in enumerate(rows):
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


def _mover_warp(rows):
    for nch in rows:
        for _ in range(4):
            yield ("sync", 9, None)
        for c in range(nch + 2):
            yield ("sync", 7, None)
            if 1 <= c <= nch:
                yield ("sync", 7, None)
                yield ("arrive", 1 + (c - 1) % 3, ("D", c - 1))
            if c >= 2:
                yield ("sync", 4 + (c - 2) % 3, ("V", c - 2))


def _run(rows, nwm, nmov, seed, tails=()):
    rng = random.Random(seed)
    counts = {9: nwm + nmov, 7: nmov, 8: nwm}
    for s in range(3):
        counts[1 + s] = counts[4 + s] = nwm + nmov
    warps = ([_mma_warp(rows) for _ in range(nwm - len(tails))] + [_mma_warp(rows, t) for t in tails]
             + [_mover_warp(rows) for _ in range(nmov)])
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
    for rows in ([1], [2], [3], [1, 4, 2, 7, 3], [5, 1, 1, 6], [10, 9, 8]):
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


# ---- register-split kernel with the alpha scatter on the tail warps -------
#
# Big MMA warps: D gathered (sync 1+s), MMA, barrier 8, write V, arrive 4+s.
# Tail warps: D gathered (sync 1+s), MMA, (partials), barrier 8, write their
# V rows, then wait for every V row (sync 4+s), read V for the alpha scatter
# and release the stage (arrive 10+s).  Movers: as above, and before the
# copies of tile c >= 3 of a row they wait for the tail's release of tile
# c-3 (sync 10+s); at the end of a row they wait for the releases of its
# last (up to three) tiles.  The model tracks what each stage holds and who
# still has to read it: a stage is refilled only after both scatters read V.

def _wsr2_bm(rows):
    for r, nch in enumerate(rows):
        for _ in range(4):
            yield ("sync", 9, None)
        for c in range(nch):
            s = c % 3
            yield ("sync", 1 + s, ("D", c))
            yield ("readD", s, (r, c))
            yield ("sync", 8, None)
            yield ("writeV", s, (r, c))
            yield ("arrive", 4 + s, ("V", c))


def _wsr2_tail(rows, who):
    t = 0
    for r, nch in enumerate(rows):
        for _ in range(4):
            yield ("sync", 9, None)
        for c in range(nch):
            s = c % 3
            yield ("sync", 1 + s, ("D", c))
            yield ("readD", s, (r, c))
            if who[1] == 1:
                yield ("write", (t & 1, who[0]), (r, c))
            yield ("sync", 8, None)
            if who[1] == 0:
                yield ("read", (t & 1, who[0]), (r, c))
            yield ("writeV", s, (r, c))
            yield ("sync", 4 + s, ("V", c))
            yield ("readV", s, (r, c))
            yield ("arrive", 10 + s, ("R", c))
            t += 1


def _wsr2_mover(rows):
    for r, nch in enumerate(rows):
        for _ in range(4):
            yield ("sync", 9, None)
        for c in range(nch + 2):
            yield ("sync", 7, None)
            if c < nch:
                if c >= 3:
                    yield ("sync", 10 + c % 3, ("R", c - 3))
                yield ("copy", c % 3, (r, c))
            if 1 <= c <= nch:
                yield ("sync", 7, None)
                yield ("arrive", 1 + (c - 1) % 3, ("D", c - 1))
            if c >= 2:
                yield ("sync", 4 + (c - 2) % 3, ("V", c - 2))
                yield ("readV", (c - 2) % 3, (r, c - 2))
        for t in range(max(0, nch - 3), nch):
            yield ("sync", 10 + t % 3, ("R", t))


def _run_wsr2(rows, seed, nbig=8, ntail=4, nmov=4):
    rng = random.Random(seed)
    nall = nbig + ntail + nmov
    counts = {9: nall, 7: nmov, 8: nbig + ntail}
    for s in range(3):
        counts[1 + s] = counts[4 + s] = nall
        counts[10 + s] = ntail + nmov
    tails = [(0, 0), (1, 0), (0, 1), (1, 1)][:ntail]
    warps = ([_wsr2_bm(rows) for _ in range(nbig)] + [_wsr2_tail(rows, w) for w in tails]
             + [_wsr2_mover(rows) for _ in range(nmov)])
    kinds = ["bm"] * nbig + ["tail"] * ntail + ["mov"] * nmov
    stage = {s: None for s in range(3)}      # what the stage holds: ("D"|"V", tile)
    pending = {s: set() for s in range(3)}   # warps that still have to read V of the stage
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
        if op in ("write", "read"):
            if op == "write":
                slots[bid] = tag
            else:
                assert slots.get(bid) == tag, ("partial sum of another tile", bid, slots.get(bid), tag)
            advance(i)
            continue
        if op == "copy":
            assert not pending[bid], ("stage refilled before its V was read", bid, pending[bid])
            stage[bid] = ("D", tag)
            advance(i)
            continue
        if op == "readD":
            assert stage[bid] == ("D", tag), ("MMA reads a stage that is not its D", bid, stage[bid], tag)
            advance(i)
            continue
        if op == "writeV":
            if stage[bid] != ("V", tag):
                stage[bid] = ("V", tag)
                pending[bid] = {j for j, k in enumerate(kinds) if k != "bm"}
            advance(i)
            continue
        if op == "readV":
            assert stage[bid] == ("V", tag), ("scatter reads a stage that is not its V", bid, stage[bid], tag)
            pending[bid].discard(i)
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


def test_wsr_tail_scatter_protocol():
    """The register-split kernel with the alpha scatter on the tail warps:
    no deadlock, no generation mixing tiles, MMA warps read only D of their
    tile, both scatters read V of their tile, and no stage is refilled while
    a scatter still has to read it."""
    for rows in ([1], [2], [3], [4], [1, 4, 2, 7, 3], [5, 1, 1, 6], [10, 9, 8]):
        for seed in range(40):
            _run_wsr2(rows, seed)
