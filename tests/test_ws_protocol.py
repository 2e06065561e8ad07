"""CPU: the named-barrier protocol of the warp-specialised sigma kernel
(pyscf-forge_b200/csrc/sigma_ws.cu), restated as the sequence of barrier
operations each warp role executes, run under random schedules: no schedule
deadlocks, no barrier generation mixes two tiles, and no arrival is left
over at the end.  Barrier ids and counts are those of the kernel: 9 = row
setup (all warps), 1+s / 4+s = "D of stage s gathered" / "V of stage s
written" (all warps; one role arrives, the other waits), 7 = movers, 8 = MMA
warps."""
import random

import pytest


def _mma_warp(rows):
    for nch in rows:
        for _ in range(4):  # ws_row_setup (3) + after the fold (1)
            yield ("sync", 9, None)
        for c in range(nch):
            s = c % 3
            yield ("sync", 1 + s, ("D", c))
            yield ("sync", 8, None)
            yield ("arrive", 4 + s, ("V", c))


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


def _run(rows, nwm, nmov, seed):
    rng = random.Random(seed)
    counts = {9: nwm + nmov, 7: nmov, 8: nwm}
    for s in range(3):
        counts[1 + s] = counts[4 + s] = nwm + nmov
    warps = [_mma_warp(rows) for _ in range(nwm)] + [_mover_warp(rows) for _ in range(nmov)]
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
