"""A model of the mbarrier protocol of the tensor-core kernel (lakde_b200/csrc/tc.cu,
tc_kernel): the metadata warp, the two gather warps, the converter warps
(which also run the epilogue) and the MMA warp as coroutines, copies and MMA
completions landing asynchronously (copies in any order, MMA completions in
issue order), mbarriers with the hardware's phase-parity wait.  Random
schedules of random row structures must finish without deadlock, and no
buffer (metadata slot, raw stage or A tile, B stage, TMEM accumulator) may be
rewritten before its last reader is done.  E-step / predictive density: two A
tiles filled in place by the gather (rempty = that tile's MMAs done);
M-step: two raw stages and one A tile (rempty = raw stage converted).

The model mirrors the kernel's waits and arrivals one to one; it checks the
protocol's design, not the compiled code (the GPU tests check that)."""

import random

import pytest

NS = 8  # metadata slots (tc.cu: NS)
NGW = 2  # gather warps (tc.cu: NGW)


class Bar:
    """mbarrier: arrival count, transaction bytes, completed phases."""

    def __init__(self, count):
        self.count, self.pending, self.tx, self.completed = count, count, 0, 0

    def arrive(self, tx=0):
        self.tx += tx
        self.pending -= 1
        self._check()

    def complete_tx(self, b):
        self.tx -= b
        self._check()

    def _check(self):
        assert self.pending >= 0, "more arrivals than the phase expects"
        if self.pending == 0 and self.tx == 0:
            self.completed += 1
            self.pending = self.count

    def ready(self, parity):
        # try_wait.parity(P) succeeds once the phase with parity P has completed
        return (self.completed & 1) != parity


def simulate(rows, mode, seed, stall=False):
    """Runs one schedule; returns "ok" or "deadlock" (asserts on early reuse)."""
    rng = random.Random(seed)
    dual = mode != "M"
    mfull = [Bar(32) for _ in range(NS)]
    mempty = [Bar(1) for _ in range(NS)]
    rfull = [Bar(32 * NGW + 1) for _ in range(2)]
    rempty = [Bar(1) for _ in range(2)]
    bfull = [Bar(1) for _ in range(2)]
    bempty = [Bar(1) for _ in range(2)]
    mma_done = [Bar(1) for _ in range(2)]
    conv = [Bar(256) for _ in range(2)]
    events, mmaq = [], []
    slots = [None] * NS
    buf = [None, None]
    landed = [[None] * NGW for _ in range(2)]
    bst = [None, None]
    st = dict(epi_done=-1, conv_done=-1, mma_done=-1)
    tiles = [(r, j == 0, j == n - 1) for r, n in enumerate(rows) for j in range(n)]
    T = len(tiles)

    def producer():
        bpar, bused = [0, 0], [0, 0]
        for i in range(T + 1):
            ms = i % NS
            if i >= NS:
                yield ("wait", mempty[ms], (i // NS - 1) & 1)
            assert st["epi_done"] >= i - NS, ("metadata slot reused before its epilogue", i)
            if i == T:
                slots[ms] = ("stop", i)
            else:
                r, first, last = tiles[i]
                bs = r & 1
                meta = dict(tile=i, row=r, first=first, last=last, bs=bs, bph=None, reused=0)
                if first:
                    meta["bph"], meta["reused"] = bpar[bs], bused[bs]
                    bpar[bs] ^= 1
                    bused[bs] = 1
                slots[ms] = meta
            for _ in range(32):
                mfull[ms].arrive()
            if i == T:
                return
            yield ("step",)

    def gatherer(gw):
        first_tile = True
        for i in range(T + 1):
            ms, s = i % NS, i & 1
            yield ("wait", mfull[ms], (i // NS) & 1)
            meta = slots[ms]
            if isinstance(meta, tuple):
                return
            if i >= 2:
                yield ("wait", rempty[s], (i // 2 - 1) & 1)
            if dual:
                assert st["mma_done"] >= i - 2, ("A tile overwritten under its MMAs", i)
            else:
                assert st["conv_done"] >= i - 2, ("raw stage overwritten before conversion", i)
            if gw == 0 and mode != "M" and meta["first"]:
                if meta["reused"]:
                    yield ("wait", bempty[meta["bs"]], meta["bph"] ^ 1)
                prev = [k for k, tt in enumerate(tiles) if tt[0] == meta["row"] - 2]
                if prev:
                    assert st["mma_done"] >= max(prev), ("B stage overwritten under its MMAs", i)
                bfull[meta["bs"]].arrive(tx=256)

                def wland(b=meta["bs"], row=meta["row"]):
                    bst[b] = row
                    bfull[b].complete_tx(256)

                events.append(wland)
            if gw == 0:
                rfull[s].arrive(tx=64 + (16 if stall and first_tile else 0))
                events.append(lambda s=s: rfull[s].complete_tx(64))
            first_tile = False
            for _ in range(32):
                def rland(s=s, i=i, gw=gw):
                    landed[s][gw] = i
                    if all(x == i for x in landed[s]):
                        buf[s] = i
                    rfull[s].arrive()

                events.append(rland)
            yield ("step",)

    def consumer():
        for t in range(T + 1):
            ms, s = t % NS, t & 1
            yield ("wait", mfull[ms], (t // NS) & 1)
            meta = slots[ms]
            stop = isinstance(meta, tuple)
            if not stop:
                yield ("wait", rfull[s], (t // 2) & 1)
            if not dual and t > 0:
                yield ("wait", mma_done[(t - 1) & 1], ((t - 1) // 2) & 1)
            if t >= 2:  # thread 0 after the top barrier: tile t - 2's epilogue ran
                mempty[(t - 2) % NS].arrive()
            if not stop:
                assert buf[s] == t, ("rows not landed", t)
                if not dual:
                    assert st["mma_done"] >= t - 1, ("A tile rewritten under its MMAs", t)
                st["conv_done"] = t
                for _ in range(256):
                    conv[s].arrive()
            if t > 0:
                if dual:
                    yield ("wait", mma_done[(t - 1) & 1], ((t - 1) // 2) & 1)
                assert st["mma_done"] >= t - 1
                st["epi_done"] = t - 1
            if stop:
                return
            yield ("step",)

    def mma():
        for t in range(T + 1):
            ms, s = t % NS, t & 1
            yield ("wait", mfull[ms], (t // NS) & 1)
            meta = slots[ms]
            if isinstance(meta, tuple):
                return
            if mode != "M" and meta["first"]:
                yield ("wait", bfull[meta["bs"]], meta["bph"])
                assert bst[meta["bs"]] == meta["row"], ("wrong W cores", t)
            yield ("wait", conv[s], (t // 2) & 1)
            assert st["conv_done"] >= t
            assert st["epi_done"] >= t - 2, ("accumulator reused before its epilogue", t)
            if not dual:
                rempty[s].arrive()

            def mland(t=t, s=s, bs=meta["bs"], row=meta["row"], last=meta["last"]):
                if mode != "M":
                    assert bst[bs] == row, ("W cores changed under the MMAs", t)
                if dual:
                    assert buf[s] == t, ("A tile changed under the MMAs", t)
                st["mma_done"] = t
                mma_done[s].arrive()
                if dual:
                    rempty[s].arrive()
                if mode != "M" and last:
                    bempty[bs].arrive()

            mmaq.append(mland)
            yield ("step",)

    actors = [producer()] + [gatherer(gw) for gw in range(NGW)] + [consumer(), mma()]
    waiting = [None] * len(actors)
    alive = [True] * len(actors)
    for _ in range(10**6):
        if not any(alive):
            return "ok"
        progressed = False
        order = list(range(len(actors)))
        rng.shuffle(order)
        for a in order:
            if not alive[a]:
                continue
            if waiting[a] is not None:
                if not waiting[a][1].ready(waiting[a][2]):
                    continue
                waiting[a] = None
            try:
                op = next(actors[a])
                if op[0] == "wait":
                    waiting[a] = op
                progressed = True
            except StopIteration:
                alive[a] = False
                progressed = True
        if events and rng.random() < 0.6:
            events.pop(rng.randrange(len(events)))()
            progressed = True
        if mmaq and rng.random() < 0.4:
            mmaq.pop(0)()
            progressed = True
        if not progressed:
            if events:
                events.pop(rng.randrange(len(events)))()
            elif mmaq:
                mmaq.pop(0)()
            else:
                return "deadlock"
    raise AssertionError("schedule did not finish")


@pytest.mark.parametrize("mode", ["E", "M", "P"])
def test_random_schedules_finish_without_early_reuse(mode):
    for seed in range(150):
        rng = random.Random(seed)
        rows = [rng.randint(1, 4) for _ in range(rng.randint(0, 12))]
        assert simulate(rows, mode, seed) == "ok", (mode, seed, rows)


def test_a_stage_that_never_completes_blocks_the_consumers():
    """The kernel's time-out hook (a stage expecting 16 bytes no copy delivers)
    leaves the consumers waiting; in the kernel that wait is bounded."""
    assert simulate([1, 1], "E", 1, stall=True) == "deadlock"
