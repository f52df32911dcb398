"""A randomised model of the barrier protocol of the fused inference kernel
(k_sur_infer, two tiles in flight): the weight loader, the MMA issuer, the 16
epilogue warps and the 4 feature/decode warps as interleaved processes, the
tensor-core work as an in-order queue whose commits arrive on mbarriers, and
the bulk copies as transfers that land in any order.  Every run must finish
without a deadlock, no mbarrier wait may pass on a phase other than the one it
waits for (a waiter at most one phase behind), and no MMA may read a buffer
version other than the one it needs or have a buffer rewritten under it.

The model follows the kernel's loops: the loader streams the hidden layers'
stages in the MMAs' order (pair of tiles, layer, slot); the MMAs of layer 0
wait for the slot's features and for the decode of the slot's previous tile,
those of layer L >= 1 for the epilogue of layer L - 1; the epilogues wait for
the MMAs of their layer; the feature warps write tile t + 2's features once
tile t's first layer has read its slot, and decode tile t after its output
layer."""
import random
from collections import Counter

import pytest

K_STAGES, K_LAYER_STAGES = 4, 8


class Bar:
    def __init__(self, name, count):
        self.name, self.count, self.pending, self.completed = name, count, 0, 0

    def arrive(self, n=1):
        self.pending += n
        assert self.pending <= self.count, (self.name, "too many arrivals")
        if self.pending == self.count:
            self.pending = 0
            self.completed += 1


class Pipeline:
    def __init__(self, tiles, seed):
        self.rng = random.Random(seed)
        self.T = tiles
        self.B = {}
        for q in range(K_STAGES):
            self.B[("full", q)] = Bar(("full", q), 1)
            self.B[("empty", q)] = Bar(("empty", q), 1)
        for q in range(2):
            for name, count in (("feat_full", 4), ("x0_free", 1), ("mma_done", 1), ("epi_done", 16),
                                ("out_done", 1), ("out_free", 4)):
                self.B[(name, q)] = Bar((name, q), count)
        self.B["res"] = Bar("res", 1)
        self.B["drain"] = Bar("drain", 1)
        self.tq = []      # tensor-core queue: ("mma", reads, writes) or ("commit", barrier)
        self.copies = []  # bulk copies in flight: (slot, version)
        self.bufs = {("act", 0): None, ("act", 1): None, ("x0", 0): None, ("x0", 1): None,
                     ("acc", 0): None, ("acc", 1): None}
        for q in range(K_STAGES):
            self.bufs[("stage", q)] = None
        self.pending_reads = Counter()
        self.epi_written = Counter()
        self.feat_written = Counter()
        self.decoded = Counter()

    # an mbarrier parity wait: passes once the phase with this parity has
    # completed; the waiter expects completion number k + 1
    def wait_ok(self, bar, parity, k):
        b = self.B[bar]
        ok = (b.completed & 1) != parity
        if ok:
            assert b.completed == k + 1, ("phase overrun or early pass", bar, b.completed, k)
        return ok

    def write(self, buf, version):
        assert self.pending_reads[buf] == 0, ("buffer rewritten under a pending MMA read", buf)
        self.bufs[buf] = version

    def issue_mma(self, reads, writes):
        for r, _ in reads:
            self.pending_reads[r] += 1
        self.tq.append(("mma", reads, writes))

    def step_tensor(self):
        op = self.tq.pop(0)
        if op[0] == "mma":
            for r, v in op[1]:
                assert self.bufs[r] == v, ("MMA read the wrong data", r, self.bufs[r], v)
                self.pending_reads[r] -= 1
            for w, v in op[2]:
                self.bufs[w] = v
        else:
            self.B[op[1]].arrive()

    def pairs(self):
        for p in range((self.T + 1) // 2):
            yield p, range(2 * p, min(2 * p + 2, self.T))

    def loader(self):
        self.copies.append(("res", None))
        si = 0
        for _, tiles in self.pairs():
            for L in (1, 2, 3):
                for _t in tiles:
                    for g in range(K_LAYER_STAGES):
                        slot = si % K_STAGES
                        if si >= K_STAGES:
                            k = si // K_STAGES - 1
                            yield lambda slot=slot, k=k: self.wait_ok(("empty", slot), k & 1, k)
                        self.copies.append((slot, (L, g, si)))
                        si += 1
                        yield None

    def mma(self):
        yield lambda: self.wait_ok("res", 0, 0)
        si = 0
        for _, tiles in self.pairs():
            for L in range(5):
                for t in tiles:
                    q, k = t & 1, t >> 1
                    if L == 0:
                        yield lambda q=q, k=k: self.wait_ok(("feat_full", q), k & 1, k)
                        if k >= 1:
                            yield lambda q=q, k=k: self.wait_ok(("out_free", q), (k - 1) & 1, k - 1)
                        self.issue_mma([(("x0", q), ("feat", t))], [(("acc", q), (t, 0))])
                        self.tq.append(("commit", ("x0_free", q)))
                        self.tq.append(("commit", ("mma_done", q)))
                        yield None
                        continue
                    e = 4 * k + L - 1
                    yield lambda q=q, e=e: self.wait_ok(("epi_done", q), e & 1, e)
                    if L < 4:
                        for g in range(K_LAYER_STAGES):
                            slot, n = si % K_STAGES, si // K_STAGES
                            yield lambda slot=slot, n=n: self.wait_ok(("full", slot), n & 1, n)
                            self.issue_mma([(("act", q), (t, L - 1)), (("stage", slot), (L, g, si))],
                                           [(("acc", q), (t, L))])
                            self.tq.append(("commit", ("empty", slot)))
                            si += 1
                            yield None
                        self.tq.append(("commit", ("mma_done", q)))
                    else:
                        self.issue_mma([(("act", q), (t, 3))], [(("acc", q), (t, 4))])
                        self.tq.append(("commit", ("out_done", q)))
                    yield None
        self.tq.append(("commit", "drain"))
        yield lambda: self.wait_ok("drain", 0, 0)

    def epilogue(self):
        for _, tiles in self.pairs():
            for L in range(4):
                for t in tiles:
                    q, k = t & 1, t >> 1
                    e = 4 * k + L
                    yield lambda q=q, e=e: self.wait_ok(("mma_done", q), e & 1, e)
                    assert self.bufs[("acc", q)] == (t, L), ("epilogue read the wrong accumulator", t, L)
                    yield None
                    assert self.pending_reads[("act", q)] == 0, ("activations written under an MMA", t, L)
                    self.epi_written[(t, L)] += 1
                    if self.epi_written[(t, L)] == 16:
                        self.write(("act", q), (t, L))
                    self.B[("epi_done", q)].arrive()
                    yield None

    def io(self):
        for t in range(min(2, self.T)):
            self.feat_written[t] += 1
            if self.feat_written[t] == 4:
                self.write(("x0", t & 1), ("feat", t))
            self.B[("feat_full", t & 1)].arrive()
            yield None
        for it in range(self.T):
            q, k = it & 1, it >> 1
            if it + 2 < self.T:
                yield lambda q=q, k=k: self.wait_ok(("x0_free", q), k & 1, k)
                assert self.pending_reads[("x0", q)] == 0, ("features written under an MMA", it + 2)
                self.feat_written[it + 2] += 1
                if self.feat_written[it + 2] == 4:
                    self.write(("x0", q), ("feat", it + 2))
                self.B[("feat_full", q)].arrive()
                yield None
            yield lambda q=q, k=k: self.wait_ok(("out_done", q), k & 1, k)
            assert self.bufs[("acc", q)] == (it, 4), ("decode read the wrong accumulator", it)
            self.B[("out_free", q)].arrive()
            self.decoded[it] += 1
            yield None

    def run(self):
        roles = {"load": self.loader(), "mma": self.mma()}
        for w in range(16):
            roles[("epi", w)] = self.epilogue()
        for w in range(4):
            roles[("io", w)] = self.io()
        blocked = {r: None for r in roles}
        while roles or self.tq or self.copies:
            choices = [("role", r) for r in roles if blocked[r] is None or blocked[r]()]
            if self.tq:
                choices.append(("tensor", None))
            if self.copies:
                choices.append(("copy", None))
            assert choices, ("deadlock", sorted(map(str, roles)))
            kind, r = self.rng.choice(choices)
            if kind == "tensor":
                self.step_tensor()
            elif kind == "copy":
                i = self.rng.randrange(len(self.copies)) if self.rng.random() < 0.3 else 0
                slot, v = self.copies.pop(i)
                if slot == "res":
                    self.B["res"].arrive()
                else:
                    self.write(("stage", slot), v)
                    self.B[("full", slot)].arrive()
            else:
                blocked[r] = None
                try:
                    blocked[r] = next(roles[r])
                except StopIteration:
                    del roles[r], blocked[r]
        assert self.decoded == Counter({t: 4 for t in range(self.T)})


@pytest.mark.parametrize("tiles", [0, 1, 2, 3, 4, 5, 8, 13])
def test_pipeline_model_has_no_deadlock_or_hazard(tiles):
    for seed in range(12):
        Pipeline(tiles, seed * 7919 + tiles).run()


class WithoutOutFree(Pipeline):
    """A broken protocol: a slot's next first layer does not wait for the
    decode of the slot's previous tile, so it may overwrite the accumulator
    the decode has not read yet."""

    def wait_ok(self, bar, parity, k):
        if isinstance(bar, tuple) and bar[0] == "out_free":
            return True
        return super().wait_ok(bar, parity, k)


def test_pipeline_model_catches_a_missing_wait():
    caught = 0
    for seed in range(40):
        try:
            WithoutOutFree(6, seed).run()
        except AssertionError:
            caught += 1
    assert caught > 0
