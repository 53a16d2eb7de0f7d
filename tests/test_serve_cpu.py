"""Host logic of the serving loop, against a fake batch (no GPU): arrivals,
FIFO admission with back-fill by footprint, retirement and statistics."""
import numpy as np

from hormone_b200 import serve


class FakeBatch:
    """Each simulation needs `cells` units of a pool and finishes after
    ceil(cells/100) steps."""

    def __init__(self, pool):
        self.pool, self.used, self.sims, self.next = pool, 0, {}, 0
        self.max_sims = 64
        self.max_live = 0

    def capacity(self, cfg):
        return int(np.prod(cfg["n"])) <= self.pool

    def add(self, cfg, prims):
        need = int(np.prod(cfg["n"]))
        if self.used + need > self.pool:
            return None
        s = self.next
        self.next += 1
        self.sims[s] = {"need": need, "left": -(-need // 100), "tn": 0}
        self.used += need
        self.max_live = max(self.max_live, len(self.sims))
        return s

    def set_held(self, slots):
        self.held = set(slots)

    def step(self, n):
        for s, v in self.sims.items():
            if s in getattr(self, "held", ()):
                continue
            k = min(n, v["left"])
            v["left"] -= k
            v["tn"] += k

    def poll(self):
        m = self.next + 1
        t, tn, done, err = np.zeros(m), np.zeros(m, int), np.zeros(m, int), np.zeros(m, int)
        for s, v in self.sims.items():
            tn[s], done[s] = v["tn"], v["left"] == 0
        return t, tn, done, err

    def download(self, s):
        return {"tn": self.sims[s]["tn"]}

    def remove(self, s):
        self.used -= self.sims.pop(s)["need"]


def test_request_stream_is_seeded_and_in_range():
    a = serve.make_requests(50, rate=10.0, seed=3, max_cells=16 ** 3)
    b = serve.make_requests(50, rate=10.0, seed=3, max_cells=16 ** 3)
    assert [r.cells for r in a] == [r.cells for r in b]
    assert all(np.diff([r.arrival for r in a]) >= 0)
    for r in a:
        assert 0.05 <= r.cfg["t_end"] <= 0.2
        assert r.cfg["gamma"] in (1.6666666666666667, 1.4, 2.0)
        if r.kind.startswith("riemann"):
            d = r.prims["d"]
            assert 0.01 <= d.min() and d.max() <= 10.0


def test_serving_admits_as_memory_frees_and_reports_latency():
    reqs = serve.make_requests(20, rate=1e9, seed=1, max_cells=4096, min_cells=256)
    fake = FakeBatch(pool=6000)
    stats = serve.serve(reqs, fake, chunk=3, realtime=False)
    assert stats.completed == 20 and stats.failed == 0
    assert fake.max_live >= 2
    assert fake.used == 0 and not fake.sims
    assert all(r.steps == -(-r.cells // 100) for r in reqs)
    s = stats.summary()
    assert s["p99_s"] >= s["p50_s"]


def test_request_larger_than_the_pool_fails_instead_of_blocking():
    reqs = serve.make_requests(3, rate=1e9, seed=2, max_cells=4096, min_cells=2048)
    fake = FakeBatch(pool=1000)
    stats = serve.serve(reqs, fake, chunk=1, realtime=False)
    assert stats.failed == 3 and stats.completed == 0


class TimedFake(FakeBatch):
    """A batch whose step costs time in proportion to the live cells (every
    step advances every live simulation), on a clock of its own."""

    def __init__(self, pool):
        super().__init__(pool)
        self.t = 0.0
        self.peak_cells = 0

    def add(self, cfg, prims):
        s = super().add(cfg, prims)
        if s is not None and len(self.sims) > 1:
            self.peak_cells = max(self.peak_cells, self.used)
        return s

    def step(self, n):
        held = getattr(self, "held", set())
        self.t += n * (sum(v["need"] for s, v in self.sims.items() if s not in held) * 1e-6 + 1e-5)
        super().step(n)


def test_shortest_first_under_a_cell_cap_cuts_the_median_latency():
    """Admitting by estimated work under a cap on the live cells finishes the
    small requests before the large ones run: the median time-to-solution
    falls, every request still completes with the same steps, and the cap
    holds whenever more than one simulation is live."""
    res = {}
    for policy, cap in (("fifo", None), ("sjf", 3000)):
        reqs = serve.make_requests(40, rate=1e9, seed=4, max_cells=4096, min_cells=64)
        fake = TimedFake(pool=10 ** 6)
        stats = serve.serve(reqs, fake, chunk=2, realtime=False, clock=lambda: fake.t, policy=policy,
                            live_cells=cap)
        assert stats.completed == 40 and stats.failed == 0
        assert all(r.steps == -(-r.cells // 100) for r in reqs)
        if cap is not None:
            assert fake.peak_cells <= cap
        res[policy] = stats.summary()
    assert res["sjf"]["p50_s"] < 0.5 * res["fifo"]["p50_s"], res


class CFLFake(TimedFake):
    """Steps to the end grow with the cells along the longest axis (the CFL
    condition), while a step costs time in proportion to the live cells,
    plus a fixed launch cost."""

    def add(self, cfg, prims):
        s = super().add(cfg, prims)
        if s is not None:
            self.sims[s]["left"] = max(int(v) for v in cfg["n"])
        return s

    def step(self, n):
        held = getattr(self, "held", set())
        self.t += n * (sum(v["need"] for s, v in self.sims.items() if s not in held) * 1e-9 + 1e-4)
        FakeBatch.step(self, n)


def shaped_requests(count, seed):
    """Requests with the serving stream's shapes (cells log-uniform from
    256 to 128^3, 1-D/2-D/3-D) but no state: the fake batch needs only n."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        dim = int(rng.integers(1, 4))
        cells = float(np.exp(rng.uniform(np.log(256), np.log(128 ** 3))))
        n_ax = int(min(max(round(cells ** (1.0 / dim)), 8), {1: 16384, 2: 1024, 3: 128}[dim]))
        n = [n_ax if d < dim else 1 for d in range(3)]
        out.append(serve.Request(r, {"n": n, "t_end": 0.1}, {}, 0.0, cells=int(np.prod(n))))
    return out


def test_priority_steps_cut_the_median_latency_and_keep_every_result():
    """Holding the long simulations while the short ones take extra steps:
    each simulation still takes exactly its own steps, and the median
    time-to-solution falls below FIFO's at about the same wall time."""
    res = {}
    for policy in ("fifo", "priority"):
        reqs = shaped_requests(80, seed=4)
        fake = CFLFake(pool=10 ** 9)
        stats = serve.serve(reqs, fake, chunk=8, realtime=False, clock=lambda: fake.t, policy=policy)
        assert stats.completed == 80 and stats.failed == 0
        assert all(r.steps == max(int(v) for v in r.cfg["n"]) for r in reqs)
        res[policy] = stats.summary()
    assert res["priority"]["p50_s"] < 0.8 * res["fifo"]["p50_s"], res
    assert res["priority"]["wall_s"] < 1.05 * res["fifo"]["wall_s"], res


def test_unknown_policy_is_refused():
    import pytest

    with pytest.raises(ValueError):
        serve.serve([], FakeBatch(pool=10), policy="lifo")
