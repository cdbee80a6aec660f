"""Host logic of the continuous-batching server (no device): admission by slots
and HBM budget, FIFO without head-of-line blocking across size classes, exact
step counts per request, slot reuse, rejection, percentiles and the seeded
arrival process.  The pools here are fakes that count the steps each slot took,
so the test checks that every request is advanced exactly its own number of
steps no matter which other requests share its pool."""

import math

import numpy as np
import pytest

from BoundaryLayerDynamics import serving as S


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class FakePool:
    """A pool with `members` slots whose "state" is the number of steps taken;
    a tick of n steps keeps it busy for n * cost seconds of the fake clock."""

    def __init__(self, members, clock, cost):
        self.members = members
        self.clock = clock
        self.cost = cost
        self.active = np.zeros(members, dtype=np.int32)
        self.steps = np.zeros(members, dtype=np.int64)
        self.params = {}
        self.loaded = {}
        self.diverge_at = {}
        self.busy_until = 0.0
        self.ticks = 0

    def set_field(self, f, values, member):
        assert self.idle(), "a pool is loaded only between ticks"
        self.loaded.setdefault(member, []).append(f)
        self.steps[member] = 0

    def init_random_field(self, f, base, scale, distribution, seed, member):
        assert self.idle(), "a pool is loaded only between ticks"
        self.loaded.setdefault(member, []).append(f)
        self.steps[member] = 0

    def set_member_params(self, m, cs=None, z0=None, forcing=None):
        self.params[m] = (z0, forcing)

    def prepare_member(self, m):
        pass

    def set_active(self, mask):
        self.active = np.array(mask, dtype=np.int32)

    def get_state(self, m):
        return {"steps": int(self.steps[m]), "params": self.params[m]}

    def step_async(self, n, dt):
        assert self.idle(), "one tick at a time per pool"
        self.steps += n * (self.active != 0)
        self.busy_until = self.clock.t + n * self.cost
        self.ticks += 1

    def idle(self):
        return self.clock.t >= self.busy_until

    def sync(self):
        from BoundaryLayerDynamics._capi import DivergenceError
        self.clock.t = max(self.clock.t, self.busy_until)
        if any(self.active[m] and self.steps[m] >= s for m, s in self.diverge_at.items()):
            raise DivergenceError(-3, "The simulation has diverged.")

    def diverged_members(self):
        out = [m for m, s in self.diverge_at.items() if self.active[m] and self.steps[m] >= s]
        for m in out:
            del self.diverge_at[m]
        return out


def _server(capacity, budget=10**12, slot_bytes=None, tick=10, keep=True):
    clock = FakeClock()
    pools = {s: FakePool(c, clock, cost=1e-4 * s[0] / 64) for s, c in capacity.items()}
    sb = slot_bytes or {s: 10**6 * s[0] for s in capacity}
    srv = S.Server(pools, sb, budget, tick=tick, keep_results=keep, clock=clock, sleep=clock.sleep, poll=1e-5)
    return srv, pools, clock


def _reqs(n, rate, sizes, steps=500, seed=5):
    return S.make_requests(n, rate, seed=seed, sizes=sizes, probs=[1.0 / len(sizes)] * len(sizes), steps=steps,
                           materialize=False)


def test_poisson_arrivals_seeded_and_rate():
    a = S.poisson_arrivals(50.0, 20000, seed=3)
    b = S.poisson_arrivals(50.0, 20000, seed=3)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0)
    assert abs(20000 / a[-1] - 50.0) / 50.0 < 0.03


def test_make_requests_draws():
    reqs = S.make_requests(4000, 10.0, seed=1, materialize=False)
    sizes = [r.size for r in reqs]
    for s, p in zip(S.SIZES, S.PROBS):
        assert abs(sizes.count(s) / len(reqs) - p) < 0.03
    z0 = np.array([r.z0 for r in reqs])
    assert z0.min() >= 1e-5 and z0.max() <= 1e-3
    lz = np.log10(z0)
    assert abs(lz.mean() + 4.0) < 0.05        # log-uniform on [1e-5, 1e-3]
    f = np.array([r.forcing for r in reqs])
    assert f.min() >= 0.5 and f.max() <= 1.5


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert S.percentile(v, 50) == 50
    assert S.percentile(v, 99) == 99
    assert S.percentile(v, 100) == 100
    assert S.percentile([3.0], 99) == 3.0
    assert math.isnan(S.percentile([], 50))


def test_plan_capacity_within_budget():
    sb = {(64, 32): 40e6, (128, 64): 300e6, (192, 96): 1.0e9, (256, 128): 2.4e9}
    probs = dict(zip(S.SIZES, S.PROBS))
    for budget in (5e9, 20e9, 60e9):
        cap = S.plan_capacity(budget, sb, probs)
        assert all(c >= 1 for c in cap.values())
        assert sum(cap[s] * sb[s] for s in sb) <= budget
    cap = S.plan_capacity(60e9, sb, probs)
    assert cap[(64, 32)] > cap[(128, 64)] > cap[(192, 96)] > cap[(256, 128)]   # follows the mix
    with pytest.raises(ValueError):
        S.plan_capacity(1e9, sb, probs)


def test_scheduler_admission_budget_and_fifo():
    a, b = (32, 16), (48, 24)
    sch = S.Scheduler({a: 2, b: 1}, {a: 10, b: 25}, budget=40)
    reqs = [S.Request(i, s, 5, 0.0, 1e-4, 1.0, i) for i, s in enumerate([b, b, a, a, a])]
    for r in reqs:
        assert sch.submit(r)
    got = sch.admit()
    # b takes its only slot (25 bytes); the second b waits without blocking the a
    # requests behind it; one a fits (35 bytes resident), a second would make 45 > 40
    assert [(r.rid, s, slot) for r, s, slot in got] == [(0, b, 0), (2, a, 0)]
    assert [r.rid for r in sch.queue] == [1, 3, 4]
    assert sch.resident == 35
    assert sch.next_tick(10) == 5
    done = sch.advance(5)
    assert sorted(r.rid for r, _, _ in done) == [0, 2]
    for r, s, slot in done:
        sch.release(s, slot)
    assert sch.resident == 0
    got = sch.admit()
    assert [(r.rid, s, slot) for r, s, slot in got] == [(1, b, 0), (3, a, 0)]


def test_scheduler_rejects():
    a = (32, 16)
    sch = S.Scheduler({a: 1}, {a: 100}, budget=50)
    r = S.Request(0, a, 5, 0.0, 1e-4, 1.0, 0)
    assert not sch.submit(r) and r.status == "rejected" and "budget" in r.error
    sch = S.Scheduler({a: 1}, {a: 10}, budget=50)
    r = S.Request(1, (99, 9), 5, 0.0, 1e-4, 1.0, 0)
    assert not sch.submit(r) and r.status == "rejected" and "no pool" in r.error
    r = S.Request(2, a, 0, 0.0, 1e-4, 1.0, 0)
    assert not sch.submit(r) and r.status == "rejected"


def test_server_exact_steps_and_slot_reuse():
    caps = {(32, 16): 3, (48, 24): 2}
    srv, pools, clock = _server(caps, tick=7)
    reqs = _reqs(40, rate=400.0, sizes=list(caps), steps=50)
    st = srv.run(reqs)
    assert st["completed"] == 40 and st["rejected"] == 0
    for r in reqs:
        assert r.result["steps"] == 50, (r.rid, r.result)          # exactly its own steps
        assert r.result["params"] == (r.z0, r.forcing)              # its own parameters
        assert r.done >= r.admitted >= r.arrival
    # continuous batching: some requests ran together in one pool
    assert srv.ticks < sum(math.ceil(50 / 7) for _ in reqs)
    assert srv.ticks == sum(p.ticks for p in pools.values())
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    assert st["updates_per_s"] > 0


def test_server_budget_limits_residency():
    caps = {(32, 16): 4}
    sb = {(32, 16): 100}
    srv, pools, clock = _server(caps, budget=250, slot_bytes=sb, tick=5)
    reqs = _reqs(12, rate=1e6, sizes=[(32, 16)], steps=10)        # all arrive at once
    st = srv.run(reqs)
    assert st["completed"] == 12
    assert st["peak_resident_bytes"] == 200                         # never a third slot
    assert max(int(p.active.sum()) for p in pools.values()) <= 2


def test_server_isolates_a_diverged_member():
    caps = {(32, 16): 3}
    srv, pools, clock = _server(caps, tick=5)
    reqs = _reqs(3, rate=1e6, sizes=[(32, 16)], steps=20)
    pools[(32, 16)].diverge_at[1] = 10                              # the request in slot 1 blows up
    st = srv.run(reqs)
    assert st["diverged"] == 1 and st["completed"] == 2
    bad = [r for r in reqs if r.status == "diverged"][0]
    assert "diverged" in bad.error
    for r in reqs:
        if r.status == "done":
            assert r.result["steps"] == 20


def test_server_pools_advance_independently():
    """A small request finishes while a large pool is still busy with long ticks."""
    small, large = (32, 16), (256, 128)
    clock = FakeClock()
    pools = {small: FakePool(2, clock, cost=1e-5), large: FakePool(2, clock, cost=1e-2)}
    srv = S.Server(pools, {small: 1, large: 1}, 10**9, tick=10, keep_results=True, clock=clock,
                   sleep=clock.sleep, poll=1e-5)
    big = S.Request(0, large, 50, 0.0, 1e-4, 1.0, 0)
    tiny = S.Request(1, small, 50, 0.001, 1e-4, 1.0, 1)
    srv.run([big, tiny])
    assert big.status == tiny.status == "done"
    assert tiny.result["steps"] == 50 and big.result["steps"] == 50
    assert tiny.latency < 0.01 < big.latency          # 50 x 1e-5 s vs 50 x 1e-2 s of device time


# ------------------------------------------------------ admission by free HBM (elastic pools)
def _elastic(slots, pool_bytes, budget, tick=5, costs=None):
    clock = FakeClock()
    made = []

    def factory(size, n):
        p = FakePool(n, clock, cost=(costs or {}).get(size, 1e-4))
        made.append((size, p))
        return p
    srv = S.ElasticServer(factory, slots, pool_bytes, budget, tick=tick, keep_results=True, clock=clock,
                          sleep=clock.sleep, poll=1e-5)
    return srv, clock, made


def test_elastic_scheduler_reclaims_idle_pools_for_a_large_request():
    small, large = (32, 16), (128, 64)
    sch = S.ElasticScheduler({small: 2, large: 1}, {small: 30, large: 100}, budget=100)
    created, destroyed = [], []
    create = lambda pid, size: created.append((pid, size))
    destroy = lambda pid: destroyed.append(pid)
    ready = lambda pid: True
    reqs = [S.Request(i, s, 5, 0.0, 1e-4, 1.0, i) for i, s in enumerate([small, small, small, large, small])]
    for r in reqs:
        assert sch.submit(r)
    got = sch.admit(ready, create, destroy)
    # two small pools (60 of 100 bytes) take the three small requests; the large one
    # does not fit and blocks new pools for the small request behind it, which
    # still finds the free slot of the second small pool
    assert [(r.rid, pid) for r, pid, _ in got] == [(0, 0), (1, 0), (2, 1), (4, 1)]
    assert [r.rid for r in sch.queue] == [3] and sch.allocated == 60
    for r, pid, slot in list(got):
        sch.release(pid, slot)
    got = sch.admit(ready, create, destroy)        # both small pools idle: released, large pool made
    assert destroyed == [0, 1] and [(r.rid, pid) for r, pid, _ in got] == [(3, 2)]
    assert sch.allocated == 100 and sch.peak_resident == 100


def test_elastic_server_serves_a_large_request_between_small_ones():
    small, large = (32, 16), (256, 128)
    srv, clock, made = _elastic({small: 4, large: 1}, {small: 40, large: 100}, budget=120, tick=5,
                                costs={small: 1e-4, large: 1e-3})
    reqs = [S.Request(i, small, 20, 1e-4 * i, 1e-4, 1.0, i) for i in range(10)]
    reqs.append(S.Request(10, large, 20, 2e-4, 1e-4, 1.0, 10))
    reqs += [S.Request(11 + i, small, 20, 3e-4 + 1e-4 * i, 1e-4, 1.0, 11 + i) for i in range(10)]
    st = srv.run(reqs)
    assert st["completed"] == len(reqs) and st["rejected"] == 0
    for r in reqs:
        assert r.result["steps"] == 20
    big = reqs[10]
    assert big.status == "done"
    assert st["peak_resident_bytes"] <= 120
    assert st["pools_released"] >= 1                     # small pools gave their memory back
    assert {s for s, _ in made} == {small, large}


def test_elastic_server_exact_steps_many_sizes():
    sizes = [(32, 16), (48, 24), (64, 32)]
    slots = {(32, 16): 3, (48, 24): 2, (64, 32): 1}
    pb = {(32, 16): 30, (48, 24): 50, (64, 32): 70}
    srv, clock, made = _elastic(slots, pb, budget=150, tick=7)
    reqs = S.make_requests(60, 2000.0, seed=9, sizes=sizes, probs=[1 / 3] * 3, steps=30, materialize=False)
    st = srv.run(reqs)
    assert st["completed"] == 60
    for r in reqs:
        assert r.result["steps"] == 30 and r.result["params"] == (r.z0, r.forcing)
    assert st["peak_resident_bytes"] <= 150
