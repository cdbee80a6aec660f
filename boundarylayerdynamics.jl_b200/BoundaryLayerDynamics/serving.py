"""Served stream of LES requests with continuous batching on one device.

Each request is an independent half-channel LES (rough wall below, free slip
above, static Smagorinsky, forcing on vel1) of one of a few grid sizes, run for
a fixed number of SSP-RK33 steps from its own seeded initial field, roughness
length and forcing.  The server keeps one pool per size class: a batched handle
(``Model(..., members=slots)``) whose member slots hold the requests' states
resident in HBM.  Pool capacities are carved out of an HBM budget, and a
request is admitted when its class has a free slot and its bytes fit in the
budget left.  Requests that arrive while others run join at the next tick: the
new member is loaded, projected and given its rates (``prepare_member``), and its
slot is switched on in the device-side active mask, so the already-captured step
graphs advance it together with the members in flight.  Every pool advances on
its own stream in ticks of ``tick`` steps, so the classes run concurrently on
the device and a small request does not wait for the ticks of a large pool.  A
finished member's slot is switched off and reused.

``Scheduler`` is the host-side admission logic alone (no device), so it can be
tested and reasoned about on its own; ``Server`` binds it to pools of models.
"""

import math
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads

# the served mix: (n, n3) size classes and their probabilities
SIZES = ((64, 32), (128, 64), (192, 96), (256, 128))
PROBS = (0.4, 0.3, 0.2, 0.1)
LES_SIZE = (2 * math.pi, math.pi, 1.0)


@dataclass
class Request:
    rid: int
    size: tuple          # (n, n3): resolution (n, n, n3)
    steps: int
    arrival: float       # seconds after the start of the stream
    z0: float
    forcing: float
    seed: int
    status: str = "pending"      # pending, queued, running, done, rejected, diverged
    error: str = ""
    admitted: float = float("nan")
    done: float = float("nan")
    result: dict = None
    fields: tuple = field(default=None, repr=False)   # physical (u, v, w) initial field

    @property
    def points(self):
        n, n3 = self.size
        return n * n * n3

    @property
    def latency(self):
        return self.done - self.arrival


def spec_for(size, z0=workloads.LES_Z0, forcing=1.0, seed=0, dt=1e-4, steps=500):
    n, n3 = size
    return workloads.les_spec(n, n3, LES_SIZE, seed=seed, z0=z0, forcing=forcing, dt=dt, steps=steps)


def poisson_arrivals(rate, n, seed):
    """Arrival times of a seeded Poisson process of ``rate`` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def make_requests(n, rate, seed=7, sizes=SIZES, probs=PROBS, steps=500, materialize=True):
    """``n`` seeded requests: Poisson arrivals, sizes drawn with ``probs``,
    z0 ~ logU[1e-5, 1e-3] and vel1 forcing ~ U[0.5, 1.5] per request."""
    rng = np.random.default_rng(seed + 1)
    times = poisson_arrivals(rate, n, seed)
    idx = rng.choice(len(sizes), size=n, p=np.asarray(probs) / np.sum(probs))
    z0 = np.exp(rng.uniform(math.log(1e-5), math.log(1e-3), size=n))
    forcing = rng.uniform(0.5, 1.5, size=n)
    reqs = []
    for i in range(n):
        r = Request(rid=i, size=tuple(sizes[idx[i]]), steps=steps, arrival=float(times[i]), z0=float(z0[i]),
                    forcing=float(forcing[i]), seed=seed * 1000 + i)
        if materialize:
            r.fields = initial_fields(r)
        reqs.append(r)
    return reqs


def initial_fields(req):
    """The request's seeded log-law-plus-noise initial field on its default grid."""
    return workloads.initial_fields(spec_for(req.size, z0=req.z0, forcing=req.forcing, seed=req.seed))


def percentile(values, q):
    """Nearest-rank percentile (q in [0, 100])."""
    v = np.sort(np.asarray(values, dtype=float))
    if v.size == 0:
        return float("nan")
    k = max(0, int(math.ceil(q / 100.0 * v.size)) - 1)
    return float(v[k])


class Scheduler:
    """Slots per size class, an HBM budget and a FIFO queue (host logic only).

    ``capacity[size]`` slots exist per class and each occupied slot holds
    ``slot_bytes[size]`` bytes of the budget.  Requests are admitted in arrival
    order; a request whose class is full (or whose bytes do not fit the budget
    left) waits without blocking requests of other classes behind it.  A request
    of an unknown size, or one that could never fit, is rejected at submission.
    """

    def __init__(self, capacity, slot_bytes, budget):
        self.capacity = dict(capacity)
        self.slot_bytes = dict(slot_bytes)
        self.budget = int(budget)
        self.free = {s: list(range(c)) for s, c in self.capacity.items()}
        self.running = {s: {} for s in self.capacity}     # size -> slot -> [request, steps left]
        self.queue = []
        self.resident = 0
        self.peak_resident = 0

    def submit(self, req):
        if req.size not in self.capacity or self.capacity[req.size] < 1:
            req.status, req.error = "rejected", f"no pool serves size {req.size}"
            return False
        if self.slot_bytes[req.size] > self.budget:
            req.status, req.error = "rejected", "request exceeds the HBM budget"
            return False
        if req.steps < 1:
            req.status, req.error = "rejected", "a request needs at least one step"
            return False
        req.status = "queued"
        self.queue.append(req)
        return True

    def admit(self, ready=None):
        """Pops every queued request that fits now (and whose pool is ``ready``,
        when given); returns [(request, size, slot)]."""
        out, keep = [], []
        for r in self.queue:
            need = self.slot_bytes[r.size]
            if (ready is None or ready(r.size)) and self.free[r.size] and self.resident + need <= self.budget:
                slot = self.free[r.size].pop(0)
                self.running[r.size][slot] = [r, r.steps]
                self.resident += need
                self.peak_resident = max(self.peak_resident, self.resident)
                r.status = "running"
                out.append((r, r.size, slot))
            else:
                keep.append(r)
        self.queue = keep
        return out

    def busy(self):
        return [s for s in self.capacity if self.running[s]]

    def mask(self, size):
        m = np.zeros(self.capacity[size], dtype=np.int32)
        for slot in self.running[size]:
            m[slot] = 1
        return m

    def next_tick(self, tick):
        """Steps the next tick may take without running any member past its end."""
        left = [v[1] for s in self.capacity for v in self.running[s].values()]
        return min([tick] + left) if left else 0

    def advance(self, nsteps, size=None):
        """Counts ``nsteps`` steps for every running request (of one pool, when
        ``size`` is given); returns the finished ones."""
        done = []
        for s in (self.capacity if size is None else (size,)):
            for slot, v in list(self.running[s].items()):
                v[1] -= nsteps
                if v[1] <= 0:
                    done.append((v[0], s, slot))
        return done

    def next_tick_of(self, size, tick):
        """Steps the next tick of one pool may take without running a member past its end."""
        left = [v[1] for v in self.running[size].values()]
        return min([tick] + left) if left else 0

    def release(self, size, slot):
        r, _ = self.running[size].pop(slot)
        self.free[size].append(slot)
        self.free[size].sort()
        self.resident -= self.slot_bytes[size]
        return r


def plan_capacity(budget, slot_bytes, probs, max_slots=64):
    """Slots per class from the HBM budget.  Members of every class advance
    together (one step graph per tick for all busy pools), so a request's time in
    the system hardly depends on its size, and by Little's law the number of
    resident requests of a class is proportional to its arrival probability:
    slots are given in proportion to the probabilities, scaled to fill the budget,
    at least one per class."""
    sizes = list(slot_bytes)
    scale = budget / sum(probs[s] * slot_bytes[s] for s in sizes)
    cap = {s: max(1, min(max_slots, int(probs[s] * scale))) for s in sizes}
    while sum(cap[s] * slot_bytes[s] for s in sizes) > budget:
        s = max((s for s in sizes if cap[s] > 1), key=lambda s: cap[s] * slot_bytes[s], default=None)
        if s is None:
            raise ValueError("the HBM budget does not hold one slot of every size class")
        cap[s] -= 1
    return cap


def estimate_slot_bytes(size, precision="mixed", device=0, members=2):
    """Device bytes per member slot of a pool of ``size``: the difference of two
    probe handles with ``members`` and one member (autotuning skipped)."""
    api = sys.modules[__package__]
    import os
    old = os.environ.get("BLD_NO_AUTOTUNE")
    os.environ["BLD_NO_AUTOTUNE"] = "1"
    try:
        one = workloads.build(spec_for(size), api, precision=precision, members=1, device=device)
        b1 = one.info.device_bytes
        del one
        more = workloads.build(spec_for(size), api, precision=precision, members=members, device=device)
        bm = more.info.device_bytes
        del more
    finally:
        if old is None:
            del os.environ["BLD_NO_AUTOTUNE"]
        else:
            os.environ["BLD_NO_AUTOTUNE"] = old
    per = (bm - b1) / (members - 1)
    return int(per), int(b1 - per)


class Server:
    """Continuous-batching server over one pool per size class.

    ``pools``: size -> model-like object with ``members`` slots and the slot API
    (``set_field``, ``set_member_params``, ``prepare_member``, ``set_active``,
    ``get_state``, ``diverged_members``) and asynchronous stepping
    (``step_async``, ``idle``, ``sync``).  Every pool advances on its own stream
    in ticks of up to ``tick`` steps (graph launches) with no host wait: the loop
    only polls which pools finished their tick, harvests their finished requests,
    admits queued requests into pools that are between ticks and launches their
    next tick.  Pools therefore run concurrently on the device and a small
    request is not held back by the ticks of a large pool.
    """

    def __init__(self, pools, slot_bytes, budget, dt=1e-4, tick=10, keep_results=False,
                 clock=time.perf_counter, sleep=time.sleep, poll=1e-4):
        self.pools = dict(pools)
        self.sched = Scheduler({s: p.members for s, p in self.pools.items()}, slot_bytes, budget)
        self.dt = float(dt)
        self.tick = int(tick)
        self.keep_results = keep_results
        self.clock = clock
        self.sleep = sleep
        self.poll = float(poll)
        self.ticks = 0
        self.launch_steps = 0
        for p in self.pools.values():
            p.set_active(np.zeros(p.members, dtype=np.int32))

    @classmethod
    def create(cls, budget, sizes=SIZES, probs=PROBS, precision="mixed", device=0, capacity=None, **kw):
        """Pools for ``sizes`` sized from the HBM ``budget`` (bytes)."""
        api = sys.modules[__package__]
        est = {tuple(s): estimate_slot_bytes(tuple(s), precision, device) for s in sizes}
        slot_bytes = {s: v[0] for s, v in est.items()}
        if capacity is None:
            fixed = sum(v[1] for v in est.values())
            capacity = plan_capacity(budget - fixed, slot_bytes, dict(zip(map(tuple, sizes), probs)))
        pools = {s: workloads.build(spec_for(s), api, precision=precision, members=capacity[s], device=device)
                 for s in est}
        return cls(pools, slot_bytes, budget, **kw)

    def _load(self, req, size, slot):
        pool = self.pools[size]
        u, v, w = req.fields if req.fields is not None else initial_fields(req)
        pool.set_field("vel1", u, member=slot)
        pool.set_field("vel2", v, member=slot)
        pool.set_field("vel3", w, member=slot)
        pool.set_member_params(slot, z0=req.z0, forcing=req.forcing)
        pool.prepare_member(slot)

    def _fail(self, req, size, slot, status, msg):
        req.status, req.error = status, msg
        req.done = self.clock() - self.t0
        self.sched.release(size, slot)

    def run(self, requests):
        """Serves ``requests`` (arrival times relative to the call); returns the statistics."""
        from ._capi import DivergenceError
        pending = sorted(requests, key=lambda r: r.arrival)
        inflight = {s: 0 for s in self.pools}        # steps of the tick on the device, 0 = idle
        self.t0 = self.clock()
        i = 0
        while i < len(pending) or self.sched.queue or self.sched.busy() or any(inflight.values()):
            progressed = False
            now = self.clock() - self.t0
            while i < len(pending) and pending[i].arrival <= now:
                self.sched.submit(pending[i])
                i += 1
            # ticks that finished: divergence check, finished requests, slots freed
            for size, pool in self.pools.items():
                n = inflight[size]
                if not n or not pool.idle():
                    continue
                progressed = True
                inflight[size] = 0
                try:
                    pool.sync()
                except DivergenceError:
                    for slot in pool.diverged_members():
                        if slot in self.sched.running[size]:
                            r = self.sched.running[size][slot][0]
                            self._fail(r, size, slot, "diverged", "The simulation has diverged.")
                finished = self.sched.advance(n, size)
                for req, s, slot in finished:
                    if self.keep_results:
                        req.result = pool.get_state(slot)
                    req.done = self.clock() - self.t0
                    req.status = "done"
                    self.sched.release(s, slot)
                pool.set_active(self.sched.mask(size))
            # admissions into pools between ticks
            changed = set()
            for req, size, slot in self.sched.admit(ready=lambda s: inflight[s] == 0):
                progressed = True
                req.admitted = self.clock() - self.t0
                try:
                    self._load(req, size, slot)
                except DivergenceError as e:
                    self.pools[size].diverged_members()
                    self._fail(req, size, slot, "diverged", str(e))
                    continue
                changed.add(size)
            for size in changed:
                self.pools[size].set_active(self.sched.mask(size))
            # next ticks of the idle pools that hold requests
            for size, pool in self.pools.items():
                if inflight[size] or not self.sched.running[size]:
                    continue
                n = self.sched.next_tick_of(size, self.tick)
                pool.step_async(n, self.dt)
                inflight[size] = n
                self.ticks += 1
                self.launch_steps += n
                progressed = True
            if not progressed:
                if any(inflight.values()):
                    self.sleep(self.poll)
                elif i < len(pending):
                    self.sleep(max(self.poll, pending[i].arrival - (self.clock() - self.t0)))
        return self.stats(requests)

    def stats(self, requests):
        done = [r for r in requests if r.status == "done"]
        lat = [r.latency for r in done]
        t_end = max([r.done for r in done], default=0.0)
        t_start = min([r.arrival for r in requests], default=0.0)
        span = max(t_end - t_start, 1e-12)
        upd = sum(r.points * r.steps for r in done)
        return {
            "requests": len(requests),
            "completed": len(done),
            "rejected": sum(r.status == "rejected" for r in requests),
            "diverged": sum(r.status == "diverged" for r in requests),
            "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else float("nan"),
            "makespan_s": span,
            "updates_per_s": upd / span,
            "ticks": self.ticks,
            "capacity": {f"{s[0]}^2x{s[1]}": self.sched.capacity[s] for s in self.sched.capacity},
            "peak_resident_bytes": self.sched.peak_resident,
            "budget_bytes": self.sched.budget,
        }


def calibrate_rate(server, probs=PROBS, steps=500, load=0.8, sample_steps=20):
    """Arrival rate that offers ``load`` of the pools' measured batched capacity:
    per class, the time of ``sample_steps`` steps with every slot busy, divided by
    the slots, gives the device time of one request; the rate is
    ``load / sum(p_c * steps * t_c)``."""
    per_request = {}
    for size, pool in server.pools.items():
        pool.set_active(np.ones(pool.members, dtype=np.int32))
        for m in range(pool.members):
            pool.set_state({}, member=m)
            pool.prepare_member(m)
        pool.step(2, server.dt)
        pool.sync()
        t = time.perf_counter()
        pool.step(sample_steps, server.dt)
        pool.sync()
        dt = time.perf_counter() - t
        pool.set_active(np.zeros(pool.members, dtype=np.int32))
        per_request[size] = dt / sample_steps * steps / pool.members
    mean = sum(p * per_request[s] for s, p in zip(server.pools, probs))
    return load / mean, per_request


# ----------------------------------------------------------- admission by free HBM
class ElasticScheduler:
    """Admission against the HBM budget that is actually free (host logic only).

    Pools are created on demand, one kind per size class with ``pool_slots[size]``
    member slots holding ``pool_bytes[size]`` bytes, and released when another
    request needs their memory: a queued request takes a free slot of a pool of
    its size; failing that a new pool, if the bytes left allow; failing that the
    pools with no member in flight are released, least recently used first,
    until the new pool fits.  Requests are served first come, first served per
    size without blocking other sizes, except that while the oldest waiting
    request cannot find memory no new pool is created for a later one: free
    slots of existing pools still fill, but a stream of small requests cannot
    starve a large one of the memory the idle pools give back.
    """

    def __init__(self, pool_slots, pool_bytes, budget):
        self.pool_slots = dict(pool_slots)
        self.pool_bytes = dict(pool_bytes)
        self.budget = int(budget)
        self.pools = {}          # pid -> {"size", "free": [slots], "running": {slot: [req, steps left]}, "used"}
        self.queue = []
        self.allocated = 0
        self.peak_resident = 0
        self.created = 0
        self.released = 0
        self._next = 0
        self._clock = 0

    @property
    def resident(self):
        return self.allocated

    def submit(self, req):
        if req.size not in self.pool_slots or self.pool_slots[req.size] < 1:
            req.status, req.error = "rejected", f"no pool serves size {req.size}"
            return False
        if self.pool_bytes[req.size] > self.budget:
            req.status, req.error = "rejected", "request exceeds the HBM budget"
            return False
        if req.steps < 1:
            req.status, req.error = "rejected", "a request needs at least one step"
            return False
        req.status = "queued"
        self.queue.append(req)
        return True

    def _free_pool(self, size, ready):
        for pid, p in self.pools.items():
            if p["size"] == size and p["free"] and ready(pid):
                return pid
        return None

    def _reclaim(self, need, ready, destroy):
        idle = sorted((p["used"], pid) for pid, p in self.pools.items() if not p["running"] and ready(pid))
        if self.allocated - sum(self.pool_bytes[self.pools[pid]["size"]] for _, pid in idle) + need > self.budget:
            return                                   # releasing every idle pool would not be enough
        for _, pid in idle:
            if self.allocated + need <= self.budget:
                break
            self.allocated -= self.pool_bytes[self.pools[pid]["size"]]
            del self.pools[pid]
            self.released += 1
            destroy(pid)

    def admit(self, ready, create, destroy):
        """Admits every queued request that finds a slot now; returns [(request, pid, slot)].
        ``ready(pid)``: the pool is between ticks; ``create(pid, size)`` makes a pool;
        ``destroy(pid)`` frees one."""
        out, keep = [], []
        blocked = False
        self._clock += 1
        for r in self.queue:
            pid = self._free_pool(r.size, ready)
            need = self.pool_bytes[r.size]
            if pid is None and not blocked:
                if self.allocated + need > self.budget:
                    self._reclaim(need, ready, destroy)
                if self.allocated + need <= self.budget:
                    pid = self._next
                    self._next += 1
                    create(pid, r.size)
                    self.pools[pid] = {"size": r.size, "free": list(range(self.pool_slots[r.size])), "running": {},
                                       "used": self._clock}
                    self.allocated += need
                    self.created += 1
                    self.peak_resident = max(self.peak_resident, self.allocated)
            if pid is None:
                blocked = blocked or self.allocated + need > self.budget
                keep.append(r)
                continue
            p = self.pools[pid]
            slot = p["free"].pop(0)
            p["running"][slot] = [r, r.steps]
            p["used"] = self._clock
            r.status = "running"
            out.append((r, pid, slot))
        self.queue = keep
        return out

    def busy(self):
        return [pid for pid, p in self.pools.items() if p["running"]]

    def mask(self, pid):
        p = self.pools[pid]
        m = np.zeros(self.pool_slots[p["size"]], dtype=np.int32)
        for slot in p["running"]:
            m[slot] = 1
        return m

    def next_tick_of(self, pid, tick):
        left = [v[1] for v in self.pools[pid]["running"].values()]
        return min([tick] + left) if left else 0

    def advance(self, nsteps, pid):
        done = []
        for slot, v in list(self.pools[pid]["running"].items()):
            v[1] -= nsteps
            if v[1] <= 0:
                done.append((v[0], pid, slot))
        return done

    def release(self, pid, slot):
        p = self.pools[pid]
        r, _ = p["running"].pop(slot)
        p["free"].append(slot)
        p["free"].sort()
        p["used"] = self._clock
        return r


def pool_slots_for(slot_bytes, target=1 << 30, max_slots=16):
    """Member slots per pool of each size: as many as fit ``target`` bytes (at
    least one, at most ``max_slots``), so that small requests share a pool and a
    released pool gives back a useful amount of memory."""
    return {s: max(1, min(max_slots, int(target // b))) for s, b in slot_bytes.items()}


class ElasticServer:
    """Continuous-batching server whose pools come and go with the load.

    ``factory(size, slots)`` builds a model-like pool (the slot API of
    ``Server``); the ``ElasticScheduler`` decides when pools are created and
    released against the HBM budget.  Every pool advances on its own stream in
    ticks of up to ``tick`` steps; the host loop polls finished ticks, harvests
    finished requests, releases idle pools whose memory a waiting request needs,
    admits requests between ticks and launches the next ticks.
    """

    def __init__(self, factory, pool_slots, pool_bytes, budget, dt=1e-4, tick=10, keep_results=False,
                 clock=time.perf_counter, sleep=time.sleep, poll=1e-4):
        self.factory = factory
        self.sched = ElasticScheduler(pool_slots, pool_bytes, budget)
        self.pools = {}
        self.dt = float(dt)
        self.tick = int(tick)
        self.keep_results = keep_results
        self.clock = clock
        self.sleep = sleep
        self.poll = float(poll)
        self.ticks = 0
        self.launch_steps = 0

    @classmethod
    def create(cls, budget, sizes=SIZES, precision="mixed", device=0, target=1 << 30, **kw):
        """Pools of ``sizes`` created on demand within ``budget`` bytes of HBM."""
        api = sys.modules[__package__]
        est = {tuple(s): estimate_slot_bytes(tuple(s), precision, device) for s in sizes}
        slot_bytes = {s: v[0] for s, v in est.items()}
        slots = pool_slots_for(slot_bytes, target)
        pool_bytes = {s: est[s][1] + slots[s] * est[s][0] for s in est}

        def factory(size, n):
            return workloads.build(spec_for(size), api, precision=precision, members=n, device=device)
        return cls(factory, slots, pool_bytes, budget, **kw)

    def _create(self, pid, size):
        pool = self.factory(size, self.sched.pool_slots[size])
        pool.set_active(np.zeros(pool.members, dtype=np.int32))
        self.pools[pid] = pool

    def _destroy(self, pid):
        del self.pools[pid]

    def _load(self, req, pid, slot):
        pool = self.pools[pid]
        if req.fields is not None:
            u, v, w = req.fields
            pool.set_field("vel1", u, member=slot)
            pool.set_field("vel2", v, member=slot)
            pool.set_field("vel3", w, member=slot)
        else:   # the seeded initial field generated on the device
            workloads.initialize_on_device(spec_for(req.size, z0=req.z0, forcing=req.forcing, seed=req.seed),
                                           pool, req.seed, member=slot)
        pool.set_member_params(slot, z0=req.z0, forcing=req.forcing)
        pool.prepare_member(slot)

    def _fail(self, req, pid, slot, status, msg):
        req.status, req.error = status, msg
        req.done = self.clock() - self.t0
        self.sched.release(pid, slot)

    def run(self, requests):
        """Serves ``requests`` (arrival times relative to the call); returns the statistics."""
        from ._capi import DivergenceError
        pending = sorted(requests, key=lambda r: r.arrival)
        inflight = {}                                   # pid -> steps of its tick on the device
        self.t0 = self.clock()
        i = 0
        while i < len(pending) or self.sched.queue or self.sched.busy() or any(inflight.values()):
            progressed = False
            now = self.clock() - self.t0
            while i < len(pending) and pending[i].arrival <= now:
                self.sched.submit(pending[i])
                i += 1
            for pid, pool in list(self.pools.items()):
                n = inflight.get(pid, 0)
                if not n or not pool.idle():
                    continue
                progressed = True
                inflight[pid] = 0
                try:
                    pool.sync()
                except DivergenceError:
                    for slot in pool.diverged_members():
                        if slot in self.sched.pools[pid]["running"]:
                            r = self.sched.pools[pid]["running"][slot][0]
                            self._fail(r, pid, slot, "diverged", "The simulation has diverged.")
                for req, p, slot in self.sched.advance(n, pid):
                    if self.keep_results:
                        req.result = pool.get_state(slot)
                    req.done = self.clock() - self.t0
                    req.status = "done"
                    self.sched.release(p, slot)
                pool.set_active(self.sched.mask(pid))
            changed = set()

            def destroy(pid):
                inflight.pop(pid, None)
                self._destroy(pid)
            for req, pid, slot in self.sched.admit(ready=lambda p: not inflight.get(p, 0), create=self._create,
                                                   destroy=destroy):
                progressed = True
                req.admitted = self.clock() - self.t0
                try:
                    self._load(req, pid, slot)
                except DivergenceError as e:
                    self.pools[pid].diverged_members()
                    self._fail(req, pid, slot, "diverged", str(e))
                    continue
                changed.add(pid)
            for pid in changed:
                self.pools[pid].set_active(self.sched.mask(pid))
            for pid, pool in self.pools.items():
                if inflight.get(pid, 0) or not self.sched.pools[pid]["running"]:
                    continue
                n = self.sched.next_tick_of(pid, self.tick)
                pool.step_async(n, self.dt)
                inflight[pid] = n
                self.ticks += 1
                self.launch_steps += n
                progressed = True
            if not progressed:
                if any(inflight.values()):
                    self.sleep(self.poll)
                elif i < len(pending):
                    self.sleep(max(self.poll, pending[i].arrival - (self.clock() - self.t0)))
        return self.stats(requests)

    def stats(self, requests):
        done = [r for r in requests if r.status == "done"]
        lat = [r.latency for r in done]
        t_end = max([r.done for r in done], default=0.0)
        t_start = min([r.arrival for r in requests], default=0.0)
        span = max(t_end - t_start, 1e-12)
        upd = sum(r.points * r.steps for r in done)
        return {
            "requests": len(requests),
            "completed": len(done),
            "rejected": sum(r.status == "rejected" for r in requests),
            "diverged": sum(r.status == "diverged" for r in requests),
            "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else float("nan"),
            "makespan_s": span,
            "updates_per_s": upd / span,
            "ticks": self.ticks,
            "slots_per_pool": {f"{s[0]}^2x{s[1]}": n for s, n in self.sched.pool_slots.items()},
            "pools_created": self.sched.created,
            "pools_released": self.sched.released,
            "peak_resident_bytes": self.sched.peak_resident,
            "budget_bytes": self.sched.budget,
        }


def calibrate_rate_elastic(server, probs=PROBS, steps=500, load=0.8, sample_steps=20):
    """``calibrate_rate`` for an ``ElasticServer``: one full pool per size class is
    built, timed with every slot busy and released again."""
    per_request = {}
    for size in server.sched.pool_slots:
        pool = server.factory(size, server.sched.pool_slots[size])
        pool.set_active(np.ones(pool.members, dtype=np.int32))
        for m in range(pool.members):
            pool.set_state({}, member=m)
            pool.prepare_member(m)
        pool.step(2, server.dt)
        pool.sync()
        t = time.perf_counter()
        pool.step(sample_steps, server.dt)
        pool.sync()
        per_request[size] = (time.perf_counter() - t) / sample_steps * steps / pool.members
        del pool
    mean = sum(p * per_request[s] for s, p in zip(server.sched.pool_slots, probs))
    return load / mean, per_request
