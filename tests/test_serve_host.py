"""Host logic of the serving layer (admission, batching, ordering) on the CPU.

The GPU pool is replaced by a fake with the same interface whose "step"
completes at once and whose result is a running sum of the system's
gradients, so per-system order and isolation are visible in the results.
"""
import time
from types import SimpleNamespace

import numpy as np
import pytest

from maos_b200 import serve


class FakePool:
    def __init__(self, stype):
        self.type = stype
        self.cap = stype.capacity
        self.owner = [None] * self.cap
        self.queue = {}
        self.inflight = None
        self.state = {}
        self.launches = []

    def free_slots(self):
        return [i for i, o in enumerate(self.owner) if o is None]

    def admit(self, system):
        slot = self.free_slots()[0]
        self.owner[slot] = system
        self.queue[system] = []
        self.state[slot] = np.zeros(self.type.nact)
        return slot

    def release(self, system):
        self.owner[self.owner.index(system)] = None
        self.queue.pop(system, None)

    take_batch = serve.Pool.take_batch

    def try_launch(self, drop_stale=False):
        if self.inflight is not None:
            return []
        batch, dropped = self.take_batch(drop_stale)
        if batch:
            for slot, req in batch:
                self.state[slot] = self.state[slot] + req.grad[: self.type.nact]
            self.launches.append(sorted(s for s, _ in batch))
            self.inflight = batch
        return dropped

    def poll(self, now_fn):
        if self.inflight is None:
            return []
        t = now_fn()
        for slot, req in self.inflight:
            req.result = self.state[slot].copy()
            req.t_done = t
        done = [r for _, r in self.inflight]
        self.inflight = None
        return done

    def close(self):
        pass


def _types(cap=(2, 1)):
    t = []
    for k, c in enumerate(cap):
        tomo = SimpleNamespace(ngrad=8 + k, nx_total=10, pmap=SimpleNamespace(n=4), wfs=[0], fdpcg=None)
        fit = SimpleNamespace(nact=3 + k, thetax=[0.0], floc=SimpleNamespace(n=4), maxit=4)
        t.append(serve.SystemType(f"t{k}", tomo, fit, capacity=c))
    return t


def test_footprint_counts_vectors():
    t = _types()[0]
    assert serve.slot_footprint_bytes(t) == 4 * (6 * 10 + 2 * 8 + 2 * 1 * 4 + 5 * 3 + 2 * 1 * 4)


def test_admission_budget_and_fifo_waiters():
    types = _types((2, 2))
    srv = serve.Server(types, hbm_budget=250, pool_factory=FakePool, slot_bytes=[100, 100])
    assert srv.register(0, 0, 0.0)
    assert srv.register(1, 1, 0.0)
    assert not srv.register(2, 0, 0.0)      # budget: 300 > 250
    assert not srv.register(3, 1, 0.0)      # FIFO: waits behind system 2
    assert srv.used == 200
    srv.release(0, 1.0)
    assert srv.admitted(2) and not srv.admitted(3)
    srv.release(1, 2.0)
    assert srv.admitted(3)
    with pytest.raises(KeyError):
        srv.submit(serve.Request(0.0, 0, 0, np.zeros(8)))
    with pytest.raises(KeyError):
        srv.release(0, 3.0)


def test_capacity_bounds_admission():
    types = _types((1, 1))
    srv = serve.Server(types, hbm_budget=10 ** 9, pool_factory=FakePool)
    assert srv.register(0, 0, 0.0)
    assert not srv.register(1, 0, 0.0)      # pool 0 full
    assert not srv.register(2, 1, 0.0)      # behind the FIFO head
    srv.release(0, 1.0)
    assert srv.admitted(1) and srv.admitted(2)


def test_batches_take_one_request_per_system_in_order():
    types = _types((2, 1))
    srv = serve.Server(types, hbm_budget=10 ** 9, pool_factory=FakePool)
    for s, p in ((0, 0), (1, 0), (2, 1)):
        srv.register(s, p, 0.0)
    g = {s: [np.full(8 + (s == 2), float(10 * s + k)) for k in range(3)] for s in range(3)}
    for k in range(3):
        for s in range(3):
            srv.submit(serve.Request(float(k), s, k, g[s][k]))
    clock = iter(range(100))
    while not srv.idle():
        srv.step(lambda: float(next(clock)))
    srv.step(lambda: 99.0)
    assert len(srv.completed) == 9
    assert srv.pools[0].launches == [[0, 1]] * 3 and srv.pools[1].launches == [[0]] * 3
    for r in srv.completed:
        want = sum(g[r.system][k][: types[srv.system_pool[r.system]].nact] for k in range(r.step + 1))
        np.testing.assert_array_equal(r.result, want)


def test_drop_stale_keeps_newest():
    types = _types((1, 1))
    srv = serve.Server(types, hbm_budget=10 ** 9, pool_factory=FakePool, drop_stale=True)
    srv.register(0, 0, 0.0)
    for k in range(4):
        srv.submit(serve.Request(float(k), 0, k, np.full(8, 1.0 + k)))
    srv.step(lambda: 5.0)
    srv.step(lambda: 6.0)
    assert [r.step for r in srv.completed] == [3]
    assert sorted(r.step for r in srv.dropped) == [0, 1, 2]
    np.testing.assert_array_equal(srv.completed[0].result, np.full(3, 4.0))


def test_run_served_poisson_with_departures():
    types = _types((2, 1))
    rng = np.random.default_rng(0)
    systems = [(k % 2, 2000.0, rng.standard_normal((3, 9))) for k in range(5)]
    srv, done, wall = serve.run_served(types, systems, duration=0.2, hbm_budget=10 ** 9,
                                       steps_per_system=5, seed=2, pool_factory=FakePool)
    assert len(done) == 25
    for sid in range(5):
        rs = sorted((r for r in done if r.system == sid), key=lambda r: r.step)
        assert [r.step for r in rs] == list(range(5))
        nact = types[systems[sid][0]].nact
        acc = np.zeros(nact)
        for k, r in enumerate(rs):
            acc = acc + systems[sid][2][k % 3][:nact]
            np.testing.assert_allclose(r.result, acc)
    st = serve.latency_stats(done)
    assert st["n"] == 25 and st["p99_ms"] >= st["p50_ms"] >= 0
    # waiters got slots as others left (3 systems of type 0 for 2 slots, 2 of type 1 for 1 slot)
    assert len(srv.admit_log) == 5


def test_priorities_favour_cheap_steps():
    t = _types((1, 1))
    t[0].tomo.cfg = SimpleNamespace(tomo_maxit=30)
    t[1].tomo.cfg = SimpleNamespace(tomo_maxit=30)
    t[1].tomo.nx_total = 1000
    assert serve.step_cost(t[0]) < serve.step_cost(t[1])
    p = serve.stream_priorities(t)
    assert p[0] <= p[1]   # lower number = higher priority in CUDA
