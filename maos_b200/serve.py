"""Serving: many concurrent AO systems of mixed sizes on one GPU.

No counterpart in the reference, which runs one reconstructor per simulation
(``curecon_t``, cuda/recon.cu:477).  Here each system type (e.g. 8 m SCAO,
8 m LTAO, 30 m MCAO) owns a *pool*: one reconstructor whose ``capacity``
instance slots share that type's operator tables, with every slot's
warm-start state (layer OPD, DM commands) kept on the device between its
steps.  A system is *admitted* into a free slot when the device-memory
footprint of the admitted set stays within the budget; otherwise it waits
until another system leaves.  Requests (one reconstruction step each) arrive
from the systems as independent streams, and the server loop batches
continuously:

* whenever a pool is idle and has queued requests, it takes the oldest queued
  step of every system that has one (or, with ``drop_stale``, the newest,
  counting the older ones as dropped frames), writes those gradients into the
  systems' slots, marks exactly those slots active and launches one graph of
  tomography + fit on the pool's own stream (``mb_recon_serve_step``: the
  uploads, the masked step and the downloads in one call);
* pools run on separate streams, so batches of different sizes overlap on the
  device; the streams carry priorities by step cost (cheapest highest), so
  short steps are not queued behind long ones on the SMs;
* requests that arrive while a batch is in flight wait for the next one;
* when a batch completes, each active slot's DM commands have been copied
  back and the request's latency (arrival to result on the host) is recorded.

Inactive slots are skipped by every kernel (their blocks return at once), so
a system's result does not depend on which other systems share its batch.
"""
from __future__ import annotations

import heapq
import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np


@dataclass
class SystemType:
    name: str
    tomo: object       # geometry.TomoSystem
    fit: object        # fit_setup.FitSystem
    capacity: int

    @property
    def ngrad(self) -> int:
        return int(self.tomo.ngrad)

    @property
    def nact(self) -> int:
        return int(self.fit.nact)


@dataclass(order=True)
class Request:
    t_arrival: float
    system: int = field(compare=False)
    step: int = field(compare=False)
    grad: np.ndarray = field(compare=False, repr=False)
    t_done: float = field(default=math.nan, compare=False)
    result: Optional[np.ndarray] = field(default=None, compare=False, repr=False)
    dropped: bool = field(default=False, compare=False)


def step_cost(stype: SystemType) -> float:
    """Relative device work of one step of one system (unknowns x iterations)."""
    t = stype.tomo
    return float(t.nx_total) * (t.cfg.tomo_maxit + 2) + float(stype.nact) * (stype.fit.maxit + 2)


def stream_priorities(types: List[SystemType]) -> List[int]:
    """CUDA stream priority per pool: the cheapest system type gets the
    highest priority, so short steps are not queued behind long ones on the
    SMs (shortest job first); distinct costs map onto the device's range."""
    try:
        import torch
        least, greatest = torch.cuda.Stream.priority_range()
    except Exception:
        least, greatest = 0, 0
    order = sorted(set(step_cost(t) for t in types))
    levels = list(range(greatest, least + 1))  # greatest (highest priority) first
    out = []
    for t in types:
        k = order.index(step_cost(t))
        out.append(levels[min(k, len(levels) - 1)] if len(order) > 1 else least)
    return out


def slot_footprint_bytes(stype: SystemType) -> int:
    """Device bytes one slot of this type holds (vectors, scratch, spectra)."""
    t = stype.tomo
    nx, ng, npup, nw = t.nx_total, t.ngrad, t.pmap.n, len(t.wfs)
    f = stype.fit
    floats = 6 * nx + 2 * ng + 2 * nw * npup + 5 * f.nact + 2 * len(f.thetax) * f.floc.n
    if getattr(t, "fdpcg", None) is not None:
        floats += 4 * nx  # two complex64 spectra
    return 4 * int(floats)


class Pool:
    """One reconstructor with `capacity` slots for one system type."""

    def __init__(self, stype: SystemType, device: int = 0, priority: int = 0, autotune: bool = False):
        import torch
        from .recon import Reconstructor
        self.type = stype
        self.cap = stype.capacity
        self.R = Reconstructor(stype.tomo, nbatch=self.cap, fit=stype.fit, device=device)
        # autotune (off by default): it tunes the full-capacity step alone on
        # the GPU, while a pool serves masked partial batches beside other
        # pools; its choice of programmatic dependent launch there cost the
        # 30 m pool of the served mix (p99 10 ms against 6.4 ms untuned)
        if autotune:
            self.R.autotune(reps=5)
        self.stream = torch.cuda.Stream(device=device, priority=priority)
        self.owner: List[Optional[int]] = [None] * self.cap
        self.queue: Dict[int, List[Request]] = {}
        self.inflight: Optional[Tuple[object, List[Tuple[int, Request]]]] = None
        self.g_host = torch.empty(self.cap * stype.ngrad, dtype=torch.float32).pin_memory()
        self.a_host = torch.empty(self.cap * stype.nact, dtype=torch.float32).pin_memory()
        self.batches = 0
        self.slot_steps = 0

    def free_slots(self) -> List[int]:
        return [i for i, o in enumerate(self.owner) if o is None]

    def admit(self, system: int) -> int:
        slot = self.free_slots()[0]
        self.owner[slot] = system
        self.queue[system] = []
        self.R.reset_slot(slot, self.stream.cuda_stream)
        return slot

    def release(self, system: int):
        self.owner[self.owner.index(system)] = None
        self.queue.pop(system, None)

    def take_batch(self, drop_stale: bool) -> Tuple[List[Tuple[int, Request]], List[Request]]:
        """Pick one request per system with queued work; returns (batch, dropped)."""
        batch, dropped = [], []
        for slot, sysid in enumerate(self.owner):
            q = self.queue.get(sysid) if sysid is not None else None
            if not q:
                continue
            if drop_stale and len(q) > 1:
                dropped += q[:-1]
                del q[:-1]
            batch.append((slot, q.pop(0)))
        for r in dropped:
            r.dropped = True
        return batch, dropped

    def try_launch(self, drop_stale: bool = False) -> List[Request]:
        """Launch one masked step if idle and there is work; returns dropped requests."""
        import torch
        if self.inflight is not None:
            return []
        batch, dropped = self.take_batch(drop_stale)
        if not batch:
            return dropped
        ng = self.type.ngrad
        mask = np.zeros(self.cap, dtype=np.int32)
        gh = self.g_host.numpy()
        for slot, req in batch:
            gh[slot * ng:(slot + 1) * ng] = req.grad
            mask[slot] = 1
        self.R.serve_step(mask, self.g_host.data_ptr(), self.a_host.data_ptr(), self.stream.cuda_stream)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.inflight = (ev, batch)
        self.batches += 1
        self.slot_steps += len(batch)
        return dropped

    def poll(self, now_fn: Callable[[], float]) -> List[Request]:
        if self.inflight is None:
            return []
        ev, batch = self.inflight
        if not ev.query():
            return []
        t = now_fn()
        na = self.type.nact
        ah = self.a_host.numpy()
        done = []
        for slot, req in batch:
            req.result = ah[slot * na:(slot + 1) * na].copy()
            req.t_done = t
            done.append(req)
        self.inflight = None
        return done

    def close(self):
        self.R.close()


class MvmPool(Pool):
    """A pool served by the control-matrix MVM instead of the iterative
    reconstructor: `capacity` rows of a batched MVM (BF16 by default) of the
    type's control matrix.  The MVM keeps no state between steps, so a slot
    only maps a system to a row; rows of systems without a request carry zero
    gradients."""

    def __init__(self, stype: SystemType, M, dtype: int = 1, device: int = 0, priority: int = 0):
        import ctypes as C
        import torch
        from . import native
        self.type = stype
        self.cap = stype.capacity
        self.lib = native.load()
        Mc = np.asfortranarray(M, dtype=np.float64)
        h = C.c_void_p()
        native.check(self.lib.mb_mvm_create(Mc.ctypes.data_as(C.POINTER(C.c_double)), int(M.shape[0]),
                                            int(M.shape[1]), int(dtype), self.cap, C.byref(h)), "mb_mvm_create")
        self.h = h
        self.stream = torch.cuda.Stream(device=device, priority=priority)
        self.owner = [None] * self.cap
        self.queue = {}
        self.inflight = None
        self.g_host = torch.zeros(self.cap * stype.ngrad, dtype=torch.float32).pin_memory()
        self.a_host = torch.empty(self.cap * stype.nact, dtype=torch.float32).pin_memory()
        self.g_dev = torch.zeros(self.cap * stype.ngrad, dtype=torch.float32, device=f"cuda:{device}")
        self.a_dev = torch.empty(self.cap * stype.nact, dtype=torch.float32, device=f"cuda:{device}")
        self.batches = 0
        self.slot_steps = 0

    def admit(self, system: int) -> int:
        slot = self.free_slots()[0]
        self.owner[slot] = system
        self.queue[system] = []
        return slot

    def try_launch(self, drop_stale: bool = False) -> List[Request]:
        import ctypes as C
        import torch
        from . import native
        if self.inflight is not None:
            return []
        batch, dropped = self.take_batch(drop_stale)
        if not batch:
            return dropped
        ng, na = self.type.ngrad, self.type.nact
        gh = self.g_host.numpy()
        for slot, req in batch:
            gh[slot * ng:(slot + 1) * ng] = req.grad
        # rows of idle slots keep stale gradients: their commands are never read,
        # so only the rows up to the last active slot travel
        top = max(slot for slot, _ in batch) + 1
        with torch.cuda.stream(self.stream):
            self.g_dev[:top * ng].copy_(self.g_host[:top * ng], non_blocking=True)
            native.check(self.lib.mb_mvm_apply_device(self.h, C.c_void_p(self.g_dev.data_ptr()),
                                                      C.c_void_p(self.a_dev.data_ptr()),
                                                      C.c_void_p(self.stream.cuda_stream)), "mb_mvm_apply_device")
            self.a_host[:top * na].copy_(self.a_dev[:top * na], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.inflight = (ev, batch)
        self.batches += 1
        self.slot_steps += len(batch)
        return dropped

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_mvm_free(self.h)
            self.h = None


class Server:
    """Admission, continuous batching and latency accounting over pools.

    `pool_factory(stype)` builds one pool per system type (``Pool`` on a
    GPU); the server only uses the pool interface (owner, queue, inflight,
    free_slots, admit, release, try_launch, poll, close)."""

    def __init__(self, types: List[SystemType], hbm_budget: int,
                 pool_factory: Optional[Callable[[SystemType], object]] = None,
                 drop_stale: bool = False, slot_bytes: Optional[List[int]] = None, prioritize: bool = True):
        if pool_factory is None:
            prio = stream_priorities(types) if prioritize else [0] * len(types)
            self.pools = [Pool(t, priority=p) for t, p in zip(types, prio)]
        else:
            self.pools = [pool_factory(t) for t in types]
        self.slot_bytes = slot_bytes or [slot_footprint_bytes(t) for t in types]
        self.budget = int(hbm_budget)
        self.used = 0
        self.drop_stale = drop_stale
        self.system_pool: Dict[int, int] = {}
        self.waiting: List[Tuple[int, int]] = []   # (system, pool) awaiting admission, FIFO
        self.completed: List[Request] = []
        self.dropped: List[Request] = []
        self.admit_log: List[Tuple[float, int]] = []

    def register(self, system: int, pool: int, now: float) -> bool:
        """Ask to admit a system; returns True if it got a slot now."""
        self.system_pool[system] = pool
        if not self.waiting and self._fits(pool):
            self._admit(system, pool, now)
            return True
        self.waiting.append((system, pool))
        return False

    def _fits(self, pool: int) -> bool:
        return bool(self.pools[pool].free_slots()) and self.used + self.slot_bytes[pool] <= self.budget

    def _admit(self, system: int, pool: int, now: float):
        self.pools[pool].admit(system)
        self.used += self.slot_bytes[pool]
        self.admit_log.append((now, system))

    def release(self, system: int, now: float):
        pool = self.system_pool[system]
        p = self.pools[pool]
        if system not in p.owner:
            raise KeyError(f"system {system} is not admitted")
        p.release(system)
        self.used -= self.slot_bytes[pool]
        # strict FIFO: admit from the head while the head fits, so a large
        # system is not starved by smaller ones arriving after it
        while self.waiting and self._fits(self.waiting[0][1]):
            s, q = self.waiting.pop(0)
            self._admit(s, q, now)

    def admitted(self, system: int) -> bool:
        pool = self.system_pool.get(system)
        return pool is not None and system in self.pools[pool].owner

    def submit(self, req: Request):
        if not self.admitted(req.system):
            raise KeyError(f"system {req.system} is not admitted")
        self.pools[self.system_pool[req.system]].queue[req.system].append(req)

    def step(self, now_fn: Callable[[], float]) -> int:
        """Collect finished batches and launch idle pools that have work."""
        n = 0
        for p in self.pools:
            self.completed += p.poll(now_fn)
            before = p.inflight
            self.dropped += p.try_launch(self.drop_stale)
            if p.inflight is not None and before is None:
                n += 1
        return n

    def idle(self) -> bool:
        return all(p.inflight is None and not any(p.queue.values()) for p in self.pools)

    def close(self):
        for p in self.pools:
            p.close()


def run_served(types: List[SystemType], systems: List[Tuple[int, float, np.ndarray]],
               duration: float, hbm_budget: int, steps_per_system: Optional[int] = None,
               seed: int = 0, drop_stale: bool = False, pool_factory=None,
               clock: Callable[[], float] = time.perf_counter, server: Optional[Server] = None):
    """Serve Poisson request streams in real time.

    systems: (pool index, request rate in Hz, gradient frames [nframe][ngrad]).
    Each system asks for admission at t=0 (in order); a system leaves after
    ``steps_per_system`` completed requests (if given), freeing its slot for
    waiters.  Arrivals stop at ``duration``; the loop then drains the queues.
    Returns (server, completed requests, wall seconds)."""
    import gc
    rng = np.random.default_rng(seed)
    srv = server or Server(types, hbm_budget, pool_factory=pool_factory, drop_stale=drop_stale)
    gc_was = gc.isenabled()
    gc.disable()  # no collector pauses inside the real-time loop
    try:
        return _serve_loop(srv, systems, duration, steps_per_system, rng, clock)
    finally:
        if gc_was:
            gc.enable()


def _serve_loop(srv, systems, duration, steps_per_system, rng, clock):
    t0 = clock()
    now = lambda: clock() - t0  # noqa: E731
    events = []  # (time, system, step)
    for sid, (pool, rate, frames) in enumerate(systems):
        srv.register(sid, pool, 0.0)
        heapq.heappush(events, (rng.exponential(1.0 / rate), sid, 0))
    done_count = {sid: 0 for sid in range(len(systems))}
    pending: Dict[int, List[Request]] = {sid: [] for sid in range(len(systems))}
    waiting = set()  # systems with requests not yet handed to the server
    left = set()
    while True:
        tn = now()
        while events and events[0][0] <= tn:
            ta, sid, k = heapq.heappop(events)
            pool, rate, frames = systems[sid]
            pending[sid].append(Request(ta, sid, k, frames[k % len(frames)]))
            waiting.add(sid)
            more = steps_per_system is None or k + 1 < steps_per_system
            if more and ta < duration:
                heapq.heappush(events, (ta + rng.exponential(1.0 / rate), sid, k + 1))
        for sid in list(waiting):
            if srv.admitted(sid):
                for r in pending[sid]:
                    srv.submit(r)
                pending[sid] = []
                waiting.discard(sid)
        before = len(srv.completed)
        srv.step(now)
        for req in srv.completed[before:]:
            done_count[req.system] += 1
            if (steps_per_system is not None and done_count[req.system] >= steps_per_system
                    and req.system not in left):
                left.add(req.system)
                srv.release(req.system, now())
        if not events and srv.idle() and not waiting:
            break
        if tn > duration * 4 + 30:
            break
    return srv, srv.completed, now()


def latency_stats(reqs: List[Request]) -> dict:
    lat = np.array([r.t_done - r.t_arrival for r in reqs if math.isfinite(r.t_done)]) * 1e3
    if lat.size == 0:
        return {"n": 0}
    return {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max())}
