"""Serving on the GPU: masked steps of instance slots.

A slot's result must not depend on which other slots run in the same batch:
every kernel skips the blocks of inactive slots and all reductions are per
slot in a fixed order, so the comparison "alone" vs "in the mix" is exact.
The served result is also checked against the FP64 oracle (tomography then
fit, warm-started over the steps), and a short real-time served run of a
mixed workload is replayed system by system on standalone reconstructors.
"""
import numpy as np
import pytest

from oracle.recon_oracle import FitOracle, TomoOracle, fit_solve, tomo_solve

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-4  # DM command vector vs the FP64 oracle, same iteration counts


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _grads(s, nstep, nsys, seed):
    rng = np.random.default_rng(seed)
    g0 = rng.standard_normal((nsys, s.ngrad)) * 1e-6
    return [(g0 + k * rng.standard_normal((nsys, s.ngrad)) * 1e-7).astype(np.float32) for k in range(nstep)]


def _run_slots(R, frames, masks):
    """frames[k][slot] uploaded for the active slots of masks[k]; returns [k][slot] commands."""
    import torch
    st = torch.cuda.Stream()
    sp = st.cuda_stream
    out = []
    for g, m in zip(frames, masks):
        gd = torch.tensor(g, device="cuda")
        for slot in np.nonzero(m)[0]:
            R.slot_upload(int(slot), gd[slot].data_ptr(), sp)
        R.step_slots(m, sp)
        a = torch.empty((R.nbatch, R.nact), dtype=torch.float32, device="cuda")
        a.zero_()
        torch.cuda.synchronize()
        for slot in np.nonzero(m)[0]:
            R.slot_download(int(slot), a[slot].data_ptr(), sp)
        st.synchronize()
        out.append(a.cpu().numpy())
    return out


@pytest.fixture(scope="module", params=["ltao_8m", "mcao_30m"])
def system(request):
    from conftest import get_fit, get_system
    return request.param, get_system(request.param), get_fit(request.param)


def test_alone_equals_in_the_mix(system):
    from maos_b200.recon import Reconstructor
    name, s, fs = system
    nb, slot, nstep = 4, 2, 3
    frames = _grads(s, nstep, nb, seed=7)
    alone = Reconstructor(s, nbatch=nb, fit=fs)
    mix = Reconstructor(s, nbatch=nb, fit=fs)
    try:
        only = np.zeros(nb, np.int32)
        only[slot] = 1
        a1 = _run_slots(alone, frames, [only] * nstep)
        # in the mix: every slot runs, slot 0 sits out the middle step
        masks = [np.ones(nb, np.int32), np.array([0, 1, 1, 1], np.int32), np.ones(nb, np.int32)]
        a2 = _run_slots(mix, frames, masks)
        for k in range(nstep):
            assert np.array_equal(a1[k][slot], a2[k][slot]), f"step {k}: slot result depends on the batch"
            assert np.all(a1[k][[0, 1, 3]] == 0)   # nothing downloaded for idle slots
        # slot 0 skipped step 1: its step-2 result equals a run that never saw frame 1
        ref = Reconstructor(s, nbatch=nb, fit=fs)
        try:
            m0 = np.array([1, 0, 0, 0], np.int32)
            a3 = _run_slots(ref, [frames[0], frames[2]], [m0, m0])
            assert np.array_equal(a3[1][0], a2[2][0])
        finally:
            ref.close()
    finally:
        alone.close()
        mix.close()


def test_slot_matches_oracle(system):
    from maos_b200.recon import Reconstructor
    name, s, fs = system
    nb, slot = 3, 1
    frames = _grads(s, 2, nb, seed=11)
    R = Reconstructor(s, nbatch=nb, fit=fs)
    try:
        m = np.zeros(nb, np.int32)
        m[slot] = 1
        got = _run_slots(R, frames, [m, m])
    finally:
        R.close()
    to, fo = TomoOracle(s), FitOracle(s, fs)
    x1, _ = tomo_solve(to, frames[0][slot].astype(np.float64))
    w1, _ = fit_solve(fo, x1)
    x2, _ = tomo_solve(to, frames[1][slot].astype(np.float64), x0=x1)
    w2, _ = fit_solve(fo, x2, a0=w1)
    assert rel(got[0][slot], w1) < SOLVE_TOL
    assert rel(got[1][slot], w2) < SOLVE_TOL


def test_reset_slot_restarts_cold():
    from conftest import get_fit, get_system
    from maos_b200.recon import Reconstructor
    s, fs = get_system("ltao_8m"), get_fit("ltao_8m")
    nb = 2
    frames = _grads(s, 3, nb, seed=5)
    R = Reconstructor(s, nbatch=nb, fit=fs)
    try:
        m = np.array([1, 1], np.int32)
        first = _run_slots(R, frames[:1], [m])[0]
        _run_slots(R, frames[1:2], [m])
        R.reset_slot(0)
        again = _run_slots(R, frames[:1], [np.array([1, 0], np.int32)])[0]
        assert np.array_equal(first[0], again[0])
    finally:
        R.close()


def test_served_mix_replays_standalone():
    """A short real-time served run of two system types, replayed per system."""
    from conftest import get_fit, get_system
    from maos_b200 import serve
    from maos_b200.recon import Reconstructor
    types = [serve.SystemType("scao_8m", get_system("scao_8m"), get_fit("scao_8m"), capacity=3),
             serve.SystemType("ltao_8m", get_system("ltao_8m"), get_fit("ltao_8m"), capacity=2)]
    rng = np.random.default_rng(3)
    systems = []
    for sid in range(5):
        t = types[sid % 2]
        fr = (rng.standard_normal((4, t.ngrad)) * 1e-6).astype(np.float32)
        systems.append((sid % 2, 400.0, fr))
    nsteps = 6
    budget = sum(serve.slot_footprint_bytes(t) * t.capacity for t in types)
    srv, done, wall = serve.run_served(types, systems, duration=5.0, hbm_budget=budget,
                                       steps_per_system=nsteps, seed=1)
    try:
        assert len(done) == 5 * nsteps
        assert not srv.dropped
        by_sys = {}
        for r in done:
            by_sys.setdefault(r.system, []).append(r)
        for sid, reqs in by_sys.items():
            reqs.sort(key=lambda r: r.step)
            assert [r.step for r in reqs] == list(range(nsteps))
            t = types[systems[sid][0]]
            R = Reconstructor(t.tomo, nbatch=1, fit=t.fit)
            try:
                m = np.ones(1, np.int32)
                want = _run_slots(R, [systems[sid][2][k % 4][None] for k in range(nsteps)], [m] * nsteps)
            finally:
                R.close()
            for k in range(nsteps):
                assert rel(reqs[k].result, want[k][0]) < 1e-4, (sid, k)
        st = serve.latency_stats(done)
        assert st["n"] == 5 * nsteps and st["p99_ms"] > 0
    finally:
        srv.close()


def test_served_through_bf16_mvm():
    """Systems served by MvmPool get M_bf16 g for their own gradients (1e-5)."""
    import torch
    from conftest import get_fit, get_system
    from maos_b200 import serve
    t = serve.SystemType("scao_8m", get_system("scao_8m"), get_fit("scao_8m"), capacity=5)
    rng = np.random.default_rng(4)
    M = rng.standard_normal((t.nact, t.ngrad)) * 1e-2
    systems = [(0, 300.0, (rng.standard_normal((4, t.ngrad)) * 1e-6).astype(np.float32)) for _ in range(5)]
    srv, done, wall = serve.run_served([t], systems, duration=5.0, hbm_budget=1 << 40, steps_per_system=4, seed=2,
                                       pool_factory=lambda st: serve.MvmPool(st, M, dtype=1))
    try:
        assert len(done) == 20
        Mb = torch.from_numpy(M).to(torch.bfloat16).to(torch.float64).numpy()
        for r in done:
            g = systems[r.system][2][r.step % 4].astype(np.float64)
            want = Mb @ g
            assert rel(r.result, want) < 1e-5
    finally:
        srv.close()
