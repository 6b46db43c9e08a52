"""Benchmark of the per-step wavefront reconstruction on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl reference]

Workload (one "step"): the 30 m NFIRAOS-like MCAO system (6 LGS, 60x60
subapertures, 33,840 gradients, 6 layers / 27,648 unknowns, 2 DMs / 9,745
actuators, 9 fit directions), seeded frozen-flow von Karman gradients in,
warm-started FP32 FDPCG tomography with 30 iterations, then the DM-fit CG with
4 iterations, actuator commands out -- for B independent instances resident on
each GPU.  The instances share the operator tables and advance together in
one CUDA graph.  The line also carries the control-matrix MVM alternative at
the same size (M = 9,745 x 33,840) in FP32, BF16 and FP8-E4M3.

value     aggregate steps/s over all GPUs (N * B * K / max-over-ranks device time),
          inputs resident in HBM, L2 flushed (256 MiB write) before every step.
e2e       the same metric through the C ABI with host buffers
          (mb_recon_serve_step: pinned FP32 gradients in, pinned FP32 DM
          commands out, copies inside the timed region); the FP64 gpu_tomo +
          gpu_fit shaped calls are reported beside it.
roofline  the kernel with the largest share of the step, its algorithmic bytes
          per launch over its measured launch time, against the measured HBM
          copy bandwidth.
cpu_baseline  the reference's own CPU reconstruction (compiled from its
          sources into oracle/_ref) timed on this host's cores on a bounded
          sample of the same workload.

Multi-GPU (--gpus N, launched by torch.distributed.run): every rank owns its
own B instances (weak scaling; no data-path collective), ranks meet at a
barrier around the timed region and the slowest rank's time is used.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = "mcao_30m"
WORKLOAD_TEXT = "mcao_30m: FDPCG tomography 30 it + DM fit CG 4 it, warm start"
METRIC = "recon steps/s (30 m MCAO: FP32 FDPCG tomography 30 it + DM fit 4 it)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mvm-batch", type=int, default=1)
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--precision-steps", type=int, default=2000)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-wfs", action="store_true")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, batch: int):
    """DRAM bytes per launch from the committed ncu summary, scaled to `batch`."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == kernel:
            b0, by = int(f[1]), float(f[2])
            return by * batch / b0
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "20"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.p is None:
            return out
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(nm)
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


class RefRunner:
    """The reference's own CPU reconstruction (oracle/_ref) on this host's cores."""

    def __init__(self, sysm, frames, fit=None):
        from oracle import refbridge
        self.ncores = os.cpu_count() or 1
        self.frames = frames
        self.maxit = sysm.cfg.tomo_maxit
        self.nx = int(sysm.nx_total)
        self.fit_maxit = fit.maxit if fit is not None else 0
        self.R = refbridge.RefProcess(nthread=self.ncores)
        self.R.call("setup", refbridge.system_desc(sysm, split=1))
        self.R.call("fdpcg_set", sysm.fdpcg.Mbinv, sysm.fdpcg.perm, sysm.fdpcg.scale)
        # the assembled fit (the reference default): setup_fit, then muv_solve's FR and pcg on FL
        self.assembled = fit is not None and hasattr(fit, "FLM")
        if self.assembled:
            self.R.call("fit_assemble", refbridge.fit_assembled_desc(fit, sysm.cfg))
        elif fit is not None:
            self.R.call("fit_setup", refbridge.fit_desc(fit))
        self.x = None
        self.a = None
        self.k = 0

    def step(self):
        g = self.frames[self.k % len(self.frames)]
        b = self.R.call("tomoR", g)
        self.x, _ = self.R.call("pcg", b, self.x, int(self.x is not None), self.maxit, 1)
        if self.fit_maxit and self.assembled:
            fb = self.R.call("fitas_rhs", self.x)
            self.a, _ = self.R.call("fitas_pcg", fb, self.a, int(self.a is not None), self.fit_maxit)
        elif self.fit_maxit:
            fb = self.R.call("fitR", self.x)
            self.a, _ = self.R.call("fit_pcg", fb, self.a, int(self.a is not None), self.fit_maxit)
        self.k += 1

    def precond_ms(self, reps: int = 20) -> float:
        """ms per call of the reference's fdpcg_precond alone (its FFTs run on
        the FFTW-API shim, FFTW being absent here), with the worker round trip."""
        import numpy as np
        r = np.random.default_rng(1).standard_normal(self.nx)
        self.R.call("fdpcg_precond", r)
        t0 = time.perf_counter()
        for _ in range(reps):
            self.R.call("fdpcg_precond", r)
        return (time.perf_counter() - t0) / reps * 1000.0

    def rate(self, seconds: float):
        """Run warm steps for about `seconds`; returns (steps/s, steps, elapsed)."""
        n = 0
        t0 = time.perf_counter()
        while True:
            self.step()
            n += 1
            dt = time.perf_counter() - t0
            if dt >= seconds or n >= 1000:
                return n / dt, n, dt

    def close(self):
        self.R.close()


def fft_note(rate: float, precond_ms: float, maxit: int) -> dict:
    """The share of the reference CPU step spent in its FDPCG preconditioner
    (whose FFTs run on this build's FFTW-API shim), and the step rate with
    that share removed: a bound on how much a faster FFT library could give."""
    step_ms = 1000.0 / rate
    pre = precond_ms * maxit
    rest = max(step_ms - pre, 1e-9)
    return {"fdpcg_precond_ms_per_call": precond_ms, "fdpcg_precond_share_of_step": min(pre / step_ms, 1.0),
            "value_without_fdpcg_precond": 1000.0 / rest,
            "fft_note": "the reference's FFTs run on this build's FFTW-API shim (FFTW is absent); "
                        "value_without_fdpcg_precond removes the whole preconditioner (FFTs and block solve) "
                        "from the CPU step, the most a faster FFT library could give"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from maos_b200 import config, fit_assemble, geometry, turbulence
    sysm = geometry.build_tomo(config.PRESETS[WORKLOAD]())
    fit = fit_assemble.build_fit_assembled(sysm)
    frames = turbulence.gradient_frames(sysm, seed=1, nframe=4)
    run = RefRunner(sysm, frames, fit)
    for _ in range(max(1, args.warmup)):
        run.step()
    per = args.cpu_seconds / max(1, args.steps)
    rates = []
    total = 0
    for _ in range(args.steps):
        r, n, _dt = run.rate(per)
        rates.append(r)
        total += n
    pms = run.precond_ms()
    run.close()
    value = statistics.median(rates)
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded von Karman frozen-flow gradients)",
            "config": {"workload": WORKLOAD_TEXT, "instances": 1},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": run.ncores, "kind": "reference",
                             "sample": f"{total} warm reference CPU steps in {args.steps} samples",
                             **fft_note(value, pms, sysm.cfg.tomo_maxit)},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def mvm_rates(lib, native, nact: int, ngrad: int, batch: int, stream, M=None):
    """Control-matrix MVM steps/s per storage type (M: the built control
    matrix, else a random matrix of the system's size)."""
    import ctypes as C
    import numpy as np
    import torch
    if M is None:
        M = np.random.default_rng(3).standard_normal((nact, ngrad)) * 1e-3
    M = np.asfortranarray(M, dtype=np.float64)
    g = torch.randn(batch, ngrad, device="cuda")
    out = torch.empty(batch, nact, device="cuda")
    res = {"batch": batch, "shape": [nact, ngrad]}
    peak, _ = measured_peaks()
    for name, dt in (("fp32", 0), ("bf16", 1), ("fp8_e4m3", 2)):
        h = C.c_void_p()
        native.check(lib.mb_mvm_create(M.ctypes.data_as(C.POINTER(C.c_double)), nact, ngrad, dt, batch,
                                       C.byref(h)), "mb_mvm_create")
        sp = stream.cuda_stream
        with torch.cuda.stream(stream):
            for _ in range(3):
                lib.mb_mvm_apply_device(h, C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(sp))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            n = 20
            e0.record(stream)
            for _ in range(n):
                lib.mb_mvm_apply_device(h, C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(sp))
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / n
        nbytes = lib.mb_mvm_bytes(h)
        res[name] = {"steps_per_s": batch * 1000.0 / ms, "ms": ms, "matrix_bytes": int(nbytes),
                     "hbm_frac": nbytes / (ms / 1000.0) / 1e9 / peak}
        lib.mb_mvm_free(h)
    del M
    return res


def wfs_rates(sysm, fit, batch: int, stream, cpu: bool = True):
    """Geometric WFS gradients on the device (mb_geom_wfs_grad: every WFS
    of ``batch`` instances, each with its own atmosphere, through the DMs,
    with noise) per step, and the reference's CPU geometric gradients of one
    instance (prop_grid + GS0 from oracle/_ref) on this host's cores."""
    import numpy as np
    import torch
    from maos_b200 import wfs_setup
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    geom = wfs_setup.build_geom_wfs(sysm)
    atms = [FrozenFlowAtmosphere(sysm.cfg, 100 + i) for i in range(4)]
    W = GeomWfs.for_system(sysm, [atms[i % 4] for i in range(batch)], fit=fit, nbatch=batch, geom=geom)
    dm = torch.randn(batch, W.nact, device="cuda") * 1e-7
    with torch.cuda.stream(stream):
        for k in range(3):
            W.grad(k, dm=dm, seed=1, stream=stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        n = 20
        e0.record(stream)
        for k in range(n):
            W.grad(k, dm=dm, seed=1, stream=stream)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    P = [geom.powfs[geom.wfs_powfs[i]] for i in range(geom.nwfs)]
    pts = sum((p.nxsa + 2) ** 2 * len(p.ix0) for p in P)
    nmap = len(sysm.cfg.atm_ht) + len(fit.dms)
    res = {"instances": batch, "ms": ms, "steps_per_s": batch * 1000.0 / ms, "kernel": "k_wfs_geom",
           "wfs": geom.nwfs, "subapertures": int(sum(len(p.ix0) for p in P)), "points_per_subaperture_side": P[0].nxsa,
           "maps": nmap, "interpolations_per_s": pts * nmap * batch / (ms / 1000.0),
           "data": "seeded von Karman layers (4 seeds over the instances), random DM commands, noise on"}
    W.close()
    if cpu:
        from oracle import refbridge
        if refbridge.available():
            a0 = atms[0]
            o = -a0.n / 2 * a0.dx
            maps = [(sc, a0.dx, o, o, float(h), float(a0.vx[l]), float(a0.vy[l]), 1.0, 1)
                    for l, (sc, h) in enumerate(zip(a0.screens, sysm.cfg.atm_ht))]
            a = dm[0].double().cpu().numpy()
            off = fit.act_offsets()
            for k, d in enumerate(fit.dms):
                maps.append((a[off[k]:off[k + 1]].reshape(d.amap.ny, d.amap.nx), d.amap.dx, d.amap.ox, d.amap.oy,
                             d.ht, 0.0, 0.0, -1.0, 0))
            ncores = os.cpu_count() or 1
            w0 = sysm.wfs[0]
            with refbridge.RefProcess(nthread=ncores) as R:
                R.call("wfs_gs0", w0.salocx, w0.salocy, w0.dsa, P[0].nxsa, sysm.cfg.D, sysm.cfg.din)
                R.call("wfs_geom_grads", geom.thetax, geom.thetay, geom.hs, maps, sysm.cfg.sim_dt, 0)
                t0 = time.perf_counter()
                nstep = 0
                while nstep < 3 or (time.perf_counter() - t0 < 5.0 and nstep < 20):
                    R.call("wfs_geom_grads", geom.thetax, geom.thetay, geom.hs, maps, sysm.cfg.sim_dt, nstep)
                    nstep += 1
                dt = time.perf_counter() - t0
            res["cpu_reference"] = {"steps_per_s": nstep / dt, "cores": ncores, "kind": "reference",
                                    "sample": f"{nstep} steps of one instance (prop_grid of every map onto every "
                                              f"WFS's points, then GS0) in {dt:.1f} s"}
    return res


def closed_loop_rates(sysm, fit, R, batch: int, stream, nstep: int = 20):
    """The whole loop on the device for ``batch`` instances: geometric WFS
    (through the DMs, noise on) -> tomography + fit (the graph step of R) ->
    servo (type I, gain 0.5) -> DM commands, per step; CUDA events around
    ``nstep`` steps after 3 warm-up steps."""
    import torch
    from maos_b200 import wfs_setup
    from maos_b200.servo import Servo
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    nact = int(fit.nact)
    atms = [FrozenFlowAtmosphere(sysm.cfg, 200 + i) for i in range(4)]
    W = GeomWfs.for_system(sysm, [atms[i % 4] for i in range(batch)], fit=fit, nbatch=batch,
                           geom=wfs_setup.build_geom_wfs(sysm))
    S = Servo(batch * nact, ep=[[0.5]], dt=sysm.cfg.sim_dt)
    dm = torch.zeros(batch, nact, dtype=torch.float32, device="cuda")
    fa = R.fit_solution()   # the fit's commands, in place on the device
    R.reset()
    sp = stream.cuda_stream

    def step(k):
        g = W.grad(k, dm=dm, seed=1, stream=stream)
        R.step_device(g.data_ptr(), sp)
        cmd = S.filter(fa.reshape(-1).double(), stream=stream)
        dm.copy_(cmd.view(batch, nact))

    with torch.cuda.stream(stream):
        for k in range(3):
            step(k)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(3, 3 + nstep):
            step(k)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nstep
    W.close()
    S.close()
    R.reset()
    return {"instances": batch, "ms_per_step": ms, "steps_per_s": batch * 1000.0 / ms,
            "step": "mb_geom_wfs_grad -> mb_recon_step_device -> mb_servo_filter -> DM commands, no host copy",
            "data": "seeded von Karman layers with frozen flow (4 seeds over the instances), noise on"}


def single_instance_rates(preset: str, nsteps: int = 200, warmup: int = 5):
    """One instance alone: the plain single-instance FP32 path (graph step of
    tomography + fit, gradients resident) with per-step CUDA events and the
    L2 flushed before every step; steps/s and p50/p99 step latency."""
    import numpy as np
    import torch
    from maos_b200 import config, fit_assemble, geometry, turbulence
    from maos_b200.recon import Reconstructor
    sysm = geometry.build_tomo(config.PRESETS[preset]())
    fit = fit_assemble.build_fit_assembled(sysm)
    frames = turbulence.gradient_frames(sysm, seed=1, nframe=4)
    g = torch.tensor(frames, dtype=torch.float32, device="cuda")
    R = Reconstructor(sysm, nbatch=1, fit=fit)
    rows, _ = R.autotune(reps=20)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
    with torch.cuda.stream(stream):
        for k in range(warmup):
            R.step_device(g[k % 4].data_ptr(), sp)
        for k in range(nsteps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            R.step_device(g[k % 4].data_ptr(), sp)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    t = sorted(a.elapsed_time(b) for a, b in ev)
    updates = table_updates(R, sysm)
    R.close()
    out = {"instances": 1, "steps": nsteps, "steps_per_s": 1000.0 * nsteps / sum(t),
           "latency_ms": {"p50": statistics.median(t), "p99": t[min(nsteps - 1, int(math.ceil(0.99 * nsteps)) - 1)],
                          "max": t[-1]},
           "pupil_rows": rows, "tomo": f"{'FDPCG' if sysm.cfg.tomo_precond else 'CG'} {sysm.cfg.tomo_maxit} it",
           "fit_it": fit.maxit}
    if updates:
        out["table_updates_ms"] = updates
    return out


def table_updates(R, sysm, reps: int = 5):
    """Host wall time (to completion on the device) of the reconstructor's
    table updates, each rebuilding every table it affects on the GPU:
    gpu_update_recon for one WFS (its NEA and tip/tilt projector, then the
    FDPCG data term and blocks from the new mean NEA) and gpu_update_recon_cn2
    (the L2 weights and the FDPCG blocks, no host tables).  The median of
    `reps` calls, the original values re-installed each time."""
    import numpy as np
    import torch
    if sysm.fdpcg is None:
        return None
    w = sysm.wfs[1]
    nsa = w.nsa
    neai = np.stack([w.saneai[:nsa], w.saneai[nsa:], np.zeros(nsa)], axis=1).ravel()
    neam = np.asarray(sysm.fdpcg.geom["neam"], dtype=np.float64)
    l2c = np.asarray(sysm.l2c, dtype=np.float64)
    tn, tc = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        R.update_nea(1, neai, w.PTT)
        R.update_neam(neam)
        torch.cuda.synchronize()
        tn.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        R.update_cn2(l2c)
        torch.cuda.synchronize()
        tc.append(time.perf_counter() - t0)
    return {"nea_one_wfs_with_fdpcg_rebuild": 1e3 * statistics.median(tn),
            "cn2_with_fdpcg_rebuild": 1e3 * statistics.median(tc)}


SERVE_MIX = (("scao_8m", 26), ("ltao_8m", 26), ("mcao_30m", 12))


def grouped_mix(nsteps: int = 30, warmup: int = 3):
    """The served mix's 64 instances of three geometries (26 8 m SCAO, 26 8 m
    LTAO, 12 30 m MCAO) all stepped at once, two ways: one group graph per
    step (mb_group_step_device: the tomography operators one launch over all
    64 instances) and the three reconstructors' own step graphs on three
    streams.  Device time per step (CUDA events, L2 flushed before every
    step), instance steps/s and kernel launches per step."""
    import numpy as np
    import torch
    from maos_b200 import config, fit_assemble, geometry, turbulence
    from maos_b200.recon import Reconstructor, ReconGroup
    rs, gs = [], []
    for name, n in SERVE_MIX:
        sysm = geometry.build_tomo(config.PRESETS[name]())
        R = Reconstructor(sysm, nbatch=n, fit=fit_assemble.build_fit_assembled(sysm))
        R.autotune(reps=5)
        rs.append(R)
        fr = turbulence.gradient_frames(sysm, seed=5, nframe=4).astype(np.float32)
        gs.append(torch.tensor(np.stack([fr[k % 4] for k in range(n)]), device="cuda"))
    G = ReconGroup(rs)
    lib = rs[0].lib
    main = torch.cuda.Stream()
    side = [torch.cuda.Stream() for _ in rs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ninst = sum(n for _, n in SERVE_MIX)

    def run(grouped: bool):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        for k in range(warmup + nsteps):
            with torch.cuda.stream(main):
                flush.fill_(float(k))
                if k >= warmup:
                    ev[k - warmup][0].record(main)
                if grouped:
                    G.step_device([g.data_ptr() for g in gs], main.cuda_stream)
                else:
                    for R, g, q in zip(rs, gs, side):
                        q.wait_stream(main)
                        R.step_device(g.data_ptr(), q.cuda_stream)
                    for q in side:
                        main.wait_stream(q)
                if k >= warmup:
                    ev[k - warmup][1].record(main)
        torch.cuda.synchronize()
        t = sorted(a.elapsed_time(b) for a, b in ev)
        return {"ms_per_step": statistics.median(t), "instance_steps_per_s": 1000.0 * ninst / statistics.median(t)}

    lib.mb_kernel_launches(1)
    pools = run(False)
    pools["launches_per_step"] = lib.mb_kernel_launches(1) / (warmup + nsteps)
    grouped = run(True)
    grouped["launches_per_step"] = lib.mb_kernel_launches(1) / (warmup + nsteps)
    G.close()
    for R in rs:
        R.close()
    return {"mix": " + ".join(f"{n} {name}" for name, n in SERVE_MIX), "instances": ninst,
            "step": "tomography (FDPCG 30 it for mcao_30m, CG 30 it for the 8 m types) + assembled fit 4 it",
            "group": grouped, "three_streams": pools}


def served_mix(seconds: float, mcao_frames=None, mvm: bool = False, rate_scale: float = 1.0):
    """The served mix: 64 systems (26 8 m SCAO, 26 8 m LTAO, 12 30 m MCAO), each
    sending Poisson requests at a rate drawn from U[500, 1000] Hz (times
    rate_scale), all admitted, warm state resident, newest frame wins when a
    system falls behind.
    mvm: every type is served by the BF16 MVM of its control matrix (built on
    the GPU by batched solves) instead of the iterative reconstructor."""
    import numpy as np
    import torch
    from maos_b200 import config, fit_assemble, geometry, serve, turbulence
    rng = np.random.default_rng(17)
    types, frames = [], []
    for name, n in SERVE_MIX:
        sysm = geometry.build_tomo(config.PRESETS[name]())
        fs = fit_assemble.build_fit_assembled(sysm)
        types.append(serve.SystemType(name, sysm, fs, capacity=n))
        if name == "mcao_30m" and mcao_frames is not None:
            fr = np.asarray(mcao_frames, dtype=np.float32)
        else:
            fr = turbulence.gradient_frames(sysm, seed=5, nframe=4).astype(np.float32)
        frames.append(fr)
    systems = []
    for t, (name, n) in enumerate(SERVE_MIX):
        for _ in range(n):
            systems.append((t, rate_scale * float(rng.uniform(500.0, 1000.0)), frames[t]))
    budget = sum(serve.slot_footprint_bytes(t) * t.capacity for t in types)
    build_s = None
    if mvm:
        from maos_b200.mvm_build import build_control_matrix
        t0 = time.perf_counter()
        Ms = {t.name: build_control_matrix(t.tomo, t.fit, rhs_batch=256, tomo_maxit=90, fit_maxit=40)[0]
              for t in types}
        build_s = time.perf_counter() - t0
        srv = serve.Server(types, 1 << 62, drop_stale=True,
                           pool_factory=lambda t: serve.MvmPool(t, Ms[t.name], dtype=1))
        del Ms
        import ctypes as C
        for p in srv.pools:  # warm
            for _ in range(3):
                p.lib.mb_mvm_apply_device(p.h, C.c_void_p(p.g_dev.data_ptr()), C.c_void_p(p.a_dev.data_ptr()),
                                          C.c_void_p(p.stream.cuda_stream))
    else:
        srv = serve.Server(types, budget, drop_stale=True)
        # warm the graphs of every pool (all slots), then reset the state
        for p in srv.pools:
            m = np.ones(p.cap, np.int32)
            for _ in range(3):
                p.R.serve_step(m, p.g_host.data_ptr(), p.a_host.data_ptr(), p.stream.cuda_stream)
    torch.cuda.synchronize()
    srv, done, wall = serve.run_served(types, systems, duration=seconds, hbm_budget=budget, seed=3,
                                       server=srv)
    offered = [0] * len(types)
    for r in done + srv.dropped:
        offered[systems[r.system][0]] += 1
    out = {"mix": " + ".join(f"{n} {name}" for name, n in SERVE_MIX),
           "path": "BF16 MVM of each type's control matrix" if mvm else "FDPCG/CG tomography + fit, FP32",
           "control_matrix_build_s": build_s,
           "rate_hz": f"U[{500 * rate_scale:g},{1000 * rate_scale:g}] Poisson per system", "seconds": seconds,
           "policy": "one masked batch per pool in flight, newest frame wins",
           "hbm_budget_bytes": int(budget),
           "served_steps_per_s": len(done) / seconds, "offered_per_s": (len(done) + len(srv.dropped)) / seconds,
           "dropped_frac": len(srv.dropped) / max(1, len(done) + len(srv.dropped)),
           "latency_ms": serve.latency_stats(done), "per_type": {}}
    for t, (name, n) in enumerate(SERVE_MIX):
        d = [r for r in done if systems[r.system][0] == t]
        nd = sum(1 for r in srv.dropped if systems[r.system][0] == t)
        out["per_type"][name] = {"systems": n, "served_per_s": len(d) / seconds,
                                 "dropped_frac": nd / max(1, len(d) + nd),
                                 "batches": srv.pools[t].batches,
                                 "mean_batch": srv.pools[t].slot_steps / max(1, srv.pools[t].batches),
                                 "latency_ms": serve.latency_stats(d)}
    srv.close()
    return out


def run_gpu(args):
    import numpy as np
    import torch
    from maos_b200 import config, fit_assemble, fit_setup, geometry, native, turbulence
    from maos_b200.recon import Reconstructor

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    sysm = geometry.build_tomo(config.PRESETS[WORKLOAD]())
    # the reference's default fit: assembled FR/FL over the in-pupil actuators
    # with slaving, extrapolation and tikcr (gpu.fit=1, fit.square=0)
    fit = fit_assemble.build_fit_assembled(sysm)
    # the device WFS and closed loop ray-trace DM maps: the grid-form fit
    # (gpu.fit=2, fit.square=1) drives them
    fit_grid = fit_setup.build_fit(sysm)
    B = args.batch
    nframe = 4
    # gradients: 4 frozen-flow frames for each of 4 seeds, tiled over instances
    seeds = [1 + 101 * rank + k for k in range(4)]
    fr = np.stack([turbulence.gradient_frames(sysm, seed=s, nframe=nframe) for s in seeds])
    grads = np.stack([np.stack([fr[b % len(seeds), k] for b in range(B)]) for k in range(nframe)])
    grads_dev = torch.tensor(grads, dtype=torch.float32, device="cuda")  # [nframe][B][ngrad]
    host_grads = [np.ascontiguousarray(grads[k]) for k in range(nframe)]

    lib = native.load()
    R = Reconstructor(sysm, nbatch=B, device=local, fit=fit)
    # the pupil-row blocking of the LHS kernel, measured for this batch (outside the timed region)
    tuned_rows, tuned_ms = R.autotune(reps=20)
    tuned_fd = {"fdpcg_form": R.fdpcg_mode(-1), "fdpcg_block_solve_instances_per_cta": R.fdpcg_shape()} \
        if sysm.fdpcg is not None else {}
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(k):
        R.step_device(grads_dev[k % nframe].data_ptr(), sp)

    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            step(k)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    lib.mb_kernel_launches(1)
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            step(k)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    launches = lib.mb_kernel_launches(1)
    clocks = clk.stop()
    times = [a.elapsed_time(b) for a, b in ev]
    total = sum(times)
    t = torch.tensor([total], dtype=torch.float64, device="cuda")
    if dist:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_max = float(t.item())
    value = world * B * args.steps / (total_max / 1000.0)
    times_sorted = sorted(times)
    p50 = statistics.median(times)
    p99 = times_sorted[min(len(times) - 1, int(math.ceil(0.99 * len(times))) - 1)]

    # end to end through the C ABI with host buffers: every step copies that
    # step's FP32 gradients from pinned host memory, runs the graph step and
    # copies the DM commands back to pinned host memory
    # (mb_recon_serve_step with every slot active), timed on the host clock
    K2 = max(3, min(args.steps, 20))
    allslots = np.ones(B, np.int32)
    g_pin = [torch.tensor(host_grads[k], dtype=torch.float32).pin_memory() for k in range(nframe)]
    a_pin = torch.empty((B, int(fit.nact)), dtype=torch.float32).pin_memory()

    def e2e_step(k):
        R.serve_step(allslots, g_pin[k % nframe].data_ptr(), a_pin.data_ptr(), sp)
        stream.synchronize()

    for k in range(2):
        e2e_step(k)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(K2):
        e2e_step(k)
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * B * K2 / float(te.item())
    # the reference-shaped FP64 calls (gpu_tomo then gpu_fit, pageable host
    # arrays converted on the host), for comparison
    for k in range(2):
        R.tomo_only(host_grads[k % nframe])
        R.fit()
    t0 = time.perf_counter()
    for k in range(K2):
        R.tomo_only(host_grads[k % nframe])
        R.fit()
    fp64_api_value = B * K2 / (time.perf_counter() - t0)

    # roofline of every kernel of a CG iteration and of the dominant one (live
    # CUDA-event timing on the reconstructor's stream; algorithmic bytes per
    # launch with the tables the instances share counted once per launch)
    ns = lib.mb_num_stages()
    import ctypes as C
    ms = (C.c_float * ns)()
    by = (C.c_double * ns)()
    lp = (C.c_int * ns)()
    native.check(lib.mb_time_stages(R.h, 20, ms, by, lp), "mb_time_stages")
    peak, peak_kind = measured_peaks()
    stages = []
    for i in range(ns):
        if lp[i] <= 0 or ms[i] <= 0:
            continue
        gbs = by[i] / (ms[i] / 1000.0) / 1e9
        stages.append({"name": lib.mb_stage_name(i).decode(), "ms_per_launch": ms[i], "bytes_per_launch": by[i],
                       "launches_per_step": lp[i], "share_ms": ms[i] * lp[i], "achieved_gbs": gbs,
                       "frac": gbs / peak})
    tot_stage = sum(s["share_ms"] for s in stages) or 1.0
    dom = max(stages, key=lambda s: s["share_ms"])
    roof = {"bound": "hbm", "kernel": dom["name"], "achieved": dom["achieved_gbs"], "peak": peak,
            "unit": "GB/s", "frac": dom["frac"], "peak_source": peak_kind,
            "traffic": ncu_traffic(dom["name"], B),
            "bytes_per_launch": dom["bytes_per_launch"], "ms_per_launch": dom["ms_per_launch"],
            "share_of_step": dom["share_ms"] / tot_stage,
            "kernels": [{k: (round(v, 6) if isinstance(v, float) else v) for k, v in s.items()} for s in stages],
            "note": "instances' working set is L2-resident: latency-bound kernels, fractions of the HBM copy "
                    "bandwidth are low by construction"}

    # control matrix of this system (batched cold solves of unit gradients,
    # 256 per launch) and the storage precision of its MVM on frozen flow
    Mctl, precision = None, None
    if world == 1 and args.precision_steps > 0:
        from maos_b200 import mvm_precision
        from maos_b200.mvm_build import build_control_matrix
        Mctl, build = build_control_matrix(sysm, fit, rhs_batch=256, tomo_maxit=90, fit_maxit=40)
        precision = mvm_precision.study(sysm, fit, Mctl, nsteps=args.precision_steps)
        precision["control_matrix_build"] = build
    mvm_line = mvm_rates(lib, native, int(fit.nact), int(sysm.ngrad), args.mvm_batch, stream, Mctl)
    mvm_line["matrix"] = "built control matrix" if Mctl is not None else "random, same shape"
    if precision is not None:
        mvm_line["precision"] = precision
    del Mctl

    wfs_line = wfs_rates(sysm, fit_grid, B, stream, cpu=(rank == 0 and not args.no_cpu_baseline)) \
        if world == 1 and not args.no_wfs else None

    loop_line = None
    if world == 1 and not args.no_wfs:
        Rg = Reconstructor(sysm, nbatch=B, device=local, fit=fit_grid)
        Rg.autotune(reps=10)
        loop_line = closed_loop_rates(sysm, fit_grid, Rg, B, stream)
        loop_line["fit"] = "grid form (DM maps on full grids)"
        Rg.close()

    single = None
    if world == 1:
        single = {name: single_instance_rates(name) for name in ("mcao_30m", "ltao_8m")}

    grouped = None
    if world == 1 and not args.no_serve:
        grouped = grouped_mix()

    served = served_mvm = served_low = None
    if world == 1 and not args.no_serve and args.serve_seconds > 0:
        served = served_mix(args.serve_seconds, mcao_frames=fr[0])
        # the same systems at a quarter of the rates, which one GPU sustains
        served_low = served_mix(args.serve_seconds, mcao_frames=fr[0], rate_scale=0.25)
        served_mvm = served_mix(args.serve_seconds, mcao_frames=fr[0], mvm=True)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import refbridge
        if refbridge.available():
            run = RefRunner(sysm, fr[0], fit)
            run.step()
            rate, n, dt = run.rate(args.cpu_seconds)
            pms = run.precond_ms()
            run.close()
            cpu = {"value": rate, "unit": "steps/s", "cores": run.ncores, "kind": "reference",
                   "sample": f"{n} warm steps of one {WORKLOAD} instance in {dt:.1f} s",
                   **fft_note(rate, pms, sysm.cfg.tomo_maxit)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded von Karman frozen-flow gradients, 4 seeds x 4 frames)",
                "config": {"workload": WORKLOAD_TEXT,
                           "instances_per_gpu": B, "ngrad": int(sysm.ngrad), "nact": int(fit.nact),
                           "nxtot": int(sysm.nx_total), "l2": "flushed before every step (256 MiB write)",
                           "parallelism": f"replicas x{world}",
                           "autotune": {"pupil_rows": tuned_rows, **tuned_fd,
                                        "lhs_ms_by_rows": {str(k): round(v, 4) for k, v in tuned_ms.items()}}},
                "latency_ms": {"p50": p50, "p99": p99, "note": "one batched step of all instances"},
                "single_instance": single,
                "e2e": {"value": e2e_value, "unit": "steps/s",
                        "h2d_bytes_per_step": int(B * sysm.ngrad * 4),
                        "d2h_bytes_per_step": int(B * fit.nact * 4),
                        "api": "mb_recon_serve_step, pinned FP32 host buffers",
                        "fp64_gpu_tomo_gpu_fit_steps_per_s": fp64_api_value},
                "mvm": mvm_line,
                "wfs_gradients": wfs_line,
                "closed_loop": loop_line,
                "grouped_mix": grouped,
                "served": served,
                "served_sustained_rate": served_low,
                "served_mvm": served_mvm,
                "gpu_launches": int(launches), "clocks": clocks, "roofline": roof,
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    R.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
