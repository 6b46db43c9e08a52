"""Device geometric WFS (``mb_geom_wfs_*`` through ``maos_b200.wfs``) against
the FP64 oracle (``oracle/wfs_oracle.py``, whose ray tracing and GS0 are
pinned to the reference's ``prop_grid`` and ``mkg``): open and closed loop,
moving atmosphere, noise drawn draw by draw, batched instances with their
own atmospheres.  Tolerance: relative L2 error 2e-5 of the gradient vector
(FP32 OPD and stencil sums against FP64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-5


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / np.linalg.norm(b))


def _screens(atm, dms_cmd=None, fit=None):
    from oracle import wfs_oracle
    n, dx = atm.n, atm.dx
    o = -n / 2 * dx
    layers = [wfs_oracle.Screen(s, o, o, dx, float(h), float(atm.vx[l]), float(atm.vy[l]))
              for l, (s, h) in enumerate(zip(atm.screens, atm.cfg.atm_ht))]
    dms = []
    if dms_cmd is not None:
        off = fit.act_offsets()
        for k, dm in enumerate(fit.dms):
            a = dms_cmd[off[k]:off[k + 1]].reshape(dm.amap.ny, dm.amap.nx)
            dms.append(wfs_oracle.Screen(a, dm.amap.ox, dm.amap.oy, dm.amap.dx, dm.ht))
    return layers, dms


@pytest.fixture(scope="module")
def ltao():
    from conftest import get_system
    from maos_b200 import wfs_setup
    s = get_system("ltao_8m")
    return s, wfs_setup.build_geom_wfs(s)


def test_open_loop_matches_oracle(ltao):
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    from oracle import wfs_oracle
    s, geom = ltao
    atm = FrozenFlowAtmosphere(s.cfg, 3)
    W = GeomWfs.for_system(s, atm, geom=geom)
    layers, _ = _screens(atm)
    for isim in (0, 37):
        g = W.grad(isim).cpu().numpy()[0]
        ref = wfs_oracle.geom_grads(geom, layers, [], isim, s.cfg.sim_dt)
        assert rel(g, ref) < TOL, isim
    W.close()


def test_closed_loop_30m_with_noise_matches_oracle():
    import torch
    from conftest import get_system
    from maos_b200 import fit_setup, wfs_setup
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    from oracle import wfs_oracle
    s = get_system("mcao_30m")
    fit = fit_setup.build_fit(s)
    geom = wfs_setup.build_geom_wfs(s)
    atm = FrozenFlowAtmosphere(s.cfg, 5)
    W = GeomWfs.for_system(s, atm, fit=fit, geom=geom)
    rng = np.random.default_rng(2)
    a = (rng.standard_normal(fit.nact) * 2e-7).astype(np.float32)
    dm = torch.as_tensor(a, device="cuda")[None, :]
    layers, dms = _screens(atm, a.astype(np.float64), fit)
    gs0 = [p.gs0() for p in geom.powfs]
    g = W.grad(123, dm=dm).cpu().numpy()[0]
    ref = wfs_oracle.geom_grads(geom, layers, dms, 123, s.cfg.sim_dt, gs0=gs0)
    assert rel(g, ref) < TOL
    # the DMs change the gradients: the closed-loop term is really there
    g_ol = W.grad(123).cpu().numpy()[0]
    assert rel(g_ol, ref) > 100 * TOL
    # noise: the same draws as the oracle's generator
    gn = W.grad(123, dm=dm, seed=99).cpu().numpy()[0]
    refn = ref + wfs_oracle.geom_noise(geom, 99, 123)
    assert rel(gn, refn) < TOL
    noise = gn - g
    sig = np.concatenate([np.concatenate([geom.nea[i][0], geom.nea[i][1]]) for i in range(geom.nwfs)])
    z = noise / sig
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1.0) < 0.05
    W.close()


def test_batched_instances_have_their_own_atmosphere(ltao):
    import torch
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    from oracle import wfs_oracle
    s, geom = ltao
    atms = [FrozenFlowAtmosphere(s.cfg, 10 + i) for i in range(3)]
    W = GeomWfs.for_system(s, atms, nbatch=3, geom=geom)
    g = W.grad(5, seed=7).cpu().numpy()
    for i in range(3):
        layers, _ = _screens(atms[i])
        ref = wfs_oracle.geom_grads(geom, layers, [], 5, s.cfg.sim_dt, seed=7, inst=i)
        assert rel(g[i], ref) < TOL, i
    W1 = GeomWfs.for_system(s, atms[1], geom=geom)
    g1 = W1.grad(5).cpu().numpy()[0]
    g0 = W.grad(5).cpu().numpy()[1]
    assert np.array_equal(g1, g0)   # an instance's result does not depend on the batch
    W.close()
    W1.close()


def test_invalid_arguments_raise(ltao):
    from maos_b200.native import MbError
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    s, geom = ltao
    W = GeomWfs.for_system(s, FrozenFlowAtmosphere(s.cfg, 1), geom=geom)
    with pytest.raises(MbError):
        W.grad(-1)
    with pytest.raises(MbError):
        W.set_atm(1, 0, np.zeros(4))
    W.close()


def test_loop_closes_on_the_device():
    """WFS -> tomography + fit -> servo -> DMs -> WFS, all on the GPU, on a
    frozen atmosphere: the closed-loop gradients shrink to the fitting error."""
    import torch
    from conftest import get_fit, get_system
    from maos_b200.recon import Reconstructor
    from maos_b200.servo import Servo
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    s = get_system("scao_8m")
    fit = get_fit("scao_8m")
    W = GeomWfs.for_system(s, FrozenFlowAtmosphere(s.cfg, 2), fit=fit)
    R = Reconstructor(s, nbatch=1, fit=fit)
    S = Servo(fit.nact, ep=[[0.5]], dt=s.cfg.sim_dt)
    st = torch.cuda.current_stream()
    dm = torch.zeros(1, fit.nact, dtype=torch.float32, device="cuda")
    fa = torch.zeros(fit.nact, dtype=torch.float32, device="cuda")
    rms = []
    for k in range(20):
        g = W.grad(0, dm=dm)
        rms.append(float(g.norm()))
        R.step_device(g.data_ptr(), st.cuda_stream)
        if k % 2:   # the commands through a copy, or in place on the device
            R.slot_download(0, fa.data_ptr(), st.cuda_stream)
        else:
            fa.copy_(R.fit_solution()[0])
        cmd = S.filter(fa.double(), stream=st)
        dm.copy_(cmd.float()[None, :])
    torch.cuda.synchronize()
    print("closed-loop gradient rms / open loop:", [round(r / rms[0], 4) for r in rms])
    assert rms[-1] < 0.3 * rms[0]
    assert rms[-1] <= 1.05 * min(rms[10:])
    R.close()
    S.close()
    W.close()


def test_widest_subaperture_window_matches_oracle():
    """34 OPD points across a subaperture (the widest window, 36 x 36: four
    columns beyond the warp's 32 lanes)."""
    from conftest import get_fit, get_system
    from maos_b200 import wfs_setup
    from maos_b200.turbulence import FrozenFlowAtmosphere
    from maos_b200.wfs import GeomWfs
    from oracle import wfs_oracle
    s = get_system("scao_8m")
    fit = get_fit("scao_8m")
    geom = wfs_setup.build_geom_wfs(s, sim_dx=s.wfs[0].dsa / 34)
    assert geom.powfs[0].nxsa == 34
    atm = FrozenFlowAtmosphere(s.cfg, 6)
    W = GeomWfs.for_system(s, atm, fit=fit, geom=geom)
    import torch
    a = (np.random.default_rng(4).standard_normal(fit.nact) * 1e-7).astype(np.float32)
    g = W.grad(9, dm=torch.as_tensor(a, device="cuda")[None, :], seed=3).cpu().numpy()[0]
    layers, dms = _screens(atm, a.astype(np.float64), fit)
    ref = wfs_oracle.geom_grads(geom, layers, dms, 9, s.cfg.sim_dt, seed=3)
    assert rel(g, ref) < TOL
    W.close()
