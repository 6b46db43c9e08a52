"""Uneven instances advanced together (mb_group_*).

Three reconstructors of different geometries and batch sizes -- 8 m SCAO
(2 instances), 8 m LTAO (plain CG, 2 instances) and 30 m MCAO (FDPCG,
3 instances) -- are stepped by one group graph in which the tomography
operators are single launches over all their instances.  Every instance's DM
commands must equal those of its own reconstructor stepped alone, bit for bit
(the group runs each member's own arithmetic), over two warm-started steps;
and the group step must take fewer kernel launches than the three steps
alone.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MEMBERS = (("scao_8m", 2), ("ltao_8m", 2), ("mcao_30m", 3))


@pytest.fixture(scope="module")
def group():
    from conftest import get_fit_assembled, get_system
    from maos_b200 import turbulence
    from maos_b200.recon import Reconstructor, ReconGroup
    rs, grads = [], []
    for name, nb in MEMBERS:
        s = get_system(name)
        R = Reconstructor(s, nbatch=nb, fit=get_fit_assembled(name))
        rs.append(R)
        fr = turbulence.gradient_frames(s, seed=3, nframe=2 * nb).astype(np.float32)
        grads.append(torch.tensor(fr.reshape(2, nb, -1), device="cuda"))
    G = ReconGroup(rs)
    yield rs, G, grads
    G.close()
    for R in rs:
        R.close()


def _commands(rs):
    torch.cuda.synchronize()
    return [R.fit_solution().cpu().numpy().copy() for R in rs]


def test_group_step_equals_members_alone(group):
    rs, G, grads = group
    lib = rs[0].lib
    alone = []
    lib.mb_kernel_launches(1)
    for R in rs:
        R.reset()
    for step in range(2):
        for R, g in zip(rs, grads):
            R.step_device(g[step].data_ptr())
        alone.append(_commands(rs))
    n_alone = lib.mb_kernel_launches(1) / 2
    together = []
    for R in rs:
        R.reset()
    for step in range(2):
        G.step_device([g[step].data_ptr() for g in grads])
        together.append(_commands(rs))
    n_group = lib.mb_kernel_launches(1) / 2
    for step in range(2):
        for i, (name, nb) in enumerate(MEMBERS):
            a, b = alone[step][i], together[step][i]
            assert a.shape == (nb, rs[i].nact)
            assert np.all(np.isfinite(b)) and np.abs(a).max() > 0
            assert np.array_equal(a, b), (name, step, float(np.abs(a - b).max()))
    assert G.graph_kernels == n_group
    assert n_group < n_alone, (n_group, n_alone)
    print(f"kernel launches per step: group {n_group:.0f}, members alone {n_alone:.0f}")


def test_group_follows_a_member_table_update(group):
    """After a member's tables change (here a re-autotune, which recaptures
    the member's graph), the group recaptures before its next step and still
    matches the member alone."""
    rs, G, grads = group
    rs[2].autotune(reps=3)
    for R in rs:
        R.reset()
    G.step_device([g[0].data_ptr() for g in grads])
    together = _commands(rs)
    for R in rs:
        R.reset()
    for R, g in zip(rs, grads):
        R.step_device(g[0].data_ptr())
    alone = _commands(rs)
    for i in range(len(rs)):
        assert np.array_equal(alone[i], together[i])
