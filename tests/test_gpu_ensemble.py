"""GPU: the ensemble path (cf_create_batch / cf_step_batch) against the same
channels stepped one at a time, and against the oracle.

An ensemble runs the same arithmetic as a single handle (only the parameter
staging differs), so every member must match its stand-alone twin to
rounding; one member is also checked against the CPU oracle at the step
tolerance.
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LX, LZ = 2 * np.pi / 1.14, 2 * np.pi / 2.5


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def members():
    g1 = cfb200.Grid(16, 17, 16, LX, LZ)
    g2 = cfb200.Grid(24, 25, 20, 2 * np.pi, np.pi)
    out = []
    for nu in (1 / 300, 1 / 400, 1 / 500):
        out.append(dict(grid=g1, profile="couette", nu=nu, dt=0.01))
    for nu in (1 / 1000, 1 / 1500):
        out.append(dict(grid=g2, profile="poiseuille", nu=nu, dt=0.005, bulkvelocity=(2 / 3, 0.0)))
    # the Chebyshev length of the 48x49x48 ensemble members (P = 48)
    g3 = cfb200.Grid(12, 49, 10, LX, LZ)
    for nu in (1 / 350, 1 / 450):
        out.append(dict(grid=g3, profile="couette", nu=nu, dt=0.01))
    return out


def twin(m):
    kw = {k: v for k, v in m.items() if k not in ("grid", "profile", "nu", "dt")}
    return cfb200.ChannelFlowProblem(m["grid"], m["profile"], m["nu"], m["dt"], **kw)


def test_ensemble_matches_single_instances():
    ms = members()
    ens = cfb200.Ensemble(ms)
    assert len(ens) == 7
    twins = []
    for i, (m, inst) in enumerate(zip(ms, ens.instances)):
        cfb200.random_state(inst, 0.1, seed=100 + i)
        U, P = inst.get_state()
        t = twin(m)
        t.set_state(U, P)
        twins.append(t)
    nsteps = 15
    ens.step(nsteps)
    ens.step(nsteps)
    # three size classes, 12 launches per class per step
    assert ens.launches() == 12 * 3 * nsteps
    # the autotuner's choice per class is recorded (whatever it chose, the
    # arithmetic per column is the same, so the twins below agree to rounding)
    sched = ens.schedule()
    assert sched.count("column kernel ncol=") == 3, sched
    for inst, t in zip(ens.instances, twins):
        t.advance(0.0, 2 * nsteps)
        Ue, Pe = inst.get_state()
        Ut, Pt = t.get_state()
        assert np.all(np.isfinite(Ue))
        assert rel(Ue, Ut) <= 1e-13
        assert rel(Pe, Pt) <= 1e-11
        t.close()
    ens.close()


@pytest.mark.parametrize("which", [3, 6])
def test_ensemble_member_matches_oracle(which):
    ms = members()
    ens = cfb200.Ensemble(ms)
    m = ms[which]
    g = m["grid"]
    if m["profile"] == "poiseuille":
        ref = O.poiseuille(g.Nx, g.Ny, g.Nz, g.Lx, g.Lz, m["nu"], m["dt"], bulkvelocity=m["bulkvelocity"])
    else:
        ref = O.couette(g.Nx, g.Ny, g.Nz, g.Lx, g.Lz, m["nu"], m["dt"])
    U, P = ref.random_state(seed=7, amp=0.1)
    inst = ens.instances[which]
    inst.set_state(U, P)
    Ur, Pr = U.copy(), P.copy()
    ref.step(Ur, Pr, 10)
    ens.step(10)
    Ue, _ = inst.get_state()
    assert rel(Ue, Ur) <= 1e-12
    ens.close()
