"""GPU: the engine on the reference's strongly nonlinear validation case, the
archived Waleffe R400 Couette equilibria (validation/waleffe_equilibrium.jl:
84-154), run as the reference runs it: each branch at (Ny, N) = (35, 32) and
(49, 48), the pressure from the stationary Stokes balance, then Flows
intervals (t - 0.25, t) for t = 0.25, 0.5 with dt = 0.025 and 0.0125
(cfb200.flow, the Flows adapter's protocol).  Every recorded value of the
reference's run (validation/results/waleffe.csv) is matched with the
tolerances of the oracle's test (energy and dissipation 1e-12 relative,
power input 2e-12, drift 1e-11), and the state agrees with the oracle's to
1e-12 after each interval.  The diagnostics are evaluated by the oracle's
transforms (the checker) on the engine's state.
"""
import numpy as np
import pytest

import cfb200
import waleffe as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.parametrize("branch", ["LB", "UB"])
@pytest.mark.parametrize("Ny,N", [(35, 32), (49, 48)])
def test_waleffe_equilibrium_engine(branch, Ny, N):
    U0 = W.perturbation(branch, Ny, N)
    chk = O.couette(N, Ny, N, W.LX, W.LZ, W.NU, 0.025)
    e0 = W.diagnostics(chk, U0)[0]
    _, P0, _ = chk.stokes(chk.nonlinear(U0), nu=W.NU, lam=0.0)
    g = cfb200.Grid(N, Ny, N, W.LX, W.LZ)
    for dt in (0.025, 0.0125):
        pb = cfb200.CouetteFlow(g, W.NU, dt)
        ref = O.couette(N, Ny, N, W.LX, W.LZ, W.NU, dt)
        flow = cfb200.flow(pb)
        st = cfb200.State(U0.copy(), P0.copy())
        Ur, Pr = U0.copy(), P0.copy()
        for t in (0.25, 0.5):
            flow(st, (t - 0.25, t))
            ref.step(Ur, Pr, int(round(0.25 / dt)))
            assert np.linalg.norm(st.U - Ur) <= 1e-12 * np.linalg.norm(Ur)
            gd = W.golden(branch, Ny, N, dt, t)
            e, d, i = W.diagnostics(chk, st.U)
            drift = np.sqrt(W.diagnostics(chk, st.U - U0)[0] / e0)
            assert rel(e, gd["energy"]) < 1e-12, (dt, t, e, gd["energy"])
            assert rel(d, gd["dissipation"]) < 1e-12, (dt, t, d, gd["dissipation"])
            assert rel(i, gd["input"]) < 2e-12, (dt, t, i, gd["input"])
            assert rel(drift, gd["drift"]) < 1e-11, (dt, t, drift, gd["drift"])
        pb.close()
