"""The oracle on the reference's strongly nonlinear validation case: the
archived Waleffe R400 Couette equilibria (lower and upper branch) at
(Ny, N) = (35, 32) and (49, 48), stepped with dt = 0.025 and 0.0125 to
t = 0.25 and 0.5 by the rotational form (validation/waleffe_equilibrium.jl:
84-154).  Every recorded value of the reference's run
(validation/results/waleffe.csv) is matched: initial energy, the defect of
the stationary Stokes balance, and energy, dissipation, wall power input and
drift after each interval.

Tolerances (relative): energy and dissipation 1e-12, power input 2e-12
(a sum of wall derivatives), the defect and the drift 1e-11 (norms of
differences ~1e-5 .. 5e-4 of the state, so rounding of the state is amplified
by their inverse).  The oracle agrees to ~1e-14 on energy and dissipation and
~3e-13 on the power input.
"""
import numpy as np
import pytest

import waleffe as W
from oracle import oracle as O


def rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.parametrize("branch", ["LB", "UB"])
@pytest.mark.parametrize("Ny,N", [(35, 32), (49, 48)])
def test_waleffe_equilibrium_oracle(branch, Ny, N):
    U0 = W.perturbation(branch, Ny, N)
    ref = O.couette(N, Ny, N, W.LX, W.LZ, W.NU, 0.025)
    e0, d0, i0 = W.diagnostics(ref, U0)
    g = W.golden(branch, Ny, N, 0.025, 0.25)
    assert rel(e0, g["energy_initial"]) < 1e-12
    assert abs(i0 / d0 - 1) < 1e-3
    # pressure from the stationary Stokes balance with the imported source
    src = ref.nonlinear(U0)
    resp, P0, _ = ref.stokes(src, nu=W.NU, lam=0.0)
    defect = np.sqrt(W.diagnostics(ref, resp - U0)[0] / e0)
    assert rel(defect, g["defect"]) < 1e-11
    for dt in (0.025, 0.0125):
        pb = O.couette(N, Ny, N, W.LX, W.LZ, W.NU, dt)
        U, P = U0.copy(), P0.copy()
        for t in (0.25, 0.5):
            pb.step(U, P, int(round(0.25 / dt)))
            gd = W.golden(branch, Ny, N, dt, t)
            e, d, i = W.diagnostics(pb, U)
            drift = np.sqrt(W.diagnostics(pb, U - U0)[0] / e0)
            assert rel(e, gd["energy"]) < 1e-12, (dt, t, e, gd["energy"])
            assert rel(d, gd["dissipation"]) < 1e-12, (dt, t, d, gd["dissipation"])
            assert rel(i, gd["input"]) < 2e-12, (dt, t, i, gd["input"])
            assert rel(drift, gd["drift"]) < 1e-11, (dt, t, drift, gd["drift"])
