"""GPU: the mixed-precision step (FP32 periodic transforms and products,
tensor-core Chebyshev transforms with TF32 heads and remainders, FP64
Stokes solve) against the FP64 step of the oracle and of the engine.

The nonlinear term carries FP32 rounding (~1e-7 relative), which the step
passes to the velocity through dt * N; the tolerances below (1e-5 relative L2
on the velocity, 1e-6 on the kinetic energy) bound that, and the divergence
and the constant-flux constraint must hold as in the FP64 form (they are
imposed by the FP64 Stokes solve).  With the state stored in FP32
("mixed-f32state") the new state is rounded to FP32 after every stage, so the
divergence holds to that rounding (bound 1e-6 below) instead of to FP64
rounding; the mean-flow mode stays FP64, so the bulk velocity still holds to
1e-9.
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C1 = dict(Nx=32, Ny=33, Nz=32, Lx=2 * np.pi / 1.14, Lz=2 * np.pi / 2.5)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


MIXED = ["mixed", "mixed-tc", "mixed-bf16", "mixed-f32state"]
# divergence bound: FP64 rounding, or the FP32 rounding of a stored state
DIV_TOL = {"mixed-f32state": 1e-6}


@pytest.mark.parametrize("precision", MIXED)
def test_mixed_couette_matches_oracle(precision):
    c = C1
    g = cfb200.Grid(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"])
    mx = cfb200.CouetteFlow(g, 1 / 400, 0.01, precision=precision)
    ref = O.couette(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"], 1 / 400, 0.01)
    U, P = ref.random_state(seed=1, amp=0.1)
    mx.set_state(U, P)
    Ur, Pr = U.copy(), P.copy()
    ref.step(Ur, Pr, 10)
    mx.advance(0.0, 10)
    Um, _ = mx.get_state()
    assert np.all(np.isfinite(Um))
    e10 = rel(Um, Ur)
    assert e10 <= 1e-5, e10
    ref.step(Ur, Pr, 90)
    mx.advance(0.0, 90)
    Um, _ = mx.get_state()
    e100 = rel(Um, Ur)
    assert e100 <= 1e-5, e100
    dm, dr = mx.diagnostics(), ref.diagnostics(Ur)
    assert abs(dm[0] - dr[0]) <= 1e-6 * abs(dr[0])
    assert dm[2] <= DIV_TOL.get(precision, 1e-10)  # divergence
    mx.close()


@pytest.mark.parametrize("precision", MIXED)
def test_mixed_poiseuille_flux_matches_fp64_engine(precision):
    g = cfb200.Grid(24, 25, 20, 2 * np.pi, np.pi)
    kw = dict(bulkvelocity=(2 / 3, 0.0))
    f64 = cfb200.PoiseuilleFlow(g, 1 / 1500, 0.005, **kw)
    mx = cfb200.PoiseuilleFlow(g, 1 / 1500, 0.005, precision=precision, **kw)
    st = cfb200.random_state(f64, 0.1, seed=4)
    mx.set_state(st.U, st.P)
    _, g64 = f64.advance(0.0, 20)
    _, gmx = mx.advance(0.0, 20)
    U64, _ = f64.get_state()
    Umx, _ = mx.get_state()
    assert rel(Umx, U64) <= 1e-5
    # the mean gradient carries the FP32 rounding of the bulk mean of N_x
    # (order 0.1 here) in absolute terms; the gradient itself is ~3e-4
    assert abs(gmx[0] - g64[0]) <= 1e-6
    # the perturbation's bulk velocity stays at its target (the FP64 constraint)
    ny = g.Ny
    n = np.arange(ny)
    w = np.zeros(ny)
    w[0::2] = 1.0 / (1.0 - n[0::2].astype(float) ** 2)
    assert abs(np.dot(w, Umx[0, :, 0, 0].real) - np.dot(w, U64[0, :, 0, 0].real)) <= 1e-9
    f64.close()
    mx.close()


@pytest.mark.parametrize("precision", MIXED)
# (384, 17, 4) and (341, 17, 4): the FP32 in-place x-pass at the padded
# lengths 576 and 512
@pytest.mark.parametrize("dims", [(9, 17, 7), (16, 17, 16), (48, 33, 40), (8, 257, 6), (384, 17, 4), (341, 17, 4)])
def test_mixed_one_step_sizes(dims, precision):
    Nx, Ny, Nz = dims
    g = cfb200.Grid(Nx, Ny, Nz, 5.3, 7.1)
    ref = O.couette(Nx, Ny, Nz, 5.3, 7.1, 1 / 300, 0.01)
    mx = cfb200.CouetteFlow(g, 1 / 300, 0.01, precision=precision)
    U, P = ref.random_state(seed=3, amp=0.2)
    mx.set_state(U, P)
    ref.step(U, P, 2)
    mx.advance(0.0, 2)
    Um, _ = mx.get_state()
    assert rel(Um, U) <= 1e-5
    mx.close()


def test_mixed_large_ny_without_tensor_cores():
    # the in-kernel FP64 Chebyshev transforms have no Ny limit of the
    # tensor-core images (Ny <= 512)
    g = cfb200.Grid(8, 577, 6, 5.3, 7.1)
    with pytest.raises(cfb200.CFError):
        cfb200.CouetteFlow(g, 1 / 300, 0.01, precision="mixed-tc")
    ref = O.couette(8, 577, 6, 5.3, 7.1, 1 / 300, 0.01)
    mx = cfb200.CouetteFlow(g, 1 / 300, 0.01, precision="mixed")
    U, P = ref.random_state(seed=3, amp=0.2)
    mx.set_state(U, P)
    ref.step(U, P, 1)
    mx.advance(0.0, 1)
    Um, _ = mx.get_state()
    assert rel(Um, U) <= 1e-5
    mx.close()


def test_f32state_round_trips_and_steps():
    # the state crosses the C ABI in FP64: before a step the FP64 copy comes
    # back unchanged; a step advances the FP32 state, and the next read is its
    # FP64 widening (equal to an FP32 rounding of the FP64 engine's state to
    # within the step's own FP32 error)
    c = C1
    g = cfb200.Grid(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"])
    mx = cfb200.CouetteFlow(g, 1 / 400, 0.01, precision="mixed-f32state")
    ref = O.couette(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"], 1 / 400, 0.01)
    U, P = ref.random_state(seed=2, amp=0.1)
    mx.set_state(U, P)
    U1, P1 = mx.get_state()
    assert np.array_equal(U1, U) and np.array_equal(P1, P)
    mx.advance(0.0, 3)
    U3, _ = mx.get_state()
    # every value is an FP32 number after a step, except the mean-flow mode
    # (kx = kz = 0, stored in FP64)
    rest = U3.copy()
    rest[:, :, 0, 0] = 0
    assert np.array_equal(rest, rest.astype(np.complex64).astype(np.complex128))
    m = U3[:, :, 0, 0]
    assert not np.array_equal(m, m.astype(np.complex64).astype(np.complex128))
    ref.step(U, P, 3)
    assert rel(U3, U) <= 1e-5
    # diagnostics read the widened state; a new state written through the
    # ABI replaces the stepped one
    d = mx.diagnostics()
    assert abs(d[0] - ref.diagnostics(U3)[0]) <= 1e-12 * abs(d[0])
    mx.set_state(U1, P1)
    assert np.array_equal(mx.get_state()[0], U1)
    # the host-buffer step runs as set, step and get
    Uh, Ph = U1.copy(), P1.copy()
    cfb200.step_(mx, Uh, Ph, 0.0, 3)
    assert np.array_equal(Uh, U3)
    mx.close()


def test_f32state_rejects_a_step_of_another_duration():
    g = cfb200.Grid(16, 17, 16, 5.3, 7.1)
    mx = cfb200.CouetteFlow(g, 1 / 400, 0.01, precision="mixed-f32state")
    with pytest.raises(cfb200.CFError) as e:
        mx.advance_dt(0.0, 0.004)
    assert e.value.code == cfb200.CF_E_UNSUPPORTED
    mx.close()
