"""GPU: the convective and divergence nonlinear forms (src/nonlinear.jl:113-167)
and the Flows adapter's shortened final step (ext/ChannelFlowFlowsExt.jl:36-52)
against the oracle, through the C ABI.

Tolerances are those of the rotational form (test_gpu_parity.py): the
nonlinear term to 1e-13 of its largest coefficient (scaled by (Ny-1)/16 for
the divergence form's y derivative of the products), the velocity to 1e-12
relative L2 after a few steps and 1e-11 after 100, the stage pressure to 1e-9.
The reference's own CUDA test runs the same three forms for five steps at
N = 8, 9, 16 (test/cuda/runtests.jl:29-66).
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FORMS = ["convective", "divergence"]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def pair(Nx, Ny, Nz, Lx, Lz, nu, dt, form, profile="couette", bulkvelocity=None):
    g = cfb200.Grid(Nx, Ny, Nz, Lx, Lz)
    if profile == "couette":
        return (cfb200.CouetteFlow(g, nu, dt, form=form),
                O.couette(Nx, Ny, Nz, Lx, Lz, nu, dt, form=form))
    return (cfb200.PoiseuilleFlow(g, nu, dt, bulkvelocity=bulkvelocity, form=form),
            O.poiseuille(Nx, Ny, Nz, Lx, Lz, nu, dt, bulkvelocity=bulkvelocity, form=form))


@pytest.mark.parametrize("form", FORMS)
def test_analytic_nonlinear_forms(form):
    # test_nonlinear.jl:1-38: total velocity (y^2 + y, 1, 0) gives -(2y + 1) e_x
    g = cfb200.Grid(5, 9, 5, 2 * np.pi, 2 * np.pi)
    gpu = cfb200.ChannelFlowProblem(g, lambda y: y, 0.01, 0.01, form=form)
    ref = O.OracleProblem(5, 9, 5, 2 * np.pi, 2 * np.pi, 0.01, 0.01, lambda y: y, form=form)
    U = np.stack([ref.spectral(lambda x, y, z: y**2 + 0 * x), ref.spectral(lambda x, y, z: 1.0 + 0 * x),
                  ref.zeros()])
    saved = U.copy()
    N = gpu.nonlinear(U)
    assert np.max(np.abs(ref.ifft(N[0]) - ref.sample(lambda x, y, z: -(2 * y + 1) + 0 * x))) < 2e-11
    assert np.max(np.abs(ref.ifft(N[1]))) < 2e-11
    assert np.max(np.abs(ref.ifft(N[2]))) < 2e-11
    assert np.array_equal(U, saved)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("dims", [(16, 17, 16), (9, 17, 7), (6, 13, 10), (48, 33, 40), (8, 81, 1), (384, 17, 4)])
def test_nonlinear_term_forms(form, dims):
    # (384, 17, 4): padded x length 576, the x-pass with in-place transforms
    Nx, Ny, Nz = dims
    gpu, ref = pair(Nx, Ny, Nz, 5.3, 7.1, 0.01, 0.01, form)
    U = ref.synth(seed=3, amp=0.2)
    N_ref = ref.nonlinear(U)
    N_gpu = gpu.nonlinear(U)
    # the divergence form differentiates the transformed products in y, which
    # scales their rounding by up to 2P per degree (3.2e-13 of max |N| at Ny = 81)
    tol = 1e-13 if form == "convective" else 1e-13 * max(1.0, (Ny - 1) / 16)
    assert np.max(np.abs(N_gpu - N_ref)) <= tol * max(1.0, np.max(np.abs(N_ref)))
    N_na = gpu.nonlinear_noalloc(U)
    assert np.array_equal(N_na, N_gpu)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("N", [8, 9, 16])
def test_five_steps_like_reference_cuda_test(form, N):
    # test/cuda/runtests.jl:29-66: Grid(N, 17, N, 2pi, 2pi), Couette Re=400,
    # dt=0.01, random state of amplitude 0.05, five steps
    gpu, ref = pair(N, 17, N, 2 * np.pi, 2 * np.pi, 1 / 400, 0.01, form)
    U, P = ref.random_state(seed=12, amp=0.05)
    gpu.set_state(U, P)
    gpu.advance(0.0, 5)
    Ug, Pg = gpu.get_state()
    ref.step(U, P, 5)
    assert rel(Ug, U) <= 1e-12
    assert rel(Pg, P) <= 1e-9
    assert gpu.diagnostics()[2] < 2e-9  # divergence


@pytest.mark.parametrize("form", FORMS)
def test_couette_100_steps(form):
    c = dict(Nx=32, Ny=33, Nz=32, Lx=2 * np.pi / 1.14, Lz=2 * np.pi / 2.5)
    gpu, ref = pair(**c, nu=1 / 400, dt=0.01, form=form)
    U, P = ref.random_state(seed=1, amp=0.1)
    gpu.set_state(U, P)
    gpu.advance(0.0, 100)
    Ug, Pg = gpu.get_state()
    ref.step(U, P, 100)
    assert rel(Ug, U) <= 1e-11
    assert rel(Pg, P) <= 1e-8


@pytest.mark.parametrize("form", FORMS)
def test_poiseuille_bulk_flux_forms(form):
    nu = (2 / 3) / 2800
    gpu, ref = pair(32, 33, 24, 4 * np.pi, 4 * np.pi / 3, nu, 0.005, form, profile="poiseuille",
                    bulkvelocity=(2 / 3, 0.0))
    U, P = ref.random_state(seed=4, amp=0.2, shape=1, rho=0.7)
    gpu.set_state(U, P)
    _, gg = gpu.advance(0.0, 20)
    Ug, _ = gpu.get_state()
    go = ref.step(U, P, 20)
    assert rel(Ug, U) <= 1e-11
    assert abs(gg[0] - go[0]) <= 1e-13 + 1e-8 * abs(go[0])


@pytest.mark.parametrize("form", FORMS)
def test_random_state_and_pressure_forms(form):
    # pressure.jl:95-104 with the form's own nonlinear term (the ordinary pressure)
    gpu, ref = pair(16, 17, 12, 5.3, 7.1, 1 / 400, 0.01, form)
    st = cfb200.random_state(gpu, 0.1, seed=9)
    Ur, Pr = ref.random_state(seed=9, amp=0.1)
    assert np.max(np.abs(st.U - Ur)) < 1e-11 * np.max(np.abs(Ur))
    assert np.max(np.abs(st.P - Pr)) < 1e-9 * np.max(np.abs(Pr))


@pytest.mark.parametrize("form", FORMS)
def test_laminar_couette_pressure_vanishes(form):
    # test_projection.jl:77-87 holds y^2/2 - 1/6 for the rotational form's
    # modified pressure; the ordinary pressure of laminar Couette flow is uniform
    g = cfb200.Grid(5, 9, 5, 2 * np.pi, 2 * np.pi)
    gpu = cfb200.CouetteFlow(g, 0.01, 0.01, form=form)
    U = cfb200.project_(np.zeros((3,) + g.spectralsize, np.complex128), gpu)
    assert np.max(np.abs(cfb200.pressure(U, gpu))) < 2e-12


def test_exact_viscous_decay_convective():
    # test/cuda/runtests.jl:123-140: x-independent streamwise velocity
    # cos(pi y/2) cos(z), zero base profile, convective form: amplitude
    # exp(-nu (pi^2/4 + 1) t) to rtol 2e-8 after 50 steps
    g = cfb200.Grid(8, 33, 8, 2 * np.pi, 2 * np.pi)
    nu, dt, stop = 0.1, 0.002, 0.1
    gpu = cfb200.ChannelFlowProblem(g, lambda y: 0.0 * y, nu, dt, form="convective")
    ref = O.OracleProblem(8, 33, 8, 2 * np.pi, 2 * np.pi, nu, dt, lambda y: 0.0 * y, form="convective")
    prof = ref.spectral(lambda x, y, z: np.cos(np.pi * y / 2) * np.cos(z) + 0 * x)
    st = cfb200.zero_state(g)
    st.U[0] = prof
    st.P[...] = cfb200.pressure(st.U, gpu)
    cfb200.flow(gpu)(st, (0.0, stop))
    exact = prof * np.exp(-nu * (np.pi**2 / 4 + 1) * stop)
    assert np.max(np.abs(st.U[0] - exact)) <= 2e-10 + 2e-8 * np.max(np.abs(exact))


@pytest.mark.parametrize("profile", ["couette", "poiseuille"])
def test_shortened_final_step(profile):
    # test/cuda/runtests.jl:104-118: an interval ending between nominal steps
    # (0, 0.025) with dt = 0.01: two nominal steps and one of 0.005 with its
    # own factors; the nominal factors stay for later steps
    kw = {"bulkvelocity": (2 / 3, 0.0)} if profile == "poiseuille" else {}
    g = cfb200.Grid(8, 17, 8, 2 * np.pi, 2 * np.pi)
    if profile == "couette":
        gpu = cfb200.CouetteFlow(g, 1 / 400, 0.01)
        ref = O.couette(8, 17, 8, 2 * np.pi, 2 * np.pi, 1 / 400, 0.01)
    else:
        gpu = cfb200.PoiseuilleFlow(g, 1 / 400, 0.01, **kw)
        ref = O.poiseuille(8, 17, 8, 2 * np.pi, 2 * np.pi, 1 / 400, 0.01, **kw)
    U, P = ref.random_state(seed=82, amp=0.02)
    st = cfb200.State(U.copy(), P.copy())
    assert cfb200.flow(gpu)(st, (0.0, 0.025)) is st
    ref.step(U, P, 2)
    ref.step_dt(U, P, 0.005)
    assert rel(st.U, U) <= 1e-12
    assert rel(st.P, P) <= 1e-9
    # the nominal step is unchanged after the shortened one
    gpu.set_state(st.U, st.P)
    t, _ = gpu.advance(0.025, 3)
    ref.step(U, P, 3)
    Ug, _ = gpu.get_state()
    assert abs(t - 0.055) < 1e-14
    assert rel(Ug, U) <= 1e-12


def test_step_dt_nominal_is_step():
    g = cfb200.Grid(16, 17, 16, 5.3, 7.1)
    a = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    b = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    st = cfb200.random_state(a, 0.1, seed=3)
    b.set_state(st.U, st.P)
    a.advance(0.0, 1)
    t, _ = b.advance_dt(0.0, 0.01)
    assert t == 0.01
    assert np.array_equal(a.get_state()[0], b.get_state()[0])
    # a repeated shortened step reuses its factors (and agrees with a fresh handle)
    c = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    c.set_state(st.U, st.P)
    b.set_state(st.U, st.P)
    b.advance_dt(0.0, 0.004)
    b.advance_dt(0.004, 0.004)
    c.advance_dt(0.0, 0.004)
    c.advance_dt(0.004, 0.004)
    assert np.array_equal(b.get_state()[0], c.get_state()[0])


def test_mixed_and_ensembles_need_rotational_form():
    g = cfb200.Grid(16, 17, 16, 5.3, 7.1)
    with pytest.raises(cfb200.CFError):
        cfb200.CouetteFlow(g, 1 / 400, 0.01, form="convective", precision="mixed")
    with pytest.raises(cfb200.CFError):
        cfb200.Ensemble([dict(grid=g, profile="couette", nu=1 / 400, dt=0.01, form="divergence")])
