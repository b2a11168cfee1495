"""GPU parity of the CUDA engine against the CPU oracle, through the C ABI.

Tolerances (FP64 plain form): velocity agrees to <= 1e-12 relative L2 after a
few steps and <= 1e-11 after 100 steps (32x33x32 Couette, Re=400).  The stage
pressure is looser (<= 1e-9 .. 1e-8): its top Chebyshev modes come from the
tau correction, sigma = (shift*v_{P-1} + (Dp)_{P-1} - Ry_{P-1})/(1 - sigma0),
a difference of large terms multiplied by the auxiliary pressure response, so
rounding differences in v are amplified in p.  A pressure error is a pure
gradient in the next stage's source, which the Stokes solve absorbs into the
new pressure, so it never reaches the velocity.  The reference's own CPU/GPU
parity tests allow the same order (rtol 2e-10 after 5 steps at 16^3 and 1e-8
on 32^3..128^3, test/cuda/runtests.jl:61,170).
"""
import json
import os

import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C1 = dict(Nx=32, Ny=33, Nz=32, Lx=2 * np.pi / 1.14, Lz=2 * np.pi / 2.5)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def pair(Nx, Ny, Nz, Lx, Lz, nu, dt, profile="couette", **kw):
    g = cfb200.Grid(Nx, Ny, Nz, Lx, Lz)
    if profile == "couette":
        return cfb200.CouetteFlow(g, nu, dt, **kw), O.couette(Nx, Ny, Nz, Lx, Lz, nu, dt, **_oc(kw))
    return cfb200.PoiseuilleFlow(g, nu, dt, **kw), O.poiseuille(Nx, Ny, Nz, Lx, Lz, nu, dt, **kw)


def _oc(kw):
    if "bulkvelocity" in kw:
        return {"constraint": ("bulkvelocity", kw["bulkvelocity"])}
    if "pressuregradient" in kw:
        return {"constraint": ("pressuregradient", kw["pressuregradient"])}
    return {}


# (384, 9, 48) and (341, 9, 6): the in-place x-pass at the padded lengths 576
# and 512 (Nx = 341: Nxp = 512)
@pytest.mark.parametrize("dims", [(16, 17, 16), (32, 33, 32), (8, 9, 8), (9, 17, 7), (8, 81, 1), (6, 13, 10),
                                  (48, 9, 384), (384, 9, 48), (341, 9, 6)])
def test_nonlinear_term(dims):
    Nx, Ny, Nz = dims
    gpu, ref = pair(Nx, Ny, Nz, 5.3, 7.1, 0.01, 0.01)
    U = ref.synth(seed=3, amp=0.2)
    N_ref = ref.nonlinear(U)
    N_gpu = gpu.nonlinear(U)
    assert np.max(np.abs(N_gpu - N_ref)) <= 1e-13 * max(1.0, np.max(np.abs(N_ref)))


def test_projection_and_pressure():
    gpu, ref = pair(24, 25, 20, 5.3, 7.1, 1 / 300, 0.01, profile="poiseuille", bulkvelocity=(2 / 3, 0.0))
    U = ref.synth(seed=5, amp=0.1)
    Ur = ref.project(U)
    Ug = cfb200.project_(U.copy(), gpu)
    assert np.max(np.abs(Ug - Ur)) < 1e-11 * np.max(np.abs(Ur))
    Pr = ref.pressure(Ur)
    Pg = cfb200.pressure(Ur, gpu)
    assert np.max(np.abs(Pg - Pr)) < 1e-9 * max(1.0, np.max(np.abs(Pr)))


def test_random_state_matches_oracle():
    gpu, ref = pair(16, 17, 12, 5.3, 7.1, 1 / 400, 0.01)
    st = cfb200.random_state(gpu, 0.1, seed=9, shape=0)
    Ur, Pr = ref.random_state(seed=9, amp=0.1, shape=0)
    assert np.max(np.abs(st.U - Ur)) < 1e-11 * np.max(np.abs(Ur))
    assert np.max(np.abs(st.P - Pr)) < 1e-9 * np.max(np.abs(Pr))


@pytest.mark.parametrize("dims", [(16, 17, 16), (8, 9, 8), (9, 17, 7), (6, 13, 10)])
def test_one_step(dims):
    Nx, Ny, Nz = dims
    gpu, ref = pair(Nx, Ny, Nz, 5.3, 7.1, 1 / 400, 0.01)
    U, P = ref.random_state(seed=2, amp=0.1)
    gpu.set_state(U, P)
    gpu.advance(0.0, 1)
    Ug, Pg = gpu.get_state()
    ref.step(U, P, 1)
    assert rel(Ug, U) < 1e-12 and rel(Pg, P) < 1e-9


def test_c1_couette_100_steps():
    # Plain FP64 Couette Re=400, 32x33x32, Lx=2pi/1.14, Lz=2pi/2.5, dt=0.01, amplitude 0.1
    gpu, ref = pair(**C1, nu=1 / 400, dt=0.01)
    U, P = ref.random_state(seed=1, amp=0.1, shape=0)
    gpu.set_state(U, P)
    t, _ = gpu.advance(0.0, 100)
    Ug, Pg = gpu.get_state()
    ref.step(U, P, 100)
    assert abs(t - 1.0) < 1e-12
    assert rel(Ug, U) <= 1e-11
    assert rel(Pg, P) <= 1e-8
    dg = gpu.diagnostics()
    do = ref.diagnostics(U)
    assert abs(dg[0] - do[0]) <= 1e-11 * abs(do[0])  # kinetic energy
    assert abs(dg[1] - do[1]) <= 1e-11 * abs(do[1])  # dissipation
    assert dg[2] < 2e-9  # divergence


def test_poiseuille_bulk_flux():
    # constant flux with Ub = 1 - y^2 (device-side flux gradient, no host round trip)
    nu = (2 / 3) / 2800
    gpu, ref = pair(32, 33, 24, 4 * np.pi, 4 * np.pi / 3, nu, 0.005, profile="poiseuille", bulkvelocity=(2 / 3, 0.0))
    U, P = ref.random_state(seed=4, amp=0.2, shape=1, rho=0.7)
    gpu.set_state(U, P)
    _, gg = gpu.advance(0.0, 20)
    Ug, Pg = gpu.get_state()
    go = ref.step(U, P, 20)
    assert rel(Ug, U) <= 1e-11
    assert abs(gg[0] - go[0]) <= 1e-13 + 1e-8 * abs(go[0])
    assert abs(gg[1] - go[1]) <= 1e-13 + 1e-8 * abs(go[1])


def test_prescribed_gradient_poiseuille():
    nu = 1 / 2000
    gpu, ref = pair(16, 33, 16, 2 * np.pi, np.pi, nu, 0.01, profile="poiseuille")
    U, P = ref.random_state(seed=8, amp=0.05)
    gpu.set_state(U, P)
    gpu.advance(0.0, 10)
    Ug, _ = gpu.get_state()
    ref.step(U, P, 10)
    assert rel(Ug, U) <= 1e-12


def test_larger_grid_one_step():
    gpu, ref = pair(64, 65, 64, 2 * np.pi, 2 * np.pi, 1 / 400, 0.002)
    U, P = ref.random_state(seed=6, amp=0.1)
    gpu.set_state(U, P)
    gpu.advance(0.0, 2)
    Ug, Pg = gpu.get_state()
    ref.step(U, P, 2)
    assert rel(Ug, U) <= 1e-12 and rel(Pg, P) <= 1e-8


def test_tollmien_schlichting_on_gpu():
    # validation/tollmien_schlichting.jl on the engine; golden error from the reference run
    from test_oracle_validation import GOLD, poiseuille_ts_mode

    s, mu_, mv, mp = poiseuille_ts_mode(81)
    nu, amp, T = 1 / 8000, 1e-7, 50.0
    gold = {r["dt"]: r["error"] for r in GOLD["ts_convergence"]}
    errors = []
    for dt in (0.4, 0.2, 0.1):
        gpu = cfb200.PoiseuilleFlow(cfb200.Grid(8, 81, 1, 2 * np.pi, 2 * np.pi), nu, dt)
        st = cfb200.zero_state(gpu.grid)
        st.U[0][:, 0, 1] = amp / 2 * mu_
        st.U[1][:, 0, 1] = amp / 2 * mv
        st.P[:, 0, 1] = amp / 2 * mp
        init = st.U.copy()
        gpu.set_state(st.U, st.P)
        gpu.advance(0.0, int(round(T / dt)))
        U, _ = gpu.get_state()
        exact = init * np.exp((0.002664410371 - 0.2470750602j) * T)
        err = np.sqrt(np.sum(np.abs(U - exact) ** 2) / np.sum(np.abs(exact) ** 2))
        assert abs(err / gold[dt] - 1) < 1e-4, (dt, err, gold[dt])
        errors.append(err)
    assert errors[0] / errors[1] > 3.5 and errors[1] / errors[2] > 3.5


def test_step_interface_host_buffers():
    gpu, ref = pair(16, 17, 16, 5.3, 7.1, 1 / 400, 0.01)
    U, P = ref.random_state(seed=12, amp=0.05)
    Uh, Ph = U.copy(), P.copy()
    t = cfb200.step_(gpu, Uh, Ph, 0.25, nsteps=3)
    ref.step(U, P, 3)
    assert abs(t - 0.28) < 1e-14
    assert rel(Uh, U) < 1e-12


def test_handles_of_different_grids_coexist():
    # 16x17x16 and 24x25x20 share the run-time-sized kernel instantiations;
    # creating the smaller handle last must not restrict the larger one
    big, ref_big = pair(24, 25, 20, 2 * np.pi, np.pi, 1 / 1000, 0.005, profile="poiseuille",
                        bulkvelocity=(2 / 3, 0.0))
    small, _ = pair(16, 17, 16, 5.3, 7.1, 1 / 300, 0.01)
    U, P = ref_big.random_state(seed=12, amp=0.1)
    big.set_state(U, P)
    big.advance(0.0, 3)
    ref_big.step(U, P, 3)
    Ug, _ = big.get_state()
    assert rel(Ug, U) <= 1e-12
    cfb200.random_state(small, 0.1, seed=1)
    big.close()
    small.close()


@pytest.mark.parametrize("dims,profile", [((16, 17, 16), "couette"), ((9, 17, 7), "couette"),
                                          ((24, 25, 20), "poiseuille")])
def test_device_diagnostics_match_oracle(dims, profile):
    Nx, Ny, Nz = dims
    kw = {"bulkvelocity": (2 / 3, 0.0)} if profile == "poiseuille" else {}
    gpu, ref = pair(Nx, Ny, Nz, 5.3, 7.1, 1 / 300, 0.01, profile=profile, **kw)
    U, P = ref.random_state(seed=21, amp=0.3)
    gpu.set_state(U, P)
    dg, do = gpu.diagnostics(), ref.diagnostics(U)
    for i in (0, 1):  # kinetic energy, dissipation
        assert abs(dg[i] - do[i]) <= 1e-12 * abs(do[i])
    assert abs(dg[2] - do[2]) <= 1e-12 + 1e-9 * abs(do[2])  # max |div|
    for i in (3, 4):  # wall shear of the mean mode
        assert abs(dg[i] - do[i]) <= 1e-12 * max(1.0, abs(do[i]))
    gpu.close()


@pytest.mark.parametrize("form", ["rotational", "convective", "divergence"])
@pytest.mark.parametrize("dims", [(8, 193, 6), (6, 385, 4)])
def test_long_columns_all_forms(dims, form):
    # Chebyshev lengths 192 and 384 (compile-time column kernels whose nodal
    # outputs are transformed two at a time) against the oracle
    Nx, Ny, Nz = dims
    g = cfb200.Grid(Nx, Ny, Nz, 5.3, 7.1)
    gpu = cfb200.CouetteFlow(g, 1 / 300, 0.01, form=form)
    ref = O.couette(Nx, Ny, Nz, 5.3, 7.1, 1 / 300, 0.01, form=form)
    U, P = ref.random_state(seed=7, amp=0.2)
    gpu.set_state(U, P)
    gpu.advance(0.0, 2)
    ref.step(U, P, 2)
    Ug, Pg = gpu.get_state()
    assert rel(Ug, U) <= 1e-12
    assert rel(Pg, P) <= 1e-9
    gpu.close()


# The column kernels are compiled per Chebyshev length (P = 32, 48, 64, 96,
# 128, 192, 256, 384) and the x-pass per padded length; these grids run the
# instantiations that the timed workloads use: P = 256 (384x257x384), P = 128
# (128x129x128), P = 48 (the 48x49x48 ensemble members), and P = 256 together
# with the 576-point in-place x-pass and with the 576-point z kernels.
@pytest.mark.parametrize("form", ["rotational", "convective", "divergence"])
@pytest.mark.parametrize("dims", [(8, 257, 6), (16, 129, 12), (12, 49, 10), (384, 257, 4), (4, 257, 384)])
def test_timed_lengths_all_forms(dims, form):
    Nx, Ny, Nz = dims
    g = cfb200.Grid(Nx, Ny, Nz, 2 * np.pi, np.pi)
    nu = (2 / 3) / 10900
    gpu = cfb200.PoiseuilleFlow(g, nu, 0.002, bulkvelocity=(2 / 3, 0.0), form=form)
    ref = O.poiseuille(Nx, Ny, Nz, 2 * np.pi, np.pi, nu, 0.002, bulkvelocity=(2 / 3, 0.0), form=form)
    U, P = ref.random_state(seed=31, amp=0.1, shape=1, rho=0.8)
    gpu.set_state(U, P)
    _, gg = gpu.advance(0.0, 3)
    go = ref.step(U, P, 3)
    Ug, Pg = gpu.get_state()
    assert rel(Ug, U) <= 1e-12
    # The stage pressure's tau-corrected top modes carry the amplified
    # rounding of v (see the header); at Ny = 257 and nu = 6e-5 the reference's
    # own CPU/GPU bound (rtol 1e-8, test/cuda/runtests.jl:170) applies to the
    # modified pressure.  The ordinary pressure of the convective and
    # divergence forms lacks the |u|^2/2 that dominates the modified one, so
    # the same absolute rounding is ~30x larger relative to it (measured
    # 1.4e-8 .. 1.2e-7).  It never reaches the velocity, held at 1e-12 above.
    assert rel(Pg, P) <= (1e-8 if form == "rotational" else 3e-7)
    assert abs(gg[0] - go[0]) <= 1e-13 + 1e-9 * abs(go[0])
    gpu.close()


def test_c2_poiseuille_flux_20_steps():
    # 128x129x128 constant-flux Poiseuille, Re_bulk = 2800, Lx = 4 pi,
    # Lz = 4 pi / 3, dt = 0.005, amplitude 0.2 with the k^-2 x 0.7^n spectrum:
    # velocity, energy, dissipation, wall shear and divergence against the oracle
    nu = (2 / 3) / 2800
    gpu, ref = pair(128, 129, 128, 4 * np.pi, 4 * np.pi / 3, nu, 0.005, profile="poiseuille",
                    bulkvelocity=(2 / 3, 0.0))
    U, P = ref.random_state(seed=2, amp=0.2, shape=1, rho=0.7)
    gpu.set_state(U, P)
    t, gg = gpu.advance(0.0, 20)
    go = ref.step(U, P, 20)
    Ug, Pg = gpu.get_state()
    assert abs(t - 0.1) < 1e-12
    assert rel(Ug, U) <= 1e-11
    assert rel(Pg, P) <= 1e-8
    assert abs(gg[0] - go[0]) <= 1e-13 + 1e-9 * abs(go[0])
    dg, do = gpu.diagnostics(), ref.diagnostics(U)
    assert abs(dg[0] - do[0]) <= 1e-11 * abs(do[0])  # kinetic energy
    assert abs(dg[1] - do[1]) <= 1e-11 * abs(do[1])  # dissipation
    assert dg[2] < 1e-8  # divergence
    for i in (3, 4):  # wall shear of the mean mode
        assert abs(dg[i] - do[i]) <= 1e-11 * max(1e-3, abs(do[i]))
    gpu.close()
