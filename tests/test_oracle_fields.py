"""Known-answer tests pinning the oracle's transforms, operators, nonlinear term,
projection, pressure and diagnostics.

Ported from the reference's test/test_ffts.jl, test/test_operators.jl,
test/test_nonlinear.jl, test/test_projection.jl and test/test_postprocessing.jl.
"""
import numpy as np
import pytest

from helpers import bulkmean
from oracle import oracle as O


def make(Nx, Ny, Nz, Lx, Lz, profile=lambda y: 0.0 * y, nu=0.01, dt=0.01, **kw):
    return O.OracleProblem(Nx, Ny, Nz, Lx, Lz, nu, dt, profile, **kw)


@pytest.mark.parametrize("NxNz", [(6, 8), (7, 9), (6, 9), (7, 8)])
def test_analytic_transforms(NxNz):
    # test_ffts.jl:1-45
    Nx, Nz = NxNz
    pb = make(Nx, 9, Nz, 5.3, 7.1)
    a, b = 2 * np.pi / 5.3, 2 * np.pi / 7.1
    u = pb.sample(lambda x, y, z: 2 + 0.3 * y + (2 * y**2 - 1) * np.cos(a * x) * np.sin(b * z))
    U = pb.fft(u)
    exact = pb.zeros()
    exact[0, 0, 0], exact[1, 0, 0] = 2, 0.3
    exact[2, 1, 1], exact[2, -1, 1] = -0.25j, 0.25j
    assert np.max(np.abs(U - exact)) < 2e-13
    assert np.max(np.abs(pb.ifft(U) - u)) < 2e-13
    U3 = pb.fft(np.full(pb.physshape, 3.0))
    exact[:] = 0
    exact[0, 0, 0] = 3
    assert np.max(np.abs(U3 - exact)) < 2e-13


def test_nyquist_filtered():
    pb = make(6, 9, 8, 2 * np.pi, 2 * np.pi)
    U = pb.spectral(lambda x, y, z: np.cos(3 * x) + np.cos(4 * z))
    assert np.max(np.abs(U)) < 2e-13


@pytest.mark.parametrize("N", [7, 8])
def test_quadratic_product_padding(N):
    # test_ffts.jl:56-73
    pb = make(N, 9, N, 2 * np.pi, 2 * np.pi)
    for f in (lambda x, y, z: np.cos(3 * x) ** 2, lambda x, y, z: np.cos(3 * z) ** 2):
        U = pb.spectral(f)
        exact = pb.zeros()
        exact[0, 0, 0] = 0.5
        assert np.max(np.abs(U - exact)) < 2e-13


@pytest.mark.parametrize("N", [7, 8])
def test_highest_chebyshev_coefficient(N):
    # test_ffts.jl:75-95
    pb = make(N, 35, N, 2 * np.pi, 2 * np.pi)
    u = pb.sample(lambda x, y, z: np.cos(34 * np.arccos(np.clip(y, -1, 1))) * np.cos(2 * x) * np.cos(2 * z))
    U = pb.fft(u)
    expected = pb.zeros()
    expected[34, 2, 2] = expected[34, -2, 2] = 0.25
    assert np.max(np.abs(U - expected)) < 2e-12
    assert np.max(np.abs(pb.ifft(U) - u)) < 2e-12


@pytest.mark.parametrize("Ny", [9, 17])
@pytest.mark.parametrize("NxNz", [(40, 42), (41, 43)])
def test_analytic_derivatives(Ny, NxNz):
    # test_operators.jl:1-95
    Nx, Nz = NxNz
    pb = make(Nx, Ny, Nz, 5.3, 7.1)
    a, b = 2 * np.pi / 5.3, 2 * np.pi / 7.1
    p = lambda y: 1 + 2 * y + 3 * y**2 + 4 * y**3
    dp = lambda y: 2 + 6 * y + 12 * y**2
    d2p = lambda y: 6 + 24 * y
    h = lambda x, z: np.exp(np.cos(a * x) + np.cos(b * z) - 2)
    f = lambda x, y, z: p(y) * h(x, z)
    fx = lambda x, y, z: -a * p(y) * np.sin(a * x) * h(x, z)
    fy = lambda x, y, z: dp(y) * h(x, z)
    fz = lambda x, y, z: -b * p(y) * np.sin(b * z) * h(x, z)
    lap = lambda x, y, z: (d2p(y) + p(y) * (a**2 * (np.sin(a * x) ** 2 - np.cos(a * x))
                                            + b**2 * (np.sin(b * z) ** 2 - np.cos(b * z)))) * h(x, z)
    U = pb.spectral(f)
    for op, exp in (("ddx1", fx), ("ddx2", fy), ("ddx3", fz)):
        out = pb.operator(op, U)
        assert np.max(np.abs(pb.ifft(out) - pb.sample(exp))) < 2e-10
        pb.operator(op, U, out=out, add=True)
        assert np.max(np.abs(pb.ifft(out) - 2 * pb.sample(exp))) < 4e-10
    out = pb.operator("laplacian", U)
    assert np.max(np.abs(pb.ifft(out) - pb.sample(lap))) < 2e-9
    V = np.stack([U, U, U])
    W = pb.curl(V)
    for comp, exp in enumerate(((fy, fz), (fz, fx), (fx, fy))):
        target = pb.sample(exp[0]) - pb.sample(exp[1])
        assert np.max(np.abs(pb.ifft(W[comp]) - target)) < 4e-10
    d = pb.div(V)
    assert np.max(np.abs(pb.ifft(d) - pb.sample(fx) - pb.sample(fy) - pb.sample(fz))) < 3e-10


def test_analytic_nonlinear_rotational():
    # test_nonlinear.jl:1-38 (rotational form): U = (y^2, 1, 0), base = y
    pb = make(5, 9, 5, 2 * np.pi, 2 * np.pi, profile=lambda y: y)
    U = np.stack([pb.spectral(lambda x, y, z: y**2 + 0 * x), pb.spectral(lambda x, y, z: 1.0 + 0 * x),
                  pb.zeros()])
    saved = U.copy()
    N = pb.nonlinear(U)
    exps = (lambda x, y, z: -(2 * y + 1) + 0 * x, lambda x, y, z: (y**2 + y) * (2 * y + 1) + 0 * x,
            lambda x, y, z: 0 * x)
    for i in range(3):
        assert np.max(np.abs(pb.ifft(N[i]) - pb.sample(exps[i]))) < 2e-11
    assert np.array_equal(U, saved)


@pytest.mark.parametrize("form", ["convective", "divergence"])
def test_analytic_nonlinear_forms(form):
    # test_nonlinear.jl:1-38 (convective and divergence forms): the total
    # velocity (y^2 + y, 1, 0) is divergence-free, so both give -(2y + 1) e_x
    pb = make(5, 9, 5, 2 * np.pi, 2 * np.pi, profile=lambda y: y, form=form)
    U = np.stack([pb.spectral(lambda x, y, z: y**2 + 0 * x), pb.spectral(lambda x, y, z: 1.0 + 0 * x),
                  pb.zeros()])
    saved = U.copy()
    for _ in range(2):  # repeated calls reuse the work arrays
        N = pb.nonlinear(U)
        assert np.max(np.abs(pb.ifft(N[0]) - pb.sample(lambda x, y, z: -(2 * y + 1) + 0 * x))) < 2e-11
        assert np.max(np.abs(pb.ifft(N[1]))) < 2e-11
        assert np.max(np.abs(pb.ifft(N[2]))) < 2e-11
    assert np.array_equal(U, saved)


def test_unknown_form_rejected():
    with pytest.raises(ValueError):
        make(5, 9, 5, 2 * np.pi, 2 * np.pi, form="skew")


def check_constraints(pb, U):
    # helpers.jl:77-87
    assert np.max(np.abs(pb.div(U))) < 2e-9
    signs = (-1.0) ** np.arange(pb.Ny)
    for i in range(3):
        assert np.max(np.abs(U[i].sum(axis=0))) < 2e-10
        assert np.max(np.abs(np.tensordot(signs, U[i], axes=(0, 0)))) < 2e-10


@pytest.mark.parametrize("NxNz", [(40, 42), (41, 43)])
def test_analytic_projection(NxNz):
    # test_projection.jl:1-55
    Nx, Nz = NxNz
    pb = make(Nx, 13, Nz, 5.3, 7.1)
    a, b = 2 * np.pi / 5.3, 2 * np.pi / 7.1
    q = lambda y: (1 - y**2) ** 2
    dq = lambda y: -4 * y + 4 * y**3
    h = lambda x, z: np.exp(np.cos(a * x) + np.cos(b * z) - 2)
    hx = lambda x, z: -a * np.sin(a * x) * h(x, z)
    hz = lambda x, z: -b * np.sin(b * z) * h(x, z)
    exact = (lambda x, y, z: dq(y) * h(x, z), lambda x, y, z: -q(y) * hx(x, z), lambda x, y, z: 0 * x)
    corr = (lambda x, y, z: q(y) * hx(x, z), lambda x, y, z: dq(y) * h(x, z), lambda x, y, z: q(y) * hz(x, z))
    U = np.stack([pb.spectral(lambda x, y, z, i=i: exact[i](x, y, z) + corr[i](x, y, z)) for i in range(3)])
    U = pb.project(U)
    for i in range(3):
        assert np.max(np.abs(pb.ifft(U[i]) - pb.sample(exact[i]))) < 2e-10
    check_constraints(pb, U)
    U2 = pb.project(U)
    assert np.max(np.abs(U2 - U)) < 2e-11


def test_projection_bulk_constraint():
    pb = make(5, 9, 5, 2 * np.pi, 2 * np.pi, constraint=("bulkvelocity", (0.2, -0.1)))
    U = pb.project(pb.zeros(3))
    assert abs(bulkmean(U[0][:, 0, 0]).real - 0.2) < 2e-12
    assert abs(bulkmean(U[2][:, 0, 0]).real + 0.1) < 2e-12
    check_constraints(pb, U)


def test_laminar_couette_modified_pressure():
    # test_projection.jl:77-87
    pb = make(5, 9, 5, 2 * np.pi, 2 * np.pi, profile=lambda y: y)
    U = pb.project(pb.zeros(3))
    P = pb.pressure(U)
    assert np.max(np.abs(pb.ifft(P) - pb.sample(lambda x, y, z: y**2 / 2 - 1 / 6 + 0 * x))) < 2e-10


@pytest.mark.parametrize("form", ["convective", "divergence"])
def test_laminar_couette_physical_pressure(form):
    # pressure.jl:86-92: for the convective and divergence forms P is the
    # ordinary pressure, which is uniform (zero in the zero-mean gauge) for
    # laminar Couette flow, where (u.grad)u = 0
    pb = make(5, 9, 5, 2 * np.pi, 2 * np.pi, profile=lambda y: y, form=form)
    U = pb.project(pb.zeros(3))
    P = pb.pressure(U)
    assert np.max(np.abs(P)) < 2e-12


def test_random_state_admissible():
    pb = make(8, 17, 8, 2 * np.pi, 2 * np.pi, profile=lambda y: y)
    U, P = pb.random_state(7, 0.1)
    U2, P2 = pb.random_state(7, 0.1)
    assert np.array_equal(U, U2) and np.array_equal(P, P2)
    assert np.max(np.abs(U)) > 0
    check_constraints(pb, U)
    # real-data round trip keeps the k = 0 conjugate pairs
    for i in range(3):
        assert np.max(np.abs(pb.fft(pb.ifft(U[i])) - U[i])) < 2e-11


def test_energy_and_dissipation():
    # test_postprocessing.jl:1-30
    nu = 0.01
    pb = make(8, 17, 8, 2 * np.pi, 2 * np.pi, nu=nu)
    U = np.stack([pb.spectral(lambda x, y, z: y + 0 * x), pb.zeros(), pb.zeros()])
    d = pb.diagnostics(U)
    assert abs(d[0] - 1 / 6) < 2e-14 and abs(d[1] - nu) < 2e-14
    assert abs(pb.dot(U, U) - 1 / 3) < 2e-14
    V = np.stack([pb.spectral(lambda x, y, z: 1 - y**2 + 0 * x), pb.zeros(), pb.zeros()])
    assert abs(pb.dot(U, V)) < 2e-14
    d = pb.diagnostics(V)
    assert abs(d[0] - 4 / 15) < 2e-14 and abs(d[1] - 4 * nu / 3) < 2e-14
    assert pb.diagnostics(pb.zeros(3))[0] == 0
