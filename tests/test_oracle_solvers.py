"""Known-answer tests pinning the oracle's solvers.

Ported from the reference's test/test_helmoltz.jl, test/test_batchedinfluence.jl
and test/test_stokes.jl (same manufactured solutions, same tolerances).  Every
Helmholtz case runs with both oracle Helmholtz paths (dense LU of the explicit
tau system and the quasi-tridiagonal elimination).
"""
import numpy as np
import pytest

from helpers import bulkmean, check_stokes, coefficients, derivative, wallvalue
from oracle import oracle as O


@pytest.fixture(params=["dense", "quasitri"])
def method(request):
    O.set_helmholtz_method(request.param)
    yield request.param
    O.set_helmholtz_method("auto", 65)


def test_helmholtz_analytic_cubic(method):
    # test_helmoltz.jl:1-29
    for Ny in (8, 9, 17):
        exact = lambda y: 0.7 + 0.3 * y - 0.2 * y**2 + 0.1 * y**3
        for nu, lam in ((0.1, 0.0), (0.03, 2.5)):
            for amp in (1.0, -0.4):
                forcing = lambda y: amp * (nu * (-0.4 + 0.6 * y) - lam * exact(y))
                rhs = coefficients(forcing, Ny).real
                expected = coefficients(lambda y: amp * exact(y), Ny).real
                out = O.helmholtz(rhs, nu, lam, amp * exact(1), amp * exact(-1))
                assert np.max(np.abs(out - expected)) < 2e-12
                assert abs(wallvalue(out, "right") - amp * exact(1)) < 2e-12
                assert abs(wallvalue(out, "left") - amp * exact(-1)) < 2e-12


def test_helmholtz_paths_agree_large_shift():
    # dense LU vs quasi-tridiagonal at the shifts and sizes of the benchmark grids
    rng = np.random.default_rng(3)
    for Ny in (33, 65, 129, 257):
        f = rng.standard_normal(Ny) / (1 + np.arange(Ny)) ** 2
        for th0, th1 in ((1.0, 0.25), (1.0, 1e4), (1 / 16350, 4000 + 1e3 / 16350), (1.0, 0.0)):
            O.set_helmholtz_method("dense")
            a = O.helmholtz(f, th0, th1, 0.3, -0.2)
            O.set_helmholtz_method("quasitri")
            b = O.helmholtz(f, th0, th1, 0.3, -0.2)
            O.set_helmholtz_method("auto", 65)
            assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(a)))


def test_neumann_paths_agree():
    rng = np.random.default_rng(4)
    for Ny in (9, 33, 129):
        f = rng.standard_normal(Ny) / (1 + np.arange(Ny)) ** 2
        for kap2 in (0.25, 3.0, 900.0):
            O.set_helmholtz_method("dense")
            a = O.helmholtz(f, 1.0, kap2, 0.3, -0.7, neumann=True)
            O.set_helmholtz_method("quasitri")
            b = O.helmholtz(f, 1.0, kap2, 0.3, -0.7, neumann=True)
            O.set_helmholtz_method("auto", 65)
            assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, np.max(np.abs(a)))
            # wall derivative data and retained tau rows
            n = np.arange(Ny)
            assert abs(np.sum(n**2 * a) - 0.3) < 1e-10
            assert abs(np.sum((-1.0) ** (n + 1) * n**2 * a) + 0.7) < 1e-10
            res = derivative(derivative(a)) - kap2 * a - f
            assert np.max(np.abs(res[: Ny - 2])) < 1e-9 * max(1, kap2)


MODES = ((1.25, 0.0), (0.0, -2.0), (1.25, -1.75), (1.25, 1.75))


@pytest.mark.parametrize("batched", [False, True])
def test_complex_primitive_variable_mode(method, batched):
    # test_helmoltz.jl:153-216 (manufactured divergence-free solution)
    for Ny in (9, 17, 33):
        for k, l in MODES:
            nu, lam = 0.03, 2.5
            kap2 = k * k + l * l
            shift = lam + nu * kap2
            c = 0.7 + 0.2j
            cq = 0.15 - 0.1j
            cp = 0.4 - 0.3j
            vfun = lambda y: c * (1 - y**2) ** 2 * (1 + 0.2 * y)
            dvfun = lambda y: c * (-4 * y + 4 * y**3 + 0.2 * (1 - 6 * y**2 + 5 * y**4))
            d2vfun = lambda y: c * (-4 + 12 * y**2 + 0.2 * (-12 * y + 20 * y**3))
            d3vfun = lambda y: c * (24 * y + 0.2 * (-12 + 60 * y**2))
            qfun = lambda y: cq * (1 - y**2) * (1 + 0.3 * y)
            d2qfun = lambda y: cq * (-2 - 1.8 * y)
            ufun = lambda y: 1j * k / kap2 * dvfun(y) + l * qfun(y)
            wfun = lambda y: 1j * l / kap2 * dvfun(y) - k * qfun(y)
            pfun = lambda y: cp * (1 + y + 0.2 * y**3)
            dpfun = lambda y: cp * (1 + 0.6 * y**2)
            Rx = coefficients(lambda y: shift * ufun(y) - nu * (1j * k / kap2 * d3vfun(y) + l * d2qfun(y))
                              + 1j * k * pfun(y), Ny)
            Ry = coefficients(lambda y: shift * vfun(y) - nu * d2vfun(y) + dpfun(y), Ny)
            Rz = coefficients(lambda y: shift * wfun(y) - nu * (1j * l / kap2 * d3vfun(y) - k * d2qfun(y))
                              + 1j * l * pfun(y), Ny)
            u, v, w, p = O.influence_solve(Ny, k, l, nu, lam, Rx, Ry, Rz, batched=batched)
            for field, exact in zip((u, v, w, p), (ufun, vfun, wfun, pfun)):
                assert np.max(np.abs(field - coefficients(exact, Ny))) < 2e-10
            e = check_stokes(k, l, shift, nu, u, v, w, p, Rx, Ry, Rz)
            assert e["div"] < 2e-10 and e["momentum"] < 2e-10
            assert e["walls"] < 2e-11 and e["dv_walls"] < 2e-11


def test_high_degree_forcing_tau(method):
    # test_helmoltz.jl:218-230 and the low-degree regression :367-384
    Ny = 17
    n = np.arange(Ny)
    R = [(np.sin((j + 1) * (n + 1)) + 1j * np.cos((j + 2) * (n + 1))) / (n + 1) ** 2 for j in (1, 2, 3)]
    u, v, w, p = O.influence_solve(Ny, 1.25, -1.75, 0.03, 2.5, *R)
    e = check_stokes(1.25, -1.75, 2.5 + 0.03 * (1.25**2 + 1.75**2), 0.03, u, v, w, p, *R)
    assert e["div"] < 2e-10 and e["momentum"] < 2e-10 and e["walls"] < 2e-11 and e["dv_walls"] < 2e-11
    for Ny in (5, 9):
        for lam in (0.0, 2.5):
            n = np.arange(Ny)
            R = [(np.sin(j + n) + 1j * np.cos(2 * j + n)) / (n + 1) for j in (1, 2, 3)]
            u, v, w, p = O.influence_solve(Ny, 2.0, -2.0, 1.0, lam, *R)
            e = check_stokes(2.0, -2.0, lam + 8.0, 1.0, u, v, w, p, *R)
            assert e["div"] < 2e-10 and e["momentum"] < 2e-10 and e["walls"] < 2e-11 and e["dv_walls"] < 2e-11


def test_influence_rejects_bad_sizes():
    with pytest.raises(ValueError):
        O.influence_solve(10, 1, 1, 0.1, 2, np.zeros(10), np.zeros(10), np.zeros(10))
    with pytest.raises(ValueError):
        O.influence_solve(9, 0, 0, 0.1, 2, np.zeros(9), np.zeros(9), np.zeros(9))


def test_mean_mode(method):
    # test_helmoltz.jl:151-277
    for Ny in (9, 16, 33):
        for lam in (0.0, 2.5):
            nu = 0.03
            grads, means = (-0.7, 0.3), (0.48, -0.2)
            ufun = lambda y: (1 - y**2) * (0.7 + 0.2 * y + 0.1 * y**2)
            wfun = lambda y: (1 - y**2) * (-0.3 + 0.15 * y)
            pfun = lambda y: y + 0.4 * (y**2 - 1 / 3) + 0.2 * y**3
            Rx = coefficients(lambda y: lam * ufun(y) + nu * (1.2 + 1.2 * y + 1.2 * y**2) + grads[0], Ny)
            Ry = coefficients(lambda y: 1 + 0.8 * y + 0.6 * y**2, Ny)
            Rz = coefficients(lambda y: lam * wfun(y) - nu * (0.6 - 0.9 * y) + grads[1], Ny)
            for fixed in (False, True):
                kw = {"bulkvelocity": means} if fixed else {"pressuregradient": grads}
                (u, v, w, p), actual = O.mean_solve(Ny, nu, lam, Rx, Ry, Rz, **kw)
                assert all(abs(a - b) < 2e-11 for a, b in zip(actual, grads))
                for field, exact in zip((u, w, p), (ufun, wfun, pfun)):
                    assert np.max(np.abs(field - coefficients(exact, Ny))) < 2e-10
                assert np.all(v == 0)
                assert abs(bulkmean(p)) < 2e-12
                assert abs(bulkmean(u) - means[0]) < 2e-11
                assert abs(bulkmean(w) - means[1]) < 2e-11
                assert np.max(np.abs(derivative(p) - Ry)) < 2e-10
                for field, rhs, g in ((u, Rx, actual[0]), (w, Rz, actual[1])):
                    res = lam * field - nu * derivative(derivative(field)) - rhs
                    res[0] += g
                    assert np.max(np.abs(res[: Ny - 2])) < 2e-10
                    assert abs(wallvalue(field, "right")) < 2e-11 and abs(wallvalue(field, "left")) < 2e-11
    # complex high-degree forcing and pressure truncation at the last coefficient
    Ny, nu, lam = 17, 0.03, 2.5
    n = np.arange(Ny)
    zero = [np.zeros(Ny, complex)] * 3
    (u, v, w, p), g = O.mean_solve(Ny, nu, lam, *zero)
    assert g == (0.0, 0.0) and not np.any(u) and not np.any(p)
    R = [(np.sin(i * (n + 1)) + 1j * np.cos((i + 1) * (n + 1))) / (n + 1) ** 2 for i in (1, 2, 3)]
    (u, v, w, p), g = O.mean_solve(Ny, nu, lam, *R, bulkvelocity=(0.2, -0.1))
    assert abs(bulkmean(u).real - 0.2) < 2e-12 and abs(bulkmean(w).real + 0.1) < 2e-12
    assert abs(bulkmean(p)) < 2e-12
    normal = derivative(p) - R[1]
    assert np.max(np.abs(normal[: Ny - 1])) < 2e-11
    assert abs(normal[-1] + R[1][-1]) < 2e-12
    # golden value: test_helmoltz.jl:273-275
    small = [np.zeros(5, complex)] * 3
    (u, v, w, p), g = O.mean_solve(5, nu, 0.0, *small, bulkvelocity=(2 / 3, 0))
    assert abs(g[0] + 2 * nu) < 2e-12 and abs(g[1]) < 2e-12
    assert np.allclose(u, [0.5, 0, -0.5, 0, 0], atol=1e-14)


def test_batched_versus_scalar(method):
    # test_batchedinfluence.jl:1-28
    rng = np.random.default_rng(0)
    for Ny in (5, 9, 17, 33):
        for lam in (0.0, 3.0):
            ks, ls = [1.0, 0.0, 1.25, 2.0], [0.0, -2.0, 1.75, -0.5]
            nu = 0.03
            for k, l in zip(ks, ls):
                R = [rng.standard_normal(Ny) + 1j * rng.standard_normal(Ny) for _ in range(3)]
                a = O.influence_solve(Ny, k, l, nu, lam, *R, batched=True)
                b = O.influence_solve(Ny, k, l, nu, lam, *R, batched=False)
                for x, y in zip(a, b):
                    assert np.allclose(x, y, rtol=2e-11, atol=2e-11)
                e = check_stokes(k, l, lam + nu * (k * k + l * l), nu, *a, *R)
                assert e["div"] < 2e-10 and e["momentum"] < 2e-10 and e["walls"] < 2e-11


@pytest.mark.parametrize("NxNz", [(6, 6), (5, 5), (6, 5), (5, 6), (1, 5), (5, 1), (1, 1), (2, 2)])
@pytest.mark.parametrize("profile", ["poiseuille", "couette"])
def test_stokes_assembly(NxNz, profile):
    # test_stokes.jl:1-131
    Nx, Nz = NxNz
    Ny, nu, lam = 9, 0.03, 2.5
    Lx, Lz = 5.3, 7.1
    grads = (-0.4, 0.15)
    prof, base_mean = ((lambda y: 1 - y * y), 2 / 3) if profile == "poiseuille" else ((lambda y: y), 0.0)
    pb = O.OracleProblem(Nx, Ny, Nz, Lx, Lz, 0.1, 0.01, prof)
    Nxh = Nx // 2 + 1
    R = pb.zeros(3)
    exact = pb.zeros(3)
    exactP = pb.zeros()
    zmodes = list(range(0, (Nz - 1) // 2 + 1)) + list(range(-(Nz // 2), 0))
    for iz, mz in enumerate(zmodes):
        for ix, mx in enumerate(range(0, Nx // 2 + 1)):
            if (Nx % 2 == 0 and mx == Nx // 2) or (Nz % 2 == 0 and mz == -(Nz // 2)):
                R[:, :, iz, ix] = 7 + 3j
                continue
            k, l = 2 * np.pi * mx / Lx, 2 * np.pi * mz / Lz
            if mx == 0 and mz == 0:
                uf, vf, wf = (lambda y: 0.2 * (1 - y**2)), (lambda y: 0.0 * y), (lambda y: -0.1 * (1 - y**2))
                d2uf, d2vf, d2wf = (lambda y: -0.4 + 0 * y), (lambda y: 0 * y), (lambda y: 0.2 + 0 * y)
                pf, dpf = (lambda y: 0.3 * y + 0.2 * (y**2 - 1 / 3)), (lambda y: 0.3 + 0.4 * y)
                mean = True
            else:
                k2 = k * k + l * l
                a, b = 0.1 / (1 + mx**2 + mz**2), 0.05j
                vf = lambda y, a=a: a * (1 - y**2) ** 2
                dvf = lambda y, a=a: a * (-4 * y + 4 * y**3)
                d2vf = lambda y, a=a: a * (-4 + 12 * y**2)
                d3vf = lambda y, a=a: 24 * a * y
                uf = lambda y, k=k, l=l, k2=k2, b=b, dvf=dvf: 1j * k / k2 * dvf(y) + l * b * (1 - y**2)
                wf = lambda y, k=k, l=l, k2=k2, b=b, dvf=dvf: 1j * l / k2 * dvf(y) - k * b * (1 - y**2)
                d2uf = lambda y, k=k, l=l, k2=k2, b=b, d3vf=d3vf: 1j * k / k2 * d3vf(y) - 2 * l * b
                d2wf = lambda y, k=k, l=l, k2=k2, b=b, d3vf=d3vf: 1j * l / k2 * d3vf(y) + 2 * k * b
                pf, dpf = (lambda y: 0.3 + 0.2 * y + 0.1 * y**2), (lambda y: 0.2 + 0.2 * y)
                mean = False
            shift = lam + nu * (k * k + l * l)
            rx = lambda y, uf=uf, d2uf=d2uf, k=k, mean=mean, shift=shift, pf=pf: \
                shift * uf(y) - nu * d2uf(y) + (grads[0] if mean else 1j * k * pf(y))
            ry = lambda y, vf=vf, d2vf=d2vf, dpf=dpf, shift=shift: shift * vf(y) - nu * d2vf(y) + dpf(y)
            rz = lambda y, wf=wf, d2wf=d2wf, l=l, mean=mean, shift=shift, pf=pf: \
                shift * wf(y) - nu * d2wf(y) + (grads[1] if mean else 1j * l * pf(y))
            for dst, f in ((exact[0], uf), (exact[1], vf), (exact[2], wf), (exactP, pf)):
                dst[:, iz, ix] = coefficients(f, Ny)
            for i, f in enumerate((rx, ry, rz)):
                R[i][:, iz, ix] = coefficients(f, Ny)
    saved = R.copy()
    for fixed in (False, True):
        if fixed:
            U, P, g = pb.stokes(R, nu=nu, lam=lam, bulkvelocity=(base_mean + 0.2 * 2 / 3, -0.1 * 2 / 3))
        else:
            U, P, g = pb.stokes(R, nu=nu, lam=lam, pressuregradient=grads)
        assert all(abs(a - b) < 2e-11 for a, b in zip(g, grads))
        for i in range(3):
            assert np.max(np.abs(U[i] - exact[i])) < 2e-10
        assert np.max(np.abs(P - exactP)) < 2e-10
        assert np.array_equal(R, saved)
        assert np.max(np.abs(pb.div(U))) < 2e-10
        assert abs(bulkmean(U[0][:, 0, 0]).real - 0.2 * 2 / 3) < 2e-11
        assert abs(bulkmean(U[2][:, 0, 0]).real + 0.1 * 2 / 3) < 2e-11
        assert abs(bulkmean(P[:, 0, 0])) < 2e-12


def test_stokes_wrapper_validation():
    with pytest.raises(ValueError):
        O.OracleProblem(5, 10, 5, 5.3, 7.1, 0.03, 0.01, lambda y: y)
    with pytest.raises(ValueError):
        O.OracleProblem(0, 9, 5, 5.3, 7.1, 0.03, 0.01, lambda y: y)
    with pytest.raises(ValueError):
        O.OracleProblem(5, 9, 5, 5.3, 7.1, 0.03, 0.0, lambda y: y)
