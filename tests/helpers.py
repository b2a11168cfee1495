"""Shared helpers mirroring the reference's test/helpers.jl.

`coefficients` builds Chebyshev coefficients with scipy's DCT-I, independently
of the oracle's transforms (helpers.jl:5-11); `bulkmean` integrates with
Gauss-Legendre quadrature (helpers.jl:23-32); `wallvalue` evaluates T_n(+-1).
"""
import numpy as np
import scipy.fft
import scipy.linalg


def lobatto(Ny):
    y = np.cos(np.pi * np.arange(Ny) / (Ny - 1))
    y[np.arange(Ny) * 2 == Ny - 1] = 0.0
    return y


def coefficients(f, Ny):
    P = Ny - 1
    vals = np.array([f(v) for v in lobatto(Ny)], dtype=complex)
    a = (scipy.fft.dct(vals.real, type=1) + 1j * scipy.fft.dct(vals.imag, type=1)) / P
    a[0] /= 2
    a[-1] /= 2
    return a


def wallvalue(a, side):
    n = np.arange(len(a))
    return np.sum(a * (1.0 if side == "right" else (-1.0) ** n))


def derivative(a):
    """Chebyshev derivative by the descending recurrence (operators.jl:38-61)."""
    a = np.asarray(a)
    P = len(a) - 1
    b = np.zeros_like(a)
    if P >= 1:
        b[P - 1] = 2 * P * a[P]
    for n in range(P - 2, -1, -1):
        b[n] = b[n + 2] + 2 * (n + 1) * a[n + 1]
    b[0] *= 0.5
    return b


def wall_diff(a, side):
    n = np.arange(len(a))
    w = n.astype(float) ** 2
    if side == "left":
        w = w * (-1.0) ** (n + 1)
    return np.sum(w * a)


def bulkmean(a):
    N = len(a)
    off = np.array([n / np.sqrt(4.0 * n * n - 1) for n in range(1, N)])
    nodes, vecs = scipy.linalg.eigh_tridiagonal(np.zeros(N), off)
    C = np.cos(np.outer(np.arccos(np.clip(nodes, -1, 1)), np.arange(N)))
    return np.sum(vecs[0, :] ** 2 * (C @ a))


def check_stokes(k, l, lam_full, nu, u, v, w, p, Rx, Ry, Rz):
    """Residual checks of test_helmoltz.jl:122-151 for one mode; returns max errors."""
    P = len(p) - 1
    dp = derivative(p)
    div = 1j * k * u + derivative(v) + 1j * l * w
    errs = {"div": np.max(np.abs(div))}
    mom = 0.0
    walls = 0.0
    for field, src, gradp in ((u, Rx, 1j * k * p), (v, Ry, dp), (w, Rz, 1j * l * p)):
        res = lam_full * field - nu * derivative(derivative(field)) + gradp - src
        mom = max(mom, np.max(np.abs(res[: P - 1])))
        walls = max(walls, abs(wallvalue(field, "left")), abs(wallvalue(field, "right")))
    errs["momentum"] = mom
    errs["walls"] = walls
    errs["dv_walls"] = max(abs(wall_diff(v, "left")), abs(wall_diff(v, "right")))
    return errs
