"""Physics validations pinning the oracle to the reference's recorded outputs.

The golden values come from the reference's own validation runs
(validation/results/{decay,ts_convergence,ts_history}.csv, copied into
tests/golden/validation_golden.json by tests/golden/make_golden.py).  The
reference ran those cases with its convective form; this oracle restates the
rotational form, whose velocity evolution is the same discrete problem up to
the gradient absorbed in the modified pressure and the y-aliasing of that
gradient, so the recorded field errors and energy ratios are matched to many
digits (tolerances stated per test).
"""
import json
import os

import numpy as np
import pytest
import scipy.linalg

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "validation_golden.json")))


def cc_weights(Ny):
    j = np.arange(Ny)
    C = np.cos(np.pi * np.outer(j, j) / (Ny - 1))
    moments = np.array([2 / (1 - n * n) if n % 2 == 0 else 0.0 for n in range(Ny)])
    return np.linalg.solve(C.T, moments)


@pytest.mark.parametrize("flow,profile,grad", [("Poiseuille", lambda y: 1 - y * y, -2 / 100), ("Couette", lambda y: y, 0.0)])
@pytest.mark.parametrize("n", [1, 3])
def test_viscous_decay(flow, profile, grad, n):
    # validation/viscous_decay.jl:5-87
    Re, A, T = 100.0, 0.1, 4.0
    nu = 1 / Re
    alpha = n * np.pi / 2
    mu = nu * (alpha**2 + 1)
    gold = {(r["dt"], r["t"]): r for r in GOLD["decay"] if r["flow"] == flow and r["n"] == n}
    errors = []
    for dt in (0.5, 0.25, 0.125):
        pb = O.OracleProblem(5, 33, 8, 2 * np.pi, 2 * np.pi, nu, dt, profile,
                             constraint=("pressuregradient", (grad, 0.0)))
        w = cc_weights(33)
        energy = lambda u: np.sum(w * np.sum(u * u, axis=(1, 2))) / (4 * pb.Nxp * pb.Nzp)
        init = pb.sample(lambda x, y, z: A * np.sin(alpha * (y + 1)) * np.cos(z) + 0 * x)
        E0 = energy(init)
        assert abs(E0 / (A * A / 8) - 1) < 1e-12
        U = pb.zeros(3)
        U[0] = pb.fft(init)
        P = pb.zeros()
        steps = int(round(T / 2 / dt))
        for t in (T / 2, T):
            pb.step(U, P, steps)
            u = pb.ifft(U[0])
            expected = init * np.exp(-mu * t)
            err = np.max(np.abs(u - expected)) / np.max(np.abs(expected))
            ratio = energy(u) / E0
            assert err < 1e-3
            assert abs(ratio / np.exp(-2 * mu * t) - 1) < 2e-3
            # reference-recorded values (same discretisation in time and y)
            g = gold[(dt, t)]
            assert abs(ratio - g["energy_ratio"]) < 1e-10, (ratio, g["energy_ratio"])
            assert abs(err - g["error"]) < 1e-9 * max(1.0, g["error"]) + 1e-11
            assert np.max(np.abs(U[1])) < 1e-11 and np.max(np.abs(U[2])) < 1e-11
            assert np.max(np.abs(U[0][:, 0, 0])) < 1e-10
            if t == T:
                errors.append(err)
    assert 3.5 < errors[0] / errors[1] < 4.5
    assert 3.5 < errors[1] / errors[2] < 4.5


def poiseuille_ts_mode(Ny):
    """Orr-Sommerfeld mode alpha=1, Re=8000 (validation/tollmien_schlichting.jl:13-66)."""
    S = np.zeros((Ny, Ny - 4))
    for k in range(Ny - 4):
        S[k, k] = 1
        S[k + 2, k] = -2 * (k + 2) / (k + 3)
        S[k + 4, k] = (k + 1) / (k + 3)
    D = np.zeros((Ny, Ny))
    for n in range(1, Ny):
        for k in range(n - 1, -1, -2):
            D[k, n] = n if k == 0 else 2 * n
    y = np.cos(np.pi * (np.arange(2 * Ny) + 0.5) / (2 * Ny))
    C = np.cos(np.outer(np.arccos(y), np.arange(Ny)))
    I = np.eye(Ny)
    V, L = C @ S, C @ (D @ D - I) @ S
    DD = D @ D - I
    A = V.T @ (C @ DD @ DD @ S / 8000 - 1j * (1 - y**2)[:, None] * L - 2j * V)
    B = V.T @ L
    vals, vecs = scipy.linalg.eig(A.astype(complex), B.astype(complex))
    target = 0.002664410371 - 0.2470750602j
    idx = np.argmin(np.abs(vals - target))
    s, c = vals[idx], vecs[:, idx]
    v = S @ c
    u = 1j * D @ v
    scale = np.max(np.sqrt(np.abs(C @ u) ** 2 + np.abs(C @ v) ** 2))
    u, v = u / scale, v / scale
    Y = np.zeros((Ny, Ny))
    Y[1, 0] = 1
    for n in range(1, Ny):
        Y[n - 1, n] = 0.5
        if n + 1 < Ny:
            Y[n + 1, n] = 0.5
    p = (-1j * (I - Y @ Y) @ u + 2 * Y @ v + DD @ u / 8000 - s * u) / 1j
    return s, u, v, p


@pytest.mark.slow
def test_tollmien_schlichting_wave():
    # validation/tollmien_schlichting.jl:73-158, against ts_convergence.csv and ts_history.csv
    reference = 0.002664410371 - 0.2470750602j
    s, mu_, mv, mp = poiseuille_ts_mode(81)
    assert abs(s - reference) < 5e-10
    nu, amp, T = 1 / 8000, 1e-7, 50.0
    gold_conv = {r["dt"]: r for r in GOLD["ts_convergence"]}
    gold_hist = {(r["dt"], r["t"]): r for r in GOLD["ts_history"]}
    errors = []
    for dt in (0.4, 0.2, 0.1):
        pb = O.OracleProblem(8, 81, 1, 2 * np.pi, 2 * np.pi, nu, dt, lambda y: 1 - y * y,
                             constraint=("pressuregradient", (-2 * nu, 0.0)))
        U = pb.zeros(3)
        P = pb.zeros()
        U[0][:, 0, 1] = amp / 2 * mu_
        U[1][:, 0, 1] = amp / 2 * mv
        P[:, 0, 1] = amp / 2 * mp
        init = U.copy()
        v0 = init[1][:, 0, 1]
        previous, phase = 1.0 + 0j, 0.0
        steps = int(round(10 / dt))
        for t in np.arange(10.0, T + 1e-9, 10.0):
            pb.step(U, P, steps)
            modal = np.vdot(v0, U[1][:, 0, 1]) / np.vdot(v0, v0)
            phase += np.angle(modal / previous)
            previous = modal
            g = gold_hist[(dt, float(t))]
            assert abs(abs(modal) - g["amplitude"]) < 1e-9 * g["amplitude"], (abs(modal), g["amplitude"])
            assert abs(phase - g["phase"]) < 1e-9 * abs(g["phase"])
            assert np.max(np.abs(U[2])) < 1e-13
        exact = init * np.exp(reference * T)
        err = np.sqrt(np.sum(np.abs(U - exact) ** 2) / np.sum(np.abs(exact) ** 2))
        assert err < 5e-3
        assert abs(err / gold_conv[dt]["error"] - 1) < 1e-4, (err, gold_conv[dt]["error"])
        errors.append(err)
    assert errors[0] / errors[1] > 3.5 and errors[1] / errors[2] > 3.5 and errors[-1] < 1e-5
