"""The reference's Waleffe-equilibrium validation (validation/waleffe_equilibrium.jl)
restated for the tests: the archived R400 Couette equilibria (fixtures made by
tests/golden/make_waleffe.py) placed on a DNS grid, the reference's volume
and wall diagnostics, and its run protocol.  Recorded outputs of the
reference's own run: validation/results/waleffe.csv (in
tests/golden/validation_golden.json, key "waleffe").
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NU = 1 / 400
LX, LZ = 2 * np.pi / 1.14, 2 * np.pi / 2.5
GOLD = json.load(open(os.path.join(HERE, "golden", "validation_golden.json")))["waleffe"]


def perturbation(branch, Ny, N):
    """waleffe_equilibrium(branch, Ny, N) (waleffe_equilibrium.jl:13-53): the
    archived spectrum copied onto the (Ny, N, N) grid, storage (3, Ny, Nz, Nxh),
    minus the laminar y = T_1 in the streamwise mean."""
    spec = np.load(os.path.join(HERE, "golden", f"waleffe_{branch}.npz"))["spec"]
    U = np.zeros((3, Ny, N, N // 2 + 1), np.complex128)
    for l in range(-15, 16):
        U[:, :34, l % N, :16] = spec[:, :, l + 15, :]
    U[0, 1, 0, 0] -= 1.0
    return U


def weights(Ny):
    """Unweighted Chebyshev (Clenshaw-Curtis) quadrature at the Lobatto nodes
    (waleffe_equilibrium.jl:63-64)."""
    C = np.cos(np.pi * np.outer(np.arange(Ny), np.arange(Ny)) / (Ny - 1))
    m = np.array([2 / (1 - j * j) if j % 2 == 0 else 0.0 for j in range(Ny)])
    return np.linalg.solve(C.T, m)


def diagnostics(ref, U):
    """equilibrium_diagnostics(U) (waleffe_equilibrium.jl:60-83) with the
    oracle's transforms and derivatives: energy of U, dissipation and wall
    power input of the total flow (base Couette du/dy = 1 added)."""
    Ny, Nzp, Nxp = ref.physshape
    w = weights(Ny)

    def average(a):  # a: (Ny, Nzp, Nxp)
        return float(np.sum(w * a.sum(axis=(1, 2)))) / (2 * Nxp * Nzp)

    energy = sum(average(ref.ifft(U[i]) ** 2) for i in range(3)) / 2
    diss, inp = 0.0, 0.0
    for i in range(3):
        for j, op in enumerate(("ddx1", "ddx2", "ddx3")):
            d = ref.ifft(ref.operator(op, U[i]))
            if i == 0 and j == 1:
                d = d + 1.0
                inp = (d[0].sum() + d[-1].sum()) / (800 * Nxp * Nzp)
            diss += average(d ** 2) / 400
    return energy, diss, inp


def golden(branch, Ny, N, dt, t):
    for r in GOLD:
        if (r["branch"], int(r["Ny"]), int(r["N"]), r["dt"], r["t"]) == (branch, Ny, N, dt, t):
            return r
    raise KeyError((branch, Ny, N, dt, t))
