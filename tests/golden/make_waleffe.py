"""Extract the Waleffe R400 Couette equilibria used by the reference's
validation/waleffe_equilibrium.jl into tests/golden/waleffe_{LB,UB}.npz.

The archives (validation/data/RRC.a1.14.g2.5.R400.{LB,UB}.tar.gz of a
ChannelFlow.jl checkout; Waleffe's ECS database, Re=400, alpha=1.14,
gamma=2.5) hold the total velocity as 34 ordinary Chebyshev coefficients on a
32x32 periodic mesh (Fortran order x, z, degree) and a stats file of mean and
rms profiles at 34 Gauss points.  As the reference's importer does
(waleffe_equilibrium.jl:13-53), this script checks the Gauss points, the mean
profile and the three rms profiles against the stats file, Fourier-transforms
x and z (divided by the 1024 mesh points), checks that both Nyquist planes
vanish, and keeps the modes k = 0..15, l = -15..15, n = 0..33 that the
importer copies onto a DNS grid.  Stored: `spec` complex128 (3, 34, 31, 16)
indexed (component, n, l + 15, k), total velocity (the laminar T_1 of u is
removed by the test when it builds the perturbation state).

    python tests/golden/make_waleffe.py /path/to/ChannelFlow.jl
"""
import io
import os
import sys
import tarfile

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_waleffe.py /path/to/ChannelFlow.jl")
src = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))
for branch in ("LB", "UB"):
    name = f"RRC.a1.14.g2.5.R400.{branch}"
    with tarfile.open(os.path.join(src, "validation", "data", name + ".tar.gz")) as tar:
        member = lambda m: tar.extractfile(f"{name}.{m}").read().decode()  # noqa: E731
        lines = [ln for ln in member("stats").split("\n") if not ln.strip().startswith("%")]
        stats = np.array(" ".join(lines).split(), dtype=float).reshape(34, 5)
        y = np.cos(np.pi * (np.arange(34) + 0.5) / 34)
        C = np.cos(np.pi * np.outer(np.arange(34) + 0.5, np.arange(34)) / 34)
        assert np.max(np.abs(stats[:, 0] - y)) < 5e-9
        spec = np.zeros((3, 34, 31, 16), np.complex128)
        for i, comp in enumerate("uvw"):
            data = np.array(member(comp + ".asc").split(), dtype=float)
            assert data.size == 32 * 32 * 34
            raw = data.reshape(34, 32, 32)  # (n, z, x): Fortran (x, z, n)
            values = C @ raw.reshape(34, -1)
            means = values.sum(axis=1) / 1024
            rms = np.sqrt(((values - means[:, None]) ** 2).sum(axis=1) / 1024)
            if i == 0:
                assert np.max(np.abs(means - stats[:, 1])) < 5e-8
            assert np.max(np.abs(rms - stats[:, i + 2])) < 5e-8
            # rfft over x (last axis) and full fft over z: (n, z, kx)
            sp = np.fft.fft(np.fft.rfft(raw, axis=2), axis=1) / 1024
            assert np.max(np.abs(sp[:, :, 16])) < 1e-12 and np.max(np.abs(sp[:, 16, :])) < 1e-12
            for l in range(-15, 16):
                spec[i, :, l + 15, :] = sp[:, l % 32, :16]
    dest = os.path.join(here, f"waleffe_{branch}.npz")
    np.savez_compressed(dest, spec=spec)
    print("wrote", dest, os.path.getsize(dest), "bytes")
