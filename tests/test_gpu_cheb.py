"""GPU: Chebyshev transforms on the tensor cores (tcgen05, FP32 accumulation)
against FP64 matrix products in numpy, with both operand splits: TF32 heads
and remainders (three TF32 products) and three BF16 pieces (six BF16
products).

The transform is the mixed-precision path's replacement of the DCT-I of the
FP64 column kernel; it must reach FP32-level accuracy: max error <= 1e-5 of
the largest output (TF32 alone would give ~1e-3, one BF16 piece ~1e-2).
"""
import numpy as np
import pytest

import cfb200

pytestmark = pytest.mark.gpu


def cheb_matrix(Ny, inverse, scale=1.0):
    P = Ny - 1
    n = np.arange(Ny)
    C = np.cos(np.pi * np.outer(n, n) / P)
    if inverse:
        return C
    e = np.where((n == 0) | (n == P), 0.5, 1.0)
    w = np.where((n == 0) | (n == P), 1.0, 2.0)
    return scale * e[:, None] * C * w[None, :]


@pytest.mark.parametrize("split", ["tf32", "bf16"])
@pytest.mark.parametrize("Ny,C", [(33, 1088), (129, 1090), (257, 300), (17, 5), (385, 260)])
@pytest.mark.parametrize("inverse", [True, False])
def test_cheb_transform_matches_fp64(Ny, C, inverse, split):
    rng = np.random.default_rng(Ny * 7 + C)
    X = rng.standard_normal((2, Ny, C)).astype(np.float32)
    scale = 1.0 / (Ny - 1) if not inverse else 1.0
    Y = cfb200.cheb_transform(X, inverse, scale, split=split)
    T = cheb_matrix(Ny, inverse, scale)
    ref = np.einsum("nk,fkc->fnc", T, X.astype(np.float64))
    err = np.max(np.abs(Y - ref)) / np.max(np.abs(ref))
    assert err <= 1e-5, err


@pytest.mark.parametrize("split", ["tf32", "bf16"])
def test_cheb_round_trip(split):
    # forward (normalised by 1/P) then inverse restores nodal values
    Ny, C = 65, 640
    rng = np.random.default_rng(3)
    X = rng.standard_normal((1, Ny, C)).astype(np.float32)
    A = cfb200.cheb_transform(X, False, 1.0 / (Ny - 1), split=split)
    Xr = cfb200.cheb_transform(A, True, split=split)
    assert np.max(np.abs(Xr - X)) <= 1e-5 * np.max(np.abs(X))
