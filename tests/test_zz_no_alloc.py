"""GPU: cf_nonlinear_noalloc (fixed device scratch, no allocation) against
cf_nonlinear on the same handle and input, two calls of each in a row.

Both run the same kernels on the same data, so the results are bit-identical.
This file is collected last so the check also runs after every other GPU test
of the session has used the library.
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LX, LZ = 2 * np.pi / 1.14, 2 * np.pi / 2.5


def test_noalloc_matches_nonlinear_twice():
    g = cfb200.Grid(32, 33, 32, LX, LZ)
    pb = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    ref = O.couette(32, 33, 32, LX, LZ, 1 / 400, 0.01)
    U = ref.synth(seed=11, amp=0.1)
    for _ in range(2):
        N_alloc = pb.nonlinear(U)
        N_fixed = pb.nonlinear_noalloc(U)
        assert np.array_equal(N_fixed, N_alloc)
    N_ref = ref.nonlinear(U)
    assert np.max(np.abs(N_fixed - N_ref)) <= 1e-13 * max(1.0, np.max(np.abs(N_ref)))
    pb.close()


def test_noalloc_rejects_grids_over_the_scratch_limit():
    # 128x129x128: 3 * Nr * 16 bytes = 51.5 MB > 16 MiB
    pb = cfb200.CouetteFlow(cfb200.Grid(128, 129, 128, LX, LZ), 1 / 400, 0.01)
    U = np.zeros((3, 129, 128, 65), dtype=np.complex128)
    with pytest.raises(cfb200.CFError):
        pb.nonlinear_noalloc(U)
    pb.close()
