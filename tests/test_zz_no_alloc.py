"""GPU: cf_nonlinear_noalloc, the nonlinear term staged in the library's fixed
device scratch, for callers that must not allocate device memory while they
run (e.g. a host framework whose memory pool is frozen or accounted).

It is checked against cf_nonlinear on the same handle and input, two calls of
each in a row (the same kernels on the same data: bit-identical), and
against the oracle.  On a fresh handle the call must leave the handle's own
device memory and the device's free memory unchanged.  This file is
collected last, so the check also runs after every other GPU test of the
session has used the library, and it passes alone in a fresh process.
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LX, LZ = 2 * np.pi / 1.14, 2 * np.pi / 2.5


def _free_bytes():
    torch = pytest.importorskip("torch")
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_noalloc_allocates_nothing_on_a_fresh_handle():
    g = cfb200.Grid(32, 33, 32, LX, LZ)
    ref = O.couette(32, 33, 32, LX, LZ, 1 / 400, 0.01)
    U = ref.synth(seed=11, amp=0.1)
    # a first handle loads every kernel the call uses
    warm = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    warm.nonlinear_noalloc(U)
    pb = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    held = pb.device_bytes()
    _free_bytes()  # torch's own first use of the device happens here
    free0 = _free_bytes()
    N = pb.nonlinear_noalloc(U)
    free1 = _free_bytes()
    assert pb.device_bytes() == held
    assert free1 == free0
    N_ref = ref.nonlinear(U)
    assert np.max(np.abs(N - N_ref)) <= 1e-13 * max(1.0, np.max(np.abs(N_ref)))
    # cf_nonlinear allocates its staging on first use: the counter sees it
    pb.nonlinear(U)
    assert pb.device_bytes() > held
    warm.close()
    pb.close()


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
    with pytest.raises(cfb200.CFError) as e:
        pb.nonlinear_noalloc(U)
    assert e.value.code == cfb200.CF_E_ARG
    pb.close()
