"""GPU: failure reporting without a GPU fault, and the power input.

* A NaN placed in the uploaded state (on the host) reaches the mean mode
  within one stage; the step reports CF_E_NONFINITE instead of returning
  garbage, as the reference's production driver aborts on a non-finite
  state (examples/mkm590/run.jl:225-226).  The flag is cleared once reported.
* The bounded waits of the TMA z kernels and of the tensor-core transform
  are given a limit of zero polls through the test hook: the first wait
  gives up at once, the kernel lets its own copies (or MMAs) in flight finish,
  and the call returns CF_E_CUDA; with the default limit restored the same
  handle gives the same results as before.  No wait is left spinning.
* power_input (src/postprocessing.jl:113-128): laminar values of the
  reference's tests (test/cuda/runtests.jl:145) and a random state against
  a NumPy restatement.
"""
import numpy as np
import pytest

import cfb200
from helpers import bulkmean, wall_diff, wallvalue
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LX, LZ = 2 * np.pi / 1.14, 2 * np.pi / 2.5


def test_nonfinite_state_is_reported_and_cleared():
    g = cfb200.Grid(16, 17, 16, LX, LZ)
    pb = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    st = cfb200.random_state(pb, 0.1, seed=3)
    U, P = st.U.copy(), st.P.copy()
    U[0, 3, 2, 1] = np.nan  # (n, l, k) = (3, 2, 1): not a Nyquist mode
    pb.set_state(U, P)
    with pytest.raises(cfb200.CFError) as e:
        pb.advance(0.0, 1)
    assert e.value.code == cfb200.CF_E_NONFINITE
    # the flag is reported once; a finite state steps again
    pb.set_state(st.U, st.P)
    pb.advance(0.0, 2)
    Ug, _ = pb.get_state()
    assert np.all(np.isfinite(Ug))
    U[0, 3, 2, 1] = np.inf
    pb.set_state(U, P)
    with pytest.raises(cfb200.CFError) as e:
        pb.advance(0.0, 1)
    assert e.value.code == cfb200.CF_E_NONFINITE
    pb.close()


def test_tma_wait_gives_up_and_handle_recovers():
    # Nz = 384 (padded 576): two columns per z block, the TMA z kernels
    g = cfb200.Grid(4, 17, 384, LX, LZ)
    pb = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    ref = O.couette(4, 17, 384, LX, LZ, 1 / 400, 0.01)
    U = ref.synth(seed=5, amp=0.1)
    N0 = pb.nonlinear(U)
    pb.set_wait_limit(0)
    with pytest.raises(cfb200.CFError) as e:
        pb.nonlinear(U)
    assert e.value.code == cfb200.CF_E_CUDA and "wait" in str(e.value)
    Ur, Pr = ref.random_state(seed=5, amp=0.1)
    pb.set_state(Ur, Pr)
    with pytest.raises(cfb200.CFError) as e:
        pb.advance(0.0, 1)
    assert e.value.code == cfb200.CF_E_CUDA
    pb.set_wait_limit(-1)
    assert np.array_equal(pb.nonlinear(U), N0)
    pb.set_state(Ur, Pr)
    pb.advance(0.0, 2)
    ref.step(Ur, Pr, 2)
    Ug, _ = pb.get_state()
    assert np.linalg.norm(Ug - Ur) <= 1e-12 * np.linalg.norm(Ur)
    pb.close()


def test_tensor_core_wait_gives_up_and_handle_recovers():
    # Ny = 65: the folded transform (producers, MMA thread and epilogue
    # handing stages and accumulators to each other through mbarriers); with a
    # zero poll limit the first wait that is not already complete gives up,
    # every role leaves, and the kernel waits for its MMAs before freeing TMEM
    g = cfb200.Grid(16, 65, 12, LX, LZ)
    pb = cfb200.CouetteFlow(g, 1 / 400, 0.01, precision="mixed-tc")
    st = cfb200.random_state(pb, 0.1, seed=8)
    pb.set_state(st.U, st.P)
    pb.advance(0.0, 1)
    U1, P1 = pb.get_state()
    pb.set_wait_limit(0)
    pb.set_state(st.U, st.P)
    with pytest.raises(cfb200.CFError) as e:
        pb.advance(0.0, 1)
    assert e.value.code == cfb200.CF_E_CUDA
    pb.set_wait_limit(-1)
    pb.set_state(st.U, st.P)
    pb.advance(0.0, 1)
    U2, P2 = pb.get_state()
    assert np.array_equal(U1, U2) and np.array_equal(P1, P2)
    pb.close()


def _power_input(U, nu, base, grad):
    # postprocessing.jl:113-128 on the (0,0) columns, base added to u
    tot = 0.0
    for i, gi in ((0, grad[0]), (2, grad[1])):
        a = U[i][:, 0, 0].copy()
        if i == 0 and base is not None:
            a = a + base
        up, lo = wallvalue(a, "right"), wallvalue(a, "left")
        tot += nu / 2 * np.real(np.conj(up) * wall_diff(a, "right") - np.conj(lo) * wall_diff(a, "left"))
        tot -= gi * np.real(bulkmean(a))
    return tot


def test_power_input():
    nu = 1 / 400
    g = cfb200.Grid(16, 33, 12, LX, LZ)
    # laminar Couette: nu; laminar Poiseuille driven by (nu <Ub''>, 0) = (-2 nu, 0): 4 nu / 3
    z = cfb200.zero_state(g)
    pc = cfb200.CouetteFlow(g, nu, 0.01)
    pc.set_state(z.U, z.P)
    assert abs(pc.power_input(with_base=True) - nu) < 1e-14
    assert pc.power_input() == 0.0
    pp = cfb200.PoiseuilleFlow(g, nu, 0.01, bulkvelocity=(2 / 3, 0.0))
    pp.set_state(z.U, z.P)
    assert abs(pp.power_input((-2 * nu, 0.0), with_base=True) - 4 * nu / 3) < 1e-14
    # a random state, perturbation and total
    st = cfb200.random_state(pp, 0.2, seed=4)
    ref = O.poiseuille(16, 33, 12, LX, LZ, nu, 0.01, bulkvelocity=(2 / 3, 0.0))
    for grad in ((0.0, 0.0), (-2 * nu, 0.3)):
        for base in (None, ref.base):
            want = _power_input(st.U, nu, base, grad)
            got = pp.power_input(grad, with_base=base is not None)
            assert abs(got - want) <= 1e-13 * max(1.0, abs(want))
    pc.close()
    pp.close()
