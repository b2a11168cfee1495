"""GPU: step! on host buffers through cf_step_host (cnrk2.jl:149-207 with CPU
fields), which moves the state over PCIe in kz-plane chunks overlapped with
the first and last column kernels.

The pipelined call must give exactly (bit for bit) what cf_set_state +
cf_step + cf_get_state give: the chunks only split the column range of the
same kernels.  Grids cover an odd number of kx modes (Nxh odd: chunk bounds on
even kz planes), fewer kz planes than chunks, Nz = 1, one and several steps
(the middle ones from the step's CUDA graph), the three nonlinear forms and
the mixed precisions (the tensor-core form runs unchunked).  The last stage
of a host step skips the nodal fields of a following stage; a later cf_step
recomputes them from the state, which the chained cases check.
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make(dims, form="rotational", precision="fp64", profile="couette"):
    Nx, Ny, Nz = dims
    g = cfb200.Grid(Nx, Ny, Nz, 5.3, 7.1)
    if profile == "couette":
        return cfb200.CouetteFlow(g, 1 / 400, 0.01, form=form, precision=precision)
    return cfb200.PoiseuilleFlow(g, 1 / 400, 0.01, bulkvelocity=(2 / 3, 0.0), form=form, precision=precision)


def start(pb, seed=5):
    st = cfb200.random_state(pb, 0.1, seed=seed)
    return st.U.copy(), st.P.copy()


def plain(pb, U, P, t, n):
    pb.set_state(U, P)
    t2, _ = pb.advance(t, n)
    Ug, Pg = pb.get_state()
    return Ug, Pg, t2


@pytest.mark.parametrize("dims", [(16, 17, 16), (12, 17, 10), (16, 33, 5), (8, 17, 1), (32, 33, 30)])
@pytest.mark.parametrize("nsteps", [1, 3])
def test_host_step_equals_set_step_get(dims, nsteps):
    a, b = make(dims, profile="poiseuille"), make(dims, profile="poiseuille")
    U, P = start(a)
    Ug, Pg, tg = plain(a, U, P, 0.5, nsteps)
    Uh, Ph = U.copy(), P.copy()
    th = cfb200.step_(b, Uh, Ph, 0.5, nsteps)
    assert th == tg
    assert np.array_equal(Uh, Ug)
    assert np.array_equal(Ph, Pg)
    a.close()
    b.close()


@pytest.mark.parametrize("form", ["rotational", "convective", "divergence"])
def test_chained_host_steps_and_device_steps_agree(form):
    # host, host, then a device step (stale nodal fields recomputed) against
    # three device steps from the same state
    dims = (16, 17, 12)
    a, b = make(dims, form=form), make(dims, form=form)
    U, P = start(a, seed=8)
    a.set_state(U, P)
    a.advance(0.0, 3)
    Ua, Pa = a.get_state()
    Uh, Ph = U.copy(), P.copy()
    t = cfb200.step_(b, Uh, Ph, 0.0, 1)
    t = cfb200.step_(b, Uh, Ph, t, 1)
    b.advance(t, 1)
    Ub, Pb = b.get_state()
    assert np.array_equal(Ub, Ua)
    assert np.array_equal(Pb, Pa)
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["mixed", "mixed-tc", "mixed-f32state"])
def test_host_step_mixed(precision):
    dims = (16, 17, 16)
    a, b = make(dims, precision=precision), make(dims, precision=precision)
    U, P = start(a, seed=2)
    Ug, Pg, _ = plain(a, U, P, 0.0, 2)
    Uh, Ph = U.copy(), P.copy()
    cfb200.step_(b, Uh, Ph, 0.0, 2)
    assert np.array_equal(Uh, Ug)
    assert np.array_equal(Ph, Pg)
    a.close()
    b.close()


def test_host_step_matches_oracle_and_other_layouts():
    # against the oracle, with a strided (non-contiguous) view as the buffer
    Nx, Ny, Nz = 16, 17, 16
    g = cfb200.Grid(Nx, Ny, Nz, 5.3, 7.1)
    gpu = cfb200.CouetteFlow(g, 1 / 400, 0.01)
    ref = O.couette(Nx, Ny, Nz, 5.3, 7.1, 1 / 400, 0.01)
    U, P = ref.random_state(seed=12, amp=0.05)
    big = np.zeros((3, Ny, Nz, 2 * (Nx // 2 + 1)), np.complex128)
    Uv = big[..., ::2]
    Uv[...] = U
    Ph = P.copy()
    t = cfb200.step_(gpu, Uv, Ph, 0.0, 2)
    ref.step(U, P, 2)
    assert abs(t - 0.02) < 1e-15
    assert np.linalg.norm(Uv - U) <= 1e-12 * np.linalg.norm(U)
    assert np.all(big[..., 1::2] == 0)
    gpu.close()
