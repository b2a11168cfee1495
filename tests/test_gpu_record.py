"""GPU: diagnostics recorded on the device between steps (cf_step_record).

The rows must equal what a caller gets by stepping and then asking for the
diagnostics and the power input through the synchronous entry points (the
same kernels on the same state: bit-identical), and the last row must match
the oracle's diagnostics of its own trajectory (FP64 step parity plus the
1e-12 bound of the diagnostics test).
"""
import numpy as np
import pytest

import cfb200
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pair(precision="fp64"):
    g = cfb200.Grid(24, 25, 20, 2 * np.pi, np.pi)
    kw = dict(bulkvelocity=(2 / 3, 0.0))
    a = cfb200.PoiseuilleFlow(g, 1 / 1500, 0.005, precision=precision, **kw)
    b = cfb200.PoiseuilleFlow(g, 1 / 1500, 0.005, precision=precision, **kw)
    return g, a, b


@pytest.mark.parametrize("precision", ["fp64", "mixed-f32state"])
def test_recorded_rows_equal_synchronous_diagnostics(precision):
    g, a, b = _pair(precision)
    st = cfb200.random_state(a, 0.1, seed=7)
    b.set_state(st.U, st.P)
    t_a, g_a, rows = a.advance_recorded(0.0, 23, 5)
    assert rows.shape == (4, 9)
    t_b = 0.0
    for r in range(4):
        t_b, g_b = b.advance(t_b, 5)
        d = b.diagnostics()
        pin = b.power_input(pressuregradient=g_b, with_base=True)
        assert rows[r, 0] == pytest.approx(t_b, abs=1e-12)
        assert np.array_equal(rows[r, 1:6], d), (r, rows[r, 1:6], d)
        assert tuple(rows[r, 6:8]) == g_b
        assert rows[r, 8] == pin
    t_b, g_b = b.advance(t_b, 3)
    assert t_a == pytest.approx(t_b) and g_a == g_b
    assert np.array_equal(a.get_state()[0], b.get_state()[0])
    a.close()
    b.close()


def test_recorded_rows_match_the_oracle():
    Nx, Ny, Nz = 16, 17, 16
    g = cfb200.Grid(Nx, Ny, Nz, 5.3, 7.1)
    gpu = cfb200.CouetteFlow(g, 1 / 300, 0.01)
    ref = O.couette(Nx, Ny, Nz, 5.3, 7.1, 1 / 300, 0.01)
    U, P = ref.random_state(seed=5, amp=0.2)
    gpu.set_state(U, P)
    _, _, rows = gpu.advance_recorded(0.0, 10, 5)
    for r in range(2):
        ref.step(U, P, 5)
        do = ref.diagnostics(U)
        assert abs(rows[r, 1] - do[0]) <= 1e-11 * abs(do[0])
        assert abs(rows[r, 2] - do[1]) <= 1e-11 * abs(do[1])
        for i in (3, 4):
            assert abs(rows[r, 1 + i] - do[i]) <= 1e-11 * max(1.0, abs(do[i]))
    gpu.close()


def test_record_rejects_bad_cadence():
    g = cfb200.Grid(8, 9, 8, 5.3, 7.1)
    pb = cfb200.CouetteFlow(g, 1 / 300, 0.01)
    with pytest.raises(cfb200.CFError) as e:
        pb.advance_recorded(0.0, 4, 0)
    assert e.value.code == cfb200.CF_E_ARG
    pb.close()
