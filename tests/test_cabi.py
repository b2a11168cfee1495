"""C-ABI checks that need no GPU: the library loads, every function declared
in include/cfb200.h is exported, and calls fail cleanly without a device."""
import ctypes
import os
import re

import pytest

import cfb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "cfb200.h")).read()
    return sorted(set(re.findall(r"\b(cf_[a-z_]+)\s*\(", src)))


def test_header_matches_python_binding():
    assert sorted(cfb200.EXPORTS) == [n for n in declared() if n in cfb200.EXPORTS]
    assert set(declared()) <= set(cfb200.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = cfb200.lib()
    for name in declared():
        assert hasattr(L, name), name


def test_errors_are_reported_not_crashed():
    # argument validation happens before any device work (stokes.jl:35, stokes.jl:36-38)
    with pytest.raises(cfb200.CFError) as e:
        cfb200.CouetteFlow(cfb200.Grid(8, 10, 8, 6.28, 6.28), 0.01, 0.01)
    assert e.value.code == -1 and "odd Ny" in str(e.value)
    with pytest.raises(cfb200.CFError):
        cfb200.CouetteFlow(cfb200.Grid(8, 9, 8, 6.28, 6.28), 0.01, 0.0)
    with pytest.raises(ValueError):
        cfb200.ChannelFlowProblem(cfb200.Grid(8, 9, 8, 6.28, 6.28), "couette", 0.01, 0.01,
                                  pressuregradient=(0, 0), bulkvelocity=(0, 0))


def test_form_validation_before_device_work():
    g = cfb200.Grid(8, 9, 8, 6.28, 6.28)
    with pytest.raises(ValueError):
        cfb200.CouetteFlow(g, 0.01, 0.01, form="skew-symmetric")
    # the mixed precision runs the rotational form only (CF_E_UNSUPPORTED)
    with pytest.raises(cfb200.CFError) as e:
        cfb200.CouetteFlow(g, 0.01, 0.01, form="divergence", precision="mixed")
    assert e.value.code == -5
    # an out-of-range cf_config.form is CF_E_ARG
    cfg, _, _ = cfb200._make_config(g, "couette", 0.01, 0.01)
    cfg.form = 7
    h = ctypes.c_void_p()
    assert cfb200.lib().cf_create(ctypes.byref(cfg), ctypes.byref(h)) == -1


def test_step_entry_points_reject_null_handles():
    # every step entry point checks its handle and arguments before any CUDA call
    L = cfb200.lib()
    t = ctypes.c_double()
    buf = (ctypes.c_double * 4)()
    assert L.cf_step(None, 0.0, 1, ctypes.byref(t), None) == -1
    assert L.cf_step_dt(None, 0.0, 0.01, ctypes.byref(t), None) == -1
    assert L.cf_step_host(None, buf, buf, 0.0, 1, ctypes.byref(t), None) == -1
    assert "null" in L.cf_last_error().decode()


@pytest.mark.parametrize("dims, field, value, code, words", [
    ((8, 17, 8), "nu", float("inf"), -1, "nu must be finite"),
    ((8, 17, 8), "dt", -0.01, -1, "dt must be finite"),
    ((8, 17, 8), "precision", 7, -1, "unknown precision"),
    ((8, 577, 6), "precision", 2, -5, "Ny <= 512"),
    ((74, 17, 8), None, None, -5, "padded x length"),
    ((8, 17, 74), None, None, -5, "padded z length"),
    ((8, 1025, 6), None, None, -5, "Ny too large"),
])
def test_sizes_and_modes_rejected_before_device_work(dims, field, value, code, words):
    # cf_create checks the configuration before it creates a stream or
    # allocates (no GPU needed): 3/2-padded lengths with a prime factor above
    # 31 (74 -> 111 = 3 x 37), a column too long for the shared memory of the
    # column kernel, the tensor-core transforms beyond Ny = 512
    g = cfb200.Grid(*dims, 6.28, 6.28)
    cfg, _, _ = cfb200._make_config(g, "couette", 0.01, 0.01)
    if field:
        setattr(cfg, field, value)
    h = ctypes.c_void_p()
    assert cfb200.lib().cf_create(ctypes.byref(cfg), ctypes.byref(h)) == code
    assert words in cfb200.lib().cf_last_error().decode()
    assert not h.value
