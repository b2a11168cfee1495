"""cfb200 -- B200-native CNRK2 engine for ChannelFlow.jl's time step.

Host-side mirror of the reference's Julia API for this path (ChannelFlow.jl
src/grids.jl, src/problem.jl, src/initialization.jl, src/timesteppers/cnrk2.jl),
bound to the C ABI of ``libcfb200.so`` (include/cfb200.h) with ctypes.  The
compute runs only in the CUDA library: importing works without a GPU, but every
operation that needs the engine raises if the library or the device is
missing -- there is no CPU fallback.

Arrays follow the reference storage: a spectral field is complex128 of shape
``(Ny, Nz, Nx//2+1)`` in C order (Julia's ``(Nx/2+1, Nz, Ny)`` column-major
with k fastest); a velocity is ``(3, Ny, Nz, Nx//2+1)``.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfb200.so")
_lib = None
_D = ctypes.POINTER(ctypes.c_double)


class CFError(RuntimeError):
    """Error returned by the engine (the reference raises ArgumentError/DimensionMismatch)."""

    def __init__(self, code, msg):
        super().__init__(f"cfb200 error {code}: {msg}")
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("Lx", ctypes.c_double), ("Lz", ctypes.c_double),
                ("nu", ctypes.c_double), ("dt", ctypes.c_double),
                ("profile", ctypes.c_int), ("base_values", _D),
                ("constraint", ctypes.c_int), ("c1", ctypes.c_double), ("c2", ctypes.c_double),
                ("precision", ctypes.c_int), ("form", ctypes.c_int)]

PRECISIONS = {"fp64": 0, "mixed": 1, "mixed-tc": 2, "mixed-bf16": 3, "mixed-f32state": 4}
# NonLinearTerm forms (src/nonlinear.jl:10-17): CF_FORM_* of cfb200.h
FORMS = {"rotational": 0, "convective": 1, "divergence": 2}


EXPORTS = ["cf_create", "cf_destroy", "cf_set_constraint", "cf_set_state", "cf_get_state",
           "cf_set_state_device", "cf_get_state_device", "cf_step", "cf_nonlinear", "cf_project",
           "cf_pressure", "cf_random_state", "cf_diagnostics", "cf_sync", "cf_last_launch_count",
           "cf_stream", "cf_last_error", "cf_step_profiled", "cf_nonlinear_noalloc", "cf_create_batch",
           "cf_destroy_batch", "cf_batch_size", "cf_batch_instance", "cf_step_batch",
           "cf_batch_last_launch_count", "cf_batch_stream", "cf_cheb_transform", "cf_step_dt",
           "cf_step_host", "cf_power_input", "cf_device_bytes", "cf_set_wait_limit", "cf_cheb_transform_split",
           "cf_batch_schedule", "cf_step_record"]

# return codes of cfb200.h
CF_E_ARG, CF_E_SINGULAR, CF_E_NOMEM, CF_E_CUDA, CF_E_UNSUPPORTED, CF_E_NONFINITE = -1, -2, -3, -4, -5, -6


def lib():
    """Load libcfb200.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.cf_last_error.restype = ctypes.c_char_p
        L.cf_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_void_p)]
        L.cf_destroy.argtypes = [ctypes.c_void_p]
        L.cf_destroy.restype = None
        L.cf_set_constraint.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.cf_set_state.argtypes = [ctypes.c_void_p, _D, _D]
        L.cf_get_state.argtypes = [ctypes.c_void_p, _D, _D]
        L.cf_set_state_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.cf_get_state_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.cf_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _D, _D]
        L.cf_step_dt.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D, _D]
        L.cf_step_host.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double, ctypes.c_int, _D, _D]
        L.cf_nonlinear.argtypes = [ctypes.c_void_p, _D, _D]
        L.cf_nonlinear_noalloc.argtypes = [ctypes.c_void_p, _D, _D]
        L.cf_cheb_transform.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                        ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.cf_create_batch.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.cf_destroy_batch.argtypes = [ctypes.c_void_p]
        L.cf_destroy_batch.restype = None
        L.cf_batch_size.argtypes = [ctypes.c_void_p]
        L.cf_batch_instance.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_batch_instance.restype = ctypes.c_void_p
        L.cf_step_batch.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cf_batch_last_launch_count.argtypes = [ctypes.c_void_p]
        L.cf_batch_stream.argtypes = [ctypes.c_void_p]
        L.cf_batch_stream.restype = ctypes.c_void_p
        L.cf_batch_schedule.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.cf_project.argtypes = [ctypes.c_void_p, _D]
        L.cf_pressure.argtypes = [ctypes.c_void_p, _D, _D]
        L.cf_random_state.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double]
        L.cf_diagnostics.argtypes = [ctypes.c_void_p, _D]
        L.cf_step_profiled.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _D, _D]
        L.cf_sync.argtypes = [ctypes.c_void_p]
        L.cf_last_launch_count.argtypes = [ctypes.c_void_p]
        L.cf_stream.argtypes = [ctypes.c_void_p]
        L.cf_stream.restype = ctypes.c_void_p
        L.cf_power_input.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        L.cf_step_record.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D, _D]
        L.cf_device_bytes.argtypes = [ctypes.c_void_p]
        L.cf_device_bytes.restype = ctypes.c_longlong
        L.cf_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_long]
        L.cf_cheb_transform_split.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                              ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_int]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise CFError(rc, lib().cf_last_error().decode())


def _ptr(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


class Grid:
    """Grid(Nx, Ny, Nz, Lx, Lz) (src/grids.jl:27-30): Lobatto y, upper wall first."""

    def __init__(self, Nx, Ny, Nz, Lx, Lz):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Lx, self.Lz = float(Lx), float(Lz)
        n = np.arange(self.Ny)
        self.y = np.cos(np.pi * n / (self.Ny - 1))
        self.y[2 * n == self.Ny - 1] = 0.0

    @property
    def spectralsize(self):
        return (self.Ny, self.Nz, self.Nx // 2 + 1)

    def physicalsize(self, padded=True):
        if padded:
            return (self.Ny, (3 * self.Nz + 1) // 2, (3 * self.Nx + 1) // 2)
        return (self.Ny, self.Nz, self.Nx)

    def __eq__(self, other):
        return isinstance(other, Grid) and (self.Nx, self.Ny, self.Nz, self.Lx, self.Lz) == (
            other.Nx, other.Ny, other.Nz, other.Lx, other.Lz)

    def __repr__(self):
        return f"Grid({self.Nx}, {self.Ny}, {self.Nz}, {self.Lx}, {self.Lz})"


class State:
    """State(U, P) (src/state.jl:18-34): perturbation velocity and stage pressure."""

    def __init__(self, U, P):
        self.U = U
        self.P = P

    def velocity(self):
        return self.U

    def stagepressure(self):
        return self.P

    def copy(self):
        return State(self.U.copy(), self.P.copy())


def zero_state(grid):
    """zero_state(grid) (src/initialization.jl:16)."""
    return State(np.zeros((3,) + grid.spectralsize, np.complex128), np.zeros(grid.spectralsize, np.complex128))


def _make_config(grid, profile, nu, dt, pressuregradient=None, bulkvelocity=None, forcing=None, form=None,
                 precision="fp64"):
    """cf_config of ChannelFlowProblem(grid, profile, nu, dt; ...); returns
    (config, base-profile array kept alive for the call, constraint)."""
    if pressuregradient is not None and bulkvelocity is not None:
        raise ValueError("specify either pressuregradient or bulkvelocity")
    if forcing is not None:
        raise ValueError("only NoForcing is accelerated by the engine")
    form = "rotational" if form is None else form
    if form not in FORMS:
        raise ValueError(f"form must be one of {sorted(FORMS)}")
    if bulkvelocity is not None:
        constraint = ("bulkvelocity", tuple(float(v) for v in bulkvelocity))
    else:
        pg = (0.0, 0.0) if pressuregradient is None else pressuregradient
        constraint = ("pressuregradient", tuple(float(v) for v in pg))
    cfg = _Config()
    cfg.Nx, cfg.Ny, cfg.Nz = grid.Nx, grid.Ny, grid.Nz
    cfg.Lx, cfg.Lz, cfg.nu, cfg.dt = grid.Lx, grid.Lz, float(nu), float(dt)
    base = None
    if profile == "couette":
        cfg.profile = 0
    elif profile == "poiseuille":
        cfg.profile = 1
    else:
        cfg.profile = 2
        base = np.ascontiguousarray([float(profile(v)) for v in grid.y], dtype=np.float64)
        cfg.base_values = _ptr(base)
    cfg.constraint = 1 if constraint[0] == "bulkvelocity" else 0
    cfg.c1, cfg.c2 = constraint[1]
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    cfg.precision = PRECISIONS[precision]
    cfg.form = FORMS[form]
    return cfg, base, constraint


class ChannelFlowProblem:
    """ChannelFlowProblem(grid, profile, nu, dt; pressuregradient | bulkvelocity,
    form) (src/problem.jl:69-107) with NoForcing, on the B200.

    ``profile`` is "couette", "poiseuille" or a callable Ub(y); ``form`` is the
    nonlinear form, "rotational" (default), "convective" or "divergence"
    (src/nonlinear.jl:10-17).
    """

    def __init__(self, grid, profile, nu, dt, pressuregradient=None, bulkvelocity=None, forcing=None, form=None,
                 precision="fp64"):
        cfg, self._base, self.constraint = _make_config(grid, profile, nu, dt, pressuregradient, bulkvelocity,
                                                        forcing, form, precision)
        self.precision = precision
        self.form = "rotational" if form is None else form
        self.grid = grid
        self.nu, self.dt = float(nu), float(dt)
        h = ctypes.c_void_p()
        _check(lib().cf_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._owned = True

    @classmethod
    def _borrow(cls, handle, grid, nu, dt, constraint):
        """View of a handle owned elsewhere (an ensemble instance)."""
        self = cls.__new__(cls)
        self.grid, self.nu, self.dt, self.constraint = grid, float(nu), float(dt), constraint
        self._base = None
        self.precision = "fp64"
        self.form = "rotational"
        self._h = ctypes.c_void_p(handle)
        self._owned = False
        return self

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            if getattr(self, "_owned", True):
                _lib.cf_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------ device-resident state
    def set_state(self, U, P):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        P = np.ascontiguousarray(P, dtype=np.complex128)
        assert U.shape == (3,) + self.grid.spectralsize and P.shape == self.grid.spectralsize
        _check(lib().cf_set_state(self._h, _ptr(U.view(np.float64)), _ptr(P.view(np.float64))))

    def get_state(self, out=None):
        """Download the state; out=(U, P) writes into the caller's contiguous
        complex128 arrays (e.g. pinned buffers) instead of new ones."""
        if out is None:
            U = np.zeros((3,) + self.grid.spectralsize, np.complex128)
            P = np.zeros(self.grid.spectralsize, np.complex128)
        else:
            U, P = out
            if not (U.dtype == np.complex128 and P.dtype == np.complex128 and U.flags["C_CONTIGUOUS"]
                    and P.flags["C_CONTIGUOUS"] and U.shape == (3,) + self.grid.spectralsize
                    and P.shape == self.grid.spectralsize):
                raise ValueError("out must be contiguous complex128 arrays of the state's shapes")
        _check(lib().cf_get_state(self._h, _ptr(U.view(np.float64)), _ptr(P.view(np.float64))))
        return U, P

    def advance(self, t, nsteps=1):
        """Advance the engine-resident state nsteps steps; returns (t + nsteps*dt, last gradients)."""
        tout = ctypes.c_double()
        g = np.zeros(2)
        _check(lib().cf_step(self._h, float(t), int(nsteps), ctypes.byref(tout), _ptr(g)))
        return tout.value, tuple(g)

    def advance_dt(self, t, dt):
        """One step of duration dt (the Flows adapter's step,
        ext/ChannelFlowFlowsExt.jl:36-52; factors for a dt other than the
        nominal one are built on first use and kept); returns (t + dt, gradients)."""
        tout = ctypes.c_double()
        g = np.zeros(2)
        _check(lib().cf_step_dt(self._h, float(t), float(dt), ctypes.byref(tout), _ptr(g)))
        return tout.value, tuple(g)

    def advance_profiled(self, t, nsteps=1):
        """As advance() without the graph; returns (t_out, ms per kernel class
        [z-inverse, x-pass, z-forward, column, forward and inverse tensor-core
        Chebyshev transforms (mixed precision)] summed over the steps)."""
        tout = ctypes.c_double()
        ms = np.zeros(6)
        _check(lib().cf_step_profiled(self._h, float(t), int(nsteps), ctypes.byref(tout), _ptr(ms)))
        return tout.value, ms

    def stream_ptr(self):
        return lib().cf_stream(self._h)

    def launches(self):
        return lib().cf_last_launch_count(self._h)

    def sync(self):
        _check(lib().cf_sync(self._h))

    # ------------------------------------------------ operators
    def nonlinear(self, U):
        """NonLinearTerm(t, U, N) of the problem's form (src/nonlinear.jl:113-193)."""
        U = np.ascontiguousarray(U, dtype=np.complex128)
        N = np.zeros_like(U)
        _check(lib().cf_nonlinear(self._h, _ptr(U.view(np.float64)), _ptr(N.view(np.float64))))
        return N

    def nonlinear_noalloc(self, U):
        """nonlinear() staged in the library's fixed device scratch (allocates
        nothing; grids with 3 * Nr * 16 bytes <= 16 MiB)."""
        U = np.ascontiguousarray(U, dtype=np.complex128)
        N = np.zeros_like(U)
        _check(lib().cf_nonlinear_noalloc(self._h, _ptr(U.view(np.float64)), _ptr(N.view(np.float64))))
        return N

    def diagnostics(self):
        out = np.zeros(5)
        _check(lib().cf_diagnostics(self._h, _ptr(out)))
        return out

    RECORD_COLUMNS = ("t", "kinetic_energy", "dissipation", "max_div", "wall_shear_upper", "wall_shear_lower",
                      "dPdx", "dPdz", "power_input")

    def advance_recorded(self, t, nsteps, every):
        """Advance nsteps steps with the diagnostics recorded on the device
        after every `every` steps (cf_step_record; no host synchronisation
        between steps): returns (t + nsteps*dt, last gradients, rows), rows an
        (nsteps // every, 9) array with the columns RECORD_COLUMNS."""
        rows = np.zeros((int(nsteps) // int(every), 9)) if every > 0 else np.zeros((0, 9))
        buf = rows if rows.size else np.zeros(9)
        tout = ctypes.c_double()
        g = np.zeros(2)
        _check(lib().cf_step_record(self._h, float(t), int(nsteps), int(every), _ptr(buf), ctypes.byref(tout), _ptr(g)))
        return tout.value, tuple(g), rows

    def power_input(self, pressuregradient=(0.0, 0.0), with_base=False):
        """power_input(U, nu; pressuregradient) (src/postprocessing.jl:113-128) of
        the engine's velocity; with_base adds the base profile first (total flow)."""
        out = np.zeros(1)
        _check(lib().cf_power_input(self._h, 1 if with_base else 0, float(pressuregradient[0]),
                                    float(pressuregradient[1]), _ptr(out)))
        return float(out[0])

    def device_bytes(self):
        """Device memory held by the handle (bytes)."""
        return int(lib().cf_device_bytes(self._h))

    def set_wait_limit(self, spins):
        """Test hook: polls after which a kernel's first bounded wait gives up
        (negative restores the default)."""
        _check(lib().cf_set_wait_limit(self._h, int(spins)))


class Ensemble:
    """Many independent channels advanced together (cf_create_batch): each
    member is given as (grid, profile, nu, dt, constraint keywords) and is
    reachable as an ordinary problem through ``instances``; ``step`` advances
    all of them with one graph per step, every kernel launched once per size
    class."""

    def __init__(self, members):
        members = list(members)
        n = len(members)
        cfgs = (_Config * n)()
        self._keep = []
        specs = []
        for i, m in enumerate(members):
            kw = dict(m)
            grid, profile, nu, dt = kw.pop("grid"), kw.pop("profile"), kw.pop("nu"), kw.pop("dt")
            cfg, base, constraint = _make_config(grid, profile, nu, dt, **kw)
            cfgs[i] = cfg
            self._keep.append(base)
            specs.append((grid, nu, dt, constraint))
        h = ctypes.c_void_p()
        _check(lib().cf_create_batch(cfgs, n, ctypes.byref(h)))
        self._h = h
        self.instances = []
        for i, (grid, nu, dt, constraint) in enumerate(specs):
            ih = lib().cf_batch_instance(self._h, i)
            self.instances.append(ChannelFlowProblem._borrow(ih, grid, nu, dt, constraint))

    def __len__(self):
        return len(self.instances)

    def step(self, nsteps=1):
        """nsteps CNRK2 steps of every member (asynchronous on the ensemble's stream)."""
        _check(lib().cf_step_batch(self._h, int(nsteps)))

    def stream_ptr(self):
        return lib().cf_batch_stream(self._h)

    def launches(self):
        return lib().cf_batch_last_launch_count(self._h)

    def schedule(self):
        """The autotuner's choice per size class (and the candidates' timings)."""
        buf = ctypes.create_string_buffer(1 << 16)
        n = lib().cf_batch_schedule(self._h, buf, len(buf))
        if n < 0:
            _check(n)
        return buf.value.decode()

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            for p in self.instances:
                p._h = None
            _lib.cf_destroy_batch(self._h)
            self._h = None

    def __del__(self):
        self.close()


def cheb_transform(X, inverse, scale=1.0, split="tf32"):
    """Chebyshev transform along axis 1 of float32 X (fields, Ny, C) on the
    tensor cores: inverse -> values at the Lobatto nodes; forward -> scaled
    coefficients with halved end coefficients.  split: "tf32" (heads and
    remainders) or "bf16" (three BF16 pieces)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    nf, Ny, C = X.shape
    Y = np.zeros_like(X)
    fp = ctypes.POINTER(ctypes.c_float)
    code = {"tf32": 0, "bf16": 1}[split]
    _check(lib().cf_cheb_transform_split(X.ctypes.data_as(fp), Y.ctypes.data_as(fp), Ny, C, nf,
                                         1 if inverse else 0, float(scale), code))
    return Y


def CouetteFlow(grid, nu, dt, **kw):
    """CouetteFlow(grid, nu, dt) (src/problem.jl:122-123): Ub = y."""
    return ChannelFlowProblem(grid, "couette", nu, dt, **kw)


def PoiseuilleFlow(grid, nu, dt, bulkvelocity=None, pressuregradient=None, **kw):
    """PoiseuilleFlow(grid, nu, dt) (src/problem.jl:137-144): Ub = 1 - y^2, default gradient (-2nu, 0)."""
    if bulkvelocity is None and pressuregradient is None:
        pressuregradient = (-2 * nu, 0.0)
    return ChannelFlowProblem(grid, "poiseuille", nu, dt, bulkvelocity=bulkvelocity,
                              pressuregradient=pressuregradient, **kw)


def project_(U, problem):
    """project!(U, problem) (src/pressure.jl:36-54); U updated in place and returned."""
    assert U.dtype == np.complex128 and U.flags["C_CONTIGUOUS"]
    _check(lib().cf_project(problem.handle, _ptr(U.view(np.float64))))
    return U


def pressure(U, problem):
    """pressure(U, problem) (src/pressure.jl:95-104): the modified pressure for
    the rotational form, the ordinary pressure for the other two."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    P = np.zeros(problem.grid.spectralsize, np.complex128)
    _check(lib().cf_pressure(problem.handle, _ptr(U.view(np.float64)), _ptr(P.view(np.float64))))
    return P


def random_state(problem, epsilon, seed=1, shape=0, rho=0.8):
    """random_state(problem, epsilon) (src/initialization.jl:32-51) with a seeded
    spectral generator: returns a host State and leaves it resident in the engine."""
    if epsilon < 0:
        raise ValueError("epsilon must be non-negative")
    _check(lib().cf_random_state(problem.handle, int(seed), float(epsilon), int(shape), float(rho)))
    U, P = problem.get_state()
    return State(U, P)


def step_(problem, U, P, t, nsteps=1):
    """step!(scheme, nlterm, U, P, t; constraint...) (src/timesteppers/cnrk2.jl:149-207).

    Host buffers U, P are advanced in place (upload, nsteps device steps,
    download) and t + nsteps*dt is returned.  Contiguous complex128 buffers go
    through cf_step_host, which overlaps the transfers with the first and last
    column kernels; others through a contiguous copy.
    """
    if U.shape != (3,) + problem.grid.spectralsize or P.shape != problem.grid.spectralsize:
        raise ValueError("fields must have the resolved spectral size")
    direct = all(a.dtype == np.complex128 and a.flags["C_CONTIGUOUS"] and a.flags["WRITEABLE"] for a in (U, P))
    Uc, Pc = (U, P) if direct else (np.ascontiguousarray(U, np.complex128), np.ascontiguousarray(P, np.complex128))
    tout = ctypes.c_double()
    _check(lib().cf_step_host(problem._h, _ptr(Uc.view(np.float64)), _ptr(Pc.view(np.float64)), float(t),
                              int(nsteps), ctypes.byref(tout), None))
    if not direct:
        U[...] = Uc
        P[...] = Pc
    return tout.value


def _download_into(problem, U, P):
    """The engine state into the caller's arrays: directly when they are
    contiguous complex128 (pinned buffers stay pinned), else through a copy."""
    if U.dtype == np.complex128 and P.dtype == np.complex128 and U.flags["C_CONTIGUOUS"] and P.flags["C_CONTIGUOUS"]:
        problem.get_state(out=(U, P))
    else:
        U2, P2 = problem.get_state()
        U[...] = U2
        P[...] = P2


def flow(problem):
    """Flows.flow(problem) (ext/ChannelFlowFlowsExt.jl:28-29): a callable
    (state, (t0, t1)) -> state advancing a host State in place from t0 to t1
    with the nominal step and a final step shortened to end on t1 (run with
    its own factors, cf_step_dt; test/test_timestepping.jl:31-41).  A
    remainder below 1e-10 of the nominal step is not stepped."""

    def run(state, span):
        t0, t1 = float(span[0]), float(span[1])
        if not t1 >= t0:
            raise ValueError("the interval must not run backwards")
        if state.U.shape != (3,) + problem.grid.spectralsize or state.P.shape != problem.grid.spectralsize:
            raise ValueError("the state does not belong to the problem's grid")
        dt = problem.dt
        problem.set_state(state.U, state.P)
        nfull = int(np.floor((t1 - t0) / dt * (1 + 1e-12)))
        t = t0
        if nfull:
            t, _ = problem.advance(t, nfull)
            t = t0 + nfull * dt
        rest = t1 - t
        if rest > 1e-10 * dt:
            t, _ = problem.advance_dt(t, rest)
        _download_into(problem, state.U, state.P)
        return state

    return run


def kinetic_energy_of(problem):
    return problem.diagnostics()[0]
