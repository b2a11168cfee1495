"""ctypes wrapper of the CPU FP64 oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the engine (``cfb200``) never does.  It loads
``oracle/liboracle_cf.so`` built from ``cf_oracle.cpp`` (``make -C oracle``).

Array conventions: spectral fields are complex128 arrays of shape
``(Ny, Nz, Nxh)`` (C order), i.e. the reference's column-major ``(k, l, n)``
storage with k fastest (src/grids.jl:71-74).  Velocity is ``(3, Ny, Nz, Nxh)``.
Padded physical fields are float64 ``(Ny, Nzp, Nxp)``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_cf.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)

# NonLinearTerm forms (src/nonlinear.jl:10-17)
FORMS = {"rotational": 0, "convective": 1, "divergence": 2}


def build():
    """Compile the oracle library (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "cf_oracle.cpp")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_last_error.restype = ctypes.c_char_p
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [_D, ctypes.c_int] + [ctypes.c_double] * 2
        L.or_destroy.argtypes = [ctypes.c_void_p]
        L.or_set_form.argtypes = [ctypes.c_void_p, ctypes.c_int]
        for name in ("or_prepare",):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.or_step.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int, _D]
        L.or_step_dt.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double, _D]
        L.or_nonlinear.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_stage.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
        L.or_inverse.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_forward.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_operator.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, ctypes.c_int]
        L.or_curl.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_stokes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _D, _D,
                                ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        L.or_project.argtypes = [ctypes.c_void_p, _D]
        L.or_pressure.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_dot.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_dot.restype = ctypes.c_double
        L.or_diagnostics.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_synth.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_int, ctypes.c_double, _D]
        L.or_get_base.argtypes = [ctypes.c_void_p, _D, _D]
        L.or_fft.argtypes = [_D, ctypes.c_int, ctypes.c_int]
        L.or_redft00.argtypes = [_D, ctypes.c_int]
        L.or_chebcoeffs.argtypes = [_D, _D, ctypes.c_int]
        L.or_diff.argtypes = [_D, _D, ctypes.c_int]
        L.or_helmholtz.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _D,
                                   ctypes.c_double, ctypes.c_double, _D]
        L.or_influence_solve.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_int] + [_D] * 7
        L.or_influence_responses.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [_D, _D]
        L.or_mean_solve.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double] + [_D] * 8
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_set_sample_div.argtypes = [ctypes.c_long]
        L.or_get_threads.restype = ctypes.c_int
        L.or_set_helmholtz_method.argtypes = [ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def _err():
    return lib().or_last_error().decode()


def set_threads(n):
    lib().or_set_threads(int(n))


def get_threads():
    return lib().or_get_threads()


def set_sample_div(d):
    """Timing only: every independent loop of a stage runs over 1/d of its range."""
    lib().or_set_sample_div(int(d))


def set_helmholtz_method(method, dense_max_ny=0):
    """method: 'auto' (dense LU for Ny <= dense_max_ny), 'dense' or 'quasitri'."""
    m = {"auto": 0, "dense": 1, "quasitri": 2}[method]
    lib().or_set_helmholtz_method(m, int(dense_max_ny))


# ---------------------------------------------------------------- 1-D helpers
def fft(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().or_fft(_p(x.view(np.float64)), len(x), sign)
    return x


def redft00(x):
    x = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().or_redft00(_p(x.view(np.float64)), len(x))
    return x


def chebcoeffs(values):
    v = np.ascontiguousarray(values, dtype=np.float64)
    out = np.zeros_like(v)
    lib().or_chebcoeffs(_p(v), _p(out), len(v))
    return out


def diff(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros_like(a)
    lib().or_diff(_p(a), _p(out), len(a))
    return out


def helmholtz(f, theta0, theta1, bp, bm, neumann=False):
    """Tau solve of rows 0..P-2 of (theta0*D^2 - theta1) a = f with wall data (bp at +1, bm at -1)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros_like(f)
    lib().or_helmholtz(len(f), theta0, theta1, int(neumann), _p(f), bp, bm, _p(out))
    return out


def influence_solve(Ny, k, l, nu, lam, Rx, Ry, Rz, batched=False):
    """One Fourier mode of the Stokes problem (influence.jl solve!); returns u, v, w, p."""
    R = [np.ascontiguousarray(x, dtype=np.complex128) for x in (Rx, Ry, Rz)]
    out = [np.zeros(Ny, np.complex128) for _ in range(4)]
    rc = lib().or_influence_solve(Ny, k, l, nu, lam, int(batched), *[_p(x.view(np.float64)) for x in R],
                                  *[_p(x.view(np.float64)) for x in out])
    if rc != 0:
        raise ValueError(_err())
    return out


def influence_responses(Ny, k, l, nu, lam):
    out = np.zeros(6 * Ny)
    extra = np.zeros(6)
    rc = lib().or_influence_responses(Ny, k, l, nu, lam, _p(out), _p(extra))
    if rc != 0:
        raise ValueError(_err())
    return out.reshape(6, Ny), extra


def mean_solve(Ny, nu, lam, Rx, Ry, Rz, pressuregradient=None, bulkvelocity=None):
    if pressuregradient is not None and bulkvelocity is not None:
        raise ValueError("specify either pressuregradient or bulkvelocity")
    mode, c = (1, bulkvelocity) if bulkvelocity is not None else (0, pressuregradient or (0.0, 0.0))
    R = [np.ascontiguousarray(x, dtype=np.complex128) for x in (Rx, Ry, Rz)]
    out = [np.zeros(Ny, np.complex128) for _ in range(4)]
    grads = np.zeros(2)
    rc = lib().or_mean_solve(Ny, nu, lam, mode, float(c[0]), float(c[1]), *[_p(x.view(np.float64)) for x in R],
                             *[_p(x.view(np.float64)) for x in out], _p(grads))
    if rc != 0:
        raise ValueError(_err())
    return out, tuple(grads)


# ------------------------------------------------------------------ problem
class OracleProblem:
    """CPU restatement of ChannelFlowProblem + CNRK2 + NonLinearTerm.

    ``constraint`` is ("pressuregradient", (gx, gz)) or ("bulkvelocity", (ub, wb)).
    ``form`` is the nonlinear form (src/nonlinear.jl:10-17): "rotational"
    (default), "convective" or "divergence".
    """

    def __init__(self, Nx, Ny, Nz, Lx, Lz, nu, dt, profile, constraint=("pressuregradient", (0.0, 0.0)),
                 form="rotational"):
        self.Nx, self.Ny, self.Nz, self.Lx, self.Lz = Nx, Ny, Nz, float(Lx), float(Lz)
        self.nu, self.dt = float(nu), float(dt)
        self.Nxh = Nx // 2 + 1
        self.Nxp = (3 * Nx + 1) // 2
        self.Nzp = (3 * Nz + 1) // 2
        self.y = np.cos(np.pi * np.arange(Ny) / (Ny - 1))
        self.y[np.arange(Ny) * 2 == Ny - 1] = 0.0  # cospi(1/2) is exact zero
        base_values = np.ascontiguousarray(np.array([profile(v) for v in self.y], dtype=np.float64))
        kind, vals = constraint
        self.cmode = 1 if kind == "bulkvelocity" else 0
        self.constraint = (kind, tuple(float(v) for v in vals))
        h = lib().or_create(Nx, Ny, Nz, self.Lx, self.Lz, self.nu, self.dt, _p(base_values), self.cmode,
                            float(vals[0]), float(vals[1]))
        if not h:
            raise ValueError(_err())
        self._h = ctypes.c_void_p(h)
        if form not in FORMS:
            raise ValueError(f"unknown nonlinear form {form!r}")
        self.form = form
        if lib().or_set_form(self._h, FORMS[form]) != 0:
            raise ValueError(_err())
        self.base = np.zeros(Ny)
        self.basecurv = np.zeros(Ny)
        lib().or_get_base(self._h, _p(self.base), _p(self.basecurv))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.or_destroy(h)
            self._h = None

    @property
    def shape(self):
        return (self.Ny, self.Nz, self.Nxh)

    @property
    def physshape(self):
        return (self.Ny, self.Nzp, self.Nxp)

    def zeros(self, ncomp=None):
        s = self.shape if ncomp is None else (ncomp,) + self.shape
        return np.zeros(s, np.complex128)

    def prepare(self):
        rc = lib().or_prepare(self._h)
        if rc != 0:
            raise ValueError(_err())

    def step(self, U, P, nsteps=1):
        """CNRK2 step! in place on U (3,Ny,Nz,Nxh) and P (Ny,Nz,Nxh); returns last gradients."""
        assert U.dtype == np.complex128 and U.flags["C_CONTIGUOUS"] and U.shape == (3,) + self.shape
        assert P.dtype == np.complex128 and P.flags["C_CONTIGUOUS"] and P.shape == self.shape
        g = np.zeros(2)
        rc = lib().or_step(self._h, _p(U.view(np.float64)), _p(P.view(np.float64)), int(nsteps), _p(g))
        if rc != 0:
            raise ValueError(_err())
        return tuple(g)

    def step_dt(self, U, P, dt):
        """One step of duration dt (a shortened final step) in place; returns the gradients."""
        assert U.dtype == np.complex128 and U.flags["C_CONTIGUOUS"] and U.shape == (3,) + self.shape
        assert P.dtype == np.complex128 and P.flags["C_CONTIGUOUS"] and P.shape == self.shape
        g = np.zeros(2)
        rc = lib().or_step_dt(self._h, _p(U.view(np.float64)), _p(P.view(np.float64)), float(dt), _p(g))
        if rc != 0:
            raise ValueError(_err())
        return tuple(g)

    def stage(self, U, P, j):
        """One CNRK2 stage j in place (a bounded sample of a step's work)."""
        rc = lib().or_stage(self._h, _p(U.view(np.float64)), _p(P.view(np.float64)), int(j))
        if rc != 0:
            raise ValueError(_err())

    def nonlinear(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        N = self.zeros(3)
        lib().or_nonlinear(self._h, _p(U.view(np.float64)), _p(N.view(np.float64)))
        return N

    def ifft(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        u = np.zeros(self.physshape)
        lib().or_inverse(self._h, _p(U.view(np.float64)), _p(u))
        return u

    def fft(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        U = self.zeros()
        lib().or_forward(self._h, _p(u), _p(U.view(np.float64)))
        return U

    def operator(self, op, U, out=None, add=False):
        ops = {"ddx1": 1, "ddx2": 2, "ddx3": 3, "laplacian": 4}
        U = np.ascontiguousarray(U, dtype=np.complex128)
        O = self.zeros() if out is None else out
        lib().or_operator(self._h, ops[op], _p(U.view(np.float64)), _p(O.view(np.float64)), int(add))
        return O

    def curl(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        O = self.zeros(3)
        lib().or_curl(self._h, _p(U.view(np.float64)), _p(O.view(np.float64)))
        return O

    def div(self, U):
        out = self.operator("ddx1", U[0])
        self.operator("ddx2", U[1], out=out, add=True)
        self.operator("ddx3", U[2], out=out, add=True)
        return out

    def stokes(self, R, stage=None, nu=None, lam=None, pressuregradient=None, bulkvelocity=None):
        """StokesSolver solve!: with the stage bank (stage=0,1,2) or a fresh (nu, lam) bank."""
        R = np.ascontiguousarray(R, dtype=np.complex128)
        U = self.zeros(3)
        P = self.zeros()
        g = np.zeros(2)
        if bulkvelocity is not None:
            mode, c = 1, bulkvelocity
        else:
            mode, c = 0, pressuregradient or (0.0, 0.0)
        j = -1 if stage is None else int(stage)
        rc = lib().or_stokes(self._h, j, float(nu or 0.0), float(lam or 0.0), _p(U.view(np.float64)),
                             _p(P.view(np.float64)), _p(R.view(np.float64)), mode, float(c[0]), float(c[1]), _p(g))
        if rc != 0:
            raise ValueError(_err())
        return U, P, tuple(g)

    def project(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128).copy()
        rc = lib().or_project(self._h, _p(U.view(np.float64)))
        if rc != 0:
            raise ValueError(_err())
        return U

    def pressure(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        P = self.zeros()
        lib().or_pressure(self._h, _p(U.view(np.float64)), _p(P.view(np.float64)))
        return P

    def dot(self, U, V):
        U = np.ascontiguousarray(U, dtype=np.complex128)
        V = np.ascontiguousarray(V, dtype=np.complex128)
        if U.ndim == 4:
            return sum(self.dot(U[i], V[i]) for i in range(3))
        return lib().or_dot(self._h, _p(U.view(np.float64)), _p(V.view(np.float64)))

    def diagnostics(self, U):
        """[kinetic energy, dissipation, max |div|, nu*u'(+1), nu*u'(-1)] of the perturbation."""
        U = np.ascontiguousarray(U, dtype=np.complex128)
        out = np.zeros(5)
        lib().or_diagnostics(self._h, _p(U.view(np.float64)), _p(out))
        return out

    def synth(self, seed, amp, shape=0, rho=0.8):
        U = self.zeros(3)
        lib().or_synth(self._h, int(seed), float(amp), int(shape), float(rho), _p(U.view(np.float64)))
        return U

    def random_state(self, seed, amp, shape=0, rho=0.8):
        """Seeded synthetic state: spectral Gaussian -> project! -> pressure (modified)."""
        U = self.project(self.synth(seed, amp, shape, rho))
        P = self.pressure(U)
        return U, P

    # --------------------------------------------------- sampling helpers
    def sample(self, f):
        """Sample f(x, y, z) on the padded physical mesh, storage (Ny, Nzp, Nxp)."""
        x = self.Lx * np.arange(self.Nxp) / self.Nxp
        z = self.Lz * np.arange(self.Nzp) / self.Nzp
        Y, Z, X = np.meshgrid(self.y, z, x, indexing="ij")
        return np.ascontiguousarray(np.broadcast_to(f(X, Y, Z), (self.Ny, self.Nzp, self.Nxp)), dtype=np.float64)

    def spectral(self, f):
        return self.fft(self.sample(f))


def couette(Nx, Ny, Nz, Lx, Lz, nu, dt, **kw):
    return OracleProblem(Nx, Ny, Nz, Lx, Lz, nu, dt, lambda y: y, **kw)


def poiseuille(Nx, Ny, Nz, Lx, Lz, nu, dt, bulkvelocity=None, pressuregradient=None, form="rotational"):
    if bulkvelocity is not None:
        c = ("bulkvelocity", bulkvelocity)
    else:
        c = ("pressuregradient", pressuregradient if pressuregradient is not None else (-2 * nu, 0.0))
    return OracleProblem(Nx, Ny, Nz, Lx, Lz, nu, dt, lambda y: 1 - y * y, constraint=c, form=form)
