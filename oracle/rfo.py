"""ctypes binding of the CPU FP64 oracle (oracle/_build/librfo.so).

Test infrastructure only: tests/, the package smoke check and bench.py's
CPU-baseline leg import this module as the checker.  The product path never
does.  See rfo.h for the reference lines each routine restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librfo.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class RfoParams(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int),
        ("N", ctypes.c_int),
        ("NoQI", ctypes.c_int),
        ("analytic", ctypes.c_int),
        ("direct", ctypes.c_int),
        ("restart", ctypes.c_int),
        ("max_iters", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("eps", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("ext_force", ctypes.c_double * 3),
        ("threads", ctypes.c_int),
    ]


def build(reference="/root/reference"):
    """Compile the oracle with its Makefile (g++, OpenMP); where the
    reference's sources are present, also its own CUDA program (_ref/, the
    reference-gpu arm of bench.py).  A failure of that second build is
    reported and leaves the oracle usable."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    if os.path.isdir(os.path.join(reference, "src")):
        r = subprocess.run(["make", "-s", "-C", _HERE, "ref-gpu", f"REFERENCE={reference}"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            print("reference CUDA program not built:", (r.stdout + r.stderr)[-400:])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.rfo_quadrature.argtypes = [ctypes.c_int, _dp, _dp]
        L.rfo_legendre.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.rfo_analytic_moments.argtypes = [_dp, _dp, _dp, ctypes.c_int, _dp]
        L.rfo_assemble_system.argtypes = [ctypes.POINTER(RfoParams), _dp, _dp, _dp, _dp]
        L.rfo_assemble_rows.argtypes = [ctypes.POINTER(RfoParams), _dp, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.rfo_solve_direct.argtypes = [ctypes.c_int, _dp, _dp]
        L.rfo_solve_gmres.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, _ip, _dp, ctypes.c_int]
        L.rfo_matvec.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
        L.rfo_matvec.restype = None
        L.rfo_matvec_rect.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong, _dp, _dp, ctypes.c_int]
        L.rfo_matvec_rect.restype = None
        L.rfo_velocities.argtypes = [ctypes.POINTER(RfoParams), _dp, _dp, _dp, _dp, _dp]
        L.rfo_velocities_rows.argtypes = [ctypes.POINTER(RfoParams), _dp, _dp, _dp, ctypes.c_int,
                                          ctypes.c_int, _dp, _dp]
        L.rfo_sim_create.argtypes = [ctypes.POINTER(RfoParams), _dp, _dp]
        L.rfo_sim_create.restype = ctypes.c_void_p
        L.rfo_sim_destroy.argtypes = [ctypes.c_void_p]
        L.rfo_sim_step.argtypes = [ctypes.c_void_p]
        L.rfo_sim_last.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.rfo_sim_solve_info.argtypes = [ctypes.c_void_p, _ip, _ip, _dp]
        L.rfo_sim_timings.argtypes = [ctypes.c_void_p, _dp]
        L.rfo_sim_assemble_part.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.rfo_sim_finish_step.argtypes = [ctypes.c_void_p]
        L.rfo_generate_layout.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_ulonglong, _dp, _dp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_dp)


def make_params(M, N=5, NoQI=8, eps=0.01, dt=0.1, analytic=True, direct=False, restart=10,
                max_iters=100, tol=1e-5, ext_force=(0.0, 0.0, -1.0), threads=0):
    p = RfoParams()
    p.M, p.N, p.NoQI = M, N, NoQI
    p.analytic, p.direct = int(bool(analytic)), int(bool(direct))
    p.restart, p.max_iters, p.tol = restart, max_iters, tol
    p.eps, p.dt = eps, dt
    p.ext_force[:] = list(ext_force)
    p.threads = threads
    return p


def quadrature(NoQI):
    pv = np.zeros(3 * NoQI)
    wv = np.zeros(3 * NoQI)
    lib().rfo_quadrature(NoQI, _ptr(pv), _ptr(wv))
    return pv, wv


def analytic_moments(xb, pb, xbar, N):
    out = np.zeros(7 * (N + 1))
    xb, pb, xbar = (np.ascontiguousarray(v, dtype=np.float64) for v in (xb, pb, xbar))
    lib().rfo_analytic_moments(_ptr(xb), _ptr(pb), _ptr(xbar), N, _ptr(out))
    return out.reshape(7, N + 1)


def assemble_system(params, X, T):
    """Return (A column-major as an (n, n) Fortran-ordered array, b)."""
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
    n = 3 * params.N * params.M
    A = np.zeros((n, n), dtype=np.float64, order="F")
    b = np.zeros(n)
    rc = lib().rfo_assemble_system(ctypes.byref(params), _ptr(X), _ptr(T), _ptr(A), _ptr(b))
    assert rc == 0
    return A, b


def assemble_rows(params, X, T, i0, i1):
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
    n = 3 * params.N * params.M
    rows = 3 * params.N * (i1 - i0)
    A = np.zeros((rows, n), dtype=np.float64, order="F")
    b = np.zeros(rows)
    rc = lib().rfo_assemble_rows(ctypes.byref(params), _ptr(X), _ptr(T), i0, i1, _ptr(A), _ptr(b))
    assert rc == 0
    return A, b


def solve_direct(A, b):
    A2 = np.array(A, dtype=np.float64, order="F", copy=True)
    x = np.array(b, dtype=np.float64, copy=True)
    rc = lib().rfo_solve_direct(len(x), _ptr(A2), _ptr(x))
    assert rc == 0, rc
    return x


def solve_gmres(A, b, x0=None, restart=10, max_iters=100, tol=1e-5, threads=0):
    A = np.asfortranarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    it = ctypes.c_int(0)
    be = ctypes.c_double(0)
    info = lib().rfo_solve_gmres(len(b), _ptr(A), _ptr(b), _ptr(x), restart, max_iters, tol,
                                 ctypes.byref(it), ctypes.byref(be), threads)
    return x, info, it.value, be.value


def matvec(A, x, threads=0):
    A = np.asfortranarray(A, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    lib().rfo_matvec(len(x), _ptr(A), _ptr(x), _ptr(y), threads)
    return y


def matvec_rect(A, x, threads=0):
    A = np.asfortranarray(A, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(A.shape[0])
    lib().rfo_matvec_rect(A.shape[0], A.shape[1], _ptr(A), A.shape[0], _ptr(x), _ptr(y), threads)
    return y


def velocities(params, X, T, coeffs):
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    V = np.zeros(3 * params.M)
    W = np.zeros(3 * params.M)
    rc = lib().rfo_velocities(ctypes.byref(params), _ptr(X), _ptr(T), _ptr(c), _ptr(V), _ptr(W))
    assert rc == 0
    return V, W


def velocities_rows(params, X, T, coeffs, i0, i1):
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1)
    T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    V = np.zeros(3 * (i1 - i0))
    W = np.zeros(3 * (i1 - i0))
    rc = lib().rfo_velocities_rows(ctypes.byref(params), _ptr(X), _ptr(T), _ptr(c), i0, i1, _ptr(V), _ptr(W))
    assert rc == 0
    return V, W


def generate_layout(M, distribution="uniform", box=5.0, min_dist=0.2, seed=1000):
    """Seeded synthetic layout, bit-identical to the product's generator
    (centres uniform in [0, box)^3 or isotropic normal with deviation box,
    minimum centre distance by rejection, orientations uniform on the sphere)."""
    pos = np.zeros(3 * M)
    ori = np.zeros(3 * M)
    dist = {"uniform": 0, "gaussian": 1}[distribution]
    rc = lib().rfo_generate_layout(M, dist, box, min_dist, seed, _ptr(pos), _ptr(ori))
    if rc != 0:
        raise ValueError(f"invalid layout request: M={M} {distribution} box={box} min_dist={min_dist}")
    return pos.reshape(M, 3), ori.reshape(M, 3)


class Simulation:
    """Oracle time stepper: advect_fibers.f90:437-593 over any number of steps."""

    def __init__(self, params, X0, T0):
        self.params = params
        X0 = np.ascontiguousarray(X0, dtype=np.float64).reshape(-1)
        T0 = np.ascontiguousarray(T0, dtype=np.float64).reshape(-1)
        self._h = lib().rfo_sim_create(ctypes.byref(params), _ptr(X0), _ptr(T0))
        assert self._h

    def step(self):
        return lib().rfo_sim_step(self._h)

    def assemble_part(self, i0, i1):
        """Rows of the current step's system for target fibers [i0, i1)."""
        rc = lib().rfo_sim_assemble_part(self._h, i0, i1)
        assert rc == 0, rc
        return rc

    def finish_step(self):
        """Solve, velocities and advection of the system assembled by the parts."""
        return lib().rfo_sim_finish_step(self._h)

    def last(self):
        M, N = self.params.M, self.params.N
        n = 3 * N * M
        b, x = np.zeros(n), np.zeros(n)
        V, W, X, T = (np.zeros(3 * M) for _ in range(4))
        lib().rfo_sim_last(self._h, _ptr(b), _ptr(x), _ptr(V), _ptr(W), _ptr(X), _ptr(T))
        return dict(BVec=b, XVec=x, TRANSVel=V, ROTVel=W, POS=X, ORIENT=T)

    def solve_info(self):
        info, it, be = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        lib().rfo_sim_solve_info(self._h, ctypes.byref(info), ctypes.byref(it), ctypes.byref(be))
        return info.value, it.value, be.value

    def timings(self):
        t = np.zeros(4)
        lib().rfo_sim_timings(self._h, _ptr(t))
        return t

    def close(self):
        if self._h:
            lib().rfo_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
