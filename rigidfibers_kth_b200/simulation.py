"""Host-side mirror of the reference's ``Simulation`` class and file formats.

The reference drives one simulation through ``Simulation(Configuration)`` and
``Simulation::step(current_timestep)``, which calls ``assembleSystem``,
``solveSystem``, ``updateVelocities`` and ``updateFibers(first_timestep)``
(src/simulation.h:36-87, src/simulation.cu:279-424).  ``Simulation`` here has
the same methods, backed by the C ABI of librigidfibers.so: every phase runs
in CUDA on the GPU, with host arrays copied in and out at the boundary.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


@dataclass
class FiberParams:
    """``FiberParams`` of src/common.h:49-68 plus the solver options of run*.in."""

    slenderness: float = 0.01
    timestep: float = 0.1
    num_fibers: int = 0
    num_timesteps: int = 10
    num_terms_in_force_expansion: int = 5
    num_quadrature_intervals: int = 8
    use_analytical_integration: int = 1
    use_direct_solver: int = 0
    gmres_restart: int = 10
    gmres_max_iters: int = 100
    gmres_tol: float = 1e-5
    external_force: tuple = (0.0, 0.0, -1.0)
    precision: int = L.PREC_FP64
    preconditioner: int = L.PC_NONE
    velocity_mode: int = L.VEL_RECOMPUTE
    device: int = 0
    max_refinements: int = 30
    cluster_size: int = 8
    inner_tol: float = 1e-3
    near_field_c: float = 6.0
    shard_index: int = 0
    shard_count: int = 1
    pc_damping: float = 0.85

    def to_c(self):
        p = L.RfParams()
        L.lib().rf_params_default(ctypes.byref(p))
        for name in (
            "slenderness", "timestep", "num_fibers", "num_timesteps", "num_terms_in_force_expansion",
            "num_quadrature_intervals", "use_analytical_integration", "use_direct_solver", "gmres_restart",
            "gmres_max_iters", "gmres_tol", "precision", "preconditioner", "velocity_mode", "device",
            "max_refinements", "cluster_size", "inner_tol", "near_field_c", "shard_index", "shard_count",
            "pc_damping",
        ):
            setattr(p, name, getattr(self, name))
        p.external_force[:] = list(self.external_force)
        return p


@dataclass
class Configuration:
    """``Configuration`` of src/parameters.h:27-31: parameters and the initial layout."""

    parameters: FiberParams
    initial_positions: np.ndarray
    initial_orientations: np.ndarray


def parse_parameter_file(path):
    """Positional v1 parameter file (src/parameters.cc:124-180; run100.in, run100_iter.in).

    Line 3 N, 4 eps, 5 dt, 6 steps, 9 NoQI, 10 analytic flag, 11 direct flag,
    and for GMRES 12 restart, 13 max iterations, 14 tolerance.
    """
    vals = []
    with open(path) as f:
        for line in f:
            tok = line.split("!")[0].split()
            vals.append(tok[0] if tok else None)
    p = FiberParams()
    p.num_terms_in_force_expansion = int(vals[2])
    p.slenderness = float(vals[3])
    p.timestep = float(vals[4])
    p.num_timesteps = int(vals[5])
    p.num_quadrature_intervals = int(vals[8])
    p.use_analytical_integration = int(vals[9])
    p.use_direct_solver = int(vals[10])
    if len(vals) > 13 and vals[11] is not None:
        p.gmres_restart = int(vals[11])
        p.gmres_max_iters = int(vals[12])
        p.gmres_tol = float(vals[13])
    return p


def parse_layout_file(path):
    """Layout file: M, then per fiber the centre and the orientation (3 numbers each).

    Both reference layouts read the same way: the CUDA parser takes two lines
    per fiber (src/parameters.cc:186-227), the Fortran driver a list-directed
    read of six numbers (fortran/advect_fibers.f90:318-321).
    """
    vals = open(path).read().split()
    M = int(vals[0])
    nums = np.array([float(v) for v in vals[1 : 1 + 6 * M]], dtype=np.float64).reshape(M, 6)
    return M, nums[:, 0:3].copy(), nums[:, 3:6].copy()


def write_layout_file(path, positions, orientations):
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    ori = np.asarray(orientations, dtype=np.float64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"{len(pos)}\n")
        for p, t in zip(pos, ori):
            f.write(f"{p[0]:.16f} {p[1]:.16f} {p[2]:.16f}\n{t[0]:.16f} {t[1]:.16f} {t[2]:.16f}\n")


def parse_configuration_files(parameters_filename, layout_filename):
    """``Parameters::parseConfigurationFiles`` (src/parameters.cc:24-43)."""
    params = parse_parameter_file(parameters_filename)
    M, pos, ori = parse_layout_file(layout_filename)
    params.num_fibers = M
    return Configuration(params, pos, ori)


def generate_layout(M, distribution="uniform", box=5.0, min_dist=0.2, seed=1000):
    """Seeded synthetic layout (C++ generator in the library).

    distribution "uniform": centres uniform in [0, box]^3; "gaussian":
    isotropic normal with standard deviation box.  Minimum centre distance by
    rejection; orientations uniform on the sphere.
    """
    pos = np.zeros(3 * M)
    ori = np.zeros(3 * M)
    dist = {"uniform": 0, "gaussian": 1}[distribution]
    L.check(L.lib().rf_generate_layout(M, dist, box, min_dist, seed, _ptr(pos), _ptr(ori)))
    return pos.reshape(M, 3), ori.reshape(M, 3)


def min_segment_distance(positions, orientations):
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
    ori = np.ascontiguousarray(orientations, dtype=np.float64).reshape(-1)
    return L.lib().rf_min_segment_distance(len(pos) // 3, _ptr(pos), _ptr(ori))


def shard_range(M, shard_count, shard_index):
    """Target fibers [t0, t1) of row-block shard `shard_index` of `shard_count`."""
    t0, t1 = ctypes.c_int32(), ctypes.c_int32()
    L.check(L.lib().rf_shard_range(M, shard_count, shard_index, ctypes.byref(t0), ctypes.byref(t1)))
    return t0.value, t1.value


def _load_torch_nccl():
    """Make the library use PyTorch's NCCL: the library loads NCCL at run time
    and reuses a copy already in the process; loading an older system copy
    first would break a later ``import torch`` in the same process."""
    try:
        import torch  # noqa: F401  (loads its NCCL with libtorch_cuda)
    except ImportError:
        pass


def shard_unique_id():
    """A new NCCL id (128 bytes) for the shards' communicator; made on one rank
    and sent to the others by the caller (e.g. torch.distributed)."""
    _load_torch_nccl()
    buf = ctypes.create_string_buffer(128)
    L.check(L.lib().rf_shard_unique_id(buf))
    return buf.raw


class Simulation:
    """Simulation(Configuration) with the reference's step API, on the GPU.

    With ``nccl_id`` (and the parameters' shard_index / shard_count) the
    handle is one row-block shard of a system split over GPUs, one process
    per GPU (rf_create_sharded: collective over the shards)."""

    def __init__(self, configuration, nccl_id=None, **overrides):
        if isinstance(configuration, FiberParams):
            raise TypeError("Simulation takes a Configuration (parameters + layout)")
        params = configuration.parameters
        for k, v in overrides.items():
            setattr(params, k, v)
        pos = np.ascontiguousarray(configuration.initial_positions, dtype=np.float64).reshape(-1)
        ori = np.ascontiguousarray(configuration.initial_orientations, dtype=np.float64).reshape(-1)
        params.num_fibers = len(pos) // 3
        self.params = params
        self.M = params.num_fibers
        self.N = params.num_terms_in_force_expansion
        self.n = 3 * self.N * self.M
        self._c = params.to_c()
        h = ctypes.c_void_p()
        if nccl_id is None:
            st = L.lib().rf_create(ctypes.byref(self._c), _ptr(pos), _ptr(ori), ctypes.byref(h))
        else:
            assert len(nccl_id) == 128
            _load_torch_nccl()
            st = L.lib().rf_create_sharded(ctypes.byref(self._c), _ptr(pos), _ptr(ori), bytes(nccl_id), ctypes.byref(h))
        L.check(st, None)
        self._h = h
        self.last_status = L.RF_OK

    # -- reference step API ------------------------------------------------
    def step(self, current_timestep):
        st = L.lib().rf_step(self._h, current_timestep)
        self.last_status = st
        if st not in (L.RF_OK, L.RF_ERR_NOT_CONVERGED):
            L.check(st, self._h)
        return st

    def assemble_system(self):
        L.check(L.lib().rf_assemble_system(self._h), self._h)

    def solve_system(self):
        st = L.lib().rf_solve_system(self._h)
        self.last_status = st
        if st not in (L.RF_OK, L.RF_ERR_NOT_CONVERGED):
            L.check(st, self._h)
        return st

    def update_velocities(self):
        L.check(L.lib().rf_update_velocities(self._h), self._h)

    def update_fibers(self, first_timestep):
        L.check(L.lib().rf_update_fibers(self._h, int(bool(first_timestep))), self._h)

    # camelCase aliases of the reference method names
    assembleSystem = assemble_system
    solveSystem = solve_system
    updateVelocities = update_velocities
    updateFibers = update_fibers

    # -- data access ---------------------------------------------------------
    def state(self):
        pos = np.zeros(3 * self.M)
        ori = np.zeros(3 * self.M)
        L.check(L.lib().rf_get_state(self._h, _ptr(pos), _ptr(ori)), self._h)
        return pos, ori

    def set_state(self, positions, orientations):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        ori = np.ascontiguousarray(orientations, dtype=np.float64).reshape(-1)
        L.check(L.lib().rf_set_state(self._h, _ptr(pos), _ptr(ori)), self._h)

    def velocities(self):
        v = np.zeros(3 * self.M)
        w = np.zeros(3 * self.M)
        L.check(L.lib().rf_get_velocities(self._h, _ptr(v), _ptr(w)), self._h)
        return v, w

    def coeffs(self):
        x = np.zeros(self.n)
        L.check(L.lib().rf_get_coeffs(self._h, _ptr(x)), self._h)
        return x

    def rhs(self):
        b = np.zeros(self.n)
        L.check(L.lib().rf_get_rhs(self._h, _ptr(b)), self._h)
        return b

    def matrix(self):
        A = np.zeros((self.n, self.n), order="F")
        L.check(L.lib().rf_get_matrix(self._h, _ptr(A)), self._h)
        return A

    def matrix_rows(self, row0, rows, inner=False):
        """Rows [row0, row0 + rows) of the stored matrix as an FP64 (rows, n)
        array; inner=True reads the inner solve's copy (BF16 where stored)."""
        A = np.zeros((rows, self.n), order="F")
        L.check(L.lib().rf_get_matrix_rows(self._h, int(bool(inner)), row0, rows, _ptr(A)), self._h)
        return A

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        L.check(L.lib().rf_matvec(self._h, _ptr(x), _ptr(y)), self._h)
        return y

    def matvec_free(self, x):
        """y = A x without forming A (the reference's mat_prod), FP64."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        L.check(L.lib().rf_matvec_free(self._h, _ptr(x), _ptr(y)), self._h)
        return y

    def solve_stats(self):
        s = L.RfSolveStats()
        L.check(L.lib().rf_get_solve_stats(self._h, ctypes.byref(s)), self._h)
        return dict(converged=bool(s.converged), iterations=s.iterations, matvecs=s.matvecs,
                    refinements=s.refinements, residual=s.residual, seconds=s.seconds,
                    pc_fallback=bool(s.pc_fallback), precision_fallback=bool(s.precision_fallback),
                    preconditioned=bool(s.preconditioned))

    def history(self):
        a = [np.zeros(3 * self.M) for _ in range(4)]
        L.check(L.lib().rf_get_history(self._h, *[_ptr(v) for v in a]), self._h)
        return a

    def set_history(self, prev_pos, prev_orient, prev_vel, prev_rot, coeffs):
        arrs = [np.ascontiguousarray(v, dtype=np.float64).reshape(-1) for v in
                (prev_pos, prev_orient, prev_vel, prev_rot, coeffs)]
        L.check(L.lib().rf_set_history(self._h, *[_ptr(v) for v in arrs]), self._h)

    def stream(self):
        return L.lib().rf_get_stream(self._h)

    def mark(self, slot):
        """Record device-time marker ``slot`` (0..15) on the handle's stream."""
        L.check(L.lib().rf_timer_mark(self._h, slot), self._h)

    def elapsed_ms(self, start, end):
        ms = L.lib().rf_timer_elapsed_ms(self._h, start, end)
        if ms < 0:
            raise RuntimeError("timer slots not recorded")
        return ms

    # -- learned / cluster preconditioner -------------------------------------
    def set_mlp_weights(self, weights):
        w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        fp = ctypes.POINTER(ctypes.c_float)
        L.check(L.lib().rf_set_mlp_weights(self._h, w.ctypes.data_as(fp), w.size), self._h)

    PAIRS = 8  # coupling blocks per fiber (RF_MLP_PAIRS)

    def features(self):
        """Pair features ((M * 8) x 144, fiber-major) of the current state in each fiber's frame."""
        f = np.zeros((self.M * self.PAIRS, 144), dtype=np.float32)
        L.check(L.lib().rf_compute_features(self._h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self._h)
        return f

    def cluster_targets(self):
        """Exact coupling blocks of the local-cluster inverses ((M * 8) x 225), in
        each fiber's frame with the neighbour's canonical sign; needs an assembled system."""
        t = np.zeros((self.M * self.PAIRS, 225), dtype=np.float32)
        L.check(L.lib().rf_compute_cluster_targets(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                self._h)
        return t

    def profile_matvec(self, reps=10):
        """(ms per product, bytes of A per product) of the inner-solve matvec."""
        ms, nbytes = ctypes.c_double(), ctypes.c_double()
        L.check(L.lib().rf_profile_matvec(self._h, reps, ctypes.byref(ms), ctypes.byref(nbytes)), self._h)
        return ms.value, nbytes.value

    def system_size(self):
        return L.lib().rf_system_size(self._h)

    def matrix_ld(self):
        """Leading dimension of the stored matrix (rows padded to 64)."""
        return L.lib().rf_matrix_ld(self._h)

    def gemv_timer(self, enable):
        """Start (True, counters reset) or stop live timing of the inner-solve
        products; returns (products timed, their total ms, bytes of A per product)."""
        cnt, ms, nbytes = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        L.check(L.lib().rf_gemv_timer(self._h, 1 if enable else 0, ctypes.byref(cnt), ctypes.byref(ms),
                                      ctypes.byref(nbytes)), self._h)
        return cnt.value, ms.value, nbytes.value

    def kernel_launches(self):
        return L.lib().rf_kernel_launches(self._h)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().rf_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
