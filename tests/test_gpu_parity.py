"""CUDA path vs the CPU oracle and the reference's golden vectors (needs a B200).

Tolerances (stated by the method's contract):
  * FP64 path: 1e-10 relative to the oracle, norm-wise (largest absolute
    difference over the largest entry) for A, b, coefficients and velocities.
  * GMRES results at the golden tolerance (1e-5) reproduce the Fortran
    iterates: the golden vectors to their printed precision (5e-9).
  * Mixed / FP32 paths: velocities within 1e-6 of the FP64 result, relative to
    the largest velocity.
"""
import numpy as np
import pytest

import rigidfibers_kth_b200 as rf
from conftest import CASES, GOLDEN_ATOL, QUANTITIES
from oracle import rfo

pytestmark = pytest.mark.gpu

REL64 = 1e-10


def golden_layout(golden, M=100):
    X0 = golden["layout_pos"][:M]
    T0 = golden["layout_orient"][:M]
    return X0, T0 / np.linalg.norm(T0, axis=1, keepdims=True)


def make_sim(X, T, **kw):
    p = rf.FiberParams(**kw)
    return rf.Simulation(rf.Configuration(p, X, T))


def assert_close64(got, ref, what):
    """Norm-wise relative error max|got - ref| / max|ref| <= 1e-10.

    Entries of A that come from cancelling Legendre combinations (far pairs,
    high k and l) are tiny; their elementwise relative error says nothing
    about the system, so the tolerance is taken on the largest entry."""
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max() / scale
    assert np.isfinite(got).all(), what
    assert err <= REL64, (what, err)


@pytest.mark.parametrize("analytic", [1, 0])
def test_assembly_matches_oracle_fp64(golden, analytic):
    X, T = golden_layout(golden)
    with make_sim(X, T, use_analytical_integration=analytic) as sim:
        sim.assemble_system()
        A = sim.matrix()
        b = sim.rhs()
    A_o, b_o = rfo.assemble_system(rfo.make_params(100, analytic=bool(analytic)), X, T)
    assert_close64(A, A_o, "A")
    assert_close64(b, b_o, "b")


@pytest.mark.parametrize("case", [c for c in CASES])
def test_two_steps_match_golden(golden, case):
    """The golden vectors of all four reference runs, the direct-solver cases
    through the device LU (dgesv in the reference)."""
    X0, T0 = golden["layout_pos"], golden["layout_orient"]
    with make_sim(X0, T0, use_analytical_integration=int("analytic" in case),
                  use_direct_solver=int("direct" in case)) as sim:
        for step in (0, 1):
            sim.assemble_system()
            b = sim.rhs()
            assert sim.solve_system() == 0
            x = sim.coeffs()
            sim.update_velocities()
            V, W = sim.velocities()
            sim.update_fibers(step == 0)
            P, O = sim.state()
            out = dict(BVec=b, XVec=x, TRANSVel=V, ROTVel=W, POS=P, ORIENT=O)
            for q in QUANTITIES:
                err = np.abs(out[q] - golden[f"{case}/{step}_{q}"]).max()
                assert err <= GOLDEN_ATOL, (case, step, q, err)


@pytest.mark.parametrize("M", [100, 300])
def test_direct_solver_matches_oracle_lu(M):
    """Device LU with partial pivoting (panels of 64; n = 1500 and 4500, the
    last panel partial) against the oracle's LU (LAPACK dgesv's algorithm) of
    the same matrix: coefficients within 1e-10, the device's backward error at
    rounding level, and A left in place (the factors have their own buffer)."""
    pos, ori = rf.generate_layout(M, "uniform", 5.0 * (M / 300) ** (1 / 3), 0.2, seed=1900 + M)
    with make_sim(pos, ori, slenderness=1e-3, use_direct_solver=1) as sim:
        sim.assemble_system()
        A0 = sim.matrix()
        b = sim.rhs()
        assert sim.solve_system() == 0
        x = sim.coeffs()
        st = sim.solve_stats()
        A1 = sim.matrix()
        y = sim.matvec(x)
    assert st["converged"] and st["iterations"] == 0
    assert st["residual"] <= 1e-13
    assert np.linalg.norm(y - b) / np.linalg.norm(b) <= 1e-13
    assert np.array_equal(A0, A1)
    x_o = rfo.solve_direct(A0, b)
    assert np.abs(x - x_o).max() <= 1e-10 * np.abs(x_o).max()


def _dgesv(A, b, lda_pad=0):
    """rf_dgesv through the C ABI on a host copy of A with lda = n + lda_pad."""
    import ctypes

    from rigidfibers_kth_b200 import _lib as L

    n = len(b)
    Ah = np.zeros((n + lda_pad, n), order="F")
    Ah[:n, :] = A
    Ah[n:, :] = np.nan  # rows past n must never be read
    x = np.zeros(n)
    piv = np.zeros(n, dtype=np.int32)
    info = ctypes.c_int32(-1)
    dp = ctypes.POINTER(ctypes.c_double)
    st = L.lib().rf_dgesv(n, Ah.ctypes.data_as(dp), n + lda_pad, np.ascontiguousarray(b).ctypes.data_as(dp),
                          x.ctypes.data_as(dp), piv.ctypes.data, ctypes.byref(info), 0)
    L.check(st)
    assert np.all(np.isnan(Ah[n:, :])) and np.array_equal(Ah[:n, :], A)  # A left unchanged
    return x, piv, info.value


def test_dgesv_general_matrix_pivots_like_lapack():
    """The system matrices of fiber layouts are close to the identity and
    need no row interchange, so the device LU's pivot search and swaps are
    checked on general matrices: random N(0, 1) entries (a row interchange in
    almost every column), n = 777 (the last 64-column panel and 8-column
    sub-panel partial), padded leading dimension.  Pivots equal LAPACK's
    (scipy's dgetrf, 1-based), x matches the oracle's LU to 1e-10 and the
    backward error is at rounding level; a matrix with a zero column reports
    LAPACK's info."""
    import scipy.linalg as sl

    rng = np.random.default_rng(777)
    n = 777
    A = rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    x, piv, info = _dgesv(A, b, lda_pad=5)
    assert info == 0
    _, piv_ref = sl.lu_factor(A)
    assert np.sum(piv_ref != np.arange(n)) > n // 2  # pivoting really happens
    assert np.array_equal(piv, piv_ref + 1)
    x_o = rfo.solve_direct(A, b)
    assert np.abs(x - x_o).max() <= 1e-10 * np.abs(x_o).max()
    assert np.linalg.norm(A @ x - b) / (np.linalg.norm(A) * np.linalg.norm(x)) <= 1e-14
    A0 = A.copy()
    A0[:, 100] = 0.0
    _, _, info0 = _dgesv(A0, b)
    assert info0 == 101


@pytest.mark.parametrize("n", [1, 7, 8, 63, 64, 65, 130])
def test_dgesv_panel_edges(n):
    """Sizes at the edges of the 8-column sub-panels and 64-column panels
    (one column, a partial sub-panel, exactly one sub-panel or panel, one
    column more): pivots equal LAPACK's and x solves the system."""
    import scipy.linalg as sl

    rng = np.random.default_rng(1000 + n)
    A = rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    x, piv, info = _dgesv(A, b, lda_pad=3)
    assert info == 0
    assert np.array_equal(piv, sl.lu_factor(A)[1] + 1)
    x_ref = np.linalg.solve(A, b)
    assert np.abs(x - x_ref).max() <= 1e-10 * max(1.0, np.abs(x_ref).max())


def test_direct_solver_steps_match_gmres():
    """Three time steps with the LU and with GMRES at 1e-13 agree."""
    pos, ori = rf.generate_layout(200, "uniform", 4.0, 0.2, seed=1950)
    out = []
    for kw in (dict(use_direct_solver=1), dict(gmres_tol=1e-13, gmres_max_iters=2000)):
        with make_sim(pos, ori, slenderness=1e-3, **kw) as sim:
            for t in range(3):
                sim.step(t)
            out.append(sim.state() + sim.velocities())
    for a, b in zip(*out):
        assert np.abs(a - b).max() <= 1e-10 * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("layout", ["one", "near pair", "far pair"])
@pytest.mark.parametrize("path", ["fp64", "direct", "fp32", "mixed-bf16", "mixed-fp32"])
def test_one_and_two_fibers_every_path(layout, path):
    """The smallest systems through every solver path (one fiber: A = I,
    b = 0, only the local velocity term; two fibers 0.5 or 8 apart: one near
    or one far pair, a CTA whose other warps hold no target), two steps,
    against the oracle's velocities and positions of the same steps."""
    pos = {"one": [[0.0, 0.0, 0.0]], "near pair": [[0.0, 0.0, 0.0], [0.5, 0.1, 0.0]],
           "far pair": [[0.0, 0.0, 0.0], [8.0, 1.0, -2.0]]}[layout]
    ori = [[0.0, 0.6, 0.8], [1.0, 0.0, 0.0]][: len(pos)]
    pos, ori = np.array(pos), np.array(ori)
    kw = {"fp64": dict(gmres_tol=1e-13, gmres_max_iters=500), "direct": dict(use_direct_solver=1),
          "fp32": dict(precision=rf.PREC_FP32, gmres_tol=1e-6),
          "mixed-bf16": dict(precision=rf.PREC_MIXED_BF16, gmres_tol=1e-12, velocity_mode=rf.VEL_REUSE),
          "mixed-fp32": dict(precision=rf.PREC_MIXED_FP32, gmres_tol=1e-12)}[path]
    M = len(pos)
    o = rfo.Simulation(rfo.make_params(M, eps=1e-3, tol=1e-13, max_iters=500), pos, ori)
    tol = {"fp64": 1e-10, "direct": 1e-10, "fp32": 1e-4}.get(path, 1e-6)
    with make_sim(pos, ori, slenderness=1e-3, **kw) as sim:
        for t in range(2):
            assert sim.step(t) == 0
            o.step()
            ref = o.last()
            V, W = sim.velocities()
            P, T = sim.state()
            for got, want in ((V, ref["TRANSVel"]), (W, ref["ROTVel"]), (P, ref["POS"]), (T, ref["ORIENT"])):
                assert np.isfinite(got).all()
                assert np.abs(got - want).max() <= tol * max(1.0, np.abs(want).max()), (t, path, layout)
    o.close()


@pytest.mark.parametrize("analytic", [1, 0])
def test_matrix_free_product_matches_assembled_matrix(golden, analytic):
    """rf_matvec_free (mat_prod: A x without forming A) against the oracle's
    assembled matrix and against the handle's own stored FP64 matrix, for the
    analytic and the numeric inner integral; also from a mixed-precision
    handle, whose product is FP64 all the same."""
    X, T = golden_layout(golden)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(1500)
    with make_sim(X, T, use_analytical_integration=analytic) as sim:
        sim.assemble_system()
        y_stored = sim.matvec(x)
        y_free = sim.matvec_free(x)
    A_o, _ = rfo.assemble_system(rfo.make_params(100, analytic=bool(analytic)), X, T)
    y_o = A_o @ x
    assert_close64(y_free, y_o, "matrix-free vs oracle A x")
    assert_close64(y_free, y_stored, "matrix-free vs stored A x")
    with make_sim(X, T, use_analytical_integration=analytic, precision=rf.PREC_MIXED_BF16) as sim:
        y_mixed = sim.matvec_free(x)  # no assembly needed: the state alone defines A
    assert_close64(y_mixed, y_o, "matrix-free from a mixed handle")


def test_gmres_iterates_match_oracle(golden):
    """Same CERFACS control flow: same iteration counts, iterates within 1e-10."""
    X, T = golden_layout(golden)
    with make_sim(X, T, gmres_tol=1e-8, gmres_restart=5, gmres_max_iters=200) as sim:
        sim.assemble_system()
        sim.solve_system()
        x = sim.coeffs()
        st = sim.solve_stats()
    A_o, b_o = rfo.assemble_system(rfo.make_params(100), X, T)
    x_o, info, iters, be = rfo.solve_gmres(A_o, b_o, restart=5, max_iters=200, tol=1e-8)
    assert info == 0 and st["converged"]
    assert st["iterations"] == iters
    assert np.abs(x - x_o).max() <= 1e-10 * np.abs(x_o).max()


@pytest.mark.parametrize("analytic", [1, 0])
def test_velocities_match_oracle(golden, analytic):
    X, T = golden_layout(golden)
    with make_sim(X, T, use_analytical_integration=analytic, gmres_tol=1e-12, gmres_max_iters=500) as sim:
        sim.assemble_system()
        sim.solve_system()
        x = sim.coeffs()
        sim.update_velocities()
        V, W = sim.velocities()
    V_o, W_o = rfo.velocities(rfo.make_params(100, analytic=bool(analytic)), X, T, x)
    assert_close64(V, V_o, "V")
    assert_close64(W, W_o, "W")


def test_velocity_reuse_matches_recompute(golden):
    X, T = golden_layout(golden)
    out = {}
    for mode in (rf.VEL_RECOMPUTE, rf.VEL_REUSE):
        with make_sim(X, T, velocity_mode=mode, gmres_tol=1e-12, gmres_max_iters=500) as sim:
            sim.step(0)
            out[mode] = sim.velocities() + sim.state()
    for a, b in zip(out[rf.VEL_RECOMPUTE], out[rf.VEL_REUSE]):
        assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(a).max())


def oracle_sensitivity(p, pos, ori, return_perturbed=False):
    """How far the oracle moves A when its inputs move by one unit in the last
    place: the conditioning limit of the reference formulas on this layout.

    The analytic integral uses a forward recursion below c = 10
    (Int_analytical.f90:123-136) whose rounding errors grow with c and are then
    cancelled by the Legendre combinations; two correct FP64 evaluations of
    the reference formula (different libm log, summation order) agree only to
    this level."""
    pos2 = perturb_1ulp(pos)
    A1, _ = rfo.assemble_system(p, pos, ori)
    A2, _ = rfo.assemble_system(p, pos2, ori)
    sens = np.abs(A2 - A1).max() / np.abs(A1).max()
    return (sens, A1, pos2) if return_perturbed else (sens, A1)


def perturb_1ulp(pos, seed=0):
    """Every coordinate moved by about one unit in the last place, up or down."""
    rng = np.random.default_rng(seed)
    return pos * (1 + 2.2e-16 * rng.choice([-1, 1], pos.shape))


def test_random_layout_m300_fp64(golden):
    """Uniform cube, eps 1e-3: A within max(1e-10, 3x the oracle's own
    1-ulp sensitivity); coefficients and velocities within max(1e-10, 3x the
    oracle's 1-ulp sensitivity of its LU solution and of its velocities)."""
    pos, ori = rf.generate_layout(300, "uniform", 5.0, 0.2, seed=1002)
    with make_sim(pos, ori, slenderness=1e-3, gmres_tol=1e-12, gmres_max_iters=1000) as sim:
        sim.assemble_system()
        A = sim.matrix()
        b = sim.rhs()
        sim.solve_system()
        x = sim.coeffs()
        sim.update_velocities()
        V, W = sim.velocities()
    p = rfo.make_params(300, eps=1e-3)
    sens, A_o, pos2 = oracle_sensitivity(p, pos, ori, return_perturbed=True)
    _, b_o = rfo.assemble_system(p, pos, ori)
    errA = np.abs(A - A_o).max() / np.abs(A_o).max()
    assert errA <= max(REL64, 3 * sens), (errA, sens)
    assert_close64(b, b_o, "b")
    x_o = rfo.solve_direct(A_o, b_o)
    V_o, W_o = rfo.velocities(p, pos, ori, x_o)
    # the same chain from the perturbed inputs: the oracle's own spread
    A_2, b_2 = rfo.assemble_system(p, pos2, ori)
    x_2 = rfo.solve_direct(A_2, b_2)
    V_2, W_2 = rfo.velocities(p, pos2, ori, x_2)
    for got, ref, alt, what in ((x, x_o, x_2, "x"), (V, V_o, V_2, "V"), (W, W_o, W_2, "W")):
        spread = np.abs(alt - ref).max() / np.abs(ref).max()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= max(REL64, 3 * spread), (what, err, spread)


def test_well_separated_layout_fp64():
    """Sparse layout (no pair close to the recursion switch at high order):
    the 1e-10 contract holds outright."""
    pos, ori = rf.generate_layout(200, "uniform", 40.0, 3.0, seed=1010)
    with make_sim(pos, ori, slenderness=1e-3, gmres_tol=1e-13, gmres_max_iters=1000) as sim:
        sim.assemble_system()
        A, b = sim.matrix(), sim.rhs()
        sim.solve_system()
        x = sim.coeffs()
        sim.update_velocities()
        V, W = sim.velocities()
    p = rfo.make_params(200, eps=1e-3)
    A_o, b_o = rfo.assemble_system(p, pos, ori)
    assert_close64(A, A_o, "A")
    assert_close64(b, b_o, "b")
    x_o = rfo.solve_direct(A_o, b_o)
    assert_close64(x, x_o, "x")
    V_o, W_o = rfo.velocities(p, pos, ori, x_o)
    assert_close64(V, V_o, "V")
    assert_close64(W, W_o, "W")


@pytest.mark.parametrize("N,NoQI", [(1, 1), (3, 4), (8, 16), (5, 3)])
def test_expansion_and_quadrature_sizes(N, NoQI):
    pos, ori = rf.generate_layout(24, "uniform", 3.0, 0.2, seed=7)
    for analytic in (1, 0):
        with make_sim(pos, ori, num_terms_in_force_expansion=N, num_quadrature_intervals=NoQI,
                      use_analytical_integration=analytic) as sim:
            sim.assemble_system()
            A, b = sim.matrix(), sim.rhs()
        A_o, b_o = rfo.assemble_system(rfo.make_params(24, N=N, NoQI=NoQI, analytic=bool(analytic)), pos, ori)
        assert_close64(A, A_o, f"A N={N} NoQI={NoQI}")
        assert_close64(b, b_o, f"b N={N} NoQI={NoQI}")


def test_two_fibers_and_nearly_collinear_pairs():
    # two fibers almost on one axis and a perpendicular pair
    pos = np.array([[0.0, 0.0, 0.0], [1e-3, 0.0, 3.0], [4.0, 0.0, 0.0]])
    ori = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    with make_sim(pos, ori) as sim:
        sim.assemble_system()
        A, b = sim.matrix(), sim.rhs()
    A_o, b_o = rfo.assemble_system(rfo.make_params(3), pos, ori)
    assert_close64(A, A_o, "A nearly collinear")
    assert_close64(b, b_o, "b nearly collinear")


def test_exactly_collinear_fibers_report_nan():
    """A target point on the extension of a source fiber's axis puts log(0)
    into the reference formula (Int_analytical.f90:113); the reference and the
    oracle produce non-finite entries, the solve reports RF_ERR_NAN."""
    pos = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 3.0], [4.0, 0.0, 0.0]])
    ori = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    A_o, _ = rfo.assemble_system(rfo.make_params(3), pos, ori)
    assert not np.isfinite(A_o).all()
    with make_sim(pos, ori) as sim:
        sim.assemble_system()
        with pytest.raises(rf.RfError) as e:
            sim.solve_system()
        assert e.value.status == 6


def test_distant_pair_near_source_axis_mixed_path():
    """Two fibers 88 half-lengths apart, the target points within 1e-4 of the
    source fiber's axis (a pair met in a sedimenting cloud).  The reference's
    closed forms for the n = 0, 1 moments divide differences of O(1) terms by
    d = c - b^2/4, tiny here: in FP64 they lose all digits of S_1 and the
    block of this pair comes out as large as its true entries
    (Int_analytical.f90:162-196).  The mixed path integrates this far pair by
    the FP32 backward recursion alone, down to n = 0.  Truth: FP64 numeric
    integration (24-point composite Gauss rule over the source), exact to
    rounding for a source this far away.  Bound, on the largest deviation
    relative to the largest entry of A as elsewhere: 1e-8 (the blocks of this
    pair are 1.7e-7 at most; the FP32 far field deviates by 3e-10)."""
    p = np.array([0.00162206, 0.0257636, 0.99966675])
    t = np.array([0.00973097, 0.11302506, -0.99354449])
    pos = np.array([[0.0, 0.0, 0.0], 88.0 * p + np.array([0.0, 1e-4, 0.0]), [3.0, 0.0, 0.0]])
    ori = np.array([p, t, [1.0, 0.0, 0.0]])
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)

    def matrix(**kw):
        with make_sim(pos, ori, slenderness=1e-3, **kw) as s:
            s.assemble_system()
            return s.matrix().astype(np.float64)

    A_num = matrix(use_analytical_integration=0)
    A_mix = matrix(precision=rf.PREC_MIXED_FP32, velocity_mode=rf.VEL_REUSE)
    A_64 = matrix()
    scale = np.abs(A_num).max()
    n = 15  # 3N rows per fiber
    for ti, si in ((1, 0), (0, 1)):
        blk = (slice(n * ti, n * ti + n), slice(n * si, n * si + n))
        e_mix = np.abs(A_mix[blk] - A_num[blk]).max() / scale
        e_64 = np.abs(A_64[blk] - A_num[blk]).max() / scale
        assert e_mix <= 1e-8, (ti, si, e_mix, e_64)


def _fp64_reference(pos, ori, eps, tol=1e-12):
    with make_sim(pos, ori, slenderness=eps, gmres_tol=tol, gmres_max_iters=2000) as sim:
        sim.assemble_system()
        sim.solve_system()
        x = sim.coeffs()
        sim.update_velocities()
        V, W = sim.velocities()
    return x, V, W


def _split_layout(kind, M):
    if kind == "cloud":  # the sedimenting-cloud density of the M=4000 benchmark: many near pairs
        return rf.generate_layout(M, "gaussian", 3.0 * (M / 4000) ** (1 / 3), 0.2, seed=1700 + M)
    return rf.generate_layout(M, "uniform", 5.0 * (M / 1000) ** (1 / 3), 0.2, seed=1800 + M)


@pytest.mark.parametrize("kind", ["cloud", "uniform"])
@pytest.mark.parametrize("prec", [rf.PREC_MIXED_BF16, rf.PREC_FP32])
def test_split_assembly_matches_fp64_matrix(kind, prec):
    """FP32 far pairs + FP64 near pairs against the FP64 system, M not a multiple of 32.

    Entry-wise the FP32 storage alone rounds at 6e-8 of each entry; the bound is
    on the largest deviation relative to the largest entry.  The plain FP32
    method (PREC_FP32) integrates every pair in FP32, including the forward
    recursion of the moments near the source fiber, which amplifies FP32
    rounding by up to ~1e5 for nearly touching pairs; its bound only guards
    against gross errors (its velocities are checked against FP64 below).
    """
    M = 333
    pos, ori = _split_layout(kind, M)
    with make_sim(pos, ori, slenderness=1e-3) as s64:
        s64.assemble_system()
        A64, b64 = s64.matrix(), s64.rhs()
    with make_sim(pos, ori, slenderness=1e-3, precision=prec, velocity_mode=rf.VEL_REUSE) as s:
        s.assemble_system()
        A, b = s.matrix(), s.rhs()
    tol = 1e-6 if prec == rf.PREC_MIXED_BF16 else 5e-2
    err = np.abs(A - A64).max() / np.abs(A64).max()
    assert err <= tol, err
    eb = np.linalg.norm(b - b64) / np.linalg.norm(b64)
    assert eb <= tol, eb


@pytest.mark.parametrize("layout", ["uniform", "cloud"])
@pytest.mark.parametrize("vmode", [rf.VEL_RECOMPUTE, rf.VEL_REUSE])
@pytest.mark.parametrize("prec", [rf.PREC_MIXED_BF16, rf.PREC_MIXED_FP32])
def test_mixed_precision_velocity_error(prec, vmode, layout):
    if layout == "uniform":
        pos, ori = rf.generate_layout(400, "uniform", 5.0, 0.2, seed=1003)
    else:
        pos, ori = _split_layout("cloud", 400)
    x64, V64, W64 = _fp64_reference(pos, ori, 1e-3)
    with make_sim(pos, ori, slenderness=1e-3, precision=prec, gmres_tol=1e-10, gmres_max_iters=200,
                  velocity_mode=vmode) as sim:
        sim.assemble_system()
        assert sim.solve_system() == 0
        st = sim.solve_stats()
        x = sim.coeffs()
        sim.update_velocities()
        V, W = sim.velocities()
    assert st["refinements"] >= 1 and st["residual"] <= 1e-10
    ev = np.abs(V - V64).max() / np.abs(V64).max()
    ew = np.abs(W - W64).max() / np.abs(W64).max()
    assert ev <= 1e-6 and ew <= 1e-6, (ev, ew)


@pytest.mark.parametrize("N,NoQI", [(1, 8), (2, 4), (3, 8), (4, 6), (6, 8)])
def test_mixed_precision_other_expansion_orders(N, NoQI):
    """The split assembly for every expansion order it takes (N = 1..4 here,
    5 above; its far kernel stages 3N-row column segments whose bulk copies
    have N-dependent sizes) and the tile kernel's mixed mode beyond it
    (N = 6): BF16 storage with FP64 refinement, reuse velocities, against the
    FP64 path on a 200-fiber cloud (a ragged last warp of targets)."""
    pos, ori = _split_layout("cloud", 200)
    common = dict(slenderness=1e-3, num_terms_in_force_expansion=N, num_quadrature_intervals=NoQI)
    with make_sim(pos, ori, gmres_tol=1e-12, gmres_max_iters=1000, **common) as s64:
        s64.assemble_system()
        s64.solve_system()
        s64.update_velocities()
        V64, W64 = s64.velocities()
    with make_sim(pos, ori, precision=rf.PREC_MIXED_BF16, gmres_tol=1e-10, gmres_max_iters=300,
                  velocity_mode=rf.VEL_REUSE, **common) as sim:
        sim.assemble_system()
        assert sim.solve_system() == 0
        sim.update_velocities()
        V, W = sim.velocities()
    ev = np.abs(V - V64).max() / np.abs(V64).max()
    ew = np.abs(W - W64).max() / np.abs(W64).max()
    assert ev <= 1e-6 and ew <= 1e-6, (N, NoQI, ev, ew)


def test_fp32_variant():
    pos, ori = rf.generate_layout(300, "uniform", 5.0, 0.2, seed=1002)
    x64, V64, W64 = _fp64_reference(pos, ori, 1e-3)
    with make_sim(pos, ori, slenderness=1e-3, precision=rf.PREC_FP32, gmres_tol=1e-5) as sim:
        sim.assemble_system()
        assert sim.solve_system() == 0
        sim.update_velocities()
        V, W = sim.velocities()
    assert np.abs(V - V64).max() / np.abs(V64).max() <= 1e-4
    assert np.abs(W - W64).max() / np.abs(W64).max() <= 1e-3


def test_not_converged_status_and_state_still_advances(golden):
    X, T = golden_layout(golden)
    with make_sim(X, T, gmres_tol=1e-15, gmres_max_iters=3) as sim:
        st = sim.step(0)
        assert st == 4  # RF_ERR_NOT_CONVERGED
        s = sim.solve_stats()
        assert not s["converged"] and s["iterations"] == 3
        P, _ = sim.state()
        assert np.isfinite(P).all()


@pytest.mark.parametrize("pc", [rf.PC_NONE, rf.PC_LEARNED])
def test_mixed_not_converged_status_and_state_still_advances(golden, pc):
    """The mixed path with a refinement budget too small for the tolerance:
    the step reports RF_ERR_NOT_CONVERGED with the reached residual, the state
    still advances, and the next step runs."""
    import os

    X, T = golden_layout(golden)
    with make_sim(X, T, gmres_tol=1e-10, precision=rf.PREC_MIXED_BF16, velocity_mode=rf.VEL_REUSE,
                  max_refinements=1, preconditioner=pc) as sim:
        if pc == rf.PC_LEARNED:
            sim.set_mlp_weights(np.load(os.path.join(os.path.dirname(rf.__file__), "mlp_weights.npy")))
        assert sim.step(0) == 4  # RF_ERR_NOT_CONVERGED
        s = sim.solve_stats()
        assert not s["converged"] and s["refinements"] == 1 and 1e-10 < s["residual"] < 1e-2
        P, _ = sim.state()
        assert np.isfinite(P).all()
        assert sim.step(1) == 4
        assert np.isfinite(sim.state()[0]).all()


def test_checkpoint_resume_matches_uninterrupted(golden):
    X, T = golden_layout(golden, 60)
    kw = dict(gmres_tol=1e-10, gmres_max_iters=300)
    with make_sim(X, T, **kw) as a:
        for s in range(3):
            a.step(s)
        ref = a.state()
    with make_sim(X, T, **kw) as b:
        b.step(0)
        pos, ori = b.state()
        hist = b.history()
        x = b.coeffs()
    with make_sim(pos, ori, **kw) as c:
        c.set_history(*hist, x)
        c.step(1)
        c.step(2)
        got = c.state()
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-11


@pytest.mark.parametrize("prec", [rf.PREC_MIXED_BF16, rf.PREC_MIXED_FP32])
def test_mixed_precision_error_every_step_m2000(prec):
    """M = 2000 fibers in a cube of side 6.5, 50 steps of the mixed path (BF16
    or FP32 storage, FP64 refinement to 1e-10).  At every step the velocities
    and coefficients are compared with an FP64 solve of the same state: the
    velocity error stays within 1e-6 of the largest velocity over the run.
    The coefficient bound is looser: the FP32 rounding of A is amplified by the
    conditioning of the state (fibers of this cloud touch: minimum segment
    distance 0), and at one step of this run (t = 42, FP32 storage) the FP64
    solve itself is off by 2e-5: an ejected fiber 88 half-lengths below lies
    on another fiber's axis, where the reference's closed-form moments lose
    their digits (test_distant_pair_near_source_axis_mixed_path)."""
    M, steps = 2000, 50
    pos, ori = rf.generate_layout(M, "uniform", 6.5, 0.2, seed=1003)
    mixed = make_sim(pos, ori, slenderness=1e-3, precision=prec, gmres_tol=1e-10, gmres_max_iters=300,
                     velocity_mode=rf.VEL_REUSE)
    ref = make_sim(pos, ori, slenderness=1e-3, gmres_tol=1e-12, gmres_max_iters=2000)
    worst_v, worst_x = 0.0, (0.0, -1)
    try:
        for t in range(steps):
            mixed.assemble_system()
            assert mixed.solve_system() == 0
            mixed.update_velocities()
            V, W = mixed.velocities()
            x = mixed.coeffs()
            P, T = mixed.state()
            ref.set_state(P, T)
            ref.assemble_system()
            ref.solve_system()
            ref.update_velocities()
            V64, W64 = ref.velocities()
            x64 = ref.coeffs()
            ev = max(np.abs(V - V64).max() / np.abs(V64).max(), np.abs(W - W64).max() / np.abs(W64).max())
            ex = np.abs(x - x64).max() / np.abs(x64).max()
            worst_v = max(worst_v, ev)
            worst_x = max(worst_x, (ex, t))
            assert ev <= 1e-6, (t, ev)
            mixed.update_fibers(t == 0)
    finally:
        mixed.close()
        ref.close()
    assert worst_x[0] <= 1e-4, worst_x


# ---------------------------------------------------------------- the benchmark configurations
def test_config1_trajectory_fp64_matches_oracle():
    """Configuration 1 as specified (M = 100, centres uniform in a cube of
    side 2.5 by seeded rejection with minimum distance 0.2, eps 1e-3, N = 5,
    8 x 3 Gauss points, dt 0.1, Euler then multistep, GMRES(10) to 1e-10):
    the whole 10-step FP64 trajectory against the oracle's.

    Tolerance per quantity and step: max(1e-10, 3 x the spread between the
    oracle's trajectory and the oracle's trajectory from initial positions
    moved by one unit in the last place).  This layout is dense (fibers of
    length 2 at centre distance 0.2), so the forward recursion of the
    reference formula near c = 10 amplifies rounding and two correct FP64
    evaluations agree only to that spread."""
    pos, ori = rf.generate_layout(100, "uniform", 2.5, 0.2, seed=1001)
    p = rfo.make_params(100, eps=1e-3, dt=0.1, max_iters=300, tol=1e-10)
    o1 = rfo.Simulation(p, pos, ori)
    o2 = rfo.Simulation(p, perturb_1ulp(pos), ori)
    worst = {}
    with make_sim(pos, ori, slenderness=1e-3, timestep=0.1, gmres_tol=1e-10, gmres_max_iters=300) as sim:
        for step in range(10):
            sim.assemble_system()
            assert sim.solve_system() == 0
            x = sim.coeffs()
            sim.update_velocities()
            V, W = sim.velocities()
            sim.update_fibers(step == 0)
            P, O = sim.state()
            assert o1.step() == 0 and o2.step() == 0
            r1, r2 = o1.last(), o2.last()
            got = dict(XVec=x, TRANSVel=V, ROTVel=W, POS=P, ORIENT=O)
            for q, v in got.items():
                scale = np.abs(r1[q]).max()
                spread = np.abs(r2[q] - r1[q]).max() / scale
                err = np.abs(v - r1[q]).max() / scale
                tol = max(REL64, 3 * spread)
                assert err <= tol, (step, q, err, spread)
                worst[q] = max(worst.get(q, 0.0), err)
    print("configuration 1, worst norm-wise error over 10 steps:", worst)


CONFIG_LAYOUTS = {
    # configuration 2: M = 1000, uniform cube of side 5; configuration 4: the
    # M = 4000 cloud (isotropic Gaussian centres, sigma 3); both seeded as the
    # benchmark runs them
    "cfg2": (1000, "uniform", 5.0, 1002),
    "cfg4": (4000, "gaussian", 3.0, 1004),
}


def _sample_targets(M):
    return [(0, 8), (M // 2 - 4, M // 2 + 4), (M - 8, M)]


@pytest.mark.parametrize("cfg", ["cfg2", "cfg4"])
def test_config_matrix_rows_fp64_match_oracle(cfg):
    """The FP64 assembly (one CTA per target tile) at the benchmark's own
    sizes: rows of 24 target fibers (first, middle, last: every source) and the
    whole right-hand side against the oracle, A within max(1e-10, 3 x the
    oracle's 1-ulp sensitivity on the same rows), b within 1e-10."""
    M, dist, box, seed = CONFIG_LAYOUTS[cfg]
    pos, ori = rf.generate_layout(M, dist, box, 0.2, seed=seed)
    p = rfo.make_params(M, eps=1e-3)
    pos2 = perturb_1ulp(pos)
    n3 = 15
    with make_sim(pos, ori, slenderness=1e-3) as sim:
        sim.assemble_system()
        b = sim.rhs()
        for i0, i1 in _sample_targets(M):
            A = sim.matrix_rows(i0 * n3, (i1 - i0) * n3)
            A_o, b_o = rfo.assemble_rows(p, pos, ori, i0, i1)
            A_2, _ = rfo.assemble_rows(p, pos2, ori, i0, i1)
            scale = np.abs(A_o).max()
            sens = np.abs(A_2 - A_o).max() / scale
            err = np.abs(A - A_o).max() / scale
            assert err <= max(REL64, 3 * sens), (cfg, i0, err, sens)
            eb = np.abs(b[i0 * n3:i1 * n3] - b_o).max() / np.abs(b_o).max()
            assert eb <= REL64, (cfg, i0, eb)


@pytest.mark.parametrize("cfg", ["cfg2", "cfg4"])
def test_config_matrix_rows_split_kernel_match_oracle(cfg):
    """The split mixed-precision assembly (FP32 far pairs, FP64 near pairs) at
    the benchmark's sizes against the oracle on the same sampled rows: the FP32
    matrix (the refinement residual's) within 1e-6 of max|A|, the BF16 copy
    (the inner solve's) within BF16 rounding of each entry (2^-8 relative, the
    FP32 deviation on top), b within 1e-6 of max|b|."""
    M, dist, box, seed = CONFIG_LAYOUTS[cfg]
    pos, ori = rf.generate_layout(M, dist, box, 0.2, seed=seed)
    p = rfo.make_params(M, eps=1e-3)
    n3 = 15
    with make_sim(pos, ori, slenderness=1e-3, precision=rf.PREC_MIXED_BF16, velocity_mode=rf.VEL_REUSE) as sim:
        sim.assemble_system()
        b = sim.rhs()
        for i0, i1 in _sample_targets(M):
            A32 = sim.matrix_rows(i0 * n3, (i1 - i0) * n3)
            A16 = sim.matrix_rows(i0 * n3, (i1 - i0) * n3, inner=True)
            A_o, b_o = rfo.assemble_rows(p, pos, ori, i0, i1)
            scale = np.abs(A_o).max()
            err32 = np.abs(A32 - A_o).max() / scale
            assert err32 <= 1e-6, (cfg, i0, err32)
            excess = np.abs(A16 - A_o) - (2.0 ** -8 * np.abs(A_o) + 1e-6 * scale)
            assert excess.max() <= 0.0, (cfg, i0, excess.max() / scale)
            assert not np.array_equal(A16, A32)  # the inner copy really is the rounded one
            # b sums M far contributions evaluated in FP32 per entry, which cancel
            # for some targets: the largest deviation relative to the largest
            # entry of b, as for A
            eb = np.abs(b[i0 * n3:i1 * n3] - b_o).max() / np.abs(b).max()
            assert eb <= 1e-6, (cfg, i0, eb)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["cloud", "uniform"])
def test_split_storage_rebuilds_the_fp32_matrix_exactly(kind):
    """The BF16 path stores its FP32 matrix as two 16-bit planes.  The FP32
    entries rebuilt from them equal, bit for bit, those the FP32 mixed path
    stores as FP32 words (the same assembly kernels), and the high plane is
    the top half of each FP32 word rounded half away from zero."""
    M = 600
    if kind == "cloud":
        pos, ori = rf.generate_layout(M, "gaussian", 3.0 * (M / 4000) ** (1 / 3), 0.2, seed=1720)
    else:
        pos, ori = rf.generate_layout(M, "uniform", 4.0, 0.2, seed=1721)
    rows = {}
    for prec in (rf.PREC_MIXED_BF16, rf.PREC_MIXED_FP32):
        p = rf.FiberParams(slenderness=1e-3, precision=prec, velocity_mode=rf.VEL_REUSE)
        with rf.Simulation(rf.Configuration(p, pos, ori)) as sim:
            sim.assemble_system()
            n = sim.n
            rows[prec] = [sim.matrix_rows(r0, 45) for r0 in (0, n // 2 - 45, n - 45)]
            if prec == rf.PREC_MIXED_BF16:
                hi = [sim.matrix_rows(r0, 45, inner=True) for r0 in (0, n // 2 - 45, n - 45)]
    for a, b, h in zip(rows[rf.PREC_MIXED_BF16], rows[rf.PREC_MIXED_FP32], hi):
        assert np.array_equal(a, b)
        u = a.astype(np.float32).view(np.uint32)
        want = ((u + np.uint32(0x8000)) >> np.uint32(16)).astype(np.uint32) << np.uint32(16)
        assert np.array_equal(h.astype(np.float32).view(np.uint32), want)
