"""The CPU oracle against the reference's own golden vectors (no GPU).

tests/reference/100_{analytic,numeric}_{direct,gmres}/{0,1}_*.ref of the
reference were written by its Fortran program (F16.8); the oracle must
reproduce all 48 of them to the printed precision.
"""
import numpy as np
import pytest

from conftest import CASES, GOLDEN_ATOL, QUANTITIES
from oracle import rfo


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_golden_two_steps(golden, case):
    X0, T0 = golden["layout_pos"], golden["layout_orient"]
    p = rfo.make_params(100, analytic="analytic" in case, direct="direct" in case)
    sim = rfo.Simulation(p, X0, T0)
    for step in (0, 1):
        assert sim.step() == 0
        out = sim.last()
        for q in QUANTITIES:
            ref = golden[f"{case}/{step}_{q}"]
            assert out[q].shape == ref.shape
            err = np.abs(out[q] - ref).max()
            assert err <= GOLDEN_ATOL, (case, step, q, err)
    if "gmres" in case:
        info, iters, be = sim.solve_info()
        assert info == 0 and 1 <= iters <= 100 and be <= 1e-5


def test_gmres_tight_matches_lu():
    rng = np.random.default_rng(3)
    n = 300
    A = np.eye(n) + 0.3 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    x_lu = rfo.solve_direct(A, b)
    x_gm, info, iters, be = rfo.solve_gmres(A, b, restart=10, max_iters=2000, tol=1e-13)
    assert info == 0
    assert np.abs(x_gm - x_lu).max() <= 1e-10 * np.abs(x_lu).max()
    assert np.allclose(x_lu, np.linalg.solve(A, b), rtol=1e-11, atol=1e-12)


def test_gmres_budget_reports_not_converged():
    rng = np.random.default_rng(4)
    n = 200
    A = np.eye(n) + 2.0 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    _, info, iters, be = rfo.solve_gmres(A, b, restart=5, max_iters=7, tol=1e-14)
    assert info == -4 and iters == 7 and be > 1e-14


def test_analytic_matches_fine_quadrature():
    """Int_analytical moments against brute-force quadrature of the same integrals."""
    rng = np.random.default_rng(5)
    s, w = np.polynomial.legendre.leggauss(400)
    for trial in range(20):
        xb = rng.uniform(-1, 1, 3)
        pb = rng.standard_normal(3)
        pb /= np.linalg.norm(pb)
        # target point at distance 0.5 .. 6 from the source centre, off-axis
        xbar = xb + rng.uniform(0.5, 6.0) * rng.standard_normal(3) / np.sqrt(3)
        N = 5
        L = rfo.analytic_moments(xb, pb, xbar, N)
        R0 = xbar - xb
        R = np.linalg.norm(R0[None, :] - s[:, None] * pb[None, :], axis=1)
        if R.min() < 0.3:
            continue
        # the Legendre combinations cancel: accuracy is relative to the
        # magnitude of the plain moments int 1/R^p; the reference's forward
        # recursion keeps about 11 of those digits at m = 5
        scale = np.array([np.sum(w / R), np.sum(w / R**3), np.sum(w / R**3), np.sum(w / R**3),
                          np.sum(w / R**5), np.sum(w / R**5), np.sum(w / R**5)])
        for m in range(N + 1):
            Pm = np.polynomial.legendre.Legendre.basis(m)(s)
            ref = np.array([np.sum(w * Pm / R), np.sum(w * Pm / R**3), np.sum(w * s * Pm / R**3),
                            np.sum(w * s * s * Pm / R**3), np.sum(w * Pm / R**5), np.sum(w * s * Pm / R**5),
                            np.sum(w * s * s * Pm / R**5)])
            err = np.abs(L[:, m] - ref)
            assert np.all(err <= 1e-10 * scale + 1e-9 * np.abs(ref)), (trial, m, err / scale)


def test_oracle_matvec_and_rows_consistent(golden):
    X0, T0 = golden["layout_pos"][:30], golden["layout_orient"][:30]
    T0 = T0 / np.linalg.norm(T0, axis=1, keepdims=True)
    p = rfo.make_params(30)
    A, b = rfo.assemble_system(p, X0, T0)
    rows, brows = rfo.assemble_rows(p, X0, T0, 7, 13)
    assert np.array_equal(rows, A[7 * 15 : 13 * 15, :])
    assert np.array_equal(brows, b[7 * 15 : 13 * 15])
    x = np.random.default_rng(0).standard_normal(A.shape[0])
    assert np.allclose(rfo.matvec(A, x), A @ x, rtol=1e-13, atol=1e-13)
    # the diagonal blocks are the identity (matrix_assembly.f90:489-492)
    for i in range(30):
        assert np.array_equal(A[i * 15 : (i + 1) * 15, i * 15 : (i + 1) * 15], np.eye(15))


def test_flop_count_of_the_reference_assembly():
    """oracle/count_flops.py: the counted work per ordered pair behind the
    assembly roofline (two sqrt and two log per Gauss point and 24 points)."""
    from oracle import count_flops

    fwd, bwd = count_flops.pair_cost(4.0), count_flops.pair_cost(40.0)
    assert fwd["sqrt"] == bwd["sqrt"] == 48 and fwd["log"] == bwd["log"] == 48
    assert bwd["div"] > fwd["div"]  # the backward recursion divides by c at every one of its 26 steps
    assert 2.5e4 < fwd["add"] + fwd["mul"] < bwd["add"] + bwd["mul"] < 4.0e4
    # the figure bench.py reports the assembly throughput against (6.9 % of the
    # Gauss points of the M = 4000 cloud in the forward-recursion range)
    import bench

    near = 0.069
    mixed = near * (fwd["add"] + fwd["mul"]) + (1 - near) * (bwd["add"] + bwd["mul"])
    assert abs(mixed - bench.ASM_FLOPS_PER_PAIR) < 1.0


@pytest.mark.parametrize("case", ["100_analytic_gmres", "100_numeric_direct"])
def test_step_in_parts_equals_whole_step(golden, case):
    """The CPU baseline times one whole step as row slices of the assembly
    followed by the rest of the step; the parts give the whole step's
    results bit for bit, over two steps (Euler, then multistep)."""
    X0, T0 = golden["layout_pos"], golden["layout_orient"]
    p = rfo.make_params(100, analytic="analytic" in case, direct="direct" in case)
    whole = rfo.Simulation(p, X0, T0)
    parts = rfo.Simulation(p, X0, T0)
    for step in (0, 1):
        assert whole.step() == 0
        for i0, i1 in [(0, 13), (13, 13), (13, 60), (60, 99), (99, 100)]:
            parts.assemble_part(i0, i1)
        assert parts.finish_step() == 0
        a, b = whole.last(), parts.last()
        for q in QUANTITIES:
            assert np.array_equal(a[q], b[q]), (step, q)
        for q in QUANTITIES:
            assert np.abs(b[q] - golden[f"{case}/{step}_{q}"]).max() <= GOLDEN_ATOL


def test_oracle_layout_matches_product_generator_bit_for_bit():
    """rfo.generate_layout (oracle side, used by the CPU baseline so that it
    never loads the product library) reproduces rf_generate_layout exactly,
    for both distributions and the benchmark configurations' seeds.  The
    product call is host code of librigidfibers.so: no GPU is needed."""
    import rigidfibers_kth_b200 as rf

    for M, dist, box, seed in [(100, "uniform", 2.5, 1001), (1000, "uniform", 5.0, 1002),
                               (2000, "uniform", 6.5, 1003), (4000, "gaussian", 3.0, 1004),
                               (8000, "uniform", 10.0, 1005), (333, "gaussian", 1.0, 7), (50, "uniform", 1.0, 0)]:
        po, oo = rfo.generate_layout(M, dist, box, 0.2, seed)
        pg, og = rf.generate_layout(M, dist, box, 0.2, seed)
        assert np.array_equal(po, pg) and np.array_equal(oo, og), (M, dist, seed)
        d = np.linalg.norm(po[:, None, :] - po[None, :, :], axis=2) if M <= 1000 else None
        if d is not None:
            assert d[~np.eye(M, dtype=bool)].min() >= 0.2
        assert np.allclose(np.linalg.norm(oo, axis=1), 1.0, atol=1e-15)
    with pytest.raises(ValueError):
        rfo.generate_layout(10**6, "uniform", 1.0, 0.2, 1)  # cannot be packed
