"""Host-side checks of the C ABI library (no GPU needed)."""
import ctypes
import os

import numpy as np
import pytest

import rigidfibers_kth_b200 as rf
from rigidfibers_kth_b200 import _lib as L
from rigidfibers_kth_b200.simulation import _ptr


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = L.declared_symbols()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_default_matches_reference_run_file():
    p = L.RfParams()
    L.lib().rf_params_default(ctypes.byref(p))
    assert p.num_terms_in_force_expansion == 5 and p.num_quadrature_intervals == 8
    assert p.slenderness == 0.01 and p.timestep == 0.1
    assert p.gmres_restart == 10 and p.gmres_max_iters == 100 and p.gmres_tol == 1e-5
    assert list(p.external_force) == [0.0, 0.0, -1.0]
    assert p.pc_damping == 0.85
    assert ctypes.sizeof(L.RfParams) == 152
    assert ctypes.sizeof(L.RfSolveStats) == 48


def test_create_rejects_bad_arguments():
    lib = L.lib()
    pos, ori = np.zeros(6), np.array([0, 0, 1.0, 1.0, 0, 0])
    pos[3] = 3.0
    p = rf.FiberParams(num_fibers=2).to_c()
    h = ctypes.c_void_p()
    bad = []
    for field, val in [("num_terms_in_force_expansion", 9), ("num_quadrature_intervals", 0),
                       ("slenderness", 0.0), ("precision", 7), ("gmres_restart", 0), ("pc_damping", -0.5),
                       ("pc_damping", 2.5), ("pc_damping", float("nan"))]:
        q = rf.FiberParams(num_fibers=2).to_c()
        setattr(q, field, val)
        bad.append(lib.rf_create(ctypes.byref(q), _ptr(pos), _ptr(ori), ctypes.byref(h)))
    assert all(s == 1 for s in bad), bad
    nanpos = pos.copy()
    nanpos[0] = np.nan
    assert lib.rf_create(ctypes.byref(p), _ptr(nanpos), _ptr(ori), ctypes.byref(h)) == 6
    q = rf.FiberParams(num_fibers=0).to_c()
    assert lib.rf_create(ctypes.byref(q), _ptr(pos), _ptr(ori), ctypes.byref(h)) == 1
    assert b"num_fibers" in lib.rf_last_error(None)
    # one fiber is a valid system, but a block preconditioner needs neighbours
    q = rf.FiberParams(num_fibers=1, preconditioner=rf.PC_LEARNED).to_c()
    assert lib.rf_create(ctypes.byref(q), _ptr(pos), _ptr(ori), ctypes.byref(h)) == 1
    assert b"two fibers" in lib.rf_last_error(None)


def test_generator_deterministic_and_spaced():
    pos1, ori1 = rf.generate_layout(300, "uniform", 5.0, 0.2, seed=1002)
    pos2, ori2 = rf.generate_layout(300, "uniform", 5.0, 0.2, seed=1002)
    pos3, _ = rf.generate_layout(300, "uniform", 5.0, 0.2, seed=1003)
    assert np.array_equal(pos1, pos2) and np.array_equal(ori1, ori2)
    assert not np.array_equal(pos1, pos3)
    assert pos1.min() >= 0.0 and pos1.max() < 5.0
    d = np.linalg.norm(pos1[:, None, :] - pos1[None, :, :], axis=2)
    d[np.arange(300), np.arange(300)] = np.inf
    assert d.min() >= 0.2
    assert np.allclose(np.linalg.norm(ori1, axis=1), 1.0, atol=1e-14)
    # orientations roughly uniform: mean direction near zero
    assert np.abs(ori1.mean(axis=0)).max() < 0.15
    g, _ = rf.generate_layout(2000, "gaussian", 3.0, 0.2, seed=1004)
    assert abs(g.std() - 3.0) < 0.2


def test_min_segment_distance():
    pos = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.0], [10, 10, 10.0]])
    ori = np.array([[1.0, 0, 0], [1.0, 0, 0], [0, 0, 1.0]])
    assert abs(rf.min_segment_distance(pos, ori) - 0.5) < 1e-12
    pos = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.3]])
    ori = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    assert abs(rf.min_segment_distance(pos, ori) - 0.3) < 1e-12


def test_parameter_and_layout_files(tmp_path):
    run = tmp_path / "run_iter.in"
    run.write_text("2 !Label\n100 !file\n5 !N\n0.01 !eps\n0.1 !dt\n10 !steps\n1\n10\n8 !NoQI\n1 !an\n0 !gmres\n"
                   "10 !restart\n100 !maxit\n1e-5 !tol\n")
    p = rf.parse_parameter_file(str(run))
    assert (p.num_terms_in_force_expansion, p.num_quadrature_intervals, p.use_analytical_integration,
            p.use_direct_solver, p.gmres_restart, p.gmres_max_iters) == (5, 8, 1, 0, 10, 100)
    assert p.slenderness == 0.01 and p.gmres_tol == 1e-5
    pos, ori = rf.generate_layout(7, "uniform", 3.0, 0.2, seed=1)
    lay = tmp_path / "XcT_init7.in"
    rf.write_layout_file(str(lay), pos, ori)
    M, p2, o2 = rf.parse_layout_file(str(lay))
    assert M == 7 and np.allclose(p2, pos, atol=1e-15) and np.allclose(o2, ori, atol=1e-15)
    cfg = rf.parse_configuration_files(str(run), str(lay))
    assert cfg.parameters.num_fibers == 7


def test_direct_solver_needs_fp64():
    """The device LU is FP64 only: asking for it with a mixed precision is
    rejected before any device work (no GPU needed)."""
    pos, ori = rf.generate_layout(4, "uniform", 3.0, 0.2, seed=1)
    with pytest.raises(rf.RfError) as e:
        rf.Simulation(rf.Configuration(rf.FiberParams(use_direct_solver=1, precision=rf.PREC_MIXED_BF16), pos, ori))
    assert e.value.status == 1 and "RF_PREC_FP64" in str(e.value)


def test_dgesv_rejects_bad_arguments():
    """rf_dgesv checks its arguments before any device work."""
    lib = L.lib()
    A, b, x = np.eye(3), np.ones(3), np.zeros(3)
    info = ctypes.c_int32(-1)
    dp = ctypes.POINTER(ctypes.c_double)
    Ap, bp, xp = (v.ctypes.data_as(dp) for v in (A, b, x))
    assert lib.rf_dgesv(3, None, 3, bp, xp, None, ctypes.byref(info), 0) == 1  # RF_ERR_INVALID_ARG
    assert lib.rf_dgesv(3, Ap, 2, bp, xp, None, ctypes.byref(info), 0) == 1  # RF_ERR_INVALID_ARG
    assert lib.rf_dgesv(0, Ap, 3, bp, xp, None, ctypes.byref(info), 0) == 1  # RF_ERR_INVALID_ARG
    assert b"rf_dgesv" in lib.rf_last_error(None)


def test_create_without_gpu_fails_cleanly():
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("GPU present")
    pos, ori = rf.generate_layout(4, "uniform", 3.0, 0.2, seed=1)
    with pytest.raises(rf.RfError) as e:
        rf.Simulation(rf.Configuration(rf.FiberParams(), pos, ori))
    assert e.value.status == 7
