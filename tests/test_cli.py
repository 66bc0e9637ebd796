"""Command-line driver: file formats on the CPU, the golden runs on the GPU.

The reference's golden vectors are the Fortran program's per-step dumps
(F16.8, one value per line) renamed {step}_{Quantity}.ref; the driver writes
the same files, so the GPU test reads them back and compares them with the
golden values to the printed precision (two roundings of 5e-9 each plus the
path's own 5e-9 agreement)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import CASES, GOLDEN_ATOL, QUANTITIES, ROOT
from rigidfibers_kth_b200 import cli

RUN_FILE = """{label}     !Label of run
100  !Label of indata file
5     !Number of terms in the force expansion
0.01  !Size of epsilon
0.1   !Timestep
{steps}    !No. of timesteps
{save}     !Save interval
{per_file}    !Number of timesteps saved in one file
8     !Number of quad.intervals
{analytic}     !Using analytical integration 1 (0 numerical)
{direct}     !Using GMRES (1 direct solver)
10    !Restart parameter
100   !Max iter
1e-5  !Tolerance
"""


def write_inputs(tmp, pos, ori, analytic=1, direct=0, steps=2, label=2, save=1, per_file=10):
    run = tmp / "run.in"
    run.write_text(RUN_FILE.format(label=label, steps=steps, save=save, per_file=per_file, analytic=analytic,
                                   direct=direct))
    lay = tmp / "XcT_init.in"
    with open(lay, "w") as f:
        f.write(f"{len(pos)}\n")
        for p, t in zip(pos, ori):
            f.write(" ".join(f"{v:.17g}" for v in (*p, *t)) + "\n")
    return str(run), str(lay)


def read_values(path):
    with open(path) as f:
        return np.array([float(v) for v in f.read().split()])


def test_number_formats():
    assert cli.fmt_f16(0.43388838) == "      0.43388838"
    assert cli.fmt_f16(-0.96867518) == "     -0.96867518"
    assert len(cli.fmt_f16(-12.5)) == 16
    assert cli.fmt_f24(-1.25) == "     -1.2500000000000000"
    assert cli.fmt_cuda(-1.5) == "     -1.50000000"
    assert cli.fmt_cuda(12.25) == "      12.25000000"


def test_parameter_labels_and_direct_mapping(tmp_path):
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    ori = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    run, lay = write_inputs(tmp_path, pos, ori, direct=1, label=7, save=2, per_file=3)
    assert cli.run_labels(run) == dict(label=7, layout_label=100, save_interval=2, saves_per_file=3)
    args = cli.parse_args([run, lay, "--precision", "mixed-bf16", "--velocities", "reuse"])
    cfg, notes = cli.configuration(args)
    p = cfg.parameters
    assert p.num_fibers == 2 and p.use_direct_solver == 0 and p.gmres_tol == 1e-13 and len(notes) == 1
    assert p.precision == cli.PRECISIONS["mixed-bf16"] and p.velocity_mode == cli.VELOCITY_MODES["reuse"]


def test_trajectory_files_roll_over(tmp_path):
    M, n = 2, 30
    w = cli.TrajectoryWriter(str(tmp_path), 4, save_interval=1, saves_per_file=2)
    pos = np.arange(3 * M, dtype=float)
    w.initial(pos, pos)
    for tt in (1, 2, 3):
        w.after_step(tt, 3, pos + tt, pos, pos, pos, np.full(n, tt, dtype=float))
    w.close()
    rec = M * (3 + 1 + 3 + 1)  # per record: 3 lines, blank, 3 lines, blank per fiber
    lines = lambda name: open(tmp_path / name).read().splitlines()
    assert len(lines("XcTData4_p1")) == 3 * rec and len(lines("XcTData4_p2")) == rec
    assert len(lines("VelRotData4_p1")) == 3 * rec
    assert len(lines("Coeffvec4_p1")) == 2 * (n + 1) and len(lines("Coeffvec4_p2")) == n + 1
    assert read_values(tmp_path / "Coeffvec4_p2").tolist() == [3.0] * n
    first = read_values(tmp_path / "XcTData4_p1")[: 6 * M]
    assert np.array_equal(first[:3], pos[:3])
    assert not read_values(tmp_path / "VelRotData4_p1")[: 6 * M].any()
    assert lines("XcTData4_p1")[0] == cli.fmt_f24(0.0)


def test_fortran_dumps_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    q = {name: rng.standard_normal(12) for name in ("BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT")}
    A = rng.standard_normal((4, 4))
    cli.write_fortran_dumps(str(tmp_path), "0_", q, A)
    for name, v in q.items():
        assert np.abs(read_values(tmp_path / f"0_{name}.out") - v).max() <= 5e-9 + 1e-15
    rows = open(tmp_path / "0_AMat.out").read().splitlines()
    assert len(rows) == 4 and all(len(r) == 4 * 16 for r in rows)
    assert np.abs(read_values(tmp_path / "0_AMat.out").reshape(4, 4) - A).max() <= 5e-9 + 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_cli_reproduces_golden_dumps(golden, tmp_path, case):
    pos, ori = golden["layout_pos"], golden["layout_orient"]
    run, lay = write_inputs(tmp_path, pos, ori, analytic=int("analytic" in case), direct=int("direct" in case))
    out = tmp_path / "out"
    assert cli.main([run, lay, "--dumps", "fortran", "--keep-steps", "--out", str(out), "--quiet"]) == 0
    for step in (0, 1):
        for q in QUANTITIES:
            got = read_values(out / f"{step}_{q}.out")
            ref = golden[f"{case}/{step}_{q}"]
            assert got.shape == ref.shape
            assert np.abs(got - ref).max() <= 2 * GOLDEN_ATOL + 5e-9, (case, step, q)


@pytest.mark.gpu
def test_cli_module_entry_writes_trajectory(golden, tmp_path):
    pos, ori = golden["layout_pos"], golden["layout_orient"]
    run, lay = write_inputs(tmp_path, pos, ori, steps=3, label=5, save=1, per_file=2)
    out = tmp_path / "out"
    r = subprocess.run([sys.executable, "-m", "rigidfibers_kth_b200", run, lay, "--trajectory", "--dumps", "cuda",
                        "--out", str(out)], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "Timestep 3 of 3" in r.stdout
    M = len(pos)
    xct = read_values(out / "XcTData5_p1").reshape(3, M, 2, 3)  # initial, step 1, step 2
    unit = ori / np.linalg.norm(ori, axis=1, keepdims=True)
    assert np.abs(xct[0, :, 0] - pos).max() <= 1e-15
    assert min(np.abs(xct[0, :, 1] - ori).max(), np.abs(xct[0, :, 1] - unit).max()) <= 1e-15
    assert np.abs(xct[2, :, 0].ravel() - golden["100_analytic_gmres/1_POS"]).max() <= 2 * GOLDEN_ATOL
    last = read_values(out / "XcTData5_p2").reshape(M, 2, 3)  # step 3
    assert np.abs(read_values(out / "positions.out") - last[:, 0].ravel()).max() <= 5e-9 + 1e-15
    assert read_values(out / "Coeffvec5_p2").size == 15 * M
