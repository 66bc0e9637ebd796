"""Command-line driver: the reference's programs on this library.

    python -m rigidfibers_kth_b200 PARAMETERS LAYOUT [options]

Mirrors the two reference drivers.  The CUDA program ``fibers <parameters>
<layout>`` (src/main.cu:26-67, src/fiberopt.h) reads a positional parameter
file and a layout file and calls ``Simulation::step`` in a time loop; the
Fortran program (fortran/advect_fibers.f90:182-593) reads the same two files
and writes the trajectory and the per-step dumps.  Outputs, all optional:

  --dumps fortran  after each step BVec.out, XVec.out, TRANSVel.out,
                   ROTVel.out, POS.out, ORIENT.out (and AMat.out with
                   --matrix): F16.8, one value per line, a matrix row per line
                   (fortran/coeffs_and_vels.f90:420-436,524-529,733-745;
                   advect_fibers.f90:529-539).  The reference's golden vectors
                   (tests/reference/*/{step}_{Quantity}.ref) are these files;
                   --keep-steps writes them as {step}_{Quantity}.out instead
                   of overwriting.
  --dumps cuda     a_matrix.out (with --matrix), b_vector.out, x_vector.out,
                   positions.out, orientations.out, t_vel.out, r_vel.out:
                   fixed 8 decimals after five spaces (negative values) or six
                   (src/simulation.cu:426-603).
  --trajectory     XcTData<label>_p<k>, VelRotData<label>_p<k>,
                   Coeffvec<label>_p<k>: F24.16, one value per line, a blank
                   record after each 3-vector (advect_fibers.f90:394-424,
                   540-591).  The first record is the initial state with zero
                   velocities; a new file k starts every
                   save_interval * saves_per_file steps.  Unlike the Fortran,
                   which reopens the first coefficient file when it rolls over
                   (filename3 is never renamed), the coefficient file rolls
                   over with the other two.

The parameter file's solver settings apply: GMRES, or the device LU when
line 11 asks for the direct solver.  The LU is FP64 only; with a mixed or
FP32 precision a direct request is solved by GMRES to 1e-13 instead (which
agrees with the LU solution far below the printed precision).
"""
import argparse
import os
import sys
import time

import numpy as np

from . import _lib as L
from .simulation import Configuration, Simulation, parse_layout_file, parse_parameter_file

PRECISIONS = {"fp64": L.PREC_FP64, "fp32": L.PREC_FP32, "mixed-bf16": L.PREC_MIXED_BF16,
              "mixed-fp32": L.PREC_MIXED_FP32}
PRECONDITIONERS = {"none": L.PC_NONE, "cluster": L.PC_CLUSTER, "learned": L.PC_LEARNED}
VELOCITY_MODES = {"recompute": L.VEL_RECOMPUTE, "reuse": L.VEL_REUSE}


def run_labels(path):
    """Lines 1, 2, 7 and 8 of the positional parameter file: run label, layout
    label, save interval, saves per file (advect_fibers.f90:182-200)."""
    vals = []
    with open(path) as f:
        for line in f:
            tok = line.split("!")[0].split()
            vals.append(tok[0] if tok else None)

    def num(i, default):
        try:
            return int(vals[i])
        except (IndexError, TypeError, ValueError):
            return default

    return dict(label=num(0, 0), layout_label=num(1, 0), save_interval=max(1, num(6, 1)),
                saves_per_file=max(1, num(7, 10)))


def fmt_f16(v):
    """Fortran F16.8 (gfortran: right-justified, leading zero kept)."""
    return f"{v:16.8f}"


def fmt_f24(v):
    """Fortran F24.16."""
    return f"{v:24.16f}"


def fmt_cuda(v):
    """std::fixed << setprecision(8) after five spaces (v < 0) or six."""
    return ("     " if v < 0 else "      ") + f"{v:.8f}"


def write_column(path, values, fmt):
    with open(path, "w") as f:
        f.write("".join(fmt(v) + "\n" for v in values))


def write_matrix_rows(path, A, fmt, sep=""):
    """One line per row of A (column-major storage, printed by rows)."""
    with open(path, "w") as f:
        for row in np.asarray(A):
            f.write(sep.join(fmt(v) for v in row) + "\n")


def write_fortran_dumps(out, prefix, q, A=None):
    for name in ("BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT"):
        write_column(os.path.join(out, f"{prefix}{name}.out"), q[name], fmt_f16)
    if A is not None:
        write_matrix_rows(os.path.join(out, f"{prefix}AMat.out"), A, fmt_f16)


def write_cuda_dumps(out, q, A=None):
    for fname, name in (("b_vector.out", "BVec"), ("x_vector.out", "XVec"), ("positions.out", "POS"),
                        ("orientations.out", "ORIENT"), ("t_vel.out", "TRANSVel"), ("r_vel.out", "ROTVel")):
        write_column(os.path.join(out, fname), q[name], fmt_cuda)
    if A is not None:
        write_matrix_rows(os.path.join(out, "a_matrix.out"), A, fmt_cuda)


class TrajectoryWriter:
    """XcTData / VelRotData / Coeffvec files of the Fortran driver."""

    def __init__(self, out, label, save_interval, saves_per_file):
        self.out, self.label = out, label
        self.save_interval, self.saves_per_file = save_interval, saves_per_file
        self.part = 0
        self.files = None

    def _open(self):
        self.close()
        self.part += 1
        self.files = [open(os.path.join(self.out, f"{stem}{self.label}_p{self.part}"), "w")
                      for stem in ("XcTData", "VelRotData", "Coeffvec")]

    @staticmethod
    def _vectors(f, first, second):
        a = np.asarray(first).reshape(-1, 3)
        b = np.asarray(second).reshape(-1, 3)
        for u, w in zip(a, b):
            f.write("".join(fmt_f24(v) + "\n" for v in u) + "  \n")
            f.write("".join(fmt_f24(v) + "\n" for v in w) + "  \n")

    def initial(self, pos, ori):
        self._open()
        self._vectors(self.files[0], pos, ori)
        zero = np.zeros(np.asarray(pos).size)
        self._vectors(self.files[1], zero, zero)

    def after_step(self, tt, num_steps, pos, ori, vel, rot, coeffs):
        """tt = 1-based step number, called after the step's advection."""
        if tt % self.save_interval == 0:
            self._vectors(self.files[0], pos, ori)
            self._vectors(self.files[1], vel, rot)
            self.files[2].write("".join(fmt_f24(v) + "\n" for v in coeffs) + "  \n")
        if tt % (self.save_interval * self.saves_per_file) == 0 and tt < num_steps:
            self._open()

    def close(self):
        for f in self.files or ():
            f.close()
        self.files = None


def parse_args(argv=None):
    ap = argparse.ArgumentParser(prog="python -m rigidfibers_kth_b200",
                                 description="Rigid fibers in Stokes flow (the reference's parameter and layout files).")
    ap.add_argument("parameters", help="positional parameter file (run*.in)")
    ap.add_argument("layout", help="layout file (XcT_init*.in): M, then centre and orientation per fiber")
    ap.add_argument("--steps", type=int, default=None, help="time steps (default: the parameter file's)")
    ap.add_argument("--out", default=".", help="output directory")
    ap.add_argument("--dumps", choices=["none", "fortran", "cuda"], default="none")
    ap.add_argument("--matrix", action="store_true", help="also dump the n x n matrix (large)")
    ap.add_argument("--keep-steps", action="store_true", help="fortran dumps as {step}_{Quantity}.out")
    ap.add_argument("--trajectory", action="store_true", help="write the Fortran trajectory files")
    ap.add_argument("--precision", choices=sorted(PRECISIONS), default="fp64")
    ap.add_argument("--preconditioner", choices=sorted(PRECONDITIONERS), default="none")
    ap.add_argument("--velocities", choices=sorted(VELOCITY_MODES), default="recompute")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "mlp_weights.npy"),
                    help="MLP weights of the learned preconditioner")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--quiet", action="store_true")
    return ap.parse_args(argv)


def configuration(args):
    params = parse_parameter_file(args.parameters)
    M, pos, ori = parse_layout_file(args.layout)
    params.num_fibers = M
    notes = []
    params.precision = PRECISIONS[args.precision]
    if params.use_direct_solver and params.precision != L.PREC_FP64:
        params.use_direct_solver = 0
        params.gmres_tol = min(params.gmres_tol, 1e-13)
        params.gmres_max_iters = max(params.gmres_max_iters, 1000)
        notes.append("direct solver requested with a reduced precision: solved by GMRES to 1e-13 (the LU is FP64 only)")
    params.preconditioner = PRECONDITIONERS[args.preconditioner]
    params.velocity_mode = VELOCITY_MODES[args.velocities]
    params.device = args.device
    return Configuration(params, pos, ori), notes


def main(argv=None):
    args = parse_args(argv)
    cfg, notes = configuration(args)
    p = cfg.parameters
    labels = run_labels(args.parameters)
    steps = p.num_timesteps if args.steps is None else args.steps
    os.makedirs(args.out, exist_ok=True)
    say = (lambda *a: None) if args.quiet else (lambda *a: print(*a, flush=True))
    say(f"     [CPU]      : M = {p.num_fibers}, N = {p.num_terms_in_force_expansion}, eps = {p.slenderness}, "
        f"dt = {p.timestep}, NoQI = {p.num_quadrature_intervals}, "
        f"{'analytic' if p.use_analytical_integration else 'numeric'} integration, "
        f"GMRES({p.gmres_restart}) tol {p.gmres_tol:g} max {p.gmres_max_iters}, {steps} steps")
    for n in notes:
        say(f"     [CPU]      : {n}")
    traj = None
    with Simulation(cfg) as sim:
        if p.preconditioner == L.PC_LEARNED:
            sim.set_mlp_weights(np.load(args.weights))
        if args.trajectory:
            traj = TrajectoryWriter(args.out, labels["label"], labels["save_interval"], labels["saves_per_file"])
            traj.initial(*sim.state())
        phase_ms = np.zeros(4)
        t0 = time.perf_counter()
        try:
            for step in range(steps):
                say(f"     [CPU]      : Timestep {step + 1} of {steps}")
                sim.mark(0)
                sim.assemble_system()
                sim.mark(1)
                status = sim.solve_system()
                sim.mark(2)
                sim.update_velocities()
                sim.mark(3)
                if status == L.RF_ERR_NOT_CONVERGED:
                    say(f"     [GPU]      : GMRES did not converge in step {step + 1}")
                q = None
                if args.dumps != "none" or traj is not None:
                    vel, rot = sim.velocities()
                    q = dict(BVec=sim.rhs(), XVec=sim.coeffs(), TRANSVel=vel, ROTVel=rot)
                    A = sim.matrix() if args.matrix and args.dumps != "none" else None
                sim.update_fibers(step == 0)
                sim.mark(4)
                for k in range(4):
                    phase_ms[k] += sim.elapsed_ms(k, k + 1)
                if q is not None:
                    q["POS"], q["ORIENT"] = sim.state()
                    if args.dumps == "fortran":
                        write_fortran_dumps(args.out, f"{step}_" if args.keep_steps else "", q, A)
                    elif args.dumps == "cuda":
                        write_cuda_dumps(args.out, q, A)
                    if traj is not None:
                        traj.after_step(step + 1, steps, q["POS"], q["ORIENT"], q["TRANSVel"], q["ROTVel"],
                                        q["XVec"])
        finally:
            if traj is not None:
                traj.close()
        wall = time.perf_counter() - t0
    names = ("assemble_system", "solve_system", "update_velocities", "update_fibers")
    for name, ms in zip(names, phase_ms):
        say(f"     [GPU]      : {name:<18} {ms / max(steps, 1):10.3f} ms per step")
    say(f"     [CPU]      : {steps} steps in {wall:.3f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
