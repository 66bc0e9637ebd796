#!/usr/bin/env python
"""Time steps/s of the rigid-fiber step at M=4000 (clustered sedimenting cloud).

Workload (one "step" = assemble -> solve -> velocities -> advect of the whole
suspension): M = 4000 fibers, centres isotropic Gaussian sigma 3 with minimum
centre distance 0.2 (seed 1004), orientations uniform on the sphere, half
length 1, eps = 1e-3, N = 5 Legendre terms, 8 x 3 Gauss points, dt = 0.1,
gravity (0,0,-1) per fiber, GMRES restart 10, FP64 residual tolerance 1e-10.
Synthetic, seeded data; no dataset is involved.

Arms:
  default            the product path: BF16-stored A for the inner GMRES (FP32
                     accumulation), FP64-residual iterative refinement against
                     the FP32-stored A, block preconditioner, velocities from
                     the stored projection panels.  The plain FP64 GPU path
                     (the reference method unchanged) is timed in the same run
                     for the speed-up and the velocity error.
  --impl reference   the CPU implementation of the path (the FP64 oracle, an
                     OpenMP restatement of the reference Fortran, which cannot
                     be built here: no Fortran compiler) on all host threads:
                     the timed iterations are the parts of ONE whole time step
                     of the workload (row slices of the assembly, then the
                     GMRES solve, velocities and advection), so their summed
                     time is a measured step; nothing is extrapolated.  It
                     never loads the product library.
  --impl reference-gpu
                     the reference's own CUDA program (oracle/_ref/fibers_gpu,
                     built unmodified from its sources) on the only case it is
                     compiled for, the M=100 golden case, beside this
                     library's plain FP64 path on the same case.  Not the
                     benchmark workload: the program's sizes are compile-time
                     constants.

Multi-GPU: every rank runs an independent replica (the reference has no
parallelism beyond one device); value = steps of all ranks / max time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s at M=4000 fibers: BF16+FP64-refine+learned vs plain FP64 GPU, ≤1e-6 err"
WORKLOAD = dict(M=4000, distribution="gaussian", box=3.0, min_dist=0.2, seed=1004, eps=1e-3, N=5, NoQI=8, dt=0.1,
                restart=10, tol=1e-10)
# FP64 GMRES matrix-vector products per step on this workload (the CPU sample
# cannot solve the full 60000 x 60000 system in a bounded time; the count is
# the one the same GMRES takes on it, from the FP64 run of this benchmark).
FP64_MATVECS_PER_STEP = 26
L2_BYTES = 126 * 1024 * 1024
# DRAM bytes (read + write) per stored element of A of one BF16 product, from
# an ncu capture of the product at M = 1000 (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch over 15040 x 15000 stored elements);
# scaled to the workload's matrix size (the traffic grows with the elements
# streamed)
TRAFFIC_PER_ELEMENT = (451.270656e6 + 7.171840e6) / (15040 * 15000)
# Algorithmic work of the assembly: add and multiply flops per ordered fiber
# pair of the reference formulas (FMA = 2), counted by the oracle's flop
# counter on this workload's initial layout (6.9 % of the Gauss points in the
# forward-recursion range); FP32 CUDA-core nominal peak of the B200 (148 SMs x
# 128 lanes x 2 flops x 1.965 GHz) for the split assembly, whose far field is FP32
ASM_FLOPS_PER_PAIR = 34916.0
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12

# The other configurations of the benchmark (seeded synthetic layouts; half
# length 1, eps 1e-3, N = 5, 8 x 3 Gauss points, gravity (0,0,-1), minimum
# centre distance 0.2).  Each arm runs the configuration's whole trajectory
# from the initial layout; the velocity error is taken against an FP64 solve
# (tol 1e-12) of the same state at the listed steps (1-based).  Arms: (name,
# precision, GMRES tolerance, preconditioner, velocities).
CONFIGS = {
    1: dict(M=100, distribution="uniform", box=2.5, seed=1001, dt=0.1, steps=10, check=(1, 10),
            arms=[("fp64", "PREC_FP64", 1e-10, "PC_NONE", "VEL_RECOMPUTE")]),
    2: dict(M=1000, distribution="uniform", box=5.0, seed=1002, dt=0.1, steps=100, check=(1, 50, 100),
            arms=[("fp64", "PREC_FP64", 1e-10, "PC_NONE", "VEL_RECOMPUTE"),
                  ("fp32", "PREC_FP32", 1e-5, "PC_NONE", "VEL_RECOMPUTE")]),
    3: dict(M=2000, distribution="uniform", box=6.5, seed=1003, dt=0.1, steps=50, check=tuple(range(1, 51)),
            arms=[("bf16+fp64-refine", "PREC_MIXED_BF16", 1e-10, "PC_NONE", "VEL_REUSE"),
                  ("fp32+fp64-refine", "PREC_MIXED_FP32", 1e-10, "PC_NONE", "VEL_REUSE")]),
    5: dict(M=8000, distribution="uniform", box=10.0, seed=1005, dt=0.05, steps=100, check=(1, 50, 100),
            arms=[("bf16+fp64-refine+learned", "PREC_MIXED_BF16", 1e-10, "PC_LEARNED", "VEL_REUSE"),
                  ("fp32", "PREC_FP32", 1e-5, "PC_NONE", "VEL_RECOMPUTE")]),
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    ap.add_argument("--M", type=int, default=WORKLOAD["M"], help="override the number of fibers (smoke runs)")
    ap.add_argument("--precision", choices=["bf16", "fp32"], default="bf16")
    ap.add_argument("--pc", choices=["learned", "cluster", "none"], default="learned")
    ap.add_argument("--weights", default=os.path.join(ROOT, "rigidfibers_kth_b200", "mlp_weights.npy"))
    ap.add_argument("--pc-damping", type=float, default=None,
                    help="damping of the preconditioner's coupling blocks (default: the library's)")
    ap.add_argument("--near-c", type=float, default=None,
                    help="squared distance below which a pair's integrals stay FP64 (default: the library's, 6; "
                         "smaller values are raised to 6)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4, 5], default=4,
                    help="workload: 4 = the M=4000 benchmark (default); 1, 2, 3, 5 = the other configurations, each "
                         "run over its whole trajectory from the initial layout (CONFIGS)")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_setup(timeout_s=300):
    """One process per GPU (torchrun env); NCCL with GPUs, gloo without (CPU tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            backend = "nccl"
        else:
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- workload description
def workload_config(M, world):
    """The `config` of the JSON line: the workload only, identical for the
    product arm and the reference arm (what each arm runs is under `arm`)."""
    n = 3 * WORKLOAD["N"] * M
    return {
        "workload": f"M={M} fibers, clustered cloud (Gaussian centres sigma {WORKLOAD['box']}, min centre "
                    f"distance {WORKLOAD['min_dist']}, seed {WORKLOAD['seed']}), eps {WORKLOAD['eps']}, "
                    f"N={WORKLOAD['N']}, 8x3 Gauss points, dt {WORKLOAD['dt']}, GMRES({WORKLOAD['restart']}) to an "
                    f"FP64 residual of {WORKLOAD['tol']}",
        "system": f"{n} x {n} dense",
        "l2": "inputs larger than L2 (FP64 A {:.1f} GB, BF16 A {:.1f} GB)".format(n * n * 8e-9, n * n * 2e-9),
        "parallelism": f"replicas x{world}",
    }


# ---------------------------------------------------------------- product arm
# block damping (FiberParams.pc_damping) of the preconditioned arms; None: the library's default
PC_DAMPING = None
# near-pair threshold (FiberParams.near_field_c) of the mixed arms; None: the library's default
NEAR_C = None


def make_sim(rf, pos, ori, device, precision, pc, velocity_mode, tol=WORKLOAD["tol"]):
    p = rf.FiberParams(slenderness=WORKLOAD["eps"], timestep=WORKLOAD["dt"],
                       num_terms_in_force_expansion=WORKLOAD["N"], num_quadrature_intervals=WORKLOAD["NoQI"],
                       gmres_restart=WORKLOAD["restart"], gmres_tol=tol, gmres_max_iters=300,
                       precision=precision, preconditioner=pc, velocity_mode=velocity_mode, device=device)
    if PC_DAMPING is not None:
        p.pc_damping = PC_DAMPING
    if NEAR_C is not None:
        p.near_field_c = NEAR_C
    return rf.Simulation(rf.Configuration(p, pos, ori))


def timed_steps(sim, steps, warmup, world, first_index=0, collect_stats=False):
    """Device time of `steps` steps after `warmup` untimed ones (marker 0 -> 1).
    Returns (ms, kernel launches or the per-step solve statistics, next step index)."""
    t = first_index
    for _ in range(warmup):
        sim.step(t)
        t += 1
    barrier(world)
    launches0 = sim.kernel_launches()
    stats = []
    sim.mark(0)
    for _ in range(steps):
        sim.step(t)
        if collect_stats:
            stats.append(sim.solve_stats())
        t += 1
    sim.mark(1)
    ms = sim.elapsed_ms(0, 1)
    launches = sim.kernel_launches() - launches0
    barrier(world)
    return ms, (stats if collect_stats else launches), t


def read_only_bandwidth(device, gib=4, reps=5):
    """HBM bandwidth of a read-only stream on this GPU: a reduction over a
    buffer far larger than L2 (torch's sum kernel), best of `reps`, CUDA
    events.  The product kernels only read A, so this is the ceiling they
    are compared with beside the measured copy bandwidth."""
    try:
        import torch

        x = torch.ones(gib * (1 << 28), dtype=torch.float32, device=f"cuda:{device}")
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        best = None
        for _ in range(reps + 1):
            s.record()
            x.sum()
            e.record()
            e.synchronize()
            ms = s.elapsed_time(e)
            best = ms if best is None else min(best, ms)
        del x
        torch.cuda.empty_cache()
        return gib * (1 << 30) / (best * 1e-3) / 1e9
    except Exception:
        return None


def phase_breakdown(sim, t, steps=5):
    """Device time of each phase of a step (assembly, solve, velocities,
    advection), averaged over `steps` steps from step index t (the solve's
    iterations vary from step to step).  Returns the phases and the
    velocities of the first of these steps."""
    acc = np.zeros(4)
    vel = None
    for i in range(steps):
        sim.mark(2)
        sim.assemble_system()
        sim.mark(3)
        sim.solve_system()
        sim.mark(4)
        sim.update_velocities()
        sim.mark(5)
        sim.update_fibers(t + i == 0)
        sim.mark(6)
        acc += [sim.elapsed_ms(2, 3), sim.elapsed_ms(3, 4), sim.elapsed_ms(4, 5), sim.elapsed_ms(5, 6)]
        if i == 0:
            vel = sim.velocities()
    acc /= steps
    return dict(assemble=float(acc[0]), solve=float(acc[1]), velocities=float(acc[2]), advect=float(acc[3]),
                steps_averaged=steps), vel


def cpu_baseline_sample(pos, ori, matvecs):
    """Oracle (OpenMP FP64 restatement of the reference Fortran) on a bounded
    sample: the rows of S target fibers for assembly and velocities (all 4000
    sources) and `matvecs` products with those rows; scaled by M/S."""
    from oracle import rfo

    M = len(pos)
    S = max(1, min(M, 200 * M // 4000))
    p = rfo.make_params(M, N=WORKLOAD["N"], NoQI=WORKLOAD["NoQI"], eps=WORKLOAD["eps"], dt=WORKLOAD["dt"])
    t0 = time.perf_counter()
    A, _ = rfo.assemble_rows(p, pos, ori, 0, S)
    t1 = time.perf_counter()
    x = np.ones(A.shape[1]) * 1e-3
    for _ in range(matvecs):
        rfo.matvec_rect(A, x)
    t2 = time.perf_counter()
    rfo.velocities_rows(p, pos, ori, np.zeros(A.shape[1]), 0, S)
    t3 = time.perf_counter()
    sample_s = t3 - t0
    step_s = sample_s * M / S
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"rows of {S} of {M} target fibers: assembly {t1 - t0:.2f}s, {matvecs} FP64 row matvecs "
                      f"{t2 - t1:.2f}s, velocities {t3 - t2:.2f}s; scaled by M/S = {M / S:.0f}"}


def run_ours(args):
    world, rank, local = dist_setup()
    import rigidfibers_kth_b200 as rf

    M = args.M
    pos, ori = rf.generate_layout(M, WORKLOAD["distribution"], WORKLOAD["box"], WORKLOAD["min_dist"],
                                  seed=WORKLOAD["seed"] + rank)
    prec = rf.PREC_MIXED_BF16 if args.precision == "bf16" else rf.PREC_MIXED_FP32
    pc = {"none": rf.PC_NONE, "cluster": rf.PC_CLUSTER, "learned": rf.PC_LEARNED}[args.pc]
    sim = make_sim(rf, pos, ori, local, prec, pc, rf.VEL_REUSE)
    if pc == rf.PC_LEARNED:
        sim.set_mlp_weights(np.load(args.weights))
    clocks = ClockSampler(local)
    # warm-up, then the timed region with clock sampling
    t = 0
    for _ in range(args.warmup):
        sim.step(t)
        t += 1
    barrier(world)
    clocks.start()
    launches0 = sim.kernel_launches()
    sim.gemv_timer(True)   # events around every inner-solve product of the timed region
    sim.mark(0)
    stats = []
    for _ in range(args.steps):
        sim.step(t)
        stats.append(sim.solve_stats())
        t += 1
    sim.mark(1)
    ms = sim.elapsed_ms(0, 1)
    gemv_count, gemv_ms, gemv_bytes = sim.gemv_timer(False)
    launches = sim.kernel_launches() - launches0
    clk = clocks.stop()
    barrier(world)
    ms = max_over_ranks(ms, world)
    value = world * args.steps / (ms * 1e-3)

    # the state after every timed step; the first phase step below computes its velocities
    P_end, O_end = sim.state()
    t_end = t
    phases, (V_end, W_end) = phase_breakdown(sim, t)
    t += phases["steps_averaged"]
    mv_ms, mv_bytes = sim.profile_matvec(reps=10)
    matrix_ld = sim.matrix_ld()
    solve_stats = stats[-1]
    sim.close()

    # end to end through the public API with host buffers, over the same step
    # window from the same initial layout: W untimed steps, then K steps that
    # each upload the state, step, and download the velocities and the state
    sim = make_sim(rf, pos, ori, local, prec, pc, rf.VEL_REUSE)
    if pc == rf.PC_LEARNED:
        sim.set_mlp_weights(np.load(args.weights))
    te = 0
    for _ in range(args.warmup):
        sim.step(te)
        te += 1
    hp, ho = sim.state()
    hp = np.ascontiguousarray(hp)
    ho = np.ascontiguousarray(ho)
    barrier(world)
    sim.mark(7)
    for _ in range(args.steps):
        sim.set_state(hp, ho)
        sim.step(te)
        te += 1
        v, w = sim.velocities()
        hp, ho = sim.state()
    sim.mark(8)
    e2e_ms = max_over_ranks(sim.elapsed_ms(7, 8), world)
    e2e_value = world * args.steps / (e2e_ms * 1e-3)
    sim.close()

    out = None
    if rank == 0:
        # the comparison arms on the same workload and the same step window
        # (W untimed steps from the initial layout, then K timed steps)
        plain = None
        pc_none = None
        verr = None
        window = {"warmup_steps": args.warmup, "timed_steps": args.steps}
        if not args.no_plain:
            # plain FP64 GPU path: the reference method unchanged
            sim64 = make_sim(rf, pos, ori, local, rf.PREC_FP64, rf.PC_NONE, rf.VEL_RECOMPUTE)
            ms64, _, t64 = timed_steps(sim64, args.steps, args.warmup, 1)
            plain = {"value": args.steps / (ms64 * 1e-3), "unit": "steps/s", "ms_per_step": ms64 / args.steps,
                     "window": window}
            plain["phases_ms"] = phase_breakdown(sim64, t64)[0]
            plain["matvecs_per_step"] = sim64.solve_stats()["matvecs"]
            sim64.close()
            # the product path without a block preconditioner (the learned
            # blocks' fallback: the diagonal blocks of A are the identity)
            if pc != rf.PC_NONE:
                simn = make_sim(rf, pos, ori, local, prec, rf.PC_NONE, rf.VEL_REUSE)
                msn, its_n, tn = timed_steps(simn, args.steps, args.warmup, 1, collect_stats=True)
                ph_n = phase_breakdown(simn, tn)[0]
                simn.close()
                pc_none = {"value": args.steps / (msn * 1e-3), "unit": "steps/s", "ms_per_step": msn / args.steps,
                           "window": window, "mean_inner_iterations": float(np.mean([s["iterations"] for s in its_n])),
                           "mean_products": float(np.mean([s["matvecs"] for s in its_n])),
                           "solve_ms_phase_steps": ph_n["solve"]}
            # velocity error of the product path against an FP64 solve (tol
            # 1e-12) of the same state: the initial layout and the state after
            # all timed steps
            ref = make_sim(rf, pos, ori, local, rf.PREC_FP64, rf.PC_NONE, rf.VEL_RECOMPUTE, tol=1e-12)
            ref.assemble_system(); ref.solve_system(); ref.update_velocities()
            V64, W64 = ref.velocities()
            chk = make_sim(rf, pos, ori, local, prec, pc, rf.VEL_REUSE)
            if pc == rf.PC_LEARNED:
                chk.set_mlp_weights(np.load(args.weights))
            chk.assemble_system(); chk.solve_system(); chk.update_velocities()
            V, W = chk.velocities()
            chk.close()
            ref.set_state(P_end, O_end)
            ref.assemble_system(); ref.solve_system(); ref.update_velocities()
            V64e, W64e = ref.velocities()
            ref.close()

            def rel(a, b):
                return float(np.abs(a - b).max() / np.abs(b).max())

            verr = {"translational": max(rel(V, V64), rel(V_end, V64e)),
                    "rotational": max(rel(W, W64), rel(W_end, W64e)),
                    "initial_state": {"translational": rel(V, V64), "rotational": rel(W, W64)},
                    "after_timed_steps": {"translational": rel(V_end, V64e), "rotational": rel(W_end, W64e),
                                          "step": t_end},
                    "bound": 1e-6, "norm": "max over fibers / max |FP64 velocity| of the same state"}
        iters = [s["iterations"] for s in stats]
        learned = {"mean_inner_iterations": float(np.mean(iters)),
                   "mean_products": float(np.mean([s["matvecs"] for s in stats])),
                   "solve_ms_phase_steps": phases["solve"],
                   "steps_not_converged": sum(int(not s["converged"]) for s in stats),
                   "fallbacks_to_no_preconditioner": sum(int(s["pc_fallback"]) for s in stats),
                   "steps_preconditioned": sum(int(s["preconditioned"]) for s in stats)}
        # roofline of the dominant kernel: the inner-solve product (BF16 A), timed
        # live over the timed region with events on the handle's stream
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        per_launch = gemv_ms / max(1, gemv_count)
        achieved = gemv_bytes / (per_launch * 1e-3) / 1e9 if gemv_count else None
        n_el = float(matrix_ld) * 3 * WORKLOAD["N"] * M
        read_peak = read_only_bandwidth(local)
        roof = {"bound": "hbm", "kernel": "gemv_partial_kernel + gemv_reduce_kernel (BF16 A x FP32 x)",
                "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak if achieved else None,
                "traffic": TRAFFIC_PER_ELEMENT * n_el if TRAFFIC_PER_ELEMENT else None,
                "peak_source": ("measured copy bandwidth (read + write bytes of a device copy; a read-only stream "
                                "such as the product can exceed it)") if "hbm_gbs" in peaks else "fallback",
                "read_only_peak": read_peak,
                "frac_of_read_only": achieved / read_peak if (achieved and read_peak) else None,
                "algorithmic_bytes": gemv_bytes, "ms_per_launch": per_launch, "launches_timed": gemv_count,
                "share_of_timed_region": gemv_ms / ms,
                "isolated_ms_per_launch": mv_ms}
        cpu = None if args.no_cpu else cpu_baseline_sample(pos, ori, FP64_MATVECS_PER_STEP)
        n = 3 * WORKLOAD["N"] * M
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bf16+fp32+fp64",
            "data": "synthetic",
            "config": workload_config(M, world),
            "arm": {"precision": args.precision + " A (inner GMRES) + FP32 A (FP64-accumulated residual) + FP64 "
                                 "refinement", "preconditioner": args.pc,
                    "pc_damping": PC_DAMPING if PC_DAMPING is not None else "library default",
                    "near_field_c": NEAR_C if NEAR_C is not None else "library default",
                    "velocities": "stored P0/P1 projection panels"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 2 * 3 * M * 8,
                    "d2h_bytes_per_step": 4 * 3 * M * 8},
            "gpu_launches": int(launches),
            "clocks": clk,
            "phases_ms": phases,
            "solve": solve_stats,
            "preconditioner": {args.pc: learned, "none": pc_none},
            "plain_fp64": plain,
            "speedup_vs_plain_fp64": (value / world) / plain["value"] if plain else None,
            "velocity_error": verr,
            "assembly": {"ms": phases["assemble"], "counted_tflop": ASM_FLOPS_PER_PAIR * M * (M - 1) / 1e12,
                         "achieved_tflops": ASM_FLOPS_PER_PAIR * M * (M - 1) / 1e12 / (phases["assemble"] * 1e-3),
                         "peak_tflops": FP32_NOMINAL_TFLOPS, "peak_source": "FP32 CUDA-core nominal",
                         "frac": ASM_FLOPS_PER_PAIR * M * (M - 1) / 1e12 / (phases["assemble"] * 1e-3)
                         / FP32_NOMINAL_TFLOPS,
                         # the matrix (BF16 with FP32 storage: two 16-bit planes, 4 bytes per
                         # entry; FP32 storage alone: 4) and the two FP32 velocity panels
                         "written_gb": (3 * WORKLOAD["N"] * M) * 1.0 * (3 * WORKLOAD["N"] * M) * 4e-9
                         + 2 * 3 * M * (3 * WORKLOAD["N"] * M) * 4e-9,
                         "note": "split assembly (classify, near, far, finish), mean of the phase steps; counted work of "
                                 "the reference formulas at the initial layout"},
        }
    sim.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return out


# ---------------------------------------------------------------- other configurations
def config_sim(rf, cfg, pos, ori, device, precision, tol, pc, velocity_mode):
    p = rf.FiberParams(slenderness=1e-3, timestep=cfg["dt"], num_terms_in_force_expansion=5,
                       num_quadrature_intervals=8, gmres_restart=10, gmres_tol=tol,
                       gmres_max_iters=300 if tol >= 1e-10 else 2000, precision=precision, preconditioner=pc,
                       velocity_mode=velocity_mode, device=device)
    if PC_DAMPING is not None:
        p.pc_damping = PC_DAMPING
    if NEAR_C is not None:
        p.near_field_c = NEAR_C
    return rf.Simulation(rf.Configuration(p, pos, ori))


def run_config(args):
    """One configuration of the benchmark other than the M=4000 headline: every
    arm over the whole trajectory (device time of all steps, events on the
    handle's stream), the roofline of its matrix-vector products (timed live),
    the velocity error at the configuration's check steps against FP64, and the
    CPU oracle on the same layout (full steps at M=100, the bounded row sample
    otherwise)."""
    world, rank, local = dist_setup()
    import rigidfibers_kth_b200 as rf

    cfg = CONFIGS[args.config]
    M, steps = cfg["M"], cfg["steps"]
    pos, ori = rf.generate_layout(M, cfg["distribution"], cfg["box"], 0.2, seed=cfg["seed"] + rank)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    arms, checks = {}, {}
    clocks = ClockSampler(local)
    clocks.start()
    for name, prec, tol, pc, vel in cfg["arms"]:
        sim = config_sim(rf, cfg, pos, ori, local, getattr(rf, prec), tol, getattr(rf, pc), getattr(rf, vel))
        if pc == "PC_LEARNED":
            sim.set_mlp_weights(np.load(args.weights))
        barrier(world)
        sim.gemv_timer(True)
        launches0 = sim.kernel_launches()
        total_ms, iters, saved, failed, unconverged, fallbacks, preconditioned = 0.0, [], [], None, 0, 0, 0
        for t in range(steps):
            pre = sim.state() if (t + 1) in cfg["check"] else None
            sim.mark(0)
            try:
                sim.step(t)
            except rf.RfError as e:  # reported in the arm's entry; the other arms still run
                failed = f"step {t + 1}: {e}"
                break
            sim.mark(1)
            total_ms += sim.elapsed_ms(0, 1)
            ss = sim.solve_stats()
            iters.append(ss["iterations"])
            unconverged += int(not ss["converged"])
            fallbacks += int(ss["pc_fallback"])
            preconditioned += int(ss["preconditioned"])
            if pre is not None:
                saved.append((t + 1, pre, sim.velocities()))
        count, gms, gbytes = sim.gemv_timer(False)
        launches = sim.kernel_launches() - launches0
        sim.close()
        barrier(world)
        total_ms = max_over_ranks(total_ms, world)
        per = gms / max(count, 1)
        ach = gbytes / (per * 1e-3) / 1e9 if count else None
        done = len(iters)
        arms[name] = {"value": world * done / (total_ms * 1e-3) if done else None, "unit": "steps/s",
                      "ms_per_step": total_ms / done if done else None, "steps_completed": done, "failed": failed,
                      "gmres_tol": tol, "mean_iterations": float(np.mean(iters)) if iters else None,
                      "max_iterations": int(max(iters)) if iters else None,
                      "steps_not_converged": unconverged, "preconditioner_fallbacks": fallbacks,
                      "steps_preconditioned": preconditioned,
                      "gpu_launches": int(launches),
                      "products": {"bytes": gbytes, "ms_per_launch": per, "launches": count, "achieved_gbs": ach,
                                   "frac": ach / hbm_peak if ach else None,
                                   "share_of_run": gms / total_ms if total_ms else None}}
        checks[name] = saved
    clk = clocks.stop()
    # velocity error at the check steps against an FP64 solve of the same state
    # (after the arms: at M = 8000 the FP64 matrix alone takes 115 GB)
    ref = config_sim(rf, cfg, pos, ori, local, rf.PREC_FP64, 1e-12, rf.PC_NONE, rf.VEL_RECOMPUTE)
    # the oracle (CPU FP64: assembly, GMRES to 1e-12, velocities) on the same
    # states where that is bounded: every check step up to M = 1000, the
    # first, middle and last check step at M = 2000, none beyond (the FP64
    # matrix of M = 8000 alone is 115 GB)
    oracle_steps = set()
    if rank == 0 and not args.no_cpu and M <= 2000:
        cs = list(cfg["check"])
        oracle_steps = set(cs) if M <= 1000 else {cs[0], cs[len(cs) // 2], cs[-1]}
    oracle_cache = {}

    def oracle_velocities(key, P, T):
        if key not in oracle_cache:
            from oracle import rfo

            p = rfo.make_params(M, eps=1e-3, dt=cfg["dt"])
            A_o, b_o = rfo.assemble_system(p, P, T)
            x_o, info, _, _ = rfo.solve_gmres(A_o, b_o, restart=10, max_iters=3000, tol=1e-12)
            del A_o
            oracle_cache[key] = rfo.velocities(p, P, T, x_o)
        return oracle_cache[key]

    def rel(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())

    fp64_vs_oracle = []
    for name, saved in checks.items():
        errs, oerrs = [], []
        for step, (P, T), (V, W) in saved:
            ref.set_state(P, T)
            ref.assemble_system()
            ref.solve_system()
            ref.update_velocities()
            V64, W64 = ref.velocities()
            errs.append((step, rel(V, V64), rel(W, W64)))
            if step in oracle_steps:
                Vo, Wo = oracle_velocities((name, step), P, T)
                oerrs.append((step, rel(V, Vo), rel(W, Wo)))
                fp64_vs_oracle.append((name, step, rel(V64, Vo), rel(W64, Wo)))
        e = max(errs, key=lambda w: max(w[1], w[2])) if errs else None
        arms[name]["velocity_error"] = None if e is None else {
            "steps_checked": [w[0] for w in errs] if len(errs) <= 5 else f"1..{errs[-1][0]}",
            "worst_step": e[0], "translational": e[1], "rotational": e[2],
            "norm": "max over fibers / max |FP64 velocity| of the same state"}
        if oerrs:
            eo = max(oerrs, key=lambda w: max(w[1], w[2]))
            arms[name]["velocity_error_vs_oracle"] = {
                "steps_checked": [w[0] for w in oerrs], "worst_step": eo[0], "translational": eo[1],
                "rotational": eo[2], "norm": "max over fibers / max |oracle velocity| of the same state; the "
                                             "oracle solves with GMRES(10) to 1e-12 on the host"}
    ref.close()
    out = None
    if rank == 0:
        first = cfg["arms"][0][0]
        cpu = None
        if not args.no_cpu:
            if M <= 100:
                from oracle import rfo

                o = rfo.Simulation(rfo.make_params(M, eps=1e-3, dt=cfg["dt"], max_iters=300, tol=1e-10), pos, ori)
                t0 = time.perf_counter()
                for _ in range(steps):
                    o.step()
                cpu_s = (time.perf_counter() - t0) / steps
                o.close()
                cpu = {"value": 1.0 / cpu_s, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                       "sample": f"all {steps} steps of the oracle (FP64, GMRES tol 1e-10)"}
            else:
                cpu = cpu_baseline_sample(pos, ori, FP64_MATVECS_PER_STEP)
        arm = arms[first]
        prod = arm["products"]
        out = {
            "metric": f"steps/s, configuration {args.config} (M={M}): " + " vs ".join(a[0] for a in cfg["arms"]),
            "value": arm["value"], "unit": "steps/s", "n_gpus": world, "steps": steps, "warmup": 0,
            "ms_per_step": arm["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": first, "data": "synthetic",
            "config": {"workload": f"M={M} fibers, centres {cfg['distribution']} in a cube of side {cfg['box']} "
                                   f"(seed {cfg['seed']}), eps 1e-3, N=5, 8x3 Gauss points, dt {cfg['dt']}, "
                                   f"{steps} steps from the initial layout",
                       "timing": "device time of every step of the trajectory, first step included",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": f"matrix-vector products of the {first} arm",
                         "achieved": prod["achieved_gbs"], "peak": hbm_peak, "unit": "GB/s", "frac": prod["frac"],
                         "traffic": None,
                         "peak_source": "measured (copy)" if "hbm_gbs" in peaks else "fallback"},
            "cpu_baseline": cpu,
            "arms": arms,
            "gpu_fp64_vs_oracle": None if not fp64_vs_oracle else {
                "translational": max(w[2] for w in fp64_vs_oracle), "rotational": max(w[3] for w in fp64_vs_oracle),
                "states": len(fp64_vs_oracle),
                "note": "the GPU FP64 reference (tol 1e-12) of the velocity checks against the oracle"},
            "clocks": clk,
        }
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return out


# ---------------------------------------------------------------- reference arm
def probe_fortran():
    """Is the reference's own CPU program buildable on this host?  It needs a
    Fortran compiler and LAPACK/BLAS (fortran/Makefile: gfortran, -llapack
    -lblas)."""
    import shutil

    compilers = {c: shutil.which(c) for c in ("gfortran", "f95", "flang", "flang-new", "ifx", "ifort")}
    try:
        libs = subprocess.run(["ldconfig", "-p"], capture_output=True, text=True, timeout=30).stdout
        lapack = sorted({ln.split()[0] for ln in libs.splitlines() if "lapack" in ln.lower()})
    except (OSError, subprocess.SubprocessError):
        lapack = []
    found = {c: p for c, p in compilers.items() if p}
    return {"fortran_compilers": found or "none", "lapack": lapack or "none",
            "buildable": bool(found) and bool(lapack)}


def step_in_parts(sim, parts):
    """One whole oracle time step split into `parts` timed pieces: with
    parts >= 2, parts - 1 row slices of the assembly (contiguous target
    fibers) and a last part that solves, computes the velocities and advects;
    with parts = 1 the step in one piece.  Returns the wall time of each part."""
    M = sim.params.M
    slices = max(1, parts - 1) if parts > 1 else 1
    bounds = [round(k * M / slices) for k in range(slices + 1)]
    times = []
    for k in range(slices):
        t0 = time.perf_counter()
        sim.assemble_part(bounds[k], bounds[k + 1])
        if parts == 1:
            sim.finish_step()
        times.append(time.perf_counter() - t0)
    if parts > 1:
        t0 = time.perf_counter()
        sim.finish_step()
        times.append(time.perf_counter() - t0)
    return times


def run_reference(args):
    """The reference method on the host cores: the FP64 oracle (an OpenMP
    restatement of the reference Fortran) over whole time steps of the
    benchmark workload.  The W warm-up iterations are the parts of the first
    (forward Euler) step, the K timed iterations those of the second
    (multistep) step: value = 1 step / the summed time of the K parts.  Only
    the oracle library is loaded (the layout comes from its restatement of
    the product's generator)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle import rfo

    M = args.M
    pos, ori = rfo.generate_layout(M, WORKLOAD["distribution"], WORKLOAD["box"], WORKLOAD["min_dist"],
                                   seed=WORKLOAD["seed"])
    p = rfo.make_params(M, N=WORKLOAD["N"], NoQI=WORKLOAD["NoQI"], eps=WORKLOAD["eps"], dt=WORKLOAD["dt"],
                        restart=WORKLOAD["restart"], max_iters=300, tol=WORKLOAD["tol"])
    sim = rfo.Simulation(p, pos, ori)
    warm = step_in_parts(sim, args.warmup) if args.warmup > 0 else []
    steps = max(1, args.steps)
    parts = step_in_parts(sim, steps)
    info, iters, be = sim.solve_info()
    phases = sim.timings()
    sim.close()
    step_s = float(sum(parts))
    value = 1.0 / step_s
    n = 3 * WORKLOAD["N"] * M
    sample = (f"one whole FP64 time step (the second, multistep) of the M={M} workload in {len(parts)} timed parts: "
              f"assembly of all {M} targets' rows {phases[0]:.2f}s, GMRES {iters} iterations to {be:.1e} "
              f"{phases[1]:.2f}s, velocities {phases[2]:.2f}s, advection {phases[3]:.3f}s; A held in host memory "
              f"({n * n * 8e-9:.1f} GB)")
    try:
        host_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
    except (ValueError, OSError):
        host_gb = None
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": step_s * 1e3 / len(parts),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(M, world),
        "arm": {"implementation": "FP64 oracle (OpenMP C++ restatement of the reference Fortran advect_fibers: "
                                  "analytic assembly, restarted GMRES with MGS and Givens, velocities, advection)",
                "timing": "the K timed iterations are the K parts of one whole time step; value = 1 / their summed "
                          "time; ms_per_step = the mean part",
                "warmup": f"the first (Euler) step in {len(warm)} parts, {sum(warm):.1f}s" if warm else "none",
                "gmres": {"info": info, "iterations": iters, "residual": be},
                "host_memory_gb": host_gb,
                "reference_fortran": probe_fortran()},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


REF_GPU_EXE = os.path.join(ROOT, "oracle", "_ref", "fibers_gpu")
# The one case the reference's CUDA program runs: its kernels are compiled for
# 100 fibers, eps 0.01, N = 5 and 8 x 3 Gauss points (src/kernels/constants.cu),
# its GMRES tolerance is fixed at 1e-5 (src/simulation.cu:337) and it stops
# after the first time step (src/main.cu:62-65).  That is the reference's own
# golden case: the XcT_init100.in layout with the run100_iter.in parameters
# (v1 parameter file, one value per line, src/parameters.cc:124-180).
REF_GPU_PARAMS = ["golden", "XcT_init100", "5", "0.01", "0.1", "10", "1", "1", "8", "1", "0", "10", "100", "1e-5"]
REF_GPU_PHASES = ("assemble_system", "solve_system", "update_velocities", "update_fibers_firststep")


def _ref_gpu_phases(out):
    """Seconds per phase from the program's own event timers: lines
    "[BENCHMARK]   : <name> : <last>(<average>) sec" (src/performance.cc)."""
    phases = {}
    for line in out.splitlines():
        if "[BENCHMARK]" in line:
            f = line.split(":")
            if len(f) >= 3:
                phases[f[1].strip()] = float(f[2].strip().split("(")[0])
    return phases


def _rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    if a.shape != b.shape:
        return None
    return float(np.abs(a - b).max() / max(1e-300, np.abs(b).max()))


def run_reference_gpu(args):
    """The reference's own CUDA program (oracle/_ref/fibers_gpu, built from its
    sources by oracle/Makefile) on the only case it is compiled for, beside
    this library's plain FP64 path on the same case.  Each of the W + K runs
    is one process that takes one (forward Euler) time step; the step time is
    the sum of the program's own CUDA-event phase timers (assembly, ViennaCL
    GMRES, velocities, advection; its text dump of A, b and x is not timed).
    Accuracy: its b and x against the reference Fortran's golden vectors."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    g = np.load(os.path.join(ROOT, "tests", "golden", "golden_m100.npz"))
    X0, T0 = g["layout_pos"], g["layout_orient"]
    gold_b, gold_x = g["100_analytic_gmres/0_BVec"], g["100_analytic_gmres/0_XVec"]
    config = {"workload": "reference golden case: M=100 (XcT_init100.in), eps 0.01, N=5, 8x3 Gauss points, "
                          "GMRES(10) tol 1e-5, first (Euler) step, FP64", "M": 100, "parallelism": "single GPU"}
    base = {"impl": "reference-gpu", "metric": "steps/s of the first time step of the M=100 golden case",
            "unit": "steps/s", "n_gpus": 1, "higher_is_better": True, "data": "the reference's golden layout",
            "config": config}
    if not os.path.exists(REF_GPU_EXE):
        return dict(base, unavailable="oracle/_ref/fibers_gpu not built (oracle/Makefile ref-gpu needs the "
                                      "reference's sources)")
    runs = []
    with tempfile.TemporaryDirectory() as d:
        par, lay = os.path.join(d, "run100_iter.in"), os.path.join(d, "XcT_init100.in")
        with open(par, "w") as f:
            f.write("\n".join(REF_GPU_PARAMS) + "\n")
        with open(lay, "w") as f:
            f.write(f"{len(X0)}\n")
            for p, t in zip(X0, T0):
                f.write(f"{p[0]:.16f} {p[1]:.16f} {p[2]:.16f}\n{t[0]:.16f} {t[1]:.16f} {t[2]:.16f}\n")
        for _ in range(args.warmup + max(1, args.steps)):
            r = subprocess.run([REF_GPU_EXE, par, lay], capture_output=True, text=True, timeout=600)
            ph = _ref_gpu_phases(r.stdout)
            if r.returncode != 0 or not all(n in ph for n in REF_GPU_PHASES):
                tail = (r.stdout + r.stderr).strip().splitlines()[-3:]
                return dict(base, unavailable=f"reference CUDA program exited {r.returncode}: {' | '.join(tail)}")
            runs.append(ph)
    # the program writes its last step's b and x next to itself (src/simulation.cu:468-546)
    out_dir = os.path.dirname(REF_GPU_EXE)
    acc = {}
    for name, gold in (("b", gold_b), ("x", gold_x)):
        path = os.path.join(out_dir, f"{name}_vector.out")
        acc[name] = _rel_err(np.loadtxt(path), gold) if os.path.exists(path) else None
    timed = runs[args.warmup:]
    step_s = [sum(ph[n] for n in REF_GPU_PHASES) for ph in timed]
    ref_phases = {n: 1e3 * float(np.mean([ph[n] for ph in timed])) for n in REF_GPU_PHASES}

    # this library's plain FP64 path, the same case and tolerance, timed on its stream
    import rigidfibers_kth_b200 as rf

    # a fresh run each time, like the program's one step per process (GMRES
    # from a zero initial guess; handle creation and upload not timed)
    ours, ours_acc = [], {}
    for k in range(args.warmup + max(1, args.steps)):
        with rf.Simulation(rf.Configuration(rf.FiberParams(device=0), X0, T0)) as sim:
            sim.mark(0); sim.assemble_system(); sim.mark(1); sim.solve_system(); sim.mark(2)
            sim.update_velocities(); sim.mark(3); sim.update_fibers(True); sim.mark(4)
            if k >= args.warmup:
                ours.append([sim.elapsed_ms(i, i + 1) for i in range(4)])
            ours_acc = {"b": _rel_err(sim.rhs(), gold_b), "x": _rel_err(sim.coeffs(), gold_x)}
    ours = np.array(ours)
    ours_ms = float(ours.sum(axis=1).mean())
    ref_ms = 1e3 * float(np.mean(step_s))
    return dict(base, value=1e3 / ref_ms, steps=len(timed), warmup=args.warmup, ms_per_step=ref_ms,
                dtype="f64 storage (float transcendentals, src/kernels/assemble_system.cu:21)",
                phases_ms=ref_phases, error_vs_fortran_golden=acc,
                product_same_case={"value": 1e3 / ours_ms, "ms_per_step": ours_ms,
                                   "phases_ms": dict(zip(REF_GPU_PHASES, map(float, ours.mean(axis=0)))),
                                   "error_vs_fortran_golden": ours_acc,
                                   "path": "plain FP64 (RF_PREC_FP64, CERFACS GMRES(10) tol 1e-5)"})


def main():
    global PC_DAMPING, NEAR_C
    args = parse_args()
    PC_DAMPING = args.pc_damping
    NEAR_C = args.near_c
    if args.impl == "reference":
        out = run_reference(args)
    elif args.impl == "reference-gpu":
        out = run_reference_gpu(args)
    else:
        out = run_ours(args) if args.config == 4 else run_config(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
