"""Benchmark: gradient evaluations of log pi(theta | y) per second on one
spatio-temporal INLA workload (default: Gaussian DEMF(1,2,1), ns = 1500,
nt = 100, nb = 6, 600 observations per step; BTA blocks 1500 x 1500).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = full gradient evaluations (f(theta) and grad f) at ``--batch``
theta points (the candidates of a line search, default 3), the unit counted
being one gradient evaluation.  ``ours`` uses the adjoint path (one
factorisation and selected inversion of Q_c and of Q_prior per point, all 2K
matrices factored and inverted together); the single-point adjoint and the
plain FP64 central-difference path (2d+1 evaluations of f, one after another,
as the reference computes it) are timed beside it.
With N > 1 (torchrun) every rank evaluates its own replica (independent theta
points, no collective on the data path); the reported value is the total over
ranks divided by the slowest rank's device time.

``--impl reference`` times the CPU oracle (NumPy/SciPy LAPACK restatement of
the reference's Serinv path) on the host cores on a bounded sample: one f(theta)
on the workload truncated to ``--cpu-nt`` time steps, scaled to the full
workload and to the 2d+1 evaluations of a finite-difference gradient.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "grad log pi(theta|y) evals/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="gst_1500x100")
    p.add_argument("--cpu-nt", type=int, default=10)
    p.add_argument("--fd-steps", type=int, default=1)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU-oracle baseline sample")
    p.add_argument("--batch", type=int, default=3,
                   help="theta points per step (a line-search batch), factorised together")
    p.add_argument("--precision", default="i8slice", choices=["fp64", "tf32x3", "i8slice"],
                   help="arithmetic of the selected inversions behind the adjoint gradient")
    return p.parse_args()


def dist_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------ replicas
def replica_theta(theta, rank):
    """Each rank evaluates its own theta points (independent replicas, no
    collective on the data path)."""
    return np.asarray(theta, dtype=np.float64) + 1e-3 * rank


def step_points(theta, step, K):
    """The K candidates of one step; theta moves between steps as in an
    optimiser, so warm starts of a Newton iteration see a new point."""
    base = theta + 0.005 * (step % 4)
    return [base + 1e-3 * j for j in range(K)]


def max_over_ranks(t, world, device=None):
    """Slowest rank's time (the job ends when it does)."""
    if world <= 1:
        return float(t)
    import torch

    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
    return float(tt.item())


def job_rate(units_per_rank, world, t_max):
    """Whole-job throughput: the units all ranks processed / the slowest time."""
    return units_per_rank * world / t_max


# ----------------------------------------------------------------- CPU port
def cpu_sample(workload, nt_sample, reps=1):
    """Time one f(theta) of the CPU oracle on the workload truncated to
    nt_sample time steps; returns (seconds per full FD gradient, description)."""
    from dalia_b200 import synth
    from oracle import coreg_ref, model_ref

    coreg = workload in synth.COREG_CONFIGS
    cfg = dict(synth.COREG_CONFIGS[workload] if coreg else synth.CONFIGS[workload])
    nt_full = cfg["nt"]
    cfg["nt"] = min(nt_sample, nt_full)
    if coreg:
        om = coreg_ref.CoregionalOracle(synth.make_coregional_problem(seed=0, **cfg))
    else:
        om = model_ref.OracleModel(synth.make_problem(seed=0, **cfg))
    th = np.asarray(cfg["theta"], dtype=np.float64)
    om.evaluate_f(th)  # warm-up (BLAS thread pool, caches)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        om.evaluate_f(th)
        ts.append(time.perf_counter() - t0)
    t_f = min(ts) * nt_full / cfg["nt"]
    d = th.size
    t_grad = t_f * (2 * d + 1)
    desc = (f"one f(theta) of the CPU oracle (NumPy/SciPy LAPACK) on {workload} truncated to nt={cfg['nt']} "
            f"of {nt_full}, scaled linearly in nt and by 2d+1={2 * d + 1} evaluations per FD gradient")
    return t_grad, desc


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    ts = []
    desc = ""
    for i in range(args.warmup + args.steps):
        t, desc = cpu_sample(args.workload, args.cpu_nt)
        if i >= args.warmup:
            ts.append(t)
    t_step = statistics.median(ts)
    value = 1.0 / t_step
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "evals/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_step * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "path": "central finite differences, FP64, CPU oracle"},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""
    A = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    B = torch.randn_like(A)
    for _ in range(2):
        A @ B
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        A @ B
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del A, B
    torch.cuda.empty_cache()
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


def run_ours(args):
    import torch

    from dalia_b200 import _lib, synth
    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.model import SpatioTemporalModel

    rank, world, local = dist_info()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()

    coreg = args.workload in synth.COREG_CONFIGS
    cfg = synth.COREG_CONFIGS[args.workload] if coreg else synth.CONFIGS[args.workload]
    prob = synth.make_config(args.workload, seed=0)
    model = (CoregionalModel if coreg else SpatioTemporalModel)(prob, device=dev, selinv_precision=args.precision)
    n, b, a = model.nt, model.b, model.nb
    # replicas evaluate different theta points (a line-search batch)
    theta = replica_theta(cfg["theta"], rank)

    peak = measured_fp64_peak(torch, dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    K = max(1, args.batch)

    def step_thetas(step):
        return step_points(theta, step, K)

    # ---- warm-up
    nwarm = max(args.warmup, 3)
    for s in range(nwarm):
        model.objective_adjoint_batched(step_thetas(s))
    barrier()

    # ---- one profiled step, events around every launch: the per-category
    # split and the dominant kernel category.  Only that category's launches
    # carry events in the timed region (events around all ~1400 launches of a
    # step cost ~2.5 %).
    import ctypes

    pre_ms = (ctypes.c_double * 8)()
    pre_cnt = (ctypes.c_longlong * 8)()
    lib.bta_prof_read(None, None)
    lib.bta_prof_mask(0xFF)
    lib.bta_prof_enable(1)
    model.objective_adjoint_batched(step_thetas(nwarm + 2 * args.steps))
    lib.bta_prof_enable(0)
    lib.bta_prof_read(pre_ms, pre_cnt)
    # the 8-bit-slice GEMM's digit pre-pass counts towards the GEMM's time
    dom = max((0, 1), key=lambda c: pre_ms[0] if c == 0 else pre_ms[1] + pre_ms[5])
    barrier()

    # ---- device-timed steps: K-point adjoint gradient batches (events around
    # the dominant category's launches)
    clock = ClockSampler(local)
    clock.start()
    lib.bta_prof_mask(1 if dom == 0 else (1 << 1) | (1 << 5))
    lib.bta_prof_enable(1)
    launches0 = lib.bta_launch_count()
    work0 = dict(model.work)
    step_th = [step_thetas(nwarm + s) for s in range(args.steps)]
    barrier()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record()
    fallbacks = 0
    resid_max = 0.0
    for s in range(args.steps):
        model.objective_adjoint_batched(step_th[s])
        fallbacks += sum(1 for c in model.last_check if c["fallback"])
        resid_max = max([resid_max] + [max(c["residual_c"], c["residual_p"]) for c in model.last_check])
    e1.record()
    barrier()
    launches = lib.bta_launch_count() - launches0
    work = {k: model.work[k] - work0[k] for k in work0}
    lib.bta_prof_enable(0)
    ms_cat = (ctypes.c_double * 8)()
    cnt_cat = (ctypes.c_longlong * 8)()
    lib.bta_prof_read(ms_cat, cnt_cat)
    lib.bta_prof_mask(0xFF)
    clocks = clock.stop()
    t_dev = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)
    value = job_rate(K * args.steps, world, t_dev)

    # ---- single-point adjoint latency
    barrier()
    s0, s1 = torch.cuda.Event(True), torch.cuda.Event(True)
    s0.record()
    for s in range(args.steps):
        model.objective_adjoint(step_thetas(s)[0])
    s1.record()
    barrier()
    single_rate = args.steps / (s0.elapsed_time(s1) * 1e-3)

    # ---- end to end through the public call, host thetas in, host gradients out
    barrier()
    t0 = time.perf_counter()
    for s in range(args.steps):
        th_host = [np.array(t) for t in step_thetas(nwarm + args.steps + s)]  # host buffers
        fs, gs = model.objective_adjoint_batched(th_host)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = job_rate(K * args.steps, world, t_e2e)
    f, g = fs[0], gs[0]
    coef_bytes = model.slots[0].coef_host[0].numel() * 8
    h2d = K * 2 * coef_bytes
    d2h = K * ((5 + 3 * (2 * n - 1) * 4 + a * a) * 8) + 16

    # ---- plain FP64 finite differences (the reference's algorithm)
    # accuracy of the reduced-precision selected inversion against FP64 at one
    # point (outside every timed region)
    accuracy = {"fallbacks_in_timed_region": fallbacks, "max_identity_residual": resid_max}
    if args.precision != "fp64":
        fr, gr = model.objective_adjoint_batched([theta])
        f64, g64 = model.objective_adjoint_batched([theta], precision="fp64")
        accuracy["grad_rel_err_vs_fp64"] = float(np.linalg.norm(np.asarray(gr[0]) - np.asarray(g64[0]))
                                                 / np.linalg.norm(np.asarray(g64[0])))
        accuracy["f_rel_err_vs_fp64"] = abs(fr[0] - f64[0]) / abs(f64[0])
    fd_rate = None
    if args.fd_steps > 0:
        barrier()
        f0, f1 = torch.cuda.Event(True), torch.cuda.Event(True)
        f0.record()
        for _ in range(args.fd_steps):
            model.objective_fd(theta)
        f1.record()
        barrier()
        fd_rate = args.fd_steps / (f0.elapsed_time(f1) * 1e-3)
    # the same stencil with its 2d+1 points factorised in batches (Gaussian)
    fdb_rate = None
    if args.fd_steps > 0 and model.gaussian:
        barrier()
        f0, f1 = torch.cuda.Event(True), torch.cuda.Event(True)
        f0.record()
        for _ in range(args.fd_steps):
            model.objective_fd_batched(theta)
        f1.record()
        barrier()
        fdb_rate = args.fd_steps / (f0.elapsed_time(f1) * 1e-3)

    # ---- roofline of the dominant kernel category
    names = {0: "panel (tile-DAG BTA panel Cholesky)",
             1: {"fp64": "gemm (grouped FP64 DMMA GEMM)",
                 "tf32x3": "gemm (split-TF32 tcgen05 GEMM)",
                 "i8slice": "gemm (8-bit-slice tcgen05 GEMM incl. digit pre-pass)"}[args.precision]}
    # algorithmic flops issued in the timed region (every Newton factorisation
    # of a non-Gaussian likelihood included)
    tot_flops = {0: work["factor"], 1: work["selinv_gemm"]}
    cat_ms = {0: ms_cat[0], 1: ms_cat[1] + ms_cat[5]}
    achieved = tot_flops[dom] / (cat_ms[dom] * 1e-3) / 1e12
    traffic = None
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(names[dom].split()[0])
        except Exception:
            traffic = None
    dom_peak, peak_src = peak, "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)"
    if dom == 1 and args.precision == "i8slice":
        # FP64-equivalent ceiling of 28 int8 digit products per product: the
        # dense int8 rate taken as twice the measured bf16 burst
        try:
            bf16 = float(json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))["bf16_tflops"])
        except Exception:
            bf16 = 1590.0
        dom_peak = 2 * bf16 / 28
        peak_src = f"2 x measured bf16 burst ({bf16:.0f} TF/s) / 28 digit products (int8 ceiling, FP64-equivalent)"
    roofline = {
        "bound": "tensor",
        "kernel": names[dom],
        "achieved": achieved,
        "peak": dom_peak,
        "unit": "TFLOP/s",
        "frac": achieved / dom_peak,
        "peak_source": peak_src,
        "avg_launch_ms": cat_ms[dom] / max(cnt_cat[dom], 1),
        "launches": int(cnt_cat[dom]),
        "traffic": traffic,
    }
    # per-category split of the profiled step (events around every launch)
    kernel_ms = {k: pre_ms[i] for i, k in enumerate(["panel", "gemm", "sweep", "trtri", "other", "slice"])}

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            t_cpu, desc = cpu_sample(args.workload, args.cpu_nt)
            cpu = {"value": 1.0 / t_cpu, "unit": "evals/s", "cores": os.cpu_count(), "kind": "port", "sample": desc}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": "evals/s", "cores": os.cpu_count(), "kind": "port", "sample": repr(exc)}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "evals/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": t_dev / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else f"f64 + {args.precision} block products",
            "data": "synthetic",
            "config": {
                "workload": args.workload,
                "ns": model.ns, "variates": model.nv, "block": b, "nt": n, "nb": a, "obs_per_step": cfg["no"],
                "theta": list(cfg["theta"]),
                "path": f"adjoint gradient, selected inversion in {args.precision} (factorisations, log-dets, solves "
                        f"FP64); {K} theta points per step (line-search batch), theta moved "
                        f"between steps; Q_c and Q_prior of all points factorised and selected-inverted together",
                "theta_points_per_step": K,
                "parallelism": f"replicas x{world}",
                "likelihood": cfg.get("likelihood", "gaussian"),
                "l2": f"inputs larger than L2 (BTA matrix {model.Qc.buf.numel() * 8 / 1e9:.1f} GB each)",
            },
            "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "mixed_accuracy": accuracy,
            "fd_fp64_evals_per_s": fd_rate,
            "fd_fp64_batched_stencil_evals_per_s": fdb_rate,
            "adjoint_single_point_evals_per_s": single_rate,
            "speedup_vs_fd_fp64": (value / fd_rate) if fd_rate else None,
            # per-step work of the timed region over the profiled step's kernel times
            "bta_factor_tflops": tot_flops[0] / args.steps / max(pre_ms[0] * 1e-3, 1e-12) / 1e12,
            "bta_selinv_gemm_tflops": tot_flops[1] / args.steps / max((pre_ms[1] + pre_ms[5]) * 1e-3, 1e-12) / 1e12,
            "kernel_ms_source": "one profiled step before the timed region (events around every launch); "
                                "in the timed region only the roofline kernel's launches carry events",
            "newton_steps_per_point": (work["newton_steps"] / (K * args.steps)) if not model.gaussian else None,
            "kernel_ms_per_step": kernel_ms,
            "f": f,
            "grad": list(map(float, g)),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
