"""Benchmark: gradient evaluations of log pi(theta | y) per second on one
spatio-temporal INLA workload (default: Gaussian DEMF(1,2,1), ns = 1500,
nt = 100, nb = 6, 600 observations per step; BTA blocks 1500 x 1500).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--batch K] [--precision fp64|i8slice|tf32x3]

One step = full gradient evaluations (f(theta) and grad f) at ``--batch``
theta points (candidates of a line search or points of a stencil, default
6), the unit counted
being one gradient evaluation.  ``ours`` uses the adjoint path (one
factorisation and selected inversion of Q_c and of Q_prior per point, all 2K
matrices factored and inverted together); the single-point adjoint and the
plain FP64 central-difference paths (2d+1 evaluations of f, one after
another as the reference computes them, and the same stencil with its points
factorised together) are timed beside it, warm, over ``--fd-steps`` repeats.
A mixed-size workload (``synth.MIXED_BATCHES``) evaluates the points of
several models -- instances of different block sizes -- in shared launches.
With N > 1 (torchrun) every rank evaluates its own replica (independent theta
points, no collective on the data path); the reported value is the total over
ranks divided by the slowest rank's device time.

``--impl reference`` times the CPU oracle (NumPy/SciPy LAPACK restatement of
the reference's Serinv path) on the host cores: every step is one f(theta) on
the workload truncated to ``--cpu-nt`` time steps, scaled to the full workload
and to the 2d+1 evaluations of a finite-difference gradient; one f(theta) on
the whole workload (``--ref-full-nt``) checks that linear scaling in nt.
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


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="gst_1500x100")
    p.add_argument("--cpu-nt", type=int, default=10)
    p.add_argument("--ref-full-nt", type=int, default=1,
                   help="reference arm: also time one f(theta) on the untruncated workload (0: skip)")
    p.add_argument("--fd-steps", type=int, default=3, help="timed repeats of each FD path (after one warm-up)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU-oracle baseline sample")
    p.add_argument("--batch", type=int, default=6,
                   help="theta points per step (e.g. line-search candidates or stencil points), factorised "
                        "together; reduced to what device memory holds")
    p.add_argument("--precision", default="i8slice", choices=["fp64", "tf32x3", "i8slice"],
                   help="arithmetic of the selected inversions behind the adjoint gradient")
    p.add_argument("--factor-precision", default="auto", choices=["fp64", "i8slice", "auto"],
                   help="arithmetic of the factorisations' previous-column Schur updates in the adjoint path "
                        "(auto: 8-bit slices for blocks of 1500 and wider; with --precision fp64 the whole "
                        "path is FP64)")
    return p.parse_args(argv)


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


# ------------------------------------------------------------- workloads
def members(workload):
    """[(single workload, theta points per step or None)] of a workload: one
    member for a plain workload, several for a mixed-size batch."""
    from dalia_b200 import synth

    if workload in synth.MIXED_BATCHES:
        return list(synth.MIXED_BATCHES[workload])
    if workload in synth.CONFIGS or workload in synth.COREG_CONFIGS:
        return [(workload, None)]
    raise SystemExit(f"unknown workload {workload!r}")


def config_of(name):
    from dalia_b200 import synth

    return synth.COREG_CONFIGS[name] if name in synth.COREG_CONFIGS else synth.CONFIGS[name]


# ----------------------------------------------------------------- CPU port
_ORACLES = {}


def cpu_sample(workload, nt_sample, reps=1):
    """Time one f(theta) of the CPU oracle on the workload truncated to
    nt_sample time steps; returns (seconds per full FD gradient, description,
    seconds of the sampled f).  A mixed-size batch is timed member by member
    and weighted by its points per step (seconds per gradient, averaged).
    The oracle model of a (workload, nt) is built and warmed up once per
    process."""
    from dalia_b200 import synth
    from oracle import coreg_ref, model_ref

    mem = members(workload)
    total_pts = sum(k or 1 for _, k in mem)
    t_grad, descs, t_sample = 0.0, [], 0.0
    for name, k in mem:
        coreg = name in synth.COREG_CONFIGS
        cfg = dict(config_of(name))
        nt_full = cfg["nt"]
        cfg["nt"] = min(nt_sample, nt_full)
        th = np.asarray(cfg["theta"], dtype=np.float64)
        om = _ORACLES.get((name, cfg["nt"]))
        if om is None:
            if coreg:
                om = coreg_ref.CoregionalOracle(synth.make_coregional_problem(seed=0, **cfg))
            else:
                om = model_ref.OracleModel(synth.make_problem(seed=0, **cfg))
            om.evaluate_f(th)  # warm-up (BLAS thread pool, caches)
            _ORACLES[(name, cfg["nt"])] = om
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            om.evaluate_f(th)
            ts.append(time.perf_counter() - t0)
        t_sample += min(ts)
        t_f = min(ts) * nt_full / cfg["nt"]
        d = th.size
        t_grad += (k or 1) / total_pts * t_f * (2 * d + 1)
        descs.append(f"{name}: one f(theta) truncated to nt={cfg['nt']} of {nt_full}, scaled linearly in nt "
                     f"and by 2d+1={2 * d + 1} evaluations per FD gradient")
    desc = "CPU oracle (NumPy/SciPy LAPACK): " + "; ".join(descs)
    return t_grad, desc, t_sample


def full_nt_check(workload, max_s=150.0):
    """One f(theta) of the CPU oracle on the untruncated (first) member of the
    workload, against the linear extrapolation from a 10-step sample; skipped
    when the extrapolation says it would take longer than max_s."""
    from dalia_b200 import synth
    from oracle import coreg_ref, model_ref

    name = members(workload)[0][0]
    cfg = dict(config_of(name))
    make = (lambda c: coreg_ref.CoregionalOracle(synth.make_coregional_problem(seed=0, **c))) \
        if name in synth.COREG_CONFIGS else (lambda c: model_ref.OracleModel(synth.make_problem(seed=0, **c)))
    th = np.asarray(cfg["theta"], dtype=np.float64)
    small = dict(cfg, nt=min(10, cfg["nt"]))
    os_ = make(small)
    os_.evaluate_f(th)
    t0 = time.perf_counter()
    os_.evaluate_f(th)
    t_small = time.perf_counter() - t0
    extrap = t_small * cfg["nt"] / small["nt"]
    out = {"workload": name, "nt": cfg["nt"], "f_nt10_s": t_small, "extrapolated_full_s": extrap}
    if extrap > max_s:
        out["skipped"] = f"extrapolated {extrap:.0f} s > {max_s:.0f} s"
        return out
    om = make(cfg)
    t0 = time.perf_counter()
    om.evaluate_f(th)
    t_full = time.perf_counter() - t0
    out.update({"f_full_nt_s": t_full, "measured_over_extrapolated": t_full / extrap})
    return out


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    ts = []
    desc = ""
    for i in range(args.warmup + args.steps):
        t, desc, _ = cpu_sample(args.workload, args.cpu_nt)
        if i >= args.warmup:
            ts.append(t)
    t_step = statistics.median(ts)
    value = 1.0 / t_step
    check = None
    if getattr(args, "ref_full_nt", 0):
        try:
            check = full_nt_check(args.workload)
        except MemoryError as exc:  # config 4 needs ~64 GB of host memory per matrix
            check = {"skipped": repr(exc)}
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
        "nt_scaling_check": check,
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


def panel_bytes_per_launch(b, a, count):
    """Algorithmic DRAM bytes of one block-column launch of the factorisation
    over count matrices: D_i, L_i and Ab_i read and written once, the previous
    column's L_{i-1} and Ab_{i-1} read once."""
    return count * 8 * (2 * (2 * b * b + a * b) + b * b + a * b)


def roofline_traffic(workload, kernel, shape):
    """DRAM bytes per launch of the dominant kernel: the ncu capture of the
    same launch shape if one is committed, else the capture of the nearest
    shape scaled by the algorithmic bytes per launch (said in the source)."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        tab = json.load(open(path))
    except Exception:
        return None, "no capture"
    caps = tab.get("captures", {})
    b, a, count = shape
    for key, cap in caps.items():
        if kernel in cap and tuple(cap.get("shape", ())) == (b, a, count):
            return float(cap[kernel]), f"ncu capture {key} (same launch shape)"
    for key, cap in caps.items():
        if kernel in cap and "shape" in cap:
            cb, ca, cc = cap["shape"]
            if kernel == "panel":
                scale = panel_bytes_per_launch(b, a, count) / panel_bytes_per_launch(cb, ca, cc)
            else:
                scale = (b * b * count) / (cb * cb * cc)
            return float(cap[kernel]) * scale, (f"ncu capture {key} (launch shape b={cb}, a={ca}, {cc} matrices) "
                                                f"scaled by algorithmic bytes per launch x{scale:.3f}")
    return None, "no capture"


def run_ours(args):
    import ctypes

    import torch

    from dalia_b200 import _lib, synth
    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.model import SpatioTemporalModel, adjoint_group

    rank, world, local = dist_info()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()

    mem = members(args.workload)
    models, thetas, Ks = [], [], []
    for name, k in mem:
        prob = synth.make_config(name, seed=0)
        cls = CoregionalModel if name in synth.COREG_CONFIGS else SpatioTemporalModel
        m = cls(prob, device=dev, selinv_precision=args.precision, factor_precision=args.factor_precision)
        models.append(m)
        # replicas evaluate different theta points (a line-search batch)
        thetas.append(replica_theta(config_of(name)["theta"], rank))
        Ks.append(k if k is not None else max(1, args.batch))
    mixed = len(models) > 1
    # the arithmetic the factorisations' Schur updates run in ("auto" resolved)
    from dalia_b200.model import _factor_arith
    factor_arith = _factor_arith(args.factor_precision, models, args.precision)
    factor_desc = factor_arith if args.factor_precision != "auto" else f"{factor_arith} (auto by block size)"
    if not mixed:
        # Q_c, Q_prior and Q_c's block inverses of every point stay resident
        m = models[0]
        per = (m.Qc.buf.numel() + m.Qp.buf.numel() + m.nt * m.b * m.b) * 8
        free, _ = torch.cuda.mem_get_info(dev)
        Ks[0] = int(max(1, min(Ks[0], (free - (8 << 30)) // per + 1)))
    units = sum(Ks)
    model = models[0]

    peak = measured_fp64_peak(torch, dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    def step_jobs(step):
        return [(m, step_points(th, step, k)) for m, th, k in zip(models, thetas, Ks)]

    def run_step(step, precision=None):
        jobs = step_jobs(step)
        if mixed:
            return adjoint_group(jobs, precision or args.precision)
        m, pts = jobs[0]
        return [m.objective_adjoint_batched(pts, precision)]

    def checks():
        return [c for m in models for c in m.last_check]

    def work_sum():
        return {k: sum(m.work[k] for m in models) for k in models[0].work}

    # ---- warm-up, then further untimed steps while the autotuner is still
    # trying candidates for a launch shape of the step (bounded)
    nwarm = max(args.warmup, 3)
    for s in range(nwarm):
        run_step(s)
    extra = 0
    while lib.bta_tune_pending() > 0 and extra < 12:
        run_step(nwarm + extra)
        extra += 1
    barrier()

    # ---- one profiled step, events around every launch: the per-category
    # split and the dominant kernel category.  Only that category's launches
    # carry events in the timed region (events around all ~1400 launches of a
    # step cost ~2.5 %).
    pre_ms = (ctypes.c_double * 8)()
    pre_cnt = (ctypes.c_longlong * 8)()
    lib.bta_prof_read(None, None)
    lib.bta_prof_mask(0xFF)
    lib.bta_prof_enable(1)
    pre_work0 = work_sum()
    run_step(nwarm + 2 * args.steps)
    # the profiled step's own algorithmic work (a point that falls back or
    # runs in FP64 after a failed check makes steps differ in work)
    pre_work = {k: v - pre_work0[k] for k, v in work_sum().items()}
    lib.bta_prof_enable(0)
    lib.bta_prof_read(pre_ms, pre_cnt)
    # kernel groups: 0 the panel kernel, 1 the selected inversion's GEMM, 2 the
    # factorisation's Schur-update GEMM (reduced-precision factor updates);
    # an 8-bit-slice GEMM's digit pre-pass counts towards its GEMM's time
    groups = {0: (0,), 1: (1, 5), 2: (6,)}
    dom = max(groups, key=lambda g: sum(pre_ms[c] for c in groups[g]))
    barrier()

    # ---- device-timed steps: K-point adjoint gradient batches (events around
    # the dominant category's launches)
    clock = ClockSampler(local)
    clock.start()
    lib.bta_prof_mask(sum(1 << c for c in groups[dom]))
    lib.bta_prof_enable(1)
    launches0 = lib.bta_launch_count()
    work0 = work_sum()
    barrier()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record()
    fallbacks = demoted = 0
    resid_max = 0.0
    for s in range(args.steps):
        run_step(nwarm + s)
        fallbacks += sum(1 for c in checks() if c["fallback"])
        demoted += sum(1 for c in checks() if c.get("demoted"))
        resid_max = max([resid_max] + [max(c["residual_c"], c["residual_p"]) for c in checks()])
    e1.record()
    barrier()
    launches = lib.bta_launch_count() - launches0
    work = {k: v - work0[k] for k, v in work_sum().items()}
    lib.bta_prof_enable(0)
    ms_cat = (ctypes.c_double * 8)()
    cnt_cat = (ctypes.c_longlong * 8)()
    lib.bta_prof_read(ms_cat, cnt_cat)
    lib.bta_prof_mask(0xFF)
    clocks = clock.stop()
    t_dev = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)
    value = job_rate(units * args.steps, world, t_dev)

    # ---- single-point adjoint latency (first member)
    barrier()
    s0, s1 = torch.cuda.Event(True), torch.cuda.Event(True)
    s0.record()
    for s in range(args.steps):
        model.objective_adjoint(step_points(thetas[0], s, 1)[0])
    s1.record()
    barrier()
    single_rate = args.steps / (s0.elapsed_time(s1) * 1e-3)

    # ---- end to end through the public call, host thetas in, host gradients out
    barrier()
    t0 = time.perf_counter()
    for s in range(args.steps):
        out = run_step(nwarm + args.steps + s)  # host theta arrays in, host f / gradients out
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = job_rate(units * args.steps, world, t_e2e)
    f, g = out[0][0][0], out[0][1][0]
    h2d = sum(k * 2 * m.slots[0].coef_host[0].numel() * 8 for m, k in zip(models, Ks))
    d2h = sum(k * ((5 + 3 * (2 * m.nt - 1) * 4 * m.nv * m.nv + m.nb * m.nb) * 8) + 16 for m, k in zip(models, Ks))

    # ---- accuracy of the reduced-precision selected inversion against FP64,
    # per result, at one point of the first member (outside every timed region)
    accuracy = {"fallbacks_in_timed_region": fallbacks, "fp64_after_failed_check_in_timed_region": demoted,
                "max_identity_residual": resid_max}
    if args.precision != "fp64":
        sl = model.slots[0]

        def results(prec):
            fr, gr = model.objective_adjoint_batched([thetas[0]], precision=prec)
            dsel = torch.cat([torch.diagonal(sl.Qc.D, dim1=1, dim2=2).reshape(-1), torch.diagonal(sl.Qc.T)])
            return fr[0], np.asarray(gr[0]), float(sl.scal[0]), sl.x.cpu().numpy(), dsel.cpu().numpy()

        fr, gr, ldr, xr, sr = results(args.precision)
        f64, g64, ld64, x64, s64 = results("fp64")
        accuracy.update({
            "grad_rel_err_vs_fp64": float(np.linalg.norm(gr - g64) / np.linalg.norm(g64)),
            "f_rel_err_vs_fp64": abs(fr - f64) / abs(f64),
            "logdet_qc_rel_err_vs_fp64": abs(ldr - ld64) / abs(ld64),
            "solution_rel_err_vs_fp64": float(np.linalg.norm(xr - x64) / np.linalg.norm(x64)),
            "selinv_diag_rel_err_vs_fp64": float(np.max(np.abs(sr - s64) / np.abs(s64))),
            "note": ("the factorisations' Schur updates and the selected inversion's block products differ; "
                     "POTRF, log-determinant sums and sweeps are FP64 in both") if factor_arith != "fp64"
            else "factorisations, log-determinants and solves are FP64 in both; the selected inversion's "
                 "block products differ",
        })

    # ---- plain FP64 finite differences (the reference's algorithm), warm:
    # one untimed evaluation of each path, then --fd-steps timed repeats.
    # A mixed batch: one point per member, weighted by its points per step.
    def fd_rate(batched):
        t_units = 0.0
        for m, th, k in zip(models, thetas, Ks):
            if batched and not m.gaussian:
                return None
            fn = m.objective_fd_batched if batched else m.objective_fd
            fn(th)  # warm-up: slots, workspaces, task lists
            barrier()
            f0, f1 = torch.cuda.Event(True), torch.cuda.Event(True)
            f0.record()
            for _ in range(args.fd_steps):
                fn(th)
            f1.record()
            barrier()
            t_units += k * (f0.elapsed_time(f1) * 1e-3) / args.fd_steps
        return units / t_units

    fd_seq = fd_rate(False) if args.fd_steps > 0 else None
    fd_bat = fd_rate(True) if args.fd_steps > 0 else None

    # ---- roofline of the dominant kernel group
    names = {0: "panel (tile-DAG BTA panel Cholesky)",
             1: {"fp64": "gemm (grouped FP64 DMMA GEMM)",
                 "tf32x3": "gemm (split-TF32 tcgen05 GEMM)",
                 "i8slice": "gemm (8-bit-slice tcgen05 GEMM incl. digit pre-pass)"}[args.precision],
             2: "gemm (8-bit-slice tcgen05 GEMM of the factorisation's Schur updates incl. digit pre-pass)"}
    # algorithmic flops issued in the timed region (every Newton factorisation
    # of a non-Gaussian likelihood included)
    tot_flops = {0: work["factor"] - work["factor_schur"], 1: work["selinv_gemm"], 2: work["factor_schur"]}
    cat_ms = {g: sum(ms_cat[c] for c in cs) for g, cs in groups.items()}
    achieved = tot_flops[dom] / (cat_ms[dom] * 1e-3) / 1e12
    # launch shape of the first member: block, arrow, matrices per launch
    shape = (model.b, model.nb, 2 * Ks[0])
    traffic, traffic_src = roofline_traffic(args.workload, names[dom].split()[0], shape)
    dom_peak, peak_src = peak, "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)"
    try:
        bf16 = float(json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))["bf16_tflops"])
        bf16_src = "measured"
    except Exception:
        bf16, bf16_src = 1590.0, "fallback"
    if (dom == 1 and args.precision == "i8slice") or dom == 2:
        # FP64-equivalent ceiling of 28 int8 digit products per product: the
        # dense int8 rate taken as twice the bf16 burst
        dom_peak = 2 * bf16 / 28
        peak_src = (f"2 x {bf16_src} bf16 burst ({bf16:.0f} TF/s) / 28 digit products "
                    f"(int8 ceiling, FP64-equivalent)")
    # the panel kernel's own rate in the profiled step, whichever group dominates
    panel_rate = (pre_work["factor"] - pre_work["factor_schur"]) / max(pre_ms[0] * 1e-3, 1e-12) / 1e12
    roofline = {
        "bound": "tensor",
        "kernel": names[dom],
        "achieved": achieved,
        "peak": dom_peak,
        "unit": "TFLOP/s",
        "frac": achieved / dom_peak,
        "peak_source": peak_src,
        "avg_launch_ms": cat_ms[dom] / max(cnt_cat[groups[dom][0]], 1),
        "launches": int(cnt_cat[groups[dom][0]]),
        "traffic": traffic,
        "traffic_source": traffic_src,
    }
    # per-category split of the profiled step (events around every launch)
    kernel_ms = {k: pre_ms[i] for i, k in enumerate(["panel", "gemm", "sweep", "trtri", "other", "slice",
                                                    "factor_gemm"])}

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            t_cpu, desc, _ = cpu_sample(args.workload, args.cpu_nt)
            cpu = {"value": 1.0 / t_cpu, "unit": "evals/s", "cores": os.cpu_count(), "kind": "port", "sample": desc}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": "evals/s", "cores": os.cpu_count(), "kind": "port", "sample": repr(exc)}

    if rank == 0:
        cfg0 = config_of(mem[0][0])
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
            "dtype": "f64" if args.precision == "fp64" else (
                f"f64 + {args.precision} selected-inversion products"
                + (f" + {factor_arith} factor Schur updates" if factor_arith != "fp64" else "")),
            "data": "synthetic",
            "config": {
                "workload": args.workload,
                "members": [{"workload": name, "block": m.b, "nt": m.nt, "nb": m.nb, "variates": m.nv,
                             "ns": m.ns, "points_per_step": k} for (name, _), m, k in zip(mem, models, Ks)],
                "obs_per_step": cfg0["no"],
                "theta": list(cfg0["theta"]),
                "path": f"adjoint gradient, selected inversion in {args.precision}, factorisations' Schur updates "
                        f"in {factor_desc} (POTRF, log-dets, "
                        f"solves FP64); {units} theta points per step, theta moved between steps; Q_c and Q_prior of all "
                        f"points factorised and selected-inverted together"
                        + ("; members of different block sizes share every launch" if mixed else ""),
                "theta_points_per_step": units,
                "parallelism": f"replicas x{world}",
                "likelihood": cfg0.get("likelihood", "gaussian"),
                "l2": f"inputs larger than L2 (BTA matrix {model.Qc.buf.numel() * 8 / 1e9:.2f} GB each)",
            },
            "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "autotune": {"decisions": _lib.tune_report(), "extra_warmup_steps": extra,
                         "pending_after_warmup": int(lib.bta_tune_pending())},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "mixed_accuracy": accuracy,
            "fd_fp64_evals_per_s": fd_seq,
            "fd_fp64_batched_stencil_evals_per_s": fd_bat,
            "fd_timing": f"warm (one untimed evaluation first), {args.fd_steps} timed repeats per path",
            "adjoint_single_point_evals_per_s": single_rate,
            "speedup_vs_fd_fp64": (value / fd_seq) if fd_seq else None,
            "speedup_vs_fd_fp64_batched": (value / fd_bat) if fd_bat else None,
            # per-step work of the timed region over the profiled step's kernel times
            "bta_factor_tflops": pre_work["factor"] / max((pre_ms[0] + pre_ms[6]) * 1e-3, 1e-12) / 1e12,
            "panel_roofline": {"achieved": panel_rate, "peak": peak, "unit": "TFLOP/s", "frac": panel_rate / peak,
                               "source": "profiled step; algorithmic flops of the panel kernel's share of the "
                                         "factorisation over its time, vs the in-run cuBLAS DGEMM"},
            "bta_selinv_gemm_tflops": pre_work["selinv_gemm"] / max((pre_ms[1] + pre_ms[5]) * 1e-3, 1e-12) / 1e12,
            "kernel_ms_source": "one profiled step before the timed region (events around every launch); "
                                "in the timed region only the roofline kernel's launches carry events",
            "newton_steps_per_point": (work["newton_steps"] / (units * args.steps)) if not model.gaussian else None,
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
