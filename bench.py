#!/usr/bin/env python
"""Benchmark of the Horn-Schunck hot path on B200: HS Mpix-iters/s and % HBM roofline.

Workload (default): one 1920x1080 FP32 pair (blur 3 px, flow up to 2 px, seed 1000 +
rank), alpha 1, 500 Jacobi sweeps, temporally blocked.  One step = one
hs_forward call (derivatives + 500 sweeps) with the inputs already in HBM, captured once
as a CUDA graph and replayed (the eager call is timed beside it).  Between steps a
256 MiB buffer is written to flush L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 run under torchrun: every rank processes its own pair (pairs are independent;
no collective on the data path), `value` = all ranks' pixel-iterations / the slowest
rank's time.  `--impl reference` times the reference-kernel restatement on the host
cores (the reference's OpenCL backend cannot run here).  Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "HS Mpix-iters/s fwd and fwd+bwd (batched vs plain) on 1 B200; % HBM roofline"
UNIT = "Mpix-iters/s"
BYTES_PER_PX_PASS = 28  # read Ix, Iy, It, u, v; write u, v (FP32)
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sweeps-per-pass", type=int, default=0, help="0 = autotuned")
    ap.add_argument("--layout", type=int, default=0,
                    help="with --sweeps-per-pass: 1 = 2 columns per lane, 2 = 4, 0 = by image size")
    ap.add_argument("--exact", action="store_true", help="bit-exact operation order")
    ap.add_argument("--cpu-sample-sweeps", type=int, default=20)
    ap.add_argument("--shape", default="", help="HxW override (profiling cases)")
    ap.add_argument("--iters", type=int, default=0, help="sweep count override")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-pairs", type=int, default=64,
                    help="pairs of the mixed batch (a prefix of the 64-pair list)")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-sweeps-per-pass", type=int, default=0,
                    help="batched leg: sweeps per pass (0 = autotuned with the rows per tile)")
    ap.add_argument("--batch-rows", type=int, default=0, help="batched leg: rows per tile")
    ap.add_argument("--batch-layout", type=int, default=0,
                    help="batched leg: 1 = 2 columns per lane, 2 = 4, 0 = by pair size")
    ap.add_argument("--no-train", action="store_true")
    ap.add_argument("--train-sweeps-per-pass", type=int, default=5)
    ap.add_argument("--no-pyramid", action="store_true")
    ap.add_argument("--no-cg", action="store_true")
    ap.add_argument("--no-exact-form", action="store_true",
                    help="skip the exact-form leg (its autotuning launches every depth)")
    ap.add_argument("--pyramid-pairs", type=int, default=8)
    ap.add_argument("--no-hm", action="store_true", help="skip the @hm drop-in leg")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5], parts[6], parts[7], parts[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[2:]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------ CPU leg

def c1_sample_rate(O, I0, I1, alpha, sweeps, steps, warm=1):
    """(Mpix-iters/s, seconds) of `steps` warm calls of the C restatement, each running the
    derivatives and `sweeps` sweeps of the whole image (the same loop for the CPU baseline
    and for --impl reference)."""
    for _ in range(warm):
        O.c_hs_forward(I0, I1, alpha, sweeps)
    tot = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        O.c_hs_forward(I0, I1, alpha, sweeps)
        tot += time.perf_counter() - t0
    H, W = I0.shape
    return H * W * sweeps * steps / tot / 1e6, tot


def cpu_leg_timings(I0, I1, alpha, args):
    """The CPU baseline: the reference-kernel restatement (two fused kernels per sweep,
    FP32, OpenMP) timed on the host cores before any GPU work, on bounded samples:
    the 1080p pair (all cores and 1 thread), the whole 256x256 x100 workload, and the
    first 8 pairs of the mixed batch at their full sweep counts."""
    from hindemith_b200 import synthetic
    from oracle import hs_oracle as O

    O.lib()
    cores = O.c_num_threads()
    sweeps = args.cpu_sample_sweeps
    value, _ = c1_sample_rate(O, I0, I1, alpha, sweeps, args.steps, warm=max(args.warmup, 1))
    H, W = I0.shape
    out = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"{W}x{H}, {sweeps} sweeps per step x {args.steps} warm steps (bounded "
                     f"sample of the 500-sweep workload), derivatives included"}
    try:
        O.c_set_num_threads(1)
        one, _ = c1_sample_rate(O, I0, I1, alpha, 5, 2)
    finally:
        O.c_set_num_threads(cores)
    out["one_thread"] = {"value": one, "unit": UNIT, "cores": 1,
                         "sample": f"{W}x{H}, 5 sweeps per step x 2 warm steps"}
    c0 = synthetic.plain_256()
    a0, b0, _, _ = synthetic.generate(c0)
    v0, _ = c1_sample_rate(O, a0, b0, c0.alpha, c0.iters, 5)
    out["c0"] = {"value": v0, "unit": UNIT, "cores": cores,
                 "sample": "256x256, the whole 100-sweep workload, 5 warm steps"}
    sub = synthetic.batch_mixed()[:8]
    pairs = [synthetic.generate(sp) for sp in sub]
    t = 0.0
    for (a, b, _, _), sp in zip(pairs, sub):
        t0 = time.perf_counter()
        O.c_hs_forward(a, b, sp.alpha, sp.iters)
        t += time.perf_counter() - t0
    pix = sum(sp.H * sp.W * sp.iters for sp in sub)
    out["c2_subset"] = {"value": pix / t / 1e6, "unit": UNIT, "cores": cores,
                        "sample": f"the first 8 pairs of the 64-pair mixed batch at their full "
                                  f"sweep counts ({pix / 1e9:.2f} Gpix-it), one pass each; the "
                                  f"rate per pixel-iteration stands for the whole batch"}
    return out


def _flow_err(u, v, ru, rv):
    d = float(max(np.abs(u - ru).max(), np.abs(v - rv).max()))
    scale = float(max(np.abs(ru).max(), np.abs(rv).max(), 1e-30))
    return {"max_abs": d, "rel": d / scale}


def cpu_leg_errors(checks):
    """The checker half of the CPU leg: each flow the GPU legs computed, against the FP64
    oracle (errors: max-abs over u and v; rel = max-abs / max |reference flow|).  Gradients
    against the FP64 reverse-mode oracle and FP64 central differences.  Outside every timed
    region."""
    from oracle import hs_oracle as O

    out = {"definition": "max_abs = max |gpu - fp64| over u and v; rel = max_abs / max |fp64 "
                         "flow|; tolerance 1e-4 max-abs (flows), 1e-3 relative (gradients)"}
    for name in ("c0", "c1"):
        if name not in checks:
            continue
        c = checks[name]
        u64, v64 = O.c_hs_forward(c["I0"], c["I1"], c["alpha"], c["iters"], np.float64)
        e = {"fast": _flow_err(c["fast"][0], c["fast"][1], u64, v64), "fast_config": c["fast_cfg"]}
        if "exact" in c:
            ru, rv = O.c_hs_forward(c["I0"], c["I1"], c["alpha"], c["iters"])
            e["exact"] = _flow_err(c["exact"][0], c["exact"][1], u64, v64)
            e["exact"]["bit_identical_to_fp32_oracle"] = bool(
                np.array_equal(c["exact"][0].view(np.uint32), ru.view(np.uint32))
                and np.array_equal(c["exact"][1].view(np.uint32), rv.view(np.uint32)))
            e["exact_config"] = c["exact_cfg"]
        out[name] = e
    if "c2" in checks:
        worst, per = None, []
        for (a, b, alpha, iters), (u, v) in zip(checks["c2"]["pairs"], checks["c2"]["flows"]):
            u64, v64 = O.c_hs_forward(a, b, alpha, iters, np.float64)
            e = _flow_err(u, v, u64, v64)
            per.append(e["max_abs"])
            if worst is None or e["max_abs"] > worst["max_abs"]:
                worst = e
        out["c2"] = {"pairs": len(per), "max_abs_worst_pair": worst["max_abs"],
                     "rel_worst_pair": worst["rel"], "max_abs_median_pair": float(np.median(per)),
                     "config": checks["c2"]["cfg"]}
    if "c3" in checks:
        out["c3"] = grad_errors(O, checks["c3"])
    if "c4" in checks:
        c = checks["c4"]
        u64, v64 = O.coarse_to_fine_f64(c["I0"], c["I1"], 1.0, c["levels"], c["iters"])
        out["c4"] = dict(_flow_err(c["flow"][0], c["flow"][1], u64, v64),
                         sample=c["sample"])
    return out


def grad_errors(O, c):
    """FP32 gradients of the mean-EPE loss (config 3 settings on a 64x64 crop) against the
    FP64 reverse-mode oracle, and against FP64 central differences at the 4 pixels of each
    image with the largest gradient and for alpha."""
    I0, I1, ut, vt = (np.asarray(x, np.float64) for x in (c["I0"], c["I1"], c["ut"], c["vt"]))
    iters, alpha = c["iters"], c["alpha"]
    n = I0.size
    u, v = O.c_hs_forward(I0, I1, alpha, iters, np.float64)
    r = np.sqrt((u - ut) ** 2 + (v - vt) ** 2 + 1e-12)
    r0, r1, ra, _ = O.hs_adjoint_f64(I0, I1, alpha, iters, (u - ut) / (n * r), (v - vt) / (n * r))
    g0, g1, ga = c["g0"], c["g1"], c["ga"]

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))

    def loss(i0, i1, al):
        uu, vv = O.c_hs_forward(i0, i1, al, iters, np.float64)
        return np.sqrt((uu - ut) ** 2 + (vv - vt) ** 2 + 1e-12).mean()

    h, fd_rel = 1e-4, []
    for g, which in ((g0, 0), (g1, 1)):
        for flat in np.argsort(-np.abs(g).ravel())[:4]:
            i, j = divmod(int(flat), g.shape[1])
            p, m = [I0.copy(), I1.copy()], [I0.copy(), I1.copy()]
            p[which][i, j] += h
            m[which][i, j] -= h
            fd = (loss(*p, alpha) - loss(*m, alpha)) / (2 * h)
            fd_rel.append(abs(g[i, j] - fd) / abs(fd))
    fda = (loss(I0, I1, alpha + h) - loss(I0, I1, alpha - h)) / (2 * h)
    return {"sample": c["sample"],
            "dI0_rel_vs_fp64_adjoint": rel(g0, r0), "dI1_rel_vs_fp64_adjoint": rel(g1, r1),
            "dalpha_rel_vs_fp64_adjoint": abs(ga - ra) / abs(ra),
            "fd_rel_max_8_pixels": float(max(fd_rel)), "dalpha_rel_vs_fd": abs(ga - fda) / abs(fda)}


def cpu_baselines_other():
    """The CPU restatements of the other operators, each on a bounded sample, on all host
    cores (the matrix powers, the preconditioners, LK and the DIA product are OpenMP loops;
    the Brox matrix fill is serial), as rates comparable to the GPU legs."""
    import numpy as np

    from oracle import hs_oracle as O

    rng = np.random.default_rng(1)

    def timed(fn, *a):
        fn(*a)  # warm
        t0 = time.perf_counter()
        fn(*a)
        return time.perf_counter() - t0

    out = {"cores": O.c_num_threads(), "kind": "port"}
    H = W = 1024
    Ix, Iy, r0, r1, d0, d1, od = (rng.standard_normal((H, W)).astype(np.float32) for _ in range(7))
    t = timed(O.c_hs_matrix_powers, 0.5, Ix, Iy, r0, r1, 9)
    out["matrix_powers"] = {"sample": "1024x1024, 9 steps", "ms_per_2048sq_call": t * 4e3}
    t = timed(O.c_apply_hs_precond, 0.25, d0, d1, od, r0, r1)
    out["hs_preconditioner"] = {"sample": "1024x1024", "ms_per_2048sq_call": t * 4e3}
    Hl, Wl = 270, 480
    t = timed(O.c_lk_least_squares, Ix[:Hl, :Wl], Iy[:Hl, :Wl], r0[:Hl, :Wl], 5)
    out["lk"] = {"sample": "480x270, radius 5", "ms_per_1080p_call": t * 16e3}
    psi = np.abs(d0) + 0.1
    t = timed(O.c_set_brox_matrix, psi, 0.5, np.zeros((5, H, W), np.float32))
    data = O.c_set_brox_matrix(psi, 0.5, np.zeros((5, H, W), np.float32))
    t2 = timed(O.c_spmv_dia2d, data, O.BROX_OFFX, O.BROX_OFFY, r0)
    t3 = timed(O.c_apply_brox_precond, data[2], d0, d1, od, r0, r1)
    out["brox"] = {"sample": "1024x1024", "set_matrix_ms_per_2048sq": t * 4e3,
                   "spmv_ms_per_2048sq": t2 * 4e3, "preconditioner_ms_per_2048sq": t3 * 4e3}
    return out


def headline_config(workload, H, W, iters, alpha, world):
    """The headline workload's config, one dict for both arms (GPU and host cores)."""
    return {"workload": workload, "H": H, "W": W, "iters": iters, "alpha": alpha,
            "pairs_per_rank": 1, "parallelism": f"replicas x{world}",
            "l2": "GPU arm: flushed between steps (256 MiB write); the 41 MB working set of "
                  "one pair is L2-resident within a step"}


def run_reference(args, rank, world):
    """--impl reference: the host-core restatement of the reference's kernels."""
    from hindemith_b200 import synthetic

    if rank != 0:
        return None
    spec = synthetic.plain_1080p()
    I0, I1, _, _ = synthetic.generate(spec)
    from oracle import hs_oracle as O

    O.lib()
    sweeps = args.cpu_sample_sweeps
    value, tot = c1_sample_rate(O, I0, I1, spec.alpha, sweeps, args.steps, warm=max(args.warmup, 1))
    cb = {"value": value, "unit": UNIT, "cores": O.c_num_threads(), "kind": "port",
          "sample": f"{spec.W}x{spec.H}, {sweeps} sweeps per step x {args.steps} warm steps "
                    f"(bounded sample of the {spec.iters}-sweep workload), derivatives included"}
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": headline_config("hs_plain_1920x1080_500sweeps", spec.H, spec.W, spec.iters,
                                      spec.alpha, world),
            "sample_sweeps_per_step": sweeps,
            "host_run": "rank 0 runs the host cores; no GPU L2 is involved",
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}



# ------------------------------------------------------------------ extra workloads

def timed_events(fn, k, warmup, flush, stream, label):
    """Sum of K per-step CUDA-event durations (s); L2 flushed between steps."""
    import torch

    for _ in range(warmup):
        fn()
        flush.zero_()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(k)]
    torch.cuda.nvtx.range_push(label)
    for a, b in evs:
        a.record(stream)
        fn()
        b.record(stream)
        flush.zero_()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs) / 1e3


def measure_batched(args, rank, flush, peak, checks=None):
    """The mixed batch (64 pairs, 320x240 .. 2048x2048, alpha in [0.5, 2], 100/200/500
    sweeps): one graph-captured persistent launch, against one plain hs_forward per pair."""
    import torch

    from hindemith_b200 import _lib as L
    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic
    from hindemith_b200.batched import BatchPlan

    from hindemith_b200.autotune import best_batch_config

    specs = synthetic.batch_mixed()[: args.batch_pairs]
    for sp in specs:
        sp.seed += 100 * rank
    shape = [(sp.H, sp.W, sp.alpha, sp.iters) for sp in specs]
    if args.batch_sweeps_per_pass > 0:
        T, rows, layout = args.batch_sweeps_per_pass, args.batch_rows, args.batch_layout
    else:
        T, rows, layout = best_batch_config(shape, fast_math=not args.exact)
    cfg = L.make_config(sweeps_per_pass=T, rows_per_segment=rows, fast_math=not args.exact,
                        layout=layout)
    plan = BatchPlan([(sp.H, sp.W, sp.alpha, sp.iters) for sp in specs], cfg)
    host_pairs = []
    for i, sp in enumerate(specs):
        I0, I1, _, _ = synthetic.generate(sp)
        plan.I0[i].copy_(torch.from_numpy(I0))
        plan.I1[i].copy_(torch.from_numpy(I1))
        if checks is not None:
            host_pairs.append((I0, I1, sp.alpha, sp.iters))
    plan.capture()
    stream = torch.cuda.current_stream()
    t_b = timed_events(plan.replay, args.steps, 3, flush, stream, "timed_batched")
    plan.check()
    outs = [D.empty_planes(2, sp.H, sp.W) for sp in specs]
    # the per-pair calls at the same depth and layout (so the flows are bit-identical), with
    # the per-pair segment rule rather than the batch's tile height
    plain_cfg = L.make_config(sweeps_per_pass=T, fast_math=not args.exact, layout=layout)

    def plain():
        for i, sp in enumerate(specs):
            D.hs_forward(plan.I0[i], plan.I1[i], sp.alpha, sp.iters, plain_cfg, out=(outs[i][0], outs[i][1]))

    t_p = timed_events(plain, max(1, args.steps // 4), 1, flush, stream, "timed_plain_loop")
    same = all(torch.equal(plan.u[i], outs[i][0]) and torch.equal(plan.v[i], outs[i][1])
               for i in range(len(specs)))
    px_it = plan.pixel_iters
    passes = sum(sp.H * sp.W * ((sp.iters + T - 1) // T) for sp in specs)
    achieved = BYTES_PER_PX_PASS * passes * args.steps / t_b / 1e9

    # the same batch at depth 4, where a pass is closer to HBM-bound than issue-bound
    cfg3 = L.make_config(sweeps_per_pass=4, rows_per_segment=96, fast_math=not args.exact,
                         layout=1 if args.exact else 2)
    plan3 = BatchPlan([(sp.H, sp.W, sp.alpha, sp.iters) for sp in specs], cfg3)
    for i in range(len(specs)):
        plan3.I0[i].copy_(plan.I0[i])
        plan3.I1[i].copy_(plan.I1[i])
    plan3.capture()
    t3 = timed_events(plan3.replay, args.steps, 3, flush, stream, "timed_batched_T4")
    plan3.check()
    passes3 = sum(sp.H * sp.W * ((sp.iters + 3) // 4) for sp in specs)
    ach3 = BYTES_PER_PX_PASS * passes3 * args.steps / t3 / 1e9
    same3 = all(torch.equal(plan3.u[i], plan.u[i]) and torch.equal(plan3.v[i], plan.v[i])
                for i in range(len(specs)))
    del plan3
    if checks is not None:
        checks["c2"] = {"pairs": host_pairs,
                        "flows": [(plan.u[i].cpu().numpy(), plan.v[i].cpu().numpy())
                                  for i in range(len(specs))],
                        "cfg": {"sweeps_per_pass": T, "rows_per_tile": rows, "layout": layout,
                                "fast_math": not args.exact}}
    return {
        "workload": f"hs_batched_{len(specs)}pairs_mixed", "pairs": len(specs),
        "mpix": round(sum(sp.H * sp.W for sp in specs) / 1e6, 3), "pix_iters": px_it,
        "sweeps_per_pass": T, "rows_per_tile": rows, "columns_per_lane": 2 * layout if layout else "auto",
        "autotuned": args.batch_sweeps_per_pass == 0,
        "launch": "one persistent kernel per batch, CUDA graph replay",
        "value": px_it * args.steps / t_b / 1e6, "unit": UNIT,
        "ms_per_step": t_b / args.steps * 1e3,
        "plain_loop": {"value": px_it * max(1, args.steps // 4) / t_p / 1e6,
                       "ms_per_step": t_p / max(1, args.steps // 4) * 1e3,
                       "launch": "one hs_forward call per pair, same depth and layout, "
                                 "per-pair segment rows"},
        "identical_to_plain": bool(same),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "bytes_per_px_pass": BYTES_PER_PX_PASS},
        "at_depth_4": {"value": px_it * args.steps / t3 / 1e6, "ms_per_step": t3 / args.steps * 1e3,
                       "rows_per_tile": 96, "columns_per_lane": 2 if args.exact else 4,
                       "identical": bool(same3),
                       "roofline": {"achieved": ach3, "peak": peak, "unit": "GB/s",
                                    "frac": ach3 / peak}},
    }


def measure_train(args, rank, flush, checks=None):
    """Differentiable workload: 16 pairs of 512x512, 200 sweeps, alpha learnable (1.0),
    mean end-point error to the synthetic flow, checkpoints every 10 sweeps; the batched
    training API (one launch per pass for all pairs)."""
    import torch

    from hindemith_b200 import _lib as L
    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic
    from hindemith_b200.autograd import horn_schunck_batch
    from hindemith_b200.loss import mean_epe_batch

    specs = synthetic.batch_512(16)
    data = []
    for sp in specs:
        sp.seed += 100 * rank
        I0, I1, ut, vt = synthetic.generate(sp)
        data.append(tuple(D.as_plane(torch.from_numpy(a).cuda()) for a in (I0, I1, ut, vt)))
    T = args.train_sweeps_per_pass
    cfg = L.make_config(sweeps_per_pass=T, fast_math=not args.exact)
    alpha = torch.tensor(1.0, device="cuda", requires_grad=True)

    def fwd():
        with torch.no_grad():
            horn_schunck_batch([(d[0], d[1]) for d in data], alpha, 200, 10, cfg)

    def fwd_bwd():
        alpha.grad = None
        xs = [(d[0].detach().requires_grad_(True), d[1].detach().requires_grad_(True)) for d in data]
        outs = horn_schunck_batch(xs, alpha, 200, 10, cfg)
        mean_epe_batch(outs, [(d[2], d[3]) for d in data]).backward()

    stream = torch.cuda.current_stream()
    k = max(1, args.steps // 4)
    t_f_eager = timed_events(fwd, k, 3, flush, stream, "timed_train_fwd_eager")
    t_fb_eager = timed_events(fwd_bwd, k, 3, flush, stream, "timed_train_fwd_bwd_eager")

    # Both as CUDA graphs: a launch of this workload's passes takes about 50 us of device
    # time, close to what the host needs to enqueue one, so the eager timings carry host
    # time.  The graphs hold the same launches.
    def fwd_bwd_fn():
        # fresh leaves per call: an autograd leaf remembers the stream it was first used on
        a = alpha.detach().requires_grad_(True)
        xs = [(d[0].detach().requires_grad_(True), d[1].detach().requires_grad_(True)) for d in data]
        outs = horn_schunck_batch(xs, a, 200, 10, cfg)
        loss = mean_epe_batch(outs, [(d[2], d[3]) for d in data])
        return (loss, *torch.autograd.grad(loss, [a] + [t for p in xs for t in p]))

    graphs = []
    for fn in (fwd, fwd_bwd_fn):
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            fn()
        stream.wait_stream(side)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            keep = fn()
        graphs.append((g, keep))
    torch.cuda.synchronize()
    t_f = timed_events(graphs[0][0].replay, k, 3, flush, stream, "timed_train_fwd")
    t_fb = timed_events(graphs[1][0].replay, k, 3, flush, stream, "timed_train_fwd_bwd")
    del graphs
    px_it = sum(sp.H * sp.W * sp.iters for sp in specs)

    # the single-pair form (horn_schunck: hs_forward_train + hs_backward) on pair 0
    from hindemith_b200.autograd import horn_schunck

    def one_fwd():
        with torch.no_grad():
            horn_schunck(data[0][0], data[0][1], alpha, 200, 10, cfg)

    def one_fwd_bwd():
        alpha.grad = None
        x0 = data[0][0].detach().requires_grad_(True)
        x1 = data[0][1].detach().requires_grad_(True)
        u, v = horn_schunck(x0, x1, alpha, 200, 10, cfg)
        mean_epe_batch([(u, v)], [(data[0][2], data[0][3])]).backward()

    t1f = timed_events(one_fwd, k, 3, flush, stream, "timed_single_fwd")
    t1fb = timed_events(one_fwd_bwd, k, 3, flush, stream, "timed_single_fwd_bwd")
    single = {"workload": "one 512x512 pair, 200 sweeps, checkpoints every 10",
              "api": "horn_schunck (hs_forward_train + hs_backward)",
              "fwd_ms": t1f / k * 1e3, "fwd_bwd_ms": t1fb / k * 1e3,
              "fwd_bwd_over_fwd": t1fb / t1f}
    if checks is not None:
        # the gradient check: pair 0's top-left 64x64 crop, the same settings and config
        I0, I1, ut, vt = (a[:64, :64].copy() for a in synthetic.generate(specs[0]))
        a = torch.tensor(1.0, device="cuda", requires_grad=True)
        xs = [(D.as_plane(torch.from_numpy(I0).cuda()).requires_grad_(True),
               D.as_plane(torch.from_numpy(I1).cuda()).requires_grad_(True))]
        outs = horn_schunck_batch(xs, a, 200, 10, cfg)
        mean_epe_batch(outs, [(D.as_plane(torch.from_numpy(ut).cuda()),
                               D.as_plane(torch.from_numpy(vt).cuda()))]).backward()
        checks["c3"] = {"I0": I0, "I1": I1, "ut": ut, "vt": vt, "iters": 200, "alpha": 1.0,
                        "g0": xs[0][0].grad.cpu().numpy(), "g1": xs[0][1].grad.cpu().numpy(),
                        "ga": float(a.grad),
                        "sample": "pair 0 of the 16x512x512 batch, top-left 64x64 crop, 200 "
                                  "sweeps, checkpoints every 10, mean EPE, the timed config"}
    return {"workload": "hs_train_16x512x512_200sweeps_ckpt10", "pix_iters": px_it,
            "sweeps_per_pass": T, "api": "horn_schunck_batch (hs_forward_train_batched + hs_backward_batched) + mean_epe_batch",
            "timed": "forward, and forward + loss + backward, each captured once as a CUDA graph "
                     "and replayed",
            "fwd_ms": t_f / k * 1e3, "fwd_bwd_ms": t_fb / k * 1e3,
            "fwd_bwd_over_fwd": t_fb / t_f,
            "eager": {"fwd_ms": t_f_eager / k * 1e3, "fwd_bwd_ms": t_fb_eager / k * 1e3,
                      "fwd_bwd_over_fwd": t_fb_eager / t_f_eager},
            "fwd_value": px_it * k / t_f / 1e6,
            "value": px_it * k / t_fb / 1e6, "unit": UNIT + " (forward+backward)",
            "single_pair": single}


def measure_pyramid(args, rank, flush, checks=None):
    """Coarse-to-fine workload: 8 pairs of 2048x2048 with flow up to 12 px, 4 levels
    (binomial blur + decimation), warp of I1 by the upsampled flow at each finer level,
    100 sweeps per level checkpointed every 10, loss = mean end-point error; forward and
    backward through all levels captured in ONE CUDA graph and replayed."""
    import torch

    from hindemith_b200 import _lib as L
    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic
    from hindemith_b200.loss import mean_epe_batch
    from hindemith_b200.pyramid import coarse_to_fine

    specs = synthetic.batch_pyramid(args.pyramid_pairs)
    levels, iters = 4, 100
    data = []
    for sp in specs:
        sp.seed += 100 * rank
        I0, I1, ut, vt = synthetic.generate(sp)
        data.append(tuple(D.as_plane(torch.from_numpy(a).cuda()) for a in (I0, I1, ut, vt)))
    cfg = L.make_config(sweeps_per_pass=args.train_sweeps_per_pass, fast_math=not args.exact)
    alpha0 = torch.tensor(1.0, device="cuda")

    def fwd_bwd():
        # fresh leaves per call: an autograd leaf remembers the stream it was first used on
        alpha = alpha0.detach().requires_grad_(True)
        xs = [(d[0].detach().requires_grad_(True), d[1].detach().requires_grad_(True))
              for d in data]
        flows = coarse_to_fine(xs, alpha, levels, iters, 10, cfg)
        loss = mean_epe_batch(flows, [(d[2], d[3]) for d in data])
        return (loss, *torch.autograd.grad(loss, [alpha] + [t for p in xs for t in p]))

    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated()
    torch.cuda.reset_peak_memory_stats()
    eager = fwd_bwd()
    torch.cuda.synchronize()
    eager_peak = torch.cuda.max_memory_allocated() - base
    del eager
    stream = torch.cuda.current_stream()
    k = max(1, args.steps // 4)
    t_eager = timed_events(fwd_bwd, k, 1, flush, stream, "timed_pyramid_eager")
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        fwd_bwd()
    stream.wait_stream(side)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        outs = fwd_bwd()
    torch.cuda.synchronize()
    graph_peak = torch.cuda.max_memory_allocated() - base
    t_graph = timed_events(graph.replay, k, 3, flush, stream, "timed_pyramid_graph")
    loss = float(outs[0].detach())
    px_it = sum(sum(((sp.H + (1 << l) - 1) >> l) * ((sp.W + (1 << l) - 1) >> l)
                    for l in range(levels)) * iters for sp in specs)
    del outs, graph
    if checks is not None:
        with torch.no_grad():
            flow = coarse_to_fine([(data[0][0], data[0][1])], alpha0, levels, iters, 10, cfg)[0]
        checks["c4"] = {"I0": data[0][0].cpu().numpy(), "I1": data[0][1].cpu().numpy(),
                        "levels": levels, "iters": iters,
                        "flow": (flow[0].cpu().numpy(), flow[1].cpu().numpy()),
                        "sample": "pair 0 of the 8x2048x2048 batch, 4 levels x 100 sweeps, "
                                  "the timed config"}
    return {"workload": f"hs_pyramid_{len(specs)}x2048x2048_4levels_100sweeps_ckpt10",
            "pix_iters_fwd": px_it, "sweeps_per_pass": args.train_sweeps_per_pass,
            "api": "pyramid.coarse_to_fine (hs_blur_down, hs_upsample2, hs_warp, batched HS) "
                   "+ torch.autograd.grad, one CUDA graph",
            "fwd_bwd_ms": t_graph / k * 1e3, "fwd_bwd_eager_ms": t_eager / k * 1e3,
            "value": px_it * k / t_graph / 1e6, "unit": UNIT + " (forward+backward, all levels)",
            "loss": loss, "peak_device_bytes": int(max(eager_peak, graph_peak)),
            "peak_device_bytes_eager": int(eager_peak), "peak_device_bytes_graph": int(graph_peak),
            "input_bytes": int(base)}


def flow_magnitude(I0, I1, Dx, Dy, Dt, eps):
    """A generic @hm program (not the HS loop): derivative stencils, gradient magnitude,
    its normalisation by the plane sum."""
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    m = sqrt(Ix * Ix + Iy * Iy + eps)  # noqa: F821 (the @hm surface's sqrt)
    return m / sum2d(m), It  # noqa: F821


def measure_fusion_flow(args, rank, flush, peak):
    """Generic fusion (the program above at 1920x1080, fused vs one operator per statement),
    Lucas-Kanade (1920x1080, radius 5) and the Brox pieces (2048x2048)."""
    import numpy as np
    import torch

    from hindemith_b200 import SpMat2D, brox_offsets, hm, hs_derivative_stencils
    from hindemith_b200 import device as D
    from hindemith_b200 import flow as FL
    from hindemith_b200 import hindemith as HM

    stream = torch.cuda.current_stream()
    k = max(1, args.steps)
    g = torch.Generator(device="cuda")
    g.manual_seed(11 + rank)
    H, W = 1080, 1920
    I0, I1 = (torch.rand((H, W), device="cuda", generator=g) for _ in range(2))
    Dx, Dy, Dt = hs_derivative_stencils()
    out = {}
    f = hm(flow_magnitude)
    kw = dict(I0=I0, I1=I1, Dx=Dx, Dy=Dy, Dt=Dt, eps=np.float32(1e-3))
    old = dict(HM.defines)
    try:
        for fuse in (True, False):
            HM.defines["hs_fuse"] = fuse
            t = timed_events(lambda: f(**kw), k, 3, flush, stream, "timed_fusion")
            out["fused_ms" if fuse else "unfused_ms"] = t / k * 1e3
            if fuse:
                out["fused_kernels_per_call"] = HM.state["last_stats"].get("fused_launches", 0)
    finally:
        HM.defines.clear()
        HM.defines.update(old)
    # fused bytes: read I0, I1 (twice: two groups read what they need) + write It, n, m once
    out["fused_bytes_per_px"] = 4 * (2 + 1 + 1 + 1 + 1)
    out["fused_gbs"] = out["fused_bytes_per_px"] * H * W / (out["fused_ms"] / 1e3) / 1e9
    err, Ix, Iy = D.empty_planes(3, H, W)
    for p in (err, Ix, Iy):
        p.copy_(torch.rand((H, W), device="cuda", generator=g) - 0.5)
    t = timed_events(lambda: FL.lk_least_squares(err, Ix, Iy, 5), k, 3, flush, stream, "timed_lk")
    lk_flops = H * W * (2 * 5) ** 2 * 10
    # The window sums' adds are fixed by the reference order (5 per window cell, 100 cells);
    # they bound the kernel on the FP32 pipe (128 lanes per SM per clock).
    lk_adds = H * W * (2 * 5) ** 2 * 5
    fp32_peak = torch.cuda.get_device_properties(0).multi_processor_count * 128 * 1965e6
    out["lk"] = {"workload": "lk_least_squares_1920x1080_radius5", "ms": t / k * 1e3,
                 "gflops": lk_flops * k / t / 1e9, "bound": "fp32 pipe",
                 "roofline": {"order_fixed_adds_per_px": 500, "achieved_tops": lk_adds * k / t / 1e12,
                              "peak_tops": fp32_peak / 1e12, "frac": lk_adds * k / t / fp32_peak,
                              "peak_source": "SMs x 128 FP32 lanes x clocks.max.sm (1965 MHz)"}}
    Hb = Wb = 2048
    psi, x, d0, d1, od = D.empty_planes(5, Hb, Wb)
    for p in (psi, x, d0, d1, od):
        p.copy_(torch.rand((Hb, Wb), device="cuda", generator=g) + 0.1)
    offx, offy = brox_offsets()
    A = FL.DeviceSpMat2D.from_host(SpMat2D(np.zeros((5, Hb, Wb), np.float32), offx, offy))
    t_set = timed_events(lambda: FL.set_brox_matrix(A, psi, 0.5), k, 3, flush, stream, "timed_brox_set")
    t_mv = timed_events(lambda: FL.spmv_dia2d(A, x), k, 3, flush, stream, "timed_spmv")
    t_pc = timed_events(lambda: FL.apply_brox_preconditioner(A, d0, d1, od, x, psi), k, 3, flush,
                        stream, "timed_brox_precond")
    px = Hb * Wb
    out["brox"] = {"workload": "brox_2048x2048",
                   "set_matrix": {"ms": t_set / k * 1e3, "gbs": 24 * px * k / t_set / 1e9},
                   "spmv_dia2d": {"ms": t_mv / k * 1e3, "gbs": 28 * px * k / t_mv / 1e9},
                   "preconditioner": {"ms": t_pc / k * 1e3, "gbs": 36 * px * k / t_pc / 1e9},
                   "peak_gbs": peak}
    out["workload"] = ("flow_magnitude_1920x1080 (@hm call end to end, including the host "
                       "read of sum2d; fused vs one operator per statement)")
    return out


def hs_program(I0, I1, Dx, Dy, Dt, A, alpha, u, v):
    """The Horn-Schunck program as a Hindemith user writes it (integer-literal loop bound,
    alpha squared by a scalar statement): the drop-in's own workload."""
    alpha2 = alpha * alpha
    Ix = Dx * I0 + Dx * I1
    Iy = Dy * I0 + Dy * I1
    It = Dt * I1 - Dt * I0
    den = alpha2 + Ix * Ix + Iy * Iy
    for i in range(500):
        ubar = A * u
        vbar = A * v
        t = (Ix * ubar + Iy * vbar + It) / den
        u = ubar - Ix * t
        v = vbar - Iy * t
    return u, v


def measure_hm(args, rank, flush, I0, I1, I0h, I1h, spec):
    """The drop-in: the Horn-Schunck program above through @hm at 1920x1080 x500, with no
    tuning keys in `defines` (the front end autotunes the fused sweep per shape), in the
    exact form (the default: the reference's FP32 operation order) and the fast form;
    device-resident torch inputs, and NumPy host inputs (copies in and out included)."""
    import numpy as np
    import torch

    from hindemith_b200 import hm, hs_average_stencil, hs_derivative_stencils
    from hindemith_b200 import hindemith as HM

    stream = torch.cuda.current_stream()
    f = hm(hs_program)
    Dx, Dy, Dt = hs_derivative_stencils()
    A = hs_average_stencil()
    z = torch.zeros_like(I0)
    zh = np.zeros_like(I0h)
    k = max(1, args.steps // 2)
    px_it = spec.H * spec.W * 500
    out = {"workload": "hs_program_1920x1080_500sweeps via @hm (keyword arguments, no defines)"}
    old = dict(HM.defines)
    try:
        for form, fast in (("exact", False), ("fast", True)):
            HM.defines.clear()
            if fast:
                HM.defines["hs_fast_math"] = True
            kw = dict(I0=I0, I1=I1, Dx=Dx, Dy=Dy, Dt=Dt, A=A, alpha=np.float32(spec.alpha),
                      u=z, v=z)
            f(**kw)  # compile + autotune (cached per shape)
            t = timed_events(lambda: f(**kw), k, 3, flush, stream, f"timed_hm_{form}")
            kwh = dict(kw, I0=I0h, I1=I1h, u=zh, v=zh)
            th = timed_events(lambda: f(**kwh), k, 1, flush, stream, f"timed_hm_{form}_numpy")
            out[form] = {"value": px_it * k / t / 1e6, "unit": UNIT, "ms_per_call": t / k * 1e3,
                         "numpy_in_out": {"value": px_it * k / th / 1e6, "unit": UNIT,
                                          "ms_per_call": th / k * 1e3}}
    finally:
        HM.defines.clear()
        HM.defines.update(old)
    return out


def measure_cg(args, rank, flush, peak):
    """Horn-Schunck as a linear system at 2048x2048: 9 Krylov powers of the HS operator
    (hs_matrix_powers, 4 powers per pass) and one block-Jacobi preconditioner application,
    as HBM GB/s against the measured peak."""
    import torch

    from hindemith_b200 import _lib as L
    from hindemith_b200 import cg
    from hindemith_b200 import device as D

    H = W = 2048
    g = torch.Generator(device="cuda")
    g.manual_seed(5 + rank)
    planes = D.empty_planes(7, H, W)
    for p in planes:
        p.copy_(torch.rand((H, W), device="cuda", generator=g) - 0.5)
    Ix, Iy, r0, r1, d0, d1, od = planes
    steps, depth = 9, 4
    cfg = L.make_config(sweeps_per_pass=depth)
    stream = torch.cuda.current_stream()
    k = max(1, args.steps)

    def powers():
        cg.hs_matrix_powers(0.5, Ix, Iy, r0, r1, steps, cfg)

    def precond():
        cg.apply_hs_preconditioner(0.25, d0, d1, od, r0, r1)

    t_mp = timed_events(powers, k, 3, flush, stream, "timed_matrix_powers")
    t_pc = timed_events(precond, k, 3, flush, stream, "timed_preconditioner")
    passes = (steps - 1 + depth - 1) // depth
    # each pass reads one power (u, v) and Ix, Iy: 16 B/px; every power V[0..steps-1] is
    # written once: 8 B/px each (V[0] by the first pass, from the r it reads)
    mp_bytes = H * W * (16 * passes + 8 * steps)
    pc_bytes = H * W * 28
    mp_gbs = mp_bytes * k / t_mp / 1e9
    pc_gbs = pc_bytes * k / t_pc / 1e9
    return {"workload": "hs_matrix_powers_2048x2048_9steps + hs_apply_hs_preconditioner_2048x2048",
            "matrix_powers": {"ms": t_mp / k * 1e3, "powers_per_pass": depth,
                              "bytes_per_call": mp_bytes, "achieved_gbs": mp_gbs,
                              "frac": mp_gbs / peak},
            "preconditioner": {"ms": t_pc / k * 1e3, "bytes_per_call": pc_bytes,
                               "achieved_gbs": pc_gbs, "frac": pc_gbs / peak}}


def e2e_pipelined(I0h, I1h, alpha, iters, cfg, steps, flush, dist=None):
    """Seconds for `steps` host-to-host hs_forward steps.  Copies in and out run on their
    own streams (double-buffered device planes), so step k+1's inputs arrive and step
    k-1's flow leaves while step k sweeps."""
    import torch

    from hindemith_b200 import device as D

    H, W = I0h.shape
    comp = torch.cuda.current_stream()
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()
    I0p = torch.from_numpy(I0h).pin_memory()
    I1p = torch.from_numpy(I1h).pin_memory()
    outs_h = [torch.empty((2, H, W), dtype=torch.float32).pin_memory() for _ in range(2)]
    ins_d = [D.empty_planes(2, H, W) for _ in range(2)]
    outs_d = [D.empty_planes(2, H, W) for _ in range(2)]

    def run(n, after=None):
        h2d = [torch.cuda.Event() for _ in range(n)]
        done = [torch.cuda.Event() for _ in range(n)]
        d2h = [torch.cuda.Event() for _ in range(n)]

        def copy_in(k):
            with torch.cuda.stream(cin):
                if after is not None:
                    cin.wait_event(after)
                if k >= 2:
                    cin.wait_event(done[k - 2])  # step k-2's sweeps are done with ins_d[b]
                ins_d[k & 1][0].copy_(I0p, non_blocking=True)
                ins_d[k & 1][1].copy_(I1p, non_blocking=True)
                h2d[k].record(cin)

        copy_in(0)
        for k in range(n):
            b = k & 1
            if k + 1 < n:
                copy_in(k + 1)
            comp.wait_event(h2d[k])
            if k >= 2:
                comp.wait_event(d2h[k - 2])  # outs_d[b] has left
            D.hs_forward(ins_d[b][0], ins_d[b][1], alpha, iters, cfg, out=(outs_d[b][0], outs_d[b][1]))
            done[k].record(comp)
            flush.zero_()
            with torch.cuda.stream(cout):
                cout.wait_event(done[k])
                outs_h[b].copy_(outs_d[b], non_blocking=True)
                d2h[k].record(cout)
        return d2h[-1]

    for _ in range(2):
        run(2)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(comp)
    last = run(steps, after=start)
    comp.wait_event(last)
    end.record(comp)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return start.elapsed_time(end) / 1e3


# ------------------------------------------------------------------ GPU arm

def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch

    from hindemith_b200 import _lib as L
    from hindemith_b200 import device as D
    from hindemith_b200 import synthetic
    from hindemith_b200 import autotune
    from hindemith_b200.replicas import job_rate, max_over_ranks, rank_seed

    spec = synthetic.plain_1080p()
    spec.seed = rank_seed(spec.seed, rank)
    workload = "hs_plain_1920x1080_500sweeps"
    if args.shape:
        spec.H, spec.W = (int(x) for x in args.shape.lower().split("x"))
        workload = f"hs_plain_{spec.W}x{spec.H}"
    if args.iters > 0:
        spec.iters = args.iters
        workload += f"_{spec.iters}sweeps" if args.shape else ""
    I0h, I1h, _, _ = synthetic.generate(spec)
    H, W, iters, alpha = spec.H, spec.W, spec.iters, spec.alpha
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    # The CPU baseline runs first, before this process touches CUDA (the driver's threads
    # take host cycles once a context exists: about 20 % of the 16-core rate was measured
    # lost), with the same warm loop as --impl reference.
    cpu_times = cpu_leg_timings(I0h, I1h, alpha, args) if cpu_leg else None

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device (libhsflow has no CPU path)")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    warmup = max(args.warmup, 3)
    checks = {}
    I0 = D.as_plane(torch.from_numpy(I0h).cuda())
    I1 = D.as_plane(torch.from_numpy(I1h).cuda())
    ld = D.ld_of(I0)
    stream = torch.cuda.current_stream()

    if args.sweeps_per_pass > 0:
        T, seg, layout = args.sweeps_per_pass, 0, args.layout
    else:
        T, seg, layout = autotune.best_sweep_config(H, W, ld, fast_math=not args.exact, sweeps=iters)
    cfg = L.make_config(sweeps_per_pass=T, rows_per_segment=seg, fast_math=not args.exact,
                        layout=layout)
    # the layout the library runs (hs_config.layout 0 chooses by image size)
    wide = (not args.exact) and (layout == 2 or (layout == 0 and H * W >= 2_000_000))
    passes = (iters + T - 1) // T
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    uv = D.empty_planes(2, H, W)
    u, v = uv[0], uv[1]

    def step():
        D.hs_forward(I0, I1, alpha, iters, cfg, out=(u, v))

    def timed(fn, k, w, label):
        for _ in range(w):
            fn()
            flush.zero_()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(k)]
        torch.cuda.nvtx.range_push(label)
        for a, b in evs:
            a.record(stream)
            fn()
            b.record(stream)
            flush.zero_()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / 1e3  # seconds

    # The step (derivatives, zeroing, all passes: one hs_forward call) as one CUDA graph, so
    # that host launch jitter stays out of the device timing; the eager call is timed too.
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        for _ in range(2):
            step()
    stream.wait_stream(side)
    torch.cuda.synchronize()
    step_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(step_graph):
        step()
    torch.cuda.synchronize()

    with ClockSampler(torch.cuda.current_device()) as clk:
        t_step = timed(step_graph.replay, args.steps, warmup, "timed_step")
        t_step_eager = timed(step, args.steps, warmup, "timed_step_eager")
        # sweep passes alone (the dominant kernel), same configuration, for the roofline
        Ixyt = D.hs_derivs(I0, I1)
        us, vs = D.empty_planes(2, H, W)

        def sweeps_only():
            D.hs_sweeps(*Ixyt, alpha * alpha, iters, us, vs, cfg)

        us.zero_(), vs.zero_()
        t_sweeps = timed(sweeps_only, args.steps, 2, "timed_sweeps")
        # the same step in the exact form (the drop-in's default: the reference program's
        # FP32 operations one rounding at a time, 2 columns per lane, its own tuned depth)
        t_exact = None
        if not args.exact and not args.shape and not args.no_exact_form:
            Te, sege, _ = autotune.best_sweep_config(H, W, ld, fast_math=False, sweeps=iters)
            cfg_e = L.make_config(sweeps_per_pass=Te, rows_per_segment=sege)

            def exact_step():
                D.hs_forward(I0, I1, alpha, iters, cfg_e, out=(u, v))

            t_exact = timed(exact_step, max(1, args.steps // 2), 2, "timed_exact")
        # end to end through the public API: every step copies its pair in from pinned
        # host memory and its flow out to pinned host memory; the copies of one step overlap
        # the sweeps of the previous one (a copy stream, double-buffered device planes), as
        # a frame pipeline would run.  Timed from the first copy-in to the last copy-out,
        # with the L2 flush between steps on the compute stream (counted).
        t_e2e = e2e_pipelined(I0h, I1h, alpha, iters, cfg, args.steps, flush, dist)
    clocks = clk.summary()
    if cpu_leg:
        # flows of the timed configurations, for the checker (outside the timed regions)
        fu, fv = D.hs_forward(I0, I1, alpha, iters, cfg)
        c1 = {"I0": I0h, "I1": I1h, "alpha": alpha, "iters": iters,
              "fast": (fu.cpu().numpy(), fv.cpu().numpy()),
              "fast_cfg": {"sweeps_per_pass": T, "rows_per_segment": seg, "layout": layout,
                           "fast_math": not args.exact}}
        if t_exact is not None:
            eu, ev = D.hs_forward(I0, I1, alpha, iters, cfg_e)
            c1["exact"] = (eu.cpu().numpy(), ev.cpu().numpy())
            c1["exact_cfg"] = {"sweeps_per_pass": Te, "rows_per_segment": sege}
        checks["c1"] = c1
        if not args.shape:
            c0 = synthetic.plain_256()
            a0, b0, _, _ = synthetic.generate(c0)
            d0, d1 = D.as_plane(torch.from_numpy(a0).cuda()), D.as_plane(torch.from_numpy(b0).cuda())
            T0, s0, l0 = autotune.best_sweep_config(c0.H, c0.W, D.ld_of(d0), fast_math=True,
                                                    sweeps=c0.iters)
            cf0 = L.make_config(sweeps_per_pass=T0, rows_per_segment=s0, fast_math=True, layout=l0)
            fu, fv = D.hs_forward(d0, d1, c0.alpha, c0.iters, cf0)
            eu, ev = D.hs_forward(d0, d1, c0.alpha, c0.iters)  # the library's default config
            checks["c0"] = {"I0": a0, "I1": b0, "alpha": c0.alpha, "iters": c0.iters,
                            "fast": (fu.cpu().numpy(), fv.cpu().numpy()),
                            "fast_cfg": {"sweeps_per_pass": T0, "rows_per_segment": s0,
                                         "layout": l0, "fast_math": True},
                            "exact": (eu.cpu().numpy(), ev.cpu().numpy()),
                            "exact_cfg": "hs_config zeroed (library default)"}

    t_step, t_step_eager, t_sweeps, t_e2e = max_over_ranks([t_step, t_step_eager, t_sweeps, t_e2e])
    if t_exact is not None:
        t_exact = max_over_ranks([t_exact])[0]

    px_iters = H * W * iters * args.steps * world
    value = job_rate(H * W * iters * args.steps, world, t_step) / 1e6
    e2e_value = job_rate(H * W * iters * args.steps, world, t_e2e) / 1e6
    peak, peak_kind = load_peaks()
    launch_s = t_sweeps / (args.steps * passes)
    achieved = BYTES_PER_PX_PASS * H * W / launch_s / 1e9
    # the wide kernel's main loop is unrolled from 3 Mpx up (kUnrollPixels in hs_sweep.cu),
    # the 2-column kernel's at depths 1 and 2
    big = H * W >= 3000000
    kernel = (f"hs_stream_w_kernel<{T},{'true' if big else 'false'}>" if wide else
              f"hs_stream_kernel<{T},{'false' if args.exact else 'true'},"
              f"{'true' if T <= 2 else 'false'}>")
    # ncu figures of this very kernel at this shape (profiles/), when one was captured
    traffic, prof = None, {}
    tpath = os.path.join(HERE, "profiles", "sweep_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            prof = json.load(f)["kernels"].get(f"{kernel}|{W}x{H}", {})
        traffic = prof.get("dram_bytes")
    # issue slots the launch used: its warp instructions over the SMSPs' slots in its time
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    issue_frac = (prof["inst"] / (launch_s * torch.cuda.get_device_properties(0).multi_processor_count
                                  * 4 * sm_mhz * 1e6) if "inst" in prof else None)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": warmup, "ms_per_step": t_step / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded blurred noise + sinusoidal flow; see hindemith_b200/synthetic.py)",
        "config": headline_config(workload, H, W, iters, alpha, world),
        "tuning": {"sweeps_per_pass": T, "rows_per_segment": seg,
                   "columns_per_lane": 4 if wide else 2, "fast_math": not args.exact,
                   "autotuned": args.sweeps_per_pass == 0},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": kernel, "peak_source": peak_kind,
                     "bytes_per_launch": BYTES_PER_PX_PASS * H * W,
                     "avg_launch_us": launch_s * 1e6,
                     "traffic_source": prof.get("summary"),
                     "issue_slot_frac": issue_frac,
                     "note": "at 1920x1080 the pair's 41.5 MB working set is L2-resident within "
                             "a step: the kernel is issue/latency-bound, so issue_slot_frac (the "
                             "profiled warp instructions per launch over 4 issue slots x SMs x "
                             "the sampled SM clock x the live launch time) is its binding "
                             "fraction"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * H * W * 4,
                "d2h_bytes_per_step": 2 * H * W * 4, "ms_per_step": t_e2e / args.steps * 1e3,
                "pipeline": "pinned host -> device -> pinned host every step; copy-in and "
                            "copy-out streams overlap step k+1's and k-1's copies with step k's "
                            "sweeps"},
        "step": {"timed": "one hs_forward call per step, captured once as a CUDA graph and "
                          "replayed (the eager call beside it)",
                 "eager_ms_per_step": t_step_eager / args.steps * 1e3,
                 "eager_value": job_rate(H * W * iters * args.steps, world, t_step_eager) / 1e6},
        "exact_form": (None if t_exact is None else
                       {"value": H * W * iters * max(1, args.steps // 2) / t_exact / 1e6,
                        "unit": UNIT, "sweeps_per_pass": Te, "rows_per_segment": sege,
                        "note": "bit-identical to the reference's FP32 semantics"}),
        "gpu_launches": (1 + passes) * args.steps,
        "clocks": clocks,
    }
    # the batched and differentiable workloads are single-GPU measurements
    if world == 1 and not args.no_batched and not args.shape:
        line["batched"] = measure_batched(args, rank, flush, peak, checks if cpu_leg else None)
    if world == 1 and not args.no_train and not args.shape:
        line["fwd_bwd"] = measure_train(args, rank, flush, checks if cpu_leg else None)
    if world == 1 and not args.no_cg and not args.shape:
        line["cg"] = measure_cg(args, rank, flush, peak)
        line["fusion_lk_brox"] = measure_fusion_flow(args, rank, flush, peak)
    if world == 1 and not args.no_pyramid and not args.shape:
        line["pyramid"] = measure_pyramid(args, rank, flush, checks if cpu_leg else None)
    if world == 1 and not args.no_hm and not args.shape:
        line["hm_dropin"] = measure_hm(args, rank, flush, I0, I1, I0h, I1h, spec)
    if cpu_leg:
        line["cpu_baseline"] = cpu_times
        if "cg" in line:
            line["cpu_baseline_other_operators"] = cpu_baselines_other()
        line["errors_vs_fp64_oracle"] = cpu_leg_errors(checks)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
