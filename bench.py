#!/usr/bin/env python
"""Kernel-sum benchmark of the B200 LDDMM hot path.

Workload (the kernel-sum microbenchmark configuration): N = M = 1,048,576
points uniform in [0,1]^3 (seeded), momenta a ~ N(0,1)^3 on the sources and
p ~ N(0,1)^3 on the targets; Gaussian kernel sigma = 0.05 and order-3
Laplacian (Matern) kernel sigma = 0.05.  One step evaluates, in FP32 with
compensated accumulation (FP64 outputs):
    applyK      K(x, y) a                 (Gaussian)
    applyDiffKT grad_x <p, K(x, y) a>     (Gaussian)
    applyK / applyDiffKT                  (Laplacian order 3)
i.e. 4 * N * M target-source pairs.  Metric: kernel-sum pairs/s (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): each rank sweeps its own seeded instance (weak scaling,
no data-path collective); the time is the max over ranks.
The reference arm (--impl reference) times the reference algorithm's CPU
implementation (the FP64 C/OpenMP restatement of kernelFunctions.f90) on all
host cores, on a bounded sample of target rows against all sources.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIGMA = 0.05
OPS = [  # name, kernel, op, flops/pair, FMA-pipe instr/pair, XU ops/pair (per-pair counts of the workload table)
    ("applyK_gauss", "gauss", "K", 15, 10, 1),
    ("applyDiffKT_gauss", "gauss", "DKT", 21, 14, 1),
    ("applyK_lap3", "laplacian", "K", 24, 16, 2),
    ("applyDiffKT_lap3", "laplacian", "DKT", 28, 19, 2),
]
LAUNCHES_PER_OP = {"K": 5, "DKT": 6}  # pack x2 (+1 or 2 value packs), sweep, combine


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--seed", type=int, default=20240601)
    ap.add_argument("--cpu-seconds", type=float, default=16.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    return ap.parse_args()


def make_inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, 3))
    y = rng.uniform(0, 1, (n, 3))
    a = rng.standard_normal((n, 3))
    p = rng.standard_normal((n, 3))
    return x, y, a, p


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[1:]:   # first sample may precede the load
            parts = [q.strip() for q in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_median": float(np.median(power)) if power else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def gpu_id_for(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


# ---------------------------------------------------------------------------
# reference arm: the CPU implementation of the reference algorithm
# ---------------------------------------------------------------------------
def cpu_sample_rows(oracle, x, y, a, p, budget_s):
    """Chooses a target-row sample size so the 4 ops take about budget_s."""
    rows = 16
    t0 = time.perf_counter()
    oracle.applyk(x[:rows], y, a, SIGMA, 10)
    dt = max(time.perf_counter() - t0, 1e-4)
    per_row_all_ops = dt / rows * 4.5     # Laplacian and derivative sums cost a bit more
    return int(max(16, min(len(x), budget_s / per_row_all_ops)))


def cpu_ops(oracle, xs, y, a, ps):
    out = {}
    t = {}
    for name, kname, op, *_ in OPS:
        order = 10 if kname == "gauss" else 3
        t0 = time.perf_counter()
        if op == "K":
            out[name] = oracle.applyk(xs, y, a, SIGMA, order)
        else:
            out[name] = oracle.applykdifft(xs, y, ps[None], a[None], SIGMA, order)
        t[name] = time.perf_counter() - t0
    return out, t


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_num_threads(cores)
    x, y, a, p = make_inputs(args.n, args.seed)
    rows = cpu_sample_rows(oracle, x, y, a, p, budget_s=max(2.0, 150.0 / max(1, args.steps + args.warmup)))
    rng = np.random.default_rng(args.seed + 1)
    times = []
    for s in range(args.warmup + args.steps):
        idx = rng.choice(args.n, rows, replace=False)
        t0 = time.perf_counter()
        cpu_ops(oracle, x[idx], y, a, p[idx])
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    pairs = 4.0 * rows * args.n
    ms = 1e3 * float(np.mean(times))
    value = pairs / (ms / 1e3)
    sample = "%d random target rows x %d sources per op, 4 ops per step (FP64, OpenMP)" % (rows, args.n)
    line = {
        "impl": "reference", "metric": "kernel-sum pairs/s", "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform cube)",
        "config": {"workload": "kernel-sum microbenchmark N=M=%d, d=3, gauss+laplacian3 sigma=%g, applyK+applyDiffKT"
                   % (args.n, SIGMA), "sample_rows": rows, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU algorithm = C/OpenMP FP64 restatement of py-lddmm/kernelFunctions.f90 "
                "(the f2py Fortran cannot be built here: no Fortran compiler)",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def measure_peaks(torch, lib, dev):
    """FP32 FMA and MUFU ex2 issue rates of this GPU (instr/s, all SMs)."""
    from registration_b200 import _lib
    from registration_b200.device import ptr, stream_handle
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, threads = sms * 8, 256
    out = torch.empty(blocks * threads, dtype=torch.float32, device=dev)
    res = {}
    for what, iters in ((0, 20000), (1, 4000)):
        for _ in range(2):
            _lib.call("lddmm_probe_launch", what, blocks, threads, iters, ptr(out), stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = None
        for _ in range(3):
            e0.record()
            _lib.call("lddmm_probe_launch", what, blocks, threads, iters, ptr(out), stream_handle())
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        res["ffma" if what == 0 else "ex2"] = blocks * threads * 8.0 * iters / best
    return res


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    from registration_b200 import kernelFunctions as kf
    from registration_b200.device import workspace

    n = args.n
    x, y, a, p = make_inputs(n, args.seed + 7919 * rank)
    xd, yd, ad, pd = (torch.from_numpy(v).to(dev) for v in (x, y, a, p))
    kernels = {"gauss": kf.Kernel(name="gauss", sigma=SIGMA), "laplacian": kf.Kernel(name="laplacian", sigma=SIGMA,
                                                                                     order=3)}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    def run_op(op, K, xs, ys, as_, ps):
        if op[2] == "K":
            return K.applyK(ys, as_, firstVar=xs)
        return K.applyDiffKT(ys, [ps], [as_], firstVar=xs)

    outs = {}

    def step(record=None):
        for op in OPS:
            K = kernels[op[1]]
            if record is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
            outs[op[0]] = run_op(op, K, xd, yd, ad, pd)
            if record is not None:
                e1.record()
                record.setdefault(op[0], []).append((e0, e1))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_id_for(local))
    clocks.start()
    time.sleep(0.3)
    rec = {}
    step_events = []
    for _ in range(args.steps):
        flush.zero_()   # L2 flush between timed iterations (outside the step's events)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        step(rec)
        s1.record()
        step_events.append((s0, s1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = [s0.elapsed_time(s1) for s0, s1 in step_events]
    op_ms = {k: float(np.mean([e0.elapsed_time(e1) for e0, e1 in v])) for k, v in rec.items()}
    total_s = sum(step_ms) / 1e3
    if world > 1:
        t = torch.tensor([total_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_s = float(t.item())
    pairs_step = 4.0 * n * n
    value = world * pairs_step * args.steps / total_s
    ms_per_step = 1e3 * total_s / args.steps

    # ---- end to end through the public API with host arrays -----------------
    pin = {}
    for k, v in (("x", x), ("y", y), ("a", a), ("p", p)):
        t = torch.empty(v.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = v
        pin[k] = t.numpy()
    h2d = d2h = 0
    for op in OPS:
        h2d += 3 * n * 3 * 8 if op[2] == "K" else 4 * n * 3 * 8
        d2h += n * 3 * 8
    e2e_steps = max(1, min(args.steps, 3))
    for op in OPS:   # warm
        run_op(op, kernels[op[1]], pin["x"], pin["y"], pin["a"], pin["p"])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for op in OPS:
            r = run_op(op, kernels[op[1]], pin["x"], pin["y"], pin["a"], pin["p"])
            assert isinstance(r, np.ndarray)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * pairs_step * e2e_steps / e2e_s

    line = None
    if rank == 0:
        # ---- measured issue-rate peaks and the roofline of the dominant kernel
        from registration_b200 import _lib
        peaks = measure_peaks(torch, _lib, dev)
        dom = max(op_ms, key=op_ms.get)
        opd = [o for o in OPS if o[0] == dom][0]
        pairs_s = n * n / (op_ms[dom] / 1e3)
        peak_pairs = min(peaks["ffma"] / opd[4], peaks["ex2"] / opd[5])
        bound = "fp32-fma" if peaks["ffma"] / opd[4] <= peaks["ex2"] / opd[5] else "xu-ex2"
        per_op = {}
        for o in OPS:
            ps_ = n * n / (op_ms[o[0]] / 1e3)
            pk = min(peaks["ffma"] / o[4], peaks["ex2"] / o[5])
            per_op[o[0]] = {"ms": op_ms[o[0]], "pairs_per_s": ps_, "frac_of_measured_peak": ps_ / pk,
                            "tflops": ps_ * o[3] / 1e12}
        roof = {"bound": bound, "achieved": pairs_s / 1e9, "peak": peak_pairs / 1e9, "unit": "Gpair/s",
                "frac": pairs_s / peak_pairs, "traffic": None, "kernel": "sweep_kernel<%s>" % dom,
                "fma_instr_per_pair": opd[4], "xu_per_pair": opd[5], "flops_per_pair": opd[3],
                "achieved_tflops": pairs_s * opd[3] / 1e12,
                "peak_source": "measured in this run: FP32 FFMA %.3g instr/s, MUFU ex2 %.3g instr/s (probe kernels)"
                               % (peaks["ffma"], peaks["ex2"]),
                "duration_ms": op_ms[dom]}

        # ---- FP64 GPU comparator on a target subset
        fp64 = None
        if not args.no_fp64:
            sub = min(n, 1 << 16)
            k64 = {"gauss": kf.Kernel(name="gauss", sigma=SIGMA, precision="fp64"),
                   "laplacian": kf.Kernel(name="laplacian", sigma=SIGMA, order=3, precision="fp64")}
            xs_d, ps_d = xd[:sub].contiguous(), pd[:sub].contiguous()
            for op in OPS:
                run_op(op, k64[op[1]], xs_d, yd, ad, ps_d)
            torch.cuda.synchronize()
            f64_ms = {}
            f64_out = {}
            for op in OPS:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                f64_out[op[0]] = run_op(op, k64[op[1]], xs_d, yd, ad, ps_d)
                e1.record()
                e1.synchronize()
                f64_ms[op[0]] = e0.elapsed_time(e1)
            fp64 = {"pairs_per_s": 4.0 * sub * n / (sum(f64_ms.values()) / 1e3),
                    "sample": "%d targets x %d sources per op" % (sub, n),
                    "speedup_fp32c_over_fp64": (4.0 * n * n / (sum(op_ms.values()) / 1e3)) /
                                               (4.0 * sub * n / (sum(f64_ms.values()) / 1e3))}

        # ---- CPU baseline leg (FP64 oracle on a row sample) + accuracy check
        cpu = None
        acc = None
        if not args.no_cpu_baseline:
            import oracle
            oracle.build()
            cores = os.cpu_count() or 1
            oracle.set_num_threads(cores)
            rows = cpu_sample_rows(oracle, x, y, a, p, args.cpu_seconds)
            rng = np.random.default_rng(args.seed + 3)
            idx = np.sort(rng.choice(min(n, 1 << 16), min(rows, 1 << 16), replace=False))
            ref_out, ref_t = cpu_ops(oracle, x[idx], y, a, p[idx])
            cpu_pairs_s = 4.0 * len(idx) * n / sum(ref_t.values())
            cpu = {"value": cpu_pairs_s, "unit": "pairs/s", "cores": cores, "kind": "port",
                   "sample": "%d target rows x %d sources, 4 ops (FP64 C/OpenMP restatement of "
                             "kernelFunctions.f90)" % (len(idx), n)}
            acc = {}
            for o in OPS:
                ours = outs[o[0]][idx.tolist()].cpu().numpy() if hasattr(outs[o[0]], "cpu") else outs[o[0]][idx]
                ref = ref_out[o[0]]
                acc[o[0]] = {
                    "fp32c_rel_l2_global": float(np.linalg.norm(ours - ref) / np.linalg.norm(ref)),
                    "fp32c_rel_l2_row_max": float((np.linalg.norm(ours - ref, axis=1) /
                                                   np.maximum(np.linalg.norm(ref, axis=1), 1e-300)).max()),
                }
                if fp64 is not None:
                    o64 = f64_out[o[0]][idx.tolist()].cpu().numpy()
                    acc[o[0]]["fp64_rel_l2_global"] = float(np.linalg.norm(o64 - ref) / np.linalg.norm(ref))

        launches = args.steps * sum(LAUNCHES_PER_OP[o[2]] for o in OPS)
        line = {
            "metric": "kernel-sum pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (compensated), f64 out",
            "data": "synthetic: seeded uniform [0,1]^3 points, N(0,1) momenta",
            "config": {"workload": "kernel-sum microbenchmark N=M=%d, d=3, gauss + laplacian(order 3) sigma=%g, "
                                   "applyK + applyDiffKT per step" % (n, SIGMA),
                       "pairs_per_step_per_gpu": pairs_step, "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": "independent instance per GPU" if world > 1 else "single GPU"},
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "api": "registration_b200.kernelFunctions.Kernel.applyK/applyDiffKT on "
                                               "pinned numpy arrays"},
            "gpu_launches": launches, "clocks": clk, "per_op": per_op, "accuracy_vs_fp64_oracle": acc,
            "fp64_gpu_path": fp64,
        }
        print(json.dumps(line), flush=True)
    workspace.clear()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
