"""Benchmark of the B200 Poisson solve: 512^3 FP64 solve points/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--grid NX NY NZ] [--precision fp64|fp32]

One step = one solve (the five passes) of one 512^3 FP64 grid whose f is the
reference's analytic right-hand side.  As in the reference harness
(FishFry.hpp:173-187) the field is re-initialised before every solve outside
the timed region (the solve destroys its density argument); each solve is
timed with CUDA events on the solve's stream, and `value` is points/s over the
K timed solves.  Inputs are 1.07 GB per field, larger than the 126 MB L2, so
no L2 flush is needed between steps.

Under torchrun (N > 1) every rank solves its own grid (replicas, weak
scaling: the single-grid solve has no exchange step on one GPU); the time is
the max over ranks.

--impl reference times the reference algorithm on the host cores: the
reference has no CPU code path, so this is the oracle's OpenMP restatement
(oracle/), on all host threads; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, nargs=3, default=[512, 512, 512])
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def bytes_model(n, precision, launches=3):
    """Algorithmic HBM bytes per launch (each field read and written once):
    R = real field, H = half spectrum (ni*nj*(nk/2+1) complex).  Five
    launches (one per pass): 2R + 8H; three launches (z/y fused through L2):
    R+H, 2H, H+R = 2R + 4H.  Also returns the five-pass total, the model the
    solve-level roofline is quoted against."""
    esz = 8 if precision == "fp64" else 4
    N = n[0] * n[1] * n[2]
    R = N * esz
    H = n[0] * n[1] * (n[2] // 2 + 1) * 2 * esz
    five = [R + H, 2 * H, 2 * H, 2 * H, H + R]
    per_launch = five if launches == 5 else [R + H, 2 * H, H + R]
    return per_launch, sum(per_launch), sum(five)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if r[3 + q].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model


def oracle_baseline(n, threads=None, steps=1, warmup=1):
    """Times the oracle's OpenMP FP64 solve of grid n on the host cores."""
    import numpy as np
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    cores = O.get_threads()
    f = O.init_f(n)
    for _ in range(warmup):
        O.solve(f)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        O.solve(f)
        times.append(time.perf_counter() - t)
    del np
    return times, cores


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.grid
    N = n[0] * n[1] * n[2]
    times, cores = oracle_baseline(n, steps=args.steps, warmup=args.warmup)
    total = sum(times)
    value = N * args.steps / total
    line = {
        "impl": "reference", "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid",
        "config": {"workload": "%dx%dx%d FP64 Poisson solve" % tuple(n), "grid": list(n), "precision": "fp64",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": "%d full %dx%dx%d solves on %s" % (args.steps, *n, cpu_info() or "host")},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU code path; this is the oracle's OpenMP restatement of its algorithm",
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    import fishfry_b200 as ff

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = tuple(args.grid)
    N = n[0] * n[1] * n[2]
    prec = ff.FF_FP64 if args.precision == "fp64" else ff.FF_FP32
    dt = torch.float64 if prec == ff.FF_FP64 else torch.float32
    esz = 8 if prec == ff.FF_FP64 else 4
    plan = ff.Plan(n, precision=prec)
    count = plan.nbytes // esz
    stream = torch.cuda.Stream(device=dev)
    d = torch.empty(count, dtype=dt, device=dev)
    p = torch.empty(count, dtype=dt, device=dev)
    f0 = torch.empty(N, dtype=dt, device=dev)
    ff.init_field(n, f0, None, prec)
    torch.cuda.synchronize()

    def step(times_out=None):
        with torch.cuda.stream(stream):
            d[:N].copy_(f0)                   # untimed: restore the destroyed input
        ms, tot = plan.solve(d, p, stream=stream, timed=True)
        if times_out is not None:
            times_out.append((ms, tot))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    rec = []
    for _ in range(args.steps):
        step(rec)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(t for _, t in rec)
    nph = plan.phases()
    pass_ms = [sum(r[0][q] for r in rec) / len(rec) for q in range(nph)]
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * N * args.steps / (total_ms * 1e-3)

    # correctness of the last solve (outside timing)
    norms = ff.rel_norms(n, p, None, prec)

    # end to end through the public API with host buffers: pinned f -> device,
    # solve, phi -> pinned host, every step
    e2e = None
    if not args.no_e2e:
        hf = torch.empty(N, dtype=dt, pin_memory=True)
        hp = torch.empty(N, dtype=dt, pin_memory=True)
        hf.copy_(f0.cpu())
        for _ in range(2):
            with torch.cuda.stream(stream):
                d[:N].copy_(hf, non_blocking=True)
            plan.solve(d, p, stream=stream)
            with torch.cuda.stream(stream):
                hp.copy_(p[:N], non_blocking=True)
        stream.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                d[:N].copy_(hf, non_blocking=True)
            plan.solve(d, p, stream=stream)
            with torch.cuda.stream(stream):
                hp.copy_(p[:N], non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_ms = float(te.item())
        e2e = {"value": world * N * args.steps / (e2e_ms * 1e-3), "unit": "points/s",
               "h2d_bytes_per_step": N * esz, "d2h_bytes_per_step": N * esz,
               "ms_per_step": e2e_ms / args.steps}

    if rank == 0:
        per_pass_bytes, total_bytes, five_pass_bytes = bytes_model(n, args.precision, nph)
        names = ff.phase_names(plan)
        top = max(range(len(pass_ms)), key=lambda q: pass_ms[q])
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        peak = peaks.get("hbm_gbs")
        peak_src = "measured" if peak else "fallback"
        peak = peak or 6650.0
        achieved = per_pass_bytes[top] / (pass_ms[top] * 1e-3) / 1e9
        traffic = None
        try:
            tr = json.load(open(PROFILE_TRAFFIC))
            key = "%dx%dx%d_%s" % (*n, args.precision)
            traffic = tr.get(key, {}).get(names[top])
        except (OSError, ValueError):
            pass
        solve_gbs = total_bytes / (ms_per_step * 1e-3) / 1e9
        five_gbs = five_pass_bytes / (ms_per_step * 1e-3) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            times, cores = oracle_baseline(n, steps=1, warmup=0)
            cpu = {"value": N / times[0], "unit": "points/s", "cores": cores, "kind": "port",
                   "sample": "one full %dx%dx%d FP64 solve of the oracle (OpenMP) on %s" % (*n, cpu_info() or "host")}
        line = {
            "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == ff.FF_FP64 else "f32",
            "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid (x = -pi + i*2*pi/n)",
            "config": {"workload": "%dx%dx%d %s Poisson solve, 5 passes" % (*n, args.precision.upper()),
                       "grid": list(n), "precision": args.precision,
                       "parallelism": "replicas x%d" % world if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (%.2f GB per field > 126 MB)" % (N * esz / 1e9)},
            "roofline": {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes": per_pass_bytes[top]},
            "solve_roofline": {"achieved": solve_gbs, "frac": solve_gbs / peak, "algorithmic_bytes": total_bytes,
                               "launches": nph,
                               "five_pass_model": {"bytes": five_pass_bytes, "equivalent_gbs": five_gbs,
                                                   "frac_of_8TBs": five_gbs / 8000.0}},
            "passes_ms": dict(zip(names, pass_ms)),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": nph * args.steps,
            "clocks": clk,
            "check": {"rel_l1_l2_linf_vs_analytic": norms},
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
