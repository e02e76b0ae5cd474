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

The default line also carries the other two parts of the headline metric,
each measured in the same run with its own clock record and error figures
(skipped with --no-extras, and under torchrun):
  batch      256 seeded grids, dims iid {32..128}: FP32 and FP64 batched
             solves/s against a loop of plain FP64 solves of the same grids,
             max relative L2 against those plain FP64 solves;
  serve      Poisson request streams (dims 5-smooth in [32, 512], log-uniform
             points): p50/p99 at 1000 requests/s with FP32:FP64 1:1, solves/s
             at saturation for the 1:1 mix and for FP32 alone, against plain
             FP64 and FP32 loops over the same requests; FP32 error against
             the plain FP64 solve;
  precision  1024^3 FP32 (FP64 twiddles and 1/k^2) with 64 seeded modes:
             points/s and relative L2/Linf against the FP64 solve of the same f.

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
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum, bytes per
# launch) of each pass, from one `ncu --set full` capture of each kernel; the
# captures' summaries and commands are profiles/passes_fp64_512cube_ncu_full.txt,
# profiles/passes_fp32_512cube_ncu_full.txt and
# profiles/passes_fp64_1024x512x256_ncu_full.txt.
MEASURED_TRAFFIC = {
    ("512x512x512", "fp64"): {
        "Real-to-complex FFT in Z": 2.10596e9, "Forward FFT in Y": 2.10300e9, "X FFTs and filter": 2.12535e9,
        "Backward FFT in Y": 2.10666e9, "Complex-to-real FFT in Z": 2.10525e9,
    },
    ("512x512x512", "fp32"): {
        "Real-to-complex FFT in Z": 1.03033e9, "Forward FFT in Y": 1.02935e9, "X FFTs and filter": 1.02789e9,
        "Backward FFT in Y": 1.04324e9, "Complex-to-real FFT in Z": 1.03176e9,
    },
    ("1024x512x256", "fp64"): {
        "Real-to-complex FFT in Z": 2.10856e9, "Forward FFT in Y": 2.11018e9, "X FFTs and filter": 2.25988e9,
        "Backward FFT in Y": 2.11315e9, "Complex-to-real FFT in Z": 2.11120e9,
    },
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, nargs=3, default=[512, 512, 512])
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["solve", "precision", "batch", "serve"], default="solve",
                    help="solve: one grid (default); precision: 1024^3 FP32 with random modes; "
                         "batch: 256 seeded grids; serve: Poisson request stream")
    ap.add_argument("--requests", type=int, default=10000, help="serve: requests per arrival rate")
    ap.add_argument("--rates", type=float, nargs="+", default=[100, 200, 500, 1000, 2000, 5000],
                    help="serve: arrival rates (requests/s)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM admission budget")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--no-tune", action="store_true", help="batch: default tile shapes, no autotuning")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the batch, serve and precision keys")
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
    """SM clocks and clock-event (throttle) reasons sampled every few ms by
    NVML while the timed region runs; nvidia-smi at 200 ms when the NVML
    bindings are missing."""

    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_s=0.005):
        self.device = device
        self.period = period_s
        self.rows = []          # (sm_mhz, max_mhz, reason bitmask)
        self.stop_flag = threading.Event()
        self.thread = None
        self.proc = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        prop = torch.cuda.get_device_properties(self.device)
        try:
            bus = "%08x:%02x:%02x.0" % (prop.pci_domain_id, prop.pci_bus_id, prop.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            return self._start_smi()
        self.source = "nvml"

        def loop():
            while not self.stop_flag.is_set():
                try:
                    self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx, int(reasons(h))))
                except Exception:
                    pass
                time.sleep(self.period)
        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def _start_smi(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.source = "nvidia-smi"

        def read():
            for line in self.proc.stdout:
                r = [x.strip() for x in line.split(",")]
                if len(r) == 7 and r[0].replace(".", "").isdigit():
                    bits = sum(b for q, (_, b) in enumerate(self.REASON_BITS) if r[3 + q].lower().startswith("active"))
                    self.rows.append((float(r[0]), float(r[1]), bits))
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def stop(self):
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.thread.join(timeout=5)
        rows = list(self.rows)
        reasons = sorted({name for _, _, bits in rows for name, b in self.REASON_BITS if bits & b})
        return {"sm_mhz": statistics.median(r[0] for r in rows) if rows else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None, "reasons": reasons,
                "samples": len(rows), "source": self.source}


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


def reference_sample_grid(n, steps, budget_s=150.0):
    """The largest cube sample (of the workload's kind, at most n) whose
    steps + warm-up finish within budget_s on the host cores, from a timed
    128^3 solve scaled by N log N."""
    import math
    from oracle import oracle as O
    f = O.init_f((128, 128, 128))
    t = time.perf_counter()
    O.solve(f)
    t128 = time.perf_counter() - t
    N = n[0] * n[1] * n[2]
    for m in (512, 384, 256, 192, 128, 96, 64):
        M = m ** 3
        if M > N:
            continue
        est = t128 * (M / 128 ** 3) * (math.log(M) / math.log(128 ** 3))
        if est * steps <= budget_s:
            return (m, m, m) if M < N else tuple(n)
    return (64, 64, 64)


def scipy_yardstick(n, threads):
    """A library yardstick on the host cores: the same spectral solve with
    scipy.fft (pocketfft) rfftn/irfftn on all threads, one timed solve of the
    FP64 analytic f (seconds, points/s)."""
    import numpy as np
    import scipy.fft as sf
    from oracle import oracle as O
    f = O.init_f(tuple(n))
    kx = [np.minimum(np.arange(m), m - np.arange(m)).astype(np.float64) for m in n[:2]]
    kz = np.arange(n[2] // 2 + 1, dtype=np.float64)
    k2 = kx[0][:, None, None] ** 2 + kx[1][None, :, None] ** 2 + kz[None, None, :] ** 2
    k2[0, 0, 0] = np.inf
    t = time.perf_counter()
    s = sf.rfftn(f, workers=threads)
    s *= -1.0 / k2
    phi = sf.irfftn(s, s=f.shape, workers=threads)
    dt = time.perf_counter() - t
    del phi
    return dt, f.size / dt


def solve_config(n, precision, world):
    """The `config` of the solve workload, identical in both arms."""
    esz = 8 if precision == "fp64" else 4
    N = n[0] * n[1] * n[2]
    return {"workload": "%dx%dx%d %s Poisson solve" % (*n, precision.upper()), "grid": list(n),
            "precision": precision, "parallelism": "replicas x%d" % world if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (%.2f GB per field > 126 MB)" % (N * esz / 1e9)}


def reference_binary_on_gpu(n=(256, 256, 256), runs=10):
    """The reference itself on this GPU: its own ParisPencil.cpp + main.cpp with
    cuFFT (oracle/_ref/fishfry_ref, built from the reference's sources with a
    one-rank MPI stub), and this build's driver with the same arguments; both
    print the reference harness's per-run Time (host wall time of a solve,
    FishFry.hpp:198).  256^3 is the largest cube the reference launches on one
    GPU.  Returns None where the reference binary was not built."""
    import re
    ref = os.path.join(ROOT, "oracle", "_ref", "fishfry_ref")
    ours = os.path.join(ROOT, "fishfry_b200", "bin", "fishfry")
    if not (os.path.exists(ref) and os.path.exists(ours)):
        return None
    args = ["1", "1", "1"] + [str(x) for x in n] + [str(runs)]
    out = {}
    for name, exe in (("reference", ref), ("fishfry_b200", ours)):
        r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=300)
        if r.returncode != 0:
            return {"error": "%s exited %d: %s" % (name, r.returncode, r.stderr[-200:])}
        times = [float(m.group(2)) for m in re.finditer(r"^(\d+): Time (\S+)", r.stdout, re.M) if m.group(1) != "0"]
        l2 = re.search(r"L_2 (\S+)", r.stdout)
        out[name] = {"ms_per_solve": 1e3 * statistics.median(times), "runs": len(times),
                     "rel_l2_vs_analytic": float(l2.group(1)) if l2 else None}
    out["grid"] = list(n)
    out["speedup"] = out["reference"]["ms_per_solve"] / out["fishfry_b200"]["ms_per_solve"]
    out["what"] = ("median per-run Time of the reference harness's printout (host wall time of one solve), "
                   "the reference with cuFFT vs this build, same arguments, same GPU")
    return out


def run_reference(args):
    """The reference's algorithm on the host cores: each step one oracle
    solve (ParisPencil's FFT solve restated in C++/OpenMP) of a sample grid
    sized so that the whole run stays within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sample = reference_sample_grid(args.grid, args.steps + args.warmup)
    N = sample[0] * sample[1] * sample[2]
    times, cores = oracle_baseline(sample, steps=args.steps, warmup=args.warmup)
    total = sum(times)
    value = N * args.steps / total
    line = {
        "impl": "reference", "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid",
        "config": solve_config(tuple(args.grid), "fp64", args.gpus),
        "sample_grid": list(sample),
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": "%d solves of a %dx%dx%d sample grid on %s" % (args.steps, *sample,
                                                                                cpu_info() or "host")},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU code path; this is the oracle's OpenMP restatement of its algorithm",
    }
    print(json.dumps(line), flush=True)


def job_time_ms(local_ms, world, device):
    """The job's time: the max over ranks of each rank's timed region (every
    rank receives it).  One rank per GPU; on the CPU (gloo) for tests."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(points_per_rank, steps, job_ms, world):
    """Whole-job points/s of N replicas (weak scaling: every rank solves its
    own grid of points_per_rank points per step)."""
    return world * points_per_rank * steps / (job_ms * 1e-3)


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
    total_ms = job_time_ms(total_ms, world, dev)
    ms_per_step = total_ms / args.steps
    value = replicas_value(N, args.steps, total_ms, world)

    # correctness of the last solve (outside timing)
    norms = ff.rel_norms(n, p, None, prec)

    # end to end through the public API with host buffers: every step copies
    # its f from pinned host memory to the device, solves, and copies phi back
    # to pinned host memory.  Steps are pipelined over two buffer sets: the
    # input copy of step s+1 and the output copy of step s-1 run on their own
    # streams while step s solves (PCIe is full duplex).
    e2e = None
    if not args.no_e2e:
        hf = torch.empty(N, dtype=dt, pin_memory=True)
        hp = [torch.empty(N, dtype=dt, pin_memory=True) for _ in range(2)]
        hf.copy_(f0.cpu())
        ref = p[:N].clone()                        # phi of the device-timed solves
        dd = [d, torch.empty_like(d)]
        pp = [p, torch.empty_like(p)]
        s_in = torch.cuda.Stream(device=dev)
        s_out = torch.cuda.Stream(device=dev)

        def pipeline(nsteps):
            loaded = [torch.cuda.Event() for _ in range(nsteps)]
            solved = [torch.cuda.Event() for _ in range(nsteps)]
            drained = [torch.cuda.Event() for _ in range(nsteps)]
            for q in range(nsteps):
                b = q % 2
                with torch.cuda.stream(s_in):
                    if q >= 2:
                        s_in.wait_event(solved[q - 2])     # buffer set b free again
                    dd[b][:N].copy_(hf, non_blocking=True)
                    loaded[q].record(s_in)
                stream.wait_event(loaded[q])
                if q >= 2:
                    stream.wait_event(drained[q - 2])      # phi of step q-2 read out
                plan.solve(dd[b], pp[b], stream=stream)
                solved[q].record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(solved[q])
                    hp[b].copy_(pp[b][:N], non_blocking=True)
                    drained[q].record(s_out)
            return drained[nsteps - 1]

        pipeline(2).synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        last = pipeline(args.steps)
        s_out.wait_event(last)
        e1.record(s_out)
        e1.synchronize()
        e2e_ms = job_time_ms(e0.elapsed_time(e1), world, dev)
        same = bool(torch.equal(hp[(args.steps - 1) % 2].to(dev), ref))
        e2e = {"value": replicas_value(N, args.steps, e2e_ms, world), "unit": "points/s",
               "h2d_bytes_per_step": N * esz, "d2h_bytes_per_step": N * esz,
               "ms_per_step": e2e_ms / args.steps, "pipelined": "two buffer sets, copies on their own streams",
               "result_matches_device_timed_solve": same}

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
        traffic = MEASURED_TRAFFIC.get(("%dx%dx%d" % n, args.precision), {}).get(names[top])
        solve_gbs = total_bytes / (ms_per_step * 1e-3) / 1e9
        five_gbs = five_pass_bytes / (ms_per_step * 1e-3) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            times, cores = oracle_baseline(n, steps=1, warmup=0)
            cpu = {"value": N / times[0], "unit": "points/s", "cores": cores, "kind": "port",
                   "sample": "one full %dx%dx%d FP64 solve of the oracle (OpenMP) on %s" % (*n, cpu_info() or "host")}
            try:
                sec, pps = scipy_yardstick(n, cores)
                cpu["scipy_fft_yardstick"] = {"value": pps, "unit": "points/s", "seconds": sec, "workers": cores,
                                              "what": "scipy.fft rfftn, -1/k^2, irfftn (pocketfft), one solve"}
            except Exception as e:   # a missing scipy does not cost the line
                cpu["scipy_fft_yardstick"] = {"unavailable": str(e)[:120]}
            try:
                rg = reference_binary_on_gpu()
                if rg is not None:
                    cpu["reference_binary_on_gpu"] = rg
            except Exception as e:
                cpu["reference_binary_on_gpu"] = {"error": str(e)[:200]}
        line = {
            "metric": "512^3 FP64 solve points/s", "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == ff.FF_FP64 else "f32",
            "data": "synthetic: analytic f of FishFry.hpp:22-44 on the reference grid (x = -pi + i*2*pi/n)",
            "config": solve_config(n, args.precision, world),
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
    plan.close()
    del d, p, f0
    if e2e is not None:
        del dd, pp, hf, hp, ref
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_extras:
        # the other parts of the headline metric, each with its own clocks
        for key, fn in (("batch", extra_batch), ("serve", extra_serve), ("precision", extra_precision)):
            t = time.perf_counter()
            try:
                line[key] = fn(args)
            except Exception as e:   # an extra that fails does not cost the headline line
                line[key] = {"error": "%s: %s" % (type(e).__name__, str(e)[:300])}
            line[key]["wall_s"] = time.perf_counter() - t
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def modes_for(ff, n, seed, count=64, kmax=32, sigma=0.1):
    """The seeded random-mode term: count modes, integer 0 < |k| <= kmax,
    alias-free on grid n, amplitudes N(0, sigma), phases U[0, 2 pi)."""
    return ff.modes_generate(seed, count, kmax, ff.alias_free_kaxis(n), sigma)


def rel_l2_dev(torch, a, b):
    a = a.double()
    b = b.double()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def precision_measure(n, steps, warmup, seed):
    """FP64 and FP32 solves of grid n, f = analytic + 64 seeded modes: ms per
    solve (CUDA events), and the FP32 error against the FP64 solve of the
    same f and against the analytic potential, all computed on the device."""
    import torch

    import fishfry_b200 as ff
    N = n[0] * n[1] * n[2]
    modes = modes_for(ff, n, seed)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    res = {}
    clocks = ClockSampler(0)
    for prec in (ff.FF_FP64, ff.FF_FP32):
        dt = torch.float64 if prec == ff.FF_FP64 else torch.float32
        plan = ff.Plan(n, precision=prec)
        esz = 8 if prec == ff.FF_FP64 else 4
        d = torch.empty(plan.nbytes // esz, dtype=dt, device=dev)
        p = torch.empty_like(d)
        f0 = torch.empty(N, dtype=dt, device=dev)
        ff.init_field(n, f0, modes, prec)
        times = []
        for it in range(max(warmup, 3) + steps):
            if it == max(warmup, 3) and prec == ff.FF_FP32:
                clocks.start()
            with torch.cuda.stream(stream):
                d[:N].copy_(f0)
            ms, tot = plan.solve(d, p, stream=stream, timed=True)
            if it >= max(warmup, 3):
                times.append(tot)
        res[prec] = {"ms": sum(times) / len(times), "phi": p[:N].clone(),
                     "norms": ff.rel_norms(n, p, modes, prec)}
        plan.close()
        del d, p, f0
        torch.cuda.empty_cache()
    clk = clocks.stop()
    p64, p32 = res[ff.FF_FP64]["phi"], res[ff.FF_FP32]["phi"]
    diff = (p32.double() - p64)
    out = {"grid": list(n), "fp32_ms_per_solve": res[ff.FF_FP32]["ms"], "fp64_ms_per_solve": res[ff.FF_FP64]["ms"],
           "fp32_points_per_s": N / (res[ff.FF_FP32]["ms"] * 1e-3),
           "fp64_points_per_s": N / (res[ff.FF_FP64]["ms"] * 1e-3),
           "fp32_vs_fp64_solve": {"rel_l2": rel_l2_dev(torch, p32, p64),
                                  "rel_linf": float(diff.abs().max() / p64.abs().max())},
           "fp32_vs_analytic_rel_l1_l2_linf": res[ff.FF_FP32]["norms"],
           "fp64_vs_analytic_rel_l1_l2_linf": res[ff.FF_FP64]["norms"],
           "data": "analytic f (FishFry.hpp:22-44) + 64 seeded modes, |k| <= 32, a ~ N(0, 0.1), seed %d" % seed,
           "steps": steps, "clocks": clk}
    del res, p64, p32, diff
    torch.cuda.empty_cache()
    return out


def extra_precision(args):
    return precision_measure((1024, 1024, 1024), min(args.steps, 5), 3, args.seed)


def run_precision(args):
    """1024^3 FP32 solve of analytic f + 64 seeded modes; error against the
    FP64 solve of the same input and against the analytic potential."""
    n = tuple(args.grid) if args.grid != [512, 512, 512] else (1024, 1024, 1024)
    r = precision_measure(n, args.steps, args.warmup, args.seed)
    line = {
        "metric": "1024^3 FP32 solve points/s (precision form)", "value": r["fp32_points_per_s"],
        "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["fp32_ms_per_solve"], "higher_is_better": True, "dtype": "f32",
        "data": "synthetic: " + r["data"],
        "config": {"workload": "%dx%dx%d FP32 (FP64 twiddles and 1/k^2)" % n, "modes_seed": args.seed},
    }
    line.update({k: v for k, v in r.items() if k not in ("data",)})
    print(json.dumps(line), flush=True)


def batch_dims(seed=2024, count=256, choices=(32, 48, 64, 80, 96, 128)):
    import numpy as np
    rng = np.random.default_rng(seed)
    return [tuple(int(x) for x in rng.choice(choices, 3)) for _ in range(count)]


def batch_measure(steps, warmup, seed, tune=True):
    """256 grids with dims iid from {32, 48, 64, 80, 96, 128}: batched solves
    (five persistent launches, graph replay, tuned tiles) in FP64 and FP32
    against a loop of single-grid FP64 solves of the same grids; errors
    against those plain FP64 solves, computed on the device."""
    import torch

    import fishfry_b200 as ff
    dims = batch_dims()
    pts = sum(a * b * c for a, b, c in dims)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    K, W = steps, max(warmup, 3)
    out = {}
    pristine = {}
    clocks = ClockSampler(0)
    for prec in (ff.FF_FP64, ff.FF_FP32):
        dt = torch.float64 if prec == ff.FF_FP64 else torch.float32
        esz = 8 if prec == ff.FF_FP64 else 4
        b = ff.Batch(dims, precision=prec)
        d = [torch.empty(nb // esz, dtype=dt, device=dev) for nb in b.nbytes]
        p = [torch.empty(nb // esz, dtype=dt, device=dev) for nb in b.nbytes]
        t_tune = time.perf_counter()
        if tune:
            b.tune(d, p, stream=stream, reps=3)
        t_tune = time.perf_counter() - t_tune
        f0 = []
        for g, n in enumerate(dims):
            x = torch.empty(n[0] * n[1] * n[2], dtype=dt, device=dev)
            ff.init_field(n, x, modes_for(ff, n, seed + g), prec)
            f0.append(x)
        pristine[prec] = f0

        def restore():
            with torch.cuda.stream(stream):
                for g in range(len(dims)):
                    d[g][:f0[g].numel()].copy_(f0[g])

        tot = []
        for it in range(W + K):
            if it == W and prec == ff.FF_FP32:
                clocks.start()
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.solve(d, p, stream=stream)
            e1.record(stream)
            e1.synchronize()
            if it >= W:
                tot.append(e0.elapsed_time(e1))
        b.check(stream)
        ms = sorted(tot)[len(tot) // 2]
        out[prec] = {"ms": ms, "solves_per_s": len(dims) / (ms * 1e-3), "points_per_s": pts / (ms * 1e-3),
                     "tune_s": t_tune, "phi": [x[:f.numel()].clone() for x, f in zip(p, f0)]}
        b.close()
        del d, p
        torch.cuda.empty_cache()
    clk = clocks.stop()
    # loop of single-grid FP64 solves (the plain method, one plan per grid)
    plans = [ff.Plan(n) for n in dims]
    ds = [torch.empty(pl.nbytes // 8, dtype=torch.float64, device=dev) for pl in plans]
    ps = [torch.empty_like(x) for x in ds]
    tot = []
    for it in range(W + K):
        with torch.cuda.stream(stream):
            for g in range(len(dims)):
                ds[g][:pristine[ff.FF_FP64][g].numel()].copy_(pristine[ff.FF_FP64][g])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for pl, x, y in zip(plans, ds, ps):
            pl.solve(x, y, stream=stream)
        e1.record(stream)
        e1.synchronize()
        if it >= W:
            tot.append(e0.elapsed_time(e1))
    loop_ms = sorted(tot)[len(tot) // 2]
    # accuracy: FP32 batch vs the plain FP64 solve; FP64 batch vs plain FP64
    err32 = max(rel_l2_dev(torch, a, y[:a.numel()]) for a, y in zip(out[ff.FF_FP32]["phi"], ps))
    err64 = max(rel_l2_dev(torch, a, y[:a.numel()]) for a, y in zip(out[ff.FF_FP64]["phi"], ps))
    for pl in plans:
        pl.close()
    del ds, ps, pristine
    loop = {"ms": loop_ms, "solves_per_s": len(dims) / (loop_ms * 1e-3)}
    res = {
        "grids": len(dims), "points_per_batch": pts, "steps": K, "tiles": "tuned" if tune else "default",
        "fp32_batch": {k: v for k, v in out[ff.FF_FP32].items() if k != "phi"},
        "fp64_batch": {k: v for k, v in out[ff.FF_FP64].items() if k != "phi"},
        "fp64_loop_of_plain_solves": loop,
        "fp32_batch_vs_fp64_loop": out[ff.FF_FP32]["solves_per_s"] / loop["solves_per_s"],
        "fp64_batch_vs_fp64_loop": out[ff.FF_FP64]["solves_per_s"] / loop["solves_per_s"],
        "max_rel_l2_vs_plain_fp64": {"fp32_batch": err32, "fp64_batch": err64},
        "data": "analytic f + 64 seeded modes per grid (dims seed 2024, modes seed %d + grid index)" % seed,
        "clocks": clk,
    }
    del out
    torch.cuda.empty_cache()
    return res


def extra_batch(args):
    return batch_measure(min(args.steps, 10), 3, args.seed, tune=not args.no_tune)


def run_batch(args):
    r = batch_measure(args.steps, args.warmup, args.seed, tune=not args.no_tune)
    line = {
        "metric": "FP32 batched solves/s (256 grids, dims iid {32..128})",
        "value": r["fp32_batch"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["fp32_batch"]["ms"], "higher_is_better": True, "dtype": "f32",
        "data": "synthetic: " + r["data"], "config": {
            "workload": "256 grids, dims seed 2024, five persistent launches per solve (CUDA graph), %s tiles" %
                        r["tiles"], "points_per_batch": r["points_per_batch"]},
    }
    line.update({k: v for k, v in r.items() if k not in ("data",)})
    print(json.dumps(line), flush=True)


def _smooth235(n):
    for q in (2, 3, 5):
        while n % q == 0:
            n //= q
    return n == 1


SMOOTH = [n for n in range(32, 513) if _smooth235(n)]


def serve_dims(rng):
    """A 5-smooth triple in [32, 512]^3 whose point count is log-uniform in
    [32^3, 512^3]: the nearest product among 16 seeded (a, b) draws."""
    import math
    target = math.exp(rng.uniform(math.log(32 ** 3), math.log(512 ** 3)))
    best = None
    for _ in range(16):
        a = SMOOTH[rng.integers(len(SMOOTH))]
        b = SMOOTH[rng.integers(len(SMOOTH))]
        c = min(SMOOTH, key=lambda x: abs(math.log(a * b * x / target)))
        err = abs(math.log(a * b * c / target))
        if best is None or err < best[0]:
            best = (err, (int(a), int(b), int(c)))
    return best[1]


def serve_stream(srv, reqs, gaps, src):
    """Submits reqs = [(dims, precision)] with inter-arrival gaps (s) from a
    producer thread, takes completions in completion order, releases them at
    once, and returns the server's statistics of the stream."""
    import threading
    srv.reset_stats()
    ready = threading.Event()

    def producer():
        t = time.perf_counter()
        for q, (n, prec) in enumerate(reqs):
            t += gaps[q]
            while True:
                now = time.perf_counter()
                if now >= t:
                    break
                if t - now > 0.002:
                    time.sleep(t - now - 0.001)
            srv.submit(n, src[prec], prec)
            if q == 0:
                ready.set()

    th = threading.Thread(target=producer)
    th.start()
    ready.wait()
    for _ in range(len(reqs)):
        rid = srv.next()[0]
        srv.release(rid)
    th.join()
    srv.check()
    st = srv.stats()
    return {"requests": len(reqs), "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
            "max_ms": st["max_ms"], "solves_per_s": st["solves_per_s"], "points_per_s": st["points_per_s"],
            "completed": st["completed"], "peak_gb": st["peak_bytes"] / 1e9, "steps": st["steps"],
            "launches": st["launches"], "max_active": st["max_active"]}


def serve_sources(torch, ff, dev, seed):
    """One device source field per precision: request inputs are read from it
    (the solve's work does not depend on the values); the accuracy sample uses
    proper fields."""
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    return {ff.FF_FP64: torch.randn(512 ** 3, dtype=torch.float64, device=dev, generator=gen),
            ff.FF_FP32: torch.randn(512 ** 3, dtype=torch.float32, device=dev, generator=gen)}


def serve_warm(srv, ff, src):
    """Every axis length's tables resident in both precisions."""
    warm = []
    for L in SMOOTH:
        for prec in (ff.FF_FP64, ff.FF_FP32):
            warm.append(srv.submit((L, 32, 32), src[prec], prec))
    for rid in warm:
        srv.wait(rid)
        srv.release(rid)


def serve_plain_loops(torch, ff, dev, dims, src):
    """The plain method on the same requests: single-grid solves one after
    another (plans made beforehand; each request's field copied in first, as
    the server copies it), FP64 and FP32; solves/s of the second pass."""
    plain = {}
    for prec in (ff.FF_FP64, ff.FF_FP32):
        dt = torch.float64 if prec == ff.FF_FP64 else torch.float32
        plans = {n: ff.Plan(n, precision=prec) for n in set(dims)}
        cap = max(pl.nbytes for pl in plans.values())
        esz = 8 if prec == ff.FF_FP64 else 4
        d = torch.empty(cap // esz, dtype=dt, device=dev)
        p = torch.empty_like(d)
        st = torch.cuda.Stream(device=dev)
        for rep in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for n in dims:
                N = n[0] * n[1] * n[2]
                with torch.cuda.stream(st):
                    d[:N].copy_(src[prec][:N])
                plans[n].solve(d, p, stream=st, nbytes=cap)
            e1.record(st)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        plain["fp64" if prec == ff.FF_FP64 else "fp32"] = {"solves_per_s": len(dims) / (ms * 1e-3),
                                                           "requests": len(dims)}
        for pl in plans.values():
            pl.close()
        del d, p
        torch.cuda.empty_cache()
    return plain


def serve_accuracy(torch, ff, dev, seed, budget_gb, count=8, max_points=256 ** 3):
    """FP32 requests through the server against the plain FP64 solve of the
    same f (analytic + 64 seeded modes); the worst relative L2."""
    import numpy as np
    srv = ff.Server(int(min(budget_gb, 40) * 1e9), max_active=64)
    rng = np.random.default_rng(seed)
    worst = 0.0
    checked = 0
    for q in range(4 * count):
        if checked == count:
            break
        n = serve_dims(rng)
        N = n[0] * n[1] * n[2]
        if N > max_points:
            continue
        f64 = torch.empty(N, dtype=torch.float64, device=dev)
        ff.init_field(n, f64, modes_for(ff, n, seed + q), ff.FF_FP64)
        f32 = f64.float()
        rid = srv.submit(n, f32, ff.FF_FP32)
        srv.wait(rid)
        o32 = torch.empty(N, dtype=torch.float32, device=dev)
        srv.fetch(rid, o32)
        plan = ff.Plan(n)
        d = torch.empty(plan.nbytes // 8, dtype=torch.float64, device=dev)
        p = torch.empty_like(d)
        d[:N].copy_(f32.double())
        plan.solve(d, p)
        worst = max(worst, rel_l2_dev(torch, o32, p[:N]))
        plan.close()
        checked += 1
    srv.close()
    return worst, checked


def serve_measure(seed, budget_gb, requests, rate_low=1000.0, rate_sat=5000.0, plain_sample=400):
    """Short request streams through one server: the 1:1 FP32:FP64 mix at
    rate_low (latency) and at rate_sat (saturation, solves/s), the FP32 lane
    alone at rate_sat on the same dims, and the plain FP64 / FP32 loops over
    those dims."""
    import numpy as np
    import torch

    import fishfry_b200 as ff
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    src = serve_sources(torch, ff, dev, seed)
    srv = ff.Server(int(budget_gb * 1e9), max_active=4096)
    serve_warm(srv, ff, src)
    rng = np.random.default_rng(seed + 1000)
    low = [(serve_dims(rng), int(rng.integers(2))) for _ in range(requests)]
    gaps_low = rng.exponential(1.0 / rate_low, requests)
    sat = [(serve_dims(rng), int(rng.integers(2))) for _ in range(requests)]
    gaps_sat = rng.exponential(1.0 / rate_sat, requests)
    clocks = ClockSampler(0)
    clocks.start()
    r_low = serve_stream(srv, low, gaps_low, src)
    r_sat = serve_stream(srv, sat, gaps_sat, src)
    r_32 = serve_stream(srv, [(n, ff.FF_FP32) for n, _ in sat], gaps_sat, src)
    clk = clocks.stop()
    srv.close()
    dims = [n for n, _ in sat[:plain_sample]]
    plain = serve_plain_loops(torch, ff, dev, dims, src)
    del src
    torch.cuda.empty_cache()
    worst, checked = serve_accuracy(torch, ff, dev, seed, budget_gb)
    r_low["rate"] = rate_low
    r_sat["rate"] = rate_sat
    r_32["rate"] = rate_sat
    return {
        "mix_1to1_at_%g_per_s" % rate_low: r_low,
        "mix_1to1_at_%g_per_s" % rate_sat: r_sat,
        "fp32_only_at_%g_per_s" % rate_sat: r_32,
        "plain_loop_on_the_saturation_dims": plain,
        "p50_ms_at_%g_per_s" % rate_low: r_low["p50_ms"], "p99_ms_at_%g_per_s" % rate_low: r_low["p99_ms"],
        "served_mix_vs_plain_fp64": r_sat["solves_per_s"] / plain["fp64"]["solves_per_s"],
        "served_fp32_vs_plain_fp64": r_32["solves_per_s"] / plain["fp64"]["solves_per_s"],
        "fp32_vs_plain_fp64_rel_l2_max": worst, "accuracy_requests": checked,
        "budget_gb": budget_gb,
        "data": "request dims log-uniform in points (5-smooth, 32..512 per axis), seed %d" % seed,
        "clocks": clk,
    }


def extra_serve(args):
    return serve_measure(args.seed, args.budget_gb, requests=min(args.requests, 1500))


def run_serve(args):
    """Poisson arrival stream of mixed-size FP32/FP64 requests through the
    request loop; p50/p99 latency and solves/s per arrival rate."""
    import numpy as np
    import torch

    import fishfry_b200 as ff
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    src = serve_sources(torch, ff, dev, args.seed)
    results = []
    for rate in args.rates:
        t_rate = time.perf_counter()
        rng = np.random.default_rng(args.seed + int(rate))
        reqs = [(serve_dims(rng), int(rng.integers(2))) for _ in range(args.requests)]
        gaps = rng.exponential(1.0 / rate, args.requests)
        srv = ff.Server(int(args.budget_gb * 1e9), max_active=4096)
        serve_warm(srv, ff, src)
        r = serve_stream(srv, reqs, gaps, src)
        srv.close()
        r["rate"] = rate
        print("serve rate %g: %d requests in %.1f s, p50 %.3f ms, p99 %.3f ms, %.0f solves/s" % (
            rate, r["completed"], time.perf_counter() - t_rate, r["p50_ms"], r["p99_ms"], r["solves_per_s"]),
            file=sys.stderr, flush=True)
        results.append(r)
    rng = np.random.default_rng(args.seed + 7)
    plain = serve_plain_loops(torch, ff, dev, [serve_dims(rng) for _ in range(min(400, args.requests))], src)
    del src
    torch.cuda.empty_cache()
    worst, checked = serve_accuracy(torch, ff, dev, args.seed, args.budget_gb)
    line = {
        "metric": "served solves/s and p99 latency (Poisson arrivals, dims 32..512, FP32:FP64 1:1)",
        "value": max(r["solves_per_s"] for r in results), "unit": "solves/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32+f64",
        "data": "synthetic: request dims log-uniform in points (5-smooth, 32..512 per axis)",
        "config": {"workload": "continuous batching request loop", "requests_per_rate": args.requests,
                   "budget_gb": args.budget_gb, "seed": args.seed},
        "rates": results,
        "plain_loop_on_the_same_mix": plain,
        "served_at_saturation_vs_plain_fp64": max(r["solves_per_s"] for r in results) / plain["fp64"]["solves_per_s"],
        "fp32_vs_plain_fp64_rel_l2_max": worst, "accuracy_requests": checked,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
