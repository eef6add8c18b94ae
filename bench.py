"""Benchmark of the batched C2C tensor-core FFT on B200.

Default workload (the configuration the headline metric is quoted on):
1D forward C2C FFT, N = 2^20, batch 64, FP16 interleaved complex input
(re/im uniform in [-1, 1), seed 1), plain FP16 form with per-stage 1/16
scaling.  The split hi+lo form (same FP16 input, FP32 output) is measured
on the same data and reported under "split".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2]
    python bench.py --impl reference ...   # CPU FFT on the host cores

One step = one exec of the plan over the whole batch.  Inputs (256 MiB FP16)
are larger than L2 (126 MB), so no flush is needed between steps.  With
N > 1 (torchrun) every rank runs its own replica of the batch (transforms are
independent: weak scaling, no collective on the data path); value is the
sum over ranks, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import threading
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (dims, batch, seed, description)
    "c1": ((4096,), 256, 0, "1D N=4096 batch 256"),
    "c2": ((1 << 20,), 64, 1, "1D N=2^20 batch 64"),
    "c3": ((1024, 1024), 16, 2, "2D 1024x1024 batch 16"),
    "c4": ((256, 256, 256), 1, 3, "3D 256^3 batch 1"),
}


def flops_5nlogn(dims, batch):
    n = int(np.prod(dims))
    return 5.0 * n * np.log2(n) * batch


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled from a thread every ~0.2 ms (the timed regions last
    milliseconds), nvidia-smi at 100 ms as a fallback.  Reads only."""

    HW_SLOWDOWN, SW_POWER_CAP, SW_THERMAL, HW_THERMAL = 0x8, 0x4, 0x20, 0x40

    def __init__(self, local_rank: int):
        self.local_rank = local_rank
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.thread = None
        self.proc = None
        self.stop_flag = False

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.local_rank)
        try:
            bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.local_rank)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            reasons_fn = (getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None)
                          or nv.nvmlDeviceGetCurrentClocksThrottleReasons)

            def poll():
                while not self.stop_flag:
                    try:
                        self.samples.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        r = reasons_fn(h)
                    except Exception:
                        break
                    for bit, nm in ((self.HW_SLOWDOWN, "hw_slowdown"),
                                    (self.HW_THERMAL, "hw_thermal_slowdown"),
                                    (self.SW_THERMAL, "sw_thermal_slowdown"),
                                    (self.SW_POWER_CAP, "sw_power_cap")):
                        if r & bit:
                            self.reasons.add(nm)
                    time.sleep(0.0002)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            while not self.samples and self.thread.is_alive():
                time.sleep(0.0005)  # first sample before the timed region
            return
        except Exception:
            self.thread = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.local_rank), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag = True
            self.thread.join(timeout=5)
        elif self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                return None
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in out.strip().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.samples.append(float(f[1]))
                    self.max_mhz = float(f[2])
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        self.reasons.add(nm)
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


def make_input(dims, batch, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float16)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float16)
    return np.stack([re, im], -1).reshape(-1)  # interleaved FP16


def time_steps(fn, steps, warmup, torch, stream, barrier):
    for _ in range(warmup):
        fn()
    barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(steps):
        starts[i].record(stream)
        fn()
        ends[i].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    total = t0.elapsed_time(t1)
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    return total / steps, per


def uneven_shapes(seed=4):
    """The uneven-batch workload: 4096 1D transforms with N = 2^e, e uniform
    in 8..16, and 64 2D transforms with Nx, Ny uniform in {128, 256, 512}
    (numpy PCG64, seed 4), ordered by shape so that equal shapes lie
    contiguously (the plan batches them)."""
    rng = np.random.default_rng(seed)
    e = rng.integers(8, 17, 4096)
    sides = np.array([128, 256, 512])
    nx = sides[rng.integers(0, 3, 64)]
    ny = sides[rng.integers(0, 3, 64)]
    shapes = [(1 << int(k),) for k in e] + [(int(a), int(b)) for a, b in zip(nx, ny)]
    return sorted(shapes, key=lambda s: (len(s), s))


def bench_uneven(args, torch, mc, stream, barrier, peak, gmax=lambda v: v):
    """Both forms on the uneven batch: one plan over 4160 descriptors (one
    per transform); returns its timings (the maximum over ranks, `gmax`)
    next to the summed ideal HBM time (one read of the input plus one write
    of the output at `peak`)."""
    shapes = uneven_shapes()
    descs, off = [], 0
    for s in shapes:
        n = int(np.prod(s))
        descs.append((s, 1, off, off))
        off += n
    total = off
    flops = sum(5.0 * np.prod(s) * np.log2(np.prod(s)) for s in shapes)
    rng = np.random.default_rng(4)
    host = rng.uniform(-1, 1, 2 * total).astype(np.float16)
    x = torch.from_numpy(host.view(np.uint16)).to("cuda").view(torch.complex32)
    out = {"workload": "4096 1D transforms N=2^8..2^16 + 64 2D transforms with 128..512 sides "
                       "(seed 4), forward", "transforms": len(shapes), "points": total}
    sptr = stream.cuda_stream
    for name, prec, flags, obytes in (("plain", mc.PREC_FP16, mc.FLAG_NONE, 4),
                                      ("split", mc.PREC_SPLIT, mc.FLAG_INPUT_F16, 8)):
        y = torch.empty(total * obytes // 4, dtype=torch.complex32, device="cuda")
        with mc.Plan(descs=descs, precision=prec, flags=flags) as p:
            info = p.info()
            ms, _ = time_steps(lambda: p.exec_ptr(x.data_ptr(), y.data_ptr(), mc.FORWARD, sptr),
                               args.steps, args.warmup, torch, stream, barrier)
            p.check_status()
        ms = gmax(ms)
        ideal_ms = total * (4 + obytes) / (peak * 1e9) * 1e3
        out[name] = {"ms_per_exec": round(ms, 4), "gflops": round(flops / (ms * 1e-3) / 1e9, 1),
                     "ideal_hbm_ms": round(ideal_ms, 4), "vs_ideal": round(ms / ideal_ms, 3),
                     "launches_per_exec": info.launches, "passes": info.num_passes}
        del y
    return out


def max_over_ranks(values, dist, device):
    """Each value's maximum over all ranks (a timing of the whole job is
    its slowest rank's); identity without a process group."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def job_rate(work_per_rank, world, ms):
    """Whole-job throughput of N replicas: all ranks' work over the slowest
    rank's time (work units per second)."""
    return world * work_per_rank / (ms * 1e-3)


def run_ours(args, rank, world, local_rank):
    import torch

    import mcfft_b200 as mc

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod

    def barrier():
        if dist is not None:
            dist.barrier()

    dims, batch, seed, desc = CONFIGS[args.config]
    n = int(np.prod(dims))
    elems = n * batch
    host = make_input(dims, batch, seed)
    x = torch.from_numpy(host.view(np.uint16).copy()).to(dev).view(torch.complex32)
    y = torch.empty(elems, dtype=torch.complex32, device=dev)
    ys = torch.empty(elems, dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    plan = mc.Plan(dims, batch, mc.PREC_FP16)
    splan = mc.Plan(dims, batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16)
    info = plan.info()
    sinfo = splan.info()

    def step_plain():
        plan.exec_ptr(x.data_ptr(), y.data_ptr(), mc.FORWARD, sptr)

    def step_split():
        splan.exec_ptr(x.data_ptr(), ys.data_ptr(), mc.FORWARD, sptr)

    sampler = ClockSampler(local_rank)
    sampler.start()
    ms, per = time_steps(step_plain, args.steps, args.warmup, torch, stream, barrier)
    clocks = sampler.stop()
    plan.check_status()
    ms_split, per_split = time_steps(step_split, args.steps, args.warmup, torch, stream, barrier)
    splan.check_status()

    # End to end through the C ABI with page-locked host buffers
    # (mcfftExecHost): every step copies the whole input in and the whole
    # output out, pipelined over chunks of whole transforms.
    h_in = torch.from_numpy(host.view(np.uint16).copy()).pin_memory()
    h_out = torch.empty(elems * 2, dtype=torch.float16).pin_memory()

    def step_e2e():
        plan.exec_host_ptr(h_in.data_ptr(), h_out.data_ptr(), mc.FORWARD, sptr)

    ms_e2e, _ = time_steps(step_e2e, max(3, args.steps // 4), max(3, args.warmup), torch, stream,
                           barrier)
    plan.check_status()

    def gmax(v):
        return max_over_ranks([v], dist, dev)[0]

    ms = gmax(ms)
    ms_split = gmax(ms_split)
    ms_e2e = gmax(ms_e2e)
    fl = flops_5nlogn(dims, batch)
    value = job_rate(fl, world, ms) / 1e9
    value_split = job_rate(fl, world, ms_split) / 1e9
    value_e2e = job_rate(fl, world, ms_e2e) / 1e9

    peak, peak_kind = read_peaks()
    bytes_alg = info.in_bytes + info.out_bytes
    bytes_alg_split = sinfo.in_bytes + sinfo.out_bytes
    kern_ms = statistics.mean(per)
    achieved = bytes_alg / (kern_ms * 1e-3) / 1e9
    achieved_split = bytes_alg_split / (statistics.mean(per_split) * 1e-3) / 1e9
    traffic = traffic_split = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath)).get(args.config, {})
            traffic, traffic_split = tj.get("plain"), tj.get("split")
        except Exception:
            traffic = traffic_split = None

    result = None
    if rank == 0:
        result = {
            "metric": "FFT GFLOP/s (5N log2N) + HBM% roofline, split-prec vs FP16 at stated L2 err",
            "value": round(value, 2),
            "unit": "GFLOP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f16 (fp32 accumulate)",
            "data": "synthetic: re/im uniform [-1,1) from numpy PCG64 seed %d, rounded to FP16" % seed,
            "config": {"workload": f"{desc}, forward C2C, plain FP16 form", "dims": list(dims),
                       "batch": batch, "parallelism": f"replicas x{world}",
                       "l2": "inputs (%d MiB) larger than L2; no flush" % (elems * 4 >> 20),
                       "passes": info.num_passes},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_exec": bytes_alg,
                         "note": "exec = %d pass launches; achieved = (input + output bytes) / "
                                 "mean CUDA-event exec time" % info.num_passes},
            "split": {"value": round(value_split, 2), "unit": "GFLOP/s",
                      "ms_per_step": round(ms_split, 5),
                      "ratio_vs_plain": round(value_split / value, 4),
                      "roofline_frac": round(achieved_split / peak, 4),
                      "algorithmic_bytes_per_exec": bytes_alg_split,
                      "traffic": traffic_split,
                      "form": "FP16 input split hi+lo, FP32 output"},
            "e2e": {"value": round(value_e2e, 2), "unit": "GFLOP/s",
                    "h2d_bytes_per_step": int(elems * 4), "d2h_bytes_per_step": int(elems * 4),
                    "ms_per_step": round(ms_e2e, 4)},
            "gpu_launches": info.num_passes * args.steps,
            "clocks": clocks,
        }
    if args.config == "c2" and not args.no_uneven:
        ub = bench_uneven(args, torch, mc, stream, barrier, peak, gmax)
        if result is not None:
            result["uneven_batch"] = ub
    plan.close()
    splan.close()
    return result, host, dims, batch


def cpu_fft_rate(dims, batch, seed, budget_s=15.0):
    """Time the oracle's FP64 FFT (OpenMP, all host threads) on a bounded
    sample of the workload.  Returns (GFLOP/s, threads, sample text)."""
    from oracle import oracle
    n = int(np.prod(dims))
    per_tx = max(1, min(batch, int(2 ** 22 // n) or 1))
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-1, 1, (per_tx, n)) + 1j * rng.uniform(-1, 1, (per_tx, n)))
    oracle.fftnd(x[:1], list(dims))  # warm (builds the library)
    t0 = time.perf_counter()
    reps = 0
    while True:
        oracle.fftnd(x, list(dims))
        reps += 1
        if time.perf_counter() - t0 > budget_s or reps >= 200:
            break
    dt = time.perf_counter() - t0
    threads = os.cpu_count() or 1
    fl = flops_5nlogn(dims, per_tx) * reps
    return fl / dt / 1e9, threads, f"{reps} x {per_tx} transform(s) of {list(dims)} in {dt:.1f} s"


def accuracy_sample(host, dims, batch):
    """rel-L2 of both forms on the first transform of the workload vs the
    FP64 oracle (part of the CPU-baseline leg: the oracle is the checker)."""
    import torch

    import mcfft_b200 as mc
    from oracle import oracle
    n = int(np.prod(dims))
    one = host[: 2 * n]
    x = torch.from_numpy(one.view(np.uint16).copy()).cuda().view(torch.complex32)
    xd = one.astype(np.float64)
    ref = oracle.fftnd((xd[0::2] + 1j * xd[1::2]).reshape((1,) + tuple(dims)), list(dims)).reshape(-1)
    out = {}
    for name, prec, flags in (("plain", mc.PREC_FP16, 0), ("split", mc.PREC_SPLIT, mc.FLAG_INPUT_F16)):
        with mc.Plan(dims, 1, prec, flags) as p:
            if prec == mc.PREC_FP16:
                y = torch.empty(n, dtype=torch.complex32, device="cuda")
            else:
                y = torch.empty(n, dtype=torch.complex64, device="cuda")
            p.exec_ptr(x.data_ptr(), y.data_ptr(), mc.FORWARD, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            if prec == mc.PREC_FP16:
                h = y.view(torch.uint16).cpu().numpy().view(np.float16).astype(np.float64)
                yc = (h[0::2] + 1j * h[1::2]) * 2.0 ** (-p.info().scale_log2)
            else:
                yc = y.cpu().numpy().astype(np.complex128)
        rel, mx = oracle.error_norms(yc, ref)
        out[name] = {"rel_l2": float("%.3e" % rel), "max_rel": float("%.3e" % mx)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch leg")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dims, batch, seed, desc = CONFIGS[args.config]

    if args.impl == "reference":
        # The reference's own implementation is HIP/rocWMMA and cannot be
        # built here; its CPU-side equivalent is the FP64 FFT oracle, timed on
        # the host cores over a bounded sample of the same workload.
        if rank != 0:
            return 0
        per_step_s = max(1.0, 20.0 / max(1, args.steps + args.warmup))
        rate, threads, sample = cpu_fft_rate(dims, batch, seed, budget_s=per_step_s * args.steps)
        fl = flops_5nlogn(dims, batch)
        line = {
            "metric": "FFT GFLOP/s (5N log2N) + HBM% roofline, split-prec vs FP16 at stated L2 err",
            "value": round(rate, 3), "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(fl / (rate * 1e9) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic, same shapes as the GPU arm",
            "config": {"workload": f"{desc}, forward C2C", "dims": list(dims), "batch": batch},
            "impl": "reference",
            "cpu_baseline": {"value": round(rate, 3), "unit": "GFLOP/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(rate, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    result, host, dims, batch = run_ours(args, rank, world, local_rank)
    if rank == 0:
        if not args.no_cpu and world == 1:  # the CPU baseline is timed at N = 1 only
            rate, threads, sample = cpu_fft_rate(dims, batch, seed)
            result["cpu_baseline"] = {"value": round(rate, 3), "unit": "GFLOP/s", "cores": threads,
                                      "kind": "port", "sample": "FP64 oracle FFT: " + sample}
            result["error"] = accuracy_sample(host, dims, batch)
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
