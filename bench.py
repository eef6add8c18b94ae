"""Benchmark of the batched C2C tensor-core FFT on B200.

Default workload (the configuration the headline metric is quoted on):
1D forward C2C FFT, N = 2^20, batch 64, FP16 interleaved complex input
(re/im uniform in [-1, 1), seed 1), plain FP16 form with per-stage 1/16
scaling.  The split hi+lo form (same FP16 input, FP32 output) is measured
on the same data and reported under "split", the uneven batch under
"uneven_batch".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2]
    python bench.py --impl reference ...   # CPU FFT on the host cores

Configurations (tests/workloads.py): c1 1D 4096 x 256; c2 1D 2^20 x 64; c3
2D 1024^2 x 16 (split form with FP32 input; errors also for the
wide-range input); c4 3D 256^3 (split form with FP32 input, forward and
inverse); c5 the uneven batch alone.

One step = one exec of the plan over the whole batch.  Inputs of c2 (256 MiB
FP16) are larger than L2 (126 MB), so no flush is needed between its steps.
With N > 1 every rank runs its own replica of the batch (transforms are
independent: weak scaling, no collective on the data path); value is the
sum over ranks, time is the max over ranks.  Without torchrun, --gpus N > 1
relaunches this script under torch.distributed.run with N ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import threading
import socket
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tests import workloads as W  # noqa: E402

METRIC = "FFT GFLOP/s (5N log2N) + HBM% roofline, split-prec vs FP16 at stated L2 err"
CONFIGS = dict(W.CONFIGS)
CONFIGS["c5"] = (None, None, 4, "uneven batch: 4096 1D (N=2^8..2^16) + 64 2D (128..512 sides)")
# split form input type per configuration: FP16 where it is compared with the
# plain form on the same input (c1, c2, c5), FP32 as c3 / c4 state it
SPLIT_IN_F16 = {"c1": True, "c2": True, "c3": False, "c4": False, "c5": True}

flops_5nlogn = W.flops_5nlogn


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


def interleaved(x: np.ndarray, f16: bool) -> np.ndarray:
    """complex128 -> interleaved FP16 (as uint16) or FP32 complex, flat."""
    flat = np.ascontiguousarray(x.reshape(-1))
    if f16:
        ri = np.stack([flat.real, flat.imag], -1).astype(np.float16)
        return ri.reshape(-1).view(np.uint16)
    return flat.astype(np.complex64)


def storage_rounded(x: np.ndarray, f16: bool) -> np.ndarray:
    if f16:
        return (x.real.astype(np.float16).astype(np.float64)
                + 1j * x.imag.astype(np.float16).astype(np.float64))
    return x.astype(np.complex64).astype(np.complex128)


def config_input(name):
    """(complex128 input, dims, batch) of a configuration (c1..c4)."""
    dims, batch, seed, _ = CONFIGS[name]
    if name == "c4":
        return W.plane_waves(seed=seed), dims, batch
    return W.uniform((batch,) + tuple(dims), seed), dims, batch


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


def device_errors(mc, torch, y, out_f16, ref, seg_off, scales):
    """Per-segment errors of device result y against the complex128 host
    reference, reduced in FP64 on the GPU (mcfftErrorNorms)."""
    rd = torch.from_numpy(np.ascontiguousarray(ref.reshape(-1)).view(np.float64)).cuda()
    res = mc.error_norms(y.data_ptr(), out_f16, rd.data_ptr(), seg_off, scales,
                         torch.cuda.current_stream().cuda_stream)
    del rd
    return {"rel_l2": float("%.3e" % max(r["rel_l2"] for r in res)),
            "max_rel": float("%.3e" % max(r["max_rel"] for r in res)),
            "get_error": float("%.3e" % max(r["get_error"] for r in res)),
            "transforms": len(res)}


def bench_uneven(args, torch, mc, stream, barrier, peak, gmax=lambda v: v, errors=False):
    """Both forms on the uneven batch: one plan over 4160 descriptors (one
    per transform, laid out in `args.uneven_order`); returns its timings (the
    maximum over ranks, `gmax`) next to the summed ideal HBM time (one read
    of the input plus one write of the output at `peak`), and with `errors`
    the worst per-transform error of each form against the FP64 oracle."""
    shapes, offs, total = W.uneven_layout(args.uneven_order)
    descs = [(s, 1, o, o) for s, o in zip(shapes, offs)]
    flops = sum(flops_5nlogn(s) for s in shapes)
    xc = W.uneven_input(total)
    x = torch.from_numpy(interleaved(xc, True).copy()).to("cuda").view(torch.complex32)
    out = {"workload": "4096 1D transforms N=2^8..2^16 + 64 2D transforms with 128..512 sides "
                       "(seed 4), forward, descriptors in %s order" % args.uneven_order,
           "transforms": len(shapes), "points": total}
    ref = None
    if errors:
        from oracle import oracle
        xr = storage_rounded(xc, True)
        ref = np.empty_like(xr)
        by_shape = {}
        for i, s in enumerate(shapes):
            by_shape.setdefault(s, []).append(i)
        for s, idx in by_shape.items():
            n = int(np.prod(s))
            stack = np.stack([xr[offs[i]:offs[i] + n] for i in idx]).reshape((len(idx),) + s)
            o = oracle.fftnd(stack, list(s)).reshape(len(idx), n)
            for j, i in enumerate(idx):
                ref[offs[i]:offs[i] + n] = o[j]
    sptr = stream.cuda_stream
    for name, prec, flags, obytes in (("plain", mc.PREC_FP16, mc.FLAG_NONE, 4),
                                      ("split", mc.PREC_SPLIT, mc.FLAG_INPUT_F16, 8)):
        y = torch.empty(total, dtype=torch.complex32 if obytes == 4 else torch.complex64,
                        device="cuda")
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
        if ref is not None:
            # undo the plain form's output scale 2^-log2(N) of each transform
            scales = [int(np.log2(np.prod(s))) if obytes == 4 else 0 for s in shapes]
            out[name]["error"] = device_errors(mc, torch, y, obytes == 4, ref, offs + [total],
                                               scales)
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

    def gmax(v):
        return max_over_ranks([v], dist, dev)[0]

    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    peak, peak_kind = read_peaks()
    accuracy = rank == 0 and world == 1 and not args.no_cpu

    if args.config == "c5":
        sampler = ClockSampler(local_rank)
        sampler.start()
        ub = bench_uneven(args, torch, mc, stream, barrier, peak, gmax, errors=accuracy)
        clocks = sampler.stop()
        if rank != 0:
            return None, None
        pl = ub["plain"]
        flops = sum(flops_5nlogn(s) for s in W.uneven_layout(args.uneven_order)[0])
        achieved = ub["points"] * 8 / (pl["ms_per_exec"] * 1e-3) / 1e9
        result = {
            "metric": METRIC, "value": round(job_rate(flops, world, pl["ms_per_exec"]) / 1e9, 2),
            "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": pl["ms_per_exec"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 (fp32 accumulate)",
            "data": "synthetic: re/im uniform [-1,1) from numpy PCG64 seed 4, rounded to FP16",
            "config": {"workload": ub["workload"], "parallelism": f"replicas x{world}",
                       "l2": "inputs (%d MiB) larger than L2; no flush" % (ub["points"] * 4 >> 20)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_kind": peak_kind},
            "uneven_batch": ub, "gpu_launches": pl["launches_per_exec"] * args.steps,
            "clocks": clocks,
        }
        return result, None

    xc, dims, batch = config_input(args.config)
    n = int(np.prod(dims))
    elems = n * batch
    s16 = SPLIT_IN_F16[args.config]
    host16 = interleaved(xc, True)
    x = torch.from_numpy(host16.copy()).to(dev).view(torch.complex32)
    xs = x if s16 else torch.from_numpy(interleaved(xc, False)).to(dev)
    y = torch.empty(elems, dtype=torch.complex32, device=dev)
    ys = torch.empty(elems, dtype=torch.complex64, device=dev)

    plan = mc.Plan(dims, batch, mc.PREC_FP16)
    splan = mc.Plan(dims, batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16 if s16 else mc.FLAG_NONE)
    info = plan.info()
    sinfo = splan.info()

    def step_plain():
        plan.exec_ptr(x.data_ptr(), y.data_ptr(), mc.FORWARD, sptr)

    def step_split():
        splan.exec_ptr(xs.data_ptr(), ys.data_ptr(), mc.FORWARD, sptr)

    sampler = ClockSampler(local_rank)
    sampler.start()
    ms, per = time_steps(step_plain, args.steps, args.warmup, torch, stream, barrier)
    clocks = sampler.stop()
    plan.check_status()
    ms_split, per_split = time_steps(step_split, args.steps, args.warmup, torch, stream, barrier)
    splan.check_status()
    ms_inv = None
    if args.config == "c4":
        # the inverse of the split form's forward output, back to the input
        zs = torch.empty_like(ys)
        ms_inv, _ = time_steps(lambda: splan.exec_ptr(ys.data_ptr(), zs.data_ptr(), mc.INVERSE, sptr),
                               args.steps, args.warmup, torch, stream, barrier)
        splan.check_status()

    # End to end through the C ABI with page-locked host buffers
    # (mcfftExecHost): every step copies the whole input in and the whole
    # output out, pipelined over chunks of whole transforms.
    h_in = torch.from_numpy(host16.copy()).pin_memory()
    h_out = torch.empty(elems * 2, dtype=torch.float16).pin_memory()

    def step_e2e():
        plan.exec_host_ptr(h_in.data_ptr(), h_out.data_ptr(), mc.FORWARD, sptr)

    ms_e2e, _ = time_steps(step_e2e, max(3, args.steps // 4), max(3, args.warmup), torch, stream,
                           barrier)
    plan.check_status()
    del h_in, h_out

    ms = gmax(ms)
    ms_split = gmax(ms_split)
    ms_e2e = gmax(ms_e2e)
    if ms_inv is not None:
        ms_inv = gmax(ms_inv)
    fl = flops_5nlogn(dims, batch)
    value = job_rate(fl, world, ms) / 1e9
    value_split = job_rate(fl, world, ms_split) / 1e9
    value_e2e = job_rate(fl, world, ms_e2e) / 1e9

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
        split_form = ("FP16 input split hi+lo, FP32 output" if s16 else
                      "FP32 input split hi+lo, FP32 output")
        result = {
            "metric": METRIC,
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
            "data": "synthetic: %s, numpy PCG64 seed %d, rounded to FP16 (split: %s)" % (
                "8 plane waves + Gaussian noise" if args.config == "c4" else "re/im uniform [-1,1)",
                CONFIGS[args.config][2], "FP16" if s16 else "FP32"),
            "config": {"workload": f"{CONFIGS[args.config][3]}, forward C2C, plain FP16 form",
                       "dims": list(dims), "batch": batch, "parallelism": f"replicas x{world}",
                       "l2": ("inputs (%d MiB) larger than L2; no flush" % (elems * 4 >> 20)
                              if elems * 4 > 126e6 else
                              "inputs (%d MiB) fit in L2; not flushed (L2-warm)" % (elems * 4 >> 20)),
                       "passes": info.num_passes},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_exec": bytes_alg,
                         "note": "exec = %d launch(es); achieved = (input + output bytes) / "
                                 "mean CUDA-event exec time" % info.launches},
            "split": {"value": round(value_split, 2), "unit": "GFLOP/s",
                      "ms_per_step": round(ms_split, 5),
                      "ratio_vs_plain": round(value_split / value, 4),
                      "roofline_frac": round(achieved_split / peak, 4),
                      "algorithmic_bytes_per_exec": bytes_alg_split,
                      "traffic": traffic_split,
                      "form": split_form},
            "e2e": {"value": round(value_e2e, 2), "unit": "GFLOP/s",
                    "h2d_bytes_per_step": int(elems * 4), "d2h_bytes_per_step": int(elems * 4),
                    "ms_per_step": round(ms_e2e, 4)},
            "gpu_launches": info.launches * args.steps,
            "clocks": clocks,
        }
        if ms_inv is not None:
            result["split"]["inverse_ms_per_step"] = round(ms_inv, 5)
    if args.config == "c2" and not args.no_uneven:
        ub = bench_uneven(args, torch, mc, stream, barrier, peak, gmax, errors=accuracy)
        if result is not None:
            result["uneven_batch"] = ub
    if accuracy:
        result["error"] = accuracy_all(args.config, xc, dims, batch, plan, splan, s16, x, xs,
                                       torch, mc)
    plan.close()
    splan.close()
    return result, (dims, batch)


def accuracy_all(name, xc, dims, batch, plan, splan, s16, x, xs, torch, mc):
    """rel-L2, max error and the reference harness's get_error of every
    transform of the workload, both forms, against the FP64 oracle on the
    same storage-rounded input; the norms are reduced on the GPU.  c3 adds
    the wide-range input, c4 the inverse and the round trip."""
    from oracle import oracle
    n = int(np.prod(dims))
    seg = [i * n for i in range(batch + 1)]
    sptr = torch.cuda.current_stream().cuda_stream
    out = {}

    def run(p, xin, out_dt, direction=mc.FORWARD):
        yy = torch.empty(n * batch, dtype=out_dt, device="cuda")
        p.exec_ptr(xin.data_ptr(), yy.data_ptr(), direction, sptr)
        torch.cuda.synchronize()
        p.check_status()
        return yy

    def one(xin_c, tag):
        ref16 = oracle.fftnd(storage_rounded(xin_c, True).reshape((batch,) + tuple(dims)), list(dims))
        xd16 = torch.from_numpy(interleaved(xin_c, True).copy()).cuda().view(torch.complex32)
        yp = run(plan, xd16, torch.complex32)
        out[tag + "plain"] = device_errors(mc, torch, yp, True, ref16, seg,
                                           [-plan.info().scale_log2] * batch)
        del yp
        if s16:
            ref_s, xd = ref16, xd16
        else:
            ref_s = oracle.fftnd(storage_rounded(xin_c, False).reshape((batch,) + tuple(dims)),
                                 list(dims))
            xd = torch.from_numpy(interleaved(xin_c, False)).cuda()
        del ref16
        ys_ = run(splan, xd, torch.complex64)
        out[tag + "split"] = device_errors(mc, torch, ys_, False, ref_s, seg, None)
        return ys_

    ys_ = one(xc, "")
    if name == "c3":
        one(W.wide_range((batch,) + tuple(dims), CONFIGS["c3"][2]), "wide_")
    if name == "c4":
        z = run(splan, ys_, torch.complex64, mc.INVERSE)
        yh = ys_.cpu().numpy().astype(np.complex128).reshape((batch,) + tuple(dims))
        out["split_inverse"] = device_errors(mc, torch, z, False,
                                             oracle.fftnd(yh, list(dims), sign=+1), seg, None)
        out["split_roundtrip"] = device_errors(mc, torch, z, False,
                                               storage_rounded(xc, False) * n, seg, None)
    return out


def workload_groups(name, order="sorted"):
    """The workload as (shape, transform count) groups."""
    if name == "c5":
        groups = {}
        for s in W.uneven_layout(order)[0]:
            groups[s] = groups.get(s, 0) + 1
        return list(groups.items())
    dims, batch, _, _ = CONFIGS[name]
    return [(tuple(dims), batch)]


def _sample(work, frac, dt, seed=0):
    rng = np.random.default_rng(seed)
    data = []
    for s, c in work:
        cnt = max(1, int(round(c * frac)))
        data.append((s, (rng.uniform(-1, 1, (cnt,) + s)
                         + 1j * rng.uniform(-1, 1, (cnt,) + s)).astype(dt)))
    return data, sum(flops_5nlogn(s, a.shape[0]) for s, a in data)


def _fft_all(sfft, data, threads):
    for s, a in data:
        sfft.fftn(a, axes=tuple(range(1, 1 + len(s))), workers=threads)


def cpu_fft_rate(work, budget_s=15.0, threads=None):
    """The CPU FFT baseline: scipy.fft (pocketfft) in single and double
    precision on all host threads, timed on a bounded sample of the
    workload (the same fraction of every transform group, at most 2^23
    points).  Returns (GFLOP/s of the faster precision, threads, sample
    text, its numpy dtype)."""
    import scipy.fft as sfft
    threads = threads or os.cpu_count() or 1
    points = sum(int(np.prod(s)) * c for s, c in work)
    frac = min(1.0, float(2 ** 23) / points)
    rates = {}
    for dt in (np.complex64, np.complex128):
        data, fl = _sample(work, frac, dt)
        _fft_all(sfft, data, threads)  # warm
        t0 = time.perf_counter()
        reps = 0
        while True:
            _fft_all(sfft, data, threads)
            reps += 1
            if time.perf_counter() - t0 > budget_s / 2 or reps >= 500:
                break
        dt_s = time.perf_counter() - t0
        rates[dt] = (fl * reps / dt_s / 1e9, reps, dt_s)
    best = max(rates, key=lambda k: rates[k][0])
    other = np.complex128 if best is np.complex64 else np.complex64
    r, reps, dt_s = rates[best]
    sample = ("scipy.fft (pocketfft) %s, %d workers: %d rep(s) of %.3g%% of the workload's "
              "transforms in %.1f s (%s: %.2f GFLOP/s)" % (
                  np.dtype(best).name, threads, reps, 100 * frac, dt_s, np.dtype(other).name,
                  rates[other][0]))
    return r, threads, sample, best


def reference_arm(args, rank):
    """`--impl reference`: the reference has no CPU FFT of its own (its
    accuracy harness calls FFTW double on the host, benchmark/accuracy_1d.cpp:
    12-24) and its GPU code is HIP for AMD GPUs; the FFTW stand-in here is
    scipy.fft (pocketfft, the faster of single and double precision) on all
    host threads.  Each step is one whole pass over the workload (every
    transform) when that keeps the run within about two minutes, else the
    same fraction of every transform group; timed on the host clock.  Rank 0
    alone runs."""
    if rank != 0:
        return 0
    import scipy.fft as sfft
    threads = os.cpu_count() or 1
    work = workload_groups(args.config, args.uneven_order)
    desc = CONFIGS[args.config][3]
    fl = sum(flops_5nlogn(s, c) for s, c in work)
    rate, _, _, dt = cpu_fft_rate(work, budget_s=2.0, threads=threads)
    est_step = fl / (rate * 1e9)
    frac = min(1.0, 120.0 / max(1e-9, est_step * (args.steps + args.warmup)))
    data, fl_step = _sample(work, frac, dt)
    for _ in range(args.warmup):
        _fft_all(sfft, data, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _fft_all(sfft, data, threads)
    ms_per_step = (time.perf_counter() - t0) / args.steps * 1e3
    value = fl_step / (ms_per_step * 1e-3) / 1e9
    sample = ("scipy.fft (pocketfft) %s, %d workers; each step %s" % (
        np.dtype(dt).name, threads,
        "the whole workload" if frac >= 1.0 else "%.1f%% of every transform group" % (100 * frac)))
    cfg = {"workload": f"{desc}, forward C2C"}
    if args.config != "c5":
        cfg.update(dims=list(CONFIGS[args.config][0]), batch=CONFIGS[args.config][1])
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64" if dt is np.complex64 else "c128",
        "data": "synthetic, same shapes as the GPU arm", "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "GFLOP/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def relaunch_cmd(argv, nproc, port):
    """torch.distributed.run command that runs this script on `nproc` ranks
    of this node (rendezvous on 127.0.0.1)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={nproc}", "--master-addr", "127.0.0.1", "--master-port", str(port),
            os.path.join(ROOT, "bench.py"), *argv]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    # the uneven batch's descriptors as drawn (the plan groups them by shape
    # whatever their order); "sorted" hands them over already grouped
    ap.add_argument("--uneven-order", default="draw", choices=["draw", "sorted", "shuffled"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and error legs")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch leg")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    if args.gpus < 1:
        print("--gpus must be at least 1", file=sys.stderr)
        return 2

    launched = "WORLD_SIZE" in os.environ
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank)

    if launched and world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU",
              file=sys.stderr)
        return 2
    if not launched and args.gpus > 1:
        # one process per GPU: run this script under torch.distributed.run
        return subprocess.call(relaunch_cmd(argv, args.gpus, _free_port()))

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    result, _ = run_ours(args, rank, world, local_rank)
    if rank == 0:
        if not args.no_cpu and world == 1:
            # the CPU baseline is timed at N = 1 only
            rate, threads, sample, _ = cpu_fft_rate(workload_groups(args.config, args.uneven_order))
            result["cpu_baseline"] = {"value": round(rate, 3), "unit": "GFLOP/s",
                                      "cores": threads, "kind": "port", "sample": sample}
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
