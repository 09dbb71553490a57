"""Benchmark of the B200 snapshot imager (one JSON line on stdout).

Workload: the W-projection snapshot of the reference's headline
configuration -- 4096 x 4096 image, 1 arcsec cells, 1,000,000 visibilities
with uvw uniform in a uv disk and w ~ U[-2000, 2000] lambda, 20 point sources
(log-uniform 0.1-10 Jy) plus 0.05 Jy noise, Gaussian-Sinc AA kernel S=3,
32 w-planes, W-kernel support <= 16 (1 % truncation), oversampling 8.
Synthetic, seeded data (no dataset exists for it).

A step = one full imaging pass of one snapshot through the library (prepass,
W-planes and FP64 W-kernels, binning, gridding, cuFFT c2r, gcf/normalise).
value = visibilities imaged per second (Mvis/s), compensated FP32 (FP32C),
inputs resident in HBM, L2 flushed (256 MB write) before every timed step.
The FP64 plain form is timed the same way and reported beside it together
with the FP32C image's error against it.  e2e = the same metric through the
host-buffer C-ABI call (stpgpu_image_visibilities_ex with host pointers) from
pinned memory, host->device copies and the image read-back inside the timed
region.

--impl reference times the reference's algorithm on the host cores (the CPU
oracle port compiled with the reference's release flags, OpenMP threads in
place of TBB, scipy FFT with all threads) on a bounded sample of the workload.
Multi-GPU (torchrun): independent snapshots per rank (replicas; no collective
on the data path), barrier + max-over-ranks timing.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mvis/s imaged, comp-FP32 vs FP64 GPU at ≤1e-5 peak-rel err; p50/p99 snapshot ms"
WORKLOAD = ("W-projection snapshot imager: 4096^2 image, 1 arcsec cells, 1M visibilities, uv disk, "
            "w~U[-2000,2000] lambda, 32 w-planes, W-kernel support<=16 (1% truncation), GaussianSinc S=3, os=8")
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def _peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for k, nm in enumerate(names):
                    if f[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def job_rates(local_ms, units_per_rank_step, steps, device=None):
    """Whole-job throughput of replicas: every rank processed `units_per_rank_step` units per step for
    `steps` steps in local_ms[k] milliseconds (one entry per timed arm); the job's time is the MAX over
    ranks (all ranks take this collective in the same order), and the rate counts the units of all ranks.
    Returns (rates in M units/s, max times in ms)."""
    import torch

    ws = 1
    tt = torch.tensor([float(x) for x in local_ms], dtype=torch.float64, device=device)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        ws = torch.distributed.get_world_size()
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
    mx = [float(x) for x in tt.cpu()]
    return [ws * units_per_rank_step * steps / (m / 1e3) / 1e6 for m in mx], mx


def run_gpu(args):
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import CONFIG2_IMAGER, config2

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    ctx = capi.Context(local)
    snap = config2(seed=2 + rank)
    N = snap.image_size
    n = snap.vis.size
    kw = dict(CONFIG2_IMAGER)
    dev = torch.device("cuda", local)
    dv = torch.from_numpy(snap.vis).to(dev)
    dw = torch.from_numpy(snap.weights).to(dev)
    duvw = torch.from_numpy(np.ascontiguousarray(snap.uvw.T)).to(dev)  # (3, n): column-major n x 3
    out32 = torch.empty(N * N, dtype=torch.float32, device=dev)
    out64 = torch.empty(N * N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def step(prec):
        out = out64 if prec == capi.FP64 else out32
        odt = capi.F64 if prec == capi.FP64 else capi.F32
        return ctx.image_visibilities(dv, dw, duvw, N, snap.cell_size, precision=prec, out_dtype=odt,
                                      device_ptrs=True, image_out=out, **kw)[2]

    def timed(prec, steps, warmup, phases=False):
        ctx.set_timing(phases)
        for _ in range(warmup):
            step(prec)
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        times, grid_ms, launches, info = [], [], 0, None
        with torch.cuda.stream(st):
            for _ in range(steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                info = step(prec)
                e1.record(st)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                grid_ms.append(list(info.phase_ms))
                launches += info.n_launches
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        ctx.set_timing(False)
        return times, grid_ms, launches, info

    # parity of the two arms (FP32C against the FP64 plain form)
    step(capi.FP64)
    torch.cuda.synchronize(dev)
    ref64 = out64.double().clone()
    step(capi.FP32C)
    torch.cuda.synchronize(dev)
    d = out32.double() - ref64
    peak = float(ref64.abs().max())
    peak_rel = float(d.abs().max()) / peak
    rms_rel = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref64))

    t64, ph64, l64, info64 = timed(capi.FP64, args.steps, args.warmup)
    with Clocks(local) as clk:
        t32, ph32, l32, info32 = timed(capi.FP32C, args.steps, args.warmup)
    clocks = clk.summary()
    _, ph, _, _ = timed(capi.FP32C, max(3, min(args.steps, 10)), 1, phases=True)

    (value, value64), (tot32, tot64) = job_rates([sum(t32), sum(t64)], n, args.steps, device=dev)

    # ---- e2e: host buffers (pinned), H2D + image D2H inside the timed region
    pv = torch.from_numpy(snap.vis).pin_memory()
    pw = torch.from_numpy(snap.weights).pin_memory()
    puvw = torch.from_numpy(np.ascontiguousarray(snap.uvw.T).reshape(-1)).pin_memory()  # u[], v[], w[]
    pimg = torch.empty(N * N, dtype=torch.float32).pin_memory()
    from fastimaging_b200.capi import AProjPars, ImagerInfo, ImagerPars, WProjPars
    import ctypes

    ip = ImagerPars(N, 0, snap.cell_size, 1.0, kw["kernel_func"], kw["kernel_support"], 0, kw["oversampling"], 0, 1,
                    0, 0)
    wp = WProjPars(kw["num_wplanes"], kw["max_wpconv_support"], kw["undersampling_opt"], kw["kernel_trunc_perc"], 0,
                   0, 0, 0)
    ap = AProjPars(0, 0.0, 0.0, 0, 0.0)
    einfo = ImagerInfo()

    def e2e_step():
        r = ctx.L.stpgpu_image_visibilities_ex(ctx.h, ctypes.c_void_p(pv.data_ptr()), capi.C128,
                                               ctypes.c_void_p(pw.data_ptr()), ctypes.c_void_p(puvw.data_ptr()), n,
                                               ctypes.byref(ip), ctypes.byref(wp), ctypes.byref(ap), capi.FP32C,
                                               ctypes.c_void_p(pimg.data_ptr()), None, capi.F32, 0,
                                               ctypes.byref(einfo))
        if r != 0:
            raise RuntimeError(ctx.L.stpgpu_last_error(ctx.h).decode())
        return einfo.device_ms

    for _ in range(args.warmup):
        e2e_step()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        e2e_ms.append(e2e_step())  # device events around H2D .. D2H on the library stream
    (e2e_single,), _ = job_rates([sum(e2e_ms)], n, args.steps, device=dev)
    h2d = snap.vis.nbytes + snap.weights.nbytes + snap.uvw.nbytes
    d2h = N * N * 4
    assert abs(float(pimg.double().max()) - float(out32.double().max())) <= 1e-6 * peak

    # e2e of a stream of snapshots: the K steps in one stpgpu_image_batch call with host buffers, each step's
    # H2D, imaging and image D2H on one of the worker streams, so transfers overlap other steps' compute
    uvw_pinned = torch.from_numpy(np.ascontiguousarray(snap.uvw.T)).pin_memory()  # (3, n): column-major n x 3
    outs_pinned = [torch.empty(N * N, dtype=torch.float32).pin_memory() for _ in range(args.steps)]
    bkw = dict(kw, image_size=N, cell_size=snap.cell_size)
    bsnaps = [dict(bkw, vis=pv.numpy(), weights=pw.numpy(), uvw=uvw_pinned.numpy().T,
                   image=o.numpy().reshape(N, N, order="F")) for o in outs_pinned]
    for _ in range(max(2, args.warmup)):
        ctx.image_batch(bsnaps, precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=False)
    # three timed repetitions of the whole batch call; the median is reported, with the spread
    e2e_reps = []
    for _ in range(3):
        flush.zero_()
        torch.cuda.synchronize(dev)
        _, _, bi = ctx.image_batch(bsnaps, precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=False)
        e2e_reps.append(bi.device_ms)
    (e2e_value,), _ = job_rates([float(np.median(e2e_reps))], n, args.steps, device=dev)
    e2e_spread = [round(n * args.steps / (t * 1e-3) / 1e6, 2) for t in sorted(e2e_reps, reverse=True)]
    for o in outs_pinned:
        assert abs(float(o.double().max()) - float(out32.double().max())) <= 1e-6 * peak

    # ---- roofline of the dominant phase (phase timers over the timed FP32C steps)
    ph = np.array(ph)  # steps x [grid init, grid loop, FFT, normalise]
    mean_ph = ph.mean(axis=0)
    names = ["grid_init", "grid_loop", "fft_c2r", "normalise"]
    hbm, peak_kind = _peaks()
    rows = N // 2 + 1
    items = info32.n_grid_items
    # algorithmic bytes per launch of each phase
    alg = {
        # grid loop: one 28-byte item record per gridded visibility read once, the half-plane grid written
        # once (FP32 complex); the tile lists' replication is overhead, not algorithmic traffic
        "grid_loop": int(info32.n_good_vis) * 28 + rows * N * 8,
        # c2r FFT: read the half-plane grid, write the N x N image (FP32)
        "fft_c2r": rows * N * 8 + N * N * 4,
        # normalise: read image, write image (FP32)
        "normalise": N * N * 4 * 2,
        # prepass + W-planes + binning: read vis/uvw/weights, write items, lists
        "grid_init": n * (16 + 24 + 8) + n * 28 + items * 4 * 2,
    }
    # the dominant kernel: the tile gridder is the single most expensive launch of a step (the
    # grid-init phase is ~20 short kernels, none above ~45 us)
    dom = names.index("grid_loop")
    dom_name = names[dom]
    achieved = alg[dom_name] / (mean_ph[dom] / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(dom_name)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": "tile gridder, autotuned form (grid_loop phase)", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_source": peak_kind, "traffic": traffic,
                "phase_ms": {k: round(float(v), 4) for k, v in zip(names, mean_ph)},
                "algorithmic_bytes": alg[dom_name],
                # every phase against the same HBM peak (algorithmic bytes / its phase time)
                "phase_frac": {k: round(alg[k] / (float(v) / 1e3) / 1e9 / hbm, 4) for k, v in zip(names, mean_ph)
                               if v > 0}}
    # the whole snapshot: vis/uvw/weights in, the half-plane grid written and read once, the image written
    # once (FP32), against the step time
    snap_bytes = n * (16 + 24 + 8) + 2 * rows * N * 8 + N * N * 4
    t_roof_ms = snap_bytes / (hbm * 1e9) * 1e3
    roofline["snapshot"] = {"algorithmic_bytes": int(snap_bytes), "t_roof_ms": round(t_roof_ms, 4),
                            "frac": round(t_roof_ms / (tot32 / args.steps), 4)}

    p50 = float(np.percentile(t32, 50))
    p99 = float(np.percentile(t32, 99))
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mvis/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(tot32 / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (two-sum compensated), FP64 W-kernels/uvw/normalise",
        "data": "synthetic (seeded point sources + noise, config-2 shapes)",
        "config": {"workload": WORKLOAD, "n_vis": n, "image_size": N, "precision": "fp32c",
                   "l2": "flushed (256 MB write) before each timed step", "inputs": "resident in HBM",
                   "parallelism": f"replicas x{ws}"},
        "fp64": {"value": round(value64, 2), "ms_per_step": round(tot64 / args.steps, 4)},
        "fp32c_over_fp64": round(value / value64, 3),
        "error_vs_fp64": {"peak_rel": peak_rel, "rms_rel": rms_rel, "tolerance": 1e-5},
        "latency_ms": {"p50": round(p50, 4), "p99": round(p99, 4)},
        "roofline": roofline,
        "e2e": {"value": round(e2e_value, 2), "unit": "Mvis/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "repetitions_Mvis_per_s": e2e_spread,
                "mode": "the timed steps as one stpgpu_image_batch call from page-locked host buffers (per step: "
                        "H2D of vis/weights/uvw, imaging, D2H of the FP32 image; steps overlap on 8 streams)",
                "single_call": {"value": round(e2e_single, 2),
                                "mode": "one stpgpu_image_visibilities_ex call per step, host buffers"}},
        "gpu_launches": int(l32),
        "clocks": clocks,
    }
    if ws == 1 and not args.headline_only:
        line.update(run_config1_and_source_finder(ctx))
        line["batched"] = run_batched(ctx, min(args.steps, 10), args.warmup)
        line["precision_study"] = run_precision(ctx)
        line["fma_peaks"] = fma_peaks(local)
        line["large_support"] = run_large_support(ctx, line["fma_peaks"])
        line["serving"] = run_serving()
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, snap)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def fma_peaks(device=0):
    """FP32 / FP64 FMA throughput of the device (TFLOP/s), from the probe library built beside the imager."""
    import ctypes

    lib = ctypes.CDLL(os.path.join(ROOT, "fastimaging_b200", "libstpgpu_peaks.so"))
    lib.stpgpu_peaks_fma_tflops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    out = {}
    for name, fp64 in (("fp32_tflops", 0), ("fp64_tflops", 1)):
        v = ctypes.c_double()
        if lib.stpgpu_peaks_fma_tflops(device, fp64, ctypes.byref(v)) != 0:
            raise RuntimeError("FMA probe failed")
        out[name] = round(v.value, 1)
    out["how"] = "independent FMA chains on every SM, best of 5 launches (2 flops per FMA)"
    return out


def run_large_support(ctx, peaks, steps=3):
    """The W-projection snapshot with untruncated W-kernels (kernel_trunc_perc 0: every plane keeps the
    maximum support 16, 33 x 33 complex taps per visibility): the regime where the gridder's complex taps,
    not memory, set the bound.  Algorithmic flops = 8 per tap (complex kernel x complex visibility and the
    accumulation), taps = gridded items x 33^2 (an upper bound: taps that fall beyond the half plane are
    not gridded)."""
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import CONFIG2_IMAGER, config2

    s = config2(seed=2)
    kw = dict(CONFIG2_IMAGER, kernel_trunc_perc=0.0)
    N, n = s.image_size, s.vis.size
    dev = torch.device("cuda", 0)
    dv = torch.from_numpy(s.vis).to(dev)
    dw = torch.from_numpy(s.weights).to(dev)
    duvw = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).to(dev)
    outs = {capi.FP64: torch.empty(N * N, dtype=torch.float64, device=dev),
            capi.FP32C: torch.empty(N * N, dtype=torch.float32, device=dev)}
    res = {}
    for prec, name in ((capi.FP32C, "fp32c"), (capi.FP64, "fp64")):
        odt = capi.F64 if prec == capi.FP64 else capi.F32
        # an untimed call first: the autotuner picks this size class's gridder layout
        ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec, out_dtype=odt, device_ptrs=True,
                               image_out=outs[prec], **kw)
        ctx.set_timing(True)
        infos = []
        for rep in range(steps + 2):
            _, _, info = ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec, out_dtype=odt,
                                                device_ptrs=True, image_out=outs[prec], **kw)
            torch.cuda.synchronize(dev)
            if rep >= 2:
                infos.append(info)
        ctx.set_timing(False)
        total = [sum(i.phase_ms) for i in infos]
        grid = [i.phase_ms[1] for i in infos]
        taps = int(infos[-1].n_grid_items) * (2 * infos[-1].max_plane_support + 1) ** 2
        flops = 8.0 * taps
        g = float(np.median(grid))
        achieved = flops / (g * 1e-3) / 1e12
        peak = peaks["fp64_tflops" if prec == capi.FP64 else "fp32_tflops"]
        res[name] = {"Mvis_per_s": round(n / (float(np.median(total)) * 1e-3) / 1e6, 2),
                     "ms": round(float(np.median(total)), 3), "grid_loop_ms": round(g, 3),
                     "max_plane_support": int(infos[-1].max_plane_support), "taps": taps,
                     "roofline": {"bound": "fp", "kernel": "tile gridder (grid_loop phase)",
                                  "achieved": round(achieved, 2), "peak": peak, "unit": "TFLOP/s",
                                  "frac": round(achieved / peak, 4), "peak_source": "measured (FMA probe)"}}
    d = outs[capi.FP32C].double() - outs[capi.FP64]
    res["fp32c_error_vs_fp64"] = float(d.abs().max() / outs[capi.FP64].abs().max())
    res["fp32c_over_fp64"] = round(res["fp32c"]["Mvis_per_s"] / res["fp64"]["Mvis_per_s"], 3)
    res["workload"] = "as the headline, kernel_trunc_perc 0 (W-kernel support 16 on every plane)"
    return res


def run_batched(ctx, steps, warmup):
    """64 snapshots of uneven sizes (visibility counts log-uniform 50k-2M, images 1024^2-8192^2, W-projection)
    through stpgpu_image_batch (FP32C, graph replay), and the same snapshots through single FP64 calls."""
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import config4

    cases = config4()
    nv = sum(s.vis.size for s, _ in cases)
    snaps, outs64 = [], {}
    for s, kw in cases:
        d = dict(kw)
        d["vis"] = torch.from_numpy(s.vis).cuda()
        d["weights"] = torch.from_numpy(s.weights).cuda()
        d["uvw"] = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda()
        d["image"] = torch.empty(kw["image_size"] ** 2, dtype=torch.float32, device="cuda")
        snaps.append(d)
    for _ in range(max(3, warmup)):
        _, _, bi = ctx.image_batch(snaps, precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=True)
    ms = []
    for _ in range(steps):
        _, infos, bi = ctx.image_batch(snaps, precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=True)
        ms.append(bi.device_ms)
    graph = bi.graph
    st = torch.cuda.ExternalStream(ctx.stream)

    def single_loop(prec):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for (s, kw), d in zip(cases, snaps):
            k = {x: v for x, v in kw.items() if x not in ("image_size", "cell_size")}
            if prec == capi.FP64:
                out = outs64.setdefault(kw["image_size"], torch.empty(kw["image_size"] ** 2, dtype=torch.float64,
                                                                      device="cuda"))
                ctx.image_visibilities(d["vis"], d["weights"], d["uvw"], kw["image_size"], kw["cell_size"],
                                       precision=capi.FP64, out_dtype=capi.F64, device_ptrs=True, image_out=out, **k)
            else:
                ctx.image_visibilities(d["vis"], d["weights"], d["uvw"], kw["image_size"], kw["cell_size"],
                                       precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=True,
                                       image_out=d["image"], **k)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    single_loop(capi.FP64)  # tunes and allocates
    t64 = min(single_loop(capi.FP64) for _ in range(2))
    single_loop(capi.FP32C)
    t32 = min(single_loop(capi.FP32C) for _ in range(2))
    batch_ms = float(np.median(ms))
    v = nv / (batch_ms / 1e3) / 1e6
    v64 = nv / (t64 / 1e3) / 1e6
    del snaps, outs64
    torch.cuda.empty_cache()
    return {"workload": "64 snapshots: visibilities log-uniform 50k-2M (total %d), images from {1024,2048,4096,8192}^2, "
                        "w ~ U[-w_max, w_max], w_max ~ U[0, 2000], GaussianSinc/PSWF, W-projection 16 planes" % nv,
            "value": round(v, 2), "unit": "Mvis/s", "ms_per_batch_p50": round(batch_ms, 3),
            "ms_per_batch_p99": round(float(np.percentile(ms, 99)), 3), "graph_replay": bool(graph),
            "fp64_single_calls": {"value": round(v64, 2), "ms": round(t64, 3)},
            "fp32c_single_calls": {"value": round(nv / (t32 / 1e3) / 1e6, 2), "ms": round(t32, 3)},
            "batched_fp32c_over_fp64_plain": round(v / v64, 3)}


def run_serving(rates=(10.0, 20.0, 50.0, 100.0, 200.0, 500.0), seconds=2.0, slots=4):
    """Poisson arrivals of imaging + source-finding requests (FP32C images, 5 sigma detection, 3 sigma
    analysis, BINAPPROX, 8-connectivity) sampled from a pool of config-4-sized snapshots with 50 point and
    5 extended sources, at offered rates from 10 to 500 requests/s; latency = submit -> done of each request
    (host clock).  A rate of at least 100 requests whose completed throughput falls below 95 % of the offered
    one is past saturation (the queue grows for the length of the run) and is marked so."""
    import numpy as np

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import config5_pool

    import torch

    # request inputs in page-locked host memory (as a receiving front end would hold them); the service
    # returns the islands, not the images
    pool = [((torch.from_numpy(s.vis).pin_memory(), torch.from_numpy(s.weights).pin_memory(),
              torch.from_numpy(np.ascontiguousarray(s.uvw.T)).pin_memory()), kw, s.vis.size)
            for s, kw in config5_pool()]
    rng = np.random.default_rng(55)
    out = []
    for rate in rates:
        srv = capi.Server(slots=slots, hbm_budget_bytes=64 << 30, precision=capi.FP32C)
        try:
            # warm-up: every template once on every slot (buffers, cuFFT plans, gridder tuning), so that
            # the timed arrivals allocate nothing
            for (v, w, uvw), kw, _ in pool:
                srv.prepare(v, w, uvw, find_sources=True, want_image=False, **kw)
            n_req = max(4, int(rate * seconds))
            gaps = rng.exponential(1.0 / rate, size=n_req)
            picks = rng.integers(0, len(pool), size=n_req)
            t_start = time.perf_counter()
            tickets, due = [], 0.0
            for g, p in zip(gaps, picks):
                due += g
                delay = due - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                (v, w, uvw), kw, _ = pool[p]
                tickets.append(srv.submit(v, w, uvw, find_sources=True, want_image=False, **kw))
            lat, nvis, nisl = [], 0, 0
            for t, p in zip(tickets, picks):
                _, _, isl, res = srv.wait(t)
                lat.append(res.done_ms - res.submit_ms)
                nvis += pool[p][2]
                nisl += len(isl)
            wall = time.perf_counter() - t_start
            st = srv.stats()
        finally:
            srv.close()
        out.append({"offered_rps": rate, "requests": len(tickets), "completed_rps": round(len(tickets) / wall, 2),
                    "p50_ms": round(float(np.percentile(lat, 50)), 2),
                    "p99_ms": round(float(np.percentile(lat, 99)), 2), "mean_ms": round(float(np.mean(lat)), 2),
                    "Mvis_per_s": round(nvis / wall / 1e6, 1), "islands_per_request": round(nisl / len(tickets), 1),
                    "peak_in_flight": int(st.peak_in_flight), "slots": slots,
                    "saturated": bool(len(tickets) >= 100 and len(tickets) / wall < 0.95 * rate)})
    return out


def run_config1_and_source_finder(ctx):
    """The reference's CPU-runnable plain imager (2048^2, 100k complex128 visibilities, w = 0, GaussianSinc
    S=3 os=8, FP64) on the GPU against the CPU oracle; then the source finder (5 sigma detection, 3 sigma
    analysis, BINAPPROX, 8-connectivity) on that image and on the 4096^2 headline image, device-resident."""
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import CONFIG1_IMAGER, CONFIG2_IMAGER, config1, config2
    from oracle import stp_oracle as orc

    s = config1()
    N = s.image_size
    dv = torch.from_numpy(s.vis).cuda()
    dw = torch.from_numpy(s.weights).cuda()
    duvw = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda()
    o64 = torch.empty(N * N, dtype=torch.float64, device="cuda")
    st = torch.cuda.ExternalStream(ctx.stream)

    def timed(fn, reps=5):
        for _ in range(2):
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    img = lambda: ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=capi.FP64, out_dtype=capi.F64,
                                         device_ptrs=True, image_out=o64, **CONFIG1_IMAGER)
    t1 = timed(img)
    img()
    torch.cuda.synchronize()
    gpu = o64.cpu().numpy().reshape(N, N).T
    ref, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, N, s.cell_size, threads=len(os.sched_getaffinity(0)),
                                    fast=False, **CONFIG1_IMAGER)
    err = float(np.max(np.abs(gpu - ref)) / np.max(np.abs(ref)))
    out = {"config1": {"workload": "plain imager 2048^2, 100k complex128 visibilities, w = 0, GaussianSinc S=3 "
                                   "os=8, FP64", "ms": round(t1, 4),
                       "Mvis_per_s": round(s.vis.size / (t1 / 1e3) / 1e6, 1),
                       "peak_rel_err_vs_oracle": err, "tolerance": 1e-10}}
    res = []
    s2 = config2()
    N2 = s2.image_size
    o2 = torch.empty(N2 * N2, dtype=torch.float32, device="cuda")
    ctx.image_visibilities(torch.from_numpy(s2.vis).cuda(), torch.from_numpy(s2.weights).cuda(),
                           torch.from_numpy(np.ascontiguousarray(s2.uvw.T)).cuda(), N2, s2.cell_size,
                           precision=capi.FP32C, out_dtype=capi.F32, device_ptrs=True, image_out=o2,
                           **CONFIG2_IMAGER)
    torch.cuda.synchronize()
    for name, im, n in (("2048^2 FP64 image", o64, N), ("4096^2 FP32 image", o2, N2)):
        lab = torch.empty(n * n, dtype=torch.int32, device="cuda")
        call = lambda: ctx.source_find(im, 5.0, 3.0, device_ptrs=True, rows=n, cols=n, label_out=lab)
        t = timed(call, 5)
        isl, _, info = call()
        res.append({"image": name, "ms": round(t, 3), "Mpix_per_s": round(n * n / (t / 1e3) / 1e6, 1),
                    "islands": len(isl), "labels_pos": int(info.n_labels_pos), "labels_neg": int(info.n_labels_neg)})
    out["source_finder"] = res
    return out


def run_precision(ctx):
    """8192^2 image, 4M complex64 visibilities Gaussian-concentrated in uv, PSWF S=4 os=16: FP32 naive and
    FP32 compensated images against the FP64 image of the same library (itself pinned to the oracle)."""
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200.synthetic import CONFIG3_IMAGER, config3

    s = config3()
    N = s.image_size
    dv = torch.from_numpy(s.vis).cuda()
    dw = torch.from_numpy(s.weights).cuda()
    duvw = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda()
    o64 = torch.empty(N * N, dtype=torch.float64, device="cuda")
    o32 = torch.empty(N * N, dtype=torch.float32, device="cuda")
    out = {"workload": "8192^2, 4M complex64 visibilities, uv Gaussian (sigma 0.25 of the radius), PSWF S=4 os=16, "
                       "analytic gcf"}
    ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=capi.FP64, out_dtype=capi.F64, device_ptrs=True,
                           image_out=o64, **CONFIG3_IMAGER)
    torch.cuda.synchronize()
    ref = o64.clone()
    peak = float(ref.abs().max())
    norm = float(torch.linalg.vector_norm(ref))
    # inner half of the field (|x|, |y| < N/4 from the phase centre; the image is unshifted, so these are the
    # first and last N/4 rows and columns), away from the edges where the analytic PSWF correction is smallest
    q = N // 4
    idx = torch.cat([torch.arange(0, q), torch.arange(N - q, N)]).cuda()
    for name, prec in (("fp32_naive", capi.FP32), ("fp32_compensated", capi.FP32C)):
        ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec, out_dtype=capi.F32, device_ptrs=True,
                               image_out=o32, **CONFIG3_IMAGER)
        torch.cuda.synchronize()
        d = o32.double() - ref
        d2 = d.view(N, N).index_select(0, idx).index_select(1, idx)
        out[name] = {"max_abs_over_peak": float(d.abs().max()) / peak,
                     "rms_rel": float(torch.linalg.vector_norm(d)) / norm,
                     "inner_half_field_max_abs_over_peak": float(d2.abs().max()) / peak}
    for prec, name in ((capi.FP64, "fp64"), (capi.FP32C, "fp32c")):
        t = []
        for _ in range(3):
            o = o64 if prec == capi.FP64 else o32
            _, _, info = ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec,
                                                out_dtype=capi.F64 if prec == capi.FP64 else capi.F32,
                                                device_ptrs=True, image_out=o, **CONFIG3_IMAGER)
        st = torch.cuda.ExternalStream(ctx.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(3):
            o = o64 if prec == capi.FP64 else o32
            ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec,
                                   out_dtype=capi.F64 if prec == capi.FP64 else capi.F32, device_ptrs=True,
                                   image_out=o, **CONFIG3_IMAGER)
        e1.record(st)
        e1.synchronize()
        t.append(e0.elapsed_time(e1) / 3)
        out[name + "_Mvis_per_s"] = round(s.vis.size / (t[0] / 1e3) / 1e6, 1)
    del dv, dw, duvw, o64, o32, ref
    torch.cuda.empty_cache()
    return out


def _cpu_one(snap, threads, fast=True):
    from fastimaging_b200.synthetic import CONFIG2_IMAGER
    from oracle import stp_oracle as orc

    kw = {k: v for k, v in CONFIG2_IMAGER.items()}
    t0 = time.perf_counter()
    orc.image_visibilities(snap.vis, snap.weights, snap.uvw, snap.image_size, snap.cell_size, threads=threads,
                           fast=fast, **kw)
    return time.perf_counter() - t0


def _cpu_host():
    """The host the CPU figures ran on: model name, logical CPUs, the affinity set used."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    aff = sorted(os.sched_getaffinity(0))
    return {"cpu_model": model, "nproc": os.cpu_count(), "affinity_count": len(aff),
            "affinity": f"{aff[0]}-{aff[-1]}" if aff and aff[-1] - aff[0] + 1 == len(aff) else ",".join(map(str, aff))}


def _cpu_extra(threads):
    """Further CPU-port figures on the same host: the plain 2048^2 imager (config 1) and the source finder
    on serving-size images (the oracle port's labelling is serial, as the reference's merge step)."""
    from fastimaging_b200 import synthetic as syn
    from oracle import stp_oracle as orc

    out = {}
    s = syn.config1()
    t0 = time.perf_counter()
    img, _ = orc.image_visibilities(s.vis, s.weights, s.uvw, s.image_size, s.cell_size, threads=threads, fast=True,
                                    **syn.CONFIG1_IMAGER)
    dt = time.perf_counter() - t0
    out["config1_plain_2048"] = {"Mvis_per_s": round(s.vis.size / dt / 1e6, 3), "s": round(dt, 3)}
    for size, seed in ((2048, 51), (4096, 52)):
        snap = syn.make_snapshot(seed, 300_000, size, 1.0, n_src=50, flux=(0.5, 10.0), noise_sigma=0.05,
                                 w_range=(-500.0, 500.0), n_extended=5)
        kw = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, gridding_correction=True,
                  analytic_gcf=False, num_wplanes=16, max_wpconv_support=16, undersampling_opt=1,
                  kernel_trunc_perc=1.0)
        im, _ = orc.image_visibilities(snap.vis, snap.weights, snap.uvw, size, 1.0, threads=threads, fast=True, **kw)
        t0 = time.perf_counter()
        orc.source_find(im, 5.0, 3.0, 0.0, True, 5, orc.BINAPPROX, False, False, True, 5)
        dt = time.perf_counter() - t0
        out[f"source_finder_{size}"] = {"Mpix_per_s": round(size * size / dt / 1e6, 2), "ms": round(dt * 1e3, 1)}
    return out


def cpu_baseline(args, snap, budget_s=20.0):
    threads = len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    times = []
    t_start = time.perf_counter()
    while True:
        times.append(_cpu_one(snap, threads))
        if time.perf_counter() - t_start > budget_s or len(times) >= 3:
            break
    n = snap.vis.size
    v = n * len(times) / sum(times) / 1e6
    return {"value": round(v, 3), "unit": "Mvis/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} full config-2 snapshot(s) ({n} vis, 4096^2) through the CPU oracle port "
                      f"(-O3 -ffast-math, OpenMP residue-partitioned gridder, scipy FFT workers={threads})",
            "host": _cpu_host(), "other_workloads": _cpu_extra(threads)}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from fastimaging_b200.synthetic import config2

    snap = config2(seed=2)
    threads = len(os.sched_getaffinity(0))
    for _ in range(max(0, min(args.warmup, 1))):
        _cpu_one(snap, threads)
    times = [_cpu_one(snap, threads) for _ in range(max(1, min(args.steps, 3)))]
    n = snap.vis.size
    v = n * len(times) / sum(times) / 1e6
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": "Mvis/s", "n_gpus": ws, "steps": len(times),
        "warmup": min(args.warmup, 1), "ms_per_step": round(1e3 * sum(times) / len(times), 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded point sources + noise, config-2 shapes)",
        "config": {"workload": WORKLOAD, "n_vis": n, "image_size": snap.image_size, "precision": "fp64"},
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 3), "unit": "Mvis/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} full config-2 snapshot(s) through the CPU oracle port of the "
                                   f"reference algorithm (reference C++ needs Armadillo/TBB, absent)",
                         "host": _cpu_host()},
        "e2e": {"value": round(v, 3), "unit": "Mvis/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_profile_calls(args):
    """A few library calls and nothing else, for ncu captures: imaging calls of one workload, or
    source-finder calls on the headline image (device pointers, no timing)."""
    import numpy as np
    import torch

    from fastimaging_b200 import capi
    from fastimaging_b200 import synthetic as syn

    ctx = capi.Context(0)
    try:
        if args.section == "imager_call":
            s = {1: syn.config1, 2: syn.config2, 3: syn.config3}[args.cfg]()
            kw = dict({1: syn.CONFIG1_IMAGER, 2: syn.CONFIG2_IMAGER, 3: syn.CONFIG3_IMAGER}[args.cfg])
            if args.trunc is not None:
                kw["kernel_trunc_perc"] = args.trunc
            prec = {"fp64": capi.FP64, "fp32": capi.FP32, "fp32c": capi.FP32C}[args.prec]
            N = s.image_size
            out = torch.empty(N * N, dtype=torch.float64 if prec == capi.FP64 else torch.float32, device="cuda")
            dv = torch.from_numpy(s.vis).cuda()
            dw = torch.from_numpy(s.weights).cuda()
            duvw = torch.from_numpy(np.ascontiguousarray(s.uvw.T)).cuda()
            def call():
                return ctx.image_visibilities(dv, dw, duvw, N, s.cell_size, precision=prec,
                                              out_dtype=capi.F64 if prec == capi.FP64 else capi.F32,
                                              device_ptrs=True, image_out=out, **kw)

            for _ in range(args.calls):
                _, _, info = call()
            torch.cuda.synchronize()
            print(json.dumps({"section": "imager_call", "cfg": args.cfg, "prec": args.prec,
                              "n_grid_items": int(info.n_grid_items), "max_plane_support": int(info.max_plane_support),
                              "flags": int(info.flags)}))
            if args.timeline:
                print_timeline(call)
        else:
            s = syn.config2()
            img, _, _ = ctx.image_visibilities(s.vis, s.weights, s.uvw, 4096, s.cell_size, precision=capi.FP32C,
                                               out_dtype=capi.F32, **syn.CONFIG2_IMAGER)
            dimg = torch.from_numpy(np.asfortranarray(img).reshape(-1, order="F").copy()).cuda()
            lab = torch.empty(4096 * 4096, dtype=torch.int32, device="cuda")
            def call():
                return ctx.source_find(dimg, 5.0, 3.0, 0.0, True, 5, capi.BINAPPROX, False, False, True, 5,
                                       device_ptrs=True, rows=4096, cols=4096, label_out=lab)

            for _ in range(args.calls):
                isl, _, info = call()
            torch.cuda.synchronize()
            print(json.dumps({"section": "sf_call", "islands": len(isl)}))
            if args.timeline:
                print_timeline(call)
    finally:
        ctx.close()


def print_timeline(call):
    """Device timeline of one warm call (after the calls above, so a repeated device-pointer call replays its
    CUDA graph), recorded by the CUDA activity API through torch.profiler: the L2 is flushed (a 256 MB write)
    before each of three calls and the last is printed, one JSON line per kernel or copy: start offset, duration
    and the idle gap before it, in microseconds."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    marks = []
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(3):
            flush.zero_()
            torch.cuda.synchronize()
            call()
            torch.cuda.synchronize()
    with tempfile.TemporaryDirectory() as td:
        fn = os.path.join(td, "trace.json")
        prof.export_chrome_trace(fn)
        with open(fn) as f:
            tr = json.load(f)
    ev = [e for e in tr["traceEvents"]
          if e.get("ph") == "X" and e.get("cat") in ("kernel", "gpu_memcpy", "gpu_memset")]
    ev.sort(key=lambda e: e["ts"])
    calls, cur = [], []
    for e in ev:  # the flush kernels separate the calls
        if "at::native" in e["name"] or "FillFunctor" in e["name"]:
            if cur:
                calls.append(cur)
            cur = []
            continue
        cur.append(e)
    if cur:
        calls.append(cur)
    last = calls[-1]
    t0 = last[0]["ts"]
    prev = t0
    for e in last:
        marks.append({"kernel": e["name"][:100], "start_us": round(e["ts"] - t0, 1), "us": round(e["dur"], 1),
                      "gap_us": round(e["ts"] - prev, 1)})
        prev = max(prev, e["ts"] + e["dur"])
    for m in marks:
        print(json.dumps(m))
    print(json.dumps({"span_us": round(prev - t0, 1), "launches": len(last)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the batched, precision-study and serving sections")
    ap.add_argument("--section", choices=["config1_sf", "imager_call", "sf_call"], default=None,
                    help="run one section alone, for profiling: config1_sf (the plain 2048^2 imager and the "
                         "source finder, JSON), imager_call (--calls imaging calls of --cfg in --prec, device "
                         "pointers), sf_call (--calls source-finder calls on the 4096^2 FP32 headline image)")
    ap.add_argument("--cfg", type=int, choices=[1, 2, 3], default=2, help="imager_call: workload 1, 2 or 3")
    ap.add_argument("--prec", choices=["fp64", "fp32", "fp32c"], default="fp32c", help="imager_call: precision")
    ap.add_argument("--trunc", type=float, default=None, help="imager_call: W-kernel truncation percentage")
    ap.add_argument("--calls", type=int, default=2, help="imager_call / sf_call: number of calls")
    ap.add_argument("--timeline", action="store_true",
                    help="imager_call / sf_call: then print the device timeline of one warm call")
    args = ap.parse_args()
    if args.section in ("imager_call", "sf_call"):
        run_profile_calls(args)
        return
    if args.section == "config1_sf":
        from fastimaging_b200 import capi

        ctx = capi.Context(0)
        try:
            print(json.dumps(run_config1_and_source_finder(ctx)), flush=True)
        finally:
            ctx.close()
        return
    if args.warmup < 3 and args.impl != "reference":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
