#!/usr/bin/env python
"""Benchmark of the CTF-estimation hot path on B200.

Workload (one "step"): the uneven batch -- 256 independent synthetic
micrographs, each a seeded pick of 4096 x 4096, 5760 x 4092 or 3838 x 3710
float32 at 0.8-1.5 A/px (rescaled to >= 1.2 A/px like the reference),
defocus 5000-40000 A, astigmatism 0-1000 A at a random angle, dose
0.5-2 e/A^2 -- searched in one gcf_run_batch_mode call.

  value  : micrographs/s of the learned + batched + BF16 contraction path
           (GCF_SEARCH_LEARNED when trained weights are present, else
           GCF_SEARCH_BF16) with the rescale as two BF16 tensor-core
           products (GCF_RESCALE_GEMM; `fast_with_cufft_rescale` is the same
           path with the reference's cuFFT rescale), micrographs resident in
           HBM, device time from CUDA events on the library stream
  plain  : the same batch through this project's plain FP32 exhaustive
           search and the cuFFT rescale, batched (one GCF_SEARCH_PLAIN call) and in the
           reference's single-file mode (one call per micrograph)
  e2e    : the headline path with pinned HOST buffers, host clock around the
           call: host->device copies of the 256 images and the result rows
           are inside the timed region
  defocus_error : the fast path against the plain path on the same batch
           (median |d defocus|, fraction within one search step) and both
           against the generator's truth

Secondary figures on the same line: the 41-tilt 4096^2 series at 1.35 A/px
through the reference's series policy (plain search), one 4096^2
micrograph at 1.0 A/px (rescale path) in single-file mode, and the mixed
stream of 2000 uneven micrographs with 8 tilt series of 61 tilts.

Rank r of N processes its own batch (seeded by r): weak scaling, replicas
only, no data-path collective.  `--impl reference` times the reference's own
CUDA implementation of the path, built from its sources, on a rotating
sample of the same batch (single-file mode, as the reference runs
independent micrographs).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BATCH = 256
METRIC = "4096^2 micrographs/s, learned+batched+BF16 vs plain GPU path; defocus error (A)"
SERIES_PX = 1.35
# DRAM bytes (read + write) of k_fused_spectrum per algorithmic byte (the
# images read once), from ncu dram__bytes_read.sum + dram__bytes_write.sum of
# the first tile launch of `bench.py --batch 16 --steps 1 --warmup 3
# --no-secondary --no-cpu-baseline --no-autotune --no-graphs --mode bf16`
# (16 micrographs of this workload, 904.6 MB of algorithmic bytes)
TILE_KERNEL_TRAFFIC_RATIO = (1_028_731_000 + 62_378_752) / 904_559_168
TILE_KERNEL_TRAFFIC_CAPTURE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the first k_fused_spectrum launch "
                               "of bench.py --batch 16 (16 micrographs of this workload), per algorithmic byte, "
                               "scaled by this launch's algorithmic bytes")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--batch", type=int, default=N_BATCH)
    ap.add_argument("--mode", default="auto", choices=["auto", "bf16", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rescale-compare", action="store_true",
                    help="only rescale one frame of each raw size of the batch (3838x3710 @ 0.9, 5760x4092 @ 0.8, "
                         "4096x4096 @ 1.0 A/px) through both rescale implementations, 2 + 5 calls each "
                         "(for a profiler's launch list), and print their wall-clock times")
    ap.add_argument("--rescale", default="gemm", choices=["gemm", "cufft", "lines"],
                    help="rescale of the headline path (the plain path always takes cuFFT, the reference's calls)")
    ap.add_argument("--no-graphs", action="store_true", help="launch every kernel from the host")
    ap.add_argument("--no-autotune", action="store_true", help="default shapes instead of the autotuner's")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the tilt-series and 1.0 A/px single-micrograph figures")
    ap.add_argument("--shrink", type=int, default=1,
                    help="divide the micrograph sizes by this factor (quick checks only)")
    return ap.parse_args()


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


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


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        busy = [r for r in rows if r[0] > 0.5 * r[1]] or rows
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, v in zip(names, r[2:]):
                if v.lower() == "active":
                    reasons.add(k)
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": rows[0][1],
                "reasons": sorted(reasons), "samples": len(rows)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "_fallback": True}


def batch_specs(n, seed, shrink=1):
    from gctffind_b200 import synth
    sizes = tuple((w // shrink // 2 * 2, h // shrink // 2 * 2) for w, h in synth.UNEVEN_SIZES)
    return synth.uneven_batch_specs(n, seed=seed, sizes=sizes)


def make_batch(rank, n, device, shrink=1):
    import torch
    from gctffind_b200 import synth
    specs = batch_specs(n, 2 + rank, shrink)
    imgs = [synth.make_micrograph(s, device=device) for s in specs]
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    return specs, imgs


def workload_name(n):
    return (f"uneven batch of {n} independent micrographs (4096x4096 / 5760x4092 / 3838x3710 float32, "
            "0.8-1.5 A/px rescaled to >= 1.2, df 5000-40000 A, astig 0-1000 A, dose 0.5-2 e/A^2), "
            "one search per micrograph")


def search_step(spec_mean):
    """The plain search's last mean-defocus step (max(20 A, range / 31) with
    range 0.525 * 0.2 * mean, FindCTF/CFindDefocus2D.cpp:166-182, 296-300)."""
    return max(20.0, 0.105 * spec_mean / 31.0)


def defocus_error(fast, plain, specs):
    import numpy as np
    from gctffind_b200 import synth
    d_fp, within, d_ft, d_pt = [], [], [], []
    for f, p, s in zip(fast, plain, specs):
        mf, mp = 0.5 * (f.df_min + f.df_max), 0.5 * (p.df_min + p.df_max)
        mt = 0.5 * (s.df_min + s.df_max)
        step = search_step(mp)
        d_fp.append(abs(mf - mp))
        within.append(abs(f.df_min - p.df_min) <= step and abs(f.df_max - p.df_max) <= step)
        if synth.inside_reference_envelope(s):
            d_ft.append(abs(mf - mt))
            d_pt.append(abs(mp - mt))
    return {"median_abs_ddf_vs_plain_A": round(float(np.median(d_fp)), 2),
            "p90_abs_ddf_vs_plain_A": round(float(np.percentile(d_fp, 90)), 2),
            "frac_within_one_step_of_plain": round(float(np.mean(within)), 4),
            "median_abs_ddf_vs_truth_A": {"fast": round(float(np.median(d_ft)), 2) if d_ft else None,
                                          "plain": round(float(np.median(d_pt)), 2) if d_pt else None,
                                          "micrographs": len(d_ft),
                                          "note": "inside the reference's search envelope"},
            "one_step": "max(20 A, 0.105 * mean / 31): the plain search's last mean-defocus step"}


def timed_batch(ctx, imgs, pxs, op, mode, steps, warmup, world, tag=""):
    import torch
    for _ in range(warmup):
        ctx.run_batch(imgs, pxs, op, mode=mode)
    barrier(world)
    torch.cuda.synchronize()
    dev_ms, launches, stage, ftimes, fcounts = 0.0, 0, {}, {}, {}
    graph_launches = 0
    res = None
    torch.cuda.nvtx.range_push(f"timed_mode{mode}{tag}")
    for _ in range(steps):
        res = ctx.run_batch(imgs, pxs, op, mode=mode)
        st = ctx.stage_times()
        dev_ms += st["total"]
        for k, v in st.items():
            stage[k] = stage.get(k, 0.0) + v / steps
        launches += ctx.launch_count()
        graph_launches += ctx.graph_info()["graph_launches"]
        if mode != 0:
            for k, v in ctx.fast_times().items():
                ftimes[k] = ftimes.get(k, 0.0) + v / steps
            fcounts = ctx.fast_counts()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier(world)
    return {"ms": max_over_ranks(dev_ms / steps, world), "results": res, "stage": stage,
            "launches": launches // steps, "fast_ms": ftimes, "fast_counts": fcounts,
            "search_counts": ctx.search_counts(), "graph_launches_per_step": graph_launches / steps,
            "graph": ctx.graph_info()}


def timed_single_file(ctx, imgs, pxs, op, steps, world):
    """The reference's single-file mode: one plain search call per
    micrograph, one pass over the batch per step."""
    import torch
    for k in range(len(imgs)):
        ctx.run_batch([imgs[k]], [pxs[k]], op, mode=0)
    barrier(world)
    torch.cuda.synchronize()
    dev_ms = 0.0
    t0 = time.perf_counter()
    for _ in range(steps):
        for k in range(len(imgs)):
            ctx.run_batch([imgs[k]], [pxs[k]], op, mode=0)
            dev_ms += ctx.stage_times()["total"]
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1000.0 / steps
    barrier(world)
    return max_over_ranks(dev_ms / steps, world), max_over_ranks(wall, world)


def cpu_baseline(host, specs, budget_s=20.0):
    """FP64 OpenMP oracle on the host cores: the plain full search (rescale,
    spectrum, 1D + 2D) of the batch's micrographs in order, as many as fit
    the time budget (at least one)."""
    from gctffind_b200 import synth
    from oracle import oracle as O
    O.build()
    cores = O.num_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    done = 0
    for img, s in zip(host, specs):
        if done and time.perf_counter() - t0 > budget_s:
            break
        nw, nh, px_n, _ = O.rescale_dims(img.shape[1], img.shape[0], s.pixel_size)
        im = O.rescale(img, s.pixel_size) if px_n != s.pixel_size else img
        O.find_ctf_image(im, px_n, O.params(pixel_size=px_n, tile_size=512), mode=0)
        done += 1
    dt = time.perf_counter() - t0
    del synth
    return {"value": done / dt, "unit": "micrographs/s", "cores": cores, "kind": "port",
            "sample": f"the first {done} micrographs of the batch (rescale + spectrum + 1D + 2D full "
                      f"search), FP64 oracle, {cores} OpenMP threads, {dt:.1f} s"}


def stream_figures(ctx, G, fast_mode, world, rank, n_batches=8, per_batch=250, series_tilts=61, lines_ctx=None,
                   fast_rescale=0):
    """The mixed stream: 2000 micrographs of the uneven mix in batches of 250,
    interleaved with 8 tilt series of 61 tilts (-60..+60 deg in 2 deg
    steps, 4096^2 at 1.35 A/px).  Each batch and series is made on the
    device (not timed) and then timed, device time from the library's CUDA
    events: the batches through the headline search and through the plain
    search, the series through the reference's series policy (the series
    search is the plain one in both columns).  Each batch's first call also
    makes a cuFFT plan for every new rescaled size (the pixel size varies
    continuously); that call (headline search, cuFFT rescale) is reported on
    its own, and the timed calls run with the plans made: the headline
    search with its rescale (fast_rescale), the plain search with cuFFT's.  With lines_ctx (a context whose
    rescale is the library's line transforms, which make no plans), each
    batch's first and second calls through it are reported as well.
    Defocus error: the headline search against the plain one on the 2000
    micrographs."""
    import numpy as np
    import torch
    from gctffind_b200 import synth
    op = G.make_optics()
    fast_ms = plain_ms = first_ms = lines_first_ms = lines_ms = 0.0
    n_mics = 0
    fast_res, plain_res, specs_all = [], [], []
    for b in range(n_batches):
        specs = synth.uneven_batch_specs(per_batch, seed=1000 + 17 * rank + b)
        imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
        pxs = [s.pixel_size for s in specs]
        torch.cuda.synchronize()
        if lines_ctx is not None:
            lines_ctx.run_batch(imgs, pxs, op, mode=fast_mode)
            lines_first_ms += lines_ctx.stage_times()["total"]
            lines_ctx.run_batch(imgs, pxs, op, mode=fast_mode)
            lines_ms += lines_ctx.stage_times()["total"]
        ctx.set_rescale_impl(G.GCF_RESCALE_CUFFT)
        ctx.run_batch(imgs, pxs, op, mode=fast_mode)
        first_ms += ctx.stage_times()["total"]
        ctx.set_rescale_impl(fast_rescale)
        fast_res += ctx.run_batch(imgs, pxs, op, mode=fast_mode)
        fast_ms += ctx.stage_times()["total"]
        ctx.set_rescale_impl(G.GCF_RESCALE_CUFFT)
        plain_res += ctx.run_batch(imgs, pxs, op, mode=G.GCF_SEARCH_PLAIN)
        plain_ms += ctx.stage_times()["total"]
        specs_all += specs
        n_mics += per_batch
        del imgs
        torch.cuda.empty_cache()
        sspecs = synth.tilt_series_specs(n_tilts=series_tilts, step_deg=2.0, size=4096, pixel_size=SERIES_PX,
                                         dose=3.0, df0=float(np.random.default_rng(b).uniform(15000, 35000)),
                                         seed=500 + 13 * rank + b)
        simgs = [synth.make_micrograph(s, device="cuda") for s in sspecs]
        order = G.series_order(synth.tilt_angles(series_tilts, 2.0)).order
        torch.cuda.synchronize()
        ctx.run_series(simgs, G.make_optics(pixel_size=SERIES_PX), order, is_tomo=True)
        t = ctx.stage_times()["total"]
        fast_ms += t
        plain_ms += t
        first_ms += t
        lines_first_ms += t
        lines_ms += t
        n_mics += series_tilts
        del simgs
        torch.cuda.empty_cache()
    fast_ms = max_over_ranks(fast_ms, world)
    plain_ms = max_over_ranks(plain_ms, world)
    lines = None
    if lines_ctx is not None:
        lines = {"first_call_value": round(world * n_mics / (max_over_ranks(lines_first_ms, world) / 1000.0), 2),
                 "value": round(world * n_mics / (max_over_ranks(lines_ms, world) / 1000.0), 2),
                 "note": "the batches' rescale through the library's line transforms (gcf_resize.cu), which "
                         "make no plans: each batch's first call and its second call; series as above"}
    return {"workload": f"stream of {n_batches * per_batch} micrographs (uneven mix, batches of {per_batch}) "
                        f"interleaved with {n_batches} tilt series of {series_tilts} x 4096^2 (2 deg steps), "
                        "in HBM; each batch / series timed once on the device",
            "value": round(world * n_mics / (fast_ms / 1000.0), 2), "unit": "micrographs/s",
            "plain_value": round(world * n_mics / (plain_ms / 1000.0), 2),
            "first_call_value": round(world * n_mics / (max_over_ranks(first_ms, world) / 1000.0), 2),
            "first_call_note": "each batch's first call (cuFFT rescale), cuFFT plans of its new rescaled sizes "
                               "included",
            "speedup_vs_plain": round(plain_ms / fast_ms, 3), "micrographs": n_mics,
            "defocus_error": defocus_error(fast_res, plain_res, specs_all),
            "rescale_lines": lines}


def series_figures(ctx, G, steps, warmup, world, rank):
    """41-tilt 4096^2 series at 1.35 A/px, reference series policy, plain
    search: device-resident and end to end (full spectra requested, as the
    reference's CFindSeriesCtfs produces them per package)."""
    import torch
    from gctffind_b200 import synth
    specs = synth.tilt_series_specs(n_tilts=41, step_deg=3.0, size=4096, pixel_size=SERIES_PX, dose=3.0,
                                    df0=30000.0, seed=1 + rank)
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    order = G.series_order(synth.tilt_angles(41, 3.0)).order
    op = G.make_optics(pixel_size=SERIES_PX)
    for _ in range(warmup):
        ctx.run_series(imgs, op, order, is_tomo=True, want_full=True)
    torch.cuda.synchronize()
    ms = 0.0
    for _ in range(steps):
        ctx.run_series(imgs, op, order, is_tomo=True, want_full=True)
        ms += ctx.stage_times()["total"]
    ms = max_over_ranks(ms / steps, world)
    host = [im.cpu().pin_memory() for im in imgs]
    del imgs
    torch.cuda.empty_cache()
    ctx.run_series(host, op, order, is_tomo=True, want_full=True)
    wall = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.run_series(host, op, order, is_tomo=True, want_full=True)
        wall += time.perf_counter() - t0
    wall = max_over_ranks(wall / steps * 1000.0, world)
    return {"workload": "tilt series 41 x 4096^2 float32 @ 1.35 A/px, 3 e/A^2, df 30000 A + tilt gradient; "
                        "CFindSeriesCtfs policy (zero tilt full, rest refined), plain FP32 search, full "
                        "diagnostic spectra returned",
            "value": round(world * 41 / (ms / 1000.0), 2), "unit": "micrographs/s", "ms_per_step": round(ms, 3),
            "e2e": {"value": round(world * 41 / (wall / 1000.0), 2), "unit": "micrographs/s",
                    "ms_per_step": round(wall, 3), "h2d_bytes_per_step": 41 * 4096 * 4096 * 4,
                    "d2h_bytes_per_step": 41 * (512 * 512 * 4 + 40), "timing": "host clock around the call"}}


def single_1p0(ctx, G, steps):
    """One 4096^2 micrograph at 1.0 A/px (Fourier-cropped to 3412^2 at
    1.2 A/px first), plain search, single-file mode."""
    import torch
    from gctffind_b200 import synth
    spec = synth.MicrographSpec(width=4096, height=4096, pixel_size=1.0, df_min=14850.0, df_max=15150.0,
                                azimuth_deg=20.0, dose=1.0, seed=2024)
    img = synth.make_micrograph(spec, device="cuda")
    op = G.make_optics()
    for _ in range(3):
        ctx.run_batch([img], [1.0], op, mode=0)
    ms, st = 0.0, {}
    for _ in range(steps):
        r = ctx.run_batch([img], [1.0], op, mode=0)[0]
        s = ctx.stage_times()
        ms += s["total"]
        for k, v in s.items():
            st[k] = st.get(k, 0.0) + v / steps
    torch.cuda.synchronize()
    return {"workload": "one 4096^2 micrograph @ 1.0 A/px (rescaled to 3412^2 @ 1.2 A/px), df 15000 A, "
                        "astig 300 A at 20 deg, 1 e/A^2; plain search, one call",
            "value": round(1000.0 / (ms / steps), 2), "unit": "micrographs/s", "ms": round(ms / steps, 3),
            "stage_ms": {k: round(v, 3) for k, v in st.items()},
            "result": {"df_min": round(r.df_min, 1), "df_max": round(r.df_max, 1), "azimuth": round(r.azimuth, 2)}}


def h2d_rate(src, device):
    """Host -> device copy rate of this box (GB/s): one pinned micrograph
    copied 8 times, CUDA events around the copies."""
    import torch
    dst = torch.empty(src.shape, dtype=src.dtype, device=f"cuda:{device}")
    dst.copy_(src, non_blocking=True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(8):
        dst.copy_(src, non_blocking=True)
    b.record()
    b.synchronize()
    return round(8 * src.numel() * 4 / (a.elapsed_time(b) / 1000.0) / 1e9, 1)


def tile_kernel_roofline(stage, imgs_dims, pk):
    """k_fused_spectrum (+ its cluster-less companion) over every tile of the
    batch: algorithmic bytes = each (rescaled) image the kernel reads, read
    once; time = the union of its launches inside the timed calls."""
    ms = stage.get("tile_kernel", 0.0)
    algo = sum(4 * w * h for w, h in imgs_dims)
    achieved = algo / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
    peak = pk.get("hbm_gbs", 6650.0)
    # FFT work of the same launch: 512^2 tiles at a 256 stride (CGenAvgSpectrum's
    # layout), 2.5 N log2 N flops per real 2D FFT of N = 512^2 points plus the
    # taper, mean and |F| per pixel
    tiles = sum(max(0, (w - 256) // 256) * max(0, (h - 256) // 256) for w, h in imgs_dims)
    flops = tiles * (2.5 * 512 * 512 * 18 + 6 * 512 * 512)
    tflops = flops / (ms / 1000.0) / 1e12 if ms > 0 else 0.0
    return {"kernel": "k_fused_spectrum (8-CTA clusters) + k_fused_spectrum_solo (the SMs the clusters leave free)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": "fallback" if pk.get("_fallback") else "measured",
            "traffic": int(algo * TILE_KERNEL_TRAFFIC_RATIO),
            "traffic_source": TILE_KERNEL_TRAFFIC_CAPTURE,
            "algorithmic_bytes_per_launch": algo, "launch_ms": round(ms, 3),
            "compute": {"tiles": tiles, "fft_flops_per_launch": flops, "achieved_tflops": round(tflops, 2),
                        "fp32_nominal_tflops": 74.4, "frac_of_nominal_fp32": round(tflops / 74.4, 4),
                        "note": "the kernel is bound by FP32 issue and shared-memory exchanges, not HBM: a tile "
                                "costs ~13.4 MFLOP per 1 MB read"}}


def run_reference(args, rank, world):
    """--impl reference: the reference's own CTF path (built from its
    sources, oracle/_ref/libgcfref.so) on the same B200, in its single-file
    mode, on a rotating sample of the batch: step k takes micrographs
    3k, 3k+1, 3k+2 (mod the batch), so the steps together cover different
    sizes and pixel sizes.  Rank 0 alone runs it."""
    if rank != 0:
        return 0
    import numpy as np
    import torch
    from oracle import refimpl
    on_gpu = torch.cuda.is_available()
    n = args.batch
    per_step = 3
    need = min(n, (args.warmup + args.steps) * per_step)
    from gctffind_b200 import synth
    specs = batch_specs(n, 2, args.shrink)
    sel = [specs[i % n] for i in range(need)]
    host = [synth.make_micrograph(s, device="cuda" if on_gpu else "cpu").cpu().numpy() for s in sel]
    if on_gpu:
        torch.cuda.empty_cache()
    workload = workload_name(n)
    if not (on_gpu and refimpl.available()):
        cb = cpu_baseline(host, sel, budget_s=30.0 if args.shrink == 1 else 2.0)
        line = {"metric": METRIC, "value": round(cb["value"], 4), "unit": "micrographs/s", "n_gpus": 1,
                "steps": 1, "warmup": 0, "ms_per_step": round(1000.0 / cb["value"], 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": workload, "note": "reference CUDA build unavailable here: FP64 oracle "
                                                         "port on the host"},
                "cpu_baseline": cb,
                "e2e": {"value": round(cb["value"], 4), "unit": "micrographs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    secs, cnt = [], 0
    for k in range(args.warmup + args.steps):
        t = 0.0
        for q in range(per_step):
            i = (k * per_step + q) % len(sel)
            _, _, dt = refimpl.run_series([host[i]], sel[i].pixel_size, [0], is_tomo=False, tile=512)
            t += dt
        if k >= args.warmup:
            secs.append(t)
            cnt += per_step
    total = sum(secs)
    v = cnt / total
    sizes = sorted({(s.width, s.height) for s in sel[args.warmup * per_step:]})
    sample = (f"reference CUDA build on the B200 (GCtfFind has no CPU path), single-file mode: {per_step} "
              f"micrographs per step from the batch, different ones each step ({cnt} timed, sizes {sizes}); "
              f"host clock around CFindSeriesCtfs::DoIt per micrograph, images in host memory")
    line = {"metric": METRIC, "value": round(v, 4), "unit": "micrographs/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 * total / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload, "tile": 512, "search": "the reference's FP32 search",
                       "ranks": "rank 0 only (n_gpus counts the GPUs this line used)"},
            "cpu_baseline": {"value": round(v, 4), "unit": "micrographs/s", "cores": 1, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(v, 4), "unit": "micrographs/s",
                    "h2d_bytes_per_step": int(np.mean([4 * s.width * s.height for s in sel]) * per_step),
                    "d2h_bytes_per_step": per_step * 20}}
    print(json.dumps(line), flush=True)
    return 0


def rescale_compare(G, dev):
    """One frame of each raw size below 1.2 A/px of the uneven batch through
    gcf_rescale with the line transforms, the tensor-core products and cuFFT;
    wall clock per call (the rescaled frame is copied to the host by the
    call)."""
    import numpy as np
    import torch
    ctx = G.Context(dev, 512, 0)
    rng = np.random.default_rng(0)
    out = []
    for (w, h, px) in [(3838, 3710, 0.9), (5760, 4092, 0.8), (4096, 4096, 1.0)]:
        img = torch.from_numpy(rng.poisson(2.0, size=(h, w)).astype(np.float32)).to(f"cuda:{dev}")
        for name, impl in (("lines", G.GCF_RESCALE_LINES), ("gemm", G.GCF_RESCALE_GEMM),
                           ("cufft", G.GCF_RESCALE_CUFFT)):
            ctx.set_rescale_impl(impl)
            for _ in range(2):
                ctx.rescale(img, px)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(5):
                ctx.rescale(img, px)
            torch.cuda.synchronize()
            out.append({"raw": [w, h], "px": px, "impl": name,
                        "wall_ms_per_call": round((time.perf_counter() - t0) / 5 * 1e3, 3)})
    ctx.close()
    print(json.dumps({"rescale_compare": out, "note": "wall clock includes the copy of the rescaled frame to "
                      "the host; kernel times come from a profiler's launch list of this command"}))
    return 0


def main():
    args = parse()
    rank, world, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    import numpy as np
    import torch
    import gctffind_b200 as G
    torch.cuda.set_device(local)
    if args.rescale_compare:
        return rescale_compare(G, local)
    ctx = G.Context(local, 512, 0)
    op = G.make_optics()
    # the project's autotuner picks the tile-kernel shape and the contraction
    # tile; repeated batch calls run as captured CUDA graphs
    tuning = None if args.no_autotune else ctx.autotune()
    ctx.set_graphs(not args.no_graphs)
    specs, imgs = make_batch(rank, args.batch, f"cuda:{local}", args.shrink)
    pxs = [s.pixel_size for s in specs]
    learned = args.mode == "learned" or (args.mode == "auto" and G.learned_available())
    fast_mode = G.GCF_SEARCH_LEARNED if learned else G.GCF_SEARCH_BF16
    if learned:
        G.load_learned(ctx)
    fast_rescale = {"gemm": G.GCF_RESCALE_GEMM, "cufft": G.GCF_RESCALE_CUFFT,
                    "lines": G.GCF_RESCALE_LINES}[args.rescale]

    clk = ClockSampler(local)
    clk.start()
    # ---- the headline path, device-resident ----
    ctx.set_rescale_impl(fast_rescale)
    torch.cuda.nvtx.range_push("fast_steps")
    fast = timed_batch(ctx, imgs, pxs, op, fast_mode, args.steps, args.warmup, world)
    torch.cuda.nvtx.range_pop()
    # ---- the contraction search without the network (what the network saves) ----
    nonet = timed_batch(ctx, imgs, pxs, op, G.GCF_SEARCH_BF16, args.steps, min(args.warmup, 2), world) \
        if learned else None
    # ---- plain FP32 search with the reference's cuFFT rescale: batched, and single-file mode ----
    ctx.set_rescale_impl(G.GCF_RESCALE_CUFFT)
    plain = timed_batch(ctx, imgs, pxs, op, G.GCF_SEARCH_PLAIN, args.steps, min(args.warmup, 2), world)
    single_ms, single_wall = timed_single_file(ctx, imgs, pxs, op, max(1, min(args.steps, 2)), world)
    # ---- the headline search with the cuFFT rescale (what the tensor-core rescale saves) ----
    fast_cufft = timed_batch(ctx, imgs, pxs, op, fast_mode, args.steps, min(args.warmup, 2), world,
                             tag="_cufft_rescale") if fast_rescale != G.GCF_RESCALE_CUFFT else None
    ctx.set_rescale_impl(fast_rescale)
    # ---- end to end: pinned host inputs, host clock around the call ----
    host = [im.cpu().pin_memory() for im in imgs]
    dims = [(G.rescale_dims(s.width, s.height, s.pixel_size)[0], G.rescale_dims(s.width, s.height, s.pixel_size)[1])
            for s in specs]
    del imgs
    torch.cuda.empty_cache()
    for _ in range(2):   # the second call captures the graph the timed calls replay
        ctx.run_batch(host, pxs, op, mode=fast_mode)
    barrier(world)
    e2e_wall = 0.0
    e2e_stage = {}
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.run_batch(host, pxs, op, mode=fast_mode)
        e2e_wall += time.perf_counter() - t0
        for k, v in ctx.stage_times().items():
            e2e_stage[k] = e2e_stage.get(k, 0.0) + v / args.steps
    e2e_graph = ctx.graph_info()
    e2e_ms = max_over_ranks(e2e_wall / args.steps * 1000.0, world)
    pcie = h2d_rate(host[0], local)
    clocks = clk.stop()
    n = args.batch
    value = world * n / (fast["ms"] / 1000.0)
    pk = peaks()
    fc, ft = fast["fast_counts"], fast["fast_ms"]
    prod_ms = ft.get("product", 0.0)
    tflops = 2.0 * fc.get("tensor_macs", 0) / (prod_ms / 1000.0) / 1e12 if prod_ms > 0 else 0.0
    bf16_peak = pk.get("bf16_tflops", 1590.0)
    line = {"metric": METRIC, "value": round(value, 2), "unit": "micrographs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(fast["ms"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32",
            "data": "synthetic",
            "config": {"workload": workload_name(n), "search": ["bf16", "learned"][int(learned)],
                       "rescale": args.rescale,
                       "tile": 512, "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2 ({sum(4 * s.width * s.height for s in specs) / 1e9:.1f} GB "
                             "per step)"},
            "plain": {"batched": {"value": round(world * n / (plain["ms"] / 1000.0), 2), "ms_per_step": round(plain["ms"], 3),
                                  "stage_ms": {k: round(v, 3) for k, v in plain["stage"].items()}},
                      "single_file": {"value": round(world * n / (single_ms / 1000.0), 2),
                                      "ms_per_step": round(single_ms, 3),
                                      "wall_ms_per_step": round(single_wall, 3),
                                      "note": "one plain call per micrograph (the reference's single-file mode); "
                                              "device time summed over the calls"}},
            "speedup": {"vs_plain_single_file": round(single_ms / fast["ms"], 3),
                        "vs_plain_batched": round(plain["ms"] / fast["ms"], 3)},
            "bf16_without_network": None if nonet is None else {
                "value": round(world * n / (nonet["ms"] / 1000.0), 2), "ms_per_step": round(nonet["ms"], 3),
                "search_ms": round(nonet["stage"].get("search1d", 0.0) + nonet["stage"].get("search2d", 0.0), 3),
                "table_candidates": nonet["fast_counts"].get("table_cand"),
                "tensor_macs": nonet["fast_counts"].get("tensor_macs"),
                "learned_search_ms": round(fast["stage"].get("search1d", 0.0) + fast["stage"].get("search2d", 0.0), 3),
                "learned_network_ms": round(ft.get("network", 0.0), 3),
                "note": "the same batch through the contraction search without the learned window; "
                        "learned_search_ms is the headline's search1d + search2d, learned_network_ms its "
                        "network (inputs and layers), which runs before the search stages"},
            "fast_with_cufft_rescale": None if fast_cufft is None else {
                "value": round(world * n / (fast_cufft["ms"] / 1000.0), 2),
                "ms_per_step": round(fast_cufft["ms"], 3),
                "stage_ms": {k: round(v, 3) for k, v in fast_cufft["stage"].items()},
                "defocus_error": defocus_error(fast_cufft["results"], plain["results"], specs),
                "note": "the headline search with the reference's cuFFT rescale instead of the tensor-core one"},
            "defocus_error": defocus_error(fast["results"], plain["results"], specs),
            "stage_ms_per_step": {k: round(v, 3) for k, v in fast["stage"].items()},
            "contraction": {"stage_ms": {k: round(v, 3) for k, v in ft.items()}, "counts": fc,
                            "tensor_tflops": round(tflops, 1), "peak_tflops": bf16_peak,
                            "frac": round(tflops / bf16_peak, 4),
                            "fp32_candidates_fast": fast["search_counts"]["cand2d"],
                            "fp32_candidates_plain": plain["search_counts"]["cand2d"]},
            "e2e": {"value": round(world * n / (e2e_ms / 1000.0), 2), "unit": "micrographs/s",
                    "h2d_bytes_per_step": sum(4 * s.width * s.height for s in specs),
                    "d2h_bytes_per_step": n * 40, "ms_per_step": round(e2e_ms, 3),
                    "timing": "host clock around gcf_run_batch_mode (pinned host images)",
                    "stage_ms": {k: round(v, 3) for k, v in e2e_stage.items()},
                    "graph_launches": e2e_graph["graph_launches"],
                    "pcie_h2d_gbs": pcie,
                    "pcie_bound_ms": round(sum(4 * s.width * s.height for s in specs) / pcie / 1e6, 1)},
            "gpu_launches": fast["launches"],
            "cuda_graphs": {"graph_launches_per_step": fast["graph_launches_per_step"],
                            "graph_nodes": fast["graph"]["nodes"],
                            "library_kernels_in_graph": fast["graph"]["kernels"],
                            "note": "each timed step is one graph launch holding gpu_launches kernels of this "
                                    "library (plus cuFFT's lowpass kernels, and its rescale kernels when the "
                                    "rescale takes cuFFT) when graph_launches_per_step "
                                    "is 1"},
            "autotune": tuning,
            "roofline": tile_kernel_roofline(fast["stage"], dims, pk),
            "clocks": clocks}
    if not args.no_secondary:
        line["series_41x4096"] = series_figures(ctx, G, max(2, min(args.steps, 3)), 2, world, rank)
        ctx.set_rescale_impl(G.GCF_RESCALE_CUFFT)
        line["single_4096_1p0"] = single_1p0(ctx, G, max(2, min(args.steps, 5)))
        lines_ctx = G.Context(local, 512, 0)
        lines_ctx.set_rescale_impl(G.GCF_RESCALE_LINES)
        if fast_mode == G.GCF_SEARCH_LEARNED:
            G.load_learned(lines_ctx)
        line["stream_2000_plus_8x61"] = stream_figures(ctx, G, fast_mode, world, rank, lines_ctx=lines_ctx,
                                                       fast_rescale=fast_rescale)
        lines_ctx.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline([h.numpy() for h in host], specs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
