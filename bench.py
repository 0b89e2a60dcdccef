#!/usr/bin/env python
"""Benchmark of the CTF-estimation hot path on B200.

Workload (one "step"): a synthetic tilt series of 41 micrographs, 4096 x 4096
float32 at 1.35 A/px (-60..+60 degrees in 3-degree steps, 3 e/A^2 per tilt,
defocus 30000 A at 0 degrees with a per-column gradient set by the tilt,
astigmatism uniform in 0-800 A at a random angle), processed with the
reference's series policy (CFindSeriesCtfs: zero tilt full search, every
other tilt refined around the best-scoring earlier one) through the C ABI
call gcf_run_series.

  value : micrographs/s with the series already resident in HBM
          (device pointers), device time from CUDA events on the library stream
  e2e   : the same call with pinned HOST buffers; the host->device copy of
          the 41 images and the device->host read of the results are inside
          the timed region

Rank r of N processes its own series (seeded by r): weak scaling, replicas
only, no data-path collective.  `--impl reference` times the reference's own
CUDA implementation of the path, built from its sources, on the same GPU
(the FP64 host oracle when that build is absent).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TILTS = 41
SIZE = 4096
PX = 1.35
METRIC = "4096^2 micrographs/s (tilt series, plain FP32 search)"
# DRAM bytes (read + write) of one micrograph's share of k_fused_spectrum,
# from ncu dram__bytes_read.sum + dram__bytes_write.sum on a 3-micrograph
# launch of the same kernel divided by 3 (profiles/k_fused_spectrum_3x4096.md)
TILE_KERNEL_TRAFFIC_PER_MICROGRAPH = (262_052_608 + 11_340_544) // 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--spectrum", default="auto", choices=["auto", "fused", "cufft"])
    ap.add_argument("--n-tilts", type=int, default=N_TILTS)
    ap.add_argument("--size", type=int, default=SIZE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--trace", default=None,
                    help="after the timed steps, record one device-resident step with the CUDA "
                         "activity tracer (torch.profiler) and write a Chrome trace here")
    return ap.parse_args()


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        import torch
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


def make_series(rank, n_tilts, size, device):
    import torch
    from gctffind_b200 import synth
    specs = synth.tilt_series_specs(n_tilts=n_tilts, step_deg=3.0, size=size, pixel_size=PX,
                                    dose=3.0, df0=30000.0, seed=1 + rank)
    imgs = [synth.make_micrograph(s, device=device) for s in specs]
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    return specs, imgs


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "_fallback": True}


def cpu_baseline(imgs_host, order, budget_s=25.0):
    """FP64 OpenMP oracle on the host cores: the zero-tilt full search plus
    refinements of the next tilts in processing order, as many as fit the
    time budget (at least one)."""
    from oracle import oracle as O
    O.build()
    cores = O.num_threads(os.cpu_count() or 1)
    p = O.params(pixel_size=PX, tile_size=512)
    t0 = time.perf_counter()
    z = order[0]
    r0 = O.find_ctf_image(imgs_host[z], PX, p, mode=0)
    done = 1
    for idx in order[1:]:
        if time.perf_counter() - t0 > budget_s:
            break
        dmin, dmax = r0.df_min, r0.df_max
        mean = 0.5 * (dmin + dmax)
        rin = [mean, max(mean * 0.5, 5000.0 * PX * PX), (dmax - dmin) * 0.5 / mean, 0.0,
               r0.azimuth, 0.0, r0.ext_phase, 0.0]
        O.find_ctf_image(imgs_host[idx], PX, p, mode=1, refine_in=rin)
        done += 1
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "micrographs/s", "cores": cores, "kind": "port",
            "sample": f"{done} of the series' 4096^2 micrographs (zero-tilt full search + "
                      f"{done - 1} refinements), FP64 oracle, {cores} OpenMP threads, {dt:.1f} s"}


def _reference_cuda_step(host, order, tilts, sample_refines):
    """One step of the reference arm on the reference's own CUDA build:
    the zero-tilt full search alone, then the zero tilt plus
    `sample_refines` packages spread evenly over the rest of the processing
    order (high tilts refine at a different cost than low ones).  Returns
    (seconds of the full search, mean seconds of one refined package)."""
    from oracle import refimpl
    rest = order[1:]
    stride = max(1, len(rest) // max(1, sample_refines))
    sub = [order[0]] + rest[stride - 1::stride][:sample_refines]
    imgs = [host[i] for i in sub]
    t = [tilts[i] for i in sub]
    _, _, t_full = refimpl.run_series(imgs[:1], PX, [0], tilts=t[:1], tile=512)
    _, _, t_sub = refimpl.run_series(imgs, PX, list(range(len(imgs))), tilts=t, tile=512)
    return t_full, max(t_sub - t_full, 0.0) / max(1, len(sub) - 1)


def run_reference(args, rank, world):
    """--impl reference: the reference implementation of the path on this
    box.  GCtfFind has no CPU path: its own CUDA code, built from its
    sources (oracle/_ref/libgcfref.so), runs on the same B200 when present;
    otherwise the FP64 oracle port times the host cores."""
    if rank != 0:
        return 0
    import torch
    from gctffind_b200 import synth
    from gctffind_b200.api import series_order
    from oracle import refimpl
    on_gpu = torch.cuda.is_available()
    specs, imgs = make_series(0, args.n_tilts, args.size, "cuda" if on_gpu else "cpu")
    host = [im.cpu().numpy() for im in imgs]
    del imgs
    if on_gpu:
        torch.cuda.empty_cache()
    tilts = synth.tilt_angles(args.n_tilts, 3.0)
    order = series_order(tilts).order
    n = args.n_tilts
    workload = (f"tilt series {n} x {args.size}^2 float32 @ {PX} A/px, CFindSeriesCtfs policy "
                "(zero tilt full, rest refined)")
    if on_gpu and refimpl.available():
        k_ref = min(8, n - 1)
        fulls, refs = [], []
        for k in range(args.warmup + args.steps):
            tf, tr = _reference_cuda_step(host, order, tilts, k_ref)
            if k >= args.warmup:
                fulls.append(tf)
                refs.append(tr)
        t_full, t_ref = statistics.median(fulls), statistics.median(refs)
        t_series = t_full + (n - 1) * t_ref
        v = n / t_series
        sample = (f"reference CUDA build on the B200 (GCtfFind has no CPU path): per step the "
                  f"zero-tilt full search ({t_full:.2f} s) and {k_ref} refined tilts spread over "
                  f"the processing order "
                  f"({t_ref:.2f} s each, medians over {args.steps} steps); value = {n} / "
                  f"(full + {n - 1} x refine) = {t_series:.1f} s per series")
        line = {"metric": METRIC, "value": round(v, 4), "unit": "micrographs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 * t_series, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": workload, "tile": 512, "l2": "inputs larger than L2",
                           "timing": "host wall clock around CFindSeriesCtfs::DoIt (it blocks on "
                                     "every candidate), images in host memory"},
                "cpu_baseline": {"value": round(v, 4), "unit": "micrographs/s", "cores": 1,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": round(v, 4), "unit": "micrographs/s",
                        "h2d_bytes_per_step": n * args.size * args.size * 4,
                        "d2h_bytes_per_step": n * (512 * 512 * 4 + 20)}}
        print(json.dumps(line), flush=True)
        return 0
    vals = []
    cb = None
    for k in range(max(1, args.warmup) + max(1, args.steps)):
        cb = cpu_baseline(host, order, budget_s=8.0)
        if k >= max(1, args.warmup):
            vals.append(cb["value"])
        if len(vals) >= args.steps:
            break
    v = statistics.median(vals)
    cb["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "micrographs/s", "n_gpus": world,
            "steps": len(vals), "warmup": args.warmup, "ms_per_step": 1000.0 * n / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload + " (sampled: zero-tilt full search + refinements)",
                       "l2": "inputs larger than L2",
                       "note": "reference CUDA build unavailable here: FP64 oracle port on the host"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "micrographs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    import numpy as np
    import torch
    import gctffind_b200 as G
    from gctffind_b200 import synth
    torch.cuda.set_device(local)
    specs, imgs = make_series(rank, args.n_tilts, args.size, f"cuda:{local}")
    order = G.series_order(synth.tilt_angles(args.n_tilts, 3.0)).order
    ctx = G.Context(local, 512, 0)
    if args.spectrum == "cufft":
        ctx.set_spectrum_impl(G.GCF_SPECT_CUFFT)
    elif args.spectrum == "fused":
        ctx.set_spectrum_impl(G.GCF_SPECT_FUSED)
    else:
        try:
            ctx.set_spectrum_impl(G.GCF_SPECT_FUSED)
        except G.GcfError:
            ctx.set_spectrum_impl(G.GCF_SPECT_CUFFT)
    op = G.make_optics(pixel_size=PX)

    # ---- device-resident inputs -------------------------------------------------
    # clocks are sampled from the warm-up on through the end-to-end steps, so
    # the short device-resident region gets samples on both sides as well
    clk = ClockSampler(local)
    clk.start()
    for _ in range(args.warmup):
        ctx.run_series(imgs, op, order, is_tomo=True)
    barrier(world)
    torch.cuda.synchronize()
    dev_ms, stage = 0.0, {}
    launches = 0
    results = None
    torch.cuda.nvtx.range_push("device_steps")   # lets ncu --nvtx-include select the timed launches
    counts = None
    for _ in range(args.steps):
        results = ctx.run_series(imgs, op, order, is_tomo=True)
        counts = ctx.search_counts()
        st = ctx.stage_times()
        dev_ms += st["total"]
        for k, v in st.items():
            stage[k] = stage.get(k, 0.0) + v
        launches += ctx.launch_count()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(world)
    t_step = max_over_ranks(dev_ms / args.steps, world)
    value = world * args.n_tilts / (t_step / 1000.0)

    # ---- end to end: pinned host inputs, H2D + results D2H inside the timed region ----
    host = [im.cpu().pin_memory() for im in imgs]
    for _ in range(max(1, min(args.warmup, 2))):
        ctx.run_series(host, op, order, is_tomo=True)
    barrier(world)
    e2e_ms = 0.0
    torch.cuda.nvtx.range_push("e2e_steps")
    for _ in range(args.steps):
        ctx.run_series(host, op, order, is_tomo=True)
        e2e_ms += ctx.stage_times()["total"]
    torch.cuda.nvtx.range_pop()
    clocks = clk.stop()
    barrier(world)
    t_e2e = max_over_ranks(e2e_ms / args.steps, world)
    e2e = world * args.n_tilts / (t_e2e / 1000.0)
    h2d = sum(int(im.numel()) * 4 for im in imgs)
    d2h = args.n_tilts * 40

    if args.trace and rank == 0:
        # kernel start/end times on every stream, recorded without serialising
        # the launches (unlike ncu): shows how the searches overlap the tiles
        from torch.profiler import profile, ProfilerActivity
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            ctx.run_series(imgs, op, order, is_tomo=True)
            torch.cuda.synchronize()
        prof.export_chrome_trace(args.trace)

    # ---- roofline of the dominant kernel: the fused tile-spectrum kernel.
    # In a series step its launches share the GPU with the searches, so it is
    # timed alone here: a batch call makes one launch over all micrographs of
    # the series and runs the searches only after it ----
    pk = peaks()
    pxs = [PX] * args.n_tilts
    ctx.run_batch(imgs, pxs, op)
    kt = []
    st2d = []
    torch.cuda.nvtx.range_push("tile_kernel_alone")   # ncu --nvtx-include selects these launches
    for _ in range(max(1, min(args.steps, 3))):
        ctx.run_batch(imgs, pxs, op)
        bt = ctx.stage_times()
        kt.append(bt["tile_kernel"])
        st2d.append(bt["search2d"])
    torch.cuda.nvtx.range_pop()
    kern_ms = statistics.median(kt)
    bcounts = ctx.search_counts()
    T = 512
    ov = T // 2
    nt1 = ((args.size - ov) // (T - ov)) ** 2            # tiles per micrograph
    nch = -(-nt1 // 24)                                   # work items per micrograph (<= 24 tiles)
    img_bytes = args.n_tilts * 4 * args.size * args.size  # every pixel read once
    part_bytes = args.n_tilts * nch * (T // 2 + 1) * T * 4  # per-item partial spectra written
    algo_bytes = img_bytes + part_bytes
    # real 2D FFT of a T x T tile: 2.5 T^2 log2(T^2) flops, plus mean removal,
    # taper, |F| and accumulation (~6 flops per pixel)
    tile_flops = 2.5 * T * T * 2 * 9 + 6 * T * T
    algo_flops = args.n_tilts * nt1 * tile_flops
    sec = kern_ms / 1000.0
    achieved = algo_bytes / sec / 1e9 if sec > 0 else 0.0
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12          # nominal FP32 FMA rate at max clock
    roof = {"kernel": "k_fused_spectrum (8-CTA clusters) + k_fused_spectrum_solo (the SMs the clusters leave "
                      "free): one launch pair over all tiles of the series, timed alone",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": pk.get("hbm_gbs"),
            "unit": "GB/s", "frac": round(achieved / pk.get("hbm_gbs", 6650.0), 4),
            "traffic": TILE_KERNEL_TRAFFIC_PER_MICROGRAPH * args.n_tilts if TILE_KERNEL_TRAFFIC_PER_MICROGRAPH else None,
            "peak_source": "fallback" if pk.get("_fallback") else "measured",
            "algorithmic_bytes_per_launch": algo_bytes, "launch_ms": round(kern_ms, 3),
            "compute": {"flops_per_launch": algo_flops,
                        "achieved_tflops": round(algo_flops / sec / 1e12, 2) if sec > 0 else 0.0,
                        "fp32_peak_tflops": round(fp32_peak, 1), "peak_source": "nominal FP32 FMA",
                        "frac": round(algo_flops / sec / 1e12 / fp32_peak, 4) if sec > 0 else 0.0}}

    # ---- the candidate contraction: 2 flops (model x spectrum multiply-add)
    # per (candidate, in-band pixel) pair, counted on the device; its rate is
    # taken on the batch call, whose 2D searches (41 full Do2D) run alone ----
    s2d_ms = statistics.median(st2d)
    bflops = 2 * bcounts["pairs2d"]
    search = {"per_step": dict(counts, flops=2 * (counts["pairs2d"] + counts["pairs1d"])),
              "batch_full_search": {"cand2d": bcounts["cand2d"], "flops_2d": bflops,
                                    "ms_2d_stage": round(s2d_ms, 3),
                                    "achieved_tflops": round(bflops / (s2d_ms * 1e-3) / 1e12, 2) if s2d_ms > 0 else 0.0,
                                    "fp32_peak_tflops": round(fp32_peak, 1),
                                    "frac": round(bflops / (s2d_ms * 1e-3) / 1e12 / fp32_peak, 4) if s2d_ms > 0 else 0.0,
                                    "note": f"{args.n_tilts} full searches (Do2D) after one tile launch"}}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "micrographs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"tilt series {args.n_tilts} x {args.size}^2 float32 @ {PX} A/px, "
                                   "3 e/A^2, df 30000 A + tilt gradient, astig 0-800 A; "
                                   "CFindSeriesCtfs policy (zero tilt full, rest refined)",
                       "tile": 512, "spectrum": ["fused", "cufft"][0 if args.spectrum == "fused" else 1]
                       if args.spectrum != "auto" else "auto",
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (2.75 GB per step)"},
            "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in stage.items()},
            "e2e": {"value": round(e2e, 2), "unit": "micrographs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(t_e2e, 3)},
            "gpu_launches": launches,
            "roofline": roof,
            "search": search,
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        host_np = [h.numpy() for h in host]
        line["cpu_baseline"] = cpu_baseline(host_np, order)
    if rank == 0:
        r0 = results[order[0]]
        line["sample_result"] = {"zero_tilt": {"df_min": round(r0.df_min, 1), "df_max": round(r0.df_max, 1),
                                               "azimuth": round(r0.azimuth, 2), "score": round(r0.score, 4)},
                                 "truth": {"df_min": round(specs[order[0]].df_min, 1),
                                           "df_max": round(specs[order[0]].df_max, 1),
                                           "azimuth": round(specs[order[0]].azimuth_deg, 2)}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
