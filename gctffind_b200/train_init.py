#!/usr/bin/env python
"""Trains the learned initialiser on the GPU and writes its weights.

    python -m gctffind_b200.train_init [--samples 1048576] [--batch 256]

Training data: `samples` synthetic (256-bin rotational profile, 256 x 256
polar half spectrum) pairs, visited `epochs` times, that the library itself
generates on the GPU
(gcf_nn_train): the expected averaged spectrum of the micrograph model --
white object, CTF with the parameter draw of the uneven batch (mean defocus
5000-40000 A, astigmatism 0-1000 A at a uniform angle, pixel size
0.8-1.5 A rescaled to >= 1.2 A, dose 0.5-2 e/A^2), B-factor envelope,
smooth background and shot noise -- background-removed and lowpassed by the
library's own post-processing.  The network, its forward and backward passes
and the Adam updates are the library's BF16 tensor-core kernels.

Evaluation on `eval` held-out samples (a different generator seed): each is
searched three ways -- the plain FP32 exhaustive search, the BF16 contraction
search without the network, and the learned window search -- and the summary
(defocus error against the plain search, the fraction within one search step,
the fallback rate and the table candidates each method scored) is written
beside the weights as JSON.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

TRAIN_SEED = 20240611     # generator seed of the training pairs
EVAL_SEED = 99173         # generator seed of the held-out pairs (never trained on)


def one_step(mean_a: float) -> float:
    """The plain search's last mean-defocus step: max(20 A, 0.105 * mean / 31)
    (the final mRefineDfMean pass, FindCTF/CFindDefocus2D.cpp:166-182, 296-300)."""
    return max(20.0, 0.105 * mean_a / 31.0)


def compare(fast, plain):
    """Median |d mean defocus| (A) and fraction within one search step of the
    plain search (both defocus extremes)."""
    d, within = [], []
    for f, p in zip(fast, plain):
        mf, mp = 0.5 * (f.df_min + f.df_max), 0.5 * (p.df_min + p.df_max)
        st = one_step(mp)
        d.append(abs(mf - mp))
        within.append(abs(f.df_min - p.df_min) <= st and abs(f.df_max - p.df_max) <= st)
    return float(np.median(d)), float(np.mean(within)), float(np.percentile(d, 99))


def truth_error(res, params):
    """Median |d mean defocus| (A) against the generator's parameters
    (params[:, 0] = mean defocus in A)."""
    return float(np.median([abs(0.5 * (r.df_min + r.df_max) - p[0]) for r, p in zip(res, params)]))


def evaluate(ctx, G, op, n, seed=EVAL_SEED, first=0):
    """Plain, BF16 and learned searches of n held-out synthetic spectra."""
    out = {}
    plain, prm = ctx.nn_eval_synthetic(op, seed, first, n, G.GCF_SEARCH_PLAIN)
    cplain = ctx.search_counts()
    bf16, _ = ctx.nn_eval_synthetic(op, seed, first, n, G.GCF_SEARCH_BF16)
    cb = ctx.fast_counts()
    learned, _ = ctx.nn_eval_synthetic(op, seed, first, n, G.GCF_SEARCH_LEARNED)
    cl = ctx.fast_counts()
    for name, res, cnt in (("bf16", bf16, cb), ("learned", learned, cl)):
        med, frac, p99 = compare(res, plain)
        out[name] = {"median_abs_ddf_vs_plain_A": round(med, 2), "p99_abs_ddf_vs_plain_A": round(p99, 2),
                     "frac_within_one_step_of_plain": round(frac, 5),
                     "median_abs_ddf_vs_truth_A": round(truth_error(res, prm), 2),
                     "table_candidates_per_micrograph": round(cnt["table_cand"] / n, 1),
                     "fp32_rescored_per_micrograph": round(cnt["rescored"] / n, 1),
                     "fallbacks": int(cnt["fallbacks"])}
    out["plain"] = {"median_abs_ddf_vs_truth_A": round(truth_error(plain, prm), 2),
                    "fp32_candidates_per_micrograph": round(cplain["cand2d"] / n, 1)}
    out["held_out"] = {"n": n, "seed": seed, "first": first}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--samples", type=int, default=1 << 20)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--epochs", type=int, default=4,
                    help="passes over the same samples; each pass decays from half the previous pass's rate")
    ap.add_argument("--init-seed", type=int, default=7)
    ap.add_argument("--eval", type=int, default=10000)
    ap.add_argument("--out", default=None, help="weights file (default: the package's weights/ctf_init.bin)")
    ap.add_argument("--gpu", type=int, default=0)
    a = ap.parse_args(argv)
    import gctffind_b200 as G
    out = a.out or G.WEIGHTS_PATH
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    ctx = G.Context(a.gpu, 512, 0)
    op = G.make_optics()
    ctx.nn_init(a.init_seed)
    steps = max(1, a.samples // a.batch)
    t0 = time.perf_counter()
    losses = np.concatenate([ctx.nn_train(op, steps=steps, batch=a.batch, seed=TRAIN_SEED, first=0,
                                          lr=a.lr * 0.5 ** e) for e in range(a.epochs)])
    train_s = time.perf_counter() - t0
    if not np.all(np.isfinite(losses)):
        raise RuntimeError("training diverged")
    ctx.save_weights(out)
    summary = {"training": {"pairs": steps * a.batch, "batch": a.batch, "epochs": a.epochs,
                            "steps": steps * a.epochs, "lr": a.lr,
                            "schedule": "Adam; per epoch a cosine decay to 5 % of that epoch's rate, "
                                        "the rate halved from epoch to epoch", "generator_seed": TRAIN_SEED,
                            "init_seed": a.init_seed, "seconds": round(train_s, 2),
                            "loss_first_100": round(float(losses[:100].mean()), 5),
                            "loss_last_100": round(float(losses[-100:].mean()), 5)}}
    if a.eval > 0:
        t0 = time.perf_counter()
        summary["evaluation"] = evaluate(ctx, G, op, a.eval)
        summary["evaluation"]["seconds"] = round(time.perf_counter() - t0, 2)
    ctx.close()
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary))
    return 0


if __name__ == "__main__":
    sys.exit(main())
