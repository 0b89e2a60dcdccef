"""The learned initialiser on the GPU: its BF16 forward/backward kernels
against the FP64 oracle (oracle/nn_oracle.py), training by the library's
own kernels, and the learned window search against the plain search.

Gradient check bars.  The library stores activations and gradients in
BF16 (8 significant bits) between layers and multiplies BF16 operands with
FP32 accumulation.  (1) Against the oracle that rounds to BF16 at the same
points (products and sums in FP64): per layer a relative L2 error <= 1e-2
and cosine similarity >= 0.9999 -- what remains is FP32 accumulation and
the rare ReLU input that lands on the other side of zero.  (2) Against the
plain FP64 oracle (BF16 weights, unrounded activations), the cost of the
BF16 storage itself: loss within 2e-2 relative, predictions within 2e-2 of
their spread, each layer's gradient within a relative L2 error of 0.15 and
cosine similarity >= 0.99.
"""
import numpy as np
import pytest

from oracle import nn_oracle as N

pytestmark = pytest.mark.gpu


def test_gradients_match_oracle(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    ctx.nn_init(11)
    op = G.make_optics()
    x1, x2, t, p = ctx.nn_synth_inputs(op, seed=5, first=0, n=4)
    assert np.all(np.isfinite(x1)) and np.all(np.isfinite(x2))
    # inputs are standardised over their non-empty cells
    assert abs(float(x1[x1 != 0].mean())) < 0.05 and 0.9 < float(x1[x1 != 0].std()) < 1.1
    params = ctx.nn_params()
    loss, grads, pred = ctx.nn_forward_backward(x1, x2, t)
    ctx.close()
    # the oracle sees the BF16-rounded inputs the library used
    for emulate, rel_bar, cos_bar in ((True, 1e-2, 0.9999), (False, 0.15, 0.99)):
        oloss, ograds, opred = N.forward_backward(params, N.bf16(x1), N.bf16(x2), t, emulate_bf16=emulate)
        assert abs(loss - oloss) <= 2e-2 * abs(oloss), (emulate, loss, oloss)
        assert np.abs(pred - opred).max() <= 2e-2 * (np.abs(opred).max() + 1e-3), (emulate, pred, opred)
        for k, ((gw, gb), (ow, ob)) in enumerate(zip(N.split(grads), N.split(ograds))):
            for a, b in ((gw, ow), (gb, ob)):
                a = a.ravel().astype(np.float64)
                b = b.ravel()
                nb = np.linalg.norm(b)
                if nb == 0:
                    assert np.linalg.norm(a) == 0
                    continue
                rel = np.linalg.norm(a - b) / nb
                cos = float(a @ b / (np.linalg.norm(a) * nb + 1e-300))
                assert rel <= rel_bar and cos >= cos_bar, (emulate, k, rel, cos)


def test_forward_through_the_persistent_product(gpu_lib):
    """40 samples: the first two convolutions have 1280 and 320 tiles of 128
    im2col rows, enough for the persistent tensor-core product (one CTA per
    SM); loss and predictions against the BF16-emulating oracle as in the
    gradient check."""
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    ctx.nn_init(13)
    op = G.make_optics()
    x1, x2, t, p = ctx.nn_synth_inputs(op, seed=9, first=0, n=40)
    params = ctx.nn_params()
    loss, grads, pred = ctx.nn_forward_backward(x1, x2, t)
    ctx.close()
    oloss, ograds, opred = N.forward_backward(params, N.bf16(x1), N.bf16(x2), t, emulate_bf16=True)
    assert abs(loss - oloss) <= 2e-2 * abs(oloss), (loss, oloss)
    assert np.abs(pred - opred).max() <= 2e-2 * (np.abs(opred).max() + 1e-3)
    for (gw, gb), (ow, ob) in zip(N.split(grads), N.split(ograds)):
        a, b = gw.ravel().astype(np.float64), ow.ravel()
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b)


@pytest.mark.parametrize("px", [1.2, 1.35, 1.5])
def test_network_inputs_match_oracle(gpu_lib, px):
    """The polar binning of a background-removed half spectrum (k_nn_input)
    against oracle/nn_oracle.py polar_inputs.  Both round the bin indices in
    float32, but the library's atan2f and fused multiply-adds may move a
    pixel that sits on a bin edge to the neighbouring bin: at most 0.5 % of
    the bins may differ by more than the BF16 rounding of the output
    (2^-7 relative + 0.02), and the empty bins must be the same up to 0.5 %."""
    from gctffind_b200 import synth
    G = gpu_lib
    spec = synth.MicrographSpec(width=2048, height=2048, pixel_size=px, df_min=17800.0, df_max=18300.0,
                                azimuth_deg=30.0, seed=5)
    img = synth.make_micrograph(spec).numpy()
    ctx = G.Context(0, 512, 0)
    ctx.setup(G.make_optics(pixel_size=px), 2048, 2048)
    ctx.gen_half_spectrum(img)
    half = ctx.half_spectrum(raw=False)
    x1, x2 = ctx.nn_inputs(half, px)
    ctx.close()
    o1, o2 = N.polar_inputs(half, px)
    for g, o in ((x1[0], o1), (x2[0], o2)):
        bad = np.abs(g - o) > 2.0 ** -7 * np.abs(o) + 0.02
        assert bad.mean() <= 5e-3, (px, int(bad.sum()), g.size)
        assert abs(int((g != 0).sum()) - int((o != 0).sum())) <= 5e-3 * g.size
    assert 0.9 < float(x2[0][x2[0] != 0].std()) < 1.1


def test_training_lowers_the_loss_and_weights_round_trip(gpu_lib, tmp_path):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    op = G.make_optics()
    ctx.nn_init(3)
    losses = ctx.nn_train(op, steps=200, batch=64, seed=77, first=0, lr=1e-3)
    assert np.all(np.isfinite(losses))
    first, last = float(losses[:20].mean()), float(losses[-20:].mean())
    assert last < 0.5 * first, (first, last)
    path = str(tmp_path / "w.bin")
    ctx.save_weights(path)
    w = ctx.nn_params()
    ctx2 = G.Context(0, 512, 0)
    ctx2.load_weights(path)
    assert np.array_equal(ctx2.nn_params(), w)
    ctx.close()
    ctx2.close()


def test_learned_search_needs_weights(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    img = np.zeros((1024, 1024), np.float32)
    with pytest.raises(G.GcfError):
        ctx.run_batch([img], [1.35], G.make_optics(), mode=G.GCF_SEARCH_LEARNED)
    ctx.close()


def test_trained_network_gain_on_held_out_spectra(gpu_lib):
    """The trained weights shipped with the package (written by
    `python -m gctffind_b200.train_init`) on 1024 held-out synthetic spectra
    (a generator seed never trained on), each searched three ways: the plain
    FP32 exhaustive search, the BF16 contraction search without the network
    and the learned window search.  Bar: the learned search lands within one
    search step of the plain one for >= 99 % of the spectra with a median
    |d defocus| <= 20 A, falls back to the full search for at most 3 % beyond
    the spectra whose CC is below the threshold anyway, and
    scores fewer than half the table candidates of the search without the
    network -- what the network gains."""
    from gctffind_b200 import train_init as TI
    G = gpu_lib
    assert G.learned_available(), "trained weights missing: run python -m gctffind_b200.train_init"
    ctx = G.Context(0, 512, 0)
    op = G.make_optics()
    G.load_learned(ctx)
    n = 1024
    plain, prm = ctx.nn_eval_synthetic(op, TI.EVAL_SEED, 0, n, G.GCF_SEARCH_PLAIN)
    bf16, _ = ctx.nn_eval_synthetic(op, TI.EVAL_SEED, 0, n, G.GCF_SEARCH_BF16)
    cb = ctx.fast_counts()
    assert ctx.fast_times()["network"] == 0.0
    learned, _ = ctx.nn_eval_synthetic(op, TI.EVAL_SEED, 0, n, G.GCF_SEARCH_LEARNED)
    cl = ctx.fast_counts()
    assert ctx.fast_times()["network"] > 0.0   # its inputs and layers, timed on the device
    ctx.close()
    med_b, frac_b, _ = TI.compare(bf16, plain)
    med_l, frac_l, _ = TI.compare(learned, plain)
    assert frac_b >= 0.99 and med_b <= 20.0, (frac_b, med_b)
    assert frac_l >= 0.99 and med_l <= 20.0, (frac_l, med_l)
    # fallbacks: the refined CC below the threshold (low-dose spectra, where
    # the full search finds no better) or an optimum at the window's edge
    low_cc = sum(r.score < 0.1 for r in bf16)
    assert cl["fallbacks"] <= low_cc + 0.03 * n, (cl, low_cc)
    assert cl["table_cand"] < 0.5 * cb["table_cand"], (cl, cb)
    # both stay as close to the generator's truth as the plain search
    assert TI.truth_error(learned, prm) <= TI.truth_error(plain, prm) + 20.0


def test_learned_threshold_sends_searches_to_the_full_search(gpu_lib):
    """gcf_set_learned_threshold: with the CC threshold at 1 every learned
    search falls back to the full contraction search, so the learned method
    returns the BF16 method's results; values outside [-1, 1] are rejected."""
    from gctffind_b200 import synth
    G = gpu_lib
    specs = [synth.MicrographSpec(width=1536, height=1536, pixel_size=1.3, df_min=12000.0 + 3000 * k,
                                  df_max=12400.0 + 3000 * k, azimuth_deg=20.0 * k, dose=2.0, seed=600 + k)
             for k in range(4)]
    imgs = [synth.make_micrograph(s, device="cuda") for s in specs]
    op = G.make_optics()
    ctx = G.Context(0, 512, 0)
    G.load_learned(ctx)
    bf16 = ctx.run_batch(imgs, [1.3] * 4, op, mode=G.GCF_SEARCH_BF16)
    ctx.set_learned_threshold(1.0)
    learned = ctx.run_batch(imgs, [1.3] * 4, op, mode=G.GCF_SEARCH_LEARNED)
    assert ctx.fast_counts()["fallbacks"] == 4
    assert [r.as_dict() for r in learned] == [r.as_dict() for r in bf16]
    with pytest.raises(G.GcfError):
        ctx.set_learned_threshold(1.5)
    ctx.close()


def test_set_params_round_trip_and_size_check(gpu_lib):
    G = gpu_lib
    ctx = G.Context(0, 512, 0)
    ctx.nn_init(5)
    p = ctx.nn_params() * 0.5
    ctx.nn_set_params(p)
    assert np.array_equal(ctx.nn_params(), p.astype(np.float32))
    with pytest.raises(G.GcfError):
        ctx.nn_set_params(p[:-1])
    ctx.close()
