"""The learned block-match proposals, on the GPU.

1. The network's gradients from the library's CUDA backward kernels equal the
   FP64 oracle's (oracle/mlp_fp64.py, itself checked by finite differences)
   within 2e-2 of the largest gradient (the products use BF16 weights and
   accumulate in FP32; the oracle uses the same BF16 weights in float64).
2. Training with the CUDA kernels lowers the loss on a learnable task.
3. The learned form at a 33 x 33 x 5 window (bm_range 16, radius 2): trained
   on other clips' full-search targets, it is run three ways on a held-out
   clip.  With the recall threshold above 1 every tile falls back to the full
   search and the output equals the plain form's bit for bit.  With 0 the
   learned rows always stand.  With the default 0.9 the per-tile check
   decides.  The test states what the network gains: the share of tiles
   whose learned rows stand, the shortlist recall, and the PSNR each way.
"""
import numpy as np
import pytest

import learned as LR
import mlp_fp64 as M
import synth
import vnlbgpu_lib as lib

pytestmark = pytest.mark.gpu


def test_gradients_match_the_fp64_oracle():
    import torch

    shape = (12, 16, 3, 40)
    net = lib.MLP(*shape, max_batch=64, seed=1)
    rng = np.random.default_rng(2)
    x = rng.normal(0.0, 1.0, (32, shape[0])).astype(np.float32)
    t = rng.integers(-1, shape[3], (32, 3)).astype(np.int32)
    t[:, 0] = np.abs(t[:, 0])
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    torch.cuda.synchronize()
    grads, loss = net.gradients(dx.data_ptr(), dt.data_ptr(), 32, 3)
    want_loss, want = M.loss_and_gradients(net.get_weights(), shape, x, t)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    err = np.abs(grads - want).max() / np.abs(want).max()
    print(f"gradient max error / max gradient {err:.2e}")
    assert err <= 2e-2


def test_tensor_core_output_layer_and_radix_shortlist():
    """The shortlist path (vnlbgpu_mlp_shortlist, as the learned form runs
    it): the output layer on the tensor cores (tcgen05, BF16 activations and
    weights, FP32 accumulation) at the 33 x 33 x 5 window's shape (5445 offsets, hidden
    128), a batch that is no multiple of the 128-row tile and outputs that
    are no multiple of the 256-column tile, then the top 64 by radix select.
    Against the FP64 oracle of the same arithmetic (activations rounded to
    BF16 before the output layer) the shortlists share at least 98% of their
    ids (the hidden layers' FP32 sums can move an activation across a BF16
    rounding boundary, which reorders near-ties at the 64th place)."""
    import torch

    shape = (45, 128, 3, 5445)
    net = lib.MLP(*shape, max_batch=512, seed=11)
    rng = np.random.default_rng(12)
    x = rng.normal(0.0, 1.0, (300, shape[0])).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    out = torch.empty((300, 64), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    net.shortlist(dx.data_ptr(), 300, 64, out.data_ptr())
    got = out.cpu().numpy()
    z = M.forward_logits(net.get_weights(), shape, x, bf16_last_input=True)
    want = np.argsort(-z, axis=1, kind="stable")[:, :64]
    assert got.min() >= 0 and got.max() < shape[3]
    assert all(len(set(r.tolist())) == 64 for r in got)  # 64 distinct ids per row
    overlap = np.mean([len(set(g.tolist()) & set(w.tolist())) / 64.0 for g, w in zip(got, want)])
    print(f"shortlist overlap with the FP64 oracle {overlap:.4f}")
    assert overlap >= 0.98


def test_training_lowers_the_loss():
    rng = np.random.default_rng(4)
    n, inputs, outputs = 4096, 20, 50
    x = rng.normal(0.0, 1.0, (n, inputs)).astype(np.float32)
    proj = rng.normal(0.0, 1.0, (inputs, outputs))
    scores = x @ proj
    order = np.argsort(-scores, axis=1)
    t = order[:, :2].astype(np.int32)  # the two best classes of a linear map
    net = lib.MLP(inputs, 64, 2, outputs, max_batch=512, seed=5)
    losses = LR.train(net, x, t, steps=400, batch=512, lr=3e-3)
    first, last = np.mean(losses[:10]), np.mean(losses[-10:])
    print(f"loss {first:.3f} -> {last:.3f}")
    assert last < 0.6 * first


@pytest.mark.timeout(900)
def test_learned_form_on_a_33x33x5_window():
    kw = dict(block_size=8, block_step=8, group_size=8, bm_range=16, radius=2, patch_time=1, rank=8, cap_factor=4.0,
              variance_threshold=1.1, weight_alpha=0.75, weight_beta=0.35, weight_gamma=1.0)
    w, h, frames, planes, sigma = 160, 128, 7, 3, 20.0
    train_clips = LR.synthetic_clips(w, h, frames, planes, sigma, seeds=(101, 102, 103))
    clean, noisy = synth.make_clip(w, h, frames, planes, sigma, seed=104)
    inputs, outputs = LR.network_shape(lib.STAGE_BASIC, planes, kw, noisy, sigma)
    assert (inputs, outputs) == (5 * 1 * 9, 5 * 33 * 33)
    feats, targets = LR.training_pairs(lib.STAGE_BASIC, train_clips, sigma, kw)
    net = lib.MLP(inputs, 128, 3, outputs, max_batch=4096, seed=6)
    losses = LR.train(net, feats, targets, steps=300, batch=1024, lr=1e-3)
    hold_f, hold_t = LR.training_pairs(lib.STAGE_BASIC, [noisy], sigma, kw)
    rec = LR.recall(net, hold_f, hold_t, 64)

    plain = LR.session(lib.STAGE_BASIC, noisy, sigma, kw).render_clip()
    results = {}
    for threshold in (1.5, 0.0, 0.9):
        s = LR.session(lib.STAGE_BASIC, noisy, sigma, kw, form="learned")
        s.set_learned(net, shortlist=64, recall_threshold=threshold, tile=64)
        out = s.render_clip()
        st = s.stats()
        s.close()
        results[threshold] = (out, st)
    print(f"loss {np.mean(losses[:10]):.3f} -> {np.mean(losses[-10:]):.3f}; held-out recall@64 {rec:.3f}")
    for threshold, (out, st) in results.items():
        kept = 1.0 - st["learned_fallback_tiles"] / max(1, st["learned_tiles"])
        print(f"threshold {threshold}: tiles {st['learned_tiles']}, learned rows kept in {kept:.1%}; "
              f"PSNR {synth.psnr(out, clean):.4f} dB (plain {synth.psnr(plain, clean):.4f})")
        assert np.isfinite(out).all()
    # a shortlisted candidate gets the full search's distance bits: the rows
    # both matchers keep have equal distances
    s = LR.session(lib.STAGE_BASIC, noisy, sigma, kw, form="learned")
    s.set_learned(net, shortlist=64, recall_threshold=0.0, tile=64)
    learned_rows = s.diag_anchor(2)
    s.close()
    s = LR.session(lib.STAGE_BASIC, noisy, sigma, kw)
    plain_rows = s.diag_anchor(2)
    s.close()
    place = lambda r: (int(r["x"]), int(r["y"]), int(r["frame"]))
    common = 0
    for gi in range(len(plain_rows["counts"])):
        a = plain_rows["grid_rows"][gi][: plain_rows["counts"][gi]]
        b = learned_rows["grid_rows"][gi][: learned_rows["counts"][gi]]
        ka = {place(x): np.float32(x["distance"]).view(np.uint32) for x in a}
        kb = {place(x): np.float32(x["distance"]).view(np.uint32) for x in b}
        for pos in set(ka) & set(kb):
            assert ka[pos] == kb[pos], (gi, pos)
            common += 1
    assert common > len(plain_rows["counts"])  # more than the anchors themselves
    full, st = results[1.5]
    assert st["learned_fallback_tiles"] == st["learned_tiles"] > 0
    assert np.array_equal(full.view(np.uint32), plain.view(np.uint32))
    assert results[0.0][1]["learned_fallback_tiles"] == 0
    # learned rows are a subset search: never better matches than the full one,
    # so the quality can only drop, and by a bounded amount at this noise
    assert synth.psnr(results[0.0][0], clean) >= synth.psnr(plain, clean) - 1.0
