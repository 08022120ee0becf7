"""GPU: the corrector's tensor-core convolutions against plain PyTorch FP32
references of the same ops (BF16-rounded inputs, FP32 accumulation), and
its training loop end to end (loss goes down; the untrained corrector is
the bilinear interpolation)."""
import ctypes as C

import numpy as np
import pytest

import tsuner_b200 as T
from tsuner_b200 import corrector as K

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = torch.nn.functional


def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def bf16(x):
    return x.to(torch.bfloat16)


def nhwc(x):  # [n][c][h][w] -> [n][h][w][c] contiguous
    return x.permute(0, 2, 3, 1).contiguous()


def wk_from_torch(w):  # torch [cout][cin][3][3] -> [cout][tap][cin]
    return w.permute(0, 2, 3, 1).reshape(32, 9, 32).contiguous()


def ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def conv(X, Wk, bias=None, relu=0, gate=None, out_fp32=True):
    n, h, w, _ = X.shape
    Yf = torch.zeros((n, h, w, 32), device=X.device, dtype=torch.float32) if out_fp32 else None
    Yb = None if out_fp32 else torch.zeros((n, h, w, 32), device=X.device, dtype=torch.bfloat16)
    rc = T.lib().tsu_corr_conv3x3(ptr(X), n, h, w, ptr(Wk), ptr(bias), relu, ptr(gate), ptr(Yb), ptr(Yf), None)
    assert rc == 0, T.lib().tsu_corr_last_error()
    assert T.lib().tsu_corr_status() == 0
    return Yf if out_fp32 else Yb


def rand_case(n, h, w, seed):
    g = torch.Generator().manual_seed(seed)
    X = bf16(torch.randn(n, 32, h, w, generator=g))
    Wt = bf16(torch.randn(32, 32, 3, 3, generator=g) * 0.1)
    b = torch.randn(32, generator=g) * 0.1
    return X, Wt, b


@pytest.mark.parametrize("shape", [(1, 16, 8), (2, 37, 29), (1, 130, 67)])
def test_conv_forward_fp32_out(shape):
    d = dev()
    n, h, w = shape
    X, Wt, b = rand_case(n, h, w, 1)
    ref = F.conv2d(X.float().to(d), Wt.float().to(d), b.to(d), padding=1)
    Y = conv(nhwc(X).to(d), wk_from_torch(Wt).to(d), b.to(d), relu=0)
    err = (Y - nhwc(ref)).abs().max().item()
    assert err <= 1e-4 * max(1.0, ref.abs().max().item()), err


@pytest.mark.parametrize("shape", [(2, 40, 24), (1, 37, 29), (3, 16, 8), (1, 130, 67)])
def test_conv_forward_relu_bf16_out_and_gate(shape):
    """BF16 output goes through the staged, row-coalesced epilogue; ragged
    widths and heights leave partial tile rows and partial warps."""
    d = dev()
    n, h, w = shape
    X, Wt, b = rand_case(n, h, w, 2)
    G = bf16(torch.randn(n, h, w, 32)).to(d)
    ref = torch.relu(F.conv2d(X.float().to(d), Wt.float().to(d), b.to(d), padding=1))
    ref = nhwc(ref) * (G.float() > 0)
    Y = conv(nhwc(X).to(d), wk_from_torch(Wt).to(d), b.to(d), relu=1, gate=G, out_fp32=False)
    # one BF16 rounding of the FP32 result
    err = (Y.float() - ref).abs()
    assert (err <= 2.0 ** -8 * ref.abs() + 1e-6).all(), err.max().item()
    assert bool(((ref == 0) == (Y.float() == 0)).all())


@pytest.mark.parametrize("shape", [(1, 37, 29), (2, 64, 64)])
def test_conv_forward_bf16_out_no_gate(shape):
    d = dev()
    n, h, w = shape
    X, Wt, b = rand_case(n, h, w, 6)
    ref = nhwc(F.conv2d(X.float().to(d), Wt.float().to(d), b.to(d), padding=1))
    Y = conv(nhwc(X).to(d), wk_from_torch(Wt).to(d), b.to(d), relu=0, out_fp32=False)
    err = (Y.float() - ref).abs()
    assert (err <= 2.0 ** -8 * ref.abs() + 1e-6).all(), err.max().item()


def test_conv_input_gradient_with_flipped_weights():
    """dX = conv(dZ, Wt[cin][8 - tap][cout] = W[cout][tap][cin]) is the input
    gradient of the forward convolution."""
    d = dev()
    X, Wt, _ = rand_case(1, 33, 20, 3)
    dZ = bf16(torch.randn(1, 32, 33, 20) * 0.5)
    ref = torch.nn.grad.conv2d_input(X.shape, Wt.float().to(d), dZ.float().to(d), padding=1)
    wk = wk_from_torch(Wt)  # [cout][tap][cin]
    flip = wk.flip(1).permute(2, 1, 0).contiguous()  # [cin][tap'][cout], tap' = 8 - tap
    Y = conv(nhwc(dZ).to(d), flip.to(d), None, relu=0)
    err = (Y - nhwc(ref)).abs().max().item()
    assert err <= 1e-4 * max(1.0, ref.abs().max().item()), err


@pytest.mark.parametrize("shape", [(1, 16, 8), (3, 45, 27)])
def test_conv_weight_and_bias_gradient(shape):
    d = dev()
    n, h, w = shape
    X, Wt, _ = rand_case(n, h, w, 4)
    dZ = bf16(torch.randn(n, 32, h, w) * 0.5)
    ref_w = torch.nn.grad.conv2d_weight(X.float().to(d), Wt.shape, dZ.float().to(d), padding=1)
    ref_b = dZ.float().sum(dim=(0, 2, 3)).to(d)
    dW = torch.zeros(32, 9, 32, device=d)
    db = torch.zeros(32, device=d)
    Xd, Zd = nhwc(X).to(d), nhwc(dZ).to(d)  # keep both alive across the call
    rc = T.lib().tsu_corr_conv3x3_wgrad(ptr(Xd), ptr(Zd), n, h, w, ptr(dW), ptr(db), None)
    assert rc == 0
    assert T.lib().tsu_corr_status() == 0
    scale = max(1.0, ref_w.abs().max().item())
    err = (dW - wk_from_torch(ref_w)).abs().max().item()
    assert err <= 1e-4 * scale, err
    assert (db - ref_b).abs().max().item() <= 1e-4 * max(1.0, ref_b.abs().max().item())


def synthetic_samples(n, ny, f, seed):
    """Coarse maps and fine targets with a learnable relation: fine maximum
    depth = interpolated coarse + sub-grid bathymetry detail where wet."""
    rng = np.random.default_rng(seed)
    Hf = (20.0 + 5.0 * np.sin(np.arange(ny) / 3.0)[None, :] + rng.normal(0, 1.0, (ny, ny))).astype(np.float32)
    Hc = K.block_mean(Hf, f).astype(np.float32)
    coarse, fine = [], []
    for _ in range(n):
        a = rng.uniform(0.5, 2.0)
        hc = (Hc + a).astype(np.float32)
        dbc = np.full_like(Hc, 0.01 * a)
        coarse.append(np.stack([hc, dbc, Hc]))
        fine.append(np.stack([Hf + a, np.full_like(Hf, 0.01 * a)]).astype(np.float32))
    return Hf, np.stack(coarse), np.stack(fine)


def test_untrained_corrector_is_interpolation_and_training_lowers_loss():
    dev()
    ny, f = 64, 4
    Hf, coarse, fine = synthetic_samples(12, ny, f, 5)
    c = K.Corrector(ny, ny, f, max_batch=4, seed=3)
    try:
        c.set_site(Hf)
        c.add_samples(coarse, fine)
        oh, ob, bh, bb = c.predict(0, 2)
        assert np.array_equal(oh, bh) and np.array_equal(ob, bb)  # zero last layer
        loss = c.train(ntrain=12, iters=150, batch=4, lr=2e-3, seed=1)
        assert np.isfinite(loss).all()
        assert loss[-10:].mean() < 0.5 * loss[:5].mean(), (loss[:5], loss[-10:])
        oh2, _, _, _ = c.predict(0, 2)
        before = np.sqrt(((bh - fine[:2, 0]) ** 2).mean())
        after = np.sqrt(((oh2 - fine[:2, 0]) ** 2).mean())
        assert after < before, (before, after)
        Wt, B = c.weights()
        assert np.isfinite(Wt).all() and np.abs(Wt[-1]).max() > 0
    finally:
        c.close()


def test_options_weight_large_residuals_and_clip_depth():
    dev()
    ny, f = 64, 4
    Hf, coarse, fine = synthetic_samples(8, ny, f, 7)
    first = []
    for wbig in (0.0, 4.0):
        c = K.Corrector(ny, ny, f, max_batch=4, seed=3)
        try:
            c.set_site(Hf)
            c.set_options(wbig, False)
            c.add_samples(coarse, fine)
            loss = c.train(ntrain=8, iters=40, batch=4, lr=2e-3, seed=1)
            assert np.isfinite(loss).all() and loss[-5:].mean() < loss[:3].mean()
            first.append(float(loss[0]))
            oh, _, _, _ = c.predict(0, 8)
            c.set_options(wbig, True)
            ohc, _, _, _ = c.predict(0, 8)
            assert (ohc >= 0).all()
            assert np.array_equal(ohc, np.maximum(oh, 0.0))
        finally:
            c.close()
    # same weights and batch at the first step: the weighted loss is larger
    assert first[1] > first[0], first


def test_envelope_clamps_residuals_to_the_training_envelope():
    """envelope k: each predicted residual lies within k times the largest
    residual the training targets hold at that pixel (here computed on the
    host from the same targets)."""
    dev()
    ny, f = 64, 4
    Hf, coarse, fine = synthetic_samples(8, ny, f, 8)
    c = K.Corrector(ny, ny, f, max_batch=4, seed=5)
    try:
        c.set_site(Hf)
        c.add_samples(coarse, fine)
        c.train(ntrain=6, iters=60, batch=4, lr=3e-3, seed=2)
        oh, ob, bh, bb = c.predict(6, 2)
        _, _, th, tb = c.predict(0, 6)   # the interpolation of the training samples
        env_h = np.abs(fine[:6, 0] - th).max(axis=0)
        env_b = np.abs(fine[:6, 1] - tb).max(axis=0)
        for k in (0.5, 1.0):
            c.set_options(0.0, False, k)
            ch, cb, bh2, bb2 = c.predict(6, 2)
            assert np.array_equal(bh2, bh) and np.array_equal(bb2, bb)
            # float32 normalisation of the residuals: a few ulp of slack
            assert (np.abs(ch - bh) <= k * env_h * (1 + 1e-5) + 1e-5).all()
            assert (np.abs(cb - bb) <= k * env_b * (1 + 1e-5) + 1e-6).all()
            inside = np.abs(oh - bh) < 0.9 * k * env_h  # unclamped residuals inside the envelope stay
            assert np.allclose(ch[inside], oh[inside], rtol=0, atol=1e-5)
    finally:
        c.close()
    c = K.Corrector(ny, ny, f, max_batch=4, seed=3)
    try:
        for bad in ((-1.0, 0, 0.0), (0.0, 2, 0.0), (0.0, 0, -1.0)):
            assert T.lib().tsu_corr_set_options(c._h, *bad) != 0
    finally:
        c.close()


def test_set_weights_round_trip_and_conv_bench():
    dev()
    ny, f = 32, 4
    Hf, coarse, fine = synthetic_samples(2, ny, f, 6)
    c = K.Corrector(ny, ny, f, max_batch=2, seed=4)
    try:
        c.set_site(Hf)
        c.add_samples(coarse, fine)
        Wt, B = c.weights()
        Wt2 = Wt * 0.5
        c.set_weights(Wt2, B + 1.0)
        Wr, Br = c.weights()
        assert np.array_equal(Wr, Wt2) and np.array_equal(Br, B + 1.0)
        ms, tf = c.bench_conv(2, 3)
        assert ms > 0 and tf > 0
    finally:
        c.close()


def test_held_out_sources_improve_on_interpolation():
    """The whole pipeline at a small size: pairs from FP32 ensembles on a 128^2
    site (coarse 32^2), held-out sources compared with the FP64 plain fine
    solve.  With the options the bench uses (large-residual weight 16, depth
    clip, envelope 1) the corrector's maximum-depth and bed-change RMSE are
    below those of the interpolation alone, and its maximum-depth L-inf is
    not more than 10 % above it (the L-inf comes from a few pixels and varies
    from seed to seed; the bench reports it at 512^2)."""
    dev()
    n, f, t_end = 128, 4, 300.0
    site = K.make_site(n=n, factor=f, dx=20.0)
    train, test = K.make_sources(48, seed=11), K.make_sources(8, seed=12)
    fine = K.solve_fp32(site.H, site.mask, site.dx, site.slr, train, t_end)
    coarse_train = K.coarse_inputs(site, train, t_end)
    coarse_test = K.coarse_inputs(site, test, t_end)
    truth = K.solve_fp64(site.H, site.mask, site.dx, site.slr, test, t_end)
    c = K.Corrector(n, n, f, max_batch=8, seed=7)
    try:
        c.set_site(site.H)
        c.set_options(16.0, True, 1.0)
        c.add_samples(coarse_train, fine)
        c.add_samples(coarse_test, truth)
        for k, (it, lr) in enumerate([(400, 1e-3), (200, 3e-4), (200, 1e-4)]):
            c.train(len(train), it, batch=8, lr=lr, seed=1 + k)
        oh, ob, bh, bb = c.predict(len(train), len(test))
    finally:
        c.close()
    region = (truth[:, 0] > 0) | (oh != 0) | (bh != 0)
    ew, e0 = K.errors((oh, ob), truth, region), K.errors((bh, bb), truth, region)
    print("held out: corrector %s, interpolation %s" % (ew, e0))
    assert (oh >= 0).all()
    assert ew["hmax_rmse_m"] < e0["hmax_rmse_m"]
    assert ew["db_rmse_m"] < e0["db_rmse_m"]
    assert ew["hmax_linf_m"] <= 1.1 * e0["hmax_linf_m"]


_PLAIN_RUN = """
import sys, ctypes as C, numpy as np, torch
import tsuner_b200 as T
g = torch.Generator().manual_seed(21)
X = torch.randn(3, 40, 72, 32, generator=g).to(torch.bfloat16).cuda()
Wk = (torch.randn(32, 9, 32, generator=g) * 0.1).to(torch.bfloat16).cuda()
b = (torch.randn(32, generator=g) * 0.1).cuda()
Y = torch.zeros((3, 40, 72, 32), device="cuda", dtype=torch.float32)
rc = T.lib().tsu_corr_conv3x3(C.c_void_p(X.data_ptr()), 3, 40, 72, C.c_void_p(Wk.data_ptr()),
                              C.c_void_p(b.data_ptr()), 1, None, None, C.c_void_p(Y.data_ptr()), None)
assert rc == 0 and T.lib().tsu_corr_status() == 0
np.save(sys.argv[1], Y.cpu().numpy())
"""


def test_both_forward_kernels_give_identical_outputs(tmp_path):
    """The warp-specialised forward kernel (default) and conv3x3_fwd_kernel
    (TSU_CONV_FWD=plain) issue the same MMAs in the same order and share the
    epilogue: their outputs are equal value for value.  The kernel is chosen
    once per process, so each runs in its own."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for name in ("ws", "plain"):
        env = dict(os.environ, TSU_CONV_FWD=name)
        path = str(tmp_path / (name + ".npy"))
        r = subprocess.run([sys.executable, "-c", _PLAIN_RUN, path], env=env, cwd=root, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        out[name] = np.load(path)
    assert np.abs(out["ws"]).max() > 0
    assert np.array_equal(out["ws"], out["plain"])


def test_training_is_reproducible():
    """The weight gradient adds its per-CTA partials in a fixed order, so two
    trainings from the same seed on the same samples give the same weights
    bit for bit (the loss sums may differ in their last bits)."""
    dev()
    ny, f = 64, 4
    Hf, coarse, fine = synthetic_samples(8, ny, f, 9)
    out = []
    for _ in range(2):
        c = K.Corrector(ny, ny, f, max_batch=4, seed=3)
        try:
            c.set_site(Hf)
            c.add_samples(coarse, fine)
            c.train(ntrain=8, iters=30, batch=4, lr=2e-3, seed=5)
            out.append(c.weights())
        finally:
            c.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
