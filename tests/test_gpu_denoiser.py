"""The learned denoiser's kernels against a plain PyTorch FP32 reference of
the same network.

The reference runs the same architecture (3x3 convolutions 16-32-32 / 64 /
96 / 128 with 2x2 average pooling, nearest upsampling and skip concatenation,
leaky ReLU 0.1) in FP32 on values rounded to BF16 where the library stores
BF16 (weights, activations); the library accumulates in FP32 on tensor
cores, so the two differ only by summation order and the BF16 rounding of
nearby values.  Bars: forward output within 2e-2 of its scale (max abs) and
1e-3 RMS; after one Adam step (whose first update is -lr * sign(gradient))
the update's sign equals the reference gradient's sign on >= 99% of the
parameters whose gradient is at least 1% of the largest in their layer, and
the gradient itself (read back without a step) has a cosine similarity of
at least 0.997 and a relative L2 error of at most 8e-2 in every layer; with
every pre-activation positive (no leaky-ReLU kink between the two forward
passes) at most 2e-2.
"""
import ctypes

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import arbor_b200 as ab

pytestmark = pytest.mark.gpu

SPEC = [(16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1), (64, 96, 1), (96, 96, 1), (96, 128, 1), (128, 128, 1), (224, 96, 1),
        (96, 96, 1), (160, 64, 1), (64, 64, 1), (96, 32, 1), (32, 32, 1), (32, 16, 0)]


def bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


def unpack(params):
    """Flat FP32 parameters -> [(weight [cout][cin][3][3], bias)] per layer."""
    out, off = [], 0
    for cin, cout, _ in SPEC:
        n = cout * 9 * cin
        w = params[off:off + n].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()
        off += n
        b = params[off:off + cout]
        off += cout
        out.append((w, b))
    assert off == params.numel()
    return out


def reference_forward(layers, feat):
    """feat: [N, 16, H, W] FP32 (BF16 values).  Returns the FP32 output [N, 16, H, W]."""
    def conv(i, x):
        w, b = layers[i]
        y = F.conv2d(x, bf(w), b, padding=1)
        return bf(F.leaky_relu(y, 0.1)) if SPEC[i][2] else y

    def pool(x):
        return bf(F.avg_pool2d(x, 2))

    def upcat(skip, low):
        return torch.cat([skip, F.interpolate(low, scale_factor=2, mode="nearest")], 1)

    e0 = conv(1, conv(0, feat))
    e1 = conv(3, conv(2, pool(e0)))
    e2 = conv(5, conv(4, pool(e1)))
    b3 = conv(7, conv(6, pool(e2)))
    d2 = conv(9, conv(8, upcat(e2, b3)))
    d1 = conv(11, conv(10, upcat(e1, d2)))
    d0 = conv(13, conv(12, upcat(e0, d1)))
    return conv(14, d0)


class Net:
    def __init__(self, batch, w, h, seed=3):
        self.lib = ab.lib()
        self.h = ctypes.c_void_p()
        st = self.lib.arbor_denoiser_create(ctypes.byref(self.h), batch, w, h, seed, None)
        assert st == ab.OK, ab.last_error()
        n = ctypes.c_size_t()
        assert self.lib.arbor_denoiser_param_count(self.h, ctypes.byref(n)) == ab.OK
        self.count = n.value

    def params(self):
        p = np.zeros(self.count, np.float32)
        assert self.lib.arbor_denoiser_get_params(self.h, p.ctypes.data, p.size) == ab.OK
        return torch.from_numpy(p)

    def close(self):
        self.lib.arbor_denoiser_destroy(self.h)


def random_inputs(batch, w, h, seed=0):
    g = torch.Generator().manual_seed(seed)
    noisy = torch.rand(batch, h, w, 4, generator=g) * 2.0
    target = noisy * (0.7 + 0.6 * torch.rand(batch, h, w, 4, generator=g))
    feat = torch.zeros(batch, h, w, 16)
    feat[..., :10] = torch.rand(batch, h, w, 10, generator=g) * 2.0 - 0.5
    feat[..., :3] = torch.log1p(noisy[..., :3])  # as arbor_denoiser_features lays them out
    return bf(feat), noisy, target


def to_dev_bf16(feat):
    return feat.to(torch.bfloat16).contiguous().cuda().view(torch.int16)


def test_forward_matches_fp32_reference(cuda):
    batch, w, h = 2, 48, 32
    net = Net(batch, w, h)
    try:
        layers = unpack(net.params())
        feat, noisy, _ = random_inputs(1, w, h)
        fdev = to_dev_bf16(feat)
        ndev = noisy.contiguous().cuda()
        out = torch.zeros(h * w * 4, device="cuda")
        st = net.lib.arbor_denoiser_infer(net.h, fdev.data_ptr(), ndev.data_ptr(), out.data_ptr(), w, h)
        assert st == ab.OK, ab.last_error()
        torch.cuda.synchronize()
        got = out.cpu().view(h, w, 4)[..., :3]
        ref_out = reference_forward(layers, feat.permute(0, 3, 1, 2))[0, :3].permute(1, 2, 0)
        want = torch.expm1(torch.log1p(noisy[0, ..., :3].clamp(min=0)) + ref_out)
        err = (got - want).abs()
        scale = want.abs().max().item()
        rms = err.pow(2).mean().sqrt().item()
        print(f"[denoiser forward] max abs err {err.max().item():.3g} (scale {scale:.3g}), rms {rms:.3g}")
        assert err.max().item() <= 2e-2 * max(1.0, scale)
        assert rms <= 1e-3 * max(1.0, scale)
    finally:
        net.close()


def test_first_adam_step_follows_reference_gradient(cuda):
    batch, w, h = 2, 32, 32
    net = Net(batch, w, h, seed=5)
    try:
        p0 = net.params()
        layers = unpack(p0.clone())
        feat, noisy, target = random_inputs(batch, w, h, seed=1)
        # reference gradient of the same loss
        params = [t.clone().requires_grad_(True) for pair in layers for t in pair]
        ref_layers = [(params[2 * i], params[2 * i + 1]) for i in range(len(SPEC))]
        out = reference_forward(ref_layers, feat.permute(0, 3, 1, 2))[:, :3].permute(0, 2, 3, 1)
        pred = torch.log1p(noisy[..., :3].clamp(min=0)) + out
        loss = (pred - torch.log1p(target[..., :3].clamp(min=0))).abs().mean()
        loss.backward()
        gref = torch.cat([torch.cat([params[2 * i].grad.permute(0, 2, 3, 1).reshape(-1), params[2 * i + 1].grad]) for i in range(len(SPEC))])
        lr = 1e-4
        lval = ctypes.c_float()
        # device copies held in names: a temporary's memory could be reused before the call reads it
        fdev, ndev, tdev = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        st = net.lib.arbor_denoiser_train_step(net.h, fdev.data_ptr(), ndev.data_ptr(), tdev.data_ptr(), batch, w, h, lr, ctypes.byref(lval))
        assert st == ab.OK, ab.last_error()
        p1 = net.params()
        step = (p0 - p1) / lr  # = sign(gradient) where the gradient is not tiny
        # parameters whose reference gradient is at least 1% of the largest in their layer
        big = torch.zeros_like(gref, dtype=torch.bool)
        off = 0
        for cin, cout, _ in SPEC:
            n = cout * 9 * cin + cout
            seg = gref[off:off + n].abs()
            big[off:off + n] = seg > 1e-2 * seg.max()
            off += n
        agree = (torch.sign(step[big]) == torch.sign(gref[big])).float().mean().item()
        print(f"[denoiser backward] loss {lval.value:.5f} (reference {loss.item():.5f}); update sign agrees on {agree:.4f} "
              f"of {int(big.sum())} parameters")
        assert abs(lval.value - loss.item()) <= 2e-3 * max(1.0, loss.item())
        assert agree >= 0.99
    finally:
        net.close()


def test_gradient_matches_reference(cuda):
    """The backward kernels' gradient (arbor_denoiser_gradient) against the
    FP32 autograd gradient of the same loss on the same BF16 values: per
    layer, cosine similarity >= 0.997 and relative L2 error <= 8e-2
    (measured worst layer 0.9987 and 5.2e-2 on this case, mostly from
    pre-activations on different sides of leaky ReLU's kink in the two
    forward passes: test_gradient_in_the_linear_regime); the loss within
    2e-3 of the reference's.  The parameters are unchanged."""
    batch, w, h = 2, 32, 32
    net = Net(batch, w, h, seed=5)
    try:
        p0 = net.params()
        layers = unpack(p0.clone())
        feat, noisy, target = random_inputs(batch, w, h, seed=1)
        params = [t.clone().requires_grad_(True) for pair in layers for t in pair]
        ref_layers = [(params[2 * i], params[2 * i + 1]) for i in range(len(SPEC))]
        out = reference_forward(ref_layers, feat.permute(0, 3, 1, 2))[:, :3].permute(0, 2, 3, 1)
        pred = torch.log1p(noisy[..., :3].clamp(min=0)) + out
        loss = (pred - torch.log1p(target[..., :3].clamp(min=0))).abs().mean()
        loss.backward()
        gref = torch.cat([torch.cat([params[2 * i].grad.permute(0, 2, 3, 1).reshape(-1), params[2 * i + 1].grad]) for i in range(len(SPEC))])
        grad = np.zeros(p0.numel(), np.float32)
        lval = ctypes.c_float()
        fdev, ndev, tdev = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        st = net.lib.arbor_denoiser_gradient(net.h, fdev.data_ptr(), ndev.data_ptr(), tdev.data_ptr(), batch, w, h, grad.ctypes.data, grad.size,
                                             ctypes.byref(lval))
        assert st == ab.OK, ab.last_error()
        g = torch.from_numpy(grad)
        assert torch.equal(net.params(), p0), "the gradient call must not change the parameters"
        off, worst_cos, worst_rel = 0, 1.0, 0.0
        for cin, cout, _ in SPEC:
            n = cout * 9 * cin + cout
            a_, b_ = g[off:off + n].double(), gref[off:off + n].double()
            cos = float((a_ @ b_) / (a_.norm() * b_.norm() + 1e-30))
            rel = float((a_ - b_).norm() / (b_.norm() + 1e-30))
            worst_cos, worst_rel = min(worst_cos, cos), max(worst_rel, rel)
            off += n
        print(f"[denoiser gradient] loss {lval.value:.6f} (reference {loss.item():.6f}); worst layer cosine {worst_cos:.6f}, "
              f"relative L2 error {worst_rel:.4f}")
        assert abs(lval.value - loss.item()) <= 2e-3 * max(1.0, loss.item())
        assert worst_cos >= 0.997
        assert worst_rel <= 8e-2
    finally:
        net.close()


def test_gradient_in_the_linear_regime(cuda):
    """The backward kernels' arithmetic alone.  In the randomly initialised
    network above, some pre-activations sit so close to zero that the
    library's and the reference's forward passes (same BF16 values,
    different FP32 summation orders) put them on different sides of leaky
    ReLU's kink: there the two backward passes scale the gradient by 1 and
    by 0.1.  With the library's own loss signs given to the reference the
    error stays at 4.9 % (measured), so the kink, not the loss, is the
    source of the 5 % allowed above.  Here
    every pre-activation is positive by construction (biases 4, weights at
    a fifth of He scale), so both networks are linear and every loss term's
    sign is the same (the prediction exceeds the target by about 3 in
    log space): per layer, relative L2 error <= 2e-2 and cosine >= 0.9998
    (measured at most 6.1e-3)."""
    batch, w, h = 2, 32, 32
    net = Net(batch, w, h, seed=5)
    try:
        g = torch.Generator().manual_seed(9)
        flat = []
        for cin, cout, _ in SPEC:
            std = 0.2 * (2.0 / (9 * cin)) ** 0.5
            flat.append((torch.randn(cout, cin, 3, 3, generator=g) * std).permute(0, 2, 3, 1).reshape(-1))
            flat.append(torch.full((cout,), 4.0))
        p0 = torch.cat(flat).contiguous()
        pn = p0.numpy()
        assert net.lib.arbor_denoiser_set_params(net.h, pn.ctypes.data, pn.size) == ab.OK, ab.last_error()
        layers = unpack(p0.clone())
        feat, noisy, target = random_inputs(batch, w, h, seed=1)
        params = [t.clone().requires_grad_(True) for pair in layers for t in pair]
        ref_layers = [(params[2 * i], params[2 * i + 1]) for i in range(len(SPEC))]
        out = reference_forward(ref_layers, feat.permute(0, 3, 1, 2))[:, :3].permute(0, 2, 3, 1)
        resid = torch.log1p(noisy[..., :3].clamp(min=0)) + out - torch.log1p(target[..., :3].clamp(min=0))
        assert bool((resid > 0.5).all()), "every loss term must keep its sign"
        resid.abs().mean().backward()
        gref = torch.cat([torch.cat([params[2 * i].grad.permute(0, 2, 3, 1).reshape(-1), params[2 * i + 1].grad]) for i in range(len(SPEC))])
        grad = np.zeros(net.count, np.float32)
        lval = ctypes.c_float()
        fdev, ndev, tdev = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        st = net.lib.arbor_denoiser_gradient(net.h, fdev.data_ptr(), ndev.data_ptr(), tdev.data_ptr(), batch, w, h, grad.ctypes.data, grad.size,
                                             ctypes.byref(lval))
        assert st == ab.OK, ab.last_error()
        gl = torch.from_numpy(grad)
        off, worst_cos, worst_rel = 0, 1.0, 0.0
        for cin, cout, _ in SPEC:
            n = cout * 9 * cin + cout
            a_, b_ = gl[off:off + n].double(), gref[off:off + n].double()
            worst_cos = min(worst_cos, float((a_ @ b_) / (a_.norm() * b_.norm() + 1e-30)))
            worst_rel = max(worst_rel, float((a_ - b_).norm() / (b_.norm() + 1e-30)))
            off += n
        print(f"[denoiser gradient, linear regime] worst layer cosine {worst_cos:.6f}, relative L2 error {worst_rel:.4f}")
        assert worst_cos >= 0.9998
        assert worst_rel <= 2e-2
    finally:
        net.close()


def test_training_reduces_loss(cuda):
    batch, w, h = 2, 32, 32
    net = Net(batch, w, h, seed=9)
    try:
        feat, noisy, _ = random_inputs(batch, w, h, seed=2)
        target = noisy * 1.5  # a correction the network can learn from its radiance input
        f, n, t = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        losses = []
        for _ in range(60):
            lv = ctypes.c_float()
            assert net.lib.arbor_denoiser_train_step(net.h, f.data_ptr(), n.data_ptr(), t.data_ptr(), batch, w, h, 2e-3,
                                                     ctypes.byref(lv)) == ab.OK
            losses.append(lv.value)
        print(f"[denoiser training] loss {losses[0]:.4f} -> {losses[-1]:.4f}")
        assert losses[-1] < 0.5 * losses[0]
    finally:
        net.close()


def test_accumulate_and_features(cuda):
    lib = ab.lib()
    x = torch.rand(1000, device="cuda")
    s = torch.rand(1000, device="cuda")
    want = 0.5 * s + x
    assert lib.arbor_accumulate(s.data_ptr(), x.data_ptr(), 1000, 0.5, None) == ab.OK
    torch.cuda.synchronize()
    assert torch.equal(s, want)
    w, h = 16, 8
    lin, gui, nrm, hit = (torch.rand(w * h * 4, device="cuda") for _ in range(4))
    fil = torch.rand(w * h * 4, device="cuda")
    feat = torch.zeros(w * h * 16, dtype=torch.int16, device="cuda")
    assert lib.arbor_denoiser_features(lin.data_ptr(), gui.data_ptr(), nrm.data_ptr(), hit.data_ptr(), fil.data_ptr(), w, h,
                                       feat.data_ptr(), None) == ab.OK
    torch.cuda.synchronize()
    f = feat.view(torch.bfloat16).float().view(-1, 16).cpu()
    L, G, N, T, Q = (v.view(-1, 4).cpu() for v in (lin, gui, nrm, hit, fil))
    assert torch.allclose(f[:, 0:3], bf(torch.log1p(L[:, :3])), atol=0, rtol=0)
    assert torch.allclose(f[:, 3:6], bf(G[:, :3]), atol=0, rtol=0)
    assert torch.allclose(f[:, 6:9], bf(N[:, :3]), atol=0, rtol=0)
    assert torch.allclose(f[:, 9], bf(torch.log1p(T[:, 0]) * 0.25), atol=1e-2, rtol=0)
    assert torch.allclose(f[:, 10:13], bf(torch.log1p(Q[:, :3])), atol=0, rtol=0)
    assert (f[:, 13:] == 0).all()


def test_rejections(cuda):
    lib = ab.lib()
    h = ctypes.c_void_p()
    assert lib.arbor_denoiser_create(ctypes.byref(h), 1, 30, 32, 1, None) == ab.ERR_VALUE
    assert lib.arbor_denoiser_create(ctypes.byref(h), 1, 32, 32, 1, None) == ab.OK
    z = torch.zeros(32 * 32 * 16, device="cuda")
    assert lib.arbor_denoiser_infer(h, z.data_ptr(), z.data_ptr(), z.data_ptr(), 64, 64) == ab.ERR_LIMIT
    assert lib.arbor_denoiser_train_step(h, z.data_ptr(), z.data_ptr(), z.data_ptr(), 1, 32, 32, float("nan"), None) == ab.ERR_VALUE
    assert lib.arbor_denoiser_destroy(h) == ab.OK


@pytest.mark.parametrize("w,h", [(200, 64), (256, 128)])
def test_tcgen05_forward_matches_mma_sync(cuda, w, h):
    """The forward convolutions on tcgen05 (TMEM accumulators) against the
    mma.sync kernels on the same BF16 inputs and weights.  Both add the same
    K = 16 products into FP32 in the same order (input-channel chunk, tap,
    16 channels), so they may agree exactly; the bar allows neighbouring BF16
    roundings.  200 pixels per row leaves a partial 128-pixel tile."""
    net = Net(1, w, h, seed=4)
    try:
        feat, noisy, _ = random_inputs(1, w, h, seed=3)
        fdev, ndev = to_dev_bf16(feat), noisy.contiguous().cuda()
        outs = {}
        for tc in (1, 0):  # tcgen05 first, on freshly allocated activation buffers
            assert net.lib.arbor_denoiser_set_backend(net.h, tc) == ab.OK
            out = torch.zeros(h * w * 4, device="cuda")
            assert net.lib.arbor_denoiser_infer(net.h, fdev.data_ptr(), ndev.data_ptr(), out.data_ptr(), w, h) == ab.OK, ab.last_error()
            assert net.lib.arbor_denoiser_check(net.h) == ab.OK, ab.last_error()
            outs[tc] = out.cpu().view(h, w, 4)[..., :3]
        err = (outs[1] - outs[0]).abs()
        scale = outs[0].abs().max().item()
        rms = err.pow(2).mean().sqrt().item()
        print(f"[tcgen05 vs mma.sync {w}x{h}] max abs diff {err.max().item():.3g} (scale {scale:.3g}), rms {rms:.3g}")
        assert torch.isfinite(outs[1]).all()
        assert err.max().item() <= 1e-2 * max(1.0, scale)
        assert rms <= 5e-4 * max(1.0, scale)
    finally:
        net.close()


def train(net, feat, noisy, target, steps, lr=2e-3, batch=2, w=32, h=32):
    f, n, t = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
    for _ in range(steps):
        assert net.lib.arbor_denoiser_train_step(net.h, f.data_ptr(), n.data_ptr(), t.data_ptr(), batch, w, h, lr, None) == ab.OK, \
            ab.last_error()
    return net.params()


def test_training_is_deterministic_and_gradient_leaves_no_state(cuda):
    """Weight and bias gradients are folded in a fixed order (no atomics), so
    training is reproducible bit for bit; and arbor_denoiser_gradient leaves
    the parameters, the Adam moments and the gradient accumulator as it found
    them: gradient() then three train steps gives exactly the parameters of
    three train steps alone."""
    batch, w, h = 2, 32, 32
    feat, noisy, target = random_inputs(batch, w, h, seed=6)
    a, b = Net(batch, w, h, seed=8), Net(batch, w, h, seed=8)
    try:
        grad = np.zeros(a.count, np.float32)
        f, n, t = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        assert a.lib.arbor_denoiser_gradient(a.h, f.data_ptr(), n.data_ptr(), t.data_ptr(), batch, w, h, grad.ctypes.data, grad.size,
                                             None) == ab.OK, ab.last_error()
        g2 = np.zeros(a.count, np.float32)
        assert a.lib.arbor_denoiser_gradient(a.h, f.data_ptr(), n.data_ptr(), t.data_ptr(), batch, w, h, g2.ctypes.data, g2.size,
                                             None) == ab.OK
        assert np.array_equal(grad, g2), "the same gradient twice"
        pa = train(a, feat, noisy, target, 3)
        pb = train(b, feat, noisy, target, 3)
        print(f"[denoiser determinism] parameters differ at {int((pa != pb).sum())} of {pa.numel()}")
        assert torch.equal(pa, pb)
    finally:
        a.close()
        b.close()


def test_backward_data_pass_on_tcgen05_matches_mma_sync(cuda):
    """The gradient with the forward and backward data convolutions on
    tcgen05 against the same gradient with every convolution on mma.sync:
    both accumulate the same K = 16 products in the same order, but a
    product rounded to a neighbouring BF16 value in one stored activation or
    gradient (relative 2^-8) propagates through the 15 layers; the bar:
    relative L2 difference <= 2e-2 per layer (measured 1.05e-2 worst)."""
    batch, w, h = 2, 64, 32
    feat, noisy, target = random_inputs(batch, w, h, seed=7)
    net = Net(batch, w, h, seed=10)
    try:
        f, n, t = to_dev_bf16(feat), noisy.contiguous().cuda(), target.contiguous().cuda()
        grads = {}
        for tc in (1, 0):
            assert net.lib.arbor_denoiser_set_backend(net.h, tc) == ab.OK
            g = np.zeros(net.count, np.float32)
            assert net.lib.arbor_denoiser_gradient(net.h, f.data_ptr(), n.data_ptr(), t.data_ptr(), batch, w, h, g.ctypes.data, g.size,
                                                   None) == ab.OK, ab.last_error()
            assert net.lib.arbor_denoiser_check(net.h) == ab.OK, ab.last_error()
            grads[tc] = torch.from_numpy(g).double()
        off, worst = 0, 0.0
        for cin, cout, _ in SPEC:
            k = cout * 9 * cin + cout
            a_, b_ = grads[1][off:off + k], grads[0][off:off + k]
            worst = max(worst, float((a_ - b_).norm() / (b_.norm() + 1e-30)))
            off += k
        exact = int((grads[1] == grads[0]).sum())
        print(f"[denoiser backward tcgen05 vs mma.sync] worst layer relative difference {worst:.3g}; {exact} of {net.count} equal")
        assert worst <= 2e-2
    finally:
        net.close()


def test_trained_network_beats_filter_lighting_on_rendered_views(cuda):
    """What the learned path gains over the method without it: trained for
    1500 steps on 24 tracer-rendered views (1-spp inputs, 64-spp targets,
    128x128 crops at the full-HD pixel angle, sun shadows on), the network at
    1 spp beats filterLighting at 1 spp by >= 1 dB PSNR (after resolvePixels'
    tone mapping, mean over 6 held-out views; measured +2.7 dB)."""
    import math

    import denoise_train as dt
    import workloads

    S, spp = 128, 64
    seeds = workloads.batch_seeds(4)
    scenes = {}
    fr = dt.Frame(S, S)

    def scene_of(k):
        if k not in scenes:
            scenes[k] = dt.Scene(seeds[k])
        return scenes[k]

    train = [dt.render_pair(fr, scene_of(k), C, spp, eval_baselines=False) for k, C in dt.view_states(24, seeds, S, seed=21)]
    evals = [dt.render_pair(fr, scene_of(k), C, spp, eval_baselines=True) | {"C": C} for k, C in dt.view_states(6, seeds, S, seed=22)]
    feats = torch.stack([r["feat"] for r in train])
    base = torch.stack([r["base"] for r in train])
    target = torch.stack([r["target"] for r in train])
    net = Net(4, S, S, seed=7)
    try:
        rng = np.random.default_rng(3)
        for step in range(1500):
            i = int(rng.integers(0, len(train) - 4 + 1))
            lr = 1e-5 + 0.5 * (2e-3 - 1e-5) * (1.0 + math.cos(math.pi * step / 1500))
            assert net.lib.arbor_denoiser_train_step(net.h, feats[i].data_ptr(), base[i].data_ptr(), target[i].data_ptr(), 4, S, S, lr,
                                                     None) == ab.OK, ab.last_error()
        den = torch.zeros(S * S * 4, device="cuda")
        gain, filt, dens = [], [], []
        for e in evals:
            assert net.lib.arbor_denoiser_infer(net.h, e["feat"].data_ptr(), e["base"].data_ptr(), den.data_ptr(), S, S) == ab.OK
            ex = float(e["C"][20])
            ref = dt.tonemap(e["target"], S, S, ex)
            f1 = dt.psnr(dt.tonemap(e["filter1"], S, S, ex), ref)
            d1 = dt.psnr(dt.tonemap(den, S, S, ex), ref)
            filt.append(f1)
            dens.append(d1)
        print(f"[denoiser gain] held-out PSNR: filterLighting 1 spp {np.mean(filt):.2f} dB, denoiser 1 spp {np.mean(dens):.2f} dB")
        assert np.mean(dens) >= np.mean(filt) + 1.0
    finally:
        net.close()
