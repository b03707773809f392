"""The learned pilot's kernels against PyTorch references.

Each tensor-core kernel is compared with a float64 PyTorch convolution of the
same BF16-rounded operands:
* the 48 -> 48 3 x 3 convolution (bias + ReLU, bias only, and the data
  gradient -- the transposed, flipped convolution masked by the layer input);
* the weight / bias gradient of such a layer.
A BF16 output is the rounding of an FP32 sum, so the bar is one BF16 rounding
(2^-8 relative) plus FP32 accumulation error; FP32 outputs (gradients) are held
to 1e-3 relative to the largest entry.

The whole network is compared with a float64 emulation that rounds weights and
activations to BF16 where the kernels do: the forward output, the loss, and the
full parameter gradient of one training step (against autograd). The training
step stores layer gradients in BF16, so the gradient bar is 3 % relative L2 per
layer and 0.999 cosine similarity.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C = 48


@pytest.fixture(scope="module")
def ctx(bm3d_lib):
    import isp_mw_b200
    c = isp_mw_b200.Context(0)
    yield c
    c.close()


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _conv48(ctx, x, W, b, aux, mode):
    import torch
    n, h, w, _ = x.shape
    y = torch.empty_like(x)
    rc = ctx.lib.bm3d_pilot_conv48(ctx.h, n, h, w, x.data_ptr(), W.data_ptr(),
                                   None if b is None else b.data_ptr(),
                                   None if aux is None else aux.data_ptr(), mode, y.data_ptr(),
                                   _stream())
    ctx._check(rc)
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("shape", [(2, 37, 53), (1, 8, 16), (3, 19, 7)])
def test_conv48_forward_matches_torch(ctx, shape):
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cuda").manual_seed(1)
    n, h, w = shape
    x = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    W = torch.randn(C, C, 3, 3, device="cuda", generator=g) * 0.05
    b = torch.randn(C, device="cuda", generator=g) * 0.1
    xr = x.double().permute(0, 3, 1, 2)
    Wr = W.bfloat16().double()
    lin = F.conv2d(xr, Wr, b.double(), padding=1).permute(0, 2, 3, 1)
    for mode, ref in ((0, torch.relu(lin)), (1, lin)):
        y = _conv48(ctx, x, W, b, None, mode).double()
        d = (y - ref).abs()
        bar = ref.abs() * 2.0 ** -8 + 1e-4 * ref.abs().max()
        assert bool((d <= bar).all()), (mode, float((d - bar).max()))


def test_conv48_data_gradient_matches_torch(ctx):
    import torch
    import torch.nn.functional as F
    g = torch.Generator(device="cuda").manual_seed(2)
    n, h, w = 2, 29, 41
    grad = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    aux = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    W = torch.randn(C, C, 3, 3, device="cuda", generator=g) * 0.05
    y = _conv48(ctx, grad, W, None, aux, 2).double()
    gx = F.conv_transpose2d(grad.double().permute(0, 3, 1, 2), W.bfloat16().double(), padding=1)
    ref = gx.permute(0, 2, 3, 1) * (aux.double() > 0)
    d = (y - ref).abs()
    bar = ref.abs() * 2.0 ** -8 + 1e-4 * ref.abs().max()
    assert bool((d <= bar).all()), float((d - bar).max())


@pytest.mark.parametrize("shape", [(2, 37, 53), (1, 8, 16), (3, 19, 7), (1, 1080, 1920)])
def test_conv48_tma_pipeline_equals_cp_async_kernel(ctx, shape):
    """The warp-specialised TMA pipeline (8 x 16 tiles, TMA halo loads and
    stores) and the cp.async kernel (16 x 8 tiles) issue the same MMAs per
    output pixel: identical BF16 outputs in every mode, ragged edges included."""
    import torch
    lib = ctx.lib
    g = torch.Generator(device="cuda").manual_seed(4)
    n, h, w = shape
    x = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    aux = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    W = torch.randn(C, C, 3, 3, device="cuda", generator=g) * 0.05
    b = torch.randn(C, device="cuda", generator=g) * 0.1
    try:
        for mode in (0, 1, 2):
            out = {}
            for which in (1, 2):
                assert lib.bm3d_pilot_set_conv_kernel(which) == 0
                out[which] = _conv48(ctx, x, W, b if mode < 2 else None, aux if mode == 2 else None,
                                     mode)
                assert lib.bm3d_pilot_conv_kernel() == which
            assert torch.equal(out[1], out[2]), (mode, (out[1].float() - out[2].float()).abs().max())
    finally:
        lib.bm3d_pilot_set_conv_kernel(0)
    _conv48(ctx, x, W, b, None, 0)
    assert lib.bm3d_pilot_conv_kernel() == 3  # forward layers default to the N = 144 pipeline
    _conv48(ctx, x, W, None, aux, 2)
    assert lib.bm3d_pilot_conv_kernel() == 2  # data gradients to the N = 48 one


@pytest.mark.parametrize("shape", [(2, 37, 53), (1, 8, 16), (3, 19, 7), (1, 1080, 1920),
                                   (2, 17, 13)])
def test_conv48_n144_matches_torch_and_n48(ctx, shape):
    """The N = 144 forward pipeline (three column taps per MMA, their partial
    sums added across TMEM lanes): against float64 PyTorch on BF16 operands,
    and against the N = 48 pipeline to within one BF16 rounding (the two add
    the same FP32 products in a different order)."""
    import torch
    import torch.nn.functional as F
    lib = ctx.lib
    g = torch.Generator(device="cuda").manual_seed(6)
    n, h, w = shape
    x = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    W = torch.randn(C, C, 3, 3, device="cuda", generator=g) * 0.05
    b = torch.randn(C, device="cuda", generator=g) * 0.1
    lin = F.conv2d(x.double().permute(0, 3, 1, 2), W.bfloat16().double(), b.double(),
                   padding=1).permute(0, 2, 3, 1)
    try:
        for mode, ref in ((0, torch.relu(lin)), (1, lin)):
            assert lib.bm3d_pilot_set_conv_kernel(3) == 0
            y3 = _conv48(ctx, x, W, b, None, mode)
            assert lib.bm3d_pilot_conv_kernel() == 3
            d = (y3.double() - ref).abs()
            bar = ref.abs() * 2.0 ** -8 + 1e-4 * ref.abs().max()
            assert bool((d <= bar).all()), (mode, float((d - bar).max()))
            assert lib.bm3d_pilot_set_conv_kernel(2) == 0
            y2 = _conv48(ctx, x, W, b, None, mode).float()
            assert bool(((y3.float() - y2).abs() <= y2.abs() * 2.0 ** -7 + 1e-6).all())
    finally:
        lib.bm3d_pilot_set_conv_kernel(0)


def test_wgrad48_matches_torch(ctx):
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    n, h, w = 2, 45, 38
    x = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    gr = torch.randn(n, h, w, C, device="cuda", generator=g).bfloat16()
    dw = torch.empty(C, C, 3, 3, device="cuda")
    db = torch.empty(C, device="cuda")
    rc = ctx.lib.bm3d_pilot_wgrad48(ctx.h, n, h, w, x.data_ptr(), gr.data_ptr(), dw.data_ptr(),
                                    db.data_ptr(), _stream())
    ctx._check(rc)
    torch.cuda.synchronize()
    ref_w = torch.nn.grad.conv2d_weight(x.double().permute(0, 3, 1, 2), (C, C, 3, 3),
                                        gr.double().permute(0, 3, 1, 2), padding=1)
    ref_b = gr.double().sum(dim=(0, 1, 2))
    for got, ref in ((dw.double(), ref_w), (db.double(), ref_b)):
        d = (got - ref).abs().max().item()
        assert d <= 1e-3 * ref.abs().max().item(), d


# ---- the whole network ------------------------------------------------------

def _split(params):
    """FP32 parameter vector -> per-layer (W, b) in PyTorch order."""
    off = 0
    layers = []
    for cin, cout in [(2, C)] + [(C, C)] * 6 + [(C, 1)]:
        nw = cout * cin * 9
        W = params[off:off + nw].reshape(cout, cin, 3, 3)
        off += nw
        b = params[off:off + cout]
        off += cout
        layers.append((W, b))
    assert off == params.numel()
    return layers


def _bf16(t):
    """BF16 rounding that passes gradients straight through."""
    return t + (t.bfloat16().double() - t).detach()


def _emulate(params, noisy, sigma):
    """float64 forward rounding where the kernels round: layer 1 FP32 weights,
    BF16 output; layers 2-7 BF16 weights, BF16 outputs; layer 8 FP32 weights on
    BF16 inputs, plus the noisy plane."""
    import torch
    import torch.nn.functional as F
    L = _split(params)
    smap = sigma.view(-1, 1, 1, 1) * torch.ones_like(noisy).unsqueeze(1)
    x = torch.cat([noisy.unsqueeze(1), smap], dim=1)
    x = _bf16(torch.relu(F.conv2d(x, L[0][0], L[0][1], padding=1)))
    for W, b in L[1:7]:
        x = _bf16(torch.relu(F.conv2d(x, _bf16(W), b, padding=1)))
    return noisy + F.conv2d(x, L[7][0], L[7][1], padding=1)[:, 0]


def _data(n, h, w, seed):
    import torch
    from isp_mw_b200 import synth
    rng = np.random.default_rng(seed)
    sig = rng.uniform(5, 50, n).astype(np.float32)
    pairs = [synth.pair(h, w, float(s), seed + i) for i, s in enumerate(sig)]
    noisy = np.stack([p[1] for p in pairs])
    clean = np.stack([p[0] for p in pairs])
    return (torch.from_numpy(noisy).cuda(), torch.from_numpy(clean).cuda(),
            torch.from_numpy(sig / 255.0).cuda())


def test_pilot_forward_matches_emulation(ctx):
    import torch
    import isp_mw_b200
    p = isp_mw_b200.Pilot(ctx, seed=5)
    noisy, _, sigma = _data(3, 40, 56, 11)
    out = torch.empty_like(noisy)
    p.estimate(out, noisy, sigma.cpu().numpy())
    ref = _emulate(torch.from_numpy(p.params()).cuda().double(), noisy.double(), sigma.double())
    d = (out.double() - ref).abs().max().item()
    assert d <= 2e-3 * ref.abs().max().item(), d
    # host planes give the same estimate
    host = np.empty(noisy.shape, np.float32)
    p.estimate(host, noisy.cpu().numpy(), sigma.cpu().numpy())
    assert np.array_equal(host, out.cpu().numpy())
    p.close()


def test_pilot_layer_timing(ctx):
    """bm3d_pilot_set_timing / bm3d_pilot_layer_ms: eight positive layer
    times, the 48 -> 48 layers the bulk of the pass."""
    import torch
    import isp_mw_b200
    p = isp_mw_b200.Pilot(ctx, seed=12)
    noisy, _, sigma = _data(2, 256, 320, 61)
    out = torch.empty_like(noisy)
    p.set_timing(True)
    p.estimate(out, noisy, sigma.cpu().numpy())
    ms = p.layer_ms()
    p.set_timing(False)
    assert ms.shape == (8,) and (ms > 0).all(), ms
    p.close()


def test_pilot_gradient_matches_autograd(ctx):
    import torch
    import isp_mw_b200
    p = isp_mw_b200.Pilot(ctx, seed=6)
    noisy, clean, sigma = _data(4, 48, 40, 21)
    params = p.params()
    loss = p.train_step(noisy, clean, sigma, lr=1e-12)
    grad = torch.from_numpy(p.grad()).double()
    pt = torch.from_numpy(params).cuda().double().requires_grad_(True)
    out = _emulate(pt, noisy.double(), sigma.double())
    # squared error scaled to a common noise level, (25/255 / sigma)^2 per image
    q = ((25.0 / 255.0) / sigma.double()) ** 2
    ref_loss = (q.view(-1, 1, 1) * (out - clean.double()) ** 2).mean()
    ref_loss.backward()
    ref = pt.grad.cpu()
    assert abs(loss - ref_loss.item()) <= 1e-3 * ref_loss.item(), (loss, ref_loss.item())
    off = 0
    for W, b in _split(torch.arange(params.size)):
        for part in (W, b):
            sl = slice(off, off + part.numel())
            off += part.numel()
            g, r = grad[sl], ref[sl]
            rel = ((g - r).norm() / r.norm()).item()
            cos = (torch.dot(g, r) / (g.norm() * r.norm())).item()
            assert rel <= 0.03 and cos >= 0.999, (sl, rel, cos)
    p.close()


def test_pilot_training_reduces_loss(ctx):
    import isp_mw_b200
    p = isp_mw_b200.Pilot(ctx, seed=7)
    noisy, clean, sigma = _data(8, 64, 64, 31)
    first = p.train_step(noisy, clean, sigma, lr=1e-3)
    for _ in range(60):
        last = p.train_step(noisy, clean, sigma, lr=1e-3)
    assert last < 0.7 * first, (first, last)
    p.close()


def test_pilot_checkpoint_round_trip(ctx, tmp_path):
    import torch
    import isp_mw_b200
    a = isp_mw_b200.Pilot(ctx, seed=8)
    noisy, clean, sigma = _data(2, 32, 48, 41)
    a.train_step(noisy, clean, sigma, lr=1e-3)
    path = str(tmp_path / "pilot.bin")
    a.save(path)
    b = isp_mw_b200.Pilot(ctx, seed=9)
    b.load(path)
    assert np.array_equal(a.params(), b.params())
    ya, yb = torch.empty_like(noisy), torch.empty_like(noisy)
    a.estimate(ya, noisy, sigma.cpu().numpy())
    b.estimate(yb, noisy, sigma.cpu().numpy())
    assert torch.equal(ya, yb)
    # the optimiser state came along: the next steps agree too (to float
    # rounding: the loss and the small layers' gradients are summed with atomics)
    la = a.train_step(noisy, clean, sigma, lr=1e-3)
    lb = b.train_step(noisy, clean, sigma, lr=1e-3)
    assert abs(la - lb) <= 1e-9 * abs(la)
    np.testing.assert_allclose(a.params(), b.params(), rtol=1e-5, atol=1e-7)
    a.close()
    b.close()


def test_pilot_full_is_final_stage_on_pilot_estimate(ctx):
    import isp_mw_b200
    from isp_mw_b200 import synth
    p = isp_mw_b200.Pilot(ctx, seed=10)
    _, noisy = synth.pair(120, 176, 25.0, 51)
    sp = [synth.sigma_param(25.0)] * 3
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    full = np.empty_like(noisy)
    p.full(f, full, noisy)
    est = np.empty_like(noisy)
    # the noise level bm3d_pilot_full derives from the final stage's sigma
    p.estimate(est, noisy, np.float32(f.sigma[0] / np.sqrt(3.0) / 255.0))
    want = np.empty_like(noisy)
    ctx.stage(f, True, want, noisy, est)
    assert np.array_equal(full, want)
    p.close()
