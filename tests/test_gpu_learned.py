"""GPU tests of the learned stage's kernels and network against plain PyTorch
FP32 references (extension; no reference counterpart).

BF16 operands are exact in FP32, so the tensor-core products match the FP32
reference exactly and only the accumulation order and the BF16 rounding of
the stored outputs differ: layer outputs within 1e-2 of the output range,
FP32 weight gradients within 1e-3.  The whole network (14 BF16 layers)
within 3e-2 of the range of its residual; gradients are checked through the
first Adam step, whose update is the gradient's sign.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _tw(w):
    """(cout, 9, cin) -> torch conv weight (cout, cin, 3, 3)"""
    cout, _, cin = w.shape
    return w.reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()


@pytest.mark.parametrize("cin,cout,B,H,W", [(16, 32, 2, 16, 32), (32, 64, 1, 24, 48),
                                            (96, 32, 2, 8, 16), (64, 128, 1, 16, 16),
                                            (128, 256, 1, 16, 32), (192, 64, 1, 8, 32),
                                            (128, 384, 1, 8, 16), (384, 128, 1, 8, 16),
                                            (32, 96, 2, 8, 16), (256, 256, 1, 8, 32),
                                            (32, 32, 2, 256, 512), (64, 64, 1, 128, 256),
                                            (96, 32, 1, 64, 256), (16, 32, 1, 40, 128),
                                            (32, 96, 1, 16, 256), (64, 128, 1, 16, 128),
                                            (32, 64, 3, 24, 384)])
def test_conv3x3_matches_torch(cin, cout, B, H, W):
    """The tensor-core (tcgen05) paths: the tiled form for every channel-chunk /
    output-tile configuration, the row-streaming form (W % 128 == 0, weights in
    shared memory) including partial strips, and images with many tiles or
    strips per persistent CTA."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(cin + cout)
    x = torch.randn((B, H, W, cin), device="cuda", generator=g).bfloat16()
    w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
    b = torch.randn(cout, device="cuda", generator=g)
    y = learned.conv3x3(x, w, b, relu=True)
    ref = F.relu(F.conv2d(x.float().permute(0, 3, 1, 2), _tw(w.float()), b, padding=1))
    ref = ref.permute(0, 2, 3, 1)
    torch.cuda.synchronize()
    tol = 1e-2 * float(ref.abs().max())
    assert float((y.float() - ref).abs().max()) <= tol


def test_conv3x3_unaligned_output_slice_uses_mma_path():
    """An output channel offset that is not a multiple of 8 goes to the
    mma.sync kernel; same results."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(17)
    B, H, W, cin, cout = 1, 16, 32, 32, 32
    x = torch.randn((B, H, W, cin), device="cuda", generator=g).bfloat16()
    w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
    yb = torch.zeros((B, H, W, 38), dtype=torch.bfloat16, device="cuda")
    learned.conv3x3(x, w, None, y=yb, y_co=2, relu=False)
    ref = F.conv2d(x.float().permute(0, 3, 1, 2), _tw(w.float()), padding=1).permute(0, 2, 3, 1)
    torch.cuda.synchronize()
    assert float((yb[..., 2:34].float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
    assert float(yb[..., :2].float().abs().max()) == 0.0


def test_conv3x3_row_form_slices_and_mask():
    """Row-streaming form with channel slices and the ReLU-mask epilogue (the
    data-gradient use)."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(23)
    B, H, W, cin, cout = 2, 24, 256, 32, 64
    xb = torch.randn((B, H, W, 96), device="cuda", generator=g).bfloat16()
    w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
    mask = torch.randn((B, H, W, 96), device="cuda", generator=g).bfloat16()
    yb = torch.zeros((B, H, W, 128), dtype=torch.bfloat16, device="cuda")
    learned.conv3x3(xb, w, None, cin=cin, x_co=32, y=yb, y_co=64, cout=cout, mask=mask, m_co=32,
                    relu=False)
    ref = F.conv2d(xb[..., 32:64].float().permute(0, 3, 1, 2), _tw(w.float()), padding=1)
    ref = ref.permute(0, 2, 3, 1) * (mask[..., 32:96].float() > 0)
    torch.cuda.synchronize()
    assert float((yb[..., 64:128].float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
    assert float(yb[..., :64].float().abs().max()) == 0.0


def test_conv3x3_channel_slices_and_mask():
    """Input and output as channel slices of wider buffers, mask epilogue."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(7)
    B, H, W, cin, cout = 1, 16, 32, 32, 32
    xb = torch.randn((B, H, W, 96), device="cuda", generator=g).bfloat16()
    w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
    mask = torch.randn((B, H, W, 64), device="cuda", generator=g).bfloat16()
    yb = torch.zeros((B, H, W, 96), dtype=torch.bfloat16, device="cuda")
    learned.conv3x3(xb, w, None, cin=cin, x_co=64, y=yb, y_co=32, cout=cout, mask=mask, m_co=32,
                    relu=False)
    ref = F.conv2d(xb[..., 64:96].float().permute(0, 3, 1, 2), _tw(w.float()), padding=1)
    ref = ref.permute(0, 2, 3, 1) * (mask[..., 32:64].float() > 0)
    torch.cuda.synchronize()
    assert float((yb[..., 32:64].float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max())
    assert float(yb[..., :32].float().abs().max()) == 0.0
    assert float(yb[..., 64:].float().abs().max()) == 0.0


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 64), (96, 32), (64, 128)])
def test_data_gradient_matches_torch(cin, cout):
    torch = _torch()
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(cin * 3 + cout)
    B, H, W = 2, 16, 32
    w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
    dy = torch.randn((B, H, W, cout), device="cuda", generator=g).bfloat16()
    if cin % 32:  # data gradients of 16-channel inputs are not produced
        pytest.skip("16-channel data gradient not used")
    dx = learned.conv3x3(dy, learned.flip_weights(w), None, relu=False)
    ref = torch.nn.grad.conv2d_input((B, cin, H, W), _tw(w.float()),
                                     dy.float().permute(0, 3, 1, 2), padding=1)
    ref = ref.permute(0, 2, 3, 1)
    torch.cuda.synchronize()
    assert float((dx.float() - ref).abs().max()) <= 1e-2 * float(ref.abs().max())


@pytest.mark.parametrize("cin,cout,B,H,W", [(16, 32, 2, 16, 64), (32, 64, 2, 16, 64),
                                            (96, 32, 2, 16, 64), (64, 128, 2, 16, 64),
                                            (32, 256, 2, 16, 64), (384, 128, 1, 16, 32),
                                            (192, 64, 1, 16, 32), (128, 384, 1, 8, 32),
                                            (32, 32, 4, 64, 128)])
def test_weight_gradient_matches_torch(cin, cout, B, H, W):
    """The tcgen05 weight gradient (split-K over pixel blocks, MN-major
    operands, 16-byte atomics): every output/input channel tiling and many
    blocks per CTA."""
    torch = _torch()
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(cin + 5 * cout)
    x = torch.randn((B, H, W, cin), device="cuda", generator=g).bfloat16()
    dy = torch.randn((B, H, W, cout), device="cuda", generator=g).bfloat16()
    dw = torch.zeros((cout, 9, cin), device="cuda")
    learned.conv3x3_wgrad(x, dy, dw)
    ref = torch.nn.grad.conv2d_weight(x.float().permute(0, 3, 1, 2), (cout, cin, 3, 3),
                                      dy.float().permute(0, 3, 1, 2), padding=1)
    ref = ref.permute(0, 2, 3, 1).reshape(cout, 9, cin)
    torch.cuda.synchronize()
    assert float((dw - ref).abs().max()) <= 1e-3 * float(ref.abs().max())


def _torch_unet(p, scale):
    """The same network in plain PyTorch FP32 (weights rounded to BF16 as the
    kernels use them)."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    layers, hw, hb = learned.split_params(p)
    ws = [(_tw(torch.from_numpy(w.copy()).cuda().bfloat16().float()),
           torch.from_numpy(b.copy()).cuda()) for w, b in layers]
    hw_t = torch.from_numpy(hw.copy()).cuda()

    def net(x):
        B, H, W = x.shape
        x16 = torch.zeros((B, 16, H, W), device="cuda")
        x16[:, 0] = x * scale
        c = lambda t, k: F.relu(F.conv2d(t, ws[k][0], ws[k][1], padding=1))
        up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")
        s1 = c(c(x16, 0), 1)
        s2 = c(c(F.max_pool2d(s1, 2), 2), 3)
        s3 = c(c(F.max_pool2d(s2, 2), 4), 5)
        bott = c(c(F.max_pool2d(s3, 2), 6), 7)
        d3 = c(c(torch.cat([up(bott), s3], 1), 8), 9)
        d2 = c(c(torch.cat([up(d3), s2], 1), 10), 11)
        d1 = c(c(torch.cat([up(d2), s1], 1), 12), 13)
        out = x * scale + torch.einsum("bchw,c->bhw", d1, hw_t) + float(hb)
        return out / scale
    return net


def test_unet_forward_matches_torch():
    torch = _torch()
    from ctas_b200 import learned
    with learned.UNet(seed=3, scale=2.0) as net:
        p = net.get_params()
        layers, hw, hb = learned.split_params(p)
        rng = np.random.default_rng(1)
        p[-33:-1] = rng.standard_normal(32).astype(np.float32) * 0.1   # a non-zero head
        p[-1] = 0.05
        net.set_params(p)
        g = torch.Generator(device="cuda").manual_seed(2)
        x = torch.rand((2, 64, 128), device="cuda", generator=g)
        y = net.forward(x)
        ref = _torch_unet(p, 2.0)(x)
        torch.cuda.synchronize()
        r = (ref - x)
        assert float(((y - x) - r).abs().max()) <= 3e-2 * float(r.abs().max())


def test_unet_gradient_signs_match_torch():
    """The first Adam step moves every parameter by lr * sign(gradient) (up to
    eps): its sign must agree with PyTorch autograd on the same loss wherever
    the gradient is not tiny."""
    torch = _torch()
    from ctas_b200 import learned
    with learned.UNet(seed=11, scale=1.0) as net:
        p = net.get_params()
        rng = np.random.default_rng(4)
        p[-33:-1] = rng.standard_normal(32).astype(np.float32) * 0.1
        net.set_params(p)
        g = torch.Generator(device="cuda").manual_seed(5)
        x = torch.rand((2, 64, 128), device="cuda", generator=g)
        t = x + 0.1 * torch.randn((2, 64, 128), device="cuda", generator=g)
        # autograd on the FP32 network
        pt = torch.from_numpy(p.copy()).cuda().requires_grad_(True)

        def net_from(vec):
            import torch.nn.functional as F
            o, ws = 0, []
            for cin, cout in learned.LAYERS:
                w = vec[o:o + cout * 9 * cin].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2)
                o += cout * 9 * cin
                b = vec[o:o + cout]
                o += cout
                ws.append((w, b))
            hw, hb = vec[o:o + 32], vec[o + 32]
            B, H, W = x.shape
            x16 = torch.zeros((B, 16, H, W), device="cuda")
            x16[:, 0] = x
            c = lambda tt, k: F.relu(F.conv2d(tt, ws[k][0], ws[k][1], padding=1))
            up = lambda tt: F.interpolate(tt, scale_factor=2, mode="nearest")
            s1 = c(c(x16, 0), 1)
            s2 = c(c(F.max_pool2d(s1, 2), 2), 3)
            s3 = c(c(F.max_pool2d(s2, 2), 4), 5)
            bott = c(c(F.max_pool2d(s3, 2), 6), 7)
            d3 = c(c(torch.cat([up(bott), s3], 1), 8), 9)
            d2 = c(c(torch.cat([up(d3), s2], 1), 10), 11)
            d1 = c(c(torch.cat([up(d2), s1], 1), 12), 13)
            return x + torch.einsum("bchw,c->bhw", d1, hw) + hb

        loss = ((net_from(pt) - t) ** 2).mean()
        loss.backward()
        grad = pt.grad.detach().cpu().numpy()
        lr = 1e-4
        net.train_step(x, t, lr)
        delta = net.get_params() - p
        big = np.abs(grad) > 1e-2 * np.abs(grad).max()
        agree = np.mean(np.sign(delta[big]) == -np.sign(grad[big]))
        assert big.sum() > 1000
        assert agree >= 0.97, agree


def test_unet_training_reduces_loss():
    """Learning a fixed smoothing of the input: the loss falls."""
    torch = _torch()
    import torch.nn.functional as F
    from ctas_b200 import learned
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.rand((4, 64, 128), device="cuda", generator=g)
    k = torch.ones((1, 1, 5, 5), device="cuda") / 25.0
    t = F.conv2d(x[:, None], k, padding=2)[:, 0].contiguous()
    with learned.UNet(seed=1, scale=1.0) as net:
        losses = [net.train_step(x, t, 1e-3) for _ in range(60)]
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])


def test_unet_shape_errors():
    torch = _torch()
    from ctas_b200 import _lib, learned
    with learned.UNet(seed=0) as net:
        with pytest.raises(_lib.CtasError) as e:
            net.forward(torch.zeros((1, 60, 128), device="cuda"))
        assert e.value.code == _lib.E_SHAPE
