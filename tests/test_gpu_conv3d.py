"""The surrogate's BF16 tensor-core convolutions (xac_conv3d_*) against torch's FP32 conv3d on the same
BF16-rounded operands: forward (FP32 and BF16 outputs, GELU epilogue), data gradient through the adjoint
weights, weight and bias gradients, determinism, and a whole-model gradient check."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from xadvcool_b200 import surrogate as S

pytestmark = pytest.mark.gpu

SHAPES = [  # N, D, H, W, Ci, Co, ksize
    (1, 4, 6, 10, 16, 16, 3),
    (2, 5, 7, 9, 48, 32, 3),
    (1, 4, 8, 19, 192, 64, 3),
    (1, 3, 4, 6, 256, 128, 3),
    (2, 4, 6, 10, 16, 16, 1),
    (1, 3, 5, 7, 32, 48, 3),
    (1, 3, 4, 6, 64, 192, 3),
    (1, 2, 4, 5, 16, 144, 3),
    (1, 8, 32, 38, 64, 64, 3),     # many 128-voxel tiles, ragged last tile
    (2, 4, 16, 19, 128, 256, 3),
    (1, 3, 9, 11, 256, 48, 1),
    (1, 16, 32, 40, 16, 16, 3),
]


def _torch_w(w_bf, ksize):
    taps, Co, Ci = w_bf.shape
    k = 3 if ksize == 3 else 1
    return w_bf.float().view(k, k, k, Co, Ci).permute(3, 4, 0, 1, 2).contiguous()


def _ref_conv(x_bf, w_bf, b, ksize):
    xt = x_bf.float().permute(0, 4, 1, 2, 3)
    y = F.conv3d(xt, _torch_w(w_bf, ksize), b, padding=ksize // 2)
    return y.permute(0, 2, 3, 4, 1)


def _rand(shape, gen, scale=1.0):
    return (torch.randn(shape, generator=gen) * scale).cuda()


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_fp32_out(cuda, shape):
    N, D, H, W, Ci, Co, k = shape
    g = torch.Generator().manual_seed(1)
    x = _rand((N, D, H, W, Ci), g).to(S.BF16)
    w = _rand((27 if k == 3 else 1, Co, Ci), g, 0.1).to(S.BF16)
    b = _rand((Co,), g)
    y = S.conv_forward(x, w, b, k, out_fp32=True)
    assert S.kernel_status() == 0
    ref = _ref_conv(x, w, b, k)
    scale = (x.float().abs().amax() * w.float().abs().sum(dim=(0, 2)).amax()).item()
    # FP32 accumulation of exact BF16 products: only the summation order differs
    assert (y - ref).abs().max().item() <= 1e-5 * scale


@pytest.mark.parametrize("act", [0, 1])
def test_forward_bf16_out_and_gelu(cuda, act):
    N, D, H, W, Ci, Co, k = 2, 4, 6, 10, 32, 32, 3
    g = torch.Generator().manual_seed(2)
    x = _rand((N, D, H, W, Ci), g).to(S.BF16)
    w = _rand((27, Co, Ci), g, 0.05).to(S.BF16)
    b = _rand((Co,), g, 0.1)
    y = S.conv_forward(x, w, b, k, act=act)
    ref = _ref_conv(x, w, b, k)
    if act:
        ref = F.gelu(ref)
    assert y.dtype == torch.bfloat16
    # one BF16 rounding of the output: relative 2^-8
    err = (y.float() - ref).abs()
    assert (err <= 2.0 ** -8 * ref.abs() + 1e-3).all()


@pytest.mark.parametrize("shape", SHAPES)
def test_data_and_weight_grads(cuda, shape):
    N, D, H, W, Ci, Co, k = shape
    g = torch.Generator().manual_seed(3)
    x = _rand((N, D, H, W, Ci), g).to(S.BF16)
    w = _rand((27 if k == 3 else 1, Co, Ci), g, 0.1).to(S.BF16)
    dy = _rand((N, D, H, W, Co), g).to(S.BF16)
    # torch reference gradients in FP32 on the same BF16 operands
    xr = x.float().requires_grad_(True)
    wr = w.float().requires_grad_(True)
    br = torch.zeros(Co, device="cuda", requires_grad=True)
    yr = _ref_conv(xr, wr, br, k)
    yr.backward(dy.float())
    dx = S.conv_forward(dy, S.adjoint_weights(w), None, k, out_fp32=True)
    dw, db = S.conv_weight_grad(x, dy, k, True)
    sx = (dy.float().abs().amax() * w.float().abs().sum(dim=(0, 1)).amax()).item()
    assert (dx - xr.grad).abs().max().item() <= 1e-5 * sx
    V = N * D * H * W
    sw = (dy.float().abs().amax() * x.float().abs().amax()).item() * V
    # the weight-gradient kernel rounds nothing: BF16 operands, FP32 sums in a different order
    assert (dw - wr.grad).abs().max().item() <= 1e-6 * sw
    assert (db - br.grad).abs().max().item() <= 1e-6 * dy.float().abs().amax().item() * V


def test_weight_grad_deterministic(cuda):
    g = torch.Generator().manual_seed(4)
    x = _rand((2, 8, 16, 40, 32), g).to(S.BF16)
    dy = _rand((2, 8, 16, 40, 16), g).to(S.BF16)
    a = S.conv_weight_grad(x, dy, 3, True)
    b = S.conv_weight_grad(x, dy, 3, True)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_rejects_bad_channels(cuda):
    from xadvcool_b200._capi import XacError
    x = torch.zeros((1, 2, 2, 2, 8), dtype=S.BF16, device="cuda")
    w = torch.zeros((27, 16, 8), dtype=S.BF16, device="cuda")
    with pytest.raises(XacError):
        S.conv_forward(x, w, None, 3)


def test_model_gradients_match_torch(cuda):
    """The whole network on the kernels vs the same network on torch's FP32 conv3d (same BF16 roundings)."""
    model = S.Surrogate("cuda", seed=0)
    g = torch.Generator().manual_seed(5)
    x = _rand((1, 8, 16, 24, 16), g).to(S.BF16)
    x[..., 3:] = 0
    tgt = _rand((1, 8, 16, 24, S.OUT_FIELDS), g)
    loss = F.mse_loss(model.forward(x)[..., :S.OUT_FIELDS], tgt)
    loss.backward()
    ours = {k: v.grad.clone() for k, v in model.params.items()}
    for v in model.params.values():
        v.grad = None
    loss_ref = F.mse_loss(model.forward(x, S.torch_conv3d)[..., :S.OUT_FIELDS], tgt)
    loss_ref.backward()
    assert abs(loss.item() - loss_ref.item()) <= 0.02 * loss_ref.item()
    for k, v in model.params.items():
        ref = v.grad
        if ref.abs().max() == 0:
            assert ours[k].abs().max() == 0, k
            continue
        cos = torch.nn.functional.cosine_similarity(ours[k].flatten(), ref.flatten(), dim=0).item()
        # BF16 activations and BF16 upstream gradients on the kernel path: gradients agree in direction
        assert cos > 0.98, (k, cos)


def test_training_reduces_loss(cuda):
    """AdamW steps on a fixed synthetic pair lower the loss (the whole training loop runs on the kernels)."""
    torch.manual_seed(0)
    model = S.Surrogate("cuda", seed=1)
    x = torch.zeros(1, 8, 16, 24, 16)
    x[..., 0] = (torch.rand(1, 8, 16, 24) > 0.4).float()
    x[..., 1] = torch.rand(1, 8, 16, 24)
    x = x.to(S.BF16).cuda()
    y = torch.zeros(1, 8, 16, 24, S.OUT_FIELDS, device="cuda")
    y[..., 0] = x[..., 0].float() * (1 + x[..., 1].float())
    y[..., 4] = x[..., 1].float() ** 2
    hist = S.train(model, [(x, y)], epochs=40, batch=1, lr=3e-3)
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.3 * hist[0], hist
