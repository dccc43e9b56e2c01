"""Learned warm start: a 3-D convolutional encoder-decoder that predicts the converged u, p, T of a cold-plate
design from its mask and heat map, so the solver can start from those fields instead of rest.

Architecture (after the reference's 3-D U-Net, benchmark/models/unet3d.py:11-125, resized): four levels with
16, 32, 64, 128 channels, two 3x3x3 convolution - GroupNorm - GELU units per level (unet3d.py:11-26), 2x
average pooling down, nearest 2x upsampling + skip concatenation up, and a 1x1 head. Weights are kept in FP32
(the optimiser's copy) and run in BF16. Every convolution - forward, data gradient and weight gradient - is
libxac.so's BF16 tensor-core implicit GEMM with FP32 accumulation (csrc/conv3d.cu). GroupNorm, pooling,
upsampling, concatenation, GELU, the loss and AdamW (benchmark/train.py:128-141) are torch tensor operations
around those kernels.

Volumes are channels-last, [batch][z][y][x][channel], x padded from 148 to 152 so three poolings divide it.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import torch
import torch.nn.functional as F

from . import _capi
from ._tensors import stream_ptr

BF16 = torch.bfloat16
IN_FEATURES = 3  # fluid indicator, heat map, inlet speed (x20)
OUT_FIELDS = 5   # ux/u_in, uy/u_in, uz/u_in, (rho-1)/u_in, (T - T_in)/heat_power
CH = (16, 32, 64, 128)


def _pad16(c):
    return (c + 15) // 16 * 16


# ------------------------------------------------------------------------------------------------ kernels
def _on_one_gpu(**tensors) -> None:
    """The convolution kernels take raw device pointers: every operand must be a CUDA tensor of one device (a host
    tensor would hand the kernel a host address)."""
    dev = None
    for name, t in tensors.items():
        if t is None:
            continue
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise ValueError(f"{name}: the convolution kernels need a CUDA tensor (there is no CPU path)")
        if dev is not None and t.device != dev:
            raise ValueError(f"{name}: on {t.device}, the other operands are on {dev}")
        dev = t.device


def conv_forward(x: torch.Tensor, w_bf: torch.Tensor, bias: torch.Tensor | None, ksize: int, act: int = 0,
                 out_fp32: bool = False) -> torch.Tensor:
    """x: [N,D,H,W,Ci] bf16; w_bf: [taps,Co,Ci] bf16; bias fp32 [Co] or None -> [N,D,H,W,Co]."""
    _on_one_gpu(x=x, w=w_bf, bias=bias)
    N, D, H, W, Ci = x.shape
    taps, Co, Ci_w = w_bf.shape
    assert Ci_w == Ci and taps == (27 if ksize == 3 else 1)
    x = x.contiguous()
    out = torch.empty((N, D, H, W, Co), dtype=torch.float32 if out_fp32 else BF16, device=x.device)
    _capi.call("xac_conv3d_forward", x.data_ptr(), N, D, H, W, Ci, w_bf.contiguous().data_ptr(),
               bias.data_ptr() if bias is not None else None, Co, ksize, act,
               None if out_fp32 else out.data_ptr(), out.data_ptr() if out_fp32 else None, stream_ptr(x.device))
    return out


def conv_weight_grad(x: torch.Tensor, dy: torch.Tensor, ksize: int, with_bias: bool):
    _on_one_gpu(x=x, dy=dy)
    N, D, H, W, Ci = x.shape
    Co = dy.shape[-1]
    taps = 27 if ksize == 3 else 1
    cnt = C.c_longlong()
    _capi.call("xac_conv3d_partial_floats", N, D, H, W, Ci, Co, ksize, C.byref(cnt))
    partial = torch.empty(int(cnt.value), dtype=torch.float32, device=x.device)
    dw = torch.empty((taps, Co, Ci), dtype=torch.float32, device=x.device)
    db = torch.empty(Co, dtype=torch.float32, device=x.device) if with_bias else None
    _capi.call("xac_conv3d_weight_grad", x.contiguous().data_ptr(), N, D, H, W, Ci, dy.contiguous().data_ptr(), Co,
               ksize, partial.data_ptr(), dw.data_ptr(), db.data_ptr() if db is not None else None,
               stream_ptr(x.device))
    return dw, db


def kernel_status() -> int:
    """Reads and clears the convolution kernels' device status (0: every bounded wait completed)."""
    v = C.c_int()
    _capi.call("xac_conv3d_status", C.byref(v))
    return int(v.value)


def adjoint_weights(w_bf: torch.Tensor) -> torch.Tensor:
    """Weights of the data gradient: flipped taps, input and output channels swapped."""
    return w_bf.flip(0).transpose(1, 2).contiguous()


class _Conv3d(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w, b, ksize, out_fp32):
        w_bf = w.to(BF16)
        ctx.save_for_backward(x, w_bf)
        ctx.ksize = ksize
        ctx.has_bias = b is not None
        return conv_forward(x, w_bf, b, ksize, out_fp32=out_fp32)

    @staticmethod
    def backward(ctx, dy):
        x, w_bf = ctx.saved_tensors
        dy = dy.to(BF16).contiguous()
        dx = conv_forward(dy, adjoint_weights(w_bf), None, ctx.ksize) if ctx.needs_input_grad[0] else None
        dw, db = conv_weight_grad(x, dy, ctx.ksize, ctx.has_bias)
        return dx, dw, db, None, None


def conv3d(x, w, b, ksize=3, out_fp32=False):
    """Differentiable convolution on the BF16 kernels; w is the FP32 master copy [taps, Co, Ci]."""
    return _Conv3d.apply(x, w, b, ksize, out_fp32)


def torch_conv3d(x, w, b, ksize=3, out_fp32=False):
    """Stand-in for :func:`conv3d` with torch's FP32 conv3d on the same BF16 roundings (test reference; runs on
    the CPU too): x [N,D,H,W,Ci] bf16, w [taps,Co,Ci] FP32 master weights."""
    taps, Co, Ci = w.shape
    k = 3 if ksize == 3 else 1
    wt = w.to(BF16).float().view(k, k, k, Co, Ci).permute(3, 4, 0, 1, 2)
    y = F.conv3d(x.float().permute(0, 4, 1, 2, 3), wt, b, padding=k // 2).permute(0, 2, 3, 4, 1)
    return y if out_fp32 else y.to(BF16)


# ------------------------------------------------------------------------------------------------ model
class Surrogate:
    """The encoder-decoder; parameters are FP32 tensors (w: [taps, Co, Ci], b: [Co])."""

    def __init__(self, device="cuda", seed=0):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        self.params = {}

        def layer(name, ci, co, k=3):
            taps = 27 if k == 3 else 1
            fan_in = taps * ci
            w = torch.randn((taps, _pad16(co), _pad16(ci)), generator=g) * math.sqrt(2.0 / fan_in)
            w[:, co:, :] = 0.0
            w[:, :, ci:] = 0.0
            self.params[name + ".w"] = w.to(self.device).requires_grad_(True)
            self.params[name + ".b"] = torch.zeros(_pad16(co), device=self.device).requires_grad_(True)
            if k == 3:  # GroupNorm scale and shift
                self.params[name + ".g"] = torch.ones(co, device=self.device).requires_grad_(True)
                self.params[name + ".s"] = torch.zeros(co, device=self.device).requires_grad_(True)

        c0, c1, c2, c3 = CH
        layer("e0a", IN_FEATURES, c0)
        layer("e0b", c0, c0)
        layer("e1a", c0, c1)
        layer("e1b", c1, c1)
        layer("e2a", c1, c2)
        layer("e2b", c2, c2)
        layer("b3a", c2, c3)
        layer("b3b", c3, c3)
        layer("d2a", c3 + c2, c2)
        layer("d2b", c2, c2)
        layer("d1a", c2 + c1, c1)
        layer("d1b", c1, c1)
        layer("d0a", c1 + c0, c0)
        layer("d0b", c0, c0)
        layer("head", c0, OUT_FIELDS, k=1)
        self.norm = None  # per-channel (mean, std) of the targets

    def parameters(self):
        return list(self.params.values())

    @staticmethod
    def groups(c):
        return max(1, min(8, c // 4))

    def _unit(self, x, name, conv):
        """conv -> GroupNorm -> GELU, channels-last, normalisation in FP32."""
        y = conv(x, self.params[name + ".w"], self.params[name + ".b"], 3, False)
        N, C = y.shape[0], y.shape[-1]
        G = self.groups(C)
        h = y.float().reshape(N, -1, G, C // G)
        mean = h.mean(dim=(1, 3), keepdim=True)
        var = h.var(dim=(1, 3), unbiased=False, keepdim=True)
        h = ((h - mean) * torch.rsqrt(var + 1e-5)).reshape(y.shape)
        return F.gelu(h * self.params[name + ".g"] + self.params[name + ".s"]).to(BF16)

    def _block(self, x, name, conv):
        return self._unit(self._unit(x, name + "a", conv), name + "b", conv)

    @staticmethod
    def _pool(x):
        N, D, H, W, Cc = x.shape
        return x.view(N, D // 2, 2, H // 2, 2, W // 2, 2, Cc).float().mean(dim=(2, 4, 6)).to(BF16)

    @staticmethod
    def _up(x):
        N, D, H, W, Cc = x.shape
        return x[:, :, None, :, None, :, None, :].expand(N, D, 2, H, 2, W, 2, Cc).reshape(N, 2 * D, 2 * H, 2 * W, Cc)

    def forward(self, x, conv=None):
        """x: [N, 32, 128, 152, 16] bf16 features -> [N, 32, 128, 152, 16] fp32 (first 5 channels used).

        ``conv(x, w, b, ksize, out_fp32)`` defaults to the tensor-core kernels (:func:`conv3d`); tests pass a
        torch stand-in to check the rest of the network against them."""
        conv = conv or conv3d
        e0 = self._block(x, "e0", conv)
        e1 = self._block(self._pool(e0), "e1", conv)
        e2 = self._block(self._pool(e1), "e2", conv)
        b3 = self._block(self._pool(e2), "b3", conv)
        d2 = self._block(torch.cat([self._up(b3), e2], dim=-1), "d2", conv)
        d1 = self._block(torch.cat([self._up(d2), e1], dim=-1), "d1", conv)
        d0 = self._block(torch.cat([self._up(d1), e0], dim=-1), "d0", conv)
        return conv(d0, self.params["head.w"], self.params["head.b"], 1, True)

    def state_dict(self):
        sd = {k: v.detach().cpu() for k, v in self.params.items()}
        if self.norm is not None:
            sd["norm.mean"], sd["norm.std"] = (t.cpu() for t in self.norm)
        return sd

    def load_state_dict(self, sd):
        for k, v in sd.items():
            if k.startswith("norm."):
                continue
            self.params[k] = v.to(self.device).requires_grad_(True)
        if "norm.mean" in sd:
            self.norm = (sd["norm.mean"].to(self.device), sd["norm.std"].to(self.device))


WEIGHTS = Path(__file__).resolve().parent / "weights" / "surrogate_gyroid148.pt"


def save_weights(model: Surrogate, path=WEIGHTS):
    """Convolution weights in BF16 (the precision the kernels read them in), everything else in FP32."""
    sd = {k: (v.to(BF16) if k.endswith(".w") else v) for k, v in model.state_dict().items()}
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    torch.save(sd, path)


def load_pretrained(device="cuda", path=WEIGHTS) -> Surrogate:
    """The surrogate trained on the seeded 148x128x32 gyroid cold plates (python -m xadvcool_b200.warmstart)."""
    if not Path(path).exists():
        raise FileNotFoundError(f"no trained surrogate weights at {path}")
    m = Surrogate(device)
    m.load_state_dict({k: (v.float() if k.endswith(".w") else v) for k, v in torch.load(path).items()})
    return m


# ------------------------------------------------------------------------------------------------ data
NXP = 152


BC_SOLID, BC_INLET = 1, 2


def _dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(device)


def features(mask: np.ndarray, heat_source: np.ndarray | None, u_in: float, device="cuda") -> torch.Tensor:
    """[1, nz, ny, 152, 16] bf16 input volume from a reference-layout design, assembled on the device: fluid
    indicator, heat map normalised to max 1 (z=0 floor when absent, as src/simulation.py:79-85), 20 u_in; x is
    padded with solid."""
    nx, ny, nz = mask.shape
    x = torch.zeros((1, nz, ny, NXP, 16), dtype=BF16, device=device)
    x[0, :, :, :nx, 0] = (_dev(mask, np.int32, device) != BC_SOLID).permute(2, 1, 0).to(BF16)
    if heat_source is not None:
        h = _dev(heat_source, np.float32, device)
        x[0, :, :, :nx, 1] = (h / h.max().clamp_min(1e-30)).permute(2, 1, 0).to(BF16)
    else:
        x[0, 0, :, :nx, 1] = 1.0
    x[..., 2] = 20.0 * u_in
    return x


def targets(rho: torch.Tensor, u: torch.Tensor, T: torch.Tensor, u_in: float, heat_power: float, t_in=25.0):
    """Raw fields (reference layout) -> [1, nz, ny, 152, 5] fp32 scaled targets."""
    nx = rho.shape[0]
    out = torch.zeros((1, rho.shape[2], rho.shape[1], NXP, OUT_FIELDS), device=rho.device)
    out[0, :, :, :nx, 0:3] = u.permute(2, 1, 0, 3) / u_in
    out[0, :, :, :nx, 3] = (rho.permute(2, 1, 0) - 1.0) / u_in
    out[0, :, :, :nx, 4] = (T.permute(2, 1, 0) - t_in) / heat_power
    return out


def fields_from_prediction(pred: torch.Tensor, shape, u_in: float, heat_power: float, mask: np.ndarray,
                           t_in=25.0, mask_dev: torch.Tensor | None = None):
    """Prediction [1, nz, ny, 152, >=5] (denormalised scaled targets) -> rho, u, T in the reference layout.

    Solid cells get rho = 1, u = 0. Inlet cells get the cold-start state rho = 1, u = 0, T = t_in
    (src/simulation.py:63-73): the velocity inlet rebuilds its populations from its own post-collision values
    only (fluid_engine3d.py:196-224), so its density keeps a memory of its initial value that sets the inflow
    mass flux for the whole solve. Starting it exactly as a cold start does makes its trajectory, and so the
    converged delta_P, the cold solve's."""
    nx, ny, nz = shape
    p = pred[0, :, :, :nx, :OUT_FIELDS].permute(2, 1, 0, 3)  # [nx, ny, nz, 5]
    u = (p[..., 0:3] * u_in).contiguous()
    rho = (1.0 + p[..., 3] * u_in).contiguous()
    T = (t_in + p[..., 4] * heat_power).contiguous()
    m = mask_dev if mask_dev is not None else _dev(mask, np.int32, pred.device)
    solid, inlet = m == BC_SOLID, m == BC_INLET
    u[solid | inlet] = 0.0
    rho[solid | inlet] = 1.0
    T[inlet] = t_in
    return rho.float(), u.float(), T.float()


def predict(model: Surrogate, mask, heat_source, u_in, heat_power, device="cuda"):
    """Warm-start fields for one design (reference layout)."""
    with torch.no_grad():
        x = features(mask, heat_source, u_in, device)
        y = model.forward(x)[..., :OUT_FIELDS]
        mean, std = model.norm
        y = y * std + mean
        return fields_from_prediction(y, mask.shape, u_in, heat_power, mask)


def train(model: Surrogate, samples, epochs=20, batch=2, lr=5e-4, weight_decay=1e-4, clip=1.0, log=None, conv=None):
    """samples: list of (features [1,...,16] bf16, targets [1,...,5] fp32) on the device. AdamW with a one-cycle
    schedule, MSE on normalised targets, gradient-norm clipping."""
    tgt = torch.cat([t for _, t in samples], 0)
    mean = tgt.mean(dim=(0, 1, 2, 3))
    std = tgt.std(dim=(0, 1, 2, 3)).clamp_min(1e-6)
    model.norm = (mean, std)
    opt = torch.optim.AdamW(model.parameters(), lr=lr, weight_decay=weight_decay)
    steps = epochs * math.ceil(len(samples) / batch)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=steps, pct_start=0.1)
    g = torch.Generator().manual_seed(0)
    hist = []
    for ep in range(epochs):
        order = torch.randperm(len(samples), generator=g).tolist()
        tot = 0.0
        for i in range(0, len(order), batch):
            idx = order[i:i + batch]
            x = torch.cat([samples[k][0] for k in idx], 0)
            y = (torch.cat([samples[k][1] for k in idx], 0) - mean) / std
            pred = model.forward(x, conv)[..., :OUT_FIELDS]
            loss = F.mse_loss(pred, y)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            if clip:
                torch.nn.utils.clip_grad_norm_(model.parameters(), clip)
            opt.step()
            sched.step()
            tot += float(loss.detach()) * len(idx)
        hist.append(tot / len(samples))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return hist
