"""Argument checking between torch CUDA tensors and the C ABI (raw device pointers)."""
from __future__ import annotations

import torch


def dev_ptr(t: torch.Tensor, dtype: torch.dtype, name: str, shape=None) -> int:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch.Tensor, got {type(t).__name__}")
    if not t.is_cuda:
        raise ValueError(f"{name}: must be a CUDA tensor (the solver has no CPU path)")
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name}: expected shape {tuple(shape)}, got {tuple(t.shape)}")
    return t.data_ptr()


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def dims3(t: torch.Tensor, name: str):
    if t.dim() != 3:
        raise ValueError(f"{name}: expected a 3-D (nx, ny, nz) tensor, got shape {tuple(t.shape)}")
    return tuple(int(s) for s in t.shape)
