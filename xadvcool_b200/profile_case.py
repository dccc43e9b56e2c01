"""A small, repeatable profiling case for the fused step: the 148x128x32 gyroid (seed 0) in a developed state.

    python -m xadvcool_b200.profile_case --save state.bin            # 4000 steps, then save the state
    python -m xadvcool_b200.profile_case --load state.bin --steps 2  # restore, then 2 steps in a profiler range

    python -m xadvcool_b200.profile_case --warm 1 --steps 1 --chunk 100  # one step, then one 100-step call

The third form runs the step loop as the solver does (100 steps per call, one CUDA graph), for captures of the
DRAM traffic per launch with L2 as the previous step left it.

The second form launches only a handful of small kernels before the profiled range
(cudaProfilerStart/Stop), so a profiler attached with --profile-from-start off sees a developed-flow step
after few prior launches.

    python -m xadvcool_b200.profile_case --conv b3b --steps 2   # one surrogate convolution layer, batch 4

runs the named layer of the warm-start surrogate (forward convolution on the tensor-core kernel, the 148x128x32
volume padded to 152 in x) inside the profiler range, after one untimed launch.
"""
from __future__ import annotations

import argparse

import torch

from . import designs
from .lattice import Lattice


CONV_LAYERS = {  # name: (D, H, W, Ci, Co) at batch 4
    "e0b": (32, 128, 152, 16, 16), "e1b": (16, 64, 76, 32, 32), "e2b": (8, 32, 38, 64, 64),
    "b3b": (4, 16, 19, 128, 128), "d2a": (8, 32, 38, 192, 64), "d0a": (32, 128, 152, 48, 16),
}


def conv_case(name, steps):
    from . import surrogate as S
    D, H, W, Ci, Co = CONV_LAYERS[name]
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((4, D, H, W, Ci), device="cuda", generator=g).to(S.BF16)
    w = (torch.randn((27, Co, Ci), device="cuda", generator=g) * 0.05).to(S.BF16)
    b = torch.zeros(Co, device="cuda")
    S.conv_forward(x, w, b, 3)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(steps):
        y = S.conv_forward(x, w, b, 3)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(f"conv case {name}: {tuple(y.shape)}, status {S.kernel_status()}")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--save")
    ap.add_argument("--load")
    ap.add_argument("--warm", type=int, default=4000)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--chunk", type=int, default=1, help="steps per call inside the profiled range")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--block", type=int, default=128)
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--conv", choices=sorted(CONV_LAYERS), help="profile one surrogate convolution layer instead")
    a = ap.parse_args(argv)
    if a.conv:
        conv_case(a.conv, a.steps)
        return
    mask, hs, u_in, _ = designs.gyroid_design(0)
    lat = Lattice(mask, heat_source=hs, tau_fluid=0.55, u_inlet_val=u_in, precision=a.precision)
    lat.tune(a.block, a.variant)
    if a.load:
        with open(a.load, "rb") as f:
            lat.load_state(f.read())
    else:
        lat.step(a.warm)
    if a.save:
        with open(a.save, "wb") as f:
            f.write(lat.save_state())
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(a.steps):
        lat.step(a.chunk)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    st = lat.stats()
    print(f"profile case: step {lat.steps_done}, max|u| {st[0]:.4f}, max T {st[11]:.3f}")


if __name__ == "__main__":
    main()
