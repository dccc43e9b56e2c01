// Dispatch of the fused step over compile-time row lengths (each instantiation makes every population offset
// an immediate). Included once per storage type by step_f32.cu / step_f16.cu / step_bf16.cu, which compile in
// parallel.
#pragma once

#include "lattice_kernels.cuh"

namespace xac {

template <typename S, bool kMacro, bool kOwn>
void launch_step_rows(const StepLaunch& a) {
  const unsigned grid = (unsigned)(((long long)a.p.g.rows * a.p.g.pitch + a.block - 1) / a.block);
#define XAC_STEP(KT)                                                                                               \
  coupled_step_kernel<S, kMacro, kOwn, KT><<<grid, a.block, 0, a.stream>>>(                                     \
      (const S*)a.Pin, (S*)a.Pout, (const S*)a.Qin, (S*)a.Qout, a.link, a.qsrc, a.u_in, a.rho, a.ux, a.uy, a.uz, \
      a.T0, a.p)
  switch (a.p.g.pitch) {
    case 32: XAC_STEP(32); break;
    case 64: XAC_STEP(64); break;
    case 96: XAC_STEP(96); break;
    case 128: XAC_STEP(128); break;
    case 160: XAC_STEP(160); break;
    case 192: XAC_STEP(192); break;
    case 224: XAC_STEP(224); break;
    case 256: XAC_STEP(256); break;
    default: XAC_STEP(0);
  }
#undef XAC_STEP
}

template <typename S>
void launch_coupled_step(const StepLaunch& a) {
  if (a.macro && a.own) launch_step_rows<S, true, true>(a);
  else if (a.macro) launch_step_rows<S, true, false>(a);
  else if (a.own) launch_step_rows<S, false, true>(a);
  else launch_step_rows<S, false, false>(a);
}

}  // namespace xac
