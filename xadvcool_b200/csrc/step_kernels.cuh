// Dispatch of the fused step over compile-time row lengths (each instantiation makes every thermal population
// offset an immediate). Included once per storage mode (fluid storage SP, thermal storage SQ) by step_f32.cu /
// step_f16.cu / step_bf16.cu / step_f32t16.cu, which compile in parallel.
#pragma once

#include "lattice_kernels.cuh"

namespace xac {

template <typename SP, typename SQ, bool kMacro, bool kOwn>
void launch_step_rows(const StepLaunch& a) {
  const unsigned grid = (unsigned)(((long long)a.p.g.rows * a.p.g.pitch + a.block - 1) / a.block);
  if (a.variant == 1 && a.p.g.pitch >= 64 && a.p.g.pitch <= 256) {
    // one block per row; the kernel's compile-time row length is its block size
#define XAC_QSTAGE(KT)                                                                                             \
  coupled_qstage_kernel<SP, SQ, kMacro, kOwn, KT><<<(unsigned)a.p.g.rows, KT, StageQ<SQ, KT>::kLen * sizeof(SQ), \
                                                   a.stream>>>(                                                   \
      (const SP*)a.Pin, (SP*)a.Pout, (const SQ*)a.Qin, (SQ*)a.Qout, a.link, a.qsrc, a.u_in, a.rho, a.ux, a.uy,     \
      a.uz, a.T0, a.p)
    switch (a.p.g.pitch) {
      case 64: XAC_QSTAGE(64); return;
      case 96: XAC_QSTAGE(96); return;
      case 128: XAC_QSTAGE(128); return;
      case 160: XAC_QSTAGE(160); return;
      case 192: XAC_QSTAGE(192); return;
      case 224: XAC_QSTAGE(224); return;
      case 256: XAC_QSTAGE(256); return;
      default: break;
    }
#undef XAC_QSTAGE
  }
#define XAC_STEP(KT)                                                                                               \
  coupled_step_kernel<SP, SQ, kMacro, kOwn, KT><<<grid, a.block, 0, a.stream>>>(                               \
      (const SP*)a.Pin, (SP*)a.Pout, (const SQ*)a.Qin, (SQ*)a.Qout, a.link, a.qsrc, a.u_in, a.rho, a.ux, a.uy,     \
      a.uz, a.T0, a.p)
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

template <typename SP, typename SQ>
void launch_coupled_step(const StepLaunch& a) {
  if (a.macro && a.own) launch_step_rows<SP, SQ, true, true>(a);
  else if (a.macro) launch_step_rows<SP, SQ, true, false>(a);
  else if (a.own) launch_step_rows<SP, SQ, false, true>(a);
  else launch_step_rows<SP, SQ, false, false>(a);
}

}  // namespace xac
