// Fused step kernels with __nv_bfloat16 fluid populations and __half thermal populations (see step_kernels.cuh):
// BF16's 8-bit significand is used for the fluid lattice only.
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<__nv_bfloat16, __half>(const StepLaunch&);
}  // namespace xac
