// Shared definitions of libxac.so: D3Q19 constants, error plumbing, launch helpers.
// The direction order, weights and opposite map follow src/fluid_engine3d.py:11-53.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/xac.h"

namespace xac {

constexpr int kQ = 19;
enum : int { kFluid = XAC_BC_FLUID, kSolid = XAC_BC_SOLID, kInlet = XAC_BC_INLET, kOutlet = XAC_BC_OUTLET };

// src/fluid_engine3d.py:19-39
__host__ __device__ constexpr int ex_of(int i) {
  constexpr int t[kQ] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  return t[i];
}
__host__ __device__ constexpr int ey_of(int i) {
  constexpr int t[kQ] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
  return t[i];
}
__host__ __device__ constexpr int ez_of(int i) {
  constexpr int t[kQ] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  return t[i];
}
// src/fluid_engine3d.py:51-53
__host__ __device__ constexpr int opp_of(int i) {
  constexpr int t[kQ] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
  return t[i];
}
// weight class: 0 rest (1/3), 1 face (1/18), 2 edge (1/36); src/fluid_engine3d.py:42-47
__host__ __device__ constexpr int wclass_of(int i) { return i == 0 ? 0 : (i < 7 ? 1 : 2); }

// The reference builds W_CONST from Python doubles and stores float32; these are those roundings.
__device__ __forceinline__ float w_of(int i) {
  return wclass_of(i) == 0 ? (float)(1.0 / 3.0) : (wclass_of(i) == 1 ? (float)(1.0 / 18.0) : (float)(1.0 / 36.0));
}

// e_i . u exactly as the reference evaluates float(ex)*ux + float(ey)*uy + float(ez)*uz: products with 0 are
// dropped (they only change the sign of a zero sum), products with +-1 are exact.
template <int I>
__device__ __forceinline__ float edotu(float ux, float uy, float uz) {
  constexpr int a = ex_of(I), b = ey_of(I), c = ez_of(I);
  float s = 0.0f;
  bool have = false;
  if (a != 0) { s = a > 0 ? ux : -ux; have = true; }
  if (b != 0) { float t = b > 0 ? uy : -uy; s = have ? s + t : t; have = true; }
  if (c != 0) { float t = c > 0 ? uz : -uz; s = have ? s + t : t; have = true; }
  return s;
}

// Second-order equilibrium, reference operand order: (w*rho) * (((1 + 3eu) + 4.5eu^2) - 1.5usq).
__device__ __forceinline__ float feq_term(float w_rho, float eu, float usq15) {
  return w_rho * (((1.0f + 3.0f * eu) + 4.5f * (eu * eu)) - usq15);
}

// Thread-local error message behind xac_last_error().
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define XAC_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return ::xac::cuda_status(_e, #call); \
  } while (0)

#define XAC_REQUIRE(cond, ...)       \
  do {                               \
    if (!(cond)) {                   \
      ::xac::set_error(__VA_ARGS__); \
      return XAC_EINVAL;             \
    }                                \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace xac
