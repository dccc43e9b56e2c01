// Device kernels of the fused lattice (internal layout).
//
// Internal layout: cell c = (z*ny + y)*nx + x (x fastest, the flow/streaming axis); populations are
// structure-of-arrays planes pop[i*N + c], N = cell count rounded up to 64 (256-byte aligned planes).
//
// Scheme. Both lattices store POST-COLLISION populations and every step is one pull pass:
//   fluid:   F^k(x)   = stream(P^{k-1})(x)  ->  rho^k, u^k  ->  P^k(x) = collide(F^k)
//   thermal: G^{k-1}(x) = tstream(Q^{k-1})(x) -> T^{k-1} -> Q^k(x) = tcollide(G^{k-1}, u^k, T^{k-1})
// which reproduces the reference order of one graph replay (src/simulation.py:93-100): its thermal
// collision of step k uses u after this step's fluid streaming and T of the previous step. The very
// first step reads the initial thermal populations G^0 unstreamed (kOwn).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "xac_internal.cuh"

namespace xac {

// ---- packed per-cell link word -------------------------------------------------------------
// bits 0..18 : fluid pull of direction i bounces back (source out of the domain or solid)
// bits 20..21: cell label (XAC_BC_*)
// bit  22    : heated (heat_source * heat_power > 0)
constexpr int kTypeShift = 20;
constexpr uint32_t kHeatedBit = 1u << 22;
__device__ __forceinline__ int link_type(uint32_t lw) { return (int)((lw >> kTypeShift) & 3u); }

struct Geom {
  int nx, ny, nz;
  long long ncell;  // nx*ny*nz
  long long N;      // population plane stride (elements)
};

// ---- population storage -------------------------------------------------------------------
// FP32 stores the population itself. The 16-bit forms store the deviation from the rest
// equilibrium w_i*ref (ref = 1 for the fluid, T_inlet for the thermal lattice) and do all
// arithmetic in float32.
template <typename S>
struct Pop;
template <>
struct Pop<float> {
  static __device__ __forceinline__ float ld(const float* p, float) { return __ldg(p); }
  static __device__ __forceinline__ void st(float* p, float v, float) { *p = v; }
};
template <>
struct Pop<__half> {
  static __device__ __forceinline__ float ld(const __half* p, float base) { return __half2float(__ldg(p)) + base; }
  static __device__ __forceinline__ void st(__half* p, float v, float base) { *p = __float2half_rn(v - base); }
};
template <>
struct Pop<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p, float base) {
    return __bfloat162float(__ldg(p)) + base;
  }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float v, float base) {
    *p = __float2bfloat16_rn(v - base);
  }
};

struct StepParams {
  Geom g;
  float tau_f;    // fluid tau
  float tau_tf;   // thermal tau in fluid
  float tau_ts;   // thermal tau in solid
  float T_in;     // inlet temperature (thermal_engine3d.py:151)
  float rho_out;  // outlet density (simulation.py:61)
  float T_ref;    // thermal rest reference for 16-bit storage
};

// Equilibrium for all 19 directions with reference operand order, collision into out[].
#define XAC_FOR19(M) M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16) M(17) M(18)

template <typename S, bool kMacro, bool kOwn>
__global__ void __launch_bounds__(256) coupled_step_kernel(const S* __restrict__ Pin, S* __restrict__ Pout,
                                                           const S* __restrict__ Qin, S* __restrict__ Qout,
                                                           const uint32_t* __restrict__ link,
                                                           const float* __restrict__ qsrc,
                                                           const float* __restrict__ u_in_ptr,
                                                           float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                           float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                           const float* __restrict__ T0, StepParams p) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= p.g.ncell) return;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz;
  const long long nxy = (long long)nx * ny;
  const long long N = p.g.N;
  const int x = (int)(c % nx);
  const long long t = c / nx;
  const int y = (int)(t % ny);
  const int z = (int)(t / ny);
  const uint32_t lw = __ldg(link + c);
  const int type = link_type(lw);

  float ux = 0.0f, uy = 0.0f, uz = 0.0f;

  // ------------------------------------------------------------------ fluid lattice
  if (type != kSolid) {
    float F[kQ];
    if (type == kInlet) {
      // src/fluid_engine3d.py:197-244: no pull; unknown populations from the known ones
      float k[kQ];
#define XAC_LD_OWN(I) k[I] = Pop<S>::ld(Pin + (long long)I * N + c, w_of(I));
      XAC_FOR19(XAC_LD_OWN)
#undef XAC_LD_OWN
      const float ux_in = __ldg(u_in_ptr);
      const float rn = (((((((((k[0] + k[3]) + k[4]) + k[5]) + k[6]) + k[15]) + k[16]) + k[17]) + k[18]) +
                         2.0f * ((((k[2] + k[8]) + k[10]) + k[12]) + k[14])) /
                        (1.0f - ux_in);
      const float c23 = 2.0f / 3.0f, c16 = 1.0f / 6.0f;
      F[0] = k[0];
      F[1] = k[2] + (c23 * rn) * ux_in;
      F[2] = k[2];
      F[3] = k[3];
      F[4] = k[4];
      F[5] = k[5];
      F[6] = k[6];
      F[7] = k[10] + (c16 * rn) * ux_in;
      F[8] = k[8];
      F[9] = k[8] + (c16 * rn) * ux_in;
      F[10] = k[10];
      F[11] = k[14] + (c16 * rn) * ux_in;
      F[12] = k[12];
      F[13] = k[12] + (c16 * rn) * ux_in;
      F[14] = k[14];
      F[15] = k[15];
      F[16] = k[16];
      F[17] = k[17];
      F[18] = k[18];
    } else if (type == kOutlet) {
      // src/fluid_engine3d.py:247-259: copy post-collision (x-1) and rescale to rho_outlet
      const long long s = x > 0 ? c - 1 : c;
      float sum = 0.0f;
#define XAC_LD_OUT(I)                                     \
  F[I] = Pop<S>::ld(Pin + (long long)I * N + s, w_of(I)); \
  sum += F[I];
      XAC_FOR19(XAC_LD_OUT)
#undef XAC_LD_OUT
      if (sum > 1e-6f) {
        const float sc = p.rho_out / sum;
#pragma unroll
        for (int i = 0; i < kQ; ++i) F[i] *= sc;
      }
    } else {
      // src/fluid_engine3d.py:262-272: pull, halfway bounce-back on out-of-domain or solid sources
#define XAC_LD_PULL(I)                                                                                      \
  {                                                                                                         \
    constexpr int o = opp_of(I);                                                                            \
    const long long off = (long long)ex_of(I) + (long long)ey_of(I) * nx + (long long)ez_of(I) * nxy;       \
    const S* src = ((lw >> I) & 1u) ? (Pin + (long long)o * N + c) : (Pin + (long long)I * N + c - off);    \
    F[I] = Pop<S>::ld(src, w_of(I));                                                                        \
  }
      XAC_FOR19(XAC_LD_PULL)
#undef XAC_LD_PULL
    }
    // src/fluid_engine3d.py:85-113 moments, reference summation order
    float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      r += F[i];
      if (ex_of(i) != 0) mx += ex_of(i) > 0 ? F[i] : -F[i];
      if (ey_of(i) != 0) my += ey_of(i) > 0 ? F[i] : -F[i];
      if (ez_of(i) != 0) mz += ez_of(i) > 0 ? F[i] : -F[i];
    }
    if (r > 1e-10f) {
      ux = mx / r;
      uy = my / r;
      uz = mz / r;
    }
    if (kMacro) {
      rho_o[c] = r;
      ux_o[c] = ux;
      uy_o[c] = uy;
      uz_o[c] = uz;
    }
    // src/fluid_engine3d.py:157-173 BGK with the equilibrium in registers
    const float omega = 1.0f / p.tau_f;
    const float usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#define XAC_COLLIDE(I)                                                               \
  {                                                                                  \
    const float fe = feq_term(w_of(I) * r, edotu<I>(ux, uy, uz), usq15);            \
    Pop<S>::st(Pout + (long long)I * N + c, F[I] - omega * (F[I] - fe), w_of(I));    \
  }
    XAC_FOR19(XAC_COLLIDE)
#undef XAC_COLLIDE
  } else if (kMacro) {
    // solid populations are never streamed (fluid_engine3d.py:193-194): moments of the frozen values
    float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const float v = Pop<S>::ld(Pin + (long long)i * N + c, w_of(i));
      r += v;
      if (ex_of(i) != 0) mx += ex_of(i) > 0 ? v : -v;
      if (ey_of(i) != 0) my += ey_of(i) > 0 ? v : -v;
      if (ez_of(i) != 0) mz += ez_of(i) > 0 ? v : -v;
    }
    rho_o[c] = r;
    ux_o[c] = r > 1e-10f ? mx / r : 0.0f;
    uy_o[c] = r > 1e-10f ? my / r : 0.0f;
    uz_o[c] = r > 1e-10f ? mz / r : 0.0f;
  }

  // ------------------------------------------------------------------ thermal lattice
  const float Tb = p.T_ref;
  float G[kQ];
  float T;
  if (kOwn) {
#define XAC_LD_G0(I) G[I] = Pop<S>::ld(Qin + (long long)I * N + c, w_of(I) * Tb);
    XAC_FOR19(XAC_LD_G0)
#undef XAC_LD_G0
    T = __ldg(T0 + c);
  } else {
    if (type == kInlet) {
      // src/thermal_engine3d.py:160-165
#pragma unroll
      for (int i = 0; i < kQ; ++i) G[i] = w_of(i) * p.T_in;
    } else if (type == kOutlet) {
      // src/thermal_engine3d.py:170-177
      const long long s = x > 0 ? c - 1 : c;
#define XAC_LD_GOUT(I) G[I] = Pop<S>::ld(Qin + (long long)I * N + s, w_of(I) * Tb);
      XAC_FOR19(XAC_LD_GOUT)
#undef XAC_LD_GOUT
    } else {
      // src/thermal_engine3d.py:180-211: pull; x<0 sources are the inlet equilibrium, x>=nx sources copy the
      // own value, other out-of-domain sources bounce back (adiabatic walls)
#define XAC_LD_GPULL(I)                                                                                        \
  {                                                                                                            \
    constexpr int a = ex_of(I), b = ey_of(I), d = ez_of(I);                                                    \
    const bool xlo = (a == 1 && x == 0);                                                                       \
    const bool xhi = (a == -1 && x == nx - 1);                                                                 \
    const bool wall = (b == 1 && y == 0) || (b == -1 && y == ny - 1) || (d == 1 && z == 0) ||                 \
                      (d == -1 && z == nz - 1);                                                                \
    const long long off = (long long)a + (long long)b * nx + (long long)d * nxy;                               \
    /* the address is always in bounds: x<0 sources read the own cell and the value is replaced */         \
    const S* src = (xhi || xlo) ? (Qin + (long long)I * N + c)                                                 \
                                : (wall ? (Qin + (long long)opp_of(I) * N + c) : (Qin + (long long)I * N + c - off)); \
    const float v = Pop<S>::ld(src, w_of(I) * Tb);                                                             \
    G[I] = xlo ? w_of(I) * p.T_in : v;                                                                         \
  }
      XAC_FOR19(XAC_LD_GPULL)
#undef XAC_LD_GPULL
    }
    // src/thermal_engine3d.py:214-224
    T = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += G[i];
  }
  // src/thermal_engine3d.py:105-145: tau by phase, u = 0 in solids, source w_i (1 - omega/2) q
  const bool solid = type == kSolid;
  const float omega_t = 1.0f / (solid ? p.tau_ts : p.tau_tf);
  const float srcf = 1.0f - 0.5f * omega_t;
  const float q = (lw & kHeatedBit) ? __ldg(qsrc + c) : 0.0f;
  if (solid) {
    ux = 0.0f;
    uy = 0.0f;
    uz = 0.0f;
  }
  const float usq15t = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#define XAC_TCOLLIDE(I)                                                          \
  {                                                                              \
    const float ge = feq_term(w_of(I) * T, edotu<I>(ux, uy, uz), usq15t);       \
    float v = G[I] - omega_t * (G[I] - ge);                                      \
    if (q > 0.0f) v += (w_of(I) * srcf) * q;                                     \
    Pop<S>::st(Qout + (long long)I * N + c, v, w_of(I) * Tb);                    \
  }
  XAC_FOR19(XAC_TCOLLIDE)
#undef XAC_TCOLLIDE
}

// T^k = sum of the streamed thermal populations, without storing them (stats / field export steps).
template <typename S>
__global__ void __launch_bounds__(256) thermal_finalize_kernel(const S* __restrict__ Qin,
                                                               const uint32_t* __restrict__ link,
                                                               float* __restrict__ T_o, StepParams p) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= p.g.ncell) return;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz;
  const long long nxy = (long long)nx * ny;
  const long long N = p.g.N;
  const int x = (int)(c % nx);
  const long long t = c / nx;
  const int y = (int)(t % ny);
  const int z = (int)(t / ny);
  const int type = link_type(__ldg(link + c));
  const float Tb = p.T_ref;
  float T = 0.0f;
  if (type == kInlet) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += w_of(i) * p.T_in;
  } else if (type == kOutlet) {
    const long long s = x > 0 ? c - 1 : c;
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += Pop<S>::ld(Qin + (long long)i * N + s, w_of(i) * Tb);
  } else {
#define XAC_T_PULL(I)                                                                                          \
  {                                                                                                            \
    constexpr int a = ex_of(I), b = ey_of(I), d = ez_of(I);                                                    \
    const bool xlo = (a == 1 && x == 0);                                                                       \
    const bool xhi = (a == -1 && x == nx - 1);                                                                 \
    const bool wall = (b == 1 && y == 0) || (b == -1 && y == ny - 1) || (d == 1 && z == 0) ||                 \
                      (d == -1 && z == nz - 1);                                                                \
    const long long off = (long long)a + (long long)b * nx + (long long)d * nxy;                               \
    const S* src = (xhi || xlo) ? (Qin + (long long)I * N + c)                                                 \
                                : (wall ? (Qin + (long long)opp_of(I) * N + c) : (Qin + (long long)I * N + c - off)); \
    const float v = Pop<S>::ld(src, w_of(I) * Tb);                                                             \
    T += xlo ? w_of(I) * p.T_in : v;                                                                           \
  }
    XAC_FOR19(XAC_T_PULL)
#undef XAC_T_PULL
  }
  T_o[c] = T;
}

}  // namespace xac
