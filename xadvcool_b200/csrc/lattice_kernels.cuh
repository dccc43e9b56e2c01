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
// bit  23/24 : x == 0 / x == nx-1
// bits 26..29: y == 0, y == ny-1, z == 0, z == nz-1; bit 25 = any of them
// bit  30    : solid cell whose population sector also holds a non-solid cell (it stores w_i so that every
//              fluid-output sector is written whole)
// With these bits a step needs no integer division to locate a cell.
constexpr int kTypeShift = 20;
constexpr uint32_t kHeatedBit = 1u << 22;
constexpr uint32_t kXLoBit = 1u << 23;
constexpr uint32_t kXHiBit = 1u << 24;
constexpr uint32_t kYZBit = 1u << 25;
constexpr uint32_t kYLoBit = 1u << 26;
constexpr uint32_t kYHiBit = 1u << 27;
constexpr uint32_t kZLoBit = 1u << 28;
constexpr uint32_t kZHiBit = 1u << 29;
constexpr uint32_t kFillBit = 1u << 30;  // solid cell sharing a 32-byte DRAM sector with a non-solid cell
__device__ __forceinline__ int link_type(uint32_t lw) { return (int)((lw >> kTypeShift) & 3u); }

// wall bits that make the thermal source of direction I leave the domain through a y/z face
__host__ __device__ constexpr uint32_t wall_bits(int I) {
  return (ey_of(I) == 1 ? kYLoBit : 0u) | (ey_of(I) == -1 ? kYHiBit : 0u) | (ez_of(I) == 1 ? kZLoBit : 0u) |
         (ez_of(I) == -1 ? kZHiBit : 0u);
}

struct Geom {
  int nx, ny, nz;
  long long ncell;  // nx*ny*nz
  long long N;      // population plane stride (elements)
};

// ---- population storage -------------------------------------------------------------------
// FP32 stores the population itself. The 16-bit forms store the deviation from the rest
// equilibrium w_i*ref (ref = 1 for the fluid, T_inlet for the thermal lattice) and do all
// arithmetic in float32.
// kCoherent loads go through L2 (ld.global.cg): needed when the data was written earlier in the same launch
// (the persistent batch kernel); otherwise the read-only path (ld.global.nc) is used.
template <typename S>
struct Pop;
template <>
struct Pop<float> {
  template <bool kCoherent = false>
  static __device__ __forceinline__ float ld(const float* p, float) {
    return kCoherent ? __ldcg(p) : __ldg(p);
  }
  static __device__ __forceinline__ void st(float* p, float v, float) { *p = v; }
};
template <>
struct Pop<__half> {
  template <bool kCoherent = false>
  static __device__ __forceinline__ float ld(const __half* p, float base) {
    return __half2float(kCoherent ? __ldcg(p) : __ldg(p)) + base;
  }
  static __device__ __forceinline__ void st(__half* p, float v, float base) { *p = __float2half_rn(v - base); }
};
template <>
struct Pop<__nv_bfloat16> {
  template <bool kCoherent = false>
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p, float base) {
    return __bfloat162float(kCoherent ? __ldcg(p) : __ldg(p)) + base;
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
  // 1/tau and 1 - omega/2 computed once on the device (the same IEEE float division as in the reference's
  // kernels, hoisted out of the per-cell work): fluid omega, thermal omega fluid/solid, source factor fluid/solid
  float omega_f, omega_tf, omega_ts, srcf_f, srcf_s;
  // element offsets: plane[i] = i*N; pull[i] = i*N - (ex + ey*nx + ez*nx*ny), so that the source of direction i
  // for cell c is pop[c + pull[i]] and its own value is pop[c + plane[i]] (32-bit indices: all are below 19 N).
  int32_t plane[kQ];
  int32_t pull[kQ];
};

#define XAC_FOR19(M) M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16) M(17) M(18)

// Lanes sharing one 32-byte DRAM sector of a population plane (planes are 256-byte aligned).
template <typename S>
__device__ __forceinline__ unsigned sector_group(int lane) {
  return sizeof(S) == 4 ? (0xFFu << (lane & ~7)) : (0xFFFFu << (lane & ~15));
}

// The three parts of one coupled step of cell c (see the scheme at the top of this file). Solid cells carry no
// fluid work: their fluid populations are the rest equilibrium w_i for ever (fluid_engine3d.py:193-194 never
// streams them, and they start at rho=1, u=0); a solid lane still stores w_i when a fluid lane shares its
// sector, so every sector of the fluid output is written whole.
// Population (direction i, cell c) is element c + plane[i] of its array; a pulled source is c + pull[i]. Both
// indices are formed in 32 bits (every one is non-negative and below 19 N) so each access costs one integer add
// and one widening multiply-add off the array base.

// fluid lattice of a non-solid cell: pull with the boundary rules, moments, BGK collision; returns u
template <typename S, bool kMacro, bool kCoherent = false>
__device__ __forceinline__ void fluid_cell(const uint32_t c, const S* __restrict__ Pin, S* __restrict__ Pout,
                                           const float* __restrict__ u_in_ptr, float* __restrict__ rho_o,
                                           float* __restrict__ ux_o, float* __restrict__ uy_o,
                                           float* __restrict__ uz_o, const StepParams& p, const uint32_t lw,
                                           float& ux, float& uy, float& uz) {
  const int type = link_type(lw);
  const S* __restrict__ Pc = Pin + c;  // outlet cells copy from Pc - 1
  float F[kQ];
  if (type == kInlet) {
    // src/fluid_engine3d.py:197-244: no pull; unknown populations from the known ones
    float k[kQ];
#define XAC_LD_OWN(I) k[I] = Pop<S>::template ld<kCoherent>(Pin + (c + p.plane[I]), w_of(I));
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
    const S* __restrict__ Ps = (lw & kXLoBit) ? Pc : Pc - 1;
    float sum = 0.0f;
#define XAC_LD_OUT(I)                              \
F[I] = Pop<S>::template ld<kCoherent>(Ps + p.plane[I], w_of(I));     \
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
F[I] = ((lw >> I) & 1u) ? Pop<S>::template ld<kCoherent>(Pin + (c + p.plane[opp_of(I)]), w_of(I)) : Pop<S>::template ld<kCoherent>(Pin + (c + p.pull[I]), w_of(I));
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
  const float omega = p.omega_f;
  const float usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#define XAC_COLLIDE(I)                                                            \
{                                                                               \
  const float fe = feq_term(w_of(I) * r, edotu<I>(ux, uy, uz), usq15);         \
  Pop<S>::st(Pout + (c + p.plane[I]), F[I] - omega * (F[I] - fe), w_of(I));             \
}
  XAC_FOR19(XAC_COLLIDE)
#undef XAC_COLLIDE
}

// fluid lattice of a solid cell: moments of the frozen populations on macro steps, w_i fill of shared sectors
template <typename S, bool kMacro, bool kCoherent = false>
__device__ __forceinline__ void solid_cell(const uint32_t c, const S* __restrict__ Pin, S* __restrict__ Pout,
                                           float* __restrict__ rho_o, float* __restrict__ ux_o,
                                           float* __restrict__ uy_o, float* __restrict__ uz_o,
                                           const StepParams& p, const bool fill_solid) {
  if (kMacro) {
    // moments of the frozen solid populations, as the reference's macroscopic kernel computes them
    float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const float v = Pop<S>::template ld<kCoherent>(Pin + (c + p.plane[i]), w_of(i));
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
  if (fill_solid) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) Pop<S>::st(Pout + (c + p.plane[i]), w_of(i), w_of(i));
  }
}

// thermal lattice of any cell, with the cell's fluid velocity u (0 in solids)
template <typename S, bool kOwn, bool kCoherent = false>
__device__ __forceinline__ void thermal_cell(const uint32_t c, const S* __restrict__ Qin, S* __restrict__ Qout,
                                             const float* __restrict__ qsrc, const float* __restrict__ T0,
                                             const StepParams& p, const uint32_t lw, const float ux, const float uy,
                                             const float uz) {
  const int type = link_type(lw);
  const S* __restrict__ Qc = Qin + c;  // outlet cells copy from Qc - 1
  const float Tb = p.T_ref;
  float G[kQ];
  float T;
  if (kOwn) {
#define XAC_LD_G0(I) G[I] = Pop<S>::template ld<kCoherent>(Qin + (c + p.plane[I]), w_of(I) * Tb);
    XAC_FOR19(XAC_LD_G0)
#undef XAC_LD_G0
    T = kCoherent ? __ldcg(T0 + c) : __ldg(T0 + c);
  } else {
    if (type == kInlet) {
      // src/thermal_engine3d.py:160-165
#pragma unroll
      for (int i = 0; i < kQ; ++i) G[i] = w_of(i) * p.T_in;
    } else if (type == kOutlet) {
      // src/thermal_engine3d.py:170-177
      const S* __restrict__ Qs = (lw & kXLoBit) ? Qc : Qc - 1;
#define XAC_LD_GOUT(I) G[I] = Pop<S>::template ld<kCoherent>(Qs + p.plane[I], w_of(I) * Tb);
      XAC_FOR19(XAC_LD_GOUT)
#undef XAC_LD_GOUT
    } else if (!(lw & kYZBit)) {
      // src/thermal_engine3d.py:180-211, cells away from the y/z faces: plain pull, except x<0 sources (inlet
      // equilibrium) and x>=nx sources (own value). Addresses stay in bounds: an x<0 source reads the own cell.
#define XAC_LD_GFAST(I)                                                                                        \
  {                                                                                                            \
    if (ex_of(I) == 1)                                                                                         \
      G[I] = (lw & kXLoBit) ? w_of(I) * p.T_in : Pop<S>::template ld<kCoherent>(Qin + (c + p.pull[I]), w_of(I) * Tb);                     \
    else if (ex_of(I) == -1)                                                                                   \
      G[I] = (lw & kXHiBit) ? Pop<S>::template ld<kCoherent>(Qin + (c + p.plane[I]), w_of(I) * Tb) : Pop<S>::template ld<kCoherent>(Qin + (c + p.pull[I]), w_of(I) * Tb); \
    else                                                                                                       \
      G[I] = Pop<S>::template ld<kCoherent>(Qin + (c + p.pull[I]), w_of(I) * Tb);                                                         \
  }
      XAC_FOR19(XAC_LD_GFAST)
#undef XAC_LD_GFAST
    } else {
      // the same rule with adiabatic bounce-back at the y/z faces
#define XAC_LD_GSLOW(I)                                                                                        \
  {                                                                                                            \
    const bool xlo = ex_of(I) == 1 && (lw & kXLoBit);                                                          \
    const bool xhi = ex_of(I) == -1 && (lw & kXHiBit);                                                         \
    const bool wall = (lw & wall_bits(I)) != 0u;                                                               \
    if (xlo)                                                                                                   \
      G[I] = w_of(I) * p.T_in;                                                                                 \
    else if (xhi)                                                                                              \
      G[I] = Pop<S>::template ld<kCoherent>(Qin + (c + p.plane[I]), w_of(I) * Tb);                                                        \
    else if (wall)                                                                                             \
      G[I] = Pop<S>::template ld<kCoherent>(Qin + (c + p.plane[opp_of(I)]), w_of(I) * Tb);                                                \
    else                                                                                                       \
      G[I] = Pop<S>::template ld<kCoherent>(Qin + (c + p.pull[I]), w_of(I) * Tb);                                                         \
  }
      XAC_FOR19(XAC_LD_GSLOW)
#undef XAC_LD_GSLOW
    }
    // src/thermal_engine3d.py:214-224
    T = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += G[i];
  }
  // src/thermal_engine3d.py:105-145: tau by phase, u = 0 in solids, source w_i (1 - omega/2) q
  const bool solid = type == kSolid;
  const float omega_t = solid ? p.omega_ts : p.omega_tf;
  const float srcf = solid ? p.srcf_s : p.srcf_f;
  const float q = (lw & kHeatedBit) ? __ldg(qsrc + c) : 0.0f;
  const float usq15t = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#define XAC_TCOLLIDE(I)                                                          \
  {                                                                              \
    const float ge = feq_term(w_of(I) * T, edotu<I>(ux, uy, uz), usq15t);       \
    float v = G[I] - omega_t * (G[I] - ge);                                      \
    if (q > 0.0f) v += (w_of(I) * srcf) * q;                                     \
    Pop<S>::st(Qout + (c + p.plane[I]), v, w_of(I) * Tb);                                \
  }
  XAC_FOR19(XAC_TCOLLIDE)
#undef XAC_TCOLLIDE
}

template <typename S, bool kMacro, bool kOwn, bool kCoherent = false>
__device__ __forceinline__ void coupled_cell(const uint32_t c, const S* __restrict__ Pin, S* __restrict__ Pout,
                                             const S* __restrict__ Qin, S* __restrict__ Qout,
                                             const uint32_t* __restrict__ link, const float* __restrict__ qsrc,
                                             const float* __restrict__ u_in_ptr, float* __restrict__ rho_o,
                                             float* __restrict__ ux_o, float* __restrict__ uy_o,
                                             float* __restrict__ uz_o, const float* __restrict__ T0,
                                             const StepParams& p, const bool valid, const uint32_t lw,
                                             const bool fill_solid) {
  const bool fluid = valid && link_type(lw) != kSolid;
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
  if (fluid)
    fluid_cell<S, kMacro, kCoherent>(c, Pin, Pout, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, lw, ux, uy, uz);
  else if (valid)
    solid_cell<S, kMacro, kCoherent>(c, Pin, Pout, rho_o, ux_o, uy_o, uz_o, p, fill_solid);
  if (!valid) return;
  thermal_cell<S, kOwn, kCoherent>(c, Qin, Qout, qsrc, T0, p, lw, ux, uy, uz);
}

// kCells cells per thread, at a stride of one block, so each load instruction stays coalesced.
template <typename S, bool kMacro, bool kOwn, int kCells>
__global__ void __launch_bounds__(256) coupled_step_kernel(const S* __restrict__ Pin, S* __restrict__ Pout,
                                                           const S* __restrict__ Qin, S* __restrict__ Qout,
                                                           const uint32_t* __restrict__ link,
                                                           const float* __restrict__ qsrc,
                                                           const float* __restrict__ u_in_ptr,
                                                           float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                           float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                           const float* __restrict__ T0, StepParams p) {
  const uint32_t base = blockIdx.x * blockDim.x * kCells + threadIdx.x;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < kCells; ++j) {
    const uint32_t c = base + j * blockDim.x;
    const bool valid = c < (uint32_t)p.g.ncell;
    const uint32_t lw = valid ? __ldg(link + c) : ((uint32_t)kSolid << kTypeShift);
    const unsigned fluid_lanes = __ballot_sync(0xffffffffu, valid && link_type(lw) != kSolid);
    coupled_cell<S, kMacro, kOwn>(c, Pin, Pout, Qin, Qout, link, qsrc, u_in_ptr, rho_o, ux_o, uy_o, uz_o, T0, p,
                                  valid, lw, (fluid_lanes & sector_group<S>(lane)) != 0u);
  }
}

// ---- pair-compacted step ------------------------------------------------------------------------
// A warp owns 64 consecutive cells, two groups of 32. When the two groups hold at most 32 non-solid cells
// between them (the usual case in a porous design), the fluid lattice of all of them runs in ONE pass over a
// compacted list - lane l takes the l-th non-solid cell - instead of two passes with the solid lanes idle. Each
// lane then gets its own cells' velocities back by shuffles and runs the thermal lattice of its two cells.
// Every cell runs exactly the arithmetic of coupled_cell, so results are identical.
template <typename S, bool kMacro, bool kOwn>
__global__ void __launch_bounds__(256) coupled_pair_kernel(const S* __restrict__ Pin, S* __restrict__ Pout,
                                                           const S* __restrict__ Qin, S* __restrict__ Qout,
                                                           const uint32_t* __restrict__ link,
                                                           const float* __restrict__ qsrc,
                                                           const float* __restrict__ u_in_ptr,
                                                           float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                           float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                           const float* __restrict__ T0, StepParams p) {
  __shared__ uint8_t slot[8][32];  // per warp: lane l of the compacted pass works on cell base + slot[l]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp) * 64u;
  const uint32_t ncell = (uint32_t)p.g.ncell;
  const uint32_t c0 = base + lane, c1 = base + 32u + lane;
  const bool v0 = c0 < ncell, v1 = c1 < ncell;
  const uint32_t solid_word = (uint32_t)kSolid << kTypeShift;
  const uint32_t lw0 = v0 ? __ldg(link + c0) : solid_word, lw1 = v1 ? __ldg(link + c1) : solid_word;
  const bool f0 = v0 && link_type(lw0) != kSolid, f1 = v1 && link_type(lw1) != kSolid;
  const unsigned m0 = __ballot_sync(0xffffffffu, f0), m1 = __ballot_sync(0xffffffffu, f1);
  const int k0 = __popc(m0), k1 = __popc(m1);
  float ux0 = 0.0f, uy0 = 0.0f, uz0 = 0.0f, ux1 = 0.0f, uy1 = 0.0f, uz1 = 0.0f;
  if (k0 + k1 <= 32) {
    const unsigned below = (1u << lane) - 1u;
    const int r0 = __popc(m0 & below), r1 = k0 + __popc(m1 & below);
    if (f0) slot[warp][r0] = (uint8_t)lane;
    if (f1) slot[warp][r1] = (uint8_t)(32 + lane);
    __syncwarp();
    const bool work = lane < k0 + k1;
    const int src = work ? slot[warp][lane] : 0;
    const uint32_t a = __shfl_sync(0xffffffffu, lw0, src & 31), b = __shfl_sync(0xffffffffu, lw1, src & 31);
    float ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (work)
      fluid_cell<S, kMacro>(base + (uint32_t)src, Pin, Pout, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, src < 32 ? a : b,
                            ux, uy, uz);
    const float a0 = __shfl_sync(0xffffffffu, ux, r0 & 31), a1 = __shfl_sync(0xffffffffu, uy, r0 & 31),
                a2 = __shfl_sync(0xffffffffu, uz, r0 & 31);
    const float b0 = __shfl_sync(0xffffffffu, ux, r1 & 31), b1 = __shfl_sync(0xffffffffu, uy, r1 & 31),
                b2 = __shfl_sync(0xffffffffu, uz, r1 & 31);
    if (f0) {
      ux0 = a0;
      uy0 = a1;
      uz0 = a2;
    }
    if (f1) {
      ux1 = b0;
      uy1 = b1;
      uz1 = b2;
    }
    __syncwarp();
  } else {
    if (f0) fluid_cell<S, kMacro>(c0, Pin, Pout, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, lw0, ux0, uy0, uz0);
    if (f1) fluid_cell<S, kMacro>(c1, Pin, Pout, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, lw1, ux1, uy1, uz1);
  }
  const unsigned sg = sector_group<S>(lane);
  if (v0 && !f0) solid_cell<S, kMacro>(c0, Pin, Pout, rho_o, ux_o, uy_o, uz_o, p, (m0 & sg) != 0u);
  if (v1 && !f1) solid_cell<S, kMacro>(c1, Pin, Pout, rho_o, ux_o, uy_o, uz_o, p, (m1 & sg) != 0u);
  if (v0) thermal_cell<S, kOwn>(c0, Qin, Qout, qsrc, T0, p, lw0, ux0, uy0, uz0);
  if (v1) thermal_cell<S, kOwn>(c1, Qin, Qout, qsrc, T0, p, lw1, ux1, uy1, uz1);
}

// ---- class-grouped step -------------------------------------------------------------------------
// Cells are visited through an index list grouped by class, so a warp never mixes them:
//   bulk fluid : fluid label, not on a y/z face  -> both lattices, plain pull, no boundary branches
//   bulk solid : solid label, not on a y/z face  -> thermal lattice only, with u = 0, where the second-order
//                equilibrium w_i T (1 + 3e.u + 4.5(e.u)^2 - 1.5u^2) evaluates to exactly w_i T
//   other      : inlet, outlet and y/z-face cells -> the general per-cell path
// Every cell runs exactly the arithmetic of coupled_cell, so results are identical.
enum CellClass : int { kClassBulkFluid = 0, kClassBulkSolid = 1, kClassOther = 2 };
constexpr uint32_t kNoCell = 0xFFFFFFFFu;

template <typename S, bool kOwn>
__device__ __forceinline__ void thermal_bulk_pull(const S* __restrict__ Qc, const uint32_t lw, const StepParams& p,
                                                  const float* __restrict__ T0, const uint32_t c, float (&G)[kQ],
                                                  float& T) {
  const float Tb = p.T_ref;
  if (kOwn) {
#define XAC_LD_G0(I) G[I] = Pop<S>::ld(Qc + p.plane[I], w_of(I) * Tb);
    XAC_FOR19(XAC_LD_G0)
#undef XAC_LD_G0
    T = __ldg(T0 + c);
    return;
  }
#define XAC_LD_GFAST(I)                                                                                        \
  {                                                                                                            \
    if (ex_of(I) == 1)                                                                                         \
      G[I] = (lw & kXLoBit) ? w_of(I) * p.T_in : Pop<S>::ld(Qc + p.pull[I], w_of(I) * Tb);                     \
    else if (ex_of(I) == -1)                                                                                   \
      G[I] = (lw & kXHiBit) ? Pop<S>::ld(Qc + p.plane[I], w_of(I) * Tb) : Pop<S>::ld(Qc + p.pull[I], w_of(I) * Tb); \
    else                                                                                                       \
      G[I] = Pop<S>::ld(Qc + p.pull[I], w_of(I) * Tb);                                                         \
  }
  XAC_FOR19(XAC_LD_GFAST)
#undef XAC_LD_GFAST
  T = 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) T += G[i];
}

template <typename S, bool kMacro, bool kOwn>
__device__ __forceinline__ void bulk_fluid_cell(const uint32_t c, const uint32_t lw, const S* __restrict__ Pin,
                                                S* __restrict__ Pout, const S* __restrict__ Qin,
                                                S* __restrict__ Qout, const float* __restrict__ qsrc,
                                                float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                const float* __restrict__ T0, const StepParams& p) {
  const S* __restrict__ Pc = Pin + c;
  S* __restrict__ Po = Pout + c;
  float F[kQ];
#define XAC_LD_PULL(I)                                                                                      \
  F[I] = ((lw >> I) & 1u) ? Pop<S>::ld(Pc + p.plane[opp_of(I)], w_of(I)) : Pop<S>::ld(Pc + p.pull[I], w_of(I));
  XAC_FOR19(XAC_LD_PULL)
#undef XAC_LD_PULL
  float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    r += F[i];
    if (ex_of(i) != 0) mx += ex_of(i) > 0 ? F[i] : -F[i];
    if (ey_of(i) != 0) my += ey_of(i) > 0 ? F[i] : -F[i];
    if (ez_of(i) != 0) mz += ez_of(i) > 0 ? F[i] : -F[i];
  }
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
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
  const float omega = p.omega_f;
  const float usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#define XAC_COLLIDE(I)                                                            \
  {                                                                               \
    const float fe = feq_term(w_of(I) * r, edotu<I>(ux, uy, uz), usq15);         \
    Pop<S>::st(Po + p.plane[I], F[I] - omega * (F[I] - fe), w_of(I));             \
  }
  XAC_FOR19(XAC_COLLIDE)
#undef XAC_COLLIDE
  float G[kQ], T;
  thermal_bulk_pull<S, kOwn>(Qin + c, lw, p, T0, c, G, T);
  S* __restrict__ Qo = Qout + c;
  const float omega_t = p.omega_tf, srcf = p.srcf_f;
  const float q = (lw & kHeatedBit) ? __ldg(qsrc + c) : 0.0f;
  const float usq15t = 1.5f * ((ux * ux + uy * uy) + uz * uz);
  const float Tb = p.T_ref;
#define XAC_TCOLLIDE(I)                                                          \
  {                                                                              \
    const float ge = feq_term(w_of(I) * T, edotu<I>(ux, uy, uz), usq15t);       \
    float v = G[I] - omega_t * (G[I] - ge);                                      \
    if (q > 0.0f) v += (w_of(I) * srcf) * q;                                     \
    Pop<S>::st(Qo + p.plane[I], v, w_of(I) * Tb);                                \
  }
  XAC_FOR19(XAC_TCOLLIDE)
#undef XAC_TCOLLIDE
}

template <typename S, bool kMacro, bool kOwn>
__device__ __forceinline__ void bulk_solid_cell(const uint32_t c, const uint32_t lw, S* __restrict__ Pout,
                                                const S* __restrict__ Qin, S* __restrict__ Qout,
                                                const float* __restrict__ qsrc, float* __restrict__ rho_o,
                                                float* __restrict__ ux_o, float* __restrict__ uy_o,
                                                float* __restrict__ uz_o, const float* __restrict__ T0,
                                                const StepParams& p) {
  if (kMacro) {
    // the frozen solid populations are w_i: rho = sum of w_i in order, u = 0
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) r += w_of(i);
    rho_o[c] = r;
    ux_o[c] = 0.0f;
    uy_o[c] = 0.0f;
    uz_o[c] = 0.0f;
  }
  if (lw & kFillBit) {
    S* __restrict__ Po = Pout + c;
#pragma unroll
    for (int i = 0; i < kQ; ++i) Pop<S>::st(Po + p.plane[i], w_of(i), w_of(i));
  }
  float G[kQ], T;
  thermal_bulk_pull<S, kOwn>(Qin + c, lw, p, T0, c, G, T);
  S* __restrict__ Qo = Qout + c;
  const float omega_t = p.omega_ts, srcf = p.srcf_s;
  const float q = (lw & kHeatedBit) ? __ldg(qsrc + c) : 0.0f;
  const float Tb = p.T_ref;
#define XAC_TCOLLIDE_S(I)                                                        \
  {                                                                              \
    const float ge = w_of(I) * T;                                                \
    float v = G[I] - omega_t * (G[I] - ge);                                      \
    if (q > 0.0f) v += (w_of(I) * srcf) * q;                                     \
    Pop<S>::st(Qo + p.plane[I], v, w_of(I) * Tb);                                \
  }
  XAC_FOR19(XAC_TCOLLIDE_S)
#undef XAC_TCOLLIDE_S
}

// cells: the three class lists concatenated, each padded with kNoCell to a multiple of 512 so that every
// block (<= 512 threads, a divisor of 512) sees one class. class_end: end of each class in the list.
template <typename S, bool kMacro, bool kOwn>
__global__ void __launch_bounds__(256) coupled_step_grouped_kernel(
    const uint32_t* __restrict__ cells, uint32_t end_fluid, uint32_t end_solid, const S* __restrict__ Pin,
    S* __restrict__ Pout, const S* __restrict__ Qin, S* __restrict__ Qout, const uint32_t* __restrict__ link,
    const float* __restrict__ qsrc, const float* __restrict__ u_in_ptr, float* __restrict__ rho_o,
    float* __restrict__ ux_o, float* __restrict__ uy_o, float* __restrict__ uz_o, const float* __restrict__ T0,
    StepParams p) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t c = __ldg(cells + idx);
  if (c == kNoCell) return;
  const uint32_t lw = __ldg(link + c);
  const uint32_t first = blockIdx.x * blockDim.x;
  if (first < end_fluid) {
    bulk_fluid_cell<S, kMacro, kOwn>(c, lw, Pin, Pout, Qin, Qout, qsrc, rho_o, ux_o, uy_o, uz_o, T0, p);
  } else if (first < end_solid) {
    bulk_solid_cell<S, kMacro, kOwn>(c, lw, Pout, Qin, Qout, qsrc, rho_o, ux_o, uy_o, uz_o, T0, p);
  } else {
    coupled_cell<S, kMacro, kOwn>(c, Pin, Pout, Qin, Qout, link, qsrc, u_in_ptr, rho_o, ux_o, uy_o, uz_o, T0, p,
                                  true, lw, (lw & kFillBit) != 0u);
  }
}

// omega and source factors, computed with the device's IEEE division once per lattice
static __global__ void relaxation_factors_kernel(float tau_f, float tau_tf, float tau_ts, float* out) {
  const float of = 1.0f / tau_f, otf = 1.0f / tau_tf, ots = 1.0f / tau_ts;
  out[0] = of;
  out[1] = otf;
  out[2] = ots;
  out[3] = 1.0f - 0.5f * otf;
  out[4] = 1.0f - 0.5f * ots;
}

// T^k = sum of the streamed thermal populations, without storing them (stats / field export steps).
template <typename S>
__global__ void __launch_bounds__(256) thermal_finalize_kernel(const S* __restrict__ Qin,
                                                               const uint32_t* __restrict__ link,
                                                               float* __restrict__ T_o, StepParams p) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (uint32_t)p.g.ncell) return;
  const uint32_t lw = __ldg(link + c);
  const int type = link_type(lw);
  const float Tb = p.T_ref;
  const S* __restrict__ Qc = Qin + c;
  float T = 0.0f;
  if (type == kInlet) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += w_of(i) * p.T_in;
  } else if (type == kOutlet) {
    const S* __restrict__ Qs = (lw & kXLoBit) ? Qc : Qc - 1;
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += Pop<S>::ld(Qs + p.plane[i], w_of(i) * Tb);
  } else {
#define XAC_T_PULL(I)                                                                                          \
  {                                                                                                            \
    const bool xlo = ex_of(I) == 1 && (lw & kXLoBit);                                                          \
    const bool xhi = ex_of(I) == -1 && (lw & kXHiBit);                                                         \
    const bool wall = (lw & wall_bits(I)) != 0u;                                                               \
    float v;                                                                                                   \
    if (xlo)                                                                                                   \
      v = w_of(I) * p.T_in;                                                                                    \
    else if (xhi)                                                                                              \
      v = Pop<S>::ld(Qc + p.plane[I], w_of(I) * Tb);                                                           \
    else if (wall)                                                                                             \
      v = Pop<S>::ld(Qc + p.plane[opp_of(I)], w_of(I) * Tb);                                                   \
    else                                                                                                       \
      v = Pop<S>::ld(Qc + p.pull[I], w_of(I) * Tb);                                                            \
    T += v;                                                                                                    \
  }
    XAC_FOR19(XAC_T_PULL)
#undef XAC_T_PULL
  }
  T_o[c] = T;
}

}  // namespace xac
