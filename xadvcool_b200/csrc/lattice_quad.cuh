// Quad variant of the fused coupled step: one thread owns 4 consecutive cells along x (the contiguous axis)
// and moves whole quads with 128-bit (FP32) / 64-bit (16-bit storage) loads and stores.
//
// Requirements (checked on the host): nx % 4 == 0, inlet cells only at x == 0, outlet cells only at x == nx-1.
// Then a quad never straddles a row, every population plane quad is 16-byte aligned, and the pull sources of
// a quad for direction i are one aligned quad of the source row plus, for ex = +-1, one element across the
// quad edge (read by a 32-bit load). Quads on a y/z face row take the per-cell path of lattice_kernels.cuh.
// The arithmetic of every cell is the per-cell kernel's, operation for operation, so both give the same bits.
#pragma once

#include "lattice_kernels.cuh"

namespace xac {

template <typename S>
struct QuadIO;
template <>
struct QuadIO<float> {
  static __device__ __forceinline__ void ld(float (&v)[4], const float* p, float) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
  static __device__ __forceinline__ void st(float* p, const float (&v)[4], float) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct QuadIO<__half> {
  static __device__ __forceinline__ void ld(float (&v)[4], const __half* p, float base) {
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&t.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&t.y));
    v[0] = a.x + base;
    v[1] = a.y + base;
    v[2] = b.x + base;
    v[3] = b.y + base;
  }
  static __device__ __forceinline__ void st(__half* p, const float (&v)[4], float base) {
    __half2 a = __floats2half2_rn(v[0] - base, v[1] - base);
    __half2 b = __floats2half2_rn(v[2] - base, v[3] - base);
    uint2 t;
    t.x = *reinterpret_cast<uint32_t*>(&a);
    t.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = t;
  }
};
template <>
struct QuadIO<__nv_bfloat16> {
  static __device__ __forceinline__ void ld(float (&v)[4], const __nv_bfloat16* p, float base) {
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&t.y));
    v[0] = a.x + base;
    v[1] = a.y + base;
    v[2] = b.x + base;
    v[3] = b.y + base;
  }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, const float (&v)[4], float base) {
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0] - base, v[1] - base);
    __nv_bfloat162 b = __floats2bfloat162_rn(v[2] - base, v[3] - base);
    uint2 t;
    t.x = *reinterpret_cast<uint32_t*>(&a);
    t.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = t;
  }
};

// sum of the rest weights in the reference's order: rho of a solid cell (its populations are w_i)
__device__ __forceinline__ float solid_rho() {
  float r = 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) r += w_of(i);
  return r;
}

template <typename S, bool kMacro, bool kOwn>
#ifndef XAC_QUAD_MIN_BLOCKS
#define XAC_QUAD_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(256, XAC_QUAD_MIN_BLOCKS) coupled_step_quad_kernel(const S* __restrict__ Pin, S* __restrict__ Pout,
                                                                const S* __restrict__ Qin, S* __restrict__ Qout,
                                                                const uint32_t* __restrict__ link,
                                                                const float* __restrict__ qsrc,
                                                                const float* __restrict__ u_in_ptr,
                                                                float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                                float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                                const float* __restrict__ T0, StepParams p) {
  const uint32_t c0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4u;
  const bool valid = c0 < (uint32_t)p.g.ncell;
  const int lane = threadIdx.x & 31;
  uint32_t lw[4];
  {
    const uint4 L = valid ? __ldg(reinterpret_cast<const uint4*>(link + c0))
                          : make_uint4(0u, 0u, 0u, 0u) ;
    lw[0] = L.x;
    lw[1] = L.y;
    lw[2] = L.z;
    lw[3] = L.w;
  }
  int ty[4];
  bool isfl[4];
  bool anyfluid = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    ty[k] = valid ? link_type(lw[k]) : (int)kSolid;
    isfl[k] = ty[k] != kSolid;
    anyfluid |= isfl[k];
  }
  // sectors are 8 FP32 / 16 16-bit cells: 2 or 4 quads (lanes) per sector
  const unsigned fb = __ballot_sync(0xffffffffu, anyfluid);
  const unsigned grp = sizeof(S) == 4 ? (0x3u << (lane & ~1)) : (0xFu << (lane & ~3));
  const bool sector_fluid = (fb & grp) != 0u;
  if (!valid) return;

  const bool yz = (lw[0] & kYZBit) != 0u;  // the four cells share y and z
  if (yz) {
    // y/z face rows: the per-cell path, cell by cell
#pragma unroll 1
    for (int k = 0; k < 4; ++k)
      coupled_cell<S, kMacro, kOwn>(c0 + k, Pin, Pout, Qin, Qout, link, qsrc, u_in_ptr, rho_o, ux_o, uy_o, uz_o, T0,
                                    p, true, lw[k], sector_fluid);
    return;
  }

  const bool xlo = (lw[0] & kXLoBit) != 0u;  // cell 0 at x = 0
  const bool xhi = (lw[3] & kXHiBit) != 0u;  // cell 3 at x = nx-1
  const bool inlet0 = ty[0] == kInlet;       // only possible with xlo
  const bool outlet3 = ty[3] == kOutlet;     // only possible with xhi
  float ux[4] = {0.0f, 0.0f, 0.0f, 0.0f}, uy[4] = {0.0f, 0.0f, 0.0f, 0.0f}, uz[4] = {0.0f, 0.0f, 0.0f, 0.0f};

  // ------------------------------------------------------------------ fluid lattice
  if (anyfluid) {
    float F[kQ][4];
    // src/fluid_engine3d.py:262-272 for the quad: aligned quad of the source row, the cross-edge element, and
    // the own opposite value where a cell bounces back
#define XAC_Q_PULL(I)                                                                                          \
  {                                                                                                            \
    constexpr int a = ex_of(I);                                                                                \
    const S* src = Pin + c0 + p.pull[I];                                                                       \
    float v[4];                                                                                                \
    if (a == 0) {                                                                                              \
      QuadIO<S>::ld(v, src, w_of(I));                                                                          \
      F[I][0] = v[0];                                                                                          \
      F[I][1] = v[1];                                                                                          \
      F[I][2] = v[2];                                                                                          \
      F[I][3] = v[3];                                                                                          \
    } else if (a == 1) {                                                                                       \
      QuadIO<S>::ld(v, src + 1, w_of(I));                                                                      \
      F[I][0] = ((lw[0] >> I) & 1u) ? 0.0f : Pop<S>::ld(src, w_of(I));                                         \
      F[I][1] = v[0];                                                                                          \
      F[I][2] = v[1];                                                                                          \
      F[I][3] = v[2];                                                                                          \
    } else {                                                                                                   \
      QuadIO<S>::ld(v, src - 1, w_of(I));                                                                      \
      F[I][0] = v[1];                                                                                          \
      F[I][1] = v[2];                                                                                          \
      F[I][2] = v[3];                                                                                          \
      F[I][3] = ((lw[3] >> I) & 1u) ? 0.0f : Pop<S>::ld(src + 3, w_of(I));                                     \
    }                                                                                                          \
    const uint32_t bb = ((lw[0] >> I) & 1u) | (((lw[1] >> I) & 1u) << 1) | (((lw[2] >> I) & 1u) << 2) |      \
                        (((lw[3] >> I) & 1u) << 3);                                                            \
    if (bb) {                                                                                                  \
      float o[4];                                                                                              \
      QuadIO<S>::ld(o, Pin + c0 + p.plane[opp_of(I)], w_of(I));                                                \
      if (bb & 1u) F[I][0] = o[0];                                                                             \
      if (bb & 2u) F[I][1] = o[1];                                                                             \
      if (bb & 4u) F[I][2] = o[2];                                                                             \
      if (bb & 8u) F[I][3] = o[3];                                                                             \
    }                                                                                                          \
  }
    XAC_FOR19(XAC_Q_PULL)
#undef XAC_Q_PULL
    if (xlo && inlet0) {
      // src/fluid_engine3d.py:197-244: the inlet cell (x = 0, cell 0) uses its own populations
#pragma unroll
      for (int i = 0; i < kQ; ++i) F[i][0] = Pop<S>::ld(Pin + c0 + p.plane[i], w_of(i));
      const float ux_in = __ldg(u_in_ptr);
      const float rn = (((((((((F[0][0] + F[3][0]) + F[4][0]) + F[5][0]) + F[6][0]) + F[15][0]) + F[16][0]) +
                          F[17][0]) + F[18][0]) +
                        2.0f * ((((F[2][0] + F[8][0]) + F[10][0]) + F[12][0]) + F[14][0])) /
                       (1.0f - ux_in);
      const float c23 = 2.0f / 3.0f, c16 = 1.0f / 6.0f;
      F[1][0] = F[2][0] + (c23 * rn) * ux_in;
      F[7][0] = F[10][0] + (c16 * rn) * ux_in;
      F[9][0] = F[8][0] + (c16 * rn) * ux_in;
      F[11][0] = F[14][0] + (c16 * rn) * ux_in;
      F[13][0] = F[12][0] + (c16 * rn) * ux_in;
    }
    if (xhi && outlet3) {
      // src/fluid_engine3d.py:247-259: the outlet cell (x = nx-1, cell 3) copies x-1 and rescales
      float sum = 0.0f;
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        F[i][3] = Pop<S>::ld(Pin + c0 + 2 + p.plane[i], w_of(i));
        sum += F[i][3];
      }
      if (sum > 1e-6f) {
        const float sc = p.rho_out / sum;
#pragma unroll
        for (int i = 0; i < kQ; ++i) F[i][3] *= sc;
      }
    }
    // moments (src/fluid_engine3d.py:85-113) and BGK (src/fluid_engine3d.py:157-173), cell by cell
    float rr[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        r += F[i][k];
        if (ex_of(i) != 0) mx += ex_of(i) > 0 ? F[i][k] : -F[i][k];
        if (ey_of(i) != 0) my += ey_of(i) > 0 ? F[i][k] : -F[i][k];
        if (ez_of(i) != 0) mz += ez_of(i) > 0 ? F[i][k] : -F[i][k];
      }
      if (isfl[k] && r > 1e-10f) {
        ux[k] = mx / r;
        uy[k] = my / r;
        uz[k] = mz / r;
      }
      rr[k] = isfl[k] ? r : solid_rho();
    }
    if (kMacro) {
      *reinterpret_cast<float4*>(rho_o + c0) = make_float4(rr[0], rr[1], rr[2], rr[3]);
      *reinterpret_cast<float4*>(ux_o + c0) = make_float4(ux[0], ux[1], ux[2], ux[3]);
      *reinterpret_cast<float4*>(uy_o + c0) = make_float4(uy[0], uy[1], uy[2], uy[3]);
      *reinterpret_cast<float4*>(uz_o + c0) = make_float4(uz[0], uz[1], uz[2], uz[3]);
    }
    const float omega = p.omega_f;
    float usq15[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) usq15[k] = 1.5f * ((ux[k] * ux[k] + uy[k] * uy[k]) + uz[k] * uz[k]);
#define XAC_Q_COLLIDE(I)                                                                          \
  {                                                                                               \
    float o[4];                                                                                   \
    _Pragma("unroll") for (int k = 0; k < 4; ++k) {                                               \
      const float fe = feq_term(w_of(I) * rr[k], edotu<I>(ux[k], uy[k], uz[k]), usq15[k]);       \
      o[k] = isfl[k] ? F[I][k] - omega * (F[I][k] - fe) : w_of(I);                                \
    }                                                                                             \
    QuadIO<S>::st(Pout + c0 + p.plane[I], o, w_of(I));                                            \
  }
    XAC_FOR19(XAC_Q_COLLIDE)
#undef XAC_Q_COLLIDE
  } else {
    if (kMacro) {
      const float r = solid_rho();
      *reinterpret_cast<float4*>(rho_o + c0) = make_float4(r, r, r, r);
      *reinterpret_cast<float4*>(ux_o + c0) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      *reinterpret_cast<float4*>(uy_o + c0) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      *reinterpret_cast<float4*>(uz_o + c0) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (sector_fluid) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        const float o[4] = {w_of(i), w_of(i), w_of(i), w_of(i)};
        QuadIO<S>::st(Pout + c0 + p.plane[i], o, w_of(i));
      }
    }
  }

  // keep the thermal loads behind the fluid stores: the two 76-value working sets are never live together
  asm volatile("" ::: "memory");

  // ------------------------------------------------------------------ thermal lattice
  const float Tb = p.T_ref;
  float G[kQ][4];
  float T[4];
  if (kOwn) {
#define XAC_Q_G0(I) QuadIO<S>::ld(G[I], Qin + c0 + p.plane[I], w_of(I) * Tb);
    XAC_FOR19(XAC_Q_G0)
#undef XAC_Q_G0
    const float4 t = __ldg(reinterpret_cast<const float4*>(T0 + c0));
    T[0] = t.x;
    T[1] = t.y;
    T[2] = t.z;
    T[3] = t.w;
  } else {
    // src/thermal_engine3d.py:180-211 away from the y/z faces: plain pull; the x = 0 cell takes the inlet
    // equilibrium from x < 0 sources, the x = nx-1 cell its own value from x >= nx sources
#define XAC_Q_GPULL(I)                                                                                         \
  {                                                                                                            \
    constexpr int a = ex_of(I);                                                                                \
    const S* src = Qin + c0 + p.pull[I];                                                                       \
    float v[4];                                                                                                \
    if (a == 0) {                                                                                              \
      QuadIO<S>::ld(G[I], src, w_of(I) * Tb);                                                                  \
    } else if (a == 1) {                                                                                       \
      QuadIO<S>::ld(v, src + 1, w_of(I) * Tb);                                                                 \
      G[I][0] = xlo ? w_of(I) * p.T_in : Pop<S>::ld(src, w_of(I) * Tb);                                        \
      G[I][1] = v[0];                                                                                          \
      G[I][2] = v[1];                                                                                          \
      G[I][3] = v[2];                                                                                          \
    } else {                                                                                                   \
      QuadIO<S>::ld(v, src - 1, w_of(I) * Tb);                                                                 \
      G[I][0] = v[1];                                                                                          \
      G[I][1] = v[2];                                                                                          \
      G[I][2] = v[3];                                                                                          \
      G[I][3] = Pop<S>::ld(xhi ? (Qin + c0 + 3 + p.plane[I]) : (src + 3), w_of(I) * Tb);                       \
    }                                                                                                          \
  }
    XAC_FOR19(XAC_Q_GPULL)
#undef XAC_Q_GPULL
    if (xlo && inlet0) {
      // src/thermal_engine3d.py:160-165
#pragma unroll
      for (int i = 0; i < kQ; ++i) G[i][0] = w_of(i) * p.T_in;
    }
    if (xhi && outlet3) {
      // src/thermal_engine3d.py:170-177: the outlet copies x-1, the quad's cell 2
#pragma unroll
      for (int i = 0; i < kQ; ++i) G[i][3] = Pop<S>::ld(Qin + c0 + 2 + p.plane[i], w_of(i) * Tb);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float t = 0.0f;
#pragma unroll
      for (int i = 0; i < kQ; ++i) t += G[i][k];
      T[k] = t;
    }
  }
  // src/thermal_engine3d.py:105-145
  float om[4], sf[4], q[4], usq15t[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const bool solid = !isfl[k];
    om[k] = solid ? p.omega_ts : p.omega_tf;
    sf[k] = solid ? p.srcf_s : p.srcf_f;
    q[k] = (lw[k] & kHeatedBit) ? __ldg(qsrc + c0 + k) : 0.0f;
    usq15t[k] = 1.5f * ((ux[k] * ux[k] + uy[k] * uy[k]) + uz[k] * uz[k]);
  }
#define XAC_Q_TCOLLIDE(I)                                                                     \
  {                                                                                           \
    float o[4];                                                                               \
    _Pragma("unroll") for (int k = 0; k < 4; ++k) {                                           \
      const float ge = feq_term(w_of(I) * T[k], edotu<I>(ux[k], uy[k], uz[k]), usq15t[k]);   \
      float v = G[I][k] - om[k] * (G[I][k] - ge);                                             \
      if (q[k] > 0.0f) v += (w_of(I) * sf[k]) * q[k];                                         \
      o[k] = v;                                                                               \
    }                                                                                         \
    QuadIO<S>::st(Qout + c0 + p.plane[I], o, w_of(I) * Tb);                                   \
  }
  XAC_FOR19(XAC_Q_TCOLLIDE)
#undef XAC_Q_TCOLLIDE
}

}  // namespace xac
