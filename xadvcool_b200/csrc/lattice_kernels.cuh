// Device kernels of the fused lattice (internal layout).
//
// Internal layout. Cells are numbered c = (z*ny + y)*nx + x (x fastest, the flow/streaming axis) for the link
// words, the heat source and the macroscopic fields.
//
// Thermal populations (every cell conducts heat) are stored row-tiled: a row (y, z) holds the 19 directions one
// after another, each a run of `pitch` = nx rounded up to 32 values:
//     pop[guard + ((z*ny + y)*19 + i)*pitch + x]
// so a direction's value of a row's neighbour in x, y or in the same row is at a compile-time distance
// (i*pitch - ex - ey*19*pitch) from the cell, and only z neighbours need another base pointer (one slab of
// ny*19*pitch values away). Rows of `guard` = (ny + 2)*19*pitch zero values before and after the array keep every
// source address that a bounce-back lane might form inside the allocation.
//
// Fluid populations exist for non-solid cells only: a solid cell's are the rest equilibrium w_i for ever (it
// starts at rho = 1, u = 0 and is never streamed, src/fluid_engine3d.py:193-194). They are stored direction-major
// over the non-solid cells in cell order:
//     pf[i*ns + k],   k = number of non-solid cells before the cell
// and a step finds k of a cell and of its pull sources in the rows above, below and beside it from a per-row table
// (FluidAt). A warp's fluid lanes then read and write one contiguous run per direction, and no solid bytes move:
// on a 63%-solid gyroid this is 55 instead of 152 fluid bytes per cell and step.
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
__device__ __forceinline__ int link_type(uint32_t lw) { return (int)((lw >> kTypeShift) & 3u); }

// wall bits that make the thermal source of direction I leave the domain through a y/z face
__host__ __device__ constexpr uint32_t wall_bits(int I) {
  return (ey_of(I) == 1 ? kYLoBit : 0u) | (ey_of(I) == -1 ? kYHiBit : 0u) | (ez_of(I) == 1 ? kZLoBit : 0u) |
         (ez_of(I) == -1 ? kZHiBit : 0u);
}

struct Geom {
  int nx, ny, nz;
  long long ncell;  // nx*ny*nz
  int pitch;        // population row length: nx rounded up to 32
  int rows;         // ny*nz
  long long guard;  // zero elements before the first and after the last row of a population array
  long long N;      // elements of one thermal population array: rows*19*pitch + 2*guard
  int nt;           // 32-cell words of a row: pitch / 32
  long long ns;     // slots of a fluid population run: the non-solid cells, rounded up to a multiple of 32
  long long np;     // elements of one fluid population array: 19*ns
};

// row length, a compile-time constant when kT > 0
template <int kT>
__host__ __device__ __forceinline__ int row_len(const Geom& g) {
  return kT > 0 ? kT : g.pitch;
}
// element of (direction 0, this row, x) for compact cell (row r, x)
__device__ __forceinline__ uint32_t pop_base(uint32_t r, uint32_t x, const Geom& g, int pitch) {
  return (uint32_t)g.guard + r * (uint32_t)(kQ * pitch) + x;
}

// ---- population storage -------------------------------------------------------------------
// FP32 stores the population itself. The 16-bit forms store the deviation from the rest
// equilibrium w_i*ref (ref = 1 for the fluid, T_inlet for the thermal lattice) and do all
// arithmetic in float32.
// Load modes: 0 = read-only path (ld.global.nc); 1 = through L2 (ld.global.cg), needed when the data was written
// earlier in the same launch (the persistent batch kernel); 2 = plain load (values staged in shared memory).
template <typename S>
struct Pop;
template <>
struct Pop<float> {
  template <int kLd = 0>
  static __device__ __forceinline__ float ld(const float* p, float) {
    return kLd == 2 ? *p : (kLd == 1 ? __ldcg(p) : __ldg(p));
  }
  static __device__ __forceinline__ void st(float* p, float v, float) { *p = v; }
};
template <>
struct Pop<__half> {
  template <int kLd = 0>
  static __device__ __forceinline__ float ld(const __half* p, float base) {
    return __half2float(kLd == 2 ? *p : (kLd == 1 ? __ldcg(p) : __ldg(p))) + base;
  }
  static __device__ __forceinline__ void st(__half* p, float v, float base) { *p = __float2half_rn(v - base); }
};
template <>
struct Pop<__nv_bfloat16> {
  template <int kLd = 0>
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p, float base) {
    return __bfloat162float(kLd == 2 ? *p : (kLd == 1 ? __ldcg(p) : __ldg(p))) + base;
  }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float v, float base) {
    *p = __float2bfloat16_rn(v - base);
  }
};
// Storage of each precision mode: fluid populations P, thermal populations Q. BF16's 8-bit significand is used for
// the fluid lattice only: a thermal population's deviation from w_i*T_inlet is dominated by its advective part
// w_i*T*3(e_i.u) (~0.2 at T = 25, |u| = 0.05), so the temperature signal w_i*(T - T_inlet) must be resolved far
// below it, which FP16's 11-bit significand does to ~1e-4 and BF16's 8 bits do not.
template <int kPrecision>
struct Storage;
template <>
struct Storage<XAC_FP32> {
  using P = float;
  using Q = float;
};
template <>
struct Storage<XAC_FP16> {
  using P = __half;
  using Q = __half;
};
template <>
struct Storage<XAC_BF16> {
  using P = __nv_bfloat16;
  using Q = __half;
};
template <>
struct Storage<XAC_FP32_T16> {
  using P = float;
  using Q = __half;
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
  // 1 = the step runs its blocks in reverse order. The host sets it on every other step, so each step starts on
  // the rows the previous step wrote last, which are still in L2 (31.6 vs 32.4 us per 148x128x32 step)
  uint32_t reverse;
  unsigned* status;  // per-lattice device word: bit 0 = a bounded wait in a step kernel ran out
  const uint2* ftab;  // non-solid cell table of the fluid populations (FluidAt)
};

// One cell's view of a population array in global memory: the cell's own position (direction 0) and the same x
// in the rows one z-slab below (source of directions with ez = +1) and above (ez = -1). own(i) is the cell's
// direction i, pull<I>() the source of direction I (a compile-time offset from one of the three pointers when
// kT > 0).
template <typename S, int kT>
struct Rows {
  const S* c;
  const S* zm;
  const S* zp;
  int RL;
  __device__ __forceinline__ const S* own(int i) const { return c + i * (kT > 0 ? kT : RL); }
  template <int I>
  __device__ __forceinline__ const S* pull() const {
    const int T = kT > 0 ? kT : RL;
    const S* b = ez_of(I) > 0 ? zm : (ez_of(I) < 0 ? zp : c);
    return b + (I * T - ex_of(I) - ey_of(I) * kQ * T);
  }
};
// Runtime row length: one base pointer and 32-bit element indices (every index of a population array fits in 31
// bits), so an address is formed right before its load instead of 19 64-bit pointers living at once.
template <typename S>
struct Rows<S, 0> {
  const S* base;
  uint32_t c, zm, zp;
  int RL;
  __device__ __forceinline__ const S* own(int i) const { return base + (c + (uint32_t)(i * RL)); }
  template <int I>
  __device__ __forceinline__ const S* pull() const {
    const uint32_t b = ez_of(I) > 0 ? zm : (ez_of(I) < 0 ? zp : c);
    return base + (b + (uint32_t)((I - ey_of(I) * kQ) * RL - ex_of(I)));
  }
};
template <int kT, typename S>
__device__ __forceinline__ Rows<S, kT> rows_at(const S* base, uint32_t e0, const Geom& g, int pitch) {
  if constexpr (kT > 0) {
    const long long slab = (long long)g.ny * kQ * pitch;
    return {base + e0, base + e0 - slab, base + e0 + slab, pitch};
  } else {
    const uint32_t slab = (uint32_t)g.ny * kQ * (uint32_t)pitch;
    return {base, e0, e0 - slab, e0 + slab, pitch};
  }
}

// ---- fluid populations of the non-solid cells -------------------------------------------------------------
// Table entry ftab[(r + ny + 1)*nt + w] of the 32-cell word w of row r: .x = bit b set when cell x = 32w + b is
// not solid, .y = k of the word's first cell (the non-solid cells before it). ny + 1 rows with an empty mask lie
// before and after the grid, so the rows above and below any row, in y and z, have an entry.
// The eight rows other than its own that a cell's pulls read, by (e_y, e_z) of the direction; the source row is
// r - e_y - e_z*ny.
__host__ __device__ constexpr int fluid_row_slot(int ey, int ez) {
  return ey == 1 && ez == 0 ? 0 : ey == -1 && ez == 0 ? 1 : ey == 0 && ez == 1 ? 2 : ey == 0 && ez == -1 ? 3
       : ey == 1 && ez == 1 ? 4 : ey == -1 && ez == -1 ? 5 : ey == 1 && ez == -1 ? 6 : 7;
}
__host__ __device__ constexpr int fluid_row_ey(int j) { return j == 0 || j == 4 || j == 6 ? 1 : j == 1 || j == 5 || j == 7 ? -1 : 0; }
__host__ __device__ constexpr int fluid_row_ez(int j) { return j == 2 || j == 4 || j == 7 ? 1 : j == 3 || j == 5 || j == 6 ? -1 : 0; }

// One non-solid cell's view of a fluid population array: own(i) is its direction i, pull<I>() the source of
// direction I when that source is a non-solid cell (a solid or off-grid source is a bounce-back, which reads
// own(opp)). rk[j] is the number of non-solid cells before the cell's x in row slot j; the source of a
// direction with e_x = 0 is that cell, with e_x = +1 the one before it (x-1 is non-solid), with e_x = -1 the next
// one (x+1), which is one further when x itself is non-solid in that row (bit j of nb).
template <typename S>
struct FluidAt {
  const S* base;
  uint32_t ns, k, nb;
  uint32_t rk[8];
  __device__ __forceinline__ const S* own(int i) const { return base + ((uint32_t)i * ns + k); }
  template <int I>
  __device__ __forceinline__ const S* pull() const {
    uint32_t s;
    if constexpr (ey_of(I) == 0 && ez_of(I) == 0) {
      s = k - (uint32_t)ex_of(I);
    } else {
      constexpr int j = fluid_row_slot(ey_of(I), ez_of(I));
      s = rk[j];
      if constexpr (ex_of(I) == 1) s -= 1u;
      if constexpr (ex_of(I) == -1) s += (nb >> j) & 1u;
    }
    return base + ((uint32_t)I * ns + s);
  }
};
// table entry of the word holding cell (row r, x)
__host__ __device__ __forceinline__ uint32_t ftab_index(const Geom& g, uint32_t r, uint32_t x) {
  return (r + (uint32_t)g.ny + 1u) * (uint32_t)g.nt + (x >> 5);
}
// the view of cell (row r, x), which must be non-solid; the nine table loads are the same for a whole warp
template <typename S>
__device__ __forceinline__ FluidAt<S> fluid_at(const S* base, uint32_t r, uint32_t x, const Geom& g,
                                               const uint2* __restrict__ ftab) {
  FluidAt<S> a;
  a.base = base;
  a.ns = (uint32_t)g.ns;
  const uint32_t below = (1u << (x & 31u)) - 1u, bit = x & 31u;
  const uint32_t t0 = ftab_index(g, r, x);
  const uint2 e = __ldg(ftab + t0);
  a.k = e.y + (uint32_t)__popc(e.x & below);
  a.nb = 0u;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int dr = -fluid_row_ey(j) - fluid_row_ez(j) * g.ny;
    const uint2 n = __ldg(ftab + (t0 + (uint32_t)(dr * g.nt)));
    a.rk[j] = n.y + (uint32_t)__popc(n.x & below);
    a.nb |= ((n.x >> bit) & 1u) << j;
  }
  return a;
}

#define XAC_FOR19(M) M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16) M(17) M(18)

// Lanes sharing one 32-byte DRAM sector of a thermal population row (rows start on 32-value boundaries).
template <typename S>
__device__ __forceinline__ unsigned sector_group(int lane) {
  return sizeof(S) == 4 ? (0xFFu << (lane & ~7)) : (0xFFFFu << (lane & ~15));
}

// The three parts of one coupled step of cell c (see the scheme at the top of this file). Solid cells carry no
// fluid work and store no fluid populations: theirs are the rest equilibrium w_i for ever
// (fluid_engine3d.py:193-194 never streams them, and they start at rho=1, u=0).
// c is the cell index (link word, heat source, fields); P is the cell's view of the input fluid populations and
// Po its own slot in the output (direction i at +i*ns); Q is its row view of the input thermal populations and Qo
// its own position in the output (direction i at +i*pitch).

// fluid lattice of a non-solid cell: pull with the boundary rules, moments, BGK collision; returns u
template <typename S, bool kMacro, int kLd, class Acc>
__device__ __forceinline__ void fluid_cell(const uint32_t c, const Acc& P, S* __restrict__ Po,
                                           const float* __restrict__ u_in_ptr, float* __restrict__ rho_o,
                                           float* __restrict__ ux_o, float* __restrict__ uy_o,
                                           float* __restrict__ uz_o, const StepParams& p, const uint32_t lw,
                                           float& ux, float& uy, float& uz) {
  const int type = link_type(lw);
  float F[kQ];
  if (type == kInlet) {
    // src/fluid_engine3d.py:197-244: no pull; unknown populations from the known ones
    float k[kQ];
#define XAC_LD_OWN(I) k[I] = Pop<S>::template ld<kLd>(P.own(I), w_of(I));
    XAC_FOR19(XAC_LD_OWN)
#undef XAC_LD_OWN
    // the batch kernel's pump controller changes the inlet within a launch: read it through L2 there
    const float ux_in = kLd == 1 ? __ldcg(u_in_ptr) : __ldg(u_in_ptr);
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
    // src/fluid_engine3d.py:247-259: copy post-collision (x-1) and rescale to rho_outlet. The x-1 cell is the
    // previous non-solid cell when it is not solid (link bit 1: the source of direction 1 is x-1), and holds the
    // rest equilibrium w_i when it is.
    const int dxo = (lw & kXLoBit) ? 0 : -1;
    const bool west_solid = dxo != 0 && ((lw >> 1) & 1u);
    float sum = 0.0f;
#define XAC_LD_OUT(I)                                                                        \
F[I] = west_solid ? w_of(I) : Pop<S>::template ld<kLd>(P.own(I) + dxo, w_of(I));             \
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
F[I] = ((lw >> I) & 1u) ? Pop<S>::template ld<kLd>(P.own(opp_of(I)), w_of(I)) : Pop<S>::template ld<kLd>(P.template pull<I>(), w_of(I));
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
  Pop<S>::st(Po + (I) * P.ns, F[I] - omega * (F[I] - fe), w_of(I));           \
}
  XAC_FOR19(XAC_COLLIDE)
#undef XAC_COLLIDE
}

// fluid lattice of a solid cell: on macro steps the moments of its frozen populations, which are the rest
// equilibrium w_i (summed in the order of the reference's macroscopic kernel, so rho and u carry the same bits)
template <bool kMacro>
__device__ __forceinline__ void solid_cell(const uint32_t c, float* __restrict__ rho_o, float* __restrict__ ux_o,
                                           float* __restrict__ uy_o, float* __restrict__ uz_o) {
  if (kMacro) {
    float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const float v = w_of(i);
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
}

// thermal lattice of any cell, with the cell's fluid velocity u (0 in solids)
template <typename S, bool kOwn, int kLd, int kT, class Acc>
__device__ __forceinline__ void thermal_cell(const uint32_t c, const Acc& Q, S* __restrict__ Qo,
                                             const float* __restrict__ qsrc, const float* __restrict__ T0,
                                             const StepParams& p, const uint32_t lw, const float ux, const float uy,
                                             const float uz) {
  const int type = link_type(lw);
  const int RL = row_len<kT>(p.g);
  const float Tb = p.T_ref;
  float G[kQ];
  float T;
  if (kOwn) {
#define XAC_LD_G0(I) G[I] = Pop<S>::template ld<kLd>(Q.own(I), w_of(I) * Tb);
    XAC_FOR19(XAC_LD_G0)
#undef XAC_LD_G0
    T = kLd == 1 ? __ldcg(T0 + c) : __ldg(T0 + c);  // T0 lives in global memory
  } else {
    if (type == kInlet) {
      // src/thermal_engine3d.py:160-165
#pragma unroll
      for (int i = 0; i < kQ; ++i) G[i] = w_of(i) * p.T_in;
    } else if (type == kOutlet) {
      // src/thermal_engine3d.py:170-177
      const int dxo = (lw & kXLoBit) ? 0 : -1;
#define XAC_LD_GOUT(I) G[I] = Pop<S>::template ld<kLd>(Q.own(I) + dxo, w_of(I) * Tb);
      XAC_FOR19(XAC_LD_GOUT)
#undef XAC_LD_GOUT
    } else if (!(lw & kYZBit)) {
      // src/thermal_engine3d.py:180-211, cells away from the y/z faces: plain pull, except x<0 sources (inlet
      // equilibrium) and x>=nx sources (own value). Addresses stay in bounds: an x<0 source reads the own cell.
#define XAC_LD_GFAST(I)                                                                                        \
  {                                                                                                            \
    if (ex_of(I) == 1)                                                                                         \
      G[I] = (lw & kXLoBit) ? w_of(I) * p.T_in : Pop<S>::template ld<kLd>(Q.template pull<I>(), w_of(I) * Tb);                     \
    else if (ex_of(I) == -1)                                                                                   \
      G[I] = (lw & kXHiBit) ? Pop<S>::template ld<kLd>(Q.own(I), w_of(I) * Tb) : Pop<S>::template ld<kLd>(Q.template pull<I>(), w_of(I) * Tb); \
    else                                                                                                       \
      G[I] = Pop<S>::template ld<kLd>(Q.template pull<I>(), w_of(I) * Tb);                                                         \
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
      G[I] = Pop<S>::template ld<kLd>(Q.own(I), w_of(I) * Tb);                                                        \
    else if (wall)                                                                                             \
      G[I] = Pop<S>::template ld<kLd>(Q.own(opp_of(I)), w_of(I) * Tb);                                                \
    else                                                                                                       \
      G[I] = Pop<S>::template ld<kLd>(Q.template pull<I>(), w_of(I) * Tb);                                                         \
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
    Pop<S>::st(Qo + (I) * RL, v, w_of(I) * Tb);                                \
  }
  XAC_FOR19(XAC_TCOLLIDE)
#undef XAC_TCOLLIDE
}

// cell c = (row r, x); its thermal populations start at element e0; SP / SQ: fluid / thermal storage
template <typename SP, typename SQ, bool kMacro, bool kOwn, int kLd, int kT>
__device__ __forceinline__ void coupled_cell(const uint32_t c, const uint32_t r, const uint32_t x, const uint32_t e0,
                                             const SP* __restrict__ Pin, SP* __restrict__ Pout,
                                             const SQ* __restrict__ Qin, SQ* __restrict__ Qout,
                                             const float* __restrict__ qsrc, const float* __restrict__ u_in_ptr,
                                             float* __restrict__ rho_o, float* __restrict__ ux_o,
                                             float* __restrict__ uy_o, float* __restrict__ uz_o,
                                             const float* __restrict__ T0, const StepParams& p, const bool valid,
                                             const uint32_t lw) {
  const int RL = row_len<kT>(p.g);
  const bool fluid = valid && link_type(lw) != kSolid;
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
  if (fluid) {
    const FluidAt<SP> P = fluid_at(Pin, r, x, p.g, p.ftab);
    fluid_cell<SP, kMacro, kLd>(c, P, Pout + P.k, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, lw, ux, uy, uz);
  } else if (valid) {
    solid_cell<kMacro>(c, rho_o, ux_o, uy_o, uz_o);
  }
  if (!valid) return;
  thermal_cell<SQ, kOwn, kLd, kT>(c, rows_at<kT>(Qin, e0, p.g, RL), Qout + e0, qsrc, T0, p, lw, ux, uy, uz);
}

// Padding positions (x >= nx) of a row's last, partly valid sector store a thermal value too, so that the sector
// is written whole (no read-modify-write in L2); the values are never read.
template <typename SQ, int kT>
__device__ __forceinline__ void pad_fill(bool valid, unsigned valid_lanes, int lane, SQ* __restrict__ Qout,
                                         uint32_t e0, const Geom& g) {
  if (valid) return;
  const int RL = row_len<kT>(g);
  if (valid_lanes & sector_group<SQ>(lane)) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) Pop<SQ>::st(Qout + e0 + i * RL, 0.0f, 0.0f);
  }
}

// One thread per row position: block-consecutive threads walk x along a row (a warp never spans two rows, the
// row length being a multiple of 32); positions x >= nx are padding. kT > 0 makes the row length and every
// thermal population offset compile-time constants; kT = 0 reads it from the geometry.
template <typename SP, typename SQ, bool kMacro, bool kOwn, int kT>
__global__ void __launch_bounds__(256) coupled_step_kernel(const SP* __restrict__ Pin, SP* __restrict__ Pout,
                                                           const SQ* __restrict__ Qin, SQ* __restrict__ Qout,
                                                           const uint32_t* __restrict__ link,
                                                           const float* __restrict__ qsrc,
                                                           const float* __restrict__ u_in_ptr,
                                                           float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                           float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                           const float* __restrict__ T0, StepParams p) {
  const int RL = row_len<kT>(p.g);
  const uint32_t blk = p.reverse ? gridDim.x - 1u - blockIdx.x : blockIdx.x;
  const uint32_t pos = blk * blockDim.x + threadIdx.x;
  const uint32_t r = pos / (uint32_t)RL, x = pos - r * (uint32_t)RL;
  if (r >= (uint32_t)p.g.rows) return;  // whole warps
  const int lane = threadIdx.x & 31;
  const bool valid = x < (uint32_t)p.g.nx;
  const uint32_t c = r * (uint32_t)p.g.nx + x;
  const uint32_t lw = valid ? __ldg(link + c) : ((uint32_t)kSolid << kTypeShift);
  const uint32_t e0 = pop_base(r, x, p.g, RL);
  coupled_cell<SP, SQ, kMacro, kOwn, 0, kT>(c, r, x, e0, Pin, Pout, Qin, Qout, qsrc, u_in_ptr, rho_o, ux_o, uy_o,
                                            uz_o, T0, p, valid, lw);
  pad_fill<SQ, kT>(valid, __ballot_sync(0xffffffffu, valid), lane, Qout, e0, p.g);
}

// ---- thermal rows staged in shared memory (launch variant 1) ------------------------------------------
// One block per row, blockDim = the row length. Thread 0 starts bulk copies (cp.async.bulk, completion counted on
// an mbarrier) of the thermal input the row needs: the row's own 19 directions (one contiguous run) and, for the 16
// directions whose source row differs (e_y or e_z != 0), that direction's run of the source row. The threads run
// the fluid lattice from global memory meanwhile, then wait for the copies (bounded) and run the thermal lattice
// from shared memory. Every cell runs the arithmetic of coupled_cell, so results are identical.
template <typename S, int kT>
struct StageQ {
  static constexpr int kPad = 16 / (int)sizeof(S);  // 16 bytes of room on both sides of a run
  static constexpr int kOwn = kPad + kQ * kT + kPad;
  static constexpr int kSlot = kPad + kT + kPad;
  static constexpr int kLen = kOwn + 16 * kSlot;  // elements
};
// a cell's view of the staged thermal input: own run (direction 0 at this x) and slot 0 (direction 3 at this x)
template <typename S, int kT>
struct SmemRows {
  const S* c;
  const S* s0;
  __device__ __forceinline__ const S* own(int i) const { return c + i * kT; }
  template <int I>
  __device__ __forceinline__ const S* pull() const {
    if (ey_of(I) == 0 && ez_of(I) == 0) return c + I * kT - ex_of(I);
    return s0 + (I - 3) * StageQ<S, kT>::kSlot - ex_of(I);
  }
};

__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool bar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t limit = 1u << 22) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <typename SP, typename SQ, bool kMacro, bool kOwn, int kT>
__global__ void __launch_bounds__(kT) coupled_qstage_kernel(const SP* __restrict__ Pin, SP* __restrict__ Pout,
                                                            const SQ* __restrict__ Qin, SQ* __restrict__ Qout,
                                                            const uint32_t* __restrict__ link,
                                                            const float* __restrict__ qsrc,
                                                            const float* __restrict__ u_in_ptr,
                                                            float* __restrict__ rho_o, float* __restrict__ ux_o,
                                                            float* __restrict__ uy_o, float* __restrict__ uz_o,
                                                            const float* __restrict__ T0, StepParams p) {
  using St = StageQ<SQ, kT>;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  SQ* sq = reinterpret_cast<SQ*>(sm_raw);
  __shared__ __align__(8) uint64_t bar;
  const uint32_t r = p.reverse ? gridDim.x - 1u - blockIdx.x : blockIdx.x, x = threadIdx.x;
  const int lane = x & 31;
  const uint32_t b = sh_addr(&bar);
  if (x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (x == 0) {
    const uint32_t run = (uint32_t)(kT * sizeof(SQ));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"((kQ + 16) * run) : "memory");
    const SQ* row0 = Qin + p.g.guard;
    bulk_copy(sh_addr(sq + St::kPad), row0 + (long long)r * kQ * kT, kQ * run, b);
#pragma unroll
    for (int i = 3; i < kQ; ++i) {
      const long long rs = (long long)r - ey_of(i) - (long long)ez_of(i) * p.g.ny;  // guards cover rows off the grid
      bulk_copy(sh_addr(sq + St::kOwn + (i - 3) * St::kSlot + St::kPad), row0 + (rs * kQ + i) * kT, run, b);
    }
  }
  const bool valid = x < (uint32_t)p.g.nx;
  const uint32_t c = r * (uint32_t)p.g.nx + x;
  const uint32_t lw = valid ? __ldg(link + c) : ((uint32_t)kSolid << kTypeShift);
  const uint32_t e0 = pop_base(r, x, p.g, kT);
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
  if (valid && link_type(lw) != kSolid) {
    const FluidAt<SP> P = fluid_at(Pin, r, x, p.g, p.ftab);
    fluid_cell<SP, kMacro, 0>(c, P, Pout + P.k, u_in_ptr, rho_o, ux_o, uy_o, uz_o, p, lw, ux, uy, uz);
  } else if (valid) {
    solid_cell<kMacro>(c, rho_o, ux_o, uy_o, uz_o);
  }
  const bool ok = bar_wait_bounded(b, 0);
  if (!ok && x == 0) atomicOr(p.status, 1u);
  if (valid && ok)
    thermal_cell<SQ, kOwn, 2, kT>(c, SmemRows<SQ, kT>{sq + St::kPad + x, sq + St::kOwn + St::kPad + x}, Qout + e0,
                                 qsrc, T0, p, lw, ux, uy, uz);
  pad_fill<SQ, kT>(valid, __ballot_sync(0xffffffffu, valid), lane, Qout, e0, p.g);
}

// Arguments of one fused step launch; launch_coupled_step<SP, SQ> (step_kernels.cuh, one translation unit per
// storage mode) picks the instantiation whose compile-time row length matches the lattice.
struct StepLaunch {
  const void* Pin;
  void* Pout;
  const void* Qin;
  void* Qout;
  const uint32_t* link;
  const float* qsrc;
  const float* u_in;
  float *rho, *ux, *uy, *uz;
  const float* T0;
  StepParams p;
  int block;
  int variant;  // 0: one thread per row position; 1: thermal rows staged in shared memory (compile-time pitch)
  bool macro, own;
  cudaStream_t stream;
};
template <typename SP, typename SQ>
void launch_coupled_step(const StepLaunch& a);

// omega and source factors, computed with the device's IEEE division once per lattice
static __global__ void relaxation_factors_kernel(float tau_f, float tau_tf, float tau_ts, float* out) {
  const float of = 1.0f / tau_f, otf = 1.0f / tau_tf, ots = 1.0f / tau_ts;
  out[0] = of;
  out[1] = otf;
  out[2] = ots;
  out[3] = 1.0f - 0.5f * otf;
  out[4] = 1.0f - 0.5f * ots;
}

// T^k = sum of the streamed thermal populations of compact cell c, without storing them (stats / field export
// steps and the batch kernel's stats steps).
template <typename S, bool kCoherent>
__device__ __forceinline__ float finalize_T_cell(const S* __restrict__ Qin, const uint32_t* __restrict__ link,
                                                 const StepParams& p, uint32_t c) {
  const uint32_t lw = __ldg(link + c);
  const int type = link_type(lw);
  const float Tb = p.T_ref;
  const int RL = p.g.pitch;
  const uint32_t r = c / (uint32_t)p.g.nx, x = c - r * (uint32_t)p.g.nx;
  const Rows<S, 0> Q = rows_at<0>(Qin, pop_base(r, x, p.g, RL), p.g, RL);
  float T = 0.0f;
  if (type == kInlet) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += w_of(i) * p.T_in;
  } else if (type == kOutlet) {
    const int dxo = (lw & kXLoBit) ? 0 : -1;
#pragma unroll
    for (int i = 0; i < kQ; ++i) T += Pop<S>::template ld<kCoherent>(Q.own(i) + dxo, w_of(i) * Tb);
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
      v = Pop<S>::template ld<kCoherent>(Q.own(I), w_of(I) * Tb);                                               \
    else if (wall)                                                                                             \
      v = Pop<S>::template ld<kCoherent>(Q.own(opp_of(I)), w_of(I) * Tb);                                     \
    else                                                                                                       \
      v = Pop<S>::template ld<kCoherent>(Q.template pull<I>(), w_of(I) * Tb);                                \
    T += v;                                                                                                    \
  }
    XAC_FOR19(XAC_T_PULL)
#undef XAC_T_PULL
  }
  return T;
}

template <typename S>
__global__ void __launch_bounds__(256) thermal_finalize_kernel(const S* __restrict__ Qin,
                                                               const uint32_t* __restrict__ link,
                                                               float* __restrict__ T_o, StepParams p) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (uint32_t)p.g.ncell) return;
  T_o[c] = finalize_T_cell<S, false>(Qin, link, p, c);
}

}  // namespace xac
