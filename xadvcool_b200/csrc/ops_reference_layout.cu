// Unfused per-operator kernels in the reference layout f[19][nx][ny][nz] (z fastest).
// Each kernel restates one Warp kernel of the reference with the same operand order, so that
// validate_analytical.py-style drivers port 1:1 and every operator can be checked on its own.
// One thread per cell; consecutive threads walk z, the contiguous axis of that layout.
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <vector>

#include "xac_internal.cuh"

namespace xac {

namespace {

struct Dims {
  int nx, ny, nz;
  long long n;  // cells
};

__device__ __forceinline__ void decompose(long long c, const Dims& d, int& x, int& y, int& z) {
  z = (int)(c % d.nz);
  long long t = c / d.nz;
  y = (int)(t % d.ny);
  x = (int)(t / d.ny);
}

__device__ __forceinline__ long long cell_of(int x, int y, int z, const Dims& d) {
  return ((long long)x * d.ny + y) * d.nz + z;
}

// The operators below run in the reference's float32 (T = float) and, for the FP64 solve, in double. These are the
// equilibrium pieces of xac_internal.cuh for any arithmetic type; for float they are the same operations.
template <typename T>
__device__ __forceinline__ T w_t(int i) {
  return wclass_of(i) == 0 ? (T)(1.0 / 3.0) : (wclass_of(i) == 1 ? (T)(1.0 / 18.0) : (T)(1.0 / 36.0));
}
template <int I, typename T>
__device__ __forceinline__ T edotu_t(T ux, T uy, T uz) {
  constexpr int a = ex_of(I), b = ey_of(I), c = ez_of(I);
  T s = T(0);
  bool have = false;
  if (a != 0) { s = a > 0 ? ux : -ux; have = true; }
  if (b != 0) { T t = b > 0 ? uy : -uy; s = have ? s + t : t; have = true; }
  if (c != 0) { T t = c > 0 ? uz : -uz; s = have ? s + t : t; have = true; }
  return s;
}
template <typename T>
__device__ __forceinline__ T feq_t(T w_rho, T eu, T usq15) {
  return w_rho * (((T(1) + T(3) * eu) + T(4.5) * (eu * eu)) - usq15);
}
// e_i . u of direction i (a runtime index inside an unrolled loop)
template <typename T>
__device__ __forceinline__ T edotu_at(int i, T ux, T uy, T uz) {
  switch (i) {
#define XAC_CASE(I) case I: return edotu_t<I>(ux, uy, uz);
    XAC_CASE(0) XAC_CASE(1) XAC_CASE(2) XAC_CASE(3) XAC_CASE(4) XAC_CASE(5) XAC_CASE(6) XAC_CASE(7)
    XAC_CASE(8) XAC_CASE(9) XAC_CASE(10) XAC_CASE(11) XAC_CASE(12) XAC_CASE(13) XAC_CASE(14) XAC_CASE(15)
    XAC_CASE(16) XAC_CASE(17) XAC_CASE(18)
#undef XAC_CASE
    default: return T(0);
  }
}

// src/fluid_engine3d.py:58-80 (also the thermal twin with T in place of rho, thermal_engine3d.py:7-47)
template <typename T, bool kThermal>
__global__ void equilibrium_kernel(const T* __restrict__ scal, const T* __restrict__ u,
                                   const int32_t* __restrict__ mask, T* __restrict__ out, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  T s = scal[c];
  T ux = u[3 * c], uy = u[3 * c + 1], uz = u[3 * c + 2];
  if (kThermal && mask[c] == kSolid) { ux = T(0); uy = T(0); uz = T(0); }
  T usq15 = T(1.5) * ((ux * ux + uy * uy) + uz * uz);
#pragma unroll
  for (int i = 0; i < kQ; ++i) out[(long long)i * d.n + c] = feq_t(w_t<T>(i) * s, edotu_at(i, ux, uy, uz), usq15);
}

// src/fluid_engine3d.py:85-113
template <typename T>
__global__ void macroscopic_kernel(const T* __restrict__ f, T* __restrict__ rho, T* __restrict__ u, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  T r = T(0), mx = T(0), my = T(0), mz = T(0);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    T v = f[(long long)i * d.n + c];
    r += v;
    mx += v * (T)ex_of(i);
    my += v * (T)ey_of(i);
    mz += v * (T)ez_of(i);
  }
  rho[c] = r;
  if (r > (T)1e-10) {
    u[3 * c] = mx / r;
    u[3 * c + 1] = my / r;
    u[3 * c + 2] = mz / r;
  } else {
    u[3 * c] = T(0);
    u[3 * c + 1] = T(0);
    u[3 * c + 2] = T(0);
  }
}

// src/fluid_engine3d.py:118-136
__global__ void bgk_collision_kernel(const float* __restrict__ fo, const float* __restrict__ fe,
                                     float* __restrict__ fp, const int32_t* __restrict__ mask, float tau, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int m = mask[c];
  float omega = 1.0f / tau;
  bool act = (m == kFluid || m == kInlet || m == kOutlet);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long k = (long long)i * d.n + c;
    fp[k] = act ? fo[k] - omega * (fo[k] - fe[k]) : fo[k];
  }
}

// src/fluid_engine3d.py:141-176
template <typename T>
__global__ void fused_collision_kernel(const T* __restrict__ fo, const T* __restrict__ rho, const T* __restrict__ u,
                                       T* __restrict__ fp, const int32_t* __restrict__ mask, T tau, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int m = mask[c];
  T omega = T(1) / tau;
  if (m == kFluid || m == kInlet || m == kOutlet) {
    T r = rho[c];
    T ux = u[3 * c], uy = u[3 * c + 1], uz = u[3 * c + 2];
    T usq15 = T(1.5) * ((ux * ux + uy * uy) + uz * uz);
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      long long k = (long long)i * d.n + c;
      T f = fo[k];
      fp[k] = f - omega * (f - feq_t(w_t<T>(i) * r, edotu_at(i, ux, uy, uz), usq15));
    }
  } else {
#pragma unroll
    for (int i = 0; i < kQ; ++i) fp[(long long)i * d.n + c] = fo[(long long)i * d.n + c];
  }
}

// src/fluid_engine3d.py:181-272
template <typename T>
__global__ void streaming_kernel(const T* __restrict__ fp, T* __restrict__ fs, const int32_t* __restrict__ mask,
                                 const T* __restrict__ u_inlet, T rho_outlet, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int x, y, z;
  decompose(c, d, x, y, z);
  int m = mask[c];
  const long long N = d.n;
  if (m == kSolid) return;
  if (m == kInlet) {
    T ux_in = u_inlet[0];
    T f0 = fp[c], f2 = fp[2 * N + c], f3 = fp[3 * N + c], f4 = fp[4 * N + c], f5 = fp[5 * N + c];
    T f6 = fp[6 * N + c], f8 = fp[8 * N + c], f10 = fp[10 * N + c], f12 = fp[12 * N + c];
    T f14 = fp[14 * N + c], f15 = fp[15 * N + c], f16 = fp[16 * N + c], f17 = fp[17 * N + c];
    T f18 = fp[18 * N + c];
    T rn = (((((((((f0 + f3) + f4) + f5) + f6) + f15) + f16) + f17) + f18) +
                T(2) * ((((f2 + f8) + f10) + f12) + f14)) /
               (T(1) - ux_in);
    const T c23 = T(2) / T(3), c16 = T(1) / T(6);
    fs[c] = f0;
    fs[1 * N + c] = f2 + (c23 * rn) * ux_in;
    fs[2 * N + c] = f2;
    fs[3 * N + c] = f3;
    fs[4 * N + c] = f4;
    fs[5 * N + c] = f5;
    fs[6 * N + c] = f6;
    fs[7 * N + c] = f10 + (c16 * rn) * ux_in;
    fs[8 * N + c] = f8;
    fs[9 * N + c] = f8 + (c16 * rn) * ux_in;
    fs[10 * N + c] = f10;
    fs[11 * N + c] = f14 + (c16 * rn) * ux_in;
    fs[12 * N + c] = f12;
    fs[13 * N + c] = f12 + (c16 * rn) * ux_in;
    fs[14 * N + c] = f14;
    fs[15 * N + c] = f15;
    fs[16 * N + c] = f16;
    fs[17 * N + c] = f17;
    fs[18 * N + c] = f18;
    return;
  }
  if (m == kOutlet) {
    long long s = cell_of(x > 0 ? x - 1 : 0, y, z, d);
    T v[kQ];
    T sum = T(0);
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      v[i] = fp[(long long)i * N + s];
      sum += v[i];
    }
    if (sum > (T)1e-6) {
      T sc = rho_outlet / sum;
#pragma unroll
      for (int i = 0; i < kQ; ++i) v[i] *= sc;
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) fs[(long long)i * N + c] = v[i];
    return;
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    int sx = x - ex_of(i), sy = y - ey_of(i), sz = z - ez_of(i);
    bool bb = sx < 0 || sx >= d.nx || sy < 0 || sy >= d.ny || sz < 0 || sz >= d.nz;
    long long s = bb ? c : cell_of(sx, sy, sz, d);
    if (!bb) bb = mask[s] == kSolid;
    fs[(long long)i * N + c] = bb ? fp[(long long)opp_of(i) * N + c] : fp[(long long)i * N + s];
  }
}

// src/thermal_engine3d.py:49-86 (kFused=false, g_eq given) and :91-145 (kFused=true, g_eq in registers)
template <typename T, bool kFused>
__global__ void thermal_collision_kernel(const T* __restrict__ go, const T* __restrict__ ge, const T* __restrict__ u,
                                         const T* __restrict__ Tf, T* __restrict__ gn, const int32_t* __restrict__ mask,
                                         T tau_f, T tau_s, const T* __restrict__ hs, T power, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  bool solid = mask[c] == kSolid;
  T tau = solid ? tau_s : tau_f;
  T omega = T(1) / tau;
  T q = hs[c] * power;
  T srcf = T(1) - T(0.5) * omega;
  T t = T(0), ux = T(0), uy = T(0), uz = T(0), usq15 = T(0);
  if (kFused) {
    t = Tf[c];
    if (!solid) { ux = u[3 * c]; uy = u[3 * c + 1]; uz = u[3 * c + 2]; }
    usq15 = T(1.5) * ((ux * ux + uy * uy) + uz * uz);
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long k = (long long)i * d.n + c;
    T g = go[k];
    T geq = kFused ? feq_t(w_t<T>(i) * t, edotu_at(i, ux, uy, uz), usq15) : ge[k];
    T v = g - omega * (g - geq);
    if (q > T(0)) v += (w_t<T>(i) * srcf) * q;
    gn[k] = v;
  }
}

// src/thermal_engine3d.py:147-211
template <typename T>
__global__ void thermal_streaming_kernel(const T* __restrict__ gp, T* __restrict__ gs, const int32_t* __restrict__ mask,
                                         T T_in, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int x, y, z;
  decompose(c, d, x, y, z);
  int m = mask[c];
  const long long N = d.n;
  if (m == kInlet) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) gs[(long long)i * N + c] = w_t<T>(i) * T_in;
    return;
  }
  if (m == kOutlet) {
    long long s = cell_of(x > 0 ? x - 1 : 0, y, z, d);
#pragma unroll
    for (int i = 0; i < kQ; ++i) gs[(long long)i * N + c] = gp[(long long)i * N + s];
    return;
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    int sx = x - ex_of(i), sy = y - ey_of(i), sz = z - ez_of(i);
    T v;
    if (sx < 0) v = w_t<T>(i) * T_in;
    else if (sx >= d.nx) v = gp[(long long)i * N + c];
    else if (sy < 0 || sy >= d.ny || sz < 0 || sz >= d.nz) v = gp[(long long)opp_of(i) * N + c];
    else v = gp[(long long)i * N + cell_of(sx, sy, sz, d)];
    gs[(long long)i * N + c] = v;
  }
}

// src/thermal_engine3d.py:214-224
template <typename T>
__global__ void thermal_macroscopic_kernel(const T* __restrict__ g, T* __restrict__ Tf, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  T s = T(0);
#pragma unroll
  for (int i = 0; i < kQ; ++i) s += g[(long long)i * d.n + c];
  Tf[c] = s;
}

// ---- test-only operators of validate_analytical.py ---------------------------------------------

// :21-30
__global__ void dirichlet_plane_kernel(float* __restrict__ g, float T_val, int x_plane, Dims d) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)d.ny * d.nz) return;
  int y = (int)(t / d.nz), z = (int)(t % d.nz);
  long long c = cell_of(x_plane, y, z, d);
#pragma unroll
  for (int i = 0; i < kQ; ++i) g[(long long)i * d.n + c] = w_of(i) * T_val;
}

__device__ __forceinline__ int wrap(int a, int n) { return (a + n) % n; }

// :255-273 and :607-621
__global__ void periodic_stream_kernel(const float* __restrict__ fp, float* __restrict__ fs, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int x, y, z;
  decompose(c, d, x, y, z);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long s = cell_of(wrap(x - ex_of(i), d.nx), wrap(y - ey_of(i), d.ny), wrap(z - ez_of(i), d.nz), d);
    fs[(long long)i * d.n + c] = fp[(long long)i * d.n + s];
  }
}

// :377-395
__global__ void forced_bgk_kernel(const float* __restrict__ fo, const float* __restrict__ fe,
                                  float* __restrict__ fn, const int32_t* __restrict__ mask, float tau, float force_x,
                                  Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  float omega = 1.0f / tau;
  bool act = mask[c] != kSolid;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long k = (long long)i * d.n + c;
    float src = ((w_of(i) * 3.0f) * (float)ex_of(i)) * force_x;
    fn[k] = act ? (fo[k] - omega * (fo[k] - fe[k])) + src : fo[k];
  }
}

// :397-420
__global__ void periodic_stream_solids_kernel(const float* __restrict__ fp, float* __restrict__ fs,
                                              const int32_t* __restrict__ mask, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  if (mask[c] == kSolid) return;
  int x, y, z;
  decompose(c, d, x, y, z);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long s = cell_of(wrap(x - ex_of(i), d.nx), wrap(y - ey_of(i), d.ny), wrap(z - ez_of(i), d.nz), d);
    bool bb = mask[s] == kSolid;
    fs[(long long)i * d.n + c] = bb ? fp[(long long)opp_of(i) * d.n + c] : fp[(long long)i * d.n + s];
  }
}

// :502-538
__global__ void couette_stream_kernel(const float* __restrict__ fp, float* __restrict__ fs,
                                      const int32_t* __restrict__ mask, float u_wall_x, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  if (mask[c] == kSolid) return;
  int x, y, z;
  decompose(c, d, x, y, z);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    int sx = wrap(x - ex_of(i), d.nx), sy = wrap(y - ey_of(i), d.ny), sz = z - ez_of(i);
    float v;
    if (sz < 0) {
      v = fp[(long long)opp_of(i) * d.n + c];
    } else if (sz >= d.nz) {
      float mom = ((6.0f * w_of(i)) * (float)ex_of(i)) * u_wall_x;
      v = fp[(long long)opp_of(i) * d.n + c] + mom;
    } else {
      long long s = cell_of(sx, sy, sz, d);
      v = mask[s] == kSolid ? fp[(long long)opp_of(i) * d.n + c] : fp[(long long)i * d.n + s];
    }
    fs[(long long)i * d.n + c] = v;
  }
}

constexpr int kBlock = 256;

template <typename T>
__global__ void fill_kernel(T* __restrict__ p, T v, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

int check_dims(int nx, int ny, int nz, Dims& d) {
  XAC_REQUIRE(nx > 0 && ny > 0 && nz > 0, "lattice dimensions must be positive (got %d x %d x %d)", nx, ny, nz);
  XAC_REQUIRE((long long)nx * ny * nz * kQ < (1LL << 40), "lattice too large");
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.n = (long long)nx * ny * nz;
  return XAC_OK;
}

int post_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, what);
  return XAC_OK;
}

}  // namespace

}  // namespace xac

using namespace xac;

#define XAC_DIMS()                             \
  Dims d;                                      \
  {                                            \
    int _r = check_dims(nx, ny, nz, d);        \
    if (_r != XAC_OK) return _r;               \
  }

extern "C" {

int xac_equilibrium(const float* rho, const float* u, float* f_eq, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(rho && u && f_eq, "xac_equilibrium: null pointer");
  equilibrium_kernel<float, false><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(rho, u, nullptr, f_eq, d);
  return post_launch("xac_equilibrium");
}

int xac_macroscopic(const float* f, float* rho, float* u, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f && rho && u, "xac_macroscopic: null pointer");
  macroscopic_kernel<float><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f, rho, u, d);
  return post_launch("xac_macroscopic");
}

int xac_bgk_collision(const float* f_old, const float* f_eq, float* f_post, const int32_t* mask, float tau, int nx,
                      int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_old && f_eq && f_post && mask, "xac_bgk_collision: null pointer");
  bgk_collision_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_old, f_eq, f_post, mask, tau, d);
  return post_launch("xac_bgk_collision");
}

int xac_fused_collision(const float* f_old, const float* rho, const float* u, float* f_post, const int32_t* mask,
                        float tau, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_old && rho && u && f_post && mask, "xac_fused_collision: null pointer");
  fused_collision_kernel<float><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_old, rho, u, f_post, mask, tau,
                                                                                  d);
  return post_launch("xac_fused_collision");
}

int xac_stream(const float* f_post, float* f_streamed, const int32_t* mask, const float* u_inlet, float rho_outlet,
               int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_post && f_streamed && mask && u_inlet, "xac_stream: null pointer");
  XAC_REQUIRE(f_post != f_streamed, "xac_stream: input and output must be distinct buffers");
  streaming_kernel<float><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_post, f_streamed, mask, u_inlet,
                                                                            rho_outlet, d);
  return post_launch("xac_stream");
}

int xac_thermal_equilibrium(const float* u, const float* T, float* g_eq, const int32_t* mask, int nx, int ny, int nz,
                            void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(u && T && g_eq && mask, "xac_thermal_equilibrium: null pointer");
  equilibrium_kernel<float, true><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(T, u, mask, g_eq, d);
  return post_launch("xac_thermal_equilibrium");
}

int xac_thermal_bgk_collision(const float* g_old, const float* g_eq, float* g_new, const int32_t* mask,
                              float tau_fluid, float tau_solid, const float* heat_source, float heat_power, int nx,
                              int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_old && g_eq && g_new && mask && heat_source, "xac_thermal_bgk_collision: null pointer");
  thermal_collision_kernel<float, false><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(
      g_old, g_eq, nullptr, nullptr, g_new, mask, tau_fluid, tau_solid, heat_source, heat_power, d);
  return post_launch("xac_thermal_bgk_collision");
}

int xac_fused_thermal_collision(const float* g_old, const float* u, const float* T, float* g_new,
                                const int32_t* mask, float tau_fluid, float tau_solid, const float* heat_source,
                                float heat_power, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_old && u && T && g_new && mask && heat_source, "xac_fused_thermal_collision: null pointer");
  thermal_collision_kernel<float, true><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(
      g_old, nullptr, u, T, g_new, mask, tau_fluid, tau_solid, heat_source, heat_power, d);
  return post_launch("xac_fused_thermal_collision");
}

int xac_thermal_stream(const float* g_post, float* g_streamed, const int32_t* mask, float T_inlet, int nx, int ny,
                       int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_post && g_streamed && mask, "xac_thermal_stream: null pointer");
  XAC_REQUIRE(g_post != g_streamed, "xac_thermal_stream: input and output must be distinct buffers");
  thermal_streaming_kernel<float><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(g_post, g_streamed, mask,
                                                                                    T_inlet, d);
  return post_launch("xac_thermal_stream");
}

int xac_thermal_macroscopic(const float* g, float* T, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g && T, "xac_thermal_macroscopic: null pointer");
  thermal_macroscopic_kernel<float><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(g, T, d);
  return post_launch("xac_thermal_macroscopic");
}

int xac_test_dirichlet_plane(float* g, float T_val, int x_plane, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g, "xac_test_dirichlet_plane: null pointer");
  XAC_REQUIRE(x_plane >= 0 && x_plane < nx, "xac_test_dirichlet_plane: x_plane %d out of range", x_plane);
  dirichlet_plane_kernel<<<grid_for((long long)ny * nz, kBlock), kBlock, 0, as_stream(stream)>>>(g, T_val, x_plane,
                                                                                                 d);
  return post_launch("xac_test_dirichlet_plane");
}

int xac_test_periodic_stream(const float* f_post, float* f_streamed, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_post && f_streamed && f_post != f_streamed, "xac_test_periodic_stream: bad buffers");
  periodic_stream_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_post, f_streamed, d);
  return post_launch("xac_test_periodic_stream");
}

int xac_test_forced_bgk(const float* f_old, const float* f_eq, float* f_new, const int32_t* mask, float tau,
                        float force_x, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_old && f_eq && f_new && mask, "xac_test_forced_bgk: null pointer");
  forced_bgk_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_old, f_eq, f_new, mask, tau, force_x,
                                                                             d);
  return post_launch("xac_test_forced_bgk");
}

int xac_test_periodic_stream_solids(const float* f_post, float* f_streamed, const int32_t* mask, int nx, int ny,
                                    int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_post && f_streamed && mask && f_post != f_streamed, "xac_test_periodic_stream_solids: bad buffers");
  periodic_stream_solids_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_post, f_streamed, mask,
                                                                                          d);
  return post_launch("xac_test_periodic_stream_solids");
}

int xac_test_couette_stream(const float* f_post, float* f_streamed, const int32_t* mask, float u_wall_x, int nx,
                            int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_post && f_streamed && mask && f_post != f_streamed, "xac_test_couette_stream: bad buffers");
  couette_stream_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_post, f_streamed, mask, u_wall_x,
                                                                                 d);
  return post_launch("xac_test_couette_stream");
}

// FP64 solve of src/simulation.py:60-100 (cold start, then the six-kernel step) in the reference layout, every
// operator above instantiated in double: the FP64 oracle on the GPU for the error of the reduced-precision storage
// forms. Inputs are prepared as the reference prepares them (the heat map normalised to its maximum in float32, the
// thermal taus derived in double).
int xac_reference_run_fp64(const xac_desc* desc, int steps, double* rho_out, double* u_out, double* T_out,
                           void* stream) {
  XAC_REQUIRE(desc && desc->mask, "xac_reference_run_fp64: null descriptor or mask");
  XAC_REQUIRE(steps >= 0, "xac_reference_run_fp64: negative step count %d", steps);
  XAC_REQUIRE(desc->nx >= 1 && desc->ny >= 1 && desc->nz >= 1, "xac_reference_run_fp64: bad lattice size");
  XAC_REQUIRE(desc->tau_fluid > 0.5 && desc->Pr > 0, "xac_reference_run_fp64: tau_fluid must exceed 0.5, Pr > 0");
  const int nx = desc->nx, ny = desc->ny, nz = desc->nz;
  const Dims d{nx, ny, nz, (long long)nx * ny * nz};
  const size_t n = (size_t)d.n;
  for (size_t c = 0; c < n; ++c)
    XAC_REQUIRE(desc->mask[c] >= 0 && desc->mask[c] <= 3, "xac_reference_run_fp64: mask value %d is not a BC label",
                (int)desc->mask[c]);
  // simulation.py:77-86: the map (default 1 on the z = 0 plane) divided by its maximum, in float32
  std::vector<float> hs32(n, 0.0f);
  if (desc->heat_source) {
    std::memcpy(hs32.data(), desc->heat_source, n * sizeof(float));
  } else {
    for (size_t xy = 0; xy < (size_t)nx * ny; ++xy) hs32[xy * nz] = 1.0f;
  }
  float mx = -INFINITY;
  for (float v : hs32) mx = v > mx ? v : mx;
  if (mx > 0.0f)
    for (float& v : hs32) v = v / mx;
  std::vector<double> hs(hs32.begin(), hs32.end());
  const double tau_th_f = 0.5 + ((desc->tau_fluid - 0.5) / desc->Pr);  // simulation.py:70-71
  const double tau_th_s = 0.5 + desc->k_ratio * (tau_th_f - 0.5);
  cudaStream_t s = as_stream(stream);
  double *f0 = nullptr, *f1 = nullptr, *g0 = nullptr, *g1 = nullptr, *rho = nullptr, *u = nullptr, *T = nullptr,
         *hsd = nullptr, *uin = nullptr;
  int32_t* mask = nullptr;
  auto release = [&]() {
    for (void* p : {(void*)f0, (void*)f1, (void*)g0, (void*)g1, (void*)rho, (void*)u, (void*)T, (void*)hsd,
                    (void*)uin, (void*)mask})
      cudaFree(p);
  };
  cudaError_t e = cudaSuccess;
  for (double** p : {&f0, &f1, &g0, &g1})
    if (e == cudaSuccess) e = cudaMalloc(p, kQ * n * sizeof(double));
  for (double** p : {&rho, &T, &hsd})
    if (e == cudaSuccess) e = cudaMalloc(p, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&u, 3 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&uin, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&mask, n * sizeof(int32_t));
  if (e != cudaSuccess) {
    release();
    return cuda_status(e, "xac_reference_run_fp64: allocation");
  }
  const unsigned grid = grid_for(d.n, kBlock);
  const double u_in = desc->u_inlet;
  fill_kernel<double><<<grid, kBlock, 0, s>>>(rho, 1.0, d.n);
  fill_kernel<double><<<grid_for(3 * d.n, kBlock), kBlock, 0, s>>>(u, 0.0, 3 * d.n);
  fill_kernel<double><<<grid, kBlock, 0, s>>>(T, desc->t_inlet, d.n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mask, desc->mask, n * sizeof(int32_t), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hsd, hs.data(), n * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(uin, &u_in, sizeof(double), cudaMemcpyHostToDevice, s);
  // simulation.py:89-90 cold start
  equilibrium_kernel<double, true><<<grid, kBlock, 0, s>>>(T, u, mask, g0, d);
  equilibrium_kernel<double, false><<<grid, kBlock, 0, s>>>(rho, u, nullptr, f0, d);
  // simulation.py:93-100, one replay of the six-kernel graph per step
  for (int k = 0; k < steps && e == cudaSuccess; ++k) {
    fused_collision_kernel<double><<<grid, kBlock, 0, s>>>(f0, rho, u, f1, mask, desc->tau_fluid, d);
    streaming_kernel<double><<<grid, kBlock, 0, s>>>(f1, f0, mask, uin, desc->rho_outlet, d);
    macroscopic_kernel<double><<<grid, kBlock, 0, s>>>(f0, rho, u, d);
    thermal_collision_kernel<double, true><<<grid, kBlock, 0, s>>>(g0, nullptr, u, T, g1, mask, tau_th_f, tau_th_s,
                                                                   hsd, desc->heat_power, d);
    thermal_streaming_kernel<double><<<grid, kBlock, 0, s>>>(g1, g0, mask, desc->t_inlet, d);
    thermal_macroscopic_kernel<double><<<grid, kBlock, 0, s>>>(g0, T, d);
    if ((k & 255) == 255) e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess && rho_out) e = cudaMemcpyAsync(rho_out, rho, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && u_out) e = cudaMemcpyAsync(u_out, u, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && T_out) e = cudaMemcpyAsync(T_out, T, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  release();
  if (e != cudaSuccess) return cuda_status(e, "xac_reference_run_fp64");
  return XAC_OK;
}

}  // extern "C"
