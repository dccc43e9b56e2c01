// Unfused per-operator kernels in the reference layout f[19][nx][ny][nz] (z fastest).
// Each kernel restates one Warp kernel of the reference with the same operand order, so that
// validate_analytical.py-style drivers port 1:1 and every operator can be checked on its own.
// One thread per cell; consecutive threads walk z, the contiguous axis of that layout.
#include <cstdarg>
#include <cmath>

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

// src/fluid_engine3d.py:58-80 (also the thermal twin with T in place of rho, thermal_engine3d.py:7-47)
template <bool kThermal>
__global__ void equilibrium_kernel(const float* __restrict__ scal, const float* __restrict__ u,
                                   const int32_t* __restrict__ mask, float* __restrict__ out, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  float s = scal[c];
  float ux = u[3 * c], uy = u[3 * c + 1], uz = u[3 * c + 2];
  if (kThermal && mask[c] == kSolid) { ux = 0.0f; uy = 0.0f; uz = 0.0f; }
  float usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    float eu;
    switch (i) {
#define XAC_CASE(I) case I: eu = edotu<I>(ux, uy, uz); break;
      XAC_CASE(0) XAC_CASE(1) XAC_CASE(2) XAC_CASE(3) XAC_CASE(4) XAC_CASE(5) XAC_CASE(6) XAC_CASE(7)
      XAC_CASE(8) XAC_CASE(9) XAC_CASE(10) XAC_CASE(11) XAC_CASE(12) XAC_CASE(13) XAC_CASE(14) XAC_CASE(15)
      XAC_CASE(16) XAC_CASE(17) XAC_CASE(18)
#undef XAC_CASE
      default: eu = 0.0f;
    }
    out[(long long)i * d.n + c] = feq_term(w_of(i) * s, eu, usq15);
  }
}

// src/fluid_engine3d.py:85-113
__global__ void macroscopic_kernel(const float* __restrict__ f, float* __restrict__ rho, float* __restrict__ u,
                                   Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  float r = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    float v = f[(long long)i * d.n + c];
    r += v;
    mx += v * (float)ex_of(i);
    my += v * (float)ey_of(i);
    mz += v * (float)ez_of(i);
  }
  rho[c] = r;
  if (r > 1e-10f) {
    u[3 * c] = mx / r;
    u[3 * c + 1] = my / r;
    u[3 * c + 2] = mz / r;
  } else {
    u[3 * c] = 0.0f;
    u[3 * c + 1] = 0.0f;
    u[3 * c + 2] = 0.0f;
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
__global__ void fused_collision_kernel(const float* __restrict__ fo, const float* __restrict__ rho,
                                       const float* __restrict__ u, float* __restrict__ fp,
                                       const int32_t* __restrict__ mask, float tau, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int m = mask[c];
  float omega = 1.0f / tau;
  if (m == kFluid || m == kInlet || m == kOutlet) {
    float r = rho[c];
    float ux = u[3 * c], uy = u[3 * c + 1], uz = u[3 * c + 2];
    float usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float eu;
      switch (i) {
#define XAC_CASE(I) case I: eu = edotu<I>(ux, uy, uz); break;
        XAC_CASE(0) XAC_CASE(1) XAC_CASE(2) XAC_CASE(3) XAC_CASE(4) XAC_CASE(5) XAC_CASE(6) XAC_CASE(7)
        XAC_CASE(8) XAC_CASE(9) XAC_CASE(10) XAC_CASE(11) XAC_CASE(12) XAC_CASE(13) XAC_CASE(14) XAC_CASE(15)
        XAC_CASE(16) XAC_CASE(17) XAC_CASE(18)
#undef XAC_CASE
        default: eu = 0.0f;
      }
      long long k = (long long)i * d.n + c;
      float f = fo[k];
      fp[k] = f - omega * (f - feq_term(w_of(i) * r, eu, usq15));
    }
  } else {
#pragma unroll
    for (int i = 0; i < kQ; ++i) fp[(long long)i * d.n + c] = fo[(long long)i * d.n + c];
  }
}

// src/fluid_engine3d.py:181-272
__global__ void streaming_kernel(const float* __restrict__ fp, float* __restrict__ fs,
                                 const int32_t* __restrict__ mask, const float* __restrict__ u_inlet,
                                 float rho_outlet, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int x, y, z;
  decompose(c, d, x, y, z);
  int m = mask[c];
  const long long N = d.n;
  if (m == kSolid) return;
  if (m == kInlet) {
    float ux_in = u_inlet[0];
    float f0 = fp[c], f2 = fp[2 * N + c], f3 = fp[3 * N + c], f4 = fp[4 * N + c], f5 = fp[5 * N + c];
    float f6 = fp[6 * N + c], f8 = fp[8 * N + c], f10 = fp[10 * N + c], f12 = fp[12 * N + c];
    float f14 = fp[14 * N + c], f15 = fp[15 * N + c], f16 = fp[16 * N + c], f17 = fp[17 * N + c];
    float f18 = fp[18 * N + c];
    float rn = (((((((((f0 + f3) + f4) + f5) + f6) + f15) + f16) + f17) + f18) +
                2.0f * ((((f2 + f8) + f10) + f12) + f14)) /
               (1.0f - ux_in);
    const float c23 = 2.0f / 3.0f, c16 = 1.0f / 6.0f;
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
    float v[kQ];
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      v[i] = fp[(long long)i * N + s];
      sum += v[i];
    }
    if (sum > 1e-6f) {
      float sc = rho_outlet / sum;
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
template <bool kFused>
__global__ void thermal_collision_kernel(const float* __restrict__ go, const float* __restrict__ ge,
                                         const float* __restrict__ u, const float* __restrict__ T,
                                         float* __restrict__ gn, const int32_t* __restrict__ mask, float tau_f,
                                         float tau_s, const float* __restrict__ hs, float power, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  bool solid = mask[c] == kSolid;
  float tau = solid ? tau_s : tau_f;
  float omega = 1.0f / tau;
  float q = hs[c] * power;
  float srcf = 1.0f - 0.5f * omega;
  float t = 0.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f, usq15 = 0.0f;
  if (kFused) {
    t = T[c];
    if (!solid) { ux = u[3 * c]; uy = u[3 * c + 1]; uz = u[3 * c + 2]; }
    usq15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    long long k = (long long)i * d.n + c;
    float g = go[k];
    float geq;
    if (kFused) {
      float eu;
      switch (i) {
#define XAC_CASE(I) case I: eu = edotu<I>(ux, uy, uz); break;
        XAC_CASE(0) XAC_CASE(1) XAC_CASE(2) XAC_CASE(3) XAC_CASE(4) XAC_CASE(5) XAC_CASE(6) XAC_CASE(7)
        XAC_CASE(8) XAC_CASE(9) XAC_CASE(10) XAC_CASE(11) XAC_CASE(12) XAC_CASE(13) XAC_CASE(14) XAC_CASE(15)
        XAC_CASE(16) XAC_CASE(17) XAC_CASE(18)
#undef XAC_CASE
        default: eu = 0.0f;
      }
      geq = feq_term(w_of(i) * t, eu, usq15);
    } else {
      geq = ge[k];
    }
    float v = g - omega * (g - geq);
    if (q > 0.0f) v += (w_of(i) * srcf) * q;
    gn[k] = v;
  }
}

// src/thermal_engine3d.py:147-211
__global__ void thermal_streaming_kernel(const float* __restrict__ gp, float* __restrict__ gs,
                                         const int32_t* __restrict__ mask, float T_in, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  int x, y, z;
  decompose(c, d, x, y, z);
  int m = mask[c];
  const long long N = d.n;
  if (m == kInlet) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) gs[(long long)i * N + c] = w_of(i) * T_in;
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
    float v;
    if (sx < 0) v = w_of(i) * T_in;
    else if (sx >= d.nx) v = gp[(long long)i * N + c];
    else if (sy < 0 || sy >= d.ny || sz < 0 || sz >= d.nz) v = gp[(long long)opp_of(i) * N + c];
    else v = gp[(long long)i * N + cell_of(sx, sy, sz, d)];
    gs[(long long)i * N + c] = v;
  }
}

// src/thermal_engine3d.py:214-224
__global__ void thermal_macroscopic_kernel(const float* __restrict__ g, float* __restrict__ T, Dims d) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) s += g[(long long)i * d.n + c];
  T[c] = s;
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
  equilibrium_kernel<false><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(rho, u, nullptr, f_eq, d);
  return post_launch("xac_equilibrium");
}

int xac_macroscopic(const float* f, float* rho, float* u, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f && rho && u, "xac_macroscopic: null pointer");
  macroscopic_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f, rho, u, d);
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
  fused_collision_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_old, rho, u, f_post, mask, tau,
                                                                                  d);
  return post_launch("xac_fused_collision");
}

int xac_stream(const float* f_post, float* f_streamed, const int32_t* mask, const float* u_inlet, float rho_outlet,
               int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(f_post && f_streamed && mask && u_inlet, "xac_stream: null pointer");
  XAC_REQUIRE(f_post != f_streamed, "xac_stream: input and output must be distinct buffers");
  streaming_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(f_post, f_streamed, mask, u_inlet,
                                                                            rho_outlet, d);
  return post_launch("xac_stream");
}

int xac_thermal_equilibrium(const float* u, const float* T, float* g_eq, const int32_t* mask, int nx, int ny, int nz,
                            void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(u && T && g_eq && mask, "xac_thermal_equilibrium: null pointer");
  equilibrium_kernel<true><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(T, u, mask, g_eq, d);
  return post_launch("xac_thermal_equilibrium");
}

int xac_thermal_bgk_collision(const float* g_old, const float* g_eq, float* g_new, const int32_t* mask,
                              float tau_fluid, float tau_solid, const float* heat_source, float heat_power, int nx,
                              int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_old && g_eq && g_new && mask && heat_source, "xac_thermal_bgk_collision: null pointer");
  thermal_collision_kernel<false><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(
      g_old, g_eq, nullptr, nullptr, g_new, mask, tau_fluid, tau_solid, heat_source, heat_power, d);
  return post_launch("xac_thermal_bgk_collision");
}

int xac_fused_thermal_collision(const float* g_old, const float* u, const float* T, float* g_new,
                                const int32_t* mask, float tau_fluid, float tau_solid, const float* heat_source,
                                float heat_power, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_old && u && T && g_new && mask && heat_source, "xac_fused_thermal_collision: null pointer");
  thermal_collision_kernel<true><<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(
      g_old, nullptr, u, T, g_new, mask, tau_fluid, tau_solid, heat_source, heat_power, d);
  return post_launch("xac_fused_thermal_collision");
}

int xac_thermal_stream(const float* g_post, float* g_streamed, const int32_t* mask, float T_inlet, int nx, int ny,
                       int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g_post && g_streamed && mask, "xac_thermal_stream: null pointer");
  XAC_REQUIRE(g_post != g_streamed, "xac_thermal_stream: input and output must be distinct buffers");
  thermal_streaming_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(g_post, g_streamed, mask,
                                                                                    T_inlet, d);
  return post_launch("xac_thermal_stream");
}

int xac_thermal_macroscopic(const float* g, float* T, int nx, int ny, int nz, void* stream) {
  XAC_DIMS();
  XAC_REQUIRE(g && T, "xac_thermal_macroscopic: null pointer");
  thermal_macroscopic_kernel<<<grid_for(d.n, kBlock), kBlock, 0, as_stream(stream)>>>(g, T, d);
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

}  // extern "C"
