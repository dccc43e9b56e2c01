// Deterministic FP64 reductions over a 3-D field view: the stats of src/fluid_engine3d.py:277-312 and
// src/thermal_engine3d.py:226-243 (which the reference accumulates with float atomics in no fixed order)
// and the scalar metrics of generate_dataset.py:57-179. Each block reduces its cells with warp shuffles
// into one row of partials; a single-block pass combines the rows in block order.
#pragma once

#include "lattice_kernels.cuh"

namespace xac {

// A read-only view of rho, u, T and the cell labels in either layout.
struct FieldView {
  const float* rho;
  const float* ux;
  const float* uy;
  const float* uz;
  int ustride;  // element stride between cells of one u component (3 = AoS vec3, 1 = SoA)
  const float* T;
  const int32_t* mask;   // reference labels, or
  const uint32_t* link;  // packed link words (internal layout)
  long long sx, sy, sz;  // element strides of the scalar fields along x, y, z
  int nx, ny, nz;
};

__device__ __forceinline__ int view_type(const FieldView& v, long long cell) {
  return v.mask ? (int)v.mask[cell] : link_type(v.link[cell]);
}

enum ReduceOp : int { kSum = 0, kMax = 1, kMin = 2 };

template <int K>
struct ReduceSpec {
  int op[K];
};

__device__ __forceinline__ double combine(int op, double a, double b) {
  return op == kSum ? a + b : (op == kMax ? fmax(a, b) : fmin(a, b));
}
__device__ __forceinline__ double identity(int op) {
  return op == kSum ? 0.0 : (op == kMax ? -INFINITY : INFINITY);
}

// Block-level reduction of K values per thread; thread 0 writes out[0..K).
template <int K>
__device__ __forceinline__ void block_reduce(double (&acc)[K], const ReduceSpec<K>& spec, double* out) {
  __shared__ double sm[32][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = combine(spec.op[k], v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sm[warp][k] = v;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double v = lane < nw ? sm[lane][k] : identity(spec.op[k]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = combine(spec.op[k], v, __shfl_down_sync(0xffffffffu, v, o));
      if (lane == 0) out[k] = v;
    }
  }
}

// Combine nrows rows of K partials; one warp per column, lanes stride the rows and a fixed shuffle tree
// finishes, so the result does not depend on scheduling (launch with 32*K threads).
template <int K>
__global__ void combine_rows_kernel(const double* __restrict__ rows, int nrows, ReduceSpec<K> spec,
                                    double* __restrict__ out) {
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= K) return;
  const int op = spec.op[k];
  double v = identity(op);
  // a lane combines rows lane, lane+32, lane+64, ... in that order; eight loads are issued before they are
  // combined, which hides their latency without changing the order
  for (int r0 = lane; r0 < nrows; r0 += 32 * 8) {
    double t[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = r0 + 32 * j;
      t[j] = r < nrows ? rows[(long long)r * K + k] : identity(op);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (r0 + 32 * j < nrows) v = combine(op, v, t[j]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = combine(op, v, __shfl_down_sync(0xffffffffu, v, o));
  if (lane == 0) out[k] = v;
}

// ---- convergence / divergence stats (XAC_ST_* order) --------------------------------------------
constexpr int kNStats = XAC_NSTATS;

inline ReduceSpec<kNStats> stats_spec() {
  ReduceSpec<kNStats> s{};
  for (int k = 0; k < kNStats; ++k) s.op[k] = kSum;
  s.op[XAC_ST_MAX_V] = kMax;
  s.op[XAC_ST_MAX_T] = kMax;
  return s;
}

// Stats of one cell added into acc (XAC_ST_* slots). Field reads go through L2 (they may have been written
// earlier in the same launch by other blocks).
__device__ __forceinline__ void stats_accumulate(const FieldView& v, int x, int y, int z, double (&acc)[kNStats]) {
  const long long cell = x * v.sx + y * v.sy + z * v.sz;
  const int m = view_type(v, cell);
  const float ux = __ldcg(v.ux + cell * v.ustride), uy = __ldcg(v.uy + cell * v.ustride),
              uz = __ldcg(v.uz + cell * v.ustride);
  const float vsq = (ux * ux + uy * uy) + uz * uz;
  const float vmag = sqrtf(vsq);
  const float r = __ldcg(v.rho + cell), T = __ldcg(v.T + cell);
  if (!isfinite(vmag) || !isfinite(T)) acc[XAC_ST_NONFINITE] += 1.0;
  acc[XAC_ST_SUM_KE] += (double)vsq;
  if (m != kSolid) {
    acc[XAC_ST_MAX_V] = fmax(acc[XAC_ST_MAX_V], (double)vmag);
    acc[XAC_ST_SUM_V] += (double)vmag;
    acc[XAC_ST_COUNT] += 1.0;
    acc[XAC_ST_SUM_RHO] += (double)r;
  }
  if (x == 1) {
    acc[XAC_ST_SUM_RHO_IN] += (double)r;
    acc[XAC_ST_C_IN] += 1.0;
  }
  if (x == v.nx - 2) {
    acc[XAC_ST_SUM_RHO_OUT] += (double)r;
    acc[XAC_ST_C_OUT] += 1.0;
  }
  if (m == kOutlet) {
    acc[XAC_ST_SUM_UX_OUT] += (double)ux;
    acc[XAC_ST_C_OUTLET] += 1.0;
    acc[XAC_ST_Q_OUT] += (double)(ux * T);
    acc[XAC_ST_Q_OUT_COUNT] += 1.0;
  }
  acc[XAC_ST_MAX_T] = fmax(acc[XAC_ST_MAX_T], (double)T);
  acc[XAC_ST_SUM_T] += (double)T;
  acc[XAC_ST_COUNT_T] += 1.0;
}

// One row of partial stats for the 1024-cell tile `tile` (cells enumerated x fastest). The tile is reduced as 8
// chunks of 128 cells, each by one warp: every lane adds its 4 cells (lane, lane+32, lane+64, lane+96 of the
// chunk) in order, then a fixed butterfly combines the lanes; the chunks are combined in order by one thread.
// The row does not depend on the block size that computes it. Every thread of the block must call.
constexpr int kStatsTile = 1024;   // cells per partial row
constexpr int kStatsChunk = 128;   // cells per warp chunk
constexpr int kStatsBlock = 256;   // threads of the kernels that compute the rows
__device__ __forceinline__ void stats_tile_row(const FieldView& v, long long tile, const ReduceSpec<kNStats>& spec,
                                               double* __restrict__ row) {
  __shared__ double chunk[kStatsTile / kStatsChunk][kNStats];
  const long long n = (long long)v.nx * v.ny * v.nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int ch = warp; ch < kStatsTile / kStatsChunk; ch += nwarps) {
    double acc[kNStats];
#pragma unroll
    for (int k = 0; k < kNStats; ++k) acc[k] = identity(spec.op[k]);
#pragma unroll
    for (int j = 0; j < kStatsChunk / 32; ++j) {
      const long long i = tile * kStatsTile + ch * kStatsChunk + j * 32 + lane;
      if (i < n) {  // lattices stay below 2^31 cells: 32-bit decomposition
        const unsigned iu = (unsigned)i, nx = (unsigned)v.nx, ny = (unsigned)v.ny;
        const unsigned t = iu / nx;
        stats_accumulate(v, (int)(iu - t * nx), (int)(t % ny), (int)(t / ny), acc);
      }
    }
#pragma unroll
    for (int k = 0; k < kNStats; ++k) {
      double a = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a = combine(spec.op[k], a, __shfl_xor_sync(0xffffffffu, a, o));
      if (lane == 0) chunk[ch][k] = a;
    }
  }
  __syncthreads();
  if (threadIdx.x < kNStats) {
    const int k = threadIdx.x;
    double a = identity(spec.op[k]);
    for (int ch = 0; ch < kStatsTile / kStatsChunk; ++ch) a = combine(spec.op[k], a, chunk[ch][k]);
    row[k] = a;
  }
  __syncthreads();
}

inline long long stats_tiles(long long ncell) { return (ncell + kStatsTile - 1) / kStatsTile; }

static __global__ void __launch_bounds__(256) stats_partials_kernel(FieldView v, ReduceSpec<kNStats> spec,
                                                             double* __restrict__ rows) {
  stats_tile_row(v, blockIdx.x, spec, rows + (long long)blockIdx.x * kNStats);
}

// ---- scalar metrics (generate_dataset.py:57-179) ------------------------------------------------
enum MetricSlot : int {
  kM_QVOL = 0,       // sum ux over outlet-labelled cells of plane x = nx-1
  kM_N_IN,           // non-solid cells of plane x = 1
  kM_RHO_IN,         //   sum rho there
  kM_N_OUT,          // non-solid cells of plane x = nx-2
  kM_RHO_OUT,        //   sum rho there
  kM_TS_MAX,         // floor z = 0, x in [buf, buf+core_nx), y < core_ny
  kM_TS_SUM,
  kM_TS_SQ,
  kM_TS_MIN,
  kM_TS_N,
  kM_QOUT,           // sum ux*T over outlet-labelled cells of plane x = nx-1
  kM_TF_SUM,         // T over non-solid cells of the core box [buf, nx-buf) x [1, ny-1) x [4, nz-2)
  kM_TF_N,
  kM_RHO1_ALL,       // sum rho over all cells of plane x = 1
  kM_RHO2_ALL,       // sum rho over all cells of plane x = nx-2
  kM_MAXV,           // max |u| over all cells
  kM_MAXT,
  kM_TSUM_ALL,
  kM_VFLUID,         // non-solid cells of the core box (compute_hydraulic_diameter)
  kM_FACES,          // solid/non-solid face pairs inside the core box
  kM_CORE_SOLID,     // solid cells in x in [buf, nx-buf) (compute_porosity)
  kNMetrics
};

inline ReduceSpec<kNMetrics> metric_spec() {
  ReduceSpec<kNMetrics> s{};
  for (int k = 0; k < kNMetrics; ++k) s.op[k] = kSum;
  s.op[kM_TS_MAX] = kMax;
  s.op[kM_TS_MIN] = kMin;
  s.op[kM_MAXV] = kMax;
  s.op[kM_MAXT] = kMax;
  return s;
}

struct MetricBox {
  int buf, core_nx, core_ny;
};

static __global__ void __launch_bounds__(256) metric_partials_kernel(FieldView v, MetricBox b, ReduceSpec<kNMetrics> spec,
                                                              double* __restrict__ rows) {
  double acc[kNMetrics];
#pragma unroll
  for (int k = 0; k < kNMetrics; ++k) acc[k] = identity(spec.op[k]);
  const long long n = (long long)v.nx * v.ny * v.nz;
  const int nx = v.nx, ny = v.ny, nz = v.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long t = i / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    const long long cell = x * v.sx + y * v.sy + z * v.sz;
    const int m = view_type(v, cell);
    const bool solid = m == kSolid;
    const float ux = v.ux[cell * v.ustride], uy = v.uy[cell * v.ustride], uz = v.uz[cell * v.ustride];
    const float r = v.rho[cell], T = v.T[cell];
    if (x == nx - 1 && m == kOutlet) {
      acc[kM_QVOL] += (double)ux;
      acc[kM_QOUT] += (double)ux * (double)T;
    }
    if (x == 1) {
      acc[kM_RHO1_ALL] += (double)r;
      if (!solid) {
        acc[kM_N_IN] += 1.0;
        acc[kM_RHO_IN] += (double)r;
      }
    }
    if (x == nx - 2) {
      acc[kM_RHO2_ALL] += (double)r;
      if (!solid) {
        acc[kM_N_OUT] += 1.0;
        acc[kM_RHO_OUT] += (double)r;
      }
    }
    if (z == 0 && x >= b.buf && x < b.buf + b.core_nx && y < b.core_ny) {
      acc[kM_TS_MAX] = fmax(acc[kM_TS_MAX], (double)T);
      acc[kM_TS_MIN] = fmin(acc[kM_TS_MIN], (double)T);
      acc[kM_TS_SUM] += (double)T;
      acc[kM_TS_SQ] += (double)T * (double)T;
      acc[kM_TS_N] += 1.0;
    }
    const bool in_core = x >= b.buf && x < nx - b.buf && y >= 1 && y < ny - 1 && z >= 4 && z < nz - 2;
    if (in_core) {
      if (!solid) {
        acc[kM_TF_SUM] += (double)T;
        acc[kM_TF_N] += 1.0;
        acc[kM_VFLUID] += 1.0;
      }
      // faces to the +x, +y, +z neighbour when it is inside the core box too
      if (x + 1 < nx - b.buf && (view_type(v, cell + v.sx) == kSolid) != solid) acc[kM_FACES] += 1.0;
      if (y + 1 < ny - 1 && (view_type(v, cell + v.sy) == kSolid) != solid) acc[kM_FACES] += 1.0;
      if (z + 1 < nz - 2 && (view_type(v, cell + v.sz) == kSolid) != solid) acc[kM_FACES] += 1.0;
    }
    if (x >= b.buf && x < nx - b.buf && solid) acc[kM_CORE_SOLID] += 1.0;
    const double vm = sqrt((double)ux * ux + (double)uy * uy + (double)uz * uz);
    acc[kM_MAXV] = fmax(acc[kM_MAXV], vm);
    acc[kM_MAXT] = fmax(acc[kM_MAXT], (double)T);
    acc[kM_TSUM_ALL] += (double)T;
  }
  block_reduce<kNMetrics>(acc, spec, rows + (long long)blockIdx.x * kNMetrics);
}

// ---- physical validators (analyze_dataset.py:184-323) ------------------------------------------
enum ValidateSlot : int {
  kV_MDOT_IN = 0,  // sum rho*ux over non-solid cells of plane x = 1            (:201-206)
  kV_MDOT_OUT,     // the same over plane x = nx-2
  kV_MAXV,         // max |u| over non-solid cells                             (:214-216)
  kV_RHODEV,       // max |rho - 1| over non-solid cells                       (:222)
  kV_TMIN,         // min T over non-solid cells                               (:229)
  kV_NFLUID,       // non-solid cells
  kV_RHO1_ALL,     // sum rho over all cells of plane x = 1                    (:236-238)
  kV_RHO2_ALL,     // the same over plane x = nx-2
  kV_DIV_SUM,      // sum |div u| over non-solid interior cells (central differences, :257-263)
  kV_DIV_MAX,
  kV_DIV_N,
  kV_QSRC,         // sum of the injected source heat_power * map over all cells
  kV_ADV_IN,       // sum ux over inlet cells of plane x = 0                   (:294-297)
  kV_ADV_OUT,      // sum ux*T over outlet cells of plane x = nx-1
  kV_DIFF_IN,      // sum over plane x = 1 of -k(cell) * (T[1] - T[0])          (:300-306)
  kV_DIFF_OUT,     // sum over plane x = nx-2 of -k(cell) * (T[nx-1] - T[nx-2])
  kNValidate
};

inline ReduceSpec<kNValidate> validate_spec() {
  ReduceSpec<kNValidate> s{};
  for (int k = 0; k < kNValidate; ++k) s.op[k] = kSum;
  s.op[kV_MAXV] = kMax;
  s.op[kV_RHODEV] = kMax;
  s.op[kV_TMIN] = kMin;
  s.op[kV_DIV_MAX] = kMax;
  return s;
}

// q: heat source per cell (compact order of the view, may be null); k_fluid / k_solid: thermal conductivities
// (tau_th - 0.5) / 3 of the two phases (:280-281). Per-cell differences are formed in float32 like the
// reference's float32 arrays; sums are FP64.
static __global__ void __launch_bounds__(256) validate_partials_kernel(FieldView v, const float* __restrict__ q,
                                                                double k_fluid, double k_solid,
                                                                ReduceSpec<kNValidate> spec,
                                                                double* __restrict__ rows) {
  double acc[kNValidate];
#pragma unroll
  for (int k = 0; k < kNValidate; ++k) acc[k] = identity(spec.op[k]);
  const long long n = (long long)v.nx * v.ny * v.nz;
  const int nx = v.nx, ny = v.ny, nz = v.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long t = i / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    const long long cell = x * v.sx + y * v.sy + z * v.sz;
    const int m = view_type(v, cell);
    const bool fluid = m != kSolid;
    const float ux = v.ux[cell * v.ustride], uy = v.uy[cell * v.ustride], uz = v.uz[cell * v.ustride];
    const float r = v.rho[cell], T = v.T[cell];
    if (q) acc[kV_QSRC] += (double)q[i];
    if (x == 1) {
      acc[kV_RHO1_ALL] += (double)r;
      if (fluid) acc[kV_MDOT_IN] += (double)(r * ux);
      acc[kV_DIFF_IN] += -(fluid ? k_fluid : k_solid) * (double)(T - v.T[cell - v.sx]);
    }
    if (x == nx - 2) {
      acc[kV_RHO2_ALL] += (double)r;
      if (fluid) acc[kV_MDOT_OUT] += (double)(r * ux);
      acc[kV_DIFF_OUT] += -(fluid ? k_fluid : k_solid) * (double)(v.T[cell + v.sx] - T);
    }
    if (x == 0 && m == kInlet) acc[kV_ADV_IN] += (double)ux;
    if (x == nx - 1 && m == kOutlet) acc[kV_ADV_OUT] += (double)(ux * T);
    if (fluid) {
      acc[kV_NFLUID] += 1.0;
      const float vm = sqrtf(ux * ux + uy * uy + uz * uz);
      acc[kV_MAXV] = fmax(acc[kV_MAXV], (double)vm);
      acc[kV_RHODEV] = fmax(acc[kV_RHODEV], (double)fabsf(r - 1.0f));
      acc[kV_TMIN] = fmin(acc[kV_TMIN], (double)T);
      if (x >= 1 && x < nx - 1 && y >= 1 && y < ny - 1 && z >= 1 && z < nz - 1) {
        const long long us = v.ustride;
        const float dux = (v.ux[(cell + v.sx) * us] - v.ux[(cell - v.sx) * us]) / 2.0f;
        const float duy = (v.uy[(cell + v.sy) * us] - v.uy[(cell - v.sy) * us]) / 2.0f;
        const float duz = (v.uz[(cell + v.sz) * us] - v.uz[(cell - v.sz) * us]) / 2.0f;
        const double d = fabs((double)((dux + duy) + duz));
        acc[kV_DIV_SUM] += d;
        acc[kV_DIV_MAX] = fmax(acc[kV_DIV_MAX], d);
        acc[kV_DIV_N] += 1.0;
      }
    }
  }
  block_reduce<kNValidate>(acc, spec, rows + (long long)blockIdx.x * kNValidate);
}

}  // namespace xac
