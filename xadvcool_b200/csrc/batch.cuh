// Batched persistent solve: many designs of uneven lattice sizes advanced by ONE cooperative launch.
//
// Every resident block loops over steps. In a step it takes tiles (one cell per thread, `blockDim` cells per
// tile) from the concatenated tile list of the still-active designs, then meets the other blocks at a grid
// barrier. On a stats step (every stats_every steps, src/simulation.py:123) the blocks also finalise T and
// reduce the stats of every active design into 1024-cell tile rows, one block per design combines its rows and
// applies the relative-rate convergence test and divergence guard of src/simulation.py:134-156, and converged
// or diverged designs retire: the next steps skip their tiles and the remaining work is redistributed over all
// blocks. The per-tile reduction is the single-lattice one, so a design solved in a batch takes exactly the
// steps and ends with exactly the bits of the same design solved alone.
//
// Designs may join a running batch (xac_batch_admit): each keeps the global step at which it started, always a
// multiple of stats_every, and everything that depends on a design's own step count (its first step, its buffer
// parity, its step limit, the convergence rule's minimum and the pump's start) is taken relative to that start.
// Designs of xac_batch_run all start at step 0.
//
// The barrier waits are bounded: a wait that exceeds the spin limit records XAC_ETIMEOUT in the control block
// and every block leaves the kernel.
#pragma once

#include "lattice_kernels.cuh"
#include "reductions.cuh"

namespace xac {

constexpr int kMaxBatch = 1024;

struct BatchDesign {
  StepParams p;
  const void* P[2];
  const void* Q[2];
  const uint32_t* link;
  const float* qsrc;
  float* u_in;  // inlet velocity (device): the constant-power pump updates it
  float *rho, *ux, *uy, *uz, *T;
  uint32_t ncell, tiles, stat_tiles, row_base;
  long long min_steps;
  long long start;  // global step at which the design joined the batch (a multiple of stats_every)
  // run state, owned by the device during a run
  int active, converged, diverged, pad;
  long long steps;
  double prev_ke, prev_max_T, prev_Q, d_ke, dT, dQ;
  double last[kNStats];
};

struct BatchCtl {
  unsigned bar_count;
  unsigned bar_gen;
  int err;
  int all_done;
  long long step;   // steps done by every active design
  int n_active;
  int pad;
  uint32_t active[kMaxBatch];
  uint32_t prefix[kMaxBatch + 1];       // step tiles of active designs, exclusive prefix
  uint32_t stat_prefix[kMaxBatch + 1];  // stats tiles of active designs, exclusive prefix
};

// Bounded sense-counting grid barrier over the co-resident blocks of a cooperative launch.
__device__ __forceinline__ bool grid_sync(BatchCtl* ctl, unsigned long long spin_limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &ctl->bar_gen;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&ctl->bar_count, 0u);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      unsigned long long spins = 0;
      while (*gen == g) {
        if (++spins > spin_limit) {
          atomicExch(&ctl->err, XAC_ETIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)&ctl->err == 0;
}

__device__ __forceinline__ int find_slot(const uint32_t* prefix, int n, uint32_t t) {
  int lo = 0, hi = n;  // prefix[lo] <= t < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldcg(prefix + mid) <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}
// the same search over a copy of the prefix in shared memory, starting from slot lo (prefix[lo] <= t)
__device__ __forceinline__ int find_slot_shared(const uint32_t* prefix, int lo, int n, uint32_t t) {
  int hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// tile = blockDim consecutive row positions (rows of `pitch` positions, x >= nx padding), one per thread
template <typename SP, typename SQ, bool kMacro, bool kOwn>
__device__ __forceinline__ void batch_step_tile(const BatchDesign& d, uint32_t tile, int cur) {
  const uint32_t pos = tile * blockDim.x + threadIdx.x;
  const uint32_t pitch = (uint32_t)d.p.g.pitch;
  const uint32_t r = pos / pitch, x = pos - r * pitch;
  if (r >= (uint32_t)d.p.g.rows) return;  // whole warps (the pitch is a multiple of 32)
  const bool valid = x < (uint32_t)d.p.g.nx;
  const uint32_t c = r * (uint32_t)d.p.g.nx + x;
  const uint32_t lw = valid ? __ldg(d.link + c) : ((uint32_t)kSolid << kTypeShift);
  const int lane = threadIdx.x & 31;
  const uint32_t e0 = pop_base(r, x, d.p.g, (int)pitch);
  coupled_cell<SP, SQ, kMacro, kOwn, 1, 0>(c, r, x, e0, (const SP*)d.P[cur], (SP*)d.P[cur ^ 1], (const SQ*)d.Q[cur],
                                            (SQ*)d.Q[cur ^ 1], d.qsrc, d.u_in, d.rho, d.ux, d.uy, d.uz, d.T, d.p,
                                            valid, lw);
  pad_fill<SQ, 0>(valid, __ballot_sync(0xffffffffu, valid), lane, (SQ*)d.Q[cur ^ 1], e0, d.p.g);
}

struct BatchRun {
  int steps;           // steps in this launch
  long long max_steps;
  int stats_every;
  double tol_ke, tol_T;
  unsigned long long spin_limit;
  int constant_power;  // pump_mode == "constant_power" (src/simulation.py:139-146)
  double target_power;
};

template <typename SP, typename SQ>
#ifndef XAC_BATCH_MIN_BLOCKS
#define XAC_BATCH_MIN_BLOCKS 4  // at most 64 registers; 3 and 5 blocks per SM measured slower
#endif
__global__ void __launch_bounds__(256, XAC_BATCH_MIN_BLOCKS) batch_persistent_kernel(BatchDesign* __restrict__ D, BatchCtl* __restrict__ ctl,
                                                               double* __restrict__ rows, BatchRun run) {
  __shared__ double st[kNStats];
  ReduceSpec<kNStats> spec;
#pragma unroll
  for (int k = 0; k < kNStats; ++k) spec.op[k] = (k == XAC_ST_MAX_V || k == XAC_ST_MAX_T) ? kMax : kSum;
  __shared__ BatchDesign dsh;
  __shared__ uint32_t s_prefix[kMaxBatch + 1];
  long long step = ctl->step;
  for (int it = 0; it < run.steps; ++it) {
    if (*(volatile int*)&ctl->all_done || *(volatile int*)&ctl->err) break;
    // control-block fields change during the launch (retirement): read them through L2
    const int na = *(volatile int*)&ctl->n_active;
    const uint32_t total = __ldcg(ctl->prefix + na);
    const long long s1 = step + 1;
    const bool stats = (s1 % run.stats_every) == 0;  // designs start on stats boundaries: the same for each
    // ---- one coupled step of every active design
    // The tile prefix of the active designs goes to shared memory once per step. A block's tiles t rise, so
    // their design slot k only moves forward: the search starts from the last slot, and the design's
    // descriptor is copied to shared memory only when the slot changes.
    for (int i = threadIdx.x; i <= na; i += blockDim.x) s_prefix[i] = __ldcg(ctl->prefix + i);
    __syncthreads();
    int kcur = -1;
    for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
      const int k = (kcur >= 0 && t < s_prefix[kcur + 1]) ? kcur : find_slot_shared(s_prefix, kcur < 0 ? 0 : kcur, na, t);
      if (k != kcur) {
        __syncthreads();  // the previous design's tiles are done with dsh
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&D[__ldcg(ctl->active + k)]);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&dsh);
        for (uint32_t w = threadIdx.x; w < sizeof(BatchDesign) / 4; w += blockDim.x) dst[w] = __ldcg(src + w);
        __syncthreads();
        kcur = k;
      }
      const uint32_t tile = t - s_prefix[k];
      const BatchDesign& d = dsh;
      const long long ls = step - d.start;  // the design's own step count
      const bool own = ls == 0;
      const bool macro = stats || ls + 1 == run.max_steps;
      const int cur = (int)(ls & 1);
      if (own) {
        if (macro) batch_step_tile<SP, SQ, true, true>(d, tile, cur);
        else batch_step_tile<SP, SQ, false, true>(d, tile, cur);
      } else if (macro) {
        batch_step_tile<SP, SQ, true, false>(d, tile, cur);
      } else {
        batch_step_tile<SP, SQ, false, false>(d, tile, cur);
      }
    }
    if (!grid_sync(ctl, run.spin_limit)) break;
    if (stats) {
      // ---- T of the new state and 1024-cell tile rows of stats
      const uint32_t stotal = __ldcg(ctl->stat_prefix + na);
      for (uint32_t t = blockIdx.x; t < stotal; t += gridDim.x) {
        const int k = find_slot(ctl->stat_prefix, na, t);
        const BatchDesign& d = D[__ldcg(ctl->active + k)];  // geometry and pointers never change
        const uint32_t tile = t - __ldcg(ctl->stat_prefix + k);
        const SQ* Qnew = (const SQ*)d.Q[((step - d.start) & 1) ^ 1];
        for (uint32_t c = tile * kStatsTile + threadIdx.x; c < (tile + 1) * kStatsTile && c < d.ncell;
             c += blockDim.x)
          d.T[c] = finalize_T_cell<SQ, true>(Qnew, d.link, d.p, c);
        __syncthreads();
        FieldView v{};
        v.rho = d.rho;
        v.ux = d.ux;
        v.uy = d.uy;
        v.uz = d.uz;
        v.ustride = 1;
        v.T = d.T;
        v.mask = nullptr;
        v.link = d.link;
        v.sx = 1;
        v.sy = d.p.g.nx;
        v.sz = (long long)d.p.g.nx * d.p.g.ny;
        v.nx = d.p.g.nx;
        v.ny = d.p.g.ny;
        v.nz = d.p.g.nz;
        stats_tile_row(v, tile, spec, rows + ((long long)d.row_base + tile) * kNStats);
      }
      if (!grid_sync(ctl, run.spin_limit)) break;
      // ---- per-design combine and decision (src/simulation.py:128-156)
      for (int k = blockIdx.x; k < na; k += gridDim.x) {
        BatchDesign& d = D[__ldcg(ctl->active + k)];
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int col = warp; col < kNStats; col += nw) {
          const int op = spec.op[col];
          double a = identity(op);
          for (uint32_t r = lane; r < d.stat_tiles; r += 32)
            a = combine(op, a, __ldcg(rows + ((long long)d.row_base + r) * kNStats + col));
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) a = combine(op, a, __shfl_down_sync(0xffffffffu, a, o));
          if (lane == 0) st[col] = a;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          const double ke = st[XAC_ST_SUM_KE], max_T = st[XAC_ST_MAX_T], Q_out = st[XAC_ST_Q_OUT],
                       max_v = st[XAC_ST_MAX_V];
          const long long s1d = s1 - d.start;  // the design's own step count after this step
          const bool past = s1d > run.stats_every;
          // the previous check of this design may have run on another block: read through L2
          const double pke = __ldcg(&d.prev_ke), pT = __ldcg(&d.prev_max_T), pQ = __ldcg(&d.prev_Q);
          d.d_ke = past ? fabs(ke - pke) / (pke + 1e-9) / run.stats_every : 0.0;
          d.dT = past ? fabs(max_T - pT) / (pT + 1e-9) / run.stats_every : 0.0;
          d.dQ = past ? fabs(Q_out - pQ) / (fabs(pQ) + 1e-12) / run.stats_every : 1.0;
          d.prev_ke = ke;
          d.prev_max_T = max_T;
          d.prev_Q = Q_out;
          if (run.constant_power && s1d > 2000) {
            // src/simulation.py:139-146, the controller of xac_lattice_run on this design's stats
            double ue = (double)__ldcg(d.u_in);
            const double rin = st[XAC_ST_C_IN] > 0 ? st[XAC_ST_SUM_RHO_IN] / st[XAC_ST_C_IN] : 1.0;
            const double rout = st[XAC_ST_C_OUT] > 0 ? st[XAC_ST_SUM_RHO_OUT] / st[XAC_ST_C_OUT] : 1.0;
            const double dP = (rin - rout) / 3.0;
            const double pw = dP * (ue * st[XAC_ST_C_IN]);
            ue = ue + 0.005 * (run.target_power - pw);
            ue = ue < 0.0001 ? 0.0001 : (ue > 0.15 ? 0.15 : ue);
            __stcg(d.u_in, (float)ue);
          }
          for (int j = 0; j < kNStats; ++j) d.last[j] = st[j];
          d.steps = s1d;
          if (s1d > d.min_steps && d.d_ke < run.tol_ke && d.dT < run.tol_T && d.dQ < run.tol_T) {
            d.converged = 1;
            d.active = 0;
          } else if (st[XAC_ST_NONFINITE] > 0 || max_v > 0.17 || max_T > 1e4) {
            d.diverged = 1;
            d.active = 0;
          }
        }
        __syncthreads();
      }
      if (!grid_sync(ctl, run.spin_limit)) break;
      // ---- retire: rebuild the active lists
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        int m = 0;
        uint32_t acc = 0, sacc = 0;
        for (int k = 0; k < na; ++k) {
          const uint32_t i = __ldcg(ctl->active + k);
          if (__ldcg(&D[i].active)) {
            ctl->active[m] = i;
            ctl->prefix[m] = acc;
            ctl->stat_prefix[m] = sacc;
            acc += D[i].tiles;  // constant fields
            sacc += D[i].stat_tiles;
            ++m;
          }
        }
        ctl->prefix[m] = acc;
        ctl->stat_prefix[m] = sacc;
        ctl->n_active = m;
        if (m == 0) ctl->all_done = 1;
        __threadfence();
      }
      if (!grid_sync(ctl, run.spin_limit)) break;
    }
    step = s1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && *(volatile int*)&ctl->err == 0) ctl->step = step;
}

}  // namespace xac
