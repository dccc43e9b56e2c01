// Lattice object of libxac.so: owns the fused-step state of one design and implements the
// xac_lattice_* entry points (the path of src/simulation.py:14-162).
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <map>
#include <tuple>
#include <type_traits>
#include <mutex>
#include <utility>
#include <vector>

#include "batch.cuh"
#include "lattice_kernels.cuh"
#include "reductions.cuh"

namespace xac {

// ---------------------------------------------------------------- error plumbing
namespace {
thread_local char g_err[512] = "";
}
void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  return e == cudaErrorMemoryAllocation ? XAC_ENOMEM : XAC_ECUDA;
}

namespace {

constexpr int kBlock = 256;

// ---------------------------------------------------------------- layout / setup kernels
// reference index r = (x*ny + y)*nz + z  <->  internal index c = (z*ny + y)*nx + x
__device__ __forceinline__ long long ref_index(int x, int y, int z, int ny, int nz) {
  return ((long long)x * ny + y) * nz + z;
}

__global__ void build_link_kernel(const uint8_t* __restrict__ type, const float* __restrict__ qsrc,
                                  uint32_t* __restrict__ link, Geom g) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= g.ncell) return;
  const int x = (int)(c % g.nx);
  const long long t = c / g.nx;
  const int y = (int)(t % g.ny), z = (int)(t / g.ny);
  uint32_t w = 0;
#pragma unroll
  for (int i = 1; i < kQ; ++i) {
    const int sx = x - ex_of(i), sy = y - ey_of(i), sz = z - ez_of(i);
    bool bb = sx < 0 || sx >= g.nx || sy < 0 || sy >= g.ny || sz < 0 || sz >= g.nz;
    if (!bb) bb = type[((long long)sz * g.ny + sy) * g.nx + sx] == kSolid;
    if (bb) w |= 1u << i;
  }
  w |= (uint32_t)(type[c] & 3) << kTypeShift;
  if (qsrc[c] > 0.0f) w |= kHeatedBit;
  if (x == 0) w |= kXLoBit;
  if (x == g.nx - 1) w |= kXHiBit;
  if (y == 0) w |= kYLoBit;
  if (y == g.ny - 1) w |= kYHiBit;
  if (z == 0) w |= kZLoBit;
  if (z == g.nz - 1) w |= kZHiBit;
  if (w & (kYLoBit | kYHiBit | kZLoBit | kZHiBit)) w |= kYZBit;
  link[c] = w;
}

// ref-layout fields (any may be null = cold-start constant) -> internal rho, ux, uy, uz, T
__global__ void import_fields_kernel(const float* __restrict__ rho_r, const float* __restrict__ u_r,
                                     const float* __restrict__ T_r, const uint8_t* __restrict__ type, float T_cold,
                                     float* __restrict__ rho, float* __restrict__ ux, float* __restrict__ uy,
                                     float* __restrict__ uz, float* __restrict__ T, Geom g) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= g.ncell) return;
  const int x = (int)(c % g.nx);
  const long long t = c / g.nx;
  const int y = (int)(t % g.ny), z = (int)(t / g.ny);
  const long long r = ref_index(x, y, z, g.ny, g.nz);
  const bool solid = type[c] == kSolid;
  rho[c] = (rho_r && !solid) ? rho_r[r] : 1.0f;
  ux[c] = (u_r && !solid) ? u_r[3 * r] : 0.0f;
  uy[c] = (u_r && !solid) ? u_r[3 * r + 1] : 0.0f;
  uz[c] = (u_r && !solid) ? u_r[3 * r + 2] : 0.0f;
  T[c] = T_r ? T_r[r] : T_cold;
}

// simulation.py:89-90 (equilibria) followed by the fluid collision of the reference's first replay
// (simulation.py:94), which this scheme performs ahead of the first streaming step.
template <typename SP, typename SQ>
__global__ void init_state_kernel(const float* __restrict__ rho, const float* __restrict__ ux,
                                  const float* __restrict__ uy, const float* __restrict__ uz,
                                  const float* __restrict__ T, const uint8_t* __restrict__ type, SP* __restrict__ P0,
                                  SP* __restrict__ P1, SQ* __restrict__ Q0, StepParams p) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= p.g.ncell) return;
  const int RL = p.g.pitch;
  const uint32_t row = (uint32_t)(c / p.g.nx), x = (uint32_t)(c - (long long)row * p.g.nx);
  const long long e0 = pop_base(row, x, p.g, RL);
  const float r = rho[c], vx = ux[c], vy = uy[c], vz = uz[c];
  const bool solid = type[c] == kSolid;
  const float usq15 = 1.5f * ((vx * vx + vy * vy) + vz * vz);
  const float omega = 1.0f / p.tau_f;
  const float Tc = T[c];
  const float tx = solid ? 0.0f : vx, ty = solid ? 0.0f : vy, tz = solid ? 0.0f : vz;
  const float usq15t = 1.5f * ((tx * tx + ty * ty) + tz * tz);
  // fluid populations of non-solid cells only (a solid cell's are w_i: rho = 1 and u = 0 there)
  uint32_t k = 0;
  if (!solid) {
    const uint2 e = p.ftab[ftab_index(p.g, row, x)];
    k = e.y + (uint32_t)__popc(e.x & ((1u << (x & 31u)) - 1u));
  }
#define XAC_INIT(I)                                                                   \
  {                                                                                   \
    if (!solid) {                                                                     \
      const float fe = feq_term(w_of(I) * r, edotu<I>(vx, vy, vz), usq15);           \
      const float pc = fe - omega * (fe - fe);                                        \
      Pop<SP>::st(P0 + k + (long long)I * p.g.ns, pc, w_of(I));                      \
      Pop<SP>::st(P1 + k + (long long)I * p.g.ns, pc, w_of(I));                      \
    }                                                                                 \
    const float ge = feq_term(w_of(I) * Tc, edotu<I>(tx, ty, tz), usq15t);           \
    Pop<SQ>::st(Q0 + e0 + (long long)I * RL, ge, w_of(I) * p.T_ref);                 \
  }
  XAC_FOR19(XAC_INIT)
#undef XAC_INIT
}

// internal -> reference layout export
__global__ void export_fields_kernel(const float* __restrict__ rho, const float* __restrict__ ux,
                                     const float* __restrict__ uy, const float* __restrict__ uz,
                                     const float* __restrict__ T, float* __restrict__ rho_r, float* __restrict__ u_r,
                                     float* __restrict__ T_r, Geom g) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= g.ncell) return;
  const int z = (int)(r % g.nz);
  const long long t = r / g.nz;
  const int y = (int)(t % g.ny), x = (int)(t / g.ny);
  const long long c = ((long long)z * g.ny + y) * g.nx + x;
  if (rho_r) rho_r[r] = rho[c];
  if (u_r) {
    u_r[3 * r] = ux[c];
    u_r[3 * r + 1] = uy[c];
    u_r[3 * r + 2] = uz[c];
  }
  if (T_r) T_r[r] = T[c];
}

__global__ void set_scalar_kernel(float* dst, float v) { *dst = v; }

// Memory-pattern probe of the fused step (SP / SQ: unsigned words of the fluid / thermal storage size): the
// threads, the link-word and table reads, the population addresses (fluid pulls of the non-solid cells with the
// bounce-back reads their link bits select, thermal pulls from the neighbours) and the whole-sector fills of the
// thermal padding lanes that coupled_step_kernel has, with no arithmetic: every value read is stored unchanged at
// the cell's own position of the other buffer. Its time is the floor the step's memory access pattern sets. (At the domain faces the thermal
// rules read the cell's own row instead of a neighbour: the probe pulls there too, which reads padding or guard
// values.)
template <typename SP, typename SQ, int kT>
__global__ void __launch_bounds__(256) pattern_copy_kernel(const SP* __restrict__ Pin, SP* __restrict__ Pout,
                                                           const SQ* __restrict__ Qin, SQ* __restrict__ Qout,
                                                           const uint32_t* __restrict__ link,
                                                           const uint2* __restrict__ ftab, Geom g, uint32_t reverse) {
  const int RL = row_len<kT>(g);
  const uint32_t blk = reverse ? gridDim.x - 1u - blockIdx.x : blockIdx.x;
  const uint32_t pos = blk * blockDim.x + threadIdx.x;
  const uint32_t r = pos / (uint32_t)RL, x = pos - r * (uint32_t)RL;
  if (r >= (uint32_t)g.rows) return;  // whole warps (the row length is a multiple of 32)
  const int lane = threadIdx.x & 31;
  const bool valid = x < (uint32_t)g.nx;
  const uint32_t c = r * (uint32_t)g.nx + x;
  const uint32_t lw = valid ? __ldg(link + c) : ((uint32_t)kSolid << kTypeShift);
  const bool fluid = valid && link_type(lw) != kSolid;
  const bool fill_q = (__ballot_sync(0xffffffffu, valid) & sector_group<SQ>(lane)) != 0u;
  const uint32_t e0 = pop_base(r, x, g, RL);
  if (fluid) {
    const FluidAt<SP> P = fluid_at(Pin, r, x, g, ftab);
#define XAC_PC_P(I) Pout[P.k + (I) * P.ns] = ((lw >> (I)) & 1u) ? __ldg(P.own(opp_of(I))) : __ldg(P.template pull<I>());
    XAC_FOR19(XAC_PC_P)
#undef XAC_PC_P
  }
  if (valid) {
    const Rows<SQ, kT> Q = rows_at<kT>(Qin, e0, g, RL);
#define XAC_PC_Q(I) Qout[e0 + (I) * RL] = __ldg(Q.template pull<I>());
    XAC_FOR19(XAC_PC_Q)
#undef XAC_PC_Q
  } else if (fill_q) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) Qout[e0 + i * RL] = SQ{};
  }
}

// The probe moves bits only: each storage type is copied as the unsigned word of its size.
template <size_t kBytes>
using RawWord = typename std::conditional<kBytes == 4, unsigned int, unsigned short>::type;

template <typename SP0, typename SQ0>
void launch_pattern_copy(const void* Pin, void* Pout, const void* Qin, void* Qout, const uint32_t* link,
                         const uint2* ftab, const Geom& g, int block, uint32_t reverse, cudaStream_t s) {
  using SP = RawWord<sizeof(SP0)>;
  using SQ = RawWord<sizeof(SQ0)>;
  const unsigned grid = (unsigned)(((long long)g.rows * g.pitch + block - 1) / block);
#define XAC_PC(KT)                                                                                                 \
  pattern_copy_kernel<SP, SQ, KT><<<grid, block, 0, s>>>((const SP*)Pin, (SP*)Pout, (const SQ*)Qin, (SQ*)Qout, \
                                                          link, ftab, g, reverse)
  switch (g.pitch) {
    case 32: XAC_PC(32); break;
    case 64: XAC_PC(64); break;
    case 96: XAC_PC(96); break;
    case 128: XAC_PC(128); break;
    case 160: XAC_PC(160); break;
    case 192: XAC_PC(192); break;
    case 224: XAC_PC(224); break;
    case 256: XAC_PC(256); break;
    default: XAC_PC(0);
  }
#undef XAC_PC
}

template <typename T>
int dmalloc(T** p, size_t count, const char* what) {
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T) + 16);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_status(e, what);
  }
  return XAC_OK;
}

int reduction_blocks(long long n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long want = (n + kBlock * 8 - 1) / (kBlock * 8);
  long long cap = (long long)sms * 4;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (int)want;
}

}  // namespace

// ---------------------------------------------------------------- device-resident run loop
// State of xac_lattice_run's convergence loop while a CUDA graph runs it: one while-node iteration is
// stats_every steps, T, the stats, and run_decision_kernel, which repeats the host loop's arithmetic
// (simulation.py:121-156) in double and sets the graph's loop condition.
struct RunCtl {
  long long start;      // lattice step count when the run began
  long long step;       // steps of this run done
  long long min_steps;  // no convergence before this many steps of the run
  long long max_iters;  // stats intervals this launch may run
  long long iters;
  int stats_every, constant_power, stop, diverged;
  double tol_ke, tol_T, target_power;
  double prev_ke, prev_max_T, prev_Q, d_ke, dT, dQ;
  float u_in;
  int pad;
  double last[kNStats];
};

static __global__ void run_decision_kernel(const double* __restrict__ st, RunCtl* c, float* u_in_dev,
                                           cudaGraphConditionalHandle h) {
  c->step += c->stats_every;
  c->iters += 1;
  const double max_v = st[XAC_ST_MAX_V], ke = st[XAC_ST_SUM_KE], max_T = st[XAC_ST_MAX_T], Q_out = st[XAC_ST_Q_OUT];
  const long long at = c->start + c->step;
  const bool past = at > c->stats_every;
  c->d_ke = past ? fabs(ke - c->prev_ke) / (c->prev_ke + 1e-9) / c->stats_every : 0.0;
  c->dT = past ? fabs(max_T - c->prev_max_T) / (c->prev_max_T + 1e-9) / c->stats_every : 0.0;
  c->dQ = past ? fabs(Q_out - c->prev_Q) / (fabs(c->prev_Q) + 1e-12) / c->stats_every : 1.0;
  c->prev_ke = ke;
  c->prev_max_T = max_T;
  c->prev_Q = Q_out;
  if (c->constant_power && at > 2000) {
    double ue = (double)c->u_in;
    const double rin = st[XAC_ST_C_IN] > 0 ? st[XAC_ST_SUM_RHO_IN] / st[XAC_ST_C_IN] : 1.0;
    const double rout = st[XAC_ST_C_OUT] > 0 ? st[XAC_ST_SUM_RHO_OUT] / st[XAC_ST_C_OUT] : 1.0;
    const double dP = (rin - rout) / 3.0;
    const double pw = dP * (ue * st[XAC_ST_C_IN]);
    ue = ue + 0.005 * (c->target_power - pw);
    ue = ue < 0.0001 ? 0.0001 : (ue > 0.15 ? 0.15 : ue);
    c->u_in = (float)ue;
    *u_in_dev = (float)ue;
  }
  for (int k = 0; k < kNStats; ++k) c->last[k] = st[k];
  bool stop = false;
  if (c->step > c->min_steps && c->d_ke < c->tol_ke && c->dT < c->tol_T && c->dQ < c->tol_T) {
    stop = true;
  } else if (st[XAC_ST_NONFINITE] > 0 || max_v > 0.17 || max_T > 1e4) {
    c->diverged = 1;
    stop = true;
  }
  if (c->iters >= c->max_iters) stop = true;
  c->stop = stop ? 1 : 0;
  cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// ---------------------------------------------------------------- the lattice object
struct LatticeImpl {
  Geom g{};
  int precision = XAC_FP32;
  size_t p_elem = 4, q_elem = 4;  // bytes per fluid / thermal population
  double tau_fluid = 0.6, Pr = 7.0, k_ratio = 628.0, u_inlet_nominal = 0.03, rho_outlet = 1.0, t_inlet = 25.0,
         heat_power = 0.1;
  float tau_th_f = 0.5f, tau_th_s = 0.5f;
  float relax[5] = {1.0f, 1.0f, 1.0f, 0.5f, 0.5f};  // omega_f, omega_tf, omega_ts, srcf_f, srcf_s (device-computed)
  float u_in_host = 0.0f;
  int tune_block = 128;  // threads per block of the step kernel
  int tune_variant = 0;  // 0: one thread per row position; 1: thermal rows staged in shared memory
  unsigned* status = nullptr;  // device word set by a step kernel whose bounded wait ran out
  // set once the status word was seen non-zero: a staged step gave up on its copies, so the thermal populations it
  // wrote are not the step's; the lattice refuses work until init_fields / load_state rewrites its populations
  bool failed = false;
  int refuse(const char* fn) const {
    set_error("%s: this lattice stopped being usable when a staged step kernel gave up waiting for its copies; "
              "re-initialise it (init_fields) or load a saved state", fn);
    return XAC_ETIMEOUT;
  }

  void* P[2] = {nullptr, nullptr};
  void* Qb[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t* type = nullptr;
  uint32_t* link = nullptr;
  uint2* ftab = nullptr;  // non-solid cell table of the fluid populations
  uint32_t nonsolid = 0;  // non-solid cells (the fluid populations' slots in use)
  float* qsrc = nullptr;
  float* u_in = nullptr;
  float *rho = nullptr, *ux = nullptr, *uy = nullptr, *uz = nullptr, *T = nullptr;
  double* rows = nullptr;  // reduction partials
  double* red_out = nullptr;
  double* host_out = nullptr;  // pinned
  int red_blocks = 1;
  long long step = 0;
  bool own_pending = true;    // next step reads the initial thermal populations unstreamed

  // src/simulation.py:102-104: no convergence before min(0.6 max_steps, max(5000, 2 nx / u_in)) steps
  long long reference_min_steps(int max_steps) const {
    const int a = (int)(0.6 * max_steps);
    const double mu = u_inlet_nominal > 1e-6 ? u_inlet_nominal : 1e-6;
    int b = (int)(2.0 * g.nx / mu);
    if (b < 5000) b = 5000;
    return a < b ? a : b;
  }
  long long macro_step = 0;   // rho/u arrays hold the fields of this step
  long long T_step = 0;       // T array holds the field of this step
  cudaStream_t capture = nullptr;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // (n, parity) -> n steps with macro output at the end
  std::map<std::pair<int, int>, cudaGraphExec_t> run_graphs;  // (stats_every, parity) -> device-resident run loop
  RunCtl* run_ctl = nullptr;       // device
  RunCtl* run_ctl_host = nullptr;  // pinned
  std::mutex mu;

  StepParams params() const {
    StepParams p;
    p.g = g;
    p.tau_f = (float)tau_fluid;
    p.tau_tf = tau_th_f;
    p.tau_ts = tau_th_s;
    p.T_in = (float)t_inlet;
    p.rho_out = (float)rho_outlet;
    p.T_ref = precision == XAC_FP32 ? 0.0f : (float)t_inlet;
    p.omega_f = relax[0];
    p.omega_tf = relax[1];
    p.omega_ts = relax[2];
    p.srcf_f = relax[3];
    p.srcf_s = relax[4];
    p.status = status;
    p.ftab = ftab;
    p.reverse = (uint32_t)cur;  // sweep direction alternates with the buffer parity
    return p;
  }

  ~LatticeImpl() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto& kv : run_graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(run_ctl);
    if (run_ctl_host) cudaFreeHost(run_ctl_host);
    for (void* b : {P[0], P[1], Qb[0], Qb[1]}) cudaFree(b);
    cudaFree(type);
    cudaFree(link);
    cudaFree(ftab);
    cudaFree(qsrc);
    cudaFree(status);
    cudaFree(u_in);
    cudaFree(rho);
    cudaFree(ux);
    cudaFree(uy);
    cudaFree(uz);
    cudaFree(T);
    cudaFree(rows);
    cudaFree(red_out);
    if (host_out) cudaFreeHost(host_out);
    if (capture) cudaStreamDestroy(capture);
  }

  template <int kPrec>
  int launch_step(cudaStream_t s, bool macro, bool own) {
    const StepParams p = params();
    StepLaunch a{P[cur], P[cur ^ 1], Qb[cur], Qb[cur ^ 1], link, qsrc, u_in, rho, ux, uy, uz, T, p, tune_block,
                 tune_variant, macro, own, s};
    launch_coupled_step<typename Storage<kPrec>::P, typename Storage<kPrec>::Q>(a);
    cur ^= 1;
    return XAC_OK;
  }

  int launch_step_any(cudaStream_t s, bool macro, bool own) {
    switch (precision) {
      case XAC_FP16: return launch_step<XAC_FP16>(s, macro, own);
      case XAC_BF16: return launch_step<XAC_BF16>(s, macro, own);
      case XAC_FP32_T16: return launch_step<XAC_FP32_T16>(s, macro, own);
      default: return launch_step<XAC_FP32>(s, macro, own);
    }
  }

  // T of the current state into the T field (the thermal populations' storage type follows the precision mode)
  void launch_finalize_T(cudaStream_t s) {
    const StepParams p = params();
    const unsigned grid = grid_for(g.ncell, kBlock);
    if (precision == XAC_FP32)
      thermal_finalize_kernel<float><<<grid, kBlock, 0, s>>>((const float*)Qb[cur], link, T, p);
    else
      thermal_finalize_kernel<__half><<<grid, kBlock, 0, s>>>((const __half*)Qb[cur], link, T, p);
  }

  // n plain steps (no own step), the last one writing rho/u
  int launch_plain(cudaStream_t s, int n) {
    for (int k = 0; k < n; ++k) {
      int r = launch_step_any(s, k == n - 1, false);
      if (r != XAC_OK) return r;
    }
    return XAC_OK;
  }

  // n >= 8 plain steps from the cached graph of n steps for the current buffer parity (captured on first use)
  int launch_graph(cudaStream_t s, int n) {
    auto key = std::make_pair(n, cur);
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      if (!capture) XAC_CUDA(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking));
      const int saved = cur;
      cudaGraph_t graph = nullptr;
      XAC_CUDA(cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal));
      launch_plain(capture, n);
      cudaError_t e = cudaStreamEndCapture(capture, &graph);
      cur = saved;
      if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
      cudaGraphExec_t exec = nullptr;
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
      it = graphs.emplace(key, exec).first;
    }
    XAC_CUDA(cudaGraphLaunch(it->second, s));
    if (n & 1) cur ^= 1;
    return XAC_OK;
  }

  // Long runs go as graphs of at most kGraphSteps steps (an even count, so the same graph serves every chunk);
  // each chunk's last step also writes rho/u, which changes no population.
  static constexpr int kGraphSteps = 512;
  int steps(int n, cudaStream_t s) {
    if (n <= 0) return XAC_OK;
    if (own_pending) {
      launch_step_any(s, n == 1, true);
      own_pending = false;
      step += 1;
      --n;
      XAC_CUDA(cudaGetLastError());
    }
    if (n > 0) {
      const int total = n;
      for (; n > kGraphSteps; n -= kGraphSteps) {
        int r = launch_graph(s, kGraphSteps);
        if (r != XAC_OK) return r;
      }
      if (n >= 8) {
        int r = launch_graph(s, n);
        if (r != XAC_OK) return r;
      } else {
        launch_plain(s, n);
      }
      step += total;
      XAC_CUDA(cudaGetLastError());
    }
    macro_step = step;
    return XAC_OK;
  }

  // The device-resident run loop for the current buffer parity: a graph whose while node repeats
  // { every plain steps, T, stats, run_decision_kernel } until the decision kernel clears the condition.
  // every must be even (the parity is the same at each iteration).
  int run_graph(int every, cudaGraphExec_t* out) {
    auto key = std::make_pair(every, cur);
    auto it = run_graphs.find(key);
    if (it != run_graphs.end()) {
      *out = it->second;
      return XAC_OK;
    }
    if (!capture) XAC_CUDA(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking));
    if (!run_ctl) XAC_CUDA(cudaMalloc(&run_ctl, sizeof(RunCtl)));
    if (!run_ctl_host) XAC_CUDA(cudaMallocHost(&run_ctl_host, sizeof(RunCtl)));
    cudaGraph_t graph = nullptr;
    XAC_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &np);
    const int saved = cur;
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(capture, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaGraphDestroy(graph);
      return cuda_status(e, "run loop graph");
    }
    launch_plain(capture, every);
    launch_finalize_T(capture);
    const auto spec = stats_spec();
    const int ntiles = (int)stats_tiles(g.ncell);
    stats_partials_kernel<<<ntiles, kStatsBlock, 0, capture>>>(view(), spec, rows);
    combine_rows_kernel<kNStats><<<1, 32 * kNStats, 0, capture>>>(rows, ntiles, spec, red_out);
    run_decision_kernel<<<1, 1, 0, capture>>>(red_out, run_ctl, u_in, h);
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(capture, &body);
    cur = saved;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_status(e, "run loop graph");
    run_graphs.emplace(key, exec);
    *out = exec;
    return XAC_OK;
  }

  int finalize_T(cudaStream_t s) {
    if (T_step == step) return XAC_OK;
    launch_finalize_T(s);
    XAC_CUDA(cudaGetLastError());
    T_step = step;
    return XAC_OK;
  }

  FieldView view() const {
    FieldView v{};
    v.rho = rho;
    v.ux = ux;
    v.uy = uy;
    v.uz = uz;
    v.ustride = 1;
    v.T = T;
    v.mask = nullptr;
    v.link = link;
    v.sx = 1;
    v.sy = g.nx;
    v.sz = (long long)g.nx * g.ny;
    v.nx = g.nx;
    v.ny = g.ny;
    v.nz = g.nz;
    return v;
  }
};

// ---------------------------------------------------------------- shared reduction drivers
// rows must hold stats_tiles(cells) * kNStats doubles
int run_stats(const FieldView& v, double* rows, double* dev_out, double* host_out, cudaStream_t s) {
  const auto spec = stats_spec();
  const int ntiles = (int)stats_tiles((long long)v.nx * v.ny * v.nz);
  stats_partials_kernel<<<ntiles, kStatsBlock, 0, s>>>(v, spec, rows);
  combine_rows_kernel<kNStats><<<1, 32 * kNStats, 0, s>>>(rows, ntiles, spec, dev_out);
  XAC_CUDA(cudaGetLastError());
  XAC_CUDA(cudaMemcpyAsync(host_out, dev_out, kNStats * sizeof(double), cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

int run_metrics(const FieldView& v, MetricBox b, double* rows, int nblocks, double* dev_out, double* host_raw,
                cudaStream_t s) {
  const auto spec = metric_spec();
  metric_partials_kernel<<<nblocks, kBlock, 0, s>>>(v, b, spec, rows);
  combine_rows_kernel<kNMetrics><<<1, 32 * kNMetrics, 0, s>>>(rows, nblocks, spec, dev_out);
  XAC_CUDA(cudaGetLastError());
  XAC_CUDA(cudaMemcpyAsync(host_raw, dev_out, kNMetrics * sizeof(double), cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

// generate_dataset.py:57-179 assembled from the FP64 partial sums.
void assemble_scalars(const double* m, int nx, int ny, int nz, int buf, double t_inlet, double tau_fluid, double Pr,
                      double u_inlet, double* out) {
  for (int k = 0; k < XAC_NSCALARS; ++k) out[k] = 0.0;
  const double Q_vol = m[kM_QVOL];
  const double rho_in = m[kM_N_IN] > 0 ? m[kM_RHO_IN] / m[kM_N_IN] : 1.0;
  const double rho_out = m[kM_N_OUT] > 0 ? m[kM_RHO_OUT] / m[kM_N_OUT] : 1.0;
  const double dP = (rho_in - rho_out) / 3.0;
  const double P_pump = std::fabs(dP * Q_vol);
  const double ts_n = m[kM_TS_N] > 0 ? m[kM_TS_N] : 1.0;
  const double Tmax_s = m[kM_TS_MAX], Tmin_s = m[kM_TS_MIN];
  const double Tavg_s = m[kM_TS_SUM] / ts_n;
  const double var = m[kM_TS_SQ] / ts_n - Tavg_s * Tavg_s;
  const double sigma = std::sqrt(var > 0 ? var : 0.0);
  const double total_flux = Q_vol;
  const double Tout_avg = std::fabs(total_flux) > 1e-12 ? m[kM_QOUT] / total_flux : t_inlet;
  const double Q_out_flux = m[kM_QOUT], Q_in_flux = t_inlet * total_flux;
  const double dq = Q_out_flux - Q_in_flux;
  const double Q_abs = std::fabs(dq) > 1e-12 ? std::fabs(dq) : 1e-12;
  const double R_th = (Tmax_s - t_inlet) / Q_abs;
  const double Tf_avg = m[kM_TF_N] > 0 ? m[kM_TF_SUM] / m[kM_TF_N] : t_inlet;
  const double dT_conv = Tavg_s - Tf_avg;
  const double V_fluid = m[kM_VFLUID], A_wet = m[kM_FACES];
  const double Dh = A_wet > 0 ? 4.0 * V_fluid / A_wet : (double)ny;
  const double h_avg = (std::fabs(dT_conv) > 1e-6 && A_wet > 0) ? Q_abs / (A_wet * std::fabs(dT_conv)) : 0.0;
  const double tau_th_f = 0.5 + (tau_fluid - 0.5) / Pr;
  const double k_f = (1.0 / 3.0) * (tau_th_f - 0.5);
  const double Nu = k_f > 1e-12 ? h_avg * Dh / k_f : 0.0;
  const double L = nx - 2 * buf;
  const double rho_avg = (rho_in + rho_out) / 2.0;
  const double f = u_inlet > 1e-12 ? (std::fabs(dP) * Dh) / (2.0 * L * rho_avg * u_inlet * u_inlet) : 0.0;
  const double COP = P_pump > 1e-12 ? Q_abs / P_pump : 0.0;
  out[XAC_SC_DP] = dP;
  out[XAC_SC_RTH] = R_th;
  out[XAC_SC_NU] = Nu;
  out[XAC_SC_F_FRICTION] = f;
  out[XAC_SC_P_PUMP] = P_pump;
  out[XAC_SC_COP] = COP;
  out[XAC_SC_Q_VOL] = Q_vol;
  out[XAC_SC_T_MAX_SURFACE] = Tmax_s;
  out[XAC_SC_T_AVG_SURFACE] = Tavg_s;
  out[XAC_SC_DELTA_T_MAX] = Tmax_s - Tmin_s;
  out[XAC_SC_SIGMA_T] = sigma;
  out[XAC_SC_FLUID_TEMP_RISE] = Tout_avg - t_inlet;
  const double plane = (double)ny * nz;
  out[XAC_SC_PRESSURE_DROP_ALL] = (m[kM_RHO1_ALL] / plane - m[kM_RHO2_ALL] / plane) / 3.0;
  out[XAC_SC_MAX_VELOCITY] = m[kM_MAXV];
  out[XAC_SC_MAX_TEMPERATURE] = m[kM_MAXT];
  out[XAC_SC_MEAN_TEMPERATURE] = m[kM_TSUM_ALL] / ((double)nx * ny * nz);
  out[XAC_SC_DH] = Dh;
  out[XAC_SC_V_FLUID] = V_fluid;
  out[XAC_SC_A_WETTED] = A_wet;
  const double core_size = (double)(nx - 2 * buf) * ny * nz;
  out[XAC_SC_POROSITY] = core_size > 0 ? 1.0 - m[kM_CORE_SOLID] / core_size : 0.0;
  out[XAC_SC_Q_ABSORBED] = Q_abs;
  out[XAC_SC_DT_CONV] = dT_conv;
  out[XAC_SC_RHO_AVG] = rho_avg;
}

}  // namespace xac

struct xac_lattice {
  xac::LatticeImpl impl;
};

using namespace xac;

namespace {

// Normalised heat source times power, internal layout; simulation.py:77-86 and thermal_engine3d.py:116-117.
// Table of the fluid populations' non-solid cells (FluidAt): per 32-cell word of each row its non-solid mask and
// the number of non-solid cells before it, with ny + 1 empty rows before and after the grid. Sets g.nt, g.ns and
// g.np. type is in cell order c = (z*ny + y)*nx + x.
std::vector<uint2> fluid_table(const uint8_t* type, Geom& g, uint32_t* nonsolid) {
  g.nt = g.pitch / 32;
  const long long guard_rows = g.ny + 1;
  std::vector<uint2> tab((size_t)((g.rows + 2 * guard_rows) * g.nt), make_uint2(0u, 0u));
  uint32_t k = 0;
  for (long long r = 0; r < g.rows; ++r)
    for (int w = 0; w < g.nt; ++w) {
      uint32_t m = 0;
      for (int b = 0; b < 32; ++b) {
        const int x = 32 * w + b;
        if (x < g.nx && type[r * g.nx + x] != kSolid) m |= 1u << b;
      }
      tab[(size_t)((r + guard_rows) * g.nt + w)] = make_uint2(m, k);
      k += (uint32_t)__builtin_popcount(m);
    }
  // rows after the grid: empty words whose count is the total
  for (size_t t = (size_t)((g.rows + guard_rows) * g.nt); t < tab.size(); ++t) tab[t].y = k;
  *nonsolid = k;
  g.ns = ((long long)k + 31) / 32 * 32;
  if (g.ns == 0) g.ns = 32;
  g.np = (long long)kQ * g.ns;
  return tab;
}

std::vector<float> host_qsrc(const xac_desc* d) {
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  const size_t n = (size_t)nx * ny * nz;
  std::vector<float> hs(n, 0.0f);
  if (d->heat_source) {
    std::memcpy(hs.data(), d->heat_source, n * sizeof(float));
  } else {
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y) hs[((size_t)x * ny + y) * nz + 0] = 1.0f;
  }
  float mx = -INFINITY;
  bool nan = false;
  for (size_t i = 0; i < n; ++i) {
    if (std::isnan(hs[i])) nan = true;
    if (hs[i] > mx) mx = hs[i];
  }
  if (!nan && mx > 0.0f)
    for (size_t i = 0; i < n; ++i) hs[i] = hs[i] / mx;
  const float power = (float)d->heat_power;
  std::vector<float> q(n);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z)
        q[((size_t)z * ny + y) * nx + x] = hs[((size_t)x * ny + y) * nz + z] * power;
  return q;
}

int create_impl(const xac_desc* d, LatticeImpl& L, cudaStream_t s) {
  XAC_REQUIRE(d, "xac_lattice_create: null descriptor");
  XAC_REQUIRE(d->nx >= 3 && d->ny >= 1 && d->nz >= 1, "xac_lattice_create: lattice %d x %d x %d too small", d->nx,
              d->ny, d->nz);
  XAC_REQUIRE(((long long)d->ny * d->nz + 2LL * (d->ny + 2)) * kQ * ((d->nx + 31) / 32 * 32) < (1LL << 31),
              "xac_lattice_create: lattice too large (19 x padded cells must stay below 2^31)");
  XAC_REQUIRE(d->mask, "xac_lattice_create: null mask");
  XAC_REQUIRE(d->tau_fluid > 0.5, "xac_lattice_create: tau_fluid must exceed 0.5 (got %g)", d->tau_fluid);
  XAC_REQUIRE(d->Pr > 0, "xac_lattice_create: Pr must be positive");
  XAC_REQUIRE(d->precision == XAC_FP32 || d->precision == XAC_FP16 || d->precision == XAC_BF16 ||
                  d->precision == XAC_FP32_T16,
              "xac_lattice_create: unknown precision %d", d->precision);
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  const long long n = (long long)nx * ny * nz;
  L.g.nx = nx;
  L.g.ny = ny;
  L.g.nz = nz;
  L.g.ncell = n;
  L.g.pitch = (nx + 31) / 32 * 32;
  L.g.rows = ny * nz;
  L.g.guard = (long long)(ny + 2) * kQ * L.g.pitch;
  L.g.N = (long long)L.g.rows * kQ * L.g.pitch + 2 * L.g.guard;
  L.precision = d->precision;
  L.p_elem = (d->precision == XAC_FP32 || d->precision == XAC_FP32_T16) ? 4 : 2;
  L.q_elem = d->precision == XAC_FP32 ? 4 : 2;
  L.tau_fluid = d->tau_fluid;
  L.Pr = d->Pr;
  L.k_ratio = d->k_ratio;
  L.u_inlet_nominal = d->u_inlet;
  L.rho_outlet = d->rho_outlet;
  L.t_inlet = d->t_inlet;
  L.heat_power = d->heat_power;
  // simulation.py:70-71 in double, handed to the kernels as float32 like Warp's float parameters
  const double tth_f = 0.5 + ((d->tau_fluid - 0.5) / d->Pr);
  const double tth_s = 0.5 + d->k_ratio * (tth_f - 0.5);
  L.tau_th_f = (float)tth_f;
  L.tau_th_s = (float)tth_s;
  L.u_in_host = (float)d->u_inlet;

  std::vector<uint8_t> type(n);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        const int32_t m = d->mask[((size_t)x * ny + y) * nz + z];
        XAC_REQUIRE(m >= 0 && m <= 3, "xac_lattice_create: mask value %d at (%d,%d,%d) is not a BC label", (int)m, x, y,
                    z);
        type[((size_t)z * ny + y) * nx + x] = (uint8_t)m;
      }
  std::vector<float> q = host_qsrc(d);
  const std::vector<uint2> ftab = fluid_table(type.data(), L.g, &L.nonsolid);
  const size_t p_bytes = (size_t)L.g.np * L.p_elem, q_bytes = (size_t)L.g.N * L.q_elem;
  for (int b = 0; b < 2; ++b) {
    XAC_CUDA(cudaMalloc(&L.P[b], p_bytes));
    XAC_CUDA(cudaMalloc(&L.Qb[b], q_bytes));
  }
  int r;
  if ((r = dmalloc(&L.type, n, "alloc type")) != XAC_OK) return r;
  if ((r = dmalloc(&L.link, n, "alloc link")) != XAC_OK) return r;
  if ((r = dmalloc(&L.ftab, ftab.size(), "alloc fluid table")) != XAC_OK) return r;
  if ((r = dmalloc(&L.qsrc, n, "alloc qsrc")) != XAC_OK) return r;
  if ((r = dmalloc(&L.u_in, 1, "alloc u_in")) != XAC_OK) return r;
  if ((r = dmalloc(&L.status, 1, "alloc status")) != XAC_OK) return r;
  XAC_CUDA(cudaMemsetAsync(L.status, 0, sizeof(unsigned), s));
  for (float** f : {&L.rho, &L.ux, &L.uy, &L.uz, &L.T})
    if ((r = dmalloc(f, n, "alloc fields")) != XAC_OK) return r;
  L.red_blocks = reduction_blocks(n);
  {
    const size_t metric_rows = (size_t)L.red_blocks * kNMetrics, stat_rows = (size_t)stats_tiles(n) * kNStats;
    if ((r = dmalloc(&L.rows, metric_rows > stat_rows ? metric_rows : stat_rows, "alloc rows")) != XAC_OK) return r;
  }
  if ((r = dmalloc(&L.red_out, 64, "alloc red_out")) != XAC_OK) return r;
  XAC_CUDA(cudaMallocHost(&L.host_out, 64 * sizeof(double)));
  // guards, row padding and the unused fluid slots are never used as values; keep them defined
  for (int b = 0; b < 2; ++b) {
    XAC_CUDA(cudaMemsetAsync(L.P[b], 0, p_bytes, s));
    XAC_CUDA(cudaMemsetAsync(L.Qb[b], 0, q_bytes, s));
  }
  XAC_CUDA(cudaMemcpyAsync(L.type, type.data(), n, cudaMemcpyHostToDevice, s));
  XAC_CUDA(cudaMemcpyAsync(L.ftab, ftab.data(), ftab.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
  XAC_CUDA(cudaMemcpyAsync(L.qsrc, q.data(), n * sizeof(float), cudaMemcpyHostToDevice, s));
  set_scalar_kernel<<<1, 1, 0, s>>>(L.u_in, L.u_in_host);
  relaxation_factors_kernel<<<1, 1, 0, s>>>((float)L.tau_fluid, L.tau_th_f, L.tau_th_s, (float*)L.red_out);
  XAC_CUDA(cudaMemcpyAsync(L.relax, L.red_out, sizeof(L.relax), cudaMemcpyDeviceToHost, s));
  build_link_kernel<<<grid_for(n, kBlock), kBlock, 0, s>>>(L.type, L.qsrc, L.link, L.g);
  XAC_CUDA(cudaGetLastError());
  // host vectors go out of scope: make the copies complete first
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

int init_impl(LatticeImpl& L, const float* rho, const float* u, const float* T, cudaStream_t s) {
  const unsigned grid = grid_for(L.g.ncell, kBlock);
  import_fields_kernel<<<grid, kBlock, 0, s>>>(rho, u, T, L.type, (float)L.t_inlet, L.rho, L.ux, L.uy, L.uz, L.T,
                                               L.g);
  const StepParams p = L.params();
  switch (L.precision) {
    case XAC_FP16:
      init_state_kernel<__half, __half><<<grid, kBlock, 0, s>>>(L.rho, L.ux, L.uy, L.uz, L.T, L.type,
                                                                      (__half*)L.P[0], (__half*)L.P[1],
                                                                      (__half*)L.Qb[0], p);
      break;
    case XAC_BF16:
      init_state_kernel<__nv_bfloat16, __half><<<grid, kBlock, 0, s>>>(L.rho, L.ux, L.uy, L.uz, L.T, L.type,
                                                                             (__nv_bfloat16*)L.P[0],
                                                                             (__nv_bfloat16*)L.P[1],
                                                                             (__half*)L.Qb[0], p);
      break;
    case XAC_FP32_T16:
      init_state_kernel<float, __half><<<grid, kBlock, 0, s>>>(L.rho, L.ux, L.uy, L.uz, L.T, L.type,
                                                                     (float*)L.P[0], (float*)L.P[1],
                                                                     (__half*)L.Qb[0], p);
      break;
    default:
      init_state_kernel<float, float><<<grid, kBlock, 0, s>>>(L.rho, L.ux, L.uy, L.uz, L.T, L.type, (float*)L.P[0],
                                                               (float*)L.P[1], (float*)L.Qb[0], p);
  }
  XAC_CUDA(cudaGetLastError());
  L.cur = 0;
  L.step = 0;
  L.own_pending = true;
  L.macro_step = 0;
  L.T_step = 0;
  return XAC_OK;
}

}  // namespace

extern "C" {

const char* xac_last_error(void) { return xac::g_err; }
int xac_version(void) { return 10000; }

int xac_lattice_create(const xac_desc* desc, xac_lattice** out, void* stream) {
  XAC_REQUIRE(out, "xac_lattice_create: null output handle");
  *out = nullptr;
  xac_lattice* lat = new (std::nothrow) xac_lattice();
  if (!lat) {
    set_error("xac_lattice_create: host allocation failed");
    return XAC_ENOMEM;
  }
  cudaStream_t s = as_stream(stream);
  int r = create_impl(desc, lat->impl, s);
  if (r == XAC_OK) r = init_impl(lat->impl, nullptr, nullptr, nullptr, s);
  if (r != XAC_OK) {
    delete lat;
    return r;
  }
  *out = lat;
  return XAC_OK;
}

int xac_lattice_destroy(xac_lattice* lat) {
  if (!lat) return XAC_OK;
  cudaDeviceSynchronize();
  delete lat;
  return XAC_OK;
}

int xac_lattice_init_fields(xac_lattice* lat, const float* rho, const float* u, const float* T, void* stream) {
  XAC_REQUIRE(lat, "xac_lattice_init_fields: null lattice");
  std::lock_guard<std::mutex> g(lat->impl.mu);
  LatticeImpl& L = lat->impl;
  XAC_CUDA(cudaMemsetAsync(L.status, 0, sizeof(unsigned), as_stream(stream)));
  L.failed = false;
  return init_impl(L, rho, u, T, as_stream(stream));
}

int xac_test_set_step_status(xac_lattice* lat, unsigned value, void* stream) {
  XAC_REQUIRE(lat, "xac_test_set_step_status: null lattice");
  std::lock_guard<std::mutex> g(lat->impl.mu);
  cudaStream_t s = as_stream(stream);
  XAC_CUDA(cudaMemcpyAsync(lat->impl.status, &value, sizeof(value), cudaMemcpyHostToDevice, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

int xac_lattice_step(xac_lattice* lat, int n, void* stream) {
  XAC_REQUIRE(lat, "xac_lattice_step: null lattice");
  XAC_REQUIRE(n >= 0, "xac_lattice_step: negative step count %d", n);
  std::lock_guard<std::mutex> g(lat->impl.mu);
  if (lat->impl.failed) return lat->impl.refuse("xac_lattice_step");
  return lat->impl.steps(n, as_stream(stream));
}

int xac_lattice_stats(xac_lattice* lat, double* out_host, void* stream) {
  XAC_REQUIRE(lat && out_host, "xac_lattice_stats: null pointer");
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  if (L.failed) return L.refuse("xac_lattice_stats");
  cudaStream_t s = as_stream(stream);
  int r = L.finalize_T(s);
  if (r != XAC_OK) return r;
  r = run_stats(L.view(), L.rows, L.red_out, L.host_out, s);
  if (r != XAC_OK) return r;
  std::memcpy(out_host, L.host_out, kNStats * sizeof(double));
  if (L.tune_variant == 1) {  // the staged kernel's bounded wait reports here
    unsigned st = 0;
    XAC_CUDA(cudaMemcpyAsync(&st, L.status, sizeof(st), cudaMemcpyDeviceToHost, s));
    XAC_CUDA(cudaStreamSynchronize(s));
    if (st) {
      L.failed = true;
      set_error("xac_lattice_stats: a staged step kernel gave up waiting for its copies (status %u); the lattice "
                "refuses further work until init_fields or load_state", st);
      return XAC_ETIMEOUT;
    }
  }
  return XAC_OK;
}

int xac_lattice_fields(xac_lattice* lat, float* rho, float* u, float* T, void* stream) {
  XAC_REQUIRE(lat, "xac_lattice_fields: null lattice");
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  if (L.failed) return L.refuse("xac_lattice_fields");
  cudaStream_t s = as_stream(stream);
  if (T) {
    int r = L.finalize_T(s);
    if (r != XAC_OK) return r;
  }
  export_fields_kernel<<<grid_for(L.g.ncell, kBlock), kBlock, 0, s>>>(L.rho, L.ux, L.uy, L.uz, L.T, rho, u, T, L.g);
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}

int xac_lattice_set_inlet(xac_lattice* lat, double u_inlet, void* stream) {
  XAC_REQUIRE(lat, "xac_lattice_set_inlet: null lattice");
  XAC_REQUIRE(std::isfinite(u_inlet) && u_inlet < 1.0, "xac_lattice_set_inlet: u_inlet %g out of range", u_inlet);
  lat->impl.u_in_host = (float)u_inlet;
  set_scalar_kernel<<<1, 1, 0, as_stream(stream)>>>(lat->impl.u_in, (float)u_inlet);
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}

int xac_lattice_get_inlet(xac_lattice* lat, double* u_inlet, void*) {
  XAC_REQUIRE(lat && u_inlet, "xac_lattice_get_inlet: null pointer");
  *u_inlet = (double)lat->impl.u_in_host;
  return XAC_OK;
}

int xac_lattice_pattern_copy(xac_lattice* lat, int launches, double* us_per_launch, void* stream) {
  XAC_REQUIRE(lat && us_per_launch, "xac_lattice_pattern_copy: null pointer");
  XAC_REQUIRE(launches >= 1 && launches <= 100000, "xac_lattice_pattern_copy: launches %d out of 1..100000",
              launches);
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  cudaStream_t s = as_stream(stream);
  auto launch = [&](int k) {
    const int c = k & 1;
    switch (L.precision) {
      case XAC_FP16:
        launch_pattern_copy<__half, __half>(L.P[c], L.P[c ^ 1], L.Qb[c], L.Qb[c ^ 1], L.link, L.ftab, L.g, L.tune_block, c, s);
        break;
      case XAC_BF16:
        launch_pattern_copy<__nv_bfloat16, __half>(L.P[c], L.P[c ^ 1], L.Qb[c], L.Qb[c ^ 1], L.link, L.ftab, L.g,
                                                        L.tune_block, c, s);
        break;
      case XAC_FP32_T16:
        launch_pattern_copy<float, __half>(L.P[c], L.P[c ^ 1], L.Qb[c], L.Qb[c ^ 1], L.link, L.ftab, L.g, L.tune_block, c,
                                                s);
        break;
      default:
        launch_pattern_copy<float, float>(L.P[c], L.P[c ^ 1], L.Qb[c], L.Qb[c ^ 1], L.link, L.ftab, L.g, L.tune_block, c, s);
    }
  };
  for (int k = 0; k < 4; ++k) launch(k);  // warm-up
  cudaEvent_t a = nullptr, b = nullptr;
  XAC_CUDA(cudaEventCreate(&a));
  cudaError_t e = cudaEventCreate(&b);
  if (e == cudaSuccess) e = cudaEventRecord(a, s);
  for (int k = 0; e == cudaSuccess && k < launches; ++k) launch(k);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(b, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_status(e, "xac_lattice_pattern_copy");
  *us_per_launch = (double)ms * 1e3 / launches;
  // the probe left copies, not a physical state: start the lattice over from the cold start
  return init_impl(L, nullptr, nullptr, nullptr, s);
}

int xac_lattice_tune(xac_lattice* lat, int block, int variant) {
  XAC_REQUIRE(lat, "xac_lattice_tune: null lattice");
  XAC_REQUIRE(block == 64 || block == 128 || block == 256, "xac_lattice_tune: block must be 64, 128 or 256 (got %d)",
              block);
  XAC_REQUIRE(variant == 0 || variant == 1, "xac_lattice_tune: variant must be 0 or 1 (got %d)", variant);
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  if (L.tune_block != block || L.tune_variant != variant) {
    for (auto& kv : L.graphs) cudaGraphExecDestroy(kv.second);
    L.graphs.clear();
    for (auto& kv : L.run_graphs) cudaGraphExecDestroy(kv.second);
    L.run_graphs.clear();
  }
  L.tune_block = block;
  L.tune_variant = variant;
  return XAC_OK;
}

int xac_lattice_get_tune(const xac_lattice* lat, int* block, int* variant) {
  XAC_REQUIRE(lat && block && variant, "xac_lattice_get_tune: null pointer");
  *block = lat->impl.tune_block;
  *variant = lat->impl.tune_variant;
  return XAC_OK;
}

int xac_lattice_steps_done(const xac_lattice* lat, long long* steps) {
  XAC_REQUIRE(lat && steps, "xac_lattice_steps_done: null pointer");
  *steps = lat->impl.step;
  return XAC_OK;
}

int xac_lattice_scalars(xac_lattice* lat, const xac_scalar_params* prm, double* out_host, void* stream) {
  XAC_REQUIRE(lat && prm && out_host, "xac_lattice_scalars: null pointer");
  LatticeImpl& L = lat->impl;
  XAC_REQUIRE(prm->buf >= 0 && 2 * prm->buf < L.g.nx, "xac_lattice_scalars: bad buffer length %d", prm->buf);
  std::lock_guard<std::mutex> g(L.mu);
  if (L.failed) return L.refuse("xac_lattice_scalars");
  cudaStream_t s = as_stream(stream);
  int r = L.finalize_T(s);
  if (r != XAC_OK) return r;
  MetricBox b{prm->buf, prm->core_nx, prm->core_ny};
  r = run_metrics(L.view(), b, L.rows, L.red_blocks, L.red_out, L.host_out, s);
  if (r != XAC_OK) return r;
  assemble_scalars(L.host_out, L.g.nx, L.g.ny, L.g.nz, prm->buf, prm->t_inlet, prm->tau_fluid, prm->Pr,
                   prm->u_inlet, out_host);
  return XAC_OK;
}

int xac_lattice_validate(xac_lattice* lat, double* out_host, void* stream) {
  XAC_REQUIRE(lat && out_host, "xac_lattice_validate: null pointer");
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  if (L.failed) return L.refuse("xac_lattice_validate");
  cudaStream_t s = as_stream(stream);
  int r = L.finalize_T(s);  // rho and u are written by the last step of every step call
  if (r != XAC_OK) return r;
  // analyze_dataset.py:274-281 in double
  const double tth_f = 0.5 + (L.tau_fluid - 0.5) / L.Pr, tth_s = 0.5 + L.k_ratio * (tth_f - 0.5);
  const double k_fluid = (1.0 / 3.0) * (tth_f - 0.5), k_solid = (1.0 / 3.0) * (tth_s - 0.5);
  const auto spec = validate_spec();
  validate_partials_kernel<<<L.red_blocks, kBlock, 0, s>>>(L.view(), L.qsrc, k_fluid, k_solid, spec, L.rows);
  combine_rows_kernel<kNValidate><<<1, 32 * kNValidate, 0, s>>>(L.rows, L.red_blocks, spec, L.red_out);
  XAC_CUDA(cudaGetLastError());
  XAC_CUDA(cudaMemcpyAsync(L.host_out, L.red_out, kNValidate * sizeof(double), cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  std::memcpy(out_host, L.host_out, kNValidate * sizeof(double));
  return XAC_OK;
}

int xac_lattice_state_bytes(const xac_lattice* lat, size_t* bytes) {
  XAC_REQUIRE(lat && bytes, "xac_lattice_state_bytes: null pointer");
  const LatticeImpl& L = lat->impl;
  *bytes = 64 + (size_t)L.g.np * L.p_elem + (size_t)L.g.N * L.q_elem + 5 * (size_t)L.g.ncell * sizeof(float);
  return XAC_OK;
}

int xac_lattice_save_state(xac_lattice* lat, void* host_dst, size_t bytes, void* stream) {
  XAC_REQUIRE(lat && host_dst, "xac_lattice_save_state: null pointer");
  size_t need = 0;
  xac_lattice_state_bytes(lat, &need);
  XAC_REQUIRE(bytes >= need, "xac_lattice_save_state: buffer of %zu bytes, need %zu", bytes, need);
  LatticeImpl& L = lat->impl;
  std::lock_guard<std::mutex> g(L.mu);
  if (L.failed) return L.refuse("xac_lattice_save_state");
  cudaStream_t s = as_stream(stream);
  int r = L.finalize_T(s);
  if (r != XAC_OK) return r;
  int64_t hdr[8] = {0x58414332, L.g.nx, L.g.ny, L.g.nz, L.precision, L.step, L.own_pending ? 1 : 0, 0};
  float u_in = L.u_in_host;
  std::memcpy(&hdr[7], &u_in, sizeof(float));
  std::memcpy(reinterpret_cast<char*>(&hdr[7]) + 4, &L.nonsolid, sizeof(uint32_t));
  char* dst = (char*)host_dst;
  std::memcpy(dst, hdr, 64);
  const size_t pb = (size_t)L.g.np * L.p_elem, qb = (size_t)L.g.N * L.q_elem;
  const size_t nf = (size_t)L.g.ncell * sizeof(float);
  XAC_CUDA(cudaMemcpyAsync(dst + 64, L.P[L.cur], pb, cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaMemcpyAsync(dst + 64 + pb, L.Qb[L.cur], qb, cudaMemcpyDeviceToHost, s));
  const float* f[5] = {L.rho, L.ux, L.uy, L.uz, L.T};
  for (int k = 0; k < 5; ++k)
    XAC_CUDA(cudaMemcpyAsync(dst + 64 + pb + qb + k * nf, f[k], nf, cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

int xac_lattice_load_state(xac_lattice* lat, const void* host_src, size_t bytes, void* stream) {
  XAC_REQUIRE(lat && host_src, "xac_lattice_load_state: null pointer");
  size_t need = 0;
  xac_lattice_state_bytes(lat, &need);
  XAC_REQUIRE(bytes >= need, "xac_lattice_load_state: buffer of %zu bytes, need %zu", bytes, need);
  LatticeImpl& L = lat->impl;
  int64_t hdr[8];
  std::memcpy(hdr, host_src, 64);
  uint32_t nonsolid = 0;
  std::memcpy(&nonsolid, reinterpret_cast<const char*>(&hdr[7]) + 4, sizeof(uint32_t));
  XAC_REQUIRE(hdr[0] == 0x58414332 && hdr[1] == L.g.nx && hdr[2] == L.g.ny && hdr[3] == L.g.nz &&
                  hdr[4] == L.precision && nonsolid == L.nonsolid,
              "xac_lattice_load_state: state was saved from a different lattice (size, precision or mask)");
  std::lock_guard<std::mutex> g(L.mu);
  cudaStream_t s = as_stream(stream);
  const char* src = (const char*)host_src;
  const size_t pb = (size_t)L.g.np * L.p_elem, qb = (size_t)L.g.N * L.q_elem;
  const size_t nf = (size_t)L.g.ncell * sizeof(float);
  XAC_CUDA(cudaMemcpyAsync(L.P[0], src + 64, pb, cudaMemcpyHostToDevice, s));
  XAC_CUDA(cudaMemcpyAsync(L.Qb[0], src + 64 + pb, qb, cudaMemcpyHostToDevice, s));
  float* f[5] = {L.rho, L.ux, L.uy, L.uz, L.T};
  for (int k = 0; k < 5; ++k)
    XAC_CUDA(cudaMemcpyAsync(f[k], src + 64 + pb + qb + k * nf, nf, cudaMemcpyHostToDevice, s));
  float u_in;
  std::memcpy(&u_in, &hdr[7], sizeof(float));
  L.u_in_host = u_in;
  set_scalar_kernel<<<1, 1, 0, s>>>(L.u_in, u_in);
  XAC_CUDA(cudaMemsetAsync(L.status, 0, sizeof(unsigned), s));
  XAC_CUDA(cudaStreamSynchronize(s));
  L.failed = false;
  L.cur = 0;
  L.step = hdr[5];
  L.own_pending = hdr[6] != 0;
  L.macro_step = L.step;
  L.T_step = L.step;
  return XAC_OK;
}

// ---- test-only: bounded waits that run out ----------------------------------------------------------------
// The staged step kernel waits on an mbarrier, the batched kernel at a grid barrier; both waits are bounded.
// Here one block waits on an mbarrier that nothing arrives on, and a two-block grid meets at the batch kernel's
// grid barrier with one block that never arrives: both waits must give up after `limit` polls and report,
// and the context stays usable.
static __global__ void test_mbarrier_timeout_kernel(uint32_t limit, unsigned* status) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = sh_addr(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = bar_wait_bounded(b, 0, limit);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (!ok) atomicOr(status, 1u);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(b) : "memory");
  }
}

static __global__ void test_grid_barrier_timeout_kernel(BatchCtl* ctl, unsigned long long limit, unsigned* status) {
  if (blockIdx.x == gridDim.x - 1) return;  // this block never arrives
  if (!grid_sync(ctl, limit) && threadIdx.x == 0) atomicOr(status, 2u);
}

extern "C" int xac_test_bounded_waits(unsigned limit, unsigned* status_out, void* stream) {
  XAC_REQUIRE(status_out, "xac_test_bounded_waits: null pointer");
  XAC_REQUIRE(limit > 0 && limit <= (1u << 20), "xac_test_bounded_waits: limit %u out of (0, 2^20]", limit);
  cudaStream_t s = as_stream(stream);
  unsigned* st = nullptr;
  BatchCtl* ctl = nullptr;
  XAC_CUDA(cudaMalloc(&st, sizeof(unsigned)));
  cudaError_t e = cudaMalloc(&ctl, sizeof(BatchCtl));
  if (e == cudaSuccess) e = cudaMemsetAsync(st, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctl, 0, sizeof(BatchCtl), s);
  if (e == cudaSuccess) {
    test_mbarrier_timeout_kernel<<<1, 32, 0, s>>>(limit, st);
    test_grid_barrier_timeout_kernel<<<2, 32, 0, s>>>(ctl, (unsigned long long)limit, st);
    e = cudaGetLastError();
  }
  unsigned host = 0;
  int err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&host, st, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &ctl->err, sizeof(err), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(st);
  cudaFree(ctl);
  if (e != cudaSuccess) return cuda_status(e, "xac_test_bounded_waits");
  *status_out = host | (err == XAC_ETIMEOUT ? 4u : 0u);  // bit 2: the grid barrier recorded XAC_ETIMEOUT
  return XAC_OK;
}

// simulation.py:102-162
int xac_lattice_run(xac_lattice* lat, const xac_run_opts* o, xac_run_result* res, void* stream) {
  XAC_REQUIRE(lat && o && res, "xac_lattice_run: null pointer");
  XAC_REQUIRE(o->stats_every > 0 && o->max_steps >= 0, "xac_lattice_run: bad options");
  LatticeImpl& L = lat->impl;
  if (L.failed) return L.refuse("xac_lattice_run");
  std::memset(res, 0, sizeof(*res));
  const long long min_steps = o->min_steps > 0 ? o->min_steps : L.reference_min_steps(o->max_steps);
  double prev_ke = 0.0, prev_max_T = 0.0, d_ke = 0.0, dT = 0.0, prev_Q = 0.0, dQ = 1.0;
  double st[kNStats];
  const long long start = L.step;
  long long step = 0;
  int diverged = 0;
  bool tried_device = false;
  while (step < o->max_steps) {
    int chunk = o->stats_every - (int)((start + step) % o->stats_every);
    if (step + chunk > o->max_steps) chunk = (int)(o->max_steps - step);
    int r = xac_lattice_step(lat, chunk, stream);
    if (r != XAC_OK) return r;
    step += chunk;
    if ((start + step) % o->stats_every != 0) continue;
    r = xac_lattice_stats(lat, st, stream);
    if (r != XAC_OK) return r;
    const double max_v = st[XAC_ST_MAX_V], ke = st[XAC_ST_SUM_KE], max_T = st[XAC_ST_MAX_T],
                 Q_out = st[XAC_ST_Q_OUT];
    const bool past = (start + step) > o->stats_every;
    d_ke = past ? std::fabs(ke - prev_ke) / (prev_ke + 1e-9) / o->stats_every : 0.0;
    dT = past ? std::fabs(max_T - prev_max_T) / (prev_max_T + 1e-9) / o->stats_every : 0.0;
    dQ = past ? std::fabs(Q_out - prev_Q) / (std::fabs(prev_Q) + 1e-12) / o->stats_every : 1.0;
    prev_ke = ke;
    prev_max_T = max_T;
    prev_Q = Q_out;
    if (o->constant_power && (start + step) > 2000) {
      double ue = (double)L.u_in_host;
      const double rin = st[XAC_ST_C_IN] > 0 ? st[XAC_ST_SUM_RHO_IN] / st[XAC_ST_C_IN] : 1.0;
      const double rout = st[XAC_ST_C_OUT] > 0 ? st[XAC_ST_SUM_RHO_OUT] / st[XAC_ST_C_OUT] : 1.0;
      const double dP = (rin - rout) / 3.0;
      const double pw = dP * (ue * st[XAC_ST_C_IN]);
      ue = ue + 0.005 * (o->target_power - pw);
      ue = ue < 0.0001 ? 0.0001 : (ue > 0.15 ? 0.15 : ue);
      r = xac_lattice_set_inlet(lat, ue, stream);
      if (r != XAC_OK) return r;
    }
    std::memcpy(res->last_stats, st, sizeof(st));
    if (step > min_steps && d_ke < o->tol_ke && dT < o->tol_T && dQ < o->tol_T) break;
    if (st[XAC_ST_NONFINITE] > 0 || max_v > 0.17 || max_T > 1e4) {
      diverged = 1;
      break;
    }
    // After the first check, the remaining whole stats intervals run as one graph launch with the loop on the
    // device (same arithmetic, same decisions); the host reads the loop state back once.
    const long long iters = (o->max_steps - step) / o->stats_every;
    if (!tried_device && o->stats_every % 2 == 0 && o->stats_every >= 8 && iters >= 2 && !L.own_pending &&
        (start + step) % o->stats_every == 0) {
      tried_device = true;
      cudaStream_t s = as_stream(stream);
      std::lock_guard<std::mutex> g(L.mu);
      cudaGraphExec_t ex = nullptr;
      r = L.run_graph(o->stats_every, &ex);
      if (r != XAC_OK) return r;
      RunCtl& c = *L.run_ctl_host;
      std::memset(&c, 0, sizeof(c));
      c.start = start;
      c.step = step;
      c.min_steps = min_steps;
      c.max_iters = iters;
      c.stats_every = o->stats_every;
      c.constant_power = o->constant_power;
      c.tol_ke = o->tol_ke;
      c.tol_T = o->tol_T;
      c.target_power = o->target_power;
      c.prev_ke = prev_ke;
      c.prev_max_T = prev_max_T;
      c.prev_Q = prev_Q;
      c.d_ke = d_ke;
      c.dT = dT;
      c.dQ = dQ;
      c.u_in = L.u_in_host;
      XAC_CUDA(cudaMemcpyAsync(L.run_ctl, &c, sizeof(RunCtl), cudaMemcpyHostToDevice, s));
      XAC_CUDA(cudaGraphLaunch(ex, s));
      XAC_CUDA(cudaMemcpyAsync(&c, L.run_ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s));
      XAC_CUDA(cudaStreamSynchronize(s));
      L.step += c.step - step;
      L.macro_step = L.step;
      L.T_step = L.step;
      L.u_in_host = c.u_in;
      step = c.step;
      prev_ke = c.prev_ke;
      prev_max_T = c.prev_max_T;
      prev_Q = c.prev_Q;
      d_ke = c.d_ke;
      dT = c.dT;
      dQ = c.dQ;
      std::memcpy(res->last_stats, c.last, sizeof(c.last));
      if (L.tune_variant == 1) {  // the staged kernel's bounded wait reports here
        unsigned stw = 0;
        XAC_CUDA(cudaMemcpy(&stw, L.status, sizeof(stw), cudaMemcpyDeviceToHost));
        if (stw) {
          L.failed = true;
          set_error("xac_lattice_run: a staged step kernel gave up waiting for its copies (status %u); the lattice "
                    "refuses further work until init_fields or load_state", stw);
          return XAC_ETIMEOUT;
        }
      }
      if (c.diverged) {
        diverged = 1;
        break;
      }
      if (step > min_steps && d_ke < o->tol_ke && dT < o->tol_T && dQ < o->tol_T) break;
    }
  }
  res->steps = step;
  res->converged = (step > min_steps && d_ke < o->tol_ke && dT < o->tol_T && dQ < o->tol_T) ? 1 : 0;
  res->diverged = diverged;
  res->d_ke = d_ke;
  res->dT_conv = dT;
  res->dQ_conv = dQ;
  res->u_inlet_final = (double)L.u_in_host;
  return XAC_OK;
}

// Deterministic stats of arbitrary reference-layout fields (the two reference stats kernels, merged).
int xac_stats_fields(const float* rho, const float* u, const float* T, const int32_t* mask, int nx, int ny, int nz,
                     double* out_host, void* stream) {
  XAC_REQUIRE(rho && u && T && mask && out_host, "xac_stats_fields: null pointer");
  XAC_REQUIRE(nx > 0 && ny > 0 && nz > 0, "xac_stats_fields: bad dimensions");
  cudaStream_t s = as_stream(stream);
  const long long n = (long long)nx * ny * nz;
  double* rows = nullptr;
  double* dout = nullptr;
  double* hout = nullptr;
  int r = dmalloc(&rows, (size_t)stats_tiles(n) * kNStats, "alloc rows");
  if (r == XAC_OK) r = dmalloc(&dout, kNStats, "alloc out");
  if (r == XAC_OK && cudaMallocHost(&hout, kNStats * sizeof(double)) != cudaSuccess) r = XAC_ENOMEM;
  if (r == XAC_OK) {
    FieldView v{};
    v.rho = rho;
    v.ux = u;
    v.uy = u + 1;
    v.uz = u + 2;
    v.ustride = 3;
    v.T = T;
    v.mask = mask;
    v.link = nullptr;
    v.sx = (long long)ny * nz;
    v.sy = nz;
    v.sz = 1;
    v.nx = nx;
    v.ny = ny;
    v.nz = nz;
    r = run_stats(v, rows, dout, hout, s);
    if (r == XAC_OK) std::memcpy(out_host, hout, kNStats * sizeof(double));
  }
  cudaFree(rows);
  cudaFree(dout);
  if (hout) cudaFreeHost(hout);
  return r;
}

int xac_scalars_fields(const float* rho, const float* u, const float* T, const int32_t* mask, int nx, int ny, int nz,
                       const xac_scalar_params* prm, double* out_host, void* stream) {
  XAC_REQUIRE(rho && u && T && mask && prm && out_host, "xac_scalars_fields: null pointer");
  XAC_REQUIRE(nx > 0 && ny > 0 && nz > 0, "xac_scalars_fields: bad dimensions");
  XAC_REQUIRE(prm->buf >= 0 && 2 * prm->buf < nx, "xac_scalars_fields: bad buffer length %d", prm->buf);
  cudaStream_t s = as_stream(stream);
  const long long n = (long long)nx * ny * nz;
  const int nb = reduction_blocks(n);
  double* rows = nullptr;
  double* dout = nullptr;
  double* hout = nullptr;
  int r = dmalloc(&rows, (size_t)nb * kNMetrics, "alloc rows");
  if (r == XAC_OK) r = dmalloc(&dout, kNMetrics, "alloc out");
  if (r == XAC_OK && cudaMallocHost(&hout, kNMetrics * sizeof(double)) != cudaSuccess) r = XAC_ENOMEM;
  if (r == XAC_OK) {
    FieldView v{};
    v.rho = rho;
    v.ux = u;
    v.uy = u + 1;
    v.uz = u + 2;
    v.ustride = 3;
    v.T = T;
    v.mask = mask;
    v.link = nullptr;
    v.sx = (long long)ny * nz;
    v.sy = nz;
    v.sz = 1;
    v.nx = nx;
    v.ny = ny;
    v.nz = nz;
    MetricBox b{prm->buf, prm->core_nx, prm->core_ny};
    r = run_metrics(v, b, rows, nb, dout, hout, s);
    if (r == XAC_OK)
      assemble_scalars(hout, nx, ny, nz, prm->buf, prm->t_inlet, prm->tau_fluid, prm->Pr, prm->u_inlet, out_host);
  }
  cudaFree(rows);
  cudaFree(dout);
  if (hout) cudaFreeHost(hout);
  return r;
}

}  // extern "C"

// =====================================================================================================
// Batch of designs advanced by one persistent cooperative launch (batch.cuh)
// =====================================================================================================
struct xac_batch {
  std::vector<xac_lattice*> lats;  // slot -> design (open batches: nullptr for a free slot)
  // open batches (xac_batch_open): designs join and leave while the batch runs
  enum : int { kFree = 0, kPending = 1, kActive = 2, kDone = 3 };
  bool open = false;
  std::vector<int> state;      // per slot
  std::vector<double> gpu_s;   // per slot: its share of the launches' wall time since it joined
  long long gstep = 0;         // global step of the batch
  long long graph_launches = 0, direct_launches = 0;
  int precision = XAC_FP32;
  int block = 128;              // threads per block (= cells per tile)
  int steps_per_launch = 1000;  // steps one launch may advance
  BatchDesign* dD = nullptr;
  BatchCtl* dC = nullptr;
  double* drows = nullptr;
  size_t rows_cap = 0;
  BatchCtl* hC = nullptr;  // pinned
  std::vector<BatchDesign> hD;
  // captured persistent launches, keyed by every launch option they hold; the device pointers they hold (designs,
  // control block, stats rows) are the batch's for its lifetime, except the stats rows of an open batch, whose
  // reallocation drops every cached graph
  std::map<std::tuple<int, long long, int, double, double, int, double>, cudaGraphExec_t> graphs;
  void drop_graphs() {
    for (auto& kv : graphs)
      if (kv.second) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }
  cudaStream_t capture = nullptr;
  ~xac_batch() {
    drop_graphs();
    if (capture) cudaStreamDestroy(capture);
    cudaFree(dD);
    cudaFree(dC);
    cudaFree(drows);
    if (hC) cudaFreeHost(hC);
    for (auto* l : lats) delete l;
  }
};

namespace {

template <typename SP, typename SQ>
int batch_launch(xac_batch* b, const BatchRun& run, cudaStream_t s, bool use_graph) {
  int dev = 0, sms = 0, per_sm = 0;
  XAC_CUDA(cudaGetDevice(&dev));
  XAC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  XAC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent_kernel<SP, SQ>, b->block, 0));
  XAC_REQUIRE(per_sm > 0, "xac_batch_run: the persistent kernel does not fit on an SM with %d threads", b->block);
  const int grid = sms * per_sm;  // every block resident: the grid barrier cannot deadlock
  BatchDesign* D = b->dD;
  BatchCtl* C = b->dC;
  double* rows = b->drows;
  BatchRun r = run;
  void* args[] = {&D, &C, &rows, &r};
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(b->block);
  cfg.dynamicSmemBytes = 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (use_graph) {
    const auto key =
        std::make_tuple(run.steps, run.max_steps, run.stats_every, run.tol_ke, run.tol_T, run.constant_power,
                        run.target_power);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      if (!b->capture) XAC_CUDA(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
      cudaGraph_t graph = nullptr;
      cfg.stream = b->capture;
      XAC_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = cudaLaunchKernelExC(&cfg, (const void*)batch_persistent_kernel<SP, SQ>, args);
      cudaError_t ce = cudaStreamEndCapture(b->capture, &graph);
      cudaGraphExec_t exec = nullptr;
      if (le == cudaSuccess && ce == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        it = b->graphs.emplace(key, exec).first;
      } else {
        // the driver could not capture a cooperative launch: launch directly from now on
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        b->graphs.emplace(key, (cudaGraphExec_t) nullptr);
        it = b->graphs.find(key);
      }
    }
    if (it->second) {
      XAC_CUDA(cudaGraphLaunch(it->second, s));
      ++b->graph_launches;
      return XAC_OK;
    }
  }
  cfg.stream = s;
  XAC_CUDA(cudaLaunchKernelExC(&cfg, (const void*)batch_persistent_kernel<SP, SQ>, args));
  ++b->direct_launches;
  return XAC_OK;
}

int batch_launch_any(xac_batch* b, const BatchRun& run, cudaStream_t s, bool use_graph) {
  switch (b->precision) {
    case XAC_FP16: return batch_launch<__half, __half>(b, run, s, use_graph);
    case XAC_BF16: return batch_launch<__nv_bfloat16, __half>(b, run, s, use_graph);
    case XAC_FP32_T16: return batch_launch<float, __half>(b, run, s, use_graph);
    default: return batch_launch<float, float>(b, run, s, use_graph);
  }
}

// Descriptor of design L for the persistent kernel, joining the batch at global step `start`.
void fill_design(BatchDesign& d, LatticeImpl& L, int block, long long min_steps, long long start) {
  d = BatchDesign{};
  d.p = L.params();
  d.P[0] = L.P[0];
  d.P[1] = L.P[1];
  d.Q[0] = L.Qb[0];
  d.Q[1] = L.Qb[1];
  d.link = L.link;
  d.qsrc = L.qsrc;
  d.u_in = L.u_in;
  d.rho = L.rho;
  d.ux = L.ux;
  d.uy = L.uy;
  d.uz = L.uz;
  d.T = L.T;
  d.ncell = (uint32_t)L.g.ncell;
  d.tiles = (uint32_t)(((long long)L.g.rows * L.g.pitch + block - 1) / block);  // row positions
  d.stat_tiles = (uint32_t)stats_tiles(L.g.ncell);
  d.min_steps = min_steps;
  d.start = start;
  d.active = 1;
  d.dQ = 1.0;
}

// Control block of a launch over the designs in `act` (slot indices, ascending): active list, tile prefixes and
// the stats rows of each design (packed in list order).
void build_ctl(xac_batch* b, const std::vector<int>& act, long long step) {
  std::memset(b->hC, 0, sizeof(BatchCtl));
  uint32_t acc = 0, sacc = 0;
  for (size_t k = 0; k < act.size(); ++k) {
    BatchDesign& d = b->hD[act[k]];
    d.row_base = sacc;
    b->hC->active[k] = (uint32_t)act[k];
    b->hC->prefix[k] = acc;
    b->hC->stat_prefix[k] = sacc;
    acc += d.tiles;
    sacc += d.stat_tiles;
  }
  b->hC->prefix[act.size()] = acc;
  b->hC->stat_prefix[act.size()] = sacc;
  b->hC->n_active = (int)act.size();
  b->hC->all_done = act.empty() ? 1 : 0;
  b->hC->step = step;
}

// A finished design's outcome, and its lattice left at its last step (fields, stats and scalars then read it).
void finish_design(xac_batch* b, int slot, long long steps, float u_fin, const xac_run_opts* o, xac_run_result& rr) {
  const BatchDesign& d = b->hD[slot];
  std::memset(&rr, 0, sizeof(rr));
  rr.steps = steps;
  rr.diverged = d.diverged;
  rr.converged = d.converged ? 1 : (!d.diverged && steps > d.min_steps && d.d_ke < o->tol_ke && d.dT < o->tol_T &&
                                    d.dQ < o->tol_T);
  rr.d_ke = d.d_ke;
  rr.dT_conv = d.dT;
  rr.dQ_conv = d.dQ;
  rr.u_inlet_final = (double)u_fin;
  std::memcpy(rr.last_stats, d.last, sizeof(d.last));
  LatticeImpl& L = b->lats[slot]->impl;
  L.u_in_host = u_fin;
  L.step = steps;
  L.cur = (int)(steps & 1);
  L.own_pending = steps == 0;
  L.macro_step = steps;
  L.T_step = (steps % o->stats_every == 0) ? steps : -1;
}

}  // namespace

extern "C" {

int xac_batch_create(const xac_desc* descs, int n, xac_batch** out, void* stream) {
  XAC_REQUIRE(out && descs, "xac_batch_create: null pointer");
  XAC_REQUIRE(n >= 1 && n <= kMaxBatch, "xac_batch_create: batch size %d outside 1..%d", n, kMaxBatch);
  *out = nullptr;
  for (int i = 1; i < n; ++i)
    XAC_REQUIRE(descs[i].precision == descs[0].precision, "xac_batch_create: designs must share one precision");
  xac_batch* b = new (std::nothrow) xac_batch();
  if (!b) {
    set_error("xac_batch_create: host allocation failed");
    return XAC_ENOMEM;
  }
  b->precision = descs[0].precision;
  for (int i = 0; i < n; ++i) {
    xac_lattice* l = nullptr;
    int r = xac_lattice_create(&descs[i], &l, stream);
    if (r != XAC_OK) {
      delete b;
      return r;
    }
    b->lats.push_back(l);
  }
  size_t rows = 0;
  for (auto* l : b->lats) rows += (size_t)stats_tiles(l->impl.g.ncell);
  b->rows_cap = rows;
  int r = XAC_OK;
  if ((r = dmalloc(&b->dD, (size_t)n, "alloc batch designs")) != XAC_OK ||
      (r = dmalloc(&b->dC, 1, "alloc batch control")) != XAC_OK ||
      (r = dmalloc(&b->drows, rows * kNStats, "alloc batch rows")) != XAC_OK) {
    delete b;
    return r;
  }
  if (cudaMallocHost(&b->hC, sizeof(BatchCtl)) != cudaSuccess) {
    delete b;
    set_error("xac_batch_create: pinned allocation failed");
    return XAC_ENOMEM;
  }
  *out = b;
  return XAC_OK;
}

int xac_batch_destroy(xac_batch* b) {
  if (!b) return XAC_OK;
  cudaDeviceSynchronize();
  delete b;
  return XAC_OK;
}

int xac_batch_size(const xac_batch* b, int* n) {
  XAC_REQUIRE(b && n, "xac_batch_size: null pointer");
  *n = (int)b->lats.size();
  return XAC_OK;
}

int xac_batch_lattice(xac_batch* b, int i, xac_lattice** lat) {
  XAC_REQUIRE(b && lat, "xac_batch_lattice: null pointer");
  XAC_REQUIRE(i >= 0 && i < (int)b->lats.size(), "xac_batch_lattice: index %d out of range", i);
  XAC_REQUIRE(b->lats[i], "xac_batch_lattice: slot %d holds no design", i);
  *lat = b->lats[i];
  return XAC_OK;
}

int xac_batch_tune(xac_batch* b, int block, int steps_per_launch) {
  XAC_REQUIRE(b, "xac_batch_tune: null batch");
  XAC_REQUIRE(block == 64 || block == 128 || block == 256, "xac_batch_tune: block must be 64, 128 or 256");
  XAC_REQUIRE(steps_per_launch >= 1, "xac_batch_tune: steps_per_launch must be positive");
  if (b->block != block) {
    b->drop_graphs();
  }
  b->block = block;
  b->steps_per_launch = steps_per_launch;
  return XAC_OK;
}

int xac_batch_get_tune(const xac_batch* b, int* block, int* steps_per_launch) {
  XAC_REQUIRE(b && block && steps_per_launch, "xac_batch_get_tune: null pointer");
  *block = b->block;
  *steps_per_launch = b->steps_per_launch;
  return XAC_OK;
}

int xac_batch_run(xac_batch* b, const xac_run_opts* o, xac_run_result* res, void* stream) {
  XAC_REQUIRE(b && o && res, "xac_batch_run: null pointer");
  XAC_REQUIRE(!b->open, "xac_batch_run: an open batch advances with xac_batch_advance");
  XAC_REQUIRE(o->stats_every > 0 && o->max_steps >= 0, "xac_batch_run: bad options");
  cudaStream_t s = as_stream(stream);
  const int n = (int)b->lats.size();
  b->hD.assign(n, BatchDesign{});
  std::vector<int> act(n);
  for (int i = 0; i < n; ++i) {
    LatticeImpl& L = b->lats[i]->impl;
    XAC_REQUIRE(L.step == 0 && L.own_pending,
                "xac_batch_run: design %d is not at step 0 (create it or re-initialise it with init_fields)", i);
    fill_design(b->hD[i], L, b->block, o->min_steps > 0 ? o->min_steps : L.reference_min_steps(o->max_steps), 0);
    act[i] = i;
  }
  build_ctl(b, act, 0);
  XAC_CUDA(cudaMemcpyAsync(b->dD, b->hD.data(), n * sizeof(BatchDesign), cudaMemcpyHostToDevice, s));
  XAC_CUDA(cudaMemcpyAsync(b->dC, b->hC, sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
  BatchRun run{};
  run.max_steps = o->max_steps;
  run.stats_every = o->stats_every;
  run.tol_ke = o->tol_ke;
  run.tol_T = o->tol_T;
  run.spin_limit = 1ull << 27;  // about 10 s of polling before a wait reports XAC_ETIMEOUT
  run.constant_power = o->constant_power;
  run.target_power = o->target_power;
  long long done = 0;
  while (done < o->max_steps && !b->hC->all_done) {
    const long long left = o->max_steps - done;
    run.steps = (int)(left < b->steps_per_launch ? left : b->steps_per_launch);
    int r = batch_launch_any(b, run, s, true);
    if (r != XAC_OK) return r;
    XAC_CUDA(cudaMemcpyAsync(b->hC, b->dC, 32, cudaMemcpyDeviceToHost, s));  // barrier words, err, done, step
    XAC_CUDA(cudaStreamSynchronize(s));
    if (b->hC->err) {
      set_error("xac_batch_run: a grid-barrier wait gave up (device status %d)", b->hC->err);
      return XAC_ETIMEOUT;
    }
    done = b->hC->step;
  }
  XAC_CUDA(cudaMemcpyAsync(b->hD.data(), b->dD, n * sizeof(BatchDesign), cudaMemcpyDeviceToHost, s));
  std::vector<float> u_fin(n);
  for (int i = 0; i < n; ++i)  // the inlet velocities the pump left (one small copy per design)
    XAC_CUDA(cudaMemcpyAsync(&u_fin[i], b->lats[i]->impl.u_in, sizeof(float), cudaMemcpyDeviceToHost, s));
  XAC_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < n; ++i) finish_design(b, i, b->hD[i].active ? done : b->hD[i].steps, u_fin[i], o, res[i]);
  return XAC_OK;
}

int xac_batch_launch_counts(const xac_batch* b, long long* graph_launches, long long* direct_launches) {
  XAC_REQUIRE(b && graph_launches && direct_launches, "xac_batch_launch_counts: null pointer");
  *graph_launches = b->graph_launches;
  *direct_launches = b->direct_launches;
  return XAC_OK;
}

int xac_batch_open(int precision, xac_batch** out) {
  XAC_REQUIRE(out, "xac_batch_open: null pointer");
  XAC_REQUIRE(precision == XAC_FP32 || precision == XAC_FP16 || precision == XAC_BF16 || precision == XAC_FP32_T16,
              "xac_batch_open: unknown precision %d", precision);
  *out = nullptr;
  xac_batch* b = new (std::nothrow) xac_batch();
  if (!b) {
    set_error("xac_batch_open: host allocation failed");
    return XAC_ENOMEM;
  }
  b->open = true;
  b->precision = precision;
  b->hD.assign(kMaxBatch, BatchDesign{});
  int r = XAC_OK;
  if ((r = dmalloc(&b->dD, (size_t)kMaxBatch, "alloc batch designs")) != XAC_OK ||
      (r = dmalloc(&b->dC, 1, "alloc batch control")) != XAC_OK) {
    delete b;
    return r;
  }
  if (cudaMallocHost(&b->hC, sizeof(BatchCtl)) != cudaSuccess) {
    delete b;
    set_error("xac_batch_open: pinned allocation failed");
    return XAC_ENOMEM;
  }
  *out = b;
  return XAC_OK;
}

int xac_batch_admit(xac_batch* b, const xac_desc* desc, int* slot, void* stream) {
  XAC_REQUIRE(b && desc && slot, "xac_batch_admit: null pointer");
  XAC_REQUIRE(b->open, "xac_batch_admit: not an open batch (create it with xac_batch_open)");
  XAC_REQUIRE(desc->precision == b->precision, "xac_batch_admit: design precision %d differs from the batch's %d",
              desc->precision, b->precision);
  int k = 0;
  while (k < (int)b->lats.size() && b->state[k] != xac_batch::kFree) ++k;
  XAC_REQUIRE(k < kMaxBatch, "xac_batch_admit: all %d slots hold designs (release finished ones first)", kMaxBatch);
  xac_lattice* l = nullptr;
  int r = xac_lattice_create(desc, &l, stream);
  if (r != XAC_OK) return r;
  if (k == (int)b->lats.size()) {
    b->lats.push_back(nullptr);
    b->state.push_back(xac_batch::kFree);
    b->gpu_s.push_back(0.0);
  }
  b->lats[k] = l;
  b->state[k] = xac_batch::kPending;
  b->gpu_s[k] = 0.0;
  *slot = k;
  return XAC_OK;
}

int xac_batch_release(xac_batch* b, int slot) {
  XAC_REQUIRE(b, "xac_batch_release: null batch");
  XAC_REQUIRE(b->open, "xac_batch_release: not an open batch");
  XAC_REQUIRE(slot >= 0 && slot < (int)b->lats.size() && b->state[slot] != xac_batch::kFree,
              "xac_batch_release: slot %d holds no design", slot);
  XAC_REQUIRE(b->state[slot] != xac_batch::kActive, "xac_batch_release: design %d is still running", slot);
  xac_lattice_destroy(b->lats[slot]);
  b->lats[slot] = nullptr;
  b->state[slot] = xac_batch::kFree;
  return XAC_OK;
}

int xac_batch_advance(xac_batch* b, const xac_run_opts* o, long long steps, int* n_finished, int* slots,
                      xac_run_result* results, double* gpu_seconds, void* stream) {
  XAC_REQUIRE(b && o && n_finished && slots && results && gpu_seconds, "xac_batch_advance: null pointer");
  XAC_REQUIRE(b->open, "xac_batch_advance: not an open batch (create it with xac_batch_open)");
  XAC_REQUIRE(o->stats_every > 0 && o->max_steps > 0 && steps >= 0, "xac_batch_advance: bad options");
  cudaStream_t s = as_stream(stream);
  *n_finished = 0;
  BatchRun run{};
  run.max_steps = o->max_steps;
  run.stats_every = o->stats_every;
  run.tol_ke = o->tol_ke;
  run.tol_T = o->tol_T;
  run.spin_limit = 1ull << 27;
  run.constant_power = o->constant_power;
  run.target_power = o->target_power;
  const int nslots = (int)b->lats.size();
  long long left = steps;
  while (left > 0) {
    // waiting designs join on a stats boundary
    const bool boundary = b->gstep % o->stats_every == 0;
    bool waiting = false;
    std::vector<int> act;
    for (int k = 0; k < nslots; ++k) {
      if (b->state[k] == xac_batch::kPending) {
        if (boundary) {
          LatticeImpl& L = b->lats[k]->impl;
          XAC_REQUIRE(L.step == 0 && L.own_pending, "xac_batch_advance: design %d is not at step 0", k);
          fill_design(b->hD[k], L, b->block, o->min_steps > 0 ? o->min_steps : L.reference_min_steps(o->max_steps),
                      b->gstep);
          b->state[k] = xac_batch::kActive;
          b->gpu_s[k] = 0.0;
        } else {
          waiting = true;
        }
      }
      if (b->state[k] == xac_batch::kActive) act.push_back(k);
    }
    if (act.empty()) {
      if (!waiting) break;
      b->gstep += o->stats_every - b->gstep % o->stats_every;  // nothing runs until the next boundary
      continue;
    }
    long long n = left < b->steps_per_launch ? left : b->steps_per_launch;
    for (int k : act) {  // no design passes its own step limit inside a launch
      const long long to_limit = b->hD[k].start + o->max_steps - b->gstep;
      if (to_limit < n) n = to_limit;
    }
    if (waiting && o->stats_every - b->gstep % o->stats_every < n) n = o->stats_every - b->gstep % o->stats_every;
    size_t rows = 0;
    for (int k : act) rows += b->hD[k].stat_tiles;
    if (rows > b->rows_cap) {
      b->drop_graphs();  // they hold the old rows pointer
      XAC_CUDA(cudaStreamSynchronize(s));
      cudaFree(b->drows);
      b->drows = nullptr;
      b->rows_cap = 0;
      int r = dmalloc(&b->drows, rows * kNStats + rows / 2 * kNStats, "alloc batch rows");
      if (r != XAC_OK) return r;
      b->rows_cap = rows + rows / 2;
    }
    build_ctl(b, act, b->gstep);
    XAC_CUDA(cudaMemcpyAsync(b->dD, b->hD.data(), nslots * sizeof(BatchDesign), cudaMemcpyHostToDevice, s));
    XAC_CUDA(cudaMemcpyAsync(b->dC, b->hC, sizeof(BatchCtl), cudaMemcpyHostToDevice, s));
    run.steps = (int)n;
    const auto t0 = std::chrono::steady_clock::now();
    int r = batch_launch_any(b, run, s, n == b->steps_per_launch);
    if (r != XAC_OK) return r;
    XAC_CUDA(cudaMemcpyAsync(b->hC, b->dC, 32, cudaMemcpyDeviceToHost, s));
    XAC_CUDA(cudaMemcpyAsync(b->hD.data(), b->dD, nslots * sizeof(BatchDesign), cudaMemcpyDeviceToHost, s));
    XAC_CUDA(cudaStreamSynchronize(s));
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (b->hC->err) {
      set_error("xac_batch_advance: a grid-barrier wait gave up (device status %d)", b->hC->err);
      return XAC_ETIMEOUT;
    }
    const long long ran = b->hC->step - b->gstep;
    b->gstep = b->hC->step;
    left -= ran;
    // the launch's wall time, shared by the designs in proportion to their tiles
    double tiles = 0.0;
    for (int k : act) tiles += b->hD[k].tiles;
    for (int k : act) b->gpu_s[k] += dt * b->hD[k].tiles / tiles;
    for (int k : act) {
      const BatchDesign& d = b->hD[k];
      const long long own = b->gstep - d.start;
      if (d.active && own < o->max_steps) continue;
      float u_fin = 0.0f;
      XAC_CUDA(cudaMemcpy(&u_fin, b->lats[k]->impl.u_in, sizeof(float), cudaMemcpyDeviceToHost));
      const int m = (*n_finished)++;
      slots[m] = k;
      gpu_seconds[m] = b->gpu_s[k];
      finish_design(b, k, d.active ? own : d.steps, u_fin, o, results[m]);
      b->state[k] = xac_batch::kDone;
    }
    if (ran == 0 || *n_finished > 0) break;  // the caller may refill the finished designs' slots now
  }
  return XAC_OK;
}

// Device bytes a lattice of this descriptor allocates (populations, link words, fields, reduction rows).
int xac_lattice_footprint(const xac_desc* d, unsigned long long* bytes) {
  XAC_REQUIRE(d && bytes, "xac_lattice_footprint: null pointer");
  XAC_REQUIRE(d->nx >= 1 && d->ny >= 1 && d->nz >= 1, "xac_lattice_footprint: bad lattice size");
  const long long n = (long long)d->nx * d->ny * d->nz;
  const long long pitch = (d->nx + 31) / 32 * 32;
  const long long N = ((long long)d->ny * d->nz + 2LL * (d->ny + 2)) * kQ * pitch;
  // fluid populations of the non-solid cells (all cells when no mask is given)
  long long nonsolid = n;
  if (d->mask) {
    nonsolid = 0;
    for (long long c = 0; c < n; ++c) nonsolid += d->mask[c] != kSolid;
  }
  const long long NP = kQ * ((nonsolid + 31) / 32 * 32 + (nonsolid == 0 ? 32 : 0));
  const long long ftab = ((long long)d->ny * d->nz + 2LL * (d->ny + 1)) * (pitch / 32) * 8;
  const long long p_elem = (d->precision == XAC_FP32 || d->precision == XAC_FP32_T16) ? 4 : 2;
  const long long q_elem = d->precision == XAC_FP32 ? 4 : 2;
  const long long metric_rows = (long long)reduction_blocks(n) * kNMetrics, stat_rows = stats_tiles(n) * kNStats;
  *bytes = (unsigned long long)(2 * NP * p_elem + 2 * N * q_elem + ftab + n * (1 + 4 + 4 + 5 * 4) +
                                8 * (metric_rows > stat_rows ? metric_rows : stat_rows) + 64 * 8 + 64);
  return XAC_OK;
}

}  // extern "C"
