// xac_stats_fields_noalloc: the deterministic FP64 stats of caller fields without any memory allocation.
//
// xac_stats_fields allocates its reduction partials, its device result and a pinned host buffer on every call.
// Some callers cannot allocate: code that runs while a CUDA stream is being captured (an allocation there is
// illegal or lands in the captured graph), code running under a strict memory-pool or memory-budget policy, or
// a host that has handed every free byte of the device to its own allocator. This entry point takes its
// scratch from a fixed array in the library's device image instead, and writes its result to a device buffer
// the caller provides, so it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits and rules, also stated in include/xac.h:
//   * at most kNoAllocMaxCells = 2,097,152 cells per call; larger lattices are rejected with XAC_EINVAL;
//   * the scratch (2,048 x 17 doubles, 278 KB) lives in every GPU that loads the library, until exit;
//   * every call on a device shares that one array: calls whose GPU work overlaps (other streams, other host
//     threads) race on it; each call rewrites all the partial rows it reads, so nothing needs clearing;
//   * the first call on each device resolves the array's device address (cudaGetSymbolAddress, with that device
//     current); make that first call before any stream capture.
#include <cstdio>
#include <mutex>

#include "reductions.cuh"

namespace xac {
namespace {

constexpr long long kNoAllocMaxCells = 1LL << 21;
constexpr int kNoAllocMaxTiles = (int)((kNoAllocMaxCells + kStatsTile - 1) / kStatsTile);
constexpr int kMaxDevices = 64;

// Partial rows of the stats reduction, one per 1024-cell tile. In host code this name is only a handle for
// cudaGetSymbolAddress: kernels receive the device address returned by it.
static __device__ __align__(256) double g_noalloc_rows[kNoAllocMaxTiles * kNStats];

double* g_rows_addr[kMaxDevices] = {};
std::mutex g_rows_mu;

// Device address of g_noalloc_rows on the current device, resolved once per device.
int scratch_rows(double** out) {
  int dev = 0;
  XAC_CUDA(cudaGetDevice(&dev));
  XAC_REQUIRE(dev >= 0 && dev < kMaxDevices, "xac_stats_fields_noalloc: device ordinal %d not supported", dev);
  std::lock_guard<std::mutex> g(g_rows_mu);
  if (!g_rows_addr[dev]) {
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_rows);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_rows)");
    g_rows_addr[dev] = p;
  }
  *out = g_rows_addr[dev];
  return XAC_OK;
}

__global__ void __launch_bounds__(256) noalloc_rows_kernel(FieldView v, ReduceSpec<kNStats> spec,
                                                           double* __restrict__ rows) {
  stats_tile_row(v, blockIdx.x, spec, rows + (long long)blockIdx.x * kNStats);
}

}  // namespace
}  // namespace xac

using namespace xac;

extern "C" int xac_stats_fields_noalloc(const float* rho, const float* u, const float* T, const int32_t* mask,
                                        int nx, int ny, int nz, double* out_dev, void* stream) {
  XAC_REQUIRE(rho && u && T && mask && out_dev, "xac_stats_fields_noalloc: null pointer");
  XAC_REQUIRE(nx > 0 && ny > 0 && nz > 0, "xac_stats_fields_noalloc: bad dimensions");
  const long long n = (long long)nx * ny * nz;
  XAC_REQUIRE(n <= kNoAllocMaxCells,
              "xac_stats_fields_noalloc: %lld cells exceed the fixed scratch of %lld cells; use xac_stats_fields",
              n, kNoAllocMaxCells);
  double* rows = nullptr;
  const int r = scratch_rows(&rows);
  if (r != XAC_OK) return r;
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
  const auto spec = stats_spec();
  const int ntiles = (int)stats_tiles(n);
  cudaStream_t s = as_stream(stream);
  noalloc_rows_kernel<<<ntiles, kStatsBlock, 0, s>>>(v, spec, rows);
  combine_rows_kernel<kNStats><<<1, 32 * kNStats, 0, s>>>(rows, ntiles, spec, out_dev);
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}
