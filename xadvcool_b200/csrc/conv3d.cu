// 3-D convolutions of the warm-start surrogate as BF16 tensor-core implicit GEMMs with FP32 accumulation.
//
// Layout: activations channels-last, x fastest: act[n][z][y][x][c] (BF16); weights w[tap][co][ci] (BF16,
// ci fastest), tap = (dz+1)*9 + (dy+1)*3 + (dx+1) for a 3x3x3 kernel (tap 0 only for 1x1x1); zero padding.
//
//   forward   out[v][co] = act( bias[co] + sum_{tap,ci} w[tap][co][ci] * in[v + off(tap)][ci] )
//             GEMM M = voxels, N = Co, K = taps * Ci, on tcgen05 (128 voxels x Co per CTA, accumulator in TMEM).
//   data grad the forward kernel applied to d_out with the flipped, transposed weights
//             w'[26 - tap][ci][co] = w[tap][co][ci] (the adjoint of a zero-padded convolution).
//   weight grad dw[tap][co][ci] = sum_v d_out[v][co] * in[v + off(tap)][ci]
//             GEMM M = taps * Co, N = Ci, K = voxels on tcgen05, split over voxel chunks; partials reduced in a
//             fixed order.
//
// Ci and Co must be multiples of 16 (the model pads its 3 input channels and 5 output channels to 16).
#include <cuda_bf16.h>

#include <cstdint>

#include "xac_internal.cuh"

namespace xac {
namespace {

struct ConvShape {
  int N, D, H, W;  // batch, z, y, x
  int Ci, Co;
  int ksize;  // 1 or 3
};



__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// voxel index -> (n, z, y, x); returns the neighbour voxel index for tap offsets, or -1 outside the volume
struct VoxelCoord {
  int n, z, y, x;
};
// volumes stay below 2^31 voxels (checked on the host): 32-bit decoding
__device__ __forceinline__ VoxelCoord decode(long long v, const ConvShape& s) {
  VoxelCoord c;
  const unsigned u = (unsigned)v, W = (unsigned)s.W, H = (unsigned)s.H, D = (unsigned)s.D;
  unsigned t = u / W;
  c.x = (int)(u - t * W);
  unsigned t2 = t / H;
  c.y = (int)(t - t2 * H);
  t = t2 / D;
  c.z = (int)(t2 - t * D);
  c.n = (int)t;
  return c;
}
__device__ __forceinline__ long long neighbour(const VoxelCoord& c, int dz, int dy, int dx, const ConvShape& s) {
  const int z = c.z + dz, y = c.y + dy, x = c.x + dx;
  if (z < 0 || z >= s.D || y < 0 || y >= s.H || x < 0 || x >= s.W) return -1;
  return (((long long)c.n * s.D + z) * s.H + y) * s.W + x;
}

// ---- forward / data grad on the 5th-generation tensor cores (tcgen05) ------------------------------------
// One CTA of 128 threads computes a 128-voxel x Co tile: D[128][Co] (FP32, in tensor memory) =
// sum over K = taps x Ci of A[voxel][k] * B[co][k]. K is walked in stages of one tap x BK channels:
//   * all 128 threads gather the stage's operands into shared memory with 16-byte cp.async copies (zero-filled
//     where the neighbour is outside the volume), A row r = voxel m0 + r, B row n = output channel n;
//   * one thread issues the stage's BK/16 tcgen05.mma (kind::f16, BF16 in, FP32 accumulate) and a
//     tcgen05.commit that frees the stage when those MMAs have read it;
//   * a ring of kStages stages overlaps the gathers with the MMAs (mbarriers "full" and "empty").
// Shared-memory operand layout (K-major, no swizzle): 16-byte chunks of 8 channels, [BK/8][rows][8], so a core
// matrix (8 rows x 16 bytes) is 128 contiguous bytes, 8-row groups are 128 bytes apart (stride byte offset) and
// the two 8-channel halves of one K = 16 MMA step are rows*16 bytes apart (leading byte offset).
// Epilogue: warp w reads tensor-memory lanes 32w..32w+31 (its voxels) 16 columns at a time, adds the bias,
// applies GELU if asked, and stores BF16 or FP32.
// Every wait is bounded: a wait that runs out sets g_conv_status, the CTA stops issuing work, waits (bounded) for
// the MMAs it issued, frees its tensor memory and returns.
constexpr int kTcM = 128;
constexpr int kTcStages = 4;
constexpr uint32_t kTcSpin = 1u << 22;
__device__ unsigned int g_conv_status;  // bit 0: a wait ran out

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = kTcSpin) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicOr(&g_conv_status, 1u);
  return false;
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle (layout type 0), descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major, N = n, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcConv {
  int BK;          // channels per stage (16..64, divides Ci)
  int kt;          // stages of K: taps * Ci / BK
  uint32_t ncols;  // tensor-memory columns allocated (power of two >= max(32, Co))
};

__global__ void __launch_bounds__(128, 1) conv_fwd_tc_kernel(const __nv_bfloat16* __restrict__ in,
                                                             const __nv_bfloat16* __restrict__ w,
                                                             const float* __restrict__ bias, ConvShape s, int act,
                                                             TcConv t, __nv_bfloat16* __restrict__ out_bf16,
                                                             float* __restrict__ out_f32) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[2 * kTcStages + 1];  // full[s], empty[s], done
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Co = s.Co, BK = t.BK, chunks = BK >> 3;
  const long long V = (long long)s.N * s.D * s.H * s.W;
  const long long m0 = (long long)blockIdx.x * kTcM;
  const uint32_t a_bytes = kTcM * BK * 2, b_bytes = (uint32_t)Co * BK * 2, stage_bytes = a_bytes + b_bytes;
  const uint32_t sbase = smem_addr(smem);
  const uint32_t bar0 = smem_addr(bars);
  auto full = [&](int st) { return bar0 + 8u * st; };
  auto empty = [&](int st) { return bar0 + 8u * (kTcStages + st); };
  const uint32_t done_bar = bar0 + 8u * (2 * kTcStages);

  if (tid == 0) {
    for (int st = 0; st < kTcStages; ++st) {
      mbar_init(full(st), 128);
      mbar_init(empty(st), 1);
    }
    mbar_init(done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(t.ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  // this thread's A row: voxel m0 + tid
  const long long v = m0 + tid;
  const bool vrow = v < V;
  const VoxelCoord vc = decode(vrow ? v : 0, s);
  const int ci_chunks = s.Ci / BK;
  const uint32_t idesc = tc_idesc(Co);

  auto load_stage = [&](int k, int st) {
    const int tap = k / ci_chunks, kc = k - tap * ci_chunks;
    const int dz = s.ksize == 3 ? tap / 9 - 1 : 0, dy = s.ksize == 3 ? (tap / 3) % 3 - 1 : 0,
              dx = s.ksize == 3 ? tap % 3 - 1 : 0;
    const long long nb = vrow ? neighbour(vc, dz, dy, dx, s) : -1;
    const uint32_t a_st = sbase + (uint32_t)st * stage_bytes, b_st = a_st + a_bytes;
    const __nv_bfloat16* asrc = nb >= 0 ? in + nb * s.Ci + kc * BK : in;
    for (int j = 0; j < chunks; ++j)
      cp_async16(a_st + (uint32_t)(j * kTcM + tid) * 16u, asrc + (nb >= 0 ? j * 8 : 0), nb >= 0 ? 16u : 0u);
    const __nv_bfloat16* wt = w + ((long long)tap * Co) * s.Ci + kc * BK;
    for (int e = tid; e < Co * chunks; e += 128) {
      const int n = e / chunks, j = e - n * chunks;
      cp_async16(b_st + (uint32_t)(j * Co + n) * 16u, wt + (long long)n * s.Ci + j * 8, 16u);
    }
  };
  auto mma_stage = [&](int k, int st) {
    const uint32_t a_st = sbase + (uint32_t)st * stage_bytes, b_st = a_st + a_bytes;
    for (int q = 0; q < BK / 16; ++q) {
      const uint64_t ad = smem_desc(a_st + (uint32_t)(2 * q) * kTcM * 16u, kTcM * 16u, 128u);
      const uint64_t bd = smem_desc(b_st + (uint32_t)(2 * q) * Co * 16u, (uint32_t)Co * 16u, 128u);
      tc_mma(tmem, ad, bd, idesc, (k > 0 || q > 0) ? 1u : 0u);
    }
    tc_commit(empty(st));
  };

  const int KT = t.kt;
  for (int k = 0; k < KT + kTcStages - 1; ++k) {
    if (k < KT) {
      const int st = k % kTcStages;
      if (k >= kTcStages && !mbar_wait(empty(st), ((k / kTcStages) - 1) & 1)) abort_flag = 1;
      if (abort_flag) break;
      load_stage(k, st);
    }
    cp_async_commit();
    const int kc = k - (kTcStages - 1);  // the stage whose copies this thread now completes
    if (kc >= 0) {
      cp_async_wait<kTcStages - 1>();
      fence_proxy_async();
      mbar_arrive(full(kc % kTcStages));
      if (warp == 0) {  // the whole warp waits, lane 0 issues
        if (mbar_wait(full(kc % kTcStages), (kc / kTcStages) & 1)) {
          tc_fence_after();
          if (lane == 0) mma_stage(kc, kc % kTcStages);
        } else {
          abort_flag = 1;
        }
        __syncwarp();
      }
    }
    if (abort_flag) break;
  }
  cp_async_wait<0>();
  // the last commit (or, after an abort, a fresh one) arrives on done_bar when every issued MMA has finished
  if (tid == 0) tc_commit(done_bar);
  const int drained = mbar_wait(done_bar, 0) ? 1 : 0;
  const bool ok = __syncthreads_and(drained) && !abort_flag;  // uniform: every thread has left the loop
  tc_fence_after();
  if (ok) {
    const long long vr = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < Co; c0 += 16) {
      float x[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, x);
      if (vr < V) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          float y = x[i] + (bias ? __ldg(bias + c0 + i) : 0.0f);
          x[i] = act == 1 ? gelu(y) : y;
        }
        if (out_bf16) {
          uint4 pk[2];
          uint32_t* pw = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            __nv_bfloat162 b2 = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
            pw[i] = *reinterpret_cast<uint32_t*>(&b2);
          }
          uint4* dst = reinterpret_cast<uint4*>(out_bf16 + vr * Co + c0);
          dst[0] = pk[0];
          dst[1] = pk[1];
        } else {
          float4* dst = reinterpret_cast<float4*>(out_f32 + vr * Co + c0);
#pragma unroll
          for (int i = 0; i < 4; ++i) dst[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(t.ncols));
  }
}

// ---- weight grad on the tensor cores (tcgen05) --------------------------------------------------------
// With u = v + off(tap): dw[tap][co][ci] = sum_u d_out[u - off(tap)][co] * in[u][ci], a GEMM with rows
// m = tap * Co + co (M = taps * Co), columns ci (N = Ci) and K = voxels. A CTA computes 128 rows x Ci columns in
// tensor memory over one chunk of kWgKC voxels (split K), 64 voxels per stage:
//   A (MN-major): A[m][u] = d_out[u - off(tap)][co], zero where u - off(tap) leaves the volume;
//   B (MN-major): B[u][ci] = in[u][ci].
// Shared-memory layout of both: core matrices of 8 M (or N) values x 8 voxels, 128 contiguous bytes each (one
// voxel's 8 values per 16-byte row); M/N groups 128 bytes apart (stride byte offset), 8-voxel groups one group
// row apart (leading byte offset). The chunk's partial goes to partial[chunk][m][ci]; the chunks are added in
// order by wgrad_reduce_kernel (deterministic). Bounded waits as in the forward kernel.
constexpr int kWgKC = 4096;  // voxels per CTA
constexpr int kWgBK = 64;    // voxels per stage

__global__ void __launch_bounds__(128, 1) conv_wgrad_tc_kernel(const __nv_bfloat16* __restrict__ in,
                                                               const __nv_bfloat16* __restrict__ dout, ConvShape s,
                                                               uint32_t ncols, float* __restrict__ partial) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[2 * kTcStages + 1];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Ci = s.Ci, Co = s.Co, taps = s.ksize == 3 ? 27 : 1, Mtot = taps * Co;
  const long long V = (long long)s.N * s.D * s.H * s.W;
  const int m0 = blockIdx.x * kTcM;
  const long long u_begin = (long long)blockIdx.y * kWgKC;
  const long long u_left = V - u_begin;
  const int KT = (int)(((u_left < kWgKC ? u_left : kWgKC) + kWgBK - 1) / kWgBK);
  const uint32_t a_bytes = kTcM * kWgBK * 2, b_bytes = (uint32_t)kWgBK * Ci * 2, stage_bytes = a_bytes + b_bytes;
  const uint32_t a_lbo = (kTcM / 8) * 128u, b_lbo = (uint32_t)(Ci / 8) * 128u;
  const uint32_t sbase = smem_addr(smem);
  const uint32_t bar0 = smem_addr(bars);
  auto full = [&](int st) { return bar0 + 8u * st; };
  auto empty = [&](int st) { return bar0 + 8u * (kTcStages + st); };
  const uint32_t done_bar = bar0 + 8u * (2 * kTcStages);
  if (tid == 0) {
    for (int st = 0; st < kTcStages; ++st) {
      mbar_init(full(st), 128);
      mbar_init(empty(st), 1);
    }
    mbar_init(done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = tc_idesc(Ci) | (1u << 15) | (1u << 16);  // A and B MN-major
  const int ul = tid & 63, g0 = tid >> 6;  // this thread's voxel in a stage, and first M / N group
  const int kg = ul >> 3, krow = ul & 7;

  auto load_stage = [&](int k, int st) {
    const uint32_t a_st = sbase + (uint32_t)st * stage_bytes, b_st = a_st + a_bytes;
    const long long u = u_begin + (long long)k * kWgBK + ul;
    const bool uok = u < V && k * kWgBK + ul < kWgKC;
    const VoxelCoord cu = decode(uok ? u : 0, s);
    for (int j = 0; j < 8; ++j) {
      const int mg = g0 + 2 * j, m = m0 + mg * 8;
      long long src = -1;
      int co = 0;
      if (uok && m < Mtot) {
        const int tap = m / Co;
        co = m - tap * Co;
        const int dz = s.ksize == 3 ? tap / 9 - 1 : 0, dy = s.ksize == 3 ? (tap / 3) % 3 - 1 : 0,
                  dx = s.ksize == 3 ? tap % 3 - 1 : 0;
        src = neighbour(cu, -dz, -dy, -dx, s);
      }
      cp_async16(a_st + ((uint32_t)(kg * (kTcM / 8) + mg) * 8u + krow) * 16u,
                 src >= 0 ? (const void*)(dout + src * Co + co) : (const void*)dout, src >= 0 ? 16u : 0u);
    }
    for (int ng = g0; ng < Ci / 8; ng += 2)
      cp_async16(b_st + ((uint32_t)(kg * (Ci / 8) + ng) * 8u + krow) * 16u,
                 uok ? (const void*)(in + u * Ci + ng * 8) : (const void*)in, uok ? 16u : 0u);
  };
  auto mma_stage = [&](int k, int st) {
    const uint32_t a_st = sbase + (uint32_t)st * stage_bytes, b_st = a_st + a_bytes;
    for (int q = 0; q < kWgBK / 16; ++q) {
      const uint64_t ad = smem_desc(a_st + (uint32_t)(2 * q) * a_lbo, a_lbo, 128u);
      const uint64_t bd = smem_desc(b_st + (uint32_t)(2 * q) * b_lbo, b_lbo, 128u);
      tc_mma(tmem, ad, bd, idesc, (k > 0 || q > 0) ? 1u : 0u);
    }
    tc_commit(empty(st));
  };

  for (int k = 0; k < KT + kTcStages - 1; ++k) {
    if (k < KT) {
      const int st = k % kTcStages;
      if (k >= kTcStages && !mbar_wait(empty(st), ((k / kTcStages) - 1) & 1)) abort_flag = 1;
      if (abort_flag) break;
      load_stage(k, st);
    }
    cp_async_commit();
    const int kc = k - (kTcStages - 1);
    if (kc >= 0) {
      cp_async_wait<kTcStages - 1>();
      fence_proxy_async();
      mbar_arrive(full(kc % kTcStages));
      if (warp == 0) {
        if (mbar_wait(full(kc % kTcStages), (kc / kTcStages) & 1)) {
          tc_fence_after();
          if (lane == 0) mma_stage(kc, kc % kTcStages);
        } else {
          abort_flag = 1;
        }
        __syncwarp();
      }
    }
    if (abort_flag) break;
  }
  cp_async_wait<0>();
  if (tid == 0) tc_commit(done_bar);
  const int drained = mbar_wait(done_bar, 0) ? 1 : 0;
  const bool ok = __syncthreads_and(drained) && !abort_flag;
  tc_fence_after();
  if (ok) {
    const int m = m0 + warp * 32 + lane;
    float* dst = partial + ((long long)blockIdx.y * Mtot + m) * Ci;
    for (int c0 = 0; c0 < Ci; c0 += 16) {
      float x[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, x);
      if (m < Mtot) {
        float4* d4 = reinterpret_cast<float4*>(dst + c0);
#pragma unroll
        for (int i = 0; i < 4; ++i) d4[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
}

// dw[t][co][ci] = sum over chunks in order; db[co] = sum of d_out over voxels (block per co, fixed order)
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int nchunks, long long per_chunk,
                                    float* __restrict__ dw) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= per_chunk) return;
  float s = 0.0f;
  for (int k = 0; k < nchunks; ++k) s += partial[(long long)k * per_chunk + e];
  dw[e] = s;
}

// db[co] = sum over voxels of d_out: 256 blocks stride over voxels (consecutive threads read consecutive channels),
// each block reduces its channel sums in a fixed order into one partial row, a second pass adds the rows in order
constexpr int kBiasBlocks = 256;
__global__ void bias_grad_partial_kernel(const __nv_bfloat16* __restrict__ dout, long long V, int Co,
                                         float* __restrict__ partial) {
  __shared__ float part[256];
  const int c = threadIdx.x % Co, lanes = blockDim.x / Co, g = threadIdx.x / Co;
  float s = 0.0f;
  if (g < lanes)
    for (long long v = (long long)blockIdx.x * lanes + g; v < V; v += (long long)gridDim.x * lanes)
      s += __bfloat162float(dout[v * Co + c]);
  part[threadIdx.x] = s;
  __syncthreads();
  if ((int)threadIdx.x < Co) {
    float t = 0.0f;
    for (int k = 0; k < lanes; ++k) t += part[k * Co + threadIdx.x];
    partial[(long long)blockIdx.x * Co + threadIdx.x] = t;
  }
}

__global__ void bias_grad_final_kernel(const float* __restrict__ partial, int nblocks, int Co, float* __restrict__ db) {
  const int c = threadIdx.x;
  if (c >= Co) return;
  float t = 0.0f;
  for (int b = 0; b < nblocks; ++b) t += partial[(long long)b * Co + c];
  db[c] = t;
}

int check_shape(const ConvShape& s) {
  XAC_REQUIRE(s.N > 0 && s.D > 0 && s.H > 0 && s.W > 0, "conv3d: bad volume");
  XAC_REQUIRE((long long)s.N * s.D * s.H * s.W < (1LL << 31), "conv3d: volume must stay below 2^31 voxels");
  XAC_REQUIRE(s.Ci % 16 == 0 && s.Co % 16 == 0 && s.Ci <= 256 && s.Co <= 256 && s.Ci >= 16 && s.Co >= 16,
              "conv3d: channels must be multiples of 16 with Ci, Co <= 256 (got %d -> %d)", s.Ci, s.Co);
  XAC_REQUIRE(s.ksize == 1 || s.ksize == 3, "conv3d: kernel size must be 1 or 3");
  return XAC_OK;
}

}  // namespace
}  // namespace xac

using namespace xac;

extern "C" {

int xac_conv3d_forward(const void* in, int N, int D, int H, int W, int Ci, const void* weight, const float* bias,
                       int Co, int ksize, int activation, void* out_bf16, float* out_f32, void* stream) {
  ConvShape s{N, D, H, W, Ci, Co, ksize};
  int r = check_shape(s);
  if (r != XAC_OK) return r;
  XAC_REQUIRE(in && weight && (out_bf16 || out_f32) && !(out_bf16 && out_f32),
              "xac_conv3d_forward: give exactly one output");
  XAC_REQUIRE(activation == 0 || activation == 1, "xac_conv3d_forward: activation must be 0 (none) or 1 (GELU)");
  const long long V = (long long)N * D * H * W;
  TcConv t;
  t.BK = 64;
  while (Ci % t.BK != 0) t.BK -= 16;  // 64, 48, 32 or 16
  t.kt = (ksize == 3 ? 27 : 1) * (Ci / t.BK);
  t.ncols = 32;
  while ((int)t.ncols < Co) t.ncols <<= 1;
  const size_t smem = (size_t)kTcStages * (kTcM + Co) * t.BK * 2;
  static bool attr_set = false;  // the attribute is per device function; set once per process
  if (!attr_set) {
    XAC_CUDA(cudaFuncSetAttribute(conv_fwd_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((size_t)kTcStages * (kTcM + 256) * 64 * 2)));
    attr_set = true;
  }
  const unsigned grid = (unsigned)((V + kTcM - 1) / kTcM);
  conv_fwd_tc_kernel<<<grid, 128, smem, as_stream(stream)>>>((const __nv_bfloat16*)in,
                                                             (const __nv_bfloat16*)weight, bias, s, activation, t,
                                                             (__nv_bfloat16*)out_bf16, out_f32);
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}

// partial must hold ceil(V / 2048) * taps * Co * Ci floats; dw receives taps * Co * Ci floats, db Co floats
int xac_conv3d_weight_grad(const void* in, int N, int D, int H, int W, int Ci, const void* dout, int Co, int ksize,
                           float* partial, float* dw, float* db, void* stream) {
  ConvShape s{N, D, H, W, Ci, Co, ksize};
  int r = check_shape(s);
  if (r != XAC_OK) return r;
  XAC_REQUIRE(in && dout && partial && dw, "xac_conv3d_weight_grad: null pointer");
  const long long V = (long long)N * D * H * W;
  const int taps = ksize == 3 ? 27 : 1;
  const int nchunks = (int)((V + kWgKC - 1) / kWgKC);
  uint32_t ncols = 32;
  while ((int)ncols < Ci) ncols <<= 1;
  static bool attr_set = false;
  if (!attr_set) {
    XAC_CUDA(cudaFuncSetAttribute(conv_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((size_t)kTcStages * (kTcM * kWgBK + kWgBK * 256) * 2)));
    attr_set = true;
  }
  const dim3 grid((unsigned)((taps * Co + kTcM - 1) / kTcM), (unsigned)nchunks);
  const size_t smem = (size_t)kTcStages * (kTcM * kWgBK + kWgBK * Ci) * 2;
  cudaStream_t st = as_stream(stream);
  conv_wgrad_tc_kernel<<<grid, 128, smem, st>>>((const __nv_bfloat16*)in, (const __nv_bfloat16*)dout, s, ncols,
                                                 partial);
  const long long per_chunk = (long long)taps * Co * Ci;
  wgrad_reduce_kernel<<<(unsigned)((per_chunk + 255) / 256), 256, 0, st>>>(partial, nchunks, per_chunk, dw);
  if (db) {
    // the bias partials reuse the head of `partial` after the weight reduction has consumed it
    bias_grad_partial_kernel<<<kBiasBlocks, 256, 0, st>>>((const __nv_bfloat16*)dout, V, Co, partial);
    bias_grad_final_kernel<<<1, Co, 0, st>>>(partial, kBiasBlocks, Co, db);
  }
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}

// Test-only: the convolution kernels' mbarrier wait on a barrier that nothing completes must give up after
// `limit` polls and set g_conv_status (read and cleared by xac_conv3d_status).
static __global__ void test_conv_wait_timeout_kernel(uint32_t limit) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = smem_addr(&bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_wait(b, 0, limit);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(b) : "memory");
  }
}

int xac_test_conv_wait_timeout(unsigned limit, void* stream) {
  XAC_REQUIRE(limit > 0 && limit <= (1u << 20), "xac_test_conv_wait_timeout: limit %u out of (0, 2^20]", limit);
  cudaStream_t s = as_stream(stream);
  test_conv_wait_timeout_kernel<<<1, 32, 0, s>>>(limit);
  XAC_CUDA(cudaGetLastError());
  XAC_CUDA(cudaStreamSynchronize(s));
  return XAC_OK;
}

int xac_conv3d_status(int* flags) {
  XAC_REQUIRE(flags, "xac_conv3d_status: null pointer");
  unsigned int v = 0, zero = 0;
  XAC_CUDA(cudaMemcpyFromSymbol(&v, g_conv_status, sizeof(v)));
  XAC_CUDA(cudaMemcpyToSymbol(g_conv_status, &zero, sizeof(zero)));
  *flags = (int)v;
  return XAC_OK;
}

int xac_conv3d_partial_floats(int N, int D, int H, int W, int Ci, int Co, int ksize, long long* count) {
  XAC_REQUIRE(count, "xac_conv3d_partial_floats: null pointer");
  const long long V = (long long)N * D * H * W;
  const long long w = ((V + kWgKC - 1) / kWgKC) * (ksize == 3 ? 27 : 1) * (long long)Co * Ci;
  const long long b = (long long)kBiasBlocks * Co;
  *count = w > b ? w : b;
  return XAC_OK;
}

}  // extern "C"
