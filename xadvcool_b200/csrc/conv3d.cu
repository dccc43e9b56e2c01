// 3-D convolutions of the warm-start surrogate as BF16 tensor-core implicit GEMMs with FP32 accumulation.
//
// Layout: activations channels-last, x fastest: act[n][z][y][x][c] (BF16); weights w[tap][co][ci] (BF16,
// ci fastest), tap = (dz+1)*9 + (dy+1)*3 + (dx+1) for a 3x3x3 kernel (tap 0 only for 1x1x1); zero padding.
//
//   forward   out[v][co] = act( bias[co] + sum_{tap,ci} w[tap][co][ci] * in[v + off(tap)][ci] )
//             GEMM M = voxels, N = Co, K = taps * Ci; each warp owns 16 voxels x all Co.
//   data grad the forward kernel applied to d_out with the flipped, transposed weights
//             w'[26 - tap][ci][co] = w[tap][co][ci] (the adjoint of a zero-padded convolution).
//   weight grad dw[tap][co][ci] = sum_v d_out[v][co] * in[v + off(tap)][ci]
//             GEMM M = Co, N = Ci, K = voxels, split over voxel chunks; partials reduced in a fixed order.
//
// Tensor-core instruction: mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32. Ci and Co must be multiples of
// 16 (the model pads its 4 input channels and 5 output channels to 16).
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

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) {
  return __ldg(reinterpret_cast<const unsigned int*>(p));
}

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

// ---- forward / data grad -----------------------------------------------------------------------------
// 4 warps per block, 16 voxels per warp, NT n-tiles of 8 output channels per warp: block (x, y) computes channels
// [y*NT*8, (y+1)*NT*8) of voxels [64x, 64x + 64).
template <int NT>
__global__ void __launch_bounds__(128) conv_fwd_kernel(const __nv_bfloat16* __restrict__ in,
                                                       const __nv_bfloat16* __restrict__ w,
                                                       const float* __restrict__ bias, ConvShape s, int act,
                                                       __nv_bfloat16* __restrict__ out_bf16,
                                                       float* __restrict__ out_f32) {
  const long long V = (long long)s.N * s.D * s.H * s.W;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long v0 = ((long long)blockIdx.x * 4 + warp) * 16;
  if (v0 >= V) return;
  const int cobase = blockIdx.y * NT * 8;
  const int r = lane >> 2, cq = (lane & 3) * 2;
  // the two voxels (rows r and r+8) this lane loads A fragments for
  const long long va = v0 + r, vb = v0 + r + 8;
  const VoxelCoord ca = decode(va < V ? va : 0, s), cb = decode(vb < V ? vb : 0, s);
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
  const int taps = s.ksize == 3 ? 27 : 1;
  for (int tap = 0; tap < taps; ++tap) {
    const int dz = s.ksize == 3 ? tap / 9 - 1 : 0, dy = s.ksize == 3 ? (tap / 3) % 3 - 1 : 0,
              dx = s.ksize == 3 ? tap % 3 - 1 : 0;
    const long long na = va < V ? neighbour(ca, dz, dy, dx, s) : -1;
    const long long nb = vb < V ? neighbour(cb, dz, dy, dx, s) : -1;
    const __nv_bfloat16* wt = w + (long long)tap * s.Co * s.Ci;
    for (int ci0 = 0; ci0 < s.Ci; ci0 += 16) {
      uint32_t a[4];
      a[0] = na >= 0 ? ld_pair(in + na * s.Ci + ci0 + cq) : 0u;
      a[1] = nb >= 0 ? ld_pair(in + nb * s.Ci + ci0 + cq) : 0u;
      a[2] = na >= 0 ? ld_pair(in + na * s.Ci + ci0 + cq + 8) : 0u;
      a[3] = nb >= 0 ? ld_pair(in + nb * s.Ci + ci0 + cq + 8) : 0u;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const __nv_bfloat16* wb = wt + (long long)(cobase + j * 8 + r) * s.Ci + ci0 + cq;
        const uint32_t b[2] = {ld_pair(wb), ld_pair(wb + 8)};
        mma_bf16_16816(acc[j], a, b);
      }
    }
  }
  // epilogue: rows r, r+8; columns j*8 + cq, +1
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int co = cobase + j * 8 + cq;
    const float b0 = bias ? bias[co] : 0.0f, b1 = bias ? bias[co + 1] : 0.0f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long v = h == 0 ? va : vb;
      if (v >= V) continue;
      float x0 = acc[j][2 * h] + b0, x1 = acc[j][2 * h + 1] + b1;
      if (act == 1) {
        x0 = gelu(x0);
        x1 = gelu(x1);
      }
      if (out_bf16) {
        __nv_bfloat162 pr = __floats2bfloat162_rn(x0, x1);
        *reinterpret_cast<__nv_bfloat162*>(out_bf16 + v * s.Co + co) = pr;
      } else {
        *reinterpret_cast<float2*>(out_f32 + v * s.Co + co) = make_float2(x0, x1);
      }
    }
  }
}

// ---- weight grad ------------------------------------------------------------------------------------
// Block: one tap, one 16 (co) x 16 (ci) tile, one chunk of voxels (the GEMM's K). 4 warps split the chunk's k16
// steps; their partials are added in warp order through shared memory. Output: partial[chunk][tap][co][ci].
constexpr int kWgChunk = 2048;
__global__ void __launch_bounds__(128) conv_wgrad_kernel(const __nv_bfloat16* __restrict__ in,
                                                         const __nv_bfloat16* __restrict__ dout, ConvShape s,
                                                         float* __restrict__ partial) {
  const long long V = (long long)s.N * s.D * s.H * s.W;
  const int tap = blockIdx.y, chunk = blockIdx.x;
  const int ci_tiles = s.Ci / 16;
  const int co0 = (blockIdx.z / ci_tiles) * 16, ci0 = (blockIdx.z % ci_tiles) * 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = lane >> 2, cq = (lane & 3) * 2;
  const int dz = s.ksize == 3 ? tap / 9 - 1 : 0, dy = s.ksize == 3 ? (tap / 3) % 3 - 1 : 0,
            dx = s.ksize == 3 ? tap % 3 - 1 : 0;
  float acc[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
  auto pack = [](float lo, float hi) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&p);
  };
  const long long vbeg = (long long)chunk * kWgChunk;
  for (long long k0 = vbeg + warp * 16; k0 < vbeg + kWgChunk && k0 < V; k0 += 64) {
    // A = d_out^T: rows co0 + r (+8), cols voxels k0 + cq (+1), +8 (+9)
    const long long vk[4] = {k0 + cq, k0 + cq + 1, k0 + cq + 8, k0 + cq + 9};
    float dv[2][4];
    long long nv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool ok = vk[q] < V;
      dv[0][q] = ok ? __bfloat162float(dout[vk[q] * s.Co + co0 + r]) : 0.0f;
      dv[1][q] = ok ? __bfloat162float(dout[vk[q] * s.Co + co0 + r + 8]) : 0.0f;
      nv[q] = ok ? neighbour(decode(vk[q], s), dz, dy, dx, s) : -1;
    }
    const uint32_t a[4] = {pack(dv[0][0], dv[0][1]), pack(dv[1][0], dv[1][1]), pack(dv[0][2], dv[0][3]),
                           pack(dv[1][2], dv[1][3])};
    // B = shifted input: rows voxels vk, cols ci0 + j*8 + r
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ci = ci0 + j * 8 + r;
      float bv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = nv[q] >= 0 ? __bfloat162float(in[nv[q] * s.Ci + ci]) : 0.0f;
      const uint32_t b[2] = {pack(bv[0], bv[1]), pack(bv[2], bv[3])};
      mma_bf16_16816(acc[j], a, b);
    }
  }
  __shared__ float red[4][16][16];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int ci = j * 8 + cq;
    red[warp][r][ci] = acc[j][0];
    red[warp][r][ci + 1] = acc[j][1];
    red[warp][r + 8][ci] = acc[j][2];
    red[warp][r + 8][ci + 1] = acc[j][3];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 256; e += blockDim.x) {
    const int row = e >> 4, col = e & 15;
    const float v = ((red[0][row][col] + red[1][row][col]) + red[2][row][col]) + red[3][row][col];
    partial[(((long long)chunk * gridDim.y + tap) * s.Co + co0 + row) * s.Ci + ci0 + col] = v;
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
  // output channels per block: the widest multiple of 16 up to 128 that divides Co
  int slice = 128;
  while (Co % slice != 0) slice -= 16;
  const dim3 grid((unsigned)((V + 63) / 64), (unsigned)(Co / slice));
  cudaStream_t st = as_stream(stream);
  const auto* x = (const __nv_bfloat16*)in;
  const auto* wt = (const __nv_bfloat16*)weight;
  auto* ob = (__nv_bfloat16*)out_bf16;
  switch (slice / 8) {
#define XAC_CO(NT) \
  case NT: conv_fwd_kernel<NT><<<grid, 128, 0, st>>>(x, wt, bias, s, activation, ob, out_f32); break;
    XAC_CO(2) XAC_CO(4) XAC_CO(6) XAC_CO(8) XAC_CO(10) XAC_CO(12) XAC_CO(14) XAC_CO(16)
#undef XAC_CO
    default: set_error("xac_conv3d_forward: unsupported channel slice %d", slice); return XAC_EINVAL;
  }
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
  const int nchunks = (int)((V + kWgChunk - 1) / kWgChunk);
  dim3 grid(nchunks, taps, (Co / 16) * (Ci / 16));
  cudaStream_t st = as_stream(stream);
  conv_wgrad_kernel<<<grid, 128, 0, st>>>((const __nv_bfloat16*)in, (const __nv_bfloat16*)dout, s, partial);
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

int xac_conv3d_partial_floats(int N, int D, int H, int W, int Ci, int Co, int ksize, long long* count) {
  XAC_REQUIRE(count, "xac_conv3d_partial_floats: null pointer");
  const long long V = (long long)N * D * H * W;
  const long long w = ((V + kWgChunk - 1) / kWgChunk) * (ksize == 3 ? 27 : 1) * (long long)Co * Ci;
  const long long b = (long long)kBiasBlocks * Co;
  *count = w > b ? w : b;
  return XAC_OK;
}

}  // extern "C"
