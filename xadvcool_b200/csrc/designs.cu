// Cold-plate designs built on the device: the reference's generate_mask families (src/geometry.py:339-526,
// parameters mapped on the host by xadvcool_b200.designs.reference_spec) and the seeded benchmark designs, the
// per-cell evaluation of xadvcool_b200.designs.build_from_spec
// (straight channels, src/geometry.py:385-434; staggered pin fins; gyroid / Schwarz P / Schwarz D TPMS,
// src/geometry.py:476-495; the frame of src/geometry.py:510-524) and the Gaussian-hotspot floor map. The random
// draws stay on the host (numpy's generator), so a seed gives the same design either way. Every expression keeps
// the host's operand order in double precision (compiled without FMA contraction); the heat map is rounded to
// float32 once, as the host does.
#include <cmath>
#include <cstdint>

#include "xac_internal.cuh"

namespace xac {
namespace {

constexpr int kBase = 4, kTop = 1;  // base plate and lid thickness (src/geometry.py:516-517)

__device__ bool straight_wall(int y, int ny, int width, int n) {
  const int total = n * width;
  if (total >= ny) return false;
  const double gap = (double)(ny - total) / (n + 1);
  const int y_end = (int)gap;
  if (y < y_end) return true;
  double pos = gap;
  for (int i = 0; i < n; ++i) {
    pos += width;
    const int y0 = (int)pos;
    const int y1 = i == n - 1 ? ny : (int)(pos + gap);
    if (y0 < ny && y >= y0 && y < y1) return true;
    pos += gap;
  }
  return false;
}

// Python's float remainder (sign of the divisor), exact like numpy's
__device__ double floor_mod(double a, double b) {
  double m = fmod(a, b);
  if (m != 0.0 && ((m < 0.0) != (b < 0.0))) m += b;
  return m;
}

__global__ void design_kernel(xac_design_spec sp, int32_t* __restrict__ mask, float* __restrict__ heat) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nx = sp.nx, ny = sp.ny, nz = sp.nz;
  if (i >= (long long)nx * ny * nz) return;
  // reference layout [x][y][z], z fastest
  const int z = (int)(i % nz);
  const long long t = i / nz;
  const int y = (int)(t % ny), x = (int)(t / ny);
  const int core = nx - 2 * sp.buf;
  bool solid = false;
  const int xc = x - sp.buf;
  const int family = sp.family & ~XAC_DESIGN_BELOW;
  if (xc >= 0 && xc < core && family != XAC_DESIGN_EMPTY) {
    if (family == XAC_DESIGN_STRAIGHT) {
      solid = straight_wall(y, ny, (int)sp.p0, (int)sp.p1);
    } else if (family == XAC_DESIGN_PIN_FIN) {
      const double radius = sp.p0, pitch = sp.p1, h = pitch / 2;
      const long long ip = (long long)pitch;
      const double ax = (double)(xc % ip) - h, ay = (double)(y % ip) - h;
      const double da = ax * ax + ay * ay;
      const double bx = floor_mod((double)xc - h, pitch) - h, by = floor_mod((double)y - h, pitch) - h;
      const double db = bx * bx + by * by;
      solid = (da < db ? da : db) < radius * radius;
    } else {
      const double omega = 2.0 * M_PI / sp.p0;
      const double wx = (double)xc * omega, wy = (double)y * omega, wz = (double)z * omega;
      double f;
      if (family == XAC_DESIGN_GYROID) {
        f = (sin(wx) * cos(wy) + sin(wy) * cos(wz)) + sin(wz) * cos(wx);
      } else if (family == XAC_DESIGN_SCHWARZ_P) {
        f = (cos(wx) + cos(wy)) + cos(wz);
      } else {
        f = ((sin(wx) * sin(wy) * sin(wz) + sin(wx) * cos(wy) * cos(wz)) + cos(wx) * sin(wy) * cos(wz)) +
            cos(wx) * cos(wy) * sin(wz);
      }
      const bool inside = (sp.family & XAC_DESIGN_BELOW) ? f < sp.p1 : f > sp.p1;
      solid = inside && !(xc < sp.margin || xc >= core - sp.margin);
    }
  }
  int m = solid ? XAC_BC_SOLID : XAC_BC_FLUID;
  if (y == 0 || y == ny - 1 || z < kBase || z >= nz - kTop) m = XAC_BC_SOLID;
  const bool opening = y >= 1 && y < ny - 1 && z >= kBase && z < nz - kTop;
  if (x == 0 && opening) m = XAC_BC_INLET;
  if (x == nx - 1 && opening) m = XAC_BC_OUTLET;
  mask[i] = m;
  float h = 0.0f;
  if (z == 0 && xc >= 0 && xc < core) {
    double hm = sp.background;
    for (int k = 0; k < sp.n_hot; ++k) {
      const double dx = (double)xc - sp.hot[k][0], dy = (double)y - sp.hot[k][1], s = sp.hot[k][2];
      hm += sp.hot[k][3] * exp(-(dx * dx + dy * dy) / (2.0 * (s * s)));
    }
    h = (float)hm;
  }
  heat[i] = h;
}

}  // namespace
}  // namespace xac

using namespace xac;

extern "C" int xac_design_build(const xac_design_spec* spec, int32_t* mask_dev, float* heat_dev, void* stream) {
  XAC_REQUIRE(spec && mask_dev && heat_dev, "xac_design_build: null pointer");
  const xac_design_spec& s = *spec;
  XAC_REQUIRE(s.nx >= 3 && s.ny >= 3 && s.nz > kBase + kTop && s.buf >= 0 && 2 * s.buf < s.nx,
              "xac_design_build: bad shape %d x %d x %d (buffer %d)", s.nx, s.ny, s.nz, s.buf);
  const int fam = s.family & ~XAC_DESIGN_BELOW;
  XAC_REQUIRE(fam >= XAC_DESIGN_EMPTY && fam <= XAC_DESIGN_SCHWARZ_D &&
                  (!(s.family & XAC_DESIGN_BELOW) || fam >= XAC_DESIGN_GYROID),
              "xac_design_build: family %d", s.family);
  XAC_REQUIRE(s.n_hot >= 0 && s.n_hot <= XAC_DESIGN_MAX_HOT, "xac_design_build: %d hotspots (at most %d)", s.n_hot,
              XAC_DESIGN_MAX_HOT);
  XAC_REQUIRE(fam != XAC_DESIGN_PIN_FIN || s.p1 >= 1.0, "xac_design_build: pin pitch must be >= 1");
  XAC_REQUIRE(fam < XAC_DESIGN_GYROID || s.p0 > 0.0, "xac_design_build: TPMS cell size must be positive");
  const long long n = (long long)s.nx * s.ny * s.nz;
  design_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(s, mask_dev, heat_dev);
  XAC_CUDA(cudaGetLastError());
  return XAC_OK;
}
