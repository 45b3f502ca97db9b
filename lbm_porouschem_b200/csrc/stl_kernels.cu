// stl_kernels.cu -- voxelisation of a closed triangle mesh (STL) onto the lattice,
// the geometry step in front of the lattice update (include/lbm_b200.h,
// lbm_voxelise_stl).
//
// The reference reads the mesh with pyvista, voxelises it and samples the voxels
// onto the grid, then derives a surface weight from the number of solid face
// neighbours (src/LBM/GEO/STL.py:147-268).  Here a cell is solid when its centre
// lies inside the mesh, decided by ray parity along x:
//   1. stl_toggle: one thread per triangle.  For every cell-centre line (y, z) that
//      crosses the triangle's projection onto the y-z plane, the crossing x is
//      found and a toggle bit is flipped (atomicXor) at the first cell whose centre
//      lies beyond it.  Points on a shared edge or vertex are counted once: the
//      triangle is oriented counter-clockwise in (y, z) and an edge contains its
//      points only if it is a "top" or "left" edge (the rasteriser's rule).
//   2. stl_prefix: one thread per x row; a prefix XOR of the toggle bits (32 at a
//      time, with a carry between words) gives inside / outside.
//   3. stl_surface: solid flag and surface weight of every cell of the domain, from
//      the 6 (2D: 4) face neighbours on a grid padded by one cell, as the reference
//      pads its sampling grid.
// The grid is voxelised with one cell of padding on each side (z too in 3D);
// cell centres are at ((i + 0.5) dx, (j + 0.5) dx, (k + 0.5) dx) for the domain's
// cells (i, j, k), and the 2D lattice is the plane z = 0.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "lbm_b200.h"

namespace lbm {
namespace capi {
int fail(int code, const std::string& msg);
}
}  // namespace lbm

namespace {

struct StlGrid {
  int px, py, pz;  // padded grid
  int nxw;         // 32-bit toggle words per padded x row
  int dim;
  double dx;
};

__device__ __forceinline__ bool edge_has(double w, double dy, double dz) {
  // inside the edge, or on a top/left edge of a counter-clockwise triangle
  return w > 0.0 || (w == 0.0 && (dz < 0.0 || (dz == 0.0 && dy > 0.0)));
}

__global__ void __launch_bounds__(256) stl_toggle(const float* __restrict__ tri, long long ntri, StlGrid g,
                                                  uint32_t* __restrict__ tog) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ntri; t += stride) {
    const float* v = tri + 9 * t;
    double x0 = v[0], y0 = v[1], z0 = v[2];
    double x1 = v[3], y1 = v[4], z1 = v[5];
    double x2 = v[6], y2 = v[7], z2 = v[8];
    // orientation in the y-z plane; a triangle seen edge-on covers no line
    const double area = (y1 - y0) * (z2 - z0) - (z1 - z0) * (y2 - y0);
    if (area == 0.0) continue;
    if (area < 0.0) {
      double s = x1; x1 = x2; x2 = s;
      s = y1; y1 = y2; y2 = s;
      s = z1; z1 = z2; z2 = s;
    }
    // cell-centre lines inside the projected bounding box (padded index = domain index + 1)
    const double ymin = fmin(y0, fmin(y1, y2)), ymax = fmax(y0, fmax(y1, y2));
    int j0 = (int)ceil(ymin / g.dx - 0.5) + 1, j1 = (int)floor(ymax / g.dx - 0.5) + 1;
    j0 = max(j0, 0);
    j1 = min(j1, g.py - 1);
    int k0 = 0, k1 = 0;
    if (g.dim == 3) {
      const double zmin = fmin(z0, fmin(z1, z2)), zmax = fmax(z0, fmax(z1, z2));
      k0 = max((int)ceil(zmin / g.dx - 0.5) + 1, 0);
      k1 = min((int)floor(zmax / g.dx - 0.5) + 1, g.pz - 1);
    }
    for (int k = k0; k <= k1; ++k) {
      const double pz = g.dim == 3 ? (k - 1 + 0.5) * g.dx : 0.0;
      if (g.dim == 2 && !(fmin(z0, fmin(z1, z2)) <= 0.0 && fmax(z0, fmax(z1, z2)) >= 0.0)) break;
      for (int j = j0; j <= j1; ++j) {
        const double py = (j - 1 + 0.5) * g.dx;
        // edge functions (twice the signed sub-areas opposite each vertex)
        const double w0 = (y2 - y1) * (pz - z1) - (z2 - z1) * (py - y1);
        const double w1 = (y0 - y2) * (pz - z2) - (z0 - z2) * (py - y2);
        const double w2 = (y1 - y0) * (pz - z0) - (z1 - z0) * (py - y0);
        if (!(edge_has(w0, y2 - y1, z2 - z1) && edge_has(w1, y0 - y2, z0 - z2) && edge_has(w2, y1 - y0, z1 - z0)))
          continue;
        const double xc = (w0 * x0 + w1 * x1 + w2 * x2) / (w0 + w1 + w2);
        // first padded cell whose centre lies beyond the crossing
        const double fi = floor(xc / g.dx - 0.5) + 2.0;
        if (fi >= (double)g.px) continue;
        const int i = fi < 0.0 ? 0 : (int)fi;
        atomicXor(&tog[(size_t)(i >> 5) + (size_t)g.nxw * ((size_t)j + (size_t)g.py * k)], 1u << (i & 31));
      }
    }
  }
}

__global__ void __launch_bounds__(256) stl_prefix(const uint32_t* __restrict__ tog, StlGrid g,
                                                  uint8_t* __restrict__ inside) {
  const size_t rows = (size_t)g.py * g.pz;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
    uint32_t carry = 0;
    for (int w = 0; w < g.nxw; ++w) {
      uint32_t p = tog[(size_t)w + (size_t)g.nxw * r];
      p ^= p << 1;
      p ^= p << 2;
      p ^= p << 4;
      p ^= p << 8;
      p ^= p << 16;  // bit b: parity of bits 0..b
      p ^= carry;
      carry = (p >> 31) ? 0xffffffffu : 0u;
      const int nb = min(32, g.px - 32 * w);
      for (int b = 0; b < nb; ++b) inside[r * g.px + 32 * w + b] = (uint8_t)((p >> b) & 1u);
    }
  }
}

__global__ void __launch_bounds__(256) stl_surface(const uint8_t* __restrict__ inside, StlGrid g, int nx, int ny,
                                                   int nz, uint8_t* __restrict__ solid, float* __restrict__ surface) {
  const size_t n = (size_t)nx * ny * nz;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t pxy = (size_t)g.px * g.py;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));
    const int pzi = g.dim == 3 ? z + 1 : 0;
    const size_t q = (size_t)(x + 1) + (size_t)g.px * (y + 1) + pxy * pzi;
    const uint8_t s = inside[q];
    solid[c] = s;
    if (surface) {
      float wgt = 0.0f;
      if (s) {
        int cnt = inside[q - 1] + inside[q + 1] + inside[q - g.px] + inside[q + g.px];
        if (g.dim == 3) {
          cnt += inside[q - pxy] + inside[q + pxy];
          // src/LBM/GEO/STL.py:237-255
          const float tab3[7] = {6.0f, 4.0f, 3.0f, 2.0f, 1.414f, 1.0f, 0.0f};
          wgt = tab3[cnt];
        } else {
          // src/LBM/GEO/STL.py:217-235
          const float tab2[5] = {4.0f, 2.0f, 1.414f, 1.0f, 0.0f};
          wgt = tab2[cnt];
        }
      }
      surface[c] = wgt;
    }
  }
}

StlGrid stl_grid(int nx, int ny, int nz, int dim, double dx) {
  StlGrid g;
  g.px = nx + 2;
  g.py = ny + 2;
  g.pz = dim == 3 ? nz + 2 : 1;
  g.nxw = (g.px + 31) / 32;
  g.dim = dim;
  g.dx = dx;
  return g;
}

size_t stl_toggle_bytes(const StlGrid& g) { return (size_t)4 * g.nxw * g.py * g.pz; }
size_t stl_work_bytes(const StlGrid& g) {
  return (stl_toggle_bytes(g) + 255) / 256 * 256 + (size_t)g.px * g.py * g.pz;
}

int stl_check(int32_t nx, int32_t ny, int32_t nz, int32_t dim) {
  using lbm::capi::fail;
  if (dim != 2 && dim != 3) return fail(LBM_ERR_ARG, "dim must be 2 or 3");
  if (nx < 1 || ny < 1 || nz < 1 || (dim == 2 && nz != 1)) return fail(LBM_ERR_ARG, "bad lattice size");
  if ((double)(nx + 2) * (ny + 2) * (nz + 2) >= 2147483647.0) return fail(LBM_ERR_SIZE, "lattice too large");
  return LBM_OK;
}

}  // namespace

extern "C" {

int32_t lbm_stl_work_bytes(int32_t nx, int32_t ny, int32_t nz, int32_t dim, size_t* bytes) {
  const int rc = stl_check(nx, ny, nz, dim);
  if (rc) return rc;
  if (!bytes) return lbm::capi::fail(LBM_ERR_ARG, "bytes is NULL");
  *bytes = stl_work_bytes(stl_grid(nx, ny, nz, dim, 1.0));
  return LBM_OK;
}

int32_t lbm_voxelise_stl(const float* triangles, int64_t ntri, int32_t nx, int32_t ny, int32_t nz, int32_t dim,
                         double dx, void* work, size_t work_bytes, uint8_t* solid, float* surface, void* stream) {
  using lbm::capi::fail;
  int rc = stl_check(nx, ny, nz, dim);
  if (rc) return rc;
  if (ntri < 0 || (ntri > 0 && !triangles)) return fail(LBM_ERR_ARG, "triangles is NULL");
  if (!(dx > 0)) return fail(LBM_ERR_ARG, "dx must be > 0");
  if (!solid) return fail(LBM_ERR_ARG, "solid is NULL");
  const StlGrid g = stl_grid(nx, ny, nz, dim, dx);
  if (!work || work_bytes < stl_work_bytes(g)) return fail(LBM_ERR_ARG, "work buffer missing or too small");
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t* tog = (uint32_t*)work;
  uint8_t* inside = (uint8_t*)work + (stl_toggle_bytes(g) + 255) / 256 * 256;
  cudaError_t e = cudaMemsetAsync(tog, 0, stl_toggle_bytes(g), st);
  if (e != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  if (ntri > 0) {
    const long long blocks = (ntri + 255) / 256;
    stl_toggle<<<(unsigned)(blocks < 8192 ? blocks : 8192), 256, 0, st>>>(triangles, ntri, g, tog);
  }
  const size_t rows = (size_t)g.py * g.pz;
  stl_prefix<<<(unsigned)((rows + 255) / 256 < 8192 ? (rows + 255) / 256 : 8192), 256, 0, st>>>(tog, g, inside);
  const size_t n = (size_t)nx * ny * nz;
  stl_surface<<<(unsigned)((n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384), 256, 0, st>>>(inside, g, nx, ny, nz,
                                                                                             solid, surface);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("stl kernels: ") + cudaGetErrorString(e));
  return LBM_OK;
}

}  // extern "C"
