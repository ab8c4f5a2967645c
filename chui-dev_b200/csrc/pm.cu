// Particle-mesh long-range force on the B200: periodic CIC/TSC mass assignment,
// cuFFT real-to-complex transform, one fused k-space pass (Green's function x
// assignment-window deconvolution x Gaussian split filter x spectral gradient,
// emitting the three force spectra), three complex-to-real transforms, and
// CIC/TSC force interpolation.
//
// Reference: src/gravity/pm_solver.cpp -- makeAxisStencil :925-951,
// assignDensityImpl :3842-4565, solvePoissonPeriodicImpl :4581-4940,
// ensureSpectralAxisMetadata :2398-2466, applyDerivedPoissonOperator
// :2557-2656, fillGradientSpectrum :2658-2706, interpolateForcesImpl
// :5735-5953.
//
// Layout in HBM: one in-place FFT array per force component, nx*ny*nzp reals
// (nzp = 2*(nz/2+1), FFTW/cuFFT padded rows). grid[0] carries the density
// (minus its mean), is transformed in place, and is overwritten by the F_x
// spectrum; grid[1], grid[2] receive F_y, F_z. Mixed precision keeps the mesh
// in FP32; the FP64 configuration uses double grids and Z2D/D2Z plans.
#include <cuda_runtime.h>

#include <type_traits>
#include <cufft.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "context.cuh"

namespace chui {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

struct PmGeom {
  int64_t n[3];
  int64_t nzc, nzp;
  double L[3];
  double inv_d[3];
  int scheme;
  int periodic;  // 0: isolated/open (no wrap; cells outside the mesh dropped)
};

PmGeom geomOf(const Context& c) {
  PmGeom g;
  g.n[0] = c.cfg.pm_grid_nx;
  g.n[1] = c.cfg.pm_grid_ny;
  g.n[2] = c.cfg.pm_grid_nz;
  g.nzc = g.n[2] / 2 + 1;
  g.nzp = 2 * g.nzc;
  g.L[0] = c.cfg.box_x;
  g.L[1] = c.cfg.box_y;
  g.L[2] = c.cfg.box_z;
  for (int a = 0; a < 3; ++a) g.inv_d[a] = static_cast<double>(g.n[a]) / g.L[a];
  g.scheme = c.cfg.assignment_scheme;
  g.periodic = c.cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_PERIODIC ? 1 : 0;
  return g;
}

// positionInsideOpenDomain (pm_solver.cpp:117-119)
__device__ __forceinline__ bool insideOpen(double v, double box) { return v >= 0.0 && v < box; }

// wrapPosition (pm_solver.cpp:112-115): fmod is exact, so cell indices match.
__device__ __forceinline__ double wrapPosition(double v, double box) {
  const double w = fmod(v, box);
  return w < 0.0 ? w + box : w;
}

__device__ __forceinline__ int64_t wrapIndex(int64_t i, int64_t n) {
  int64_t w = i % n;
  return w < 0 ? w + n : w;
}

struct Stencil {
  int64_t off0;
  double w[3];
};

// makeAxisStencil (pm_solver.cpp:925-951).
__device__ __forceinline__ Stencil makeStencil(double gp, int scheme) {
  Stencil s;
  if (scheme == 0) {
    const double base = floor(gp);
    const double t = gp - base;
    s.off0 = static_cast<int64_t>(base);
    s.w[0] = 1.0 - t;
    s.w[1] = t;
    s.w[2] = 0.0;
  } else {
    const double center = floor(gp + 0.5);
    const double d = gp - center;
    s.off0 = static_cast<int64_t>(center) - 1;
    s.w[0] = 0.5 * ((0.5 - d) * (0.5 - d));
    s.w[1] = 0.75 - d * d;
    s.w[2] = 0.5 * ((0.5 + d) * (0.5 + d));
  }
  return s;
}

template <class R>
__global__ void fillKernel(R* grid, size_t count, R value) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    grid[i] = value;
  }
}

// Mass assignment: one thread per particle, `taps`^3 atomic adds into the FP32
// (or FP64) padded grid; the 1/cell_volume normalization is folded into the
// per-particle mass.
template <class R>
__global__ void depositKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, const double* __restrict__ m,
                              double uniform_mass, double inv_cell_volume, PmGeom g, R* grid) {
  const int taps = g.scheme == 0 ? 2 : 3;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const Stencil sx = makeStencil(wrapPosition(x[i], g.L[0]) * g.inv_d[0], g.scheme);
    const Stencil sy = makeStencil(wrapPosition(y[i], g.L[1]) * g.inv_d[1], g.scheme);
    const Stencil sz = makeStencil(wrapPosition(z[i], g.L[2]) * g.inv_d[2], g.scheme);
    const double mass = (m ? m[i] : uniform_mass) * inv_cell_volume;
    for (int a = 0; a < taps; ++a) {
      const int64_t ix = wrapIndex(sx.off0 + a, g.n[0]);
      for (int b = 0; b < taps; ++b) {
        const int64_t iy = wrapIndex(sy.off0 + b, g.n[1]);
        const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp;
        const double wxy = sx.w[a] * sy.w[b];
        for (int cc = 0; cc < taps; ++cc) {
          const int64_t iz = wrapIndex(sz.off0 + cc, g.n[2]);
          atomicAdd(grid + row + iz, static_cast<R>(mass * (wxy * sz.w[cc])));
        }
      }
    }
  }
}

// Mass assignment over tree-ordered sources (double4 {position, mass}),
// accumulated per block in a shared-memory tile. A block takes chunks of
// kDepositChunk consecutive tree positions, which occupy a compact region;
// it finds the chunk's base-cell bounding box, and when the stencil box fits
// the tile it deposits into shared memory and then adds the tile's nonzero
// cells to the grid (one global atomic per touched cell instead of taps^3 per
// particle). Each thread takes a contiguous run of the chunk and sums the
// stencils of consecutive particles with the same base cell in registers
// (dense regions repeat base cells along tree order), so shared-memory
// atomics are issued once per run of equal cells and lanes of a warp work in
// different places. Chunks that straddle the periodic boundary or are too
// spread out deposit with global atomics. Weights and cells are those of
// depositKernel (same stencil arithmetic); only the summation order differs.
#ifndef CHUI_DEPOSIT_CHUNK
#define CHUI_DEPOSIT_CHUNK 2048
#endif
constexpr int kDepositChunk = CHUI_DEPOSIT_CHUNK;
constexpr int kDepositTileBytes = 32768;

template <class R, int kTaps>
__device__ __forceinline__ void tileFlush(R* tile, int e1, int e2, int lx, int ly, int lz, const R (&acc)[kTaps * kTaps * kTaps]) {
#pragma unroll
  for (int a = 0; a < kTaps; ++a)
#pragma unroll
    for (int b = 0; b < kTaps; ++b)
#pragma unroll
      for (int c = 0; c < kTaps; ++c) {
        const R v = acc[(a * kTaps + b) * kTaps + c];
        if (v != R(0)) atomicAdd(tile + ((lx + a) * e1 + (ly + b)) * e2 + (lz + c), v);
      }
}

template <class R, int kTaps>
__global__ void __launch_bounds__(256) depositTiledKernel(int64_t n, const double4* __restrict__ src,
                                                          double inv_cell_volume, PmGeom g, R* grid) {
  __shared__ __align__(16) unsigned char tile_raw[kDepositTileBytes];
  __shared__ int box_lo[3], box_hi[3];
  R* tile = reinterpret_cast<R*>(tile_raw);
  constexpr int kTileCells = kDepositTileBytes / static_cast<int>(sizeof(R));
  const int64_t chunks = (n + kDepositChunk - 1) / kDepositChunk;
  for (int64_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x) {
    const int64_t begin = chunk * kDepositChunk;
    const int count = static_cast<int>(n - begin < kDepositChunk ? n - begin : kDepositChunk);
    if (threadIdx.x < 3) {
      box_lo[threadIdx.x] = INT_MAX;
      box_hi[threadIdx.x] = INT_MIN;
    }
    __syncthreads();
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
      const double4 p = src[begin + i];
      const double v[3] = {p.x, p.y, p.z};
      for (int a = 0; a < 3; ++a) {
        const int o = static_cast<int>(makeStencil(wrapPosition(v[a], g.L[a]) * g.inv_d[a], g.scheme).off0);
        lo[a] = min(lo[a], o);
        hi[a] = max(hi[a], o);
      }
    }
    for (int a = 0; a < 3; ++a) {
      for (int off = 16; off > 0; off >>= 1) {
        lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
        hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
      }
    }
    if ((threadIdx.x & 31) == 0) {
      for (int a = 0; a < 3; ++a) {
        atomicMin(box_lo + a, lo[a]);
        atomicMax(box_hi + a, hi[a]);
      }
    }
    __syncthreads();
    const int b0 = box_lo[0], b1 = box_lo[1], b2 = box_lo[2];
    const int e0 = box_hi[0] - b0 + kTaps, e1 = box_hi[1] - b1 + kTaps, e2 = box_hi[2] - b2 + kTaps;
    const int64_t cells = static_cast<int64_t>(e0) * e1 * e2;
    if (cells <= kTileCells) {
      const int tc = static_cast<int>(cells);
      for (int t = threadIdx.x; t < tc; t += blockDim.x) tile[t] = R(0);
      __syncthreads();
      // contiguous run per thread, equal base cells summed in registers
      const int per = (count + static_cast<int>(blockDim.x) - 1) / static_cast<int>(blockDim.x);
      const int i0 = static_cast<int>(threadIdx.x) * per;
      const int i1 = min(i0 + per, count);
      R acc[kTaps * kTaps * kTaps];
#pragma unroll
      for (int t = 0; t < kTaps * kTaps * kTaps; ++t) acc[t] = R(0);
      int cx = INT_MIN, cy = 0, cz = 0;
      for (int i = i0; i < i1; ++i) {
        const double4 p = src[begin + i];
        const Stencil s0 = makeStencil(wrapPosition(p.x, g.L[0]) * g.inv_d[0], g.scheme);
        const Stencil s1 = makeStencil(wrapPosition(p.y, g.L[1]) * g.inv_d[1], g.scheme);
        const Stencil s2 = makeStencil(wrapPosition(p.z, g.L[2]) * g.inv_d[2], g.scheme);
        const int lx = static_cast<int>(s0.off0) - b0, ly = static_cast<int>(s1.off0) - b1,
                  lz = static_cast<int>(s2.off0) - b2;
        if (lx != cx || ly != cy || lz != cz) {
          if (cx != INT_MIN) tileFlush<R, kTaps>(tile, e1, e2, cx, cy, cz, acc);
#pragma unroll
          for (int t = 0; t < kTaps * kTaps * kTaps; ++t) acc[t] = R(0);
          cx = lx;
          cy = ly;
          cz = lz;
        }
        const double mass = p.w * inv_cell_volume;
#pragma unroll
        for (int a = 0; a < kTaps; ++a)
#pragma unroll
          for (int b = 0; b < kTaps; ++b) {
            const double wxy = s0.w[a] * s1.w[b];
#pragma unroll
            for (int c = 0; c < kTaps; ++c) acc[(a * kTaps + b) * kTaps + c] += static_cast<R>(mass * (wxy * s2.w[c]));
          }
      }
      if (cx != INT_MIN) tileFlush<R, kTaps>(tile, e1, e2, cx, cy, cz, acc);
      __syncthreads();
      for (int t = threadIdx.x; t < tc; t += blockDim.x) {
        const R v = tile[t];
        if (v == R(0)) continue;
        const int lz = t % e2;
        const int ly = (t / e2) % e1;
        const int lx = t / (e1 * e2);
        const int64_t ix = wrapIndex(b0 + lx, g.n[0]);
        const int64_t iy = wrapIndex(b1 + ly, g.n[1]);
        const int64_t iz = wrapIndex(b2 + lz, g.n[2]);
        atomicAdd(grid + (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp + iz, v);
      }
    } else {
      for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double4 p = src[begin + i];
        const Stencil s0 = makeStencil(wrapPosition(p.x, g.L[0]) * g.inv_d[0], g.scheme);
        const Stencil s1 = makeStencil(wrapPosition(p.y, g.L[1]) * g.inv_d[1], g.scheme);
        const Stencil s2 = makeStencil(wrapPosition(p.z, g.L[2]) * g.inv_d[2], g.scheme);
        const double mass = p.w * inv_cell_volume;
        for (int a = 0; a < kTaps; ++a) {
          const int64_t ix = wrapIndex(s0.off0 + a, g.n[0]);
          for (int b = 0; b < kTaps; ++b) {
            const int64_t iy = wrapIndex(s1.off0 + b, g.n[1]);
            const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp;
            const double wxy = s0.w[a] * s1.w[b];
            for (int cc = 0; cc < kTaps; ++cc) {
              const int64_t iz = wrapIndex(s2.off0 + cc, g.n[2]);
              atomicAdd(grid + row + iz, static_cast<R>(mass * (wxy * s2.w[cc])));
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

template <class R>
void launchDepositTiled(int64_t n, const double4* src, double inv_cell_volume, const PmGeom& g, R* grid,
                        cudaStream_t s) {
  const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((n + kDepositChunk - 1) / kDepositChunk, 148 * 8));
  noteLaunch();
  if (g.scheme == 0) {
    depositTiledKernel<R, 2><<<blocks, 256, 0, s>>>(n, src, inv_cell_volume, g, grid);
  } else {
    depositTiledKernel<R, 3><<<blocks, 256, 0, s>>>(n, src, inv_cell_volume, g, grid);
  }
}

// Same assignment into a compact FP64 grid (diagnostic density output).
__global__ void depositCompactKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                     const double* __restrict__ z, const double* __restrict__ m,
                                     double uniform_mass, PmGeom g, double* grid) {
  const int taps = g.scheme == 0 ? 2 : 3;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // isolated/open: particles outside [0, L) and cells outside the mesh are
    // dropped (pm_solver.cpp:4016-4049)
    if (!g.periodic && !(insideOpen(x[i], g.L[0]) && insideOpen(y[i], g.L[1]) && insideOpen(z[i], g.L[2]))) continue;
    const Stencil sx = makeStencil((g.periodic ? wrapPosition(x[i], g.L[0]) : x[i]) * g.inv_d[0], g.scheme);
    const Stencil sy = makeStencil((g.periodic ? wrapPosition(y[i], g.L[1]) : y[i]) * g.inv_d[1], g.scheme);
    const Stencil sz = makeStencil((g.periodic ? wrapPosition(z[i], g.L[2]) : z[i]) * g.inv_d[2], g.scheme);
    const double mass = m ? m[i] : uniform_mass;
    for (int a = 0; a < taps; ++a) {
      const int64_t ox = sx.off0 + a;
      if (!g.periodic && (ox < 0 || ox >= g.n[0])) continue;
      const int64_t ix = g.periodic ? wrapIndex(ox, g.n[0]) : ox;
      for (int b = 0; b < taps; ++b) {
        const int64_t oy = sy.off0 + b;
        if (!g.periodic && (oy < 0 || oy >= g.n[1])) continue;
        const int64_t iy = g.periodic ? wrapIndex(oy, g.n[1]) : oy;
        for (int cc = 0; cc < taps; ++cc) {
          const int64_t oz = sz.off0 + cc;
          if (!g.periodic && (oz < 0 || oz >= g.n[2])) continue;
          const int64_t iz = g.periodic ? wrapIndex(oz, g.n[2]) : oz;
          const double w = sx.w[a] * sy.w[b] * sz.w[cc];
          atomicAdd(grid + (static_cast<size_t>(ix) * g.n[1] + iy) * g.n[2] + iz, mass * w);
        }
      }
    }
  }
}

__global__ void scaleKernel(double* v, size_t count, double factor) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    v[i] /= factor;
  }
}

__global__ void cellsKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, PmGeom g, int64_t* cells) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double p[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      const Stencil s = makeStencil(wrapPosition(p[a], g.L[a]) * g.inv_d[a], g.scheme);
      cells[3 * i + a] = wrapIndex(s.off0, g.n[a]);
    }
  }
}

// Fused k-space pass over the half spectrum: Psi = G(k) rho_k with
// G = -4 pi G_N W(k)^-2 exp(-(|k| r_s)^2) / k^2 / M (k = 0 -> 0), then
// F_a = -i g_a Psi with g_a = k_a except the Nyquist index of an even axis.
// Reads rho_k once and writes three spectra (F_x in place).
template <class R, class C>
__global__ void greenGradientKernel(PmGeom g, const double* __restrict__ tab, double prefactor,
                                    double rs, int deconv, C* c0, C* c1, C* c2) {
  const int64_t nx = g.n[0], ny = g.n[1], nzc = g.nzc;
  const double* kx = tab;
  const double* ky = kx + nx;
  const double* kz = ky + ny;
  const double* wx = kz + nzc;
  const double* wy = wx + nx;
  const double* wz = wy + ny;
  const double* gx = wz + nzc;
  const double* gy = gx + nx;
  const double* gz = gy + ny;
  const size_t total = static_cast<size_t>(nx) * ny * nzc;
  for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int64_t iz = static_cast<int64_t>(idx % nzc);
    const size_t row = idx / nzc;
    const int64_t iy = static_cast<int64_t>(row % ny);
    const int64_t ix = static_cast<int64_t>(row / ny);
    const double k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
    double op = 0.0;
    if (k2 != 0.0) {
      double window = 1.0;
      if (deconv) {
        const double tw = wx[ix] * wy[iy] * wz[iz];
        const double w2 = tw * tw;
        window = 1.0 / (w2 > 1.0e-12 ? w2 : 1.0e-12);
      }
      const double prod = sqrt(k2) * rs;
      op = prefactor * window * exp(-(prod * prod)) / k2;
    }
    const C rho = c0[idx];
    const R re = static_cast<R>(op) * rho.x;
    const R im = static_cast<R>(op) * rho.y;
    const R ga = static_cast<R>(gx[ix]);
    const R gb = static_cast<R>(gy[iy]);
    const R gc = static_cast<R>(gz[iz]);
    C fx, fy, fz;
    fx.x = ga * im;
    fx.y = -ga * re;
    fy.x = gb * im;
    fy.y = -gb * re;
    fz.x = gc * im;
    fz.y = -gc * re;
    c0[idx] = fx;
    c1[idx] = fy;
    c2[idx] = fz;
  }
}

// taps^3 stencil gathers of the three padded force grids at one position
// (interpolateForcesImpl, pm_solver.cpp:5735-5953); isolated/open
// boundaries: no force outside [0, L), cells outside the mesh skipped.
template <class R>
__device__ __forceinline__ void gatherForce(const PmGeom& g, const R* __restrict__ fxg, const R* __restrict__ fyg,
                                            const R* __restrict__ fzg, double px, double py, double pz, R& gx,
                                            R& gy, R& gz) {
  gx = gy = gz = R(0);
  if (!g.periodic && !(insideOpen(px, g.L[0]) && insideOpen(py, g.L[1]) && insideOpen(pz, g.L[2]))) return;
  const int taps = g.scheme == 0 ? 2 : 3;
  const Stencil s0 = makeStencil((g.periodic ? wrapPosition(px, g.L[0]) : px) * g.inv_d[0], g.scheme);
  const Stencil s1 = makeStencil((g.periodic ? wrapPosition(py, g.L[1]) : py) * g.inv_d[1], g.scheme);
  const Stencil s2 = makeStencil((g.periodic ? wrapPosition(pz, g.L[2]) : pz) * g.inv_d[2], g.scheme);
  for (int a = 0; a < taps; ++a) {
    const int64_t ox = s0.off0 + a;
    if (!g.periodic && (ox < 0 || ox >= g.n[0])) continue;
    const int64_t ix = g.periodic ? wrapIndex(ox, g.n[0]) : ox;
    for (int b = 0; b < taps; ++b) {
      const int64_t oy = s1.off0 + b;
      if (!g.periodic && (oy < 0 || oy >= g.n[1])) continue;
      const int64_t iy = g.periodic ? wrapIndex(oy, g.n[1]) : oy;
      const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp;
      const R wab = static_cast<R>(s0.w[a] * s1.w[b]);
      for (int cc = 0; cc < taps; ++cc) {
        const int64_t oz = s2.off0 + cc;
        if (!g.periodic && (oz < 0 || oz >= g.n[2])) continue;
        const int64_t iz = g.periodic ? wrapIndex(oz, g.n[2]) : oz;
        const R w = wab * static_cast<R>(s2.w[cc]);
        gx += w * fxg[row + iz];
        gy += w * fyg[row + iz];
        gz += w * fzg[row + iz];
      }
    }
  }
}

// The same gathers from the interleaved field of a periodic mixed-precision
// mesh: one 16-byte record {F_x, F_y, F_z, 0} per cell, row-major without the
// FFT padding, so each stencil cell costs one sector instead of one in each
// of three grids. Weights, products and sums are those of gatherForce<float>.
__device__ __forceinline__ void gatherForce4(const PmGeom& g, const float4* __restrict__ f4, double px, double py,
                                             double pz, float& gx, float& gy, float& gz) {
  gx = gy = gz = 0.f;
  const int taps = g.scheme == 0 ? 2 : 3;
  const Stencil s0 = makeStencil(wrapPosition(px, g.L[0]) * g.inv_d[0], g.scheme);
  const Stencil s1 = makeStencil(wrapPosition(py, g.L[1]) * g.inv_d[1], g.scheme);
  const Stencil s2 = makeStencil(wrapPosition(pz, g.L[2]) * g.inv_d[2], g.scheme);
  for (int a = 0; a < taps; ++a) {
    const int64_t ix = wrapIndex(s0.off0 + a, g.n[0]);
    for (int b = 0; b < taps; ++b) {
      const int64_t iy = wrapIndex(s1.off0 + b, g.n[1]);
      const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.n[2];
      const float wab = static_cast<float>(s0.w[a] * s1.w[b]);
      for (int cc = 0; cc < taps; ++cc) {
        const int64_t iz = wrapIndex(s2.off0 + cc, g.n[2]);
        const float w = wab * static_cast<float>(s2.w[cc]);
        const float4 v = f4[row + iz];
        gx += w * v.x;
        gy += w * v.y;
        gz += w * v.z;
      }
    }
  }
}

// {F_x, F_y, F_z, 0} per cell from the three padded real grids.
__global__ void interleaveForceKernel(PmGeom g, const float* __restrict__ fx, const float* __restrict__ fy,
                                      const float* __restrict__ fz, float4* out) {
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t row = i / static_cast<size_t>(g.n[2]);
    const size_t src = row * static_cast<size_t>(g.nzp) + (i - row * static_cast<size_t>(g.n[2]));
    out[i] = make_float4(fx[src], fy[src], fz[src], 0.f);
  }
}

// Interpolation and the total force of a solve in one pass over the active
// slots: the stencil gathers, the walk's part (written at the slot), and the
// total and optional lanes written once (TreePmForceAccumulatorView's accel,
// long-range, short-range and nearest-pair lanes, tree_pm_coupling.cpp:1961-1978),
// with no long-range lane round trip through memory.
template <class R>
__global__ void interpolateCombineKernel(int64_t nt, const uint32_t* __restrict__ active,
                                         const double* __restrict__ tx, const double* __restrict__ ty,
                                         const double* __restrict__ tz, int64_t n, const double* __restrict__ sx_pos,
                                         const double* __restrict__ sy_pos, const double* __restrict__ sz_pos,
                                         PmGeom g, const R* __restrict__ fxg, const R* __restrict__ fyg,
                                         const R* __restrict__ fzg, const float4* __restrict__ f4, int with_pm,
                                         const double* __restrict__ tree,
                                         const double* __restrict__ near, double* ax, double* ay, double* az,
                                         double* lx, double* ly, double* lz, double* sx, double* sy, double* sz,
                                         double* snear) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nt;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t row = tx ? kInvalid : (active ? active[k] : static_cast<uint32_t>(k));
    R gx = R(0), gy = R(0), gz = R(0);
    if (with_pm) {
      double px, py, pz;
      if (tx) {
        px = tx[k];
        py = ty[k];
        pz = tz[k];
      } else {
        px = sx_pos[row];
        py = sy_pos[row];
        pz = sz_pos[row];
      }
      if constexpr (std::is_same<R, float>::value) {
        if (f4) gatherForce4(g, f4, px, py, pz, gx, gy, gz);
        else gatherForce<R>(g, fxg, fyg, fzg, px, py, pz, gx, gy, gz);
      } else {
        gatherForce<R>(g, fxg, fyg, fzg, px, py, pz, gx, gy, gz);
      }
    }
    const double pmx = static_cast<double>(gx), pmy = static_cast<double>(gy), pmz = static_cast<double>(gz);
    const double trx = tree[k], try_ = tree[nt + k], trz = tree[2 * nt + k];
    ax[k] = pmx + trx;
    ay[k] = pmy + try_;
    az[k] = pmz + trz;
    if (lx) {
      lx[k] = pmx;
      ly[k] = pmy;
      lz[k] = pmz;
    }
    if (row < n) {
      if (sx) {
        sx[row] = trx;
        sy[row] = try_;
        sz[row] = trz;
      }
      if (snear) snear[row] = near[k];
    }
  }
}

// Force interpolation at targets: taps^3 gathers from the three padded
// force grids. Targets are active slots (rows of the source arrays) or
// explicit positions.
template <class R>
__global__ void interpolateKernel(int64_t nt, const uint32_t* __restrict__ order,
                                  const uint32_t* __restrict__ active,
                                  const double* __restrict__ tx, const double* __restrict__ ty,
                                  const double* __restrict__ tz, const double* __restrict__ sx,
                                  const double* __restrict__ sy, const double* __restrict__ sz,
                                  PmGeom g, const R* __restrict__ fxg, const R* __restrict__ fyg,
                                  const R* __restrict__ fzg, const float4* __restrict__ f4, double* ax, double* ay,
                                  double* az) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < nt;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // slot k: the j-th target, or the j-th entry of a visit-order slice
    // (written at j)
    const int64_t k = order ? static_cast<int64_t>(order[j]) : j;
    double px, py, pz;
    if (tx) {
      px = tx[k];
      py = ty[k];
      pz = tz[k];
    } else {
      const int64_t row = active ? static_cast<int64_t>(active[k]) : k;
      px = sx[row];
      py = sy[row];
      pz = sz[row];
    }
    R gx, gy, gz;
    if constexpr (std::is_same<R, float>::value) {
      if (f4) gatherForce4(g, f4, px, py, pz, gx, gy, gz);
      else gatherForce<R>(g, fxg, fyg, fzg, px, py, pz, gx, gy, gz);
    } else {
      gatherForce<R>(g, fxg, fyg, fzg, px, py, pz, gx, gy, gz);
    }
    const int64_t o = order ? j : k;
    ax[o] = static_cast<double>(gx);
    ay[o] = static_cast<double>(gy);
    az[o] = static_cast<double>(gz);
  }
}

// ---- isolated/open boundaries (solvePoissonIsolatedOpen, pm_solver.cpp:4942-5337) ----
// Padded mesh: px = 2 nx, py = 2 ny, pz = 2 nz in the in-place real layout with
// rows of pzp = 2 (pz/2 + 1) reals; the physical mesh is the corner ix < nx,
// iy < ny, iz < nz.
struct IsoGeom {
  int64_t px, py, pz, pzp;
};

template <class R>
__global__ void depositIsolatedKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                      const double* __restrict__ z, const double* __restrict__ m,
                                      double uniform_mass, double inv_cell_volume, PmGeom g, IsoGeom q, R* pad) {
  const int taps = g.scheme == 0 ? 2 : 3;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (!(insideOpen(x[i], g.L[0]) && insideOpen(y[i], g.L[1]) && insideOpen(z[i], g.L[2]))) continue;
    const Stencil sx = makeStencil(x[i] * g.inv_d[0], g.scheme);
    const Stencil sy = makeStencil(y[i] * g.inv_d[1], g.scheme);
    const Stencil sz = makeStencil(z[i] * g.inv_d[2], g.scheme);
    const double mass = (m ? m[i] : uniform_mass) * inv_cell_volume;
    for (int a = 0; a < taps; ++a) {
      const int64_t ix = sx.off0 + a;
      if (ix < 0 || ix >= g.n[0]) continue;
      for (int b = 0; b < taps; ++b) {
        const int64_t iy = sy.off0 + b;
        if (iy < 0 || iy >= g.n[1]) continue;
        const size_t row = (static_cast<size_t>(ix) * q.py + iy) * q.pzp;
        const double wxy = sx.w[a] * sy.w[b];
        for (int cc = 0; cc < taps; ++cc) {
          const int64_t iz = sz.off0 + cc;
          if (iz < 0 || iz >= g.n[2]) continue;
          atomicAdd(pad + row + iz, static_cast<R>(mass * (wxy * sz.w[cc])));
        }
      }
    }
  }
}

// The split Green function on the padded mesh at minimum-image separations:
// -erf(r / 2 r_s) / r, and -1 / (sqrt(pi) r_s) at r = 0 (pm_solver.cpp:5150-5204).
template <class R>
__global__ void isoKernelFillKernel(PmGeom g, IsoGeom q, double dx, double dy, double dz, double rs, R* pad) {
  const size_t total = static_cast<size_t>(q.px) * q.py * q.pz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int64_t iz = static_cast<int64_t>(i % q.pz);
    const int64_t iy = static_cast<int64_t>((i / q.pz) % q.py);
    const int64_t ix = static_cast<int64_t>(i / (static_cast<size_t>(q.pz) * q.py));
    const double rx = static_cast<double>(ix <= g.n[0] ? ix : ix - q.px) * dx;
    const double ry = static_cast<double>(iy <= g.n[1] ? iy : iy - q.py) * dy;
    const double rz = static_cast<double>(iz <= g.n[2] ? iz : iz - q.pz) * dz;
    const double r = sqrt(rx * rx + ry * ry + rz * rz);
    const double kernel = r > 0.0 ? -erf(0.5 * r / rs) / r : -1.0 / (sqrt(kPi) * rs);
    pad[(static_cast<size_t>(ix) * q.py + iy) * q.pzp + iz] = static_cast<R>(kernel);
  }
}

// The kernel is real and even on the padded mesh, so its spectrum is real:
// keep the real part, scaled by G dV / (px py pz) (the convolution's prefactor
// and the unnormalized inverse transform, pm_solver.cpp:5207-5222).
template <class R, class C>
__global__ void isoKernelExtractKernel(size_t count, const C* __restrict__ spec, double scale, R* out) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    out[i] = static_cast<R>(static_cast<double>(spec[i].x) * scale);
  }
}

template <class R, class C>
__global__ void isoMultiplyKernel(size_t count, C* spec, const R* __restrict__ kern) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const R k = kern[i];
    C v = spec[i];
    v.x *= k;
    v.y *= k;
    spec[i] = v;
  }
}

// Force = -gradient of the potential: central differences inside, one-sided
// second-order differences on the faces (pm_solver.cpp:5240-5265). Writes the
// force meshes in the periodic layout the interpolation reads.
template <class R>
__global__ void isoGradientKernel(PmGeom g, IsoGeom q, double dx, double dy, double dz, const R* __restrict__ phi,
                                  R* fx, R* fy, R* fz) {
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const size_t total = static_cast<size_t>(nx) * ny * nz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int64_t iz = static_cast<int64_t>(i % nz);
    const int64_t iy = static_cast<int64_t>((i / nz) % ny);
    const int64_t ix = static_cast<int64_t>(i / (static_cast<size_t>(nz) * ny));
    auto P = [&](int64_t a, int64_t b, int64_t c) -> double {
      return static_cast<double>(phi[(static_cast<size_t>(a) * q.py + b) * q.pzp + c]);
    };
    double gx, gy, gz;
    if (ix == 0) gx = (-3.0 * P(0, iy, iz) + 4.0 * P(1, iy, iz) - P(2, iy, iz)) / (2.0 * dx);
    else if (ix + 1 == nx) gx = (3.0 * P(nx - 1, iy, iz) - 4.0 * P(nx - 2, iy, iz) + P(nx - 3, iy, iz)) / (2.0 * dx);
    else gx = (P(ix + 1, iy, iz) - P(ix - 1, iy, iz)) / (2.0 * dx);
    if (iy == 0) gy = (-3.0 * P(ix, 0, iz) + 4.0 * P(ix, 1, iz) - P(ix, 2, iz)) / (2.0 * dy);
    else if (iy + 1 == ny) gy = (3.0 * P(ix, ny - 1, iz) - 4.0 * P(ix, ny - 2, iz) + P(ix, ny - 3, iz)) / (2.0 * dy);
    else gy = (P(ix, iy + 1, iz) - P(ix, iy - 1, iz)) / (2.0 * dy);
    if (iz == 0) gz = (-3.0 * P(ix, iy, 0) + 4.0 * P(ix, iy, 1) - P(ix, iy, 2)) / (2.0 * dz);
    else if (iz + 1 == nz) gz = (3.0 * P(ix, iy, nz - 1) - 4.0 * P(ix, iy, nz - 2) + P(ix, iy, nz - 3)) / (2.0 * dz);
    else gz = (P(ix, iy, iz + 1) - P(ix, iy, iz - 1)) / (2.0 * dz);
    const size_t o = (static_cast<size_t>(ix) * ny + iy) * g.nzp + iz;
    fx[o] = static_cast<R>(-gx);
    fy[o] = static_cast<R>(-gy);
    fz[o] = static_cast<R>(-gz);
  }
}

inline unsigned gridFor(size_t n, int block) {
  size_t b = (n + block - 1) / block;
  if (b > 148u * 32u) b = 148u * 32u;
  return static_cast<unsigned>(b ? b : 1);
}

inline double sincHost(double v) {
  // pm_solver.cpp:121-126
  if (std::fabs(v) < 1.0e-12) return 1.0;
  return std::sin(v) / v;
}

bool isMixed(const Context& c) { return c.cfg.precision == CHUI_TREEPM_MIXED; }

// ---- adjoint (transposes of the PM force map) ----

// Derivatives of the stencil weights with respect to the grid coordinate gp
// (same base cell as makeStencil).
__device__ __forceinline__ Stencil makeStencilGrad(double gp, int scheme) {
  Stencil s;
  if (scheme == 0) {
    s.off0 = static_cast<int64_t>(floor(gp));
    s.w[0] = -1.0;
    s.w[1] = 1.0;
    s.w[2] = 0.0;
  } else {
    const double center = floor(gp + 0.5);
    const double d = gp - center;
    s.off0 = static_cast<int64_t>(center) - 1;
    s.w[0] = -(0.5 - d);
    s.w[1] = -2.0 * d;
    s.w[2] = 0.5 + d;
  }
  return s;
}

// Transpose of the interpolation a_k = sum_c W(x_k - c) F(c) for cotangents
// a_bar: position gradient sum_b a_bar_b sum_c grad W F_b(c) (written to g),
// and the cotangent grids B_b(c) += W(x_k - c) a_bar_b (atomics).
template <class R>
__global__ void pmInterpAdjointKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                      const double* __restrict__ z, const double* __restrict__ cx,
                                      const double* __restrict__ cy, const double* __restrict__ cz, PmGeom g,
                                      const R* __restrict__ f0, const R* __restrict__ f1, const R* __restrict__ f2,
                                      R* b0, R* b1, R* b2, double* gx, double* gy, double* gz) {
  const int taps = g.scheme == 0 ? 2 : 3;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double gp0 = wrapPosition(x[k], g.L[0]) * g.inv_d[0];
    const double gp1 = wrapPosition(y[k], g.L[1]) * g.inv_d[1];
    const double gp2 = wrapPosition(z[k], g.L[2]) * g.inv_d[2];
    const Stencil s0 = makeStencil(gp0, g.scheme), s1 = makeStencil(gp1, g.scheme), s2 = makeStencil(gp2, g.scheme);
    const Stencil d0 = makeStencilGrad(gp0, g.scheme), d1 = makeStencilGrad(gp1, g.scheme),
                  d2 = makeStencilGrad(gp2, g.scheme);
    const double ax = cx[k], ay = cy[k], az = cz[k];
    double ox = 0.0, oy = 0.0, oz = 0.0;
    for (int a = 0; a < taps; ++a) {
      const int64_t ix = wrapIndex(s0.off0 + a, g.n[0]);
      for (int b = 0; b < taps; ++b) {
        const int64_t iy = wrapIndex(s1.off0 + b, g.n[1]);
        const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp;
        for (int cc = 0; cc < taps; ++cc) {
          const int64_t iz = wrapIndex(s2.off0 + cc, g.n[2]);
          const size_t at = row + iz;
          const double dot = ax * static_cast<double>(f0[at]) + ay * static_cast<double>(f1[at]) +
                             az * static_cast<double>(f2[at]);
          ox += d0.w[a] * s1.w[b] * s2.w[cc] * dot;
          oy += s0.w[a] * d1.w[b] * s2.w[cc] * dot;
          oz += s0.w[a] * s1.w[b] * d2.w[cc] * dot;
          const double w = s0.w[a] * s1.w[b] * s2.w[cc];
          atomicAdd(b0 + at, static_cast<R>(w * ax));
          atomicAdd(b1 + at, static_cast<R>(w * ay));
          atomicAdd(b2 + at, static_cast<R>(w * az));
        }
      }
    }
    gx[k] = ox * g.inv_d[0];
    gy[k] = oy * g.inv_d[1];
    gz[k] = oz * g.inv_d[2];
  }
}

// Transpose of the three gradient operators F_b = C2R(-i g_b op R2C(rho)):
// each is a real circulant with an odd kernel, so its transpose is its
// negative and rho_bar = -sum_b C2R(-i g_b op B_b^) = C2R(sum_b i g_b op B_b^).
// Writes that spectrum into c0 (in place of B_0^).
template <class R, class C>
__global__ void pmSpectrumAdjointKernel(PmGeom g, const double* __restrict__ tab, double prefactor, double rs,
                                        int deconv, C* c0, const C* __restrict__ c1, const C* __restrict__ c2) {
  const int64_t nx = g.n[0], ny = g.n[1], nzc = g.nzc;
  const double* kx = tab;
  const double* ky = kx + nx;
  const double* kz = ky + ny;
  const double* wx = kz + nzc;
  const double* wy = wx + nx;
  const double* wz = wy + ny;
  const double* gx = wz + nzc;
  const double* gy = gx + nx;
  const double* gz = gy + ny;
  const size_t total = static_cast<size_t>(nx) * ny * nzc;
  for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int64_t iz = static_cast<int64_t>(idx % nzc);
    const size_t row = idx / nzc;
    const int64_t iy = static_cast<int64_t>(row % ny);
    const int64_t ix = static_cast<int64_t>(row / ny);
    const double k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
    double op = 0.0;
    if (k2 != 0.0) {
      double window = 1.0;
      if (deconv) {
        const double tw = wx[ix] * wy[iy] * wz[iz];
        const double w2 = tw * tw;
        window = 1.0 / (w2 > 1.0e-12 ? w2 : 1.0e-12);
      }
      const double prod = sqrt(k2) * rs;
      op = prefactor * window * exp(-(prod * prod)) / k2;
    }
    const C v0 = c0[idx], v1 = c1[idx], v2 = c2[idx];
    // sum_b g_b (re_b + i im_b) = (sr + i si); times i op -> (-op si, op sr)
    const double sr = gx[ix] * static_cast<double>(v0.x) + gy[iy] * static_cast<double>(v1.x) +
                      gz[iz] * static_cast<double>(v2.x);
    const double si = gx[ix] * static_cast<double>(v0.y) + gy[iy] * static_cast<double>(v1.y) +
                      gz[iz] * static_cast<double>(v2.y);
    C out;
    out.x = static_cast<R>(-op * si);
    out.y = static_cast<R>(op * sr);
    c0[idx] = out;
  }
}

// Transpose of the mass deposit rho(c) = sum_j m_j W(x_j - c) / V_cell:
// g_j += (m_j / V_cell) sum_c rho_bar(c) grad W(x_j - c). The grid's row
// stride is g.nzp (padded FFT layout or compact nz).
template <class R>
__global__ void pmDepositAdjointKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                       const double* __restrict__ z, const double* __restrict__ m,
                                       double uniform_mass, double inv_cell_volume, PmGeom g,
                                       const R* __restrict__ rho_bar, int accumulate, double* gx, double* gy,
                                       double* gz) {
  const int taps = g.scheme == 0 ? 2 : 3;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double gp0 = wrapPosition(x[k], g.L[0]) * g.inv_d[0];
    const double gp1 = wrapPosition(y[k], g.L[1]) * g.inv_d[1];
    const double gp2 = wrapPosition(z[k], g.L[2]) * g.inv_d[2];
    const Stencil s0 = makeStencil(gp0, g.scheme), s1 = makeStencil(gp1, g.scheme), s2 = makeStencil(gp2, g.scheme);
    const Stencil d0 = makeStencilGrad(gp0, g.scheme), d1 = makeStencilGrad(gp1, g.scheme),
                  d2 = makeStencilGrad(gp2, g.scheme);
    double ox = 0.0, oy = 0.0, oz = 0.0;
    for (int a = 0; a < taps; ++a) {
      const int64_t ix = wrapIndex(s0.off0 + a, g.n[0]);
      for (int b = 0; b < taps; ++b) {
        const int64_t iy = wrapIndex(s1.off0 + b, g.n[1]);
        const size_t row = (static_cast<size_t>(ix) * g.n[1] + iy) * g.nzp;
        for (int cc = 0; cc < taps; ++cc) {
          const int64_t iz = wrapIndex(s2.off0 + cc, g.n[2]);
          const double v = static_cast<double>(rho_bar[row + iz]);
          ox += d0.w[a] * s1.w[b] * s2.w[cc] * v;
          oy += s0.w[a] * d1.w[b] * s2.w[cc] * v;
          oz += s0.w[a] * s1.w[b] * d2.w[cc] * v;
        }
      }
    }
    const double f = (m ? m[k] : uniform_mass) * inv_cell_volume;
    ox *= f * g.inv_d[0];
    oy *= f * g.inv_d[1];
    oz *= f * g.inv_d[2];
    if (accumulate) {
      gx[k] += ox;
      gy[k] += oy;
      gz[k] += oz;
    } else {
      gx[k] = ox;
      gy[k] = oy;
      gz[k] = oz;
    }
  }
}

}  // namespace

int pmPrepare(Context& c) {
  if (c.fft_ready) return 0;
  const PmGeom g = geomOf(c);
  const bool mixed = isMixed(c);
  const size_t elem = mixed ? sizeof(float) : sizeof(double);
  const size_t padded = static_cast<size_t>(g.n[0]) * g.n[1] * g.nzp;
  for (auto& b : c.grid) {
    if (ensure(b, padded * elem) != cudaSuccess) {
      c.last_error = "PM mesh allocation failed";
      return CHUI_TREEPM_ENOMEM;
    }
  }
  const int nx = static_cast<int>(g.n[0]), ny = static_cast<int>(g.n[1]), nz = static_cast<int>(g.n[2]);
  if (cufftPlan3d(&c.plan_r2c, nx, ny, nz, mixed ? CUFFT_R2C : CUFFT_D2Z) != CUFFT_SUCCESS ||
      cufftPlan3d(&c.plan_c2r, nx, ny, nz, mixed ? CUFFT_C2R : CUFFT_Z2D) != CUFFT_SUCCESS) {
    c.last_error = "cuFFT plan creation failed";
    return CHUI_TREEPM_EDEVICE;
  }
  // Axis metadata (ensureSpectralAxisMetadata, pm_solver.cpp:2398-2466) plus
  // the gradient wave numbers with the even-axis Nyquist zeroed (:2679-2705).
  std::vector<double> tab;
  const int expo = c.cfg.assignment_scheme == CHUI_TREEPM_CIC ? 2 : 3;
  std::vector<double> k[3], w[3], gk[3];
  for (int a = 0; a < 3; ++a) {
    const int64_t count = a == 2 ? g.nzc : g.n[a];
    const double dk = 2.0 * kPi / g.L[a];
    for (int64_t i = 0; i < count; ++i) {
      const int64_t mode = (a == 2) ? i : (i <= g.n[a] / 2 ? i : i - g.n[a]);
      const double kk = dk * static_cast<double>(mode);
      k[a].push_back(kk);
      w[a].push_back(c.cfg.window_deconvolution
                         ? std::pow(sincHost(0.5 * kk * g.L[a] / static_cast<double>(g.n[a])),
                                    static_cast<double>(expo))
                         : 1.0);
      gk[a].push_back((g.n[a] % 2 == 0 && i == g.n[a] / 2) ? 0.0 : kk);
    }
  }
  for (int a = 0; a < 3; ++a) tab.insert(tab.end(), k[a].begin(), k[a].end());
  for (int a = 0; a < 3; ++a) tab.insert(tab.end(), w[a].begin(), w[a].end());
  for (int a = 0; a < 3; ++a) tab.insert(tab.end(), gk[a].begin(), gk[a].end());
  if (ensure(c.axis_tables, tab.size() * sizeof(double)) != cudaSuccess ||
      cudaMemcpy(c.axis_tables.ptr, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    c.last_error = "PM axis table upload failed";
    return CHUI_TREEPM_EDEVICE;
  }
  c.fft_ready = true;
  return 0;
}

void pmDestroy(Context& c) {
  if (c.plan_r2c) cufftDestroy(c.plan_r2c);
  if (c.plan_c2r) cufftDestroy(c.plan_c2r);
  c.plan_r2c = c.plan_c2r = 0;
  c.fft_ready = false;
  if (c.iso_r2c) cufftDestroy(c.iso_r2c);
  if (c.iso_c2r) cufftDestroy(c.iso_c2r);
  c.iso_r2c = c.iso_c2r = 0;
  c.iso_ready = false;
  release(c.iso_pad);
  release(c.iso_kernel);
  for (auto& b : c.grid) release(b);
  for (auto& b : c.adj_grid) release(b);
  release(c.axis_tables);
}

namespace {

IsoGeom isoGeomOf(const PmGeom& g) {
  IsoGeom q;
  q.px = 2 * g.n[0];
  q.py = 2 * g.n[1];
  q.pz = 2 * g.n[2];
  q.pzp = 2 * (q.pz / 2 + 1);
  return q;
}

// Padded plans, buffers and the Green function's spectrum (computed once per
// configuration, as the reference caches its kernel, pm_solver.cpp:5148-5206).
template <class R, class C>
int isoPrepare(Context& c, const PmGeom& g, cudaStream_t s) {
  if (c.iso_ready) return 0;
  const IsoGeom q = isoGeomOf(g);
  const bool mixed = sizeof(R) == 4;
  const size_t padded = static_cast<size_t>(q.px) * q.py * q.pzp;
  const size_t half = static_cast<size_t>(q.px) * q.py * (q.pz / 2 + 1);
  if (ensure(c.iso_pad, padded * sizeof(R)) != cudaSuccess || ensure(c.iso_kernel, half * sizeof(R)) != cudaSuccess) {
    c.last_error = "isolated PM workspace allocation failed";
    return CHUI_TREEPM_ENOMEM;
  }
  if (cufftPlan3d(&c.iso_r2c, static_cast<int>(q.px), static_cast<int>(q.py), static_cast<int>(q.pz),
                  mixed ? CUFFT_R2C : CUFFT_D2Z) != CUFFT_SUCCESS ||
      cufftPlan3d(&c.iso_c2r, static_cast<int>(q.px), static_cast<int>(q.py), static_cast<int>(q.pz),
                  mixed ? CUFFT_C2R : CUFFT_Z2D) != CUFFT_SUCCESS) {
    c.last_error = "cuFFT plan creation failed (isolated PM)";
    return CHUI_TREEPM_EDEVICE;
  }
  cufftSetStream(c.iso_r2c, s);
  cufftSetStream(c.iso_c2r, s);
  const double dx = g.L[0] / static_cast<double>(g.n[0]), dy = g.L[1] / static_cast<double>(g.n[1]),
               dz = g.L[2] / static_cast<double>(g.n[2]);
  const int block = 256;
  { noteLaunch(); isoKernelFillKernel<R><<<gridFor(static_cast<size_t>(q.px) * q.py * q.pz, block), block, 0, s>>>(
      g, q, dx, dy, dz, c.rs, c.iso_pad.as<R>()); }
  cufftResult fr = mixed ? cufftExecR2C(c.iso_r2c, c.iso_pad.as<cufftReal>(), c.iso_pad.as<cufftComplex>())
                         : cufftExecD2Z(c.iso_r2c, c.iso_pad.as<cufftDoubleReal>(), c.iso_pad.as<cufftDoubleComplex>());
  if (fr != CUFFT_SUCCESS) {
    c.last_error = "cuFFT forward transform failed (isolated PM kernel)";
    return CHUI_TREEPM_EDEVICE;
  }
  const double scale = c.cfg.gravitational_constant * (dx * dy * dz) /
                       (static_cast<double>(q.px) * static_cast<double>(q.py) * static_cast<double>(q.pz));
  { noteLaunch(); isoKernelExtractKernel<R, C><<<gridFor(half, block), block, 0, s>>>(half, c.iso_pad.as<C>(), scale,
                                                                                     c.iso_kernel.as<R>()); }
  c.iso_ready = true;
  return 0;
}

template <class R, class C>
int isoRefresh(Context& c, const PmGeom& g, int64_t n, const double* x, const double* y, const double* z,
               const double* m, double uniform_mass, cudaStream_t s) {
  int rc = isoPrepare<R, C>(c, g, s);
  if (rc) return rc;
  const IsoGeom q = isoGeomOf(g);
  const bool mixed = sizeof(R) == 4;
  const size_t padded = static_cast<size_t>(q.px) * q.py * q.pzp;
  const size_t half = static_cast<size_t>(q.px) * q.py * (q.pz / 2 + 1);
  const double dx = g.L[0] / static_cast<double>(g.n[0]), dy = g.L[1] / static_cast<double>(g.n[1]),
               dz = g.L[2] / static_cast<double>(g.n[2]);
  const int block = 256;
  cufftSetStream(c.iso_r2c, s);
  cufftSetStream(c.iso_c2r, s);
  cudaMemsetAsync(c.iso_pad.ptr, 0, padded * sizeof(R), s);
  if (n > 0)
    { noteLaunch(); depositIsolatedKernel<R><<<gridFor(n, block), block, 0, s>>>(
        n, x, y, z, m, uniform_mass, 1.0 / (dx * dy * dz), g, q, c.iso_pad.as<R>()); }
  cufftResult fr = mixed ? cufftExecR2C(c.iso_r2c, c.iso_pad.as<cufftReal>(), c.iso_pad.as<cufftComplex>())
                         : cufftExecD2Z(c.iso_r2c, c.iso_pad.as<cufftDoubleReal>(), c.iso_pad.as<cufftDoubleComplex>());
  if (fr != CUFFT_SUCCESS) {
    c.last_error = "cuFFT forward transform failed (isolated PM)";
    return CHUI_TREEPM_EDEVICE;
  }
  { noteLaunch(); isoMultiplyKernel<R, C><<<gridFor(half, block), block, 0, s>>>(half, c.iso_pad.as<C>(),
                                                                                c.iso_kernel.as<R>()); }
  fr = mixed ? cufftExecC2R(c.iso_c2r, c.iso_pad.as<cufftComplex>(), c.iso_pad.as<cufftReal>())
             : cufftExecZ2D(c.iso_c2r, c.iso_pad.as<cufftDoubleComplex>(), c.iso_pad.as<cufftDoubleReal>());
  if (fr != CUFFT_SUCCESS) {
    c.last_error = "cuFFT inverse transform failed (isolated PM)";
    return CHUI_TREEPM_EDEVICE;
  }
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  { noteLaunch(); isoGradientKernel<R><<<gridFor(cells, block), block, 0, s>>>(
      g, q, dx, dy, dz, c.iso_pad.as<R>(), c.grid[0].as<R>(), c.grid[1].as<R>(), c.grid[2].as<R>()); }
  return 0;
}

}  // namespace

int pmRefresh(Context& c, int64_t n, const double* x, const double* y, const double* z,
              const double* m, double uniform_mass, double total_mass, cudaStream_t s,
              const double4* tree_sources) {
  c.pm_f4_ready = false;
  int rc = pmPrepare(c);
  if (rc) return rc;
  if (c.cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_PERIODIC) {
    const PmGeom gi = geomOf(c);
    rc = isMixed(c) ? isoRefresh<float, cufftComplex>(c, gi, n, x, y, z, m, uniform_mass, s)
                    : isoRefresh<double, cufftDoubleComplex>(c, gi, n, x, y, z, m, uniform_mass, s);
    if (rc) return rc;
    if (cudaGetLastError() != cudaSuccess) {
      c.last_error = "PM kernel launch failed";
      return CHUI_TREEPM_EDEVICE;
    }
    c.pm_field_valid = true;
    c.pm_field_box[0] = gi.L[0];
    c.pm_field_box[1] = gi.L[1];
    c.pm_field_box[2] = gi.L[2];
    return 0;
  }
  const PmGeom g = geomOf(c);
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  const size_t padded = static_cast<size_t>(g.n[0]) * g.n[1] * g.nzp;
  const double volume = g.L[0] * g.L[1] * g.L[2];
  const double cell_volume = volume / static_cast<double>(cells);
  // Mean subtraction (pm_solver.cpp:4676-4707) folded into the fill value:
  // the mean density is total mass / box volume, which the deposit conserves.
  const double mean = total_mass / volume;
  const bool mixed = isMixed(c);
  const int block = 256;
  if (mixed) {
    { noteLaunch(); fillKernel<float><<<gridFor(padded, block), block, 0, s>>>(c.grid[0].as<float>(), padded,
                                                               static_cast<float>(-mean)); }
    if (n > 0 && tree_sources)
      launchDepositTiled<float>(n, tree_sources, 1.0 / cell_volume, g, c.grid[0].as<float>(), s);
    else if (n > 0)
      { noteLaunch(); depositKernel<float><<<gridFor(n, block), block, 0, s>>>(n, x, y, z, m, uniform_mass,
                                                               1.0 / cell_volume, g, c.grid[0].as<float>()); }
  } else {
    { noteLaunch(); fillKernel<double><<<gridFor(padded, block), block, 0, s>>>(c.grid[0].as<double>(), padded, -mean); }
    if (n > 0 && tree_sources)
      launchDepositTiled<double>(n, tree_sources, 1.0 / cell_volume, g, c.grid[0].as<double>(), s);
    else if (n > 0)
      { noteLaunch(); depositKernel<double><<<gridFor(n, block), block, 0, s>>>(n, x, y, z, m, uniform_mass,
                                                                1.0 / cell_volume, g, c.grid[0].as<double>()); }
  }
  cufftSetStream(c.plan_r2c, s);
  cufftSetStream(c.plan_c2r, s);
  const double prefactor = -4.0 * kPi * c.cfg.gravitational_constant / static_cast<double>(cells);
  const size_t total = static_cast<size_t>(g.n[0]) * g.n[1] * g.nzc;
  cufftResult fr;
  if (mixed) {
    fr = cufftExecR2C(c.plan_r2c, c.grid[0].as<cufftReal>(), c.grid[0].as<cufftComplex>());
    if (fr != CUFFT_SUCCESS) {
      c.last_error = "cuFFT R2C failed";
      return CHUI_TREEPM_EDEVICE;
    }
    { noteLaunch(); greenGradientKernel<float, cufftComplex><<<gridFor(total, block), block, 0, s>>>(
        g, c.axis_tables.as<double>(), prefactor, c.rs, c.cfg.window_deconvolution,
        c.grid[0].as<cufftComplex>(), c.grid[1].as<cufftComplex>(), c.grid[2].as<cufftComplex>()); }
    for (int a = 0; a < 3; ++a) {
      fr = cufftExecC2R(c.plan_c2r, c.grid[a].as<cufftComplex>(), c.grid[a].as<cufftReal>());
      if (fr != CUFFT_SUCCESS) {
        c.last_error = "cuFFT C2R failed";
        return CHUI_TREEPM_EDEVICE;
      }
    }
    // the interpolation's interleaved copy of the field
    if (ensure(c.grid_f4, cells * sizeof(float4))) {
      c.last_error = "PM interleaved field allocation failed";
      return CHUI_TREEPM_ENOMEM;
    }
    { noteLaunch(); interleaveForceKernel<<<gridFor(cells, block), block, 0, s>>>(
        g, c.grid[0].as<float>(), c.grid[1].as<float>(), c.grid[2].as<float>(), c.grid_f4.as<float4>()); }
    c.pm_f4_ready = true;
  } else {
    fr = cufftExecD2Z(c.plan_r2c, c.grid[0].as<cufftDoubleReal>(), c.grid[0].as<cufftDoubleComplex>());
    if (fr != CUFFT_SUCCESS) {
      c.last_error = "cuFFT D2Z failed";
      return CHUI_TREEPM_EDEVICE;
    }
    { noteLaunch(); greenGradientKernel<double, cufftDoubleComplex><<<gridFor(total, block), block, 0, s>>>(
        g, c.axis_tables.as<double>(), prefactor, c.rs, c.cfg.window_deconvolution,
        c.grid[0].as<cufftDoubleComplex>(), c.grid[1].as<cufftDoubleComplex>(),
        c.grid[2].as<cufftDoubleComplex>()); }
    for (int a = 0; a < 3; ++a) {
      fr = cufftExecZ2D(c.plan_c2r, c.grid[a].as<cufftDoubleComplex>(), c.grid[a].as<cufftDoubleReal>());
      if (fr != CUFFT_SUCCESS) {
        c.last_error = "cuFFT Z2D failed";
        return CHUI_TREEPM_EDEVICE;
      }
    }
  }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM kernel launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  c.pm_field_valid = true;
  c.pm_field_box[0] = g.L[0];
  c.pm_field_box[1] = g.L[1];
  c.pm_field_box[2] = g.L[2];
  return 0;
}

int pmInterpolate(Context& c, int64_t nt, const uint32_t* active, const double* tx,
                  const double* ty, const double* tz, const double* sx, const double* sy,
                  const double* sz, double* ax, double* ay, double* az, cudaStream_t s,
                  const uint32_t* order) {
  if (nt == 0) return 0;
  const PmGeom g = geomOf(c);
  const int block = 256;
  if (isMixed(c)) {
    { noteLaunch(); interpolateKernel<float><<<gridFor(nt, block), block, 0, s>>>(
        nt, order, active, tx, ty, tz, sx, sy, sz, g, c.grid[0].as<float>(), c.grid[1].as<float>(),
        c.grid[2].as<float>(), c.pm_f4_ready ? c.grid_f4.as<float4>() : nullptr, ax, ay, az); }
  } else {
    { noteLaunch(); interpolateKernel<double><<<gridFor(nt, block), block, 0, s>>>(
        nt, order, active, tx, ty, tz, sx, sy, sz, g, c.grid[0].as<double>(), c.grid[1].as<double>(),
        c.grid[2].as<double>(), nullptr, ax, ay, az); }
  }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM interpolation launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

int pmInterpolateCombine(Context& c, int64_t nt, const uint32_t* active, const double* tx, const double* ty,
                         const double* tz, int64_t n, const double* px, const double* py, const double* pz,
                         bool with_pm, const double* tree, const double* near, double* ax, double* ay, double* az,
                         double* lx, double* ly, double* lz, double* sx, double* sy, double* sz, double* snear,
                         cudaStream_t s) {
  if (nt == 0) return 0;
  const PmGeom g = geomOf(c);
  const int block = 256;
  if (isMixed(c)) {
    { noteLaunch(); interpolateCombineKernel<float><<<gridFor(nt, block), block, 0, s>>>(
        nt, active, tx, ty, tz, n, px, py, pz, g, c.grid[0].as<float>(), c.grid[1].as<float>(),
        c.grid[2].as<float>(), c.pm_f4_ready ? c.grid_f4.as<float4>() : nullptr, with_pm ? 1 : 0, tree, near, ax, ay, az, lx, ly, lz, sx, sy, sz, snear); }
  } else {
    { noteLaunch(); interpolateCombineKernel<double><<<gridFor(nt, block), block, 0, s>>>(
        nt, active, tx, ty, tz, n, px, py, pz, g, c.grid[0].as<double>(), c.grid[1].as<double>(),
        c.grid[2].as<double>(), nullptr, with_pm ? 1 : 0, tree, near, ax, ay, az, lx, ly, lz, sx, sy, sz, snear); }
  }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM interpolation launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

int pmDensityOnly(Context& c, int64_t n, const double* x, const double* y, const double* z,
                  const double* m, double uniform_mass, double* rho, cudaStream_t s) {
  const PmGeom g = geomOf(c);
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  const int block = 256;
  if (cudaMemsetAsync(rho, 0, cells * sizeof(double), s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  if (n > 0)
    { noteLaunch(); depositCompactKernel<<<gridFor(n, block), block, 0, s>>>(n, x, y, z, m, uniform_mass, g, rho); }
  const double cell_volume = (g.L[0] * g.L[1] * g.L[2]) / static_cast<double>(cells);
  { noteLaunch(); scaleKernel<<<gridFor(cells, block), block, 0, s>>>(rho, cells, cell_volume); }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM density launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

// Density into a caller-provided compact FP64 grid, with no allocation (the
// allocation-free entry point): zero the grid, deposit, divide by the cell
// volume. Same kernels and arithmetic as pmDensityOnly.
int pmDensityInto(const chui_treepm_config& cfg, int64_t n, const double* x, const double* y, const double* z,
                  const double* m, double uniform_mass, double* rho, cudaStream_t s) {
  PmGeom g;
  g.n[0] = cfg.pm_grid_nx;
  g.n[1] = cfg.pm_grid_ny;
  g.n[2] = cfg.pm_grid_nz;
  g.nzc = g.n[2] / 2 + 1;
  g.nzp = 2 * g.nzc;
  g.L[0] = cfg.box_x;
  g.L[1] = cfg.box_y;
  g.L[2] = cfg.box_z;
  for (int a = 0; a < 3; ++a) g.inv_d[a] = static_cast<double>(g.n[a]) / g.L[a];
  g.scheme = cfg.assignment_scheme;
  g.periodic = cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_PERIODIC ? 1 : 0;
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  const int block = 256;
  if (cudaMemsetAsync(rho, 0, cells * sizeof(double), s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  if (n > 0)
    { noteLaunch(); depositCompactKernel<<<gridFor(n, block), block, 0, s>>>(n, x, y, z, m, uniform_mass, g, rho); }
  const double cell_volume = (g.L[0] * g.L[1] * g.L[2]) / static_cast<double>(cells);
  { noteLaunch(); scaleKernel<<<gridFor(cells, block), block, 0, s>>>(rho, cells, cell_volume); }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

// PM part of the force VJP at positions (x, y, z): refreshes the PM field at
// these positions, then g = J_pm^T a_bar (written, not accumulated).
int pmForceVjp(Context& c, int64_t n, const double* x, const double* y, const double* z, const double* m,
               double uniform_mass, double total_mass, const double* cx, const double* cy, const double* cz,
               double* gx, double* gy, double* gz, cudaStream_t s, const double4* tree_sources) {
  int rc = pmRefresh(c, n, x, y, z, m, uniform_mass, total_mass, s, tree_sources);
  if (rc) return rc;
  if (n == 0) return 0;
  const PmGeom g = geomOf(c);
  const bool mixed = isMixed(c);
  const size_t elem = mixed ? sizeof(float) : sizeof(double);
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  const size_t padded = static_cast<size_t>(g.n[0]) * g.n[1] * g.nzp;
  const size_t total = static_cast<size_t>(g.n[0]) * g.n[1] * g.nzc;
  const double cell_volume = (g.L[0] * g.L[1] * g.L[2]) / static_cast<double>(cells);
  const double prefactor = -4.0 * kPi * c.cfg.gravitational_constant / static_cast<double>(cells);
  for (auto& b : c.adj_grid) {
    if (ensure(b, padded * elem) != cudaSuccess) {
      c.last_error = "PM adjoint mesh allocation failed";
      return CHUI_TREEPM_ENOMEM;
    }
    cudaMemsetAsync(b.ptr, 0, padded * elem, s);
  }
  const int block = 256;
  cufftSetStream(c.plan_r2c, s);
  cufftSetStream(c.plan_c2r, s);
  cufftResult fr = CUFFT_SUCCESS;
  if (mixed) {
    { noteLaunch(); pmInterpAdjointKernel<float><<<gridFor(n, block), block, 0, s>>>(
        n, x, y, z, cx, cy, cz, g, c.grid[0].as<float>(), c.grid[1].as<float>(), c.grid[2].as<float>(),
        c.adj_grid[0].as<float>(), c.adj_grid[1].as<float>(), c.adj_grid[2].as<float>(), gx, gy, gz); }
    for (int a = 0; a < 3 && fr == CUFFT_SUCCESS; ++a)
      fr = cufftExecR2C(c.plan_r2c, c.adj_grid[a].as<cufftReal>(), c.adj_grid[a].as<cufftComplex>());
    if (fr == CUFFT_SUCCESS) {
      { noteLaunch(); pmSpectrumAdjointKernel<float, cufftComplex><<<gridFor(total, block), block, 0, s>>>(
          g, c.axis_tables.as<double>(), prefactor, c.rs, c.cfg.window_deconvolution,
          c.adj_grid[0].as<cufftComplex>(), c.adj_grid[1].as<cufftComplex>(), c.adj_grid[2].as<cufftComplex>()); }
      fr = cufftExecC2R(c.plan_c2r, c.adj_grid[0].as<cufftComplex>(), c.adj_grid[0].as<cufftReal>());
    }
    if (fr == CUFFT_SUCCESS)
      { noteLaunch(); pmDepositAdjointKernel<float><<<gridFor(n, block), block, 0, s>>>(
          n, x, y, z, m, uniform_mass, 1.0 / cell_volume, g, c.adj_grid[0].as<float>(), 1, gx, gy, gz); }
  } else {
    { noteLaunch(); pmInterpAdjointKernel<double><<<gridFor(n, block), block, 0, s>>>(
        n, x, y, z, cx, cy, cz, g, c.grid[0].as<double>(), c.grid[1].as<double>(), c.grid[2].as<double>(),
        c.adj_grid[0].as<double>(), c.adj_grid[1].as<double>(), c.adj_grid[2].as<double>(), gx, gy, gz); }
    for (int a = 0; a < 3 && fr == CUFFT_SUCCESS; ++a)
      fr = cufftExecD2Z(c.plan_r2c, c.adj_grid[a].as<cufftDoubleReal>(), c.adj_grid[a].as<cufftDoubleComplex>());
    if (fr == CUFFT_SUCCESS) {
      { noteLaunch(); pmSpectrumAdjointKernel<double, cufftDoubleComplex><<<gridFor(total, block), block, 0, s>>>(
          g, c.axis_tables.as<double>(), prefactor, c.rs, c.cfg.window_deconvolution,
          c.adj_grid[0].as<cufftDoubleComplex>(), c.adj_grid[1].as<cufftDoubleComplex>(),
          c.adj_grid[2].as<cufftDoubleComplex>()); }
      fr = cufftExecZ2D(c.plan_c2r, c.adj_grid[0].as<cufftDoubleComplex>(), c.adj_grid[0].as<cufftDoubleReal>());
    }
    if (fr == CUFFT_SUCCESS)
      { noteLaunch(); pmDepositAdjointKernel<double><<<gridFor(n, block), block, 0, s>>>(
          n, x, y, z, m, uniform_mass, 1.0 / cell_volume, g, c.adj_grid[0].as<double>(), 1, gx, gy, gz); }
  }
  if (fr != CUFFT_SUCCESS) {
    c.last_error = "cuFFT failed in the PM adjoint";
    return CHUI_TREEPM_EDEVICE;
  }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM adjoint launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

// Transpose of the density (mass / cell volume, compact FP64 grid):
// g_j = (m_j / V_cell) sum_c rho_bar(c) grad W(x_j - c).
int pmDensityVjp(Context& c, int64_t n, const double* x, const double* y, const double* z, const double* m,
                 double uniform_mass, const double* rho_bar, double* gx, double* gy, double* gz, cudaStream_t s) {
  if (n == 0) return 0;
  PmGeom g = geomOf(c);
  g.nzp = g.n[2];  // compact rows
  const size_t cells = static_cast<size_t>(g.n[0]) * g.n[1] * g.n[2];
  const double cell_volume = (g.L[0] * g.L[1] * g.L[2]) / static_cast<double>(cells);
  { noteLaunch(); pmDepositAdjointKernel<double><<<gridFor(n, 256), 256, 0, s>>>(
      n, x, y, z, m, uniform_mass, 1.0 / cell_volume, g, rho_bar, 0, gx, gy, gz); }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM density adjoint launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

int pmCells(Context& c, int64_t n, const double* x, const double* y, const double* z,
            int64_t* cells, cudaStream_t s) {
  const PmGeom g = geomOf(c);
  if (n > 0) { noteLaunch(); cellsKernel<<<gridFor(n, 256), 256, 0, s>>>(n, x, y, z, g, cells); }
  if (cudaGetLastError() != cudaSuccess) {
    c.last_error = "PM cell launch failed";
    return CHUI_TREEPM_EDEVICE;
  }
  return 0;
}

}  // namespace chui
