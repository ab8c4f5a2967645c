// C-ABI of the B200 TreePM solver (include/chui_treepm.h): context lifecycle,
// input validation with the reference's error semantics, host/device staging,
// and the orchestration of one solve (TreePmCoordinator::solveActiveSetWithPmCadence,
// tree_pm_coupling.cpp:2282-3518): PM refresh -> periodic tree build ->
// residual walk -> PM interpolation -> accumulation.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "context.cuh"

namespace chui {

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (bytes <= b.bytes && b.ptr) return cudaSuccess;
  if (b.ptr) cudaFree(b.ptr);
  b.ptr = nullptr;
  b.bytes = 0;
  const size_t want = bytes ? bytes : 16;
  cudaError_t e = cudaMalloc(&b.ptr, want);
  if (e == cudaSuccess) b.bytes = want;
  return e;
}

void release(DevBuf& b) {
  if (b.ptr) cudaFree(b.ptr);
  b.ptr = nullptr;
  b.bytes = 0;
}

namespace {
std::atomic<uint64_t> g_launches{0};
}
void noteLaunch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launchCount() { return g_launches.load(std::memory_order_relaxed); }

const char* statusText(uint32_t bits) {
  if (bits & kStatusStackOverflow) return "TreePM residual traversal stack overflow";
  if (bits & kStatusDepthExceeded) return "Tree gravity maximum depth contract exceeded";
  if (bits & kStatusNonFinite) return "TreePM sources require finite coordinates and finite non-negative masses";
  if (bits & kStatusNegativeMass) return "TreePM sources require finite coordinates and finite non-negative masses";
  if (bits & kStatusIndexRange) return "TreePM active index exceeds particle count";
  return "";
}

namespace {

inline unsigned gridFor(size_t n, int block) {
  size_t b = (n + block - 1) / block;
  if (b > 148u * 32u) b = 148u * 32u;
  return static_cast<unsigned>(b ? b : 1);
}

// min/max per axis, finiteness, non-negative mass and mass sum in one pass.
__global__ void sourceReduceKernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                   const double* __restrict__ z, const double* __restrict__ m,
                                   unsigned long long* out, double* mass_sum, uint32_t* status) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double msum = 0.0, mlo = INFINITY, mhi = -INFINITY;
  uint32_t bad = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double p[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      if (!isfinite(p[a])) bad |= kStatusNonFinite;
      lo[a] = fmin(lo[a], p[a]);
      hi[a] = fmax(hi[a], p[a]);
    }
    if (m) {
      const double mi = m[i];
      if (!isfinite(mi)) bad |= kStatusNonFinite;
      if (mi < 0.0) bad |= kStatusNegativeMass;
      msum += mi;
      mlo = fmin(mlo, mi);
      mhi = fmax(mhi, mi);
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    msum += __shfl_xor_sync(0xffffffffu, msum, off);
    mlo = fmin(mlo, __shfl_xor_sync(0xffffffffu, mlo, off));
    mhi = fmax(mhi, __shfl_xor_sync(0xffffffffu, mhi, off));
    bad |= __shfl_xor_sync(0xffffffffu, bad, off);
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(out + a, orderedBits(lo[a]));
      atomicMax(out + 3 + a, orderedBits(hi[a]));
    }
    if (m) {
      atomicAdd(mass_sum, msum);
      atomicMin(out + 8, orderedBits(mlo));
      atomicMax(out + 9, orderedBits(mhi));
    }
    if (bad) atomicOr(status, bad);
  }
}

__global__ void activeCheckKernel(int64_t nt, const uint32_t* __restrict__ active, int64_t n, int explicit_targets,
                                  uint32_t* status) {
  uint32_t bad = 0;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nt;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t r = active[k];
    if (r >= n && !(explicit_targets && r == kInvalid)) bad = kStatusIndexRange;
  }
  if (bad) atomicOr(status, bad);
}

// Softening lanes must be finite and non-negative
// (validateTreePmPreflight, tree_pm_coupling.cpp:440-449).
__global__ void softeningCheckKernel(int64_t n, const double* __restrict__ eps, uint32_t* status) {
  uint32_t bad = 0;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double e = eps[k];
    if (!(isfinite(e) && e >= 0.0)) bad = kStatusNonFinite;
  }
  if (bad) atomicOr(status, bad);
}

// accel = PM + tree (active order); optional source-indexed tree-only and
// nearest-pair lanes (TreePmForceAccumulatorView::addShortRangeToActiveSlot and
// noteNearestPairToActiveSlot, tree_pm_coupling.cpp:1961-1978).
// Total = PM + tree per target. Over all nt slots (order == nullptr), or over
// the count targets of a visit-order slice, whose PM and tree parts and
// outputs are all compact (entry j is slot order[j]; long_range copies too).
__global__ void combineKernel(int64_t count, const uint32_t* __restrict__ order, int64_t nt,
                              const uint32_t* __restrict__ active, int64_t n,
                              const double* __restrict__ pmx, const double* __restrict__ pmy,
                              const double* __restrict__ pmz, const double* __restrict__ tr,
                              const double* __restrict__ near, double* ax, double* ay, double* az,
                              double* lx, double* ly, double* lz,
                              double* sx, double* sy, double* sz, double* snear) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < count;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = order ? static_cast<int64_t>(order[j]) : j;
    const double tx = tr[j], ty = tr[nt + j], tz = tr[2 * nt + j];
    const double px = pmx ? pmx[j] : 0.0, py = pmy ? pmy[j] : 0.0, pz = pmz ? pmz[j] : 0.0;
    ax[j] = px + tx;
    ay[j] = py + ty;
    az[j] = pz + tz;
    if (lx) {
      lx[j] = px;
      ly[j] = py;
      lz[j] = pz;
    }
    const uint32_t row = active ? active[k] : static_cast<uint32_t>(k);
    if (row < n) {
      if (sx) {
        sx[row] = tx;
        sy[row] = ty;
        sz[row] = tz;
      }
      if (snear) snear[row] = near[j];
    }
  }
}

// applyPeculiarVelocityKick (src/workflows/gravity_runtime.cpp:3043-3059).
__global__ void kickKernel(int64_t n, double* vx, double* vy, double* vz, const double* __restrict__ ax,
                           const double* __restrict__ ay, const double* __restrict__ az, double kick, double drag) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    vx[i] = fma(kick, ax[i], drag * vx[i]);
    vy[i] = fma(kick, ay[i], drag * vy[i]);
    vz[i] = fma(kick, az[i], drag * vz[i]);
  }
}

// FP64 global checks: out = {sum m v (3), sum m a (3), sum m v^2 / 2, sum m}.
// Block partial sums in FP64, one atomicAdd per block and quantity.
__global__ void momentumEnergyKernel(int64_t n, const double* __restrict__ m, double uniform_mass,
                                     const double* __restrict__ vx, const double* __restrict__ vy,
                                     const double* __restrict__ vz, const double* __restrict__ ax,
                                     const double* __restrict__ ay, const double* __restrict__ az, double* out) {
  double q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double mi = m ? m[i] : uniform_mass;
    const double u[3] = {vx[i], vy[i], vz[i]};
    q[0] += mi * u[0];
    q[1] += mi * u[1];
    q[2] += mi * u[2];
    if (ax) {
      q[3] += mi * ax[i];
      q[4] += mi * ay[i];
      q[5] += mi * az[i];
    }
    q[6] += 0.5 * mi * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    q[7] += mi;
  }
  __shared__ double part[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 8; ++k) {
    for (int off = 16; off > 0; off >>= 1) q[k] += __shfl_xor_sync(0xffffffffu, q[k], off);
    if (lane == 0) part[k][warp] = q[k];
  }
  __syncthreads();
  if (warp == 0) {
    const int warps = blockDim.x >> 5;
    for (int k = 0; k < 8; ++k) {
      double v = lane < warps ? part[k][lane] : 0.0;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) atomicAdd(out + k, v);
    }
  }
}

// g += t (the short-range part of the force VJP onto the PM part).
__global__ void addKernel(int64_t n, double* gx, double* gy, double* gz, const double* __restrict__ t) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    gx[i] += t[i];
    gy[i] += t[n + i];
    gz[i] += t[2 * n + i];
  }
}

// Transpose of one KDK step (kick K1 with drag1, drift D, kick K2 with drag2)
// applied after the force VJP g at the step's end positions:
//   x_bar += g;  vh_bar = drag2 v_bar + D x_bar;  v_bar = drag1 vh_bar;
//   a_bar = K1 vh_bar (+ K2 v_bar from the previous step's closing kick,
//   which acts at the same positions, unless this is the first step).
__global__ void kdkAdjointKernel(int64_t n, const double* __restrict__ gx, const double* __restrict__ gy,
                                 const double* __restrict__ gz, double* xb, double* yb, double* zb, double* vxb,
                                 double* vyb, double* vzb, double* axb, double* ayb, double* azb, double D,
                                 double K1, double K2, double drag1, double drag2, int first_step) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double px = xb[i] + gx[i], py = yb[i] + gy[i], pz = zb[i] + gz[i];
    const double hx = fma(D, px, drag2 * vxb[i]);
    const double hy = fma(D, py, drag2 * vyb[i]);
    const double hz = fma(D, pz, drag2 * vzb[i]);
    const double vx = drag1 * hx, vy = drag1 * hy, vz = drag1 * hz;
    xb[i] = px;
    yb[i] = py;
    zb[i] = pz;
    vxb[i] = vx;
    vyb[i] = vy;
    vzb[i] = vz;
    const double k2 = first_step ? 0.0 : K2;
    axb[i] = fma(K1, hx, k2 * vx);
    ayb[i] = fma(K1, hy, k2 * vy);
    azb[i] = fma(K1, hz, k2 * vz);
  }
}

// Drift + core::canonicalPeriodicPosition (include/cosmosim/core/periodic_domain.hpp:8-16;
// src/workflows/reference_runtime_composition.cpp:76-107).
__device__ __forceinline__ double canonicalPosition(double v, double box) {
  double w = fmod(v, box);
  if (w < 0.0) w += box;
  if (!(w < box)) w = 0.0;
  return w;
}

__global__ void driftKernel(int64_t n, double* x, double* y, double* z, const double* __restrict__ vx,
                            const double* __restrict__ vy, const double* __restrict__ vz, double drift,
                            double bx, double by, double bz) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // box lengths 0: isolated/open boundaries, positions are not wrapped
    const double nx = fma(vx[i], drift, x[i]), ny = fma(vy[i], drift, y[i]), nz = fma(vz[i], drift, z[i]);
    x[i] = bx > 0.0 ? canonicalPosition(nx, bx) : nx;
    y[i] = by > 0.0 ? canonicalPosition(ny, by) : ny;
    z[i] = bz > 0.0 ? canonicalPosition(nz, bz) : nz;
  }
}

// ---- Gaussian long-range coefficient polynomial (host) ----------------------

double hostH(double t) {
  // H(t) = L(sqrt t)/t^(3/2) (tree_pm_split_kernel.hpp:109-116 and :90-107)
  const double c = 2.25675833419102514779231780624309034;
  if (t < 0.015625) {
    return c * (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
                t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
  }
  const double q = std::sqrt(t);
  return (std::erf(q) - 0.5 * c * q * std::exp(-t)) / (t * q);
}

// H'(t) (the adjoint's kernel derivative): Taylor series below t = 1, closed
// form above (see residualDerivOverR).
double hostHp(double t) {
  if (t < 1.0) {
    double sum = 0.0, term = 1.0;
    for (int k = 0; k <= 20; ++k) {
      const double v = term / (2.0 * k + 5.0);
      sum += (k & 1) ? v : -v;
      term *= t / (k + 1.0);
    }
    return 2.25675833419102514779231780624309034 * sum;
  }
  const double q = std::sqrt(t);
  const double e = std::exp(-t);
  const double L = std::erf(q) - 1.12837916709551257389615890312154517 * q * e;
  return 1.12837916709551257389615890312154517 * e / t - 1.5 * L / (t * t * q);
}

// H''(t): Taylor series (4/sqrt(pi)) sum_k (-1)^k t^k / (k! (2k+7)) below
// t = 1, closed form -(2/sqrt(pi)) e^{-t} (1/t + 2.5/t^2) + 3.75 L(sqrt t) / t^{7/2}
// above (the derivative of H'(t) above).
double hostHpp(double t) {
  if (t < 1.0) {
    double sum = 0.0, term = 1.0;
    for (int k = 0; k <= 20; ++k) {
      const double v = term / (2.0 * k + 7.0);
      sum += (k & 1) ? -v : v;
      term *= t / (k + 1.0);
    }
    return 2.25675833419102514779231780624309034 * sum;
  }
  const double q = std::sqrt(t);
  const double e = std::exp(-t);
  const double L = std::erf(q) - 1.12837916709551257389615890312154517 * q * e;
  return -1.12837916709551257389615890312154517 * e * (1.0 / t + 2.5 / (t * t)) + 3.75 * L / (t * t * t * q);
}

// Chebyshev interpolation of f on [0, t_cut] rewritten as a polynomial in
// s = t * 2 / t_cut - 1 (FP32 coefficients).
template <class F>
PolyH fitChebyshev(F func, double t_cut, double tolerance = 2.0e-6, int short_terms = 12) {
  PolyH best;
  best.max_rel_error = 1e300;
  // The kernels evaluate a short form (`short_terms`) or kPolyMaxTerms terms
  // (unused high coefficients are zero); try the short one first.
  for (int deg : {short_terms - 1, kPolyMaxTerms - 1}) {
    const int m = deg + 1;
    std::vector<double> f(m), cheb(m, 0.0);
    const double pi = 3.141592653589793238462643383279502884;
    for (int k = 0; k < m; ++k) {
      const double xk = std::cos(pi * (k + 0.5) / m);
      f[k] = func((xk + 1.0) * 0.5 * t_cut);
    }
    for (int j = 0; j < m; ++j) {
      double sum = 0.0;
      for (int k = 0; k < m; ++k) sum += f[k] * std::cos(pi * j * (k + 0.5) / m);
      cheb[j] = (j == 0 ? 1.0 : 2.0) * sum / m;
    }
    // Chebyshev -> monomial in s
    std::vector<double> mono(m, 0.0), tkm1(m, 0.0), tk(m, 0.0), tkp1(m, 0.0);
    tkm1[0] = 1.0;
    if (m > 1) tk[1] = 1.0;
    for (int i = 0; i < m; ++i) mono[i] += cheb[0] * tkm1[i];
    if (m > 1)
      for (int i = 0; i < m; ++i) mono[i] += cheb[1] * tk[i];
    for (int j = 2; j < m; ++j) {
      std::fill(tkp1.begin(), tkp1.end(), 0.0);
      for (int i = 0; i < m; ++i) {
        if (i + 1 < m) tkp1[i + 1] += 2.0 * tk[i];
        tkp1[i] -= tkm1[i];
      }
      for (int i = 0; i < m; ++i) mono[i] += cheb[j] * tkp1[i];
      tkm1 = tk;
      tk = tkp1;
    }
    PolyH p;
    p.terms = m;
    p.scale = static_cast<float>(2.0 / t_cut);
    for (int i = 0; i < m; ++i) p.c[i] = static_cast<float>(mono[i]);
    double err = 0.0;
    for (int k = 0; k <= 4000; ++k) {
      const double t = t_cut * k / 4000.0;
      const float s = std::fmaf(static_cast<float>(t), p.scale, -1.0f);
      float h = p.c[m - 1];
      for (int i = m - 2; i >= 0; --i) h = std::fmaf(h, s, p.c[i]);
      const double ref = func(t);
      err = std::max(err, std::fabs(static_cast<double>(h) - ref) / std::fabs(ref));
    }
    p.max_rel_error = err;
    if (err < best.max_rel_error) best = p;
    if (err < tolerance) break;
  }
  return best;
}

// H for the pair kernel: 9 terms (2.9e-5 relative at r_cut/r_s = 5) keep
// FMAs out of the issue-bound walk; at 256^3 the forces then differ from the
// FP64 solve by median 2.5e-7, p99 3.0e-6 (10 terms: 1.9e-7, 2.0e-6);
// configurations the short form cannot fit take the long one.
#ifndef CHUI_PAIR_TOLERANCE
#define CHUI_PAIR_TOLERANCE 5.0e-5
#endif
PolyH fitPoly(double t_cut) { return fitChebyshev(hostH, t_cut, CHUI_PAIR_TOLERANCE, kPairPolyTerms); }

int fail(Context& c, int code, const std::string& msg) {
  c.last_error = msg;
  return code;
}

int validateConfig(const chui_treepm_config& cfg, std::string& err) {
  if (cfg.pm_grid_nx <= 0 || cfg.pm_grid_ny <= 0 || cfg.pm_grid_nz <= 0) {
    err = "numerics.treepm_pm_grid_n{xyz} must all be > 0";
    return CHUI_TREEPM_EINVAL;
  }
  if (!(std::isfinite(cfg.box_x) && std::isfinite(cfg.box_y) && std::isfinite(cfg.box_z)) || cfg.box_x <= 0 ||
      cfg.box_y <= 0 || cfg.box_z <= 0 || !std::isfinite(cfg.gravitational_constant) ||
      cfg.gravitational_constant <= 0) {
    err = "TreePM requires finite positive box axes, scale factor, and gravitational constants";
    return CHUI_TREEPM_EINVAL;
  }
  if (!std::isfinite(cfg.asmth_cells) || cfg.asmth_cells <= 0) {
    err = "TreePM asmth_cells must be > 0";
    return CHUI_TREEPM_EINVAL;
  }
  if (!std::isfinite(cfg.rcut_cells) || cfg.rcut_cells <= 0) {
    err = "TreePM rcut_cells must be > 0";
    return CHUI_TREEPM_EINVAL;
  }
  if (!std::isfinite(cfg.opening_theta) || cfg.opening_theta <= 0 || cfg.max_leaf_size <= 0 ||
      !std::isfinite(cfg.softening) || cfg.softening < 0 ||
      (cfg.opening_criterion < 0 || cfg.opening_criterion > 2) ||
      (cfg.multipole_order != 0 && cfg.multipole_order != 2)) {
    err = "TreePM tree options are invalid";
    return CHUI_TREEPM_EINVAL;
  }
  if (cfg.assignment_scheme != CHUI_TREEPM_CIC && cfg.assignment_scheme != CHUI_TREEPM_TSC) {
    err = "TreePM PM assignment scheme is invalid";
    return CHUI_TREEPM_EINVAL;
  }
  // validateTreePmOptions (tree_pm_coupling.cpp:300-340)
  if (!std::isfinite(cfg.relative_force_tolerance) || cfg.relative_force_tolerance <= 0.0 ||
      !std::isfinite(cfg.relative_force_acceleration_floor) || cfg.relative_force_acceleration_floor <= 0.0 ||
      !std::isfinite(cfg.adaptive_maximum_opening_angle) || cfg.adaptive_maximum_opening_angle <= 0.0 ||
      cfg.adaptive_maximum_opening_angle > 1.0) {
    err = "TreePM tree options are invalid";
    return CHUI_TREEPM_EINVAL;
  }
  if (cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_PERIODIC &&
      cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_ISOLATED_OPEN) {
    err = "TreePM PM boundary condition is invalid";
    return CHUI_TREEPM_EINVAL;
  }
  if (cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_ISOLATED_OPEN) {
    // validatePmSolveOptions (pm_solver.cpp:1664-1667) and solvePoissonIsolatedOpen (:5069-5071)
    if (cfg.window_deconvolution) {
      err = "isolated PM currently does not support window deconvolution";
      return CHUI_TREEPM_EINVAL;
    }
    if (cfg.pm_grid_nx < 3 || cfg.pm_grid_ny < 3 || cfg.pm_grid_nz < 3) {
      err = "PmSolver::solvePoissonIsolatedOpen requires nx,ny,nz >= 3 for one-sided boundary gradients";
      return CHUI_TREEPM_EINVAL;
    }
  }
  if (cfg.diagnostics < 0 || cfg.diagnostics > 2) {
    err = "diagnostics must be 0 (production walk), 1 (the reference's per-node walk and counters) or 2 "
          "(production walk with its own counters and the nearest-pair lane)";
    return CHUI_TREEPM_EINVAL;
  }
  if (cfg.acceptance_policy != CHUI_TREEPM_POLICY_STRICT && cfg.acceptance_policy != CHUI_TREEPM_POLICY_ADAPTIVE) {
    err = "TreePM acceptance policy is invalid";
    return CHUI_TREEPM_EINVAL;
  }
  if ((cfg.adaptive_error_estimator != CHUI_TREEPM_ESTIMATOR_RESIDUAL_DERIVATIVE &&
       cfg.adaptive_error_estimator != CHUI_TREEPM_ESTIMATOR_RELATIVE_MONOPOLE) ||
      (cfg.cutoff_node_policy != CHUI_TREEPM_CUTOFF_CONTAIN_NODE &&
       cfg.cutoff_node_policy != CHUI_TREEPM_CUTOFF_COM_DISTANCE)) {
    err = "TreePM adaptive estimator or cutoff-node policy is invalid";
    return CHUI_TREEPM_EINVAL;
  }
  if (cfg.precision != CHUI_TREEPM_MIXED && cfg.precision != CHUI_TREEPM_FP64) {
    err = "precision must be CHUI_TREEPM_MIXED or CHUI_TREEPM_FP64";
    return CHUI_TREEPM_EINVAL;
  }
  const double spacing = std::cbrt((cfg.box_x / cfg.pm_grid_nx) * (cfg.box_y / cfg.pm_grid_ny) *
                                   (cfg.box_z / cfg.pm_grid_nz));
  const double cutoff = cfg.rcut_cells * spacing;
  const double half_short = 0.5 * std::min({cfg.box_x, cfg.box_y, cfg.box_z});
  if (cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_PERIODIC && cutoff >= std::nextafter(half_short, 0.0)) {
    err = "Periodic TreePM requires cutoff_radius_comoving < half the shortest box axis; cutoff_radius_comoving=" +
          std::to_string(cutoff) + ", half_shortest_axis=" + std::to_string(half_short) +
          "; the short-range tree evaluates one minimum image per source";
    return CHUI_TREEPM_EINVAL;
  }
  return 0;
}

void applyConfig(Context& c, const chui_treepm_config& cfg) {
  c.cfg = cfg;
  // makeTreePmSplitPolicyFromMeshSpacing (tree_pm_split_kernel.hpp:50-63) with the
  // mesh spacing of gravity_runtime.cpp:586-590.
  c.spacing = std::cbrt((cfg.box_x / static_cast<double>(cfg.pm_grid_nx)) *
                        (cfg.box_y / static_cast<double>(cfg.pm_grid_ny)) *
                        (cfg.box_z / static_cast<double>(cfg.pm_grid_nz)));
  c.rs = cfg.asmth_cells * c.spacing;
  c.cutoff = cfg.rcut_cells * c.spacing;
  const double t_cut = (c.cutoff * c.cutoff) / (4.0 * c.rs * c.rs) * (1.0 + 1.0e-5);
  c.poly = fitPoly(t_cut);
  c.dpoly = fitChebyshev(hostHp, t_cut);
  // H'' scales the quadrupole's second-derivative term only: 1e-5 suffices
  c.ddpoly = fitChebyshev(hostHpp, t_cut, 1.0e-5);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Stage a host array into a device buffer (or pass a device pointer through).
template <class T>
int stageIn(Context& c, DevBuf& buf, const T* src, int64_t count, int memory, cudaStream_t s, const T** out) {
  if (src == nullptr || count == 0) {
    *out = src;
    if (count == 0 && src == nullptr) return 0;
    if (count == 0) return 0;
    return 0;
  }
  if (memory == CHUI_TREEPM_DEVICE) {
    *out = src;
    return 0;
  }
  if (ensure(buf, count * sizeof(T)) != cudaSuccess) return fail(c, CHUI_TREEPM_ENOMEM, "device staging allocation failed");
  if (cudaMemcpyAsync(buf.ptr, src, count * sizeof(T), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return fail(c, CHUI_TREEPM_EDEVICE, "host-to-device copy failed");
  *out = buf.as<T>();
  return 0;
}

}  // namespace

int sourceBounds(Context& c, int64_t n, const double* x, const double* y, const double* z, const double* m,
                 double lo[3], double hi[3], double* mass_sum, uint32_t* status_bits, cudaStream_t s,
                 double* mass_range) {
  auto* sc = c.scalars.as<unsigned long long>();
  unsigned long long init[10] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, 0ull, 0ull, ~0ull, 0ull};
  cudaMemcpyAsync(sc, init, sizeof(init), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(c.status.ptr, 0, 4, s);
  if (n > 0)
    { noteLaunch(); sourceReduceKernel<<<std::min(gridFor(n, 256), kReduceBlocks), 256, 0, s>>>(n, x, y, z, m, sc, reinterpret_cast<double*>(sc + 6),
                                                       c.status.as<uint32_t>()); }
  unsigned long long hb[10];
  uint32_t st = 0;
  cudaMemcpyAsync(hb, sc, sizeof(hb), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&st, c.status.ptr, 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(c, CHUI_TREEPM_EDEVICE, "source reduction failed");
  for (int a = 0; a < 3; ++a) {
    lo[a] = n > 0 ? fromOrderedBits(hb[a]) : INFINITY;
    hi[a] = n > 0 ? fromOrderedBits(hb[3 + a]) : -INFINITY;
  }
  double ms;
  std::memcpy(&ms, &hb[6], 8);
  *mass_sum = ms;
  *status_bits = st;
  if (mass_range) {
    mass_range[0] = (m && n > 0) ? fromOrderedBits(hb[8]) : 0.0;
    mass_range[1] = (m && n > 0) ? fromOrderedBits(hb[9]) : 0.0;
  }
  return 0;
}

}  // namespace chui

using chui::Context;

namespace {
// Text of the last failed chui_treepm_create on this thread (no handle exists).
thread_local std::string g_create_error;
}  // namespace

namespace chui {
namespace {

// One array of a host-memory elementwise step: copied in (host_in), updated
// on the device (dev), copied back (host_out, or NULL for inputs only).
struct HostLane {
  const double* host_in;
  double* dev;
  double* host_out;
};

// Host-memory kick and drift in chunks on two streams: each chunk's copies
// in, its kernel and its copies out are ordered on one stream, so a chunk's
// host-to-device copy overlaps the previous chunk's kernel and device-to-host
// copy (the copy engines move both directions at once). The caller's stream
// orders the whole step: the two streams start after its pending work and it
// waits for both before the call returns.
template <class Launch>
int pipelineHostStep(Context& c, int64_t n, cudaStream_t s, const HostLane* lanes, int count, Launch launch) {
  if (!c.pipe_ready) {
    for (auto& st : c.pipe_stream)
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
    for (auto& e : c.pipe_ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
    c.pipe_ready = true;
  }
  cudaEventRecord(c.pipe_ev[2], s);
  for (auto& st : c.pipe_stream) cudaStreamWaitEvent(st, c.pipe_ev[2], 0);
  constexpr int64_t kChunk = int64_t(1) << 22;  // 4 Mi elements: 32 MiB per array
  int64_t k = 0;
  for (int64_t b = 0; b < n; b += kChunk, ++k) {
    cudaStream_t st = c.pipe_stream[k & 1];
    const int64_t len = n - b < kChunk ? n - b : kChunk;
    for (int l = 0; l < count; ++l)
      cudaMemcpyAsync(lanes[l].dev + b, lanes[l].host_in + b, static_cast<size_t>(len) * 8, cudaMemcpyHostToDevice, st);
    launch(b, len, st);
    for (int l = 0; l < count; ++l)
      if (lanes[l].host_out)
        cudaMemcpyAsync(lanes[l].host_out + b, lanes[l].dev + b, static_cast<size_t>(len) * 8, cudaMemcpyDeviceToHost,
                        st);
  }
  for (int j = 0; j < 2; ++j) {
    cudaEventRecord(c.pipe_ev[j], c.pipe_stream[j]);
    cudaStreamWaitEvent(s, c.pipe_ev[j], 0);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

}  // namespace
}  // namespace chui

// ---- Lambda-CDM step factors (host) ----
namespace lcdm {

// H(a) in s^-1 for the background (LambdaCdmBackground::hubbleSi without
// radiation species).
struct Background {
  double h0_si, om, ol, orad, ok;
  double hubble(double a) const {
    const double a2 = a * a, a3 = a2 * a, a4 = a2 * a2;
    return h0_si * std::sqrt(orad / a4 + om / a3 + ok / a2 + ol);
  }
};

// Midpoint rule over [a0, a1] with `samples` cells of integrand(a_mid).
template <class F>
double midpoint(double a0, double a1, unsigned samples, F integrand) {
  const double da = (a1 - a0) / static_cast<double>(samples);
  if (da == 0.0) return 0.0;
  double sum = 0.0;
  for (unsigned i = 0; i < samples; ++i) sum += integrand(a0 + (static_cast<double>(i) + 0.5) * da);
  return sum * da;
}

// Cosmic time from a0 to a1: integral da / (a H).
double cosmicTime(const Background& b, double a0, double a1, unsigned samples) {
  return midpoint(a0, a1, samples, [&](double a) { return 1.0 / (a * b.hubble(a)); });
}

// Scale factor after dt seconds from a0: bracket by doubling, then bisect.
int advanceScaleFactor(const Background& b, double a0, double dt_si, double* out) {
  if (dt_si == 0.0) {
    *out = a0;
    return 0;
  }
  constexpr unsigned kSamples = 64;
  double hi = a0 * 1.001;
  if (hi <= a0) hi = a0 + 1.0e-12;
  for (int iter = 0; iter < 256 && cosmicTime(b, a0, hi, kSamples) < dt_si; ++iter) {
    hi *= 2.0;
    if (!std::isfinite(hi) || hi > 1.0e12) return CHUI_TREEPM_ERANGE;
  }
  if (cosmicTime(b, a0, hi, kSamples) < dt_si) return CHUI_TREEPM_ERANGE;
  double lo = a0;
  for (int iter = 0; iter < 96; ++iter) {
    const double mid = 0.5 * (lo + hi);
    if (cosmicTime(b, a0, mid, kSamples) < dt_si) lo = mid;
    else hi = mid;
  }
  *out = 0.5 * (lo + hi);
  return 0;
}

}  // namespace lcdm

extern "C" {

int chui_treepm_config_default(chui_treepm_config* cfg) {
  if (!cfg) return CHUI_TREEPM_EINVAL;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->pm_grid_nx = cfg->pm_grid_ny = cfg->pm_grid_nz = 16;  // config.hpp:778-780
  cfg->box_x = cfg->box_y = cfg->box_z = 1.0;
  cfg->asmth_cells = 1.25;                                    // config.hpp:783
  cfg->rcut_cells = 6.25;                                     // config.hpp:784
  cfg->opening_theta = 0.7;                                   // tree_gravity.hpp:33
  cfg->opening_criterion = CHUI_TREEPM_OPEN_COM_DISTANCE;     // tree_gravity.hpp:34
  cfg->multipole_order = 2;                                   // tree_gravity.hpp:35
  cfg->max_leaf_size = 16;                                    // tree_gravity.hpp:37
  cfg->assignment_scheme = CHUI_TREEPM_CIC;                   // pm_solver.hpp:231
  cfg->window_deconvolution = 0;                              // pm_solver.hpp:232
  cfg->gravitational_constant = 1.0;
  cfg->softening = 0.0;
  cfg->acceptance_policy = CHUI_TREEPM_POLICY_STRICT;            // tree_pm_coupling.hpp:247
  cfg->precision = CHUI_TREEPM_MIXED;
  cfg->device = 0;
  cfg->diagnostics = 0;  // the production walk
  cfg->adaptive_error_estimator = CHUI_TREEPM_ESTIMATOR_RESIDUAL_DERIVATIVE;  // tree_pm_coupling.hpp:249
  cfg->cutoff_node_policy = CHUI_TREEPM_CUTOFF_CONTAIN_NODE;                  // tree_pm_coupling.hpp:250
  cfg->adaptive_maximum_opening_angle = 0.25;                                 // tree_pm_coupling.hpp:248
  cfg->relative_force_tolerance = 0.005;                                      // tree_gravity.hpp:39
  cfg->relative_force_acceleration_floor = 1.0e-30;                           // tree_gravity.hpp:40
  cfg->group_walk_enabled = 0;                                                // tree_pm_coupling.hpp:257
  cfg->gaussian_pair_lookup = 0;                                              // tree_pm_coupling.hpp:266
  cfg->boundary_condition = CHUI_TREEPM_BOUNDARY_PERIODIC;                    // pm_solver.hpp:236
  cfg->short_range_only = 0;                                                  // tree_pm_coupling.hpp:292
  return 0;
}

int chui_treepm_create(const chui_treepm_config* cfg, void** handle) {
  if (!cfg || !handle) return CHUI_TREEPM_EINVAL;
  *handle = nullptr;
  std::string err;
  int rc = chui::validateConfig(*cfg, err);
  if (rc) {
    g_create_error = err;
    return rc;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    g_create_error = "no CUDA device is available";
    return CHUI_TREEPM_EDEVICE;
  }
  if (cfg->device < 0 || cfg->device >= ndev) {
    g_create_error = "device ordinal out of range";
    return CHUI_TREEPM_EINVAL;
  }
  Context* c = new (std::nothrow) Context();
  if (!c) {
    g_create_error = "context allocation failed";
    return CHUI_TREEPM_ENOMEM;
  }
  c->device = cfg->device;
  chui::DeviceGuard guard(c->device);
  chui::applyConfig(*c, *cfg);
  if (chui::ensure(c->status, 64) != cudaSuccess || chui::ensure(c->scalars, 64 * 8) != cudaSuccess) {
    delete c;
    g_create_error = "device allocation failed";
    return CHUI_TREEPM_ENOMEM;
  }
  g_create_error.clear();
  for (auto& e : c->ev) cudaEventCreate(&e);
  c->events_ready = true;
  *handle = c;
  return 0;
}

void chui_treepm_destroy(void* handle) {
  if (!handle) return;
  Context* c = static_cast<Context*>(handle);
  {
    chui::DeviceGuard guard(c->device);
    cudaDeviceSynchronize();
    chui::pmDestroy(*c);
    chui::DevBuf* bufs[] = {&c->in_x, &c->in_y, &c->in_z, &c->in_m, &c->in_active, &c->in_tx, &c->in_ty, &c->in_tz, &c->in_prev,
                            &c->grp_leaf, &c->grp_start, &c->grp_rec, &c->grp_list, &c->grp_done, &c->gauss_tab,
                            &c->out_acc[0], &c->out_acc[1], &c->out_acc[2], &c->out_pm[0], &c->out_pm[1],
                            &c->out_pm[2], &c->out_tree[0], &c->out_tree[1], &c->out_tree[2], &c->out_near,
                            &c->status, &c->scalars, &c->ux, &c->uy, &c->uz, &c->bucket_min, &c->bucket_max, &c->gap_min, &c->gap_max, &c->gap_flag, &c->gap_off, &c->grid_f4, &c->cp_levels,
                            &c->keys_a, &c->keys_b, &c->idx_a, &c->idx_b, &c->idx_c, &c->idx_d,
                            &c->path_words, &c->common_prefix, &c->node_count_per_pos, &c->node_offset,
                            &c->leaf_of_pos, &c->inv_pos, &c->sort_hist, &c->sort_counts,
                            &c->sort_totals, &c->sort_keys, &c->sort_vals, &c->node_geom, &c->node_com,
                            &c->node_quad, &c->node_f4, &c->node_mq, &c->node_child, &c->node_range, &c->node_parent, &c->node_depth,
                            &c->node_counter, &c->sorted_index, &c->pos_of_row, &c->src_f4, &c->src_d4, &c->src_u4, &c->src_cot,
                            &c->target_order, &c->morton_keys, &c->walk_counters, &c->work_counter,
                            &c->tree_acc, &c->tree_near, &c->walk_cost, &c->out_lr[0], &c->out_lr[1],
                            &c->out_lr[2]};
    for (auto* b : bufs) chui::release(*b);
    if (c->events_ready)
      for (auto& e : c->ev) cudaEventDestroy(e);
    if (c->pipe_ready) {
      for (auto& st : c->pipe_stream) cudaStreamDestroy(st);
      for (auto& e : c->pipe_ev) cudaEventDestroy(e);
    }
  }
  delete c;
}

int chui_treepm_set_config(void* handle, const chui_treepm_config* cfg) {
  if (!handle || !cfg) return CHUI_TREEPM_EINVAL;
  Context* c = static_cast<Context*>(handle);
  std::string err;
  int rc = chui::validateConfig(*cfg, err);
  if (rc) return chui::fail(*c, rc, err);
  if (cfg->pm_grid_nx != c->cfg.pm_grid_nx || cfg->pm_grid_ny != c->cfg.pm_grid_ny ||
      cfg->pm_grid_nz != c->cfg.pm_grid_nz || cfg->device != c->cfg.device)
    return chui::fail(*c, CHUI_TREEPM_EINVAL, "PM solver/grid shape mismatch: the mesh is fixed at creation");
  chui::DeviceGuard guard(c->device);
  const bool pm_changed = cfg->precision != c->cfg.precision || cfg->assignment_scheme != c->cfg.assignment_scheme ||
                          cfg->window_deconvolution != c->cfg.window_deconvolution || cfg->box_x != c->cfg.box_x ||
                          cfg->box_y != c->cfg.box_y || cfg->box_z != c->cfg.box_z ||
                          cfg->asmth_cells != c->cfg.asmth_cells ||
                          cfg->boundary_condition != c->cfg.boundary_condition ||
                          cfg->gravitational_constant != c->cfg.gravitational_constant;
  if (pm_changed) {
    cudaDeviceSynchronize();
    chui::pmDestroy(*c);
    c->pm_field_valid = false;
    c->pm_f4_ready = false;
  }
  chui::applyConfig(*c, *cfg);
  return 0;
}

const char* chui_treepm_last_error(const void* handle) {
  if (!handle) return g_create_error.c_str();
  return static_cast<const Context*>(handle)->last_error.c_str();
}

int chui_treepm_kdk_factors_lcdm(const chui_treepm_cosmology* cosmo, double a, double dt, double factors[10]) {
  if (!cosmo || !factors) return CHUI_TREEPM_EINVAL;
  const chui_treepm_cosmology& c = *cosmo;
  const double dens[4] = {c.omega_matter, c.omega_lambda, c.omega_radiation, c.omega_curvature};
  for (double d : dens)
    if (!std::isfinite(d)) return CHUI_TREEPM_EINVAL;
  if (!(std::isfinite(c.hubble_param) && c.hubble_param > 0.0) || c.omega_matter < 0.0 || c.omega_lambda < 0.0 ||
      c.omega_radiation < 0.0 ||
      std::fabs(c.omega_matter + c.omega_lambda + c.omega_radiation + c.omega_curvature - 1.0) > 1.0e-10 ||
      !(std::isfinite(c.time_si_per_code) && c.time_si_per_code > 0.0) || !(std::isfinite(a) && a > 0.0) ||
      !(std::isfinite(dt) && dt > 0.0))
    return CHUI_TREEPM_EINVAL;
  // 100 km/s/Mpc in s^-1 (1 pc = 3.0856775814913673e16 m)
  const double h100_si = (100.0 * 1.0e3) / (1.0e6 * 3.0856775814913673e16);
  const lcdm::Background b{c.hubble_param * h100_si, c.omega_matter, c.omega_lambda, c.omega_radiation,
                     c.omega_curvature};
  const double dt_si = dt * c.time_si_per_code;
  double a_mid = 0.0, a_end = 0.0;
  int rc = lcdm::advanceScaleFactor(b, a, 0.5 * dt_si, &a_mid);
  if (!rc) rc = lcdm::advanceScaleFactor(b, a, dt_si, &a_end);
  if (rc) return rc;
  constexpr unsigned kSamples = 64;
  // integral dt / a = integral da / (a^2 H); kick factors divide by the end scale factor
  const auto drift_like = [&](double a0, double a1) {
    return lcdm::midpoint(a0, a1, kSamples, [&](double x) { return 1.0 / (x * x * b.hubble(x)); });
  };
  const auto source_like = [&](double a0, double a1) {
    return lcdm::midpoint(a0, a1, kSamples, [&](double x) { return 1.0 / (x * x * x * b.hubble(x)); });
  };
  factors[0] = drift_like(a, a_end) / c.time_si_per_code;
  factors[1] = drift_like(a, a_mid) / a_mid / c.time_si_per_code;
  factors[2] = drift_like(a_mid, a_end) / a_end / c.time_si_per_code;
  factors[3] = a / a_mid;
  factors[4] = a_mid / a_end;
  factors[5] = source_like(a, a_mid) / c.time_si_per_code;
  factors[6] = source_like(a_mid, a_end) / c.time_si_per_code;
  factors[7] = a_mid;
  factors[8] = a_end;
  factors[9] = a / a_end;
  for (int k = 0; k < 10; ++k)
    if (!std::isfinite(factors[k])) return CHUI_TREEPM_ERANGE;
  return 0;
}

int chui_treepm_kdk_factors_static(double dt, double factors[5]) {
  if (!factors || !(dt > 0.0) || !std::isfinite(dt)) return CHUI_TREEPM_EINVAL;
  factors[0] = dt;
  factors[1] = 0.5 * dt;
  factors[2] = 0.5 * dt;
  factors[3] = 1.0;
  factors[4] = 1.0;
  return 0;
}

// The solve over the visit positions [visit_begin, visit_end) of the targets
// (ranged == false: all of them, outputs in active-slot order; ranged: outputs
// compact in visit order).
static int solveVisitRange(void* handle, const chui_treepm_sources* src, const chui_treepm_accumulator* acc,
                           int refresh_long_range_field, int memory, void* stream, chui_treepm_stats* stats,
                           int64_t visit_begin, int64_t visit_end, bool ranged) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  c.last_error.clear();
  if (!src || !acc) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources and accumulator are required");
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  const int64_t n = src->count;
  const int64_t nt = acc->active_index ? acc->active_count : (acc->target_x ? acc->active_count : n);
  if (n < 0 || nt < 0) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM requires non-negative extents");
  if (!ranged) {
    visit_begin = 0;
    visit_end = nt;
  } else if (visit_begin < 0 || visit_end < visit_begin || visit_end > nt ||
             (visit_begin % 64 != 0 && visit_begin != nt) || (visit_end % 64 != 0 && visit_end != nt)) {
    return chui::fail(c, CHUI_TREEPM_EINVAL,
                      "TreePM visit range must satisfy 0 <= begin <= end <= target count with both ends multiples "
                      "of 64 or the target count");
  }
  // outputs per call: every target, or the slice's targets in visit order
  const int64_t nout = visit_end - visit_begin;
  c.visit_count = -1;
  if (n > static_cast<int64_t>(0xFFFFFFFEu))
    return chui::fail(c, CHUI_TREEPM_ERANGE, "Tree gravity source count exceeds the 32-bit tree-index contract");
  if (n > 0 && (!src->x || !src->y || !src->z))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM requires position and mass spans with equal extent");
  if (!src->mass && !(std::isfinite(src->uniform_mass) && src->uniform_mass >= 0.0))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources require finite coordinates and finite non-negative masses");
  const bool explicit_targets = acc->target_x != nullptr;
  if (explicit_targets && (!acc->target_y || !acc->target_z))
    return chui::fail(c, CHUI_TREEPM_EINVAL,
                      "TreePM independent target coordinate triplet must be entirely present or absent");
  if (!explicit_targets && (acc->target_y || acc->target_z))
    return chui::fail(c, CHUI_TREEPM_EINVAL,
                      "TreePM independent target coordinate triplet must be entirely present or absent");
  if (nout > 0 && (!acc->accel_x || !acc->accel_y || !acc->accel_z))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM force accumulator spans must have matching active-set extent");
  if (explicit_targets && (acc->short_range_x || acc->nearest_pair_r2))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "Tree component output requires source-indexed full source extents");
  const bool lr = acc->long_range_x || acc->long_range_y || acc->long_range_z;
  const bool sr = acc->short_range_x || acc->short_range_y || acc->short_range_z;
  if ((lr && !(acc->long_range_x && acc->long_range_y && acc->long_range_z)) ||
      (sr && !(acc->short_range_x && acc->short_range_y && acc->short_range_z)))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM force accumulator spans must have matching active-set extent");

  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint64_t launches_before = chui::launchCount();
  cudaEventRecord(c.ev[0], s);
  int rc;
  const double *x, *y, *z, *m, *tx = nullptr, *ty = nullptr, *tz = nullptr;
  const uint32_t* active = nullptr;
  if ((rc = chui::stageIn(c, c.in_x, src->x, n, memory, s, &x)) || (rc = chui::stageIn(c, c.in_y, src->y, n, memory, s, &y)) ||
      (rc = chui::stageIn(c, c.in_z, src->z, n, memory, s, &z)) ||
      (rc = chui::stageIn(c, c.in_m, src->mass, src->mass ? n : 0, memory, s, &m)))
    return rc;
  if (acc->active_index && (rc = chui::stageIn(c, c.in_active, acc->active_index, nt, memory, s, &active))) return rc;
  const double* prev = nullptr;
  if (acc->previous_acceleration_magnitude &&
      (rc = chui::stageIn(c, c.in_prev, acc->previous_acceleration_magnitude, nt, memory, s, &prev)))
    return rc;
  if (explicit_targets &&
      ((rc = chui::stageIn(c, c.in_tx, acc->target_x, nt, memory, s, &tx)) ||
       (rc = chui::stageIn(c, c.in_ty, acc->target_y, nt, memory, s, &ty)) ||
       (rc = chui::stageIn(c, c.in_tz, acc->target_z, nt, memory, s, &tz))))
    return rc;
  if (!src->mass) m = nullptr;
  // per-particle softening lanes (resolved epsilons)
  c.soft_rows = nullptr;
  c.soft_targets = nullptr;
  if (explicit_targets && src->softening && !acc->target_softening)
    return chui::fail(c, CHUI_TREEPM_EINVAL,
                      "TreePM independent targets require target-owned softening/species sidecars when source "
                      "sidecars are present");
  if (src->softening && (rc = chui::stageIn(c, c.in_eps, src->softening, n, memory, s, &c.soft_rows))) return rc;
  if (acc->target_softening &&
      (rc = chui::stageIn(c, c.in_teps, acc->target_softening, nt, memory, s, &c.soft_targets)))
    return rc;
  if (c.soft_rows || c.soft_targets) {
    uint32_t bits = 0;
    cudaMemsetAsync(c.status.ptr, 0, 4, s);
    if (c.soft_rows && n > 0)
      { chui::noteLaunch(); chui::softeningCheckKernel<<<chui::gridFor(n, 256), 256, 0, s>>>(n, c.soft_rows, c.status.as<uint32_t>()); }
    if (c.soft_targets && nt > 0)
      { chui::noteLaunch(); chui::softeningCheckKernel<<<chui::gridFor(nt, 256), 256, 0, s>>>(nt, c.soft_targets, c.status.as<uint32_t>()); }
    cudaMemcpyAsync(&bits, c.status.ptr, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return chui::fail(c, CHUI_TREEPM_EDEVICE, "CUDA error");
    if (bits) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM softening sidecars require finite non-negative values");
  }

  // validateTreePmPreflight (tree_pm_coupling.cpp:244-481)
  double lo[3], hi[3], mass_sum = 0.0, mass_range[2] = {0.0, 0.0};
  uint32_t st = 0;
  if ((rc = chui::sourceBounds(c, n, x, y, z, m, lo, hi, &mass_sum, &st, s, mass_range))) return rc;
  if (st) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources require finite coordinates and finite non-negative masses");
  if (explicit_targets && nt > 0) {
    double tlo[3], thi[3], dummy;
    if ((rc = chui::sourceBounds(c, nt, tx, ty, tz, nullptr, tlo, thi, &dummy, &st, s))) return rc;
    if (st) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM target positions must be finite");
  }
  if (active && nt > 0) {
    cudaMemsetAsync(c.status.ptr, 0, 4, s);
    { chui::noteLaunch(); chui::activeCheckKernel<<<chui::gridFor(nt, 256), 256, 0, s>>>(nt, active, n, explicit_targets ? 1 : 0,
                                                                  c.status.as<uint32_t>()); }
    cudaMemcpyAsync(&st, c.status.ptr, 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (st) {
      return chui::fail(c, CHUI_TREEPM_ERANGE,
                        explicit_targets
                            ? "TreePM explicit target source identity must be local or the invalid local-index sentinel"
                            : "TreePM active index exceeds particle count");
    }
  } else if (!active && !explicit_targets && nt > n) {
    return chui::fail(c, CHUI_TREEPM_ERANGE, "TreePM active index exceeds particle count");
  }
  const double total_mass = m ? mass_sum : static_cast<double>(n) * src->uniform_mass;

  // short-range only: no PM refresh, interpolation or reuse
  const bool short_only = c.cfg.short_range_only != 0;
  if (short_only) refresh_long_range_field = 0;
  // cached-field reuse needs a compatible field (tree_pm_coupling.cpp:2483-2532)
  if (!refresh_long_range_field && !short_only &&
      (!c.pm_field_valid || c.pm_field_box[0] != c.cfg.box_x || c.pm_field_box[1] != c.cfg.box_y ||
       c.pm_field_box[2] != c.cfg.box_z)) {
    return chui::fail(c, CHUI_TREEPM_ESTATE, "TreePM long-range reuse requested without a compatible PM field");
  }

  // periodic tree build (first: the PM deposit reads the tree-ordered sources);
  // equal masses travel as one value instead of a lane of scattered reads
  const bool equal_masses = m && mass_range[0] == mass_range[1];
  if ((rc = chui::treeBuild(c, n, x, y, z, equal_masses ? nullptr : m,
                            equal_masses ? mass_range[0] : src->uniform_mass, lo, hi, s))) {
    if (c.last_error.empty()) c.last_error = "TreePM tree build failed";
    return rc;
  }
  double nlo[3], nhi[3];
  if ((rc = chui::treeNodeBounds(c, nlo, nhi, s))) return chui::fail(c, rc, "node bounds failed");
  if ((rc = chui::treeOrderTargets(c, nt, active, explicit_targets ? 1 : 0, n, s)))
    return chui::fail(c, rc, "target ordering failed");
  cudaEventRecord(c.ev[1], s);

  // PM refresh (tiled deposit over the tree-ordered sources)
  if (refresh_long_range_field &&
      (rc = chui::pmRefresh(c, n, x, y, z, m, src->uniform_mass, total_mass, s,
                            n > 0 ? c.src_d4.as<double4>() : nullptr)))
    return rc;
  cudaEventRecord(c.ev[2], s);

  // residual walk
  chui::WalkParams wp;
  // isolated/open: no periodic images (tree_pm_coupling.cpp:3560-3562)
  const bool periodic = c.cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_PERIODIC;
  wp.box[0] = periodic ? c.cfg.box_x : 0.0;
  wp.box[1] = periodic ? c.cfg.box_y : 0.0;
  wp.box[2] = periodic ? c.cfg.box_z : 0.0;
  for (int a = 0; a < 3; ++a) wp.inv_box[a] = periodic ? 1.0 / wp.box[a] : 0.0;
  for (int a = 0; a < 3; ++a) {
    wp.src_lo[a] = lo[a];
    wp.src_hi[a] = hi[a];
    wp.node_lo[a] = nlo[a];
    wp.node_hi[a] = nhi[a];
  }
  wp.rs = c.rs;
  wp.cutoff = c.cutoff;
  wp.cutoff2 = c.cutoff * c.cutoff;
  wp.G = c.cfg.gravitational_constant;
  wp.eps = c.cfg.softening;
  wp.theta = c.cfg.opening_theta;
  wp.exact_half = periodic ? 0.5 * std::min({c.cfg.box_x, c.cfg.box_y, c.cfg.box_z}) - c.cutoff : INFINITY;
  wp.criterion = c.cfg.opening_criterion;
  wp.quadrupole = c.cfg.multipole_order == 2 ? 1 : 0;
  wp.policy = c.cfg.acceptance_policy;
  wp.estimator = c.cfg.adaptive_error_estimator;
  wp.com_cutoff = c.cfg.acceptance_policy == CHUI_TREEPM_POLICY_ADAPTIVE &&
                  c.cfg.cutoff_node_policy == CHUI_TREEPM_CUTOFF_COM_DISTANCE;
  wp.angle = c.cfg.adaptive_maximum_opening_angle;
  wp.rel_tol = c.cfg.relative_force_tolerance;
  wp.floor_ = c.cfg.relative_force_acceleration_floor;
  wp.gauss_lookup = c.cfg.gaussian_pair_lookup ? 1 : 0;
  // one mass for every source (no mass lane, or equal entries): the walk
  // queue then carries a lane mask instead of a mass
  wp.uniform_mass = !m || mass_range[0] == mass_range[1];
  wp.m0_f = static_cast<float>(m ? mass_range[0] : src->uniform_mass);
  {
    // group walk eligibility (tree_pm_coupling.cpp:3840-3870, 3922-3925, 4282-4286)
    const double inv_2a2 = (0.25 / c.rs) / c.rs, inv_8a3 = ((0.125 / c.rs) / c.rs) / c.rs;
    const double t_cut = (0.25 * wp.cutoff2 / c.rs) / c.rs;
    // (no group walk with per-particle softening: tree_pm_coupling.cpp:3858-3859)
    wp.group_walk = !c.soft_rows && !c.soft_targets && c.cfg.group_walk_enabled &&
                    c.cfg.acceptance_policy == CHUI_TREEPM_POLICY_ADAPTIVE &&
                    c.cfg.adaptive_error_estimator == CHUI_TREEPM_ESTIMATOR_RELATIVE_MONOPOLE &&
                    c.cfg.gaussian_pair_lookup && std::isnormal(inv_2a2) && std::isnormal(inv_8a3) &&
                    std::isfinite(t_cut) && t_cut < 63.0;
  }
  wp.inv_4rs2_f = static_cast<float>(0.25 / (c.rs * c.rs));
  wp.inv_8rs3_f = static_cast<float>(0.125 / (c.rs * c.rs * c.rs));
  wp.cut2_f = static_cast<float>(c.cutoff * c.cutoff);
  wp.eps2_f = static_cast<float>(c.cfg.softening * c.cfg.softening);
  wp.G_f = static_cast<float>(c.cfg.gravitational_constant);
  cudaMemsetAsync(c.status.ptr, 0, 4, s);
  // the production walk also counts and records nearest pairs when asked to,
  // or when the caller wants the nearest-pair lane
  c.walk_instrument = c.cfg.diagnostics == 2 || acc->nearest_pair_r2 != nullptr;
  // outputs at slots (a slice's compactly, with per-block cycles)
  if (n > 0 && (rc = chui::walkRun(c, nt, active, tx, ty, tz, x, y, z, prev, wp, n, s, visit_begin, visit_end,
                                     ranged, ranged)))
    return chui::fail(c, rc, rc == CHUI_TREEPM_ENOTSUP
                                 ? "the mixed-precision pair kernel's constants (H(t)/(8 r_s^3)) overflow FP32 for "
                                   "this split scale; use precision FP64"
                                 : "residual walk launch failed");
  if (n == 0 && nt > 0) {
    if (chui::ensure(c.tree_acc, nt * 3 * 8) || chui::ensure(c.tree_near, nt * 8))
      return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    cudaMemsetAsync(c.tree_acc.ptr, 0, nt * 3 * 8, s);
    std::vector<double> inf(nt, INFINITY);
    cudaMemcpyAsync(c.tree_near.ptr, inf.data(), nt * 8, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  }
  cudaEventRecord(c.ev[3], s);

  // outputs
  double *ax, *ay, *az, *pmx, *pmy, *pmz, *sx = nullptr, *sy = nullptr, *sz = nullptr, *snear = nullptr;
  if (memory == CHUI_TREEPM_DEVICE) {
    ax = acc->accel_x;
    ay = acc->accel_y;
    az = acc->accel_z;
    sx = acc->short_range_x;
    sy = acc->short_range_y;
    sz = acc->short_range_z;
    snear = acc->nearest_pair_r2;
  } else {
    for (int a = 0; a < 3; ++a)
      if (chui::ensure(c.out_acc[a], std::max<int64_t>(nout, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    ax = c.out_acc[0].as<double>();
    ay = c.out_acc[1].as<double>();
    az = c.out_acc[2].as<double>();
    if (sr) {
      for (int a = 0; a < 3; ++a)
        if (chui::ensure(c.out_tree[a], std::max<int64_t>(n, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
      sx = c.out_tree[0].as<double>();
      sy = c.out_tree[1].as<double>();
      sz = c.out_tree[2].as<double>();
      cudaMemcpyAsync(sx, acc->short_range_x, n * 8, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(sy, acc->short_range_y, n * 8, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(sz, acc->short_range_z, n * 8, cudaMemcpyHostToDevice, s);
    }
    if (acc->nearest_pair_r2) {
      if (chui::ensure(c.out_near, std::max<int64_t>(n, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
      snear = c.out_near.as<double>();
      cudaMemcpyAsync(snear, acc->nearest_pair_r2, n * 8, cudaMemcpyHostToDevice, s);
    }
  }
  // a visit range interpolates into slot-indexed scratch; the combine writes
  // the slice's long-range lanes compactly
  double *lx = nullptr, *ly = nullptr, *lz = nullptr;
  if (lr && memory == CHUI_TREEPM_DEVICE && !ranged) {
    pmx = acc->long_range_x;
    pmy = acc->long_range_y;
    pmz = acc->long_range_z;
  } else {
    for (int a = 0; a < 3; ++a)
      if (chui::ensure(c.out_pm[a], std::max<int64_t>(nt, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    pmx = c.out_pm[0].as<double>();
    pmy = c.out_pm[1].as<double>();
    pmz = c.out_pm[2].as<double>();
  }
  const uint32_t* slice = ranged && nout > 0 ? c.target_order.as<uint32_t>() + visit_begin : nullptr;
  if (ranged && lr) {
    if (memory == CHUI_TREEPM_DEVICE) {
      lx = acc->long_range_x;
      ly = acc->long_range_y;
      lz = acc->long_range_z;
    } else {
      for (int a = 0; a < 3; ++a)
        if (chui::ensure(c.out_lr[a], std::max<int64_t>(nout, 1) * 8))
          return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
      lx = c.out_lr[0].as<double>();
      ly = c.out_lr[1].as<double>();
      lz = c.out_lr[2].as<double>();
    }
  }
  if (!ranged) {
    // interpolation and the total in one pass over the slots
    if (nt > 0 &&
        (rc = chui::pmInterpolateCombine(c, nt, active, tx, ty, tz, explicit_targets ? 0 : n, x, y, z, !short_only,
                                         c.tree_acc.as<double>(), c.tree_near.as<double>(), ax, ay, az,
                                         lr ? pmx : nullptr, lr ? pmy : nullptr, lr ? pmz : nullptr, sx, sy, sz, snear,
                                         s)))
      return rc;
  } else {
    if (short_only) {
      for (double* p : {pmx, pmy, pmz}) cudaMemsetAsync(p, 0, static_cast<size_t>(nt) * 8, s);
    } else if ((rc = chui::pmInterpolate(c, nout, active, tx, ty, tz, x, y, z, pmx, pmy, pmz, s, slice))) {
      return rc;
    }
    if (nout > 0)
      { chui::noteLaunch(); chui::combineKernel<<<chui::gridFor(nout, 256), 256, 0, s>>>(
            nout, slice, nt, active, explicit_targets ? 0 : n, pmx, pmy, pmz, c.tree_acc.as<double>(),
            c.tree_near.as<double>(), ax, ay, az, lx, ly, lz, sx, sy, sz, snear); }
  }
  c.visit_count = nt;
  cudaEventRecord(c.ev[4], s);
  uint32_t walk_status = 0;
  cudaMemcpyAsync(&walk_status, c.status.ptr, 4, cudaMemcpyDeviceToHost, s);
  unsigned long long counters[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (n > 0 && nt > 0 && c.walk_counters.ptr)
    cudaMemcpyAsync(counters, c.walk_counters.ptr, sizeof(counters), cudaMemcpyDeviceToHost, s);
  if (memory == CHUI_TREEPM_HOST && nout > 0) {
    cudaMemcpyAsync(acc->accel_x, ax, nout * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(acc->accel_y, ay, nout * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(acc->accel_z, az, nout * 8, cudaMemcpyDeviceToHost, s);
    if (lr) {
      cudaMemcpyAsync(acc->long_range_x, ranged ? lx : pmx, nout * 8, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(acc->long_range_y, ranged ? ly : pmy, nout * 8, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(acc->long_range_z, ranged ? lz : pmz, nout * 8, cudaMemcpyDeviceToHost, s);
    }
    if (sr) {
      cudaMemcpyAsync(acc->short_range_x, sx, n * 8, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(acc->short_range_y, sy, n * 8, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(acc->short_range_z, sz, n * 8, cudaMemcpyDeviceToHost, s);
    }
    if (acc->nearest_pair_r2) cudaMemcpyAsync(acc->nearest_pair_r2, snear, n * 8, cudaMemcpyDeviceToHost, s);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return chui::fail(c, CHUI_TREEPM_EDEVICE, std::string("CUDA error: ") + cudaGetErrorString(e));
  if (walk_status) return chui::fail(c, CHUI_TREEPM_ERANGE, chui::statusText(walk_status));
  chui_treepm_stats stt{};
  stt.visited_nodes = counters[0];
  stt.accepted_nodes = counters[1];
  stt.opened_nodes = counters[2];
  stt.direct_pair_evaluations = counters[3];
  stt.cutoff_pruned_nodes = counters[4];
  stt.cutoff_skipped_pairs = counters[5];
  stt.accepted_internal_multipoles = counters[6];
  stt.accepted_leaves = counters[7];
  stt.node_count = static_cast<uint64_t>(c.n_nodes);
  stt.maximum_depth = c.max_depth;
  stt.path_words = static_cast<uint32_t>(c.path_words_used);
  stt.kernel_launches = chui::launchCount() - launches_before;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]);
  stt.tree_build_ms = ms;
  cudaEventElapsedTime(&ms, c.ev[1], c.ev[2]);
  stt.pm_ms = ms;
  cudaEventElapsedTime(&ms, c.ev[2], c.ev[3]);
  stt.walk_ms = ms;
  cudaEventElapsedTime(&ms, c.ev[0], c.ev[4]);
  stt.total_ms = ms;
  c.last_stats = stt;
  if (stats) *stats = stt;
  return 0;
}

int chui_treepm_solve(void* handle, const chui_treepm_sources* src, const chui_treepm_accumulator* acc,
                      int refresh_long_range_field, int memory, void* stream, chui_treepm_stats* stats) {
  return solveVisitRange(handle, src, acc, refresh_long_range_field, memory, stream, stats, 0, -1, false);
}

int chui_treepm_solve_visit_range(void* handle, const chui_treepm_sources* src, const chui_treepm_accumulator* acc,
                                  int refresh_long_range_field, int memory, void* stream, chui_treepm_stats* stats,
                                  int64_t visit_begin, int64_t visit_end) {
  return solveVisitRange(handle, src, acc, refresh_long_range_field, memory, stream, stats, visit_begin, visit_end,
                         true);
}

int chui_treepm_walk_cost(void* handle, int64_t begin, int64_t end, float* cost, int memory, void* stream) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  c.last_error.clear();
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  if (c.visit_count < 0) return chui::fail(c, CHUI_TREEPM_ESTATE, "TreePM walk cost requested before a solve");
  if (begin < 0 || end < begin || end > c.visit_count || (begin % 32 != 0 && begin != end))
    return chui::fail(c, CHUI_TREEPM_EINVAL,
                      "TreePM walk cost range must lie in the last solve's targets and start at a multiple of 32");
  const int64_t chunks = (end - begin + 31) / 32;
  if (chunks == 0) return 0;
  if (!cost) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM walk cost output is required");
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const cudaMemcpyKind kind = memory == CHUI_TREEPM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const size_t have = c.walk_cost.bytes / sizeof(float);
  const int64_t first = begin / 32;
  if (static_cast<size_t>(first + chunks) <= have) {
    cudaMemcpyAsync(cost, c.walk_cost.as<float>() + first, static_cast<size_t>(chunks) * sizeof(float), kind, s);
  } else if (memory == CHUI_TREEPM_HOST) {
    std::fill(cost, cost + chunks, 0.0f);  // no walk ran (no sources)
  } else {
    cudaMemsetAsync(cost, 0, static_cast<size_t>(chunks) * sizeof(float), s);
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return chui::fail(c, CHUI_TREEPM_EDEVICE, std::string("CUDA error: ") + cudaGetErrorString(e));
  return 0;
}

int chui_treepm_visit_order(void* handle, int64_t begin, int64_t end, uint32_t* slots, int memory, void* stream) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  c.last_error.clear();
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  if (c.visit_count < 0) return chui::fail(c, CHUI_TREEPM_ESTATE, "TreePM visit order requested before a solve");
  if (begin < 0 || end < begin || end > c.visit_count)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM visit order range exceeds the last solve's target count");
  if (end > begin && !slots) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM visit order output is required");
  if (end == begin) return 0;
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemcpyAsync(slots, c.target_order.as<uint32_t>() + begin, static_cast<size_t>(end - begin) * 4,
                  memory == CHUI_TREEPM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return chui::fail(c, CHUI_TREEPM_EDEVICE, std::string("CUDA error: ") + cudaGetErrorString(e));
  return 0;
}

int chui_treepm_force_vjp(void* handle, const chui_treepm_sources* src, const double* cot_x, const double* cot_y,
                          const double* cot_z, double* grad_x, double* grad_y, double* grad_z, int memory,
                          void* stream, chui_treepm_stats* stats) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  c.last_error.clear();
  if (c.cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_PERIODIC)
    return chui::fail(c, CHUI_TREEPM_ENOTSUP, "the force VJP supports periodic boundaries only");
  if (!src) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources are required");
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  const int64_t n = src->count;
  if (n < 0) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM requires non-negative extents");
  if (n > static_cast<int64_t>(0xFFFFFFFEu))
    return chui::fail(c, CHUI_TREEPM_ERANGE, "Tree gravity source count exceeds the 32-bit tree-index contract");
  if (n > 0 && (!src->x || !src->y || !src->z || !cot_x || !cot_y || !cot_z || !grad_x || !grad_y || !grad_z))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "force VJP requires positions, cotangents and gradients of equal extent");
  if (!src->mass && !(std::isfinite(src->uniform_mass) && src->uniform_mass >= 0.0))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources require finite coordinates and finite non-negative masses");
  if (src->softening)
    return chui::fail(c, CHUI_TREEPM_ENOTSUP, "the force VJP supports uniform softening only");
  c.soft_rows = nullptr;
  c.soft_targets = nullptr;
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint64_t launches_before = chui::launchCount();
  cudaEventRecord(c.ev[0], s);
  int rc;
  const double *x, *y, *z, *m, *cx, *cy, *cz;
  if ((rc = chui::stageIn(c, c.in_x, src->x, n, memory, s, &x)) || (rc = chui::stageIn(c, c.in_y, src->y, n, memory, s, &y)) ||
      (rc = chui::stageIn(c, c.in_z, src->z, n, memory, s, &z)) ||
      (rc = chui::stageIn(c, c.in_m, src->mass, src->mass ? n : 0, memory, s, &m)) ||
      (rc = chui::stageIn(c, c.in_tx, cot_x, n, memory, s, &cx)) ||
      (rc = chui::stageIn(c, c.in_ty, cot_y, n, memory, s, &cy)) ||
      (rc = chui::stageIn(c, c.in_tz, cot_z, n, memory, s, &cz)))
    return rc;
  if (!src->mass) m = nullptr;
  double lo[3], hi[3], mass_sum = 0.0;
  uint32_t st = 0;
  if ((rc = chui::sourceBounds(c, n, x, y, z, m, lo, hi, &mass_sum, &st, s))) return rc;
  if (st) return chui::fail(c, CHUI_TREEPM_EINVAL, "TreePM sources require finite coordinates and finite non-negative masses");
  const double total_mass = m ? mass_sum : static_cast<double>(n) * src->uniform_mass;
  double *gx = grad_x, *gy = grad_y, *gz = grad_z;
  if (memory == CHUI_TREEPM_HOST) {
    for (int a = 0; a < 3; ++a)
      if (chui::ensure(c.out_acc[a], std::max<int64_t>(n, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    gx = c.out_acc[0].as<double>();
    gy = c.out_acc[1].as<double>();
    gz = c.out_acc[2].as<double>();
  }
  // tree for these positions, every particle a target in tree order
  c.visit_count = -1;
  if (n > 0) {
    if ((rc = chui::treeBuild(c, n, x, y, z, m, src->uniform_mass, lo, hi, s))) {
      if (c.last_error.empty()) c.last_error = "TreePM tree build failed";
      return rc;
    }
    if ((rc = chui::treeOrderTargets(c, n, nullptr, 0, n, s))) return chui::fail(c, rc, "target ordering failed");
  }
  cudaEventRecord(c.ev[1], s);
  // PM part (refreshes the PM field at these positions)
  if ((rc = chui::pmForceVjp(c, n, x, y, z, m, src->uniform_mass, total_mass, cx, cy, cz, gx, gy, gz, s,
                             n > 0 ? c.src_d4.as<double4>() : nullptr)))
    return chui::fail(c, rc, c.last_error.empty() ? "PM adjoint failed" : c.last_error);
  cudaEventRecord(c.ev[2], s);
  chui::WalkParams wp{};
  wp.box[0] = c.cfg.box_x;
  wp.box[1] = c.cfg.box_y;
  wp.box[2] = c.cfg.box_z;
  for (int a = 0; a < 3; ++a) wp.inv_box[a] = 1.0 / wp.box[a];
  wp.rs = c.rs;
  wp.cutoff = c.cutoff;
  wp.cutoff2 = c.cutoff * c.cutoff;
  wp.G = c.cfg.gravitational_constant;
  wp.eps = c.cfg.softening;
  wp.inv_4rs2_f = static_cast<float>(0.25 / (c.rs * c.rs));
  wp.inv_8rs3_f = static_cast<float>(0.125 / (c.rs * c.rs * c.rs));
  wp.cut2_f = static_cast<float>(c.cutoff * c.cutoff);
  wp.eps2_f = static_cast<float>(c.cfg.softening * c.cfg.softening);
  wp.G_f = static_cast<float>(c.cfg.gravitational_constant);
  cudaMemsetAsync(c.status.ptr, 0, 4, s);
  if (n > 0) {
    if (chui::ensure(c.tree_acc, static_cast<size_t>(n) * 3 * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    double* t = c.tree_acc.as<double>();
    if ((rc = chui::walkVjpRun(c, n, x, y, z, m, src->uniform_mass, cx, cy, cz, wp, t, t + n, t + 2 * n, s)))
      return chui::fail(c, rc, "adjoint walk launch failed");
    cudaEventRecord(c.ev[3], s);
    { chui::noteLaunch(); chui::addKernel<<<chui::gridFor(n, 256), 256, 0, s>>>(n, gx, gy, gz, t); }
  } else {
    cudaEventRecord(c.ev[3], s);
  }
  cudaEventRecord(c.ev[4], s);
  uint32_t walk_status = 0;
  cudaMemcpyAsync(&walk_status, c.status.ptr, 4, cudaMemcpyDeviceToHost, s);
  if (memory == CHUI_TREEPM_HOST && n > 0) {
    cudaMemcpyAsync(grad_x, gx, n * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(grad_y, gy, n * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(grad_z, gz, n * 8, cudaMemcpyDeviceToHost, s);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return chui::fail(c, CHUI_TREEPM_EDEVICE, std::string("CUDA error: ") + cudaGetErrorString(e));
  if (walk_status) return chui::fail(c, CHUI_TREEPM_ERANGE, chui::statusText(walk_status));
  if (stats) {
    chui_treepm_stats stt{};
    stt.node_count = static_cast<uint64_t>(c.n_nodes);
    stt.maximum_depth = c.max_depth;
    stt.path_words = static_cast<uint32_t>(c.path_words_used);
    stt.kernel_launches = chui::launchCount() - launches_before;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]);
    stt.tree_build_ms = ms;
    cudaEventElapsedTime(&ms, c.ev[1], c.ev[2]);
    stt.pm_ms = ms;
    cudaEventElapsedTime(&ms, c.ev[2], c.ev[3]);
    stt.walk_ms = ms;
    cudaEventElapsedTime(&ms, c.ev[0], c.ev[4]);
    stt.total_ms = ms;
    *stats = stt;
  }
  return 0;
}

int chui_pm_density_vjp(void* handle, const chui_treepm_sources* src, const double* rho_bar, double* grad_x,
                        double* grad_y, double* grad_z, int memory, void* stream) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  if (c.cfg.boundary_condition != CHUI_TREEPM_BOUNDARY_PERIODIC)
    return chui::fail(c, CHUI_TREEPM_ENOTSUP, "the density VJP supports periodic boundaries only");
  if (!src || !rho_bar || (src->count > 0 && (!src->x || !src->y || !src->z || !grad_x || !grad_y || !grad_z)))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "density VJP requires positions, a cotangent grid and gradients");
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = src->count;
  const size_t cells = static_cast<size_t>(c.cfg.pm_grid_nx) * c.cfg.pm_grid_ny * c.cfg.pm_grid_nz;
  const double *x, *y, *z, *m, *rb;
  int rc;
  if ((rc = chui::stageIn(c, c.in_x, src->x, n, memory, s, &x)) || (rc = chui::stageIn(c, c.in_y, src->y, n, memory, s, &y)) ||
      (rc = chui::stageIn(c, c.in_z, src->z, n, memory, s, &z)) ||
      (rc = chui::stageIn(c, c.in_m, src->mass, src->mass ? n : 0, memory, s, &m)) ||
      (rc = chui::stageIn(c, c.in_tx, rho_bar, static_cast<int64_t>(cells), memory, s, &rb)))
    return rc;
  if (!src->mass) m = nullptr;
  double *gx = grad_x, *gy = grad_y, *gz = grad_z;
  if (memory == CHUI_TREEPM_HOST) {
    for (int a = 0; a < 3; ++a)
      if (chui::ensure(c.out_acc[a], std::max<int64_t>(n, 1) * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    gx = c.out_acc[0].as<double>();
    gy = c.out_acc[1].as<double>();
    gz = c.out_acc[2].as<double>();
  }
  if ((rc = chui::pmDensityVjp(c, n, x, y, z, m, src->uniform_mass, rb, gx, gy, gz, s))) return rc;
  if (memory == CHUI_TREEPM_HOST && n > 0) {
    cudaMemcpyAsync(grad_x, gx, n * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(grad_y, gy, n * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(grad_z, gz, n * 8, cudaMemcpyDeviceToHost, s);
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "density VJP failed");
}

int chui_treepm_kdk_adjoint(void* handle, int64_t n, const double* gx, const double* gy, const double* gz,
                            double* x_bar_x, double* x_bar_y, double* x_bar_z, double* v_bar_x, double* v_bar_y,
                            double* v_bar_z, double* a_bar_x, double* a_bar_y, double* a_bar_z, double drift_factor,
                            double kick1, double kick2, double drag1, double drag2, int first_step, void* stream) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  if (n < 0 || (n > 0 && (!gx || !gy || !gz || !x_bar_x || !x_bar_y || !x_bar_z || !v_bar_x || !v_bar_y ||
                          !v_bar_z || !a_bar_x || !a_bar_y || !a_bar_z)))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "KDK adjoint requires device arrays of equal extent");
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n > 0)
    { chui::noteLaunch(); chui::kdkAdjointKernel<<<chui::gridFor(n, 256), 256, 0, s>>>(
        n, gx, gy, gz, x_bar_x, x_bar_y, x_bar_z, v_bar_x, v_bar_y, v_bar_z, a_bar_x, a_bar_y, a_bar_z,
        drift_factor, kick1, kick2, drag1, drag2, first_step); }
  return cudaGetLastError() == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "KDK adjoint launch failed");
}

int chui_treepm_momentum_energy(void* handle, int64_t n, const double* mass, double uniform_mass, const double* vx,
                                const double* vy, const double* vz, const double* ax, const double* ay,
                                const double* az, int memory, void* stream, double out[8]) {
  if (!handle || !out) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  if (n < 0 || (n > 0 && (!vx || !vy || !vz)) || ((ax || ay || az) && !(ax && ay && az)))
    return chui::fail(c, CHUI_TREEPM_EINVAL, "momentum/energy check requires velocity arrays (and all or no accelerations)");
  if (memory != CHUI_TREEPM_HOST && memory != CHUI_TREEPM_DEVICE)
    return chui::fail(c, CHUI_TREEPM_EINVAL, "memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double *m, *u[3], *a[3] = {nullptr, nullptr, nullptr};
  int rc;
  if ((rc = chui::stageIn(c, c.in_m, mass, mass ? n : 0, memory, s, &m)) ||
      (rc = chui::stageIn(c, c.in_x, vx, n, memory, s, &u[0])) || (rc = chui::stageIn(c, c.in_y, vy, n, memory, s, &u[1])) ||
      (rc = chui::stageIn(c, c.in_z, vz, n, memory, s, &u[2])))
    return rc;
  if (ax && ((rc = chui::stageIn(c, c.in_tx, ax, n, memory, s, &a[0])) ||
             (rc = chui::stageIn(c, c.in_ty, ay, n, memory, s, &a[1])) ||
             (rc = chui::stageIn(c, c.in_tz, az, n, memory, s, &a[2]))))
    return rc;
  if (!mass) m = nullptr;
  double* d = c.scalars.as<double>();
  cudaMemsetAsync(d, 0, 8 * sizeof(double), s);
  if (n > 0)
    { chui::noteLaunch(); chui::momentumEnergyKernel<<<std::min<unsigned>(chui::gridFor(n, 256), 148u * 4u), 256, 0, s>>>(
        n, m, uniform_mass, u[0], u[1], u[2], a[0], a[1], a[2], d); }
  cudaMemcpyAsync(out, d, 8 * sizeof(double), cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "momentum/energy check failed");
}

int chui_pm_assign_density(void* handle, const chui_treepm_sources* src, double* density, int memory, void* stream) {
  if (!handle || !src || !density) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = src->count;
  const double *x, *y, *z, *m;
  int rc;
  if ((rc = chui::stageIn(c, c.in_x, src->x, n, memory, s, &x)) || (rc = chui::stageIn(c, c.in_y, src->y, n, memory, s, &y)) ||
      (rc = chui::stageIn(c, c.in_z, src->z, n, memory, s, &z)) ||
      (rc = chui::stageIn(c, c.in_m, src->mass, src->mass ? n : 0, memory, s, &m)))
    return rc;
  if (!src->mass) m = nullptr;
  const size_t cells = static_cast<size_t>(c.cfg.pm_grid_nx) * c.cfg.pm_grid_ny * c.cfg.pm_grid_nz;
  double* rho = density;
  chui::DevBuf tmp;
  if (memory == CHUI_TREEPM_HOST) {
    if (chui::ensure(tmp, cells * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    rho = tmp.as<double>();
  }
  rc = chui::pmDensityOnly(c, n, x, y, z, m, src->uniform_mass, rho, s);
  if (!rc && memory == CHUI_TREEPM_HOST) cudaMemcpyAsync(density, rho, cells * 8, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) rc = CHUI_TREEPM_EDEVICE;
  chui::release(tmp);
  return rc;
}

int chui_pm_cells(void* handle, const chui_treepm_sources* src, int64_t* cells, int memory, void* stream) {
  if (!handle || !src || !cells) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = src->count;
  const double *x, *y, *z;
  int rc;
  if ((rc = chui::stageIn(c, c.in_x, src->x, n, memory, s, &x)) || (rc = chui::stageIn(c, c.in_y, src->y, n, memory, s, &y)) ||
      (rc = chui::stageIn(c, c.in_z, src->z, n, memory, s, &z)))
    return rc;
  int64_t* out = cells;
  chui::DevBuf tmp;
  if (memory == CHUI_TREEPM_HOST) {
    if (chui::ensure(tmp, std::max<int64_t>(n, 1) * 3 * 8)) return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    out = tmp.as<int64_t>();
  }
  rc = chui::pmCells(c, n, x, y, z, out, s);
  if (!rc && memory == CHUI_TREEPM_HOST && n > 0) cudaMemcpyAsync(cells, out, n * 3 * 8, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) rc = CHUI_TREEPM_EDEVICE;
  chui::release(tmp);
  return rc;
}

int chui_treepm_tree_build_info(const void* handle, int32_t info[3]) {
  if (!handle || !info) return CHUI_TREEPM_EINVAL;
  const Context& c = *static_cast<const Context*>(handle);
  info[0] = c.unwrap_sorted_axes;
  info[1] = c.large_leaf;
  info[2] = c.path_levels_retried;
  return 0;
}

int chui_treepm_tree_node_count(const void* handle, int64_t* node_count) {
  if (!handle || !node_count) return CHUI_TREEPM_EINVAL;
  *node_count = static_cast<const Context*>(handle)->n_nodes;
  return 0;
}

int chui_treepm_dump_tree(void* handle, const chui_treepm_tree_dump* d) {
  if (!handle || !d) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  chui::DeviceGuard guard(c.device);
  const int64_t nn = c.n_nodes;
  if (cudaDeviceSynchronize() != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  // n is the size of the last solve's source set; sorted_index holds n entries
  const int64_t n = static_cast<int64_t>(c.sorted_index.bytes / 4);
  (void)n;
  auto copy = [](void* dst, const void* srcp, size_t bytes) {
    if (dst && bytes) cudaMemcpy(dst, srcp, bytes, cudaMemcpyDeviceToHost);
  };
  std::vector<double> geom(nn * 4), com(nn * 4), quad(nn * 8);
  std::vector<uint32_t> child(nn * 8);
  std::vector<uint4> range(nn);
  copy(geom.data(), c.node_geom.ptr, nn * 32);
  copy(com.data(), c.node_com.ptr, nn * 32);
  copy(quad.data(), c.node_quad.ptr, nn * 64);
  copy(child.data(), c.node_child.ptr, nn * 32);
  copy(range.data(), c.node_range.ptr, nn * 16);
  for (int64_t k = 0; k < nn; ++k) {
    if (d->center_x) d->center_x[k] = geom[4 * k];
    if (d->center_y) d->center_y[k] = geom[4 * k + 1];
    if (d->center_z) d->center_z[k] = geom[4 * k + 2];
    if (d->half_size) d->half_size[k] = geom[4 * k + 3];
    if (d->com_x) d->com_x[k] = com[4 * k];
    if (d->com_y) d->com_y[k] = com[4 * k + 1];
    if (d->com_z) d->com_z[k] = com[4 * k + 2];
    if (d->mass) d->mass[k] = com[4 * k + 3];
    double* qs[7] = {d->quad_xx, d->quad_xy, d->quad_xz, d->quad_yy, d->quad_yz, d->quad_zz, d->second_moment_trace};
    for (int q = 0; q < 7; ++q)
      if (qs[q]) qs[q][k] = quad[8 * k + q];
    if (d->child_count) d->child_count[k] = range[k].z;
    if (d->particle_begin) d->particle_begin[k] = range[k].x;
    if (d->particle_count) d->particle_count[k] = range[k].y;
    if (d->child_index)
      for (int o = 0; o < 8; ++o) d->child_index[8 * k + o] = child[8 * k + o];
  }
  return 0;
}

int chui_treepm_dump_particles(void* handle, int64_t n, double* ux, double* uy, double* uz, uint64_t* morton_sorted,
                               uint32_t* sorted_index, double anchors[3]) {
  if (!handle) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  chui::DeviceGuard guard(c.device);
  if (cudaDeviceSynchronize() != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  if (ux) cudaMemcpy(ux, c.ux.ptr, n * 8, cudaMemcpyDeviceToHost);
  if (uy) cudaMemcpy(uy, c.uy.ptr, n * 8, cudaMemcpyDeviceToHost);
  if (uz) cudaMemcpy(uz, c.uz.ptr, n * 8, cudaMemcpyDeviceToHost);
  if (morton_sorted) {
    // the tree build keeps each particle's key; the sorted list is formed here
    if (chui::ensure(c.keys_b, n * 8)) return CHUI_TREEPM_ENOMEM;
    const unsigned long long* kin = c.morton_keys.as<unsigned long long>();
    unsigned long long* kout = c.keys_b.as<unsigned long long>();
    if (int rc = chui::radixSortKeysU64(c, 1, &kin, &kout, n, 63, nullptr)) return rc;
    if (cudaMemcpy(morton_sorted, kout, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  }
  if (sorted_index) cudaMemcpy(sorted_index, c.sorted_index.ptr, n * 4, cudaMemcpyDeviceToHost);
  if (anchors)
    for (int a = 0; a < 3; ++a) anchors[a] = c.tree_anchor[a];
  return 0;
}

int chui_treepm_kick(void* handle, int64_t n, double* vx, double* vy, double* vz, const double* ax, const double* ay,
                     const double* az, double kick_factor, double drag_factor, int memory, void* stream) {
  if (!handle || n < 0) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  if (n == 0) return 0;
  chui::DeviceGuard guard(c.device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *dvx = vx, *dvy = vy, *dvz = vz;
  const double *dax = ax, *day = ay, *daz = az;
  if (memory == CHUI_TREEPM_HOST) {
    if (chui::ensure(c.in_x, n * 8) || chui::ensure(c.in_y, n * 8) || chui::ensure(c.in_z, n * 8) ||
        chui::ensure(c.out_acc[0], n * 8) || chui::ensure(c.out_acc[1], n * 8) || chui::ensure(c.out_acc[2], n * 8))
      return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    double* v[3] = {c.in_x.as<double>(), c.in_y.as<double>(), c.in_z.as<double>()};
    double* a[3] = {c.out_acc[0].as<double>(), c.out_acc[1].as<double>(), c.out_acc[2].as<double>()};
    const chui::HostLane lanes[6] = {{vx, v[0], vx}, {vy, v[1], vy}, {vz, v[2], vz},
                                     {ax, a[0], nullptr}, {ay, a[1], nullptr}, {az, a[2], nullptr}};
    const int rc = chui::pipelineHostStep(c, n, s, lanes, 6, [&](int64_t b, int64_t len, cudaStream_t st) {
      chui::noteLaunch();
      chui::kickKernel<<<chui::gridFor(len, 256), 256, 0, st>>>(len, v[0] + b, v[1] + b, v[2] + b, a[0] + b, a[1] + b,
                                                                a[2] + b, kick_factor, drag_factor);
    });
    if (rc) return chui::fail(c, rc, "kick failed");
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "kick failed");
  }
  { chui::noteLaunch(); chui::kickKernel<<<chui::gridFor(n, 256), 256, 0, s>>>(n, dvx, dvy, dvz, dax, day, daz, kick_factor, drag_factor); }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "kick failed");
}

int chui_treepm_drift(void* handle, int64_t n, double* x, double* y, double* z, const double* vx, const double* vy,
                      const double* vz, double drift_factor, int memory, void* stream) {
  if (!handle || n < 0) return CHUI_TREEPM_EINVAL;
  Context& c = *static_cast<Context*>(handle);
  if (n == 0) return 0;
  chui::DeviceGuard guard(c.device);
  // isolated/open boundaries: no wrap (box lengths 0 in the kernel)
  const bool periodic = c.cfg.boundary_condition == CHUI_TREEPM_BOUNDARY_PERIODIC;
  const double per_box[3] = {periodic ? c.cfg.box_x : 0.0, periodic ? c.cfg.box_y : 0.0, periodic ? c.cfg.box_z : 0.0};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *dx = x, *dy = y, *dz = z;
  const double *dvx = vx, *dvy = vy, *dvz = vz;
  if (memory == CHUI_TREEPM_HOST) {
    if (chui::ensure(c.in_x, n * 8) || chui::ensure(c.in_y, n * 8) || chui::ensure(c.in_z, n * 8) ||
        chui::ensure(c.out_acc[0], n * 8) || chui::ensure(c.out_acc[1], n * 8) || chui::ensure(c.out_acc[2], n * 8))
      return chui::fail(c, CHUI_TREEPM_ENOMEM, "allocation failed");
    double* p[3] = {c.in_x.as<double>(), c.in_y.as<double>(), c.in_z.as<double>()};
    double* v[3] = {c.out_acc[0].as<double>(), c.out_acc[1].as<double>(), c.out_acc[2].as<double>()};
    const chui::HostLane lanes[6] = {{x, p[0], x}, {y, p[1], y}, {z, p[2], z},
                                     {vx, v[0], nullptr}, {vy, v[1], nullptr}, {vz, v[2], nullptr}};
    const int rc = chui::pipelineHostStep(c, n, s, lanes, 6, [&](int64_t b, int64_t len, cudaStream_t st) {
      chui::noteLaunch();
      chui::driftKernel<<<chui::gridFor(len, 256), 256, 0, st>>>(len, p[0] + b, p[1] + b, p[2] + b, v[0] + b, v[1] + b,
                                                                 v[2] + b, drift_factor, per_box[0], per_box[1],
                                                                 per_box[2]);
    });
    if (rc) return chui::fail(c, rc, "drift failed");
  } else {
    chui::noteLaunch();
    chui::driftKernel<<<chui::gridFor(n, 256), 256, 0, s>>>(n, dx, dy, dz, dvx, dvy, dvz, drift_factor, per_box[0],
                                                           per_box[1], per_box[2]);
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : chui::fail(c, CHUI_TREEPM_EDEVICE, "drift failed");
}

}  // extern "C"

// ---- allocation-free density (chui_pm_assign_density_static) ----

// Accumulation grid of chui_pm_assign_density_static, one per device (module
// globals are per device). Zero at module load; every call zeroes it again
// before depositing.
static __device__ __align__(256) double g_static_density[CHUI_PM_STATIC_MAX_CELLS];

namespace {
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;                              // one call at a time per process
void* g_static_density_ptr[kStaticMaxDevices] = {};     // device address, looked up on first use

bool onDevice(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

int staticFail(int code, const std::string& msg) {
  g_create_error = msg;
  return code;
}
}  // namespace

extern "C" {

int chui_pm_assign_density_static(const chui_treepm_config* cfg, const chui_treepm_sources* src, double* density,
                                  int density_memory, void* stream) {
  if (!cfg || !src || !density) return staticFail(CHUI_TREEPM_EINVAL, "config, sources and density must be non-null");
  std::string err;
  int rc = chui::validateConfig(*cfg, err);
  if (rc) return staticFail(rc, err);
  const double cells_d = static_cast<double>(cfg->pm_grid_nx) * static_cast<double>(cfg->pm_grid_ny) *
                         static_cast<double>(cfg->pm_grid_nz);
  if (cells_d > static_cast<double>(CHUI_PM_STATIC_MAX_CELLS)) {
    return staticFail(CHUI_TREEPM_ERANGE, "PM mesh of " + std::to_string(static_cast<long long>(cells_d)) +
                                              " cells exceeds the static scratch grid of " +
                                              std::to_string(CHUI_PM_STATIC_MAX_CELLS) + " cells");
  }
  const size_t cells = static_cast<size_t>(cells_d);
  if (density_memory != CHUI_TREEPM_HOST && density_memory != CHUI_TREEPM_DEVICE)
    return staticFail(CHUI_TREEPM_EINVAL, "density_memory must be CHUI_TREEPM_HOST or CHUI_TREEPM_DEVICE");
  const int64_t n = src->count;
  if (n < 0) return staticFail(CHUI_TREEPM_EINVAL, "source count must be >= 0");
  if (n > 0 && (!src->x || !src->y || !src->z))
    return staticFail(CHUI_TREEPM_EINVAL, "source positions must be non-null");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return staticFail(CHUI_TREEPM_EDEVICE, "no CUDA device is available");
  if (cfg->device < 0 || cfg->device >= ndev || cfg->device >= kStaticMaxDevices)
    return staticFail(CHUI_TREEPM_EINVAL, "device ordinal out of range");

  std::lock_guard<std::mutex> lock(g_static_mutex);
  chui::DeviceGuard guard(cfg->device);
  if (n > 0 && (!onDevice(src->x, cfg->device) || !onDevice(src->y, cfg->device) ||
                !onDevice(src->z, cfg->device) || (src->mass && !onDevice(src->mass, cfg->device))))
    return staticFail(CHUI_TREEPM_EINVAL, "positions and masses must be device memory on the configured device");
  if (density_memory == CHUI_TREEPM_DEVICE && !onDevice(density, cfg->device))
    return staticFail(CHUI_TREEPM_EINVAL, "density must be device memory on the configured device");
  void*& scratch = g_static_density_ptr[cfg->device];
  if (scratch == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_density);
    if (e != cudaSuccess || p == nullptr)
      return staticFail(CHUI_TREEPM_EDEVICE, std::string("static scratch lookup failed: ") + cudaGetErrorString(e));
    scratch = p;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* grid = static_cast<double*>(scratch);
  rc = chui::pmDensityInto(*cfg, n, src->x, src->y, src->z, src->mass, src->uniform_mass, grid, s);
  if (rc) return staticFail(rc, "PM density launch failed");
  if (cudaMemcpyAsync(density, grid, cells * sizeof(double),
                      density_memory == CHUI_TREEPM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                      s) != cudaSuccess)
    return staticFail(CHUI_TREEPM_EDEVICE, "density copy failed");
  if (cudaStreamSynchronize(s) != cudaSuccess) return staticFail(CHUI_TREEPM_EDEVICE, "PM density kernels failed");
  return 0;
}

}  // extern "C"
