// Shared device/host helpers for the B200 TreePM kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <cmath>

namespace chui {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kMaxDepth = 64;            // tree_gravity.hpp:17 (kMaximumTreeDepth)
constexpr int kLevelsPerWord = 21;       // 3 octant bits per level, 63 bits per path word
// Grid of the reductions whose warps end in atomics on a few adjacent words:
// four blocks per SM keep those atomics (serialised on one L2 line) to a few
// thousand while the grid-stride loops still stream at full bandwidth.
constexpr unsigned kReduceBlocks = 148u * 4u;
constexpr int kLeafOrderMax = 1024;      // largest leaf ordered in place (larger: one more global sort)
constexpr int kMaxPathWords = 4;         // 84 levels > kMaxDepth
constexpr int kWalkWarpsPerBlock = 4;
constexpr int kStackCap = 1 + 7 * kMaxDepth;  // tree_pm_coupling.cpp:899-925 stack bound
constexpr int kPolyMaxTerms = 20;
#ifndef CHUI_PAIR_TERMS
#define CHUI_PAIR_TERMS 9
#endif
constexpr int kPairPolyTerms = CHUI_PAIR_TERMS;  // short form of the pair kernel's H(t) polynomial

// Status bits written by kernels instead of trapping.
enum StatusBits : uint32_t {
  kStatusOk = 0u,
  kStatusNonFinite = 1u << 0,
  kStatusStackOverflow = 1u << 1,
  kStatusDepthExceeded = 1u << 2,
  kStatusNeedMorePathWords = 1u << 3,
  kStatusNegativeMass = 1u << 4,
  kStatusIndexRange = 1u << 5,
  kStatusLargeLeaf = 1u << 6,  // a leaf above the within-leaf ordering limit (not an error)
};

// Periodic nearest-image metric (internal/tree_pm_geometry.hpp:12-32): bounded
// deltas use one conditional shift, the narrow tie band and unbounded deltas
// use delta - L*rint(delta/L).
struct Metric {
  double length;
  int bounded;
};

__host__ __device__ inline Metric makeMetric(double lo, double hi, double target, double length) {
  Metric m;
  m.length = length;
  m.bounded = isfinite(lo) && isfinite(hi) && (lo - target >= -length) && (hi - target <= length);
  return m;
}

__device__ __forceinline__ double applyMetric(const Metric& m, double delta) {
  if (!(m.length > 0.0)) return delta;
  const double half = 0.5 * m.length;
  if (!m.bounded || fabs(fabs(delta) - half) <= 4.0 * DBL_EPSILON * m.length) {
    return delta - m.length * rint(delta / m.length);
  }
  return delta > half ? delta - m.length : (delta < -half ? delta + m.length : delta);
}

// treePmSquaredDistanceWithinCutoff (internal/tree_pm_geometry.hpp:51-60).
__device__ __forceinline__ bool isNormalDouble(double v) {
  const double a = fabs(v);
  return a >= DBL_MIN && a <= DBL_MAX;
}

__device__ __forceinline__ bool withinCutoff(double d2, double cutoff, double cutoff2) {
  if (!isNormalDouble(cutoff2) || !isfinite(d2) || fabs(d2 - cutoff2) <= 8.0 * DBL_EPSILON * cutoff2) {
    return sqrt(d2) <= cutoff;
  }
  return d2 <= cutoff2;
}

// Order-preserving integer encoding of doubles for atomic min/max.
__host__ __device__ inline unsigned long long orderedBits(double v) {
  unsigned long long b;
  memcpy(&b, &v, sizeof(b));
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double fromOrderedBits(unsigned long long b) {
  b = (b & 0x8000000000000000ull) ? (b & 0x7FFFFFFFFFFFFFFFull) : ~b;
  double v;
  memcpy(&v, &b, sizeof(v));
  return v;
}

// --- Gaussian split law -----------------------------------------------------
// FP64 forms follow include/cosmosim/gravity/tree_pm_split_kernel.hpp.
__device__ inline double shortRangeFactor(double r, double rs) {
  if (r <= 0.0) return 1.0;
  const double q = (0.5 * r) / rs;
  if (isinf(q)) return 0.0;
  return erfc(q) + 2.0 * 0.564189583547756286948079451560772586 * q * exp(-q * q);
}

__device__ inline double longRangeFactor(double r, double rs) {
  if (r <= 0.0) return 0.0;
  const double q = (0.5 * r) / rs;
  if (isinf(q)) return 1.0;
  if (q < 0.125) {
    const double t = q * q;
    const double h = 4.0 * 0.564189583547756286948079451560772586 *
        (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
         t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
    return q * q * q * h;
  }
  return erf(q) - 2.0 * 0.564189583547756286948079451560772586 * q * exp(-q * q);
}

__device__ inline double coefficientSeries(double t) {
  return 2.25675833419102514779231780624309034 *
         (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
          t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
}

__device__ inline double longRangeInvR3(double r, double rs) {
  const double q = (0.5 * r) / rs;
  if (q < 0.125) return ((0.125 * coefficientSeries(q * q) / rs) / rs) / rs;
  return ((longRangeFactor(r, rs) / r) / r) / r;
}

__device__ inline double softenedInvR3(double r2, double eps) {
  const double s2 = r2 + eps * eps;
  if (s2 <= 0.0) return 0.0;
  return 1.0 / (s2 * sqrt(s2));
}

// K_soft - K_long (tree_pm_split_kernel.hpp:204-228).
__device__ inline double residualInvR3(double r2, double eps, double rs) {
  if (r2 <= 0.0) {
    if (eps == 0.0) return softenedInvR3(r2, eps);
    const double k = 0.094031597257959381158013241926795431;
    if (eps <= rs) {
      const double ratio = eps / rs;
      const double c = 1.0 - k * ratio * ratio * ratio;
      return ((c / eps) / eps) / eps;
    }
    const double ratio = rs / eps;
    const double c = ratio * ratio * ratio - k;
    return ((c / rs) / rs) / rs;
  }
  return softenedInvR3(r2, eps) - longRangeInvR3(sqrt(r2), rs);
}

// (dK/dr) / r of K = K_soft - K_long at r^2 = r2 > 0, FP64. K_long = H(t) / (8 r_s^3)
// with H(t) = L(q) / q^3, t = q^2 = r^2 / (4 r_s^2), L(q) = erf(q) - 2 q e^{-q^2} / sqrt(pi),
// so dK_long/dr / r = H'(t) / (16 r_s^5). H'(t) from its Taylor series
// (4/sqrt(pi)) sum_m (-1)^{m+1} t^m / (m! (2m+5)) for t < 1, else from
// H'(t) = (2/sqrt(pi)) e^{-t} / t - 1.5 L(sqrt t) / t^{5/2}.
__device__ inline double residualDerivOverR(double r2, double eps, double rs) {
  const double s2 = r2 + eps * eps;
  const double soft = -3.0 / (s2 * s2 * sqrt(s2));
  const double t = r2 / (4.0 * rs * rs);
  double hp;
  if (t < 1.0) {
    double sum = 0.0, term = 1.0;  // term = t^m / m!
    for (int k = 0; k <= 20; ++k) {
      const double v = term / (2.0 * k + 5.0);
      sum += (k & 1) ? v : -v;
      term *= t / (k + 1.0);
    }
    hp = 2.25675833419102514779231780624309034 * sum;
  } else {
    const double q = sqrt(t);
    const double e = exp(-t);
    const double L = erf(q) - 1.12837916709551257389615890312154517 * q * e;
    hp = 1.12837916709551257389615890312154517 * e / t - 1.5 * L / (t * t * q);
  }
  const double rs2 = rs * rs;
  return soft - hp / (16.0 * rs2 * rs2 * rs);
}

}  // namespace chui
