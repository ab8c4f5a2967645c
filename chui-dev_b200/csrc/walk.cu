// Short-range residual walk on the B200: the FLOP sink of the TreePM force.
//
// Reference: evaluateTargetAgainstLocalTree, tree_pm_coupling.cpp:4026-4272
// (per-target DFS, periodic node metric, AABB cutoff prune, leaf pairs with
// K_soft - K_long inside r_cut, strict acceptance of internal nodes,
// screened-quadrupole multipoles monopolePlusQuadrupoleAccelPeriodicReference
// :743-827, children pushed in reverse octant order :916-925).
//
// Design: one warp walks 32 targets that are consecutive in tree order
// (spatially coherent), sharing one DFS stack in shared memory. Every lane
// makes the reference's own decision for every node it reaches, in FP64
// (prune / leaf pairs / accept multipole / open); the warp descends into a
// node's children when any lane opens it, and a lane that pruned or accepted
// a node skips that node's subtree (nodes are numbered in preorder, so the
// subtree is the index range [node, subtree_end)). Each lane therefore sees
// exactly the nodes, pairs and multipoles of its own walk.
//
// Leaf sources are staged through shared memory per warp chunk of 32 and
// broadcast to the lanes. Mixed precision: each source is stored as an FP32
// offset from its leaf's FP64 centre; the target's offset to that centre is
// formed in FP64 (the node metric) and rounded once, so the pair separation
// is an FP32 difference of two small node-relative vectors. The residual
// kernel K = (r^2+eps^2)^-3/2 - H(t)/(8 r_s^3), t = r^2/(4 r_s^2), uses one
// rsqrt and a polynomial for H fitted per configuration (no erf/exp per
// pair). Per-leaf FP32 partial sums are added into FP64 accumulators. The
// FP64 configuration evaluates the reference's formulas (source metric per
// pair, erf/exp residual) unchanged.
//
// With diagnostics on, the walk reproduces the reference's node counters
// exactly. With diagnostics off (production), a small opened node is
// evaluated as one block of sources instead of being descended: its lanes
// get every source inside r_cut, which is the reference's pair set except
// where a deeper node would have been accepted as a strict multipole (those
// few are summed as pairs, which moves forces by far less than the mixed
// precision does); the number of warp traversal steps drops several-fold,
// and no counters are kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <type_traits>
#include <vector>

#include "context.cuh"

namespace chui {
namespace {

struct WalkArgs {
  int64_t nt;       // targets
  int64_t v0, v1;   // visit positions walked: [v0, v1) of the nt
  float* chunk_cost;  // SM cycles spent per 32 visit positions (index base / 32), nullable
  int out_compact;    // outputs at visit position - v0 (a visit-range solve) instead of the slot
  int64_t n;        // sources
  const uint32_t* order;   // visit position -> active slot
  const uint32_t* active;  // slot -> source row (nullable: slot == row)
  const double* tx;        // explicit target positions (nullable)
  const double* ty;
  const double* tz;
  const double* sx;        // caller source positions
  const double* sy;
  const double* sz;
  const uint32_t* pos_of_row;
  const double4* geom;
  const double4* com;
  const double* quad;
  const uint32_t* child;
  const uint4* range;
  const float4* src_f4;
  const double4* src_d4;
  const float4* node_f4;
  const float4* node_mq;   // per node 2 x float4: {mass, Mxx, Mxy, Mxz}, {Myy, Myz, Mzz, trace}
  const double4* src_u4;   // tree-ordered unwrapped positions + mass
  const double* prev;      // per slot |a_previous| (nullable: no history)
  // per-particle softening (all nullable: uniform wp.eps): tree-order and
  // row-order source epsilons, per-slot target epsilons, per-node {min, max}
  const double* src_eps;
  const double* row_eps;
  const double* tgt_eps;
  const double2* node_soft;
  // group walk
  const uint32_t* leaf_of_pos;  // tree position -> leaf node
  uint32_t* grp_start;          // visit position -> visit position of its group's first target
  double4* grp_rec;             // at a group start v: [2v] {centre, a_min}, [2v+1] {half, targets or 0 if ineligible}
  uint32_t* grp_list;           // eligible group starts
  unsigned char* grp_done;      // per slot: evaluated by the group walk
  const double2* gauss;         // Gaussian Hermite table {value, slope} (4097 knots)
  double* out_x;   // per slot, short-range part
  double* out_y;
  double* out_z;
  double* out_near;
  unsigned long long* counters;
  uint32_t* work;
  uint32_t* status;
  PolyH poly;
  PolyH dpoly;     // H'(t)
  PolyH ddpoly;    // H''(t)
  float inv_16rs5_f;
  float inv_32rs7_f;
  int mult_f32;    // accepted multipoles in FP32 (the split constants are normal floats)
  int mpoly12;     // H' and H'' fits have at most 12 terms
  // Packed (f32x2) operands of the pair loop, each value in both halves, so
  // that two queued sources share every FP32 instruction: the coefficients
  // of -H(t)/(8 r_s^3) (minus the long-range kernel K_long), the scale and
  // offset taking r^2 + eps^2 to the polynomial variable s = r^2 sc - 1, and
  // eps^2. cut2e = r_cut^2 + eps^2 is the cutoff test on r^2 + eps^2.
  float2 pk2[kPolyMaxTerms];
  float2 sc2, soff2, eps2_2;
  float2 mone2;  // {-1, -1}: s from r^2 itself (per-pair softening)
  float cut2e;
  // diagnostics 2 (or a requested nearest-pair lane): the counting instances
  // walk with subtree blocks (the production traversal) -- blocks -- and the
  // FP64 production walk counts and records nearest pairs -- instrument
  int blocks;
  int instrument;
  WalkParams wp;
};

__device__ __forceinline__ float polyH(const PolyH& p, float t) {
  const float s = fmaf(t, p.scale, -1.0f);
  float h = p.c[p.terms - 1];
  for (int k = p.terms - 2; k >= 0; --k) h = fmaf(h, s, p.c[k]);
  return h;
}

// Fixed-length Horner form (coefficients beyond p.terms are zero).
template <int kTerms>
__device__ __forceinline__ float polyHFixed(const PolyH& p, float t) {
  const float s = fmaf(t, p.scale, -1.0f);
  float h = p.c[kTerms - 1];
#pragma unroll
  for (int k = kTerms - 2; k >= 0; --k) h = fmaf(h, s, p.c[k]);
  return h;
}

// monopolePlusQuadrupoleAccelPeriodicReference (tree_pm_coupling.cpp:743-827), FP64.
__device__ __forceinline__ void multipoleForce(const WalkArgs& a, uint32_t node, double dx, double dy, double dz,
                               double eps_t, double& ax, double& ay, double& az) {
  const WalkParams& w = a.wp;
  const double rs = w.rs;
  const double4 cm = a.com[node];
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double safe_r2 = fmax(r2, 1.0e-30);
  const double r = sqrt(safe_r2);
  // max(node softening maximum, target) (tree_pm_coupling.cpp:749-757)
  const double pe = fmax(a.node_soft ? a.node_soft[node].y : w.eps, eps_t);
  const double denom = fmax(r2 + pe * pe, 1.0e-30);
  const double soft = 1.0 / (denom * sqrt(denom));
  const double split = shortRangeFactor(r, rs);
  const double newton = 1.0 / (safe_r2 * r);
  const double radial = soft + (split - 1.0) * newton;
  const double G = w.G;
  double fx = G * cm.w * radial * dx;
  double fy = G * cm.w * radial * dy;
  double fz = G * cm.w * radial * dz;
  if (w.quadrupole) {
    const double* q = a.quad + 8 * static_cast<size_t>(node);
    const double tr = q[6];
    const double mxx = (q[0] + tr) / 3.0, mxy = q[1] / 3.0, mxz = q[2] / 3.0;
    const double myy = (q[3] + tr) / 3.0, myz = q[4] / 3.0, mzz = (q[5] + tr) / 3.0;
    const double mdx = mxx * dx + mxy * dy + mxz * dz;
    const double mdy = mxy * dx + myy * dy + myz * dz;
    const double mdz = mxz * dx + myz * dy + mzz * dz;
    const double dmd = dx * mdx + dy * mdy + dz * mdz;
    const double k = 0.564189583547756286948079451560772586;
    const double rs2 = rs * rs;
    const double ex = exp(-r2 / (4.0 * rs2));
    const double sf = -0.5 * k * r2 * ex / (rs * rs2);
    const double ss = k * ex * (-r / (rs * rs2) + 0.25 * r * r2 / (rs * rs2 * rs2));
    const double s1 = -3.0 * r / (denom * denom * sqrt(denom));
    const double s2 = -3.0 / (denom * denom * sqrt(denom)) + 15.0 * r2 / (denom * denom * denom * sqrt(denom));
    const double n1 = -3.0 / (safe_r2 * safe_r2);
    const double n2 = 12.0 / (safe_r2 * safe_r2 * r);
    const double rf = s1 + sf * newton + (split - 1.0) * n1;
    const double rsec = s2 + ss * newton + 2.0 * sf * n1 + (split - 1.0) * n2;
    const double f1 = rf / r;
    const double cr = rsec / r2 - rf / (r2 * r);
    fx += G * (mdx * f1 + 0.5 * tr * dx * f1 + 0.5 * dx * dmd * cr);
    fy += G * (mdy * f1 + 0.5 * tr * dy * f1 + 0.5 * dy * dmd * cr);
    fz += G * (mdz * f1 + 0.5 * tr * dz * f1 + 0.5 * dz * dmd * cr);
  }
  ax += fx;
  ay += fy;
  az += fz;
}

// |d|^2 summed as the reference does, ((dx dx + dy dy) + dz dz) with every
// operation rounded on its own (no FMA contraction), so acceptance decisions
// see the reference's exact value.
__device__ __forceinline__ double norm2rn(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Per-target acceleration history: present and finite
// (tree_pm_coupling.cpp:4467-4472); magnitude 0 when absent.
struct History {
  bool avail;
  double mag;
};

__device__ __forceinline__ History loadHistory(const double* prev, uint32_t slot, bool valid) {
  History h{false, 0.0};
  if (prev && valid) {
    const double v = prev[slot];
    h.avail = isfinite(v);
    h.mag = h.avail ? v : 0.0;
  }
  return h;
}

// residualAccuracyProxy (internal/tree_pm_acceptance.hpp:20-51) with uniform
// softening (node softening max = the target's). Scalars by value: a
// reference into the kernel's parameter block would force a local copy of it.
__device__ __noinline__ double residualProxy(double G, double eps, double rs, double half, double com_offset,
                                            double mass, double r2) {
  if (!(r2 > 0.0) || !isfinite(r2)) return INFINITY;
  const double r = sqrt(r2);
  const double d = r2 + eps * eps;
  const double inv_d5 = 1.0 / (d * d * sqrt(d));
  const double inv_r3 = 1.0 / (r2 * r);
  const double inv_r4 = 1.0 / (r2 * r2);
  const double long_factor = longRangeFactor(r, rs);
  const double q = r / (2.0 * rs);
  const double exponential = exp(-q * q);
  const double k_inv_sqrt_pi = 0.564189583547756286948079451560772586;
  const double scale3 = rs * rs * rs;
  const double s_first = -0.5 * k_inv_sqrt_pi * r2 * exponential / scale3;
  const double s_second = k_inv_sqrt_pi * exponential * (-r / scale3 + 0.25 * r * r2 / (scale3 * rs * rs));
  const double first = -3.0 * r * inv_d5 + s_first * inv_r3 - 3.0 * (-long_factor) * inv_r4;
  const double second = -3.0 * inv_d5 + 15.0 * r2 * inv_d5 / d + s_second * inv_r3 - 6.0 * s_first * inv_r4 +
                        12.0 * (-long_factor) * inv_r4 / r;
  const double width = 2.0 * half;
  const double rho = sqrt(3.0) * half + com_offset;
  const double proxy =
      G * mass * fmax(width * width * inv_r4, 0.5 * rho * rho * (3.0 * fabs(first) + fabs(r * second - first)));
  return isfinite(proxy) && proxy >= 0.0 ? proxy : INFINITY;
}

// A target's softening: its own lane, else its source row's epsilon, else
// the configured one (targetSofteningEpsilonUnchecked, tree_softening.hpp:90-110).
__device__ __forceinline__ double targetEps(const WalkArgs& a, uint32_t slot, uint32_t row, bool valid) {
  if (!valid) return a.wp.eps;
  if (a.tgt_eps) return a.tgt_eps[slot];
  if (a.row_eps && row < a.n) return a.row_eps[row];
  return a.wp.eps;
}

// A source's softening by tree position.
__device__ __forceinline__ double sourceEps(const WalkArgs& a, uint32_t pos) {
  return a.src_eps ? a.src_eps[pos] : a.wp.eps;
}

// max(node softening maximum, target): the multipole and proxy softening.
__device__ __forceinline__ double nodeEps(const WalkArgs& a, uint32_t node, double eps_t) {
  return fmax(a.node_soft ? a.node_soft[node].y : a.wp.eps, eps_t);
}

// passesSofteningEnvelopeGuard (internal/tree_interaction_common.hpp:77-89)
// at r = sqrt(max(r^2, 1e-30)): nodes whose sources' softenings differ are
// accepted only beyond 2h + 2 max(node maximum, target).
__device__ __forceinline__ bool softeningGuard(const WalkArgs& a, uint32_t node, double half, double r2,
                                               double eps_t) {
  if (!a.node_soft) return true;
  const double2 ns = a.node_soft[node];
  if (ns.y - ns.x <= 1.0e-12) return true;
  return sqrt(fmax(r2, 1.0e-30)) > 2.0 * half + 2.0 * fmax(ns.y, eps_t);
}

// Acceptance of an internal node (acceptTreePmNode, internal/tree_pm_acceptance.hpp:53-139,
// with acceptNodeByMac and acceptNodeByComDistanceMac of
// internal/tree_interaction_common.hpp:36-75). Softening is uniform, so the
// softening envelope guard passes.
template <bool kAdaptive>
__device__ __forceinline__ bool acceptNode(const WalkParams& w, double half, double com_offset, double mass,
                                           bool inside, bool within, double r2, const History& hist,
                                           bool soft_ok = true, double eps_node = -1.0) {
  const double r = sqrt(fmax(r2, 1.0e-30));
  const double width = 2.0 * half;
  if (eps_node < 0.0) eps_node = w.eps;
  if (!soft_ok) return false;  // passesSofteningEnvelopeGuard
  if constexpr (!kAdaptive) {
    const bool envelope_ok = w.quadrupole && (width / r) < 0.08;
    bool mac_ok;
    if (inside) {
      mac_ok = false;
    } else if (w.criterion == 0) {
      mac_ok = (width / sqrt(r2 + 1.0e-30)) < w.theta;
    } else if (w.criterion == 1 || !hist.avail) {
      mac_ok = ((width + com_offset) / sqrt(r2 + 1.0e-30)) < w.theta;
    } else {
      const double scale = fmax(fabs(hist.mag), w.floor_);
      mac_ok = w.G * mass * width * width <= w.rel_tol * scale * r2 * r2;
    }
    return mac_ok && envelope_ok && within && !inside && isfinite(r2);
  }
  const bool envelope_ok = (width / r) < w.angle;
  if (!envelope_ok || inside || !within || !isfinite(r2)) return false;
  if (hist.avail && hist.mag > w.floor_) {
    const double allowance = w.rel_tol * hist.mag;
    const double inv_r4 = 1.0 / (r2 * r2);
    const double lower = w.G * mass * (width * width * inv_r4);
    if (isfinite(allowance) && isfinite(lower) && lower > allowance) return false;
    if (w.estimator == 1) return isfinite(allowance) && isfinite(lower);
    const double est = residualProxy(w.G, eps_node, w.rs, half, com_offset, mass, r2);
    return isfinite(est) && isfinite(allowance) && est <= allowance;
  }
  return ((width + com_offset) / sqrt(r2 + 1.0e-30)) < w.theta;
}

// ---- Gaussian pair lookup and the group walk (FP64) ------------------------

constexpr int kGaussCells = 4096;                  // tree_pm_split_kernel.hpp:136-138
constexpr double kGaussStep = 64.0 / kGaussCells;

// Cubic Hermite evaluation of H(t) from the reference's table
// (TreePmGaussianCoefficientTable::dimensionlessCoefficient, :150-164).
__device__ __forceinline__ double gaussHermite(const double2* g, double t) {
  const double cell = t / kGaussStep;
  const int i = static_cast<int>(cell);
  const double u = cell - static_cast<double>(i);
  const double u2 = u * u;
  const double u3 = u2 * u;
  const double2 k0 = g[i], k1 = g[i + 1];
  return (2 * u3 - 3 * u2 + 1) * k0.x + (u3 - 2 * u2 + u) * k0.y + (-2 * u3 + 3 * u2) * k1.x + (u3 - u2) * k1.y;
}

// Per-target direct pair with the Gaussian lookup (tree_pm_coupling.cpp:4221-4226).
__device__ __forceinline__ double gaussResidualInvR3(const WalkArgs& a, double r2, double eps) {
  const double rs = a.wp.rs;
  const double inv_2a2 = (0.25 / rs) / rs, inv_8a3 = ((0.125 / rs) / rs) / rs;
  const double t = r2 * inv_2a2;
  double long_inv_r3;
  if (t < 64.0) {
    const double coeff = t < 0.015625 ? coefficientSeries(t) : gaussHermite(a.gauss, t);
    long_inv_r3 = coeff * inv_8a3;
  } else {
    long_inv_r3 = longRangeInvR3(sqrt(r2), rs);
  }
  return softenedInvR3(r2, eps) - long_inv_r3;
}

// treePmGroupNearestImage (internal/tree_pm_group_walk.hpp:70-76), unfused:
// delta - L nearbyint(delta / L). The quotient only chooses the integer; a
// product with 1/L chooses the same one unless the quotient lies within 1e-6
// of a half-integer (the products differ by ulps), where the division is made.
__device__ __forceinline__ double groupImage(double delta, double length, double inv_length) {
  if (!(length > 0.0)) return delta;
  const double q = delta * inv_length;
  double k = rint(q);
  if (fabs(fabs(q - k) - 0.5) < 1.0e-6) k = rint(__ddiv_rn(delta, length));
  return __dsub_rn(delta, __dmul_rn(length, k));
}

struct GroupBox {
  double c[3], h[3], a_min;
};

// Node decision of the group walk (buildTreePmGroupInteractionList,
// internal/tree_pm_group_walk.hpp:78-154): 0 prune, 1 accept (leaf or
// multipole), 2 open. The reference's FP64 arithmetic, unfused.
__device__ __forceinline__ int groupDecisionNode(const WalkArgs& a, uint32_t node, const GroupBox& gb,
                                                 const double4 g, bool is_leaf) {
  const WalkParams& w = a.wp;
  const double h = g.w;
  const double cc[3] = {g.x, g.y, g.z};
  double gap2 = 0.0, far2 = 0.0;
  for (int ax = 0; ax < 3; ++ax) {
    const double d = fabs(groupImage(cc[ax] - gb.c[ax], w.box[ax], w.inv_box[ax]));
    const double gap = fmax(0.0, __dsub_rn(__dsub_rn(d, h), gb.h[ax]));
    const double far = __dadd_rn(__dadd_rn(d, h), gb.h[ax]);
    gap2 = __dadd_rn(gap2, __dmul_rn(gap, gap));
    far2 = __dadd_rn(far2, __dmul_rn(far, far));
  }
  if (gap2 > w.cutoff2) return 0;
  if (is_leaf) return 1;
  bool accept = gap2 > 0.0 && (w.com_cutoff || far2 <= w.cutoff2);
  if (accept) {
    const double4 cm = a.com[node];
    const double mc[3] = {cm.x, cm.y, cm.z};
    double r_min2 = 0.0;
    for (int ax = 0; ax < 3; ++ax) {
      const double gap = fmax(0.0, __dsub_rn(fabs(groupImage(mc[ax] - gb.c[ax], w.box[ax], w.inv_box[ax])), gb.h[ax]));
      r_min2 = __dadd_rn(r_min2, __dmul_rn(gap, gap));
    }
    const double width2 = 4.0 * h * h;
    const double rel_over_g = w.rel_tol / w.G;
    accept = r_min2 > 0.0 && width2 < (w.angle * w.angle) * r_min2 &&
             cm.w * width2 <= rel_over_g * gb.a_min * r_min2 * r_min2;
  }
  return accept ? 1 : 2;
}

__device__ __forceinline__ int groupDecision(const WalkArgs& a, uint32_t node, const GroupBox& gb) {
  return groupDecisionNode(a, node, gb, a.geom[node], a.range[node].z == 0);
}

inline unsigned groupGrid(int64_t n, int block) {
  const int64_t g = (n + block - 1) / block;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 64)));
}

__global__ void leafOfPosKernel(int64_t nodes, const uint4* __restrict__ range, uint32_t* leaf_of_pos) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nodes;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint4 rg = range[k];
    if (rg.z != 0) continue;
    for (uint32_t q = rg.x; q < rg.x + rg.y; ++q) leaf_of_pos[q] = static_cast<uint32_t>(k);
  }
}

__device__ __forceinline__ uint32_t leafOfVisit(const WalkArgs& a, int64_t v, uint32_t* slot_out, uint32_t* row_out) {
  const uint32_t slot = a.order[v];
  const uint32_t row = a.active ? a.active[slot] : slot;
  *slot_out = slot;
  *row_out = row;
  return row < a.n ? a.leaf_of_pos[a.pos_of_row[row]] : kInvalid;
}

// Groups: maximal runs of visit positions with the same source leaf inside one
// residual block of 64 (tree_pm_coupling.cpp:4498-4560, legacy grouping). At a
// group start: the group box (reference = first target, nearest-image deltas),
// the smallest previous |a|, and eligibility (every target with history above
// the floor and a bounded source metric; :4326-4368).
__global__ void groupSetupKernel(WalkArgs a, uint32_t* count) {
  const WalkParams& w = a.wp;
  // [v0, v1) starts and ends on a residual block boundary (or at nt), so no
  // group crosses it
  for (int64_t v = a.v0 + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < a.v1;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t slot, row;
    const uint32_t leaf = leafOfVisit(a, v, &slot, &row);
    const int64_t block0 = v & ~static_cast<int64_t>(63);
    int64_t st = v;
    if (leaf != kInvalid) {
      uint32_t s2, r2;
      while (st > block0 && leafOfVisit(a, st - 1, &s2, &r2) == leaf) --st;
    }
    a.grp_start[v] = static_cast<uint32_t>(st);
    if (st != v) continue;
    const int64_t block1 = min(block0 + 64, a.nt);
    int64_t e = v + 1;
    if (leaf != kInvalid) {
      uint32_t s2, r2;
      while (e < block1 && leafOfVisit(a, e, &s2, &r2) == leaf) ++e;
    }
    bool ok = leaf != kInvalid;
    double ref[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, a_min = INFINITY;
    for (int64_t q = v; q < e && ok; ++q) {
      uint32_t sq, rq;
      leafOfVisit(a, q, &sq, &rq);
      const double pv = a.prev ? a.prev[sq] : NAN;
      if (!(isfinite(pv) && pv > w.floor_)) {
        ok = false;
        break;
      }
      a_min = fmin(a_min, pv);
      const double pos[3] = {a.tx ? a.tx[sq] : a.sx[rq], a.ty ? a.ty[sq] : a.sy[rq], a.tz ? a.tz[sq] : a.sz[rq]};
      for (int ax = 0; ax < 3; ++ax) {
        if (!makeMetric(w.src_lo[ax], w.src_hi[ax], pos[ax], w.box[ax]).bounded) ok = false;
        if (q == v) {
          ref[ax] = pos[ax];
          continue;
        }
        const double d = groupImage(pos[ax] - ref[ax], w.box[ax], w.inv_box[ax]);
        lo[ax] = fmin(lo[ax], d);
        hi[ax] = fmax(hi[ax], d);
      }
    }
    double c[3], h[3];
    for (int ax = 0; ax < 3; ++ax) {
      c[ax] = ref[ax] + 0.5 * (lo[ax] + hi[ax]);
      h[ax] = 0.5 * (hi[ax] - lo[ax]);
    }
    a.grp_rec[2 * v] = make_double4(c[0], c[1], c[2], a_min);
    a.grp_rec[2 * v + 1] = make_double4(h[0], h[1], h[2], ok ? static_cast<double>(e - v) : 0.0);
    if (ok) a.grp_list[atomicAdd(count, 1u)] = static_cast<uint32_t>(v);
  }
}

// The FP64 group walk: one warp per eligible group (its targets on the lanes,
// 32 at a time), one warp-uniform walk building the shared list; each lane
// evaluates the accepted leaves' pairs with the Hermite table (leaves whose
// cell lies beyond r_cut are culled per target, as the reference does) and the
// accepted multipoles at its own COM distance (pruned beyond r_cut under
// COM-distance cutoff nodes), accumulateTreePmGroupCulledLeaves and
// evaluate_target_group (tree_pm_coupling.cpp:4369-4420). Summation order:
// leaves and multipoles as the walk meets them.
__global__ void __launch_bounds__(kWalkWarpsPerBlock * 32) groupWalkKernel(WalkArgs a, const uint32_t* groups,
                                                                           uint32_t n_groups) {
  __shared__ uint32_t stack_sm[kWalkWarpsPerBlock][kStackCap];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint32_t* stack = stack_sm[warp];
  const WalkParams& w = a.wp;
  const double lx = w.box[0], ly = w.box[1], lz = w.box[2];
  const double inv_2a2 = (0.25 / w.rs) / w.rs, inv_8a3 = ((0.125 / w.rs) / w.rs) / w.rs;
  const double t_limit = 63.99999999999999;  // nextafter(64, 0)
  const double eps2 = w.eps * w.eps;
  const double cull2 = w.cutoff2 * (1.0 + 1.0e-9);
  unsigned long long cnt_visited = 0, cnt_accepted = 0, cnt_opened = 0, cnt_pairs = 0, cnt_pruned = 0,
                     cnt_multi = 0, cnt_leaves = 0;
  for (uint32_t gi = blockIdx.x * kWalkWarpsPerBlock + warp; gi < n_groups; gi += gridDim.x * kWalkWarpsPerBlock) {
    const uint32_t v0 = groups[gi];
    const double4 r0 = a.grp_rec[2 * static_cast<size_t>(v0)], r1 = a.grp_rec[2 * static_cast<size_t>(v0) + 1];
    GroupBox gb;
    gb.c[0] = r0.x; gb.c[1] = r0.y; gb.c[2] = r0.z; gb.a_min = r0.w;
    gb.h[0] = r1.x; gb.h[1] = r1.y; gb.h[2] = r1.z;
    const int count = static_cast<int>(r1.w);
    for (int chunk = 0; chunk < count; chunk += 32) {
      const bool valid = chunk + lane < count;
      uint32_t slot = 0, row = kInvalid;
      double px = 0.0, py = 0.0, pz = 0.0;
      if (valid) {
        leafOfVisit(a, v0 + chunk + lane, &slot, &row);
        px = a.tx ? a.tx[slot] : a.sx[row];
        py = a.ty ? a.ty[slot] : a.sy[row];
        pz = a.tz ? a.tz[slot] : a.sz[row];
      }
      const uint32_t self_pos = (valid && row < a.n) ? a.pos_of_row[row] : kInvalid;
      const double toff[3] = {groupImage(px - gb.c[0], lx, w.inv_box[0]), groupImage(py - gb.c[1], ly, w.inv_box[1]),
                                groupImage(pz - gb.c[2], lz, w.inv_box[2])};
      Metric nm[3];
      const double pt[3] = {px, py, pz};
      for (int ax = 0; ax < 3; ++ax) nm[ax] = makeMetric(w.node_lo[ax], w.node_hi[ax], pt[ax], w.box[ax]);
      const bool count_walk = lane == 0 && chunk == 0;
      double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0, nearest = INFINITY;
      if (lane == 0) stack[0] = 0u;
      int sp = 1;
      __syncwarp();
      bool overflow = false;
      while (sp > 0) {
        const uint32_t node = stack[sp - 1];
        --sp;
        __syncwarp();
        const int d = groupDecision(a, node, gb);  // identical on every lane
        if (count_walk) {
          ++cnt_visited;
          cnt_pruned += d == 0 ? 1 : 0;
        }
        if (d == 0) continue;
        const uint4 rg = a.range[node];
        if (d == 1 && rg.z == 0) {
          if (count_walk) {
            ++cnt_leaves;
            ++cnt_accepted;
          }
          if (valid) {
            const double4 g = a.geom[node];
            const double h = g.w;
            const double lc[3] = {groupImage(g.x - gb.c[0], lx, w.inv_box[0]), groupImage(g.y - gb.c[1], ly, w.inv_box[1]),
                                  groupImage(g.z - gb.c[2], lz, w.inv_box[2])};
            double g2 = 0.0;
            for (int ax = 0; ax < 3; ++ax) {
              const double off = lc[ax] - toff[ax], hl = 0.5 * w.box[ax];
              const double dd = off > hl ? off - w.box[ax] : (off < -hl ? off + w.box[ax] : off);
              const double gg = fmax(0.0, fabs(dd) - h);
              g2 = __dadd_rn(g2, __dmul_rn(gg, gg));
            }
            if (!(g2 > cull2)) {
              double sx = 0.0, sy = 0.0, sz = 0.0;
              for (uint32_t j = rg.x; j < rg.x + rg.y; ++j) {
                const double4 sv = a.src_d4[j];
                double dx = sv.x - px, dy = sv.y - py, dz = sv.z - pz;
                dx = dx > 0.5 * lx ? dx - lx : (dx < -0.5 * lx ? dx + lx : dx);
                dy = dy > 0.5 * ly ? dy - ly : (dy < -0.5 * ly ? dy + ly : dy);
                dz = dz > 0.5 * lz ? dz - lz : (dz < -0.5 * lz ? dz + lz : dz);
                const double r2 = norm2rn(dx, dy, dz);
                const bool inside = j != self_pos && r2 <= w.cutoff2;
                const double t = fmin(r2 * inv_2a2, t_limit);
                const double coeff_long = gaussHermite(a.gauss, t) * inv_8a3;
                const double dn = r2 + eps2;
                const double softened = 1.0 / (dn * sqrt(dn));
                const double factor = (inside && r2 > 0.0) ? (softened - coeff_long) * w.G * sv.w : 0.0;
                sx += factor * dx;
                sy += factor * dy;
                sz += factor * dz;
                cnt_pairs += inside ? 1 : 0;
                nearest = inside ? fmin(nearest, r2) : nearest;
              }
              acc_x += sx;
              acc_y += sy;
              acc_z += sz;
            }
          }
          continue;
        }
        if (d == 1) {
          if (count_walk) {
            ++cnt_multi;
            ++cnt_accepted;
          }
          if (valid) {
            const double4 cm = a.com[node];
            const double dx = applyMetric(nm[0], cm.x - px);
            const double dy = applyMetric(nm[1], cm.y - py);
            const double dz = applyMetric(nm[2], cm.z - pz);
            if (w.com_cutoff && norm2rn(dx, dy, dz) > w.cutoff2) {
              ++cnt_pruned;
            } else {
              multipoleForce(a, node, dx, dy, dz, w.eps, acc_x, acc_y, acc_z);
            }
          }
          continue;
        }
        if (count_walk) ++cnt_opened;
        const uint32_t ch = lane < 8 ? a.child[8 * static_cast<size_t>(node) + lane] : kInvalid;
        const unsigned cmask = __ballot_sync(0xffffffffu, ch != kInvalid) & 0xFFu;
        const int nc = __popc(cmask);
        if (sp + nc > kStackCap) {
          overflow = true;
          break;
        }
        if (ch != kInvalid) stack[sp + __popc(cmask >> (lane + 1))] = ch;
        sp += nc;
        __syncwarp();
      }
      if (overflow && lane == 0) atomicOr(a.status, kStatusStackOverflow);
      if (valid) {
        const int64_t o = a.out_compact ? static_cast<int64_t>(v0) + chunk + lane - a.v0 : slot;
        a.out_x[o] = acc_x;
        a.out_y[o] = acc_y;
        a.out_z[o] = acc_z;
        a.out_near[o] = nearest;
        a.grp_done[slot] = 1;
      }
      __syncwarp();
    }
  }
  unsigned long long c[8] = {cnt_visited, cnt_accepted, cnt_opened, cnt_pairs, cnt_pruned, 0ull, cnt_multi, cnt_leaves};
  for (int k = 0; k < 8; ++k) {
    for (int off = 16; off > 0; off >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], off);
  }
  if (lane == 0) {
    for (int k = 0; k < 8; ++k) atomicAdd(a.counters + k, c[k]);
  }
}

template <bool kMixed, bool kEpsZero>
__global__ void __launch_bounds__(kWalkWarpsPerBlock * 32) walkKernel(WalkArgs a) {
  __shared__ uint32_t stack_sm[kWalkWarpsPerBlock][kStackCap];
  __shared__ long long item_start_sm[kWalkWarpsPerBlock];
  __shared__ float4 src_f_sm[kWalkWarpsPerBlock][32];
  __shared__ double4 src_d_sm[kWalkWarpsPerBlock][32];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint32_t* stack = stack_sm[warp];
  const WalkParams& w = a.wp;
  unsigned long long cnt_visited = 0, cnt_accepted = 0, cnt_opened = 0, cnt_pairs = 0, cnt_pruned = 0,
                     cnt_skips = 0, cnt_multi = 0, cnt_leaves = 0;

  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = static_cast<uint32_t>(a.v0) + atomicAdd(a.work, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= a.v1) break;
    if (lane == 0 && a.chunk_cost) item_start_sm[warp] = clock64();
    const int64_t v = static_cast<int64_t>(base) + lane;
    const bool valid = v < a.v1;
    uint32_t slot = 0, row = kInvalid;
    double px = 0.0, py = 0.0, pz = 0.0;
    if (valid) {
      slot = a.order[v];
      row = a.active ? a.active[slot] : slot;
      if (a.tx) {
        px = a.tx[slot];
        py = a.ty[slot];
        pz = a.tz[slot];
      } else {
        px = a.sx[row];
        py = a.sy[row];
        pz = a.sz[row];
      }
    }
    const bool skip_self = valid && row < a.n;
    const uint32_t self_pos = skip_self ? a.pos_of_row[row] : kInvalid;
    const double eps_t = targetEps(a, slot, row, valid);
    const History hist = loadHistory(a.prev, slot, valid);
    // targets the group walk evaluated take no per-target walk
    const bool grouped = valid && a.grp_done != nullptr && a.grp_done[slot] != 0;
    Metric sm[3], nm[3];
    const double pt[3] = {px, py, pz};
    for (int ax_ = 0; ax_ < 3; ++ax_) {
      sm[ax_] = makeMetric(w.src_lo[ax_], w.src_hi[ax_], pt[ax_], w.box[ax_]);
      nm[ax_] = makeMetric(w.node_lo[ax_], w.node_hi[ax_], pt[ax_], w.box[ax_]);
    }
    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    double nearest = INFINITY;
    float nearest_f = INFINITY;
    uint32_t skip_until = 0;
    int sp = 0;
    if (lane == 0) stack[0] = 0u;
    sp = 1;
    __syncwarp();
    bool overflow = false;
    while (sp > 0) {
      const uint32_t node = stack[sp - 1];
      --sp;
      __syncwarp();
      const bool act = valid && !grouped && node >= skip_until;
      if (!__any_sync(0xffffffffu, act)) continue;
      const double4 g = a.geom[node];
      const uint4 rg = a.range[node];
      const double h = g.w;
      const double ndx = applyMetric(nm[0], g.x - px);
      const double ndy = applyMetric(nm[1], g.y - py);
      const double ndz = applyMetric(nm[2], g.z - pz);
      const double ax_abs = fabs(ndx), ay_abs = fabs(ndy), az_abs = fabs(ndz);
      const double ex = fmax(0.0, ax_abs - h), ey = fmax(0.0, ay_abs - h), ez = fmax(0.0, az_abs - h);
      bool prune = !withinCutoff(ex * ex + ey * ey + ez * ez, w.cutoff, w.cutoff2);
      if (act) {
        ++cnt_visited;
        cnt_pruned += prune ? 1 : 0;
      }
      const bool is_leaf = rg.z == 0;
      if (is_leaf) {
        const bool want = act && !prune;
        if (!__any_sync(0xffffffffu, want)) continue;
        if (want) {
          ++cnt_accepted;
          ++cnt_leaves;
        }
        const uint32_t begin = rg.x, count = rg.y;
        // Node-relative FP32 offsets select the right periodic image only for
        // leaves smaller than L/2 - r_cut; larger (tiny-N) leaves use the exact path.
        if (kMixed && h < w.exact_half) {
          const float ndfx = static_cast<float>(ndx), ndfy = static_cast<float>(ndy),
                      ndfz = static_cast<float>(ndz);
          float fx = 0.f, fy = 0.f, fz = 0.f;
          for (uint32_t chunk = 0; chunk < count; chunk += 32) {
            const uint32_t k = chunk + lane;
            if (k < count) src_f_sm[warp][lane] = a.src_f4[begin + k];
            __syncwarp();
            const uint32_t m = min(32u, count - chunk);
            if (want) {
              for (uint32_t j = 0; j < m; ++j) {
                const float4 s = src_f_sm[warp][j];
                const float dx = s.x + ndfx, dy = s.y + ndfy, dz = s.z + ndfz;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const bool in = r2 <= w.cut2_f && (begin + chunk + j) != self_pos;
                cnt_pairs += in ? 1 : 0;
                cnt_skips += (!in && (begin + chunk + j) != self_pos) ? 1 : 0;
                nearest_f = in ? fminf(nearest_f, r2) : nearest_f;
                const float t = r2 * w.inv_4rs2_f;
                const float hh = polyH(a.poly, t);
                const float s2 = kEpsZero ? r2 : r2 + w.eps2_f;
                const float rinv = rsqrtf(s2);
                const float k3 = fmaf(-hh, w.inv_8rs3_f, rinv * rinv * rinv);
                const float f = (in && r2 > 0.f) ? w.G_f * s.w * k3 : 0.f;
                fx = fmaf(f, dx, fx);
                fy = fmaf(f, dy, fy);
                fz = fmaf(f, dz, fz);
              }
            }
            __syncwarp();
          }
          acc_x += static_cast<double>(fx);
          acc_y += static_cast<double>(fy);
          acc_z += static_cast<double>(fz);
        } else {
          float nearest_mixed = INFINITY;
          for (uint32_t chunk = 0; chunk < count; chunk += 32) {
            const uint32_t k = chunk + lane;
            if (k < count) src_d_sm[warp][lane] = a.src_d4[begin + k];
            __syncwarp();
            const uint32_t m = min(32u, count - chunk);
            if (want) {
              for (uint32_t j = 0; j < m; ++j) {
                if ((begin + chunk + j) == self_pos) continue;
                const double4 s = src_d_sm[warp][j];
                const double dx = applyMetric(sm[0], s.x - px);
                const double dy = applyMetric(sm[1], s.y - py);
                const double dz = applyMetric(sm[2], s.z - pz);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > w.cutoff2) {
                  ++cnt_skips;
                  continue;
                }
                nearest = fmin(nearest, r2);
                nearest_mixed = fminf(nearest_mixed, static_cast<float>(r2));
                ++cnt_pairs;
                if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
                // max(source, target) softening (tree_pm_coupling.cpp:4208-4212)
                const double pe = fmax(sourceEps(a, begin + chunk + j), eps_t);
                const double f = (w.gauss_lookup && r2 > 0.0 ? gaussResidualInvR3(a, r2, pe)
                                                             : residualInvR3(r2, pe, w.rs)) *
                                 w.G;
                acc_x += f * s.w * dx;
                acc_y += f * s.w * dy;
                acc_z += f * s.w * dz;
              }
            }
            __syncwarp();
          }
          nearest_f = fminf(nearest_f, nearest_mixed);
        }
        continue;
      }
      // internal node
      const double4 cm = a.com[node];
      const double off = a.quad[8 * static_cast<size_t>(node) + 7];
      // the adaptive policy tests containment for every target (tree_pm_coupling.cpp:4090-4092)
      const bool inside = (skip_self || w.policy == 1) && ax_abs <= h && ay_abs <= h && az_abs <= h;
      const double mx = ax_abs + h, my = ay_abs + h, mz = az_abs + h;
      const bool within = w.com_cutoff || withinCutoff(mx * mx + my * my + mz * mz, w.cutoff, w.cutoff2);
      const double dx = applyMetric(nm[0], cm.x - px);
      const double dy = applyMetric(nm[1], cm.y - py);
      const double dz = applyMetric(nm[2], cm.z - pz);
      const double r2 = norm2rn(dx, dy, dz);
      bool accept = act && !prune &&
                    (w.policy == 1 ? acceptNode<true>(w, h, off, cm.w, inside, within, r2, hist,
                                                      softeningGuard(a, node, h, r2, eps_t), nodeEps(a, node, eps_t))
                                   : acceptNode<false>(w, h, off, cm.w, inside, within, r2, hist,
                                                       softeningGuard(a, node, h, r2, eps_t), nodeEps(a, node, eps_t)));
      // COM-distance cutoff nodes: accepted beyond r_cut means pruned (:4129-4132)
      if (accept && w.com_cutoff && r2 > w.cutoff2) {
        accept = false;
        prune = true;
        ++cnt_pruned;
      }
      const bool open = act && !prune && !accept;
      if (accept) {
        ++cnt_accepted;
        ++cnt_multi;
        multipoleForce(a, node, dx, dy, dz, eps_t, acc_x, acc_y, acc_z);
      }
      if (act && (prune || accept)) skip_until = rg.w;
      if (open) ++cnt_opened;
      if (__any_sync(0xffffffffu, open)) {
        const uint32_t ch = lane < 8 ? a.child[8 * static_cast<size_t>(node) + lane] : kInvalid;
        const unsigned mask = __ballot_sync(0xffffffffu, ch != kInvalid) & 0xFFu;
        const int nc = __popc(mask);
        if (sp + nc > kStackCap) {
          overflow = true;
          break;
        }
        if (ch != kInvalid) {
          // highest octant deepest in the stack: octant 0 is popped first
          const int pos = sp + __popc(mask >> (lane + 1));
          stack[pos] = ch;
        }
        sp += nc;
        __syncwarp();
      }
    }
    if (overflow) {
      if (lane == 0) atomicOr(a.status, kStatusStackOverflow);
    }
    if constexpr (kMixed) nearest = static_cast<double>(nearest_f);
    if (valid && !grouped) {
      const int64_t o = a.out_compact ? v - a.v0 : slot;
      a.out_x[o] = acc_x;
      a.out_y[o] = acc_y;
      a.out_z[o] = acc_z;
      a.out_near[o] = nearest;
    }
    if (lane == 0 && a.chunk_cost) a.chunk_cost[base >> 5] = static_cast<float>(clock64() - item_start_sm[warp]);
    __syncwarp();
  }
  // counters: warp reduction then one atomic each
  unsigned long long c[8] = {cnt_visited, cnt_accepted, cnt_opened, cnt_pairs,
                             cnt_pruned, cnt_skips, cnt_multi, cnt_leaves};
  for (int k = 0; k < 8; ++k) {
    for (int off = 16; off > 0; off >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], off);
  }
  if (lane == 0) {
    for (int k = 0; k < 8; ++k) atomicAdd(a.counters + k, c[k]);
  }
}

constexpr int kQueue = 64;   // sources per warp batch
constexpr int kMultList = 4; // accepted multipoles per lane before a flush (4 against 8: group walk 209 -> 202 ms)

// Subtree blocks of the production walk (diagnostics off): an opened node
// with at most kBulkCount sources and half-size at most kBulkHalf * r_cut is
// evaluated as one block of sources by the lanes that opened it.
#ifndef CHUI_BULK_COUNT
#define CHUI_BULK_COUNT 2048  // 1024: 192.8 ms, 2048: 190.3, 4096: 190.4 at 256^3 (strict, packed pair loop)
#endif
#ifndef CHUI_BULK_HALF
#define CHUI_BULK_HALF 1.0
#endif
#ifndef CHUI_PAIR_UNROLL
#define CHUI_PAIR_UNROLL 4  // source pairs per unrolled step of the pair loop
#endif
#ifndef CHUI_WALK_MIN_BLOCKS_STRICT
#define CHUI_WALK_MIN_BLOCKS_STRICT 6  // the strict, uniform-mass production instances (80 registers)
#endif
#ifndef CHUI_WALK_MIN_BLOCKS
#define CHUI_WALK_MIN_BLOCKS 5  // resident blocks per SM the register budget is sized for
#endif
#ifndef CHUI_WALK_MIN_BLOCKS_ADAPTIVE
#define CHUI_WALK_MIN_BLOCKS_ADAPTIVE 6  // the adaptive, uniform-mass production instances (fast deck: 149.8 -> 147.2 ms at 256^3)
#endif
// Under the adaptive policy most opened nodes have deeper accepted
// multipoles, so blocks pay only for small nodes; evaluating their sources as
// pairs is at least as accurate as the multipoles it replaces.
#ifndef CHUI_BULK_COUNT_ADAPTIVE
#define CHUI_BULK_COUNT_ADAPTIVE 256
#endif
constexpr uint32_t kBulkCount = CHUI_BULK_COUNT;
#ifndef CHUI_BULK_COUNT_VJP
#define CHUI_BULK_COUNT_VJP 1024  // the adjoint walk's blocks
#endif
constexpr uint32_t kBulkCountVjp = CHUI_BULK_COUNT_VJP;
constexpr uint32_t kBulkCountAdaptive = CHUI_BULK_COUNT_ADAPTIVE;
constexpr double kBulkHalf = CHUI_BULK_HALF;
constexpr int kPairUnroll = CHUI_PAIR_UNROLL;

// The fitted polynomial at t = r^2 / (4 r_s^2), straight from r^2: s =
// r^2 * sc - 1 with sc = scale / (4 r_s^2), then Horner (kTerms - 1 FMAs).
// The walk is issue-bound, so the fewest instructions win over a shorter
// dependency chain (the unrolled queue loop supplies the parallelism).
template <int kTerms>
__device__ __forceinline__ float hornerR2(const PolyH& p, float r2, float sc) {
  const float s = fmaf(r2, sc, -1.0f);
  float h = p.c[kTerms - 1];
#pragma unroll
  for (int k = kTerms - 2; k >= 0; --k) h = fmaf(h, s, p.c[k]);
  return h;
}

// The same Horner chain for two sources at once (packed FP32: one f32x2 FMA
// per term serves both halves); c2 holds each coefficient in both halves,
// s = r2 * sc2 + off2.
template <int kTerms>
__device__ __forceinline__ float2 hornerR2x2(const float2* c2, float2 r2, float2 sc2, float2 off2) {
  const float2 s = __ffma2_rn(r2, sc2, off2);
  float2 h = c2[kTerms - 1];
#pragma unroll
  for (int k = kTerms - 2; k >= 0; --k) h = __ffma2_rn(h, s, c2[k]);
  return h;
}

// monopolePlusQuadrupoleAccelPeriodicReference (tree_pm_coupling.cpp:743-827)
// in FP32, without the G factor, added to (fx, fy, fz). With t = r^2/(4 r_s^2)
// and H the fitted long-range kernel: K = (r^2+eps^2)^-3/2 - H(t)/(8 r_s^3),
// K'/r = -3 (r^2+eps^2)^-5/2 - H'(t)/(16 r_s^5) and
// (K'' - K'/r)/r^2 = 15 (r^2+eps^2)^-7/2 - H''(t)/(32 r_s^7); the force is
// M K d + f1 (Md + tr d / 2) + cr (d.Md) d / 2 with f1 = K'/r, cr the last.
template <bool kEpsZero, int kTerms>
__device__ __forceinline__ void multipoleF32(const WalkArgs& a, uint32_t node, float dx, float dy, float dz, float sc,
                                             float& fx, float& fy, float& fz, float eps2) {
  const float4 q0 = a.node_mq[2 * static_cast<size_t>(node)];
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float den = kEpsZero ? r2 : r2 + eps2;
  const float rinv = rsqrtf(den);
  const float rinv2 = rinv * rinv;
  const float rinv3 = rinv2 * rinv;
  const float k = fmaf(-hornerR2<kTerms>(a.poly, r2, sc), a.wp.inv_8rs3_f, rinv3);
  float s = q0.x * k;
  if (a.wp.quadrupole) {
    const float4 q1 = a.node_mq[2 * static_cast<size_t>(node) + 1];
    const float rinv5 = rinv3 * rinv2;
    // H' and H'' have their own fitted lengths (warp-uniform choice)
    const float h1 = a.mpoly12 ? hornerR2<12>(a.dpoly, r2, sc) : hornerR2<kPolyMaxTerms>(a.dpoly, r2, sc);
    const float h2 = a.mpoly12 ? hornerR2<12>(a.ddpoly, r2, sc) : hornerR2<kPolyMaxTerms>(a.ddpoly, r2, sc);
    const float f1 = fmaf(-h1, a.inv_16rs5_f, -3.0f * rinv5);
    const float cr = fmaf(-h2, a.inv_32rs7_f, 15.0f * rinv5 * rinv2);
    const float mdx = fmaf(q0.y, dx, fmaf(q0.z, dy, q0.w * dz));
    const float mdy = fmaf(q0.z, dx, fmaf(q1.x, dy, q1.y * dz));
    const float mdz = fmaf(q0.w, dx, fmaf(q1.y, dy, q1.z * dz));
    const float dmd = fmaf(dx, mdx, fmaf(dy, mdy, dz * mdz));
    s = fmaf(0.5f, fmaf(q1.w, f1, dmd * cr), s);
    fx = fmaf(mdx, f1, fmaf(s, dx, fx));
    fy = fmaf(mdy, f1, fmaf(s, dy, fy));
    fz = fmaf(mdz, f1, fmaf(s, dz, fz));
  } else {
    fx = fmaf(s, dx, fx);
    fy = fmaf(s, dy, fy);
    fz = fmaf(s, dz, fz);
  }
}

// Exact (FP64, reference formulas) decision for one lane at one node: prune,
// and for internal nodes accept/open, plus the COM offset for a multipole.
struct ExactDecision {
  bool prune, accept;
  double dx, dy, dz;
};

template <bool kAdaptive>
__device__ __forceinline__ ExactDecision exactNodeDecision(const WalkArgs& a, uint32_t node, double px, double py,
                                                        double pz, bool skip_self, const History& hist,
                                                        double eps_t) {
  const WalkParams& w = a.wp;
  ExactDecision d{};
  const double4 g = a.geom[node];
  const uint4 rg4 = a.range[node];
  const Metric mx = makeMetric(w.node_lo[0], w.node_hi[0], px, w.box[0]);
  const Metric my = makeMetric(w.node_lo[1], w.node_hi[1], py, w.box[1]);
  const Metric mz = makeMetric(w.node_lo[2], w.node_hi[2], pz, w.box[2]);
  const double h = g.w;
  const double ndx = applyMetric(mx, g.x - px), ndy = applyMetric(my, g.y - py), ndz = applyMetric(mz, g.z - pz);
  const double ax = fabs(ndx), ay = fabs(ndy), az = fabs(ndz);
  const double ex = fmax(0.0, ax - h), ey = fmax(0.0, ay - h), ez = fmax(0.0, az - h);
  d.prune = !withinCutoff(ex * ex + ey * ey + ez * ez, w.cutoff, w.cutoff2);
  d.accept = false;
  if (d.prune || rg4.z == 0) return d;
  const double4 cm = a.com[node];
  const double off = a.quad[8 * static_cast<size_t>(node) + 7];
  const bool inside = (skip_self || kAdaptive) && ax <= h && ay <= h && az <= h;
  const double qx = ax + h, qy = ay + h, qz = az + h;
  const bool within = (kAdaptive && w.com_cutoff) || withinCutoff(qx * qx + qy * qy + qz * qz, w.cutoff, w.cutoff2);
  d.dx = applyMetric(mx, cm.x - px);
  d.dy = applyMetric(my, cm.y - py);
  d.dz = applyMetric(mz, cm.z - pz);
  const double r2 = norm2rn(d.dx, d.dy, d.dz);
  d.accept = acceptNode<kAdaptive>(w, h, off, cm.w, inside, within, r2, hist, softeningGuard(a, node, h, r2, eps_t),
                                   nodeEps(a, node, eps_t));
  if (kAdaptive && d.accept && w.com_cutoff && r2 > w.cutoff2) {  // accepted beyond r_cut: pruned
    d.accept = false;
    d.prune = true;
  }
  return d;
}

// Exact FP64 pairs of one leaf for the lanes in `want` (reference formulas,
// per-pair source metric): used where the shared FP32 frame cannot serve.
__device__ __forceinline__ void exactLeafPairs(const WalkArgs& a, double4* stage, uint32_t begin, uint32_t count,
                                            bool want, double px, double py, double pz, uint32_t self_pos, double eps_t,
                                            double& ax, double& ay, double& az, double& nearest,
                                            unsigned long long& pairs, unsigned long long& skips) {
  const WalkParams& w = a.wp;
  const int lane = threadIdx.x & 31;
  const Metric mx = makeMetric(w.src_lo[0], w.src_hi[0], px, w.box[0]);
  const Metric my = makeMetric(w.src_lo[1], w.src_hi[1], py, w.box[1]);
  const Metric mz = makeMetric(w.src_lo[2], w.src_hi[2], pz, w.box[2]);
  for (uint32_t chunk = 0; chunk < count; chunk += 32) {
    const uint32_t k = chunk + lane;
    if (k < count) stage[lane] = a.src_d4[begin + k];
    __syncwarp();
    const uint32_t m = min(32u, count - chunk);
    if (want) {
      for (uint32_t j = 0; j < m; ++j) {
        if ((begin + chunk + j) == self_pos) continue;
        const double4 sv = stage[j];
        const double dx = applyMetric(mx, sv.x - px), dy = applyMetric(my, sv.y - py), dz = applyMetric(mz, sv.z - pz);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > w.cutoff2) {
          ++skips;
          continue;
        }
        nearest = fmin(nearest, r2);
        ++pairs;
        if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
        const double f = residualInvR3(r2, fmax(sourceEps(a, begin + chunk + j), eps_t), w.rs) * w.G;
        ax += f * sv.w * dx;
        ay += f * sv.w * dy;
        az += f * sv.w * dz;
      }
    }
    __syncwarp();
  }
}

// Nearest image of a frame offset on an axis of length L (inv_l = 1/L); L = 0
// (isolated/open boundaries) has no images. The reciprocal replaces a division
// per axis and node: the shared frame is only used where offsets stay well
// inside half a box, so the rounding of d/L cannot pick another image.
__device__ __forceinline__ double frameImage(double d, double L, double inv_l) {
  return L > 0.0 ? d - L * rint(d * inv_l) : d;
}

// Comparison a < b decided in FP32 with a guard band (relative, plus an
// absolute bound `err` on the inputs' own error): returns +1 (certainly true),
// -1 (certainly false) or 0 (too close to call in FP32).
__device__ __forceinline__ int certainLess(float a, float b, float err = 0.f) {
  const float band = fmaf(2.0e-5f, fabsf(a) + fabsf(b), err) + 1.0e-30f;
  if (a < b - band) return 1;
  if (a > b + band) return -1;
  return 0;
}

// Mixed-precision walk (the product path).
//
// Traversal order and every per-lane decision are those of the reference's
// evaluateTargetAgainstLocalTree. Each warp works in one FP64 reference frame
// (its first target): a node's centre offset is formed once in FP64 and
// rounded, and each lane decides prune / accept / open in FP32 with a guard
// band; only lanes whose FP32 test lands inside the band re-decide with the
// exact FP64 reference arithmetic, so decisions equal the reference's.
// Accepted leaves are appended to a shared-memory queue (sources outside the
// group's cutoff sphere are dropped at enqueue) tagged with the ballot of
// accepting lanes, and evaluated 64 sources at a time in FP32.
// kMode: 0 strict policy without acceleration history, 1 strict policy with
// the relative-force MAC and history, 2 adaptive-relative policy, 3 adaptive
// with the group walk: lanes whose group is eligible take their group's
// decision (made in FP64 by the group's first lane in the warp and broadcast),
// the others the per-target adaptive decision.
// kUniform (production, contiguous targets, one source mass): queue entries
// carry the lane mask in place of the mass, so each entry is one 16-byte load
// and the mass multiplies the flush's partial sums once.
//
// kF64 (strict policy, no diagnostics): the same traversal, decisions and
// subtree blocks with every pair in FP64 -- queue entries are FP64 offsets
// formed from the tree-frame FP64 positions, pairs take the reference's
// formulas (erf/exp residual, or its Gaussian table) and accepted multipoles
// the FP64 screened quadrupole. This is the production solver in FP64, the
// comparator for the mixed-precision speed-up.
//
// kSoft: per-particle softening -- each queued source carries its epsilon,
// pairs take max(source, target), multipoles max(node maximum, target), and
// nodes whose sources' softenings differ are decided in FP64 (the envelope
// guard); masses travel with the sources.
template <bool kEpsZero, int kTerms, bool kDiag, bool kContiguous, int kMode, bool kUniform = false,
          bool kCost = false, bool kF64 = false, bool kSoft = false>
__global__ void __launch_bounds__(kWalkWarpsPerBlock * 32,
                                  (kMode == 0 && kUniform)   ? CHUI_WALK_MIN_BLOCKS_STRICT
                                  : (kMode == 2 && kUniform) ? CHUI_WALK_MIN_BLOCKS_ADAPTIVE
                                                             : CHUI_WALK_MIN_BLOCKS)
    walkFastKernel(WalkArgs a) {
  static_assert(!kF64 || (kMode <= 1 && !kDiag && !kUniform), "FP64 production walk: strict policy only");
  static_assert(!kSoft || (!kUniform && !kEpsZero && !kF64 && kMode <= 2), "per-particle softening instances");
  // counters and the nearest-pair lane: the counting instances (kDiag), and
  // the FP64 production walk on request
  const bool inst = kDiag || (kF64 && a.instrument != 0);
  constexpr bool kAdaptive = kMode >= 2;
  constexpr bool kGroup = kMode == 3;
  constexpr bool kHistory = kMode != 0;
  constexpr int kList = kAdaptive ? kMultList : 1;
  // sources per warp batch: longer for the strict walk (fewer flushes; 256
  // against 64 took 224.1 to 219.8 ms at 256^3), the adaptive instances'
  // shared memory (lane multipole lists) keeps them at 64 for occupancy
  constexpr int kQueueLen = kAdaptive ? kQueue : 4 * kQueue;
  static_assert(kQueueLen % 2 == 0, "the queue holds pairs of sources");
  __shared__ long long item_start_sm[kWalkWarpsPerBlock];
  __shared__ uint32_t stack_sm[kWalkWarpsPerBlock][kStackCap];
  // The queue holds sources in pairs, laid out for packed FP32 evaluation:
  // pair p is q_src[2p] = {x0, x1, y0, y1}, q_src[2p+1] = {z0, z1, w0, w1}
  // (w: mass, or the lane mask under kUniform), and q_meta[p] = {mask0,
  // mask1, tree position 0, tree position 1} when masses travel separately.
  __shared__ float4 q_src[kWalkWarpsPerBlock][kF64 ? 2 : kQueueLen];
  __shared__ uint4 q_meta[kWalkWarpsPerBlock][kF64 ? 1 : kQueueLen / 2];
  // kSoft: each queued source's softening (entry k at [k]; a pair reads a float2)
  __shared__ __align__(8) float q_eps[kWalkWarpsPerBlock][kSoft ? kQueueLen : 2];
  // kF64: FP64 offsets + mass, and {lane mask, tree position}
  constexpr int kQ64 = kF64 ? kQueueLen / 2 : 1;
  __shared__ double4 q64[kWalkWarpsPerBlock][kQ64];
  __shared__ uint2 q64m[kWalkWarpsPerBlock][kQ64];
  __shared__ float4 m_list[kWalkWarpsPerBlock][kList][32];
  __shared__ double4 exact_sm[kWalkWarpsPerBlock][32];
  // per-lane FP64 target position and accumulators, kept in shared memory
  // rather than registers: they are touched once per flush or exact decision,
  // and the registers they would hold buy the pair loop occupancy and ILP
  __shared__ double lane_sm[kF64 ? 9 : 6][kWalkWarpsPerBlock][32];
  // group walk: each deciding lane's group box {centre, half, a_min}, read at
  // every node visit (components outermost: no bank conflicts)
  __shared__ double gbox_sm[kGroup ? 7 : 1][kWalkWarpsPerBlock][32];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t lane_bit = 1u << lane;
  uint32_t* stack = stack_sm[warp];
  const WalkParams& w = a.wp;
  // no image ambiguity without periodic boundaries
  const double half_min_box = w.box[0] > 0.0 ? 0.5 * fmin(w.box[0], fmin(w.box[1], w.box[2])) : INFINITY;
  const double* inv_l = w.inv_box;
  const float cut2 = w.cut2_f;
  const float cut_f = static_cast<float>(w.cutoff);
  const float env2 = 0.0064f;  // 0.08^2
  const float theta2 = static_cast<float>(w.theta * w.theta);
  const float angle2 = static_cast<float>(w.angle * w.angle);
  const double bulk_half = kBulkHalf * w.cutoff;
  const float sc_r2 = w.inv_4rs2_f * a.poly.scale;
  const float g_pair = kUniform ? w.G_f * w.m0_f : w.G_f;  // factor on the flush's partial sums

  while (true) {
    uint32_t cnt_visited = 0, cnt_accepted = 0, cnt_opened = 0, cnt_pairs = 0, cnt_pruned = 0, cnt_skips = 0,
             cnt_multi = 0, cnt_leaves = 0;
    uint32_t base = 0;
    if (lane == 0) base = static_cast<uint32_t>(a.v0) + atomicAdd(a.work, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= a.v1) break;
    if constexpr (kCost) {
      // reading the clock costs the walk ~1.5 % in code generation, so only
      // the instances behind a visit-range solve do it
      if (lane == 0) item_start_sm[warp] = clock64();
    }
    const int64_t v = static_cast<int64_t>(base) + lane;
    const bool valid = v < a.v1;
    uint32_t slot = 0, row = kInvalid;
    double& px = lane_sm[0][warp][lane];
    double& py = lane_sm[1][warp][lane];
    double& pz = lane_sm[2][warp][lane];
    px = 0.0;
    py = 0.0;
    pz = 0.0;
    if (valid) {
      slot = a.order[v];
      row = a.active ? a.active[slot] : slot;
      if (a.tx) {
        px = a.tx[slot];
        py = a.ty[slot];
        pz = a.tz[slot];
      } else {
        px = a.sx[row];
        py = a.sy[row];
        pz = a.sz[row];
      }
    }
    const double rx = __shfl_sync(0xffffffffu, px, 0);
    const double ry = __shfl_sync(0xffffffffu, py, 0);
    const double rz = __shfl_sync(0xffffffffu, pz, 0);
    double ox = px - rx, oy = py - ry, oz = pz - rz;
    ox = frameImage(ox, w.box[0], inv_l[0]);
    oy = frameImage(oy, w.box[1], inv_l[1]);
    oz = frameImage(oz, w.box[2], inv_l[2]);
    double rga = valid ? fmax(fabs(ox), fmax(fabs(oy), fabs(oz))) : 0.0;
    double rg2 = valid ? ox * ox + oy * oy + oz * oz : 0.0;
    for (int off = 16; off > 0; off >>= 1) {
      rga = fmax(rga, __shfl_xor_sync(0xffffffffu, rga, off));
      rg2 = fmax(rg2, __shfl_xor_sync(0xffffffffu, rg2, off));
    }
    const float tfx = static_cast<float>(ox), tfy = static_cast<float>(oy), tfz = static_cast<float>(oz);
    if constexpr (kF64) {
      lane_sm[6][warp][lane] = ox;
      lane_sm[7][warp][lane] = oy;
      lane_sm[8][warp][lane] = oz;
    }
    // FP64 cull radius of the queue (kF64): r_cut + the warp's target spread
    const double cull2d = kF64 ? (w.cutoff + sqrt(rg2)) * (w.cutoff + sqrt(rg2)) * (1.0 + 1.0e-12) : 0.0;
    const float cull = static_cast<float>(w.cutoff + sqrt(rg2));
    const float cull2 = cull * cull * 1.0001f;
    const float rga_f = static_cast<float>(rga);
    const bool skip_self = valid && row < a.n;
    const uint32_t self_pos = skip_self ? a.pos_of_row[row] : kInvalid;
    const History hist = loadHistory(kHistory ? a.prev : nullptr, slot, valid);
    // the target's softening (uniform: the configured one)
    const double eps_t_d = kSoft ? targetEps(a, slot, row, valid) : w.eps;
    const float eps_t_f = static_cast<float>(eps_t_d);
    // group walk: the lane's group (start visit position), eligibility, and the
    // lane deciding for it in this warp (the group's first lane here); only the
    // warp holding a group's first target counts the group walk's node counters
    uint32_t g_start = 0;
    bool in_group = false;
    int leader = lane;
    bool count_walk = false;
    if constexpr (kGroup) {
      g_start = valid ? a.grp_start[v] : 0xFFFFFFFFu;
      in_group = valid && a.grp_rec[2 * static_cast<size_t>(g_start) + 1].w > 0.0;
      const uint32_t up = __shfl_up_sync(0xffffffffu, g_start, 1);
      const unsigned run_start = __ballot_sync(0xffffffffu, lane == 0 || up != g_start);
      leader = 31 - __clz(run_start & ((2u << lane) - 1u));
      count_walk = in_group && leader == lane && static_cast<int64_t>(g_start) == v;
      if (in_group && leader == lane) {
        const double4 r0 = a.grp_rec[2 * static_cast<size_t>(g_start)];
        const double4 r1 = a.grp_rec[2 * static_cast<size_t>(g_start) + 1];
        gbox_sm[0][warp][lane] = r0.x;
        gbox_sm[1][warp][lane] = r0.y;
        gbox_sm[2][warp][lane] = r0.z;
        gbox_sm[3][warp][lane] = r1.x;
        gbox_sm[4][warp][lane] = r1.y;
        gbox_sm[5][warp][lane] = r1.z;
        gbox_sm[6][warp][lane] = r0.w;
      }
      __syncwarp();
    }
    // relative criterion in FP32: the allowance alpha |a_prev| (adaptive, with
    // usable history) or alpha max(|a_prev|, floor) (strict relative MAC, any
    // finite history); FP32 tests are used only where it is a normal float
    const bool rel_test = kAdaptive ? (hist.avail && hist.mag > w.floor_) : (kHistory && hist.avail);
    float allow_f = 0.f;
    if (rel_test) {
      allow_f = static_cast<float>(kAdaptive ? w.rel_tol * hist.mag : w.rel_tol * fmax(fabs(hist.mag), w.floor_));
      if (!(allow_f >= FLT_MIN && allow_f <= FLT_MAX)) allow_f = 0.f;  // FP32 cannot decide: exact path
    }
    double& acc_x = lane_sm[3][warp][lane];
    double& acc_y = lane_sm[4][warp][lane];
    double& acc_z = lane_sm[5][warp][lane];
    acc_x = 0.0;
    acc_y = 0.0;
    acc_z = 0.0;
    float nearest_f = INFINITY;
    double nearest_d = INFINITY;  // FP64 pairs (exact leaf pairs, the FP64 production walk)
    uint32_t skip_until = 0;
    int qn = 0;  // warp's source queue length
    int mn = 0;  // this lane's multipole list length
    if (lane == 0) stack[0] = 0u;
    int sp = 1;
    __syncwarp();
    bool overflow = false;

    // Pair loop over the queue, two sources per step in packed FP32 (f32x2
    // FMA/ADD/MUL: one instruction serves both sources of a pair); lane
    // masks, cutoff tests and rsqrt stay per source.
    auto flush32 = [&]() {
      if (qn & 1) {
        // pad to whole pairs with an entry no lane takes (mask 0, mass 0)
        if (lane == 0) {
          float* qf = reinterpret_cast<float*>(&q_src[warp][qn - 1]);
          qf[1] = 0.f;
          qf[3] = 0.f;
          qf[5] = 0.f;
          qf[7] = 0.f;
          if constexpr (!kUniform) {
            uint32_t* qm = reinterpret_cast<uint32_t*>(&q_meta[warp][qn >> 1]);
            qm[1] = 0u;
            qm[3] = kInvalid;
          }
          if constexpr (kSoft) q_eps[warp][qn] = 0.f;
        }
        __syncwarp();
      }
      const float2 ntx = make_float2(-tfx, -tfx), nty = make_float2(-tfy, -tfy), ntz = make_float2(-tfz, -tfz);
      float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;
      uint32_t pairs = 0, skips = 0;
      const int np = (qn + 1) >> 1;
      auto pairStep = [&](auto count_tag, int p, float2& fx, float2& fy, float2& fz) {
        constexpr bool kCount = decltype(count_tag)::value;
        const float4 A = q_src[warp][2 * p];
        const float4 B = q_src[warp][2 * p + 1];
        const float2 dx = __fadd2_rn(make_float2(A.x, A.y), ntx);
        const float2 dy = __fadd2_rn(make_float2(A.z, A.w), nty);
        const float2 dz = __fadd2_rn(make_float2(B.x, B.y), ntz);
        // r^2 + eps^2 in one chain (eps^2 is the first addend); the polynomial
        // variable and the cutoff test take it with eps^2 folded into their
        // constants. Diagnostics test the cutoff on r^2 itself, as the
        // reference does, and report it for the nearest pair.
        // kSoft: r^2, then r^2 + max(eps_source, eps_target)^2 per source
        float2 r2e, r2;
        if constexpr (kSoft) {
          r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
          const float2 es = *reinterpret_cast<const float2*>(&q_eps[warp][2 * p]);
          const float2 ep = make_float2(fmaxf(es.x, eps_t_f), fmaxf(es.y, eps_t_f));
          r2e = __ffma2_rn(ep, ep, r2);
        } else {
          r2e = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, a.eps2_2)));
          r2 = kDiag ? __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz))) : r2e;
        }
        const float cut_t = (kDiag || kSoft) ? cut2 : a.cut2e;
        bool mine0, mine1;
        if constexpr (kUniform) {
          mine0 = (__float_as_uint(B.z) & lane_bit) != 0u;
          mine1 = (__float_as_uint(B.w) & lane_bit) != 0u;
        } else {
          const uint4 M = q_meta[warp][p];
          mine0 = kContiguous ? (M.x & lane_bit) != 0u : ((M.x & lane_bit) != 0u && M.z != self_pos);
          mine1 = kContiguous ? (M.y & lane_bit) != 0u : ((M.y & lane_bit) != 0u && M.w != self_pos);
        }
        const bool in0 = mine0 && r2.x <= cut_t;
        const bool in1 = mine1 && r2.y <= cut_t;
        if constexpr (kCount) {
          pairs += (in0 ? 1u : 0u) + (in1 ? 1u : 0u);
          // the group walk's pair kernel counts no skipped pairs
          skips += ((mine0 && !in0 && !in_group) ? 1u : 0u) + ((mine1 && !in1 && !in_group) ? 1u : 0u);
          nearest_f = in0 ? fminf(nearest_f, r2.x) : nearest_f;
          nearest_f = in1 ? fminf(nearest_f, r2.y) : nearest_f;
        }
        const float2 klong = kSoft ? hornerR2x2<kTerms>(a.pk2, r2, a.sc2, a.mone2)     // -K_long
                                   : hornerR2x2<kTerms>(a.pk2, r2e, a.sc2, a.soff2);
        const float2 rinv = make_float2(rsqrtf(r2e.x), rsqrtf(r2e.y));
        float2 k3 = __ffma2_rn(__fmul2_rn(rinv, rinv), rinv, klong);  // K_soft - K_long
        if constexpr (!kUniform) k3 = __fmul2_rn(k3, make_float2(B.z, B.w));
        // coincident sources contribute nothing: with eps > 0 the kernel is
        // finite there and d = 0; with eps = 0 the zero-distance test avoids inf * 0
        const float2 f = make_float2((kEpsZero ? (in0 && r2e.x > 0.f) : in0) ? k3.x : 0.f,
                                     (kEpsZero ? (in1 && r2e.y > 0.f) : in1) ? k3.y : 0.f);
        fx = __ffma2_rn(f, dx, fx);
        fy = __ffma2_rn(f, dy, fy);
        fz = __ffma2_rn(f, dz, fz);
      };
#pragma unroll (kPairUnroll)
      for (int p = 0; p < np; ++p) pairStep(std::integral_constant<bool, kDiag>{}, p, fx, fy, fz);
      acc_x += static_cast<double>(g_pair * (fx.x + fx.y));
      acc_y += static_cast<double>(g_pair * (fy.x + fy.y));
      acc_z += static_cast<double>(g_pair * (fz.x + fz.y));
      cnt_pairs += pairs;
      cnt_skips += skips;
      qn = 0;
      __syncwarp();
    };

    // kF64: every queued source in FP64 with the reference's pair formula.
    auto flush64 = [&]() {
      const double tx = lane_sm[6][warp][lane], ty = lane_sm[7][warp][lane], tz = lane_sm[8][warp][lane];
      double fx = 0.0, fy = 0.0, fz = 0.0;
      for (int k = 0; k < qn; ++k) {
        const double4 e = q64[warp][k];
        const uint2 meta = q64m[warp][k];
        const double dx = e.x - tx, dy = e.y - ty, dz = e.z - tz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const bool mine = (meta.x & lane_bit) != 0u && (kContiguous || meta.y != self_pos);
        const bool in = mine && r2 <= w.cutoff2 && (!kEpsZero || r2 > 0.0);
        if (inst) {
          cnt_pairs += in ? 1u : 0u;
          cnt_skips += (mine && !in) ? 1u : 0u;
          nearest_d = in ? fmin(nearest_d, r2) : nearest_d;
        }
        if (in) {
          const double pe = fmax(sourceEps(a, meta.y), eps_t_d);
          const double kr = w.gauss_lookup ? gaussResidualInvR3(a, r2, pe) : residualInvR3(r2, pe, w.rs);
          const double f = kr * e.w;
          fx += f * dx;
          fy += f * dy;
          fz += f * dz;
        }
      }
      acc_x += w.G * fx;
      acc_y += w.G * fy;
      acc_z += w.G * fz;
      qn = 0;
      __syncwarp();
    };
    auto flush = [&]() {
      if constexpr (kF64) flush64();
      else flush32();
    };

    // Accepted multipoles wait in a per-lane list and are evaluated together:
    // the lanes step through their own lists in lockstep, so a warp pays for
    // the longest list rather than for every node some lane accepted.
    auto mflush = [&]() {
      const int kmax = __reduce_max_sync(0xffffffffu, mn);
      float fx = 0.f, fy = 0.f, fz = 0.f;
      for (int k = 0; k < kmax; ++k) {
        if (k < mn) {
          const float4 e = m_list[warp][k][lane];
          const uint32_t mnode = __float_as_uint(e.w);
          float me2 = w.eps2_f;
          if constexpr (kSoft) {
            const float me = static_cast<float>(nodeEps(a, mnode, eps_t_d));
            me2 = me * me;
          }
          multipoleF32<kEpsZero, kTerms>(a, mnode, e.x, e.y, e.z, sc_r2, fx, fy, fz, me2);
        }
      }
      acc_x += static_cast<double>(w.G_f * fx);
      acc_y += static_cast<double>(w.G_f * fy);
      acc_z += static_cast<double>(w.G_f * fz);
      mn = 0;
      __syncwarp();
    };

    // Append sources [begin, begin+count) for the lanes in `mask`, as FP32
    // offsets from the warp's reference target; sources outside the group's
    // cutoff sphere are dropped. Leaf records are offsets from the leaf centre
    // (src_f4); subtree blocks read tree-frame FP64 positions (src_u4). Either
    // way the offset is formed in FP64 and rounded once.
    auto enqueue = [&](uint32_t begin, uint32_t count, uint32_t mask, bool whole, const double4& g, double cdx,
                       double cdy, double cdz) {
      if constexpr (kF64) {
        for (uint32_t chunk = 0; chunk < count; chunk += 32) {
          const uint32_t k = chunk + lane;
          double4 e = make_double4(0.0, 0.0, 0.0, 0.0);
          bool keep = false;
          if (k < count) {
            const double4 u = a.src_u4[begin + k];
            e = make_double4((u.x - g.x) + cdx, (u.y - g.y) + cdy, (u.z - g.z) + cdz, u.w);
            keep = e.x * e.x + e.y * e.y + e.z * e.z <= cull2d;
          }
          const uint32_t keep_mask = __ballot_sync(0xffffffffu, keep);
          const int c = __popc(keep_mask);
          if (qn + c > kQ64) flush();
          if (keep) {
            const int slot_q = qn + __popc(keep_mask & (lane_bit - 1u));
            uint32_t m = mask;
            if constexpr (kContiguous) {
              const uint32_t rel = begin + k - base;
              if (rel < 32u) m &= ~(1u << rel);
            }
            q64[warp][slot_q] = e;
            q64m[warp][slot_q] = make_uint2(m, begin + k);
          }
          __syncwarp();
          qn += c;
        }
        return;
      }
      for (uint32_t chunk = 0; chunk < count; chunk += 32) {
        const uint32_t k = chunk + lane;
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
        bool keep = false;
        if (k < count) {
          if (whole) {
            const double4 u = a.src_u4[begin + k];
            e = make_float4(static_cast<float>((u.x - g.x) + cdx), static_cast<float>((u.y - g.y) + cdy),
                            static_cast<float>((u.z - g.z) + cdz), static_cast<float>(u.w));
          } else {
            const float4 sv = a.src_f4[begin + k];
            e = make_float4(static_cast<float>(static_cast<double>(sv.x) + cdx),
                            static_cast<float>(static_cast<double>(sv.y) + cdy),
                            static_cast<float>(static_cast<double>(sv.z) + cdz), sv.w);
          }
          keep = fmaf(e.x, e.x, fmaf(e.y, e.y, e.z * e.z)) <= cull2;
        }
        const uint32_t keep_mask = __ballot_sync(0xffffffffu, keep);
        const int c = __popc(keep_mask);
        if (qn + c > kQueueLen) flush();
        if (keep) {
          const int slot_q = qn + __popc(keep_mask & (lane_bit - 1u));
          uint32_t m = mask;
          if constexpr (kContiguous) {
            // targets are tree positions base..base+31: drop the source's own lane
            const uint32_t rel = begin + k - base;
            if (rel < 32u) m &= ~(1u << rel);
          }
          // pair layout (see q_src): entry slot_q is half (slot_q & 1) of pair slot_q / 2
          float* qf = reinterpret_cast<float*>(&q_src[warp][slot_q & ~1]);
          const int hq = slot_q & 1;
          qf[hq] = e.x;
          qf[2 + hq] = e.y;
          qf[4 + hq] = e.z;
          qf[6 + hq] = kUniform ? __uint_as_float(m) : e.w;
          if constexpr (!kUniform) {
            uint32_t* qm = reinterpret_cast<uint32_t*>(&q_meta[warp][slot_q >> 1]);
            qm[hq] = m;
            qm[2 + hq] = begin + k;
          }
          if constexpr (kSoft) q_eps[warp][slot_q] = static_cast<float>(sourceEps(a, begin + k));
        }
        __syncwarp();
        qn += c;
      }
    };

    while (sp > 0) {
      const uint32_t node = stack[sp - 1];
      --sp;
      __syncwarp();
      const bool act = valid && node >= skip_until;
      if (!__any_sync(0xffffffffu, act)) continue;
      const double4 g = a.geom[node];
      const uint4 rg4 = a.range[node];
      const double h = g.w;
      const bool is_leaf = rg4.z == 0;
      // warp-uniform FP64 centre offset from the reference target
      double cdx = g.x - rx, cdy = g.y - ry, cdz = g.z - rz;
      cdx = frameImage(cdx, w.box[0], inv_l[0]);
      cdy = frameImage(cdy, w.box[1], inv_l[1]);
      cdz = frameImage(cdz, w.box[2], inv_l[2]);
      const double cmax = fmax(fabs(cdx), fmax(fabs(cdy), fabs(cdz)));
      const bool fast_frame = h < 64.0 * w.cutoff && cmax + rga < half_min_box * (1.0 - 1.0e-9);
      bool prune = false, accept = false, need_exact = !fast_frame;
      float dxc = 0.f, dyc = 0.f, dzc = 0.f;  // COM offset of an accepted node (FP32)
      if constexpr (kGroup) {
        const bool lead = in_group && act && leader == lane;
        int gd = 0;
        if (__any_sync(0xffffffffu, lead)) {
          if (lead) {
            GroupBox gb;
            for (int c = 0; c < 3; ++c) {
              gb.c[c] = gbox_sm[c][warp][lane];
              gb.h[c] = gbox_sm[3 + c][warp][lane];
            }
            gb.a_min = gbox_sm[6][warp][lane];
            gd = groupDecisionNode(a, node, gb, g, is_leaf);
          }
        }
        gd = __shfl_sync(0xffffffffu, gd, leader);
        if (in_group) {
          need_exact = false;
          prune = gd == 0;
          accept = gd == 1;
        }
      }
      if (act && fast_frame && !in_group) {
        const float hf = static_cast<float>(h);
        // bound on the error of each FP32 offset component below (centre and
        // target offsets rounded once, one subtraction, the COM offset added)
        const float fe = 2.4e-7f * (static_cast<float>(cmax) + rga_f + hf);
        const float cut_e = 4.0f * cut_f * fe;
        const float ndx = static_cast<float>(cdx) - tfx;
        const float ndy = static_cast<float>(cdy) - tfy;
        const float ndz = static_cast<float>(cdz) - tfz;
        const float ax = fabsf(ndx), ay = fabsf(ndy), az = fabsf(ndz);
        const float ex = fmaxf(0.f, ax - hf), ey = fmaxf(0.f, ay - hf), ez = fmaxf(0.f, az - hf);
        const int keep = certainLess(fmaf(ex, ex, fmaf(ey, ey, ez * ez)), cut2, cut_e);
        if (keep == 0) {
          need_exact = true;
        } else {
          prune = keep < 0;
          if (!prune && !is_leaf) {
            // inside (target within the node cube), cutoff containment, envelope, MAC;
            // each +1 certainly true, -1 certainly false, 0 too close to call in FP32
            // Under the strict policy the inside test never decides: a target
            // inside the node cube is within 2 sqrt(3) h of the COM (which lies in
            // the cube), so 2h/r >= 0.58 fails the 0.08 envelope, and without
            // quadrupoles nothing is accepted. Only the adaptive envelope (angle
            // up to 1) needs it.
            int cin = -1;
            if (kAdaptive) {
              const int ix = certainLess(ax, hf, fe), iy = certainLess(ay, hf, fe), iz = certainLess(az, hf, fe);
              if (ix < 0 || iy < 0 || iz < 0) cin = -1;  // outside on some axis
              else cin = (ix > 0 && iy > 0 && iz > 0) ? 1 : 0;
            }
            int within = 1;
            if (!(kAdaptive && w.com_cutoff)) {
              const float qx = ax + hf, qy = ay + hf, qz = az + hf;
              within = certainLess(fmaf(qx, qx, fmaf(qy, qy, qz * qz)), cut2, cut_e);
            }
            const float4 nf = a.node_f4[node];
            dxc = ndx + nf.x;
            dyc = ndy + nf.y;
            dzc = ndz + nf.z;
            const float r2c = fmaf(dxc, dxc, fmaf(dyc, dyc, dzc * dzc));
            const float w2 = 4.0f * hf * hf;
            // bound on the error of r2c (an approximate root suffices for a bound)
            const float r2c_e = 4.0f * (r2c * rsqrtf(r2c)) * fe;
            int env, mac;
            if constexpr (kAdaptive) {
              env = certainLess(w2, angle2 * r2c, angle2 * r2c_e);
            } else {
              env = w.quadrupole ? certainLess(w2, env2 * r2c, env2 * r2c_e) : -1;
            }
            if (rel_test) {
              // G M w^2 / r^4 against the allowance (relative monopole: lower <= allowance
              // accepts; residual derivative: lower > allowance rejects, else the FP64 proxy)
              const float gm = w.G_f * a.node_mq[2 * static_cast<size_t>(node)].x;
              const float ir = __fdividef(1.0f, r2c);  // within the band's relative 2e-5
              const float lower = gm * (w2 * ir) * ir;
              const int over = (allow_f > 0.f && isfinite(lower))
                                   ? certainLess(allow_f, lower, 2.0f * lower * (r2c_e / r2c))
                                   : 0;
              if (!kAdaptive || w.estimator == 1) mac = -over;
              else mac = over > 0 ? -1 : 0;
            } else {
              const float macl = (!kAdaptive && w.criterion == 0) ? w2 : (2.0f * hf + nf.w) * (2.0f * hf + nf.w);
              mac = certainLess(macl, theta2 * r2c, theta2 * r2c_e);
            }
            if (cin > 0 || within < 0 || env < 0 || mac < 0) {
              accept = false;  // some condition certainly fails
            } else if (cin == 0 || within == 0 || env == 0 || mac == 0) {
              need_exact = true;
            } else {
              accept = true;
              if (kAdaptive && w.com_cutoff) {
                // accepted with its COM beyond r_cut: pruned (tree_pm_coupling.cpp:4129-4132)
                const int beyond = certainLess(cut2, r2c, r2c_e);
                if (beyond > 0) {
                  accept = false;
                  prune = true;
                } else if (beyond == 0) {
                  accept = false;
                  need_exact = true;
                }
              }
            }
          }
        }
      }
      // a group lane's accepted multipole: its own COM offset, and under
      // COM-distance cutoff nodes no contribution beyond r_cut (the node stays
      // accepted for the walk; the reference counts it pruned for this target)
      bool com_skip = false;
      if (kGroup && in_group && act && accept && !is_leaf) {
        bool exact_com = !fast_frame;
        if (fast_frame) {
          const float4 nf = a.node_f4[node];
          dxc = (static_cast<float>(cdx) - tfx) + nf.x;
          dyc = (static_cast<float>(cdy) - tfy) + nf.y;
          dzc = (static_cast<float>(cdz) - tfz) + nf.z;
          if (w.com_cutoff) {
            const float fe = 2.4e-7f * (static_cast<float>(cmax) + rga_f + static_cast<float>(h));
            const float r2c = fmaf(dxc, dxc, fmaf(dyc, dyc, dzc * dzc));
            const int beyond = certainLess(cut2, r2c, 4.0f * (r2c * rsqrtf(r2c)) * fe);
            if (beyond > 0) com_skip = true;
            else if (beyond == 0) exact_com = true;
          }
        }
        if (exact_com) {
          const double4 cm = a.com[node];
          const double ex = applyMetric(makeMetric(w.node_lo[0], w.node_hi[0], px, w.box[0]), cm.x - px);
          const double ey = applyMetric(makeMetric(w.node_lo[1], w.node_hi[1], py, w.box[1]), cm.y - py);
          const double ez = applyMetric(makeMetric(w.node_lo[2], w.node_hi[2], pz, w.box[2]), cm.z - pz);
          com_skip = w.com_cutoff && norm2rn(ex, ey, ez) > w.cutoff2;
          dxc = static_cast<float>(ex);
          dyc = static_cast<float>(ey);
          dzc = static_cast<float>(ez);
        }
        if (inst && com_skip) ++cnt_pruned;
      }
      if constexpr (kSoft) {
        // a node whose sources' softenings differ: the envelope guard decides
        // with the reference's FP64 arithmetic
        if (act && !is_leaf && !prune && !in_group && a.node_soft) {
          const double2 ns = a.node_soft[node];
          if (ns.y - ns.x > 1.0e-12) need_exact = true;
        }
      }
      if (act && need_exact) {
        const ExactDecision d = exactNodeDecision<kAdaptive>(a, node, px, py, pz, skip_self, hist, eps_t_d);
        prune = d.prune;
        accept = d.accept;
        dxc = static_cast<float>(d.dx);
        dyc = static_cast<float>(d.dy);
        dzc = static_cast<float>(d.dz);
      }
      // node counters: per lane, or once per group under the group walk
      const bool count_node = !kGroup || !in_group || count_walk;
      if (inst && act && count_node) {
        ++cnt_visited;
        cnt_pruned += prune ? 1 : 0;
      }
      if (is_leaf) {
        const bool want = act && !prune;
        const uint32_t mask = __ballot_sync(0xffffffffu, want);
        if (mask == 0u) continue;
        if (inst && want && count_node) {
          ++cnt_accepted;
          ++cnt_leaves;
        }
        const uint32_t begin = rg4.x, count = rg4.y;
        if (w.cutoff + h + rga < half_min_box && h < w.exact_half) {
          enqueue(begin, count, mask, false, g, cdx, cdy, cdz);
        } else {
          unsigned long long p = 0, sk = 0;
          exactLeafPairs(a, exact_sm[warp], begin, count, want, px, py, pz, self_pos, eps_t_d, acc_x, acc_y, acc_z,
                         nearest_d, p, sk);
          cnt_pairs += static_cast<uint32_t>(p);
          cnt_skips += static_cast<uint32_t>(sk);
        }
        continue;
      }
      // internal node
      const bool do_accept = act && !prune && accept;
      const bool open = act && !prune && !accept;
      if (do_accept) {
        if (inst && count_node) {
          ++cnt_accepted;
          ++cnt_multi;
        }
      }
      if (do_accept && !com_skip) {
        if (!kF64 && a.mult_f32 && fmaf(dxc, dxc, fmaf(dyc, dyc, dzc * dzc)) >= fmaxf(1.0e-8f * cut2, 1.0e-10f)) {
          if constexpr (kAdaptive) {
            m_list[warp][mn][lane] = make_float4(dxc, dyc, dzc, __uint_as_float(node));
            ++mn;
          } else {
            // few multipoles under the strict policy: evaluated where accepted
            float fx = 0.f, fy = 0.f, fz = 0.f;
            float me2 = w.eps2_f;
            if constexpr (kSoft) {
              const float me = static_cast<float>(nodeEps(a, node, eps_t_d));
              me2 = me * me;
            }
            multipoleF32<kEpsZero, kTerms>(a, node, dxc, dyc, dzc, sc_r2, fx, fy, fz, me2);
            acc_x += static_cast<double>(w.G_f * fx);
            acc_y += static_cast<double>(w.G_f * fy);
            acc_z += static_cast<double>(w.G_f * fz);
          }
        } else {
          // FP64 multipole: FP32 powers of 1/r could overflow this close to the
          // COM, or the FP32 split constants are out of range for this r_s
          const ExactDecision d = exactNodeDecision<kAdaptive>(a, node, px, py, pz, skip_self, hist, eps_t_d);
          multipoleForce(a, node, d.dx, d.dy, d.dz, eps_t_d, acc_x, acc_y, acc_z);
        }
      }
      if constexpr (kAdaptive) {
        if (__any_sync(0xffffffffu, mn == kList)) mflush();
      }
      if (act && (prune || accept)) skip_until = rg4.w;
      if (inst && open && count_node) ++cnt_opened;
      if (__any_sync(0xffffffffu, open)) {
        constexpr uint32_t kBlock = kAdaptive ? kBulkCountAdaptive : kBulkCount;
        if (kBlock > 0 && (!kDiag || a.blocks)) {
          // Subtree block: the lanes that opened this small node take every
          // source in it within r_cut (per-pair test, as in the leaf path)
          // instead of descending. This is the reference's pair set except
          // where a deeper node would have been accepted as a strict
          // multipole; those few are evaluated as the pairs they stand for.
          if (fast_frame && rg4.y <= kBlock && h <= bulk_half && w.cutoff + h + rga < half_min_box &&
              h < w.exact_half) {
            enqueue(rg4.x, rg4.y, __ballot_sync(0xffffffffu, open), true, g, cdx, cdy, cdz);
            continue;
          }
        }
        const uint32_t ch = lane < 8 ? a.child[8 * static_cast<size_t>(node) + lane] : kInvalid;
        const unsigned cmask = __ballot_sync(0xffffffffu, ch != kInvalid) & 0xFFu;
        const int nc = __popc(cmask);
        if (sp + nc > kStackCap) {
          overflow = true;
          break;
        }
        if (ch != kInvalid) stack[sp + __popc(cmask >> (lane + 1))] = ch;
        sp += nc;
        __syncwarp();
      }
    }
    if (qn > 0) flush();
    if constexpr (kAdaptive) {
      if (__any_sync(0xffffffffu, mn > 0)) mflush();
    }
    if (overflow && lane == 0) atomicOr(a.status, kStatusStackOverflow);
    if (valid) {
      const int64_t o = a.out_compact ? v - a.v0 : slot;
      a.out_x[o] = acc_x;
      a.out_y[o] = acc_y;
      a.out_z[o] = acc_z;
      a.out_near[o] = inst ? fmin(static_cast<double>(nearest_f), nearest_d) : INFINITY;
    }
    if (inst) {
      uint32_t c[8] = {cnt_visited, cnt_accepted, cnt_opened, cnt_pairs, cnt_pruned, cnt_skips, cnt_multi, cnt_leaves};
      for (int k = 0; k < 8; ++k) {
        for (int off = 16; off > 0; off >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], off);
      }
      if (lane == 0) {
        for (int k = 0; k < 8; ++k) atomicAdd(a.counters + k, static_cast<unsigned long long>(c[k]));
      }
    }
    if constexpr (kCost) {
      if (lane == 0) a.chunk_cost[base >> 5] = static_cast<float>(clock64() - item_start_sm[warp]);
    }
    __syncwarp();
  }
}

// ---- adjoint: vector-Jacobian product of the short-range force ----------

struct VjpArgs {
  int64_t n;                    // particles (every particle is a target)
  const uint32_t* order;        // visit position -> row (tree order)
  const double* sx;             // caller positions
  const double* sy;
  const double* sz;
  const double* m;              // masses (nullable: uniform_mass)
  double uniform_mass;
  const double* cx;             // cotangents a_bar per row
  const double* cy;
  const double* cz;
  const double4* geom;
  const uint4* range;
  const uint32_t* child;
  const double4* src_d4;        // tree order: caller position + mass
  const double4* src_c4;        // tree order: cotangent
  double* out_x;                // per row: x_bar of the short-range force (times G)
  double* out_y;
  double* out_z;
  uint32_t* work;
  uint32_t* status;
  PolyH poly;
  PolyH dpoly;
  WalkParams wp;
  float inv_16rs5_f;
  // the FP32 instance's packed pair loop: each coefficient in both halves, the
  // polynomial variables' scales and the kernel constants as pairs
  float2 pk2[kPolyMaxTerms];
  float2 dk2[kPolyMaxTerms];
  float2 sc2, dsc2, mone2, eps2_2, m8_2, m16_2, mthree2;
};

template <class Real>
struct VjpQueue;
template <>
struct VjpQueue<float> {
  using V4 = float4;
};
template <>
struct VjpQueue<double> {
  using V4 = double4;
};

// x_bar_k = G sum_j M(d) (m_k a_bar_j - m_j a_bar_k), d = x_j - x_k, over every
// source j within r_cut of target k (j != k, d != 0), M(d) = K I + (K'/r) d d^T
// the Jacobian of the pair force d -> K(|d|) d. Because M is even in d and the
// pair set {|d| <= r_cut} is symmetric, this gathers both the target-side and
// the source-side derivatives without scattering.
//
// Traversal: a node is kept while the r_cut sphere of some lane may reach its
// cube (each lane with its own minimum image, so groups of targets that are
// far apart in the box still prune); leaves and nodes of at most kBulkCountVjp
// sources are enqueued whole, keeping sources inside the sphere of the lanes
// that need the node; every pair decision is the per-pair cutoff test. Queue
// entries are FP64-formed minimum-image offsets from the warp's reference
// target; when r_cut plus the group radius reaches half the box, each pair
// takes its own minimum image.
template <class Real, bool kEpsZero, int kTerms>
__global__ void __launch_bounds__(kWalkWarpsPerBlock * 32, 4) walkVjpKernel(VjpArgs a) {
  using V4 = typename VjpQueue<Real>::V4;
  // FP32: sources in pairs for packed arithmetic, pair p = {x0, x1, y0, y1},
  // {z0, z1, m0, m1}, {cx0, cx1, cy0, cy1}, {cz0, cz1, -, -} (cotangents c)
  constexpr bool kPacked = sizeof(Real) == 4;
  __shared__ uint32_t stack_sm[kWalkWarpsPerBlock][kStackCap];
  __shared__ V4 q_pos[kWalkWarpsPerBlock][kPacked ? 1 : kQueue];
  __shared__ V4 q_cot[kWalkWarpsPerBlock][kPacked ? 1 : kQueue];
  __shared__ float4 q_pair[4][kWalkWarpsPerBlock][kPacked ? kQueue / 2 : 1];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint32_t* stack = stack_sm[warp];
  const WalkParams& w = a.wp;
  const double half_min_box = 0.5 * fmin(w.box[0], fmin(w.box[1], w.box[2]));
  const double inv_box[3] = {1.0 / w.box[0], 1.0 / w.box[1], 1.0 / w.box[2]};
  const Real cut2 = static_cast<Real>(w.cutoff2);
  const Real box_r[3] = {static_cast<Real>(w.box[0]), static_cast<Real>(w.box[1]), static_cast<Real>(w.box[2])};
  const Real inv_box_r[3] = {static_cast<Real>(inv_box[0]), static_cast<Real>(inv_box[1]),
                             static_cast<Real>(inv_box[2])};
  const double bulk_half = kBulkHalf * w.cutoff;

  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.work, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= a.n) break;
    const int64_t v = static_cast<int64_t>(base) + lane;
    const bool valid = v < a.n;
    uint32_t row = 0;
    double px = 0.0, py = 0.0, pz = 0.0, mk = 0.0, ckx = 0.0, cky = 0.0, ckz = 0.0;
    if (valid) {
      row = a.order[v];
      px = a.sx[row];
      py = a.sy[row];
      pz = a.sz[row];
      mk = a.m ? a.m[row] : a.uniform_mass;
      ckx = a.cx[row];
      cky = a.cy[row];
      ckz = a.cz[row];
    }
    const double rx = __shfl_sync(0xffffffffu, px, 0);
    const double ry = __shfl_sync(0xffffffffu, py, 0);
    const double rz = __shfl_sync(0xffffffffu, pz, 0);
    double ox = px - rx, oy = py - ry, oz = pz - rz;
    ox -= w.box[0] * rint(ox * inv_box[0]);
    oy -= w.box[1] * rint(oy * inv_box[1]);
    oz -= w.box[2] * rint(oz * inv_box[2]);
    double rg2 = valid ? ox * ox + oy * oy + oz * oz : 0.0;
    for (int off = 16; off > 0; off >>= 1) rg2 = fmax(rg2, __shfl_xor_sync(0xffffffffu, rg2, off));
    const double reach = w.cutoff + sqrt(rg2);       // group sphere radius
    const bool pair_image = reach >= half_min_box * (1.0 - 1.0e-9);
    const Real tx = static_cast<Real>(ox), ty = static_cast<Real>(oy), tz = static_cast<Real>(oz);
    const Real mkr = static_cast<Real>(mk);
    const Real ckxr = static_cast<Real>(ckx), ckyr = static_cast<Real>(cky), ckzr = static_cast<Real>(ckz);
    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    int qn = 0;
    if (lane == 0) stack[0] = 0u;
    int sp = 1;
    __syncwarp();
    bool overflow = false;

    // entry k of the queue (either layout)
    auto entryAt = [&](int k, V4& e, V4& cj) {
      if constexpr (kPacked) {
        const int h = k & 1;
        const float* qa = reinterpret_cast<const float*>(&q_pair[0][warp][k >> 1]);
        const float* qb = reinterpret_cast<const float*>(&q_pair[1][warp][k >> 1]);
        const float* qc = reinterpret_cast<const float*>(&q_pair[2][warp][k >> 1]);
        const float* qd = reinterpret_cast<const float*>(&q_pair[3][warp][k >> 1]);
        e = make_float4(qa[h], qa[2 + h], qb[h], qb[2 + h]);
        cj = make_float4(qc[h], qc[2 + h], qd[h], 0.f);
      } else {
        e = q_pos[warp][k];
        cj = q_cot[warp][k];
      }
    };

    auto flush = [&]() {
      Real gx = 0, gy = 0, gz = 0;
      if constexpr (kPacked) {
        if (!pair_image) {
          // two sources per step in packed FP32; an odd queue's last pair has
          // a second half of zero mass and zero cotangent (it adds exactly 0)
          if (qn & 1) {
            if (lane == 0) {
              for (int t = 0; t < 4; ++t) {
                float* q = reinterpret_cast<float*>(&q_pair[t][warp][qn >> 1]);
                q[1] = 0.f;
                q[3] = 0.f;
              }
            }
            __syncwarp();
          }
          const float2 ntx = make_float2(-tx, -tx), nty = make_float2(-ty, -ty), ntz = make_float2(-tz, -tz);
          const float2 mk2 = make_float2(mkr, mkr);
          const float2 nck0 = make_float2(-ckxr, -ckxr), nck1 = make_float2(-ckyr, -ckyr),
                       nck2 = make_float2(-ckzr, -ckzr);
          float2 g0 = make_float2(0.f, 0.f), g1 = g0, g2 = g0;
          const int np = (qn + 1) >> 1;
#pragma unroll 2
          for (int p = 0; p < np; ++p) {
            const float4 A = q_pair[0][warp][p];
            const float4 B = q_pair[1][warp][p];
            const float4 C = q_pair[2][warp][p];
            const float4 D = q_pair[3][warp][p];
            const float2 dx = __fadd2_rn(make_float2(A.x, A.y), ntx);
            const float2 dy = __fadd2_rn(make_float2(A.z, A.w), nty);
            const float2 dz = __fadd2_rn(make_float2(B.x, B.y), ntz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const bool in0 = valid && r2.x <= cut2 && r2.x > 0.f;
            const bool in1 = valid && r2.y <= cut2 && r2.y > 0.f;
            const float2 hh = hornerR2x2<(kTerms == 12 ? kPairPolyTerms : kTerms)>(a.pk2, r2, a.sc2, a.mone2);
            const float2 hp = hornerR2x2<kTerms>(a.dk2, r2, a.dsc2, a.mone2);
            const float2 s2 = kEpsZero ? r2 : __fadd2_rn(r2, a.eps2_2);
            const float2 rinv = make_float2(rsqrtf(s2.x), rsqrtf(s2.y));
            const float2 rinv2 = __fmul2_rn(rinv, rinv);
            const float2 rinv3 = __fmul2_rn(rinv2, rinv);
            const float2 K = __ffma2_rn(hh, a.m8_2, rinv3);  // r^-3 - H/(8 r_s^3)
            const float2 Kp = __ffma2_rn(hp, a.m16_2, __fmul2_rn(__fmul2_rn(rinv3, rinv2), a.mthree2));
            const float2 mj = make_float2(B.z, B.w);
            const float2 c0 = __ffma2_rn(mk2, make_float2(C.x, C.y), __fmul2_rn(mj, nck0));
            const float2 c1 = __ffma2_rn(mk2, make_float2(C.z, C.w), __fmul2_rn(mj, nck1));
            const float2 c2 = __ffma2_rn(mk2, make_float2(D.x, D.y), __fmul2_rn(mj, nck2));
            const float2 dc = __fmul2_rn(__ffma2_rn(dx, c0, __ffma2_rn(dy, c1, __fmul2_rn(dz, c2))), Kp);
            // select, not multiply: K and K' are infinite for the excluded self pair
            const float2 Ks = make_float2(in0 ? K.x : 0.f, in1 ? K.y : 0.f);
            const float2 dcs = make_float2(in0 ? dc.x : 0.f, in1 ? dc.y : 0.f);
            g0 = __ffma2_rn(Ks, c0, __ffma2_rn(dcs, dx, g0));
            g1 = __ffma2_rn(Ks, c1, __ffma2_rn(dcs, dy, g1));
            g2 = __ffma2_rn(Ks, c2, __ffma2_rn(dcs, dz, g2));
          }
          acc_x += static_cast<double>(g0.x + g0.y);
          acc_y += static_cast<double>(g1.x + g1.y);
          acc_z += static_cast<double>(g2.x + g2.y);
          qn = 0;
          __syncwarp();
          return;
        }
      }
#pragma unroll 2
      for (int k = 0; k < qn; ++k) {
        V4 e, cj;
        entryAt(k, e, cj);
        Real dx = static_cast<Real>(e.x) - tx, dy = static_cast<Real>(e.y) - ty, dz = static_cast<Real>(e.z) - tz;
        if (pair_image) {
          dx -= box_r[0] * rint(dx * inv_box_r[0]);
          dy -= box_r[1] * rint(dy * inv_box_r[1]);
          dz -= box_r[2] * rint(dz * inv_box_r[2]);
        }
        const Real r2 = dx * dx + dy * dy + dz * dz;
        const bool in = valid && r2 <= cut2 && r2 > Real(0);
        Real K, Kp;
        if constexpr (sizeof(Real) == 4) {
          // H in its pair-kernel length when it fits (the short fit has 9 terms)
          const float hh = hornerR2<(kTerms == 12 ? kPairPolyTerms : kTerms)>(a.poly, r2, w.inv_4rs2_f * a.poly.scale);
          const float hp = hornerR2<kTerms>(a.dpoly, r2, w.inv_4rs2_f * a.dpoly.scale);
          const float s2 = kEpsZero ? r2 : r2 + w.eps2_f;
          const float rinv = rsqrtf(s2);
          const float rinv2 = rinv * rinv;
          const float rinv3 = rinv2 * rinv;
          K = fmaf(-hh, w.inv_8rs3_f, rinv3);
          Kp = fmaf(-hp, a.inv_16rs5_f, -3.0f * rinv3 * rinv2);
        } else {
          const double rr = in ? r2 : 1.0;
          K = residualInvR3(rr, w.eps, w.rs);
          Kp = residualDerivOverR(rr, w.eps, w.rs);
        }
        const Real c0 = mkr * static_cast<Real>(cj.x) - static_cast<Real>(e.w) * ckxr;
        const Real c1 = mkr * static_cast<Real>(cj.y) - static_cast<Real>(e.w) * ckyr;
        const Real c2 = mkr * static_cast<Real>(cj.z) - static_cast<Real>(e.w) * ckzr;
        const Real dc = (dx * c0 + dy * c1 + dz * c2) * Kp;
        // select, not multiply: K and K' are infinite for the excluded self pair
        gx += in ? K * c0 + dc * dx : Real(0);
        gy += in ? K * c1 + dc * dy : Real(0);
        gz += in ? K * c2 + dc * dz : Real(0);
      }
      acc_x += static_cast<double>(gx);
      acc_y += static_cast<double>(gy);
      acc_z += static_cast<double>(gz);
      qn = 0;
      __syncwarp();
    };

    auto enqueue = [&](uint32_t begin, uint32_t count, uint32_t mask) {
      // sphere of the lanes that need the node (their offsets, FP64)
      const int first = __ffs(mask) - 1;
      const double scx = __shfl_sync(0xffffffffu, ox, first);
      const double scy = __shfl_sync(0xffffffffu, oy, first);
      const double scz = __shfl_sync(0xffffffffu, oz, first);
      double d2 = 0.0;
      if ((mask >> lane) & 1u) {
        const double ux = ox - scx, uy = oy - scy, uz = oz - scz;
        d2 = ux * ux + uy * uy + uz * uz;
      }
      for (int off = 16; off > 0; off >>= 1) d2 = fmax(d2, __shfl_xor_sync(0xffffffffu, d2, off));
      const double sr = w.cutoff + sqrt(d2);
      const double sr2 = sr * sr * (1.0 + 1.0e-6);
      // a sphere reaching half the box keeps everything; in warps whose pairs
      // take their own minimum image, the distance to its centre is wrapped too
      const bool keep_all = sr >= half_min_box * (1.0 - 1.0e-9);
      for (uint32_t chunk = 0; chunk < count; chunk += 32) {
        const uint32_t k = chunk + lane;
        bool keep = false;
        double ex = 0.0, ey = 0.0, ez = 0.0;
        double4 sv = make_double4(0.0, 0.0, 0.0, 0.0), cv = sv;
        if (k < count) {
          sv = a.src_d4[begin + k];
          ex = sv.x - rx;
          ey = sv.y - ry;
          ez = sv.z - rz;
          ex -= w.box[0] * rint(ex * inv_box[0]);
          ey -= w.box[1] * rint(ey * inv_box[1]);
          ez -= w.box[2] * rint(ez * inv_box[2]);
          double qx = ex - scx, qy = ey - scy, qz = ez - scz;
          if (pair_image) {
            qx -= w.box[0] * rint(qx * inv_box[0]);
            qy -= w.box[1] * rint(qy * inv_box[1]);
            qz -= w.box[2] * rint(qz * inv_box[2]);
          }
          keep = keep_all || qx * qx + qy * qy + qz * qz <= sr2;
          if (keep) cv = a.src_c4[begin + k];
        }
        const uint32_t keep_mask = __ballot_sync(0xffffffffu, keep);
        const int c = __popc(keep_mask);
        if (qn + c > kQueue) flush();
        if (keep) {
          const int slot_q = qn + __popc(keep_mask & ((1u << lane) - 1u));
          V4 e, cj;
          e.x = static_cast<Real>(ex);
          e.y = static_cast<Real>(ey);
          e.z = static_cast<Real>(ez);
          e.w = static_cast<Real>(sv.w);
          cj.x = static_cast<Real>(cv.x);
          cj.y = static_cast<Real>(cv.y);
          cj.z = static_cast<Real>(cv.z);
          cj.w = Real(0);
          if constexpr (kPacked) {
            const int hq = slot_q & 1;
            float* qa = reinterpret_cast<float*>(&q_pair[0][warp][slot_q >> 1]);
            float* qb = reinterpret_cast<float*>(&q_pair[1][warp][slot_q >> 1]);
            float* qc = reinterpret_cast<float*>(&q_pair[2][warp][slot_q >> 1]);
            float* qd = reinterpret_cast<float*>(&q_pair[3][warp][slot_q >> 1]);
            qa[hq] = e.x;
            qa[2 + hq] = e.y;
            qb[hq] = e.z;
            qb[2 + hq] = e.w;
            qc[hq] = cj.x;
            qc[2 + hq] = cj.y;
            qd[hq] = cj.z;
          } else {
            q_pos[warp][slot_q] = e;
            q_cot[warp][slot_q] = cj;
          }
        }
        __syncwarp();
        qn += c;
      }
    };

    while (sp > 0) {
      const uint32_t node = stack[sp - 1];
      --sp;
      __syncwarp();
      const double4 g = a.geom[node];
      const uint4 rg4 = a.range[node];
      const double h = g.w;
      // lanes whose r_cut sphere may reach the node cube: each lane takes its
      // own minimum image of the cube centre, so the test holds however far
      // apart the warp's targets are (only cubes with h + r_cut >= L/2, near
      // the root, are never pruned)
      bool need = valid;
      if (valid && h + w.cutoff < half_min_box * (1.0 - 1.0e-9)) {
        double dx = g.x - px, dy = g.y - py, dz = g.z - pz;
        dx -= w.box[0] * rint(dx * inv_box[0]);
        dy -= w.box[1] * rint(dy * inv_box[1]);
        dz -= w.box[2] * rint(dz * inv_box[2]);
        const double ex = fmax(0.0, fabs(dx) - h), ey = fmax(0.0, fabs(dy) - h), ez = fmax(0.0, fabs(dz) - h);
        need = ex * ex + ey * ey + ez * ez <= w.cutoff2 * (1.0 + 1.0e-9);
      }
      const uint32_t need_mask = __ballot_sync(0xffffffffu, need);
      if (need_mask == 0u) continue;
      if (rg4.z == 0 || (rg4.y <= kBulkCountVjp && h <= bulk_half)) {
        enqueue(rg4.x, rg4.y, need_mask);
        continue;
      }
      const uint32_t ch = lane < 8 ? a.child[8 * static_cast<size_t>(node) + lane] : kInvalid;
      const unsigned cmask = __ballot_sync(0xffffffffu, ch != kInvalid) & 0xFFu;
      const int nc = __popc(cmask);
      if (sp + nc > kStackCap) {
        overflow = true;
        break;
      }
      if (ch != kInvalid) stack[sp + __popc(cmask >> (lane + 1))] = ch;
      sp += nc;
      __syncwarp();
    }
    if (qn > 0) flush();
    if (overflow && lane == 0) atomicOr(a.status, kStatusStackOverflow);
    if (valid) {
      a.out_x[row] = w.G * acc_x;
      a.out_y[row] = w.G * acc_y;
      a.out_z[row] = w.G * acc_z;
    }
    __syncwarp();
  }
}

// Cotangents gathered into tree order (double4 {a_bar, 0}).
__global__ void packCotangentKernel(int64_t n, const uint32_t* __restrict__ sorted, const double* __restrict__ cx,
                                    const double* __restrict__ cy, const double* __restrict__ cz, double4* out) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint32_t s = sorted[t];
    out[t] = make_double4(cx[s], cy[s], cz[s], 0.0);
  }
}

template <class Kernel>
int launchVjp(Kernel kernel, const VjpArgs& args, cudaStream_t s) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWalkWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int64_t warps_needed = (args.n + 31) / 32;
  int64_t blocks = static_cast<int64_t>(sms) * per_sm;
  const int64_t max_useful = (warps_needed + kWalkWarpsPerBlock - 1) / kWalkWarpsPerBlock;
  if (blocks > max_useful) blocks = max_useful;
  if (blocks < 1) blocks = 1;
  { noteLaunch(); kernel<<<static_cast<unsigned>(blocks), kWalkWarpsPerBlock * 32, 0, s>>>(args); }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

template <class Kernel>
int launchPersistent(Kernel kernel, const WalkArgs& args, cudaStream_t s) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWalkWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int64_t warps_needed = (args.v1 - args.v0 + 31) / 32;
  int64_t blocks = static_cast<int64_t>(sms) * per_sm;
  const int64_t max_useful = (warps_needed + kWalkWarpsPerBlock - 1) / kWalkWarpsPerBlock;
  if (blocks > max_useful) blocks = max_useful;
  if (blocks < 1) blocks = 1;
  { noteLaunch(); kernel<<<static_cast<unsigned>(blocks), kWalkWarpsPerBlock * 32, 0, s>>>(args); }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

template <bool kMixed, bool kEpsZero>
int launchWalk(const WalkArgs& args, cudaStream_t s) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, walkKernel<kMixed, kEpsZero>,
                                                kWalkWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int64_t warps_needed = (args.v1 - args.v0 + 31) / 32;
  int64_t blocks = static_cast<int64_t>(sms) * per_sm;
  const int64_t max_useful = (warps_needed + kWalkWarpsPerBlock - 1) / kWalkWarpsPerBlock;
  if (blocks > max_useful) blocks = max_useful;
  if (blocks < 1) blocks = 1;
  { noteLaunch(); walkKernel<kMixed, kEpsZero><<<static_cast<unsigned>(blocks), kWalkWarpsPerBlock * 32, 0, s>>>(args); }
  return cudaGetLastError() == cudaSuccess ? 0 : CHUI_TREEPM_EDEVICE;
}

// Host copy of the Gaussian long-range force factor L(q) for the table.
double hostLongRangeFactor(double r, double rs) {
  if (r <= 0.0) return 0.0;
  const double q = (0.5 * r) / rs;
  if (std::isinf(q)) return 1.0;
  const double k = 0.564189583547756286948079451560772586;
  if (q < 0.125) {
    const double t = q * q;
    const double h = 4.0 * k * (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
                     t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
    return q * q * q * h;
  }
  return std::erf(q) - 2.0 * k * q * std::exp(-q * q);
}

// TreePmGaussianCoefficientTable's knots (tree_pm_split_kernel.hpp:170-181),
// uploaded once per context.
int ensureGaussTable(Context& c, cudaStream_t s) {
  if (c.gauss_ready) return 0;
  if (ensure(c.gauss_tab, (kGaussCells + 1) * sizeof(double2))) return CHUI_TREEPM_ENOMEM;
  std::vector<double2> tab(kGaussCells + 1);
  const double k = 0.564189583547756286948079451560772586;
  for (int i = 0; i <= kGaussCells; ++i) {
    const double t = static_cast<double>(i) * kGaussStep;
    const double q = std::sqrt(t);
    const double value = i == 0 ? 4.0 * k / 3.0 : hostLongRangeFactor(q, 0.5) / (t * q);
    const double derivative = i == 0 ? -4.0 * k / 5.0 : (2.0 * k * std::exp(-t) - 1.5 * value) / t;
    tab[i] = make_double2(value, kGaussStep * derivative);
  }
  cudaMemcpyAsync(c.gauss_tab.ptr, tab.data(), tab.size() * sizeof(double2), cudaMemcpyHostToDevice, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
  c.gauss_ready = true;
  return 0;
}

}  // namespace

int walkRun(Context& c, int64_t nt, const uint32_t* active, const double* tx, const double* ty,
            const double* tz, const double* sx, const double* sy, const double* sz,
            const double* prev_acc, const WalkParams& wp, int64_t n, cudaStream_t s,
            int64_t visit_begin, int64_t visit_end, bool compact, bool record_cost) {
  if (visit_end < 0) visit_end = nt;
  if (nt == 0) return 0;
  // counters and per-chunk walk cycles start at zero even when the visit
  // range is empty (the solve reads the counters back either way)
  const size_t chunks = static_cast<size_t>((nt + 31) / 32);
  if (ensure(c.walk_cost, chunks * sizeof(float)) || ensure(c.walk_counters, 8 * sizeof(unsigned long long)))
    return CHUI_TREEPM_ENOMEM;
  cudaMemsetAsync(c.walk_cost.ptr, 0, chunks * sizeof(float), s);
  cudaMemsetAsync(c.walk_counters.ptr, 0, 8 * sizeof(unsigned long long), s);
  if (visit_end <= visit_begin) return 0;
  if (ensure(c.tree_acc, static_cast<size_t>(nt) * 3 * sizeof(double)) ||
      ensure(c.tree_near, static_cast<size_t>(nt) * sizeof(double)) || ensure(c.work_counter, 4))
    return CHUI_TREEPM_ENOMEM;
  cudaMemsetAsync(c.work_counter.ptr, 0, 4, s);
  WalkArgs a;
  a.nt = nt;
  a.v0 = visit_begin;
  a.v1 = visit_end;
  a.out_compact = compact ? 1 : 0;
  a.n = n;
  a.order = c.target_order.as<uint32_t>();
  a.active = active;
  a.tx = tx;
  a.ty = ty;
  a.tz = tz;
  a.sx = sx;
  a.sy = sy;
  a.sz = sz;
  a.pos_of_row = c.pos_of_row.as<uint32_t>();
  a.geom = c.node_geom.as<double4>();
  a.com = c.node_com.as<double4>();
  a.quad = c.node_quad.as<double>();
  a.child = c.node_child.as<uint32_t>();
  a.range = c.node_range.as<uint4>();
  a.src_f4 = c.src_f4.as<float4>();
  a.src_d4 = c.src_d4.as<double4>();
  a.node_f4 = c.node_f4.as<float4>();
  a.node_mq = c.node_mq.as<float4>();
  a.src_u4 = c.src_u4.as<double4>();
  a.prev = prev_acc;
  const bool soft = c.soft_rows != nullptr || c.soft_targets != nullptr;
  a.src_eps = c.soft_rows ? c.src_eps.as<double>() : nullptr;
  a.row_eps = c.soft_rows;
  a.tgt_eps = c.soft_targets;
  a.node_soft = c.soft_rows ? c.node_soft.as<double2>() : nullptr;
  a.leaf_of_pos = nullptr;
  a.grp_start = nullptr;
  a.grp_rec = nullptr;
  a.grp_list = nullptr;
  a.grp_done = nullptr;
  a.gauss = nullptr;
  if (wp.gauss_lookup || wp.group_walk) {
    if (int rc = ensureGaussTable(c, s)) return rc;
    a.gauss = c.gauss_tab.as<double2>();
  }
  double* acc = c.tree_acc.as<double>();
  a.out_x = acc;
  a.out_y = acc + nt;
  a.out_z = acc + 2 * nt;
  a.out_near = c.tree_near.as<double>();
  a.counters = c.walk_counters.as<unsigned long long>();
  a.work = c.work_counter.as<uint32_t>();
  // per-block cycles for visit-range solves (FP64 walk, and the mixed walk's
  // production instances: no diagnostics, every source a target, one mass)
  a.chunk_cost = record_cost ? c.walk_cost.as<float>() : nullptr;
  a.status = c.status.as<uint32_t>();
  a.poly = c.poly;
  a.dpoly = c.dpoly;
  a.ddpoly = c.ddpoly;
  {
    const double rs2 = c.rs * c.rs;
    const double i5 = 1.0 / (16.0 * rs2 * rs2 * c.rs), i7 = 1.0 / (32.0 * rs2 * rs2 * rs2 * c.rs);
    a.inv_16rs5_f = static_cast<float>(i5);
    a.inv_32rs7_f = static_cast<float>(i7);
    a.mult_f32 = (i5 >= FLT_MIN && i5 <= 1.0e30 && i7 >= FLT_MIN && i7 <= 1.0e30) ? 1 : 0;
    a.mpoly12 = (c.dpoly.terms <= 12 && c.ddpoly.terms <= 12) ? 1 : 0;
  }
  {
    // K_long = H(t)/(8 r_s^3): the pair loop evaluates -K_long directly from
    // the H coefficients scaled by -1/(8 r_s^3), at s = (r^2 + eps^2) sc + soff
    // with soff = -1 - eps^2 sc (that is s = r^2 sc - 1, eps^2 folded in)
    const double kscale = -0.125 / (c.rs * c.rs * c.rs);
    for (int k = 0; k < kPolyMaxTerms; ++k) {
      const float v = static_cast<float>(static_cast<double>(c.poly.c[k]) * kscale);
      if (!std::isfinite(v)) return CHUI_TREEPM_ENOTSUP;  // r_s outside the FP32 pair kernel's range
      a.pk2[k] = make_float2(v, v);
    }
    const float sc = wp.inv_4rs2_f * c.poly.scale;  // the r^2 -> s scale, rounded as the multipoles round it
    a.sc2 = make_float2(sc, sc);
    const float soff = static_cast<float>(-1.0 - static_cast<double>(wp.eps2_f) * static_cast<double>(sc));
    a.soff2 = make_float2(soff, soff);
    a.eps2_2 = make_float2(wp.eps2_f, wp.eps2_f);
    a.cut2e = wp.cut2_f + wp.eps2_f;
    a.mone2 = make_float2(-1.0f, -1.0f);
  }
  // diagnostics 2 or a nearest-pair lane: counted walk over the production traversal
  a.instrument = c.walk_instrument ? 1 : 0;
  a.blocks = c.cfg.diagnostics != 1 ? 1 : 0;
  a.wp = wp;
  uint32_t* group_count = nullptr;
  if (wp.group_walk) {
    if (ensure(c.grp_leaf, static_cast<size_t>(n) * 4) || ensure(c.grp_start, static_cast<size_t>(nt) * 4) ||
        ensure(c.grp_rec, static_cast<size_t>(nt) * 2 * sizeof(double4)) ||
        ensure(c.grp_list, static_cast<size_t>(nt) * 4) || ensure(c.grp_done, static_cast<size_t>(nt)) ||
        ensure(c.work_counter, 16))
      return CHUI_TREEPM_ENOMEM;
    a.leaf_of_pos = c.grp_leaf.as<uint32_t>();
    a.grp_start = c.grp_start.as<uint32_t>();
    a.grp_rec = c.grp_rec.as<double4>();
    a.grp_list = c.grp_list.as<uint32_t>();
    a.grp_done = c.grp_done.as<unsigned char>();
    group_count = c.work_counter.as<uint32_t>() + 1;
    cudaMemsetAsync(c.grp_done.ptr, 0, static_cast<size_t>(nt), s);
    cudaMemsetAsync(group_count, 0, 4, s);
    { noteLaunch(); leafOfPosKernel<<<groupGrid(c.n_nodes, 256), 256, 0, s>>>(c.n_nodes, a.range, c.grp_leaf.as<uint32_t>()); }
    { noteLaunch(); groupSetupKernel<<<groupGrid(visit_end - visit_begin, 256), 256, 0, s>>>(a, group_count); }
  }
  const bool mixed = c.cfg.precision == CHUI_TREEPM_MIXED;
  const bool eps_zero = wp.eps == 0.0;
  if (mixed) {
    // full solves visit targets in tree order, so a warp's targets are tree
    // positions base..base+31 and self pairs are excluded by the lane mask
    const bool contiguous = active == nullptr && tx == nullptr && nt == n;
    // the counting instances: diagnostics 1 (per node) and 2 or a nearest-pair
    // lane (with subtree blocks: the production traversal)
    const bool diag = c.cfg.diagnostics == 1 || c.walk_instrument;
    const bool uniform = wp.uniform_mass != 0;
    const int mode = wp.policy == CHUI_TREEPM_POLICY_ADAPTIVE ? (wp.group_walk ? 3 : 2)
                                                               : (wp.criterion == 2 && prev_acc ? 1 : 0);
    if (soft) {
      // per-particle softening: masses travel with the sources, the long H
      // form (any configuration), no group walk
#define CHUI_WALK_SOFT(DIAG, CONT, MODE) \
  walkFastKernel<false, kPolyMaxTerms, DIAG, CONT, MODE, false, false, false, true>
#define CHUI_WALK_SOFT2(MODE)                                                                          \
  if (diag) return contiguous ? launchPersistent(CHUI_WALK_SOFT(true, true, MODE), a, s)                  \
                              : launchPersistent(CHUI_WALK_SOFT(true, false, MODE), a, s);                \
  return contiguous ? launchPersistent(CHUI_WALK_SOFT(false, true, MODE), a, s)                          \
                    : launchPersistent(CHUI_WALK_SOFT(false, false, MODE), a, s);
      if (mode >= 2) { CHUI_WALK_SOFT2(2) }
      if (mode == 1) { CHUI_WALK_SOFT2(1) }
      CHUI_WALK_SOFT2(0)
#undef CHUI_WALK_SOFT2
#undef CHUI_WALK_SOFT
    }
#define CHUI_WALK_DISPATCH2(EPS, TERMS, ADP)                                                           \
    if (diag) return contiguous ? launchPersistent(walkFastKernel<EPS, TERMS, true, true, ADP>, a, s)     \
                                : launchPersistent(walkFastKernel<EPS, TERMS, true, false, ADP>, a, s);   \
    if (contiguous && uniform)                                                                         \
      return a.chunk_cost ? launchPersistent(walkFastKernel<EPS, TERMS, false, true, ADP, true, true>, a, s)    \
                          : launchPersistent(walkFastKernel<EPS, TERMS, false, true, ADP, true>, a, s);         \
    if (contiguous) return launchPersistent(walkFastKernel<EPS, TERMS, false, true, ADP>, a, s);             \
    return launchPersistent(walkFastKernel<EPS, TERMS, false, false, ADP>, a, s);
#define CHUI_WALK_DISPATCH(EPS, TERMS)                  \
    if (mode == 3) { CHUI_WALK_DISPATCH2(EPS, TERMS, 3) } \
    if (mode == 2) { CHUI_WALK_DISPATCH2(EPS, TERMS, 2) } \
    if (mode == 1) { CHUI_WALK_DISPATCH2(EPS, TERMS, 1) } \
    CHUI_WALK_DISPATCH2(EPS, TERMS, 0)
    if (c.poly.terms <= kPairPolyTerms) {
      if (eps_zero) { CHUI_WALK_DISPATCH(true, kPairPolyTerms) }
      CHUI_WALK_DISPATCH(false, kPairPolyTerms)
    }
    if (eps_zero) { CHUI_WALK_DISPATCH(true, kPolyMaxTerms) }
    CHUI_WALK_DISPATCH(false, kPolyMaxTerms)
#undef CHUI_WALK_DISPATCH
#undef CHUI_WALK_DISPATCH2
  }
  if (!mixed && !soft && c.cfg.diagnostics != 1 && wp.policy == CHUI_TREEPM_POLICY_STRICT && !wp.group_walk &&
      !(wp.criterion == 2 && prev_acc)) {
    // the production solver in FP64 (same traversal and subtree blocks as the
    // mixed walk, FP64 pairs and multipoles)
    const bool contiguous = active == nullptr && tx == nullptr && nt == n;
#define CHUI_WALK64(EPS, CONT, COST) walkFastKernel<EPS, kPairPolyTerms, false, CONT, 0, false, COST, true>
    if (contiguous) {
      if (a.chunk_cost) return eps_zero ? launchPersistent(CHUI_WALK64(true, true, true), a, s)
                                        : launchPersistent(CHUI_WALK64(false, true, true), a, s);
      return eps_zero ? launchPersistent(CHUI_WALK64(true, true, false), a, s)
                      : launchPersistent(CHUI_WALK64(false, true, false), a, s);
    }
    return eps_zero ? launchPersistent(CHUI_WALK64(true, false, false), a, s)
                    : launchPersistent(CHUI_WALK64(false, false, false), a, s);
#undef CHUI_WALK64
  }
  if (wp.group_walk) {
    uint32_t n_groups = 0;
    cudaMemcpyAsync(&n_groups, group_count, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return CHUI_TREEPM_EDEVICE;
    if (n_groups > 0) {
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const int64_t want = (static_cast<int64_t>(n_groups) + kWalkWarpsPerBlock - 1) / kWalkWarpsPerBlock;
      const unsigned blocks = static_cast<unsigned>(std::min<int64_t>(want, static_cast<int64_t>(sms) * 8));
      { noteLaunch(); groupWalkKernel<<<blocks, kWalkWarpsPerBlock * 32, 0, s>>>(a, c.grp_list.as<uint32_t>(), n_groups); }
      if (cudaGetLastError() != cudaSuccess) return CHUI_TREEPM_EDEVICE;
    }
  }
  return launchWalk<false, false>(a, s);
}

int walkVjpRun(Context& c, int64_t n, const double* sx, const double* sy, const double* sz, const double* m,
               double uniform_mass, const double* cx, const double* cy, const double* cz, const WalkParams& wp,
               double* gx, double* gy, double* gz, cudaStream_t s) {
  if (n == 0) return 0;
  if (ensure(c.src_cot, static_cast<size_t>(n) * sizeof(double4)) || ensure(c.work_counter, 4))
    return CHUI_TREEPM_ENOMEM;
  { noteLaunch(); packCotangentKernel<<<static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 148 * 32)), 256, 0, s>>>(
      n, c.sorted_index.as<uint32_t>(), cx, cy, cz, c.src_cot.as<double4>()); }
  cudaMemsetAsync(c.work_counter.ptr, 0, 4, s);
  VjpArgs a;
  a.n = n;
  a.order = c.target_order.as<uint32_t>();
  a.sx = sx;
  a.sy = sy;
  a.sz = sz;
  a.m = m;
  a.uniform_mass = uniform_mass;
  a.cx = cx;
  a.cy = cy;
  a.cz = cz;
  a.geom = c.node_geom.as<double4>();
  a.range = c.node_range.as<uint4>();
  a.child = c.node_child.as<uint32_t>();
  a.src_d4 = c.src_d4.as<double4>();
  a.src_c4 = c.src_cot.as<double4>();
  a.out_x = gx;
  a.out_y = gy;
  a.out_z = gz;
  a.work = c.work_counter.as<uint32_t>();
  a.status = c.status.as<uint32_t>();
  a.poly = c.poly;
  a.dpoly = c.dpoly;
  a.wp = wp;
  const double rs2 = c.rs * c.rs;
  a.inv_16rs5_f = static_cast<float>(1.0 / (16.0 * rs2 * rs2 * c.rs));
  for (int k = 0; k < kPolyMaxTerms; ++k) {
    a.pk2[k] = make_float2(c.poly.c[k], c.poly.c[k]);
    a.dk2[k] = make_float2(c.dpoly.c[k], c.dpoly.c[k]);
  }
  const float sc = wp.inv_4rs2_f * c.poly.scale, dsc = wp.inv_4rs2_f * c.dpoly.scale;
  a.sc2 = make_float2(sc, sc);
  a.dsc2 = make_float2(dsc, dsc);
  a.mone2 = make_float2(-1.f, -1.f);
  a.eps2_2 = make_float2(wp.eps2_f, wp.eps2_f);
  a.m8_2 = make_float2(-wp.inv_8rs3_f, -wp.inv_8rs3_f);
  a.m16_2 = make_float2(-a.inv_16rs5_f, -a.inv_16rs5_f);
  a.mthree2 = make_float2(-3.f, -3.f);
  const bool eps_zero = wp.eps == 0.0;
  if (c.cfg.precision == CHUI_TREEPM_MIXED) {
    if (c.poly.terms <= kPairPolyTerms && c.dpoly.terms <= 12)
      return eps_zero ? launchVjp(walkVjpKernel<float, true, 12>, a, s) : launchVjp(walkVjpKernel<float, false, 12>, a, s);
    return eps_zero ? launchVjp(walkVjpKernel<float, true, kPolyMaxTerms>, a, s)
                    : launchVjp(walkVjpKernel<float, false, kPolyMaxTerms>, a, s);
  }
  return launchVjp(walkVjpKernel<double, false, 12>, a, s);
}

}  // namespace chui
