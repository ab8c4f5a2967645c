// Internal state of one TreePM solver instance (the object behind the C-ABI
// handle) and the declarations shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/chui_treepm.h"
#include "common.cuh"

namespace chui {

// Grow-only device allocation.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

cudaError_t ensure(DevBuf& b, size_t bytes);
void release(DevBuf& b);

// Coefficients of the FP32 Gaussian long-range coefficient H(t) = L(q)/q^3,
// t = q^2 = r^2/(4 r_s^2), as a polynomial in s = t*scale - 1 on [0, t_cut].
struct PolyH {
  int terms = 0;              // degree + 1
  float scale = 0.f;          // 2 / t_cut
  float c[kPolyMaxTerms] = {};
  double max_rel_error = 0.0;
};

// Per-solve scalar geometry shared with the walk kernel.
struct WalkParams {
  double box[3];
  double inv_box[3];              // 1/box (0 for isolated/open boundaries)
  double src_lo[3], src_hi[3];    // bounds of the caller's source coordinates
  double node_lo[3], node_hi[3];  // bounds of node centres and COMs
  double rs, cutoff, cutoff2;
  double G, eps;
  double theta;
  double exact_half;  // leaves with half >= this use the exact FP64 pair path
  int criterion;   // 0 geometric, 1 COM distance, 2 relative (no history: COM distance)
  int quadrupole;
  int policy;      // 0 strict reference, 1 adaptive relative
  int estimator;   // adaptive: 0 residual derivative, 1 relative monopole
  int com_cutoff;  // adaptive with COM-distance cutoff nodes
  int group_walk;  // the group walk is active for this solve
  int gauss_lookup;  // Gaussian Hermite table for FP64 direct pairs
  int uniform_mass;  // every source has mass m0
  float m0_f;
  double angle;    // adaptive_maximum_opening_angle
  double rel_tol;  // relative_force_tolerance
  double floor_;   // relative_force_acceleration_floor_code
  float inv_4rs2_f;   // 1/(4 r_s^2)
  float inv_8rs3_f;   // 1/(8 r_s^3)
  float cut2_f;
  float eps2_f;
  float G_f;
};

struct Context {
  chui_treepm_config cfg{};
  int device = 0;
  double spacing = 0.0, rs = 0.0, cutoff = 0.0;
  PolyH poly;
  PolyH dpoly;   // H'(t): the adjoint walk and FP32 multipoles
  PolyH ddpoly;  // H''(t): FP32 quadrupoles
  std::string last_error;

  // PM (cuFFT, in-place padded real layout nx*ny*2*(nz/2+1))
  bool fft_ready = false;
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  // isolated/open PM: zero-padded (2nx, 2ny, 2nz) in-place real/half-spectrum
  // array, the split Green function's (real) spectrum scaled by G dV / pad size
  bool iso_ready = false;
  cufftHandle iso_r2c = 0, iso_c2r = 0;
  DevBuf iso_pad, iso_kernel;
  DevBuf grid[3];            // grid[0] holds the density then F_x; grid[1], grid[2] F_y, F_z
  DevBuf grid_f4;            // periodic mixed: {F_x, F_y, F_z, 0} per cell for the interpolation
  bool pm_f4_ready = false;  // grid_f4 holds the current field
  DevBuf adj_grid[3];        // adjoint: cotangent grids B_x, B_y, B_z; adj_grid[0] then holds rho_bar
  DevBuf axis_tables;        // kx, ky, kz, wx, wy, wz (FP64)
  bool pm_field_valid = false;
  double pm_field_box[3] = {0, 0, 0};

  // staged inputs / outputs
  DevBuf in_x, in_y, in_z, in_m, in_active, in_tx, in_ty, in_tz, in_prev;
  // per-particle softening of the current solve: row-order source epsilons and
  // active-slot target epsilons (staged inputs), the tree-order copy, and each
  // node's {min, max} source epsilon
  DevBuf in_eps, in_teps, src_eps, node_soft;
  const double* soft_rows = nullptr;     // null: uniform (config) source softening
  const double* soft_targets = nullptr;  // null: targets take their source row's epsilon
  // group walk: leaf per tree position, per visit position the group start and
  // the group record (centre + a_min, half + flags), the eligible group starts,
  // per-slot "evaluated by a group" flags, the Gaussian Hermite table
  DevBuf grp_leaf, grp_start, grp_rec, grp_list, grp_done, gauss_tab;
  bool gauss_ready = false;
  DevBuf out_acc[3], out_pm[3], out_tree[3], out_near, out_lr[3];
  // targets of the last successful solve (its visit order is target_order);
  // -1 before one
  int64_t visit_count = -1;
  DevBuf status;       // uint32 status word + scalar results (reduction scratch)
  DevBuf scalars;      // reduction outputs (64 x u64)
  std::vector<unsigned long long> host_scalars;

  // tree construction
  DevBuf ux, uy, uz;             // unwrapped FP64 coordinates (tree frame)
  DevBuf bucket_min, bucket_max;  // unwrap gap buckets {min, max}; bucket_max is also tree-path sort scratch
  DevBuf gap_min, gap_max, gap_flag, gap_off;  // non-empty gap buckets in order, their flags and offsets
  DevBuf keys_a, keys_b, idx_a, idx_b, idx_c, idx_d;
  DevBuf path_words;             // kMaxPathWords * n u64
  DevBuf common_prefix;          // int8/int32 per sorted position
  DevBuf cp_levels;              // block minima of the common prefix (levels 1..)
  DevBuf node_count_per_pos, node_offset;  // per sorted position (n+1)
  DevBuf leaf_of_pos, inv_pos;
  // radix sort and scan scratch (sort.cu)
  DevBuf sort_hist, sort_counts, sort_totals, sort_keys, sort_vals;
  int64_t n_nodes = 0;
  uint32_t max_depth = 0;
  int path_words_used = 0;
  int unwrap_sorted_axes = 0;  // axes whose unwrap sorted the coordinates (bit a)
  int prev_tree_depth = 0;     // depth of the previous tree built by this context (0: none)
  int large_leaf = 0;
  int path_levels_retried = 0;  // the last build repeated the path sort with every level          // the last build ordered a leaf above kLeafOrderMax globally
  double tree_anchor[3] = {0, 0, 0};

  // nodes (SoA, FP64 geometry/moments)
  DevBuf node_geom;    // double4 {cx, cy, cz, half}
  DevBuf node_com;     // double4 {comx, comy, comz, mass}
  DevBuf node_quad;    // 8 doubles per node {qxx, qxy, qxz, qyy, qyz, qzz, trace, com_center_offset}
  DevBuf node_mq;      // 2 x float4 per node: {mass, Mxx, Mxy, Mxz}, {Myy, Myz, Mzz, trace}, M = (Q + tr I)/3
  DevBuf node_f4;      // float4 {com - centre (x, y, z), |centre - com|}: FP32 node frame of the walk
  DevBuf node_child;   // 8 u32 per node
  DevBuf node_range;   // uint4 {begin, count, child_count | leaf flag, subtree_end}
  DevBuf node_parent;  // u32
  DevBuf node_depth;   // u32
  DevBuf node_counter; // u32 (bottom-up completion counters)
  DevBuf sorted_index; // u32 per tree position: caller row
  DevBuf pos_of_row;   // u32 per caller row: tree position
  DevBuf src_f4;       // float4 per tree position: offset from leaf centre (FP32) + mass
  DevBuf src_d4;       // double4 per tree position: caller position + mass (FP64 path)
  DevBuf src_u4;       // double4 per tree position: unwrapped (tree frame) position + mass (moments, walk)
  DevBuf src_cot;      // double4 per tree position: force cotangent (adjoint walk)
  DevBuf target_order; // visit order of active slots
  DevBuf morton_keys;  // Morton key of each particle (row order)

  // walk
  DevBuf walk_counters;  // 8 x u64
  DevBuf walk_cost;      // per 32 visit positions: SM cycles of the last walk (float)
  DevBuf work_counter;   // u32 dynamic scheduling
  DevBuf tree_acc;       // double3 per active slot (short-range part)
  DevBuf tree_near;      // double per active slot
  // the production walk counts its traversal and pairs and records the
  // nearest-pair r^2 (diagnostics 2, or a nearest-pair lane requested)
  bool walk_instrument = false;

  cudaEvent_t ev[8] = {};
  bool events_ready = false;
  // host-memory kick and drift: two copy/compute streams and their events
  cudaStream_t pipe_stream[2] = {};
  cudaEvent_t pipe_ev[3] = {};
  bool pipe_ready = false;
  chui_treepm_stats last_stats{};
};

// ---- PM (pm.cu) ----
int pmPrepare(Context& c);
// tree_sources (nullable): the same sources in tree order as double4
// {position, mass} (Context::src_d4 after treeBuild); selects the tiled deposit.
int pmRefresh(Context& c, int64_t n, const double* x, const double* y, const double* z,
              const double* m, double uniform_mass, double total_mass, cudaStream_t s,
              const double4* tree_sources = nullptr);
// CIC/TSC interpolation of the cached force grids at targets (active slots);
// with `order`, only the nt slots order[0..nt) (a visit-order slice), written
// compactly (entry j is slot order[j]).
int pmInterpolate(Context& c, int64_t nt, const uint32_t* active, const double* tx,
                  const double* ty, const double* tz, const double* sx, const double* sy,
                  const double* sz, double* ax, double* ay, double* az, cudaStream_t s,
                  const uint32_t* order = nullptr);
// Interpolation and the solve's total force over the nt active slots (tree:
// the walk's slot-indexed output, 3 lanes of nt; positions: explicit targets
// or the sources' rows): the accel (and optional long-range) lanes at slots,
// the optional source-indexed short-range and nearest-pair lanes at rows
// below n.
int pmInterpolateCombine(Context& c, int64_t nt, const uint32_t* active, const double* tx, const double* ty,
                         const double* tz, int64_t n, const double* px, const double* py, const double* pz,
                         bool with_pm, const double* tree, const double* near, double* ax, double* ay, double* az,
                         double* lx, double* ly, double* lz, double* sx, double* sy, double* sz, double* snear,
                         cudaStream_t s);
int pmDensityOnly(Context& c, int64_t n, const double* x, const double* y, const double* z,
                  const double* m, double uniform_mass, double* rho_out, cudaStream_t s);
int pmCells(Context& c, int64_t n, const double* x, const double* y, const double* z,
            int64_t* cells, cudaStream_t s);
// Adjoint of the PM force at positions (x, y, z) for cotangents c: g = J_pm^T c
// (refreshes the PM field at these positions first).
int pmForceVjp(Context& c, int64_t n, const double* x, const double* y, const double* z, const double* m,
               double uniform_mass, double total_mass, const double* cx, const double* cy, const double* cz,
               double* gx, double* gy, double* gz, cudaStream_t s, const double4* tree_sources = nullptr);
// Adjoint of the compact FP64 density for a cotangent grid rho_bar.
int pmDensityVjp(Context& c, int64_t n, const double* x, const double* y, const double* z, const double* m,
                 double uniform_mass, const double* rho_bar, double* gx, double* gy, double* gz, cudaStream_t s);
// Density into a caller-provided compact grid of nx*ny*nz doubles; no allocation.
int pmDensityInto(const chui_treepm_config& cfg, int64_t n, const double* x, const double* y, const double* z,
                  const double* m, double uniform_mass, double* rho, cudaStream_t s);
void pmDestroy(Context& c);

// ---- tree (tree.cu) ----
int treeBuild(Context& c, int64_t n, const double* x, const double* y, const double* z,
              const double* m, double uniform_mass, const double src_lo[3], const double src_hi[3],
              cudaStream_t s);
int treeNodeBounds(Context& c, double lo[3], double hi[3], cudaStream_t s);
int treeOrderTargets(Context& c, int64_t nt, const uint32_t* active, int explicit_targets, int64_t n,
                     cudaStream_t s);

// ---- sort and scan (sort.cu) ----
// Stable LSD radix sorts by the low end_bit bits (8-bit digits; digits equal
// for every key are skipped); kin and kout must differ.
int radixSortPairsU64(Context& c, const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin,
                      uint32_t* vout, int64_t n, int end_bit, cudaStream_t s);
// batch (<= 3) independent keys-only sorts of n keys each, in the same launches
int radixSortKeysU64(Context& c, int batch, const unsigned long long* const* kin, unsigned long long* const* kout,
                     int64_t n, int end_bit, cudaStream_t s);
int radixSortPairsU32(Context& c, const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
                      int64_t n, int end_bit, cudaStream_t s);
int exclusiveScanU32(Context& c, const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s);
// Maximum of n values, returned to the host (synchronises the stream).
int maxU32(Context& c, const uint32_t* in, int64_t n, uint32_t* result, cudaStream_t s);

// ---- walk (walk.cu) ----
// Targets are the visit positions [visit_begin, visit_end) of the nt targets
// (visit_end < 0: all of them); outputs land at the targets' slots, or with
// compact at visit position - visit_begin.
int walkRun(Context& c, int64_t nt, const uint32_t* active, const double* tx, const double* ty,
            const double* tz, const double* sx, const double* sy, const double* sz,
            const double* prev_acc, const WalkParams& wp, int64_t n, cudaStream_t s,
            int64_t visit_begin = 0, int64_t visit_end = -1, bool compact = false, bool record_cost = false);

// Adjoint of the short-range force for all n particles (targets in tree
// order, after treeBuild and treeOrderTargets with the full set):
// g = G sum_j M(d) (m_k c_j - m_j c_k) per row.
int walkVjpRun(Context& c, int64_t n, const double* sx, const double* sy, const double* sz, const double* m,
               double uniform_mass, const double* cx, const double* cy, const double* cz, const WalkParams& wp,
               double* gx, double* gy, double* gz, cudaStream_t s);

// ---- reductions / small kernels (abi.cu) ----
int sourceBounds(Context& c, int64_t n, const double* x, const double* y, const double* z,
                 const double* m, double lo[3], double hi[3], double* mass_sum,
                 uint32_t* status_bits, cudaStream_t s, double* mass_range = nullptr);

const char* statusText(uint32_t bits);

// Count of this library's own kernel launches (cuFFT internals excluded),
// reported per solve in chui_treepm_stats::kernel_launches.
void noteLaunch();
uint64_t launchCount();

}  // namespace chui
