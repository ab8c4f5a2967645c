// C++20 host shim: the reference's gravity-solver interface over the B200
// C-ABI (include/chui_treepm.h).
//
// A CHUI host compiles against this header instead of
// include/cosmosim/gravity/tree_pm_coupling.hpp and links
// libchui_treepm.so; GravityRuntimeImpl keeps calling
// solveActiveSetWithPmCadence with the same spans, accumulator view, options
// and refresh flag (src/workflows/gravity_runtime.cpp:2408). The types below
// carry the field names and meaning of the reference's TreePmOptions,
// TreePmForceAccumulatorView and PmGridShape for the periodic strict path;
// C-ABI status codes are rethrown as the reference's exception types
// (std::invalid_argument, std::out_of_range / std::overflow_error,
// std::runtime_error, std::bad_alloc).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <new>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/chui_treepm.h"

namespace chui::b200 {

using TreeLocalIndex = std::uint32_t;
inline constexpr TreeLocalIndex kInvalidTreeLocalIndex = 0xFFFFFFFFu;

// include/cosmosim/gravity/pm_solver.hpp (PmGridShape)
struct PmGridShape {
  std::size_t nx = 0, ny = 0, nz = 0;
  [[nodiscard]] bool isValid() const noexcept { return nx > 0 && ny > 0 && nz > 0; }
};

enum class PmAssignmentScheme { kCic, kTsc };
enum class PmBoundaryCondition { kPeriodic, kIsolatedOpen };
enum class TreeOpeningCriterion { kBarnesHutGeometric, kBarnesHutComDistance, kRelativeForceError };
enum class TreeMultipoleOrder { kMonopole = 0, kQuadrupole = 2 };
enum class TreePmAcceptancePolicy { kStrictReference, kAdaptiveRelative };
enum class TreePmAdaptiveErrorEstimator { kResidualDerivative, kRelativeMonopole };
enum class TreePmCutoffNodePolicy { kContainNode, kComDistance };
enum class Precision { kMixed, kFp64 };
// B200 extension: which walk serves the solve. kAuto: the production walk,
// counting its own traversal (kProductionCounters) when the caller passes a
// TreePmDiagnostics, else uncounted (kProduction). kReferenceCounters: the
// per-node walk whose counters equal the reference's (parity checks).
enum class WalkDiagnostics { kAuto, kProduction, kReferenceCounters, kProductionCounters };

// The option fields the periodic TreePM path consumes (tree_pm_coupling.hpp:243-332,
// tree_gravity.hpp:30-43, pm_solver.hpp:223-254, tree_pm_split_kernel.hpp:20-27).
struct PmSolveOptions {
  double box_size_x_mpc_comoving = 0.0;
  double box_size_y_mpc_comoving = 0.0;
  double box_size_z_mpc_comoving = 0.0;
  double box_size_mpc_comoving = 0.0;
  double gravitational_constant_code = 1.0;
  PmAssignmentScheme assignment_scheme = PmAssignmentScheme::kCic;
  bool enable_window_deconvolution = false;
  PmBoundaryCondition boundary_condition = PmBoundaryCondition::kPeriodic;
};

struct TreeSofteningPolicy {
  double epsilon_comoving = 0.0;
};

struct TreeGravityOptions {
  double opening_theta = 0.7;
  TreeOpeningCriterion opening_criterion = TreeOpeningCriterion::kBarnesHutComDistance;
  TreeMultipoleOrder multipole_order = TreeMultipoleOrder::kQuadrupole;
  double gravitational_constant_code = 1.0;
  std::size_t max_leaf_size = 16;
  double relative_force_tolerance = 0.005;
  double relative_force_acceleration_floor_code = 1.0e-30;
  TreeSofteningPolicy softening{};
};

struct TreePmSplitPolicy {
  double asmth_cells = 1.25;
  double rcut_cells = 6.25;
};

struct TreePmOptions {
  PmSolveOptions pm_options{};
  TreeGravityOptions tree_options{};
  TreePmSplitPolicy split_policy{};
  TreePmAcceptancePolicy acceptance_policy = TreePmAcceptancePolicy::kStrictReference;
  double adaptive_maximum_opening_angle = 0.25;
  TreePmAdaptiveErrorEstimator adaptive_error_estimator = TreePmAdaptiveErrorEstimator::kResidualDerivative;
  TreePmCutoffNodePolicy cutoff_node_policy = TreePmCutoffNodePolicy::kContainNode;
  bool group_walk_enabled = false;
  bool gaussian_pair_lookup_enabled = false;
  bool short_range_only = false;  // the integrator's split operator: residual only, no PM
  Precision precision = Precision::kMixed;  // B200 extension: FP64 runs the same solver in double
  WalkDiagnostics walk_diagnostics = WalkDiagnostics::kAuto;  // B200 extension
  int device = 0;
};

// tree_pm_coupling.hpp:127-165
struct TreePmForceAccumulatorView {
  std::span<const TreeLocalIndex> active_particle_index;
  std::span<double> accel_x_comoving;
  std::span<double> accel_y_comoving;
  std::span<double> accel_z_comoving;
  std::span<const double> previous_acceleration_magnitude_code{};
  std::span<const double> target_pos_x_comoving{};
  std::span<const double> target_pos_y_comoving{};
  std::span<const double> target_pos_z_comoving{};
  std::span<double> long_range_accel_x_comoving{};
  std::span<double> long_range_accel_y_comoving{};
  std::span<double> long_range_accel_z_comoving{};
  std::span<double> short_range_accel_x_comoving{};
  std::span<double> short_range_accel_y_comoving{};
  std::span<double> short_range_accel_z_comoving{};
  std::span<double> short_range_nearest_pair_r2_comoving{};
};

// The TreePmTraversalCounters fields the walk produces (tree_pm_coupling.hpp:39-60):
// equal to the reference's with WalkDiagnostics::kReferenceCounters; the
// production walk's own traversal (subtree blocks) with kProductionCounters.
struct TreePmTraversalCounters {
  std::uint64_t visited_nodes = 0;
  std::uint64_t accepted_nodes = 0;
  std::uint64_t opened_nodes = 0;
  std::uint64_t direct_pair_evaluations = 0;
  std::uint64_t cutoff_pruned_nodes = 0;
  std::uint64_t cutoff_skipped_pairs = 0;
  std::uint64_t accepted_internal_multipoles = 0;
  std::uint64_t accepted_leaves = 0;
  std::uint64_t targets = 0;
};

// The subset of TreePmDiagnostics (tree_pm_coupling.hpp:334-470) a
// single-device periodic solve defines. GravityRuntimeImpl checks
// pm_solve_count / pm_reuse_count against its cadence decision right after
// the call (src/workflows/gravity_runtime.cpp:2418-2424).
struct TreePmDiagnostics {
  TreePmTraversalCounters local_traversal{};
  std::uint64_t local_source_count = 0;
  std::uint64_t local_active_target_count = 0;
  std::uint64_t local_tree_node_count = 0;
  std::uint64_t pm_solve_count = 0;
  std::uint64_t pm_reuse_count = 0;
  double mesh_spacing_comoving = 0.0;
  double asmth_cells = 0.0;
  double rcut_cells = 0.0;
  double split_scale_comoving = 0.0;
  double cutoff_radius_comoving = 0.0;
  std::uint64_t residual_pruned_nodes = 0;
  std::uint64_t residual_pair_skips_cutoff = 0;
  std::uint64_t residual_pair_evaluations = 0;
  std::uint64_t local_pair_evaluations = 0;
  chui_treepm_stats stats{};  // raw C-ABI record (maximum depth, launches, ...)
};

// Phase timings in the shape of TreePmProfileEvent (tree_pm_coupling.hpp:505-524)
// and TreeGravityProfile (tree_gravity.hpp:45-59); device times from CUDA events.
struct TreeGravityProfile {
  double build_ms = 0.0;
  double multipole_ms = 0.0;
  double traversal_ms = 0.0;
  std::uint64_t build_count = 0;
  std::uint64_t visited_nodes = 0;
  std::uint64_t accepted_nodes = 0;
  std::uint64_t opened_nodes = 0;
  std::uint64_t particle_particle_interactions = 0;
  std::uint64_t traversed_target_count = 0;
  std::uint64_t actual_node_count = 0;
};

struct TreePmProfileEvent {
  double pm_ms = 0.0;  // PM refresh (deposit, FFTs, Green, gradient) and interpolation
  TreeGravityProfile tree_profile{};
  double tree_short_range_ms = 0.0;
  double coupling_overhead_ms = 0.0;
  double source_preprocess_ms = 0.0;
};

// tree_softening.hpp:26-47: per-particle softening sidecars. Resolved here
// into the C-ABI's epsilon lanes with the reference's rules
// (resolveSourceSofteningEpsilon :152-180, targetSofteningEpsilonUnchecked
// :90-110, sourceSofteningIsProvablyUniform tree_gravity.cpp:82-94).
struct TreeSofteningSpeciesPolicy {
  static constexpr std::size_t kSpeciesCapacity = 6;  // core::k_particle_species_count
  std::array<double, kSpeciesCapacity> epsilon_comoving_by_species{};
  bool enabled = false;
};

struct TreeSofteningView {
  std::span<const std::uint32_t> source_species_tag{};
  std::span<const double> source_particle_epsilon_comoving{};
  std::span<const std::uint8_t> source_particle_epsilon_override_mask{};
  std::span<const std::uint32_t> target_species_tag{};
  std::span<const double> target_particle_epsilon_comoving{};
  std::span<const std::uint8_t> target_particle_epsilon_override_mask{};
  TreeSofteningSpeciesPolicy species_policy{};
};

namespace softening_detail {

inline double validated(double v, const char* what) {
  if (!std::isfinite(v) || v < 0.0) throw std::invalid_argument(std::string(what) + " must be finite and non-negative");
  return v;
}

inline double speciesEpsilon(const TreeSofteningSpeciesPolicy& p, std::uint32_t tag, const char* what) {
  if (tag >= p.epsilon_comoving_by_species.size())
    throw std::invalid_argument("species tag is outside the canonical species range");
  return validated(p.epsilon_comoving_by_species[tag], what);
}

// Per-source epsilons, or empty when the sources are provably uniform.
inline std::vector<double> resolveSources(std::size_t n, double fallback, const TreeSofteningView& v) {
  const bool species = v.species_policy.enabled && !v.source_species_tag.empty();
  if (v.source_particle_epsilon_comoving.empty() && v.source_particle_epsilon_override_mask.empty() && !species)
    return {};
  if ((!v.source_particle_epsilon_comoving.empty() && v.source_particle_epsilon_comoving.size() != n) ||
      (!v.source_particle_epsilon_override_mask.empty() && v.source_particle_epsilon_override_mask.size() != n) ||
      (!v.source_species_tag.empty() && v.source_species_tag.size() != n))
    throw std::invalid_argument("TreePM softening/species sidecar extent mismatch");
  std::vector<double> eps(n, validated(fallback, "Tree softening epsilon_comoving"));
  for (std::size_t i = 0; i < n; ++i) {
    if (!v.source_particle_epsilon_comoving.empty() && !v.source_particle_epsilon_override_mask.empty() &&
        v.source_particle_epsilon_override_mask[i] != 0U) {
      eps[i] = validated(v.source_particle_epsilon_comoving[i], "source softening override");
    } else if (species) {
      eps[i] = speciesEpsilon(v.species_policy, v.source_species_tag[i], "source species softening");
    }
  }
  return eps;
}

// Per-active-slot target epsilons, or empty when the library's default (a
// target that is a source takes its source epsilon, others the configured
// one) gives the same values.
inline std::vector<double> resolveTargets(std::span<const std::uint32_t> rows, std::size_t sources,
                                          const std::vector<double>& source_eps, double fallback,
                                          const TreeSofteningView& v) {
  const bool target_species = v.species_policy.enabled && !v.target_species_tag.empty();
  if (v.target_particle_epsilon_comoving.empty() && !target_species) return {};
  const std::size_t nt = rows.size();
  if ((!v.target_particle_epsilon_comoving.empty() && v.target_particle_epsilon_comoving.size() != nt) ||
      (!v.target_particle_epsilon_override_mask.empty() && v.target_particle_epsilon_override_mask.size() != nt) ||
      (!v.target_species_tag.empty() && v.target_species_tag.size() != nt))
    throw std::invalid_argument("TreePM softening/species sidecar extent mismatch");
  std::vector<double> eps(nt);
  for (std::size_t k = 0; k < nt; ++k) {
    const std::size_t row = rows[k];
    if (!v.target_particle_epsilon_comoving.empty() && !v.target_particle_epsilon_override_mask.empty() &&
        v.target_particle_epsilon_override_mask[k] != 0U) {
      eps[k] = validated(v.target_particle_epsilon_comoving[k], "target softening override");
    } else if (target_species) {
      eps[k] = speciesEpsilon(v.species_policy, v.target_species_tag[k], "target species softening");
    } else if (v.target_particle_epsilon_comoving.empty() && row < sources) {
      eps[k] = source_eps.empty() ? fallback : source_eps[row];
    } else if (v.species_policy.enabled && row < v.source_species_tag.size()) {
      eps[k] = speciesEpsilon(v.species_policy, v.source_species_tag[row], "target species softening");
    } else {
      eps[k] = fallback;
    }
  }
  return eps;
}

}  // namespace softening_detail

class TreePmCoordinator {
 public:
  explicit TreePmCoordinator(PmGridShape pm_shape) : m_shape(pm_shape) {
    if (!m_shape.isValid()) throw std::invalid_argument("numerics.treepm_pm_grid_n{xyz} must all be > 0");
  }
  ~TreePmCoordinator() { chui_treepm_destroy(m_handle); }
  TreePmCoordinator(const TreePmCoordinator&) = delete;
  TreePmCoordinator& operator=(const TreePmCoordinator&) = delete;

  void solveActiveSetWithPmCadence(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                                   std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                                   const TreePmForceAccumulatorView& accumulator, const TreePmOptions& options,
                                   bool refresh_long_range_field, TreePmProfileEvent* profile = nullptr,
                                   TreePmDiagnostics* diagnostics = nullptr,
                                   const TreeSofteningView& softening_view = {}) {
    solve(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, accumulator, options, refresh_long_range_field,
          profile, diagnostics, softening_view, false, 0, 0);
  }

  // One shard of the solve, for processes that each hold every source (no
  // counterpart in the reference): only the targets at visit positions
  // [visit_begin, visit_end) of the accumulator's active set are walked, and
  // accel_* / long_range_* hold visit_end - visit_begin entries in visit
  // order; visitOrder() names their active slots. Both ends are multiples of
  // 64 or the active count.
  void solveVisitRange(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                       std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                       const TreePmForceAccumulatorView& accumulator, const TreePmOptions& options,
                       bool refresh_long_range_field, std::size_t visit_begin, std::size_t visit_end,
                       TreePmProfileEvent* profile = nullptr, TreePmDiagnostics* diagnostics = nullptr) {
    solve(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, accumulator, options, refresh_long_range_field,
          profile, diagnostics, {}, true, visit_begin, visit_end);
  }

  // Active slots at visit positions [begin, end) of the last solve.
  std::vector<std::uint32_t> visitOrder(std::size_t begin, std::size_t end) const {
    std::vector<std::uint32_t> slots(end > begin ? end - begin : 0);
    check(chui_treepm_visit_order(m_handle, static_cast<std::int64_t>(begin), static_cast<std::int64_t>(end),
                                  slots.data(), CHUI_TREEPM_HOST, nullptr));
    return slots;
  }

  void solveActiveSet(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                      std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                      const TreePmForceAccumulatorView& accumulator, const TreePmOptions& options,
                      TreePmProfileEvent* profile = nullptr, TreePmDiagnostics* diagnostics = nullptr,
                      const TreeSofteningView& softening_view = {}) {
    solveActiveSetWithPmCadence(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, accumulator, options,
                                true, profile, diagnostics, softening_view);
  }

 private:
  void solve(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
             std::span<const double> pos_z_comoving, std::span<const double> mass_code,
             const TreePmForceAccumulatorView& accumulator, const TreePmOptions& options,
             bool refresh_long_range_field, TreePmProfileEvent* profile, TreePmDiagnostics* diagnostics,
             const TreeSofteningView& softening_view, bool ranged, std::size_t visit_begin, std::size_t visit_end) {
    if (pos_x_comoving.size() != pos_y_comoving.size() || pos_x_comoving.size() != pos_z_comoving.size() ||
        pos_x_comoving.size() != mass_code.size()) {
      throw std::invalid_argument("TreePM requires position and mass spans with equal extent");
    }
    const std::size_t targets = accumulator.active_particle_index.size();
    const std::size_t outputs = ranged ? (visit_end > visit_begin ? visit_end - visit_begin : 0) : targets;
    if (accumulator.accel_x_comoving.size() != outputs || accumulator.accel_y_comoving.size() != outputs ||
        accumulator.accel_z_comoving.size() != outputs) {
      throw std::invalid_argument("TreePM force accumulator spans must have matching active-set extent");
    }
    if (!accumulator.previous_acceleration_magnitude_code.empty() &&
        accumulator.previous_acceleration_magnitude_code.size() != targets) {
      throw std::invalid_argument("TreePM force accumulator spans must have matching active-set extent");
    }
    configure(options, diagnostics != nullptr);
    // per-particle softening: resolved epsilon lanes
    const double eps0 = options.tree_options.softening.epsilon_comoving;
    m_source_eps = softening_detail::resolveSources(pos_x_comoving.size(), eps0, softening_view);
    m_target_eps = softening_detail::resolveTargets(accumulator.active_particle_index, pos_x_comoving.size(),
                                                    m_source_eps, eps0, softening_view);
    chui_treepm_sources src{};
    src.count = static_cast<std::int64_t>(pos_x_comoving.size());
    src.x = pos_x_comoving.data();
    src.y = pos_y_comoving.data();
    src.z = pos_z_comoving.data();
    src.mass = mass_code.data();
    src.softening = m_source_eps.empty() ? nullptr : m_source_eps.data();
    chui_treepm_accumulator acc{};
    acc.active_count = static_cast<std::int64_t>(targets);
    acc.active_index = accumulator.active_particle_index.data();
    acc.accel_x = accumulator.accel_x_comoving.data();
    acc.accel_y = accumulator.accel_y_comoving.data();
    acc.accel_z = accumulator.accel_z_comoving.data();
    acc.target_softening = m_target_eps.empty() ? nullptr : m_target_eps.data();
    if (!accumulator.previous_acceleration_magnitude_code.empty()) {
      acc.previous_acceleration_magnitude = accumulator.previous_acceleration_magnitude_code.data();
    }
    if (!accumulator.target_pos_x_comoving.empty()) {
      acc.target_x = accumulator.target_pos_x_comoving.data();
      acc.target_y = accumulator.target_pos_y_comoving.data();
      acc.target_z = accumulator.target_pos_z_comoving.data();
    }
    if (!accumulator.long_range_accel_x_comoving.empty()) {
      acc.long_range_x = accumulator.long_range_accel_x_comoving.data();
      acc.long_range_y = accumulator.long_range_accel_y_comoving.data();
      acc.long_range_z = accumulator.long_range_accel_z_comoving.data();
    }
    if (!accumulator.short_range_accel_x_comoving.empty()) {
      if (accumulator.short_range_accel_x_comoving.size() != pos_x_comoving.size()) {
        throw std::invalid_argument("Tree component output requires source-indexed full source extents");
      }
      acc.short_range_x = accumulator.short_range_accel_x_comoving.data();
      acc.short_range_y = accumulator.short_range_accel_y_comoving.data();
      acc.short_range_z = accumulator.short_range_accel_z_comoving.data();
      for (const TreeLocalIndex row : accumulator.active_particle_index) {
        if (row < pos_x_comoving.size()) {
          // the reference resets each active row before accumulating (tree_pm_coupling.cpp:2417-2424)
          accumulator.short_range_accel_x_comoving[row] = 0.0;
          accumulator.short_range_accel_y_comoving[row] = 0.0;
          accumulator.short_range_accel_z_comoving[row] = 0.0;
        }
      }
    }
    if (!accumulator.short_range_nearest_pair_r2_comoving.empty()) {
      acc.nearest_pair_r2 = accumulator.short_range_nearest_pair_r2_comoving.data();
    }
    if (!accumulator.long_range_accel_x_comoving.empty() && accumulator.long_range_accel_x_comoving.size() != outputs) {
      throw std::invalid_argument("TreePM force accumulator spans must have matching active-set extent");
    }
    chui_treepm_stats stats{};
    if (ranged) {
      check(chui_treepm_solve_visit_range(m_handle, &src, &acc, refresh_long_range_field ? 1 : 0, CHUI_TREEPM_HOST,
                                          nullptr, &stats, static_cast<std::int64_t>(visit_begin),
                                          static_cast<std::int64_t>(visit_end)));
    } else {
      check(chui_treepm_solve(m_handle, &src, &acc, refresh_long_range_field ? 1 : 0, CHUI_TREEPM_HOST, nullptr,
                              &stats));
    }
    // a visit-range solve walks only its slice's targets
    if (diagnostics != nullptr) fillDiagnostics(stats, pos_x_comoving.size(), outputs, refresh_long_range_field, *diagnostics);
    if (profile != nullptr) {
      *profile = TreePmProfileEvent{};
      profile->pm_ms = stats.pm_ms;
      profile->source_preprocess_ms = stats.tree_build_ms;
      profile->tree_short_range_ms = stats.walk_ms;
      profile->coupling_overhead_ms = stats.total_ms - stats.pm_ms - stats.tree_build_ms - stats.walk_ms;
      TreeGravityProfile& t = profile->tree_profile;
      t.build_ms = stats.tree_build_ms;
      t.traversal_ms = stats.walk_ms;
      t.build_count = 1;
      t.visited_nodes = stats.visited_nodes;
      t.accepted_nodes = stats.accepted_nodes;
      t.opened_nodes = stats.opened_nodes;
      t.particle_particle_interactions = stats.direct_pair_evaluations;
      t.traversed_target_count = outputs;
      t.actual_node_count = stats.node_count;
    }
  }

  void fillDiagnostics(const chui_treepm_stats& s, std::size_t sources, std::size_t targets, bool refresh,
                       TreePmDiagnostics& d) const {
    d = TreePmDiagnostics{};
    d.stats = s;
    TreePmTraversalCounters& c = d.local_traversal;
    c.visited_nodes = s.visited_nodes;
    c.accepted_nodes = s.accepted_nodes;
    c.opened_nodes = s.opened_nodes;
    c.direct_pair_evaluations = s.direct_pair_evaluations;
    c.cutoff_pruned_nodes = s.cutoff_pruned_nodes;
    c.cutoff_skipped_pairs = s.cutoff_skipped_pairs;
    c.accepted_internal_multipoles = s.accepted_internal_multipoles;
    c.accepted_leaves = s.accepted_leaves;
    c.targets = targets;
    d.local_source_count = sources;
    d.local_active_target_count = targets;
    d.local_tree_node_count = s.node_count;
    // short-range only: neither a PM solve nor a reuse (gravity_runtime.cpp:2418-2424)
    d.pm_solve_count = refresh && !m_short_only ? 1U : 0U;
    d.pm_reuse_count = refresh || m_short_only ? 0U : 1U;
    d.mesh_spacing_comoving = m_spacing;
    d.asmth_cells = m_asmth;
    d.rcut_cells = m_rcut;
    d.split_scale_comoving = m_asmth * m_spacing;
    d.cutoff_radius_comoving = m_rcut * m_spacing;
    d.residual_pruned_nodes = s.cutoff_pruned_nodes;
    d.residual_pair_skips_cutoff = s.cutoff_skipped_pairs;
    d.residual_pair_evaluations = s.direct_pair_evaluations;
    d.local_pair_evaluations = s.direct_pair_evaluations;
  }

  void configure(const TreePmOptions& o, bool counters_wanted) {
    chui_treepm_config c{};
    chui_treepm_config_default(&c);
    c.pm_grid_nx = static_cast<std::int64_t>(m_shape.nx);
    c.pm_grid_ny = static_cast<std::int64_t>(m_shape.ny);
    c.pm_grid_nz = static_cast<std::int64_t>(m_shape.nz);
    const double scalar = o.pm_options.box_size_mpc_comoving;
    c.box_x = o.pm_options.box_size_x_mpc_comoving > 0.0 ? o.pm_options.box_size_x_mpc_comoving : scalar;
    c.box_y = o.pm_options.box_size_y_mpc_comoving > 0.0 ? o.pm_options.box_size_y_mpc_comoving : scalar;
    c.box_z = o.pm_options.box_size_z_mpc_comoving > 0.0 ? o.pm_options.box_size_z_mpc_comoving : scalar;
    if (o.tree_options.gravitational_constant_code != o.pm_options.gravitational_constant_code) {
      throw std::invalid_argument("TreePM PM and tree gravitational_constant_code values must match");
    }
    c.gravitational_constant = o.pm_options.gravitational_constant_code;
    c.asmth_cells = o.split_policy.asmth_cells;
    c.rcut_cells = o.split_policy.rcut_cells;
    c.opening_theta = o.tree_options.opening_theta;
    c.opening_criterion = static_cast<std::int32_t>(o.tree_options.opening_criterion);
    c.multipole_order = static_cast<std::int32_t>(o.tree_options.multipole_order);
    c.max_leaf_size = static_cast<std::int64_t>(o.tree_options.max_leaf_size);
    c.assignment_scheme = o.pm_options.assignment_scheme == PmAssignmentScheme::kTsc ? CHUI_TREEPM_TSC : CHUI_TREEPM_CIC;
    c.window_deconvolution = o.pm_options.enable_window_deconvolution ? 1 : 0;
    c.boundary_condition = o.pm_options.boundary_condition == PmBoundaryCondition::kIsolatedOpen
                               ? CHUI_TREEPM_BOUNDARY_ISOLATED_OPEN
                               : CHUI_TREEPM_BOUNDARY_PERIODIC;
    c.softening = o.tree_options.softening.epsilon_comoving;
    c.acceptance_policy = o.acceptance_policy == TreePmAcceptancePolicy::kStrictReference ? CHUI_TREEPM_POLICY_STRICT
                                                                                        : CHUI_TREEPM_POLICY_ADAPTIVE;
    c.adaptive_error_estimator = o.adaptive_error_estimator == TreePmAdaptiveErrorEstimator::kRelativeMonopole
                                     ? CHUI_TREEPM_ESTIMATOR_RELATIVE_MONOPOLE
                                     : CHUI_TREEPM_ESTIMATOR_RESIDUAL_DERIVATIVE;
    c.cutoff_node_policy = o.cutoff_node_policy == TreePmCutoffNodePolicy::kComDistance
                               ? CHUI_TREEPM_CUTOFF_COM_DISTANCE
                               : CHUI_TREEPM_CUTOFF_CONTAIN_NODE;
    c.adaptive_maximum_opening_angle = o.adaptive_maximum_opening_angle;
    c.relative_force_tolerance = o.tree_options.relative_force_tolerance;
    c.relative_force_acceleration_floor = o.tree_options.relative_force_acceleration_floor_code;
    c.group_walk_enabled = o.group_walk_enabled ? 1 : 0;
    c.gaussian_pair_lookup = o.gaussian_pair_lookup_enabled ? 1 : 0;
    c.precision = o.precision == Precision::kFp64 ? CHUI_TREEPM_FP64 : CHUI_TREEPM_MIXED;
    c.short_range_only = o.short_range_only ? 1 : 0;
    m_short_only = o.short_range_only;
    switch (o.walk_diagnostics) {
      case WalkDiagnostics::kAuto: c.diagnostics = counters_wanted ? 2 : 0; break;
      case WalkDiagnostics::kProduction: c.diagnostics = 0; break;
      case WalkDiagnostics::kReferenceCounters: c.diagnostics = 1; break;
      case WalkDiagnostics::kProductionCounters: c.diagnostics = 2; break;
    }
    c.device = o.device;
    // split scale and cutoff are in units of the mean mesh spacing (gravity_runtime.cpp:586-590)
    m_spacing = std::cbrt((c.box_x / c.pm_grid_nx) * (c.box_y / c.pm_grid_ny) * (c.box_z / c.pm_grid_nz));
    m_asmth = c.asmth_cells;
    m_rcut = c.rcut_cells;
    if (m_handle == nullptr) {
      check(chui_treepm_create(&c, &m_handle));
    } else {
      check(chui_treepm_set_config(m_handle, &c));
    }
  }

  void check(int rc) const {
    if (rc == CHUI_TREEPM_OK) return;
    const std::string msg = chui_treepm_last_error(m_handle);
    switch (rc) {
      case CHUI_TREEPM_EINVAL:
      case CHUI_TREEPM_ENOTSUP:
        throw std::invalid_argument(msg);
      case CHUI_TREEPM_ERANGE:
        if (msg.find("overflow") != std::string::npos || msg.find("depth") != std::string::npos) {
          throw std::overflow_error(msg);
        }
        throw std::out_of_range(msg);
      case CHUI_TREEPM_ENOMEM:
        throw std::bad_alloc();
      default:
        throw std::runtime_error(msg.empty() ? "B200 TreePM failure" : msg);
    }
  }

  PmGridShape m_shape;
  void* m_handle = nullptr;
  std::vector<double> m_source_eps, m_target_eps;
  bool m_short_only = false;
  double m_spacing = 0.0;
  double m_asmth = 0.0;
  double m_rcut = 0.0;
};

}  // namespace chui::b200
