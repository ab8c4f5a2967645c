// The B200 TreePM solver behind the reference's own types.
//
// Compiled inside a CHUI build (its include/ and generated configuration on
// the include path), this class takes exactly what GravityRuntimeImpl passes to
// cosmosim::gravity::TreePmCoordinator::solveActiveSetWithPmCadence
// (src/workflows/gravity_runtime.cpp:2408-2418): the source spans, the
// reference's TreePmForceAccumulatorView, TreePmOptions, TreeSofteningView,
// TreePmProfileEvent and TreePmDiagnostics. A host swaps the coordinator's
// type for this one (one declaration) and links libchui_treepm.so; the call
// site, the option mapping (gravity_runtime.cpp:469-608) and the cadence check
// after the call stay as they are.
//
// Per-particle softening is resolved with the reference's own inline rules
// (resolveSourceSofteningEpsilon, targetSofteningEpsilonUnchecked from
// include/cosmosim/gravity/tree_softening.hpp). Options that only select an
// implementation of the same arithmetic on the CPU (leaf SIMD, residual
// lookup tables, radial coefficients, tree reuse and refit, diagnostic
// reductions, exchange batching) are accepted and have no effect here;
// options for paths this single-device solver does not have (zoom
// correction, the size-capped group walk) are rejected with
// std::invalid_argument.
#pragma once

#include <cstddef>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <vector>

#include "cosmosim/gravity/tree_pm_coupling.hpp"
#include "tree_pm_coordinator.hpp"

namespace chui::b200::cosmosim_adapter {

namespace cg = cosmosim::gravity;

class TreePmCoordinator {
 public:
  explicit TreePmCoordinator(cg::PmGridShape pm_shape)
      : m_impl(chui::b200::PmGridShape{pm_shape.nx, pm_shape.ny, pm_shape.nz}) {}

  // B200 extension: precision and walk (FP64 runs the same solver in double).
  void setPrecision(Precision precision) { m_precision = precision; }
  void setWalkDiagnostics(WalkDiagnostics mode) { m_walk = mode; }
  void setDevice(int device) { m_device = device; }

  void solveActiveSetWithPmCadence(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                                   std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                                   const cg::TreePmForceAccumulatorView& accumulator, const cg::TreePmOptions& options,
                                   bool refresh_long_range_field, cg::TreePmProfileEvent* profile = nullptr,
                                   cg::TreePmDiagnostics* diagnostics = nullptr,
                                   const cg::TreeSofteningView& softening_view = {}) {
    const chui::b200::TreePmOptions o = mapOptions(options);
    // the reference's softening resolution, handed over as resolved lanes
    const std::size_t n = pos_x_comoving.size();
    chui::b200::TreeSofteningView resolved{};
    std::vector<double> source_eps, target_eps;
    std::vector<std::uint8_t> source_mask, target_mask;
    const bool uniform = softening_view.source_particle_epsilon_comoving.empty() &&
                         softening_view.source_particle_epsilon_override_mask.empty() &&
                         (!softening_view.species_policy.enabled || softening_view.source_species_tag.empty());
    if (!uniform) {
      source_eps.resize(n);
      for (std::size_t i = 0; i < n; ++i)
        source_eps[i] = cg::resolveSourceSofteningEpsilon(i, options.tree_options.softening, softening_view);
      source_mask.assign(n, 1U);
      resolved.source_particle_epsilon_comoving = source_eps;
      resolved.source_particle_epsilon_override_mask = source_mask;
    }
    const auto rows = accumulator.active_particle_index;
    const bool target_lanes = !softening_view.target_particle_epsilon_comoving.empty() ||
                              (softening_view.species_policy.enabled && !softening_view.target_species_tag.empty());
    if (target_lanes) {
      const cg::ResolvedSourceSofteningView src_view{
          .representation = uniform ? cg::ResolvedSourceSofteningRepresentation::kUniform
                                    : cg::ResolvedSourceSofteningRepresentation::kMaterialized,
          .source_count = n,
          .uniform_epsilon_comoving = options.tree_options.softening.epsilon_comoving,
          .materialized_epsilon_comoving = source_eps,
      };
      const cg::ValidatedTargetSofteningView view{
          .target_epsilon_comoving = softening_view.target_particle_epsilon_comoving,
          .target_override_mask = softening_view.target_particle_epsilon_override_mask,
          .target_species_tag = softening_view.target_species_tag,
          .resolved_source_softening = src_view,
          .source_species_tag = softening_view.source_species_tag,
          .fallback = options.tree_options.softening,
          .species_policy_enabled = softening_view.species_policy.enabled,
          .species_epsilon_comoving = softening_view.species_policy.epsilon_comoving_by_species,
      };
      target_eps.resize(rows.size());
      for (std::size_t k = 0; k < rows.size(); ++k)
        target_eps[k] = cg::targetSofteningEpsilonUnchecked(k, rows[k], view);
      target_mask.assign(rows.size(), 1U);
      resolved.target_particle_epsilon_comoving = target_eps;
      resolved.target_particle_epsilon_override_mask = target_mask;
    }
    chui::b200::TreePmForceAccumulatorView acc{accumulator.active_particle_index, accumulator.accel_x_comoving,
                                               accumulator.accel_y_comoving, accumulator.accel_z_comoving};
    acc.previous_acceleration_magnitude_code = accumulator.previous_acceleration_magnitude_code;
    acc.target_pos_x_comoving = accumulator.target_pos_x_comoving;
    acc.target_pos_y_comoving = accumulator.target_pos_y_comoving;
    acc.target_pos_z_comoving = accumulator.target_pos_z_comoving;
    acc.long_range_accel_x_comoving = accumulator.long_range_accel_x_comoving;
    acc.long_range_accel_y_comoving = accumulator.long_range_accel_y_comoving;
    acc.long_range_accel_z_comoving = accumulator.long_range_accel_z_comoving;
    acc.short_range_accel_x_comoving = accumulator.short_range_accel_x_comoving;
    acc.short_range_accel_y_comoving = accumulator.short_range_accel_y_comoving;
    acc.short_range_accel_z_comoving = accumulator.short_range_accel_z_comoving;
    acc.short_range_nearest_pair_r2_comoving = accumulator.short_range_nearest_pair_r2_comoving;
    chui::b200::TreePmProfileEvent prof{};
    chui::b200::TreePmDiagnostics diag{};
    m_impl.solveActiveSetWithPmCadence(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, acc, o,
                                       refresh_long_range_field, profile ? &prof : nullptr,
                                       diagnostics ? &diag : nullptr, resolved);
    if (profile != nullptr) {
      *profile = cg::TreePmProfileEvent{};
      profile->pm_profile.total_ms = prof.pm_ms;
      profile->tree_profile.build_ms = prof.tree_profile.build_ms;
      profile->tree_profile.full_rebuild_ms = prof.tree_profile.build_ms;
      profile->tree_profile.traversal_ms = prof.tree_profile.traversal_ms;
      profile->tree_profile.build_count = prof.tree_profile.build_count;
      profile->tree_profile.visited_nodes = prof.tree_profile.visited_nodes;
      profile->tree_profile.accepted_nodes = prof.tree_profile.accepted_nodes;
      profile->tree_profile.opened_nodes = prof.tree_profile.opened_nodes;
      profile->tree_profile.particle_particle_interactions = prof.tree_profile.particle_particle_interactions;
      profile->tree_profile.traversed_target_count = prof.tree_profile.traversed_target_count;
      profile->tree_profile.actual_node_count = prof.tree_profile.actual_node_count;
      profile->tree_short_range_ms = prof.tree_short_range_ms;
      profile->coupling_overhead_ms = prof.coupling_overhead_ms;
      profile->source_preprocess_ms = prof.source_preprocess_ms;
    }
    if (diagnostics != nullptr) {
      *diagnostics = cg::TreePmDiagnostics{};
      cg::TreePmTraversalCounters& c = diagnostics->local_traversal;
      c.visited_nodes = diag.local_traversal.visited_nodes;
      c.accepted_nodes = diag.local_traversal.accepted_nodes;
      c.opened_nodes = diag.local_traversal.opened_nodes;
      c.direct_pair_evaluations = diag.local_traversal.direct_pair_evaluations;
      c.cutoff_pruned_nodes = diag.local_traversal.cutoff_pruned_nodes;
      c.cutoff_skipped_pairs = diag.local_traversal.cutoff_skipped_pairs;
      c.accepted_internal_multipoles = diag.local_traversal.accepted_internal_multipoles;
      c.accepted_leaves = diag.local_traversal.accepted_leaves;
      c.targets = diag.local_traversal.targets;
      diagnostics->local_source_count = diag.local_source_count;
      diagnostics->local_active_target_count = diag.local_active_target_count;
      diagnostics->local_tree_node_count = diag.local_tree_node_count;
      diagnostics->pm_solve_count = diag.pm_solve_count;
      diagnostics->pm_reuse_count = diag.pm_reuse_count;
      diagnostics->mesh_spacing_comoving = diag.mesh_spacing_comoving;
      diagnostics->asmth_cells = diag.asmth_cells;
      diagnostics->rcut_cells = diag.rcut_cells;
      diagnostics->split_scale_comoving = diag.split_scale_comoving;
      diagnostics->cutoff_radius_comoving = diag.cutoff_radius_comoving;
      diagnostics->residual_pruned_nodes = diag.residual_pruned_nodes;
      diagnostics->residual_pair_skips_cutoff = diag.residual_pair_skips_cutoff;
      diagnostics->residual_pair_evaluations = diag.residual_pair_evaluations;
      diagnostics->local_pair_evaluations = diag.local_pair_evaluations;
    }
  }

  void solveActiveSet(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                      std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                      const cg::TreePmForceAccumulatorView& accumulator, const cg::TreePmOptions& options,
                      cg::TreePmProfileEvent* profile = nullptr, cg::TreePmDiagnostics* diagnostics = nullptr,
                      const cg::TreeSofteningView& softening_view = {}) {
    solveActiveSetWithPmCadence(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, accumulator, options, true,
                                profile, diagnostics, softening_view);
  }

 private:
  chui::b200::TreePmOptions mapOptions(const cg::TreePmOptions& r) const {
    if (r.enable_zoom_long_range_correction)
      throw std::invalid_argument("B200 TreePM: the zoom long-range correction is not supported");
    if (r.group_walk_enabled && r.group_walk_target_group_size != 0U)
      throw std::invalid_argument("B200 TreePM: group_walk_target_group_size must be 0 (leaf groups)");
    if (r.tree_options.softening.kernel != cg::TreeSofteningKernel::kPlummer)
      throw std::invalid_argument("Unsupported tree softening kernel");
    chui::b200::TreePmOptions o;
    o.pm_options.box_size_x_mpc_comoving = r.pm_options.box_size_x_mpc_comoving;
    o.pm_options.box_size_y_mpc_comoving = r.pm_options.box_size_y_mpc_comoving;
    o.pm_options.box_size_z_mpc_comoving = r.pm_options.box_size_z_mpc_comoving;
    o.pm_options.box_size_mpc_comoving = r.pm_options.box_size_mpc_comoving;
    o.pm_options.gravitational_constant_code = r.pm_options.gravitational_constant_code;
    o.pm_options.assignment_scheme = r.pm_options.assignment_scheme == cg::PmAssignmentScheme::kTsc
                                         ? PmAssignmentScheme::kTsc
                                         : PmAssignmentScheme::kCic;
    o.pm_options.enable_window_deconvolution = r.pm_options.enable_window_deconvolution;
    o.pm_options.boundary_condition = r.pm_options.boundary_condition == cg::PmBoundaryCondition::kIsolatedOpen
                                          ? PmBoundaryCondition::kIsolatedOpen
                                          : PmBoundaryCondition::kPeriodic;
    o.tree_options.opening_theta = r.tree_options.opening_theta;
    o.tree_options.opening_criterion =
        r.tree_options.opening_criterion == cg::TreeOpeningCriterion::kBarnesHutGeometric
            ? TreeOpeningCriterion::kBarnesHutGeometric
            : (r.tree_options.opening_criterion == cg::TreeOpeningCriterion::kRelativeForceError
                   ? TreeOpeningCriterion::kRelativeForceError
                   : TreeOpeningCriterion::kBarnesHutComDistance);
    o.tree_options.multipole_order = r.tree_options.multipole_order == cg::TreeMultipoleOrder::kMonopole
                                         ? TreeMultipoleOrder::kMonopole
                                         : TreeMultipoleOrder::kQuadrupole;
    o.tree_options.gravitational_constant_code = r.tree_options.gravitational_constant_code;
    o.tree_options.max_leaf_size = r.tree_options.max_leaf_size;
    o.tree_options.relative_force_tolerance = r.tree_options.relative_force_tolerance;
    o.tree_options.relative_force_acceleration_floor_code = r.tree_options.relative_force_acceleration_floor_code;
    o.tree_options.softening.epsilon_comoving = r.tree_options.softening.epsilon_comoving;
    o.split_policy.asmth_cells = r.split_policy.asmth_cells;
    o.split_policy.rcut_cells = r.split_policy.rcut_cells;
    o.acceptance_policy = r.acceptance_policy == cg::TreePmAcceptancePolicy::kAdaptiveRelative
                              ? TreePmAcceptancePolicy::kAdaptiveRelative
                              : TreePmAcceptancePolicy::kStrictReference;
    o.adaptive_maximum_opening_angle = r.adaptive_maximum_opening_angle;
    o.adaptive_error_estimator = r.adaptive_error_estimator == cg::TreePmAdaptiveErrorEstimator::kRelativeMonopole
                                     ? TreePmAdaptiveErrorEstimator::kRelativeMonopole
                                     : TreePmAdaptiveErrorEstimator::kResidualDerivative;
    o.cutoff_node_policy = r.cutoff_node_policy == cg::TreePmCutoffNodePolicy::kComDistance
                               ? TreePmCutoffNodePolicy::kComDistance
                               : TreePmCutoffNodePolicy::kContainNode;
    o.group_walk_enabled = r.group_walk_enabled;
    o.gaussian_pair_lookup_enabled = r.gaussian_pair_lookup_enabled;
    o.short_range_only = r.short_range_only;
    o.precision = m_precision;
    o.walk_diagnostics = m_walk;
    o.device = m_device;
    return o;
  }

  chui::b200::TreePmCoordinator m_impl;
  Precision m_precision = Precision::kMixed;
  WalkDiagnostics m_walk = WalkDiagnostics::kAuto;
  int m_device = 0;
};

}  // namespace chui::b200::cosmosim_adapter
