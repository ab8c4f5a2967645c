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

#include <cstddef>
#include <cstdint>
#include <new>
#include <span>
#include <stdexcept>
#include <string>

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
enum class TreeOpeningCriterion { kBarnesHutGeometric, kBarnesHutComDistance, kRelativeForceError };
enum class TreeMultipoleOrder { kMonopole = 0, kQuadrupole = 2 };
enum class TreePmAcceptancePolicy { kStrictReference, kAdaptiveRelative };
enum class Precision { kMixed, kFp64 };

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
  Precision precision = Precision::kMixed;  // B200 extension: FP64 runs the same solver in double
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

// The counters of TreePmTraversalCounters plus the phase timings.
struct TreePmDiagnostics {
  chui_treepm_stats stats{};
};

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
                                   bool refresh_long_range_field, TreePmDiagnostics* diagnostics = nullptr) {
    if (pos_x_comoving.size() != pos_y_comoving.size() || pos_x_comoving.size() != pos_z_comoving.size() ||
        pos_x_comoving.size() != mass_code.size()) {
      throw std::invalid_argument("TreePM requires position and mass spans with equal extent");
    }
    const std::size_t targets = accumulator.active_particle_index.size();
    if (accumulator.accel_x_comoving.size() != targets || accumulator.accel_y_comoving.size() != targets ||
        accumulator.accel_z_comoving.size() != targets) {
      throw std::invalid_argument("TreePM force accumulator spans must have matching active-set extent");
    }
    configure(options);
    chui_treepm_sources src{};
    src.count = static_cast<std::int64_t>(pos_x_comoving.size());
    src.x = pos_x_comoving.data();
    src.y = pos_y_comoving.data();
    src.z = pos_z_comoving.data();
    src.mass = mass_code.data();
    chui_treepm_accumulator acc{};
    acc.active_count = static_cast<std::int64_t>(targets);
    acc.active_index = accumulator.active_particle_index.data();
    acc.accel_x = accumulator.accel_x_comoving.data();
    acc.accel_y = accumulator.accel_y_comoving.data();
    acc.accel_z = accumulator.accel_z_comoving.data();
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
    chui_treepm_stats stats{};
    check(chui_treepm_solve(m_handle, &src, &acc, refresh_long_range_field ? 1 : 0, CHUI_TREEPM_HOST, nullptr,
                            &stats));
    if (diagnostics != nullptr) diagnostics->stats = stats;
  }

  void solveActiveSet(std::span<const double> pos_x_comoving, std::span<const double> pos_y_comoving,
                      std::span<const double> pos_z_comoving, std::span<const double> mass_code,
                      const TreePmForceAccumulatorView& accumulator, const TreePmOptions& options,
                      TreePmDiagnostics* diagnostics = nullptr) {
    solveActiveSetWithPmCadence(pos_x_comoving, pos_y_comoving, pos_z_comoving, mass_code, accumulator, options,
                                true, diagnostics);
  }

 private:
  void configure(const TreePmOptions& o) {
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
    c.softening = o.tree_options.softening.epsilon_comoving;
    c.acceptance_policy = o.acceptance_policy == TreePmAcceptancePolicy::kStrictReference ? 0 : 1;
    c.precision = o.precision == Precision::kFp64 ? CHUI_TREEPM_FP64 : CHUI_TREEPM_MIXED;
    c.device = o.device;
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
};

}  // namespace chui::b200
