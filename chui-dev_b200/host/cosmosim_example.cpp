// Example host program: the reference runtime's call into the TreePM
// coordinator (src/workflows/gravity_runtime.cpp:2383-2424), compiled against
// the reference's own headers with the B200 coordinator type in place of
// cosmosim::gravity::TreePmCoordinator. Reads a problem (n, box, mesh, theta,
// leaf, eps, deconvolution flag, softening-lane flag as doubles/int64, then x,
// y, z, m and, with the flag, per-source epsilons and override masks as
// doubles), solves all particles with a PM refresh, checks the runtime's
// cadence invariant on the diagnostics, solves again reusing the PM field,
// and writes both accelerations.
//   g++ -std=c++20 -O2 -I<CHUI>/include -I<generated config> cosmosim_example.cpp
//       -L../_build -lchui_treepm -o cosmosim_example
#include <cstdint>
#include <cstdio>
#include <exception>
#include <numeric>
#include <vector>

#include "cosmosim_tree_pm_coordinator.hpp"

namespace gravity = cosmosim::gravity;

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: cosmosim_example <in.bin> <out.bin>\n");
    return 2;
  }
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::int64_t n = 0, mesh = 0, leaf = 0, deconv = 0, has_soft = 0;
  double box = 0, theta = 0, eps = 0;
  bool ok = std::fread(&n, 8, 1, f) == 1 && std::fread(&box, 8, 1, f) == 1 && std::fread(&mesh, 8, 1, f) == 1 &&
            std::fread(&theta, 8, 1, f) == 1 && std::fread(&leaf, 8, 1, f) == 1 && std::fread(&eps, 8, 1, f) == 1 &&
            std::fread(&deconv, 8, 1, f) == 1 && std::fread(&has_soft, 8, 1, f) == 1;
  std::vector<double> x(n), y(n), z(n), m(n), src_eps, mask_d;
  for (auto* v : {&x, &y, &z, &m}) ok = ok && std::fread(v->data(), 8, n, f) == static_cast<std::size_t>(n);
  if (has_soft) {
    src_eps.resize(n);
    mask_d.resize(n);
    ok = ok && std::fread(src_eps.data(), 8, n, f) == static_cast<std::size_t>(n) &&
         std::fread(mask_d.data(), 8, n, f) == static_cast<std::size_t>(n);
  }
  std::fclose(f);
  if (!ok) return 2;
  std::vector<std::uint8_t> src_mask(mask_d.size());
  for (std::size_t i = 0; i < mask_d.size(); ++i) src_mask[i] = mask_d[i] != 0.0 ? 1U : 0U;
  try {
    // the runtime's option mapping (gravity_runtime.cpp:469-608)
    gravity::TreePmOptions options;
    options.pm_options.box_size_x_mpc_comoving = box;
    options.pm_options.box_size_y_mpc_comoving = box;
    options.pm_options.box_size_z_mpc_comoving = box;
    options.pm_options.box_size_mpc_comoving = box;
    options.pm_options.gravitational_constant_code = 1.0;
    options.pm_options.assignment_scheme = gravity::PmAssignmentScheme::kCic;
    options.pm_options.enable_window_deconvolution = deconv != 0;
    options.tree_options.gravitational_constant_code = 1.0;
    options.tree_options.opening_theta = theta;
    options.tree_options.max_leaf_size = static_cast<std::size_t>(leaf);
    options.tree_options.softening.epsilon_comoving = eps;
    options.split_policy.asmth_cells = 1.25;
    options.split_policy.rcut_cells = 6.25;
    chui::b200::cosmosim_adapter::TreePmCoordinator coordinator(
        gravity::PmGridShape{static_cast<std::size_t>(mesh), static_cast<std::size_t>(mesh),
                             static_cast<std::size_t>(mesh)});
    std::vector<std::uint32_t> active(n);
    std::iota(active.begin(), active.end(), 0u);
    std::vector<double> ax(n), ay(n), az(n), bx(n), by(n), bz(n);
    gravity::TreePmForceAccumulatorView accumulator{active, ax, ay, az};
    gravity::TreePmDiagnostics diagnostics;
    const gravity::TreeSofteningView softening_view{
        .source_species_tag = {},
        .source_particle_epsilon_comoving = std::span<const double>(src_eps.data(), src_eps.size()),
        .source_particle_epsilon_override_mask = std::span<const std::uint8_t>(src_mask.data(), src_mask.size()),
        .target_species_tag = {},
        .target_particle_epsilon_comoving = {},
        .target_particle_epsilon_override_mask = {},
        .species_policy = {},
    };
    for (const bool refresh : {true, false}) {
      gravity::TreePmProfileEvent tree_pm_profile;
      gravity::TreePmForceAccumulatorView acc = refresh ? accumulator : gravity::TreePmForceAccumulatorView{active, bx, by, bz};
      coordinator.solveActiveSetWithPmCadence(x, y, z, m, acc, options, refresh, &tree_pm_profile, &diagnostics,
                                              softening_view);
      // the runtime's cadence check right after the call
      const std::uint64_t expected_pm_solve_count = refresh ? 1U : 0U;
      if (diagnostics.pm_solve_count != expected_pm_solve_count ||
          diagnostics.pm_reuse_count != (options.short_range_only ? 0U : 1U - expected_pm_solve_count)) {
        std::fprintf(stderr, "TreePM solver PM solve/reuse outcome disagrees with the cadence directive\n");
        return 4;
      }
      if (diagnostics.residual_pair_evaluations == 0 || tree_pm_profile.tree_profile.actual_node_count == 0) {
        std::fprintf(stderr, "missing diagnostics\n");
        return 5;
      }
    }
    std::FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    for (const auto* v : {&ax, &ay, &az, &bx, &by, &bz}) std::fwrite(v->data(), 8, v->size(), o);
    std::fclose(o);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
  return 0;
}
