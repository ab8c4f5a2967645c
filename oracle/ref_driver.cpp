// Test infrastructure (oracle): driver around the reference's own TreePM path.
//
// Reads a binary problem file (written by oracle/refio.py), runs
// cosmosim::gravity::TreePmCoordinator::solveActiveSet
// (include/cosmosim/gravity/tree_pm_coupling.hpp:575-584) with the same options
// a CHUI deck maps through GravityRuntimeImpl (src/workflows/gravity_runtime.cpp:469-608),
// and writes the accelerations plus the tree the coordinator built, so the
// repository's CPU restatement (oracle/treepm_oracle.c) and the CUDA path can be
// pinned against the reference itself. Optionally times repeated solves (the
// CPU-baseline arm of bench.py) and applies one KDK step with the reference's
// kick/drift formulas (src/workflows/gravity_runtime.cpp:3043-3059,
// src/workflows/reference_runtime_composition.cpp:49-107).
//
// Private coordinator state (the built tree, unwrapped coordinates, anchors) is
// read through the standard explicit-instantiation member-pointer idiom; the
// reference sources are compiled unmodified.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "cosmosim/core/cosmology.hpp"
#include "cosmosim/core/periodic_domain.hpp"
#include "cosmosim/core/time_integration.hpp"
#include "cosmosim/gravity/pm_solver.hpp"
#include "cosmosim/gravity/tree_pm_coupling.hpp"
#include "support/periodic_ewald_reference.hpp"

namespace cg = cosmosim::gravity;

// ---- member access idiom -------------------------------------------------
template <typename Tag, typename Tag::type Member>
struct Expose {
  friend typename Tag::type get(Tag) { return Member; }
};
struct TreeSolverTag {
  using type = cg::TreeGravitySolver cg::TreePmCoordinator::*;
  friend type get(TreeSolverTag);
};
struct TreeXTag {
  using type = std::vector<double> cg::TreePmCoordinator::*;
  friend type get(TreeXTag);
};
struct TreeYTag {
  using type = std::vector<double> cg::TreePmCoordinator::*;
  friend type get(TreeYTag);
};
struct TreeZTag {
  using type = std::vector<double> cg::TreePmCoordinator::*;
  friend type get(TreeZTag);
};
struct AnchorTag {
  using type = std::array<double, 3U> cg::TreePmCoordinator::*;
  friend type get(AnchorTag);
};
template struct Expose<TreeSolverTag, &cg::TreePmCoordinator::m_tree_solver>;
template struct Expose<TreeXTag, &cg::TreePmCoordinator::m_tree_source_x_comoving>;
template struct Expose<TreeYTag, &cg::TreePmCoordinator::m_tree_source_y_comoving>;
template struct Expose<TreeZTag, &cg::TreePmCoordinator::m_tree_source_z_comoving>;
template struct Expose<AnchorTag, &cg::TreePmCoordinator::m_tree_unwrap_anchor>;

// ---- binary io --------------------------------------------------------------
struct Reader {
  FILE* f;
  template <class T>
  T get() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("truncated input");
    return v;
  }
  template <class T>
  std::vector<T> vec(std::size_t n) {
    std::vector<T> v(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) throw std::runtime_error("truncated input");
    return v;
  }
};
struct Writer {
  FILE* f;
  template <class T>
  void put(T v) { std::fwrite(&v, sizeof(T), 1, f); }
  template <class T>
  void vec(const std::vector<T>& v) {
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
  }
};

struct Problem {
  std::int64_t n = 0;
  double box[3]{};
  std::int64_t mesh[3]{};
  double asmth = 1.25, rcut = 6.25, theta = 0.5, g = 1.0, eps = 0.0, scale_factor = 1.0;
  std::int64_t leaf = 16, scheme = 0, deconv = 0, criterion = 1, order = 2, n_active = 0;
  std::int64_t dump_tree = 1, dump_density = 0, kdk = 0, repeats = 0, ewald = 0;
  double drift = 0, kick1 = 0, kick2 = 0, drag1 = 1, drag2 = 1;
  std::vector<double> x, y, z, m, vx, vy, vz;
  std::vector<std::uint32_t> active;
  // optional trailing "CHUIADP1" block: acceptance policy and acceleration history
  std::int64_t policy = 0, estimator = 0, cutoff_policy = 0, has_prev = 0;
  double adaptive_angle = 0.25, rel_tol = 0.005, accel_floor = 1.0e-30;
  std::vector<double> prev;
  // optional "CHUIGRP1" block after it: group walk and Gaussian pair lookup
  std::int64_t group_walk = 0, gaussian_lookup = 0;
  // optional "CHUIISO1" block after it: PM boundary condition (1 isolated/open)
  std::int64_t boundary = 0;
  // optional "CHUISOF1" block: per-particle softening sidecars of a
  // TreeSofteningView (source epsilon + override mask, target epsilon + mask)
  std::vector<double> src_eps, tgt_eps;
  std::vector<std::uint8_t> src_mask, tgt_mask;
};

Problem readProblem(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) throw std::runtime_error("cannot open input");
  Reader r{f};
  char magic[8];
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "CHUIIN01", 8) != 0) {
    throw std::runtime_error("bad magic");
  }
  Problem p;
  p.n = r.get<std::int64_t>();
  for (double& b : p.box) b = r.get<double>();
  for (std::int64_t& m : p.mesh) m = r.get<std::int64_t>();
  p.asmth = r.get<double>();
  p.rcut = r.get<double>();
  p.theta = r.get<double>();
  p.g = r.get<double>();
  p.eps = r.get<double>();
  p.scale_factor = r.get<double>();
  p.leaf = r.get<std::int64_t>();
  p.scheme = r.get<std::int64_t>();
  p.deconv = r.get<std::int64_t>();
  p.criterion = r.get<std::int64_t>();
  p.order = r.get<std::int64_t>();
  p.n_active = r.get<std::int64_t>();
  p.dump_tree = r.get<std::int64_t>();
  p.dump_density = r.get<std::int64_t>();
  p.kdk = r.get<std::int64_t>();
  p.repeats = r.get<std::int64_t>();
  p.ewald = r.get<std::int64_t>();
  p.drift = r.get<double>();
  p.kick1 = r.get<double>();
  p.kick2 = r.get<double>();
  p.drag1 = r.get<double>();
  p.drag2 = r.get<double>();
  const auto n = static_cast<std::size_t>(p.n);
  p.x = r.vec<double>(n);
  p.y = r.vec<double>(n);
  p.z = r.vec<double>(n);
  p.m = r.vec<double>(n);
  p.vx = r.vec<double>(n);
  p.vy = r.vec<double>(n);
  p.vz = r.vec<double>(n);
  p.active = r.vec<std::uint32_t>(static_cast<std::size_t>(p.n_active));
  // tagged trailing blocks, in any order
  char tail[8];
  while (std::fread(tail, 1, 8, f) == 8) {
    if (std::memcmp(tail, "CHUIADP1", 8) == 0) {
      p.policy = r.get<std::int64_t>();
      p.estimator = r.get<std::int64_t>();
      p.cutoff_policy = r.get<std::int64_t>();
      p.has_prev = r.get<std::int64_t>();
      p.adaptive_angle = r.get<double>();
      p.rel_tol = r.get<double>();
      p.accel_floor = r.get<double>();
      if (p.has_prev) p.prev = r.vec<double>(static_cast<std::size_t>(p.n_active ? p.n_active : p.n));
    } else if (std::memcmp(tail, "CHUIGRP1", 8) == 0) {
      p.group_walk = r.get<std::int64_t>();
      p.gaussian_lookup = r.get<std::int64_t>();
    } else if (std::memcmp(tail, "CHUIISO1", 8) == 0) {
      p.boundary = r.get<std::int64_t>();
    } else if (std::memcmp(tail, "CHUISOF1", 8) == 0) {
      const auto ns = static_cast<std::size_t>(r.get<std::int64_t>());
      p.src_eps = r.vec<double>(ns);
      p.src_mask = r.vec<std::uint8_t>(ns);
      const auto nt = static_cast<std::size_t>(r.get<std::int64_t>());
      p.tgt_eps = r.vec<double>(nt);
      p.tgt_mask = r.vec<std::uint8_t>(nt);
    } else {
      throw std::runtime_error("bad trailing block");
    }
  }
  std::fclose(f);
  return p;
}

cg::TreePmOptions makeOptions(const Problem& p) {
  cg::TreePmOptions o;
  o.pm_options.box_size_x_mpc_comoving = p.box[0];
  o.pm_options.box_size_y_mpc_comoving = p.box[1];
  o.pm_options.box_size_z_mpc_comoving = p.box[2];
  o.pm_options.box_size_mpc_comoving = p.box[0];
  o.pm_options.scale_factor = p.scale_factor;
  o.pm_options.gravitational_constant_code = p.g;
  o.pm_options.assignment_scheme = p.scheme == 1 ? cg::PmAssignmentScheme::kTsc : cg::PmAssignmentScheme::kCic;
  o.pm_options.enable_window_deconvolution = p.deconv != 0;
  o.pm_options.boundary_condition =
      p.boundary == 1 ? cg::PmBoundaryCondition::kIsolatedOpen : cg::PmBoundaryCondition::kPeriodic;
  o.tree_options.gravitational_constant_code = p.g;
  o.tree_options.opening_theta = p.theta;
  o.tree_options.opening_criterion = p.criterion == 0 ? cg::TreeOpeningCriterion::kBarnesHutGeometric
      : (p.criterion == 2 ? cg::TreeOpeningCriterion::kRelativeForceError
                          : cg::TreeOpeningCriterion::kBarnesHutComDistance);
  o.tree_options.multipole_order = p.order == 0 ? cg::TreeMultipoleOrder::kMonopole : cg::TreeMultipoleOrder::kQuadrupole;
  o.tree_options.max_leaf_size = static_cast<std::size_t>(p.leaf);
  o.tree_options.softening.epsilon_comoving = p.eps;
  o.tree_options.relative_force_tolerance = p.rel_tol;
  o.tree_options.relative_force_acceleration_floor_code = p.accel_floor;
  o.acceptance_policy = p.policy == 1 ? cg::TreePmAcceptancePolicy::kAdaptiveRelative
                                      : cg::TreePmAcceptancePolicy::kStrictReference;
  o.adaptive_maximum_opening_angle = p.adaptive_angle;
  o.adaptive_error_estimator = p.estimator == 1 ? cg::TreePmAdaptiveErrorEstimator::kRelativeMonopole
                                                : cg::TreePmAdaptiveErrorEstimator::kResidualDerivative;
  o.cutoff_node_policy = p.cutoff_policy == 1 ? cg::TreePmCutoffNodePolicy::kComDistance
                                              : cg::TreePmCutoffNodePolicy::kContainNode;
  o.group_walk_enabled = p.group_walk != 0;
  o.gaussian_pair_lookup_enabled = p.gaussian_lookup != 0;
  o.split_policy = cg::makeTreePmSplitPolicyFromMeshSpacing(
      p.asmth, p.rcut,
      std::cbrt((p.box[0] / static_cast<double>(p.mesh[0])) * (p.box[1] / static_cast<double>(p.mesh[1])) *
                (p.box[2] / static_cast<double>(p.mesh[2]))));
  return o;
}

// --kdk-factors h omega_m omega_lambda omega_r omega_k time_si_per_code a dt:
// the reference's CosmologicalTimeline::prepareStep factors, one per line.
int kdkFactors(char** argv) {
  cosmosim::core::CosmologyBackgroundConfig cfg;
  cfg.hubble_param = std::stod(argv[2]);
  cfg.omega_matter = std::stod(argv[3]);
  cfg.omega_lambda = std::stod(argv[4]);
  cfg.omega_radiation = std::stod(argv[5]);
  cfg.omega_curvature = std::stod(argv[6]);
  const cosmosim::core::LambdaCdmBackground background(cfg);
  const cosmosim::core::CosmologicalTimeline timeline(&background, std::stod(argv[7]));
  const auto st = timeline.prepareStep(0.0, std::stod(argv[8]), std::stod(argv[9]));
  const double v[10] = {st.drift_factor_code, st.first_kick_factor_code, st.second_kick_factor_code,
                        st.first_hubble_drag_factor, st.second_hubble_drag_factor, st.first_source_kick_factor_code,
                        st.second_source_kick_factor_code, st.scale_factor_midpoint, st.scale_factor_end,
                        st.hubble_drag_factor};
  for (double x : v) std::printf("%.17g\n", x);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 10 && std::strcmp(argv[1], "--kdk-factors") == 0) {
    try {
      return kdkFactors(argv);
    } catch (const std::exception& e) {
      std::fprintf(stderr, "treepm_ref error: %s\n", e.what());
      return 1;
    }
  }
  if (argc != 3) {
    std::fprintf(stderr, "usage: treepm_ref <input.bin> <output.bin>\n");
    return 2;
  }
  try {
    Problem p = readProblem(argv[1]);
    const auto n = static_cast<std::size_t>(p.n);
    std::vector<std::uint32_t> active = p.active;
    if (active.empty()) {
      active.resize(n);
      std::iota(active.begin(), active.end(), 0U);
    }
    const std::size_t na = active.size();
    const cg::TreePmOptions options = makeOptions(p);
    cg::TreePmCoordinator coordinator(cg::PmGridShape{static_cast<std::size_t>(p.mesh[0]),
        static_cast<std::size_t>(p.mesh[1]), static_cast<std::size_t>(p.mesh[2])});

    std::vector<double> ax(na), ay(na), az(na), lx(na), ly(na), lz(na);
    std::vector<double> sx(n), sy(n), sz(n), nearest(n);
    cg::TreePmForceAccumulatorView acc{active, ax, ay, az};
    acc.long_range_accel_x_comoving = lx;
    acc.long_range_accel_y_comoving = ly;
    acc.long_range_accel_z_comoving = lz;
    acc.short_range_accel_x_comoving = sx;
    acc.short_range_accel_y_comoving = sy;
    acc.short_range_accel_z_comoving = sz;
    acc.short_range_nearest_pair_r2_comoving = nearest;
    if (p.has_prev) acc.previous_acceleration_magnitude_code = p.prev;

    cg::TreePmProfileEvent profile{};
    cg::TreePmDiagnostics diagnostics{};
    cg::TreeSofteningView softening{};
    softening.source_particle_epsilon_comoving = p.src_eps;
    softening.source_particle_epsilon_override_mask = p.src_mask;
    softening.target_particle_epsilon_comoving = p.tgt_eps;
    softening.target_particle_epsilon_override_mask = p.tgt_mask;
    const auto t0 = std::chrono::steady_clock::now();
    coordinator.solveActiveSet(p.x, p.y, p.z, p.m, acc, options, &profile, &diagnostics, softening);
    const double first_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    std::vector<double> times, rep_phases;  // rep_phases: {pm, tree build, traversal} ms per repeat
    for (std::int64_t rep = 0; rep < p.repeats; ++rep) {
      cg::TreePmProfileEvent prof{};
      const auto t1 = std::chrono::steady_clock::now();
      coordinator.solveActiveSet(p.x, p.y, p.z, p.m, acc, options, &prof, nullptr, softening);
      times.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count());
      rep_phases.push_back(prof.pm_profile.total_ms);
      rep_phases.push_back(prof.tree_profile.full_rebuild_ms);
      rep_phases.push_back(prof.tree_profile.traversal_ms);
    }

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) throw std::runtime_error("cannot open output");
    Writer w{f};
    std::fwrite("CHUIOUT1", 1, 8, f);
    w.put<std::int64_t>(p.n);
    w.put<std::int64_t>(static_cast<std::int64_t>(na));
    w.vec(ax); w.vec(ay); w.vec(az);
    w.vec(lx); w.vec(ly); w.vec(lz);
    w.vec(sx); w.vec(sy); w.vec(sz);
    w.vec(nearest);
    // timing: first solve wall, profile phases, repeats
    w.put<double>(first_ms);
    w.put<double>(profile.pm_profile.total_ms);
    w.put<double>(profile.tree_profile.full_rebuild_ms);
    w.put<double>(profile.tree_profile.traversal_ms);
    w.put<std::int64_t>(static_cast<std::int64_t>(times.size()));
    w.vec(times);
    const auto& lt = diagnostics.local_traversal;
    const std::uint64_t counters[8] = {lt.visited_nodes, lt.accepted_nodes, lt.opened_nodes,
        lt.direct_pair_evaluations, lt.cutoff_pruned_nodes, lt.cutoff_skipped_pairs,
        lt.accepted_internal_multipoles, lt.accepted_leaves};
    for (std::uint64_t c : counters) w.put<std::uint64_t>(c);

    // tree
    const cg::TreeGravitySolver& tree = coordinator.*get(TreeSolverTag());
    const auto& nodes = tree.nodes();
    const auto& ordering = tree.ordering();
    const std::size_t nn = p.dump_tree ? nodes.size() : 0U;
    w.put<std::int64_t>(static_cast<std::int64_t>(nn));
    if (p.dump_tree) {
      // isolated/open boundaries build the tree on the caller's coordinates
      const bool unwrapped = !(coordinator.*get(TreeXTag())).empty();
      w.vec(unwrapped ? coordinator.*get(TreeXTag()) : p.x);
      w.vec(unwrapped ? coordinator.*get(TreeYTag()) : p.y);
      w.vec(unwrapped ? coordinator.*get(TreeZTag()) : p.z);
      const auto anchors = coordinator.*get(AnchorTag());
      for (double a : anchors) w.put<double>(a);
      w.vec(ordering.morton_key);
      w.vec(ordering.sorted_particle_index);
      w.vec(nodes.center_x_comoving); w.vec(nodes.center_y_comoving); w.vec(nodes.center_z_comoving);
      w.vec(nodes.half_size_comoving); w.vec(nodes.mass_code);
      w.vec(nodes.com_x_comoving); w.vec(nodes.com_y_comoving); w.vec(nodes.com_z_comoving);
      w.vec(nodes.quad_xx); w.vec(nodes.quad_xy); w.vec(nodes.quad_xz);
      w.vec(nodes.quad_yy); w.vec(nodes.quad_yz); w.vec(nodes.quad_zz);
      w.vec(nodes.second_moment_trace);
      std::vector<std::uint32_t> child_count(nodes.child_count.begin(), nodes.child_count.end());
      w.vec(child_count);
      w.vec(nodes.child_index);
      w.vec(nodes.particle_begin);
      w.vec(nodes.particle_count);
    }

    // optional CIC/TSC density from the reference's PmSolver::assignDensity
    const std::size_t cells = static_cast<std::size_t>(p.mesh[0] * p.mesh[1] * p.mesh[2]);
    w.put<std::int64_t>(p.dump_density ? static_cast<std::int64_t>(cells) : 0);
    if (p.dump_density) {
      const cg::PmGridShape shape{static_cast<std::size_t>(p.mesh[0]), static_cast<std::size_t>(p.mesh[1]),
          static_cast<std::size_t>(p.mesh[2])};
      cg::PmGridStorage grid(shape);
      cg::PmSolver solver(shape);
      solver.assignDensity(grid, p.x, p.y, p.z, p.m, options.pm_options);
      const auto density = static_cast<const cg::PmGridStorage&>(grid).density();
      std::vector<double> d(density.begin(), density.end());
      w.vec(d);
    }

    // optional one KDK step: kick(a_old) -> drift+wrap -> solve -> kick(a_new)
    w.put<std::int64_t>(p.kdk);
    if (p.kdk) {
      if (na != n) throw std::runtime_error("KDK requires the full active set");
      std::vector<double> x = p.x, y = p.y, z = p.z, vx = p.vx, vy = p.vy, vz = p.vz;
      for (std::size_t k = 0; k < na; ++k) {
        const std::size_t i = active[k];
        vx[i] = p.drag1 * vx[i] + p.kick1 * ax[k];
        vy[i] = p.drag1 * vy[i] + p.kick1 * ay[k];
        vz[i] = p.drag1 * vz[i] + p.kick1 * az[k];
      }
      for (std::size_t i = 0; i < n; ++i) {
        x[i] += vx[i] * p.drift;
        y[i] += vy[i] * p.drift;
        z[i] += vz[i] * p.drift;
        x[i] = cosmosim::core::canonicalPeriodicPosition(x[i], p.box[0]);
        y[i] = cosmosim::core::canonicalPeriodicPosition(y[i], p.box[1]);
        z[i] = cosmosim::core::canonicalPeriodicPosition(z[i], p.box[2]);
      }
      std::vector<double> bx(na), by(na), bz(na);
      cg::TreePmForceAccumulatorView acc2{active, bx, by, bz};
      coordinator.solveActiveSet(x, y, z, p.m, acc2, options);
      for (std::size_t k = 0; k < na; ++k) {
        const std::size_t i = active[k];
        vx[i] = p.drag2 * vx[i] + p.kick2 * bx[k];
        vy[i] = p.drag2 * vy[i] + p.kick2 * by[k];
        vz[i] = p.drag2 * vz[i] + p.kick2 * bz[k];
      }
      w.vec(x); w.vec(y); w.vec(z); w.vec(vx); w.vec(vy); w.vec(vz);
      w.vec(bx); w.vec(by); w.vec(bz);
    }

    // optional FP64 Ewald accelerations for the first `ewald` active targets
    // (tests/support/periodic_ewald_reference.hpp:87-91), alpha = 2.5/L,
    // images +-3, modes +-10 (tests/validation/test_tree_pm_ewald_accuracy.cpp:695-706)
    w.put<std::int64_t>(p.ewald);
    if (p.ewald) {
      namespace ts = cosmosim::test_support;
      std::vector<ts::PeriodicEwaldSource> sources(n);
      for (std::size_t i = 0; i < n; ++i) sources[i] = {{p.x[i], p.y[i], p.z[i]}, p.m[i]};
      const std::size_t nt = std::min<std::size_t>(static_cast<std::size_t>(p.ewald), na);
      std::vector<ts::PeriodicEwaldTarget> targets(nt);
      for (std::size_t k = 0; k < nt; ++k) {
        const std::size_t i = active[k];
        targets[k] = {{p.x[i], p.y[i], p.z[i]}, i};
      }
      ts::PeriodicEwaldOptions eo;
      eo.gravitational_constant = p.g;
      eo.alpha_inverse_length = 2.5 / std::min({p.box[0], p.box[1], p.box[2]});
      eo.real_image_limits = {3, 3, 3};
      eo.reciprocal_mode_limits = {10, 10, 10};
      eo.plummer_softening_epsilon = p.eps;
      const auto e = ts::periodicEwaldAccelerations(sources, targets,
          ts::PeriodicEwaldBox{p.box[0], p.box[1], p.box[2]}, eo);
      std::vector<double> ex(nt), ey(nt), ez(nt);
      for (std::size_t k = 0; k < nt; ++k) { ex[k] = e[k].x; ey[k] = e[k].y; ez[k] = e[k].z; }
      w.vec(ex); w.vec(ey); w.vec(ez);
    }
    // per-repeat phase times (trailing block, read when present)
    std::fwrite("CHUIREP1", 1, 8, f);
    w.put<std::int64_t>(static_cast<std::int64_t>(times.size()));
    w.vec(rep_phases);
    std::fclose(f);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "treepm_ref error: %s\n", e.what());
    return 1;
  }
  return 0;
}
