// Example host program: a CHUI-style caller driving the B200 solver through the
// C++ shim exactly as GravityRuntimeImpl drives TreePmCoordinator. Reads a
// binary problem (n, box, mesh, theta, leaf, eps, then x, y, z, m as doubles),
// solves all particles once with refresh and once reusing the PM field, checks
// that two visit-range shards reassemble the first solve, and writes the
// accelerations of both full solves as doubles.
//   g++ -std=c++20 -O2 shim_example.cpp -L../_build -lchui_treepm -o shim_example
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <numeric>
#include <utility>
#include <vector>

#include "tree_pm_coordinator.hpp"

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: shim_example <in.bin> <out.bin>\n");
    return 2;
  }
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::int64_t n = 0, mesh = 0, leaf = 0;
  double box = 0, theta = 0, eps = 0;
  bool ok = std::fread(&n, 8, 1, f) == 1 && std::fread(&box, 8, 1, f) == 1 && std::fread(&mesh, 8, 1, f) == 1 &&
            std::fread(&theta, 8, 1, f) == 1 && std::fread(&leaf, 8, 1, f) == 1 && std::fread(&eps, 8, 1, f) == 1;
  std::vector<double> x(n), y(n), z(n), m(n);
  for (auto* v : {&x, &y, &z, &m}) ok = ok && std::fread(v->data(), 8, n, f) == static_cast<std::size_t>(n);
  std::fclose(f);
  if (!ok) return 2;
  try {
    namespace cb = chui::b200;
    cb::TreePmCoordinator coordinator(cb::PmGridShape{static_cast<std::size_t>(mesh), static_cast<std::size_t>(mesh),
                                                      static_cast<std::size_t>(mesh)});
    cb::TreePmOptions options;
    options.pm_options.box_size_mpc_comoving = box;
    options.tree_options.opening_theta = theta;
    options.tree_options.max_leaf_size = static_cast<std::size_t>(leaf);
    options.tree_options.softening.epsilon_comoving = eps;
    std::vector<std::uint32_t> active(n);
    std::iota(active.begin(), active.end(), 0u);
    std::vector<double> ax(n), ay(n), az(n), bx(n), by(n), bz(n);
    cb::TreePmForceAccumulatorView acc{active, ax, ay, az};
    cb::TreePmProfileEvent profile;
    cb::TreePmDiagnostics diag;
    coordinator.solveActiveSet(x, y, z, m, acc, options, &profile, &diag);
    if (diag.pm_solve_count != 1 || diag.pm_reuse_count != 0 || diag.local_traversal.targets != static_cast<std::uint64_t>(n) ||
        diag.local_traversal.visited_nodes == 0 || profile.tree_profile.actual_node_count == 0) {
      std::fprintf(stderr, "unexpected diagnostics after a refresh solve\n");
      return 4;
    }
    // the default walk is the production one (subtree blocks): fewer node
    // visits than the per-node walk whose counters equal the reference's
    {
      cb::TreePmOptions per_node = options;
      per_node.walk_diagnostics = cb::WalkDiagnostics::kReferenceCounters;
      std::vector<double> px(n), py(n), pz(n);
      cb::TreePmForceAccumulatorView pacc{active, px, py, pz};
      cb::TreePmDiagnostics ref_diag;
      coordinator.solveActiveSet(x, y, z, m, pacc, per_node, nullptr, &ref_diag);
      // (pairs: the production set is a superset, up to FP32 rounding at r_cut)
      const auto& pt = diag.local_traversal;
      const auto& rt = ref_diag.local_traversal;
      if (!(pt.visited_nodes < rt.visited_nodes) ||
          static_cast<double>(pt.direct_pair_evaluations) < 0.999 * static_cast<double>(rt.direct_pair_evaluations)) {
        std::fprintf(stderr, "the default walk is not the production walk: visits %llu vs %llu, pairs %llu vs %llu\n",
                     static_cast<unsigned long long>(pt.visited_nodes), static_cast<unsigned long long>(rt.visited_nodes),
                     static_cast<unsigned long long>(pt.direct_pair_evaluations),
                     static_cast<unsigned long long>(rt.direct_pair_evaluations));
        return 7;
      }
      coordinator.solveActiveSet(x, y, z, m, acc, options, &profile, &diag);
    }
    cb::TreePmForceAccumulatorView acc2{active, bx, by, bz};
    coordinator.solveActiveSetWithPmCadence(x, y, z, m, acc2, options, false, nullptr, &diag);
    // the integrator's cadence check (gravity_runtime.cpp:2418-2424)
    if (diag.pm_solve_count != 0 || diag.pm_reuse_count != 1) {
      std::fprintf(stderr, "unexpected PM cadence diagnostics after a reuse solve\n");
      return 5;
    }
    // two shards of the visit order reassemble the full solve (PM field reused)
    {
      const std::size_t half = (static_cast<std::size_t>(n) / 2) / 64 * 64;
      double worst = 0.0, scale = 0.0;
      for (double v : ax) scale = std::max(scale, std::fabs(v));
      for (const auto& [b, e] : {std::pair<std::size_t, std::size_t>{0, half},
                                std::pair<std::size_t, std::size_t>{half, static_cast<std::size_t>(n)}}) {
        std::vector<double> sx(e - b), sy(e - b), sz(e - b);
        cb::TreePmForceAccumulatorView part{active, sx, sy, sz};
        // the same walk as the full solve (counted: diagnostics requested)
        cb::TreePmDiagnostics shard_diag;
        coordinator.solveVisitRange(x, y, z, m, part, options, false, b, e, nullptr, &shard_diag);
        const std::vector<std::uint32_t> slots = coordinator.visitOrder(b, e);
        for (std::size_t j = 0; j < slots.size(); ++j) worst = std::max(worst, std::fabs(sx[j] - ax[slots[j]]));
      }
      if (!(worst <= 1e-12 * scale)) {
        std::fprintf(stderr, "visit-range shards differ from the full solve by %g\n", worst);
        return 6;
      }
    }
    std::FILE* o = std::fopen(argv[2], "wb");
    for (auto* v : {&ax, &ay, &az, &bx, &by, &bz}) std::fwrite(v->data(), 8, n, o);
    std::fclose(o);
    // error path: a cutoff beyond half the box must raise std::invalid_argument
    cb::TreePmOptions bad = options;
    bad.split_policy.rcut_cells = 1.0e6;
    try {
      cb::TreePmCoordinator other(cb::PmGridShape{static_cast<std::size_t>(mesh), static_cast<std::size_t>(mesh),
                                                  static_cast<std::size_t>(mesh)});
      other.solveActiveSet(x, y, z, m, acc, bad);
      std::fprintf(stderr, "expected std::invalid_argument\n");
      return 3;
    } catch (const std::invalid_argument&) {
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "shim_example: %s\n", e.what());
    return 1;
  }
  return 0;
}
