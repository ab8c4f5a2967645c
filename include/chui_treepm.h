/* chui_treepm.h -- C-ABI of the B200 TreePM gravity solver.
 *
 * Drop-in boundary for CHUI's periodic TreePM force path. A C++ host binds it
 * behind the same interface as cosmosim::gravity::TreePmCoordinator
 * (include/cosmosim/gravity/tree_pm_coupling.hpp:527-814 in the reference);
 * chui-dev_b200/host/tree_pm_coordinator.hpp is that shim. Plain pointers and
 * sizes only; no C++ or torch types cross this boundary.
 *
 * Conventions
 *  - Every entry point returns 0 on success or a CHUI_TREEPM_E* code; the text
 *    of the last error is available from chui_treepm_last_error().
 *  - Pointers are host memory when `memory == CHUI_TREEPM_HOST`, device memory
 *    of the context's GPU when `memory == CHUI_TREEPM_DEVICE`.
 *  - `stream` is a cudaStream_t (NULL: the context's own stream). Calls with
 *    host memory return after the results are in the host buffers; calls with
 *    device memory return after the work is complete on `stream` as well (the
 *    solver reads a status word back to report kernel-side errors).
 *  - One context must not be used from two threads at once.
 */
#ifndef CHUI_TREEPM_H
#define CHUI_TREEPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHUI_TREEPM_ABI_VERSION 2

enum {
  CHUI_TREEPM_OK = 0,
  CHUI_TREEPM_EINVAL = 22,      /* std::invalid_argument in the reference */
  CHUI_TREEPM_ERANGE = 34,      /* std::out_of_range / std::overflow_error (index, depth, stack) */
  CHUI_TREEPM_ENOMEM = 12,      /* allocation failure (MemoryAdmissionError / bad_alloc) */
  CHUI_TREEPM_ESTATE = 71,      /* std::runtime_error: e.g. PM reuse without a valid field */
  CHUI_TREEPM_EDEVICE = 5,      /* CUDA / cuFFT failure */
  CHUI_TREEPM_ENOTSUP = 95      /* option outside the implemented periodic strict path */
};

enum { CHUI_TREEPM_HOST = 0, CHUI_TREEPM_DEVICE = 1 };
enum { CHUI_TREEPM_MIXED = 0, CHUI_TREEPM_FP64 = 1 };
enum { CHUI_TREEPM_CIC = 0, CHUI_TREEPM_TSC = 1 };
enum {
  CHUI_TREEPM_OPEN_GEOMETRIC = 0,     /* TreeOpeningCriterion::kBarnesHutGeometric */
  CHUI_TREEPM_OPEN_COM_DISTANCE = 1,  /* TreeOpeningCriterion::kBarnesHutComDistance */
  CHUI_TREEPM_OPEN_RELATIVE = 2       /* TreeOpeningCriterion::kRelativeForceError */
};
/* TreePmAcceptancePolicy, TreePmAdaptiveErrorEstimator, TreePmCutoffNodePolicy
 * (include/cosmosim/gravity/tree_pm_coupling.hpp:172-199) */
enum { CHUI_TREEPM_POLICY_STRICT = 0, CHUI_TREEPM_POLICY_ADAPTIVE = 1 };
enum { CHUI_TREEPM_ESTIMATOR_RESIDUAL_DERIVATIVE = 0, CHUI_TREEPM_ESTIMATOR_RELATIVE_MONOPOLE = 1 };
enum { CHUI_TREEPM_CUTOFF_CONTAIN_NODE = 0, CHUI_TREEPM_CUTOFF_COM_DISTANCE = 1 };
/* PmBoundaryCondition (include/cosmosim/gravity/pm_solver.hpp:78-81) */
enum { CHUI_TREEPM_BOUNDARY_PERIODIC = 0, CHUI_TREEPM_BOUNDARY_ISOLATED_OPEN = 1 };

/* Solver configuration: the `.param.txt` [numerics] treepm_* knobs
 * (include/cosmosim/core/config.hpp:776-821) after GravityRuntimeImpl's
 * mapping to TreePmOptions (src/workflows/gravity_runtime.cpp:469-608). */
typedef struct {
  int64_t pm_grid_nx, pm_grid_ny, pm_grid_nz; /* treepm_pm_grid_n{x,y,z} */
  double box_x, box_y, box_z;                 /* cosmology box_size_{x,y,z}_mpc_comoving */
  double asmth_cells;                         /* treepm_asmth_cells: r_s in mesh cells */
  double rcut_cells;                          /* treepm_rcut_cells: r_cut in mesh cells */
  double opening_theta;                       /* treepm_tree_opening_theta */
  int32_t opening_criterion;                  /* treepm_tree_opening_criterion */
  int32_t multipole_order;                    /* 0 monopole, 2 quadrupole (the reference default) */
  int64_t max_leaf_size;                      /* treepm_tree_max_leaf_size */
  int32_t assignment_scheme;                  /* treepm_assignment_scheme: CIC or TSC */
  int32_t window_deconvolution;               /* treepm_enable_window_deconvolution */
  double gravitational_constant;              /* G in code units (PM and tree share it) */
  double softening;                           /* Plummer epsilon, comoving (gravity_softening_kpc_comoving * 1e-3) */
  int32_t acceptance_policy;                  /* CHUI_TREEPM_POLICY_*: treepm_adaptive_acceptance_enabled */
  int32_t precision;                          /* CHUI_TREEPM_MIXED or CHUI_TREEPM_FP64 */
  int32_t device;                             /* CUDA device ordinal */
  int32_t diagnostics;                        /* 0 (default): the production walk (subtree blocks), no
                                                 counters; it still fills a requested nearest-pair lane.
                                                 1: the reference's per-node walk, traversal counters
                                                 equal to the reference's, nearest-pair r^2.
                                                 2: the production walk with its own counters (its
                                                 traversal's node visits and in-cutoff pairs) and the
                                                 nearest-pair lane */
  /* adaptive-relative policy (TreePmOptions, tree_pm_coupling.hpp:243-332) */
  int32_t adaptive_error_estimator;           /* CHUI_TREEPM_ESTIMATOR_*: treepm_adaptive_error_estimator */
  int32_t cutoff_node_policy;                 /* CHUI_TREEPM_CUTOFF_*: treepm_cutoff_node_policy */
  double adaptive_maximum_opening_angle;      /* (0, 1]; 0.25 */
  /* relative criteria (TreeGravityOptions, tree_gravity.hpp:30-43) */
  double relative_force_tolerance;            /* alpha; 0.005 */
  double relative_force_acceleration_floor;   /* code units; 1e-30 */
  /* TreePmOptions::group_walk_enabled: one conservative walk per leaf of targets
   * (effective with the adaptive policy, relative_monopole and the Gaussian pair
   * lookup, as in the reference; other cases use the per-target walk) */
  int32_t group_walk_enabled;
  /* TreePmOptions::gaussian_pair_lookup_enabled: direct pairs take the Gaussian
   * long-range coefficient from the reference's cubic Hermite table */
  int32_t gaussian_pair_lookup;
  /* PmSolveOptions::boundary_condition (mode.gravity_boundary): periodic, or
   * isolated/open -- zero-padded PM with the split Green function, the tree
   * on the caller's coordinates and no periodic images in the walk. The
   * adjoint entry points support periodic boundaries only. */
  int32_t boundary_condition;
  /* TreePmOptions::short_range_only (tree_pm_coupling.hpp:289-292): the
   * integrator's split operator -- only the short-range residual force, no PM
   * refresh, interpolation or reuse (long-range lanes are zero). */
  int32_t short_range_only;
} chui_treepm_config;

/* Counters named as TreePmTraversalCounters (tree_pm_coupling.hpp:39-87) plus
 * device timings of the last solve. */
typedef struct {
  uint64_t visited_nodes, accepted_nodes, opened_nodes, direct_pair_evaluations;
  uint64_t cutoff_pruned_nodes, cutoff_skipped_pairs, accepted_internal_multipoles, accepted_leaves;
  uint64_t node_count;
  uint32_t maximum_depth;
  uint32_t path_words;
  double pm_ms, tree_build_ms, walk_ms, total_ms;
  uint64_t kernel_launches;   /* this library's own kernels launched by the solve */
} chui_treepm_stats;

/* Sources: TreePmCoordinator::solveActiveSet's pos_{x,y,z}_comoving and
 * mass_code spans. mass may be NULL for a uniform mass population.
 * softening (optional): each source's resolved Plummer epsilon (comoving),
 * the materialized lane of TreeGravitySolver::resolvedSourceSoftening
 * (include/cosmosim/gravity/tree_softening.hpp:46-67, resolved from a
 * TreeSofteningView by resolveSourceSofteningEpsilon, :152-180); NULL: every
 * source takes config.softening. A pair uses max(epsilon_source,
 * epsilon_target) and an accepted node max(node maximum, epsilon_target)
 * (:229-233); nodes whose sources' epsilons differ are accepted only beyond
 * 2h + 2 max(node maximum, epsilon_target) (passesSofteningEnvelopeGuard). */
typedef struct {
  int64_t count;
  const double *x, *y, *z;
  const double *mass;
  double uniform_mass;
  const double *softening;
} chui_treepm_sources;

/* Accumulator: TreePmForceAccumulatorView (tree_pm_coupling.hpp:127-165).
 * active_index may be NULL for "all sources in row order". target_{x,y,z}
 * (optional) give explicit target positions, in which case active_index
 * entries may be 0xFFFFFFFF for targets without a source identity. Output
 * lanes other than accel_* are optional (NULL). long_range_* are in active-slot
 * order; short_range_* and nearest_pair_r2 are source-indexed like the
 * reference's tree-only lanes. */
typedef struct {
  int64_t active_count;
  const uint32_t *active_index;
  double *accel_x, *accel_y, *accel_z;
  const double *target_x, *target_y, *target_z;
  double *long_range_x, *long_range_y, *long_range_z;
  double *short_range_x, *short_range_y, *short_range_z;
  double *nearest_pair_r2;
  /* previous_acceleration_magnitude_code: per active slot |a_previous| for the
   * relative criteria, or NULL (no history). Non-finite entries mean "no
   * history" for that target: the COM-distance fallback. */
  const double *previous_acceleration_magnitude;
  /* target_softening (optional): per active slot, the target's resolved
   * epsilon (resolveTargetSofteningEpsilon, tree_softening.hpp:182-226);
   * NULL: a target that is a source takes its source epsilon, others
   * config.softening. Explicit targets with a source softening lane need it
   * (tree_pm_coupling.cpp:3962-3971). */
  const double *target_softening;
} chui_treepm_accumulator;

/* Defaults of TreePmOptions / TreeGravityOptions (tree_gravity.hpp:30-43,
 * tree_pm_coupling.hpp:243-332) for a 16^3 mesh on a unit box. */
int chui_treepm_config_default(chui_treepm_config *config);

/* TreePmCoordinator::TreePmCoordinator(PmGridShape) (tree_pm_coupling.hpp:545-551):
 * owns the PM mesh, FFT plans, tree and scratch on `config->device`. */
int chui_treepm_create(const chui_treepm_config *config, void **handle);

/* ~TreePmCoordinator(). NULL is accepted. */
void chui_treepm_destroy(void *handle);

/* Replace the options used by later solves (TreePmOptions passed per call in
 * the reference). The mesh shape is fixed at creation, as PmGridShape is. */
int chui_treepm_set_config(void *handle, const chui_treepm_config *config);

/* Text of the last error on this handle ("" when none). With a NULL handle:
 * the text of the last failed chui_treepm_create on the calling thread. */
const char *chui_treepm_last_error(const void *handle);

/* TreePmCoordinator::solveActiveSetWithPmCadence (tree_pm_coupling.hpp:563-573,
 * tree_pm_coupling.cpp:2282-3518): PM refresh (deposit, FFT, Green x split
 * filter, spectral gradient) when refresh_long_range_field != 0 (otherwise the
 * cached field must match, as :2483-2532 requires), PM interpolation, periodic
 * tree build, short-range residual walk, accumulation. stats may be NULL. */
int chui_treepm_solve(void *handle, const chui_treepm_sources *sources,
                      const chui_treepm_accumulator *accumulator, int refresh_long_range_field,
                      int memory, void *stream, chui_treepm_stats *stats);

/* One shard of a solve: the same solve restricted to the targets at visit
 * positions [visit_begin, visit_end). No counterpart in the reference, whose
 * ranks each own their particles (the MPI slab/LET path of
 * tree_pm_coupling.cpp); here every process holds all sources, builds the same
 * tree and PM field, and walks a slice of the common visit order, so the
 * shards' union is the full solve.
 *
 * The visit order is the order the walk takes targets in: tree order for a
 * full solve (no active_index, no explicit targets), else the active slots
 * sorted by tree position. Both ends must be multiples of 64 or the target
 * count, so that no group of targets (residual blocks of 64) is split. accel_* and long_range_* hold
 * visit_end - visit_begin entries, entry j being the target at visit position
 * visit_begin + j; short_range_* and nearest_pair_r2 stay source-indexed (only
 * the slice's entries are written). chui_treepm_visit_order gives the slots. */
int chui_treepm_solve_visit_range(void *handle, const chui_treepm_sources *sources,
                                  const chui_treepm_accumulator *accumulator, int refresh_long_range_field,
                                  int memory, void *stream, chui_treepm_stats *stats, int64_t visit_begin,
                                  int64_t visit_end);

/* Active slots (particle rows for a full solve) at visit positions
 * [begin, end) of the last successful solve, into slots (end - begin
 * entries, host or device memory). CHUI_TREEPM_ESTATE before any solve. */
int chui_treepm_visit_order(void *handle, int64_t begin, int64_t end, uint32_t *slots, int memory,
                            void *stream);

/* Device cycles the residual walk of the last successful solve spent on each
 * block of 32 visit positions: cost[k] covers positions begin + 32k ..
 * begin + 32k + 31 (SM clock cycles). Recorded by visit-range solves in FP64
 * and by the mixed walk's production form (diagnostics off, every source a
 * target, one mass for all sources); 0 elsewhere, where nothing was walked,
 * and for targets taken by the group walk. begin must be a multiple of 32;
 * cost holds ceil((end - begin) / 32) entries. No counterpart in the
 * reference; it lets a sharded solve cut the visit order into slices of equal
 * walk time. */
int chui_treepm_walk_cost(void *handle, int64_t begin, int64_t end, float *cost, int memory, void *stream);

/* PmSolver::assignDensity (pm_solver.hpp:469-482, pm_solver.cpp:3842-4565):
 * periodic CIC/TSC density (mass / cell volume) in compact nx*ny*nz row-major
 * order, written as FP64. */
int chui_pm_assign_density(void *handle, const chui_treepm_sources *sources, double *density,
                           int memory, void *stream);

/* Allocation-free form of chui_pm_assign_density. No counterpart in the
 * reference, which always allocates its mesh.
 *
 * For callers that must not allocate device memory during the call: code
 * running while another allocator (a framework's caching pool) holds the
 * device's free memory, where cudaMalloc would fail, and code that must not
 * pay cudaFree's device-wide synchronisation between steps. It takes no
 * handle (creating one allocates). The accumulation grid is a fixed scratch
 * array inside the library, CHUI_PM_STATIC_MAX_CELLS doubles (2 MiB) per
 * device, so meshes with nx*ny*nz above that fail with CHUI_TREEPM_ERANGE.
 * Positions and masses (mass may be NULL: uniform_mass) must be device memory
 * on config->device; density (nx*ny*nz doubles, row-major, mass / cell volume)
 * is host or device memory as density_memory says. The call zeroes the
 * scratch grid itself; nothing has to start at zero.
 *
 * The first call on a device also looks up the scratch address (a one-time
 * per-device set-up). All calls on a device in one process share the scratch
 * grid and overlapping calls would race, so each call holds a process-wide
 * lock and synchronises its stream (cudaStreamSynchronize) before returning.
 * Errors: chui_treepm_last_error(NULL) describes the last failure. */
#define CHUI_PM_STATIC_MAX_CELLS 262144
int chui_pm_assign_density_static(const chui_treepm_config *config, const chui_treepm_sources *sources,
                                  double *density, int density_memory, void *stream);

/* Base mesh cell per axis of each particle's assignment stencil after the
 * periodic wrap (makeAxisStencil / wrapIndex, pm_solver.cpp:103-116, :925-951):
 * cells[3*i + a]. The parity check on cell indices uses this. */
int chui_pm_cells(void *handle, const chui_treepm_sources *sources, int64_t *cells, int memory,
                  void *stream);

/* Tree parity dump after the last solve (TreeGravitySolver::nodes() and
 * ::ordering(), tree_gravity.hpp:195-198; unwrapped coordinates and anchors of
 * tree_pm_coupling.cpp:3183-3194). Host memory. Pass NULL for unwanted arrays.
 * node arrays hold node_count entries (child_index 8 per node). */
typedef struct {
  double *center_x, *center_y, *center_z, *half_size, *mass, *com_x, *com_y, *com_z;
  double *quad_xx, *quad_xy, *quad_xz, *quad_yy, *quad_yz, *quad_zz, *second_moment_trace;
  uint32_t *child_count, *child_index, *particle_begin, *particle_count;
} chui_treepm_tree_dump;
int chui_treepm_tree_node_count(const void *handle, int64_t *node_count);
int chui_treepm_dump_tree(void *handle, const chui_treepm_tree_dump *dump);

/* Which form the last tree build took (no counterpart in the reference; the
 * tree is the same either way): info[0] has bit a set when axis a's periodic
 * unwrap sorted the coordinates because its gap buckets could hide the
 * largest gap; info[1] is 1 when a leaf held more particles than the
 * in-place within-leaf ordering takes and the Morton order was sorted;
 * info[2] is 1 when the octant paths, first sorted by the levels the
 * context's previous tree needed, were sorted again by every level. */
int chui_treepm_tree_build_info(const void *handle, int32_t info[3]);

/* Particle-level parity dump after the last solve of n sources: unwrapped
 * tree-frame coordinates (m_tree_source_{x,y,z}_comoving), Morton keys in
 * sorted order (TreeMortonOrdering::morton_key), the final particle order
 * (TreeMortonOrdering::sorted_particle_index) and the three unwrap anchors
 * (m_tree_unwrap_anchor). Host memory; NULL skips an array. */
int chui_treepm_dump_particles(void *handle, int64_t n, double *ux, double *uy, double *uz,
                               uint64_t *morton_key, uint32_t *sorted_particle_index,
                               double anchors[3]);

/* KDK building blocks. Kick: u <- drag*u + kick*a (applyPeculiarVelocityKick,
 * src/workflows/gravity_runtime.cpp:3043-3059). Drift: x <- canonical(x + u*D)
 * (src/workflows/reference_runtime_composition.cpp:49-107 with
 * core::canonicalPeriodicPosition, include/cosmosim/core/periodic_domain.hpp:8-16),
 * using the context's box. */
int chui_treepm_kick(void *handle, int64_t n, double *vx, double *vy, double *vz,
                     const double *ax, const double *ay, const double *az, double kick_factor,
                     double drag_factor, int memory, void *stream);
int chui_treepm_drift(void *handle, int64_t n, double *x, double *y, double *z,
                      const double *vx, const double *vy, const double *vz, double drift_factor,
                      int memory, void *stream);

/* Non-cosmological KDK factors of CosmologicalTimeline::prepareStep without a
 * background (src/core/time_integration.cpp:429-441): D = dt, K1 = K2 = dt/2,
 * drag = 1. factors = {drift, kick1, kick2, drag1, drag2}. */
int chui_treepm_kdk_factors_static(double dt, double factors[5]);

/* Flat or curved Lambda-CDM background without radiation species
 * (CosmologyBackgroundConfig, include/cosmosim/core/cosmology.hpp:49-56):
 * E(a)^2 = Omega_r a^-4 + Omega_m a^-3 + Omega_k a^-2 + Omega_Lambda, the
 * densities summing to 1 within 1e-10; H0 = h x 100 km/s/Mpc. */
typedef struct {
  double hubble_param;
  double omega_matter, omega_lambda, omega_radiation, omega_curvature;
  double time_si_per_code; /* seconds per code time unit */
} chui_treepm_cosmology;

/* Cosmological KDK factors of one step of dt_code from scale factor a
 * (CosmologicalTimeline::prepareStep with a background,
 * src/core/time_integration.cpp:409-458; the factors of
 * computeComovingDriftFactor / KickFactor / SourceKickFactor /
 * HubbleDragFactor, :3530-3595, as 64-sample midpoint integrals over a; the
 * midpoint and end scale factors by advanceScaleFactorByCosmicTime,
 * :3469-3517). factors = {drift, kick1, kick2, drag1, drag2, source_kick1,
 * source_kick2, a_midpoint, a_end, drag (whole step)}: the kick and drift of
 * chui_treepm_kick / chui_treepm_drift take factors[0..4]. */
int chui_treepm_kdk_factors_lcdm(const chui_treepm_cosmology *cosmology, double scale_factor, double dt_code,
                                 double factors[10]);

/* Global FP64 momentum and energy checks over n particles: out = {sum m v_x,
 * sum m v_y, sum m v_z, sum m a_x, sum m a_y, sum m a_z, sum m |v|^2 / 2,
 * sum m}. mass may be NULL (uniform_mass); a_* may all be NULL. Reductions run
 * in FP64 on the device. */
int chui_treepm_momentum_energy(void *handle, int64_t n, const double *mass, double uniform_mass,
                                const double *vx, const double *vy, const double *vz, const double *ax,
                                const double *ay, const double *az, int memory, void *stream, double out[8]);

/* ---- Adjoint (no counterpart in the reference) ----------------------------
 * Reverse-mode building blocks for gradients of a loss on final positions or
 * density with respect to initial conditions. */

/* grad = J^T cot for the full TreePM acceleration a(x) of all sources (every
 * particle a target): PM part transposed exactly (interpolation, k-space
 * gradient operators, deposit); short-range part over the tree rebuilt for
 * these positions, as the pair-force Jacobian of every pair inside r_cut
 * (accepted strict multipoles are differentiated as the pairs they stand
 * for). cot and grad are source-indexed. The PM field cached for cadence
 * reuse afterwards holds these positions' field. stats may be NULL. */
int chui_treepm_force_vjp(void *handle, const chui_treepm_sources *sources, const double *cot_x,
                          const double *cot_y, const double *cot_z, double *grad_x, double *grad_y,
                          double *grad_z, int memory, void *stream, chui_treepm_stats *stats);

/* grad_j = sum_c rho_bar(c) d rho(c) / d x_j for the density of
 * chui_pm_assign_density (compact nx*ny*nz row-major cotangent). */
int chui_pm_density_vjp(void *handle, const chui_treepm_sources *sources, const double *rho_bar,
                        double *grad_x, double *grad_y, double *grad_z, int memory, void *stream);

/* Transpose of one KDK step (kick1/drag1, drift, kick2/drag2), in place on
 * device arrays, given g = chui_treepm_force_vjp at the step's end positions
 * for the pending force cotangent a_bar:
 *   x_bar += g; vh = drag2 v_bar + D x_bar; v_bar = drag1 vh;
 *   a_bar = kick1 vh + (first_step ? 0 : kick2 v_bar)   (cotangent at the start positions). */
int chui_treepm_kdk_adjoint(void *handle, int64_t n, const double *gx, const double *gy, const double *gz,
                            double *x_bar_x, double *x_bar_y, double *x_bar_z, double *v_bar_x,
                            double *v_bar_y, double *v_bar_z, double *a_bar_x, double *a_bar_y,
                            double *a_bar_z, double drift_factor, double kick1, double kick2, double drag1,
                            double drag2, int first_step, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CHUI_TREEPM_H */
