/* Test infrastructure (oracle): plain-C CPU restatement of the reference's
 * periodic TreePM force path (CHUI, src/gravity/). It is the checker for the
 * CUDA path in chui-dev_b200/csrc: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline arm may load it. It is never part of the product.
 *
 * Parity of this restatement is pinned against the reference itself
 * (oracle/_ref/treepm_ref, compiled from the reference's sources by
 * oracle/Makefile.ref) through the fixtures in tests/golden/.
 */
#ifndef CHUI_TREEPM_ORACLE_H
#define CHUI_TREEPM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double box[3];         /* periodic box lengths (Mpc/h comoving) */
  int64_t mesh[3];       /* PM mesh nx, ny, nz */
  double asmth_cells;    /* split scale r_s in mesh cells */
  double rcut_cells;     /* short-range cutoff in mesh cells */
  double theta;          /* opening angle */
  double G;              /* gravitational constant, code units */
  double epsilon;        /* uniform Plummer softening (comoving) */
  int64_t leaf_size;     /* max particles per leaf */
  int32_t scheme;        /* 0 CIC, 1 TSC */
  int32_t deconvolution; /* assignment-window deconvolution on/off */
  int32_t criterion;     /* 0 geometric, 1 COM distance, 2 relative force */
  int32_t quadrupole;    /* 1 quadrupole multipoles, 0 monopole */
  /* TreePmOptions acceptance policy (tree_pm_coupling.hpp:243-332) */
  int32_t policy;        /* 0 strict reference, 1 adaptive relative */
  int32_t estimator;     /* adaptive: 0 residual derivative, 1 relative monopole */
  int32_t cutoff_policy; /* adaptive: 0 contain node, 1 COM distance */
  int32_t reserved;
  double adaptive_angle; /* adaptive_maximum_opening_angle */
  double rel_tol;        /* tree relative_force_tolerance (alpha) */
  double accel_floor;    /* tree relative_force_acceleration_floor_code */
  int32_t group_walk;      /* TreePmOptions::group_walk_enabled (leaf grouping, blocks of 64) */
  int32_t gaussian_lookup; /* TreePmOptions::gaussian_pair_lookup_enabled (Hermite pair table) */
  int32_t boundary;        /* PmBoundaryCondition: 0 periodic, 1 isolated/open */
  int32_t reserved2;
} oracle_params;

typedef struct {
  uint64_t visited, accepted, opened, pairs, pruned, pair_skips, multipoles, leaves;
} oracle_counters;

typedef struct oracle_tree oracle_tree;

double oracle_mesh_spacing(const oracle_params *p);

/* PM (src/gravity/pm_solver.cpp) */
void oracle_pm_cells(int64_t n, const double *x, const double *y, const double *z,
                     const oracle_params *p, int64_t *base_cells /* 3*n: ix0,iy0,iz0 */);
void oracle_pm_density(int64_t n, const double *x, const double *y, const double *z,
                       const double *m, const oracle_params *p, double *rho /* nx*ny*nz */);
void oracle_pm_force_grids(int64_t n, const double *x, const double *y, const double *z,
                           const double *m, const oracle_params *p,
                           double *fx, double *fy, double *fz);
void oracle_pm_interpolate(const oracle_params *p, const double *fx, const double *fy,
                           const double *fz, int64_t nt, const double *tx, const double *ty,
                           const double *tz, double *ax, double *ay, double *az);

/* Tree (src/gravity/tree_pm_coupling.cpp:141-218, tree_ordering.cpp, tree_gravity.cpp) */
double oracle_unwrap_axis(int64_t n, const double *in, double box, int canonical, double *out);
oracle_tree *oracle_tree_build(int64_t n, const double *ux, const double *uy, const double *uz,
                               const double *m, const oracle_params *p, int *status);
int64_t oracle_tree_node_count(const oracle_tree *t);
uint32_t oracle_tree_max_depth(const oracle_tree *t);
/* field ids: 0 morton(u64,n) 1 sorted(u32,n) 2 cx 3 cy 4 cz 5 half 6 mass 7 comx 8 comy 9 comz
   10 qxx 11 qxy 12 qxz 13 qyy 14 qyz 15 qzz 16 trace (f64,nodes) 17 child_count(u32)
   18 child_index(u32, 8*nodes) 19 particle_begin(u32) 20 particle_count(u32) */
void oracle_tree_copy(const oracle_tree *t, int field, void *dst);
void oracle_tree_free(oracle_tree *t);

/* Full periodic TreePM solve (TreePmCoordinator::solveActiveSet, strict policy).
 * active may be NULL (all particles); outputs are in active-slot order; any
 * output pointer may be NULL. Returns 0 on success. */
int oracle_treepm_solve(int64_t n, const double *x, const double *y, const double *z,
                        const double *m, int64_t n_active, const uint32_t *active,
                        const oracle_params *p, double *ax, double *ay, double *az,
                        double *pm_ax, double *pm_ay, double *pm_az, double *tree_ax,
                        double *tree_ay, double *tree_az, double *nearest_r2,
                        oracle_counters *counters);

/* As oracle_treepm_solve, with the previous-step acceleration magnitudes of
 * the targets (active-slot order; NULL: no history), which the relative
 * criterion and the adaptive policy read. */
int oracle_treepm_solve2(int64_t n, const double *x, const double *y, const double *z,
                         const double *m, int64_t n_active, const uint32_t *active,
                         const oracle_params *p, const double *prev_acc, double *ax, double *ay,
                         double *az, double *pm_ax, double *pm_ay, double *pm_az, double *tree_ax,
                         double *tree_ay, double *tree_az, double *nearest_r2,
                         oracle_counters *counters);

/* KDK pieces (src/workflows/gravity_runtime.cpp:3043-3059,
 * src/workflows/reference_runtime_composition.cpp:76-107) */
void oracle_kick(int64_t n, double *vx, double *vy, double *vz, const double *ax,
                 const double *ay, const double *az, double kick, double drag);
void oracle_drift(int64_t n, double *x, double *y, double *z, const double *vx,
                  const double *vy, const double *vz, double drift, const double box[3]);

/* Scalar kernels, exposed for unit tests (tree_pm_split_kernel.hpp:90-131,204-228) */
double oracle_long_range_factor(double r, double rs);
double oracle_short_range_factor(double r, double rs);
double oracle_residual_inv_r3(double r2, double eps, double rs);

#ifdef __cplusplus
}
#endif

#endif
