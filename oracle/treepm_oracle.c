/* Test infrastructure (oracle): CPU restatement of the reference's periodic
 * TreePM path, see treepm_oracle.h. Each function names the reference lines it
 * restates. FP64 throughout, OpenMP over independent targets/lines only, so
 * results do not depend on the thread count.
 */
#include "treepm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft.h"

static const double k_pi = 3.141592653589793238462643383279502884;
static const double k_inv_sqrt_pi = 0.564189583547756286948079451560772586;
static const double k_inv_six_sqrt_pi = 0.094031597257959381158013241926795431;

double oracle_mesh_spacing(const oracle_params *p) {
  /* gravity_runtime.cpp:586-590: cbrt of the product of axis spacings */
  return cbrt((p->box[0] / (double)p->mesh[0]) * (p->box[1] / (double)p->mesh[1]) *
              (p->box[2] / (double)p->mesh[2]));
}

/* ---------------------------------------------------------------- split law */

/* tree_pm_split_kernel.hpp:66-76 */
double oracle_short_range_factor(double r, double rs) {
  if (r <= 0.0) return 1.0;
  const double q = (0.5 * r) / rs;
  if (isinf(q)) return 0.0;
  return erfc(q) + 2.0 * k_inv_sqrt_pi * q * exp(-q * q);
}

/* tree_pm_split_kernel.hpp:90-107 */
double oracle_long_range_factor(double r, double rs) {
  if (r <= 0.0) return 0.0;
  const double q = (0.5 * r) / rs;
  if (isinf(q)) return 1.0;
  if (q < 0.125) {
    const double t = q * q;
    const double h = 4.0 * k_inv_sqrt_pi *
                     (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
                      t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
    return q * q * q * h;
  }
  return erf(q) - 2.0 * k_inv_sqrt_pi * q * exp(-q * q);
}

/* tree_pm_split_kernel.hpp:111-116 */
static double coefficient_series(double t) {
  const double c = 2.25675833419102514779231780624309034;
  return c * (1.0 / 3.0 + t * (-1.0 / 5.0 + t * (1.0 / 14.0 + t * (-1.0 / 54.0 +
              t * (1.0 / 264.0 + t * (-1.0 / 1560.0 + t * (1.0 / 10800.0 - t / 85680.0)))))));
}

/* tree_pm_split_kernel.hpp:118-128 */
static double long_range_inv_r3(double r, double rs) {
  const double q = (0.5 * r) / rs;
  if (q < 0.125) return ((0.125 * coefficient_series(q * q) / rs) / rs) / rs;
  return ((oracle_long_range_factor(r, rs) / r) / r) / r;
}

/* tree_softening.hpp:243-253 */
static double softened_inv_r3(double r2, double eps) {
  const double s2 = r2 + eps * eps;
  if (s2 <= 0.0) return 0.0;
  return 1.0 / (s2 * sqrt(s2));
}

/* tree_pm_split_kernel.hpp:204-228 */
double oracle_residual_inv_r3(double r2, double eps, double rs) {
  if (r2 <= 0.0) {
    if (eps == 0.0) return softened_inv_r3(r2, eps);
    if (eps <= rs) {
      const double ratio = eps / rs;
      const double c = 1.0 - k_inv_six_sqrt_pi * ratio * ratio * ratio;
      return ((c / eps) / eps) / eps;
    }
    const double ratio = rs / eps;
    const double c = ratio * ratio * ratio - k_inv_six_sqrt_pi;
    return ((c / rs) / rs) / rs;
  }
  return softened_inv_r3(r2, eps) - long_range_inv_r3(sqrt(r2), rs);
}

/* ---------------------------------------------------------------------- PM */

/* pm_solver.cpp:112-115 */
static double wrap_position(double x, double box) {
  const double w = fmod(x, box);
  return w < 0.0 ? w + box : w;
}

/* pm_solver.cpp:103-110 */
static int64_t wrap_index(int64_t i, int64_t n) {
  int64_t w = i % n;
  if (w < 0) w += n;
  return w;
}

typedef struct {
  int64_t off[3];
  double w[3];
  int count;
} stencil1d;

/* pm_solver.cpp:925-951 (makeAxisStencil) */
static stencil1d make_stencil(double gp, int scheme) {
  stencil1d s;
  if (scheme == 0) {
    const double base = floor(gp);
    const int64_t i0 = (int64_t)base;
    const double t = gp - base;
    s.off[0] = i0;
    s.off[1] = i0 + 1;
    s.off[2] = 0;
    s.w[0] = 1.0 - t;
    s.w[1] = t;
    s.w[2] = 0.0;
    s.count = 2;
  } else {
    const double center = floor(gp + 0.5);
    const int64_t ic = (int64_t)center;
    const double d = gp - center;
    s.off[0] = ic - 1;
    s.off[1] = ic;
    s.off[2] = ic + 1;
    s.w[0] = 0.5 * ((0.5 - d) * (0.5 - d));
    s.w[1] = 0.75 - d * d;
    s.w[2] = 0.5 * ((0.5 + d) * (0.5 + d));
    s.count = 3;
  }
  return s;
}

void oracle_pm_cells(int64_t n, const double *x, const double *y, const double *z,
                     const oracle_params *p, int64_t *base) {
  const double inv[3] = {(double)p->mesh[0] / p->box[0], (double)p->mesh[1] / p->box[1],
                         (double)p->mesh[2] / p->box[2]};
  for (int64_t i = 0; i < n; ++i) {
    const double pos[3] = {x[i], y[i], z[i]};
    for (int a = 0; a < 3; ++a) {
      const stencil1d s = make_stencil(wrap_position(pos[a], p->box[a]) * inv[a], p->scheme);
      base[3 * i + a] = wrap_index(s.off[0], p->mesh[a]);
    }
  }
}

/* assignDensityImpl serial periodic branch, pm_solver.cpp:4015-4057, then
 * the /cell_volume normalization :4544-4554. Compact (nx, ny, nz) layout. */
/* positionInsideOpenDomain, pm_solver.cpp:117-119 */
static int inside_open(double v, double box) { return v >= 0.0 && v < box; }

void oracle_pm_density(int64_t n, const double *x, const double *y, const double *z,
                       const double *m, const oracle_params *p, double *rho) {
  const int64_t nx = p->mesh[0], ny = p->mesh[1], nz = p->mesh[2];
  const size_t cells = (size_t)nx * ny * nz;
  memset(rho, 0, sizeof(double) * cells);
  const double inv_dx = (double)nx / p->box[0];
  const double inv_dy = (double)ny / p->box[1];
  const double inv_dz = (double)nz / p->box[2];
  const int per = p->boundary == 0;
  for (int64_t i = 0; i < n; ++i) {
    /* isolated/open: particles outside [0, L) and stencil cells outside the mesh are skipped (:4016-4049) */
    if (!per && !(inside_open(x[i], p->box[0]) && inside_open(y[i], p->box[1]) && inside_open(z[i], p->box[2])))
      continue;
    const stencil1d sx = make_stencil((per ? wrap_position(x[i], p->box[0]) : x[i]) * inv_dx, p->scheme);
    const stencil1d sy = make_stencil((per ? wrap_position(y[i], p->box[1]) : y[i]) * inv_dy, p->scheme);
    const stencil1d sz = make_stencil((per ? wrap_position(z[i], p->box[2]) : z[i]) * inv_dz, p->scheme);
    for (int a = 0; a < sx.count; ++a) {
      if (!per && (sx.off[a] < 0 || sx.off[a] >= nx)) continue;
      const int64_t ix = per ? wrap_index(sx.off[a], nx) : sx.off[a];
      for (int b = 0; b < sy.count; ++b) {
        if (!per && (sy.off[b] < 0 || sy.off[b] >= ny)) continue;
        const int64_t iy = per ? wrap_index(sy.off[b], ny) : sy.off[b];
        for (int c = 0; c < sz.count; ++c) {
          if (!per && (sz.off[c] < 0 || sz.off[c] >= nz)) continue;
          const int64_t iz = per ? wrap_index(sz.off[c], nz) : sz.off[c];
          const double w = sx.w[a] * sy.w[b] * sz.w[c];
          rho[((size_t)ix * ny + iy) * nz + iz] += m[i] * w;
        }
      }
    }
  }
  const double cell_volume = (p->box[0] * p->box[1] * p->box[2]) / (double)cells;
  for (size_t c = 0; c < cells; ++c) rho[c] /= cell_volume;
}

static double sinc(double v) {
  /* pm_solver.cpp:121-126 */
  if (fabs(v) < 1.0e-12) return 1.0;
  return sin(v) / v;
}

/* solvePoissonPeriodicImpl spectral branch, pm_solver.cpp:4676-4707 (mean
 * subtraction), :4712 (r2c), applyDerivedPoissonOperator :2557-2656 with the
 * axis metadata of ensureSpectralAxisMetadata :2398-2466, fillGradientSpectrum
 * :2658-2706 and the normalized c2r per axis :4865-4924. */
/* solvePoissonIsolatedOpen single-rank path, pm_solver.cpp:4942-5337: zero-padded
 * (2n)^3 complex convolution of the density with the split Green function
 * -erf(r / 2 r_s) / r (r = 0: -1 / (sqrt(pi) r_s)), potential = G dV conv / pad_total,
 * force = -gradient by central differences, one-sided second order at the faces. */
static void pm_force_grids_isolated(int64_t n, const double *x, const double *y, const double *z,
                                    const double *m, const oracle_params *p, double *fx, double *fy,
                                    double *fz) {
  const int64_t nx = p->mesh[0], ny = p->mesh[1], nz = p->mesh[2];
  const size_t cells = (size_t)nx * ny * nz;
  const int64_t px = 2 * nx, py = 2 * ny, pz = 2 * nz;
  const size_t pad_total = (size_t)px * py * pz;
  double *rho = (double *)malloc(sizeof(double) * cells);
  oracle_pm_density(n, x, y, z, m, p, rho);
  double *rk = (double *)calloc(2 * pad_total, sizeof(double));
  for (int64_t ix = 0; ix < nx; ++ix)
    for (int64_t iy = 0; iy < ny; ++iy)
      for (int64_t iz = 0; iz < nz; ++iz) rk[2 * (((size_t)ix * py + iy) * pz + iz)] = rho[((size_t)ix * ny + iy) * nz + iz];
  free(rho);
  oracle_fft3d_c2c(rk, (int)px, (int)py, (int)pz, -1);
  const double dx = p->box[0] / (double)nx, dy = p->box[1] / (double)ny, dz = p->box[2] / (double)nz;
  const double rs = p->asmth_cells * oracle_mesh_spacing(p);
  double *kk = (double *)calloc(2 * pad_total, sizeof(double));
  for (int64_t ix = 0; ix < px; ++ix) {
    const double rx = (double)(ix <= nx ? ix : ix - px) * dx;
    for (int64_t iy = 0; iy < py; ++iy) {
      const double ry = (double)(iy <= ny ? iy : iy - py) * dy;
      for (int64_t iz = 0; iz < pz; ++iz) {
        const double rz = (double)(iz <= nz ? iz : iz - pz) * dz;
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        double kernel;
        if (r > 0.0) {
          kernel = rs > 0.0 ? -erf(0.5 * r / rs) / r : -1.0 / r;
        } else {
          kernel = -1.0 / (sqrt(acos(-1.0)) * rs);
        }
        kk[2 * (((size_t)ix * py + iy) * pz + iz)] = kernel;
      }
    }
  }
  oracle_fft3d_c2c(kk, (int)px, (int)py, (int)pz, -1);
  for (size_t i = 0; i < pad_total; ++i) {
    const double ar = rk[2 * i], ai = rk[2 * i + 1], br = kk[2 * i], bi = kk[2 * i + 1];
    rk[2 * i] = ar * br - ai * bi;
    rk[2 * i + 1] = ar * bi + ai * br;
  }
  free(kk);
  oracle_fft3d_c2c(rk, (int)px, (int)py, (int)pz, +1);
  const double prefactor = p->G * (dx * dy * dz);
  double *phi = (double *)malloc(sizeof(double) * cells);
  for (int64_t ix = 0; ix < nx; ++ix)
    for (int64_t iy = 0; iy < ny; ++iy)
      for (int64_t iz = 0; iz < nz; ++iz) {
        double value = rk[2 * (((size_t)ix * py + iy) * pz + iz)];
        value /= (double)pad_total;
        phi[((size_t)ix * ny + iy) * nz + iz] = prefactor * value;
      }
  free(rk);
#define PHI(a, b, c) phi[((size_t)(a) * ny + (b)) * nz + (c)]
  for (int64_t ix = 0; ix < nx; ++ix)
    for (int64_t iy = 0; iy < ny; ++iy)
      for (int64_t iz = 0; iz < nz; ++iz) {
        double gx, gy, gz;
        if (ix == 0) gx = (-3.0 * PHI(0, iy, iz) + 4.0 * PHI(1, iy, iz) - PHI(2, iy, iz)) / (2.0 * dx);
        else if (ix + 1 == nx) gx = (3.0 * PHI(nx - 1, iy, iz) - 4.0 * PHI(nx - 2, iy, iz) + PHI(nx - 3, iy, iz)) / (2.0 * dx);
        else gx = (PHI(ix + 1, iy, iz) - PHI(ix - 1, iy, iz)) / (2.0 * dx);
        if (iy == 0) gy = (-3.0 * PHI(ix, 0, iz) + 4.0 * PHI(ix, 1, iz) - PHI(ix, 2, iz)) / (2.0 * dy);
        else if (iy + 1 == ny) gy = (3.0 * PHI(ix, ny - 1, iz) - 4.0 * PHI(ix, ny - 2, iz) + PHI(ix, ny - 3, iz)) / (2.0 * dy);
        else gy = (PHI(ix, iy + 1, iz) - PHI(ix, iy - 1, iz)) / (2.0 * dy);
        if (iz == 0) gz = (-3.0 * PHI(ix, iy, 0) + 4.0 * PHI(ix, iy, 1) - PHI(ix, iy, 2)) / (2.0 * dz);
        else if (iz + 1 == nz) gz = (3.0 * PHI(ix, iy, nz - 1) - 4.0 * PHI(ix, iy, nz - 2) + PHI(ix, iy, nz - 3)) / (2.0 * dz);
        else gz = (PHI(ix, iy, iz + 1) - PHI(ix, iy, iz - 1)) / (2.0 * dz);
        const size_t c = ((size_t)ix * ny + iy) * nz + iz;
        fx[c] = -gx;
        fy[c] = -gy;
        fz[c] = -gz;
      }
#undef PHI
  free(phi);
}

void oracle_pm_force_grids(int64_t n, const double *x, const double *y, const double *z,
                           const double *m, const oracle_params *p,
                           double *fx, double *fy, double *fz) {
  if (p->boundary == 1) {
    pm_force_grids_isolated(n, x, y, z, m, p, fx, fy, fz);
    return;
  }
  const int64_t nx = p->mesh[0], ny = p->mesh[1], nz = p->mesh[2];
  const size_t cells = (size_t)nx * ny * nz;
  const int64_t nzc = nz / 2 + 1;
  const size_t ccells = (size_t)nx * ny * nzc;
  double *rho = (double *)malloc(sizeof(double) * cells);
  oracle_pm_density(n, x, y, z, m, p, rho);
  double sum = 0.0;
  for (size_t c = 0; c < cells; ++c) sum += rho[c];
  const double mean = sum / (double)cells;
  for (size_t c = 0; c < cells; ++c) rho[c] -= mean;
  double *phik = (double *)malloc(sizeof(double) * 2 * ccells);
  oracle_fft3d_r2c(rho, (size_t)nz, phik, (int)nx, (int)ny, (int)nz);
  free(rho);

  const double rs = p->asmth_cells * oracle_mesh_spacing(p);
  const double dk[3] = {2.0 * k_pi / p->box[0], 2.0 * k_pi / p->box[1], 2.0 * k_pi / p->box[2]};
  const int expo = p->scheme == 0 ? 2 : 3;
  double *kx = (double *)malloc(sizeof(double) * nx), *wx = (double *)malloc(sizeof(double) * nx);
  double *ky = (double *)malloc(sizeof(double) * ny), *wy = (double *)malloc(sizeof(double) * ny);
  double *kz = (double *)malloc(sizeof(double) * nzc), *wz = (double *)malloc(sizeof(double) * nzc);
  for (int64_t i = 0; i < nx; ++i) {
    const int64_t mode = i <= nx / 2 ? i : i - nx;
    kx[i] = dk[0] * (double)mode;
    wx[i] = p->deconvolution ? pow(sinc(0.5 * kx[i] * p->box[0] / (double)nx), (double)expo) : 1.0;
  }
  for (int64_t i = 0; i < ny; ++i) {
    const int64_t mode = i <= ny / 2 ? i : i - ny;
    ky[i] = dk[1] * (double)mode;
    wy[i] = p->deconvolution ? pow(sinc(0.5 * ky[i] * p->box[1] / (double)ny), (double)expo) : 1.0;
  }
  for (int64_t i = 0; i < nzc; ++i) {
    kz[i] = dk[2] * (double)i;
    wz[i] = p->deconvolution ? pow(sinc(0.5 * kz[i] * p->box[2] / (double)nz), (double)expo) : 1.0;
  }
  const double prefactor = -4.0 * k_pi * p->G;
  for (int64_t ix = 0; ix < nx; ++ix) {
    for (int64_t iy = 0; iy < ny; ++iy) {
      for (int64_t iz = 0; iz < nzc; ++iz) {
        const size_t idx = ((size_t)ix * ny + iy) * nzc + iz;
        const double k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
        if (k2 == 0.0) {
          phik[2 * idx] = 0.0;
          phik[2 * idx + 1] = 0.0;
          continue;
        }
        double window_correction = 1.0;
        if (p->deconvolution) {
          const double tw = wx[ix] * wy[iy] * wz[iz];
          const double w2 = tw * tw;
          window_correction = 1.0 / (w2 > 1.0e-12 ? w2 : 1.0e-12);
        }
        const double prod = sqrt(k2) * rs;
        const double split = exp(-(prod * prod));
        const double op = prefactor * window_correction * split * 1.0 / k2;
        phik[2 * idx] *= op;
        phik[2 * idx + 1] *= op;
      }
    }
  }
  double *gk = (double *)malloc(sizeof(double) * 2 * ccells);
  double *outs[3] = {fx, fy, fz};
  const double norm = 1.0 / (double)cells;
  for (int axis = 0; axis < 3; ++axis) {
    for (int64_t ix = 0; ix < nx; ++ix) {
      for (int64_t iy = 0; iy < ny; ++iy) {
        for (int64_t iz = 0; iz < nzc; ++iz) {
          const size_t idx = ((size_t)ix * ny + iy) * nzc + iz;
          double g;
          if (axis == 0) g = (nx % 2 == 0 && ix == nx / 2) ? 0.0 : kx[ix];
          else if (axis == 1) g = (ny % 2 == 0 && iy == ny / 2) ? 0.0 : ky[iy];
          else g = (nz % 2 == 0 && iz == nz / 2) ? 0.0 : kz[iz];
          /* (0, -g) * (re, im) = (g*im, -g*re) */
          const double re = phik[2 * idx], im = phik[2 * idx + 1];
          gk[2 * idx] = -(-g) * im;
          gk[2 * idx + 1] = (-g) * re;
        }
      }
    }
    oracle_fft3d_c2r(gk, outs[axis], (size_t)nz, (int)nx, (int)ny, (int)nz);
    for (size_t c = 0; c < cells; ++c) outs[axis][c] *= norm;
  }
  free(gk);
  free(phik);
  free(kx); free(ky); free(kz); free(wx); free(wy); free(wz);
}

/* interpolateForcesImpl serial periodic branch, pm_solver.cpp:5898-5953 */
void oracle_pm_interpolate(const oracle_params *p, const double *fx, const double *fy,
                           const double *fz, int64_t nt, const double *tx, const double *ty,
                           const double *tz, double *ax, double *ay, double *az) {
  const int64_t nx = p->mesh[0], ny = p->mesh[1], nz = p->mesh[2];
  const double inv_dx = (double)nx / p->box[0];
  const double inv_dy = (double)ny / p->box[1];
  const double inv_dz = (double)nz / p->box[2];
  const int per = p->boundary == 0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nt; ++i) {
    if (!per && !(inside_open(tx[i], p->box[0]) && inside_open(ty[i], p->box[1]) && inside_open(tz[i], p->box[2]))) {
      ax[i] = ay[i] = az[i] = 0.0; /* :5905-5913 */
      continue;
    }
    const stencil1d sx = make_stencil((per ? wrap_position(tx[i], p->box[0]) : tx[i]) * inv_dx, p->scheme);
    const stencil1d sy = make_stencil((per ? wrap_position(ty[i], p->box[1]) : ty[i]) * inv_dy, p->scheme);
    const stencil1d sz = make_stencil((per ? wrap_position(tz[i], p->box[2]) : tz[i]) * inv_dz, p->scheme);
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int a = 0; a < sx.count; ++a) {
      if (!per && (sx.off[a] < 0 || sx.off[a] >= nx)) continue;
      const int64_t ix = per ? wrap_index(sx.off[a], nx) : sx.off[a];
      for (int b = 0; b < sy.count; ++b) {
        if (!per && (sy.off[b] < 0 || sy.off[b] >= ny)) continue;
        const int64_t iy = per ? wrap_index(sy.off[b], ny) : sy.off[b];
        for (int c = 0; c < sz.count; ++c) {
          if (!per && (sz.off[c] < 0 || sz.off[c] >= nz)) continue;
          const int64_t iz = per ? wrap_index(sz.off[c], nz) : sz.off[c];
          const double w = sx.w[a] * sy.w[b] * sz.w[c];
          const size_t idx = ((size_t)ix * ny + iy) * nz + iz;
          gx += w * fx[idx];
          gy += w * fy[idx];
          gz += w * fz[idx];
        }
      }
    }
    ax[i] = gx;
    ay[i] = gy;
    az[i] = gz;
  }
}

/* ------------------------------------------------------------- unwrapping */

static int cmp_u64(const void *a, const void *b) {
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* unwrapPeriodicAxis, tree_pm_coupling.cpp:141-218 (the IEEE-bit radix sort of
 * :94-135 is a sort of non-negative doubles; qsort of the same bits yields the
 * same order). */
double oracle_unwrap_axis(int64_t n, const double *in, double box, int canonical, double *out) {
  if (n == 0) return 0.0;
  uint64_t *bits = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    double v = canonical ? in[i] : in[i] - box * floor(in[i] / box);
    if (v >= box) v = 0.0;
    else if (v < 0.0) v += box;
    if (v == 0.0) v = 0.0;
    out[i] = v;
    memcpy(&bits[i], &v, sizeof(double));
  }
  qsort(bits, (size_t)n, sizeof(uint64_t), cmp_u64);
  double anchor;
  memcpy(&anchor, &bits[0], sizeof(double));
  if (n > 1) {
    double largest = -1.0, best = anchor;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t nxt = (i + 1) % n;
      double cur, cand;
      memcpy(&cur, &bits[i], sizeof(double));
      memcpy(&cand, &bits[nxt], sizeof(double));
      const double next_value = nxt == 0 ? cand + box : cand;
      const double gap = next_value - cur;
      if (gap > largest || (gap == largest && cand < best)) {
        largest = gap;
        best = cand;
      }
    }
    anchor = best;
  }
  for (int64_t i = 0; i < n; ++i) {
    if (out[i] < anchor) out[i] += box;
  }
  free(bits);
  return anchor;
}

/* ------------------------------------------------------------------ tree */

struct oracle_tree {
  int64_t n, n_nodes, cap;
  uint32_t max_depth;
  uint64_t *morton;
  uint32_t *sorted;
  uint32_t *scratch;
  double *cx, *cy, *cz, *half, *mass, *comx, *comy, *comz;
  double *q[6], *trace, *smin, *smax;
  uint32_t *child_count, *child_index, *pbegin, *pcount;
  int status;
};

/* tree_ordering.cpp:73-85 */
static uint64_t expand_bits21(uint32_t v) {
  uint64_t x = v & 0x1FFFFFu;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

static void tree_reserve(oracle_tree *t, int64_t need) {
  if (need <= t->cap) return;
  int64_t cap = t->cap ? t->cap : 64;
  while (cap < need) cap *= 2;
  double **dl[] = {&t->cx, &t->cy, &t->cz, &t->half, &t->mass, &t->comx, &t->comy, &t->comz,
                   &t->q[0], &t->q[1], &t->q[2], &t->q[3], &t->q[4], &t->q[5], &t->trace,
                   &t->smin, &t->smax};
  for (size_t k = 0; k < sizeof(dl) / sizeof(dl[0]); ++k)
    *dl[k] = (double *)realloc(*dl[k], sizeof(double) * (size_t)cap);
  t->child_count = (uint32_t *)realloc(t->child_count, sizeof(uint32_t) * (size_t)cap);
  t->child_index = (uint32_t *)realloc(t->child_index, sizeof(uint32_t) * 8 * (size_t)cap);
  t->pbegin = (uint32_t *)realloc(t->pbegin, sizeof(uint32_t) * (size_t)cap);
  t->pcount = (uint32_t *)realloc(t->pcount, sizeof(uint32_t) * (size_t)cap);
  t->cap = cap;
}

/* octantForParticle, tree_gravity.cpp:50-61 */
static int octant_of(double x, double y, double z, double cx, double cy, double cz) {
  return ((x >= cx) << 2) | ((y >= cy) << 1) | (z >= cz);
}

/* buildNodeRecursive, tree_gravity.cpp:1081-1206 */
static uint32_t build_node(oracle_tree *t, const double *px, const double *py, const double *pz,
                           uint32_t begin, uint32_t end, double cx, double cy, double cz,
                           double half, uint32_t depth, int64_t leaf) {
  if (depth > 64) {
    t->status = 3;
    return 0xFFFFFFFFu;
  }
  if (depth > t->max_depth) t->max_depth = depth;
  const int64_t idx = t->n_nodes;
  tree_reserve(t, idx + 1);
  t->n_nodes = idx + 1;
  t->cx[idx] = cx;
  t->cy[idx] = cy;
  t->cz[idx] = cz;
  t->half[idx] = half;
  t->mass[idx] = 0.0;
  t->comx[idx] = cx;
  t->comy[idx] = cy;
  t->comz[idx] = cz;
  for (int k = 0; k < 6; ++k) t->q[k][idx] = 0.0;
  t->trace[idx] = 0.0;
  t->smin[idx] = INFINITY;
  t->smax[idx] = 0.0;
  t->child_count[idx] = 0;
  for (int k = 0; k < 8; ++k) t->child_index[8 * idx + k] = 0xFFFFFFFFu;
  t->pbegin[idx] = begin;
  t->pcount[idx] = end - begin;
  if ((int64_t)(end - begin) <= leaf || half <= 1.0e-12) return (uint32_t)idx;

  uint32_t count[8] = {0}, off[9];
  for (uint32_t i = begin; i < end; ++i) {
    const uint32_t s = t->sorted[i];
    ++count[octant_of(px[s], py[s], pz[s], cx, cy, cz)];
  }
  off[0] = begin;
  for (int k = 0; k < 8; ++k) off[k + 1] = off[k] + count[k];
  uint32_t cursor[8];
  for (int k = 0; k < 8; ++k) cursor[k] = off[k];
  for (uint32_t i = begin; i < end; ++i) {
    const uint32_t s = t->sorted[i];
    t->scratch[cursor[octant_of(px[s], py[s], pz[s], cx, cy, cz)]++] = s;
  }
  memcpy(t->sorted + begin, t->scratch + begin, sizeof(uint32_t) * (end - begin));
  uint32_t children = 0;
  for (int o = 0; o < 8; ++o) {
    if (off[o] == off[o + 1]) continue;
    const double ch = 0.5 * half;
    const double ccx = cx + ((o & 4) ? ch : -ch);
    const double ccy = cy + ((o & 2) ? ch : -ch);
    const double ccz = cz + ((o & 1) ? ch : -ch);
    const uint32_t c = build_node(t, px, py, pz, off[o], off[o + 1], ccx, ccy, ccz, ch, depth + 1, leaf);
    if (t->status) return 0xFFFFFFFFu;
    t->child_index[8 * idx + o] = c;
    ++children;
  }
  t->child_count[idx] = children;
  return (uint32_t)idx;
}

/* accumulateMultipoles, tree_gravity.cpp:1208-1380 (uniform softening
 * representation: every node's softening min/max is the uniform epsilon). */
static void accumulate(oracle_tree *t, const double *px, const double *py, const double *pz,
                       const double *m, uint32_t node, int quad, double eps) {
  if (t->child_count[node] == 0) {
    const uint32_t b = t->pbegin[node], e = b + t->pcount[node];
    double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    t->smin[node] = eps;
    t->smax[node] = eps;
    for (uint32_t i = b; i < e; ++i) {
      const uint32_t s = t->sorted[i];
      total += m[s];
      wx += m[s] * px[s];
      wy += m[s] * py[s];
      wz += m[s] * pz[s];
    }
    t->mass[node] = total;
    if (total > 0.0) {
      t->comx[node] = wx / total;
      t->comy[node] = wy / total;
      t->comz[node] = wz / total;
    }
    if (quad && total > 0.0) {
      const double cx = t->comx[node], cy = t->comy[node], cz = t->comz[node];
      double ixx = 0, ixy = 0, ixz = 0, iyy = 0, iyz = 0, izz = 0;
      for (uint32_t i = b; i < e; ++i) {
        const uint32_t s = t->sorted[i];
        const double rx = px[s] - cx, ry = py[s] - cy, rz = pz[s] - cz;
        ixx += m[s] * rx * rx;
        ixy += m[s] * rx * ry;
        ixz += m[s] * rx * rz;
        iyy += m[s] * ry * ry;
        iyz += m[s] * ry * rz;
        izz += m[s] * rz * rz;
      }
      const double tr = ixx + iyy + izz;
      t->trace[node] = tr;
      t->q[0][node] = 3.0 * ixx - tr;
      t->q[1][node] = 3.0 * ixy;
      t->q[2][node] = 3.0 * ixz;
      t->q[3][node] = 3.0 * iyy - tr;
      t->q[4][node] = 3.0 * iyz;
      t->q[5][node] = 3.0 * izz - tr;
    }
    return;
  }
  double total = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  for (int o = 0; o < 8; ++o) {
    const uint32_t c = t->child_index[8 * node + o];
    if (c == 0xFFFFFFFFu) continue;
    accumulate(t, px, py, pz, m, c, quad, eps);
    if (t->smin[c] < t->smin[node]) t->smin[node] = t->smin[c];
    if (t->smax[c] > t->smax[node]) t->smax[node] = t->smax[c];
    total += t->mass[c];
    wx += t->mass[c] * t->comx[c];
    wy += t->mass[c] * t->comy[c];
    wz += t->mass[c] * t->comz[c];
  }
  t->mass[node] = total;
  if (total > 0.0) {
    t->comx[node] = wx / total;
    t->comy[node] = wy / total;
    t->comz[node] = wz / total;
  }
  if (!quad || total <= 0.0) return;
  const double cx = t->comx[node], cy = t->comy[node], cz = t->comz[node];
  double qxx = 0, qxy = 0, qxz = 0, qyy = 0, qyz = 0, qzz = 0, tr = 0;
  for (int o = 0; o < 8; ++o) {
    const uint32_t c = t->child_index[8 * node + o];
    if (c == 0xFFFFFFFFu) continue;
    const double dx = t->comx[c] - cx, dy = t->comy[c] - cy, dz = t->comz[c] - cz;
    const double mc = t->mass[c];
    const double d2 = dx * dx + dy * dy + dz * dz;
    qxx += t->q[0][c] + mc * (3.0 * dx * dx - d2);
    qxy += t->q[1][c] + mc * (3.0 * dx * dy);
    qxz += t->q[2][c] + mc * (3.0 * dx * dz);
    qyy += t->q[3][c] + mc * (3.0 * dy * dy - d2);
    qyz += t->q[4][c] + mc * (3.0 * dy * dz);
    qzz += t->q[5][c] + mc * (3.0 * dz * dz - d2);
    tr += t->trace[c] + mc * d2;
  }
  t->q[0][node] = qxx;
  t->q[1][node] = qxy;
  t->q[2][node] = qxz;
  t->q[3][node] = qyy;
  t->q[4][node] = qyz;
  t->q[5][node] = qzz;
  t->trace[node] = tr;
}

static void bounds_of(int64_t n, const double *x, double *lo, double *hi) {
  *lo = INFINITY;
  *hi = -INFINITY;
  for (int64_t i = 0; i < n; ++i) {
    if (x[i] < *lo) *lo = x[i];
    if (x[i] > *hi) *hi = x[i];
  }
}

/* TreeGravitySolver::build, tree_gravity.cpp:343-524, with
 * buildMortonOrderingInPlace (tree_ordering.cpp:128-171) and its stable
 * 8-pass byte radix sort (:13-71). */
oracle_tree *oracle_tree_build(int64_t n, const double *ux, const double *uy, const double *uz,
                               const double *m, const oracle_params *p, int *status) {
  oracle_tree *t = (oracle_tree *)calloc(1, sizeof(oracle_tree));
  t->n = n;
  t->morton = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1));
  t->sorted = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  t->scratch = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  if (n == 0) {
    if (status) *status = 0;
    return t;
  }
  double lo[3], hi[3];
  bounds_of(n, ux, &lo[0], &hi[0]);
  bounds_of(n, uy, &lo[1], &hi[1]);
  bounds_of(n, uz, &lo[2], &hi[2]);
  double max_extent = hi[0] - lo[0];
  if (hi[1] - lo[1] > max_extent) max_extent = hi[1] - lo[1];
  if (hi[2] - lo[2] > max_extent) max_extent = hi[2] - lo[2];
  const double extent = max_extent > 1.0e-12 ? max_extent : 1.0e-12;
  const double grid = (double)((1u << 21) - 1u);
  for (int64_t i = 0; i < n; ++i) {
    double v[3] = {(ux[i] - lo[0]) / extent, (uy[i] - lo[1]) / extent, (uz[i] - lo[2]) / extent};
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
      const double c = v[a] < 0.0 ? 0.0 : (v[a] > 1.0 ? 1.0 : v[a]);
      q[a] = (uint32_t)llround(c * grid);
    }
    t->sorted[i] = (uint32_t)i;
    t->morton[i] = (expand_bits21(q[0]) << 2) | (expand_bits21(q[1]) << 1) | expand_bits21(q[2]);
  }
  /* stable LSD radix, 8 byte passes */
  uint64_t *kb = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
  uint32_t *ib = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
  uint64_t *ks = t->morton, *kd = kb;
  uint32_t *is = t->sorted, *id = ib;
  for (int pass = 0; pass < 8; ++pass) {
    const int shift = pass * 8;
    size_t cnt[256] = {0}, off[256];
    for (int64_t i = 0; i < n; ++i) ++cnt[(ks[i] >> shift) & 0xFF];
    off[0] = 0;
    for (int b = 1; b < 256; ++b) off[b] = off[b - 1] + cnt[b - 1];
    for (int64_t i = 0; i < n; ++i) {
      const size_t d = off[(ks[i] >> shift) & 0xFF]++;
      kd[d] = ks[i];
      id[d] = is[i];
    }
    uint64_t *tk = ks; ks = kd; kd = tk;
    uint32_t *ti = is; is = id; id = ti;
  }
  /* eight passes leave the result in the primary arrays */
  free(kb);
  free(ib);

  const double mext = max_extent > 1.0e-10 ? max_extent : 1.0e-10;
  const double rcx = 0.5 * (lo[0] + hi[0]);
  const double rcy = 0.5 * (lo[1] + hi[1]);
  const double rcz = 0.5 * (lo[2] + hi[2]);
  const double root_half = 0.5 * mext * (1.0 + 1.0e-8);
  build_node(t, ux, uy, uz, 0, (uint32_t)n, rcx, rcy, rcz, root_half, 0, p->leaf_size);
  if (t->status == 0) accumulate(t, ux, uy, uz, m, 0, p->quadrupole, p->epsilon);
  if (status) *status = t->status;
  return t;
}

int64_t oracle_tree_node_count(const oracle_tree *t) { return t->n_nodes; }
uint32_t oracle_tree_max_depth(const oracle_tree *t) { return t->max_depth; }

void oracle_tree_copy(const oracle_tree *t, int field, void *dst) {
  const size_t nn = (size_t)t->n_nodes, n = (size_t)t->n;
  const double *d[] = {t->cx, t->cy, t->cz, t->half, t->mass, t->comx, t->comy, t->comz,
                       t->q[0], t->q[1], t->q[2], t->q[3], t->q[4], t->q[5], t->trace};
  if (field == 0) memcpy(dst, t->morton, sizeof(uint64_t) * n);
  else if (field == 1) memcpy(dst, t->sorted, sizeof(uint32_t) * n);
  else if (field >= 2 && field <= 16) memcpy(dst, d[field - 2], sizeof(double) * nn);
  else if (field == 17) memcpy(dst, t->child_count, sizeof(uint32_t) * nn);
  else if (field == 18) memcpy(dst, t->child_index, sizeof(uint32_t) * 8 * nn);
  else if (field == 19) memcpy(dst, t->pbegin, sizeof(uint32_t) * nn);
  else if (field == 20) memcpy(dst, t->pcount, sizeof(uint32_t) * nn);
}

void oracle_tree_free(oracle_tree *t) {
  if (!t) return;
  double *dl[] = {t->cx, t->cy, t->cz, t->half, t->mass, t->comx, t->comy, t->comz, t->q[0],
                  t->q[1], t->q[2], t->q[3], t->q[4], t->q[5], t->trace, t->smin, t->smax};
  for (size_t k = 0; k < sizeof(dl) / sizeof(dl[0]); ++k) free(dl[k]);
  free(t->child_count);
  free(t->child_index);
  free(t->pbegin);
  free(t->pcount);
  free(t->morton);
  free(t->sorted);
  free(t->scratch);
  free(t);
}

/* ------------------------------------------------------------------ walk */

typedef struct {
  double length;
  int bounded;
} metric;

/* TreePmPeriodicMetric, internal/tree_pm_geometry.hpp:12-32 */
static double metric_apply(metric mt, double delta) {
  if (!(mt.length > 0.0)) return delta;
  const double half = 0.5 * mt.length;
  if (!mt.bounded || fabs(fabs(delta) - half) <= 4.0 * DBL_EPSILON * mt.length)
    return delta - mt.length * nearbyint(delta / mt.length);
  return delta > half ? delta - mt.length : (delta < -half ? delta + mt.length : delta);
}

static metric metric_make(double lo, double hi, double target, double length) {
  metric mt;
  mt.length = length;
  mt.bounded = isfinite(lo) && isfinite(hi) && lo - target >= -length && hi - target <= length;
  return mt;
}

/* treePmSquaredDistanceWithinCutoff, internal/tree_pm_geometry.hpp:51-60 */
static int within_cutoff(double d2, double cutoff, double cutoff2) {
  if (!isnormal(cutoff2) || !isfinite(d2) || fabs(d2 - cutoff2) <= 8.0 * DBL_EPSILON * cutoff2)
    return sqrt(d2) <= cutoff;
  return d2 <= cutoff2;
}

/* TreePmGaussianCoefficientTable (tree_pm_split_kernel.hpp:130-186): cubic
 * Hermite interpolation of H(t) = L(sqrt t)/t^(3/2) on t in [0, 64], 4096 cells,
 * slopes pre-scaled by the cell width. */
#define GAUSS_CELLS 4096
static const double k_gauss_step = 64.0 / GAUSS_CELLS;
typedef struct {
  double value[GAUSS_CELLS + 1];
  double slope[GAUSS_CELLS + 1];
} gauss_table;

static void gauss_table_init(gauss_table *g) {
  const double two_inv_sqrt_pi = 1.12837916709551257389615890312154517;
  for (int i = 0; i <= GAUSS_CELLS; ++i) {
    const double t = (double)i * k_gauss_step;
    const double q = sqrt(t);
    g->value[i] = i == 0 ? coefficient_series(0.0) : oracle_long_range_factor(q, 0.5) / (t * q);
    const double derivative = i == 0 ? -4.0 * k_inv_sqrt_pi / 5.0 : (two_inv_sqrt_pi * exp(-t) - 1.5 * g->value[i]) / t;
    g->slope[i] = k_gauss_step * derivative;
  }
}

static double gauss_hermite(const gauss_table *g, double t) {
  const double cell = t / k_gauss_step;
  const size_t i = (size_t)cell;
  const double u = cell - (double)i;
  const double u2 = u * u;
  const double u3 = u2 * u;
  return (2 * u3 - 3 * u2 + 1) * g->value[i] + (u3 - 2 * u2 + u) * g->slope[i] + (-2 * u3 + 3 * u2) * g->value[i + 1] +
         (u3 - u2) * g->slope[i + 1];
}

/* dimensionlessCoefficient (tree_pm_split_kernel.hpp:150-164) */
static double gauss_coefficient(const gauss_table *g, double t) {
  if (t < 0.015625) return coefficient_series(t);
  if (!(t < 64.0)) return long_range_inv_r3(sqrt(t), 0.5);
  return gauss_hermite(g, t);
}

/* longRangeInvR3 of the table (tree_pm_split_kernel.hpp:143-149) */
static double gauss_long_inv_r3(const gauss_table *g, double r2, double a) {
  const double t = 0.25 * (r2 / a) / a;
  if (!(t >= 0.0) || t >= 64.0) return long_range_inv_r3(sqrt(r2), a);
  return ((0.125 * gauss_coefficient(g, t) / a) / a) / a;
}

typedef struct {
  const oracle_tree *t;
  const oracle_params *p;
  const double *ox, *oy, *oz, *om; /* caller positions/masses gathered into tree order */
  double src_lo[3], src_hi[3], node_lo[3], node_hi[3];
  double rs, cutoff, cutoff2;
  const gauss_table *gt;      /* Gaussian pair lookup (NULL: analytic) */
  double inv_2a2, inv_8a3;    /* 1/(2 r_s)^2, 1/(8 r_s^3) */
  int scaling_ok;             /* both normal (tree_pm_coupling.cpp:3922-3925) */
  double len[3];              /* periodic box lengths; 0 for isolated/open (:3560-3562) */
} walk_ctx;

/* monopolePlusQuadrupoleAccelPeriodicReference, tree_pm_coupling.cpp:743-827 */
static void multipole_force(const walk_ctx *w, uint32_t node, double dx, double dy, double dz,
                            double eps_t, double *acc) {
  const oracle_tree *t = w->t;
  const double rs = w->rs;
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double safe_r2 = r2 > 1.0e-30 ? r2 : 1.0e-30;
  const double r = sqrt(safe_r2);
  const double pe = t->smax[node] > eps_t ? t->smax[node] : eps_t;
  const double eps2 = pe * pe;
  const double denom = (r2 + eps2) > 1.0e-30 ? (r2 + eps2) : 1.0e-30;
  const double soft = 1.0 / (denom * sqrt(denom));
  const double split = oracle_short_range_factor(r, rs);
  const double newton = 1.0 / (safe_r2 * r);
  const double radial = soft + (split - 1.0) * newton;
  const double G = w->p->G;
  double ax = G * t->mass[node] * radial * dx;
  double ay = G * t->mass[node] * radial * dy;
  double az = G * t->mass[node] * radial * dz;
  if (w->p->quadrupole) {
    const double tr = t->trace[node];
    const double mxx = (t->q[0][node] + tr) / 3.0, mxy = t->q[1][node] / 3.0,
                 mxz = t->q[2][node] / 3.0, myy = (t->q[3][node] + tr) / 3.0,
                 myz = t->q[4][node] / 3.0, mzz = (t->q[5][node] + tr) / 3.0;
    const double mdx = mxx * dx + mxy * dy + mxz * dz;
    const double mdy = mxy * dx + myy * dy + myz * dz;
    const double mdz = mxz * dx + myz * dy + mzz * dz;
    const double dmd = dx * mdx + dy * mdy + dz * mdz;
    const double rs2 = rs * rs;
    const double ex = exp(-r2 / (4.0 * rs2));
    const double sf = -0.5 * k_inv_sqrt_pi * r2 * ex / (rs * rs2);
    const double ss = k_inv_sqrt_pi * ex * (-r / (rs * rs2) + 0.25 * r * r2 / (rs * rs2 * rs2));
    const double soft1 = -3.0 * r / (denom * denom * sqrt(denom));
    const double soft2 = -3.0 / (denom * denom * sqrt(denom)) + 15.0 * r2 / (denom * denom * denom * sqrt(denom));
    const double n1 = -3.0 / (safe_r2 * safe_r2);
    const double n2 = 12.0 / (safe_r2 * safe_r2 * r);
    const double rf = soft1 + sf * newton + (split - 1.0) * n1;
    const double rsec = soft2 + ss * newton + 2.0 * sf * n1 + (split - 1.0) * n2;
    const double f1 = rf / r;
    const double cr = rsec / r2 - rf / (r2 * r);
    ax += G * (mdx * f1 + 0.5 * tr * dx * f1 + 0.5 * dx * dmd * cr);
    ay += G * (mdy * f1 + 0.5 * tr * dy * f1 + 0.5 * dy * dmd * cr);
    az += G * (mdz * f1 + 0.5 * tr * dz * f1 + 0.5 * dz * dmd * cr);
  }
  acc[0] += ax;
  acc[1] += ay;
  acc[2] += az;
}

static double com_center_offset(const oracle_tree *t, uint32_t node) {
  const double ox = t->cx[node] - t->comx[node];
  const double oy = t->cy[node] - t->comy[node];
  const double oz = t->cz[node] - t->comz[node];
  return sqrt(ox * ox + oy * oy + oz * oz);
}

/* acceptNodeByComDistanceMac, internal/tree_interaction_common.hpp:36-43 */
static int com_distance_mac(double theta, double h, double off, double r2) {
  const double r = sqrt(r2 + 1.0e-30);
  return ((2.0 * h + off) / r) < theta;
}

/* passesSofteningEnvelopeGuard, internal/tree_interaction_common.hpp:77-89 */
static int softening_ok(const oracle_tree *t, uint32_t node, double r, double eps_t) {
  if (t->smax[node] - t->smin[node] <= 1.0e-12) return 1;
  const double pe = t->smax[node] > eps_t ? t->smax[node] : eps_t;
  return r > (2.0 * t->half[node] + 2.0 * pe);
}

/* Strict-reference acceptance, internal/tree_pm_acceptance.hpp:170-255 with
 * acceptNodeByMac (internal/tree_interaction_common.hpp:45-75): COM-distance
 * or geometric MAC, or the relative-force criterion when the target has an
 * acceleration history. */
static int accept_strict(const walk_ctx *w, uint32_t node, int inside, int within, double r2,
                         double eps_t, int prev_avail, double prev_mag) {
  const oracle_tree *t = w->t;
  const double h = t->half[node];
  const double r = sqrt(r2 > 1.0e-30 ? r2 : 1.0e-30);
  const int soft_ok = softening_ok(t, node, r, eps_t);
  const int envelope_ok = w->p->quadrupole && (2.0 * h / r) < 0.08;
  int mac_ok;
  if (inside) {
    mac_ok = 0;
  } else if (w->p->criterion == 0) {
    mac_ok = (2.0 * h / sqrt(r2 + 1.0e-30)) < w->p->theta;
  } else if (w->p->criterion == 1 || !prev_avail) {
    mac_ok = com_distance_mac(w->p->theta, h, com_center_offset(t, node), r2);
  } else {
    const double scale = fabs(prev_mag) > w->p->accel_floor ? fabs(prev_mag) : w->p->accel_floor;
    const double width = 2.0 * h;
    const double estimated = w->p->G * t->mass[node] * width * width;
    const double allowed = w->p->rel_tol * scale * r2 * r2;
    mac_ok = estimated <= allowed;
  }
  return mac_ok && envelope_ok && soft_ok && within && !inside && isfinite(r2);
}

/* residualAccuracyProxy, internal/tree_pm_acceptance.hpp:20-51 (same order of
 * operations: the proxy is compared with alpha |a_previous|). */
static double residual_proxy(const walk_ctx *w, uint32_t node, double r2, double eps_t) {
  const oracle_tree *t = w->t;
  if (!(r2 > 0.0) || !isfinite(r2)) return INFINITY;
  const double rs = w->rs;
  const double r = sqrt(r2);
  const double eps = t->smax[node] > eps_t ? t->smax[node] : eps_t;
  const double d = r2 + eps * eps;
  const double inv_d5 = 1.0 / (d * d * sqrt(d));
  const double inv_r3 = 1.0 / (r2 * r);
  const double inv_r4 = 1.0 / (r2 * r2);
  const double long_factor = oracle_long_range_factor(r, rs);
  const double q = r / (2.0 * rs);
  const double exponential = exp(-q * q);
  const double scale3 = rs * rs * rs;
  const double s_first = -0.5 * k_inv_sqrt_pi * r2 * exponential / scale3;
  const double s_second = k_inv_sqrt_pi * exponential * (-r / scale3 + 0.25 * r * r2 / (scale3 * rs * rs));
  const double first = -3.0 * r * inv_d5 + s_first * inv_r3 - 3.0 * (-long_factor) * inv_r4;
  const double second = -3.0 * inv_d5 + 15.0 * r2 * inv_d5 / d + s_second * inv_r3 - 6.0 * s_first * inv_r4 +
                        12.0 * (-long_factor) * inv_r4 / r;
  const double width = 2.0 * t->half[node];
  const double rho = sqrt(3.0) * t->half[node] + com_center_offset(t, node);
  const double a = width * width * inv_r4;
  const double b = 0.5 * rho * rho * (3.0 * fabs(first) + fabs(r * second - first));
  const double proxy = w->p->G * t->mass[node] * (a > b ? a : b);
  return isfinite(proxy) && proxy >= 0.0 ? proxy : INFINITY;
}

/* Adaptive-relative acceptance, internal/tree_pm_acceptance.hpp:170-255:
 * opening-angle envelope, then the relative monopole (or residual-derivative)
 * estimate against alpha |a_previous|, or the COM-distance MAC without history. */
static int accept_adaptive(const walk_ctx *w, uint32_t node, int inside, int within, double r2, double eps_t,
                           int prev_avail, double prev_mag) {
  const oracle_tree *t = w->t;
  const double h = t->half[node];
  const double r = sqrt(r2 > 1.0e-30 ? r2 : 1.0e-30);
  const int soft_ok = softening_ok(t, node, r, eps_t);
  const int envelope_ok = (2.0 * h / r) < w->p->adaptive_angle;
  if (!envelope_ok || !soft_ok || inside || !within || !isfinite(r2)) return 0;
  const int history_ok = prev_avail && isfinite(prev_mag) && prev_mag > w->p->accel_floor;
  int mac_ok;
  if (history_ok) {
    const double allowance = w->p->rel_tol * prev_mag;
    const double width = 2.0 * h;
    const double inv_r4 = 1.0 / (r2 * r2);
    const double lower = w->p->G * t->mass[node] * (width * width * inv_r4);
    if (isfinite(allowance) && isfinite(lower) && lower > allowance) {
      mac_ok = 0;
    } else if (w->p->estimator == 1) {
      mac_ok = isfinite(allowance) && isfinite(lower);
    } else {
      const double est = residual_proxy(w, node, r2, eps_t);
      mac_ok = isfinite(est) && isfinite(allowance) && est <= allowance;
    }
  } else {
    mac_ok = com_distance_mac(w->p->theta, h, com_center_offset(t, node), r2);
  }
  return mac_ok;
}

/* evaluateTargetAgainstLocalTree, tree_pm_coupling.cpp:4026-4272 (no lookup
 * tables, no SIMD staging: the reference defaults). */
static void walk_target(const walk_ctx *w, double px, double py, double pz, uint32_t self,
                        int skip_self, double eps_t, int prev_avail, double prev_mag, uint32_t *stack,
                        size_t stack_cap, double out[4], oracle_counters *cnt) {
  const int adaptive = w->p->policy == 1;
  const int com_cutoff = adaptive && w->p->cutoff_policy == 1;
  const oracle_tree *t = w->t;
  double acc[3] = {0.0, 0.0, 0.0};
  double nearest = INFINITY;
  if (t->n_nodes == 0) {
    out[0] = out[1] = out[2] = 0.0;
    out[3] = nearest;
    return;
  }
  const double tg[3] = {px, py, pz};
  metric sm[3], nm[3];
  for (int a = 0; a < 3; ++a) {
    sm[a] = metric_make(w->src_lo[a], w->src_hi[a], tg[a], w->len[a]);
    nm[a] = metric_make(w->node_lo[a], w->node_hi[a], tg[a], w->len[a]);
  }
  size_t sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const uint32_t node = stack[--sp];
    ++cnt->visited;
    const double h = t->half[node];
    const double ndx = metric_apply(nm[0], t->cx[node] - px);
    const double ndy = metric_apply(nm[1], t->cy[node] - py);
    const double ndz = metric_apply(nm[2], t->cz[node] - pz);
    const double ax_ = fabs(ndx), ay_ = fabs(ndy), az_ = fabs(ndz);
    const double ex = ax_ - h > 0.0 ? ax_ - h : 0.0;
    const double ey = ay_ - h > 0.0 ? ay_ - h : 0.0;
    const double ez = az_ - h > 0.0 ? az_ - h : 0.0;
    const double min2 = ex * ex + ey * ey + ez * ez;
    if (!within_cutoff(min2, w->cutoff, w->cutoff2)) {
      ++cnt->pruned;
      continue;
    }
    const int is_leaf = t->child_count[node] == 0;
    int accept = is_leaf;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    if (!is_leaf) {
      /* the adaptive policy tests containment for every target (:4090-4092) */
      const int inside = (skip_self || adaptive) && ax_ <= h && ay_ <= h && az_ <= h;
      const double mx = ax_ + h, my = ay_ + h, mz = az_ + h;
      const int within = com_cutoff || within_cutoff(mx * mx + my * my + mz * mz, w->cutoff, w->cutoff2);
      dx = metric_apply(nm[0], t->comx[node] - px);
      dy = metric_apply(nm[1], t->comy[node] - py);
      dz = metric_apply(nm[2], t->comz[node] - pz);
      const double r2 = dx * dx + dy * dy + dz * dz;
      accept = adaptive ? accept_adaptive(w, node, inside, within, r2, eps_t, prev_avail, prev_mag)
                        : accept_strict(w, node, inside, within, r2, eps_t, prev_avail, prev_mag);
      /* kComDistance: an accepted node whose COM lies beyond r_cut is pruned (:4129-4132) */
      if (accept && com_cutoff && r2 > w->cutoff2) {
        ++cnt->pruned;
        continue;
      }
    }
    if (accept) {
      ++cnt->accepted;
      if (is_leaf) {
        ++cnt->leaves;
        const uint32_t b = t->pbegin[node], e = b + t->pcount[node];
        for (uint32_t s = b; s < e; ++s) {
          if (skip_self && t->sorted[s] == self) continue;
          const double sx = metric_apply(sm[0], w->ox[s] - px);
          const double sy = metric_apply(sm[1], w->oy[s] - py);
          const double sz = metric_apply(sm[2], w->oz[s] - pz);
          const double sr2 = sx * sx + sy * sy + sz * sz;
          if (sr2 > w->cutoff2) {
            ++cnt->pair_skips;
            continue;
          }
          if (sr2 < nearest) nearest = sr2;
          ++cnt->pairs;
          if (sx == 0.0 && sy == 0.0 && sz == 0.0) continue;
          const double pe = w->p->epsilon > eps_t ? w->p->epsilon : eps_t;
          double res;
          if (w->gt != NULL && sr2 > 0.0) {
            /* Gaussian pair lookup (tree_pm_coupling.cpp:4221-4226) */
            const double gt_t = w->scaling_ok ? sr2 * w->inv_2a2 : 64.0;
            const double long_inv_r3 =
                gt_t < 64.0 ? gauss_coefficient(w->gt, gt_t) * w->inv_8a3 : gauss_long_inv_r3(w->gt, sr2, w->rs);
            res = softened_inv_r3(sr2, pe) - long_inv_r3;
          } else {
            res = oracle_residual_inv_r3(sr2, pe, w->rs);
          }
          const double f = res * w->p->G;
          acc[0] += f * w->om[s] * sx;
          acc[1] += f * w->om[s] * sy;
          acc[2] += f * w->om[s] * sz;
        }
      } else {
        ++cnt->multipoles;
        multipole_force(w, node, dx, dy, dz, eps_t, acc);
      }
    } else {
      ++cnt->opened;
      for (int o = 7; o >= 0; --o) {
        const uint32_t c = t->child_index[8 * node + o];
        if (c != 0xFFFFFFFFu && sp < stack_cap) stack[sp++] = c;
      }
    }
  }
  out[0] = acc[0];
  out[1] = acc[1];
  out[2] = acc[2];
  out[3] = nearest;
}


/* ---------------------------------------------------------- group walk */
/* Opt-in group walk (TreePmOptions::group_walk_enabled, adaptive relative
 * monopole with the Gaussian pair table): internal/tree_pm_group_walk.hpp and
 * its driver tree_pm_coupling.cpp:4287-4560. Legacy grouping only
 * (group_walk_target_group_size = 0: the active targets of one source leaf,
 * consecutive in visit order inside one residual block of 64). */

/* treePmGroupNearestImage, tree_pm_group_walk.hpp:70-76 */
static double group_nearest_image(double delta, double length) {
  if (!(length > 0.0)) return delta;
  return delta - length * nearbyint(delta / length);
}

typedef struct {
  uint32_t *mult;
  size_t n_mult;
  uint32_t *leaf_begin, *leaf_end;
  double *leaf_dx, *leaf_dy, *leaf_dz, *leaf_h;
  size_t n_leaf;
} group_list;

/* buildTreePmGroupInteractionList, tree_pm_group_walk.hpp:78-154 */
static void group_build_list(const walk_ctx *w, const double center[3], const double half[3], double a_min,
                             uint32_t *stack, size_t stack_cap, group_list *out, oracle_counters *cnt) {
  const oracle_tree *t = w->t;
  const int contain = !(w->p->policy == 1 && w->p->cutoff_policy == 1);
  const double rel_over_g = w->p->rel_tol / w->p->G;
  const double angle2 = w->p->adaptive_angle * w->p->adaptive_angle;
  out->n_mult = out->n_leaf = 0;
  if (t->n_nodes == 0) return;
  size_t sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const uint32_t node = stack[--sp];
    ++cnt->visited;
    const double h = t->half[node];
    const double dc[3] = {group_nearest_image(t->cx[node] - center[0], w->len[0]),
                          group_nearest_image(t->cy[node] - center[1], w->len[1]),
                          group_nearest_image(t->cz[node] - center[2], w->len[2])};
    double gap2 = 0.0, far2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double ad = fabs(dc[a]);
      const double gap = ad - h - half[a] > 0.0 ? ad - h - half[a] : 0.0;
      const double far = ad + h + half[a];
      gap2 += gap * gap;
      far2 += far * far;
    }
    if (gap2 > w->cutoff2) {
      ++cnt->pruned;
      continue;
    }
    if (t->child_count[node] == 0) {
      ++cnt->leaves;
      ++cnt->accepted;
      const size_t k = out->n_leaf++;
      out->leaf_begin[k] = t->pbegin[node];
      out->leaf_end[k] = t->pbegin[node] + t->pcount[node];
      out->leaf_dx[k] = dc[0];
      out->leaf_dy[k] = dc[1];
      out->leaf_dz[k] = dc[2];
      out->leaf_h[k] = h;
      continue;
    }
    int accept = gap2 > 0.0 && (!contain || far2 <= w->cutoff2);
    if (accept) {
      const double dm[3] = {group_nearest_image(t->comx[node] - center[0], w->len[0]),
                            group_nearest_image(t->comy[node] - center[1], w->len[1]),
                            group_nearest_image(t->comz[node] - center[2], w->len[2])};
      double r_min2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double gap = fabs(dm[a]) - half[a] > 0.0 ? fabs(dm[a]) - half[a] : 0.0;
        r_min2 += gap * gap;
      }
      const double width2 = 4.0 * h * h;
      accept = r_min2 > 0.0 && width2 < angle2 * r_min2 &&
               t->mass[node] * width2 <= rel_over_g * a_min * r_min2 * r_min2;
    }
    if (accept) {
      ++cnt->multipoles;
      ++cnt->accepted;
      out->mult[out->n_mult++] = node;
    } else {
      ++cnt->opened;
      for (int o = 7; o >= 0; --o) {
        const uint32_t c = t->child_index[8 * node + o];
        if (c != 0xFFFFFFFFu && sp < stack_cap) stack[sp++] = c;
      }
    }
  }
}

/* accumulateTreePmGroupPairsImpl, tree_pm_group_walk.hpp:191-246 (owned
 * targets: the self pair excluded by source identity, distinct coincident
 * sources counted) */
static void group_pairs(const walk_ctx *w, double px, double py, double pz, size_t begin, size_t end,
                        uint32_t self_row, double acc[3], uint64_t *pairs, double *nearest) {
  const oracle_tree *t = w->t;
  const double lx = w->len[0], ly = w->len[1], lz = w->len[2];
  const double hx = 0.5 * lx, hy = 0.5 * ly, hz = 0.5 * lz;
  const double t_limit = nextafter(64.0, 0.0);
  const double eps2 = w->p->epsilon * w->p->epsilon;
  double sx = 0.0, sy = 0.0, sz = 0.0, near = *nearest;
  uint64_t counted = 0;
  for (size_t j = begin; j < end; ++j) {
    double dx = w->ox[j] - px, dy = w->oy[j] - py, dz = w->oz[j] - pz;
    dx = dx > hx ? dx - lx : (dx < -hx ? dx + lx : dx);
    dy = dy > hy ? dy - ly : (dy < -hy ? dy + ly : dy);
    dz = dz > hz ? dz - lz : (dz < -hz ? dz + lz : dz);
    const double r2 = dx * dx + dy * dy + dz * dz;
    const int is_self = self_row != 0xFFFFFFFFu && t->sorted[j] == self_row;
    const int inside = !is_self && r2 <= w->cutoff2;
    const double tt = r2 * w->inv_2a2 < t_limit ? r2 * w->inv_2a2 : t_limit;
    const double coefficient_long = gauss_hermite(w->gt, tt) * w->inv_8a3;
    const double d = r2 + eps2;
    const double softened = 1.0 / (d * sqrt(d));
    const double factor = inside && r2 > 0.0 ? (softened - coefficient_long) * w->p->G * w->om[j] : 0.0;
    sx += factor * dx;
    sy += factor * dy;
    sz += factor * dz;
    counted += inside ? 1u : 0u;
    near = fmin(near, inside ? r2 : near);
  }
  *nearest = near;
  acc[0] += sx;
  acc[1] += sy;
  acc[2] += sz;
  *pairs += counted;
}

/* One group through the shared list (evaluate_target_group,
 * tree_pm_coupling.cpp:4326-4422). Returns 0 when the group falls back to
 * per-target walks (history or geometry), before any accumulation. */
static int group_evaluate(const walk_ctx *w, const double *tx, const double *ty, const double *tz,
                          const uint32_t *rows, const double *prev, const int64_t *slots, size_t count,
                          uint32_t *stack, size_t stack_cap, group_list *list, double *res, oracle_counters *cnt) {
  const double len[3] = {w->len[0], w->len[1], w->len[2]};
  double a_min = INFINITY, ref[3] = {0, 0, 0}, low[3] = {0, 0, 0}, high[3] = {0, 0, 0};
  for (size_t i = 0; i < count; ++i) {
    const int64_t k = slots[i];
    const double pv = prev ? prev[k] : NAN;
    if (!(isfinite(pv) && pv > w->p->accel_floor)) return 0;
    if (pv < a_min) a_min = pv;
    const double pos[3] = {tx[k], ty[k], tz[k]};
    for (int a = 0; a < 3; ++a) {
      if (!metric_make(w->src_lo[a], w->src_hi[a], pos[a], len[a]).bounded) return 0;
      if (i == 0) {
        ref[a] = pos[a];
        continue;
      }
      const double delta = group_nearest_image(pos[a] - ref[a], len[a]);
      if (delta < low[a]) low[a] = delta;
      if (delta > high[a]) high[a] = delta;
    }
  }
  double center[3], half[3];
  for (int a = 0; a < 3; ++a) {
    center[a] = ref[a] + 0.5 * (low[a] + high[a]);
    half[a] = 0.5 * (high[a] - low[a]);
  }
  group_build_list(w, center, half, a_min, stack, stack_cap, list, cnt);
  const int com_cutoff = w->p->policy == 1 && w->p->cutoff_policy == 1;
  const double cull2 = w->cutoff2 * (1.0 + 1.0e-9);
  for (size_t i = 0; i < count; ++i) {
    const int64_t k = slots[i];
    const double px = tx[k], py = ty[k], pz = tz[k];
    double acc[3] = {0.0, 0.0, 0.0}, nearest = INFINITY;
    uint64_t pairs = 0;
    const double toff[3] = {group_nearest_image(px - center[0], len[0]), group_nearest_image(py - center[1], len[1]),
                            group_nearest_image(pz - center[2], len[2])};
    /* accumulateTreePmGroupCulledLeaves, tree_pm_group_walk.hpp:284-341 */
    size_t run_begin = 0, run_end = 0;
    int run_open = 0;
    for (size_t l = 0; l < list->n_leaf; ++l) {
      const double h = list->leaf_h[l];
      const double off[3] = {list->leaf_dx[l] - toff[0], list->leaf_dy[l] - toff[1], list->leaf_dz[l] - toff[2]};
      double g2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double hl = 0.5 * len[a];
        const double d = off[a] > hl ? off[a] - len[a] : (off[a] < -hl ? off[a] + len[a] : off[a]);
        const double g = fabs(d) - h > 0.0 ? fabs(d) - h : 0.0;
        g2 += g * g;
      }
      if (g2 > cull2) continue;
      const size_t b = list->leaf_begin[l], e = list->leaf_end[l];
      if (run_open && run_end == b) {
        run_end = e;
        continue;
      }
      if (run_open) group_pairs(w, px, py, pz, run_begin, run_end, rows[k], acc, &pairs, &nearest);
      run_begin = b;
      run_end = e;
      run_open = 1;
    }
    if (run_open) group_pairs(w, px, py, pz, run_begin, run_end, rows[k], acc, &pairs, &nearest);
    cnt->pairs += pairs;
    metric nm[3];
    const double pos[3] = {px, py, pz};
    for (int a = 0; a < 3; ++a) nm[a] = metric_make(w->node_lo[a], w->node_hi[a], pos[a], len[a]);
    const oracle_tree *t = w->t;
    for (size_t q = 0; q < list->n_mult; ++q) {
      const uint32_t node = list->mult[q];
      const double dx = metric_apply(nm[0], t->comx[node] - px);
      const double dy = metric_apply(nm[1], t->comy[node] - py);
      const double dz = metric_apply(nm[2], t->comz[node] - pz);
      if (com_cutoff && dx * dx + dy * dy + dz * dz > w->cutoff2) {
        ++cnt->pruned;
        continue;
      }
      multipole_force(w, node, dx, dy, dz, w->p->epsilon, acc);
    }
    res[4 * k + 0] = acc[0];
    res[4 * k + 1] = acc[1];
    res[4 * k + 2] = acc[2];
    res[4 * k + 3] = nearest;
  }
  return 1;
}

static int cmp_visit(const void *a, const void *b) {
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* solveActiveSetWithPmCadence (tree_pm_coupling.cpp:2282-3518) restricted to
 * the single-rank periodic strict path: PM refresh + interpolation, periodic
 * unwrap + tree build, then the residual walk per active target. */
int oracle_treepm_solve(int64_t n, const double *x, const double *y, const double *z,
                        const double *m, int64_t n_active, const uint32_t *active,
                        const oracle_params *p, double *ax, double *ay, double *az,
                        double *pm_ax, double *pm_ay, double *pm_az, double *tree_ax,
                        double *tree_ay, double *tree_az, double *nearest_r2,
                        oracle_counters *counters) {
  return oracle_treepm_solve2(n, x, y, z, m, n_active, active, p, NULL, ax, ay, az, pm_ax, pm_ay, pm_az,
                              tree_ax, tree_ay, tree_az, nearest_r2, counters);
}

int oracle_treepm_solve2(int64_t n, const double *x, const double *y, const double *z,
                         const double *m, int64_t n_active, const uint32_t *active,
                         const oracle_params *p, const double *prev_acc, double *ax, double *ay,
                         double *az, double *pm_ax, double *pm_ay, double *pm_az, double *tree_ax,
                         double *tree_ay, double *tree_az, double *nearest_r2,
                         oracle_counters *counters) {
  const int64_t na = active ? n_active : n;
  const double delta = oracle_mesh_spacing(p);
  const double rs = p->asmth_cells * delta;
  const double cutoff = p->rcut_cells * delta;
  double src_lo[3] = {INFINITY, INFINITY, INFINITY}, src_hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  const double *pos[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) {
    for (int64_t i = 0; i < n; ++i) {
      if (pos[a][i] < src_lo[a]) src_lo[a] = pos[a][i];
      if (pos[a][i] > src_hi[a]) src_hi[a] = pos[a][i];
    }
  }
  const double min_box = fmin(p->box[0], fmin(p->box[1], p->box[2]));
  if (p->boundary == 0 && !(cutoff < nextafter(0.5 * min_box, 0.0))) return 1; /* :374-381 */

  /* targets */
  double *tx = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  double *ty = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  double *tz = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  for (int64_t k = 0; k < na; ++k) {
    const int64_t i = active ? active[k] : k;
    tx[k] = x[i];
    ty[k] = y[i];
    tz[k] = z[i];
  }
  /* PM */
  const size_t cells = (size_t)p->mesh[0] * p->mesh[1] * p->mesh[2];
  double *fx = (double *)malloc(sizeof(double) * cells);
  double *fy = (double *)malloc(sizeof(double) * cells);
  double *fz = (double *)malloc(sizeof(double) * cells);
  oracle_pm_force_grids(n, x, y, z, m, p, fx, fy, fz);
  double *lx = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  double *ly = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  double *lz = (double *)malloc(sizeof(double) * (size_t)(na ? na : 1));
  oracle_pm_interpolate(p, fx, fy, fz, na, tx, ty, tz, lx, ly, lz);
  free(fx);
  free(fy);
  free(fz);

  /* tree: periodic unwrap (canonical flag as tree_pm_coupling.cpp:3183-3194) */
  double *ux = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *uy = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *uz = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *u[3] = {ux, uy, uz};
  for (int a = 0; a < 3; ++a) {
    if (p->boundary != 0) { /* isolated/open: the tree takes the caller's coordinates (:3179-3196) */
      memcpy(u[a], pos[a], sizeof(double) * (size_t)n);
      continue;
    }
    const int canonical = src_lo[a] >= 0.0 && src_hi[a] < p->box[a];
    oracle_unwrap_axis(n, pos[a], p->box[a], canonical, u[a]);
  }
  int status = 0;
  oracle_tree *t = oracle_tree_build(n, ux, uy, uz, m, p, &status);
  free(ux);
  free(uy);
  free(uz);
  if (status != 0) {
    oracle_tree_free(t);
    free(tx); free(ty); free(tz); free(lx); free(ly); free(lz);
    return 2;
  }
  walk_ctx w;
  memset(&w, 0, sizeof(w));
  w.t = t;
  w.p = p;
  w.rs = rs;
  for (int a = 0; a < 3; ++a) w.len[a] = p->boundary == 0 ? p->box[a] : 0.0;
  w.cutoff = cutoff;
  w.cutoff2 = cutoff * cutoff;
  for (int a = 0; a < 3; ++a) {
    w.src_lo[a] = src_lo[a];
    w.src_hi[a] = src_hi[a];
    w.node_lo[a] = INFINITY;
    w.node_hi[a] = -INFINITY;
  }
  /* node coordinate bounds over centers and COMs (tree_pm_coupling.cpp:3223-3242) */
  const double *nc[3] = {t->cx, t->cy, t->cz}, *nm[3] = {t->comx, t->comy, t->comz};
  for (int a = 0; a < 3; ++a) {
    for (int64_t k = 0; k < t->n_nodes; ++k) {
      w.node_lo[a] = fmin(w.node_lo[a], fmin(nc[a][k], nm[a][k]));
      w.node_hi[a] = fmax(w.node_hi[a], fmax(nc[a][k], nm[a][k]));
    }
  }
  /* tree-order copies of the caller's positions (:3736-3800) */
  double *ox = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *oy = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *oz = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *om = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  for (int64_t s = 0; s < n; ++s) {
    const uint32_t r = t->sorted[s];
    ox[s] = x[r];
    oy[s] = y[r];
    oz[s] = z[r];
    om[s] = m[r];
  }
  w.ox = ox;
  w.oy = oy;
  w.oz = oz;
  w.om = om;
  gauss_table *gt = NULL;
  if (p->gaussian_lookup) {
    gt = (gauss_table *)malloc(sizeof(gauss_table));
    gauss_table_init(gt);
  }
  w.gt = gt;
  w.inv_2a2 = (0.25 / rs) / rs;
  w.inv_8a3 = ((0.125 / rs) / rs) / rs;
  w.scaling_ok = isnormal(w.inv_2a2) && isnormal(w.inv_8a3);
  const size_t stack_cap = 1 + 7 * (size_t)t->max_depth;
  oracle_counters total;
  memset(&total, 0, sizeof(total));
  double *res = (double *)malloc(sizeof(double) * 4 * (size_t)(na ? na : 1));
  unsigned char *done = (unsigned char *)calloc((size_t)(na ? na : 1), 1);

  /* group walk eligibility (tree_pm_coupling.cpp:3840-3870, 4282-4286) */
  const double t_cut_group = (0.25 * w.cutoff2 / rs) / rs;
  const int group_active = p->group_walk && p->policy == 1 && p->estimator == 1 && gt != NULL && t->n_nodes > 0 &&
                           isfinite(t_cut_group) && t_cut_group < 63.0 && w.scaling_ok;
  if (group_active) {
    /* visit order: stable sort of active slots by the tree position of their row (:3808-3838) */
    uint32_t *pos_of_row = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    for (int64_t s2 = 0; s2 < n; ++s2) pos_of_row[t->sorted[s2]] = (uint32_t)s2;
    uint64_t *keyed = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(na ? na : 1));
    uint32_t *rows = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(na ? na : 1));
    for (int64_t k = 0; k < na; ++k) {
      const uint32_t row = active ? active[k] : (uint32_t)k;
      rows[k] = row;
      const uint64_t key = (int64_t)row < n ? pos_of_row[row] : 0xFFFFFFFFu;
      keyed[k] = (key << 32) | (uint64_t)k; /* ties keep slot order: a stable sort */
    }
    qsort(keyed, (size_t)na, sizeof(uint64_t), cmp_visit);
    uint32_t *leaf_of_pos = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    for (int64_t s2 = 0; s2 < n; ++s2) leaf_of_pos[s2] = 0xFFFFFFFFu;
    for (int64_t nd = 0; nd < t->n_nodes; ++nd) {
      if (t->child_count[nd] != 0) continue;
      for (uint32_t q = t->pbegin[nd]; q < t->pbegin[nd] + t->pcount[nd]; ++q) leaf_of_pos[q] = (uint32_t)nd;
    }
    const int64_t blocks = (na + 63) / 64;
#pragma omp parallel
    {
      uint32_t *stack = (uint32_t *)malloc(sizeof(uint32_t) * (stack_cap + 8));
      group_list list;
      const size_t cap = (size_t)t->n_nodes;
      list.mult = (uint32_t *)malloc(sizeof(uint32_t) * cap);
      list.leaf_begin = (uint32_t *)malloc(sizeof(uint32_t) * cap);
      list.leaf_end = (uint32_t *)malloc(sizeof(uint32_t) * cap);
      list.leaf_dx = (double *)malloc(sizeof(double) * cap);
      list.leaf_dy = (double *)malloc(sizeof(double) * cap);
      list.leaf_dz = (double *)malloc(sizeof(double) * cap);
      list.leaf_h = (double *)malloc(sizeof(double) * cap);
      int64_t slots[64];
      oracle_counters local;
      memset(&local, 0, sizeof(local));
#pragma omp for schedule(dynamic, 1)
      for (int64_t b = 0; b < blocks; ++b) {
        const int64_t v_end = (b + 1) * 64 < na ? (b + 1) * 64 : na;
        int64_t v = b * 64;
        while (v < v_end) {
          const int64_t k0 = (int64_t)(keyed[v] & 0xFFFFFFFFu);
          const uint32_t r0 = rows[k0];
          const uint32_t leaf = (int64_t)r0 < n ? leaf_of_pos[pos_of_row[r0]] : 0xFFFFFFFFu;
          int64_t g_end = v + 1;
          if (leaf != 0xFFFFFFFFu) {
            while (g_end < v_end) {
              const uint32_t rr = rows[(int64_t)(keyed[g_end] & 0xFFFFFFFFu)];
              if (!((int64_t)rr < n && leaf_of_pos[pos_of_row[rr]] == leaf)) break;
              ++g_end;
            }
            const size_t count = (size_t)(g_end - v);
            for (size_t i = 0; i < count; ++i) slots[i] = (int64_t)(keyed[v + (int64_t)i] & 0xFFFFFFFFu);
            if (group_evaluate(&w, tx, ty, tz, rows, prev_acc, slots, count, stack, stack_cap, &list, res, &local))
              for (size_t i = 0; i < count; ++i) done[slots[i]] = 1;
          }
          v = g_end;
        }
      }
#pragma omp critical
      {
        total.visited += local.visited;
        total.accepted += local.accepted;
        total.opened += local.opened;
        total.pairs += local.pairs;
        total.pruned += local.pruned;
        total.pair_skips += local.pair_skips;
        total.multipoles += local.multipoles;
        total.leaves += local.leaves;
      }
      free(list.mult); free(list.leaf_begin); free(list.leaf_end);
      free(list.leaf_dx); free(list.leaf_dy); free(list.leaf_dz); free(list.leaf_h);
      free(stack);
    }
    free(pos_of_row); free(keyed); free(rows); free(leaf_of_pos);
  }

#pragma omp parallel
  {
    uint32_t *stack = (uint32_t *)malloc(sizeof(uint32_t) * (stack_cap + 8));
    oracle_counters local;
    memset(&local, 0, sizeof(local));
#pragma omp for schedule(dynamic, 64)
    for (int64_t k = 0; k < na; ++k) {
      if (done[k]) continue;
      const uint32_t self = active ? active[k] : (uint32_t)k;
      /* history per active slot: present and finite (tree_pm_coupling.cpp:4467-4472) */
      const int avail = prev_acc != NULL && isfinite(prev_acc[k]);
      walk_target(&w, tx[k], ty[k], tz[k], self, 1, p->epsilon, avail, avail ? prev_acc[k] : 0.0, stack,
                  stack_cap, res + 4 * k, &local);
    }
#pragma omp critical
    {
      total.visited += local.visited;
      total.accepted += local.accepted;
      total.opened += local.opened;
      total.pairs += local.pairs;
      total.pruned += local.pruned;
      total.pair_skips += local.pair_skips;
      total.multipoles += local.multipoles;
      total.leaves += local.leaves;
    }
    free(stack);
  }
  for (int64_t k = 0; k < na; ++k) {
    if (ax) ax[k] = lx[k] + res[4 * k + 0];
    if (ay) ay[k] = ly[k] + res[4 * k + 1];
    if (az) az[k] = lz[k] + res[4 * k + 2];
    if (tree_ax) tree_ax[k] = res[4 * k + 0];
    if (tree_ay) tree_ay[k] = res[4 * k + 1];
    if (tree_az) tree_az[k] = res[4 * k + 2];
    if (nearest_r2) nearest_r2[k] = res[4 * k + 3];
  }
  free(res);
  free(done);
  free(gt);
  if (pm_ax) memcpy(pm_ax, lx, sizeof(double) * (size_t)na);
  if (pm_ay) memcpy(pm_ay, ly, sizeof(double) * (size_t)na);
  if (pm_az) memcpy(pm_az, lz, sizeof(double) * (size_t)na);
  if (counters) *counters = total;
  free(ox); free(oy); free(oz); free(om);
  free(tx); free(ty); free(tz); free(lx); free(ly); free(lz);
  oracle_tree_free(t);
  return 0;
}

/* applyPeculiarVelocityKick, gravity_runtime.cpp:3043-3059 */
void oracle_kick(int64_t n, double *vx, double *vy, double *vz, const double *ax,
                 const double *ay, const double *az, double kick, double drag) {
  for (int64_t i = 0; i < n; ++i) {
    /* the reference build contracts these to fused multiply-adds */
    vx[i] = fma(kick, ax[i], drag * vx[i]);
    vy[i] = fma(kick, ay[i], drag * vy[i]);
    vz[i] = fma(kick, az[i], drag * vz[i]);
  }
}

/* canonicalPeriodicPosition, include/cosmosim/core/periodic_domain.hpp:8-16 */
static double canonical(double v, double box) {
  double w = fmod(v, box);
  if (w < 0.0) w += box;
  if (!(w < box)) w = 0.0;
  return w;
}

/* drift task, reference_runtime_composition.cpp:76-107 */
void oracle_drift(int64_t n, double *x, double *y, double *z, const double *vx,
                  const double *vy, const double *vz, double drift, const double box[3]) {
  for (int64_t i = 0; i < n; ++i) {
    /* the reference build contracts x += v * D to a fused multiply-add */
    x[i] = fma(vx[i], drift, x[i]);
    y[i] = fma(vy[i], drift, y[i]);
    z[i] = fma(vz[i], drift, z[i]);
    x[i] = canonical(x[i], box[0]);
    y[i] = canonical(y[i], box[1]);
    z[i] = canonical(z[i], box[2]);
  }
}
