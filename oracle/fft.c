/* Test infrastructure (oracle): double-precision 3-D FFT, see fft.h.
 *
 * Power-of-two lengths use an iterative radix-2 Cooley-Tukey transform with
 * twiddles evaluated directly as cos/sin of 2*pi*k/n (no recurrence drift);
 * other lengths use a direct DFT with the same exact-angle twiddles. The 3-D
 * transform is three passes of 1-D transforms over lines, OpenMP-parallel over
 * lines when compiled with -fopenmp.
 */
#include "fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double k_two_pi = 6.283185307179586476925286766559;

typedef struct {
  int n;
  int pow2;
  double *tw; /* cos/sin pairs, n entries (angle 2*pi*k/n) */
  int *rev;   /* bit reversal permutation (pow2 only) */
} line_plan;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void plan_init(line_plan *p, int n) {
  p->n = n;
  p->pow2 = is_pow2(n);
  p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    /* reduce k/n to keep the angle small and exact-ish */
    const double a = k_two_pi * (double)k / (double)n;
    p->tw[2 * k] = cos(a);
    p->tw[2 * k + 1] = sin(a);
  }
  p->rev = NULL;
  if (p->pow2) {
    p->rev = (int *)malloc(sizeof(int) * (size_t)n);
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
      p->rev[i] = r;
    }
  }
}

static void plan_free(line_plan *p) {
  free(p->tw);
  free(p->rev);
}

/* One line, interleaved complex, contiguous. scratch holds 2n doubles. */
static void line_fft(const line_plan *p, double *x, int sign, double *scratch) {
  const int n = p->n;
  if (n == 1) return;
  if (p->pow2) {
    for (int i = 0; i < n; ++i) {
      const int r = p->rev[i];
      if (r > i) {
        double t0 = x[2 * i], t1 = x[2 * i + 1];
        x[2 * i] = x[2 * r];
        x[2 * i + 1] = x[2 * r + 1];
        x[2 * r] = t0;
        x[2 * r + 1] = t1;
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1;
      const int step = n / len;
      for (int start = 0; start < n; start += len) {
        for (int k = 0; k < half; ++k) {
          const double wr = p->tw[2 * (k * step)];
          const double wi = (double)sign * p->tw[2 * (k * step) + 1];
          double *a = x + 2 * (start + k);
          double *b = x + 2 * (start + k + half);
          const double br = b[0] * wr - b[1] * wi;
          const double bi = b[0] * wi + b[1] * wr;
          b[0] = a[0] - br;
          b[1] = a[1] - bi;
          a[0] += br;
          a[1] += bi;
        }
      }
    }
    return;
  }
  for (int k = 0; k < n; ++k) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; ++j) {
      const int m = (int)(((long long)j * k) % n);
      const double wr = p->tw[2 * m];
      const double wi = (double)sign * p->tw[2 * m + 1];
      sr += x[2 * j] * wr - x[2 * j + 1] * wi;
      si += x[2 * j] * wi + x[2 * j + 1] * wr;
    }
    scratch[2 * k] = sr;
    scratch[2 * k + 1] = si;
  }
  memcpy(x, scratch, sizeof(double) * 2 * (size_t)n);
}

/* Transform along one axis of a (d0, d1, d2) complex array. */
static void axis_pass(double *data, int d0, int d1, int d2, int axis, int sign) {
  const int n = axis == 0 ? d0 : (axis == 1 ? d1 : d2);
  line_plan plan;
  plan_init(&plan, n);
  const long long lines = (long long)d0 * d1 * d2 / n;
#pragma omp parallel
  {
    double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)n);
    double *scratch = buf + 2 * n;
#pragma omp for schedule(static)
    for (long long l = 0; l < lines; ++l) {
      size_t base, stride;
      if (axis == 2) {
        base = (size_t)l * (size_t)d2;
        stride = 1;
      } else if (axis == 1) {
        const long long i0 = l / d2, i2 = l % d2;
        base = (size_t)i0 * (size_t)d1 * (size_t)d2 + (size_t)i2;
        stride = (size_t)d2;
      } else {
        base = (size_t)l; /* l = i1*d2 + i2 */
        stride = (size_t)d1 * (size_t)d2;
      }
      for (int j = 0; j < n; ++j) {
        buf[2 * j] = data[2 * (base + j * stride)];
        buf[2 * j + 1] = data[2 * (base + j * stride) + 1];
      }
      line_fft(&plan, buf, sign, scratch);
      for (int j = 0; j < n; ++j) {
        data[2 * (base + j * stride)] = buf[2 * j];
        data[2 * (base + j * stride) + 1] = buf[2 * j + 1];
      }
    }
    free(buf);
  }
  plan_free(&plan);
}

void oracle_fft3d_c2c(double *data, int n0, int n1, int n2, int sign) {
  axis_pass(data, n0, n1, n2, 2, sign);
  axis_pass(data, n0, n1, n2, 1, sign);
  axis_pass(data, n0, n1, n2, 0, sign);
}

void oracle_fft3d_r2c(const double *in, size_t in_row_stride, double *out,
                      int n0, int n1, int n2) {
  const size_t total = (size_t)n0 * n1 * n2;
  const int nzc = n2 / 2 + 1;
  double *work = (double *)malloc(sizeof(double) * 2 * total);
  for (size_t row = 0; row < (size_t)n0 * n1; ++row) {
    for (int k = 0; k < n2; ++k) {
      work[2 * (row * n2 + k)] = in[row * in_row_stride + k];
      work[2 * (row * n2 + k) + 1] = 0.0;
    }
  }
  oracle_fft3d_c2c(work, n0, n1, n2, -1);
  for (size_t row = 0; row < (size_t)n0 * n1; ++row) {
    for (int k = 0; k < nzc; ++k) {
      out[2 * (row * nzc + k)] = work[2 * (row * n2 + k)];
      out[2 * (row * nzc + k) + 1] = work[2 * (row * n2 + k) + 1];
    }
  }
  free(work);
}

void oracle_fft3d_c2r(const double *in, double *out, size_t out_row_stride,
                      int n0, int n1, int n2) {
  const size_t total = (size_t)n0 * n1 * n2;
  const int nzc = n2 / 2 + 1;
  double *work = (double *)malloc(sizeof(double) * 2 * total);
  /* Rebuild the full Hermitian spectrum: X[i0,i1,k] = conj(X[-i0,-i1,-k]). */
  for (int i0 = 0; i0 < n0; ++i0) {
    for (int i1 = 0; i1 < n1; ++i1) {
      const size_t row = (size_t)i0 * n1 + i1;
      const size_t mrow = (size_t)((n0 - i0) % n0) * n1 + (size_t)((n1 - i1) % n1);
      for (int k = 0; k < n2; ++k) {
        double re, im;
        if (k < nzc) {
          re = in[2 * (row * nzc + k)];
          im = in[2 * (row * nzc + k) + 1];
        } else {
          const int mk = n2 - k;
          re = in[2 * (mrow * nzc + mk)];
          im = -in[2 * (mrow * nzc + mk) + 1];
        }
        work[2 * (row * n2 + k)] = re;
        work[2 * (row * n2 + k) + 1] = im;
      }
    }
  }
  oracle_fft3d_c2c(work, n0, n1, n2, +1);
  for (size_t row = 0; row < (size_t)n0 * n1; ++row) {
    for (int k = 0; k < n2; ++k) out[row * out_row_stride + k] = work[2 * (row * n2 + k)];
  }
  free(work);
}
