/* Test infrastructure (oracle): FFTW3-API subset over oracle/fft.c (see fftw3.h).
 * In-place r2c/c2r plans (in == out) use FFTW's padded row layout of
 * 2*(n2/2+1) reals; out-of-place plans use dense rows, as FFTW defines.
 */
#include "fftw3.h"

#include <stdlib.h>
#include <string.h>

#include "../fft.h"

enum { k_r2c = 0, k_c2r = 1, k_c2c = 2 };

struct chui_oracle_fftw_plan_s {
  int kind;
  int n0, n1, n2;
  int sign;
  void *in;
  void *out;
};

static fftw_plan make_plan(int kind, int n0, int n1, int n2, void *in, void *out, int sign) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return NULL;
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags) {
  (void)flags;
  return make_plan(k_r2c, n0, n1, n2, in, out, -1);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags) {
  (void)flags;
  return make_plan(k_c2r, n0, n1, n2, in, out, +1);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags) {
  (void)flags;
  return make_plan(k_c2c, n0, n1, n2, in, out, sign);
}

void fftw_execute(const fftw_plan p) {
  if (p == NULL) return;
  const size_t padded = 2 * (size_t)(p->n2 / 2 + 1);
  if (p->kind == k_r2c) {
    const size_t stride = p->in == p->out ? padded : (size_t)p->n2;
    oracle_fft3d_r2c((const double *)p->in, stride, (double *)p->out, p->n0, p->n1, p->n2);
  } else if (p->kind == k_c2r) {
    const size_t stride = p->in == p->out ? padded : (size_t)p->n2;
    oracle_fft3d_c2r((const double *)p->in, (double *)p->out, stride, p->n0, p->n1, p->n2);
  } else {
    const size_t total = (size_t)p->n0 * p->n1 * p->n2;
    if (p->in != p->out) memcpy(p->out, p->in, sizeof(double) * 2 * total);
    oracle_fft3d_c2c((double *)p->out, p->n0, p->n1, p->n2, p->sign);
  }
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}
