/* Test infrastructure (oracle): a small double-precision 3-D FFT.
 *
 * Used by the CPU restatement of the TreePM path (oracle/treepm_oracle.c) and
 * by the FFTW-API subset shim (oracle/fftw_shim) that lets the reference's own
 * PM code run its FFTW branch (src/gravity/pm_solver.cpp:2248-2266, :2708-2723)
 * without FFTW being installed. Never linked into the product library.
 *
 * Conventions follow FFTW3's published definitions: forward = exp(-2*pi*i*jk/n),
 * backward = exp(+2*pi*i*jk/n), both unnormalized; r2c/c2r use the half
 * spectrum along the last axis (n2/2+1 complex values per row).
 */
#ifndef CHUI_ORACLE_FFT_H
#define CHUI_ORACLE_FFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* In-place complex 3-D transform of an n0*n1*n2 array of interleaved
 * (re, im) doubles in row-major order. sign = -1 forward, +1 backward. */
void oracle_fft3d_c2c(double *data, int n0, int n1, int n2, int sign);

/* Real -> half-spectrum. `in` holds n0*n1*n2 reals with row stride
 * `in_row_stride` (n2 for dense, 2*(n2/2+1) for FFTW in-place layout);
 * `out` receives n0*n1*(n2/2+1) complex values. in and out may alias. */
void oracle_fft3d_r2c(const double *in, size_t in_row_stride, double *out,
                      int n0, int n1, int n2);

/* Half-spectrum -> real (unnormalized backward). `in` holds n0*n1*(n2/2+1)
 * complex values; `out` receives reals with row stride `out_row_stride`.
 * in and out may alias. */
void oracle_fft3d_c2r(const double *in, double *out, size_t out_row_stride,
                      int n0, int n1, int n2);

#ifdef __cplusplus
}
#endif

#endif
