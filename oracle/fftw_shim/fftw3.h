/* Test infrastructure (oracle): the subset of the public FFTW3 API that the
 * reference's PM solver calls (src/gravity/pm_solver.cpp:2093-2128 plans for
 * the isolated workspace, :2248-2266 periodic r2c/c2r plans, :2711/:2722
 * execute, :1985-1998 destroy, :61-62 threads). FFTW itself is not installed
 * here; these declarations carry only FFTW's published names and signatures and
 * are implemented by fftw3_shim.c on top of oracle/fft.c. Only the oracle build
 * of the reference (oracle/_ref) links it.
 */
#ifndef CHUI_ORACLE_FFTW3_SHIM_H
#define CHUI_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct chui_oracle_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_EXHAUSTIVE (1U << 3)

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup(void);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif
