/* chui_treepm_diag.h -- measurement helpers of the B200 TreePM solver.
 *
 * Not part of the reference-facing boundary (no counterpart in the reference):
 * the residual walk is bound by the FP32 pipes, so its roofline needs a
 * measured FP32 FMA throughput of the GPU, which this probe provides.
 */
#ifndef CHUI_TREEPM_DIAG_H
#define CHUI_TREEPM_DIAG_H

#ifdef __cplusplus
extern "C" {
#endif

/* Measured FP32 FMA throughput of `device` in TFLOP/s (an FMA counts 2). */
int chui_treepm_probe_fp32_peak(int device, double *tflops);

#ifdef __cplusplus
}
#endif

#endif
