/*
 * adamantine_b200 -- diagnostic entry points (no counterpart in the
 * reference). They exist so that tests can check building blocks of the
 * kernels on the GPU.
 */
#ifndef ADAMANTINE_B200_DIAG_H
#define ADAMANTINE_B200_DIAG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y[i] = reciprocal of x[i] as computed by the tile kernel (Newton-Raphson on
 * the hardware estimate), and y_ref[i] = 1.0 / x[i] (IEEE division); device
 * pointers, n values, on the CUDA default stream; synchronizes. */
int adm_diag_reciprocal(double const *x, double *y, double *y_ref, int64_t n);

/* FP64 FMA throughput of the device in TFLOP/s (2 FLOP per FMA), measured
 * with independent FMA chains on every SM; the FP64 roofline denominator.
 * Best of five timed launches after one warm-up; synchronizes. */
int adm_diag_fp64_fma_rate(int device, double *tflops);

/* Runs the kernels' bounded mbarrier wait (a wall-time limit of limit_us
 * microseconds on the GPU's global timer, 1..10^6; the kernels use 2 s) on a
 * barrier that nothing arrives at; *timed_out = 1 when the wait gave up and
 * reported it (the path a TMA copy that never lands takes). The GPU keeps
 * running. */
int adm_diag_wait_timeout(long long limit_us, int32_t *timed_out);

#ifdef __cplusplus
}
#endif

#endif
