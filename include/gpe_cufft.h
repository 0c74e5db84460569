/*
 * gpe_cufft.h -- the dipolar convolution through cuFFT, kept only as a timed
 * comparison for the solver's own FFT passes (libgpe_cufft.so; libgpe.so
 * never calls cuFFT).
 *
 * Replaces nothing on the solver's path: it re-runs the reference's cuFFT
 * pipeline of calcpsidd2_mem (src/imag3d-mpicuda/imag3d-mpicuda.cu:1460-1510,
 * plans :1092-1126) on one GPU so that its time can be set beside the
 * solver's (gpe_time_calcpsidd2 in gpe.h) on the same grid and inputs.
 */
#ifndef GPE_CUFFT_H
#define GPE_CUFFT_H

#include "gpe.h"

#ifdef __cplusplus
extern "C" {
#endif

/* phi = IFFT_unnormalised[Udd(k) FFT[|psi|^2]] with the boundary planes,
 * computed by cuFFT.  p: grid, spacings, cutoff, mode (psi real or
 * interleaved complex) and precision (FP64: D2Z/Z2Z/Z2D; mixed: R2C/C2C/C2R
 * on FP32 data); p->device selects the GPU (-1 = current).  psi: host
 * x-major array.  variant 0 follows the reference's call structure (the
 * one-rank transpose copies and one Z2Z execution along x per y line, as the
 * host loop of imag3d-mpicuda.cu:1472-1485); variant 1 uses one batched Z2Z
 * plan along x and no copies.  After one untimed convolution, nrep
 * convolutions are timed with CUDA events: *ms (may be NULL) receives the
 * mean milliseconds per convolution and phi (host, nx*ny*nz doubles, may be
 * NULL) the last result.  Allocates its own device buffers and plans. */
gpe_status gpe_cufft_convolution(const gpe_params *p, const double *psi, int variant, int nrep, double *phi,
                                 double *ms);
/* Message of the last failure of gpe_cufft_convolution on this thread. */
const char *gpe_cufft_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GPE_CUFFT_H */
