// kernels.cuh -- device kernels of one split step and of the observables.
//
// Layouts in HBM (dense, no pitch):
//   psi   [nx][ny][nz]        R (imaginary time) or complex R (real time)
//   spec  [nzh][nx][ny]       complex R, nzh = nz/2+1  (plane-major half spectrum)
//   phi   [nx][ny][nz]        R, unnormalised inverse FFT (the reference's psidd2)
//   udd   [nzh][nx/2+1][ny/2+1] FP64 octant of Udd(k) (depends on kx^2, ky^2, kz^2)
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace gpe {

struct Dims {
   int nx, ny, nz, nzh;
   int nzp;  // row pitch of the half spectrum in complex elements: nzh, or
             // nzh rounded up to even for complex64 so rows stay 16-byte multiples
   long long nxy, npts;
};

// Device-resident step state shared by the kernels of a step.
struct State {
   double norm;    // last pre-renormalisation norm
   double scale;   // pending 1/norm not yet applied to psi (1 when applied)
   double scale2;  // scale * scale, applied to |psi|^2 spectra
   double g, gd;   // couplings of the current step
   double pad[2];
   unsigned int ticket;  // CTAs of k_norm_final done (back to 0 after each launch)
   unsigned int pad_u;
};

template <class R, bool CPLX> struct Tr {
   using P = typename psi_elem<R, CPLX>::type;
   using C = cpx<R>;
};

// ---- rounding-exact helpers (no FMA contraction) --------------------------
__device__ __forceinline__ double mrn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double arn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mrn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float arn(float a, float b) { return __fadd_rn(a, b); }

// Trap potential recomputed from 1D tables exactly as initpot
// (imag3d-mpicuda.cu:872-889): 0.5 * par * (g2 x^2 + n2 y^2 + l2 z^2).
struct Trap {
   const double *x2, *y2, *z2;
   const float *x2f, *y2f, *z2f;  // FP32 copies (mixed precision)
   double hp;  // 0.5 * par
   double vg2, vn2, vl2;
   __device__ __forceinline__ double v(int i, int j, int k) const {
      double s = arn(arn(mrn(vg2, x2[i]), mrn(vn2, y2[j])), mrn(vl2, z2[k]));
      return mrn(hp, s);
   }
};

// Separable trap factors of calcnu in imaginary time.  V = 0.5 par (g2 x^2 +
// n2 y^2 + l2 z^2) is a sum over the axes, so exp(-dt V) is a product of one
// factor per axis; the factors are tabulated per axis on the host (long
// double) and only the nonlinear part of the exponent is evaluated per point.
// The tables are FP64 for FP64 handles and FP32 for mixed-precision ones.
struct LinPhase {
   const void *ex, *ey, *ez;
};

// exp(t) for the nonlinear part of the step's exponent, which is small in
// practice: Taylor series on |t| <= 1/8 (through t^10; the first omitted
// term is below 3e-18) and on |t| <= 0.5 (through t^16; below 2.2e-20
// relative), the library function beyond.  The short series is the common
// case: with it the 256^3 FP64 imaginary-time step (dt = 4e-3, g = 200)
// measured 0.667 -> 0.663 ms on B200.
__device__ __forceinline__ double exp_small(double t) {
   if (fabs(t) > 0.5) return exp(t);
   constexpr double f2 = 1. / 2, f3 = f2 / 3, f4 = f3 / 4, f5 = f4 / 5, f6 = f5 / 6, f7 = f6 / 7, f8 = f7 / 8,
                    f9 = f8 / 9, f10 = f9 / 10, f11 = f10 / 11, f12 = f11 / 12, f13 = f12 / 13, f14 = f13 / 14,
                    f15 = f14 / 15, f16 = f15 / 16;
   if (fabs(t) <= 0.125) {
      double e = f10;
      e = fma(e, t, f9);
      e = fma(e, t, f8);
      e = fma(e, t, f7);
      e = fma(e, t, f6);
      e = fma(e, t, f5);
      e = fma(e, t, f4);
      e = fma(e, t, f3);
      e = fma(e, t, f2);
      e = fma(e, t, 1.);
      return fma(e, t, 1.);
   }
   double e = f16;
   e = fma(e, t, f15);
   e = fma(e, t, f14);
   e = fma(e, t, f13);
   e = fma(e, t, f12);
   e = fma(e, t, f11);
   e = fma(e, t, f10);
   e = fma(e, t, f9);
   e = fma(e, t, f8);
   e = fma(e, t, f7);
   e = fma(e, t, f6);
   e = fma(e, t, f5);
   e = fma(e, t, f4);
   e = fma(e, t, f3);
   e = fma(e, t, f2);
   e = fma(e, t, 1.);
   return fma(e, t, 1.);
}

// calcnu of one FP64 element with the trap factor lin = exp(-dt V) from the
// axis tables: the same step as nu_op up to rounding.
__device__ __forceinline__ double nu_split(double p, double phi, double lin, double g, double gd, double dt,
                                           double invN) {
   const double thn = dt * fma(p * p, g, (phi * invN) * gd);
   return p * (lin * exp_small(-thn));
}
// calcnu on one element (imag3d-mpicuda.cu:1759-1783, real3d:1856-1883).
template <class R>
__device__ __forceinline__ R nu_op(R p, R phi, R V, R g, R gd, R dt, R invN) {
   R psi2lin = mrn(mrn(p, p), g);
   R psidd2lin = mrn(phi * invN, gd);
   R pt = mrn(dt, arn(arn(V, psi2lin), psidd2lin));
   return p * exp(-pt);
}
template <class R>
__device__ __forceinline__ cpx<R> nu_op(cpx<R> p, R phi, R V, R g, R gd, R dt, R invN) {
   R psi2lin = mrn(arn(mrn(p.x, p.x), mrn(p.y, p.y)), g);
   R psidd2lin = mrn(phi * invN, gd);
   R pt = mrn(dt, arn(arn(V, psi2lin), psidd2lin));
   R s, c;
   sincos(-pt, &s, &c);
   return cmul(p, mk<R>(c, s));
}

}  // namespace gpe
