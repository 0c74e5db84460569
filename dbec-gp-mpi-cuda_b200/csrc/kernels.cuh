// kernels.cuh -- device kernels of one split step and of the observables.
//
// Layouts in HBM (dense, no pitch):
//   psi   [nx][ny][nz]        R (imaginary time) or complex R (real time)
//   beta  same as psi         Thomas scratch
//   spec  [nzh][nx][ny]       complex R, nzh = nz/2+1  (plane-major half spectrum)
//   phi   [nx][ny][nz]        R, unnormalised inverse FFT (the reference's psidd2)
//   udd   [nzh][nx/2+1][ny/2+1] FP64 octant of Udd(k) (depends on kx^2, ky^2, kz^2)
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace gpe {

struct Dims {
   int nx, ny, nz, nzh;
   long long nxy, npts;
};

// Thomas coefficients of one axis (gencoef, imag3d-mpicuda.cu:894-931 and
// real3d-mpicuda.cu:991-1035): alpha/gamma are double (imaginary time) or
// double2 (real time) arrays of n-1 entries.
struct Coef {
   const void *alpha;
   const void *gamma;
   double2 A, A0r, mA;
};

// Device-resident step state shared by the kernels of a step.
struct State {
   double norm;    // last pre-renormalisation norm
   double scale;   // pending 1/norm not yet applied to psi (1 when applied)
   double scale2;  // scale * scale, applied to |psi|^2 spectra
   double g, gd;   // couplings of the current step
   double pad[3];
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
   double hp;  // 0.5 * par
   double vg2, vn2, vl2;
   __device__ __forceinline__ double v(int i, int j, int k) const {
      double s = arn(arn(mrn(vg2, x2[i]), mrn(vn2, y2[j])), mrn(vl2, z2[k]));
      return mrn(hp, s);
   }
};

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

// ---- coefficient access ---------------------------------------------------
template <class R, bool CPLX> struct CoefT;
template <class R> struct CoefT<R, false> {
   using P = R;
   __device__ static P al(const Coef &c, int i) { return (R) ((const double *) c.alpha)[i]; }
   __device__ static P ga(const Coef &c, int i) { return (R) ((const double *) c.gamma)[i]; }
   __device__ static P A(const Coef &c) { return (R) c.A.x; }
   __device__ static P A0r(const Coef &c) { return (R) c.A0r.x; }
   __device__ static P mA(const Coef &c) { return (R) c.mA.x; }
   __device__ static P mul(P a, P b) { return a * b; }
   __device__ static P fma_(P a, P b, P d) { return fma(a, b, d); }
};
template <class R> struct CoefT<R, true> {
   using P = cpx<R>;
   __device__ static P cv(double2 v) { return mk<R>((R) v.x, (R) v.y); }
   __device__ static P al(const Coef &c, int i) { return cv(((const double2 *) c.alpha)[i]); }
   __device__ static P ga(const Coef &c, int i) { return cv(((const double2 *) c.gamma)[i]); }
   __device__ static P A(const Coef &c) { return cv(c.A); }
   __device__ static P A0r(const Coef &c) { return cv(c.A0r); }
   __device__ static P mA(const Coef &c) { return cv(c.mA); }
   __device__ static P mul(P a, P b) { return cmul(a, b); }
   __device__ static P fma_(P a, P b, P d) {
      P r;
      r.x = fma(a.x, b.x, d.x);
      r.x = fma(-a.y, b.y, r.x);
      r.y = fma(a.x, b.y, d.y);
      r.y = fma(a.y, b.x, r.y);
      return r;
   }
};

// ---------------------------------------------------------------------------
// Thomas sweep along one line held in global memory, one thread per line
// (calclux/y/z_kernel, imag3d-mpicuda.cu:1802-1942).  load(i) yields psi[i]
// (with calcnu applied on the fly where fused); beta is the scratch line.
template <class R, bool CPLX, bool SIMP, class LoadF>
__device__ __forceinline__ double thomas_line(typename Tr<R, CPLX>::P *psi, typename Tr<R, CPLX>::P *beta,
                                              long long st, int n, const Coef &cf, LoadF load, double h) {
   using K = CoefT<R, CPLX>;
   using P = typename Tr<R, CPLX>::P;
   const P A = K::A(cf), A0r = K::A0r(cf), mA = K::mA(cf);
   P nxt = load(n - 1);
   P cur = load(n - 2);
   P bcur = nxt;
   beta[(long long) (n - 2) * st] = bcur;
   for (int i = n - 2; i > 0; i--) {
      P prv = load(i - 1);
      P c = K::mul(mA, nxt);
      c = (P) cadd_any(c, K::mul(A0r, cur));
      c = (P) csub_any(c, K::mul(A, prv));
      P bprev = K::mul(K::ga(cf, i), csub_any(K::mul(A, bcur), c));
      beta[(long long) (i - 1) * st] = bprev;
      bcur = bprev;
      nxt = cur;
      cur = prv;
   }
   Simpson sp;
   if (SIMP) { sp.init(n); sp.add(0, 0.); }
   P p = zero_of<P>();
   psi[0] = p;
   for (int i = 0; i < n - 2; i++) {
      p = K::fma_(K::al(cf, i), p, beta[(long long) i * st]);
      psi[(long long) (i + 1) * st] = p;
      if (SIMP) sp.add(i + 1, (double) dens2(p));
   }
   psi[(long long) (n - 1) * st] = zero_of<P>();
   if (SIMP) { sp.add(n - 1, 0.); return sp.finish(h); }
   return 0.;
}

}  // namespace gpe
