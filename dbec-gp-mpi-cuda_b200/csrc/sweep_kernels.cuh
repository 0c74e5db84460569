// sweep_kernels.cuh -- Crank-Nicolson Thomas sweeps along x, y and z
// (calclux/calcluy/calcluz_kernel, imag3d-mpicuda.cu:1802-1942,
// real3d-mpicuda.cu:1902-2040) on whole lines staged in shared memory.
//
// A CTA owns TW lines.  The lines are brought in by one TMA tensor load (x
// and y sweeps: box of TW z-columns by the whole line) or by one bulk copy
// per row (z sweep), so every HBM access is a full 128-byte row segment and
// no transpose is needed.  The per-axis coefficient tables are read through
// the L1 cache, which the CTAs of an SM share.  Each line is split into P segments of m points,
// one thread per (line, segment); the two first-order recurrences of the
// Thomas algorithm
//    beta[i-1] = gamma[i] (A beta[i] - c_i),      i = n-2 .. 1
//    psi'[i+1] = alpha[i] psi'[i] + beta[i],      i = 0 .. n-3
// run locally from a zero carry-in, and the true values follow from the
// carries by the exact decomposition value = local + prefix_product * carry,
// with the prefix products of (gamma_i A) and alpha_i precomputed per axis
// (tables M and N).  The result equals the sequential recurrence up to
// rounding.
#pragma once

#include <type_traits>

#include "kernels.cuh"
#include "tma.cuh"

namespace gpe {

// Segment tables of one axis.
struct SegTab {
   const void *al, *ga;  // alpha, gamma padded to n entries (double or double2;
                         // float or float2 for the FP32 sweeps)
   const void *M, *N;    // prefix products, n entries each
   double2 A, A0r, mA;
   int n, m, P;
};

template <class R, bool CPLX> struct SegOps {
   using P = typename Tr<R, CPLX>::P;
   // table entry i: FP64 tables for FP64 sweeps, their once-rounded FP32
   // copies for FP32 sweeps
   __device__ static P ld(const void *t, int i) {
      if constexpr (std::is_same<R, float>::value) {
         if constexpr (CPLX) return __ldg((const float2 *) t + i);
         else return __ldg((const float *) t + i);
      } else if constexpr (CPLX) {
         const double2 v = __ldg((const double2 *) t + i);
         return mk<R>((R) v.x, (R) v.y);
      } else {
         return (R) __ldg((const double *) t + i);
      }
   }
   // the same from a table staged in shared memory
   __device__ static P lds(const void *t, int i) {
      if constexpr (CPLX) {
         const double2 v = ((const double2 *) t)[i];
         return mk<R>((R) v.x, (R) v.y);
      } else {
         return (R) ((const double *) t)[i];
      }
   }
   __device__ static P cv(double2 v) {
      if constexpr (CPLX) return mk<R>((R) v.x, (R) v.y);
      else return (R) v.x;
   }
   __device__ static P mul(P a, P b) {
      if constexpr (CPLX) return cmul(a, b);
      else return a * b;
   }
   // One backward Thomas step of the Crank-Nicolson system.  With the
   // coefficients of gencoef, minusA = -A and A0r = 1 + 2A in both modes
   // (imag: A = -c/2 real; real: A = -i c/2), so the right-hand side
   //    r = minusA psi[i+1] + A0r psi[i] - A psi[i-1] = psi[i] + A t,
   //    t = 2 psi[i] - psi[i+1] - psi[i-1],
   // and gamma (A beta - r) = gamma (A (beta - t) - psi[i]).  `a` is A's
   // real (imag mode) or imaginary (real mode) part.
   //
   // FP32 real time: gamma = -1 / (A0 + A alpha) is -1 plus a small complex
   // number (about i c), and a once-rounded FP32 gamma is off by up to half
   // an FP32 ulp of 1 at every index, the same error at every step: the
   // solve is then not unitary and the norm and mu drift linearly (1.7e-5
   // and 5.7e-5 after 200 steps of a 32x30x40 test, the error of the whole
   // mixed path; rounding alpha, A, psi, phi or the calcnu phase factor to
   // FP32 instead changes mu by at most 2e-8 there, measured with the FP64
   // oracle).  So the FP32 table holds gamma + 1, whose rounding error is
   // that of the small part, and gamma u = (gamma + 1) u - u costs the same
   // two multiply-adds per component.
   __device__ static P back_step(P b, P w2, P w1, P w0, P g, R a) {
      if constexpr (CPLX) {
         const R tx = fma((R) 2, w1.x, -w2.x) - w0.x, ty = fma((R) 2, w1.y, -w2.y) - w0.y;
         const R dx = b.x - tx, dy = b.y - ty;
         const R ux = fma(-a, dy, -w1.x), uy = fma(a, dx, -w1.y);
         P r;
         if constexpr (std::is_same<R, float>::value) {  // g = gamma + 1
            r.x = fma(g.x, ux, fma(-g.y, uy, -ux));
            r.y = fma(g.x, uy, fma(g.y, ux, -uy));
         } else {
            r.x = fma(g.x, ux, -g.y * uy);
            r.y = fma(g.x, uy, g.y * ux);
         }
         return r;
      } else {
         const R t = fma((R) 2, w1, -w2) - w0;
         return g * fma(a, b - t, -w1);
      }
   }
   __device__ static P fma_(P a, P b, P c) {  // a * b + c
      if constexpr (CPLX) {
         P r;
         r.x = fma(a.x, b.x, c.x);
         r.x = fma(-a.y, b.y, r.x);
         r.y = fma(a.x, b.y, c.y);
         r.y = fma(a.y, b.x, r.y);
         return r;
      } else {
         return fma(a, b, c);
      }
   }
};

// Segmented Thomas sweep of line c held in shared memory at
// s[i * es + c * cs], i in [0, n).  Called by all threads of the CTA; thread
// t = p * TW + c owns recurrence indices [p m, hf] of line c.  A warp holds
// SPW = 32 / TW consecutive segments of each of its TW lines.  blk is a
// shared scratch of 2 * (NW + 1) * TW elements (NW warps hold segments).
// Writes the swept line back in place.  When simp_w and simp_w2 are
// non-null, *simp receives this thread's share of sum_i simp_w[i] |psi'_i|^2
// and *simp2 that of sum_i simp_w2[i] |psi'_i|^2.  When only simp_w is
// non-null, *simp receives the share with the interior Simpson weights, 4 at
// odd i and 2 at even i, applied by parity without reading the table (a
// segment starts at an even index, m being even); the caller adds the end
// correction of an even-length line (simp_w's other entries).  Every
// value of the line the recurrence reads goes through xf(value, i) first
// (the fused calcnu of the x sweep; identity otherwise); a thread reads its
// own points and the two above its segment, so no transformed copy of the
// line is stored.
//
// Carries: segment p maps the value entering at its top (index hf+1) to the
// value at its bottom (index lo) by the affine map x -> b + a x with
// a = M[lo], b = beta~[lo]; the value entering segment p is the composition
// of the maps of all segments above it: a suffix scan, done with shuffles
// inside a warp and a short chain over the warps above.  The forward
// recurrence composes x -> psi'~[hf+1] + N[hf+1] x from the bottom (prefix).
struct NoXf {
   template <class P> __device__ __forceinline__ P operator()(P v, int) const { return v; }
};

template <class R, bool CPLX, int MSEG, int TWC = 0, class XF = NoXf, bool STAB = false>
__device__ __forceinline__ void seg_sweep(typename Tr<R, CPLX>::P *s, int es, int cs, int c, int p, int tw_arg,
                                          const SegTab &tb, typename Tr<R, CPLX>::P *blk, const double *simp_w,
                                          double *simp, const double *simp_w2 = nullptr,
                                          double *simp2 = nullptr, const XF &xf = XF()) {
   using Op = SegOps<R, CPLX>;
   using P = typename Tr<R, CPLX>::P;
   const int TW = TWC > 0 ? TWC : tw_arg;  // lines per CTA (compile time when TWC > 0)
   const int n = tb.n, m = tb.m, NP = tb.P;
   const int SPW = 32 / TW;              // segments of one line inside a warp
   const int NW = (NP + SPW - 1) / SPW;  // warps that hold segments
   const int lane = threadIdx.x & 31, j = lane / TW, w = threadIdx.x >> 5;
   const bool act = p < NP;
   const int lo = p * m;
   const bool top = (p == NP - 1);
   const int hf = top ? n - 3 : lo + m - 1;  // last owned recurrence index
   const int K = hf - lo + 1;                // owned points, 1 <= K <= MSEG
   const R a = CPLX ? (R) tb.A.y : (R) tb.A.x;
   P *line = s + c * cs;
   auto L = [&](int i) -> P { return xf(line[i * es], i); };
   // coefficient tables: global (read-only path) or staged in shared memory
   auto T = [&](const void *t, int i) -> P { return STAB ? Op::lds(t, i) : Op::ld(t, i); };
   P *ba = blk, *bb = blk + (NW + 1) * TW;  // per-warp block maps [NW][TW]
   const unsigned fullmask = 0xffffffffu;

   // ---- backward local recurrence: bt[q] = beta~[lo + q]
   P bt[MSEG];
   if (act) {
      P b = top ? L(n - 1) : zero_of<P>();  // beta[n-2] = psi[n-1] is exact
      // the step producing beta[lo+q] uses i = lo+q+1: psi[i+1], psi[i], psi[i-1]
      P w2 = L(lo + K + 1);
      P w1 = L(lo + K);
#pragma unroll
      for (int q = MSEG - 1; q >= 0; q--) {
         if (q < K) {
            const P w0 = L(lo + q);
            b = Op::back_step(b, w2, w1, w0, T(tb.ga, lo + q + 1), a);
            bt[q] = b;
            w2 = w1;
            w1 = w0;
         }
      }
   }
   // ---- suffix scan of the backward maps: in-warp, then over the warps above
   P sa = zero_of<P>(), sb = zero_of<P>();
   if (act) {
      sa = top ? zero_of<P>() : T(tb.M, lo);
      sb = bt[0];
   }
   for (int dd = 1; dd < SPW; dd <<= 1) {
      const P a2 = shfl_down_any(fullmask, sa, dd * TW), b2 = shfl_down_any(fullmask, sb, dd * TW);
      if (j + dd < SPW && p + dd < NP) {
         sb = Op::fma_(sa, b2, sb);
         sa = Op::mul(sa, a2);
      }
   }
   if (j == 0 && w < NW) {
      ba[w * TW + c] = sa;
      bb[w * TW + c] = sb;
   }
   __syncthreads();  // also: every read of the line is complete before it is rewritten
   P bin = zero_of<P>();
   {
      // value entering the top segment of this warp from the warps above
      P x = zero_of<P>();
      for (int ww = NW - 1; ww > w; ww--) x = Op::fma_(ba[ww * TW + c], x, bb[ww * TW + c]);
      const P here = Op::fma_(sa, x, sb);  // beta at the bottom of this segment
      const P nxt = shfl_down_any(fullmask, here, TW);
      bin = (j + 1 < SPW) ? nxt : x;
      if (!act || top) bin = zero_of<P>();
   }
   __syncthreads();  // the block maps are reused below

   // ---- forward local recurrence: bt[q] becomes psi'~[lo + q + 1]
   P v = zero_of<P>();
   sa = zero_of<P>();
   if (act) {
#pragma unroll
      for (int q = 0; q < MSEG; q++) {
         if (q < K) {
            const int i = lo + q;
            const P beta = Op::fma_(T(tb.M, i), bin, bt[q]);
            v = Op::fma_(T(tb.al, i), v, beta);
            bt[q] = v;
         }
      }
      sa = T(tb.N, hf + 1);
   }
   // ---- prefix scan of the forward maps
   sb = v;
   for (int dd = 1; dd < SPW; dd <<= 1) {
      const P a2 = shfl_up_any(fullmask, sa, dd * TW), b2 = shfl_up_any(fullmask, sb, dd * TW);
      if (j >= dd) {
         sb = Op::fma_(sa, b2, sb);
         sa = Op::mul(sa, a2);
      }
   }
   if (j == SPW - 1 && w < NW) {
      ba[w * TW + c] = sa;
      bb[w * TW + c] = sb;
   }
   __syncthreads();
   double acc = 0., acc2 = 0., acc_o = 0., acc_e = 0.;
   {
      P x = zero_of<P>();  // psi' entering the first segment of this warp
      for (int ww = 0; ww < w; ww++) x = Op::fma_(ba[ww * TW + c], x, bb[ww * TW + c]);
      const P upto = Op::fma_(sa, x, sb);  // psi'[hf + 1] of this segment
      const P prv = shfl_up_any(fullmask, upto, TW);
      const P fin = (j >= 1) ? prv : x;  // psi'[lo]
      if (act) {
#pragma unroll
         for (int q = 0; q < MSEG; q++) {
            if (q < K) {
               const int k = lo + q + 1;
               const P val = Op::fma_(T(tb.N, k), fin, bt[q]);
               line[k * es] = val;
               if (simp_w) {
                  const double f = (double) dens2(val);
                  if (simp_w2) {
                     acc += simp_w[k] * f;
                     acc2 += simp_w2[k] * f;
                  } else if (q & 1) {  // k = lo + q + 1 even
                     acc_e += f;
                  } else {
                     acc_o += f;
                  }
               }
            }
         }
         if (p == 0) line[0] = zero_of<P>();
         if (top) line[(n - 1) * es] = zero_of<P>();
      }
   }
   if (simp) *simp = simp_w2 ? acc : fma(4., acc_o, 2. * acc_e);
   if (simp2) *simp2 = acc2;
}

// exp(-i t) = (cos t, -sin t) for the nonlinear part of the real-time phase,
// which is small in practice: Maclaurin series on |t| <= 1/32 (through t^7
// for sin and t^6 for cos; the first omitted terms are below 3e-18 relative
// to sin and 3e-17 to cos) and on |t| <= 0.25 (through t^11 and t^12; below
// 3e-18), the library sincos beyond.  The short series is the common case:
// with it the 256^3 FP64 real-time step (dt = 4e-4, g = 200) measured 0.817
// -> 0.815 ms on B200.
__device__ __forceinline__ double2 expi_small(double t) {
   if (fabs(t) > 0.25) {
      double sn, cs;
      sincos(-t, &sn, &cs);
      return make_double2(cs, sn);
   }
   constexpr double s3 = 1. / 6, s5 = s3 / 20, s7 = s5 / 42, s9 = s7 / 72, s11 = s9 / 110;
   constexpr double c2 = 1. / 2, c4 = c2 / 12, c6 = c4 / 30, c8 = c6 / 56, c10 = c8 / 90, c12 = c10 / 132;
   const double t2 = t * t;
   if (fabs(t) <= 0.03125) {
      double sq = fma(-s7, t2, s5);
      sq = fma(sq, t2, -s3);
      const double sn = fma(sq * t2, t, t);
      double cq = fma(-c6, t2, c4);
      cq = fma(cq, t2, -c2);
      const double cs = fma(cq, t2, 1.);
      return make_double2(cs, -sn);
   }
   double sp = fma(-s11, t2, s9);
   sp = fma(sp, t2, -s7);
   sp = fma(sp, t2, s5);
   sp = fma(sp, t2, -s3);
   const double sn = fma(sp * t2, t, t);
   double cp = fma(c12, t2, -c10);
   cp = fma(cp, t2, c8);
   cp = fma(cp, t2, -c6);
   cp = fma(cp, t2, c4);
   cp = fma(cp, t2, -c2);
   const double cs = fma(cp, t2, 1.);
   return make_double2(cs, -sn);
}

// FP64 calcnu over a staged tile before its sweep (the x sweep's fused
// calcnu_kernel, imag3d-mpicuda.cu:1759, real3d-mpicuda.cu:1856), one z
// column per thread, with the pending 1/norm applied first.  Tile t of the
// sweep covers z columns [z0, z0 + TW) of plane `other` (y for the x sweep,
// x for the y sweep); xtab is calcnu's per-x table staged in shared memory
// (imaginary time: exp(-dt V_x); real time: the phase exp(-i dt V_x)).  The
// trap part of the exponent is a product of per-axis factors (V is a sum
// over the axes), so only the nonlinear part is evaluated per point, by a
// series.  The caller synchronises the CTA afterwards.
template <class R, bool CPLX, int AXIS>
__device__ __forceinline__ void nu_pass_fp64(typename Tr<R, CPLX>::P *tile, const R *ptile, int n, int lg, int c,
                                             int other, int z0, const Dims &d, const Trap &trap, const LinPhase &lin,
                                             const double *xtab, double g, double gd, double dt, double scale) {
   const R invN = (R) (1.0 / (double) d.npts);
   const int k = z0 + c;
   if (k >= d.nz) return;
   const int step = blockDim.x >> lg;
   if constexpr (!CPLX && AXIS == 0) {
      // imaginary time: trap factor exp(-dt V) from the axis tables, series
      // for the nonlinear part (measured faster than exp of the sum; in real
      // time CUDA's sincos of the sum measured faster than the split, so real
      // time keeps nu_op)
      const double eyz = __ldg((const double *) lin.ey + other) * __ldg((const double *) lin.ez + k);
      for (int ii = threadIdx.x >> lg; ii < n; ii += step) {
         const int e = (ii << lg) + c;
         const double lx = xtab[ii] * eyz;
         tile[e] = nu_split(scl(tile[e], scale), (double) ptile[e], lx, g, gd, dt, (double) invN);
      }
   } else if constexpr (CPLX && AXIS == 0) {
      // real time: psi exp(-i dt V_x) exp(-i dt (V_y + V_z)) exp(-i dt (g |psi|^2 + gd phi / N))
      const double2 ey = __ldg((const double2 *) lin.ey + other), ez = __ldg((const double2 *) lin.ez + k);
      const double2 eyz = cmul(ey, ez);
      const double2 *ex = (const double2 *) xtab;
      for (int ii = threadIdx.x >> lg; ii < n; ii += step) {
         const int e = (ii << lg) + c;
         const double2 p = scl(tile[e], scale);
         const double thn = dt * fma(fma(p.x, p.x, p.y * p.y), g, ((double) ptile[e] * invN) * gd);
         tile[e] = cmul(p, cmul(cmul(ex[ii], eyz), expi_small(thn)));
      }
   } else {
      // Trap::v with the terms of the two fixed coordinates hoisted
      const double tz = mrn(trap.vl2, trap.z2[k]);
      const double to = AXIS == 0 ? mrn(trap.vn2, trap.y2[other]) : mrn(trap.vg2, trap.x2[other]);
      const double *va = AXIS == 0 ? xtab : trap.y2;
      const double ca = AXIS == 0 ? trap.vg2 : trap.vn2;
#pragma unroll 2
      for (int ii = threadIdx.x >> lg; ii < n; ii += step) {
         const int e = (ii << lg) + c;
         const double sv = AXIS == 0 ? arn(arn(mrn(ca, va[ii]), to), tz) : arn(arn(to, mrn(ca, va[ii])), tz);
         const R V = (R) mrn(trap.hp, sv);
         tile[e] = nu_op<R>(scl(tile[e], scale), ptile[e], V, (R) g, (R) gd, (R) dt, invN);
      }
   }
}

// calcnu of the mixed-precision x sweep, applied as the sweep's recurrence
// reads each point (measured faster than a separate pass over the tile in
// FP32; slower in FP64, where a thread's extra evaluations for the two points
// above its segment cost more), entirely in FP32 like the step's other
// exponentials: real time recomputes V from the FP32 trap tables (the order
// of Trap::v) and takes sincosf of the exponent; imaginary time multiplies the
// FP32 trap factors exp(-dt V_x) exp(-dt V_y) exp(-dt V_z) and takes expf of
// the nonlinear part only.  The pending 1/norm is applied first.
template <bool CPLX> struct NuTrap32 {
   const float *ptile;  // phi tile, row stride tw
   int tw;
   const float *va;     // along the line: x^2 (real time) or exp(-dt V_x) (imaginary time)
   float ca, to, tz, hp;  // real time: V = hp ((ca va + to) + tz)
   float lfix;            // imaginary time: exp(-dt V_y) exp(-dt V_z) of this column
   float scale, g, gd, dt, invN;
   template <class P> __device__ __forceinline__ P operator()(P v, int i) const {
      const float phi = ptile[i * tw];
      if constexpr (CPLX) {
         const float2 p = make_float2(v.x * scale, v.y * scale);
         const float sv = __fadd_rn(__fadd_rn(__fmul_rn(ca, va[i]), to), tz);
         return nu_op<float>(p, phi, __fmul_rn(hp, sv), g, gd, dt, invN);
      } else {
         const float p = v * scale;
         const float thn = dt * fmaf(p * p, g, (phi * invN) * gd);
         return p * ((va[i] * lfix) * expf(-thn));
      }
   }
};

// The calcnu functor of tile column c of an x sweep tile covering z columns
// [z0, z0 + TW) of plane y = other (mixed precision).
template <bool CPLX>
__device__ __forceinline__ NuTrap32<CPLX> nu_reads_fp32(const float *ptile_c, int TW, int other, int z0, int c,
                                                        const Dims &d, const Trap &trap, const LinPhase &lin, double g,
                                                        double gd, double dt, double scale) {
   const int k = min(z0 + c, d.nz - 1);  // columns past nz are zero fill, never stored
   NuTrap32<CPLX> f;
   f.ptile = ptile_c;
   f.tw = TW;
   f.scale = (float) scale;
   f.g = (float) g;
   f.gd = (float) gd;
   f.dt = (float) dt;
   f.invN = (float) (1.0 / (double) d.npts);
   if constexpr (CPLX) {
      f.va = trap.x2f;
      f.ca = (float) trap.vg2;
      f.to = __fmul_rn((float) trap.vn2, trap.y2f[other]);
      f.tz = __fmul_rn((float) trap.vl2, trap.z2f[k]);
      f.hp = (float) trap.hp;
      f.lfix = 0.f;
   } else {
      f.va = (const float *) lin.ex;
      f.lfix = __ldg((const float *) lin.ey + other) * __ldg((const float *) lin.ez + k);
      f.ca = f.to = f.tz = f.hp = 0.f;
   }
   return f;
}

// ---------------------------------------------------------------------------
// Persistent pipelined CTAs.  A CTA walks the tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... through S shared-memory stages: while it sweeps
// tile i, the TMA engine already loads tile i+1 into the next stage and
// stores tile i-1 from the previous one.  Thread 0 issues every copy; before
// refilling a stage it waits until the bulk store that last read the stage
// has finished reading (all but the newest S-2 store groups: wait_stage_free).
//
// Resident CTAs per SM the sweep kernels are compiled for (register
// budget): [0] plain sweeps, [1] the x sweep fused with calcnu, whose tile
// also stages phi.  The host never launches more per SM.  Three CTAs (80
// registers) spill the 16-point segments and measured slower on B200.
constexpr int kSweepCtas[2] = {2, 2};


// x or y sweep.  Tile: TW consecutive z columns of one y (x sweep) or one x
// (y sweep) plane, the whole line along the swept axis, brought in by TMA.
// With NU the x sweep first applies the pending 1/norm and calcnu to the tile
// (needs phi).
template <class R, bool CPLX, int AXIS, bool NU, int MSEG, int S, int TWC>
__global__ void __launch_bounds__(256, kSweepCtas[NU ? 1 : 0]) k_sweep_xy(const __grid_constant__ CUtensorMap tm_psi,
                                                     const __grid_constant__ CUtensorMap tm_phi, Dims d, SegTab tb,
                                                     Trap trap, LinPhase lin, double g, double gd, double dt,
                                                     const State *__restrict__ st, int tw_arg, int boxn, int nbox,
                                                     uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   using P = typename Tr<R, CPLX>::P;
   const int TW = TWC > 0 ? TWC : tw_arg;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t full[S];
   const int n = tb.n;
   const int rows = boxn * nbox;  // rows staged (>= n)
   constexpr int E = CPLX ? 2 : 1;
   const uint32_t psi_bytes = (uint32_t) (rows * TW * sizeof(P));
   const uint32_t phi_bytes = NU ? (uint32_t) (rows * TW * sizeof(R)) : 0u;
   const uint32_t stage_bytes = (psi_bytes + phi_bytes + 127u) & ~127u;
   // layout: S stages of (tile | phi tile) | block maps  (TMA targets 128-byte aligned)
   unsigned char *base = (unsigned char *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   P *blk = (P *) (base + S * stage_bytes);
   const int nzb = (d.nz + TW - 1) / TW;
   const int ntiles = (AXIS == 0 ? d.ny : d.nx) * nzb;
   auto copy_tile = [&](int t, int q, bool load) {
      const int other = t / nzb, z0 = (t - other * nzb) * TW;
      P *tile = (P *) (base + q * stage_bytes);
      R *ptile = (R *) (tile + rows * TW);
      if (load) mbar_arrive_expect_tx(&full[q], psi_bytes + phi_bytes);
      for (int b = 0; b < nbox; b++) {
         const int a0 = b * boxn;
         if (load) {
            if (AXIS == 0) tma_load_3d(tile + a0 * TW, &tm_psi, E * z0, other, a0, &full[q]);
            else tma_load_3d(tile + a0 * TW, &tm_psi, E * z0, a0, other, &full[q]);
            if (NU) {
               if (AXIS == 0) tma_load_3d(ptile + a0 * TW, &tm_phi, z0, other, a0, &full[q]);
               else tma_load_3d(ptile + a0 * TW, &tm_phi, z0, a0, other, &full[q]);
            }
         } else {
            if (AXIS == 0) tma_store_3d(&tm_psi, E * z0, other, a0, tile + a0 * TW);
            else tma_store_3d(&tm_psi, E * z0, a0, other, tile + a0 * TW);
         }
      }
      if (!load) bulk_commit();
   };
   // FP64: calcnu's per-x factor (the phase exp(-i dt V_x) in real time,
   // exp(-dt V_x) in imaginary time) staged once per CTA after the block
   // maps, the shared tiles leaving little L1 for the tables (real-time x
   // sweep 223 -> 219 us at 256^3 when it held x^2; the FP32 sweep reads its
   // tables from global)
   double *xtab = (double *) (blk + 2 * (((tb.P + 32 / TW - 1) / (32 / TW)) + 1) * TW);
   if constexpr (NU && AXIS == 0 && std::is_same<R, double>::value) {
      // imaginary time: exp(-dt V_x); real time: (cos, sin) of -dt V_x
      const double *src = (const double *) lin.ex;
      for (int e = threadIdx.x; e < (CPLX ? 2 : 1) * n; e += blockDim.x) xtab[e] = src[e];
   }
   if (threadIdx.x == 0) {
      for (int q = 0; q < S; q++) mbar_init(&full[q], 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0 && (int) blockIdx.x < ntiles) copy_tile(blockIdx.x, 0, true);
   const double scale = NU ? st->scale : 1.;
   const int lg = __ffs(TW) - 1;  // TW is a power of two
   const int c = threadIdx.x & (TW - 1), p = threadIdx.x >> lg;
   int i = 0;
   for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
      const int q = i % S;
      if (threadIdx.x == 0 && t + (int) gridDim.x < ntiles) {
         wait_stage_free<S>();
         copy_tile(t + gridDim.x, (i + 1) % S, true);
      }
      // a timed-out copy makes the whole CTA leave together
      if (__syncthreads_or(!mbar_wait(&full[q], (i / S) & 1, err))) break;
      P *tile = (P *) (base + q * stage_bytes);
      const int other = t / nzb, z0 = (t - other * nzb) * TW;
      if constexpr (NU && std::is_same<R, double>::value) {
         nu_pass_fp64<R, CPLX, AXIS>(tile, (const R *) (tile + rows * TW), n, lg, c, other, z0, d, trap, lin, xtab, g,
                                     gd, dt, scale);
         __syncthreads();
      }
      if constexpr (NU && std::is_same<R, float>::value) {
         static_assert(AXIS == 0, "calcnu is fused into the x sweep only");
         const NuTrap32<CPLX> xf = nu_reads_fp32<CPLX>((const float *) (tile + rows * TW) + c, TW, other, z0, c, d,
                                                       trap, lin, g, gd, dt, scale);
         seg_sweep<R, CPLX, MSEG, TWC>(tile, TW, 1, c, p, TW, tb, blk, nullptr, nullptr, nullptr, nullptr, xf);
      } else {
         seg_sweep<R, CPLX, MSEG, TWC>(tile, TW, 1, c, p, TW, tb, blk, nullptr, nullptr);
      }
      fence_proxy_async();
      __syncthreads();
      if (threadIdx.x == 0) copy_tile(t, q, false);
   }
   if (threadIdx.x == 0) bulk_wait_all();
}

// The z sweep of one staged tile of TR rows (nr of them inside the grid)
// starting at grid row row0, with the Simpson row partials of MOM >= 1; ends
// with the tile written back in shared memory and a CTA barrier (the caller
// then stores it).
template <class R, bool CPLX, int MOM, int MSEG, int TWC, bool STAB>
__device__ __forceinline__ void zsweep_tile(typename Tr<R, CPLX>::P *tile, int nr, int TR, int LS, int c, int p,
                                            const SegTab &tbs, typename Tr<R, CPLX>::P *blk, double *part,
                                            double *part2, const double *__restrict__ wz,
                                            const double *__restrict__ wz2, double hz3, double *__restrict__ rowsum,
                                            double *__restrict__ rowsum2, long long row0) {
   using P = typename Tr<R, CPLX>::P;
   constexpr bool SIMP = MOM >= 1;
   if (nr < TR) {  // rows beyond the grid are zero so their sweep stays finite
      for (int e = threadIdx.x; e < (TR - nr) * LS; e += blockDim.x) tile[nr * LS + e] = zero_of<P>();
      __syncthreads();
   }
   double my = 0., my2 = 0.;
   seg_sweep<R, CPLX, MSEG, TWC, NoXf, STAB>(tile, 1, LS, c, p, TR, tbs, blk, SIMP ? wz : nullptr, SIMP ? &my : nullptr,
                                             MOM == 2 ? wz2 : nullptr, MOM == 2 ? &my2 : nullptr);
   if (SIMP && p < tbs.P) part[p * TR + c] = my;
   if (MOM == 2 && p < tbs.P) part2[p * TR + c] = my2;
   fence_proxy_async();
   __syncthreads();
   // row rr's sums on the last warp, so that warp 0 (whose thread 0 issues
   // the tile's store and the next load) goes on at once (TR <= 32)
   const int rr = (int) threadIdx.x - ((int) blockDim.x - 32);
   if (SIMP && rr >= 0 && rr < nr) {
      double sum = 0.;
      for (int pp = 0; pp < tbs.P; pp++) sum += part[pp * TR + rr];
      if (MOM == 1 && !(tbs.n & 1)) {
         // the end correction of an even nz: the weights of points nz-2 and
         // nz-3 are 3 and 3.75 where the interior weights give 2 and 4
         const int n = tbs.n;
         const typename Tr<R, CPLX>::P *row = tile + rr * LS;
         sum += (double) dens2(row[n - 2]) - 0.25 * (double) dens2(row[n - 3]);
      }
      rowsum[row0 + rr] = sum * hz3;
      if (MOM == 2) {
         double sum2 = 0.;
         for (int pp = 0; pp < tbs.P; pp++) sum2 += part2[pp * TR + rr];
         rowsum2[row0 + rr] = sum2 * hz3;
      }
   }
}

// z sweep.  Tile: TR consecutive (x, y) rows, each copied by one bulk copy to
// a padded shared row (stride LS elements).  With MOM >= 1 every row also
// yields its Simpson integral of |psi'|^2 over z (simpint, diffint.cu:106),
// for the norm of the step (rowsum); with MOM = 2 also that of z^2 |psi'|^2
// (rowsum2), the row partials of calcrms, so an rms sample after the step
// needs no extra pass over psi.
template <class R, bool CPLX, int MOM, int MSEG, int S, int TWC>
__global__ void __launch_bounds__(256, kSweepCtas[0]) k_sweep_z(typename Tr<R, CPLX>::P *__restrict__ psi, Dims d, SegTab tb,
                                                    int tr_arg, int LS, const double *__restrict__ wz,
                                                    const double *__restrict__ wz2, double hz3,
                                                    double *__restrict__ rowsum, double *__restrict__ rowsum2,
                                                    uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   const int TR = TWC > 0 ? TWC : tr_arg;
   using P = typename Tr<R, CPLX>::P;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t full[S];
   const int nz = d.nz;
   const uint32_t row_bytes = (uint32_t) (nz * sizeof(P));
   const uint32_t stage_bytes = ((uint32_t) (TR * LS * sizeof(P)) + 127u) & ~127u;
   // layout: S stages of rows | block maps | Simpson partials
   unsigned char *base = (unsigned char *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   const int NW = (tb.P + 32 / TR - 1) / (32 / TR);
   P *blk = (P *) (base + S * stage_bytes);
   double *part = (double *) (blk + 2 * (NW + 1) * TR);
   double *part2 = part + tb.P * TR;
   // FP64: the coefficient tables (alpha, gamma, M, N) staged once per CTA,
   // the shared rows leaving little L1 for them (z sweep 129 -> 128 us real,
   // 94 -> 93 us imaginary time at 256^3; FP32 measured slower with it)
   constexpr bool STAB = std::is_same<R, double>::value;
   constexpr int TE = CPLX ? 2 : 1;  // doubles per entry
   double *tabs = part2 + tb.P * TR;
   SegTab tbs = tb;
   if constexpr (STAB) {
      const void *src[4] = {tb.al, tb.ga, tb.M, tb.N};
      for (int a = 0; a < 4; a++)
         for (int e = threadIdx.x; e < tb.n * TE; e += blockDim.x) tabs[a * tb.n * TE + e] = ((const double *) src[a])[e];
      tbs.al = tabs;
      tbs.ga = tabs + tb.n * TE;
      tbs.M = tabs + 2 * tb.n * TE;
      tbs.N = tabs + 3 * tb.n * TE;
   }
   const int ntiles = (int) ((d.nxy + TR - 1) / TR);
   auto nrows = [&](int t) -> int {
      const long long r0 = (long long) t * TR;
      return (int) ((d.nxy - r0) < TR ? (d.nxy - r0) : TR);
   };
   auto copy_tile = [&](int t, int q, bool load) {
      P *tile = (P *) (base + q * stage_bytes);
      const int nr = nrows(t);
      if (load) mbar_arrive_expect_tx(&full[q], row_bytes * nr);
      for (int r = 0; r < nr; r++) {
         P *g = psi + ((long long) t * TR + r) * nz;
         if (load) bulk_load(tile + r * LS, g, row_bytes, &full[q]);
         else bulk_store(g, tile + r * LS, row_bytes);
      }
      if (!load) bulk_commit();
   };
   if (threadIdx.x == 0) {
      for (int q = 0; q < S; q++) mbar_init(&full[q], 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0 && (int) blockIdx.x < ntiles) copy_tile(blockIdx.x, 0, true);
   const int c = threadIdx.x % TR, p = threadIdx.x / TR;
   int i = 0;
   for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
      const int q = i % S;
      if (threadIdx.x == 0 && t + (int) gridDim.x < ntiles) {
         wait_stage_free<S>();
         copy_tile(t + gridDim.x, (i + 1) % S, true);
      }
      if (__syncthreads_or(!mbar_wait(&full[q], (i / S) & 1, err))) break;
      P *tile = (P *) (base + q * stage_bytes);
      zsweep_tile<R, CPLX, MOM, MSEG, TWC, STAB>(tile, nrows(t), TR, LS, c, p, tbs, blk, part, part2, wz, wz2, hz3,
                                                rowsum, rowsum2, (long long) t * TR);
      if (threadIdx.x == 0) copy_tile(t, q, false);
   }
   if (threadIdx.x == 0) bulk_wait_all();
}

}  // namespace gpe
