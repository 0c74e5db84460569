// fft.cuh -- shared-memory mixed-radix Stockham FFT used by every FFT pass
// of the dipolar convolution (the reference calls cuFFT D2Z/Z2Z/Z2D here,
// src/imag3d-mpicuda/imag3d-mpicuda.cu:1460-1510; this is a project-written
// transform, not cuFFT's).
//
// A CTA transforms L lines of length n held in shared memory in the
// interleaved layout [j][L]: element j of line l at base[j * L + l].  L is
// 128 bytes of elements (8 complex doubles, 16 complex floats), so the L
// threads that handle one butterfly position of the L lines touch one
// 128-byte row: bank-conflict free.  This is also the layout a TMA box of L
// columns by the whole line lands in.
//
// Radices 2, 3, 4, 5, 8 and (FP32, 16 points per thread) 16.  Each radix-r
// stage (autosort Stockham, decimation in time) computes
//   j in [0, n/r), k = j mod Ns,  v[t] = src[j + t n/r] * W^(t k n/(Ns r))
//   v = DFT_r(v),  dst[(j / Ns) Ns r + k + t Ns] = v[t],  Ns *= r
// leaving the result in natural order; src and dst are the same buffer, the
// reads of a stage finishing (barrier) before its writes start.  W = exp(-2 pi i / n) comes from a
// table of the n-th roots computed on the host in long double (twmul > 1
// reads a table of a longer transform with stride twmul).  Inverse
// transforms use conjugated twiddles and are unnormalised, like cuFFT's
// CUFFT_INVERSE.
#pragma once

#include "common.cuh"

namespace gpe {

constexpr int kMaxStages = 12;

struct FftPlan {
   int n;
   int nst;
   int rad[kMaxStages];
   int ns[kMaxStages];             // Ns before the stage
   unsigned magic[kMaxStages];     // ceil(2^32 / Ns): j / Ns == umulhi(j, magic) for j < 2^16
};

// ---- small DFT kernels (constants are exact values of cos/sin) -------------
template <class C, bool INV> __device__ __forceinline__ void dft2(C *v) {
   C a = v[0], b = v[1];
   v[0] = cadd(a, b);
   v[1] = csub(a, b);
}

template <class C, bool INV> __device__ __forceinline__ void dft3(C *v) {
   using R = decltype(v[0].x);
   const R s3 = (R) 0.86602540378443864676;  // sin(2 pi / 3)
   C a = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
   C m = csub(a, cscale(t1, (R) 0.5));
   C r = cscale(mul_mi<C, INV>(t2), s3);  // -i s3 t2 (forward)
   v[0] = cadd(a, t1);
   v[1] = cadd(m, r);
   v[2] = csub(m, r);
}

template <class C, bool INV> __device__ __forceinline__ void dft4(C *v) {
   C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
   C t2 = cadd(v[1], v[3]), t3 = mul_mi<C, INV>(csub(v[1], v[3]));
   v[0] = cadd(t0, t2);
   v[2] = csub(t0, t2);
   v[1] = cadd(t1, t3);
   v[3] = csub(t1, t3);
}

template <class C, bool INV> __device__ __forceinline__ void dft5(C *v) {
   using R = decltype(v[0].x);
   const R c1 = (R) 0.30901699437494742410, c2 = (R) -0.80901699437494742410;
   const R s1 = (R) 0.95105651629515357212, s2 = (R) 0.58778525229247312917;
   C a0 = v[0];
   C b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
   C d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
   C p1 = cadd(a0, cadd(cscale(b1, c1), cscale(b2, c2)));
   C p2 = cadd(a0, cadd(cscale(b1, c2), cscale(b2, c1)));
   C q1 = mul_mi<C, INV>(cadd(cscale(d1, s1), cscale(d2, s2)));
   C q2 = mul_mi<C, INV>(csub(cscale(d1, s2), cscale(d2, s1)));
   v[0] = cadd(a0, cadd(b1, b2));
   v[1] = cadd(p1, q1);
   v[4] = csub(p1, q1);
   v[2] = cadd(p2, q2);
   v[3] = csub(p2, q2);
}

template <class C, bool INV> __device__ __forceinline__ void dft8(C *v) {
   using R = decltype(v[0].x);
   const R h = (R) 0.70710678118654752440;  // 1/sqrt(2)
   C e[4] = {v[0], v[2], v[4], v[6]};
   C o[4] = {v[1], v[3], v[5], v[7]};
   dft4<C, INV>(e);
   dft4<C, INV>(o);
   // o[k] *= W8^k (forward W8 = (1 - i)/sqrt2)
   C w1, w3;
   if (INV) {
      w1.x = (o[1].x - o[1].y) * h; w1.y = (o[1].x + o[1].y) * h;     // (1+i)/sqrt2
      w3.x = (-o[3].x - o[3].y) * h; w3.y = (o[3].x - o[3].y) * h;    // (-1+i)/sqrt2
   } else {
      w1.x = (o[1].x + o[1].y) * h; w1.y = (o[1].y - o[1].x) * h;     // (1-i)/sqrt2
      w3.x = (-o[3].x + o[3].y) * h; w3.y = (-o[3].x - o[3].y) * h;   // (-1-i)/sqrt2
   }
   C w2 = mul_mi<C, INV>(o[2]);
   v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
   v[1] = cadd(e[1], w1);   v[5] = csub(e[1], w1);
   v[2] = cadd(e[2], w2);   v[6] = csub(e[2], w2);
   v[3] = cadd(e[3], w3);   v[7] = csub(e[3], w3);
}

// 16-point DFT as 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2): a DFT4 over n1 for
// every n2, the twiddles W16^(n2 k1), a DFT4 over n2 for every k1.
template <class C, bool INV> __device__ __forceinline__ void dft16(C *v) {
   using R = decltype(v[0].x);
   const R c1 = (R) 0.92387953251128675613, s1 = (R) 0.38268343236508977173;  // cos, sin(pi / 8)
   const R h = (R) 0.70710678118654752440;
   C y[4][4];
#pragma unroll
   for (int n2 = 0; n2 < 4; n2++) {
      C t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      dft4<C, INV>(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; k1++) y[n2][k1] = t[k1];
   }
   // W16^m, m = n2 k1 in {1, 2, 3, 2, 4, 6, 3, 6, 9} (forward: exp(-2 pi i m / 16))
   const R sg = INV ? (R) 1 : (R) -1;
   auto tw = [&](C a, R wr, R wi) -> C { C r; r.x = a.x * wr - a.y * wi; r.y = a.x * wi + a.y * wr; return r; };
   y[1][1] = tw(y[1][1], c1, sg * s1);
   y[1][2] = tw(y[1][2], h, sg * h);
   y[1][3] = tw(y[1][3], s1, sg * c1);
   y[2][1] = tw(y[2][1], h, sg * h);
   y[2][2] = mul_mi<C, INV>(y[2][2]);
   y[2][3] = tw(y[2][3], -h, sg * h);
   y[3][1] = tw(y[3][1], s1, sg * c1);
   y[3][2] = tw(y[3][2], -h, sg * h);
   y[3][3] = tw(y[3][3], -c1, -sg * s1);
#pragma unroll
   for (int k1 = 0; k1 < 4; k1++) {
      C t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      dft4<C, INV>(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
   }
}

template <int R, class C, bool INV> __device__ __forceinline__ void dftr(C *v) {
   if constexpr (R == 2) dft2<C, INV>(v);
   else if constexpr (R == 3) dft3<C, INV>(v);
   else if constexpr (R == 4) dft4<C, INV>(v);
   else if constexpr (R == 5) dft5<C, INV>(v);
   else if constexpr (R == 16) dft16<C, INV>(v);
   else dft8<C, INV>(v);
}

// One stage on one buffer: every thread first reads and transforms all its
// butterflies of the stage (at most PPT values of the L n points per
// thread, PPT * blockDim.x >= n L), the CTA synchronises, then every thread
// writes its results.  Half the shared memory of a ping-pong pair of
// buffers, for one more barrier per stage.
template <int RAD, int L, class C, bool INV, int PPT>
__device__ __forceinline__ void fft_stage_ip(C *buf, int n, int Ns, unsigned magic, const C *__restrict__ tw,
                                             int twmul) {
   constexpr int MAXU = (PPT + RAD - 1) / RAD;  // butterflies per thread
   const int nr = n / RAD;
   const int nb = nr * L;
   const int twstep = (n / (Ns * RAD)) * twmul;
   C v[MAXU][RAD];
#pragma unroll
   for (int u = 0; u < MAXU; u++) {
      const int b = threadIdx.x + u * blockDim.x;
      if (b < nb) {
         const int l = b % L;
         const int j = b / L;
         const int g = Ns == 1 ? j : (int) __umulhi((unsigned) j, magic);
         const int k = j - g * Ns;
         const C *src = buf + j * L + l;
#pragma unroll
         for (int t = 0; t < RAD; t++) v[u][t] = src[t * nr * L];
         if (Ns > 1) {
#pragma unroll
            for (int t = 1; t < RAD; t++) {
               C w = tw[t * k * twstep];
               if (INV) w.y = -w.y;
               v[u][t] = cmul(v[u][t], w);
            }
         }
         dftr<RAD, C, INV>(v[u]);
      }
   }
   __syncthreads();
#pragma unroll
   for (int u = 0; u < MAXU; u++) {
      const int b = threadIdx.x + u * blockDim.x;
      if (b < nb) {
         const int l = b % L;
         const int j = b / L;
         const int g = Ns == 1 ? j : (int) __umulhi((unsigned) j, magic);
         const int k = j - g * Ns;
         C *dst = buf + (g * Ns * RAD + k) * L + l;
#pragma unroll
         for (int t = 0; t < RAD; t++) dst[t * Ns * L] = v[u][t];
      }
   }
   __syncthreads();
}

// Full in-place transform of L interleaved lines in buf (PPT as above).
template <int L, class C, bool INV, int PPT>
__device__ __forceinline__ void fft_lines_ip(C *buf, const FftPlan &pl, const C *tw, int twmul) {
   // make_plan orders the stages by radix (16, 8, 4, 2, 3, 5): one loop per
   // radix (a switch over the radix inside one loop made ptxas spill the
   // values held across the barriers).  Radix 16 only where a thread holds
   // 16 points (PPT >= 16, the FP32 passes).
   int st = 0;
   if constexpr (PPT >= 16)
      for (; st < pl.nst && pl.rad[st] == 16; st++)
         fft_stage_ip<16, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
   for (; st < pl.nst && pl.rad[st] == 8; st++) fft_stage_ip<8, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
   for (; st < pl.nst && pl.rad[st] == 4; st++) fft_stage_ip<4, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
   for (; st < pl.nst && pl.rad[st] == 2; st++) fft_stage_ip<2, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
   for (; st < pl.nst && pl.rad[st] == 3; st++) fft_stage_ip<3, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
   for (; st < pl.nst && pl.rad[st] == 5; st++) fft_stage_ip<5, L, C, INV, PPT>(buf, pl.n, pl.ns[st], pl.magic[st], tw, twmul);
}

}  // namespace gpe
