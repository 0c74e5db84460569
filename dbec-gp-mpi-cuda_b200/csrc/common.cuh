// common.cuh -- element types, complex helpers and the Simpson accumulator
// shared by every kernel of the B200 dipolar GP solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gpe {

template <class R> struct vec2;
template <> struct vec2<double> { using type = double2; };
template <> struct vec2<float> { using type = float2; };

template <class R> using cpx = typename vec2<R>::type;

template <class R> __host__ __device__ __forceinline__ cpx<R> mk(R x, R y) { cpx<R> r; r.x = x; r.y = y; return r; }
template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
   C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <class C> __host__ __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
template <class C, class S> __host__ __device__ __forceinline__ C cscale(C a, S s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
// Complex float adds, subtracts and real scalings as one packed two-lane
// FP32 instruction each on sm_100 (PTX add/sub/mul.rn.f32x2, each lane
// rounded as the scalar instruction rounds it; the compiler no longer fuses
// such a multiply with a following add, which moves FP32 results by a last
// bit), and a complex product as a packed multiply and a packed
// multiply-add.  The FP32 FFT stages are mostly such operations and are
// bound by instruction issue (mixed 256^3 step 0.439 -> 0.428 ms for the
// adds, subtracts and scalings, 0.415 -> 0.411 ms for the products).
__device__ __forceinline__ unsigned long long f2_pack(float2 v) {
   unsigned long long r;
   asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
   return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r) {
   float2 v;
   asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
   return v;
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
   unsigned long long r;
   asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
   return f2_unpack(r);
#else
   return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
   unsigned long long r;
   asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
   return f2_unpack(r);
#else
   return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
#ifdef __CUDA_ARCH__
   unsigned long long r;
   asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(make_float2(s, s))));
   return f2_unpack(r);
#else
   return make_float2(a.x * s, a.y * s);
#endif
}

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
#ifdef __CUDA_ARCH__
   // (a.x b.x, a.x b.y) + (-a.y b.y, a.y b.x)
   unsigned long long t, r;
   asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(f2_pack(make_float2(a.x, a.x))), "l"(f2_pack(b)));
   asm("fma.rn.f32x2 %0, %1, %2, %3;"
       : "=l"(r)
       : "l"(f2_pack(make_float2(-a.y, a.y))), "l"(f2_pack(make_float2(b.y, b.x))), "l"(t));
   return f2_unpack(r);
#else
   return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
#endif
}

// multiply by -i (forward) or +i (inverse)
template <class C, bool INV> __host__ __device__ __forceinline__ C mul_mi(C a) {
   C r;
   if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
   return r;
}

// generic add/sub over real and complex psi elements
__host__ __device__ __forceinline__ double cadd_any(double a, double b) { return a + b; }
__host__ __device__ __forceinline__ float cadd_any(float a, float b) { return a + b; }
__host__ __device__ __forceinline__ double2 cadd_any(double2 a, double2 b) { return cadd(a, b); }
__host__ __device__ __forceinline__ float2 cadd_any(float2 a, float2 b) { return cadd(a, b); }
__host__ __device__ __forceinline__ double csub_any(double a, double b) { return a - b; }
__host__ __device__ __forceinline__ float csub_any(float a, float b) { return a - b; }
__host__ __device__ __forceinline__ double2 csub_any(double2 a, double2 b) { return csub(a, b); }
__host__ __device__ __forceinline__ float2 csub_any(float2 a, float2 b) { return csub(a, b); }

// warp shuffles of real or complex elements
__device__ __forceinline__ double shfl_down_any(unsigned m, double v, int d) { return __shfl_down_sync(m, v, d); }
__device__ __forceinline__ float shfl_down_any(unsigned m, float v, int d) { return __shfl_down_sync(m, v, d); }
__device__ __forceinline__ double2 shfl_down_any(unsigned m, double2 v, int d) {
   return make_double2(__shfl_down_sync(m, v.x, d), __shfl_down_sync(m, v.y, d));
}
__device__ __forceinline__ float2 shfl_down_any(unsigned m, float2 v, int d) {
   return make_float2(__shfl_down_sync(m, v.x, d), __shfl_down_sync(m, v.y, d));
}
__device__ __forceinline__ double shfl_up_any(unsigned m, double v, int d) { return __shfl_up_sync(m, v, d); }
__device__ __forceinline__ float shfl_up_any(unsigned m, float v, int d) { return __shfl_up_sync(m, v, d); }
__device__ __forceinline__ double2 shfl_up_any(unsigned m, double2 v, int d) {
   return make_double2(__shfl_up_sync(m, v.x, d), __shfl_up_sync(m, v.y, d));
}
__device__ __forceinline__ float2 shfl_up_any(unsigned m, float2 v, int d) {
   return make_float2(__shfl_up_sync(m, v.x, d), __shfl_up_sync(m, v.y, d));
}

// psi element: real R in imaginary time, complex in real time
template <class R, bool CPLX> struct psi_elem { using type = R; };
template <class R> struct psi_elem<R, true> { using type = cpx<R>; };

template <class R> __device__ __forceinline__ R dens(R v) { return v * v; }
template <class R> __device__ __forceinline__ R dens(typename vec2<R>::type v) { return v.x * v.x + v.y * v.y; }
__device__ __forceinline__ double dens2(double v) { return v * v; }
__device__ __forceinline__ double dens2(double2 v) { return v.x * v.x + v.y * v.y; }
__device__ __forceinline__ float dens2(float v) { return v * v; }
__device__ __forceinline__ float dens2(float2 v) { return v.x * v.x + v.y * v.y; }

__device__ __forceinline__ double scl(double v, double s) { return v * s; }
__device__ __forceinline__ double2 scl(double2 v, double s) { return make_double2(v.x * s, v.y * s); }
__device__ __forceinline__ float scl(float v, double s) { return (float) (v * s); }
__device__ __forceinline__ float2 scl(float2 v, double s) { return make_float2((float) (v.x * s), (float) (v.y * s)); }

template <class T> __device__ __forceinline__ T zero_of();
template <> __device__ __forceinline__ double zero_of<double>() { return 0.; }
template <> __device__ __forceinline__ float zero_of<float>() { return 0.f; }
template <> __device__ __forceinline__ double2 zero_of<double2>() { return make_double2(0., 0.); }
template <> __device__ __forceinline__ float2 zero_of<float2>() { return make_float2(0.f, 0.f); }

// Composite Simpson rule accumulated while walking a line in index order,
// with the reference's three partial sums and end correction
// (src/utils/diffint.cu:37-66): odd samples (sumi), the even sample before
// each odd one (sumj) and the even sample after it (sumk).
struct Simpson {
   double si, sj, sk, f1, f2, f3;  // f1 = f[N-1] candidate chain
   long n;
   __host__ __device__ __forceinline__ void init(long N) { si = sj = sk = f1 = f2 = f3 = 0.; n = N; }
   __host__ __device__ __forceinline__ void add(long k, double f) {
      if (k & 1) {
         if (k < n - 1) si += f;
      } else {
         if (k < n - 2) sj += f;
         if (k >= 2) sk += f;
      }
      f3 = f2; f2 = f1; f1 = f;
   }
   // after add() was called for k = 0..N-1 in order
   __host__ __device__ __forceinline__ double finish(double h) const {
      double sum = sj + 4. * si + sk;
      if (n % 2 == 0) sum += (5. * f1 + 8. * f2 - f3) / 4.;
      return sum * h / 3.;
   }
};

// Weight of sample k in simpint over N samples (src/utils/diffint.cu:37-66),
// in units of h/3: 1, 4, 2, ..., 4, 1 over the first odd count of samples,
// plus the end correction (5 f[N-1] + 8 f[N-2] - f[N-3]) / 4 for even N.
__host__ __device__ __forceinline__ double simp_w(int k, int N) {
   const int mm = (N & 1) ? N : N - 1;
   double w = k < mm ? ((k == 0 || k == mm - 1) ? 1. : ((k & 1) ? 4. : 2.)) : 0.;
   if (!(N & 1)) {
      if (k == N - 1) w += 1.25;
      else if (k == N - 2) w += 2.;
      else if (k == N - 3) w -= 0.25;
   }
   return w;
}

// Simpson over an array in memory, the reference's loop verbatim in order.
__host__ __device__ __forceinline__ double simpint_arr(double h, const double *f, long N, long st = 1) {
   double sumi = 0., sumj = 0., sumk = 0.;
   for (long c = 1; c < N - 1; c += 2) {
      sumi += f[c * st];
      sumj += f[(c - 1) * st];
      sumk += f[(c + 1) * st];
   }
   double sum = sumj + 4. * sumi + sumk;
   if (N % 2 == 0) sum += (5. * f[(N - 1) * st] + 8. * f[(N - 2) * st] - f[(N - 3) * st]) / 4.;
   return sum * h / 3.;
}

}  // namespace gpe
