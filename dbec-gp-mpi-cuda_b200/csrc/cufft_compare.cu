// cufft_compare.cu -- the dipolar convolution phi = IFFT[Udd * FFT[|psi|^2]]
// through cuFFT, kept only as a timed comparison for the project-written FFT
// passes of libgpe.so (which never calls cuFFT).  Built as its own library,
// libgpe_cufft.so, so that the solver does not link cuFFT at all.
//
// Two call structures:
//  variant 0, the reference's (calcpsidd2_mem, imag3d-mpicuda.cu:1460-1510,
//    plans :1092-1126): |psi|^2 into a real buffer, D2Z 2D over (y, z)
//    batched over x, the one-rank "transpose" (a device copy of the whole
//    half spectrum into the transposed buffer, whose layout equals the
//    original's at one rank), one Z2Z 1D execution along x per y (the host
//    loop of :1472-1476, stride ny (nz/2+1), batch nz/2+1), the Udd multiply,
//    the inverse host loop, the copy back, Z2D and the boundary planes;
//  variant 1, the library at its best: the same without the copies, and one
//    batched Z2Z plan along x over all (y, kz) lines per direction.
// FP64 grids use D2Z/Z2Z/Z2D, mixed-precision grids R2C/C2C/C2R.  Udd is the
// same octant table as the solver's (initpotdd, imag3d-mpicuda.cu:945-980),
// multiplied by a plain elementwise kernel.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <type_traits>
#include <string>
#include <vector>

#include "gpe.h"
#include "gpe_cufft.h"

namespace {

thread_local std::string g_cerr;

gpe_status cfail(gpe_status st, const std::string &m) {
   g_cerr = m;
   return st;
}

const char *cufft_name(cufftResult r) {
   switch (r) {
   case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
   case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
   case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
   case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
   case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
   default: return "cufft error";
   }
}

#define CC(call)                                                                                          \
   do {                                                                                                   \
      cudaError_t e_ = (call);                                                                            \
      if (e_ != cudaSuccess) {                                                                            \
         (void) cudaGetLastError();                                                                       \
         return cfail(e_ == cudaErrorMemoryAllocation ? GPE_ERR_OOM : GPE_ERR_CUDA,                       \
                      std::string(#call) + ": " + cudaGetErrorString(e_));                                 \
      }                                                                                                   \
   } while (0)
#define CF(call)                                                                                          \
   do {                                                                                                   \
      cufftResult r_ = (call);                                                                            \
      if (r_ != CUFFT_SUCCESS) return cfail(GPE_ERR_CUDA, std::string(#call) + ": " + cufft_name(r_));    \
   } while (0)

cufftResult exec_r2c(cufftHandle p, double *i, cufftDoubleComplex *o) { return cufftExecD2Z(p, i, o); }
cufftResult exec_r2c(cufftHandle p, float *i, cufftComplex *o) { return cufftExecR2C(p, i, o); }
cufftResult exec_c2r(cufftHandle p, cufftDoubleComplex *i, double *o) { return cufftExecZ2D(p, i, o); }
cufftResult exec_c2r(cufftHandle p, cufftComplex *i, float *o) { return cufftExecC2R(p, i, o); }
cufftResult exec_c2c(cufftHandle p, cufftDoubleComplex *i, cufftDoubleComplex *o, int dir) {
   return cufftExecZ2Z(p, i, o, dir);
}
cufftResult exec_c2c(cufftHandle p, cufftComplex *i, cufftComplex *o, int dir) { return cufftExecC2C(p, i, o, dir); }

// |psi|^2 (calcpsi2_kernel, imag3d-mpicuda.cu:1168; real3d-mpicuda.cu:1277)
template <class R, int E>
__global__ void k_dens(const R *__restrict__ psi, R *__restrict__ rho, long long n) {
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < n; q += (long long) gridDim.x * blockDim.x) {
      if (E == 1) {
         const R v = psi[q];
         rho[q] = v * v;
      } else {
         const R a = psi[2 * q], b = psi[2 * q + 1];
         rho[q] = a * a + b * b;
      }
   }
}

// spec[x][y][kz] *= Udd(|kx|, |ky|, kz) (calcpsidd2_kernel1, imag3d-mpicuda.cu:1571)
template <class R, class C>
__global__ void k_udd(C *__restrict__ spec, const double *__restrict__ udd, int nx, int ny, int nzh) {
   const long long n = (long long) nx * ny * nzh;
   const int nyh = ny / 2 + 1;
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < n; q += (long long) gridDim.x * blockDim.x) {
      const int k = (int) (q % nzh);
      const long long r = q / nzh;
      const int y = (int) (r % ny), x = (int) (r / ny);
      const int ax = x <= nx / 2 ? x : nx - x, ay = y <= ny / 2 ? y : ny - y;
      const R u = (R) udd[((long long) ax * nyh + ay) * nzh + k];
      C v = spec[q];
      v.x *= u;
      v.y *= u;
      spec[q] = v;
   }
}

// Boundary planes of phi at one rank (calcpsidd2_kernel2a/2b,
// imag3d-mpicuda.cu:1591-1625); the read and write sets are disjoint.
template <class R>
__global__ void k_planes(R *__restrict__ phi, int nx, int ny, int nz) {
   const long long nyz = (long long) ny * nz;
   const long long nxpl = (long long) (ny - 1) * (nz - 1);   // x = nx-1 plane
   const long long nypl = (long long) (nx - 1) * (nz - 1);   // y = ny-1 plane
   const long long nzpl = (long long) (nx - 1) * (ny - 1);   // z = nz-1 plane
   const long long tot = nxpl + nypl + nzpl;
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < tot; q += (long long) gridDim.x * blockDim.x) {
      if (q < nxpl) {
         const long long j = q / (nz - 1), k = q % (nz - 1);
         phi[(nx - 1) * nyz + j * nz + k] = phi[j * nz + k];
      } else if (q < nxpl + nypl) {
         const long long e = q - nxpl, i = e / (nz - 1), k = e % (nz - 1);
         phi[i * nyz + (long long) (ny - 1) * nz + k] = phi[i * nyz + k];
      } else {
         const long long e = q - nxpl - nypl, i = e / (ny - 1), j = e % (ny - 1);
         phi[i * nyz + j * nz + nz - 1] = phi[i * nyz + j * nz];
      }
   }
}

// initpotdd on the octant |kx| <= nx/2, |ky| <= ny/2, kz <= nz/2, with the
// reference's truncated pi (imag3d-mpicuda.cu:69, 945-980).
std::vector<double> udd_octant(const gpe_params *p) {
   const double pi = 3.14159265358979;
   const long nx = p->nx, ny = p->ny, nz = p->nz, nxh = nx / 2 + 1, nyh = ny / 2 + 1, nzh = nz / 2 + 1;
   const double dkx = 2. * pi / (nx * p->dx), dky = 2. * pi / (ny * p->dy), dkz = 2. * pi / (nz * p->dz);
   const double R = p->cutoff;
   std::vector<double> u((size_t) (nxh * nyh * nzh));
   for (long i = 0; i < nxh; i++)
      for (long j = 0; j < nyh; j++)
         for (long k = 0; k < nzh; k++) {
            const double kx = i * dkx, ky = j * dky, kz = k * dkz;
            const double kx2 = kx * kx, ky2 = ky * ky, kz2 = kz * kz;
            const double xk = std::sqrt(kz2 + kx2 + ky2);
            const double tmp = 1. + 3. * std::cos(xk * R) / (xk * xk * R * R) - 3. * std::sin(xk * R) / (xk * xk * xk * R * R * R);
            u[(size_t) ((i * nyh + j) * nzh + k)] = (4. * pi * (3. * kz2 / (kx2 + ky2 + kz2) - 1.) / 3.) * tmp;
         }
   u[0] = 0.;
   return u;
}

template <class R> struct Bufs {
   using C = typename std::conditional<sizeof(R) == 8, cufftDoubleComplex, cufftComplex>::type;
   R *psi = nullptr, *rho = nullptr, *phi = nullptr;
   C *spec = nullptr, *specT = nullptr;
   double *udd = nullptr;
   cufftHandle fr = 0, br = 0, fx = 0;
   bool have_fr = false, have_br = false, have_fx = false;
   cudaStream_t st = nullptr;
   cudaEvent_t a = nullptr, b = nullptr;
   ~Bufs() {
      if (have_fr) cufftDestroy(fr);
      if (have_br) cufftDestroy(br);
      if (have_fx) cufftDestroy(fx);
      void *ptrs[] = {psi, rho, phi, spec, specT, udd};
      for (void *q : ptrs)
         if (q) cudaFree(q);
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
      if (st) cudaStreamDestroy(st);
   }
};

template <class R>
gpe_status run(const gpe_params *p, const double *psi_h, int variant, int nrep, double *phi_h, double *ms) {
   using B = Bufs<R>;
   using C = typename B::C;
   constexpr cufftType R2C = sizeof(R) == 8 ? CUFFT_D2Z : CUFFT_R2C;
   constexpr cufftType C2R = sizeof(R) == 8 ? CUFFT_Z2D : CUFFT_C2R;
   constexpr cufftType C2C = sizeof(R) == 8 ? CUFFT_Z2Z : CUFFT_C2C;
   B b;
   const int nx = (int) p->nx, ny = (int) p->ny, nz = (int) p->nz, nzh = nz / 2 + 1;
   const long long npts = (long long) nx * ny * nz, nspec = (long long) nx * ny * nzh;
   const int E = p->mode == GPE_MODE_REAL ? 2 : 1;
   if (p->device >= 0) CC(cudaSetDevice(p->device));
   CC(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
   CC(cudaEventCreate(&b.a));
   CC(cudaEventCreate(&b.b));
   CC(cudaMalloc(&b.psi, sizeof(R) * E * npts));
   CC(cudaMalloc(&b.rho, sizeof(R) * npts));
   CC(cudaMalloc(&b.phi, sizeof(R) * npts));
   CC(cudaMalloc(&b.spec, sizeof(C) * nspec));
   if (variant == 0) CC(cudaMalloc(&b.specT, sizeof(C) * nspec));
   {
      std::vector<R> h((size_t) (E * npts));
      for (size_t q = 0; q < h.size(); q++) h[q] = (R) psi_h[q];
      CC(cudaMemcpy(b.psi, h.data(), sizeof(R) * h.size(), cudaMemcpyHostToDevice));
      const std::vector<double> u = udd_octant(p);
      CC(cudaMalloc(&b.udd, sizeof(double) * u.size()));
      CC(cudaMemcpy(b.udd, u.data(), sizeof(double) * u.size(), cudaMemcpyHostToDevice));
   }
   // plans (imag3d-mpicuda.cu:1092-1126): 2D (y, z) batched over x, and the
   // x transform with stride ny * nzh over the (y, kz) lines
   int n2[2] = {ny, nz};
   int inr[2] = {ny, nz}, onc[2] = {ny, nzh};
   CF(cufftPlanMany(&b.fr, 2, n2, inr, 1, ny * nz, onc, 1, ny * nzh, R2C, nx));
   b.have_fr = true;
   CF(cufftPlanMany(&b.br, 2, n2, onc, 1, ny * nzh, inr, 1, ny * nz, C2R, nx));
   b.have_br = true;
   int n1[1] = {nx}, emb[1] = {nx};
   const int xbatch = variant == 0 ? nzh : ny * nzh;
   CF(cufftPlanMany(&b.fx, 1, n1, emb, ny * nzh, 1, emb, ny * nzh, 1, C2C, xbatch));
   b.have_fx = true;
   CF(cufftSetStream(b.fr, b.st));
   CF(cufftSetStream(b.br, b.st));
   CF(cufftSetStream(b.fx, b.st));
   const unsigned grid = 148 * 8;
   auto conv = [&]() -> gpe_status {
      if (E == 1) k_dens<R, 1><<<grid, 256, 0, b.st>>>(b.psi, b.rho, npts);
      else k_dens<R, 2><<<grid, 256, 0, b.st>>>(b.psi, b.rho, npts);
      CC(cudaGetLastError());
      CF(exec_r2c(b.fr, b.rho, b.spec));
      C *xs = b.spec;
      if (variant == 0) {
         CC(cudaMemcpyAsync(b.specT, b.spec, sizeof(C) * nspec, cudaMemcpyDeviceToDevice, b.st));
         xs = b.specT;
         for (int y = 0; y < ny; y++) CF(exec_c2c(b.fx, xs + (long long) y * nzh, xs + (long long) y * nzh, CUFFT_FORWARD));
      } else {
         CF(exec_c2c(b.fx, xs, xs, CUFFT_FORWARD));
      }
      k_udd<R, C><<<grid, 256, 0, b.st>>>(xs, b.udd, nx, ny, nzh);
      CC(cudaGetLastError());
      if (variant == 0) {
         for (int y = 0; y < ny; y++) CF(exec_c2c(b.fx, xs + (long long) y * nzh, xs + (long long) y * nzh, CUFFT_INVERSE));
         CC(cudaMemcpyAsync(b.spec, b.specT, sizeof(C) * nspec, cudaMemcpyDeviceToDevice, b.st));
      } else {
         CF(exec_c2c(b.fx, xs, xs, CUFFT_INVERSE));
      }
      CF(exec_c2r(b.br, b.spec, b.phi));
      k_planes<R><<<grid, 256, 0, b.st>>>(b.phi, nx, ny, nz);
      CC(cudaGetLastError());
      return GPE_OK;
   };
   gpe_status s = conv();  // warm-up (plan work areas, module loading)
   if (s != GPE_OK) return s;
   CC(cudaEventRecord(b.a, b.st));
   for (int r = 0; r < nrep && s == GPE_OK; r++) s = conv();
   if (s != GPE_OK) return s;
   CC(cudaEventRecord(b.b, b.st));
   CC(cudaEventSynchronize(b.b));
   float f = 0.f;
   CC(cudaEventElapsedTime(&f, b.a, b.b));
   if (ms) *ms = f / nrep;
   if (phi_h) {
      std::vector<R> h((size_t) npts);
      CC(cudaMemcpyAsync(h.data(), b.phi, sizeof(R) * npts, cudaMemcpyDeviceToHost, b.st));
      CC(cudaStreamSynchronize(b.st));
      for (size_t q = 0; q < h.size(); q++) phi_h[q] = h[q];
   }
   return GPE_OK;
}

}  // namespace

extern "C" gpe_status gpe_cufft_convolution(const gpe_params *p, const double *psi, int variant, int nrep,
                                            double *phi, double *ms) {
   if (!p || !psi) return cfail(GPE_ERR_PARAM, "null parameters or psi");
   if (variant != 0 && variant != 1) return cfail(GPE_ERR_PARAM, "variant must be 0 or 1");
   if (nrep < 1) return cfail(GPE_ERR_PARAM, "nrep must be >= 1");
   if (p->nx < 4 || p->ny < 4 || p->nz < 4 || p->nx > 4096 || p->ny > 4096 || p->nz > 4096 || p->nx % 2 || p->ny % 2 ||
       p->nz % 2)
      return cfail(GPE_ERR_PARAM, "grid sizes must be even, in [4, 4096]");
   if (p->mode != GPE_MODE_IMAG && p->mode != GPE_MODE_REAL) return cfail(GPE_ERR_PARAM, "mode must be 0 or 1");
   return p->precision == GPE_PREC_MIXED ? run<float>(p, psi, variant, nrep, phi, ms)
                                         : run<double>(p, psi, variant, nrep, phi, ms);
}

extern "C" const char *gpe_cufft_last_error(void) { return g_cerr.c_str(); }
