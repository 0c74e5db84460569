// solver.cu -- handle, tables and the C ABI (include/gpe.h) of the B200
// dipolar Gross-Pitaevskii solver.  Host code only orchestrates; every
// operator on psi runs in the kernels of step_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <type_traits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "gpe.h"
#include "internal.h"
#include "step_kernels.cuh"
#include "sweep_kernels.cuh"
#include "batch_kernels.cuh"

using namespace gpe;

// The reference's truncated pi (imag3d-mpicuda.cu:69).
static const double kRefPi = 3.14159265358979;

static thread_local std::string g_err;

namespace gpe {
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace gpe

static gpe_status fail(gpe_status st, const std::string &msg) {
   g_err = msg;
   return st;
}

// On failure the runtime's last-error slot is cleared so that a non-sticky
// error is reported once, by the call that caused it.
#define CK(call)                                                                                   \
   do {                                                                                           \
      cudaError_t e_ = (call);                                                                    \
      if (e_ != cudaSuccess) {                                                                    \
         (void) cudaGetLastError();                                                               \
         return fail(e_ == cudaErrorMemoryAllocation ? GPE_ERR_OOM : GPE_ERR_CUDA,                \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                          \
      }                                                                                           \
   } while (0)

#define CKL()                                                                                      \
   do {                                                                                           \
      cudaError_t e_ = cudaGetLastError();                                                        \
      if (e_ != cudaSuccess) return fail(GPE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
   } while (0)

#define CKS(expr)                                                                                  \
   do {                                                                                           \
      gpe_status s_ = (expr);                                                                     \
      if (s_ != GPE_OK) return s_;                                                                \
   } while (0)

struct gpe_solver {
   gpe_params p;
   int dev = 0;
   cudaStream_t st = nullptr;
   bool own_stream = false;
   bool cplx = false, fp32 = false;
   Dims d{};
   double par = 1.;
   FftPlan px{}, py{}, ph{};  // x, y lines and half-length z lines
   int LSr = 0, LSo = 0;                  // shared row strides of the z passes
   CUtensorMap tm_spec_y{}, tm_spec_x{};  // spectrum tiles of the y and x passes
   int boxy = 0, nboxy = 1, boxx = 0, nboxx = 1;
   int Ly = 8, Lx = 8;  // kz columns per tile of the y and x passes
   gpe_tuning tune{};   // requested tile configuration (0 = default heuristic)
   // bumped whenever the tiles are planned again (their tables reallocated):
   // batches built over this handle rebuild their descriptors when it moves
   unsigned long long plan_gen = 0;
   size_t esz_psi = 8, esz_c = 16, esz_r = 8;
   void *psi = nullptr, *spec = nullptr, *phi = nullptr;
   void *twx = nullptr, *twy = nullptr, *twz = nullptr;
   double *udd = nullptr;
   void *alpha[3] = {nullptr, nullptr, nullptr}, *gamma[3] = {nullptr, nullptr, nullptr};
   double2 A[3], A0r[3], mA[3];
   double *x2 = nullptr, *y2 = nullptr, *z2 = nullptr;
   float *x2f = nullptr, *y2f = nullptr, *z2f = nullptr;  // FP32 copies (mixed precision)
   void *lin[3] = {nullptr, nullptr, nullptr};  // per-axis trap factors of calcnu, imag (LinPhase)
   double *rowA = nullptr, *rowB = nullptr, *tmp = nullptr, *obs = nullptr;
   double *rms_buf = nullptr;  // rms samples of gpe_run, kRmsSlots x 4 doubles

   long long row_cap = 0;  // doubles in rowA / rowB: the largest of nx*ny, nx*nz, ny*nz
   State *state = nullptr;
   std::vector<double> hx, hy, hz, hx2, hy2, hz2;
   long long launches = 0;
   size_t obs_cap = 0;
   // sweep configuration per axis (x, y: TMA tensor tiles; z: bulk rows)
   struct Sweep {
      int TW = 8, MSEG = 8, boxn = 0, nbox = 1, LS = 0, S = 2, ctas = 1;
      size_t smem = 0;
      CUtensorMap tm_psi{}, tm_phi{};
      SegTab tab{};
      void *M = nullptr, *N = nullptr;
      // mixed precision: alpha, gamma, M, N rounded once to FP32 (the values
      // the FP32 sweeps would otherwise round from the FP64 tables at every use)
      void *t32[4] = {nullptr, nullptr, nullptr, nullptr};
   } sw[3];
   double *wz = nullptr;      // Simpson weights along z (norm partials)
   double *wz2 = nullptr;     // wz[k] * z[k]^2 (rms partials)
   int nsm = 148;             // streaming multiprocessors of the device
   uint32_t *err = nullptr;   // device status word (bounded waits)
   // per-kernel profiling: when prof_ev is set, mark() records an event
   // after every kernel of a step
   cudaEvent_t *prof_ev = nullptr;
   int prof_i = 0, prof_cap = 0;
};

// rms samples gpe_run keeps on the device before copying them out (a run with
// more samples copies every full batch of slots while it continues)
constexpr long kRmsSlots = 256;

static void mark(gpe_solver *s) {
   if (s->prof_ev && s->prof_i < s->prof_cap) cudaEventRecord(s->prof_ev[s->prof_i++], s->st);
}

// ---------------------------------------------------------------- planning
// Radices in the order the stages are grouped (fft_lines_ip loops over them
// in this order); max_radix 8, 4 or 2 drops the larger powers of two.  Radix
// 16 is for the FP32 passes only, whose threads hold 16 points.
static bool make_plan(int n, FftPlan &pl, int max_radix = 8) {
   pl.n = n;
   pl.nst = 0;
   int m = n;
   static const int pref[] = {16, 8, 4, 2, 3, 5};
   for (int r : pref) {
      if ((r == 16 || r == 8 || r == 4) && r > max_radix) continue;
      while (m % r == 0 && pl.nst < kMaxStages) { pl.rad[pl.nst++] = r; m /= r; }
   }
   int ns = 1;
   for (int st = 0; st < pl.nst; st++) {
      pl.ns[st] = ns;
      // ceil(2^32 / ns): umulhi(j, magic) == j / ns for j, ns < 2^16; ns = 1 wraps to 0
      pl.magic[st] = ns == 1 ? 0u : (unsigned) ((0x100000000ULL + (unsigned long long) ns - 1) / (unsigned long long) ns);
      ns *= pl.rad[st];
   }
   return m == 1;
}

static gpe_status validate(const gpe_params *p) {
   if (!p) return fail(GPE_ERR_PARAM, "null parameters");
   if (p->mode != GPE_MODE_IMAG && p->mode != GPE_MODE_REAL) return fail(GPE_ERR_PARAM, "mode must be 0 (imag) or 1 (real)");
   if (p->precision != GPE_PREC_FP64 && p->precision != GPE_PREC_MIXED) return fail(GPE_ERR_PARAM, "precision must be 0 or 1");
   const long n[3] = {p->nx, p->ny, p->nz};
   for (int a = 0; a < 3; a++) {
      if (n[a] < 8 || n[a] > 1024) return fail(GPE_ERR_PARAM, "grid sizes must be in [8, 1024]");
      if (n[a] % 2) return fail(GPE_ERR_PARAM, "grid sizes must be even (k-grid of initpotdd)");
      FftPlan pl;
      if (!make_plan((int) n[a], pl)) return fail(GPE_ERR_PARAM, "grid sizes must factor into 2, 3 and 5");
   }
   if (!(p->dx > 0 && p->dy > 0 && p->dz > 0 && p->dt > 0)) return fail(GPE_ERR_PARAM, "DX, DY, DZ, DT must be positive");
   if (!(p->cutoff > 0)) return fail(GPE_ERR_PARAM, "CUTOFF must be positive");
   if (p->precision == GPE_PREC_MIXED && p->nz % 4)
      return fail(GPE_ERR_PARAM, "mixed precision needs NZ divisible by 4 (16-byte FP32 rows)");
   return GPE_OK;
}

static size_t psi_esz(const gpe_params *p) {
   size_t r = (p->precision == GPE_PREC_MIXED) ? 4 : 8;
   return p->mode == GPE_MODE_REAL ? 2 * r : r;
}

extern "C" gpe_status gpe_device_bytes(const gpe_params *p, long long *bytes) {
   CKS(validate(p));
   const long long npts = p->nx * p->ny * p->nz;
   const long long nzh = p->nz / 2 + 1;
   const size_t r = (p->precision == GPE_PREC_MIXED) ? 4 : 8;
   long long b = 0;
   b += npts * (long long) psi_esz(p);                   // psi
   const long long nzp = (p->precision == GPE_PREC_MIXED) ? (nzh + 1) & ~1LL : nzh;
   b += nzp * p->nx * p->ny * (long long) (2 * r);       // spectrum (rows padded to 16 bytes)
   b += npts * (long long) r;                            // phi
   b += nzh * (p->nx / 2 + 1) * (p->ny / 2 + 1) * 8;     // Udd octant
   b += 4 * std::max(p->nx * p->ny, std::max(p->nx * p->nz, p->ny * p->nz)) * 8;  // row sums
   b += 1 << 20;                                         // tables, state
   if (bytes) *bytes = b;
   return GPE_OK;
}

// ------------------------------------------------------------------ tables
template <class T> static gpe_status upload(void **dst, const T *src, size_t n) {
   CK(cudaMalloc(dst, sizeof(T) * n));
   CK(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
   return GPE_OK;
}

static gpe_status make_twiddles(gpe_solver *s, int n, void **dst) {
   std::vector<double2> t(n);
   for (int m = 0; m < n; m++) {
      const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double) m / (long double) n;
      t[m] = make_double2((double) cosl(a), (double) sinl(a));
   }
   if (s->fp32) {
      std::vector<float2> f(n);
      for (int m = 0; m < n; m++) f[m] = make_float2((float) t[m].x, (float) t[m].y);
      return upload(dst, f.data(), n);
   }
   return upload(dst, t.data(), n);
}

// gencoef (imag3d-mpicuda.cu:894-931, real3d-mpicuda.cu:991-1035).
static gpe_status make_coef(gpe_solver *s, int ax, long n, double d2) {
   const double c = s->p.dt / d2 / (3. - s->par);
   typedef std::complex<double> Z;
   Z A0, A0r, A, mA;
   if (!s->cplx) {
      A0 = 1. + c; A0r = 1. - c; A = -0.5 * c; mA = -A;
   } else {
      A0 = Z(1., c); A0r = std::conj(A0); A = Z(0., -0.5 * c); mA = Z(0., -A.imag());
   }
   std::vector<Z> al(n - 1), ga(n - 1);
   al[n - 2] = 0.;
   ga[n - 2] = Z(-1.) / A0;
   for (long i = n - 2; i > 0; i--) {
      al[i - 1] = A * ga[i];
      ga[i - 1] = Z(-1.) / (A0 + A * al[i - 1]);
   }
   s->A[ax] = make_double2(A.real(), A.imag());
   s->A0r[ax] = make_double2(A0r.real(), A0r.imag());
   s->mA[ax] = make_double2(mA.real(), mA.imag());
   // uploaded padded to n entries (the last is 0 and never used) so that the
   // sweep kernels can bulk-copy them in 16-byte multiples
   if (!s->cplx) {
      std::vector<double> a(n, 0.), g(n, 0.);
      for (long i = 0; i < n - 1; i++) { a[i] = al[i].real(); g[i] = ga[i].real(); }
      CKS(upload(&s->alpha[ax], a.data(), n));
      CKS(upload(&s->gamma[ax], g.data(), n));
   } else {
      std::vector<double2> a(n, make_double2(0., 0.)), g(n, make_double2(0., 0.));
      for (long i = 0; i < n - 1; i++) {
         a[i] = make_double2(al[i].real(), al[i].imag());
         g[i] = make_double2(ga[i].real(), ga[i].imag());
      }
      CKS(upload(&s->alpha[ax], a.data(), n));
      CKS(upload(&s->gamma[ax], g.data(), n));
   }
   return GPE_OK;
}

// Segment tables of the parallel Thomas sweep of axis ax (line length n,
// segment length m, P segments; the last segment ends at n-3):
//   M[i] = prod_{j=i+1}^{H_p+1} gamma[j] A   for i in segment p < P-1
//   N[k] = prod_{j=lo_p}^{k-1} alpha[j]       for k in (lo_p, hf_p + 1]
// computed in long double and rounded once.
static gpe_status make_segtab(gpe_solver *s, int ax, long n, double d2, int m, int P) {
   // the z sweep's Simpson partials take the weight of a point from its
   // parity within the segment, so segments start at even indices
   if (m % 2) return fail(GPE_ERR_PARAM, "segment length must be even");
   typedef std::complex<long double> Z;
   const long double c = (long double) s->p.dt / (long double) d2 / (3.L - (long double) s->par);
   Z A0, A;
   if (!s->cplx) { A0 = 1.L + c; A = -0.5L * c; }
   else { A0 = Z(1.L, c); A = Z(0.L, -0.5L * c); }
   // coefficients as uploaded (double), promoted: the tables multiply exactly those
   std::vector<Z> al(n - 1), ga(n - 1);
   {
      std::vector<double> ad((size_t) (s->cplx ? 2 : 1) * (n - 1)), gd((size_t) (s->cplx ? 2 : 1) * (n - 1));
      CK(cudaMemcpy(ad.data(), s->alpha[ax], sizeof(double) * ad.size(), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(gd.data(), s->gamma[ax], sizeof(double) * gd.size(), cudaMemcpyDeviceToHost));
      for (long i = 0; i < n - 1; i++) {
         al[i] = s->cplx ? Z(ad[2 * i], ad[2 * i + 1]) : Z(ad[i], 0.L);
         ga[i] = s->cplx ? Z(gd[2 * i], gd[2 * i + 1]) : Z(gd[i], 0.L);
      }
      const double2 Ad = s->A[ax];
      A = Z(Ad.x, Ad.y);
   }
   std::vector<Z> M(n, Z(0)), N(n, Z(0));
   for (int p = 0; p < P; p++) {
      const long lo = (long) p * m;
      const bool top = p == P - 1;
      const long hf = top ? n - 3 : lo + m - 1;
      if (!top) {
         Z r = 1;
         for (long i = hf; i >= lo; i--) { r *= ga[i + 1] * A; M[i] = r; }
      }
      Z r = 1;
      for (long i = lo; i <= hf; i++) { r *= al[i]; N[i + 1] = r; }
   }
   if (!s->cplx) {
      std::vector<double> a(n), b(n);
      for (long i = 0; i < n; i++) { a[i] = (double) M[i].real(); b[i] = (double) N[i].real(); }
      CKS(upload(&s->sw[ax].M, a.data(), n));
      CKS(upload(&s->sw[ax].N, b.data(), n));
   } else {
      std::vector<double2> a(n), b(n);
      for (long i = 0; i < n; i++) {
         a[i] = make_double2((double) M[i].real(), (double) M[i].imag());
         b[i] = make_double2((double) N[i].real(), (double) N[i].imag());
      }
      CKS(upload(&s->sw[ax].M, a.data(), n));
      CKS(upload(&s->sw[ax].N, b.data(), n));
   }
   SegTab &t = s->sw[ax].tab;
   t.al = s->alpha[ax];
   t.ga = s->gamma[ax];
   t.M = s->sw[ax].M;
   t.N = s->sw[ax].N;
   if (s->fp32) {
      // FP32 copies of the FP64 tables (alpha and gamma stay FP64 in HBM as
      // computed; the FP32 kernels read these once-rounded copies).  In real
      // time the gamma copy holds gamma + 1 (SegOps::back_step): gamma is -1
      // plus a small number, which FP32 keeps to its own relative precision.
      const void *src[4] = {s->alpha[ax], s->gamma[ax], s->sw[ax].M, s->sw[ax].N};
      const size_t nd = (size_t) n * (s->cplx ? 2 : 1);
      std::vector<double> h(nd);
      std::vector<float> f(nd);
      for (int q = 0; q < 4; q++) {
         if (s->sw[ax].t32[q]) cudaFree(s->sw[ax].t32[q]);
         s->sw[ax].t32[q] = nullptr;
         CK(cudaMemcpy(h.data(), src[q], sizeof(double) * nd, cudaMemcpyDeviceToHost));
         const bool shift = q == 1 && s->cplx;
         for (size_t e = 0; e < nd; e++) f[e] = (float) (shift && e % 2 == 0 ? h[e] + 1. : h[e]);
         CKS(upload(&s->sw[ax].t32[q], f.data(), nd));
      }
      t.al = s->sw[ax].t32[0];
      t.ga = s->sw[ax].t32[1];
      t.M = s->sw[ax].t32[2];
      t.N = s->sw[ax].t32[3];
   }
   t.A = s->A[ax];
   t.A0r = s->A0r[ax];
   t.mA = s->mA[ax];
   t.n = (int) n;
   t.m = m;
   t.P = P;
   return GPE_OK;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static gpe_status encoder(EncodeTiledFn *fn) {
   static EncodeTiledFn cached = nullptr;
   if (!cached) {
      void *f = nullptr;
      cudaDriverEntryPointQueryResult q;
      CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
      if (!f || q != cudaDriverEntryPointSuccess) return fail(GPE_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
      cached = (EncodeTiledFn) f;
   }
   *fn = cached;
   return GPE_OK;
}

// 3D tensor map over a [nx][ny][w * nz] array of `esz`-byte scalars with box
// {bw, by, bx} (innermost first).
// Rows are `pitch` elements apart (pitch = w_nz when 0).
static gpe_status make_tmap(CUtensorMap *m, void *base, size_t esz, long w_nz, long ny, long nx, int bw, int by, int bx,
                            long pitch = 0) {
   EncodeTiledFn enc;
   CKS(encoder(&enc));
   if (pitch == 0) pitch = w_nz;
   cuuint64_t dims[3] = {(cuuint64_t) w_nz, (cuuint64_t) ny, (cuuint64_t) nx};
   cuuint64_t strides[2] = {(cuuint64_t) (pitch * esz), (cuuint64_t) (pitch * esz * ny)};
   cuuint32_t box[3] = {(cuuint32_t) bw, (cuuint32_t) by, (cuuint32_t) bx};
   cuuint32_t es[3] = {1, 1, 1};
   CUresult r = enc(m, esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims,
                    strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
   if (r != CUDA_SUCCESS) return fail(GPE_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int) r) + ")");
   return GPE_OK;
}

// Candidates (lines per CTA TW, segment length MSEG, segments P) for a sweep
// over lines of length n, widest tile first: TW from `tw_base` (a 128-byte
// row) down to 2, and for each TW every segment length with at most 256
// threads (TW * P), shortest first; prim[c] marks the shortest segment of
// each TW (the most threads), the built-in choice.  Lines of 16-byte elements
// keep 8-point segments (16 would spill registers); 4-byte elements may use
// 32-point segments, which keep 64-byte tile rows on 512-point lines.
constexpr int kSweepCand = 16;
static int sweep_candidates(int n, int tw_base, int esz, int *TW, int *MSEG, int *P, bool *prim) {
   const bool wide = esz == 16;
   const int ms[3] = {8, 16, 32};
   const int nms = wide ? 1 : (esz == 4 ? 3 : 2);
   int k = 0;
   for (int tw = tw_base; tw >= 2 && k < kSweepCand; tw /= 2) {
      bool first = true;
      for (int mi = 0; mi < nms && k < kSweepCand; mi++) {
         const int p = (n - 2 + ms[mi] - 1) / ms[mi];
         if (tw * p <= 256) {
            TW[k] = tw; MSEG[k] = ms[mi]; P[k] = p; prim[k] = first;
            first = false;
            k++;
         }
      }
   }
   if (k == 0) {
      TW[0] = 2; MSEG[0] = wide ? 8 : 16; P[0] = (n - 2 + MSEG[0] - 1) / MSEG[0]; prim[0] = true;
      k = 1;
   }
   return k;
}

// Tile configuration of the sweeps and of the y / x FFT passes, and the FFT
// plans: the heuristics below, or the values of s->tune where set.  May be
// called again (gpe_set_tuning); it reuploads only the segment tables.
static gpe_status plan_tiles(gpe_solver *s) {
   s->plan_gen++;
   const Dims &d = s->d;
   const size_t esz = s->esz_psi, rsz = s->esz_r;
   const int E = s->cplx ? 2 : 1;
   const int tw_base = (int) (128 / esz);
   const long nn[3] = {d.nx, d.ny, d.nz};
   const double h2[3] = {s->p.dx * s->p.dx, s->p.dy * s->p.dy, s->p.dz * s->p.dz};
   const size_t sm_cap = 227 * 1024;
   for (int ax = 0; ax < 3; ax++) {
      auto &w = s->sw[ax];
      // the widest tile for which as many CTAs as the kernels are compiled for
      // fit on an SM with a 2-stage pipeline (else the widest tile, fewer CTAs)
      const int max_ctas = kSweepCtas[ax == 0 ? 1 : 0];
      int cTW[kSweepCand], cM[kSweepCand], cP[kSweepCand];
      bool prim[kSweepCand];
      const int nc = sweep_candidates((int) nn[ax], tw_base, (int) esz, cTW, cM, cP, prim);
      auto sizes = [&](int TW, int P, size_t &stage, size_t &fixed) {
         const int spw = 32 / TW;
         const size_t blk = 2 * (size_t) ((P + spw - 1) / spw + 1) * TW * esz;
         if (ax < 2) {
            const long rows = (long) std::min<long>(nn[ax], 256) * ((nn[ax] + 255) / 256);
            stage = (rows * TW * esz + (ax == 0 ? rows * TW * rsz : 0) + 127) & ~(size_t) 127;
            // FP64 x sweep: calcnu's per-x table staged in shared memory
            fixed = 128 + blk + (ax == 0 && !s->fp32 ? (size_t) nn[0] * (s->cplx ? 16 : 8) : 0);
         } else {
            stage = ((size_t) TW * (d.nz + 16 / esz) * esz + 127) & ~(size_t) 127;
            // FP64: the four coefficient tables staged in shared memory
            fixed = 128 + blk + 2 * (size_t) P * TW * sizeof(double) +
                    (s->fp32 ? 0 : 4 * (size_t) nn[2] * (s->cplx ? 16 : 8));
         }
      };
      auto fits = [&](int c) {
         size_t st_, fx_;
         sizes(cTW[c], cP[c], st_, fx_);
         return (fx_ + 2 * st_) * max_ctas <= sm_cap;
      };
      const int want_tw = s->tune.sweep_tw[ax], want_ms = s->tune.sweep_seg[ax];
      // a candidate matching the fields that are set (an unset segment
      // length means the shortest of that TW; an unset TW the widest tile
      // that fits, else the widest)
      auto match = [&](int c) { return (want_tw <= 0 || cTW[c] == want_tw) && (want_ms <= 0 ? prim[c] : cM[c] == want_ms); };
      int pick = -1;
      if (want_tw > 0 || want_ms > 0) {
         for (int c = 0; c < nc && pick < 0; c++)
            if (match(c) && (want_tw > 0 || fits(c))) pick = c;
         for (int c = 0; c < nc && pick < 0; c++)
            if (match(c)) pick = c;
         if (pick < 0) return fail(GPE_ERR_PARAM, "tuning: sweep_tw / sweep_seg not available for this line length");
      } else {
         // FP32 real z lines of 100 points or more: 32-point segments when
         // that leaves at least four per line (128^3 z sweep 20.1 -> 16.6 us
         // on B200; shorter lines, and the x and y sweeps, measured no faster
         // or slower with them solo), on 16-row tiles where those fit (with
         // a 3-stage pipeline, below: mixed 256^3 step 0.4117 -> 0.4088 ms,
         // 512x512x256 1.676 -> 1.666 ms)
         if (ax == 2 && esz == 4) {
            for (int c = 0; c < nc && pick < 0; c++)
               if (cM[c] == 32 && cP[c] >= 4 && cTW[c] == 16 && fits(c)) pick = c;
            for (int c = 0; c < nc && pick < 0; c++)
               if (cM[c] == 32 && cP[c] >= 4 && fits(c)) pick = c;
         }
         for (int c = 0; c < nc && pick < 0; c++)
            if (prim[c] && fits(c)) pick = c;
         if (pick < 0) pick = 0;
      }
      w.TW = cTW[pick];
      w.MSEG = cM[pick];
      const int P = cP[pick];
      if (w.M) cudaFree(w.M);
      if (w.N) cudaFree(w.N);
      w.M = w.N = nullptr;
      CKS(make_segtab(s, ax, nn[ax], h2[ax], w.MSEG, P));
      size_t stage = 0, fixed = 0;
      sizes(w.TW, P, stage, fixed);
      if (ax < 2) {
         w.boxn = (int) std::min<long>(nn[ax], 256);
         w.nbox = (int) ((nn[ax] + w.boxn - 1) / w.boxn);
         const int by = ax == 1 ? w.boxn : 1, bx = ax == 0 ? w.boxn : 1;
         CKS(make_tmap(&w.tm_psi, s->psi, s->fp32 ? 4 : 8, E * d.nz, d.ny, d.nx, E * w.TW, by, bx));
         CKS(make_tmap(&w.tm_phi, s->phi, rsz, d.nz, d.ny, d.nx, w.TW, by, bx));
      } else {
         w.LS = (int) (d.nz + 16 / esz);
      }
      // as many resident CTAs as allowed, then the deepest pipeline (2 or 3
      // stages) that keeps them
      // default depth: 3 for the TMA tensor tiles of the x / y sweeps, 2 for
      // the z sweep's bulk-copied rows (measured faster on B200 at 256^3, both
      // modes)
      // (FP32 real z sweeps on 16-row tiles of 32-point segments: 3)
      const bool z16 = ax == 2 && esz == 4 && w.TW == 16 && w.MSEG == 32;
      const int s_hi = s->tune.sweep_stages[ax] > 0 ? s->tune.sweep_stages[ax] : ((ax == 2 && !z16) ? 2 : 3);
      const int s_lo = s->tune.sweep_stages[ax] > 0 ? s->tune.sweep_stages[ax] : 2;
      if (s_lo < 2 || s_hi > 3) return fail(GPE_ERR_PARAM, "tuning: sweep_stages must be 2 or 3");
      // the register budget of max_ctas CTAs of 256 threads holds more CTAs
      // of fewer threads
      const int thr = (w.TW * P + 31) & ~31;
      const int ct_max = std::min(32, 256 * max_ctas / thr);
      w.ctas = 0;
      for (int ct = ct_max; ct >= 1 && !w.ctas; ct--)
         for (int S = s_hi; S >= s_lo && !w.ctas; S--)
            if ((fixed + S * stage) * ct <= sm_cap) { w.ctas = ct; w.S = S; }
      if (!w.ctas) return fail(GPE_ERR_PARAM, "grid too large for the sweep tiles (shared memory)");
      w.smem = fixed + w.S * stage;
   }
   // spectrum tiles: spec[x][y][kz] viewed as [nx][ny][2 nzh] scalars; L kz
   // columns (at most a 128-byte row) per tile, halved (down to 2) until a
   // tile of a whole line holds at most 256 PPT points (32 KB), the in-place
   // FFT's register budget; the CTA has one thread per PPT points of its tile
   {
      s->boxy = (int) std::min<long>(d.ny, 256);
      s->nboxy = (d.ny + s->boxy - 1) / s->boxy;
      s->boxx = (int) std::min<long>(d.nx, 256);
      s->nboxx = (d.nx + s->boxx - 1) / s->boxx;
      const long ppt = s->fp32 ? 16 : 8;  // FftL<R>::PPT
      // FP64 starts from 4 columns: on B200 the 128-thread CTAs of 4-column
      // tiles (eight per SM) measured faster than 8-column tiles (four per
      // SM): y pass 60 -> 56 us, 256^3 step 0.870 -> 0.863 ms.  FP32 starts
      // from 8 columns (64-byte rows): mixed 256^3 step 0.412 -> 0.403 ms
      // against 16 columns, 128^3 0.103 -> 0.102 ms, 512x512x256 (8 columns
      // either way) unchanged
      auto pickL = [&](long rows) {
         int L = s->fp32 ? 8 : 4;
         while (L > 2 && rows * L > 256 * ppt) L /= 2;
         return L;
      };
      s->Ly = pickL((long) s->boxy * s->nboxy);
      s->Lx = pickL((long) s->boxx * s->nboxx);
      const long rows[2] = {(long) s->boxy * s->nboxy, (long) s->boxx * s->nboxx};
      int *Ls[2] = {&s->Ly, &s->Lx};
      for (int a = 0; a < 2; a++) {
         const int L = s->tune.fft_tile[a];
         if (L == 0) continue;
         if ((L & (L - 1)) || L < 2 || L > 128 / (int) s->esz_c || rows[a] * L > 256 * ppt)
            return fail(GPE_ERR_PARAM, "tuning: fft_tile must be a power of two, >= 2, at most a 128-byte row and "
                                       "at most 256 PPT points per tile");
         *Ls[a] = L;
      }
      // FP32 passes hold 16 points per thread and default to radix-16 stages
      // (two stages instead of three for 128- and 256-point lines)
      const int mr = s->tune.fft_max_radix > 0 ? s->tune.fft_max_radix : (s->fp32 ? 16 : 8);
      if (mr != 16 && mr != 8 && mr != 4 && mr != 2)
         return fail(GPE_ERR_PARAM, "tuning: fft_max_radix must be 16, 8, 4 or 2");
      if (mr == 16 && !s->fp32) return fail(GPE_ERR_PARAM, "tuning: radix 16 is for mixed precision only");
      make_plan(d.nx, s->px, mr);
      make_plan(d.ny, s->py, mr);
      make_plan(d.nz / 2, s->ph, mr);
      CKS(make_tmap(&s->tm_spec_y, s->spec, rsz, 2 * d.nzh, d.ny, d.nx, 2 * s->Ly, s->boxy, 1, 2 * d.nzp));
      CKS(make_tmap(&s->tm_spec_x, s->spec, rsz, 2 * d.nzh, d.ny, d.nx, 2 * s->Lx, 1, s->boxx, 2 * d.nzp));
   }
   return GPE_OK;
}

// Simpson weights along z and the device status word (once per handle).
static gpe_status setup_static(gpe_solver *s) {
   const Dims &d = s->d;
   // Simpson weights along z: sum_k wz[k] f[k] * dz / 3 equals simpint (diffint.cu:37-66)
   std::vector<double> wz(d.nz, 0.);
   const int N = d.nz, mm = (N % 2) ? N : N - 1;
   for (int k = 0; k < mm; k++) wz[k] = (k == 0 || k == mm - 1) ? 1. : ((k % 2) ? 4. : 2.);
   if (N % 2 == 0) { wz[N - 1] += 5. / 4.; wz[N - 2] += 8. / 4.; wz[N - 3] -= 1. / 4.; }
   void *t = nullptr;
   CKS(upload(&t, wz.data(), wz.size()));
   s->wz = (double *) t;
   std::vector<double> wz2(d.nz);
   for (int k = 0; k < N; k++) {
      const double z = (k - d.nz / 2) * s->p.dz;  // the mesh of initpsi
      wz2[k] = wz[k] * (z * z);
   }
   CKS(upload(&t, wz2.data(), wz2.size()));
   s->wz2 = (double *) t;
   CK(cudaMalloc(&s->err, sizeof(uint32_t)));
   CK(cudaMemset(s->err, 0, sizeof(uint32_t)));
   return GPE_OK;
}

// initpotdd (imag3d-mpicuda.cu:945-980) on the octant |kx| <= nx/2,
// |ky| <= ny/2, kz <= nz/2, stored [|kx|][|ky|][kz]: Udd depends on kx^2,
// ky^2, kz^2 only, and the squares of the reference's negative k values equal
// those of the octant.
static gpe_status make_udd(gpe_solver *s) {
   const long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
   const long nxh = nx / 2 + 1, nyh = ny / 2 + 1, nzh = nz / 2 + 1;
   const double pi = kRefPi, cutoff = s->p.cutoff;
   const double dkx = 2. * pi / (nx * s->p.dx), dky = 2. * pi / (ny * s->p.dy), dkz = 2. * pi / (nz * s->p.dz);
   std::vector<double> kx2(nxh), ky2(nyh), kz2(nzh);
   for (long i = 0; i < nxh; i++) { double k = i * dkx; kx2[i] = k * k; }
   for (long i = 0; i < nyh; i++) { double k = i * dky; ky2[i] = k * k; }
   for (long i = 0; i < nzh; i++) { double k = i * dkz; kz2[i] = k * k; }
   std::vector<double> u((size_t) (nzh * nxh * nyh));
   for (long i = 0; i < nxh; i++)
      for (long j = 0; j < nyh; j++)
         for (long k = 0; k < nzh; k++) {
            const double xk = std::sqrt(kz2[k] + kx2[i] + ky2[j]);
            const double tmp = 1. + 3. * std::cos(xk * cutoff) / (xk * xk * cutoff * cutoff) -
                               3. * std::sin(xk * cutoff) / (xk * xk * xk * cutoff * cutoff * cutoff);
            u[(size_t) ((i * nyh + j) * nzh + k)] = (4. * pi * (3. * kz2[k] / (kx2[i] + ky2[j] + kz2[k]) - 1.) / 3.) * tmp;
         }
   u[0] = 0.;  // imag3d-mpicuda.cu:975-977
   void *dp = nullptr;
   CKS(upload(&dp, u.data(), u.size()));
   s->udd = (double *) dp;
   return GPE_OK;
}

static void free_all(gpe_solver *s) {
   void *ptrs[] = {s->psi, s->spec, s->phi, s->twx, s->twy, s->twz, s->udd, s->x2, s->y2, s->z2, s->x2f, s->y2f, s->z2f,
                   s->rowA, s->rowB, s->tmp, s->obs, s->state, s->rms_buf};
   for (void *q : ptrs)
      if (q) cudaFree(q);
   for (int a = 0; a < 3; a++) {
      if (s->alpha[a]) cudaFree(s->alpha[a]);
      if (s->gamma[a]) cudaFree(s->gamma[a]);
      if (s->sw[a].M) cudaFree(s->sw[a].M);
      if (s->sw[a].N) cudaFree(s->sw[a].N);
      for (void *q : s->sw[a].t32)
         if (q) cudaFree(q);
   }
   if (s->wz) cudaFree(s->wz);
   for (void *q : s->lin)
      if (q) cudaFree(q);
   if (s->wz2) cudaFree(s->wz2);
   if (s->err) cudaFree(s->err);
   if (s->own_stream && s->st) cudaStreamDestroy(s->st);
}

static gpe_status create_impl(const gpe_params *p, void *stream, gpe_solver *s) {
   s->p = *p;
   s->cplx = p->mode == GPE_MODE_REAL;
   s->fp32 = p->precision == GPE_PREC_MIXED;
   s->par = (p->opt == 2) ? 2. : 1.;
   if (p->device >= 0) CK(cudaSetDevice(p->device));
   CK(cudaGetDevice(&s->dev));
   CK(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, s->dev));
   if (stream) {
      s->st = (cudaStream_t) stream;
   } else {
      CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
      s->own_stream = true;
   }
   Dims &d = s->d;
   d.nx = (int) p->nx; d.ny = (int) p->ny; d.nz = (int) p->nz; d.nzh = d.nz / 2 + 1;
   d.nzp = s->fp32 ? (d.nzh + 1) & ~1 : d.nzh;
   d.nxy = (long long) d.nx * d.ny;
   d.npts = d.nxy * d.nz;
   const size_t r = s->fp32 ? 4 : 8;
   s->esz_r = r;
   s->esz_c = 2 * r;
   s->esz_psi = psi_esz(p);
   s->LSr = (int) (d.nz + 16 / s->esz_psi);
   s->LSo = (int) (d.nz + 16 / s->esz_r);

   CK(cudaMalloc(&s->psi, s->esz_psi * d.npts));
   CK(cudaMalloc(&s->spec, s->esz_c * (size_t) d.nzp * d.nxy));
   CK(cudaMalloc(&s->phi, r * d.npts));
   CK(cudaMemset(s->psi, 0, s->esz_psi * d.npts));
   s->row_cap = std::max(d.nxy, std::max((long long) d.nx * d.nz, (long long) d.ny * d.nz));
   CK(cudaMalloc(&s->rowA, sizeof(double) * s->row_cap));
   CK(cudaMalloc(&s->rowB, sizeof(double) * s->row_cap));
   CK(cudaMalloc(&s->tmp, sizeof(double) * std::max<long long>(d.nxy, std::max(d.nx, std::max(d.ny, d.nz))) * 2));
   s->obs_cap = 64;
   CK(cudaMalloc(&s->obs, sizeof(double) * s->obs_cap));
   CK(cudaMalloc(&s->rms_buf, sizeof(double) * 4 * kRmsSlots));
   CK(cudaMalloc(&s->state, sizeof(State)));
   State st0{};
   st0.norm = 1.; st0.scale = 1.; st0.scale2 = 1.;
   CK(cudaMemcpy(s->state, &st0, sizeof(State), cudaMemcpyHostToDevice));

   CKS(make_twiddles(s, d.nx, &s->twx));
   CKS(make_twiddles(s, d.ny, &s->twy));
   CKS(make_twiddles(s, d.nz, &s->twz));
   CKS(make_coef(s, 0, d.nx, p->dx * p->dx));
   CKS(make_coef(s, 1, d.ny, p->dy * p->dy));
   CKS(make_coef(s, 2, d.nz, p->dz * p->dz));
   CKS(make_udd(s));
   CKS(plan_tiles(s));
   CKS(setup_static(s));

   // space mesh (initpsi, imag3d-mpicuda.cu:842-855)
   const long nx2 = d.nx / 2, ny2 = d.ny / 2, nz2 = d.nz / 2;
   s->hx.resize(d.nx); s->hy.resize(d.ny); s->hz.resize(d.nz);
   s->hx2.resize(d.nx); s->hy2.resize(d.ny); s->hz2.resize(d.nz);
   for (long i = 0; i < d.nx; i++) { s->hx[i] = (i - nx2) * p->dx; s->hx2[i] = s->hx[i] * s->hx[i]; }
   for (long j = 0; j < d.ny; j++) { s->hy[j] = (j - ny2) * p->dy; s->hy2[j] = s->hy[j] * s->hy[j]; }
   for (long k = 0; k < d.nz; k++) { s->hz[k] = (k - nz2) * p->dz; s->hz2[k] = s->hz[k] * s->hz[k]; }
   void *t = nullptr;
   CKS(upload(&t, s->hx2.data(), d.nx)); s->x2 = (double *) t;
   CKS(upload(&t, s->hy2.data(), d.ny)); s->y2 = (double *) t;
   CKS(upload(&t, s->hz2.data(), d.nz)); s->z2 = (double *) t;
   if (s->fp32) {
      const std::vector<double> *sq[3] = {&s->hx2, &s->hy2, &s->hz2};
      float **dst[3] = {&s->x2f, &s->y2f, &s->z2f};
      for (int a = 0; a < 3; a++) {
         std::vector<float> f(sq[a]->begin(), sq[a]->end());
         CKS(upload(&t, f.data(), f.size()));
         *dst[a] = (float *) t;
      }
   }
   // trap factors per axis for calcnu: exp(-dt 0.5 par c x^2) in imaginary
   // time; in real time (FP64) the phases exp(-i dt 0.5 par c x^2), stored as
   // (cos, sin) pairs
   if (s->cplx && !s->fp32) {
      const long double hp = 0.5L * (long double) s->par, dt = (long double) p->dt;
      const long double cf[3] = {(long double) p->gamma * p->gamma, (long double) p->nu * p->nu,
                                 (long double) p->lambda * p->lambda};
      const std::vector<double> *sq[3] = {&s->hx2, &s->hy2, &s->hz2};
      for (int a = 0; a < 3; a++) {
         const size_t n = sq[a]->size();
         std::vector<double2> tab(n);
         for (size_t i = 0; i < n; i++) {
            const long double th = -dt * hp * cf[a] * (long double) (*sq[a])[i];
            tab[i] = make_double2((double) cosl(th), (double) sinl(th));
         }
         CKS(upload(&s->lin[a], tab.data(), tab.size()));
      }
   }
   if (!s->cplx) {
      const long double hp = 0.5L * (long double) s->par, dt = (long double) p->dt;
      const long double cf[3] = {(long double) p->gamma * p->gamma, (long double) p->nu * p->nu,
                                 (long double) p->lambda * p->lambda};
      const std::vector<double> *sq[3] = {&s->hx2, &s->hy2, &s->hz2};
      for (int a = 0; a < 3; a++) {
         const size_t n = sq[a]->size();
         std::vector<double> tab(n);
         for (size_t i = 0; i < n; i++) tab[i] = (double) expl(-dt * hp * cf[a] * (long double) (*sq[a])[i]);
         if (s->fp32) {
            std::vector<float> f(tab.begin(), tab.end());
            CKS(upload(&s->lin[a], f.data(), f.size()));
         } else {
            CKS(upload(&s->lin[a], tab.data(), tab.size()));
         }
      }
   }
   CK(cudaDeviceSynchronize());
   return GPE_OK;
}

extern "C" gpe_status gpe_create(const gpe_params *p, void *stream, gpe_solver **out) {
   if (!out) return fail(GPE_ERR_PARAM, "null output handle");
   *out = nullptr;
   CKS(validate(p));
   gpe_solver *s = new gpe_solver();
   gpe_status st = create_impl(p, stream, s);
   if (st != GPE_OK) {
      std::string keep = g_err;
      free_all(s);
      delete s;
      g_err = keep;
      return st;
   }
   *out = s;
   return GPE_OK;
}

extern "C" void gpe_destroy(gpe_solver *s) {
   if (!s) return;
   if (s->st) cudaStreamSynchronize(s->st);
   free_all(s);
   delete s;
}

extern "C" const char *gpe_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------------ launches
static Trap trap_of(const gpe_solver *s) {
   Trap t;
   t.x2 = s->x2; t.y2 = s->y2; t.z2 = s->z2;
   t.x2f = s->x2f; t.y2f = s->y2f; t.z2f = s->z2f;
   t.hp = 0.5 * s->par;
   t.vg2 = s->p.gamma * s->p.gamma;
   t.vn2 = s->p.nu * s->p.nu;
   t.vl2 = s->p.lambda * s->p.lambda;
   return t;
}

static unsigned blocks_for(long long n, int bs) { return (unsigned) ((n + bs - 1) / bs); }

// Launch on the handle's stream with programmatic dependent launch: the
// kernel may be scheduled while its predecessor finishes its last wave (its
// CTAs call pdl_trigger / pdl_wait before touching memory), which hides the
// gap between the kernels of a step (FP64 0.880 -> 0.872 ms real, 0.722 ->
// 0.712 ms imaginary time; mixed precision 0.429 -> 0.415 ms at 256^3 and
// 0.107 -> 0.103 ms at 128^3, 512x512x256 unchanged at 1.69 ms, on B200).
template <class... KP, class... A>
static gpe_status launch_pdl(void (*k)(KP...), dim3 grid, dim3 block, size_t smem, const gpe_solver *s, A... args) {
   cudaLaunchAttribute at[1];
   at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
   at[0].val.programmaticStreamSerializationAllowed = 1;
   cudaLaunchConfig_t cfg{};
   cfg.gridDim = grid;
   cfg.blockDim = block;
   cfg.dynamicSmemBytes = smem;
   cfg.stream = s->st;
   cfg.attrs = at;
   cfg.numAttrs = 1;
   CK(cudaLaunchKernelEx(&cfg, k, ((KP) args)...));
   return GPE_OK;
}

template <class R, bool CPLX> struct Impl {
   using P = typename Tr<R, CPLX>::P;
   using C = cpx<R>;

   static gpe_status smem_attr(const void *f, size_t bytes) {
      if (bytes > 48 * 1024) CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes));
      return GPE_OK;
   }

   // runs f(std::integral_constant<int, v>) for v in {2, 4, 8, 16} (tile
   // widths) or {8, 16, 32} (points per thread)
   template <class F> static gpe_status with_L(int L, F f) {
      if (L == 16) return f(std::integral_constant<int, 16>());
      if (L == 8) return f(std::integral_constant<int, 8>());
      if (L == 4) return f(std::integral_constant<int, 4>());
      return f(std::integral_constant<int, 2>());
   }
   template <class F> static gpe_status with_ppt(int ppt, F f) {
      if (ppt <= 8) return f(std::integral_constant<int, 8>());
      if (ppt <= 16) return f(std::integral_constant<int, 16>());
      return f(std::integral_constant<int, 32>());
   }
   // points per thread of the z passes: (nz/2) L over 256 threads, at least
   // 16 in FP32 (the radix-16 stages need them)
   static int zppt(const gpe_solver *s, int L) {
      const int p = (int) (((s->d.nz / 2) * L + 255) / 256);
      return s->fp32 ? std::max(p, 16) : p;
   }
   // threads of a z inverse pass CTA, and of a forward pass CTA over real
   // rows: PPT points each of the L half-length lines (the forward passes
   // over complex rows keep 256: sized CTAs measured slower there, 101 -> 105
   // us at 256^3 complex FP64)
   static unsigned z_threads(const gpe_solver *s, int L, int ppt) {
      const long t = ((long) (s->d.nz / 2) * L + ppt - 1) / ppt;
      return (unsigned) std::min<long>(256, std::max<long>(32, (t + 31) / 32 * 32));
   }

   // threads of a y / x pass CTA: PPT points each over a tile of rows x L
   // (at most 256: the kernels' register budget)
   static unsigned fft_threads(long rows, int L) {
      const long t = (rows * L + FftL<R>::PPT - 1) / FftL<R>::PPT;
      return (unsigned) std::min<long>(256, std::max<long>(32, (t + 31) / 32 * 32));
   }

   template <bool INV, int L> static gpe_status yfft(gpe_solver *s) {
      const Dims &d = s->d;
      const int nkb = (d.nzh + L - 1) / L;
      const size_t smy = 128 + (size_t) s->boxy * s->nboxy * L * sizeof(C) + d.ny * sizeof(C);
      CKS(smem_attr((const void *) k_yfft<R, INV, L>, smy));
      CKS(launch_pdl(k_yfft<R, INV, L>, (unsigned) (d.nx * nkb), fft_threads(s->boxy * s->nboxy, L), smy, s, s->tm_spec_y, d, s->py,
                     (const C *) s->twy, s->boxy, s->nboxy, s->err));
      CKL();
      mark(s);
      return GPE_OK;
   }

   template <int L> static gpe_status xconv(gpe_solver *s) {
      const Dims &d = s->d;
      const int nkb = (d.nzh + L - 1) / L;
      const size_t sm = 128 + (size_t) s->boxx * s->nboxx * L * sizeof(C) + d.nx * sizeof(C) +
                        (size_t) (d.nx / 2 + 1) * L * sizeof(double);
      CKS(smem_attr((const void *) k_xconv<R, L>, sm));
      CKS(launch_pdl(k_xconv<R, L>, (unsigned) (d.ny * nkb), fft_threads(s->boxx * s->nboxx, L), sm, s, s->tm_spec_x, d, s->px, (const C *) s->twx, s->udd,
                                                                 s->state, s->boxx, s->nboxx, s->err));
      CKL();
      mark(s);
      return GPE_OK;
   }

   // z pass kernels for a tile of L rows
   template <int L> static gpe_status zfwd_L(gpe_solver *s, size_t sm, bool sized) {
      const Dims &d = s->d;
      return with_ppt(zppt(s, L), [&](auto pc) {
         constexpr int PPT = decltype(pc)::value;
         CKS(smem_attr((const void *) k_zfwd<R, CPLX, PPT, L>, sm));
         const unsigned nt = sized ? z_threads(s, L, PPT) : 256u;
         CKS(launch_pdl(k_zfwd<R, CPLX, PPT, L>, blocks_for(d.nxy, L), nt, sm, s, (const P *) s->psi, (C *) s->spec, d,
                        s->ph, (const C *) s->twz, s->LSr, s->err));
         CKL();
         mark(s);
         return GPE_OK;
      });
   }

   template <int L> static gpe_status zinv_L(gpe_solver *s, size_t sm) {
      const Dims &d = s->d;
      return with_ppt(zppt(s, L), [&](auto pc) {
         constexpr int PPT = decltype(pc)::value;
         CKS(smem_attr((const void *) k_zinv<R, PPT, L>, sm));
         CKS(launch_pdl(k_zinv<R, PPT, L>, blocks_for(d.nxy, L), z_threads(s, L, PPT), sm, s, (const C *) s->spec, (R *) s->phi, d, s->ph,
                        (const C *) s->twz, s->LSo, s->err));
         CKL();
         mark(s);
         return GPE_OK;
      });
   }

   // shared memory of the z passes for L rows; the rows per CTA start at the
   // preferred value and halve (down to 4) until the tile fits
   static size_t zfwd_smem(const gpe_solver *s, int L) {
      const Dims &d = s->d;
      return 128 + (size_t) L * s->LSr * sizeof(P) + (size_t) (d.nz / 2) * L * sizeof(C) + d.nz * sizeof(C);
   }
   static size_t zinv_smem(const gpe_solver *s, int L) {
      const Dims &d = s->d;
      const size_t in_el = std::max((size_t) L * d.nzp, ((size_t) L * s->LSo * sizeof(R) + sizeof(C) - 1) / sizeof(C));
      return 128 + ((in_el + 7) & ~(size_t) 7) * sizeof(C) + (size_t) (d.nz / 2) * L * sizeof(C) + d.nz * sizeof(C);
   }
   template <class SM> static int zrows(const gpe_solver *s, int pref, SM smem) {
      int L = pref;
      while (L > 4 && smem(s, L) > 227 * 1024) L /= 2;
      return L;
   }
   template <class F> static gpe_status with_zrows(int L, F f) {
      if (L == 16) return f(std::integral_constant<int, 16>());
      if (L == 8) return f(std::integral_constant<int, 8>());
      return f(std::integral_constant<int, 4>());
   }

   static gpe_status psidd2(gpe_solver *s) {
      const Dims &d = s->d;
      {
         // real rows: 8-row tiles on CTAs sized to them, except FP64 rows
         // shorter than 128 points, which keep 16 rows on 256 threads (sized
         // CTAs of 32 threads measured slower at 64^3: 8.8 -> 10.8 us)
         const bool sized = !CPLX && (sizeof(R) == 4 || d.nz >= 128);
         const int L = zrows(s, (!CPLX && !sized) ? 16 : ZRows<R, CPLX>::fwd, zfwd_smem);
         const size_t sm = zfwd_smem(s, L);
         CKS(with_zrows(L, [&](auto lc) { return zfwd_L<decltype(lc)::value>(s, sm, sized); }));
      }
      CKS(with_L(s->Ly, [&](auto Lc) { return yfft<false, decltype(Lc)::value>(s); }));
      CKS(with_L(s->Lx, [&](auto Lc) { return xconv<decltype(Lc)::value>(s); }));
      CKS(with_L(s->Ly, [&](auto Lc) { return yfft<true, decltype(Lc)::value>(s); }));
      {
         const int L = zrows(s, ZRows<R, CPLX>::inv, zinv_smem);
         const size_t sm = zinv_smem(s, L);
         CKS(with_zrows(L, [&](auto lc) { return zinv_L<decltype(lc)::value>(s, sm); }));
      }
      CKS(launch_pdl(k_phifix<R>, (unsigned) std::max<long>(1, (d.ny - 1) + (d.nx - 1)),
                     (unsigned) std::min<long>(256, std::max<long>(32, (d.nz - 1 + 31) / 32 * 32)), 0, s, (R *) s->phi, d));
      CKL();
      mark(s);
      s->launches += 6;
      return GPE_OK;
   }

   template <int AXIS, bool NU, int MSEG, int S, int TWC> static gpe_status sweep_xy_launch_t(gpe_solver *s, double g, double gd) {
      auto &w = s->sw[AXIS];
      const Dims &d = s->d;
      const void *f = (const void *) k_sweep_xy<R, CPLX, AXIS, NU, MSEG, S, TWC>;
      CKS(smem_attr(f, w.smem));
      const int nzb = (d.nz + w.TW - 1) / w.TW;
      const int ntiles = (AXIS == 0 ? d.ny : d.nx) * nzb;
      const unsigned grid = (unsigned) std::min(ntiles, w.ctas * s->nsm);
      CKS(launch_pdl(k_sweep_xy<R, CPLX, AXIS, NU, MSEG, S, TWC>, grid, ((w.TW * w.tab.P + 31) & ~31), w.smem, s,
          w.tm_psi, w.tm_phi, d, w.tab, trap_of(s), LinPhase{s->lin[0], s->lin[1], s->lin[2]}, g, gd, s->p.dt,
          s->state, w.TW, w.boxn, w.nbox, s->err));
      CKL();
      mark(s);
      s->launches++;
      return GPE_OK;
   }

   // FP64 tiles of 8 or 16 lines use kernels compiled for that width
   template <int AXIS, bool NU, int MSEG, int S> static gpe_status sweep_xy_launch(gpe_solver *s, double g, double gd) {
      if constexpr (std::is_same<R, double>::value) {
         if (s->sw[AXIS].TW == 8) return sweep_xy_launch_t<AXIS, NU, MSEG, S, 8>(s, g, gd);
         if (s->sw[AXIS].TW == 16) return sweep_xy_launch_t<AXIS, NU, MSEG, S, 16>(s, g, gd);
      }
      return sweep_xy_launch_t<AXIS, NU, MSEG, S, 0>(s, g, gd);
   }

   // 32-point segments exist for FP32 real lines only (register budget)
   static constexpr bool kSeg32 = std::is_same<R, float>::value && !CPLX;

   template <int AXIS, bool NU> static gpe_status sweep_xy(gpe_solver *s, double g, double gd) {
      const auto &w = s->sw[AXIS];
      if constexpr (kSeg32)
         if (w.MSEG == 32)
            return w.S == 3 ? sweep_xy_launch<AXIS, NU, 32, 3>(s, g, gd) : sweep_xy_launch<AXIS, NU, 32, 2>(s, g, gd);
      if (w.MSEG == 8) return w.S == 3 ? sweep_xy_launch<AXIS, NU, 8, 3>(s, g, gd) : sweep_xy_launch<AXIS, NU, 8, 2>(s, g, gd);
      return w.S == 3 ? sweep_xy_launch<AXIS, NU, 16, 3>(s, g, gd) : sweep_xy_launch<AXIS, NU, 16, 2>(s, g, gd);
   }

   // x sweep; with nu the pending 1/norm and calcnu are applied on load
   // (calcnu_kernel imag3d-mpicuda.cu:1759 fused with calclux_kernel :1802).
   static gpe_status xsweep(gpe_solver *s, bool nu, double g, double gd) {
      return nu ? sweep_xy<0, true>(s, g, gd) : sweep_xy<0, false>(s, g, gd);
   }

   static gpe_status ysweep(gpe_solver *s) { return sweep_xy<1, false>(s, 0., 0.); }

   template <int MOM, int MSEG, int S, int TWC> static gpe_status sweep_z_launch_t(gpe_solver *s) {
      auto &w = s->sw[2];
      const Dims &d = s->d;
      const void *f = (const void *) k_sweep_z<R, CPLX, MOM, MSEG, S, TWC>;
      CKS(smem_attr(f, w.smem));
      const long long ntiles = (d.nxy + w.TW - 1) / w.TW;
      const unsigned grid = (unsigned) std::min<long long>(ntiles, (long long) w.ctas * s->nsm);
      CKS(launch_pdl(k_sweep_z<R, CPLX, MOM, MSEG, S, TWC>, grid, ((w.TW * w.tab.P + 31) & ~31), w.smem, s,
          (P *) s->psi, d, w.tab, w.TW, w.LS, s->wz, s->wz2, s->p.dz / 3., s->rowA, s->rowB, s->err));
      CKL();
      mark(s);
      s->launches++;
      return GPE_OK;
   }

   template <int MOM, int MSEG, int S> static gpe_status sweep_z_launch(gpe_solver *s) {
      if constexpr (std::is_same<R, double>::value) {
         if (s->sw[2].TW == 8) return sweep_z_launch_t<MOM, MSEG, S, 8>(s);
         if (s->sw[2].TW == 16) return sweep_z_launch_t<MOM, MSEG, S, 16>(s);
      }
      return sweep_z_launch_t<MOM, MSEG, S, 0>(s);
   }

   template <int MOM> static gpe_status zsweep_m(gpe_solver *s) {
      const auto &w = s->sw[2];
      if constexpr (kSeg32)
         if (w.MSEG == 32) return w.S == 3 ? sweep_z_launch<MOM, 32, 3>(s) : sweep_z_launch<MOM, 32, 2>(s);
      if (w.MSEG == 8) return w.S == 3 ? sweep_z_launch<MOM, 8, 3>(s) : sweep_z_launch<MOM, 8, 2>(s);
      return w.S == 3 ? sweep_z_launch<MOM, 16, 3>(s) : sweep_z_launch<MOM, 16, 2>(s);
   }

   // z sweep; mom 1: each row also yields its Simpson integral of |psi|^2
   // (norm); mom 2: and of z^2 |psi|^2 (rms row partials)
   static gpe_status zsweep(gpe_solver *s, int mom) {
      if (mom == 2) return zsweep_m<2>(s);
      return mom == 1 ? zsweep_m<1>(s) : zsweep_m<0>(s);
   }

   static gpe_status norm_final(gpe_solver *s, double *dev_out) {
      CKS(launch_pdl(k_norm_final, blocks_for(s->d.nx, kNormRowsPerCta), 32 * kNormRowsPerCta, 0, s,
          s->rowA, s->d, s->p.dx, s->p.dy, s->state, s->tmp, dev_out));
      CKL();
      mark(s);
      s->launches++;
      return GPE_OK;
   }

   static gpe_status apply_scale(gpe_solver *s) {
      k_apply_scale<R, CPLX><<<592, 256, 0, s->st>>>((P *) s->psi, s->d.npts, s->state);
      CKL();
      k_state_set<<<1, 1, 0, s->st>>>(s->state, 1.);
      CKL();
      s->launches += 2;
      return GPE_OK;
   }

   static gpe_status calcnorm(gpe_solver *s, bool renorm) {
      const Dims &d = s->d;
      k_rows_dens<R, CPLX><<<blocks_for(d.nxy, 128), 128, 0, s->st>>>((const P *) s->psi, d, s->p.dz, s->rowA, nullptr,
                                                                     s->z2);
      CKL();
      CKS(norm_final(s, s->obs));
      s->launches++;
      if (renorm) {
         CKS(apply_scale(s));
      } else {
         k_state_set<<<1, 1, 0, s->st>>>(s->state, 1.);
         CKL();
      }
      return GPE_OK;
   }

   static gpe_status rms(gpe_solver *s, double *dev_out) {
      const Dims &d = s->d;
      k_rows_dens<R, CPLX><<<blocks_for(d.nxy, 128), 128, 0, s->st>>>((const P *) s->psi, d, s->p.dz, s->rowA, s->rowB,
                                                                     s->z2);
      CKL();
      s->launches++;
      return rms_final(s, dev_out);
   }

   // rms from the row partials in rowA / rowB (k_rows_dens, or the z sweep
   // of the step with mom = 2)
   static gpe_status rms_final(gpe_solver *s, double *dev_out) {
      const Dims &d = s->d;
      CKS(launch_pdl(k_rms_final, blocks_for(d.nx, kNormRowsPerCta), 32 * kNormRowsPerCta, 0, s,
          s->rowA, s->rowB, d, s->p.dx, s->p.dy, s->x2, s->y2, s->state, s->tmp, dev_out));
      CKL();
      s->launches++;
      return GPE_OK;
   }

   static gpe_status muen(gpe_solver *s, double g, double gd, double *dev_out) {
      const Dims &d = s->d;
      CKS(psidd2(s));
      k_muen_rows<R, CPLX><<<blocks_for(d.nxy, 128), 128, 0, s->st>>>((const P *) s->psi, (const R *) s->phi, d,
                                                                     trap_of(s), g, gd, s->p.dx, s->p.dy, s->p.dz,
                                                                     s->par, s->rowA, s->rowB);
      CKL();
      k_xy_final<<<1, 256, sizeof(double) * d.nx, s->st>>>(s->rowA, d, s->p.dx, s->p.dy, dev_out);
      CKL();
      k_xy_final<<<1, 256, sizeof(double) * d.nx, s->st>>>(s->rowB, d, s->p.dx, s->p.dy, dev_out + 1);
      CKL();
      s->launches += 3;
      return GPE_OK;
   }

   // One split step (imag3d-mpicuda.cu:319-324): calcpsidd2, calcnu (fused
   // into the x sweep), x, y, z sweeps, and in imaginary time the norm.
   // rms_rows: (real time) the z sweep also leaves the rms row partials of
   // the new psi in rowA / rowB for rms_final.
   static gpe_status step(gpe_solver *s, double g, double gd, double *dev_norm, bool rms_rows = false) {
      CKS(psidd2(s));
      CKS(xsweep(s, true, g, gd));
      CKS(ysweep(s));
      const bool imag = !CPLX;
      CKS(zsweep(s, imag ? 1 : (rms_rows ? 2 : 0)));
      if (imag) CKS(norm_final(s, dev_norm));
      return GPE_OK;
   }

   static gpe_status calcnu(gpe_solver *s, double g, double gd) {
      k_calcnu<R, CPLX><<<592, 256, 0, s->st>>>((P *) s->psi, (const R *) s->phi, s->d, trap_of(s), g, gd, s->p.dt);
      CKL();
      s->launches++;
      return GPE_OK;
   }

   static gpe_status density(gpe_solver *s, int kind, long sx, long sy, long sz, double *out, long cap, long *count);

   // ---- batched launches: geometry and descriptor of this instance
   static gpe_status geom(gpe_solver *s, int Ly, int Lx, BatchGeom *g) {
      const Dims &d = s->d;
      *g = BatchGeom{};
      g->Ly = s->Ly;
      g->Lx = s->Lx;
      if (Ly <= 0 || Lx <= 0) return GPE_OK;
      // z passes: 8-row tiles on CTAs sized to them
      constexpr int L = 8;
      const int zp = zppt(s, L);
      const int ppt = zp <= 8 ? 8 : (zp <= 16 ? 16 : 32);
      g->zppt = ppt;
      g->tiles[kPZfwd] = g->tiles[kPZinv] = (d.nxy + L - 1) / L;
      g->threads[kPZfwd] = g->threads[kPZinv] = z_threads(s, L, ppt);
      g->smem[kPZfwd] = zfwd_smem(s, L);
      g->smem[kPZinv] = zinv_smem(s, L);
      if (g->smem[kPZfwd] > 227 * 1024 || g->smem[kPZinv] > 227 * 1024)
         return fail(GPE_ERR_PARAM, "batch: z rows too long for 8-row tiles");
      // y / x passes
      const long ry = (long) s->boxy * s->nboxy, rx = (long) s->boxx * s->nboxx;
      if (ry * Ly > 256L * FftL<R>::PPT || rx * Lx > 256L * FftL<R>::PPT)
         return fail(GPE_ERR_PARAM, "batch: FFT tile too wide for this grid");
      g->tiles[kPYfft] = g->tiles[kPYinv] = (long long) d.nx * ((d.nzh + Ly - 1) / Ly);
      g->tiles[kPXconv] = (long long) d.ny * ((d.nzh + Lx - 1) / Lx);
      g->threads[kPYfft] = g->threads[kPYinv] = fft_threads(ry, Ly);
      g->threads[kPXconv] = fft_threads(rx, Lx);
      g->smem[kPYfft] = g->smem[kPYinv] = 128 + (size_t) ry * Ly * sizeof(C) + d.ny * sizeof(C);
      g->smem[kPXconv] = 128 + (size_t) rx * Lx * sizeof(C) + d.nx * sizeof(C) + (size_t) (d.nx / 2 + 1) * Lx * sizeof(double);
      // boundary planes of phi
      g->tiles[kPPhifix] = std::max<long>(1, (d.ny - 1) + (d.nx - 1));
      g->threads[kPPhifix] = (unsigned) std::min<long>(256, std::max<long>(32, (d.nz - 1 + 31) / 32 * 32));
      // sweeps
      const size_t esz = s->esz_psi;
      for (int ax = 0; ax < 3; ax++) {
         const auto &w = s->sw[ax];
         const int TW = w.TW, P = w.tab.P, spw = 32 / TW;
         const int kp = kPXsweep + ax;
         g->mseg[ax] = w.MSEG;
         g->threads[kp] = (unsigned) ((TW * P + 31) & ~31);
         const int nzb = (d.nz + TW - 1) / TW;
         g->tiles[kp] = ax == 0 ? (long long) d.ny * nzb : (ax == 1 ? (long long) d.nx * nzb : (d.nxy + TW - 1) / TW);
         size_t stage;
         if (ax < 2) {
            const size_t rows = (size_t) w.boxn * w.nbox;
            stage = rows * TW * esz + (ax == 0 ? rows * TW * s->esz_r : 0);
         } else {
            stage = (size_t) TW * w.LS * esz;
         }
         g->stage[ax] = (uint32_t) ((stage + 127) & ~(size_t) 127);
         g->blk[ax] = (uint32_t) ((2 * (size_t) ((P + spw - 1) / spw + 1) * TW * esz + 15) & ~(size_t) 15);
         if (!s->fp32) {
            if (ax == 0) g->extra[ax] = (uint32_t) (d.nx * (s->cplx ? 16 : 8));
            if (ax == 2) g->extra[ax] = (uint32_t) (4 * (size_t) d.nz * (s->cplx ? 16 : 8));
         }
         if (ax == 2) g->part = (uint32_t) (((size_t) P * TW * sizeof(double) + 15) & ~(size_t) 15);
      }
      // norm (imaginary time)
      g->tiles[kPNorm] = s->cplx ? 0 : (d.nx + kNormRowsPerCta - 1) / kNormRowsPerCta;
      g->threads[kPNorm] = 32 * kNormRowsPerCta;
      return GPE_OK;
   }

   static gpe_status desc(gpe_solver *s, int Ly, int Lx, double g, double gd, BatchDesc *D) {
      const Dims &d = s->d;
      std::memset((void *) D, 0, sizeof(BatchDesc));
      D->tm_psi[0] = s->sw[0].tm_psi;
      D->tm_psi[1] = s->sw[1].tm_psi;
      D->tm_phi = s->sw[0].tm_phi;
      CKS(make_tmap(&D->tm_spec_y, s->spec, s->esz_r, 2 * d.nzh, d.ny, d.nx, 2 * Ly, s->boxy, 1, 2 * d.nzp));
      CKS(make_tmap(&D->tm_spec_x, s->spec, s->esz_r, 2 * d.nzh, d.ny, d.nx, 2 * Lx, 1, s->boxx, 2 * d.nzp));
      for (int ax = 0; ax < 3; ax++) {
         const auto &w = s->sw[ax];
         SweepView &v = D->sv[ax];
         v.tb = w.tab;
         v.trap = trap_of(s);
         v.lin = LinPhase{s->lin[0], s->lin[1], s->lin[2]};
         v.d = d;
         v.st = s->state;
         v.err = s->err;
         v.psi = s->psi;
         v.wz = s->wz;
         v.wz2 = s->wz2;
         v.rowsum = s->rowA;
         v.rowsum2 = s->rowB;
         v.g = g;
         v.gd = gd;
         v.dt = s->p.dt;
         v.hz3 = s->p.dz / 3.;
         v.TW = w.TW;
         v.boxn = w.boxn;
         v.nbox = w.nbox;
         v.LS = w.LS;
      }
      D->px = s->px;
      D->py = s->py;
      D->ph = s->ph;
      D->d = d;
      D->psi = s->psi;
      D->spec = s->spec;
      D->phi = s->phi;
      D->twx = s->twx;
      D->twy = s->twy;
      D->twz = s->twz;
      D->udd = s->udd;
      D->state = s->state;
      D->err = s->err;
      D->rowA = s->rowA;
      D->xs = s->tmp;
      D->hx = s->p.dx;
      D->hy = s->p.dy;
      D->LSr = s->LSr;
      D->LSo = s->LSo;
      D->boxy = s->boxy;
      D->nboxy = s->nboxy;
      D->boxx = s->boxx;
      D->nboxx = s->nboxx;
      D->Ly = Ly;
      D->Lx = Lx;
      return GPE_OK;
   }
};

template <class R, bool CPLX>
gpe_status Impl<R, CPLX>::density(gpe_solver *s, int kind, long sx, long sy, long sz, double *out, long cap,
                                  long *count) {
   const Dims &d = s->d;
   const P *psi = (const P *) s->psi;
   const double hh[3] = {s->p.dx, s->p.dy, s->p.dz};
   const int n[3] = {d.nx, d.ny, d.nz};
   const std::vector<double> *crd[3] = {&s->hx, &s->hy, &s->hz};
   const long stp[3] = {sx, sy, sz};
   std::vector<double> buf;
   long o = 0;
   auto need = [&](long m) -> gpe_status {
      if (m > cap) return fail(GPE_ERR_PARAM, "density output buffer too small");
      return GPE_OK;
   };
   if (kind >= GPE_DEN_1D_X && kind <= GPE_DEN_1D_Z) {
      // axis integrated first, then the second one (reference nesting)
      const int keep = kind - GPE_DEN_1D_X;
      const int first = (keep == 2) ? 1 : 2;   // z (or y for the z profile)
      const int second = (keep == 0) ? 1 : 0;  // y for x profile, x otherwise
      const int o1 = first == 0 ? 1 : 0, o2 = first == 2 ? 1 : 2;  // axes of the 2D result
      if ((long long) n[o1] * n[o2] > s->row_cap) return fail(GPE_ERR_STATE, "row buffer too small");
      k_lineint_psi<R, CPLX><<<blocks_for((long long) n[o1] * n[o2], 128), 128, 0, s->st>>>(psi, d, first, hh[first],
                                                                                          s->rowA);
      CKL();
      const int ax = (second == o1) ? 0 : 1;  // integrate rows (0) or columns (1)
      const int m = n[keep];
      k_lineint_arr<<<blocks_for(m, 128), 128, 0, s->st>>>(s->rowA, n[o1], n[o2], ax == 0 ? 0 : 1, hh[second], s->tmp);
      CKL();
      s->launches += 2;
      buf.resize(m);
      CK(cudaMemcpyAsync(buf.data(), s->tmp, sizeof(double) * m, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      for (long c = 0; c < m; c += stp[keep]) {
         CKS(need(o + 2));
         out[o++] = (*crd[keep])[c];
         out[o++] = buf[c];
      }
   } else if (kind >= GPE_DEN_2D_XY && kind <= GPE_DEN_2D_YZ) {
      const int integ = 2 - (kind - GPE_DEN_2D_XY);  // xy -> z, xz -> y, yz -> x
      const int a1 = integ == 0 ? 1 : 0, a2 = integ == 2 ? 1 : 2;
      if ((long long) n[a1] * n[a2] > s->row_cap) return fail(GPE_ERR_STATE, "row buffer too small");
      k_lineint_psi<R, CPLX><<<blocks_for((long long) n[a1] * n[a2], 128), 128, 0, s->st>>>(psi, d, integ, hh[integ],
                                                                                          s->rowA);
      CKL();
      s->launches++;
      buf.resize((size_t) n[a1] * n[a2]);
      CK(cudaMemcpyAsync(buf.data(), s->rowA, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      for (long u = 0; u < n[a1]; u += stp[a1])
         for (long v = 0; v < n[a2]; v += stp[a2]) {
            CKS(need(o + 3));
            out[o++] = (*crd[a1])[u];
            out[o++] = (*crd[a2])[v];
            out[o++] = buf[(size_t) u * n[a2] + v];
         }
   } else if (kind >= GPE_DEN_3D_XY0 && kind <= GPE_DEN_3D_0YZ) {
      const int fixed = 2 - (kind - GPE_DEN_3D_XY0);  // xy0 -> z fixed, x0z -> y, 0yz -> x
      const int a1 = fixed == 0 ? 1 : 0, a2 = fixed == 2 ? 1 : 2;
      int lo[3] = {0, 0, 0}, hi[3] = {d.nx, d.ny, d.nz}, sp[3] = {(int) sx, (int) sy, (int) sz};
      lo[fixed] = n[fixed] / 2; hi[fixed] = lo[fixed] + 1; sp[fixed] = 1;
      const long na = (n[a1] + stp[a1] - 1) / stp[a1], nb = (n[a2] + stp[a2] - 1) / stp[a2];
      double *dv = nullptr;
      CK(cudaMalloc(&dv, sizeof(double) * na * nb));
      k_gather_dens<R, CPLX><<<blocks_for(na * nb, 256), 256, 0, s->st>>>(psi, d, lo[0], hi[0], sp[0], lo[1], hi[1], sp[1],
                                                                         lo[2], hi[2], sp[2], dv);
      s->launches++;
      buf.resize(na * nb);
      cudaError_t e1 = cudaGetLastError();
      cudaError_t e2 = cudaMemcpyAsync(buf.data(), dv, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost, s->st);
      cudaError_t e3 = cudaStreamSynchronize(s->st);
      cudaFree(dv);
      if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return fail(GPE_ERR_CUDA, "density cut failed");
      for (long u = 0; u < na; u++)
         for (long v = 0; v < nb; v++) {
            CKS(need(o + 3));
            out[o++] = (*crd[a1])[u * stp[a1]];
            out[o++] = (*crd[a2])[v * stp[a2]];
            out[o++] = buf[(size_t) u * nb + v];
         }
   } else if (kind == GPE_DEN_3D) {
      const long na = (d.nx + sx - 1) / sx, nb = (d.ny + sy - 1) / sy, nc = (d.nz + sz - 1) / sz;
      CKS(need(na * nb * nc));
      double *dv = nullptr;
      CK(cudaMalloc(&dv, sizeof(double) * na * nb * nc));
      k_gather_dens<R, CPLX><<<592, 256, 0, s->st>>>(psi, d, 0, d.nx, (int) sx, 0, d.ny, (int) sy, 0, d.nz, (int) sz, dv);
      s->launches++;
      cudaError_t e1 = cudaGetLastError();
      cudaError_t e2 = cudaMemcpyAsync(out, dv, sizeof(double) * na * nb * nc, cudaMemcpyDeviceToHost, s->st);
      cudaError_t e3 = cudaStreamSynchronize(s->st);
      cudaFree(dv);
      if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return fail(GPE_ERR_CUDA, "density copy failed");
      o = na * nb * nc;
   } else {
      return fail(GPE_ERR_PARAM, "unknown density kind");
   }
   if (count) *count = o;
   return GPE_OK;
}

#define DISPATCH(s, CALL)                                                                 \
   (((s)->fp32) ? (((s)->cplx) ? Impl<float, true>::CALL : Impl<float, false>::CALL)     \
                : (((s)->cplx) ? Impl<double, true>::CALL : Impl<double, false>::CALL))

#define CHECK_HANDLE(s) \
   if (!(s)) return fail(GPE_ERR_PARAM, "null solver handle")

// ------------------------------------------------------------------ psi I/O
// FP64 psi is copied as is (the host layout equals the device layout); the
// mixed-precision handle converts through a host float buffer.
extern "C" gpe_status gpe_set_psi(gpe_solver *s, const double *psi) {
   CHECK_HANDLE(s);
   if (!psi) return fail(GPE_ERR_PARAM, "null psi");
   CK(cudaSetDevice(s->dev));
   const size_t nd = (size_t) s->d.npts * (s->cplx ? 2 : 1);
   if (s->fp32) {
      std::vector<float> b(nd);
      for (size_t q = 0; q < nd; q++) b[q] = (float) psi[q];
      CK(cudaMemcpyAsync(s->psi, b.data(), sizeof(float) * nd, cudaMemcpyHostToDevice, s->st));
      CK(cudaStreamSynchronize(s->st));
   } else {
      CK(cudaMemcpyAsync(s->psi, psi, sizeof(double) * nd, cudaMemcpyHostToDevice, s->st));
      CK(cudaStreamSynchronize(s->st));
   }
   k_state_set<<<1, 1, 0, s->st>>>(s->state, 1.);
   CKL();
   return GPE_OK;
}

extern "C" gpe_status gpe_get_psi(gpe_solver *s, double *psi) {
   CHECK_HANDLE(s);
   if (!psi) return fail(GPE_ERR_PARAM, "null psi");
   CK(cudaSetDevice(s->dev));
   const size_t nd = (size_t) s->d.npts * (s->cplx ? 2 : 1);
   if (s->fp32) {
      std::vector<float> b(nd);
      CK(cudaMemcpyAsync(b.data(), s->psi, sizeof(float) * nd, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      for (size_t q = 0; q < nd; q++) psi[q] = b[q];
   } else {
      CK(cudaMemcpyAsync(psi, s->psi, sizeof(double) * nd, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
   }
   return GPE_OK;
}

// initpsi Gaussian (imag3d-mpicuda.cu:835-867), evaluated on the host like
// the reference and uploaded.
extern "C" gpe_status gpe_init_gaussian(gpe_solver *s) {
   CHECK_HANDLE(s);
   const double pi = kRefPi;
   const double cpsi = std::sqrt(pi * std::sqrt(pi / (s->p.gamma * s->p.nu * s->p.lambda)));
   const Dims &d = s->d;
   std::vector<double> re((size_t) d.npts * (s->cplx ? 2 : 1), 0.);
   for (long i = 0; i < d.nx; i++)
      for (long j = 0; j < d.ny; j++)
         for (long k = 0; k < d.nz; k++) {
            const double tmp = std::exp(-0.5 * (s->p.gamma * s->hx2[i] + s->p.nu * s->hy2[j] + s->p.lambda * s->hz2[k]));
            re[(size_t) ((i * d.ny + j) * d.nz + k) * (s->cplx ? 2 : 1)] = tmp / cpsi;
         }
   return gpe_set_psi(s, re.data());
}

extern "C" gpe_status gpe_init_density(gpe_solver *s, const double *rho) {
   CHECK_HANDLE(s);
   if (!rho) return fail(GPE_ERR_PARAM, "null density");
   CK(cudaSetDevice(s->dev));
   double *dr = nullptr;
   CK(cudaMalloc(&dr, sizeof(double) * s->d.npts));
   cudaError_t e = cudaMemcpyAsync(dr, rho, sizeof(double) * s->d.npts, cudaMemcpyHostToDevice, s->st);
   if (e == cudaSuccess) {
      if (s->fp32)
         s->cplx ? k_init_density<float, true><<<592, 256, 0, s->st>>>((float2 *) s->psi, dr, s->d.npts)
                 : k_init_density<float, false><<<592, 256, 0, s->st>>>((float *) s->psi, dr, s->d.npts);
      else
         s->cplx ? k_init_density<double, true><<<592, 256, 0, s->st>>>((double2 *) s->psi, dr, s->d.npts)
                 : k_init_density<double, false><<<592, 256, 0, s->st>>>((double *) s->psi, dr, s->d.npts);
      e = cudaGetLastError();
   }
   cudaError_t e2 = cudaStreamSynchronize(s->st);
   cudaFree(dr);
   if (e != cudaSuccess || e2 != cudaSuccess) return fail(GPE_ERR_CUDA, "init from density failed");
   s->launches++;
   k_state_set<<<1, 1, 0, s->st>>>(s->state, 1.);
   CKL();
   return GPE_OK;
}

// -------------------------------------------------------------- operators
// Reads and clears the device status word; a bounded wait that gave up turns
// into GPE_ERR_TIMEOUT.
static gpe_status check_err(gpe_solver *s) {
   uint32_t e = 0;
   CK(cudaMemcpyAsync(&e, s->err, sizeof(e), cudaMemcpyDeviceToHost, s->st));
   CK(cudaStreamSynchronize(s->st));
   if (e) {
      CK(cudaMemsetAsync(s->err, 0, sizeof(uint32_t), s->st));
      return fail(GPE_ERR_TIMEOUT, "a bounded device wait for a bulk copy gave up");
   }
   return GPE_OK;
}

static gpe_status read_obs(gpe_solver *s, double *dst, int n, int off = 0) {
   CK(cudaMemcpyAsync(dst, s->obs + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
   CK(cudaStreamSynchronize(s->st));
   return GPE_OK;
}

extern "C" gpe_status gpe_calcnorm(gpe_solver *s, int renormalize, double *norm) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   CKS(DISPATCH(s, calcnorm(s, renormalize != 0)));
   double v = 0;
   CKS(read_obs(s, &v, 1));
   if (norm) *norm = v;
   return GPE_OK;
}

extern "C" gpe_status gpe_run(gpe_solver *s, long nsteps, double *g, double *gd, double g_inc, double gd_inc,
                              double *last_norm, long rms_every, double *rms_out) {
   CHECK_HANDLE(s);
   if (!g || !gd) return fail(GPE_ERR_PARAM, "null coupling pointers");
   if (nsteps < 0) return fail(GPE_ERR_PARAM, "negative step count");
   CK(cudaSetDevice(s->dev));
   const bool imag = !s->cplx;
   const long nrms = (rms_every > 0) ? (nsteps + rms_every - 1) / rms_every : 0;
   if (nrms > 0 && !rms_out) return fail(GPE_ERR_PARAM, "rms_out required when rms_every > 0");
   // rms samples land in the handle's preallocated slots (no allocation and
   // no implicit synchronisation inside the run); every kRmsSlots samples the
   // full batch is copied out
   long flushed = 0;  // samples already copied to rms_out
   auto flush = [&](long upto) -> gpe_status {
      if (upto <= flushed) return GPE_OK;
      CK(cudaMemcpyAsync(rms_out + 4 * flushed, s->rms_buf, sizeof(double) * 4 * (upto - flushed),
                         cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      flushed = upto;
      return GPE_OK;
   };
   gpe_status st = GPE_OK;
   for (long c = 0; c < nsteps && st == GPE_OK; c++) {
      *g += g_inc;
      *gd += gd_inc;
      const bool rms_here = rms_every > 0 && c % rms_every == 0;
      double *slot = nullptr;
      if (rms_here) {
         const long idx = c / rms_every;
         if (idx - flushed == kRmsSlots) st = flush(idx);
         slot = s->rms_buf + 4 * (idx - flushed);
      }
      // real time: the step's z sweep leaves the rms row partials (no extra
      // pass over psi); imaginary time: renormalise first, then a full rms
      if (st == GPE_OK) st = DISPATCH(s, step(s, *g, *gd, s->obs, rms_here && !imag));
      if (st == GPE_OK && rms_here) {
         if (imag) {
            st = DISPATCH(s, apply_scale(s));
            if (st == GPE_OK) st = DISPATCH(s, rms(s, slot));
         } else {
            st = DISPATCH(s, rms_final(s, slot));
         }
      }
   }
   if (st == GPE_OK && imag && nsteps > 0) st = DISPATCH(s, apply_scale(s));
   if (st == GPE_OK && last_norm && imag && nsteps > 0) st = read_obs(s, last_norm, 1);
   if (st == GPE_OK && nrms > 0) st = flush(nrms);
   if (st == GPE_OK) {
      cudaError_t e = cudaStreamSynchronize(s->st);
      if (e != cudaSuccess) st = fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   }
   if (st == GPE_OK) st = check_err(s);
   return st;
}

extern "C" gpe_status gpe_calcmuen(gpe_solver *s, double g, double gd, double *mu, double *en) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   CKS(DISPATCH(s, muen(s, g, gd, s->obs + 8)));
   double v[2];
   CKS(read_obs(s, v, 2, 8));
   if (mu) *mu = v[0];
   if (en) *en = v[1];
   return GPE_OK;
}

extern "C" gpe_status gpe_calcrms(gpe_solver *s, double *rms) {
   CHECK_HANDLE(s);
   if (!rms) return fail(GPE_ERR_PARAM, "null rms");
   CK(cudaSetDevice(s->dev));
   CKS(DISPATCH(s, rms(s, s->obs + 16)));
   return read_obs(s, rms, 4, 16);
}

extern "C" gpe_status gpe_psi_center2(gpe_solver *s, double *value) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   const Dims &d = s->d;
   const long long q = ((long long) (d.nx / 2) * d.ny + d.ny / 2) * d.nz + d.nz / 2;
   double v[2] = {0, 0};
   if (s->fp32) {
      float f[2] = {0, 0};
      CK(cudaMemcpyAsync(f, (char *) s->psi + q * s->esz_psi, s->esz_psi, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      v[0] = f[0]; v[1] = s->cplx ? f[1] : 0.;
   } else {
      CK(cudaMemcpyAsync(v, (char *) s->psi + q * s->esz_psi, s->esz_psi, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      if (!s->cplx) v[1] = 0.;
   }
   if (value) *value = v[0] * v[0] + v[1] * v[1];
   return GPE_OK;
}

extern "C" gpe_status gpe_density(gpe_solver *s, int kind, long sx, long sy, long sz, double *out, long cap,
                                  long *count) {
   CHECK_HANDLE(s);
   if (!out) return fail(GPE_ERR_PARAM, "null output");
   if (sx < 1 || sy < 1 || sz < 1) return fail(GPE_ERR_PARAM, "OUTSTPX/Y/Z must be >= 1");
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, density(s, kind, sx, sy, sz, out, cap, count));
}

extern "C" gpe_status gpe_calcpsidd2(gpe_solver *s) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, psidd2(s));
}

extern "C" gpe_status gpe_get_phi(gpe_solver *s, double *phi) {
   CHECK_HANDLE(s);
   if (!phi) return fail(GPE_ERR_PARAM, "null phi");
   CK(cudaSetDevice(s->dev));
   const long long n = s->d.npts;
   if (s->fp32) {
      std::vector<float> b((size_t) n);
      CK(cudaMemcpyAsync(b.data(), s->phi, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
      for (long long q = 0; q < n; q++) phi[q] = b[(size_t) q];
   } else {
      CK(cudaMemcpyAsync(phi, s->phi, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
      CK(cudaStreamSynchronize(s->st));
   }
   return GPE_OK;
}

extern "C" gpe_status gpe_calcnu(gpe_solver *s, double g, double gd) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, calcnu(s, g, gd));
}

extern "C" gpe_status gpe_calclux(gpe_solver *s) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, xsweep(s, false, 0., 0.));
}

extern "C" gpe_status gpe_calcluy(gpe_solver *s) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, ysweep(s));
}

extern "C" gpe_status gpe_calcluz(gpe_solver *s) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   return DISPATCH(s, zsweep(s, 0));
}

extern "C" gpe_status gpe_synchronize(gpe_solver *s) {
   CHECK_HANDLE(s);
   CK(cudaStreamSynchronize(s->st));
   return check_err(s);
}

extern "C" gpe_status gpe_selftest_wait_timeout(gpe_solver *s, unsigned spins) {
   CHECK_HANDLE(s);
   if (spins < 1 || spins > (1u << 16)) return fail(GPE_ERR_PARAM, "spins must be in [1, 65536]");
   CK(cudaSetDevice(s->dev));
   k_wait_selftest<<<1, 32, 0, s->st>>>(spins, s->err);
   CKL();
   s->launches++;
   return GPE_OK;
}

extern "C" gpe_status gpe_launch_count(gpe_solver *s, long long *count) {
   CHECK_HANDLE(s);
   if (count) *count = s->launches;
   return GPE_OK;
}

extern "C" gpe_status gpe_time_steps(gpe_solver *s, long nsteps, double g, double gd, double *ms) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   cudaEvent_t a, b;
   CK(cudaEventCreate(&a));
   CK(cudaEventCreate(&b));
   CK(cudaEventRecord(a, s->st));
   gpe_status st = GPE_OK;
   for (long c = 0; c < nsteps && st == GPE_OK; c++) st = DISPATCH(s, step(s, g, gd, nullptr));
   if (st == GPE_OK && !s->cplx) st = DISPATCH(s, apply_scale(s));
   CK(cudaEventRecord(b, s->st));
   CK(cudaEventSynchronize(b));
   float f = 0;
   CK(cudaEventElapsedTime(&f, a, b));
   cudaEventDestroy(a);
   cudaEventDestroy(b);
   if (ms) *ms = f;
   return st;
}

extern "C" gpe_status gpe_time_calcpsidd2(gpe_solver *s, long nrep, double *ms) {
   CHECK_HANDLE(s);
   if (nrep < 1) return fail(GPE_ERR_PARAM, "nrep must be >= 1");
   CK(cudaSetDevice(s->dev));
   CKS(DISPATCH(s, psidd2(s)));  // untimed warm-up
   cudaEvent_t a, b;
   CK(cudaEventCreate(&a));
   CK(cudaEventCreate(&b));
   CK(cudaEventRecord(a, s->st));
   gpe_status st = GPE_OK;
   for (long c = 0; c < nrep && st == GPE_OK; c++) st = DISPATCH(s, psidd2(s));
   CK(cudaEventRecord(b, s->st));
   CK(cudaEventSynchronize(b));
   float f = 0;
   CK(cudaEventElapsedTime(&f, a, b));
   cudaEventDestroy(a);
   cudaEventDestroy(b);
   if (ms) *ms = f / nrep;
   if (st == GPE_OK) st = check_err(s);
   return st;
}

// ------------------------------------------------------------ profiling
static const char *kStepKernels[] = {"zfwd_r2c", "yfft_fwd", "xconv_udd", "yfft_inv", "zinv_c2r",
                                     "phi_boundary", "xsweep_calcnu", "ysweep", "zsweep", "norm_final"};

extern "C" const char *gpe_step_kernel_name(gpe_solver *s, int i) {
   const int n = (s && s->cplx) ? 9 : 10;
   if (i < 0 || i >= n) return nullptr;
   if (i == 8 && s && !s->cplx) return "zsweep_norm";
   return kStepKernels[i];
}

// Compulsory bytes of one launch of kernel i for this pass structure.
extern "C" double gpe_step_kernel_bytes(gpe_solver *s, int i) {
   if (!s) return 0.;
   const Dims &d = s->d;
   const double sp = (double) s->esz_psi, sc = (double) s->esz_c, r = (double) s->esz_r;
   const double npts = (double) d.npts, half = (double) d.nzh * (double) d.nxy;
   const double oct = (double) d.nzh * (d.nx / 2 + 1) * (d.ny / 2 + 1) * 8.;
   const double planes = ((double) (d.ny - 1) * (d.nz - 1) + (double) (d.nx - 1) * (d.nz - 1)) * 2. * r;
   switch (i) {
   case 0: return npts * sp + half * sc;
   case 1: case 3: return 2. * half * sc;
   case 2: return 2. * half * sc + oct;
   case 4: return half * sc + npts * r;
   case 5: return planes;
   case 6: return npts * (2. * sp + r);
   case 7: return 2. * npts * sp;
   case 8: return 2. * npts * sp + (s->cplx ? 0. : 8. * (double) d.nxy);
   case 9: return s->cplx ? 0. : 8. * (double) d.nxy;
   default: return 0.;
   }
}

extern "C" gpe_status gpe_profile_step(gpe_solver *s, long nsteps, double g, double gd, double *ms, int cap,
                                       int *count) {
   CHECK_HANDLE(s);
   if (!ms || nsteps < 1) return fail(GPE_ERR_PARAM, "profile needs an output array and nsteps >= 1");
   CK(cudaSetDevice(s->dev));
   const int nk = s->cplx ? 9 : 10;
   if (cap < nk) return fail(GPE_ERR_PARAM, "profile output array too small");
   std::vector<cudaEvent_t> ev((size_t) (nsteps * (nk + 1)));
   for (auto &e : ev) CK(cudaEventCreate(&e));
   std::vector<double> acc(nk, 0.);
   gpe_status st = GPE_OK;
   for (long c = 0; c < nsteps && st == GPE_OK; c++) {
      cudaEvent_t *base = ev.data() + c * (nk + 1);
      cudaEventRecord(base[0], s->st);
      s->prof_ev = base + 1;
      s->prof_i = 0;
      s->prof_cap = nk;
      st = DISPATCH(s, step(s, g, gd, nullptr));
      s->prof_ev = nullptr;
   }
   if (st == GPE_OK && !s->cplx) st = DISPATCH(s, apply_scale(s));
   cudaError_t e = cudaStreamSynchronize(s->st);
   if (st == GPE_OK && e != cudaSuccess) st = fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   if (st == GPE_OK) {
      for (long c = 0; c < nsteps; c++) {
         cudaEvent_t *base = ev.data() + c * (nk + 1);
         for (int i = 0; i < nk; i++) {
            float f = 0.f;
            cudaEventElapsedTime(&f, base[i], base[i + 1]);
            acc[i] += f;
         }
      }
      for (int i = 0; i < nk; i++) ms[i] = acc[i] / (double) nsteps;
      if (count) *count = nk;
   }
   for (auto &x : ev) cudaEventDestroy(x);
   return st;
}

// ------------------------------------------------------------------ tuning
extern "C" gpe_status gpe_get_tuning(gpe_solver *s, gpe_tuning *t) {
   CHECK_HANDLE(s);
   if (!t) return fail(GPE_ERR_PARAM, "null tuning");
   for (int a = 0; a < 3; a++) {
      t->sweep_tw[a] = s->sw[a].TW;
      t->sweep_stages[a] = s->sw[a].S;
      t->sweep_seg[a] = s->sw[a].MSEG;
   }
   t->fft_tile[0] = s->Ly;
   t->fft_tile[1] = s->Lx;
   t->fft_max_radix = s->tune.fft_max_radix > 0 ? s->tune.fft_max_radix : (s->fp32 ? 16 : 8);
   return GPE_OK;
}

extern "C" gpe_status gpe_set_tuning(gpe_solver *s, const gpe_tuning *t) {
   CHECK_HANDLE(s);
   CK(cudaSetDevice(s->dev));
   CK(cudaStreamSynchronize(s->st));  // queued kernels still read the old tables
   const gpe_tuning old = s->tune;
   s->tune = t ? *t : gpe_tuning{};
   gpe_status st = plan_tiles(s);
   if (st != GPE_OK) {
      const std::string msg = g_err;
      s->tune = old;
      plan_tiles(s);
      return fail(st, msg);
   }
   return GPE_OK;
}

// Per-kernel times of the step (index as gpe_step_kernel_name) for the
// configuration in use; psi advances by warm + nsteps steps.
static gpe_status time_kernels(gpe_solver *s, double g, double gd, int nsteps, double *ms) {
   double warm[10];
   int cnt = 0;
   CKS(gpe_profile_step(s, 1, g, gd, warm, 10, &cnt));
   return gpe_profile_step(s, nsteps, g, gd, ms, 10, &cnt);
}

extern "C" gpe_status gpe_autotune(gpe_solver *s, double g, double gd, int nsteps, gpe_tuning *best) {
   CHECK_HANDLE(s);
   if (nsteps < 1) return fail(GPE_ERR_PARAM, "autotune needs nsteps >= 1");
   CK(cudaSetDevice(s->dev));
   gpe::Stash keep;  // psi and the step state, put back at the end
   CKS(gpe::stash_take(s, &keep));
   const gpe_tuning start = s->tune;
   gpe_tuning pick = start;
   double best_sweep[3] = {1e30, 1e30, 1e30}, best_y = 1e30, best_x = 1e30, best_fft = 1e30;
   const int ksw[3] = {6, 7, 8};  // x, y, z sweeps in the kernel list
   gpe_status st = GPE_OK;
   // sweeps: every available (lines per CTA, segment length) pair with both
   // pipeline depths; the three axes are timed together, candidate c of
   // each (its last one once an axis has fewer)
   {
      const long nn[3] = {s->d.nx, s->d.ny, s->d.nz};
      int cTW[3][kSweepCand], cM[3][kSweepCand], cP[kSweepCand], nc[3];
      bool prim[kSweepCand];
      for (int a = 0; a < 3; a++)
         nc[a] = sweep_candidates((int) nn[a], (int) (128 / s->esz_psi), (int) s->esz_psi, cTW[a], cM[a], cP, prim);
      const int ncmax = std::max(nc[0], std::max(nc[1], nc[2]));
      for (int c = 0; c < ncmax && st == GPE_OK; c++)
         for (int S = 2; S <= 3 && st == GPE_OK; S++) {
            gpe_tuning t = start;
            for (int a = 0; a < 3; a++) {
               t.sweep_tw[a] = cTW[a][std::min(c, nc[a] - 1)];
               t.sweep_seg[a] = cM[a][std::min(c, nc[a] - 1)];
               t.sweep_stages[a] = S;
            }
            s->tune = t;
            if (plan_tiles(s) != GPE_OK) continue;  // does not fit: skip
            double ms[10];
            st = time_kernels(s, g, gd, nsteps, ms);
            for (int a = 0; a < 3 && st == GPE_OK; a++)
               if (ms[ksw[a]] < best_sweep[a]) {
                  best_sweep[a] = ms[ksw[a]];
                  pick.sweep_tw[a] = t.sweep_tw[a];
                  pick.sweep_seg[a] = t.sweep_seg[a];
                  pick.sweep_stages[a] = S;
               }
         }
   }
   // FFT: tile widths of the y and x passes, then the largest radix
   for (int L = 128 / (int) s->esz_c; L >= 2 && st == GPE_OK; L /= 2) {
      gpe_tuning t = pick;
      t.fft_tile[0] = t.fft_tile[1] = L;
      s->tune = t;
      if (plan_tiles(s) != GPE_OK) continue;
      double ms[10];
      st = time_kernels(s, g, gd, nsteps, ms);
      if (st != GPE_OK) break;
      if (ms[1] + ms[3] < best_y) { best_y = ms[1] + ms[3]; pick.fft_tile[0] = L; }
      if (ms[2] < best_x) { best_x = ms[2]; pick.fft_tile[1] = L; }
   }
   for (int r = s->fp32 ? 16 : 8; r >= 2 && st == GPE_OK; r /= 2) {
      gpe_tuning t = pick;
      t.fft_max_radix = r;
      s->tune = t;
      if (plan_tiles(s) != GPE_OK) continue;
      double ms[10];
      st = time_kernels(s, g, gd, nsteps, ms);
      if (st != GPE_OK) break;
      const double f = ms[0] + ms[1] + ms[2] + ms[3] + ms[4];
      if (f < best_fft) { best_fft = f; pick.fft_max_radix = r; }
   }
   // the per-kernel choices are combined: keep them only if whole steps
   // (launched as a run launches them, each kernel overlapping the drain of
   // the one before) are faster than with the configuration the tuner
   // started from (on B200 the combined picks once made the mixed real-time
   // step 13 % slower)
   if (st == GPE_OK) {
      double t_pick = 1e30, t_start = 1e30;
      const gpe_tuning cand[2] = {pick, start};
      double *tt[2] = {&t_pick, &t_start};
      for (int k = 0; k < 2 && st == GPE_OK; k++) {
         s->tune = cand[k];
         st = plan_tiles(s);
         double ms = 0.;
         if (st == GPE_OK) st = gpe_time_steps(s, 1, g, gd, &ms);
         for (int r = 0; r < 2 && st == GPE_OK; r++) {
            st = gpe_time_steps(s, 2 * nsteps, g, gd, &ms);
            *tt[k] = std::min(*tt[k], ms);
         }
      }
      if (st == GPE_OK && t_pick >= t_start) pick = start;
   }
   s->tune = st == GPE_OK ? pick : start;
   gpe_status st2 = plan_tiles(s);
   gpe_status st3 = gpe::stash_restore(s, &keep);
   if (st != GPE_OK) return st;
   if (st2 != GPE_OK) return st2;
   if (st3 != GPE_OK) return st3;
   if (best) return gpe_get_tuning(s, best);  // every field filled in
   return GPE_OK;
}

// ------------------------------------------------------ hooks (internal.h)
namespace gpe {

gpe_status queue_steps(gpe_solver *s, long nsteps, double g, double gd) {
   CHECK_HANDLE(s);
   for (long c = 0; c < nsteps; c++) CKS(DISPATCH(s, step(s, g, gd, nullptr)));
   return GPE_OK;
}

gpe_status queue_finish(gpe_solver *s) {
   CHECK_HANDLE(s);
   if (!s->cplx) return DISPATCH(s, apply_scale(s));
   return GPE_OK;
}

gpe_status queue_muen(gpe_solver *s, double g, double gd) {
   CHECK_HANDLE(s);
   return DISPATCH(s, muen(s, g, gd, s->obs + 8));
}

gpe_status read_muen(gpe_solver *s, double *mu, double *en) {
   CHECK_HANDLE(s);
   double v[2];
   CKS(read_obs(s, v, 2, 8));
   CKS(check_err(s));
   if (mu) *mu = v[0];
   if (en) *en = v[1];
   return GPE_OK;
}

cudaStream_t stream_of(gpe_solver *s) { return s->st; }
gpe_status params_of(gpe_solver *s, gpe_params *p) {
   CHECK_HANDLE(s);
   *p = s->p;
   return GPE_OK;
}
int device_of(gpe_solver *s) { return s->dev; }
long long kernels_per_step(gpe_solver *s) { return s->cplx ? 9 : 10; }
unsigned long long plan_generation(gpe_solver *s) { return s->plan_gen; }
gpe_status tuning_as_set(gpe_solver *s, gpe_tuning *t) {
   CHECK_HANDLE(s);
   *t = s->tune;
   return GPE_OK;
}

gpe_status batch_geom(gpe_solver *s, int Ly, int Lx, BatchGeom *geom) {
   CHECK_HANDLE(s);
   return DISPATCH(s, geom(s, Ly, Lx, geom));
}

gpe_status batch_desc(gpe_solver *s, int Ly, int Lx, double g, double gd, BatchDesc *out) {
   CHECK_HANDLE(s);
   return DISPATCH(s, desc(s, Ly, Lx, g, gd, out));
}

static_assert(sizeof(State) <= sizeof(Stash::state), "step state larger than its stash");

gpe_status stash_take(gpe_solver *s, Stash *k) {
   CHECK_HANDLE(s);
   if (!k || k->psi) return fail(GPE_ERR_PARAM, "stash: null or already holding a copy");
   CK(cudaSetDevice(s->dev));
   k->bytes = s->esz_psi * (size_t) s->d.npts;
   CK(cudaMalloc(&k->psi, k->bytes));
   cudaError_t e = cudaMemcpyAsync(k->psi, s->psi, k->bytes, cudaMemcpyDeviceToDevice, s->st);
   if (e == cudaSuccess) e = cudaMemcpyAsync(k->state, s->state, sizeof(State), cudaMemcpyDeviceToHost, s->st);
   if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
   if (e != cudaSuccess) {
      stash_drop(k);
      return fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   }
   return GPE_OK;
}

gpe_status stash_restore(gpe_solver *s, Stash *k) {
   CHECK_HANDLE(s);
   if (!k || !k->psi) return fail(GPE_ERR_PARAM, "stash: nothing to restore");
   CK(cudaSetDevice(s->dev));
   cudaError_t e = cudaMemcpyAsync(s->psi, k->psi, k->bytes, cudaMemcpyDeviceToDevice, s->st);
   if (e == cudaSuccess) e = cudaMemcpyAsync(s->state, k->state, sizeof(State), cudaMemcpyHostToDevice, s->st);
   if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
   stash_drop(k);
   if (e != cudaSuccess) return fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   return GPE_OK;
}

void stash_drop(Stash *k) {
   if (k && k->psi) cudaFree(k->psi);
   if (k) k->psi = nullptr;
}

}  // namespace gpe

// --------------------------------------------------------------- snapshots
namespace {
struct SnapHeader {
   char magic[8];           // "GPESNAP1"
   uint32_t header_bytes;   // 192 (the header is zero-padded to that size)
   uint32_t version;        // 1
   gpe_params p;
   double g, gd;
   long long step;
   unsigned long long payload_bytes;
   unsigned long long fnv1a;
};
static_assert(sizeof(gpe_params) == 104, "gpe_params layout");
constexpr size_t kSnapHeaderBytes = 192;
static_assert(sizeof(SnapHeader) <= kSnapHeaderBytes, "snapshot header size");

unsigned long long fnv1a(const unsigned char *p, size_t n) {
   unsigned long long h = 1469598103934665603ULL;
   for (size_t i = 0; i < n; i++) {
      h ^= p[i];
      h *= 1099511628211ULL;
   }
   return h;
}
}  // namespace

extern "C" gpe_status gpe_snapshot_save(gpe_solver *s, const char *path, double g, double gd, long long step) {
   CHECK_HANDLE(s);
   if (!path) return fail(GPE_ERR_PARAM, "null path");
   CK(cudaSetDevice(s->dev));
   State st{};
   CK(cudaMemcpyAsync(&st, s->state, sizeof(State), cudaMemcpyDeviceToHost, s->st));
   CK(cudaStreamSynchronize(s->st));
   if (st.scale != 1.) CKS(DISPATCH(s, apply_scale(s)));
   const size_t nbytes = s->esz_psi * (size_t) s->d.npts;
   std::vector<unsigned char> buf(kSnapHeaderBytes + nbytes, 0);
   CK(cudaMemcpyAsync(buf.data() + kSnapHeaderBytes, s->psi, nbytes, cudaMemcpyDeviceToHost, s->st));
   CK(cudaStreamSynchronize(s->st));
   SnapHeader h{};
   std::memcpy(h.magic, "GPESNAP1", 8);
   h.header_bytes = (uint32_t) kSnapHeaderBytes;
   h.version = 1;
   h.p = s->p;
   h.g = g;
   h.gd = gd;
   h.step = step;
   h.payload_bytes = nbytes;
   h.fnv1a = fnv1a(buf.data() + kSnapHeaderBytes, nbytes);
   std::memcpy(buf.data(), &h, sizeof(h));
   FILE *f = std::fopen(path, "wb");
   if (!f) return fail(GPE_ERR_IO, std::string("cannot create ") + path);
   const size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
   const int c = std::fclose(f);
   if (w != buf.size() || c != 0) return fail(GPE_ERR_IO, std::string("short write to ") + path);
   return GPE_OK;
}

extern "C" gpe_status gpe_snapshot_load(gpe_solver *s, const char *path, double *g, double *gd, long long *step) {
   CHECK_HANDLE(s);
   if (!path) return fail(GPE_ERR_PARAM, "null path");
   FILE *f = std::fopen(path, "rb");
   if (!f) return fail(GPE_ERR_IO, std::string("cannot open ") + path);
   SnapHeader h{};
   unsigned char hb[kSnapHeaderBytes];
   const size_t r = std::fread(hb, 1, kSnapHeaderBytes, f);
   std::memcpy(&h, hb, sizeof(h));
   if (r != kSnapHeaderBytes || std::memcmp(h.magic, "GPESNAP1", 8) != 0 || h.version != 1 ||
       h.header_bytes != kSnapHeaderBytes) {
      std::fclose(f);
      return fail(GPE_ERR_IO, std::string(path) + " is not a version-1 solver snapshot");
   }
   if (h.p.nx != s->p.nx || h.p.ny != s->p.ny || h.p.nz != s->p.nz || h.p.mode != s->p.mode ||
       h.p.precision != s->p.precision) {
      std::fclose(f);
      return fail(GPE_ERR_PARAM, "snapshot grid, mode or precision differs from the handle's");
   }
   const size_t nbytes = s->esz_psi * (size_t) s->d.npts;
   std::vector<unsigned char> buf(nbytes);
   const size_t rp = h.payload_bytes == nbytes ? std::fread(buf.data(), 1, nbytes, f) : 0;
   std::fclose(f);
   if (rp != nbytes || fnv1a(buf.data(), nbytes) != h.fnv1a)
      return fail(GPE_ERR_IO, std::string(path) + ": payload short or checksum mismatch");
   CK(cudaSetDevice(s->dev));
   CK(cudaMemcpyAsync(s->psi, buf.data(), nbytes, cudaMemcpyHostToDevice, s->st));
   CK(cudaStreamSynchronize(s->st));
   k_state_set<<<1, 1, 0, s->st>>>(s->state, 1.);
   CKL();
   if (g) *g = h.g;
   if (gd) *gd = h.gd;
   if (step) *step = h.step;
   return GPE_OK;
}
