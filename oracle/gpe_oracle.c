/*
 * gpe_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain FP64 CPU restatement of one MPI rank of the reference programs
 * src/imag3d-mpicuda/imag3d-mpicuda.cu ("imag") and
 * src/real3d-mpicuda/real3d-mpicuda.cu ("real"), with
 * src/utils/diffint.cu ("diffint").  At one rank every distributed transpose
 * of the reference is the identity, so the x sweep and the x FFT read x lines
 * directly.  The FFT is this file's own mixed-radix Cooley-Tukey (cuFFT's
 * arithmetic is closed; only the transform it computes is restated).
 *
 * Parallelised with OpenMP over independent lines/planes only; every
 * reduction runs sequentially in the reference's nested order.
 */
#include "gpe_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* The reference's truncated pi (imag:69, real:71). */
#define REF_PI 3.14159265358979

/* ------------------------------------------------------------------ FFT */

typedef struct {
   long n;
   int nf;
   int f[64];
   cplx *tw; /* tw[e] = exp(-2 pi i e / n), e in [0, n) */
} fftplan;

static int fft_factor(long n, int *f) {
   int nf = 0;
   static const int pref[] = {4, 2, 3, 5, 7};
   long m = n;
   for (int pi = 0; pi < 5; pi++) {
      while (m % pref[pi] == 0) { f[nf++] = pref[pi]; m /= pref[pi]; }
   }
   /* any leftover prime factor is handled by a generic radix */
   for (long p = 11; m > 1; p += 2) {
      while (m % p == 0) { f[nf++] = (int) p; m /= p; }
   }
   return nf;
}

static void fft_plan_init(fftplan *P, long n) {
   P->n = n;
   P->nf = fft_factor(n, P->f);
   P->tw = (cplx *) malloc(sizeof(cplx) * (size_t) n);
   for (long e = 0; e < n; e++) {
      long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double) e / (long double) n;
      P->tw[e] = (double) cosl(a) + I * (double) sinl(a);
   }
}

static void fft_plan_free(fftplan *P) { free(P->tw); }

static inline cplx fft_w(const fftplan *P, long e, int inv) {
   cplx w = P->tw[e % P->n];
   return inv ? conj(w) : w;
}

/* Decimation-in-time recursion: out[0..n) = DFT of in[0], in[is], ... */
static void fft_rec(const cplx *in, long is, cplx *out, long n, const fftplan *P,
                    int level, long twmul, int inv) {
   if (n == 1) { out[0] = in[0]; return; }
   int r = P->f[level];
   long m = n / r;
   for (int q = 0; q < r; q++)
      fft_rec(in + q * is, is * r, out + q * m, m, P, level + 1, twmul * r, inv);
   cplx t[64], y[64];
   for (long k = 0; k < m; k++) {
      for (int q = 0; q < r; q++) t[q] = out[q * m + k] * fft_w(P, (long) q * k * twmul, inv);
      for (int s = 0; s < r; s++) {
         cplx acc = 0;
         for (int q = 0; q < r; q++) acc += t[q] * fft_w(P, (long) ((q * s) % r) * m * twmul, inv);
         y[s] = acc;
      }
      for (int s = 0; s < r; s++) out[k + s * m] = y[s];
   }
}

/* In-place transform of a strided line through a scratch of 2n. */
static void fft_line(cplx *a, long stride, const fftplan *P, int inv, cplx *scratch) {
   long n = P->n;
   for (long j = 0; j < n; j++) scratch[j] = a[j * stride];
   fft_rec(scratch, 1, scratch + n, n, P, 0, 1, inv);
   for (long j = 0; j < n; j++) a[j * stride] = scratch[n + j];
}

void orc_fft_1d(long n, double *re, double *im, int inverse) {
   fftplan P;
   fft_plan_init(&P, n);
   cplx *a = (cplx *) malloc(sizeof(cplx) * (size_t) n);
   cplx *sc = (cplx *) malloc(sizeof(cplx) * (size_t) (2 * n));
   for (long j = 0; j < n; j++) a[j] = re[j] + I * im[j];
   fft_line(a, 1, &P, inverse, sc);
   for (long j = 0; j < n; j++) { re[j] = creal(a[j]); im[j] = cimag(a[j]); }
   free(a); free(sc);
   fft_plan_free(&P);
}

/* ------------------------------------------------------------ solver state */

struct orc {
   orc_params p;
   double par;
   long nx2, ny2, nz2, nzh;
   double *x, *y, *z, *x2, *y2, *z2;
   /* Crank-Nicolson coefficients per axis (imag: real values in complex). */
   cplx A0[3], A0r[3], A[3], mA[3];
   cplx *calpha[3], *cgamma[3];
   cplx *psi;     /* [nx][ny][nz] */
   cplx *beta;    /* [nx][ny][nz] Thomas scratch */
   double *phi;   /* [nx][ny][nz] dipolar term (unnormalised inverse FFT) */
   cplx *spec;    /* [nx][ny][nzh] */
   double *potdd; /* [nx][ny][nzh] half spectrum of Udd */
   fftplan fx, fy, fz;
};

void orc_set_threads(int n) {
#ifdef _OPENMP
   if (n > 0) omp_set_num_threads(n);
#else
   (void) n;
#endif
}

static inline double pot_at(const orc_t *s, long i, long j, long k) {
   /* initpot (imag:872-889): 0.5 * par * (gamma^2 x^2 + nu^2 y^2 + lambda^2 z^2) */
   double vg2 = s->p.gamma * s->p.gamma, vn2 = s->p.nu * s->p.nu, vl2 = s->p.lambda * s->p.lambda;
   return 0.5 * s->par * (vg2 * s->x2[i] + vn2 * s->y2[j] + vl2 * s->z2[k]);
}

/* gencoef (imag:894-931 real, real:991-1035 complex). */
static void gencoef_axis(orc_t *s, int ax, long n, double d2) {
   double c = s->p.dt / d2 / (3. - s->par);
   if (s->p.mode == 0) {
      s->A0[ax] = 1. + c;
      s->A0r[ax] = 1. - c;
      s->A[ax] = -0.5 * c;
      s->mA[ax] = -s->A[ax];
   } else {
      s->A0[ax] = 1. + I * c;
      s->A0r[ax] = conj(s->A0[ax]);
      s->A[ax] = I * (-0.5 * c);
      s->mA[ax] = I * (-cimag(s->A[ax]));
   }
   cplx *al = s->calpha[ax] = (cplx *) calloc((size_t) (n - 1), sizeof(cplx));
   cplx *ga = s->cgamma[ax] = (cplx *) calloc((size_t) (n - 1), sizeof(cplx));
   al[n - 2] = 0.;
   ga[n - 2] = -1. / s->A0[ax];
   for (long i = n - 2; i > 0; i--) {
      al[i - 1] = s->A[ax] * ga[i];
      ga[i - 1] = -1. / (s->A0[ax] + s->A[ax] * al[i - 1]);
   }
}

/* initpotdd (imag:945-980): half spectrum kz < Nz/2+1 only. */
static void initpotdd(orc_t *s) {
   const long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, nzh = s->nzh;
   double pi = REF_PI, cutoff = s->p.cutoff;
   double dkx = 2. * pi / (nx * s->p.dx), dky = 2. * pi / (ny * s->p.dy), dkz = 2. * pi / (nz * s->p.dz);
   double *kx2 = (double *) malloc(sizeof(double) * nx), *ky2 = (double *) malloc(sizeof(double) * ny),
          *kz2 = (double *) malloc(sizeof(double) * nz);
   for (long i = 0; i < nx; i++) { double k = (i < s->nx2) ? i * dkx : (i - s->nx2 - s->nx2) * dkx; kx2[i] = k * k; }
   for (long i = 0; i < ny; i++) { double k = (i < s->ny2) ? i * dky : (i - s->ny2 - s->ny2) * dky; ky2[i] = k * k; }
   for (long i = 0; i < nz; i++) { double k = (i < s->nz2) ? i * dkz : (i - s->nz2 - s->nz2) * dkz; kz2[i] = k * k; }
   s->potdd = (double *) malloc(sizeof(double) * (size_t) (nx * ny * nzh));
#pragma omp parallel for collapse(2)
   for (long i = 0; i < nx; i++)
      for (long j = 0; j < ny; j++)
         for (long k = 0; k < nzh; k++) {
            double xk = sqrt(kz2[k] + kx2[i] + ky2[j]);
            double tmp = 1. + 3. * cos(xk * cutoff) / (xk * xk * cutoff * cutoff)
                         - 3. * sin(xk * cutoff) / (xk * xk * xk * cutoff * cutoff * cutoff);
            s->potdd[(i * ny + j) * nzh + k] = (4. * pi * (3. * kz2[k] / (kx2[i] + ky2[j] + kz2[k]) - 1.) / 3.) * tmp;
         }
   s->potdd[0] = 0.;
   free(kx2); free(ky2); free(kz2);
}

orc_t *orc_create(const orc_params *p) {
   if (p->nx < 4 || p->ny < 4 || p->nz < 4 || (p->nx % 2) || (p->ny % 2) || (p->nz % 2)) return NULL;
   orc_t *s = (orc_t *) calloc(1, sizeof(orc_t));
   s->p = *p;
   s->par = (p->opt == 2) ? 2. : 1.;
   s->nx2 = p->nx / 2; s->ny2 = p->ny / 2; s->nz2 = p->nz / 2;
   s->nzh = s->nz2 + 1;
   long nx = p->nx, ny = p->ny, nz = p->nz;
   s->x = malloc(sizeof(double) * nx); s->x2 = malloc(sizeof(double) * nx);
   s->y = malloc(sizeof(double) * ny); s->y2 = malloc(sizeof(double) * ny);
   s->z = malloc(sizeof(double) * nz); s->z2 = malloc(sizeof(double) * nz);
   /* space mesh from initpsi (imag:842-855) */
   for (long i = 0; i < nx; i++) { s->x[i] = (i - s->nx2) * p->dx; s->x2[i] = s->x[i] * s->x[i]; }
   for (long j = 0; j < ny; j++) { s->y[j] = (j - s->ny2) * p->dy; s->y2[j] = s->y[j] * s->y[j]; }
   for (long k = 0; k < nz; k++) { s->z[k] = (k - s->nz2) * p->dz; s->z2[k] = s->z[k] * s->z[k]; }
   gencoef_axis(s, 0, nx, p->dx * p->dx);
   gencoef_axis(s, 1, ny, p->dy * p->dy);
   gencoef_axis(s, 2, nz, p->dz * p->dz);
   size_t npts = (size_t) (nx * ny * nz);
   s->psi = (cplx *) calloc(npts, sizeof(cplx));
   s->beta = (cplx *) calloc(npts, sizeof(cplx));
   s->phi = (double *) calloc(npts, sizeof(double));
   s->spec = (cplx *) calloc((size_t) (nx * ny * s->nzh), sizeof(cplx));
   initpotdd(s);
   fft_plan_init(&s->fx, nx);
   fft_plan_init(&s->fy, ny);
   fft_plan_init(&s->fz, nz);
   return s;
}

void orc_destroy(orc_t *s) {
   if (!s) return;
   free(s->x); free(s->y); free(s->z); free(s->x2); free(s->y2); free(s->z2);
   for (int a = 0; a < 3; a++) { free(s->calpha[a]); free(s->cgamma[a]); }
   free(s->psi); free(s->beta); free(s->phi); free(s->spec); free(s->potdd);
   fft_plan_free(&s->fx); fft_plan_free(&s->fy); fft_plan_free(&s->fz);
   free(s);
}

#define IDX(i, j, k) (((i) * s->p.ny + (j)) * s->p.nz + (k))

void orc_init_gaussian(orc_t *s) {
   /* initpsi (imag:835-867): cpsi = sqrt(pi * sqrt(pi / (gamma nu lambda))) */
   double pi = REF_PI;
   double cpsi = sqrt(pi * sqrt(pi / (s->p.gamma * s->p.nu * s->p.lambda)));
#pragma omp parallel for collapse(2)
   for (long i = 0; i < s->p.nx; i++)
      for (long j = 0; j < s->p.ny; j++)
         for (long k = 0; k < s->p.nz; k++) {
            double tmp = exp(-0.5 * (s->p.gamma * s->x2[i] + s->p.nu * s->y2[j] + s->p.lambda * s->z2[k]));
            s->psi[IDX(i, j, k)] = tmp / cpsi;
         }
}

void orc_init_from_density(orc_t *s, const double *rho) {
   size_t n = (size_t) (s->p.nx * s->p.ny * s->p.nz);
   for (size_t q = 0; q < n; q++) s->psi[q] = sqrt(rho[q]);
}

void orc_set_psi(orc_t *s, const double *re, const double *im) {
   size_t n = (size_t) (s->p.nx * s->p.ny * s->p.nz);
   for (size_t q = 0; q < n; q++) s->psi[q] = re[q] + I * (im ? im[q] : 0.);
}

void orc_get_psi(const orc_t *s, double *re, double *im) {
   size_t n = (size_t) (s->p.nx * s->p.ny * s->p.nz);
   for (size_t q = 0; q < n; q++) { re[q] = creal(s->psi[q]); if (im) im[q] = cimag(s->psi[q]); }
}

void orc_get_phi(const orc_t *s, double *phi) {
   memcpy(phi, s->phi, sizeof(double) * (size_t) (s->p.nx * s->p.ny * s->p.nz));
}

void orc_get_potdd(const orc_t *s, double *out) {
   memcpy(out, s->potdd, sizeof(double) * (size_t) (s->p.nx * s->p.ny * s->nzh));
}

static inline double dens(const orc_t *s, cplx v) {
   if (s->p.mode == 0) { double r = creal(v); return r * r; }
   return creal(v) * creal(v) + cimag(v) * cimag(v);
}

/* simpint (diffint:37-66), same three accumulators and the same order. */
double orc_simpint(double h, const double *f, long N) {
   double sumi = 0., sumj = 0., sumk = 0.;
   for (long cnti = 1; cnti < N - 1; cnti += 2) {
      sumi += f[cnti];
      sumj += f[cnti - 1];
      sumk += f[cnti + 1];
   }
   double sum = sumj + 4. * sumi + sumk;
   if (N % 2 == 0) sum += (5. * f[N - 1] + 8. * f[N - 2] - f[N - 3]) / 4.;
   return sum * h / 3.;
}

/* Integral of f[nx][ny][nz] in the reference's nesting: z rows, then y, then x
 * (simpint3d_kernel diffint:106, simpint2d_kernel diffint:95, simpint_gpu). */
static double integrate_xyz(const orc_t *s, const double *f) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
   double *tx = (double *) malloc(sizeof(double) * nx);
#pragma omp parallel
   {
      double *ty = (double *) malloc(sizeof(double) * ny);
#pragma omp for
      for (long i = 0; i < nx; i++) {
         for (long j = 0; j < ny; j++) ty[j] = orc_simpint(s->p.dz, f + (i * ny + j) * nz, nz);
         tx[i] = orc_simpint(s->p.dy, ty, ny);
      }
      free(ty);
   }
   double r = orc_simpint(s->p.dx, tx, nx);
   free(tx);
   return r;
}

double orc_calcnorm(orc_t *s, int renormalize) {
   size_t n = (size_t) (s->p.nx * s->p.ny * s->p.nz);
   double *f = (double *) malloc(sizeof(double) * n);
#pragma omp parallel for
   for (size_t q = 0; q < n; q++) f[q] = dens(s, s->psi[q]);
   double norm = sqrt(integrate_xyz(s, f));
   free(f);
   if (renormalize) {
      /* calcnorm_kernel (imag:1220-1233): psi *= 1 / norm */
      double tmp = 1. / norm;
#pragma omp parallel for
      for (size_t q = 0; q < n; q++) s->psi[q] = creal(s->psi[q]) * tmp + I * (cimag(s->psi[q]) * tmp);
   }
   return norm;
}

void orc_calcpsidd2(orc_t *s) {
   const long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, nzh = s->nzh;
   cplx *sp = s->spec;
   /* calcpsi2 + D2Z along z (2D {Ny, Nz} plan; its z part here) */
#pragma omp parallel
   {
      cplx *row = (cplx *) malloc(sizeof(cplx) * nz);
      cplx *sc = (cplx *) malloc(sizeof(cplx) * 2 * (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
#pragma omp for collapse(2)
      for (long i = 0; i < nx; i++)
         for (long j = 0; j < ny; j++) {
            for (long k = 0; k < nz; k++) row[k] = dens(s, s->psi[IDX(i, j, k)]);
            fft_line(row, 1, &s->fz, 0, sc);
            for (long k = 0; k < nzh; k++) sp[(i * ny + j) * nzh + k] = row[k];
         }
      /* y part of the D2Z */
#pragma omp for collapse(2)
      for (long i = 0; i < nx; i++)
         for (long k = 0; k < nzh; k++) fft_line(sp + i * ny * nzh + k, nzh, &s->fy, 0, sc);
      /* Z2Z along x, multiply by Udd (calcpsidd2_kernel1 imag:1571), inverse along x */
#pragma omp for collapse(2)
      for (long j = 0; j < ny; j++)
         for (long k = 0; k < nzh; k++) {
            cplx *line = sp + j * nzh + k;
            long st = ny * nzh;
            fft_line(line, st, &s->fx, 0, sc);
            for (long i = 0; i < nx; i++) {
               double t = s->potdd[(i * ny + j) * nzh + k];
               line[i * st] = creal(line[i * st]) * t + I * (cimag(line[i * st]) * t);
            }
            fft_line(line, st, &s->fx, 1, sc);
         }
      /* Z2D 2D {Ny, Nz}: inverse along y, then the Hermitian inverse along z */
#pragma omp for collapse(2)
      for (long i = 0; i < nx; i++)
         for (long k = 0; k < nzh; k++) fft_line(sp + i * ny * nzh + k, nzh, &s->fy, 1, sc);
#pragma omp for collapse(2)
      for (long i = 0; i < nx; i++)
         for (long j = 0; j < ny; j++) {
            const cplx *h = sp + (i * ny + j) * nzh;
            for (long k = 0; k < nz; k++) row[k] = (k < nzh) ? h[k] : conj(h[nz - k]);
            fft_line(row, 1, &s->fz, 1, sc);
            for (long k = 0; k < nz; k++) s->phi[IDX(i, j, k)] = creal(row[k]);
         }
      free(row); free(sc);
   }
   /* boundary planes at one rank: cudaMemcpy of plane 0, kernel2a (imag:1591),
    * kernel2b (imag:1605) with last = 1.  Plane 0 is untouched by 2b for
    * k < Nz-1 and j < Ny-1, so copying from phi itself is equivalent. */
   for (long j = 0; j < ny - 1; j++)
      for (long k = 0; k < nz - 1; k++) s->phi[IDX(nx - 1, j, k)] = s->phi[IDX(0, j, k)];
   for (long i = 0; i < nx - 1; i++) {
      for (long k = 0; k < nz - 1; k++) s->phi[IDX(i, ny - 1, k)] = s->phi[IDX(i, 0, k)];
      for (long j = 0; j < ny - 1; j++) s->phi[IDX(i, j, nz - 1)] = s->phi[IDX(i, j, 0)];
   }
}

void orc_calcnu(orc_t *s, double g, double gd) {
   size_t n = (size_t) (s->p.nx * s->p.ny * s->p.nz);
   long nn = s->p.nx * s->p.ny * s->p.nz;
   double dt = s->p.dt;
#pragma omp parallel for collapse(2)
   for (long i = 0; i < s->p.nx; i++)
      for (long j = 0; j < s->p.ny; j++)
         for (long k = 0; k < s->p.nz; k++) {
            size_t q = (size_t) IDX(i, j, k);
            cplx psit = s->psi[q];
            double psidd2lin = (s->phi[q] / nn) * gd;
            double pottmp = pot_at(s, i, j, k);
            if (s->p.mode == 0) {
               /* calcnu_kernel imag:1759-1783 */
               double p = creal(psit);
               double psi2lin = p * p * g;
               pottmp = dt * (pottmp + psi2lin + psidd2lin);
               s->psi[q] = p * exp(-pottmp);
            } else {
               /* calcnu_kernel real:1856-1883: psi * (cos(-th), sin(-th)) */
               double psi2lin = dens(s, psit) * g;
               pottmp = dt * (pottmp + psi2lin + psidd2lin);
               cplx e = cos(-pottmp) + I * sin(-pottmp);
               s->psi[q] = psit * e;
            }
         }
   (void) n;
}

/* One Thomas sweep along a line: elements a[0], a[st], ..., beta alongside.
 * calclux_kernel (imag:1802-1844) / calcluz_kernel real:2014-2040. */
static void thomas_line(orc_t *s, int ax, long n, cplx *a, cplx *b, long st) {
   const cplx A = s->A[ax], A0r = s->A0r[ax], mA = s->mA[ax];
   const cplx *al = s->calpha[ax], *ga = s->cgamma[ax];
   b[(n - 2) * st] = a[(n - 1) * st];
   for (long i = n - 2; i > 0; i--) {
      cplx c = mA * a[(i + 1) * st] + A0r * a[i * st] - A * a[(i - 1) * st];
      b[(i - 1) * st] = ga[i] * (A * b[i * st] - c);
   }
   a[0] = 0.;
   for (long i = 0; i < n - 2; i++) a[(i + 1) * st] = al[i] * a[i * st] + b[i * st];
   a[(n - 1) * st] = 0.;
}

void orc_calclux(orc_t *s) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
#pragma omp parallel for collapse(2)
   for (long j = 0; j < ny; j++)
      for (long k = 0; k < nz; k++)
         thomas_line(s, 0, nx, s->psi + IDX(0, j, k), s->beta + IDX(0, j, k), ny * nz);
}

void orc_calcluy(orc_t *s) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
#pragma omp parallel for collapse(2)
   for (long i = 0; i < nx; i++)
      for (long k = 0; k < nz; k++)
         thomas_line(s, 1, ny, s->psi + IDX(i, 0, k), s->beta + IDX(i, 0, k), nz);
}

void orc_calcluz(orc_t *s) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
#pragma omp parallel for collapse(2)
   for (long i = 0; i < nx; i++)
      for (long j = 0; j < ny; j++)
         thomas_line(s, 2, nz, s->psi + IDX(i, j, 0), s->beta + IDX(i, j, 0), 1);
}

void orc_run(orc_t *s, long nsteps, double *g, double *gd, double g_inc, double gd_inc, double *norm) {
   double nrm = NAN;
   for (long c = 0; c < nsteps; c++) {
      *g += g_inc;
      *gd += gd_inc;
      orc_calcpsidd2(s);
      orc_calcnu(s, *g, *gd);
      orc_calclux(s);
      orc_calcluy(s);
      orc_calcluz(s);
      if (s->p.mode == 0) nrm = orc_calcnorm(s, 1);
   }
   if (norm) *norm = nrm;
}

/* 4th-order first derivative with the reference's edge rules
 * (calcmuen_kernel1x imag:1293-1338). */
static inline double fd(const double *f, long i, long n, long st, double h) {
   if (i == 0 || i == n - 1) return 0.;
   if (i == 1) return (f[2 * st] - f[0]) / (2. * h);
   if (i == n - 2) return (f[(n - 1) * st] - f[(n - 3) * st]) / (2. * h);
   return (f[(i - 2) * st] - 8. * f[(i - 1) * st] + 8. * f[(i + 1) * st] - f[(i + 2) * st]) / (12. * h);
}

void orc_calcmuen(orc_t *s, double g, double gd, double *mu, double *en) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, nn = nx * ny * nz;
   size_t n = (size_t) nn;
   orc_calcpsidd2(s);
   /* imag differentiates psi, real differentiates |psi| (real:1401) */
   double *a = (double *) malloc(sizeof(double) * n);
   double *tmu = (double *) malloc(sizeof(double) * n), *ten = (double *) malloc(sizeof(double) * n);
#pragma omp parallel for
   for (size_t q = 0; q < n; q++) a[q] = (s->p.mode == 0) ? creal(s->psi[q]) : cabs(s->psi[q]);
   double par = s->par;
#pragma omp parallel for collapse(2)
   for (long i = 0; i < nx; i++)
      for (long j = 0; j < ny; j++)
         for (long k = 0; k < nz; k++) {
            size_t q = (size_t) IDX(i, j, k);
            double dxv = fd(a + IDX(0, j, k), i, nx, ny * nz, s->p.dx);
            double dyv = fd(a + IDX(i, 0, k), j, ny, nz, s->p.dy);
            double dzv = fd(a + IDX(i, j, 0), k, nz, 1, s->p.dz);
            double dpsi = (dxv * dxv) / (3. - par);
            dpsi += (dyv * dyv) / (3. - par);
            dpsi += (dzv * dzv) / (3. - par);
            double psi2 = dens(s, s->psi[q]);
            double psi2lin = psi2 * g;
            double psidd2lin = (s->phi[q] / nn) * gd;
            double tmppot = pot_at(s, i, j, k);
            tmu[q] = (tmppot + psi2lin + psidd2lin) * psi2 + dpsi;
            ten[q] = (tmppot + 0.5 * psi2lin + 0.5 * psidd2lin) * psi2 + dpsi;
         }
   *mu = integrate_xyz(s, tmu);
   *en = integrate_xyz(s, ten);
   free(a); free(tmu); free(ten);
}

void orc_calcrms(orc_t *s, double *rms) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
   size_t n = (size_t) (nx * ny * nz);
   double *f = (double *) malloc(sizeof(double) * n);
   const double *w[3] = {s->x2, s->y2, s->z2};
   for (int ax = 0; ax < 3; ax++) {
#pragma omp parallel for collapse(2)
      for (long i = 0; i < nx; i++)
         for (long j = 0; j < ny; j++)
            for (long k = 0; k < nz; k++) {
               size_t q = (size_t) IDX(i, j, k);
               long c = (ax == 0) ? i : (ax == 1) ? j : k;
               f[q] = w[ax][c] * dens(s, s->psi[q]);
            }
      rms[1 + ax] = sqrt(integrate_xyz(s, f));
   }
   rms[0] = sqrt(rms[1] * rms[1] + rms[2] * rms[2] + rms[3] * rms[3]);
   free(f);
}

double orc_psi_center2(const orc_t *s) {
   cplx v = s->psi[(s->nx2 * s->p.ny + s->ny2) * s->p.nz + s->nz2];
   return dens(s, v);
}

/* Density files (imag:1944-2399).  Integrals use the reference's nesting. */
long orc_density(orc_t *s, int kind, long sx, long sy, long sz, double *out) {
   long nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
   long o = 0;
   double *ty = (double *) malloc(sizeof(double) * (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
   double *tz = (double *) malloc(sizeof(double) * (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
   double *tx = (double *) malloc(sizeof(double) * nx);
#define D(i, j, k) dens(s, s->psi[IDX(i, j, k)])
   switch (kind) {
   case 0: /* outdenx: z then y (imag:1944-1962) */
      for (long i = 0; i < nx; i += sx) {
         for (long j = 0; j < ny; j++) {
            for (long k = 0; k < nz; k++) tz[k] = D(i, j, k);
            ty[j] = orc_simpint(s->p.dz, tz, nz);
         }
         out[o++] = s->x[i];
         out[o++] = orc_simpint(s->p.dy, ty, ny);
      }
      break;
   case 1: /* outdeny: z then x (imag:1985-2004) */
      for (long j = 0; j < ny; j += sy) {
         for (long i = 0; i < nx; i++) {
            for (long k = 0; k < nz; k++) tz[k] = D(i, j, k);
            tx[i] = orc_simpint(s->p.dz, tz, nz);
         }
         out[o++] = s->y[j];
         out[o++] = orc_simpint(s->p.dx, tx, nx);
      }
      break;
   case 2: /* outdenz: y then x (imag:2023-2050) */
      for (long k = 0; k < nz; k += sz) {
         for (long i = 0; i < nx; i++) {
            for (long j = 0; j < ny; j++) ty[j] = D(i, j, k);
            tx[i] = orc_simpint(s->p.dy, ty, ny);
         }
         out[o++] = s->z[k];
         out[o++] = orc_simpint(s->p.dx, tx, nx);
      }
      break;
   case 3: /* outdenxy: integrate z (imag:2072-2098) */
      for (long i = 0; i < nx; i += sx)
         for (long j = 0; j < ny; j += sy) {
            for (long k = 0; k < nz; k++) tz[k] = D(i, j, k);
            out[o++] = s->x[i]; out[o++] = s->y[j]; out[o++] = orc_simpint(s->p.dz, tz, nz);
         }
      break;
   case 4: /* outdenxz: integrate y (imag:2119-2145) */
      for (long i = 0; i < nx; i += sx)
         for (long k = 0; k < nz; k += sz) {
            for (long j = 0; j < ny; j++) ty[j] = D(i, j, k);
            out[o++] = s->x[i]; out[o++] = s->z[k]; out[o++] = orc_simpint(s->p.dy, ty, ny);
         }
      break;
   case 5: /* outdenyz: integrate x (imag:2166-2194) */
      for (long j = 0; j < ny; j += sy)
         for (long k = 0; k < nz; k += sz) {
            for (long i = 0; i < nx; i++) tx[i] = D(i, j, k);
            out[o++] = s->y[j]; out[o++] = s->z[k]; out[o++] = orc_simpint(s->p.dx, tx, nx);
         }
      break;
   case 6: /* outpsi2xy: plane z = Nz/2 (imag:2215-2254) */
      for (long i = 0; i < nx; i += sx)
         for (long j = 0; j < ny; j += sy) { out[o++] = s->x[i]; out[o++] = s->y[j]; out[o++] = D(i, j, s->nz2); }
      break;
   case 7: /* outpsi2xz: plane y = Ny/2 (imag:2256-2293) */
      for (long i = 0; i < nx; i += sx)
         for (long k = 0; k < nz; k += sz) { out[o++] = s->x[i]; out[o++] = s->z[k]; out[o++] = D(i, s->ny2, k); }
      break;
   case 8: /* outpsi2yz: plane x = Nx/2 (imag:2295-2353) */
      for (long j = 0; j < ny; j += sy)
         for (long k = 0; k < nz; k += sz) { out[o++] = s->y[j]; out[o++] = s->z[k]; out[o++] = D(s->nx2, j, k); }
      break;
   case 9: /* outdenxyz: raw 3D (imag:2355-2399) */
      for (long i = 0; i < nx; i += sx)
         for (long j = 0; j < ny; j += sy)
            for (long k = 0; k < nz; k += sz) out[o++] = D(i, j, k);
      break;
   default:
      o = -1;
   }
#undef D
   free(ty); free(tz); free(tx);
   return o;
}
