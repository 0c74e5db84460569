/*
 * gpe_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU FP64 restatement of the dipolar Gross-Pitaevskii split-step
 * Crank-Nicolson propagator of DBEC-GP-MPI-CUDA (imag3d-mpicuda and
 * real3d-mpicuda) at one MPI rank.  Only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py may load this library.
 *
 * Every function cites the reference file:line it restates, relative to the
 * reference project root ("imag" = src/imag3d-mpicuda/imag3d-mpicuda.cu,
 * "real" = src/real3d-mpicuda/real3d-mpicuda.cu).
 */
#ifndef GPE_ORACLE_H
#define GPE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors the reference's readpar() globals (imag:650-829, real:675-883). */
typedef struct {
   int mode;        /* 0 = imaginary time (real psi), 1 = real time (complex psi) */
   int opt;         /* OPTION: par = 2 if opt == 2 else 1 (imag:201-202) */
   long nx, ny, nz;
   double dx, dy, dz, dt;
   double gamma, nu, lambda;
   double cutoff;
} orc_params;

typedef struct orc orc_t;

orc_t *orc_create(const orc_params *p);
void orc_destroy(orc_t *s);
void orc_set_threads(int n);

/* initpsi Gaussian (imag:835-867, real:914-923). */
void orc_init_gaussian(orc_t *s);
/* psi = (sqrt(rho), 0) as real3d reads imag3d-den.bin (real:925-947). */
void orc_init_from_density(orc_t *s, const double *rho);
void orc_set_psi(orc_t *s, const double *re, const double *im);
void orc_get_psi(const orc_t *s, double *re, double *im);

/* calcnorm (imag:1194-1233 with renormalisation, real:1304-1322 without). */
double orc_calcnorm(orc_t *s, int renormalize);
/* calcpsidd2_mem (imag:1460-1510): phi = IFFT[Udd * FFT[|psi|^2]] + boundary planes. */
void orc_calcpsidd2(orc_t *s);
void orc_get_phi(const orc_t *s, double *phi);
void orc_get_potdd(const orc_t *s, double *potdd_half);
/* calcnu (imag:1752-1783, real:1849-1883); uses phi from orc_calcpsidd2. */
void orc_calcnu(orc_t *s, double g, double gd);
/* Crank-Nicolson Thomas sweeps (imag:1790-1942, real:1890-2040). */
void orc_calclux(orc_t *s);
void orc_calcluy(orc_t *s);
void orc_calcluz(orc_t *s);
/* One full step loop, as the phase loops in imag:315-325 / real:334-338:
 * before each step g += g_inc, gd += gd_inc (pass 0 for fixed couplings).
 * In imaginary time each step ends with calcnorm(renormalize); the last
 * pre-renormalisation norm is returned in *norm (NaN in real time). */
void orc_run(orc_t *s, long nsteps, double *g, double *gd, double g_inc, double gd_inc, double *norm);
/* calcmuen (imag:1250-1450, real:1339-1543): mu and E (not divided by par). */
void orc_calcmuen(orc_t *s, double g, double gd, double *mu, double *en);
/* calcrms (imag:1639-1744): rms[0]=<r>, rms[1..3]=<x>,<y>,<z>. */
void orc_calcrms(orc_t *s, double *rms);
/* |psi(Nx/2, Ny/2, Nz/2)|^2 as printed in the out file (imag:246). */
double orc_psi_center2(const orc_t *s);
/* Density outputs (imag:1944-2399); out receives the same doubles the
 * reference writes to the file (pairs, triples or the raw 3D block).
 * kind: 0..2 = 1d x/y/z, 3..5 = 2d xy/xz/yz, 6..8 = 3d cuts xy0/x0z/0yz,
 * 9 = 3D density.  Returns the number of doubles written. */
long orc_density(orc_t *s, int kind, long outstpx, long outstpy, long outstpz, double *out);

/* Standalone FFT used by the oracle (tests pin it against numpy). */
void orc_fft_1d(long n, double *re, double *im, int inverse);

/* composite Simpson rule exactly as diffint.cu:37-66 */
double orc_simpint(double h, const double *f, long n);

#ifdef __cplusplus
}
#endif

#endif
