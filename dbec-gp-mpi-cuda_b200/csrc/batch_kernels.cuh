// batch_kernels.cuh -- one launch per pass of the split step over many
// independent solves (gpe_batch_* in include/gpe.h).
//
// The reference runs one solve per MPI job; a batch steps many solves with
// their own grids, parameters and couplings together.  Every pass of the step
// (z forward FFT, y FFT, x convolution, inverse y FFT, z inverse FFT, phi
// boundary planes, x sweep with calcnu, y sweep, z sweep, norm) is ONE launch
// over the tiles of all instances of a group (same mode and precision): a
// per-instance descriptor table in device memory holds each instance's
// dimensions, pointers, FFT plans, coefficient tables, couplings and TMA
// tensor maps, and a work list per pass maps a tile to its instance and its
// place in that instance.  The per-tile arithmetic is the single
// solve's own (the *_body functions of step_kernels.cuh and the sweep helpers
// of sweep_kernels.cuh), so an instance's step is bit for bit its solo step.
//
// Tensor maps read from global memory are acquired through the tensormap
// proxy (fence.proxy.tensormap::generic.acquire) by the thread that issues
// the copies, before their first use in the CTA (and again whenever a
// persistent CTA moves on to another instance).
#pragma once

#include "step_kernels.cuh"
#include "sweep_kernels.cuh"

namespace gpe {

// Everything one sweep tile of one instance needs.
struct SweepView {
   SegTab tb;
   Trap trap;
   LinPhase lin;
   Dims d;
   const State *st;
   uint32_t *err;
   void *psi;               // z sweep: psi rows
   const double *wz, *wz2;  // z sweep: Simpson weights (norm, rms partials)
   double *rowsum, *rowsum2;
   double g, gd, dt, hz3;
   int TW, boxn, nbox, LS;
};

// Passes of the step (work-list index).
enum BatchPass { kPZfwd = 0, kPYfft, kPXconv, kPYinv, kPZinv, kPPhifix, kPXsweep, kPYsweep, kPZsweep, kPNorm, kNPass };

// One instance of a batch.  Tensor maps need 64-byte alignment; the table is
// a cudaMalloc'd array of these.
struct alignas(64) BatchDesc {
   CUtensorMap tm_psi[2];  // x and y sweep tiles of psi
   CUtensorMap tm_phi;     // x sweep tiles of phi
   CUtensorMap tm_spec_y, tm_spec_x;
   SweepView sv[3];
   FftPlan px, py, ph;
   Dims d;
   void *psi, *spec, *phi;
   const void *twx, *twy, *twz;
   const double *udd;
   State *state;
   uint32_t *err;
   double *rowA, *xs;
   double hx, hy;
   int LSr, LSo, boxy, nboxy, boxx, nboxx, Ly, Lx;
};

// Launch geometry of one instance under the batch's fixed tile choices (z
// passes: 8-row tiles; y / x passes: Ly / Lx kz columns; sweeps: the
// instance's own lines per CTA and segments, 2-stage pipelines).
struct BatchGeom {
   long long tiles[kNPass];  // CTAs (FFT passes, norm, planes) or tiles (sweeps)
   unsigned threads[kNPass];
   size_t smem[kNPass];      // dynamic shared memory of one CTA (FFT passes)
   int zppt;                 // points per thread of the z passes
   int mseg[3];              // compile-time segment bound of each sweep
   uint32_t stage[3];        // sweeps: bytes of one pipeline stage
   uint32_t blk[3];          // sweeps: bytes of the block maps
   uint32_t extra[3];        // sweeps: FP64 tables (x: calcnu table; z: coefficient tables)
   uint32_t part;            // z sweep: bytes of one Simpson partial array
   int Ly, Lx;               // the instance's own FFT tile widths
};

__device__ __forceinline__ void tmap_acquire(const CUtensorMap *m) {
   asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// Work list of a pass: entry t packs the instance owning tile t (high
// kInstBits bits) and the tile's index within that instance (low bits), so a
// CTA finds its instance with one load.
constexpr int kInstBits = 12;
constexpr int kLocalBits = 32 - kInstBits;
struct TileRef {
   int inst, local;
};
__device__ __forceinline__ TileRef tile_ref(const unsigned *__restrict__ work, int t) {
   const unsigned w = __ldg(work + t);
   return TileRef{(int) (w >> kLocalBits), (int) (w & ((1u << kLocalBits) - 1u))};
}

// Copies a plan into shared memory (every thread of the CTA calls it); the
// FFT stages index its arrays with run-time stage numbers.
__device__ __forceinline__ void stage_plan(FftPlan &dst, const FftPlan &src) {
   constexpr int W = (int) (sizeof(FftPlan) / sizeof(int));
   static_assert(sizeof(FftPlan) % sizeof(int) == 0, "plan size");
   for (int e = threadIdx.x; e < W; e += blockDim.x) ((int *) &dst)[e] = ((const int *) &src)[e];
   __syncthreads();
}

// ---------------------------------------------------------------- FFT passes
// One CTA per tile; tile numbering of each instance as its single-solve grid.

template <class R, bool CPLX, int PPT, int L>
__global__ void __launch_bounds__(256, L >= 16 ? 3 : 4) kb_zfwd(const BatchDesc *__restrict__ tab,
                                                                const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   __shared__ FftPlan pl;
   stage_plan(pl, D.ph);
   const Dims d = D.d;
   zfwd_body<R, CPLX, PPT, L>((const typename Tr<R, CPLX>::P *) D.psi, (cpx<R> *) D.spec, d, pl,
                              (const cpx<R> *) D.twz, D.LSr, D.err, (long long) r.local * L);
}

template <class R, bool INV, int L>
__global__ void __launch_bounds__(256, 4) kb_yfft(const BatchDesc *__restrict__ tab,
                                                  const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   __shared__ FftPlan pl;
   if (threadIdx.x == 0) tmap_acquire(&D.tm_spec_y);
   stage_plan(pl, D.py);
   const Dims d = D.d;
   const int nkb = (d.nzh + L - 1) / L;
   const int x = r.local / nkb, k0 = (r.local - x * nkb) * L;
   yfft_body<R, INV, L>(&D.tm_spec_y, d, pl, (const cpx<R> *) D.twy, D.boxy, D.nboxy, D.err, x, k0);
}

template <class R, int L>
__global__ void __launch_bounds__(256, 4) kb_xconv(const BatchDesc *__restrict__ tab,
                                                   const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   __shared__ FftPlan pl;
   if (threadIdx.x == 0) tmap_acquire(&D.tm_spec_x);
   stage_plan(pl, D.px);
   const Dims d = D.d;
   const int nkb = (d.nzh + L - 1) / L;
   const int y = r.local / nkb, k0 = (r.local - y * nkb) * L;
   xconv_body<R, L>(&D.tm_spec_x, d, pl, (const cpx<R> *) D.twx, D.udd, D.state, D.boxx, D.nboxx, D.err, y, k0);
}

template <class R, int PPT, int L>
__global__ void __launch_bounds__(256, L >= 16 ? 3 : 4) kb_zinv(const BatchDesc *__restrict__ tab,
                                                                const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   __shared__ FftPlan pl;
   stage_plan(pl, D.ph);
   const Dims d = D.d;
   zinv_body<R, PPT, L>((const cpx<R> *) D.spec, (R *) D.phi, d, pl, (const cpx<R> *) D.twz, D.LSo, D.err,
                        (long long) r.local * L);
}

template <class R>
__global__ void kb_phifix(const BatchDesc *__restrict__ tab, const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   const Dims d = D.d;
   phifix_body<R>((R *) D.phi, d, r.local);
}

static __global__ void __launch_bounds__(32 * kNormRowsPerCta) kb_norm_final(const BatchDesc *__restrict__ tab,
                                                                             const unsigned *__restrict__ work) {
   const TileRef r = tile_ref(work, blockIdx.x);
   const BatchDesc &D = tab[r.inst];
   const Dims d = D.d;
   norm_final_body(D.rowA, d, D.hx, D.hy, D.state, D.xs, nullptr, r.local,
                   (d.nx + kNormRowsPerCta - 1) / kNormRowsPerCta);
}

// ------------------------------------------------------------------- sweeps
// Persistent pipelined CTAs over the tiles of all instances (the pipeline of
// k_sweep_xy / k_sweep_z): while a CTA sweeps tile t, tile t + gridDim.x
// (possibly of another instance) is loading.  Every stage has room for the
// largest tile of the group (stage_bytes); the view of the tile's instance
// is copied into shared memory when the instance changes from one tile of
// the CTA to the next, and so are the FP64 tables the single-solve kernels
// stage once per CTA.

// Words of a view copied by the CTA (every thread calls it).
__device__ __forceinline__ void copy_view(SweepView &dst, const SweepView &src) {
   constexpr int W = (int) (sizeof(SweepView) / sizeof(int));
   static_assert(sizeof(SweepView) % sizeof(int) == 0, "view size");
   for (int e = threadIdx.x; e < W; e += blockDim.x) ((int *) &dst)[e] = ((const int *) &src)[e];
}

template <class R, bool CPLX, int AXIS, bool NU, int MSEG, int S>
__global__ void __launch_bounds__(256, kSweepCtas[NU ? 1 : 0]) kb_sweep_xy(const BatchDesc *__restrict__ tab,
                                                                           const unsigned *__restrict__ work,
                                                                           int ntiles, uint32_t stage_bytes,
                                                                           uint32_t blk_bytes) {
   using P = typename Tr<R, CPLX>::P;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t full[S];
   __shared__ __align__(16) SweepView sv;
   constexpr int E = CPLX ? 2 : 1;
   // layout: S stages of (tile | phi tile) | block maps | FP64 calcnu table
   unsigned char *base = (unsigned char *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   P *blk = (P *) (base + S * stage_bytes);
   double *xtab = (double *) ((unsigned char *) blk + blk_bytes);
   // tile t of the work list: its instance and its place in that instance
   int acq = -1;  // thread 0: the instance whose tensor maps it last acquired
   auto copy_tile = [&](int t, int q, bool load) {
      const TileRef r = tile_ref(work, t);
      const BatchDesc &D = tab[r.inst];
      const SweepView &v = D.sv[AXIS];
      const int TW = v.TW, rows = v.boxn * v.nbox, nzb = (v.d.nz + TW - 1) / TW;
      const int other = r.local / nzb, z0 = (r.local - other * nzb) * TW;
      P *tile = (P *) (base + q * stage_bytes);
      R *ptile = (R *) (tile + rows * TW);
      const CUtensorMap *tm_psi = &D.tm_psi[AXIS];
      if (r.inst != acq) {
         tmap_acquire(tm_psi);
         if (NU) tmap_acquire(&D.tm_phi);
         acq = r.inst;
      }
      if (load) {
         mbar_arrive_expect_tx(&full[q], (uint32_t) (rows * TW * sizeof(P)) + (NU ? (uint32_t) (rows * TW * sizeof(R)) : 0u));
      }
      for (int b = 0; b < v.nbox; b++) {
         const int a0 = b * v.boxn;
         if (load) {
            if (AXIS == 0) tma_load_3d(tile + a0 * TW, tm_psi, E * z0, other, a0, &full[q]);
            else tma_load_3d(tile + a0 * TW, tm_psi, E * z0, a0, other, &full[q]);
            if (NU) {
               if (AXIS == 0) tma_load_3d(ptile + a0 * TW, &D.tm_phi, z0, other, a0, &full[q]);
               else tma_load_3d(ptile + a0 * TW, &D.tm_phi, z0, a0, other, &full[q]);
            }
         } else {
            if (AXIS == 0) tma_store_3d(tm_psi, E * z0, other, a0, tile + a0 * TW);
            else tma_store_3d(tm_psi, E * z0, a0, other, tile + a0 * TW);
         }
      }
      if (!load) bulk_commit();
   };
   if (threadIdx.x == 0) {
      for (int q = 0; q < S; q++) mbar_init(&full[q], 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0 && (int) blockIdx.x < ntiles) copy_tile(blockIdx.x, 0, true);
   int cur = -1;  // instance whose view is in sv
   int it = 0;
   for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
      const int q = it % S;
      if (threadIdx.x == 0 && t + (int) gridDim.x < ntiles) {
         wait_stage_free<S>();
         copy_tile(t + gridDim.x, (it + 1) % S, true);
      }
      // the view and table of this tile's instance (the barrier after the
      // copy wait publishes them)
      const TileRef r = tile_ref(work, t);
      const int i = r.inst;
      if (i != cur) {
         // every thread has finished with the previous view and table
         __syncthreads();
         const BatchDesc &D = tab[i];
         copy_view(sv, D.sv[AXIS]);
         if constexpr (NU && AXIS == 0 && std::is_same<R, double>::value) {
            const SweepView &v = D.sv[AXIS];
            const double *src = (const double *) v.lin.ex;
            for (int e = threadIdx.x; e < (CPLX ? 2 : 1) * v.tb.n; e += blockDim.x) xtab[e] = src[e];
         }
         cur = i;
      }
      if (__syncthreads_or(!mbar_wait(&full[q], (it / S) & 1, tab[i].err))) break;
      const int TW = sv.TW, rows = sv.boxn * sv.nbox, nzb = (sv.d.nz + TW - 1) / TW;
      const int lg = __ffs(TW) - 1;
      const int c = threadIdx.x & (TW - 1), p = threadIdx.x >> lg;
      const int other = r.local / nzb, z0 = (r.local - other * nzb) * TW;
      P *tile = (P *) (base + q * stage_bytes);
      const double scale = NU ? sv.st->scale : 1.;
      if constexpr (NU && std::is_same<R, double>::value) {
         nu_pass_fp64<R, CPLX, AXIS>(tile, (const R *) (tile + rows * TW), sv.tb.n, lg, c, other, z0, sv.d, sv.trap,
                                     sv.lin, xtab, sv.g, sv.gd, sv.dt, scale);
         __syncthreads();
      }
      if constexpr (NU && std::is_same<R, float>::value) {
         static_assert(AXIS == 0, "calcnu is fused into the x sweep only");
         const NuTrap32<CPLX> xf = nu_reads_fp32<CPLX>((const float *) (tile + rows * TW) + c, TW, other, z0, c, sv.d,
                                                       sv.trap, sv.lin, sv.g, sv.gd, sv.dt, scale);
         seg_sweep<R, CPLX, MSEG, 0>(tile, TW, 1, c, p, TW, sv.tb, blk, nullptr, nullptr, nullptr, nullptr, xf);
      } else {
         seg_sweep<R, CPLX, MSEG, 0>(tile, TW, 1, c, p, TW, sv.tb, blk, nullptr, nullptr);
      }
      fence_proxy_async();
      __syncthreads();
      if (threadIdx.x == 0) copy_tile(t, q, false);
   }
   if (threadIdx.x == 0) bulk_wait_all();
}

template <class R, bool CPLX, int MOM, int MSEG, int S>
__global__ void __launch_bounds__(256, kSweepCtas[0]) kb_sweep_z(const BatchDesc *__restrict__ tab,
                                                                 const unsigned *__restrict__ work, int ntiles,
                                                                 uint32_t stage_bytes, uint32_t blk_bytes,
                                                                 uint32_t part_bytes) {
   using P = typename Tr<R, CPLX>::P;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t full[S];
   __shared__ __align__(16) SweepView sv;
   // layout: S stages of rows | block maps | Simpson partials (2 arrays) | FP64 tables
   unsigned char *base = (unsigned char *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   P *blk = (P *) (base + S * stage_bytes);
   double *part = (double *) ((unsigned char *) blk + blk_bytes);
   double *part2 = (double *) ((unsigned char *) part + part_bytes);
   double *tabs = (double *) ((unsigned char *) part2 + part_bytes);
   // FP64: the coefficient tables staged in shared memory, as k_sweep_z does
   constexpr bool STAB = std::is_same<R, double>::value;
   constexpr int TE = CPLX ? 2 : 1;
   // one bulk copy per row, issued by the 32 lanes of warp 0 (the short rows
   // of small grids make many small copies); every lane commits and waits
   // for its own store groups
   const int lane = threadIdx.x & 31;
   auto copy_tile = [&](int t, int q, bool load) {
      const TileRef r = tile_ref(work, t);
      const SweepView &v = tab[r.inst].sv[2];
      const int TR = v.TW, nz = v.d.nz;
      const long long r0 = (long long) r.local * TR;
      const int nr = (int) ((v.d.nxy - r0) < TR ? (v.d.nxy - r0) : TR);
      const uint32_t row_bytes = (uint32_t) (nz * sizeof(P));
      P *tile = (P *) (base + q * stage_bytes);
      if (load && lane == 0) mbar_arrive_expect_tx(&full[q], row_bytes * nr);
      __syncwarp();
      for (int rr = lane; rr < nr; rr += 32) {
         P *g = (P *) v.psi + (r0 + rr) * nz;
         if (load) bulk_load(tile + rr * v.LS, g, row_bytes, &full[q]);
         else bulk_store(g, tile + rr * v.LS, row_bytes);
      }
      if (!load) bulk_commit();
   };
   if (threadIdx.x == 0) {
      for (int q = 0; q < S; q++) mbar_init(&full[q], 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x < 32 && (int) blockIdx.x < ntiles) copy_tile(blockIdx.x, 0, true);
   int cur = -1;
   int it = 0;
   for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
      const int q = it % S;
      if (threadIdx.x < 32 && t + (int) gridDim.x < ntiles) {
         wait_stage_free<S>();
         copy_tile(t + gridDim.x, (it + 1) % S, true);
      }
      const TileRef r = tile_ref(work, t);
      const int i = r.inst;
      if (i != cur) {
         // every thread has finished with the previous view and tables
         __syncthreads();
         const SweepView &v = tab[i].sv[2];
         copy_view(sv, v);
         if constexpr (STAB) {
            const void *src[4] = {v.tb.al, v.tb.ga, v.tb.M, v.tb.N};
            for (int a = 0; a < 4; a++)
               for (int e = threadIdx.x; e < v.tb.n * TE; e += blockDim.x)
                  tabs[a * v.tb.n * TE + e] = ((const double *) src[a])[e];
         }
         cur = i;
      }
      if (__syncthreads_or(!mbar_wait(&full[q], (it / S) & 1, tab[i].err))) break;
      SegTab tbs = sv.tb;
      if constexpr (STAB) {
         const int nn = sv.tb.n * TE;
         tbs.al = tabs;
         tbs.ga = tabs + nn;
         tbs.M = tabs + 2 * nn;
         tbs.N = tabs + 3 * nn;
      }
      const int TR = sv.TW;
      const int c = threadIdx.x % TR, p = threadIdx.x / TR;
      const long long r0 = (long long) r.local * TR;
      const int nr = (int) ((sv.d.nxy - r0) < TR ? (sv.d.nxy - r0) : TR);
      P *tile = (P *) (base + q * stage_bytes);
      zsweep_tile<R, CPLX, MOM, MSEG, 0, STAB>(tile, nr, TR, sv.LS, c, p, tbs, blk, part, part2, sv.wz, sv.wz2, sv.hz3,
                                               sv.rowsum, sv.rowsum2, r0);
      if (threadIdx.x < 32) copy_tile(t, q, false);
   }
   if (threadIdx.x < 32) bulk_wait_all();
}

}  // namespace gpe
