// step_kernels.cuh -- kernels of the split step (dipolar convolution passes,
// fused calcnu + sweeps, norm) and of the observables.
#pragma once

#include "kernels.cuh"
#include "tma.cuh"

namespace gpe {

// ===========================================================================
// Dipolar convolution phi = IFFT[Udd * FFT[|psi|^2]] (calcpsidd2_mem,
// imag3d-mpicuda.cu:1460-1510) as four FFT passes over the half spectrum
// spec[x][y][kz], kz in [0, nz/2], plus the boundary planes.
//
// z passes: each real row of length nz is transformed as a complex line of
// length h = nz/2 (z[m] = x[2m] + i x[2m+1]) and split/merged with
//   X[k] = E + W^k O,  E = (Z_k + conj Z_{h-k})/2,  O = (Z_k - conj Z_{h-k})/(2i)
// (forward) and Z_k = (X_k + conj X_{h-k}) + i (X_k - conj X_{h-k}) W^-k
// (inverse), W = exp(-2 pi i / nz).  Rows arrive and leave by bulk copies.
// y and x passes: a TMA box of L kz columns by the whole line lands in the
// interleaved layout the FFT engine works in.
// ===========================================================================

// L: lines per tile of the z passes (128-byte rows); PPT: points per thread
// of the y and x passes, whose tile width the host picks so that a tile of a
// whole line holds at most 256 PPT points (32 KB).
template <class R> struct FftL {
   static constexpr int L = 128 / (2 * (int) sizeof(R));
   static constexpr int PPT = sizeof(R) == 8 ? 8 : 16;
};

// Preferred rows per CTA of the z passes.  Forward: 16 over complex FP32
// rows, so that the radix-8 stages (nz/2-point lines) keep all 256 threads
// busy; 8 over complex FP64 rows (4 KB each), which measured faster with four
// CTAs per SM; 8 over real rows on a CTA sized to them (128 threads at nz =
// 256; 512x512x256 FP32 280 -> 238 us, 256^3 FP64 93 -> 87 us), where the
// host keeps 16 rows on 256 threads for FP64 rows shorter than 128 points.
// Inverse: 8 rows on a CTA sized to them (128 threads at nz = 256), six
// per SM, measured faster than 16 rows on 256 threads (256^3 FP64 82 -> 78
// us, 512x512x256 FP32 238 -> 210 us).  The host halves the rows while the
// tile does not fit shared memory.
template <class R, bool CPLX> struct ZRows {
   static constexpr int fwd = (sizeof(R) == 4 && CPLX) ? 16 : 8;
   static constexpr int inv = 8;
};

// |psi|^2 of L rows (row stride LS elements) packed as complex lines of
// length h = nz/2 in the interleaved layout: buf[m L + l] = (rho[2m], rho[2m+1]).
template <class R, bool CPLX, int L>
__device__ __forceinline__ void zfwd_pack(const typename Tr<R, CPLX>::P *rows, int LS, cpx<R> *buf, int h) {
   for (int e = threadIdx.x; e < h * L; e += blockDim.x) {
      const int l = e % L, m = e / L;
      const typename Tr<R, CPLX>::P *rw = rows + l * LS + 2 * m;
      buf[e] = mk<R>(dens2(rw[0]), dens2(rw[1]));
   }
}

// Real-FFT split of the transformed lines Z into half-spectrum rows
// out[l pitch + k], k < nzh, zero padding for nzh <= k < nzp, rows l < nr.
template <class R, int L>
__device__ __forceinline__ void zfwd_split(const cpx<R> *Z, const cpx<R> *tw, int h, int nzh, int nzp,
                                           cpx<R> *out, long long pitch, int nr) {
   using C = cpx<R>;
   for (int e = threadIdx.x; e < nzp * L; e += blockDim.x) {
      const int l = e % L, k = e / L;
      if (l >= nr) continue;
      if (k >= nzh) {  // row padding
         out[l * pitch + k] = mk<R>(0, 0);
         continue;
      }
      const C a = Z[(k == h ? 0 : k) * L + l];
      const C b = cconj(Z[(k == 0 ? 0 : h - k) * L + l]);
      const C E = cscale(cadd(a, b), (R) 0.5);
      const C t = csub(a, b);
      const C O = mk<R>(t.y * (R) 0.5, -t.x * (R) 0.5);
      out[l * pitch + k] = cadd(E, cmul(tw[k], O));
   }
}

// Pass 1: |psi|^2 rows -> half spectrum rows (L rows per CTA).
// Register budget: four CTAs per SM for 8-row tiles, three for 16-row tiles
// (whose shared tiles allow no more; measured faster with the larger budget).
// The pass over the tile of L rows starting at row r0 (shared by the single
// solve's kernel and the batched one).
template <class R, bool CPLX, int PPT, int L>
__device__ __forceinline__ void zfwd_body(const typename Tr<R, CPLX>::P *__restrict__ psi, cpx<R> *__restrict__ spec,
                                          const Dims &d, const FftPlan &ph, const cpx<R> *__restrict__ twz, int LSr,
                                          uint32_t *err, long long r0) {
   using C = cpx<R>;
   using P = typename Tr<R, CPLX>::P;

   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t bar;
   const int nz = d.nz, h = nz / 2, nzh = d.nzh, nzp = d.nzp;
   // layout: rows [L][LSr] (later the output rows [L][nzp]) | FFT buffer | twiddles
   P *rows = (P *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   C *buf = (C *) (rows + L * LSr);
   C *tw = buf + h * L;
   const int nr = (int) ((d.nxy - r0) < L ? (d.nxy - r0) : L);
   const uint32_t row_bytes = (uint32_t) (nz * sizeof(P));
   if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&bar, row_bytes * nr + (uint32_t) (nz * sizeof(C)));
      bulk_load(tw, twz, (uint32_t) (nz * sizeof(C)), &bar);
      for (int r = 0; r < nr; r++) bulk_load(rows + r * LSr, psi + (r0 + r) * nz, row_bytes, &bar);
   }
   for (int e = threadIdx.x; e < (L - nr) * LSr; e += blockDim.x) rows[nr * LSr + e] = zero_of<P>();
   if (__syncthreads_or(!mbar_wait(&bar, 0, err))) return;
   zfwd_pack<R, CPLX, L>(rows, LSr, buf, h);
   __syncthreads();
   fft_lines_ip<L, C, false, PPT>(buf, ph, tw, 2);
   C *out = (C *) rows;  // [L][nzp]; the rows are no longer read
   zfwd_split<R, L>(buf, tw, h, nzh, nzp, out, nzp, L);
   fence_proxy_async();
   __syncthreads();
   if (threadIdx.x == 0) {
      bulk_store(spec + r0 * nzp, out, (uint32_t) (nr * nzp * sizeof(C)));
      bulk_commit();
      bulk_wait_all();
   }
}

template <class R, bool CPLX, int PPT, int L>
__global__ void __launch_bounds__(256, L >= 16 ? 3 : 4) k_zfwd(const typename Tr<R, CPLX>::P *__restrict__ psi,
                                              cpx<R> *__restrict__ spec, Dims d, FftPlan ph,
                                              const cpx<R> *__restrict__ twz, int LSr, uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   zfwd_body<R, CPLX, PPT, L>(psi, spec, d, ph, twz, LSr, err, (long long) blockIdx.x * L);
}

// Passes 2 and 4: FFT along y of L kz columns of one x plane.  The host sizes
// the CTA at one thread per PPT points of the tile (128 threads for the
// 4-column FP64 tiles, so that eight fit on an SM); the register budget
// (launch bounds 256 x 4) allows any of these sizes.
template <class R, bool INV, int L>
__device__ __forceinline__ void yfft_body(const CUtensorMap *tm, const Dims &d, const FftPlan &py,
                                          const cpx<R> *__restrict__ twy, int boxn, int nbox, uint32_t *err, int x,
                                          int k0) {
   using C = cpx<R>;
   constexpr int PPT = FftL<R>::PPT;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t bar;
   const int ny = d.ny, rows = boxn * nbox;
   C *buf = (C *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   C *tw = buf + rows * L;
   if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&bar, (uint32_t) (rows * L * sizeof(C) + ny * sizeof(C)));
      bulk_load(tw, twy, (uint32_t) (ny * sizeof(C)), &bar);
      for (int b = 0; b < nbox; b++) tma_load_3d(buf + b * boxn * L, tm, 2 * k0, b * boxn, x, &bar);
   }
   if (__syncthreads_or(!mbar_wait(&bar, 0, err))) return;
   fft_lines_ip<L, C, INV, PPT>(buf, py, tw, 1);
   fence_proxy_async();
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int b = 0; b < nbox; b++) tma_store_3d(tm, 2 * k0, b * boxn, x, buf + b * boxn * L);
      bulk_commit();
      bulk_wait_all();
   }
}

template <class R, bool INV, int L>
__global__ void __launch_bounds__(256, 4) k_yfft(const __grid_constant__ CUtensorMap tm, Dims d, FftPlan py,
                                                 const cpx<R> *__restrict__ twy, int boxn, int nbox, uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   const int nkb = (d.nzh + L - 1) / L;
   const int x = blockIdx.x / nkb, k0 = (blockIdx.x - x * nkb) * L;
   yfft_body<R, INV, L>(&tm, d, py, twy, boxn, nbox, err, x, k0);
}

// Pass 3: FFT along x, multiply by Udd(k) * scale^2, inverse FFT along x, for
// L kz columns of one y plane.  Udd octant layout [|kx|][|ky|][kz].  CTA size
// as for the y passes.
template <class R, int L>
__device__ __forceinline__ void xconv_body(const CUtensorMap *tm, const Dims &d, const FftPlan &px,
                                           const cpx<R> *__restrict__ twx, const double *__restrict__ udd,
                                           const State *__restrict__ st, int boxn, int nbox, uint32_t *err, int y,
                                           int k0) {
   using C = cpx<R>;
   constexpr int PPT = FftL<R>::PPT;
   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t bar;
   const int nx = d.nx, ny = d.ny, rows = boxn * nbox;
   C *buf = (C *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   C *tw = buf + rows * L;
   double *ud = (double *) (tw + nx);  // Udd of this y plane and these columns, [|kx|][L]
   const int nxh = nx / 2 + 1, nyh = ny / 2 + 1, nzh = d.nzh;
   const int ay = (y <= ny / 2) ? y : ny - y;
   if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&bar, (uint32_t) (rows * L * sizeof(C) + nx * sizeof(C)));
      bulk_load(tw, twx, (uint32_t) (nx * sizeof(C)), &bar);
      for (int b = 0; b < nbox; b++) tma_load_3d(buf + b * boxn * L, tm, 2 * k0, y, b * boxn, &bar);
   }
   // the Udd factors of the tile travel while the tile and the forward FFT do
   // (loaded after the FFT, their latency measured exposed)
   for (int e = threadIdx.x; e < nxh * L; e += blockDim.x) {
      const int ax = e / L, c = e - ax * L;
      const int k = k0 + c < nzh ? k0 + c : nzh - 1;
      cp_async8(ud + e, udd + ((long long) ax * nyh + ay) * nzh + k);
   }
   if (__syncthreads_or(!mbar_wait(&bar, 0, err))) {
      cp_async_wait_all();
      return;
   }
   fft_lines_ip<L, C, false, PPT>(buf, px, tw, 1);
   cp_async_wait_all();
   __syncthreads();
   C *res = buf;
   const double s2 = st->scale2;
   for (int e = threadIdx.x; e < nx * L; e += blockDim.x) {
      const int xx = e / L, c = e - xx * L;
      const int ax = (xx <= nx / 2) ? xx : nx - xx;
      const R u = (R) (ud[ax * L + c] * s2);
      res[e] = cscale(res[e], u);
   }
   __syncthreads();
   fft_lines_ip<L, C, true, PPT>(buf, px, tw, 1);
   fence_proxy_async();
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int b = 0; b < nbox; b++) tma_store_3d(tm, 2 * k0, y, b * boxn, buf + b * boxn * L);
      bulk_commit();
      bulk_wait_all();
   }
}

template <class R, int L>
__global__ void __launch_bounds__(256, 4) k_xconv(const __grid_constant__ CUtensorMap tm, Dims d, FftPlan px,
                                                  const cpx<R> *__restrict__ twx, const double *__restrict__ udd,
                                                  const State *__restrict__ st, int boxn, int nbox, uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   const int nkb = (d.nzh + L - 1) / L;
   const int y = blockIdx.x / nkb, k0 = (blockIdx.x - y * nkb) * L;
   xconv_body<R, L>(&tm, d, px, twx, udd, st, boxn, nbox, err, y, k0);
}

// Pass 5: half spectrum rows -> phi rows (unnormalised inverse, Hermitian).
template <class R, int PPT, int L>
__device__ __forceinline__ void zinv_body(const cpx<R> *__restrict__ spec, R *__restrict__ phi, const Dims &d,
                                          const FftPlan &ph, const cpx<R> *__restrict__ twz, int LSo, uint32_t *err,
                                          long long r0) {
   using C = cpx<R>;

   extern __shared__ __align__(16) unsigned char smem_raw[];
   __shared__ __align__(8) uint64_t bar;
   const int nz = d.nz, h = nz / 2, nzp = d.nzp;
   // layout: input rows [L][nzp] (later the phi rows [L][LSo]) | FFT buffer | twiddles
   C *in = (C *) (((uintptr_t) smem_raw + 127) & ~(uintptr_t) 127);
   const int in_elems = ((L * nzp) > (L * LSo + 1) / 2 ? (L * nzp) : (L * LSo + 1) / 2);
   C *buf = in + ((in_elems + 7) & ~7);
   C *tw = buf + h * L;
   const int nr = (int) ((d.nxy - r0) < L ? (d.nxy - r0) : L);
   if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&bar, (uint32_t) (nr * nzp * sizeof(C) + nz * sizeof(C)));
      bulk_load(tw, twz, (uint32_t) (nz * sizeof(C)), &bar);
      bulk_load(in, spec + r0 * nzp, (uint32_t) (nr * nzp * sizeof(C)), &bar);
   }
   for (int e = threadIdx.x; e < (L - nr) * nzp; e += blockDim.x) in[nr * nzp + e] = mk<R>(0, 0);
   if (__syncthreads_or(!mbar_wait(&bar, 0, err))) return;
   for (int e = threadIdx.x; e < h * L; e += blockDim.x) {
      const int l = e % L, k = e / L;
      C a = in[l * nzp + k];
      C b = in[l * nzp + h - k];
      if (k == 0) { a.y = 0; b.y = 0; }  // DC and Nyquist bins are real
      b = cconj(b);
      const C E = cadd(a, b);
      const C O = cmul(csub(a, b), cconj(tw[k]));
      buf[e] = mk<R>(E.x - O.y, E.y + O.x);
   }
   __syncthreads();
   fft_lines_ip<L, C, true, PPT>(buf, ph, tw, 2);
   const C *z = buf;
   R *out = (R *) in;  // [L][LSo]
   for (int e = threadIdx.x; e < h * L; e += blockDim.x) {
      const int l = e % L, m = e / L;
      const C v = z[e];
      out[l * LSo + 2 * m] = v.x;
      out[l * LSo + 2 * m + 1] = v.y;
   }
   __syncthreads();
   // boundary plane z = nz-1 <- z = 0 for x < nx-1, y < ny-1, inside the row
   // (the z part of calcpsidd2_kernel2b, imag3d-mpicuda.cu:1605-1625)
   if (threadIdx.x < nr) {
      const long long row = r0 + threadIdx.x;
      const long long x = row / d.ny, y = row - x * d.ny;
      if (x < d.nx - 1 && y < d.ny - 1) out[threadIdx.x * LSo + nz - 1] = out[threadIdx.x * LSo];
   }
   fence_proxy_async();
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int r = 0; r < nr; r++) bulk_store(phi + (r0 + r) * nz, out + r * LSo, (uint32_t) (nz * sizeof(R)));
      bulk_commit();
      bulk_wait_all();
   }
}

template <class R, int PPT, int L>
__global__ void __launch_bounds__(256, L >= 16 ? 3 : 4) k_zinv(const cpx<R> *__restrict__ spec, R *__restrict__ phi, Dims d,
                                                 FftPlan ph, const cpx<R> *__restrict__ twz, int LSo, uint32_t *err) {
   pdl_trigger();
   pdl_wait();
   zinv_body<R, PPT, L>(spec, phi, d, ph, twz, LSo, err, (long long) blockIdx.x * L);
}

// Boundary planes of phi at one rank (calcpsidd2_kernel2a/2b with last = 1,
// imag3d-mpicuda.cu:1591-1625): x = nx-1 <- x = 0 and y = ny-1 <- y = 0 here,
// each excluding the other two last indices; z = nz-1 <- z = 0 is done inside
// the rows by k_zinv.  The read and write sets are disjoint, so both copies
// run concurrently.  One CTA per copied row: blocks [0, ny-1) the rows (nx-1,
// j) <- (0, j), blocks [ny-1, ny-1 + nx-1) the rows (i, ny-1) <- (i, 0), the
// first nz-1 points of each (the grid has at least one block).
template <class R>
__device__ __forceinline__ void phifix_body(R *__restrict__ phi, const Dims &d, int b) {
   long long dst, src;
   if (b < d.ny - 1) {
      dst = ((long long) (d.nx - 1) * d.ny + b) * d.nz;
      src = (long long) b * d.nz;
   } else if (b - (d.ny - 1) < d.nx - 1) {
      const long long i = b - (d.ny - 1);
      dst = (i * d.ny + d.ny - 1) * d.nz;
      src = i * d.ny * d.nz;
   } else {
      return;
   }
   for (int k = threadIdx.x; k < d.nz - 1; k += blockDim.x) phi[dst + k] = phi[src + k];
}

template <class R>
__global__ void k_phifix(R *__restrict__ phi, Dims d) {
   pdl_trigger();
   pdl_wait();
   phifix_body<R>(phi, d, blockIdx.x);
}

// Self-test of the bounded waits: one CTA waits on an mbarrier that expects
// 16 bytes of a transaction no copy will ever deliver.  No copy is issued, so
// nothing is in flight when the wait gives up after `spins` polls; the CTA
// then leaves together, exactly as a step kernel whose tile never arrived,
// and the handle's status word reports the timeout.
static __global__ void k_wait_selftest(uint32_t spins, uint32_t *err) {
   __shared__ __align__(8) uint64_t bar;
   if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      fence_mbar_init();
   }
   __syncthreads();
   if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16u);
   if (__syncthreads_or(!mbar_wait_n(&bar, 0, err, spins))) return;
}

// ===========================================================================
// Sweeps.
// ===========================================================================

// Standalone calcnu (operator-level entry point).
template <class R, bool CPLX>
__global__ void k_calcnu(typename Tr<R, CPLX>::P *__restrict__ psi, const R *__restrict__ phi, Dims d, Trap trap,
                         double g, double gd, double dt) {
   const R invN = (R) (1.0 / (double) d.npts);
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < d.npts; q += (long long) gridDim.x * blockDim.x) {
      const int k = (int) (q % d.nz);
      const long long r = q / d.nz;
      const int j = (int) (r % d.ny), i = (int) (r / d.ny);
      psi[q] = nu_op<R>(psi[q], phi[q], (R) trap.v(i, j, k), (R) g, (R) gd, (R) dt, invN);
   }
}

// ===========================================================================
// Reductions.
// ===========================================================================

// Per-row Simpson of |psi|^2 along z (no sweep).
template <class R, bool CPLX>
__global__ void k_rows_dens(const typename Tr<R, CPLX>::P *__restrict__ psi, Dims d, double hz,
                            double *__restrict__ rowA, double *__restrict__ rowB, const double *__restrict__ z2) {
   const long long row = (long long) blockIdx.x * blockDim.x + threadIdx.x;
   if (row >= d.nxy) return;
   const auto *ps = psi + row * d.nz;
   Simpson a, b;
   a.init(d.nz);
   b.init(d.nz);
   for (int k = 0; k < d.nz; k++) {
      const double f = (double) dens2(ps[k]);
      a.add(k, f);
      if (rowB) b.add(k, z2[k] * f);
   }
   rowA[row] = a.finish(hz);
   if (rowB) rowB[row] = b.finish(hz);
}

// norm = sqrt(S_x S_y rowsum) (calcnorm, imag3d-mpicuda.cu:1194-1218), stores
// norm, scale = 1/norm and scale^2 in the state.  Each warp forms the
// weighted Simpson sum over y of one x row (shuffle reduction) into xs[i];
// the last CTA to finish integrates xs over x.  The kernel is latency-bound
// (a few kB of row sums): loads are issued ahead of the sums and the final
// sum uses the whole CTA (16 -> 10 us at 256^3).
constexpr int kNormRowsPerCta = 8;
// CTA `cta` of the `ncta` CTAs that reduce one solve's row sums.
__device__ __forceinline__ void norm_final_body(const double *__restrict__ rowsum, const Dims &d, double hx, double hy,
                                                State *st, double *xs, double *out_norm, int cta, int ncta) {
   const int lane = threadIdx.x & 31;
   const int i = cta * kNormRowsPerCta + (threadIdx.x >> 5);
   if (i < d.nx) {
      // a warp per x row; the loads of a lane are issued before the sums
      const double *r = rowsum + (long long) i * d.ny;
      constexpr int U = 8;
      double acc = 0.;
      for (int j0 = 0; j0 < d.ny; j0 += 32 * U) {
         double v[U];
#pragma unroll
         for (int u = 0; u < U; u++) {
            const int j = j0 + lane + 32 * u;
            v[u] = j < d.ny ? r[j] : 0.;
         }
#pragma unroll
         for (int u = 0; u < U; u++) {
            const int j = j0 + lane + 32 * u;
            if (j < d.ny) acc = fma(simp_w(j, d.ny), v[u], acc);
         }
      }
      for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) xs[i] = acc * hy / 3.;
   }
   __threadfence();
   __syncthreads();
   __shared__ bool last;
   __shared__ double red[32 * kNormRowsPerCta];
   if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == (unsigned) ncta - 1;
   __syncthreads();
   if (!last) return;
   // last CTA: every thread takes its strided share of the x rows, then a
   // fixed-order tree over the CTA
   __threadfence();
   double acc = 0.;
   for (int k = threadIdx.x; k < d.nx; k += blockDim.x) acc = fma(simp_w(k, d.nx), __ldcg(xs + k), acc);
   red[threadIdx.x] = acc;
   __syncthreads();
   for (int h = blockDim.x / 2; h >= 32; h >>= 1) {
      if ((int) threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
   }
   if (threadIdx.x >= 32) return;
   acc = red[threadIdx.x];
   for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
   if (lane == 0) {
      const double nrm = sqrt(acc * hx / 3.);
      const double t = 1. / nrm;
      st->norm = nrm;
      st->scale = t;
      st->scale2 = t * t;
      st->ticket = 0u;
      if (out_norm) *out_norm = nrm;
   }
}

static __global__ void __launch_bounds__(32 * kNormRowsPerCta) k_norm_final(const double *__restrict__ rowsum, Dims d,
                                                                     double hx, double hy, State *st, double *xs,
                                                                     double *out_norm) {
   pdl_trigger();
   pdl_wait();
   norm_final_body(rowsum, d, hx, hy, st, xs, out_norm, blockIdx.x, gridDim.x);
}

// psi *= scale (calcnorm_kernel, imag3d-mpicuda.cu:1220-1233).
template <class R, bool CPLX>
__global__ void k_apply_scale(typename Tr<R, CPLX>::P *__restrict__ psi, long long n, const State *__restrict__ st) {
   const double s = st->scale;
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < n; q += (long long) gridDim.x * blockDim.x)
      psi[q] = scl(psi[q], s);
}

static __global__ void k_state_set(State *st, double scale) {
   st->scale = scale;
   st->scale2 = scale * scale;
}

// calcrms (imag3d-mpicuda.cu:1639-1744) from the row partials rowA = S_z
// |psi|^2 and rowB = S_z z^2 |psi|^2: <x^2> = S_x x^2 S_y rowA, <y^2> =
// S_x S_y y^2 rowA, <z^2> = S_x S_y rowB; out = (r, rx, ry, rz).  Each warp
// forms the three weighted Simpson sums over y of one x row into xs[3 nx];
// the last CTA to finish integrates them over x.
static __global__ void __launch_bounds__(32 * kNormRowsPerCta) k_rms_final(const double *__restrict__ rowA,
                                                                    const double *__restrict__ rowB, Dims d, double hx,
                                                                    double hy, const double *__restrict__ x2,
                                                                    const double *__restrict__ y2, State *st,
                                                                    double *xs, double *__restrict__ out) {
   pdl_trigger();
   pdl_wait();
   const int lane = threadIdx.x & 31;
   const int i = blockIdx.x * kNormRowsPerCta + (threadIdx.x >> 5);
   if (i < d.nx) {
      const double *ra = rowA + (long long) i * d.ny, *rb = rowB + (long long) i * d.ny;
      double a = 0., b = 0., c = 0.;
      for (int j = lane; j < d.ny; j += 32) {
         const double w = simp_w(j, d.ny);
         a = fma(w, ra[j], a);
         b = fma(w, rb[j], b);
         c = fma(w * y2[j], ra[j], c);
      }
      for (int o = 16; o; o >>= 1) {
         a += __shfl_xor_sync(0xffffffffu, a, o);
         b += __shfl_xor_sync(0xffffffffu, b, o);
         c += __shfl_xor_sync(0xffffffffu, c, o);
      }
      if (lane == 0) {
         xs[i] = x2[i] * a * hy / 3.;
         xs[d.nx + i] = c * hy / 3.;
         xs[2 * d.nx + i] = b * hy / 3.;
      }
   }
   __threadfence();
   __syncthreads();
   __shared__ bool last;
   if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
   __syncthreads();
   if (!last || threadIdx.x >= 32) return;
   __threadfence();
   double m[3] = {0., 0., 0.};
   for (int k = lane; k < d.nx; k += 32) {
      const double w = simp_w(k, d.nx);
      for (int q = 0; q < 3; q++) m[q] = fma(w, __ldcg(xs + q * d.nx + k), m[q]);
   }
   for (int q = 0; q < 3; q++)
      for (int o = 16; o; o >>= 1) m[q] += __shfl_xor_sync(0xffffffffu, m[q], o);
   if (lane == 0) {
      const double rx = sqrt(m[0] * hx / 3.), ry = sqrt(m[1] * hx / 3.), rz = sqrt(m[2] * hx / 3.);
      out[1] = rx;
      out[2] = ry;
      out[3] = rz;
      out[0] = sqrt(rx * rx + ry * ry + rz * rz);
      st->ticket = 0u;
   }
}

// Generic S_x S_y of a per-row array (mu, E, norm).
static __global__ void k_xy_final(const double *__restrict__ rowA, Dims d, double hx, double hy, double *__restrict__ out) {
   extern __shared__ double tx[];
   for (int i = threadIdx.x; i < d.nx; i += blockDim.x) tx[i] = simpint_arr(hy, rowA + (long long) i * d.ny, d.ny);
   __syncthreads();
   if (threadIdx.x == 0) *out = simpint_arr(hx, tx, d.nx);
}

// 4th-order first derivative with the reference's edge rules
// (calcmuen_kernel1x/1y/1z, imag3d-mpicuda.cu:1293-1422).
template <class F>
__device__ __forceinline__ double fd4(F f, int i, int n, double h) {
   if (i == 0 || i == n - 1) return 0.;
   if (i == 1) return (f(2) - f(0)) / (2. * h);
   if (i == n - 2) return (f(n - 1) - f(n - 3)) / (2. * h);
   return (f(i - 2) - 8. * f(i - 1) + 8. * f(i + 1) - f(i + 2)) / (12. * h);
}

// Per-row Simpson of the mu and E integrands (calcmuen_kernel2,
// imag3d-mpicuda.cu:1424-1450); real time differentiates |psi| (real:1401).
template <class R, bool CPLX>
__global__ void k_muen_rows(const typename Tr<R, CPLX>::P *__restrict__ psi, const R *__restrict__ phi, Dims d,
                            Trap trap, double g, double gd, double dx, double dy, double dz, double par,
                            double *__restrict__ rowMu, double *__restrict__ rowEn) {
   const long long row = (long long) blockIdx.x * blockDim.x + threadIdx.x;
   if (row >= d.nxy) return;
   const int i = (int) (row / d.ny), j = (int) (row - (long long) i * d.ny);
   const long long sx = (long long) d.ny * d.nz, sy = d.nz;
   const auto *base = psi + row * d.nz;
   const double invN = 1.0 / (double) d.npts;
   auto amp = [&](const typename Tr<R, CPLX>::P &v) -> double {
      if (CPLX) return sqrt((double) dens2(v));
      return (double) *(const R *) &v;
   };
   Simpson smu, sen;
   smu.init(d.nz);
   sen.init(d.nz);
   for (int k = 0; k < d.nz; k++) {
      const auto *pk = base + k;
      const double ddx = fd4([&](int q) { return amp(pk[(long long) (q - i) * sx]); }, i, d.nx, dx);
      const double ddy = fd4([&](int q) { return amp(pk[(long long) (q - j) * sy]); }, j, d.ny, dy);
      const double ddz = fd4([&](int q) { return amp(base[q]); }, k, d.nz, dz);
      double dpsi = (ddx * ddx) / (3. - par);
      dpsi += (ddy * ddy) / (3. - par);
      dpsi += (ddz * ddz) / (3. - par);
      const double psi2 = (double) dens2(*pk);
      const double psi2lin = psi2 * g;
      const double psidd2lin = ((double) phi[row * d.nz + k] * invN) * gd;
      const double tmppot = trap.v(i, j, k);
      smu.add(k, (tmppot + psi2lin + psidd2lin) * psi2 + dpsi);
      sen.add(k, (tmppot + 0.5 * psi2lin + 0.5 * psidd2lin) * psi2 + dpsi);
   }
   rowMu[row] = smu.finish(dz);
   rowEn[row] = sen.finish(dz);
}

// ---- density outputs -------------------------------------------------------
// Line integral of |psi|^2 along `axis` for every line; out is indexed by the
// two remaining axes in (x, y, z) order.
template <class R, bool CPLX>
__global__ void k_lineint_psi(const typename Tr<R, CPLX>::P *__restrict__ psi, Dims d, int axis, double h,
                              double *__restrict__ out) {
   const int n[3] = {d.nx, d.ny, d.nz};
   const long long s[3] = {(long long) d.ny * d.nz, d.nz, 1};
   const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
   const long long nl = (long long) n[a1] * n[a2];
   const long long l = (long long) blockIdx.x * blockDim.x + threadIdx.x;
   if (l >= nl) return;
   const long long u = l / n[a2], v = l - u * n[a2];
   const auto *p = psi + u * s[a1] + v * s[a2];
   Simpson sp;
   sp.init(n[axis]);
   for (int c = 0; c < n[axis]; c++) sp.add(c, (double) dens2(p[(long long) c * s[axis]]));
   out[l] = sp.finish(h);
}

// out[u] = Simpson along axis `ax` (0 rows, 1 columns) of a [n0][n1] array.
static __global__ void k_lineint_arr(const double *__restrict__ a, int n0, int n1, int ax, double h, double *__restrict__ out) {
   const int l = blockIdx.x * blockDim.x + threadIdx.x;
   if (ax == 1) {
      if (l < n0) out[l] = simpint_arr(h, a + (long long) l * n1, n1, 1);
   } else {
      if (l < n1) out[l] = simpint_arr(h, a + l, n0, n1);
   }
}

// |psi|^2 gathered on a strided sub-grid of a box (3D cuts and raw density).
template <class R, bool CPLX>
__global__ void k_gather_dens(const typename Tr<R, CPLX>::P *__restrict__ psi, Dims d, int i0, int i1, int si,
                              int j0, int j1, int sj, int k0, int k1, int sk, double *__restrict__ out) {
   const long long ni = (i1 - i0 + si - 1) / si, nj = (j1 - j0 + sj - 1) / sj, nk = (k1 - k0 + sk - 1) / sk;
   const long long tot = ni * nj * nk;
   for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < tot; e += (long long) gridDim.x * blockDim.x) {
      const long long a = e / (nj * nk), r = e - a * nj * nk, b = r / nk, c = r - b * nk;
      const long long i = i0 + a * si, j = j0 + b * sj, k = k0 + c * sk;
      out[e] = (double) dens2(psi[(i * d.ny + j) * d.nz + k]);
   }
}

template <class R, bool CPLX>
__global__ void k_init_density(typename Tr<R, CPLX>::P *__restrict__ psi, const double *__restrict__ rho, long long n) {
   using P = typename Tr<R, CPLX>::P;
   for (long long q = blockIdx.x * (long long) blockDim.x + threadIdx.x; q < n; q += (long long) gridDim.x * blockDim.x) {
      const double a = sqrt(rho[q]);
      P v = zero_of<P>();
      if constexpr (CPLX) v.x = (R) a; else v = (R) a;
      psi[q] = v;
   }
}

}  // namespace gpe
