// noalloc.cu -- norm of a device-resident wave function without any device
// allocation.
//
// The regular entry point gpe_calcnorm works on a handle whose device memory
// gpe_create allocated.  Some callers cannot allocate device memory where they
// need the norm: a latency-critical loop that must not take the implicit
// device synchronisation of cudaMalloc/cudaFree, or a process whose device
// memory is owned entirely by another allocator (a framework's caching
// allocator or a fixed pool).  gpe_norm_noalloc serves them: the caller
// passes psi and the output slot in device memory, and the only scratch, one
// Simpson partial per (x, y) row, lives in the file-scope array below.
//
// Limits and sharing:
//  - the scratch holds kNoAllocMaxRows doubles (2 MiB), so nx * ny must not
//    exceed 262144; nx and nz are also limited to 1024 (the final reduction's
//    shared row and the solver's own grid limit);
//  - psi must be aligned to its element (8 bytes in imaginary time, 16 bytes
//    for interleaved complex psi) and norm_dev to 8 bytes; anything else is
//    refused before a launch, since a misaligned load would fault the
//    caller's context;
//  - every device that loads this library keeps the array until the process
//    exits;
//  - the array's device address is looked up (cudaGetSymbolAddress, with the
//    calling device current) the first time a CUDA context calls, and cached
//    per context: a context created later (after cudaDeviceReset, or another
//    driver-API context) looks it up again, so a stale address is never used.
//    Make that first call before any stream capture;
//  - all calls on a device share the array; calls whose kernels overlap on
//    the GPU (different streams, no ordering between them) race on it.  Calls
//    on one stream are ordered and safe.  Every call overwrites all nx * ny
//    entries it reads, so nothing has to be cleared between calls.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "gpe.h"

namespace gpe {
void set_last_error(const std::string &msg);  // defined with gpe_last_error in solver.cu
}

namespace {

constexpr long kNoAllocMaxRows = 1L << 18;  // 2 MiB of doubles
constexpr int kNoAllocMaxN = 1024;
constexpr int kMaxContexts = 64;
constexpr int kRowsPerCta = 8;  // one warp per (x, y) row

static __device__ __align__(256) double g_noalloc_rows[kNoAllocMaxRows];

// Device address of g_noalloc_rows per CUDA context (the host-side symbol is
// only a stand-in), keyed by the driver's context id, which is unique for the
// life of the process.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
std::mutex g_mu;
struct CacheEntry {
   unsigned long long ctx_id;
   double *rows;
};
CacheEntry g_cache[kMaxContexts];
int g_ncache = 0;

gpe_status na_fail(gpe_status st, const std::string &m) {
   gpe::set_last_error(m);  // read back through gpe_last_error()
   return st;
}

// Id of the calling thread's current context.
gpe_status current_ctx_id(unsigned long long *id) {
   static CtxGetCurrentFn get_cur = nullptr;
   static CtxGetIdFn get_id = nullptr;
   if (!get_cur || !get_id) {
      void *f1 = nullptr, *f2 = nullptr;
      cudaDriverEntryPointQueryResult q1, q2;
      if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
          cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess || !f1 || !f2 ||
          q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess) {
         (void) cudaGetLastError();
         return na_fail(GPE_ERR_UNSUPPORTED, "gpe_norm_noalloc: cuCtxGetCurrent / cuCtxGetId unavailable");
      }
      get_cur = (CtxGetCurrentFn) f1;
      get_id = (CtxGetIdFn) f2;
   }
   CUcontext ctx = nullptr;
   if (get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS)
      return na_fail(GPE_ERR_CUDA, "gpe_norm_noalloc: no current CUDA context");
   return GPE_OK;
}

// Simpson partial of |psi|^2 along z for every (x, y) row, one warp per row
// (lanes read consecutive z points, so a warp's loads are coalesced).
template <class P>
__global__ void __launch_bounds__(32 * kRowsPerCta) k_noalloc_rows(const P *__restrict__ psi, long long nxy, int nz,
                                                                   double hz, double *__restrict__ rows) {
   const int lane = threadIdx.x & 31;
   const long long r = (long long) blockIdx.x * kRowsPerCta + (threadIdx.x >> 5);
   if (r >= nxy) return;
   const P *ps = psi + r * nz;
   double acc = 0.;
   for (int k = lane; k < nz; k += 32) acc = fma(gpe::simp_w(k, nz), gpe::dens2(ps[k]), acc);
   for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
   if (lane == 0) rows[r] = acc * hz / 3.;
}

// norm = sqrt(S_x S_y rows) in the order of calcnorm (Simpson over y per x,
// then over x): a warp per x row, then the first warp over x.
__global__ void __launch_bounds__(256) k_noalloc_final(const double *__restrict__ rows, int nx, int ny, double hx,
                                                       double hy, double *__restrict__ norm_out) {
   __shared__ double tx[kNoAllocMaxN];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
   for (int i = w; i < nx; i += nw) {
      const double *ri = rows + (long long) i * ny;
      double acc = 0.;
      for (int j = lane; j < ny; j += 32) acc = fma(gpe::simp_w(j, ny), ri[j], acc);
      for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) tx[i] = acc * hy / 3.;
   }
   __syncthreads();
   if (w != 0) return;
   double acc = 0.;
   for (int i = lane; i < nx; i += 32) acc = fma(gpe::simp_w(i, nx), tx[i], acc);
   for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
   if (lane == 0) *norm_out = sqrt(acc * hx / 3.);
}

}  // namespace

extern "C" gpe_status gpe_norm_noalloc(const void *psi_dev, int mode, long nx, long ny, long nz, double dx, double dy,
                                       double dz, double *norm_dev, void *stream) {
   // every argument is checked before any CUDA call
   if (!psi_dev || !norm_dev) return na_fail(GPE_ERR_PARAM, "psi and norm must be device pointers");
   if (mode != GPE_MODE_IMAG && mode != GPE_MODE_REAL) return na_fail(GPE_ERR_PARAM, "mode must be 0 (imag) or 1 (real)");
   const uintptr_t psi_align = mode == GPE_MODE_REAL ? 16 : 8;
   if ((uintptr_t) psi_dev % psi_align)
      return na_fail(GPE_ERR_PARAM, mode == GPE_MODE_REAL ? "gpe_norm_noalloc: complex psi must be 16-byte aligned"
                                                          : "gpe_norm_noalloc: psi must be 8-byte aligned");
   if ((uintptr_t) norm_dev % 8) return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: norm_dev must be 8-byte aligned");
   if (nx < 4 || ny < 4 || nz < 4) return na_fail(GPE_ERR_PARAM, "grid sizes must be at least 4");
   if (nx > kNoAllocMaxN) return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: nx exceeds 1024");
   if (nz > kNoAllocMaxN) return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: nz exceeds 1024");
   // ny is bounded before the product so that nx * ny cannot wrap
   if (ny > kNoAllocMaxRows || nx * ny > kNoAllocMaxRows)
      return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: nx * ny exceeds the 262144-row scratch (2 MiB)");
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return na_fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   unsigned long long ctx_id = 0;
   if (current_ctx_id(&ctx_id) != GPE_OK) {
      // no context current on this thread yet: cudaSetDevice initialises and
      // binds the device's primary context (it allocates no device memory)
      e = cudaSetDevice(dev);
      if (e != cudaSuccess) return na_fail(GPE_ERR_CUDA, cudaGetErrorString(e));
      gpe_status s = current_ctx_id(&ctx_id);
      if (s != GPE_OK) return s;
   }
   double *rows = nullptr;
   {
      std::lock_guard<std::mutex> lk(g_mu);
      for (int c = 0; c < g_ncache; c++)
         if (g_cache[c].ctx_id == ctx_id) rows = g_cache[c].rows;
      if (!rows) {
         void *ptr = nullptr;
         e = cudaGetSymbolAddress(&ptr, g_noalloc_rows);
         if (e != cudaSuccess) {
            (void) cudaGetLastError();
            return na_fail(GPE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
         }
         rows = (double *) ptr;
         // the oldest entry makes room when the table is full
         if (g_ncache == kMaxContexts) {
            for (int c = 1; c < kMaxContexts; c++) g_cache[c - 1] = g_cache[c];
            g_ncache--;
         }
         g_cache[g_ncache++] = CacheEntry{ctx_id, rows};
      }
   }
   cudaStream_t st = (cudaStream_t) stream;
   const long long nxy = (long long) nx * ny;
   const unsigned grid = (unsigned) ((nxy + kRowsPerCta - 1) / kRowsPerCta);
   if (mode == GPE_MODE_IMAG)
      k_noalloc_rows<double><<<grid, 32 * kRowsPerCta, 0, st>>>((const double *) psi_dev, nxy, (int) nz, dz, rows);
   else
      k_noalloc_rows<double2><<<grid, 32 * kRowsPerCta, 0, st>>>((const double2 *) psi_dev, nxy, (int) nz, dz, rows);
   k_noalloc_final<<<1, 256, 0, st>>>(rows, (int) nx, (int) ny, dx, dy, norm_dev);
   e = cudaGetLastError();
   if (e != cudaSuccess) return na_fail(GPE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
   return GPE_OK;
}
