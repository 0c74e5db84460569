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
//    exceed 262144; nx is also limited to 1024 by the final reduction;
//  - every device that loads this library keeps the array until the process
//    exits;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make
//    that first call before any stream capture;
//  - all calls on a device share the array; calls whose kernels overlap on
//    the GPU (different streams, no ordering between them) race on it.  Calls
//    on one stream are ordered and safe.  Every call overwrites all nx * ny
//    entries it reads, so nothing has to be cleared between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "gpe.h"

namespace gpe {
void set_last_error(const std::string &msg);  // defined with gpe_last_error in solver.cu
}

namespace {

constexpr long kNoAllocMaxRows = 1L << 18;  // 2 MiB of doubles
constexpr int kNoAllocMaxNx = 1024;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_rows[kNoAllocMaxRows];

// Device address of g_noalloc_rows per device ordinal, looked up once per
// device with that device current (the host-side symbol is only a stand-in).
std::mutex g_mu;
double *g_rows_dev[kMaxDevices] = {nullptr};

gpe_status na_fail(gpe_status st, const std::string &m) {
   gpe::set_last_error(m);  // read back through gpe_last_error()
   return st;
}

template <class P>
__global__ void k_noalloc_rows(const P *__restrict__ psi, long long nxy, int nz, double hz, double *__restrict__ rows) {
   const long long r = (long long) blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= nxy) return;
   const P *ps = psi + r * nz;
   gpe::Simpson sp;
   sp.init(nz);
   for (int k = 0; k < nz; k++) sp.add(k, gpe::dens2(ps[k]));
   rows[r] = sp.finish(hz);
}

// norm = sqrt(S_x S_y rows) in the order of calcnorm (simpint over y per x,
// then over x).
__global__ void k_noalloc_final(const double *__restrict__ rows, int nx, int ny, double hx, double hy,
                                double *__restrict__ norm_out) {
   __shared__ double tx[kNoAllocMaxNx];
   for (int i = threadIdx.x; i < nx; i += blockDim.x) tx[i] = gpe::simpint_arr(hy, rows + (long long) i * ny, ny);
   __syncthreads();
   if (threadIdx.x == 0) *norm_out = sqrt(gpe::simpint_arr(hx, tx, nx));
}

}  // namespace

extern "C" gpe_status gpe_norm_noalloc(const void *psi_dev, int mode, long nx, long ny, long nz, double dx, double dy,
                                       double dz, double *norm_dev, void *stream) {
   if (!psi_dev || !norm_dev) return na_fail(GPE_ERR_PARAM, "psi and norm must be device pointers");
   if (mode != GPE_MODE_IMAG && mode != GPE_MODE_REAL) return na_fail(GPE_ERR_PARAM, "mode must be 0 (imag) or 1 (real)");
   if (nx < 4 || ny < 4 || nz < 4) return na_fail(GPE_ERR_PARAM, "grid sizes must be at least 4");
   if (nx > kNoAllocMaxNx) return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: nx exceeds 1024");
   if (nx * ny > kNoAllocMaxRows)
      return na_fail(GPE_ERR_PARAM, "gpe_norm_noalloc: nx * ny exceeds the 262144-row scratch (2 MiB)");
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return na_fail(GPE_ERR_CUDA, cudaGetErrorString(e));
   if (dev < 0 || dev >= kMaxDevices) return na_fail(GPE_ERR_UNSUPPORTED, "device ordinal out of range");
   double *rows = nullptr;
   {
      std::lock_guard<std::mutex> lk(g_mu);
      if (!g_rows_dev[dev]) {
         void *ptr = nullptr;
         e = cudaGetSymbolAddress(&ptr, g_noalloc_rows);
         if (e != cudaSuccess) {
            (void) cudaGetLastError();
            return na_fail(GPE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
         }
         g_rows_dev[dev] = (double *) ptr;
      }
      rows = g_rows_dev[dev];
   }
   cudaStream_t st = (cudaStream_t) stream;
   const long long nxy = (long long) nx * ny;
   const unsigned grid = (unsigned) ((nxy + 127) / 128);
   if (mode == GPE_MODE_IMAG)
      k_noalloc_rows<double><<<grid, 128, 0, st>>>((const double *) psi_dev, nxy, (int) nz, dz, rows);
   else
      k_noalloc_rows<double2><<<grid, 128, 0, st>>>((const double2 *) psi_dev, nxy, (int) nz, dz, rows);
   k_noalloc_final<<<1, 256, 0, st>>>(rows, (int) nx, (int) ny, dx, dy, norm_dev);
   e = cudaGetLastError();
   if (e != cudaSuccess) return na_fail(GPE_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
   return GPE_OK;
}
