// batch.cu -- many independent solves stepped together (gpe_batch_* in
// include/gpe.h).
//
// Every instance is a complete solver handle (its own device buffers, tables
// and step state).  Instances of the same mode and precision form a group;
// one batch step is, per group, ONE launch per pass of the split step over
// the tiles of all its instances (batch_kernels.cuh): a per-instance
// descriptor table in device memory (dimensions, pointers, FFT plans,
// coefficient tables, couplings, tensor maps) and per-pass work lists of tile
// offsets.  The step's launches are captured once into a CUDA graph and the
// graph is relaunched for every step, so the host cost of a batch step is one
// graph launch and the GPU sees a few wide launches instead of many narrow
// ones.  New couplings are written into the descriptor table (the graph stays
// valid); a new tile configuration (gpe_batch_autotune) rebuilds the tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "batch_kernels.cuh"
#include "gpe.h"
#include "internal.h"

using namespace gpe;

namespace {

// One group: instances of one (mode, precision), with the aggregated launch
// geometry of its passes.
struct Group {
   bool cplx = false, fp32 = false;
   std::vector<int> members;  // instance indices
   int Ly = 0, Lx = 0;        // FFT tile widths (the narrowest of the members)
   BatchGeom geo{};           // maxima over the members (tiles: sums)
   long long off[kNPass + 1] = {};  // start of each pass's work list in dwork
   BatchDesc *dtab = nullptr;        // device descriptor table
   unsigned *dwork = nullptr;        // device work lists (TileRef packed per tile)
   int sweep_grid[3] = {0, 0, 0};
   size_t sweep_smem[3] = {0, 0, 0};
};

}  // namespace

struct gpe_batch {
   std::vector<gpe_solver *> inst;
   std::vector<double> g, gd;
   int dev = 0;
   int nsm = 148;
   cudaStream_t master = nullptr;
   cudaEvent_t fork = nullptr;
   std::vector<Group> groups;
   bool tables = false;  // groups and device tables built
   std::vector<unsigned long long> gen;  // instances' plan generations the tables were built for
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   long long kernels_per_step = 0;
   long long launches = 0;
   // a view over handles owned by someone else (the request server), stepping
   // on the caller's stream: destroying it leaves the handles and the stream
   bool view = false;
};

namespace {

gpe_status bfail(gpe_status st, const std::string &m) {
   gpe::set_last_error(m);
   return st;
}

#define BCK(x)                                                                        \
   do {                                                                               \
      cudaError_t e_ = (x);                                                           \
      if (e_ != cudaSuccess) return bfail(GPE_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
   } while (0)
#define BCKS(...)                     \
   do {                               \
      gpe_status s_ = (__VA_ARGS__);  \
      if (s_ != GPE_OK) return s_;    \
   } while (0)

void drop_graph(gpe_batch *b) {
   if (b->exec) cudaGraphExecDestroy(b->exec);
   if (b->graph) cudaGraphDestroy(b->graph);
   b->exec = nullptr;
   b->graph = nullptr;
}

void drop_tables(gpe_batch *b) {
   drop_graph(b);
   for (Group &G : b->groups) {
      if (G.dtab) cudaFree(G.dtab);
      if (G.dwork) cudaFree(G.dwork);
   }
   b->groups.clear();
   b->tables = false;
}

// Tables (and the captured step) built before an instance's tiles were
// planned again (gpe_set_tuning or gpe_autotune on its handle) are dropped,
// so the next step rebuilds them: the old descriptors still point at the
// instance's freed segment tables and carry its old tile geometry.
void refresh(gpe_batch *b) {
   if (!b->tables) return;
   for (size_t i = 0; i < b->inst.size(); i++)
      if (i >= b->gen.size() || gpe::plan_generation(b->inst[i]) != b->gen[i]) {
         drop_tables(b);
         return;
      }
}

constexpr size_t kSmemCap = 227 * 1024;

// Descriptors of a group (host copy), in member order.
gpe_status group_descs(gpe_batch *b, const Group &G, std::vector<BatchDesc> &h) {
   h.resize(G.members.size());
   for (size_t k = 0; k < G.members.size(); k++) {
      const int i = G.members[k];
      BCKS(gpe::batch_desc(b->inst[i], G.Ly, G.Lx, b->g[i], b->gd[i], &h[k]));
   }
   return GPE_OK;
}

// Groups, aggregated geometry, work lists and device tables.
gpe_status build_tables(gpe_batch *b) {
   drop_tables(b);
   BCK(cudaSetDevice(b->dev));
   std::map<std::pair<int, int>, int> gi;
   for (size_t i = 0; i < b->inst.size(); i++) {
      gpe_params p;
      BCKS(gpe::params_of(b->inst[i], &p));
      const auto key = std::make_pair(p.mode, p.precision);
      auto it = gi.find(key);
      if (it == gi.end()) {
         Group G;
         G.cplx = p.mode == GPE_MODE_REAL;
         G.fp32 = p.precision == GPE_PREC_MIXED;
         b->groups.push_back(G);
         it = gi.emplace(key, (int) b->groups.size() - 1).first;
      }
      b->groups[it->second].members.push_back((int) i);
   }
   for (Group &G : b->groups) {
      const int n = (int) G.members.size();
      G.Ly = G.Lx = 1 << 30;
      for (int i : G.members) {
         BatchGeom own;
         BCKS(gpe::batch_geom(b->inst[i], 0, 0, &own));
         G.Ly = std::min(G.Ly, own.Ly);
         G.Lx = std::min(G.Lx, own.Lx);
      }
      if (n > (1 << kInstBits)) return bfail(GPE_ERR_PARAM, "batch: at most 4096 instances of one mode and precision");
      BatchGeom &A = G.geo;
      A = BatchGeom{};
      std::vector<BatchGeom> geo(n);
      for (int k = 0; k < n; k++) {
         BatchGeom &g = geo[k];
         BCKS(gpe::batch_geom(b->inst[G.members[k]], G.Ly, G.Lx, &g));
         for (int q = 0; q < kNPass; q++) {
            if (g.tiles[q] > (1LL << kLocalBits)) return bfail(GPE_ERR_PARAM, "batch: too many tiles in one instance");
            A.tiles[q] += g.tiles[q];
            A.threads[q] = std::max(A.threads[q], g.threads[q]);
            A.smem[q] = std::max(A.smem[q], g.smem[q]);
         }
         A.zppt = std::max(A.zppt, g.zppt);
         for (int a = 0; a < 3; a++) {
            A.mseg[a] = std::max(A.mseg[a], g.mseg[a]);
            A.stage[a] = std::max(A.stage[a], g.stage[a]);
            A.blk[a] = std::max(A.blk[a], g.blk[a]);
            A.extra[a] = std::max(A.extra[a], g.extra[a]);
         }
         A.part = std::max(A.part, g.part);
      }
      for (long long t : A.tiles)
         if (t > (1LL << 31) - 1) return bfail(GPE_ERR_PARAM, "batch: too many tiles in one pass");
      // sweeps: 2-stage pipelines; as many CTAs per SM as shared memory and
      // the kernels' register budget allow
      for (int a = 0; a < 3; a++) {
         size_t sm = 128 + 2 * (size_t) A.stage[a] + A.blk[a] + A.extra[a];
         if (a == 2) sm += 2 * (size_t) A.part;
         if (sm > kSmemCap) return bfail(GPE_ERR_PARAM, "batch: sweep tiles exceed shared memory");
         // the kernels' register budget holds kSweepCtas CTAs of 256 threads,
         // so more of fewer threads
         const int cap0 = a == 0 ? kSweepCtas[1] : kSweepCtas[0];
         const int cap = std::max(1, std::min(32, 256 * cap0 / std::max(32, (int) A.threads[kPXsweep + a])));
         const int ctas = std::max(1, std::min(cap, (int) (kSmemCap / sm)));
         G.sweep_smem[a] = sm;
         G.sweep_grid[a] = (int) std::min<long long>(A.tiles[kPXsweep + a], (long long) ctas * b->nsm);
      }
      // work lists: every pass's tiles, instance by instance
      G.off[0] = 0;
      for (int q = 0; q < kNPass; q++) G.off[q + 1] = G.off[q] + A.tiles[q];
      std::vector<unsigned> work((size_t) G.off[kNPass]);
      for (int q = 0; q < kNPass; q++) {
         size_t e = (size_t) G.off[q];
         for (int k = 0; k < n; k++)
            for (long long t = 0; t < geo[k].tiles[q]; t++) work[e++] = ((unsigned) k << kLocalBits) | (unsigned) t;
      }
      std::vector<BatchDesc> h;
      BCKS(group_descs(b, G, h));
      BCK(cudaMalloc(&G.dtab, sizeof(BatchDesc) * h.size()));
      BCK(cudaMalloc(&G.dwork, sizeof(unsigned) * std::max<size_t>(1, work.size())));
      BCK(cudaMemcpyAsync(G.dtab, h.data(), sizeof(BatchDesc) * h.size(), cudaMemcpyHostToDevice, b->master));
      BCK(cudaMemcpyAsync(G.dwork, work.data(), sizeof(unsigned) * work.size(), cudaMemcpyHostToDevice, b->master));
   }
   BCK(cudaStreamSynchronize(b->master));
   b->gen.clear();
   for (gpe_solver *s : b->inst) b->gen.push_back(gpe::plan_generation(s));
   b->tables = true;
   return GPE_OK;
}

template <class K, class... A>
gpe_status launch(K kern, unsigned grid, unsigned block, size_t smem, cudaStream_t st, A... args) {
   if (grid == 0) return GPE_OK;
   if (smem > 48 * 1024)
      BCK(cudaFuncSetAttribute((const void *) kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
   kern<<<grid, block, smem, st>>>(args...);
   BCK(cudaGetLastError());
   return GPE_OK;
}

// The passes of one batch step of group G, on stream st.
template <class R, bool CPLX> struct BatchStep {
   using C = cpx<R>;
   template <class F> static gpe_status with_ppt(int ppt, F f) {
      if (ppt <= 8) return f(std::integral_constant<int, 8>());
      if (ppt <= 16) return f(std::integral_constant<int, 16>());
      return f(std::integral_constant<int, 32>());
   }
   template <class F> static gpe_status with_L(int L, F f) {
      if (L >= 16) return f(std::integral_constant<int, 16>());
      if (L == 8) return f(std::integral_constant<int, 8>());
      if (L == 4) return f(std::integral_constant<int, 4>());
      return f(std::integral_constant<int, 2>());
   }
   template <class F> static gpe_status with_mseg(int m, F f) {
      if constexpr (std::is_same<R, float>::value && !CPLX)
         if (m > 16) return f(std::integral_constant<int, 32>());
      if (m > 8) return f(std::integral_constant<int, 16>());
      return f(std::integral_constant<int, 8>());
   }

   // ev (may be null): an event recorded after every pass, index = pass
   static gpe_status run(const Group &G, cudaStream_t st, long long *kernels, cudaEvent_t *ev = nullptr) {
      const BatchGeom &A = G.geo;
      const BatchDesc *tab = G.dtab;
      auto S = [&](int q) { return (const unsigned *) (G.dwork + G.off[q]); };
      auto T = [&](int q) { return (unsigned) A.tiles[q]; };
      constexpr int ZL = 8;
      auto mark = [&](int q) -> gpe_status {
         if (ev) BCK(cudaEventRecord(ev[q], st));
         return GPE_OK;
      };
      BCKS(with_ppt(A.zppt, [&](auto pc) {
         constexpr int PPT = decltype(pc)::value;
         return launch(kb_zfwd<R, CPLX, PPT, ZL>, T(kPZfwd), A.threads[kPZfwd], A.smem[kPZfwd], st, tab, S(kPZfwd));
      }));
      BCKS(mark(kPZfwd));
      BCKS(with_L(G.Ly, [&](auto lc) {
         constexpr int L = decltype(lc)::value;
         return launch(kb_yfft<R, false, L>, T(kPYfft), A.threads[kPYfft], A.smem[kPYfft], st, tab, S(kPYfft));
      }));
      BCKS(mark(kPYfft));
      BCKS(with_L(G.Lx, [&](auto lc) {
         constexpr int L = decltype(lc)::value;
         return launch(kb_xconv<R, L>, T(kPXconv), A.threads[kPXconv], A.smem[kPXconv], st, tab, S(kPXconv));
      }));
      BCKS(mark(kPXconv));
      BCKS(with_L(G.Ly, [&](auto lc) {
         constexpr int L = decltype(lc)::value;
         return launch(kb_yfft<R, true, L>, T(kPYinv), A.threads[kPYinv], A.smem[kPYinv], st, tab, S(kPYinv));
      }));
      BCKS(mark(kPYinv));
      BCKS(with_ppt(A.zppt, [&](auto pc) {
         constexpr int PPT = decltype(pc)::value;
         return launch(kb_zinv<R, PPT, ZL>, T(kPZinv), A.threads[kPZinv], A.smem[kPZinv], st, tab, S(kPZinv));
      }));
      BCKS(mark(kPZinv));
      BCKS(launch(kb_phifix<R>, T(kPPhifix), A.threads[kPPhifix], 0, st, tab, S(kPPhifix)));
      BCKS(mark(kPPhifix));
      BCKS(with_mseg(A.mseg[0], [&](auto mc) {
         constexpr int M = decltype(mc)::value;
         return launch(kb_sweep_xy<R, CPLX, 0, true, M, 2>, (unsigned) G.sweep_grid[0], A.threads[kPXsweep],
                       G.sweep_smem[0], st, tab, S(kPXsweep), (int) A.tiles[kPXsweep], A.stage[0], A.blk[0]);
      }));
      BCKS(mark(kPXsweep));
      BCKS(with_mseg(A.mseg[1], [&](auto mc) {
         constexpr int M = decltype(mc)::value;
         return launch(kb_sweep_xy<R, CPLX, 1, false, M, 2>, (unsigned) G.sweep_grid[1], A.threads[kPYsweep],
                       G.sweep_smem[1], st, tab, S(kPYsweep), (int) A.tiles[kPYsweep], A.stage[1], A.blk[1]);
      }));
      BCKS(mark(kPYsweep));
      BCKS(with_mseg(A.mseg[2], [&](auto mc) {
         constexpr int M = decltype(mc)::value;
         constexpr int MOM = CPLX ? 0 : 1;
         return launch(kb_sweep_z<R, CPLX, MOM, M, 2>, (unsigned) G.sweep_grid[2], A.threads[kPZsweep],
                       G.sweep_smem[2], st, tab, S(kPZsweep), (int) A.tiles[kPZsweep], A.stage[2], A.blk[2],
                       A.part);
      }));
      BCKS(mark(kPZsweep));
      if (!CPLX) BCKS(launch(kb_norm_final, T(kPNorm), A.threads[kPNorm], 0, st, tab, S(kPNorm)));
      BCKS(mark(kPNorm));
      *kernels += CPLX ? 9 : 10;
      return GPE_OK;
   }
};

// ev (may be null): per group, kNPass events recorded after its passes
gpe_status queue_step(gpe_batch *b, cudaStream_t st, long long *kernels, cudaEvent_t *ev = nullptr) {
   for (size_t gi = 0; gi < b->groups.size(); gi++) {
      const Group &G = b->groups[gi];
      cudaEvent_t *e = ev ? ev + gi * kNPass : nullptr;
      if (G.fp32)
         BCKS(G.cplx ? BatchStep<float, true>::run(G, st, kernels, e) : BatchStep<float, false>::run(G, st, kernels, e));
      else
         BCKS(G.cplx ? BatchStep<double, true>::run(G, st, kernels, e) : BatchStep<double, false>::run(G, st, kernels, e));
   }
   return GPE_OK;
}

// Captures one batch step (every group's passes) on the master stream.
gpe_status capture(gpe_batch *b) {
   drop_graph(b);
   BCK(cudaSetDevice(b->dev));
   if (!b->tables) BCKS(build_tables(b));
   // the instances' own queued work comes first
   for (gpe_solver *s : b->inst) {
      BCK(cudaEventRecord(b->fork, gpe::stream_of(s)));
      BCK(cudaStreamWaitEvent(b->master, b->fork, 0));
   }
   BCK(cudaStreamSynchronize(b->master));
   BCK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeRelaxed));
   long long kernels = 0;
   gpe_status st = queue_step(b, b->master, &kernels);
   cudaGraph_t graph = nullptr;
   cudaError_t e = cudaStreamEndCapture(b->master, &graph);
   if (st != GPE_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
   }
   if (e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return bfail(GPE_ERR_CUDA, std::string("batch step capture: ") + cudaGetErrorString(e));
   }
   b->graph = graph;
   BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
   b->kernels_per_step = kernels;
   return GPE_OK;
}

// Orders the master stream after every instance's queued work.
gpe_status fan_in(gpe_batch *b) {
   for (gpe_solver *s : b->inst) {
      BCK(cudaEventRecord(b->fork, gpe::stream_of(s)));
      BCK(cudaStreamWaitEvent(b->master, b->fork, 0));
   }
   return GPE_OK;
}

// Makes every instance stream wait for the work queued on the master stream.
gpe_status fan_out(gpe_batch *b) {
   BCK(cudaEventRecord(b->fork, b->master));
   for (gpe_solver *s : b->inst) BCK(cudaStreamWaitEvent(gpe::stream_of(s), b->fork, 0));
   return GPE_OK;
}

}  // namespace

extern "C" gpe_status gpe_batch_create(const gpe_params *params, const double *g, const double *gd, int n,
                                       gpe_batch **out) {
   if (!out || !params || !g || !gd || n < 1) return bfail(GPE_ERR_PARAM, "batch: null argument or n < 1");
   *out = nullptr;
   gpe_batch *b = new gpe_batch();
   b->g.assign(g, g + n);
   b->gd.assign(gd, gd + n);
   gpe_status st = GPE_OK;
   for (int i = 0; i < n && st == GPE_OK; i++) {
      gpe_solver *s = nullptr;
      st = gpe_create(&params[i], nullptr, &s);
      if (st == GPE_OK) b->inst.push_back(s);
      // mixed-precision imaginary time: 32-point segments in the y and z
      // sweeps (fewer threads per tile, more CTAs per SM in the batched
      // launches: 64-instance batch 1.95 -> 1.83 ms on B200; solo the small
      // grids measured slower with them, so this is the batch's default
      // only), the z sweep on 16-row tiles with a 3-stage pipeline (1.758 ->
      // 1.740 ms)
      if (st == GPE_OK && params[i].mode == GPE_MODE_IMAG && params[i].precision == GPE_PREC_MIXED) {
         gpe_tuning t{};
         t.sweep_seg[1] = t.sweep_seg[2] = 32;
         t.sweep_tw[2] = 16;
         t.sweep_stages[2] = 3;
         st = gpe_set_tuning(s, &t);
      }
   }
   cudaError_t e = cudaSuccess;
   if (st == GPE_OK) {
      b->dev = gpe::device_of(b->inst[0]);
      for (gpe_solver *s : b->inst)
         if (gpe::device_of(s) != b->dev) st = bfail(GPE_ERR_PARAM, "batch: all instances must use one device");
   }
   if (st == GPE_OK) e = cudaSetDevice(b->dev);
   if (st == GPE_OK && e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
   if (st == GPE_OK && e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
   if (st == GPE_OK && e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
   if (st == GPE_OK && e != cudaSuccess) st = bfail(GPE_ERR_CUDA, cudaGetErrorString(e));
   if (st != GPE_OK) {
      const std::string keep = gpe_last_error();
      gpe_batch_destroy(b);
      gpe::set_last_error(keep);
      return st;
   }
   *out = b;
   return GPE_OK;
}

extern "C" void gpe_batch_destroy(gpe_batch *b) {
   if (!b) return;
   cudaSetDevice(b->dev);
   if (b->master) cudaStreamSynchronize(b->master);
   drop_tables(b);
   if (!b->view)
      for (gpe_solver *s : b->inst) gpe_destroy(s);
   if (b->fork) cudaEventDestroy(b->fork);
   if (b->master && !b->view) cudaStreamDestroy(b->master);
   delete b;
}

// ------------------------------------------------------ views (internal.h)
namespace gpe {

gpe_status batch_view_create(int dev, cudaStream_t stream, gpe_batch **out) {
   if (!out) return bfail(GPE_ERR_PARAM, "batch view: null output");
   gpe_batch *b = new gpe_batch();
   b->view = true;
   b->dev = dev;
   b->master = stream;
   cudaError_t e = cudaSetDevice(dev);
   if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
   if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
   if (e != cudaSuccess) {
      delete b;
      return bfail(GPE_ERR_CUDA, cudaGetErrorString(e));
   }
   *out = b;
   return GPE_OK;
}

gpe_status batch_view_set(gpe_batch *b, const std::vector<gpe_solver *> &inst, const std::vector<double> &g,
                          const std::vector<double> &gd) {
   if (!b || !b->view) return bfail(GPE_ERR_PARAM, "batch view: not a view");
   drop_tables(b);
   b->inst = inst;
   b->g = g;
   b->gd = gd;
   return GPE_OK;
}

gpe_status batch_view_queue(gpe_batch *b, long nsteps) {
   if (!b || nsteps < 0) return bfail(GPE_ERR_PARAM, "batch view: null or negative step count");
   if (b->inst.empty() || nsteps == 0) return GPE_OK;
   BCK(cudaSetDevice(b->dev));
   refresh(b);
   if (!b->exec) BCKS(capture(b));
   for (long c = 0; c < nsteps; c++) BCK(cudaGraphLaunch(b->exec, b->master));
   b->launches += b->kernels_per_step * nsteps;
   return GPE_OK;
}

}  // namespace gpe

extern "C" gpe_status gpe_batch_solver(gpe_batch *b, int i, gpe_solver **s) {
   if (!b || !s || i < 0 || i >= (int) b->inst.size()) return bfail(GPE_ERR_PARAM, "batch: bad instance index");
   *s = b->inst[i];
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_set_couplings(gpe_batch *b, const double *g, const double *gd) {
   if (!b || !g || !gd) return bfail(GPE_ERR_PARAM, "batch: null argument");
   b->g.assign(g, g + b->inst.size());
   b->gd.assign(gd, gd + b->inst.size());
   refresh(b);
   if (!b->tables) return GPE_OK;
   // rewrite the descriptor tables in place, in stream order after any batch
   // step already queued; the captured graph reads them at run time
   BCK(cudaSetDevice(b->dev));
   for (const Group &G : b->groups) {
      std::vector<BatchDesc> h;
      BCKS(group_descs(b, G, h));
      BCK(cudaMemcpyAsync(G.dtab, h.data(), sizeof(BatchDesc) * h.size(), cudaMemcpyHostToDevice, b->master));
      BCK(cudaStreamSynchronize(b->master));
   }
   return GPE_OK;
}

// Milliseconds per batch step with the instances' tiles as they are now: the
// step is captured for them, one untimed step, then the best of two runs of
// nsteps steps.
static gpe_status time_batch(gpe_batch *b, int nsteps, double *ms) {
   drop_tables(b);
   double t = 0., best = 1e30;
   BCKS(gpe_batch_time_steps(b, 1, &t));
   for (int r = 0; r < 2; r++) {
      BCKS(gpe_batch_time_steps(b, nsteps, &t));
      best = std::min(best, t / nsteps);
   }
   *ms = best;
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_autotune(gpe_batch *b, int nsteps) {
   if (!b) return bfail(GPE_ERR_PARAM, "batch: null handle");
   if (nsteps < 1) return bfail(GPE_ERR_PARAM, "batch autotune needs nsteps >= 1");
   BCK(cudaSetDevice(b->dev));
   const size_t n = b->inst.size();
   // every instance's psi and step state, put back at the end
   std::vector<gpe::Stash> keep(n);
   std::vector<gpe_tuning> start(n);
   gpe_status st = GPE_OK;
   for (size_t i = 0; i < n && st == GPE_OK; i++) {
      st = gpe::tuning_as_set(b->inst[i], &start[i]);
      if (st == GPE_OK) st = gpe::stash_take(b->inst[i], &keep[i]);
   }
   // the batch step with the tiles the instances start from
   double t_start = 0., t_tuned = 0.;
   if (st == GPE_OK) st = time_batch(b, nsteps, &t_start);
   // one autotuned representative per (grid, mode, precision)
   std::map<std::tuple<long, long, long, int, int>, gpe_tuning> done;
   for (size_t i = 0; i < n && st == GPE_OK; i++) {
      gpe_params p;
      gpe_solver *s = b->inst[i];
      st = gpe::params_of(s, &p);
      if (st != GPE_OK) break;
      const auto key = std::make_tuple(p.nx, p.ny, p.nz, p.mode, p.precision);
      auto it = done.find(key);
      if (it == done.end()) {
         gpe_tuning best;
         st = gpe_autotune(s, b->g[i], b->gd[i], nsteps, &best);
         if (st == GPE_OK) done[key] = best;
      } else {
         st = gpe_set_tuning(s, &it->second);
      }
   }
   // a tile that is fastest for one instance's own launches need not be for
   // the batched launches (one grid over all instances of a group, with other
   // occupancy): the per-grid choices stay only if the batch step is faster
   if (st == GPE_OK) st = time_batch(b, nsteps, &t_tuned);
   if (st != GPE_OK || t_tuned >= t_start)
      for (size_t i = 0; i < n; i++) {
         gpe_status s2 = gpe_set_tuning(b->inst[i], &start[i]);
         if (st == GPE_OK) st = s2;
      }
   drop_tables(b);
   for (size_t i = 0; i < n; i++) {
      gpe_status s2 = keep[i].psi ? gpe::stash_restore(b->inst[i], &keep[i]) : GPE_OK;
      if (st == GPE_OK) st = s2;
   }
   return st;
}

extern "C" gpe_status gpe_batch_run(gpe_batch *b, long nsteps) {
   if (!b || nsteps < 0) return bfail(GPE_ERR_PARAM, "batch: null handle or negative step count");
   BCK(cudaSetDevice(b->dev));
   if (nsteps == 0) return GPE_OK;
   refresh(b);
   if (!b->exec) BCKS(capture(b));
   BCKS(fan_in(b));
   for (long c = 0; c < nsteps; c++) BCK(cudaGraphLaunch(b->exec, b->master));
   b->launches += b->kernels_per_step * nsteps;
   BCKS(fan_out(b));
   for (gpe_solver *s : b->inst) BCKS(gpe::queue_finish(s));
   for (gpe_solver *s : b->inst) BCKS(gpe_synchronize(s));
   BCK(cudaStreamSynchronize(b->master));
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_time_steps(gpe_batch *b, long nsteps, double *ms) {
   if (!b || nsteps < 1) return bfail(GPE_ERR_PARAM, "batch: null handle or nsteps < 1");
   BCK(cudaSetDevice(b->dev));
   refresh(b);
   if (!b->exec) BCKS(capture(b));
   BCKS(fan_in(b));
   cudaEvent_t e0, e1;
   BCK(cudaEventCreate(&e0));
   BCK(cudaEventCreate(&e1));
   BCK(cudaEventRecord(e0, b->master));
   for (long c = 0; c < nsteps; c++) BCK(cudaGraphLaunch(b->exec, b->master));
   BCK(cudaEventRecord(e1, b->master));
   BCK(cudaEventSynchronize(e1));
   float f = 0.f;
   BCK(cudaEventElapsedTime(&f, e0, e1));
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   b->launches += b->kernels_per_step * nsteps;
   gpe_status st = fan_out(b);
   for (gpe_solver *s : b->inst)
      if (st == GPE_OK) st = gpe::queue_finish(s);
   for (gpe_solver *s : b->inst)
      if (st == GPE_OK) st = gpe_synchronize(s);
   if (ms) *ms = f;
   return st;
}

extern "C" gpe_status gpe_batch_profile_step(gpe_batch *b, long nsteps, double *ms, int cap, int *count) {
   if (!b || !ms || nsteps < 1) return bfail(GPE_ERR_PARAM, "batch: null argument or nsteps < 1");
   if (cap < kNPass) return bfail(GPE_ERR_PARAM, "batch: profile output array too small");
   BCK(cudaSetDevice(b->dev));
   refresh(b);
   if (!b->tables) BCKS(build_tables(b));
   BCKS(fan_in(b));
   const size_t ng = b->groups.size();
   std::vector<cudaEvent_t> ev((size_t) nsteps * (ng * kNPass + 1));
   for (auto &e : ev) BCK(cudaEventCreate(&e));
   long long kernels = 0;
   gpe_status st = GPE_OK;
   for (long c = 0; c < nsteps && st == GPE_OK; c++) {
      cudaEvent_t *base = ev.data() + c * (ng * kNPass + 1);
      cudaEventRecord(base[0], b->master);
      st = queue_step(b, b->master, &kernels, base + 1);
   }
   cudaError_t e = cudaStreamSynchronize(b->master);
   if (st == GPE_OK && e != cudaSuccess) st = bfail(GPE_ERR_CUDA, cudaGetErrorString(e));
   if (st == GPE_OK) {
      for (int q = 0; q < kNPass; q++) ms[q] = 0.;
      for (long c = 0; c < nsteps; c++) {
         cudaEvent_t *base = ev.data() + c * (ng * kNPass + 1);
         for (size_t k = 0; k < ng * kNPass; k++) {
            float f = 0.f;
            cudaEventElapsedTime(&f, base[k], base[k + 1]);
            ms[k % kNPass] += f / nsteps;
         }
      }
      if (count) *count = kNPass;
      b->launches += kernels;
   }
   for (auto &x : ev) cudaEventDestroy(x);
   if (st == GPE_OK) st = fan_out(b);
   for (gpe_solver *s : b->inst)
      if (st == GPE_OK) st = gpe::queue_finish(s);
   for (gpe_solver *s : b->inst)
      if (st == GPE_OK) st = gpe_synchronize(s);
   return st;
}

extern "C" gpe_status gpe_batch_launch_count(gpe_batch *b, long long *count) {
   if (!b) return bfail(GPE_ERR_PARAM, "batch: null handle");
   if (count) *count = b->launches;
   return GPE_OK;
}
