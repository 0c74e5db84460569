// batch.cu -- many independent solves stepped together (gpe_batch_* in
// include/gpe.h).
//
// Every instance is a complete solver handle with its own stream.  One batch
// step is one split step of every instance; the step is captured once into a
// CUDA graph (fork from a master stream, one branch per instance on its own
// stream, join back) and that graph is relaunched for every step, so the
// kernels of small instances, which cannot fill the GPU alone, run side by
// side, and the per-step host cost is one graph launch.  The per-instance
// descriptor table is the list of handles with their parameters, couplings
// and tile configuration (gpe_batch_autotune picks the configuration per
// distinct grid).
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "gpe.h"
#include "internal.h"

struct gpe_batch {
   std::vector<gpe_solver *> inst;
   std::vector<double> g, gd;
   int dev = 0;
   cudaStream_t master = nullptr;
   cudaEvent_t fork = nullptr;
   std::vector<cudaEvent_t> join;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   long long kernels_per_step = 0;
   long long launches = 0;
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

void drop_graph(gpe_batch *b) {
   if (b->exec) cudaGraphExecDestroy(b->exec);
   if (b->graph) cudaGraphDestroy(b->graph);
   b->exec = nullptr;
   b->graph = nullptr;
}

// Captures one batch step: master -> fork -> every instance's step on its
// stream -> join -> master.
gpe_status capture(gpe_batch *b) {
   drop_graph(b);
   BCK(cudaSetDevice(b->dev));
   for (gpe_solver *s : b->inst) BCK(cudaStreamSynchronize(gpe::stream_of(s)));
   BCK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeRelaxed));
   gpe_status st = GPE_OK;
   cudaError_t e = cudaEventRecord(b->fork, b->master);
   long long kernels = 0;
   for (size_t i = 0; i < b->inst.size() && e == cudaSuccess && st == GPE_OK; i++) {
      cudaStream_t si = gpe::stream_of(b->inst[i]);
      e = cudaStreamWaitEvent(si, b->fork, 0);
      if (e != cudaSuccess) break;
      st = gpe::queue_steps(b->inst[i], 1, b->g[i], b->gd[i]);
      kernels += gpe::kernels_per_step(b->inst[i]);
      if (st == GPE_OK) e = cudaEventRecord(b->join[i], si);
      if (e == cudaSuccess && st == GPE_OK) e = cudaStreamWaitEvent(b->master, b->join[i], 0);
   }
   cudaGraph_t graph = nullptr;
   cudaError_t e2 = cudaStreamEndCapture(b->master, &graph);
   if (st != GPE_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
   }
   if (e != cudaSuccess || e2 != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return bfail(GPE_ERR_CUDA, std::string("batch step capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
   }
   b->graph = graph;
   BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
   b->kernels_per_step = kernels;
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
   }
   cudaError_t e = cudaSuccess;
   if (st == GPE_OK) {
      b->dev = gpe::device_of(b->inst[0]);
      for (gpe_solver *s : b->inst)
         if (gpe::device_of(s) != b->dev) st = bfail(GPE_ERR_PARAM, "batch: all instances must use one device");
   }
   if (st == GPE_OK) e = cudaSetDevice(b->dev);
   if (st == GPE_OK && e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
   if (st == GPE_OK && e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
   b->join.assign(b->inst.size(), nullptr);
   for (size_t i = 0; i < b->join.size() && st == GPE_OK && e == cudaSuccess; i++)
      e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
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
   if (!b->inst.empty()) cudaSetDevice(b->dev);
   if (b->master) cudaStreamSynchronize(b->master);
   drop_graph(b);
   for (gpe_solver *s : b->inst) gpe_destroy(s);
   for (cudaEvent_t e : b->join)
      if (e) cudaEventDestroy(e);
   if (b->fork) cudaEventDestroy(b->fork);
   if (b->master) cudaStreamDestroy(b->master);
   delete b;
}

extern "C" gpe_status gpe_batch_solver(gpe_batch *b, int i, gpe_solver **s) {
   if (!b || !s || i < 0 || i >= (int) b->inst.size()) return bfail(GPE_ERR_PARAM, "batch: bad instance index");
   *s = b->inst[i];
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_set_couplings(gpe_batch *b, const double *g, const double *gd) {
   if (!b || !g || !gd) return bfail(GPE_ERR_PARAM, "batch: null argument");
   b->g.assign(g, g + b->inst.size());
   b->gd.assign(gd, gd + b->inst.size());
   drop_graph(b);
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_autotune(gpe_batch *b, int nsteps) {
   if (!b) return bfail(GPE_ERR_PARAM, "batch: null handle");
   drop_graph(b);
   // one autotuned representative per (grid, mode, precision)
   std::map<std::tuple<long, long, long, int, int>, gpe_tuning> done;
   for (size_t i = 0; i < b->inst.size(); i++) {
      gpe_params p;
      gpe_solver *s = b->inst[i];
      gpe_status st = gpe::params_of(s, &p);
      if (st != GPE_OK) return st;
      const auto key = std::make_tuple(p.nx, p.ny, p.nz, p.mode, p.precision);
      auto it = done.find(key);
      if (it == done.end()) {
         gpe_tuning best;
         st = gpe_autotune(s, b->g[i], b->gd[i], nsteps, &best);
         if (st != GPE_OK) return st;
         done[key] = best;
      } else {
         st = gpe_set_tuning(s, &it->second);
         if (st != GPE_OK) return st;
      }
   }
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_run(gpe_batch *b, long nsteps) {
   if (!b || nsteps < 0) return bfail(GPE_ERR_PARAM, "batch: null handle or negative step count");
   BCK(cudaSetDevice(b->dev));
   if (nsteps == 0) return GPE_OK;
   if (!b->exec) {
      gpe_status st = capture(b);
      if (st != GPE_OK) return st;
   }
   for (long c = 0; c < nsteps; c++) BCK(cudaGraphLaunch(b->exec, b->master));
   b->launches += b->kernels_per_step * nsteps;
   gpe_status st = fan_out(b);
   if (st != GPE_OK) return st;
   for (gpe_solver *s : b->inst) {
      st = gpe::queue_finish(s);
      if (st != GPE_OK) return st;
   }
   for (gpe_solver *s : b->inst) {
      st = gpe_synchronize(s);
      if (st != GPE_OK) return st;
   }
   BCK(cudaStreamSynchronize(b->master));
   return GPE_OK;
}

extern "C" gpe_status gpe_batch_time_steps(gpe_batch *b, long nsteps, double *ms) {
   if (!b || nsteps < 1) return bfail(GPE_ERR_PARAM, "batch: null handle or nsteps < 1");
   BCK(cudaSetDevice(b->dev));
   if (!b->exec) {
      gpe_status st = capture(b);
      if (st != GPE_OK) return st;
   }
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

extern "C" gpe_status gpe_batch_launch_count(gpe_batch *b, long long *count) {
   if (!b) return bfail(GPE_ERR_PARAM, "batch: null handle");
   if (count) *count = b->launches;
   return GPE_OK;
}
