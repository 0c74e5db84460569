// server.cpp -- request server with continuous batching (gpe_server_* in
// include/gpe.h).
//
// One worker thread owns the GPU work.  Each turn of its loop it
//   1. admits queued requests in arrival order while the summed
//      gpe_device_bytes of the active solves stays within the HBM budget and
//      fewer than max_active are running (psi is created on the device and
//      stays there until the request retires);
//   2. queues the next chunk of steps (plus, for a ground state, its mu) for
//      active solves that have none in flight, in order of least remaining
//      work (grid points x steps left), as long as the grid points of the
//      chunks in flight stay within kFillPoints (the first always goes), each
//      solve on its own stream with an event recorded behind it: the solves
//      run side by side on the GPU, each at its own pace, and short requests
//      are not held behind long ones;
//   3. polls the chunks' events; for every finished chunk it checks
//      convergence (ground state: relative change of mu between checks below
//      tol; evolution: all steps done) and retires finished solves, freeing
//      their memory for the next admissions.
// Requests arriving while others run are admitted on the next turn.
// A solve's arithmetic does not depend on what else is running: every solve
// has its own handle, stream and buffers, and its chunk boundaries depend only
// on its own request.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "gpe.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Active {
   long long id = 0;
   gpe_request rq{};
   gpe_solver *s = nullptr;
   long long bytes = 0;
   long steps = 0;
   double mu_prev = NAN;
   double t_submit = 0., t_start = 0.;
   gpe_status st = GPE_OK;
   bool done = false;
   bool inflight = false;
   bool cancel = false;  // gpe_server_cancel: retire at the next chunk boundary
   cudaEvent_t ev = nullptr;
   cudaStream_t stream = nullptr;  // created by the server with a priority
};

// Grid points of the chunks kept in flight at once: about two 256^3 solves,
// more than enough to fill the GPU, so admitting more only shares it.
constexpr long long kFillPoints = 2LL * 256 * 256 * 256;

long long npts_of(const gpe_request &rq) { return (long long) rq.p.nx * rq.p.ny * rq.p.nz; }

struct Pending {
   long long id;
   gpe_request rq;
   double t_submit;
};

gpe_status sfail(gpe_status st, const std::string &m) {
   gpe::set_last_error(m);
   return st;
}

}  // namespace

struct gpe_server {
   int device = 0;
   long long budget = 0;
   int max_active = 1;
   Clock::time_point t0;
   std::mutex mu;
   std::condition_variable cv_work, cv_done;
   std::deque<Pending> queue;
   std::map<long long, gpe_result> results;
   std::set<long long> cancel_req;  // ids of admitted requests to cancel
   long long next_id = 1;
   bool stopping = false;
   double stats[4] = {0, 0, 0, 0};
   std::thread worker;

   double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

   void finish(Active &a) {
      gpe_result r{};
      r.id = a.id;
      r.status = a.st;
      r.steps = a.steps;
      r.t_submit = a.t_submit;
      r.t_start = a.t_start;
      r.mu = r.en = r.norm = NAN;
      if (a.cancel && a.st == GPE_OK) r.status = GPE_ERR_CANCELLED;
      if (a.st == GPE_OK && !a.cancel) {
         gpe_status st = gpe::queue_muen(a.s, a.rq.g, a.rq.gd);
         if (st == GPE_OK) st = gpe::read_muen(a.s, &r.mu, &r.en);
         if (st == GPE_OK) st = gpe_calcnorm(a.s, 0, &r.norm);
         if (st == GPE_OK) st = gpe_calcrms(a.s, r.rms);
         r.status = st;
      }
      gpe_destroy(a.s);
      a.s = nullptr;
      if (a.ev) cudaEventDestroy(a.ev);
      a.ev = nullptr;
      if (a.stream) cudaStreamDestroy(a.stream);
      a.stream = nullptr;
      r.t_done = now();
      std::lock_guard<std::mutex> lk(mu);
      results[a.id] = r;
      cancel_req.erase(a.id);
      stats[0] += 1;
      cv_done.notify_all();
   }

   // chunk of steps for one active solve
   long chunk(const Active &a) const {
      const long left = a.rq.max_steps - a.steps;
      return std::max(0L, std::min(a.rq.check_every, left));
   }

   int prio_lo = 0, prio_mid = 0, prio_hi = 0;

   void run() {
      cudaSetDevice(device);
      int least = 0, greatest = 0;
      if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) {
         prio_lo = least;
         prio_hi = greatest;
         prio_mid = (least + greatest) / 2;
      }
      std::vector<Active> active;
      long long used = 0;
      for (;;) {
         // 1. admission (arrival order, stop at the first that does not fit)
         std::vector<Pending> admit;
         {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && queue.empty()) {
               if (stopping) break;
               cv_work.wait_for(lk, std::chrono::milliseconds(2));
               continue;
            }
            long long plan = used;
            while (!queue.empty() && (int) (active.size() + admit.size()) < max_active) {
               long long bytes = 0;
               if (gpe_device_bytes(&queue.front().rq.p, &bytes) != GPE_OK) bytes = 0;
               if (plan + bytes > budget && !(active.empty() && admit.empty())) break;
               plan += bytes;
               admit.push_back(queue.front());
               queue.pop_front();
            }
         }
         for (const Pending &pd : admit) {
            Active a;
            a.id = pd.id;
            a.rq = pd.rq;
            a.t_submit = pd.t_submit;
            a.t_start = now();
            gpe_device_bytes(&a.rq.p, &a.bytes);
            if (a.bytes > budget) {
               a.st = sfail(GPE_ERR_BUDGET, "request exceeds the server's HBM budget");
            } else {
               // smaller solves on higher-priority streams: when the GPU is
               // shared, the CTA scheduler serves them first, so short requests
               // are not held back by long ones (shortest work first)
               const long long npts = a.rq.p.nx * a.rq.p.ny * a.rq.p.nz;
               const int pr = npts <= 64 * 64 * 64 ? prio_hi : (npts <= 128 * 128 * 128 ? prio_mid : prio_lo);
               if (cudaStreamCreateWithPriority(&a.stream, cudaStreamNonBlocking, pr) != cudaSuccess)
                  a.st = sfail(GPE_ERR_CUDA, "server: stream creation failed");
               else
                  a.st = gpe_create(&a.rq.p, a.stream, &a.s);
               if (a.st == GPE_OK) a.st = gpe_init_gaussian(a.s);
               if (a.st == GPE_OK && a.rq.kind == GPE_REQ_GROUND) {
                  double nrm;
                  a.st = gpe_calcnorm(a.s, 1, &nrm);
               }
            }
            if (a.st != GPE_OK) {
               if (a.s) {
                  gpe_destroy(a.s);
                  a.s = nullptr;
               }
               if (a.stream) cudaStreamDestroy(a.stream);
               gpe_result r{};
               r.id = a.id;
               r.status = a.st;
               r.t_submit = a.t_submit;
               r.t_start = a.t_start;
               r.t_done = now();
               std::lock_guard<std::mutex> lk(mu);
               results[a.id] = r;
               cancel_req.erase(a.id);
               stats[0] += 1;
               cv_done.notify_all();
               continue;
            }
            used += a.bytes;
            active.push_back(a);
         }
         {
            std::lock_guard<std::mutex> lk(mu);
            stats[1] = std::max(stats[1], (double) active.size());
            stats[2] = std::max(stats[2], (double) used);
         }
         if (active.empty()) continue;
         // cancellations: a solve stops at its next chunk boundary (never with
         // a chunk of its kernels in flight)
         {
            std::lock_guard<std::mutex> lk(mu);
            for (Active &a : active)
               if (cancel_req.count(a.id)) a.cancel = true;
         }
         for (Active &a : active)
            if (a.cancel && !a.inflight) a.done = true;
         // 2. next chunks, least remaining work first, within the fill budget
         long long fill = 0;
         for (const Active &a : active)
            if (a.inflight) fill += npts_of(a.rq);
         std::vector<Active *> order;
         for (Active &a : active)
            if (!a.inflight && !a.done) order.push_back(&a);
         std::sort(order.begin(), order.end(), [](const Active *x, const Active *y) {
            return npts_of(x->rq) * (x->rq.max_steps - x->steps) < npts_of(y->rq) * (y->rq.max_steps - y->steps);
         });
         for (Active *ap : order) {
            Active &a = *ap;
            if (fill > 0 && fill + npts_of(a.rq) > kFillPoints) continue;
            fill += npts_of(a.rq);
            if (!a.ev && cudaEventCreateWithFlags(&a.ev, cudaEventDisableTiming) != cudaSuccess) {
               a.st = sfail(GPE_ERR_CUDA, "server: event creation failed");
               a.done = true;
               continue;
            }
            const long n = chunk(a);
            a.st = gpe::queue_steps(a.s, n, a.rq.g, a.rq.gd);
            if (a.st == GPE_OK) a.st = gpe::queue_finish(a.s);
            if (a.st == GPE_OK && a.rq.kind == GPE_REQ_GROUND) a.st = gpe::queue_muen(a.s, a.rq.g, a.rq.gd);
            if (a.st == GPE_OK && cudaEventRecord(a.ev, gpe::stream_of(a.s)) != cudaSuccess)
               a.st = sfail(GPE_ERR_CUDA, "server: event record failed");
            a.steps += n;
            if (a.st != GPE_OK) {
               a.done = true;
               continue;
            }
            a.inflight = true;
            std::lock_guard<std::mutex> lk(mu);
            stats[3] += 1;
         }
         // 3. finished chunks: check, retire
         bool progressed = false;
         for (Active &a : active) {
            if (!a.inflight) continue;
            const cudaError_t q = cudaEventQuery(a.ev);
            if (q == cudaErrorNotReady) continue;
            a.inflight = false;
            progressed = true;
            if (q != cudaSuccess) {
               a.st = sfail(GPE_ERR_CUDA, cudaGetErrorString(q));
               a.done = true;
               continue;
            }
            if (a.rq.kind == GPE_REQ_GROUND) {
               double m = NAN, e = NAN;
               a.st = gpe::read_muen(a.s, &m, &e);
               if (a.st == GPE_OK && std::isfinite(a.mu_prev) && std::fabs(m - a.mu_prev) < a.rq.tol * std::fabs(m))
                  a.done = true;
               a.mu_prev = m;
            } else {
               a.st = gpe_synchronize(a.s);
            }
            if (a.steps >= a.rq.max_steps || a.st != GPE_OK || a.cancel) a.done = true;
         }
         for (Active &a : active)
            if (a.done && !a.inflight) {
               used -= a.bytes;
               finish(a);
            }
         active.erase(std::remove_if(active.begin(), active.end(),
                                     [](const Active &a) { return a.done && !a.inflight && !a.s; }),
                      active.end());
         if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
   }
};

extern "C" gpe_status gpe_server_create(int device, long long hbm_budget_bytes, int max_active, gpe_server **out) {
   if (!out || hbm_budget_bytes <= 0 || max_active < 1)
      return sfail(GPE_ERR_PARAM, "server: null handle, budget <= 0 or max_active < 1");
   *out = nullptr;
   int dev = device;
   if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return sfail(GPE_ERR_CUDA, "server: no current device");
   gpe_server *sv = new gpe_server();
   sv->device = dev;
   sv->budget = hbm_budget_bytes;
   sv->max_active = max_active;
   sv->t0 = Clock::now();
   sv->worker = std::thread([sv] { sv->run(); });
   *out = sv;
   return GPE_OK;
}

extern "C" void gpe_server_destroy(gpe_server *sv) {
   if (!sv) return;
   {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->stopping = true;
   }
   sv->cv_work.notify_all();
   if (sv->worker.joinable()) sv->worker.join();
   delete sv;
}

extern "C" gpe_status gpe_server_submit(gpe_server *sv, const gpe_request *rq, long long *id) {
   if (!sv || !rq) return sfail(GPE_ERR_PARAM, "server: null argument");
   if (rq->kind != GPE_REQ_GROUND && rq->kind != GPE_REQ_EVOLVE) return sfail(GPE_ERR_PARAM, "server: unknown kind");
   if (rq->kind == GPE_REQ_GROUND && rq->p.mode != GPE_MODE_IMAG)
      return sfail(GPE_ERR_PARAM, "server: a ground-state request runs in imaginary time");
   if (rq->kind == GPE_REQ_EVOLVE && rq->p.mode != GPE_MODE_REAL)
      return sfail(GPE_ERR_PARAM, "server: an evolution request runs in real time");
   if (rq->check_every < 1 || rq->max_steps < 1) return sfail(GPE_ERR_PARAM, "server: check_every, max_steps >= 1");
   long long bytes = 0;
   gpe_status st = gpe_device_bytes(&rq->p, &bytes);  // validates the grid
   if (st != GPE_OK) return st;
   std::lock_guard<std::mutex> lk(sv->mu);
   if (sv->stopping) return sfail(GPE_ERR_STATE, "server: stopping");
   const long long i = sv->next_id++;
   sv->queue.push_back({i, *rq, sv->now()});
   if (id) *id = i;
   sv->cv_work.notify_all();
   return GPE_OK;
}

extern "C" gpe_status gpe_server_wait(gpe_server *sv, long long id, double timeout_s, gpe_result *res) {
   if (!sv) return sfail(GPE_ERR_PARAM, "server: null handle");
   std::unique_lock<std::mutex> lk(sv->mu);
   auto ready = [&] { return sv->results.count(id) > 0; };
   if (timeout_s < 0) {
      sv->cv_done.wait(lk, ready);
   } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
      return sfail(GPE_ERR_TIMEOUT, "server: request not finished in time");
   }
   if (res) *res = sv->results[id];
   return GPE_OK;
}

extern "C" gpe_status gpe_server_cancel(gpe_server *sv, long long id) {
   if (!sv) return sfail(GPE_ERR_PARAM, "server: null handle");
   std::lock_guard<std::mutex> lk(sv->mu);
   if (id < 1 || id >= sv->next_id) return sfail(GPE_ERR_PARAM, "server: unknown request id");
   if (sv->results.count(id)) return sfail(GPE_ERR_STATE, "server: request already finished");
   for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it)
      if (it->id == id) {
         // still queued: never admitted, nothing on the device
         gpe_result r{};
         r.id = id;
         r.status = GPE_ERR_CANCELLED;
         r.mu = r.en = r.norm = NAN;
         r.t_submit = it->t_submit;
         r.t_start = r.t_done = sv->now();
         sv->queue.erase(it);
         sv->results[id] = r;
         sv->stats[0] += 1;
         sv->cv_done.notify_all();
         return GPE_OK;
      }
   sv->cancel_req.insert(id);  // admitted: the worker retires it at the next chunk boundary
   return GPE_OK;
}

extern "C" gpe_status gpe_server_stats(gpe_server *sv, double *stats) {
   if (!sv || !stats) return sfail(GPE_ERR_PARAM, "server: null argument");
   std::lock_guard<std::mutex> lk(sv->mu);
   for (int i = 0; i < 4; i++) stats[i] = sv->stats[i];
   return GPE_OK;
}
