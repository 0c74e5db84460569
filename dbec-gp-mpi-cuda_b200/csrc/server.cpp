// server.cpp -- request server with continuous batching (gpe_server_* in
// include/gpe.h).
//
// One worker thread owns the GPU work.  Active solves live in lanes: a lane
// holds the solves of one size class (up to 64^3, 128^3, larger), mode and
// precision, has its own CUDA stream (smaller classes at higher priority)
// and steps all its solves together with the batched launches of batch.cu
// (one launch per pass over the lane's descriptor table, captured as one CUDA
// graph per step).  Each turn of the loop the worker
//   1. admits queued requests in arrival order while the summed
//      gpe_device_bytes of the active solves stays within the HBM budget and
//      fewer than max_active are running (psi is created on the device and
//      stays there until the request retires); a lane whose stepping set
//      changed is captured again before its next chunk;
//   2. for every lane with no chunk in flight (smallest size class first),
//      queues a chunk of batched steps for the members with the least
//      remaining work while the grid points in flight over all lanes stay
//      within a budget of about two 256^3 solves (the others wait, resident),
//      ending at the nearest chunk boundary of those members (a solve's
//      boundaries: every check_every steps and its last step), then, for the
//      members at a boundary, the pending renormalisation and (ground state)
//      mu, and an event behind it;
//   3. polls the lanes' events; at a finished chunk it checks the members at
//      a boundary (ground state: relative change of mu since the previous
//      check below tol; evolution: all steps done), retires finished solves
//      and frees their memory for the next admissions.
// Requests arriving while others run join a lane at its next chunk boundary.
// A solve's arithmetic does not depend on what else is running: a batched
// step is the solve's own step bit for bit, and its renormalisations and mu
// checks fall on its own boundaries, exactly as when it runs alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "gpe.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

int size_class(const gpe_params &p) {
   const long long n = (long long) p.nx * p.ny * p.nz;
   return n <= 64LL * 64 * 64 ? 0 : (n <= 128LL * 128 * 128 ? 1 : 2);
}

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
   bool cancel = false;  // gpe_server_cancel: retire at the next chunk boundary
   bool due = false;     // the chunk in flight ends at one of its boundaries
   bool on = false;      // stepping in the current chunk
};

// Grid points stepping at once over all lanes: about two 256^3 solves,
// enough to fill the GPU; beyond that, stepping more solves together only
// shares it, so the solves with the least remaining work step first and the
// others wait, resident, for their turn.
constexpr long long kFillPoints = 2LL * 256 * 256 * 256;

long long npts_of(const gpe_request &rq) { return (long long) rq.p.nx * rq.p.ny * rq.p.nz; }

// Solves of one (size class, mode, precision), stepped together.
struct Lane {
   cudaStream_t stream = nullptr;
   gpe_batch *view = nullptr;
   std::vector<std::unique_ptr<Active>> members;
   std::vector<Active *> stepping;  // the members of the batch view
   long long pts = 0;               // grid points of the chunk in flight
   bool inflight = false;
   cudaEvent_t ev = nullptr;
};

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
   std::map<std::tuple<int, int, int>, Lane> lanes;
   int nactive = 0;
   long long used = 0;

   double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

   void post(const gpe_result &r) {
      std::lock_guard<std::mutex> lk(mu);
      results[r.id] = r;
      cancel_req.erase(r.id);
      stats[0] += 1;
      cv_done.notify_all();
   }

   // Retires a solve of a lane with no chunk in flight: observables (unless
   // failed or cancelled), then its memory.
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
         // the solve ended at a boundary, where its renormalisation was applied
         gpe_status st = gpe::queue_muen(a.s, a.rq.g, a.rq.gd);
         if (st == GPE_OK) st = gpe::read_muen(a.s, &r.mu, &r.en);
         if (st == GPE_OK) st = gpe_calcnorm(a.s, 0, &r.norm);
         if (st == GPE_OK) st = gpe_calcrms(a.s, r.rms);
         r.status = st;
      }
      gpe_destroy(a.s);
      a.s = nullptr;
      used -= a.bytes;
      nactive--;
      r.t_done = now();
      post(r);
   }

   // steps from a's current count to its next boundary
   static long to_boundary(const Active &a) {
      const long left = a.rq.max_steps - a.steps;
      const long k = a.rq.check_every - a.steps % a.rq.check_every;
      return std::max(0L, std::min(k, left));
   }

   void admit(const Pending &pd) {
      auto a = std::make_unique<Active>();
      a->id = pd.id;
      a->rq = pd.rq;
      a->t_submit = pd.t_submit;
      a->t_start = now();
      gpe_device_bytes(&a->rq.p, &a->bytes);
      if (a->bytes > budget) {
         a->st = sfail(GPE_ERR_BUDGET, "request exceeds the server's HBM budget");
      } else {
         const int cls = size_class(a->rq.p);
         Lane &L = lanes[std::make_tuple(cls, a->rq.p.mode, a->rq.p.precision)];
         if (!L.stream) {
            // smaller classes on higher-priority streams: when the GPU is
            // shared, the CTA scheduler serves them first, so short requests
            // are not held back by long ones
            int least = 0, greatest = 0;
            cudaDeviceGetStreamPriorityRange(&least, &greatest);
            const int pr = cls == 0 ? greatest : (cls == 1 ? (least + greatest) / 2 : least);
            if (cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, pr) != cudaSuccess ||
                cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming) != cudaSuccess)
               a->st = sfail(GPE_ERR_CUDA, "server: stream creation failed");
            else
               a->st = gpe::batch_view_create(device, L.stream, &L.view);
         }
         if (a->st == GPE_OK) a->st = gpe_create(&a->rq.p, L.stream, &a->s);
         if (a->st == GPE_OK) a->st = gpe_init_gaussian(a->s);
         if (a->st == GPE_OK && a->rq.kind == GPE_REQ_GROUND) {
            double nrm;
            a->st = gpe_calcnorm(a->s, 1, &nrm);
         }
         if (a->st == GPE_OK) {
            used += a->bytes;
            nactive++;
            L.members.push_back(std::move(a));
            return;
         }
      }
      if (a->s) gpe_destroy(a->s);
      gpe_result r{};
      r.id = a->id;
      r.status = a->st;
      r.mu = r.en = r.norm = NAN;
      r.t_submit = a->t_submit;
      r.t_start = a->t_start;
      r.t_done = now();
      post(r);
   }

   // Queues the next chunk of lane L (no chunk in flight): the members with
   // the least remaining work (grid points x steps left) while their points
   // fit `avail` (the first also when nothing else is in flight) step to the
   // nearest of their boundaries.
   void launch_chunk(Lane &L, long long avail, bool first_always) {
      L.pts = 0;
      if (L.members.empty()) return;
      std::vector<Active *> order;
      for (auto &a : L.members) order.push_back(a.get());
      std::stable_sort(order.begin(), order.end(), [](const Active *x, const Active *y) {
         return npts_of(x->rq) * (x->rq.max_steps - x->steps) < npts_of(y->rq) * (y->rq.max_steps - y->steps);
      });
      std::vector<Active *> sel;
      long long pts = 0;
      for (Active *a : order) {
         if (pts + npts_of(a->rq) > avail && !(sel.empty() && first_always)) continue;
         sel.push_back(a);
         pts += npts_of(a->rq);
      }
      if (sel.empty()) return;  // waits for budget
      if (sel != L.stepping) {
         std::vector<gpe_solver *> inst;
         std::vector<double> g, gd;
         for (Active *a : sel) {
            inst.push_back(a->s);
            g.push_back(a->rq.g);
            gd.push_back(a->rq.gd);
         }
         gpe_status st = gpe::batch_view_set(L.view, inst, g, gd);
         if (st != GPE_OK) {
            for (auto &a : L.members) {
               a->st = st;
               a->done = true;
            }
            L.stepping.clear();
            return;
         }
         L.stepping = sel;
      }
      for (auto &a : L.members) a->on = a->due = false;
      long n = 1L << 62;
      for (Active *a : sel) n = std::min(n, to_boundary(*a));
      gpe_status st = n > 0 ? gpe::batch_view_queue(L.view, n) : GPE_OK;
      for (Active *a : sel) {
         a->on = true;
         a->steps += n;
         a->due = st == GPE_OK && (a->steps % a->rq.check_every == 0 || a->steps >= a->rq.max_steps);
         if (st != GPE_OK) {
            a->st = st;
            a->done = true;
         } else if (a->due) {
            a->st = gpe::queue_finish(a->s);
            if (a->st == GPE_OK && a->rq.kind == GPE_REQ_GROUND) a->st = gpe::queue_muen(a->s, a->rq.g, a->rq.gd);
            if (a->st != GPE_OK) a->done = true;
         }
      }
      if (cudaEventRecord(L.ev, L.stream) != cudaSuccess) {
         for (auto &a : L.members) {
            a->st = sfail(GPE_ERR_CUDA, "server: event record failed");
            a->done = true;
         }
         return;
      }
      L.inflight = true;
      L.pts = pts;
      std::lock_guard<std::mutex> lk(mu);
      stats[3] += 1;
   }

   // A finished chunk of lane L: checks at the members' boundaries.
   void chunk_done(Lane &L, cudaError_t q) {
      L.inflight = false;
      for (auto &a : L.members) {
         if (a->done || !a->on) continue;
         if (q != cudaSuccess) {
            a->st = sfail(GPE_ERR_CUDA, cudaGetErrorString(q));
            a->done = true;
            continue;
         }
         if (!a->on || !a->due) continue;
         if (a->rq.kind == GPE_REQ_GROUND) {
            double m = NAN, e = NAN;
            a->st = gpe::read_muen(a->s, &m, &e);
            if (a->st == GPE_OK && std::isfinite(a->mu_prev) && std::fabs(m - a->mu_prev) < a->rq.tol * std::fabs(m))
               a->done = true;
            a->mu_prev = m;
         } else {
            a->st = gpe_synchronize(a->s);
         }
         if (a->steps >= a->rq.max_steps || a->st != GPE_OK) a->done = true;
      }
   }

   // Retires the finished and cancelled members of lane L (no chunk in flight).
   void retire(Lane &L) {
      {
         std::lock_guard<std::mutex> lk(mu);
         for (auto &a : L.members)
            if (cancel_req.count(a->id)) a->cancel = true;
      }
      bool changed = false;
      for (auto &a : L.members)
         if (a->done || a->cancel) {
            finish(*a);
            changed = true;
         }
      if (!changed) return;
      L.members.erase(std::remove_if(L.members.begin(), L.members.end(),
                                     [](const std::unique_ptr<Active> &a) { return a->s == nullptr; }),
                      L.members.end());
      L.stepping.clear();  // the view is set again before the next chunk
   }

   void run() {
      cudaSetDevice(device);
      for (;;) {
         // 1. admission (arrival order, stop at the first that does not fit)
         std::vector<Pending> admit_now;
         {
            std::unique_lock<std::mutex> lk(mu);
            if (nactive == 0 && queue.empty()) {
               if (stopping) break;
               cv_work.wait_for(lk, std::chrono::milliseconds(2));
               continue;
            }
            long long plan = used;
            int act = nactive;
            while (!queue.empty() && act < max_active) {
               long long bytes = 0;
               if (gpe_device_bytes(&queue.front().rq.p, &bytes) != GPE_OK) bytes = 0;
               if (plan + bytes > budget && act > 0) break;
               plan += bytes;
               act++;
               admit_now.push_back(queue.front());
               queue.pop_front();
            }
         }
         for (const Pending &pd : admit_now) admit(pd);
         {
            std::lock_guard<std::mutex> lk(mu);
            stats[1] = std::max(stats[1], (double) nactive);
            stats[2] = std::max(stats[2], (double) used);
         }
         // 2./3. per lane: a finished chunk is checked, finished solves
         // retire, the next chunk goes out
         bool progressed = false;
         for (auto &kv : lanes) {
            Lane &L = kv.second;
            if (!L.inflight) continue;
            const cudaError_t q = cudaEventQuery(L.ev);
            if (q == cudaErrorNotReady) continue;
            chunk_done(L, q);
            progressed = true;
         }
         // lanes in size-class order (smallest first) share one budget of
         // grid points in flight
         long long busy = 0;
         for (auto &kv : lanes)
            if (kv.second.inflight) busy += kv.second.pts;
         for (auto &kv : lanes) {
            Lane &L = kv.second;
            if (L.inflight) continue;
            retire(L);
            launch_chunk(L, kFillPoints - busy, busy == 0);
            busy += L.pts;
         }
         if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
      for (auto &kv : lanes) {
         Lane &L = kv.second;
         if (L.view) gpe_batch_destroy(L.view);
         if (L.ev) cudaEventDestroy(L.ev);
         if (L.stream) cudaStreamDestroy(L.stream);
      }
      lanes.clear();
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
   sv->cancel_req.insert(id);  // admitted: retired at its lane's next chunk boundary
   return GPE_OK;
}

extern "C" gpe_status gpe_server_stats(gpe_server *sv, double *stats) {
   if (!sv || !stats) return sfail(GPE_ERR_PARAM, "server: null argument");
   std::lock_guard<std::mutex> lk(sv->mu);
   for (int i = 0; i < 4; i++) stats[i] = sv->stats[i];
   return GPE_OK;
}
