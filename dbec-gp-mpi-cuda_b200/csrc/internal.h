// internal.h -- hooks of the solver handle for the batch runner and the
// request server, which live in the same library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "gpe.h"

namespace gpe {

void set_last_error(const std::string &msg);
// Queues nsteps split steps at fixed couplings on the handle's stream, with no
// synchronisation; in imaginary time the last renormalisation stays pending.
gpe_status queue_steps(gpe_solver *s, long nsteps, double g, double gd);
// Queues the pending renormalisation (imaginary time; nothing in real time).
gpe_status queue_finish(gpe_solver *s);
// Queues calcmuen into the handle's observable slots; read_muen synchronises
// the stream and returns mu and E.
gpe_status queue_muen(gpe_solver *s, double g, double gd);
gpe_status read_muen(gpe_solver *s, double *mu, double *en);
cudaStream_t stream_of(gpe_solver *s);
gpe_status params_of(gpe_solver *s, gpe_params *p);
int device_of(gpe_solver *s);
long long kernels_per_step(gpe_solver *s);
// Counts the handle's tile plannings (gpe_set_tuning, gpe_autotune): a batch
// compares it with the value its descriptors were built for.
unsigned long long plan_generation(gpe_solver *s);
// The tile choices as set (zeros where the planner picks): gpe_set_tuning
// with them re-plans the handle exactly as before.
gpe_status tuning_as_set(gpe_solver *s, gpe_tuning *t);

// Batched launches (batch.cu): the instance's launch geometry under the
// batch's tile choices with y / x FFT tiles of Ly / Lx columns (Ly = Lx = 0:
// only geom->Ly / Lx, the instance's own widths, are filled in), and its
// descriptor with those tiles and couplings g, gd.
struct BatchDesc;
struct BatchGeom;

// A batch view over handles owned elsewhere (the request server): its steps
// are queued on `stream` (every handle of the view must use that stream);
// destroying it (gpe_batch_destroy) leaves the handles and the stream.
// batch_view_set replaces the members (the step is captured again at the
// next batch_view_queue); batch_view_queue queues nsteps batched steps and
// returns without waiting.
gpe_status batch_view_create(int dev, cudaStream_t stream, gpe_batch **out);
gpe_status batch_view_set(gpe_batch *b, const std::vector<gpe_solver *> &inst, const std::vector<double> &g,
                          const std::vector<double> &gd);
gpe_status batch_view_queue(gpe_batch *b, long nsteps);
gpe_status batch_geom(gpe_solver *s, int Ly, int Lx, BatchGeom *geom);
gpe_status batch_desc(gpe_solver *s, int Ly, int Lx, double g, double gd, BatchDesc *out);

// A device copy of psi and a host copy of the step state (pending
// renormalisation, couplings): stash_take makes it (one cudaMalloc, after the
// handle's queued work), stash_restore writes it back and frees the copy,
// stash_drop frees it without writing back.  Trial steps run in between.
struct Stash {
   void *psi = nullptr;
   size_t bytes = 0;
   unsigned char state[64];
};
gpe_status stash_take(gpe_solver *s, Stash *k);
gpe_status stash_restore(gpe_solver *s, Stash *k);
void stash_drop(Stash *k);

}  // namespace gpe
