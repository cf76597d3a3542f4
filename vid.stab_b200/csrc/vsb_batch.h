/*
 * vsb_batch.h -- internal C interface of the batched multi-stream device
 * path (vsb_batch.cu).  Plain C types only.
 */
#ifndef VSB_BATCH_H
#define VSB_BATCH_H

#include <stdint.h>

#include "vsb_device.h"

#ifdef __cplusplus
extern "C" {
#endif

/* what the device path needs of one stream (planar luma only) */
typedef struct {
  int width, height;
  int blur_size;         /* < 2: no blur */
  int nc, nf;            /* coarse / fine field counts */
  const int16_t* xy;     /* coarse x[nc], coarse y[nc], fine x[nf], fine y[nf] */
  vsbd_geom coarse, fine;
  double coarse_thr;     /* contrast threshold of the coarse fields */
} vsbd_batch_stream;

typedef struct vsbd_batch vsbd_batch;

/* Allocates the device state of n streams, tunes the search tilings of
   every distinct field geometry in the persistent kernel and captures the
   two stage graphs.  Returns 0 or -1 (vsbd_error()). */
int vsbd_batch_create(vsbd_batch** out, int n, const vsbd_batch_stream* streams);
void vsbd_batch_destroy(vsbd_batch* b);

/* Stage A of one step: plane 0 of every stream's new frame (device
   addresses with on_device, else host), blur, coarse search of every coarse
   field, min/max of every field.  Blocks until the results are on the host
   (vsbd_batch_results_a). */
int vsbd_batch_stage_a(vsbd_batch* b, const uint8_t* const* planes, const int* pitches,
                       int on_device);
void vsbd_batch_results_a(const vsbd_batch* b, int stream, const uint8_t** minmax,
                          const vsbd_result** coarse);

/* Stage B: the fine work lists (items[s] of nitems[s]; NULL or 0 for none);
   fres[s] receives stream s's results.  Blocks. */
int vsbd_batch_stage_b(vsbd_batch* b, const vsbd_item* const* items, const int* nitems,
                       const vsbd_result** fres);

/* stream s's current blurred frame becomes its previous one */
void vsbd_batch_commit(vsbd_batch* b, int stream);

/* Overlapped steps: stage A enqueued only and collected later, at most two
   in flight (mode 0: the current step; 1: the next one, into every stream's
   third plane slot; 2: the one after, into the previous step's slot, once
   the current step's fine stage is collected); stage B enqueued on a second
   stream and collected later.  vsbd_batch_stage_a_collect takes the older
   stage A in flight and makes its results the ones vsbd_batch_results_a
   returns; vsbd_batch_drain waits for all. */
int vsbd_batch_stage_a_issue(vsbd_batch* b, const uint8_t* const* planes, const int* pitches,
                             int on_device, int mode);
int vsbd_batch_stage_a_collect(vsbd_batch* b);
void vsbd_batch_drain(vsbd_batch* b);
int vsbd_batch_stage_b_issue(vsbd_batch* b, const vsbd_item* const* items, const int* nitems);
int vsbd_batch_stage_b_collect(vsbd_batch* b, const vsbd_result** fres);

/* limits of the persistent kernel's bounded waits (polls, SM clock cycles) */
int vsbd_batch_set_wait_limit(vsbd_batch* b, unsigned spins, long long cycles);
/* test hook: stage A's work list leaves out stream s's blur items (s < 0:
   the full list again), so that stream's waits run out */
int vsbd_batch_withhold_blur(vsbd_batch* b, int stream);

/* The learned search proposal for every stream (params: the network's
   parameters in device order, on the host; NULL: the dense search again).
   fine_radius >= 0: the fine fields take the narrowed search in a window
   of that radius around the coarse model's prediction; < 0: the dense
   search.
   The network, the priors of streams with passes[s] == 2, the narrowed
   searches and the dense search of the items that fell back all become
   work items of the persistent kernel.  No step may be in flight. */
int vsbd_batch_set_proposal(vsbd_batch* b, const void* params, float scale, float radius,
                            float conf_min, float match_bound, float fine_radius,
                            const int* passes);
/* stream s's proposal counts of the last collected stages (coarse fields
   searched with the proposal, those that fell back; fine items that fell
   back) */
int vsbd_batch_proposal_counts(const vsbd_batch* b, int s, int* coarse_items, int* coarse_fb,
                               int* fine_fb);

long vsbd_batch_launches(const vsbd_batch* b);
/* persistent grid: CTAs, threads per CTA, dynamic shared memory per CTA */
int vsbd_batch_grid(const vsbd_batch* b, int* ctas, int* threads, long* smem);
/* geometry class k of the batch: desc[0..11] = lattice rows per thread,
   layout (1, 2 or 3: DGeom::ta), lattice columns and rows per CTA, field strips, threads, shared
   memory bytes, CTAs per field, search items per step, tuned time of those
   items alone in the persistent kernel (ns), field size, lattice points.
   Returns the number of classes (also for k out of range). */
int vsbd_batch_class(const vsbd_batch* b, int k, int* desc);

#ifdef __cplusplus
}
#endif
#endif
