/*
 * vs_batch.c -- the detect pass over many independent streams at once
 * (declared in vidstab_b200_ext.h; no reference counterpart: the reference
 * runs one VSMotionDetect per stream).
 *
 * Every stream is a VSMotionDetect of its own (fields, selection, simple
 * model, tripod state: the same host code as vsMotionDetection), without
 * per-detector device state.  A batch step runs the device work of all
 * streams as two persistent-kernel launches (vsb_batch.cu) with the
 * per-stream host phases in between.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vidstab_b200.h"
#include "vsb_batch.h"
#include "vsb_host.h"

struct vsb_batch {
  int n;
  VSMotionDetect* md;
  vsbd_batch* dev;
  vsb_frame_work* w;
  int* search;
  const vsbd_item** items;
  int* nitems;
  const vsbd_result** fres;
  FILE** trf; /* per stream: the .trf file its motions go to (NULL: none) */
  int pn_on;  /* a learned search proposal is set */
  long long pn_stats[8]; /* as vsb_proposal_stats */
};

/* proposal counts of stream s's collected stage A (coarse) or stage B
   (fine, nitems items) */
static void tally(vsb_batch* b, int s, int fine, int nitems) {
  int ci = 0, cfb = 0, ffb = 0;
  /* fine fields take the dense search: nothing to count */
  if (fine) return;
  if (!b->pn_on || vsbd_batch_proposal_counts(b->dev, s, &ci, &cfb, &ffb) != 0) return;
  const int items = fine ? nitems : ci, fb = fine ? ffb : cfb;
  b->pn_stats[0] += items;
  b->pn_stats[1] += fb;
  b->pn_stats[4 + 2 * fine] += items;
  b->pn_stats[5 + 2 * fine] += fb;
}

int vsb_batch_set_proposal(vsb_batch* b, const void* blob, long bytes) {
  if (!b) return VS_ERROR;
  if (!blob) {
    if (vsbd_batch_set_proposal(b->dev, NULL, 0, 0, 0, 0, 0, NULL) != 0) return VS_ERROR;
    b->pn_on = 0;
    return VS_OK;
  }
  vsb_pnet_settings p;
  if (vsb_pnet_parse(blob, bytes, -1.0, NAN, -1.0, &p) != VS_OK) return VS_ERROR;
  int* passes = (int*)malloc(sizeof(int) * (size_t)b->n);
  if (!passes) return VS_ERROR;
  /* as a single detector: two network passes for very shaky footage */
  for (int s = 0; s < b->n; s++) passes[s] = b->md[s].conf.shakiness >= 8 ? 2 : 1;
  /* fine fields: the dense search, as a single detector's default */
  int rc = vsbd_batch_set_proposal(b->dev, p.params, p.scale, p.radius, p.conf_min,
                                   p.match_bound, -1.0f, passes);
  free(passes);
  if (rc != 0) return VS_ERROR;
  b->pn_on = 1;
  memset(b->pn_stats, 0, sizeof(b->pn_stats));
  return VS_OK;
}

int vsb_batch_proposal_stats(const vsb_batch* b, long long* stats) {
  if (!b || !stats || !b->pn_on) return VS_ERROR;
  memcpy(stats, b->pn_stats, sizeof(b->pn_stats));
  return VS_OK;
}

/* after a stream's frame ended (frame number advanced, as vidstabdetect
   writes after vsMotionDetection): its motions to the stream's .trf */
static int write_trf(vsb_batch* b, int s, const LocalMotions* lms) {
  if (!b->trf || !b->trf[s]) return VS_OK;
  if (vsWriteToFile(&b->md[s], b->trf[s], lms) != VS_OK) {
    vs_log_error("vsb_batch", "writing the .trf of stream %d failed\n", s);
    return VS_ERROR;
  }
  return VS_OK;
}

int vsb_batch_set_wait_limit(vsb_batch* b, unsigned spins, long long cycles) {
  if (!b) return VS_ERROR;
  return vsbd_batch_set_wait_limit(b->dev, spins, cycles) == 0 ? VS_OK : VS_ERROR;
}

int vsb_batch_test_withhold_blur(vsb_batch* b, int stream) {
  if (!b) return VS_ERROR;
  return vsbd_batch_withhold_blur(b->dev, stream) == 0 ? VS_OK : VS_ERROR;
}

int vsb_batch_close_trf(vsb_batch* b) {
  if (!b) return VS_ERROR;
  int rc = VS_OK;
  if (b->trf)
    for (int s = 0; s < b->n; s++)
      if (b->trf[s] && fclose(b->trf[s]) != 0) rc = VS_ERROR;
  free(b->trf);
  b->trf = NULL;
  return rc;
}

int vsb_batch_open_trf(vsb_batch* b, const char* const* paths, int serialization_mode) {
  if (!b || !paths) return VS_ERROR;
  vsb_batch_close_trf(b);
  b->trf = (FILE**)calloc((size_t)b->n, sizeof(FILE*));
  if (!b->trf) return VS_ERROR;
  for (int s = 0; s < b->n; s++) {
    if (!paths[s]) continue;
    b->md[s].serializationMode = serialization_mode;
    b->trf[s] = fopen(paths[s], "wb");
    if (!b->trf[s] || vsPrepareFile(&b->md[s], b->trf[s]) != VS_OK) {
      vs_log_error("vsb_batch", "cannot start the .trf of stream %d (%s)\n", s, paths[s]);
      vsb_batch_close_trf(b);
      return VS_ERROR;
    }
  }
  return VS_OK;
}

void vsb_batch_free(vsb_batch* b) {
  if (!b) return;
  vsb_batch_close_trf(b);
  vsbd_batch_destroy(b->dev);
  if (b->md)
    for (int s = 0; s < b->n; s++)
      if (b->md[s].initialized) vsMotionDetectionCleanup(&b->md[s]);
  free(b->md);
  free(b->w);
  free(b->search);
  free(b->items);
  free(b->nitems);
  free(b->fres);
  free(b);
}

vsb_batch* vsb_batch_create(int n, const int* widths, const int* heights, int pformat,
                            const VSMotionDetectConfig* conf) {
  if (n < 1 || !widths || !heights || !conf) return NULL;
  if (pformat <= PF_NONE || pformat >= PF_PACKED) {
    vsbd_set_error("the batched path takes planar pixel formats only");
    return NULL;
  }
  vsb_batch* b = (vsb_batch*)calloc(1, sizeof(vsb_batch));
  b->n = n;
  b->md = (VSMotionDetect*)calloc((size_t)n, sizeof(VSMotionDetect));
  b->w = (vsb_frame_work*)calloc((size_t)n, sizeof(vsb_frame_work));
  b->search = (int*)calloc((size_t)n, sizeof(int));
  b->items = (const vsbd_item**)calloc((size_t)n, sizeof(vsbd_item*));
  b->nitems = (int*)calloc((size_t)n, sizeof(int));
  b->fres = (const vsbd_result**)calloc((size_t)n, sizeof(vsbd_result*));
  vsb_md_layout* lay = (vsb_md_layout*)calloc((size_t)n, sizeof(vsb_md_layout));
  vsbd_batch_stream* ds = (vsbd_batch_stream*)calloc((size_t)n, sizeof(vsbd_batch_stream));
  int ok = b->md && b->w && b->search && b->items && b->nitems && b->fres && lay && ds;
  for (int s = 0; ok && s < n; s++) {
    VSFrameInfo fi;
    VSMotionDetectConfig c = conf[s];
    c.show = 0; /* no host frame to draw into */
    if (!vsFrameInfoInit(&fi, widths[s], heights[s], (VSPixelFormat)pformat) ||
        vsb_md_init(&b->md[s], &c, &fi, 0, &lay[s]) != VS_OK) {
      ok = 0;
      break;
    }
    ds[s].width = widths[s];
    ds[s].height = heights[s];
    ds[s].blur_size = lay[s].blur;
    ds[s].nc = lay[s].nc;
    ds[s].nf = lay[s].nf;
    ds[s].xy = lay[s].xy;
    ds[s].coarse = lay[s].coarse;
    ds[s].fine = lay[s].fine;
    ds[s].coarse_thr = b->md[s].fieldscoarse.contrastThreshold;
  }
  if (ok && vsbd_batch_create(&b->dev, n, ds) != 0) ok = 0;
  for (int s = 0; lay && s < n; s++) vsb_md_layout_free(&lay[s]);
  free(lay);
  free(ds);
  if (!ok) {
    vsb_batch_free(b);
    return NULL;
  }
  return b;
}

int vsb_batch_detect(vsb_batch* b, const uint8_t* const* planes, const int* pitches,
                     int on_device, LocalMotions* motions) {
  if (!b || !planes || !pitches || !motions) return VS_ERROR;
  for (int s = 0; s < b->n; s++)
    if (vsb_frame_begin(&b->md[s], &b->search[s]) != VS_OK) return VS_ERROR;
  /* wall time: [0] stage A, [1] host part A, [2] stage B, [3] host part B */
  double t0 = vsb_now_s(), prof[4];
  if (vsbd_batch_stage_a(b->dev, planes, pitches, on_device) != 0) {
    vs_log_error("vsb_batch", "GPU stage A failed: %s\n", vsbd_error());
    return VS_ERROR;
  }
  double t1 = vsb_now_s();
  for (int s = 0; s < b->n; s++) {
    b->items[s] = NULL;
    b->nitems[s] = 0;
    if (!b->search[s]) continue;
    const uint8_t* mm;
    const vsbd_result* cres;
    vsbd_batch_results_a(b->dev, s, &mm, &cres);
    tally(b, s, 0, 0);
    vsb_frame_host_a(&b->md[s], mm, cres, &b->w[s]);
    if (b->w[s].fine_pass) {
      b->items[s] = b->w[s].items;
      b->nitems[s] = b->w[s].nitems;
    }
  }
  double t2 = vsb_now_s();
  if (vsbd_batch_stage_b(b->dev, b->items, b->nitems, b->fres) != 0) {
    vs_log_error("vsb_batch", "GPU stage B failed: %s\n", vsbd_error());
    for (int s = 0; s < b->n; s++)
      if (b->search[s]) vsb_frame_discard(&b->w[s]);
    return VS_ERROR;
  }
  double t3 = vsb_now_s();
  for (int s = 0; s < b->n; s++)
    if (b->search[s] && b->nitems[s] > 0) tally(b, s, 1, b->nitems[s]);
  int trf_rc = VS_OK;
  /* the host parts of every stream first: a failed allocation in one drops
     the step for all, before any stream's frame ends */
  int bad = -1;
  for (int s = 0; s < b->n; s++) {
    int rc = b->search[s] ? vsb_frame_host_b(&b->md[s], b->fres[s], &b->w[s], &motions[s])
                          : vsb_frame_first(&b->md[s], &motions[s]);
    if (rc != VS_OK) {
      bad = s;
      for (int q = 0; q < s; q++) vs_vector_del(&motions[q]);
      for (int q = s + 1; q < b->n; q++)
        if (b->search[q]) vsb_frame_discard(&b->w[q]);
      break;
    }
  }
  if (bad >= 0) return VS_ERROR;
  for (int s = 0; s < b->n; s++) {
    if (vsb_frame_end(&b->md[s])) vsbd_batch_commit(b->dev, s);
    if (write_trf(b, s, &motions[s]) != VS_OK) trf_rc = VS_ERROR;
  }
  prof[0] = t1 - t0;
  prof[1] = t2 - t1;
  prof[2] = t3 - t2;
  prof[3] = vsb_now_s() - t3;
  vsb_prof_add(prof, b->n);
  return trf_rc;
}

/* a step's motions into the record array */
static long emit_step(vsb_batch* b, LocalMotions* lms, int k, LocalMotion* rec, long total,
                      long cap, int* counts) {
  for (int s = 0; s < b->n; s++) {
    int m = vs_vector_size(&lms[s]);
    if (counts) counts[(size_t)k * b->n + s] = m;
    for (int i = 0; i < m; i++) {
      if (rec && total < cap) rec[total] = *LMGet(&lms[s], i);
      total++;
    }
    vs_vector_del(&lms[s]);
  }
  return total;
}

/* Overlap needs every stream's current frame to become its previous one
   (no virtual tripod) and every stream past its first frame. */
static int can_overlap(const vsb_batch* b, int check_seen) {
  for (int s = 0; s < b->n; s++) {
    if (b->md[s].conf.virtualTripod >= 1) return 0;
    if (check_seen && !b->md[s].hasSeenOneFrame) return 0;
  }
  return 1;
}

/* Steps k0.. with consecutive steps overlapped on the GPU.  Two stage As
   are kept in flight: step k+1's runs while the host selects step k's
   fields and step k's fine search runs after it, and step k+2's is enqueued
   as soon as step k's fine search is collected, so the GPU works while the
   host assembles step k's motions.  Same results as vsb_batch_detect step
   by step. */
static long run_overlapped(vsb_batch* b, const uint8_t* const* clips, const long* frame_bytes,
                           const int* pitches, int k0, int nframes, int on_device,
                           const uint8_t** planes, LocalMotions* lms, LocalMotion* rec,
                           long total, long cap, int* counts) {
  for (int s = 0; s < b->n; s++) planes[s] = clips[s] + (size_t)k0 * frame_bytes[s];
  if (vsbd_batch_stage_a(b->dev, planes, pitches, on_device) != 0) {
    vs_log_error("vsb_batch", "GPU stage A failed: %s\n", vsbd_error());
    return -1;
  }
  if (k0 + 1 < nframes) {
    for (int s = 0; s < b->n; s++) planes[s] = clips[s] + (size_t)(k0 + 1) * frame_bytes[s];
    if (vsbd_batch_stage_a_issue(b->dev, planes, pitches, on_device, 1) != 0) {
      vs_log_error("vsb_batch", "GPU stage A failed: %s\n", vsbd_error());
      vsbd_batch_drain(b->dev);
      return -1;
    }
  }
  for (int k = k0; k < nframes; k++) {
    /* wall time: [0] waiting for stage A, [1] host part A, [2] waiting for
       stage B, [3] host part B */
    double t0 = vsb_now_s(), prof[4] = { 0, 0, 0, 0 };
    for (int s = 0; s < b->n; s++) {
      const uint8_t* mm;
      const vsbd_result* cres;
      if (vsb_frame_begin(&b->md[s], &b->search[s]) != VS_OK || !b->search[s]) {
        for (int q = 0; q < s; q++) vsb_frame_discard(&b->w[q]);
        vsbd_batch_drain(b->dev);
        return -1;
      }
      vsbd_batch_results_a(b->dev, s, &mm, &cres);
      tally(b, s, 0, 0);
      vsb_frame_host_a(&b->md[s], mm, cres, &b->w[s]);
      b->items[s] = b->w[s].fine_pass ? b->w[s].items : NULL;
      b->nitems[s] = b->w[s].fine_pass ? b->w[s].nitems : 0;
    }
    double t1 = vsb_now_s();
    prof[1] = t1 - t0;
    int rc = vsbd_batch_stage_b_issue(b->dev, b->items, b->nitems);
    if (rc == 0) rc = vsbd_batch_stage_b_collect(b->dev, b->fres);
    if (rc == 0)
      for (int s = 0; s < b->n; s++)
        if (b->nitems[s] > 0) tally(b, s, 1, b->nitems[s]);
    double t2 = vsb_now_s();
    prof[2] = t2 - t1;
    if (rc == 0 && k + 2 < nframes) {
      for (int s = 0; s < b->n; s++) planes[s] = clips[s] + (size_t)(k + 2) * frame_bytes[s];
      rc = vsbd_batch_stage_a_issue(b->dev, planes, pitches, on_device, 2);
    }
    if (rc != 0) {
      vs_log_error("vsb_batch", "GPU stage failed: %s\n", vsbd_error());
      vsbd_batch_drain(b->dev);
      for (int s = 0; s < b->n; s++) vsb_frame_discard(&b->w[s]);
      return -1;
    }
    int trf_rc = VS_OK;
    if (!b->trf) {
      /* no .trf to write: each stream's motions go straight into the
         record array, without an allocation per motion */
      for (int s = 0; s < b->n; s++) {
        const int nrec = vsb_frame_host_b_records(&b->md[s], b->fres[s], &b->w[s],
                                                  total < cap ? rec + total : NULL,
                                                  total < cap ? cap - total : 0);
        if (nrec < 0) {
          for (int q = s + 1; q < b->n; q++) vsb_frame_discard(&b->w[q]);
          vsbd_batch_drain(b->dev);
          return -1;
        }
        if (counts) counts[(size_t)k * b->n + s] = nrec;
        total += nrec;
      }
      for (int s = 0; s < b->n; s++)
        if (vsb_frame_end(&b->md[s])) vsbd_batch_commit(b->dev, s);
      double t3 = vsb_now_s();
      prof[3] = t3 - t2;
      if (k + 1 < nframes && vsbd_batch_stage_a_collect(b->dev) != 0) {
        vs_log_error("vsb_batch", "GPU stage A failed: %s\n", vsbd_error());
        vsbd_batch_drain(b->dev);
        return -1;
      }
      prof[0] = vsb_now_s() - t3;
      vsb_prof_add(prof, b->n);
      continue;
    }
    for (int s = 0; s < b->n; s++)
      if (vsb_frame_host_b(&b->md[s], b->fres[s], &b->w[s], &lms[s]) != VS_OK) {
        for (int q = 0; q < s; q++) vs_vector_del(&lms[q]);
        for (int q = s + 1; q < b->n; q++) vsb_frame_discard(&b->w[q]);
        vsbd_batch_drain(b->dev);
        return -1;
      }
    for (int s = 0; s < b->n; s++) {
      if (vsb_frame_end(&b->md[s])) vsbd_batch_commit(b->dev, s);
      if (write_trf(b, s, &lms[s]) != VS_OK) trf_rc = VS_ERROR;
    }
    total = emit_step(b, lms, k, rec, total, cap, counts);
    if (trf_rc != VS_OK) {
      vsbd_batch_drain(b->dev);
      return -1;
    }
    double t3 = vsb_now_s();
    prof[3] = t3 - t2;
    if (k + 1 < nframes && vsbd_batch_stage_a_collect(b->dev) != 0) {
      vs_log_error("vsb_batch", "GPU stage A failed: %s\n", vsbd_error());
      vsbd_batch_drain(b->dev);
      return -1;
    }
    prof[0] = vsb_now_s() - t3;
    vsb_prof_add(prof, b->n);
  }
  return total;
}

long vsb_batch_run(vsb_batch* b, const uint8_t* const* clips, const long* frame_bytes,
                   const int* pitches, int nframes, int on_device, void* out, long out_cap,
                   int* counts) {
  if (!b || !clips || !frame_bytes || !pitches || nframes < 0) return -1;
  const uint8_t** planes = (const uint8_t**)malloc(sizeof(uint8_t*) * (size_t)b->n);
  LocalMotions* lms = (LocalMotions*)malloc(sizeof(LocalMotions) * (size_t)b->n);
  LocalMotion* rec = (LocalMotion*)out;
  long total = 0;
  int k = 0;
  const int overlap = can_overlap(b, 0);
  for (; k < nframes && total >= 0; k++) {
    if (overlap && can_overlap(b, 1) && nframes - k > 1) {
      total = run_overlapped(b, clips, frame_bytes, pitches, k, nframes, on_device, planes, lms,
                             rec, total, out_cap, counts);
      break;
    }
    for (int s = 0; s < b->n; s++) planes[s] = clips[s] + (size_t)k * frame_bytes[s];
    if (vsb_batch_detect(b, planes, pitches, on_device, lms) != VS_OK) {
      total = -1;
      break;
    }
    total = emit_step(b, lms, k, rec, total, out_cap, counts);
  }
  free(planes);
  free(lms);
  return total;
}

long vsb_batch_launch_count(const vsb_batch* b) { return b ? vsbd_batch_launches(b->dev) : 0; }

int vsb_batch_class(const vsb_batch* b, int k, int* desc) {
  return b ? vsbd_batch_class(b->dev, k, desc) : -1;
}

int vsb_batch_grid(const vsb_batch* b, int* ctas, int* threads, long* smem) {
  return b && vsbd_batch_grid(b->dev, ctas, threads, smem) == 0 ? VS_OK : VS_ERROR;
}
