/*
 * vs_l2t.c -- the second pass's drop-in entry points (src/localmotion2transform.c
 * :40-121 and :220-284 of the reference): one global transform per frame from
 * the frame's LocalMotions.  The fit itself runs on the GPU for every frame at
 * once (vsb_l2t.cu); this file gathers the caller's vectors into one record
 * array, writes the results back and produces the reference's
 * global_motions.trf lines.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vidstab_b200.h"
#include "vsb_device.h"

/* src/vidstabdefines.h:49 */
#define VS_DEBUG_LEVEL 2

/* frame k's records go to recs[first[k] .. first[k+1]) */
static int gather(const VSManyLocalMotions* motions, int len, LocalMotion** recs, long** first) {
  long total = 0;
  int k, i;
  *recs = NULL;
  *first = (long*)malloc(sizeof(long) * (size_t)(len + 1));
  if (!*first) return -1;
  for (k = 0; k < len; k++) {
    const LocalMotions* lms = VSMLMGet(motions, k);
    (*first)[k] = total;
    total += lms ? vs_vector_size(lms) : 0;
  }
  (*first)[len] = total;
  *recs = (LocalMotion*)malloc(sizeof(LocalMotion) * (size_t)(total > 0 ? total : 1));
  if (!*recs) {
    free(*first);
    *first = NULL;
    return -1;
  }
  for (k = 0; k < len; k++) {
    const LocalMotions* lms = VSMLMGet(motions, k);
    const int n = lms ? vs_vector_size(lms) : 0;
    for (i = 0; i < n; i++) (*recs)[(*first)[k] + i] = *LMGet(lms, i);
  }
  return 0;
}

/* the frame's line of global_motions.trf (src/localmotion2transform.c:225,
   :279-282) */
static void store_line(FILE* f, const VSTransform* t, int nmotions, double residual, int rounds) {
  if (!f) return;
  if (nmotions == 0)
    fprintf(f, "0 0 0 0 0 %i\n# no fields\n", t->extra);
  else
    fprintf(f, "0 %f %f %f %f %i\n#\t\t\t\t\t %f %i\n", t->x, t->y, t->alpha, t->zoom, t->extra,
            residual, rounds);
}

static void debug_line(const VSTransformData* td, const int* info, int nmotions,
                       double residual) {
  if (nmotions > 0 && (td->conf.verbose & VS_DEBUG_LEVEL))
    vs_log_info(td->conf.modName, "disabled (%i+%i)/%i,\tresidual: %f (%i)\n", info[1], info[2],
                nmotions, residual, info[0]);
}

int vsLocalmotions2Transforms(VSTransformData* td, const VSManyLocalMotions* motions,
                              VSTransformations* trans) {
  const int len = motions ? vs_vector_size(motions) : 0;
  FILE* f = NULL;
  int k;
  if (!td || !trans) return VS_ERROR;
  if (td->conf.estimateLensDistortion && td->conf.simpleMotionCalculation == 0) {
    vsbd_set_error("vsLocalmotions2Transforms: the lens-distortion estimate is not supported");
    vs_log_error(td->conf.modName ? td->conf.modName : "vidstab_b200",
                 "vsLocalmotions2Transforms: the lens-distortion estimate is not supported; "
                 "set conf.estimateLensDistortion = 0\n");
    return VS_ERROR;
  }
  trans->ts = (VSTransform*)vs_malloc(sizeof(VSTransform) * (size_t)(len > 0 ? len : 1));
  if (!trans->ts) return VS_ERROR;
  if (td->conf.storeTransforms) f = fopen("global_motions.trf", "w");

  if (td->conf.simpleMotionCalculation == 0) {
    LocalMotion* recs = NULL;
    long* first = NULL;
    double* resid = NULL;
    int* info = NULL;
    int rc = gather(motions, len, &recs, &first);
    if (rc == 0) {
      resid = (double*)malloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
      info = (int*)malloc(sizeof(int) * 3 * (size_t)(len > 0 ? len : 1));
      rc = (resid && info) ? 0 : -1;
    }
    if (rc == 0)
      rc = vsb_motions_to_transforms(recs, first, len, td->fiSrc.width, td->fiSrc.height,
                                     td->conf.fov, td->conf.smoothZoom, trans->ts, resid, info);
    if (rc == 0) {
      for (k = 0; k < len; k++) {
        const int n = (int)(first[k + 1] - first[k]);
        debug_line(td, info + 3 * k, n, resid[k]);
        store_line(f, &trans->ts[k], n, resid[k], info[3 * k]);
      }
    } else {
      vs_log_error(td->conf.modName ? td->conf.modName : "vidstab_b200",
                   "vsLocalmotions2Transforms: %s\n", vsb_last_error());
    }
    free(recs);
    free(first);
    free(resid);
    free(info);
    if (rc != 0) {
      if (f) fclose(f);
      vs_free(trans->ts);
      trans->ts = NULL;
      return VS_ERROR;
    }
  } else {
    for (k = 0; k < len; k++)
      trans->ts[k] = vsSimpleMotionsToTransform(td->fiSrc, td->conf.modName, VSMLMGet(motions, k));
  }
  trans->len = len;
  if (f) fclose(f);
  return VS_OK;
}

VSTransform vsMotionsToTransform(VSTransformData* td, const LocalMotions* motions, FILE* f) {
  VSTransform t = null_transform();
  const int n = motions ? vs_vector_size(motions) : 0;
  LocalMotion* recs;
  long first[2] = {0, n};
  double resid = 0.0;
  int info[3] = {0, 0, 0};
  int i;
  if (!td) return t;
  recs = (LocalMotion*)malloc(sizeof(LocalMotion) * (size_t)(n > 0 ? n : 1));
  if (!recs) {
    t.extra = 1;
    return t;
  }
  for (i = 0; i < n; i++) recs[i] = *LMGet(motions, i);
  if (vsb_motions_to_transforms(recs, first, 1, td->fiSrc.width, td->fiSrc.height, td->conf.fov,
                                td->conf.smoothZoom, &t, &resid, info) != 0) {
    vs_log_error(td->conf.modName ? td->conf.modName : "vidstab_b200",
                 "vsMotionsToTransform: %s\n", vsb_last_error());
    t = null_transform();
    t.extra = 1;
  } else {
    debug_line(td, info, n, resid);
    store_line(f, &t, n, resid, info[0]);
  }
  free(recs);
  return t;
}
