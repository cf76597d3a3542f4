/*
 * vs_motionmodel.c -- the simple global model the detect pass fits to the
 * coarse local motions to centre the fine search (the counterpart of
 * src/localmotion2transform.c:336-402 of the reference).  Built with the
 * reference build's floating-point flags; the operation order is the
 * reference's because the result is truncated to whole pixels per fine
 * field and any last-bit difference could move a search window.
 */
#include <math.h>
#include <stdlib.h>

#include "vidstab_b200.h"
#include "vsb_host.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* rotation of one field about the centre, 0 for fields near it */
double vsCalcAngle(const LocalMotion* lm, int center_x, int center_y) {
  if (abs(lm->f.x - center_x) + abs(lm->f.y - center_y) < lm->f.size * 2) return 0;
  double a1 = atan2(lm->f.y - center_y, lm->f.x - center_x);
  double a2 = atan2(lm->f.y - center_y + lm->v.y, lm->f.x - center_x + lm->v.x);
  double diff = a2 - a1;
  return (diff > M_PI) ? diff - 2 * M_PI : ((diff < -M_PI) ? diff + 2 * M_PI : diff);
}

VSTransform vsSimpleMotionsToTransform(VSFrameInfo fi, const char* modName,
                                       const LocalMotions* motions) {
  int center_x = 0;
  int center_y = 0;
  VSTransform t = null_transform();
  if (motions == 0) return t;
  int num_motions = vs_vector_size(motions);
  if (num_motions < 1) return t;
  double* angles = (double*)vs_malloc(sizeof(double) * num_motions);
  if (!angles) { /* counted as a failed allocation: the frame is dropped */
    vsb_note_oom();
    return t;
  }
  LocalMotion meanmotion;
  int i;

  for (i = 0; i < num_motions; i++) {
    center_x += LMGet(motions, i)->f.x;
    center_y += LMGet(motions, i)->f.y;
  }
  center_x /= num_motions;
  center_y /= num_motions;

  meanmotion = cleanmean_localmotions(motions);

  if (num_motions < 6) {
    t.alpha = 0; /* too few fields for a rotation estimate */
  } else {
    for (i = 0; i < num_motions; i++) {
      LocalMotion m = sub_localmotion(LMGet(motions, i), &meanmotion);
      angles[i] = vsCalcAngle(&m, center_x, center_y);
    }
    double min, max;
    t.alpha = -cleanmean(angles, num_motions, &min, &max);
    if (max - min > 1.0) {
      t.alpha = 0;
      vs_log_info(modName, "too large variation in angle(%f)\n", max - min);
    }
  }
  vs_free(angles);
  /* rotation about the frame centre instead of the fields' centre */
  double p_x = (center_x - fi.width / 2);
  double p_y = (center_y - fi.height / 2);
  t.x = meanmotion.v.x + (cos(t.alpha) - 1) * p_x - sin(t.alpha) * p_y;
  t.y = meanmotion.v.y + sin(t.alpha) * p_x + (cos(t.alpha) - 1) * p_y;
  return t;
}
