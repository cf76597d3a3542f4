/*
 * vs_transform.c -- transform and local-motion helpers of the detect pass
 * (the API of src/transformtype_operations.h:44-173 of the reference).
 *
 * The floating-point routines here decide output bits of the detect pass:
 * cleanmean() gives the mean-match threshold of the fine fields and
 * prepare_transform()/transform_vec() give every fine field's search
 * offset.  They keep the reference's operation order and this file is built
 * with the reference build's floating-point flags (-O3 -msse2 -ffast-math),
 * so that the compiler makes the same choices for the same expressions.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vidstab_b200.h"
#include "vsb_host.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

VSTransform new_transform(double x, double y, double alpha, double zoom, double barrel,
                          double rshutter, int extra) {
  VSTransform t;
  t.x = x;
  t.y = y;
  while (alpha < -M_PI) alpha += 2.0 * M_PI;
  while (alpha > M_PI) alpha -= 2.0 * M_PI;
  t.alpha = alpha;
  t.zoom = zoom;
  t.barrel = barrel;
  t.rshutter = rshutter;
  t.extra = extra;
  return t;
}

VSTransform null_transform(void) { return new_transform(0, 0, 0, 0, 0, 0, 0); }

VSTransform add_transforms(const VSTransform* a, const VSTransform* b) {
  VSTransform t;
  t.x = a->x + b->x;
  t.y = a->y + b->y;
  t.alpha = a->alpha + b->alpha;
  t.zoom = a->zoom + b->zoom;
  t.barrel = a->barrel + b->barrel;
  t.rshutter = a->rshutter + b->rshutter;
  t.extra = a->extra || b->extra;
  return t;
}

VSTransform sub_transforms(const VSTransform* a, const VSTransform* b) {
  VSTransform t;
  t.x = a->x - b->x;
  t.y = a->y - b->y;
  t.alpha = a->alpha - b->alpha;
  t.zoom = a->zoom - b->zoom;
  t.barrel = a->barrel - b->barrel;
  t.rshutter = a->rshutter - b->rshutter;
  t.extra = a->extra || b->extra;
  return t;
}

VSTransform mult_transform(const VSTransform* a, double f) {
  VSTransform t;
  t.x = a->x * f;
  t.y = a->y * f;
  t.alpha = a->alpha * f;
  t.zoom = a->zoom * f;
  t.barrel = a->barrel * f;
  t.rshutter = a->rshutter * f;
  t.extra = a->extra;
  return t;
}

void storeVSTransform(FILE* f, const VSTransform* t) {
  fprintf(f, "Trans %lf %lf %lf %lf %i\n", t->x, t->y, t->alpha, t->zoom, t->extra);
}

/* similarity model of src/transformtype.c:162-184 (the rotational field-of-
   view model belongs to the transform pass and is not built here: f = 0) */
PreparedTransform prepare_transform(const VSTransform* t, const VSFrameInfo* fi) {
  PreparedTransform pt;
  memset(pt.r, 0, sizeof(pt.r));
  pt.t = t;
  double z = 1.0 + t->zoom / 100.0;
  pt.zcos_a = z * cos(t->alpha);
  pt.zsin_a = z * sin(t->alpha);
  pt.c_x = fi->width / 2;
  pt.c_y = fi->height / 2;
  pt.z = z;
  pt.f = 0.0;
  return pt;
}

/* src/transformtype.c:193-209 */
void transform_vec_double(double* x, double* y, const PreparedTransform* pt, const Vec* v) {
  double rx = v->x - pt->c_x;
  double ry = v->y - pt->c_y;
  if (pt->f > 0.0) {
    double X = pt->r[0] * rx + pt->r[1] * ry + pt->r[2] * pt->f;
    double Y = pt->r[3] * rx + pt->r[4] * ry + pt->r[5] * pt->f;
    double Z = pt->r[6] * rx + pt->r[7] * ry + pt->r[8] * pt->f;
    *x = pt->z * pt->f * X / Z + pt->c_x;
    *y = pt->z * pt->f * Y / Z + pt->c_y;
    return;
  }
  *x = pt->zcos_a * rx + pt->zsin_a * ry + pt->t->x + pt->c_x;
  *y = -pt->zsin_a * rx + pt->zcos_a * ry + pt->t->y + pt->c_y;
}

/* the double position is truncated to int16 (src/transformtype.c:186-191) */
Vec transform_vec(const PreparedTransform* pt, const Vec* v) {
  double x, y;
  transform_vec_double(&x, &y, pt, v);
  Vec r = { (int16_t)x, (int16_t)y };
  return r;
}

Vec sub_vec(Vec a, Vec b) {
  Vec r = { (int16_t)(a.x - b.x), (int16_t)(a.y - b.y) };
  return r;
}

Vec add_vec(Vec a, Vec b) {
  Vec r = { (int16_t)(a.x + b.x), (int16_t)(a.y + b.y) };
  return r;
}

Vec field_to_vec(Field f) {
  Vec r = { f.x, f.y };
  return r;
}

int cmp_double(const void* t1, const void* t2) {
  double a = *(const double*)t1, b = *(const double*)t2;
  return a < b ? -1 : (a > b ? 1 : 0);
}

int cmp_int(const void* t1, const void* t2) {
  int a = *(const int*)t1, b = *(const int*)t2;
  return a < b ? -1 : (a > b ? 1 : 0);
}

/* mean without the lowest and highest fifth; sorts ds
   (src/transformtype.c:445-459, same summation loop) */
double cleanmean(double* ds, int len, double* minimum, double* maximum) {
  int cut = len / 5;
  double sum = 0;
  int i = 0;
  qsort(ds, len, sizeof(double), cmp_double);
  for (i = cut; i < len - cut; i++) {
    sum += ds[i];
  }
  if (minimum) *minimum = ds[cut];
  if (maximum) *maximum = ds[len - cut - 1];
  return sum / (len - (2.0 * cut));
}

LocalMotion null_localmotion(void) {
  LocalMotion lm;
  memset(&lm, 0, sizeof(lm));
  return lm;
}

int* localmotions_getx(const LocalMotions* lms) {
  int n = vs_vector_size(lms);
  int* xs = (int*)vs_malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  if (!xs) {
    vsb_note_oom();
    return NULL;
  }
  for (int i = 0; i < n; i++) xs[i] = LMGet(lms, i)->v.x;
  return xs;
}

int* localmotions_gety(const LocalMotions* lms) {
  int n = vs_vector_size(lms);
  int* ys = (int*)vs_malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  if (!ys) {
    vsb_note_oom();
    return NULL;
  }
  for (int i = 0; i < n; i++) ys[i] = LMGet(lms, i)->v.y;
  return ys;
}

LocalMotion sub_localmotion(const LocalMotion* a, const LocalMotion* b) {
  LocalMotion r = *a;
  r.v.x -= b->v.x;
  r.v.y -= b->v.y;
  return r;
}

/* trimmed mean of the shifts; the sums and the quotient live in the int16
   members of a Vec (src/transformtype.c:513-534) */
LocalMotion cleanmean_localmotions(const LocalMotions* lms) {
  int len = vs_vector_size(lms);
  int i, cut = len / 5;
  int* xs = localmotions_getx(lms);
  int* ys = localmotions_gety(lms);
  LocalMotion m = null_localmotion();
  if (!xs || !ys) { /* counted as a failed allocation: the frame is dropped */
    if (xs) vs_free(xs);
    if (ys) vs_free(ys);
    return m;
  }
  m.v.x = 0;
  m.v.y = 0;
  qsort(xs, len, sizeof(int), cmp_int);
  for (i = cut; i < len - cut; i++) m.v.x += xs[i];
  qsort(ys, len, sizeof(int), cmp_int);
  for (i = cut; i < len - cut; i++) m.v.y += ys[i];
  vs_free(xs);
  vs_free(ys);
  m.v.x /= (len - (2.0 * cut));
  m.v.y /= (len - (2.0 * cut));
  return m;
}

VSArray localmotionsGetMatch(const LocalMotions* lms) {
  VSArray m = vs_array_new(vs_vector_size(lms));
  for (int i = 0; i < m.len; i++) m.dat[i] = LMGet(lms, i)->match;
  return m;
}

/* src/boxblur.c:109-122: odd, at least 3, at most half the smaller frame
   dimension; below 2 nothing is blurred.  The requested size is unsigned
   there, so is the lower clamp. */
int vsb_blur_size(int requested, int width, int height) {
  unsigned int s = (unsigned int)requested;
  if (s < 2) return (int)s;
  s = (s / 2) * 2 + 1;
  if (s < 3u) s = 3u;
  int hi = VS_MIN(height / 2, width / 2);
  if ((long)s > (long)hi) s = (unsigned int)(hi < 0 ? 0 : hi);
  return (int)s;
}
