/*
 * vsoracle.c -- TEST INFRASTRUCTURE ONLY (see vsoracle.h).
 *
 * CPU restatement of the reference's motion-detection pass.  Every function
 * names the reference lines whose behaviour it restates; the code is written
 * for clarity (direct window sums, full SADs, explicit spiral legs), not for
 * speed.  Floating-point steps that decide output bits (contrast, match,
 * the cleaned means, the coarse-to-fine transform) keep the reference's
 * operation order and are compiled with the reference build's flags
 * (oracle/Makefile).
 */
#include "vsoracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------------ */
/* box blur                                                                  */
/* ------------------------------------------------------------------------ */

/* src/boxblur.c:109-122: below 2 the frame is copied; otherwise the size is
   made odd, at least 3 and at most half the smaller frame dimension.  The
   requested size is unsigned in the reference, and the lower clamp is an
   unsigned comparison. */
int orc_blur_size(int requested, int width, int height) {
  unsigned int s = (unsigned int)requested;
  if (s < 2) return (int)s;
  s = (s / 2) * 2 + 1;
  if (s < 3u) s = 3u;
  int hi = imin(height / 2, width / 2);
  if ((long)s > (long)hi) s = (unsigned int)hi;
  return (int)s;
}

/* Both reference passes keep a running sum over the window
   [i - size/2, i + size/2] with indices clamped to the row (edge pixels
   replicated) and emit floor(sum / size) as an 8-bit value
   (src/boxblur.c:206-236 and :299-327; the magic reciprocal of :69-85 is an
   exact floor division).  Restated here as a direct window sum. */
void orc_blur_hori(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int size) {
  int half = size / 2;
  for (int y = 0; y < height; y++) {
    const uint8_t* s = src + (long)y * src_ls;
    uint8_t* d = dst + (long)y * dst_ls;
    for (int x = 0; x < width; x++) {
      uint32_t acc = 0;
      for (int k = -half; k <= half; k++) acc += s[iclamp(x + k, 0, width - 1)];
      d[x] = (uint8_t)(acc / (uint32_t)size);
    }
  }
}

void orc_blur_vert(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int size) {
  int half = size / 2;
  for (int y = 0; y < height; y++) {
    uint8_t* d = dst + (long)y * dst_ls;
    for (int x = 0; x < width; x++) {
      uint32_t acc = 0;
      for (int k = -half; k <= half; k++)
        acc += src[(long)iclamp(y + k, 0, height - 1) * src_ls + x];
      d[x] = (uint8_t)(acc / (uint32_t)size);
    }
  }
}

/* src/boxblur.c:104-161 with BoxBlurNoColor: luma only */
void orc_blur_luma(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int stepSize) {
  int size = orc_blur_size(stepSize, width, height);
  if (size < 2) {
    for (int y = 0; y < height; y++)
      memcpy(dst + (long)y * dst_ls, src + (long)y * src_ls, (size_t)width);
    return;
  }
  uint8_t* tmp = (uint8_t*)malloc((size_t)width * height);
  orc_blur_hori(tmp, width, src, src_ls, width, height, size);
  orc_blur_vert(dst, dst_ls, tmp, width, width, height, size);
  free(tmp);
}

/* ------------------------------------------------------------------------ */
/* SAD and contrast                                                          */
/* ------------------------------------------------------------------------ */

/* src/motiondetect.c:971-996.  The early exit there only ever returns a
   value above the running minimum, and the caller only tests
   `error < minerror`, so the full sum selects the same minimum. */
uint32_t orc_sad(const uint8_t* I1, int ls1, const uint8_t* I2, int ls2,
                 int fx, int fy, int size, int bpp, int dx, int dy) {
  int h = size / 2;
  const uint8_t* a = I1 + (long)(fx - h) * bpp + (long)(fy - h) * ls1;
  const uint8_t* b = I2 + (long)(fx - h + dx) * bpp + (long)(fy - h + dy) * ls2;
  uint32_t sum = 0;
  for (int r = 0; r < size; r++) {
    for (int k = 0; k < size * bpp; k++) sum += (uint32_t)abs((int)a[k] - (int)b[k]);
    a += ls1;
    b += ls2;
  }
  return sum;
}

/* src/motiondetect.c:389-407 */
void orc_minmax(const uint8_t* I, int ls, int fx, int fy, int size, int bpp,
                uint8_t* mn, uint8_t* mx) {
  int h = size / 2;
  uint8_t lo = 255, hi = 0;
  for (int r = 0; r < size; r++) {
    const uint8_t* p = I + (long)(fx - h) * bpp + (long)(fy - h + r) * ls;
    for (int k = 0; k < size; k++) {
      uint8_t v = p[(long)k * bpp];
      if (v < lo) lo = v;
      if (v > hi) hi = v;
    }
  }
  *mn = lo;
  *mx = hi;
}

/* src/motiondetect.c:406: Michelson contrast with a 0.1 guard, in double */
double orc_contrast_from_minmax(int mn, int mx) {
  return (mx - mn) / (mx + mn + 0.1);
}

/* ------------------------------------------------------------------------ */
/* search                                                                    */
/* ------------------------------------------------------------------------ */

/* The outgoing square spiral of src/motiondetect.c:465-518: legs of length
   1,1,2,2,3,3,... in the directions +x, +y, -x, -y (repeating), one lattice
   step per move, starting at the origin.  Every point is visited before
   moving on; the walk ends at the first point outside the square
   |i|,|j| <= maxShift. */
int orc_spiral(int maxShift, int step, int* di, int* dj, int cap) {
  static const int mvx[4] = { 1, 0, -1, 0 };
  static const int mvy[4] = { 0, 1, 0, -1 };
  int i = 0, j = 0, n = 0;
  int leg = 0;
  for (;;) {
    int len = leg / 2 + 1;
    int d = leg % 4;
    for (int s = 0; s < len; s++) {
      if (i < -maxShift || i > maxShift || j < -maxShift || j > maxShift) return n;
      if (n < cap) { di[n] = i; dj[n] = j; }
      n++;
      i += mvx[d] * step;
      j += mvy[d] * step;
    }
    leg++;
  }
}

/* src/motiondetect.c:439-586 */
int orc_search_planar(const uint8_t* curr, int ls_c, const uint8_t* prev, int ls_p,
                      int fx, int fy, int size, int maxShift, int stepSize,
                      int ox, int oy, int* tx, int* ty, uint32_t* minerror) {
  int cap = (2 * (maxShift / (stepSize > 0 ? stepSize : 1)) + 3);
  cap = cap * cap;
  int* di = (int*)malloc(sizeof(int) * cap);
  int* dj = (int*)malloc(sizeof(int) * cap);
  int n = orc_spiral(maxShift, stepSize, di, dj, cap);
  uint32_t best = UINT_MAX;
  int bx = 0, by = 0;
  for (int k = 0; k < n && k < cap; k++) {
    uint32_t e = orc_sad(curr, ls_c, prev, ls_p, fx, fy, size, 1, di[k] + ox, dj[k] + oy);
    if (e < best) { best = e; bx = di[k]; by = dj[k]; }
  }
  free(di);
  free(dj);
  /* refinement around the best point, halving the step each round
     (src/motiondetect.c:545-567); the centre itself is not re-evaluated */
  int s = stepSize;
  while (s > 1) {
    int h = s / 2, r = s - h;
    int cx = bx, cy = by;
    for (int i = cx - r; i <= cx + r; i += h)
      for (int j = cy - r; j <= cy + r; j += h) {
        if (i == cx && j == cy) continue;
        uint32_t e = orc_sad(curr, ls_c, prev, ls_p, fx, fy, size, 1, i + ox, j + oy);
        if (e < best) { best = e; bx = i; by = j; }
      }
    s /= 2;
  }
  *tx = bx;
  *ty = by;
  *minerror = best;
  /* asymmetric range test of src/motiondetect.c:573-574 (s is the final step) */
  if (abs(bx) >= maxShift + s - 1 || abs(by) >= maxShift + s) return 0;
  return 1;
}

/* src/motiondetect.c:591-660: raster scan from -maxShift after the origin,
   one refinement ring at step 1 */
int orc_search_packed(const uint8_t* curr, int ls_c, const uint8_t* prev, int ls_p,
                      int fx, int fy, int size, int bpp, int maxShift, int stepSize,
                      int ox, int oy, int* tx, int* ty, uint32_t* minerror) {
  int bx = 0, by = 0;
  uint32_t best = orc_sad(curr, ls_c, prev, ls_p, fx, fy, size, bpp, ox, oy);
  for (int i = -maxShift; i <= maxShift; i += stepSize)
    for (int j = -maxShift; j <= maxShift; j += stepSize) {
      if (i == 0 && j == 0) continue;
      uint32_t e = orc_sad(curr, ls_c, prev, ls_p, fx, fy, size, bpp, i + ox, j + oy);
      if (e < best) { best = e; bx = i; by = j; }
    }
  if (stepSize > 1) {
    int cx = bx, cy = by, r = stepSize - 1;
    for (int i = cx - r; i <= cx + r; i++)
      for (int j = cy - r; j <= cy + r; j++) {
        if (i == cx && j == cy) continue;
        uint32_t e = orc_sad(curr, ls_c, prev, ls_p, fx, fy, size, bpp, i + ox, j + oy);
        if (e < best) { best = e; bx = i; by = j; }
      }
  }
  *tx = bx;
  *ty = by;
  *minerror = best;
  if (abs(bx) >= maxShift + stepSize - 1 || abs(by) >= maxShift + stepSize - 1) return 0;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */

/* src/motiondetect.c:314-358 */
static int orc_init_fields(orc_fields* fs, int W, int H, int accuracy, int size, int maxShift,
                           int stepSize, int keepBorder, int spacing, double thr) {
  fs->size = size;
  fs->maxShift = maxShift;
  fs->stepSize = stepSize;
  fs->contrastThreshold = thr;
  int rows = imax(3, (H - maxShift * 2) / (size + spacing) - 1);
  int cols = imax(3, (W - maxShift * 2) / (size + spacing) - 1);
  fs->num = rows * cols;
  fs->rows = rows;
  fs->x = (int16_t*)malloc(sizeof(int16_t) * fs->num);
  fs->y = (int16_t*)malloc(sizeof(int16_t) * fs->num);
  if (!fs->x || !fs->y) return 0;
  int border = keepBorder ? size / 2 + maxShift + stepSize : stepSize;
  int sx = (W - 2 * border) / imax(cols - 1, 1);
  int sy = (H - 2 * border) / imax(rows - 1, 1);
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) {
      fs->x[r * cols + c] = (int16_t)(border + c * sx);
      fs->y[r * cols + c] = (int16_t)(border + r * sy);
    }
  fs->maxFields = accuracy * fs->num / 15;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* field selection (src/motiondetect.c:662-743)                              */
/* ------------------------------------------------------------------------ */

typedef struct { double contrast; int index; } orc_ci;

/* descending by contrast, ties compare equal (src/motiondetect.c:665-669) */
static int orc_cmp_ci(const void* a, const void* b) {
  double x = ((const orc_ci*)a)->contrast, y = ((const orc_ci*)b)->contrast;
  return x < y ? 1 : (x > y ? -1 : 0);
}

/* Fills sel[] with the selected (index, contrast) pairs in the order the
   reference appends them; returns their number. */
static int orc_select(const orc_fields* fs, const double* contrast, orc_ci* sel) {
  int n = fs->num, nsel = 0;
  orc_ci* all = (orc_ci*)malloc(sizeof(orc_ci) * n);
  orc_ci* seg = (orc_ci*)malloc(sizeof(orc_ci) * n);
  for (int i = 0; i < n; i++) {
    all[i].contrast = contrast[i] < fs->contrastThreshold ? 0 : contrast[i];
    all[i].index = i;
  }
  memcpy(seg, all, sizeof(orc_ci) * n);
  int nseg = fs->rows + 1;
  int seglen = n / (fs->rows + 1) + 1;
  for (int s = 0; s < nseg; s++) {
    int a = seglen * s, b = imin(seglen * (s + 1), n);
    if (b - a > 0) qsort(seg + a, (size_t)(b - a), sizeof(orc_ci), orc_cmp_ci);
    for (int j = 0; j < fs->maxFields / nseg; j++) {
      if (a + j >= b) continue;
      if (seg[a + j].contrast > 0) {
        sel[nsel++] = all[seg[a + j].index];
        seg[a + j].contrast = 0;
      }
    }
  }
  int remaining = fs->maxFields - nsel;
  if (remaining > 0) {
    qsort(seg, (size_t)n, sizeof(orc_ci), orc_cmp_ci);
    for (int j = 0; j < remaining; j++)
      if (seg[j].contrast > 0) sel[nsel++] = seg[j];
  }
  free(all);
  free(seg);
  return nsel;
}

/* ------------------------------------------------------------------------ */
/* coarse -> fine transform (src/localmotion2transform.c:336-402,            */
/* src/transformtype.c:158-209, :445-461, :513-534)                          */
/* ------------------------------------------------------------------------ */

static int orc_cmp_double(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}
static int orc_cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

__attribute__((noinline)) double orc_cleanmean(double* ds, int len, double* mn, double* mx) {
  int cut = len / 5;
  double sum = 0;
  int i = 0;
  qsort(ds, len, sizeof(double), orc_cmp_double);
  for (i = cut; i < len - cut; i++) {
    sum += ds[i];
  }
  if (mn) *mn = ds[cut];
  if (mx) *mx = ds[len - cut - 1];
  return sum / (len - (2.0 * cut));
}

/* the cleaned mean shift is accumulated and stored in int16 fields
   (Vec, src/transformtype.c:513-534); kept out of line and returned by
   value as the reference's cleanmean_localmotions is, so that the compiler
   treats the caller's expressions alike */
typedef struct { int16_t x, y; } orc_vec;
typedef struct { orc_vec v; int16_t pad[3]; double c, m; } orc_meanlm;

__attribute__((noinline)) static orc_meanlm orc_cleanmean_shift(const orc_lm* lms, int n) {
  int cut = n / 5;
  int* xs = (int*)malloc(sizeof(int) * n);
  int* ys = (int*)malloc(sizeof(int) * n);
  for (int i = 0; i < n; i++) { xs[i] = lms[i].vx; ys[i] = lms[i].vy; }
  orc_meanlm m;
  memset(&m, 0, sizeof(m));
  qsort(xs, n, sizeof(int), orc_cmp_int);
  for (int i = cut; i < n - cut; i++) m.v.x += xs[i];
  qsort(ys, n, sizeof(int), orc_cmp_int);
  for (int i = cut; i < n - cut; i++) m.v.y += ys[i];
  free(xs);
  free(ys);
  m.v.x /= (n - (2.0 * cut));
  m.v.y /= (n - (2.0 * cut));
  return m;
}

/* src/localmotion2transform.c:336-349 */
__attribute__((noinline)) static double orc_angle(int fx, int fy, int fsize, int vx, int vy, int cx,
                                                 int cy) {
  if (abs(fx - cx) + abs(fy - cy) < fsize * 2) return 0;
  double a1 = atan2(fy - cy, fx - cx);
  double a2 = atan2(fy - cy + vy, fx - cx + vx);
  double diff = a2 - a1;
  return (diff > M_PI) ? diff - 2 * M_PI : ((diff < -M_PI) ? diff + 2 * M_PI : diff);
}

typedef struct { double x, y, alpha, zoom, barrel, rshutter; int extra; } orc_trans;

/* src/localmotion2transform.c:352-402: centre of the fields, trimmed mean
   shift, trimmed mean rotation (from 6 fields on), rotation re-centred on
   the frame centre */
static orc_trans orc_model(int width, int height, const orc_lm* lms, int n) {
  orc_trans t;
  memset(&t, 0, sizeof(t));
  if (n < 1) return t;
  int cx = 0, cy = 0;
  double* angles = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n; i++) { cx += lms[i].fx; cy += lms[i].fy; }
  cx /= n;
  cy /= n;
  orc_meanlm mean = orc_cleanmean_shift(lms, n);
  if (n < 6) {
    t.alpha = 0;
  } else {
    for (int i = 0; i < n; i++) {
      int16_t vx = (int16_t)(lms[i].vx - mean.v.x), vy = (int16_t)(lms[i].vy - mean.v.y);
      angles[i] = orc_angle(lms[i].fx, lms[i].fy, lms[i].fsize, vx, vy, cx, cy);
    }
    double mn, mx;
    t.alpha = -orc_cleanmean(angles, n, &mn, &mx);
    if (mx - mn > 1.0) t.alpha = 0;
  }
  free(angles);
  double p_x = (cx - width / 2);
  double p_y = (cy - height / 2);
  t.x = mean.v.x + (cos(t.alpha) - 1) * p_x - sin(t.alpha) * p_y;
  t.y = mean.v.y + sin(t.alpha) * p_x + (cos(t.alpha) - 1) * p_y;
  return t;
}

void orc_simple_transform(int width, int height, const orc_lm* lms, int n, double* out) {
  orc_trans t = orc_model(width, height, lms, n);
  out[0] = t.x;
  out[1] = t.y;
  out[2] = t.alpha;
  out[3] = t.zoom;
}

/* prepare_transform + transform_vec for the similarity model
   (src/transformtype.c:162-191, :207-208): the frame centre is integer,
   the new position is truncated to int16, the offset is the difference.
   Both steps stay out of line, as in the reference where they live in
   another translation unit than their caller. */
typedef struct { const orc_trans* t; double zcos, zsin, cx, cy, f, z; } orc_prep;

__attribute__((noinline)) static orc_prep orc_prepare(const orc_trans* t, int W, int H) {
  orc_prep p;
  p.t = t;
  double z = 1.0 + t->zoom / 100.0;
  p.zcos = z * cos(t->alpha);
  p.zsin = z * sin(t->alpha);
  p.cx = W / 2;
  p.cy = H / 2;
  p.z = z;
  p.f = 0.0;
  return p;
}

__attribute__((noinline)) static orc_vec orc_apply(const orc_prep* p, int16_t vx, int16_t vy) {
  double rx = vx - p->cx;
  double ry = vy - p->cy;
  double x = p->zcos * rx + p->zsin * ry + p->t->x + p->cx;
  double y = -p->zsin * rx + p->zcos * ry + p->t->y + p->cy;
  orc_vec r = { (int16_t)x, (int16_t)y };
  return r;
}

static void orc_field_offset(const orc_trans* t, int W, int H, int fx, int fy,
                             int16_t* ox, int16_t* oy) {
  orc_prep p = orc_prepare(t, W, H);
  orc_vec n = orc_apply(&p, (int16_t)fx, (int16_t)fy);
  *ox = (int16_t)(n.x - fx);
  *oy = (int16_t)(n.y - fy);
}

/* offset of a field for the transform {x, y, alpha, zoom} (test hook) */
void orc_offset(const double* t4, int W, int H, int fx, int fy, int16_t* ox, int16_t* oy) {
  orc_trans t;
  memset(&t, 0, sizeof(t));
  t.x = t4[0];
  t.y = t4[1];
  t.alpha = t4[2];
  t.zoom = t4[3];
  orc_field_offset(&t, W, H, fx, fy, ox, oy);
}

/* ------------------------------------------------------------------------ */
/* the pass                                                                  */
/* ------------------------------------------------------------------------ */

struct orc_md {
  int W, H, pformat, bpp, planar;
  int stepSize, accuracy, shakiness, tripod;
  double mincontrast;
  orc_fields coarse, fine;
  uint8_t* curr;
  uint8_t* prev;
  int ls;
  const uint8_t* last;   /* blurred plane of the most recent frame */
  int hasSeenOneFrame;
  int frameNum;
};

orc_md* orc_md_new(int W, int H, int pformat, int stepSize, int accuracy, int shakiness,
                   double mincontrast, int tripod) {
  if (pformat <= -1 || pformat == ORC_PF_PACKED || pformat >= ORC_PF_NUMBER) return NULL;
  if (W <= 0 || H <= 0) return NULL;
  orc_md* md = (orc_md*)calloc(1, sizeof(orc_md));
  md->W = W;
  md->H = H;
  md->pformat = pformat;
  md->planar = pformat < ORC_PF_PACKED;
  md->bpp = pformat == ORC_PF_RGBA ? 4 : (md->planar ? 1 : 3);
  /* parameter clamps of src/motiondetect.c:121-130 */
  shakiness = imin(10, imax(1, shakiness));
  accuracy = imin(15, imax(1, accuracy));
  if (accuracy < shakiness / 2) accuracy = shakiness / 2;
  if (accuracy > 9 && stepSize > 6) stepSize = 6;
  md->stepSize = stepSize;
  md->accuracy = accuracy;
  md->shakiness = shakiness;
  md->tripod = tripod;
  md->mincontrast = mincontrast;
  /* geometry of src/motiondetect.c:132-149; the +16 rounding always adds */
  int m = imin(W, H);
  int maxShift = imax(16, m / 7);
  int fsize = imax(16, m / 10);
  int fsizeFine = imax(6, m / 60);
  fsize = (fsize / 16 + 1) * 16;
  fsizeFine = (fsizeFine / 16 + 1) * 16;
  orc_init_fields(&md->coarse, W, H, accuracy, fsize, maxShift, stepSize, 1, 0, mincontrast);
  orc_init_fields(&md->fine, W, H, accuracy, fsizeFine, fsizeFine, 2, 1, fsizeFine,
                  mincontrast / 2);
  md->ls = W * md->bpp;
  md->curr = (uint8_t*)calloc((size_t)md->ls * H, 1);
  md->prev = (uint8_t*)calloc((size_t)md->ls * H, 1);
  return md;
}

const orc_fields* orc_md_fields(const orc_md* md, int which) {
  return which ? &md->fine : &md->coarse;
}
const uint8_t* orc_md_curr(const orc_md* md) { return md->last; }
int orc_md_frame_num(const orc_md* md) { return md->frameNum; }

void orc_md_free(orc_md* md) {
  if (!md) return;
  free(md->coarse.x); free(md->coarse.y);
  free(md->fine.x); free(md->fine.y);
  free(md->curr);
  free(md->prev);
  free(md);
}

/* (c0 + c1 + c2) / 3 as the reference's fast-math build evaluates it:
   ((c0 + c1) + c2) times the double nearest 1/3 (pinned against the
   reference by tests/test_oracle_pin.py) */
__attribute__((optimize("no-fast-math"), noinline)) static double orc_mean3(double a, double b,
                                                                             double c) {
  double s = a + b;
  s = s + c;
  return s * (1.0 / 3.0);
}

static double orc_field_contrast(const orc_md* md, int fx, int fy, int size) {
  uint8_t mn, mx;
  if (md->planar) {
    orc_minmax(md->curr, md->ls, fx, fy, size, 1, &mn, &mx);
    return orc_contrast_from_minmax(mn, mx);
  }
  /* src/motiondetect.c:370-377: mean of the three colour channels */
  double c[3];
  for (int ch = 0; ch < 3; ch++) {
    orc_minmax(md->curr + ch, md->ls, fx, fy, size, md->bpp, &mn, &mx);
    c[ch] = orc_contrast_from_minmax(mn, mx);
  }
  return orc_mean3(c[0], c[1], c[2]);
}

/* calcTransFields (src/motiondetect.c:752-807) for one field set; with
   use_offset the per-field search centre follows the transform t and fields
   whose search window would leave the frame are dropped
   (src/motiondetect.c:418-434) */
static int orc_trans_fields(orc_md* md, const orc_fields* fs, int use_offset, const orc_trans* t,
                            orc_lm* out) {
  double* con = (double*)malloc(sizeof(double) * fs->num);
  orc_ci* sel = (orc_ci*)malloc(sizeof(orc_ci) * (fs->num + 1));
  for (int i = 0; i < fs->num; i++) con[i] = orc_field_contrast(md, fs->x[i], fs->y[i], fs->size);
  int nsel = orc_select(fs, con, sel);
  int nout = 0;
  for (int k = 0; k < nsel; k++) {
    int i = sel[k].index;
    int fx = fs->x[i], fy = fs->y[i];
    int16_t ox = 0, oy = 0;
    if (use_offset) {
      orc_field_offset(t, md->W, md->H, fx, fy, &ox, &oy);
      int border = fs->size / 2 + fs->maxShift + fs->stepSize;
      int x = fx + ox, y = fy + oy;
      if (x - border < 0 || x + border >= md->W || y - border < 0 || y + border >= md->H)
        continue;
    }
    int tx, ty, ok;
    uint32_t e;
    if (md->planar)
      ok = orc_search_planar(md->curr, md->ls, md->prev, md->ls, fx, fy, fs->size, fs->maxShift,
                             fs->stepSize, ox, oy, &tx, &ty, &e);
    else
      ok = orc_search_packed(md->curr, md->ls, md->prev, md->ls, fx, fy, fs->size, md->bpp,
                             fs->maxShift, fs->stepSize, ox, oy, &tx, &ty, &e);
    if (!ok) continue;
    orc_lm* lm = &out[nout++];
    memset(lm, 0, sizeof(*lm));
    lm->vx = (int16_t)(tx + ox);
    lm->vy = (int16_t)(ty + oy);
    lm->fx = (int16_t)fx;
    lm->fy = (int16_t)fy;
    lm->fsize = (int16_t)fs->size;
    lm->match = ((double)e) / (fs->size * fs->size);
    lm->contrast = sel[k].contrast;
  }
  free(con);
  free(sel);
  return nout;
}

int orc_md_frame(orc_md* md, const uint8_t* plane0, int linesize, orc_lm* out, int cap) {
  int W = md->W, H = md->H;
  if (md->planar) {
    orc_blur_luma(md->curr, md->ls, plane0, linesize, W, H, md->stepSize);
  } else {
    for (int y = 0; y < H; y++)
      memcpy(md->curr + (long)y * md->ls, plane0 + (long)y * linesize, (size_t)md->ls);
  }
  int lead_in = md->tripod >= 1 && md->frameNum < md->tripod;
  int n = 0;
  if (md->hasSeenOneFrame && !lead_in) {
    orc_lm* coarse = (orc_lm*)malloc(sizeof(orc_lm) * (md->coarse.num + 1));
    orc_lm* fine = (orc_lm*)malloc(sizeof(orc_lm) * (md->fine.num + 1));
    int nc = orc_trans_fields(md, &md->coarse, 0, NULL, coarse);
    int nf = 0;
    if (nc >= 1) {
      orc_trans t = orc_model(W, H, coarse, nc);
      int nf2 = orc_trans_fields(md, &md->fine, 1, &t, fine);
      double* matches = (double*)malloc(sizeof(double) * nc);
      for (int i = 0; i < nc; i++) matches[i] = coarse[i].match;
      double meanMatch = orc_cleanmean(matches, nc, NULL, NULL);
      free(matches);
      for (int i = 0; i < nf2; i++)
        if (fine[i].match <= meanMatch) fine[nf++] = fine[i];
    }
    for (int i = 0; i < nc; i++) { if (n < cap) out[n] = coarse[i]; n++; }
    for (int i = 0; i < nf; i++) { if (n < cap) out[n] = fine[i]; n++; }
    free(coarse);
    free(fine);
  } else {
    md->hasSeenOneFrame = 1;
  }
  md->last = md->curr;
  if (md->tripod < 1 || md->frameNum < md->tripod) {
    uint8_t* t = md->prev;
    md->prev = md->curr;
    md->curr = t;
  }
  md->frameNum++;
  return n;
}
