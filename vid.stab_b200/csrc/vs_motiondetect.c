/*
 * vs_motiondetect.c -- the detect API (src/motiondetect.h:121-147 of the
 * reference) over the sm_100a kernels.
 *
 * Per frame (src/motiondetect.c:191-305):
 *   stage A on the GPU: upload plane 0, box-blur it, 8-bit min/max of every
 *       coarse and fine field, full coarse search of every coarse field
 *       (speculatively: selection cannot shrink the work below "every field
 *       with enough contrast" at the default accuracy 15, and searching all
 *       saves a host round trip), one copy back;
 *   host: contrasts, field selection with a stable merge sort that gives
 *       the permutation glibc's qsort gives with the reference's comparator
 *       (the tie order decides which fields are kept and
 *       the output order), coarse LocalMotions, the simple global model, the
 *       per-field fine offsets;
 *   stage B on the GPU: fine search of the selected fine fields, copy back;
 *   host: mean-match filter, concatenation.
 *
 * Device state lives in a table keyed by the VSMotionDetect address, since
 * the struct layout is ABI and has no slot for it.  This file is compiled
 * with strict IEEE arithmetic: the two divisions it performs (contrast and
 * match) are single divisions in the reference as well.
 */
#include <limits.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "vidstab_b200.h"
#include "vsb_device.h"
#include "vsb_host.h"

/* (contrast, field index) as the reference sorts it (src/motiondetect.c:54-57) */
typedef struct {
  double contrast;
  int index;
} contrast_idx;

struct md_state {
  const VSMotionDetect* key;
  vsbd_ctx* dev;
  int planar, bpp, nch;
  double* con_c;       /* coarse contrasts */
  double* con_f;       /* fine contrasts */
  contrast_idx* ci;    /* selection scratch: original, */
  contrast_idx* seg;   /* per-segment sorted copy, */
  contrast_idx* sel;   /* result in append order */
  contrast_idx* tmp;   /* merge buffer of the sort */
  vsbd_item* items;    /* fine work list */
  int* item_sel;       /* fine item -> position in sel */
  long frames;
  struct md_state* next;
};
typedef struct md_state md_state;

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static md_state* g_states = NULL;

static md_state* state_find(const VSMotionDetect* md) {
  pthread_mutex_lock(&g_lock);
  md_state* s = g_states;
  while (s && s->key != md) s = s->next;
  pthread_mutex_unlock(&g_lock);
  return s;
}

static void state_free(md_state* s) {
  if (!s) return;
  vsbd_destroy(s->dev);
  free(s->con_c);
  free(s->con_f);
  free(s->ci);
  free(s->seg);
  free(s->sel);
  free(s->tmp);
  free(s->items);
  free(s->item_sel);
  free(s);
}

static void state_remove(const VSMotionDetect* md) {
  pthread_mutex_lock(&g_lock);
  md_state** pp = &g_states;
  while (*pp && (*pp)->key != md) pp = &(*pp)->next;
  md_state* s = *pp;
  if (s) *pp = s->next;
  pthread_mutex_unlock(&g_lock);
  state_free(s);
}

static void state_insert(md_state* s) {
  pthread_mutex_lock(&g_lock);
  s->next = g_states;
  g_states = s;
  pthread_mutex_unlock(&g_lock);
}

vsbd_ctx* vsb_md_device(const VSMotionDetect* md) {
  md_state* s = state_find(md);
  return s ? s->dev : NULL;
}

/* ------------------------------------------------------------------------ */

VSMotionDetectConfig vsMotionDetectGetDefaultConfig(const char* modName) {
  VSMotionDetectConfig conf;
  memset(&conf, 0, sizeof(conf));
  conf.stepSize = 6;
  conf.accuracy = 15;
  conf.shakiness = 5;
  conf.virtualTripod = 0;
  conf.contrastThreshold = 0.25;
  conf.show = 0;
  conf.modName = modName;
  conf.numThreads = 0;
  return conf;
}

void vsMotionDetectGetConfig(VSMotionDetectConfig* conf, const VSMotionDetect* md) {
  if (md && conf) *conf = md->conf;
}

const VSFrameInfo* vsMotionDetectGetFrameInfo(const VSMotionDetect* md) { return &md->fi; }

/* field grid of src/motiondetect.c:314-358 */
static int init_fields(VSMotionDetect* md, VSMotionDetectFields* fs, int size, int maxShift,
                       int stepSize, int keepBorder, int spacing, double thr) {
  fs->fieldSize = size;
  fs->maxShift = maxShift;
  fs->stepSize = stepSize;
  fs->useOffset = 0;
  fs->contrastThreshold = thr;
  int rows = VS_MAX(3, (md->fi.height - maxShift * 2) / (size + spacing) - 1);
  int cols = VS_MAX(3, (md->fi.width - maxShift * 2) / (size + spacing) - 1);
  fs->fieldNum = rows * cols;
  fs->fieldRows = rows;
  fs->fields = (Field*)vs_malloc(sizeof(Field) * (size_t)fs->fieldNum);
  if (!fs->fields) {
    vs_log_error(md->conf.modName, "malloc failed!\n");
    return 0;
  }
  int border = keepBorder ? size / 2 + maxShift + stepSize : stepSize;
  int sx = (md->fi.width - 2 * border) / VS_MAX(cols - 1, 1);
  int sy = (md->fi.height - 2 * border) / VS_MAX(rows - 1, 1);
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) {
      Field* f = &fs->fields[r * cols + c];
      f->x = (int16_t)(border + c * sx);
      f->y = (int16_t)(border + r * sy);
      f->size = (int16_t)size;
    }
  fs->maxFields = md->conf.accuracy * fs->fieldNum / 15;
  vs_log_info(md->conf.modName, "Fieldsize: %i, Maximal translation: %i pixel\n", size, maxShift);
  vs_log_info(md->conf.modName, "Number of used measurement fields: %i out of %i\n",
              fs->maxFields, fs->fieldNum);
  return 1;
}

/* Candidate geometry of one field set for the GPU search.
   Planar: the spiral of src/motiondetect.c:465-518 visits exactly the square
   lattice |i|,|j| <= K*step, K = maxShift/step; rank = visiting index.
   Packed: (0,0) first, then the raster i = -maxShift, -maxShift+step, ...
   (outer), j likewise (inner) of :613-628. */
int vsb_build_geom(vsbd_geom* g, int32_t** order_out, int size, int bpp, int maxShift,
                      int step, int planar) {
  memset(g, 0, sizeof(*g));
  g->size = size;
  g->bpp = bpp;
  g->step = step;
  int32_t* order = NULL;
  if (planar) {
    int K = maxShift / step;
    g->na = g->nb = 2 * K + 1;
    g->ax0 = g->by0 = -K * step;
    order = (int32_t*)malloc(sizeof(int32_t) * (size_t)g->na * g->nb);
    if (!order) return -1;
    for (int k = 0; k < g->na * g->nb; k++) order[k] = -1;
    /* walk the spiral: legs of 1,1,2,2,3,3,... lattice steps, turning
       +x -> +y -> -x -> -y */
    int a = 0, b = 0, rank = 0, leg = 0, done = 0;
    while (!done) {
      int len = leg / 2 + 1, d = leg & 3;
      for (int s = 0; s < len; s++) {
        if (a < -K || a > K || b < -K || b > K) { done = 1; break; }
        order[(b + K) * g->na + (a + K)] = rank++;
        a += d == 0 ? 1 : (d == 2 ? -1 : 0);
        b += d == 1 ? 1 : (d == 3 ? -1 : 0);
      }
      leg++;
    }
    for (int k = 0; k < g->na * g->nb; k++)
      if (order[k] < 0) { free(order); return -1; }
    int s = step;
    while (s > 1) {
      if (g->nstages >= VSBD_MAX_STAGES) { free(order); return -1; }
      int h = s / 2;
      g->st_r[g->nstages] = s - h;
      g->st_h[g->nstages] = h;
      g->nstages++;
      s = h;
    }
    g->limx = maxShift + s - 1;
    g->limy = maxShift + s;
  } else {
    g->na = g->nb = (2 * maxShift) / step + 1;
    g->ax0 = g->by0 = -maxShift;
    g->has_origin = 1;
    order = (int32_t*)malloc(sizeof(int32_t) * (size_t)g->na * g->nb);
    if (!order) return -1;
    for (int a = 0; a < g->na; a++)
      for (int b = 0; b < g->nb; b++) order[b * g->na + a] = 1 + a * g->nb + b;
    if (step > 1) {
      g->st_r[0] = step - 1;
      g->st_h[0] = 1;
      g->nstages = 1;
    }
    g->limx = g->limy = maxShift + step - 1;
  }
  g->order = order;
  *order_out = order;
  return 0;
}

/* how far a search can reach from the field's lattice centre */
static void geom_reach(const vsbd_geom* g, int* lo, int* hi) {
  int refine = 0;
  for (int k = 0; k < g->nstages; k++) refine += g->st_r[k];
  *lo = g->ax0 - refine;
  *hi = g->ax0 + (g->na - 1) * g->step + refine;
  if (g->has_origin) {
    if (*lo > 0) *lo = 0;
    if (*hi < 0) *hi = 0;
  }
}

/* every read of a coarse search and of a field's min/max stays inside the
   frame; the reference has undefined behaviour otherwise */
static int geometry_fits(const VSMotionDetect* md, const VSMotionDetectFields* fs,
                         const vsbd_geom* g, int searched_without_offset) {
  int lo, hi;
  geom_reach(g, &lo, &hi);
  for (int i = 0; i < fs->fieldNum; i++) {
    int x0 = fs->fields[i].x - fs->fieldSize / 2, y0 = fs->fields[i].y - fs->fieldSize / 2;
    if (x0 < 0 || y0 < 0 || x0 + fs->fieldSize > md->fi.width || y0 + fs->fieldSize > md->fi.height)
      return 0;
    if (searched_without_offset &&
        (x0 + lo < 0 || y0 + lo < 0 || x0 + fs->fieldSize + hi > md->fi.width ||
         y0 + fs->fieldSize + hi > md->fi.height))
      return 0;
  }
  return 1;
}

int vsMotionDetectInit(VSMotionDetect* md, const VSMotionDetectConfig* conf, const VSFrameInfo* fi) {
  return vsb_md_init(md, conf, fi, 1, NULL);
}

void vsb_md_layout_free(vsb_md_layout* lay) {
  if (!lay) return;
  free(lay->order_c);
  free(lay->order_f);
  free(lay->xy);
  memset(lay, 0, sizeof(*lay));
}

int vsb_md_init(VSMotionDetect* md, const VSMotionDetectConfig* conf, const VSFrameInfo* fi,
                int with_device, vsb_md_layout* lay) {
  if (!md || !conf || !fi) return VS_ERROR;
  if (!with_device && !lay) return VS_ERROR;
  md->conf = *conf;
  md->fi = *fi;
  if (fi->pFormat <= PF_NONE || fi->pFormat == PF_PACKED || fi->pFormat >= PF_NUMBER) {
    vs_log_warn(md->conf.modName, "unsupported Pixel Format (%i)\n", md->fi.pFormat);
    return VS_ERROR;
  }
  /* a detector re-initialised without cleanup drops its previous device state */
  state_remove(md);

  vsFrameNull(&md->curr);
  vsFrameNull(&md->currorig);
  vsFrameNull(&md->currtmp);
  vsFrameNull(&md->prev);
  md->hasSeenOneFrame = 0;
  md->frameNum = 0;
  md->fieldscoarse.fields = NULL;
  md->fieldsfine.fields = NULL;
  md->initialized = 0;

  /* read before written, as in the reference: anything but the two valid
     modes (a zeroed struct included) becomes binary */
  if (md->serializationMode != ASCII_SERIALIZATION_MODE &&
      md->serializationMode != BINARY_SERIALIZATION_MODE)
    md->serializationMode = BINARY_SERIALIZATION_MODE;

  md->conf.shakiness = VS_MIN(10, VS_MAX(1, md->conf.shakiness));
  md->conf.accuracy = VS_MIN(15, VS_MAX(1, md->conf.accuracy));
  if (md->conf.accuracy < md->conf.shakiness / 2) {
    vs_log_info(md->conf.modName, "Accuracy should not be lower than shakiness/2 -- fixed");
    md->conf.accuracy = md->conf.shakiness / 2;
  }
  if (md->conf.accuracy > 9 && md->conf.stepSize > 6) {
    vs_log_info(md->conf.modName, "For high accuracy use lower stepsize  -- set to 6 now");
    md->conf.stepSize = 6;
  }
  if (md->conf.stepSize < 1) {
    /* the reference's spiral never terminates for a step of 0 */
    vs_log_error(md->conf.modName, "stepsize must be at least 1 (got %i)\n", md->conf.stepSize);
    return VS_ERROR;
  }

  /* fixed geometry of src/motiondetect.c:132-149; the rounding to the next
     multiple of 16 always adds */
  int minDimension = VS_MIN(md->fi.width, md->fi.height);
  int maxShift = VS_MAX(16, minDimension / 7);
  int fieldSize = VS_MAX(16, minDimension / 10);
  int fieldSizeFine = VS_MAX(6, minDimension / 60);
  fieldSize = (fieldSize / 16 + 1) * 16;
  fieldSizeFine = (fieldSizeFine / 16 + 1) * 16;
  if (!init_fields(md, &md->fieldscoarse, fieldSize, maxShift, md->conf.stepSize, 1, 0,
                   md->conf.contrastThreshold))
    return VS_ERROR;
  if (!init_fields(md, &md->fieldsfine, fieldSizeFine, fieldSizeFine, 2, 1, fieldSizeFine,
                   md->conf.contrastThreshold / 2)) {
    vs_free(md->fieldscoarse.fields);
    md->fieldscoarse.fields = NULL;
    return VS_ERROR;
  }

  md_state* st = (md_state*)calloc(1, sizeof(md_state));
  if (!st) {
    vs_log_error(md->conf.modName, "malloc failed!\n");
    vs_free(md->fieldscoarse.fields);
    vs_free(md->fieldsfine.fields);
    md->fieldscoarse.fields = NULL;
    md->fieldsfine.fields = NULL;
    return VS_ERROR;
  }
  st->key = md;
  st->planar = md->fi.pFormat < PF_PACKED;
  st->bpp = st->planar ? 1 : md->fi.bytesPerPixel;
  st->nch = st->planar ? 1 : 3;
  int nc = md->fieldscoarse.fieldNum, nf = md->fieldsfine.fieldNum;
  int nmax = VS_MAX(nc, nf) + 1;
  st->con_c = (double*)malloc(sizeof(double) * (size_t)(nc + 1));
  st->con_f = (double*)malloc(sizeof(double) * (size_t)(nf + 1));
  st->ci = (contrast_idx*)malloc(sizeof(contrast_idx) * (size_t)nmax);
  st->seg = (contrast_idx*)malloc(sizeof(contrast_idx) * (size_t)nmax);
  st->sel = (contrast_idx*)malloc(sizeof(contrast_idx) * (size_t)nmax);
  st->tmp = (contrast_idx*)malloc(sizeof(contrast_idx) * (size_t)nmax);
  st->items = (vsbd_item*)malloc(sizeof(vsbd_item) * (size_t)(nf + 1));
  st->item_sel = (int*)malloc(sizeof(int) * (size_t)(nf + 1));

  vsbd_geom gc, gf;
  int32_t *oc = NULL, *of = NULL;
  int ok = st->con_c && st->con_f && st->ci && st->seg && st->sel && st->tmp && st->items &&
           st->item_sel;
  ok = ok && vsb_build_geom(&gc, &oc, fieldSize, st->bpp, maxShift, md->conf.stepSize, st->planar) == 0;
  ok = ok && vsb_build_geom(&gf, &of, fieldSizeFine, st->bpp, fieldSizeFine, 2, st->planar) == 0;
  if (ok && (!geometry_fits(md, &md->fieldscoarse, &gc, 1) ||
             !geometry_fits(md, &md->fieldsfine, &gf, 0))) {
    vs_log_error(md->conf.modName,
                 "frame %ix%i is too small for the measurement-field layout (fields or their "
                 "search range would leave the frame)\n",
                 md->fi.width, md->fi.height);
    ok = 0;
  }
  if (ok) {
    int16_t* xy = (int16_t*)malloc(sizeof(int16_t) * 2 * (size_t)(nc + nf + 1));
    if (!xy) {
      ok = 0;
      nc = nf = 0; /* nothing to fill */
    }
    for (int i = 0; i < nc; i++) {
      xy[i] = md->fieldscoarse.fields[i].x;
      xy[nc + i] = md->fieldscoarse.fields[i].y;
    }
    for (int i = 0; i < nf; i++) {
      xy[2 * nc + i] = md->fieldsfine.fields[i].x;
      xy[2 * nc + nf + i] = md->fieldsfine.fields[i].y;
    }
    int blur = st->planar ? vsb_blur_size(md->conf.stepSize, md->fi.width, md->fi.height) : 0;
    if (!ok) {
      /* no memory for the field table */
    } else if (!with_device) {
      /* the caller runs the device work (batched streams): hand it the layout */
      lay->coarse = gc;
      lay->fine = gf;
      lay->order_c = oc;
      lay->order_f = of;
      lay->xy = xy;
      lay->nc = nc;
      lay->nf = nf;
      lay->blur = blur;
      oc = of = NULL;
      xy = NULL;
    } else if (vsbd_create(&st->dev, md->fi.width, md->fi.height, st->bpp, blur, st->nch, &gc,
                           xy, xy + nc, nc, &gf, xy + 2 * nc, xy + 2 * nc + nf, nf,
                           md->fieldscoarse.contrastThreshold) != 0) {
      vs_log_error(md->conf.modName, "GPU initialisation failed: %s\n", vsbd_error());
      ok = 0;
    }
    free(xy);
  }
  free(oc);
  free(of);
  if (!ok) {
    state_free(st);
    vs_free(md->fieldscoarse.fields);
    vs_free(md->fieldsfine.fields);
    md->fieldscoarse.fields = NULL;
    md->fieldsfine.fields = NULL;
    return VS_ERROR;
  }
  if (with_device)
    vs_log_info(md->conf.modName, "GPU: sm_100a kernels, blur size %i\n",
                st->planar ? vsb_blur_size(md->conf.stepSize, md->fi.width, md->fi.height) : 0);
  state_insert(st);
  md->initialized = 2;
  return VS_OK;
}

void vsMotionDetectionCleanup(VSMotionDetect* md) {
  state_remove(md);
  if (md->fieldscoarse.fields) {
    vs_free(md->fieldscoarse.fields);
    md->fieldscoarse.fields = 0;
  }
  if (md->fieldsfine.fields) {
    vs_free(md->fieldsfine.fields);
    md->fieldsfine.fields = 0;
  }
  vsFrameFree(&md->prev);
  vsFrameFree(&md->curr);
  vsFrameFree(&md->currtmp);
  md->initialized = 0;
}

/* ------------------------------------------------------------------------ */
/* field selection (src/motiondetect.c:662-743)                              */
/* ------------------------------------------------------------------------ */

/* Sorts by descending contrast, keeping the order of equal contrasts.  The
   reference sorts with libc qsort and a comparator that orders by
   descending contrast and calls equal contrasts equal (cmp_contrast_idx,
   src/motiondetect.c:665-669); glibc's qsort is a stable merge sort at
   these sizes, so the permutation is the stable one, which this sort gives
   without a comparator call per comparison.  tmp holds n elements. */
static void sort_contrast_desc(contrast_idx* a, int n, contrast_idx* tmp) {
  if (n < 2) return;
  if (n <= 24) {
    for (int i = 1; i < n; i++) {
      contrast_idx x = a[i];
      int j = i;
      while (j > 0 && a[j - 1].contrast < x.contrast) {
        a[j] = a[j - 1];
        j--;
      }
      a[j] = x;
    }
    return;
  }
  int h = n / 2;
  sort_contrast_desc(a, h, tmp);
  sort_contrast_desc(a + h, n - h, tmp);
  int i = 0, j = h, k = 0;
  while (i < h && j < n) tmp[k++] = a[j].contrast > a[i].contrast ? a[j++] : a[i++];
  while (i < h) tmp[k++] = a[i++];
  while (j < n) tmp[k++] = a[j++];
  memcpy(a, tmp, sizeof(contrast_idx) * (size_t)n);
}

/* fills st->sel in the reference's append order; returns the count */
static int select_fields(md_state* st, const VSMotionDetectFields* fs, const double* contrast) {
  int n = fs->fieldNum, nsel = 0;
  contrast_idx* ci = st->ci;
  contrast_idx* seg = st->seg;
  for (int i = 0; i < n; i++) {
    ci[i].contrast = contrast[i] < fs->contrastThreshold ? 0 : contrast[i];
    ci[i].index = i;
  }
  memcpy(seg, ci, sizeof(contrast_idx) * (size_t)n);
  int numsegms = fs->fieldRows + 1;
  int segmlen = n / (fs->fieldRows + 1) + 1;
  int per_seg = fs->maxFields / numsegms;
  for (int s = 0; s < numsegms; s++) {
    int a = segmlen * s;
    int b = VS_MIN(segmlen * (s + 1), n);
    sort_contrast_desc(seg + a, b - a > 0 ? b - a : 0, st->tmp);
    for (int j = 0; j < per_seg; j++) {
      if (a + j >= b) continue;
      if (seg[a + j].contrast > 0) {
        st->sel[nsel++] = ci[seg[a + j].index];
        seg[a + j].contrast = 0;
      }
    }
  }
  int remaining = fs->maxFields - nsel;
  if (remaining > 0) {
    sort_contrast_desc(seg, n, st->tmp);
    for (int j = 0; j < remaining; j++)
      if (seg[j].contrast > 0) st->sel[nsel++] = seg[j];
  }
  return nsel;
}

/* Mean of the three channel contrasts of a packed field
   (src/motiondetect.c:374-376).  The reference's fast-math build evaluates
   `(c0 + c1 + c2) / 3` as ((c0 + c1) + c2) times the double nearest 1/3;
   that order is written out here in strict arithmetic so that no compiler
   choice can change it. */
double vsb_mean3(double a, double b, double c) {
  double s = a + b;
  s = s + c;
  return s * (1.0 / 3.0);
}

/* Michelson contrast of one field from its 8-bit extremes
   (src/motiondetect.c:406; packed: mean over three channels, :374-376) */
static void field_contrasts(const md_state* st, const uint8_t* mm, int n, double* out) {
  for (int i = 0; i < n; i++) {
    const uint8_t* p = mm + (size_t)i * st->nch * 2;
    if (st->nch == 1) {
      int mini = p[0], maxi = p[1];
      out[i] = (maxi - mini) / (maxi + mini + 0.1);
    } else {
      double c[3];
      for (int k = 0; k < 3; k++) {
        int mini = p[2 * k], maxi = p[2 * k + 1];
        c[k] = (maxi - mini) / (maxi + mini + 0.1);
      }
      out[i] = vsb_mean3(c[0], c[1], c[2]);
    }
  }
}

static LocalMotion make_lm(const Field* f, int vx, int vy, double contrast, uint32_t sad) {
  LocalMotion lm = null_localmotion();
  lm.f = *f;
  lm.v.x = (int16_t)vx;
  lm.v.y = (int16_t)vy;
  lm.contrast = contrast;
  lm.match = ((double)sad) / (f->size * f->size);
  return lm;
}

static short match_at_most(void* thresh, void* lm) {
  return ((LocalMotion*)lm)->match <= *(double*)thresh ? 1 : 0;
}

int vsb_frame_begin(VSMotionDetect* md, int* search) {
  if (!md || md->initialized != 2) {
    vs_log_error(md ? md->conf.modName : "vid.stab", "motion detection is not initialised\n");
    return VS_ERROR;
  }
  if (!state_find(md)) {
    vs_log_error(md->conf.modName, "no device state for this detector\n");
    return VS_ERROR;
  }
  int leadIn = md->conf.virtualTripod >= 1 && md->frameNum < md->conf.virtualTripod;
  *search = md->hasSeenOneFrame && !leadIn;
  return VS_OK;
}

int vsb_frame_host_a(VSMotionDetect* md, const uint8_t* mm, const vsbd_result* cres,
                     vsb_frame_work* w) {
  md_state* st = state_find(md);
  VSMotionDetectFields* fc = &md->fieldscoarse;
  VSMotionDetectFields* ff = &md->fieldsfine;
  w->oom0 = vsb_oom_count();
  vs_vector_init(&w->coarse, fc->maxFields);
  vs_vector_init(&w->fine, 0);
  w->fine_pass = 0;
  w->nitems = 0;
  w->items = st->items;
  field_contrasts(st, mm, fc->fieldNum, st->con_c);
  field_contrasts(st, mm + (size_t)fc->fieldNum * st->nch * 2, ff->fieldNum, st->con_f);

  int nsel = select_fields(st, fc, st->con_c);
  for (int k = 0; k < nsel; k++) {
    int i = st->sel[k].index;
    const vsbd_result* r = &cres[i];
    if (!r->ok) continue;
    LocalMotion lm = make_lm(&fc->fields[i], r->tx, r->ty, st->sel[k].contrast, r->sad);
    vs_vector_append_dup(&w->coarse, &lm, sizeof(LocalMotion));
  }
  int num_motions = vs_vector_size(&w->coarse);
  if (num_motions < 1) {
    vs_log_warn(md->conf.modName, "too low contrast. (no translations are detected in frame %i)\n",
                md->frameNum);
    return VS_OK;
  }
  VSTransform t = vsSimpleMotionsToTransform(md->fi, md->conf.modName, &w->coarse);
  ff->offset = t;
  ff->useOffset = 1;
  int nfs = select_fields(st, ff, st->con_f);
  int nitems = 0;
  PreparedTransform pt = prepare_transform(&ff->offset, &md->fi);
  int border = ff->fieldSize / 2 + ff->maxShift + ff->stepSize;
  for (int k = 0; k < nfs; k++) {
    const Field* f = &ff->fields[st->sel[k].index];
    Vec pos = { f->x, f->y };
    Vec off = sub_vec(transform_vec(&pt, &pos), pos);
    int x = pos.x + off.x, y = pos.y + off.y;
    if (x - border < 0 || x + border >= md->fi.width || y - border < 0 ||
        y + border >= md->fi.height)
      continue; /* the shifted search would leave the frame (:429-433) */
    st->items[nitems].x = f->x;
    st->items[nitems].y = f->y;
    st->items[nitems].ox = off.x;
    st->items[nitems].oy = off.y;
    st->item_sel[nitems] = k;
    nitems++;
  }
  w->fine_pass = 1;
  w->nitems = nitems;
  return VS_OK;
}

int vsb_frame_host_b(VSMotionDetect* md, const vsbd_result* fres, vsb_frame_work* w,
                     LocalMotions* motions) {
  md_state* st = state_find(md);
  VSMotionDetectFields* ff = &md->fieldsfine;
  if (w->fine_pass) {
    /* the fine motions in item order, kept when their match is at most the
       coarse motions' trimmed mean (src/motiondetect.c:268-283); each one is
       built on the stack and only a kept one is allocated */
    VSArray q = localmotionsGetMatch(&w->coarse);
    double meanMatch = cleanmean(q.dat, q.len, NULL, NULL);
    for (int m = 0; m < w->nitems; m++) {
      if (!fres[m].ok) continue;
      const contrast_idx* s = &st->sel[st->item_sel[m]];
      LocalMotion lm = make_lm(&ff->fields[s->index], fres[m].tx + st->items[m].ox,
                               fres[m].ty + st->items[m].oy, s->contrast, fres[m].sad);
      if (match_at_most(&meanMatch, &lm)) vs_vector_append_dup(&w->fine, &lm, sizeof(LocalMotion));
    }
    vs_array_free(q);
  }
  if (vsb_oom_count() != w->oom0) {
    /* an allocation through the host's hooks failed: no partial result */
    vsb_frame_discard(w);
    vs_vector_init(motions, 0);
    vs_log_error(md->conf.modName, "out of memory in frame %i: frame dropped\n", md->frameNum);
    return VS_ERROR;
  }
  if (md->conf.show) vsb_draw_motions(md, &w->coarse, &w->fine);
  *motions = vs_vector_concat(&w->coarse, &w->fine);
  if (vsb_oom_count() != w->oom0) {
    vsb_frame_discard(w);
    vs_log_error(md->conf.modName, "out of memory in frame %i: frame dropped\n", md->frameNum);
    return VS_ERROR;
  }
  vs_vector_fini(&w->coarse);
  vs_vector_fini(&w->fine);
  return VS_OK;
}

int vsb_frame_host_b_records(VSMotionDetect* md, const vsbd_result* fres, vsb_frame_work* w,
                             LocalMotion* rec, long cap) {
  md_state* st = state_find(md);
  VSMotionDetectFields* ff = &md->fieldsfine;
  long n = 0;
  for (int i = 0; i < vs_vector_size(&w->coarse); i++, n++)
    if (rec && n < cap) rec[n] = *LMGet(&w->coarse, i);
  if (w->fine_pass) {
    VSArray q = localmotionsGetMatch(&w->coarse);
    double meanMatch = cleanmean(q.dat, q.len, NULL, NULL);
    for (int m = 0; m < w->nitems; m++) {
      if (!fres[m].ok) continue;
      const contrast_idx* s = &st->sel[st->item_sel[m]];
      LocalMotion lm = make_lm(&ff->fields[s->index], fres[m].tx + st->items[m].ox,
                               fres[m].ty + st->items[m].oy, s->contrast, fres[m].sad);
      if (match_at_most(&meanMatch, &lm)) {
        if (rec && n < cap) rec[n] = lm;
        n++;
      }
    }
    vs_array_free(q);
  }
  const int failed = vsb_oom_count() != w->oom0;
  vsb_frame_discard(w);
  if (failed) {
    vs_log_error(md->conf.modName, "out of memory in frame %i: frame dropped\n", md->frameNum);
    return -1;
  }
  return (int)n;
}

void vsb_frame_discard(vsb_frame_work* w) {
  vs_vector_del(&w->coarse);
  vs_vector_del(&w->fine);
}

int vsb_frame_first(VSMotionDetect* md, LocalMotions* motions) {
  if (vs_vector_init(motions, 1) != VS_OK) {
    vs_log_error(md->conf.modName, "out of memory in frame %i: frame dropped\n", md->frameNum);
    return VS_ERROR;
  }
  md->hasSeenOneFrame = 1;
  return VS_OK;
}

int vsb_frame_end(VSMotionDetect* md) {
  md_state* st = state_find(md);
  int commit = md->conf.virtualTripod < 1 || md->frameNum < md->conf.virtualTripod;
  md->frameNum++;
  if (st) st->frames++;
  return commit;
}

/* process-wide wall-time profile of the per-frame path (seconds): device
   stage A, host part A, device stage B, host part B (read by benchmarks) */
static double g_prof[4];
static long g_prof_frames;

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

void vsb_prof_add(const double* sec, long frames) {
  pthread_mutex_lock(&g_lock);
  for (int k = 0; k < 4; k++) g_prof[k] += sec[k];
  g_prof_frames += frames;
  pthread_mutex_unlock(&g_lock);
}

double vsb_now_s(void) { return now_s(); }

void vsb_host_profile(double* sec, long* frames, int reset) {
  pthread_mutex_lock(&g_lock);
  if (sec)
    for (int k = 0; k < 4; k++) sec[k] = g_prof[k];
  if (frames) *frames = g_prof_frames;
  if (reset) {
    memset(g_prof, 0, sizeof(g_prof));
    g_prof_frames = 0;
  }
  pthread_mutex_unlock(&g_lock);
}

int vsb_detect_common(VSMotionDetect* md, LocalMotions* motions, const uint8_t* host, int linesize,
                      const uint8_t* dev, int pitch) {
  int search = 0;
  if (!motions || vsb_frame_begin(md, &search) != VS_OK) return VS_ERROR;
  md_state* st = state_find(md);
  const uint8_t* mm = NULL;
  const vsbd_result* cres = NULL;
  double t[5] = { now_s(), 0, 0, 0, 0 };
  VSB_RANGE("vsb device stage A");
  const int rca = vsbd_stage_a(st->dev, host, linesize, dev, pitch, search, &mm, &cres);
  VSB_RANGE_END();
  if (rca != 0) {
    vs_log_error(md->conf.modName, "GPU stage A failed: %s\n", vsbd_error());
    return VS_ERROR;
  }
  t[1] = now_s();
  t[2] = t[3] = t[1];
  if (search) {
    vsb_frame_work w;
    VSB_RANGE("vsb host part A");
    vsb_frame_host_a(md, mm, cres, &w);
    VSB_RANGE_END();
    t[2] = now_s();
    const vsbd_result* fres = NULL;
    VSB_RANGE("vsb device stage B");
    const int rcb = w.fine_pass ? vsbd_stage_b(st->dev, w.items, w.nitems, &fres) : 0;
    VSB_RANGE_END();
    if (rcb != 0) {
      vs_log_error(md->conf.modName, "GPU stage B failed: %s\n", vsbd_error());
      vsb_frame_discard(&w);
      return VS_ERROR;
    }
    t[3] = now_s();
    VSB_RANGE("vsb host part B");
    const int rch = vsb_frame_host_b(md, fres, &w, motions);
    VSB_RANGE_END();
    if (rch != VS_OK) return VS_ERROR;
  } else if (vsb_frame_first(md, motions) != VS_OK) {
    return VS_ERROR;
  }
  if (vsb_frame_end(md)) vsbd_commit_prev(st->dev);
  t[4] = now_s();
  pthread_mutex_lock(&g_lock);
  for (int k = 0; k < 4; k++) g_prof[k] += t[k + 1] - t[k];
  g_prof_frames++;
  pthread_mutex_unlock(&g_lock);
  return VS_OK;
}

/* Copies a frame's motions into the record array and frees them. */
static long append_records(LocalMotions* lms, LocalMotion* rec, long total, long cap, int* count) {
  int n = vs_vector_size(lms);
  if (count) *count = n;
  for (int i = 0; i < n; i++) {
    if (rec && total < cap) rec[total] = *LMGet(lms, i);
    total++;
  }
  vs_vector_del(lms);
  return total;
}

int vsb_can_overlap(const VSMotionDetect* md) {
  md_state* st = state_find(md);
  return st && md->conf.virtualTripod < 1 && !md->conf.show && vsbd_can_overlap(st->dev);
}

/* Issues stage A of frame j of the clip (the frame after the last one
   issued) and, for host frames, copies frame j+1 into its upload slot
   (j+1) % 3; frame j was copied into slot j % 3 before.  0 or -1. */
static int issue_next_frame(VSMotionDetect* md, md_state* st, const uint8_t* frames,
                            long frame_bytes, int linesize, int nframes, int on_device, int j) {
  if ((on_device ? vsbd_stage_a_next_issue(st->dev, NULL, linesize,
                                           frames + (size_t)j * frame_bytes, linesize)
                 : vsbd_stage_a_next_issue_uploaded(st->dev, j % 3)) != 0 ||
      (!on_device && j + 1 < nframes &&
       vsbd_upload(st->dev, frames + (size_t)(j + 1) * frame_bytes, linesize, (j + 1) % 3) != 0)) {
    vs_log_error(md->conf.modName, "GPU stage A failed: %s\n", vsbd_error());
    return -1;
  }
  return 0;
}

/* A clip through the detector with consecutive frames overlapped on the
   GPU: stage A of frame k+1 (blur, min/max, coarse search) is enqueued
   before the host selects frame k's fields, and runs on one stream while
   the host works and frame k's fine search runs on the other; host frames
   are copied one frame further ahead on a third stream.  Same results, frame by frame,
   as calling vsMotionDetection (or vsb_motion_detection_device) in order.
   Plane 0 of frame k is at frames + k*frame_bytes (host memory, or device
   memory with on_device).  Returns the total number of records, or -1. */
long vsb_detect_run_overlapped(VSMotionDetect* md, const uint8_t* frames, long frame_bytes,
                               int linesize, int nframes, int on_device, LocalMotion* rec,
                               long out_cap, int* counts) {
  md_state* st = state_find(md);
  long total = 0;
  int k = 0;
  if (!st) return -1;
  /* the first frame only primes the detector */
  while (k < nframes && !md->hasSeenOneFrame) {
    LocalMotions lms;
    const uint8_t* src = frames + (size_t)k * frame_bytes;
    if (vsb_detect_common(md, &lms, on_device ? NULL : src, linesize, on_device ? src : NULL,
                          linesize) != VS_OK)
      return -1;
    total = append_records(&lms, rec, total, out_cap, counts ? counts + k : NULL);
    k++;
  }
  if (k >= nframes) return total;
  const uint8_t* mm = NULL;
  const vsbd_result* cres = NULL;
  {
    int search = 0;
    const uint8_t* src = frames + (size_t)k * frame_bytes;
    if (vsb_frame_begin(md, &search) != VS_OK || !search) return -1;
    if (vsbd_stage_a(st->dev, on_device ? NULL : src, linesize, on_device ? src : NULL, linesize,
                     1, &mm, &cres) != 0) {
      vs_log_error(md->conf.modName, "GPU stage A failed: %s\n", vsbd_error());
      return -1;
    }
  }
  /* Host frames travel ahead of their stage A: frame j is copied into
     upload slot j % 3 on the copy stream.  Plain search: two frames' stage A
     are kept in flight, so frame k+2's stage A is issued right after frame
     k's fine stage, before the host waits for that stage and assembles frame
     k; the GPU then has queued work while the host does.  With a proposal
     network frame k+1's stage A is not issued before frame k's fine stage
     (the network kernel fills every SM's shared memory and would hold the
     fine stage back), and while its verification runs only one frame's
     stage A is kept in flight. */
  const int a_first = !vsbd_proposal_on(st->dev);
  const int depth = vsbd_pipeline_depth(st->dev);
  int issued = k; /* the last frame whose stage A is issued */
  if (!on_device && k + 1 < nframes &&
      vsbd_upload(st->dev, frames + (size_t)(k + 1) * frame_bytes, linesize, (k + 1) % 3) != 0) {
    vs_log_error(md->conf.modName, "GPU upload failed: %s\n", vsbd_error());
    return -1;
  }
  if (a_first && issued + 1 < nframes) {
    if (issue_next_frame(md, st, frames, frame_bytes, linesize, nframes, on_device, issued + 1))
      goto fail;
    issued++;
  }
  for (; k < nframes; k++) {
    int search = 0;
    if (vsb_frame_begin(md, &search) != VS_OK || !search) goto fail;
    vsb_frame_work w;
    VSB_RANGE("vsb host part A");
    vsb_frame_host_a(md, mm, cres, &w);
    VSB_RANGE_END();
    if (vsbd_stage_b_issue(st->dev, w.items, w.fine_pass ? w.nitems : 0) != 0) {
      vs_log_error(md->conf.modName, "GPU stage B failed: %s\n", vsbd_error());
      vsb_frame_discard(&w);
      goto fail;
    }
    while (issued < k + depth && issued + 1 < nframes) {
      if (issue_next_frame(md, st, frames, frame_bytes, linesize, nframes, on_device,
                           issued + 1)) {
        const vsbd_result* unused;
        vsb_frame_discard(&w);
        vsbd_stage_b_collect(st->dev, &unused);
        goto fail;
      }
      issued++;
    }
    const vsbd_result* fres = NULL;
    if (vsbd_stage_b_collect(st->dev, &fres) != 0) {
      vs_log_error(md->conf.modName, "GPU stage B failed: %s\n", vsbd_error());
      vsb_frame_discard(&w);
      goto fail;
    }
    VSB_RANGE("vsb host part B");
    const int nrec = vsb_frame_host_b_records(md, fres, &w, total < out_cap ? rec + total : NULL,
                                              total < out_cap ? out_cap - total : 0);
    VSB_RANGE_END();
    if (nrec < 0) goto fail;
    if (vsb_frame_end(md)) vsbd_commit_prev(st->dev);
    if (counts) counts[k] = nrec;
    total += nrec;
    if (k + 1 < nframes && vsbd_stage_a_next_collect(st->dev, &mm, &cres) != 0) {
      vs_log_error(md->conf.modName, "GPU stage A failed: %s\n", vsbd_error());
      goto fail;
    }
  }
  return total;
fail:
  /* let the stage A's still in flight finish */
  while (vsbd_stage_a_next_collect(st->dev, &mm, &cres) == 0) {
  }
  return -1;
}

/* Many detectors stepped together by one host thread: for each frame, the
   stage A of every detector is enqueued before any is collected, then each
   detector's host part A runs and its fine stage is enqueued, then each fine
   stage is collected and its motions assembled.  The GPU overlaps the
   streams' stages while the host works on the others.  Same results, stream
   by stream, as each detector's own frame loop.  Records are appended frame
   by frame, detector by detector; counts[k*n + s].  Returns the number of
   records, or -1. */
long vsb_detect_multi_impl(VSMotionDetect** mds, int n, const uint8_t* const* clips,
                      const long* frame_bytes, const int* linesizes, int nframes, int on_device,
                      LocalMotion* rec, long out_cap, int* counts) {
  long total = 0;
  if (!mds || n < 1 || !clips || !frame_bytes || !linesizes || nframes < 0) return -1;
  md_state** st = (md_state**)malloc(sizeof(md_state*) * (size_t)n);
  vsb_frame_work* w = (vsb_frame_work*)malloc(sizeof(vsb_frame_work) * (size_t)n);
  int* search = (int*)malloc(sizeof(int) * (size_t)n);
  int* ok = (int*)calloc((size_t)n, sizeof(int));
  long rc = -1;
  if (!st || !w || !search || !ok) goto done;
  for (int s = 0; s < n; s++)
    if (!(st[s] = state_find(mds[s]))) goto done;
  for (int k = 0; k < nframes; k++) {
    for (int s = 0; s < n; s++) {
      const uint8_t* src = clips[s] + (size_t)k * frame_bytes[s];
      if (vsb_frame_begin(mds[s], &search[s]) != VS_OK ||
          vsbd_stage_a_issue(st[s]->dev, on_device ? NULL : src, linesizes[s],
                             on_device ? src : NULL, linesizes[s], search[s]) != 0) {
        vs_log_error(mds[s]->conf.modName, "GPU stage A failed: %s\n", vsbd_error());
        goto done;
      }
    }
    for (int s = 0; s < n; s++) {
      const uint8_t* mm = NULL;
      const vsbd_result* cres = NULL;
      ok[s] = 0;
      if (vsbd_stage_a_next_collect(st[s]->dev, &mm, &cres) != 0) goto done;
      if (!search[s]) continue;
      vsb_frame_host_a(mds[s], mm, cres, &w[s]);
      ok[s] = 1;
      if (vsbd_stage_b_issue(st[s]->dev, w[s].items, w[s].fine_pass ? w[s].nitems : 0) != 0)
        goto done;
    }
    for (int s = 0; s < n; s++) {
      int nrec = 0;
      if (search[s]) {
        const vsbd_result* fres = NULL;
        if (vsbd_stage_b_collect(st[s]->dev, &fres) != 0) goto done;
        ok[s] = 0;
        nrec = vsb_frame_host_b_records(mds[s], fres, &w[s], total < out_cap ? rec + total : NULL,
                                        total < out_cap ? out_cap - total : 0);
        if (nrec < 0) {
          for (int q = s + 1; q < n; q++)
            if (search[q]) vsbd_stage_b_collect(st[q]->dev, &fres);
          goto done;
        }
      } else {
        LocalMotions lms;
        if (vsb_frame_first(mds[s], &lms) != VS_OK) goto done;
        vs_vector_del(&lms);
      }
      if (vsb_frame_end(mds[s])) vsbd_commit_prev(st[s]->dev);
      if (counts) counts[(size_t)k * n + s] = nrec;
      total += nrec;
    }
  }
  rc = total;
done:
  if (rc < 0 && w && ok)
    for (int s = 0; s < n; s++)
      if (ok[s]) vsb_frame_discard(&w[s]);
  free(st);
  free(w);
  free(search);
  free(ok);
  return rc;
}

int vsMotionDetection(VSMotionDetect* md, LocalMotions* motions, VSFrame* frame) {
  if (!md || !frame || !frame->data[0]) return VS_ERROR;
  md->currorig = *frame;
  return vsb_detect_common(md, motions, frame->data[0], frame->linesize[0], NULL, 0);
}
