/*
 * ref_driver.c -- test infrastructure only (a checker, never the product).
 *
 * Thin C driver over the UNMODIFIED reference library (oracle/_ref/
 * libvidstab_ref.so, compiled from the reference sources by oracle/Makefile).
 * It runs the reference's own public detect API the way a host application
 * does (src/motiondetect.h:121-147: vsMotionDetectInit, then
 * vsMotionDetection once per frame, then vsMotionDetectionCleanup) over a
 * clip held in one buffer, and flattens every frame's LocalMotions into
 * plain 32-byte records so that Python can compare them field by field.
 * It also exposes the reference's leaf kernels (blur passes, SAD, contrast,
 * field search) for unit-level pinning of the oracle restatement, and the
 * second pass (local motions -> per-frame transforms) over a whole clip.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "motiondetect.h"
#include "motiondetect_internal.h"
#include "localmotion2transform.h"
#include "transform.h"
#include "serialize.h"
#include "boxblur.h"
#include "transformtype_operations.h"
#include "motiondetect_opt.h"

/* not declared in boxblur.h; exported by boxblur.c:190,247 */
void boxblur_hori_C(unsigned char* dest, const unsigned char* src,
                    int width, int height, int dest_strive, int src_strive, int size);
void boxblur_vert_C(unsigned char* dest, const unsigned char* src,
                    int width, int height, int dest_strive, int src_strive, int size);

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

int vsref_sizeof_localmotion(void) { return (int)sizeof(LocalMotion); }
int vsref_sizeof_motiondetect(void) { return (int)sizeof(VSMotionDetect); }

static void quiet_log(void) { vs_log_level = 0; }

/* Runs detect over `nframes` frames.  Frame k's plane 0 starts at
 * frames + k*frame_bytes with the given linesize (bytes); for planar formats
 * the chroma planes point at a shared grey buffer (the planar detect path never
 * reads them, src/boxblur.c:154 BoxBlurNoColor).  Records of frame k are
 * appended to `out` (capacity out_cap records); counts[k] receives their
 * number (or -1 on error).  Returns the total number of records, or -1.
 * *elapsed receives the wall time of the vsMotionDetection loop alone.
 * If trf_path is not NULL the .trf file is written as the ffmpeg filter does
 * (vsPrepareFile once, vsWriteToFile after every frame). */
long vsref_detect_clip(int width, int height, int pformat,
                       const uint8_t* frames, long frame_bytes, int linesize,
                       int nframes, int stepSize, int accuracy, int shakiness,
                       double mincontrast, int tripod, int show, int numThreads,
                       int serializationMode, const char* trf_path,
                       LocalMotion* out, long out_cap, int* counts, double* elapsed,
                       uint8_t* show_out) {
  VSFrameInfo fi;
  VSMotionDetect md;
  VSMotionDetectConfig conf;
  long total = 0;
  int k;
  uint8_t* chroma = NULL;
  uint8_t* work = NULL;
  FILE* trf = NULL;
  double t_acc = 0.0;

  quiet_log();
  if (!vsFrameInfoInit(&fi, width, height, (VSPixelFormat)pformat)) return -1;
  conf = vsMotionDetectGetDefaultConfig("vsref");
  conf.stepSize = stepSize;
  conf.accuracy = accuracy;
  conf.shakiness = shakiness;
  conf.contrastThreshold = mincontrast;
  conf.virtualTripod = tripod;
  conf.show = show;
  conf.numThreads = numThreads;
  memset(&md, 0, sizeof(md));
  md.serializationMode = serializationMode;
  if (vsMotionDetectInit(&md, &conf, &fi) != VS_OK) return -1;
  if (trf_path) {
    trf = fopen(trf_path, "wb");
    if (!trf || vsPrepareFile(&md, trf) != VS_OK) {
      if (trf) fclose(trf);
      vsMotionDetectionCleanup(&md);
      return -1;
    }
  }
  chroma = (uint8_t*)malloc((size_t)width * height + 64);
  memset(chroma, 128, (size_t)width * height + 64);
  if (show) work = (uint8_t*)malloc((size_t)frame_bytes);

  for (k = 0; k < nframes; k++) {
    VSFrame f;
    LocalMotions lms;
    int n, i;
    const uint8_t* src = frames + (size_t)k * frame_bytes;
    memset(&f, 0, sizeof(f));
    if (show) { memcpy(work, src, (size_t)frame_bytes); src = work; }
    f.data[0] = (uint8_t*)src;
    f.linesize[0] = linesize;
    if (pformat < PF_PACKED) {
      int p;
      for (p = 1; p < fi.planes; p++) {
        f.data[p] = chroma;
        f.linesize[p] = width >> vsGetPlaneWidthSubS(&fi, p);
      }
    }
    double t0 = now_s();
    if (vsMotionDetection(&md, &lms, &f) != VS_OK) { counts[k] = -1; total = -1; break; }
    t_acc += now_s() - t0;
    n = vs_vector_size(&lms);
    counts[k] = n;
    for (i = 0; i < n; i++) {
      if (out && total < out_cap) out[total] = *LMGet(&lms, i);
      total++;
    }
    if (trf) vsWriteToFile(&md, trf, &lms);
    if (show && show_out) memcpy(show_out + (size_t)k * frame_bytes, work, (size_t)frame_bytes);
    vs_vector_del(&lms);
  }
  if (trf) fclose(trf);
  vsMotionDetectionCleanup(&md);
  free(chroma);
  free(work);
  if (elapsed) *elapsed = t_acc;
  return total;
}

/* the reference's luma prefilter: boxblurPlanar with BoxBlurNoColor on a GRAY8
   frame (src/boxblur.c:104-161), linesizes in bytes */
void vsref_boxblur_plane(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                         int width, int height, int size) {
  VSFrameInfo fi;
  VSFrame d, s, tmp;
  vsFrameInfoInit(&fi, width, height, PF_GRAY8);
  vsFrameNull(&d); vsFrameNull(&s);
  d.data[0] = dst; d.linesize[0] = dst_ls;
  s.data[0] = (uint8_t*)src; s.linesize[0] = src_ls;
  vsFrameAllocate(&tmp, &fi);
  boxblurPlanar(&d, &s, &tmp, &fi, (unsigned)size, BoxBlurNoColor);
  vsFrameFree(&tmp);
}

void vsref_boxblur_hori(uint8_t* dst, const uint8_t* src, int w, int h, int dst_ls,
                        int src_ls, int size) {
  boxblur_hori_C(dst, src, w, h, dst_ls, src_ls, size);
}

void vsref_boxblur_vert(uint8_t* dst, const uint8_t* src, int w, int h, int dst_ls,
                        int src_ls, int size) {
  boxblur_vert_C(dst, src, w, h, dst_ls, src_ls, size);
}

/* plain C SAD of the reference (src/motiondetect.c:971-996) */
unsigned int vsref_sad(const uint8_t* I1, const uint8_t* I2, int ls1, int ls2, int height,
                       int fx, int fy, int size, int dx, int dy, unsigned int threshold) {
  Field f;
  f.x = (int16_t)fx; f.y = (int16_t)fy; f.size = (int16_t)size;
  return compareSubImg_thr((unsigned char*)I1, (unsigned char*)I2, &f, ls1, ls2, height,
                           1, dx, dy, threshold);
}

/* the dispatched (SIMD) SAD the reference detect actually calls */
unsigned int vsref_sad_dispatch(const uint8_t* I1, const uint8_t* I2, int ls1, int ls2,
                                int height, int fx, int fy, int size, int dx, int dy,
                                unsigned int threshold) {
  Field f;
  vs_simd_init();
  f.x = (int16_t)fx; f.y = (int16_t)fy; f.size = (int16_t)size;
  return compareSubImg((unsigned char*)I1, (unsigned char*)I2, &f, ls1, ls2, height,
                       1, dx, dy, threshold);
}

double vsref_contrast(const uint8_t* I, int ls, int height, int fx, int fy, int size) {
  Field f;
  f.x = (int16_t)fx; f.y = (int16_t)fy; f.size = (int16_t)size;
  return contrastSubImg((unsigned char*)I, &f, ls, height, 1);
}

const char* vsref_simd_name(void) { return vs_simd_active_name(); }

/* The field geometry vsMotionDetectInit lays out (src/motiondetect.c:132-158,
   :314-358).  xy receives 2*n int16 pairs (coarse fields then fine fields);
   info receives {coarse n, size, maxShift, stepSize, maxFields, rows,
                  fine n, size, maxShift, stepSize, maxFields, rows}. */
int vsref_field_layout(int width, int height, int stepSize, int accuracy, int shakiness,
                       int16_t* xy, int cap, int* info) {
  VSFrameInfo fi;
  VSMotionDetect md;
  VSMotionDetectConfig conf;
  int i, n = 0;
  quiet_log();
  if (!vsFrameInfoInit(&fi, width, height, PF_GRAY8)) return -1;
  conf = vsMotionDetectGetDefaultConfig("vsref");
  conf.stepSize = stepSize; conf.accuracy = accuracy; conf.shakiness = shakiness;
  memset(&md, 0, sizeof(md));
  if (vsMotionDetectInit(&md, &conf, &fi) != VS_OK) return -1;
  VSMotionDetectFields* fs[2] = { &md.fieldscoarse, &md.fieldsfine };
  for (int s = 0; s < 2; s++) {
    info[6 * s + 0] = fs[s]->fieldNum;
    info[6 * s + 1] = fs[s]->fieldSize;
    info[6 * s + 2] = fs[s]->maxShift;
    info[6 * s + 3] = fs[s]->stepSize;
    info[6 * s + 4] = fs[s]->maxFields;
    info[6 * s + 5] = fs[s]->fieldRows;
    for (i = 0; i < fs[s]->fieldNum; i++) {
      if (n < cap) { xy[2 * n] = fs[s]->fields[i].x; xy[2 * n + 1] = fs[s]->fields[i].y; }
      n++;
    }
  }
  vsMotionDetectionCleanup(&md);
  return n;
}

/* The reference's per-field search (calcFieldTransPlanar,
   src/motiondetect.c:439-586) on caller-provided blurred planes, without an
   offset: returns match (or -1 when rejected) and the shift in *vx,*vy. */
double vsref_field_search(const uint8_t* curr, const uint8_t* prev, int width, int height,
                          int fx, int fy, int size, int maxShift, int stepSize,
                          int* vx, int* vy) {
  VSFrameInfo fi;
  VSMotionDetect md;
  VSMotionDetectFields fs;
  Field f;
  LocalMotion lm;
  quiet_log();
  vsFrameInfoInit(&fi, width, height, PF_GRAY8);
  memset(&md, 0, sizeof(md));
  memset(&fs, 0, sizeof(fs));
  md.fi = fi;
  md.curr.data[0] = (uint8_t*)curr; md.curr.linesize[0] = width;
  md.prev.data[0] = (uint8_t*)prev; md.prev.linesize[0] = width;
  fs.maxShift = maxShift; fs.stepSize = stepSize; fs.useOffset = 0;
  f.x = (int16_t)fx; f.y = (int16_t)fy; f.size = (int16_t)size;
  vs_simd_init();
  lm = calcFieldTransPlanar(&md, &fs, &f, 0);
  *vx = lm.v.x; *vy = lm.v.y;
  return lm.match;
}

/* vsSimpleMotionsToTransform over flat records
   (src/localmotion2transform.c:352-402); out = {x, y, alpha, zoom} */
void vsref_simple_transform(int width, int height, const LocalMotion* lms, int n, double* out) {
  VSFrameInfo fi;
  LocalMotions v;
  int i;
  quiet_log();
  vsFrameInfoInit(&fi, width, height, PF_GRAY8);
  vs_vector_init(&v, n > 0 ? n : 1);
  for (i = 0; i < n; i++) vs_vector_append_dup(&v, (void*)&lms[i], sizeof(LocalMotion));
  VSTransform t = vsSimpleMotionsToTransform(fi, "vsref", &v);
  out[0] = t.x; out[1] = t.y; out[2] = t.alpha; out[3] = t.zoom;
  vs_vector_del(&v);
}

/* the fine-search offset of one field for transform t4 = {x, y, alpha, zoom}:
   prepare_transform + transform_vec - position, as fieldSearchOffset does
   (src/motiondetect.c:418-427) */
void vsref_field_offset(const double* t4, int width, int height, int fx, int fy,
                        int16_t* ox, int16_t* oy) {
  VSFrameInfo fi;
  VSTransform t = null_transform();
  vsFrameInfoInit(&fi, width, height, PF_GRAY8);
  t.x = t4[0]; t.y = t4[1]; t.alpha = t4[2]; t.zoom = t4[3];
  PreparedTransform pt = prepare_transform(&t, &fi);
  Vec pos = { (int16_t)fx, (int16_t)fy };
  Vec off = sub_vec(transform_vec(&pt, &pos), pos);
  *ox = off.x;
  *oy = off.y;
}

double vsref_cleanmean(double* ds, int len, double* mn, double* mx) {
  return cleanmean(ds, len, mn, mx);
}

/* contrast of a packed field as the reference's packed detect computes it
   (contrastSubImgPacked, src/motiondetect.c:370-377) */
double vsref_contrast_packed(const uint8_t* I, int linesize, int width, int height, int bpp,
                             int fx, int fy, int size) {
  VSMotionDetect md;
  Field f;
  memset(&md, 0, sizeof(md));
  vsFrameInfoInit(&md.fi, width, height, bpp == 4 ? PF_RGBA : PF_RGB24);
  md.curr.data[0] = (uint8_t*)I;
  md.curr.linesize[0] = linesize;
  f.x = (int16_t)fx; f.y = (int16_t)fy; f.size = (int16_t)size;
  return contrastSubImgPacked(&md, &f);
}

/* exported by src/localmotion2transform.c:140 but not declared in its header */
double calcTransformQuality(VSArray params, void* dat);

/* ---- second pass: local motions -> one transform per frame ---------------
 * Runs the reference's vsLocalmotions2Transforms (src/localmotion2transform.c:
 * 40-121) over a clip whose frame k holds the records recs[first[k] ..
 * first[k+1]).  The VSTransformData is the reference's own default transform
 * configuration (src/transform.c vsTransformGetDefaultConfig) with the lens
 * estimate switched off and fov / smoothZoom / simpleMotionCalculation set
 * from the arguments.  *elapsed receives the wall time of the call alone. */
int vsref_motions_to_transforms(int width, int height, const LocalMotion* recs,
                                const long* first, int nframes, double fov, int smoothZoom,
                                int simple, VSTransform* out, double* elapsed) {
  VSTransformData td;
  VSManyLocalMotions mlms;
  VSTransformations trans;
  int k, rc;
  quiet_log();
  memset(&td, 0, sizeof(td));
  if (!vsFrameInfoInit(&td.fiSrc, width, height, PF_YUV420P)) return -1;
  td.fiDest = td.fiSrc;
  td.conf = vsTransformGetDefaultConfig("vsref");
  td.conf.estimateLensDistortion = 0;
  td.conf.fov = fov;
  td.conf.smoothZoom = smoothZoom;
  td.conf.simpleMotionCalculation = simple;
  vs_vector_init(&mlms, nframes > 0 ? nframes : 1);
  for (k = 0; k < nframes; k++) {
    LocalMotions lms;
    long i;
    vs_vector_init(&lms, (int)(first[k + 1] - first[k]) + 1);
    for (i = first[k]; i < first[k + 1]; i++)
      vs_vector_append_dup(&lms, (void*)&recs[i], sizeof(LocalMotion));
    vs_vector_append_dup(&mlms, &lms, sizeof(LocalMotions));
  }
  vsTransformationsInit(&trans);
  double t0 = now_s();
  rc = vsLocalmotions2Transforms(&td, &mlms, &trans);
  if (elapsed) *elapsed = now_s() - t0;
  for (k = 0; rc == VS_OK && k < trans.len && k < nframes; k++) out[k] = trans.ts[k];
  vsTransformationsCleanup(&trans);
  for (k = 0; k < vs_vector_size(&mlms); k++) vs_vector_del(VSMLMGet(&mlms, k));
  vs_vector_del(&mlms);
  return rc == VS_OK ? 0 : -1;
}

/* calcTransformQuality (src/localmotion2transform.c:140-172) on one frame's
 * records with the given mask / missmatch array (updated in place). */
double vsref_transform_quality(int width, int height, const LocalMotion* recs, int n,
                               const double* params4, double fov, double* missmatches) {
  VSTransformData td;
  LocalMotions lms;
  struct { VSTransformData* td; const LocalMotions* motions; VSArray mm; } dat;
  VSArray p;
  double r;
  int i;
  memset(&td, 0, sizeof(td));
  vsFrameInfoInit(&td.fiSrc, width, height, PF_YUV420P);
  td.conf = vsTransformGetDefaultConfig("vsref");
  td.conf.fov = fov;
  vs_vector_init(&lms, n + 1);
  for (i = 0; i < n; i++) vs_vector_append_dup(&lms, (void*)&recs[i], sizeof(LocalMotion));
  dat.td = &td;
  dat.motions = &lms;
  dat.mm.dat = missmatches;
  dat.mm.len = n;
  p = vs_array((double*)params4, 4);
  r = calcTransformQuality(p, &dat);
  vs_array_free(p);
  vs_vector_del(&lms);
  return r;
}

/* layout of the structures the second pass reads through a caller's pointer */
int vsref_transform_layout(long* out, int cap) {
  long v[] = {
    (long)sizeof(VSTransformData), (long)sizeof(VSTransformConfig),
    (long)sizeof(VSTransformations),
    (long)offsetof(VSTransformData, fiSrc), (long)offsetof(VSTransformData, conf),
    (long)offsetof(VSTransformData, initialized),
    (long)offsetof(VSTransformConfig, modName), (long)offsetof(VSTransformConfig, verbose),
    (long)offsetof(VSTransformConfig, simpleMotionCalculation),
    (long)offsetof(VSTransformConfig, storeTransforms),
    (long)offsetof(VSTransformConfig, smoothZoom),
    (long)offsetof(VSTransformConfig, estimateLensDistortion),
    (long)offsetof(VSTransformConfig, lensK), (long)offsetof(VSTransformConfig, fov),
    (long)offsetof(VSTransformations, ts), (long)offsetof(VSTransformations, len),
  };
  int n = (int)(sizeof(v) / sizeof(v[0])), i;
  for (i = 0; i < n && i < cap; i++) out[i] = v[i];
  return n;
}

/* The transform pass's input path as a host application takes it: the
 * reference's vsReadLocalMotionsFile on a .trf file, then
 * vsLocalmotions2Transforms (lens estimate off; storeTransforms writes
 * global_motions.trf into the working directory).  Returns the number of
 * frames (their transforms in out[0 .. min(n, cap))) or -1. */
int vsref_trf_to_transforms(const char* trf_path, int width, int height, double fov,
                            int smoothZoom, int store, VSTransform* out, int cap) {
  VSTransformData td;
  VSManyLocalMotions mlms;
  VSTransformations trans;
  FILE* f;
  int k, n, rc;
  quiet_log();
  f = fopen(trf_path, "rb");
  if (!f) return -1;
  memset(&mlms, 0, sizeof(mlms));
  rc = vsReadLocalMotionsFile(f, &mlms);
  fclose(f);
  if (rc != VS_OK) return -1;
  memset(&td, 0, sizeof(td));
  vsFrameInfoInit(&td.fiSrc, width, height, PF_YUV420P);
  td.fiDest = td.fiSrc;
  td.conf = vsTransformGetDefaultConfig("vsref");
  td.conf.estimateLensDistortion = 0;
  td.conf.fov = fov;
  td.conf.smoothZoom = smoothZoom;
  td.conf.storeTransforms = store;
  vsTransformationsInit(&trans);
  rc = vsLocalmotions2Transforms(&td, &mlms, &trans);
  n = rc == VS_OK ? trans.len : -1;
  for (k = 0; k < n && k < cap; k++) out[k] = trans.ts[k];
  vsTransformationsCleanup(&trans);
  for (k = 0; k < vs_vector_size(&mlms); k++) vs_vector_del(VSMLMGet(&mlms, k));
  vs_vector_del(&mlms);
  return n;
}
