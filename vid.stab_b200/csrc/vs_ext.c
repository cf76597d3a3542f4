/*
 * vs_ext.c -- entry points without a counterpart in the reference
 * (declared in vidstab_b200_ext.h).
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "vidstab_b200.h"
#include "vsb_host.h"

const char* vsb_last_error(void) { return vsbd_error(); }

int vsb_device_count(void) { return vsbd_device_count(); }

int vsb_sizeof(const char* t) {
  if (!t) return -1;
  if (!strcmp(t, "VSMotionDetect")) return (int)sizeof(VSMotionDetect);
  if (!strcmp(t, "VSMotionDetectConfig")) return (int)sizeof(VSMotionDetectConfig);
  if (!strcmp(t, "VSMotionDetectFields")) return (int)sizeof(VSMotionDetectFields);
  if (!strcmp(t, "VSFrameInfo")) return (int)sizeof(VSFrameInfo);
  if (!strcmp(t, "VSFrame")) return (int)sizeof(VSFrame);
  if (!strcmp(t, "VSTransform")) return (int)sizeof(VSTransform);
  if (!strcmp(t, "LocalMotion")) return (int)sizeof(LocalMotion);
  if (!strcmp(t, "VSVector")) return (int)sizeof(VSVector);
  if (!strcmp(t, "Field")) return (int)sizeof(Field);
  if (!strcmp(t, "PreparedTransform")) return (int)sizeof(PreparedTransform);
  if (!strcmp(t, "VSTransformData")) return (int)sizeof(VSTransformData);
  if (!strcmp(t, "VSTransformConfig")) return (int)sizeof(VSTransformConfig);
  if (!strcmp(t, "VSTransformations")) return (int)sizeof(VSTransformations);
  return -1;
}

int vsb_transform_layout(long* out, int cap) {
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

int vsb_motion_detection_device(VSMotionDetect* md, LocalMotions* motions, const uint8_t* d_plane0,
                                int pitch) {
  if (!md || !d_plane0) return VS_ERROR;
  VSFrame none;
  vsFrameNull(&none);
  md->currorig = none;
  return vsb_detect_common(md, motions, NULL, 0, d_plane0, pitch);
}

long vsb_launch_count(const VSMotionDetect* md) { return vsbd_launches(vsb_md_device(md)); }

int vsb_search_tiling(const VSMotionDetect* md, int fine, int* desc) {
  return vsbd_search_tiling(vsb_md_device(md), fine, desc) == 0 ? VS_OK : VS_ERROR;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

long vsb_detect_clip(int width, int height, int pformat, const uint8_t* frames, long frame_bytes,
                     int linesize, int nframes, int on_device, int stepSize, int accuracy,
                     int shakiness, double mincontrast, int tripod, int show,
                     int serializationMode, const char* trf_path, void* out, long out_cap,
                     int* counts, double* elapsed, uint8_t* show_out) {
  VSFrameInfo fi;
  VSMotionDetect md;
  VSMotionDetectConfig conf;
  LocalMotion* rec = (LocalMotion*)out;
  long total = 0;
  FILE* trf = NULL;
  uint8_t* work = NULL;
  uint8_t* chroma = NULL;
  double t_acc = 0.0;
  if (!vsFrameInfoInit(&fi, width, height, (VSPixelFormat)pformat)) return -1;
  conf = vsMotionDetectGetDefaultConfig("vsb");
  conf.stepSize = stepSize;
  conf.accuracy = accuracy;
  conf.shakiness = shakiness;
  conf.contrastThreshold = mincontrast;
  conf.virtualTripod = tripod;
  conf.show = on_device ? 0 : show;
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
  if (conf.show) work = (uint8_t*)malloc((size_t)frame_bytes);
  chroma = (uint8_t*)calloc((size_t)width * height + 64, 1);
  for (int k = 0; k < nframes; k++) {
    LocalMotions lms;
    const uint8_t* src = frames + (size_t)k * frame_bytes;
    int rc;
    double t0;
    if (on_device) {
      t0 = now_s();
      rc = vsb_motion_detection_device(&md, &lms, src, linesize);
    } else {
      VSFrame f;
      memset(&f, 0, sizeof(f));
      if (work) {
        memcpy(work, src, (size_t)frame_bytes);
        src = work;
      }
      f.data[0] = (uint8_t*)src;
      f.linesize[0] = linesize;
      if (pformat < PF_PACKED)
        for (int p = 1; p < fi.planes; p++) {
          f.data[p] = chroma;
          f.linesize[p] = width >> vsGetPlaneWidthSubS(&fi, p);
        }
      t0 = now_s();
      rc = vsMotionDetection(&md, &lms, &f);
    }
    if (rc != VS_OK) {
      counts[k] = -1;
      total = -1;
      break;
    }
    t_acc += now_s() - t0;
    int n = vs_vector_size(&lms);
    counts[k] = n;
    for (int i = 0; i < n; i++) {
      if (rec && total < out_cap) rec[total] = *LMGet(&lms, i);
      total++;
    }
    if (trf) vsWriteToFile(&md, trf, &lms);
    if (work && show_out) memcpy(show_out + (size_t)k * frame_bytes, work, (size_t)frame_bytes);
    vs_vector_del(&lms);
  }
  if (trf) fclose(trf);
  vsMotionDetectionCleanup(&md);
  free(work);
  free(chroma);
  if (elapsed) *elapsed = t_acc;
  return total;
}

/* frames through the per-frame entry points, one call per frame */
static long run_per_frame(VSMotionDetect* md, const uint8_t* frames, long frame_bytes,
                          int linesize, int nframes, int on_device, LocalMotion* rec,
                          long out_cap, int* counts) {
  long total = 0;
  for (int k = 0; k < nframes; k++) {
    LocalMotions lms;
    const uint8_t* src = frames + (size_t)k * frame_bytes;
    int rc;
    if (on_device) {
      rc = vsb_motion_detection_device(md, &lms, src, linesize);
    } else {
      /* only plane 0 is read; the other plane pointers stay valid memory */
      VSFrame f;
      memset(&f, 0, sizeof(f));
      for (int p = 0; p < 4; p++) {
        f.data[p] = (uint8_t*)src;
        f.linesize[p] = linesize;
      }
      rc = vsMotionDetection(md, &lms, &f);
    }
    if (rc != VS_OK) {
      if (counts) counts[k] = -1;
      return -1;
    }
    int n = vs_vector_size(&lms);
    if (counts) counts[k] = n;
    for (int i = 0; i < n; i++) {
      if (rec && total < out_cap) rec[total] = *LMGet(&lms, i);
      total++;
    }
    vs_vector_del(&lms);
  }
  return total;
}

long vsb_detect_run(VSMotionDetect* md, const uint8_t* frames, long frame_bytes, int linesize,
                    int nframes, int on_device, void* out, long out_cap, int* counts) {
  if (!md || !frames || nframes < 0) return -1;
  if (nframes > 1 && vsb_can_overlap(md))
    return vsb_detect_run_overlapped(md, frames, frame_bytes, linesize, nframes, on_device,
                                     (LocalMotion*)out, out_cap, counts);
  return run_per_frame(md, frames, frame_bytes, linesize, nframes, on_device, (LocalMotion*)out,
                       out_cap, counts);
}

long vsb_detect_frames(VSMotionDetect* md, const uint8_t* frames, long frame_bytes, int linesize,
                       int nframes, int on_device, void* out, long out_cap, int* counts) {
  if (!md || !frames || nframes < 0) return -1;
  return run_per_frame(md, frames, frame_bytes, linesize, nframes, on_device, (LocalMotion*)out,
                       out_cap, counts);
}

long vsb_detect_multi(VSMotionDetect** mds, int n, const uint8_t* const* clips,
                      const long* frame_bytes, const int* linesizes, int nframes, int on_device,
                      void* out, long out_cap, int* counts) {
  return vsb_detect_multi_impl(mds, n, clips, frame_bytes, linesizes, nframes, on_device,
                               (LocalMotion*)out, out_cap, counts);
}

int vsb_boxblur_host(uint8_t* dst, const uint8_t* src, int width, int height, int size) {
  return vsbd_blur_host(dst, src, width, height, size) == 0 ? VS_OK : VS_ERROR;
}

int vsb_boxblur_host_tile(uint8_t* dst, const uint8_t* src, int width, int height, int size,
                          int shape) {
  return vsbd_blur_host_shape(dst, src, width, height, size, shape) == 0 ? VS_OK : VS_ERROR;
}

int vsb_blur_tiling(const VSMotionDetect* md, int* desc) {
  return vsbd_blur_tiling(vsb_md_device(md), desc) == 0 ? VS_OK : VS_ERROR;
}

int vsb_field_minmax_host(const uint8_t* img, int width, int height, int bpp, int channels,
                          const int16_t* x, const int16_t* y, int n, int size, uint8_t* out) {
  return vsbd_minmax_host(img, width, height, bpp, channels, x, y, n, size, out) == 0 ? VS_OK
                                                                                       : VS_ERROR;
}

int vsb_field_search_host(const uint8_t* curr, const uint8_t* prev, int width, int height,
                          int size, int maxShift, int stepSize, int packed_bpp, const int16_t* x,
                          const int16_t* y, const int16_t* ox, const int16_t* oy, int n, int tiles,
                          uint32_t* sad, int16_t* tx, int16_t* ty, int32_t* ok) {
  vsbd_geom g;
  int32_t* order = NULL;
  int planar = packed_bpp <= 0;
  if (vsb_build_geom(&g, &order, size, planar ? 1 : packed_bpp, maxShift, stepSize, planar) != 0)
    return VS_ERROR;
  vsbd_item* items = (vsbd_item*)malloc(sizeof(vsbd_item) * (size_t)(n > 0 ? n : 1));
  vsbd_result* res = (vsbd_result*)malloc(sizeof(vsbd_result) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    items[i].x = x[i];
    items[i].y = y[i];
    items[i].ox = ox ? ox[i] : 0;
    items[i].oy = oy ? oy[i] : 0;
  }
  int rc = n > 0 ? vsbd_search_host(curr, prev, width, height, &g, items, n, tiles, res) : 0;
  for (int i = 0; rc == 0 && i < n; i++) {
    sad[i] = res[i].sad;
    tx[i] = res[i].tx;
    ty[i] = res[i].ty;
    ok[i] = res[i].ok;
  }
  free(items);
  free(res);
  free(order);
  return rc == 0 ? VS_OK : VS_ERROR;
}

int vsb_set_kernel_timing(VSMotionDetect* md, int on) {
  return vsbd_set_timing(vsb_md_device(md), on) == 0 ? VS_OK : VS_ERROR;
}

int vsb_kernel_times(const VSMotionDetect* md, double* ms, long* count) {
  return vsbd_kernel_times(vsb_md_device(md), ms, count) == 0 ? VS_OK : VS_ERROR;
}

int vsb_sad_peak(int variant, double* byteops_per_s) {
  return vsbd_sad_peak(variant, byteops_per_s) == 0 ? VS_OK : VS_ERROR;
}

long long vsb_test_device_alloc(int fail_after, int sticky) {
  return vsbd_test_device_alloc(fail_after, sticky);
}

void vsb_counters(long long* launches, long long* h2d_bytes, long long* d2h_bytes) {
  vsbd_counters(launches, h2d_bytes, d2h_bytes);
}

int vsb_field_search_noalloc(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int size,
                             int maxShift, int stepSize, const void* d_fields, int n,
                             void* d_results, void* stream) {
  return vsbd_search_noalloc(d_curr, d_prev, pitch, size, maxShift, stepSize, d_fields, n,
                             d_results, stream) == 0
             ? VS_OK
             : VS_ERROR;
}

int vsb_set_search_mode(VSMotionDetect* md, int pruned) {
  return vsbd_set_search_mode(vsb_md_device(md), pruned) == 0 ? VS_OK : VS_ERROR;
}

void vsb_set_default_search_mode(int pruned) { vsbd_set_default_search_mode(pruned); }
