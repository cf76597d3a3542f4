/*
 * vsb_host.h -- internal declarations shared by the host C files.
 */
#ifndef VSB_HOST_H
#define VSB_HOST_H

#include "vidstab_b200.h"
#include "vsb_device.h"

#ifdef __cplusplus
extern "C" {
#endif

/* a failed allocation through vs_malloc / vs_zalloc / vs_realloc (counted
   per thread), and the count so far */
void vsb_note_oom(void);
int vsb_oom_count(void);

/* effective box size of the luma prefilter for a requested size
   (src/boxblur.c:109-122); < 2 means no blur */
int vsb_blur_size(int requested, int width, int height);

/* (a + b + c) / 3 with the reference build's floating-point flags */
double vsb_mean3(double a, double b, double c);

/* the `show` overlay of src/motiondetect.c:271-286 into md->currorig */
void vsb_draw_motions(VSMotionDetect* md, LocalMotions* coarse, LocalMotions* fine);

/* one frame of the detect pass from host (host != NULL) or device memory */
int vsb_detect_common(VSMotionDetect* md, LocalMotions* motions, const uint8_t* host,
                      int linesize, const uint8_t* dev, int pitch);

/* candidate geometry of a field set (spiral for planar, raster for
   packed); *order_out must be freed by the caller */
int vsb_build_geom(vsbd_geom* g, int32_t** order_out, int size, int bpp, int maxShift, int step,
                   int planar);

/* Field layout and candidate geometry of a detector initialised without
   device state (vsb_md_init with_device = 0): the caller runs the device
   work.  xy: coarse x[nc], coarse y[nc], fine x[nf], fine y[nf]. */
typedef struct {
  vsbd_geom coarse, fine;
  int32_t* order_c;
  int32_t* order_f;
  int16_t* xy;
  int nc, nf, blur;
} vsb_md_layout;

/* vsMotionDetectInit with or without the per-detector device state */
int vsb_md_init(VSMotionDetect* md, const VSMotionDetectConfig* conf, const VSFrameInfo* fi,
                int with_device, vsb_md_layout* lay);
void vsb_md_layout_free(vsb_md_layout* lay);

/* One frame in phases (src/motiondetect.c:191-305), the device stages
   between them run by the caller:
     vsb_frame_begin      checks; *search = 0 for the first frame and the
                          tripod lead-in (vsb_frame_first then)
     [stage A: blur, field min/max, coarse search]
     vsb_frame_host_a     contrasts, selection, coarse motions, the simple
                          model and the fine work list (w->items[0..nitems),
                          valid until the next frame of this detector)
     [stage B, when w->fine_pass: fine search of the work list]
     vsb_frame_host_b     fine motions, mean-match filter, show, result;
                          VS_ERROR (nothing returned, the frame to be
                          dropped) if an allocation failed in either part
     vsb_frame_end        frame count; returns 1 if the current blurred
                          frame becomes the previous one */
typedef struct {
  LocalMotions coarse, fine;
  int fine_pass;
  int nitems;
  const vsbd_item* items;
  int oom0; /* vsb_oom_count() when the frame's host work began */
} vsb_frame_work;
int vsb_frame_begin(VSMotionDetect* md, int* search);
int vsb_frame_host_a(VSMotionDetect* md, const uint8_t* mm, const vsbd_result* cres,
                     vsb_frame_work* w);
int vsb_frame_host_b(VSMotionDetect* md, const vsbd_result* fres, vsb_frame_work* w,
                     LocalMotions* motions);
void vsb_frame_discard(vsb_frame_work* w);
/* vsb_frame_host_b for a frame loop whose output is a record array: the
   frame's motions (coarse, then the kept fine ones) written to rec[0 ..)
   (at most cap of them) without allocating each motion; returns their
   number, or -1 (nothing valid, the frame to be dropped) if an allocation
   failed.  The work's vectors are released either way. */
int vsb_frame_host_b_records(VSMotionDetect* md, const vsbd_result* fres, vsb_frame_work* w,
                             LocalMotion* rec, long cap);
int vsb_frame_first(VSMotionDetect* md, LocalMotions* motions);
int vsb_frame_end(VSMotionDetect* md);

/* whether vsb_detect_run_overlapped may serve this detector (no tripod,
   no overlay, a device configuration whose stages share no scratch) */
int vsb_can_overlap(const VSMotionDetect* md);

/* NVTX ranges around the per-frame stages (header-only NVTX: no cost
   unless a profiler is attached), so a profile of any host program shows
   device stage A, host part A, device stage B and host part B by name */
#include <nvtx3/nvToolsExt.h>
#define VSB_RANGE(name) nvtxRangePushA(name)
#define VSB_RANGE_END() nvtxRangePop()

/* a serialized proposal network ("VSBP" blob) checked and read; radius,
   conf_min (NaN) and match_bound below zero take the blob's values */
typedef struct {
  const void* params; /* the device-order parameters inside the blob */
  float scale, radius, conf_min, match_bound;
} vsb_pnet_settings;
int vsb_pnet_parse(const void* blob, long bytes, double radius, double conf_min,
                   double match_bound, vsb_pnet_settings* out);
long vsb_detect_run_overlapped(VSMotionDetect* md, const uint8_t* frames, long frame_bytes,
                               int linesize, int nframes, int on_device, LocalMotion* rec,
                               long out_cap, int* counts);

long vsb_detect_multi_impl(VSMotionDetect** mds, int n, const uint8_t* const* clips,
                           const long* frame_bytes, const int* linesizes, int nframes,
                           int on_device, LocalMotion* rec, long out_cap, int* counts);

/* adds wall times (device stage A, host A, device stage B, host B) of
   `frames` frames to the profile vsb_host_profile reads; monotonic clock */
void vsb_prof_add(const double* sec, long frames);
double vsb_now_s(void);

/* device context of an initialised detector (NULL if none) */
vsbd_ctx* vsb_md_device(const VSMotionDetect* md);

#ifdef __cplusplus
}
#endif
#endif
