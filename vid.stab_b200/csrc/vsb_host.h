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

/* device context of an initialised detector (NULL if none) */
vsbd_ctx* vsb_md_device(const VSMotionDetect* md);

#ifdef __cplusplus
}
#endif
#endif
