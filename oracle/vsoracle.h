/*
 * vsoracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of vid.stab's motion-detection pass
 * (vsMotionDetectInit / vsMotionDetection, src/motiondetect.c:83-305 of the
 * reference) used as the checker for the CUDA product path.  Only tests/,
 * the smoke check and bench.py's CPU-baseline leg may load it; the product
 * library never links or calls it.
 *
 * Parity of this restatement is pinned against the unmodified reference
 * library compiled from its own sources (oracle/_ref, see oracle/Makefile)
 * by tests/test_oracle_pin.py and by the committed fixtures in tests/golden/.
 */
#ifndef VSORACLE_H
#define VSORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same memory layout as the reference's LocalMotion (src/transformtype.h:64-69)
   on x86-64: five int16 values, padding, two doubles (32 bytes). */
typedef struct {
  int16_t vx, vy;
  int16_t fx, fy, fsize;
  int16_t pad_;
  double contrast;
  double match;
} orc_lm;

/* pixel formats, numbered as src/frameinfo.h:34-48 */
enum { ORC_PF_GRAY8 = 0, ORC_PF_YUV420P = 1, ORC_PF_YUVA420P = 7, ORC_PF_PACKED = 8,
       ORC_PF_RGB24 = 9, ORC_PF_BGR24 = 10, ORC_PF_RGBA = 11, ORC_PF_NUMBER = 12 };

/* ---- leaf operations ---------------------------------------------------- */

/* effective odd box size boxblurPlanar uses for a requested size
   (src/boxblur.c:109-122); returns <2 when the reference copies instead */
int orc_blur_size(int requested, int width, int height);

/* one separable box pass: clamped-window sum divided by size, truncated to
   8 bits (src/boxblur.c:190-238 horizontal, :247-332 vertical) */
void orc_blur_hori(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int size);
void orc_blur_vert(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int size);

/* the luma prefilter of one frame: size = orc_blur_size(stepSize); horizontal
   then vertical pass through an 8-bit intermediate (src/boxblur.c:104-161) */
void orc_blur_luma(uint8_t* dst, int dst_ls, const uint8_t* src, int src_ls,
                   int width, int height, int stepSize);

/* full sum of absolute differences of a size x size field (bpp bytes per
   pixel) at centre (fx,fy) of I1 against I2 displaced by (dx,dy)
   (src/motiondetect.c:971-996 without the early exit) */
uint32_t orc_sad(const uint8_t* I1, int ls1, const uint8_t* I2, int ls2,
                 int fx, int fy, int size, int bpp, int dx, int dy);

/* 8-bit minimum and maximum over the field of one channel
   (src/motiondetect.c:389-407) */
void orc_minmax(const uint8_t* I, int ls, int fx, int fy, int size, int bpp,
                uint8_t* mn, uint8_t* mx);
double orc_contrast_from_minmax(int mn, int mx);

/* lattice points of the outgoing spiral, in visiting order
   (src/motiondetect.c:465-518); returns the count, writes up to cap points */
int orc_spiral(int maxShift, int step, int* di, int* dj, int cap);

/* planar field search (src/motiondetect.c:439-586) around offset (ox,oy):
   returns 1 and the best shift (relative to the offset) and its SAD, or 0 if
   the shift is rejected by the final range test */
int orc_search_planar(const uint8_t* curr, int ls_c, const uint8_t* prev, int ls_p,
                      int fx, int fy, int size, int maxShift, int stepSize,
                      int ox, int oy, int* tx, int* ty, uint32_t* minerror);

/* packed field search (src/motiondetect.c:591-660) */
int orc_search_packed(const uint8_t* curr, int ls_c, const uint8_t* prev, int ls_p,
                      int fx, int fy, int size, int bpp, int maxShift, int stepSize,
                      int ox, int oy, int* tx, int* ty, uint32_t* minerror);

/* ---- field geometry (src/motiondetect.c:132-158, :314-358) -------------- */
typedef struct {
  int num, size, maxShift, stepSize, maxFields, rows;
  double contrastThreshold;
  int16_t* x;
  int16_t* y;
} orc_fields;

/* ---- the whole pass ----------------------------------------------------- */
typedef struct orc_md orc_md;

/* vsMotionDetectInit (src/motiondetect.c:83-165); NULL on unsupported input.
   shakiness/accuracy/stepSize are clamped as the reference does. */
orc_md* orc_md_new(int width, int height, int pformat, int stepSize, int accuracy,
                   int shakiness, double mincontrast, int tripod);
/* read back the geometry: which = 0 coarse, 1 fine */
const orc_fields* orc_md_fields(const orc_md* md, int which);
/* vsMotionDetection (src/motiondetect.c:191-305) on plane 0 of one frame.
   Writes up to cap records, returns their number (<0 on error). */
int orc_md_frame(orc_md* md, const uint8_t* plane0, int linesize, orc_lm* out, int cap);
/* the blurred current frame of the last call (W x H, linesize W*bpp) */
const uint8_t* orc_md_curr(const orc_md* md);
int orc_md_frame_num(const orc_md* md);
void orc_md_free(orc_md* md);

/* vsSimpleMotionsToTransform (src/localmotion2transform.c:352-402); out =
   {x, y, alpha, zoom} */
void orc_simple_transform(int width, int height, const orc_lm* lms, int n, double* out);

/* fine-search offset of a field for the transform {x, y, alpha, zoom}
   (src/motiondetect.c:418-427 with src/transformtype.c:158-209) */
void orc_offset(const double* t4, int W, int H, int fx, int fy, int16_t* ox, int16_t* oy);

/* cleanmean of src/transformtype.c:445-461 (sorts ds) */
double orc_cleanmean(double* ds, int len, double* mn, double* mx);

#ifdef __cplusplus
}
#endif
#endif
