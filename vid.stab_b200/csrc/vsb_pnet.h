/*
 * vsb_pnet.h -- internal interface of the learned search proposal
 * (vsb_pnet.cu) for the detector shim (vsb_device.cu).  C++ only.
 *
 * The proposal network reads, per search item, a 32x32 crop pair of the
 * blurred current and previous planes (2x2 averages of a 64x64 window) and
 * predicts the item's displacement and a confidence.  The narrowed search
 * evaluates only the lattice points around the prediction, then runs the
 * reference's refinement; items whose proposal is not trusted are flagged
 * for the exact full search.
 */
#ifndef VSB_PNET_H
#define VSB_PNET_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "vsb_device.h"
#include "vsb_search.cuh"

/* parameter counts: bf16 weights, then f32 biases (device buffer order) */
#define PN_NW1 1024
#define PN_NW 9216
#define PN_NFC 1536
#define PN_NB16 (PN_NW1 + 3 * PN_NW + PN_NFC)
#define PN_NF32 131
#define PN_F32_OFFSET (PN_NB16 * 2)
#define PN_PARAM_BYTES (PN_F32_OFFSET + PN_NF32 * 4)
/* stored activations of one item for the backward pass (bf16) */
#define PN_ACT_ELEMS (32 * 32 * 32 + 16 * 16 * 32 + 8 * 8 * 32 + 4 * 4 * 32)
/* fp32 gradient work space of one item */
#define PN_WORK_ELEMS (32 * 32 * 32 + 16 * 16 * 32 + 8 * 8 * 32 + 4 * 4 * 32)

/* per-item fallback flags written by the narrowed search */
#define PN_FB_ACCEPT 0
#define PN_FB_FULL 1
#define PN_FB_UNUSED 2

/* settings of the narrowed search */
struct PNSearch {
  float scale;      /* network (dx, dy) units -> pixels */
  float radius;     /* window: lattice points bracketing prediction +- radius, plus one ring */
  float conf_min;   /* confidence logit below which the full search runs */
  unsigned sad_bound; /* refined SAD above which the full search runs */
};

/* network forward for n items: crops taken from the planes (prepared ==
   NULL; items give the centres and offsets) or read from prepared inputs
   [n][32][32][2] bf16; raw outputs out[n][3].  err (device-visible word,
   may be NULL) is raised when the kernel's bounded wait for the tensor
   cores gave up.  Returns launches (1) or -1. */
int vsbpn_infer(const void* d_params, const uint8_t* curr, const uint8_t* prev, int pitch, int W,
                int H, const vsbd_item* items, const void* prepared, int n, float* out,
                unsigned* err, cudaStream_t st);

/* narrowed search of n items of field set g: results into res, flags into
   fb (PN_FB_*); skip (may be NULL) marks items never used.  Items that fall
   back are appended to fb_list (*fb_count, which the caller zeroes).  With
   prior != NULL the proposal is prior[item] + the network's prediction.
   Returns launches or -1. */
int vsbpn_narrow(const DGeom& g, const uint8_t* curr, const uint8_t* prev, int pitch,
                 const vsbd_item* items, int n, const float* pout, const short2* prior,
                 const PNSearch& ps, const uint8_t* skip, vsbd_result* res, uint8_t* fb,
                 int* fb_count, int* fb_list, cudaStream_t st);

/* Global motion prior of n coarse items from a first network pass (median
   translation of the confident predictions, least-squares rotation about the
   frame centre): items2 = items with the prior as search offset (the second
   pass's crops), prior = the rounded model displacement per item (added to
   the second pass's prediction).  One launch. */
int vsbpn_prior(const vsbd_item* items, const float* pout, int n, float scale, float conf_min,
                const uint8_t* skip, int W, int H, vsbd_item* items2, short2* prior,
                cudaStream_t st);

/* crops of n items into inputs [n][32][32][2] bf16 (training data) */
int vsbpn_crops(const uint8_t* curr, const uint8_t* prev, int pitch, int W, int H,
                const vsbd_item* items, int n, void* inputs, cudaStream_t st);

/* training-data labels of n searched items (kind 0 coarse, 1 fine) */
struct PNLabel {
  int16_t tx, ty;
  uint32_t sad;
  uint8_t kind, ok, use, pad;
};
int vsbpn_labels(const vsbd_result* res, const uint8_t* skip, int n, int kind, PNLabel* out,
                 cudaStream_t st);

#endif
