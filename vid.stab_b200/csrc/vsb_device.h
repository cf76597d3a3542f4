/*
 * vsb_device.h -- internal C interface between the host C library and the
 * sm_100a CUDA code (vsb_device.cu).  Plain C types only.
 */
#ifndef VSB_DEVICE_H
#define VSB_DEVICE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One search item: a field centre and the displacement the lattice is
   centred on (zero for the coarse pass, the transform-derived offset for the
   fine pass). */
typedef struct {
  int16_t x, y;
  int16_t ox, oy;
} vsbd_item;

/* Result of one item: minimal SAD, the best displacement relative to the
   item's offset, and whether it passed the final range test. */
typedef struct {
  uint32_t sad;
  int16_t tx, ty;
  int32_t ok;
} vsbd_result;

#define VSBD_MAX_STAGES 8

/* Candidate geometry of one field set.
   Lattice point (a,b), 0<=a<na, 0<=b<nb, is the displacement
   (ax0 + a*step, by0 + b*step).  order[b*na + a] is its rank in the
   reference's visiting order: the lowest (SAD, rank) wins.  With has_origin
   the displacement (0,0) is evaluated first with rank 0 (raster scans).
   Refinement stage k evaluates the (2*r/h+1)^2 grid of spacing h around the
   current best (i outer, j inner), the centre excluded.  A result is rejected
   when |tx| >= limx or |ty| >= limy. */
typedef struct {
  int size, bpp, step;
  int na, nb, ax0, by0;
  int has_origin;
  int nstages;
  int st_r[VSBD_MAX_STAGES];
  int st_h[VSBD_MAX_STAGES];
  int limx, limy;
  const int32_t* order; /* host array, na*nb */
} vsbd_geom;

typedef struct vsbd_ctx vsbd_ctx;

/* Creates the device state of one detector.  blur_size < 2 means no blur
   (the plane is used as is; packed formats).  channels: 1 planar, 3 packed
   (contrast over the colour channels).  coarse_threshold: the coarse
   fields' contrast threshold (fields below it are never selected and the
   pruned search skips them).  Returns 0 or -1 (vsbd_error()). */
int vsbd_create(vsbd_ctx** out, int width, int height, int bpp, int blur_size, int channels,
                const vsbd_geom* coarse, const int16_t* cx, const int16_t* cy, int nc,
                const vsbd_geom* fine, const int16_t* fx, const int16_t* fy, int nf,
                double coarse_threshold);

/* 1: exact pruned search (partial-row bounds, survivors only; default),
   0: dense search of every candidate.  Both give identical results. */
int vsbd_set_search_mode(vsbd_ctx* c, int pruned);
/* the strategy detectors created later start with (-1: environment) */
void vsbd_set_default_search_mode(int pruned);
void vsbd_destroy(vsbd_ctx* c);

/* Stage A of one frame: take plane 0 (host pointer + linesize, or a device
   pointer + pitch when dev != NULL), blur it into the current buffer and,
   when search != 0, compute every field's (min,max) and run the coarse
   search of every coarse field against the previous buffer.  Blocks until
   the results are on the host.  minmax: (nc+nf)*channels (min,max) byte
   pairs, coarse first; coarse: nc results. */
int vsbd_stage_a(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev, int pitch,
                 int search, const uint8_t** minmax, const vsbd_result** coarse);

/* Stage B: fine search of n items against the previous buffer; blocks. */
int vsbd_stage_b(vsbd_ctx* c, const vsbd_item* items, int n, const vsbd_result** fine);

/* The current buffer becomes the previous one. */
void vsbd_commit_prev(vsbd_ctx* c);

/* Overlapped frames (a frame loop that knows the next frame): while the
   current frame's fine search runs (vsbd_stage_b_issue ... _collect, on a
   second stream), stage A of the next frame is enqueued
   (vsbd_stage_a_next_issue: its plane goes to the third buffer and is
   searched against the current frame's) and collected after the commit
   (vsbd_stage_a_next_collect).  Only when vsbd_can_overlap(c). */
int vsbd_can_overlap(const vsbd_ctx* c);
/* stage A of the current frame, enqueued only (collect with
   vsbd_stage_a_next_collect): lets one host thread keep several detectors'
   stages in flight */
int vsbd_stage_a_issue(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev,
                       int pitch, int search);
int vsbd_stage_a_next_issue(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev,
                            int pitch);
int vsbd_stage_a_next_collect(vsbd_ctx* c, const uint8_t** minmax, const vsbd_result** coarse);
/* A host frame copied ahead into upload slot 0 or 1 on a copy stream of its
   own, so that the copy overlaps the stages of earlier frames; then the next
   frame's stage A from that slot (it waits for the copy on the device).  A
   slot may be refilled once the stage A that read it has been collected. */
int vsbd_upload(vsbd_ctx* c, const uint8_t* host, int linesize, int slot);
/* whether the detector searches with a proposal network */
int vsbd_proposal_on(const vsbd_ctx* c);
/* frames whose stage A a frame loop may keep in flight (1 or 2) */
int vsbd_pipeline_depth(const vsbd_ctx* c);
int vsbd_stage_a_next_issue_uploaded(vsbd_ctx* c, int slot);
int vsbd_stage_b_issue(vsbd_ctx* c, const vsbd_item* items, int n);
int vsbd_stage_b_collect(vsbd_ctx* c, const vsbd_result** fine);

/* the search tiling the detector runs for its coarse (fine = 0) or fine
   fields: desc[0..7] = rows per thread, columns per thread, lattice columns
   and rows per CTA, field strips, threads, shared memory bytes, CTAs per item */
int vsbd_search_tiling(const vsbd_ctx* c, int fine, int* desc);

/* the prefilter's tile (desc[0] width, desc[1] height) and its tuned time
   per frame in ns (desc[2]; 0 when not tuned) */
int vsbd_blur_tiling(const vsbd_ctx* c, int* desc);

/* Kernel launches issued on behalf of this detector so far. */
long vsbd_launches(const vsbd_ctx* c);

/* per-kernel CUDA-event timing (indices VSBD_KT_*); with a proposal
   network, COARSE and FINE time the narrowed searches, PNET the network and
   FALLBACK the full searches of the items that fell back */
#define VSBD_KT_BLUR 0
#define VSBD_KT_MINMAX 1
#define VSBD_KT_COARSE 2
#define VSBD_KT_FINE 3
#define VSBD_KT_PNET 4
#define VSBD_KT_FALLBACK 5
#define VSBD_NKT 6

/* ---- learned search proposal (vsb_pnet.cu) ---- */

/* Turns the proposal on for this detector (params: the network's bf16
   weights followed by its f32 biases, pn_param_bytes() bytes, host memory)
   or off (params NULL).  scale: network units -> pixels; radius: pixels
   around the prediction; conf_min: confidence logit threshold;
   match_bound: largest trusted refined SAD per pixel.  Planar only. */
int vsbd_set_proposal(vsbd_ctx* c, const void* params, float scale, float radius, float conf_min,
                      float match_bound);
long vsbd_pnet_param_bytes(void);
/* fine fields take the network's proposal (fine_net 1) or the coarse
   model's prediction, i.e. zero residual (0, the default); fine_radius:
   their window radius in pixels (< 0: 4 px around the model, the blob's
   radius around the network) */
int vsbd_set_proposal_scope(vsbd_ctx* c, int fine_net, float fine_radius);
/* coarse fields: 1 network pass, or 2 (the second with crops re-centred on
   the global motion model fitted to the first pass's predictions) */
int vsbd_set_proposal_passes(vsbd_ctx* c, int passes);
/* with verify on, every stage also runs the full search and compares */
int vsbd_set_proposal_verify(vsbd_ctx* c, int on);
/* [0] items searched with a proposal, [1] of them fell back, [2] items
   verified against the full search, [3] of them identical; [4]/[5] and
   [6]/[7] searched / fell back of the coarse and the fine items */
int vsbd_proposal_stats(const vsbd_ctx* c, long long* st);
/* Training-data log: every searched item's network input (d_inputs, 4096
   bytes each) and full-search label (d_labels, 12 bytes each) appended,
   up to cap items; NULL turns it off.  Plain (full-search) detectors only. */
int vsbd_set_field_log(vsbd_ctx* c, void* d_inputs, void* d_labels, long cap);
long vsbd_field_log_count(const vsbd_ctx* c);

/* network kernels (device pointers; stream may be NULL) */
int vsbd_pnet_forward_train(const void* d_params, const void* d_input, int n, void* d_acts,
                            float* d_out, void* stream);
int vsbd_pnet_backward(const void* d_params, const void* d_input, const void* d_acts, int n,
                       const float* d_dout, float* d_grad, void* d_work, void* stream);
int vsbd_pnet_infer(const void* d_params, const void* d_input, int n, float* d_out, void* stream);
int vsbd_pnet_infer_items(const void* d_params, const uint8_t* d_curr, const uint8_t* d_prev,
                          int pitch, int width, int height, const void* d_items, int n,
                          float* d_out, void* stream);
int vsbd_pnet_crops(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int width,
                    int height, const void* d_items, int n, void* d_input, void* stream);
int vsbd_pnet_narrow_host(const uint8_t* curr, const uint8_t* prev, int width, int height,
                          const vsbd_geom* g, const vsbd_item* items, int n, const float* pout,
                          float scale, float radius, float conf_min, unsigned sad_bound,
                          vsbd_result* out, uint8_t* flags);
int vsbd_set_timing(vsbd_ctx* c, int on);
int vsbd_kernel_times(const vsbd_ctx* c, double* ms, long* n);

/* byte-absdiff throughput of a register-only SAD loop (see vsb_device.cu) */
int vsbd_sad_peak(int variant, double* byteops_per_s);

/* process-wide totals: kernel launches, host-to-device and device-to-host
   bytes of the per-frame path */
void vsbd_counters(long long* launches, long long* h2d, long long* d2h);

/* device allocations made so far; fail_after >= 0 makes the allocation that
   many calls later fail (sticky: that one and all later ones), -1 disarms */
long long vsbd_test_device_alloc(int fail_after, int sticky);

/* Message of the last failure on this thread. */
const char* vsbd_error(void);
void vsbd_set_error(const char* msg);

/* the field search with all scratch in a static device array (vsb_noalloc.cu) */
int vsbd_search_noalloc(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int size,
                        int maxShift, int stepSize, const void* d_items, int n, void* d_results,
                        void* stream);

/* ---- kernel-level entry points for parity tests (host buffers in/out) --- */
int vsbd_blur_host(uint8_t* dst, const uint8_t* src, int width, int height, int size);
int vsbd_blur_host_shape(uint8_t* dst, const uint8_t* src, int width, int height, int size,
                         int shape);
int vsbd_minmax_host(const uint8_t* img, int width, int height, int bpp, int channels,
                     const int16_t* x, const int16_t* y, int n, int size, uint8_t* out);
int vsbd_search_host(const uint8_t* curr, const uint8_t* prev, int width, int height,
                     const vsbd_geom* g, const vsbd_item* items, int n, int tiles_hint,
                     vsbd_result* out);
int vsbd_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
