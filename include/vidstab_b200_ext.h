/*
 * vidstab_b200_ext.h -- entry points of libvidstab_b200 without a
 * counterpart in the reference library.  All take plain pointers and sizes;
 * "device" pointers are CUDA device addresses on the detector's GPU.
 */
#ifndef VIDSTAB_B200_EXT_H
#define VIDSTAB_B200_EXT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct _vsmotiondetect;
struct vsvector_;

/* Message of the last GPU-side failure on this thread ("" if none). */
VS_API const char* vsb_last_error(void);

/* Number of CUDA devices visible to the process. */
VS_API int vsb_device_count(void);

/* sizeof of the public structs as compiled into the library (ABI checks). */
VS_API int vsb_sizeof(const char* type_name);

/* vsMotionDetection with plane 0 already in device memory (e.g. decoded on
   the GPU): same results, no host-to-device copy of the frame.  Planar
   formats read the luma plane, packed formats the interleaved plane;
   pitch is in bytes.  The `show` overlay is not drawn (no host frame). */
VS_API int vsb_motion_detection_device(struct _vsmotiondetect* md, struct vsvector_* motions,
                                       const uint8_t* d_plane0, int pitch);

/* Search strategy of a detector: 0 (default) the dense search of every
   candidate; 1 the exact pruned search -- every candidate's SAD over the
   first quarter of its field's rows bounds its full SAD from below;
   candidates whose bound exceeds the full SAD of the best-bounded few cannot
   win and are not completed.  Both give identical LocalMotions.
   VSB_PRUNED_SEARCH in the environment makes 1 the default. */
VS_API int vsb_set_search_mode(struct _vsmotiondetect* md, int pruned);
/* The strategy detectors initialised from now on start with (-1: back to the
   environment's choice). */
VS_API void vsb_set_default_search_mode(int pruned);

/* The search tiling the detector picked (cost model + timing at init) for
   its coarse (fine = 0) or fine (1) fields: desc[0..7] = lattice rows per
   thread, layout (1: one lattice column per thread; 2: two, aligned by
   shifts; 3: two of one byte alignment, read from word-aligned window
   copies; 4: as 3 from one window copy, the odd columns against a copy of
   the field shifted by two bytes), lattice columns and rows per CTA, field
   strips, threads per CTA,
   shared memory bytes per CTA, CTAs per field. */
VS_API int vsb_search_tiling(const struct _vsmotiondetect* md, int fine, int* desc);

/* The prefilter of the detector: desc[0], desc[1] the width and height
   (output pixels per CTA) of the separate blur's tile, picked by timing at
   init, desc[2] its time per frame in ns (0 when it was not timed), desc[3]
   1 when the blur and the field min/max run as one launch (k_blurmm; planar
   frames, box sizes 3..9), in which case the tile is not used. */
VS_API int vsb_blur_tiling(const struct _vsmotiondetect* md, int* desc);

/* Kernel launches issued for this detector so far. */
VS_API long vsb_launch_count(const struct _vsmotiondetect* md);

/* Runs the detect API over a clip, frame by frame, the way a host filter
   does: vsMotionDetectInit, vsMotionDetection per frame (frame k's plane 0
   at frames + k*frame_bytes, row distance linesize; or, with on_device,
   device memory read through vsb_motion_detection_device), then cleanup.
   Every frame's motions are appended to `out` (up to out_cap records) and
   counts[k] receives their number.  If trf_path is not NULL the .trf file is
   written as vidstabdetect writes it.  *elapsed receives the wall time of the
   per-frame loop.  Returns the number of records, or -1. */
VS_API long vsb_detect_clip(int width, int height, int pformat, const uint8_t* frames,
                            long frame_bytes, int linesize, int nframes, int on_device,
                            int stepSize, int accuracy, int shakiness, double mincontrast,
                            int tripod, int show, int serializationMode, const char* trf_path,
                            void* out, long out_cap, int* counts, double* elapsed,
                            uint8_t* show_out);

/* Runs nframes frames through an initialised detector, in order, the way a
   host filter calls vsMotionDetection (on_device = 0: frame k's plane 0 at
   frames + k*frame_bytes in host memory, show not drawn) or
   vsb_motion_detection_device (on_device = 1: device addresses).  The
   LocalMotions of every frame are appended to out (at most out_cap records,
   LocalMotion layout) and freed; counts[k] receives their number.  The
   detector's state (previous frame, frame number) carries over between
   calls.  Without tripod mode or overlay, and with the dense search, frame
   k+1's blur, min/max and coarse search run on the GPU while frame k's fine
   search runs and its motions are assembled (for the plain search also while
   frame k's fields are selected), and host frames are copied one frame
   further ahead on a stream of their own (same results).
   Returns the number of records, or -1. */
VS_API long vsb_detect_run(struct _vsmotiondetect* md, const uint8_t* frames, long frame_bytes,
                           int linesize, int nframes, int on_device, void* out, long out_cap,
                           int* counts);

/* As vsb_detect_run, without the overlap: each frame is one call of
   vsMotionDetection (or vsb_motion_detection_device) that returns only
   when the frame's motions are complete -- the call sequence of a host
   filter such as vidstabdetect, timed as the drop-in's per-frame path. */
VS_API long vsb_detect_frames(struct _vsmotiondetect* md, const uint8_t* frames,
                              long frame_bytes, int linesize, int nframes, int on_device,
                              void* out, long out_cap, int* counts);

/* Many initialised detectors (one per stream, any mix of resolutions, with
   or without a search proposal) stepped together by the calling thread:
   every frame, the coarse stage of every detector is enqueued before any is
   waited for, so the streams' GPU work overlaps while the host selects and
   assembles the others' motions.  Frame k of stream s at clips[s] + k *
   frame_bytes[s] (host memory, or device memory with on_device), row pitch
   linesizes[s].  Records are appended frame by frame, stream by stream
   (LocalMotion layout, at most out_cap); counts[k*n + s] receives each
   frame's count.  Each stream's motions are its detector's own.  Returns
   the number of records, or -1. */
VS_API long vsb_detect_multi(struct _vsmotiondetect** mds, int n, const uint8_t* const* clips,
                             const long* frame_bytes, const int* linesizes, int nframes,
                             int on_device, void* out, long out_cap, int* counts);

/* Per-kernel device time: with timing on, CUDA events bracket every kernel
   of the detector on its stream.  ms[k] and count[k] for k = 0 blur,
   1 field min/max, 2 coarse search, 3 fine search, 4 proposal network,
   5 full searches of items that fell back (6 entries each; with a proposal,
   2 and 3 time the narrowed searches).
   Turning timing on resets the totals. */
VS_API int vsb_set_kernel_timing(struct _vsmotiondetect* md, int on);
VS_API int vsb_kernel_times(const struct _vsmotiondetect* md, double* ms, long* count);

/* Process-wide totals since load: kernels launched by the detect path, and
   bytes it copied host-to-device (frames, work lists) and device-to-host
   (per-field results). */
VS_API void vsb_counters(long long* launches, long long* h2d_bytes, long long* d2h_bytes);

/* Process-wide wall time of the per-frame path since load or the last
   reset, summed over frames: sec[0] device stage A (frame upload, blur,
   min/max, coarse search, results back), sec[1] host part A (selection,
   coarse motions, the simple model, fine work list), sec[2] device stage B
   (fine search), sec[3] host part B (fine motions, mean-match filter,
   result); *frames the number of frames.  Batched steps (vsb_batch_detect,
   vsb_batch_run) add their stage times the same way, each step counting
   one frame per stream; overlapped steps count the time spent waiting for
   each stage rather than its duration. */
VS_API void vsb_host_profile(double* sec, long* frames, int reset);

/* Test hook for the out-of-memory paths, host side only: returns the number
   of device allocations (cudaMalloc) the library has made since load; with
   fail_after >= 0 the allocation fail_after calls from now fails with
   cudaErrorMemoryAllocation (sticky != 0: that one and every later one),
   -1 disarms it.  The calls that meet the failure return VS_ERROR (or NULL)
   with the reason in vsb_last_error() and free what they had allocated. */
VS_API long long vsb_test_device_alloc(int fail_after, int sticky);

/* Measured byte-absolute-difference throughput (per second) of the GPU's
   packed SAD instruction sequence in a register-only loop: variant 0 the
   accumulate form the kernels use, 1 and 2 alternative formulations. */
VS_API int vsb_sad_peak(int variant, double* byteops_per_s);

/* ---- kernel-level entry points (host buffers in and out; for testing) ---- */

/* luma prefilter of one W x H plane (tight rows) with box size `size`
   (already clamped; < 2 copies) */
VS_API int vsb_boxblur_host(uint8_t* dst, const uint8_t* src, int width, int height, int size);
/* the same with vector-blur tile shape `shape` (0: 256x32, 1: 128x16,
   2: 128x32, 3: 64x32; shapes 1-3 serve box sizes up to 17, larger boxes
   take shape 0) */
VS_API int vsb_boxblur_host_tile(uint8_t* dst, const uint8_t* src, int width, int height,
                                 int size, int shape);

/* per-field, per-channel 8-bit (min,max) of an interleaved image with bpp
   bytes per pixel: out[(i*channels+c)*2 + {0,1}] */
VS_API int vsb_field_minmax_host(const uint8_t* img, int width, int height, int bpp,
                                 int channels, const int16_t* x, const int16_t* y, int n,
                                 int size, uint8_t* out);

/* planar field search exactly as vsMotionDetection runs it for one field
   set: spiral lattice of the given step within maxShift plus refinement, for
   n fields with centres (x,y) and lattice offsets (ox,oy).  Writes per field
   {sad, tx, ty, ok}; tx,ty relative to the offset.  tiles > 0 forces the
   number of CTAs per field. */
VS_API int vsb_field_search_host(const uint8_t* curr, const uint8_t* prev, int width,
                                 int height, int size, int maxShift, int stepSize, int packed_bpp,
                                 const int16_t* x, const int16_t* y, const int16_t* ox,
                                 const int16_t* oy, int n, int tiles, uint32_t* sad,
                                 int16_t* tx, int16_t* ty, int32_t* ok);

/* ---- allocation-free search (no counterpart in the reference) ----------
   For callers that cannot let a library allocate GPU memory: hosts that own
   all device memory through their own pools or budgets, where a cudaMalloc
   they did not make breaks the pool's accounting or the budget.  It runs
   the planar per-field search of vsMotionDetection (spiral lattice of
   maxShift/stepSize steps, halving refinement, range test) and allocates
   nothing: its scratch (per-field running minimum and completion counter,
   lattice rank tables; at most 4096 fields per call, 32768 lattice points
   and maxShift + stepSize <= 32767) lives in one static device array of
   311,300 bytes that every GPU loading the library holds until the process
   exits.
     d_curr, d_prev: blurred planes on the current device, 16-byte aligned,
       row pitch `pitch` a multiple of 16 bytes, readable up to 256 bytes past
       the end of their last row; every field's whole search window must lie
       inside the planes.
     d_fields: n records {int16 x, y, ox, oy} (centre, lattice offset).
     d_results: n records {uint32 sad; int16 tx, ty; int32 ok} (shift
       relative to the offset; ok = passed the range test).
     stream: a cudaStream_t (NULL: legacy default stream); the call is
       asynchronous on it.
   The first call on a device resolves the array's device address; make that
   first call before any stream capture.  All calls share the one array and
   it keeps the last call's contents, so calls whose GPU work overlaps (two
   streams, two host threads) race: serialize them.  Larger inputs are
   rejected with VS_ERROR and a message in vsb_last_error(). */
VS_API int vsb_field_search_noalloc(const uint8_t* d_curr, const uint8_t* d_prev, int pitch,
                                    int size, int maxShift, int stepSize, const void* d_fields,
                                    int n, void* d_results, void* stream);

/* ---- batched multi-stream detect (no reference counterpart: the reference
   runs one VSMotionDetect per stream; each stream here gives exactly the
   LocalMotions a VSMotionDetect of its own would give) ---- */
typedef struct vsb_batch vsb_batch;

/* n independent streams; stream s has frames of widths[s] x heights[s] in
   the planar format pformat and the configuration conf[s] (show is not
   drawn).  One step of all streams runs as two launches of one persistent
   kernel, each replayed from a captured CUDA graph; the search tilings of
   every distinct field geometry are picked at creation by timing candidate
   shapes in that kernel.  Returns NULL on failure (vsb_last_error()). */
VS_API vsb_batch* vsb_batch_create(int n, const int* widths, const int* heights, int pformat,
                                   const VSMotionDetectConfig* conf);
/* One frame of every stream: plane 0 of stream s at planes[s] with row
   pitch pitches[s] (device addresses with on_device != 0, else host
   memory).  motions[s] receives the stream's LocalMotions (free with
   vs_vector_del).  Returns VS_OK or VS_ERROR. */
VS_API int vsb_batch_detect(vsb_batch* b, const uint8_t* const* planes, const int* pitches,
                            int on_device, LocalMotions* motions);
/* nframes steps over clips: frame k of stream s at clips[s] + k *
   frame_bytes[s].  Records are appended step by step, stream by stream
   (LocalMotion layout, at most out_cap); counts[k*n + s] receives each
   frame's count.  Without virtual tripod on any stream, consecutive steps
   overlap on the GPU: step k+1's upload, blur, min/max and coarse search
   run on one CUDA stream while step k's fine search runs on another and the
   host assembles step k's motions (the results are vsb_batch_detect's, step
   by step).  Returns the number of records, or -1. */
VS_API long vsb_batch_run(vsb_batch* b, const uint8_t* const* clips, const long* frame_bytes,
                          const int* pitches, int nframes, int on_device, void* out,
                          long out_cap, int* counts);
VS_API void vsb_batch_free(vsb_batch* b);
/* The .trf output of vidstabdetect for batched streams: paths[s] (NULL:
   none) is created and started for stream s in serialization_mode
   (ASCII_SERIALIZATION_MODE or BINARY_SERIALIZATION_MODE), and every later
   step (vsb_batch_detect, vsb_batch_run) appends that stream's frame to it,
   byte for byte what vsWriteToFile writes after vsMotionDetection for a
   detector of its own.  Closing (or vsb_batch_free) ends the files.  Returns
   VS_OK or VS_ERROR (no file stays open then). */
VS_API int vsb_batch_open_trf(vsb_batch* b, const char* const* paths, int serialization_mode);
VS_API int vsb_batch_close_trf(vsb_batch* b);
/* Limits of the persistent kernel's bounded waits: a search or min/max item
   that waits for its stream's blur tiles gives up after `spins` polls
   (100 ns apart) or `cycles` SM clock cycles, whichever comes first; the
   step then fails with VS_ERROR ("a wait for blur tiles gave up" in
   vsb_last_error()), the step's frame is dropped for every stream, and the
   next step starts clean.  Defaults 2^24 polls and 8e9 cycles; a wait only
   runs out when the device work list is broken. */
VS_API int vsb_batch_set_wait_limit(vsb_batch* b, unsigned spins, long long cycles);
/* Fault injection for tests, on the host side: stage A's work list leaves
   out stream `stream`'s blur tiles (a negative stream restores the full
   list), so that stream's waits run out and the step fails as above.  No
   GPU fault is involved: the waits end at their limits. */
VS_API int vsb_batch_test_withhold_blur(vsb_batch* b, int stream);
/* persistent-kernel launches so far */
VS_API long vsb_batch_launch_count(const vsb_batch* b);
/* the persistent grid: CTAs, threads per CTA, dynamic shared memory per CTA */
VS_API int vsb_batch_grid(const vsb_batch* b, int* ctas, int* threads, long* smem);
/* the search tiling of geometry class k (streams whose coarse or fine fields
   share size, shift range and step share a class): desc[0..11] = lattice
   rows per thread, layout (as vsb_search_tiling), lattice columns and rows per CTA, field
   strips, threads, shared memory bytes per CTA, CTAs per field, search items
   per step, time of those items alone in the persistent kernel when tuned
   (ns), field size, lattice points per field.  Returns the number of classes
   (for any k, desc untouched when k is out of range), -1 without a batch. */
VS_API int vsb_batch_class(const vsb_batch* b, int k, int* desc);
/* The learned search proposal (blob as for vsb_set_proposal below) for
   every stream of the batch; NULL returns them to the dense search.  The
   network, the global-motion prior of streams with shakiness >= 8 (two
   network passes, as a single detector), the narrowed searches and the
   dense search of the items that fell back all become work items of the
   same persistent kernel: each step stays two graph launches.  A stream's
   results equal those of a detector of its own given the same blob.  No
   step may be in flight.  Returns VS_OK or VS_ERROR. */
VS_API int vsb_batch_set_proposal(vsb_batch* b, const void* blob, long bytes);
/* counts since vsb_batch_set_proposal, as vsb_proposal_stats: [0] items
   searched with the proposal, [1] of them fell back to the full search,
   [4], [5] coarse items / fallbacks ([2], [3], [6], [7] stay 0: the
   batch has no verify mode and searches fine fields densely) */
VS_API int vsb_batch_proposal_stats(const vsb_batch* b, long long* stats);

/* ---- learned search proposal (no reference counterpart) ----------------
   The reference searches every field over its whole candidate lattice.  A
   detector given a proposal network first predicts each field's
   displacement from a 32x32 crop pair (2x2 averages of the 64x64
   neighbourhood in the blurred current and previous planes), evaluates only
   the lattice points that bracket prediction +- radius plus one ring around
   them, and refines the winner exactly as the full search does.  An item
   falls back to the exact full search when the network's confidence logit
   is below conf_min, when the winner lies on the ring, or when the refined
   SAD per field pixel exceeds match_bound.  Planar formats only.

   blob: a serialized network (header "VSBP", version 1, its bf16 weights and
   f32 biases, and the radius / conf_min / match_bound it was calibrated
   with); NULL returns the detector to the plain full search. */
VS_API int vsb_set_proposal(struct _vsmotiondetect* md, const void* blob, long bytes);
/* as vsb_set_proposal, overriding the blob's radius (if >= 0), conf_min
   (if not NaN) and match_bound (if >= 0) */
VS_API int vsb_set_proposal_ex(struct _vsmotiondetect* md, const void* blob, long bytes,
                               double radius, double conf_min, double match_bound);
/* How the fine fields are searched with a proposal.  By default
   (fine_net = 0, fine_radius < 0) they take the exact dense search of the
   plain detector: their window is already centred on the coarse model's
   prediction and small.  fine_net = 0 with fine_radius >= 0: a narrowed
   window of that radius around the coarse model's prediction (zero
   residual), with the same fallbacks.  fine_net = 1: the network predicts
   them too (radius fine_radius, or the blob's radius when negative).
   fine_radius is at most 16 pixels. */
VS_API int vsb_set_proposal_scope(struct _vsmotiondetect* md, int fine_net, double fine_radius);
/* Network passes over the coarse fields: 1, or 2 -- the first pass's
   predictions give the frame a global motion model (median translation,
   least-squares rotation about the centre); the second pass re-centres
   every coarse crop on the model and predicts the residual.  For motions
   beyond the network's reach (64x64 crops).  vsb_set_proposal picks 2 when
   the detector's shakiness is 8 or more, else 1. */
VS_API int vsb_set_proposal_passes(struct _vsmotiondetect* md, int passes);
/* With verify on, every stage also runs the full search of every item and
   counts the items whose result (SAD, shift, range test) is identical. */
VS_API int vsb_set_proposal_verify(struct _vsmotiondetect* md, int on);
/* stats[0] items searched with the proposal, [1] of them fell back to the
   full search, [2] items verified, [3] of them identical to the full search,
   [4] coarse items searched, [5] of them fell back, [6] fine items searched,
   [7] of them fell back (8 entries) */
VS_API int vsb_proposal_stats(const struct _vsmotiondetect* md, long long* stats);

/* Training-data log of a plain detector: for every item the full search
   runs on (coarse fields, then the frame's fine fields), the network input
   (4096 bytes: [32][32][2] bf16) is appended to d_inputs and the label
   {int16 tx, ty; uint32 sad; uint8 kind (0 coarse, 1 fine), ok, use (field
   passes the contrast threshold), pad} (12 bytes) to d_labels, until cap
   items; d_inputs NULL turns it off.  Device memory of the detector's GPU. */
VS_API int vsb_set_field_log(struct _vsmotiondetect* md, void* d_inputs, void* d_labels, long cap);
VS_API long vsb_field_log_count(const struct _vsmotiondetect* md);

/* Network kernels for the offline trainer and tests (device pointers,
   stream a cudaStream_t or NULL).  d_params: n_bf16 bf16 weights then n_f32
   f32 biases; inputs [n][32][32][2] bf16; outputs [n][3] f32 (dx, dy in
   units of the blob's scale, confidence logit). */
VS_API int vsb_pnet_sizes(long* n_bf16, long* n_f32, long* act_bytes_per_item,
                          long* work_bytes_per_item);
/* training forward (fp32 FMA); stores the activations the backward needs */
VS_API int vsb_pnet_forward_train(const void* d_params, const void* d_input, int n, void* d_acts,
                                  float* d_out, void* stream);
/* gradient of sum(out * d_dout) w.r.t. the parameters, fp32 in parameter
   order (overwritten); d_work: work_bytes_per_item * n bytes */
VS_API int vsb_pnet_backward(const void* d_params, const void* d_input, const void* d_acts, int n,
                             const float* d_dout, float* d_grad, void* d_work, void* stream);
/* the detector's inference kernel (tensor cores) on prepared inputs */
VS_API int vsb_pnet_infer(const void* d_params, const void* d_input, int n, float* d_out,
                          void* stream);
/* the same kernel taking its inputs straight from two blurred planes, for
   n items {int16 x, y, ox, oy}, as a detector runs it */
VS_API int vsb_pnet_infer_items(const void* d_params, const uint8_t* d_curr,
                                const uint8_t* d_prev, int pitch, int width, int height,
                                const void* d_items, int n, float* d_out, void* stream);
/* network inputs of n items {int16 x, y, ox, oy} on two blurred planes */
VS_API int vsb_pnet_crops(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int width,
                          int height, const void* d_items, int n, void* d_input, void* stream);
/* narrowed search of one planar field set on host planes, given raw network
   outputs pout[n][3]: per item the result (as vsb_field_search_host) and
   the fallback flag (0 accepted, 1 falls back; the full search is not run) */
VS_API int vsb_pnet_narrow_host(const uint8_t* curr, const uint8_t* prev, int width, int height,
                                int size, int maxShift, int stepSize, const int16_t* x,
                                const int16_t* y, const int16_t* ox, const int16_t* oy, int n,
                                const float* pout, float scale, float radius, float conf_min,
                                uint32_t sad_bound, uint32_t* sad, int16_t* tx, int16_t* ty,
                                int32_t* ok, uint8_t* flags);

/* ---- second pass over many frames (vsLocalmotions2Transforms' fit,
   src/localmotion2transform.c:137-330, one GPU warp per frame) ---------
   Frame k's LocalMotions are recs[first[k] .. first[k+1]) (32-byte
   records).  Per frame: out[k] the transform vsMotionsToTransform returns,
   residual[k] the final objective value (NaN for a frame without motions),
   info[3k..3k+2] = gradient-descent rounds as the reference counts them (the
   last number of its global_motions.trf line), fields disabled for their
   match quality, fields disabled as outliers.  width/height: the frame;
   fov: degrees across the width (0: similarity model); smooth_zoom 0 drops
   the fitted zoom.  residual and info may be NULL.  One frame may hold up to
   vsb_motions_to_transforms_capacity() motions.  Host pointers; blocking. */
VS_API int vsb_motions_to_transforms(const LocalMotion* recs, const long* first, int nframes,
                                     int width, int height, double fov, int smooth_zoom,
                                     VSTransform* out, double* residual, int* info);
/* the same on device pointers, enqueued on `stream` (a cudaStream_t or
   NULL); max_motions: the largest first[k+1] - first[k] (shared memory is
   sized by it; a frame holding more is not fitted: extra = 1, info rounds
   -1) */
VS_API int vsb_motions_to_transforms_device(const LocalMotion* d_recs, const long* d_first,
                                            int nframes, int max_motions, int width, int height,
                                            double fov, int smooth_zoom, VSTransform* d_out,
                                            double* d_residual, int* d_info, void* stream);
VS_API int vsb_motions_to_transforms_capacity(void);
/* sizes and member offsets of VSTransformData, VSTransformConfig and
   VSTransformations, in a fixed order (ABI checks) */
VS_API int vsb_transform_layout(long* out, int cap);
/* kernel launches of the second pass since the library was loaded */
VS_API long vsb_motions_to_transforms_launches(void);

#ifdef __cplusplus
}
#endif
#endif
