/*
 * vsb_device.cu -- sm_100a kernels of the motion-detection pass and the thin
 * C shim the host library calls (declared in vsb_device.h).
 *
 * Kernels (one frame of one stream):
 *   k_blur      separable box prefilter, both passes fused in one shared
 *               memory tile (src/boxblur.c:104-332 of the reference)
 *   k_minmax    8-bit min/max of every measurement field (the integer part of
 *               src/motiondetect.c:389-407; the double contrast is formed on
 *               the host with the reference's expression)
 *   k_search    per-field SAD search: CTAs split a field's candidate lattice,
 *               each computes full SADs against a shared-memory window of the
 *               previous frame and folds (SAD, visiting rank) into one 64-bit
 *               atomicMin per field; the last CTA of a field runs the
 *               dependent refinement rounds and the range test
 *               (src/motiondetect.c:439-586 planar, :591-660 packed).
 */
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "vsb_device.h"
#include "vsb_plan.h"
#include "vsb_pnet.h"
#include "vsb_prefilter.cuh"
#include "vsb_search.cuh"
#include "vsb_sweep.cuh"
#include "vsb_blurmm.cuh"
#include "vsb_finewarp.cuh"

/* ------------------------------------------------------------------------ */
/* error plumbing                                                            */
/* ------------------------------------------------------------------------ */
static thread_local char g_err[512];

static void set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
}
static void set_msg(const char* m) { snprintf(g_err, sizeof(g_err), "%s", m); }

/* process-wide counters: kernels launched and bytes copied host<->device by
   the per-frame path (read by benchmarks) */
static unsigned long long g_nlaunch = 0, g_nh2d = 0, g_nd2h = 0;
static void count_launches(long n) { __atomic_fetch_add(&g_nlaunch, (unsigned long long)n, __ATOMIC_RELAXED); }
static void count_h2d(size_t b) { __atomic_fetch_add(&g_nh2d, (unsigned long long)b, __ATOMIC_RELAXED); }
static void count_d2h(size_t b) { __atomic_fetch_add(&g_nd2h, (unsigned long long)b, __ATOMIC_RELAXED); }

extern "C" void vsbd_counters(long long* launches, long long* h2d, long long* d2h) {
  if (launches) *launches = (long long)__atomic_load_n(&g_nlaunch, __ATOMIC_RELAXED);
  if (h2d) *h2d = (long long)__atomic_load_n(&g_nh2d, __ATOMIC_RELAXED);
  if (d2h) *d2h = (long long)__atomic_load_n(&g_nd2h, __ATOMIC_RELAXED);
}

extern "C" const char* vsbd_error(void) { return g_err; }

/* device allocations: counted, and the one `g_alloc_fail` calls from now
   fails (and, sticky, every later one) -- a test hook for the out-of-memory
   paths; (cudaMalloc) names the runtime's function, not the counting macro */
static long long g_alloc_calls = 0;
static int g_alloc_fail = -1, g_alloc_sticky = 0;
extern "C" cudaError_t vsbd_dev_malloc(void** p, size_t bytes) {
  __atomic_fetch_add(&g_alloc_calls, 1ll, __ATOMIC_RELAXED);
  int k = __atomic_load_n(&g_alloc_fail, __ATOMIC_RELAXED);
  if (k == 0) {
    if (!g_alloc_sticky) __atomic_store_n(&g_alloc_fail, -1, __ATOMIC_RELAXED);
    *p = NULL;
    return cudaErrorMemoryAllocation;
  }
  if (k > 0) __atomic_store_n(&g_alloc_fail, k - 1, __ATOMIC_RELAXED);
  return (cudaMalloc)(p, bytes);
}

extern "C" long long vsbd_test_device_alloc(int fail_after, int sticky) {
  g_alloc_sticky = sticky;
  __atomic_store_n(&g_alloc_fail, fail_after < 0 ? -1 : fail_after, __ATOMIC_RELAXED);
  return __atomic_load_n(&g_alloc_calls, __ATOMIC_RELAXED);
}

#define CK(call)                                 \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) {                     \
      set_err(#call, e_);                        \
      return -1;                                 \
    }                                            \
  } while (0)

/* ------------------------------------------------------------------------ */
/* box blur                                                                  */
/* ------------------------------------------------------------------------ */

/* One CTA blurs a BT_H x BT_W output tile (blur_tile). */
__global__ void __launch_bounds__(256) k_blur(const uint8_t* __restrict__ src, int sp,
                                              uint8_t* __restrict__ dst, int dp, int W, int H,
                                              int half, BlurDiv dv) {
  __shared__ __align__(16) uint8_t tile[BT_SMEM];
  blur_tile(src, sp, dst, dp, W, H, half, dv, blockIdx.x, blockIdx.y, tile);
}

/* Fallback for windows wider than the fused tile's halo: one thread per row,
   then one per column, each with a running sum (same arithmetic). */
__global__ void k_blur_rows(const uint8_t* __restrict__ src, int sp, uint8_t* __restrict__ dst,
                            int dp, int W, int H, int half, BlurDiv dv) {
  int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= H) return;
  const uint8_t* s = src + (size_t)y * sp;
  uint8_t* d = dst + (size_t)y * dp;
  unsigned acc = 0;
  for (int k = -half; k <= half; k++) acc += s[min(max(k, 0), W - 1)];
  for (int x = 0; x < W; x++) {
    d[x] = (uint8_t)blur_div(acc, dv);
    acc += s[min(x + half + 1, W - 1)];
    acc -= s[max(x - half, 0)];
  }
}

__global__ void k_blur_cols(const uint8_t* __restrict__ src, int sp, uint8_t* __restrict__ dst,
                            int dp, int W, int H, int half, BlurDiv dv) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  unsigned acc = 0;
  for (int k = -half; k <= half; k++) acc += src[(size_t)min(max(k, 0), H - 1) * sp + x];
  for (int y = 0; y < H; y++) {
    dst[(size_t)y * dp + x] = (uint8_t)blur_div(acc, dv);
    acc += src[(size_t)min(y + half + 1, H - 1) * sp + x];
    acc -= src[(size_t)max(y - half, 0) * sp + x];
  }
}

/* Planar prefilter with vector memory access: one CTA of 256 threads
   blurs a BH x BW output tile (BW a multiple of 64 up to 256, BH a multiple
   of 1024/BW), for a window half-width HALF known at compile time; the
   tile shape is picked per detector by timing (autotune_blur).  Input rows (clamped to the frame) are staged with 16-byte
   loads from 16 bytes left of the tile to 16 bytes right of it (tiles
   touching the left or right frame edge load bytewise with clamped
   columns).  The horizontal pass gives each task a run of 16 outputs of one
   row: the bytes it needs are read as words once, the window sum slides
   along the run, and the 16 results are stored as one 16-byte vector.  The
   vertical pass runs 4-column sliding sums down a quarter of the tile and
   stores words.  Same arithmetic as blur_tile (window sums, floor division
   by the size). */
#define BF_MAXHALF 16
template <int HALF, int BF_W = 256, int BF_H = 32>
__global__ void __launch_bounds__(256) k_blur_fast(const uint8_t* __restrict__ src, int sp,
                                                   uint8_t* __restrict__ dst, int dp, int W, int H,
                                                   BlurDiv dv) {
  constexpr int BF_RAWP = BF_W + 32;
  constexpr int PARTS = 1024 / BF_W; /* vertical pass: threads per column group */
  static_assert(BF_W % 64 == 0 && BF_W <= 256 && BF_H % PARTS == 0, "blur tile shape");
  __shared__ __align__(16) uint8_t raw[(BF_H + 2 * HALF) * BF_RAWP];
  __shared__ __align__(16) uint8_t hor[(BF_H + 2 * HALF) * BF_W];
  constexpr int ROWS = BF_H + 2 * HALF, WIN = 2 * HALF + 1;
  const int x0 = blockIdx.x * BF_W, y0 = blockIdx.y * BF_H;
  const bool interior = x0 >= 16 && x0 + BF_W + 16 <= W;
  if (interior) {
    for (int i = threadIdx.x; i < ROWS * (BF_RAWP / 16); i += blockDim.x) {
      const int r = i / (BF_RAWP / 16), v = i - r * (BF_RAWP / 16);
      const int gy = min(max(y0 - HALF + r, 0), H - 1);
      *(uint4*)(raw + r * BF_RAWP + (v << 4)) =
          *(const uint4*)(src + (size_t)gy * sp + x0 - 16 + (v << 4));
    }
  } else {
    for (int i = threadIdx.x; i < ROWS * BF_RAWP; i += blockDim.x) {
      const int r = i / BF_RAWP, c = i - r * BF_RAWP;
      const int gy = min(max(y0 - HALF + r, 0), H - 1);
      const int gx = min(max(x0 - 16 + c, 0), W - 1);
      raw[r * BF_RAWP + c] = src[(size_t)gy * sp + gx];
    }
  }
  __syncthreads();
  /* runs of 16 outputs at columns c0 .. c0+15 need raw bytes
     16 + c0 - HALF .. 16 + c0 + 15 + HALF; read the words from 16 + c0 - 16 */
  constexpr int NW = (16 + 15 + HALF) / 4 + 1; /* the words holding bytes c0 .. c0 + 31 + HALF */
  for (int t = threadIdx.x; t < ROWS * (BF_W / 16); t += blockDim.x) {
    const int r = t / (BF_W / 16), c0 = (t - r * (BF_W / 16)) * 16;
    const uint32_t* wp = (const uint32_t*)(raw + r * BF_RAWP + c0); /* byte 16 + c0 - 16 */
    uint32_t wv[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) wv[k] = wp[k];
    /* byte b of the staged row relative to c0 - 16 + 16 = c0: index 16 + b */
#define BYTE_AT(b) ((wv[(16 + (b)) >> 2] >> (((16 + (b)) & 3) * 8)) & 0xffu)
    unsigned acc = 0;
#pragma unroll
    for (int k = -HALF; k <= HALF; k++) acc += BYTE_AT(k);
    uint32_t o[4] = { 0u, 0u, 0u, 0u };
#pragma unroll
    for (int q = 0; q < 16; q++) {
      if (q > 0) acc += BYTE_AT(q + HALF) - BYTE_AT(q - 1 - HALF);
      o[q >> 2] |= blur_div(acc, dv) << (8 * (q & 3));
    }
#undef BYTE_AT
    *(uint4*)(hor + r * BF_W + c0) = make_uint4(o[0], o[1], o[2], o[3]);
  }
  __syncthreads();
  /* thread: 4 columns (cg), a part of the tile rows */
  const int cg = threadIdx.x % (BF_W / 4), part = threadIdx.x / (BF_W / 4);
  const int gx = x0 + cg * 4;
  if (gx >= W) return;
  const int rb = part * (BF_H / PARTS);
  unsigned a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
  for (int k = 0; k < WIN; k++) {
    const unsigned w = *(const unsigned*)(hor + (rb + k) * BF_W + cg * 4);
    a0 += w & 0xff;
    a1 += (w >> 8) & 0xff;
    a2 += (w >> 16) & 0xff;
    a3 += w >> 24;
  }
  const bool full4 = gx + 4 <= W;
#pragma unroll
  for (int r = rb; r < rb + BF_H / PARTS; r++) {
    if (r > rb) {
      const unsigned wi = *(const unsigned*)(hor + (r + WIN - 1) * BF_W + cg * 4);
      const unsigned wo = *(const unsigned*)(hor + (r - 1) * BF_W + cg * 4);
      a0 += (wi & 0xff) - (wo & 0xff);
      a1 += ((wi >> 8) & 0xff) - ((wo >> 8) & 0xff);
      a2 += ((wi >> 16) & 0xff) - ((wo >> 16) & 0xff);
      a3 += (wi >> 24) - (wo >> 24);
    }
    const int gy = y0 + r;
    if (gy >= H) break;
    const unsigned o = blur_div(a0, dv) | (blur_div(a1, dv) << 8) | (blur_div(a2, dv) << 16) |
                       (blur_div(a3, dv) << 24);
    uint8_t* d = dst + (size_t)gy * dp + gx;
    if (full4) {
      *(unsigned*)d = o;
    } else {
      for (int k = 0; k < 4 && gx + k < W; k++) d[k] = (uint8_t)(o >> (8 * k));
    }
  }
}

/* tile shapes (width, height) of the vector blur; shape 0 serves every
   half-width, the others half-widths up to 8 (box sizes up to 17) */
#define VSB_BLUR_SHAPES 4
static const int g_blur_shape[VSB_BLUR_SHAPES][2] = { { 256, 32 }, { 128, 16 }, { 128, 32 },
                                                      { 64, 32 } };

static int blur_shape_ok(int shape, int half) {
  if (shape == 0) return half >= 1 && half <= BF_MAXHALF;
  return shape > 0 && shape < VSB_BLUR_SHAPES && half >= 1 && half <= 8;
}

/* k_blur_fast for the window half-width of the plane and a tile shape */
static void launch_blur_fast(int shape, cudaStream_t st, const uint8_t* src, int sp, uint8_t* dst,
                             int dp, int W, int H, int half, BlurDiv dv) {
  const dim3 grid((W + g_blur_shape[shape][0] - 1) / g_blur_shape[shape][0],
                  (H + g_blur_shape[shape][1] - 1) / g_blur_shape[shape][1]);
#define VSB_BLURH(K, BW, BH) \
  case K: k_blur_fast<K, BW, BH><<<grid, 256, 0, st>>>(src, sp, dst, dp, W, H, dv); break;
#define VSB_BLUR8(BW, BH) \
  VSB_BLURH(1, BW, BH) VSB_BLURH(2, BW, BH) VSB_BLURH(3, BW, BH) VSB_BLURH(4, BW, BH) \
  VSB_BLURH(5, BW, BH) VSB_BLURH(6, BW, BH) VSB_BLURH(7, BW, BH) VSB_BLURH(8, BW, BH)
  if (shape == 0) {
    switch (half) {
      VSB_BLUR8(256, 32)
      VSB_BLURH(9, 256, 32) VSB_BLURH(10, 256, 32) VSB_BLURH(11, 256, 32)
      VSB_BLURH(12, 256, 32) VSB_BLURH(13, 256, 32) VSB_BLURH(14, 256, 32)
      VSB_BLURH(15, 256, 32) VSB_BLURH(16, 256, 32)
      default: break;
    }
  } else if (shape == 1) {
    switch (half) { VSB_BLUR8(128, 16) default: break; }
  } else if (shape == 2) {
    switch (half) { VSB_BLUR8(128, 32) default: break; }
  } else {
    switch (half) { VSB_BLUR8(64, 32) default: break; }
  }
#undef VSB_BLUR8
#undef VSB_BLURH
}

/* launches the prefilter of one plane with vector-blur tile shape `shape`
   (where the plane allows the vector blur); returns the number of kernels */
static int launch_blur(const uint8_t* src, int sp, uint8_t* dst, int dp, int W, int H, int size,
                       uint8_t* tmp, int tp, cudaStream_t st, int shape = 0) {
  int half = size / 2;
  BlurDiv dv;
  make_div(size, half, &dv);
  if (half >= 1 && half <= BF_MAXHALF &&
      ((((uintptr_t)src | (uintptr_t)sp | (uintptr_t)dst | (uintptr_t)dp) & 15) == 0)) {
    launch_blur_fast(blur_shape_ok(shape, half) ? shape : 0, st, src, sp, dst, dp, W, H, half, dv);
    return 1;
  }
  if (half <= BT_MAXHALF) {
    dim3 grid((W + BT_W - 1) / BT_W, (H + BT_H - 1) / BT_H);
    k_blur<<<grid, 256, 0, st>>>(src, sp, dst, dp, W, H, half, dv);
    return 1;
  }
  k_blur_rows<<<(H + 127) / 128, 128, 0, st>>>(src, sp, tmp, tp, W, H, half, dv);
  k_blur_cols<<<(W + 127) / 128, 128, 0, st>>>(tmp, tp, dst, dp, W, H, half, dv);
  return 2;
}

/* ------------------------------------------------------------------------ */
/* field min / max                                                           */
/* ------------------------------------------------------------------------ */

/* One CTA per field (minmax_field). */
__global__ void __launch_bounds__(256) k_minmax(const uint8_t* __restrict__ img, int pitch,
                                                const int16_t* __restrict__ xs,
                                                const int16_t* __restrict__ ys, int S, int bpp,
                                                int nch, uint8_t* __restrict__ out, double thr,
                                                uint8_t* __restrict__ skip) {
  const int f = blockIdx.x;
  minmax_field(img, pitch, xs[f], ys[f], S, bpp, nch, f, out, thr, skip);
}

/* bytes b of a word with lo <= b < hi (byte offsets) set to 0xff */
__device__ __forceinline__ unsigned byte_mask(int lo, int hi) {
  unsigned m = 0;
#pragma unroll
  for (int b = 0; b < 4; b++)
    if (b >= lo && b < hi) m |= 0xffu << (8 * b);
  return m;
}

/* Planar 8-bit min/max of both field sets in one launch: blocks [0, nc)
   take the coarse fields (size Sc, threshold thr, skip flags), the rest the
   fine fields (size Sf).  Rows are read with 16-byte loads; bytes outside
   the field are masked to the neutral value.  Same outputs as minmax_field
   (the contrast is the reference's double expression). */
__global__ void __launch_bounds__(256) k_minmax_planar(const uint8_t* __restrict__ img, int pitch,
                                                       const int16_t* __restrict__ xy, int nc,
                                                       int nf, int Sc, int Sf,
                                                       uint8_t* __restrict__ out, double thr,
                                                       uint8_t* __restrict__ skip) {
  __shared__ unsigned smn[8], smx[8];
  const int f = blockIdx.x;
  const bool coarse = f < nc;
  const int S = coarse ? Sc : Sf;
  const int x = coarse ? xy[f] : xy[2 * nc + (f - nc)];
  const int y = coarse ? xy[nc + f] : xy[2 * nc + nf + (f - nc)];
  const int x0 = x - S / 2, y0 = y - S / 2;
  const int xa = x0 & ~15;
  const int nv = (x0 + S - xa + 15) >> 4;
  unsigned mn = 0xffffffffu, mx = 0u;
  for (int i = threadIdx.x; i < S * nv; i += blockDim.x) {
    const int r = i / nv, v = i - r * nv;
    const int bx = xa + (v << 4);
    const uint4 q = *(const uint4*)(img + (size_t)(y0 + r) * pitch + bx);
    const unsigned w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int b0 = bx + 4 * k;
      const unsigned m = byte_mask(x0 - b0, x0 + S - b0);
      mn = __vminu4(mn, w[k] | ~m);
      mx = __vmaxu4(mx, w[k] & m);
    }
  }
  unsigned bmn = min(min(mn & 0xff, (mn >> 8) & 0xff), min((mn >> 16) & 0xff, mn >> 24));
  unsigned bmx = max(max(mx & 0xff, (mx >> 8) & 0xff), max((mx >> 16) & 0xff, mx >> 24));
  bmn = __reduce_min_sync(0xffffffffu, bmn);
  bmx = __reduce_max_sync(0xffffffffu, bmx);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smn[warp] = bmn;
    smx[warp] = bmx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      bmn = min(bmn, smn[w]);
      bmx = max(bmx, smx[w]);
    }
    out[f * 2 + 0] = (uint8_t)bmn;
    out[f * 2 + 1] = (uint8_t)bmx;
    if (coarse && skip) {
      const double con = (double)((int)bmx - (int)bmn) / ((double)((int)bmx + (int)bmn) + 0.1);
      skip[f] = !(con >= thr && con > 0.0);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* SAD search (kernels in vsb_search.cuh)                                    */
/* ------------------------------------------------------------------------ */


#define VSB_MAX_DEVICES 64

static int current_device(void) {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev >= 0 && dev < VSB_MAX_DEVICES ? dev : 0;
}

/* SMs of the current device (kept per device; a benign race fills an entry
   with the same value twice at worst) */
static int sm_count(void) {
  static int n[VSB_MAX_DEVICES];
  const int dev = current_device();
  int v = __atomic_load_n(&n[dev], __ATOMIC_RELAXED);
  if (!v) {
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (v <= 0) v = 148;
    __atomic_store_n(&n[dev], v, __ATOMIC_RELAXED);
  }
  return v;
}

/* raises a kernel's dynamic shared-memory limit only when a launch needs
   more than this device already allows it (the attribute call costs
   microseconds of host time per launch otherwise); slot names the kernel */
static cudaError_t ensure_smem(const void* fn, int slot, size_t smem) {
  static size_t done[16][64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 16 && slot >= 0 && slot < 64 && done[dev][slot] >= smem) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && dev >= 0 && dev < 16 && slot >= 0 && slot < 64) done[dev][slot] = smem;
  return e;
}

/* largest dynamic shared memory one search CTA may request on this device
   (the kernels' static shared memory counts against the opt-in limit) */
static size_t search_smem_limit(void) {
  static size_t lims[VSB_MAX_DEVICES];
  const int dev = current_device();
  size_t lim = __atomic_load_n(&lims[dev], __ATOMIC_RELAXED);
  if (!lim) {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t stat = 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_lattice<4>) == cudaSuccess) stat = fa.sharedSizeBytes;
    if (cudaFuncGetAttributes(&fa, k_lattice<2>) == cudaSuccess && fa.sharedSizeBytes > stat)
      stat = fa.sharedSizeBytes;
    if (cudaFuncGetAttributes(&fa, k_lattice<8>) == cudaSuccess && fa.sharedSizeBytes > stat)
      stat = fa.sharedSizeBytes;
    lim = optin > 0 ? (size_t)optin - stat - 64 : 48 * 1024;
    __atomic_store_n(&lims[dev], lim, __ATOMIC_RELAXED);
  }
  return lim;
}

/* registers per thread of the search kernel for TB rows and TA columns per
   thread */
static int lattice_regs(int TB, int TA) {
  static int r[5][9] = { { 0 } };
  if (TB < 1 || TB > 8 || TA < 1 || TA > 4) return 0;
  if (!r[TA][TB]) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaErrorInvalidValue;
    if (TA == 1) {
      if (TB == 2) e = cudaFuncGetAttributes(&fa, k_lattice<2>);
      if (TB == 4) e = cudaFuncGetAttributes(&fa, k_lattice<4>);
      if (TB == 8) e = cudaFuncGetAttributes(&fa, k_lattice<8>);
    } else if (TA == 2) {
      if (TB == 2) e = cudaFuncGetAttributes(&fa, k_lattice<2, false, 2>);
      if (TB == 4) e = cudaFuncGetAttributes(&fa, k_lattice<4, false, 2>);
    } else if (TA == 3) {
      if (TB == 2) e = cudaFuncGetAttributes(&fa, k_lattice<2, false, 3>);
      if (TB == 4) e = cudaFuncGetAttributes(&fa, k_lattice<4, false, 3>);
    } else {
      if (TB == 2) e = cudaFuncGetAttributes(&fa, k_lattice<2, false, 4>);
      if (TB == 4) e = cudaFuncGetAttributes(&fa, k_lattice<4, false, 4>);
    }
    r[TA][TB] = e == cudaSuccess ? fa.numRegs : 64;
  }
  return r[TA][TB];
}

/* Candidate tile shapes (columns x rows of the lattice per CTA, rows per
   thread, field strips) with their modelled time: SAD issue slots of the CTA
   times the waves of CTAs the SMs can hold at once (shared memory, threads
   and registers), with a penalty below 16 resident warps per SM, plus the
   staging of the window.  Forced values (> 0) pin a dimension.  Returns the
   number of candidates written (best first, at most cap). */

static int tile_candidates(const DGeom& g, int nitems, int tb_force, int strip_force,
                           int nab_force, int nbb_force, TileCand* out, int cap,
                           int max_threads = 512, int ta_force = 0) {
  const size_t lim = search_smem_limit();
  const int sms = sm_count();
  int n = 0;
  const int tbs[3] = { 4, 2, 8 };
  const int sb = g.step * g.bpp;
  for (int tv = 0; tv < 12; tv++) {
    /* layouts: 1 one column per thread, 2 two with shifts, 3 two from aligned
       window copies, 4 two from one copy and a shifted field copy */
    const int ti = tv % 3, TA = 1 + tv / 3;
    int TB = tbs[ti];
    if (tb_force > 0 && TB != tb_force) continue;
    if (TA >= 2 && (TB > 4 || sb > 8 || g.rows > 0)) continue;
    if (TA == 3 && (sb & 1)) continue;
    if (TA == 4 && (sb & 3) != 2) continue;
    if (ta_force > 0 && TA != ta_force) continue;
    for (int ns = 1; ns <= 8; ns *= 2) {
      if (strip_force > 0 && ns != strip_force) continue;
      const int rows = geom_rows(g);
      if (rows % ns) continue;
      int Rs = rows / ns;
      if (Rs < 4) continue;
      /* two-column layouts need nab even (a multiple of 4 for aligned copies
         of a step of 2 mod 4 bytes): the even split rounded up */
      const int nab_mul = TA == 1 ? 1 : (TA == 4 || (TA == 3 && (sb & 3)) ? 4 : 2);
      int nab_prev = -1;
      for (int ka = 1; ka <= 16; ka++) {
        int nab = (g.na + ka - 1) / ka;
        nab = (nab + nab_mul - 1) / nab_mul * nab_mul;
        if (nab_force > 0) nab = nab_force;
        if (nab_force <= 0 && nab == nab_prev) continue;
        nab_prev = nab;
        for (int m = 1; m * TB <= ((g.nb + TB - 1) / TB) * TB; m++) {
          int nbb = m * TB;
          if (nbb_force > 0) nbb = nbb_force;
          if (nbb % TB) break;
          if (nab % nab_mul) continue;
          DGeom t = g;
          t.tb = TB;
          t.ta = TA;
          t.nab = nab;
          t.nbb = nbb;
          t.nstrip = ns;
          t.nta = (g.na + nab - 1) / nab;
          t.ntb = (g.nb + nbb - 1) / nbb;
          /* layout 4: even-column pairs in the first half of the block, odd
             ones in the second, each half whole warps */
          int threads = TA == 4 ? 2 * (((nab / 4) * (nbb / TB) * ns + 31) & ~31)
                                : (nab / (TA == 1 ? 1 : 2)) * (nbb / TB) * ns;
          threads = (threads + 31) & ~31;
          if (threads > max_threads || threads < 32) {
            if (nbb_force > 0) break;
            continue;
          }
          t.threads = threads;
          TileLayout L = tile_layout(t);
          if (L.total > lim) {
            if (nbb_force > 0) break;
            continue;
          }
          long ctas = (long)nitems * t.nta * t.ntb;
          int cps = (int)((228 * 1024) / (L.total + 1024));
          if (2048 / threads < cps) cps = 2048 / threads;
          int regs = lattice_regs(TB, TA);
          if (regs > 0 && 65536 / (threads * regs) < cps) cps = 65536 / (threads * regs);
          if (cps > 32) cps = 32;
          if (cps < 1) {
            if (nbb_force > 0) break;
            continue;
          }
          double eff = (double)Rs / (Rs + g.step * (TB - 1));
          double work = (double)nab * nbb * rows * L.rowW / eff; /* lane-SAD4 slots */
          double warps = (double)cps * threads / 32.0;
          double occ = warps >= 16 ? 1.0 : warps / 16.0;
          long waves = (ctas + (long)sms * cps - 1) / ((long)sms * cps);
          double clk = (double)waves * cps *
                       (work / 64.0 / occ + (double)window_copies(t) * L.WH_alloc * L.WP / 32.0);
          /* two columns per thread load each window word once for both (fewer
             shared-memory loads per SAD than the model counts) */
          if (TA == 2) clk *= 0.85;
          /* ... and with aligned window copies they need no shifts */
          if (TA >= 3) clk *= 0.7;
          /* keep the cap best, sorted */
          int pos = n < cap ? n : cap;
          while (pos > 0 && out[pos - 1].clk > clk) {
            if (pos < cap) out[pos] = out[pos - 1];
            pos--;
          }
          if (pos < cap) {
            out[pos].clk = clk;
            out[pos].g = t;
            if (n < cap) n++;
          }
          if (nbb_force > 0) break;
        }
        if (nab_force > 0) break;
      }
    }
  }
  return n;
}

static int geom_upload(const vsbd_geom* h, int nitems, int tiles_hint, GeomDev* out) {
  memset(out, 0, sizeof(*out));
  DGeom& g = out->g;
  g.S = h->size; g.bpp = h->bpp; g.step = h->step;
  g.na = h->na; g.nb = h->nb; g.ax0 = h->ax0; g.by0 = h->by0;
  g.has_origin = h->has_origin; g.nstages = h->nstages;
  if (g.nstages > VSBD_MAX_STAGES) { set_msg("too many refinement stages"); return -1; }
  if ((g.S * g.bpp) % 16 != 0) { set_msg("field row bytes must be a multiple of 16"); return -1; }
  g.maxq = 1;
  for (int i = 0; i < g.nstages; i++) {
    g.st_r[i] = h->st_r[i];
    g.st_h[i] = h->st_h[i];
    int side = (2 * h->st_r[i]) / h->st_h[i] + 1;
    if (side * side > g.maxq) g.maxq = side * side;
  }
  g.limx = h->limx; g.limy = h->limy;
  int n = g.na * g.nb;
  int32_t* rank = (int32_t*)malloc(sizeof(int32_t) * n);
  short2* pt = (short2*)malloc(sizeof(short2) * (n + 1));
  memcpy(rank, h->order, sizeof(int32_t) * n);
  pt[0] = make_short2(0, 0);
  for (int b = 0; b < g.nb; b++)
    for (int a = 0; a < g.na; a++) {
      int k = rank[b * g.na + a];
      if (k >= 0 && k <= n) pt[k] = make_short2((short)(g.ax0 + a * g.step), (short)(g.by0 + b * g.step));
    }
  cudaError_t e1 = cudaMalloc(&out->d_order, sizeof(int32_t) * n);
  cudaError_t e2 = cudaMalloc(&out->d_point, sizeof(short2) * (n + 1));
  if (e1 == cudaSuccess) e1 = cudaMemcpy(out->d_order, rank, sizeof(int32_t) * n, cudaMemcpyHostToDevice);
  if (e2 == cudaSuccess) e2 = cudaMemcpy(out->d_point, pt, sizeof(short2) * (n + 1), cudaMemcpyHostToDevice);
  free(rank);
  free(pt);
  if (e1 != cudaSuccess || e2 != cudaSuccess) { set_err("geometry upload", e1 != cudaSuccess ? e1 : e2); return -1; }
  g.order = out->d_order;
  g.point = out->d_point;
  int tb_f = 0, ns_f = 0, nab_f = 0, nbb_f = 0, ta_f = 0;
  if (tiles_hint > 0) { /* test hook: ta*100000000 + tb*1000000 + strips*10000 + nab*100 + nbb */
    ta_f = tiles_hint / 100000000;
    tb_f = (tiles_hint / 1000000) % 100;
    ns_f = (tiles_hint / 10000) % 100;
    nab_f = (tiles_hint / 100) % 100;
    nbb_f = tiles_hint % 100;
  }
  TileCand cand[1];
  int nc = tile_candidates(g, nitems > 0 ? nitems : 1, tb_f, ns_f, nab_f, nbb_f, cand, 1, 512, ta_f);
  if (nc < 1) { set_msg("no search tiling fits in shared memory"); return -1; }
  g = cand[0].g;
  out->smem = tile_layout(g).total;
  return 0;
}

static void geom_free(GeomDev* g) {
  if (g->d_order) cudaFree(g->d_order);
  if (g->d_point) cudaFree(g->d_point);
  g->d_order = NULL;
  g->d_point = NULL;
}

template <int TB, int TA>
static int launch_lattice(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                          const vsbd_item* d_items, int n, unsigned long long* keys,
                          unsigned* tickets, vsbd_result* d_res, cudaStream_t st) {
  cudaError_t e = ensure_smem((const void*)k_lattice<TB, false, TA>,
                              (TA == 4 ? 24 : (TA == 3 ? 20 : (TA == 2 ? 11 : 0))) +
                                  (TB == 2 ? 0 : (TB == 4 ? 1 : 2)),
                              gd.smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute(k_lattice)", e);
    return -1;
  }
  dim3 grid(gd.g.nta * gd.g.ntb, n);
  k_lattice<TB, false, TA><<<grid, gd.g.threads, gd.smem, st>>>(curr, prev, pitch, gd.g, d_items,
                                                                keys, tickets, d_res);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    char what[160];
    snprintf(what, sizeof(what), "k_lattice<%d,%d> launch (%d x %d CTAs x %d threads, %zu B shared)",
             TB, TA, gd.g.nta * gd.g.ntb, n, gd.g.threads, gd.smem);
    set_err(what, e);
    return -1;
  }
  return 1;
}

static int launch_search(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                         const vsbd_item* d_items, int n, unsigned long long* keys,
                         unsigned* tickets, vsbd_result* d_res, cudaStream_t st) {
  if (n <= 0) return 0;
  switch (gd.g.tb) {
    case 2:
      if (gd.g.ta == 4) return launch_lattice<2, 4>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
      if (gd.g.ta == 3) return launch_lattice<2, 3>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
      return gd.g.ta == 2 ? launch_lattice<2, 2>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st)
                          : launch_lattice<2, 1>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
    case 4:
      if (gd.g.ta == 4) return launch_lattice<4, 4>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
      if (gd.g.ta == 3) return launch_lattice<4, 3>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
      return gd.g.ta == 2 ? launch_lattice<4, 2>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st)
                          : launch_lattice<4, 1>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
    case 8: return launch_lattice<8, 1>(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
  }
  set_msg("unsupported rows-per-thread");
  return -1;
}

/* ---- the persistent TMA-staged sweep (vsb_sweep.cuh) ---- */

/* the (step, field size) pairs the sweep is compiled for: the defaults'
   coarse fields (step 6; 48 to 112 pixels, 360p to 1080p) and fine fields
   (step 2; 16 to 48 pixels, 360p to 4K) */
#define VSB_SWEEP_CASES(X) \
  X(6, 3) X(6, 4) X(6, 5) X(6, 7) X(2, 1) X(2, 2) X(2, 3)

static bool sweep_supported(const DGeom& g) {
  if (g.bpp != 1 || g.has_origin || g.rows > 0 || g.S % 16) return false;
  const int NQ = g.S / 16;
#define VSB_SW_SUP(ST, NQv) if (g.step == ST && NQ == NQv) return true;
  VSB_SWEEP_CASES(VSB_SW_SUP)
#undef VSB_SW_SUP
  return false;
}

/* registers per thread of a sweep instantiation (0 if not compiled) */
static int sweep_regs(int step, int NQ) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaErrorInvalidValue;
#define VSB_SW_REG(ST, NQv) \
  if (step == ST && NQ == NQv) e = cudaFuncGetAttributes(&fa, k_sweep<NQv, ST>);
  VSB_SWEEP_CASES(VSB_SW_REG)
#undef VSB_SW_REG
  return e == cudaSuccess ? fa.numRegs : 0;
}

/* Candidate sweep plans, best first by a cost model: lattice-column groups
   (the whole width, or the width split in two or three), lattice rows per
   tile and field strips; the persistent grid holds as many CTAs as fit on
   the GPU at once. */
static int sweep_candidates(const DGeom& g, int nitems, TileCand* out, int cap) {
  if (!sweep_supported(g) || nitems < 1) return 0;
  const size_t lim = search_smem_limit();
  const int sms = sm_count();
  const int regs = sweep_regs(g.step, g.S / 16);
  if (regs <= 0) return 0;
  /* the plan (ncg column groups of 8, nbb lattice rows, ns field strips)
     with its modelled time, or false when it does not fit */
  auto make = [&](int ncg, int nbb, int ns, TileCand* c) -> bool {
    if (g.S % ns || g.S / ns < 2) return false;
    const int ntask = ncg * nbb * ns;
    const int threads = (ntask + 31) & ~31;
    if (threads > SW_MAX_THREADS || threads < 64) return false;
    DGeom t = g;
    t.ta = 5;
    t.tb = 1;
    t.nab = ncg * SW_TA;
    t.nbb = nbb;
    t.nta = (g.na + t.nab - 1) / t.nab;
    t.ntb = (g.nb + nbb - 1) / nbb;
    t.nstrip = ns;
    t.threads = threads;
    const SweepLayout L = sweep_layout(t);
    if (L.total > lim) return false;
    int cps = (int)((228 * 1024) / (L.total + 2048));
    if (2048 / threads < cps) cps = 2048 / threads;
    if (65536 / (threads * regs) < cps) cps = 65536 / (threads * regs);
    if (cps < 1) return false;
    if (cps > 4) cps = 4;
    const long T = (long)nitems * t.nta * t.ntb;
    t.ctas = (int)(T < (long)sms * cps ? T : (long)sms * cps);
    const long per_cta = (T + t.ctas - 1) / t.ctas;
    /* a tile's lane-SAD slots (padded columns and rows included), the
       per-row loads of each thread, and a fixed cost per tile */
    const int Rs = g.S / ns;
    const double work = (double)t.nab * nbb * g.S * (g.S / 4) +
                        (double)ntask * Rs * (sw_chunks(g.step, g.S / 16) + 2 * (g.S / 16) + 12);
    const double warps = (double)cps * threads / 32.0;
    const double occ = warps >= 12 ? 1.0 : warps / 12.0;
    c->clk = (double)per_cta * (work / (64.0 / cps) / occ + 2500.0);
    c->g = t;
    return true;
  };
  /* plans whose one tile holds an item's whole lattice (the fine fields):
     timed whatever the model says */
  TileCand whole[3];
  int nwhole = 0;
  if (g.nb <= 48)
    for (int ns = 1; ns <= 4 && nwhole < 3; ns *= 2)
      if (make((g.na + SW_TA - 1) / SW_TA, g.nb, ns, &whole[nwhole])) nwhole++;
  if (nwhole > cap / 3) nwhole = cap / 3;
  const int mcap = cap - nwhole;
  int n = 0, ncg_prev = -1;
  for (int split = 1; split <= 3; split++) {
    const int ncg = ((g.na + split - 1) / split + SW_TA - 1) / SW_TA;
    if (ncg == ncg_prev) continue;
    ncg_prev = ncg;
    for (int nbb = 1; nbb <= 24 && nbb <= g.nb; nbb++)
      for (int ns = 1; ns <= 16; ns *= 2) {
        TileCand c;
        if (!make(ncg, nbb, ns, &c)) continue;
        if (c.g.nbb == g.nb && c.g.nab >= g.na) continue; /* already among the whole plans */
        int pos = n < mcap ? n : mcap;
        while (pos > 0 && out[pos - 1].clk > c.clk) {
          if (pos < mcap) out[pos] = out[pos - 1];
          pos--;
        }
        if (pos < mcap) {
          out[pos] = c;
          if (n < mcap) n++;
        }
      }
  }
  for (int k = 0; k < nwhole; k++) out[n++] = whole[k];
  return n;
}

template <int NQ, int STEP>
static int launch_sweep_t(const DGeom& g, size_t smem, int slot, const uint8_t* curr,
                          const uint8_t* prev, int pitch, const vsbd_item* d_items, int n,
                          unsigned long long* keys, unsigned* tickets, vsbd_result* d_res,
                          unsigned* err, cudaStream_t st) {
  cudaError_t e = ensure_smem((const void*)k_sweep<NQ, STEP>, slot, smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute(k_sweep)", e);
    return -1;
  }
  k_sweep<NQ, STEP><<<g.ctas, g.threads, smem, st>>>(curr, prev, pitch, g, d_items, n, keys,
                                                     tickets, d_res, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    char what[160];
    snprintf(what, sizeof(what), "k_sweep<%d,%d> launch (%d CTAs x %d threads, %zu B shared)",
             NQ, STEP, g.ctas, g.threads, smem);
    set_err(what, e);
    return -1;
  }
  return 1;
}

/* the sweep of items[0 .. n) with plan g (ta == 5); err: a device-visible
   word the kernel raises when a wait for its copies runs out */
static int launch_sweep(const DGeom& g, const uint8_t* curr, const uint8_t* prev, int pitch,
                        const vsbd_item* d_items, int n, unsigned long long* keys,
                        unsigned* tickets, vsbd_result* d_res, unsigned* err, cudaStream_t st) {
  if (n <= 0) return 0;
  if ((pitch & 15) || ((uintptr_t)prev & 15) || ((uintptr_t)curr & 15)) {
    set_msg("the sweep needs 16-byte aligned planes and pitch");
    return -1;
  }
  const size_t smem = sweep_layout(g).total;
  const int NQ = g.S / 16;
  int slot = 40;
#define VSB_SW_LAUNCH(ST, NQv)                                                                  \
  if (g.step == ST && NQ == NQv)                                                                \
    return launch_sweep_t<NQv, ST>(g, smem, slot, curr, prev, pitch, d_items, n, keys,          \
                                   tickets, d_res, err, st);                                    \
  slot++;
  VSB_SWEEP_CASES(VSB_SW_LAUNCH)
#undef VSB_SW_LAUNCH
  set_msg("no sweep compiled for this field geometry");
  return -1;
}

/* k_fine over items[0 .. n): one CTA of `warps` warps per item, T lattice
   rows per thread (1, 2 or 4), the field rows in ns strips (1, 2 or 4) */
static int launch_fine_warp(const GeomDev& gd, int warps, int T, int ns, const uint8_t* curr,
                            const uint8_t* prev, int pitch, const vsbd_item* d_items, int n,
                            vsbd_result* d_res, cudaStream_t st) {
  if (n <= 0) return 0;
  const DGeom& g = gd.g;
  if (!fw_supported(g) || warps < 1 || warps > FW_MAX_WARPS || (T != 1 && T != 2 && T != 4) ||
      (ns != 1 && ns != 2 && ns != 4)) {
    set_msg("k_fine does not take this field geometry or configuration");
    return -1;
  }
  const int nt = 32 * warps;
  const size_t smem = fw_layout(g, nt, T, ns).total;
  if (smem > search_smem_limit()) {
    set_msg("k_fine: the search window does not fit in shared memory");
    return -1;
  }
  cudaError_t e = cudaErrorInvalidValue;
#define VSB_FW(SV, TV, SLOT)                                                                   \
  if (g.S == SV && T == TV) {                                                                \
    e = ensure_smem((const void*)k_fine<SV, TV>, SLOT, smem);                                \
    if (e == cudaSuccess)                                                                    \
      k_fine<SV, TV><<<n, nt, smem, st>>>(curr, prev, pitch, g, d_items, d_res, ns);         \
  }
  VSB_FW(16, 1, 50) VSB_FW(16, 2, 51) VSB_FW(16, 4, 52)
  VSB_FW(32, 1, 53) VSB_FW(32, 2, 54) VSB_FW(32, 4, 55)
  VSB_FW(48, 1, 56) VSB_FW(48, 2, 57) VSB_FW(48, 4, 58)
#undef VSB_FW
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("k_fine launch", e);
    return -1;
  }
  return 1;
}

/* full search of the items in list[0 .. *count), at most n of them:
   persistent CTAs, as many as fit on the GPU at once */
template <int TB, int TA>
static int launch_list_tb(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                          const vsbd_item* d_items, int n, const int* count, const int* list,
                          unsigned long long* keys, unsigned* tickets, vsbd_result* d_res,
                          cudaStream_t st) {
  cudaError_t e = ensure_smem((const void*)k_lattice_list<TB, TA>,
                              (TA == 4 ? 26 : (TA == 3 ? 22 : (TA == 2 ? 14 : 3))) +
                                  (TB == 2 ? 0 : (TB == 4 ? 1 : 2)),
                              gd.smem);
  int cps = gd.list_cps;
  if (e == cudaSuccess && cps <= 0)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, k_lattice_list<TB, TA>, gd.g.threads,
                                                      gd.smem);
  if (e != cudaSuccess) {
    set_err("k_lattice_list set-up", e);
    return -1;
  }
  long units = (long)n * gd.g.nta * gd.g.ntb;
  long grid = (long)sm_count() * (cps > 0 ? cps : 1);
  if (grid > units) grid = units;
  k_lattice_list<TB, TA><<<(unsigned)grid, gd.g.threads, gd.smem, st>>>(curr, prev, pitch, gd.g, d_items,
                                                                   count, list, keys, tickets, d_res);
  return 1;
}

static int launch_list(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                       const vsbd_item* d_items, int n, const int* count, const int* list,
                       unsigned long long* keys, unsigned* tickets, vsbd_result* d_res,
                       cudaStream_t st) {
  if (n <= 0) return 0;
  switch (gd.g.tb) {
    case 2:
      if (gd.g.ta == 4) return launch_list_tb<2, 4>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
      if (gd.g.ta == 3) return launch_list_tb<2, 3>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
      return gd.g.ta == 2 ? launch_list_tb<2, 2>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st)
                          : launch_list_tb<2, 1>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
    case 4:
      if (gd.g.ta == 4) return launch_list_tb<4, 4>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
      if (gd.g.ta == 3) return launch_list_tb<4, 3>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
      return gd.g.ta == 2 ? launch_list_tb<4, 2>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st)
                          : launch_list_tb<4, 1>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
    case 8: return launch_list_tb<8, 1>(gd, curr, prev, pitch, d_items, n, count, list, keys, tickets, d_res, st);
  }
  set_msg("unsupported rows-per-thread");
  return -1;
}

/* the partial pass: every candidate's sum over the field's first rows */
template <int TB>
static int launch_emit_tb(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                          const vsbd_item* d_items, int n, cudaStream_t st) {
  cudaError_t e = ensure_smem((const void*)k_lattice<TB, true>, TB == 2 ? 6 : (TB == 4 ? 7 : 8),
                              gd.smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute(k_lattice emit)", e);
    return -1;
  }
  dim3 grid(gd.g.nta * gd.g.ntb, n);
  k_lattice<TB, true><<<grid, gd.g.threads, gd.smem, st>>>(curr, prev, pitch, gd.g, d_items, NULL,
                                                           NULL, NULL);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    char what[160];
    snprintf(what, sizeof(what), "k_lattice<%d> partial-pass launch (%d x %d CTAs x %d threads, "
             "%zu B shared)", TB, gd.g.nta * gd.g.ntb, n, gd.g.threads, gd.smem);
    set_err(what, e);
    return -1;
  }
  return 1;
}

static int launch_emit(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                       const vsbd_item* d_items, int n, cudaStream_t st) {
  if (n <= 0) return 0;
  switch (gd.g.tb) {
    case 2: return launch_emit_tb<2>(gd, curr, prev, pitch, d_items, n, st);
    case 4: return launch_emit_tb<4>(gd, curr, prev, pitch, d_items, n, st);
    case 8: return launch_emit_tb<8>(gd, curr, prev, pitch, d_items, n, st);
  }
  set_msg("unsupported rows-per-thread");
  return -1;
}

/* Pruned search of n items: partial pass, bound + survivors, survivors'
   full SADs and refinement.  gp is the partial-pass geometry (rows < S, emit
   set), gd the full one.  Returns the number of kernels launched or -1. */
static int launch_pruned(const GeomDev& gd, const GeomDev& gp, const uint8_t* curr,
                         const uint8_t* prev, int pitch, const vsbd_item* d_items, int n,
                         const uint8_t* skip, unsigned* part, int* counts, int* lists,
                         int* boxes, unsigned long long* keys, unsigned* tickets,
                         vsbd_result* d_res, cudaStream_t st) {
  if (n <= 0) return 0;
  GeomDev p = gp;
  p.g.emit = part;
  p.g.skip = skip;
  if (launch_emit(p, curr, prev, pitch, d_items, n, st) < 0) return -1;
  DGeom g = gd.g;
  g.skip = skip;
  const size_t fs = (size_t)g.S * g.S * g.bpp + 64;
  cudaError_t e = ensure_smem((const void*)k_prune, 9, fs);
  if (e != cudaSuccess) { set_err("cudaFuncSetAttribute(k_prune)", e); return -1; }
  k_prune<<<n, 256, fs, st>>>(curr, prev, pitch, g, d_items, part, 4, keys, counts, lists, boxes);
  const size_t ss = survive_smem(g);
  e = ensure_smem((const void*)k_survive, 10, ss);
  if (e != cudaSuccess) { set_err("cudaFuncSetAttribute(k_survive)", e); return -1; }
  int chunks = 4 * sm_count() / n;
  if (chunks < 1) chunks = 1;
  if (chunks > 16) chunks = 16;
  dim3 grid(chunks, n);
  k_survive<<<grid, 256, ss, st>>>(curr, prev, pitch, g, geom_rows(gp.g), d_items, part, counts,
                                   lists, boxes, keys, tickets, d_res);
  return 3;
}

/* Times the modelled best tilings of one field set on the detector's own
   buffers and items and keeps the fastest.  The dense lattice does the same
   work whatever the pixels hold, so the contents of the buffers do not matter.
   Results are cached per (geometry, item count) for the process. */
struct TuneEntry {
  int dev, S, bpp, step, na, nb, nstages, nitems, rows;
  DGeom g;
};
/* the cache, and the tuning itself, are serialised by g_tune_lock:
   detectors may be created from several host threads at once, and timings
   taken concurrently on one GPU would mislead each other */
static TuneEntry g_tune[64];
static int g_ntune = 0;
static pthread_mutex_t g_tune_lock = PTHREAD_MUTEX_INITIALIZER;

struct TuneLock {
  TuneLock() { pthread_mutex_lock(&g_tune_lock); }
  ~TuneLock() { pthread_mutex_unlock(&g_tune_lock); }
};

static int autotune_tiling(GeomDev* gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                           const vsbd_item* d_items, int n, unsigned long long* keys,
                           unsigned* tickets, vsbd_result* d_res, cudaStream_t st,
                           unsigned* emit_buf = NULL) {
  if (n <= 0 || getenv("VSB_NO_AUTOTUNE")) return 0;
  TuneLock lock;
  const int dev = current_device();
  DGeom& g = gd->g;
  for (int i = 0; i < g_ntune; i++) {
    TuneEntry& e = g_tune[i];
    if (e.dev == dev && e.S == g.S && e.bpp == g.bpp && e.step == g.step && e.na == g.na &&
        e.nb == g.nb &&
        e.nstages == g.nstages && e.nitems == n && e.rows == g.rows) {
      DGeom t = e.g;
      t.order = g.order;
      t.point = g.point;
      g = t;
      gd->smem = tile_layout(g).total;
      return 0;
    }
  }
  /* the model's best tilings of each layout (one lattice column per thread;
     two with shifts; two from aligned window copies; two from one copy and
     a shifted field copy): the model does not
     count shared-memory loads and shifts, which is where the layouts
     differ, so all three are timed */
  TileCand cand[32];
  int nc = tile_candidates(g, n, 0, 0, 0, 0, cand, 8, 512, 1);
  nc += tile_candidates(g, n, 0, 0, 0, 0, cand + nc, 6, 512, 2);
  nc += tile_candidates(g, n, 0, 0, 0, 0, cand + nc, 8, 512, 3);
  nc += tile_candidates(g, n, 0, 0, 0, 0, cand + nc, 10, 512, 4);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  /* one candidate's time over `reps` launches after one untimed launch
     (negative if it cannot run) */
  auto time_cand = [&](const DGeom& cg, int reps) -> float {
    GeomDev t = *gd;
    t.g = cg;
    t.g.emit = emit_buf;
    t.g.skip = NULL;
    t.smem = tile_layout(t.g).total;
    auto one = [&]() {
      return emit_buf ? launch_emit(t, curr, prev, pitch, d_items, n, st)
                      : launch_search(t, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
    };
    if (one() < 0) {
      const cudaError_t le = cudaGetLastError();
      if (getenv("VSB_DEBUG_TUNE"))
        fprintf(stderr, "tiling tuning: tiling skipped (tb %d ta %d %dx%d, %d strips, %d threads: "
                "%s; %s)\n", cg.tb, cg.ta, cg.nab, cg.nbb, cg.nstrip, cg.threads, vsbd_error(),
                cudaGetErrorString(le));
      return -1.f;
    }
    cudaEventRecord(e0, st);
    for (int rep = 0; rep < reps; rep++) one();
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  /* the clocks ramp up under the first launches: warm up on the model's
     favourite before anything is timed */
  for (int w = 0; w < 3 && nc > 0; w++) time_cand(cand[0].g, 3);
  float ms_of[40];
  for (int k = 0; k < nc; k++) ms_of[k] = time_cand(cand[k].g, 3);
  /* the three fastest once more, twice each in turn, best time kept: a
     single short timing can mislead by a few percent */
  int top[3] = { -1, -1, -1 };
  for (int k = 0; k < nc; k++) {
    if (ms_of[k] < 0.f) continue;
    for (int p = 0; p < 3; p++)
      if (top[p] < 0 || ms_of[k] < ms_of[top[p]]) {
        for (int q = 2; q > p; q--) top[q] = top[q - 1];
        top[p] = k;
        break;
      }
  }
  float best_ms = 1e30f;
  DGeom best = g;
  for (int round = 0; round < 2; round++)
    for (int p = 0; p < 3; p++) {
      if (top[p] < 0) continue;
      float ms = time_cand(cand[top[p]].g, 5);
      if (ms >= 0.f && ms < best_ms) {
        best_ms = ms;
        best = cand[top[p]].g;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_err(emit_buf ? "partial-pass tiling tuning" : "search tiling tuning", le);
      return -1;
    }
  }
  best.emit = NULL;
  g = best;
  gd->smem = tile_layout(g).total;
  if (g_ntune < 64) {
    TuneEntry& e = g_tune[g_ntune++];
    e.dev = dev;
    e.S = g.S; e.bpp = g.bpp; e.step = g.step; e.na = g.na; e.nb = g.nb;
    e.nstages = g.nstages; e.nitems = n; e.rows = g.rows; e.g = g;
  }
  return 0;
}

/* Whether the persistent sweep beats the tuned per-tile search for a field
   set: the tuned tiling and the sweep's best modelled plans are timed on the
   detector's own buffers and items (the dense search does the same work
   whatever the pixels hold) and the faster is kept; cached per geometry,
   item count and device for the process.  *on = 1 with *plan the sweep's
   plan, else 0.  err: the sweep's error word (device-visible). */
struct SweepTune {
  int dev, S, step, na, nb, nstages, nitems, on;
  DGeom g;
};
static SweepTune g_swtune[64];
static int g_nswtune = 0;

static int autotune_sweep(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                          const vsbd_item* d_items, int n, unsigned long long* keys,
                          unsigned* tickets, vsbd_result* d_res, unsigned* err,
                          volatile unsigned* h_err, cudaStream_t st, DGeom* plan, int* on) {
  *on = 0;
  if (n <= 0 || !sweep_supported(gd.g) || getenv("VSB_NO_SWEEP") || getenv("VSB_NO_AUTOTUNE"))
    return 0;
  /* VSB_FORCE_SWEEP: the sweep's best plan whatever the timings say (tests) */
  const bool force = getenv("VSB_FORCE_SWEEP") != NULL;
  TuneLock lock;
  const int dev = current_device();
  const DGeom& g = gd.g;
  for (int i = 0; !force && i < g_nswtune; i++) {
    const SweepTune& e = g_swtune[i];
    if (e.dev == dev && e.S == g.S && e.step == g.step && e.na == g.na && e.nb == g.nb &&
        e.nstages == g.nstages && e.nitems == n) {
      *on = e.on;
      *plan = e.g;
      plan->order = g.order;
      plan->point = g.point;
      return 0;
    }
  }
  TileCand cand[12];
  const int nc = sweep_candidates(g, n, cand, 10);
  if (nc > 0) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time_of = [&](const DGeom* sw, int reps) -> float {
      auto one = [&]() {
        return sw ? launch_sweep(*sw, curr, prev, pitch, d_items, n, keys, tickets, d_res, err,
                                 st)
                  : launch_search(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
      };
      if (one() < 0) {
        /* a plan that cannot launch here is skipped; its error is not
           the tuning's */
        const cudaError_t le = cudaGetLastError();
        if (getenv("VSB_DEBUG_TUNE"))
          fprintf(stderr, "sweep tuning: plan skipped (%s; %s)\n", vsbd_error(),
                  cudaGetErrorString(le));
        return -1.f;
      }
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps; r++) one();
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      return ms / reps;
    };
    for (int w = 0; w < 3; w++) time_of(NULL, 3); /* clocks up */
    float lat_ms = time_of(NULL, 5);
    float ms_of[12];
    for (int k = 0; k < nc; k++) ms_of[k] = time_of(&cand[k].g, 3);
    int top[3] = { -1, -1, -1 };
    for (int k = 0; k < nc; k++) {
      if (ms_of[k] < 0.f) continue;
      for (int p = 0; p < 3; p++)
        if (top[p] < 0 || ms_of[k] < ms_of[top[p]]) {
          for (int q = 2; q > p; q--) top[q] = top[q - 1];
          top[p] = k;
          break;
        }
    }
    float best_ms = 1e30f;
    int best = -1;
    for (int round = 0; round < 2; round++) {
      const float lm = time_of(NULL, 5);
      if (lm >= 0.f && lm < lat_ms) lat_ms = lm;
      for (int p = 0; p < 3; p++) {
        if (top[p] < 0) continue;
        const float ms = time_of(&cand[top[p]].g, 5);
        if (ms >= 0.f && ms < best_ms) {
          best_ms = ms;
          best = top[p];
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_err("search sweep tuning", le);
      return -1;
    }
    if (*h_err) {
      *h_err = 0;
      set_msg("the search sweep's staging did not complete while tuning");
      return -1;
    }
    if (getenv("VSB_DEBUG_TUNE")) {
      fprintf(stderr, "sweep tuning S=%d step=%d na=%d items=%d: per-tile search %.1f us\n", g.S,
              g.step, g.na, n, 1000.f * lat_ms);
      for (int k = 0; k < nc; k++)
        fprintf(stderr, "  plan %d: %d cols x %d rows, %d strips, %d threads, %d CTAs, %zu B: "
                "%.1f us%s\n", k, cand[k].g.nab, cand[k].g.nbb, cand[k].g.nstrip,
                cand[k].g.threads, cand[k].g.ctas, sweep_layout(cand[k].g).total, 1000.f * ms_of[k],
                k == best ? " (best)" : "");
    }
    if (best >= 0 && lat_ms >= 0.f && (force || best_ms < lat_ms)) {
      *on = 1;
      *plan = cand[best].g;
    }
  }
  if (!force && g_nswtune < 64) {
    SweepTune& e = g_swtune[g_nswtune++];
    e.dev = dev; e.S = g.S; e.step = g.step; e.na = g.na; e.nb = g.nb;
    e.nstages = g.nstages; e.nitems = n; e.on = *on; e.g = *plan;
  }
  return 0;
}

/* Tiling of a field set without uploading its tables (the caller provides
   the rank tables): the cost model's best shape.  Used by the
   allocation-free entry point. */
int vsbd_plan_search(const vsbd_geom* h, int nitems, DGeom* out) {
  DGeom g;
  memset(&g, 0, sizeof(g));
  g.S = h->size; g.bpp = h->bpp; g.step = h->step;
  g.na = h->na; g.nb = h->nb; g.ax0 = h->ax0; g.by0 = h->by0;
  g.has_origin = h->has_origin; g.nstages = h->nstages;
  if (g.nstages > VSBD_MAX_STAGES) { set_msg("too many refinement stages"); return -1; }
  g.maxq = 1;
  for (int i = 0; i < g.nstages; i++) {
    g.st_r[i] = h->st_r[i];
    g.st_h[i] = h->st_h[i];
    int side = (2 * h->st_r[i]) / h->st_h[i] + 1;
    if (side * side > g.maxq) g.maxq = side * side;
  }
  g.limx = h->limx; g.limy = h->limy;
  TileCand cand[1];
  if (tile_candidates(g, nitems > 0 ? nitems : 1, 0, 0, 0, 0, cand, 1) < 1) {
    set_msg("no search tiling fits in shared memory");
    return -1;
  }
  *out = cand[0].g;
  return 0;
}

/* The fine pass on k_fine: timed against the search the detector would
   otherwise run (the sweep plan or the per-tile search), on the detector's
   own buffers and every fine field; kept when faster.  Cached per device and
   geometry.  VSB_NO_FINEWARP: never; VSB_FORCE_FINEWARP: always (tests). */
struct FineTune {
  int dev, S, step, na, nb, nstages, nitems, warps, T, ns;
};
static FineTune g_fwtune[64];
static int g_nfwtune = 0;

static int autotune_fine_warp(const GeomDev& gd, const DGeom* swplan, int sw_on,
                              const uint8_t* curr, const uint8_t* prev, int pitch,
                              const vsbd_item* d_items, int n, unsigned long long* keys,
                              unsigned* tickets, vsbd_result* d_res, unsigned* err,
                              cudaStream_t st, int* warps_out, int* t_out, int* ns_out) {
  *warps_out = 0;
  *t_out = 1;
  *ns_out = 1;
  const DGeom& g = gd.g;
  if (n <= 0 || !fw_supported(g) || getenv("VSB_NO_FINEWARP") || getenv("VSB_NO_AUTOTUNE"))
    return 0;
  const bool force = getenv("VSB_FORCE_FINEWARP") != NULL;
  if (!force && getenv("VSB_FORCE_SWEEP")) return 0; /* the sweep was asked for */
  TuneLock lock;
  const int dev = current_device();
  for (int i = 0; !force && i < g_nfwtune; i++) {
    const FineTune& e = g_fwtune[i];
    if (e.dev == dev && e.S == g.S && e.step == g.step && e.na == g.na && e.nb == g.nb &&
        e.nstages == g.nstages && e.nitems == n) {
      *warps_out = e.warps;
      *t_out = e.T;
      *ns_out = e.ns;
      return 0;
    }
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto time_of = [&](int warps, int T, int ns) -> float {
    auto one = [&]() {
      if (warps > 0)
        return launch_fine_warp(gd, warps, T, ns, curr, prev, pitch, d_items, n, d_res, st);
      return sw_on ? launch_sweep(*swplan, curr, prev, pitch, d_items, n, keys, tickets, d_res,
                                  err, st)
                   : launch_search(gd, curr, prev, pitch, d_items, n, keys, tickets, d_res, st);
    };
    if (one() < 0) {
      cudaGetLastError();
      return -1.f;
    }
    /* the best of three timings of five launches each */
    float best = 3.0e38f;
    for (int trial = 0; trial < 3; trial++) {
      cudaEventRecord(e0, st);
      for (int r = 0; r < 5; r++) one();
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      best = ms / 5 < best ? ms / 5 : best;
    }
    return best;
  };
  for (int w = 0; w < 3; w++) time_of(0, 1, 1); /* clocks up */
  const float base = time_of(0, 1, 1);
  int best_w = 0, best_t = 1, best_ns = 1;
  float best_ms = base > 0.f ? base : 3.0e38f;
  /* warp counts between the powers of two too: 6 warps fit 165 tasks (33
     lattice rows x 5 column groups) better than 8 */
  static const int kwarps[] = { 1, 2, 4, 6, 8, 10, 12, 16 };
  for (int T = 1; T <= 2; T *= 2)
    for (int ns = 1; ns <= 4; ns *= 2)
      for (int wi = 0; wi < (int)(sizeof(kwarps) / sizeof(kwarps[0])); wi++) {
        const int warps = kwarps[wi];
        /* at least a third of the threads have a task */
        if (32 * warps > 3 * fw_tasks(g, T, ns) + 32) continue;
        const float ms = time_of(warps, T, ns);
        if (getenv("VSB_DEBUG_TUNE"))
          fprintf(stderr,
                  "fine tuning S=%d items=%d: k_fine %d warps x %d rows x %d strips %.1f us "
                  "(current %.1f us)\n",
                  g.S, n, warps, T, ns, 1000.f * ms, 1000.f * base);
        if (ms > 0.f && (ms < best_ms || (force && best_w == 0))) {
          best_ms = ms;
          best_w = warps;
          best_t = T;
          best_ns = ns;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  *warps_out = best_w;
  *t_out = best_t;
  *ns_out = best_ns;
  if (!force && g_nfwtune < 64) {
    FineTune& t = g_fwtune[g_nfwtune++];
    t.dev = dev;
    t.S = g.S;
    t.step = g.step;
    t.na = g.na;
    t.nb = g.nb;
    t.nstages = g.nstages;
    t.nitems = n;
    t.warps = best_w;
    t.T = best_t;
    t.ns = best_ns;
  }
  return 0;
}

extern "C" void vsbd_set_error(const char* msg) { set_msg(msg); }

/* ------------------------------------------------------------------------ */
/* per-detector context                                                      */
/* ------------------------------------------------------------------------ */

struct vsbd_ctx {
  int dev;
  int W, H, bpp, blur, nch, pitch;
  int nc, nf;
  cudaStream_t st;
  uint8_t* d_raw;     /* input plane (blurred formats) */
  int blur_shape;     /* vector-blur tile shape (g_blur_shape), picked by timing */
  float blur_us;      /* its tuned time per frame */
  uint8_t* d_tmp;     /* row-pass buffer of the wide-window blur */
  uint8_t* d_buf[4];  /* blurred planes: slots of the current frame, the
                         previous one and up to two next ones (filled ahead
                         while the current frame's fine search runs) */
  int cur, prv;       /* slots of the current and the previous frame */
  int nxt[2], nnxt;   /* slots of next frames whose stage A is issued, in order */
  cudaStream_t st2;   /* the fine stage */
  cudaEvent_t ev_b;
  /* frames uploaded ahead of their stage A (vsbd_upload), on a copy stream
     of their own; allocated on first use */
  uint8_t* d_up[3];
  cudaStream_t st3;
  cudaEvent_t ev_up[3];
  int a_search, b_n;  /* the pending stages' search flag / item count */
  double thr_coarse;  /* contrast threshold of the coarse fields */
  int16_t* d_xy;      /* coarse x | coarse y | fine x | fine y */
  GeomDev gc, gf;
  /* the persistent sweep, where it beats the per-tile search (autotuned):
     plans of the coarse and the fine fields, on flags, and the error words
     its bounded waits raise ([0] coarse, [1] fine; mapped pinned memory) */
  DGeom swc, swf;
  int sw_c, sw_f;
  int fw_f, fw_warps, fw_t, fw_ns; /* fine pass on k_fine: warps per item, lattice rows per
                                      thread, field-row strips */
  unsigned* h_swerr;
  unsigned* d_swerr;
  vsbd_item* d_citems;
  vsbd_item* d_fitems;
  unsigned long long* d_keys;   /* coarse nc, then fine nf */
  unsigned* d_tickets;
  int mode;                     /* 0 dense search, 1 pruned search */
  GeomDev gcp, gfp;             /* partial-pass geometry (first rows of the field) */
  uint8_t* d_skip;              /* coarse fields never selected (contrast) */
  /* blur and field min/max in one launch (k_blurmm): per 128x16 warp block
     the fields meeting it, the running min/max of every field, the ticket */
  int bm_on, bm_nbx, bm_grid_x, bm_grid_y;
  int* d_bm_lofs;
  uint2* d_bm_list;
  unsigned* d_bm_acc;
  unsigned* d_bm_ticket;
  unsigned* d_part;             /* partial sums, per item per lattice point */
  int* d_lists;                 /* survivors, per item */
  int* d_counts;
  int* d_boxes;                 /* survivors' lattice bounding box, per item */
  uint8_t* d_out;               /* minmax | coarse results | coarse proposal flags |
                                   fine results | fine proposal flags */
  uint8_t* h_out;               /* pinned mirror of d_out */
  /* three such blocks: every stage A moves to the next one, so up to two
     frames' stage A can run while the host still reads an earlier frame's
     results (d_out/h_out point at the latest block) */
  uint8_t* d_outs[3];
  uint8_t* h_outs[3];
  int obuf;
  /* issued stage A's not yet collected, oldest first: their output block,
     search flag and completion event */
  int aq_blk[3], aq_search[3], naq;
  cudaEvent_t ev_ablk[3];
  uint8_t* b_hout;              /* host block the pending stage B copies into (a
                                   stage A may switch d_out/h_out meanwhile) */
  vsbd_item* h_items;           /* pinned staging of fine items */
  size_t off_coarse, off_cfb, off_fine, off_ffb, out_bytes;
  /* learned search proposal */
  void* d_pn;                   /* network parameters: bf16 weights | f32 biases */
  PNSearch pn;
  float pn_match_bound;         /* trusted refined SAD per field pixel */
  int pn_on, pn_verify;
  int pn_fine_net;              /* fine fields: 1 network proposal, 0 the coarse model's
                                   prediction (zero residual) */
  float pn_fine_radius;         /* window radius of the fine fields (< 0: the default) */
  int pn_passes;                /* coarse fields: 1 network pass, 2 with a global prior */
  vsbd_item* d_citems2;         /* second-pass items (coarse fields, prior as offset) */
  short2* d_prior;              /* per coarse field, the rounded global-model displacement */
  float* d_pout;                /* network outputs [nc + nf][3] */
  vsbd_result* d_vres;          /* verify: full-search results, coarse then fine */
  vsbd_result* h_vres;
  GeomDev gcf, gff;             /* full-search tilings for the few items that fall back */
  int fb_last[2];               /* items that fell back in the previous frame: coarse, fine */
  int* d_fbl;                   /* fallback count, then the fallback item list */
  long long pn_stats[8];        /* searched, fell back, verified, identical; then
                                   coarse searched / fell back, fine searched / fell back */
  /* training-data log */
  uint8_t* log_in;
  PNLabel* log_lab;
  long log_cap, log_n;
  long launches;
  int timing;                   /* record CUDA events around each kernel */
  cudaEvent_t ev[VSBD_NKT][2];
  double kt_ms[VSBD_NKT];
  long kt_n[VSBD_NKT];
  int kt_pending[VSBD_NKT];
};

/* per-kernel event pairs on the detector's stream; read after the sync */
static void kt_begin(vsbd_ctx* c, int k, cudaStream_t st) {
  if (c->timing) cudaEventRecord(c->ev[k][0], st);
}
static void kt_end(vsbd_ctx* c, int k, cudaStream_t st) {
  if (c->timing) {
    cudaEventRecord(c->ev[k][1], st);
    c->kt_pending[k] = 1;
  }
}
static void kt_collect(vsbd_ctx* c) {
  if (!c->timing) return;
  for (int k = 0; k < VSBD_NKT; k++)
    if (c->kt_pending[k]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->ev[k][0], c->ev[k][1]) == cudaSuccess) {
        c->kt_ms[k] += ms;
        c->kt_n[k]++;
      }
      c->kt_pending[k] = 0;
    }
}

extern "C" int vsbd_set_timing(vsbd_ctx* c, int on) {
  if (!c) return -1;
  CK(cudaSetDevice(c->dev));
  if (on && !c->ev[0][0])
    for (int k = 0; k < VSBD_NKT; k++) {
      CK(cudaEventCreate(&c->ev[k][0]));
      CK(cudaEventCreate(&c->ev[k][1]));
    }
  c->timing = on;
  for (int k = 0; k < VSBD_NKT; k++) { c->kt_ms[k] = 0; c->kt_n[k] = 0; c->kt_pending[k] = 0; }
  return 0;
}

extern "C" int vsbd_kernel_times(const vsbd_ctx* c, double* ms, long* n) {
  if (!c) return -1;
  for (int k = 0; k < VSBD_NKT; k++) { ms[k] = c->kt_ms[k]; n[k] = c->kt_n[k]; }
  return 0;
}

static size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

extern "C" int vsbd_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

extern "C" void vsbd_destroy(vsbd_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->st2) cudaStreamSynchronize(c->st2);
  for (int k = 0; k < VSBD_NKT; k++)
    if (c->ev[k][0]) { cudaEventDestroy(c->ev[k][0]); cudaEventDestroy(c->ev[k][1]); }
  cudaFree(c->d_raw);
  cudaFree(c->d_tmp);
  for (int k = 0; k < 4; k++) cudaFree(c->d_buf[k]);
  if (c->ev_b) cudaEventDestroy(c->ev_b);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st3) {
    cudaStreamSynchronize(c->st3);
    cudaStreamDestroy(c->st3);
  }
  for (int k = 0; k < 3; k++) {
    cudaFree(c->d_up[k]);
    if (c->ev_up[k]) cudaEventDestroy(c->ev_up[k]);
  }
  cudaFree(c->d_xy);
  cudaFree(c->d_citems);
  cudaFree(c->d_fitems);
  cudaFree(c->d_keys);
  cudaFree(c->d_tickets);
  for (int k = 0; k < 3; k++) {
    cudaFree(c->d_outs[k]);
    if (c->ev_ablk[k]) cudaEventDestroy(c->ev_ablk[k]);
  }
  cudaFree(c->d_skip);
  cudaFree(c->d_bm_lofs);
  cudaFree(c->d_bm_list);
  cudaFree(c->d_bm_acc);
  cudaFree(c->d_bm_ticket);
  cudaFree(c->d_part);
  cudaFree(c->d_lists);
  cudaFree(c->d_counts);
  cudaFree(c->d_boxes);
  for (int k = 0; k < 3; k++)
    if (c->h_outs[k]) cudaFreeHost(c->h_outs[k]);
  if (c->h_items) cudaFreeHost(c->h_items);
  if (c->h_swerr) cudaFreeHost(c->h_swerr);
  cudaFree(c->d_pn);
  cudaFree(c->d_pout);
  cudaFree(c->d_fbl);
  cudaFree(c->d_citems2);
  cudaFree(c->d_prior);
  cudaFree(c->d_vres);
  if (c->h_vres) cudaFreeHost(c->h_vres);
  geom_free(&c->gc);
  geom_free(&c->gf);
  /* gcp/gfp share gc/gf's tables */
  if (c->st) cudaStreamDestroy(c->st);
  free(c);
}

/* The vector blur's tile shape for a plane geometry: every shape that
   serves the window is timed on the detector's own planes and the fastest
   kept; cached per (device, width, height, box size). */
struct BlurTune {
  int dev, W, H, size, shape;
  float us;
};
static BlurTune g_blurtune[64];
static int g_nblurtune = 0;

/* Every kernel of a detector's frame prefers the largest shared-memory
   carveout: the search kernels need it, and a small-memory kernel between
   them (blur, min/max) that asked for a different split would make the SMs
   reconfigure between launches.  Set once per process (the attribute
   belongs to the function, per device context). */
static void prefer_shared_carveout(void) {
  static int done[VSB_MAX_DEVICES];
  const int dev = current_device();
  if (__atomic_load_n(&done[dev], __ATOMIC_RELAXED)) return;
  const int pref = cudaSharedmemCarveoutMaxShared;
#define VSB_CARVE(fn) cudaFuncSetAttribute((const void*)(fn), cudaFuncAttributePreferredSharedMemoryCarveout, pref);
#define VSB_CARVE_BLUR(BW, BH) \
  VSB_CARVE((k_blur_fast<1, BW, BH>)) VSB_CARVE((k_blur_fast<2, BW, BH>)) VSB_CARVE((k_blur_fast<3, BW, BH>)) \
  VSB_CARVE((k_blur_fast<4, BW, BH>)) VSB_CARVE((k_blur_fast<5, BW, BH>)) VSB_CARVE((k_blur_fast<6, BW, BH>)) \
  VSB_CARVE((k_blur_fast<7, BW, BH>)) VSB_CARVE((k_blur_fast<8, BW, BH>))
  VSB_CARVE_BLUR(256, 32)
  VSB_CARVE_BLUR(128, 16)
  VSB_CARVE_BLUR(128, 32)
  VSB_CARVE_BLUR(64, 32)
  VSB_CARVE(k_minmax_planar)
  VSB_CARVE(k_minmax)
  VSB_CARVE(k_blur)
#undef VSB_CARVE_BLUR
#undef VSB_CARVE
  cudaGetLastError(); /* a hint the device may not take is not an error */
  __atomic_store_n(&done[dev], 1, __ATOMIC_RELAXED);
}

static int autotune_blur(vsbd_ctx* c, const uint8_t* src, uint8_t* dst) {
  c->blur_shape = 0;
  c->blur_us = 0.f;
  const int half = c->blur / 2;
  if (c->blur < 2 || half > 8 || getenv("VSB_NO_AUTOTUNE")) return 0;
  TuneLock lock;
  const int dev = current_device();
  for (int i = 0; i < g_nblurtune; i++)
    if (g_blurtune[i].dev == dev && g_blurtune[i].W == c->W && g_blurtune[i].H == c->H &&
        g_blurtune[i].size == c->blur) {
      c->blur_shape = g_blurtune[i].shape;
      c->blur_us = g_blurtune[i].us;
      return 0;
    }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int round = 0; round < 3; round++)
    for (int s = 0; s < VSB_BLUR_SHAPES; s++) {
      if (!blur_shape_ok(s, half)) continue;
      launch_blur(src, c->pitch, dst, c->pitch, c->W, c->H, c->blur, c->d_tmp, c->pitch, c->st, s);
      cudaEventRecord(e0, c->st);
      for (int r = 0; r < 10; r++)
        launch_blur(src, c->pitch, dst, c->pitch, c->W, c->H, c->blur, c->d_tmp, c->pitch, c->st,
                    s);
      cudaEventRecord(e1, c->st);
      if (cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      /* the first round warms the clocks up */
      if (round > 0 && ms < best) {
        best = ms;
        c->blur_shape = s;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_err("blur tile tuning", le);
      return -1;
    }
  }
  c->blur_us = best < 1e29f ? 100.f * best : 0.f;
  if (g_nblurtune < 64) {
    BlurTune& b = g_blurtune[g_nblurtune++];
    b.dev = dev; b.W = c->W; b.H = c->H; b.size = c->blur; b.shape = c->blur_shape; b.us = c->blur_us;
  }
  return 0;
}

/* search strategy of detectors created from now on (-1: environment) */
static int g_default_mode = -1;
extern "C" void vsbd_set_default_search_mode(int pruned) { g_default_mode = pruned < 0 ? -1 : (pruned ? 1 : 0); }

/* rows of a field the pruned search's partial pass sums: a quarter, at
   least 4 (on blurred content this leaves a few percent of the candidates) */
static int partial_rows(int S) {
  int r = S / 4;
  return r < 4 ? (S < 4 ? S : 4) : r;
}

extern "C" int vsbd_set_search_mode(vsbd_ctx* c, int pruned) {
  if (!c) return -1;
  c->mode = pruned ? 1 : 0;
  return 0;
}

/* The fused prefilter's tables (planar frames, box half-width 1..4): for
   every 128-column x 16-row warp block of the frame, the fields whose
   square meets it, with the block's column range and row mask of the
   intersection; the fields' min/max accumulators start at (255.., 0). */
static int blurmm_setup(vsbd_ctx* c, const int16_t* cx, const int16_t* cy, const int16_t* fx,
                        const int16_t* fy) {
  const int half = c->blur / 2;
  const int nfield = c->nc + c->nf;
  c->bm_on = 0;
  /* VSB_NO_BLURMM: the two-launch prefilter (blur, then field min/max) */
  if (c->blur < 2 || half < 1 || half > BM_MAXHALF || c->bpp != 1 || c->nch != 1 ||
      nfield > 65535 || c->W < 4 || getenv("VSB_NO_BLURMM"))
    return 0;
  {
    /* the kernel divides by the multiply-high alone */
    BlurDiv dv;
    make_div(c->blur, half, &dv);
    if (!dv.exact) return 0;
  }
  const int nbx = (c->W + BM_COLS - 1) / BM_COLS;
  const int nbands = (c->H + BM_ROWS - 1) / BM_ROWS;
  const int gy = (nbands + BM_WARPS - 1) / BM_WARPS;
  const size_t nwb = (size_t)gy * BM_WARPS * nbx; /* every warp of the grid has a slot */
  std::vector<std::vector<uint2>> per(nwb);
  for (int f = 0; f < nfield; f++) {
    const bool coarse = f < c->nc;
    const int S = coarse ? c->gc.g.S : c->gf.g.S;
    const int x = coarse ? cx[f] : fx[f - c->nc];
    const int y = coarse ? cy[f] : fy[f - c->nc];
    const int xa = x - S / 2, ya = y - S / 2;
    if (xa < 0 || ya < 0 || xa + S > c->W || ya + S > c->H) return 0; /* not expected */
    for (int b = ya / BM_ROWS; b * BM_ROWS < ya + S; b++) {
      unsigned rows = 0;
      for (int r = 0; r < BM_ROWS; r++) {
        const int yy = b * BM_ROWS + r;
        if (yy >= ya && yy < ya + S) rows |= 1u << r;
      }
      for (int bx = xa / BM_COLS; bx * BM_COLS < xa + S; bx++) {
        const int lo = std::max(xa, bx * BM_COLS) - bx * BM_COLS;
        const int hi = std::min(xa + S, (bx + 1) * BM_COLS) - bx * BM_COLS;
        per[(size_t)b * nbx + bx].push_back(
            make_uint2((unsigned)f | ((unsigned)lo << 16) | ((unsigned)hi << 24), rows));
      }
    }
  }
  std::vector<int> ofs(nwb + 1, 0);
  std::vector<uint2> list;
  for (size_t i = 0; i < nwb; i++) {
    ofs[i] = (int)list.size();
    list.insert(list.end(), per[i].begin(), per[i].end());
  }
  ofs[nwb] = (int)list.size();
  std::vector<unsigned> acc(2 * (size_t)nfield);
  for (int f = 0; f < nfield; f++) {
    acc[2 * f] = 0xffffffffu;
    acc[2 * f + 1] = 0u;
  }
  CK(cudaMalloc(&c->d_bm_lofs, sizeof(int) * (nwb + 1)));
  CK(cudaMalloc(&c->d_bm_list, sizeof(uint2) * (list.size() + 1)));
  CK(cudaMalloc(&c->d_bm_acc, sizeof(unsigned) * (acc.size() + 2)));
  CK(cudaMalloc(&c->d_bm_ticket, sizeof(unsigned)));
  CK(cudaMemcpy(c->d_bm_lofs, ofs.data(), sizeof(int) * (nwb + 1), cudaMemcpyHostToDevice));
  if (!list.empty())
    CK(cudaMemcpy(c->d_bm_list, list.data(), sizeof(uint2) * list.size(), cudaMemcpyHostToDevice));
  if (!acc.empty())
    CK(cudaMemcpy(c->d_bm_acc, acc.data(), sizeof(unsigned) * acc.size(), cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_bm_ticket, 0, sizeof(unsigned)));
  c->bm_nbx = nbx;
  c->bm_grid_x = nbx;
  c->bm_grid_y = gy;
  c->bm_on = 1;
  return 0;
}

/* k_blurmm over plane `src` into `cur`: the blurred plane, the (min, max)
   byte pairs of every field into c->d_out and the coarse contrast flags */
static int launch_blurmm(vsbd_ctx* c, const uint8_t* src, int sp, uint8_t* cur, uint8_t* skip,
                         cudaStream_t st) {
  BMArgs A;
  A.src = src;
  A.sp = sp;
  A.dst = cur;
  A.dp = c->pitch;
  A.W = c->W;
  A.H = c->H;
  make_div(c->blur, c->blur / 2, &A.dv);
  A.lofs = c->d_bm_lofs;
  A.list = c->d_bm_list;
  A.nbx = c->bm_nbx;
  A.acc = c->d_bm_acc;
  A.ticket = c->d_bm_ticket;
  A.nc = c->nc;
  A.nfields = c->nc + c->nf;
  A.out = c->d_out;
  A.thr = c->thr_coarse;
  A.skip = skip;
  const dim3 grid(c->bm_grid_x, c->bm_grid_y);
  switch (c->blur / 2) {
    case 1: k_blurmm<1><<<grid, 32 * BM_WARPS, 0, st>>>(A); break;
    case 2: k_blurmm<2><<<grid, 32 * BM_WARPS, 0, st>>>(A); break;
    case 3: k_blurmm<3><<<grid, 32 * BM_WARPS, 0, st>>>(A); break;
    case 4: k_blurmm<4><<<grid, 32 * BM_WARPS, 0, st>>>(A); break;
    default: set_msg("k_blurmm: unsupported box size"); return -1;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_err("k_blurmm launch", e); return -1; }
  c->launches++;
  count_launches(1);
  return 0;
}

extern "C" int vsbd_create(vsbd_ctx** out, int W, int H, int bpp, int blur_size, int channels,
                           const vsbd_geom* coarse, const int16_t* cx, const int16_t* cy, int nc,
                           const vsbd_geom* fine, const int16_t* fx, const int16_t* fy, int nf,
                           double coarse_threshold) {
  *out = NULL;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev < 1) {
    set_msg("no CUDA device available (the GPU path has no CPU fallback)");
    return -1;
  }
  vsbd_ctx* c = (vsbd_ctx*)calloc(1, sizeof(vsbd_ctx));
  CK(cudaGetDevice(&c->dev));
  c->W = W; c->H = H; c->bpp = bpp; c->blur = blur_size; c->nch = channels;
  c->nc = nc; c->nf = nf;
  c->thr_coarse = coarse_threshold;
  c->pitch = (int)(((size_t)W * bpp + 127) & ~(size_t)127);
  size_t plane = (size_t)c->pitch * H + 256; /* slack: word reads past a row end */
#define CKC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { set_err(#call, e_); vsbd_destroy(c); return -1; } } while (0)
  CKC(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  if (blur_size >= 2) CKC(cudaMalloc(&c->d_raw, plane));
  if (blur_size >= 2 && blur_size / 2 > BT_MAXHALF) CKC(cudaMalloc(&c->d_tmp, plane));
  for (int k = 0; k < 4; k++) {
    CKC(cudaMalloc(&c->d_buf[k], plane));
    CKC(cudaMemset(c->d_buf[k], 0, plane));
  }
  c->cur = 0;
  c->prv = 1;
  c->nnxt = 0;
  c->pn_fine_radius = -1.f;
  c->pn_passes = 1;
  CKC(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
  CKC(cudaEventCreateWithFlags(&c->ev_b, cudaEventDisableTiming));
  CKC(cudaMalloc(&c->d_xy, sizeof(int16_t) * 2 * (nc + nf) + 16));
  CKC(cudaMemcpy(c->d_xy, cx, sizeof(int16_t) * nc, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + nc, cy, sizeof(int16_t) * nc, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + 2 * nc, fx, sizeof(int16_t) * nf, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + 2 * nc + nf, fy, sizeof(int16_t) * nf, cudaMemcpyHostToDevice));
  if (geom_upload(coarse, nc, 0, &c->gc) != 0) { vsbd_destroy(c); return -1; }
  if (geom_upload(fine, nf, 0, &c->gf) != 0) { vsbd_destroy(c); return -1; }
  /* the pruned search's partial pass sums the first rows of each field */
  c->mode = g_default_mode >= 0 ? g_default_mode : (getenv("VSB_PRUNED_SEARCH") ? 1 : 0);
  c->gcp = c->gc;
  c->gfp = c->gf;
  c->gcp.g.rows = partial_rows(c->gc.g.S);
  c->gfp.g.rows = partial_rows(c->gf.g.S);
  {
    TileCand tc[1];
    if (tile_candidates(c->gcp.g, nc, 0, 0, 0, 0, tc, 1) < 1 ||
        (c->gcp.g = tc[0].g, tile_candidates(c->gfp.g, nf, 0, 0, 0, 0, tc, 1) < 1)) {
      set_msg("no partial-pass tiling fits in shared memory");
      vsbd_destroy(c);
      return -1;
    }
    c->gfp.g = tc[0].g;
    c->gcp.smem = tile_layout(c->gcp.g).total;
    c->gfp.smem = tile_layout(c->gfp.g).total;
  }
  {
    size_t lat = (size_t)c->gc.g.na * c->gc.g.nb * nc;
    size_t latf = (size_t)c->gf.g.na * c->gf.g.nb * nf;
    if (latf > lat) lat = latf;
    CKC(cudaMalloc(&c->d_part, sizeof(unsigned) * (lat + 1)));
    CKC(cudaMalloc(&c->d_lists, sizeof(int) * (lat + 1)));
    CKC(cudaMalloc(&c->d_counts, sizeof(int) * (nc + nf + 1)));
    CKC(cudaMalloc(&c->d_boxes, sizeof(int) * 4 * (nc + nf + 1)));
    CKC(cudaMalloc(&c->d_skip, nc + 1));
    CKC(cudaMemset(c->d_skip, 0, nc + 1));
  }
  if (blurmm_setup(c, cx, cy, fx, fy) != 0) { vsbd_destroy(c); return -1; }
  /* coarse items: every coarse field, no offset */
  {
    vsbd_item* it = (vsbd_item*)malloc(sizeof(vsbd_item) * (nc + 1));
    for (int i = 0; i < nc; i++) { it[i].x = cx[i]; it[i].y = cy[i]; it[i].ox = 0; it[i].oy = 0; }
    CKC(cudaMalloc(&c->d_citems, sizeof(vsbd_item) * (nc + 1)));
    cudaError_t e3 = cudaMemcpy(c->d_citems, it, sizeof(vsbd_item) * nc, cudaMemcpyHostToDevice);
    free(it);
    CKC(e3);
  }
  CKC(cudaMalloc(&c->d_fitems, sizeof(vsbd_item) * (nf + 1)));
  CKC(cudaMallocHost(&c->h_items, sizeof(vsbd_item) * (nf + 1)));
  CKC(cudaMalloc(&c->d_keys, sizeof(unsigned long long) * (nc + nf + 2)));
  CKC(cudaMemset(c->d_keys, 0xff, sizeof(unsigned long long) * (nc + nf + 2)));
  CKC(cudaMalloc(&c->d_tickets, sizeof(unsigned) * (nc + nf + 2)));
  CKC(cudaMemset(c->d_tickets, 0, sizeof(unsigned) * (nc + nf + 2)));
  c->off_coarse = align16((size_t)(nc + nf) * channels * 2);
  c->off_cfb = c->off_coarse + align16(sizeof(vsbd_result) * (nc + 1));
  c->off_fine = c->off_cfb + align16((size_t)nc + 1);
  c->off_ffb = c->off_fine + align16(sizeof(vsbd_result) * (nf + 1));
  c->out_bytes = c->off_ffb + align16((size_t)nf + 1);
  for (int k = 0; k < 3; k++) {
    CKC(cudaMalloc(&c->d_outs[k], c->out_bytes));
    CKC(cudaMallocHost(&c->h_outs[k], c->out_bytes));
    CKC(cudaEventCreateWithFlags(&c->ev_ablk[k], cudaEventDisableTiming));
  }
  c->obuf = 0;
  c->naq = 0;
  c->d_out = c->d_outs[0];
  c->h_out = c->h_outs[0];
  /* fine items for tuning: every fine field without offset */
  {
    vsbd_item* it = (vsbd_item*)malloc(sizeof(vsbd_item) * (nf + 1));
    for (int i = 0; i < nf; i++) { it[i].x = fx[i]; it[i].y = fy[i]; it[i].ox = 0; it[i].oy = 0; }
    cudaError_t e3 = cudaMemcpy(c->d_fitems, it, sizeof(vsbd_item) * nf, cudaMemcpyHostToDevice);
    free(it);
    CKC(e3);
  }
  if (autotune_tiling(&c->gc, c->d_buf[0], c->d_buf[1], c->pitch, c->d_citems, nc, c->d_keys,
                      c->d_tickets, (vsbd_result*)(c->d_out + c->off_coarse), c->st) != 0 ||
      autotune_tiling(&c->gf, c->d_buf[0], c->d_buf[1], c->pitch, c->d_fitems, nf, c->d_keys + nc,
                      c->d_tickets + nc, (vsbd_result*)(c->d_out + c->off_fine), c->st) != 0 ||
      autotune_tiling(&c->gcp, c->d_buf[0], c->d_buf[1], c->pitch, c->d_citems, nc, NULL, NULL,
                      NULL, c->st, c->d_part) != 0 ||
      autotune_tiling(&c->gfp, c->d_buf[0], c->d_buf[1], c->pitch, c->d_fitems, nf, NULL, NULL,
                      NULL, c->st, c->d_part) != 0) {
    vsbd_destroy(c);
    return -1;
  }
  prefer_shared_carveout();
  if (autotune_blur(c, c->d_raw ? c->d_raw : c->d_buf[0], c->d_buf[2]) != 0) {
    vsbd_destroy(c);
    return -1;
  }
  /* error words: [0] coarse sweep, [1] fine sweep, [2] proposal network */
  CKC(cudaHostAlloc(&c->h_swerr, 3 * sizeof(unsigned), cudaHostAllocMapped));
  c->h_swerr[0] = c->h_swerr[1] = c->h_swerr[2] = 0;
  CKC(cudaHostGetDevicePointer((void**)&c->d_swerr, c->h_swerr, 0));
  if (autotune_sweep(c->gc, c->d_buf[0], c->d_buf[1], c->pitch, c->d_citems, nc, c->d_keys,
                     c->d_tickets, (vsbd_result*)(c->d_out + c->off_coarse), c->d_swerr,
                     c->h_swerr, c->st, &c->swc, &c->sw_c) != 0 ||
      autotune_sweep(c->gf, c->d_buf[0], c->d_buf[1], c->pitch, c->d_fitems, nf,
                     c->d_keys + nc, c->d_tickets + nc, (vsbd_result*)(c->d_out + c->off_fine),
                     c->d_swerr + 1, c->h_swerr + 1, c->st, &c->swf, &c->sw_f) != 0) {
    vsbd_destroy(c);
    return -1;
  }
  if (c->bpp == 1 && c->nch == 1 &&
      autotune_fine_warp(c->gf, &c->swf, c->sw_f, c->d_buf[0], c->d_buf[1], c->pitch, c->d_fitems,
                         nf, c->d_keys + nc, c->d_tickets + nc,
                         (vsbd_result*)(c->d_out + c->off_fine), c->d_swerr + 1, c->st,
                         &c->fw_warps, &c->fw_t, &c->fw_ns) != 0) {
    vsbd_destroy(c);
    return -1;
  }
  c->fw_f = c->fw_warps > 0;
  CKC(cudaStreamSynchronize(c->st));
#undef CKC
  *out = c;
  return 0;
}

/* whether the fine fields take the narrowed search (the network's, or a
   window around the coarse model's prediction); by default they take the
   exact dense search of the plain detector */
static bool fine_narrowed(const vsbd_ctx* c) {
  return c->pn_on && (c->pn_fine_net || c->pn_fine_radius >= 0.f);
}

/* The proposal path of one field set: network, narrowed search, full
   search of the items that fell back (and, when verifying, the full search
   of every item into d_vres + base).  fbl: this field set's fallback count
   and list. */
static int learned_search(vsbd_ctx* c, const GeomDev& gd, const GeomDev& gfull, uint8_t* cur,
                          uint8_t* prv, cudaStream_t st, const vsbd_item* items, int n, int base,
                          const uint8_t* skip, unsigned long long* keys, unsigned* tickets,
                          vsbd_result* res, uint8_t* fb, int* fbl) {
  if (n <= 0) return 0;
  float* pout = NULL;
  const short2* prior = NULL;
  if (base == 0 || c->pn_fine_net) {
    pout = c->d_pout + (size_t)3 * base;
    kt_begin(c, VSBD_KT_PNET, st);
    if (vsbpn_infer(c->d_pn, cur, prv, c->pitch, c->W, c->H, items, NULL, n, pout,
                    c->d_swerr + 2, st) < 0)
      return -1;
    c->launches++;
    count_launches(1);
    if (base == 0 && c->pn_passes == 2) {
      /* second pass: every coarse field's crop re-centred on the frame's
         global motion model from the first pass; the proposal is the model
         plus the second prediction */
      if (vsbpn_prior(items, pout, n, c->pn.scale, c->pn.conf_min, skip, c->W, c->H, c->d_citems2,
                      c->d_prior, st) < 0 ||
          vsbpn_infer(c->d_pn, cur, prv, c->pitch, c->W, c->H, c->d_citems2, NULL, n, pout,
                      c->d_swerr + 2, st) < 0)
        return -1;
      prior = c->d_prior;
      c->launches += 2;
      count_launches(2);
    }
    kt_end(c, VSBD_KT_PNET, st);
  }
  const int kt = base == 0 ? VSBD_KT_COARSE : VSBD_KT_FINE;
  kt_begin(c, kt, st);
  /* the SAD bound scales with the field's pixel count */
  PNSearch ps = c->pn;
  if (base != 0) /* fine fields: 4 px around the coarse model, the blob's radius around the network */
    ps.radius = c->pn_fine_radius >= 0.f ? c->pn_fine_radius : c->pn.radius;
  const double bound = (double)c->pn_match_bound * gd.g.S * gd.g.S;
  ps.sad_bound = bound >= 4294967295.0 ? 0xffffffffu : (unsigned)bound;
  CK(cudaMemsetAsync(fbl, 0, sizeof(int), st));
  if (vsbpn_narrow(gd.g, cur, prv, c->pitch, items, n, pout, prior, ps, skip, res, fb, fbl, fbl + 1,
                   st) < 0)
    return -1;
  kt_end(c, kt, st);
  kt_begin(c, VSBD_KT_FALLBACK, st);
  int nl = launch_list(gfull, cur, prv, c->pitch, items, n, fbl, fbl + 1, keys, tickets, res, st);
  if (nl < 0) return -1;
  kt_end(c, VSBD_KT_FALLBACK, st);
  c->launches += 1 + nl;
  count_launches(1 + nl);
  if (c->pn_verify) {
    int nv = launch_search(gd, cur, prv, c->pitch, items, n, keys, tickets, c->d_vres + base, st);
    if (nv < 0) return -1;
    c->launches += nv;
    count_launches(nv);
  }
  return 0;
}

/* counts of one stage after its results reached the host */
static void proposal_tally(vsbd_ctx* c, const uint8_t* fb, const vsbd_result* res,
                           const vsbd_result* vres, int n, int kind) {
  c->fb_last[kind] = 0;
  for (int i = 0; i < n; i++) {
    if (fb[i] == PN_FB_FULL) c->fb_last[kind]++;
    if (fb[i] == PN_FB_UNUSED) continue;
    c->pn_stats[0]++;
    c->pn_stats[4 + 2 * kind]++;
    if (fb[i] == PN_FB_FULL) {
      c->pn_stats[1]++;
      c->pn_stats[5 + 2 * kind]++;
    }
    if (c->pn_verify && vres) {
      c->pn_stats[2]++;
      if (res[i].sad == vres[i].sad && res[i].tx == vres[i].tx && res[i].ty == vres[i].ty &&
          res[i].ok == vres[i].ok)
        c->pn_stats[3]++;
    }
  }
}

/* appends the network inputs and full-search labels of n items to the log */
static int log_items(vsbd_ctx* c, uint8_t* cur, uint8_t* prv, cudaStream_t st,
                     const vsbd_item* items, int n, int kind, const vsbd_result* res,
                     const uint8_t* skip) {
  if (n <= 0 || c->log_n + n > c->log_cap) return 0;
  if (vsbpn_crops(cur, prv, c->pitch, c->W, c->H, items, n, c->log_in + (size_t)c->log_n * 4096,
                  st) < 0 ||
      vsbpn_labels(res, skip, n, kind, c->log_lab + c->log_n, st) < 0)
    return -1;
  c->launches += 2;
  count_launches(2);
  c->log_n += n;
  return 0;
}

/* Stage A of a frame whose blurred plane goes to slot ci and whose search
   runs against slot pi, enqueued on the detector's first stream, ending with
   the results' copy to the host and the stage-A event. */
static int stage_a_issue(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev,
                         int pitch, int search, int ci, int pi) {
  const int rowbytes = c->W * c->bpp;
  cudaStream_t st = c->st;
  uint8_t* cur = c->d_buf[ci];
  uint8_t* prv = c->d_buf[pi];
  if (c->naq >= 3) {
    set_msg("three stage A's already in flight");
    return -1;
  }
  c->a_search = search;
  /* this stage's results go to the next output block: the two earlier
     frames' stay readable meanwhile */
  c->obuf = (c->obuf + 1) % 3;
  c->d_out = c->d_outs[c->obuf];
  c->h_out = c->h_outs[c->obuf];
  /* the contrast flags steer the pruned and the proposal searches and mark
     the training log's unused fields */
  uint8_t* skip = (c->mode || c->pn_on || c->log_in) ? c->d_skip : NULL;
  bool fused = false; /* blur and field min/max in one launch */
  if (c->blur >= 2) {
    const uint8_t* src = dev;
    int sp = pitch;
    if (!dev) {
      CK(cudaMemcpy2DAsync(c->d_raw, c->pitch, host, linesize, rowbytes, c->H,
                           cudaMemcpyHostToDevice, st));
      count_h2d((size_t)rowbytes * c->H);
      src = c->d_raw;
      sp = c->pitch;
    }
    fused = c->bm_on &&
            ((((uintptr_t)src | (uintptr_t)sp | (uintptr_t)cur | (uintptr_t)c->pitch) & 3) == 0);
    kt_begin(c, VSBD_KT_BLUR, st);
    if (fused) {
      if (launch_blurmm(c, src, sp, cur, skip, st) != 0) return -1;
    } else {
      int nb = launch_blur(src, sp, cur, c->pitch, c->W, c->H, c->blur, c->d_tmp, c->pitch, st,
                           c->blur_shape);
      c->launches += nb;
      count_launches(nb);
    }
    kt_end(c, VSBD_KT_BLUR, st);
    CK(cudaGetLastError());
  } else {
    if (dev)
      CK(cudaMemcpy2DAsync(cur, c->pitch, dev, pitch, rowbytes, c->H, cudaMemcpyDeviceToDevice, st));
    else {
      CK(cudaMemcpy2DAsync(cur, c->pitch, host, linesize, rowbytes, c->H, cudaMemcpyHostToDevice, st));
      count_h2d((size_t)rowbytes * c->H);
    }
  }
  if (search) {
    int S = c->gc.g.S;
    vsbd_result* cres = (vsbd_result*)(c->d_out + c->off_coarse);
    if (!fused) kt_begin(c, VSBD_KT_MINMAX, st);
    if (fused) {
      /* done by k_blurmm */
    } else if (c->bpp == 1 && c->nch == 1) {
      k_minmax_planar<<<c->nc + c->nf, 256, 0, st>>>(cur, c->pitch, c->d_xy, c->nc, c->nf, S,
                                                     c->gf.g.S, c->d_out, c->thr_coarse, skip);
      c->launches++;
      count_launches(1);
    } else {
      k_minmax<<<c->nc, 256, 0, st>>>(cur, c->pitch, c->d_xy, c->d_xy + c->nc, S, c->bpp, c->nch,
                                      c->d_out, c->thr_coarse, skip);
      c->launches++;
      count_launches(1);
      if (c->nf > 0) {
        k_minmax<<<c->nf, 256, 0, st>>>(cur, c->pitch, c->d_xy + 2 * c->nc,
                                        c->d_xy + 2 * c->nc + c->nf, c->gf.g.S, c->bpp, c->nch,
                                        c->d_out + (size_t)c->nc * c->nch * 2, 0.0, NULL);
        c->launches++;
        count_launches(1);
      }
    }
    if (!fused) kt_end(c, VSBD_KT_MINMAX, st);
    if (c->pn_on) {
      if (learned_search(c, c->gc, c->fb_last[0] >= 8 ? c->gc : c->gcf, cur, prv, st, c->d_citems,
                         c->nc, 0, skip, c->d_keys, c->d_tickets, cres, c->d_out + c->off_cfb,
                         c->d_fbl) != 0)
        return -1;
    } else {
      kt_begin(c, VSBD_KT_COARSE, st);
      int nl = c->mode ? launch_pruned(c->gc, c->gcp, cur, prv, c->pitch, c->d_citems, c->nc,
                                       c->d_skip, c->d_part, c->d_counts, c->d_lists, c->d_boxes,
                                       c->d_keys, c->d_tickets, cres, st)
               : c->sw_c ? launch_sweep(c->swc, cur, prv, c->pitch, c->d_citems, c->nc, c->d_keys,
                                        c->d_tickets, cres, c->d_swerr, st)
                       : launch_search(c->gc, cur, prv, c->pitch, c->d_citems, c->nc, c->d_keys,
                                       c->d_tickets, cres, st);
      if (nl < 0) return -1;
      c->launches += nl;
      count_launches(nl);
      kt_end(c, VSBD_KT_COARSE, st);
      if (c->log_in && log_items(c, cur, prv, st, c->d_citems, c->nc, 0, cres, skip) != 0) return -1;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_out, c->d_out, c->off_fine, cudaMemcpyDeviceToHost, st));
    count_d2h(c->off_fine);
    if (c->pn_on && c->pn_verify)
      CK(cudaMemcpyAsync(c->h_vres, c->d_vres, sizeof(vsbd_result) * c->nc, cudaMemcpyDeviceToHost,
                         st));
  }
  CK(cudaEventRecord(c->ev_ablk[c->obuf], st));
  c->aq_blk[c->naq] = c->obuf;
  c->aq_search[c->naq] = search;
  c->naq++;
  return 0;
}

/* a sweep whose bounded wait ran out left its fields' keys and counters
   mid-way: report, and start them afresh */
static int sweep_failed(vsbd_ctx* c, int k) {
  if (!c->h_swerr || !((volatile unsigned*)c->h_swerr)[k]) return 0;
  cudaStreamSynchronize(c->st);
  cudaStreamSynchronize(c->st2);
  c->h_swerr[k] = 0;
  cudaMemset(c->d_keys, 0xff, sizeof(unsigned long long) * (c->nc + c->nf + 2));
  cudaMemset(c->d_tickets, 0, sizeof(unsigned) * (c->nc + c->nf + 2));
  set_msg(k ? "fine search: a wait for staged rows gave up" : "coarse search: a wait for staged rows gave up");
  return 1;
}

/* waits for the oldest issued stage A and hands out its results */
static int stage_a_collect(vsbd_ctx* c, const uint8_t** minmax, const vsbd_result** coarse) {
  if (c->naq <= 0) {
    set_msg("no stage A in flight");
    return -1;
  }
  const int blk = c->aq_blk[0], search = c->aq_search[0];
  for (int i = 1; i < c->naq; i++) {
    c->aq_blk[i - 1] = c->aq_blk[i];
    c->aq_search[i - 1] = c->aq_search[i];
  }
  c->naq--;
  CK(cudaEventSynchronize(c->ev_ablk[blk]));
  kt_collect(c);
  if (sweep_failed(c, 0)) return -1;
  if (c->h_swerr && ((volatile unsigned*)c->h_swerr)[2]) {
    c->h_swerr[2] = 0;
    set_msg("proposal network: a wait for the tensor cores gave up");
    return -1;
  }
  uint8_t* h = c->h_outs[blk];
  if (search && c->pn_on)
    proposal_tally(c, h + c->off_cfb, (const vsbd_result*)(h + c->off_coarse), c->h_vres, c->nc,
                   0);
  if (minmax) *minmax = h;
  if (coarse) *coarse = (const vsbd_result*)(h + c->off_coarse);
  return 0;
}

/* a blurred-plane slot that no frame in use holds */
static int free_slot(const vsbd_ctx* c) {
  for (int k = 0; k < 4; k++) {
    bool used = k == c->cur || k == c->prv;
    for (int i = 0; i < c->nnxt; i++) used = used || k == c->nxt[i];
    if (!used) return k;
  }
  return -1;
}

/* stage A of the frame after the last one issued: blurred into a free slot,
   searched against that frame's plane */
static int stage_a_next(vsbd_ctx* c, const uint8_t* dev, int pitch) {
  if (c->nnxt >= 2) {
    set_msg("two next frames already in flight");
    return -1;
  }
  const int slot = free_slot(c);
  const int against = c->nnxt > 0 ? c->nxt[c->nnxt - 1] : c->cur;
  if (slot < 0 || stage_a_issue(c, NULL, 0, dev, pitch, 1, slot, against) != 0) return -1;
  c->nxt[c->nnxt++] = slot;
  return 0;
}

extern "C" int vsbd_stage_a(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev,
                            int pitch, int search, const uint8_t** minmax,
                            const vsbd_result** coarse) {
  CK(cudaSetDevice(c->dev));
  if (stage_a_issue(c, host, linesize, dev, pitch, search, c->cur, c->prv) != 0) return -1;
  return stage_a_collect(c, minmax, coarse);
}

extern "C" int vsbd_stage_a_issue(vsbd_ctx* c, const uint8_t* host, int linesize,
                                  const uint8_t* dev, int pitch, int search) {
  CK(cudaSetDevice(c->dev));
  return stage_a_issue(c, host, linesize, dev, pitch, search, c->cur, c->prv);
}

extern "C" int vsbd_stage_a_next_issue(vsbd_ctx* c, const uint8_t* host, int linesize,
                                       const uint8_t* dev, int pitch) {
  CK(cudaSetDevice(c->dev));
  if (host) {
    set_msg("the next frame's stage A takes device planes (vsbd_upload for host frames)");
    return -1;
  }
  return stage_a_next(c, dev, pitch);
}

extern "C" int vsbd_proposal_on(const vsbd_ctx* c) { return c && c->pn_on; }

/* how many frames' stage A a frame loop may keep in flight: one while the
   proposal's verification runs (every stage A copies its full-search
   results into the one host array the collect tallies), else two */
extern "C" int vsbd_pipeline_depth(const vsbd_ctx* c) {
  return c && c->pn_on && c->pn_verify ? 1 : 2;
}

extern "C" int vsbd_upload(vsbd_ctx* c, const uint8_t* host, int linesize, int slot) {
  CK(cudaSetDevice(c->dev));
  if (slot < 0 || slot > 2) {
    set_msg("upload slot must be 0, 1 or 2");
    return -1;
  }
  if (!c->st3) {
    const size_t plane = (size_t)c->pitch * c->H + 256;
    for (int k = 0; k < 3; k++) {
      if (!c->d_up[k]) CK(cudaMalloc(&c->d_up[k], plane));
      if (!c->ev_up[k]) CK(cudaEventCreateWithFlags(&c->ev_up[k], cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking));
  }
  const int rowbytes = c->W * c->bpp;
  CK(cudaMemcpy2DAsync(c->d_up[slot], c->pitch, host, linesize, rowbytes, c->H,
                       cudaMemcpyHostToDevice, c->st3));
  count_h2d((size_t)rowbytes * c->H);
  CK(cudaEventRecord(c->ev_up[slot], c->st3));
  return 0;
}

extern "C" int vsbd_stage_a_next_issue_uploaded(vsbd_ctx* c, int slot) {
  CK(cudaSetDevice(c->dev));
  if (slot < 0 || slot > 2 || !c->d_up[slot]) {
    set_msg("no frame uploaded in that slot");
    return -1;
  }
  /* the next frame's stage A starts once its upload has landed */
  CK(cudaStreamWaitEvent(c->st, c->ev_up[slot], 0));
  return stage_a_next(c, c->d_up[slot], c->pitch);
}

extern "C" int vsbd_stage_a_next_collect(vsbd_ctx* c, const uint8_t** minmax,
                                         const vsbd_result** coarse) {
  CK(cudaSetDevice(c->dev));
  return stage_a_collect(c, minmax, coarse);
}

extern "C" int vsbd_stage_b_issue(vsbd_ctx* c, const vsbd_item* items, int n) {
  CK(cudaSetDevice(c->dev));
  if (n > c->nf) { set_msg("more fine items than fine fields"); return -1; }
  c->b_n = n;
  c->b_hout = c->h_out;
  if (n <= 0) return 0;
  cudaStream_t st = c->st2;
  memcpy(c->h_items, items, sizeof(vsbd_item) * n);
  CK(cudaMemcpyAsync(c->d_fitems, c->h_items, sizeof(vsbd_item) * n, cudaMemcpyHostToDevice, st));
  count_h2d(sizeof(vsbd_item) * n);
  uint8_t* cur = c->d_buf[c->cur];
  uint8_t* prv = c->d_buf[c->prv];
  vsbd_result* fres = (vsbd_result*)(c->d_out + c->off_fine);
  size_t d2h = sizeof(vsbd_result) * n;
  if (fine_narrowed(c)) {
    if (learned_search(c, c->gf, c->fb_last[1] >= 8 ? c->gf : c->gff, cur, prv, st, c->d_fitems,
                       n, c->nc, NULL, c->d_keys + c->nc, c->d_tickets + c->nc, fres,
                       c->d_out + c->off_ffb, c->d_fbl + c->nc + 2) != 0)
      return -1;
    d2h = c->off_ffb - c->off_fine + n;
  } else {
    kt_begin(c, VSBD_KT_FINE, st);
    int nl = c->mode ? launch_pruned(c->gf, c->gfp, cur, prv, c->pitch, c->d_fitems, n, NULL,
                                     c->d_part, c->d_counts + c->nc, c->d_lists,
                                     c->d_boxes + 4 * c->nc, c->d_keys + c->nc,
                                     c->d_tickets + c->nc, fres, st)
             : c->fw_f ? launch_fine_warp(c->gf, c->fw_warps, c->fw_t, c->fw_ns, cur, prv,
                                          c->pitch, c->d_fitems, n, fres, st)
             : c->sw_f ? launch_sweep(c->swf, cur, prv, c->pitch, c->d_fitems, n, c->d_keys + c->nc,
                                      c->d_tickets + c->nc, fres, c->d_swerr + 1, st)
                     : launch_search(c->gf, cur, prv, c->pitch, c->d_fitems, n, c->d_keys + c->nc,
                                     c->d_tickets + c->nc, fres, st);
    if (nl < 0) return -1;
    c->launches += nl;
    count_launches(nl);
    kt_end(c, VSBD_KT_FINE, st);
    if (c->log_in && log_items(c, cur, prv, st, c->d_fitems, n, 1, fres, NULL) != 0) return -1;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_out + c->off_fine, c->d_out + c->off_fine, d2h, cudaMemcpyDeviceToHost,
                     st));
  count_d2h(d2h);
  if (fine_narrowed(c) && c->pn_verify)
    CK(cudaMemcpyAsync(c->h_vres + c->nc, c->d_vres + c->nc, sizeof(vsbd_result) * n,
                       cudaMemcpyDeviceToHost, st));
  CK(cudaEventRecord(c->ev_b, st));
  return 0;
}

extern "C" int vsbd_stage_b_collect(vsbd_ctx* c, const vsbd_result** fine) {
  CK(cudaSetDevice(c->dev));
  uint8_t* h = c->b_hout ? c->b_hout : c->h_out;
  *fine = (const vsbd_result*)(h + c->off_fine);
  if (c->b_n <= 0) return 0;
  CK(cudaEventSynchronize(c->ev_b));
  kt_collect(c);
  if (sweep_failed(c, 1)) return -1;
  if (fine_narrowed(c))
    proposal_tally(c, h + c->off_ffb, (const vsbd_result*)(h + c->off_fine),
                   c->h_vres ? c->h_vres + c->nc : NULL, c->b_n, 1);
  return 0;
}

extern "C" int vsbd_stage_b(vsbd_ctx* c, const vsbd_item* items, int n, const vsbd_result** fine) {
  if (vsbd_stage_b_issue(c, items, n) != 0) return -1;
  return vsbd_stage_b_collect(c, fine);
}

/* the current plane becomes the previous one; the next frame takes the
   slot its issued stage A blurred into, or a free one */
extern "C" void vsbd_commit_prev(vsbd_ctx* c) {
  int f;
  if (c->nnxt > 0) {
    f = c->nxt[0];
    c->nxt[0] = c->nxt[1];
    c->nnxt--;
  } else {
    f = free_slot(c);
  }
  c->prv = c->cur;
  c->cur = f;
}

/* whether stage A of the next frame may overlap stage B of this one: the
   two stages then share no scratch (the pruned search's partial sums and
   the training log are shared, and per-kernel timing needs one stream) */
extern "C" int vsbd_can_overlap(const vsbd_ctx* c) {
  return c && c->mode == 0 && !c->log_in && !c->timing;
}

extern "C" long vsbd_launches(const vsbd_ctx* c) { return c ? c->launches : 0; }

extern "C" int vsbd_search_tiling(const vsbd_ctx* c, int fine, int* desc) {
  if (!c || !desc) return -1;
  if (fine && c->fw_f) {
    /* k_fine: layout 6, one CTA of desc[5] threads per field */
    const DGeom& g = c->gf.g;
    desc[0] = 1;
    desc[1] = 6;
    desc[2] = g.na;
    desc[3] = g.nb;
    desc[4] = c->fw_t;
    desc[5] = 32 * c->fw_warps;
    desc[6] = (int)fw_layout(g, 32 * c->fw_warps, c->fw_t, c->fw_ns).total;
    desc[7] = c->fw_ns;
    return 0;
  }
  const int sw = fine ? c->sw_f : c->sw_c;
  const DGeom& g = sw ? (fine ? c->swf : c->swc) : (fine ? c->gf.g : c->gc.g);
  desc[0] = g.tb;
  desc[1] = g.ta > 0 ? g.ta : 1;
  desc[2] = g.nab;
  desc[3] = g.nbb;
  desc[4] = g.nstrip;
  desc[5] = g.threads;
  desc[6] = (int)(sw ? sweep_layout(g).total : (fine ? c->gf.smem : c->gc.smem));
  desc[7] = sw ? g.ctas : g.nta * g.ntb;
  return 0;
}

extern "C" int vsbd_blur_tiling(const vsbd_ctx* c, int* desc) {
  if (!c || !desc) return -1;
  desc[0] = g_blur_shape[c->blur_shape][0];
  desc[1] = g_blur_shape[c->blur_shape][1];
  desc[2] = (int)(1000.f * c->blur_us);
  desc[3] = c->bm_on;
  return 0;
}

extern "C" long vsbd_pnet_param_bytes(void) { return (long)PN_PARAM_BYTES; }

extern "C" int vsbd_set_proposal(vsbd_ctx* c, const void* params, float scale, float radius,
                                 float conf_min, float match_bound) {
  if (!c) return -1;
  CK(cudaSetDevice(c->dev));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaStreamSynchronize(c->st2));
  if (!params) {
    c->pn_on = 0;
    return 0;
  }
  if (c->bpp != 1 || c->gc.g.has_origin || c->gf.g.has_origin) {
    set_msg("the search proposal serves planar formats only");
    return -1;
  }
  if (!(scale > 0.f) || !(radius >= 0.f) || !(match_bound >= 0.f)) {
    set_msg("bad proposal settings");
    return -1;
  }
  if (!c->d_pn) CK(cudaMalloc(&c->d_pn, PN_PARAM_BYTES));
  if (!c->d_pout) CK(cudaMalloc(&c->d_pout, sizeof(float) * 3 * (c->nc + c->nf + 1)));
  if (!c->d_fbl) CK(cudaMalloc(&c->d_fbl, sizeof(int) * (c->nc + c->nf + 4)));
  if (!c->d_citems2) CK(cudaMalloc(&c->d_citems2, sizeof(vsbd_item) * (c->nc + 1)));
  if (!c->d_prior) CK(cudaMalloc(&c->d_prior, sizeof(short2) * (c->nc + 1)));
  CK(cudaMemcpy(c->d_pn, params, PN_PARAM_BYTES, cudaMemcpyHostToDevice));
  /* the full search of the items that fall back: a tiling for a handful of
     items, so that one item's lattice is spread over many CTAs (the
     detector's own tiling gives each item a few CTAs, and one fallback would
     then take as long as searching every field) */
  {
    TileCand tc[1];
    c->gcf = c->gc;
    c->gff = c->gf;
    if (tile_candidates(c->gc.g, 2, 0, 0, 0, 0, tc, 1) >= 1) {
      c->gcf.g = tc[0].g;
      c->gcf.smem = tile_layout(tc[0].g).total;
    }
    if (tile_candidates(c->gf.g, 8, 0, 0, 0, 0, tc, 1) >= 1) {
      c->gff.g = tc[0].g;
      c->gff.smem = tile_layout(tc[0].g).total;
    }
    GeomDev* gs[4] = { &c->gc, &c->gf, &c->gcf, &c->gff };
    for (int k = 0; k < 4; k++) {
      GeomDev* g = gs[k];
      int cps = 0;
      cudaError_t e = cudaSuccess;
      const void* fn = NULL;
      int slot = 0;
      if (g->g.tb == 2) { fn = g->g.ta == 2 ? (const void*)k_lattice_list<2, 2> : (const void*)k_lattice_list<2, 1>; slot = g->g.ta == 2 ? 14 : 3; }
      if (g->g.tb == 4) { fn = g->g.ta == 2 ? (const void*)k_lattice_list<4, 2> : (const void*)k_lattice_list<4, 1>; slot = g->g.ta == 2 ? 15 : 4; }
      if (g->g.ta == 3 && g->g.tb == 2) { fn = (const void*)k_lattice_list<2, 3>; slot = 22; }
      if (g->g.ta == 3 && g->g.tb == 4) { fn = (const void*)k_lattice_list<4, 3>; slot = 23; }
      if (g->g.ta == 4 && g->g.tb == 2) { fn = (const void*)k_lattice_list<2, 4>; slot = 26; }
      if (g->g.ta == 4 && g->g.tb == 4) { fn = (const void*)k_lattice_list<4, 4>; slot = 27; }
      if (g->g.tb == 8) { fn = (const void*)k_lattice_list<8, 1>; slot = 5; }
      if (fn) {
        e = ensure_smem(fn, slot, g->smem);
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, fn, g->g.threads, g->smem);
      }
      if (e != cudaSuccess) {
        set_err("fallback search set-up", e);
        return -1;
      }
      g->list_cps = cps;
    }
  }
  c->pn.scale = scale;
  c->pn.radius = radius;
  c->pn.conf_min = conf_min;
  c->pn.sad_bound = 0xffffffffu;
  c->pn_match_bound = match_bound;
  c->pn_on = 1;
  return 0;
}

extern "C" int vsbd_set_proposal_scope(vsbd_ctx* c, int fine_net, float fine_radius) {
  if (!c) return -1;
  if (fine_radius > 16.f) {
    set_msg("fine proposal radius above 16 px");
    return -1;
  }
  c->pn_fine_net = fine_net ? 1 : 0;
  c->pn_fine_radius = fine_radius;
  return 0;
}

extern "C" int vsbd_set_proposal_passes(vsbd_ctx* c, int passes) {
  if (!c || passes < 1 || passes > 2) {
    set_msg("proposal passes must be 1 or 2");
    return -1;
  }
  c->pn_passes = passes;
  return 0;
}

extern "C" int vsbd_set_proposal_verify(vsbd_ctx* c, int on) {
  if (!c) return -1;
  CK(cudaSetDevice(c->dev));
  if (on && !c->d_vres) {
    CK(cudaMalloc(&c->d_vres, sizeof(vsbd_result) * (c->nc + c->nf + 1)));
    CK(cudaMallocHost(&c->h_vres, sizeof(vsbd_result) * (c->nc + c->nf + 1)));
  }
  c->pn_verify = on ? 1 : 0;
  return 0;
}

extern "C" int vsbd_proposal_stats(const vsbd_ctx* c, long long* st) {
  if (!c || !st) return -1;
  for (int k = 0; k < 8; k++) st[k] = c->pn_stats[k];
  return 0;
}

extern "C" int vsbd_set_field_log(vsbd_ctx* c, void* d_inputs, void* d_labels, long cap) {
  if (!c) return -1;
  if (d_inputs && (!d_labels || cap < 0)) {
    set_msg("field log needs inputs, labels and a capacity");
    return -1;
  }
  if (d_inputs && c->bpp != 1) {
    set_msg("the field log serves planar formats only");
    return -1;
  }
  c->log_in = (uint8_t*)d_inputs;
  c->log_lab = (PNLabel*)d_labels;
  c->log_cap = d_inputs ? cap : 0;
  c->log_n = 0;
  return 0;
}

extern "C" long vsbd_field_log_count(const vsbd_ctx* c) { return c ? c->log_n : -1; }

/* ------------------------------------------------------------------------ */
/* kernel-level entry points (parity tests)                                  */
/* ------------------------------------------------------------------------ */

extern "C" int vsbd_blur_host_shape(uint8_t* dst, const uint8_t* src, int W, int H, int size,
                                    int shape) {
  int pitch = (W + 127) & ~127;
  size_t plane = (size_t)pitch * H + 256;
  uint8_t *d_src = NULL, *d_dst = NULL, *d_tmp = NULL;
  int rc = -1;
  cudaError_t e;
  if ((e = cudaMalloc(&d_src, plane)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_dst, plane)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_tmp, plane)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMemcpy2D(d_src, pitch, src, W, W, H, cudaMemcpyHostToDevice)) != cudaSuccess) { set_err("upload", e); goto done; }
  if (size < 2) {
    e = cudaMemcpy2D(d_dst, pitch, d_src, pitch, W, H, cudaMemcpyDeviceToDevice);
  } else {
    launch_blur(d_src, pitch, d_dst, pitch, W, H, size, d_tmp, pitch, 0, shape);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) { set_err("blur", e); goto done; }
  if ((e = cudaMemcpy2D(dst, W, d_dst, pitch, W, H, cudaMemcpyDeviceToHost)) != cudaSuccess) { set_err("download", e); goto done; }
  rc = 0;
done:
  cudaFree(d_src);
  cudaFree(d_dst);
  cudaFree(d_tmp);
  return rc;
}

extern "C" int vsbd_blur_host(uint8_t* dst, const uint8_t* src, int W, int H, int size) {
  return vsbd_blur_host_shape(dst, src, W, H, size, 0);
}

extern "C" int vsbd_minmax_host(const uint8_t* img, int W, int H, int bpp, int channels,
                                const int16_t* x, const int16_t* y, int n, int size,
                                uint8_t* out) {
  int pitch = (int)(((size_t)W * bpp + 127) & ~(size_t)127);
  uint8_t *d_img = NULL, *d_out = NULL;
  int16_t* d_xy = NULL;
  int rc = -1;
  cudaError_t e;
  if ((e = cudaMalloc(&d_img, (size_t)pitch * H + 256)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_out, (size_t)n * channels * 2 + 16)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_xy, sizeof(int16_t) * 2 * n + 16)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMemcpy2D(d_img, pitch, img, (size_t)W * bpp, (size_t)W * bpp, H, cudaMemcpyHostToDevice)) != cudaSuccess) { set_err("upload", e); goto done; }
  cudaMemcpy(d_xy, x, sizeof(int16_t) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(d_xy + n, y, sizeof(int16_t) * n, cudaMemcpyHostToDevice);
  if (n > 0) k_minmax<<<n, 256>>>(d_img, pitch, d_xy, d_xy + n, size, bpp, channels, d_out, 0.0, NULL);
  if ((e = cudaGetLastError()) != cudaSuccess) { set_err("k_minmax", e); goto done; }
  if ((e = cudaMemcpy(out, d_out, (size_t)n * channels * 2, cudaMemcpyDeviceToHost)) != cudaSuccess) { set_err("download", e); goto done; }
  rc = 0;
done:
  cudaFree(d_img);
  cudaFree(d_out);
  cudaFree(d_xy);
  return rc;
}

extern "C" int vsbd_search_host(const uint8_t* curr, const uint8_t* prev, int W, int H,
                                const vsbd_geom* geom, const vsbd_item* items, int n,
                                int tiles_hint, vsbd_result* out) {
  int bpp = geom->bpp;
  int pitch = (int)(((size_t)W * bpp + 127) & ~(size_t)127);
  size_t plane = (size_t)pitch * H + 256;
  uint8_t *d_c = NULL, *d_p = NULL;
  vsbd_item* d_items = NULL;
  vsbd_result* d_res = NULL;
  unsigned long long* d_keys = NULL;
  unsigned* d_tk = NULL;
  GeomDev gd;
  memset(&gd, 0, sizeof(gd));
  int rc = -1;
  cudaError_t e;
  /* tiles_hint < 0: the sweep, with the plan of that rank in its candidate
     list (-1 the model's best); tiles_hint <= -100: k_fine, -100 - tiles_hint
     = 1000 * strips + 100 * T + warps (T lattice rows per thread; a zero
     digit means 1) */
  const int fw_code = tiles_hint <= -100 ? -100 - tiles_hint : 0;
  const int fw_warps = fw_code % 100;
  const int fw_t = (fw_code / 100) % 10 ? (fw_code / 100) % 10 : 1;
  const int fw_ns = fw_code / 1000 ? fw_code / 1000 : 1;
  if (tiles_hint <= -100) tiles_hint = 0;
  DGeom swg;
  unsigned* d_err = NULL;
  unsigned h_err = 0;
  if (geom_upload(geom, n, tiles_hint > 0 ? tiles_hint : 0, &gd) != 0) goto done;
  if (tiles_hint < 0) {
    TileCand cand[12];
    const int nc = sweep_candidates(gd.g, n, cand, 12);
    if (-tiles_hint > nc) {
      set_msg("no sweep plan of that rank for this field geometry");
      goto done;
    }
    swg = cand[-tiles_hint - 1].g;
    if ((e = cudaMalloc(&d_err, sizeof(unsigned))) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
    cudaMemset(d_err, 0, sizeof(unsigned));
  }
  if ((e = cudaMalloc(&d_c, plane)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_p, plane)) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_items, sizeof(vsbd_item) * (n + 1))) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_res, sizeof(vsbd_result) * (n + 1))) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_keys, sizeof(unsigned long long) * (n + 1))) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  if ((e = cudaMalloc(&d_tk, sizeof(unsigned) * (n + 1))) != cudaSuccess) { set_err("cudaMalloc", e); goto done; }
  cudaMemset(d_keys, 0xff, sizeof(unsigned long long) * (n + 1));
  cudaMemset(d_tk, 0, sizeof(unsigned) * (n + 1));
  cudaMemcpy2D(d_c, pitch, curr, (size_t)W * bpp, (size_t)W * bpp, H, cudaMemcpyHostToDevice);
  cudaMemcpy2D(d_p, pitch, prev, (size_t)W * bpp, (size_t)W * bpp, H, cudaMemcpyHostToDevice);
  cudaMemcpy(d_items, items, sizeof(vsbd_item) * n, cudaMemcpyHostToDevice);
  if (fw_code) {
    if (launch_fine_warp(gd, fw_warps, fw_t, fw_ns, d_c, d_p, pitch, d_items, n, d_res, 0) < 0)
      goto done;
  } else if (tiles_hint < 0) {
    if (launch_sweep(swg, d_c, d_p, pitch, d_items, n, d_keys, d_tk, d_res, d_err, 0) < 0)
      goto done;
    if ((e = cudaMemcpy(&h_err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost)) != cudaSuccess) { set_err("k_sweep", e); goto done; }
    if (h_err) { set_msg("search sweep: a wait for staged rows gave up"); goto done; }
  } else if (launch_search(gd, d_c, d_p, pitch, d_items, n, d_keys, d_tk, d_res, 0) < 0) {
    goto done;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) { set_err("k_search", e); goto done; }
  if ((e = cudaMemcpy(out, d_res, sizeof(vsbd_result) * n, cudaMemcpyDeviceToHost)) != cudaSuccess) { set_err("download", e); goto done; }
  rc = 0;
done:
  geom_free(&gd);
  cudaFree(d_c);
  cudaFree(d_p);
  cudaFree(d_items);
  cudaFree(d_res);
  cudaFree(d_keys);
  cudaFree(d_tk);
  cudaFree(d_err);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* packed-SAD throughput probe: register-only chains of one SAD formulation  */
/* ------------------------------------------------------------------------ */

template <int V>
__device__ __forceinline__ unsigned sad_variant(unsigned a, unsigned b, unsigned c) {
  if (V == 0) return sad4(a, b, c);
  if (V == 1) return __vsadu4(a, b) + c;
  return __dp4a(__vabsdiffu4(a, b), 0x01010101u, c);
}

template <int V>
__global__ void __launch_bounds__(256) k_sad_peak(unsigned* out, int iters, unsigned seed) {
  unsigned a[8], acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed * (unsigned)(k + 1) + threadIdx.x * 0x9e3779b9u;
    acc[k] = a[k] ^ 0x5a5a5a5au;
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = sad_variant<V>(a[k], acc[k], acc[k]);
  }
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += acc[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

/* byte absolute differences per second of one SAD formulation (variant 0:
   vabsdiff4 with accumulate, 1: __vsadu4 + add, 2: __vabsdiffu4 + dp4a) */
extern "C" int vsbd_sad_peak(int variant, double* byteops_per_s) {
  int blocks = sm_count() * 8, threads = 256, iters = 8192;
  unsigned* d = NULL;
  cudaEvent_t e0, e1;
  CK(cudaMalloc(&d, sizeof(unsigned) * blocks * threads));
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    if (variant == 0) k_sad_peak<0><<<blocks, threads>>>(d, iters, 12345u + rep);
    else if (variant == 1) k_sad_peak<1><<<blocks, threads>>>(d, iters, 12345u + rep);
    else k_sad_peak<2><<<blocks, threads>>>(d, iters, 12345u + rep);
    cudaEventRecord(e1);
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  *byteops_per_s = (double)blocks * threads * iters * 8.0 * 4.0 / (best * 1e-3);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* planning helpers for the batched path (vsb_plan.h)                        */
/* ------------------------------------------------------------------------ */
int vsbp_geom_upload(const vsbd_geom* h, int nitems, GeomDev* out) {
  return geom_upload(h, nitems, 0, out);
}
void vsbp_geom_free(GeomDev* g) { geom_free(g); }
int vsbp_tile_candidates(const DGeom& g, int nitems, int max_threads, TileCand* out, int cap) {
  return tile_candidates(g, nitems, 0, 0, 0, 0, out, cap, max_threads);
}
int vsbp_tile_candidates_ta(const DGeom& g, int nitems, int max_threads, TileCand* out, int cap,
                            int ta) {
  return tile_candidates(g, nitems, 0, 0, 0, 0, out, cap, max_threads, ta);
}
int vsbp_sm_count(void) { return sm_count(); }
void vsbp_set_err(const char* what, cudaError_t e) { set_err(what, e); }
void vsbp_set_msg(const char* m) { set_msg(m); }
void vsbp_count(long launches, size_t h2d, size_t d2h) {
  count_launches(launches);
  count_h2d(h2d);
  count_d2h(d2h);
}
