/*
 * vsb_prefilter.cuh -- per-tile and per-field bodies of the prefilter
 * kernels (box blur, field min/max), shared by the per-stream kernels and
 * the batched persistent kernel.
 */
#ifndef VSB_PREFILTER_CUH
#define VSB_PREFILTER_CUH

#include <cuda_runtime.h>
#include <stdint.h>

/* floor(acc / size) as a multiply-high by ceil(2^32/size): exact whenever
   acc_max * size < 2^32 (checked exhaustively on the host when the divisor
   is set up; otherwise the kernel divides) */
struct BlurDiv {
  unsigned mul;
  unsigned size;
  int exact;
};

__device__ __forceinline__ unsigned blur_div(unsigned acc, BlurDiv d) {
  return d.exact ? __umulhi(acc, d.mul) : acc / d.size;
}

#define BT_W 128
#define BT_H 32
#define BT_MAXHALF 32
#define BT_RAWP (BT_W + 2 * BT_MAXHALF + 4)
#define BT_HORP (BT_W + 4)
/* shared memory of one blur tile: raw input with halo, horizontal pass */
#define BT_SMEM ((BT_H + 2 * BT_MAXHALF) * (BT_RAWP + BT_HORP))

/* One CTA of 256 threads blurs the BT_H x BT_W output tile (bx, by).  The
   input tile plus a halo of `half` pixels is read once with clamped
   coordinates (edge replication), the horizontal pass writes 8-bit values to
   shared memory and the vertical pass runs a sliding sum down each column
   (src/boxblur.c:190-332: window sums, floor division by the size). */
__device__ __forceinline__ void blur_tile(const uint8_t* __restrict__ src, int sp,
                                          uint8_t* __restrict__ dst, int dp, int W, int H,
                                          int half, BlurDiv dv, int bx, int by, uint8_t* smem) {
  uint8_t* raw = smem;
  uint8_t* hor = smem + (BT_H + 2 * BT_MAXHALF) * BT_RAWP;
  const int x0 = bx * BT_W, y0 = by * BT_H;
  const int rows = BT_H + 2 * half, cols = BT_W + 2 * half;
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    int r = i / cols, c = i - r * cols;
    int gy = min(max(y0 - half + r, 0), H - 1);
    int gx = min(max(x0 - half + c, 0), W - 1);
    raw[r * BT_RAWP + c] = src[(size_t)gy * sp + gx];
  }
  __syncthreads();
  const int win = 2 * half + 1;
  for (int i = threadIdx.x; i < rows * BT_W; i += blockDim.x) {
    int r = i / BT_W, c = i - r * BT_W;
    unsigned acc = 0;
    for (int k = 0; k < win; k++) acc += raw[r * BT_RAWP + c + k];
    hor[r * BT_HORP + c] = (uint8_t)blur_div(acc, dv);
  }
  __syncthreads();
  /* 256 threads: column c, upper or lower half of the tile rows (threads
     beyond 256, in larger blocks, have no column) */
  if (threadIdx.x >= 2 * BT_W) return;
  const int c = threadIdx.x & (BT_W - 1);
  const int part = threadIdx.x >> 7;
  const int gx = x0 + c;
  if (gx >= W) return;
  const int rbeg = part * (BT_H / 2);
  unsigned acc = 0;
  for (int k = 0; k < win; k++) acc += hor[(rbeg + k) * BT_HORP + c];
  for (int r = rbeg; r < rbeg + BT_H / 2; r++) {
    if (r > rbeg) { /* slide: rows [r, r + win) of hor feed output row r */
      acc += hor[(r + win - 1) * BT_HORP + c];
      acc -= hor[(r - 1) * BT_HORP + c];
    }
    int gy = y0 + r;
    if (gy >= H) break;
    dst[(size_t)gy * dp + gx] = (uint8_t)blur_div(acc, dv);
  }
}

/* The same blur over a BTF_H x BTF_W output tile with vector memory access,
   for half-widths up to BTF_MAXHALF given at run time (at least 256
   threads).  Input rows with clamped coordinates are staged from 16 bytes
   left of the tile to 16 bytes right of it, with 16-byte loads when the tile
   is interior and the source 16-byte aligned, else bytewise.  The
   horizontal pass gives each task a run of 16 outputs of one row (a sliding
   window sum, one 16-byte store); the vertical pass runs 4-column sliding
   sums down a quarter of the tile and stores words (threads beyond 256 have
   no column).  Same window sums and floor division as blur_tile. */
#define BTF_W 256
#define BTF_H 32
#define BTF_MAXHALF 16
#define BTF_RAWP (BTF_W + 32)
#define BTF_SMEM ((BTF_H + 2 * BTF_MAXHALF) * (BTF_RAWP + BTF_W))

__device__ __forceinline__ void blur_tile_fast(const uint8_t* __restrict__ src, int sp,
                                               uint8_t* __restrict__ dst, int dp, int W, int H,
                                               int half, BlurDiv dv, int bx, int by,
                                               uint8_t* smem) {
  const int rows = BTF_H + 2 * half, win = 2 * half + 1;
  uint8_t* raw = smem;
  uint8_t* hor = smem + rows * BTF_RAWP;
  const int x0 = bx * BTF_W, y0 = by * BTF_H;
  const bool vec = x0 >= 16 && x0 + BTF_W + 16 <= W &&
                   ((((uintptr_t)src) | (uintptr_t)(unsigned)sp) & 15) == 0;
  if (vec) {
    for (int i = threadIdx.x; i < rows * (BTF_RAWP / 16); i += blockDim.x) {
      const int r = i / (BTF_RAWP / 16), v = i - r * (BTF_RAWP / 16);
      const int gy = min(max(y0 - half + r, 0), H - 1);
      *(uint4*)(raw + r * BTF_RAWP + (v << 4)) =
          *(const uint4*)(src + (size_t)gy * sp + x0 - 16 + (v << 4));
    }
  } else {
    for (int i = threadIdx.x; i < rows * BTF_RAWP; i += blockDim.x) {
      const int r = i / BTF_RAWP, c = i - r * BTF_RAWP;
      const int gy = min(max(y0 - half + r, 0), H - 1);
      const int gx = min(max(x0 - 16 + c, 0), W - 1);
      raw[r * BTF_RAWP + c] = src[(size_t)gy * sp + gx];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < rows * (BTF_W / 16); t += blockDim.x) {
    const int r = t / (BTF_W / 16), c0 = (t - r * (BTF_W / 16)) * 16;
    const uint8_t* rp = raw + r * BTF_RAWP + 16 + c0; /* the byte of column c0 */
    unsigned acc = 0;
    for (int k = -half; k <= half; k++) acc += rp[k];
    uint32_t o[4] = { 0u, 0u, 0u, 0u };
#pragma unroll
    for (int q = 0; q < 16; q++) {
      if (q > 0) acc += (unsigned)rp[q + half] - (unsigned)rp[q - 1 - half];
      o[q >> 2] |= blur_div(acc, dv) << (8 * (q & 3));
    }
    *(uint4*)(hor + r * BTF_W + c0) = make_uint4(o[0], o[1], o[2], o[3]);
  }
  __syncthreads();
  if (threadIdx.x >= 256) return;
  const int cg = threadIdx.x & 63, part = threadIdx.x >> 6;
  const int gx = x0 + cg * 4;
  if (gx >= W) return;
  const int rb = part * (BTF_H / 4);
  unsigned a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (int k = 0; k < win; k++) {
    const unsigned w = *(const unsigned*)(hor + (rb + k) * BTF_W + cg * 4);
    a0 += w & 0xff;
    a1 += (w >> 8) & 0xff;
    a2 += (w >> 16) & 0xff;
    a3 += w >> 24;
  }
  const bool full4 = gx + 4 <= W;
  for (int r = rb; r < rb + BTF_H / 4; r++) {
    if (r > rb) {
      const unsigned wi = *(const unsigned*)(hor + (r + win - 1) * BTF_W + cg * 4);
      const unsigned wo = *(const unsigned*)(hor + (r - 1) * BTF_W + cg * 4);
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

/* Field f of a field list, by one CTA: 8-bit min/max per channel (channel ch
   of a pixel is byte ch of its bpp bytes) into out[(f*nch + ch)*2 + {0,1}].
   With skip != NULL it also flags a field whose contrast keeps it out of the
   selection: the reference zeroes a contrast below the threshold and selects
   only positive contrasts (src/motiondetect.c:697-698, :719, :734).  The
   contrast is the reference's double expression (:389-407), evaluated in
   IEEE double like the host's ((c0 + c1) + c2) * (1/3) for three channels,
   so the flag agrees with the host's selection bit for bit. */
__device__ __forceinline__ void minmax_field(const uint8_t* __restrict__ img, int pitch, int x,
                                             int y, int S, int bpp, int nch, int f,
                                             uint8_t* __restrict__ out, double thr,
                                             uint8_t* __restrict__ skip) {
  __shared__ unsigned smn[32], smx[32];
  const int x0 = x - S / 2, y0 = y - S / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double c[3] = { 0.0, 0.0, 0.0 };
  for (int ch = 0; ch < nch; ch++) {
    unsigned mn = 255, mx = 0;
    for (int i = threadIdx.x; i < S * S; i += blockDim.x) {
      int r = i / S, col = i - r * S;
      unsigned v = img[(size_t)(y0 + r) * pitch + (size_t)(x0 + col) * bpp + ch];
      mn = min(mn, v);
      mx = max(mx, v);
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane == 0) { smn[warp] = mn; smx[warp] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) { mn = min(mn, smn[w]); mx = max(mx, smx[w]); }
      out[(f * nch + ch) * 2 + 0] = (uint8_t)mn;
      out[(f * nch + ch) * 2 + 1] = (uint8_t)mx;
      c[ch] = (double)((int)mx - (int)mn) / ((double)((int)mx + (int)mn) + 0.1);
    }
    __syncthreads();
  }
  if (skip && threadIdx.x == 0) {
    double con = c[0];
    if (nch == 3) {
      double s = __dadd_rn(c[0], c[1]);
      s = __dadd_rn(s, c[2]);
      con = __dmul_rn(s, 1.0 / 3.0);
    }
    skip[f] = !(con >= thr && con > 0.0);
  }
}

/* 8-bit min/max of one planar field by one warp (out[f*2 + {0,1}]): rows
   read with 16-byte loads from the 16-byte boundary at or left of the
   field, bytes outside the field masked to the neutral value.  The plane's
   rows must start on 16-byte boundaries, with readable bytes up to 15 past
   the field's right edge. */
__device__ __forceinline__ unsigned mm_byte_mask(int lo, int hi) {
  unsigned m = 0;
#pragma unroll
  for (int b = 0; b < 4; b++)
    if (b >= lo && b < hi) m |= 0xffu << (8 * b);
  return m;
}

__device__ __forceinline__ void minmax_field_warp(const uint8_t* __restrict__ img, int pitch,
                                                  int x, int y, int S, int f,
                                                  uint8_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int x0 = x - S / 2, y0 = y - S / 2;
  const int xa = x0 & ~15;
  const int nv = (x0 + S - xa + 15) >> 4;
  unsigned mn = 0xffffffffu, mx = 0u;
  for (int i = lane; i < S * nv; i += 32) {
    const int r = i / nv, v = i - r * nv;
    const int bx = xa + (v << 4);
    const uint4 q = *(const uint4*)(img + (size_t)(y0 + r) * pitch + bx);
    const unsigned w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int b0 = bx + 4 * k;
      const unsigned m = mm_byte_mask(x0 - b0, x0 + S - b0);
      mn = __vminu4(mn, w[k] | ~m);
      mx = __vmaxu4(mx, w[k] & m);
    }
  }
  unsigned bmn = min(min(mn & 0xff, (mn >> 8) & 0xff), min((mn >> 16) & 0xff, mn >> 24));
  unsigned bmx = max(max(mx & 0xff, (mx >> 8) & 0xff), max((mx >> 16) & 0xff, mx >> 24));
  bmn = __reduce_min_sync(0xffffffffu, bmn);
  bmx = __reduce_max_sync(0xffffffffu, bmx);
  if (lane == 0) {
    out[f * 2 + 0] = (uint8_t)bmn;
    out[f * 2 + 1] = (uint8_t)bmx;
  }
}

/* divisor set-up of the blur (host) */
static inline int make_div(int size, int half, BlurDiv* d) {
  d->size = (unsigned)size;
  d->exact = 0;
  d->mul = 0;
  if (size < 2) return 0;
  unsigned long long mul = ((1ull << 32) + (unsigned)size - 1) / (unsigned)size;
  if (mul > 0xffffffffull) return 0;
  unsigned accmax = 255u * (unsigned)(2 * half + 1);
  for (unsigned a = 0; a <= accmax; a++)
    if ((unsigned)((a * mul) >> 32) != a / (unsigned)size) return 0;
  d->mul = (unsigned)mul;
  d->exact = 1;
  return 0;
}

#endif
