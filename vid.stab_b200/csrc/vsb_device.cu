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
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vsb_device.h"

/* ------------------------------------------------------------------------ */
/* error plumbing                                                            */
/* ------------------------------------------------------------------------ */
static thread_local char g_err[512];

static void set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
}
static void set_msg(const char* m) { snprintf(g_err, sizeof(g_err), "%s", m); }

extern "C" const char* vsbd_error(void) { return g_err; }

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

/* One CTA blurs a BT_H x BT_W output tile.  The input tile plus a halo of
   `half` pixels is read once with clamped coordinates (edge replication),
   the horizontal pass writes 8-bit values to shared memory and the vertical
   pass runs a sliding sum down each column. */
__global__ void __launch_bounds__(256) k_blur(const uint8_t* __restrict__ src, int sp,
                                              uint8_t* __restrict__ dst, int dp, int W, int H,
                                              int half, BlurDiv dv) {
  __shared__ uint8_t raw[BT_H + 2 * BT_MAXHALF][BT_W + 2 * BT_MAXHALF + 4];
  __shared__ uint8_t hor[BT_H + 2 * BT_MAXHALF][BT_W + 4];
  const int x0 = blockIdx.x * BT_W, y0 = blockIdx.y * BT_H;
  const int rows = BT_H + 2 * half, cols = BT_W + 2 * half;
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    int r = i / cols, c = i - r * cols;
    int gy = min(max(y0 - half + r, 0), H - 1);
    int gx = min(max(x0 - half + c, 0), W - 1);
    raw[r][c] = src[(size_t)gy * sp + gx];
  }
  __syncthreads();
  const int win = 2 * half + 1;
  for (int i = threadIdx.x; i < rows * BT_W; i += blockDim.x) {
    int r = i / BT_W, c = i - r * BT_W;
    unsigned acc = 0;
    for (int k = 0; k < win; k++) acc += raw[r][c + k];
    hor[r][c] = (uint8_t)blur_div(acc, dv);
  }
  __syncthreads();
  /* 256 threads: column c, upper or lower half of the tile rows */
  const int c = threadIdx.x & (BT_W - 1);
  const int part = threadIdx.x >> 7;
  const int gx = x0 + c;
  if (gx >= W) return;
  const int rbeg = part * (BT_H / 2);
  unsigned acc = 0;
  for (int k = 0; k < win; k++) acc += hor[rbeg + k][c];
  for (int r = rbeg; r < rbeg + BT_H / 2; r++) {
    int gy = y0 + r;
    if (gy >= H) break;
    dst[(size_t)gy * dp + gx] = (uint8_t)blur_div(acc, dv);
    acc += hor[r + win][c];
    acc -= hor[r][c];
  }
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

static int make_div(int size, int half, BlurDiv* d) {
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

/* launches the prefilter of one plane; returns the number of kernels */
static int launch_blur(const uint8_t* src, int sp, uint8_t* dst, int dp, int W, int H, int size,
                       uint8_t* tmp, int tp, cudaStream_t st) {
  int half = size / 2;
  BlurDiv dv;
  make_div(size, half, &dv);
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

/* one CTA per field; channel ch of a pixel is byte ch of its bpp bytes */
__global__ void __launch_bounds__(256) k_minmax(const uint8_t* __restrict__ img, int pitch,
                                                const int16_t* __restrict__ xs,
                                                const int16_t* __restrict__ ys, int S, int bpp,
                                                int nch, uint8_t* __restrict__ out) {
  __shared__ unsigned smn[8], smx[8];
  const int f = blockIdx.x;
  const int x0 = xs[f] - S / 2, y0 = ys[f] - S / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int ch = 0; ch < nch; ch++) {
    unsigned mn = 255, mx = 0;
    for (int i = threadIdx.x; i < S * S; i += blockDim.x) {
      int r = i / S, c = i - r * S;
      unsigned v = img[(size_t)(y0 + r) * pitch + (size_t)(x0 + c) * bpp + ch];
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
    }
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* SAD search                                                                */
/* ------------------------------------------------------------------------ */

struct DGeom {
  int S, bpp, step, na, nb, ax0, by0, has_origin, nstages;
  int st_r[VSBD_MAX_STAGES], st_h[VSBD_MAX_STAGES];
  int limx, limy;
  int rows_per_tile;
  int maxq;                    /* largest refinement grid */
  const int32_t* order;        /* rank of lattice point (a,b) at [b*na+a] */
  const short2* point;         /* displacement of rank k */
};

/* packed 4 x u8 sum of absolute differences, accumulated */
__device__ __forceinline__ unsigned sad4(unsigned a, unsigned b, unsigned c) {
  unsigned d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

/* SAD of the staged field (rowW words per row, S rows) against the window
   bytes starting at byte column cxb of P (row pitch WP). */
__device__ __forceinline__ unsigned sad_window(const uint32_t* __restrict__ C, int rowW, int S,
                                               const uint8_t* __restrict__ P, int WP, int cxb) {
  unsigned acc = 0;
  const int sh = (cxb & 3) << 3;
  const int nq = rowW >> 2;
  for (int r = 0; r < S; r++) {
    const uint32_t* Pw = (const uint32_t*)(P + r * WP) + (cxb >> 2);
    const uint4* C4 = (const uint4*)(C + r * rowW);
    uint32_t lo = Pw[0];
    for (int q = 0; q < nq; q++) {
      uint4 c = C4[q];
      uint32_t p1 = Pw[4 * q + 1], p2 = Pw[4 * q + 2], p3 = Pw[4 * q + 3], p4 = Pw[4 * q + 4];
      acc = sad4(c.x, __funnelshift_r(lo, p1, sh), acc);
      acc = sad4(c.y, __funnelshift_r(p1, p2, sh), acc);
      acc = sad4(c.z, __funnelshift_r(p2, p3, sh), acc);
      acc = sad4(c.w, __funnelshift_r(p3, p4, sh), acc);
      lo = p4;
    }
  }
  return acc;
}

/* SAD of the staged field against the previous frame in global memory at
   byte column gxb, row gy0 (warp-cooperative: lanes take rows) */
__device__ unsigned sad_global_warp(const uint32_t* __restrict__ C, int rowW, int S,
                                    const uint8_t* __restrict__ prev, int pitch, int gxb,
                                    int gy0, int lane) {
  unsigned acc = 0;
  const int sh = (gxb & 3) << 3;
  for (int r = lane; r < S; r += 32) {
    const uint32_t* Pw = (const uint32_t*)(prev + (size_t)(gy0 + r) * pitch) + (gxb >> 2);
    const uint32_t* Cr = C + r * rowW;
    uint32_t lo = Pw[0];
    for (int w = 0; w < rowW; w++) {
      uint32_t hi = Pw[w + 1];
      acc = sad4(Cr[w], __funnelshift_r(lo, hi, sh), acc);
      lo = hi;
    }
  }
  return __reduce_add_sync(0xffffffffu, acc);
}

__device__ __forceinline__ unsigned long long warp_min64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t < v ? t : v;
  }
  return v;
}

/* grid: (tiles, items); 256 threads.  Dynamic shared memory:
   [field S*rowB][window WH*WP][refinement SADs maxq*4] */
__global__ void __launch_bounds__(256) k_search(const uint8_t* __restrict__ curr,
                                                const uint8_t* __restrict__ prev, int pitch,
                                                DGeom g, const vsbd_item* __restrict__ items,
                                                unsigned long long* __restrict__ keys,
                                                unsigned* __restrict__ tickets,
                                                vsbd_result* __restrict__ res) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ unsigned long long red[8];
  __shared__ int s_last, s_tx, s_ty;
  __shared__ unsigned s_min;
  const int item = blockIdx.y, tile = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const vsbd_item it = items[item];
  const int rowB = g.S * g.bpp, rowW = rowB >> 2;
  uint32_t* C = (uint32_t*)sm;
  const int b0 = tile * g.rows_per_tile;
  const int nbt = min(g.rows_per_tile, g.nb - b0);
  const int gx0 = (it.x - g.S / 2 + it.ox + g.ax0) * g.bpp;
  const int gy0 = it.y - g.S / 2 + it.oy + g.by0 + b0 * g.step;
  const int WWb = rowB + (g.na - 1) * g.step * g.bpp;
  const int WH = g.S + (nbt - 1) * g.step;
  const int gx0a = gx0 & ~15, e = gx0 - gx0a;
  const int nvec = (e + WWb + 15) >> 4;
  const int WP = (nvec + 1) << 4;
  uint8_t* P = sm + g.S * rowB;
  unsigned* qsad = (unsigned*)(P + (size_t)WH * WP);

  /* the current field, re-aligned to word boundaries */
  {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int sh = (cx0 & 3) << 3, cw0 = cx0 >> 2;
    for (int i = threadIdx.x; i < g.S * rowW; i += blockDim.x) {
      int r = i / rowW, w = i - r * rowW;
      const uint32_t* s = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + cw0 + w;
      C[i] = __funnelshift_r(s[0], s[1], sh);
    }
  }
  /* the window of the previous frame this CTA's candidate rows touch */
  for (int i = threadIdx.x; i < WH * nvec; i += blockDim.x) {
    int r = i / nvec, v = i - r * nvec;
    uint4 val = *(const uint4*)(prev + (size_t)(gy0 + r) * pitch + gx0a + (v << 4));
    *(uint4*)(P + r * WP + (v << 4)) = val;
  }
  __syncthreads();

  unsigned long long best = ~0ull;
  const int ncand = g.na * nbt;
  for (int c = threadIdx.x; c < ncand; c += blockDim.x) {
    int bl = c / g.na, a = c - bl * g.na;
    unsigned s = sad_window(C, rowW, g.S, P + bl * g.step * WP, WP, e + a * g.step * g.bpp);
    unsigned long long key =
        ((unsigned long long)s << 32) | (unsigned)g.order[(b0 + bl) * g.na + a];
    best = key < best ? key : best;
  }
  best = warp_min64(best);
  if (lane == 0) red[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nwarps; w++) best = red[w] < best ? red[w] : best;
    atomicMin(&keys[item], best);
    __threadfence();
    unsigned t = atomicAdd(&tickets[item], 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();

  /* last CTA of this item: origin candidate, refinement, range test */
  if (threadIdx.x == 0) {
    unsigned long long k = atomicAdd(&keys[item], 0ull);
    short2 pt = g.point[(unsigned)(k & 0xffffffffu)];
    s_min = (unsigned)(k >> 32);
    s_tx = pt.x;
    s_ty = pt.y;
  }
  __syncthreads();
  const int fx0 = (it.x - g.S / 2 + it.ox) * g.bpp, fy0 = it.y - g.S / 2 + it.oy;
  if (g.has_origin) {
    if (warp == 0) {
      unsigned s0 = sad_global_warp(C, rowW, g.S, prev, pitch, fx0, fy0, lane);
      /* rank 0 precedes every lattice rank */
      if (lane == 0 && s0 <= s_min) { s_min = s0; s_tx = 0; s_ty = 0; }
    }
    __syncthreads();
  }
  for (int st = 0; st < g.nstages; st++) {
    const int r = g.st_r[st], h = g.st_h[st];
    const int side = (2 * r) / h + 1, nq = side * side;
    const int cx = s_tx, cy = s_ty;
    for (int q = warp; q < nq; q += nwarps) {
      int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
      unsigned s = 0xffffffffu;
      if (!(i == cx && j == cy))
        s = sad_global_warp(C, rowW, g.S, prev, pitch, fx0 + i * g.bpp, fy0 + j, lane);
      if (lane == 0) qsad[q] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned m = s_min;
      int tx = cx, ty = cy;
      for (int q = 0; q < nq; q++) {
        int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
        if (i == cx && j == cy) continue;
        if (qsad[q] < m) { m = qsad[q]; tx = i; ty = j; }
      }
      s_min = m;
      s_tx = tx;
      s_ty = ty;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    vsbd_result o;
    o.sad = s_min;
    o.tx = (int16_t)s_tx;
    o.ty = (int16_t)s_ty;
    o.ok = !(abs(s_tx) >= g.limx || abs(s_ty) >= g.limy);
    res[item] = o;
    keys[item] = ~0ull;
    tickets[item] = 0u;
  }
}

/* ------------------------------------------------------------------------ */
/* geometry upload                                                           */
/* ------------------------------------------------------------------------ */

struct GeomDev {
  DGeom g;
  int32_t* d_order;
  short2* d_point;
  int tiles;
  size_t smem;
};

static size_t search_smem(const DGeom& g, int rows_per_tile) {
  int rowB = g.S * g.bpp;
  int WWb = rowB + (g.na - 1) * g.step * g.bpp;
  int WH = g.S + (rows_per_tile - 1) * g.step;
  int WP = (((15 + WWb + 15) >> 4) + 1) << 4;
  return (size_t)g.S * rowB + (size_t)WH * WP + (size_t)g.maxq * 4 + 16;
}

static int sm_count(void) {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

/* rows of the candidate lattice per CTA: enough CTAs for ~4 per SM, as long
   as the window fits the shared-memory budget */
static int pick_rows_per_tile(const DGeom& g, int nitems, int hint) {
  int rpt = g.nb;
  if (hint > 0) rpt = (g.nb + hint - 1) / hint;
  else if (nitems > 0) {
    int want = 4 * sm_count();
    int tiles = (want + nitems - 1) / nitems;
    if (tiles > g.nb) tiles = g.nb;
    if (tiles < 1) tiles = 1;
    rpt = (g.nb + tiles - 1) / tiles;
  }
  while (rpt > 1 && search_smem(g, rpt) > 200 * 1024) rpt = (rpt + 1) / 2;
  return rpt;
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
  g.rows_per_tile = pick_rows_per_tile(g, nitems, tiles_hint);
  out->tiles = (g.nb + g.rows_per_tile - 1) / g.rows_per_tile;
  out->smem = search_smem(g, g.rows_per_tile);
  if (out->smem > 227 * 1024) { set_msg("search window exceeds shared memory"); return -1; }
  return 0;
}

static void geom_free(GeomDev* g) {
  if (g->d_order) cudaFree(g->d_order);
  if (g->d_point) cudaFree(g->d_point);
  g->d_order = NULL;
  g->d_point = NULL;
}

static int launch_search(const GeomDev& gd, const uint8_t* curr, const uint8_t* prev, int pitch,
                         const vsbd_item* d_items, int n, unsigned long long* keys,
                         unsigned* tickets, vsbd_result* d_res, cudaStream_t st) {
  if (n <= 0) return 0;
  static int attr_done = 0;
  if (!attr_done) {
    cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr_done = 1;
  }
  dim3 grid(gd.tiles, n);
  k_search<<<grid, 256, gd.smem, st>>>(curr, prev, pitch, gd.g, d_items, keys, tickets, d_res);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* per-detector context                                                      */
/* ------------------------------------------------------------------------ */

struct vsbd_ctx {
  int dev;
  int W, H, bpp, blur, nch, pitch;
  int nc, nf;
  cudaStream_t st;
  uint8_t* d_raw;     /* input plane (blurred formats) */
  uint8_t* d_tmp;     /* row-pass buffer of the wide-window blur */
  uint8_t* d_buf[2];  /* blurred planes: current / previous */
  int cur;
  int16_t* d_xy;      /* coarse x | coarse y | fine x | fine y */
  GeomDev gc, gf;
  vsbd_item* d_citems;
  vsbd_item* d_fitems;
  unsigned long long* d_keys;   /* coarse nc, then fine nf */
  unsigned* d_tickets;
  uint8_t* d_out;               /* minmax | coarse results | fine results */
  uint8_t* h_out;               /* pinned mirror of d_out */
  vsbd_item* h_items;           /* pinned staging of fine items */
  size_t off_coarse, off_fine, out_bytes;
  long launches;
};

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
  cudaFree(c->d_raw);
  cudaFree(c->d_tmp);
  cudaFree(c->d_buf[0]);
  cudaFree(c->d_buf[1]);
  cudaFree(c->d_xy);
  cudaFree(c->d_citems);
  cudaFree(c->d_fitems);
  cudaFree(c->d_keys);
  cudaFree(c->d_tickets);
  cudaFree(c->d_out);
  if (c->h_out) cudaFreeHost(c->h_out);
  if (c->h_items) cudaFreeHost(c->h_items);
  geom_free(&c->gc);
  geom_free(&c->gf);
  if (c->st) cudaStreamDestroy(c->st);
  free(c);
}

extern "C" int vsbd_create(vsbd_ctx** out, int W, int H, int bpp, int blur_size, int channels,
                           const vsbd_geom* coarse, const int16_t* cx, const int16_t* cy, int nc,
                           const vsbd_geom* fine, const int16_t* fx, const int16_t* fy, int nf) {
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
  c->pitch = (int)(((size_t)W * bpp + 127) & ~(size_t)127);
  size_t plane = (size_t)c->pitch * H + 256; /* slack: word reads past a row end */
#define CKC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { set_err(#call, e_); vsbd_destroy(c); return -1; } } while (0)
  CKC(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  if (blur_size >= 2) CKC(cudaMalloc(&c->d_raw, plane));
  if (blur_size >= 2 && blur_size / 2 > BT_MAXHALF) CKC(cudaMalloc(&c->d_tmp, plane));
  CKC(cudaMalloc(&c->d_buf[0], plane));
  CKC(cudaMalloc(&c->d_buf[1], plane));
  CKC(cudaMemset(c->d_buf[0], 0, plane));
  CKC(cudaMemset(c->d_buf[1], 0, plane));
  CKC(cudaMalloc(&c->d_xy, sizeof(int16_t) * 2 * (nc + nf) + 16));
  CKC(cudaMemcpy(c->d_xy, cx, sizeof(int16_t) * nc, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + nc, cy, sizeof(int16_t) * nc, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + 2 * nc, fx, sizeof(int16_t) * nf, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(c->d_xy + 2 * nc + nf, fy, sizeof(int16_t) * nf, cudaMemcpyHostToDevice));
  if (geom_upload(coarse, nc, 0, &c->gc) != 0) { vsbd_destroy(c); return -1; }
  if (geom_upload(fine, nf, 0, &c->gf) != 0) { vsbd_destroy(c); return -1; }
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
  c->off_fine = c->off_coarse + align16(sizeof(vsbd_result) * (nc + 1));
  c->out_bytes = c->off_fine + align16(sizeof(vsbd_result) * (nf + 1));
  CKC(cudaMalloc(&c->d_out, c->out_bytes));
  CKC(cudaMallocHost(&c->h_out, c->out_bytes));
#undef CKC
  *out = c;
  return 0;
}

extern "C" int vsbd_stage_a(vsbd_ctx* c, const uint8_t* host, int linesize, const uint8_t* dev,
                            int pitch, int search, const uint8_t** minmax,
                            const vsbd_result** coarse) {
  CK(cudaSetDevice(c->dev));
  const int rowbytes = c->W * c->bpp;
  uint8_t* cur = c->d_buf[c->cur];
  uint8_t* prv = c->d_buf[c->cur ^ 1];
  if (c->blur >= 2) {
    const uint8_t* src = dev;
    int sp = pitch;
    if (!dev) {
      CK(cudaMemcpy2DAsync(c->d_raw, c->pitch, host, linesize, rowbytes, c->H,
                           cudaMemcpyHostToDevice, c->st));
      src = c->d_raw;
      sp = c->pitch;
    }
    c->launches += launch_blur(src, sp, cur, c->pitch, c->W, c->H, c->blur, c->d_tmp, c->pitch, c->st);
    CK(cudaGetLastError());
  } else {
    if (dev)
      CK(cudaMemcpy2DAsync(cur, c->pitch, dev, pitch, rowbytes, c->H, cudaMemcpyDeviceToDevice, c->st));
    else
      CK(cudaMemcpy2DAsync(cur, c->pitch, host, linesize, rowbytes, c->H, cudaMemcpyHostToDevice, c->st));
  }
  if (search) {
    int S = c->gc.g.S;
    k_minmax<<<c->nc, 256, 0, c->st>>>(cur, c->pitch, c->d_xy, c->d_xy + c->nc, S, c->bpp, c->nch, c->d_out);
    c->launches++;
    if (c->nf > 0) {
      k_minmax<<<c->nf, 256, 0, c->st>>>(cur, c->pitch, c->d_xy + 2 * c->nc, c->d_xy + 2 * c->nc + c->nf,
                                         c->gf.g.S, c->bpp, c->nch, c->d_out + (size_t)c->nc * c->nch * 2);
      c->launches++;
    }
    c->launches += launch_search(c->gc, cur, prv, c->pitch, c->d_citems, c->nc, c->d_keys, c->d_tickets,
                                 (vsbd_result*)(c->d_out + c->off_coarse), c->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_out, c->d_out, c->off_fine, cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  if (minmax) *minmax = c->h_out;
  if (coarse) *coarse = (const vsbd_result*)(c->h_out + c->off_coarse);
  return 0;
}

extern "C" int vsbd_stage_b(vsbd_ctx* c, const vsbd_item* items, int n, const vsbd_result** fine) {
  CK(cudaSetDevice(c->dev));
  if (n > c->nf) { set_msg("more fine items than fine fields"); return -1; }
  *fine = (const vsbd_result*)(c->h_out + c->off_fine);
  if (n <= 0) return 0;
  memcpy(c->h_items, items, sizeof(vsbd_item) * n);
  CK(cudaMemcpyAsync(c->d_fitems, c->h_items, sizeof(vsbd_item) * n, cudaMemcpyHostToDevice, c->st));
  uint8_t* cur = c->d_buf[c->cur];
  uint8_t* prv = c->d_buf[c->cur ^ 1];
  c->launches += launch_search(c->gf, cur, prv, c->pitch, c->d_fitems, n, c->d_keys + c->nc,
                               c->d_tickets + c->nc, (vsbd_result*)(c->d_out + c->off_fine), c->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_out + c->off_fine, c->d_out + c->off_fine, sizeof(vsbd_result) * n,
                     cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" void vsbd_commit_prev(vsbd_ctx* c) { c->cur ^= 1; }

extern "C" long vsbd_launches(const vsbd_ctx* c) { return c ? c->launches : 0; }

/* ------------------------------------------------------------------------ */
/* kernel-level entry points (parity tests)                                  */
/* ------------------------------------------------------------------------ */

extern "C" int vsbd_blur_host(uint8_t* dst, const uint8_t* src, int W, int H, int size) {
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
    launch_blur(d_src, pitch, d_dst, pitch, W, H, size, d_tmp, pitch, 0);
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
  if (n > 0) k_minmax<<<n, 256>>>(d_img, pitch, d_xy, d_xy + n, size, bpp, channels, d_out);
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
  if (geom_upload(geom, n, tiles_hint, &gd) != 0) goto done;
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
  launch_search(gd, d_c, d_p, pitch, d_items, n, d_keys, d_tk, d_res, 0);
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
  return rc;
}
