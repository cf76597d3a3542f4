/*
 * vsb_pnet_dev.cuh -- device bodies of the learned search proposal: the
 * crop of an item, the narrowed search of one item and the global motion
 * prior of a field set (the network's forward is in vsb_pnet_tc.cuh).  The
 * single-stream kernels (vsb_pnet.cu) and the batched persistent kernel
 * (vsb_batch.cu) both call them, so a batched stream computes exactly what
 * its own detector does.
 */
#ifndef VSB_PNET_DEV_CUH
#define VSB_PNET_DEV_CUH

#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "vsb_pnet.h"
#include "vsb_search.cuh"

typedef __nv_bfloat16 bf16;
namespace cg = cooperative_groups;

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }

struct PNPtr {
  const bf16 *w1, *w2, *w3, *w4, *fc;
  const float *b1, *b2, *b3, *b4, *bfc;
};

__host__ __device__ inline PNPtr pn_ptr(const void* p) {
  const bf16* w = (const bf16*)p;
  const float* f = (const float*)((const char*)p + PN_F32_OFFSET);
  PNPtr r;
  r.w1 = w;
  r.w2 = w + PN_NW1;
  r.w3 = w + PN_NW1 + PN_NW;
  r.w4 = w + PN_NW1 + 2 * PN_NW;
  r.fc = w + PN_NW1 + 3 * PN_NW;
  r.b1 = f;
  r.b2 = f + 32;
  r.b3 = f + 64;
  r.b4 = f + 96;
  r.bfc = f + 128;
  return r;
}

/* ------------------------------------------------------------------------ */
/* crop: 2x2 averages of the 64x64 windows around the item in both planes   */
/* ------------------------------------------------------------------------ */

/* value of input element (ch, r, c) of item it: bf16((sum4 - 512) / 256) */
__device__ __forceinline__ bf16 crop_value(const uint8_t* __restrict__ curr,
                                           const uint8_t* __restrict__ prev, int pitch, int W,
                                           int H, const vsbd_item& it, int ch, int r, int c) {
  const uint8_t* img = ch ? prev : curr;
  const int cx = (ch ? it.x + it.ox : it.x) - 32 + 2 * c;
  const int cy = (ch ? it.y + it.oy : it.y) - 32 + 2 * r;
  const int x0 = min(max(cx, 0), W - 1), x1 = min(max(cx + 1, 0), W - 1);
  const int y0 = min(max(cy, 0), H - 1), y1 = min(max(cy + 1, 0), H - 1);
  const uint8_t* r0 = img + (size_t)y0 * pitch;
  const uint8_t* r1 = img + (size_t)y1 * pitch;
  int s = (int)r0[x0] + (int)r0[x1] + (int)r1[x0] + (int)r1[x1];
  return __float2bfloat16_rn((float)(s - 512) / 256.0f);
}

/* block size of the inference (vsb_pnet_tc.cuh) */
#define PI_THREADS 512

/* ------------------------------------------------------------------------ */
/* narrowed search                                                           */
/* ------------------------------------------------------------------------ */

/* lattice points per axis the window can hold: the bracket of prediction
   +- radius (at most ceil(2 radius / step) + 2 points) plus the ring */
__host__ __device__ inline int narrow_span(float radius, int step) {
  return (int)ceilf(2.0f * radius / (float)step) + 4;
}

/* shared-memory layout of k_pn_narrow */
struct NarrowLayout {
  int rowW, fieldB, WP, WH, R, nq;
  size_t off_win, off_q, total;
};

#define PN_NARROW_QMAX 64 /* candidate sums of one round (lattice window or refinement grid) */

__host__ __device__ inline NarrowLayout narrow_layout(const DGeom& g, float radius) {
  NarrowLayout L;
  const int rowB = g.S * g.bpp;
  L.rowW = rowB >> 2;
  L.fieldB = ((g.S * rowB) + 15) & ~15;
  L.R = refine_reach(g);
  const int span = narrow_span(radius, g.step);
  const int wwb = rowB + ((span - 1) * g.step + 2 * L.R) * g.bpp;
  L.WP = (((15 + wwb + 15) >> 4) + 1) << 4;
  L.WH = g.S + (span - 1) * g.step + 2 * L.R;
  L.off_win = (size_t)L.fieldB + 16;
  L.off_q = L.off_win + (size_t)L.WH * L.WP + 16;
  L.nq = g.maxq > PN_NARROW_QMAX ? g.maxq : PN_NARROW_QMAX;
  /* three sum buffers: two that the CTAs of a cluster add into by turns,
     one for the totals read back */
  L.total = L.off_q + (size_t)3 * L.nq * 4 + 16;
  return L;
}

/* One warp's share of a column of NK candidates: displacements (dx, dy0 +
   k*hy), k < NK, relative to the staged window's origin, summed over field
   rows [r0, r1).  A lane owns one word of the field row (several rows at
   once when a row has fewer than 32 words), loads the field word once per
   row and applies it to every candidate of the column; partial sums are
   added to sums[k] in shared memory. */
template <int NK>
__device__ __forceinline__ void sad_column(const uint32_t* __restrict__ C, int rowW,
                                           const uint8_t* __restrict__ win, int WP, int e, int bpp,
                                           int dx, int dy0, int hy, int r0, int r1, int lane,
                                           unsigned* sums) {
  unsigned acc[NK];
#pragma unroll
  for (int k = 0; k < NK; k++) acc[k] = 0;
  const int bx = e + dx * bpp;
  const int sh = (bx & 3) << 3;
  const int WPw = WP >> 2;
  const int G = rowW < 32 ? 32 / rowW : 1;
  const int g = rowW < 32 ? lane / rowW : 0;
  const int w0 = rowW < 32 ? lane - g * rowW : lane;
  const int hyw = hy * WPw;
  if (g < G) {
    for (int w = w0; w < rowW; w += 32) {
      const uint32_t* Cw = C + w;
      const uint32_t* Pw = (const uint32_t*)win + (bx >> 2) + w;
      for (int r = r0 + g; r < r1; r += G) {
        const uint32_t c = Cw[r * rowW];
        const uint32_t* P = Pw + (r + dy0) * WPw;
#pragma unroll
        for (int k = 0; k < NK; k++) {
          const uint32_t* Q = P + k * hyw;
          acc[k] = sad4(c, __funnelshift_r(Q[0], Q[1], sh), acc[k]);
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NK; k++) {
    const unsigned v = __reduce_add_sync(0xffffffffu, acc[k]);
    if (lane == 0) atomicAdd(&sums[k], v);
  }
}

__device__ __forceinline__ void sad_column_n(int nk, const uint32_t* C, int rowW,
                                             const uint8_t* win, int WP, int e, int bpp, int dx,
                                             int dy0, int hy, int r0, int r1, int lane,
                                             unsigned* sums) {
#define VSB_SADCOL(K) \
  case K: sad_column<K>(C, rowW, win, WP, e, bpp, dx, dy0, hy, r0, r1, lane, sums); break;
  switch (nk) {
    VSB_SADCOL(1) VSB_SADCOL(2) VSB_SADCOL(3) VSB_SADCOL(4)
    VSB_SADCOL(5) VSB_SADCOL(6) VSB_SADCOL(7) VSB_SADCOL(8)
    default: break;
  }
#undef VSB_SADCOL
}

/* The SADs of a grid of candidates over field rows [rlo, rhi): columns
   i < ncol at dx0 + i*hx, rows k < nrow at dy0 + k*hy (window
   coordinates), added into sums[i*nrow + k] (zeroed first when `zero`;
   sums may be another CTA's shared memory).  The warps take (column, row
   chunk of <= 8, field-row strip) tasks. */
__device__ __forceinline__ void sad_grid(const uint32_t* C, int rowW, int rlo, int rhi,
                                         const uint8_t* win, int WP, int e, int bpp, int dx0,
                                         int hx, int ncol, int dy0, int hy, int nrow,
                                         unsigned* sums, bool zero) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (zero) {
    for (int q = threadIdx.x; q < ncol * nrow; q += blockDim.x) sums[q] = 0;
    __syncthreads();
  }
  const int nch = (nrow + 7) >> 3;
  const int units = ncol * nch;
  int strips = nwarps / units;
  if (strips < 1) strips = 1;
  const int rs = (rhi - rlo + strips - 1) / strips;
  for (int t = warp; t < units * strips; t += nwarps) {
    const int u = t % units, sidx = t / units;
    const int col = u / nch, ch = u - col * nch;
    const int k0 = ch * 8, nk = min(8, nrow - k0);
    const int r0 = rlo + sidx * rs, r1 = min(rhi, r0 + rs);
    if (r0 < r1)
      sad_column_n(nk, C, rowW, win, WP, e, bpp, dx0 + col * hx, dy0 + k0 * hy, hy, r0, r1, lane,
                   sums + col * nrow + k0);
  }
  __syncthreads();
}

/* The narrowed search of one item by the calling CTA (any multiple of 32
   threads up to 512; sm holds narrow_layout(g, ps.radius).total bytes).
   The lattice points that bracket the prediction +-
   radius, plus one ring around them, get their full SAD; the lowest (SAD,
   rank) is refined exactly as the full search refines its winner
   (src/motiondetect.c:545-567 of the reference: i outer, j inner, centre
   skipped, strict <) and range-tested (:573-574).  The window of the
   previous frame all of this can touch (the candidates plus the refinement
   reach) is staged once in shared memory with 16-byte loads.  The item
   falls back to the full search (appended to fb_list) when the confidence
   is below the threshold, the winner lies on the ring (the minimum may lie
   further out), or the refined SAD exceeds the bound. */
template <int CL>
__device__ __forceinline__ void pn_narrow_item(uint8_t* sm, const uint8_t* __restrict__ curr,
                                               const uint8_t* __restrict__ prev, int pitch,
                                               const DGeom& g, const vsbd_item* __restrict__ items,
                                               const float* __restrict__ pout,
                                               const short2* __restrict__ prior,
                                               const PNSearch& ps,
                                               const uint8_t* __restrict__ skip,
                                               vsbd_result* __restrict__ res,
                                               uint8_t* __restrict__ fb,
                                               int* __restrict__ fb_count,
                                               int* __restrict__ fb_list, int item) {
  __shared__ int s_tx, s_ty;
  __shared__ unsigned s_min;
  const NarrowLayout L = narrow_layout(g, ps.radius);
  const float* po = pout ? pout + item * 3 : NULL;
  const short2 base = prior ? prior[item] : make_short2(0, 0);
  const float px = (po ? po[0] * ps.scale : 0.f) + (float)base.x;
  const float py = (po ? po[1] * ps.scale : 0.f) + (float)base.y;
  const float cf = po ? po[2] : 3.0e38f;
  /* the bracket [lo, hi] of lattice indices covering prediction +- radius */
  int alo = 1, ahi = 0, blo = 1, bhi = 0;
  if (isfinite(px) && isfinite(py) && fabsf(px) < 30000.f && fabsf(py) < 30000.f) {
    alo = max((int)floorf((px - ps.radius - g.ax0) / g.step), 0);
    ahi = min((int)ceilf((px + ps.radius - g.ax0) / g.step), g.na - 1);
    blo = max((int)floorf((py - ps.radius - g.by0) / g.step), 0);
    bhi = min((int)ceilf((py + ps.radius - g.by0) / g.step), g.nb - 1);
  }
  const int wal = max(alo - 1, 0), wah = min(ahi + 1, g.na - 1);
  const int wbl = max(blo - 1, 0), wbh = min(bhi + 1, g.nb - 1);
  const int wa = wah - wal + 1, wb = wbh - wbl + 1;
  const int span = narrow_span(ps.radius, g.step);
  const bool unused = skip && skip[item];
  /* prediction outside the lattice, or a window that would not fit (cannot
     happen): no narrowed result */
  /* with CL > 1 the item is shared by a cluster of CL CTAs: CTA `rank`
     sums field rows [rlo, rhi) of every candidate into rank 0's sums */
  unsigned rank = 0;
  if constexpr (CL > 1) rank = cg::this_cluster().block_rank();
  const int rsz = (g.S + CL - 1) / CL;
  const int rlo = min(g.S, (int)rank * rsz), rhi = min(g.S, rlo + rsz);
  if (unused || alo > ahi || blo > bhi || wa > span || wb > span) {
    if (threadIdx.x == 0 && rank == 0) {
      vsbd_result o;
      o.sad = 0xffffffffu;
      o.tx = o.ty = 0;
      o.ok = 0;
      res[item] = o;
      fb[item] = unused ? PN_FB_UNUSED : PN_FB_FULL;
      if (!unused) fb_list[atomicAdd(fb_count, 1)] = item;
    }
    return;
  }
  const vsbd_item it = items[item];
  uint32_t* C = (uint32_t*)sm;
  uint8_t* win = sm + L.off_win;
  unsigned* qsad = (unsigned*)(sm + L.off_q);
  const int fx0 = (it.x - g.S / 2 + it.ox) * g.bpp, fy0 = it.y - g.S / 2 + it.oy;
  /* window origin: displacement (ax0 + wal*step - R, by0 + wbl*step - R) */
  const int dx0 = g.ax0 + wal * g.step - L.R, dy0 = g.by0 + wbl * g.step - L.R;
  const int wx = fx0 + dx0 * g.bpp, wy = fy0 + dy0;
  const int wxa = wx & ~15, e = wx - wxa;
  {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int sh = (cx0 & 3) << 3;
    for (int i = rlo * L.rowW + threadIdx.x; i < rhi * L.rowW; i += blockDim.x) {
      const int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + (cx0 >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
    /* the window rows the CTA's field rows meet: [rlo, rhi + wh - S) */
    const int wwb = g.S * g.bpp + ((wa - 1) * g.step + 2 * L.R) * g.bpp;
    const int wh = g.S + (wb - 1) * g.step + 2 * L.R;
    const int nv = (e + wwb + 15) >> 4;
    const int wr0 = rlo, wr1 = rhi + wh - g.S;
    for (int i = wr0 * nv + threadIdx.x; i < wr1 * nv; i += blockDim.x) {
      const int r = i / nv, v = i - r * nv;
      *(uint4*)(win + r * L.WP + (v << 4)) =
          *(const uint4*)(prev + (size_t)(wy + r) * pitch + wxa + (v << 4));
    }
  }
  __syncthreads();
  /* one round of candidate sums: qv = the totals (this CTA's qsad, or the
     totals read back from rank 0 after the cluster has added into it) */
  unsigned* qv = qsad;
  int round = 0;
  auto sums_round = [&](int dxs, int hx, int ncol, int dys, int hy, int nrow) {
    if constexpr (CL == 1) {
      sad_grid(C, L.rowW, 0, g.S, win, L.WP, e, g.bpp, dxs, hx, ncol, dys, hy, nrow, qsad, true);
    } else {
      cg::cluster_group cl = cg::this_cluster();
      unsigned* qb = qsad + (round & 1) * L.nq;
      if (rank == 0)
        for (int q = threadIdx.x; q < ncol * nrow; q += blockDim.x) qb[q] = 0;
      cl.sync();
      unsigned* qb0 = cl.map_shared_rank(qb, 0);
      sad_grid(C, L.rowW, rlo, rhi, win, L.WP, e, g.bpp, dxs, hx, ncol, dys, hy, nrow, qb0, false);
      cl.sync();
      qv = qsad + 2 * L.nq;
      for (int q = threadIdx.x; q < ncol * nrow; q += blockDim.x) qv[q] = qb0[q];
      __syncthreads();
    }
    round++;
  };
  /* lattice window: column a - wal, row b - wbl at sums[(a-wal)*wb + (b-wbl)];
     the lowest (SAD, visiting rank) by a block-wide reduction */
  sums_round(L.R, g.step, wa, L.R, g.step, wb);
  {
    __shared__ unsigned long long red[16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long best = ~0ull;
    for (int q = threadIdx.x; q < wa * wb; q += blockDim.x) {
      const int a = wal + q / wb, b = wbl + q % wb;
      const unsigned long long key =
          ((unsigned long long)qv[q] << 32) | (unsigned)g.order[b * g.na + a];
      best = key < best ? key : best;
    }
    best = warp_min64(best);
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) best = red[w] < best ? red[w] : best;
      const short2 pt = g.point[(unsigned)(best & 0xffffffffu)];
      s_min = (unsigned)(best >> 32);
      s_tx = pt.x;
      s_ty = pt.y;
    }
    __syncthreads();
  }
  const int aw = (s_tx - g.ax0) / g.step, bw = (s_ty - g.by0) / g.step;
  const bool ring = aw < alo || aw > ahi || bw < blo || bw > bhi;
  /* refinement rounds around the winner, inside the staged window: the
     side x side grid (centre included, ignored) */
  for (int st = 0; st < g.nstages; st++) {
    const int r = g.st_r[st], h = g.st_h[st];
    const int side = (2 * r) / h + 1;
    const int cx = s_tx, cy = s_ty;
    sums_round(cx - r - dx0, h, side, cy - r - dy0, h, side);
    if (threadIdx.x == 0) {
      unsigned m = s_min;
      int tx = cx, ty = cy;
      /* the reference's order: i (x) outer, j (y) inner */
      for (int ii = 0; ii < side; ii++)
        for (int jj = 0; jj < side; jj++) {
          const int i = cx - r + ii * h, j = cy - r + jj * h;
          if (i == cx && j == cy) continue;
          if (qv[ii * side + jj] < m) {
            m = qv[ii * side + jj];
            tx = i;
            ty = j;
          }
        }
      s_min = m;
      s_tx = tx;
      s_ty = ty;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && rank == 0) {
    vsbd_result o;
    o.sad = s_min;
    o.tx = (int16_t)s_tx;
    o.ty = (int16_t)s_ty;
    o.ok = !(abs(s_tx) >= g.limx || abs(s_ty) >= g.limy);
    res[item] = o;
    const bool trust = !ring && cf >= ps.conf_min && o.sad <= ps.sad_bound;
    fb[item] = trust ? PN_FB_ACCEPT : PN_FB_FULL;
    if (!trust) fb_list[atomicAdd(fb_count, 1)] = item;
  }
  /* rank 0's shared memory stays until every CTA of the cluster has read
     its last totals */
  if constexpr (CL > 1) cg::this_cluster().sync();
}

/* Global motion prior of a frame's coarse items from the first network
   pass.  Translation: the per-axis median of the confident predictions (the
   non-skipped items with a finite prediction and a logit >= conf_min; all
   non-skipped items if fewer than three are confident).  Rotation: the small
   angle about the frame centre that best fits, in least squares, the
   predictions within 8 px of that translation.  Every item gets the model's
   displacement at its centre, rounded: the search offset of its second
   network pass (items2) and the base of its proposal (prior).  Run by one
   CTA of 256 to 1024 threads, with the same result for any block size;
   buf is 4 * PN_PRIOR_MAX floats of its shared memory. */
#define PN_PRIOR_MAX 1024
__device__ __forceinline__ void pn_prior_body(float* buf, const vsbd_item* __restrict__ items,
                                              const float* __restrict__ pout, int n, float scale,
                                              float conf_min, const uint8_t* __restrict__ skip,
                                              float cx, float cy, vsbd_item* __restrict__ items2,
                                              short2* __restrict__ prior) {
  float* vx = buf;
  float* vy = buf + PN_PRIOR_MAX;
  float* jx = buf + 2 * PN_PRIOR_MAX;
  float* jy = buf + 3 * PN_PRIOR_MAX;
  __shared__ int m;
  __shared__ float med[2];
  __shared__ float sums[2][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  /* the usable predictions in item order (warp 0, 32 items per round, so
     the arrays and every sum below do not depend on scheduling or on the
     block size) */
  for (int pass = 0; pass < 2; pass++) {
    if (warp == 0) {
      int base = 0;
      for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        float px = 0.f, py = 0.f;
        bool use = i < n && !(skip && skip[i]);
        if (use) {
          px = pout[3 * i] * scale;
          py = pout[3 * i + 1] * scale;
          const float c = pout[3 * i + 2];
          use = isfinite(px) && isfinite(py) && fabsf(px) <= 4096.f && fabsf(py) <= 4096.f &&
                (pass == 1 || c >= conf_min);
        }
        const unsigned ball = __ballot_sync(0xffffffffu, use);
        const int k = base + __popc(ball & ((1u << lane) - 1u));
        if (use && k < PN_PRIOR_MAX) {
          vx[k] = px;
          vy[k] = py;
          jx[k] = -((float)items[i].y - cy); /* d(displacement)/d(angle) at the centre */
          jy[k] = (float)items[i].x - cx;
        }
        base += __popc(ball);
      }
      if (lane == 0) m = base;
    }
    __syncthreads();
    if (m >= 3 || pass == 1) break;
    __syncthreads();
  }
  const int cnt = min(m, PN_PRIOR_MAX);
  /* per-axis medians: the element whose rank (ties by index) is cnt/2 */
  if (tid == 0) med[0] = med[1] = 0.f;
  __syncthreads();
  for (int t = tid; t < 2 * cnt; t += blockDim.x) {
    const int ax = t >= cnt, k = t - ax * cnt;
    const float* v = ax ? vy : vx;
    const float x = v[k];
    int rank = 0;
    for (int j = 0; j < cnt; j++) rank += v[j] < x || (v[j] == x && j < k);
    if (rank == cnt / 2) med[ax] = x;
  }
  __syncthreads();
  /* rotation about the centre from the inliers of the translation, summed
     by the first 256 threads in a fixed order */
  float num = 0.f, den = 0.f;
  if (tid < 256)
    for (int k = tid; k < cnt; k += 256) {
      const float rx = vx[k] - med[0], ry = vy[k] - med[1];
      if (fabsf(rx) < 8.f && fabsf(ry) < 8.f) {
        num += rx * jx[k] + ry * jy[k];
        den += jx[k] * jx[k] + jy[k] * jy[k];
      }
    }
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, o);
    den += __shfl_xor_sync(0xffffffffu, den, o);
  }
  if (lane == 0 && warp < 8) {
    sums[0][warp] = num;
    sums[1][warp] = den;
  }
  __syncthreads();
  float th = 0.f;
  {
    float a = 0.f, b = 0.f;
    for (int w = 0; w < 8; w++) {
      a += sums[0][w];
      b += sums[1][w];
    }
    if (b > 0.f) th = fminf(fmaxf(a / b, -0.05f), 0.05f);
  }
  for (int i = tid; i < n; i += blockDim.x) {
    const vsbd_item it = items[i];
    const float dx = med[0] + th * -((float)it.y - cy), dy = med[1] + th * ((float)it.x - cx);
    const int ox = (int)rintf(fminf(fmaxf(dx, -4000.f), 4000.f));
    const int oy = (int)rintf(fminf(fmaxf(dy, -4000.f), 4000.f));
    vsbd_item o = it;
    o.ox = (int16_t)ox;
    o.oy = (int16_t)oy;
    items2[i] = o;
    prior[i] = make_short2((short)ox, (short)oy);
  }
}

#endif
