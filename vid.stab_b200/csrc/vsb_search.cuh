/*
 * vsb_search.cuh -- the per-field SAD search of the detect pass for sm_100a
 * (src/motiondetect.c:439-586 planar spiral, :591-660 packed raster of the
 * reference), shared by the per-stream and the batched paths.
 *
 * Work split.  A field's candidate displacements form a lattice
 * (a, b) -> (ax0 + a*step, by0 + b*step).  One CTA takes a tile of
 * nab x nbb lattice points of one field and stages, once, the field of the
 * current frame and the window of the previous frame those candidates
 * touch.  A thread owns one lattice column a and TB consecutive lattice
 * rows b, and one horizontal strip of the field's rows.  It walks the rows
 * of the window: each previous-frame row it loads serves TB candidates at
 * once (against TB different field rows, which are shared by the whole warp
 * and so read as broadcasts).  Strips are summed in shared memory.
 *
 * Every candidate gets its FULL sum of absolute differences (the reference
 * stops early once a row exceeds the running minimum, which never changes
 * which candidate wins: `error < minerror` only).  The winner is the lowest
 * (SAD, rank) pair, where rank is the candidate's position in the
 * reference's visiting order, so equal SADs resolve exactly as the
 * reference's strict `<` scan does.  CTAs of a field fold their best pair
 * into one 64-bit atomicMin; the last CTA of the field (ticket counter) runs
 * the dependent refinement rounds around the winner and the range test, and
 * resets the field's key and ticket for the next launch.
 */
#ifndef VSB_SEARCH_CUH
#define VSB_SEARCH_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "vsb_device.h"

struct DGeom {
  int S, bpp, step, na, nb, ax0, by0, has_origin, nstages;
  int st_r[VSBD_MAX_STAGES], st_h[VSBD_MAX_STAGES];
  int limx, limy;
  int maxq;             /* largest refinement grid */
  const int32_t* order; /* rank of lattice point (a,b) at [b*na + a] */
  const short2* point;  /* displacement of rank k */
  /* tiling, chosen on the host */
  int tb;               /* lattice rows per thread (the kernel's template value) */
  int nab, nbb;         /* lattice columns / rows per tile (nbb a multiple of tb) */
  int nta, ntb;         /* tiles along a / along b */
  int nstrip;           /* field rows split into this many strips */
  int threads;          /* block size */
  int ta;               /* lattice columns per thread: 1 (or 0); 2 -- a window row's words
                           then serve two candidate columns (step*bpp <= 8); 3 -- two columns
                           of one byte alignment, read from window copies staged word-aligned
                           for them (step*bpp even and <= 8): no shifts in the sums; 4 -- as 3
                           for step*bpp 2 or 6, from one window copy aligned for the even
                           columns, the odd ones summed against a copy of the field shifted
                           by two bytes (edge bytes masked) */
  int rows;             /* field rows a launch sums (0: all S); fewer rows give
                           every candidate a lower bound of its SAD */
  int ctas;             /* ta == 5 (the persistent sweep, vsb_sweep.cuh): its grid */
  unsigned* emit;       /* emit mode: per item, per lattice point, the sum */
  const uint8_t* skip;  /* emit mode: per item, nonzero = field never used */
};

__host__ __device__ inline int geom_rows(const DGeom& g) { return g.rows > 0 ? g.rows : g.S; }

/* packed 4 x u8 sum of absolute differences, accumulated */
__device__ __forceinline__ unsigned sad4(unsigned a, unsigned b, unsigned c) {
  unsigned d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

__device__ __forceinline__ unsigned long long warp_min64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t < v ? t : v;
  }
  return v;
}

/* shared-memory layout of one tile (bytes) */
struct TileLayout {
  int rowB, rowW, nq;
  int WP, WH_alloc;  /* previous-frame window: row pitch, rows */
  int RP, RH;        /* refinement window: row pitch (bytes), rows */
  int FP;            /* row pitch of the staged current-field rows */
  int CP;            /* ta == 3: distance of the second window copy from the first */
  int C1P;           /* ta == 4: row pitch of the shifted field copy (at off_C1) */
  size_t off_C1, off_P, off_part, off_q, total;
};

/* window copies of a ta == 3 tile: two when the lattice step in bytes is 2
   mod 4 (even and odd lattice columns fall on different byte alignments),
   else one */
__host__ __device__ inline int window_copies(const DGeom& g) {
  return g.ta == 3 && ((g.step * g.bpp) & 3) ? 2 : 1;
}

/* total reach of the refinement rounds around the lattice winner */
__host__ __device__ inline int refine_reach(const DGeom& g) {
  int R = 0;
  for (int k = 0; k < g.nstages; k++) R += g.st_r[k];
  return R;
}

__host__ __device__ inline TileLayout tile_layout(const DGeom& g) {
  TileLayout L;
  L.rowB = g.S * g.bpp;
  L.rowW = L.rowB >> 2;
  L.nq = L.rowW >> 2;
  int wwb = L.rowB + (g.nab - 1) * g.step * g.bpp;
  L.WP = (((15 + wwb + 15) >> 4) + 1) << 4;
  const int rows = geom_rows(g);
  L.WH_alloc = rows + (g.nbb - 1) * g.step;
  int R = refine_reach(g);
  L.RH = g.S + 2 * R;
  L.RP = ((3 + L.rowB + 2 * R * g.bpp + 8 + 15) >> 4) << 4;
  L.FP = ((L.rowB + 15 + 15) >> 4 << 4) + 16;
  L.C1P = L.rowB + 16;
  L.off_C1 = (size_t)rows * L.rowB;
  L.off_P = L.off_C1 + (g.ta == 4 ? (size_t)rows * L.C1P : 0);
  /* the second copy sits one word off a 16-byte boundary, so that a warp's
     even- and odd-column threads read different banks */
  L.CP = L.WH_alloc * L.WP + 4;
  size_t parea = (size_t)window_copies(g) * L.CP;
  size_t rarea = g.rows > 0 ? 0 : (size_t)L.RH * L.RP + 16;
  size_t farea = (size_t)rows * L.FP;
  if (rarea > parea) parea = rarea;
  if (farea > parea) parea = farea;
  L.off_part = L.off_P + parea;
  int G = g.nbb / g.tb;
  L.off_q = L.off_part + (size_t)(g.nstrip > 1 ? g.nstrip - 1 : 0) * G * g.tb * g.nab * 4;
  L.total = L.off_q + (size_t)g.maxq * 4 + 16;
  return L;
}

/* SAD of the staged field C (rowW words per row, cpw words apart) against
   rows of a row-major byte buffer whose matching field starts at byte
   column bx (any alignment) of row row0; lanes take field rows, the warp
   sums */
__device__ __forceinline__ unsigned sad_rows_warp(const uint32_t* __restrict__ C, int rowW, int cpw,
                                                  int S, const uint8_t* __restrict__ base,
                                                  size_t pitch, int bx, int row0, int lane) {
  /* lanes stride over the field's words in raster order (consecutive lanes
     read consecutive words: coalesced in global memory, conflict-free in
     shared memory); four words in flight per lane */
  unsigned acc = 0;
  const int sh = (bx & 3) << 3;
  const uint8_t* b0 = base + (size_t)row0 * pitch + (bx & ~3);
  const int total = S * rowW;
  int r = lane / rowW, w = lane - r * rowW;
  int i = lane;
  for (; i + 96 < total; i += 128) {
    uint32_t lo[4], hi[4], cw[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t* Pw = (const uint32_t*)(b0 + (size_t)r * pitch) + w;
      lo[u] = Pw[0];
      hi[u] = Pw[1];
      cw[u] = C[r * cpw + w];
      w += 32;
      while (w >= rowW) { w -= rowW; r++; }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) acc = sad4(cw[u], __funnelshift_r(lo[u], hi[u], sh), acc);
  }
  for (; i < total; i += 32) {
    const uint32_t* Pw = (const uint32_t*)(b0 + (size_t)r * pitch) + w;
    acc = sad4(C[r * cpw + w], __funnelshift_r(Pw[0], Pw[1], sh), acc);
    w += 32;
    while (w >= rowW) { w -= rowW; r++; }
  }
  return __reduce_add_sync(0xffffffffu, acc);
}

/* Last CTA of an item: origin candidate (raster scans), refinement rounds
   (i outer, j inner, centre skipped, strict <), range test, reset.  The
   window the rounds can reach (the field plus the sum of the round radii on
   every side, RH rows of RP bytes) is staged in shared memory (rwin) first.
   C: the field, rowW words per row, cpw words apart. */
static __device__ void refine_and_store(const DGeom& g, int rowW, int cpw, int RH, int RP,
                                        const vsbd_item& it, const uint32_t* C, uint8_t* rwin,
                                        const uint8_t* __restrict__ prev, int pitch,
                                        unsigned long long* keys, unsigned* tickets,
                                        vsbd_result* res, int item, unsigned* qsad) {
  __shared__ int s_tx, s_ty;
  __shared__ unsigned s_min;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
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
      unsigned s0 = sad_rows_warp(C, rowW, cpw, g.S, prev, (size_t)pitch, fx0, fy0, lane);
      if (lane == 0 && s0 <= s_min) { /* rank 0 precedes every lattice rank */
        s_min = s0;
        s_tx = 0;
        s_ty = 0;
      }
    }
    __syncthreads();
  }
  if (g.nstages > 0) {
    const int R = refine_reach(g);
    const int cx0 = s_tx, cy0 = s_ty;
    const int wx = fx0 + (cx0 - R) * g.bpp, wy = fy0 + cy0 - R;
    const int wxa = wx & ~3, off = wx - wxa;
    const int nw = RP >> 2;
    for (int i = threadIdx.x; i < RH * nw; i += blockDim.x) {
      int r = i / nw, w = i - r * nw;
      ((uint32_t*)rwin)[i] = *((const uint32_t*)(prev + (size_t)(wy + r) * pitch + wxa) + w);
    }
    __syncthreads();
    for (int st = 0; st < g.nstages; st++) {
      const int r = g.st_r[st], h = g.st_h[st];
      const int side = (2 * r) / h + 1, nq = side * side;
      const int cx = s_tx, cy = s_ty;
      for (int q = warp; q < nq; q += nwarps) {
        int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
        unsigned sd = 0xffffffffu;
        if (!(i == cx && j == cy))
          sd = sad_rows_warp(C, rowW, cpw, g.S, rwin, (size_t)RP, off + (i - cx0 + R) * g.bpp,
                             j - cy0 + R, lane);
        if (lane == 0) qsad[q] = sd;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned m = s_min;
        int tx = cx, ty = cy;
        for (int q = 0; q < nq; q++) {
          int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
          if (i == cx && j == cy) continue;
          if (qsad[q] < m) {
            m = qsad[q];
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

/* Rows [rb, re) of one thread's walk with candidates JLO..JHI of its TB all
   active: per window row the row's words are loaded once, aligned to the
   thread's column by funnel shifts, and every active candidate j adds the
   row's SAD against its own field row rho - step*j (a warp-wide broadcast).
   No condition inside, so the accumulation chains interleave. */
template <int TB, int JLO, int JHI>
__device__ __forceinline__ void rows_active(unsigned (&acc)[TB], int rb, int re, int step,
                                            const uint8_t* __restrict__ Pb, int WP, int sh,
                                            const uint4* __restrict__ C4, int nq) {
  for (int rho = rb; rho < re; rho++) {
    const uint32_t* Pw = (const uint32_t*)(Pb + rho * WP);
    const uint4* Cj[TB];
#pragma unroll
    for (int j = JLO; j <= JHI; j++) Cj[j] = C4 + (rho - step * j) * nq;
    uint32_t lo = Pw[0];
    for (int q = 0; q < nq; q++) {
      uint32_t p1 = Pw[4 * q + 1], p2 = Pw[4 * q + 2], p3 = Pw[4 * q + 3], p4 = Pw[4 * q + 4];
      uint32_t w0 = __funnelshift_r(lo, p1, sh), w1 = __funnelshift_r(p1, p2, sh);
      uint32_t w2 = __funnelshift_r(p2, p3, sh), w3 = __funnelshift_r(p3, p4, sh);
      lo = p4;
#pragma unroll
      for (int j = JLO; j <= JHI; j++) {
        uint4 c = Cj[j][q];
        acc[j] = sad4(c.x, w0, acc[j]);
        acc[j] = sad4(c.y, w1, acc[j]);
        acc[j] = sad4(c.z, w2, acc[j]);
        acc[j] = sad4(c.w, w3, acc[j]);
      }
    }
  }
}

/* one segment of rows with a constant active range [jlo, jhi]: a uniform
   switch to the body compiled for that range */
template <int TB>
__device__ __forceinline__ void rows_segment(unsigned (&acc)[TB], int jlo, int jhi, int rb, int re,
                                             int step, const uint8_t* Pb, int WP, int sh,
                                             const uint4* C4, int nq) {
#define VSB_SEG(L, H)                                                           \
  if (jlo == L && jhi == H) {                                                   \
    rows_active<TB, L, H>(acc, rb, re, step, Pb, WP, sh, C4, nq);               \
    return;                                                                     \
  }
  if constexpr (TB == 2) {
    VSB_SEG(0, 0) VSB_SEG(0, 1) VSB_SEG(1, 1)
  } else if constexpr (TB == 4) {
    VSB_SEG(0, 0) VSB_SEG(0, 1) VSB_SEG(0, 2) VSB_SEG(0, 3)
    VSB_SEG(1, 1) VSB_SEG(1, 2) VSB_SEG(1, 3)
    VSB_SEG(2, 2) VSB_SEG(2, 3)
    VSB_SEG(3, 3)
  } else if constexpr (TB == 8) {
    VSB_SEG(0, 0) VSB_SEG(0, 1) VSB_SEG(0, 2) VSB_SEG(0, 3) VSB_SEG(0, 4) VSB_SEG(0, 5)
    VSB_SEG(0, 6) VSB_SEG(0, 7) VSB_SEG(1, 1) VSB_SEG(1, 2) VSB_SEG(1, 3) VSB_SEG(1, 4)
    VSB_SEG(1, 5) VSB_SEG(1, 6) VSB_SEG(1, 7) VSB_SEG(2, 2) VSB_SEG(2, 3) VSB_SEG(2, 4)
    VSB_SEG(2, 5) VSB_SEG(2, 6) VSB_SEG(2, 7) VSB_SEG(3, 3) VSB_SEG(3, 4) VSB_SEG(3, 5)
    VSB_SEG(3, 6) VSB_SEG(3, 7) VSB_SEG(4, 4) VSB_SEG(4, 5) VSB_SEG(4, 6) VSB_SEG(4, 7)
    VSB_SEG(5, 5) VSB_SEG(5, 6) VSB_SEG(5, 7) VSB_SEG(6, 6) VSB_SEG(6, 7) VSB_SEG(7, 7)
  }
#undef VSB_SEG
}

/* Rows [rb, re) for a thread owning two lattice columns (ta == 2), the
   second DW words right of the first with its own funnel shift: each quad of
   a window row is loaded once (four new words, three carried) and serves
   both columns of every active candidate row. */
template <int TB, int JLO, int JHI, int DW>
__device__ __forceinline__ void rows_active_ta2(unsigned (&acc)[2][TB], int rb, int re, int step,
                                                const uint8_t* __restrict__ Pb, int WP, int sh0,
                                                int sh1, const uint4* __restrict__ C4, int nq) {
  for (int rho = rb; rho < re; rho++) {
    const uint32_t* Pw = (const uint32_t*)(Pb + rho * WP);
    const uint4* Cj[TB];
#pragma unroll
    for (int j = JLO; j <= JHI; j++) Cj[j] = C4 + (rho - step * j) * nq;
    uint32_t a0 = Pw[0], a1 = Pw[1], a2 = Pw[2];
    for (int q = 0; q < nq; q++) {
      const uint32_t b0 = Pw[4 * q + 3], b1 = Pw[4 * q + 4], b2 = Pw[4 * q + 5], b3 = Pw[4 * q + 6];
      const uint32_t W[7] = { a0, a1, a2, b0, b1, b2, b3 };
      const uint32_t x0 = __funnelshift_r(W[0], W[1], sh0), x1 = __funnelshift_r(W[1], W[2], sh0);
      const uint32_t x2 = __funnelshift_r(W[2], W[3], sh0), x3 = __funnelshift_r(W[3], W[4], sh0);
      const uint32_t y0 = __funnelshift_r(W[DW], W[DW + 1], sh1);
      const uint32_t y1 = __funnelshift_r(W[DW + 1], W[DW + 2], sh1);
      const uint32_t y2 = __funnelshift_r(W[DW + 2], W[DW + 3], sh1);
      const uint32_t y3 = __funnelshift_r(W[DW + 3], W[DW + 4], sh1);
      a0 = b1;
      a1 = b2;
      a2 = b3;
#pragma unroll
      for (int j = JLO; j <= JHI; j++) {
        const uint4 c = Cj[j][q];
        acc[0][j] = sad4(c.x, x0, acc[0][j]);
        acc[1][j] = sad4(c.x, y0, acc[1][j]);
        acc[0][j] = sad4(c.y, x1, acc[0][j]);
        acc[1][j] = sad4(c.y, y1, acc[1][j]);
        acc[0][j] = sad4(c.z, x2, acc[0][j]);
        acc[1][j] = sad4(c.z, y2, acc[1][j]);
        acc[0][j] = sad4(c.w, x3, acc[0][j]);
        acc[1][j] = sad4(c.w, y3, acc[1][j]);
      }
    }
  }
}

template <int TB, int DW>
__device__ __forceinline__ void rows_segment_ta2_dw(unsigned (&acc)[2][TB], int jlo, int jhi,
                                                    int rb, int re, int step, const uint8_t* Pb,
                                                    int WP, int sh0, int sh1, const uint4* C4,
                                                    int nq) {
#define VSB_SEG2(L, H)                                                                 \
  if (jlo == L && jhi == H) {                                                          \
    rows_active_ta2<TB, L, H, DW>(acc, rb, re, step, Pb, WP, sh0, sh1, C4, nq);        \
    return;                                                                            \
  }
  if constexpr (TB == 2) {
    VSB_SEG2(0, 0) VSB_SEG2(0, 1) VSB_SEG2(1, 1)
  } else if constexpr (TB == 4) {
    VSB_SEG2(0, 0) VSB_SEG2(0, 1) VSB_SEG2(0, 2) VSB_SEG2(0, 3)
    VSB_SEG2(1, 1) VSB_SEG2(1, 2) VSB_SEG2(1, 3)
    VSB_SEG2(2, 2) VSB_SEG2(2, 3)
    VSB_SEG2(3, 3)
  }
#undef VSB_SEG2
}

/* segment of a two-column thread: DW, the word distance of its second
   column (0..2), is uniform per thread and chosen once here */
template <int TB>
__device__ __forceinline__ void rows_segment_ta2(unsigned (&acc)[2][TB], int jlo, int jhi, int rb,
                                                 int re, int step, const uint8_t* Pb, int WP,
                                                 int sh0, int sh1, int dw, const uint4* C4,
                                                 int nq) {
  if (dw == 1)
    rows_segment_ta2_dw<TB, 1>(acc, jlo, jhi, rb, re, step, Pb, WP, sh0, sh1, C4, nq);
  else if (dw == 2)
    rows_segment_ta2_dw<TB, 2>(acc, jlo, jhi, rb, re, step, Pb, WP, sh0, sh1, C4, nq);
  else
    rows_segment_ta2_dw<TB, 0>(acc, jlo, jhi, rb, re, step, Pb, WP, sh0, sh1, C4, nq);
}

/* Rows [rb, re) for a thread owning two lattice columns of one byte
   alignment (ta == 3): both read whole words of a window copy staged for
   that alignment, the second DW words right of the first.  Each quad of a
   window row is four new words (DW carried): the first column sums words
   0..3 of carry+new, the second the four new ones. */
template <int TB, int JLO, int JHI, int DW>
__device__ __forceinline__ void rows_active_al(unsigned (&acc)[2][TB], int rb, int re, int step,
                                               const uint32_t* __restrict__ Pw0, int WPw,
                                               const uint4* __restrict__ C4, int nq) {
  for (int rho = rb; rho < re; rho++) {
    const uint32_t* Pw = Pw0 + rho * WPw;
    const uint4* Cj[TB];
#pragma unroll
    for (int j = JLO; j <= JHI; j++) Cj[j] = C4 + (rho - step * j) * nq;
    uint32_t cr[DW];
#pragma unroll
    for (int k = 0; k < DW; k++) cr[k] = Pw[k];
    for (int q = 0; q < nq; q++) {
      const uint32_t n0 = Pw[4 * q + DW], n1 = Pw[4 * q + DW + 1], n2 = Pw[4 * q + DW + 2],
                     n3 = Pw[4 * q + DW + 3];
      /* the first column's words: the first four of carry + new */
      uint32_t X[4];
      if constexpr (DW == 1) {
        X[0] = cr[0]; X[1] = n0; X[2] = n1; X[3] = n2;
        cr[0] = n3;
      } else if constexpr (DW == 2) {
        X[0] = cr[0]; X[1] = cr[1]; X[2] = n0; X[3] = n1;
        cr[0] = n2; cr[1] = n3;
      } else {
        X[0] = cr[0]; X[1] = cr[1]; X[2] = cr[2]; X[3] = n0;
        cr[0] = n1; cr[1] = n2; cr[2] = n3;
      }
#pragma unroll
      for (int j = JLO; j <= JHI; j++) {
        const uint4 c = Cj[j][q];
        acc[0][j] = sad4(c.x, X[0], acc[0][j]);
        acc[1][j] = sad4(c.x, n0, acc[1][j]);
        acc[0][j] = sad4(c.y, X[1], acc[0][j]);
        acc[1][j] = sad4(c.y, n1, acc[1][j]);
        acc[0][j] = sad4(c.z, X[2], acc[0][j]);
        acc[1][j] = sad4(c.z, n2, acc[1][j]);
        acc[0][j] = sad4(c.w, X[3], acc[0][j]);
        acc[1][j] = sad4(c.w, n3, acc[1][j]);
      }
    }
  }
}

template <int TB, int DW>
__device__ __forceinline__ void rows_segment_al_dw(unsigned (&acc)[2][TB], int jlo, int jhi,
                                                   int rb, int re, int step, const uint32_t* Pw0,
                                                   int WPw, const uint4* C4, int nq) {
#define VSB_SEG3(L, H)                                                      \
  if (jlo == L && jhi == H) {                                               \
    rows_active_al<TB, L, H, DW>(acc, rb, re, step, Pw0, WPw, C4, nq);      \
    return;                                                                 \
  }
  if constexpr (TB == 2) {
    VSB_SEG3(0, 0) VSB_SEG3(0, 1) VSB_SEG3(1, 1)
  } else if constexpr (TB == 4) {
    VSB_SEG3(0, 0) VSB_SEG3(0, 1) VSB_SEG3(0, 2) VSB_SEG3(0, 3)
    VSB_SEG3(1, 1) VSB_SEG3(1, 2) VSB_SEG3(1, 3)
    VSB_SEG3(2, 2) VSB_SEG3(2, 3)
    VSB_SEG3(3, 3)
  }
#undef VSB_SEG3
}

/* DW (1..3: the lattice step in bytes times the column distance, in words)
   is uniform per tile */
template <int TB>
__device__ __forceinline__ void rows_segment_al(unsigned (&acc)[2][TB], int jlo, int jhi, int rb,
                                                int re, int step, const uint32_t* Pw0, int WPw,
                                                int dw, const uint4* C4, int nq) {
  if (dw == 3)
    rows_segment_al_dw<TB, 3>(acc, jlo, jhi, rb, re, step, Pw0, WPw, C4, nq);
  else if (dw == 2)
    rows_segment_al_dw<TB, 2>(acc, jlo, jhi, rb, re, step, Pw0, WPw, C4, nq);
  else
    rows_segment_al_dw<TB, 1>(acc, jlo, jhi, rb, re, step, Pw0, WPw, C4, nq);
}

/* Rows [rb, re) for an odd-column thread of layout 4: its columns start
   two bytes into window words, the field copy C1 is shifted by two bytes
   (rowW + 1 words per row, zero outside the field), so word k of a column
   pairs with word k of C1; the halves of the first and the last word that
   lie outside the field are masked off the window words. */
template <int TB, int JLO, int JHI, int DW>
__device__ __forceinline__ void rows_active_fc(unsigned (&acc)[2][TB], int rb, int re, int step,
                                               const uint32_t* __restrict__ Pw0, int WPw,
                                               const uint4* __restrict__ C14, int nq1, int nq) {
  for (int rho = rb; rho < re; rho++) {
    const uint32_t* Pw = Pw0 + rho * WPw;
    const uint4* Cj[TB];
#pragma unroll
    for (int j = JLO; j <= JHI; j++) Cj[j] = C14 + (rho - step * j) * nq1;
    uint32_t cr[DW];
#pragma unroll
    for (int k = 0; k < DW; k++) cr[k] = Pw[k];
    cr[0] &= 0xffff0000u;
    uint32_t m = 0xffff0000u;
    for (int q = 0; q < nq; q++) {
      const uint32_t n0 = Pw[4 * q + DW], n1 = Pw[4 * q + DW + 1], n2 = Pw[4 * q + DW + 2],
                     n3 = Pw[4 * q + DW + 3];
      uint32_t X[4];
      if constexpr (DW == 1) {
        X[0] = cr[0]; X[1] = n0; X[2] = n1; X[3] = n2;
        cr[0] = n3;
      } else if constexpr (DW == 2) {
        X[0] = cr[0]; X[1] = cr[1]; X[2] = n0; X[3] = n1;
        cr[0] = n2; cr[1] = n3;
      } else {
        X[0] = cr[0]; X[1] = cr[1]; X[2] = cr[2]; X[3] = n0;
        cr[0] = n1; cr[1] = n2; cr[2] = n3;
      }
      const uint32_t y0 = n0 & m; /* the second column's first word, at q == 0 */
      m = 0xffffffffu;
#pragma unroll
      for (int j = JLO; j <= JHI; j++) {
        const uint4 c = Cj[j][q];
        acc[0][j] = sad4(c.x, X[0], acc[0][j]);
        acc[1][j] = sad4(c.x, y0, acc[1][j]);
        acc[0][j] = sad4(c.y, X[1], acc[0][j]);
        acc[1][j] = sad4(c.y, n1, acc[1][j]);
        acc[0][j] = sad4(c.z, X[2], acc[0][j]);
        acc[1][j] = sad4(c.z, n2, acc[1][j]);
        acc[0][j] = sad4(c.w, X[3], acc[0][j]);
        acc[1][j] = sad4(c.w, n3, acc[1][j]);
      }
    }
    /* word rowW = 4*nq: the field's last two bytes in its lower half */
    const uint32_t t0 = cr[0] & 0xffffu, t1 = Pw[4 * nq + DW] & 0xffffu;
#pragma unroll
    for (int j = JLO; j <= JHI; j++) {
      const uint32_t cw = ((const uint32_t*)Cj[j])[4 * nq];
      acc[0][j] = sad4(cw, t0, acc[0][j]);
      acc[1][j] = sad4(cw, t1, acc[1][j]);
    }
  }
}

template <int TB, int DW>
__device__ __forceinline__ void rows_segment_fc_dw(unsigned (&acc)[2][TB], int jlo, int jhi,
                                                   int rb, int re, int step, const uint32_t* Pw0,
                                                   int WPw, const uint4* C14, int nq1, int nq) {
#define VSB_SEG4(L, H)                                                            \
  if (jlo == L && jhi == H) {                                                     \
    rows_active_fc<TB, L, H, DW>(acc, rb, re, step, Pw0, WPw, C14, nq1, nq);      \
    return;                                                                       \
  }
  if constexpr (TB == 2) {
    VSB_SEG4(0, 0) VSB_SEG4(0, 1) VSB_SEG4(1, 1)
  } else if constexpr (TB == 4) {
    VSB_SEG4(0, 0) VSB_SEG4(0, 1) VSB_SEG4(0, 2) VSB_SEG4(0, 3)
    VSB_SEG4(1, 1) VSB_SEG4(1, 2) VSB_SEG4(1, 3)
    VSB_SEG4(2, 2) VSB_SEG4(2, 3)
    VSB_SEG4(3, 3)
  }
#undef VSB_SEG4
}

/* bytes o .. o+15 of the 32 bytes lo:hi, o = 4*wo + sh/8 (wo uniform) */
__device__ __forceinline__ uint4 extract16(uint4 lo, uint4 hi, int wo, int sh) {
  uint32_t w0, w1, w2, w3, w4;
  switch (wo) {
    case 0: w0 = lo.x; w1 = lo.y; w2 = lo.z; w3 = lo.w; w4 = hi.x; break;
    case 1: w0 = lo.y; w1 = lo.z; w2 = lo.w; w3 = hi.x; w4 = hi.y; break;
    case 2: w0 = lo.z; w1 = lo.w; w2 = hi.x; w3 = hi.y; w4 = hi.z; break;
    default: w0 = lo.w; w1 = hi.x; w2 = hi.y; w3 = hi.z; w4 = hi.w; break;
  }
  return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                    __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
}

template <int TB, bool EMIT, int AL>
__device__ void lattice_tile_ta2(const uint8_t* __restrict__ curr, const uint8_t* __restrict__ prev,
                                 int pitch, const DGeom& g, const vsbd_item* __restrict__ items,
                                 unsigned long long* __restrict__ keys,
                                 unsigned* __restrict__ tickets, vsbd_result* __restrict__ res,
                                 int item, int tile, unsigned ntiles, uint8_t* sm);

/* One lattice tile of one item, by one CTA: tile = tbi*nta + tai of the
   item's ntiles = nta*ntb tiles; sm: tile_layout(g).total bytes of shared
   memory.  The last of the item's CTAs to finish refines and stores.  TA:
   the tiling's g.ta (1 to 4; 1 for g.ta == 0). */
template <int TB, bool EMIT, int TA = 1>
__device__ __forceinline__ void lattice_tile(const uint8_t* __restrict__ curr,
                                             const uint8_t* __restrict__ prev, int pitch,
                                             const DGeom& g, const vsbd_item* __restrict__ items,
                                             unsigned long long* __restrict__ keys,
                                             unsigned* __restrict__ tickets,
                                             vsbd_result* __restrict__ res, int item, int tile,
                                             unsigned ntiles, uint8_t* sm) {
  if constexpr (TA >= 2) {
    lattice_tile_ta2<TB, EMIT, TA - 2>(curr, prev, pitch, g, items, keys, tickets, res, item,
                                       tile, ntiles, sm);
    return;
  }
  __shared__ unsigned long long red[32];
  __shared__ int s_last;
  const TileLayout L = tile_layout(g);
  const int tbi = tile / g.nta, tai = tile - tbi * g.nta;
  const vsbd_item it = items[item];
  const int a0 = tai * g.nab, b0 = tbi * g.nbb;
  const int na_t = min(g.nab, g.na - a0), nb_t = min(g.nbb, g.nb - b0);
  const int G = g.nbb / TB;
  const int rows = geom_rows(g);
  const int Rs = rows / g.nstrip;
  if (EMIT && g.skip && g.skip[item]) return; /* a field that is never selected */
  uint32_t* C = (uint32_t*)sm; /* the current field, rowB bytes per row */
  uint8_t* P = sm + L.off_P;
  unsigned* part = (unsigned*)(sm + L.off_part);
  unsigned* qsad = (unsigned*)(sm + L.off_q);

  /* the current field: rows staged with 16-byte loads in the (not yet used)
     window space, then re-aligned to word boundaries */
  {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int cx0a = cx0 & ~15, ce = cx0 - cx0a;
    const int nv = (ce + L.rowB + 15) >> 4;
    for (int i = threadIdx.x; i < rows * nv; i += blockDim.x) {
      int r = i / nv, v = i - r * nv;
      *(uint4*)(P + r * L.FP + (v << 4)) =
          *(const uint4*)(curr + (size_t)(cy0 + r) * pitch + cx0a + (v << 4));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rows * L.rowW; i += blockDim.x) {
      int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(P + r * L.FP) + (ce >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], (ce & 3) << 3);
    }
    __syncthreads();
  }
  /* the rows of the previous frame this tile's candidates touch */
  const int gx0 = (it.x - g.S / 2 + it.ox + g.ax0 + a0 * g.step) * g.bpp;
  const int gy0 = it.y - g.S / 2 + it.oy + g.by0 + b0 * g.step;
  const int gx0a = gx0 & ~15, e = gx0 - gx0a;
  {
    const int wwb = L.rowB + (na_t - 1) * g.step * g.bpp;
    const int wh = rows + (nb_t - 1) * g.step;
    const int nvec = (e + wwb + 15) >> 4;
    for (int i = threadIdx.x; i < wh * nvec; i += blockDim.x) {
      int r = i / nvec, v = i - r * nvec;
      *(uint4*)(P + r * L.WP + (v << 4)) =
          *(const uint4*)(prev + (size_t)(gy0 + r) * pitch + gx0a + (v << 4));
    }
  }
  __syncthreads();

  /* thread task: lattice column a (fastest), row group, field strip */
  const int t = threadIdx.x;
  const int ntask = g.nab * G * g.nstrip;
  const bool active = t < ntask;
  int al = t % g.nab, rest = t / g.nab;
  int grp = rest % G, st = rest / G;
  if (!active) { al = 0; grp = 0; st = 0; }
  unsigned acc[TB];
#pragma unroll
  for (int j = 0; j < TB; j++) acc[j] = 0;
  {
    const int r0 = st * Rs;
    const int cxb = e + al * g.step * g.bpp;
    const int sh = (cxb & 3) << 3;
    const uint8_t* Pb = P + (size_t)(r0 + grp * TB * g.step) * L.WP + (cxb & ~3);
    const uint4* C4 = (const uint4*)C + r0 * L.nq;
    /* walk the window rows; the field row of candidate j is rho - step*j,
       inside the strip for j in [jlo(rho), jhi(rho)], a range that changes
       only where rho or rho - Rs crosses a multiple of the step */
    const int nrho = Rs + g.step * (TB - 1);
    for (int rb = 0; rb < nrho;) {
      int jhi = min(TB - 1, rb / g.step);
      int jlo = rb < Rs ? 0 : (rb - Rs) / g.step + 1;
      int re = jhi == TB - 1 ? nrho : min(nrho, (jhi + 1) * g.step);
      int lo_next = Rs + jlo * g.step;
      if (lo_next > rb && lo_next < re) re = lo_next;
      rows_segment<TB>(acc, jlo, jhi, rb, re, g.step, Pb, L.WP, sh, C4, L.nq);
      rb = re;
    }
  }
  /* sum the strips */
  if (g.nstrip > 1) {
    if (active && st > 0)
#pragma unroll
      for (int j = 0; j < TB; j++) part[(((st - 1) * G + grp) * TB + j) * g.nab + al] = acc[j];
    __syncthreads();
    if (active && st == 0)
      for (int s2 = 1; s2 < g.nstrip; s2++)
#pragma unroll
        for (int j = 0; j < TB; j++) acc[j] += part[(((s2 - 1) * G + grp) * TB + j) * g.nab + al];
  }
  if (EMIT) {
    if (active && st == 0 && al < na_t) {
      unsigned* out = g.emit + (size_t)item * g.na * g.nb;
#pragma unroll
      for (int j = 0; j < TB; j++) {
        int bl = grp * TB + j;
        if (bl < nb_t) out[(b0 + bl) * g.na + (a0 + al)] = acc[j];
      }
    }
    return;
  }
  unsigned long long best = ~0ull;
  if (active && st == 0 && al < na_t) {
#pragma unroll
    for (int j = 0; j < TB; j++) {
      int bl = grp * TB + j;
      if (bl < nb_t) {
        unsigned long long key = ((unsigned long long)acc[j] << 32) |
                                 (unsigned)g.order[(b0 + bl) * g.na + (a0 + al)];
        best = key < best ? key : best;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  best = warp_min64(best);
  if (lane == 0) red[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nwarps; w++) best = red[w] < best ? red[w] : best;
    atomicMin(&keys[item], best);
    __threadfence();
    unsigned tk = atomicAdd(&tickets[item], 1u);
    s_last = (tk == ntiles - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  refine_and_store(g, L.rowW, L.rowW, L.RH, L.RP, it, C, P + 16, prev, pitch, keys, tickets, res,
                   item, qsad);
}

/* lattice_tile for two columns per thread, TB rows of a row group and a
   strip of the field; same sums, keys and refinement as lattice_tile.
   g.ta == 2 (AL false, nab even): thread t owns columns 2*(t % (nab/2)) and
   the next, aligned by funnel shifts.  g.ta == 3 (AL true): the columns of
   one byte alignment pair up -- a and a+2 (a = 4*(p/2) + p%2 for pair p,
   nab a multiple of 4) when the step in bytes is 2 mod 4, else a = 2p and
   a+1 -- and each alignment has its own window copy, staged so that its
   columns start on word boundaries.  g.ta == 4 (AL 2, step in bytes 2 or 6,
   nab a multiple of 4): the same pairs from one window copy aligned for the
   even columns; odd-column threads use the field copy shifted by two bytes.
   The first half of the threads takes the even columns, the second half the
   odd ones, so that no warp mixes the two loops. */
template <int TB, bool EMIT, int AL>
__device__ void lattice_tile_ta2(const uint8_t* __restrict__ curr, const uint8_t* __restrict__ prev,
                                 int pitch, const DGeom& g, const vsbd_item* __restrict__ items,
                                 unsigned long long* __restrict__ keys,
                                 unsigned* __restrict__ tickets, vsbd_result* __restrict__ res,
                                 int item, int tile, unsigned ntiles, uint8_t* sm) {
  __shared__ unsigned long long red[32];
  __shared__ int s_last;
  const TileLayout L = tile_layout(g);
  const int tbi = tile / g.nta, tai = tile - tbi * g.nta;
  const vsbd_item it = items[item];
  const int a0 = tai * g.nab, b0 = tbi * g.nbb;
  const int na_t = min(g.nab, g.na - a0), nb_t = min(g.nbb, g.nb - b0);
  const int G = g.nbb / TB;
  const int NAG = g.nab / 2;
  const int rows = geom_rows(g);
  const int Rs = rows / g.nstrip;
  if (EMIT && g.skip && g.skip[item]) return;
  uint32_t* C = (uint32_t*)sm;
  uint8_t* P = sm + L.off_P;
  unsigned* part = (unsigned*)(sm + L.off_part);
  unsigned* qsad = (unsigned*)(sm + L.off_q);
  {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int cx0a = cx0 & ~15, ce = cx0 - cx0a;
    const int nv = (ce + L.rowB + 15) >> 4;
    for (int i = threadIdx.x; i < rows * nv; i += blockDim.x) {
      int r = i / nv, v = i - r * nv;
      *(uint4*)(P + r * L.FP + (v << 4)) =
          *(const uint4*)(curr + (size_t)(cy0 + r) * pitch + cx0a + (v << 4));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rows * L.rowW; i += blockDim.x) {
      int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(P + r * L.FP) + (ce >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], (ce & 3) << 3);
    }
    __syncthreads();
  }
  const int gx0 = (it.x - g.S / 2 + it.ox + g.ax0 + a0 * g.step) * g.bpp;
  const int gy0 = it.y - g.S / 2 + it.oy + g.by0 + b0 * g.step;
  const int gx0a = gx0 & ~15, e = gx0 - gx0a;
  const int sb = g.step * g.bpp; /* lattice step in bytes */
  const int dcol = AL && (sb & 3) ? 2 : 1;
  const int ncopy = AL == 1 ? dcol : 1;
  {
    const int wwb = L.rowB + (na_t - 1) * sb;
    const int wh = rows + (nb_t - 1) * g.step;
    const int nvec = (e + wwb + 15) >> 4;
    if constexpr (AL == 0) {
      for (int i = threadIdx.x; i < wh * nvec; i += blockDim.x) {
        int r = i / nvec, v = i - r * nvec;
        *(uint4*)(P + r * L.WP + (v << 4)) =
            *(const uint4*)(prev + (size_t)(gy0 + r) * pitch + gx0a + (v << 4));
      }
    } else {
      /* copy c starts at window byte c*sb: the columns c, c + 2*dcol, ... (and
         their partners) begin on its word boundaries.  Only the aligned
         16-byte chunks the plain staging reads are read. */
      for (int c = 0; c < ncopy; c++) {
        const int bytes = L.rowB + max(na_t - 1 - c, 0) * sb;
        const int ob = e + c * sb;
        const int o = ob & 15, wo = o >> 2, sh = (o & 3) << 3, u00 = ob >> 4;
        const int nvo = (bytes + 15) >> 4;
        uint8_t* Pc = P + c * L.CP;
        for (int i = threadIdx.x; i < wh * nvo; i += blockDim.x) {
          const int r = i / nvo, v = i - r * nvo;
          const uint8_t* row = prev + (size_t)(gy0 + r) * pitch + gx0a;
          const int u0 = u00 + v;
          uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
          if (u0 < nvec) lo = *(const uint4*)(row + (u0 << 4));
          if (o && u0 + 1 < nvec) hi = *(const uint4*)(row + ((u0 + 1) << 4));
          const uint4 w = extract16(lo, hi, wo, sh);
          uint8_t* dst = Pc + r * L.WP + (v << 4);
          if (c == 0) {
            *(uint4*)dst = w;
          } else {
            uint32_t* d4 = (uint32_t*)dst;
            d4[0] = w.x;
            d4[1] = w.y;
            d4[2] = w.z;
            d4[3] = w.w;
          }
        }
      }
      if constexpr (AL == 2) {
        /* the field shifted right by two bytes: word k of row r holds field
           bytes 4k-2 .. 4k+1, zero outside the field */
        uint32_t* C1 = (uint32_t*)(sm + L.off_C1);
        const int c1w = L.C1P >> 2;
        for (int i = threadIdx.x; i < rows * c1w; i += blockDim.x) {
          const int r = i / c1w, k = i - r * c1w;
          const uint32_t lo = k > 0 && k <= L.rowW ? C[r * L.rowW + k - 1] : 0u;
          const uint32_t hi = k < L.rowW ? C[r * L.rowW + k] : 0u;
          C1[i] = __funnelshift_r(lo, hi, 16);
        }
      }
    }
  }
  __syncthreads();

  int t = threadIdx.x;
  int ntask = NAG * G * g.nstrip;
  int cls = 0;
  if constexpr (AL == 2) {
    /* halves of the block: even-column pairs, then odd-column pairs */
    const int half = (int)blockDim.x >> 1;
    cls = t >= half;
    t -= cls * half;
    ntask >>= 1;
  }
  const bool active = t < ntask;
  const int NAGc = AL == 2 ? NAG >> 1 : NAG;
  int ag = t % NAGc, rest = t / NAGc;
  int grp = rest % G, st = rest / G;
  if (!active) { ag = 0; grp = 0; st = 0; }
  if constexpr (AL == 2) ag = 2 * ag + cls;
  /* the thread's two columns and, for AL 1, the copy it reads */
  if constexpr (AL == 1) cls = dcol == 2 ? (ag & 1) : 0;
  const int al0 = dcol == 2 ? 4 * (ag >> 1) + (ag & 1) : 2 * ag;
  const int col[2] = { al0, al0 + dcol };
  unsigned acc[2][TB];
#pragma unroll
  for (int j = 0; j < TB; j++) acc[0][j] = acc[1][j] = 0;
  {
    const int r0 = st * Rs;
    const int cxb = e + al0 * sb;
    const int cxb1 = cxb + sb;
    const int sh0 = (cxb & 3) << 3, sh1 = (cxb1 & 3) << 3;
    const int dw = AL ? (sb * dcol) >> 2 : (cxb1 >> 2) - (cxb >> 2);
    const size_t rowoff = (size_t)(r0 + grp * TB * g.step) * L.WP;
    const uint8_t* Pb = P + rowoff + (cxb & ~3);
    /* AL 1: column al0 starts at byte (al0 - cls)*sb of copy cls, a word
       boundary; AL 2: at byte al0*sb of the one copy, two bytes into a word
       for the odd columns */
    const uint32_t* Pw0 =
        AL == 2 ? (const uint32_t*)(P + rowoff) + ((al0 * sb) >> 2)
                : (const uint32_t*)(P + cls * L.CP + rowoff) + (((al0 - cls) * sb) >> 2);
    const uint4* C4 = (const uint4*)C + r0 * L.nq;
    const int nrho = Rs + g.step * (TB - 1);
    for (int rb = 0; rb < nrho;) {
      int jhi = min(TB - 1, rb / g.step);
      int jlo = rb < Rs ? 0 : (rb - Rs) / g.step + 1;
      int re = jhi == TB - 1 ? nrho : min(nrho, (jhi + 1) * g.step);
      int lo_next = Rs + jlo * g.step;
      if (lo_next > rb && lo_next < re) re = lo_next;
      if constexpr (AL == 2) {
        if (cls) {
          const uint4* C14 = (const uint4*)(sm + L.off_C1) + (size_t)r0 * (L.C1P >> 4);
          if (dw == 3)
            rows_segment_fc_dw<TB, 3>(acc, jlo, jhi, rb, re, g.step, Pw0, L.WP >> 2, C14,
                                      L.C1P >> 4, L.nq);
          else
            rows_segment_fc_dw<TB, 1>(acc, jlo, jhi, rb, re, g.step, Pw0, L.WP >> 2, C14,
                                      L.C1P >> 4, L.nq);
        } else {
          rows_segment_al<TB>(acc, jlo, jhi, rb, re, g.step, Pw0, L.WP >> 2, dw, C4, L.nq);
        }
      } else if constexpr (AL == 1)
        rows_segment_al<TB>(acc, jlo, jhi, rb, re, g.step, Pw0, L.WP >> 2, dw, C4, L.nq);
      else
        rows_segment_ta2<TB>(acc, jlo, jhi, rb, re, g.step, Pb, L.WP, sh0, sh1, dw, C4, L.nq);
      rb = re;
    }
  }
  if (g.nstrip > 1) {
    if (active && st > 0)
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < TB; j++)
          part[(((st - 1) * G + grp) * TB + j) * g.nab + col[c]] = acc[c][j];
    __syncthreads();
    if (active && st == 0)
      for (int s2 = 1; s2 < g.nstrip; s2++)
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
          for (int j = 0; j < TB; j++)
            acc[c][j] += part[(((s2 - 1) * G + grp) * TB + j) * g.nab + col[c]];
  }
  if (EMIT) {
    if (active && st == 0) {
      unsigned* out = g.emit + (size_t)item * g.na * g.nb;
#pragma unroll
      for (int c = 0; c < 2; c++)
        if (col[c] < na_t)
#pragma unroll
          for (int j = 0; j < TB; j++) {
            int bl = grp * TB + j;
            if (bl < nb_t) out[(b0 + bl) * g.na + (a0 + col[c])] = acc[c][j];
          }
    }
    return;
  }
  unsigned long long best = ~0ull;
  if (active && st == 0) {
#pragma unroll
    for (int c = 0; c < 2; c++)
      if (col[c] < na_t)
#pragma unroll
        for (int j = 0; j < TB; j++) {
          int bl = grp * TB + j;
          if (bl < nb_t) {
            unsigned long long key = ((unsigned long long)acc[c][j] << 32) |
                                     (unsigned)g.order[(b0 + bl) * g.na + (a0 + col[c])];
            best = key < best ? key : best;
          }
        }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  best = warp_min64(best);
  if (lane == 0) red[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nwarps; w++) best = red[w] < best ? red[w] : best;
    atomicMin(&keys[item], best);
    __threadfence();
    unsigned tk = atomicAdd(&tickets[item], 1u);
    s_last = (tk == ntiles - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  refine_and_store(g, L.rowW, L.rowW, L.RH, L.RP, it, C, P + 16, prev, pitch, keys, tickets, res,
                   item, qsad);
}

/* grid (nta*ntb, items); block g.threads; dynamic smem tile_layout(g).total;
   TA == g.ta (1 for 0) */
template <int TB, bool EMIT = false, int TA = 1>
__global__ void __launch_bounds__(512, 1) k_lattice(const uint8_t* __restrict__ curr,
                                                  const uint8_t* __restrict__ prev, int pitch,
                                                  DGeom g, const vsbd_item* __restrict__ items,
                                                  unsigned long long* __restrict__ keys,
                                                  unsigned* __restrict__ tickets,
                                                  vsbd_result* __restrict__ res) {
  extern __shared__ __align__(16) uint8_t sm[];
  lattice_tile<TB, EMIT, TA>(curr, prev, pitch, g, items, keys, tickets, res, blockIdx.y, blockIdx.x,
                         gridDim.x, sm);
}

/* Full search of the items listed in list[0 .. *count) (indices into
   items): persistent CTAs take the (item, tile) units in turn; the last
   tile of an item to finish refines it, as in k_lattice. */
template <int TB, int TA = 1>
__global__ void __launch_bounds__(512, 1) k_lattice_list(const uint8_t* __restrict__ curr,
                                                       const uint8_t* __restrict__ prev, int pitch,
                                                       DGeom g, const vsbd_item* __restrict__ items,
                                                       const int* __restrict__ count,
                                                       const int* __restrict__ list,
                                                       unsigned long long* __restrict__ keys,
                                                       unsigned* __restrict__ tickets,
                                                       vsbd_result* __restrict__ res) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int ntiles = g.nta * g.ntb;
  const int nu = *count * ntiles;
  for (int u = blockIdx.x; u < nu; u += gridDim.x) {
    lattice_tile<TB, false, TA>(curr, prev, pitch, g, items, keys, tickets, res, list[u / ntiles],
                            u % ntiles, ntiles, sm);
    __syncthreads();
  }
}

/* Bound and survivors of one item after the partial pass (one CTA per item).
   The topk candidates with the smallest partial sums (ties by rank) get their
   full SAD; the smallest gives the bound B and the item's starting key.  A
   candidate whose partial sum exceeds B has a full SAD above B and cannot be
   the minimum (nor tie with it), so only candidates with partial <= B
   survive.  Dynamic shared memory: the field (S rows) plus the small lists. */
static __global__ void __launch_bounds__(256) k_prune(const uint8_t* __restrict__ curr,
                                               const uint8_t* __restrict__ prev, int pitch,
                                               DGeom g, const vsbd_item* __restrict__ items,
                                               const unsigned* __restrict__ part, int topk,
                                               unsigned long long* __restrict__ keys,
                                               int* __restrict__ counts, int* __restrict__ lists,
                                               int* __restrict__ boxes) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ unsigned long long red[8];
  __shared__ int chosen[8];
  __shared__ unsigned long long s_best;
  __shared__ int s_count, s_box[4];
  const int item = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int n = g.na * g.nb;
  if (topk > n) topk = n;
  if (g.skip && g.skip[item]) {
    if (threadIdx.x == 0) {
      counts[item] = 0;
      keys[item] = ~0ull;
    }
    return;
  }
  const vsbd_item it = items[item];
  const unsigned* P = part + (size_t)item * n;
  const int rowB = g.S * g.bpp, rowW = rowB >> 2;
  uint32_t* C = (uint32_t*)sm;
  {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int sh = (cx0 & 3) << 3;
    for (int i = threadIdx.x; i < g.S * rowW; i += blockDim.x) {
      int r = i / rowW, w = i - r * rowW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + (cx0 >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
  }
  if (topk > 8) topk = 8;
  for (int k = 0; k < topk; k++) {
    unsigned long long best = ~0ull;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      bool taken = false;
      for (int q = 0; q < k; q++) taken |= chosen[q] == c;
      if (taken) continue;
      unsigned long long key = ((unsigned long long)P[c] << 32) | (unsigned)g.order[c];
      best = key < best ? key : best;
    }
    best = warp_min64(best);
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < nwarps; w++) best = red[w] < best ? red[w] : best;
      short2 pt = g.point[(unsigned)(best & 0xffffffffu)];
      chosen[k] = ((pt.y - g.by0) / g.step) * g.na + (pt.x - g.ax0) / g.step;
    }
    __syncthreads();
  }
  __syncthreads();
  if (threadIdx.x == 0) s_best = ~0ull;
  __syncthreads();
  const int fx0 = (it.x - g.S / 2 + it.ox) * g.bpp, fy0 = it.y - g.S / 2 + it.oy;
  for (int k = warp; k < topk; k += nwarps) {
    int c = chosen[k];
    int a = c % g.na, b = c / g.na;
    unsigned sd = sad_rows_warp(C, rowW, rowW, g.S, prev, (size_t)pitch,
                                fx0 + (g.ax0 + a * g.step) * g.bpp, fy0 + g.by0 + b * g.step, lane);
    if (lane == 0) atomicMin(&s_best, ((unsigned long long)sd << 32) | (unsigned)g.order[c]);
  }
  if (threadIdx.x == 0) {
    s_count = 0;
    s_box[0] = s_box[1] = 1 << 30;
    s_box[2] = s_box[3] = -1;
  }
  __syncthreads();
  const unsigned B = (unsigned)(s_best >> 32);
  int* L = lists + (size_t)item * n;
  int amin = 1 << 30, bmin = 1 << 30, amax = -1, bmax = -1;
  for (int c = threadIdx.x; c < n; c += blockDim.x)
    if (P[c] <= B) {
      L[atomicAdd(&s_count, 1)] = c;
      int a = c % g.na, b = c / g.na;
      amin = min(amin, a);
      amax = max(amax, a);
      bmin = min(bmin, b);
      bmax = max(bmax, b);
    }
  atomicMin(&s_box[0], amin);
  atomicMin(&s_box[1], bmin);
  atomicMax(&s_box[2], amax);
  atomicMax(&s_box[3], bmax);
  __syncthreads();
  if (threadIdx.x == 0) {
    counts[item] = s_count;
    keys[item] = s_best;
    for (int k = 0; k < 4; k++) boxes[item * 4 + k] = s_box[k];
  }
}

/* bytes of shared memory k_survive may use for the survivors' window */
#define VSB_SURVIVE_WINDOW (96 * 1024)

/* Full SADs of the survivors (rows [rows0, S) added to their partial sums),
   folded into the item's key; the last CTA of the item refines.
   grid (chunks, items); each CTA strides over the survivors by gridDim.x. */
static __global__ void __launch_bounds__(256) k_survive(const uint8_t* __restrict__ curr,
                                                 const uint8_t* __restrict__ prev, int pitch,
                                                 DGeom g, int rows0,
                                                 const vsbd_item* __restrict__ items,
                                                 const unsigned* __restrict__ part,
                                                 const int* __restrict__ counts,
                                                 const int* __restrict__ lists,
                                                 const int* __restrict__ boxes,
                                                 unsigned long long* __restrict__ keys,
                                                 unsigned* __restrict__ tickets,
                                                 vsbd_result* __restrict__ res) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ int s_last;
  const int item = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int n = g.na * g.nb;
  const int cnt = counts[item];
  const bool skipped = g.skip && g.skip[item];
  const vsbd_item it = items[item];
  const TileLayout L = tile_layout(g);
  uint32_t* C = (uint32_t*)sm;
  bool staged = false;
  if (!skipped && (int)blockIdx.x < cnt) {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int sh = (cx0 & 3) << 3;
    for (int i = threadIdx.x; i < g.S * L.rowW; i += blockDim.x) {
      int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + (cx0 >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
    staged = true;
    __syncthreads();
    const int fx0 = (it.x - g.S / 2 + it.ox) * g.bpp, fy0 = it.y - g.S / 2 + it.oy;
    const unsigned* P = part + (size_t)item * n;
    const int* Ls = lists + (size_t)item * n;
    /* the window of the remaining rows [rows0, S) every survivor can touch:
       survivors' lattice bounding box, staged with 16-byte loads when it fits */
    const int amin = boxes[item * 4], bmin = boxes[item * 4 + 1];
    const int amax = boxes[item * 4 + 2], bmax = boxes[item * 4 + 3];
    const int rowsR = g.S - rows0;
    const int wx = fx0 + (g.ax0 + amin * g.step) * g.bpp;
    const int wy = fy0 + g.by0 + bmin * g.step + rows0;
    const int wxa = wx & ~15, we = wx - wxa;
    const int wwb = we + L.rowB + (amax - amin) * g.step * g.bpp;
    const int wh = rowsR + (bmax - bmin) * g.step;
    const int nv = (wwb + 15) >> 4;
    const int WPs = (nv + 1) << 4;
    uint8_t* win = sm + (size_t)g.S * L.rowB + 16;
    /* staging pays when this CTA's survivors read the window's bytes several
       times over; otherwise they read the frame directly */
    const int mine = (cnt - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    const bool in_smem = (size_t)wh * WPs + 16 <= VSB_SURVIVE_WINDOW &&
                         (size_t)wh * WPs <= (size_t)2 * mine * rowsR * L.rowB;
    if (in_smem) {
      for (int i = threadIdx.x; i < wh * nv; i += blockDim.x) {
        int r = i / nv, v = i - r * nv;
        *(uint4*)(win + r * WPs + (v << 4)) =
            *(const uint4*)(prev + (size_t)(wy + r) * pitch + wxa + (v << 4));
      }
      __syncthreads();
    }
    for (int q = blockIdx.x + gridDim.x * warp; q < cnt; q += gridDim.x * nwarps) {
      int c = Ls[q];
      int a = c % g.na, b = c / g.na;
      unsigned sd;
      if (in_smem)
        sd = sad_rows_warp(C + rows0 * L.rowW, L.rowW, L.rowW, rowsR, win, (size_t)WPs,
                           we + (a - amin) * g.step * g.bpp, (b - bmin) * g.step, lane);
      else
        sd = sad_rows_warp(C + rows0 * L.rowW, L.rowW, L.rowW, rowsR, prev, (size_t)pitch,
                           fx0 + (g.ax0 + a * g.step) * g.bpp, fy0 + g.by0 + b * g.step + rows0,
                           lane);
      if (lane == 0)
        atomicMin(&keys[item], ((unsigned long long)(sd + P[c]) << 32) | (unsigned)g.order[c]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned tk = atomicAdd(&tickets[item], 1u);
    s_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (skipped) {
    if (threadIdx.x == 0) {
      vsbd_result o;
      o.sad = 0xffffffffu;
      o.tx = o.ty = 0;
      o.ok = 0;
      res[item] = o;
      keys[item] = ~0ull;
      tickets[item] = 0u;
    }
    return;
  }
  if (!staged) {
    const int cx0 = (it.x - g.S / 2) * g.bpp, cy0 = it.y - g.S / 2;
    const int sh = (cx0 & 3) << 3;
    for (int i = threadIdx.x; i < g.S * L.rowW; i += blockDim.x) {
      int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + (cx0 >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
    __syncthreads();
  }
  uint8_t* rwin = sm + (size_t)g.S * L.rowB;
  unsigned* qsad = (unsigned*)(rwin + (size_t)L.RH * L.RP + 32);
  refine_and_store(g, L.rowW, L.rowW, L.RH, L.RP, it, C, rwin + 16, prev, pitch, keys, tickets,
                   res, item, qsad);
}

/* shared memory of k_survive: field, refinement window, refinement SADs */
__host__ inline size_t survive_smem(const DGeom& g) {
  DGeom f = g;
  f.rows = 0;
  TileLayout L = tile_layout(f);
  size_t ref = (size_t)L.RH * L.RP + 32 + (size_t)g.maxq * 4 + 16;
  size_t win = VSB_SURVIVE_WINDOW + 32;
  return (size_t)g.S * L.rowB + (ref > win ? ref : win);
}

/* tiling of a field set by the cost model (vsb_device.cu) */
int vsbd_plan_search(const vsbd_geom* h, int nitems, DGeom* out);

#endif
