/*
 * vsb_finewarp.cuh -- full search of small fields (the fine pass), one CTA
 * of a few warps per field (k_fine).
 *
 * A fine field's whole search fits in shared memory: for 32x32 fields with a
 * shift range of +-32 at lattice step 2 the previous-frame window is 98 x 98
 * bytes.  One CTA per item stages that window once (16-byte loads), builds
 * two byte-shifted copies of it so that every candidate column of the lattice
 * reads whole words (candidate columns 2 bytes apart fall on two alignments),
 * and sums every lattice candidate: a thread takes 8 consecutive lattice
 * columns of one lattice row and keeps 8 accumulators of packed sums of
 * absolute differences (vabsdiff4.add), the field row a broadcast from shared
 * memory.  The lowest (SAD, visiting rank) wins, as in every other search of
 * this library (the reference's strict `<` over its spiral order); the CTA
 * then refines the winner from the same staged window (src/motiondetect.c:
 * 545-567 of the reference: i outer, j inner, centre skipped, strict <) and
 * applies the range test (:573-574).  No tickets, no atomics: the CTA owns
 * the item.  Planar frames, even lattice steps (the fine pass uses 2).
 */
#ifndef VSB_FINEWARP_CUH
#define VSB_FINEWARP_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "vsb_search.cuh"

#define FW_MAX_WARPS 16

/* shared memory of one item */
struct FWLayout {
  int WH, WW;  /* window rows, bytes per row the candidates and refinement read */
  int RP;      /* staged raw row pitch (bytes, 16-aligned, with slack) */
  int WPW;     /* shifted-copy row pitch (words): a row's words, then room
                  for its skew */
  size_t off_raw, off_c0, off_c1, off_f, off_red, off_part, total;
};

/* tasks of one item: 8-column groups x blocks of T lattice rows x strips */
__host__ __device__ inline int fw_tasks(const DGeom& g, int T, int ns) {
  return ((g.na + 7) / 8) * ((g.nb + T - 1) / T) * ns;
}

__host__ __device__ inline FWLayout fw_layout(const DGeom& g, int threads, int T, int ns) {
  FWLayout L;
  const int R = refine_reach(g);
  L.WH = g.S + (g.nb - 1) * g.step + 2 * R;
  L.WW = g.S + (g.na - 1) * g.step + 2 * R;
  const int words = (15 + L.WW + 3) / 4 + 6; /* words of a copy row the sums read */
  L.WPW = words + 4;                          /* + the row skew (0..3 words) */
  L.RP = (4 * (words + 2) + 15) & ~15;        /* every raw word the copies read */
  L.off_raw = 0;
  L.off_c0 = L.off_raw + (size_t)L.WH * L.RP;
  L.off_c1 = L.off_c0 + (size_t)L.WH * L.WPW * 4;
  L.off_f = L.off_c1 + (size_t)L.WH * L.WPW * 4;
  L.off_f = (L.off_f + 15) & ~(size_t)15;
  L.off_red = L.off_f + (size_t)g.S * g.S;
  L.off_part = L.off_red + FW_MAX_WARPS * 8;
  /* the refinement's partials, or the strips' partial sums */
  const int np = ns > 1 ? fw_tasks(g, T, ns) * 8 * T : 0;
  L.total = L.off_part + (size_t)(threads > np ? threads : np) * 4 + 16;
  return L;
}

/* the fine pass's geometries this kernel takes */
__host__ __device__ inline bool fw_supported(const DGeom& g) {
  return g.bpp == 1 && !g.has_origin && g.step == 2 && (g.S == 16 || g.S == 32 || g.S == 48) &&
         g.na <= 64 && g.nb <= 64;
}

/* Copy row y starts (y >> sh) & 3 words into its slot of WPW words: the
   threads of a warp read rows 2T apart (T lattice rows each), and the skew
   spreads them over the shared-memory banks. */
__device__ __forceinline__ int fw_row(int y, int WPW, int sh) { return y * WPW + ((y >> sh) & 3); }

/* The sums of lattice columns ag*8 .. ag*8+7 and lattice rows b0 .. b0+nv-1
   (nv <= T): acc[t*8 + k] for column ag*8 + k, row b0 + t.  Column a reads,
   for field word w of row r, the window bytes at e + R + 2a + 4w: word
   J0 + jo(k) + w of copy (k & 1), whose words start s0 (even k) or s0 ^ 2
   (odd k) bytes into the raw row; LO says whether s0 < 2 (odd columns then
   start one word earlier).  The window rows are walked once: row y0 + yr
   serves lattice row b0 + t with field row yr - 2t; only field rows
   [r0, r1) (a strip) are summed. */
template <int S, bool LO, int T>
__device__ __forceinline__ void fw_sums(const uint32_t* __restrict__ F, const uint32_t* __restrict__ c0,
                                        const uint32_t* __restrict__ c1, int WPW, int sh, int y0,
                                        int nv, int J0, int r0, int r1, unsigned* acc) {
  constexpr int NW = S / 4;
#pragma unroll
  for (int k = 0; k < 8 * T; k++) acc[k] = 0;
  const int ny = r1 + 2 * (nv - 1);
#pragma unroll 1
  for (int yr = r0; yr < ny; yr++) {
    const int rw = fw_row(y0 + yr, WPW, sh) + J0;
    uint32_t x0[NW + 4], x1[NW + 4];
#pragma unroll
    for (int j = 0; j < NW + 4; j++) {
      x0[j] = c0[rw + j];
      x1[j] = c1[rw + j];
    }
#pragma unroll
    for (int t = 0; t < T; t++) {
      const int r = yr - 2 * t;
      if (t < nv && r >= r0 && r < r1) {
        uint32_t f[NW];
#pragma unroll
        for (int q = 0; q < NW / 4; q++) {
          const uint4 v = *(const uint4*)(F + r * NW + 4 * q);
          f[4 * q] = v.x;
          f[4 * q + 1] = v.y;
          f[4 * q + 2] = v.z;
          f[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
          /* even k: copy 0, word offset k/2; odd k: copy 1, offset (k-1)/2
             when s0 < 2, else (k+1)/2 */
          const int jo = (k & 1) ? (LO ? (k - 1) / 2 : (k + 1) / 2) : k / 2;
#pragma unroll
          for (int w = 0; w < NW; w++)
            acc[8 * t + k] = sad4(f[w], (k & 1) ? x1[jo + w] : x0[jo + w], acc[8 * t + k]);
        }
      }
    }
  }
}

/* The search of item `item` by the calling CTA (blockDim.x = 32 * warps,
   sm holding fw_layout(g, blockDim.x, T, ns).total bytes); a thread takes
   8 lattice columns x T lattice rows x one of ns strips of the field rows
   (the strips' partial sums are added in shared memory). */
template <int S, int T>
__device__ __forceinline__ void fine_item(uint8_t* sm, const uint8_t* __restrict__ curr,
                                          const uint8_t* __restrict__ prev, int pitch,
                                          const DGeom& g, const vsbd_item* __restrict__ items,
                                          vsbd_result* __restrict__ res, int ns, int item) {
  __shared__ int s_tx, s_ty;
  __shared__ unsigned s_min;
  constexpr int NW = S / 4;
  const int nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const FWLayout L = fw_layout(g, nt, T, ns);
  const int R = refine_reach(g);
  const vsbd_item it = items[item];
  const int cx0 = it.x - S / 2, cy0 = it.y - S / 2;
  const int fx0 = cx0 + it.ox, fy0 = cy0 + it.oy;
  const int wx0 = fx0 + g.ax0 - R, wy0 = fy0 + g.by0 - R;
  const int wxa = wx0 & ~15, e = wx0 - wxa;
  uint8_t* raw = sm + L.off_raw;
  uint32_t* c0 = (uint32_t*)(sm + L.off_c0);
  uint32_t* c1 = (uint32_t*)(sm + L.off_c1);
  uint32_t* F = (uint32_t*)(sm + L.off_f);
  unsigned long long* red = (unsigned long long*)(sm + L.off_red);
  unsigned* part = (unsigned*)(sm + L.off_part);
  /* the window (16-byte loads) and the field (word-aligned by funnel shifts) */
  {
    const int nv = L.RP >> 4, tot = L.WH * nv;
    for (int i0 = tid; i0 < tot; i0 += 4 * nt) {
      uint4 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u * nt;
        if (i < tot) {
          const int r = i / nv, c = i - r * nv;
          v[u] = *(const uint4*)(prev + (size_t)(wy0 + r) * pitch + wxa + 16 * c);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u * nt;
        if (i < tot) {
          const int r = i / nv, c = i - r * nv;
          *(uint4*)(raw + (size_t)r * L.RP + 16 * c) = v[u];
        }
      }
    }
    const int sh = (cx0 & 3) * 8;
    for (int i = tid; i < S * NW; i += nt) {
      const int r = i / NW, w = i - r * NW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch + (cx0 & ~3)) + w;
      F[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
  }
  __syncthreads();
  /* the two shifted copies: word j of copy c holds raw bytes 4j + s_c .. + 3 */
  const int s0 = (e + R) & 3, s1 = s0 ^ 2;
  const int sh = T == 4 ? 3 : T == 2 ? 2 : 1; /* log2(2T): rows between a warp's threads */
  const int nword = L.WPW - 4;
  for (int i = tid; i < L.WH * nword; i += nt) {
    const int r = i / nword, j = i - r * nword;
    const uint32_t* rw = (const uint32_t*)(raw + (size_t)r * L.RP) + j;
    const uint32_t a = rw[0], b = rw[1];
    const int o = fw_row(r, L.WPW, sh) + j;
    c0[o] = __funnelshift_r(a, b, 8 * s0);
    c1[o] = __funnelshift_r(a, b, 8 * s1);
  }
  __syncthreads();
  /* every lattice candidate: a thread takes 8 columns of one lattice row */
  const int ngrp = (g.na + 7) >> 3, nbt = (g.nb + T - 1) / T, ntask0 = ngrp * nbt;
  const int rs = S / ns; /* field rows of a strip */
  unsigned long long best = ~0ull;
  for (int t = tid; t < ntask0 * ns; t += nt) {
    const int strip = t / ntask0, t0 = t - strip * ntask0;
    const int ag = t0 / nbt, b0 = (t0 - ag * nbt) * T;
    const int nv = min(T, g.nb - b0);
    const int J0 = (e + R + 16 * ag - s0) >> 2;
    unsigned acc[8 * T];
    if (s0 < 2)
      fw_sums<S, true, T>(F, c0, c1, L.WPW, sh, R + 2 * b0, nv, J0, strip * rs, strip * rs + rs,
                          acc);
    else
      fw_sums<S, false, T>(F, c0, c1, L.WPW, sh, R + 2 * b0, nv, J0, strip * rs, strip * rs + rs,
                           acc);
    if (ns > 1) {
#pragma unroll
      for (int i = 0; i < 8 * T; i++) part[t * 8 * T + i] = acc[i];
    } else {
#pragma unroll
      for (int u = 0; u < T; u++)
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int a = ag * 8 + k, b = b0 + u;
          if (u < nv && a < g.na) {
            const unsigned long long key =
                ((unsigned long long)acc[8 * u + k] << 32) | (unsigned)g.order[b * g.na + a];
            best = key < best ? key : best;
          }
        }
    }
  }
  if (ns > 1) {
    /* each candidate's total over the strips */
    __syncthreads();
    for (int q = tid; q < ntask0 * 8 * T; q += nt) {
      const int t0 = q / (8 * T), i = q - t0 * (8 * T);
      const int ag = t0 / nbt, b = (t0 - ag * nbt) * T + i / 8, a = ag * 8 + (i & 7);
      if (b >= g.nb || a >= g.na) continue;
      unsigned sum = 0;
      for (int st = 0; st < ns; st++) sum += part[(st * ntask0 + t0) * 8 * T + i];
      const unsigned long long key =
          ((unsigned long long)sum << 32) | (unsigned)g.order[b * g.na + a];
      best = key < best ? key : best;
    }
  }
  best = warp_min64(best);
  if (lane == 0) red[warp] = best;
  __syncthreads();
  if (tid == 0) {
    for (int w2 = 1; w2 < (nt >> 5); w2++) best = red[w2] < best ? red[w2] : best;
    const short2 pt = g.point[(unsigned)(best & 0xffffffffu)];
    s_min = (unsigned)(best >> 32);
    s_tx = pt.x;
    s_ty = pt.y;
  }
  __syncthreads();
  /* refinement rounds from the staged window: candidate (i, j) reads raw
     bytes e + R + (i - ax0) + x of row R + (j - by0) + r */
  const uint32_t* raw32 = (const uint32_t*)raw;
  const int RPW = L.RP >> 2;
  for (int st = 0; st < g.nstages; st++) {
    const int r = g.st_r[st], h = g.st_h[st];
    const int side = (2 * r) / h + 1, nq = side * side;
    const int cx = s_tx, cy = s_ty;
    const int G = nt / nq;
    if (G > 0 && tid < nq * G) {
      const int q = tid % nq, grp = tid / nq;
      const int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
      const int bx = e + R + (i - g.ax0), by = R + (j - g.by0);
      const int sh = (bx & 3) * 8;
      unsigned acc = 0;
      for (int rr = grp; rr < S; rr += G) {
        const uint32_t* W = raw32 + (size_t)(by + rr) * RPW + (bx >> 2);
#pragma unroll
        for (int w = 0; w < NW; w++) acc = sad4(F[rr * NW + w], __funnelshift_r(W[w], W[w + 1], sh), acc);
      }
      part[grp * nq + q] = acc;
    }
    __syncthreads();
    if (tid == 0) {
      unsigned m = s_min;
      int tx = cx, ty = cy;
      for (int q = 0; q < nq; q++) {
        const int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
        if (i == cx && j == cy) continue;
        unsigned sd = 0;
        for (int gg = 0; gg < G; gg++) sd += part[gg * nq + q];
        if (sd < m) {
          m = sd;
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
  if (tid == 0) {
    vsbd_result o;
    o.sad = s_min;
    o.tx = (int16_t)s_tx;
    o.ty = (int16_t)s_ty;
    o.ok = !(abs(s_tx) >= g.limx || abs(s_ty) >= g.limy);
    res[item] = o;
  }
}

/* One CTA (blockDim.x = 32 * warps) per item of items[0 .. n). */
template <int S, int T>
__global__ void __launch_bounds__(FW_MAX_WARPS * 32) k_fine(const uint8_t* __restrict__ curr,
                                                          const uint8_t* __restrict__ prev,
                                                          int pitch, DGeom g,
                                                          const vsbd_item* __restrict__ items,
                                                          vsbd_result* __restrict__ res, int ns) {
  extern __shared__ __align__(16) uint8_t sm[];
  fine_item<S, T>(sm, curr, prev, pitch, g, items, res, ns, blockIdx.x);
}

#endif
