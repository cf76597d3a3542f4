/*
 * vsb_blurmm.cuh -- the planar prefilter and the field min/max in one
 * launch (k_blurmm): box blur of plane 0 (src/boxblur.c:104-332 of the
 * reference: horizontal window sums with edge replication, floor division
 * by the size, then the same vertically) and the 8-bit minimum and maximum
 * of every coarse and fine field of the blurred plane
 * (src/motiondetect.c:389-407), without a second pass over the plane.
 *
 * Work split: one warp owns a block of 128 columns x BM_ROWS rows of the
 * output, each lane 4 adjacent columns (one 32-bit word per row); a CTA
 * stacks BM_WARPS warps vertically.  A lane loads all BM_ROWS + 2*HALF input
 * words of its column group first (one memory round trip; the block's edge
 * lanes also load the words beyond it) and stages them in shared memory.
 * A rolled loop then takes one row per iteration (compact code: each warp
 * runs the body once per row, so a fully unrolled body would stall on
 * instruction fetch): the horizontal window sums from the word and its two
 * neighbours (byte permutes and packed sums of absolute differences against
 * zero), and the vertical window over the last 2*HALF+1 horizontal rows on
 * two words of 16-bit lanes (even and odd bytes).  For every field that meets
 * the block (a list made on the host when the detector is created: field,
 * column range, row mask), the warp reduces the masked output bytes and one
 * lane folds them into the field's global minimum and maximum with atomics.  The last CTA to finish (a ticket) writes the (min, max) byte
 * pairs, the coarse fields' contrast flags, and resets the accumulators and
 * the ticket for the next launch.
 */
#ifndef VSB_BLURMM_CUH
#define VSB_BLURMM_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "vsb_prefilter.cuh"

#define BM_COLS 128
#define BM_ROWS 8
#define BM_WARPS 4
#define BM_MAXHALF 4

struct BMArgs {
  const uint8_t* src;
  int sp;
  uint8_t* dst;
  int dp;
  int W, H;
  BlurDiv dv;
  const int* lofs;    /* per warp block: its first list entry (nwb + 1 entries) */
  const uint2* list;  /* x: field | clo << 16 | chi << 24 (columns of the block), y: row mask */
  int nbx;            /* warp blocks across the frame */
  unsigned* acc;      /* running min at 2f, max at 2f + 1 */
  unsigned* ticket;
  int nc, nfields;    /* coarse fields first, then the fine ones */
  uint8_t* out;       /* (min, max) byte pairs of every field */
  double thr;         /* coarse contrast threshold */
  uint8_t* skip;      /* coarse fields below it (may be NULL) */
};

/* the word of 4 bytes at columns x .. x+3 of row gy, columns clamped to the
   frame (edge replication) */
__device__ __forceinline__ uint32_t bm_word(const uint8_t* __restrict__ src, int sp, int W, int gy,
                                            int x) {
  const uint8_t* row = src + (size_t)gy * sp;
  if (x >= 0 && x + 4 <= W) return __ldg((const uint32_t*)(row + x));
  uint32_t w = 0;
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const int c = min(max(x + b, 0), W - 1);
    w |= (uint32_t)__ldg(row + c) << (8 * b);
  }
  return w;
}

/* sum of the bytes B[s .. s+n) of the 12-byte row piece B = (L, M, R) */
template <int S, int N>
__device__ __forceinline__ unsigned bm_window(uint32_t L, uint32_t M, uint32_t R) {
  unsigned acc = 0;
#pragma unroll
  for (int c = 0; c * 4 < N; c++) {
    const int s = S + 4 * c;
    const int len = (N - 4 * c) < 4 ? (N - 4 * c) : 4;
    uint32_t w;
    if (s + 3 <= 7) {
      const unsigned sel = (unsigned)(s | ((s + 1) << 4) | ((s + 2) << 8) | ((s + 3) << 12));
      w = __byte_perm(L, M, sel);
    } else {
      const int t = s - 4;
      const unsigned sel = (unsigned)(t | ((t + 1) << 4) | ((t + 2) << 8) | ((t + 3) << 12));
      w = __byte_perm(M, R, sel);
    }
    if (len < 4) w &= (1u << (8 * len)) - 1u;
    acc = __vsadu4(w, 0u) + acc;
  }
  return acc;
}

/* the four output bytes of one row piece: window sums of 2*HALF+1 bytes
   centred on bytes 4..7 of (L, M, R), each divided by the size with the
   multiply-high (exact: the largest sum times the size stays far below
   2^32 for half-widths up to 4).  For the default half-width 3 every window
   covers M: its sum is shared and each output adds the 3 bytes it takes from
   L and R, gathered by one byte permute */
template <int HALF>
__device__ __forceinline__ uint32_t bm_hrow(uint32_t L, uint32_t M, uint32_t R, unsigned mul) {
  unsigned s0, s1, s2, s3;
  if (HALF == 3) {
    const unsigned q = __vsadu4(M, 0u);
    s0 = __vsadu4(__byte_perm(L, R, 0x0321) & 0x00ffffffu, 0u) + q;
    s1 = __vsadu4(__byte_perm(L, R, 0x0432) & 0x00ffffffu, 0u) + q;
    s2 = __vsadu4(__byte_perm(L, R, 0x0543) & 0x00ffffffu, 0u) + q;
    s3 = __vsadu4(__byte_perm(L, R, 0x0654) & 0x00ffffffu, 0u) + q;
  } else {
    constexpr int WIN = 2 * HALF + 1;
    s0 = bm_window<4 - HALF, WIN>(L, M, R);
    s1 = bm_window<5 - HALF, WIN>(L, M, R);
    s2 = bm_window<6 - HALF, WIN>(L, M, R);
    s3 = bm_window<7 - HALF, WIN>(L, M, R);
  }
  return __byte_perm(__byte_perm(__umulhi(s0, mul), __umulhi(s1, mul), 0x0040),
                     __byte_perm(__umulhi(s2, mul), __umulhi(s3, mul), 0x0040), 0x5410);
}

template <int HALF>
__global__ void __launch_bounds__(32 * BM_WARPS) k_blurmm(BMArgs A) {
  static_assert(HALF >= 1 && HALF <= BM_MAXHALF, "half-width");
  const unsigned mul = A.dv.mul;
  constexpr int RIN = BM_ROWS + 2 * HALF, WIN = 2 * HALF + 1;
  constexpr int RAWP = 34; /* words of a staged row: left halo, 32 lanes, right halo */
  __shared__ uint32_t s_raw[BM_WARPS][RIN][RAWP];
  __shared__ uint32_t s_hor[BM_WARPS][RIN][32];
  __shared__ uint32_t s_out[BM_WARPS][BM_ROWS][32];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int band = blockIdx.y * BM_WARPS + warp;
  const int x0 = blockIdx.x * BM_COLS, y0 = band * BM_ROWS;
  const int x = x0 + 4 * lane;
  if (y0 < A.H) {
    /* every input word of the block first (one round trip), then shared:
       lane l loads its column group of every row, and the block's 2*RIN
       halo words (left and right of every row) are spread over the lanes */
    {
      uint32_t in[RIN];
      const bool inside = __all_sync(0xffffffffu, x0 >= 0 && x0 + BM_COLS <= A.W);
      if (inside) {
#pragma unroll
        for (int r = 0; r < RIN; r++) {
          const int gy = min(max(y0 - HALF + r, 0), A.H - 1);
          in[r] = __ldg((const uint32_t*)(A.src + (size_t)gy * A.sp + x));
        }
      } else {
#pragma unroll
        for (int r = 0; r < RIN; r++) {
          const int gy = min(max(y0 - HALF + r, 0), A.H - 1);
          in[r] = bm_word(A.src, A.sp, A.W, gy, x);
        }
      }
      uint32_t hw[(2 * RIN + 31) / 32];
#pragma unroll
      for (int u = 0; u < (2 * RIN + 31) / 32; u++) {
        const int k = lane + 32 * u, r = k >> 1;
        if (r < RIN) {
          const int gy = min(max(y0 - HALF + r, 0), A.H - 1);
          hw[u] = bm_word(A.src, A.sp, A.W, gy, (k & 1) ? x0 + BM_COLS : x0 - 4);
        }
      }
#pragma unroll
      for (int r = 0; r < RIN; r++) s_raw[warp][r][lane + 1] = in[r];
#pragma unroll
      for (int u = 0; u < (2 * RIN + 31) / 32; u++) {
        const int k = lane + 32 * u, r = k >> 1;
        if (r < RIN) s_raw[warp][r][(k & 1) ? RAWP - 1 : 0] = hw[u];
      }
    }
    __syncwarp();
    /* one row per iteration: its horizontal windows, then the vertical
       window (even / odd bytes as 16-bit lanes) over the last WIN rows */
    unsigned se = 0, so = 0;
#pragma unroll 2
    for (int r = 0; r < RIN; r++) {
      const uint32_t h = bm_hrow<HALF>(s_raw[warp][r][lane], s_raw[warp][r][lane + 1],
                                       s_raw[warp][r][lane + 2], mul);
      s_hor[warp][r][lane] = h;
      se += __byte_perm(h, 0u, 0x4240);
      so += __byte_perm(h, 0u, 0x4341);
      if (r >= WIN) {
        const uint32_t old = s_hor[warp][r - WIN][lane];
        se -= __byte_perm(old, 0u, 0x4240);
        so -= __byte_perm(old, 0u, 0x4341);
      }
      if (r >= WIN - 1) {
        const int i = r - (WIN - 1);
        const unsigned b0 = __umulhi(se & 0xffffu, mul), b2 = __umulhi(se >> 16, mul);
        const unsigned b1 = __umulhi(so & 0xffffu, mul), b3 = __umulhi(so >> 16, mul);
        const uint32_t o =
            __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
        s_out[warp][i][lane] = o;
        const int gy = y0 + i;
        if (gy < A.H && x < A.W) {
          uint8_t* d = A.dst + (size_t)gy * A.dp + x;
          if (x + 4 <= A.W) {
            *(uint32_t*)d = o;
          } else {
            for (int b = 0; x + b < A.W; b++) d[b] = (uint8_t)(o >> (8 * b));
          }
        }
      }
    }
    /* the fields meeting this block: masked min / max over the intersection
       rows of each lane's output words (written by this lane) */
    const int wb = band * A.nbx + blockIdx.x;
    const int e1 = A.lofs[wb + 1];
#pragma unroll 1
    for (int e = A.lofs[wb]; e < e1; e++) {
      const uint2 ent = A.list[e];
      const int f = (int)(ent.x & 0xffffu);
      const int clo = (int)((ent.x >> 16) & 0xffu) - 4 * lane;
      const int chi = (int)(ent.x >> 24) - 4 * lane;
      unsigned m = 0;
#pragma unroll
      for (int b = 0; b < 4; b++)
        if (b >= clo && b < chi) m |= 0xffu << (8 * b);
      const int rlo = __ffs(ent.y) - 1, rhi = 32 - __clz(ent.y);
      unsigned mn = 0xffffffffu, mx = 0u;
#pragma unroll 1
      for (int i = rlo; i < rhi; i++) {
        const uint32_t o = s_out[warp][i][lane];
        mn = __vminu4(mn, o | ~m);
        mx = __vmaxu4(mx, o & m);
      }
      mn = __vminu4(mn, mn >> 16);
      mn = __vminu4(mn, mn >> 8) & 0xffu;
      mx = __vmaxu4(mx, mx >> 16);
      mx = __vmaxu4(mx, mx >> 8) & 0xffu;
      mn = __reduce_min_sync(0xffffffffu, mn);
      mx = __reduce_max_sync(0xffffffffu, mx);
      if (lane == 0) {
        atomicMin(&A.acc[2 * f], mn);
        atomicMax(&A.acc[2 * f + 1], mx);
      }
    }
    if (lane == 0) __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(A.ticket, 1u) == gridDim.x * gridDim.y - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  /* four fields per thread and pass, their accumulators loaded together */
  for (int f0 = threadIdx.x; f0 < A.nfields; f0 += 4 * blockDim.x) {
    uint2 v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int f = f0 + u * (int)blockDim.x;
      if (f < A.nfields) v[u] = __ldcg((const uint2*)&A.acc[2 * f]);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int f = f0 + u * (int)blockDim.x;
      if (f >= A.nfields) break;
      const unsigned mn = v[u].x, mx = v[u].y;
      A.out[2 * f] = (uint8_t)mn;
      A.out[2 * f + 1] = (uint8_t)mx;
      if (f < A.nc && A.skip) {
        const double con = (double)((int)mx - (int)mn) / ((double)((int)mx + (int)mn) + 0.1);
        A.skip[f] = !(con >= A.thr && con > 0.0);
      }
      *(uint2*)&A.acc[2 * f] = make_uint2(0xffffffffu, 0u);
    }
  }
  if (threadIdx.x == 0) *A.ticket = 0u;
}

#endif
