/*
 * vsb_pnet.cu -- the learned search proposal of the detect pass on sm_100a.
 *
 * The reference searches every field over its whole candidate lattice
 * (src/motiondetect.c:439-586).  Here a small network looks at the field's
 * neighbourhood in both frames and predicts where the minimum lies; the
 * narrowed search evaluates only the lattice points around the prediction,
 * then runs the reference's refinement.  The exact full search stays the
 * fallback: it runs for every item whose proposal is not trusted (low
 * confidence, a winner on the window's outer ring, or a refined SAD above a
 * bound), so an accepted proposal only ever replaces a full search whose
 * minimum it has found.
 *
 * Network (the oracle restates it in float64): input 2 x 32 x 32 (2x2
 * averages of 64 x 64 windows of the blurred current and previous planes),
 * conv 3x3 2->32 stride 1, three conv 3x3 32->32 stride 2, each with ReLU,
 * then a 512 -> 3 linear head (dx, dy, confidence logit).  Weights and stored
 * activations are bf16, accumulation fp32.
 *
 * Kernels:
 *   k_pn_infer     the whole network per item, one CTA per item at a time,
 *                  every layer an implicit GEMM on the tensor cores
 *                  (mma m16n8k16 bf16 -> f32) from swizzled shared memory;
 *                  the crop is taken straight from the blurred planes
 *   k_pn_fwd_*     per-layer training forward (fp32 FMA), keeps activations
 *   k_pn_bwd_*     per-layer backward: input gradients and weight gradients
 *                  (fp32, weight gradients folded over the batch by atomics)
 *   k_pn_narrow    the narrowed search + refinement + fallback decision
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vsb_device.h"
#include "vsb_pnet.h"
#include "vsb_plan.h"
#include "vsb_search.cuh"

typedef __nv_bfloat16 bf16;

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

static __global__ void k_pn_crops(const uint8_t* __restrict__ curr, const uint8_t* __restrict__ prev,
                                  int pitch, int W, int H, const vsbd_item* __restrict__ items,
                                  int n, bf16* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n * 2048) return;
  const int s = (int)(i >> 11), e = (int)(i & 2047);
  const int r = e >> 6, c = (e >> 1) & 31, ch = e & 1; /* HWC order */
  out[i] = crop_value(curr, prev, pitch, W, H, items[s], ch, r, c);
}

/* ------------------------------------------------------------------------ */
/* training forward (fp32 FMA, activations stored bf16)                      */
/* ------------------------------------------------------------------------ */

/* one thread per output pixel, all 32 output channels; weights in shared
   memory as [tap][ci][co] floats (broadcast reads) */
template <int CIN, int STRIDE, int HIN, bool L1>
static __global__ void __launch_bounds__(128) k_pn_fwd_conv(const bf16* __restrict__ x,
                                                            const bf16* __restrict__ w,
                                                            const float* __restrict__ bias,
                                                            bf16* __restrict__ y, int n) {
  constexpr int HO = HIN / STRIDE;
  __shared__ __align__(16) float ws[9 * CIN * 32];
  __shared__ float bs[32];
  for (int i = threadIdx.x; i < 9 * CIN * 32; i += blockDim.x) {
    const int tap = i / (CIN * 32), r = i - tap * CIN * 32, ci = r >> 5, co = r & 31;
    ws[i] = L1 ? bf(w[co * 32 + tap * 2 + ci]) : bf(w[(tap * 32 + co) * CIN + ci]);
  }
  if (threadIdx.x < 32) bs[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n * HO * HO) return;
  const int s = (int)(idx / (HO * HO)), p = (int)(idx - (long)s * HO * HO);
  const int oy = p / HO, ox = p - oy * HO;
  float acc[32];
#pragma unroll
  for (int co = 0; co < 32; co++) acc[co] = bs[co];
  for (int tap = 0; tap < 9; tap++) {
    const int iy = oy * STRIDE + tap / 3 - 1, ix = ox * STRIDE + tap % 3 - 1;
    if (iy < 0 || iy >= HIN || ix < 0 || ix >= HIN) continue;
    const bf16* xp = x + (((size_t)s * HIN + iy) * HIN + ix) * CIN;
    float xv[CIN];
    if constexpr (CIN % 8 == 0) {
#pragma unroll
      for (int q = 0; q < CIN / 8; q++) {
        uint4 u = ((const uint4*)xp)[q];
        const bf16* h = (const bf16*)&u;
#pragma unroll
        for (int k = 0; k < 8; k++) xv[q * 8 + k] = bf(h[k]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < CIN; k++) xv[k] = bf(xp[k]);
    }
#pragma unroll
    for (int ci = 0; ci < CIN; ci++) {
      const float4* wr = (const float4*)(ws + (tap * CIN + ci) * 32);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float4 wv = wr[q];
        acc[4 * q + 0] = fmaf(xv[ci], wv.x, acc[4 * q + 0]);
        acc[4 * q + 1] = fmaf(xv[ci], wv.y, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(xv[ci], wv.z, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(xv[ci], wv.w, acc[4 * q + 3]);
      }
    }
  }
  __nv_bfloat162* yp = (__nv_bfloat162*)(y + (size_t)idx * 32);
#pragma unroll
  for (int co = 0; co < 32; co += 2)
    yp[co >> 1] = __floats2bfloat162_rn(fmaxf(acc[co], 0.f), fmaxf(acc[co + 1], 0.f));
}

/* linear head: one warp per item */
static __global__ void k_pn_fwd_fc(const bf16* __restrict__ a4, const bf16* __restrict__ wfc,
                                   const float* __restrict__ bfc, float* __restrict__ out, int n) {
  const int wid = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (wid >= n) return;
  const bf16* a = a4 + (size_t)wid * 512;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
  for (int k = lane; k < 512; k += 32) {
    const float v = bf(a[k]);
    s0 = fmaf(v, bf(wfc[k]), s0);
    s1 = fmaf(v, bf(wfc[512 + k]), s1);
    s2 = fmaf(v, bf(wfc[1024 + k]), s2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    out[wid * 3 + 0] = s0 + bfc[0];
    out[wid * 3 + 1] = s1 + bfc[1];
    out[wid * 3 + 2] = s2 + bfc[2];
  }
}

/* ------------------------------------------------------------------------ */
/* backward                                                                  */
/* ------------------------------------------------------------------------ */

/* head: input gradient d4[s][k] = sum_o dout[s][o] * Wfc[o][k] */
static __global__ void k_pn_bwd_fc_data(const float* __restrict__ dout, const bf16* __restrict__ wfc,
                                        float* __restrict__ d4, int n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n * 512) return;
  const int s = (int)(i >> 9), k = (int)(i & 511);
  d4[i] = dout[s * 3] * bf(wfc[k]) + dout[s * 3 + 1] * bf(wfc[512 + k]) +
          dout[s * 3 + 2] * bf(wfc[1024 + k]);
}

/* head: weight and bias gradients, items split over blockIdx.y (atomics) */
static __global__ void k_pn_bwd_fc_weight(const float* __restrict__ dout, const bf16* __restrict__ a4,
                                          float* __restrict__ dw, float* __restrict__ db, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x; /* 0..1535 weights, 1536..1538 biases */
  if (j >= 1539) return;
  const int chunk = (n + gridDim.y - 1) / gridDim.y;
  const int s0 = blockIdx.y * chunk, s1 = min(n, s0 + chunk);
  float acc = 0.f;
  if (j < 1536) {
    const int o = j >> 9, k = j & 511;
    for (int s = s0; s < s1; s++) acc = fmaf(dout[s * 3 + o], bf(a4[(size_t)s * 512 + k]), acc);
    atomicAdd(dw + j, acc);
  } else {
    const int o = j - 1536;
    for (int s = s0; s < s1; s++) acc += dout[s * 3 + o];
    atomicAdd(db + o, acc);
  }
}

/* input gradient of a 32 -> 32 conv: one thread per input pixel, all 32
   input channels; g = dy masked by the stored ReLU output */
template <int STRIDE, int HIN>
static __global__ void __launch_bounds__(128) k_pn_bwd_data(const float* __restrict__ dy,
                                                            const bf16* __restrict__ y,
                                                            const bf16* __restrict__ w,
                                                            float* __restrict__ dx, int n) {
  constexpr int HO = HIN / STRIDE;
  __shared__ __align__(16) float ws[9 * 32 * 32]; /* [tap][co][ci] */
  for (int i = threadIdx.x; i < 9 * 32 * 32; i += blockDim.x) ws[i] = bf(w[i]);
  __syncthreads();
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n * HIN * HIN) return;
  const int s = (int)(idx / (HIN * HIN)), p = (int)(idx - (long)s * HIN * HIN);
  const int iy = p / HIN, ix = p - iy * HIN;
  float acc[32];
#pragma unroll
  for (int k = 0; k < 32; k++) acc[k] = 0.f;
  for (int tap = 0; tap < 9; tap++) {
    const int ty = iy + 1 - tap / 3, tx = ix + 1 - tap % 3;
    if (ty < 0 || tx < 0 || ty % STRIDE || tx % STRIDE) continue;
    const int oy = ty / STRIDE, ox = tx / STRIDE;
    if (oy >= HO || ox >= HO) continue;
    const size_t o = (((size_t)s * HO + oy) * HO + ox) * 32;
    for (int co = 0; co < 32; co++) {
      const float g = bf(y[o + co]) > 0.f ? dy[o + co] : 0.f;
      if (g == 0.f) continue;
      const float4* wr = (const float4*)(ws + (tap * 32 + co) * 32);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float4 wv = wr[q];
        acc[4 * q + 0] = fmaf(g, wv.x, acc[4 * q + 0]);
        acc[4 * q + 1] = fmaf(g, wv.y, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(g, wv.z, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(g, wv.w, acc[4 * q + 3]);
      }
    }
  }
  float4* dp = (float4*)(dx + (size_t)idx * 32);
#pragma unroll
  for (int q = 0; q < 8; q++) dp[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
}

/* weight and bias gradients of a conv layer: CTAs stride over chunks of 64
   output positions, stage the masked output gradient and the im2col rows
   in shared memory, and accumulate every weight of the layer in registers
   (thread t owns weights t, t + 256, ...); one atomicAdd per weight per CTA */
#define PN_PC 64
template <int CIN, int STRIDE, int HIN, bool L1>
static __global__ void __launch_bounds__(256) k_pn_bwd_weight(const float* __restrict__ dy,
                                                              const bf16* __restrict__ y,
                                                              const bf16* __restrict__ x,
                                                              float* __restrict__ dw,
                                                              float* __restrict__ db, int n) {
  constexpr int HO = HIN / STRIDE, KC = 9 * CIN, NWT = KC * 32, PER = (NWT + 255) / 256;
  extern __shared__ __align__(16) float smf[];
  float* gs = smf;              /* [PN_PC][32] */
  float* xs = smf + PN_PC * 32; /* [PN_PC][KC] */
  float acc[PER];
#pragma unroll
  for (int j = 0; j < PER; j++) acc[j] = 0.f;
  float bacc = 0.f;
  const long P = (long)n * HO * HO;
  for (long c0 = (long)blockIdx.x * PN_PC; c0 < P; c0 += (long)gridDim.x * PN_PC) {
    __syncthreads();
    for (int i = threadIdx.x; i < PN_PC * 32; i += blockDim.x) {
      const long p = c0 + (i >> 5);
      float v = 0.f;
      if (p < P) {
        v = dy[p * 32 + (i & 31)];
        if (!(bf(y[p * 32 + (i & 31)]) > 0.f)) v = 0.f;
      }
      gs[i] = v;
    }
    for (int i = threadIdx.x; i < PN_PC * KC; i += blockDim.x) {
      const int pl = i / KC, r = i - pl * KC, tap = r / CIN, ci = r - tap * CIN;
      const long p = c0 + pl;
      float v = 0.f;
      if (p < P) {
        const int s = (int)(p / (HO * HO)), q = (int)(p - (long)s * HO * HO);
        const int oy = q / HO, ox = q - oy * HO;
        const int iy = oy * STRIDE + tap / 3 - 1, ix = ox * STRIDE + tap % 3 - 1;
        if (iy >= 0 && iy < HIN && ix >= 0 && ix < HIN)
          v = bf(x[(((size_t)s * HIN + iy) * HIN + ix) * CIN + ci]);
      }
      xs[i] = v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const int wi = threadIdx.x + 256 * j;
      if (wi < NWT) {
        const int tap = wi / (32 * CIN), r = wi - tap * 32 * CIN, co = r / CIN, ci = r - co * CIN;
        const float* gp = gs + co;
        const float* xp = xs + tap * CIN + ci;
        float a = 0.f;
#pragma unroll 8
        for (int pl = 0; pl < PN_PC; pl++) a = fmaf(gp[pl * 32], xp[pl * KC], a);
        acc[j] += a;
      }
    }
    if (threadIdx.x < 32)
      for (int pl = 0; pl < PN_PC; pl++) bacc += gs[pl * 32 + threadIdx.x];
  }
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const int wi = threadIdx.x + 256 * j;
    if (wi < NWT) {
      const int tap = wi / (32 * CIN), r = wi - tap * 32 * CIN, co = r / CIN, ci = r - co * CIN;
      atomicAdd(dw + (L1 ? co * 32 + tap * 2 + ci : wi), acc[j]);
    }
  }
  if (threadIdx.x < 32) atomicAdd(db + threadIdx.x, bacc);
}

/* ------------------------------------------------------------------------ */
/* fused inference on the tensor cores                                       */
/* ------------------------------------------------------------------------ */

/* shared memory map of k_pn_infer (bytes); 32-channel rows are 64 bytes
   with their four 16-byte chunks XOR-swizzled by bits 1-2 of the row index,
   so the 8 rows an ldmatrix phase reads fall in distinct bank groups */
#define PI_SM_W1 0                       /* [32 co][32 k] */
#define PI_SM_W2 (PI_SM_W1 + 2048)       /* [9*32 (tap,co)][32 ci] */
#define PI_SM_W3 (PI_SM_W2 + 18432)
#define PI_SM_W4 (PI_SM_W3 + 18432)
#define PI_SM_FC (PI_SM_W4 + 18432)      /* [3][512] plain */
#define PI_SM_B (PI_SM_FC + 3072)        /* f32 [131] */
#define PI_SM_IN (PI_SM_B + 528)         /* [34][34][2] zero-bordered input */
#define PI_SM_A1 (PI_SM_IN + 4624)       /* im2col of 512 conv1 pixels [512][32] */
#define PI_SM_ACT1 (PI_SM_A1 + 32768)    /* [34*34][32] */
#define PI_SM_ACT2 (PI_SM_ACT1 + 73984)  /* [18*18][32] */
#define PI_SM_ACT3 (PI_SM_ACT2 + 20736)  /* [10*10][32] */
#define PI_SM_ACT4 (PI_SM_ACT3 + 6400)   /* f32 [16][32] */
#define PI_SMEM (PI_SM_ACT4 + 2048)
#define PI_THREADS 512

__device__ __forceinline__ int swz(int row, int ch) {
  return (row << 5) | ((((ch >> 3) ^ (row >> 1)) & 3) << 3) | (ch & 7);
}

__device__ __forceinline__ void ldsm4(uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3,
                                      const bf16* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_relu(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(a, 0.f), fmaxf(b, 0.f));
  return *(uint32_t*)&h;
}

/* One m-tile (16 output pixels) of a stride-2 32->32 conv against n-tile
   pairs [np0, np0+NP): A rows from the swizzled input activation (padded
   width WP); the output pixel of the lane's A row is (oy, ox). */
template <int NP>
__device__ __forceinline__ void conv_s2_mtile(const bf16* act, int WP, int oy, int ox,
                                              const bf16* wsm, int np0, float (&acc)[2 * NP][4],
                                              int lane) {
  const int hi = lane >> 4, kq = (lane >> 3) & 1, nr = lane & 7;
#pragma unroll
  for (int t = 0; t < 2 * NP; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
#pragma unroll 1
  for (int tap = 0; tap < 9; tap++) {
    const int ky = tap / 3, kx = tap - ky * 3;
    const int arow = (2 * oy + ky) * WP + 2 * ox + kx;
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
      uint32_t a0, a1, a2, a3;
      ldsm4(a0, a1, a2, a3, act + swz(arow, ks * 16 + hi * 8));
#pragma unroll
      for (int p = 0; p < NP; p++) {
        const int wrow = tap * 32 + (2 * (np0 + p) + hi) * 8 + nr;
        uint32_t b0, b1, b2, b3;
        ldsm4(b0, b1, b2, b3, wsm + swz(wrow, ks * 16 + kq * 8));
        mma_bf16(acc[2 * p], a0, a1, a2, a3, b0, b1);
        mma_bf16(acc[2 * p + 1], a0, a1, a2, a3, b2, b3);
      }
    }
  }
}

/* grid: up to one CTA per SM, CTAs stride over the items; block PI_THREADS
   (16 warps) */
static __global__ void __launch_bounds__(PI_THREADS, 1) k_pn_infer(const void* __restrict__ params,
                                                            const uint8_t* __restrict__ curr,
                                                            const uint8_t* __restrict__ prev,
                                                            int pitch, int W, int H,
                                                            const vsbd_item* __restrict__ items,
                                                            const uint32_t* __restrict__ prepared,
                                                            int n, float* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t sm[];
  bf16* sW1 = (bf16*)(sm + PI_SM_W1);
  bf16* sW2 = (bf16*)(sm + PI_SM_W2);
  bf16* sW3 = (bf16*)(sm + PI_SM_W3);
  bf16* sW4 = (bf16*)(sm + PI_SM_W4);
  bf16* sFC = (bf16*)(sm + PI_SM_FC);
  float* sB = (float*)(sm + PI_SM_B);
  uint32_t* sIn = (uint32_t*)(sm + PI_SM_IN); /* one word = the 2 channels of a pixel */
  bf16* sA1 = (bf16*)(sm + PI_SM_A1);
  bf16* sAct1 = (bf16*)(sm + PI_SM_ACT1);
  bf16* sAct2 = (bf16*)(sm + PI_SM_ACT2);
  bf16* sAct3 = (bf16*)(sm + PI_SM_ACT3);
  float* sAct4 = (float*)(sm + PI_SM_ACT4);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const PNPtr P = pn_ptr(params);

  /* weights, swizzled 16-byte chunks; zero every bordered buffer once (the
     borders are never written again) */
  for (int i = tid; i < 32 * 4; i += PI_THREADS) {
    const int r = i >> 2, j = i & 3;
    ((uint4*)sW1)[r * 4 + (j ^ ((r >> 1) & 3))] = ((const uint4*)P.w1)[i];
  }
  for (int i = tid; i < 288 * 4; i += PI_THREADS) {
    const int r = i >> 2, j = i & 3, d = r * 4 + (j ^ ((r >> 1) & 3));
    ((uint4*)sW2)[d] = ((const uint4*)P.w2)[i];
    ((uint4*)sW3)[d] = ((const uint4*)P.w3)[i];
    ((uint4*)sW4)[d] = ((const uint4*)P.w4)[i];
  }
  for (int i = tid; i < PN_NFC / 8; i += PI_THREADS) ((uint4*)sFC)[i] = ((const uint4*)P.fc)[i];
  for (int i = tid; i < PN_NF32; i += PI_THREADS) sB[i] = P.b1[i];
  for (int i = tid; i < (PI_SM_ACT4 - PI_SM_IN) / 16; i += PI_THREADS)
    ((uint4*)(sm + PI_SM_IN))[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();

  const int hi = lane >> 4, kq = (lane >> 3) & 1, nr = lane & 7;
  const int arl = (lane & 7) + kq * 8; /* the lane's A row within an m-tile */
  const int g = lane >> 2, t2 = 2 * (lane & 3); /* accumulator row / column pair */

  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    /* 1. input planes */
    if (prepared) {
      const uint32_t* src = prepared + (size_t)s * 1024;
      for (int i = tid; i < 1024; i += PI_THREADS) sIn[((i >> 5) + 1) * 34 + (i & 31) + 1] = src[i];
    } else {
      const vsbd_item it = items[s];
      bf16* sInh = (bf16*)sIn;
      for (int i = tid; i < 2048; i += PI_THREADS) {
        const int r = i >> 6, c = (i >> 1) & 31, ch = i & 1;
        sInh[((r + 1) * 34 + c + 1) * 2 + ch] = crop_value(curr, prev, pitch, W, H, it, ch, r, c);
      }
    }
    __syncthreads();

    /* 2. conv1 (stride 1) as an im2col GEMM, 2 chunks of 16 output rows */
    for (int ck = 0; ck < 2; ck++) {
      {
        const int y = ck * 16 + (tid >> 5), x = tid & 31;
        uint32_t wv[16];
#pragma unroll
        for (int tap = 0; tap < 9; tap++) wv[tap] = sIn[(y + tap / 3) * 34 + x + tap % 3];
#pragma unroll
        for (int j = 9; j < 16; j++) wv[j] = 0u;
        uint4* dst = (uint4*)(sA1 + tid * 32);
#pragma unroll
        for (int q = 0; q < 4; q++)
          dst[q ^ ((tid >> 1) & 3)] = make_uint4(wv[4 * q], wv[4 * q + 1], wv[4 * q + 2], wv[4 * q + 3]);
      }
      __syncthreads();
#pragma unroll 1
      for (int mi = 0; mi < 2; mi++) {
        const int mt = warp * 2 + mi;
        float acc[4][4];
#pragma unroll
        for (int t = 0; t < 4; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
          uint32_t a0, a1, a2, a3;
          ldsm4(a0, a1, a2, a3, sA1 + swz(mt * 16 + arl, ks * 16 + hi * 8));
#pragma unroll
          for (int p = 0; p < 2; p++) {
            uint32_t b0, b1, b2, b3;
            ldsm4(b0, b1, b2, b3, sW1 + swz((2 * p + hi) * 8 + nr, ks * 16 + kq * 8));
            mma_bf16(acc[2 * p], a0, a1, a2, a3, b0, b1);
            mma_bf16(acc[2 * p + 1], a0, a1, a2, a3, b2, b3);
          }
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int pl = mt * 16 + g + 8 * h; /* chunk-local pixel */
          const int row = (ck * 16 + (pl >> 5) + 1) * 34 + (pl & 31) + 1;
#pragma unroll
          for (int t = 0; t < 4; t++) {
            const int ch = t * 8 + t2;
            *(uint32_t*)(sAct1 + swz(row, ch)) =
                pack_relu(acc[t][2 * h] + sB[ch], acc[t][2 * h + 1] + sB[ch + 1]);
          }
        }
      }
      __syncthreads();
    }

    /* 3. conv2: 16x16 outputs, m-tile = output row, one per warp */
    {
      const int oy = warp;
      float acc[4][4];
      conv_s2_mtile<2>(sAct1, 34, oy, arl, sW2, 0, acc, lane);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int row = (oy + 1) * 18 + g + 8 * h + 1;
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int ch = t * 8 + t2;
          *(uint32_t*)(sAct2 + swz(row, ch)) =
              pack_relu(acc[t][2 * h] + sB[32 + ch], acc[t][2 * h + 1] + sB[32 + ch + 1]);
        }
      }
    }
    __syncthreads();

    /* 4. conv3: 8x8 outputs = 4 m-tiles; warp (< 8): m-tile w/2, n-tiles 2(w&1).. */
    if (warp < 8) {
      const int mt = warp >> 1, np0 = warp & 1;
      const int px = mt * 16 + arl;
      float acc[2][4];
      conv_s2_mtile<1>(sAct2, 18, px >> 3, px & 7, sW3, np0, acc, lane);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int po = mt * 16 + g + 8 * h;
        const int row = ((po >> 3) + 1) * 10 + (po & 7) + 1;
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const int ch = (2 * np0 + t) * 8 + t2;
          *(uint32_t*)(sAct3 + swz(row, ch)) =
              pack_relu(acc[t][2 * h] + sB[64 + ch], acc[t][2 * h + 1] + sB[64 + ch + 1]);
        }
      }
    }
    __syncthreads();

    /* 5. conv4: 4x4 outputs = 1 m-tile; warps 0 and 1 take two n-tiles each */
    if (warp < 2) {
      float acc[2][4];
      conv_s2_mtile<1>(sAct3, 10, arl >> 2, arl & 3, sW4, warp, acc, lane);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int po = g + 8 * h;
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const int ch = (2 * warp + t) * 8 + t2;
#pragma unroll
          for (int e = 0; e < 2; e++)
            sAct4[po * 32 + ch + e] = __bfloat162float(
                __float2bfloat16_rn(fmaxf(acc[t][2 * h + e] + sB[96 + ch + e], 0.f)));
        }
      }
    }
    __syncthreads();

    /* 6. head */
    if (warp < 3) {
      float acc = 0.f;
      for (int k = lane; k < 512; k += 32) acc = fmaf(sAct4[k], bf(sFC[warp * 512 + k]), acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) out[(size_t)s * 3 + warp] = acc + sB[128 + warp];
    }
    __syncthreads();
  }
}

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
  int rowW, fieldB, WP, WH, R;
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
  const int q = g.maxq > PN_NARROW_QMAX ? g.maxq : PN_NARROW_QMAX;
  L.total = L.off_q + (size_t)q * 4 + 16;
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

/* The SADs of a grid of candidates: columns i < ncol at dx0 + i*hx, rows
   k < nrow at dy0 + k*hy (window coordinates), into sums[i*nrow + k].  The
   warps take (column, row chunk of <= 8, field-row strip) tasks. */
__device__ __forceinline__ void sad_grid(const uint32_t* C, int rowW, int S, const uint8_t* win,
                                         int WP, int e, int bpp, int dx0, int hx, int ncol,
                                         int dy0, int hy, int nrow, unsigned* sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int q = threadIdx.x; q < ncol * nrow; q += blockDim.x) sums[q] = 0;
  __syncthreads();
  const int nch = (nrow + 7) >> 3;
  const int units = ncol * nch;
  int strips = nwarps / units;
  if (strips < 1) strips = 1;
  const int rs = (S + strips - 1) / strips;
  for (int t = warp; t < units * strips; t += nwarps) {
    const int u = t % units, sidx = t / units;
    const int col = u / nch, ch = u - col * nch;
    const int k0 = ch * 8, nk = min(8, nrow - k0);
    const int r0 = sidx * rs, r1 = min(S, r0 + rs);
    if (r0 < r1)
      sad_column_n(nk, C, rowW, win, WP, e, bpp, dx0 + col * hx, dy0 + k0 * hy, hy, r0, r1, lane,
                   sums + col * nrow + k0);
  }
  __syncthreads();
}

/* One CTA per item.  The lattice points that bracket the prediction +-
   radius, plus one ring around them, get their full SAD; the lowest (SAD,
   rank) is refined exactly as the full search refines its winner
   (src/motiondetect.c:545-567 of the reference: i outer, j inner, centre
   skipped, strict <) and range-tested (:573-574).  The window of the
   previous frame all of this can touch (the candidates plus the refinement
   reach) is staged once in shared memory with 16-byte loads.  The item
   falls back to the full search (appended to fb_list) when the confidence
   is below the threshold, the winner lies on the ring (the minimum may lie
   further out), or the refined SAD exceeds the bound. */
static __global__ void __launch_bounds__(512) k_pn_narrow(const uint8_t* __restrict__ curr,
                                                          const uint8_t* __restrict__ prev,
                                                          int pitch, DGeom g,
                                                          const vsbd_item* __restrict__ items,
                                                          const float* __restrict__ pout,
                                                          const short2* __restrict__ prior,
                                                          PNSearch ps,
                                                          const uint8_t* __restrict__ skip,
                                                          vsbd_result* __restrict__ res,
                                                          uint8_t* __restrict__ fb,
                                                          int* __restrict__ fb_count,
                                                          int* __restrict__ fb_list) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ int s_tx, s_ty;
  __shared__ unsigned s_min;
  const int item = blockIdx.x;
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
  if (unused || alo > ahi || blo > bhi || wa > span || wb > span) {
    if (threadIdx.x == 0) {
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
    for (int i = threadIdx.x; i < g.S * L.rowW; i += blockDim.x) {
      const int r = i / L.rowW, w = i - r * L.rowW;
      const uint32_t* sw = (const uint32_t*)(curr + (size_t)(cy0 + r) * pitch) + (cx0 >> 2) + w;
      C[i] = __funnelshift_r(sw[0], sw[1], sh);
    }
    const int wwb = g.S * g.bpp + ((wa - 1) * g.step + 2 * L.R) * g.bpp;
    const int wh = g.S + (wb - 1) * g.step + 2 * L.R;
    const int nv = (e + wwb + 15) >> 4;
    for (int i = threadIdx.x; i < wh * nv; i += blockDim.x) {
      const int r = i / nv, v = i - r * nv;
      *(uint4*)(win + r * L.WP + (v << 4)) =
          *(const uint4*)(prev + (size_t)(wy + r) * pitch + wxa + (v << 4));
    }
  }
  __syncthreads();
  /* lattice window: column a - wal, row b - wbl at sums[(a-wal)*wb + (b-wbl)];
     the lowest (SAD, visiting rank) by a block-wide reduction */
  sad_grid(C, L.rowW, g.S, win, L.WP, e, g.bpp, L.R, g.step, wa, L.R, g.step, wb, qsad);
  {
    __shared__ unsigned long long red[16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long best = ~0ull;
    for (int q = threadIdx.x; q < wa * wb; q += blockDim.x) {
      const int a = wal + q / wb, b = wbl + q % wb;
      const unsigned long long key =
          ((unsigned long long)qsad[q] << 32) | (unsigned)g.order[b * g.na + a];
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
    sad_grid(C, L.rowW, g.S, win, L.WP, e, g.bpp, cx - r - dx0, h, side, cy - r - dy0, h, side,
             qsad);
    if (threadIdx.x == 0) {
      unsigned m = s_min;
      int tx = cx, ty = cy;
      /* the reference's order: i (x) outer, j (y) inner */
      for (int ii = 0; ii < side; ii++)
        for (int jj = 0; jj < side; jj++) {
          const int i = cx - r + ii * h, j = cy - r + jj * h;
          if (i == cx && j == cy) continue;
          if (qsad[ii * side + jj] < m) {
            m = qsad[ii * side + jj];
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
  if (threadIdx.x == 0) {
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
}

/* Global motion prior of a frame's coarse items from the first network
   pass.  Translation: the per-axis median of the confident predictions (the
   non-skipped items with a finite prediction and a logit >= conf_min; all
   non-skipped items if fewer than three are confident).  Rotation: the small
   angle about the frame centre that best fits, in least squares, the
   predictions within 8 px of that translation.  Every item gets the model's
   displacement at its centre, rounded: the search offset of its second
   network pass (items2) and the base of its proposal (prior).  One CTA. */
#define PN_PRIOR_MAX 1024
static __global__ void __launch_bounds__(256) k_pn_prior(const vsbd_item* __restrict__ items,
                                                         const float* __restrict__ pout, int n,
                                                         float scale, float conf_min,
                                                         const uint8_t* __restrict__ skip,
                                                         float cx, float cy,
                                                         vsbd_item* __restrict__ items2,
                                                         short2* __restrict__ prior) {
  __shared__ float vx[PN_PRIOR_MAX], vy[PN_PRIOR_MAX], jx[PN_PRIOR_MAX], jy[PN_PRIOR_MAX];
  __shared__ int m;
  __shared__ float med[2];
  __shared__ float sums[2][8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int pass = 0; pass < 2; pass++) {
    if (tid == 0) m = 0;
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
      if (skip && skip[i]) continue;
      const float px = pout[3 * i] * scale, py = pout[3 * i + 1] * scale, c = pout[3 * i + 2];
      if (!isfinite(px) || !isfinite(py) || fabsf(px) > 4096.f || fabsf(py) > 4096.f) continue;
      if (pass == 0 && !(c >= conf_min)) continue;
      const int k = atomicAdd(&m, 1);
      if (k < PN_PRIOR_MAX) {
        vx[k] = px;
        vy[k] = py;
        jx[k] = -((float)items[i].y - cy); /* d(displacement)/d(angle) at the centre */
        jy[k] = (float)items[i].x - cx;
      }
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
  /* rotation about the centre from the inliers of the translation */
  float num = 0.f, den = 0.f;
  for (int k = tid; k < cnt; k += blockDim.x) {
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
  if (lane == 0) {
    sums[0][warp] = num;
    sums[1][warp] = den;
  }
  __syncthreads();
  float th = 0.f;
  {
    float a = 0.f, b = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
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

static __global__ void k_pn_labels(const vsbd_result* __restrict__ res,
                                   const uint8_t* __restrict__ skip, int n, int kind,
                                   PNLabel* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vsbd_result r = res[i];
  PNLabel l;
  l.tx = r.tx;
  l.ty = r.ty;
  l.sad = r.sad;
  l.kind = (uint8_t)kind;
  l.ok = (uint8_t)(r.ok != 0);
  l.use = (uint8_t)(skip ? !skip[i] : 1);
  l.pad = 0;
  out[i] = l;
}

/* ------------------------------------------------------------------------ */
/* launchers                                                                 */
/* ------------------------------------------------------------------------ */

static thread_local char g_pn_err[256];
static int pn_fail(const char* what, cudaError_t e) {
  snprintf(g_pn_err, sizeof(g_pn_err), "%s: %s", what, cudaGetErrorString(e));
  vsbd_set_error(g_pn_err);
  return -1;
}
static int pn_msg(const char* m) {
  vsbd_set_error(m);
  return -1;
}

#define PCK(call)                              \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return pn_fail(#call, e_); \
  } while (0)

/* dynamic shared-memory limit of a kernel on the current device, raised
   only when a launch needs more (slot names the kernel) */
static cudaError_t pn_ensure_smem(const void* fn, int slot, size_t smem) {
  static size_t done[16][8];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 16 && done[dev][slot] >= smem) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && dev >= 0 && dev < 16) done[dev][slot] = smem;
  return e;
}

static int sm_count_cached(void) {
  static int n = 0;
  if (!n) n = vsbp_sm_count();
  return n;
}

int vsbpn_infer(const void* d_params, const uint8_t* curr, const uint8_t* prev, int pitch, int W,
                int H, const vsbd_item* items, const void* prepared, int n, float* out,
                cudaStream_t st) {
  if (n <= 0) return 0;
  PCK(pn_ensure_smem((const void*)k_pn_infer, 0, PI_SMEM));
  const int grid = min(n, sm_count_cached());
  k_pn_infer<<<grid, PI_THREADS, PI_SMEM, st>>>(d_params, curr, prev, pitch, W, H, items,
                                         (const uint32_t*)prepared, n, out);
  PCK(cudaGetLastError());
  return 1;
}

int vsbpn_narrow(const DGeom& g, const uint8_t* curr, const uint8_t* prev, int pitch,
                 const vsbd_item* items, int n, const float* pout, const short2* prior,
                 const PNSearch& ps, const uint8_t* skip, vsbd_result* res, uint8_t* fb,
                 int* fb_count, int* fb_list, cudaStream_t st) {
  if (n <= 0) return 0;
  if (g.has_origin) return pn_msg("the narrowed search serves planar field sets only");
  if (narrow_span(ps.radius, g.step) * narrow_span(ps.radius, g.step) > PN_NARROW_QMAX)
    return pn_msg("proposal radius too large for the narrowed search");
  const size_t smem = narrow_layout(g, ps.radius).total;
  if (smem > 48 * 1024) PCK(pn_ensure_smem((const void*)k_pn_narrow, 1, smem));
  k_pn_narrow<<<n, 512, smem, st>>>(curr, prev, pitch, g, items, pout, prior, ps, skip, res, fb,
                                    fb_count, fb_list);
  PCK(cudaGetLastError());
  return 1;
}

int vsbpn_crops(const uint8_t* curr, const uint8_t* prev, int pitch, int W, int H,
                const vsbd_item* items, int n, void* inputs, cudaStream_t st) {
  if (n <= 0) return 0;
  const long tot = (long)n * 2048;
  k_pn_crops<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(curr, prev, pitch, W, H, items, n,
                                                           (bf16*)inputs);
  PCK(cudaGetLastError());
  return 1;
}

int vsbpn_labels(const vsbd_result* res, const uint8_t* skip, int n, int kind, PNLabel* out,
                 cudaStream_t st) {
  if (n <= 0) return 0;
  k_pn_labels<<<(n + 127) / 128, 128, 0, st>>>(res, skip, n, kind, out);
  PCK(cudaGetLastError());
  return 1;
}

int vsbpn_prior(const vsbd_item* items, const float* pout, int n, float scale, float conf_min,
                const uint8_t* skip, int W, int H, vsbd_item* items2, short2* prior,
                cudaStream_t st) {
  if (n <= 0) return 0;
  k_pn_prior<<<1, 256, 0, st>>>(items, pout, n, scale, conf_min, skip, (float)(W / 2),
                                (float)(H / 2), items2, prior);
  PCK(cudaGetLastError());
  return 1;
}

/* activation blocks of a batch of n items inside the caller's buffer */
struct PNActs {
  bf16 *a1, *a2, *a3, *a4;
};
static PNActs pn_acts(void* base, int n) {
  PNActs a;
  a.a1 = (bf16*)base;
  a.a2 = a.a1 + (size_t)n * 32768;
  a.a3 = a.a2 + (size_t)n * 8192;
  a.a4 = a.a3 + (size_t)n * 2048;
  return a;
}

template <typename K>
static unsigned blocks_for(long threads, K) {
  return (unsigned)((threads + 127) / 128);
}

extern "C" int vsbd_pnet_forward_train(const void* d_params, const void* d_input, int n,
                                       void* d_acts, float* d_out, void* stream) {
  if (n <= 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  const PNPtr P = pn_ptr(d_params);
  const PNActs A = pn_acts(d_acts, n);
  const bf16* x = (const bf16*)d_input;
  k_pn_fwd_conv<2, 1, 32, true><<<(unsigned)(((long)n * 1024 + 127) / 128), 128, 0, st>>>(
      x, P.w1, P.b1, A.a1, n);
  k_pn_fwd_conv<32, 2, 32, false><<<(unsigned)(((long)n * 256 + 127) / 128), 128, 0, st>>>(
      A.a1, P.w2, P.b2, A.a2, n);
  k_pn_fwd_conv<32, 2, 16, false><<<(unsigned)(((long)n * 64 + 127) / 128), 128, 0, st>>>(
      A.a2, P.w3, P.b3, A.a3, n);
  k_pn_fwd_conv<32, 2, 8, false><<<(unsigned)(((long)n * 16 + 127) / 128), 128, 0, st>>>(
      A.a3, P.w4, P.b4, A.a4, n);
  k_pn_fwd_fc<<<(unsigned)(((long)n * 32 + 127) / 128), 128, 0, st>>>(A.a4, P.fc, P.bfc, d_out, n);
  PCK(cudaGetLastError());
  return 0;
}

template <int CIN, int STRIDE, int HIN, bool L1>
static int launch_bwd_weight(const float* dy, const bf16* y, const bf16* x, float* dw, float* db,
                             int n, cudaStream_t st) {
  const size_t smem = sizeof(float) * PN_PC * (32 + 9 * CIN);
  PCK(pn_ensure_smem((const void*)k_pn_bwd_weight<CIN, STRIDE, HIN, L1>,
                     2 + (CIN == 2 ? 0 : (HIN == 8 ? 1 : (HIN == 16 ? 2 : 3))), smem));
  constexpr int HO = HIN / STRIDE;
  const long chunks = ((long)n * HO * HO + PN_PC - 1) / PN_PC;
  const long cap = 2L * sm_count_cached();
  const unsigned grid = (unsigned)(chunks < cap ? chunks : cap);
  k_pn_bwd_weight<CIN, STRIDE, HIN, L1><<<grid, 256, smem, st>>>(dy, y, x, dw, db, n);
  PCK(cudaGetLastError());
  return 0;
}

extern "C" int vsbd_pnet_backward(const void* d_params, const void* d_input, const void* d_acts,
                                  int n, const float* d_dout, float* d_grad, void* d_work,
                                  void* stream) {
  if (n <= 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  const PNPtr P = pn_ptr(d_params);
  const PNActs A = pn_acts((void*)d_acts, n);
  float* d1 = (float*)d_work;
  float* d2 = d1 + (size_t)n * 32768;
  float* d3 = d2 + (size_t)n * 8192;
  float* d4 = d3 + (size_t)n * 2048;
  float* gW1 = d_grad;
  float* gW2 = gW1 + PN_NW1;
  float* gW3 = gW2 + PN_NW;
  float* gW4 = gW3 + PN_NW;
  float* gFC = gW4 + PN_NW;
  float* gB = d_grad + PN_NB16;
  PCK(cudaMemsetAsync(d_grad, 0, sizeof(float) * (PN_NB16 + PN_NF32), st));
  {
    dim3 grid((1539 + 127) / 128, (unsigned)min(64, (n + 63) / 64));
    k_pn_bwd_fc_weight<<<grid, 128, 0, st>>>(d_dout, A.a4, gFC, gB + 128, n);
  }
  k_pn_bwd_fc_data<<<(unsigned)(((long)n * 512 + 127) / 128), 128, 0, st>>>(d_dout, P.fc, d4, n);
  if (launch_bwd_weight<32, 2, 8, false>(d4, A.a4, A.a3, gW4, gB + 96, n, st)) return -1;
  k_pn_bwd_data<2, 8><<<(unsigned)(((long)n * 64 + 127) / 128), 128, 0, st>>>(d4, A.a4, P.w4, d3, n);
  if (launch_bwd_weight<32, 2, 16, false>(d3, A.a3, A.a2, gW3, gB + 64, n, st)) return -1;
  k_pn_bwd_data<2, 16><<<(unsigned)(((long)n * 256 + 127) / 128), 128, 0, st>>>(d3, A.a3, P.w3, d2, n);
  if (launch_bwd_weight<32, 2, 32, false>(d2, A.a2, A.a1, gW2, gB + 32, n, st)) return -1;
  k_pn_bwd_data<2, 32><<<(unsigned)(((long)n * 1024 + 127) / 128), 128, 0, st>>>(d2, A.a2, P.w2, d1, n);
  if (launch_bwd_weight<2, 1, 32, true>(d1, A.a1, (const bf16*)d_input, gW1, gB, n, st)) return -1;
  PCK(cudaGetLastError());
  return 0;
}

extern "C" int vsbd_pnet_infer(const void* d_params, const void* d_input, int n, float* d_out,
                               void* stream) {
  return vsbpn_infer(d_params, NULL, NULL, 0, 0, 0, NULL, d_input, n, d_out,
                     (cudaStream_t)stream) < 0 ? -1 : 0;
}

extern "C" int vsbd_pnet_infer_items(const void* d_params, const uint8_t* d_curr,
                                     const uint8_t* d_prev, int pitch, int W, int H,
                                     const void* d_items, int n, float* d_out, void* stream) {
  if (!d_curr || !d_prev || W < 1 || H < 1 || pitch < W) return pn_msg("bad plane arguments");
  return vsbpn_infer(d_params, d_curr, d_prev, pitch, W, H, (const vsbd_item*)d_items, NULL, n,
                     d_out, (cudaStream_t)stream) < 0 ? -1 : 0;
}

extern "C" int vsbd_pnet_crops(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int W,
                               int H, const void* d_items, int n, void* d_input, void* stream) {
  if (!d_curr || !d_prev || W < 1 || H < 1 || pitch < W) return pn_msg("bad plane arguments");
  return vsbpn_crops(d_curr, d_prev, pitch, W, H, (const vsbd_item*)d_items, n, d_input,
                     (cudaStream_t)stream) < 0 ? -1 : 0;
}

/* Narrowed search of one field set on host buffers (parity tests): the
   planes are uploaded with 256 bytes of slack, proposals pout[n][3] are raw
   network outputs (scaled by ps.scale).  Writes per item the result and the
   fallback flag (the full search is not run here). */
extern "C" int vsbd_pnet_narrow_host(const uint8_t* curr, const uint8_t* prev, int W, int H,
                                     const vsbd_geom* h, const vsbd_item* items, int n,
                                     const float* pout, float scale, float radius,
                                     float conf_min, unsigned sad_bound, vsbd_result* out,
                                     uint8_t* flags) {
  if (n <= 0) return 0;
  GeomDev gd;
  if (vsbp_geom_upload(h, n, &gd) != 0) return -1;
  const int pitch = (W + 127) & ~127;
  const size_t plane = (size_t)pitch * H + 256;
  uint8_t *dc = NULL, *dp = NULL, *dfb = NULL;
  vsbd_item* di = NULL;
  float* dpo = NULL;
  int* dcount = NULL;
  int* dlist = NULL;
  vsbd_result* dr = NULL;
  int rc = -1;
  cudaError_t e = cudaSuccess;
#define PTRY(call)            \
  do {                        \
    e = (call);               \
    if (e != cudaSuccess) {   \
      pn_fail(#call, e);      \
      goto done;              \
    }                         \
  } while (0)
  PTRY(cudaMalloc(&dc, plane));
  PTRY(cudaMalloc(&dp, plane));
  PTRY(cudaMemset(dc, 0, plane));
  PTRY(cudaMemset(dp, 0, plane));
  PTRY(cudaMemcpy2D(dc, pitch, curr, W, W, H, cudaMemcpyHostToDevice));
  PTRY(cudaMemcpy2D(dp, pitch, prev, W, W, H, cudaMemcpyHostToDevice));
  PTRY(cudaMalloc(&di, sizeof(vsbd_item) * n));
  PTRY(cudaMemcpy(di, items, sizeof(vsbd_item) * n, cudaMemcpyHostToDevice));
  PTRY(cudaMalloc(&dpo, sizeof(float) * 3 * n));
  PTRY(cudaMemcpy(dpo, pout, sizeof(float) * 3 * n, cudaMemcpyHostToDevice));
  PTRY(cudaMalloc(&dcount, sizeof(int)));
  PTRY(cudaMemset(dcount, 0, sizeof(int)));
  PTRY(cudaMalloc(&dlist, sizeof(int) * n));
  PTRY(cudaMalloc(&dr, sizeof(vsbd_result) * n));
  PTRY(cudaMalloc(&dfb, n));
  {
    PNSearch ps;
    ps.scale = scale;
    ps.radius = radius;
    ps.conf_min = conf_min;
    ps.sad_bound = sad_bound;
    if (vsbpn_narrow(gd.g, dc, dp, pitch, di, n, dpo, NULL, ps, NULL, dr, dfb, dcount, dlist, 0) < 0)
      goto done;
  }
  PTRY(cudaDeviceSynchronize());
  PTRY(cudaMemcpy(out, dr, sizeof(vsbd_result) * n, cudaMemcpyDeviceToHost));
  PTRY(cudaMemcpy(flags, dfb, n, cudaMemcpyDeviceToHost));
  rc = 0;
done:
#undef PTRY
  cudaFree(dc);
  cudaFree(dp);
  cudaFree(di);
  cudaFree(dpo);
  cudaFree(dcount);
  cudaFree(dlist);
  cudaFree(dr);
  cudaFree(dfb);
  vsbp_geom_free(&gd);
  return rc;
}
