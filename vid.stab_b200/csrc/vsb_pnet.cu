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
 *                  every convolution an implicit GEMM on the fifth-generation
 *                  tensor cores (tcgen05.mma bf16 -> f32, accumulators in
 *                  tensor memory, vsb_pnet_tc.cuh); the crop is taken
 *                  straight from the blurred planes
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

#include "vsb_pnet_dev.cuh"
#include "vsb_pnet_tc.cuh"

/* grid: up to one CTA per SM, CTAs stride over the items; block PI_THREADS
   (16 warps); every layer on the tensor cores (tcgen05, accumulators in
   tensor memory).  err (may be NULL) is raised when a wait for the tensor
   cores gave up. */
static __global__ void __launch_bounds__(PI_THREADS, 1) k_pn_infer(const void* __restrict__ params,
                                                            const uint8_t* __restrict__ curr,
                                                            const uint8_t* __restrict__ prev,
                                                            int pitch, int W, int H,
                                                            const vsbd_item* __restrict__ items,
                                                            const uint32_t* __restrict__ prepared,
                                                            int n, float* __restrict__ out,
                                                            unsigned* err) {
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot, phase;
  if (threadIdx.x == 0) {
    tc_mbar_init(&mbar);
    phase = 0;
  }
  tc_alloc(&tslot);
  tc_fence_before();
  pn_tc_stage(sm, params); /* ends with a barrier */
  tc_fence_after();
  const uint32_t taddr = tslot;
  pn_tc_items(sm, taddr, tc_saddr(&mbar), &phase, curr, prev, pitch, W, H, items, prepared,
              blockIdx.x, n, gridDim.x, out, err);
  tc_fence_before();
  __syncthreads();
  tc_dealloc(taddr);
}

/* CTAs of 512 threads per item (a cluster of PN_NARROW_CL, each summing a
   strip of the field rows into the first CTA's shared memory) */
#define PN_NARROW_CL 4
static __global__ void __cluster_dims__(PN_NARROW_CL, 1, 1) __launch_bounds__(512)
    k_pn_narrow(const uint8_t* __restrict__ curr,
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
  pn_narrow_item<PN_NARROW_CL>(sm, curr, prev, pitch, g, items, pout, prior, ps, skip, res, fb,
                               fb_count, fb_list, blockIdx.x / PN_NARROW_CL);
}

/* one CTA of 256 threads */
static __global__ void __launch_bounds__(256) k_pn_prior(const vsbd_item* __restrict__ items,
                                                         const float* __restrict__ pout, int n,
                                                         float scale, float conf_min,
                                                         const uint8_t* __restrict__ skip,
                                                         float cx, float cy,
                                                         vsbd_item* __restrict__ items2,
                                                         short2* __restrict__ prior) {
  __shared__ float buf[4 * PN_PRIOR_MAX];
  pn_prior_body(buf, items, pout, n, scale, conf_min, skip, cx, cy, items2, prior);
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
                unsigned* err, cudaStream_t st) {
  if (n <= 0) return 0;
  PCK(pn_ensure_smem((const void*)k_pn_infer, 0, TC_SMEM));
  const int grid = min(n, sm_count_cached());
  k_pn_infer<<<grid, PI_THREADS, TC_SMEM, st>>>(d_params, curr, prev, pitch, W, H, items,
                                         (const uint32_t*)prepared, n, out, err);
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
  k_pn_narrow<<<n * PN_NARROW_CL, 512, smem, st>>>(curr, prev, pitch, g, items, pout, prior, ps,
                                                   skip, res, fb, fb_count, fb_list);
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
  return vsbpn_infer(d_params, NULL, NULL, 0, 0, 0, NULL, d_input, n, d_out, NULL,
                     (cudaStream_t)stream) < 0 ? -1 : 0;
}

extern "C" int vsbd_pnet_infer_items(const void* d_params, const uint8_t* d_curr,
                                     const uint8_t* d_prev, int pitch, int W, int H,
                                     const void* d_items, int n, float* d_out, void* stream) {
  if (!d_curr || !d_prev || W < 1 || H < 1 || pitch < W) return pn_msg("bad plane arguments");
  return vsbpn_infer(d_params, d_curr, d_prev, pitch, W, H, (const vsbd_item*)d_items, NULL, n,
                     d_out, NULL, (cudaStream_t)stream) < 0 ? -1 : 0;
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
