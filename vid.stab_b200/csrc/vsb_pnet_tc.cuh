/*
 * vsb_pnet_tc.cuh -- the proposal network's forward pass on the fifth-
 * generation tensor cores (tcgen05.mma, kind::f16, bf16 operands from shared
 * memory, fp32 accumulators in tensor memory), one item per CTA at a time.
 *
 * Every convolution is an implicit GEMM D[pixels][32 out channels] =
 * A[pixels][9 taps x 32 in channels] * W.  The operands sit in shared memory
 * in the canonical K-major layout without swizzle: 8 rows x 16 bytes per
 * core matrix; SBO = distance between 8-row groups along M (N), LBO =
 * distance between the two 8-element core matrices of one K = 16 step.
 *
 *   conv1   im2col A1 [1024 pixels][32] (9 taps x 2 channels, zero padded),
 *           8 MMAs of M = 128 per K step, into TMEM columns 0..255
 *   conv2-4 stride 2: the input activation is stored as four parity planes
 *           per 8-channel chunk (cell = 8 channels = 16 bytes, zero borders),
 *           so tap (ky, kx) of eight consecutive output columns reads eight
 *           consecutive cells of one plane: the tap is a plain descriptor
 *           offset, no im2col copy.  M = 128 per MMA (conv2: one per half of
 *           the output columns; conv3 and conv4 use 64 and 16 of the rows)
 *
 * The epilogues read the accumulators with tcgen05.ld (one TMEM lane per
 * thread, 32 columns), add the bias, apply ReLU, round to bf16 and write the
 * next layer's planes.  The head (512 -> 3) runs on the CUDA cores.
 *
 * One thread issues the MMAs and commits them to an mbarrier; every wait is
 * bounded: a wait that gives up raises *err (if given), waits once more
 * (bounded) and the CTA releases its tensor memory and returns.
 */
#ifndef VSB_PNET_TC_CUH
#define VSB_PNET_TC_CUH

#include "vsb_pnet_dev.cuh"

/* shared memory map (bytes) */
#define TC_W1 0                     /* conv1 B: 4 K chunks x 4 channel groups x 128 */
#define TC_W2 (TC_W1 + 2048)        /* conv2 B: 9 taps x 4 K chunks x 4 groups x 128 */
#define TC_W3 (TC_W2 + 18432)
#define TC_W4 (TC_W3 + 18432)
#define TC_FC (TC_W4 + 18432)       /* head [3][512] plain */
#define TC_B (TC_FC + 3072)         /* f32 biases [131] */
#define TC_IN (TC_B + 528)          /* [34][34] words (2 channels), zero border */
#define TC_ACT1 (TC_IN + 4624)      /* conv2 A: 4 chunks x 4 parities x 17 x 17 cells */
#define TC_CH1 (4 * 17 * 17 * 16)   /* chunk stride of ACT1 */
#define TC_PL1 (17 * 17 * 16)       /* parity-plane stride of ACT1 */
#define TC_R (TC_ACT1 + 4 * TC_CH1) /* A1 during conv1; afterwards ACT2, ACT3, ACT4 */
#define TC_A1 TC_R                  /* [128 groups][4 chunks] x 128 = 65536 */
#define TC_ACT2 TC_R                /* 4 chunks x 4 parities x 9 x 9 cells */
#define TC_CH2 (4 * 9 * 9 * 16)
#define TC_PL2 (9 * 9 * 16)
#define TC_ACT3 (TC_ACT2 + 4 * TC_CH2) /* 4 chunks x 4 parities x 5 x 5 cells */
#define TC_CH3 (4 * 5 * 5 * 16)
#define TC_PL3 (5 * 5 * 16)
#define TC_ACT4 (TC_ACT3 + 4 * TC_CH3) /* f32 [16 pixels][32] */
#define TC_REND (TC_R + 65536)
#define TC_SMEM TC_REND
#define TC_TMEM_COLS 256

/* the 128-row MMAs of conv3 and conv4 read past their planes into the
   rest of region R (their extra rows are never used): keep those reads
   inside it */
static_assert(TC_ACT4 + 2048 <= TC_REND, "region R holds ACT2..ACT4");
static_assert(TC_ACT2 + 3 * TC_CH2 + 3 * TC_PL2 + (16 * 9 + 1 + 8 + 7) * 16 + 16 + TC_CH2 <= TC_REND,
              "conv3 reads stay in region R");
static_assert(TC_ACT3 + 3 * TC_CH3 + 3 * TC_PL3 + (16 * 5 + 1 + 8 + 7) * 16 + 16 + TC_CH3 <= TC_REND,
              "conv4 reads stay in region R");

__device__ __forceinline__ uint32_t tc_saddr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

/* shared-memory matrix descriptor: K-major, no swizzle (sm_100 version 1) */
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

/* instruction descriptor: kind::f16, bf16 x bf16 -> f32, both K-major,
   M = 128, N = 32 */
#define TC_IDESC ((1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24))

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
/* generic-proxy shared-memory writes become visible to the tensor cores */
__device__ __forceinline__ void tc_fence_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

/* bounded wait for the mbarrier phase `parity` to complete (every thread
   polls); returns 0 if it gave up */
__device__ __forceinline__ int tc_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return 1;
  }
  return 0;
}

/* 32 consecutive fp32 columns of this thread's TMEM lane */
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

/* an mbarrier for one arrival per phase (the commit of the MMAs) */
__device__ __forceinline__ void tc_mbar_init(uint64_t* mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc_saddr(mbar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

/* tensor memory of the CTA: allocated by warp 0 (address into *slot) */
__device__ __forceinline__ void tc_alloc(uint32_t* slot) {
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 :
                 : "r"(tc_saddr(slot)), "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr) {
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 :
                 : "r"(taddr), "r"(TC_TMEM_COLS)
                 : "memory");
}

/* bf16 pair of (relu(a), relu(b)) as one word */
__device__ __forceinline__ uint32_t tc_pack(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(a, 0.f), fmaxf(b, 0.f));
  return *(uint32_t*)&h;
}

/* Stages the weights in the canonical layouts and the biases, zeroes the
   input and ACT1 (their borders are never written again).  Block of
   PI_THREADS threads. */
__device__ __forceinline__ void pn_tc_stage(uint8_t* sm, const void* params) {
  const PNPtr P = pn_ptr(params);
  const int tid = threadIdx.x;
  /* conv1: W1 [32 co][32 k] -> core matrix (k chunk c, co group g) at (c*4 + g)*128 */
  for (int i = tid; i < 32 * 4; i += PI_THREADS) {
    const int co = i >> 2, c = i & 3;
    *(uint4*)(sm + TC_W1 + ((c * 4 + (co >> 3)) * 128) + (co & 7) * 16) =
        ((const uint4*)P.w1)[co * 4 + c];
  }
  /* conv2..4: W [9*32 (tap, co)][32 ci] -> (tap, c, g) at ((tap*4 + c)*4 + g)*128 */
  for (int i = tid; i < 288 * 4; i += PI_THREADS) {
    const int row = i >> 2, c = i & 3, tap = row >> 5, co = row & 31;
    const int d = ((tap * 4 + c) * 4 + (co >> 3)) * 128 + (co & 7) * 16;
    *(uint4*)(sm + TC_W2 + d) = ((const uint4*)P.w2)[i];
    *(uint4*)(sm + TC_W3 + d) = ((const uint4*)P.w3)[i];
    *(uint4*)(sm + TC_W4 + d) = ((const uint4*)P.w4)[i];
  }
  for (int i = tid; i < PN_NFC / 8; i += PI_THREADS)
    ((uint4*)(sm + TC_FC))[i] = ((const uint4*)P.fc)[i];
  for (int i = tid; i < PN_NF32; i += PI_THREADS) ((float*)(sm + TC_B))[i] = P.b1[i];
  for (int i = tid; i < (TC_R - TC_IN) / 16; i += PI_THREADS)
    ((uint4*)(sm + TC_IN))[i] = make_uint4(0, 0, 0, 0);
  tc_fence_smem();
  __syncthreads();
}

/* cell of 8-channel chunk c of pixel (y, x) of a stride-2 layer's input
   (H x H pixels, parity planes of P x P cells, P = H/2 + 1, chunk stride CH) */
__device__ __forceinline__ int tc_cell(int y, int x, int c, int P, int CH) {
  const int Y = y + 1, X = x + 1;
  return c * CH + (((Y & 1) * 2 + (X & 1)) * P * P + (Y >> 1) * P + (X >> 1)) * 16;
}

/* the 18 MMAs (9 taps x 2 K steps) of one 128-row tile of a stride-2 conv:
   A rows = 16 groups of 8 consecutive output columns, group j = output row
   j (its planes P cells wide, chunk stride CH), first column x0 */
__device__ __forceinline__ void tc_conv_s2(uint32_t d, uint32_t act, uint32_t w, int P, int CH,
                                           int x0) {
  const int PL = P * P * 16;
#pragma unroll 1
  for (int tap = 0; tap < 9; tap++) {
    const int ky = tap / 3, kx = tap - 3 * ky;
    const uint32_t a0 =
        act + ((ky & 1) * 2 + (kx & 1)) * PL + ((ky >> 1) * P + (kx >> 1) + x0) * 16;
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const uint64_t ad = tc_desc(a0 + 2 * s * CH, CH, P * 16);
      const uint64_t bd = tc_desc(w + (tap * 4 + 2 * s) * 4 * 128, 512, 128);
      tc_mma(d, ad, bd, tap | s);
    }
  }
}

/* The network on items s0, s0 + ds, ... below n (raw outputs out[s][3]),
   weights staged by pn_tc_stage, tensor memory at taddr (TC_TMEM_COLS
   columns), mbar an initialised mbarrier whose next phase parity is
   *phase.  Block of PI_THREADS threads.  Returns 0, or -1 when a wait for
   the tensor cores gave up (err raised). */
__device__ __forceinline__ int pn_tc_items(uint8_t* sm, uint32_t taddr, uint32_t mbar,
                                           uint32_t* phase, const uint8_t* __restrict__ curr,
                                           const uint8_t* __restrict__ prev, int pitch, int W,
                                           int H, const vsbd_item* __restrict__ items,
                                           const uint32_t* __restrict__ prepared, int s0, int n,
                                           int ds, float* __restrict__ out, unsigned* err) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = warp & 3; /* the TMEM lane quarter this warp may read */
  const float* sB = (const float*)(sm + TC_B);
  uint32_t* sIn = (uint32_t*)(sm + TC_IN);
  float* sAct4 = (float*)(sm + TC_ACT4);
  const uint32_t base = tc_saddr(sm);
  uint32_t ph = *phase;
  int ok = 1;
  /* one commit + bounded wait; the thread-sync fences order TMEM accesses
     around the barrier */
#define TC_SYNC_MMA()                                        \
  do {                                                       \
    if (tid == 0) tc_commit(mbar);                           \
    if (!tc_wait(mbar, ph)) {                                \
      ok = 0;                                                \
      if (tid == 0 && err) atomicExch(err, 1u);              \
      tc_wait(mbar, ph);                                     \
    }                                                        \
    ph ^= 1u;                                                \
    tc_fence_after();                                        \
  } while (0)

  for (int s = s0; s < n && ok; s += ds) {
    /* 1. input planes (zero border) */
    if (prepared) {
      const uint32_t* src = prepared + (size_t)s * 1024;
      for (int i = tid; i < 1024; i += PI_THREADS) sIn[((i >> 5) + 1) * 34 + (i & 31) + 1] = src[i];
    } else {
      /* the two 64 x 64 windows, row by row into region R: 80 bytes a row
         from the 16-byte boundary at or left of the window (raw byte e + j
         holds column x0 + j, e = x0 mod 16), rows and columns outside the
         frame clamped as crop_value clamps them; 16-byte loads where the
         whole row lies inside the frame, bytes elsewhere */
      const vsbd_item it = items[s];
      uint8_t* raw = sm + TC_R; /* [2 planes][64 rows][80] */
      const bool vec = (((uintptr_t)curr | (uintptr_t)prev | (uintptr_t)pitch) & 15) == 0;
      for (int i = tid; i < 2 * 64 * 5; i += PI_THREADS) {
        const int ch = i / 320, rem = i - ch * 320, r = rem / 5, v = rem - r * 5;
        const int x0 = (ch ? it.x + it.ox : it.x) - 32;
        const int y0 = (ch ? it.y + it.oy : it.y) - 32;
        const uint8_t* row = (ch ? prev : curr) + (size_t)min(max(y0 + r, 0), H - 1) * pitch;
        const int xa = x0 & ~15;
        uint8_t* dst = raw + (ch * 64 + r) * 80 + v * 16;
        if (vec && xa >= 0 && xa + 80 <= W) {
          *(uint4*)dst = *(const uint4*)(row + xa + v * 16);
        } else {
#pragma unroll
          for (int b = 0; b < 16; b++) dst[b] = row[min(max(xa + v * 16 + b, 0), W - 1)];
        }
      }
      __syncthreads();
      bf16* sInh = (bf16*)sIn;
      for (int i = tid; i < 2048; i += PI_THREADS) {
        const int r = i >> 6, c = (i >> 1) & 31, ch = i & 1;
        const int x0 = (ch ? it.x + it.ox : it.x) - 32;
        const uint8_t* q4 = raw + (ch * 64 + 2 * r) * 80 + (x0 & 15) + 2 * c;
        const int sum = (int)q4[0] + (int)q4[1] + (int)q4[80] + (int)q4[81];
        sInh[((r + 1) * 34 + c + 1) * 2 + ch] = __float2bfloat16_rn((float)(sum - 512) / 256.0f);
      }
    }
    __syncthreads();
    /* 2. im2col of conv1: pixel m -> 9 tap words + zeros, 4 chunks of 16 B
          at (m/8 * 4 + chunk) * 128 + (m%8) * 16 */
    for (int m = tid; m < 1024; m += PI_THREADS) {
      const int y = m >> 5, x = m & 31;
      uint32_t wv[16];
#pragma unroll
      for (int tap = 0; tap < 9; tap++) wv[tap] = sIn[(y + tap / 3) * 34 + x + tap % 3];
#pragma unroll
      for (int j = 9; j < 16; j++) wv[j] = 0u;
      uint8_t* dst = sm + TC_A1 + (m >> 3) * 512 + (m & 7) * 16;
#pragma unroll
      for (int c = 0; c < 4; c++)
        *(uint4*)(dst + c * 128) = make_uint4(wv[4 * c], wv[4 * c + 1], wv[4 * c + 2], wv[4 * c + 3]);
    }
    tc_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll 1
      for (int t = 0; t < 8; t++)
#pragma unroll
        for (int k = 0; k < 2; k++)
          tc_mma(taddr + t * 32, tc_desc(base + TC_A1 + t * 8192 + k * 256, 128, 512),
                 tc_desc(base + TC_W1 + k * 1024, 512, 128), k);
    }
    TC_SYNC_MMA();
    /* 3. conv1 epilogue: warp w reads tiles w/4 and w/4 + 4 of its lane
          quarter; pixel m = tile*128 + q*32 + lane */
#pragma unroll 1
    for (int t = warp >> 2; t < 8; t += 4) {
      float v[32];
      tc_ld32(taddr + ((uint32_t)(q * 32) << 16) + t * 32, v);
      const int m = t * 128 + q * 32 + lane, y = m >> 5, x = m & 31;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        uint4 o;
        o.x = tc_pack(v[8 * c + 0] + sB[8 * c + 0], v[8 * c + 1] + sB[8 * c + 1]);
        o.y = tc_pack(v[8 * c + 2] + sB[8 * c + 2], v[8 * c + 3] + sB[8 * c + 3]);
        o.z = tc_pack(v[8 * c + 4] + sB[8 * c + 4], v[8 * c + 5] + sB[8 * c + 5]);
        o.w = tc_pack(v[8 * c + 6] + sB[8 * c + 6], v[8 * c + 7] + sB[8 * c + 7]);
        *(uint4*)(sm + TC_ACT1 + tc_cell(y, x, c, 17, TC_CH1)) = o;
      }
    }
    tc_fence_before();
    __syncthreads();
    /* A1 is dead: zero ACT2 and ACT3 (borders) in region R */
    for (int i = tid; i < (TC_ACT4 - TC_ACT2) / 16; i += PI_THREADS)
      ((uint4*)(sm + TC_ACT2))[i] = make_uint4(0, 0, 0, 0);
    tc_fence_smem();
    __syncthreads();
    /* 4. conv2: two 128-row tiles (output columns 0-7, 8-15) */
    if (tid == 0) {
      tc_fence_after();
      tc_conv_s2(taddr, base + TC_ACT1, base + TC_W2, 17, TC_CH1, 0);
      tc_conv_s2(taddr + 32, base + TC_ACT1, base + TC_W2, 17, TC_CH1, 8);
    }
    TC_SYNC_MMA();
    if (warp < 8) {
      float v[32];
      const int h = warp >> 2;
      tc_ld32(taddr + ((uint32_t)(q * 32) << 16) + h * 32, v);
      const int m = q * 32 + lane, y = m >> 3, x = 8 * h + (m & 7);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        uint4 o;
        o.x = tc_pack(v[8 * c + 0] + sB[32 + 8 * c + 0], v[8 * c + 1] + sB[32 + 8 * c + 1]);
        o.y = tc_pack(v[8 * c + 2] + sB[32 + 8 * c + 2], v[8 * c + 3] + sB[32 + 8 * c + 3]);
        o.z = tc_pack(v[8 * c + 4] + sB[32 + 8 * c + 4], v[8 * c + 5] + sB[32 + 8 * c + 5]);
        o.w = tc_pack(v[8 * c + 6] + sB[32 + 8 * c + 6], v[8 * c + 7] + sB[32 + 8 * c + 7]);
        *(uint4*)(sm + TC_ACT2 + tc_cell(y, x, c, 9, TC_CH2)) = o;
      }
    }
    tc_fence_before();
    tc_fence_smem();
    __syncthreads();
    /* 5. conv3: one tile, rows 0..63 used (output row j, column r) */
    if (tid == 0) {
      tc_fence_after();
      tc_conv_s2(taddr, base + TC_ACT2, base + TC_W3, 9, TC_CH2, 0);
    }
    TC_SYNC_MMA();
    if (warp < 2) {
      float v[32];
      tc_ld32(taddr + ((uint32_t)(q * 32) << 16), v);
      const int m = q * 32 + lane, y = m >> 3, x = m & 7;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        uint4 o;
        o.x = tc_pack(v[8 * c + 0] + sB[64 + 8 * c + 0], v[8 * c + 1] + sB[64 + 8 * c + 1]);
        o.y = tc_pack(v[8 * c + 2] + sB[64 + 8 * c + 2], v[8 * c + 3] + sB[64 + 8 * c + 3]);
        o.z = tc_pack(v[8 * c + 4] + sB[64 + 8 * c + 4], v[8 * c + 5] + sB[64 + 8 * c + 5]);
        o.w = tc_pack(v[8 * c + 6] + sB[64 + 8 * c + 6], v[8 * c + 7] + sB[64 + 8 * c + 7]);
        *(uint4*)(sm + TC_ACT3 + tc_cell(y, x, c, 5, TC_CH3)) = o;
      }
    }
    tc_fence_before();
    tc_fence_smem();
    __syncthreads();
    /* 6. conv4: one tile, rows 8j + r with j, r < 4 used */
    if (tid == 0) {
      tc_fence_after();
      tc_conv_s2(taddr, base + TC_ACT3, base + TC_W4, 5, TC_CH3, 0);
    }
    TC_SYNC_MMA();
    if (warp == 0) {
      float v[32];
      tc_ld32(taddr, v);
      const int y = lane >> 3, x = lane & 7;
      if (y < 4 && x < 4) {
#pragma unroll
        for (int c = 0; c < 32; c++)
          sAct4[(y * 4 + x) * 32 + c] =
              __bfloat162float(__float2bfloat16_rn(fmaxf(v[c] + sB[96 + c], 0.f)));
      }
    }
    tc_fence_before();
    __syncthreads();
    /* 7. head */
    if (warp < 3) {
      const bf16* sFC = (const bf16*)(sm + TC_FC);
      float acc = 0.f;
      for (int k = lane; k < 512; k += 32) acc = fmaf(sAct4[k], bf(sFC[warp * 512 + k]), acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) out[(size_t)s * 3 + warp] = acc + sB[128 + warp];
    }
    __syncthreads();
  }
#undef TC_SYNC_MMA
  *phase = ph;
  return ok ? 0 : -1;
}

#endif
