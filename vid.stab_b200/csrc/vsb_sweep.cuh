/*
 * vsb_sweep.cuh -- persistent, TMA-staged SAD sweep of planar field sets
 * (the lattice and refinement search of src/motiondetect.c:439-586 in the
 * reference), for field rows of 16*NQ bytes and even lattice steps.
 *
 * Work split.  A tile is one field's lattice rows [b0, b0+nbb) across
 * 8*ncg lattice columns (the whole width for the field sizes served here).
 * The kernel is persistent: CTA c takes the tiles [c*T/G, (c+1)*T/G) of the
 * T tiles of the launch in order, so consecutive tiles mostly share a field.
 * Each tile's previous-frame window (and, when the field changes, the
 * current frame's field rows) is staged in shared memory by the TMA unit:
 * one cp.async.bulk per row, completing on an mbarrier.  Two buffers: tile
 * k+1's copies are in flight while tile k is summed.
 *
 * Sums.  A thread owns 8 consecutive lattice columns of one lattice row and
 * a strip of the field's rows.  Its columns start at byte E + c*STEP of a
 * 16-byte chunk of the window row, where E (0..15) is the same for every
 * thread of the tile (8*STEP is a multiple of 16), so the kernel selects a
 * body compiled for that E: every window word a column needs is a register
 * picked at compile time from the row's chunks, loaded with 16-byte shared
 * loads.  Instead of shifting the window into the columns' alignment, the
 * field is pre-shifted: copy F_s holds field bytes 4k-s .. 4k-s+3 in word k
 * (zero outside the field), so column c (byte offset o, s = o & 3) sums
 * word k of F_s against window word (o >> 2) + k; the s bytes before the
 * column in its first window word and the bytes after the field in its last
 * are masked off.  The packed SAD of four bytes with accumulate
 * (vabsdiff4.add) does all the arithmetic; the strips' partial sums are
 * added in shared memory.
 *
 * Winner.  Every candidate gets its full sum; the lowest (SAD, rank) pair
 * wins, rank being the candidate's position in the reference's visiting
 * order, so equal SADs resolve as its strict `<` scan does.  Each thread
 * keeps its lowest pair over the CTA's consecutive tiles of one field; after
 * its last tile of that field the CTA folds the best pair into the field's
 * 64-bit key with one atomicMin and takes a ticket.  The tile ranges are
 * fixed by the grid, so the number of CTAs that have tiles of a field is
 * known; the CTA drawing the last of those tickets runs the refinement
 * rounds and the range test and resets the key and ticket, as the
 * one-launch-per-tile search (vsb_search.cuh) does after a field's last
 * tile.
 *
 * Waits on the mbarriers are bounded (polls and clock cycles); a wait that
 * runs out raises *err, waits once more (bounded) for the CTA's copies and
 * ends the CTA.
 */
#ifndef VSB_SWEEP_CUH
#define VSB_SWEEP_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "vsb_search.cuh"

/* lattice columns per thread */
#define SW_TA 8
/* largest block */
#define SW_MAX_THREADS 512
/* bounded mbarrier wait: polls, then SM clock cycles (about 1 s) */
#define SW_WAIT_POLLS (1u << 26)
#define SW_WAIT_CYCLES 2000000000ll

/* words of a column's window row the sums read, last one included: the
   column starts at byte o = E + c*STEP of the thread's chunks */
__host__ __device__ constexpr int sw_last_word(int E, int STEP, int NQ) {
  return ((E + 7 * STEP) >> 2) + 4 * NQ - 1 + (((E + 7 * STEP) & 3) ? 1 : 0);
}
/* 16-byte chunks of a window row one thread loads (largest over E) */
__host__ __device__ constexpr int sw_chunks(int STEP, int NQ) {
  return sw_last_word(15, STEP, NQ) / 4 + 1;
}

/* shared-memory layout of the sweep for a tiling (g.ncg = g.nab / 8
   column groups, g.nbb lattice rows, g.nstrip strips) */
struct SweepLayout {
  int NQ, WPc, X, WH, FR, FCP;
  size_t win_bytes, fraw_bytes, fc_bytes;
  size_t off_win[2], off_fraw[2], off_fc, off_part, off_q, total;
};

/* chunk offset of window row r: rows STEP apart differ by an odd multiple
   of the thread stride, so the 16-byte loads of 8 consecutive threads hit
   distinct bank groups */
__host__ __device__ inline int sw_row_off(int r, int WPc, int X, int step) {
  return r * WPc + (r / step) * X;
}

__host__ __device__ inline SweepLayout sweep_layout(const DGeom& g) {
  SweepLayout L;
  L.NQ = g.S / 16;
  const int ncg = g.nab / SW_TA;
  const int cs = g.step / 2; /* chunks between column groups */
  L.WPc = (ncg - 1) * cs + sw_chunks(g.step, L.NQ);
  L.X = (((cs * ncg - g.step * L.WPc) % 8) + 8) % 8;
  L.WH = g.S + (g.nbb - 1) * g.step;
  L.FR = g.S + 16;
  L.FCP = (L.NQ + 1) * 16;
  L.win_bytes = (size_t)16 * (sw_row_off(L.WH - 1, L.WPc, L.X, g.step) + L.WPc);
  /* the refinement window of a field reuses a tile buffer */
  const int R = refine_reach(g);
  const size_t rwin = (size_t)(g.S + 2 * R) * (((3 + g.S + 2 * R + 8 + 15) >> 4) << 4) + 16;
  if (rwin > L.win_bytes) L.win_bytes = rwin;
  L.win_bytes = (L.win_bytes + 127) & ~(size_t)127;
  L.fraw_bytes = (((size_t)g.S * L.FR) + 127) & ~(size_t)127;
  L.fc_bytes = (size_t)3 * g.S * L.FCP;
  L.off_win[0] = 0;
  L.off_win[1] = L.win_bytes;
  L.off_fraw[0] = 2 * L.win_bytes;
  L.off_fraw[1] = L.off_fraw[0] + L.fraw_bytes;
  L.off_fc = L.off_fraw[1] + L.fraw_bytes;
  L.off_part = L.off_fc + L.fc_bytes;
  L.off_q = L.off_part + (size_t)g.nstrip * ncg * g.nbb * SW_TA * 4;
  L.total = L.off_q + (size_t)g.maxq * 4 + 16;
  return L;
}

/* the tile t of a launch: field, lattice block, window and field origins */
struct SweepTile {
  int item, a0, b0, na_t, nb_t;
  int gx0a, gy0, e;   /* window: 16-byte aligned start column, first row, E */
  int cx0a, cy0, ce;  /* field rows: aligned start, first row, offset */
};

__device__ __forceinline__ SweepTile sweep_tile(const DGeom& g, const vsbd_item* __restrict__ items,
                                                int t) {
  SweepTile T;
  const int per = g.nta * g.ntb;
  T.item = t / per;
  const int r = t - T.item * per;
  const int tbi = r / g.nta, tai = r - tbi * g.nta;
  T.a0 = tai * g.nab;
  T.b0 = tbi * g.nbb;
  T.na_t = min(g.nab, g.na - T.a0);
  T.nb_t = min(g.nbb, g.nb - T.b0);
  const vsbd_item it = items[T.item];
  const int gx0 = it.x - g.S / 2 + it.ox + g.ax0 + T.a0 * g.step;
  T.gy0 = it.y - g.S / 2 + it.oy + g.by0 + T.b0 * g.step;
  T.gx0a = gx0 & ~15;
  T.e = gx0 - T.gx0a;
  const int cx0 = it.x - g.S / 2;
  T.cy0 = it.y - g.S / 2;
  T.cx0a = cx0 & ~15;
  T.ce = cx0 - T.cx0a;
  return T;
}

/* ---- mbarrier and bulk-copy primitives (PTX) ---- */

__device__ __forceinline__ uint32_t sw_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void sw_bar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sw_smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void sw_bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void sw_bar_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sw_smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

/* one bulk copy global -> shared (16-byte aligned ends, size a multiple of
   16) completing on bar */
__device__ __forceinline__ void sw_bulk_load(void* dst, const void* src, unsigned bytes,
                                             uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(sw_smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(sw_smem_addr(bar))
      : "memory");
}

/* generic-proxy accesses of shared memory before the async proxy's writes */
__device__ __forceinline__ void sw_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool sw_bar_try(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sw_smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/* bounded wait for phase `parity` of bar; false if it ran out */
__device__ __forceinline__ bool sw_bar_wait(uint64_t* bar, unsigned parity) {
  const long long t0 = clock64();
  for (unsigned i = 0; i < SW_WAIT_POLLS; i++) {
    if (sw_bar_try(bar, parity)) return true;
    if ((i & 255) == 255 && clock64() - t0 > SW_WAIT_CYCLES) break;
  }
  return false;
}

/* bytes tile T's copies bring: its window rows and, with field, the rows
   of its field in the current frame */
template <int STEP>
__device__ __forceinline__ unsigned sweep_bytes(const DGeom& g, const SweepTile& T, bool field) {
  const int nvec = (T.e + (T.na_t - 1) * STEP + g.S + 15) >> 4;
  const int wh = g.S + (T.nb_t - 1) * STEP;
  const int nvf = (T.ce + g.S + 15) >> 4;
  return (unsigned)(wh * nvec * 16 + (field ? g.S * nvf * 16 : 0));
}

/* Issues tile T's copies into a buffer, one row per copy, the rows spread
   over all threads of the CTA (issuing a copy costs its thread time, so no
   warp carries them all); the buffer's mbarrier already expects their bytes
   (sweep_bytes). */
template <int STEP>
__device__ __forceinline__ void sweep_copies(const DGeom& g, const SweepLayout& L, const SweepTile& T,
                                             bool field, const uint8_t* __restrict__ curr,
                                             const uint8_t* __restrict__ prev, int pitch,
                                             uint8_t* win, uint8_t* fraw, uint64_t* bar) {
  const int nvec = (T.e + (T.na_t - 1) * STEP + g.S + 15) >> 4;
  const int wh = g.S + (T.nb_t - 1) * STEP;
  const int nvf = (T.ce + g.S + 15) >> 4;
  const int nrows = wh + (field ? g.S : 0);
  for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
    if (r < wh)
      sw_bulk_load(win + 16 * sw_row_off(r, L.WPc, L.X, STEP),
                   prev + (size_t)(T.gy0 + r) * pitch + T.gx0a, (unsigned)nvec * 16u, bar);
    else
      sw_bulk_load(fraw + (size_t)(r - wh) * L.FR,
                   curr + (size_t)(T.cy0 + r - wh) * pitch + T.cx0a, (unsigned)nvf * 16u, bar);
  }
}

/* Builds the field copies of one field from its raw rows (S = 16*NQ rows of
   S+16 bytes, the field starting at byte ce): slot 0 the field aligned
   (shift 0), slot 1 shifted by sA bytes, slot 2 by sB (slots 1 and 2 only
   for nonzero shifts).  Word k of the copy for shift s holds field bytes
   4k-s .. 4k-s+3, zero outside the field.  A thread builds one 16-byte
   quad of a copy row from five raw words. */
template <int NQ>
__device__ __forceinline__ void sweep_field_copies(const uint8_t* fraw, int ce, int sA, int sB,
                                                   uint8_t* fc) {
  constexpr int S = 16 * NQ, Q = NQ + 1, FRW = (S + 16) / 4, ROWW = 4 * NQ;
  constexpr int PER_SLOT = S * Q;
  for (int i = threadIdx.x; i < 3 * PER_SLOT; i += blockDim.x) {
    const int slot = i / PER_SLOT;
    const int j = i - slot * PER_SLOT;
    const int r = j / Q, m = j - r * Q;
    const int s = slot == 0 ? 0 : (slot == 1 ? sA : sB);
    if (slot > 0 && s == 0) continue;
    const uint32_t* row = (const uint32_t*)(fraw + (size_t)r * (S + 16));
    const int b0 = ce + 16 * m - s; /* raw byte of field byte 16m-s (at least -3) */
    const int a0 = b0 >> 2, sh = (b0 & 3) * 8;
    uint32_t w[5];
#pragma unroll
    for (int t = 0; t < 5; t++) w[t] = (a0 + t >= 0 && a0 + t < FRW) ? row[a0 + t] : 0u;
    uint32_t v[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int k = 4 * m + t;
      uint32_t x = sh ? __funnelshift_r(w[t], w[t + 1], sh) : w[t];
      if (k == 0 && s) x &= 0xffffffffu << (8 * s);
      if (k == ROWW) x &= s ? (0xffffffffu >> (32 - 8 * s)) : 0u;
      if (k > ROWW) x = 0u;
      v[t] = x;
    }
    *(uint4*)(fc + (size_t)slot * S * Q * 16 + (size_t)r * Q * 16 + 16 * m) =
        make_uint4(v[0], v[1], v[2], v[3]);
  }
}

/* The refinement of one item by the whole CTA (the rounds of
   src/motiondetect.c:545-567 after the lattice winner: i outer, j inner,
   centre skipped, strict <, then the range test of :573-574).  The window
   the rounds can reach is staged with 16-byte loads into rwin; every
   round's candidate SADs are split over the threads by (candidate, group
   of field rows) and totalled in shared memory; thread 0 then scans them
   in the reference's order.  F0: the aligned field copy ((NQ+1) quads per
   row).  Resets the item's key and ticket. */
template <int NQ>
__device__ void sweep_refine(const DGeom& g, const vsbd_item& it, const uint8_t* F0, uint8_t* rwin,
                             const uint8_t* __restrict__ prev, int pitch,
                             unsigned long long* keys, unsigned* tickets, vsbd_result* res,
                             int item, unsigned* part, unsigned* qsad) {
  constexpr int S = 16 * NQ, Q = NQ + 1;
  __shared__ int s_tx, s_ty, s_cx0, s_cy0;
  __shared__ unsigned s_min;
  if (threadIdx.x == 0) {
    const unsigned long long k = atomicAdd(&keys[item], 0ull);
    const short2 pt = g.point[(unsigned)(k & 0xffffffffu)];
    s_min = (unsigned)(k >> 32);
    s_tx = s_cx0 = pt.x;
    s_ty = s_cy0 = pt.y;
  }
  __syncthreads();
  const int R = refine_reach(g);
  const int fx0 = it.x - S / 2 + it.ox, fy0 = it.y - S / 2 + it.oy;
  if (g.nstages > 0) {
    /* rows fy0 + cy0 - R .. + S + 2R, bytes from fx0 + cx0 - R */
    const int cx0 = s_cx0, cy0 = s_cy0;
    const int wx = fx0 + cx0 - R, wy = fy0 + cy0 - R;
    const int wxa = wx & ~15, off = wx - wxa;
    const int nc = (off + S + 2 * R + 4 + 15) / 16; /* chunks a row's SADs can read */
    const int RH = S + 2 * R;
    const int tot = RH * nc;
    for (int i0 = threadIdx.x; i0 < tot; i0 += 4 * blockDim.x) {
      uint4 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u * blockDim.x;
        if (i < tot) {
          const int r = i / nc, c = i - r * nc;
          v[u] = *(const uint4*)(prev + (size_t)(wy + r) * pitch + wxa + 16 * c);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u * blockDim.x;
        if (i < tot) *(uint4*)(rwin + 16 * (size_t)i) = v[u];
      }
    }
    __syncthreads();
    const int rp = 16 * nc; /* staged row pitch */
    for (int st = 0; st < g.nstages; st++) {
      const int r = g.st_r[st], h = g.st_h[st];
      const int side = (2 * r) / h + 1, nq = side * side;
      const int cx = s_tx, cy = s_ty;
      const int G = (int)blockDim.x / nq; /* row groups */
      const int t = threadIdx.x;
      unsigned acc = 0, a1 = 0, a2 = 0, a3 = 0; /* four chains: one per word of a quad */
      if (G > 0 && t < nq * G) {
        const int q = t % nq, grp = t / nq;
        const int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
        if (!(i == cx && j == cy)) {
          const int bx = off + (i - cx0 + R); /* byte of the candidate's column 0 */
          const int sh = (bx & 3) * 8;
          for (int rr = grp; rr < S; rr += G) {
            const uint32_t* W = (const uint32_t*)(rwin + (size_t)(j - cy0 + R + rr) * rp) + (bx >> 2);
            const uint4* F = (const uint4*)(F0 + (size_t)rr * Q * 16);
            uint32_t lo = W[0];
#pragma unroll
            for (int qq = 0; qq < NQ; qq++) {
              const uint4 f = F[qq];
              const uint32_t w1 = W[4 * qq + 1], w2 = W[4 * qq + 2], w3 = W[4 * qq + 3],
                             w4 = W[4 * qq + 4];
              acc = sad4(f.x, sh ? __funnelshift_r(lo, w1, sh) : lo, acc);
              a1 = sad4(f.y, sh ? __funnelshift_r(w1, w2, sh) : w1, a1);
              a2 = sad4(f.z, sh ? __funnelshift_r(w2, w3, sh) : w2, a2);
              a3 = sad4(f.w, sh ? __funnelshift_r(w3, w4, sh) : w3, a3);
              lo = w4;
            }
          }
          acc += a1 + a2 + a3;
        } else {
          acc = 0xffffffffu; /* the centre is not a candidate */
        }
        part[grp * nq + q] = acc;
      }
      __syncthreads();
      /* each candidate's total over the row groups (the centre's is never
         compared) */
      if (threadIdx.x < nq) {
        unsigned sd = 0;
        for (int gg = 0; gg < G; gg++) sd += part[gg * nq + threadIdx.x];
        qsad[threadIdx.x] = sd;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned m = s_min;
        int tx = cx, ty = cy;
        for (int q = 0; q < nq; q++) {
          const int i = cx - r + (q / side) * h, j = cy - r + (q % side) * h;
          if (i == cx && j == cy) continue;
          const unsigned sd = qsad[q];
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

/* The sums of one thread: 8 lattice columns starting at byte E + c*STEP of
   the thread's window chunks, field rows r0 .. r0+Rs-1 against window rows
   wr0 .. wr0+Rs-1.  fA / fB: the field copies of the even / odd columns. */
template <int NQ, int STEP, int E>
__device__ __forceinline__ void sweep_sums(unsigned (&acc)[SW_TA], const uint8_t* __restrict__ win,
                                           int WPc, int X, int cgoff, int wr0,
                                           const uint8_t* __restrict__ fA,
                                           const uint8_t* __restrict__ fB, int FCP, int r0,
                                           int Rs) {
  constexpr int SA = E & 3, SB = (E + STEP) & 3;
  constexpr int NCH = sw_last_word(E, STEP, NQ) / 4 + 1;
  const uint4* __restrict__ W0 = (const uint4*)win + cgoff;
  for (int r = 0; r < Rs; r++) {
    const int wr = wr0 + r;
    const uint4* __restrict__ W4 = W0 + sw_row_off(wr, WPc, X, STEP);
    const uint4* __restrict__ FA4 = (const uint4*)(fA + (size_t)(r0 + r) * FCP);
    const uint4* __restrict__ FB4 = (const uint4*)(fB + (size_t)(r0 + r) * FCP);
    uint32_t w[4 * NCH];
#pragma unroll
    for (int j = 0; j < NCH; j++) {
      const uint4 v = W4[j];
      w[4 * j] = v.x;
      w[4 * j + 1] = v.y;
      w[4 * j + 2] = v.z;
      w[4 * j + 3] = v.w;
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const uint4 fa = FA4[q];
      const uint4 fb = SB == SA ? fa : FB4[q];
      const uint32_t fav[4] = { fa.x, fa.y, fa.z, fa.w };
      const uint32_t fbv[4] = { fb.x, fb.y, fb.z, fb.w };
      /* word-major: the eight columns' accumulations are independent, so
         consecutive packed SADs never wait on one another */
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int k = 4 * q + i;
#pragma unroll
        for (int c = 0; c < SW_TA; c++) {
          const int o = E + c * STEP, wc = o >> 2, s = o & 3;
          uint32_t ww = w[wc + k];
          if (k == 0 && s) ww &= 0xffffffffu << (8 * s);
          acc[c] = sad4(((c & 1) && SB != SA) ? fbv[i] : fav[i], ww, acc[c]);
        }
      }
    }
    /* the last word of a shifted copy: the field's final s bytes */
    if (SA) {
      const uint32_t ta = ((const uint32_t*)FA4)[4 * NQ];
#pragma unroll
      for (int c = 0; c < SW_TA; c += (SB == SA ? 1 : 2)) {
        const int o = E + c * STEP, wc = o >> 2;
        acc[c] = sad4(ta, w[wc + 4 * NQ] & (0xffffffffu >> (32 - 8 * SA)), acc[c]);
      }
    }
    if (SB && SB != SA) {
      const uint32_t tb = ((const uint32_t*)FB4)[4 * NQ];
#pragma unroll
      for (int c = 1; c < SW_TA; c += 2) {
        const int o = E + c * STEP, wc = o >> 2;
        acc[c] = sad4(tb, w[wc + 4 * NQ] & (0xffffffffu >> (32 - 8 * SB)), acc[c]);
      }
    }
  }
}

template <int NQ, int STEP>
__device__ __forceinline__ void sweep_sums_e(int E, unsigned (&acc)[SW_TA], const uint8_t* win,
                                             int WPc, int X, int cgoff, int wr0,
                                             const uint8_t* fA, const uint8_t* fB, int FCP,
                                             int r0, int Rs) {
#define SW_E(v) \
  case v: sweep_sums<NQ, STEP, v>(acc, win, WPc, X, cgoff, wr0, fA, fB, FCP, r0, Rs); break;
  switch (E) {
    SW_E(0) SW_E(1) SW_E(2) SW_E(3) SW_E(4) SW_E(5) SW_E(6) SW_E(7)
    SW_E(8) SW_E(9) SW_E(10) SW_E(11) SW_E(12) SW_E(13) SW_E(14) SW_E(15)
  }
#undef SW_E
}

/* grid: g.ctas persistent CTAs; block g.threads; dynamic shared memory
   sweep_layout(g).total.  Tiles of items[0 .. n). */
template <int NQ, int STEP>
__global__ void __launch_bounds__(SW_MAX_THREADS, 1)
    k_sweep(const uint8_t* __restrict__ curr, const uint8_t* __restrict__ prev, int pitch, DGeom g,
            const vsbd_item* __restrict__ items, int n, unsigned long long* __restrict__ keys,
            unsigned* __restrict__ tickets, vsbd_result* __restrict__ res, unsigned* err) {
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ unsigned long long red[SW_MAX_THREADS / 32];
  __shared__ int s_last;
  const SweepLayout L = sweep_layout(g);
  const int ncg = g.nab / SW_TA;
  const long T_ = (long)n * g.nta * g.ntb; /* tiles of the launch */
  const int t_begin = (int)((long)blockIdx.x * T_ / gridDim.x);
  const int t_end = (int)((long)(blockIdx.x + 1) * T_ / gridDim.x);
  const int nmine = t_end - t_begin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (nmine <= 0) return;
  uint8_t* fc = sm + L.off_fc;
  /* whether tile t needs its field staged: the first tile, a new field, or a
     new alignment of the window (which picks the field copies) */
  auto needs_field = [&](int t, const SweepTile& Tt) -> bool {
    if (t == t_begin) return true;
    const SweepTile Tp = sweep_tile(g, items, t - 1);
    return Tp.item != Tt.item || ((Tp.e ^ Tt.e) & 3);
  };
  if (threadIdx.x == 0) {
    sw_bar_init(&bars[0], 1);
    sw_bar_init(&bars[1], 1);
    sw_bar_init_fence();
    for (int k = 0; k < 2 && k < nmine; k++) {
      const SweepTile Tt = sweep_tile(g, items, t_begin + k);
      sw_bar_expect(&bars[k], sweep_bytes<STEP>(g, Tt, needs_field(t_begin + k, Tt)));
    }
  }
  __syncthreads();
  for (int k = 0; k < 2 && k < nmine; k++) {
    const SweepTile Tt = sweep_tile(g, items, t_begin + k);
    sweep_copies<STEP>(g, L, Tt, needs_field(t_begin + k, Tt), curr, prev, pitch,
                       sm + L.off_win[k], sm + L.off_fraw[k], &bars[k]);
  }
  /* thread task: column group, lattice row of the tile, field strip */
  const int tps = ncg * g.nbb;
  const int ntask = tps * g.nstrip;
  const int t = threadIdx.x;
  const bool active = t < ntask;
  const int st = active ? t / tps : 0;
  const int rem = active ? t - st * tps : 0;
  const int bl = rem / ncg, cg = rem - bl * ncg;
  const int Rs = g.S / g.nstrip;
  unsigned* part = (unsigned*)(sm + L.off_part);
  /* the lowest (SAD, rank) this thread has seen in the current field's
     tiles: the CTA folds it into the field's key once, after its last tile
     of the field */
  unsigned long long best = ~0ull;
  const int per_item = g.nta * g.ntb;
  for (int k = 0; k < nmine; k++) {
    const int tt = t_begin + k;
    const int b = k & 1;
    const SweepTile T = sweep_tile(g, items, tt);
    const bool field = needs_field(tt, T);
    const bool ok = sw_bar_wait(&bars[b], (unsigned)((k >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      /* the copies did not complete: report, give them one more bounded
         wait, and end this CTA */
      if (threadIdx.x == 0) {
        atomicExch(err, 1u);
        sw_bar_wait(&bars[b], (unsigned)((k >> 1) & 1));
        if (k + 1 < nmine) sw_bar_wait(&bars[b ^ 1], (unsigned)(((k + 1) >> 1) & 1));
      }
      return;
    }
    const int sA = T.e & 3, sB = (T.e + STEP) & 3;
    if (field) {
      sweep_field_copies<NQ>(sm + L.off_fraw[b], T.ce, sA, sB, fc);
      __syncthreads();
    }
    /* the rank of each candidate this thread totals after the sums, fetched
       now so that the load's latency hides behind them */
    constexpr int RK = 3; /* candidates per thread the prefetch covers */
    int32_t rank[RK];
#pragma unroll
    for (int u = 0; u < RK; u++) {
      const int q = threadIdx.x + u * (int)blockDim.x;
      rank[u] = -1;
      if (q < tps * SW_TA) {
        const int r2 = q / SW_TA, c = q - r2 * SW_TA;
        const int bl2 = r2 / ncg, cg2 = r2 - bl2 * ncg;
        if (bl2 < T.nb_t && cg2 * SW_TA + c < T.na_t)
          rank[u] = g.order[(size_t)(T.b0 + bl2) * g.na + T.a0 + cg2 * SW_TA + c];
      }
    }
    const uint8_t* win = sm + L.off_win[b];
    unsigned acc[SW_TA];
#pragma unroll
    for (int c = 0; c < SW_TA; c++) acc[c] = 0;
    if (active) {
      const uint8_t* fA = fc + (size_t)(sA ? 1 : 0) * g.S * L.FCP;
      const uint8_t* fB = fc + (size_t)(sB ? 2 : 0) * g.S * L.FCP;
      sweep_sums_e<NQ, STEP>(T.e, acc, win, L.WPc, L.X, cg * (STEP / 2), st * Rs + bl * STEP, fA,
                             fB, L.FCP, st * Rs, Rs);
    }
    /* every strip's partial sums go to shared memory; then the whole CTA
       totals the tile's candidates over the strips, each thread a few, and
       keeps the lowest (SAD, rank) */
    if (active) {
      uint4* p = (uint4*)(part + ((size_t)st * tps + rem) * SW_TA);
      p[0] = make_uint4(acc[0], acc[1], acc[2], acc[3]);
      p[1] = make_uint4(acc[4], acc[5], acc[6], acc[7]);
    }
    __syncthreads();
    for (int u = 0, q = threadIdx.x; q < tps * SW_TA; u++, q += blockDim.x) {
      const int r2 = q / SW_TA, c = q - r2 * SW_TA;
      const int bl2 = r2 / ncg, cg2 = r2 - bl2 * ncg;
      if (bl2 >= T.nb_t || cg2 * SW_TA + c >= T.na_t) continue;
      unsigned sum = 0;
      for (int s2 = 0; s2 < g.nstrip; s2++) sum += part[((size_t)s2 * tps + r2) * SW_TA + c];
      const int32_t rk =
          u < RK ? rank[u] : g.order[(size_t)(T.b0 + bl2) * g.na + T.a0 + cg2 * SW_TA + c];
      const unsigned long long key = ((unsigned long long)sum << 32) | (unsigned)rk;
      best = key < best ? key : best;
    }
    /* the CTA's last tile of this field: fold the field's best into its key
       and take a ticket; the field's tickets are counted per CTA that has
       tiles of it (the tile ranges are fixed by the grid) */
    const bool field_end = k + 1 == nmine || (tt + 1) / per_item != T.item;
    bool last = false;
    if (field_end) {
      best = warp_min64(best);
      if (lane == 0) red[warp] = best;
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < nwarps; w2++) best = red[w2] < best ? red[w2] : best;
        atomicMin(&keys[T.item], best);
        __threadfence();
        const unsigned tk = atomicAdd(&tickets[T.item], 1u);
        /* CTAs holding tiles of the field: with at least as many tiles as
           CTAs every CTA has some, so they are the owners of the field's
           first and last tiles and those between; with fewer, a CTA has at
           most one tile (and empty CTAs lie between the owners) */
        const long G = gridDim.x;
        const long f0 = (long)T.item * per_item, f1 = f0 + per_item - 1;
        const long c0 = ((f0 + 1) * G + T_ - 1) / T_ - 1, c1 = ((f1 + 1) * G + T_ - 1) / T_ - 1;
        const long holders = T_ >= G ? c1 - c0 + 1 : per_item;
        s_last = tk == (unsigned)(holders - 1);
      }
      __syncthreads();
      last = s_last;
      best = ~0ull;
    }
    if (last) {
      /* the field's last tile: refinement, with the aligned field copy and
         this tile's (now free) buffer as the refinement window */
      __threadfence();
      const vsbd_item it = items[T.item];
      sweep_refine<NQ>(g, it, fc, sm + L.off_win[b], prev, pitch, keys, tickets, res, T.item,
                       part, (unsigned*)(sm + L.off_q));
    }
    /* every thread's reads (and the refinement's writes) of buffer b are
       ordered before the bulk copies that refill it; the mbarrier expects
       tile k+2's bytes before any of its copies is issued */
    sw_fence_async_smem();
    const bool more = k + 2 < nmine;
    SweepTile Tn;
    bool fn = false;
    if (more) {
      Tn = sweep_tile(g, items, tt + 2);
      fn = needs_field(tt + 2, Tn);
      if (threadIdx.x == 0) sw_bar_expect(&bars[b], sweep_bytes<STEP>(g, Tn, fn));
    }
    __syncthreads();
    if (more)
      sweep_copies<STEP>(g, L, Tn, fn, curr, prev, pitch, sm + L.off_win[b], sm + L.off_fraw[b],
                         &bars[b]);
  }
}

#endif
