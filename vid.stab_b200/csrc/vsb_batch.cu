/*
 * vsb_batch.cu -- the detect pass of many independent streams at once, in
 * one persistent kernel per stage, each stage replayed from a captured CUDA
 * graph.
 *
 * A batch step advances every stream by one frame.  The device work of the
 * step is two queues of work items:
 *   stage A  blur tiles of every stream's new frame, then the coarse search
 *            tiles (field x lattice tile) of every stream, then the min/max
 *            of every stream's coarse and fine fields;
 *   stage B  the fine search tiles of the fine work lists the host built
 *            from stage A's results (selection, simple model, offsets --
 *            the same host code as the per-stream detector).
 * The persistent kernel's CTAs (as many as fit on the GPU at once) take
 * items from the queue in order with one atomic counter.  A search or
 * min/max item of a stream first waits until every blur tile of that
 * stream's frame is written: all blur items sit earlier in the queue, so they
 * were taken by CTAs that are running, and the wait always ends; it is
 * bounded anyway (time and iterations), after which the item is skipped and
 * an error flag is raised for the host.
 *
 * Each search item is exactly one CTA of the per-stream search kernel
 * (lattice_tile), with the same tiling rules, so each stream's results are
 * the per-stream detector's, bit for bit.  The tilings of every resolution
 * class are picked by timing candidate shapes in the persistent kernel itself
 * at batch creation.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vsb_batch.h"
#include "vsb_plan.h"
#include "vsb_pnet_dev.cuh"
#include "vsb_pnet_tc.cuh"
#include "vsb_prefilter.cuh"
#include "vsb_search.cuh"
#include "vsb_finewarp.cuh"

#define VSB_BATCH_THREADS 512
/* stage B (fine search only) runs the same kernel with 256-thread CTAs, two
   per SM: fine-field tiles need at most 256 threads, and a second CTA hides
   each tile's staging and reductions */
#define VSB_BATCH_THREADS_B 256
/* fields per min/max work item (one warp each; stage A has 16 warps) */
#define VSB_MM_GROUP 16
#define VSB_BATCH_MAX_STREAMS 1024
#define VSB_BATCH_MAX_CLASSES 64

/* per-stream descriptor, in device memory (rewritten every step) */
struct BStream {
  const uint8_t* src; /* raw plane 0 of this step's frame */
  int sp;             /* its row pitch */
  uint8_t* cur;       /* blurred current frame */
  uint8_t* prev;      /* blurred previous frame */
  int pitch, W, H, half;
  BlurDiv dv;
  int ntx, nty;           /* blur tiles */
  const int16_t* xy;      /* coarse x[nc], coarse y[nc], fine x[nf], fine y[nf] */
  int nc, nf, Sc, Sf;
  int gc, gf;             /* geometry classes of the coarse and fine fields */
  const vsbd_item* citems;
  unsigned long long* keys; /* coarse [0,nc), fine [nc, nc+nf) */
  unsigned* tickets;
  uint8_t* mm;            /* out: (nc+nf) (min,max) pairs */
  vsbd_result* cres;      /* out: nc */
  vsbd_result* fres;      /* out: nf */
  /* learned search proposal (pn == NULL: the dense search) */
  const void* pn;         /* network parameters */
  float* pout;            /* raw network outputs, nc x 3 */
  vsbd_item* citems2;     /* second pass: coarse items re-centred on the prior */
  short2* prior;          /* second pass: the prior's displacement per item */
  uint8_t* skip;          /* coarse fields below the contrast threshold */
  uint8_t* cfb;           /* out: coarse fallback flags (PN_FB_*) */
  int* cfl;               /* coarse items that fell back */
  int* ffl;               /* fine items that fell back */
  uint8_t* ffb;           /* fine fallback flags */
  double thr;             /* contrast threshold of the coarse fields */
  PNSearch psc, psf;      /* narrowed-search settings of coarse and fine fields */
  int fnarrow;            /* fine fields take the narrowed search (else the dense one) */
  int ffine;              /* the dense fine search runs one CTA per field (k_fine's body) */
  int passes;             /* network passes over the coarse fields (1 or 2) */
  int nchunk;             /* network items (VSB_PN_CHUNK coarse fields each) */
};

/* coarse fields per network work item: the CTA stages the weights once for
   them */
#define VSB_PN_CHUNK 8

/* stage-A work item: type 0 blur tile a; 1 min/max of fields
   a*VSB_MM_GROUP..; 2 coarse search tile a = item * ntiles + tile; with a
   search proposal: 3 first network pass over coarse fields
   a*VSB_PN_CHUNK..; 4 the stream's global motion prior; 5 second network
   pass over chunk a; 6 narrowed search of coarse field a */
struct BWork {
  int type, stream, a, pad;
};

/* default limits of the bounded waits: polls (100 ns apart) and SM clock
   cycles, about 1.7 s and 4 s on a B200 */
#define VSB_WAIT_SPINS (1u << 24)
#define VSB_WAIT_CYCLES 8000000000ll

/* control block of one stage */
struct BCtl {
  unsigned head;
  unsigned err;
  unsigned blur_done[VSB_BATCH_MAX_STREAMS];
  /* the proposal's per-stream progress: min/max items, first-pass network
     items, priors, second-pass network items, and fallbacks appended */
  unsigned mm_done[VSB_BATCH_MAX_STREAMS];
  unsigned inf_done[VSB_BATCH_MAX_STREAMS];
  unsigned prior_done[VSB_BATCH_MAX_STREAMS];
  unsigned inf2_done[VSB_BATCH_MAX_STREAMS];
  unsigned fbn[VSB_BATCH_MAX_STREAMS];
  unsigned narrow_done; /* narrowed searches finished */
  unsigned fb_head;     /* next fallback search tile */
  int nwork; /* set by the host; not cleared per launch (nor are the fields below) */
  int nnarrow; /* narrowed searches in the list (0: no fallback phase) */
  unsigned spin_limit;    /* a wait gives up after this many polls ... */
  long long cycle_limit;  /* ... or this many SM clock cycles */
};

/* Bounded wait of one CTA until the counter *p reaches target.  Returns 0
   if the wait gave up (the error flag is raised). */
__device__ __forceinline__ int wait_ge(BCtl* ctl, const unsigned* p, unsigned target) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    const long long t0 = clock64();
    const unsigned spin_limit = ctl->spin_limit;
    const long long cycle_limit = ctl->cycle_limit;
    unsigned spins = 0;
    int ok = 1;
    while (*(volatile const unsigned*)p < target) {
      if (++spins > spin_limit || clock64() - t0 > cycle_limit) {
        ok = 0;
        atomicExch(&ctl->err, 1u);
        break;
      }
      __nanosleep(100);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok;
}

/* Bounded wait until stream s has `target` blur tiles written. */
__device__ __forceinline__ int wait_blur(BCtl* ctl, int s, unsigned target) {
  return wait_ge(ctl, &ctl->blur_done[s], target);
}

/* counter += 1 once the CTA's writes are visible device-wide */
__device__ __forceinline__ void signal_done(unsigned* p) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(p, 1u);
  }
}

/* One search tile of a layout as a called (not inlined) function: each
   layout's register allocation stays its own and the persistent kernel
   compiles in a fraction of the time an inlined body of every layout takes. */
template <int TB, int TA>
__device__ __noinline__ void batch_tile(const uint8_t* __restrict__ cur,
                                        const uint8_t* __restrict__ prev, int pitch,
                                        const DGeom& g, const vsbd_item* items,
                                        unsigned long long* keys, unsigned* tickets,
                                        vsbd_result* res, int item, int tile, unsigned ntiles,
                                        uint8_t* sm) {
  lattice_tile<TB, false, TA>(cur, prev, pitch, g, items, keys, tickets, res, item, tile, ntiles,
                              sm);
}

/* The proposal's bodies as called functions (their registers stay their
   own, as with the search tiles). */
/* tensor memory of a stage-A CTA, allocated at its first network item and
   released when the CTA leaves the work list */
struct BTmem {
  uint64_t mbar;
  uint32_t taddr, phase;
  int on;
};

__device__ __noinline__ void batch_infer(uint8_t* sm, const BStream& S, const vsbd_item* items,
                                         int chunk, int staged, BTmem* tm, unsigned* err) {
  if (!tm->on) {
    if (threadIdx.x == 0) {
      tc_mbar_init(&tm->mbar);
      tm->phase = 0;
    }
    tc_alloc(&tm->taddr);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) tm->on = 1;
  }
  if (!staged) pn_tc_stage(sm, S.pn);
  const int i0 = chunk * VSB_PN_CHUNK;
  const int i1 = min(S.nc, i0 + VSB_PN_CHUNK);
  __syncthreads();
  pn_tc_items(sm, tm->taddr, tc_saddr(&tm->mbar), &tm->phase, S.cur, S.prev, S.pitch, S.W, S.H,
              items, NULL, i0, i1, 1, S.pout, err);
}

__device__ __noinline__ void batch_prior(uint8_t* sm, const BStream& S) {
  pn_prior_body((float*)sm, S.citems, S.pout, S.nc, S.psc.scale, S.psc.conf_min, S.skip,
                (float)(S.W / 2), (float)(S.H / 2), S.citems2, S.prior);
}

__device__ __noinline__ void batch_narrow(uint8_t* sm, const BStream& S, const DGeom& g,
                                          const vsbd_item* items, const float* pout,
                                          const short2* prior, const PNSearch& ps,
                                          const uint8_t* skip, vsbd_result* res, uint8_t* fb,
                                          unsigned* fbn, int* fbl, int item) {
  pn_narrow_item<1>(sm, S.cur, S.prev, S.pitch, g, items, pout, prior, ps, skip, res, fb, (int*)fbn,
                 fbl, item);
}

/* The dense search of one fine field by the CTA (k_fine's body, one
   lattice row per thread, no strips). */
__device__ __noinline__ void batch_fine(uint8_t* sm, const BStream& S, const DGeom& g,
                                        const vsbd_item* items, int item) {
  if (g.S == 16) fine_item<16, 1>(sm, S.cur, S.prev, S.pitch, g, items, S.fres, 1, item);
  else if (g.S == 32) fine_item<32, 1>(sm, S.cur, S.prev, S.pitch, g, items, S.fres, 1, item);
  else fine_item<48, 1>(sm, S.cur, S.prev, S.pitch, g, items, S.fres, 1, item);
}

__device__ __forceinline__ void search_tile(const BStream& S, const DGeom* geoms, int cls,
                                            const vsbd_item* items, unsigned long long* keys,
                                            unsigned* tickets, vsbd_result* res, int item,
                                            int tile, DGeom* sg, uint8_t* sm) {
  if (threadIdx.x == 0) *sg = geoms[cls];
  __syncthreads();
  const DGeom& g = *sg;
  const unsigned ntiles = (unsigned)(g.nta * g.ntb);
#define VSB_TILE(TBv, TAv) \
  batch_tile<TBv, TAv>(S.cur, S.prev, S.pitch, g, items, keys, tickets, res, item, tile, ntiles, sm)
  const int ta = g.ta > 0 ? g.ta : 1;
  if (g.tb == 4) {
    if (ta == 4) VSB_TILE(4, 4);
    else if (ta == 3) VSB_TILE(4, 3);
    else if (ta == 2) VSB_TILE(4, 2);
    else VSB_TILE(4, 1);
  } else {
    if (ta == 4) VSB_TILE(2, 4);
    else if (ta == 3) VSB_TILE(2, 3);
    else if (ta == 2) VSB_TILE(2, 2);
    else VSB_TILE(2, 1);
  }
#undef VSB_TILE
}

/* Stage A: the static work list `work`.  Stage B (work == NULL): item w of
   the fine search is found from the per-stream prefix sums (tile-granular;
   with a proposal, one narrowed search per fine item) and item offsets into
   the packed fine work list.  With a proposal (ctl->nnarrow > 0) the CTAs
   that find the list empty wait until every narrowed search of the launch
   is done, then share the dense search tiles of the items that fell back. */
template <int NT>
__global__ void __launch_bounds__(NT, VSB_BATCH_THREADS / NT) k_batch_t(const BWork* __restrict__ work,
                                                             const BStream* __restrict__ streams,
                                                             const DGeom* __restrict__ geoms,
                                                             BCtl* ctl, const int* __restrict__ prefix,
                                                             const int* __restrict__ item_off,
                                                             const vsbd_item* __restrict__ fitems,
                                                             int nstreams) {
  extern __shared__ __align__(16) uint8_t sm[];
  __shared__ int s_w;
  __shared__ int s_wres; /* the network's weights are staged in sm */
  __shared__ DGeom sg;
  __shared__ BTmem s_tm;
  const int nwork = ctl->nwork;
  if (threadIdx.x == 0) {
    s_wres = 0;
    s_tm.on = 0;
  }
  for (;;) {
    if (threadIdx.x == 0) s_w = (int)atomicAdd(&ctl->head, 1u);
    __syncthreads();
    const int w = s_w;
    if (w >= nwork) break;
    int keep_w = 0;
    if (work) {
      const BWork it = work[w];
      const BStream& S = streams[it.stream];
      unsigned* done = NULL; /* progress counter this item advances */
      if (it.type == 0) {
        if (S.half <= BTF_MAXHALF)
          blur_tile_fast(S.src, S.sp, S.cur, S.pitch, S.W, S.H, S.half, S.dv, it.a % S.ntx,
                         it.a / S.ntx, sm);
        else
          blur_tile(S.src, S.sp, S.cur, S.pitch, S.W, S.H, S.half, S.dv, it.a % S.ntx,
                    it.a / S.ntx, sm);
        done = &ctl->blur_done[it.stream];
      } else {
        const int ok = wait_blur(ctl, it.stream, (unsigned)(S.ntx * S.nty));
        const unsigned ngroups = (unsigned)((S.nc + S.nf + VSB_MM_GROUP - 1) / VSB_MM_GROUP);
        if (it.type == 1) {
          /* fields a*MM_GROUP .. +MM_GROUP, one warp each; with a proposal
             also the coarse contrast flags (src/motiondetect.c:389-407 of
             the reference: contrast = (max - min) / (max + min + 0.1)) */
          const int f = it.a * VSB_MM_GROUP + (int)(threadIdx.x >> 5);
          if (ok && (int)(threadIdx.x >> 5) < VSB_MM_GROUP && f < S.nc + S.nf) {
            const bool coarse = f < S.nc;
            const int x = coarse ? S.xy[f] : S.xy[2 * S.nc + (f - S.nc)];
            const int y = coarse ? S.xy[S.nc + f] : S.xy[2 * S.nc + S.nf + (f - S.nc)];
            minmax_field_warp(S.cur, S.pitch, x, y, coarse ? S.Sc : S.Sf, f, S.mm);
            if (coarse && S.skip && (threadIdx.x & 31) == 0) {
              const int mn = S.mm[2 * f], mx = S.mm[2 * f + 1];
              const double con = (double)(mx - mn) / ((double)(mx + mn) + 0.1);
              S.skip[f] = !(con >= S.thr && con > 0.0);
            }
          }
          done = &ctl->mm_done[it.stream];
        } else if (it.type == 2) {
          if (ok) {
            const DGeom* gp = &geoms[S.gc];
            const int ntiles = gp->nta * gp->ntb;
            search_tile(S, geoms, S.gc, S.citems, S.keys, S.tickets, S.cres, it.a / ntiles,
                        it.a % ntiles, &sg, sm);
          }
        } else if constexpr (NT == VSB_BATCH_THREADS) {
          /* the proposal's items: every counter they wait for is advanced by
             items earlier in the list (even when those gave up), so the
             waits end */
          const int s = it.stream;
          if (it.type == 3 || it.type == 5) {
            const int ready = ok && (it.type == 3 || wait_ge(ctl, &ctl->prior_done[s], 1u));
            if (ready) {
              batch_infer(sm, S, it.type == 3 ? S.citems : S.citems2, it.a, s_wres, &s_tm,
                          &ctl->err);
              keep_w = 1;
            }
            done = it.type == 3 ? &ctl->inf_done[s] : &ctl->inf2_done[s];
          } else if (it.type == 4) {
            if (ok && wait_ge(ctl, &ctl->mm_done[s], ngroups) &&
                wait_ge(ctl, &ctl->inf_done[s], (unsigned)S.nchunk))
              batch_prior(sm, S);
            done = &ctl->prior_done[s];
          } else if (it.type == 6) {
            unsigned* net = S.passes == 2 ? &ctl->inf2_done[s] : &ctl->inf_done[s];
            if (ok && wait_ge(ctl, &ctl->mm_done[s], ngroups) &&
                wait_ge(ctl, net, (unsigned)S.nchunk)) {
              if (threadIdx.x == 0) sg = geoms[S.gc];
              __syncthreads();
              batch_narrow(sm, S, sg, S.citems, S.pout, S.passes == 2 ? S.prior : NULL, S.psc,
                           S.skip, S.cres, S.cfb, &ctl->fbn[s], S.cfl, it.a);
            }
            done = &ctl->narrow_done;
          }
        }
      }
      if (done) signal_done(done);
    } else {
      /* stream of item w: largest s with prefix[s] <= w */
      int lo = 0, hi = nstreams - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= w) lo = mid; else hi = mid - 1;
      }
      const BStream& S = streams[lo];
      const int local = w - prefix[lo];
      if (S.fnarrow) {
        if (threadIdx.x == 0) sg = geoms[S.gf];
        __syncthreads();
        batch_narrow(sm, S, sg, fitems + item_off[lo], NULL, NULL, S.psf, NULL, S.fres, S.ffb,
                     &ctl->fbn[lo], S.ffl, local);
        signal_done(&ctl->narrow_done);
      } else if (S.ffine) {
        if (threadIdx.x == 0) sg = geoms[S.gf];
        __syncthreads();
        batch_fine(sm, S, sg, fitems + item_off[lo], local);
      } else {
        const DGeom* gp = &geoms[S.gf];
        const int ntiles = gp->nta * gp->ntb;
        search_tile(S, geoms, S.gf, fitems + item_off[lo], S.keys + S.nc, S.tickets + S.nc,
                    S.fres, local / ntiles, local % ntiles, &sg, sm);
      }
    }
    if (threadIdx.x == 0) s_wres = keep_w;
    __syncthreads();
  }
  if (s_tm.on) {
    tc_fence_before();
    __syncthreads();
    tc_dealloc(s_tm.taddr);
  }
  /* the dense search of the items whose proposal was not trusted: tile f of
     the concatenation, stream by stream, of (fallback item x search tile) */
  const int nnarrow = ctl->nnarrow;
  if (nnarrow <= 0 || !wait_ge(ctl, &ctl->narrow_done, (unsigned)nnarrow)) return;
  __shared__ int s_fs, s_fi, s_ft;
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned f = atomicAdd(&ctl->fb_head, 1u);
      int fs = -1, fi = 0, ft = 0;
      unsigned acc = 0;
      for (int q = 0; q < nstreams; q++) {
        const DGeom* gp = &geoms[work ? streams[q].gc : streams[q].gf];
        const unsigned nt = (unsigned)(gp->nta * gp->ntb);
        const unsigned c = *(volatile const unsigned*)&ctl->fbn[q] * nt;
        if (f < acc + c) {
          fs = q;
          fi = (int)((f - acc) / nt);
          ft = (int)((f - acc) % nt);
          break;
        }
        acc += c;
      }
      s_fs = fs;
      s_fi = fi;
      s_ft = ft;
    }
    __syncthreads();
    const int fs = s_fs;
    if (fs < 0) break;
    const BStream& S = streams[fs];
    if (work)
      search_tile(S, geoms, S.gc, S.citems, S.keys, S.tickets, S.cres, __ldcg(S.cfl + s_fi), s_ft,
                  &sg, sm);
    else
      search_tile(S, geoms, S.gf, fitems + item_off[fs], S.keys + S.nc, S.tickets + S.nc, S.fres,
                  __ldcg(S.ffl + s_fi), s_ft, &sg, sm);
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* host side                                                                 */
/* ------------------------------------------------------------------------ */

struct vsbd_batch {
  int dev, n, ncls;
  cudaStream_t st;
  /* geometry classes */
  GeomDev cls[VSB_BATCH_MAX_CLASSES];
  vsbd_geom cls_key[VSB_BATCH_MAX_CLASSES]; /* order: owned copy */
  int cls_items[VSB_BATCH_MAX_CLASSES];     /* search items of the class per step */
  float cls_us[VSB_BATCH_MAX_CLASSES];      /* tuned time of those items alone */
  size_t static_smem;                       /* of the kernel (larger of both block sizes) */
  int cls_nt[VSB_BATCH_MAX_CLASSES];        /* block size a class's tiling must fit */
  size_t smem_b;                            /* stage B: dynamic shared memory, grid */
  int grid_b;
  int optin;                                /* per-block shared memory limit */
  size_t nkeys;
  DGeom* d_geoms;
  /* streams */
  BStream* h_streams; /* pinned; stage A's descriptors */
  BStream* d_streams;
  BStream* h_streamsB; /* stage B's descriptors (a step's planes while stage A of
                          the next step runs) */
  BStream* d_streamsB;
  cudaStream_t st2;    /* stage B */
  cudaEvent_t evA, evB;
  uint8_t** raw;      /* per stream: raw upload buffer (host input) */
  uint8_t** buf[3];   /* per stream: blurred planes (current, previous, next) */
  int* cur;           /* per stream: slot of the current frame */
  int* prv;           /* per stream: slot of the previous frame */
  int16_t** d_xy;
  vsbd_item** d_citems;
  unsigned long long* d_keys;
  unsigned* d_tickets;
  size_t* key_off;    /* per stream: offset of its keys/tickets */
  /* results */
  uint8_t* d_resA;
  uint8_t* h_resA;
  uint8_t* h_resA2;   /* second stage-A result buffer (gA2 copies into it) */
  size_t resA_bytes;
  size_t* mm_off;
  size_t* cres_off;
  vsbd_result* d_resB;
  vsbd_result* h_resB;
  size_t* fres_off;   /* in results */
  int nf_total;
  /* stage A */
  BWork* d_workA;
  int nworkA;
  BCtl* d_ctlA;
  /* stage B */
  BCtl* d_ctlB;
  int* d_pre; /* prefix[n+1], item_off[n] */
  int* h_pre;
  vsbd_item* d_fitems;
  vsbd_item* h_fitems;
  int* h_nwork;
  /* persistent grid */
  size_t smem;
  int grid;
  cudaGraphExec_t gA, gB;
  cudaGraphExec_t gA2; /* stage A with its results copied to h_resA2 (error flag h_nwork[3]) */
  BStream* h_desc[2]; /* pinned per-buffer copies of h_streams, the source of each
                         stage A's descriptor upload */
  cudaEvent_t evA2;   /* end of a stage A of buffer 1 */
  int a_buf;          /* result buffer of the stage A issued last (0: h_resA) */
  int res_buf;        /* result buffer of the stage A collected last */
  int a_fifo[2], a_n; /* buffers of the stage As in flight, oldest first */
  int b_pending;      /* a stage B was issued and not collected */
  long launches;
  long steps;
  unsigned wait_spins;  /* limits of the bounded waits (BCtl) */
  long long wait_cycles;
  int withheld;         /* stream whose blur items stage A's list leaves out (test hook; -1) */
  /* learned search proposal (vsbd_batch_set_proposal) */
  int pn_on;
  void* d_pn;           /* network parameters */
  uint8_t* d_pnbuf;     /* every stream's proposal buffers, one allocation */
  unsigned* h_fbnB;     /* pinned: stage B's fallback count per stream */
  size_t* cfb_off;      /* per stream: coarse fallback flags in the stage-A results */
  int nnarrowA;         /* narrowed searches of a stage A (every coarse field) */
};

/* a control block as the host uploads it: zero counters, the work count and
   the wait limits */
static BCtl ctl_init(const vsbd_batch* b, int nwork, int nnarrow = 0) {
  BCtl h;
  memset(&h, 0, sizeof(h));
  h.nwork = nwork;
  h.nnarrow = nnarrow;
  h.spin_limit = b->wait_spins;
  h.cycle_limit = b->wait_cycles;
  return h;
}

#define BCK(call)                             \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) {                  \
      vsbp_set_err(#call, e_);                \
      return -1;                              \
    }                                         \
  } while (0)

static size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

static int same_geom(const vsbd_geom* a, const vsbd_geom* b) {
  if (a->size != b->size || a->bpp != b->bpp || a->step != b->step || a->na != b->na ||
      a->nb != b->nb || a->ax0 != b->ax0 || a->by0 != b->by0 || a->has_origin != b->has_origin ||
      a->nstages != b->nstages || a->limx != b->limx || a->limy != b->limy)
    return 0;
  for (int k = 0; k < a->nstages; k++)
    if (a->st_r[k] != b->st_r[k] || a->st_h[k] != b->st_h[k]) return 0;
  return memcmp(a->order, b->order, sizeof(int32_t) * (size_t)a->na * a->nb) == 0;
}

/* a tiling the persistent kernel can run: TB 2 or 4, one or two columns
   per thread, at most its block size, tile and static shared memory within
   the per-block limit */
static int tiling_ok(const vsbd_batch* b, const DGeom& g, int nt = VSB_BATCH_THREADS) {
  return (g.tb == 2 || g.tb == 4) && g.threads <= nt &&
         tile_layout(g).total + b->static_smem + 64 <= (size_t)b->optin;
}

/* the model's best tiling of class k that fits blocks of nt threads */
static int default_tiling(vsbd_batch* b, int k, int nitems, int nt) {
  TileCand cand[16];
  int nc = vsbp_tile_candidates(b->cls[k].g, nitems, nt, cand, 16);
  for (int i = 0; i < nc; i++)
    if (tiling_ok(b, cand[i].g, nt)) {
      DGeom t = cand[i].g;
      t.order = b->cls[k].g.order;
      t.point = b->cls[k].g.point;
      b->cls[k].g = t;
      b->cls[k].smem = tile_layout(t).total;
      return 0;
    }
  vsbp_set_msg("no search tiling of the batched kernel fits in shared memory");
  return -1;
}

static int class_of(vsbd_batch* b, const vsbd_geom* g, int nitems) {
  for (int k = 0; k < b->ncls; k++)
    if (same_geom(&b->cls_key[k], g)) return k;
  if (b->ncls >= VSB_BATCH_MAX_CLASSES) {
    vsbp_set_msg("too many distinct field geometries in one batch");
    return -1;
  }
  int k = b->ncls;
  if (vsbp_geom_upload(g, nitems, &b->cls[k]) != 0) return -1;
  size_t no = sizeof(int32_t) * (size_t)g->na * g->nb;
  int32_t* own = (int32_t*)malloc(no);
  if (!own) { vsbp_set_msg("out of host memory"); vsbp_geom_free(&b->cls[k]); return -1; }
  memcpy(own, g->order, no);
  b->cls_key[k] = *g;
  b->cls_key[k].order = own;
  b->ncls++;
  b->cls_nt[k] = VSB_BATCH_THREADS;
  /* the default tiling: the model's best that the persistent kernel runs */
  return default_tiling(b, k, nitems, VSB_BATCH_THREADS) == 0 ? k : -1;
}

/* shared memory of the narrowed search of class k's fields at radius r */
static size_t narrow_smem(const vsbd_batch* b, int k, float r) {
  return narrow_layout(b->cls[k].g, r).total;
}

static size_t kernel_smem(const vsbd_batch* b) {
  size_t m = BT_SMEM > BTF_SMEM ? BT_SMEM : BTF_SMEM;
  for (int k = 0; k < b->ncls; k++) {
    size_t t = tile_layout(b->cls[k].g).total;
    if (t > m) m = t;
  }
  if (b->pn_on) {
    /* the network, the prior's arrays, the coarse narrowed searches */
    if ((size_t)TC_SMEM > m) m = TC_SMEM;
    if (sizeof(float) * 4 * PN_PRIOR_MAX > m) m = sizeof(float) * 4 * PN_PRIOR_MAX;
    for (int s = 0; s < b->n; s++) {
      const size_t t = narrow_smem(b, b->h_streams[s].gc, b->h_streams[s].psc.radius);
      if (t > m) m = t;
    }
  }
  return m;
}

static int set_grid(vsbd_batch* b) {
  b->smem = kernel_smem(b);
  BCK(cudaFuncSetAttribute(k_batch_t<VSB_BATCH_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)b->smem));
  int per = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_t<VSB_BATCH_THREADS>,
                                                    VSB_BATCH_THREADS, b->smem));
  if (per < 1) {
    vsbp_set_msg("the batched kernel does not fit on an SM");
    return -1;
  }
  b->grid = per * vsbp_sm_count();
  return 0;
}

/* stage B's grid: shared memory of the classes that serve fine fields */
static int set_grid_b(vsbd_batch* b) {
  size_t m = 16;
  for (int k = 0; k < b->ncls; k++)
    if (b->cls_nt[k] == VSB_BATCH_THREADS_B && tile_layout(b->cls[k].g).total > m)
      m = tile_layout(b->cls[k].g).total;
  for (int s = 0; s < b->n; s++)
    if (b->h_streams[s].ffine) {
      const size_t t = fw_layout(b->cls[b->h_streams[s].gf].g, VSB_BATCH_THREADS_B, 1, 1).total;
      if (t > m) m = t;
    }
  if (b->pn_on)
    for (int s = 0; s < b->n; s++) {
      if (!b->h_streams[s].fnarrow) continue;
      const size_t t = narrow_smem(b, b->h_streams[s].gf, b->h_streams[s].psf.radius);
      if (t > m) m = t;
    }
  b->smem_b = m;
  BCK(cudaFuncSetAttribute(k_batch_t<VSB_BATCH_THREADS_B>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem_b));
  int per = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_t<VSB_BATCH_THREADS_B>,
                                                    VSB_BATCH_THREADS_B, b->smem_b));
  if (per < 1) {
    vsbp_set_msg("the batched fine-search kernel does not fit on an SM");
    return -1;
  }
  b->grid_b = per * vsbp_sm_count();
  return 0;
}

static int upload_geoms(vsbd_batch* b) {
  DGeom h[VSB_BATCH_MAX_CLASSES];
  for (int k = 0; k < b->ncls; k++) h[k] = b->cls[k].g;
  BCK(cudaMemcpy(b->d_geoms, h, sizeof(DGeom) * b->ncls, cudaMemcpyHostToDevice));
  return 0;
}

/* stage-A work list: blur tiles, coarse search tiles (heaviest classes
   first), min/max of every field */
/* stage-A work list of a batch with a search proposal: blur tiles, min/max
   groups, the first network pass, the priors and second pass of the
   streams that take two, then one narrowed search per coarse field */
static int build_workA_learned(vsbd_batch* b, BWork** out, int* count) {
  long total = 0;
  for (int s = 0; s < b->n; s++) {
    const BStream& S = b->h_streams[s];
    total += (long)S.ntx * S.nty + (S.nc + S.nf + VSB_MM_GROUP - 1) / VSB_MM_GROUP;
    total += (long)S.nchunk * S.passes + (S.passes == 2) + S.nc;
  }
  BWork* w = (BWork*)malloc(sizeof(BWork) * (size_t)(total + 1));
  if (!w) { vsbp_set_msg("out of host memory"); return -1; }
  long k = 0;
  for (int s = 0; s < b->n; s++)
    for (int t = 0; t < b->h_streams[s].ntx * b->h_streams[s].nty; t++) w[k++] = { 0, s, t, 0 };
  for (int s = 0; s < b->n; s++)
    for (int g = 0; g * VSB_MM_GROUP < b->h_streams[s].nc + b->h_streams[s].nf; g++)
      w[k++] = { 1, s, g, 0 };
  for (int s = 0; s < b->n; s++)
    for (int c = 0; c < b->h_streams[s].nchunk; c++) w[k++] = { 3, s, c, 0 };
  for (int s = 0; s < b->n; s++)
    if (b->h_streams[s].passes == 2) w[k++] = { 4, s, 0, 0 };
  for (int s = 0; s < b->n; s++)
    if (b->h_streams[s].passes == 2)
      for (int c = 0; c < b->h_streams[s].nchunk; c++) w[k++] = { 5, s, c, 0 };
  for (int s = 0; s < b->n; s++)
    for (int i = 0; i < b->h_streams[s].nc; i++) w[k++] = { 6, s, i, 0 };
  *out = w;
  *count = (int)k;
  return 0;
}

static int build_workA(vsbd_batch* b, BWork** out, int* count, int only_cls, int fine_cls_tune) {
  if (b->pn_on && only_cls < 0) return build_workA_learned(b, out, count);
  long total = 0;
  for (int s = 0; s < b->n; s++) {
    const BStream& S = b->h_streams[s];
    if (only_cls < 0) total += (long)S.ntx * S.nty + S.nc + S.nf;
    const int cg = fine_cls_tune ? S.gf : S.gc;
    const int ni = fine_cls_tune ? S.nf : S.nc;
    if (only_cls < 0 || cg == only_cls)
      total += (long)ni * b->cls[cg].g.nta * b->cls[cg].g.ntb;
  }
  BWork* w = (BWork*)malloc(sizeof(BWork) * (size_t)(total + 1));
  if (!w) { vsbp_set_msg("out of host memory"); return -1; }
  long k = 0;
  if (only_cls < 0)
    for (int s = 0; s < b->n; s++)
      for (int t = 0; t < b->h_streams[s].ntx * b->h_streams[s].nty; t++) w[k++] = { 0, s, t, 0 };
  /* search items, by class cost (descending) */
  int order[VSB_BATCH_MAX_CLASSES];
  for (int c = 0; c < b->ncls; c++) order[c] = c;
  for (int i = 1; i < b->ncls; i++)
    for (int j = i; j > 0; j--) {
      const DGeom& x = b->cls[order[j]].g;
      const DGeom& y = b->cls[order[j - 1]].g;
      double cx = (double)x.S * x.S * x.na * x.nb, cy = (double)y.S * y.S * y.na * y.nb;
      if (cx > cy) { int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t; }
    }
  for (int oc = 0; oc < b->ncls; oc++) {
    const int c = order[oc];
    if (only_cls >= 0 && c != only_cls) continue;
    for (int s = 0; s < b->n; s++) {
      const BStream& S = b->h_streams[s];
      const int cg = fine_cls_tune ? S.gf : S.gc;
      if (cg != c) continue;
      const int ni = fine_cls_tune ? S.nf : S.nc;
      const int nt = b->cls[c].g.nta * b->cls[c].g.ntb;
      for (int i = 0; i < ni; i++)
        for (int t = 0; t < nt; t++) w[k++] = { 2, s, i * nt + t, 0 };
    }
  }
  if (only_cls < 0)
    for (int s = 0; s < b->n; s++)
      for (int g = 0; g * VSB_MM_GROUP < b->h_streams[s].nc + b->h_streams[s].nf; g++)
        w[k++] = { 1, s, g, 0 };
  *out = w;
  *count = (int)k;
  return 0;
}

static int launch_k(vsbd_batch* b, const BWork* work, BCtl* ctl, cudaStream_t st, int nt) {
  if (nt == VSB_BATCH_THREADS_B)
    k_batch_t<VSB_BATCH_THREADS_B><<<b->grid_b, VSB_BATCH_THREADS_B, b->smem_b, st>>>(
        work, b->d_streams, b->d_geoms, ctl, b->d_pre, b->d_pre + b->n + 1, b->d_fitems, b->n);
  else
    k_batch_t<VSB_BATCH_THREADS><<<b->grid, VSB_BATCH_THREADS, b->smem, st>>>(
        work, b->d_streams, b->d_geoms, ctl, b->d_pre, b->d_pre + b->n + 1, b->d_fitems, b->n);
  BCK(cudaGetLastError());
  return 0;
}

/* Times the model's best tilings of one class inside the persistent kernel
   (the class's search items alone, all streams of the class, zero offsets)
   and keeps the fastest. */
static int autotune_class(vsbd_batch* b, int c, int is_fine) {
  int nitems = 0;
  for (int s = 0; s < b->n; s++) {
    const BStream& S = b->h_streams[s];
    if ((is_fine ? S.gf : S.gc) == c) nitems += is_fine ? S.nf : S.nc;
  }
  if (nitems == 0 || getenv("VSB_NO_AUTOTUNE")) return 0;
  /* all four layouts (one lattice column per thread; two with shifts; two
     from aligned window copies; two from one copy and a shifted field copy):
     the cost model does not see the shared-memory loads and shifts in which
     they differ */
  /* fine classes run in stage B's 256-thread blocks and are timed there */
  const int nt = b->cls_nt[c];
  const int kernel_nt = is_fine ? VSB_BATCH_THREADS_B : VSB_BATCH_THREADS;
  TileCand cand[24];
  int nc = vsbp_tile_candidates_ta(b->cls[c].g, nitems, nt, cand, 5, 1);
  nc += vsbp_tile_candidates_ta(b->cls[c].g, nitems, nt, cand + nc, 5, 2);
  nc += vsbp_tile_candidates_ta(b->cls[c].g, nitems, nt, cand + nc, 6, 3);
  nc += vsbp_tile_candidates_ta(b->cls[c].g, nitems, nt, cand + nc, 6, 4);
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  DGeom best = b->cls[c].g;
  int tried = 0;
  for (int k = 0; k < nc && tried < 18; k++) {
    if (!tiling_ok(b, cand[k].g, nt)) continue;
    tried++;
    DGeom t = cand[k].g;
    t.order = b->cls[c].g.order;
    t.point = b->cls[c].g.point;
    DGeom keep = b->cls[c].g;
    b->cls[c].g = t;
    BWork* w = NULL;
    int nw = 0;
    if ((kernel_nt == VSB_BATCH_THREADS_B ? set_grid_b(b) : set_grid(b)) != 0 ||
        upload_geoms(b) != 0 || build_workA(b, &w, &nw, c, is_fine) != 0) {
      b->cls[c].g = keep;
      free(w);
      continue;
    }
    BWork* d_w = NULL;
    cudaError_t e = cudaMalloc(&d_w, sizeof(BWork) * (size_t)(nw + 1));
    if (e == cudaSuccess) e = cudaMemcpy(d_w, w, sizeof(BWork) * nw, cudaMemcpyHostToDevice);
    free(w);
    if (e != cudaSuccess) { cudaFree(d_w); b->cls[c].g = keep; vsbp_set_err("tuning buffers", e); return -1; }
    float ms = 0.f;
    int ok = 1;
    for (int rep = 0; rep < 4 && ok; rep++) {
      /* the tuning list has no blur items: mark every stream's blur done */
      BCtl h = ctl_init(b, 0);
      for (int s = 0; s < b->n; s++)
        h.blur_done[s] = (unsigned)(b->h_streams[s].ntx * b->h_streams[s].nty);
      h.nwork = nw;
      if (cudaMemcpyAsync(b->d_ctlA, &h, sizeof(h), cudaMemcpyHostToDevice, b->st) != cudaSuccess)
        ok = 0;
      if (rep == 1) cudaEventRecord(e0, b->st);
      if (ok && launch_k(b, d_w, b->d_ctlA, b->st, kernel_nt) != 0) ok = 0;
      if (rep == 3) cudaEventRecord(e1, b->st);
      if (cudaStreamSynchronize(b->st) != cudaSuccess) ok = 0;
    }
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    cudaFree(d_w);
    b->cls[c].g = keep;
    if (ok && ms < best_ms) {
      best_ms = ms;
      best = t;
    }
    if (!ok) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BCK(cudaGetLastError());
  b->cls[c].g = best;
  b->cls[c].smem = tile_layout(best).total;
  b->cls_items[c] = nitems;
  b->cls_us[c] = best_ms < 1e29f ? 1000.f * best_ms / 3.f : 0.f;
  return 0;
}

static int capture(vsbd_batch* b, int stageB, uint8_t* h_res, int flag, cudaGraphExec_t* out) {
  cudaGraph_t g = NULL;
  BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  BCtl* ctl = stageB ? b->d_ctlB : b->d_ctlA;
  cudaMemsetAsync(ctl, 0, offsetof(BCtl, nwork), b->st);
  if (stageB)
    k_batch_t<VSB_BATCH_THREADS_B><<<b->grid_b, VSB_BATCH_THREADS_B, b->smem_b, b->st>>>(
        NULL, b->d_streamsB, b->d_geoms, ctl, b->d_pre, b->d_pre + b->n + 1, b->d_fitems, b->n);
  else
    k_batch_t<VSB_BATCH_THREADS><<<b->grid, VSB_BATCH_THREADS, b->smem, b->st>>>(
        b->d_workA, b->d_streams, b->d_geoms, ctl, b->d_pre, b->d_pre + b->n + 1, b->d_fitems,
        b->n);
  if (stageB) {
    cudaMemcpyAsync(b->h_resB, b->d_resB, sizeof(vsbd_result) * (size_t)(b->nf_total + 1),
                    cudaMemcpyDeviceToHost, b->st);
    if (b->pn_on && b->h_streams[0].fnarrow)
      cudaMemcpyAsync(b->h_fbnB, ctl->fbn, sizeof(unsigned) * b->n, cudaMemcpyDeviceToHost, b->st);
  }
  else
    cudaMemcpyAsync(h_res, b->d_resA, b->resA_bytes, cudaMemcpyDeviceToHost, b->st);
  cudaMemcpyAsync((void*)&b->h_nwork[flag], &ctl->err,
                  sizeof(unsigned), cudaMemcpyDeviceToHost, b->st);
  cudaError_t e = cudaStreamEndCapture(b->st, &g);
  if (e != cudaSuccess) { vsbp_set_err("graph capture", e); return -1; }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { vsbp_set_err("graph instantiation", e); return -1; }
  return 0;
}

extern "C" void vsbd_batch_destroy(vsbd_batch* b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->st2) cudaStreamSynchronize(b->st2);
  if (b->gA) cudaGraphExecDestroy(b->gA);
  if (b->gA2) cudaGraphExecDestroy(b->gA2);
  if (b->gB) cudaGraphExecDestroy(b->gB);
  for (int s = 0; s < b->n; s++) {
    if (b->raw) cudaFree(b->raw[s]);
    if (b->buf[0]) cudaFree(b->buf[0][s]);
    if (b->buf[1]) cudaFree(b->buf[1][s]);
    if (b->buf[2]) cudaFree(b->buf[2][s]);
    if (b->d_xy) cudaFree(b->d_xy[s]);
    if (b->d_citems) cudaFree(b->d_citems[s]);
  }
  for (int k = 0; k < b->ncls; k++) {
    vsbp_geom_free(&b->cls[k]);
    free((void*)b->cls_key[k].order);
  }
  cudaFree(b->d_geoms);
  cudaFree(b->d_streams);
  cudaFreeHost(b->h_streams);
  cudaFree(b->d_streamsB);
  cudaFreeHost(b->h_streamsB);
  if (b->evA) cudaEventDestroy(b->evA);
  if (b->evA2) cudaEventDestroy(b->evA2);
  for (int k = 0; k < 2; k++)
    if (b->h_desc[k]) cudaFreeHost(b->h_desc[k]);
  if (b->evB) cudaEventDestroy(b->evB);
  if (b->st2) cudaStreamDestroy(b->st2);
  cudaFree(b->d_keys);
  cudaFree(b->d_tickets);
  cudaFree(b->d_resA);
  cudaFreeHost(b->h_resA);
  if (b->h_resA2) cudaFreeHost(b->h_resA2);
  cudaFree(b->d_resB);
  cudaFreeHost(b->h_resB);
  cudaFree(b->d_workA);
  cudaFree(b->d_ctlA);
  cudaFree(b->d_ctlB);
  cudaFree(b->d_pre);
  cudaFreeHost(b->h_pre);
  cudaFree(b->d_fitems);
  cudaFreeHost(b->h_fitems);
  cudaFreeHost(b->h_nwork);
  cudaFree(b->d_pn);
  cudaFree(b->d_pnbuf);
  if (b->h_fbnB) cudaFreeHost(b->h_fbnB);
  free(b->cfb_off);
  free(b->raw);
  free(b->buf[0]);
  free(b->buf[1]);
  free(b->buf[2]);
  free(b->cur);
  free(b->prv);
  free(b->d_xy);
  free(b->d_citems);
  free(b->key_off);
  free(b->mm_off);
  free(b->cres_off);
  free(b->fres_off);
  if (b->st) cudaStreamDestroy(b->st);
  free(b);
}

extern "C" int vsbd_batch_create(vsbd_batch** out, int n, const vsbd_batch_stream* d) {
  *out = NULL;
  if (n < 1 || n > VSB_BATCH_MAX_STREAMS) {
    vsbp_set_msg("batch size out of range (1..1024 streams)");
    return -1;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    vsbp_set_msg("no CUDA device available (the GPU path has no CPU fallback)");
    return -1;
  }
  vsbd_batch* b = (vsbd_batch*)calloc(1, sizeof(vsbd_batch));
  cudaGetDevice(&b->dev);
  b->n = n;
  {
    cudaFuncAttributes fa, fb;
    if (cudaFuncGetAttributes(&fa, k_batch_t<VSB_BATCH_THREADS>) != cudaSuccess ||
        cudaFuncGetAttributes(&fb, k_batch_t<VSB_BATCH_THREADS_B>) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->dev) !=
            cudaSuccess) {
      vsbp_set_msg("cannot query the batched kernel");
      free(b);
      return -1;
    }
    b->static_smem = fa.sharedSizeBytes > fb.sharedSizeBytes ? fa.sharedSizeBytes
                                                             : fb.sharedSizeBytes;
  }
#define CKB(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { vsbp_set_err(#call, e_); vsbd_batch_destroy(b); return -1; } } while (0)
#define FAILB() do { vsbd_batch_destroy(b); return -1; } while (0)
  CKB(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  CKB(cudaStreamCreateWithFlags(&b->st2, cudaStreamNonBlocking));
  CKB(cudaEventCreateWithFlags(&b->evA, cudaEventDisableTiming));
  CKB(cudaEventCreateWithFlags(&b->evA2, cudaEventDisableTiming));
  CKB(cudaEventCreateWithFlags(&b->evB, cudaEventDisableTiming));
  b->raw = (uint8_t**)calloc(n, sizeof(uint8_t*));
  b->buf[0] = (uint8_t**)calloc(n, sizeof(uint8_t*));
  b->buf[1] = (uint8_t**)calloc(n, sizeof(uint8_t*));
  b->buf[2] = (uint8_t**)calloc(n, sizeof(uint8_t*));
  b->cur = (int*)calloc(n, sizeof(int));
  b->prv = (int*)calloc(n, sizeof(int));
  for (int s = 0; s < n; s++) b->prv[s] = 1;
  b->d_xy = (int16_t**)calloc(n, sizeof(int16_t*));
  b->d_citems = (vsbd_item**)calloc(n, sizeof(vsbd_item*));
  b->key_off = (size_t*)calloc(n, sizeof(size_t));
  b->mm_off = (size_t*)calloc(n, sizeof(size_t));
  b->cres_off = (size_t*)calloc(n, sizeof(size_t));
  b->fres_off = (size_t*)calloc(n, sizeof(size_t));
  b->cfb_off = (size_t*)calloc(n, sizeof(size_t));
  CKB(cudaMallocHost(&b->h_streams, sizeof(BStream) * n));
  memset(b->h_streams, 0, sizeof(BStream) * n);
  CKB(cudaMalloc(&b->d_streams, sizeof(BStream) * n));
  CKB(cudaMallocHost(&b->h_streamsB, sizeof(BStream) * n));
  for (int k = 0; k < 2; k++) CKB(cudaMallocHost(&b->h_desc[k], sizeof(BStream) * n));
  CKB(cudaMalloc(&b->d_streamsB, sizeof(BStream) * n));
  CKB(cudaMalloc(&b->d_geoms, sizeof(DGeom) * VSB_BATCH_MAX_CLASSES));
  size_t nkeys = 0, resA = 0;
  int nf_total = 0;
  for (int s = 0; s < n; s++) {
    const vsbd_batch_stream& q = d[s];
    if (q.blur_size >= 2 && q.blur_size / 2 > BT_MAXHALF) {
      vsbp_set_msg("blur window too wide for the batched kernel");
      FAILB();
    }
    BStream& S = b->h_streams[s];
    S.W = q.width;
    S.H = q.height;
    S.pitch = (int)(((size_t)q.width + 127) & ~(size_t)127);
    S.half = q.blur_size >= 2 ? q.blur_size / 2 : 0;
    make_div(q.blur_size >= 2 ? q.blur_size : 1, S.half, &S.dv);
    if (q.blur_size < 2) { S.dv.mul = 0; S.dv.size = 1; S.dv.exact = 0; }
    /* blur tiles: 256 x 32 with vector access up to half-width 16, else the
       128 x 32 byte tile */
    const int tw = S.half <= BTF_MAXHALF ? BTF_W : BT_W;
    S.ntx = (q.width + tw - 1) / tw;
    S.nty = (q.height + BT_H - 1) / BT_H;
    S.nc = q.nc;
    S.nf = q.nf;
    S.Sc = q.coarse.size;
    S.Sf = q.fine.size;
    if (q.coarse.bpp != 1 || q.fine.bpp != 1) {
      vsbp_set_msg("the batched path takes planar formats only");
      FAILB();
    }
    int gc = class_of(b, &q.coarse, q.nc);
    int gf = gc < 0 ? -1 : class_of(b, &q.fine, q.nf);
    if (gc < 0 || gf < 0) FAILB();
    S.gc = gc;
    S.gf = gf;
    size_t plane = (size_t)S.pitch * q.height + 256;
    CKB(cudaMalloc(&b->raw[s], plane));
    for (int k = 0; k < 3; k++) {
      CKB(cudaMalloc(&b->buf[k][s], plane));
      CKB(cudaMemset(b->buf[k][s], 0, plane));
    }
    CKB(cudaMalloc(&b->d_xy[s], sizeof(int16_t) * 2 * (size_t)(q.nc + q.nf) + 16));
    CKB(cudaMemcpy(b->d_xy[s], q.xy, sizeof(int16_t) * 2 * (size_t)(q.nc + q.nf),
                   cudaMemcpyHostToDevice));
    vsbd_item* it = (vsbd_item*)malloc(sizeof(vsbd_item) * (size_t)(q.nc + 1));
    for (int i = 0; i < q.nc; i++) { it[i].x = q.xy[i]; it[i].y = q.xy[q.nc + i]; it[i].ox = 0; it[i].oy = 0; }
    cudaError_t e3 = cudaMalloc(&b->d_citems[s], sizeof(vsbd_item) * (size_t)(q.nc + 1));
    if (e3 == cudaSuccess)
      e3 = cudaMemcpy(b->d_citems[s], it, sizeof(vsbd_item) * q.nc, cudaMemcpyHostToDevice);
    free(it);
    CKB(e3);
    b->key_off[s] = nkeys;
    nkeys += (size_t)q.nc + q.nf;
    b->mm_off[s] = resA;
    resA = al16(resA + 2 * (size_t)(q.nc + q.nf));
    b->cres_off[s] = resA;
    resA = al16(resA + sizeof(vsbd_result) * (size_t)q.nc);
    b->cfb_off[s] = resA;
    resA = al16(resA + (size_t)q.nc);
    b->fres_off[s] = (size_t)nf_total;
    nf_total += q.nf;
  }
  b->nf_total = nf_total;
  b->nkeys = nkeys;
  b->resA_bytes = resA + 16;
  CKB(cudaMalloc(&b->d_keys, sizeof(unsigned long long) * (nkeys + 1)));
  CKB(cudaMemset(b->d_keys, 0xff, sizeof(unsigned long long) * (nkeys + 1)));
  CKB(cudaMalloc(&b->d_tickets, sizeof(unsigned) * (nkeys + 1)));
  CKB(cudaMemset(b->d_tickets, 0, sizeof(unsigned) * (nkeys + 1)));
  CKB(cudaMalloc(&b->d_resA, b->resA_bytes));
  CKB(cudaMallocHost(&b->h_resA, b->resA_bytes));
  CKB(cudaMallocHost(&b->h_resA2, b->resA_bytes));
  CKB(cudaMalloc(&b->d_resB, sizeof(vsbd_result) * (size_t)(nf_total + 1)));
  CKB(cudaMallocHost(&b->h_resB, sizeof(vsbd_result) * (size_t)(nf_total + 1)));
  CKB(cudaMalloc(&b->d_ctlA, sizeof(BCtl)));
  CKB(cudaMalloc(&b->d_ctlB, sizeof(BCtl)));
  b->wait_spins = VSB_WAIT_SPINS;
  b->wait_cycles = VSB_WAIT_CYCLES;
  b->withheld = -1;
  {
    BCtl h = ctl_init(b, 0);
    CKB(cudaMemcpy(b->d_ctlA, &h, sizeof(h), cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(b->d_ctlB, &h, sizeof(h), cudaMemcpyHostToDevice));
  }
  CKB(cudaMalloc(&b->d_pre, sizeof(int) * (2 * (size_t)n + 2)));
  CKB(cudaMallocHost(&b->h_pre, sizeof(int) * (2 * (size_t)n + 2)));
  CKB(cudaMalloc(&b->d_fitems, sizeof(vsbd_item) * (size_t)(nf_total + 1)));
  CKB(cudaMallocHost(&b->h_fitems, sizeof(vsbd_item) * (size_t)(nf_total + 1)));
  /* [0] stage B's items, [1] its error flag, [2], [3] the error flags of
     the two stage-A graphs, [4], [5] stage B's work count and narrowed
     searches as uploaded */
  CKB(cudaMallocHost(&b->h_nwork, sizeof(int) * 8));
  memset(b->h_nwork, 0, sizeof(int) * 8);
  for (int s = 0; s < n; s++) {
    BStream& S = b->h_streams[s];
    S.src = b->raw[s];
    S.sp = S.pitch;
    S.cur = b->buf[0][s];
    S.prev = b->buf[1][s];
    S.xy = b->d_xy[s];
    S.citems = b->d_citems[s];
    S.keys = b->d_keys + b->key_off[s];
    S.tickets = b->d_tickets + b->key_off[s];
    S.mm = b->d_resA + b->mm_off[s];
    S.cres = (vsbd_result*)(b->d_resA + b->cres_off[s]);
    S.fres = b->d_resB + b->fres_off[s];
    S.cfb = b->d_resA + b->cfb_off[s];
    S.thr = d[s].coarse_thr;
  }
  CKB(cudaMemcpy(b->d_streams, b->h_streams, sizeof(BStream) * n, cudaMemcpyHostToDevice));
  /* fine items for tuning: every fine field of every stream, no offset; the
     stage-B tables of the tuning runs are not used (stage-A lists) */
  for (int s = 0, k = 0; s < n; s++)
    for (int i = 0; i < d[s].nf; i++, k++) {
      b->h_fitems[k].x = d[s].xy[2 * d[s].nc + i];
      b->h_fitems[k].y = d[s].xy[2 * d[s].nc + d[s].nf + i];
      b->h_fitems[k].ox = b->h_fitems[k].oy = 0;
    }
  /* tuning of fine classes runs through the stage-A path with citems
     replaced: point each stream's citems at its fine items for that run */
  /* classes that serve fine fields run in stage B's smaller blocks */
  for (int c = 0; c < b->ncls; c++) {
    int used_f = 0, nitems = 0;
    for (int s = 0; s < n; s++)
      if (b->h_streams[s].gf == c) {
        used_f = 1;
        nitems += b->h_streams[s].nf;
      }
    if (!used_f) continue;
    b->cls_nt[c] = VSB_BATCH_THREADS_B;
    if (b->cls[c].g.threads > VSB_BATCH_THREADS_B &&
        default_tiling(b, c, nitems, VSB_BATCH_THREADS_B) != 0)
      FAILB();
  }
  if (set_grid(b) != 0 || set_grid_b(b) != 0 || upload_geoms(b) != 0) FAILB();
  for (int c = 0; c < b->ncls; c++) {
    int used_c = 0, used_f = 0;
    for (int s = 0; s < n; s++) {
      used_c |= b->h_streams[s].gc == c;
      used_f |= b->h_streams[s].gf == c;
    }
    if (used_c && autotune_class(b, c, 0) != 0) FAILB();
    if (used_f && !used_c) {
      /* fine classes are tuned as a stage-A search over the fine items */
      vsbd_item* tmp = NULL;
      CKB(cudaMalloc(&tmp, sizeof(vsbd_item) * (size_t)(nf_total + 1)));
      cudaError_t e = cudaMemcpy(tmp, b->h_fitems, sizeof(vsbd_item) * nf_total, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) { cudaFree(tmp); CKB(e); }
      BStream* keep = (BStream*)malloc(sizeof(BStream) * n);
      memcpy(keep, b->h_streams, sizeof(BStream) * n);
      for (int s = 0; s < n; s++) {
        BStream& S = b->h_streams[s];
        S.citems = tmp + b->fres_off[s];
        S.cres = S.fres;
        S.keys += S.nc;
        S.tickets += S.nc;
        S.gc = S.gf;
      }
      e = cudaMemcpy(b->d_streams, b->h_streams, sizeof(BStream) * n, cudaMemcpyHostToDevice);
      int rc = e == cudaSuccess ? autotune_class(b, c, 1) : -1;
      memcpy(b->h_streams, keep, sizeof(BStream) * n);
      free(keep);
      cudaMemcpy(b->d_streams, b->h_streams, sizeof(BStream) * n, cudaMemcpyHostToDevice);
      cudaFree(tmp);
      if (e != cudaSuccess) CKB(e);
      if (rc != 0) FAILB();
    }
  }
  /* fine fields of the geometries k_fine takes: one CTA per field in stage
     B (VSB_BATCH_FINE_TILES: the tiles of the tuned tiling instead) */
  for (int s = 0; s < n; s++) {
    BStream& S = b->h_streams[s];
    const DGeom& g = b->cls[S.gf].g;
    S.ffine = !getenv("VSB_BATCH_FINE_TILES") && fw_supported(g) &&
              fw_layout(g, VSB_BATCH_THREADS_B, 1, 1).total + b->static_smem + 64 <=
                  (size_t)b->optin;
  }
  if (set_grid(b) != 0 || set_grid_b(b) != 0 || upload_geoms(b) != 0) FAILB();
  BWork* w = NULL;
  if (build_workA(b, &w, &b->nworkA, -1, 0) != 0) FAILB();
  cudaError_t e = cudaMalloc(&b->d_workA, sizeof(BWork) * (size_t)(b->nworkA + 1));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_workA, w, sizeof(BWork) * b->nworkA, cudaMemcpyHostToDevice);
  free(w);
  CKB(e);
  {
    BCtl h = ctl_init(b, b->nworkA);
    CKB(cudaMemcpy(b->d_ctlA, &h, sizeof(h), cudaMemcpyHostToDevice));
  }
  CKB(cudaStreamSynchronize(b->st));
  if (capture(b, 0, b->h_resA, 2, &b->gA) != 0 || capture(b, 0, b->h_resA2, 3, &b->gA2) != 0 ||
      capture(b, 1, NULL, 1, &b->gB) != 0)
    FAILB();
#undef CKB
#undef FAILB
  *out = b;
  return 0;
}

/* Stage A of a step enqueued on the first stream.  mode 0: every stream's
   frame goes to slot cur, searched against slot prv; 1: the step after the
   current one, into the third slot, against cur; 2: the step after that,
   into slot prv (free once the current step's fine stage is collected),
   against the third slot, which mode 1 filled.  At most two stage As are in
   flight; vsbd_batch_stage_a_collect takes the older. */
extern "C" int vsbd_batch_stage_a_issue(vsbd_batch* b, const uint8_t* const* planes,
                                        const int* pitches, int on_device, int mode) {
  BCK(cudaSetDevice(b->dev));
  if (b->a_n >= 2) {
    vsbp_set_msg("batched stage A: two steps already in flight");
    return -1;
  }
  size_t h2d = 0;
  for (int s = 0; s < b->n; s++) {
    BStream& S = b->h_streams[s];
    if (on_device) {
      S.src = planes[s];
      S.sp = pitches[s];
    } else {
      S.src = b->raw[s];
      S.sp = S.pitch;
      BCK(cudaMemcpy2DAsync(b->raw[s], S.pitch, planes[s], pitches[s], S.W, S.H,
                            cudaMemcpyHostToDevice, b->st));
      h2d += (size_t)S.W * S.H;
    }
    const int third = 3 - b->cur[s] - b->prv[s];
    const int ci = mode == 0 ? b->cur[s] : (mode == 1 ? third : b->prv[s]);
    const int pi = mode == 0 ? b->prv[s] : (mode == 1 ? b->cur[s] : third);
    S.cur = b->buf[ci][s];
    S.prev = b->buf[pi][s];
  }
  /* alternate result buffers (and descriptor copies): the host may still read
     the previous stage A's results while this one runs */
  b->a_buf ^= 1;
  memcpy(b->h_desc[b->a_buf], b->h_streams, sizeof(BStream) * b->n);
  BCK(cudaMemcpyAsync(b->d_streams, b->h_desc[b->a_buf], sizeof(BStream) * b->n,
                      cudaMemcpyHostToDevice, b->st));
  BCK(cudaGraphLaunch(b->a_buf ? b->gA2 : b->gA, b->st));
  BCK(cudaEventRecord(b->a_buf ? b->evA2 : b->evA, b->st));
  b->a_fifo[b->a_n++] = b->a_buf;
  b->launches++;
  vsbp_count(1, h2d + sizeof(BStream) * b->n, b->resA_bytes + 4);
  return 0;
}

extern "C" int vsbd_batch_stage_a_collect(vsbd_batch* b) {
  BCK(cudaSetDevice(b->dev));
  if (b->a_n < 1) {
    vsbp_set_msg("batched stage A: nothing in flight");
    return -1;
  }
  const int buf = b->a_fifo[0];
  b->a_fifo[0] = b->a_fifo[1];
  b->a_n--;
  BCK(cudaEventSynchronize(buf ? b->evA2 : b->evA));
  b->res_buf = buf;
  if (b->h_nwork[buf ? 3 : 2]) {
    vsbp_set_msg("batched stage A: a wait for blur tiles gave up");
    /* skipped tiles leave keys and tickets mid-way: start them afresh */
    cudaStreamSynchronize(b->st);
    b->a_n = 0;
    cudaMemset(b->d_keys, 0xff, sizeof(unsigned long long) * (b->nkeys + 1));
    cudaMemset(b->d_tickets, 0, sizeof(unsigned) * (b->nkeys + 1));
    return -1;
  }
  return 0;
}

extern "C" int vsbd_batch_set_wait_limit(vsbd_batch* b, unsigned spins, long long cycles) {
  BCK(cudaSetDevice(b->dev));
  if (spins < 1 || cycles < 1) {
    vsbp_set_msg("wait limits must be positive");
    return -1;
  }
  BCK(cudaStreamSynchronize(b->st));
  BCK(cudaStreamSynchronize(b->st2));
  b->wait_spins = spins;
  b->wait_cycles = cycles;
  BCtl h = ctl_init(b, 0);
  const size_t off = offsetof(BCtl, spin_limit);
  BCK(cudaMemcpy((uint8_t*)b->d_ctlA + off, (uint8_t*)&h + off, sizeof(BCtl) - off,
                 cudaMemcpyHostToDevice));
  BCK(cudaMemcpy((uint8_t*)b->d_ctlB + off, (uint8_t*)&h + off, sizeof(BCtl) - off,
                 cudaMemcpyHostToDevice));
  return 0;
}

/* Stage A's work list without stream s's blur items (s < 0: the full list):
   the captured graphs read the list and its length from device memory, so
   they run the new list as they are. */
extern "C" int vsbd_batch_withhold_blur(vsbd_batch* b, int stream) {
  BCK(cudaSetDevice(b->dev));
  if (stream >= b->n) {
    vsbp_set_msg("no such stream");
    return -1;
  }
  BCK(cudaStreamSynchronize(b->st));
  BCK(cudaStreamSynchronize(b->st2));
  BWork* w = NULL;
  int nw = 0;
  if (build_workA(b, &w, &nw, -1, 0) != 0) return -1;
  int k = 0;
  for (int i = 0; i < nw; i++)
    if (stream < 0 || !(w[i].type == 0 && w[i].stream == stream)) w[k++] = w[i];
  cudaError_t e = cudaMemcpy(b->d_workA, w, sizeof(BWork) * (size_t)k, cudaMemcpyHostToDevice);
  free(w);
  BCK(e);
  BCK(cudaMemcpy(&b->d_ctlA->nwork, &k, sizeof(int), cudaMemcpyHostToDevice));
  b->withheld = stream;
  return 0;
}

/* waits for every stage A in flight, keeping the last error message */
extern "C" void vsbd_batch_drain(vsbd_batch* b) {
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->st);
  b->a_n = 0;
}

extern "C" int vsbd_batch_stage_a(vsbd_batch* b, const uint8_t* const* planes, const int* pitches,
                                  int on_device) {
  if (vsbd_batch_stage_a_issue(b, planes, pitches, on_device, 0) != 0) return -1;
  return vsbd_batch_stage_a_collect(b);
}

extern "C" void vsbd_batch_results_a(const vsbd_batch* b, int s, const uint8_t** mm,
                                     const vsbd_result** cres) {
  const uint8_t* h = b->res_buf ? b->h_resA2 : b->h_resA;
  *mm = h + b->mm_off[s];
  *cres = (const vsbd_result*)(h + b->cres_off[s]);
}

/* Stage B of the current step enqueued on the second stream, with its own
   descriptors (the current and previous slots of every stream). */
extern "C" int vsbd_batch_stage_b_issue(vsbd_batch* b, const vsbd_item* const* items,
                                        const int* nitems) {
  BCK(cudaSetDevice(b->dev));
  int* pre = b->h_pre;
  int* off = b->h_pre + b->n + 1;
  int total = 0, nit = 0;
  for (int s = 0; s < b->n; s++) {
    const BStream& S = b->h_streams[s];
    const DGeom& g = b->cls[S.gf].g;
    int ni = items && items[s] ? nitems[s] : 0;
    if (ni > S.nf) {
      vsbp_set_msg("more fine items than fine fields");
      return -1;
    }
    pre[s] = total;
    off[s] = nit;
    if (ni > 0) memcpy(b->h_fitems + nit, items[s], sizeof(vsbd_item) * ni);
    nit += ni;
    /* one narrowed search per item with a narrowed fine stage, else the
       item's search tiles */
    total += S.fnarrow || S.ffine ? ni : ni * g.nta * g.ntb;
  }
  pre[b->n] = total;
  b->h_nwork[0] = total;
  b->h_nwork[4] = total;
  b->h_nwork[5] = b->pn_on && b->h_streams[0].fnarrow ? nit : 0;
  b->b_pending = total > 0;
  if (total == 0) return 0;
  for (int s = 0; s < b->n; s++) {
    b->h_streamsB[s] = b->h_streams[s];
    b->h_streamsB[s].cur = b->buf[b->cur[s]][s];
    b->h_streamsB[s].prev = b->buf[b->prv[s]][s];
  }
  BCK(cudaMemcpyAsync(b->d_streamsB, b->h_streamsB, sizeof(BStream) * b->n,
                      cudaMemcpyHostToDevice, b->st2));
  BCK(cudaMemcpyAsync(b->d_pre, b->h_pre, sizeof(int) * (2 * (size_t)b->n + 1),
                      cudaMemcpyHostToDevice, b->st2));
  BCK(cudaMemcpyAsync(b->d_fitems, b->h_fitems, sizeof(vsbd_item) * (size_t)nit,
                      cudaMemcpyHostToDevice, b->st2));
  BCK(cudaMemcpyAsync(&b->d_ctlB->nwork, &b->h_nwork[4], 2 * sizeof(int), cudaMemcpyHostToDevice,
                      b->st2));
  BCK(cudaGraphLaunch(b->gB, b->st2));
  BCK(cudaEventRecord(b->evB, b->st2));
  b->launches++;
  vsbp_count(1, sizeof(BStream) * b->n + sizeof(int) * (2 * (size_t)b->n + 2) +
                    sizeof(vsbd_item) * (size_t)nit,
             sizeof(vsbd_result) * (size_t)(b->nf_total + 1) + 4);
  return 0;
}

extern "C" int vsbd_batch_stage_b_collect(vsbd_batch* b, const vsbd_result** fres) {
  BCK(cudaSetDevice(b->dev));
  for (int s = 0; s < b->n; s++) fres[s] = b->h_resB + b->fres_off[s];
  if (!b->b_pending) return 0;
  BCK(cudaEventSynchronize(b->evB));
  b->b_pending = 0;
  if (b->h_nwork[1]) {
    vsbp_set_msg("batched stage B: the error flag was raised");
    return -1;
  }
  return 0;
}

extern "C" int vsbd_batch_stage_b(vsbd_batch* b, const vsbd_item* const* items, const int* nitems,
                                  const vsbd_result** fres) {
  if (vsbd_batch_stage_b_issue(b, items, nitems) != 0) return -1;
  return vsbd_batch_stage_b_collect(b, fres);
}

/* stream s's current frame becomes its previous one; the third slot takes
   the next frame */
extern "C" void vsbd_batch_commit(vsbd_batch* b, int s) {
  const int f = 3 - b->cur[s] - b->prv[s];
  b->prv[s] = b->cur[s];
  b->cur[s] = f;
}

/* Gives every stream the learned search proposal (params: the network's
   device-order parameters on the host) or, with params == NULL, the dense
   search again.  Rebuilds stage A's work list, the grids and the captured
   graphs; no step may be in flight. */
extern "C" int vsbd_batch_set_proposal(vsbd_batch* b, const void* params, float scale,
                                       float radius, float conf_min, float match_bound,
                                       float fine_radius, const int* passes) {
  BCK(cudaSetDevice(b->dev));
  if (b->a_n > 0 || b->b_pending) {
    vsbp_set_msg("batched proposal: a step is in flight");
    return -1;
  }
  BCK(cudaStreamSynchronize(b->st));
  BCK(cudaStreamSynchronize(b->st2));
  if (params && (!(scale > 0.f) || !(radius >= 0.f) || !(match_bound >= 0.f) ||
                 isnan(fine_radius) || fine_radius > 16.f)) {
    vsbp_set_msg("bad proposal settings");
    return -1;
  }
  if (params)
    for (int s = 0; s < b->n; s++) {
      const BStream& S = b->h_streams[s];
      const DGeom& gc = b->cls[S.gc].g;
      const DGeom& gf = b->cls[S.gf].g;
      const int sc = narrow_span(radius, gc.step);
      const int sf = fine_radius >= 0.f ? narrow_span(fine_radius, gf.step) : 0;
      if (sc * sc > PN_NARROW_QMAX || sf * sf > PN_NARROW_QMAX) {
        vsbp_set_msg("proposal radius too large for the narrowed search");
        return -1;
      }
      if (S.nc > PN_PRIOR_MAX || (passes && passes[s] != 1 && passes[s] != 2)) {
        vsbp_set_msg("batched proposal: more coarse fields than the prior takes, or bad passes");
        return -1;
      }
    }
  /* per stream: pout | citems2 | prior | skip | coarse list | fine list | fine flags */
  size_t* off = (size_t*)malloc(sizeof(size_t) * (size_t)(b->n + 1));
  if (!off) { vsbp_set_msg("out of host memory"); return -1; }
  size_t tot = 0;
  for (int s = 0; s < b->n; s++) {
    const BStream& S = b->h_streams[s];
    off[s] = tot;
    tot += al16(sizeof(float) * 3 * (size_t)S.nc) + al16(sizeof(vsbd_item) * (size_t)S.nc) +
           al16(sizeof(short2) * (size_t)S.nc) + al16((size_t)S.nc) +
           al16(sizeof(int) * (size_t)S.nc) + al16(sizeof(int) * (size_t)S.nf) + al16((size_t)S.nf);
  }
  off[b->n] = tot;
  cudaFree(b->d_pnbuf);
  b->d_pnbuf = NULL;
  b->pn_on = 0;
  if (params) {
    cudaError_t e = cudaSuccess;
    if (!b->d_pn) e = cudaMalloc(&b->d_pn, PN_PARAM_BYTES);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_pn, params, PN_PARAM_BYTES, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_pnbuf, tot + 16);
    if (e == cudaSuccess) e = cudaMemset(b->d_pnbuf, 0, tot + 16);
    if (e == cudaSuccess && !b->h_fbnB) e = cudaMallocHost(&b->h_fbnB, sizeof(unsigned) * b->n);
    if (e != cudaSuccess) {
      free(off);
      vsbp_set_err("batched proposal buffers", e);
      return -1;
    }
    b->nnarrowA = 0;
    for (int s = 0; s < b->n; s++) {
      BStream& S = b->h_streams[s];
      uint8_t* p = b->d_pnbuf + off[s];
      S.pn = b->d_pn;
      S.pout = (float*)p;
      p += al16(sizeof(float) * 3 * (size_t)S.nc);
      S.citems2 = (vsbd_item*)p;
      p += al16(sizeof(vsbd_item) * (size_t)S.nc);
      S.prior = (short2*)p;
      p += al16(sizeof(short2) * (size_t)S.nc);
      S.skip = p;
      p += al16((size_t)S.nc);
      S.cfl = (int*)p;
      p += al16(sizeof(int) * (size_t)S.nc);
      S.ffl = (int*)p;
      p += al16(sizeof(int) * (size_t)S.nf);
      S.ffb = p;
      /* the SAD bound scales with the field's pixel count */
      const double bc = (double)match_bound * b->cls[S.gc].g.S * b->cls[S.gc].g.S;
      const double bf = (double)match_bound * b->cls[S.gf].g.S * b->cls[S.gf].g.S;
      S.psc.scale = S.psf.scale = scale;
      S.psc.conf_min = S.psf.conf_min = conf_min;
      S.psc.radius = radius;
      S.psf.radius = fine_radius;
      S.psc.sad_bound = bc >= 4294967295.0 ? 0xffffffffu : (unsigned)bc;
      S.psf.sad_bound = bf >= 4294967295.0 ? 0xffffffffu : (unsigned)bf;
      S.passes = passes ? passes[s] : 1;
      S.nchunk = (S.nc + VSB_PN_CHUNK - 1) / VSB_PN_CHUNK;
      S.fnarrow = fine_radius >= 0.f;
      b->nnarrowA += S.nc;
    }
    b->pn_on = 1;
  } else {
    for (int s = 0; s < b->n; s++) {
      BStream& S = b->h_streams[s];
      S.pn = NULL;
      S.pout = NULL;
      S.citems2 = NULL;
      S.prior = NULL;
      S.skip = NULL;
      S.cfl = S.ffl = NULL;
      S.ffb = NULL;
      S.passes = 1;
      S.nchunk = 0;
      S.fnarrow = 0;
    }
    b->nnarrowA = 0;
  }
  free(off);
  if (set_grid(b) != 0 || set_grid_b(b) != 0 || upload_geoms(b) != 0) return -1;
  BWork* w = NULL;
  int nw = 0;
  if (build_workA(b, &w, &nw, -1, 0) != 0) return -1;
  cudaFree(b->d_workA);
  b->d_workA = NULL;
  cudaError_t e = cudaMalloc(&b->d_workA, sizeof(BWork) * (size_t)(nw + 1));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_workA, w, sizeof(BWork) * nw, cudaMemcpyHostToDevice);
  free(w);
  BCK(e);
  b->nworkA = nw;
  b->withheld = -1;
  {
    BCtl h = ctl_init(b, nw, b->nnarrowA);
    BCK(cudaMemcpy(b->d_ctlA, &h, sizeof(h), cudaMemcpyHostToDevice));
    BCtl hb = ctl_init(b, 0);
    BCK(cudaMemcpy(b->d_ctlB, &hb, sizeof(hb), cudaMemcpyHostToDevice));
  }
  BCK(cudaMemcpy(b->d_streams, b->h_streams, sizeof(BStream) * b->n, cudaMemcpyHostToDevice));
  if (b->gA) cudaGraphExecDestroy(b->gA);
  if (b->gA2) cudaGraphExecDestroy(b->gA2);
  if (b->gB) cudaGraphExecDestroy(b->gB);
  b->gA = b->gA2 = b->gB = NULL;
  if (capture(b, 0, b->h_resA, 2, &b->gA) != 0 || capture(b, 0, b->h_resA2, 3, &b->gA2) != 0 ||
      capture(b, 1, NULL, 1, &b->gB) != 0)
    return -1;
  return 0;
}

/* proposal counts of stream s's last collected stages: coarse fields
   searched with the proposal and how many of them fell back (from stage
   A's flags), and the fine items that fell back (stage B) */
extern "C" int vsbd_batch_proposal_counts(const vsbd_batch* b, int s, int* coarse_items,
                                          int* coarse_fb, int* fine_fb) {
  if (!b || !b->pn_on || s < 0 || s >= b->n) return -1;
  const uint8_t* fl = (b->res_buf ? b->h_resA2 : b->h_resA) + b->cfb_off[s];
  int ni = 0, nfb = 0;
  for (int i = 0; i < b->h_streams[s].nc; i++) {
    if (fl[i] == PN_FB_UNUSED) continue;
    ni++;
    nfb += fl[i] == PN_FB_FULL;
  }
  if (coarse_items) *coarse_items = ni;
  if (coarse_fb) *coarse_fb = nfb;
  if (fine_fb) *fine_fb = b->h_fbnB && b->h_streams[s].fnarrow ? (int)b->h_fbnB[s] : 0;
  return 0;
}

extern "C" long vsbd_batch_launches(const vsbd_batch* b) { return b ? b->launches : 0; }

extern "C" int vsbd_batch_class(const vsbd_batch* b, int k, int* desc) {
  if (!b) return -1;
  if (k < 0 || k >= b->ncls || !desc) return b->ncls;
  const DGeom& g = b->cls[k].g;
  desc[0] = g.tb;
  desc[1] = g.ta > 0 ? g.ta : 1;
  desc[2] = g.nab;
  desc[3] = g.nbb;
  desc[4] = g.nstrip;
  desc[5] = g.threads;
  desc[6] = (int)tile_layout(g).total;
  desc[7] = g.nta * g.ntb;
  desc[8] = b->cls_items[k];
  desc[9] = (int)(b->cls_us[k] * 1000.f);
  desc[10] = g.S;
  desc[11] = g.na * g.nb;
  return b->ncls;
}

extern "C" int vsbd_batch_grid(const vsbd_batch* b, int* ctas, int* threads, long* smem) {
  if (!b) return -1;
  *ctas = b->grid;
  *threads = VSB_BATCH_THREADS;
  *smem = (long)b->smem;
  return 0;
}
