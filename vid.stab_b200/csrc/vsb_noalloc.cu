/*
 * vsb_noalloc.cu -- the per-field SAD search for callers that cannot
 * allocate GPU memory.
 *
 * Some hosts own every byte of device memory themselves: a decoder or
 * encoder pipeline that hands out frames from a fixed pool, or a process
 * that runs under a memory budget enforced by its own allocator.  A
 * cudaMalloc behind their back would break the pool's accounting or the
 * budget, so they cannot let a library allocate.  This entry point
 * runs the same search kernel as vsMotionDetection's planar path, but all of
 * its scratch memory (per-field running minimum and completion counter, the
 * lattice's visiting-rank tables) lives in one statically sized array that
 * is part of the loaded module.  The caller passes only its own inputs (the
 * two frames, the list of fields) and its output buffer.
 */
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "vsb_device.h"
#include "vsb_search.cuh"

/* sizes of the static scratch: up to VSB_NOALLOC_MAX_ITEMS fields per call and
   lattices of up to VSB_NOALLOC_MAX_LATTICE points (e.g. maxShift/step <= 90).
   In bytes: keys 8 x 4096 + counters 4 x 4096 + rank table 4 x 32768 +
   displacement table 4 x 32769 = 311,300 (304 KiB) */
#define VSB_NOALLOC_MAX_ITEMS 4096
#define VSB_NOALLOC_MAX_LATTICE 32768
#define VSB_NOALLOC_OFF_KEYS 0
#define VSB_NOALLOC_OFF_TICKETS (VSB_NOALLOC_OFF_KEYS + 8 * VSB_NOALLOC_MAX_ITEMS)
#define VSB_NOALLOC_OFF_ORDER (VSB_NOALLOC_OFF_TICKETS + 4 * VSB_NOALLOC_MAX_ITEMS)
#define VSB_NOALLOC_OFF_POINT (VSB_NOALLOC_OFF_ORDER + 4 * VSB_NOALLOC_MAX_LATTICE)
#define VSB_NOALLOC_BYTES (VSB_NOALLOC_OFF_POINT + 4 * (VSB_NOALLOC_MAX_LATTICE + 1))

/* Held by every GPU that loads the library, until the process exits.  In
   host code this name is only a stand-in for the symbol: its device address
   comes from cudaGetSymbolAddress. */
static __device__ __align__(256) uint8_t g_noalloc_scratch[VSB_NOALLOC_BYTES];

static int fail(const char* what, cudaError_t e) {
  char msg[256];
  if (e == cudaSuccess)
    snprintf(msg, sizeof(msg), "%s", what);
  else
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  vsbd_set_error(msg);
  return -1;
}

/* device address of the scratch array, resolved once per device */
#define VSB_NOALLOC_MAX_DEVICES 64
static uint8_t* g_scratch_addr[VSB_NOALLOC_MAX_DEVICES];
static pthread_mutex_t g_scratch_lock = PTHREAD_MUTEX_INITIALIZER;

static uint8_t* scratch_on_current_device(void) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fail("cudaGetDevice", e);
    return NULL;
  }
  if (dev < 0 || dev >= VSB_NOALLOC_MAX_DEVICES) {
    fail("device index beyond the supported range", cudaSuccess);
    return NULL;
  }
  pthread_mutex_lock(&g_scratch_lock);
  uint8_t* p = g_scratch_addr[dev];
  if (!p) {
    void* addr = NULL;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess)
      fail("cudaGetSymbolAddress(g_noalloc_scratch)", e);
    else
      p = g_scratch_addr[dev] = (uint8_t*)addr;
  }
  pthread_mutex_unlock(&g_scratch_lock);
  return p;
}

/* rank of lattice point (a,b), |a|,|b| <= K, in the outgoing spiral of the
   reference (src/motiondetect.c:465-518): ring m = max(|a|,|b|) starts at rank
   (2m-1)^2 with (m, -(m-1)) and runs down the right side, left along the
   bottom, up the left side and right along the top */
__device__ __forceinline__ int spiral_rank(int a, int b) {
  int m = max(abs(a), abs(b));
  if (m == 0) return 0;
  int base = (2 * m - 1) * (2 * m - 1);
  if (a == m && b > -m) return base + b + m - 1;
  if (b == m) return base + 2 * m + (m - 1 - a);
  if (a == -m) return base + 4 * m + (m - 1 - b);
  return base + 6 * m + (a + m - 1);
}

__global__ void k_noalloc_tables(int K, int step, int32_t* order, short2* point) {
  int na = 2 * K + 1, n = na * na;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a = i % na - K, b = i / na - K;
    int r = spiral_rank(a, b);
    order[i] = r;
    point[r] = make_short2((short)(a * step), (short)(b * step));
  }
}

template <int TB, int TA>
static cudaError_t launch_tb(const DGeom& g, size_t smem, const uint8_t* curr, const uint8_t* prev,
                             int pitch, const vsbd_item* items, int n, unsigned long long* keys,
                             unsigned* tickets, vsbd_result* res, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(k_lattice<TB, false, TA>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(g.nta * g.ntb, n);
  k_lattice<TB, false, TA><<<grid, g.threads, smem, st>>>(curr, prev, pitch, g, items, keys,
                                                          tickets, res);
  return cudaGetLastError();
}

extern "C" int vsbd_search_noalloc(const uint8_t* d_curr, const uint8_t* d_prev, int pitch,
                                   int size, int maxShift, int stepSize, const void* d_items,
                                   int n, void* d_results, void* stream) {
  if (n < 0 || n > VSB_NOALLOC_MAX_ITEMS) {
    char msg[128];
    snprintf(msg, sizeof(msg), "%d fields: this entry point takes at most %d per call", n,
             VSB_NOALLOC_MAX_ITEMS);
    return fail(msg, cudaSuccess);
  }
  if (size < 16 || size % 16 || maxShift < 0 || stepSize < 1 || pitch < size || pitch % 16 ||
      ((uintptr_t)d_curr & 15) || ((uintptr_t)d_prev & 15)) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "invalid input: size %d (multiple of 16 needed), maxShift %d, step %d, pitch %d "
             "(multiple of 16 needed), planes 16-byte aligned",
             size, maxShift, stepSize, pitch);
    return fail(msg, cudaSuccess);
  }
  if (maxShift + stepSize > 32767) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "maxShift %d + step %d: shifts must stay within 16 bits (sum at most 32767)",
             maxShift, stepSize);
    return fail(msg, cudaSuccess);
  }
  const int K = maxShift / stepSize;
  const long lattice = (long)(2 * K + 1) * (2 * K + 1);
  if (lattice > VSB_NOALLOC_MAX_LATTICE) {
    char msg[128];
    snprintf(msg, sizeof(msg), "lattice of %ld candidates: this entry point takes at most %d",
             lattice, VSB_NOALLOC_MAX_LATTICE);
    return fail(msg, cudaSuccess);
  }
  if (n == 0) return 0;
  uint8_t* sc = scratch_on_current_device();
  if (!sc) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* keys = (unsigned long long*)(sc + VSB_NOALLOC_OFF_KEYS);
  unsigned* tickets = (unsigned*)(sc + VSB_NOALLOC_OFF_TICKETS);
  int32_t* order = (int32_t*)(sc + VSB_NOALLOC_OFF_ORDER);
  short2* point = (short2*)(sc + VSB_NOALLOC_OFF_POINT);

  /* the geometry of the planar search: spiral lattice, halving refinement */
  vsbd_geom h;
  memset(&h, 0, sizeof(h));
  h.size = size;
  h.bpp = 1;
  h.step = stepSize;
  h.na = h.nb = 2 * K + 1;
  h.ax0 = h.by0 = -K * stepSize;
  int s = stepSize;
  while (s > 1) {
    int hh = s / 2;
    h.st_r[h.nstages] = s - hh;
    h.st_h[h.nstages] = hh;
    h.nstages++;
    s = hh;
  }
  h.limx = maxShift + s - 1;
  h.limy = maxShift + s;
  DGeom g;
  if (vsbd_plan_search(&h, n, &g) != 0) return -1;
  g.order = order;
  g.point = point;
  const size_t smem = tile_layout(g).total;

  /* every call shares the scratch: keys start at "no candidate yet", counters
     at zero; the tables are rewritten for this call's lattice */
  cudaError_t e = cudaMemsetAsync(keys, 0xff, sizeof(unsigned long long) * n, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(tickets, 0, sizeof(unsigned) * n, st);
  if (e != cudaSuccess) return fail("clearing the scratch", e);
  int blocks = (int)((lattice + 255) / 256);
  k_noalloc_tables<<<blocks < 1024 ? blocks : 1024, 256, 0, st>>>(K, stepSize, order, point);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail("k_noalloc_tables", e);
  const vsbd_item* items = (const vsbd_item*)d_items;
  vsbd_result* res = (vsbd_result*)d_results;
  switch (g.tb) {
    case 2:
      e = g.ta == 4   ? launch_tb<2, 4>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
          : g.ta == 3 ? launch_tb<2, 3>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
          : g.ta == 2 ? launch_tb<2, 2>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
                      : launch_tb<2, 1>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st);
      break;
    case 4:
      e = g.ta == 4   ? launch_tb<4, 4>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
          : g.ta == 3 ? launch_tb<4, 3>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
          : g.ta == 2 ? launch_tb<4, 2>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st)
                      : launch_tb<4, 1>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st);
      break;
    case 8: e = launch_tb<8, 1>(g, smem, d_curr, d_prev, pitch, items, n, keys, tickets, res, st); break;
    default: return fail("unsupported tiling", cudaSuccess);
  }
  if (e != cudaSuccess) return fail("k_lattice", e);
  return 0;
}
