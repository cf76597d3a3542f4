/*
 * vsb_plan.h -- planning helpers of the search (tilings, geometry tables on
 * the device) shared by the per-stream shim (vsb_device.cu) and the batched
 * path (vsb_batch.cu).  C++ only.
 */
#ifndef VSB_PLAN_H
#define VSB_PLAN_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "vsb_device.h"
#include "vsb_search.cuh"

/* a field set's geometry with its rank/point tables in device memory */
struct GeomDev {
  DGeom g;
  int32_t* d_order;
  short2* d_point;
  size_t smem;
  int list_cps; /* CTAs per SM of the list-driven search with this tiling (0: not known) */
};

/* a tiling with its modelled cost */
struct TileCand {
  double clk;
  DGeom g;
};

/* uploads the tables and picks the cost model's best tiling */
int vsbp_geom_upload(const vsbd_geom* h, int nitems, GeomDev* out);
void vsbp_geom_free(GeomDev* g);
/* the cap best tilings (model order) with at most max_threads threads */
int vsbp_tile_candidates(const DGeom& g, int nitems, int max_threads, TileCand* out, int cap);
/* the same, with ta lattice columns per thread only (1 or 2) */
int vsbp_tile_candidates_ta(const DGeom& g, int nitems, int max_threads, TileCand* out, int cap,
                            int ta);
/* SMs of the current device */
int vsbp_sm_count(void);
void vsbp_set_err(const char* what, cudaError_t e);
void vsbp_set_msg(const char* m);
/* process-wide counters of the per-frame path */
void vsbp_count(long launches, size_t h2d, size_t d2h);

/* Every device allocation of the library's CUDA units that include this
   header goes through vsbd_dev_malloc, which counts them and can be told to
   fail one (vsb_test_device_alloc): the library's handling of an
   out-of-memory GPU is then testable without exhausting a GPU. */
extern "C" cudaError_t vsbd_dev_malloc(void** p, size_t bytes);
template <class T>
static inline cudaError_t vsbp_cuda_malloc(T** p, size_t bytes) {
  return vsbd_dev_malloc((void**)p, bytes);
}
#define cudaMalloc(p, bytes) vsbp_cuda_malloc((p), (bytes))

#endif
