/*
 * vsb_l2t.cu -- the second pass on the GPU: one global transform per frame
 * from the frame's LocalMotions, every frame of a clip (or of many streams)
 * at once, one warp per frame.
 *
 * Algorithm: vsMotionsToTransform and vsGradientDescent of the reference
 * (src/localmotion2transform.c:137-330) with calcTransformQuality as the
 * objective: the translation seed is the mean of the motions, fields whose
 * match is worse than mean + 1.5 sigma are masked, then up to three rounds
 * of a coordinate-wise finite-difference descent over (x, y, alpha, zoom)
 * (16 sweeps of the four coordinates, step sizes 0.2, 0.2, 5e-5, 0.1, grown
 * by 1.2 on success and halved on failure, stopping once the objective is
 * at most 0.01); between rounds the fields whose residual is above
 * mean + 1 sigma are masked too.
 *
 * Bit-exactness.  The reference's shipped build (-O3 -msse2 -ffast-math)
 * fixes how each expression is grouped and rounded; this file follows that
 * order, is compiled with --fmad=false (no contraction of a multiply and an
 * add into one rounding) and uses only IEEE-rounded double operations
 * except cos/sin, which come from CUDA's math library (the reference calls
 * glibc's): where the two differ in the last bit an objective value can
 * differ in its last bits, and a descent step that compares two values that
 * close can go the other way.  The pinned order:
 *   - the error sum of an objective evaluation is sequential in field order
 *     (one lane adds while the others have computed the terms);
 *   - mean() sums even and odd elements separately and adds the two partial
 *     sums, then the odd tail (the build vectorises it two-wide); stddev()
 *     is sequential;
 *   - x' = (zcos*rx + zsin*ry) + (t.x + c_x); y' = (-zsin*rx + zcos*ry) +
 *     (t.y + c_y); z = 1 + zoom*0.01; the penalty is
 *     error/num + (|alpha|*0.2 + |zoom|*0.002);
 *   - rotational model: X = (r0*rx + r1*ry) + r2*f, x' = ((z*f)*X)/Z + c_x;
 *     the focal length arrives from the host, computed there as
 *     (w/2) / tan(fov*(pi/360)).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "vidstab_b200.h"
#include "vsb_plan.h"

namespace {

constexpr int kWarp = 32;
/* shared memory per motion: packed (v.x, v.y, f.x, f.y) + the mask/residual */
constexpr int kSmemPerMotion = 16;
constexpr int kSmemLimit = 220 * 1024;

struct L2TArgs {
  const LocalMotion* recs;
  const long* first;
  int nframes;
  int max_motions; /* shared memory was sized for this many motions per frame */
  double cx, cy;   /* double(width/2), double(height/2) */
  double f;      /* focal length in pixels, 0: similarity model */
  int smooth_zoom;
  VSTransform* out;
  double* residual;
  int* info;
};

__device__ __forceinline__ double wrap_angle(double a) {
  /* new_transform, src/transformtype.c:38-58; the reference's loops never
     end for an infinite angle, these stop after 64 turns either way (an
     angle that far out comes only from a diverged objective) */
  for (int it = 0; it < 64 && a < -M_PI; it++) a += 2.0 * M_PI;
  for (int it = 0; it < 64 && a > M_PI; it++) a -= 2.0 * M_PI;
  return a;
}

/* 3x3 product a.b with the sum of each entry taken left to right
   (src/transformtype.c:130-140) */
__device__ __forceinline__ void mat3mul(const double* a, const double* b, double* out) {
  double t[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) s = s + a[3 * i + k] * b[3 * k + j];
      t[3 * i + j] = s;
    }
#pragma unroll
  for (int i = 0; i < 9; i++) out[i] = t[i];
}

/* the forward rotation of the rotational model: the transpose of
   rotation_matrix_backward(yaw, pitch, roll) (src/transformtype.c:142-156,
   :175-182) */
__device__ void rotation_forward(double yaw, double pitch, double roll, double* r) {
  const double cy = cos(-yaw), sy = sin(-yaw);
  const double cp = cos(pitch), sp = sin(pitch);
  const double cr = cos(roll), sr = sin(roll);
  const double Ry[9] = {cy, 0.0, sy, 0.0, 1.0, 0.0, -sy, 0.0, cy};
  const double Rx[9] = {1.0, 0.0, 0.0, 0.0, cp, -sp, 0.0, sp, cp};
  const double Rz[9] = {cr, -sr, 0.0, sr, cr, 0.0, 0.0, 0.0, 1.0};
  double b[9];
  mat3mul(Ry, Rx, b);
  mat3mul(b, Rz, b);
  r[0] = b[0]; r[1] = b[3]; r[2] = b[6];
  r[3] = b[1]; r[4] = b[4]; r[5] = b[7];
  r[6] = b[2]; r[7] = b[5]; r[8] = b[8];
}

struct FrameSmem {
  const short4* q; /* v.x, v.y, f.x, f.y per motion */
  double* mm;      /* < 0: field masked; else its last squared residual */
  int n;
};

/* calcTransformQuality (src/localmotion2transform.c:139-172) at p = (x, y,
   alpha, zoom): every lane computes the residuals of its fields, lane 0 adds
   them in field order; the value is returned to all lanes. */
__device__ double quality(const double* p, const FrameSmem& fs, const L2TArgs& A, int lane) {
  const double a = wrap_angle(p[2]);
  const double z = p[3];
  const double zz = 1.0 + z * 0.01;
  if (A.f > 0.0) {
    const double f = A.f;
    const double zf = zz * f;
    double r[9];
    rotation_forward(p[0] / f, p[1] / f, a, r);
    for (int i = lane; i < fs.n; i += kWarp) {
      if (fs.mm[i] >= 0.0) {
        const short4 q = fs.q[i];
        const double fx = (double)q.z, fy = (double)q.w;
        const double rx = fx - A.cx, ry = fy - A.cy;
        const double X = (r[0] * rx + r[1] * ry) + r[2] * f;
        const double Y = (r[3] * rx + r[4] * ry) + r[5] * f;
        const double Z = (r[6] * rx + r[7] * ry) + r[8] * f;
        const double vx = (zf * X) / Z + A.cx;
        const double vy = (zf * Y) / Z + A.cy;
        const double ex = (vx - fx) - (double)q.x;
        const double ey = (vy - fy) - (double)q.y;
        fs.mm[i] = ex * ex + ey * ey;
      }
    }
  } else {
    const double zc = zz * cos(a), zs = zz * sin(a);
    const double tx = p[0] + A.cx, ty = p[1] + A.cy;
    for (int i = lane; i < fs.n; i += kWarp) {
      if (fs.mm[i] >= 0.0) {
        const short4 q = fs.q[i];
        const double fx = (double)q.z, fy = (double)q.w;
        const double rx = fx - A.cx, ry = fy - A.cy;
        const double vx = (zc * rx + zs * ry) + tx;
        const double vy = ((-zs) * rx + zc * ry) + ty;
        const double ex = (vx - fx) - (double)q.x;
        const double ey = (vy - fy) - (double)q.y;
        fs.mm[i] = ex * ex + ey * ey;
      }
    }
  }
  __syncwarp();
  double v = 0.0;
  if (lane == 0) {
    /* adding +0.0 leaves a non-negative sum unchanged, so masked fields
       contribute 0.0 instead of a branch */
    double s = 0.0;
    int num = 1;
    int i = 0;
    for (; i + 4 <= fs.n; i += 4) {
      const double m0 = fs.mm[i], m1 = fs.mm[i + 1], m2 = fs.mm[i + 2], m3 = fs.mm[i + 3];
      s = s + (m0 >= 0.0 ? m0 : 0.0);
      s = s + (m1 >= 0.0 ? m1 : 0.0);
      s = s + (m2 >= 0.0 ? m2 : 0.0);
      s = s + (m3 >= 0.0 ? m3 : 0.0);
      num += (m0 >= 0.0) + (m1 >= 0.0) + (m2 >= 0.0) + (m3 >= 0.0);
    }
    for (; i < fs.n; i++) {
      const double m = fs.mm[i];
      s = s + (m >= 0.0 ? m : 0.0);
      num += (m >= 0.0);
    }
    v = s / (double)num + (fabs(a) * 0.2 + fabs(z) * 0.002);
  }
  v = __shfl_sync(0xffffffffu, v, 0);
  return v;
}

/* disableFields (src/localmotion2transform.c:204-218) with the quality
   values q[i] (q may alias mm): lanes 0 and 1 form mean()'s two interleaved
   partial sums, lane 0 the sequential stddev() sum; every lane then masks
   its fields.  Returns the number of fields masked. */
__device__ int disable_fields(double* mm, const double* q, int qstride, int n, double k,
                              int lane) {
  double part = 0.0;
  const int n0 = n / 2 * 2;
  if (lane < 2)
    for (int i = lane; i < n0; i += 2) part = part + q[(size_t)i * qstride];
  const double p1 = __shfl_sync(0xffffffffu, part, 1);
  double thresh = 0.0;
  if (lane == 0) {
    double s = part + p1;
    for (int i = n0; i < n; i++) s = s + q[(size_t)i * qstride];
    const double mu = s / (double)n;
    double d2 = 0.0;
    for (int i = 0; i < n; i++) {
      const double d = q[(size_t)i * qstride] - mu;
      d2 = d2 + d * d;
    }
    thresh = mu + k * sqrt(d2 / (double)n);
  }
  thresh = __shfl_sync(0xffffffffu, thresh, 0);
  __syncwarp();
  int cnt = 0;
  for (int i = lane; i < n; i += kWarp) {
    if (q[(size_t)i * qstride] > thresh) {
      mm[i] = -1.0;
      cnt++;
    }
  }
  __syncwarp();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  return cnt;
}

/* vsGradientDescent (src/localmotion2transform.c:288-330), N = 16 sweeps,
   threshold 0.01; x is updated in place, the final value returned */
__device__ double gradient_descent(double* x, const FrameSmem& fs, const L2TArgs& A, int lane) {
  double ss[4] = {0.2, 0.2, 0.00005, 0.1};
  double v = quality(x, fs, A, lane);
  for (int i = 0; i < 16 * 4 && v > 0.01; i++) {
    const int k = i & 3;
    const double h = ((i >> 2) & 1) ? 1e-6 : -1e-6;
    double x2[4];
#pragma unroll
    for (int j = 0; j < 4; j++) x2[j] = (j == k) ? x[j] + h : x[j];
    double v2 = quality(x2, fs, A, lane);
    const double g = (v - v2) / h;
    double sk = ss[0];
#pragma unroll
    for (int j = 1; j < 4; j++) sk = (j == k) ? ss[j] : sk;
#pragma unroll
    for (int j = 0; j < 4; j++) x2[j] = x[j] + ((j == k ? g : 0.0) * sk);
    v2 = quality(x2, fs, A, lane);
    const bool better = v2 < v;
    if (better) {
#pragma unroll
      for (int j = 0; j < 4; j++) x[j] = x2[j];
      v = v2;
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (j == k) ss[j] = better ? ss[j] * 1.2 : ss[j] / 2.0;
  }
  return v;
}

/* One warp per frame (vsMotionsToTransform, src/localmotion2transform.c:
   220-284).  Dynamic shared memory: kSmemPerMotion bytes per motion of the
   largest frame. */
__global__ void __launch_bounds__(kWarp) k_l2t(L2TArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int frame = blockIdx.x;
  const int lane = threadIdx.x;
  if (frame >= A.nframes) return;
  const long b = A.first[frame];
  const int n = (int)(A.first[frame + 1] - b);
  const LocalMotion* rec = A.recs + b;
  VSTransform t;
  t.x = t.y = t.alpha = t.zoom = t.barrel = t.rshutter = 0.0;
  t.extra = 0;
  if (n <= 0 || n > A.max_motions) {
    /* meanMotions: no fields, the frame is to be ignored later.  A frame
       larger than the launch was sized for is not fitted: flagged the same
       way, with rounds = -1 */
    if (lane == 0) {
      t.extra = 1;
      A.out[frame] = t;
      if (A.residual) A.residual[frame] = __longlong_as_double(0x7ff8000000000000ll);
      if (A.info) {
        A.info[3 * frame] = n > 0 ? -1 : 0;
        A.info[3 * frame + 1] = A.info[3 * frame + 2] = 0;
      }
    }
    return;
  }
  short4* q = reinterpret_cast<short4*>(smem);
  double* mm = reinterpret_cast<double*>(smem + (size_t)n * sizeof(short4));
  long long sx = 0, sy = 0;
  for (int i = lane; i < n; i += kWarp) {
    const short4 r = *reinterpret_cast<const short4*>(&rec[i]);
    q[i] = r;
    mm[i] = 0.0;
    sx += r.x;
    sy += r.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  __syncwarp();
  const FrameSmem fs{q, mm, n};
  /* meanMotions: the integer sums are exact in double */
  double params[4] = {(double)sx / (double)n, (double)sy / (double)n, 0.0, 0.0};
  /* the match qualities straight from the records (stride 4 doubles) */
  const double* match = reinterpret_cast<const double*>(rec) + 3;
  const int dis1 = disable_fields(mm, match, 4, n, 1.5, lane);
  int dis2 = 0, rounds = 0;
  double res[4], resid = 0.0;
  for (int k = 0; k < 3; k++) {
#pragma unroll
    for (int j = 0; j < 4; j++) res[j] = params[j];
    resid = gradient_descent(res, fs, A, lane);
    rounds = k + 1;
    if ((k == 0 && resid > 0.1) || (k == 1 && resid > 20)) {
      dis2 += disable_fields(mm, mm, 1, n, 1.0, lane);
#pragma unroll
      for (int j = 0; j < 4; j++) params[j] = res[j];
    } else {
      break;
    }
  }
  if (lane == 0) {
    t.x = res[0];
    t.y = res[1];
    t.alpha = wrap_angle(res[2]);
    t.zoom = A.smooth_zoom ? res[3] : 0.0;
    t.extra = resid > 100 ? 1 : 0;
    A.out[frame] = t;
    if (A.residual) A.residual[frame] = resid;
    if (A.info) {
      A.info[3 * frame] = rounds;
      A.info[3 * frame + 1] = dis1;
      A.info[3 * frame + 2] = dis2;
    }
  }
}

/* host-side state of the blocking entry point: device buffers grown as
   needed, one stream; a mutex serialises callers */
struct L2THost {
  std::mutex mu;
  int dev = -1;
  cudaStream_t stream = nullptr;
  LocalMotion* d_recs = nullptr;
  long* d_first = nullptr;
  VSTransform* d_out = nullptr;
  double* d_resid = nullptr;
  int* d_info = nullptr;
  size_t cap_recs = 0, cap_frames = 0;
};
L2THost g_host;
unsigned long long g_launches = 0;

int grow(L2THost& h, size_t nrecs, size_t nframes) {
  if (nrecs > h.cap_recs) {
    if (h.d_recs) cudaFree(h.d_recs);
    h.d_recs = nullptr;
    h.cap_recs = 0;
    const size_t c = nrecs + nrecs / 4 + 256;
    cudaError_t e = cudaMalloc(&h.d_recs, c * sizeof(LocalMotion));
    if (e != cudaSuccess) { vsbp_set_err("second pass: device records", e); return -1; }
    h.cap_recs = c;
  }
  if (nframes > h.cap_frames) {
    if (h.d_first) cudaFree(h.d_first);
    if (h.d_out) cudaFree(h.d_out);
    if (h.d_resid) cudaFree(h.d_resid);
    if (h.d_info) cudaFree(h.d_info);
    h.d_first = nullptr; h.d_out = nullptr; h.d_resid = nullptr; h.d_info = nullptr;
    h.cap_frames = 0;
    const size_t c = nframes + nframes / 4 + 64;
    cudaError_t e = cudaMalloc(&h.d_first, (c + 1) * sizeof(long));
    if (e == cudaSuccess) e = cudaMalloc(&h.d_out, c * sizeof(VSTransform));
    if (e == cudaSuccess) e = cudaMalloc(&h.d_resid, c * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&h.d_info, c * 3 * sizeof(int));
    if (e != cudaSuccess) { vsbp_set_err("second pass: device buffers", e); return -1; }
    h.cap_frames = c;
  }
  return 0;
}

double l2t_focal(double fov, int width) {
  /* src/transformtype.c:123-127 as the reference build evaluates it */
  if (fov <= 0.0 || fov >= 180.0 || width <= 0) return 0.0;
  return (width / 2.0) / tan(fov * (M_PI / 360.0));
}

int launch(const LocalMotion* d_recs, const long* d_first, int nframes, int max_motions,
           int width, int height, double fov, int smooth_zoom, VSTransform* d_out,
           double* d_resid, int* d_info, cudaStream_t st) {
  if (nframes < 0 || max_motions < 0 || width <= 0 || height <= 0) {
    vsbp_set_msg("second pass: invalid arguments");
    return -1;
  }
  if (nframes == 0) return 0;
  const size_t smem = (size_t)max_motions * kSmemPerMotion;
  if (smem > (size_t)kSmemLimit) {
    char m[160];
    snprintf(m, sizeof(m), "second pass: %d motions in one frame exceed the capacity of %d",
             max_motions, kSmemLimit / kSmemPerMotion);
    vsbp_set_msg(m);
    return -1;
  }
  cudaError_t e = cudaFuncSetAttribute(k_l2t, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(smem < 16 ? 16 : smem));
  if (e != cudaSuccess) { vsbp_set_err("cudaFuncSetAttribute(k_l2t)", e); return -1; }
  L2TArgs A;
  A.recs = d_recs;
  A.first = d_first;
  A.nframes = nframes;
  A.max_motions = max_motions;
  A.cx = (double)(width / 2);
  A.cy = (double)(height / 2);
  A.f = l2t_focal(fov, width);
  A.smooth_zoom = smooth_zoom;
  A.out = d_out;
  A.residual = d_resid;
  A.info = d_info;
  k_l2t<<<nframes, kWarp, smem, st>>>(A);
  e = cudaGetLastError();
  if (e != cudaSuccess) { vsbp_set_err("k_l2t launch", e); return -1; }
  __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED);
  return 0;
}

} // namespace

extern "C" int vsb_motions_to_transforms_capacity(void) { return kSmemLimit / kSmemPerMotion; }

extern "C" long vsb_motions_to_transforms_launches(void) {
  return (long)__atomic_load_n(&g_launches, __ATOMIC_RELAXED);
}

extern "C" int vsb_motions_to_transforms_device(const LocalMotion* d_recs, const long* d_first,
                                                int nframes, int max_motions, int width,
                                                int height, double fov, int smooth_zoom,
                                                VSTransform* d_out, double* d_residual,
                                                int* d_info, void* stream) {
  if (!d_first || !d_out || (nframes > 0 && max_motions > 0 && !d_recs)) {
    vsbp_set_msg("second pass: null pointer");
    return -1;
  }
  return launch(d_recs, d_first, nframes, max_motions, width, height, fov, smooth_zoom, d_out,
                d_residual, d_info, (cudaStream_t)stream);
}

extern "C" int vsb_motions_to_transforms(const LocalMotion* recs, const long* first, int nframes,
                                         int width, int height, double fov, int smooth_zoom,
                                         VSTransform* out, double* residual, int* info) {
  if (nframes < 0 || !first || (nframes > 0 && !out)) {
    vsbp_set_msg("second pass: invalid arguments");
    return -1;
  }
  if (nframes == 0) return 0;
  long maxn = 0;
  for (int k = 0; k < nframes; k++) {
    const long n = first[k + 1] - first[k];
    if (n < 0 || first[k] < 0) {
      vsbp_set_msg("second pass: frame offsets must not decrease");
      return -1;
    }
    if (n > maxn) maxn = n;
  }
  const long total = first[nframes];
  if (total > 0 && !recs) {
    vsbp_set_msg("second pass: null records");
    return -1;
  }
  if (maxn > vsb_motions_to_transforms_capacity()) {
    char m[160];
    snprintf(m, sizeof(m), "second pass: %ld motions in one frame exceed the capacity of %d",
             maxn, vsb_motions_to_transforms_capacity());
    vsbp_set_msg(m);
    return -1;
  }
  std::lock_guard<std::mutex> lk(g_host.mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { vsbp_set_err("second pass: cudaGetDevice", e); return -1; }
  if (g_host.dev != dev) {
    /* buffers of another device are not reused */
    if (g_host.dev >= 0) {
      int cur = dev;
      cudaSetDevice(g_host.dev);
      if (g_host.stream) cudaStreamDestroy(g_host.stream);
      cudaFree(g_host.d_recs); cudaFree(g_host.d_first); cudaFree(g_host.d_out);
      cudaFree(g_host.d_resid); cudaFree(g_host.d_info);
      cudaSetDevice(cur);
    }
    g_host.stream = nullptr;
    g_host.d_recs = nullptr; g_host.d_first = nullptr; g_host.d_out = nullptr;
    g_host.d_resid = nullptr; g_host.d_info = nullptr;
    g_host.cap_recs = g_host.cap_frames = 0;
    e = cudaStreamCreateWithFlags(&g_host.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { vsbp_set_err("second pass: stream", e); return -1; }
    g_host.dev = dev;
  }
  if (grow(g_host, (size_t)total, (size_t)nframes)) return -1;
  cudaStream_t st = g_host.stream;
  if (total > 0)
    e = cudaMemcpyAsync(g_host.d_recs, recs, (size_t)total * sizeof(LocalMotion),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g_host.d_first, first, (size_t)(nframes + 1) * sizeof(long),
                        cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) { vsbp_set_err("second pass: upload", e); return -1; }
  if (launch(g_host.d_recs, g_host.d_first, nframes, (int)maxn, width, height, fov, smooth_zoom,
             g_host.d_out, g_host.d_resid, g_host.d_info, st))
    return -1;
  e = cudaMemcpyAsync(out, g_host.d_out, (size_t)nframes * sizeof(VSTransform),
                      cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && residual)
    e = cudaMemcpyAsync(residual, g_host.d_resid, (size_t)nframes * sizeof(double),
                        cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && info)
    e = cudaMemcpyAsync(info, g_host.d_info, (size_t)nframes * 3 * sizeof(int),
                        cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { vsbp_set_err("second pass: download", e); return -1; }
  return 0;
}
