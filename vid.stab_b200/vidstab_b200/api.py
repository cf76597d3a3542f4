"""Python calls over the C ABI: a per-frame detector mirroring the reference
API (vsMotionDetectInit / vsMotionDetection / vsMotionDetectionCleanup) and
a clip driver that loops in C."""
import ctypes as C

import numpy as np

from ._lib import (LM_DTYPE, PF_PACKED, PF_RGBA, TRANSFORM_DTYPE, VSFrame, VSFrameInfo,
                   VSMotionDetect, VSVector, lib, ptr, vector_records)


def records_per_frame(width, height):
    """an upper bound of the LocalMotions one frame can give: every coarse
    and every fine field (fine fields are at least 16 pixels apart)"""
    return 256 + (width // 16 + 1) * (height // 16 + 1)


def _check_fits(total, out):
    """the C loops copy at most len(out) records but count them all"""
    if total > len(out):
        raise ValueError("%d LocalMotions do not fit the record buffer of %d" % (total, len(out)))


def bpp_of(pformat):
    if pformat < PF_PACKED:
        return 1
    return 4 if pformat == PF_RGBA else 3


class MotionDetector:
    """One detect stream (src/motiondetect.h:121-147 of the reference)."""

    def __init__(self, width, height, pformat=1, stepsize=6, accuracy=15, shakiness=5,
                 mincontrast=0.25, tripod=0, show=0, serialization_mode=0):
        L = lib()
        self.L = L
        self.fi = VSFrameInfo()
        if not L.vsFrameInfoInit(C.byref(self.fi), width, height, pformat):
            raise ValueError("invalid frame geometry / pixel format")
        conf = L.vsMotionDetectGetDefaultConfig(b"vidstab_b200")
        conf.stepSize, conf.accuracy, conf.shakiness = stepsize, accuracy, shakiness
        conf.contrastThreshold, conf.virtualTripod, conf.show = mincontrast, tripod, show
        self.conf = conf
        self.md = VSMotionDetect()
        self.md.serializationMode = serialization_mode
        if L.vsMotionDetectInit(C.byref(self.md), C.byref(conf), C.byref(self.fi)) != 0:
            raise RuntimeError("vsMotionDetectInit failed: %s" % L.vsb_last_error().decode())
        self.width, self.height, self.pformat = width, height, pformat
        self._chroma = np.full(width * height + 64, 128, np.uint8)

    def detect(self, plane0, linesize=None):
        """Motions of one frame given its plane 0 (host numpy array)."""
        plane0 = np.ascontiguousarray(plane0)
        f = VSFrame()
        f.data[0] = plane0.ctypes.data
        f.linesize[0] = linesize or plane0.strides[0]
        for p in range(1, self.fi.planes):
            f.data[p] = self._chroma.ctypes.data
            f.linesize[p] = self.width >> (self.fi.log2ChromaW if p in (1, 2) else 0)
        v = VSVector()
        if self.L.vsMotionDetection(C.byref(self.md), C.byref(v), C.byref(f)) != 0:
            raise RuntimeError("vsMotionDetection failed: %s" % self.L.vsb_last_error().decode())
        out = vector_records(v)
        self.L.vs_vector_del(C.byref(v))
        return out

    def detect_device(self, dptr, pitch):
        """Motions of one frame whose plane 0 is at CUDA address dptr."""
        v = VSVector()
        if self.L.vsb_motion_detection_device(C.byref(self.md), C.byref(v), C.c_void_p(dptr),
                                              pitch) != 0:
            raise RuntimeError("vsb_motion_detection_device failed: %s"
                               % self.L.vsb_last_error().decode())
        out = vector_records(v)
        self.L.vs_vector_del(C.byref(v))
        return out

    def run(self, n, frames_ptr, frame_bytes, linesize, on_device, out, counts):
        """Frames n in order through this detector in C (vsb_detect_run):
        records appended to the preallocated LM_DTYPE array out, per-frame
        counts to the int32 array counts.  Returns the number of records."""
        if len(out) * out.itemsize < 32 or len(counts) < n:
            raise ValueError("output buffers too small")
        total = self.L.vsb_detect_run(C.byref(self.md), C.c_void_p(frames_ptr), frame_bytes,
                                      linesize, n, 1 if on_device else 0, ptr(out), len(out),
                                      ptr(counts))
        if total < 0:
            raise RuntimeError("vsb_detect_run failed: %s" % self.L.vsb_last_error().decode())
        _check_fits(total, out)
        return total

    def run_frames(self, n, frames_ptr, frame_bytes, linesize, on_device, out, counts):
        """As run, one vsMotionDetection call per frame with no overlap
        between frames (vsb_detect_frames): a host filter's call sequence."""
        if len(out) * out.itemsize < 32 or len(counts) < n:
            raise ValueError("output buffers too small")
        total = self.L.vsb_detect_frames(C.byref(self.md), C.c_void_p(frames_ptr), frame_bytes,
                                         linesize, n, 1 if on_device else 0, ptr(out), len(out),
                                         ptr(counts))
        if total < 0:
            raise RuntimeError("vsb_detect_frames failed: %s" % self.L.vsb_last_error().decode())
        _check_fits(total, out)
        return total

    @property
    def frame_num(self):
        return self.md.frameNum

    def launches(self):
        return self.L.vsb_launch_count(C.byref(self.md))

    def close(self):
        if self.md is not None and self.md.initialized:
            self.L.vsMotionDetectionCleanup(C.byref(self.md))
        self.md = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent detect streams stepped together (vsb_batch_*): every
    step runs the device work of all streams in two persistent-kernel
    launches replayed from captured CUDA graphs.  Stream s gives the
    LocalMotions a MotionDetector of its own would give."""

    def __init__(self, widths, heights, pformat=1, stepsize=6, accuracy=15, shakiness=5,
                 mincontrast=0.25, tripod=0):
        L = lib()
        self.L = L
        self.n = len(widths)
        conf = L.vsMotionDetectGetDefaultConfig(b"vidstab_b200")
        conf.stepSize, conf.accuracy, conf.shakiness = stepsize, accuracy, shakiness
        conf.contrastThreshold, conf.virtualTripod = mincontrast, tripod
        confs = (type(conf) * self.n)(*([conf] * self.n))
        self.widths = np.ascontiguousarray(widths, np.int32)
        self.heights = np.ascontiguousarray(heights, np.int32)
        self.h = L.vsb_batch_create(self.n, ptr(self.widths), ptr(self.heights), pformat,
                                    C.cast(confs, C.c_void_p))
        if not self.h:
            raise RuntimeError("vsb_batch_create failed: %s" % L.vsb_last_error().decode())

    def run(self, clip_ptrs, frame_bytes, pitches, nframes, on_device, out, counts):
        """nframes steps; stream s's frame k at clip_ptrs[s] + k*frame_bytes[s].
        Records go to the preallocated LM_DTYPE array out (step by step,
        stream by stream), counts (int32, nframes*n) gets per-frame counts."""
        clips = np.ascontiguousarray(clip_ptrs, np.uint64)
        fb = np.ascontiguousarray(frame_bytes, np.int64)
        pt = np.ascontiguousarray(pitches, np.int32)
        if len(counts) < nframes * self.n:
            raise ValueError("counts too small")
        total = self.L.vsb_batch_run(self.h, ptr(clips), ptr(fb), ptr(pt), nframes,
                                     1 if on_device else 0, ptr(out), len(out), ptr(counts))
        if total < 0:
            raise RuntimeError("vsb_batch_run failed: %s" % self.L.vsb_last_error().decode())
        _check_fits(total, out)
        return total

    def detect(self, planes, pitches, on_device):
        """One step: a list of n records arrays."""
        pl = np.ascontiguousarray(planes, np.uint64)
        pt = np.ascontiguousarray(pitches, np.int32)
        vs = (VSVector * self.n)()
        if self.L.vsb_batch_detect(self.h, ptr(pl), ptr(pt), 1 if on_device else 0,
                                   C.cast(vs, C.c_void_p)) != 0:
            raise RuntimeError("vsb_batch_detect failed: %s" % self.L.vsb_last_error().decode())
        out = []
        for v in vs:
            out.append(vector_records(v))
            self.L.vs_vector_del(C.byref(v))
        return out

    def set_proposal(self, blob):
        """The learned search proposal (VSBP bytes) for every stream, as work
        items of the same persistent kernel; None: the dense search again."""
        self._blob = C.create_string_buffer(blob, len(blob)) if blob is not None else None
        if self.L.vsb_batch_set_proposal(self.h, self._blob, len(blob) if blob else 0) != 0:
            raise RuntimeError("vsb_batch_set_proposal failed: %s" %
                               self.L.vsb_last_error().decode())

    def proposal_stats(self):
        """{searched, fell_back, coarse_searched, coarse_fell_back,
        fine_searched, fine_fell_back} since set_proposal"""
        st = (C.c_longlong * 8)()
        if self.L.vsb_batch_proposal_stats(self.h, st) != 0:
            raise RuntimeError("vsb_batch_proposal_stats failed")
        v = [int(x) for x in st]
        return {"searched": v[0], "fell_back": v[1], "coarse_searched": v[4],
                "coarse_fell_back": v[5], "fine_searched": v[6], "fine_fell_back": v[7]}

    def launches(self):
        return self.L.vsb_batch_launch_count(self.h)

    def grid(self):
        a, b, c = C.c_int(), C.c_int(), C.c_long()
        self.L.vsb_batch_grid(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def open_trf(self, paths, serialization_mode=1):
        """Starts a .trf file per stream (None: no file for that stream);
        later steps append to them (vsb_batch_open_trf)."""
        enc = [p.encode() if p is not None else None for p in paths]
        arr = (C.c_char_p * self.n)(*enc)
        if self.L.vsb_batch_open_trf(self.h, C.cast(arr, C.c_void_p), serialization_mode) != 0:
            raise RuntimeError("vsb_batch_open_trf failed")

    def close_trf(self):
        if self.L.vsb_batch_close_trf(self.h) != 0:
            raise RuntimeError("vsb_batch_close_trf failed")

    def classes(self):
        """Per geometry class: the search tiling and its tuned time
        (vsb_batch_class)."""
        keys = ("rows_per_thread", "layout", "cols_per_cta", "rows_per_cta", "strips",
                "threads", "smem", "ctas_per_field", "items", "tuned_ns", "field_size",
                "lattice_points")
        n = self.L.vsb_batch_class(self.h, -1, None)
        out = []
        for k in range(n):
            d = (C.c_int * 12)()
            self.L.vsb_batch_class(self.h, k, d)
            out.append(dict(zip(keys, list(d))))
        return out

    def close(self):
        if self.h:
            self.L.vsb_batch_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def detect_multi(detectors, clip_ptrs, frame_bytes, pitches, nframes, on_device, out, counts):
    """Steps many MotionDetectors together (vsb_detect_multi): frame k of
    stream s at clip_ptrs[s] + k*frame_bytes[s].  Records go to the
    preallocated LM_DTYPE array out (frame by frame, stream by stream),
    counts (int32, nframes*n) gets per-frame counts.  Returns the number of
    records."""
    L = lib()
    n = len(detectors)
    if not getattr(L, "_multi_bound", False):
        L.vsb_detect_multi.restype = C.c_long
        L.vsb_detect_multi.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p]
        L._multi_bound = True
    mds = (C.POINTER(VSMotionDetect) * n)(*[C.pointer(d.md) for d in detectors])
    clips = np.ascontiguousarray(clip_ptrs, np.uint64)
    fb = np.ascontiguousarray(frame_bytes, np.int64)
    pt = np.ascontiguousarray(pitches, np.int32)
    if len(counts) < nframes * n:
        raise ValueError("counts too small")
    total = L.vsb_detect_multi(C.cast(mds, C.c_void_p), n, ptr(clips), ptr(fb), ptr(pt), nframes,
                               1 if on_device else 0, ptr(out), len(out), ptr(counts))
    if total < 0:
        raise RuntimeError("vsb_detect_multi failed: %s" % L.vsb_last_error().decode())
    _check_fits(total, out)
    return total


def detect_clip(frames, pformat=1, stepsize=6, accuracy=15, shakiness=5, mincontrast=0.25,
                tripod=0, show=0, serialization_mode=0, trf_path=None, on_device_ptr=None,
                frame_bytes=None, linesize=None, width=None, height=None, return_frames=False):
    """Runs the detect API over a clip in C.

    frames: numpy uint8 array (n, H, W) planar / (n, H, W*bpp) packed, or
    with on_device_ptr a CUDA address of n frames frame_bytes apart.
    Returns (records, counts, elapsed_seconds[, drawn frames])."""
    L = lib()
    if on_device_ptr is None:
        frames = np.ascontiguousarray(frames)
        n, H = frames.shape[0], frames.shape[1]
        W = frames.shape[2] // bpp_of(pformat)
        fb = frames[0].nbytes
        ls = frames.shape[2]
        src = frames.ctypes.data
    else:
        n = frames
        H, W, fb, ls, src = height, width, frame_bytes, linesize, on_device_ptr
    cap = n * records_per_frame(W, H) + 64
    out = np.zeros(cap, LM_DTYPE)
    counts = np.zeros(n, np.int32)
    el = C.c_double(0)
    drawn = np.zeros((n, fb), np.uint8) if (show and return_frames) else None
    total = L.vsb_detect_clip(W, H, pformat, C.c_void_p(src), fb, ls, n,
                              1 if on_device_ptr is not None else 0, stepsize, accuracy,
                              shakiness, mincontrast, tripod, show, serialization_mode,
                              trf_path.encode() if trf_path else None, ptr(out), cap, ptr(counts),
                              C.byref(el), ptr(drawn))
    if total < 0:
        raise RuntimeError("vsb_detect_clip failed: %s" % L.vsb_last_error().decode())
    _check_fits(total, out)
    res = (out[:total].copy(), counts, el.value)
    if return_frames:
        res = res + (drawn,)
    return res


def boxblur(plane, size):
    """GPU prefilter of one tight W x H plane with (clamped) box size."""
    L = lib()
    plane = np.ascontiguousarray(plane, dtype=np.uint8)
    H, W = plane.shape
    out = np.empty_like(plane)
    if L.vsb_boxblur_host(ptr(out), ptr(plane), W, H, size) != 0:
        raise RuntimeError(L.vsb_last_error().decode())
    return out


def boxblur_tile(plane, size, shape):
    """GPU prefilter with a given vector-blur tile shape (0: 256x32,
    1: 128x16, 2: 128x32, 3: 64x32)."""
    L = lib()
    plane = np.ascontiguousarray(plane, dtype=np.uint8)
    H, W = plane.shape
    out = np.empty_like(plane)
    if L.vsb_boxblur_host_tile(ptr(out), ptr(plane), W, H, size, shape) != 0:
        raise RuntimeError(L.vsb_last_error().decode())
    return out


def field_minmax(img, xs, ys, size, bpp=1, channels=1):
    L = lib()
    img = np.ascontiguousarray(img, dtype=np.uint8)
    H = img.shape[0]
    W = img.shape[1] // bpp
    xs = np.ascontiguousarray(xs, np.int16)
    ys = np.ascontiguousarray(ys, np.int16)
    out = np.zeros((len(xs), channels, 2), np.uint8)
    if L.vsb_field_minmax_host(ptr(img), W, H, bpp, channels, ptr(xs), ptr(ys), len(xs), size,
                               ptr(out)) != 0:
        raise RuntimeError(L.vsb_last_error().decode())
    return out


def field_search(curr, prev, xs, ys, size, max_shift, step, ox=None, oy=None, packed_bpp=0,
                 tiles=0):
    """Per-field search results (sad, tx, ty, ok) of the GPU kernel."""
    L = lib()
    curr = np.ascontiguousarray(curr, dtype=np.uint8)
    prev = np.ascontiguousarray(prev, dtype=np.uint8)
    H = curr.shape[0]
    W = curr.shape[1] // (packed_bpp or 1)
    n = len(xs)
    xs = np.ascontiguousarray(xs, np.int16)
    ys = np.ascontiguousarray(ys, np.int16)
    ox = np.ascontiguousarray(ox if ox is not None else np.zeros(n), np.int16)
    oy = np.ascontiguousarray(oy if oy is not None else np.zeros(n), np.int16)
    sad = np.zeros(n, np.uint32)
    tx = np.zeros(n, np.int16)
    ty = np.zeros(n, np.int16)
    ok = np.zeros(n, np.int32)
    if L.vsb_field_search_host(ptr(curr), ptr(prev), W, H, size, max_shift, step, packed_bpp,
                               ptr(xs), ptr(ys), ptr(ox), ptr(oy), n, tiles, ptr(sad), ptr(tx),
                               ptr(ty), ptr(ok)) != 0:
        raise RuntimeError(L.vsb_last_error().decode())
    return sad, tx, ty, ok


def motions_to_transforms(recs, counts, width, height, fov=0.0, smooth_zoom=0):
    """The second pass (vsLocalmotions2Transforms' fit, one GPU warp per
    frame) over frames whose LocalMotions are `recs` (LM_DTYPE), frame k
    holding counts[k] of them in order.  Returns (transforms as
    TRANSFORM_DTYPE, residuals, info[n, 3] = rounds, fields masked for their
    match, fields masked as outliers)."""
    L = lib()
    recs = np.ascontiguousarray(recs, LM_DTYPE)
    counts = np.asarray(counts, np.int64)
    n = len(counts)
    first = np.zeros(n + 1, np.int64)
    first[1:] = np.cumsum(counts)
    if first[-1] != len(recs):
        raise ValueError("counts add up to %d, %d records given" % (first[-1], len(recs)))
    out = np.zeros(n, TRANSFORM_DTYPE)
    resid = np.zeros(n, np.float64)
    info = np.zeros((n, 3), np.int32)
    rc = L.vsb_motions_to_transforms(ptr(recs) if len(recs) else None, ptr(first), n, width,
                                     height, fov, smooth_zoom, ptr(out), ptr(resid), ptr(info))
    if rc != 0:
        raise RuntimeError("second pass failed: %s" % L.vsb_last_error().decode())
    return out, resid, info
