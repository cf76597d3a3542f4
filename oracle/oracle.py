"""TEST INFRASTRUCTURE ONLY: Python access to the CPU checkers.

* the C restatement of the detect pass (oracle/liboracle.so, vsoracle.c);
* the unmodified reference library compiled from its sources
  (oracle/_ref/libvidstab_ref.so through oracle/_ref/libvsref_driver.so),
  available wherever `make -C oracle` ran with the reference sources present
  (the built files travel with the repository snapshot).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_DRIVER = os.path.join(REF_DIR, "libvsref_driver.so")

LM_DTYPE = np.dtype({"names": ["vx", "vy", "fx", "fy", "fsize", "contrast", "match"],
                     "formats": ["<i2", "<i2", "<i2", "<i2", "<i2", "<f8", "<f8"],
                     "offsets": [0, 2, 4, 6, 8, 16, 24], "itemsize": 32})

_orc = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def build():
    """Compiles the oracle (and the reference, when its sources exist)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        i, d, p = C.c_int, C.c_double, C.c_void_p
        L.orc_blur_size.restype = i
        L.orc_blur_size.argtypes = [i, i, i]
        L.orc_blur_hori.argtypes = [p, i, p, i, i, i, i]
        L.orc_blur_vert.argtypes = [p, i, p, i, i, i, i]
        L.orc_blur_luma.argtypes = [p, i, p, i, i, i, i]
        L.orc_sad.restype = C.c_uint32
        L.orc_sad.argtypes = [p, i, p, i, i, i, i, i, i, i]
        L.orc_minmax.argtypes = [p, i, i, i, i, i, p, p]
        L.orc_contrast_from_minmax.restype = d
        L.orc_contrast_from_minmax.argtypes = [i, i]
        L.orc_spiral.restype = i
        L.orc_spiral.argtypes = [i, i, p, p, i]
        L.orc_search_planar.restype = i
        L.orc_search_planar.argtypes = [p, i, p, i, i, i, i, i, i, i, i, p, p, p]
        L.orc_search_packed.restype = i
        L.orc_search_packed.argtypes = [p, i, p, i, i, i, i, i, i, i, i, i, p, p, p]
        L.orc_md_new.restype = p
        L.orc_md_new.argtypes = [i, i, i, i, i, i, d, i]
        L.orc_md_frame.restype = i
        L.orc_md_frame.argtypes = [p, p, i, p, i]
        L.orc_md_free.argtypes = [p]
        L.orc_md_curr.restype = p
        L.orc_md_curr.argtypes = [p]
        L.orc_simple_transform.argtypes = [i, i, p, i, p]
        L.orc_cleanmean.restype = d
        L.orc_cleanmean.argtypes = [p, i, p, p]
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_DRIVER)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference build not present (run make -C oracle where the "
                               "reference sources exist)")
        C.CDLL(os.path.join(REF_DIR, "libvidstab_ref.so"), mode=C.RTLD_GLOBAL)
        L = C.CDLL(REF_DRIVER)
        i, d, p, u = C.c_int, C.c_double, C.c_void_p, C.c_uint
        L.vsref_detect_clip.restype = C.c_long
        L.vsref_detect_clip.argtypes = [i, i, i, p, C.c_long, i, i, i, i, i, d, i, i, i, i,
                                        C.c_char_p, p, C.c_long, p, p, p]
        L.vsref_boxblur_plane.argtypes = [p, i, p, i, i, i, i]
        L.vsref_boxblur_hori.argtypes = [p, p, i, i, i, i, i]
        L.vsref_boxblur_vert.argtypes = [p, p, i, i, i, i, i]
        L.vsref_sad.restype = u
        L.vsref_sad.argtypes = [p, p, i, i, i, i, i, i, i, i, u]
        L.vsref_sad_dispatch.restype = u
        L.vsref_sad_dispatch.argtypes = [p, p, i, i, i, i, i, i, i, i, u]
        L.vsref_contrast.restype = d
        L.vsref_contrast.argtypes = [p, i, i, i, i, i]
        L.vsref_simd_name.restype = C.c_char_p
        L.vsref_field_layout.restype = i
        L.vsref_field_layout.argtypes = [i, i, i, i, i, p, i, p]
        L.vsref_field_search.restype = d
        L.vsref_field_search.argtypes = [p, p, i, i, i, i, i, i, i, p, p]
        L.vsref_simple_transform.argtypes = [i, i, p, i, p]
        L.vsref_sizeof_localmotion.restype = i
        L.vsref_sizeof_motiondetect.restype = i
        _ref = L
    return _ref


def _bpp(pformat):
    return 1 if pformat < 8 else (4 if pformat == 11 else 3)


class OracleDetector:
    """The C restatement of vsMotionDetectInit/vsMotionDetection."""

    def __init__(self, width, height, pformat=1, stepsize=6, accuracy=15, shakiness=5,
                 mincontrast=0.25, tripod=0):
        L = orc()
        self.L = L
        self.h = L.orc_md_new(width, height, pformat, stepsize, accuracy, shakiness, mincontrast,
                              tripod)
        if not self.h:
            raise ValueError("unsupported configuration")
        self.width, self.height, self.bpp = width, height, _bpp(pformat)

    def detect(self, plane0):
        plane0 = np.ascontiguousarray(plane0, np.uint8)
        out = np.zeros(4096, LM_DTYPE)
        n = self.L.orc_md_frame(self.h, _p(plane0), plane0.strides[0], _p(out), len(out))
        return out[:n].copy()

    def blurred(self):
        ptr = self.L.orc_md_curr(self.h)
        buf = (C.c_uint8 * (self.width * self.bpp * self.height)).from_address(ptr)
        return np.frombuffer(buf, np.uint8).reshape(self.height, self.width * self.bpp).copy()

    def close(self):
        if self.h:
            self.L.orc_md_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def oracle_clip(frames, pformat=1, **kw):
    det = OracleDetector(frames.shape[2] // _bpp(pformat), frames.shape[1], pformat, **kw)
    recs, counts = [], []
    for f in frames:
        r = det.detect(f)
        recs.append(r)
        counts.append(len(r))
    det.close()
    return (np.concatenate(recs) if recs else np.zeros(0, LM_DTYPE)), np.array(counts, np.int32)


def records_per_frame(width, height):
    """an upper bound of the LocalMotions one frame can give: every coarse
    and every fine field (fine fields are at least 16 pixels apart)"""
    return 256 + (width // 16 + 1) * (height // 16 + 1)


def ref_clip(frames, pformat=1, stepsize=6, accuracy=15, shakiness=5, mincontrast=0.25, tripod=0,
             show=0, threads=1, serialization_mode=0, trf_path=None, return_frames=False):
    """The unmodified reference's public detect API over a clip (CPU)."""
    L = ref()
    frames = np.ascontiguousarray(frames, np.uint8)
    n, H = frames.shape[0], frames.shape[1]
    W = frames.shape[2] // _bpp(pformat)
    cap = n * records_per_frame(W, H) + 64
    out = np.zeros(cap, LM_DTYPE)
    counts = np.zeros(n, np.int32)
    el = C.c_double(0)
    drawn = np.zeros((n, frames[0].nbytes), np.uint8) if (show and return_frames) else None
    total = L.vsref_detect_clip(W, H, pformat, _p(frames), frames[0].nbytes, frames.shape[2], n,
                                stepsize, accuracy, shakiness, mincontrast, tripod, show, threads,
                                serialization_mode, trf_path.encode() if trf_path else None,
                                _p(out), cap, _p(counts), C.byref(el), _p(drawn))
    if total < 0:
        raise RuntimeError("reference detect failed")
    if total > cap:
        raise RuntimeError("reference detect: %d records do not fit the buffer of %d" % (total, cap))
    res = (out[:total].copy(), counts, el.value)
    if return_frames:
        res = res + (drawn,)
    return res


def ref_field_layout(width, height, stepsize=6, accuracy=15, shakiness=5):
    L = ref()
    xy = np.zeros((8192, 2), np.int16)
    info = np.zeros(12, np.int32)
    n = L.vsref_field_layout(width, height, stepsize, accuracy, shakiness, _p(xy), 8192, _p(info))
    return xy[:n].copy(), info
