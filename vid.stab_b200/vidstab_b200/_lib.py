"""ctypes view of libvidstab_b200.so (the C ABI in include/vidstab_b200.h).

The shared library is built in-tree by vid.stab_b200/build.py.  Loading it
never falls back to anything: a missing library raises.
"""
import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(ROOT, "lib", "libvidstab_b200.so")

# pixel formats, src/frameinfo.h:34-48 of the reference
PF_GRAY8, PF_YUV420P, PF_YUV422P, PF_YUV444P = 0, 1, 2, 3
PF_YUV410P, PF_YUV411P, PF_YUV440P, PF_YUVA420P = 4, 5, 6, 7
PF_PACKED, PF_RGB24, PF_BGR24, PF_RGBA = 8, 9, 10, 11
ASCII_SERIALIZATION_MODE, BINARY_SERIALIZATION_MODE = 1, 2

# one LocalMotion record as laid out in memory (32 bytes on x86-64)
LM_DTYPE = np.dtype({"names": ["vx", "vy", "fx", "fy", "fsize", "contrast", "match"],
                     "formats": ["<i2", "<i2", "<i2", "<i2", "<i2", "<f8", "<f8"],
                     "offsets": [0, 2, 4, 6, 8, 16, 24], "itemsize": 32})
assert LM_DTYPE.itemsize == 32


class VSFrameInfo(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("planes", C.c_int),
                ("log2ChromaW", C.c_int), ("log2ChromaH", C.c_int), ("pFormat", C.c_int),
                ("bytesPerPixel", C.c_int)]


class VSFrame(C.Structure):
    _fields_ = [("data", C.c_void_p * 4), ("linesize", C.c_int * 4)]


class VSMotionDetectConfig(C.Structure):
    _fields_ = [("shakiness", C.c_int), ("accuracy", C.c_int), ("stepSize", C.c_int),
                ("algo", C.c_int), ("virtualTripod", C.c_int), ("show", C.c_int),
                ("contrastThreshold", C.c_double), ("modName", C.c_char_p),
                ("numThreads", C.c_int)]


class VSTransform(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("alpha", C.c_double),
                ("zoom", C.c_double), ("barrel", C.c_double), ("rshutter", C.c_double),
                ("extra", C.c_int)]


class Field(C.Structure):
    _fields_ = [("x", C.c_int16), ("y", C.c_int16), ("size", C.c_int16)]


class VSMotionDetectFields(C.Structure):
    _fields_ = [("maxShift", C.c_int), ("stepSize", C.c_int), ("fieldNum", C.c_int),
                ("maxFields", C.c_int), ("contrastThreshold", C.c_double),
                ("fieldSize", C.c_int), ("fieldRows", C.c_int), ("fields", C.POINTER(Field)),
                ("useOffset", C.c_short), ("offset", VSTransform)]


class VSMotionDetect(C.Structure):
    _fields_ = [("fi", VSFrameInfo), ("conf", VSMotionDetectConfig),
                ("fieldscoarse", VSMotionDetectFields), ("fieldsfine", VSMotionDetectFields),
                ("curr", VSFrame), ("currorig", VSFrame), ("currtmp", VSFrame),
                ("prev", VSFrame), ("hasSeenOneFrame", C.c_short), ("initialized", C.c_int),
                ("serializationMode", C.c_int), ("frameNum", C.c_int)]


# VSTransform as an array element (56 bytes + 8 padding on x86-64)
TRANSFORM_DTYPE = np.dtype({"names": ["x", "y", "alpha", "zoom", "barrel", "rshutter", "extra"],
                            "formats": ["<f8", "<f8", "<f8", "<f8", "<f8", "<f8", "<i4"],
                            "offsets": [0, 8, 16, 24, 32, 40, 48], "itemsize": 56})


class VSVector(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_void_p)), ("buffersize", C.c_int), ("nelems", C.c_int)]


class VSTransformConfig(C.Structure):
    """src/transform.h:88-150 of the reference"""
    _fields_ = [("relative", C.c_int), ("smoothing", C.c_int), ("crop", C.c_int),
                ("invert", C.c_int), ("zoom", C.c_double), ("optZoom", C.c_int),
                ("zoomSpeed", C.c_double), ("interpolType", C.c_int), ("maxShift", C.c_int),
                ("maxAngle", C.c_double), ("modName", C.c_char_p), ("verbose", C.c_int),
                ("simpleMotionCalculation", C.c_int), ("storeTransforms", C.c_int),
                ("smoothZoom", C.c_int), ("camPathAlgo", C.c_int),
                ("estimateLensDistortion", C.c_int), ("lensCorrection", C.c_int),
                ("lensK", C.c_double), ("fov", C.c_double)]


class VSLensPlaneMap(C.Structure):
    _fields_ = [("active", C.c_int), ("mode", C.c_int)] + \
        [(n, C.c_double) for n in ("k", "cdx", "cdy", "csx", "csy", "tMaxU", "tMaxD", "tDomD",
                                   "invRho2", "f")] + \
        [("sxShift", C.c_int), ("syShift", C.c_int), ("idxScaleU", C.c_int32),
         ("idxScaleD", C.c_int32), ("gU", C.c_void_p), ("gD", C.c_void_p)]


class VSTransformData(C.Structure):
    """src/transform.h:152-178 of the reference"""
    _fields_ = [("fiSrc", VSFrameInfo), ("fiDest", VSFrameInfo), ("src", VSFrame),
                ("destbuf", VSFrame), ("dest", VSFrame), ("srcMalloced", C.c_short),
                ("interpolate", C.c_void_p), ("conf", VSTransformConfig), ("lensMode", C.c_int),
                ("lensActive", C.c_int), ("lensK", C.c_double), ("lensMapK", C.c_double),
                ("lensMaps", VSLensPlaneMap * 3), ("initialized", C.c_int)]


class VSTransformations(C.Structure):
    _fields_ = [("ts", C.POINTER(VSTransform)), ("current", C.c_int), ("len", C.c_int),
                ("warned_end", C.c_short)]


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libvidstab_b200.so is not built (expected at %s); run vid.stab_b200/build.py" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    i, d, p, u8p = C.c_int, C.c_double, C.c_void_p, C.c_void_p
    L.vsMotionDetectGetDefaultConfig.restype = VSMotionDetectConfig
    L.vsMotionDetectGetDefaultConfig.argtypes = [C.c_char_p]
    L.vsMotionDetectInit.restype = i
    L.vsMotionDetectInit.argtypes = [C.POINTER(VSMotionDetect), C.POINTER(VSMotionDetectConfig),
                                     C.POINTER(VSFrameInfo)]
    L.vsMotionDetection.restype = i
    L.vsMotionDetection.argtypes = [C.POINTER(VSMotionDetect), C.POINTER(VSVector),
                                    C.POINTER(VSFrame)]
    L.vsMotionDetectionCleanup.restype = None
    L.vsMotionDetectionCleanup.argtypes = [C.POINTER(VSMotionDetect)]
    L.vsFrameInfoInit.restype = i
    L.vsFrameInfoInit.argtypes = [C.POINTER(VSFrameInfo), i, i, i]
    L.vs_vector_del.restype = i
    L.vs_vector_del.argtypes = [C.POINTER(VSVector)]
    L.vs_vector_size.restype = i
    L.vs_vector_size.argtypes = [C.POINTER(VSVector)]
    L.vsSimpleMotionsToTransform.restype = VSTransform
    L.vsSimpleMotionsToTransform.argtypes = [VSFrameInfo, C.c_char_p, C.POINTER(VSVector)]
    L.cleanmean.restype = d
    L.cleanmean.argtypes = [p, i, p, p]
    L.vsb_last_error.restype = C.c_char_p
    L.vsb_device_count.restype = i
    L.vsb_sizeof.restype = i
    L.vsb_sizeof.argtypes = [C.c_char_p]
    L.vsb_motion_detection_device.restype = i
    L.vsb_motion_detection_device.argtypes = [C.POINTER(VSMotionDetect), C.POINTER(VSVector),
                                              p, i]
    L.vsb_launch_count.restype = C.c_long
    L.vsb_launch_count.argtypes = [C.POINTER(VSMotionDetect)]
    L.vsb_detect_clip.restype = C.c_long
    L.vsb_detect_clip.argtypes = [i, i, i, p, C.c_long, i, i, i, i, i, i, d, i, i, i,
                                  C.c_char_p, p, C.c_long, p, p, p]
    L.vsb_detect_run.restype = C.c_long
    L.vsb_detect_run.argtypes = [C.POINTER(VSMotionDetect), p, C.c_long, i, i, i, p, C.c_long, p]
    L.vsb_detect_frames.restype = C.c_long
    L.vsb_detect_frames.argtypes = [C.POINTER(VSMotionDetect), p, C.c_long, i, i, i, p, C.c_long,
                                    p]
    L.vsb_batch_create.restype = p
    L.vsb_batch_create.argtypes = [i, p, p, i, p]
    L.vsb_batch_detect.restype = i
    L.vsb_batch_detect.argtypes = [p, p, p, i, p]
    L.vsb_batch_run.restype = C.c_long
    L.vsb_batch_run.argtypes = [p, p, p, p, i, i, p, C.c_long, p]
    L.vsb_batch_free.restype = None
    L.vsb_batch_free.argtypes = [p]
    L.vsb_batch_launch_count.restype = C.c_long
    L.vsb_batch_launch_count.argtypes = [p]
    L.vsb_batch_grid.restype = i
    L.vsb_batch_grid.argtypes = [p, p, p, p]
    L.vsb_batch_class.restype = i
    L.vsb_batch_class.argtypes = [p, i, p]
    L.vsb_batch_open_trf.restype = i
    L.vsb_batch_open_trf.argtypes = [p, p, i]
    L.vsb_batch_close_trf.restype = i
    L.vsb_batch_close_trf.argtypes = [p]
    L.vsb_batch_set_wait_limit.argtypes = [p, C.c_uint, C.c_longlong]
    L.vsb_batch_test_withhold_blur.argtypes = [p, i]
    L.vsb_batch_set_proposal.restype = i
    L.vsb_batch_set_proposal.argtypes = [p, p, C.c_long]
    L.vsb_batch_proposal_stats.restype = i
    L.vsb_batch_proposal_stats.argtypes = [p, p]
    L.vsb_test_device_alloc.restype = C.c_longlong
    L.vsb_test_device_alloc.argtypes = [i, i]
    L.vsb_boxblur_host.restype = i
    L.vsb_boxblur_host.argtypes = [p, p, i, i, i]
    L.vsb_boxblur_host_tile.restype = i
    L.vsb_boxblur_host_tile.argtypes = [p, p, i, i, i, i]
    L.vsb_blur_tiling.restype = i
    L.vsb_blur_tiling.argtypes = [C.POINTER(VSMotionDetect), p]
    L.vsb_field_minmax_host.restype = i
    L.vsb_field_minmax_host.argtypes = [p, i, i, i, i, p, p, i, i, p]
    L.vsb_field_search_host.restype = i
    L.vsb_field_search_host.argtypes = [p, p, i, i, i, i, i, i, p, p, p, p, i, i, p, p, p, p]
    L.vsLocalmotions2Transforms.restype = i
    L.vsLocalmotions2Transforms.argtypes = [C.POINTER(VSTransformData), C.POINTER(VSVector),
                                            C.POINTER(VSTransformations)]
    L.vsMotionsToTransform.restype = VSTransform
    L.vsMotionsToTransform.argtypes = [C.POINTER(VSTransformData), C.POINTER(VSVector), p]
    L.vsb_transform_layout.restype = i
    L.vsb_transform_layout.argtypes = [p, i]
    L.vsb_motions_to_transforms.restype = i
    L.vsb_motions_to_transforms.argtypes = [p, p, i, i, i, d, i, p, p, p]
    L.vsb_motions_to_transforms_device.restype = i
    L.vsb_motions_to_transforms_device.argtypes = [p, p, i, i, i, i, d, i, p, p, p, p]
    L.vsb_motions_to_transforms_capacity.restype = i
    L.vsb_motions_to_transforms_launches.restype = C.c_long
    _lib = L
    return L


def ptr(a):
    """Address of a numpy array's data (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def vector_records(v):
    """Copies the LocalMotions of a VSVector into a structured numpy array."""
    n = v.nelems
    out = np.zeros(n, dtype=LM_DTYPE)
    raw = out.view(np.uint8).reshape(n, 32) if n else None
    for k in range(n):
        C.memmove(raw[k].ctypes.data, v.data[k], 32)
    return out
