"""CPU-only checks of the C ABI library: it loads, exports every function and
variable include/*.h declares, its public structs have the reference's sizes,
its host-side arithmetic is bit-identical to the reference's, and the detect
path refuses to run without a GPU instead of falling back to the CPU."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200._lib import VSFrameInfo, VSVector

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")


def declared_symbols():
    names = set()
    for h in ("vidstab_b200.h", "vidstab_b200_ext.h"):
        src = open(os.path.join(REPO, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = "\n".join(l for l in src.splitlines() if not l.lstrip().startswith("#"))
        for m in re.finditer(r"VS_API\s+[^;{(]*?\b(\w+)\s*\(", src):
            names.add(m.group(1))
        for m in re.finditer(r"extern\s+VS_API\s+[\w\s\*]+?\b(\w+)\s*;", src):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol():
    L = V.lib()
    names = declared_symbols()
    assert len(names) > 80
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


@needs_ref
def test_struct_sizes_match_reference():
    L = V.lib()
    R = O.ref()
    assert L.vsb_sizeof(b"VSMotionDetect") == R.vsref_sizeof_motiondetect()
    assert L.vsb_sizeof(b"LocalMotion") == R.vsref_sizeof_localmotion() == 32
    assert C.sizeof(V._lib.VSMotionDetect) == L.vsb_sizeof(b"VSMotionDetect")
    for t, s in (("VSFrameInfo", 28), ("VSFrame", 48), ("VSTransform", 56), ("Field", 6),
                 ("VSVector", 16)):
        assert L.vsb_sizeof(t.encode()) == s, t


def _motion_vector(L, recs):
    L.vs_vector_init.argtypes = [C.POINTER(VSVector), C.c_int]
    L.vs_vector_append_dup.argtypes = [C.POINTER(VSVector), C.c_void_p, C.c_int]
    v = VSVector()
    L.vs_vector_init(C.byref(v), max(len(recs), 1))
    for k in range(len(recs)):
        L.vs_vector_append_dup(C.byref(v), C.c_void_p(recs.ctypes.data + 32 * k), 32)
    return v


@needs_ref
def test_host_model_bits_match_reference():
    """vsSimpleMotionsToTransform, cleanmean and the fine-search offsets of the
    product library against the reference's own functions"""
    L, R = V.lib(), O.ref()
    R.vsref_cleanmean.restype = C.c_double
    R.vsref_cleanmean.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(11)
    fi = VSFrameInfo()
    L.vsFrameInfoInit(C.byref(fi), 1920, 1080, 0)
    for trial in range(400):
        n = int(rng.integers(1, 80))
        recs = np.zeros(n, O.LM_DTYPE)
        recs["fx"] = rng.integers(60, 1860, n)
        recs["fy"] = rng.integers(60, 1020, n)
        recs["fsize"] = 112
        recs["vx"] = rng.integers(-30, 30, n) + int(rng.integers(-100, 100))
        recs["vy"] = rng.integers(-30, 30, n)
        recs["match"] = rng.random(n) * 20
        v = _motion_vector(L, recs)
        t = L.vsSimpleMotionsToTransform(fi, b"t", C.byref(v))
        L.vs_vector_del(C.byref(v))
        ref = np.zeros(4)
        R.vsref_simple_transform(1920, 1080, recs.ctypes.data_as(C.c_void_p), n,
                                 ref.ctypes.data_as(C.c_void_p))
        assert np.array_equal(np.array([t.x, t.y, t.alpha, t.zoom]), ref)
        d = rng.random(n) * 7
        a, b = d.copy(), d.copy()
        assert L.cleanmean(a.ctypes.data, n, None, None) == R.vsref_cleanmean(
            b.ctypes.data, n, None, None)


def test_trf_roundtrip_host():
    """.trf writer and reader of the product library (no GPU involved)"""
    L = V.lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    L.vsStoreLocalmotions.argtypes = [C.c_void_p, C.POINTER(VSVector), C.c_int]
    L.vsRestoreLocalmotions.argtypes = [C.c_void_p, C.c_int]
    L.vsRestoreLocalmotions.restype = VSVector
    recs = np.zeros(5, V.LM_DTYPE)
    recs["vx"] = [1, -2, 3, 0, 7]
    recs["fx"] = [100, 200, 300, 400, 500]
    recs["fsize"] = 32
    recs["contrast"] = [0.5, 0.25, 0.125, 1.0, 0.75]
    recs["match"] = [1.5, 2.5, 3.25, 0.0, 9.0]
    v = _motion_vector(L, recs)
    with tempfile.TemporaryDirectory() as d:
        for mode in (V.BINARY_SERIALIZATION_MODE, V.ASCII_SERIALIZATION_MODE):
            path = os.path.join(d, "m%d" % mode).encode()
            f = libc.fopen(path, b"wb")
            assert L.vsStoreLocalmotions(f, C.byref(v), mode) == 1
            libc.fclose(f)
            f = libc.fopen(path, b"rb")
            back = L.vsRestoreLocalmotions(f, mode)
            libc.fclose(f)
            got = V._lib.vector_records(back)
            L.vs_vector_del(C.byref(back))
            for k in ("vx", "vy", "fx", "fy", "fsize", "contrast", "match"):
                assert np.array_equal(got[k], recs[k]), (mode, k)
    L.vs_vector_del(C.byref(v))


@pytest.mark.skipif(V.lib().vsb_device_count() > 0, reason="checks the no-GPU behaviour")
def test_no_gpu_fails_loudly():
    with pytest.raises(RuntimeError, match="no CUDA device"):
        V.MotionDetector(640, 480, V.PF_YUV420P)


def test_init_rejects_bad_input():
    """unsupported pixel format and a frame too small for the field layout
    return VS_ERROR before any device work"""
    L = V.lib()
    fi = VSFrameInfo()
    L.vsFrameInfoInit(C.byref(fi), 640, 480, V.PF_YUV420P)
    fi.pFormat = 8  # PF_PACKED marker
    conf = L.vsMotionDetectGetDefaultConfig(b"t")
    md = V._lib.VSMotionDetect()
    assert L.vsMotionDetectInit(C.byref(md), C.byref(conf), C.byref(fi)) == -1
