"""The second pass (local motions -> one transform per frame,
src/localmotion2transform.c:40-330 of the reference) on the CPU: the oracle
restatement against the committed reference outputs and against the live
reference build, the ABI of the structures it reads, and the host-only
paths of the drop-in entry point (no GPU needed)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import transform_oracle as T
import vidstab_b200 as V
from vidstab_b200 import _lib
from vidstab_b200 import synthetic as S

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "transforms.npz")
TD = np.dtype([("x", "<f8"), ("y", "<f8"), ("alpha", "<f8"), ("zoom", "<f8"),
               ("barrel", "<f8"), ("rshutter", "<f8"), ("extra", "<i4"), ("pad", "<i4")])


def golden_cases():
    """(label, records, first, width, height, fov, smooth_zoom, reference rows)"""
    g = np.load(GOLDEN)
    cases = []
    for name in ("clip640", "clip1080"):
        recs, counts = g[name + "_recs"], g[name + "_counts"]
        W, H = (int(v) for v in g[name + "_geom"])
        first = np.zeros(len(counts) + 1, np.int64)
        first[1:] = np.cumsum(counts)
        for ci, (fov, sz) in enumerate(g["configs"]):
            cases.append(("%s/%d" % (name, ci), recs, first, W, H, float(fov), int(sz),
                          g["%s_ref%d" % (name, ci)]))
    for si, nm in enumerate(g["edge_names"]):
        r = g["edge%d_recs" % si]
        W, H = (int(v) for v in g["edge%d_geom" % si])
        for ci, (fov, sz) in enumerate(g["configs"]):
            cases.append(("%s/%d" % (nm, ci), r, np.array([0, len(r)], np.int64), W, H,
                          float(fov), int(sz), g["edge%d_ref%d" % (si, ci)]))
    return cases


def test_oracle_matches_golden():
    """every committed case, bit for bit (x, y, alpha, zoom, extra)"""
    n = 0
    for label, recs, first, W, H, fov, sz, ref in golden_cases():
        mine, _ = T.motions_to_transforms(recs, first, W, H, fov, sz)
        assert np.array_equal(mine, ref), label
        n += len(ref)
    assert n >= 100


def test_golden_covers_the_edge_cases():
    g = np.load(GOLDEN)
    names = list(g["edge_names"])
    assert {"empty", "one", "two", "translation_equal_match", "moving_object", "no_model",
            "4k_825"} <= set(names)
    # a frame without motions is flagged, as is one no model fits
    assert g["edge%d_ref0" % names.index("empty")][0, 4] == 1
    assert g["edge%d_ref0" % names.index("no_model")][0, 4] == 1
    assert g["edge%d_ref0" % names.index("moving_object")][0, 4] == 0
    # smoothZoom keeps the fitted zoom, the default drops it
    assert np.any(g["clip640_ref1"][:, 3] != 0) and np.all(g["clip640_ref0"][:, 3] == 0)


def ref_transforms(recs, first, W, H, fov, sz, simple=0):
    R = O.ref()
    R.vsref_motions_to_transforms.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                              C.c_double, C.c_int, C.c_int, C.c_void_p,
                                              C.c_void_p]
    out = np.zeros(len(first) - 1, TD)
    el = C.c_double()
    assert R.vsref_motions_to_transforms(W, H, recs.ctypes.data if len(recs) else None,
                                         first.ctypes.data, len(first) - 1, fov, sz, simple,
                                         out.ctypes.data, C.byref(el)) == 0
    return np.stack([out["x"], out["y"], out["alpha"], out["zoom"],
                     out["extra"].astype(np.float64)], 1)


@needs_ref
def test_oracle_matches_live_reference():
    """a clip the fixture does not hold (640x360, another seed), every model"""
    frames = np.asarray(S.clip(640, 360, 6, seed=29))
    recs, counts, _ = O.ref_clip(frames)
    first = np.zeros(len(counts) + 1, np.int64)
    first[1:] = np.cumsum(counts)
    for fov, sz in ((0.0, 0), (0.0, 1), (60.0, 1), (120.0, 0)):
        mine, _ = T.motions_to_transforms(recs, first, 640, 360, fov, sz)
        assert np.array_equal(mine, ref_transforms(recs, first, 640, 360, fov, sz)), (fov, sz)


@needs_ref
def test_transform_layout_matches_reference():
    L, R = V.lib(), O.ref()
    R.vsref_transform_layout.argtypes = [C.c_void_p, C.c_int]
    a = np.zeros(32, np.int64)
    b = np.zeros(32, np.int64)
    n = L.vsb_transform_layout(a.ctypes.data, 32)
    assert n == R.vsref_transform_layout(b.ctypes.data, 32) and n >= 16
    assert np.array_equal(a[:n], b[:n])
    assert C.sizeof(_lib.VSTransformData) == a[0] == L.vsb_sizeof(b"VSTransformData")
    assert C.sizeof(_lib.VSTransformConfig) == a[1] == L.vsb_sizeof(b"VSTransformConfig")
    assert C.sizeof(_lib.VSTransformations) == a[2] == L.vsb_sizeof(b"VSTransformations")
    assert _lib.VSTransformData.conf.offset == a[4]
    assert _lib.VSTransformConfig.fov.offset == a[13]


def many_motions(L, recs, first):
    """a VSManyLocalMotions (vector of LocalMotions vectors) over the records"""
    L.vs_vector_init.argtypes = [C.POINTER(_lib.VSVector), C.c_int]
    L.vs_vector_append_dup.argtypes = [C.POINTER(_lib.VSVector), C.c_void_p, C.c_int]
    L.vs_vector_get.restype = C.c_void_p
    L.vs_vector_get.argtypes = [C.POINTER(_lib.VSVector), C.c_int]
    mlms = _lib.VSVector()
    L.vs_vector_init(C.byref(mlms), max(len(first) - 1, 1))
    for k in range(len(first) - 1):
        lms = _lib.VSVector()
        n = int(first[k + 1] - first[k])
        L.vs_vector_init(C.byref(lms), max(n, 1))
        for i in range(first[k], first[k + 1]):
            L.vs_vector_append_dup(C.byref(lms), recs.ctypes.data + 32 * int(i), 32)
        L.vs_vector_append_dup(C.byref(mlms), C.addressof(lms), C.sizeof(_lib.VSVector))
    return mlms


def free_many(L, mlms):
    for k in range(L.vs_vector_size(C.byref(mlms))):
        L.vs_vector_del(C.cast(L.vs_vector_get(C.byref(mlms), k), C.POINTER(_lib.VSVector)))
    L.vs_vector_del(C.byref(mlms))


def transform_data(width, height, fov=0.0, smooth_zoom=0, simple=0, lens=0, store=0):
    td = _lib.VSTransformData()
    V.lib().vsFrameInfoInit(C.byref(td.fiSrc), width, height, 1)
    td.fiDest = td.fiSrc
    c = td.conf
    c.modName = b"vidstab_b200"
    c.smoothing, c.maxShift, c.maxAngle, c.optZoom, c.zoomSpeed = 15, -1, -1.0, 1, 0.25
    c.interpolType, c.camPathAlgo = 2, 1
    c.fov, c.smoothZoom, c.simpleMotionCalculation = fov, smooth_zoom, simple
    c.estimateLensDistortion, c.storeTransforms = lens, store
    return td


def test_lens_estimate_is_refused():
    """the lens-distortion estimate (src/localmotion2transform.c:59-105) is not
    part of this library: asked for it, the call fails before any work"""
    L = V.lib()
    recs = np.load(GOLDEN)["clip640_recs"][:50]
    mlms = many_motions(L, recs, np.array([0, 50], np.int64))
    td = transform_data(640, 480, lens=1)
    tr = _lib.VSTransformations()
    try:
        assert L.vsLocalmotions2Transforms(C.byref(td), C.byref(mlms), C.byref(tr)) != 0
        assert not tr.ts and tr.len == 0
        assert b"lens-distortion" in L.vsb_last_error()
    finally:
        free_many(L, mlms)


@needs_ref
def test_simple_motion_calculation_matches_reference():
    """conf.simpleMotionCalculation: vsSimpleMotionsToTransform per frame on
    the host, bit for bit with the reference's vsLocalmotions2Transforms"""
    L = V.lib()
    g = np.load(GOLDEN)
    recs, counts = g["clip640_recs"], g["clip640_counts"]
    first = np.zeros(len(counts) + 1, np.int64)
    first[1:] = np.cumsum(counts)
    mlms = many_motions(L, recs, first)
    td = transform_data(640, 480, simple=1, lens=1)
    tr = _lib.VSTransformations()
    try:
        assert L.vsLocalmotions2Transforms(C.byref(td), C.byref(mlms), C.byref(tr)) == 0
        assert tr.len == len(counts)
        mine = np.array([[tr.ts[k].x, tr.ts[k].y, tr.ts[k].alpha, tr.ts[k].zoom, tr.ts[k].extra]
                         for k in range(tr.len)])
        C.CDLL(None).free(C.cast(tr.ts, C.c_void_p))
    finally:
        free_many(L, mlms)
    ref = ref_transforms(recs, first, 640, 480, 0.0, 0, simple=1)
    assert np.array_equal(mine, ref)
