"""k_fine (vsb_finewarp.cuh), the full search of fine fields with one CTA of
a few warps per field, against the oracle and the reference: per-field
results for the fine geometries of 640x360 to 4K at every CTA size, window
offsets of every alignment, ties on flat and periodic frames, and whole
detect passes forced onto it."""
import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import synthetic as S
from conftest import first_difference, records_equal
from test_gpu_kernels import _blurred_pair, orc_search
from test_gpu_sweep import _fields

pytestmark = pytest.mark.gpu

# (field size, maxShift, step) of the default fine fields: 640x360 / 1280x720,
# 1920x1080, 3840x2160; plus a shorter shift range
FINE = [(16, 16, 2), (32, 32, 2), (48, 48, 2), (32, 20, 2)]


def hook(warps, rows=1, strips=1):
    """the test hook's tiles value of k_fine"""
    return -100 - (warps + (100 * rows if rows > 1 else 0) + (1000 * strips if strips > 1 else 0))


@pytest.mark.parametrize("size,ms,step", FINE)
@pytest.mark.parametrize("warps,rows,strips", [(1, 1, 1), (2, 1, 1), (8, 1, 1), (16, 1, 2),
                                               (8, 1, 4), (1, 2, 1), (4, 2, 2), (16, 2, 4),
                                               (2, 4, 1), (8, 4, 2)])
def test_fine_field_search(size, ms, step, warps, rows, strips):
    """rows: lattice rows per thread (the window rows are walked once for all
    of them); strips: the field rows split over threads, partial sums added"""
    w, h = 1280, 720
    curr, prev = _blurred_pair(w, h, seed=size + warps + rows + strips)
    xs, ys, ox, oy = _fields(w, h, size, ms, step, size * 5 + ms + warps + rows + strips)
    sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, ox, oy,
                                     tiles=hook(warps, rows, strips))
    for k in range(len(xs)):
        exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step, int(ox[k]),
                         int(oy[k]))
        assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2], bool(exp[3])), k


def test_fine_ties():
    """flat, periodic and striped frames: many equal SADs, the visiting order
    decides"""
    w, h = 320, 240
    flat = np.full((h, w), 90, np.uint8)
    yy, xx = np.mgrid[0:h, 0:w]
    periodic = (((xx // 6) + (yy // 6)) % 2 * 60 + 60).astype(np.uint8)
    stripes = ((xx % 12) * 10).astype(np.uint8)
    xs = np.array([100, 161, 222, 143], np.int16)
    ys = np.array([100, 120, 140, 117], np.int16)
    for curr, prev in [(flat, flat), (periodic, periodic), (periodic, np.roll(periodic, 3, 1)),
                       (stripes, stripes)]:
        for size, ms, step in [(32, 32, 2), (16, 16, 2)]:
            for tiles in (hook(2), hook(2, 4), hook(16, 1, 4)):
                sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, tiles=tiles)
                for k in range(len(xs)):
                    exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step)
                    assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2],
                                                                   bool(exp[3])), tiles


@pytest.mark.parametrize("w,h,n", [(640, 360, 5), (1920, 1080, 4), (3840, 2160, 3)])
def test_detect_on_fine_kernel_matches_reference(w, h, n, monkeypatch):
    monkeypatch.setenv("VSB_FORCE_FINEWARP", "1")
    frames = S.clip(w, h, n, seed=w + 11)
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    desc = (O.C.c_int * 8)()
    assert V.lib().vsb_search_tiling(O.C.byref(det.md), 1, desc) == 0
    assert desc[1] == 6, "the detector did not take k_fine"
    got = np.concatenate([det.detect(f) for f in frames])
    det.close()
    if O.ref_available():
        exp, ec, _ = O.ref_clip(np.asarray(frames), V.PF_YUV420P)
    else:
        exp, ec = O.oracle_clip(np.asarray(frames), V.PF_YUV420P)
    assert records_equal(got, exp), first_difference(got, exp)
