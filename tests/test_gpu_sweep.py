"""The persistent TMA-staged SAD sweep (vsb_sweep.cuh) against the oracle
and the reference: per-field results for every geometry it is compiled for
and several plans of each, ties on flat and periodic frames, window offsets
of every alignment, and whole detect passes forced onto the sweep."""
import os

import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import synthetic as S
from conftest import first_difference, records_equal
from test_gpu_kernels import _blurred_pair, orc_search

pytestmark = pytest.mark.gpu

# (field size, maxShift, step): the defaults' coarse fields of 640x360,
# 640x480, 1280x720, 1920x1080 and their fine fields (1080p and 4K), plus a
# shorter shift range
GEOMS = [(48, 51, 6), (64, 68, 6), (80, 102, 6), (112, 154, 6), (112, 60, 6), (16, 16, 2),
         (32, 32, 2), (48, 48, 2)]


def _fields(w, h, size, ms, step, seed):
    """fields whose window origins cover all 16 byte offsets modulo 16"""
    rng = np.random.default_rng(seed)
    reach = size // 2 + ms + step + 4
    n = 20
    xs = rng.integers(reach, w - reach - 16, n)
    xs[:16] = (xs[:16] & ~15) + np.arange(16)
    ys = rng.integers(reach, h - reach, n)
    ox = rng.integers(-3, 4, n)
    oy = rng.integers(-3, 4, n)
    return (xs.astype(np.int16), ys.astype(np.int16), ox.astype(np.int16), oy.astype(np.int16))


@pytest.mark.parametrize("size,ms,step", GEOMS)
@pytest.mark.parametrize("plan", [-1, -2, -4, -7])
def test_sweep_field_search(size, ms, step, plan):
    w, h = 1280, 720
    if size // 2 + ms + step + 4 > 340:
        w, h = 1920, 1080
    curr, prev = _blurred_pair(w, h, seed=size + step)
    xs, ys, ox, oy = _fields(w, h, size, ms, step, size * 3 + ms)
    try:
        sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, ox, oy, tiles=plan)
    except RuntimeError as e:
        if "no sweep plan of that rank" in str(e):
            pytest.skip(str(e))
        raise
    for k in range(len(xs)):
        exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step, int(ox[k]),
                         int(oy[k]))
        assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2], bool(exp[3])), k


def test_sweep_ties():
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
        for size, ms, step in [(48, 40, 6), (32, 32, 2), (16, 16, 2)]:
            for plan in (-1, -3):
                sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, tiles=plan)
                for k in range(len(xs)):
                    exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step)
                    assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2],
                                                                   bool(exp[3]))


@pytest.fixture
def forced_sweep(monkeypatch):
    monkeypatch.setenv("VSB_FORCE_SWEEP", "1")
    yield


@pytest.mark.parametrize("w,h,n", [(640, 360, 6), (1280, 720, 5), (1920, 1080, 5)])
def test_detect_on_sweep_matches_reference(w, h, n, forced_sweep):
    """whole detect passes on the sweep; the fine plan is sized for every
    fine field, so a frame's fine launch (the selected fields only) has fewer
    tiles than CTAs at 640x360 and empty CTAs lie between the CTAs holding a
    field's tiles"""
    frames = S.clip(w, h, n, seed=w + 7)
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    desc = (O.C.c_int * 8)()
    for fine in (0, 1):
        assert V.lib().vsb_search_tiling(O.C.byref(det.md), fine, desc) == 0
        assert desc[1] == 5, "the detector did not take the sweep"
    got = [det.detect(f) for f in frames]
    det.close()
    got = np.concatenate(got)
    if O.ref_available():
        exp, ec, _ = O.ref_clip(frames, V.PF_YUV420P)
    else:
        exp, ec = O.oracle_clip(frames, V.PF_YUV420P)
    assert records_equal(got, exp), first_difference(got, exp)


def test_overlapped_loop_on_sweep(forced_sweep):
    """both stages on the sweep at once (frame k's fine stage beside frame
    k+1's coarse stage) through the frame loop, against the reference"""
    import torch
    w, h, n = 1920, 1080, 12
    clip = S.clip(w, h, n, seed=91, device="cuda")
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)
    tot = det.run(n, clip.data_ptr(), w * h, w, True, rec, cnt)
    det.close()
    host = clip.cpu().numpy()
    torch.cuda.synchronize()
    if O.ref_available():
        exp, ec, _ = O.ref_clip(host, V.PF_YUV420P)
    else:
        exp, ec = O.oracle_clip(host, V.PF_YUV420P)
    assert np.array_equal(cnt, ec)
    assert records_equal(rec[:tot], exp), first_difference(rec[:tot], exp)
