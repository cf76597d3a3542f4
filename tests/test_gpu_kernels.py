"""GPU kernels through the C ABI against the oracle, bit for bit."""
import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import synthetic as S
from conftest import first_difference, records_equal

pytestmark = pytest.mark.gpu


def _p(a):
    return a.ctypes.data_as(O.C.c_void_p)


def orc_blur(src, size):
    h, w = src.shape
    L = O.orc()
    tmp = np.empty_like(src)
    out = np.empty_like(src)
    L.orc_blur_hori(_p(tmp), w, _p(src), w, w, h, size)
    L.orc_blur_vert(_p(out), w, _p(tmp), w, w, h, size)
    return out


def test_blur_geometry_sweep():
    """the geometry sweep of the reference's tests/test_boxblur.c:135-195,
    both passes fused on the GPU vs the two oracle passes"""
    widths = [1, 2, 7, 16, 17, 31, 64, 100, 127, 256, 300]
    heights = [4, 5, 16, 33, 64, 127, 560]
    sizes = [3, 5, 7, 9, 15, 31, 65, 67, 265, 267]
    n = 0
    for w in widths:
        for h in heights:
            for size in sizes:
                if size // 2 >= w or size // 2 >= h:
                    continue
                i = np.arange(w * h)
                src = ((i * 37 + (i // w) * 11 + (i % w) * 7) & 0xFF).astype(np.uint8).reshape(h, w)
                got = V.boxblur(src, size)
                exp = orc_blur(src, size)
                assert np.array_equal(got, exp), (w, h, size)
                n += 1
    assert n > 300


@pytest.mark.parametrize("shape", [0, 1, 2, 3])
def test_blur_tile_shapes(shape):
    """every tile shape the blur autotuner picks from, frame sizes that leave
    ragged edge tiles and box sizes 3 to 17, against the oracle"""
    rng = np.random.default_rng(shape)
    for w, h in [(1920, 1080), (640, 360), (333, 201), (96, 70), (1280, 720)]:
        src = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
        for size in (3, 5, 7, 9, 13, 17):
            got = V.boxblur_tile(src, size, shape)
            assert np.array_equal(got, orc_blur(src, size)), (w, h, size)


@pytest.mark.parametrize("w,h,step", [(1920, 1080, 6), (640, 480, 6), (3840, 2160, 6),
                                      (1280, 720, 14), (333, 201, 3)])
def test_blur_frame(w, h, step):
    rng = np.random.default_rng(w + h)
    src = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    size = O.orc().orc_blur_size(step, w, h)
    got = V.boxblur(src, size)
    exp = np.empty_like(src)
    O.orc().orc_blur_luma(_p(exp), w, _p(src), w, w, h, step)
    assert np.array_equal(got, exp)
    if O.ref_available():
        ref = np.empty_like(src)
        O.ref().vsref_boxblur_plane(_p(ref), w, _p(src), w, w, h, step)
        assert np.array_equal(got, ref)


def test_field_minmax():
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, size=(480, 640), dtype=np.uint8)
    img[100:200, 100:300] = 77
    for size in (16, 32, 48, 64, 112):
        xs = rng.integers(size // 2, 640 - size // 2, 40).astype(np.int16)
        ys = rng.integers(size // 2, 480 - size // 2, 40).astype(np.int16)
        xs[0], ys[0] = 150, 150  # inside the flat block for small sizes
        got = V.field_minmax(img, xs, ys, size)
        for k in range(len(xs)):
            mn, mx = O.C.c_uint8(), O.C.c_uint8()
            O.orc().orc_minmax(_p(img), 640, int(xs[k]), int(ys[k]), size, 1, O.C.byref(mn),
                               O.C.byref(mx))
            assert (got[k, 0, 0], got[k, 0, 1]) == (mn.value, mx.value)


def test_field_minmax_packed():
    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, size=(240, 320 * 4), dtype=np.uint8)
    xs = np.array([40, 100, 200, 280], np.int16)
    ys = np.array([40, 120, 100, 200], np.int16)
    got = V.field_minmax(img, xs, ys, 32, bpp=4, channels=3)
    for k in range(4):
        for ch in range(3):
            mn, mx = O.C.c_uint8(), O.C.c_uint8()
            O.orc().orc_minmax(_p(img[:, ch:]), 320 * 4, int(xs[k]), int(ys[k]), 32, 4,
                               O.C.byref(mn), O.C.byref(mx))
            assert (got[k, ch, 0], got[k, ch, 1]) == (mn.value, mx.value)


def _blurred_pair(w, h, seed, shift=(3, -2)):
    fr = S.clip(w, h, 2, seed=seed, trans_sigma=4.0)
    return fr[1], fr[0]


def orc_search(curr, prev, x, y, size, ms, step, ox=0, oy=0, bpp=0):
    tx, ty, e = O.C.c_int(), O.C.c_int(), O.C.c_uint32()
    ls = curr.shape[1]
    if bpp:
        ok = O.orc().orc_search_packed(_p(curr), ls, _p(prev), ls, x, y, size, bpp, ms, step, ox,
                                       oy, O.C.byref(tx), O.C.byref(ty), O.C.byref(e))
    else:
        ok = O.orc().orc_search_planar(_p(curr), ls, _p(prev), ls, x, y, size, ms, step, ox, oy,
                                       O.C.byref(tx), O.C.byref(ty), O.C.byref(e))
    return e.value, tx.value, ty.value, ok


def enc(tb, strips, nab, nbb, ta=0):
    """forced tiling: rows per thread, field strips, lattice columns / rows per
    CTA, layout (1 one column per thread, 2 two columns with shifts, 3 two
    columns from aligned window copies, 4 two columns from one window copy
    and a field copy shifted by two bytes)"""
    return ta * 100000000 + tb * 1000000 + strips * 10000 + nab * 100 + nbb


@pytest.mark.parametrize("size,ms,step,tiles", [(64, 40, 6, 0), (32, 32, 2, 0),
                                                (112, 60, 6, enc(4, 2, 7, 8)),
                                                (48, 30, 4, enc(2, 4, 5, 6)),
                                                (16, 16, 2, enc(8, 1, 17, 16)),
                                                (80, 45, 5, 0), (32, 20, 1, enc(4, 8, 41, 4)),
                                                (48, 33, 7, enc(8, 2, 3, 8)), (224, 40, 6, 0),
                                                (112, 154, 6, 0), (32, 32, 2, enc(4, 1, 33, 36)),
                                                (112, 60, 6, enc(4, 2, 8, 8, 2)),
                                                (112, 154, 6, enc(2, 4, 14, 10, 2)),
                                                (48, 30, 4, enc(2, 4, 6, 6, 2)),
                                                (32, 32, 2, enc(4, 1, 34, 36, 2)),
                                                (48, 33, 7, enc(4, 2, 4, 8, 2)),
                                                (32, 20, 1, enc(2, 8, 42, 4, 2)),
                                                (64, 40, 6, enc(2, 1, 2, 2, 2)),
                                                (112, 60, 6, enc(4, 2, 8, 8, 3)),
                                                (112, 154, 6, enc(2, 4, 12, 10, 3)),
                                                (48, 30, 4, enc(2, 4, 6, 6, 3)),
                                                (32, 32, 2, enc(4, 1, 36, 36, 3)),
                                                (48, 32, 8, enc(2, 2, 6, 8, 3)),
                                                (64, 40, 6, enc(2, 1, 4, 2, 3)),
                                                (224, 40, 6, enc(2, 4, 8, 6, 3)),
                                                (16, 16, 2, enc(4, 2, 4, 4, 3)),
                                                (112, 60, 6, enc(4, 2, 8, 8, 4)),
                                                (112, 154, 6, enc(2, 4, 12, 10, 4)),
                                                (32, 32, 2, enc(4, 1, 36, 36, 4)),
                                                (64, 40, 6, enc(2, 1, 4, 2, 4)),
                                                (224, 40, 6, enc(2, 4, 12, 14, 4)),
                                                (16, 16, 2, enc(4, 2, 4, 4, 4)),
                                                (80, 45, 6, enc(2, 2, 16, 14, 4))])
def test_field_search_planar(size, ms, step, tiles):
    w, h = 640, 480
    curr, prev = _blurred_pair(w, h, seed=size + step)
    rng = np.random.default_rng(size * 7 + ms)
    reach = size // 2 + ms + step + 4
    if 2 * reach >= h:
        w, h = 1280, 720
        curr, prev = _blurred_pair(w, h, seed=size + step)
    n = 24
    xs = rng.integers(reach, w - reach, n).astype(np.int16)
    ys = rng.integers(reach, h - reach, n).astype(np.int16)
    ox = rng.integers(-3, 4, n).astype(np.int16)
    oy = rng.integers(-3, 4, n).astype(np.int16)
    sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, ox, oy, tiles=tiles)
    for k in range(n):
        exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step, int(ox[k]), int(oy[k]))
        assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2], bool(exp[3])), k


def test_field_search_ties():
    """flat and periodic frames: many equal SADs, the visiting order decides"""
    w, h = 320, 240
    flat = np.full((h, w), 90, np.uint8)
    yy, xx = np.mgrid[0:h, 0:w]
    periodic = (((xx // 6) + (yy // 6)) % 2 * 60 + 60).astype(np.uint8)
    stripes = ((xx % 12) * 10).astype(np.uint8)
    xs = np.array([100, 160, 220], np.int16)
    ys = np.array([100, 120, 140], np.int16)
    for curr, prev in [(flat, flat), (periodic, periodic), (periodic, np.roll(periodic, 3, 1)),
                       (stripes, stripes)]:
        for size, ms, step in [(32, 30, 6), (32, 32, 2), (16, 16, 2)]:
            for tiles in (enc(4, 2, 5, 4), enc(4, 2, 8, 4, 3), enc(4, 2, 8, 4, 4)):
                sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, tiles=tiles)
                for k in range(3):
                    exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step)
                    assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2],
                                                                   bool(exp[3]))


@pytest.mark.parametrize("bpp", [3, 4])
def test_field_search_packed(bpp):
    w, h = 320, 240
    curr_l, prev_l = _blurred_pair(w, h, seed=11 + bpp)
    curr = S.to_packed(curr_l, bpp)
    prev = S.to_packed(prev_l, bpp)
    xs = np.array([90, 160, 230, 120], np.int16)
    ys = np.array([90, 120, 150, 130], np.int16)
    # the aligned two-column layout serves packed rows too (step 2: 6 or 8
    # bytes per lattice step)
    cases = [(32, 34, 6, 0), (16, 16, 2, 0), (16, 16, 2, enc(2, 2, 8, 4, 3))]
    if bpp == 3:  # 6 bytes per lattice step: the shifted-field layout too
        cases.append((16, 16, 2, enc(2, 2, 8, 4, 4)))
    for size, ms, step, tiles in cases:
        sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, ms, step, packed_bpp=bpp,
                                         tiles=tiles)
        for k in range(len(xs)):
            exp = orc_search(curr, prev, int(xs[k]), int(ys[k]), size, ms, step, bpp=bpp)
            assert (sad[k], tx[k], ty[k], bool(ok[k])) == (exp[0], exp[1], exp[2], bool(exp[3]))


def test_sad_peak_probe():
    d = O.C.c_double()
    assert V.lib().vsb_sad_peak(0, O.C.byref(d)) == 0
    assert d.value > 1e12


@pytest.mark.parametrize("w,h,step", [(642, 482, 6), (1000, 562, 4), (1282, 722, 8),
                                      (1921, 1081, 2), (800, 600, 5)])
def test_fused_prefilter_matches_two_launch_path(w, h, step, monkeypatch):
    """k_blurmm (blur + every field's min/max in one launch, box half-widths
    1..4) against the two-launch path (VSB_NO_BLURMM) and the reference, on
    frames whose width and height are not multiples of the 128 x 16 warp
    block (ragged last blocks, edge words loaded and stored bytewise)"""
    frames = S.clip(w, h, 3, seed=w + h)
    fused, fc, _ = V.detect_clip(frames, V.PF_GRAY8, stepsize=step)
    monkeypatch.setenv("VSB_NO_BLURMM", "1")
    two, tc, _ = V.detect_clip(frames, V.PF_GRAY8, stepsize=step)
    monkeypatch.delenv("VSB_NO_BLURMM")
    assert np.array_equal(fc, tc) and records_equal(fused, two), first_difference(fused, two)
    if O.ref_available():
        ref, rc, _ = O.ref_clip(np.asarray(frames), V.PF_GRAY8, stepsize=step)
        assert np.array_equal(fc, rc) and records_equal(fused, ref), first_difference(fused, ref)
