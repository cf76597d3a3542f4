"""The whole detect pass through the C ABI (vsMotionDetectInit /
vsMotionDetection) against the unmodified reference compiled from its
sources (oracle/_ref) and the oracle restatement: LocalMotions equal in
count, order and all seven fields, .trf files byte-identical."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import synthetic as S
from conftest import first_difference, records_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["pruned", "dense"])
def search(request):
    """runs a test under both search strategies of the library"""
    V.lib().vsb_set_default_search_mode(1 if request.param == "pruned" else 0)
    yield request.param
    V.lib().vsb_set_default_search_mode(-1)


def expected(frames, pformat=1, **kw):
    """reference output where the reference build exists, else the oracle"""
    if O.ref_available():
        r, c, _ = O.ref_clip(frames, pformat, **kw)
        return r, c
    kw2 = {k: v for k, v in kw.items() if k in ("stepsize", "accuracy", "shakiness",
                                                 "mincontrast", "tripod")}
    return O.oracle_clip(frames, pformat, **kw2)


def check(frames, pformat=1, **kw):
    got, gc, _ = V.detect_clip(frames, pformat, **kw)
    exp, ec = expected(frames, pformat, **kw)
    assert np.array_equal(gc, ec), (gc, ec)
    assert records_equal(got, exp), first_difference(got, exp)
    return got, gc


@pytest.mark.parametrize("seed", range(6))
def test_cfg0_pair(seed, search):
    A, B, _ = S.pair(640, 480, seed=seed)
    got, counts = check(np.stack([A, B]), V.PF_YUV420P)
    assert counts[0] == 0 and counts[1] > 20


@pytest.mark.parametrize("w,h,n", [(640, 360, 8), (1280, 720, 5), (1920, 1080, 4)])
def test_clip(w, h, n, search):
    frames = S.clip(w, h, n, seed=w)
    check(frames, V.PF_YUV420P)


def test_clip_4k(search):
    frames = S.clip(3840, 2160, 3, seed=4, trans_sigma=8.0, rot_sigma_deg=0.5)
    check(frames, V.PF_YUV420P, shakiness=10)


@pytest.mark.parametrize("kw", [dict(stepsize=4), dict(stepsize=5), dict(stepsize=2),
                                dict(stepsize=1), dict(accuracy=9, stepsize=8),
                                dict(accuracy=4, shakiness=8), dict(mincontrast=0.4),
                                dict(mincontrast=0.05), dict(accuracy=1)])
def test_config_variants(kw, search):
    frames = S.clip(640, 480, 4, seed=17)
    check(frames, V.PF_GRAY8, **kw)


@pytest.mark.parametrize("tripod", [1, 3])
def test_tripod(tripod, search):
    frames = S.clip(640, 360, 7, seed=23)
    got, counts = check(frames, V.PF_YUV420P, tripod=tripod)
    assert all(c == 0 for c in counts[:tripod])


@pytest.mark.parametrize("pformat,bpp", [(V.PF_RGB24, 3), (V.PF_BGR24, 3), (V.PF_RGBA, 4)])
def test_packed(pformat, bpp, search):
    frames = S.to_packed(S.clip(320, 240, 4, seed=29), bpp)
    check(frames, pformat)


def test_low_contrast_frames(search):
    """flat frames: no field passes the contrast threshold"""
    frames = np.full((3, 360, 640), 120, np.uint8)
    got, counts = check(frames, V.PF_GRAY8)
    assert counts.sum() == 0


@pytest.mark.parametrize("show", [1, 2])
def test_show_overlay(show):
    frames = S.clip(640, 360, 4, seed=31)
    got, gc, _, drawn = V.detect_clip(frames, V.PF_GRAY8, show=show, return_frames=True)
    if not O.ref_available():
        pytest.skip("overlay pixels are checked against the reference build")
    exp, ec, _, ref_drawn = O.ref_clip(frames, V.PF_GRAY8, show=show, return_frames=True)
    assert records_equal(got, exp), first_difference(got, exp)
    assert np.array_equal(drawn, ref_drawn)


@pytest.mark.parametrize("mode", [V.ASCII_SERIALIZATION_MODE, V.BINARY_SERIALIZATION_MODE, 0])
def test_trf_bytes(mode):
    if not O.ref_available():
        pytest.skip("byte comparison needs the reference build")
    frames = S.clip(640, 360, 5, seed=37)
    with tempfile.TemporaryDirectory() as d:
        a, b = os.path.join(d, "gpu.trf"), os.path.join(d, "ref.trf")
        V.detect_clip(frames, V.PF_YUV420P, serialization_mode=mode, trf_path=a)
        O.ref_clip(frames, V.PF_YUV420P, serialization_mode=mode, trf_path=b)
        assert open(a, "rb").read() == open(b, "rb").read()


def test_device_input_matches_host():
    import torch
    frames = S.clip(1280, 720, 4, seed=41)
    host, hc, _ = V.detect_clip(frames, V.PF_YUV420P)
    d = torch.from_numpy(frames).cuda()
    dev, dc, _ = V.detect_clip(4, V.PF_YUV420P, on_device_ptr=d.data_ptr(),
                               frame_bytes=frames[0].nbytes, linesize=1280, width=1280, height=720)
    assert np.array_equal(hc, dc)
    assert records_equal(host, dev)


def test_per_frame_api_and_reinit():
    frames = S.clip(640, 360, 4, seed=43)
    det = V.MotionDetector(640, 360, V.PF_YUV420P)
    got = [det.detect(f) for f in frames]
    assert det.frame_num == 4
    assert det.launches() > 0
    det.close()
    exp, ec = expected(frames, V.PF_YUV420P)
    assert records_equal(np.concatenate(got), exp)
    # a second detector in the same process gives the same results
    det2 = V.MotionDetector(640, 360, V.PF_YUV420P)
    again = np.concatenate([det2.detect(f) for f in frames])
    det2.close()
    assert records_equal(again, exp)


def test_detect_run_continues_state():
    """vsb_detect_run over a clip in two calls gives the records of one
    detect_clip run over the whole clip, from host and from device frames."""
    import torch
    frames = S.clip(640, 360, 6, seed=45)
    exp, ec, _ = V.detect_clip(frames, V.PF_YUV420P)
    d = torch.from_numpy(frames).cuda()
    fb = frames[0].nbytes
    for on_device in (False, True):
        det = V.MotionDetector(640, 360, V.PF_YUV420P)
        out = np.zeros(6 * 512, V.LM_DTYPE)
        cnt = np.zeros(6, np.int32)
        base = d.data_ptr() if on_device else frames.ctypes.data
        n1 = det.run(3, base, fb, 640, on_device, out, cnt)
        out2 = np.zeros(6 * 512, V.LM_DTYPE)
        cnt2 = np.zeros(3, np.int32)
        n2 = det.run(3, base + 3 * fb, fb, 640, on_device, out2, cnt2)
        det.close()
        assert np.array_equal(cnt[:3], ec[:3])
        assert np.array_equal(cnt2, ec[3:])
        assert records_equal(np.concatenate([out[:n1], out2[:n2]]), exp)
