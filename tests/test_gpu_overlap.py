"""The overlapped frame loop (vsb_detect_run: frame k+1's stage A on the GPU
while frame k's fine search runs) gives, frame by frame, the LocalMotions of
the per-frame API, with and without a search proposal, from host and from
device frames."""
import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import pnet
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _per_frame(det, clip, w, h):
    out, cnt = [], []
    for k in range(clip.shape[0]):
        r = det.detect_device(clip.data_ptr() + k * w * h, w)
        out.append(r)
        cnt.append(len(r))
    return np.concatenate(out), np.array(cnt, np.int32)


def _run(det, ptr, n, w, h, on_device):
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)
    tot = det.run(n, ptr, w * h, w, on_device, rec, cnt)
    return rec[:tot].copy(), cnt


@pytest.mark.parametrize("w,h", [(640, 480), (1920, 1080)])
def test_overlapped_equals_per_frame(w, h):
    n = 14
    clip = S.clip(w, h, n, seed=31, device="cuda")
    a = V.MotionDetector(w, h, V.PF_YUV420P)
    exp, ec = _per_frame(a, clip, w, h)
    b = V.MotionDetector(w, h, V.PF_YUV420P)
    got, gc = _run(b, clip.data_ptr(), n, w, h, True)
    assert np.array_equal(gc, ec) and np.array_equal(got, exp)
    host = clip.cpu().numpy()
    c = V.MotionDetector(w, h, V.PF_YUV420P)
    got2, gc2 = _run(c, host.ctypes.data, n, w, h, False)
    assert np.array_equal(gc2, ec) and np.array_equal(got2, exp)


def test_overlapped_matches_reference():
    if not O.ref_available():
        pytest.skip("reference build not present")
    w, h, n = 640, 480, 8
    host = S.clip(w, h, n, seed=32)
    clip = torch.from_numpy(host).cuda()
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    got, gc = _run(det, clip.data_ptr(), n, w, h, True)
    exp, ec, _ = O.ref_clip(host, V.PF_YUV420P)
    assert np.array_equal(gc, ec)
    for k in ("vx", "vy", "fx", "fy", "fsize", "contrast", "match"):
        assert np.array_equal(got[k], exp[k]), k


@pytest.mark.parametrize("on_device", [True, False])
def test_overlapped_with_proposal(on_device):
    """the learned frame loop, from device and from host frames, and a second
    run of the same detector that continues its state"""
    w, h, n = 1920, 1080, 12
    clip = S.clip(w, h, n, seed=33, device="cuda")
    host = clip.cpu().numpy()
    blob = pnet.load_blob()
    a = V.MotionDetector(w, h, V.PF_YUV420P)
    pnet.set_proposal(a, blob)
    exp, ec = _per_frame(a, clip, w, h)
    b = V.MotionDetector(w, h, V.PF_YUV420P)
    pnet.set_proposal(b, blob)
    got, gc = _run(b, clip.data_ptr() if on_device else host.ctypes.data, n, w, h, on_device)
    assert np.array_equal(gc, ec) and np.array_equal(got, exp)
    # a second run of the same detector continues across the lanes
    got2, gc2 = _run(b, clip.data_ptr() if on_device else host.ctypes.data, n, w, h, on_device)
    assert ec[0] == 0 and np.array_equal(gc2[1:], ec[1:])
    assert np.array_equal(got2[gc2[0]:], exp)


def test_multi_detectors_equal_their_own_runs():
    """vsb_detect_multi: mixed resolutions, one detector with the proposal and
    its two-pass prior, one in tripod mode; every stream's motions are its
    own detector's"""
    sizes = [(640, 360), (1920, 1080), (1280, 720)]
    n = 6
    clips = [S.clip(w, h, n, seed=40 + i, device="cuda") for i, (w, h) in enumerate(sizes)]
    blob = pnet.load_blob()

    def make(i):
        w, h = sizes[i]
        d = V.MotionDetector(w, h, V.PF_YUV420P, tripod=2 if i == 2 else 0)
        if i == 1:
            pnet.set_proposal(d, blob, passes=2)
        return d

    exp = []
    for i, (w, h) in enumerate(sizes):
        d = make(i)
        exp.append(_per_frame(d, clips[i], w, h))
        d.close()
    dets = [make(i) for i in range(len(sizes))]
    out = np.zeros(n * len(sizes) * 800, V.LM_DTYPE)
    counts = np.zeros(n * len(sizes), np.int32)
    tot = V.detect_multi(dets, [c.data_ptr() for c in clips], [w * h for w, h in sizes],
                         [w for w, _ in sizes], n, True, out, counts)
    cm = counts.reshape(n, len(sizes))
    pos = np.concatenate([[0], np.cumsum(cm.ravel())])
    assert pos[-1] == tot
    for s in range(len(sizes)):
        got = np.concatenate([out[pos[k * len(sizes) + s]:pos[k * len(sizes) + s + 1]]
                              for k in range(n)])
        assert np.array_equal(cm[:, s], exp[s][1])
        assert np.array_equal(got, exp[s][0])


def test_headline_clip_frame_loops_match_reference():
    """The benchmark's workload whole: the 300-frame 1920x1080 camera-walk
    clip (seed 1) through the overlapped frame loop from device and from host
    frames, and through the per-frame loop (vsb_detect_frames), each equal to
    the reference's CPU detect of the same clip, every frame, all seven fields
    (tests/test_determinism.c:356-361 of the reference)."""
    if not O.ref_available():
        pytest.skip("reference build not present")
    w, h, n = 1920, 1080, 300
    clip = S.clip(w, h, n, seed=1, device="cuda")
    host = clip.cpu().numpy()
    exp, ec, _ = O.ref_clip(host, V.PF_YUV420P, threads=8)
    a = V.MotionDetector(w, h, V.PF_YUV420P)
    got, gc = _run(a, clip.data_ptr(), n, w, h, True)
    assert np.array_equal(gc, ec)
    for k in ("vx", "vy", "fx", "fy", "fsize", "contrast", "match"):
        assert np.array_equal(got[k], exp[k]), k
    pinned = torch.from_numpy(host).pin_memory()
    b = V.MotionDetector(w, h, V.PF_YUV420P)
    got, gc = _run(b, pinned.data_ptr(), n, w, h, False)
    assert np.array_equal(gc, ec) and np.array_equal(got, exp.astype(V.LM_DTYPE))
    c = V.MotionDetector(w, h, V.PF_YUV420P)
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)
    tot = c.run_frames(n, pinned.data_ptr(), w * h, w, False, rec, cnt)
    assert np.array_equal(cnt, ec) and np.array_equal(rec[:tot], exp.astype(V.LM_DTYPE))
