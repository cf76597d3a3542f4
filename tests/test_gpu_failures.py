"""Failure handling of the GPU path, provoked on the host: no GPU fault,
trap or hang is involved.

* the batched kernel's bounded wait runs out (a stream's blur tiles left out
  of the work list, tiny limits): the step fails with a message, the next
  step is clean;
* the host's allocation hooks (vs_malloc / vs_zalloc / vs_realloc of
  src/vidstabdefines.h:84-99 in the reference) fail at every point of
  detector creation and of the first frames: each call fails cleanly
  (VS_ERROR) and a detector made afterwards gives the reference's output;
* a device allocation (cudaMalloc) fails at every point of detector and
  batch creation (the library's own counting hook): creation fails cleanly,
  without leaking device memory, and works again afterwards."""
import ctypes as C

import numpy as np
import pytest

import vidstab_b200 as V
from vidstab_b200 import synthetic as S
from conftest import records_equal
from test_hooks_host import FailingHooks

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _detect_all(det, frames):
    return [det.detect(f) for f in frames]


def test_batch_wait_gives_up_then_next_step_is_clean():
    w, h = 640, 360
    clips = [S.clip(w, h, 3, seed=900 + s) for s in range(2)]
    b = V.Batch([w, w], [h, h])
    L = V.lib()

    def step(k):
        return b.detect([c[k].ctypes.data for c in clips], [w, w], False)

    first = step(0)
    assert all(len(r) == 0 for r in first)
    assert L.vsb_batch_set_wait_limit(b.h, 64, 200000) == 0
    assert L.vsb_batch_test_withhold_blur(b.h, 1) == 0
    with pytest.raises(RuntimeError):
        step(1)
    assert "gave up" in L.vsb_last_error().decode()
    assert L.vsb_batch_test_withhold_blur(b.h, -1) == 0
    assert L.vsb_batch_set_wait_limit(b.h, 1 << 24, 8000000000) == 0
    got = step(2)  # frame 1 was dropped for both streams: 2 follows 0
    b.close()
    for s in range(2):
        d = V.MotionDetector(w, h, V.PF_YUV420P)
        exp = _detect_all(d, [clips[s][0], clips[s][2]])[1]
        d.close()
        assert len(exp) > 0 and records_equal(got[s], exp)


def test_failing_allocation_hooks_during_detect():
    w, h = 640, 360
    frames = S.clip(w, h, 3, seed=910)
    ref = V.MotionDetector(w, h, V.PF_YUV420P)
    exp = _detect_all(ref, frames)
    ref.close()
    outcomes = set()
    for after in list(range(0, 24)) + [40, 80, 160, 320, 640, 1280]:
        det = None
        with FailingHooks(after) as hk:
            try:
                det = V.MotionDetector(w, h, V.PF_YUV420P)
            except RuntimeError:
                outcomes.add("init failed")
            if det is not None:
                for k, f in enumerate(frames):
                    try:
                        got = det.detect(f)
                    except RuntimeError:
                        outcomes.add("frame %d dropped" % min(k, 1))
                        continue
                    if hk.failed == 0:
                        outcomes.add("frame ok")
        if det is not None:
            det.close()
    assert {"init failed", "frame 1 dropped", "frame ok"} <= outcomes, outcomes
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    again = _detect_all(det, frames)
    det.close()
    assert all(records_equal(a, b) for a, b in zip(again, exp))


def test_device_allocation_failure_at_creation():
    L = V.lib()
    w, h = 1280, 720
    frames = S.clip(w, h, 2, seed=920)
    torch.cuda.synchronize()
    d = V.MotionDetector(w, h, V.PF_YUV420P)  # tilings tuned and cached
    exp = _detect_all(d, frames)
    d.close()
    n0 = L.vsb_test_device_alloc(-1, 0)
    d = V.MotionDetector(w, h, V.PF_YUV420P)
    per_detector = L.vsb_test_device_alloc(-1, 0) - n0
    d.close()
    assert per_detector > 3
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(per_detector):
        L.vsb_test_device_alloc(k, 0)
        with pytest.raises(RuntimeError):
            V.MotionDetector(w, h, V.PF_YUV420P)
        assert "memory" in L.vsb_last_error().decode().lower()
    L.vsb_test_device_alloc(-1, 0)
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (8 << 20)  # nothing leaked
    d = V.MotionDetector(w, h, V.PF_YUV420P)
    assert all(records_equal(a, b) for a, b in zip(_detect_all(d, frames), exp))
    d.close()
    # batches: every allocation of a small batch's creation fails in turn
    n0 = L.vsb_test_device_alloc(-1, 0)
    V.Batch([640, 320], [360, 240]).close()
    per_batch = L.vsb_test_device_alloc(-1, 0) - n0
    for k in range(0, per_batch, max(1, per_batch // 12)):
        L.vsb_test_device_alloc(k, 0)
        with pytest.raises(RuntimeError):
            V.Batch([640, 320], [360, 240])
    L.vsb_test_device_alloc(-1, 0)
    V.Batch([640, 320], [360, 240]).close()
