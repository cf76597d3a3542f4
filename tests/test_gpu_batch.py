"""Batched multi-stream detect: every stream of a batch gives exactly the
LocalMotions of a detector of its own (which the other GPU tests pin to the
reference), across resolutions, frame counts and input kinds."""
import numpy as np
import pytest

from conftest import records_equal
import vidstab_b200 as V
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def per_stream(frames_list, **kw):
    return [V.detect_clip(f, V.PF_YUV420P, **kw)[:2] for f in frames_list]


def batch_records(b, frames_list, on_device):
    import torch
    n = len(frames_list)
    T = frames_list[0].shape[0]
    held = [torch.from_numpy(f).cuda() for f in frames_list] if on_device else frames_list
    ptrs = [h.data_ptr() if on_device else h.ctypes.data for h in held]
    fb = [f[0].nbytes for f in frames_list]
    pitches = [f.shape[2] for f in frames_list]
    out = np.zeros(T * n * 1024, V.LM_DTYPE)
    counts = np.zeros(T * n, np.int32)
    total = b.run(ptrs, fb, pitches, T, on_device, out, counts)
    counts = counts.reshape(T, n)
    # split the step-major record stream back into streams
    per = [[] for _ in range(n)]
    pos = 0
    for k in range(T):
        for s in range(n):
            per[s].append(out[pos:pos + counts[k, s]])
            pos += counts[k, s]
    assert pos == total
    return [(np.concatenate(p), counts[:, s]) for s, p in enumerate(per)]


@pytest.mark.parametrize("on_device", [False, True])
def test_batch_mixed_resolutions_match_single_streams(on_device):
    sizes = [(640, 360), (1280, 720), (640, 360), (1920, 1080), (960, 540)]
    frames = [S.clip(w, h, 5, seed=100 + i) for i, (w, h) in enumerate(sizes)]
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        got = batch_records(b, frames, on_device)
        assert b.launches() == 2 * 5 - 1  # no fine pass on the first step
    finally:
        b.close()
    for (g, gc), (e, ec) in zip(got, per_stream(frames)):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)


def test_batch_4k_and_small_together():
    sizes = [(3840, 2160), (640, 360), (640, 360)]
    frames = [S.clip(w, h, 3, seed=200 + i) for i, (w, h) in enumerate(sizes)]
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        got = batch_records(b, frames, True)
    finally:
        b.close()
    for (g, gc), (e, ec) in zip(got, per_stream(frames)):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)


def test_batch_per_step_api_and_tripod():
    sizes = [(640, 360), (640, 360)]
    frames = [S.clip(640, 360, 5, seed=300 + i) for i in range(2)]
    b = V.Batch([640, 640], [360, 360], tripod=2)
    try:
        steps = [b.detect([f[k].ctypes.data for f in frames], [640, 640], False) for k in range(5)]
    finally:
        b.close()
    for s in range(2):
        exp, ec = per_stream([frames[s]], tripod=2)[0]
        got = np.concatenate([st[s] for st in steps])
        assert np.array_equal([len(st[s]) for st in steps], ec)
        assert records_equal(got, exp)


def test_batch_many_streams_of_one_size():
    n = 24
    frames = [S.clip(640, 360, 3, seed=400 + i) for i in range(n)]
    b = V.Batch([640] * n, [360] * n)
    try:
        ctas, threads, smem = b.grid()
        assert ctas >= 148 and threads == 512 and smem > 0
        got = batch_records(b, frames, True)
    finally:
        b.close()
    for (g, gc), (e, ec) in zip(got, per_stream(frames)):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)


@pytest.mark.parametrize("on_device", [False, True])
def test_batch_run_overlap_mixed_with_per_step_calls(on_device):
    # the overlapped run continues a batch stepped by vsb_batch_detect and is
    # continued by it: the blurred-plane slots rotate consistently across both
    sizes = [(640, 360), (1280, 720), (960, 540)]
    T = 8
    frames = [S.clip(w, h, T, seed=500 + i) for i, (w, h) in enumerate(sizes)]
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        pitches = [w for w, _ in sizes]
        head = [b.detect([f[k].ctypes.data for f in frames], pitches, False) for k in range(2)]
        mid = batch_records(b, [np.ascontiguousarray(f[2:6]) for f in frames], on_device)
        tail = [b.detect([f[k].ctypes.data for f in frames], pitches, False) for k in range(6, T)]
    finally:
        b.close()
    for s, (e, ec) in enumerate(per_stream(frames)):
        got = [st[s] for st in head] + [mid[s][0]] + [st[s] for st in tail]
        cnt = [len(st[s]) for st in head] + list(mid[s][1]) + [len(st[s]) for st in tail]
        assert np.array_equal(cnt, ec)
        assert records_equal(np.concatenate(got), e)


def test_batch_run_with_tripod_stream():
    # a virtual-tripod stream keeps its reference frame: the run steps serially
    frames = [S.clip(640, 360, 6, seed=600 + i) for i in range(2)]
    b = V.Batch([640, 640], [360, 360], tripod=3)
    try:
        got = batch_records(b, frames, True)
    finally:
        b.close()
    for (g, gc), (e, ec) in zip(got, per_stream(frames, tripod=3)):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)


@pytest.mark.parametrize("mode", [1, 2])
def test_batch_trf_matches_single_stream(tmp_path, mode):
    # the batch's .trf files equal, byte for byte, those a detector of its
    # own writes for the stream; per-step calls and the overlapped run both
    # append; a stream without a path writes nothing
    sizes = [(640, 360), (1280, 720), (640, 360)]
    T = 6
    frames = [S.clip(w, h, T, seed=700 + i) for i, (w, h) in enumerate(sizes)]
    paths = [str(tmp_path / ("batch%d_%d.trf" % (mode, s))) for s in range(len(sizes))]
    paths[2] = None
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        b.open_trf(paths, mode)
        pitches = [w for w, _ in sizes]
        for k in range(2):
            b.detect([f[k].ctypes.data for f in frames], pitches, False)
        batch_records(b, [np.ascontiguousarray(f[2:]) for f in frames], True)
        b.close_trf()
    finally:
        b.close()
    for s, p in enumerate(paths):
        if p is None:
            continue
        exp = str(tmp_path / ("single%d_%d.trf" % (mode, s)))
        V.detect_clip(frames[s], V.PF_YUV420P, serialization_mode=mode, trf_path=exp)
        with open(p, "rb") as fa, open(exp, "rb") as fb:
            assert fa.read() == fb.read(), s
