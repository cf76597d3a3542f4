"""Learned search proposal inside the batched persistent kernel
(vsb_batch_set_proposal): the network passes, the global-motion prior, the
narrowed searches and the dense search of the items that fell back are work
items of the same kernel as the blur and the min/max.

Each stream must give exactly what a detector of its own with the same
network gives (those detectors are pinned to the exact full search by
tests/test_gpu_pnet*.py), and at the resolutions the packaged network is
calibrated for (1080p, 4K) its fields must agree with the plain search (the
reference's results) on at least 99.5 % of fields."""
import numpy as np
import pytest

from conftest import records_equal
import vidstab_b200 as V
from vidstab_b200 import pnet
from vidstab_b200 import synthetic as S
from test_gpu_batch import batch_records

pytestmark = pytest.mark.gpu


def learned_detectors(frames_list, blob, shakiness):
    """each stream through a learned detector of its own (stepped together)"""
    import torch
    n = len(frames_list)
    T = frames_list[0].shape[0]
    held = [torch.from_numpy(f).cuda() for f in frames_list]
    ds = []
    for f in frames_list:
        d = V.MotionDetector(f.shape[2], f.shape[1], V.PF_YUV420P, shakiness=shakiness)
        pnet.set_proposal(d, blob)
        ds.append(d)
    out = np.zeros(T * n * 4096, V.LM_DTYPE)
    counts = np.zeros(T * n, np.int32)
    try:
        total = V.detect_multi(ds, [h.data_ptr() for h in held], [f[0].nbytes for f in frames_list],
                               [f.shape[2] for f in frames_list], T, True, out, counts)
    finally:
        for d in ds:
            d.close()
    counts = counts.reshape(T, n)
    per = [[] for _ in range(n)]
    pos = 0
    for k in range(T):
        for s in range(n):
            per[s].append(out[pos:pos + counts[k, s]])
            pos += counts[k, s]
    assert pos == total
    return [(np.concatenate(p), counts[:, s]) for s, p in enumerate(per)]


def field_agreement(got, exp):
    """fields of the plain search reproduced exactly (stream by stream,
    frame by frame, same field order)"""
    same = tot = 0
    for (g, gc), (e, ec) in zip(got, exp):
        pg = pe = 0
        for a, b in zip(gc, ec):
            ga, eb = g[pg:pg + a], e[pe:pe + b]
            pg += a
            pe += b
            tot += b
            if a == b:
                same += int(sum(all(ga[k][i] == eb[k][i] for k in
                                    ("vx", "vy", "fx", "fy", "fsize", "contrast", "match"))
                                for i in range(b)))
    return same / max(tot, 1)


@pytest.mark.parametrize("on_device", [False, True])
def test_learned_batch_equals_learned_detectors(on_device):
    sizes = [(640, 360), (1280, 720), (1920, 1080), (640, 360)]
    frames = [S.clip(w, h, 5, seed=900 + i) for i, (w, h) in enumerate(sizes)]
    blob = pnet.load_blob()
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        b.set_proposal(blob)
        got = batch_records(b, frames, on_device)
        st = b.proposal_stats()
        assert b.launches() == 2 * 5 - 1  # still two launches per step
    finally:
        b.close()
    assert st["coarse_searched"] > 0 and st["fine_searched"] == 0  # fine fields: dense
    exp = learned_detectors(frames, blob, 5)
    for (g, gc), (e, ec) in zip(got, exp):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)
    # the packaged network is calibrated on 1080p fields: the agreement bound
    # holds there (smaller frames have other field sizes and shift ranges)
    k = sizes.index((1920, 1080))
    plain = V.detect_clip(frames[k], V.PF_YUV420P)[:2]
    assert field_agreement([got[k]], [plain]) >= 0.995


def test_learned_batch_two_passes_large_shake():
    """shakiness 10: every stream's coarse fields take the prior and a second
    network pass inside the persistent kernel"""
    n, w, h, T = 3, 1920, 1080, 5
    frames = [S.clip(w, h, T, seed=950 + i, trans_sigma=8.0, rot_sigma_deg=0.5) for i in range(n)]
    blob = pnet.load_blob()
    b = V.Batch([w] * n, [h] * n, shakiness=10)
    try:
        b.set_proposal(blob)
        got = batch_records(b, frames, True)
        st = b.proposal_stats()
    finally:
        b.close()
    assert st["coarse_searched"] > 0
    exp = learned_detectors(frames, blob, 10)
    for (g, gc), (e, ec) in zip(got, exp):
        assert np.array_equal(gc, ec)
        assert records_equal(g, e)
    plain = [V.detect_clip(f, V.PF_YUV420P, shakiness=10)[:2] for f in frames]
    assert field_agreement(got, plain) >= 0.995


def test_learned_batch_back_to_plain_and_per_step():
    """the proposal switched off again gives the plain batch; per-step calls
    with the proposal equal the overlapped run"""
    sizes = [(640, 360), (1280, 720)]
    frames = [S.clip(w, h, 4, seed=970 + i) for i, (w, h) in enumerate(sizes)]
    blob = pnet.load_blob()
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    try:
        b.set_proposal(blob)
        steps = [b.detect([f[k].ctypes.data for f in frames], [w for w, _ in sizes], False)
                 for k in range(4)]
        b.set_proposal(None)
        plain_again = batch_records(b, frames, False)
    finally:
        b.close()
    exp = learned_detectors(frames, blob, 5)
    for s in range(2):
        got = np.concatenate([st[s] for st in steps])
        assert records_equal(got, exp[s][0])
    # the plain steps continue the streams: frames 4..7 of the clip played twice
    for (g, gc), f in zip(plain_again, frames):
        e, ec = V.detect_clip(np.concatenate([f, f]), V.PF_YUV420P)[:2]
        assert np.array_equal(gc, ec[4:])
        assert records_equal(g, e[int(ec[:4].sum()):])
