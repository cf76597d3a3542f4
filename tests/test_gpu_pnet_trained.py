"""The packaged, trained proposal network on held-out 1080p camera-walk
clips: field agreement with the exact full search (target >= 99.5 %), and
what the network gains over the same narrowed search without it (every field
proposed at zero shift, the same fallbacks)."""
import numpy as np
import pytest

import vidstab_b200 as V
from vidstab_b200 import pnet
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu

W, H = 1920, 1080


def _run(clip, blob=None, **kw):
    n = clip.shape[0]
    det = V.MotionDetector(W, H, V.PF_YUV420P)
    if blob is not None:
        pnet.set_proposal(det, blob, verify=True, **kw)
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)
    tot = det.run(n, clip.data_ptr(), W * H, W, True, rec, cnt)
    st = pnet.proposal_stats(det) if blob is not None else None
    det.close()
    return rec[:tot].copy(), cnt, st


def _frames_identical(a, ca, b, cb):
    oa = np.concatenate([[0], np.cumsum(ca)])
    ob = np.concatenate([[0], np.cumsum(cb)])
    return sum(1 for k in range(len(ca))
               if ca[k] == cb[k] and np.array_equal(a[oa[k]:oa[k + 1]], b[ob[k]:ob[k + 1]]))


@pytest.fixture(scope="module")
def clip():
    return S.clip(W, H, 40, seed=401, device="cuda")


def test_trained_agreement_1080p(clip):
    exp, ec, _ = _run(clip)
    got, gc, st = _run(clip, pnet.load_blob())
    # the coarse fields of 39 searched frames (fine fields take the dense search)
    assert st["verified"] == st["searched"] > 2000
    assert st["agreement"] >= 0.995, st
    assert _frames_identical(exp, ec, got, gc) >= 0.95 * len(ec)


def test_network_gain_over_zero_proposal(clip):
    """the network keeps at least as many fields in agreement and sends at
    most half as many coarse fields back to the full search"""
    _, _, learned = _run(clip, pnet.load_blob())
    _, _, zero = _run(clip, pnet.zero_blob())
    assert learned["agreement"] >= zero["agreement"]
    assert learned["coarse_fell_back"] <= 0.5 * max(zero["coarse_fell_back"], 1), (learned, zero)


def test_network_gain_large_shake():
    """with the larger camera steps of the 4K configuration (N(0,8 px),
    N(0,0.5 deg)) the zero-shift proposal misses most coarse fields; the
    network keeps the narrowed search"""
    c = S.clip(W, H, 16, seed=402, device="cuda", trans_sigma=8.0, rot_sigma_deg=0.5)
    _, _, learned = _run(c, pnet.load_blob())
    _, _, zero = _run(c, pnet.zero_blob())
    assert learned["agreement"] >= 0.995
    assert learned["coarse_fell_back"] < zero["coarse_fell_back"], (learned, zero)


def test_two_pass_prior_large_shake():
    """the second network pass around the frame's global motion model (the
    default for shakiness >= 8) keeps more coarse fields on the narrowed
    search under large camera steps, with the same agreement"""
    c = S.clip(W, H, 16, seed=403, device="cuda", trans_sigma=8.0, rot_sigma_deg=0.5)
    blob = pnet.load_blob()
    _, _, one = _run(c, blob, passes=1)
    _, _, two = _run(c, blob, passes=2)
    assert two["agreement"] >= 0.995, two
    assert two["coarse_fell_back"] < one["coarse_fell_back"], (one, two)
