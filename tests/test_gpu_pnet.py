"""The learned search proposal on the GPU: every network kernel against the
float64 oracle (crops bit for bit; layer outputs and gradients within the
fp32-accumulation tolerance), the narrowed search against the exact full
search, and the detector's fallback path end to end."""
import numpy as np
import pytest

import pnet_oracle as P
import vidstab_b200 as V
from vidstab_b200 import pnet
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _params(seed):
    bits, f32 = P.init_params(seed)
    rng = np.random.default_rng(seed + 5)
    f32 = f32.copy()
    f32[:128] = rng.normal(0.05, 0.05, 128)
    f32[128:] = rng.normal(0, 0.1, 3)
    return bits, f32.astype(np.float32)


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = P.bf16_round(rng.uniform(-2, 2, (n, 32, 32, 2)))
    xt = torch.from_numpy(P.to_bf16_bits(x).view(np.int16)).cuda()
    return x, xt


def _acts(acts, n):
    a = acts.cpu().numpy().view(np.uint16)
    sizes = [(32, 32), (16, 16), (8, 8), (4, 4)]
    out, o = [], 0
    for h, w in sizes:
        k = n * h * w * 32
        out.append(P.from_bf16_bits(a[o:o + k]).reshape(n, h, w, 32))
        o += k
    return out


def test_crops_match_oracle():
    rng = np.random.default_rng(0)
    W, H = 300, 200
    curr = rng.integers(0, 256, (H, W), dtype=np.uint8)
    prev = rng.integers(0, 256, (H, W), dtype=np.uint8)
    items = np.array([[150, 100, 0, 0], [40, 40, 3, -2], [5, 3, 0, 0], [W - 2, H - 1, -1, 1],
                      [100, 150, 12, -30], [33, 190, -5, 7]], np.int16)
    got = pnet.crops(torch.from_numpy(curr).cuda(), torch.from_numpy(prev).cuda(), items)
    got = got.cpu().numpy().view(np.uint16).reshape(len(items), 32, 32, 2)
    exp = P.to_bf16_bits(P.crops(curr, prev, items.astype(int)))
    assert np.array_equal(got, exp)


def test_forward_train_layers_match_oracle():
    """each layer from the GPU's own stored input: only fp32-vs-fp64
    summation differences, which flip a bf16 rounding at most by one step"""
    n = 5
    bits, f32 = _params(1)
    p = P.unpack(bits, f32)
    x, xt = _inputs(n, 2)
    params = pnet.params_to_device(bits, f32)
    out, acts = pnet.forward_train(params, xt, n)
    a1, a2, a3, a4 = _acts(acts, n)
    ins = [x, a1, a2, a3]
    ws = [P.w1_taps(p["W1"]), p["W2"], p["W3"], p["W4"]]
    for k, (xin, got) in enumerate(zip(ins, [a1, a2, a3, a4])):
        exp = P.bf16_round(np.maximum(P.conv_fwd(xin, ws[k], p["b%d" % (k + 1)], 1 if k == 0 else 2), 0))
        close = np.abs(got - exp) <= np.abs(exp) * 2.0 ** -7 + 1e-6
        assert close.all(), (k, np.abs(got - exp).max())
        assert (got == exp).mean() > 0.99, k
    eout = a4.reshape(n, 512) @ p["Wfc"].T + p["bfc"]
    assert np.allclose(out.cpu().numpy(), eout, rtol=1e-4, atol=1e-4)


def test_backward_matches_oracle():
    """gradients of sum(out * dout) for every parameter, against the float64
    restatement evaluated on the GPU's stored activations"""
    n = 6
    bits, f32 = _params(3)
    p = P.unpack(bits, f32)
    x, xt = _inputs(n, 4)
    params = pnet.params_to_device(bits, f32)
    out, acts = pnet.forward_train(params, xt, n)
    dout = np.random.default_rng(5).normal(0, 1, (n, 3))
    grad = pnet.backward(params, xt, acts, n, torch.from_numpy(dout).float().cuda()).cpu().numpy()
    gb, gf = P.backward(p, x, tuple(_acts(acts, n)), dout.astype(np.float32).astype(np.float64))
    offs = [0, P.N_W1, P.N_W1 + P.N_W, P.N_W1 + 2 * P.N_W, P.N_W1 + 3 * P.N_W, P.N_BF16]
    for a, b in zip(offs[:-1], offs[1:]):
        g, e = grad[a:b], gb[a:b]
        assert np.abs(g - e).max() <= 1e-4 * max(np.abs(e).max(), 1e-3), (a, np.abs(g - e).max())
    g = grad[P.N_BF16:]
    assert np.abs(g - gf).max() <= 1e-4 * max(np.abs(gf).max(), 1e-3)


def test_infer_kernel_matches_forward():
    """the fused tensor-core inference (prepared inputs and crops taken from
    the planes) against the training forward and the oracle"""
    n = 333
    bits, f32 = _params(7)
    p = P.unpack(bits, f32)
    x, xt = _inputs(n, 8)
    params = pnet.params_to_device(bits, f32)
    ref, _ = pnet.forward_train(params, xt, n)
    got = pnet.infer(params, xt, n).cpu().numpy()
    ref = ref.cpu().numpy()
    d = np.abs(got - ref)
    assert d.max() < 0.05 and np.median(d) < 2e-3, (d.max(), np.median(d))
    _, eo = P.forward(p, x[:16])
    assert np.abs(got[:16] - eo).max() < 0.05
    # crops taken by the kernel itself
    rng = np.random.default_rng(9)
    W, H = 400, 300
    curr = rng.integers(0, 256, (H, W), dtype=np.uint8)
    prev = rng.integers(0, 256, (H, W), dtype=np.uint8)
    items = np.stack([rng.integers(0, W, 40), rng.integers(0, H, 40), rng.integers(-9, 10, 40),
                      rng.integers(-9, 10, 40)], 1).astype(np.int16)
    ct, pt = torch.from_numpy(curr).cuda(), torch.from_numpy(prev).cuda()
    xi = pnet.crops(ct, pt, items)
    a = pnet.infer(params, xi, len(items)).cpu().numpy()
    b = pnet.infer_items(params, ct, pt, items).cpu().numpy()
    assert np.array_equal(a, b)


def _pair(w, h, seed):
    clip = S.clip(w, h, 2, seed=seed)
    return V.boxblur(clip[1], 7), V.boxblur(clip[0], 7)


@pytest.mark.parametrize("size,max_shift,step,offs", [(64, 68, 6, 0), (16, 16, 2, 3), (32, 32, 2, 2)])
def test_narrow_finds_full_search_result(size, max_shift, step, offs):
    """with the proposal within the radius of the full search's result, the
    narrowed search reproduces it exactly and accepts it"""
    curr, prev = _pair(640, 480, 11 + size)
    m = size // 2 + max_shift + step + offs
    xs, ys = np.meshgrid(np.arange(m, 640 - m, 23), np.arange(m, 480 - m, 29))
    xs, ys = xs.ravel(), ys.ravel()
    rng = np.random.default_rng(size)
    ox = rng.integers(-offs, offs + 1, len(xs)) if offs else None
    oy = rng.integers(-offs, offs + 1, len(xs)) if offs else None
    sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, max_shift, step, ox, oy)
    for err in (0, 2):
        e = rng.integers(-err, err + 1, (len(xs), 2))
        pout = np.stack([(tx + e[:, 0]) / pnet.SCALE, (ty + e[:, 1]) / pnet.SCALE,
                         np.full(len(xs), 5.0)], 1)
        s2, x2, y2, ok2, fl = pnet.narrow_host(curr, prev, xs, ys, size, max_shift, step, pout,
                                               ox, oy)
        assert np.array_equal(s2, sad) and np.array_equal(x2, tx) and np.array_equal(y2, ty)
        assert np.array_equal(ok2, ok)
        assert (fl == 0).all()


def test_narrow_fallback_flags():
    size, max_shift, step = 64, 68, 6
    curr, prev = _pair(640, 480, 3)
    m = size // 2 + max_shift + step
    xs = np.array([m, 320, 640 - m, 200])
    ys = np.array([m, 240, 480 - m, 300])
    sad, tx, ty, ok = V.field_search(curr, prev, xs, ys, size, max_shift, step)
    good = np.stack([tx / pnet.SCALE, ty / pnet.SCALE, np.full(4, 5.0)], 1)
    # low confidence
    low = good.copy()
    low[:, 2] = -5.0
    assert (pnet.narrow_host(curr, prev, xs, ys, size, max_shift, step, low)[4] == 1).all()
    # predictions outside the lattice and non-finite ones
    bad = good.copy()
    bad[0, :2] = 1000.0
    bad[1, 0] = np.nan
    bad[2, 1] = np.inf
    fl = pnet.narrow_host(curr, prev, xs, ys, size, max_shift, step, bad)[4]
    assert list(fl) == [1, 1, 1, 0]
    # a SAD bound below every result
    fl = pnet.narrow_host(curr, prev, xs, ys, size, max_shift, step, good,
                          sad_bound=int(sad.min()) - 1)[4]
    assert (fl == 1).all()


def _clip(w, h, n, seed):
    return S.clip(w, h, n, seed=seed, device="cuda")


def _run(det, clip, w, h):
    n = clip.shape[0]
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)
    tot = det.run(n, clip.data_ptr(), w * h, w, True, rec, cnt)
    return rec[:tot].copy(), cnt


def test_detector_full_fallback_is_plain():
    """every item falling back (confidence threshold above any logit) must
    give the plain detector's LocalMotions bit for bit"""
    w, h = 640, 480
    clip = _clip(w, h, 12, 21)
    plain = V.MotionDetector(w, h, V.PF_YUV420P)
    exp, ec = _run(plain, clip, w, h)
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    pnet.set_proposal(det, pnet.zero_blob(), conf_min=1e30, verify=True, fine_net=True)
    got, gc = _run(det, clip, w, h)
    st = pnet.proposal_stats(det)
    assert np.array_equal(gc, ec)
    assert np.array_equal(got, exp)
    assert st["searched"] > 0 and st["fell_back"] == st["searched"]
    assert st["identical"] == st["verified"] == st["searched"]


def test_detector_zero_proposal_consistent():
    """the narrowed path with a proposal at zero shift: where every item
    agrees with the full search, the LocalMotions are the plain ones"""
    w, h = 640, 480
    clip = _clip(w, h, 10, 22)
    plain = V.MotionDetector(w, h, V.PF_YUV420P)
    exp, ec = _run(plain, clip, w, h)
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    # fine fields narrowed too (4 px around the coarse model's prediction)
    pnet.set_proposal(det, pnet.zero_blob(), verify=True, fine_radius=4.0)
    got, gc = _run(det, clip, w, h)
    st = pnet.proposal_stats(det)
    assert st["searched"] > 0 and st["verified"] == st["searched"]
    assert 0 < st["fell_back"] < st["searched"]
    if st["identical"] == st["verified"]:
        assert np.array_equal(got, exp)


def test_training_reduces_loss():
    """a short run of the trainer on logged pairs lowers the loss"""
    w, h = 640, 480
    clip = _clip(w, h, 16, 23)
    x, lab = pnet.field_log(clip, w, h, cap=20000)
    assert len(lab) > 1000 and (lab["use"] == 1).sum() > 500
    hist = []
    pnet.train(x, lab, steps=400, batch=256, lr=2e-3, log=hist.append)
    assert hist[-1][1] < 0.7 * hist[0][1], hist
