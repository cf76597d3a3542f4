"""CPU oracle of the learned search-proposal network (test infrastructure).

This file is a checker: only tests, the smoke entry and the benchmark's CPU
leg use it.  The product computes everything here in CUDA
(vid.stab_b200/csrc/vsb_pnet.cu).

The network has no counterpart in the reference; it narrows the reference's
per-field search (src/motiondetect.c:439-586), whose exact result stays the
arbiter.  The semantics restated here, in float64 with the GPU's storage
roundings (bf16 round-to-nearest-even of inputs, weights and stored
activations), are:

  input   per item (field centre x, y; search offset ox, oy) two 32x32
          planes: the blurred current frame around (x, y) and the blurred
          previous frame around (x+ox, y+oy), each a 64x64 window (top-left
          centre-32) averaged over 2x2 blocks, coordinates clamped to the
          frame; value bf16((sum4 - 512) / 256).  Layout [32][32][2] (HWC).
  conv1   2 -> 32, 3x3, stride 1, zero padding 1, ReLU      -> 32x32x32
  conv2   32 -> 32, 3x3, stride 2, padding 1, ReLU          -> 16x16x32
  conv3   32 -> 32, 3x3, stride 2, padding 1, ReLU          ->  8x8x32
  conv4   32 -> 32, 3x3, stride 2, padding 1, ReLU          ->  4x4x32
  head    fully connected 512 -> 3 (no activation): (dx, dy) in units of
          out_scale pixels and a confidence logit.
  Every stored activation is rounded to bf16 after the ReLU; accumulation is
  in float32 on the GPU (float64 here).

Parameter vector (the order of the device buffer):
  bf16 part: W1 [32 co][32 k] (k = tap*2 + ci, tap = ky*3 + kx; k >= 18 zero),
             W2, W3, W4 [9 tap][32 co][32 ci], Wfc [3][512] (k = (y*4+x)*32+c)
  f32 part:  b1, b2, b3, b4 [32] each, bfc [3]
"""
import numpy as np

C = 32
N_W1 = 32 * 32
N_W = 9 * 32 * 32
N_FC = 3 * 512
N_BF16 = N_W1 + 3 * N_W + N_FC
N_F32 = 4 * 32 + 3


def bf16_round(x):
    """round-to-nearest-even to bfloat16, returned as float64"""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


def to_bf16_bits(x):
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(bf16_bits, f32):
    """parameter vectors -> dict of float64 arrays"""
    w = from_bf16_bits(bf16_bits)
    o = 0
    p = {}
    p["W1"] = w[o:o + N_W1].reshape(32, 32); o += N_W1
    for k in (2, 3, 4):
        p["W%d" % k] = w[o:o + N_W].reshape(9, 32, 32); o += N_W
    p["Wfc"] = w[o:o + N_FC].reshape(3, 512); o += N_FC
    f = np.asarray(f32, dtype=np.float64)
    for k in range(4):
        p["b%d" % (k + 1)] = f[32 * k:32 * (k + 1)]
    p["bfc"] = f[128:131]
    return p


def crops(curr, prev, items):
    """network inputs [n][32][32][2] (float64 of bf16 values) of items
    (x, y, ox, oy) on blurred planes curr, prev (H x W uint8)"""
    H, W = curr.shape
    out = np.zeros((len(items), 32, 32, 2))
    i = np.arange(32)
    for n, (x, y, ox, oy) in enumerate(items):
        for ch, (img, cx, cy) in enumerate(((curr, x, y), (prev, x + ox, y + oy))):
            s = np.zeros((32, 32), np.int64)
            for dy in (0, 1):
                for dx in (0, 1):
                    ry = np.clip(cy - 32 + 2 * i + dy, 0, H - 1)
                    rx = np.clip(cx - 32 + 2 * i + dx, 0, W - 1)
                    s += img[ry][:, rx].astype(np.int64)
            out[n, :, :, ch] = bf16_round((s.astype(np.float32) - 512.0) / 256.0)
    return out


def _pad(a):
    return np.pad(a, ((0, 0), (1, 1), (1, 1), (0, 0)))


def conv_fwd(x, Wt, b, stride, layer1=False):
    """x [n][H][W][cin]; Wt [9][32][cin] (layer 1 is converted); -> pre-activation"""
    n, H, Wd, cin = x.shape
    Ho, Wo = H // stride, Wd // stride
    xp = _pad(x)
    out = np.broadcast_to(b, (n, Ho, Wo, 32)).copy()
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        patch = xp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :]
        out += np.einsum("nhwc,oc->nhwo", patch, Wt[tap])
    return out


def w1_taps(W1):
    """W1 [32][32 k] -> [9][32][2]"""
    return W1[:, :18].reshape(32, 9, 2).transpose(1, 0, 2)


def forward(p, x, rounding=True):
    """-> (acts a1..a4, out [n][3]); with rounding the stored activations are
    bf16 values (as on the GPU), without it plain float64 (for derivative
    checks of the backward restatement)"""
    rnd = bf16_round if rounding else (lambda a: a)
    a1 = rnd(np.maximum(conv_fwd(x, w1_taps(p["W1"]), p["b1"], 1), 0))
    a2 = rnd(np.maximum(conv_fwd(a1, p["W2"], p["b2"], 2), 0))
    a3 = rnd(np.maximum(conv_fwd(a2, p["W3"], p["b3"], 2), 0))
    a4 = rnd(np.maximum(conv_fwd(a3, p["W4"], p["b4"], 2), 0))
    out = a4.reshape(len(x), 512) @ p["Wfc"].T + p["bfc"]
    return (a1, a2, a3, a4), out


def conv_bwd(x, y, dy, Wt, stride):
    """gradients of one conv layer given its input x, stored output y (ReLU
    mask y > 0) and upstream dy: -> (dx, dW [9][32][cin], db [32])"""
    n, H, Wd, cin = x.shape
    Ho, Wo = H // stride, Wd // stride
    g = dy * (y > 0)
    xp = _pad(x)
    dxp = np.zeros_like(xp)
    dW = np.zeros((9, 32, cin))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        patch = xp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :]
        dW[tap] = np.einsum("nhwo,nhwc->oc", g, patch)
        dxp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :] += np.einsum(
            "nhwo,oc->nhwc", g, Wt[tap])
    return dxp[:, 1:-1, 1:-1, :], dW, g.sum(axis=(0, 1, 2))


def backward(p, x, acts, dout):
    """gradient of sum(out * dout) -> (grad bf16-part order float64, grad f32 part)"""
    a1, a2, a3, a4 = acts
    n = len(x)
    dWfc = dout.T @ a4.reshape(n, 512)
    dbfc = dout.sum(axis=0)
    d4 = (dout @ p["Wfc"]).reshape(n, 4, 4, 32)
    d3, dW4, db4 = conv_bwd(a3, a4, d4, p["W4"], 2)
    d2, dW3, db3 = conv_bwd(a2, a3, d3, p["W3"], 2)
    d1, dW2, db2 = conv_bwd(a1, a2, d2, p["W2"], 2)
    _, dW1t, db1 = conv_bwd(x, a1, d1, w1_taps(p["W1"]), 1)
    dW1 = np.zeros((32, 32))
    dW1[:, :18] = dW1t.transpose(1, 0, 2).reshape(32, 18)
    gb = np.concatenate([dW1.ravel(), dW2.ravel(), dW3.ravel(), dW4.ravel(), dWfc.ravel()])
    gf = np.concatenate([db1, db2, db3, db4, dbfc])
    return gb, gf


def init_params(seed=0):
    """He-initialised parameters: (bf16 bits, f32)"""
    rng = np.random.default_rng(seed)
    W1 = np.zeros((32, 32))
    W1[:, :18] = rng.normal(0, np.sqrt(2.0 / 18), (32, 18))
    ws = [W1.ravel()]
    for _ in range(3):
        ws.append(rng.normal(0, np.sqrt(2.0 / 288), N_W))
    ws.append(rng.normal(0, np.sqrt(1.0 / 512), N_FC))
    f = np.zeros(N_F32)
    f[:128] = 0.01
    return to_bf16_bits(np.concatenate(ws)), f.astype(np.float32)
