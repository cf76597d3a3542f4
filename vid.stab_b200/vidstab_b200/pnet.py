"""The learned search proposal: bindings, offline trainer, calibration and
the VSBP file format.

Inference runs inside the C library: a detector given a network with
vsb_set_proposal predicts every field's displacement on the GPU, searches
only around it and falls back to the exact full search where the proposal
is not trusted.  This module is the offline side.  It

* generates training pairs with a plain detector's field log (the network
  inputs of every searched field and the full-search result as the label),
* trains the network with the library's own forward and backward kernels
  (vsb_pnet_forward_train / vsb_pnet_backward behind a torch autograd
  Function; torch only holds the fp32 master weights, the loss and Adam),
* calibrates the fallback thresholds and writes the VSBP blob.
"""
import ctypes as C
import math
import os
import struct

import numpy as np

from ._lib import PF_YUV420P, lib, ptr

N_BF16, N_F32 = 30208, 131
PARAM_BYTES = 2 * N_BF16 + 4 * N_F32
ACT_BYTES = 2 * (32768 + 8192 + 2048 + 512)
WORK_BYTES = 4 * (32768 + 8192 + 2048 + 512)
INPUT_BYTES = 4096
HEADER = struct.Struct("<4siiiffff")
SCALE = 4.0  # network units -> pixels
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_BLOB = os.path.join(DATA_DIR, "pnet_1080p.vsbp")
LABEL_DTYPE = np.dtype([("tx", "<i2"), ("ty", "<i2"), ("sad", "<u4"), ("kind", "u1"),
                        ("ok", "u1"), ("use", "u1"), ("pad", "u1")])
assert LABEL_DTYPE.itemsize == 12

_bound = False


def _L():
    global _bound
    L = lib()
    if not _bound:
        p, i, f, l_ = C.c_void_p, C.c_int, C.c_float, C.c_long
        L.vsb_pnet_sizes.restype = i
        L.vsb_pnet_sizes.argtypes = [C.POINTER(l_)] * 4
        for name in ("vsb_pnet_forward_train",):
            getattr(L, name).restype = i
        L.vsb_pnet_forward_train.argtypes = [p, p, i, p, p, p]
        L.vsb_pnet_backward.restype = i
        L.vsb_pnet_backward.argtypes = [p, p, p, i, p, p, p, p]
        L.vsb_pnet_infer.restype = i
        L.vsb_pnet_infer.argtypes = [p, p, i, p, p]
        L.vsb_pnet_infer_items.restype = i
        L.vsb_pnet_infer_items.argtypes = [p, p, p, i, i, i, p, i, p, p]
        L.vsb_pnet_crops.restype = i
        L.vsb_pnet_crops.argtypes = [p, p, i, i, i, p, i, p, p]
        L.vsb_pnet_narrow_host.restype = i
        L.vsb_pnet_narrow_host.argtypes = [p, p, i, i, i, i, i, p, p, p, p, i, p, f, f, f,
                                           C.c_uint32, p, p, p, p, p]
        L.vsb_set_proposal.restype = i
        L.vsb_set_proposal.argtypes = [p, p, l_]
        L.vsb_set_proposal_ex.restype = i
        L.vsb_set_proposal_ex.argtypes = [p, p, l_, C.c_double, C.c_double, C.c_double]
        L.vsb_set_proposal_scope.restype = i
        L.vsb_set_proposal_scope.argtypes = [p, i, C.c_double]
        L.vsb_set_proposal_passes.restype = i
        L.vsb_set_proposal_passes.argtypes = [p, i]
        L.vsb_set_proposal_verify.restype = i
        L.vsb_set_proposal_verify.argtypes = [p, i]
        L.vsb_proposal_stats.restype = i
        L.vsb_proposal_stats.argtypes = [p, p]
        L.vsb_set_field_log.restype = i
        L.vsb_set_field_log.argtypes = [p, p, p, l_]
        L.vsb_field_log_count.restype = l_
        L.vsb_field_log_count.argtypes = [p]
        _bound = True
    return L


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed: %s" % (what, lib().vsb_last_error().decode()))


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


# ---------------------------------------------------------------- blobs ----

def pack_blob(bits, f32, scale=SCALE, radius=2.0, conf_min=0.0, match_bound=64.0):
    """VSBP bytes from bf16 bits (uint16[N_BF16]) and f32 biases."""
    bits = np.ascontiguousarray(bits, np.uint16)
    f32 = np.ascontiguousarray(f32, np.float32)
    assert bits.shape == (N_BF16,) and f32.shape == (N_F32,)
    return HEADER.pack(b"VSBP", 1, N_BF16, N_F32, scale, radius, conf_min, match_bound) + \
        bits.tobytes() + f32.tobytes()


def unpack_blob(blob):
    """(bits, f32, settings dict) of VSBP bytes"""
    magic, ver, nb, nf, scale, radius, conf_min, match_bound = HEADER.unpack_from(blob, 0)
    if magic != b"VSBP" or ver != 1 or nb != N_BF16 or nf != N_F32:
        raise ValueError("not a version-1 VSBP blob of this architecture")
    o = HEADER.size
    bits = np.frombuffer(blob, np.uint16, N_BF16, o).copy()
    f32 = np.frombuffer(blob, np.float32, N_F32, o + 2 * N_BF16).copy()
    return bits, f32, {"scale": scale, "radius": radius, "conf_min": conf_min,
                       "match_bound": match_bound}


def load_blob(path=None):
    with open(path or DEFAULT_BLOB, "rb") as f:
        return f.read()


def zero_blob(radius=2.0, conf_logit=10.0, match_bound=64.0):
    """The proposal without a network: every field predicted at zero shift
    with full confidence (the narrowed search around the coarse model's
    prediction, fallbacks still active)."""
    f32 = np.zeros(N_F32, np.float32)
    f32[130] = conf_logit
    return pack_blob(np.zeros(N_BF16, np.uint16), f32, SCALE, radius, 0.0, match_bound)


def set_proposal(det, blob, radius=-1.0, conf_min=float("nan"), match_bound=-1.0, verify=False,
                 fine_net=False, fine_radius=-1.0, passes=None):
    """Gives a MotionDetector the proposal (blob None: back to plain)."""
    L = _L()
    buf = C.create_string_buffer(blob, len(blob)) if blob is not None else None
    _check(L.vsb_set_proposal_ex(C.byref(det.md), buf, len(blob) if blob else 0, radius,
                                 conf_min, match_bound), "vsb_set_proposal_ex")
    _check(L.vsb_set_proposal_scope(C.byref(det.md), 1 if fine_net else 0, fine_radius),
           "vsb_set_proposal_scope")
    if passes is not None and blob is not None:
        _check(L.vsb_set_proposal_passes(C.byref(det.md), passes), "vsb_set_proposal_passes")
    _check(L.vsb_set_proposal_verify(C.byref(det.md), 1 if verify else 0), "vsb_set_proposal_verify")


def proposal_stats(det):
    st = (C.c_longlong * 8)()
    _check(_L().vsb_proposal_stats(C.byref(det.md), st), "vsb_proposal_stats")
    searched, fell, verified, same, cs, cf, fs, ff = [int(v) for v in st]
    return {"searched": searched, "fell_back": fell, "verified": verified, "identical": same,
            "fallback_rate": fell / searched if searched else 0.0,
            "agreement": same / verified if verified else None,
            "coarse_searched": cs, "coarse_fell_back": cf, "fine_searched": fs,
            "fine_fell_back": ff}


def kernel_ms(det, frames_fn):
    """per-frame device time of the detector's kernels while frames_fn runs:
    {blur, field_minmax, coarse_search, fine_search, network, fallback} in ms"""
    L = lib()
    L.vsb_set_kernel_timing.argtypes = [C.c_void_p, C.c_int]
    L.vsb_kernel_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.vsb_set_kernel_timing(C.byref(det.md), 1)
    frames_fn()
    ms = (C.c_double * 6)()
    cnt = (C.c_long * 6)()
    L.vsb_kernel_times(C.byref(det.md), ms, cnt)
    L.vsb_set_kernel_timing(C.byref(det.md), 0)
    names = ["blur", "field_minmax", "coarse_search", "fine_search", "network", "fallback"]
    return {k: (ms[i] / cnt[i] if cnt[i] else None) for i, k in enumerate(names)}


# ------------------------------------------------------- device kernels ----

def params_to_device(bits, f32, device="cuda"):
    """device parameter buffer (uint8 torch tensor) from bf16 bits + f32"""
    import torch
    buf = torch.empty(PARAM_BYTES, dtype=torch.uint8, device=device)
    buf[:2 * N_BF16].copy_(torch.from_numpy(np.ascontiguousarray(bits, np.uint16).view(np.uint8)))
    buf[2 * N_BF16:].copy_(torch.from_numpy(np.ascontiguousarray(f32, np.float32).view(np.uint8)))
    return buf


def forward_train(params, x, n):
    """(out [n][3] fp32, acts) with the training forward kernels"""
    import torch
    acts = torch.empty(n * ACT_BYTES, dtype=torch.uint8, device=x.device)
    out = torch.empty((n, 3), dtype=torch.float32, device=x.device)
    _check(_L().vsb_pnet_forward_train(params.data_ptr(), x.data_ptr(), n, acts.data_ptr(),
                                       out.data_ptr(), _stream()), "vsb_pnet_forward_train")
    return out, acts


def backward(params, x, acts, n, dout):
    """fp32 gradient [N_BF16 + N_F32] of sum(out * dout)"""
    import torch
    work = torch.empty(n * WORK_BYTES, dtype=torch.uint8, device=x.device)
    grad = torch.empty(N_BF16 + N_F32, dtype=torch.float32, device=x.device)
    dout = dout.contiguous().float()
    _check(_L().vsb_pnet_backward(params.data_ptr(), x.data_ptr(), acts.data_ptr(), n,
                                  dout.data_ptr(), grad.data_ptr(), work.data_ptr(), _stream()),
           "vsb_pnet_backward")
    return grad


def infer(params, x, n):
    """outputs of the detector's tensor-core inference kernel"""
    import torch
    out = torch.empty((n, 3), dtype=torch.float32, device=x.device)
    _check(_L().vsb_pnet_infer(params.data_ptr(), x.data_ptr(), n, out.data_ptr(), _stream()),
           "vsb_pnet_infer")
    return out


def infer_items(params, curr, prev, items):
    """the inference kernel reading its crops from two device planes"""
    import torch
    H, W = curr.shape
    it = torch.as_tensor(np.ascontiguousarray(items, np.int16), device=curr.device)
    n = it.shape[0]
    out = torch.empty((n, 3), dtype=torch.float32, device=curr.device)
    _check(_L().vsb_pnet_infer_items(params.data_ptr(), curr.data_ptr(), prev.data_ptr(),
                                     curr.stride(0), W, H, it.data_ptr(), n, out.data_ptr(),
                                     _stream()), "vsb_pnet_infer_items")
    return out


def crops(curr, prev, items):
    """network inputs (uint8 tensor [n][4096]) of items (int16 [n][4]: x, y,
    ox, oy) on two device planes (uint8 torch tensors H x W)"""
    import torch
    H, W = curr.shape
    it = torch.as_tensor(np.ascontiguousarray(items, np.int16), device=curr.device)
    n = it.shape[0]
    out = torch.empty((n, INPUT_BYTES), dtype=torch.uint8, device=curr.device)
    _check(_L().vsb_pnet_crops(curr.data_ptr(), prev.data_ptr(), curr.stride(0), W, H,
                               it.data_ptr(), n, out.data_ptr(), _stream()), "vsb_pnet_crops")
    return out


class _NetFn:
    """torch autograd Function over the library's kernels (built lazily so
    importing this module does not import torch)."""
    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            import torch

            class PNetFunction(torch.autograd.Function):
                @staticmethod
                def forward(ctx, master, x):
                    params = master_to_params(master)
                    n = x.shape[0]
                    out, acts = forward_train(params, x, n)
                    ctx.save_for_backward(params, x, acts)
                    return out

                @staticmethod
                def backward(ctx, dout):
                    params, x, acts = ctx.saved_tensors
                    return backward(params, x, acts, x.shape[0], dout), None

            cls.fn = PNetFunction
        return cls.fn


def master_to_params(master):
    """fp32 master vector -> device parameter buffer (bf16 weights, f32 biases)"""
    import torch
    buf = torch.empty(PARAM_BYTES, dtype=torch.uint8, device=master.device)
    buf[:2 * N_BF16].view(torch.bfloat16).copy_(master[:N_BF16].detach())
    buf[2 * N_BF16:].view(torch.float32).copy_(master[N_BF16:].detach())
    return buf


def init_master(seed=0, device="cuda"):
    """He-initialised fp32 master vector (parameter order)"""
    import torch
    rng = np.random.default_rng(seed)
    w1 = np.zeros((32, 32))
    w1[:, :18] = rng.normal(0, math.sqrt(2.0 / 18), (32, 18))
    parts = [w1.ravel()] + [rng.normal(0, math.sqrt(2.0 / 288), 9216) for _ in range(3)]
    parts.append(rng.normal(0, math.sqrt(1.0 / 512), 1536))
    b = np.zeros(N_F32)
    b[:128] = 0.01
    v = np.concatenate(parts + [b]).astype(np.float32)
    return torch.tensor(v, device=device, requires_grad=True)


def master_bits(master):
    import torch
    m = master.detach()
    bits = m[:N_BF16].to(torch.bfloat16).view(torch.int16).cpu().numpy().view(np.uint16)
    return bits.copy(), m[N_BF16:].cpu().numpy().astype(np.float32)


# ------------------------------------------------------- training data ----

def field_log(clip, width, height, cap, stepsize=6, accuracy=15, shakiness=5, mincontrast=0.25):
    """Runs a plain detector over a device clip (uint8 torch tensor n x H x W)
    with the field log on.  Returns (inputs uint8 [m][4096], labels numpy
    LABEL_DTYPE [m]) on the clip's device."""
    import torch
    from .api import MotionDetector
    L = _L()
    det = MotionDetector(width, height, PF_YUV420P, stepsize=stepsize, accuracy=accuracy,
                         shakiness=shakiness, mincontrast=mincontrast)
    inputs = torch.empty((cap, INPUT_BYTES), dtype=torch.uint8, device=clip.device)
    labels = torch.empty((cap, 12), dtype=torch.uint8, device=clip.device)
    _check(L.vsb_set_field_log(C.byref(det.md), inputs.data_ptr(), labels.data_ptr(), cap),
           "vsb_set_field_log")
    n = clip.shape[0]
    rec = np.zeros(n * 512 + 64, dtype=np.dtype((np.void, 32)))
    cnt = np.zeros(n, np.int32)
    det.run(n, clip.data_ptr(), width * height, width, True, rec, cnt)
    torch.cuda.synchronize()
    m = int(L.vsb_field_log_count(C.byref(det.md)))
    det.close()
    lab = labels[:m].cpu().numpy().view(LABEL_DTYPE).reshape(m)
    return inputs[:m], lab


# ------------------------------------------------------------- training ----

def train(inputs, labels, steps=3000, batch=512, lr=2e-3, seed=0, radius=2.0, log=None,
          master=None, coarse_weight=1.0):
    """Trains the network on logged pairs with the library's kernels.
    inputs: uint8 [m][4096] device tensor; labels: LABEL_DTYPE numpy;
    coarse pairs are drawn coarse_weight times as often as fine ones.
    Returns the fp32 master vector."""
    import torch
    dev = inputs.device
    use = np.nonzero(labels["use"] == 1)[0]
    x_all = inputs[torch.as_tensor(use, device=dev)]
    t_all = torch.as_tensor(np.stack([labels["tx"][use], labels["ty"][use]], 1).astype(np.float32),
                            device=dev)
    wts = torch.as_tensor(np.where(labels["kind"][use] == 0, coarse_weight, 1.0), device=dev,
                          dtype=torch.float32)
    m = x_all.shape[0]
    if master is None:
        master = init_master(seed, dev)
    opt = torch.optim.Adam([master], lr=lr)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=steps, pct_start=0.1)
    fn = _NetFn.get()
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    hist = []
    for step in range(steps):
        idx = torch.multinomial(wts, batch, replacement=True, generator=g)
        x = x_all[idx].view(torch.bfloat16).view(batch, 32, 32, 2).contiguous()
        t = t_all[idx]
        out = fn.apply(master, x)
        pred = out[:, :2] * SCALE
        err = (pred.detach() - t).abs().amax(dim=1)
        conf_t = (err <= radius).float()
        loss = torch.nn.functional.smooth_l1_loss(out[:, :2], t / SCALE, beta=0.25) + \
            0.2 * torch.nn.functional.binary_cross_entropy_with_logits(out[:, 2], conf_t)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        torch.nn.utils.clip_grad_norm_([master], 5.0)
        opt.step()
        sched.step()
        if log is not None and (step % 200 == 0 or step == steps - 1):
            rec = (step, float(loss.detach()), float(conf_t.mean()))
            hist.append(rec)
            log(rec)
    return master


def evaluate(params, inputs, labels, kind=None):
    """outputs of the inference kernel on logged items (use == 1, optional
    kind filter): (out numpy [k][3], targets [k][2], sad, kind)"""
    import torch
    sel = labels["use"] == 1
    if kind is not None:
        sel &= labels["kind"] == kind
    idx = np.nonzero(sel)[0]
    outs = []
    for a in range(0, len(idx), 8192):
        b = idx[a:a + 8192]
        x = inputs[torch.as_tensor(b, device=inputs.device)].contiguous()
        outs.append(infer(params, x, len(b)).cpu().numpy())
    out = np.concatenate(outs) if outs else np.zeros((0, 3), np.float32)
    tgt = np.stack([labels["tx"][idx], labels["ty"][idx]], 1).astype(np.float32)
    return out, tgt, labels["sad"][idx], labels["kind"][idx]


def calibrate(params, inputs, labels, sizes, radius=2.0, target=0.999, match_quantile=0.998):
    """Fallback thresholds from validation pairs: conf_min, the lowest logit
    at which at least `target` of the accepted predictions lie within the
    radius, and match_bound, a high quantile of the labels' SAD per pixel.
    sizes: {kind: field size}."""
    out, tgt, sad, kind = evaluate(params, inputs, labels)
    err = np.abs(out[:, :2] * SCALE - tgt).max(axis=1)
    hit = err <= radius
    order = np.argsort(-out[:, 2])
    cum = np.cumsum(hit[order]) / np.arange(1, len(order) + 1)
    ok = np.nonzero(cum >= target)[0]
    conf_min = float(out[order[ok[-1]], 2]) if len(ok) else float(out[:, 2].max() + 1)
    pp = np.array([sad[i] / float(sizes[int(kind[i])] ** 2) for i in range(len(sad))])
    match_bound = float(np.quantile(pp, match_quantile)) if len(pp) else 64.0
    acc = float((out[:, 2] >= conf_min).mean()) if len(out) else 0.0
    return {"conf_min": conf_min, "match_bound": match_bound, "accept_rate": acc,
            "hit_rate": float(hit.mean()) if len(hit) else 0.0,
            "mean_abs_err_px": float(np.abs(out[:, :2] * SCALE - tgt).mean()) if len(hit) else 0.0}


def narrow_host(curr, prev, xs, ys, size, max_shift, step, pout, ox=None, oy=None, scale=SCALE,
                radius=2.0, conf_min=0.0, sad_bound=0xFFFFFFFF):
    """Narrowed search of one planar field set on host planes given raw
    network outputs pout [n][3]: (sad, tx, ty, ok, flags)"""
    L = _L()
    curr = np.ascontiguousarray(curr, np.uint8)
    prev = np.ascontiguousarray(prev, np.uint8)
    H, W = curr.shape
    n = len(xs)
    xs = np.ascontiguousarray(xs, np.int16)
    ys = np.ascontiguousarray(ys, np.int16)
    ox = np.ascontiguousarray(ox if ox is not None else np.zeros(n), np.int16)
    oy = np.ascontiguousarray(oy if oy is not None else np.zeros(n), np.int16)
    po = np.ascontiguousarray(pout, np.float32).reshape(n, 3)
    sad = np.zeros(n, np.uint32)
    tx = np.zeros(n, np.int16)
    ty = np.zeros(n, np.int16)
    ok = np.zeros(n, np.int32)
    fl = np.zeros(n, np.uint8)
    _check(L.vsb_pnet_narrow_host(ptr(curr), ptr(prev), W, H, size, max_shift, step, ptr(xs),
                                  ptr(ys), ptr(ox), ptr(oy), n, ptr(po), scale, radius, conf_min,
                                  sad_bound, ptr(sad), ptr(tx), ptr(ty), ptr(ok), ptr(fl)),
           "vsb_pnet_narrow_host")
    return sad, tx, ty, ok, fl
