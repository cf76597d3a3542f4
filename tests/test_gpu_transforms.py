"""The second pass on the GPU (vsb_l2t.cu: vsLocalmotions2Transforms' fit,
one warp per frame) against the reference's outputs: the committed fixture
(tests/golden/transforms.npz, made by the reference), the live reference
build, and the drop-in entry points fed from a .trf file as the transform
pass reads it.

Tolerance.  The kernel follows the reference build's rounding step by step;
the only operations that may round differently are cos/sin (CUDA's against
glibc's).  A last-bit difference there can flip a descent step whose two
objective values are that close, after which the two descents end at
slightly different points of the same minimum.  So: every frame's `extra`
flag must agree, every value must be within TOL (pixels for x/y, radians
for alpha, percent for zoom), and at least MIN_IDENTICAL of all frames must
be bit-identical."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import _lib
from vidstab_b200 import synthetic as S
from test_transforms_host import (golden_cases, ref_transforms, many_motions, free_many,
                                  transform_data)

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")

TOL = np.array([1e-3, 1e-3, 1e-5, 1e-3])
MIN_IDENTICAL = 0.97


def rows(t):
    return np.stack([t["x"], t["y"], t["alpha"], t["zoom"], t["extra"].astype(np.float64)], 1)


def compare(mine, ref, label):
    """(identical frames, frames); asserts the tolerance"""
    assert mine.shape == ref.shape, label
    assert np.array_equal(mine[:, 4], ref[:, 4]), label
    d = np.abs(mine[:, :4] - ref[:, :4])
    assert np.all(d <= TOL), (label, d.max(0))
    return int((mine == ref).all(1).sum()), len(ref)


def test_kernel_matches_golden():
    same = total = 0
    for label, recs, first, W, H, fov, sz, ref in golden_cases():
        counts = np.diff(first)
        out, resid, info = V.motions_to_transforms(recs, counts, W, H, fov, sz)
        s, n = compare(rows(out), ref, label)
        same += s
        total += n
        # rounds 1..3 for frames with motions, 0 for empty ones
        assert np.all((info[:, 0] >= 1) == (counts > 0)) and np.all(info[:, 0] <= 3), label
    assert same >= MIN_IDENTICAL * total, (same, total)


def test_edge_shapes():
    """no frames; frames without motions only; one frame at the capacity; one
    over it (refused before any launch, the next call still works)"""
    L = V.lib()
    out, _, _ = V.motions_to_transforms(np.zeros(0, V.LM_DTYPE), [], 1920, 1080)
    assert len(out) == 0
    out, resid, info = V.motions_to_transforms(np.zeros(0, V.LM_DTYPE), [0, 0, 0], 1920, 1080)
    assert np.all(out["extra"] == 1) and np.all(np.isnan(resid)) and np.all(info == 0)
    cap = L.vsb_motions_to_transforms_capacity()
    rng = np.random.default_rng(3)
    r = np.zeros(cap + 1, V.LM_DTYPE)
    r["fx"] = rng.integers(0, 3840, cap + 1)
    r["fy"] = rng.integers(0, 2160, cap + 1)
    r["vx"] = 3
    r["vy"] = -2
    r["match"] = rng.gamma(3.0, 2.0, cap + 1)
    with pytest.raises(RuntimeError, match="capacity"):
        V.motions_to_transforms(r, [cap + 1], 3840, 2160)
    out, _, _ = V.motions_to_transforms(r[:cap], [cap], 3840, 2160)
    assert abs(out["x"][0] - 3) < 1e-3 and abs(out["y"][0] + 2) < 1e-3 and out["extra"][0] == 0


@needs_ref
def test_kernel_matches_live_reference_4k_and_batch():
    """a 4K clip's motions (760 fine fields a frame) and many streams' frames
    in one launch: each frame's result does not depend on its neighbours"""
    frames = np.asarray(S.clip(3840, 2160, 4, seed=41))
    recs, counts, _ = O.ref_clip(frames)
    first = np.zeros(len(counts) + 1, np.int64)
    first[1:] = np.cumsum(counts)
    ref = ref_transforms(recs, first, 3840, 2160, 0.0, 0)
    out, _, _ = V.motions_to_transforms(recs, counts, 3840, 2160)
    compare(rows(out), ref, "4k")
    # 64 copies of the clip in one launch give 64 copies of the result
    big_recs = np.concatenate([recs] * 64)
    big_counts = np.concatenate([counts] * 64)
    before = V.lib().vsb_motions_to_transforms_launches()
    big, _, _ = V.motions_to_transforms(big_recs, big_counts, 3840, 2160)
    assert V.lib().vsb_motions_to_transforms_launches() == before + 1
    assert np.array_equal(rows(big), np.concatenate([rows(out)] * 64))


def test_device_entry_matches_host_entry():
    """vsb_motions_to_transforms_device on device buffers, on torch's stream"""
    import torch
    L = V.lib()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "transforms.npz"))
    recs, counts = g["clip1080_recs"], g["clip1080_counts"]
    first = np.zeros(len(counts) + 1, np.int64)
    first[1:] = np.cumsum(counts)
    n = len(counts)
    host, hres, hinfo = V.motions_to_transforms(recs, counts, 1920, 1080, 70.0, 1)
    d_recs = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
    d_first = torch.from_numpy(first).cuda()
    d_out = torch.zeros(n * V.TRANSFORM_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_res = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_info = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert L.vsb_motions_to_transforms_device(d_recs.data_ptr(), d_first.data_ptr(), n,
                                              int(counts.max()), 1920, 1080, 70.0, 1,
                                              d_out.data_ptr(), d_res.data_ptr(),
                                              d_info.data_ptr(), st) == 0
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(V.TRANSFORM_DTYPE)
    assert np.array_equal(rows(out), rows(host))
    assert np.array_equal(d_res.cpu().numpy(), hres, equal_nan=True)
    assert np.array_equal(d_info.cpu().numpy().reshape(n, 3), hinfo)


def _libc():
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    return libc


@needs_ref
@pytest.mark.parametrize("fov,smooth_zoom", [(0.0, 0), (80.0, 1)])
def test_dropin_from_trf_matches_reference(tmp_path, monkeypatch, fov, smooth_zoom):
    """The transform pass's input path: a .trf written by the reference's
    detect, read back by each library's vsReadLocalMotionsFile and fitted by
    its vsLocalmotions2Transforms with storeTransforms on; the transforms and
    the global_motions.trf files of the two agree"""
    L, libc = V.lib(), _libc()
    W, H, N = 960, 540, 10
    frames = np.asarray(S.clip(W, H, N, seed=13))
    trf = str(tmp_path / "motions.trf")
    O.ref_clip(frames, trf_path=trf)
    # reference, in its own directory
    R = O.ref()
    R.vsref_trf_to_transforms.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                          C.c_int, C.c_void_p, C.c_int]
    TD = np.dtype([("x", "<f8"), ("y", "<f8"), ("alpha", "<f8"), ("zoom", "<f8"),
                   ("barrel", "<f8"), ("rshutter", "<f8"), ("extra", "<i4"), ("pad", "<i4")])
    rdir, mdir = tmp_path / "ref", tmp_path / "mine"
    rdir.mkdir()
    mdir.mkdir()
    ref = np.zeros(N + 4, TD)
    monkeypatch.chdir(rdir)
    nref = R.vsref_trf_to_transforms(trf.encode(), W, H, fov, smooth_zoom, 1, ref.ctypes.data,
                                     N + 4)
    assert nref >= N - 1
    # this library
    monkeypatch.chdir(mdir)
    L.vsReadLocalMotionsFile.restype = C.c_int
    L.vsReadLocalMotionsFile.argtypes = [C.c_void_p, C.POINTER(_lib.VSVector)]
    f = libc.fopen(trf.encode(), b"rb")
    mlms = _lib.VSVector()
    assert L.vsReadLocalMotionsFile(f, C.byref(mlms)) == 0
    libc.fclose(f)
    td = transform_data(W, H, fov=fov, smooth_zoom=smooth_zoom, store=1)
    tr = _lib.VSTransformations()
    try:
        assert L.vsLocalmotions2Transforms(C.byref(td), C.byref(mlms), C.byref(tr)) == 0
        assert tr.len == nref
        mine = np.array([[tr.ts[k].x, tr.ts[k].y, tr.ts[k].alpha, tr.ts[k].zoom, tr.ts[k].extra]
                         for k in range(tr.len)])
        C.CDLL(None).free(C.cast(tr.ts, C.c_void_p))
    finally:
        free_many(L, mlms)
    refrows = np.stack([ref["x"], ref["y"], ref["alpha"], ref["zoom"],
                        ref["extra"].astype(np.float64)], 1)[:nref]
    same, n = compare(mine, refrows, "trf")
    a = (rdir / "global_motions.trf").read_text().splitlines()
    b = (mdir / "global_motions.trf").read_text().splitlines()
    assert len(a) == len(b) == 2 * nref
    if same == n:
        assert a == b
    else:
        for la, lb in zip(a, b):
            if la.startswith("#"):
                continue
            assert np.allclose([float(v) for v in la.split()], [float(v) for v in lb.split()],
                               atol=2e-6)


def test_motions_to_transform_one_frame(tmp_path):
    """vsMotionsToTransform: one frame, its global_motions.trf line into the
    caller's FILE*; the same numbers as the batched call"""
    L, libc = V.lib(), _libc()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "transforms.npz"))
    recs, counts = g["clip640_recs"], g["clip640_counts"]
    k = 3
    lo = int(counts[:k].sum())
    r = np.ascontiguousarray(recs[lo:lo + counts[k]])
    batched, resid, info = V.motions_to_transforms(r, [len(r)], 640, 480)
    mlms = many_motions(L, r, np.array([0, len(r)], np.int64))
    lms = C.cast(L.vs_vector_get(C.byref(mlms), 0), C.POINTER(_lib.VSVector))
    path = str(tmp_path / "line.txt")
    f = libc.fopen(path.encode(), b"w")
    td = transform_data(640, 480)
    try:
        t = L.vsMotionsToTransform(C.byref(td), lms, f)
    finally:
        libc.fclose(f)
        free_many(L, mlms)
    assert (t.x, t.y, t.alpha, t.zoom, t.extra) == tuple(rows(batched)[0][:4]) + (0,)
    line = open(path).read().splitlines()
    assert line[0] == "0 %f %f %f %f %i" % (t.x, t.y, t.alpha, t.zoom, t.extra)
    assert line[1] == "#\t\t\t\t\t %f %i" % (resid[0], info[0, 0])
