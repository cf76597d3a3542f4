"""The allocation-free field search (vsb_field_search_noalloc) through the C
ABI, against the library's regular field search on the same inputs.

It exists for callers that cannot let a library allocate GPU memory (hosts
that own device memory through their own pools or budgets, or that call while
recording a CUDA graph): its scratch lives in a static device array.  The test
owns every device buffer the call touches, runs two different searches back
to back (the shared scratch must be reset between them) and repeats the first
one, comparing every field's (SAD, shift, range test) with vsb_field_search_host.
The file sorts last so that a stopping run has executed every other test
first; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import vidstab_b200 as V
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu

RES_DTYPE = np.dtype([("sad", "<u4"), ("tx", "<i2"), ("ty", "<i2"), ("ok", "<i4")])
ITEM_DTYPE = np.dtype([("x", "<i2"), ("y", "<i2"), ("ox", "<i2"), ("oy", "<i2")])


def device_plane(torch, img, pitch):
    """frame on the device with the given row pitch and 256 bytes of slack"""
    h, w = img.shape
    buf = torch.zeros(pitch * h + 256, dtype=torch.uint8, device="cuda")
    host = np.zeros(pitch * h + 256, np.uint8)
    host[:pitch * h].reshape(h, pitch)[:, :w] = img
    buf.copy_(torch.from_numpy(host))
    return buf


def noalloc(torch, L, d_curr, d_prev, pitch, size, ms, step, items):
    d_items = torch.from_numpy(items.view(np.uint8).copy()).cuda()
    d_res = torch.zeros(len(items) * RES_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    rc = L.vsb_field_search_noalloc(C.c_void_p(d_curr.data_ptr()), C.c_void_p(d_prev.data_ptr()),
                                    pitch, size, ms, step, C.c_void_p(d_items.data_ptr()),
                                    len(items), C.c_void_p(d_res.data_ptr()), None)
    assert rc == 0, L.vsb_last_error()
    torch.cuda.synchronize()
    return d_res.cpu().numpy().view(RES_DTYPE)


def regular(curr, prev, size, ms, step, items):
    sad, tx, ty, ok = V.field_search(curr, prev, items["x"], items["y"], size, ms, step,
                                     items["ox"], items["oy"])
    return sad, tx, ty, ok


def fields(w, h, size, ms, step, n, seed, offsets):
    rng = np.random.default_rng(seed)
    reach = size // 2 + ms + step + 4
    it = np.zeros(n, ITEM_DTYPE)
    it["x"] = rng.integers(reach, w - reach, n)
    it["y"] = rng.integers(reach, h - reach, n)
    if offsets:
        it["ox"] = rng.integers(-3, 4, n)
        it["oy"] = rng.integers(-3, 4, n)
    return it


def test_noalloc_matches_regular_search_twice():
    torch = pytest.importorskip("torch")
    L = V.lib()
    L.vsb_field_search_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.vsb_last_error.restype = C.c_char_p
    w, h = 1280, 720
    fr = S.clip(w, h, 2, seed=77, trans_sigma=4.0)
    curr, prev = fr[1], fr[0]
    pitch = 1280
    d_curr = device_plane(torch, curr, pitch)
    d_prev = device_plane(torch, prev, pitch)
    runs = [(112, 102, 6, fields(w, h, 112, 102, 6, 40, 1, False)),
            (32, 32, 2, fields(w, h, 32, 32, 2, 300, 2, True))]
    runs.append(runs[0])
    for size, ms, step, items in runs:
        got = noalloc(torch, L, d_curr, d_prev, pitch, size, ms, step, items)
        sad, tx, ty, ok = regular(curr, prev, size, ms, step, items)
        assert np.array_equal(got["sad"], sad)
        assert np.array_equal(got["tx"], tx)
        assert np.array_equal(got["ty"], ty)
        assert np.array_equal(got["ok"] != 0, ok != 0)


def test_noalloc_rejects_oversized_input():
    torch = pytest.importorskip("torch")
    L = V.lib()
    L.vsb_field_search_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.vsb_last_error.restype = C.c_char_p
    buf = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    # too many fields: rejected before any device work
    assert L.vsb_field_search_noalloc(p, p, 64, 32, 32, 2, p, 100000, p, None) != 0
    assert b"at most" in L.vsb_last_error()
    # a lattice larger than the scratch holds
    assert L.vsb_field_search_noalloc(p, p, 64, 32, 400, 1, p, 4, p, None) != 0
    assert b"at most" in L.vsb_last_error()
