"""The allocation-free field search (vsb_field_search_noalloc) through the C
ABI.

It exists for callers that cannot let a library allocate GPU memory: hosts
that hand out all device memory from their own pools, or hold it to a
budget, where an allocation they did not make breaks their accounting.  Its
scratch lives in a static device array instead.  The test owns every device
buffer the call touches and checks, on calls in a row that reuse the shared
scratch:

* every field's (SAD, shift, range test) equals the library's regular
  search (vsb_field_search_host) and, for a sample of fields, the oracle's
  restatement of the reference's spiral search -- over several lattice
  geometries, which also pins the entry point's own spiral rank table;
* a call allocates nothing: on the second call of each geometry the
  library's device-allocation counter does not move, a device allocation
  armed to fail is never reached, and the free device memory is unchanged;
* oversized inputs are rejected before any device work.

The file sorts last so that a stopping run has executed every other test
first; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import vidstab_b200 as V
from vidstab_b200 import synthetic as S

pytestmark = pytest.mark.gpu

RES_DTYPE = np.dtype([("sad", "<u4"), ("tx", "<i2"), ("ty", "<i2"), ("ok", "<i4")])
ITEM_DTYPE = np.dtype([("x", "<i2"), ("y", "<i2"), ("ox", "<i2"), ("oy", "<i2")])


def bind():
    L = V.lib()
    L.vsb_field_search_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.vsb_last_error.restype = C.c_char_p
    return L


def device_plane(torch, img, pitch):
    """frame on the device with the given row pitch and 256 bytes of slack"""
    h, w = img.shape
    buf = torch.zeros(pitch * h + 256, dtype=torch.uint8, device="cuda")
    host = np.zeros(pitch * h + 256, np.uint8)
    host[:pitch * h].reshape(h, pitch)[:, :w] = img
    buf.copy_(torch.from_numpy(host))
    return buf


def noalloc(torch, L, d_curr, d_prev, pitch, size, ms, step, d_items, d_res, n):
    rc = L.vsb_field_search_noalloc(C.c_void_p(d_curr.data_ptr()), C.c_void_p(d_prev.data_ptr()),
                                    pitch, size, ms, step, C.c_void_p(d_items.data_ptr()), n,
                                    C.c_void_p(d_res.data_ptr()), None)
    assert rc == 0, L.vsb_last_error()
    torch.cuda.synchronize()
    return d_res.cpu().numpy()[:n * RES_DTYPE.itemsize].view(RES_DTYPE)


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


# (field size, maxShift, step, fields, lattice offsets): the 720p coarse and
# fine geometries of vsMotionDetection, then other steps of the spiral
RUNS = [(80, 102, 6, 40, False), (16, 16, 2, 300, True), (48, 40, 4, 24, True),
        (32, 30, 3, 24, False), (64, 50, 5, 16, True), (32, 12, 1, 24, False)]


def test_noalloc_matches_regular_search_and_oracle():
    torch = pytest.importorskip("torch")
    L = bind()
    w, h = 1280, 720
    fr = S.clip(w, h, 2, seed=77, trans_sigma=4.0)
    curr, prev = fr[1], fr[0]
    pitch = 1280
    d_curr = device_plane(torch, curr, pitch)
    d_prev = device_plane(torch, prev, pitch)
    # every buffer the calls touch, allocated by the test up front
    cap = max(r[3] for r in RUNS)
    d_items = torch.zeros(cap * ITEM_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_res = torch.zeros(cap * RES_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    runs = [(s, m, st, fields(w, h, s, m, st, n, k, off)) for k, (s, m, st, n, off)
            in enumerate(RUNS)]
    runs.append(runs[0])  # the first geometry again after the scratch held others
    orc = O.orc()
    for size, ms, step, items in runs:
        n = len(items)
        d_items[:n * ITEM_DTYPE.itemsize].copy_(torch.from_numpy(items.view(np.uint8).copy()))
        # a first call (which may load kernels into the context), then a
        # second one during which any device allocation by the library fails
        got = noalloc(torch, L, d_curr, d_prev, pitch, size, ms, step, d_items, d_res, n).copy()
        allocs0 = L.vsb_test_device_alloc(0, 1)
        free0 = torch.cuda.mem_get_info()[0]
        try:
            again = noalloc(torch, L, d_curr, d_prev, pitch, size, ms, step, d_items, d_res, n)
        finally:
            allocs1 = L.vsb_test_device_alloc(-1, 0)
        assert allocs1 == allocs0, "the allocation-free search allocated device memory"
        assert torch.cuda.mem_get_info()[0] == free0
        assert np.array_equal(again, got)
        sad, tx, ty, ok = V.field_search(curr, prev, items["x"], items["y"], size, ms, step,
                                         items["ox"], items["oy"])
        assert np.array_equal(got["sad"], sad)
        assert np.array_equal(got["tx"], tx)
        assert np.array_equal(got["ty"], ty)
        assert np.array_equal(got["ok"] != 0, ok != 0)
        # the oracle's spiral search (src/motiondetect.c:439-586 restated)
        for i in range(0, n, max(1, n // 8)):
            otx, oty, oe = C.c_int(), C.c_int(), C.c_uint32()
            cur = np.ascontiguousarray(curr)
            prv = np.ascontiguousarray(prev)
            r = orc.orc_search_planar(cur.ctypes.data, w, prv.ctypes.data, w, int(items["x"][i]),
                                      int(items["y"][i]), size, ms, step, int(items["ox"][i]),
                                      int(items["oy"][i]), C.byref(otx), C.byref(oty),
                                      C.byref(oe))
            assert (got["ok"][i] != 0) == (r != 0)
            assert got["sad"][i] == oe.value
            assert (got["tx"][i], got["ty"][i]) == (otx.value, oty.value)


def test_noalloc_rejects_oversized_input():
    torch = pytest.importorskip("torch")
    L = bind()
    buf = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    # too many fields: rejected before any device work
    assert L.vsb_field_search_noalloc(p, p, 64, 32, 32, 2, p, 100000, p, None) != 0
    assert b"at most" in L.vsb_last_error()
    # a lattice larger than the scratch holds
    assert L.vsb_field_search_noalloc(p, p, 64, 32, 400, 1, p, 4, p, None) != 0
    assert b"at most" in L.vsb_last_error()
    # a shift range beyond 16 bits with a small lattice (100000 / 2000 = 50 steps)
    assert L.vsb_field_search_noalloc(p, p, 64, 32, 100000, 2000, p, 4, p, None) != 0
    assert b"16 bits" in L.vsb_last_error()
