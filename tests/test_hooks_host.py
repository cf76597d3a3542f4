"""The runtime allocation hooks (src/vidstabdefines.h:84-99 of the
reference: vs_malloc, vs_zalloc, vs_realloc are pointers a host such as
ffmpeg replaces) made to fail on the host, without a GPU: the vector and
frame helpers report VS_ERROR and leave valid state instead of crashing."""
import ctypes as C

import pytest

import vidstab_b200 as V
from vidstab_b200._lib import VSVector

_libc = C.CDLL(None)
_libc.malloc.restype = C.c_void_p
_libc.malloc.argtypes = [C.c_size_t]
_libc.calloc.restype = C.c_void_p
_libc.calloc.argtypes = [C.c_size_t, C.c_size_t]
_libc.realloc.restype = C.c_void_p
_libc.realloc.argtypes = [C.c_void_p, C.c_size_t]

MALLOC_T = C.CFUNCTYPE(C.c_void_p, C.c_size_t)
REALLOC_T = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t)


class FailingHooks:
    """Installs vs_malloc / vs_zalloc / vs_realloc that succeed `after`
    times, then fail (return NULL) until removed; counts the calls."""

    NAMES = ("vs_malloc", "vs_zalloc", "vs_realloc")

    def __init__(self, after):
        self.left = after
        self.calls = 0
        self.failed = 0

    def _ok(self):
        self.calls += 1
        if self.left == 0:
            self.failed += 1
            return False
        self.left -= 1
        return True

    def __enter__(self):
        L = V.lib()
        self.slots = [C.c_void_p.in_dll(L, n) for n in self.NAMES]
        self.saved = [s.value for s in self.slots]
        self.cbs = [MALLOC_T(lambda n: _libc.malloc(n) if self._ok() else None),
                    MALLOC_T(lambda n: _libc.calloc(1, n) if self._ok() else None),
                    REALLOC_T(lambda p, n: _libc.realloc(p, n) if self._ok() else None)]
        for s, cb in zip(self.slots, self.cbs):
            s.value = C.cast(cb, C.c_void_p).value
        return self

    def __exit__(self, *exc):
        for s, v in zip(self.slots, self.saved):
            s.value = v
        return False


def test_vector_reports_failed_allocations():
    L = V.lib()
    L.vs_vector_init.argtypes = [C.POINTER(VSVector), C.c_int]
    L.vs_vector_append_dup.argtypes = [C.POINTER(VSVector), C.c_void_p, C.c_int]
    L.vs_vector_size.argtypes = [C.POINTER(VSVector)]
    L.vs_vector_del.argtypes = [C.POINTER(VSVector)]
    item = (C.c_ubyte * 32)()
    v = VSVector()
    with FailingHooks(0) as h:
        assert L.vs_vector_init(C.byref(v), 4) != 0
        assert L.vs_vector_append_dup(C.byref(v), item, 32) != 0
        assert L.vs_vector_size(C.byref(v)) == 0
    assert h.failed >= 2
    # a vector that grows past its buffer while the reallocation fails keeps
    # its elements
    assert L.vs_vector_init(C.byref(v), 1) == 0
    assert L.vs_vector_append_dup(C.byref(v), item, 32) == 0
    with FailingHooks(1):  # the element copy succeeds, the growth fails
        assert L.vs_vector_append_dup(C.byref(v), item, 32) != 0
    assert L.vs_vector_size(C.byref(v)) == 1
    assert L.vs_vector_append_dup(C.byref(v), item, 32) == 0
    assert L.vs_vector_size(C.byref(v)) == 2
    L.vs_vector_del(C.byref(v))


def test_frame_allocate_reports_failure():
    from vidstab_b200._lib import VSFrame, VSFrameInfo
    L = V.lib()
    fi = VSFrameInfo()
    assert L.vsFrameInfoInit(C.byref(fi), 64, 48, V.PF_YUV420P)
    f = VSFrame()
    with FailingHooks(1):  # luma succeeds, the first chroma plane fails
        L.vsFrameAllocate(C.byref(f), C.byref(fi))
    L.vsFrameFree.argtypes = [C.POINTER(VSFrame)]
    L.vsFrameFree(C.byref(f))  # frees what was allocated, no crash


@pytest.mark.parametrize("after", [0, 1, 2])
def test_init_without_a_device_or_memory_fails_cleanly(after):
    """vsMotionDetectInit with failing hooks (and, in this CPU-only
    container, no GPU) returns VS_ERROR; the detector struct stays
    uninitialised"""
    with FailingHooks(after):
        with pytest.raises((RuntimeError, ValueError)):
            V.MotionDetector(640, 360, V.PF_YUV420P)
