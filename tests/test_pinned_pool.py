"""The host side's pinned-buffer pool (chiaro_b200.runtime.PinnedPool) with a fake
allocator: buffers are lent to numpy arrays, come back when the arrays (and their
views) are gone, and are handed out again, with no lock on the return path."""
import ctypes as C
import gc

import numpy as np

from chiaro_b200 import abi, runtime


class FakeLib:
    def __init__(self):
        self.blocks = {}

    def chiaro_host_alloc(self, nbytes, out):
        buf = (C.c_char * nbytes)()
        self.blocks[C.addressof(buf)] = buf
        C.cast(out, C.POINTER(C.c_void_p))[0] = C.addressof(buf)
        return abi.OK


def test_pool_lends_recycles_and_keeps_views_alive():
    lib = FakeLib()
    pool = runtime.PinnedPool(lib)
    a = pool.empty(1000, np.float32)
    a[:] = np.arange(1000)
    view = a[10:20]
    addr = a.ctypes.data
    del a
    gc.collect()
    assert view[0] == 10.0 and len(lib.blocks) == 1  # the view keeps the buffer lent
    b = pool.empty(1000, np.float32)
    assert b.ctypes.data != addr  # still lent: a new buffer
    del view
    gc.collect()
    c = pool.empty(4000 // 8, np.float64)  # same byte size: the first buffer again
    assert c.ctypes.data == addr and len(lib.blocks) == 2
    assert c.shape == (500,) and c.dtype == np.float64
    del b, c


def test_release_during_allocation_does_not_deadlock():
    lib = FakeLib()
    pool = runtime.PinnedPool(lib)
    arrays = [pool.empty(64, np.uint8) for _ in range(50)]
    del arrays
    with pool.lock:  # a finalizer that runs while the pool is busy must not block
        gc.collect()
    assert len(pool.returned) == 50
    again = [pool.empty(64, np.uint8) for _ in range(50)]
    assert len(lib.blocks) == 50 and not pool.returned
    del again


def test_pinned_pool_singleton_loads_the_library_outside_its_lock():
    assert runtime.pinned_pool() is runtime.pinned_pool()
