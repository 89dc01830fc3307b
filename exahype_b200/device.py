"""Device memory, streams and timers through the library's C ABI (no
framework dependency): enough plumbing for the tests, the benchmark and the
serving loop to hold data on the GPU and time kernels with CUDA events."""
import ctypes as C

import numpy as np

from ._lib import call, lib


class DeviceBuffer:
    """A cudaMalloc'd buffer of float64 (or int32) elements."""

    def __init__(self, n, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        self.nbytes = max(1, self.n * self.dtype.itemsize)
        p = C.c_void_p()
        call('exa_device_alloc', self.nbytes, C.byref(p))
        self.ptr = p

    @classmethod
    def from_array(cls, a, stream=None):
        a = np.ascontiguousarray(a)
        b = cls(a.size, a.dtype)
        b.upload(a, stream)
        return b

    def upload(self, a, stream=None):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.size <= self.n
        call('exa_memcpy_h2d', self.ptr, a.ctypes.data, a.nbytes, stream)
        if stream is None:
            call('exa_stream_synchronize', None)

    def download(self, out=None, stream=None):
        if out is None:
            out = np.empty(self.n, dtype=self.dtype)
        call('exa_memcpy_d2h', out.ctypes.data, self.ptr, out.nbytes, stream)
        call('exa_stream_synchronize', stream)
        return out

    def zero(self, stream=None):
        call('exa_memset_device', self.ptr, 0, self.nbytes, stream)

    def free(self):
        if self.ptr:
            call('exa_device_free', self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, n, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.nbytes = max(1, int(n) * self.dtype.itemsize)
        p = C.c_void_p()
        call('exa_host_alloc_pinned', self.nbytes, C.byref(p))
        self.ptr = p
        buf = (C.c_char * self.nbytes).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(n))

    def free(self):
        if self.ptr:
            self.array = None
            call('exa_host_free_pinned', self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Stream:
    def __init__(self):
        p = C.c_void_p()
        call('exa_stream_create', C.byref(p))
        self.ptr = p

    def synchronize(self):
        call('exa_stream_synchronize', self.ptr)

    def destroy(self):
        if self.ptr:
            call('exa_stream_destroy', self.ptr)
            self.ptr = None


class Timer:
    """CUDA-event timer recorded on a given stream."""

    def __init__(self):
        p = C.c_void_p()
        call('exa_timer_create', C.byref(p))
        self.ptr = p

    def start(self, stream=None):
        call('exa_timer_start', self.ptr, stream)

    def stop(self, stream=None):
        call('exa_timer_stop', self.ptr, stream)

    def elapsed_ms(self):
        ms = C.c_float()
        call('exa_timer_elapsed_ms', self.ptr, C.byref(ms))
        return float(ms.value)

    def __del__(self):
        try:
            if self.ptr:
                lib().exa_timer_destroy(self.ptr)
        except Exception:
            pass


def device_count():
    return lib().exa_device_count()


def launch_count():
    return int(lib().exa_launch_count())


def synchronize():
    call('exa_device_synchronize')


def diff_norms(a_ptr, b_ptr, n, stream=None):
    """Relative L2 / Linf of device array a against b (n doubles), computed on
    the device; returns dict(rel_l2, rel_linf, abs_l2, abs_linf)."""
    out = (C.c_double * 4)()
    call('exa_diff_norms', a_ptr, b_ptr, int(n), out, stream)
    return dict(rel_l2=out[0], rel_linf=out[1], abs_l2=out[2], abs_linf=out[3])
