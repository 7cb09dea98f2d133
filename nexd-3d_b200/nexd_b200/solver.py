"""Device time loop (libnexd.so): Python mirror of the reference's timeloop3D
entry point (src/timeloopMod.f90:42) over the C-ABI of include/nexd.h.

There is no CPU fallback: constructing a Solver without the CUDA library or
without a visible GPU raises.
"""
import ctypes as C

import numpy as np

from . import _abi
from .host import NexdError


def _gpu_error(ctx, status):
    buf = C.create_string_buffer(1024)
    _abi.gpu_lib().nexd_last_error(ctx, buf, len(buf))
    return NexdError(status, buf.value.decode(errors="replace"))


class Solver:
    """One device context: nexd_create on a descriptor, then run/traces."""

    def __init__(self, desc_ptr):
        lib = _abi.gpu_lib()
        ctx = C.c_void_p()
        st = lib.nexd_create(desc_ptr, C.byref(ctx))
        if st != 0:
            raise _gpu_error(None, st)
        self._ctx = ctx
        d = desc_ptr.contents
        self.nrec, self.nt, self.nbatch = d.nrec, d.nt, d.nbatch
        self.K, self.Np = d.nelem, d.Np

    def run(self, it_begin, it_end):
        st = _abi.gpu_lib().nexd_run(self._ctx, it_begin, it_end)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def traces(self, out=None):
        if out is None:
            out = np.zeros((self.nrec, self.nt, 9, self.nbatch), dtype=np.float32, order="F")
        st = _abi.gpu_lib().nexd_get_traces(self._ctx, out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return out

    def field(self, b=0):
        out = np.zeros((self.K * self.Np, 9), dtype=np.float32, order="F")
        st = _abi.gpu_lib().nexd_get_field(self._ctx, b, out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return out

    def set_field(self, q, b=0):
        q = np.asfortranarray(q, dtype=np.float32)
        st = _abi.gpu_lib().nexd_set_field(self._ctx, b, q.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def launch_count(self):
        n = C.c_int64()
        _abi.gpu_lib().nexd_launch_count(self._ctx, C.byref(n))
        return n.value

    def close(self):
        if getattr(self, "_ctx", None):
            _abi.gpu_lib().nexd_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
