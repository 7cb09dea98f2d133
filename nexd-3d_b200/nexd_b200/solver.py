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
    """One device context: nexd_create on a descriptor (nexd_create_partition
    when a halo descriptor is given), then run/traces."""

    def __init__(self, desc_ptr, halo_ptr=None):
        lib = _abi.gpu_lib()
        ctx = C.c_void_p()
        if halo_ptr is None:
            st = lib.nexd_create(desc_ptr, C.byref(ctx))
        else:
            st = lib.nexd_create_partition(desc_ptr, halo_ptr, C.byref(ctx))
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

    def state(self, which=_abi.NEXD_STATE_Q, b=0, nfields=9):
        """Copy of a state array: q (K*Np,9), theta (K*Np,6*nMB) or PML
        auxiliaries (K*Np,27)."""
        out = np.zeros((self.K * self.Np, nfields), dtype=np.float32, order="F")
        st = _abi.gpu_lib().nexd_get_state(self._ctx, which, b, out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return out

    def set_state(self, arr, which=_abi.NEXD_STATE_Q, b=0):
        arr = np.asfortranarray(arr, dtype=np.float32)
        st = _abi.gpu_lib().nexd_set_state(self._ctx, which, b, arr.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def field(self, b=0):
        return self.state(_abi.NEXD_STATE_Q, b, 9)

    def set_field(self, q, b=0):
        self.set_state(q, _abi.NEXD_STATE_Q, b)

    def step_io(self, it, stf_in, traces_out):
        """One step with host source samples in and that step's receiver samples out."""
        sp = None if stf_in is None else stf_in.ctypes.data_as(C.POINTER(C.c_float))
        st = _abi.gpu_lib().nexd_step_io(self._ctx, it, sp, traces_out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def profile(self, enable=None):
        """CUDA-event timing: enable=True (per launch + run span), "span" (run
        span only, CUDA graphs kept), False (off); without an argument return
        the per-kernel-kind counters as a dict."""
        lib = _abi.gpu_lib()
        if enable is not None:
            mode = 2 if enable == "span" else (1 if enable else 0)
            lib.nexd_profile_enable(self._ctx, mode)
            return None
        p = _abi.NexdProfile()
        lib.nexd_profile_get(self._ctx, C.byref(p))
        names = ("record", "stage_pml", "stage_main", "energy", "boundary", "halo")
        out = {n: dict(launches=p.launches[i], ms=p.ms[i], elements=p.elements[i]) for i, n in enumerate(names)}
        out["span_ms"] = p.span_ms
        return out

    def set_contraction(self, mode):
        """Element contraction arithmetic: "fp32" (CUDA cores, default),
        "bf16x3" (tcgen05 tensor cores, split BF16, FP32 accumulation),
        "fp32_pairs" (the node-pair FP32 kernel outside the NPML) or "auto"
        (per element class the fastest candidate kernel, timed on this mesh;
        the bulk-copy kernels are candidates too)."""
        m = {"fp32": _abi.NEXD_CONTRACT_FP32, "bf16x3": _abi.NEXD_CONTRACT_BF16X3,
             "auto": _abi.NEXD_CONTRACT_AUTO, "fp32_pairs": _abi.NEXD_CONTRACT_FP32_PAIRS}.get(mode, mode)
        st = _abi.gpu_lib().nexd_set_contraction(self._ctx, m)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def set_contraction_kinds(self, npml, rest):
        """Pins the kernel per element class ("fp32", "bf16x3"; "fp32_bulk"
        for the NPML elements, "fp32_pairs" for the rest), e.g. an earlier
        auto choice, without timing."""
        m = {"fp32": 0, "bf16x3": 1, "fp32_pairs": 2, "fp32_bulk": 3}
        kinds = (C.c_int32 * 2)(m.get(npml, npml), m.get(rest, rest))
        st = _abi.gpu_lib().nexd_set_contraction_kinds(self._ctx, kinds)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def contraction(self):
        """({"npml": kind, "rest": kind}, autotune ms per launch {(class, kind): ms})."""
        kinds = (C.c_int32 * 2)()
        ms = (C.c_float * 8)()
        st = _abi.gpu_lib().nexd_get_contraction(self._ctx, kinds, ms)
        if st != 0:
            raise _gpu_error(self._ctx, st)
        names = {0: "fp32", 1: "bf16x3", 2: "fp32_pairs", 3: "fp32_bulk"}
        return ({"npml": names[kinds[0]], "rest": names[kinds[1]]},
                {(cl, names[k]): ms[4 * i + k] for i, cl in enumerate(("npml", "rest")) for k in range(4)})

    def boundary_faces(self):
        """(elem, face) 1-based arrays of the absorbing faces in ghost-slot order."""
        lib = _abi.gpu_lib()
        n = C.c_int32()
        st = lib.nexd_boundary_faces(self._ctx, C.byref(n), None, None)
        if st != 0:
            raise _gpu_error(self._ctx, st)
        e = np.zeros(n.value, dtype=np.int32)
        f = np.zeros(n.value, dtype=np.int32)
        if n.value:
            st = lib.nexd_boundary_faces(self._ctx, None, e.ctypes.data_as(C.POINTER(C.c_int32)),
                                         f.ctypes.data_as(C.POINTER(C.c_int32)))
            if st != 0:
                raise _gpu_error(self._ctx, st)
        return e, f

    def set_boundary_mlp(self, params, max_reflection=0.5):
        """Learned absorbing boundary from FP32 parameters (incoming characteristics
        bounded by max_reflection times the outgoing ones), or None for the plain one."""
        lib = _abi.gpu_lib()
        if params is None:
            st = lib.nexd_set_boundary_mlp(self._ctx, None, 0, 0.0)
        else:
            p = np.ascontiguousarray(params, dtype=np.float32)
            st = lib.nexd_set_boundary_mlp(self._ctx, p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                           max_reflection)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def ghost(self, npf):
        """Exterior states of the last stage, (nbatch, nbf, 9, NpF)."""
        nbf = len(self.boundary_faces()[0])
        out = np.zeros((self.nbatch, nbf, 9, npf), dtype=np.float32)
        st = _abi.gpu_lib().nexd_get_ghost(self._ctx, out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return out

    def face_traces(self, elem, face, npf):
        """Own and neighbour traces of faces (1-based elem, face): (nbatch, nfaces, 2, 9, NpF)."""
        e = np.ascontiguousarray(elem, dtype=np.int32)
        f = np.ascontiguousarray(face, dtype=np.int32)
        out = np.zeros((self.nbatch, len(e), 2, 9, npf), dtype=np.float32)
        st = _abi.gpu_lib().nexd_get_face_traces(self._ctx, len(e), e.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 f.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return out

    def movie(self, frame, max_frames=64):
        """Per-element |u| snapshots every `frame` steps (0 switches them off)."""
        st = _abi.gpu_lib().nexd_movie(self._ctx, frame, max_frames)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def movie_frames(self):
        """Stored snapshots, (nbatch, nframes, nelem)."""
        lib = _abi.gpu_lib()
        nf = C.c_int32()
        st = lib.nexd_get_movie(self._ctx, None, C.byref(nf))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        out = np.zeros((self.nbatch, nf.value, self.K), dtype=np.float32)
        if nf.value:
            st = lib.nexd_get_movie(self._ctx, out.ctypes.data_as(C.POINTER(C.c_float)), C.byref(nf))
            if st != 0:
                raise _gpu_error(self._ctx, st)
        return out

    def pml_trigger(self, avg_window1=10, avg_window2=2, sta_lta_trigger=0.1, f0=1.0, formula=0):
        """Arm the NPML energy STA/LTA trigger (src/timeloopMod.f90:508-542)."""
        st = _abi.gpu_lib().nexd_pml_trigger(self._ctx, avg_window1, avg_window2, sta_lta_trigger, f0, formula)
        if st != 0:
            raise _gpu_error(self._ctx, st)

    def energy(self):
        """(energy history (nt, nbatch), step at which the NPML switched off per wavefield)."""
        e = np.zeros((self.nt, self.nbatch), dtype=np.float64, order="F")
        sw = np.zeros(self.nbatch, dtype=np.int32)
        st = _abi.gpu_lib().nexd_get_energy(self._ctx, e.ctypes.data_as(C.POINTER(C.c_double)),
                                            sw.ctypes.data_as(C.POINTER(C.c_int32)))
        if st != 0:
            raise _gpu_error(self._ctx, st)
        return e, sw

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


class Group:
    """Several solvers stepped together as one CUDA graph (nexd_group_*)."""

    def __init__(self, solvers):
        lib = _abi.gpu_lib()
        self._members = list(solvers)  # keeps the contexts alive
        arr = (C.c_void_p * len(self._members))(*[s._ctx.value for s in self._members])
        g = C.c_void_p()
        st = lib.nexd_group_create(arr, len(self._members), C.byref(g))
        if st != 0:
            raise _gpu_error(None, st)
        self._g = g

    def run(self, it_begin, it_end):
        st = _abi.gpu_lib().nexd_group_run(self._g, it_begin, it_end)
        if st != 0:
            raise _gpu_error(None, st)

    def autotune(self):
        d = C.c_int32()
        st = _abi.gpu_lib().nexd_group_autotune(self._g, C.byref(d))
        if st != 0:
            raise _gpu_error(None, st)
        return d.value

    def set_mode(self, mode):
        """0: one graph branch per member; 1: one persistent launch per stage for all members."""
        st = _abi.gpu_lib().nexd_group_set_mode(self._g, int(mode))
        if st != 0:
            raise _gpu_error(None, st)

    def mode(self):
        """(mode, blocks per member in mode 1, autotune ms {"branches": .., "persistent": ..})."""
        m = C.c_int32()
        blocks = (C.c_int32 * len(self._members))()
        ms = (C.c_double * 2)()
        st = _abi.gpu_lib().nexd_group_get_mode(self._g, C.byref(m), blocks, ms)
        if st != 0:
            raise _gpu_error(None, st)
        return m.value, list(blocks), {"branches": ms[0], "persistent": ms[1]}

    def span_ms(self):
        v = C.c_double()
        st = _abi.gpu_lib().nexd_group_span(self._g, C.byref(v))
        if st != 0:
            raise _gpu_error(None, st)
        return v.value

    def close(self):
        if getattr(self, "_g", None):
            _abi.gpu_lib().nexd_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
