"""Host-side mesh database (libnexd_host.so): the single-partition NEXD-3D
mesher and solver set-up that produce the nexd_desc of the C-ABI."""
import ctypes as C
import os

import numpy as np

from . import _abi


class NexdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"status {status}: {msg}")
        self.status = status


def _host_error(status):
    buf = C.create_string_buffer(1024)
    _abi.host_lib().nexd_mesh_last_error(buf, len(buf))
    return NexdError(status, buf.value.decode(errors="replace"))


def _arr(ptr, shape, dtype=np.float64):
    """numpy view (Fortran order) of a C array owned by the mesh handle."""
    n = int(np.prod(shape))
    if not ptr or n == 0:
        return np.zeros(shape, dtype=dtype, order="F")
    ctype = C.c_double if dtype == np.float64 else C.c_int32
    buf = C.cast(ptr, C.POINTER(ctype * n)).contents
    return np.frombuffer(buf, dtype=dtype, count=n).reshape(shape, order="F")


class Mesh:
    """A built database for one reference simulation directory.

    Mirrors what the reference's timeloop3D holds after readMesh/readSrc/
    readRec/prepareSources (src/timeloopMod.f90:137-356).
    """

    def __init__(self, directory, N=4, timeint=0, cfl=0.0, nt=0, t0=0.0, stf_stage_time=False,
                 init_value=1e-24, nbatch=1, database=False):
        """database=True reads directory/out/{meshVar,srcVar,recVar}000001 (the
        reference mesher's output for one partition; the order comes from the
        files) instead of running the mesher on directory/cubit."""
        lib = _abi.host_lib()
        opts = _abi.NexdBuildOpts(N=N, timeint=timeint, cfl=cfl, nt=nt, t0=t0,
                                  stf_stage_time=1 if stf_stage_time else 0, init_value=init_value,
                                  nbatch=nbatch)
        h = C.c_void_p()
        build = lib.nexd_mesh_load_database if database else lib.nexd_mesh_build
        st = build(str(directory).encode(), C.byref(opts), C.byref(h))
        if st != 0:
            raise _host_error(st)
        self._h = h
        self.desc_ptr = lib.nexd_mesh_desc(h)
        self.desc = self.desc_ptr.contents
        info = _abi.NexdMeshInfo()
        lib.nexd_mesh_get_info(h, C.byref(info))
        self.info = info
        d = self.desc
        self.N, self.Np, self.NpF, self.K = d.N, d.Np, d.NpF, d.nelem
        self.nt, self.dt = d.nt, d.dt
        self.nrec, self.nsrc, self.nbatch = d.nrec, d.nsrc, d.nbatch

    # ---- array views -------------------------------------------------
    def array(self, name):
        d, Np, NpF, K = self.desc, self.Np, self.NpF, self.K
        shapes = {
            "Dr": (Np, Np), "Ds": (Np, Np), "Dt": (Np, Np), "lift": (Np, 4 * NpF), "invmass": (Np, Np),
            "metric": (9, K), "jacobian": (K,), "fscale": (4, K), "nnormal": (3, 4, K),
            "stangential": (3, 4, K), "ttangential": (3, 4, K), "rho": (K,), "vpu": (K,), "vsu": (K,),
            "lambdau": (K,), "muu": (K,), "ylambda": (max(d.nMB, 1), K), "ymu": (max(d.nMB, 1), K),
            "wl": (max(d.nMB, 1),), "pml_profiles": (K * Np, 9), "srcInt": (Np, d.nsrc),
            "srcangle_force": (3, d.nsrc), "srcM": (6, d.nsrc), "stf": (d.stf_per_step, d.nt, d.nsrc),
            "recInt": (Np, d.nrec),
        }
        ishapes = {"fmask": (NpF, 4), "neighbor": (4, K), "face": (4, K), "ibn": (NpF, 4, K), "pmlcheck": (K,),
                   "srcelem": (d.nsrc,), "srctype": (d.nsrc,), "recelem": (d.nrec,), "srcbatch": (d.nsrc,)}
        if name in shapes:
            return _arr(getattr(d, name), shapes[name])
        if name in ishapes:
            return _arr(getattr(d, name), ishapes[name], np.int32)
        info, ng = self.info, self.info.nglob
        extra = {"vx": (info.vx, (ng,)), "vy": (info.vy, (ng,)), "vz": (info.vz, (ng,)),
                 "mass": (info.mass, (Np, Np)), "vdm": (info.vdm, (Np, Np)),
                 "src_rst": (info.src_rst, (3, d.nsrc)), "rec_rst": (info.rec_rst, (3, d.nrec))}
        if name in extra:
            return _arr(extra[name][0], extra[name][1])
        if name == "recnr":
            return _arr(info.recnr, (d.nrec,), np.int32)
        raise KeyError(name)

    def write_database(self, outdir):
        """Writes meshVar000001 (+ srcVar000001 / recVar000001) into outdir as
        the reference's mesher does for one partition."""
        os.makedirs(outdir, exist_ok=True)
        st = _abi.host_lib().nexd_mesh_write_database(self._h, str(outdir).encode())
        if st != 0:
            raise _host_error(st)

    def write_seismograms(self, outdir, traces, nt_written=None, batch=0):
        tr = np.asfortranarray(traces, dtype=np.float32)
        nt_written = self.nt if nt_written is None else nt_written
        st = _abi.host_lib().nexd_mesh_write_seismograms(
            self._h, str(outdir).encode(), tr.ctypes.data_as(C.POINTER(C.c_float)), nt_written, batch)
        if st != 0:
            raise _host_error(st)

    def close(self):
        if getattr(self, "_h", None):
            _abi.host_lib().nexd_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
