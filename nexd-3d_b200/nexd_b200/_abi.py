"""ctypes mirror of include/nexd.h and include/nexd_host.h.

The structures below are field-for-field copies of the C declarations; the
shared libraries are the in-tree builds under ``nexd-3d_b200/lib``.
"""
import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_ROOT, "lib")

NEXD_OK = 0
NEXD_ERR_INVALID = 1
NEXD_ERR_CUDA = 2
NEXD_ERR_NOMEM = 3
NEXD_ERR_UNSUPPORTED = 4
NEXD_ERR_NONFINITE = 5
NEXD_ERR_NODEVICE = 6
NEXD_ERR_TIMEOUT = 7
NEXD_FACE_PARTITION = -3
NEXD_NCOMP = 9
NEXD_ABI_VERSION = 1

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


class NexdDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("N", C.c_int32), ("Np", C.c_int32), ("NpF", C.c_int32),
        ("nelem", C.c_int32), ("nMB", C.c_int32), ("attenuation", C.c_int32), ("set_pml", C.c_int32),
        ("timeint", C.c_int32), ("nt", C.c_int32), ("dt", C.c_double), ("init_value", C.c_double),
        ("Dr", _pd), ("Ds", _pd), ("Dt", _pd), ("lift", _pd), ("invmass", _pd), ("fmask", _pi),
        ("metric", _pd), ("jacobian", _pd), ("fscale", _pd), ("nnormal", _pd), ("stangential", _pd),
        ("ttangential", _pd),
        ("rho", _pd), ("vpu", _pd), ("vsu", _pd), ("lambdau", _pd), ("muu", _pd), ("ylambda", _pd),
        ("ymu", _pd), ("wl", _pd),
        ("neighbor", _pi), ("face", _pi), ("ibn", _pi),
        ("pmlcheck", _pi), ("pml_profiles", _pd),
        ("nsrc", C.c_int32), ("srcelem", _pi), ("srctype", _pi), ("srcInt", _pd), ("srcangle_force", _pd),
        ("srcM", _pd), ("stf_per_step", C.c_int32), ("stf", _pd),
        ("nrec", C.c_int32), ("recelem", _pi), ("recInt", _pd),
        ("nbatch", C.c_int32), ("srcbatch", _pi),
    ]


class NexdHaloDesc(C.Structure):
    _fields_ = [("partition", C.c_int32), ("npeer", C.c_int32), ("peer", _pi), ("nface", _pi), ("elem", _pi),
                ("side", _pi), ("peer_index", _pi), ("peer_node", _pi)]


class NexdHaloExport(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("device", C.c_int32), ("pid", C.c_int64), ("partition", C.c_int32),
                ("nface", C.c_int32), ("nbatch", C.c_int32), ("nbuf", C.c_int32), ("ldq", C.c_int64),
                ("halo_base", C.c_int64), ("counter_slot", C.c_int32), ("reserved", C.c_int32),
                ("q", C.c_uint64 * 3), ("counters", C.c_uint64), ("q_ipc", (C.c_ubyte * 64) * 3),
                ("counters_ipc", C.c_ubyte * 64)]


class NexdPartView(C.Structure):
    _fields_ = [("desc", C.POINTER(NexdDesc)), ("halo", C.POINTER(NexdHaloDesc)), ("nelem", C.c_int32),
                ("elem_global", _pi), ("nsrc", C.c_int32), ("src_global", _pi), ("nrec", C.c_int32),
                ("rec_global", _pi)]


class NexdBuildOpts(C.Structure):
    _fields_ = [
        ("N", C.c_int32), ("timeint", C.c_int32), ("cfl", C.c_double), ("nt", C.c_int32), ("t0", C.c_double),
        ("stf_stage_time", C.c_int32), ("init_value", C.c_double), ("nbatch", C.c_int32),
    ]


class NexdMeshInfo(C.Structure):
    _fields_ = [
        ("dtfactor", C.c_double), ("dt", C.c_double), ("minGLL", C.c_double), ("cfl", C.c_double),
        ("nglob", C.c_int32), ("ncoord", C.c_int32), ("vx", _pd), ("vy", _pd), ("vz", _pd), ("mass", _pd),
        ("vdm", _pd), ("src_rst", _pd), ("rec_rst", _pd), ("recnr", _pi), ("mu", _pd), ("lambda_", _pd),
        ("n_warnings", C.c_int32),
    ]


# Entry points declared in include/*.h, per library (checked by the CPU tests).
HOST_SYMBOLS = ["nexd_mesh_build", "nexd_mesh_desc", "nexd_mesh_get_info", "nexd_mesh_write_seismograms",
                "nexd_mesh_last_error", "nexd_mesh_free", "nexd_mesh_write_database", "nexd_mesh_load_database",
                "nexd_partition_create", "nexd_partition_get", "nexd_partition_count", "nexd_partition_free"]
GPU_SYMBOLS = ["nexd_create", "nexd_create_partition", "nexd_halo_export_peer", "nexd_halo_connect",
               "nexd_halo_run", "nexd_halo_bytes", "nexd_halo_set_timeout", "nexd_run", "nexd_get_traces", "nexd_get_field", "nexd_set_field",
               "nexd_get_state", "nexd_set_state", "nexd_step_io", "nexd_pml_trigger", "nexd_get_energy",
               "nexd_set_contraction", "nexd_get_contraction", "nexd_set_contraction_kinds", "nexd_boundary_faces", "nexd_set_boundary_mlp",
               "nexd_get_ghost", "nexd_get_face_traces", "nexd_mlp_param_count", "nexd_mlp_workspace_floats",
               "nexd_mlp_forward", "nexd_mlp_loss_grad", "nexd_mlp_adam", "nexd_group_create", "nexd_group_run",
               "nexd_group_autotune", "nexd_group_span", "nexd_group_destroy", "nexd_group_set_mode",
               "nexd_group_get_mode", "nexd_movie", "nexd_get_movie",
               "nexd_wavefield_energy_noalloc", "nexd_profile_enable", "nexd_profile_get",
               "nexd_last_error", "nexd_launch_count", "nexd_destroy"]
NEXD_K_RECORD, NEXD_K_STAGE_PML, NEXD_K_STAGE_MAIN, NEXD_K_ENERGY, NEXD_K_BOUNDARY, NEXD_K_HALO, NEXD_K_COUNT = \
    0, 1, 2, 3, 4, 5, 6


class NexdProfile(C.Structure):
    _fields_ = [("launches", C.c_int64 * NEXD_K_COUNT), ("ms", C.c_double * NEXD_K_COUNT),
                ("elements", C.c_int64 * NEXD_K_COUNT), ("span_ms", C.c_double)]
NEXD_STATE_Q, NEXD_STATE_THETA, NEXD_STATE_PML = 0, 1, 2
NEXD_NOALLOC_MAX_BATCH = 64
NEXD_CONTRACT_FP32, NEXD_CONTRACT_BF16X3, NEXD_CONTRACT_AUTO, NEXD_CONTRACT_FP32_PAIRS = 0, 1, 2, 3

_host = None
_gpu = None


def _load(name):
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError(f"{name} is not built ({path} missing); run __graft_entry__.build()")
    return C.CDLL(path)


def host_lib():
    global _host
    if _host is None:
        lib = _load("libnexd_host.so")
        lib.nexd_mesh_build.argtypes = [C.c_char_p, C.POINTER(NexdBuildOpts), C.POINTER(C.c_void_p)]
        lib.nexd_mesh_build.restype = C.c_int
        lib.nexd_mesh_load_database.argtypes = [C.c_char_p, C.POINTER(NexdBuildOpts), C.POINTER(C.c_void_p)]
        lib.nexd_mesh_load_database.restype = C.c_int
        lib.nexd_mesh_write_database.argtypes = [C.c_void_p, C.c_char_p]
        lib.nexd_mesh_write_database.restype = C.c_int
        lib.nexd_mesh_desc.argtypes = [C.c_void_p]
        lib.nexd_mesh_desc.restype = C.POINTER(NexdDesc)
        lib.nexd_mesh_get_info.argtypes = [C.c_void_p, C.POINTER(NexdMeshInfo)]
        lib.nexd_mesh_get_info.restype = C.c_int
        lib.nexd_mesh_write_seismograms.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_float), C.c_int32,
                                                    C.c_int32]
        lib.nexd_mesh_write_seismograms.restype = C.c_int
        lib.nexd_mesh_last_error.argtypes = [C.c_char_p, C.c_size_t]
        lib.nexd_mesh_last_error.restype = C.c_int
        lib.nexd_mesh_free.argtypes = [C.c_void_p]
        lib.nexd_mesh_free.restype = None
        lib.nexd_partition_create.argtypes = [C.POINTER(NexdDesc), C.c_int32, _pi, _pd, C.POINTER(C.c_void_p)]
        lib.nexd_partition_create.restype = C.c_int
        lib.nexd_partition_get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(NexdPartView)]
        lib.nexd_partition_get.restype = C.c_int
        lib.nexd_partition_count.argtypes = [C.c_void_p, _pi]
        lib.nexd_partition_count.restype = C.c_int
        lib.nexd_partition_free.argtypes = [C.c_void_p]
        lib.nexd_partition_free.restype = None
        _host = lib
    return _host


def gpu_lib():
    global _gpu
    if _gpu is None:
        lib = _load("libnexd.so")
        vp = C.c_void_p
        lib.nexd_create.argtypes = [C.POINTER(NexdDesc), C.POINTER(vp)]
        lib.nexd_create_partition.argtypes = [C.POINTER(NexdDesc), C.POINTER(NexdHaloDesc), C.POINTER(vp)]
        lib.nexd_halo_export_peer.argtypes = [vp, C.c_int32, C.POINTER(NexdHaloExport)]
        lib.nexd_halo_connect.argtypes = [vp, C.c_int32, C.POINTER(NexdHaloExport)]
        lib.nexd_halo_run.argtypes = [C.POINTER(vp), C.c_int32, C.c_int32, C.c_int32]
        lib.nexd_halo_bytes.argtypes = [vp, C.POINTER(C.c_int64)]
        lib.nexd_halo_set_timeout.argtypes = [vp, C.c_double]
        lib.nexd_run.argtypes = [vp, C.c_int32, C.c_int32]
        lib.nexd_get_traces.argtypes = [vp, C.POINTER(C.c_float)]
        lib.nexd_get_field.argtypes = [vp, C.c_int32, C.POINTER(C.c_float)]
        lib.nexd_set_field.argtypes = [vp, C.c_int32, C.POINTER(C.c_float)]
        lib.nexd_get_state.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_float)]
        lib.nexd_set_state.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_float)]
        lib.nexd_step_io.argtypes = [vp, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.nexd_pml_trigger.argtypes = [vp, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_int32]
        lib.nexd_get_energy.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
        lib.nexd_set_contraction.argtypes = [vp, C.c_int32]
        lib.nexd_get_contraction.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        lib.nexd_set_contraction_kinds.argtypes = [vp, C.POINTER(C.c_int32)]
        i32p = C.POINTER(C.c_int32)
        lib.nexd_boundary_faces.argtypes = [vp, i32p, i32p, i32p]
        lib.nexd_set_boundary_mlp.argtypes = [vp, C.POINTER(C.c_float), C.c_int64, C.c_float]
        lib.nexd_get_ghost.argtypes = [vp, C.POINTER(C.c_float)]
        lib.nexd_get_face_traces.argtypes = [vp, C.c_int32, i32p, i32p, C.POINTER(C.c_float)]
        lib.nexd_mlp_param_count.argtypes = [C.c_int32, C.c_int32]
        lib.nexd_mlp_param_count.restype = C.c_int64
        lib.nexd_mlp_workspace_floats.argtypes = [C.c_int32, C.c_int32, C.c_int32]
        lib.nexd_mlp_workspace_floats.restype = C.c_int64
        lib.nexd_mlp_forward.argtypes = [C.c_int32, C.c_int32, vp, vp, C.c_int32, vp, vp, vp]
        lib.nexd_mlp_loss_grad.argtypes = [C.c_int32, C.c_int32, vp, vp, vp, C.c_int32, vp, vp, vp, vp]
        lib.nexd_mlp_adam.argtypes = [C.c_int64, vp, vp, vp, vp, C.c_int32, C.c_float, C.c_float, C.c_float,
                                      C.c_float, vp]
        lib.nexd_group_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
        lib.nexd_group_run.argtypes = [vp, C.c_int32, C.c_int32]
        lib.nexd_group_autotune.argtypes = [vp, C.POINTER(C.c_int32)]
        lib.nexd_group_span.argtypes = [vp, C.POINTER(C.c_double)]
        lib.nexd_group_set_mode.argtypes = [vp, C.c_int32]
        lib.nexd_group_get_mode.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.nexd_group_destroy.argtypes = [vp]
        lib.nexd_movie.argtypes = [vp, C.c_int32, C.c_int32]
        lib.nexd_get_movie.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        lib.nexd_wavefield_energy_noalloc.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_int32,
                                                      C.POINTER(C.c_double)]
        lib.nexd_profile_enable.argtypes = [vp, C.c_int32]
        lib.nexd_profile_get.argtypes = [vp, C.POINTER(NexdProfile)]
        lib.nexd_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        lib.nexd_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
        lib.nexd_destroy.argtypes = [vp]
        for n in GPU_SYMBOLS:
            getattr(lib, n).restype = C.c_int
        _gpu = lib
    return _gpu
