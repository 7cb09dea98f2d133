"""The C-ABI surface: both libraries load and export every entry point the
headers declare; argument validation runs without touching a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, PKG, have_gpu
from nexd_b200 import _abi, Mesh, synth


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^(?:int|int64_t|const nexd_desc\*|void)\s+(nexd_\w+)\s*\(", txt, re.M)))


def _exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_host_library_exports_header(built):
    lib = os.path.join(PKG, "lib", "libnexd_host.so")
    decl = _declared("nexd_host.h")
    assert decl == sorted(_abi.HOST_SYMBOLS)
    assert set(decl) <= _exported(lib)
    _abi.host_lib()


def test_gpu_library_exports_header():
    lib = os.path.join(PKG, "lib", "libnexd.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "lib/libnexd.so"], check=True)
    decl = _declared("nexd.h")
    assert decl == sorted(_abi.GPU_SYMBOLS)
    assert set(decl) <= _exported(lib)
    _abi.gpu_lib()  # loads (the CUDA runtime resolves lazily, no device needed)


def _err(ctx=None):
    buf = C.create_string_buffer(512)
    _abi.gpu_lib().nexd_last_error(ctx, buf, 512)
    return buf.value.decode()


def test_create_rejects_bad_descriptors(tmp_path, built):
    test_gpu_library_exports_header()
    lib = _abi.gpu_lib()
    d = str(tmp_path / "c")
    synth.write_cube(d, cells=2, nt=5)
    m = Mesh(d, N=3)
    ctx = C.c_void_p()
    assert lib.nexd_create(None, C.byref(ctx)) == _abi.NEXD_ERR_INVALID
    desc = _abi.NexdDesc.from_buffer_copy(m.desc)
    desc.abi_version = 99
    assert lib.nexd_create(C.byref(desc), C.byref(ctx)) == _abi.NEXD_ERR_INVALID
    assert "ABI" in _err()
    desc = _abi.NexdDesc.from_buffer_copy(m.desc)
    desc.N = 7
    assert lib.nexd_create(C.byref(desc), C.byref(ctx)) == _abi.NEXD_ERR_UNSUPPORTED
    desc = _abi.NexdDesc.from_buffer_copy(m.desc)
    desc.dt = -1.0
    assert lib.nexd_create(C.byref(desc), C.byref(ctx)) == _abi.NEXD_ERR_INVALID
    # a boundary face that is neither free nor absorbing
    face = m.array("face")
    nb = m.array("neighbor")
    f, e = [(f, e) for e in range(m.K) for f in range(4) if nb[f, e] == 0][0]
    old = face[f, e]
    face[f, e] = 0
    try:
        assert lib.nexd_create(m.desc_ptr, C.byref(ctx)) == _abi.NEXD_ERR_INVALID
        assert "neither free" in _err()
    finally:
        face[f, e] = old
    assert not ctx.value


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_it(tmp_path, built):
    test_gpu_library_exports_header()
    d = str(tmp_path / "c")
    synth.write_cube(d, cells=2, nt=5)
    m = Mesh(d, N=3)
    ctx = C.c_void_p()
    assert _abi.gpu_lib().nexd_create(m.desc_ptr, C.byref(ctx)) == _abi.NEXD_ERR_NODEVICE
    assert "no CUDA device" in _err()


def test_oracle_header_is_test_infrastructure():
    txt = open(os.path.join(ROOT, "oracle", "oracle.h")).read()
    assert "TEST INFRASTRUCTURE" in txt
    # the product does not link the oracle
    for lib in ("libnexd.so", "libnexd_host.so"):
        p = os.path.join(PKG, "lib", lib)
        if os.path.exists(p):
            assert not any(s.startswith("oracle_") for s in _exported(p))


def test_fortran_module_binds_declared_entry_points():
    """nexd-3d_b200/fortran/nexd_capi.f90 (the Fortran host's ISO_C_BINDING
    module) binds only names the header declares, and its nexd_desc lists the
    C struct's fields in the same order."""
    src = open(os.path.join(PKG, "fortran", "nexd_capi.f90")).read()
    bound = set(re.findall(r'bind\(C, name="(nexd_\w+)"\)', src))
    assert bound and bound <= set(_declared("nexd.h"))
    body = src[src.index("type, bind(C) :: nexd_desc"):src.index("end type nexd_desc")]
    names = []
    for line in body.splitlines()[1:]:
        if "::" in line:
            names += [n.strip() for n in line.split("::")[1].split(",")]
    assert names == [f[0] for f in _abi.NexdDesc._fields_]


def _corrupt(m, name, index, value):
    """Context manager-like helper: sets m.array(name)[index] = value and
    returns a function that restores it."""
    arr = m.array(name)
    old = arr[index].copy() if hasattr(arr[index], "copy") else arr[index]
    arr[index] = value
    def restore():
        arr[index] = old
    return restore


@pytest.mark.parametrize("case", ["neighbor", "ibn", "jacobian", "fmask_low", "fmask_high"])
def test_create_rejects_corrupt_connectivity_before_any_launch(tmp_path, built, case):
    """Descriptors corrupted on the host are refused by nexd_create's
    argument checks (NEXD_ERR_INVALID with a message) before it touches a
    device: on a machine without a GPU the answer is still INVALID, not
    NODEVICE.  The reference aborts on the same inconsistencies while it
    builds its database (src/meshMod.f90:553-596)."""
    test_gpu_library_exports_header()
    lib = _abi.gpu_lib()
    d = str(tmp_path / "c")
    synth.write_cube(d, cells=2, nt=5)
    m = Mesh(d, N=2)
    nb = m.array("neighbor")
    e, f = [(e, f) for e in range(m.K) for f in range(4) if nb[f, e] > 0][0]
    if case == "neighbor":
        restore, msg = _corrupt(m, "neighbor", (f, e), m.K + 1), "neighbor index out of range"
    elif case == "ibn":
        # a node of the element itself instead of one of the neighbour's
        restore, msg = _corrupt(m, "ibn", (0, f, e), e * m.Np + 1), "ibn does not point into the neighbour"
    elif case == "jacobian":
        restore, msg = _corrupt(m, "jacobian", e, 0.0), "zero Jacobian"
    elif case == "fmask_low":
        restore, msg = _corrupt(m, "fmask", (0, 0), 0), "fmask entry out of 1..Np"
    else:
        restore, msg = _corrupt(m, "fmask", (m.NpF - 1, 3), m.Np + 1), "fmask entry out of 1..Np"
    ctx = C.c_void_p()
    try:
        assert lib.nexd_create(m.desc_ptr, C.byref(ctx)) == _abi.NEXD_ERR_INVALID
        assert msg in _err()
        assert not ctx.value
    finally:
        restore()


def test_noalloc_energy_refuses_misaligned_pointers_without_a_device():
    """nexd_wavefield_energy_noalloc checks the caller's pointers before it
    touches the device: emat must be 16-byte aligned (read as float4), mass
    8-byte (FP64), q 4-byte.  The addresses below are never dereferenced."""
    test_gpu_library_exports_header()
    lib = _abi.gpu_lib()
    out = (C.c_double * 1)()
    ok_q, ok_e, ok_m = 0x7f0000000000, 0x7f0000100000, 0x7f0000200000
    cases = [(ok_q, ok_e + 4, ok_m, "emat must be 16-byte aligned"),
             (ok_q, ok_e + 8, ok_m, "emat must be 16-byte aligned"),
             (ok_q, ok_e, ok_m + 4, "mass must be 8-byte aligned"),
             (ok_q + 2, ok_e, ok_m, "q must be 4-byte aligned")]
    for q, emat, mass, msg in cases:
        st = lib.nexd_wavefield_energy_noalloc(q, 1000, 10, 10, 1, emat, mass, 1, out)
        assert st == _abi.NEXD_ERR_INVALID
        assert msg in _err()


def test_fortran_timeloop_replacement_fills_the_descriptor():
    """nexd-3d_b200/fortran/timeloopMod_nexd.f90 replaces the reference's
    module timeloopMod with the same public subroutine timeloop3D(par,
    myrank); it assigns every field of nexd_desc, and every nexd_* function it
    calls is bound in nexd_capi.f90 (whose bindings the header declares)."""
    src = open(os.path.join(PKG, "fortran", "timeloopMod_nexd.f90")).read()
    code = "\n".join(l.split("!")[0] for l in src.splitlines())  # comments out
    assert re.search(r"^module timeloopMod\s*$", code, re.M | re.I)
    assert re.search(r"^\s*subroutine timeloop3D\(par, myrank\)", code, re.M)
    assigned = set(re.findall(r"^\s*(?:if \(.*\) )?d%(\w+)\s*=", code, re.M))
    fields = {f[0] for f in _abi.NexdDesc._fields_}
    assert fields <= assigned, sorted(fields - assigned)
    capi = open(os.path.join(PKG, "fortran", "nexd_capi.f90")).read()
    bound = set(re.findall(r'function (nexd_\w+)\(.*bind\(C, name="\1"\)', capi.replace("&\n", "")))
    called = set(re.findall(r"\b(nexd_\w+)\s*\(", code)) - {"nexd_check", "nexd_desc"}
    assert called and called <= bound, sorted(called - bound)
    # the run and the writers of the reference stay: create, run, traces, destroy, seismograms
    for name in ("nexd_create", "nexd_run", "nexd_get_traces", "nexd_destroy", "readMesh", "prepareSources",
                 "plotPoints2D"):
        assert name in code


def test_c_harness_argument_errors_and_no_device(tmp_path, built):
    """lib/nexd_solve (harness/nexd_solve.c): usage errors return
    NEXD_ERR_INVALID; without a device it builds the mesh from the reference's
    input files and stops at nexd_create with NEXD_ERR_NODEVICE."""
    exe = os.path.join(PKG, "lib", "nexd_solve")
    subprocess.run(["make", "-s", "-C", PKG, "lib/nexd_solve"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == _abi.NEXD_ERR_INVALID and "usage" in r.stderr
    r = subprocess.run([exe, str(tmp_path), "--contraction", "fp64"], capture_output=True, text=True)
    assert r.returncode == _abi.NEXD_ERR_INVALID
    r = subprocess.run([exe, str(tmp_path / "missing")], capture_output=True, text=True)
    assert r.returncode != 0 and "building the mesh failed" in r.stderr
    if not have_gpu():
        d = str(tmp_path / "c")
        synth.write_cube(d, cells=2, nt=5)
        r = subprocess.run([exe, d, "--order", "2"], capture_output=True, text=True)
        assert r.returncode == _abi.NEXD_ERR_NODEVICE and "no CUDA device" in r.stderr
