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
