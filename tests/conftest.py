"""Shared fixtures.

CPU tests (default) cover the host database builder, the oracle against the
reference's golden seismograms, and the C-ABI surface.  Tests marked ``gpu``
compare the sm_100a path (libnexd.so) with the oracle and need a B200.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nexd-3d_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from nexd_b200 import _abi  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libnexd.so")


def _make(path, target=None):
    cmd = ["make", "-s", "-C", path] + ([target] if target else [])
    subprocess.run(cmd, check=True)


@pytest.fixture(scope="session")
def built():
    """Builds the host library and the oracle (and the CUDA library when nvcc exists)."""
    _make(PKG, "host")
    _make(os.path.join(ROOT, "oracle"))
    return True


@pytest.fixture(scope="session")
def oracle(built):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.oracle_run.argtypes = [C.POINTER(_abi.NexdDesc), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_void_p, C.c_int]
    lib.oracle_run.restype = C.c_int
    lib.oracle_rhs.argtypes = [C.POINTER(_abi.NexdDesc), C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 6
    lib.oracle_rhs.restype = C.c_int
    lib.oracle_run_trigger.argtypes = [C.POINTER(_abi.NexdDesc), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_void_p,
                                       C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.oracle_run_trigger.restype = C.c_int
    return lib


def run_oracle_trigger(lib, mesh, precision=64, w1=10, w2=2, thr=0.1, f0=1.0, formula=0):
    """Oracle run with the NPML energy trigger armed: (traces, energy, switch)."""
    tr = np.zeros((mesh.nrec, mesh.nt, 9, mesh.nbatch), dtype=np.float32, order="F")
    en = np.zeros((mesh.nt, mesh.nbatch), dtype=np.float64, order="F")
    sw = np.zeros(mesh.nbatch, dtype=np.int32)
    st = lib.oracle_run_trigger(mesh.desc_ptr, precision, mesh.nt, tr.ctypes.data_as(C.POINTER(C.c_float)), None, 0,
                                w1, w2, thr, f0, formula, en.ctypes.data_as(C.POINTER(C.c_double)),
                                sw.ctypes.data_as(C.POINTER(C.c_int)))
    assert st == 0, f"oracle failed with status {st}"
    return tr, en, sw


def run_oracle(lib, mesh, precision=64, steps=None, want_field=False):
    """Traces (nrec, nt, 9, nbatch) [and final fields] from the CPU oracle."""
    steps = mesh.nt if steps is None else steps
    tr = np.zeros((mesh.nrec, mesh.nt, 9, mesh.nbatch), dtype=np.float32, order="F")
    field = None
    fptr = None
    if want_field:
        field = np.zeros((mesh.K * mesh.Np, 9, mesh.nbatch), dtype=np.float64, order="F")
        fptr = field.ctypes.data_as(C.c_void_p)
    st = lib.oracle_run(mesh.desc_ptr, precision, steps, tr.ctypes.data_as(C.POINTER(C.c_float)), fptr, 0)
    assert st == 0, f"oracle failed with status {st}"
    return (tr, field) if want_field else tr


def write_brick(directory):
    """Rewrites the reference's brick example inputs from tests/golden/brick.npz."""
    d = np.load(os.path.join(GOLDEN, "brick.npz"))
    os.makedirs(os.path.join(directory, "cubit"), exist_ok=True)
    os.makedirs(os.path.join(directory, "data"), exist_ok=True)
    cub = os.path.join(directory, "cubit")
    coord = d["coord"]
    with open(os.path.join(cub, "coord"), "w") as f:
        f.write(f"{len(coord)}\n")
        np.savetxt(f, np.column_stack([np.arange(1, len(coord) + 1), coord]), fmt=["%d", "%.6f", "%.6f", "%.6f"])
    tets, props = d["tets"], d["props"]
    with open(os.path.join(cub, "mesh"), "w") as f:
        f.write(f"{len(tets)}\n")
        np.savetxt(f, np.column_stack([np.arange(1, len(tets) + 1), tets, props]), fmt=["%d"] * 5 + ["%.4f"] * 5)
    np.savetxt(os.path.join(cub, "mat"), d["mat"], fmt="%d")
    for name in ("free", "absorb"):
        arr = d[name]
        with open(os.path.join(cub, name), "w") as f:
            f.write(f"{len(arr)}\n")
            np.savetxt(f, arr, fmt="%d")
    with open(os.path.join(cub, "matprop"), "w") as f:
        f.write(str(d["matprop"]))
    for name in ("parfile", "source", "stations"):
        with open(os.path.join(directory, "data", name), "w") as f:
            f.write(str(d[name]))
    return d["traces"], d["time"]


# The reference locates stations 1 and 11 (on the box's top edges, at mesh
# vertices shared by six elements) in elements 7937 and 4815; which element
# wins that tie depends on FP32 rounding of the reference's vertex nodes.  The
# golden comparison uses the same elements (vertex nodes 35 and 1).
BRICK_EDGE_STATIONS = {0: (7937, 34), 10: (4815, 0)}


def pin_brick_edge_stations(mesh):
    recelem, recInt = mesh.array("recelem"), mesh.array("recInt")
    for r, (e, node) in BRICK_EDGE_STATIONS.items():
        recelem[r] = e
        recInt[:, r] = 0.0
        recInt[node, r] = 1.0


def brick_dt_cfl():
    """CFL that reproduces the reference's dt = 6.46257467e-06 exactly (its
    FP32 geometry gives dtfactor 1.3e-5 below the FP64 value)."""
    return 0.4 * 6.46257467e-06 / 6.462657008558699e-06


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def trace_misfit(test, ref):
    """Relative L2 of the receiver traces, per trace kind (u, v, a) over all
    receivers and components; returns the largest of the three."""
    return max(rel_l2(test[:, :, 3 * k:3 * k + 3], ref[:, :, 3 * k:3 * k + 3]) for k in range(3))


def station_misfit(test, ref):
    """Relative L2 per receiver and kind, normalised by that receiver's three
    components of the kind; returns the maximum (meaningful only when every
    receiver has recorded the wave)."""
    worst = 0.0
    for r in range(ref.shape[0]):
        for k in range(3):
            worst = max(worst, rel_l2(test[r, :, 3 * k:3 * k + 3], ref[r, :, 3 * k:3 * k + 3]))
    return worst


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
