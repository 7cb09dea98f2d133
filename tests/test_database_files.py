"""The reference's mesher -> solver database files (out/meshVar000001,
srcVar000001, recVar000001) written and read by libnexd_host.so.

The files are Fortran sequential unformatted records (4-byte length markers
around each record, REAL(4) / INTEGER(4) / LOGICAL(4) data, column-major
arrays).  A record parser written here, independent of the library, checks
the record list against the order and shapes of writeMeshVar
(src/meshMod.f90:1401-1504), writeSrcVar and writeRecVar
(src/sourceReceiverMod.f90:615-648) for one partition.  Reading the files back
gives the descriptor of the mesher path to FP32 rounding (the files hold
REAL(4)), and the oracle runs the same simulation from both.
"""
import os
import struct

import numpy as np
import pytest

from conftest import rel_l2, run_oracle, trace_misfit
from nexd_b200 import Mesh, NexdError, synth


def read_records(path):
    """Fortran sequential unformatted file -> list of record payloads (bytes)."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        payload = data[pos + 4:pos + 4 + n]
        (n2,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert n == n2 == len(payload), (path, len(out))
        out.append(payload)
        pos += 8 + n
    return out


def meshvar_layout(K, Np, NpF, ncoord, nmat):
    """(name, bytes) of every record writeMeshVar writes, in order."""
    nglob, nMB = K * Np, 3
    i4 = lambda name, n=1: (name, 4 * n)
    rec = [i4(n) for n in ("nglob", "nelem", "nmat", "ncoord", "pinterfaces", "mpi_nn", "mpi_nnmax", "mpi_ne",
                           "mpi_nemax", "nproc", "has_src", "has_rec", "dtfactor", "mingll_jac")]
    rec += [i4(n, Np * Np) for n in ("invVdm", "Vdm", "Dr", "Ds", "Dt", "Drw", "Dsw", "Dtw", "Vdmr", "Vdms", "Vdmt",
                                     "mass")]
    rec += [i4("lift", Np * 4 * NpF), i4("fmask", NpF * 4), i4("fmaskv", 4 * NpF)]
    rec += [i4(n, nglob) for n in ("vx", "vy", "vz")]
    rec += [i4("matval", nmat * 11)]
    rec += [i4(n, nglob) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz", "jacobian")]
    rec += [i4("mat", K), i4("ibool", Np * K)]
    rec += [i4(n, 4 * NpF * K) for n in ("nx", "ny", "nz", "sj", "fscale")]
    rec += [i4(n, 12 * K) for n in ("nnormal", "stangential", "ttangential")]
    rec += [i4("coord", 3 * ncoord), i4("elem", 4 * K), i4("neighbor", 4 * K), i4("face", 4 * K)]
    rec += [i4(n, K) for n in ("vp", "vs", "rho", "mu", "lambda", "qp", "qs", "vpu", "vsu", "muu", "lambdau")]
    rec += [i4("ylambda", nMB * K), i4("ymu", nMB * K), i4("wl", nMB), i4("pml", K)]
    rec += [i4(n) for n in ("pmlxmin", "pmlxmax", "pmlymin", "pmlymax", "pmlzmin", "pmlzmax")]
    rec += [i4("ibt", NpF * 4 * K), i4("ibn", NpF * 4 * K), i4("loc2glob_nodes", ncoord),
            i4("mpi_interface", 16 * K), i4("mpi_neighbor", 0), i4("mpi_connection", 0), i4("mpi_ninterface", 0),
            i4("mpi_ibool", 4 * K), i4("mpi_ibt", NpF * 4 * K), i4("mpi_icon", 0), i4("pml_delta")]
    return rec


@pytest.fixture(scope="module")
def twolayer(tmp_path_factory):
    """Anelastic two-layer model with an NPML (N=4) and its database files."""
    d = str(tmp_path_factory.mktemp("db") / "tl")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=40, nrec=5, nsrc=2, src_depth=(700.0, 900.0))
    m = Mesh(d, N=4)
    m.write_database(os.path.join(d, "out"))
    return d, m


def test_record_layout(twolayer):
    d, m = twolayer
    ncoord = int(open(os.path.join(d, "cubit", "coord")).readline())
    nmat = int(open(os.path.join(d, "cubit", "matprop")).readline())
    recs = read_records(os.path.join(d, "out", "meshVar000001"))
    layout = meshvar_layout(m.K, m.Np, m.NpF, ncoord, nmat)
    assert len(recs) == len(layout) == 89
    for (name, nbytes), r in zip(layout, recs):
        assert len(r) == nbytes, name
    rec = {name: r for (name, _), r in zip(layout, recs)}
    i4 = lambda name: np.frombuffer(rec[name], dtype="<i4")
    r4 = lambda name: np.frombuffer(rec[name], dtype="<f4")
    assert i4("nglob")[0] == m.K * m.Np and i4("nelem")[0] == m.K and i4("ncoord")[0] == ncoord
    assert i4("mpi_nn")[0] == 0 and i4("mpi_nemax")[0] == m.K and i4("nproc")[0] == 1
    assert i4("has_src")[0] == 1 and i4("has_rec")[0] == 1
    assert np.array_equal(i4("ibool"), np.arange(1, m.K * m.Np + 1))
    # column-major arrays as the descriptor holds them, rounded to REAL(4)
    K, Np, NpF = m.K, m.Np, m.NpF
    assert np.array_equal(i4("neighbor").reshape((4, K), order="F"), m.array("neighbor"))
    assert np.array_equal(i4("face").reshape((4, K), order="F"), m.array("face"))
    assert np.array_equal(i4("ibn").reshape((NpF, 4, K), order="F"), m.array("ibn"))
    assert np.array_equal(i4("fmask").reshape((NpF, 4), order="F"), m.array("fmask"))
    assert np.array_equal(r4("Dr").reshape((Np, Np), order="F"), m.array("Dr").astype(np.float32))
    assert np.array_equal(r4("lift").reshape((Np, 4 * NpF), order="F"), m.array("lift").astype(np.float32))
    rx = r4("rx").reshape((Np, K), order="F")
    assert np.array_equal(rx, np.broadcast_to(m.array("metric")[0].astype(np.float32), (Np, K)))
    fs = r4("fscale").reshape((NpF, 4, K), order="F")
    assert np.array_equal(fs, np.broadcast_to(m.array("fscale").astype(np.float32), (NpF, 4, K)))
    assert np.array_equal(r4("nnormal").reshape((3, 4, K), order="F"), m.array("nnormal").astype(np.float32))
    assert np.array_equal(r4("ylambda").reshape((3, K), order="F"), m.array("ylambda").astype(np.float32))
    assert np.array_equal(i4("pml"), (m.array("pmlcheck") > 0).astype(np.int32))
    # mass = invV^T invV and Vdmr = Dr V (src/meshMod.f90:607-611)
    V = r4("Vdm").reshape((Np, Np), order="F").astype(np.float64)
    invV = r4("invVdm").reshape((Np, Np), order="F").astype(np.float64)
    assert rel_l2(r4("mass").reshape((Np, Np), order="F"), invV.T @ invV) < 1e-5
    assert rel_l2(r4("Vdmr").reshape((Np, Np), order="F"), m.array("Dr") @ V) < 1e-5


def test_source_receiver_records(twolayer):
    d, m = twolayer
    s = read_records(os.path.join(d, "out", "srcVar000001"))
    n = m.nsrc
    assert [len(x) for x in s] == [4, 12 * n, 12 * n, 4 * n, 4 * n, 4 * n, 4 * n, 4 * n, 4 * n, 12 * n, 24 * n]
    assert np.frombuffer(s[0], "<i4")[0] == n
    assert np.array_equal(np.frombuffer(s[3], "<i4"), m.array("srcelem"))
    assert np.array_equal(np.frombuffer(s[2], "<f4").reshape((3, n), order="F"), m.array("src_rst").astype(np.float32))
    r = read_records(os.path.join(d, "out", "recVar000001"))
    n = m.nrec
    assert [len(x) for x in r] == [4, 12 * n, 12 * n, 4 * n, 4 * n, 4 * n]
    assert np.array_equal(np.frombuffer(r[3], "<i4"), m.array("recelem"))
    assert np.array_equal(np.frombuffer(r[5], "<i4"), m.array("recnr"))


def test_database_gives_the_mesher_descriptor(twolayer):
    d, m = twolayer
    m2 = Mesh(d, database=True)
    assert (m2.N, m2.K, m2.nsrc, m2.nrec, m2.nt) == (m.N, m.K, m.nsrc, m.nrec, m.nt)
    assert abs(m2.dt - m.dt) <= 1e-7 * m.dt
    for name in ("neighbor", "face", "ibn", "pmlcheck", "srcelem", "srctype", "recelem", "fmask"):
        assert np.array_equal(m2.array(name), m.array(name)), name
    # REAL(4) in the files: within a few FP32 ulps of the FP64 mesher values
    for name in ("metric", "jacobian", "fscale", "nnormal", "stangential", "ttangential", "rho", "vpu", "vsu",
                 "lambdau", "muu", "ylambda", "ymu", "wl", "pml_profiles", "srcInt", "recInt", "stf", "srcM",
                 "Dr", "lift", "invmass"):
        a, b = m.array(name), m2.array(name)
        assert np.abs(a - b).max() <= 4e-7 * np.abs(a).max(), name


def test_oracle_runs_the_same_simulation(tmp_path, oracle):
    d = str(tmp_path / "cube")
    synth.write_cube(d, cells=4, nt=150)
    m = Mesh(d, N=3)
    m.write_database(os.path.join(d, "out"))
    m2 = Mesh(d, database=True)
    t1 = run_oracle(oracle, m, 64)[..., 0]
    t2 = run_oracle(oracle, m2, 64)[..., 0]
    assert np.abs(t1).max() > 0
    assert trace_misfit(t2, t1) < 1e-5


def _corrupt(path, pos, data):
    with open(path, "r+b") as f:
        f.seek(pos)
        f.write(data)


def test_database_errors(tmp_path):
    d = str(tmp_path / "c")
    synth.write_cube(d, cells=2, nt=4)
    m = Mesh(d, N=2)
    out = os.path.join(d, "out")
    mv = os.path.join(out, "meshVar000001")
    with pytest.raises(NexdError, match="files not existing"):
        Mesh(d, database=True)
    m.write_database(out)
    Mesh(d, database=True)
    good = open(mv, "rb").read()
    # a partition with MPI neighbours (mpi_nn = 1): record 6 starts at 5 * 12 bytes
    _corrupt(mv, 5 * 12 + 4, struct.pack("<i", 1))
    with pytest.raises(NexdError, match="MPI interfaces"):
        Mesh(d, database=True)
    # mismatched end marker of the first record
    open(mv, "wb").write(good)
    _corrupt(mv, 8, struct.pack("<i", 5))
    with pytest.raises(NexdError, match="markers"):
        Mesh(d, database=True)
    # truncated file
    open(mv, "wb").write(good[:len(good) // 2])
    with pytest.raises(NexdError):
        Mesh(d, database=True)
    # trailing data
    open(mv, "wb").write(good + b"\0\0\0\0")
    with pytest.raises(NexdError, match="unexpected data"):
        Mesh(d, database=True)
    # operators of another node set: Dr scaled
    open(mv, "wb").write(good)
    off = sum(8 + len(r) for r in read_records(mv)[:16])  # Dr is record 17
    Np = m.Np
    dr = np.frombuffer(good[off + 4:off + 4 + 4 * Np * Np], "<f4") * 1.01
    _corrupt(mv, off + 4, dr.astype("<f4").tobytes())
    with pytest.raises(NexdError, match="do not match"):
        Mesh(d, database=True)


@pytest.mark.parametrize("N", [2, 3, 5])
def test_round_trip_other_orders(tmp_path, N):
    """The reader takes the order from the records: elastic cube at N = 2, 3,
    5 written and read back gives the mesher's descriptor."""
    d = str(tmp_path / f"cube{N}")
    synth.write_cube(d, cells=2, nt=6)
    m = Mesh(d, N=N)
    m.write_database(os.path.join(d, "out"))
    m2 = Mesh(d, N=4, database=True)  # the order argument is ignored
    assert (m2.N, m2.Np, m2.NpF, m2.K) == (m.N, m.Np, m.NpF, m.K)
    for name in ("neighbor", "face", "ibn", "fmask", "srcelem", "recelem"):
        assert np.array_equal(m2.array(name), m.array(name)), name
    for name in ("metric", "fscale", "nnormal", "Dr", "lift", "srcInt", "recInt"):
        a, b = m.array(name), m2.array(name)
        assert np.abs(a - b).max() <= 4e-7 * np.abs(a).max(), name
