"""Partitions and their halo descriptors on the CPU: the host partitioner
(nexd_partition_create) against the whole mesh's connectivity and node
coordinates, the argument checks of nexd_create_partition (answered before
any device is touched), and the rank-to-rank delivery of halo exports over
two gloo ranks.  The reference's counterparts: the mesher's partition and
interface arrays (src/meshMod.f90:382-504, 669-1110) and SendRecVar
(src/mpiMod.f90:310-351)."""
import ctypes as C
import os
import socket
import sys

import numpy as np
import pytest

from conftest import PKG
from nexd_b200 import Mesh, _abi, synth
from nexd_b200.halo import Partitions, element_centroids, route_exports


@pytest.fixture(scope="module")
def mesh(tmp_path_factory, built):
    d = str(tmp_path_factory.mktemp("p") / "twolayer")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=20, nrec=12, nsrc=3)
    return Mesh(d, N=2, stf_stage_time=True)


def _arr(ptr, n, dtype=np.int32):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def _node_xyz(m):
    info = m.info
    n = m.K * m.Np
    return np.stack([np.ctypeslib.as_array(p, shape=(n,)) for p in (info.vx, info.vy, info.vz)], axis=1)


def _check_partitions(m, ps):
    K, Np, NpF = m.K, m.Np, m.NpF
    nb_g = m.array("neighbor").astype(int)     # (4, K)
    fc_g = m.array("face").astype(int)
    fmask = m.array("fmask").astype(int) - 1   # (NpF, 4)
    xyz = _node_xyz(m)
    owner = np.full(K, -1)
    local = np.zeros(K, dtype=int)
    for i in range(ps.n):
        el = ps.elements(i) - 1
        assert (owner[el] == -1).all()
        owner[el] = i
        local[el] = np.arange(len(el))
        assert (np.diff(el) > 0).all()  # original order kept
    assert (owner >= 0).all()
    halos = {}
    for i in range(ps.n):
        d = ps.desc(i).contents
        h = ps.halo(i).contents
        el = ps.elements(i) - 1
        Kp = d.nelem
        assert Kp == len(el) and h.partition == i + 1
        nb = _arr(d.neighbor, 4 * Kp).reshape(Kp, 4)
        fc = _arr(d.face, 4 * Kp).reshape(Kp, 4)
        for li, e in enumerate(el):
            for f in range(4):
                g = nb_g[f, e]
                if g == 0:
                    assert nb[li, f] == 0 and fc[li, f] == fc_g[f, e]
                elif owner[g - 1] == i:
                    assert nb[li, f] == local[g - 1] + 1 and fc[li, f] == fc_g[f, e]
                else:
                    assert nb[li, f] == 0 and fc[li, f] == _abi.NEXD_FACE_PARTITION
        npeer = h.npeer
        peers = _arr(h.peer, npeer)
        nface = _arr(h.nface, npeer)
        tot = int(nface.sum())
        halos[i + 1] = dict(peers=list(peers), nface=list(nface), elem=_arr(h.elem, tot), side=_arr(h.side, tot),
                            pidx=_arr(h.peer_index, tot), pnode=_arr(h.peer_node, tot * NpF).reshape(tot, NpF),
                            el=el)
        assert (np.diff(peers) > 0).all()
        assert tot == int((fc == _abi.NEXD_FACE_PARTITION).sum())
    # every shared face pairs with the neighbour's face, and the node matching
    # joins nodes at the same place
    for p, hp in halos.items():
        off = 0
        for q, n in zip(hp["peers"], hp["nface"]):
            hq = halos[q]
            k = hq["peers"].index(p)
            qoff = int(sum(hq["nface"][:k]))
            for c in range(n):
                e = hp["el"][hp["elem"][off + c] - 1]
                f = hp["side"][off + c] - 1
                c2 = hp["pidx"][off + c] - 1
                e2 = hq["el"][hq["elem"][qoff + c2] - 1]
                f2 = hq["side"][qoff + c2] - 1
                assert nb_g[f, e] == e2 + 1 and nb_g[f2, e2] == e + 1
                assert hq["pidx"][qoff + c2] - 1 == c
                for j in range(NpF):
                    jj = hp["pnode"][off + c, j] - 1
                    a = xyz[e * Np + fmask[j, f]]
                    b = xyz[e2 * Np + fmask[jj, f2]]
                    assert np.allclose(a, b, atol=1e-6 * np.abs(xyz).max())
            off += n
    # sources and receivers dealt out once, in order
    recs = np.concatenate([ps.receivers(i) for i in range(ps.n)])
    assert sorted(recs) == list(range(1, m.nrec + 1))
    assert sum(ps.desc(i).contents.nsrc for i in range(ps.n)) == m.nsrc


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_bisection_partitions_are_consistent(mesh, nparts):
    ps = Partitions(mesh.desc_ptr, nparts, centroids=element_centroids(mesh))
    sizes = [ps.desc(i).contents.nelem for i in range(nparts)]
    assert sum(sizes) == mesh.K and max(sizes) - min(sizes) <= 1
    _check_partitions(mesh, ps)
    if nparts == 1:
        assert ps.halo(0).contents.npeer == 0
    ps.close()


def test_given_element_partition(mesh):
    """A partition handed in (as the reference's METIS output would be),
    scattered at random, gives many small interfaces."""
    part = np.random.default_rng(3).integers(0, 4, mesh.K).astype(np.int32)
    ps = Partitions(mesh.desc_ptr, 4, part=part)
    for i in range(4):
        assert (part[ps.elements(i) - 1] == i).all()
    _check_partitions(mesh, ps)
    ps.close()


def test_partition_errors(mesh):
    with pytest.raises(Exception, match="empty partition"):
        Partitions(mesh.desc_ptr, 3, part=np.zeros(mesh.K, dtype=np.int32))
    with pytest.raises(Exception, match="out of 0..nparts-1"):
        Partitions(mesh.desc_ptr, 2, part=np.full(mesh.K, 2, dtype=np.int32))
    with pytest.raises(Exception, match="centroids"):
        Partitions(mesh.desc_ptr, 2)
    ps = Partitions(mesh.desc_ptr, 2, centroids=element_centroids(mesh))
    with pytest.raises(Exception, match="partition already"):
        Partitions(ps.desc(0), 2, part=np.zeros(ps.desc(0).contents.nelem, dtype=np.int32))
    ps.close()


def _create_status(desc_ptr, halo_ptr):
    lib = _abi.gpu_lib()
    ctx = C.c_void_p()
    if halo_ptr is None:
        st = lib.nexd_create(desc_ptr, C.byref(ctx))
    else:
        st = lib.nexd_create_partition(desc_ptr, halo_ptr, C.byref(ctx))
    buf = C.create_string_buffer(512)
    lib.nexd_last_error(None, buf, len(buf))
    if ctx:
        lib.nexd_destroy(ctx)
    return st, buf.value.decode()


@pytest.mark.parametrize("case", ["plain_create", "missing_face", "not_shared", "peer_index", "peer_node",
                                  "self_peer"])
def test_create_partition_rejects_bad_halo_before_any_launch(mesh, case):
    """Inconsistent halo descriptors are refused with NEXD_ERR_INVALID by the
    argument checks, before a device is touched (so the same answer comes
    without a GPU)."""
    from test_abi import test_gpu_library_exports_header
    test_gpu_library_exports_header()
    ps = Partitions(mesh.desc_ptr, 2, centroids=element_centroids(mesh))
    d, h = ps.desc(0), ps.halo(0)
    hc = h.contents
    tot = int(sum(_arr(hc.nface, hc.npeer)))
    NpF = mesh.NpF
    if case == "plain_create":
        st, msg = _create_status(d, None)
        assert st == _abi.NEXD_ERR_INVALID and "nexd_create_partition" in msg
    elif case == "missing_face":
        hc.nface[0] -= 1
        st, msg = _create_status(d, h)
        hc.nface[0] += 1
        assert st == _abi.NEXD_ERR_INVALID and ("missing" in msg or "permutation" in msg)
    elif case == "not_shared":
        old = hc.side[0]
        hc.side[0] = old % 4 + 1
        st, msg = _create_status(d, h)
        hc.side[0] = old
        assert st == _abi.NEXD_ERR_INVALID and "halo" in msg
    elif case == "peer_index":
        old = hc.peer_index[0]
        hc.peer_index[0] = tot + 5
        st, msg = _create_status(d, h)
        hc.peer_index[0] = old
        assert st == _abi.NEXD_ERR_INVALID and "peer_index" in msg
    elif case == "peer_node":
        old = hc.peer_node[1]
        hc.peer_node[1] = hc.peer_node[0]
        st, msg = _create_status(d, h)
        hc.peer_node[1] = old
        assert st == _abi.NEXD_ERR_INVALID and "peer_node" in msg
    elif case == "self_peer":
        old = hc.peer[0]
        hc.peer[0] = hc.partition
        st, msg = _create_status(d, h)
        hc.peer[0] = old
        assert st == _abi.NEXD_ERR_INVALID and "neighbour" in msg
    # restored: valid, so the answer is a device one (or success on a GPU)
    st, _ = _create_status(d, h)
    assert st in (_abi.NEXD_OK, _abi.NEXD_ERR_NODEVICE, _abi.NEXD_ERR_INVALID) and st != _abi.NEXD_ERR_INVALID
    ps.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _route_main(rank, world, port, out_dir):
    sys.path.insert(0, PKG)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from nexd_b200 import replicas
    from nexd_b200.halo import route_exports
    g = replicas.init("gloo", timeout_s=60)
    part = rank + 1
    # partitions 1-2-3 in a row: each exports to its neighbours
    nbrs = [q for q in (part - 1, part + 1) if 1 <= q <= world]
    out = {q: bytes([part, q]) * 8 for q in nbrs}
    got = route_exports(g, part, out)
    g.barrier()
    g.close()
    with open(os.path.join(out_dir, f"got{rank}.txt"), "w") as f:
        f.write(repr(sorted((k, v.hex()) for k, v in got.items())))


def test_route_exports_over_three_gloo_ranks(tmp_path):
    """Halo exports reach exactly the neighbours they were made for (the
    exchange connect_ranks runs before the first step)."""
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    world, port = 3, _free_port()
    mp.start_processes(_route_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    for rank in range(world):
        part = rank + 1
        got = eval(open(tmp_path / f"got{rank}.txt").read())
        want = sorted((q, (bytes([q, part]) * 8).hex()) for q in (part - 1, part + 1) if 1 <= q <= world)
        assert got == want
    assert route_exports(type("G", (), {"dist": None, "world": 1})(), 1, {2: b"x"}) == {}
