"""Partitions of one mesh and the halo exchange between them.

The reference scales a mesh beyond one process by domain decomposition: its
mesher splits the elements with METIS and hands every rank its elements plus
the interface arrays (src/meshMod.f90:382-504, 669-1110), and the solver
exchanges the face traces of the interface faces once per RK stage
(SendRecVar, src/mpiMod.f90:310-351, called at src/timeloopMod.f90:393).

Here ``Partitions`` wraps nexd_partition_create (libnexd_host.so: the
partition and halo descriptors of every part), and the halo itself runs
inside libnexd.so: every stage each partition writes its interface traces
straight into its neighbours' halo slots and raises their arrival counters
(include/nexd.h, nexd_create_partition).  Two ways to link the partitions:

* ``PartitionedSolver``: all partitions in this process on one GPU, stepped
  together stage by stage (nexd_halo_run);
* ``connect_ranks``: one partition per process (one rank per GPU under
  torchrun); the halo exports travel between the ranks through
  torch.distributed and the library opens them with CUDA IPC, after which
  each rank calls ``Solver.run`` on its own.
"""
import ctypes as C

import numpy as np

from . import _abi
from .host import NexdError, _host_error
from .solver import Solver, _gpu_error


def element_centroids(mesh):
    """(3, K) centroids of the mesh's elements (mean of their nodes)."""
    info = _abi.NexdMeshInfo()
    st = _abi.host_lib().nexd_mesh_get_info(mesh._h, C.byref(info))
    if st != 0:
        raise _host_error(st)
    K, Np = mesh.K, mesh.Np
    out = np.empty((3, K))
    for k, ptr in enumerate((info.vx, info.vy, info.vz)):
        out[k] = np.ctypeslib.as_array(ptr, shape=(K * Np,)).reshape(K, Np).mean(axis=1)
    return np.asfortranarray(out)


class Partitions:
    """nexd_partition_create on a descriptor: ``part`` (K, 0-based) or, when
    None, recursive coordinate bisection of ``centroids`` (3, K)."""

    def __init__(self, desc_ptr, nparts, part=None, centroids=None):
        lib = _abi.host_lib()
        K = desc_ptr.contents.nelem
        self._keep = []
        pp = None
        if part is not None:
            part = np.ascontiguousarray(part, dtype=np.int32)
            if part.shape != (K,):
                raise ValueError("part must have one entry per element")
            self._keep.append(part)
            pp = part.ctypes.data_as(_abi._pi)
        cp = None
        if centroids is not None:
            centroids = np.asfortranarray(centroids, dtype=np.float64)
            self._keep.append(centroids)
            cp = centroids.ctypes.data_as(_abi._pd)
        self._h = C.c_void_p()
        st = lib.nexd_partition_create(desc_ptr, int(nparts), pp, cp, C.byref(self._h))
        if st != 0:
            raise _host_error(st)
        self._desc_ptr = desc_ptr  # the partitions share its operators
        self.n = int(nparts)
        self.views = []
        for i in range(self.n):
            v = _abi.NexdPartView()
            st = lib.nexd_partition_get(self._h, i, C.byref(v))
            if st != 0:
                raise _host_error(st)
            self.views.append(v)

    def desc(self, i):
        return self.views[i].desc

    def halo(self, i):
        return self.views[i].halo

    def elements(self, i):
        """1-based elements of the whole mesh in partition i."""
        v = self.views[i]
        return np.ctypeslib.as_array(v.elem_global, shape=(v.nelem,)).copy()

    def receivers(self, i):
        v = self.views[i]
        if v.nrec == 0:
            return np.zeros(0, dtype=np.int32)
        return np.ctypeslib.as_array(v.rec_global, shape=(v.nrec,)).copy()

    def peers(self, i):
        """Neighbour partition numbers (1-based) of partition i and the faces
        shared with each."""
        h = self.views[i].halo.contents
        if h.npeer == 0:
            return [], []
        return (list(np.ctypeslib.as_array(h.peer, shape=(h.npeer,))),
                list(np.ctypeslib.as_array(h.nface, shape=(h.npeer,))))

    def close(self):
        if getattr(self, "_h", None):
            _abi.host_lib().nexd_partition_free(self._h)
            self._h = None
            self.views = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def export_peer(solver, k):
    """The halo export of ``solver``'s partition for its k-th neighbour."""
    e = _abi.NexdHaloExport()
    st = _abi.gpu_lib().nexd_halo_export_peer(solver._ctx, k, C.byref(e))
    if st != 0:
        raise _gpu_error(solver._ctx, st)
    return e


def connect(solver, k, export):
    st = _abi.gpu_lib().nexd_halo_connect(solver._ctx, k, C.byref(export))
    if st != 0:
        raise _gpu_error(solver._ctx, st)


def halo_bytes(solver):
    n = C.c_int64()
    st = _abi.gpu_lib().nexd_halo_bytes(solver._ctx, C.byref(n))
    if st != 0:
        raise _gpu_error(solver._ctx, st)
    return int(n.value)


class PartitionedSolver:
    """Every partition of ``parts`` as a context on this GPU, linked to its
    neighbours; ``run`` steps them together (nexd_halo_run) and ``traces``
    puts the receivers back in the whole mesh's order."""

    def __init__(self, parts, nrec_total=None):
        self.parts = parts
        self.solvers = [Solver(parts.desc(i), parts.halo(i)) for i in range(parts.n)]
        self.nrec = nrec_total if nrec_total is not None else sum(s.nrec for s in self.solvers)
        self.nt = self.solvers[0].nt
        self.nbatch = self.solvers[0].nbatch
        # partition i's k-th neighbour q exports for its own index of i
        index = {}
        for i in range(parts.n):
            for k, q in enumerate(parts.peers(i)[0]):
                index[(i + 1, int(q))] = k
        for i in range(parts.n):
            for k, q in enumerate(parts.peers(i)[0]):
                q = int(q)
                connect(self.solvers[i], k, export_peer(self.solvers[q - 1], index[(q, i + 1)]))

    def run(self, it_begin, it_end):
        arr = (C.c_void_p * len(self.solvers))(*[s._ctx for s in self.solvers])
        st = _abi.gpu_lib().nexd_halo_run(arr, len(self.solvers), it_begin, it_end)
        if st != 0:
            bad = next((s._ctx for s in self.solvers), None)
            raise _gpu_error(bad, st)

    def traces(self):
        out = np.zeros((self.nrec, self.nt, 9, self.nbatch), dtype=np.float32, order="F")
        for i, s in enumerate(self.solvers):
            if s.nrec == 0:
                continue
            out[self.parts.receivers(i) - 1] = s.traces()
        return out

    def field(self, K, Np, b=0):
        """The whole mesh's wavefield (K*Np, 9) from the partitions."""
        out = np.zeros((K * Np, 9), dtype=np.float32, order="F")
        for i, s in enumerate(self.solvers):
            el = self.parts.elements(i) - 1
            rows = (el[:, None] * Np + np.arange(Np)[None, :]).ravel()
            out[rows] = s.field(b)
        return out

    def halo_bytes(self):
        return sum(halo_bytes(s) for s in self.solvers)

    def close(self):
        for s in self.solvers:
            s.close()
        self.solvers = []


def route_exports(group, partition, outgoing):
    """Delivers halo exports between ranks: ``outgoing`` maps a neighbour's
    partition number to the bytes exported for it; returns the bytes every
    neighbour exported for ``partition``, by the neighbour's number.  One
    all-gather over the group (gloo or NCCL), every rank taking part."""
    if group.dist is None or group.world == 1:
        return {}
    mine = (int(partition), {int(q): bytes(b) for q, b in outgoing.items()})
    everyone = [None] * group.world
    group.dist.all_gather_object(everyone, mine)
    got = {}
    for src, table in everyone:
        if src != partition and partition in table:
            got[src] = table[partition]
    return got


def connect_ranks(group, solver, parts, i):
    """Links partition i, run by this rank as ``solver``, to the partitions
    of the other ranks (one partition per rank): exports for every neighbour
    go out, the neighbours' exports come back and are opened, then all ranks
    meet at a barrier so that no rank writes into a neighbour before it is
    linked."""
    peers = [int(q) for q in parts.peers(i)[0]]
    outgoing = {q: bytes(export_peer(solver, k)) for k, q in enumerate(peers)}
    incoming = route_exports(group, i + 1, outgoing)
    for k, q in enumerate(peers):
        if q not in incoming:
            raise NexdError(_abi.NEXD_ERR_INVALID, f"no halo export from partition {q}")
        connect(solver, k, _abi.NexdHaloExport.from_buffer_copy(incoming[q]))
    group.barrier()
