"""Partitions with the halo exchange on one GPU (nexd_create_partition,
nexd_halo_connect, nexd_halo_run): a mesh split into 2 to 4 partitions gives
the traces and wavefield of the whole mesh in one context bit for bit (the
halo slots hold exactly the neighbour values the stage kernels would read),
for LSERK4 with attenuation and NPML, for TVD-RK3 (three wavefield buffers)
and for batched wavefields; a partition whose neighbour never writes ends its
bounded wait with NEXD_ERR_TIMEOUT.  The reference's counterpart is the
per-stage SendRecVar (src/mpiMod.f90:310-351, src/timeloopMod.f90:393) on a
METIS-partitioned mesh, whose traces do not depend on the partition."""
import numpy as np
import pytest

from conftest import run_oracle, trace_misfit
from nexd_b200 import Mesh, _abi, synth
from nexd_b200.halo import Partitions, PartitionedSolver, element_centroids, export_peer, connect
from nexd_b200.host import NexdError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver_mod():
    from nexd_b200 import solver
    return solver


def _whole(solver_mod, m, nsteps):
    s = solver_mod.Solver(m.desc_ptr)
    s.run(1, nsteps)
    out = s.traces(), s.field()
    s.close()
    return out


def _parted(m, ps, nsteps, split=None):
    p = PartitionedSolver(ps, nrec_total=m.nrec)
    if split is None:
        p.run(1, nsteps)
    else:  # several calls: the step counter and buffer parity carry over
        p.run(1, split)
        p.run(split + 1, nsteps)
    out = p.traces(), p.field(m.K, m.Np)
    p.close()
    return out


@pytest.mark.parametrize("nparts,how", [(2, "bisect"), (3, "bisect"), (4, "scatter")])
def test_partitions_match_the_whole_mesh_bit_for_bit(tmp_path, solver_mod, oracle, nparts, how):
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=40, nrec=10, src_depth=(900.0, 900.0))
    m = Mesh(d, N=3, stf_stage_time=True)
    tr0, q0 = _whole(solver_mod, m, 25)
    if how == "bisect":
        ps = Partitions(m.desc_ptr, nparts, centroids=element_centroids(m))
    else:
        ps = Partitions(m.desc_ptr, nparts, part=np.random.default_rng(5).integers(0, nparts, m.K).astype(np.int32))
    tr, q = _parted(m, ps, 25, split=11)
    assert np.array_equal(tr, tr0)
    assert np.array_equal(q, q0)
    # and the oracle on the whole mesh agrees with both
    to = run_oracle(oracle, m, precision=64, steps=25)
    assert trace_misfit(tr[:, :25], to[:, :25]) < 1e-4
    ps.close()


def test_rk3_and_batched_partitions(tmp_path, solver_mod):
    """Three wavefield buffers (TVD-RK3: the halo writes land in the buffer
    each stage reads) and two wavefields per partition."""
    d = str(tmp_path / "cube")
    synth.write_cube(d, cells=5, nt=30)
    m = Mesh(d, N=3, timeint=3)
    tr0, q0 = _whole(solver_mod, m, 17)
    ps = Partitions(m.desc_ptr, 3, centroids=element_centroids(m))
    tr, q = _parted(m, ps, 17)
    assert np.array_equal(tr, tr0) and np.array_equal(q, q0)
    ps.close()
    d = str(tmp_path / "tlb")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=20, nrec=6, nsrc=2, src_depth=(900.0, 900.0))
    m = Mesh(d, N=2, stf_stage_time=True, nbatch=2)
    tr0, _ = _whole(solver_mod, m, 14)
    ps = Partitions(m.desc_ptr, 2, centroids=element_centroids(m))
    tr, _ = _parted(m, ps, 14)
    assert np.array_equal(tr, tr0)
    ps.close()


def test_partition_errors_and_bounded_wait(tmp_path, solver_mod):
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=20, nrec=4, src_depth=(900.0, 900.0))
    m = Mesh(d, N=2, stf_stage_time=True)
    ps = Partitions(m.desc_ptr, 2, centroids=element_centroids(m))
    a = solver_mod.Solver(ps.desc(0), ps.halo(0))
    b = solver_mod.Solver(ps.desc(1), ps.halo(1))
    with pytest.raises(NexdError, match="not linked"):
        a.run(1, 1)
    with pytest.raises(NexdError) as e:
        a.pml_trigger()
    assert e.value.status == _abi.NEXD_ERR_UNSUPPORTED
    connect(a, 0, export_peer(b, 0))
    with pytest.raises(NexdError, match="another partition"):
        connect(b, 0, export_peer(b, 0))
    connect(b, 0, export_peer(a, 0))
    # partition 0 steps alone: its neighbour never writes, every arrival wait
    # runs out after its limit and the run reports it
    lib = _abi.gpu_lib()
    assert lib.nexd_halo_set_timeout(a._ctx, 0.05) == 0
    with pytest.raises(NexdError) as e:
        a.run(1, 1)
    assert e.value.status == _abi.NEXD_ERR_TIMEOUT
    a.close()
    b.close()
    ps.close()


def test_bulk_kernels_in_partitions_and_batches(tmp_path, solver_mod):
    """The stage kernels whose element-local state moves by bulk copies (NPML
    elements and the other anelastic elements), run on two wavefields per
    launch and on partitions linked by the halo exchange, give the FP32
    kernels' traces and wavefields on the whole mesh bit for bit."""
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=30, nrec=8, nsrc=2, src_depth=(900.0, 900.0))
    m = Mesh(d, N=3, stf_stage_time=True, nbatch=2)
    ref = solver_mod.Solver(m.desc_ptr)
    ref.run(1, 20)
    tr0, q0, q1 = ref.traces(), ref.field(0), ref.field(1)
    ref.close()
    s = solver_mod.Solver(m.desc_ptr)
    s.set_contraction_kinds("fp32_bulk", "fp32_bulk")
    s.run(1, 20)
    assert np.array_equal(s.traces(), tr0)
    assert np.array_equal(s.field(0), q0) and np.array_equal(s.field(1), q1)
    s.close()
    ps = Partitions(m.desc_ptr, 3, centroids=element_centroids(m))
    p = PartitionedSolver(ps, nrec_total=m.nrec)
    for sv in p.solvers:
        sv.set_contraction_kinds("fp32_bulk", "fp32_bulk")
    p.run(1, 9)
    p.run(10, 20)
    assert np.array_equal(p.traces(), tr0)
    assert np.array_equal(p.field(m.K, m.Np, 0), q0) and np.array_equal(p.field(m.K, m.Np, 1), q1)
    p.close()
    ps.close()
