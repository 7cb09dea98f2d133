"""The multi-GPU path of bench.py on CPU: two gloo ranks run the replica
plumbing (torchrun environment, barrier, max/sum reductions, whole-job
throughput, per-rank seeded sources) that bench.py runs over NCCL."""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import PKG

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    sys.path.insert(0, PKG)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from nexd_b200 import replicas, synth
    g = replicas.init("gloo", timeout_s=60)
    assert (g.rank, g.world) == (rank, world)
    g.barrier()
    seconds = 1.0 + rank          # rank 1 is the slow one
    units = 100.0 * (rank + 1)
    res = dict(max=g.max(seconds), sum=g.sum(units), agg=replicas.aggregate(g, units, seconds))
    d = os.path.join(out_dir, f"r{rank}")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=5, nrec=2, src_seed=replicas.replica_seed(2, rank))
    src = open(os.path.join(d, "data", "source")).read()
    # end of run: each replica's receiver traces (nrec, nt, 9, nbatch) gathered on rank 0
    traces = np.full((2, 5, 9, 1), float(rank + 1), dtype=np.float32, order="F")
    traces[0, :, 0, 0] = np.arange(5) + 10 * rank
    gathered = replicas.gather_traces(g, traces)
    # data-parallel network training: gradients averaged over the ranks, and
    # the ranks agree on the number of steps (the smaller shard decides)
    grads = torch.full((5,), float(rank + 1))
    replicas.allreduce_mean(g, grads)
    steps = replicas.agree_min(g, 10 + 3 * rank)
    np.save(os.path.join(out_dir, f"grad{rank}.npy"), np.append(grads.numpy(), steps))
    g.barrier()
    g.close()
    if rank == 0:
        np.save(os.path.join(out_dir, "gathered.npy"), gathered)
    else:
        assert gathered is None
    np.save(os.path.join(out_dir, f"res{rank}.npy"), np.array([res["max"], res["sum"], res["agg"]]))
    with open(os.path.join(out_dir, f"src{rank}.txt"), "w") as f:
        f.write(src)


def test_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"res{r}.npy") for r in range(world))
    # max of the times, sum of the units, whole-job throughput = sum / max
    assert np.allclose(r0, r1)
    assert r0[0] == 2.0 and r0[1] == 300.0 and np.isclose(r0[2], 150.0)
    # each rank's replica has its own seeded source
    assert open(tmp_path / "src0.txt").read() != open(tmp_path / "src1.txt").read()
    for r in range(world):
        gr = np.load(tmp_path / f"grad{r}.npy")
        assert np.allclose(gr[:5], 1.5) and gr[5] == 10
    # rank 0 holds every replica's traces in rank order
    gathered = np.load(tmp_path / "gathered.npy")
    assert gathered.shape == (2, 2, 5, 9, 1)
    for r in range(world):
        assert np.all(gathered[r, 1] == r + 1)
        assert np.array_equal(gathered[r, 0, :, 0, 0], np.arange(5) + 10 * r)


def test_single_process_group_is_local():
    sys.path.insert(0, PKG)
    from nexd_b200 import replicas
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK") if k in os.environ}
    try:
        g = replicas.init()
        assert g.dist is None and g.world == 1
        assert replicas.gather_traces(g, np.ones((2, 3))).shape == (1, 2, 3)
        assert g.max(3.0) == 3.0 and g.sum(5.0) == 5.0 and replicas.aggregate(g, 10.0, 2.0) == 5.0
        g.barrier()
        g.close()
    finally:
        os.environ.update(env)
