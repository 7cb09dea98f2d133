"""Movie snapshots on the device (nexd_movie): the per-element mean of |u|
with u integrated at every node equals the same quantity integrated on the
host from the step-by-step wavefields; graph replay gives the same frames."""
import numpy as np
import pytest

from conftest import rel_l2
from nexd_b200 import Mesh, synth

pytestmark = pytest.mark.gpu


def test_movie_frames_match_host_integration(tmp_path):
    from nexd_b200.solver import Solver
    d = str(tmp_path / "cube")
    synth.write_cube(d, cells=6, nt=12)
    m = Mesh(d, N=3, stf_stage_time=True)
    a = Solver(m.desc_ptr)
    a.movie(4, max_frames=8)
    u = np.full((m.K * m.Np, 3), 1e-24)
    want = []
    for it in range(1, 13):
        a.run(it, it)
        v = a.field()[:, 6:9].astype(np.float64)
        u += np.float32(m.dt) * v
        if it % 4 == 0:
            want.append(np.linalg.norm(u, axis=1).reshape(m.K, m.Np).mean(axis=1))
    got = a.movie_frames()[0]
    assert got.shape == (3, m.K)
    assert rel_l2(got, np.array(want)) < 1e-5
    b = Solver(m.desc_ptr)
    b.movie(4, max_frames=8)
    b.run(1, 12)
    assert np.array_equal(b.movie_frames(), a.movie_frames())
    b.movie(0)
    assert b.movie_frames().shape[1] == 0
