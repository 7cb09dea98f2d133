"""Host database builder (libnexd_host.so): operators, geometry, topology,
source/receiver location and the dt known answer of the reference's brick."""
import math
import os

import numpy as np
import pytest

from conftest import write_brick, brick_dt_cfl
from nexd_b200 import Mesh, NexdError, synth


@pytest.fixture(scope="module")
def brick_dir(tmp_path_factory, built):
    d = tmp_path_factory.mktemp("brick")
    write_brick(str(d))
    return str(d)


@pytest.fixture(scope="module")
def brick(brick_dir):
    return Mesh(brick_dir, N=4)


def small_cube(tmp_path, N, cells=4, **kw):
    d = str(tmp_path / f"cube{N}_{cells}")
    synth.write_cube(d, cells=cells, nt=10)
    return Mesh(d, N=N, **kw)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_physical_derivatives_exact(tmp_path, built, N):
    """Dx = rx Dr + sx Ds + tx Dt differentiates polynomials of degree N exactly
    on every (jittered, affine) element."""
    m = small_cube(tmp_path, N)
    Np = m.Np
    Dr, Ds, Dt = m.array("Dr"), m.array("Ds"), m.array("Dt")
    met = m.array("metric")
    vx, vy, vz = m.array("vx"), m.array("vy"), m.array("vz")
    worst = 0.0
    for e in range(0, m.K, 7):
        sl = slice(e * Np, (e + 1) * Np)
        x, y, z = vx[sl], vy[sl], vz[sl]
        rx, ry, rz, sx, sy, sz, tx, ty, tz = met[:, e]
        Dx = rx * Dr + sx * Ds + tx * Dt
        Dy = ry * Dr + sy * Ds + ty * Dt
        Dz = rz * Dr + sz * Ds + tz * Dt
        L = 2000.0
        xs, ys, zs = x / L, y / L, z / L
        f = xs ** (N - 1) * ys + zs ** N
        dfx = (N - 1) * xs ** (N - 2) * ys / L if N >= 2 else np.zeros(Np)
        dfy = xs ** (N - 1) / L
        dfz = N * zs ** (N - 1) / L
        worst = max(worst, np.abs(Dx @ f - dfx).max() * L, np.abs(Dy @ f - dfy).max() * L,
                    np.abs(Dz @ f - dfz).max() * L)
        worst = max(worst, np.abs(Dx @ np.ones(Np)).max() * L, np.abs(Dy @ x).max(), np.abs(Dx @ x - 1).max())
    assert worst < 1e-9 * 10 ** N


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_mass_and_lift(tmp_path, built, N):
    """V is orthonormal (M^-1 = V V^T) and LIFT = M^-1 E with the face mass
    matrices: M LIFT integrates a unit face function to the face area 2."""
    m = small_cube(tmp_path, N)
    M, Minv, LIFT = m.array("mass"), m.array("invmass"), m.array("lift")
    assert np.abs(M @ Minv - np.eye(m.Np)).max() < 1e-10
    E = M @ LIFT
    for f in range(4):
        blk = E[:, f * m.NpF:(f + 1) * m.NpF]
        assert abs(blk.sum() - 2.0) < 1e-10
        # E vanishes off the face's nodes
        fm = m.array("fmask")[:, f] - 1
        off = np.setdiff1d(np.arange(m.Np), fm)
        assert np.abs(blk[off]).max() < 1e-10


def test_brick_dt_known_answer(brick):
    """dt = dtfactor * cfl reproduces the reference's brick time step
    6.46257467e-06 s (golden seismogram time axis).  The reference computes the
    Jacobians in FP32 from absolute coordinates (Dr*x), which moves dtfactor by
    ~1.3e-5; the FP64 value agrees within 2e-5."""
    assert abs(brick.dt - 6.46257467e-06) / 6.46257467e-06 < 2e-5
    assert brick.K == 9859 and brick.Np == 35 and brick.NpF == 15


def test_brick_topology(brick):
    face = brick.array("face")
    nb = brick.array("neighbor")
    assert (face == -1).sum() == 220
    assert (face == -2).sum() == 1104
    # neighbour relation is symmetric and face ids point back
    K = brick.K
    for e in range(0, K, 13):
        for f in range(4):
            n = nb[f, e]
            if n > 0:
                assert nb[face[f, e] - 1, n - 1] == e + 1
    # ibn nodes coincide with this element's face nodes
    vx, vy, vz = brick.array("vx"), brick.array("vy"), brick.array("vz")
    ibn = brick.array("ibn")
    fmask = brick.array("fmask") - 1
    Np = brick.Np
    worst = 0.0
    for e in range(0, K, 11):
        for f in range(4):
            if nb[f, e] > 0:
                own = e * Np + fmask[:, f]
                oth = ibn[:, f, e] - 1
                worst = max(worst, np.abs(vx[own] - vx[oth]).max(), np.abs(vy[own] - vy[oth]).max(),
                            np.abs(vz[own] - vz[oth]).max())
    assert worst < 1e-9


def test_brick_locations(brick):
    """Located reference coordinates map back to the requested positions."""
    Np = brick.Np
    vx, vy, vz = brick.array("vx"), brick.array("vy"), brick.array("vz")
    V = brick.array("vdm")
    for arr_e, arr_i, targets in (("srcelem", "srcInt", [(5.0, 5.0, 5.0)]),
                                  ("recelem", "recInt", [(float(i), 5.0, 10.0) for i in range(11)])):
        el, w = brick.array(arr_e), brick.array(arr_i)
        for k, t in enumerate(targets):
            sl = slice((el[k] - 1) * Np, el[k] * Np)
            pos = (w[:, k] @ vx[sl], w[:, k] @ vy[sl], w[:, k] @ vz[sl])
            assert np.allclose(pos, t, atol=1e-9), (arr_e, k, pos)
            assert abs(w[:, k].sum() - 1.0) < 1e-12
    assert V.shape == (Np, Np)


def test_synth_cube_counts(tmp_path, built):
    d = str(tmp_path / "cube")
    info = synth.write_cube(d)
    m = Mesh(d, N=3)
    assert info["nelem"] == 6000 == m.K
    face = m.array("face")
    assert (face == -1).sum() == 200 and (face == -2).sum() == 1000
    assert m.nrec == 9 and m.nsrc == 1 and m.nt == 1000
    assert m.desc.timeint == 4


def test_missing_input_raises(tmp_path, built):
    with pytest.raises(NexdError):
        Mesh(str(tmp_path / "nothing"), N=3)


def test_unassigned_boundary_raises(tmp_path, built):
    d = str(tmp_path / "cube")
    synth.write_cube(d, cells=2, nt=5)
    with open(os.path.join(d, "cubit", "absorb")) as f:
        lines = f.read().splitlines()
    with open(os.path.join(d, "cubit", "absorb"), "w") as f:
        f.write(f"{int(lines[0]) - 1}\n" + "\n".join(lines[2:]) + "\n")
    with pytest.raises(NexdError, match="not assigned"):
        Mesh(d, N=2)


def test_source_search_gives_up_like_the_reference(tmp_path, built):
    """findSource (src/sourceReceiverMod.f90:243-356) starts at the element of
    the node nearest the source and gives up after 20 rejected elements with
    "could not find source": at N = 4 a source on a vertical cell edge of a
    4 x 4 x 2 box, where many tets share the nearest node, is not found. The
    same point inside a cell of a 5 x 5 x 2 box is."""
    d = str(tmp_path / "edge")
    synth.write_twolayer(d, cells=(4, 4, 2), nt=5, nrec=0, src_depth=(900.0, 900.0))
    with pytest.raises(NexdError, match="could not find source 1 at global coordinates 2000 2000 1100"):
        Mesh(d, N=4)
    d = str(tmp_path / "inside")
    synth.write_twolayer(d, cells=(5, 5, 2), nt=5, nrec=0, src_depth=(900.0, 900.0))
    assert Mesh(d, N=4).K == 300


def test_zener_fit_quality(tmp_path, built):
    """Kaeser et al. (2007) eq. 6: the fitted mechanisms reproduce 1/Q within a
    few percent across the fitted band (src/anelasticMod.f90:59-179)."""
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(4, 4, 2), nt=5, nrec=2)
    m = Mesh(d, N=2)
    wl = m.array("wl")
    yl, ymu = m.array("ylambda")[:, 0], m.array("ymu")[:, 0]
    lam_u, mu_u = m.array("lambdau")[0], m.array("muu")[0]
    # P modulus coefficients Yp = (lam Ylam + 2 mu Ymu)/(lam + 2 mu)
    yp = (lam_u * yl + 2 * mu_u * ymu) / (lam_u + 2 * mu_u)
    for y, Qt in ((yp, 400.0), (ymu, 200.0)):
        for w in np.geomspace(wl[0] * 1.2, wl[-1] / 1.2, 9):
            num = 1.0 - np.sum(wl ** 2 * y / (wl ** 2 + w ** 2))
            den = np.sum(wl * w * y / (wl ** 2 + w ** 2))
            Q = num / den
            assert abs(Q - Qt) / Qt < 0.06, (Qt, w, Q)
