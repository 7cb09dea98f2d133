"""Host side of the learned absorbing boundary (no GPU): face-frame features
and their inverse, the wide/small model pair and its element map, and the
FP64 MLP oracle against finite differences."""
import os
import sys

import numpy as np

from nexd_b200 import Mesh, boundary

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle  # noqa: E402


def _frames(rng, nf):
    n = rng.standard_normal((nf, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    a = rng.standard_normal((nf, 3))
    s = a - (a * n).sum(1, keepdims=True) * n
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    t = np.cross(n, s)
    return n, s, t, rng.uniform(5e6, 2e7, nf)


def test_features_are_characteristics():
    rng = np.random.default_rng(0)
    nf, npf = 7, 15
    n, s, t, zp = _frames(rng, nf)
    zs = zp / 1.7
    q = rng.standard_normal((nf, 9, npf)) * np.array([1e6] * 6 + [0.1] * 3)[None, :, None]
    x = boundary.characteristics(q, n, s, t, zp, zs)
    assert x.shape == (nf, 9 * npf)
    f = boundary.features(q, n, s, t, zp, zs).reshape(nf, npf, 9)
    assert np.all(f[..., :3] == 0) and np.allclose(f[..., 3:], x.reshape(nf, npf, 9)[..., 3:])
    S = np.zeros((3, 3))
    S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[1, 2], S[0, 2] = q[0, :6, 0]
    S = S + np.triu(S, 1).T
    v = q[0, 6:9, 0]
    # node 0 of face 0: incoming and outgoing P and S values over Zp
    assert np.isclose(x[0, 0], (n[0] @ S @ n[0] - zp[0] * v @ n[0]) / zp[0])
    assert np.isclose(x[0, 3], (n[0] @ S @ n[0] + zp[0] * v @ n[0]) / zp[0])
    assert np.isclose(x[0, 1], (n[0] @ S @ s[0] - zs[0] * v @ s[0]) / zp[0])
    assert np.isclose(x[0, 5], (n[0] @ S @ t[0] + zs[0] * v @ t[0]) / zp[0])
    assert np.isclose(x[0, 8], s[0] @ S @ t[0] / zp[0])
    xn, yn, r = boundary.normalise(x, 2 * x)
    assert np.allclose(np.sqrt((xn ** 2).mean(1)), 1.0) and np.allclose(yn, 2 * xn)
    # the ghost state carries the clamped incoming values as its traction
    y = boundary.incoming_only(xn * 10.0, npf)
    g = boundary.ghost_states(xn, y, r, n, s, t, zp, 0.5, npf)
    gx = boundary.characteristics(g, n, s, t, zp, zs).reshape(nf, npf, 9)
    b = 0.5 * np.abs(xn.reshape(nf, npf, 9)[..., 3:6])
    want = np.clip(y.reshape(nf, npf, 9)[..., :3], -b, b) * r[:, None, None]
    assert np.allclose(gx[..., :3], want, rtol=1e-7, atol=1e-9 * np.abs(want).max())
    assert np.allclose(gx[..., :3], gx[..., 3:6])  # zero velocity: the ghost's incoming and outgoing values agree
    assert 0 < (np.abs(want) < b * r[:, None, None] * (1 - 1e-12)).mean() < 1  # the clamp binds on some nodes


def _centroids(d):
    coord = np.loadtxt(os.path.join(d, "cubit", "coord"), skiprows=1)[:, 1:]
    tets = np.loadtxt(os.path.join(d, "cubit", "mesh"), skiprows=1)[:, 1:5].astype(int) - 1
    return coord[tets].mean(axis=1), tets, coord


def test_model_pair_maps_identical_tetrahedra(tmp_path):
    w, s = str(tmp_path / "w"), str(tmp_path / "s")
    m = boundary.write_model_pair(w, s, cells=(3, 2, 2), h=200.0, pml_cells=2, nt=5,
                                  sources=boundary.random_sources(1, (3, 2, 2), 200.0, 0, depth=(150, 250), margin=1),
                                  stations=boundary.surface_stations((3, 2, 2), 200.0, 1))
    cs, ts, xs = _centroids(s)
    cw, tw, xw = _centroids(w)
    assert len(m) == len(cs)
    assert np.allclose(cw[m], cs, atol=1e-6)
    # same local vertex order: the vertices coincide one by one
    assert np.allclose(xw[tw[m]], xs[ts], atol=1e-6)
    ms = Mesh(s, N=2)
    mw = Mesh(w, N=2)
    face = ms.array("face")
    assert (face == -2).sum() > 0 and mw.array("pmlcheck").sum() > 0
    # a small model's absorbing face is an interior face of the wide model
    e, f = np.nonzero(face.T == -2)
    assert (mw.array("face")[f, m[e]] > 0).all()


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    nin, h, B = 6, 5, 4
    p = rng.standard_normal(h * nin + h + h * h + h + nin * h + nin) * 0.5
    x, t = rng.standard_normal((B, nin)), rng.standard_normal((B, nin))
    loss, g = mlp_oracle.loss_grad(p, x, t, nin, h)
    eps = 1e-6
    for i in rng.choice(p.size, 25, replace=False):
        dp = np.zeros_like(p)
        dp[i] = eps
        fd = (mlp_oracle.loss_grad(p + dp, x, t, nin, h)[0] - mlp_oracle.loss_grad(p - dp, x, t, nin, h)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_vtk_cell_scalars_format(tmp_path):
    """movie_elem_it*.vtk in the layout of the reference's
    writeVtkTetraMeshRealdata (legacy ASCII, CELLS of 4 corners, type 10,
    CELL_DATA 'data')."""
    from nexd_b200 import synth, vtk
    d = str(tmp_path / "m")
    synth.write_cube(d, cells=2, nt=2)
    coord, tets = vtk.read_cubit_mesh(d)
    data = np.arange(len(tets), dtype=float) * 0.5
    p = vtk.write_movie(d, str(tmp_path / "out"), [data], frame_step=10)[0]
    assert p.endswith("movie_elem_it0000010.vtk")
    lines = open(p).read().split("\n")
    assert lines[:4] == ["# vtk DataFile Version 3.1", "Mesh with Data", "ASCII", "DATASET UNSTRUCTURED_GRID"]
    assert lines[4].split() == ["POINTS", str(len(coord)), "float"]
    i = lines.index(next(l for l in lines if l.startswith("CELLS")))
    assert lines[i].split()[1:] == [str(len(tets)), str(5 * len(tets))]
    cells = np.array([l.split() for l in lines[i + 1:i + 1 + len(tets)]], dtype=int)
    assert (cells[:, 0] == 4).all() and np.array_equal(cells[:, 1:], tets)
    j = lines.index(next(l for l in lines if l.startswith("CELL_DATA")))
    assert lines[j + 1] == "SCALARS data float" and lines[j + 2] == "LOOKUP_TABLE default"
    assert np.allclose(np.array(lines[j + 3:j + 3 + len(tets)], dtype=float), data)
