"""Synthetic simulation directories in the reference's input formats.

The reference meshes with Cubit and exports through cubit2dg3d.py
(simulations/*/cubit/cubit2dg3d.py); its mesher reads the exported text files
cubit/{coord,mesh,mat,matprop,free,absorb} (src/meshMod.f90:146-319) and the
solver inputs data/{parfile,source,stations} (src/parameterMod.f90:30-103,
src/sourceReceiverMod.f90:36-201).  This module writes the same files for
structured boxes split into tetrahedra (6 per hexahedron, all sharing the
hexahedron's main diagonal, which keeps neighbouring hexahedra conforming),
with seeded interior-node jitter, layered materials, NPML flags, a free top
surface and absorbing sides.  The workloads below are seeded synthetic
stand-ins; no external data set is involved.
"""
import itertools
import math
import os

import numpy as np

_PERMS = list(itertools.permutations(range(3)))


def _box_mesh(x0, x1, y0, y1, z0, z1, nx, ny, nz, jitter, seed):
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    zs = np.linspace(z0, z1, nz + 1)
    I, J, Kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    I, J, Kk = I.ravel(order="F"), J.ravel(order="F"), Kk.ravel(order="F")
    coord = np.stack([xs[I], ys[J], zs[Kk]], axis=1)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        h = np.array([(x1 - x0) / nx, (y1 - y0) / ny, (z1 - z0) / nz])
        interior = (I > 0) & (I < nx) & (J > 0) & (J < ny) & (Kk > 0) & (Kk < nz)
        d = rng.uniform(-jitter, jitter, size=coord.shape) * h
        coord[interior] += d[interior]

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    tets = []
    hi, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hi, hj, hk = hi.ravel(order="F"), hj.ravel(order="F"), hk.ravel(order="F")
    unit = np.eye(3, dtype=int)
    for perm in _PERMS:
        a, b = unit[perm[0]], unit[perm[0]] + unit[perm[1]]
        v0 = vid(hi, hj, hk)
        v1 = vid(hi + a[0], hj + a[1], hk + a[2])
        v2 = vid(hi + b[0], hj + b[1], hk + b[2])
        v3 = vid(hi + 1, hj + 1, hk + 1)
        tets.append(np.stack([v0, v1, v2, v3], axis=1))
    # order: hexahedron-major, the 6 tetrahedra of one hexahedron consecutive
    tets = np.stack(tets, axis=1).reshape(-1, 4)
    # positive orientation
    X = coord[tets]
    det = np.einsum("ki,ki->k", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]))
    neg = det < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    return coord, tets, (I, J, Kk)


def _boundary_faces(tets, ijk, nx, ny, nz):
    """Boundary faces as (elem, n1, n2, n3, side) with side in xmin,xmax,ymin,ymax,zmin,zmax."""
    I, J, Kk = ijk
    out = {s: [] for s in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    tests = [("xmin", I, 0), ("xmax", I, nx), ("ymin", J, 0), ("ymax", J, ny), ("zmin", Kk, 0), ("zmax", Kk, nz)]
    for opp in range(4):
        face = tets[:, [v for v in range(4) if v != opp]]
        for side, arr, val in tests:
            on = np.all(arr[face] == val, axis=1)
            idx = np.nonzero(on)[0]
            if len(idx):
                out[side].append(np.concatenate([idx[:, None] + 1, face[idx] + 1], axis=1))
    return {k: (np.concatenate(v) if v else np.zeros((0, 4), dtype=int)) for k, v in out.items()}


def double_couple(strike, dip, rake, m0=1.0):
    """Moment tensor (Mxx, Myy, Mzz, Mxy, Mxz, Myz) of a double couple, x east,
    y north, z up, from Aki & Richards (2002, box 4.4) in north-east-down."""
    s, d, r = math.radians(strike), math.radians(dip), math.radians(rake)
    mnn = -m0 * (math.sin(d) * math.cos(r) * math.sin(2 * s) + math.sin(2 * d) * math.sin(r) * math.sin(s) ** 2)
    mne = m0 * (math.sin(d) * math.cos(r) * math.cos(2 * s) + 0.5 * math.sin(2 * d) * math.sin(r) * math.sin(2 * s))
    mnd = -m0 * (math.cos(d) * math.cos(r) * math.cos(s) + math.cos(2 * d) * math.sin(r) * math.sin(s))
    mee = m0 * (math.sin(d) * math.cos(r) * math.sin(2 * s) - math.sin(2 * d) * math.sin(r) * math.cos(s) ** 2)
    med = -m0 * (math.cos(d) * math.cos(r) * math.sin(s) - math.cos(2 * d) * math.sin(r) * math.cos(s))
    mdd = m0 * math.sin(2 * d) * math.sin(r)
    # east-north-up: x=e, y=n, z=-d
    return (mee, mnn, mdd, mne, -med, -mnd)


def write_simulation(directory, *, box, cells, jitter=0.05, seed=1, layers=None, pml_cells=0, free_top=True,
                     parfile=None, sources=(), stations=()):
    """Write cubit/* and data/* for a structured box.

    box = (x0, x1, y0, y1, z0, z1); cells = (nx, ny, nz);
    layers: list of (z_min, vp, vs, rho, qp, qs), the first whose z_min is below
    an element's centroid applies (list top-down, last entry with z_min=-inf);
    pml_cells: NPML thickness in cells on the four sides and the bottom.
    """
    x0, x1, y0, y1, z0, z1 = box
    nx, ny, nz = cells
    os.makedirs(os.path.join(directory, "cubit"), exist_ok=True)
    os.makedirs(os.path.join(directory, "data"), exist_ok=True)
    coord, tets, ijk = _box_mesh(x0, x1, y0, y1, z0, z1, nx, ny, nz, jitter, seed)
    K = len(tets)
    if not layers:
        layers = [(-math.inf, 4000.0, 2310.0, 2700.0, 9000.0, 9000.0)]
    cen = coord[tets].mean(axis=1)
    mat = np.zeros(K, dtype=int)
    assigned = np.zeros(K, dtype=bool)
    for li, (zmin, *_r) in enumerate(layers):
        sel = (~assigned) & (cen[:, 2] > zmin)
        mat[sel] = li + 1
        assigned |= sel
    mat[~assigned] = len(layers)
    props = np.array([l[1:] for l in layers], dtype=float)[mat - 1]
    pml = np.zeros(K, dtype=int)
    if pml_cells > 0:
        hx, hy, hz = (x1 - x0) / nx, (y1 - y0) / ny, (z1 - z0) / nz
        pml = ((cen[:, 0] < x0 + pml_cells * hx) | (cen[:, 0] > x1 - pml_cells * hx) |
               (cen[:, 1] < y0 + pml_cells * hy) | (cen[:, 1] > y1 - pml_cells * hy) |
               (cen[:, 2] < z0 + pml_cells * hz)).astype(int)
    bf = _boundary_faces(tets, ijk, nx, ny, nz)
    free = bf["zmax"] if free_top else np.zeros((0, 4), dtype=int)
    absorb = np.concatenate([bf[s] for s in ("xmin", "xmax", "ymin", "ymax", "zmin")] +
                            ([] if free_top else [bf["zmax"]]))
    cub = os.path.join(directory, "cubit")
    ids = np.arange(1, len(coord) + 1)
    with open(os.path.join(cub, "coord"), "w") as f:
        f.write(f"{len(coord)}\n")
        np.savetxt(f, np.column_stack([ids, coord]), fmt=["%d", "%.9f", "%.9f", "%.9f"])
    with open(os.path.join(cub, "mesh"), "w") as f:
        f.write(f"{K}\n")
        np.savetxt(f, np.column_stack([np.arange(1, K + 1), tets + 1, props]),
                   fmt=["%d"] * 5 + ["%.6f"] * 5)
    with open(os.path.join(cub, "mat"), "w") as f:
        np.savetxt(f, np.column_stack([np.arange(1, K + 1), mat, pml]), fmt="%d")
    with open(os.path.join(cub, "matprop"), "w") as f:
        f.write(f"{len(layers)}\n")
        for i, l in enumerate(layers):
            f.write(f"{i + 1} {i + 1} {l[1]} {l[2]} {l[3]} {l[4]} {l[5]}\n")
    for name, arr in (("free", free), ("absorb", absorb)):
        with open(os.path.join(cub, name), "w") as f:
            f.write(f"{len(arr)}\n")
            if len(arr):
                np.savetxt(f, arr, fmt="%d")
    par = dict(log=".false.", external=".true.", nproc=1, vtk=".false.", movie=".false.", frame=10, timeint=4,
               nt=1000, cfl=0.3, attenuation=".false.", f0_att=1.0, fr_att=1.0, set_pml=".false.", pml_delta=0.0,
               pml_rc=0.01, pml_kmax=1.0, pml_afac=1.0, avg_window1=10, avg_window2=2, sta_lta_trigger=0.1)
    if parfile:
        par.update(parfile)
    with open(os.path.join(directory, "data", "parfile"), "w") as f:
        f.write("# Parameter file written by nexd_b200.synth\n")
        for k, v in par.items():
            f.write(f"{k:<16}= {v}\n")
    with open(os.path.join(directory, "data", "source"), "w") as f:
        f.write(f"nsrc            = {len(sources)}\n")
        for i, s in enumerate(sources):
            m = s.get("M", (0, 0, 0, 0, 0, 0))
            fd = s.get("force", (0.0, 0.0, 1.0))
            f.write(f"source          = {i + 1}\n")
            f.write(f"xsource         = {s['xyz'][0]!r}\nysource         = {s['xyz'][1]!r}\n"
                    f"zsource         = {s['xyz'][2]!r}\n")
            f.write(f"sourcetype      = {s.get('type', 0)}\nstf             = {s.get('stf', 2)}\n"
                    f"f0              = {s.get('f0', 1.0)!r}\nfactor          = {s.get('factor', 1.0)!r}\n")
            f.write(f"xangle_force    = {fd[0]!r}\nyangle_force    = {fd[1]!r}\nzangle_force    = {fd[2]!r}\n")
            for name, val in zip(("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"), m):
                f.write(f"{name:<16}= {float(val)!r}\n")
    with open(os.path.join(directory, "data", "stations"), "w") as f:
        f.write(f"{len(stations)}\n")
        for i, st in enumerate(stations):
            f.write(f"{i + 1:03d} {st[0]!r} {st[1]!r} {st[2]!r}\n")
    return dict(nelem=K, ncoord=len(coord), npml=int(pml.sum()))


# ---------------------------------------------------------------------------
# The benchmark models (sizes and material values as the benchmark workloads use them)
# ---------------------------------------------------------------------------

def write_cube(directory, *, cells=10, seed=1, nt=1000):
    """Homogeneous elastic 2 km cube, 10x10x10 hexahedra x 6 = 6,000 tets,
    free top, absorbing sides, vertical Ricker force (f0=5 Hz, t0=0.25 s) at the
    centre, 3x3 surface receivers, LSERK4 at CFL 0.3."""
    L = 2000.0
    st = [(x, y, L) for y in (500.0, 1000.0, 1500.0) for x in (500.0, 1000.0, 1500.0)]
    return write_simulation(directory, box=(0, L, 0, L, 0, L), cells=(cells, cells, cells), jitter=0.05, seed=seed,
                            layers=[(-math.inf, 4000.0, 2310.0, 2700.0, 9000.0, 9000.0)],
                            parfile=dict(timeint=4, nt=nt, cfl=0.3),
                            sources=[dict(xyz=(L / 2, L / 2, L / 2), type=0, stf=2, f0=5.0, force=(0.0, 0.0, 1.0))],
                            stations=st)


def write_twolayer(directory, *, cells=(40, 40, 20), seed=2, nt=3000, nrec=100, nsrc=1, attenuation=True,
                   pml=True, f0=3.0, src_depth=(1500.0, 1500.0), f0_range=None, src_seed=None, homogeneous=False):
    """Two-layer anelastic box 4x4x2 km (40x40x20 hexahedra x 6 = 192,000 tets):
    upper 600 m vp 3000 / vs 1730 / rho 2400 / Qp 100 / Qs 50, half-space 5000 /
    2890 / 2800 / 400 / 200; 3-cell NPML on the sides and bottom, free top;
    seeded double-couple sources (Ricker), random surface receivers.
    homogeneous: the half-space material everywhere."""
    Lx, Ly, Lz = 4000.0, 4000.0, 2000.0
    nx, ny, nz = cells
    rng = np.random.default_rng(seed if src_seed is None else src_seed)
    hx = Lx / nx
    margin = min(4 * hx, 0.25 * Lx)
    srcs = []
    for i in range(nsrc):
        strike, dip, rake = rng.uniform(0, 360), rng.uniform(10, 90), rng.uniform(-180, 180)
        depth = rng.uniform(*src_depth) if src_depth[0] != src_depth[1] else src_depth[0]
        x = Lx / 2 if nsrc == 1 else rng.uniform(margin, Lx - margin)
        y = Ly / 2 if nsrc == 1 else rng.uniform(margin, Ly - margin)
        f = f0 if f0_range is None else rng.uniform(*f0_range)
        srcs.append(dict(xyz=(float(x), float(y), float(Lz - depth)), type=1, stf=2, f0=float(f),
                         M=double_couple(strike, dip, rake, m0=1e15)))
    recs = [(float(rng.uniform(margin, Lx - margin)), float(rng.uniform(margin, Ly - margin)), Lz)
            for _ in range(nrec)]
    par = dict(timeint=4, nt=nt, cfl=0.3)
    if attenuation:
        par.update(attenuation=".true.", f0_att=round(2 * math.pi * f0, 6), fr_att=100.0)
    if pml:
        par.update(set_pml=".true.", pml_delta=3 * hx, pml_rc=0.001, pml_kmax=1.0, pml_afac=1.0)
    return write_simulation(directory, box=(0, Lx, 0, Ly, 0, Lz), cells=cells, jitter=0.05, seed=seed,
                            layers=([(-math.inf, 5000.0, 2890.0, 2800.0, 400.0, 200.0)] if homogeneous else
                                    [(Lz - 600.0, 3000.0, 1730.0, 2400.0, 100.0, 50.0),
                                     (-math.inf, 5000.0, 2890.0, 2800.0, 400.0, 200.0)]),
                            pml_cells=3 if pml else 0, parfile=par, sources=srcs, stations=recs)
