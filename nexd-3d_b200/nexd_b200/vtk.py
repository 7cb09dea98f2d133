"""Legacy-VTK output of movie snapshots, in the format of the reference's
writeVtkTetraMeshRealdata (src/vtkMod.f90:70-111): the tetrahedral mesh by its
corner vertices and one float per element (CELL_DATA), as collectMovie
writes movie_elem_it%07d.vtk (src/collectMovieMod.f90:180-185)."""
import os

import numpy as np


def read_cubit_mesh(directory):
    """Corner vertices (ncoord, 3) and tetrahedra (nelem, 4, 0-based) of a
    simulation directory's cubit/coord and cubit/mesh files."""
    coord = np.loadtxt(os.path.join(directory, "cubit", "coord"), skiprows=1, ndmin=2)[:, 1:4]
    mesh = np.loadtxt(os.path.join(directory, "cubit", "mesh"), skiprows=1, ndmin=2)
    return coord, mesh[:, 1:5].astype(np.int64) - 1


def write_cell_scalars(path, coord, tets, data):
    """One legacy ASCII VTK file: POINTS, CELLS (type 10), CELL_DATA 'data'."""
    coord = np.asarray(coord, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    data = np.asarray(data, dtype=np.float64)
    n, k = len(coord), len(tets)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.1\nMesh with Data\nASCII\nDATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {n:12d} float\n")
        np.savetxt(f, coord, fmt="%18.6e")
        f.write(f"\nCELLS {k:12d}{5 * k:12d}\n")
        np.savetxt(f, np.column_stack([np.full(k, 4), tets]), fmt="%12d")
        f.write(f"\nCELL_TYPES {k:12d}\n")
        np.savetxt(f, np.full((k, 1), 10), fmt="%d")
        f.write(f"\nCELL_DATA {k:12d}\nSCALARS data float\nLOOKUP_TABLE default\n")
        np.savetxt(f, data, fmt="%.6e")


def write_movie(directory, outdir, frames, frame_step):
    """movie_elem_it%07d.vtk for every stored frame of one wavefield (frames:
    (nframes, nelem)); frame i is step (i + 1) * frame_step."""
    coord, tets = read_cubit_mesh(directory)
    os.makedirs(outdir, exist_ok=True)
    paths = []
    for i, fr in enumerate(frames):
        p = os.path.join(outdir, f"movie_elem_it{(i + 1) * frame_step:07d}.vtk")
        write_cell_scalars(p, coord, tets, fr)
        paths.append(p)
    return paths
