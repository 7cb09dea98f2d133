"""Pack the reference's brick example into tests/golden/brick.npz.

Source: simulations/brick/{cubit,data,ref} of the NEXD-3D reference
(Cubit tetmesh of a 10 m cube, 9859 tets; z-force Ricker source; 11 surface
stations; RK2, cfl 0.4, nt 1000; golden seismograms seismo.{x,y,z}.%07d.sd{u,v,a}
produced by the reference solver in FP32).  The test suite rewrites the text
inputs from this archive, so nothing reads the reference tree at test time.

Usage: python tests/golden/make_brick_fixture.py /path/to/reference
"""
import os
import sys

import numpy as np


def main(ref_root):
    b = os.path.join(ref_root, "simulations", "brick")
    coord = np.loadtxt(os.path.join(b, "cubit", "coord"), skiprows=1)
    mesh = np.loadtxt(os.path.join(b, "cubit", "mesh"), skiprows=1)
    mat = np.loadtxt(os.path.join(b, "cubit", "mat"), dtype=np.int64)
    free = np.loadtxt(os.path.join(b, "cubit", "free"), skiprows=1, dtype=np.int64)
    absorb = np.loadtxt(os.path.join(b, "cubit", "absorb"), skiprows=1, dtype=np.int64)
    with open(os.path.join(b, "cubit", "matprop")) as f:
        matprop = f.read()
    with open(os.path.join(b, "data", "parfile")) as f:
        parfile = f.read()
    with open(os.path.join(b, "data", "source")) as f:
        source = f.read()
    with open(os.path.join(b, "data", "stations")) as f:
        stations = f.read()
    nrec = int(stations.split()[0])
    traces = np.zeros((nrec, 1000, 9), dtype=np.float32)
    time = None
    for r in range(nrec):
        for k, kind in enumerate(("sdu", "sdv", "sda")):
            for c, comp in enumerate("xyz"):
                a = np.loadtxt(os.path.join(b, "ref", f"seismo.{comp}.{r + 1:07d}.{kind}"))
                traces[r, :, 3 * k + c] = a[:, 1]
                time = a[:, 0]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "brick.npz")
    np.savez_compressed(
        out,
        coord=coord[:, 1:].astype(np.float64),
        tets=mesh[:, 1:5].astype(np.int32),
        props=mesh[:, 5:10].astype(np.float64),
        mat=mat.astype(np.int32),
        free=free.astype(np.int32),
        absorb=absorb.astype(np.int32),
        matprop=np.array(matprop),
        parfile=np.array(parfile),
        source=np.array(source),
        stations=np.array(stations),
        traces=traces,
        time=time.astype(np.float64),
    )
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python make_brick_fixture.py <path of the NEXD-3D source tree>")
    main(sys.argv[1])
