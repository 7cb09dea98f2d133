"""Full-run FP64 oracle traces for the GPU parity tests (tests/golden/fullrun_*.npz).

The correctness bar of the GPU path is the receiver traces "after the full
run" against the FP64 solver.  These fixtures hold the FP64 oracle's traces of
two seeded synthetic models over their full step counts, so that a GPU test
can check the FP32, split-BF16 tensor-core and autotuned paths over every step
without running a long CPU job:

  cube      the homogeneous elastic 2 km cube, 10x10x10 hexahedra x 6 = 6,000
            tets, N=3, free top, absorbing sides, vertical Ricker force
            (f0 = 5 Hz, t0 = 0.25 s), 9 surface receivers, 1,000 LSERK4 steps
            at CFL 0.3 (the whole workload);
  twolayer  the two-layer anelastic model family (3 Zener mechanisms, 3-cell
            NPML on the sides and bottom, free top, double-couple source) at
            10x10x5 hexahedra x 6 = 3,000 tets, N=4, 12 surface receivers,
            3,000 LSERK4 steps (the full step count of the 192,000-tet
            workload, on a mesh the CPU finishes in minutes).

Each archive stores the traces (nrec, nt, 9) in FP32 (the oracle computes in
FP64; FP32 storage is ~6e-8 relative, far below the 1e-4 bar), the final
wavefield's per-field L2 norms (FP64), and a fingerprint of the descriptor
(K, Np, dt, sums of the geometry and material arrays) that the tests compare
before they trust the traces.  The meshes are rebuilt from the same seeded
generator calls by the tests (nexd_b200.synth), so only these small archives
are stored.

Usage: python tests/golden/make_fullrun_fixtures.py [cube|twolayer ...]
(needs the host library and the oracle: make -C nexd-3d_b200 host; make -C oracle)
"""
import ctypes as C
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "nexd-3d_b200"))

from nexd_b200 import Mesh, _abi, synth  # noqa: E402

# Generator calls of the two models; the GPU tests rebuild the meshes with these.
MODELS = {
    "cube": dict(writer="write_cube", kw=dict(cells=10, nt=1000), N=3),
    "twolayer": dict(writer="write_twolayer",
                     kw=dict(cells=(10, 10, 5), nt=3000, nrec=12, src_depth=(700.0, 700.0)), N=4),
}


def build(name, directory):
    spec = MODELS[name]
    getattr(synth, spec["writer"])(directory, **spec["kw"])
    return Mesh(directory, N=spec["N"], stf_stage_time=True)


def fingerprint(m):
    """Numbers that identify the descriptor: a different mesh, node set or
    material assignment changes them."""
    return np.array([m.K, m.Np, m.nrec, m.nt, m.dt, m.array("metric").sum(), np.abs(m.array("metric")).sum(),
                     m.array("jacobian").sum(), m.array("rho").sum(), m.array("vpu").sum(),
                     float(m.array("neighbor").sum()), m.array("recInt").sum(), m.array("srcInt").sum()],
                    dtype=np.float64)


def main(names):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.oracle_run.argtypes = [C.POINTER(_abi.NexdDesc), C.c_int, C.c_int, C.POINTER(C.c_float), C.c_void_p,
                               C.c_int]
    for name in names:
        with tempfile.TemporaryDirectory() as d:
            m = build(name, d)
            tr = np.zeros((m.nrec, m.nt, 9, 1), dtype=np.float32, order="F")
            field = np.zeros((m.K * m.Np, 9, 1), dtype=np.float64, order="F")
            t0 = time.perf_counter()
            st = lib.oracle_run(m.desc_ptr, 64, m.nt, tr.ctypes.data_as(C.POINTER(C.c_float)),
                                field.ctypes.data_as(C.c_void_p), 0)
            if st != 0:
                raise SystemExit(f"oracle failed on {name}: {st}")
            out = os.path.join(HERE, f"fullrun_{name}.npz")
            np.savez_compressed(out, traces=tr[..., 0], field_norms=np.linalg.norm(field[..., 0], axis=0),
                                fingerprint=fingerprint(m), nt=np.int64(m.nt))
            print(f"{name}: K={m.K} N={m.N} nt={m.nt} oracle {time.perf_counter() - t0:.0f} s -> {out} "
                  f"({os.path.getsize(out)} bytes)", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(MODELS))
