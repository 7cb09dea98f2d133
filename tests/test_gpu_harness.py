"""The C driver lib/nexd_solve (harness/nexd_solve.c) on the reference's own
brick example: it reads the mesher inputs and data files, runs the time loop
on the GPU through the C-ABI and writes the reference's seismogram files.
Its seismograms equal the Python (ctypes) path's traces of the same
descriptor, and those of the stations that do not sit on a vertex shared by
several elements match the reference's golden seismograms."""
import os
import subprocess

import numpy as np
import pytest

from conftest import BRICK_EDGE_STATIONS, PKG, brick_dt_cfl, rel_l2, station_misfit, write_brick
from nexd_b200 import Mesh

pytestmark = pytest.mark.gpu


def _read_seismograms(outdir, recnr, nt):
    out = np.zeros((len(recnr), nt, 9))
    for r, nr in enumerate(recnr):
        for k, kind in enumerate(("sdu", "sdv", "sda")):
            for c, comp in enumerate("xyz"):
                a = np.loadtxt(os.path.join(outdir, f"seismo.{comp}.{nr:07d}.{kind}"))
                assert a.shape == (nt, 2)
                out[r, :, 3 * k + c] = a[:, 1]
    return out, a[:, 0]


def test_c_harness_runs_the_brick_example(tmp_path):
    from nexd_b200.solver import Solver
    golden, gtime = write_brick(str(tmp_path))
    exe = os.path.join(PKG, "lib", "nexd_solve")
    out = str(tmp_path / "out_c")
    r = subprocess.run([exe, str(tmp_path), "--cfl", repr(brick_dt_cfl()), "--out", out], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    m = Mesh(str(tmp_path), N=4, cfl=brick_dt_cfl())
    recnr = [int(x) for x in m.array("recnr")]
    tc, t_axis = _read_seismograms(out, recnr, m.nt)
    assert np.allclose(t_axis, np.asarray(gtime, dtype=np.float64).ravel()[:m.nt], rtol=1e-6)
    # the same descriptor through ctypes: the files hold the same traces (9 printed digits)
    s = Solver(m.desc_ptr)
    s.run(1, m.nt)
    tp = s.traces()[..., 0].astype(np.float64)
    s.close()
    assert rel_l2(tc, tp) < 1e-7
    untied = [i for i in range(len(recnr)) if i not in BRICK_EDGE_STATIONS]
    assert station_misfit(tc[untied], np.asarray(golden)[untied]) < 2e-4
