"""The CPU oracle (oracle/liboracle.so) pinned against the reference's own
golden seismograms and checked for the properties the method guarantees."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import (GOLDEN, brick_dt_cfl, pin_brick_edge_stations, run_oracle, run_oracle_trigger, trace_misfit,
                      station_misfit, write_brick, rel_l2)
from nexd_b200 import Mesh, _abi, synth


@pytest.fixture(scope="module")
def brick_dir(tmp_path_factory, built):
    d = tmp_path_factory.mktemp("brick")
    golden, time = write_brick(str(d))
    return str(d), golden, time


def test_brick_golden_fp32_rk2(brick_dir, oracle):
    """FP32 + the reference's TVD-RK2 reproduces simulations/brick/ref (33 traces
    x 3 kinds, 1000 steps) at every station within 2e-4 relative L2.

    Golden traces come from the reference run on 12 MPI ranks; the
    partitioning moves halo copies only, not arithmetic.  Stations 1 and 11 sit
    on mesh vertices shared by six elements; the reference's choice of element
    is pinned (see conftest.BRICK_EDGE_STATIONS)."""
    d, golden, time = brick_dir
    m = Mesh(d, N=4, cfl=brick_dt_cfl())
    assert abs(m.dt - 6.46257467e-06) < 1e-15
    pin_brick_edge_stations(m)
    tr = run_oracle(oracle, m, precision=32)[..., 0]
    assert tr.shape == golden.shape
    assert station_misfit(tr, golden) < 2e-4
    assert trace_misfit(tr, golden) < 1e-4
    # first sample: the start value 1e-24 interpolated (src/timeloopMod.f90:184-195)
    assert np.allclose(tr[:, 0, :], golden[:, 0, :], rtol=1e-5, atol=0)


def _cube(tmp_path, cells=2, N=2, nt=40, **kw):
    d = str(tmp_path / f"cube_{cells}_{N}")
    synth.write_cube(d, cells=cells, nt=nt)
    return Mesh(d, N=N, **kw)


def test_fp32_tracks_fp64(tmp_path, oracle):
    m = _cube(tmp_path, cells=3, N=3, nt=200, stf_stage_time=True)
    t64 = run_oracle(oracle, m, 64)
    t32 = run_oracle(oracle, m, 32)
    assert trace_misfit(t32[..., 0], t64[..., 0]) < 1e-4


def test_constant_state_interior_rhs_vanishes(tmp_path, oracle):
    """A constant wavefield has zero volume derivative and zero jumps, so the
    right-hand side vanishes on elements with only interior faces."""
    m = _cube(tmp_path, cells=3, N=3, nt=5)
    ng = m.K * m.Np
    q = np.zeros((ng, 9), order="F")
    q[:] = np.array([1.0, -2.0, 0.5, 0.3, -0.7, 0.2, 1e-3, -2e-3, 5e-4])
    rq = np.zeros_like(q)
    st = oracle.oracle_rhs(m.desc_ptr, 64, 1, 0, q.ctypes.data_as(C.c_void_p), None, None,
                           rq.ctypes.data_as(C.c_void_p), None, None)
    assert st == 0
    nb = m.array("neighbor")
    src = set(m.array("srcelem") - 1)
    interior = [e for e in range(m.K) if (nb[:, e] > 0).all() and e not in src]
    assert interior
    scale = np.abs(q).max() * 4000 / 100.0
    for e in interior:
        assert np.abs(rq[e * m.Np:(e + 1) * m.Np]).max() < 1e-9 * scale


def test_lserk4_fourth_order_in_time(tmp_path, oracle):
    """Halving dt divides the LSERK4 error by ~16 (Carpenter & Kennedy 1994):
    traces at common times of runs with cfl c, c/2, c/4, with the source time
    function sampled at the stage times."""
    runs = []
    for k, cfl in enumerate((0.2, 0.1, 0.05)):
        d = str(tmp_path / f"conv{k}")
        synth.write_cube(d, cells=2, nt=80 * 2 ** k)
        m = Mesh(d, N=3, cfl=cfl, stf_stage_time=True, t0=0.1)
        _, field = run_oracle(oracle, m, 64, want_field=True)
        runs.append(field[..., 0])
    e1 = np.linalg.norm(runs[0] - runs[2])
    e2 = np.linalg.norm(runs[1] - runs[2])
    ratio = e1 / e2
    # e(c)/e(c/2) with the c/4 run as reference: (16-1)/(1-1/16)... ~ 17 for order 4
    assert 10.0 < ratio < 25.0, ratio


def test_batch_members_are_independent(tmp_path, oracle):
    """Two wavefields sharing the mesh, one source each, equal two separate runs."""
    d = str(tmp_path / "b2")
    synth.write_twolayer(d, cells=(4, 4, 2), nt=30, nrec=3, nsrc=2, attenuation=False, pml=False,
                         src_depth=(900.0, 1200.0))
    mb = Mesh(d, N=2, nbatch=2)
    tb = run_oracle(oracle, mb, 64)
    ms = Mesh(d, N=2, nbatch=1)
    ts = run_oracle(oracle, ms, 64)[..., 0]
    # the single run has both sources in one wavefield: linear superposition
    assert rel_l2(tb[..., 0] + tb[..., 1], ts) < 1e-5


def _pml_model(tmp_path, nt=60):
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=nt, nrec=4, attenuation=False, src_depth=(800.0, 800.0))
    return Mesh(d, N=2, stf_stage_time=True)


def test_pml_energy_and_trigger(tmp_path, oracle):
    """The reference's NPML STA/LTA safeguard (src/timeloopMod.f90:508-542):
    the energy is non-negative with the physical compliance, a huge threshold
    never fires (traces unchanged), a tiny one fires right after timecrit and
    switches the NPML off."""
    m = _pml_model(tmp_path)
    base = run_oracle(oracle, m, 64)
    f0 = 10.0  # trigger frequency parameter: timecrit = 2.4/(f0 dt) steps
    timecrit = int(np.float32(2.4 / f0 / m.dt))
    assert timecrit < m.nt - 5
    tr, en, sw = run_oracle_trigger(oracle, m, 64, thr=1e30, f0=f0, formula=1)
    assert sw[0] == 0 and (en[:, 0] >= 0).all() and en[-1, 0] > 0
    assert rel_l2(tr, base) == 0.0
    tr2, en2, sw2 = run_oracle_trigger(oracle, m, 64, thr=1e-9, f0=f0, formula=1)
    assert sw2[0] == timecrit + 1
    assert rel_l2(tr2, base) > 0.0
    # The reference's own strain expression multiplies by 4mu^2+6mu*lambda
    # (src/timeloopMod.f90:493-497); at these amplitudes the FP32 window
    # averages overflow, the ratio is NaN and the trigger never fires.
    tr3, en3, sw3 = run_oracle_trigger(oracle, m, 64, thr=1e-9, f0=f0, formula=0)
    assert sw3[0] == 0 and np.isfinite(en3).all()


@pytest.mark.parametrize("name", ["cube", "twolayer"])
def test_fullrun_fixture_matches_oracle_prefix(tmp_path, oracle, name):
    """The full-run FP64 trace fixtures (tests/golden/fullrun_*.npz) belong to
    the meshes the generator rebuilds: same descriptor fingerprint, and the
    oracle's first 60 steps reproduce the stored traces' first 60 steps."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_fullrun_fixtures as fx
    ref = np.load(os.path.join(GOLDEN, f"fullrun_{name}.npz"))
    m = fx.build(name, str(tmp_path / name))
    assert np.allclose(fx.fingerprint(m), ref["fingerprint"], rtol=1e-12, atol=0)
    tr = run_oracle(oracle, m, 64, steps=60)[..., 0]
    assert np.array_equal(tr[:, :60], ref["traces"][:, :60])


def test_ref_quirks_switch_reports_the_reference_npml(tmp_path, oracle):
    """oracle_set_ref_quirks reproduces what the reference computes on the NPML
    path: bit 1 drives every PML element's auxiliary equation with the last
    element's flux (src/rungekuttaMod.f90:52-63 with the ftemp/gtemp/htemp the
    element loop leaves behind), bit 2 carries the flux columns elasticFluxes
    never writes from element to element (src/waveMod.f90:37-62).  Two-layer
    anelastic model with a 3-cell NPML around a 4 x 4 x 2-cell interior
    (3,000 tets), N=2, the reference's RK2 at CFL 0.15, 400 steps: the
    carried columns change nothing (the auxiliaries of those columns start
    at zero and stay zero), the last-element flux moves the traces by the
    deviation printed here, 4.6e-2 (the correct NPML is the default of the
    oracle and of the GPU path)."""
    oracle.oracle_set_ref_quirks.argtypes = [C.c_int]
    d = str(tmp_path / "q")
    synth.write_twolayer(d, cells=(10, 10, 5), nt=400, nrec=8, src_depth=(700.0, 700.0))
    m = Mesh(d, N=2, timeint=2, cfl=0.15)  # RK2 at N=2 is unstable at CFL 0.3
    assert m.array("pmlcheck").sum() > 0
    base = run_oracle(oracle, m, 64)[..., 0]
    try:
        assert oracle.oracle_set_ref_quirks(2) == 0
        carried = run_oracle(oracle, m, 64)[..., 0]
        assert oracle.oracle_set_ref_quirks(3) == 0
        both = run_oracle(oracle, m, 64)[..., 0]
        assert oracle.oracle_set_ref_quirks(4) == _abi.NEXD_ERR_INVALID
    finally:
        oracle.oracle_set_ref_quirks(0)
    assert np.array_equal(carried, base)
    assert np.isfinite(both).all()
    dev = trace_misfit(both, base)
    print(f"reference NPML (last-element flux) vs correct NPML: trace relative L2 {dev:.3e}")
    assert 1e-3 < dev < 0.5
    assert np.abs(both).max() < 10 * np.abs(base).max()  # a different NPML, not a blow-up
