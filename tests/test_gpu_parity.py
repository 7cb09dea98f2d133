"""GPU (libnexd.so, sm_100a, FP32) against the CPU oracle (FP64) and against
the reference's golden seismograms, through the C-ABI.

Tolerances: receiver traces within 1e-4 relative L2 of the FP64 oracle, per
trace kind (u, v, a) over all receivers; final wavefields within 1e-4; one
right-hand side within 2e-5 plus the FP32 loss of the Euler difference; the
reference's golden brick traces within 1e-4 overall and 2e-4 per station (the
reference ran in FP32 with FP32 operators).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import (brick_dt_cfl, pin_brick_edge_stations, rel_l2, run_oracle, run_oracle_trigger, trace_misfit,
                      station_misfit, write_brick)
from nexd_b200 import Mesh, NexdError, synth
from nexd_b200 import _abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Solver():
    from nexd_b200.solver import Solver as S
    return S


def _rhs_case(tmp_path, kind, N):
    d = str(tmp_path / f"{kind}{N}")
    if kind == "elastic":
        synth.write_cube(d, cells=3, nt=4)
    else:
        synth.write_twolayer(d, cells=(6, 6, 3), nt=4, nrec=4, attenuation=(kind != "pml"),
                             pml=(kind != "anelastic"))
    return Mesh(d, N=N, timeint=1)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("kind", ["elastic", "anelastic", "pml", "anelastic_pml"])
def test_single_rhs_matches_oracle(tmp_path, oracle, Solver, kind, N):
    """One forward-Euler step from random q, theta and NPML auxiliaries
    isolates one right-hand side of every updated field: (x1 - x0)/dt on the
    GPU equals the oracle's L(x0) for q, theta and F',G',H'."""
    m = _rhs_case(tmp_path, kind, N)
    rng = np.random.default_rng(N)
    ng = m.K * m.Np
    # velocity ~1, stress ~ impedance * velocity, so dt*L(q) ~ q in both blocks
    qs = np.array([1.2e7] * 6 + [1.0] * 3)
    q0 = np.asfortranarray((rng.standard_normal((ng, 9)) * qs).astype(np.float32))
    att, pml = m.desc.attenuation == 1, m.desc.set_pml == 1
    nth = 6 * m.desc.nMB
    th0 = np.asfortranarray((rng.standard_normal((ng, nth)) * 1e-4).astype(np.float32)) if att else None
    aux0 = None
    if pml:
        fs = np.array([3e10] * 6 + [4e3] * 3)
        aux0 = np.asfortranarray((rng.standard_normal((ng, 27)) * np.tile(fs, 3)).astype(np.float32))
        aux0[np.repeat(m.array("pmlcheck") == 0, m.Np)] = 0.0
    s = Solver(m.desc_ptr)
    s.set_field(q0)
    if att:
        s.set_state(th0, _abi.NEXD_STATE_THETA)
    if pml:
        s.set_state(aux0, _abi.NEXD_STATE_PML)
    s.run(1, 1)
    dt = np.float32(m.dt)
    rq = np.zeros((ng, 9), order="F")
    arq = np.zeros((ng, nth), order="F") if att else None
    auxr = np.zeros((ng, 27), order="F") if pml else None
    f64 = lambda a: None if a is None else np.asfortranarray(a.astype(np.float64))
    assert oracle.oracle_rhs(m.desc_ptr, 64, 1, 0, _ptr(f64(q0)), _ptr(f64(th0)), _ptr(f64(aux0)), _ptr(rq),
                             _ptr(arq), _ptr(auxr)) == 0
    checks = [("q", q0, s.field(), rq)]
    if att:
        checks.append(("theta", th0, s.state(_abi.NEXD_STATE_THETA, nfields=nth), arq))
    if pml:
        checks.append(("aux", aux0, s.state(_abi.NEXD_STATE_PML, nfields=27), auxr))
    for name, x0, x1, ref in checks:
        got = (x1.astype(np.float64) - x0.astype(np.float64)) / dt
        err = rel_l2(got, ref)
        # FP32 rounding of the Euler difference: |x0| / (dt |L x0|) digits are lost
        tol = 2e-5 + 8 * np.finfo(np.float32).eps * np.linalg.norm(x0) / (m.dt * np.linalg.norm(ref))
        assert err < tol, (kind, N, name, err, tol)


def test_cube_lserk4_traces(tmp_path, oracle, Solver):
    """Homogeneous 2 km cube, 6,000 tets, N=3, LSERK4: 400 steps (through the
    first P and S arrivals at the surface receivers), FP32 GPU vs FP64 oracle."""
    d = str(tmp_path / "cube")
    synth.write_cube(d, nt=400)
    m = Mesh(d, N=3, stf_stage_time=True)
    s = Solver(m.desc_ptr)
    s.run(1, 200)
    s.run(201, 400)
    tg = s.traces()[..., 0]
    to = run_oracle(oracle, m, 64)[..., 0]
    assert np.abs(to).max() > 1e-12  # the wave reached the receivers
    assert trace_misfit(tg, to) < 1e-4


def test_twolayer_anelastic_pml_traces(tmp_path, oracle, Solver):
    """Two-layer Zener + NPML model (N=4, 10x10x5 cells = 3,000 tets), LSERK4,
    moment-tensor source: 150 steps, FP32 GPU vs FP64 oracle."""
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(10, 10, 5), nt=150, nrec=12, src_depth=(900.0, 900.0))
    m = Mesh(d, N=4, stf_stage_time=True)
    assert m.array("pmlcheck").sum() > 0 and m.desc.attenuation == 1
    s = Solver(m.desc_ptr)
    s.run(1, 150)
    tg = s.traces()[..., 0]
    tg_f = s.field()
    to, fo = run_oracle(oracle, m, 64, want_field=True)
    assert trace_misfit(tg, to[..., 0]) < 1e-4
    assert rel_l2(tg_f, fo[..., 0]) < 1e-4


@pytest.mark.parametrize("timeint", [1, 2, 3])
def test_reference_integrators(tmp_path, oracle, Solver, timeint):
    """The reference's Euler / TVD-RK2 / TVD-RK3 stage updates
    (src/rungekuttaMod.f90:27-120) on the GPU vs the oracle."""
    d = str(tmp_path / f"ti{timeint}")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=60, nrec=5, src_depth=(800.0, 800.0))
    m = Mesh(d, N=3, timeint=timeint, cfl=0.1 if timeint == 1 else 0.3)
    s = Solver(m.desc_ptr)
    s.run(1, 60)
    assert trace_misfit(s.traces()[..., 0], run_oracle(oracle, m, 64)[..., 0]) < 1e-4


def test_brick_golden_on_gpu(tmp_path, Solver):
    """The reference's own brick example (9,859 tets, N=4, RK2, 1000 steps) on
    the GPU reproduces its golden seismograms within 2e-4 relative L2."""
    golden, _ = write_brick(str(tmp_path))
    m = Mesh(str(tmp_path), N=4, cfl=brick_dt_cfl())
    pin_brick_edge_stations(m)
    s = Solver(m.desc_ptr)
    s.run(1, 1000)
    tr = s.traces()[..., 0]
    assert station_misfit(tr, golden) < 2e-4
    assert trace_misfit(tr, golden) < 1e-4


def test_brick_golden_from_database_files_on_gpu(tmp_path, Solver):
    """The brick example handed over as the reference's database files
    (meshVar000001, srcVar000001, recVar000001: REAL(4) records, read as
    timeloop3D's readMesh / readSrc / readRec do) reproduces the golden
    seismograms on the GPU within the same bounds."""
    golden, _ = write_brick(str(tmp_path))
    Mesh(str(tmp_path), N=4).write_database(str(tmp_path / "out"))
    # the reference's dt = 6.46257467e-06 from the REAL(4) dtfactor of the file
    dtf = Mesh(str(tmp_path), database=True).info.dtfactor
    m = Mesh(str(tmp_path), database=True, cfl=6.46257467e-06 / dtf)
    assert m.N == 4 and abs(m.dt - 6.46257467e-06) < 1e-14
    pin_brick_edge_stations(m)
    s = Solver(m.desc_ptr)
    s.run(1, 1000)
    tr = s.traces()[..., 0]
    assert station_misfit(tr, golden) < 2e-4
    assert trace_misfit(tr, golden) < 1e-4


def test_batched_wavefields(tmp_path, Solver):
    """nbatch independent wavefields in one launch equal separate runs."""
    d = str(tmp_path / "b")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=80, nrec=4, nsrc=3, src_depth=(700.0, 1200.0))
    mb = Mesh(d, N=3, nbatch=3, stf_stage_time=True)
    sb = Solver(mb.desc_ptr)
    sb.run(1, 80)
    tb = sb.traces()
    for b in range(3):
        ms = Mesh(d, N=3, nbatch=3, stf_stage_time=True)
        # keep only source b: move the others to a wavefield that is not compared
        srcb = ms.array("srcbatch")
        stf = ms.array("stf")
        for i in range(3):
            if i != b:
                stf[:, :, i] = 0.0
        ss = Solver(ms.desc_ptr)
        ss.run(1, 80)
        ts = ss.traces()
        assert rel_l2(tb[..., b], ts[..., b]) < 1e-6
        assert srcb[b] == b


def test_step_range_and_nonfinite_errors(tmp_path, Solver):
    d = str(tmp_path / "e")
    synth.write_cube(d, cells=2, nt=5)
    m = Mesh(d, N=2)
    s = Solver(m.desc_ptr)
    with pytest.raises(NexdError) as ei:
        s.run(1, 6)
    assert ei.value.status == _abi.NEXD_ERR_INVALID
    q = s.field()
    q[:, 6] = np.nan
    s.set_field(q)
    with pytest.raises(NexdError) as ei:
        s.run(1, 2)
    assert ei.value.status == _abi.NEXD_ERR_NONFINITE


@pytest.mark.parametrize("formula", [0, 1])
def test_pml_energy_trigger_matches_oracle(tmp_path, oracle, Solver, formula):
    """Device energy reduction and STA/LTA trigger vs the oracle: energy history
    within 1e-5, the same switch-off step, and matching traces afterwards."""
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=80, nrec=4, src_depth=(800.0, 800.0))
    m = Mesh(d, N=3, stf_stage_time=True)
    f0 = 10.0  # trigger frequency parameter: timecrit = 2.4/(f0 dt) = 34 steps here
    for thr in (1e30, 1e-3):
        s = Solver(m.desc_ptr)
        s.pml_trigger(10, 2, thr, f0, formula)
        s.run(1, 80)
        eg, swg = s.energy()
        tg = s.traces()
        to, eo, swo = run_oracle_trigger(oracle, m, 64, thr=thr, f0=f0, formula=formula)
        assert rel_l2(eg, eo) < 1e-5
        assert swg[0] == swo[0]
        assert trace_misfit(tg[..., 0], to[..., 0]) < 1e-4
        if thr < 1 and formula == 1:
            assert swg[0] > 0


def test_graph_replay_matches_direct_launches(tmp_path, Solver):
    """nexd_run replays captured two-step CUDA graphs (steps counted on the
    device); with per-launch timing on it launches one kernel at a time.  Both
    orders of the same kernels give bit-identical wavefields, memory variables,
    NPML auxiliaries and traces, including odd step counts and restarts."""
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=30, nrec=4, src_depth=(800.0, 800.0))
    m = Mesh(d, N=3, stf_stage_time=True)
    a, b = Solver(m.desc_ptr), Solver(m.desc_ptr)
    b.profile(True)
    for lo, hi in ((1, 7), (8, 8), (9, 20), (21, 30)):
        a.run(lo, hi)
        b.run(lo, hi)
    p = b.profile()
    assert p["stage_main"]["launches"] == p["stage_pml"]["launches"] == 5 * 30
    assert np.array_equal(a.field(), b.field())
    nth = 6 * m.desc.nMB
    assert np.array_equal(a.state(_abi.NEXD_STATE_THETA, nfields=nth), b.state(_abi.NEXD_STATE_THETA, nfields=nth))
    assert np.array_equal(a.state(_abi.NEXD_STATE_PML, nfields=27), b.state(_abi.NEXD_STATE_PML, nfields=27))
    assert np.array_equal(a.traces(), b.traces())
    assert a.launch_count() == b.launch_count()
