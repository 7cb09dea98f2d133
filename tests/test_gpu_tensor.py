"""The tensor-core contraction (NEXD_CONTRACT_BF16X3: tcgen05, both operands
split three ways into BF16 parts, six products accumulated in FP32) and the per-class autotune (NEXD_CONTRACT_AUTO) against
the FP64 oracle and against the FP32 CUDA-core path, through the C-ABI.

Tolerances are those of the FP32 path: one right-hand side within 2e-5
relative L2 of the oracle plus the FP32 loss of the Euler difference; receiver
traces after the full run within 1e-4 relative L2 of the FP64 oracle, per
trace kind.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2, run_oracle, trace_misfit
from nexd_b200 import Mesh, NexdError, synth
from nexd_b200 import _abi
from test_gpu_parity import _ptr, _rhs_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Solver():
    from nexd_b200.solver import Solver as S
    return S


@pytest.mark.parametrize("N", [4])
@pytest.mark.parametrize("kind", ["elastic", "anelastic", "pml", "anelastic_pml"])
def test_tc_single_rhs_matches_oracle(tmp_path, oracle, Solver, kind, N):
    """One forward-Euler step from random q, theta and NPML auxiliaries: the
    tensor-core stage's (x1 - x0)/dt equals the oracle's L(x0)."""
    m = _rhs_case(tmp_path, kind, N)
    rng = np.random.default_rng(10 + N)
    ng = m.K * m.Np
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
    s.set_contraction("bf16x3")
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
        tol = 2e-5 + 8 * np.finfo(np.float32).eps * np.linalg.norm(x0) / (m.dt * np.linalg.norm(ref))
        assert err < tol, (kind, N, name, err, tol)


def test_tc_cube_traces(tmp_path, oracle, Solver):
    """Elastic cube (6,000 tets at N=4, LSERK4, 400 steps): tensor-core traces
    within 1e-4 of the FP64 oracle."""
    d = str(tmp_path / "cube")
    synth.write_cube(d, nt=400)
    m = Mesh(d, N=4, stf_stage_time=True)
    s = Solver(m.desc_ptr)
    s.set_contraction("bf16x3")
    s.run(1, 400)
    to = run_oracle(oracle, m, 64)[..., 0]
    assert np.abs(to).max() > 1e-12
    assert trace_misfit(s.traces()[..., 0], to) < 1e-4


def test_tc_twolayer_anelastic_pml_traces(tmp_path, oracle, Solver):
    """Two-layer Zener + NPML model (N=4, 3,000 tets, LSERK4, 150 steps):
    tensor-core traces and final wavefield within 1e-4 of the FP64 oracle."""
    d = str(tmp_path / "tl")
    synth.write_twolayer(d, cells=(10, 10, 5), nt=150, nrec=12, src_depth=(900.0, 900.0))
    m = Mesh(d, N=4, stf_stage_time=True)
    s = Solver(m.desc_ptr)
    s.set_contraction("bf16x3")
    s.run(1, 150)
    to, fo = run_oracle(oracle, m, 64, want_field=True)
    assert trace_misfit(s.traces()[..., 0], to[..., 0]) < 1e-4
    assert rel_l2(s.field(), fo[..., 0]) < 1e-4


@pytest.mark.parametrize("timeint", [2, 3])
def test_tc_reference_integrators(tmp_path, oracle, Solver, timeint):
    """TVD RK2 / RK3 stage updates with the tensor-core contraction."""
    d = str(tmp_path / f"ti{timeint}")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=60, nrec=5, src_depth=(800.0, 800.0))
    m = Mesh(d, N=4, timeint=timeint, cfl=0.3)
    s = Solver(m.desc_ptr)
    s.set_contraction("bf16x3")
    s.run(1, 60)
    assert trace_misfit(s.traces()[..., 0], run_oracle(oracle, m, 64)[..., 0]) < 1e-4


def test_tc_batched_and_switching(tmp_path, Solver):
    """Batched wavefields on the tensor cores equal single-wavefield runs of
    the same path; switching the contraction mid-run keeps the state."""
    d = str(tmp_path / "b")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=60, nrec=4, nsrc=2, src_depth=(700.0, 1200.0))
    mb = Mesh(d, N=4, nbatch=2, stf_stage_time=True)
    sb = Solver(mb.desc_ptr)
    sb.set_contraction("bf16x3")
    sb.run(1, 60)
    tb = sb.traces()
    for b in range(2):
        ms = Mesh(d, N=4, nbatch=2, stf_stage_time=True)
        stf = ms.array("stf")
        stf[:, :, 1 - b] = 0.0
        ss = Solver(ms.desc_ptr)
        ss.set_contraction("bf16x3")
        ss.run(1, 30)
        ss.set_contraction("fp32")
        ss.set_contraction("bf16x3")
        ss.run(31, 60)
        assert rel_l2(tb[..., b], ss.traces()[..., b]) < 1e-6
    # the two contractions agree to the split-product accuracy
    sf = Solver(mb.desc_ptr)
    sf.run(1, 60)
    assert trace_misfit(sf.traces()[..., 0], tb[..., 0]) < 1e-4


def test_tc_contraction_errors(tmp_path, Solver):
    d = str(tmp_path / "c")
    synth.write_cube(d, cells=3, nt=4)
    m = Mesh(d, N=3)  # keeps the descriptor's arrays alive while the solver is created
    s = Solver(m.desc_ptr)
    with pytest.raises(NexdError) as ei:
        s.set_contraction("bf16x3")
    assert ei.value.status == _abi.NEXD_ERR_UNSUPPORTED
    with pytest.raises(NexdError) as ei:
        s.set_contraction(7)
    assert ei.value.status == _abi.NEXD_ERR_INVALID
    s.run(1, 4)  # still runs on the FP32 path


@pytest.mark.parametrize("timeint", [4, 2])
def test_autotune_leaves_state_and_picks_valid_kinds(tmp_path, oracle, Solver, timeint):
    """The autotune's timing launches at a step boundary leave the wavefield,
    memory variables and NPML auxiliaries bit-identical; the run continues on
    the chosen kernels within the FP32 tolerance of the oracle."""
    d = str(tmp_path / "auto")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=60, nrec=6, src_depth=(900.0, 900.0))
    m = Mesh(d, N=4, timeint=timeint, stf_stage_time=(timeint == 4), cfl=0.3)
    s = Solver(m.desc_ptr)
    s.run(1, 30)
    nth = 6 * m.desc.nMB
    before = (s.field(), s.state(_abi.NEXD_STATE_THETA, nfields=nth), s.state(_abi.NEXD_STATE_PML, nfields=27))
    s.set_contraction("auto")
    after = (s.field(), s.state(_abi.NEXD_STATE_THETA, nfields=nth), s.state(_abi.NEXD_STATE_PML, nfields=27))
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    kinds, ms = s.contraction()
    assert set(kinds.values()) <= {"fp32", "bf16x3", "fp32_pairs", "fp32_bulk"}
    assert kinds["npml"] != "fp32_pairs"
    # every candidate of each class was timed, the chosen one is the fastest
    for cl, cands in (("npml", ("fp32", "bf16x3", "fp32_bulk")), ("rest", ("fp32", "bf16x3", "fp32_pairs", "fp32_bulk"))):
        assert all(ms[(cl, k)] > 0 for k in cands)
        assert ms[(cl, kinds[cl])] == min(ms[(cl, k)] for k in cands)
    s.run(31, 60)
    assert trace_misfit(s.traces()[..., 0], run_oracle(oracle, m, 64)[..., 0]) < 1e-4


@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_node_pair_kernel_is_bit_identical(tmp_path, Solver, N):
    """The node-pair FP32 kernel (elements outside the NPML) performs the
    FP32 kernel's operations in the same order: identical wavefields, memory
    variables and traces; AUTO may choose it."""
    d = str(tmp_path / "pair")
    synth.write_twolayer(d, cells=(10, 10, 5), nt=12, nrec=4, src_depth=(900.0, 900.0))
    m = Mesh(d, N=N, stf_stage_time=True)
    a, b = Solver(m.desc_ptr), Solver(m.desc_ptr)
    b.set_contraction("fp32_pairs")
    assert b.contraction()[0] == {"npml": "fp32", "rest": "fp32_pairs"}
    a.run(1, 12)
    b.run(1, 12)
    assert np.array_equal(a.field(), b.field())
    nth = 6 * m.desc.nMB
    assert np.array_equal(a.state(_abi.NEXD_STATE_THETA, nfields=nth), b.state(_abi.NEXD_STATE_THETA, nfields=nth))
    assert np.array_equal(a.traces(), b.traces())
    c = Solver(m.desc_ptr)
    c.set_contraction("auto")
    kinds, ms = c.contraction()
    assert ms[("rest", "fp32_pairs")] > 0 and ms[("rest", "fp32")] > 0


def test_pinned_kernel_kinds(tmp_path, oracle, Solver):
    """nexd_set_contraction_kinds pins the kernel per element class without
    timing: the pinned FP32 / node-pair pair is bit-identical to the FP32
    path, the tensor-core NPML kernel stays within the FP32 tolerance of the
    oracle, and kinds the class or order lacks are refused."""
    d = str(tmp_path / "pin")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=40, nrec=6, src_depth=(900.0, 900.0))
    m = Mesh(d, N=4, stf_stage_time=True)
    ref = Solver(m.desc_ptr)
    ref.run(1, 40)
    a = Solver(m.desc_ptr)
    a.set_contraction_kinds("fp32", "fp32_pairs")
    assert a.contraction()[0] == {"npml": "fp32", "rest": "fp32_pairs"}
    a.run(1, 40)
    assert np.array_equal(a.traces(), ref.traces())
    b = Solver(m.desc_ptr)
    b.set_contraction_kinds("bf16x3", "fp32")
    assert b.contraction()[0] == {"npml": "bf16x3", "rest": "fp32"}
    b.run(1, 40)
    assert trace_misfit(b.traces()[..., 0], run_oracle(oracle, m, 64)[..., 0]) < 1e-4
    with pytest.raises(NexdError) as ei:
        b.set_contraction_kinds("fp32_pairs", "fp32")  # no node-pair kernel for NPML elements
    assert ei.value.status == _abi.NEXD_ERR_INVALID
    assert b.contraction()[0] == {"npml": "bf16x3", "rest": "fp32"}  # unchanged
    d3 = str(tmp_path / "n3")
    synth.write_cube(d3, cells=3, nt=4)
    m3 = Mesh(d3, N=3)
    s3 = Solver(m3.desc_ptr)
    with pytest.raises(NexdError) as ei:
        s3.set_contraction_kinds("fp32", "bf16x3")
    assert ei.value.status == _abi.NEXD_ERR_UNSUPPORTED
    s3.run(1, 4)


@pytest.mark.parametrize("N,att,timeint", [(3, False, 4), (3, True, 4), (4, True, 4), (4, False, 4), (4, True, 2),
                                          (4, True, 3), (2, True, 4), (5, True, 4)])
def test_bulk_kernels_are_bit_identical(tmp_path, oracle, Solver, N, att, timeint):
    """The stage kernels whose element-local state moves by bulk copies (NPML
    elements: NPML auxiliaries, their residuals, damping profiles, residual of
    q and memory variables, orders 3 and 4; the other elements of anelastic
    models: memory variables, orders 2-5) perform the FP32 kernels'
    operations in the same order: identical wavefields, memory variables,
    NPML auxiliaries and traces under LSERK4 and the reference's RK2 and RK3,
    over several chunks per block and partial chunks; their traces agree with
    the FP64 oracle within the FP32 tolerance; AUTO times them."""
    d = str(tmp_path / "bulk")
    nt = 40
    synth.write_twolayer(d, cells=(10, 10, 5), nt=nt, nrec=6, src_depth=(900.0, 900.0), attenuation=att)
    m = Mesh(d, N=N, stf_stage_time=(timeint == 4), timeint=timeint, cfl=0.3 if timeint == 4 else 0.1)
    assert m.array("pmlcheck").sum() > 0
    kinds = ("fp32_bulk" if N in (3, 4) else "fp32", "fp32_bulk" if att else "fp32")
    a, b = Solver(m.desc_ptr), Solver(m.desc_ptr)
    a.set_contraction_kinds("fp32", "fp32")
    b.set_contraction_kinds(*kinds)
    assert b.contraction()[0] == {"npml": kinds[0], "rest": kinds[1]}
    a.run(1, nt)
    b.run(1, nt)
    assert np.array_equal(a.field(), b.field())
    if att:
        nth = 6 * m.desc.nMB
        assert np.array_equal(a.state(_abi.NEXD_STATE_THETA, nfields=nth), b.state(_abi.NEXD_STATE_THETA, nfields=nth))
    assert np.array_equal(a.state(_abi.NEXD_STATE_PML, nfields=27), b.state(_abi.NEXD_STATE_PML, nfields=27))
    assert np.array_equal(a.traces(), b.traces())
    assert trace_misfit(b.traces()[..., 0], run_oracle(oracle, m, 64)[..., 0]) < 1e-4
    if N == 4 and timeint == 4:
        c = Solver(m.desc_ptr)
        c.set_contraction("auto")
        kinds, ms = c.contraction()
        assert ms[("npml", "fp32_bulk")] > 0 and ms[("npml", "fp32")] > 0
        assert kinds["npml"] in ("fp32", "bf16x3", "fp32_bulk")
        if att:
            assert ms[("rest", "fp32_bulk")] > 0


@pytest.mark.parametrize("N,att", [(2, True), (5, True), (4, False)])
def test_bulk_kernels_refused_where_they_do_not_apply(tmp_path, Solver, N, att):
    """Orders 2 and 5 need more shared memory than a block can have for the
    bulk-copy NPML kernel, and elastic models have no memory variables for
    the other bulk-copy kernel: pinning them is refused, the FP32 kernels
    stay."""
    d = str(tmp_path / "nofit")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=4, nrec=2, src_depth=(900.0, 900.0), attenuation=att)
    m = Mesh(d, N=N)
    s = Solver(m.desc_ptr)
    with pytest.raises(NexdError) as ei:
        s.set_contraction_kinds("fp32_bulk", "fp32") if N != 4 else s.set_contraction_kinds("fp32", "fp32_bulk")
    assert ei.value.status == _abi.NEXD_ERR_UNSUPPORTED
    assert s.contraction()[0] == {"npml": "fp32", "rest": "fp32"}
    s.run(1, 4)
