"""Several models in one CUDA graph (nexd_group_*): a group run is
bit-identical to running its members one by one, for members of different
orders (2 to 5), sizes, rheologies and contractions (FP32, node-pair FP32,
split-BF16 tcgen05), over step pairs and a leftover step; every member's
traces agree with the FP64 oracle; the grid autotune leaves the live state
unchanged."""
import numpy as np
import pytest

from conftest import rel_l2, run_oracle, trace_misfit
from nexd_b200 import Mesh, synth
from nexd_b200 import _abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver_mod():
    from nexd_b200 import solver
    return solver


def _models(tmp_path):
    out = []
    d = str(tmp_path / "cube2")
    synth.write_cube(d, cells=4, nt=30)
    out.append((Mesh(d, N=2, stf_stage_time=True), "fp32"))
    d = str(tmp_path / "tl3")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=30, nrec=4, src_depth=(900.0, 900.0))
    out.append((Mesh(d, N=3, stf_stage_time=True), "fp32"))
    d = str(tmp_path / "tl4")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=30, nrec=4, src_depth=(900.0, 900.0), attenuation=False,
                         src_seed=7)
    out.append((Mesh(d, N=4, stf_stage_time=True), "bf16x3"))
    d = str(tmp_path / "cube2p")
    synth.write_cube(d, cells=4, nt=30, seed=3)
    out.append((Mesh(d, N=2, stf_stage_time=True), "fp32_pairs"))
    d = str(tmp_path / "tl5")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=30, nrec=4, src_depth=(900.0, 900.0), pml=False, src_seed=9)
    out.append((Mesh(d, N=5, stf_stage_time=True), "fp32"))
    d = str(tmp_path / "tl5p")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=30, nrec=4, src_depth=(900.0, 900.0), src_seed=11)
    out.append((Mesh(d, N=5, stf_stage_time=True), "fp32_pairs"))
    return out


def test_group_run_equals_member_runs(tmp_path, solver_mod):
    models = _models(tmp_path)
    alone = []
    for m, c in models:
        s = solver_mod.Solver(m.desc_ptr)
        s.set_contraction(c)
        s.run(1, 13)
        alone.append((s.field(), s.traces()))
    members = []
    for m, c in models:
        s = solver_mod.Solver(m.desc_ptr)
        s.set_contraction(c)
        members.append(s)
    g = solver_mod.Group(members)
    g.run(1, 6)       # three graph replays
    g.run(7, 13)      # three replays and a leftover step
    assert g.span_ms() > 0
    for s, (f, t) in zip(members, alone):
        assert np.array_equal(s.field(), f)
        assert np.array_equal(s.traces(), t)
    g.close()


def test_group_members_match_oracle(tmp_path, solver_mod, oracle):
    """Each member of a group (orders 2 to 5, every contraction) run for 30
    steps in the group against its own FP64 oracle run: the final wavefield
    within 1e-4 relative L2 (the receivers may not have recorded the wave yet
    after 30 steps, so the traces are compared only where they have)."""
    models = _models(tmp_path)
    members = []
    for m, c in models:
        s = solver_mod.Solver(m.desc_ptr)
        s.set_contraction(c)
        members.append(s)
    g = solver_mod.Group(members)
    g.run(1, 30)
    for (m, c), s in zip(models, members):
        to, fo = run_oracle(oracle, m, 64, want_field=True)
        assert rel_l2(s.field(), fo[..., 0]) < 1e-4, (m.N, c)
        if np.abs(to[:, :, 3:6]).max() > 1e-6 * np.abs(fo[:, 6:9]).max():
            assert trace_misfit(s.traces()[..., 0], to[..., 0]) < 1e-4, (m.N, c)
    g.close()


def test_group_autotune_keeps_state(tmp_path, solver_mod):
    models = _models(tmp_path)
    members = [solver_mod.Solver(m.desc_ptr) for m, _ in models]
    g = solver_mod.Group(members)
    g.run(1, 4)
    before = [s.field() for s in members]
    div = g.autotune()
    assert div in (1, 2, 4)
    for s, f in zip(members, before):
        assert np.array_equal(s.field(), f)
    g.run(5, 8)
    ref = [solver_mod.Solver(m.desc_ptr) for m, _ in models]
    for r in ref:
        r.run(1, 8)
    for s, r in zip(members, ref):
        assert np.array_equal(s.field(), r.field())


def test_group_errors(tmp_path, solver_mod):
    models = _models(tmp_path)
    a = solver_mod.Solver(models[0][0].desc_ptr)
    with pytest.raises(Exception):
        solver_mod.Group([a, a])
    g = solver_mod.Group([a])
    with pytest.raises(Exception):
        g.run(1, 31)  # beyond nt
    g.run(1, 2)


def _no_pml_models(tmp_path):
    """Members the single persistent launch covers: orders 2 to 5, elastic and
    anelastic, no NPML, of different sizes."""
    out = []
    d = str(tmp_path / "pc2")
    synth.write_cube(d, cells=4, nt=30)
    out.append(Mesh(d, N=2, stf_stage_time=True))
    d = str(tmp_path / "pt3")
    synth.write_twolayer(d, cells=(8, 8, 4), nt=30, nrec=4, src_depth=(900.0, 900.0), pml=False)
    out.append(Mesh(d, N=3, stf_stage_time=True))
    d = str(tmp_path / "pt4")
    synth.write_twolayer(d, cells=(10, 10, 5), nt=30, nrec=4, src_depth=(900.0, 900.0), pml=False,
                         attenuation=False, src_seed=5)
    out.append(Mesh(d, N=4, stf_stage_time=True))
    d = str(tmp_path / "pt5")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=30, nrec=4, src_depth=(900.0, 900.0), pml=False, src_seed=9)
    out.append(Mesh(d, N=5, stf_stage_time=True))
    return out


def test_group_single_persistent_launch_equals_member_runs(tmp_path, solver_mod):
    """Mode 1: every stage of all members is one launch of the multi-model
    kernel (blocks shared out over the members' work items).  Fields, memory
    variables and traces are bit-identical to each member run on its own,
    over graph-replayed step pairs and a leftover step; a group with an NPML
    member cannot use the mode."""
    meshes = _no_pml_models(tmp_path)
    alone = []
    for m in meshes:
        s = solver_mod.Solver(m.desc_ptr)
        s.run(1, 13)
        alone.append((s.field(), s.traces()))
        s.close()
    members = [solver_mod.Solver(m.desc_ptr) for m in meshes]
    g = solver_mod.Group(members)
    g.set_mode(1)
    mode, blocks, _ = g.mode()
    assert mode == 1 and all(b >= 1 for b in blocks)
    l0 = sum(s.launch_count() for s in members)
    g.run(1, 6)
    g.run(7, 13)
    # 13 steps x 5 stages: one launch per stage for the whole group
    per_step_small = sum(1 + (1 if m.nrec > 0 else 0) for m in meshes)  # tick + record per member
    assert sum(s.launch_count() for s in members) - l0 == 13 * (5 + per_step_small)
    for s, (f, t) in zip(members, alone):
        assert np.array_equal(s.field(), f)
        assert np.array_equal(s.traces(), t)
    g.close()
    d = str(tmp_path / "withpml")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=10, nrec=2, src_depth=(800.0, 800.0))
    mp = Mesh(d, N=3, stf_stage_time=True)
    h = solver_mod.Group([solver_mod.Solver(mp.desc_ptr)])
    with pytest.raises(Exception):
        h.set_mode(1)


def test_group_autotune_chooses_between_modes(tmp_path, solver_mod, oracle):
    """The group autotune times the per-member branches (grid divisors 1, 2,
    4) and the single persistent launch, keeps the faster, and the run goes on
    bit-identically to the members run alone and within the FP32 tolerance
    of the oracle."""
    meshes = _no_pml_models(tmp_path)
    members = [solver_mod.Solver(m.desc_ptr) for m in meshes]
    g = solver_mod.Group(members)
    g.run(1, 4)
    g.autotune()
    mode, blocks, ms = g.mode()
    assert mode in (0, 1) and ms["branches"] > 0 and ms["persistent"] > 0
    assert (mode == 1) == (ms["persistent"] < ms["branches"])
    g.run(5, 30)
    for m, s in zip(meshes, members):
        r = solver_mod.Solver(m.desc_ptr)
        r.run(1, 30)
        assert np.array_equal(s.field(), r.field())
        to, fo = run_oracle(oracle, m, 64, want_field=True)
        assert rel_l2(s.field(), fo[..., 0]) < 1e-4
    g.close()


def test_group_with_bulk_copy_kernels_equals_member_runs(tmp_path, solver_mod):
    """Members on the bulk-copy stage kernels (an NPML model at N=4 with both
    element classes pinned to them; an anelastic model at N=3 without NPML,
    its elements on the bulk-copy kernel of the rest) stepped together as
    graph branches give their own runs bit for bit."""
    d1 = str(tmp_path / "npml4")
    synth.write_twolayer(d1, cells=(8, 8, 4), nt=30, nrec=4, src_depth=(900.0, 900.0))
    d2 = str(tmp_path / "tl3")
    synth.write_twolayer(d2, cells=(6, 6, 3), nt=30, nrec=4, src_depth=(900.0, 900.0), pml=False, src_seed=5)
    specs = [(Mesh(d1, N=4, stf_stage_time=True), ("fp32_bulk", "fp32_bulk")),
             (Mesh(d2, N=3, stf_stage_time=True), ("fp32", "fp32_bulk"))]
    alone = []
    for m, kinds in specs:
        s = solver_mod.Solver(m.desc_ptr)
        s.set_contraction_kinds(*kinds)
        s.run(1, 13)
        alone.append((s.field(), s.traces()))
        s.close()
    members = []
    for m, kinds in specs:
        s = solver_mod.Solver(m.desc_ptr)
        s.set_contraction_kinds(*kinds)
        members.append(s)
    g = solver_mod.Group(members)
    g.run(1, 6)
    g.run(7, 13)
    for s, (f, t) in zip(members, alone):
        assert np.array_equal(s.field(), f)
        assert np.array_equal(s.traces(), t)
    g.close()
