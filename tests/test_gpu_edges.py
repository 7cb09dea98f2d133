"""Edge cases of the stage path on the GPU against the FP64 oracle, through
the C-ABI:

* one hexahedron (6 tets): a single partial chunk, every face on the free or
  absorbing boundary;
* a two-layer anelastic box so small that every element is an NPML element,
  so the other element class is empty;
* the same box with no receivers.

The reference runs all of them: its element loop walks whatever elements the
mesh holds (src/timeloopMod.f90:395-476), and a station file may list none.
The wavefield after the run agrees with the oracle's within 1e-4 relative L2,
the FP32 tolerance of the full runs. The traces agree within 1e-4 per trace
kind. Every FP32 kernel kind that applies gives the same bits, and the
per-class autotune runs with an empty class.
"""
import numpy as np
import pytest

from conftest import rel_l2, run_oracle, trace_misfit
from nexd_b200 import Mesh, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Solver():
    from nexd_b200.solver import Solver as S
    return S


def _check(oracle, Solver, m, kinds):
    """Runs the mesh once per kernel kind ("auto" or an (npml, rest) pair) and
    compares each run with the oracle; the pinned FP32 kinds with one another."""
    to, fo = run_oracle(oracle, m, 64, want_field=True)
    assert np.abs(fo).max() > 0
    first = None
    for k in kinds:
        s = Solver(m.desc_ptr)
        try:
            if k == "auto":
                s.set_contraction("auto")
            else:
                s.set_contraction_kinds(*k)
            s.run(1, m.nt)
            f, tr = s.field(), s.traces()
        finally:
            s.close()
        assert np.all(np.isfinite(f)), k
        assert rel_l2(f, fo[..., 0]) < 1e-4, k
        assert tr.shape == (m.nrec, m.nt, 9, 1)
        if m.nrec:
            assert trace_misfit(tr[..., 0], to[..., 0]) < 1e-4, k
        if k == "auto":
            continue
        if first is None:
            first = (f, tr)
        else:
            assert np.array_equal(f, first[0]) and np.array_equal(tr, first[1]), k


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
def test_single_hexahedron(tmp_path, oracle, Solver, N):
    """Six elastic tets in one chunk (fewer than a chunk holds at every order),
    free top and absorbing sides on every element."""
    d = str(tmp_path / "hex")
    synth.write_cube(d, cells=1, nt=40)
    m = Mesh(d, N=N)
    assert m.K == 6
    kinds = [("fp32", "fp32")] + ([("fp32", "fp32_pairs")] if N >= 2 else []) + ["auto"]
    _check(oracle, Solver, m, kinds)


@pytest.mark.parametrize("N", [2, 3, 4, 5])
@pytest.mark.parametrize("nrec", [3, 0])
def test_every_element_in_the_npml(tmp_path, oracle, Solver, N, nrec):
    """5 x 5 x 2 cells with the 3-cell NPML: all 300 tets are NPML elements
    and the class of the other elements is empty, with and without receivers.
    The source sits inside a cell: on a cell edge the reference's source
    search gives up after 20 elements around the nearest node."""
    d = str(tmp_path / f"allpml{nrec}")
    synth.write_twolayer(d, cells=(5, 5, 2), nt=40, nrec=nrec, src_depth=(900.0, 900.0))
    m = Mesh(d, N=N)
    assert m.K == 300 and m.array("pmlcheck").min() == 1 and m.nrec == nrec
    kinds = [("fp32", "fp32"), ("fp32", "fp32_bulk")]
    if N in (3, 4):
        kinds.append(("fp32_bulk", "fp32_bulk"))
    kinds.append("auto")
    _check(oracle, Solver, m, kinds)
