"""Size-independent checks at the benchmark's full size, through the C-ABI:
the two-layer anelastic model with the 3-cell NPML, 40 x 40 x 20 hexahedra =
192,000 tets, N = 4, LSERK4, two sources (10 Hz), 120 steps.

* Superposition. With the NPML energy trigger not armed, the solver is
  linear in the sources: one wavefield driven by both sources equals the sum
  of two batched wavefields with one source each, within 1e-5 relative L2
  (FP32 rounding of the sum). The oracle's own superposition check is the
  same at a size it finishes in seconds.
* Kernel kinds. The FP32, bulk-copy and node-pair kernels give the same bits
  at this size (about 70 chunks per block and a partial last chunk per
  class): SHA-256 digests of the wavefield, memory variables, NPML
  auxiliaries and traces match.
"""
import hashlib

import numpy as np
import pytest

from conftest import rel_l2
from nexd_b200 import Mesh, _abi, synth

pytestmark = pytest.mark.gpu

CELLS = (40, 40, 20)
NT = 120


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("full"))
    synth.write_twolayer(d, cells=CELLS, nt=NT, nrec=20, nsrc=2, f0=10.0, src_depth=(900.0, 1300.0))
    return d


@pytest.fixture(scope="module")
def Solver():
    from nexd_b200.solver import Solver as S
    return S


def _run(Solver, m, kinds, fields):
    s = Solver(m.desc_ptr)
    try:
        s.set_contraction_kinds(*kinds)
        s.run(1, NT)
        return fields(s)
    finally:
        s.close()


def test_superposition_at_full_size(model, Solver):
    mb = Mesh(model, N=4, nbatch=2)
    assert mb.K == 192000 and list(mb.array("srcbatch")) == [0, 1]
    kinds = ("fp32_bulk", "fp32_bulk")
    f0, f1 = _run(Solver, mb, kinds, lambda s: (s.field(0), s.field(1)))
    ms = Mesh(model, N=4, nbatch=1)
    assert list(ms.array("srcbatch")) == [0, 0]
    fs = _run(Solver, ms, kinds, lambda s: s.field(0))
    assert np.all(np.isfinite(fs)) and np.abs(f0).max() > 0 and np.abs(f1).max() > 0
    assert rel_l2(f0.astype(np.float64) + f1, fs) < 1e-5
    # each source contributes: neither wavefield alone is the joint one
    assert rel_l2(f0, fs) > 1e-2 and rel_l2(f1, fs) > 1e-2


def test_kernel_kinds_identical_at_full_size(model, Solver):
    m = Mesh(model, N=4)
    nth = 6 * m.desc.nMB

    def digests(s):
        arrs = (s.field(), s.state(_abi.NEXD_STATE_THETA, nfields=nth), s.state(_abi.NEXD_STATE_PML, nfields=27),
                s.traces())
        assert np.all(np.isfinite(arrs[0]))
        return [hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() for a in arrs]

    ref = _run(Solver, m, ("fp32", "fp32"), digests)
    for kinds in (("fp32_bulk", "fp32_bulk"), ("fp32_bulk", "fp32_pairs"), ("fp32", "fp32_bulk")):
        assert _run(Solver, m, kinds, digests) == ref, kinds
