"""The allocation-free energy entry point, nexd_wavefield_energy_noalloc.

Hosts whose device memory belongs to another allocator (a framework's caching
allocator, or a pool a Fortran/MPI host reserves up front), and monitoring code
that must not pay cudaMalloc's implicit device synchronisation, cannot allocate
scratch while a run is in progress.  This entry point gives them the wavefield
energy using only a fixed scratch array compiled into libnexd.so; the caller
owns every input and output.  The test checks it through the C-ABI against the
solver's own energy (nexd_pml_trigger / nexd_get_energy), which allocates its
scratch, and against the CPU oracle's energy of the same run, on two calls in
a row; that repeated calls leave the device's free memory and torch's
allocation count unchanged (the point of the entry point); and that oversized
requests and misaligned caller pointers are refused without a launch.

This file is collected last on purpose (test_zz_*), so that a run stopping at
its first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2, run_oracle_trigger
from nexd_b200 import Mesh, synth, _abi

pytestmark = pytest.mark.gpu


def _device_inputs(m, q_host, torch):
    """Device copies of the wavefield (field-major), per-element (rho, lambda,
    mu, J) and the FP64 mass matrix, allocated by the caller (here: torch)."""
    K, Np = m.K, m.Np
    q = torch.from_numpy(np.ascontiguousarray(q_host.T)).cuda()  # (9, K*Np)
    emat = np.stack([m.array("rho"), m.array("lambdau"), m.array("muu"), m.array("jacobian")], axis=1)
    emat = torch.from_numpy(np.ascontiguousarray(emat, dtype=np.float32)).cuda()  # (K, 4)
    mass = torch.from_numpy(np.ascontiguousarray(np.linalg.inv(m.array("invmass")).T)).cuda()  # row-major M(n,k)
    torch.cuda.synchronize()
    return q, emat, mass, K * Np


def _noalloc(lib, q, ldq, m, nbatch, emat, mass, formula):
    out = np.zeros(nbatch, dtype=np.float64)
    st = lib.nexd_wavefield_energy_noalloc(q.data_ptr(), ldq, m.K, m.Np, nbatch, emat.data_ptr(), mass.data_ptr(),
                                           formula, out.ctypes.data_as(C.POINTER(C.c_double)))
    return st, out


@pytest.mark.parametrize("formula", [0, 1])
def test_noalloc_energy_matches_solver_and_oracle(tmp_path, oracle, formula):
    torch = pytest.importorskip("torch")
    from nexd_b200.solver import Solver
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(6, 6, 3), nt=40, nrec=4, src_depth=(800.0, 800.0))
    m = Mesh(d, N=3, stf_stage_time=True)
    s = Solver(m.desc_ptr)
    s.pml_trigger(10, 2, 1e30, 10.0, formula)  # energy every step, trigger never fires
    _, eo, _ = run_oracle_trigger(oracle, m, 64, thr=1e30, f0=10.0, formula=formula)  # FP64 CPU energy history
    lib = _abi.gpu_lib()
    for it in (30, 31):  # two calls in a row, on consecutive wavefields
        s.run(1 if it == 30 else it, it)
        ref, _ = s.energy()
        q, emat, mass, ldq = _device_inputs(m, s.field(), torch)
        st, got = _noalloc(lib, q, ldq, m, 1, emat, mass, formula)
        assert st == 0
        assert ref[it - 1, 0] != 0.0
        assert rel_l2(got, ref[it - 1:it, 0]) < 1e-6, (it, got, ref[it - 1, 0])
        # the oracle evolves the wavefield in FP64: FP32 rounding of the state only
        assert rel_l2(got, eo[it - 1:it, 0]) < 1e-5, (it, got, eo[it - 1, 0])
    s.close()


def test_noalloc_energy_allocates_nothing(tmp_path):
    """After the first call on the device (which looks up the scratch array's
    address and loads the kernels), further calls change neither the device's
    free memory nor what torch has allocated."""
    torch = pytest.importorskip("torch")
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(5, 5, 2), nt=5, nrec=2, src_depth=(800.0, 800.0))
    m = Mesh(d, N=3)
    rng = np.random.default_rng(1)
    q_host = (rng.standard_normal((m.K * m.Np, 9)) * np.array([1e3] * 6 + [1e-3] * 3)).astype(np.float32)
    q, emat, mass, ldq = _device_inputs(m, q_host, torch)
    lib = _abi.gpu_lib()
    st, first = _noalloc(lib, q, ldq, m, 1, emat, mass, 1)
    assert st == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(5):
        st, got = _noalloc(lib, q, ldq, m, 1, emat, mass, 1)
        assert st == 0 and got[0] == first[0]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_energy_refuses_misaligned_device_pointers(tmp_path):
    """Views of caller-owned device memory at an offset that breaks the
    required alignment are refused with NEXD_ERR_INVALID (nothing runs, the
    context stays usable)."""
    torch = pytest.importorskip("torch")
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(5, 5, 2), nt=5, nrec=2, src_depth=(800.0, 800.0))
    m = Mesh(d, N=2)
    q_host = np.ones((m.K * m.Np, 9), dtype=np.float32)
    q, emat, mass, ldq = _device_inputs(m, q_host, torch)
    lib = _abi.gpu_lib()
    out = np.zeros(1, dtype=np.float64)
    ptr = out.ctypes.data_as(C.POINTER(C.c_double))
    emat_off = torch.empty(emat.numel() + 1, dtype=torch.float32, device="cuda")[1:]  # 4-byte offset
    mass_off = torch.empty(mass.numel() * 2 + 1, dtype=torch.float32, device="cuda")[1:]  # 4-byte offset
    assert lib.nexd_wavefield_energy_noalloc(q.data_ptr(), ldq, m.K, m.Np, 1, emat_off.data_ptr(), mass.data_ptr(),
                                             1, ptr) == _abi.NEXD_ERR_INVALID
    assert lib.nexd_wavefield_energy_noalloc(q.data_ptr(), ldq, m.K, m.Np, 1, emat.data_ptr(), mass_off.data_ptr(),
                                             1, ptr) == _abi.NEXD_ERR_INVALID
    st, got = _noalloc(lib, q, ldq, m, 1, emat, mass, 1)  # the aligned call still works
    assert st == 0 and got[0] > 0


def test_noalloc_energy_batched_and_limits(tmp_path):
    torch = pytest.importorskip("torch")
    d = str(tmp_path / "pml")
    synth.write_twolayer(d, cells=(5, 5, 2), nt=5, nrec=2, src_depth=(800.0, 800.0))
    m = Mesh(d, N=2)
    rng = np.random.default_rng(0)
    lib = _abi.gpu_lib()
    q1 = (rng.standard_normal((m.K * m.Np, 9)) * np.array([1e3] * 6 + [1e-3] * 3)).astype(np.float32)
    q2 = 2.0 * q1
    qa, emat, mass, ldq = _device_inputs(m, q1, torch)
    qb, _, _, _ = _device_inputs(m, q2, torch)
    qq = torch.cat([qa, qb], dim=0).contiguous()  # two wavefields, stride 9*ldq
    for _ in range(2):
        st, got = _noalloc(lib, qq, ldq, m, 2, emat, mass, 1)
        assert st == 0
        # the energy is a quadratic form: doubling the wavefield multiplies it by 4
        assert got[0] > 0 and abs(got[1] / got[0] - 4.0) < 1e-6
    # more wavefields than the static scratch holds are refused, nothing launched
    big = np.zeros(1, dtype=np.float64)
    st = lib.nexd_wavefield_energy_noalloc(qq.data_ptr(), ldq, m.K, m.Np, _abi.NEXD_NOALLOC_MAX_BATCH + 1,
                                           emat.data_ptr(), mass.data_ptr(), 1,
                                           big.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == _abi.NEXD_ERR_INVALID
