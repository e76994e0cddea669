"""Golden fixtures (tests/golden/golden_32x32.npz, written by tests/golden/make_golden.py from
the CPU restatement): the restatement must reproduce them exactly, and the CUDA path must match
them within the stated tolerances."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

from jd_lepic_b200 import _capi as capi  # noqa: E402

GOLD = os.path.join(HERE, "golden", "golden_32x32.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_oracle_reproduces_golden(oracle_lib, gold, tmp_path, monkeypatch):
    monkeypatch.setattr(make_golden, "HERE", str(tmp_path))
    fresh = make_golden.make()
    for k, v in gold.items():
        assert np.array_equal(fresh[k], v), k


@pytest.mark.gpu
def test_gpu_matches_golden(gpu_lib, gold):
    from jd_lepic_b200.simulation import GpuSimulation
    case = make_golden.golden_case()
    s = GpuSimulation(case, tile=(8, 8), load=False, capacity=4096)
    for k in range(2):
        s.put_particles(k, gold[f"p{k}"])
        assert np.array_equal(s.get_particles(k)[:, [0, 1, 3, 4, 5]], gold[f"p{k}"][:, [0, 1, 3, 4, 5]])
    s.set_phi(gold["phi"])
    E = s.efield()
    assert np.array_equal(E, gold["E"])                       # bit-exact
    s.push(1)
    for k in range(2):
        got, ref = s.get_particles(k), gold[f"pushed{k}"]
        assert got.shape == ref.shape
        assert np.abs(got[:, :2] - ref[:, :2]).max() <= 1e-6 * case.dx
        v = np.linalg.norm(ref[:, 3:], axis=1) + s.sp.vt0[k]
        assert (np.linalg.norm(got[:, 3:] - ref[:, 3:], axis=1) / v).max() <= 1e-6
    # deposition of the device's own positions must equal the FP64 deposit to 1e-12
    from oracle import oracle as O
    cfg = O.make_cfg(case, s.sp)
    for k in range(2):
        p = s.get_particles(k)
        npg = np.zeros_like(gold["np"][k])
        O.deposit(cfg, k, p, p.shape[0], O.kq_of(case.bcnd), npg)
        assert np.abs(s.grid(capi.GRID_NP + k) - npg).max() <= 1e-12 * np.abs(npg).max()
    # the Poisson solve of the golden rhs
    a = np.ascontiguousarray(gold["rhs"])
    s.check(s.lib.lepic_gpu_set_grid(s.ctx, capi.GRID_RHS, a.ctypes.data_as(C.POINTER(C.c_double))), "set")
    st = s.solve(eps=1e-10, mode=capi.POISSON_FP64_MG, phi=np.where(case.bcnd >= 1, case.phi0, 0.0))
    assert [st["cycles"], st["sweeps_fine"]] == list(gold["solve_k"])
    assert np.abs(st["phi"] - gold["phi_solved"]).max() <= 1e-13 * np.abs(gold["phi_solved"]).max()
    s.close()
