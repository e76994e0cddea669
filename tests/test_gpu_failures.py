"""Failure paths of the device path, each made on the host or by the deck, never by a GPU fault:
every call returns its status and the context stays usable afterwards.

  LEPIC_ENOTCONV   ncycl V-cycles without reaching eps (main.f90:261) -- the FP64 multigrid
                   stops after the same cycle as the oracle, with the same potential
  LEPIC_EDIVERGED  the residual grew 10x (iterative_solver.f90:39-51) -- a deck on which the
                   reference's V-cycle diverges (a 2-cell plate at 256^2: injection-coarsened
                   masks lose the conductor), the oracle diverging on it too
  LEPIC_ERANGE     Pmax = nu_max ns_coll dt > 1 (collisions.f90:119-123), the oracle too
  LEPIC_ETIMEOUT   the solvers' bounded grid barrier waits for one CTA more than launched
                   (lepic_options::barrier_extra), gives up after about 2 s and ends the kernel
A truncated backup file is in tests/test_gpu_backup.py."""
import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sim(case, **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8), **kw)


def _set_rhs(s, rhs):
    import ctypes as C
    a = np.ascontiguousarray(rhs)
    s.check(s.lib.lepic_gpu_set_grid(s.ctx, capi.GRID_RHS, a.ctypes.data_as(C.POINTER(C.c_double))), "set_grid")


def _structured_rhs(s, case):
    rhs = s.calc_rhs()
    i = np.arange(case.nx + 1)
    X, Y = np.meshgrid(i / case.nx, i / case.ny)
    return rhs + 1.6e-3 * np.sin(3 * np.pi * X) * np.sin(2 * np.pi * Y)


def test_notconv_after_ncycl_cycles(gpu_lib):
    case = configs.case0(ppc=4, nx=64, ny=64)
    s = _sim(case, config={"ncycl": 2})
    try:
        rhs = _structured_rhs(s, case)
        _set_rhs(s, rhs)
        with pytest.raises(capi.LepicError) as e:
            s.solve(eps=1e-12, mode=capi.POISSON_FP64_MG, phi=case.phi0.copy())
        assert e.value.code == capi.ENOTCONV
        got = s.grid(capi.GRID_PHI)
        cfg = O.make_cfg(case, s.sp)
        ref = case.phi0.copy()
        rc, st = O.solve(cfg, ref, rhs, case.bcnd, case.levels(), 1e-12, ncycl=2)
        assert st.k == 2 and st.res > 1e-12
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
        # the mixed solver's iteration cap
        s.set_options(mx_max_iter=1)
        with pytest.raises(capi.LepicError) as e:
            s.solve(eps=1e-12, mode=capi.POISSON_MIXED_IR, phi=case.phi0.copy())
        assert e.value.code == capi.ENOTCONV
        # the context is usable: defaults back, both solvers converge
        s.set_options(mx_max_iter=200)
        st = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR, phi=case.phi0.copy())
        assert st["res_l2_rel"] <= 1e-8
    finally:
        s.close()


def test_diverged_on_a_deck_where_the_reference_diverges(gpu_lib):
    nx = 256
    case = configs.case4(ppc=1, nx=nx, ny=nx)
    ap = max(5, int(round(40 * nx / 2048)))
    case.bcnd = configs.aperture_plate(nx, nx, thickness=2, aperture=ap)
    case.phi0 = configs.potentials(case.bcnd, {1: 0.0, 2: 1000.0, 3: -50.0})
    s = _sim(case, load=False)
    try:
        rhs = np.zeros((nx + 1, nx + 1))
        _set_rhs(s, rhs)
        cfg = O.make_cfg(case, s.sp)
        ref = case.phi0.copy()
        rc, st = O.solve(cfg, ref, rhs, case.bcnd, case.levels(), 1e-10, ncycl=200)
        assert rc == -1                                    # the oracle aborts as the reference does
        with pytest.raises(capi.LepicError) as e:
            s.solve(eps=1e-10, mode=capi.POISSON_FP64_MG, phi=case.phi0.copy())
        assert e.value.code == capi.EDIVERGED
        s.sync()                                           # the error was reported once
        st = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR, phi=case.phi0.copy())
        assert st["res_l2_rel"] <= 1e-8                    # the CG's own residual test still holds
    finally:
        s.close()


def test_range_error_when_pmax_exceeds_one(gpu_lib):
    case = configs.case0(ppc=2, nx=32, ny=32)
    case.dt = 2e-9                                         # 6e7 1/s * 10 * 2e-9 = 1.2
    s = _sim(case)
    try:
        with pytest.raises(capi.LepicError) as e:
            s.collide(11)
        assert e.value.code == capi.ERANGE
        cfg = O.make_cfg(case, s.sp)
        rc, _, _, _ = O.collisions(cfg, O.XsHolder(s.xs), [s.get_particles(0), s.get_particles(1)], seed=1)
        assert rc == -1
        s.push(1)                                          # the context stays usable
        s.sync()
    finally:
        s.close()


@pytest.mark.parametrize("mode", [capi.POISSON_FP64_MG, capi.POISSON_MIXED_IR])
def test_grid_barrier_timeout(gpu_lib, mode):
    case = configs.case0(ppc=2, nx=64, ny=64)
    s = _sim(case)
    try:
        rhs = _structured_rhs(s, case)
        _set_rhs(s, rhs)
        s.set_options(barrier_extra=1)
        with pytest.raises(capi.LepicError) as e:
            s.solve(eps=1e-8, mode=mode, phi=case.phi0.copy())
        assert e.value.code == capi.ETIMEOUT
        s.set_options(barrier_extra=0)
        st = s.solve(eps=1e-10, mode=capi.POISSON_FP64_MG, phi=case.phi0.copy())
        cfg = O.make_cfg(case, s.sp)
        ref = case.phi0.copy()
        O.solve(cfg, ref, rhs, case.bcnd, case.levels(), 1e-10)
        assert np.abs(st["phi"] - ref).max() <= 1e-13 * np.abs(ref).max()
    finally:
        s.close()
