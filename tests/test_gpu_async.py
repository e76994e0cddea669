"""The overlapped copies (lepic_gpu_iterative_solver_async, lepic_gpu_get_grid_async,
lepic_gpu_stage_solver_input): the host array receives exactly what the synchronous calls
return, once a synchronising call has returned, and one host array used for both directions
step after step (the input staged beside the push, or uploaded before the solve) gives the
same run as the synchronous solver."""
import ctypes as C

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs

pytestmark = pytest.mark.gpu


def _sim(case):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _run(how, steps=6):
    """how: 'sync' (phi in and out of the synchronous solver), 'async' (the solver's download
    overlapped), 'staged' (the next input staged beside the push, the download overlapped)."""
    case = configs.case1(ppc=8, nx=128, ny=128)
    s = _sim(case)
    try:
        lib, ctx = s.lib, s.ctx
        phi = np.ascontiguousarray(case.phi0, dtype=np.float64).copy()
        out = []
        if how == "staged":
            s.check(lib.lepic_gpu_stage_solver_input(ctx, _dp(phi)), "stage")
        for it in range(1, steps + 1):
            s.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs")
            if how == "async":
                s.check(lib.lepic_gpu_iterative_solver_async(ctx, _dp(phi), _dp(phi), 1e-8, 1), "solver_async")
            elif how == "staged":
                s.check(lib.lepic_gpu_iterative_solver_async(ctx, None, _dp(phi), 1e-8, 1), "solver_async")
            else:
                s.check(lib.lepic_gpu_iterative_solver(ctx, _dp(phi), 1e-8, 1, None), "solver")
            s.check(lib.lepic_gpu_calc_efield(ctx, None), "efield")
            if it % 3 == 1:
                for sp in range(2):
                    s.check(lib.lepic_gpu_part_sorting(ctx, sp, None), "sort")
            if how == "staged" and it < steps:
                s.check(lib.lepic_gpu_stage_solver_input(ctx, _dp(phi)), "stage")
            ps = capi.LepicPushStats()
            s.check(lib.lepic_gpu_push_deposit(ctx, it, C.byref(ps)), "push")   # synchronises
            out.append(phi.copy())
        return out, s.get_particles(0)
    finally:
        s.close()


@pytest.mark.parametrize("how", ["async", "staged"])
def test_overlapped_copies_run_equals_sync_run(gpu_lib, how):
    a, pa = _run(how)
    b, pb = _run("sync")
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(pa, pb)


def test_get_grid_async_matches_get_grid(gpu_lib):
    case = configs.case1(ppc=4, nx=128, ny=64)
    s = _sim(case)
    try:
        s.calc_rhs()
        s.solve(eps=1e-8, mode=1)
        s.efield()
        for which, shape in ((capi.GRID_PHI, (case.ny + 3, case.nx + 3)),
                             (capi.GRID_RHS, (case.ny + 1, case.nx + 1)),
                             (capi.GRID_EI, (case.ny + 3, case.nx + 3, 2))):
            out = np.full(shape, np.nan)
            s.check(s.lib.lepic_gpu_get_grid_async(s.ctx, which, _dp(out)), "get_grid_async")
            s.sync()
            np.testing.assert_array_equal(out, s.grid(which))
        # the snapshot is taken in stream order: a download enqueued before a solve holds the
        # potential before it
        before = s.grid(capi.GRID_PHI)
        early = np.full(before.shape, np.nan)
        s.check(s.lib.lepic_gpu_get_grid_async(s.ctx, capi.GRID_PHI, _dp(early)), "get_grid_async")
        s.set_phi(np.zeros_like(before))
        s.sync()
        np.testing.assert_array_equal(early, before)
        with pytest.raises(capi.LepicError):
            s.check(s.lib.lepic_gpu_get_grid_async(s.ctx, 99, _dp(early)), "get_grid_async")
    finally:
        s.close()
