"""A sort leaves its permutation pending (lepic_options.sort_defer = 1, the default): the
collisions read and write through it and the push writes the sorted order as it moves the
particles (no separate gather).  Two contexts with the same deck and seed run the same steps:
one through lepic_gpu_step with the default, one through the single-routine entry points with
sort_defer = 0 (its sorts move the records at once); after the compared steps the particles,
their order and the charge densities agree bit for bit, through sort steps, collision steps
(neutral targets, and DSMC with charged targets) and the steps after them.  A pending
permutation is also moved by the calls that read the records (get_particles here).  The first
sort after a load moves the records itself (its permutation is far from the identity)."""
import ctypes as C

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs, deck as dk
from jd_lepic_b200.simulation import GpuSimulation

pytestmark = pytest.mark.gpu


def _pair(case):
    a, b = GpuSimulation(case, tile=(8, 8)), GpuSimulation(case, tile=(8, 8))
    b.set_options(sort_defer=0)   # b's sorts move the records at once
    return a, b


def _manual_step(s, it, eps, mode):
    """main.f90:818-1090 through the separate entry points, the order lepic_gpu_step keeps."""
    g = s.case
    lib, ctx = s.lib, s.ctx
    s.check(lib.lepic_gpu_calc_rhs(ctx, None), "calc_rhs")
    s.check(lib.lepic_gpu_iterative_solver(ctx, None, eps, mode, None), "solver")
    s.check(lib.lepic_gpu_calc_efield(ctx, None), "efield")
    if it % 10 == 1:
        for sp in range(2):
            s.check(lib.lepic_gpu_part_sorting(ctx, sp, None), "sort")
    if it > 1 and it % 10 == 1:
        s.check(lib.lepic_gpu_collisions(ctx, it, None), "collisions")
    s.check(lib.lepic_gpu_push_deposit(ctx, it, None), "push")


def _compare(a, b, case, it):
    for sp in range(2):
        pa, pb = a.get_particles(sp), b.get_particles(sp)
        assert pa.shape == pb.shape, (it, sp, pa.shape, pb.shape)
        assert np.array_equal(pa, pb), (it, sp)
        np.testing.assert_array_equal(a.grid(capi.GRID_NP + sp), b.grid(capi.GRID_NP + sp))


@pytest.mark.parametrize("kind", ["neutral", "dsmc"])
def test_step_with_pending_permutation_equals_separate_calls(gpu_lib, kind):
    case = configs.case0(ppc=30, nx=64, ny=64)
    if kind == "dsmc":
        case.deck_text = dk.argon_dsmc_deck(with_neutral=True)
    a, b = _pair(case)
    try:
        for it in range(1, 26):
            a.check(a.lib.lepic_gpu_step(a.ctx, it, 1e-8, 1), "step")
            _manual_step(b, it, 1e-8, 1)
            if it in (1, 2, 11, 12, 21, 25):
                _compare(a, b, case, it)
        ma, mb = a.mcc_stats(), b.mcc_stats()
        assert ma["n_coll"] == mb["n_coll"] and sum(ma["n_coll"]) > 0
        ta, tb = capi.LepicTallies(), capi.LepicTallies()
        a.check(a.lib.lepic_gpu_get_tallies(a.ctx, C.byref(ta), 0), "tallies")
        b.check(b.lib.lepic_gpu_get_tallies(b.ctx, C.byref(tb), 0), "tallies")
        assert [list(r) for r in ta.n_loss] == [list(r) for r in tb.n_loss]
    finally:
        a.close()
        b.close()


def test_calls_between_sort_and_push_see_the_sorted_order(gpu_lib):
    """Through the single-routine entry points: a sort followed by the push (which moves the
    records as it writes them) gives the same particles as the immediate gather; a pending
    permutation is moved by the calls that read the records (the particles, the tallies)."""
    case = configs.case0(ppc=20, nx=64, ny=64)
    a, b = _pair(case)
    try:
        for s in (a, b):
            s.calc_rhs()
            s.solve(eps=1e-8, mode=1)
            s.efield()
            s.push(1)   # leaves loss holes for the sort to drop
            for sp in range(2):
                s.sort(sp)   # the first sort after the load moves the records at once
            s.push(2)
            for sp in range(2):
                s.sort(sp)   # a: pending
            s.push(3)   # a: through the pending permutation
        _compare(a, b, case, 3)
        for s in (a, b):
            for sp in range(2):
                s.sort(sp)
        for sp in range(2):   # a: moves the records first
            assert np.array_equal(a.get_particles(sp), b.get_particles(sp))
        for s in (a, b):
            s.push(4)
            for sp in range(2):
                s.sort(sp)
        ta, tb = capi.LepicTallies(), capi.LepicTallies()
        a.check(a.lib.lepic_gpu_get_tallies(a.ctx, C.byref(ta), 0), "tallies")
        b.check(b.lib.lepic_gpu_get_tallies(b.ctx, C.byref(tb), 0), "tallies")
        assert [list(r) for r in ta.n_loss] == [list(r) for r in tb.n_loss]
        assert sum(sum(r) for r in ta.n_loss) > 0
        for s in (a, b):
            s.push(5)
        _compare(a, b, case, 5)
    finally:
        a.close()
        b.close()
