"""Dielectric walls (generate_boundary.f90:149-152, part_expmover.f90:340-350, main.f90:756-809)
on the device against the oracle's restatement (o_part_mover_zd, o_dielectric_update):

  a wall loss on a dielectric label, or under one, leaves Nm q on the label's rows iy and iy+1
    of the loss cell, split by the loss point's y: per label and row within 2 particles' charge
    plus 1e-4 of the row (the device keeps positions in fixed point)
  the update adds kd dq / (Ca dy) to the dielectric labels' wall nodes of rows 2..ny (kd = 2 on
    rows 1 and ny+1) and clears dq: 1e-12 relative against the oracle on the device's own dq
  the Poisson solve keeps the charged wall nodes as Dirichlet values, and lepic_gpu_step
    applies the update before its solve."""
import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CA = 1e-7   # F/m^2


def _case():
    case = configs.case0(ppc=2, nx=64, ny=64)
    case.bcnd = configs.box_mask(case.nx, case.ny, label_left=2, label_right=3)
    case.phi0 = configs.potentials(case.bcnd, {1: 0.0, 2: 0.0, 3: 0.0})
    return case


def _sim(case, **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8), **kw)


def _wall_electrons(case, n, rng):
    """Electrons within three cells of the left and right walls moving into them, over the full
    height (the corners included: there the loss cell's label is the bottom or top wall's)."""
    p = np.zeros((n, 6))
    left = rng.random(n) < 0.5
    p[:, 0] = np.where(left, rng.uniform(0.02, 3.0, n), case.nx - rng.uniform(0.02, 3.0, n)) * case.dx
    p[:, 1] = rng.uniform(0.05, case.ny - 0.05, n) * case.dy
    sp = rng.uniform(0.5, 4.0, n) * case.dx / case.dt
    p[:, 3] = np.where(left, -sp, sp)
    p[:, 4] = rng.normal(0.0, 0.3, n) * case.dy / case.dt
    p[:, 5] = rng.normal(0.0, 1e5, n)
    p[:, 3:] = p[:, 3:].astype(np.float32)
    return p


def test_wall_charge_and_update_match_oracle(gpu_lib):
    case = _case()
    s = _sim(case, load=False, capacity=50000)
    try:
        dtype = np.zeros(16, np.int32)
        dtype[2] = dtype[3] = 1
        s.set_dielectrics(dtype, CA)
        rng = np.random.default_rng(21)
        n = 40000
        s.put_particles(0, _wall_electrons(case, n, rng))
        s.set_phi(case.phi0)
        E = s.efield()
        s.sort(0)
        p0 = s.get_particles(0)
        s.push(1)
        dq = s.dielectric_charge()
        cfg = O.make_cfg(case, s.sp)
        ref = p0.copy()
        nref, t, dq_ref = O.mover_dielec(cfg, 0, E, None, case.bcnd, ref, dtype)
        nmq = abs(s.sp.Nm[0] * s.sp.charge[0])
        lost = n - nref
        assert lost > 0.3 * n
        # every label's total: Nm q per loss (a particle within rounding of a wall may differ)
        for lab in range(16):
            assert abs(dq[lab].sum() - dq_ref[lab].sum()) <= 2.5 * nmq, lab
        assert abs(dq[2].sum()) > 0.1 * lost * nmq and abs(dq[3].sum()) > 0.1 * lost * nmq
        # the label-1 rows hold the corner losses under a dielectric (part_expmover.f90:343-345)
        assert abs(dq[1].sum()) > 0
        tol = 2.5 * nmq + 1e-4 * np.abs(dq_ref)
        bad = np.argwhere(np.abs(dq - dq_ref) > tol)
        assert bad.size == 0, (bad[:5], dq[tuple(bad[0])], dq_ref[tuple(bad[0])])
        # the update on the device's own charge
        phi0 = s.grid(capi.GRID_PHI)
        s.dielectric_update()
        phi1 = s.grid(capi.GRID_PHI)
        phi_ref = phi0.copy()
        O.dielectric_update(cfg, phi_ref, case.bcnd, dtype, dq.copy(), CA)
        np.testing.assert_allclose(phi1, phi_ref, rtol=1e-12, atol=1e-15)
        changed = phi1 != phi0
        assert changed.any()
        assert set(np.unique(case.bcnd[changed])) <= {2, 3}
        assert not changed[:2].any() and not changed[case.ny + 1:].any()   # rows 0, 1, ny+1, ny+2 stay
        assert not s.dielectric_charge().any()
        # the solve keeps the charged walls as Dirichlet values
        s.calc_rhs()
        st = s.solve(eps=1e-10, mode=1)
        assert st["res_l2_rel"] <= 1e-9
        phi2 = s.grid(capi.GRID_PHI)
        wall = case.bcnd >= 1
        np.testing.assert_array_equal(phi2[wall], phi1[wall])
    finally:
        s.close()


def test_step_applies_the_update_before_its_solve(gpu_lib):
    case = _case()
    s = _sim(case, load=False, capacity=50000)
    try:
        dtype = np.zeros(16, np.int32)
        dtype[2] = 1
        s.set_dielectrics(dtype, CA)
        rng = np.random.default_rng(5)
        s.put_particles(0, _wall_electrons(case, 20000, rng))
        s.set_phi(case.phi0)
        s.efield()
        s.sort(0)
        s.push(1)
        dq = s.dielectric_charge()
        phi0 = s.grid(capi.GRID_PHI)
        s.step(2)
        phi1 = s.grid(capi.GRID_PHI)
        expect = phi0.copy()
        O.dielectric_update(O.make_cfg(case, s.sp), expect, case.bcnd, dtype, dq.copy(), CA)
        lab2 = case.bcnd == 2
        np.testing.assert_allclose(phi1[lab2], expect[lab2], rtol=1e-12, atol=1e-15)
        assert (phi1[lab2] != 0).any()
        # label 3 is a conductor here: its wall stays at 0 V
        assert not phi1[case.bcnd == 3].any()
        # switched off: no charge kept
        s.set_dielectrics(np.zeros(16, np.int32), 0.0)
        with pytest.raises(capi.LepicError):
            s.dielectric_charge()
    finally:
        s.close()


def test_bad_dielectric_arguments(gpu_lib):
    case = _case()
    s = _sim(case, load=False, capacity=1000)
    try:
        d = np.zeros(16, np.int32)
        d[2] = 2
        with pytest.raises(capi.LepicError):
            s.set_dielectrics(d, CA)
        d[2] = 1
        with pytest.raises(capi.LepicError):
            s.set_dielectrics(d, 0.0)
    finally:
        s.close()


def test_two_ranks_summed_charge_equals_one_context(gpu_lib):
    """main.f90:758-772 with two ranks: each context holds half of the particles; their charges
    summed agree with one context holding all of them (each particle within the rounding of its
    fixed-point move), and the summed charge set on one rank gives the oracle's wall update."""
    case = _case()
    dtype = np.zeros(16, np.int32)
    dtype[2] = dtype[3] = 1
    rng = np.random.default_rng(8)
    p = _wall_electrons(case, 20000, rng)
    sims = [_sim(case, load=False, capacity=30000) for _ in range(3)]
    try:
        for s, q in zip(sims, [p, p[:10000], p[10000:]]):
            s.set_dielectrics(dtype, CA)
            s.put_particles(0, q)
            s.set_phi(case.phi0)
            s.efield()
            s.sort(0)
            s.push(1)
        nmq = abs(sims[0].sp.Nm[0] * sims[0].sp.charge[0])
        dq_sum = sims[1].dielectric_charge() + sims[2].dielectric_charge()
        dq_one = sims[0].dielectric_charge()
        assert np.all(np.abs(dq_sum - dq_one) <= 2.5 * nmq + 1e-4 * np.abs(dq_one))
        assert abs(dq_sum.sum() - dq_one.sum()) <= 2.5 * nmq
        sims[1].check(sims[1].lib.lepic_gpu_set_dielectric_charge(
            sims[1].ctx, np.ascontiguousarray(dq_sum).ctypes.data_as(capi.C.POINTER(capi.C.c_double))),
            "set_dielectric_charge")
        phi0 = sims[1].grid(capi.GRID_PHI)
        sims[1].dielectric_update()
        expect = phi0.copy()
        O.dielectric_update(O.make_cfg(case, sims[1].sp), expect, case.bcnd, dtype, dq_sum.copy(), CA)
        np.testing.assert_allclose(sims[1].grid(capi.GRID_PHI), expect, rtol=1e-12, atol=1e-15)
    finally:
        for s in sims:
            s.close()
