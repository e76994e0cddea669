"""DSMC collisions with charged targets (collisions.f90:339-418) on the B200: electron-ion
elastic scattering on the ions themselves.  Checked against properties the algorithm must
have: momentum and kinetic energy conserved by each elastic pair, every target used by one
collision (the claims), and the collision count of the rate ns_coll dt n_i(cell) sigma v."""
import math

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs, deck as dk
from jd_lepic_b200.simulation import GpuSimulation

pytestmark = pytest.mark.gpu


def dsmc_case(with_neutral=False):
    case = configs.case0(ppc=100, nx=64, ny=64)
    case.deck_text = dk.argon_dsmc_deck(with_neutral=with_neutral)
    return case


def test_dsmc_conserves_pairs_uses_each_target_once_and_has_the_rate(gpu_lib):
    case = dsmc_case()
    sim = GpuSimulation(case)
    try:
        sp = sim.sp
        sim.sort(0)
        sim.sort(1)
        before = [sim.get_particles(s) for s in (0, 1)]
        npi = sim.grid(capi.GRID_NP + 1)
        mc = sim.collide(11)
        after = [sim.get_particles(s) for s in (0, 1)]
        ncoll = mc["n_coll"][0]
        assert ncoll > 100 and mc["n_add"] == [0, 0]
        assert [len(a) for a in after] == [len(b) for b in before]
        dv = [after[s][:, 3:] - before[s][:, 3:] for s in (0, 1)]
        # one incident and one distinct target per collision
        assert np.count_nonzero(np.any(dv[0] != 0, axis=1)) == ncoll
        assert np.count_nonzero(np.any(dv[1] != 0, axis=1)) == ncoll
        # momentum and kinetic energy of the pairs (FP32 storage of the new velocities)
        dP = sum(sp.Nm[s] * sp.mass[s] * dv[s].sum(axis=0) for s in (0, 1))
        ve = np.linalg.norm(before[0][:, 3:], axis=1).mean()
        assert np.abs(dP).max() <= 1e-3 * ncoll * sp.Nm[0] * sp.mass[0] * ve
        dE = sum(0.5 * sp.Nm[s] * sp.mass[s] * ((after[s][:, 3:] ** 2).sum() - (before[s][:, 3:] ** 2).sum())
                 for s in (0, 1))
        Ee = 0.5 * sp.Nm[0] * sp.mass[0] * (before[0][:, 3:] ** 2).sum(axis=1).mean()
        assert abs(dE) <= 1e-4 * ncoll * Ee
        # the rate: sum over electrons of ns_coll dt n_i(cell) sigma v (v_rel ~ v_e, sigma = 2e-15
        # m^2 up to 20 eV), n_i the mean of the ion density at the cell's four nodes
        x, y = before[0][:, 0], before[0][:, 1]
        ix = (x / case.dx).astype(int) + 1
        iy = (y / case.dy).astype(int) + 1
        ni = 0.25 * (npi[iy, ix] + npi[iy, ix + 1] + npi[iy + 1, ix] + npi[iy + 1, ix + 1])
        v = np.linalg.norm(before[0][:, 3:], axis=1)
        E = 0.5 * sp.mass[0] * v ** 2 / dk.QE
        expect = (10 * case.dt * ni * np.where(E <= 20.0, 2.0e-15, 0.0) * v).sum()
        assert abs(ncoll - expect) < 5 * math.sqrt(expect) + 0.03 * expect
    finally:
        sim.close()


def test_dsmc_with_neutral_background_in_the_step(gpu_lib):
    case = dsmc_case(with_neutral=True)
    case.poisson_mode = 1
    case.eps = 1e-8
    sim = GpuSimulation(case)
    try:
        n0 = sim.push_stats()["np_tot"]
        for it in range(1, 23):
            sim.step(it)
        mc = sim.mcc_stats()
        assert mc["n_coll"][0] > 0 and mc["n_coll"][1] > 0     # e-Ar+ (DSMC) and e-Ar (MC)
        st = sim.push_stats()
        assert st["np_tot"][1] == n0[1] - st["n_lost"][1]      # elastic: no ion created or killed
    finally:
        sim.close()
