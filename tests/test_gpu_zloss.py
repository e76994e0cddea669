"""The 3rd virtual dimension of the 2.5D model (hz >= 0; part_expmover.f90:216-219, 269-309,
400-421) on the device against the oracle's restatement (o_part_mover_z), particle by particle:

  electrons reaching z <= 0 or z >= zmax: lost when 0.5 m vz^2 / qe >= phi(ix,iy) - phi0, else
    reflected (vz -> -vz, z -> 0.02 or 0.98 zmax); z within 1e-6 of zmax, velocities 1e-6
  positive ions: lost with probability hz 2 uB / zmax dt, both sides drawing from the same
    counter-based stream, so the same ions are lost
  P_loss(1) takes Nm q phi at each loss point (1e-9 relative), p_mac counts them in igrid 0
and z is carried by the sort, put/get, the backup and the collision products."""
import math

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs, deck as dk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sim(case, **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8), **kw)


def _case():
    case = configs.case0(ppc=2, nx=64, ny=64)
    case.zmax = 0.01         # a 1 cm deep slab: the deck's zmax with hz >= 0
    return case


def _phi(case, amp=12.0):
    i = np.arange(case.nx + 3) - 1
    X, Y = np.meshgrid(i / case.nx, i / case.ny)
    return np.where(case.bcnd >= 1, 0.0, amp * np.sin(math.pi * X) * np.sin(math.pi * Y) + 2.0)


def _tallies(s):
    import ctypes as C
    t = capi.LepicTallies()
    s.check(s.lib.lepic_gpu_get_tallies(s.ctx, C.byref(t), 0), "get_tallies")
    return t


def test_electrons_end_plates_match_oracle(gpu_lib):
    case = _case()
    s = _sim(case, load=False, capacity=50000)
    try:
        s.set_zloss(hz=1.0, phi0=-1.0)
        rng = np.random.default_rng(9)
        n = 40000
        p = np.zeros((n, 6))
        p[:, 0] = rng.uniform(2, case.nx - 2, n) * case.dx
        p[:, 1] = rng.uniform(2, case.ny - 2, n) * case.dy
        # z within a step of an end plate, z-energies from 0.1 to 40 eV, both signs
        E = rng.uniform(0.1, 40.0, n)
        vzm = np.sqrt(2 * dk.QE * E / s.sp.mass[0])
        sgn = rng.choice([-1.0, 1.0], n)
        p[:, 5] = sgn * vzm
        p[:, 2] = np.where(sgn < 0, rng.uniform(0, 1, n) * vzm * case.dt, case.zmax - rng.uniform(0, 1, n) * vzm * case.dt)
        p[:, 3:5] = rng.normal(0, 3e5, (n, 2))
        p[:, 2:] = p[:, 2:].astype(np.float32)
        s.put_particles(0, p)
        s.set_phi(_phi(case))
        E_field = s.efield()
        s.sort(0)
        p0 = s.get_particles(0)
        # the sort carried z with its particle (particles matched by their FP32 velocities)
        zof = {(a, b, c): z for z, a, b, c in zip(p[:, 2], p[:, 3], p[:, 4], p[:, 5])}
        zs = np.array([zof[(a, b, c)] for a, b, c in zip(p0[:, 3], p0[:, 4], p0[:, 5])])
        bad = np.flatnonzero(zs != p0[:, 2])
        assert bad.size == 0, (bad.size, p0[bad[:5]], zs[bad[:5]])
        s.push(1)
        got = s.get_particles(0)
        cfg = O.make_cfg(case, s.sp)
        ref = p0.copy()
        nref, t = O.mover_z(cfg, 0, E_field, None, case.bcnd, ref, _phi(case), -1.0, np.zeros((65, 65), np.float32),
                            case.nx, 1, 1.0, case.seed, 1)
        ref = ref[:nref]
        lost_ref = n - nref
        assert 0.2 * n < lost_ref < 0.8 * n                  # both outcomes occur
        gi, rj, g_only, r_only = O.align_survivors(got, ref, case.dx, case.dy)
        assert g_only + r_only <= 2
        assert np.abs(got[gi, 2] - ref[rj, 2]).max() <= 1e-6 * case.zmax
        vmag = np.linalg.norm(ref[rj, 3:], axis=1)
        assert (np.linalg.norm(got[gi, 3:] - ref[rj, 3:], axis=1) / vmag).max() <= 1e-6
        # the reflected ones sit at 0.02 or 0.98 zmax with vz reversed
        refl = np.isclose(got[:, 2], 0.02 * case.zmax, rtol=1e-6) | np.isclose(got[:, 2], 0.98 * case.zmax, rtol=1e-6)
        assert refl.sum() > 0.1 * n
        tl = _tallies(s)
        assert abs(tl.n_loss[0][0] - t.n_loss[0]) <= 2 and t.n_loss[0] == lost_ref
        P1z_ref = t.P1z
        dev_P1 = tl.P_loss[0][0] - sum(tl.P_w[0][l] for l in range(capi.MAXLABEL))
        assert dev_P1 == pytest.approx(P1z_ref, rel=1e-6)
    finally:
        s.close()


def test_ions_bohm_losses_match_oracle(gpu_lib):
    case = _case()
    s = _sim(case, load=True)
    try:
        hz = 20000.0
        s.set_zloss(hz=hz, phi0=0.0, size_na=2)
        na1 = na2 = case.nx // 2
        uB = np.zeros((2, na2 + 1, na1 + 1))
        j, i = np.meshgrid(np.arange(na2 + 1), np.arange(na1 + 1), indexing="ij")
        uB[1] = 2000.0 + 30.0 * i + 10.0 * j                   # m/s, varying over the coarse grid
        s.set_bohm_speed(uB)
        s.set_phi(_phi(case))
        E_field = s.efield()
        s.sort(1)
        p0 = s.get_particles(1)
        s.push(5)
        got = s.get_particles(1)
        cfg = O.make_cfg(case, s.sp)
        ref = p0.copy()
        nref, t = O.mover_z(cfg, 1, E_field, None, case.bcnd, ref, _phi(case), 0.0,
                            uB[1].astype(np.float32), na1, 2, hz, case.seed, 5)
        ref = ref[:nref]
        lost = p0.shape[0] - nref
        ixc = (p0[:, 0] / (2 * case.dx)).astype(int)
        iyc = (p0[:, 1] / (2 * case.dy)).astype(int)
        expect = (hz * 2 * uB[1][iyc, ixc] / case.zmax * case.dt).sum()
        assert abs(lost - expect) < 5 * math.sqrt(expect)   # the rate itself
        gi, rj, g_only, r_only = O.align_survivors(got, ref, case.dx, case.dy)
        assert g_only == 0 and r_only == 0                  # the same ions: the same draws
        assert np.abs(got[gi, 2] - ref[rj, 2]).max() <= 1e-6 * case.zmax
        tl = _tallies(s)
        assert tl.n_loss[1][0] == lost
        dev_P1 = tl.P_loss[0][1] - sum(tl.P_w[1][l] for l in range(capi.MAXLABEL))
        assert dev_P1 == pytest.approx(t.P1z, rel=1e-6)
    finally:
        s.close()


def test_z_carried_through_sort_backup_and_products(gpu_lib, tmp_path):
    case = _case()
    s = _sim(case, load=False, capacity=20000)
    b = _sim(case, load=False, capacity=20000)
    try:
        s.set_zloss(hz=1.0)
        b.set_zloss(hz=1.0)
        rng = np.random.default_rng(3)
        n = 5000
        p = np.zeros((n, 6))
        p[:, 0] = rng.uniform(1, case.nx - 1, n) * case.dx
        p[:, 1] = rng.uniform(1, case.ny - 1, n) * case.dy
        p[:, 2] = rng.uniform(0.1, 0.9, n) * case.zmax
        p[:, 4] = math.sqrt(2 * 100 * dk.QE / s.sp.mass[0])  # 100 eV: ionizing
        p[:, 2:] = p[:, 2:].astype(np.float32)
        s.put_particles(0, p)
        s.put_particles(1, p)
        s.sort(0)
        q = s.get_particles(0)
        assert np.array_equal(np.sort(q[:, 2]), np.sort(p[:, 2]))
        path = str(tmp_path / "z.bak")
        s.write_backup(path)
        b.read_backup(path)
        assert np.array_equal(b.get_particles(0), q)
        st = s.collide(11)
        prod = s.get_particles(0)[n:]
        assert prod.shape[0] > 0
        parent_z = {(round(x, 15), round(y, 15)): z for x, y, z in q[:, :3]}
        for x, y, z in prod[:, :3]:
            assert parent_z[(round(x, 15), round(y, 15))] == z
    finally:
        s.close()
        b.close()
