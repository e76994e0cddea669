"""Two wall branches of part_mover on the device against the oracle's restatement
(o_part_mover_x), particle by particle (both sides draw from the same counter streams):

  refluxing (part_expmover.f90:445-470; opt_inj = 4 with the Neumann option): a particle at
    x <= 0 is re-drawn from the shifted-Maxwellian flux and placed at x = vx r dt; positions
    within one fixed-point unit, velocities 1e-6 relative, P_loss(1) / P_loss(4) 1e-6
  secondary emission (:354-392): positive ions lost on the emitting label give INT(gam) or
    INT(gam)+1 electrons at (xg_sec, y) appended to the electrons in the ions' slot order;
    the same count, positions and velocities, P_loss(4) of the electrons 1e-9, and the
    electrons are in the step's density (1e-12 against the oracle's deposit)."""
import ctypes as C
import math

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs, deck as dk, sources as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 64


def _sim(case, **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8), **kw)


def _float_match(ref, got, rel=1e-6):
    scale = np.maximum(np.abs(ref), 1e-30)
    np.testing.assert_array_less(np.abs(got - ref), rel * scale + 1e-30 + rel * np.abs(ref).max())


def _neumann_case():
    case = configs.case0(ppc=2, nx=N, ny=N)
    b = configs.box_mask(N, N)
    b[2:N + 1, 0:2] = -2          # the x = 0 column Neumann (generate_boundary.f90:137-145)
    case.bcnd = b
    case.flag_nmn = 1
    case.phi0 = configs.potentials(b, {1: 0.0})
    return case


def _reflux_params(case, sp, s, THm, th_B):
    """sources_reflux: part_injection.f90:34-47 (electrons: vb = 0 with the Neumann option) and
    init_shifted_maxwellian_flux (:267-290)."""
    vb = 0.0 if s == 0 else math.sqrt(2 * dk.QE * THm / abs(sp.mass[s]))
    v0 = sp.vt0[s]
    vmax = (vb + math.sqrt(vb * vb + 2 * v0 * v0)) / 2
    return dict(vb=vb, fmax=vmax * math.exp(-(vmax - vb) ** 2 / v0 ** 2), vt=v0, th_B=th_B)


def test_reflux_matches_oracle(gpu_lib):
    case = _neumann_case()
    sim = _sim(case, load=False, capacity=60000)
    try:
        THm, th_B = 4.0, 0.6
        sc = S.source_config(S.SourceDeck(I_inj=-1.0, opt_inj=4, THm=THm, th_B=th_B, nu_h=-1.0),
                             case.dt, sim.sp.vt0[0])
        sim.set_sources(sc)
        rng = np.random.default_rng(17)
        cfg = O.make_cfg(case, sim.sp)
        E = np.zeros((case.ny + 3, case.nx + 3, 2))
        sim.set_phi(np.zeros((case.ny + 3, case.nx + 3)))
        sim.efield()
        for s, vmag in ((0, 1.5e6), (1, 4.0e4)):
            n = 30000
            p = np.zeros((n, 6))
            p[:, 0] = rng.uniform(0.01, 3.0, n) * case.dx
            p[:, 1] = rng.uniform(2.0, N - 2.0, n) * case.dy
            p[:, 3] = -rng.uniform(0.05, 2.0, n) * case.dx / case.dt   # 0.05 to 2 cells per step
            p[:, 4:] = rng.normal(0.0, vmag, (n, 2))
            p[:, 3:] = p[:, 3:].astype(np.float32)
            sim.put_particles(s, p)
        for s in (0, 1):
            sim.sort(s)
        before = [sim.get_particles(s) for s in (0, 1)]
        sim.push(3)
        tl = capi.LepicTallies()
        sim.check(sim.lib.lepic_gpu_get_tallies(sim.ctx, C.byref(tl), 0), "get_tallies")
        for s in (0, 1):
            got = sim.get_particles(s)
            ref = before[s].copy()
            nref, t, w, _ = O.mover_wallx(cfg, s, E, None, case.bcnd, ref, case.seed, 3,
                                          reflux=_reflux_params(case, sim.sp, s, THm, th_B))
            assert nref == ref.shape[0] == got.shape[0]        # nothing is lost
            x0 = before[s][:, 0] + case.dt * before[s][:, 3]
            refluxed = x0 <= 0.0
            assert refluxed.sum() > 1000
            # refluxed particles: new velocities from the flux, x = vx r dt (not -x)
            assert np.all(ref[refluxed, 3] > 0)
            assert np.abs(got[:, 0] - ref[:, 0]).max() <= 2e-6 * case.dx
            assert np.abs(got[:, 1] - ref[:, 1]).max() <= 2e-6 * case.dy
            _float_match(ref[:, 3:], got[:, 3:])
            assert not np.allclose(got[refluxed, 0], -x0[refluxed])
            assert tl.P_loss[0][s] == pytest.approx(w.P1r, rel=1e-6)
            assert tl.P_loss[3][s] == pytest.approx(w.P4r, rel=1e-6)
            assert w.P4r > 0
    finally:
        sim.close()


def test_secondary_emission_matches_oracle(gpu_lib):
    case = configs.case0(ppc=2, nx=N, ny=N)
    b = configs.box_mask(N, N, label_right=2)
    case.bcnd = b
    case.phi0 = configs.potentials(b, {1: 0.0, 2: 0.0})
    sim = _sim(case, load=False, capacity=200000)
    try:
        gam, xg, THm = 2.4, (N - 12) * case.dx, 3.0
        sim.set_secondary(gam, 2, xg, THm)
        rng = np.random.default_rng(23)
        cfg = O.make_cfg(case, sim.sp)
        sim.set_phi(case.phi0)
        E = sim.efield()
        ne, ni = 5000, 30000
        pe = np.zeros((ne, 6))
        pe[:, 0] = rng.uniform(5, N - 5, ne) * case.dx
        pe[:, 1] = rng.uniform(5, N - 5, ne) * case.dy
        pe[:, 3:] = rng.normal(0, 3e5, (ne, 3)).astype(np.float32)
        pi = np.zeros((ni, 6))
        pi[:, 0] = (N - rng.uniform(0.01, 3.0, ni)) * case.dx
        pi[:, 1] = rng.uniform(0.5, N - 0.5, ni) * case.dy    # the corners too (label 1 there)
        pi[:, 3] = (rng.uniform(0.2, 4.0, ni) * case.dx / case.dt).astype(np.float32)
        pi[:, 4:] = rng.normal(0, 2e3, (ni, 2)).astype(np.float32)
        sim.put_particles(0, pe)
        sim.put_particles(1, pi)
        for s in (0, 1):
            sim.sort(s)
        e0, i0 = sim.get_particles(0), sim.get_particles(1)
        sim.push(5)
        e1 = sim.get_particles(0)
        tl = capi.LepicTallies()
        sim.check(sim.lib.lepic_gpu_get_tallies(sim.ctx, C.byref(tl), 0), "get_tallies")
        # the oracle: electrons moved, then the ions with the emission
        ref_e = e0.copy()
        ne_ref, _ = O.mover(cfg, 0, E, None, case.bcnd, ref_e)
        ref_i = i0.copy()
        vt_sec = math.sqrt(2 * dk.QE * THm / abs(sim.sp.mass[0]))
        ni_ref, ti, w, emitted = O.mover_wallx(
            cfg, 1, E, None, case.bcnd, ref_i, case.seed, 5,
            secondary=dict(label=2, gam=gam, vt=vt_sec, xg=xg, Nm0=sim.sp.Nm[0], m0=sim.sp.mass[0]))
        n_sec = emitted.shape[0]
        assert ti.n_loss[2] > 5000 and n_sec > 2 * ti.n_loss[2]
        assert e1.shape[0] == ne_ref + n_sec
        tail = e1[ne_ref:]
        unit = case.dx * 2e-6
        assert np.abs(tail[:, 0] - xg).max() <= unit
        assert np.abs(tail[:, 1] - emitted[:, 1]).max() <= 2e-6 * case.dy
        _float_match(emitted[:, 3:], tail[:, 3:])
        assert np.all(tail[:, 3] < 0)                          # back into the plasma
        assert tl.n_loss[1][2] == ti.n_loss[2]
        assert tl.P_loss[3][0] == pytest.approx(w.P4sec, rel=1e-9)
        # the secondaries are in this step's electron density
        kq = O.kq_of(np.asarray(case.bcnd))
        npg = np.zeros((case.ny + 3, case.nx + 3))
        O.deposit(cfg, 0, np.ascontiguousarray(e1), e1.shape[0], kq, npg)
        dev = sim.grid(capi.GRID_NP + 0)
        assert np.abs(dev - npg).max() <= 1e-12 * np.abs(npg).max()
        # gam = 0 switches the emission off
        sim.set_secondary(0.0, 2, xg, THm)
        with pytest.raises(capi.LepicError):
            sim.set_secondary(9.0, 2, xg, THm)
    finally:
        sim.close()
