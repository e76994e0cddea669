"""Averaging diagnostics on the B200 (part_moments + calc_avg + the potential and field
averages) against the FP64 restatement.  The device sums in FP64 with atomics, so the check
is to 1e-12 of each component's largest magnitude."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import _capi as capi, configs, deck as dk
from jd_lepic_b200.simulation import GpuSimulation, species_params

pytestmark = pytest.mark.gpu

NX = 64


def get_avg(sim, size_na, reset=False):
    na = NX // size_na
    data = np.zeros((sim.sp.ntype, na + 1, na + 1, 7))
    phi = np.zeros((NX + 3, NX + 3, 3))
    cnt = C.c_int32()
    sim.check(sim.lib.lepic_gpu_get_avg(sim.ctx, data.ctypes.data_as(C.POINTER(C.c_double)),
                                        phi.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt), 1 if reset else 0),
              "get_avg")
    return data, phi, cnt.value


def close(a, b, tol=1e-12):
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() <= tol * scale, (np.abs(a - b).max(), scale)


@pytest.mark.parametrize("size_na", [1, 2, 4])
def test_averages_match_oracle(gpu_lib, size_na):
    case = configs.case0(ppc=4, nx=NX, ny=NX)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    cfg = O.make_cfg(case, sp)
    sim = GpuSimulation(case, load=False, capacity=400000)
    try:
        rng = np.random.default_rng(size_na)
        for s, vs in ((0, 1.0e6), (1, 5.0e2)):
            n = 200000
            v = np.zeros((n, 6))
            v[:, 0] = rng.random(n) * case.nx * case.dx * 0.999
            v[:, 1] = rng.random(n) * case.ny * case.dy * 0.999
            v[:, 3:] = rng.normal(0.0, vs, (n, 3)).astype(np.float32)
            v[:, 3] += vs
            sim.put_particles(s, v)
        sim.sort(0)
        sim.sort(1)
        sim.deposit()
        phi = rng.random((case.ny + 3, case.nx + 3))
        sim.set_phi(phi)
        E = sim.efield()
        sim.check(sim.lib.lepic_gpu_set_avg(sim.ctx, size_na, 0), "set_avg")
        sim.check(sim.lib.lepic_gpu_calc_avg(sim.ctx), "calc_avg")
        sim.check(sim.lib.lepic_gpu_calc_avg(sim.ctx), "calc_avg")
        data, phi_avg, cnt = get_avg(sim, size_na)
        assert cnt == 2
        kq = O.kq_of(np.asarray(case.bcnd))
        na = NX // size_na
        ref = np.zeros((sp.ntype, na + 1, na + 1, 7))
        for s in (0, 1):
            p = sim.get_particles(s)
            pm = O.part_moments(cfg, size_na, s, p, kq)
            npg = sim.grid(capi.GRID_NP + s)
            O.calc_avg(cfg, size_na, s, npg, pm, ref)
            O.calc_avg(cfg, size_na, s, npg, pm, ref)
        for s in (0, 1):
            for q in (0, 2, 3, 4):
                close(data[s, ..., q], ref[s, ..., q])
            close(data[s, ..., 1], ref[s, ..., 1], 1e-9)   # Tp: a difference of two close terms
        assert np.array_equal(phi_avg[..., 0], 2 * phi)
        assert np.array_equal(phi_avg[..., 1:], 2 * E)
        assert np.all(data[..., 5:] == 0.0)
        # reset
        get_avg(sim, size_na, reset=True)
        data2, phi2, cnt2 = get_avg(sim, size_na)
        assert cnt2 == 0 and not data2.any() and not phi2.any()
    finally:
        sim.close()


def test_step_takes_averages_at_navg(gpu_lib):
    case = configs.case0(ppc=8, nx=NX, ny=NX)
    case.poisson_mode = 1
    case.eps = 1e-8
    sim = GpuSimulation(case)
    try:
        sim.check(sim.lib.lepic_gpu_set_avg(sim.ctx, 2, 5), "set_avg")
        for it in range(1, 12):
            sim.step(it)
        data, phi, cnt = get_avg(sim, 2)
        assert cnt == 3                                   # it = 1, 6, 11
        assert data[..., 0].sum() > 0 and np.isfinite(data).all()
        # the averaged electron temperature is near the loaded 2 eV
        te = data[0, 4:-4, 4:-4, 1] / cnt
        assert 1.5 < np.median(te) < 2.5
    finally:
        sim.close()


def get_maps(sim):
    nt = sim.sp.ntype
    m = np.zeros((nt, NX + 3, NX + 3, 2))
    sim.check(sim.lib.lepic_gpu_get_source_maps(sim.ctx, m.ctypes.data_as(C.POINTER(C.c_double))), "source maps")
    return m


def test_source_sink_maps(gpu_lib):
    """ss2D with plt_src = 0: a wall loss counts at the node nearest its new position
    (part_expmover.f90:327-332), an injected particle at its cell's node (part_injection.f90:205);
    a sample adds the counts times Nm/Vc to data_pavg's columns 6 and 7 and zeroes them."""
    from jd_lepic_b200 import sources as S
    case = configs.case0(ppc=4, nx=NX, ny=NX)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    cfg = O.make_cfg(case, sp)
    sim = GpuSimulation(case, load=False, capacity=200000)
    try:
        sim.check(sim.lib.lepic_gpu_set_avg(sim.ctx, 2, 0), "set_avg")
        assert np.all(get_maps(sim) == 0.0)
        rng = np.random.default_rng(7)
        n = 3000
        v = np.zeros((n, 6))
        j = rng.integers(2, NX - 3, n)
        v[:, 0] = (0.3 + 0.4 * rng.random(n)) * case.dx          # in the first cell ...
        v[:, 1] = (j + 0.2 + 0.1 * rng.random(n)) * case.dy
        frac = 0.15 + 0.2 * rng.random(n)                         # ... and out through x = 0 to
        v[:, 3] = np.float32(-(v[:, 0] / case.dx + frac) * case.dx / case.dt)   # x in (-0.35, -0.15) dx
        keep = rng.random(n) < 0.3                                # some stay: slow, moving right
        v[keep, 3] = np.float32(1.0e3)
        sim.put_particles(0, v)
        sim.set_phi(np.zeros((NX + 3, NX + 3)))
        sim.efield()
        sim.push(1)
        m = get_maps(sim)
        lost = ~keep
        exp = np.zeros((NX + 3, NX + 3))
        np.add.at(exp, (j[lost] + 1, np.ones(lost.sum(), int)), 1.0)   # NINT(x/h) + 1 = 1, NINT(y/h) + 1 = j + 1
        assert np.array_equal(m[0, :, :, 1], exp)
        assert np.all(m[0, :, :, 0] == 0.0) and np.all(m[1] == 0.0)
        # injection: a source at each injected particle's (INT(x/h) + 1, INT(y/h) + 1)
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 0.5, 0.1, 0.5), I_inj=200.0, opt_inj=1,
                                          ni0=(1.0, 1.0), nu_h=-1.0, seed=5), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        before = [len(sim.get_particles(s)) for s in (0, 1)]
        sim.inject(2)
        m = get_maps(sim)
        for s in (0, 1):
            p = sim.get_particles(s)[before[s]:]
            assert len(p) > 100
            e = np.zeros((NX + 3, NX + 3))
            np.add.at(e, ((p[:, 1] / case.dy + 1e-9).astype(int) + 1, (p[:, 0] / case.dx + 1e-9).astype(int) + 1), 1.0)
            assert np.array_equal(m[s, :, :, 0], e)
        # a sample: columns 6, 7 against the restatement, then the counts start again
        sim.sort(0)
        sim.sort(1)
        sim.deposit()
        sim.check(sim.lib.lepic_gpu_calc_avg(sim.ctx), "calc_avg")
        data, _, _ = get_avg(sim, 2)
        kq = O.kq_of(np.asarray(case.bcnd))
        ref = np.zeros_like(data)
        for s in (0, 1):
            pm = O.part_moments(cfg, 2, s, sim.get_particles(s), kq)
            O.calc_avg(cfg, 2, s, sim.grid(capi.GRID_NP + s), pm, ref, ss=np.moveaxis(m[s], -1, 0))
            for q in (5, 6):
                close(data[s, ..., q], ref[s, ..., q])
        assert data[0, ..., 5].sum() > 0 and data[0, ..., 6].sum() > 0
        assert np.all(get_maps(sim) == 0.0)
    finally:
        sim.close()


def test_source_maps_count_collision_products(gpu_lib):
    """Collision products count as sources at the incident's cell node (collisions.f90:809):
    with 100 eV electrons on argon every ionization adds an electron and an ion there."""
    import math
    case = configs.case0(ppc=20, nx=NX, ny=NX)
    sim = GpuSimulation(case)
    try:
        sim.check(sim.lib.lepic_gpu_set_avg(sim.ctx, 1, 0), "set_avg")
        p = sim.get_particles(0)
        p[:, 3:] = 0.0
        p[:, 4] = math.sqrt(2 * 100 * 1.602e-19 / 9.109e-31)
        sim.put_particles(0, p)
        st = sim.collide(11)
        added = sim.mcc_stats()["n_add"]
        m = get_maps(sim)
        assert added[0] > 0 and added[1] == added[0]
        for s in (0, 1):
            assert m[s, ..., 0].sum() == added[s]
        # the sources sit on nodes of cells that hold electrons
        cells = np.zeros((NX + 3, NX + 3), bool)
        cells[(p[:, 1] / case.dy + 1e-9).astype(int) + 1, (p[:, 0] / case.dx + 1e-9).astype(int) + 1] = True
        assert np.all(cells[m[0, ..., 0] > 0])
    finally:
        sim.close()


def test_source_option_collision_frequencies(gpu_lib):
    """plt_src = 1 (collisions with flag_diag, collisions.f90:546-600): each 100 eV electron adds
    its ionization frequency n sigma v times Nm/Vc to the Ar+ source with CIC weights; the
    electron is not a source (it is the incident) and nothing is a sink (the electron survives,
    the target is a neutral); calc_avg takes the densities as they are."""
    import math
    case = configs.case0(ppc=8, nx=NX, ny=NX)
    E = dk.energy_grid(1e3, 50)
    sig = 2.0e-20
    case.deck_text = dk.write_deck("[Ar+]", 39.95, 0.03, "[Ar]", 0.0258,
                                   [("[e]+[Ar]->[e]+[e]+[Ar+]", "IONIZATION", 15.76, E, dk.sigma_constant(E, sig))])
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    sim = GpuSimulation(case)
    try:
        p = sim.get_particles(0)
        v = math.sqrt(2 * 100 * dk.QE / 9.10938e-31)
        p[:, 3:] = 0.0
        p[:, 4] = np.float32(v)
        sim.put_particles(0, p)
        sim.check(sim.lib.lepic_gpu_set_avg(sim.ctx, 1, 0), "set_avg")
        sim.check(sim.lib.lepic_gpu_set_source_option(sim.ctx, 1), "set_source_option")
        n_before = sim.push_stats()["np_tot"]
        sim.check(sim.lib.lepic_gpu_calc_avg(sim.ctx), "calc_avg")
        m = get_maps(sim)
        assert sim.push_stats()["np_tot"] == n_before          # no collision performed
        vc = case.dx * case.dy * case.zmax
        vf = float(np.float32(v))
        expect = len(p) * case.ngas * sig * vf * sp.Nm[1] / vc
        assert m[1, ..., 0].sum() == pytest.approx(expect, rel=1e-5)
        assert np.all(m[0, ..., 0] == 0.0) and np.all(m[..., 1] == 0.0)
        data, _, _ = get_avg(sim, 1)
        close(data[1, ..., 5], m[1, 1:NX + 2, 1:NX + 2, 0], 1e-14)
        # back to counting: the maps start from zero
        sim.check(sim.lib.lepic_gpu_set_source_option(sim.ctx, 0), "set_source_option")
        assert np.all(get_maps(sim) == 0.0)
    finally:
        sim.close()
