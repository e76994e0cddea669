"""Loss, power and collision tallies on the B200: p_mac by wall label from the push,
P_loss(3) and cnt_col from the collisions, P_loss(2)/(4) from the sources."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import _capi as capi, configs, deck as dk
from jd_lepic_b200 import sources as S
from jd_lepic_b200.simulation import GpuSimulation, species_params

pytestmark = pytest.mark.gpu


def tallies(sim, reset=False):
    t = capi.LepicTallies()
    sim.check(sim.lib.lepic_gpu_get_tallies(sim.ctx, C.byref(t), 1 if reset else 0), "get_tallies")
    return t


def test_push_loss_tallies_by_wall_label(gpu_lib):
    case = configs.case4(ppc=1, nx=64, ny=64)
    case.dt = 1e-10          # three cells per step stay far below the push's 3e8 m/s check
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    sim = GpuSimulation(case, load=False, capacity=10000)
    try:
        i0 = int(round(0.8 * 64)) + 1
        rng = np.random.default_rng(4)
        v, ex, v2 = [], {1: 0, 2: 0, 3: 0}, {1: 0.0, 2: 0.0, 3: 0.0}
        for k in range(400):
            y = (10.3 + rng.random() * 3) * case.dy
            speed = float(np.float32((3.0 + 0.5 * rng.random()) * case.dx / case.dt))
            kind = k % 4
            if kind == 0:
                p = (0.2 * case.dx, y, 0, -speed, 0, 0); lab = 3
            elif kind == 1:
                p = ((i0 - 1.3) * case.dx, y, 0, speed, 0, 0); lab = 2
            elif kind == 2:
                p = (20.4 * case.dx, 63.8 * case.dy, 0, 0, speed, 0); lab = 1
            else:
                p = (30.5 * case.dx, 30.5 * case.dy, 0, 0.1 * case.dx / case.dt, 0, 0); lab = None
            if lab:
                ex[lab] += 1
                v2[lab] += speed ** 2
            v.append(p)
        sim.put_particles(0, np.array(v))
        sim.push(1)
        t = tallies(sim)
        assert sim.push_stats()["n_lost"][0] == 300
        Ek = 0.5 * sp.Nm[0] * sp.mass[0]
        for lab in (1, 2, 3):
            assert t.n_loss[0][lab] == ex[lab]
            # the Boris rotation in Bz keeps |v| to FP32 rounding
            assert t.P_w[0][lab] == pytest.approx(Ek * v2[lab], rel=1e-5)
        assert t.P_loss[0][0] == pytest.approx(sum(t.P_w[0][l] for l in range(capi.MAXLABEL)), rel=1e-14)
        t = tallies(sim, reset=True)
        t = tallies(sim)
        assert sum(t.n_loss[0]) == 0 and t.P_loss[0][0] == 0.0
    finally:
        sim.close()


def test_collision_energy_identity_and_region_counts(gpu_lib):
    case = configs.case0(ppc=100, nx=64, ny=64)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    sim = GpuSimulation(case)
    try:
        L = case.nx * case.dx
        xl = np.array([0.0, 0.5 * L]); xr = np.array([0.5 * L, L])
        sim.check(sim.lib.lepic_gpu_set_regions(sim.ctx, 2, xl.ctypes.data_as(C.POINTER(C.c_double)),
                                                xr.ctypes.data_as(C.POINTER(C.c_double)), 0.0,
                                                case.ny * case.dy), "set_regions")
        sim.sort(0)
        sim.sort(1)
        before = [sim.get_particles(s) for s in (0, 1)]
        mc = sim.collide(11)
        after = [sim.get_particles(s) for s in (0, 1)]
        t = tallies(sim)
        assert sum(mc["n_coll"]) > 100
        dE = 0.0
        for s in (0, 1):
            Ek = 0.5 * sp.Nm[s] * sp.mass[s]
            dE += Ek * ((after[s][:, 3:] ** 2).sum() - (before[s][:, 3:] ** 2).sum())
        P3 = t.P_loss[2][0] + t.P_loss[2][1]
        assert P3 == pytest.approx(dE, rel=1e-6)
        # cnt_col(3, c, rg) = collisions of c in the region / np_tot_rg
        ix_mid = int(round(0.5 * L / case.dx)) + 1
        npg = [sim.grid(capi.GRID_NP + s) for s in (0, 1)]
        cnt3 = np.array(t.cnt_col[2])          # [c][rg]
        cnt2 = np.array(t.cnt_col[1])
        for s in (0, 1):
            k = case.dx * case.dy * case.zmax / sp.Nm[s]
            cols = [int(sim.xs.sig_list[s][q]) for q in range(int(sim.xs.p_ncol[s]))]
            tot = 0.0
            for rg, (a, b) in enumerate(((1, ix_mid), (ix_mid, case.nx + 1))):
                np_rg = k * npg[s][1:case.ny + 2, a:b + 1].sum()
                n_rg = sum(cnt3[c][rg] for c in cols) * np_rg
                assert n_rg > 0
                tot += n_rg
            # every cell lies in a region (the first that holds it), so the regions' counts add
            # up to all collisions of the species
            assert tot == pytest.approx(sum(mc["n_coll"][c] for c in cols), rel=1e-9)
            assert all(cnt2[c][0] + cnt2[c][1] <= mc["n_cand"][s] for c in cols)
            assert all(t.cnt_col[0][c][0] > 0 for c in cols)
    finally:
        sim.close()


def test_source_power_in_tallies(gpu_lib):
    case = configs.case0(ppc=8, nx=64, ny=64)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    sim = GpuSimulation(case)
    try:
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 0.5, 0.1, 0.5), nu_h=1e10, I_inj=50.0, opt_inj=1,
                                          ni0=(1.0, 1.0)), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        sim.eheating(4)
        sim.inject(4)
        st = sim.source_tallies()
        t = tallies(sim)
        assert t.P_loss[1][0] == st["P_heat"] and t.P_loss[3][0] == st["P_inj"][0] and t.P_loss[3][1] == st["P_inj"][1]
        tallies(sim, reset=True)
        assert sim.source_tallies()["P_heat"] == 0.0
    finally:
        sim.close()
