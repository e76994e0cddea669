"""The CPU restatement of the averaging diagnostics (part_moments, calc_avg: utils.f90),
pinned by the moments of a drifting Maxwellian: flux n u and temperature T come back."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import configs, deck as dk
from jd_lepic_b200.simulation import species_params


def setup(nx=32):
    case = configs.case0(ppc=4, nx=nx, ny=nx)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    return case, O.make_cfg(case, sp), sp


@pytest.mark.parametrize("size_na", [1, 2, 4])
def test_drifting_maxwellian_moments(oracle_lib, size_na):
    case, cfg, sp = setup()
    rng = np.random.default_rng(3)
    n = 400000
    T, u = 2.0, 3.0e5                                   # eV, m/s drift along x
    vt = math.sqrt(2 * dk.QE * T / abs(sp.mass[0]))
    v = np.zeros((n, 6))
    v[:, 0] = rng.random(n) * case.nx * case.dx
    v[:, 1] = rng.random(n) * case.ny * case.dy
    v[:, 3:] = rng.normal(0.0, vt / math.sqrt(2), (n, 3))
    v[:, 3] += u
    kq = O.kq_of(np.asarray(case.bcnd))
    npg = np.zeros((case.ny + 3, case.nx + 3))
    O.deposit(cfg, 0, v, n, kq, npg)
    pm = O.part_moments(cfg, size_na, 0, v, kq)
    na = case.nx // size_na
    data = np.zeros((cfg.ntype, na + 1, na + 1, 7))
    O.calc_avg(cfg, size_na, 0, npg, pm, data)
    inner = data[0, 2:-2, 2:-2]
    nd = inner[..., 0].copy()
    # flux / density = drift, temperature = T (statistical, ~n/cells particles per node)
    assert abs((inner[..., 2].sum() / nd.sum()) / u - 1) < 0.02
    assert abs(inner[..., 3].sum() / nd.sum()) < 0.02 * u
    assert abs(np.median(inner[..., 1]) / T - 1) < 0.05
    # two samples accumulate
    O.calc_avg(cfg, size_na, 0, npg, pm, data)
    assert np.allclose(data[0, 2:-2, 2:-2, 0], 2 * nd)


def test_moments_back_step_and_bounds(oracle_lib):
    case, cfg, sp = setup()
    kq = O.kq_of(np.asarray(case.bcnd))
    v = np.zeros((2, 6))
    v[0, :2] = (10.5 * case.dx, 7.5 * case.dy)
    v[0, 3:] = (2 * case.dx / case.dt, 0.0, 0.0)       # x - vx dt/2 moves it one cell left
    v[1, :2] = (0.1 * case.dx, 3.0 * case.dy)
    v[1, 3] = 1.0 * case.dx / case.dt                  # back-stepped out of the box: skipped
    pm = O.part_moments(cfg, 1, 0, v, kq)
    W = case.nx + 3
    k1 = sp.Nm[0] / (case.dx * case.dy * cfg.zmax)
    # the particle sits at x = 9.5 dx after the half step back: nodes 10 and 11 share jx
    jx = pm[1]
    assert jx.sum() == pytest.approx(k1 * 2 * case.dx / case.dt * 1.0, rel=1e-12)
    assert jx[8, 10] == pytest.approx(k1 * 0.25 * 2 * case.dx / case.dt, rel=1e-12)


def test_mover_loss_tallies_by_wall_label(oracle_lib):
    """Particles thrown at the walls of the aperture-plate geometry (left wall label 3, plate
    2, other walls 1): p_mac counts each loss under the label of its cell and its v^2."""
    case = configs.case4(ppc=1, nx=64, ny=64)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    cfg = O.make_cfg(case, sp)
    cfg.flag_B = 0
    b = np.ascontiguousarray(case.bcnd, dtype=np.int32)
    i0 = int(round(0.8 * 64)) + 1          # plate's first node
    v = []
    ex = {1: 0, 2: 0, 3: 0}
    v2 = {1: 0.0, 2: 0.0, 3: 0.0}
    rng = np.random.default_rng(4)
    for k in range(300):
        y = (10.3 + rng.random() * 3) * case.dy
        speed = (3.0 + 0.5 * rng.random()) * case.dx / case.dt   # lands inside the 4-cell plate
        kind = k % 4
        if kind == 0:   # into the left wall
            p = (0.2 * case.dx, y, 0, -speed, 0, 0); ex[3] += 1; v2[3] += speed ** 2
        elif kind == 1:  # into the plate's left face
            p = ((i0 - 1.3) * case.dx, y, 0, speed, 0, 0); ex[2] += 1; v2[2] += speed ** 2
        elif kind == 2:  # into the top wall
            p = (20.4 * case.dx, 63.8 * case.dy, 0, 0, speed, 0); ex[1] += 1; v2[1] += speed ** 2
        else:            # stays inside
            p = (30.5 * case.dx, 30.5 * case.dy, 0, 0.1 * case.dx / case.dt, 0, 0)
        v.append(p)
    vxp = np.array(v, dtype=np.float64)
    Ei = np.zeros((case.ny + 3, case.nx + 3, 2))
    n, t = O.mover(cfg, 0, Ei, None, b, vxp)
    assert n == 75 and t.n_lost == 225
    for lab in (1, 2, 3):
        assert t.n_loss[lab] == ex[lab]
        assert t.v2_loss[lab] == pytest.approx(v2[lab], rel=1e-12)
