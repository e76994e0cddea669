"""Known-answer tests that pin the CPU restatement (the oracle) of the reference routines.

The reference has no tests or golden vectors; these pin the restatement to published values
(Park-Miller minimal standard) and to analytic physics (Boris rotation, E x B drift, CIC
charge conservation, discrete Poisson solutions, MCC rate n*sigma*v)."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import configs, deck as dk
from jd_lepic_b200.simulation import species_params


def small_case(nx=32, ny=32, ppc=4):
    return configs.case0(ppc=ppc, nx=nx, ny=ny)


def cfg_for(case):
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    return O.make_cfg(case, sp), sp


def test_ran2_park_miller_minimal_standard(oracle_lib):
    # ran2.f90:1-15 is Park & Miller's minimal standard; from seed 1 the 10000th state is
    # 1043618065 (Park & Miller, CACM 31(10), 1988).
    vals, state = O.ran2_sequence(1, 10000)
    assert state == 1043618065
    assert vals[0] == 16807 / 2147483647


def test_load_gauss_moments(oracle_lib):
    rng = np.random.default_rng(1)
    vt = 3.0
    xs, ys = [], []
    L = O.lib()
    a, b = C.c_double(), C.c_double()
    for _ in range(20000):
        r = (C.c_double * 2)(*rng.random(2))
        L.o_load_gauss(C.byref(a), C.byref(b), vt, r)
        xs.append(a.value)
        ys.append(b.value)
    xs, ys = np.array(xs), np.array(ys)
    # components are normal with sigma = vt/sqrt(2)
    assert abs(xs.mean()) < 0.05 and abs(ys.mean()) < 0.05
    assert abs(xs.std() - vt / math.sqrt(2)) < 0.05
    assert abs(ys.std() - vt / math.sqrt(2)) < 0.05


def _uniform_E(case, ex=0.0, ey=0.0):
    Ei = np.zeros((case.ny + 3, case.nx + 3, 2))
    Ei[..., 0] = ex
    Ei[..., 1] = ey
    return Ei


def test_boris_gyration_angle_and_speed(oracle_lib):
    case = small_case()
    case.flag_B = 1
    case.Bc = (0.0, 0.0, 0.02)
    cfg, sp = cfg_for(case)
    Ei = _uniform_E(case)
    v0 = 1.0e5
    p = np.array([[0.5 * case.nx * case.dx, 0.5 * case.ny * case.dy, 0.0, v0, 0.0, 0.0]])
    k1 = case.dt * sp.charge[0] / (2 * sp.mass[0])
    theta = -2.0 * math.atan(k1 * 0.02)  # Boris rotation per step (q < 0: counter-clockwise)
    for _ in range(50):
        n, _t = O.mover(cfg, 0, Ei, None, case.bcnd, p)
        assert n == 1
    ang = math.atan2(p[0, 4], p[0, 3])
    expect = math.remainder(50 * theta, 2 * math.pi)
    assert abs(math.remainder(ang - expect, 2 * math.pi)) < 1e-9
    assert abs(math.hypot(p[0, 3], p[0, 4]) - v0) / v0 < 1e-12


def test_exb_drift(oracle_lib):
    case = small_case(64, 64)
    case.flag_B = 1
    case.Bc = (0.0, 0.0, 0.05)
    cfg, sp = cfg_for(case)
    ex = 1.0e3
    Ei = _uniform_E(case, ex=ex)
    p = np.array([[0.5 * case.nx * case.dx, 0.5 * case.ny * case.dy, 0.0, 0.0, 0.0, 0.0]])
    y0 = p[0, 1]
    nsteps = 4000
    for _ in range(nsteps):
        O.mover(cfg, 0, Ei, None, case.bcnd, p)
    vd = (p[0, 1] - y0) / (nsteps * case.dt)
    assert abs(vd - (-ex / 0.05)) / (ex / 0.05) < 0.02  # v_E = E x B / B^2


def test_leapfrog_constant_field(oracle_lib):
    case = small_case()
    cfg, sp = cfg_for(case)
    ey = -500.0
    Ei = _uniform_E(case, ey=ey)
    p = np.array([[0.5 * case.nx * case.dx, 0.5 * case.ny * case.dy, 0.0, 0.0, 0.0, 0.0]])
    O.mover(cfg, 0, Ei, None, case.bcnd, p)
    assert abs(p[0, 4] - sp.charge[0] / sp.mass[0] * ey * case.dt) < 1e-9 * abs(p[0, 4])


def test_wall_loss_and_compaction(oracle_lib):
    case = small_case()
    cfg, sp = cfg_for(case)
    Ei = _uniform_E(case)
    L = case.nx * case.dx
    p = np.array([[0.5 * L, 0.5 * L, 0, 0, 0, 0],
                  [0.5 * case.dx, 0.5 * L, 0, -1e8, 0, 0],   # leaves through x = 0
                  [0.3 * L, 0.6 * L, 0, 0, 0, 0]])
    n, t = O.mover(cfg, 0, Ei, None, case.bcnd, p)
    assert n == 2 and t.n_lost == 1
    assert p[1, 0] == pytest.approx(0.3 * L)  # order-preserving compaction


def test_cic_charge_conservation(oracle_lib):
    case = small_case()
    cfg, sp = cfg_for(case)
    rng = np.random.default_rng(3)
    n = 5000
    p = np.zeros((n, 6))
    p[:, 0] = rng.random(n) * case.nx * case.dx
    p[:, 1] = rng.random(n) * case.ny * case.dy
    kq = np.ones((case.ny + 3, case.nx + 3))
    npg = np.zeros_like(kq)
    O.deposit(cfg, 0, p, n, kq, npg)
    total = npg.sum() * case.dx * case.dy * case.zmax / sp.Nm[0]
    assert abs(total - n) < 1e-9 * n


def _manufactured(case):
    nx, ny = case.nx, case.ny
    i = np.arange(nx + 3) - 1
    j = np.arange(ny + 3) - 1
    X, Y = np.meshgrid(i / nx, j / ny)
    u = 3.0 * np.sin(math.pi * X) * np.sin(2 * math.pi * Y) + 2.0 * X
    return u


def _apply_A(cfg, u):
    aw = cfg.eps0 / (cfg.dx * cfg.dx)
    an = cfg.eps0 / (cfg.dy * cfg.dy)
    ac = -(2 * an + 2 * aw)
    return aw * u[1:-1, :-2] + an * u[2:, 1:-1] + an * u[:-2, 1:-1] + aw * u[1:-1, 2:] + ac * u[1:-1, 1:-1]


@pytest.mark.parametrize("n", [32, 64])
def test_mg_manufactured_solution(oracle_lib, n):
    case = small_case(n, n)
    cfg, sp = cfg_for(case)
    ue = _manufactured(case)
    b = _apply_A(cfg, ue)
    phi = np.where(case.bcnd >= 1, ue, 0.0)
    rc, st = O.solve(cfg, phi, b, case.bcnd, case.levels(), 1e-12)
    assert rc == 0
    interior = case.bcnd == -1
    assert np.abs(phi - ue)[interior].max() < 1e-8 * np.abs(ue).max()
    assert O.l2_residual(cfg, phi, b, case.bcnd) < 1e-10


def test_mg_vcycle_contracts(oracle_lib):
    case = small_case(64, 64)
    cfg, sp = cfg_for(case)
    ue = _manufactured(case)
    b = _apply_A(cfg, ue)
    phi = np.where(case.bcnd >= 1, ue, 0.0)
    res = []
    for k in range(4):
        rc, st = O.solve(cfg, phi, b, case.bcnd, case.levels(), 1e-30, ncycl=1)
        res.append(O.l2_residual(cfg, phi, b, case.bcnd))
    assert all(res[k + 1] < 0.3 * res[k] for k in range(3))


def test_sort_stable_by_cell(oracle_lib):
    case = small_case(16, 16)
    cfg, sp = cfg_for(case)
    rng = np.random.default_rng(5)
    n = 3000
    p = np.zeros((n, 6))
    p[:, 0] = rng.random(n) * case.nx * case.dx
    p[:, 1] = rng.random(n) * case.ny * case.dy
    p[:, 3] = np.arange(n)  # original index as a tag
    pl = O.sort(cfg, p, n)
    ic = (p[:, 0] / case.dx).astype(int) + case.nx * (p[:, 1] / case.dy).astype(int)
    assert np.all(np.diff(ic) >= 0)
    for c in np.unique(ic):  # stable inside each cell
        assert np.all(np.diff(p[ic == c, 3]) > 0)
    counts = np.bincount(ic, minlength=case.nx * case.ny)
    assert np.array_equal(pl[1:case.nx * case.ny + 1], np.cumsum(counts))


def test_indexx_ascending(oracle_lib):
    rng = np.random.default_rng(7)
    for n in (1, 3, 7, 8, 20, 60):
        a = rng.random(n)
        idx = (C.c_int * n)()
        O.lib().o_indexx(n, O.dp(a), idx)
        assert list(idx) == list(np.argsort(a))


def test_mcc_rate_constant_cross_section(oracle_lib):
    """Null-collision MCC with a constant elastic cross section: the number of real collisions
    per call is N * n_gas * sigma * v * ns_coll * dt (collisions.f90)."""
    case = small_case(16, 16)
    E = dk.energy_grid(1e3, 50)
    text = dk.write_deck("[Ar+]", 39.95, 0.03, "[Ar]", 0.0258,
                         [("[e]+[Ar]->[e]+[Ar]", "COLLISION", 0.0, E, dk.sigma_constant(E, 1e-19))])
    case.deck_text = text
    n = 200000
    v = 2.0e6
    p = np.zeros((n, 6))
    rng = np.random.default_rng(11)
    p[:, 0] = rng.random(n) * case.nx * case.dx
    p[:, 1] = rng.random(n) * case.ny * case.dy
    p[:, 3] = v
    sim = O.OracleSimulation(case, particles={0: p, 1: p[:10].copy()}, seed=1)
    t = sim.collide()
    nu = case.ngas * 1e-19 * v  # neutral velocity is negligible against v
    expect = n * nu * 10 * case.dt
    got = t.n_coll[0]
    assert abs(got - expect) < 5 * math.sqrt(expect)


def test_oracle_dsmc_pairs_conserve_and_targets_come_from_the_cell():
    """o_collisions_dsmc on electron-ion elastic scattering (a charged target): every collision
    changes one electron and one ion of the electron's cell (or a neighbour), and the pair
    keeps its momentum and kinetic energy."""
    import math
    from jd_lepic_b200 import configs, deck as dk
    from jd_lepic_b200.simulation import species_params
    from oracle import oracle as O
    case = configs.case0(ppc=100, nx=32, ny=32)
    case.deck_text = dk.argon_dsmc_deck()
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    cfg = O.make_cfg(case, sp)
    xsh = O.XsHolder(dk.ordering(d))
    rng = np.random.default_rng(5)
    n = case.n_particles
    parts = []
    for s in (0, 1):
        p = np.zeros((n, 6))
        p[:, 0] = rng.uniform(0, case.nx * case.dx, n)
        p[:, 1] = rng.uniform(0, case.ny * case.dy, n)
        p[:, 3:] = rng.normal(0, sp.vt0[s] / math.sqrt(2), (n, 3))
        parts.append(p)
    plist = O.sort(cfg, parts[1], n)
    kq = O.kq_of(case.bcnd)
    npg = np.zeros((2, case.ny + 3, case.nx + 3))
    for s in (0, 1):
        O.deposit(cfg, s, parts[s], n, kq, npg[s])
    red, mx = O.dens_red(cfg, npg, case.bcnd)
    cfg.np_mx[1] = mx[1]
    rc, out, tal, _ = O.collisions(cfg, xsh, parts, seed=3, plists={1: plist}, np_red=red)
    assert rc == 0
    nc = tal.n_coll[0]
    assert nc > 50 and tal.n_add[0] == tal.n_add[1] == 0
    ce = np.flatnonzero(np.any(out[0][:, 3:] != parts[0][:, 3:], axis=1))
    ci = np.flatnonzero(np.any(out[1][:, 3:] != parts[1][:, 3:], axis=1))
    # picks with replacement can hit one particle twice: a few changed particles fewer
    assert nc - 3 <= ce.size <= nc and nc - 3 <= ci.size <= nc
    dP = sp.mass[0] * (out[0][:, 3:] - parts[0][:, 3:]).sum(axis=0) + \
        sp.mass[1] * (out[1][:, 3:] - parts[1][:, 3:]).sum(axis=0)
    pe = sp.mass[0] * np.linalg.norm(parts[0][ce, 3:], axis=1).sum()
    assert np.abs(dP).max() <= 1e-9 * pe
    dE = sum(0.5 * sp.mass[s] * ((out[s][:, 3:] ** 2).sum() - (parts[s][:, 3:] ** 2).sum()) for s in (0, 1))
    Ee = 0.5 * sp.mass[0] * (parts[0][ce, 3:] ** 2).sum()
    assert abs(dE) <= 1e-9 * Ee
    # each changed ion sits in the cell of some changed electron or next to it
    cell = lambda p: ((p[:, 0] / case.dx).astype(int), (p[:, 1] / case.dy).astype(int))
    ex, ey = cell(out[0][ce])
    ix, iy = cell(out[1][ci])
    near = np.zeros(ci.size, dtype=bool)
    for k in range(ci.size):
        near[k] = np.any(np.abs(ex - ix[k]) + np.abs(ey - iy[k]) <= 1) or np.any((ey == iy[k] + 1) | (ey == iy[k] - 1))
    assert near.all()


def test_oracle_third_dimension_model():
    """o_part_mover_z (part_expmover.f90:269-309): an electron crossing an end plate with more
    z-energy than phi - phi0 is lost, with less it is reflected to 0.02 / 0.98 zmax with vz
    reversed; ions are lost at the rate hz 2 uB / zmax dt."""
    import math
    from jd_lepic_b200 import configs, deck as dk
    from jd_lepic_b200.simulation import species_params
    from oracle import oracle as O
    case = configs.case0(ppc=1, nx=16, ny=16)
    case.zmax = 0.01
    sp = species_params(case, dk.read_reactions(case.deck_text, case.ngas))
    cfg = O.make_cfg(case, sp)
    E = np.zeros((case.ny + 3, case.nx + 3, 2))
    phi = np.full((case.ny + 3, case.nx + 3), 5.0)
    me = sp.mass[0]
    v = lambda eV: math.sqrt(2 * eV * dk.QE / me)
    p = np.zeros((4, 6))
    p[:, 0] = p[:, 1] = 8.3 * case.dx
    p[0, 2], p[0, 5] = 1e-9, -v(7.0)                # 7 eV >= 5 - (-1): lost
    p[1, 2], p[1, 5] = 1e-9, -v(5.0)                # 5 eV < 6: reflected at 0.02 zmax
    p[2, 2], p[2, 5] = case.zmax - 1e-9, v(3.0)     # reflected at 0.98 zmax
    p[3, 2], p[3, 5] = 0.5 * case.zmax, v(50.0)     # stays inside
    n, t = O.mover_z(cfg, 0, E, None, case.bcnd, p, phi, -1.0, np.zeros((17, 17), np.float32), 16, 1, 1.0, 1, 1)
    assert n == 3 and t.n_loss[0] == 1
    assert p[0, 2] == pytest.approx(0.02 * case.zmax) and p[0, 5] == pytest.approx(v(5.0))
    assert p[1, 2] == pytest.approx(0.98 * case.zmax) and p[1, 5] == pytest.approx(-v(3.0))
    assert p[2, 2] == pytest.approx(0.5 * case.zmax + case.dt * v(50.0))
    assert t.P1z == pytest.approx(sp.Nm[0] * sp.charge[0] * 5.0)
    rng = np.random.default_rng(1)
    m = 20000
    ions = np.zeros((m, 6))
    ions[:, 0] = rng.uniform(1, 15, m) * case.dx
    ions[:, 1] = rng.uniform(1, 15, m) * case.dy
    ions[:, 2] = 0.5 * case.zmax
    uB = np.full((17, 17), 3000.0, np.float32)
    hz = 5e4
    n, _ = O.mover_z(cfg, 1, E, None, case.bcnd, ions, phi, 0.0, uB, 16, 1, hz, 1, 3)
    expect = m * hz * 2 * 3000.0 / case.zmax * case.dt
    assert abs((m - n) - expect) < 5 * math.sqrt(expect)


def test_oracle_dielectric_charging():
    """o_part_mover_zd / o_dielectric_update (part_expmover.f90:340-350, main.f90:756-809): an
    electron lost in the left wall at y = (iy - 0.25) h leaves 0.25 Nm q on row iy and 0.75 on
    row iy+1 of the wall's label; the update adds kd dq / (Ca dy) to that label's wall nodes of
    rows 2..ny (kd = 2 on rows 1 and ny+1) and clears dq.  A conductor label collects nothing."""
    case = configs.case0(ppc=1, nx=16, ny=16)
    case.bcnd = configs.box_mask(16, 16, label_left=2, label_right=3)
    cfg, sp = cfg_for(case)
    E = np.zeros((case.ny + 3, case.nx + 3, 2))
    dtype = np.zeros(16, np.int32)
    dtype[2] = 1
    p = np.zeros((3, 6))
    p[0, 0], p[0, 1], p[0, 3] = 0.5 * case.dx, 6.75 * case.dy, -1.0 * case.dx / case.dt  # -> x < 0: cell ix 0
    p[1, 0], p[1, 1], p[1, 3] = (case.nx - 0.5) * case.dx, 5.5 * case.dy, case.dx / case.dt  # right: a conductor
    p[2, 0], p[2, 1] = 8.0 * case.dx, 8.0 * case.dy                                          # stays
    n, t, dq = O.mover_dielec(cfg, 0, E, None, case.bcnd, p, dtype)
    nmq = sp.Nm[0] * sp.charge[0]
    assert n == 1 and t.n_lost == 2
    iy = 7                                           # floor(6.75) + 1
    assert dq[2, iy] == pytest.approx(0.25 * nmq) and dq[2, iy + 1] == pytest.approx(0.75 * nmq)
    assert np.count_nonzero(dq) == 2
    phi = np.zeros((case.ny + 3, case.nx + 3))
    Ca = 1e-7
    O.dielectric_update(cfg, phi, case.bcnd, dtype, dq, Ca)
    assert not dq.any()
    col = phi[:, 0]
    assert col[iy] == pytest.approx(0.25 * nmq / (Ca * case.dy))
    assert col[iy + 1] == pytest.approx(0.75 * nmq / (Ca * case.dy))
    assert np.count_nonzero(phi) == 4                # columns 0 and 1 of label 2, two rows
    # a loss on row 1 (the half cell) doubles, but the row lies outside 2..ny: nothing moves
    dq[2, 1] = nmq
    O.dielectric_update(cfg, phi, case.bcnd, dtype, dq, Ca)
    assert np.count_nonzero(phi) == 4
