"""CUDA path vs the CPU FP64 restatement (the oracle), through the C ABI.

Tolerances (stated per test):
  push      positions within 1e-6 * dx, velocities within 1e-6 * |v| (plus 1e-6 * vth),
            of the FP64 Boris/leap-frog oracle given the same particles and field
  deposit   charge density within 1e-12 of its maximum, against the oracle's FP64 deposition
            of the GPU's own (fixed-point) positions
  E field   bit-identical to the oracle (FP64, no FMA contraction on either side)
  rhs       bit-identical given the same np grids
  MG FP64   same V-cycle and sweep counts; phi identical to 1e-13 relative (normally exact)
  MG mixed  ||b - A u||_2 / ||b - A u_D||_2 <= 1e-8 measured in FP64 on the CPU
  sort      reference order: particle order and Plist identical (integer work, exact)
"""
import math

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def sim_for(case, tile=(8, 8), **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=tile, **kw)


def smooth_phi(case, amp=40.0):
    nx, ny = case.nx, case.ny
    i = np.arange(nx + 3) - 1
    j = np.arange(ny + 3) - 1
    X, Y = np.meshgrid(i / nx, j / ny)
    phi = amp * np.sin(math.pi * X) * np.sin(math.pi * Y) * (1 + 0.3 * np.cos(5 * X + 3 * Y))
    return np.where(case.bcnd >= 1, case.phi0, phi)


@pytest.fixture(scope="module")
def small():
    return configs.case0(ppc=20, nx=64, ny=64)


def oracle_cfg(case, sim):
    return O.make_cfg(case, sim.sp)


def assert_push_matches(case, sim, cfg, sp, E, p0, got, max_unpaired=2):
    """The device's survivors against the FP64 oracle's, particle by particle: both keep the
    initial order (part_expmover.f90:496-503), so they are aligned and every particle that both
    keep is compared; at most max_unpaired particles (within a rounding distance of a wall
    cell) may be lost on one side only.  Returns the number of compared particles."""
    ref, _, _ = O.mover_tagged(cfg, sp, E, case.Bi, case.bcnd, p0)
    gi, rj, g_only, r_only = O.align_survivors(got, ref, case.dx, case.dy)
    assert g_only + r_only <= max_unpaired, (g_only, r_only)
    assert gi.size == got.shape[0] - g_only and rj.size == ref.shape[0] - r_only
    vth = sim.sp.vt0[sp]
    dpos = np.abs(got[gi, :2] - ref[rj, :2]).max() if gi.size else 0.0
    vmag = np.linalg.norm(ref[rj, 3:], axis=1)
    dvel = (np.linalg.norm(got[gi, 3:] - ref[rj, 3:], axis=1) / (vmag + vth)).max() if gi.size else 0.0
    assert dpos <= 1e-6 * case.dx, dpos / case.dx
    assert dvel <= 1e-6, dvel
    return gi.size


def test_smoke_create_load_step(gpu_lib, small):
    s = sim_for(small)
    st0 = s.push_stats()
    assert st0["np_tot"] == [small.n_particles] * 2
    for it in range(1, 4):
        s.step(it)
    s.sync()
    st = s.push_stats()
    assert all(st["np_tot"][k] + st["n_lost"][k] == small.n_particles for k in range(2))
    s.close()


@pytest.mark.parametrize("bmode", [0, 1, 2])
def test_push_and_deposit_match_oracle(gpu_lib, bmode):
    case = configs.case0(ppc=20, nx=64, ny=64)
    if bmode == 1:
        case.flag_B, case.Bc = 1, (0.003, -0.002, 0.02)
    elif bmode == 2:
        case.flag_B = 2
        case.Bi = configs.dipole_field(case.nx, case.ny, case.dx, case.dy, bmax=0.05, bz=0.01)
    s = sim_for(case)
    s.set_phi(smooth_phi(case))
    E = s.efield()
    s.sort(0)
    s.sort(1)  # exercises the tiled shared-memory deposit window
    cfg = oracle_cfg(case, s)
    dx = case.dx
    p0 = [s.get_particles(k) for k in range(2)]
    s.push(1)
    p_all = [s.get_particles(k) for k in range(2)]
    for sp in range(2):
        assert assert_push_matches(case, s, cfg, sp, E, p0[sp], p_all[sp]) >= p0[sp].shape[0] - 2000
    # deposit: oracle FP64 CIC of the GPU's post-push positions vs the GPU's np grids
    kq = O.kq_of(case.bcnd)
    for sp in range(2):
        p = p_all[sp]
        npg = np.zeros((case.ny + 3, case.nx + 3))
        O.deposit(cfg, sp, p, p.shape[0], kq, npg)
        g = s.grid(capi.GRID_NP + sp)
        assert np.abs(g - npg).max() <= 1e-12 * np.abs(npg).max()
    s.close()


@pytest.mark.parametrize("nx", [1024, 2048])
def test_push_and_deposit_large_grid(gpu_lib, nx):
    """Grids of 1024 and up (S <= 22) deposit through per-run moments: exact integer weights,
    so the density must equal the oracle's FP64 CIC to 1e-12 and be bit-reproducible."""
    case = configs.case0(ppc=1, nx=nx, ny=nx)
    case.flag_B, case.Bc = 1, (0.0, 0.0, 0.005)
    grids = []
    for rep in range(2):
        s = sim_for(case, tile=(16, 16))
        s.set_phi(smooth_phi(case))
        E = s.efield()
        s.sort(0)
        s.sort(1)
        cfg = oracle_cfg(case, s)
        p0 = [s.get_particles(k) for k in range(2)]
        s.push(1)
        p_all = [s.get_particles(k) for k in range(2)]
        grids.append([s.grid(capi.GRID_NP + k) for k in range(2)])
        if rep == 0:
            kq = O.kq_of(case.bcnd)
            for sp in range(2):
                got = p_all[sp]
                assert_push_matches(case, s, cfg, sp, E, p0[sp], got)
                npg = np.zeros((case.ny + 3, case.nx + 3))
                O.deposit(cfg, sp, got, got.shape[0], kq, npg)
                assert np.abs(grids[0][sp] - npg).max() <= 1e-12 * np.abs(npg).max()
        s.close()
    for k in range(2):
        assert np.array_equal(grids[0][k], grids[1][k])


def test_push_and_deposit_cfg0_full_size(gpu_lib):
    """The 128x128 Ar box at its full 100 particles per cell (1.64 M per species), one push from
    a structured potential: every particle both sides keep is compared with the FP64 oracle,
    and the density with the oracle's FP64 deposition of the device's positions."""
    case = configs.case0()
    assert case.nx == 128 and case.n_particles == 1638400
    s = sim_for(case, tile=(16, 16))
    try:
        s.set_phi(smooth_phi(case))
        E = s.efield()
        s.sort(0)
        s.sort(1)
        cfg = oracle_cfg(case, s)
        p0 = [s.get_particles(k) for k in range(2)]
        s.push(1)
        kq = O.kq_of(case.bcnd)
        for sp in range(2):
            got = s.get_particles(sp)
            n_cmp = assert_push_matches(case, s, cfg, sp, E, p0[sp], got)
            assert n_cmp >= 0.9 * p0[sp].shape[0]
            npg = np.zeros((case.ny + 3, case.nx + 3))
            O.deposit(cfg, sp, got, got.shape[0], kq, npg)
            g = s.grid(capi.GRID_NP + sp)
            assert np.abs(g - npg).max() <= 1e-12 * np.abs(npg).max()
    finally:
        s.close()


def test_deposit_bit_reproducible(gpu_lib, small):
    grids = []
    for _ in range(2):
        s = sim_for(small)
        s.set_phi(smooth_phi(small))
        for it in range(1, 6):
            s.step(it)
        grids.append([s.grid(capi.GRID_NP + k) for k in range(2)])
        s.close()
    for k in range(2):
        assert np.array_equal(grids[0][k], grids[1][k])


def test_efield_bit_exact(gpu_lib, small):
    s = sim_for(small)
    phi = smooth_phi(small)
    s.set_phi(phi)
    E = s.efield()
    cfg = oracle_cfg(small, s)
    Eref = O.efield(cfg, phi, small.bcnd)
    assert np.array_equal(E, Eref)
    s.close()


def test_calc_rhs_bit_exact(gpu_lib, small):
    s = sim_for(small)
    rhs = s.calc_rhs()
    cfg = oracle_cfg(small, s)
    npg = np.stack([s.grid(capi.GRID_NP + k) for k in range(2)])
    ref = O.calc_rhs(cfg, npg)
    assert np.array_equal(rhs, ref)
    s.close()


def set_rhs(s, rhs):
    import ctypes as C
    a = np.ascontiguousarray(rhs)
    s.check(s.lib.lepic_gpu_set_grid(s.ctx, capi.GRID_RHS, a.ctypes.data_as(C.POINTER(C.c_double))), "set_grid")


def _perturbed_rhs(s, case):
    """A charge density with structure: the loaded density plus an imposed imbalance."""
    rhs = s.calc_rhs()
    i = np.arange(case.nx + 1)
    j = np.arange(case.ny + 1)
    X, Y = np.meshgrid(i / case.nx, j / case.ny)
    return rhs + 1.6e-3 * np.sin(3 * math.pi * X) * np.sin(2 * math.pi * Y)


@pytest.mark.parametrize("n,eps", [(64, 1e-10), (128, 1e-8)])
def test_mg_fp64_matches_oracle(gpu_lib, n, eps):
    case = configs.case0(ppc=4, nx=n, ny=n)
    s = sim_for(case)
    rhs = _perturbed_rhs(s, case)
    set_rhs(s, rhs)
    phi0 = case.phi0.copy()
    st = s.solve(eps=eps, mode=capi.POISSON_FP64_MG, phi=phi0)
    cfg = oracle_cfg(case, s)
    ref = case.phi0.copy()
    rc, ost = O.solve(cfg, ref, rhs, case.bcnd, case.levels(), eps)
    assert rc == 0
    assert st["cycles"] == ost.k
    assert st["sweeps_fine"] == ost.sweeps_fine
    assert np.abs(st["phi"] - ref).max() <= 1e-13 * np.abs(ref).max()
    assert abs(st["res_l1"] - ost.res) <= 1e-9 * ost.res + 1e-300
    s.close()


@pytest.mark.parametrize("mode", [capi.POISSON_MIXED_IR, capi.POISSON_FP64_PCG])
@pytest.mark.parametrize("idx,n", [(2, 64), (2, 256), (4, 256), (4, 512)])
def test_mg_mixed_precision_reaches_1e8(gpu_lib, idx, n, mode):
    case = configs.case2(ppc=2, nx=n, ny=n // 2) if idx == 2 else configs.case4(ppc=2, nx=n, ny=n)
    s = sim_for(case)
    rhs = _perturbed_rhs(s, case)
    set_rhs(s, rhs)
    phi0 = case.phi0.copy()
    st = s.solve(eps=1e-8, mode=mode, phi=phi0)
    cfg = oracle_cfg(case, s)
    res = O.l2_residual(cfg, st["phi"], rhs, case.bcnd)
    assert res <= 1e-8, res
    assert st["res_l2_rel"] <= 1e-8
    # same discrete solution as the FP64 solver: the oracle's where it finishes in seconds,
    # else the GPU FP64 V-cycle (itself checked against the oracle above) driven to 1e-12
    if n <= 256:
        ref = case.phi0.copy()
        O.solve(cfg, ref, rhs, case.bcnd, case.levels(), 1e-13)
    else:
        ref = s.solve(eps=1e-12, mode=capi.POISSON_FP64_MG_L2, phi=case.phi0.copy())["phi"]
    assert np.abs(st["phi"] - ref).max() <= 1e-5 * np.abs(ref).max()
    s.close()


def test_warm_start_extrapolation(gpu_lib):
    """lepic_gpu_set_warm_start(1): a rhs that changes linearly from step to step has a linear
    solution, so 2 phi_(n-1) - phi_(n-2) is almost the answer: fewer CG iterations than from
    phi_(n-1), the same tolerance on the true residual and the same potential."""
    case = configs.case4(ppc=2, nx=256, ny=256)
    s = sim_for(case)
    try:
        cfg = oracle_cfg(case, s)
        base = _perturbed_rhs(s, case)
        i = np.arange(case.nx + 1)
        j = np.arange(case.ny + 1)
        X, Y = np.meshgrid(i / case.nx, j / case.ny)
        step = 2.0e-4 * np.sin(math.pi * X) * np.sin(2 * math.pi * Y)
        s.check(s.lib.lepic_gpu_set_warm_start(s.ctx, 1), "set_warm_start")
        phis, cyc = [], []
        for n in range(5):
            set_rhs(s, base + n * step)
            st = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR)   # from the device's last solution
            assert st["res_l2_rel"] <= 1e-8
            cyc.append(st["cycles"])
            phis.append(s.grid(capi.GRID_PHI))
        assert O.l2_residual(cfg, phis[4], base + 4 * step, case.bcnd) <= 1e-8
        # the last step again, from phi_3 as it is
        s.check(s.lib.lepic_gpu_set_warm_start(s.ctx, 0), "set_warm_start")
        s.set_phi(phis[3])
        st = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR)
        assert st["res_l2_rel"] <= 1e-8
        assert cyc[4] < st["cycles"], (cyc, st["cycles"])
        plain = s.grid(capi.GRID_PHI)
        assert np.abs(phis[4] - plain).max() <= 1e-5 * np.abs(plain).max()
    finally:
        s.close()


def test_sort_reference_order_exact(gpu_lib):
    case = configs.case0(ppc=20, nx=64, ny=64)
    s = sim_for(case, tile=None)  # the reference's row-major cell order
    s.set_phi(smooth_phi(case))
    s.efield()
    for it in range(2, 6):  # unsort by moving without sorting
        s.push(it)
    for sp in range(2):
        p0 = s.get_particles(sp)
        pl = s.sort(sp, plist=True)
        got = s.get_particles(sp)
        ref = p0.copy()
        cfg = oracle_cfg(case, s)
        pref = O.sort(cfg, ref, ref.shape[0])
        assert np.array_equal(got, ref)
        assert np.array_equal(pl, pref)
    s.close()


def test_sort_tiled_groups_cells(gpu_lib, small):
    s = sim_for(small, tile=(8, 8))
    s.set_phi(smooth_phi(small))
    s.efield()
    for it in range(2, 6):
        s.push(it)
    p0 = s.get_particles(0)
    s.sort(0)
    p1 = s.get_particles(0)
    assert p1.shape == p0.shape
    # same multiset of particles
    a = p0[np.lexsort(p0.T[::-1])]
    b = p1[np.lexsort(p1.T[::-1])]
    assert np.array_equal(a, b)
    cx = (p1[:, 0] / small.dx).astype(int)
    cy = (p1[:, 1] / small.dy).astype(int)
    key = ((cy // 8) * (small.nx // 8) + cx // 8) * 64 + (cy % 8) * 8 + (cx % 8)
    assert np.all(np.diff(key) >= 0)
    s.close()


def test_mcc_rate_matches_n_sigma_v(gpu_lib):
    from jd_lepic_b200 import deck as dk
    case = configs.case0(ppc=50, nx=64, ny=64)
    E = dk.energy_grid(1e3, 50)
    case.deck_text = dk.write_deck("[Ar+]", 39.95, 0.03, "[Ar]", 0.0258,
                                   [("[e]+[Ar]->[e]+[Ar]", "COLLISION", 0.0, E, dk.sigma_constant(E, 1e-19))])
    s = sim_for(case)
    n = case.n_particles
    v = 2.0e6
    p = s.get_particles(0)
    p[:, 3:] = 0.0
    p[:, 3] = v
    s.put_particles(0, p)
    st = s.collide(11)
    nu = case.ngas * 1e-19 * v
    expect = n * nu * 10 * case.dt
    got = st["n_coll"][0]
    assert abs(got - expect) < 5 * math.sqrt(expect), (got, expect)
    # elastic scattering conserves the electron speed up to the neutral's recoil (m/M ~ 1e-5)
    q = s.get_particles(0)
    sp = np.linalg.norm(q[:, 3:], axis=1)
    assert np.abs(sp / v - 1).max() < 2e-3
    s.close()


def test_ionization_creates_pairs(gpu_lib):
    case = configs.case0(ppc=20, nx=64, ny=64)
    s = sim_for(case)
    p = s.get_particles(0)
    # 100 eV electrons ionise readily
    v = math.sqrt(2 * 100 * 1.602e-19 / 9.109e-31)
    p[:, 3:] = 0.0
    p[:, 4] = v
    s.put_particles(0, p)
    n_e0 = p.shape[0]
    n_i0 = s.push_stats()["np_tot"][1]
    st = s.collide(11)
    ion_reaction = 2
    nion = st["n_coll"][ion_reaction]
    assert nion > 0
    ps = s.push_stats()
    assert ps["np_tot"][0] == n_e0 + nion
    assert ps["np_tot"][1] == n_i0 + nion
    # the new electrons and ions sit at the parent's position
    e = s.get_particles(0)[n_e0:]
    assert e.shape[0] == nion
    s.close()


def test_capacity_error_is_reported(gpu_lib):
    case = configs.case0(ppc=2, nx=32, ny=32)
    s = sim_for(case, capacity=case.n_particles + 10)
    p = np.zeros((case.n_particles + 11, 6))
    p[:, 0] = 0.5 * case.nx * case.dx
    p[:, 1] = 0.5 * case.ny * case.dy
    with pytest.raises(capi.LepicError) as e:
        s.put_particles(0, p)
    assert e.value.code == capi.ECAPACITY
    s.step(1)  # the context stays usable
    s.sync()
    s.close()


@pytest.mark.parametrize("idx", [1, 2, 3, 4])
def test_config_shapes_run(gpu_lib, idx):
    kw = {1: dict(ppc=4, nx=128, ny=128, steps=12), 2: dict(ppc=4, nx=128, ny=64, steps=12),
          3: dict(ppc=4, nx=128, ny=128, steps=12), 4: dict(ppc=4, nx=256, ny=256, steps=12)}[idx]
    case = configs.make_case(idx, **kw)
    s = sim_for(case, tile=(16, 16))
    s.run(12)
    st = s.push_stats()
    assert all(x > 0 for x in st["np_tot"])
    mc = s.mcc_stats()
    assert mc["n_cand"][0] > 0
    s.close()


@pytest.mark.parametrize("mode", [capi.POISSON_MIXED_IR, capi.POISSON_FP64_PCG])
@pytest.mark.parametrize("idx,n", [(4, 512), (2, 256), (4, 2048)])
def test_mixed_tiled_smoother_matches_grid_sweeps(gpu_lib, monkeypatch, idx, n, mode):
    """The shared-memory tiles of the mixed solver's V-cycle (all half-sweeps of a stage on a
    tile plus halo, then the restriction / after the prolongation) give exactly the values of
    the grid-wide half-sweeps: same iterations, bit-identical potential.  At 2048^2 every CTA
    handles several tiles, so a tile reading a neighbour's finished values would show here."""
    case = configs.case2(ppc=2, nx=n, ny=n // 2) if idx == 2 else configs.case4(ppc=2, nx=n, ny=n)
    s = sim_for(case)
    rhs = _perturbed_rhs(s, case)
    set_rhs(s, rhs)
    tiled = s.solve(eps=1e-8, mode=mode, phi=case.phi0.copy())
    s.set_options(mx_tiled=0)
    grid = s.solve(eps=1e-8, mode=mode, phi=case.phi0.copy())
    assert tiled["cycles"] == grid["cycles"]
    assert np.array_equal(tiled["phi"], grid["phi"])
    s.close()


def test_push_fast_particles_through_the_queues(gpu_lib):
    """Particles that leave their cell every step (1-3 cells per step), unsorted and sorted, so
    that every particle takes the push's cell-change path: every particle both sides keep still
    matches the FP64 oracle, and the density its FP64 deposition."""
    case = configs.case0(ppc=4, nx=64, ny=64)
    s = sim_for(case, capacity=200000)
    try:
        rng = np.random.default_rng(11)
        n = 120000
        p = np.zeros((n, 6))
        p[:, 0] = rng.uniform(0.05, 0.95, n) * case.nx * case.dx
        p[:, 1] = rng.uniform(0.05, 0.95, n) * case.ny * case.dy
        v = rng.uniform(1.0, 3.0, n) * case.dx / case.dt
        th = rng.uniform(0, 2 * math.pi, n)
        p[:, 3], p[:, 4] = v * np.cos(th), v * np.sin(th)
        p[:, 5] = rng.normal(0, 1e5, n)
        s.put_particles(0, p)
        s.set_phi(smooth_phi(case))
        E = s.efield()
        cfg = oracle_cfg(case, s)
        kq = O.kq_of(case.bcnd)
        for it, sort_first in ((1, False), (2, True)):
            if sort_first:
                s.sort(0)
            p0 = s.get_particles(0)
            s.push(it)
            got = s.get_particles(0)
            assert assert_push_matches(case, s, cfg, 0, E, p0, got) > 0.8 * p0.shape[0]
            npg = np.zeros((case.ny + 3, case.nx + 3))
            O.deposit(cfg, 0, got, got.shape[0], kq, npg)
            assert np.abs(s.grid(capi.GRID_NP + 0) - npg).max() <= 1e-12 * np.abs(npg).max()
    finally:
        s.close()


@pytest.mark.parametrize("direct", [0, 1])
def test_mixed_coarse_solve_both_ways(gpu_lib, direct):
    """The mixed cycle's on-chip levels either solved exactly through the precomputed inverse of
    their top level (the default) or cycled by CTA 0: both preconditioners are symmetric, both
    solves reach 1e-8 on the true FP64 residual and give the FP64 multigrid's potential."""
    case = configs.case4(ppc=2, nx=512, ny=512)
    s = sim_for(case)
    try:
        s.set_options(mx_coarse_direct=direct)
        rhs = _perturbed_rhs(s, case)
        set_rhs(s, rhs)
        st = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR, phi=case.phi0.copy())
        cfg = oracle_cfg(case, s)
        assert O.l2_residual(cfg, st["phi"], rhs, case.bcnd) <= 1e-8
        ref = s.solve(eps=1e-12, mode=capi.POISSON_FP64_MG_L2, phi=case.phi0.copy())["phi"]
        assert np.abs(st["phi"] - ref).max() <= 1e-5 * np.abs(ref).max()
    finally:
        s.close()
