"""Particle sources on the B200 through the C ABI, against the CPU restatement.

eheating and part_injection draw from counter-based streams, and the oracle's _ctr form
draws the same numbers, so the check is particle by particle: the set of heated electrons,
the injected counts and cells are exact; velocities are FP32 and agree to the last bit except
where the device's and the C library's log/sincos round differently (bounded by 1e-6
relative); the FP64 power tallies agree to 1e-9 relative (summation order differs); the
charge density including the injected particles agrees to 1e-12 relative of its maximum."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import _capi as capi, configs, deck as dk
from jd_lepic_b200 import sources as S
from jd_lepic_b200.simulation import GpuSimulation, species_params

pytestmark = pytest.mark.gpu

NX = 64


def make_case(plate=False):
    case = configs.case0(ppc=4, nx=NX, ny=NX)
    if plate:
        b = np.array(case.bcnd, dtype=np.int32, copy=True)
        b[20:41, 16:25] = 1              # an embedded wall plate inside the source region
        case.bcnd = b
        case.phi0 = configs.potentials(b, {1: 0.0})
    return case


def oracle_cfg(case):
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    return O.make_cfg(case, sp), sp


def shift_of(sim):
    s = C.c_int32()
    sim.check(sim.lib.lepic_gpu_particle_arrays(sim.ctx, 0, None, None, None, None, None, None, C.byref(s)),
              "particle_arrays")
    return s.value


def rand_particles(case, n, seed, vscale):
    rng = np.random.default_rng(seed)
    v = np.zeros((n, 6))
    v[:, 0] = rng.random(n) * case.nx * case.dx * 0.999
    v[:, 1] = rng.random(n) * case.ny * case.dy * 0.999
    v[:, 3:] = rng.normal(0.0, vscale, (n, 3)).astype(np.float32)
    return v


def vt_used(sc, sp):
    vt = np.zeros(capi.MAXICP)
    if sc.flag_inj:
        vt[:] = sp.vt0[0]
    else:
        vt[:sc.n_icp] = list(sc.vt)[:sc.n_icp]
    return vt


def float_match(a, b):
    """FP32 velocities: identical except for rare last-bit differences of log/sincos."""
    a32 = a.astype(np.float32)
    same = (a32 == b).all(axis=1)
    assert same.mean() > 0.999, same.mean()
    np.testing.assert_allclose(b, a32, rtol=1e-6, atol=0)


HEAT_CASES = [
    dict(heat_region_cm=(0.16, 0.48, 0.08, 0.56), nu_h=2.0e10, I_inj=-1.0, n_icp=1),
    dict(heat_region_cm=(-0.16, -0.48, 0, 0), nu_h=2.0e9, Pabs=(100.0,), opt_inj=-1, I_inj=-1.0),
    dict(heat_region_cm=(0.08, 0.56, 0.0, 0.64), nu_h=2.0e10, I_inj=-1.0, n_icp=3,
         vt=(5.0e5, 1.0e6, 2.0e6), eheat_type=2),
    dict(heat_region_cm=(0.16, 0.48, 0.08, 0.56), nu_h=2.0e10, I_inj=10.0, opt_inj=1),
]


@pytest.mark.parametrize("kw", HEAT_CASES)
def test_eheating_matches_oracle(gpu_lib, kw):
    kw = dict(kw)
    etype = kw.pop("eheat_type", 1)
    case = make_case()
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=400000)
    try:
        sim.put_particles(0, rand_particles(case, 300000, 1, 1.0e6))
        sc = S.source_config(S.SourceDeck(**kw), case.dt, sp.vt0[0])
        sc.eheat_type = etype
        sim.set_sources(sc)
        p0 = sim.get_particles(0)
        sim.eheating(8)
        p1 = sim.get_particles(0)
        t = sim.source_tallies()
        o = p0.copy()
        P, nh = O.eheating(cfg, O.make_src(sc), o, vt_used(sc, sp), seed=sc.seed, it=8)
        assert nh > 1000 and t["n_heated"] == nh and t["n_heat_calls"] == 1
        dev_changed = np.any(p1[:, 3:] != p0[:, 3:], axis=1)
        ora_changed = np.any(o[:, 3:] != p0[:, 3:], axis=1)
        assert np.array_equal(dev_changed, ora_changed)
        assert np.array_equal(p1[:, :2], p0[:, :2])
        float_match(o[:, 3:], p1[:, 3:])
        assert t["P_heat"] == pytest.approx(P, rel=1e-9)
    finally:
        sim.close()


def test_heating_tally_and_temperature_update(gpu_lib):
    case = make_case()
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=300000)
    try:
        sim.put_particles(0, rand_particles(case, 200000, 2, 1.0e6))
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.08, 0.5, 0.0, 0.64), nu_h=1.0e9, n_icp=2,
                                          Pabs=(50.0, 80.0), I_inj=-1.0), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        sim.heating_tally()
        t = sim.source_tallies()
        Nh, E = O.heat_tally(cfg, O.make_src(sc), sim.get_particles(0))
        assert t["Nh"] == list(Nh)
        np.testing.assert_allclose(t["sum_dEk"], E, rtol=1e-12)
        # a heating step at MOD(it, ns_heat) = 0 first updates vt from the tally (one rank)
        for it in (1, 2, 3, 4):
            sim.step(it)
        t = sim.source_tallies()
        for b in range(2):
            vt = O.te_update(cfg, 1, sc.Pabs[b], sc.nu_h, t["Nh"][b], t["sum_dEk"][b], sc.vt[b])
            assert t["vt"][b] == pytest.approx(vt, rel=1e-12)
            assert t["vt"][b] != sc.vt[b]
        assert t["n_heat_calls"] == 1
    finally:
        sim.close()


INJ_CASES = [(1, (0.08, 0.4, 0.08, 0.56), {}), (1, (-0.12, -0.44, 0, 0), {}),
             (-1, (0.16, 0.32, 0.08, 0.56), {}), (-1, (-0.2, -0.4, 0, 0), {}),
             (3, (0.08, 0.4, 0.08, 0.56), dict(THm=4.0)),
             (4, (0.08, 0.4, 0.08, 0.56), dict(THm=4.0)),
             (4, (0.0, 0.3, 0.08, 0.56), dict(THm=4.0, nmn=1, th_B=0.6)),
             (-4, (0.0, 0.3, 0.08, 0.56), dict(THm=2.0, nmn=1, th_B=-0.3))]


@pytest.mark.parametrize("opt,region,extra", INJ_CASES)
def test_injection_matches_oracle(gpu_lib, opt, region, extra):
    extra = dict(extra)
    case = make_case(plate=True)
    case.flag_nmn = extra.pop("nmn", 0)
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=100000)
    try:
        sim.put_particles(0, rand_particles(case, 20000, 3, 1.0e6))
        sim.put_particles(1, rand_particles(case, 20000, 4, 3.0e2))
        phi = np.fromfunction(lambda j, i: 2.0 * i - 1.5 * j + 0.01 * i * j, (case.ny + 3, case.nx + 3))
        sim.set_phi(phi)
        sim.deposit()
        sc = S.source_config(S.SourceDeck(heat_region_cm=region, I_inj=2000.0, opt_inj=opt, ni0=(1.0, 1.0),
                                          flag_diffsrc=1, nu_h=-1.0, seed=99, **extra), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        before = [sim.get_particles(s) for s in (0, 1)]
        sim.inject(6)
        after = [sim.get_particles(s) for s in (0, 1)]
        t = sim.source_tallies()
        Sb = shift_of(sim)
        vx = [np.zeros((len(before[s]) + 40000, 6)) for s in (0, 1)]
        for s in (0, 1):
            vx[s][:len(before[s])] = before[s]
        rc, n, cnt, Pi, Ps = O.part_injection_ctr(cfg, O.make_src(sc), np.ascontiguousarray(case.bcnd, np.int32),
                                                  phi, [0, 0], sc.seed, 6, Sb, vx, [len(b) for b in before])
        assert rc == 0
        assert t["n_inj_last"] == list(cnt) and cnt[0] > 1000
        # part_injection.f90:77-79: no ions under the beam, nor from the cathode without Neumann
        assert (cnt[1] == 0) == (abs(opt) == 3 or (abs(opt) == 4 and case.flag_nmn == 0))
        unit = case.dx * 2.0 ** -Sb
        for s in (0, 1):
            assert len(after[s]) == len(before[s]) + cnt[s]
            assert np.array_equal(after[s][:len(before[s])], before[s])
            new, ref = after[s][len(before[s]):], vx[s][len(before[s]):n[s]]
            if cnt[s] == 0:
                assert t["P_inj"][s] == 0.0
                continue
            assert np.abs(new[:, :2] - ref[:, :2]).max() <= unit * 1.0001
            float_match(ref[:, 3:], new[:, 3:])
            assert t["P_inj"][s] == pytest.approx(Pi[s], rel=1e-9)
            assert t["P_src"][s] == pytest.approx(Ps[s], rel=1e-9)
        # the injected particles are in this step's density
        kq = O.kq_of(np.asarray(case.bcnd))
        for s in (0, 1):
            npg = np.zeros((case.ny + 3, case.nx + 3))
            O.deposit(cfg, s, np.ascontiguousarray(after[s]), len(after[s]), kq, npg)
            dev = sim.grid(capi.GRID_NP + s)
            assert np.abs(dev - npg).max() <= 1e-12 * np.abs(npg).max()
    finally:
        sim.close()


def test_reinjection_of_lost_ions(gpu_lib):
    case = make_case()
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=100000)
    try:
        rng = np.random.default_rng(5)
        e = rand_particles(case, 5000, 6, 1.0e5)
        ions = rand_particles(case, 5000, 7, 1.0)
        ions[:1200, 0] = rng.random(1200) * case.dx * 0.5     # next to the left wall ...
        ions[:1200, 3] = -2.0 * case.dx / case.dt             # ... and leaving through it
        sim.put_particles(0, e)
        sim.put_particles(1, ions)
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 0.5, 0.1, 0.5), I_inj=0.0, opt_inj=2,
                                          ni0=(1.0, 1.0), nu_h=-1.0, seed=3), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        sim.push(1)
        lost = sim.push_stats()["n_lost"]
        assert lost[1] >= 1200
        sim.inject(1)
        t = sim.source_tallies()
        rc, _, cnt, _, _ = O.part_injection_ctr(cfg, O.make_src(sc), np.ascontiguousarray(case.bcnd, np.int32),
                                                np.zeros((case.ny + 3, case.nx + 3)), lost, sc.seed, 1, 0,
                                                [np.zeros((20000, 6)), np.zeros((20000, 6))], [0, 0])
        assert t["n_inj_last"] == list(cnt) == [lost[1], lost[1]]
        # the next call counts only the losses since this one
        sim.push(2)
        lost2 = sim.push_stats()["n_lost"]
        sim.inject(2)
        assert sim.source_tallies()["n_inj_last"][1] == lost2[1] - lost[1]
    finally:
        sim.close()


def run_with_sources(steps=8):
    case = configs.case0(ppc=8, nx=NX, ny=NX)
    case.poisson_mode = 1
    case.eps = 1e-8
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    sim = GpuSimulation(case)
    sc = S.source_config(S.SourceDeck(heat_region_cm=(0.16, 0.48, 0.16, 0.48), nu_h=5.0e8, Pabs=(20.0,),
                                      I_inj=50.0, opt_inj=1, ni0=(1.0, 1.0), seed=11), case.dt, sp.vt0[0])
    sim.set_sources(sc)
    for it in range(1, steps + 1):
        sim.step(it)
    out = [sim.get_particles(s) for s in (0, 1)], sim.source_tallies(), sim.push_stats()
    sim.close()
    return out


def test_step_with_sources_is_reproducible_and_consistent(gpu_lib):
    (pa, ta, sa), (pb, tb, sb) = run_with_sources(), run_with_sources()
    for s in (0, 1):
        assert np.array_equal(pa[s], pb[s])
    assert ta == tb
    assert ta["n_heat_calls"] == 2                      # it = 4 and 8 (ns_heat = 4)
    assert ta["n_heated"] > 0 and ta["P_heat"] != 0.0
    assert ta["n_inj"][0] > 0 and abs(ta["n_inj"][0] - ta["n_inj"][1]) <= 8   # one rounding per step
    assert sa["np_tot"] == [len(pa[0]), len(pa[1])]


def test_source_errors(gpu_lib):
    case = make_case()
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=1000)
    try:
        lib = sim.lib
        bad = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 0.3, 0.1, 0.3), I_inj=1.0, opt_inj=5),
                              case.dt, sp.vt0[0])
        assert lib.lepic_gpu_set_sources(sim.ctx, C.byref(bad)) == capi.EINVAL
        bad = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 3.0, 0.1, 0.3), I_inj=1.0), case.dt, sp.vt0[0])
        assert lib.lepic_gpu_set_sources(sim.ctx, C.byref(bad)) == capi.EINVAL
        assert lib.lepic_gpu_eheating(sim.ctx, 4) == capi.EINVAL         # no sources yet
        # more injected particles than slots: the call fails, the context stays usable
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1, 0.5, 0.1, 0.5), I_inj=1.0e4, opt_inj=1,
                                          ni0=(1.0, 1.0), nu_h=-1.0), case.dt, sp.vt0[0])
        sim.set_sources(sc)
        assert lib.lepic_gpu_part_injection(sim.ctx, 1) == 0
        assert lib.lepic_gpu_sync(sim.ctx) == capi.ECAPACITY
        assert sim.push_stats()["np_tot"] == [0, 0]
        sim.put_particles(0, rand_particles(case, 10, 1, 1.0))
        assert len(sim.get_particles(0)) == 10
    finally:
        sim.close()


def test_region_edges_exact(gpu_lib):
    """Particles on the fixed-point values around every edge of the slit: with nu*dt = 1 every
    electron of the region is heated, so the heated set and the tally counts show the region
    test itself, which must equal the oracle's FP64 test exactly."""
    case = make_case()
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=200000)
    try:
        Sb = shift_of(sim)
        ux = case.dx * 2.0 ** -Sb
        sc = S.source_config(S.SourceDeck(heat_region_cm=(0.1234567, 0.4123457, 0.0987654, 0.5012345),
                                          nu_h=1.0 / (4 * case.dt), I_inj=-1.0), case.dt, sp.vt0[0])
        assert sc.nudt == pytest.approx(1.0)
        xa, dr = (sc.xl_pow + sc.xr_pow) / 2, (sc.xr_pow - sc.xl_pow) / 2
        xe = [sc.xl_pow, sc.xr_pow, xa - dr, xa + dr, xa]
        ye = [sc.yl_pow, sc.yr_pow, 0.5 * case.ny * case.dy]
        Xs = np.unique(np.concatenate([np.round(np.array(xe) / ux).astype(np.int64)[:, None] + np.arange(-3, 4)]))
        Ys = np.unique(np.concatenate([np.round(np.array(ye) / ux).astype(np.int64)[:, None] + np.arange(-3, 4)]))
        XX, YY = np.meshgrid(Xs, Ys)
        v = np.zeros((XX.size, 6))
        v[:, 0] = XX.ravel() * ux
        v[:, 1] = YY.ravel() * ux
        v[:, 3:] = 1.0
        sim.put_particles(0, v)
        sim.set_sources(sc)
        p0 = sim.get_particles(0)
        assert np.array_equal(p0[:, :2], v[:, :2])
        sim.heating_tally()
        sim.eheating(4)
        p1 = sim.get_particles(0)
        t = sim.source_tallies()
        o = p0.copy()
        _, nh = O.eheating(cfg, O.make_src(sc), o, vt_used(sc, sp), seed=sc.seed, it=4)
        heated_o = np.any(o[:, 3:] != p0[:, 3:], axis=1)
        heated_d = np.any(p1[:, 3:] != p0[:, 3:], axis=1)
        assert 0 < heated_o.sum() < len(v) and np.array_equal(heated_o, heated_d)
        Nh, _ = O.heat_tally(cfg, O.make_src(sc), p0)
        assert t["Nh"] == list(Nh)
    finally:
        sim.close()


def plate_case(left=True, holes=((20, 26), (38, 44))):
    case = configs.case0(ppc=4, nx=NX, ny=NX)
    b = np.array(case.bcnd, dtype=np.int32, copy=True)
    b[5:61, 40:44] = 1
    for h0, h1 in holes:
        b[h0:h1 + 1, 40:44] = -1
    if not left:
        b[2:case.ny + 1, 2:40] = 1
    case.bcnd = b
    case.phi0 = configs.potentials(b, {1: 0.0})
    return case


EMIT_CASES = [dict(left=True), dict(left=False),
              dict(left=True, chamfer=True)]


@pytest.mark.parametrize("kw", EMIT_CASES)
def test_flux_emitter_matches_oracle(gpu_lib, kw):
    left, chamfer = kw["left"], kw.get("chamfer", False)
    case = plate_case(left, holes=((28, 36),) if chamfer else ((20, 26), (38, 44)))
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=100000)
    try:
        rng = np.random.default_rng(8)
        e = rand_particles(case, 3000, 9, 1e5)
        sim.put_particles(0, e)
        sim.put_particles(1, rand_particles(case, 3000, 10, 1e2))
        xg1 = (39.5 if left else 42.5) * case.dx
        extra = dict(tag_neg=1, ptype_fx=1, tag_b=0, chamfer_m=(39.5 * case.dx, 43.5 * case.dx, 2.0e-3, 2.6e-3),
                     n_holes=1) if chamfer else {}
        deck = dict(jne=1.0e5, ptype_fx=0, THm=5.0, xg1_cm=xg1 * 100, Lg_cm=55 * case.dy * 100,
                    Lh_cm=3 * case.dy * 100, n_holes=2, nu_h=-1.0, I_inj=-1.0, seed=77)
        deck.update(extra)
        sc = S.source_config(S.SourceDeck(**deck), case.dt, sp.vt0[0], case.dy)
        sim.set_sources(sc)
        before = [sim.get_particles(s) for s in (0, 1)]
        sim.flux_emitter(5)
        after = [sim.get_particles(s) for s in (0, 1)]
        t = sim.source_tallies()
        Sb = shift_of(sim)
        vx = [np.zeros((len(before[s]) + 40000, 6)) for s in (0, 1)]
        for s in (0, 1):
            vx[s][:len(before[s])] = before[s]
        rc, n, cnt, Pi, nout = O.flux_emitter_ctr(cfg, O.make_emit(sc), np.ascontiguousarray(case.bcnd, np.int32),
                                                  sc.seed, 5, Sb, vx, [len(b) for b in before])
        assert rc == 0 and sum(cnt) > 2000
        assert t["n_emit_last"] == list(cnt) and t["n_emit_out"] == nout
        if chamfer:
            assert cnt[0] > 0 and cnt[1] > 0
        unit = case.dx * 2.0 ** -Sb
        for s in (0, 1):
            assert np.array_equal(after[s][:len(before[s])], before[s])
            new, ref = after[s][len(before[s]):], vx[s][len(before[s]):n[s]]
            assert len(new) == len(ref)
            if len(new):
                assert np.abs(new[:, :2] - ref[:, :2]).max() <= unit * 1.0001
                float_match(ref[:, 3:], new[:, 3:])
            assert t["P_inj"][s] == pytest.approx(Pi[s], rel=1e-9, abs=0.0)
        ps = sim.push_stats()
        assert ps["n_lost"] == [0, 0] or sum(ps["n_lost"]) == nout
    finally:
        sim.close()


def test_step_runs_the_emitter(gpu_lib):
    case = plate_case(True)
    case.poisson_mode = 1
    case.eps = 1e-8
    cfg, sp = oracle_cfg(case)
    sim = GpuSimulation(case, load=False, capacity=200000)
    try:
        sim.put_particles(0, rand_particles(case, 20000, 11, 1e5))
        sim.put_particles(1, rand_particles(case, 20000, 12, 1e2))
        sim.deposit()
        sc = S.source_config(S.SourceDeck(jne=2.0e4, ptype_fx=0, THm=5.0, xg1_cm=39.5 * case.dx * 100,
                                          Lg_cm=55 * case.dy * 100, Lh_cm=3 * case.dy * 100, n_holes=2,
                                          nu_h=-1.0, I_inj=-1.0, seed=5), case.dt, sp.vt0[0], case.dy)
        sim.set_sources(sc)
        per = []
        for it in range(1, 5):
            sim.step(it)
            per.append(sim.source_tallies()["n_emit_last"][0])
        t = sim.source_tallies()
        assert min(per) > 0 and t["n_emit"][0] == sum(per)
    finally:
        sim.close()
