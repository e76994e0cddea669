"""The CPU restatement of the particle sources (e_heating.f90, part_injection.f90) and the
deck conversions of ``jd_lepic_b200.sources``.

The counter-based RNG of the device path is pinned to the published Philox4x32-10 known
answers; the two oracle forms (the reference's sequential ran2 draw order and the device's
counter streams) are checked against the distributions the routines define and against
each other."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from jd_lepic_b200 import configs, deck as dk
from jd_lepic_b200 import sources as S
from jd_lepic_b200.simulation import species_params

# Random123's known-answer vectors for Philox4x32-10 (counter, key, output)
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def test_philox_known_answers(oracle_lib):
    for ctr, key, out in PHILOX_KAT:
        assert O.philox(ctr, key) == out


def setup(nx=32, ny=32):
    case = configs.case0(ppc=4, nx=nx, ny=ny)
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    return case, O.make_cfg(case, sp), sp


def src_cfg(sp, dt, **kw):
    deck = S.SourceDeck(**kw)
    return S.source_config(deck, dt, sp.vt0[0])


def electrons(case, n, seed, S_bits=None):
    """n electrons uniform in the box, velocities ~ N(0, vt0^2/2) (FP32-representable)."""
    rng = np.random.default_rng(seed)
    v = np.zeros((n, 6))
    v[:, 0] = rng.random(n) * case.nx * case.dx
    v[:, 1] = rng.random(n) * case.ny * case.dy
    v[:, 3:] = rng.normal(0.0, 1.0e6, (n, 3)).astype(np.float32)
    return v


# ---- eheating --------------------------------------------------------------------------
@pytest.mark.parametrize("disk", [0, 1])
def test_eheating_region_rate_and_power_identity(oracle_lib, disk):
    case, cfg, sp = setup()
    region = (-0.08, -0.24, 0.0, 0.0) if disk else (0.08, 0.24, 0.04, 0.28)
    sc = src_cfg(sp, case.dt, heat_region_cm=region, nu_h=2.0e10, ns_heat=4, Pabs=(0.0,))
    src = O.make_src(sc)
    v0 = electrons(case, 200000, 1)
    v = v0.copy()
    vt = np.full(16, 1.5e6)
    P, nh, _ = O.eheating(cfg, src, v, vt, iseed=12345)
    changed = np.any(v[:, 3:] != v0[:, 3:], axis=1)
    x, y = v0[:, 0], v0[:, 1]
    xa, dr = (sc.xl_pow + sc.xr_pow) / 2, (sc.xr_pow - sc.xl_pow) / 2
    if disk:
        inside = (x - xa) ** 2 + (y - case.ny * case.dy / 2) ** 2 <= dr * dr
    else:
        inside = ((x - xa) ** 2 <= dr * dr) & (y >= sc.yl_pow) & (y <= sc.yr_pow)
    assert not np.any(changed & ~inside)                     # only the region is heated
    assert changed.sum() == nh
    p = sc.nudt                                              # probability per call
    n_in = inside.sum()
    assert abs(nh - p * n_in) < 5 * math.sqrt(n_in * p * (1 - p))
    # P_loss(2) is the kinetic energy the heated electrons gained
    Ek = 0.5 * sp.Nm[0] * sp.mass[0]
    dE = Ek * ((v[:, 3:] ** 2).sum(1) - (v0[:, 3:] ** 2).sum(1))
    assert P == pytest.approx(dE.sum(), rel=1e-9)
    # eheat_type 1: the new components are normal with sigma = vt/sqrt(2)
    nv = v[changed, 3:]
    assert abs(nv.std() / (1.5e6 / math.sqrt(2)) - 1) < 0.05


def test_eheating_gaussian_profile_rate(oracle_lib):
    case, cfg, sp = setup()
    sc = src_cfg(sp, case.dt, heat_region_cm=(-0.08, -0.24, 0, 0), nu_h=1.0e8, ns_heat=4, Pabs=(100.0,),
                 opt_inj=-1, I_inj=-1.0)
    assert sc.flag_gpp == 1
    src = O.make_src(sc)
    v = electrons(case, 400000, 2)
    x, y = v[:, 0].copy(), v[:, 1].copy()
    v0 = v.copy()
    P, nh = O.eheating(cfg, src, v, np.full(16, 1e6), seed=7, it=4)
    changed = np.any(v[:, 3:] != v0[:, 3:], axis=1)
    xa, dr = (sc.xl_pow + sc.xr_pow) / 2, (sc.xr_pow - sc.xl_pow) / 2
    rp2 = (x - xa) ** 2 + (y - case.ny * case.dy / 2) ** 2
    inside = rp2 <= dr * dr
    prob = sc.nudt * 9.0 * np.exp(-9.0 * rp2 / dr ** 2)
    expect = prob[inside].sum()
    assert abs(nh - expect) < 5 * math.sqrt(expect)
    # the inner third heats far more often than the outer ring
    inner = inside & (rp2 < (dr / 3) ** 2)
    outer = inside & (rp2 > (2 * dr / 3) ** 2)
    assert changed[inner].mean() > 5 * changed[outer].mean()


def test_eheating_two_forms_agree_in_distribution(oracle_lib):
    case, cfg, sp = setup()
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.04, 0.28, 0.0, 0.32), nu_h=5.0e8, ns_heat=4, n_icp=2)
    src = O.make_src(sc)
    vt = np.zeros(16)
    vt[:2] = (1.0e6, 2.0e6)
    a = electrons(case, 200000, 3)
    b = a.copy()
    _, na, _ = O.eheating(cfg, src, a, vt, iseed=99)
    _, nb = O.eheating(cfg, src, b, vt, seed=5, it=8)
    assert abs(na - nb) < 5 * math.sqrt(na)
    ya, yb = a[:, 1], b[:, 1]
    for band, vtb in enumerate((1.0e6, 2.0e6)):
        ma = np.any(a[:, 3:] != electrons(case, 200000, 3)[:, 3:], axis=1) & ((2 * ya / (case.ny * case.dy)).astype(int) == band)
        mb = np.any(b[:, 3:] != electrons(case, 200000, 3)[:, 3:], axis=1) & ((2 * yb / (case.ny * case.dy)).astype(int) == band)
        # vx, vy come from the particle's own band; the reference's vz is the saved second
        # component of the previous heated electron's pair, which may be of the other band
        sa, sb = a[ma, 3:5].std(), b[mb, 3:].std()
        assert abs(sa / (vtb / math.sqrt(2)) - 1) < 0.06
        assert abs(sb / (vtb / math.sqrt(2)) - 1) < 0.06


def test_eheating_increment_type(oracle_lib):
    case, cfg, sp = setup()
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.0, 0.32, 0.0, 0.32), nu_h=1.0e9, ns_heat=4)
    sc.eheat_type = 2
    src = O.make_src(sc)
    v0 = electrons(case, 100000, 4)
    v = v0.copy()
    O.eheating(cfg, src, v, np.full(16, 1e5), seed=1, it=1)
    ch = np.any(v[:, 3:] != v0[:, 3:], axis=1)
    d = (v - v0)[ch, 3:]
    assert abs(d.std() / (1e5 / math.sqrt(2)) - 1) < 0.06   # increments, not replacements


def test_heat_tally_and_te_update(oracle_lib):
    case, cfg, sp = setup()
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.08, 0.24, 0.0, 0.32), nu_h=1.0e8, n_icp=2, Pabs=(50.0, 80.0))
    src = O.make_src(sc)
    v = electrons(case, 50000, 5)
    Nh, E = O.heat_tally(cfg, src, v)
    x, y = v[:, 0], v[:, 1]
    inside = (x >= sc.xl_pow) & (x <= sc.xr_pow) & (y >= sc.yl_pow) & (y <= sc.yr_pow)
    band = (2 * y / (case.ny * case.dy)).astype(int)
    Ek = 0.5 * sp.Nm[0] * sp.mass[0] * (v[:, 3:] ** 2).sum(1)
    for b in range(2):
        m = inside & (band == b)
        assert Nh[b] == m.sum()
        assert E[b] == pytest.approx(Ek[m].sum(), rel=1e-12)
        vt = O.te_update(cfg, 1, sc.Pabs[b], sc.nu_h, Nh[b], E[b], 0.0)
        Te = (2 / 3) * (E[b] + sc.Pabs[b] / sc.nu_h) / (sp.Nm[0] * dk.QE * Nh[b])
        assert vt == pytest.approx(math.sqrt(2 * dk.QE * Te / abs(sp.mass[0])), rel=1e-14)
    assert O.te_update(cfg, 1, 1.0, 1.0, 0, 0.0, 123.0) == 123.0   # no electrons: keep vt


# ---- part_injection --------------------------------------------------------------------
def plate_bcnd(case):
    """The box with an embedded wall plate (nodes 8..12 x 10..20 labelled 1)."""
    b = np.array(case.bcnd, dtype=np.int32, copy=True)
    b[10:21, 8:13] = 1
    return b


def all_walls(b, x, y, case):
    ix = (x / case.dx).astype(int) + 1
    iy = (y / case.dy).astype(int) + 1
    return (b[iy, ix] >= 1) & (b[iy, ix + 1] >= 1) & (b[iy + 1, ix + 1] >= 1) & (b[iy + 1, ix] >= 1)


@pytest.mark.parametrize("opt,region", [(1, (0.04, 0.2, 0.04, 0.28)), (1, (-0.06, -0.2, 0, 0)),
                                        (-1, (0.08, 0.16, 0.04, 0.28)), (-1, (-0.1, -0.2, 0, 0))])
def test_injection_reference_form(oracle_lib, opt, region):
    case, cfg, sp = setup()
    b = plate_bcnd(case)
    phi = np.zeros((case.ny + 3, case.nx + 3))
    sc = src_cfg(sp, case.dt, heat_region_cm=region, I_inj=400.0, opt_inj=opt, ni0=(1.0, 1.0))
    src = O.make_src(sc)
    dN = sc.I_inj * sc.ns_inj * case.dt * 1.0 / (dk.QE * sp.Nm[0])
    assert 100 < dN < 100000
    for ptype in (0, 1):
        N_inj = np.zeros(8, dtype=np.int64)
        vxp = np.zeros((int(dN) + 10, 6))
        rc, n, Pi, Ps, _ = O.part_injection(cfg, src, ptype, b, phi, N_inj, vxp, 0, 777 + ptype)
        assert rc == 0 and n == N_inj[ptype] and n in (int(dN), int(dN) + 1)
        p = vxp[:n]
        assert not np.any(all_walls(b, p[:, 0], p[:, 1], case))
        xa, dr = (sc.xl_pow + sc.xr_pow) / 2, (sc.xr_pow - sc.xl_pow) / 2
        ymid = case.ny * case.dy / 2
        if opt > 0 and sc.flag_c == 0:
            assert p[:, 0].min() >= sc.xl_pow and p[:, 0].max() <= sc.xr_pow
            assert p[:, 1].min() >= sc.yl_pow and p[:, 1].max() <= sc.yr_pow
        elif opt > 0:
            assert np.all((p[:, 0] - xa) ** 2 + (p[:, 1] - ymid) ** 2 <= dr * dr * (1 + 1e-12))
        elif sc.flag_c == 0:  # Gaussian along x, sigma = dr/sqrt(2)
            assert abs(p[:, 0].std() / (dr / math.sqrt(2)) - 1) < 0.15
        else:
            assert np.all((p[:, 0] - xa) ** 2 + (p[:, 1] - ymid) ** 2 <= 4 * dr * dr * (1 + 1e-12))
        vt = sp.vt0[ptype]
        assert abs(p[:, 4].std() / (vt / math.sqrt(2)) - 1) < 0.15
        # the first particle of the call (and every second one) has vz = vx
        assert np.all(p[0::2, 5] == p[0::2, 3])
        assert Pi == pytest.approx(0.5 * sp.Nm[ptype] * sp.mass[ptype] * (p[:, 3:] ** 2).sum(), rel=1e-9)


def test_injection_reinjects_lost_ions(oracle_lib):
    case, cfg, sp = setup()
    b = np.array(case.bcnd, dtype=np.int32)
    phi = np.zeros((case.ny + 3, case.nx + 3))
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.04, 0.28, 0.04, 0.28), I_inj=0.0, opt_inj=2, ni0=(1.0, 1.0))
    assert sc.I_inj == 0.0
    src = O.make_src(sc)
    lost = np.array([17, 53], dtype=np.int64)
    v = [np.zeros((200, 6)), np.zeros((200, 6))]
    rc, n, cnt, Pi, Ps = O.part_injection_ctr(cfg, src, b, phi, lost, 3, 10, 0, v, [0, 0])
    assert rc == 0 and list(cnt) == [53, 53]       # a pair per lost positive ion
    # the reference form: the electron count from the ions' losses, the ions their own
    N_inj = lost.copy()
    N_inj.resize(8)
    ve = np.zeros((200, 6))
    rc, ne, *_ = O.part_injection(cfg, src, 0, b, phi, N_inj, ve, 0, 5)
    assert rc == 0 and ne == 53 and N_inj[0] == 53
    rc, ni, *_ = O.part_injection(cfg, src, 1, b, phi, N_inj, np.zeros((200, 6)), 0, 6)
    assert rc == 0 and ni == 53


def test_injection_capacity_and_diffsrc(oracle_lib):
    case, cfg, sp = setup()
    b = np.array(case.bcnd, dtype=np.int32)
    phi = np.fromfunction(lambda j, i: 10.0 * i + 3.0 * j, (case.ny + 3, case.nx + 3))
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.04, 0.28, 0.04, 0.28), I_inj=40.0, opt_inj=1, ni0=(1.0, 1.0),
                 flag_diffsrc=1)
    src = O.make_src(sc)
    N_inj = np.zeros(8, dtype=np.int64)
    small = np.zeros((5, 6))
    rc, *_ = O.part_injection(cfg, src, 0, b, phi, N_inj, small, 0, 1)
    assert rc == -2                                # part_injection.f90:146-150
    big = [np.zeros((5000, 6)), np.zeros((5000, 6))]
    rc, n, cnt, Pi, Ps = O.part_injection_ctr(cfg, src, b, phi, [0, 0], 9, 3, 0, big, [0, 0])
    assert rc == 0
    for s in range(2):
        p = big[s][:cnt[s]]
        # phi is bilinear in the node indices, so the CIC interpolation is exact
        phip = 10.0 * (p[:, 0] / case.dx + 1) + 3.0 * (p[:, 1] / case.dy + 1)
        assert Ps[s] == pytest.approx((-sp.Nm[s] * sp.charge[s] * phip).sum(), rel=1e-10)


def test_injection_two_forms_agree_in_distribution(oracle_lib):
    case, cfg, sp = setup()
    b = plate_bcnd(case)
    phi = np.zeros((case.ny + 3, case.nx + 3))
    sc = src_cfg(sp, case.dt, heat_region_cm=(-0.06, -0.22, 0, 0), I_inj=8000.0, opt_inj=-1, ni0=(1.0, 1.0))
    src = O.make_src(sc)
    N_inj = np.zeros(8, dtype=np.int64)
    va = np.zeros((20000, 6))
    rc, na, *_ = O.part_injection(cfg, src, 0, b, phi, N_inj, va, 0, 42)
    vb = [np.zeros((20000, 6)), np.zeros((20000, 6))]
    rc2, nb, cnt, *_ = O.part_injection_ctr(cfg, src, b, phi, [0, 0], 11, 2, 21, vb, [0, 0])
    assert rc == 0 and rc2 == 0 and abs(na - cnt[0]) <= 1
    pa, pb = va[:na], vb[0][:cnt[0]]
    for k in (0, 1):
        assert abs(pa[:, k].mean() - pb[:, k].mean()) < 4 * pa[:, k].std() / math.sqrt(na) * 1.5
        assert abs(pa[:, k].std() / pb[:, k].std() - 1) < 0.05
    for k in (3, 4, 5):
        assert abs(pa[:, k].std() / pb[:, k].std() - 1) < 0.05
    assert np.all(pb[0::2, 5] == pb[0::2, 3])


def flux_mean(vb, vt):
    """The mean of v under the shifted-Maxwellian flux v exp(-(v - vb)^2 / vt^2) on
    [max(0, vb - 4 vt), vb + 4 vt] (part_injection.f90:239-265)."""
    v = np.linspace(max(0.0, vb - 4 * vt), vb + 4 * vt, 200001)
    f = v * np.exp(-(v - vb) ** 2 / vt ** 2)
    return float((v * f).sum() / f.sum())


@pytest.mark.parametrize("nmn", [0, 1])
def test_injection_beam_and_cathode_reference_form(oracle_lib, nmn):
    """|opt_inj| = 3: electrons only, vz shifted by the beam speed; |opt_inj| = 4: the flux
    along +x from the cathode at x = 0 (electrons half-Maxwellian with Neumann), positions
    x = vx * U(0, ns_inj dt), vy shifted by vb sin(th_B); ions only with Neumann."""
    case, cfg, sp = setup()
    cfg.flag_nmn = nmn
    b = np.array(case.bcnd, dtype=np.int32)
    phi = np.zeros((case.ny + 3, case.nx + 3))
    THm, thB = 3.0, 0.4
    for opt in (3, 4):
        sc = src_cfg(sp, case.dt, heat_region_cm=(0.04, 0.28, 0.04, 0.28), I_inj=1600.0, opt_inj=opt,
                     ni0=(1.0, 1.0), THm=THm, th_B=thB, ns_inj=2)
        src = O.make_src(sc)
        assert src.th_B == (thB if opt == 4 else 0.0)
        for ptype in (0, 1):
            N_inj = np.zeros(8, dtype=np.int64)
            vxp = np.zeros((40000, 6))
            rc, n, Pi, Ps, _ = O.part_injection(cfg, src, ptype, b, phi, N_inj, vxp, 0, 31 + ptype)
            assert rc == 0
            ions_off = opt == 3 or nmn == 0
            if ptype == 1 and ions_off:
                assert n == 0 and N_inj[1] == 0
                continue
            assert n > 3000
            p = vxp[:n]
            vt = sp.vt0[ptype]
            vb = math.sqrt(2 * dk.QE * THm / abs(sp.mass[ptype]))
            if opt == 3:
                assert abs(p[:, 5].mean() - vb) < 5 * vt / math.sqrt(2 * n)
                assert np.all(p[0::2, 5] - vb == pytest.approx(p[0::2, 3], abs=1e-9 * vb))
                continue
            if opt == 4 and ptype == 0 and nmn == 1:
                vb = 0.0
            vbt = vb * math.cos(thB)
            assert p[:, 3].min() >= max(0.0, vbt - 4 * vt) and p[:, 3].max() <= vbt + 4 * vt
            m = flux_mean(vbt, vt)
            assert abs(p[:, 3].mean() - m) < 5 * p[:, 3].std() / math.sqrt(n)
            assert abs(p[:, 4].mean() - vb * math.sin(thB)) < 5 * vt / math.sqrt(2 * n) + 1e-12
            assert abs(p[:, 5].mean()) < 5 * vt / math.sqrt(2 * n)
            t = p[:, 0] / p[:, 3]
            ns_dt = 2 * case.dt
            assert t.min() >= 0.0 and t.max() <= ns_dt * (1 + 1e-12)
            assert abs(t.mean() / (ns_dt / 2) - 1) < 0.05
            assert Pi == pytest.approx(0.5 * sp.Nm[ptype] * sp.mass[ptype] * (p[:, 3:] ** 2).sum(), rel=1e-9)


def test_cathode_two_forms_agree_in_distribution(oracle_lib):
    case, cfg, sp = setup()
    cfg.flag_nmn = 1
    b = np.array(case.bcnd, dtype=np.int32)
    phi = np.zeros((case.ny + 3, case.nx + 3))
    sc = src_cfg(sp, case.dt, heat_region_cm=(0.0, 0.2, 0.04, 0.28), I_inj=6000.0, opt_inj=4, ni0=(1.0, 1.0),
                 THm=5.0, th_B=-0.7)
    src = O.make_src(sc)
    N_inj = np.zeros(8, dtype=np.int64)
    va = np.zeros((30000, 6))
    rc, na, *_ = O.part_injection(cfg, src, 1, b, phi, N_inj, va, 0, 77)
    vb_ = [np.zeros((30000, 6)), np.zeros((30000, 6))]
    rc2, nb, cnt, *_ = O.part_injection_ctr(cfg, src, b, phi, [0, 0], 5, 4, 0, vb_, [0, 0])
    assert rc == 0 and rc2 == 0 and abs(na - cnt[1]) <= 1 and na > 5000
    pa, pb = va[:na], vb_[1][:cnt[1]]
    for k in (0, 1, 3, 4, 5):
        se = math.sqrt(pa[:, k].var() / na + pb[:, k].var() / cnt[1])
        assert abs(pa[:, k].mean() - pb[:, k].mean()) < 5 * se
        assert abs(pa[:, k].std() / pb[:, k].std() - 1) < 0.05


def test_cathode_angle():
    assert S.cathode_angle(4, 1, 0.02, 0.01) == pytest.approx(math.atan(0.5))
    assert S.cathode_angle(4, 0, 0.02, 0.01) == 0.0
    assert S.cathode_angle(-4, 1, 0.02, 0.01) == 0.0        # main.f90:450: opt_inj .eq. 4
    assert S.cathode_angle(4, 1, 0.0, 0.01) == 0.0


# ---- deck conversions ------------------------------------------------------------------
def test_source_deck_conversions():
    d = S.SourceDeck(heat_region_cm=(-1.0, -3.0, 0.5, 2.5), n_icp=-2, Pabs=(100.0, 50.0), nu_h=1.0e7,
                     I_inj=5.0, opt_inj=-2, THm=-3.0, ns_heat=4)
    c = S.source_config(d, 1e-11, 1.0e6)
    assert c.flag_c == 1 and c.xl_pow == pytest.approx(0.01) and c.xr_pow == pytest.approx(0.03)
    assert c.n_icp == 2 and c.flag_heat == 1 and c.nudt == pytest.approx(1.0e7 * 4 * 1e-11)
    assert c.flag_gpp == 1 and c.eheat_type == 1
    assert c.flag_inj == 1 and c.I_inj == 0.0        # |opt_inj| = 2 ignores I_inj
    assert c.flag_Tp == 1 and c.THm == 3.0
    off = S.source_config(S.SourceDeck(nu_h=-1.0, I_inj=-1.0), 1e-11, 1.0e6)
    assert off.flag_heat == 0 and off.flag_inj == 0 and off.flag_c == 0


# ---- part_flux_emitter -----------------------------------------------------------------
def plate_with_holes(case, i0=40, width=4, j0=5, j1=60, holes=((20, 26), (38, 44)), plasma_left=True):
    """A grid plate of wall nodes i0..i0+width-1, rows j0..j1, with apertures; the far side of
    the plate is walled off when plasma_left is False so that the plasma is on the right."""
    b = np.array(case.bcnd, dtype=np.int32, copy=True)
    b[j0:j1 + 1, i0:i0 + width] = 1
    for h0, h1 in holes:
        b[h0:h1 + 1, i0:i0 + width] = -1
    if not plasma_left:
        b[2:case.ny + 1, 2:i0] = 1
    return b


def emit_cfg(sp, case, **kw):
    d = dict(jne=1.0e5, ptype_fx=0, THm=5.0, xg1_cm=39.5 * case.dx * 100, Lg_cm=55 * case.dy * 100,
             Lh_cm=3 * case.dy * 100, n_holes=2, nu_h=-1.0, I_inj=-1.0)
    d.update(kw)
    return S.source_config(S.SourceDeck(**d), case.dt, sp.vt0[0], case.dy)


@pytest.mark.parametrize("left", [True, False])
def test_flux_emitter_reference_form(oracle_lib, left):
    case, cfg, sp = setup(64, 64)
    b = plate_with_holes(case, plasma_left=left)
    # the emission plane inside the plate's face cell on the plasma side
    xg1 = (39.5 if left else 42.5) * case.dx
    sc = emit_cfg(sp, case, xg1_cm=xg1 * 100)
    em = O.make_emit(sc)
    v = [np.zeros((50000, 6)), np.zeros((10, 6))]
    rc, n, cnt, Pi, _ = O.flux_emitter(cfg, em, b, v, [0, 0], 4242)
    Lgrd = 1 * (55 * case.dy - 3 * case.dy * 2)
    dNh = sc.js * cfg.zmax * Lgrd * case.dt / (sp.Nm[0] * dk.QE)
    assert rc == 0 and cnt[0] in (int(dNh), int(dNh) + 1) and cnt[0] > 5000 and cnt[1] == 0
    p = v[0][:n[0]]
    vt = math.sqrt(2 * dk.QE * 5.0 / abs(sp.mass[0]))
    if left:   # the flux leaves the plate towards the plasma side
        assert np.all(p[:, 3] < 0) and np.all(p[:, 0] <= xg1 + 1e-12)
    else:
        assert np.all(p[:, 3] > 0) and np.all(p[:, 0] >= xg1 - 1e-12)
    # the normal component is the Rayleigh speed of a half-Maxwellian flux, mean vt sqrt(pi)/2
    assert abs(np.abs(p[:, 3]).mean() / (vt * math.sqrt(math.pi) / 2) - 1) < 0.03
    assert abs(p[:, 4].std() / (vt / math.sqrt(2)) - 1) < 0.03
    assert abs(p[:, 5].std() / (vt / math.sqrt(2)) - 1) < 0.03
    # nothing is emitted from the apertures
    iy = (p[:, 1] / case.dy).astype(int) + 1
    assert not np.any((iy >= 21) & (iy <= 25)) and not np.any((iy >= 39) & (iy <= 43))
    assert Pi[0] == pytest.approx(0.5 * sp.Nm[0] * sp.mass[0] * (p[:, 3:] ** 2).sum(), rel=1e-9)


def test_flux_emitter_two_forms_agree(oracle_lib):
    case, cfg, sp = setup(64, 64)
    b = plate_with_holes(case)
    sc = emit_cfg(sp, case)
    em = O.make_emit(sc)
    va = [np.zeros((50000, 6)), np.zeros((10, 6))]
    vb = [np.zeros((50000, 6)), np.zeros((10, 6))]
    rc, na, ca, Pa, _ = O.flux_emitter(cfg, em, b, va, [0, 0], 99)
    rc2, nb, cb, Pb, nout = O.flux_emitter_ctr(cfg, em, b, 17, 3, 0, vb, [0, 0])
    assert rc == 0 and rc2 == 0 and abs(ca[0] - cb[0]) <= 1 and nout == 0
    pa, pb = va[0][:na[0]], vb[0][:nb[0]]
    for k in (1, 3, 4, 5):
        assert abs(pa[:, k].mean() - pb[:, k].mean()) < 5 * pa[:, k].std() / math.sqrt(len(pa))
        assert abs(pa[:, k].std() / pb[:, k].std() - 1) < 0.04
    assert Pa[0] == pytest.approx(Pb[0], rel=0.04)


def test_flux_emitter_chamfer_species(oracle_lib):
    case, cfg, sp = setup(64, 64)
    b = plate_with_holes(case, holes=((28, 36),))
    ymax = case.ny * case.dy
    # a chamfered aperture edge: from (x1, ymax/2 - y1) to (x2, ymax/2 - y2)
    ch = (39.5 * case.dx, 43.5 * case.dx, 2.0e-3, 2.6e-3)     # Lgrd = 2 (y1 + d) = 5.44 mm < ymax
    sc = emit_cfg(sp, case, tag_neg=1, ptype_fx=1, tag_b=0, chamfer_m=ch, n_holes=1, I_inj=-1.0)
    em = O.make_emit(sc)
    assert em.chamfer == 1 and em.sp_fx == 1 and em.sp_b == 0
    v = [np.zeros((100000, 6)), np.zeros((100000, 6))]
    rc, n, cnt, Pi, _ = O.flux_emitter_ctr(cfg, em, b, 5, 1, 0, v, [0, 0])
    assert rc == 0 and cnt[0] > 0 and cnt[1] > 0       # both surfaces emit
    d = math.hypot(ch[1] - ch[0], ch[3] - ch[2])
    Lgrd = 2 * (ch[2] + d)
    dNh = sc.js * cfg.zmax * Lgrd * case.dt / (sp.Nm[1] * dk.QE)
    assert cnt.sum() in (int(dNh), int(dNh) + 1)


def test_emitter_deck_conversion():
    case, cfg, sp = setup(64, 64)
    sc = emit_cfg(sp, case, Lh_cm=3.5 * case.dy * 100)
    assert sc.js == pytest.approx(1.0e6) and sc.ns_Hm == 1
    assert sc.Lh == pytest.approx(3 * case.dy)          # rounded down to the cell
    assert sc.xg1 == pytest.approx(39.5 * case.dx)
