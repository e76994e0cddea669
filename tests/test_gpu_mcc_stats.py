"""Null-collision MCC of the 5-reaction argon deck on the B200 against the oracle's collisions
(collisions.f90:1-207, collision_OMP :209-1040), matched statistically.

The two sides draw different random numbers: the device selects each slot with probability
Pmax (a Bernoulli trial per slot, drawn as geometric gaps between candidates from Philox
counter streams), the reference picks Nc = N Pmax
particles with replacement from one Park-Miller stream (collisions.f90:92-157, 273-283).  The
expected number of candidates, the per-particle collision probability and every outcome
distribution are the same, and that is what these tests check:

  * per-reaction collision counts and candidate counts agree within 4 sigma of their
    difference (Poisson counts: sigma = sqrt(n_gpu + n_oracle)), over K independent draws of
    the same particles;
  * the electrons of a 20-100 eV tail have sum(nu)/nu_max > 1 (nu_max is capped at
    nu_uplim = 6e7 1/s, main.f90:494), so the reaction taken depends on the ascending-nu order
    of indexx (collisions.f90:619-647); their per-reaction counts agree within 4 sigma;
  * post-collision electron and ion energies pass a two-sample Kolmogorov-Smirnov test at
    p > 0.01;
  * energy bookkeeping, on every event of the device: an ionization's two electrons share
    Ekr - Eth (15.76 eV), an excitation takes 11.5 eV, an elastic collision keeps the energy (to
    2e-3 of it plus 0.05 eV, the neutral's thermal motion and recoil), and the events of each
    kind number exactly the device's per-reaction counts;
  * after 100 steps of the 128x128 box at 100 particles per cell (push, Poisson, sort and MCC),
    the EEDF and the particle fluxes to the wall label agree with the oracle's own run of the
    same particles within Poisson error bars (5 sigma per EEDF bin, 4 sigma per flux).
"""
import math
import os

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs, deck as dk
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EXC, ION = 11.5, 15.76
R_ELASTIC, R_EXC, R_ION, R_CX, R_IEL = 0, 1, 2, 3, 4


def _energy(p, m):
    return 0.5 * m * (p[:, 3] ** 2 + p[:, 4] ** 2 + p[:, 5] ** 2) / dk.QE


def _isotropic(rng, n, speed):
    c = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    s = np.sqrt(1.0 - c * c)
    return np.stack([speed * s * np.cos(ph), speed * s * np.sin(ph), speed * c], axis=1)


def _particles(case, rng, n, m, T_eV, tail_frac, e_lo, e_hi):
    """Uniform positions; a Maxwellian at T_eV and a fraction with energies uniform in
    [e_lo, e_hi] eV, isotropic."""
    p = np.zeros((n, 6))
    p[:, 0] = rng.uniform(0.0, case.nx * case.dx, n)
    p[:, 1] = rng.uniform(0.0, case.ny * case.dy, n)
    nt = int(tail_frac * n)
    vt = math.sqrt(dk.QE * T_eV / m)
    p[nt:, 3:] = rng.normal(0.0, vt, (n - nt, 3))
    E = rng.uniform(e_lo, e_hi, nt)
    p[:nt, 3:] = _isotropic(rng, nt, np.sqrt(2.0 * dk.QE * E / m))
    return p


def _outcomes(before, after, m, n_prod):
    """Classifies one call's electron events: returns a dict of per-kind counts and arrays,
    and the fraction of events whose energy bookkeeping holds."""
    n0 = before.shape[0]
    e0 = _energy(before, m)
    e1 = _energy(after[:n0], m)
    changed = np.any(after[:n0, 3:] != before[:, 3:], axis=1)
    prod = after[n0:]
    assert prod.shape[0] == n_prod
    e_prod = _energy(prod, m)
    where = {(x, y): k for k, (x, y) in enumerate(zip(after[:n0, 0], after[:n0, 1])) if changed[k]}
    parent = np.array([where.get((x, y), -1) for x, y in zip(prod[:, 0], prod[:, 1])], dtype=np.int64)
    ok_ion = np.zeros(n_prod, dtype=bool)
    if n_prod:
        j = np.maximum(parent, 0)
        tol = 2e-3 * e0[j] + 0.05
        ok_ion = (parent >= 0) & (np.abs(e1[j] + e_prod - (e0[j] - ION)) <= tol)
    is_ion = np.zeros(n0, dtype=bool)
    is_ion[parent[parent >= 0]] = True
    rest = changed & ~is_ion
    d = e1 - e0
    tol = 2e-3 * e0 + 0.05
    is_exc = rest & (np.abs(d + EXC) <= tol)
    is_el = rest & (np.abs(d) <= tol)
    return {
        "n_el": int(is_el.sum()), "n_exc": int(is_exc.sum()), "n_ion": int(is_ion.sum()),
        "unclassified": int((rest & ~is_exc & ~is_el).sum()), "ok_ion": int(ok_ion.sum()),
        "n_prod": n_prod, "e_after": np.concatenate([e1[changed], e_prod]),
        "tail_el": int((is_el & (e0 > 20)).sum()), "tail_exc": int((is_exc & (e0 > 20)).sum()),
        "tail_ion": int((is_ion & (e0 > 20)).sum()),
    }


def _close(a, b, k=4.0):
    return abs(a - b) <= k * math.sqrt(max(a + b, 1.0))


def test_mcc_argon_deck_statistics_match_oracle(gpu_lib):
    from scipy.stats import ks_2samp
    from jd_lepic_b200.simulation import GpuSimulation

    case = configs.case0(ppc=25, nx=128, ny=128)     # 409,600 particles per species
    n = case.n_particles
    s = GpuSimulation(case, tile=(16, 16), load=False, capacity=n + 65536)
    try:
        me, mi = s.sp.mass[0], s.sp.mass[1]
        rng = np.random.default_rng(2024)
        s.put_particles(0, _particles(case, rng, n, me, 2.0, 0.2, 20.0, 100.0))
        s.put_particles(1, _particles(case, rng, n, mi, 0.03, 0.3, 1.0, 50.0))
        p0 = [s.get_particles(k) for k in range(2)]   # the FP32-stored state, given to both sides
        cfg = O.make_cfg(case, s.sp)
        xsh = O.XsHolder(s.xs)
        assert s.xs.ncol == 5
        K = 20
        g = {"coll": np.zeros(5, np.int64), "cand": np.zeros(2, np.int64)}
        o = {"coll": np.zeros(5, np.int64), "cand": np.zeros(2, np.int64)}
        gE, oE, gI, oI = [], [], [], []
        gt = np.zeros(3, np.int64)
        ot = np.zeros(3, np.int64)
        for k in range(K):
            s.put_particles(0, p0[0])
            s.put_particles(1, p0[1])
            m0 = s.mcc_stats()
            m1 = s.collide(11 + 10 * k)
            dcoll = np.array(m1["n_coll"]) - np.array(m0["n_coll"])
            dadd = np.array(m1["n_add"]) - np.array(m0["n_add"])
            g["coll"] += dcoll
            g["cand"] += np.array(m1["n_cand"]) - np.array(m0["n_cand"])
            ae, ai = s.get_particles(0), s.get_particles(1)
            assert ae.shape[0] == n + dadd[0] and ai.shape[0] == n + dadd[1]
            assert dadd[0] == dadd[1] == dcoll[R_ION]           # a new electron and ion per ionization
            out = _outcomes(p0[0], ae, me, int(dadd[0]))
            # the device's bookkeeping holds on every event
            assert out["ok_ion"] == out["n_prod"] == dcoll[R_ION]
            assert out["n_ion"] == dcoll[R_ION] and out["n_exc"] == dcoll[R_EXC] and out["n_el"] == dcoll[R_ELASTIC]
            assert out["unclassified"] == 0
            gE.append(out["e_after"])
            gt += [out["tail_el"], out["tail_exc"], out["tail_ion"]]
            ch = np.any(ai[:n, 3:] != p0[1][:, 3:], axis=1)
            gI.append(_energy(ai[:n][ch], mi))
            assert ch.sum() == dcoll[R_CX] + dcoll[R_IEL]
            # the oracle from the same particles, its own ran2 stream
            rc, oa, tal, _ = O.collisions(cfg, xsh, p0, seed=1000 + 7919 * k)
            assert rc == 0
            oc = np.array(tal.n_coll[:5])
            o["coll"] += oc
            o["cand"] += np.array(tal.n_cand[:2])
            oo = _outcomes(p0[0], oa[0], me, int(tal.n_add[0]))
            # picks with replacement may hit a particle twice: the oracle's classification is
            # exact up to those few
            assert oo["ok_ion"] >= oo["n_prod"] - 3 and abs(oo["n_exc"] - oc[R_EXC]) <= 3
            oE.append(oo["e_after"])
            ot += [oo["tail_el"], oo["tail_exc"], oo["tail_ion"]]
            chi = np.any(oa[1][:n, 3:] != p0[1][:, 3:], axis=1)
            oI.append(_energy(oa[1][:n][chi], mi))
        for r in range(5):
            assert _close(g["coll"][r], o["coll"][r]), (r, g["coll"], o["coll"])
        assert min(g["coll"]) > 50 and min(o["coll"]) > 50
        for sp in range(2):
            assert _close(g["cand"][sp], o["cand"][sp]), (g["cand"], o["cand"])
        # sum(nu)/nu_max > 1 in the tail: ascending-nu order decides; without it elastic (the
        # largest nu) would take every tail collision
        assert gt[2] > 0.2 * gt.sum() and gt[1] > 0
        for q in range(3):
            assert _close(gt[q], ot[q]), (gt, ot)
        pe = ks_2samp(np.concatenate(gE), np.concatenate(oE)).pvalue
        pi = ks_2samp(np.concatenate(gI), np.concatenate(oI)).pvalue
        assert pe > 0.01, pe
        assert pi > 0.01, pi
    finally:
        s.close()


def test_cfg0_100_steps_eedf_and_wall_flux_match_oracle(gpu_lib):
    """The 128x128 box at 100 particles per cell, 100 steps (MCC at steps 11, 21, ..., 91) on
    the device and in the oracle from the same initial particles."""
    import ctypes as C
    from jd_lepic_b200.simulation import GpuSimulation

    case = configs.case0()
    s = GpuSimulation(case, tile=(16, 16))
    try:
        p0 = [s.get_particles(k) for k in range(2)]
        n0 = [p.shape[0] for p in p0]
        orc = O.OracleSimulation(case, nthreads=max(1, min(32, os.cpu_count() or 1)), particles=p0, seed=1)
        o_coll = np.zeros(5, np.int64)
        o_add = np.zeros(2, np.int64)
        for it in range(1, 101):
            s.step(it)
            orc.step(it)
            if it > 1 and it % 10 == 1:
                o_coll += np.array(orc.mcc.n_coll[:5])
                o_add += np.array(orc.mcc.n_add[:2])
        s.sync()
        me = s.sp.mass[0]
        ge = _energy(s.get_particles(0), me)
        oe = _energy(orc.vxp[0][:orc.np_tot[0]], me)
        bins = np.concatenate([np.linspace(0.0, 10.0, 41), [12.0, 15.0, 20.0, 1e9]])
        hg, _ = np.histogram(ge, bins)
        ho, _ = np.histogram(oe, bins)
        z = (hg - ho) / np.sqrt(np.maximum(hg + ho, 1))
        assert np.abs(z).max() < 5.0, z
        # mean energy of the EEDF to its statistical error
        assert abs(ge.mean() - oe.mean()) <= 5 * math.sqrt(ge.var() / ge.size + oe.var() / oe.size)
        # fluxes to the wall (label 1 on all four sides): the device's p_mac tallies, the
        # oracle's particles that left (loaded + created - remaining)
        t = capi.LepicTallies()
        s.check(s.lib.lepic_gpu_get_tallies(s.ctx, C.byref(t), 0), "get_tallies")
        mc = s.mcc_stats()
        g_add = mc["n_add"]
        for sp in range(2):
            g_flux = t.n_loss[sp][1]
            assert sum(t.n_loss[sp]) == g_flux
            o_flux = n0[sp] + o_add[sp] - orc.np_tot[sp]
            assert s.push_stats()["np_tot"][sp] == n0[sp] + g_add[sp] - g_flux
            assert _close(g_flux, o_flux), (sp, g_flux, o_flux)
        assert t.n_loss[0][1] > 0
        for r in range(5):
            assert _close(mc["n_coll"][r], o_coll[r]), (r, mc["n_coll"], o_coll)
    finally:
        s.close()
