"""Species and reaction decks in the reference's text format, and the collision tables the
device consumes.

``read_reactions`` restates the parsing of ``Src/read_reactions.f90:112-365`` (IONS /
NEUTRALS / REACTION sections, ``----`` delimited tables, scale factors, reaction-type
keywords) and ``ordering`` restates ``Src/read_reactions.f90:511-697`` (union energy grid,
resampling of every cross section onto it, (sigma*v)_max with the 0.1 eV cut-off, per-species
reaction lists).  ``write_deck`` writes synthetic decks in the same format so the reader is
exercised end to end.

Species numbering is 0-based here: 0 is the electron (``read_reactions.f90:103-107``), then
the species in file order.  Neutral masses are stored negative
(``read_reactions.f90:200-205``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MAXSP = 8
MAXCOL = 64
AMU = 1.66053886e-27
ME = 9.10938188e-31
QE = float(np.float32(1.60217646e-19))  # main.f90:120 assigns a default-real literal
EPS0 = 8.854187817e-12
KB = 1.380649e-23

RTYPE_KEYWORDS = [  # read_reactions.f90:275-307, in the order the reference tests them
    ("COLLISION", 1), ("IONIZATION", 2), ("EXCITATION", 3), ("CHARGEEXCHANGE", 4),
    ("DISSOCIATION", 5),
]
RTYPE_PREFIXES = [("DATT", 2), ("DION", 2), ("DISS", 5), ("ELA", 1), ("EXC", 3), ("ION", 2),
                  ("VIBB", 3), ("VIBS", 3), ("CEX", 4), ("DRE", 5), ("RRE", 2)]


@dataclass
class Reaction:
    label: str
    reactants: list[int]
    byproducts: list[int]
    rtype: int
    eth: float
    energy: np.ndarray   # eV, scaled
    sigma: np.ndarray    # m^2, scaled


@dataclass
class Deck:
    names: list[str]
    mass: list[float]        # kg, neutrals negative
    charge: list[float]      # C
    temp: list[float]        # eV (electron temperature comes from the case)
    ni0: list[float]         # fraction for charged species, density for neutrals
    reactions: list[Reaction] = field(default_factory=list)

    @property
    def nsp(self) -> int:
        return len(self.names)

    @property
    def ntype(self) -> int:  # charged species (main.f90:175)
        return sum(1 for q in self.charge if q != 0.0)


def _rtype_of(word: str) -> int:
    w = word.strip()
    code = 0
    for kw, v in RTYPE_KEYWORDS:
        if w == kw or w == kw.lower():
            code = v
    for pre, v in RTYPE_PREFIXES:
        if w[: len(pre)] in (pre, pre.lower()):
            code = v
    return code


def read_reactions(text: str, ngas: float) -> Deck:
    """Parses a species/reaction deck (read_reactions.f90:112-365)."""
    lines = text.splitlines()
    deck = Deck(names=["[e]"], mass=[ME], charge=[-QE], temp=[0.0], ni0=[1.0])
    i = 0

    def first_token(s: str) -> str:
        t = s.split()
        return t[0][:4] if t else ""

    while i < len(lines):
        tok = first_token(lines[i])
        i += 1
        if tok in ("IONS", "Ions", "ions", "NEUT", "Neut", "neut"):
            while i < len(lines) and first_token(lines[i]) != "----":
                i += 1
            i += 1
            while i < len(lines):
                s = lines[i]
                i += 1
                if s[:6][:2] == "--":
                    break
                name = s[:6].strip()
                vals = [float(v) for v in s[6:].split()[:4]]
                m, q, t, n = vals
                q = q * QE
                m = m * AMU
                if q == 0.0:
                    n = n * ngas
                    m = -abs(m)
                deck.names.append(name)
                deck.mass.append(m)
                deck.charge.append(q)
                deck.temp.append(t)
                deck.ni0.append(n)
        elif tok in ("REAC", "Reac", "reac"):
            label = lines[i].split()[0]
            i += 1
            parts = []
            n_re = None
            pos = 0
            while pos < len(label):
                ch = label[pos]
                if ch == ">":
                    n_re = len(parts)
                if ch == "[":
                    end = label.index("]", pos)
                    nm = label[pos:end + 1]
                    if nm not in deck.names:
                        raise ValueError(f"unknown particle {nm} in reaction {label}")
                    parts.append(deck.names.index(nm))
                    pos = end
                pos += 1
            if n_re is None:
                raise ValueError(f"reaction {label} has no '->'")
            eth, _de = (float(v) for v in lines[i].split()[:2])
            i += 1
            sc1, sc2 = (float(v) for v in lines[i].split()[:2])
            i += 1
            rt = _rtype_of(lines[i].split()[0])
            i += 1
            if rt == 0:
                raise ValueError(f"unknown reaction type in {label}")
            while i < len(lines) and first_token(lines[i]) != "----":
                i += 1
            i += 1
            es, ss = [], []
            while i < len(lines):
                s = lines[i]
                i += 1
                if s.strip()[:4] == "----":
                    break
                e, sg = (float(v) for v in s.split()[:2])
                es.append(e * sc1)
                ss.append(sg * sc2)
            deck.reactions.append(Reaction(label, parts[:n_re], parts[n_re:], rt, eth * sc1,
                                           np.array(es), np.array(ss)))
    return deck


@dataclass
class XsTables:
    npt: int
    ncol: int
    sig_Er: np.ndarray        # [npt]
    sig: np.ndarray           # [ncol, npt]
    Eth: np.ndarray           # [ncol]
    col_info: np.ndarray      # [ncol, 10] int32, 0-based species
    p_ncol: np.ndarray        # [MAXSP] int32
    sig_list: np.ndarray      # [MAXSP, MAXCOL] int32
    sigv_mx: np.ndarray       # [MAXSP, MAXCOL]
    flag_ionrep: int = 0
    fEk: float = 0.5


def ordering(deck: Deck, qe: float = QE) -> XsTables:
    """Union energy grid, resampled cross sections and (sigma*v)_max
    (read_reactions.f90:511-697)."""
    ncol = len(deck.reactions)
    allE = np.concatenate([r.energy for r in deck.reactions])
    order = np.argsort(allE, kind="stable")
    union = []
    prev = 1.0e10
    for k in order:  # :563-571, drop repeated energies
        if allE[k] != prev:
            union.append(allE[k])
            prev = allE[k]
    sig_Er = np.array(union, dtype=np.float64)
    npt = len(sig_Er)
    sig = np.zeros((ncol, npt))
    sig_p = 0.0  # a subroutine local: keeps its value when no interval matches
    for icol, r in enumerate(deck.reactions):  # :592-644
        Et = np.append(r.energy, 0.0)
        St = np.append(r.sigma, 0.0)
        for ipt, ekp in enumerate(sig_Er):
            for k in range(len(r.energy)):
                ek_l, ek_r, s_l, s_r = Et[k], Et[k + 1], St[k], St[k + 1]
                if ekp < ek_l:
                    sig_p = s_l
                    break
                if ek_l <= ekp <= ek_r:
                    sig_p = s_l + (ekp - ek_l) * (s_r - s_l) / (ek_r - ek_l)
                    break
            sig[icol, ipt] = sig_p
    col_info = np.zeros((ncol, 10), dtype=np.int32)
    sig_list = np.zeros((MAXSP, MAXCOL), dtype=np.int32)
    sigv_mx = np.zeros((MAXSP, MAXCOL))
    p_ncol = np.zeros(MAXSP, dtype=np.int32)
    for icol, r in enumerate(deck.reactions):
        n_re, n_by = len(r.reactants), len(r.byproducts)
        ci = [n_re, n_by] + r.reactants + r.byproducts + [r.rtype, sum(1 for b in r.byproducts if b == 0)]
        col_info[icol, : len(ci)] = ci
        r1, r2 = ci[2], ci[3]  # col_info(icol, ind_nby+1) and col_info(icol, ind_nby+2)
        sig_list[r1, p_ncol[r1]] = icol  # :653-655
        p_ncol[r1] += 1
        m1, m2 = abs(deck.mass[r1]), abs(deck.mass[r2])
        mu = m1 * m2 / (m1 + m2)
        for ipt in range(npt):  # :657-672
            vr = math.sqrt(2.0 * sig_Er[ipt] * qe / mu)
            if sig_Er[ipt] >= 0.1:
                sigv_mx[r1, icol] = max(sigv_mx[r1, icol], vr * sig[icol, ipt])
    eth = np.array([r.eth for r in deck.reactions])
    return XsTables(npt, ncol, sig_Er, sig, eth, col_info, p_ncol, sig_list, sigv_mx)


# ------------------------------------------------------------------------------------------
# Synthetic decks (the cross sections named by the benchmark configurations)

def energy_grid(emax: float = 1.0e5, n: int = 400) -> np.ndarray:
    """0 eV followed by log-spaced points from 1 meV to emax (all reactions share it)."""
    return np.concatenate([[0.0], np.logspace(-3.0, math.log10(emax), n)])


def sigma_constant(E, s0):
    return np.full_like(E, s0)


def sigma_threshold_peak(E, eth, epk, s_pk):
    """Zero below eth, rises linearly-exponentially to s_pk at epk."""
    x = np.clip((E - eth) / (epk - eth), 0.0, None)
    return np.where(E > eth, s_pk * x * np.exp(1.0 - x), 0.0)


def sigma_lotz(E, eth, s_pk):
    """Single-shell Lotz form s(E) ~ ln(E/I)/(E I), scaled to its maximum s_pk at E = e*I."""
    with np.errstate(divide="ignore", invalid="ignore"):
        v = s_pk * math.e * eth * np.log(E / eth) / E
    return np.where(E > eth, v, 0.0)


def write_deck(ion: str, ion_mass: float, ion_temp: float, neutral: str, neu_temp: float,
               reactions: list[tuple[str, str, float, np.ndarray, np.ndarray]]) -> str:
    """Text of a deck in the reference's format (input_dir/argon.dat:1-50)."""
    out = ["IONS", "name   mass  charge  temp.(eV)  n/n0", "-" * 37,
           f"{ion:<6s}   {ion_mass:.2f}     1.     {ion_temp:.4f}   1.", "-" * 37, "",
           "NEUTRALS", "name   mass  charge  temp.(eV)  n/n0", "-" * 37,
           f"{neutral:<6s}   {-ion_mass:.2f}     0.     {neu_temp:.4f}   1.", "-" * 37, ""]
    for label, rtype, eth, E, S in reactions:
        out += ["REACTION", label, f" {eth:.4f}    0.", " 1.    1.", rtype, "-" * 60]
        out += [f"  {e:.8e}  {s:.8e}" for e, s in zip(E, S)]
        out += ["-" * 60, ""]
    return "\n".join(out) + "\n"


def argon_deck(ion_temp: float = 0.03, gas_temp_k: float = 300.0) -> str:
    """Synthetic argon set: e-Ar elastic 1e-19 m^2; excitation 11.5 eV, peak 5e-21 m^2;
    ionization 15.76 eV (Lotz), peak 3e-20 m^2; Ar+-Ar charge exchange 5e-19 m^2 and
    isotropic elastic 3e-19 m^2."""
    E = energy_grid()
    reac = [
        ("[e]+[Ar]->[e]+[Ar]", "COLLISION", 0.0, E, sigma_constant(E, 1.0e-19)),
        ("[e]+[Ar]->[e]+[Ar]", "EXCITATION", 11.5, E, sigma_threshold_peak(E, 11.5, 30.0, 5.0e-21)),
        ("[e]+[Ar]->[e]+[e]+[Ar+]", "IONIZATION", 15.76, E, sigma_lotz(E, 15.76, 3.0e-20)),
        ("[Ar+]+[Ar]->[Ar]+[Ar+]", "CHARGEEXCHANGE", 0.0, E, sigma_constant(E, 5.0e-19)),
        ("[Ar+]+[Ar]->[Ar+]+[Ar]", "COLLISION", 0.0, E, sigma_constant(E, 3.0e-19)),
    ]
    kT = KB * gas_temp_k / QE
    return write_deck("[Ar+]", 39.95, ion_temp, "[Ar]", kT, reac)


def argon_dsmc_deck(sigma: float = 2.0e-15, e_cut: float = 20.0, ion_temp: float = 0.03,
                    gas_temp_k: float = 300.0, with_neutral: bool = False) -> str:
    """Electron-ion elastic scattering on the ions themselves (a charged target, collisions by
    DSMC; the first reaction of the reference's argon set), sigma constant up to e_cut eV and
    zero above; optionally with the e-Ar elastic reaction on the background gas."""
    E = energy_grid()
    sig = np.where(np.asarray(E) <= e_cut, sigma, 0.0)
    reac = [("[e]+[Ar+]->[e]+[Ar+]", "COLLISION", 0.0, E, sig)]
    if with_neutral:
        reac.append(("[e]+[Ar]->[e]+[Ar]", "COLLISION", 0.0, E, sigma_constant(E, 1.0e-19)))
    kT = KB * gas_temp_k / QE
    return write_deck("[Ar+]", 39.95, ion_temp, "[Ar]", kT, reac)


def helium_deck(ion_temp: float = 0.03, gas_temp_k: float = 300.0) -> str:
    """Synthetic helium set: e-He elastic 6e-20 m^2; excitation 19.8 eV (peak 2e-21 m^2 at
    40 eV); ionization 24.6 eV (Lotz, peak 3.5e-21 m^2); He+-He charge exchange 3e-19 m^2."""
    E = energy_grid()
    reac = [
        ("[e]+[He]->[e]+[He]", "COLLISION", 0.0, E, sigma_constant(E, 6.0e-20)),
        ("[e]+[He]->[e]+[He]", "EXCITATION", 19.8, E, sigma_threshold_peak(E, 19.8, 40.0, 2.0e-21)),
        ("[e]+[He]->[e]+[e]+[He+]", "IONIZATION", 24.6, E, sigma_lotz(E, 24.6, 3.5e-21)),
        ("[He+]+[He]->[He]+[He+]", "CHARGEEXCHANGE", 0.0, E, sigma_constant(E, 3.0e-19)),
    ]
    kT = KB * gas_temp_k / QE
    return write_deck("[He+]", 4.0026, ion_temp, "[He]", kT, reac)
