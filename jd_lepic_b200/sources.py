"""Deck values of the particle sources -> ``lepic_source_config``.

The conversions the reference applies while reading its input deck and starting up:
the heating region in cm with a negative x bound selecting the disk (read_input.f90:43-55),
the driver count, absorbed powers and heating frequency (read_input.f90:80-89), the injected
current and its option (read_input.f90:90-98), the injected-electron temperature THm whose
sign selects flag_Tp (read_input.f90:147-151), and the derived heating parameters nudt,
eheat_type and flag_gpp (main.f90:493-500).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import _capi as capi


@dataclass
class SourceDeck:
    heat_region_cm: tuple = (0.0, 0.0, 0.0, 0.0)  # xl_pow, xr_pow, yl_pow, yr_pow [cm]
    n_icp: int = 1                                  # drivers (< 0: iterative Pabs)
    Pabs: tuple = (0.0,)                            # absorbed power per driver [W] (<= 0: fixed Te)
    nu_h: float = -1.0                              # heating frequency [1/s] (< 0: off)
    I_inj: float = -1.0                             # injected current [A] (< 0: off)
    opt_inj: int = 1                                # 1 fixed current, 2 pair per lost ion, 3 beam along z,
                                                    # 4 cathode emission at x = 0; < 0 Gaussian
    THm: float = 0.0                                # [eV]; < 0 sets flag_Tp
    ns_heat: int = 4
    ns_inj: int = 1
    ni0: tuple = (1.0,)                             # charged-species fractions
    tag_neg: int = -1                               # 0-based negative-ion species, -1 none
    flag_diffsrc: int = 0
    nproc_mpi: int = 1
    te_update: int = 1
    vt: tuple = field(default_factory=tuple)        # initial heating speed per band [m/s]
    seed: int = 12345
    # part_flux_emitter: jne [mA/cm^2] (<= 0: off), emitted species, grid plane and holes [cm]
    jne: float = 0.0
    ptype_fx: int = 0
    tag_b: int = -1                                 # 0-based chamfer-emitted species, -1 none
    xg1_cm: float = 0.0
    Lg_cm: float = 0.0
    Lh_cm: float = 0.0
    n_holes: int = 0
    chamfer_m: tuple = ()                           # chmfrd_array (x1, x2, ymax/2-y1, ymax/2-y2) [m]
    th_B: float = 0.0                               # |opt_inj| = 4: angle of B to the x axis [rad]


def cathode_angle(opt_inj: int, flag_nmn: int, Bx11: float, By11: float) -> float:
    """th_B of main.f90:450-452: atan(By/Bx) of the field at node (1, 1) when the cathode
    option runs with the Neumann boundary and Bx is not zero, else 0."""
    if opt_inj == 4 and flag_nmn == 1 and abs(Bx11) > 0.0:
        return math.atan(By11 / Bx11)
    return 0.0


def source_config(d: SourceDeck, dt: float, vt0_e: float, dy: float = 0.0) -> capi.LepicSourceConfig:
    """The lepic_source_config of a deck; vt0_e is the electron vt0 (the initial heating speed
    when the deck gives none, and the constant one when particles are injected); dy the cell
    height, to which the hole size is rounded down (generate_boundary.f90:267-270)."""
    c = capi.LepicSourceConfig()
    xl, xr, yl, yr = (v * 1e-2 for v in d.heat_region_cm)
    c.flag_c = 1 if (xl < 0.0 or xr < 0.0) else 0
    c.xl_pow, c.xr_pow, c.yl_pow, c.yr_pow = abs(xl), abs(xr), yl, yr
    n_icp = abs(int(d.n_icp))
    if not 1 <= n_icp <= capi.MAXICP:
        raise ValueError(f"n_icp={d.n_icp} out of range")
    c.n_icp = n_icp
    c.flag_heat = 0 if d.nu_h < 0.0 else 1
    c.nu_h = max(d.nu_h, 0.0)
    c.ns_heat = d.ns_heat
    c.nudt = c.nu_h * (d.ns_heat * dt)
    pabs = list(d.Pabs) + [d.Pabs[-1]] * (n_icp - len(d.Pabs))
    for b in range(n_icp):
        c.Pabs[b] = pabs[b]
    c.eheat_type = 1
    c.flag_gpp = 1 if (d.opt_inj < 0 and pabs[0] > 0.0) else 0
    c.Pabs_cor = 1.0
    vt = list(d.vt) if d.vt else [vt0_e] * n_icp
    for b in range(n_icp):
        c.vt[b] = vt[b] if b < len(vt) else vt[-1]
    c.te_update = d.te_update if pabs[0] > 0.0 else 0
    c.flag_inj = 0 if d.I_inj < 0.0 else 1
    c.I_inj = 0.0 if (d.I_inj < 0.0 or abs(d.opt_inj) == 2) else d.I_inj
    c.opt_inj = d.opt_inj
    c.ns_inj = d.ns_inj
    c.flag_Tp = 1 if d.THm < 0.0 else 0
    c.THm = abs(d.THm)
    c.flag_diffsrc = d.flag_diffsrc
    c.tag_neg = d.tag_neg
    c.nproc_mpi = d.nproc_mpi
    for s, v in enumerate(d.ni0[:capi.MAXSP]):
        c.ni0[s] = v
    c.seed = d.seed
    c.js = d.jne * 10.0 if d.jne > 0.0 else 0.0     # mA/cm^2 -> A/m^2 (part_flux_emitter.f90:22)
    c.ptype_fx = d.ptype_fx
    c.tag_b = d.tag_b
    c.ns_Hm = 1                                       # main.f90:496
    c.n_holes = d.n_holes
    c.xg1, c.Lg = d.xg1_cm * 1e-2, d.Lg_cm * 1e-2
    Lh = d.Lh_cm * 1e-2
    c.Lh = math.floor(Lh / dy) * dy if dy > 0.0 else Lh
    c.th_B = d.th_B if abs(d.opt_inj) == 4 else 0.0
    if d.chamfer_m:
        c.flag_chmfrd = 1
        for k in range(4):
            c.chmfrd[k] = d.chamfer_m[k]
    return c
