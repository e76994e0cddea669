"""Host driver over the C ABI: the in-scope part of the reference's start-up
(main.f90:140-600) and time loop (main.f90:818-1090) with every hot routine on the B200.

``species_params`` computes the per-species constants the reference derives at start-up
(vt0 = sqrt(2 qe T/|m|), Nm = n*Vc/np_cell, nu_uplim; main.f90:466-495) and is shared with
the CPU restatement so both see identical inputs.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from . import deck as dk
from .configs import Case

NU_UPLIM_E = 6.0e7   # main.f90:494
NU_UPLIM_ION = 5.0e6  # main.f90:495


@dataclass
class SpeciesParams:
    names: list
    ntype: int
    nsp: int
    charge: np.ndarray
    mass: np.ndarray
    vt0: np.ndarray
    Nm: np.ndarray
    np_mx: np.ndarray
    nu_uplim: np.ndarray


def mean_density(case: Case) -> float:
    """Cell-averaged density of the load profile (uniform: n0)."""
    if case.profile == 0:
        return case.n0
    x = (np.arange(case.nx) + 0.5) * case.dx - 0.5 * case.nx * case.dx
    y = (np.arange(case.ny) + 0.5) * case.dy - 0.5 * case.ny * case.dy
    X, Y = np.meshgrid(x, y)
    n = case.n_floor + (case.n_peak - case.n_floor) * np.exp(-(X * X + Y * Y) / (2 * case.sigma ** 2))
    return float(n.mean())


def species_params(case: Case, d: dk.Deck) -> SpeciesParams:
    nsp = d.nsp
    ntype = d.ntype
    charge = np.zeros(dk.MAXSP)
    mass = np.zeros(dk.MAXSP)
    vt0 = np.zeros(dk.MAXSP)
    Nm = np.zeros(dk.MAXSP)
    np_mx = np.zeros(dk.MAXSP)
    nu_up = np.zeros(dk.MAXSP)
    Vc = case.dx * case.dy * case.zmax
    nbar = mean_density(case)
    for s in range(nsp):
        charge[s] = d.charge[s]
        mass[s] = d.mass[s]
        T = case.te if s == 0 else d.temp[s]
        vt0[s] = math.sqrt(2.0 * dk.QE * T / abs(d.mass[s]))  # main.f90:468
        if d.charge[s] != 0.0:
            Nm[s] = nbar * Vc / case.ppc  # main.f90:471
        else:
            Nm[s] = case.ngas * Vc / case.ppc
            np_mx[s] = d.ni0[s]  # main.f90:177
    nu_up[0] = NU_UPLIM_E
    nu_up[1:ntype] = NU_UPLIM_ION
    return SpeciesParams(d.names, ntype, nsp, charge, mass, vt0, Nm, np_mx, nu_up)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


class GpuSimulation:
    """One device context running a Case through the C ABI."""

    def __init__(self, case: Case, tile=(16, 16), capacity_factor: float = 1.3, load: bool = True,
                 capacity: int | None = None, config: dict | None = None):
        self.lib = capi.load_library()
        self.case = case
        self.deck = dk.read_reactions(case.deck_text, case.ngas)
        self.xs = dk.ordering(self.deck)
        self.sp = species_params(case, self.deck)
        cfg = capi.LepicConfig()
        cfg.nx, cfg.ny = case.nx, case.ny
        cfg.dx, cfg.dy, cfg.zmax, cfg.dt = case.dx, case.dy, case.zmax, case.dt
        cfg.eps0, cfg.qe = dk.EPS0, dk.QE
        cfg.flag_pbc, cfg.flag_spec, cfg.flag_nmn = case.flag_pbc, case.flag_spec, case.flag_nmn
        cfg.flag_B = case.flag_B
        cfg.flag_B_pos = 0
        for k in range(3):
            cfg.Bc[k] = case.Bc[k]
        cfg.ntype, cfg.nsp = self.sp.ntype, self.sp.nsp
        for s in range(dk.MAXSP):
            cfg.charge[s] = self.sp.charge[s]
            cfg.mass[s] = self.sp.mass[s]
            cfg.Nm[s] = self.sp.Nm[s]
            cfg.vt0[s] = self.sp.vt0[s]
            cfg.np_mx[s] = self.sp.np_mx[s]
            cfg.nu_uplim[s] = self.sp.nu_uplim[s]
        cfg.ns_coll, cfg.nsort = 10, 10  # main.f90:479-480
        cfg.ng = case.levels()
        cfg.ncycl = 20000  # main.f90:261
        cfg.omega = 1.4    # iterative_solver.f90:28
        cap = capacity if capacity is not None else int(case.n_load * capacity_factor) + 4096
        for s in range(self.sp.ntype):
            cfg.capacity[s] = cap
        cfg.seed = case.seed
        cfg.tile_w, cfg.tile_h = (tile if tile else (0, 0))
        for k, v in (config or {}).items():   # lepic_config fields set by name (e.g. ncycl)
            setattr(cfg, k, v)
        self.cfg = cfg
        self._bcnd = np.ascontiguousarray(case.bcnd, dtype=np.int32)
        self._phi0 = np.ascontiguousarray(case.phi0, dtype=np.float64)
        self._Bi = np.ascontiguousarray(case.Bi, dtype=np.float64) if case.Bi is not None else None
        t = self.xs
        self._xs_keep = [np.ascontiguousarray(t.sig_Er), np.ascontiguousarray(t.sig),
                         np.ascontiguousarray(t.Eth), np.ascontiguousarray(t.col_info, dtype=np.int32),
                         np.ascontiguousarray(t.p_ncol, dtype=np.int32),
                         np.ascontiguousarray(t.sig_list, dtype=np.int32), np.ascontiguousarray(t.sigv_mx)]
        k = self._xs_keep
        xs = capi.LepicXsTables(t.npt, t.ncol, _dp(k[0]), _dp(k[1]), _dp(k[2]), _ip(k[3]), _ip(k[4]),
                                _ip(k[5]), _dp(k[6]), t.flag_ionrep, t.fEk)
        self._xs = xs
        self.ctx = C.c_void_p()
        rc = self.lib.lepic_gpu_create(C.byref(cfg), _ip(self._bcnd), _dp(self._phi0), _dp(self._Bi),
                                       C.byref(xs), C.byref(self.ctx))
        if rc != 0:
            msg = self.lib.lepic_gpu_last_error(None)
            raise capi.LepicError(rc, "lepic_gpu_create", msg.decode() if msg else "")
        if load:
            self.load()

    # --------------------------------------------------------------------------------------
    def check(self, rc: int, where: str):
        if rc != 0:
            msg = self.lib.lepic_gpu_last_error(self.ctx)
            raise capi.LepicError(rc, where, msg.decode() if msg else "")

    def load(self, n: int | None = None, seed: int | None = None):
        c = self.case
        spec = capi.LepicLoadSpec(n if n is not None else c.n_load, c.profile, 0.0, c.n_peak,
                                  c.n_floor, c.sigma, seed if seed is not None else c.seed)
        self.check(self.lib.lepic_gpu_load_particles(self.ctx, C.byref(spec)), "load_particles")
        self.check(self.lib.lepic_gpu_charge_deposition(self.ctx), "charge_deposition")

    def put_particles(self, ptype: int, vxp: np.ndarray):
        a = np.ascontiguousarray(vxp, dtype=np.float64)
        self.check(self.lib.lepic_gpu_put_particles(self.ctx, ptype, _dp(a), a.shape[0]), "put_particles")

    def get_particles(self, ptype: int) -> np.ndarray:
        n = C.c_int64()
        self.check(self.lib.lepic_gpu_get_particles(self.ctx, ptype, None, 0, C.byref(n)), "get_particles")
        out = np.zeros((n.value, 6))
        self.check(self.lib.lepic_gpu_get_particles(self.ctx, ptype, _dp(out), n.value, C.byref(n)),
                   "get_particles")
        return out

    def step(self, it: int):
        self.check(self.lib.lepic_gpu_step(self.ctx, it, self.case.eps, self.case.poisson_mode), "step")

    def run(self, nsteps: int, start: int = 1):
        for it in range(start, start + nsteps):
            self.step(it)
        self.sync()

    def sync(self):
        self.check(self.lib.lepic_gpu_sync(self.ctx), "sync")

    def deposit(self):
        self.check(self.lib.lepic_gpu_charge_deposition(self.ctx), "charge_deposition")

    def calc_rhs(self) -> np.ndarray:
        out = np.zeros((self.case.ny + 1, self.case.nx + 1))
        self.check(self.lib.lepic_gpu_calc_rhs(self.ctx, _dp(out)), "calc_rhs")
        return out

    def solve(self, eps: float | None = None, mode: int | None = None, phi: np.ndarray | None = None):
        st = capi.LepicSolveStats()
        arr = None
        if phi is not None:
            arr = np.ascontiguousarray(phi, dtype=np.float64).copy()
        self.check(self.lib.lepic_gpu_iterative_solver(
            self.ctx, _dp(arr), self.case.eps if eps is None else eps,
            self.case.poisson_mode if mode is None else mode, C.byref(st)), "iterative_solver")
        return {"cycles": st.cycles, "sweeps_fine": st.sweeps_fine, "res_l1": st.res_l1,
                "res_l2_rel": st.res_l2_rel, "ktot": st.ktot, "phi": arr}

    def efield(self) -> np.ndarray:
        out = np.zeros((self.case.ny + 3, self.case.nx + 3, 2))
        self.check(self.lib.lepic_gpu_calc_efield(self.ctx, _dp(out)), "calc_efield")
        return out

    def sort(self, ptype: int, plist: bool = False):
        if plist:
            n = self.case.nx + self.case.nx * self.case.ny + 2
            out = np.zeros(n, dtype=np.int32)
            self.check(self.lib.lepic_gpu_part_sorting(self.ctx, ptype, _ip(out)), "part_sorting")
            return out
        self.check(self.lib.lepic_gpu_part_sorting(self.ctx, ptype, None), "part_sorting")
        return None

    def collide(self, it: int) -> dict:
        st = capi.LepicMccStats()
        self.check(self.lib.lepic_gpu_collisions(self.ctx, it, C.byref(st)), "collisions")
        return self.mcc_stats()

    def push(self, it: int):
        self.check(self.lib.lepic_gpu_push_deposit(self.ctx, it, None), "push_deposit")

    def grid(self, which: int) -> np.ndarray:
        c = self.case
        if which == capi.GRID_RHS:
            out = np.zeros((c.ny + 1, c.nx + 1))
        elif which == capi.GRID_EI:
            out = np.zeros((c.ny + 3, c.nx + 3, 2))
        else:
            out = np.zeros((c.ny + 3, c.nx + 3))
        self.check(self.lib.lepic_gpu_get_grid(self.ctx, which, _dp(out)), "get_grid")
        return out

    def set_phi(self, phi: np.ndarray):
        a = np.ascontiguousarray(phi, dtype=np.float64)
        self.check(self.lib.lepic_gpu_set_grid(self.ctx, capi.GRID_PHI, _dp(a)), "set_grid")

    def push_stats(self) -> dict:
        st = capi.LepicPushStats()
        self.check(self.lib.lepic_gpu_get_push_stats(self.ctx, C.byref(st)), "get_push_stats")
        n = self.sp.ntype
        return {"np_tot": list(st.np_tot[:n]), "n_lost": list(st.n_lost[:n]),
                "n_dead": list(st.n_dead[:n]), "n_slots": list(st.n_slots[:n])}

    def mcc_stats(self) -> dict:
        st = capi.LepicMccStats()
        self.check(self.lib.lepic_gpu_get_mcc_stats(self.ctx, C.byref(st)), "get_mcc_stats")
        n = self.sp.ntype
        return {"n_cand": list(st.n_cand[:n]), "n_coll": list(st.n_coll[:self.xs.ncol]),
                "n_add": list(st.n_add[:n]), "n_overflow": st.n_overflow, "nu_max": list(st.nu_max[:n])}

    # particle sources (e_heating.f90, part_injection.f90) -------------------------------
    def set_sources(self, cfg: capi.LepicSourceConfig):
        self._src_cfg = cfg
        self.check(self.lib.lepic_gpu_set_sources(self.ctx, C.byref(cfg)), "set_sources")

    def set_heating(self, vt, Pabs_cor: float = 1.0):
        a = np.ascontiguousarray(vt, dtype=np.float64)
        self.check(self.lib.lepic_gpu_set_heating(self.ctx, _dp(a), a.shape[0], Pabs_cor), "set_heating")

    def eheating(self, it: int):
        self.check(self.lib.lepic_gpu_eheating(self.ctx, it), "eheating")

    def inject(self, it: int):
        self.check(self.lib.lepic_gpu_part_injection(self.ctx, it), "part_injection")

    def flux_emitter(self, it: int):
        self.check(self.lib.lepic_gpu_flux_emitter(self.ctx, it), "flux_emitter")

    def heating_tally(self):
        self.check(self.lib.lepic_gpu_heating_tally(self.ctx), "heating_tally")

    def source_tallies(self, reset: bool = False) -> dict:
        t = capi.LepicSourceTally()
        self.check(self.lib.lepic_gpu_source_tallies(self.ctx, C.byref(t), 1 if reset else 0), "source_tallies")
        n, b = self.sp.ntype, t.n_icp
        return {"P_heat": t.P_heat, "n_heated": t.n_heated, "n_heat_calls": t.n_heat_calls,
                "P_inj": list(t.P_inj[:n]), "P_src": list(t.P_src[:n]), "n_inj": list(t.n_inj[:n]),
                "n_inj_last": list(t.n_inj_last[:n]), "Nh": list(t.Nh[:b]), "sum_dEk": list(t.sum_dEk[:b]),
                "vt": list(t.vt[:b]), "n_emit": list(t.n_emit[:n]), "n_emit_last": list(t.n_emit_last[:n]),
                "n_emit_out": t.n_emit_out}

    # particle backup (main.f90:1102-1139, restart.f90:48-149) ---------------------------
    def write_backup(self, path: str, time: float = 0.0, gtype: int = 0, Pabs_cor: float = 1.0):
        self.check(self.lib.lepic_gpu_write_backup(self.ctx, path.encode(), time, gtype, Pabs_cor), "write_backup")

    def read_backup(self, path: str):
        t, pc = C.c_double(), C.c_double()
        gt = C.c_int32()
        self.check(self.lib.lepic_gpu_read_backup(self.ctx, path.encode(), C.byref(t), C.byref(gt), C.byref(pc)),
                   "read_backup")
        return t.value, gt.value, pc.value

    def set_zloss(self, hz: float, phi0: float = 0.0, size_na: int = 1):
        """The 3rd virtual dimension (hz >= 0 in the deck): z kept per particle, end-plate and
        Bohm losses in the mover (part_expmover.f90:269-309)."""
        z = capi.LepicZlossConfig(hz, phi0, size_na)
        self.check(self.lib.lepic_gpu_set_zloss(self.ctx, C.byref(z)), "set_zloss")

    def set_bohm_speed(self, uB: np.ndarray):
        """uB(na1+1, na2+1, ntype) in Fortran order: a (ntype, na2+1, na1+1) array."""
        a = np.ascontiguousarray(uB, dtype=np.float64)
        self.check(self.lib.lepic_gpu_set_bohm_speed(self.ctx, _dp(a)), "set_bohm_speed")

    def set_secondary(self, gam_sec: float, igrid_sec: int, xg_sec: float, THm: float):
        """Secondary electrons from positive ions lost on wall label igrid_sec
        (part_expmover.f90:354-392); gam_sec = 0 switches it off."""
        q = capi.LepicSecondaryConfig(gam_sec, igrid_sec, 0, xg_sec, THm)
        self.check(self.lib.lepic_gpu_set_secondary(self.ctx, C.byref(q)), "set_secondary")

    def set_dielectrics(self, dtype, Ca: float):
        """Dielectric wall labels (dtype[label] = 1; part_expmover.f90:340-350, main.f90:756-809)
        and their capacitance Ca [F/m^2]; all zeros switch the model off."""
        d = np.zeros(capi.MAXLABEL, dtype=np.int32)
        d[:len(dtype)] = dtype
        self.check(self.lib.lepic_gpu_set_dielectrics(self.ctx, d.ctypes.data_as(C.POINTER(C.c_int32)), Ca),
                   "set_dielectrics")

    def dielectric_update(self):
        self.check(self.lib.lepic_gpu_dielectric_update(self.ctx), "dielectric_update")

    def dielectric_charge(self) -> np.ndarray:
        """The charge collected on the dielectric labels since the last update: (MAXLABEL, ny+3) [C]."""
        q = np.zeros((capi.MAXLABEL, self.case.ny + 3))
        self.check(self.lib.lepic_gpu_get_dielectric_charge(self.ctx, _dp(q)), "get_dielectric_charge")
        return q

    def options(self) -> capi.LepicOptions:
        o = capi.LepicOptions()
        self.check(self.lib.lepic_gpu_get_options(self.ctx, C.byref(o)), "get_options")
        return o

    def set_options(self, **kw):
        """Changes solver settings by name (lepic_options fields); returns the previous ones."""
        old = self.options()
        o = capi.LepicOptions.from_buffer_copy(old)
        for k, v in kw.items():
            setattr(o, k, v)
        self.check(self.lib.lepic_gpu_set_options(self.ctx, C.byref(o)), "set_options")
        return old

    def stream_ptr(self) -> int:
        return self.lib.lepic_gpu_stream(self.ctx) or 0

    def close(self):
        if self.ctx:
            self.lib.lepic_gpu_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
