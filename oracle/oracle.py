"""ctypes wrapper of the CPU FP64 restatement (``lepic_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it; the product package
``jd_lepic_b200`` never imports it.

Parity against the reference's own outputs is UNPINNED (the Fortran reference cannot be
built here and ships no golden vectors); the restatement is pinned by the Park-Miller
published sequence and analytic known-answer tests in ``tests/test_oracle_kat.py``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
MAXSP = 8
MAXCOL = 64


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("lepic_oracle.c", "lepic_oracle.h", "cnn_oracle.c", "sources_oracle.c",
                                            "diag_oracle.c")]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-C", HERE, "-B" if force else "-s"], check=True, capture_output=True)
    return LIB


class OCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("zmax", C.c_double), ("xmax", C.c_double),
        ("ymax", C.c_double), ("dt", C.c_double),
        ("eps0", C.c_double), ("qe", C.c_double), ("pi", C.c_double),
        ("flag_pbc", C.c_int), ("flag_spec", C.c_int), ("flag_nmn", C.c_int),
        ("flag_B", C.c_int), ("flag_B_pos", C.c_int),
        ("Bc", C.c_double * 3),
        ("ntype", C.c_int), ("nsp", C.c_int),
        ("charge", C.c_double * MAXSP), ("mass", C.c_double * MAXSP), ("Nm", C.c_double * MAXSP),
        ("vt0", C.c_double * MAXSP), ("np_mx", C.c_double * MAXSP), ("nu_uplim", C.c_double * MAXSP),
        ("ns_coll", C.c_int), ("nsort", C.c_int),
    ]


class OXs(C.Structure):
    _fields_ = [
        ("npt", C.c_int), ("ncol", C.c_int),
        ("sig_Er", C.POINTER(C.c_double)), ("sig", C.POINTER(C.c_double)),
        ("Eth", C.POINTER(C.c_double)), ("col_info", C.POINTER(C.c_int32)),
        ("p_ncol", C.POINTER(C.c_int32)), ("sig_list", C.POINTER(C.c_int32)),
        ("sigv_mx", C.POINTER(C.c_double)),
        ("flag_ionrep", C.c_int), ("fEk", C.c_double),
    ]


class OPushTally(C.Structure):
    _fields_ = [("n_lost", C.c_int64), ("n_dead", C.c_int64), ("n_loss", C.c_int64 * 16),
                ("v2_loss", C.c_double * 16), ("P1z", C.c_double)]


class OZloss(C.Structure):
    _fields_ = [("phi0", C.c_double), ("phi", C.POINTER(C.c_double)), ("uB", C.POINTER(C.c_float)),
                ("na1", C.c_int), ("size_na", C.c_int), ("nu_fac", C.c_float),
                ("k0", C.c_uint32), ("k1", C.c_uint32), ("it", C.c_uint32)]


class OMccTally(C.Structure):
    _fields_ = [("n_cand", C.c_int64 * MAXSP), ("n_coll", C.c_int64 * MAXCOL),
                ("n_add", C.c_int64 * MAXSP), ("n_overflow", C.c_int64), ("nu_max", C.c_double * MAXSP)]


MAXICP = 16


class OSrc(C.Structure):
    _fields_ = [
        ("flag_c", C.c_int), ("xl_pow", C.c_double), ("xr_pow", C.c_double), ("yl_pow", C.c_double),
        ("yr_pow", C.c_double), ("eheat_type", C.c_int), ("flag_gpp", C.c_int), ("n_icp", C.c_int),
        ("nudt", C.c_double), ("Pabs_cor", C.c_double),
        ("opt_inj", C.c_int), ("flag_Tp", C.c_int), ("flag_diffsrc", C.c_int), ("tag_neg", C.c_int),
        ("nproc_mpi", C.c_int), ("ns_inj", C.c_int), ("I_inj", C.c_double), ("THm", C.c_double),
        ("ni0", C.c_double * MAXSP), ("th_B", C.c_double),
    ]


class OEmit(C.Structure):
    _fields_ = [
        ("js", C.c_double), ("xg1", C.c_double), ("Lg", C.c_double), ("Lh", C.c_double),
        ("n_holes", C.c_int), ("ns_Hm", C.c_int), ("n_icp", C.c_int), ("nproc_mpi", C.c_int),
        ("chamfer", C.c_int), ("chmfrd", C.c_double * 4), ("sp_fx", C.c_int), ("sp_b", C.c_int),
        ("THm", C.c_double),
    ]


class ODsmc(C.Structure):
    _fields_ = [("plist", C.POINTER(C.c_int32) * MAXSP), ("np_red", C.POINTER(C.c_double))]


class OSolveStats(C.Structure):
    _fields_ = [("k", C.c_int), ("ktot", C.c_double), ("res", C.c_double), ("sweeps_fine", C.c_int)]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
_I8 = C.POINTER(C.c_int8)
_LP = C.POINTER(C.c_int64)

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.o_ran2.restype = C.c_double
        L.o_ran2.argtypes = [C.POINTER(C.c_int32)]
        L.o_load_gauss.argtypes = [_DP, _DP, C.c_double, _DP]
        L.o_part_mover.argtypes = [C.POINTER(OCfg), C.c_int, _DP, _DP, _IP, _DP, _LP, _I8,
                                   C.POINTER(OPushTally)]
        L.o_part_mover_z.argtypes = [C.POINTER(OCfg), C.c_int, _DP, _DP, _IP, _DP, _LP, _I8,
                                     C.POINTER(OPushTally), C.POINTER(OZloss)]
        L.o_charge_deposition.argtypes = [C.POINTER(OCfg), C.c_int, _DP, C.c_int64, _DP, _DP]
        L.o_np_periodic.argtypes = [C.POINTER(OCfg), _DP, _IP]
        L.o_calc_rhs.argtypes = [C.POINTER(OCfg), _DP, _DP]
        L.o_dens_red.argtypes = [C.POINTER(OCfg), _DP, _DP, _IP]
        L.o_calc_efield.argtypes = [C.POINTER(OCfg), _DP, _DP, _IP]
        L.o_iterative_solver.restype = C.c_int
        L.o_iterative_solver.argtypes = [C.POINTER(OCfg), _DP, _DP, _IP, C.c_int, C.c_int, C.c_double,
                                         C.POINTER(OSolveStats)]
        L.o_iterative_solver_omp.restype = C.c_int
        L.o_iterative_solver_omp.argtypes = [C.POINTER(OCfg), _DP, _DP, _IP, C.c_int, C.c_int, C.c_double,
                                             C.POINTER(OSolveStats), C.c_int]
        L.o_iterative_solver_l2_omp.restype = C.c_int
        L.o_iterative_solver_l2_omp.argtypes = [C.POINTER(OCfg), _DP, _DP, _IP, C.c_int, C.c_int, C.c_double,
                                                C.POINTER(OSolveStats), C.c_int]
        L.o_sor_rb.restype = C.c_int
        L.o_sor_rb.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _DP, _DP, _IP, _DP,
                               C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        L.o_restriction.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _DP, _DP, _IP,
                                    _IP, _DP, _DP, C.c_int, C.c_int]
        L.o_prolongation.argtypes = [C.c_int, C.c_int, _DP, _DP, _IP]
        L.o_part_sorting.argtypes = [C.POINTER(OCfg), _DP, C.c_int64, _IP, _DP]
        L.o_indexx.argtypes = [C.c_int, _DP, C.POINTER(C.c_int)]
        L.o_collisions.restype = C.c_int
        L.o_collisions.argtypes = [C.POINTER(OCfg), C.POINTER(OXs), C.POINTER(_DP), _LP, _LP,
                                   C.POINTER(_I8), C.POINTER(C.c_int32), C.POINTER(OMccTally)]
        L.o_collisions_dsmc.restype = C.c_int
        L.o_collisions_dsmc.argtypes = [C.POINTER(OCfg), C.POINTER(OXs), C.POINTER(_DP), _LP, _LP,
                                        C.POINTER(_I8), C.POINTER(C.c_int32), C.POINTER(OMccTally),
                                        C.POINTER(ODsmc)]
        L.o_scatter.argtypes = [_DP, _DP, _DP, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.o_push_deposit_omp.argtypes = [C.POINTER(OCfg), C.c_int, _DP, _DP, _IP, _DP, _DP, _LP, _I8, _DP,
                                         C.c_int]
        _U32 = C.POINTER(C.c_uint32)
        L.o_philox4x32_10.argtypes = [_U32, C.c_uint32, C.c_uint32, _U32]
        L.o_u01.restype = C.c_double
        L.o_u01.argtypes = [C.c_uint32]
        L.o_eheating.argtypes = [C.POINTER(OCfg), C.POINTER(OSrc), _DP, C.c_int64, _DP, C.POINTER(C.c_int32), _DP, _LP]
        L.o_eheating_ctr.argtypes = [C.POINTER(OCfg), C.POINTER(OSrc), _DP, C.c_int64, _DP, C.c_uint64, C.c_int32,
                                     _DP, _LP]
        L.o_heat_tally.argtypes = [C.POINTER(OCfg), C.POINTER(OSrc), _DP, C.c_int64, _LP, _DP]
        L.o_te_update.restype = C.c_double
        L.o_te_update.argtypes = [C.POINTER(OCfg), C.c_int, C.c_double, C.c_double, C.c_int64, C.c_double, C.c_double]
        L.o_part_injection.restype = C.c_int
        L.o_part_injection.argtypes = [C.POINTER(OCfg), C.POINTER(OSrc), C.c_int, _IP, _DP, _LP, _DP, _LP, C.c_int64,
                                       C.POINTER(C.c_int32), _DP, _DP]
        L.o_part_injection_ctr.restype = C.c_int
        L.o_part_injection_ctr.argtypes = [C.POINTER(OCfg), C.POINTER(OSrc), _IP, _DP, _LP, C.c_uint64, C.c_int32,
                                           C.c_int, C.POINTER(_DP), _LP, _LP, _LP, _DP, _DP]
        L.o_part_flux_emitter.restype = C.c_int
        L.o_part_flux_emitter.argtypes = [C.POINTER(OCfg), C.POINTER(OEmit), _IP, C.POINTER(_DP), _LP, _LP,
                                          C.POINTER(C.c_int32), _LP, _DP]
        L.o_part_flux_emitter_ctr.restype = C.c_int
        L.o_part_flux_emitter_ctr.argtypes = [C.POINTER(OCfg), C.POINTER(OEmit), _IP, C.c_uint64, C.c_int32, C.c_int,
                                              C.POINTER(_DP), _LP, _LP, _LP, _DP, _LP]
        L.o_part_moments.argtypes = [C.POINTER(OCfg), C.c_int, C.c_int, _DP, C.c_int64, _DP, _DP]
        L.o_calc_avg.argtypes = [C.POINTER(OCfg), C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP]
        _lib = L
    return _lib


def dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


def ip(a):
    return a.ctypes.data_as(_IP) if a is not None else None


def make_cfg(case, sp) -> OCfg:
    """o_cfg from a configs.Case and simulation.SpeciesParams (the same inputs the GPU gets)."""
    from jd_lepic_b200 import deck as dk
    c = OCfg()
    c.nx, c.ny = case.nx, case.ny
    c.dx, c.dy, c.zmax = case.dx, case.dy, case.zmax
    c.xmax, c.ymax = case.nx * case.dx, case.ny * case.dy
    c.dt = case.dt
    c.eps0, c.qe, c.pi = dk.EPS0, dk.QE, 4.0 * math.atan(1.0)
    c.flag_pbc, c.flag_spec, c.flag_nmn = case.flag_pbc, case.flag_spec, case.flag_nmn
    c.flag_B = case.flag_B
    c.flag_B_pos = 0
    for k in range(3):
        c.Bc[k] = case.Bc[k]
    c.ntype, c.nsp = sp.ntype, sp.nsp
    for s in range(MAXSP):
        c.charge[s], c.mass[s], c.Nm[s] = sp.charge[s], sp.mass[s], sp.Nm[s]
        c.vt0[s], c.np_mx[s], c.nu_uplim[s] = sp.vt0[s], sp.np_mx[s], sp.nu_uplim[s]
    c.ns_coll, c.nsort = 10, 10
    return c


class XsHolder:
    """Keeps numpy buffers alive behind an OXs."""

    def __init__(self, t):
        self.arrs = [np.ascontiguousarray(t.sig_Er), np.ascontiguousarray(t.sig), np.ascontiguousarray(t.Eth),
                     np.ascontiguousarray(t.col_info, dtype=np.int32), np.ascontiguousarray(t.p_ncol, dtype=np.int32),
                     np.ascontiguousarray(t.sig_list, dtype=np.int32), np.ascontiguousarray(t.sigv_mx)]
        a = self.arrs
        self.xs = OXs(t.npt, t.ncol, dp(a[0]), dp(a[1]), dp(a[2]), ip(a[3]), ip(a[4]), ip(a[5]), dp(a[6]),
                      t.flag_ionrep, t.fEk)


def kq_of(bcnd: np.ndarray) -> np.ndarray:
    """main.f90:334-344"""
    return np.where(bcnd != -1, 2.0, 1.0)


def mover(cfg, ptype, Ei, Bi, bcnd, vxp: np.ndarray, flag_dead=None):
    n = C.c_int64(vxp.shape[0])
    t = OPushTally()
    fd = flag_dead.ctypes.data_as(_I8) if flag_dead is not None else None
    lib().o_part_mover(C.byref(cfg), ptype, dp(Ei), dp(Bi), ip(bcnd), dp(vxp), C.byref(n), fd, C.byref(t))
    return n.value, t


def zloss_keys(seed: int):
    """The device's key of the 3rd-dimension draws (push.cu, zstep)."""
    return int(seed) & 0xFFFFFFFF, ((int(seed) >> 32) ^ 0x5A10C5) & 0xFFFFFFFF


def mover_z(cfg, ptype, Ei, Bi, bcnd, vxp: np.ndarray, phi, phi0, uB, na1, size_na, hz, seed, it):
    """o_part_mover_z on vxp (n, 6) in place (z in column 2); uB: this species' (na2+1, na1+1)
    map.  Returns (n survivors, tally)."""
    n = C.c_int64(vxp.shape[0])
    t = OPushTally()
    phi_a = np.ascontiguousarray(phi, dtype=np.float64)
    ub = np.ascontiguousarray(uB, dtype=np.float32)
    k0, k1 = zloss_keys(seed)
    z = OZloss(phi0, dp(phi_a), ub.ctypes.data_as(C.POINTER(C.c_float)), na1, size_na,
               float(np.float32(hz * 2.0 / cfg.zmax * cfg.dt)), k0, k1, it)
    lib().o_part_mover_z(C.byref(cfg), ptype, dp(Ei), dp(Bi), ip(bcnd), dp(vxp), C.byref(n), None, C.byref(t),
                         C.byref(z))
    return n.value, t


class ODielec(C.Structure):
    _fields_ = [("dtype", C.POINTER(C.c_int32)), ("dq", C.POINTER(C.c_double))]


def mover_dielec(cfg, ptype, Ei, Bi, bcnd, vxp: np.ndarray, dtype):
    """o_part_mover_zd on vxp (n, 6) in place with dielectric labels dtype (16 entries); returns
    (n survivors, tally, dq (16, ny+3))."""
    n = C.c_int64(vxp.shape[0])
    t = OPushTally()
    dt = np.ascontiguousarray(dtype, dtype=np.int32)
    dq = np.zeros((16, cfg.ny + 3))
    d = ODielec(dt.ctypes.data_as(C.POINTER(C.c_int32)), dp(dq))
    lib().o_part_mover_zd(C.byref(cfg), ptype, dp(Ei), dp(Bi), ip(bcnd), dp(vxp), C.byref(n), None, C.byref(t),
                          None, C.byref(d))
    return n.value, t, dq


class OWallx(C.Structure):
    _fields_ = [("reflux", C.c_int), ("vb", C.c_double), ("fmax", C.c_double), ("vt", C.c_double),
                ("sin_thB", C.c_double), ("cos_thB", C.c_double), ("sec_label", C.c_int),
                ("gam_sec", C.c_double), ("vt_sec", C.c_double), ("xg_sec", C.c_double), ("Nm0", C.c_double),
                ("m0", C.c_double), ("sec_out", C.POINTER(C.c_double)), ("sec_cap", C.c_int64),
                ("n_sec", C.c_int64), ("k0", C.c_uint32), ("k1", C.c_uint32), ("it", C.c_uint32),
                ("P1r", C.c_double), ("P4r", C.c_double), ("P4sec", C.c_double)]


def mover_wallx(cfg, ptype, Ei, Bi, bcnd, vxp: np.ndarray, seed: int, it: int, reflux=None, secondary=None,
                sec_cap: int = 1 << 20):
    """o_part_mover_x on vxp (n, 6) in place with the device's counter streams.
    reflux: dict(vb, fmax, vt, th_B); secondary: dict(label, gam, vt, xg, Nm0, m0).
    Returns (n survivors, tally, wallx struct, emitted electrons (m, 6))."""
    n = C.c_int64(vxp.shape[0])
    t = OPushTally()
    w = OWallx()
    out = np.zeros((sec_cap, 6))
    k0, k1 = zloss_keys(seed)
    w.k0, w.k1, w.it = k0, k1, it
    if reflux:
        w.reflux = 1
        w.vb, w.fmax, w.vt = reflux["vb"], reflux["fmax"], reflux["vt"]
        w.sin_thB, w.cos_thB = math.sin(reflux["th_B"]), math.cos(reflux["th_B"])
    if secondary:
        w.sec_label, w.gam_sec, w.vt_sec = secondary["label"], secondary["gam"], secondary["vt"]
        w.xg_sec, w.Nm0, w.m0 = secondary["xg"], secondary["Nm0"], secondary["m0"]
    w.sec_out = dp(out)
    w.sec_cap = sec_cap
    lib().o_part_mover_x(C.byref(cfg), ptype, dp(Ei), dp(Bi), ip(bcnd), dp(vxp), C.byref(n), None, C.byref(t),
                         None, None, C.byref(w))
    return n.value, t, w, out[:min(w.n_sec, sec_cap)].copy()


def dielectric_update(cfg, phi: np.ndarray, bcnd, dtype, dq: np.ndarray, Ca: float):
    """o_dielectric_update: phi (ny+3, nx+3) and dq (16, ny+3) in place."""
    dt = np.ascontiguousarray(dtype, dtype=np.int32)
    lib().o_dielectric_update(C.byref(cfg), dp(phi), ip(bcnd), dt.ctypes.data_as(C.POINTER(C.c_int32)), dp(dq),
                              C.c_double(Ca))


def mover_tagged(cfg, ptype, Ei, Bi, bcnd, vxp: np.ndarray):
    """o_part_mover on a copy of vxp whose z holds each particle's index; returns the survivors
    (compacted in order, part_expmover.f90:496-503) and their indices.  z moves by dt*vz, far
    below 0.5, so rounding recovers the index."""
    ref = np.ascontiguousarray(vxp, dtype=np.float64).copy()
    ref[:, 2] = np.arange(ref.shape[0], dtype=np.float64)
    n, t = mover(cfg, ptype, Ei, Bi, bcnd, ref)
    ref = ref[:n].copy()
    ids = np.rint(ref[:, 2]).astype(np.int64)
    ref[:, 2] = 0.0
    return ref, ids, t


def align_survivors(got: np.ndarray, ref: np.ndarray, dx: float, dy: float, window: int = 8):
    """Pairs the device's survivors with the oracle's.  Both are the initial particles minus the
    lost ones, in the initial order, so they are two subsequences of one sequence that differ
    only where a particle within a rounding distance of a wall cell is lost on one side.
    Returns (gi, rj, n_gpu_only, n_ref_only): index arrays of the paired rows and the number of
    particles kept by one side only.  Two rows pair when their positions agree to 1e-3 of a cell
    (the parity tolerance is far tighter and is asserted on the pairs by the caller)."""
    ng, nr = got.shape[0], ref.shape[0]
    gi, rj = [], []
    g_only = r_only = 0
    i = j = 0

    def same(a, b):
        return abs(got[a, 0] - ref[b, 0]) <= 1e-3 * dx and abs(got[a, 1] - ref[b, 1]) <= 1e-3 * dy

    # vectorised fast path over the common prefix, then a windowed greedy walk at mismatches
    while i < ng and j < nr:
        m = min(ng - i, nr - j)
        ok = (np.abs(got[i:i + m, 0] - ref[j:j + m, 0]) <= 1e-3 * dx) & \
             (np.abs(got[i:i + m, 1] - ref[j:j + m, 1]) <= 1e-3 * dy)
        k = int(np.argmin(ok)) if not ok.all() else m
        gi.extend(range(i, i + k))
        rj.extend(range(j, j + k))
        i += k
        j += k
        if i >= ng or j >= nr:
            break
        for d in range(1, window + 1):       # the device lost ref[j .. j+d-1]
            if j + d < nr and same(i, j + d):
                r_only += d
                j += d
                break
            if i + d < ng and same(i + d, j):  # the oracle lost got[i .. i+d-1]
                g_only += d
                i += d
                break
        else:
            raise AssertionError(f"device and oracle survivors cannot be aligned at {i}/{j}")
    g_only += ng - i
    r_only += nr - j
    return np.asarray(gi, dtype=np.int64), np.asarray(rj, dtype=np.int64), g_only, r_only


DEP_SHIFT = 44   # the device's accumulators hold CIC weights in units of 2^-44


def int_deposit(X, Y, nx: int, ny: int, S: int) -> np.ndarray:
    """The device's charge accumulator of one species, restated in numpy: uint64 CIC weights of
    fixed-point positions (cell = X >> S, offset = X & (2^S - 1)), the products of the offsets
    rounded to 2^-44 (part_expmover.f90:540-575 in integer form), node i + j (nx+3) of
    np(0:nx+2, 0:ny+2).  Integer sums: any split of the particles over ranks sums to the same
    grid (calc_rho.f90:71-74)."""
    X = np.asarray(X, dtype=np.int64)
    Y = np.asarray(Y, dtype=np.int64)
    W = nx + 3
    acc = np.zeros((ny + 3) * W, dtype=np.uint64)
    mask = (1 << S) - 1
    fx = (X & mask).astype(np.uint64)
    fy = (Y & mask).astype(np.uint64)
    A = np.uint64(1 << S)
    ax, ay = A - fx, A - fy
    sh = 2 * S - DEP_SHIFT
    ix = (X >> S) + 1
    iy = (Y >> S) + 1
    for w, ddx, ddy in ((ax * ay, 0, 0), (fx * ay, 1, 0), (fx * fy, 1, 1), (ax * fy, 0, 1)):
        if sh > 0:
            w = (w + np.uint64(1 << (sh - 1))) >> np.uint64(sh)
        elif sh < 0:
            w = w << np.uint64(-sh)
        np.add.at(acc, (ix + ddx) + (iy + ddy) * W, w)
    return acc


def np_from_acc(cfg, ptype: int, acc: np.ndarray, kq: np.ndarray) -> np.ndarray:
    """np(0:nx+2, 0:ny+2) of one species from its accumulator, as the device scales it:
    kq * (k1 * (acc 2^-44)), k1 = Nm / (dx dy zmax)."""
    k1 = cfg.Nm[ptype] / (cfg.dx * cfg.dy * cfg.zmax)
    w = np.asarray(acc, dtype=np.uint64).astype(np.float64) * 5.684341886080802e-14
    return (np.asarray(kq, dtype=np.float64).ravel() * (k1 * w)).reshape(cfg.ny + 3, cfg.nx + 3)


def dens_red(cfg, npg, bcnd):
    """o_dens_red (calc_rho.f90:134-199): returns (np_red (ntype, ny+3, nx+3), np_mx[ntype])."""
    ntype = cfg.ntype
    a = np.ascontiguousarray(npg, dtype=np.float64)
    out = np.zeros((ntype, cfg.ny + 3, cfg.nx + 3))
    c = OCfg.from_buffer_copy(cfg)
    lib().o_dens_red(C.byref(c), dp(a), dp(out), ip(np.ascontiguousarray(bcnd, dtype=np.int32)))
    return out, np.array(c.np_mx[:ntype])


def deposit(cfg, ptype, vxp, n, kq, npg):
    lib().o_charge_deposition(C.byref(cfg), ptype, dp(vxp), n, dp(kq), dp(npg))


def np_periodic(cfg, npg, bcnd):
    """calc_rho.f90:1-35 on npg (ntype, ny+3, nx+3) in place."""
    assert npg.flags.c_contiguous and npg.shape[0] >= cfg.ntype
    lib().o_np_periodic(C.byref(cfg), dp(npg), ip(np.ascontiguousarray(bcnd, dtype=np.int32)))


def calc_rhs(cfg, npg):
    rhs = np.zeros((cfg.ny + 1, cfg.nx + 1))
    lib().o_calc_rhs(C.byref(cfg), dp(npg), dp(rhs))
    return rhs


def efield(cfg, phi, bcnd, Ei=None):
    if Ei is None:
        Ei = np.zeros((cfg.ny + 3, cfg.nx + 3, 2))
    lib().o_calc_efield(C.byref(cfg), dp(phi), dp(Ei), ip(bcnd))
    return Ei


def solve(cfg, phi, rhs, bcnd, ng, eps, ncycl=20000, nthreads=1, l2=False):
    """iterative_solver on phi in place; eps is the reference's normalised L1 tolerance, or with
    l2 the relative L2 residual ||b - A u|| / ||b - A u_D|| the device's L2 modes stop on."""
    st = OSolveStats()
    if l2:
        rc = lib().o_iterative_solver_l2_omp(C.byref(cfg), dp(phi), dp(rhs), ip(bcnd), ng, ncycl, eps, C.byref(st),
                                             max(1, nthreads))
    elif nthreads > 1:
        rc = lib().o_iterative_solver_omp(C.byref(cfg), dp(phi), dp(rhs), ip(bcnd), ng, ncycl, eps, C.byref(st),
                                          nthreads)
    else:
        rc = lib().o_iterative_solver(C.byref(cfg), dp(phi), dp(rhs), ip(bcnd), ng, ncycl, eps, C.byref(st))
    return rc, st


def sort(cfg, vxp, n):
    pl = np.zeros(cfg.nx + cfg.nx * cfg.ny + 2, dtype=np.int32)
    scratch = np.zeros((max(n, 1), 6))
    lib().o_part_sorting(C.byref(cfg), dp(vxp), n, ip(pl), dp(scratch))
    return pl


def ran2_sequence(seed: int, n: int) -> tuple[np.ndarray, int]:
    s = C.c_int32(seed)
    out = np.array([lib().o_ran2(C.byref(s)) for _ in range(n)])
    return out, s.value


def l2_residual(cfg, phi, rhs, bcnd):
    """||b - A u||_2 / ||b - A u_D||_2 over bcnd == -1 nodes (u_D: unknowns zeroed), FP64."""
    aw = cfg.eps0 / (cfg.dx * cfg.dx)
    an = cfg.eps0 / (cfg.dy * cfg.dy)
    ac = -(an + an + aw + aw)
    u = phi
    c = u[1:-1, 1:-1]
    Au = aw * u[1:-1, :-2] + an * u[2:, 1:-1] + an * u[:-2, 1:-1] + aw * u[1:-1, 2:] + ac * c
    m = bcnd[1:-1, 1:-1] == -1
    r = rhs - Au
    w = bcnd > 0
    ud = np.where(w, u, 0.0)
    Aud = aw * ud[1:-1, :-2] + an * ud[2:, 1:-1] + an * ud[:-2, 1:-1] + aw * ud[1:-1, 2:]
    d = rhs - Aud
    return math.sqrt(float((r[m] ** 2).sum())) / max(math.sqrt(float((d[m] ** 2).sum())), 1e-300)


def collisions(cfg, xsh, particles, seed: int, extra: int = 4096, plists=None, np_red=None):
    """o_collisions (collisions.f90:1-207, collision_OMP, SCATTER) once on copies of the given
    per-species particle arrays, the ran2 stream seeded with `seed`.  Returns (rc, arrays after
    the call with the products appended, the collision tally, flag_dead per species).
    With plists ({species: Plist of its array as sort() returns it}) and np_red (dens_red's
    (ntype, ny+3, nx+3) grids; cfg.np_mx must hold their maxima) charged targets take part
    (o_collisions_dsmc, collisions.f90:339-418)."""
    ntype = cfg.ntype
    bufs, fds = [], []
    for s in range(ntype):
        a = np.ascontiguousarray(particles[s], dtype=np.float64)
        b = np.zeros((a.shape[0] + extra, 6))
        b[:a.shape[0]] = a
        bufs.append(b)
        fds.append(np.zeros(b.shape[0], dtype=np.int8))
    arrs = (_DP * MAXSP)(*[dp(b) for b in bufs])
    npt = (C.c_int64 * MAXSP)(*[p.shape[0] for p in particles[:ntype]])
    cap = (C.c_int64 * MAXSP)(*[b.shape[0] for b in bufs])
    fdp = (_I8 * MAXSP)(*[f.ctypes.data_as(_I8) for f in fds])
    t = OMccTally()
    sd = C.c_int32(seed)
    if plists is None:
        rc = lib().o_collisions(C.byref(cfg), C.byref(xsh.xs), arrs, npt, cap, fdp, C.byref(sd), C.byref(t))
    else:
        keep = [np.ascontiguousarray(plists[s], dtype=np.int32) for s in sorted(plists)]
        red = np.ascontiguousarray(np_red, dtype=np.float64)
        d = ODsmc()
        for s, a in zip(sorted(plists), keep):
            d.plist[s] = ip(a)
        d.np_red = dp(red)
        rc = lib().o_collisions_dsmc(C.byref(cfg), C.byref(xsh.xs), arrs, npt, cap, fdp, C.byref(sd), C.byref(t),
                                     C.byref(d))
    out = [bufs[s][:npt[s]].copy() for s in range(ntype)]
    return rc, out, t, [fds[s][:npt[s]].copy() for s in range(ntype)]


class OracleSimulation:
    """The reference's step loop (main.f90:818-1090, in-scope routines) on the CPU, FP64."""

    def __init__(self, case, nthreads: int = 1, particles: dict | None = None, seed: int | None = None,
                 capacity_factor: float = 1.3):
        from jd_lepic_b200 import deck as dk
        from jd_lepic_b200.simulation import species_params
        self.case = case
        self.deck = dk.read_reactions(case.deck_text, case.ngas)
        self.tables = dk.ordering(self.deck)
        self.sp = species_params(case, self.deck)
        self.cfg = make_cfg(case, self.sp)
        self.xsh = XsHolder(self.tables)
        self.nt = nthreads
        self.bcnd = np.ascontiguousarray(case.bcnd, dtype=np.int32)
        self.phi = np.ascontiguousarray(case.phi0, dtype=np.float64).copy()
        self.kq = kq_of(self.bcnd)
        self.Bi = np.ascontiguousarray(case.Bi) if case.Bi is not None else None
        self.Ei = np.zeros((case.ny + 3, case.nx + 3, 2))
        self.ng = case.levels()
        ntype = self.sp.ntype
        nn = (case.nx + 3) * (case.ny + 3)
        self.npg = np.zeros((ntype, case.ny + 3, case.nx + 3))
        self.seed = C.c_int32(seed if seed is not None else 123456)  # main.f90:530 for iproc = 1
        self.vxp, self.np_tot, self.cap, self.flag_dead = [], [], [], []
        for s in range(ntype):
            arr = particles[s] if particles is not None else None
            n = arr.shape[0] if arr is not None else 0
            cap = max(int(n * capacity_factor) + 1024, 1024)
            buf = np.zeros((cap, 6))
            if n:
                buf[:n] = arr
            self.vxp.append(buf)
            self.np_tot.append(n)
            self.cap.append(cap)
            self.flag_dead.append(np.zeros(cap, dtype=np.int8))
        self._nn = nn
        self.deposit_all()

    def deposit_all(self):
        self.npg[:] = 0.0
        for s in range(self.sp.ntype):
            deposit(self.cfg, s, self.vxp[s], self.np_tot[s], self.kq, self.npg[s])

    def step(self, it: int, eps: float | None = None, l2: bool = False):
        case = self.case
        eps = case.eps if eps is None else eps
        self.rhs = calc_rhs(self.cfg, self.npg)
        rc, self.solve_stats = solve(self.cfg, self.phi, self.rhs, self.bcnd, self.ng, eps, nthreads=self.nt, l2=l2)
        if rc != 0:
            raise RuntimeError("oracle Poisson solve diverged")
        efield(self.cfg, self.phi, self.bcnd, self.Ei)
        if it % 10 == 1:
            for s in range(self.sp.ntype):
                if self.np_tot[s] > 0:
                    sort(self.cfg, self.vxp[s], self.np_tot[s])
        if it > 1 and it % 10 == 1:
            self.collide()
        self.npg[:] = 0.0
        for s in range(self.sp.ntype):
            n = C.c_int64(self.np_tot[s])
            lib().o_push_deposit_omp(C.byref(self.cfg), s, dp(self.Ei), dp(self.Bi), ip(self.bcnd), dp(self.kq),
                                     dp(self.vxp[s]), C.byref(n), self.flag_dead[s].ctypes.data_as(_I8),
                                     dp(self.npg[s]), self.nt)
            self.np_tot[s] = n.value

    def collide(self):
        ntype = self.sp.ntype
        arrs = (_DP * MAXSP)(*[dp(self.vxp[s]) for s in range(ntype)])
        npt = (C.c_int64 * MAXSP)(*self.np_tot)
        cap = (C.c_int64 * MAXSP)(*self.cap)
        fds = (_I8 * MAXSP)(*[self.flag_dead[s].ctypes.data_as(_I8) for s in range(ntype)])
        t = OMccTally()
        rc = lib().o_collisions(C.byref(self.cfg), C.byref(self.xsh.xs), arrs, npt, cap, fds, C.byref(self.seed),
                                C.byref(t))
        if rc != 0:
            raise RuntimeError(f"oracle collisions failed with {rc}")
        for s in range(ntype):
            self.np_tot[s] = npt[s]
        self.mcc = t
        return t


# ---------------------------------------------------------------------------------------------
# learned warm-start network (cnn_oracle.c)

CNN_CIN = (2, 16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16)
CNN_COUT = (16, 16, 32, 32, 64, 64, 64, 64, 64, 32, 16, 1)


def cnn_nparams() -> int:
    return int(lib().o_cnn_nparams())


def cnn_loss_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray, m: np.ndarray, emulate_bf16: bool = True,
                  want_grad: bool = True):
    """Forward, energy-norm loss and gradient of the warm-start network on the CPU.
    x: (N, H, W, 2), t and m: (N, H, W); H and W multiples of 8.  Returns (loss, out, grad)."""
    L = lib()
    f = L.o_cnn_loss_grad
    f.restype = C.c_double
    f.argtypes = [C.POINTER(C.c_double)] * 4 + [C.c_int] * 4 + [C.POINTER(C.c_double)] * 2
    N, H, W = t.shape
    prm = np.ascontiguousarray(params, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    tt = np.ascontiguousarray(t, dtype=np.float64)
    mm = np.ascontiguousarray(m, dtype=np.float64)
    out = np.zeros((N, H, W))
    grad = np.zeros(prm.size) if want_grad else None
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
    loss = f(dp(prm), dp(xx), dp(tt), dp(mm), N, H, W, 1 if emulate_bf16 else 0, dp(out), dp(grad))
    return loss, out, grad


def cnn_init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (std sqrt(2 / (9 cin))), zero biases, in the oracle's parameter order."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in zip(CNN_CIN, CNN_COUT):
        out.append(rng.standard_normal(co * ci * 9) * np.sqrt(2.0 / (9 * ci)))
        out.append(np.zeros(co))
    return np.concatenate(out)


# ---- particle sources (e_heating.f90, part_injection.f90) -------------------------------
def philox(ctr, key) -> tuple[int, int, int, int]:
    """Philox4x32-10 of a 4-word counter and a 2-word key."""
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    o = (C.c_uint32 * 4)()
    lib().o_philox4x32_10(c, int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF, o)
    return tuple(int(v) for v in o)


def make_src(sc) -> OSrc:
    """o_src from a lepic_source_config (ctypes structure of the product's C ABI)."""
    o = OSrc()
    for f in ("flag_c", "xl_pow", "xr_pow", "yl_pow", "yr_pow", "eheat_type", "flag_gpp", "n_icp", "nudt",
              "Pabs_cor", "opt_inj", "flag_Tp", "flag_diffsrc", "tag_neg", "nproc_mpi", "ns_inj", "I_inj", "THm", "th_B"):
        setattr(o, f, getattr(sc, f))
    for s in range(MAXSP):
        o.ni0[s] = sc.ni0[s]
    return o


def eheating(cfg, src, vxp, vt, *, iseed=None, seed=None, it=0):
    """e_heating.f90 on vxp (n, 6) in place.  iseed: the reference's ran2 form; seed/it: the
    device's counter streams.  Returns (P_heat, n_heated[, iseed])."""
    vt = np.ascontiguousarray(vt, dtype=np.float64)
    P = C.c_double(0.0)
    nh = C.c_int64(0)
    if iseed is not None:
        sd = C.c_int32(iseed)
        lib().o_eheating(C.byref(cfg), C.byref(src), dp(vxp), vxp.shape[0], dp(vt), C.byref(sd), C.byref(P),
                         C.byref(nh))
        return P.value, nh.value, sd.value
    lib().o_eheating_ctr(C.byref(cfg), C.byref(src), dp(vxp), vxp.shape[0], dp(vt), seed, it, C.byref(P), C.byref(nh))
    return P.value, nh.value


def heat_tally(cfg, src, vxp):
    Nh = np.zeros(MAXICP, dtype=np.int64)
    E = np.zeros(MAXICP)
    lib().o_heat_tally(C.byref(cfg), C.byref(src), dp(vxp), vxp.shape[0], Nh.ctypes.data_as(_LP), dp(E))
    return Nh[:src.n_icp], E[:src.n_icp]


def te_update(cfg, eheat_type, Pabs, nu_h, Nh, sum_dEk, vt_old):
    return lib().o_te_update(C.byref(cfg), eheat_type, Pabs, nu_h, int(Nh), sum_dEk, vt_old)


def part_injection(cfg, src, ptype, bcnd, phi, N_inj, vxp, n, iseed):
    """The reference's form for one species (ran2).  N_inj (int64[ntype]) in/out; vxp (cap, 6)
    receives the particles from row n.  Returns (rc, n, P_inj, P_src, iseed)."""
    nn = C.c_int64(n)
    sd = C.c_int32(iseed)
    Pi, Ps = C.c_double(0.0), C.c_double(0.0)
    rc = lib().o_part_injection(C.byref(cfg), C.byref(src), ptype, ip(bcnd), dp(phi), N_inj.ctypes.data_as(_LP),
                                dp(vxp), C.byref(nn), vxp.shape[0], C.byref(sd), C.byref(Pi), C.byref(Ps))
    return rc, nn.value, Pi.value, Ps.value, sd.value


def part_injection_ctr(cfg, src, bcnd, phi, lost, seed, it, S, vxp_list, n_list):
    """The device's form for every charged species.  vxp_list[s] (cap_s, 6) arrays receive the
    particles from row n_list[s].  Returns (rc, n, count, P_inj, P_src)."""
    ns = cfg.ntype
    lost = np.ascontiguousarray(np.resize(np.asarray(lost, dtype=np.int64), MAXSP))
    ptrs = (_DP * MAXSP)(*[dp(v) for v in vxp_list] + [None] * (MAXSP - ns))
    npa = np.zeros(MAXSP, dtype=np.int64)
    npa[:ns] = n_list
    cap = np.zeros(MAXSP, dtype=np.int64)
    cap[:ns] = [v.shape[0] for v in vxp_list]
    cnt = np.zeros(MAXSP, dtype=np.int64)
    Pi = np.zeros(MAXSP)
    Ps = np.zeros(MAXSP)
    rc = lib().o_part_injection_ctr(C.byref(cfg), C.byref(src), ip(bcnd), dp(phi), lost.ctypes.data_as(_LP), seed,
                                    it, S, ptrs, npa.ctypes.data_as(_LP), cap.ctypes.data_as(_LP),
                                    cnt.ctypes.data_as(_LP), dp(Pi), dp(Ps))
    return rc, npa[:ns].copy(), cnt[:ns].copy(), Pi[:ns].copy(), Ps[:ns].copy()


def make_emit(sc) -> OEmit:
    """o_emit from a lepic_source_config."""
    o = OEmit()
    for f in ("js", "xg1", "Lg", "Lh", "n_holes", "ns_Hm", "n_icp", "nproc_mpi", "THm"):
        setattr(o, f, getattr(sc, f))
    o.chamfer = 1 if (sc.ptype_fx == sc.tag_neg and sc.flag_chmfrd == 1) else 0
    for k in range(4):
        o.chmfrd[k] = sc.chmfrd[k]
    o.sp_fx = sc.ptype_fx
    o.sp_b = sc.tag_b if (o.chamfer and sc.tag_b >= 0) else sc.ptype_fx
    return o


def _emit_args(cfg, vxp_list, n_list):
    ns = cfg.ntype
    ptrs = (_DP * MAXSP)(*[dp(v) for v in vxp_list] + [None] * (MAXSP - ns))
    npa = np.zeros(MAXSP, dtype=np.int64)
    npa[:ns] = n_list
    cap = np.zeros(MAXSP, dtype=np.int64)
    cap[:ns] = [v.shape[0] for v in vxp_list]
    return ptrs, npa, cap, np.zeros(MAXSP, dtype=np.int64), np.zeros(MAXSP)


def flux_emitter(cfg, emit, bcnd, vxp_list, n_list, iseed):
    """The reference's form (ran2).  Returns (rc, n, count, P_inj, iseed)."""
    ptrs, npa, cap, cnt, Pi = _emit_args(cfg, vxp_list, n_list)
    sd = C.c_int32(iseed)
    rc = lib().o_part_flux_emitter(C.byref(cfg), C.byref(emit), ip(bcnd), ptrs, npa.ctypes.data_as(_LP),
                                   cap.ctypes.data_as(_LP), C.byref(sd), cnt.ctypes.data_as(_LP), dp(Pi))
    ns = cfg.ntype
    return rc, npa[:ns].copy(), cnt[:ns].copy(), Pi[:ns].copy(), sd.value


def flux_emitter_ctr(cfg, emit, bcnd, seed, it, S, vxp_list, n_list):
    """The device's form.  Returns (rc, n, count, P_inj, n_out)."""
    ptrs, npa, cap, cnt, Pi = _emit_args(cfg, vxp_list, n_list)
    out = C.c_int64(0)
    rc = lib().o_part_flux_emitter_ctr(C.byref(cfg), C.byref(emit), ip(bcnd), seed, it, S, ptrs,
                                       npa.ctypes.data_as(_LP), cap.ctypes.data_as(_LP), cnt.ctypes.data_as(_LP),
                                       dp(Pi), C.byref(out))
    ns = cfg.ntype
    return rc, npa[:ns].copy(), cnt[:ns].copy(), Pi[:ns].copy(), out.value


# ---- averaging diagnostics (utils.f90) ---------------------------------------------------
def part_moments(cfg, size_na, ptype, vxp, kq):
    na1, na2 = cfg.nx // size_na, cfg.ny // size_na
    p = np.zeros((4, na2 + 3, na1 + 3))
    lib().o_part_moments(C.byref(cfg), size_na, ptype, dp(np.ascontiguousarray(vxp)), vxp.shape[0], dp(kq), dp(p))
    return p


def calc_avg(cfg, size_na, ptype, npg, p_mts, data_pavg, ss=None):
    """data_pavg: (ntype, na2+1, na1+1, 7) array, accumulated in place; ss: the species'
    (2, ny+3, nx+3) source and sink counts (or None)."""
    src = sink = None
    if ss is not None:
        src, sink = (np.ascontiguousarray(ss[k], dtype=np.float64) for k in (0, 1))
    lib().o_calc_avg(C.byref(cfg), size_na, ptype, dp(np.ascontiguousarray(npg)), dp(p_mts), dp(data_pavg),
                     dp(src), dp(sink))
