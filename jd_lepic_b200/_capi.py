"""ctypes mirror of ``include/lepic_gpu.h`` (the C ABI of the sm_100a library).

The structures below must match the header field for field; ``tests/test_capi_cpu.py``
checks that every symbol the header declares is exported by the shared library.
The library is the in-tree ``jd_lepic_b200/_lib/liblepic_gpu.so``; if it is missing the
load fails loudly (there is no CPU fallback of the product path).
"""
from __future__ import annotations

import ctypes as C
import os

MAXSP = 8
MAXCOL = 64

OK = 0
EINVAL = -1
ENOMEM = -2
ECUDA = -3
ECAPACITY = -4
EDIVERGED = -5
ETIMEOUT = -6
ERANGE = -7
ENOTCONV = -8
ENOKERNEL = -9

ERROR_NAMES = {
    EINVAL: "LEPIC_EINVAL", ENOMEM: "LEPIC_ENOMEM", ECUDA: "LEPIC_ECUDA",
    ECAPACITY: "LEPIC_ECAPACITY", EDIVERGED: "LEPIC_EDIVERGED", ETIMEOUT: "LEPIC_ETIMEOUT",
    ERANGE: "LEPIC_ERANGE", ENOTCONV: "LEPIC_ENOTCONV", ENOKERNEL: "LEPIC_ENOKERNEL",
}

POISSON_FP64_MG = 0
POISSON_MIXED_IR = 1
POISSON_FP64_MG_L2 = 2
POISSON_LEARNED = 3
POISSON_FP64_PCG = 4

GRID_PHI = 0
GRID_RHS = 1
GRID_EI = 2
GRID_NP = 16

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "liblepic_gpu.so")


class LepicConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("zmax", C.c_double),
        ("dt", C.c_double),
        ("eps0", C.c_double), ("qe", C.c_double),
        ("flag_pbc", C.c_int32), ("flag_spec", C.c_int32), ("flag_nmn", C.c_int32),
        ("flag_B", C.c_int32),
        ("flag_B_pos", C.c_int32),
        ("Bc", C.c_double * 3),
        ("ntype", C.c_int32),
        ("nsp", C.c_int32),
        ("charge", C.c_double * MAXSP), ("mass", C.c_double * MAXSP),
        ("Nm", C.c_double * MAXSP), ("vt0", C.c_double * MAXSP),
        ("np_mx", C.c_double * MAXSP),
        ("nu_uplim", C.c_double * MAXSP),
        ("ns_coll", C.c_int32), ("nsort", C.c_int32),
        ("ng", C.c_int32),
        ("ncycl", C.c_int32),
        ("omega", C.c_double),
        ("capacity", C.c_int64 * MAXSP),
        ("seed", C.c_uint64),
        ("tile_w", C.c_int32), ("tile_h", C.c_int32),
    ]


class LepicXsTables(C.Structure):
    _fields_ = [
        ("npt", C.c_int32), ("ncol", C.c_int32),
        ("sig_Er", C.POINTER(C.c_double)),
        ("sig", C.POINTER(C.c_double)),
        ("Eth", C.POINTER(C.c_double)),
        ("col_info", C.POINTER(C.c_int32)),
        ("p_ncol", C.POINTER(C.c_int32)),
        ("sig_list", C.POINTER(C.c_int32)),
        ("sigv_mx", C.POINTER(C.c_double)),
        ("flag_ionrep", C.c_int32),
        ("fEk", C.c_double),
    ]


class LepicSolveStats(C.Structure):
    _fields_ = [
        ("cycles", C.c_int32), ("sweeps_fine", C.c_int32),
        ("res_l1", C.c_double), ("res_l2_rel", C.c_double), ("ktot", C.c_double),
    ]


class LepicPushStats(C.Structure):
    _fields_ = [
        ("np_tot", C.c_int64 * MAXSP), ("n_lost", C.c_int64 * MAXSP),
        ("n_dead", C.c_int64 * MAXSP), ("n_slots", C.c_int64 * MAXSP),
    ]


class LepicMccStats(C.Structure):
    _fields_ = [
        ("n_cand", C.c_int64 * MAXSP), ("n_coll", C.c_int64 * MAXCOL),
        ("n_add", C.c_int64 * MAXSP), ("n_overflow", C.c_int64),
        ("nu_max", C.c_double * MAXSP),
    ]


class LepicLoadSpec(C.Structure):
    _fields_ = [
        ("n_samples", C.c_int64),
        ("profile", C.c_int32),
        ("x_load", C.c_double),
        ("n_peak", C.c_double), ("n_floor", C.c_double),
        ("sigma", C.c_double),
        ("seed", C.c_uint64),
    ]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
_VP = C.c_void_p

# name -> (restype, argtypes); every function declared in include/lepic_gpu.h
class LepicCnnConfig(C.Structure):
    _fields_ = [
        ("enable_training", C.c_int32), ("warmup_solves", C.c_int32), ("steps_warmup", C.c_int32),
        ("train_every", C.c_int32), ("steps_after", C.c_int32), ("crop", C.c_int32), ("batch", C.c_int32),
        ("lr", C.c_float), ("seed", C.c_uint64),
    ]


class LepicCnnStats(C.Structure):
    _fields_ = [
        ("solves", C.c_int64), ("train_steps", C.c_int64), ("last_accepted", C.c_int32),
        ("last_res_ratio", C.c_double), ("last_loss", C.c_double),
    ]


MAXICP = 16


class LepicSourceConfig(C.Structure):
    _fields_ = [
        ("flag_c", C.c_int32), ("xl_pow", C.c_double), ("xr_pow", C.c_double), ("yl_pow", C.c_double),
        ("yr_pow", C.c_double),
        ("flag_heat", C.c_int32), ("ns_heat", C.c_int32), ("eheat_type", C.c_int32), ("flag_gpp", C.c_int32),
        ("n_icp", C.c_int32), ("te_update", C.c_int32),
        ("nudt", C.c_double), ("nu_h", C.c_double), ("Pabs", C.c_double * MAXICP), ("Pabs_cor", C.c_double),
        ("vt", C.c_double * MAXICP),
        ("flag_inj", C.c_int32), ("ns_inj", C.c_int32), ("opt_inj", C.c_int32), ("flag_Tp", C.c_int32),
        ("flag_diffsrc", C.c_int32), ("tag_neg", C.c_int32), ("nproc_mpi", C.c_int32),
        ("I_inj", C.c_double), ("THm", C.c_double), ("ni0", C.c_double * MAXSP), ("seed", C.c_uint64),
        ("js", C.c_double), ("ptype_fx", C.c_int32), ("tag_b", C.c_int32), ("ns_Hm", C.c_int32),
        ("n_holes", C.c_int32), ("xg1", C.c_double), ("Lg", C.c_double), ("Lh", C.c_double),
        ("flag_chmfrd", C.c_int32), ("chmfrd", C.c_double * 4), ("th_B", C.c_double),
    ]


class LepicSourceTally(C.Structure):
    _fields_ = [
        ("P_heat", C.c_double), ("n_heated", C.c_int64), ("n_heat_calls", C.c_int64),
        ("P_inj", C.c_double * MAXSP), ("P_src", C.c_double * MAXSP), ("n_inj", C.c_int64 * MAXSP),
        ("n_inj_last", C.c_int64 * MAXSP), ("n_icp", C.c_int32), ("Nh", C.c_int64 * MAXICP),
        ("sum_dEk", C.c_double * MAXICP), ("vt", C.c_double * MAXICP),
        ("n_emit", C.c_int64 * MAXSP), ("n_emit_last", C.c_int64 * MAXSP), ("n_emit_out", C.c_int64),
    ]


MAXLABEL = 16
MAXRG = 8


class LepicTallies(C.Structure):
    _fields_ = [
        ("n_loss", (C.c_int64 * MAXLABEL) * MAXSP), ("P_w", (C.c_double * MAXLABEL) * MAXSP),
        ("P_loss", (C.c_double * MAXSP) * 4), ("cnt_col", ((C.c_double * MAXRG) * MAXCOL) * 3),
        ("n_rg", C.c_int32),
    ]


_FP = C.POINTER(C.c_float)


class LepicZlossConfig(C.Structure):
    _fields_ = [("hz", C.c_double), ("phi0", C.c_double), ("size_na", C.c_int32)]


class LepicSecondaryConfig(C.Structure):
    _fields_ = [("gam_sec", C.c_double), ("igrid_sec", C.c_int32), ("pad", C.c_int32), ("xg_sec", C.c_double),
                ("THm", C.c_double)]


class LepicOptions(C.Structure):
    _fields_ = [("mx_nu1", C.c_int32), ("mx_nu2", C.c_int32), ("mx_nuc", C.c_int32), ("mx_omega", C.c_float),
                ("mx_onchip_bytes", C.c_int32), ("mx_tiled", C.c_int32), ("mx_max_iter", C.c_int32),
                ("mx_coarse_direct", C.c_int32),
                ("mg_small_nodes", C.c_int32), ("ctas_per_sm", C.c_int32), ("barrier_extra", C.c_int32),
                ("fortran_max_subrecord", C.c_int64), ("sort_defer", C.c_int32), ("pad", C.c_int32)]

PROTOTYPES = {
    "lepic_gpu_abi_version": (C.c_int32, []),
    "lepic_gpu_create": (C.c_int, [C.POINTER(LepicConfig), _IP, _DP, _DP, C.POINTER(LepicXsTables),
                                   C.POINTER(_VP)]),
    "lepic_gpu_destroy": (C.c_int, [_VP]),
    "lepic_gpu_stream": (_VP, [_VP]),
    "lepic_gpu_sync": (C.c_int, [_VP]),
    "lepic_gpu_last_error": (C.c_char_p, [_VP]),
    "lepic_gpu_put_particles": (C.c_int, [_VP, C.c_int32, _DP, C.c_int64]),
    "lepic_gpu_get_particles": (C.c_int, [_VP, C.c_int32, _DP, C.c_int64, C.POINTER(C.c_int64)]),
    "lepic_gpu_load_particles": (C.c_int, [_VP, C.POINTER(LepicLoadSpec)]),
    "lepic_gpu_put_particles_slabs": (C.c_int, [_VP, _DP, _IP, C.c_int64, C.c_int32, C.c_int32]),
    "lepic_gpu_get_particles_slabs": (C.c_int, [_VP, _DP, _IP, C.c_int64, C.c_int32, C.c_int32]),
    "lepic_gpu_charge_deposition": (C.c_int, [_VP]),
    "lepic_gpu_calc_rhs": (C.c_int, [_VP, _DP]),
    "lepic_gpu_dens_red": (C.c_int, [_VP, _DP, _DP]),
    "lepic_gpu_iterative_solver": (C.c_int, [_VP, _DP, C.c_double, C.c_int32, C.POINTER(LepicSolveStats)]),
    "lepic_gpu_iterative_solver_async": (C.c_int, [_VP, _DP, _DP, C.c_double, C.c_int32]),
    "lepic_gpu_get_grid_async": (C.c_int, [_VP, C.c_int32, _DP]),
    "lepic_gpu_stage_solver_input": (C.c_int, [_VP, _DP]),
    "lepic_gpu_calc_efield": (C.c_int, [_VP, _DP]),
    "lepic_gpu_part_sorting": (C.c_int, [_VP, C.c_int32, _IP]),
    "lepic_gpu_collisions": (C.c_int, [_VP, C.c_int32, C.POINTER(LepicMccStats)]),
    "lepic_gpu_push_deposit": (C.c_int, [_VP, C.c_int32, C.POINTER(LepicPushStats)]),
    "lepic_gpu_step": (C.c_int, [_VP, C.c_int32, C.c_double, C.c_int32]),
    "lepic_gpu_get_options": (C.c_int, [_VP, C.POINTER(LepicOptions)]),
    "lepic_gpu_set_options": (C.c_int, [_VP, C.POINTER(LepicOptions)]),
    "lepic_gpu_get_grid": (C.c_int, [_VP, C.c_int32, _DP]),
    "lepic_gpu_set_grid": (C.c_int, [_VP, C.c_int32, _DP]),
    "lepic_gpu_get_push_stats": (C.c_int, [_VP, C.POINTER(LepicPushStats)]),
    "lepic_gpu_get_mcc_stats": (C.c_int, [_VP, C.POINTER(LepicMccStats)]),
    "lepic_gpu_deposit_grid": (C.c_int, [_VP, C.c_int32, C.POINTER(_VP)]),
    "lepic_gpu_deposit_noalloc": (C.c_int, [_VP, _VP, _VP, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                            _VP, _VP, _VP]),
    "lepic_gpu_particle_arrays": (C.c_int, [_VP, C.c_int32, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                            C.POINTER(_VP), C.POINTER(_VP), C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int32)]),
    "lepic_gpu_set_sources": (C.c_int, [_VP, C.POINTER(LepicSourceConfig)]),
    "lepic_gpu_set_heating": (C.c_int, [_VP, _DP, C.c_int32, C.c_double]),
    "lepic_gpu_eheating": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_part_injection": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_heating_tally": (C.c_int, [_VP]),
    "lepic_gpu_flux_emitter": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_source_tallies": (C.c_int, [_VP, C.POINTER(LepicSourceTally), C.c_int32]),
    "lepic_gpu_write_backup": (C.c_int, [_VP, C.c_char_p, C.c_double, C.c_int32, C.c_double]),
    "lepic_gpu_read_backup": (C.c_int, [_VP, C.c_char_p, _DP, C.POINTER(C.c_int32), _DP]),
    "lepic_gpu_duplicate_particles": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_set_zloss": (C.c_int, [_VP, C.POINTER(LepicZlossConfig)]),
    "lepic_gpu_set_secondary": (C.c_int, [_VP, C.POINTER(LepicSecondaryConfig)]),
    "lepic_gpu_set_bohm_speed": (C.c_int, [_VP, _DP]),
    "lepic_gpu_set_dielectrics": (C.c_int, [_VP, _IP, C.c_double]),
    "lepic_gpu_dielectric_update": (C.c_int, [_VP]),
    "lepic_gpu_get_dielectric_charge": (C.c_int, [_VP, _DP]),
    "lepic_gpu_set_dielectric_charge": (C.c_int, [_VP, _DP]),
    "lepic_gpu_set_avg": (C.c_int, [_VP, C.c_int32, C.c_int32]),
    "lepic_gpu_set_regions": (C.c_int, [_VP, C.c_int32, _DP, _DP, C.c_double, C.c_double]),
    "lepic_gpu_get_tallies": (C.c_int, [_VP, C.POINTER(LepicTallies), C.c_int32]),
    "lepic_gpu_calc_avg": (C.c_int, [_VP]),
    "lepic_gpu_get_avg": (C.c_int, [_VP, _DP, _DP, C.POINTER(C.c_int32), C.c_int32]),
    "lepic_gpu_get_source_maps": (C.c_int, [_VP, _DP]),
    "lepic_gpu_set_source_option": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_set_warm_start": (C.c_int, [_VP, C.c_int32]),
    "lepic_gpu_cnn_configure": (C.c_int, [_VP, C.POINTER(LepicCnnConfig)]),
    "lepic_gpu_cnn_stats": (C.c_int, [_VP, C.POINTER(LepicCnnStats)]),
    "lepic_gpu_cnn_net": (_VP, [_VP]),
    "lepic_cnn_create": (C.c_int, [C.POINTER(_VP), C.c_uint64]),
    "lepic_cnn_destroy": (C.c_int, [_VP]),
    "lepic_cnn_nparams": (C.c_int, []),
    "lepic_cnn_params": (C.c_int, [_VP, _FP, C.c_int64, C.c_int32]),
    "lepic_cnn_loss_grad": (C.c_int, [_VP, _FP, _FP, _FP, C.c_int32, C.c_int32, C.c_int32, _FP, _FP,
                                      C.POINTER(C.c_double)]),
    "lepic_cnn_adam_step": (C.c_int, [_VP, C.c_float]),
    "lepic_cnn_last_error": (C.c_char_p, [_VP]),
}

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads the sm_100a library and binds every prototype; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing; run `python -m jd_lepic_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class LepicError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        super().__init__(f"{where} failed with {ERROR_NAMES.get(code, code)}: {detail}")
