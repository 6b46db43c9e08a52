"""ctypes binding of the C ABI declared in ``include/maos_b200.h``.

The structs below mirror the header field by field.  Loading fails loudly when
``libmaosb200.so`` is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmaosb200.so")

MB_OK = 0
MB_MVM_F32, MB_MVM_BF16, MB_MVM_FP8 = 0, 1, 2
ERRORS = {-1: "MB_EINVAL", -2: "MB_ECUDA", -3: "MB_ENOMEM", -4: "MB_ESTATE", -5: "MB_EUNSUP",
          -6: "MB_ENUM"}


class MbGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("ox", C.c_double), ("oy", C.c_double), ("ht", C.c_double)]


class MbWfsDesc(C.Structure):
    _fields_ = [("thetax", C.c_double), ("thetay", C.c_double), ("hs", C.c_double),
                ("nsa", C.c_int), ("dsa", C.c_double),
                ("salocx", C.POINTER(C.c_double)), ("salocy", C.POINTER(C.c_double)),
                ("gp_p", C.POINTER(C.c_int)), ("gp_i", C.POINTER(C.c_int)),
                ("gp_x", C.POINTER(C.c_double)), ("neai", C.POINTER(C.c_double)),
                ("ptt", C.POINTER(C.c_double))]


class MbFdpcgGeom(C.Structure):
    _fields_ = [("nxp", C.c_int), ("nyp", C.c_int), ("dxp", C.c_double), ("pos", C.c_int), ("adimx", C.c_int),
                ("adimy", C.c_int), ("gx", C.POINTER(C.c_double)), ("gy", C.POINTER(C.c_double)),
                ("nsel", C.c_int), ("sel_dx", C.POINTER(C.c_int)), ("sel_dy", C.POINTER(C.c_int)),
                ("sel_r", C.POINTER(C.c_double)), ("needscale", C.c_int), ("neam", C.POINTER(C.c_double))]


class MbFdpcgDesc(C.Structure):
    _fields_ = [("nb", C.c_int), ("bs", C.c_int), ("scale", C.c_int),
                ("perm", C.POINTER(C.c_long)), ("mbinv", C.POINTER(C.c_double)),
                ("mdata", C.POINTER(C.c_double)), ("mdiag", C.POINTER(C.c_double)),
                ("geom", C.POINTER(MbFdpcgGeom))]


class MbCsc(C.Structure):
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("p", C.POINTER(C.c_int)), ("i", C.POINTER(C.c_int)),
                ("x", C.POINTER(C.c_double))]


class MbFitDesc(C.Structure):
    _fields_ = [("floc", MbGrid), ("nfit", C.c_int), ("thetax", C.POINTER(C.c_double)),
                ("thetay", C.POINTER(C.c_double)), ("wt", C.POINTER(C.c_double)),
                ("hs", C.POINTER(C.c_double)), ("w0_p", C.POINTER(C.c_int)),
                ("w0_i", C.POINTER(C.c_int)), ("w0_x", C.POINTER(C.c_double)),
                ("w1", C.POINTER(C.c_double)), ("ndm", C.c_int), ("amap", C.POINTER(MbGrid)),
                ("nnw", C.c_int), ("nw", C.POINTER(C.c_double)), ("maxit", C.c_int),
                ("actslave", MbCsc)]


class MbFitSparseDesc(C.Structure):
    _fields_ = [("frm", MbCsc), ("nfr", C.c_int), ("fru", C.POINTER(C.c_double)), ("frv", C.POINTER(C.c_double)),
                ("flm", MbCsc), ("nfl", C.c_int), ("flu", C.POINTER(C.c_double)), ("flv", C.POINTER(C.c_double)),
                ("maxit", C.c_int)]


class MbReconDesc(C.Structure):
    _fields_ = [("pmap", MbGrid), ("nps", C.c_int), ("xmap", C.POINTER(MbGrid)),
                ("l2c", C.POINTER(C.c_double)), ("nwfs", C.c_int),
                ("wfs", C.POINTER(MbWfsDesc)), ("maxit", C.c_int), ("precond", C.c_int),
                ("split", C.c_int), ("fdpcg", C.POINTER(MbFdpcgDesc)), ("nbatch", C.c_int),
                ("fit", C.POINTER(MbFitDesc)), ("fit_sparse", C.POINTER(MbFitSparseDesc))]


_PI = C.POINTER(C.c_int)
_PD = C.POINTER(C.c_double)


class MbGeomWfsDesc(C.Structure):
    _fields_ = [("nwfs", C.c_int), ("nsa", _PI), ("nxsa", _PI), ("dx", _PD), ("gox", _PD), ("goy", _PD),
                ("thetax", _PD), ("thetay", _PD), ("hs", _PD), ("sa_ix", _PI), ("sa_iy", _PI),
                ("sa_stencil", _PI), ("nstencil", C.c_int), ("stencil_off", C.POINTER(C.c_long)),
                ("stencils", _PD), ("stencil_len", C.c_long), ("nea", _PD), ("natm", C.c_int),
                ("atm_nx", _PI), ("atm_ny", _PI), ("atm_dx", _PD), ("atm_ox", _PD), ("atm_oy", _PD),
                ("atm_ht", _PD), ("atm_vx", _PD), ("atm_vy", _PD), ("ndm", C.c_int), ("dm_nx", _PI),
                ("dm_ny", _PI), ("dm_dx", _PD), ("dm_ox", _PD), ("dm_oy", _PD), ("dm_ht", _PD),
                ("dt", C.c_double), ("nbatch", C.c_int)]


# every symbol the header declares, with (restype, argtypes)
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
SIGNATURES = {
    "mb_init": (C.c_int, [C.c_int]),
    "mb_cleanup": (None, []),
    "mb_setup_recon": (C.c_int, [C.POINTER(MbReconDesc), C.POINTER(C.c_void_p)]),
    "mb_recon_free": (None, [C.c_void_p]),
    "mb_recon_reset": (C.c_int, [C.c_void_p]),
    "mb_update_recon_nea": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "mb_update_recon_cn2": (C.c_int, [C.c_void_p, _D, C.POINTER(MbFdpcgDesc)]),
    "mb_tomo": (C.c_int, [C.c_void_p, _D, _D, _F]),
    "mb_tomo_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mb_fit": (C.c_int, [C.c_void_p, _D, _F]),
    "mb_fdpcg_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "mb_fdpcg_shape": (C.c_int, [C.c_void_p, C.c_int]),
    "mb_update_recon_neam": (C.c_int, [C.c_void_p, _D]),
    "mb_fdpcg_data": (C.c_int, [C.c_void_p, _D]),
    "mb_tomo_wfs": (C.c_int, [C.c_void_p, C.POINTER(_D), C.POINTER(_D), _F]),
    "mb_fit_opdr": (C.c_int, [C.c_void_p, C.POINTER(_D), _D, _F]),
    "mb_recon_step_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mb_group_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    "mb_group_step_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p]),
    "mb_group_graph_kernels": (C.c_long, [C.c_void_p]),
    "mb_group_free": (None, [C.c_void_p]),
    "mb_fit_solution": (C.c_void_p, [C.c_void_p]),
    "mb_nact": (C.c_long, [C.c_void_p]),
    "mb_apply_fit_R": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_apply_fit_L": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_tomo_solution": (C.c_void_p, [C.c_void_p]),
    "mb_recon_stream": (C.c_void_p, [C.c_void_p]),
    "mb_num_stages": (C.c_int, []),
    "mb_stage_name": (C.c_char_p, [C.c_int]),
    "mb_time_stages": (C.c_int, [C.c_void_p, C.c_int, _F, _D, C.POINTER(C.c_int)]),
    "mb_tomo_residual": (C.c_int, [C.c_void_p, _F]),
    "mb_recon_reset_slot": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mb_slot_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mb_slot_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mb_recon_step_slots": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p]),
    "mb_recon_serve_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p]),
    "mb_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "mb_ngrad": (C.c_long, [C.c_void_p]),
    "mb_nxtot": (C.c_long, [C.c_void_p]),
    "mb_nbatch": (C.c_int, [C.c_void_p]),
    "mb_apply_tomo_R": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_apply_tomo_L": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_apply_fdpcg": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_apply_hx": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_kernel_launches": (C.c_long, [C.c_int]),
    "mb_mvm_create": (C.c_int, [_D, C.c_long, C.c_long, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mb_mvm_free": (None, [C.c_void_p]),
    "mb_mvm_bytes": (C.c_long, [C.c_void_p]),
    "mb_recon_mvm": (C.c_int, [C.c_void_p, _D, _D]),
    "mb_mvm_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mb_mvm_apply_noalloc": (C.c_int, [C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_void_p]),
    "mb_servo_create": (C.c_int, [C.c_long, _D, C.c_int, C.c_int, _D, C.c_int, C.c_int, C.c_double,
                                  C.POINTER(C.c_void_p)]),
    "mb_servo_filter": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mb_servo_reset": (C.c_int, [C.c_void_p]),
    "mb_servo_free": (None, [C.c_void_p]),
    "mb_geom_wfs_create": (C.c_int, [C.POINTER(MbGeomWfsDesc), C.POINTER(C.c_void_p)]),
    "mb_geom_wfs_set_atm": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D]),
    "mb_geom_wfs_set_wind": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]),
    "mb_geom_wfs_grad": (C.c_int, [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_void_p]),
    "mb_geom_wfs_ngrad": (C.c_long, [C.c_void_p]),
    "mb_geom_wfs_nact": (C.c_long, [C.c_void_p]),
    "mb_geom_wfs_free": (None, [C.c_void_p]),
    "mb_error_string": (C.c_char_p, [C.c_int]),
    "mb_last_error_message": (C.c_char_p, []),
    "mb_version": (C.c_int, []),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the native library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"maos_b200 native library not built: {path} "
                           "(run python -m maos_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MbError(RuntimeError):
    def __init__(self, code: int, where: str):
        lib = load()
        msg = lib.mb_last_error_message().decode(errors="replace")
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({msg})")
        self.code = code


def check(code: int, where: str) -> None:
    if code != MB_OK:
        raise MbError(code, where)
