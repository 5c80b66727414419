"""ctypes binding of libmagic_b200.so (the C ABI in include/magic_b200.h).

The library is built in-tree (``magic_b200/csrc/build.py``).  There is no
fallback: if the library is missing or cannot be loaded, ``lib()`` raises.
"""

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmagic_b200.so")

MT_OK = 0
MT_PREC_FP64 = 0
MT_PREC_SPLIT = 1
MT_PREC_OZAKI = 2

_dp = C.c_void_p  # device pointer
_i64 = C.c_int64


class GridDesc(C.Structure):
    _fields_ = [("l_max", C.c_int), ("minc", C.c_int), ("n_theta_max", C.c_int),
                ("n_phi_max", C.c_int), ("precision", C.c_int)]


class PlanInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("l_max", "minc", "n_theta_max", "n_phi_max",
                                       "n_m_max", "lm_max", "nhs", "precision")]


class AnelParams(C.Structure):
    _fields_ = [(n, _dp) for n in ("r", "or1", "or2", "or4", "beta", "orho1", "otemp1",
                                   "visc", "lambda_")] + \
               [("LFfac", C.c_double), ("ViscHeatFac", C.c_double),
                ("OhmLossFac", C.c_double), ("l_mag", C.c_int)]


class CourantParams(C.Structure):
    _fields_ = [(n, _dp) for n in ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")] + \
               [("courfac", C.c_double), ("alffac", C.c_double), ("LFfac", C.c_double),
                ("opm", C.c_double), ("mode", C.c_int)]


class BoussIn(C.Structure):
    _fields_ = [(n, _dp) for n in ("w", "dw", "ddw", "z", "dz", "s", "b", "db", "ddb",
                                   "aj", "dj", "xi")] + [("ld", _i64)]


class BoussOut(C.Structure):
    _fields_ = [(n, _dp) for n in ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt",
                                   "VxBp", "VXir", "VXit")] + [("ld", _i64)]


class BoussParams(C.Structure):
    _fields_ = [(n, _dp) for n in ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")] + \
               [("LFfac", C.c_double), ("courfac", C.c_double), ("alffac", C.c_double),
                ("opm", C.c_double), ("l_mag", C.c_int), ("l_chem", C.c_int),
                ("cour_mode", C.c_int), ("parts", C.c_int), ("LFfac_r", _dp)]


class AnelIn(C.Structure):
    _fields_ = [(n, _dp) for n in ("w", "dw", "ddw", "z", "dz", "s", "xi", "b", "db", "ddb",
                                   "aj", "dj")] + [("ld", _i64)]


class AnelOut(C.Structure):
    _fields_ = [(n, _dp) for n in ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp",
                                   "VXir", "VXit", "heat")] + [("ld", _i64)]


class AnelStageParams(C.Structure):
    _fields_ = [(n, _dp) for n in ("r", "or1", "or2", "or4", "beta", "orho1", "orho2", "otemp1",
                                   "visc", "lambda_", "delxr2", "delxh2")] + \
               [(n, C.c_double) for n in ("LFfac", "ViscHeatFac", "OhmLossFac", "courfac",
                                          "alffac", "opm")] + \
               [("l_mag", C.c_int), ("l_chem", C.c_int), ("cour_mode", C.c_int)]


class TdIn(C.Structure):
    _fields_ = [(n, _dp) for n in ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp",
                                   "VXir", "VXit", "w", "dw", "ddw", "z", "dz")] + [("ld", _i64),
                                                                                   ("heat", _dp)]


class TdOut(C.Structure):
    _fields_ = [(n, _dp) for n in ("dwdt", "dzdt", "dpdt", "dsdt", "dxidt", "dbdt",
                                   "djdt")] + [("ld", _i64)]


class TdParams(C.Structure):
    _fields_ = [(n, _dp) for n in ("r", "or1", "or2", "or4", "orho1", "beta")] + \
               [("CorFac", C.c_double)] + \
               [(n, C.c_int) for n in ("l_double_curl", "l_heat", "l_mag", "l_chem", "l_anel")]


class FieldUpdate(C.Structure):
    _fields_ = [(n, _dp) for n in ("x", "dx", "d2x", "old", "impl", "expl0", "expl1", "top",
                                   "bot")] + \
               [("ld", _i64)] + \
               [(n, C.c_double) for n in ("w_old", "w_impl", "w_expl0", "w_expl1")] + \
               [(n, _dp) for n in ("so_l", "so_r", "ia_l", "ia_r", "ib_r", "ic_r", "ic_l",
                                   "ic_r2")]


class AmCorrection(C.Structure):
    _fields_ = [(n, _dp) for n in ("rint", "r", "am_z", "am_dz", "am_d2z")] + \
               [(n, C.c_double) for n in ("c_moi_oc", "am_start")] + \
               [(n, C.c_int) for n in ("axial", "equatorial")]


class PoloidalUpdate(C.Structure):
    _fields_ = [(n, _dp) for n in ("w", "dw", "ddw", "old", "impl", "expl0", "expl1", "p", "s",
                                   "xi")] + [("ld", _i64)] + \
               [(n, C.c_double) for n in ("w_old", "w_impl", "w_expl0", "w_expl1", "wimp_lin0",
                                          "BuoFac", "ChemFac")] + \
               [(n, _dp) for n in ("hdif", "or2", "orho1", "beta", "visc", "rgrav", "rho0", "c3",
                                   "c2n", "c1n", "c1d", "c0n")]


class WpUpdate(C.Structure):
    _fields_ = [(n, _dp) for n in ("w", "dw", "ddw", "p", "dp", "w_old", "w_impl", "w_expl0",
                                   "w_expl1", "p_old", "p_impl", "p_expl0", "p_expl1", "s",
                                   "xi")] + [("ld", _i64)] + \
               [(n, C.c_double) for n in ("w_old_wt", "w_impl_wt", "w_expl0_wt", "w_expl1_wt",
                                          "wimp_lin0", "BuoFac", "ChemFac")] + \
               [(n, _dp) for n in ("hdif", "or1", "or2", "beta", "dbeta", "visc", "dLvisc",
                                   "rgrav", "rho0")] + [("impl_interior", C.c_int),
                                                        ("p0_row0", _dp)]


class LevelCopy(C.Structure):
    _fields_ = [("src", _dp), ("dst", _dp), ("src_ld", _i64), ("dst_ld", _i64),
                ("src_col0", C.c_int), ("dst_col0", C.c_int), ("n_cols", C.c_int),
                ("pad", C.c_int)]


class EnergyArgs(C.Structure):
    _fields_ = [(n, _dp) for n in ("pol", "dpol", "tor")] + [("ld", _i64)] + \
               [(n, _dp) for n in ("or2", "cr", "rint")] + [("magnetic", C.c_int)]


# name -> (restype, argtypes)
_PROTOS = {
    "mt_plan_create": (C.c_int, [C.POINTER(GridDesc), C.POINTER(C.c_void_p)]),
    "mt_plan_destroy": (C.c_int, [C.c_void_p]),
    "mt_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    "mt_plan_copy_tables": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "mt_transform_workspace": (C.c_size_t, [C.c_void_p, C.c_int, C.c_int]),
    "mt_scal_to_spat": (C.c_int, [C.c_void_p, _dp, _i64, C.c_int, _dp, _dp, C.c_size_t, _dp]),
    "mt_scal_to_spat_noalloc": (C.c_int, [C.c_void_p, _dp, _i64, C.c_int, _dp, _dp]),
    "mt_scal_to_SH": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, _i64, _dp, C.c_size_t, _dp]),
    "mt_torpol_to_spat": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _i64, C.c_int, _dp, _dp, _dp,
                                    _dp, C.c_size_t, _dp]),
    "mt_spat_to_sphertor": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, _i64, _dp,
                                      C.c_size_t, _dp]),
    "mt_scal_to_grad_spat": (C.c_int, [C.c_void_p, _dp, _i64, C.c_int, C.c_int, _dp, _dp,
                                       _dp, C.c_size_t, _dp]),
    "mt_get_nl": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_dp), C.POINTER(_dp), _dp, _dp,
                            C.c_double, _dp]),
    "mt_get_nl_anel": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_dp), C.POINTER(_dp),
                                 C.POINTER(AnelParams), _dp]),
    "mt_courant_workspace": (C.c_size_t, [C.c_void_p, C.c_int]),
    "mt_courant": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                             C.POINTER(CourantParams), _dp, _dp, _dp, C.c_size_t, _dp]),
    "mt_nl_bouss_workspace": (C.c_size_t, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "mt_nl_bouss": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(BoussIn), C.POINTER(BoussOut),
                              C.POINTER(BoussParams), _dp, _dp, _dp, C.c_size_t, _dp]),
    "mt_nl_anel_workspace": (C.c_size_t, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "mt_nl_anel": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(AnelIn), C.POINTER(AnelOut),
                             C.POINTER(AnelStageParams), _dp, _dp, _dp, C.c_size_t, _dp]),
    "mt_radial_op_create": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    "mt_radial_op_create_dct1": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "mt_radial_op_destroy": (C.c_int, [C.c_void_p]),
    "mt_radial_op_bandwidth": (C.c_int, [C.c_void_p]),
    "mt_radial_apply": (C.c_int, [C.c_void_p, C.c_int, _dp, _i64, _dp, _i64, _dp]),
    "mt_radial_apply2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, _dp, _i64, _dp, _dp, _i64,
                                   _dp]),
    "mt_get_td": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TdIn), C.POINTER(TdOut),
                            C.POINTER(TdParams), C.c_void_p, _dp]),
    "mt_lop_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    "mt_energy_workspace": (C.c_size_t, [C.c_void_p]),
    "mt_energy": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(EnergyArgs), _dp, _dp, C.c_size_t,
                            _dp]),
    "mt_lop_create_band": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_void_p)]),
    "mt_lop_destroy": (C.c_int, [C.c_void_p]),
    "mt_update_field": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FieldUpdate), C.c_void_p,
                                  C.c_void_p, C.c_void_p, _dp]),
    "mt_correct_am": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FieldUpdate),
                                C.POINTER(AmCorrection), _dp]),
    "mt_update_poloidal": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(PoloidalUpdate), C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, _dp]),
    "mt_update_wp": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(WpUpdate), C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _dp]),
    "mt_selftest_wait_timeout": (C.c_int, [_dp, C.c_longlong, _dp]),
    "mt_copy_levels": (C.c_int, [C.c_int, _dp, C.c_int, _dp]),
    "mt_device_status": (C.c_int, [_dp, C.POINTER(C.c_int), _dp]),
    "mt_noalloc_status": (C.c_int, [C.POINTER(C.c_int), _dp]),
    "mt_last_error": (C.c_char_p, []),
}

EXPORTED = tuple(_PROTOS)

_lib = None


def lib():
    """Load (once) and return the library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m magic_b200.csrc.build` "
                "(magic_b200 has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class MagicError(RuntimeError):
    pass


def check(rc):
    if rc != MT_OK:
        msg = lib().mt_last_error().decode(errors="replace")
        raise MagicError(f"magic_b200 status {rc}: {msg}")


# Codes the split-precision kernels record in the first int of their workspace
# when a bounded wait runs out (the wait that gave up; see umma.cuh callers).
DEVICE_STATUS = {
    2: "synthesis GEMM epilogue: accumulator never became ready",
    3: "synthesis GEMM loader: operand stage never freed",
    4: "synthesis GEMM MMA issuer: operand copy never landed",
    6: "synthesis GEMM MMA issuer: accumulator never drained",
    12: "analysis GEMM epilogue: accumulators never became ready",
    13: "analysis GEMM loader: operand stage never freed",
    14: "analysis GEMM MMA issuer: operand copy never landed",
    22: "digit synthesis GEMM epilogue: accumulators never became ready",
    23: "digit synthesis GEMM loader: operand stage never freed",
    24: "digit synthesis GEMM MMA issuer: operand copy never landed",
    26: "digit synthesis GEMM MMA issuer: accumulators never drained",
    32: "digit analysis GEMM epilogue: accumulators never became ready",
    33: "digit analysis GEMM loader: operand stage never freed",
    34: "digit analysis GEMM MMA issuer: operand copy never landed",
    36: "digit analysis GEMM MMA issuer: accumulators never drained",
    99: "self-test wait (nothing arrives by design)",
}


def describe_status(code):
    """Text for a device status code (0 = every bounded wait completed)."""
    if code == 0:
        return "ok"
    return DEVICE_STATUS.get(code, "a bounded tensor-pipe wait ran out") + f" (code {code})"


def raise_device_status(code, what="split-precision call"):
    if code != 0:
        raise MagicError(f"magic_b200 device status after {what}: {describe_status(code)}; "
                         "its results are invalid")
