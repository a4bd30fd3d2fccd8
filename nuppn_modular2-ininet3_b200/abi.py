"""ctypes mirror of include/nuppn.h: knobs, network descriptor and per-zone stats.

The structures are laid out exactly as the C header declares them; ``make_desc`` keeps every numpy
array it points at alive on the returned object.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import synthnet as sn

P_D = C.POINTER(C.c_double)
P_I = C.POINTER(C.c_int32)
P_U8 = C.POINTER(C.c_uint8)

# per-zone outcome codes, utils/source/errors.F90:5-21
SLV_CNVRG, MAX_SUBSTEPS, BAD_STEP, NEG_ABUNDS, HUGE_ABUNDS, SUM_X, GOT_NAN, BAD_YE, NSE_CNVRG, \
    NSE_WEAK, SMALL_DT = range(1, 12)
BAD_INPUT = 20
ERROR_CODE = {0: "OK", 1: "CONVERGENCE", 2: "MAX_STEPS", 3: "BAD_STEP", 4: "NEGATIVE_X",
              5: "HUGE_X", 6: "SUM_X", 7: "NAN", 8: "BAD_YE", 9: "NSE_CNVRG", 10: "NSE_WEAK",
              11: "DT_UNDRFLOW", 20: "BAD_INPUT"}


class Knobs(C.Structure):
    _fields_ = [("ittd", C.c_int32), ("integration_method", C.c_int32),
                ("max_sub_steps", C.c_int32), ("interpolate_temp", C.c_int32),
                ("interpolate_dens", C.c_int32), ("screen_option", C.c_int32),
                ("detailed_balance", C.c_int32), ("weak_rates", C.c_int32),
                ("strong_rates", C.c_int32), ("decay", C.c_int32), ("i_nse", C.c_int32),
                ("nse_weak_method", C.c_int32), ("dgrd", C.c_double),
                ("grdthreshold", C.c_double), ("cyminformal", C.c_double),
                ("min_rate_ov_dt", C.c_double), ("min_t9_for_slv", C.c_double),
                ("delta_state_max", C.c_double), ("nse_min_t9", C.c_double),
                ("lu_precision", C.c_int32), ("ir_max_iters", C.c_int32),
                ("ir_rtol", C.c_double), ("threads_per_zone", C.c_int32),
                ("lu_onewarp_max", C.c_int32), ("lu_tile_max", C.c_int32),
                ("zones_per_cta", C.c_int32), ("zone_smem", C.c_int32),
                ("reserved", C.c_int32 * 3)]


def default_knobs(**over) -> Knobs:
    """&ppn_solver / &ppn_physics defaults (solver_knobs.F90:43-57, physics_knobs.F90:100-120)."""
    k = Knobs()
    k.ittd = 6
    k.integration_method = 0
    k.max_sub_steps = 4000
    k.interpolate_temp = 1
    k.interpolate_dens = 1
    k.screen_option = 2
    k.detailed_balance = 1
    k.weak_rates = 1
    k.strong_rates = 1
    k.decay = 0
    k.i_nse = 0
    k.nse_weak_method = 1
    k.dgrd = 1.0e-3
    k.grdthreshold = 1.0e-15
    k.cyminformal = 1.0e-30
    k.min_rate_ov_dt = 1.0e-99
    k.min_t9_for_slv = 0.01
    k.delta_state_max = 1.0e99
    k.nse_min_t9 = 6.0
    k.lu_precision = 0
    k.ir_max_iters = 3
    k.ir_rtol = 1.0e-14
    k.threads_per_zone = 0
    for name, val in over.items():
        setattr(k, name, val)
    return k


class NetDesc(C.Structure):
    _fields_ = [("nsp", C.c_int32), ("nre", C.c_int32), ("igamma", C.c_int32),
                ("anetw", P_D), ("znetw", P_D), ("considerisotope", P_U8), ("exmass", P_D),
                ("gspin", P_D), ("spec_part", P_I), ("k", P_I), ("ilabb", P_I),
                ("considerreaction", P_U8), ("rfac", P_D), ("src", P_I), ("src_idx", P_I),
                ("irev", P_I),
                ("rl_ncontrib", C.c_int32), ("rl_nrate", C.c_int32), ("rl_a", P_D),
                ("rl_rate", P_I), ("rl_chapter", P_I), ("rl_vflag", P_U8), ("rl_ecflag", P_U8),
                ("rl_nireac", P_I), ("rl_part", P_I), ("npart", C.c_int32), ("part_t9", P_D),
                ("part_val", P_D),
                ("vt_nrate", C.c_int32), ("vt_nterm", C.c_int32), ("vt_first", P_I),
                ("vt_terms", P_D), ("vt_dpow", P_D), ("vt_xfac", P_I),
                ("ng_kgrid", C.c_int32), ("ng_nreac", C.c_int32), ("ng_ndmax", C.c_int32),
                ("ng_t8", P_D), ("ng_flag", P_D), ("ng_ndata", P_I), ("ng_ane", P_D),
                ("ng_l10v", P_D),
                ("ff_nv", C.c_int32), ("ff_nt", C.c_int32), ("ff_nr", C.c_int32),
                ("ff_t9coo", P_D), ("ff_rhocoo", P_D), ("ff_l10v", P_D),
                ("kd_n", C.c_int32), ("kd_ne", C.c_int32), ("kd_e", P_D), ("kd_rate", P_D),
                ("nconst", C.c_int32), ("const_rate", P_D), ("vt_form", P_I)]


class ZoneStats(C.Structure):
    _fields_ = [("nsucc", C.c_int32), ("nfail", C.c_int32), ("newton_iters", C.c_int32),
                ("nfact", C.c_int32), ("nsolve", C.c_int32), ("nvar1_last", C.c_int32),
                ("ir_sweeps", C.c_int32), ("nvar1_max", C.c_int32)]


class ServeStats(C.Structure):
    """nuppn_serve_stats (include/nuppn.h)."""
    _fields_ = [("slots", C.c_int32), ("queue", C.c_int32), ("ctas", C.c_int32),
                ("pending", C.c_int32), ("in_flight", C.c_int32), ("launches", C.c_int64),
                ("published", C.c_int64), ("completed", C.c_int64), ("device_bytes", C.c_int64)]


class NetSetup(C.Structure):
    """nuppn_netsetup (include/nuppn.h)."""
    _fields_ = [("nsp", C.c_int32), ("nre", C.c_int32), ("nisomers", C.c_int32), ("nreac_isomers", C.c_int32),
                ("t9", C.c_double), ("rho", C.c_double), ("zis", C.c_void_p), ("considerisotope", C.c_void_p),
                ("anetw", C.c_void_p), ("znetw", C.c_void_p), ("isomeric_state", C.c_void_p),
                ("considerreaction", C.c_void_p), ("k", C.c_void_p), ("v", C.c_void_p), ("lab", C.c_void_p),
                ("labb", C.c_void_p), ("ilabb", C.c_void_p), ("rfac", C.c_void_p),
                ("bind_energy_diff", C.c_void_p)]


class TuneResult(C.Structure):
    _fields_ = [("threads_per_zone", C.c_int32), ("zones_per_cta", C.c_int32), ("zone_smem", C.c_int32),
                ("zones_per_sm", C.c_int32), ("ms", C.c_double), ("zone_steps_per_s", C.c_double),
                ("chosen", C.c_int32), ("reserved", C.c_int32)]


class NetInfo(C.Structure):
    _fields_ = [("nsp", C.c_int32), ("nre", C.c_int32), ("nspec_active", C.c_int32),
                ("nreac_active", C.c_int32), ("nnz_jac", C.c_int32), ("nnz_lu", C.c_int32),
                ("n_solve", C.c_int32), ("levels_lower", C.c_int32),
                ("levels_upper", C.c_int32), ("lu_flops", C.c_int64),
                ("device_bytes", C.c_int64)]


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def make_desc(net: sn.Network) -> NetDesc:
    """Descriptor pointing at contiguous copies of the network arrays (kept alive on it)."""
    keep = []

    def d(x):
        a = np.ascontiguousarray(x, dtype=np.float64)
        keep.append(a)
        return ptr(a, P_D)

    def i(x):
        a = np.ascontiguousarray(x, dtype=np.int32)
        keep.append(a)
        return ptr(a, P_I)

    def u(x):
        a = np.ascontiguousarray(x, dtype=np.uint8)
        keep.append(a)
        return ptr(a, P_U8)

    D = NetDesc()
    D.nsp, D.nre, D.igamma = net.nsp, net.nre, net.igamma
    D.anetw, D.znetw = d(net.anetw), d(net.znetw)
    D.considerisotope = u(net.considerisotope)
    D.exmass, D.gspin, D.spec_part = d(net.exmass), d(net.gspin), i(net.spec_part)
    D.k, D.ilabb = i(net.k.reshape(-1)), i(net.ilabb)
    D.considerreaction, D.rfac = u(net.considerreaction), d(net.rfac)
    D.src, D.src_idx, D.irev = i(net.src), i(net.src_idx), i(net.irev)
    D.rl_ncontrib, D.rl_nrate = len(net.rl_rate), len(net.rl_chapter)
    D.rl_a, D.rl_rate = d(net.rl_a.reshape(-1)), i(net.rl_rate)
    D.rl_chapter, D.rl_vflag, D.rl_ecflag = i(net.rl_chapter), u(net.rl_vflag), u(net.rl_ecflag)
    D.rl_nireac, D.rl_part = i(net.rl_nireac), i(net.rl_part.reshape(-1))
    D.npart, D.part_t9, D.part_val = len(net.part_val), d(net.part_t9), d(net.part_val.reshape(-1))
    D.vt_nrate, D.vt_nterm = len(net.vt_dpow), len(net.vt_terms)
    D.vt_first, D.vt_terms = i(net.vt_first), d(net.vt_terms.reshape(-1))
    D.vt_dpow, D.vt_xfac = d(net.vt_dpow), i(net.vt_xfac)
    D.ng_kgrid, D.ng_nreac = len(net.ng_t8), len(net.ng_flag)
    D.ng_ndmax = net.ng_ane.shape[1] if net.ng_ane.ndim == 2 else 1
    D.ng_t8, D.ng_flag, D.ng_ndata = d(net.ng_t8), d(net.ng_flag), i(net.ng_ndata)
    D.ng_ane, D.ng_l10v = d(net.ng_ane.reshape(-1)), d(net.ng_l10v.reshape(-1))
    D.ff_nv, D.ff_nt, D.ff_nr = len(net.ff_l10v), len(net.ff_t9coo), len(net.ff_rhocoo)
    D.ff_t9coo, D.ff_rhocoo, D.ff_l10v = d(net.ff_t9coo), d(net.ff_rhocoo), d(net.ff_l10v.reshape(-1))
    D.kd_n, D.kd_ne = len(net.kd_rate), len(net.kd_e)
    D.kd_e, D.kd_rate = d(net.kd_e), d(net.kd_rate.reshape(-1))
    D.nconst, D.const_rate = len(net.const_rate), d(net.const_rate if len(net.const_rate) else [0.0])
    vt_form = getattr(net, "vt_form", None)
    D.vt_form = i(vt_form if vt_form is not None and len(vt_form) else np.zeros(max(len(net.vt_dpow), 1)))
    D._keep = keep
    return D
