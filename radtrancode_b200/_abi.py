"""ctypes mirror of the structures declared in include/radtran_b200.h.

Only layout lives here; loading of the shared library is in ``_lib.py``.
"""
import ctypes as C

import numpy as np

RTB_OK = 0
RTB_ERR_ARG = 1
RTB_ERR_LIMIT = 2
RTB_ERR_UNSUPPORTED = 3
RTB_ERR_CUDA = 4
RTB_ERR_NOTABLE = 5
RTB_ERR_NONPD = 6
RTB_ERR_RANGE = 7
RTB_ERR_GORD = 8
RTB_ERR_BUDGET = 9

STATUS_NAMES = {
    0: "RTB_OK", 1: "RTB_ERR_ARG", 2: "RTB_ERR_LIMIT", 3: "RTB_ERR_UNSUPPORTED",
    4: "RTB_ERR_CUDA", 5: "RTB_ERR_NOTABLE", 6: "RTB_ERR_NONPD", 7: "RTB_ERR_RANGE",
    8: "RTB_ERR_GORD", 9: "RTB_ERR_BUDGET",
}

KTAB_BY_ID = -2

MAXLAY, MAXPAT, MAXGAS, MAXCON, MAXG, MAXK, MAXV, MAXPRO = 400, 200, 30, 10, 51, 30, 401, 200
CIA_NUMPAIRS, CIA_NUMT, CIA_NUMWN = 9, 25, 1501

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class RtbConv(C.Structure):
    _fields_ = [
        ("nconv", C.c_int), ("vconv", _fp),
        ("nfwhm", C.c_int), ("vfwhm", _fp), ("xfwhm", _fp),
        ("nfil", C.c_int), ("vcen", _fp), ("nsub", _ip), ("vfil", _fp), ("fil", _fp),
    ]


class RtbAtm(C.Structure):
    _fields_ = [
        ("nlayer", C.c_int), ("ngas", C.c_int), ("ncont", C.c_int), ("npath", C.c_int),
        ("npro", C.c_int), ("nv", C.c_int), ("nwave", C.c_int),
        ("ld_lay", C.c_int), ("ld_con", C.c_int), ("ld_v", C.c_int), ("ld_param", C.c_int),
        ("press", _fp), ("temp", _fp), ("delh", _fp), ("pp", _fp), ("amount", _fp), ("cont", _fp),
        ("idgas", _ip), ("isogas", _ip), ("ktab", _ip),
        ("nlayin", _ip), ("imod", _ip), ("layinc", _ip), ("scale", _fp), ("emtemp", _fp),
        ("dte", _fp), ("dam", _fp), ("dco", _fp), ("dfp", _fp),
        ("xmap", _fp),
        ("vwave", _fp), ("xsec_ext", _fp),
        ("inormal", C.c_int), ("iray", C.c_int), ("itype", C.c_int), ("ispace", C.c_int),
        ("flagh2p", C.c_int), ("ilbl", C.c_int), ("inlte", C.c_int), ("iform", C.c_int),
        ("tsurf", C.c_float), ("fwhm", C.c_float),
        ("nem", C.c_int), ("vem", _fp), ("emissivity", _fp),
        ("conv", C.POINTER(RtbConv)),
        ("hfp", _fp),
        ("radius1", C.c_float), ("radextra", C.c_float),
        ("nlte_k1", C.c_float), ("nlte_A", C.c_float),
        ("dist", C.c_float),
        ("ih2o", C.c_int), ("ich4", C.c_int), ("inh3", C.c_int), ("io3", C.c_int), ("iuvscat", C.c_int),
    ]


class RtbProfile(C.Structure):
    _fields_ = [
        ("npro", C.c_int), ("nvmr", C.c_int), ("ndust", C.c_int), ("ld_pro", C.c_int), ("ld_con", C.c_int),
        ("h", _fp), ("p", _fp), ("t", _fp), ("vmr", _fp), ("dust", _fp),
        ("molwt", C.c_float), ("radius", C.c_float),
    ]


class RtbLayerOpts(C.Structure):
    _fields_ = [
        ("nlay", C.c_int), ("laytyp", C.c_int), ("layint", C.c_int),
        ("layht", C.c_float), ("layang", C.c_float), ("base", _fp),
        ("angle", C.c_float), ("botlay", C.c_int), ("ipzen", C.c_int),
    ]


class RtbLayers(C.Structure):
    _fields_ = [
        ("ld_lay", C.c_int), ("ld_con", C.c_int),
        ("baseh", _fp), ("delh", _fp), ("basep", _fp), ("baset", _fp), ("press", _fp), ("temp", _fp),
        ("totam", _fp), ("laysf", _fp), ("amount", _fp), ("pp", _fp), ("cont", _fp),
        ("dte", _fp), ("dam", _fp), ("dco", _fp),
        ("npath", _ip), ("nlayin", _ip), ("imod", _ip), ("layinc", _ip), ("scale", _fp), ("emtemp", _fp),
    ]


class RtbFwdStats(C.Structure):
    _fields_ = [
        ("cells", C.c_longlong), ("sort_passes", C.c_longlong), ("tie_passes", C.c_longlong),
        ("exact_passes", C.c_longlong), ("irregular_passes", C.c_longlong), ("block_passes", C.c_longlong),
        ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong), ("ms_kernel", C.c_float), ("grid", C.c_int),
    ]


class RtbRetrievalSpec(C.Structure):
    _fields_ = [
        ("atm", C.POINTER(RtbAtm)), ("nscale", C.c_int), ("scale_gas", _ip),
        ("y", _fp), ("sei", C.POINTER(C.c_double)), ("sa", C.POINTER(C.c_double)),
        ("xa", _fp), ("x0", _fp),
        ("scale_model", _ip), ("nprof", C.c_int), ("prof_gas", _ip),
        ("prof", C.POINTER(RtbProfile)), ("lopts", C.POINTER(RtbLayerOpts)),
        ("ndust", C.c_int), ("dust_type", _ip),
    ]


class RtbRetrievalOpts(C.Structure):
    _fields_ = [("kiter", C.c_int), ("phlimit", C.c_float), ("dchisq_stop", C.c_float), ("max_batch", C.c_int)]


class RtbRetrievalResult(C.Structure):
    _fields_ = [
        ("x", _fp), ("yn", _fp), ("phi", C.c_float), ("chisq", C.c_float), ("alambda", C.c_float),
        ("iterations", C.c_int), ("forwards", C.c_int), ("converged", C.c_int), ("nonpd", C.c_int),
        ("ms", C.c_double),
    ]


class RtbFwdTune(C.Structure):
    _fields_ = [("schedule", C.c_int), ("blocks_per_sm", C.c_int), ("ms", C.c_float), ("candidates", C.c_int),
                ("warps", C.c_int)]


class RtbNewtonStats(C.Structure):
    _fields_ = [("retrievals", C.c_longlong), ("ms_kernel", C.c_float)]


RESULT_KEYS = ("phi", "chisq", "alambda", "iterations", "forwards", "converged", "nonpd", "ms")


def fptr(a):
    """float* of a contiguous float32 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float32 and (a.flags.c_contiguous or a.flags.f_contiguous), a.dtype
    return a.ctypes.data_as(_fp)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and (a.flags.c_contiguous or a.flags.f_contiguous), a.dtype
    return a.ctypes.data_as(_ip)


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64
    return a.ctypes.data_as(C.POINTER(C.c_double))
