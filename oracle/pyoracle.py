"""ctypes front-end of the ORACLE library (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, as the checker.  The product never imports
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from radtrancode_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

ORC_MIXED, ORC_FP64 = 0, 1


class OrcTables(C.Structure):
    _fields_ = [
        ("ntab", C.c_int), ("np", C.c_int), ("nt", C.c_int), ("ng", C.c_int),
        ("lnp", C.POINTER(C.c_float)), ("tk", C.POINTER(C.c_float)), ("delg", C.POINTER(C.c_float)),
        ("vmin", C.POINTER(C.c_float)), ("delv", C.POINTER(C.c_float)), ("nbin", C.POINTER(C.c_int)),
        ("data", C.POINTER(C.c_float)),
        ("has_cia", C.c_int), ("dnu", C.c_float), ("cia_temps", C.POINTER(C.c_double)),
        ("kcia", C.POINTER(C.c_float)),
        ("npoint", C.c_int), ("vcen", C.POINTER(C.c_float)),
        ("has_para", C.c_int), ("ipara", C.c_int), ("dnu2", C.c_float),
        ("para_temps", C.POINTER(C.c_float)), ("para_fp", C.POINTER(C.c_float)),
        ("kh2h2", C.POINTER(C.c_float)), ("kh2he", C.POINTER(C.c_float)), ("kcia5", C.POINTER(C.c_float)),
        ("e3_tran", C.POINTER(C.c_double)), ("e3_e3", C.POINTER(C.c_double)),
        ("solar_npt", C.c_int), ("solar_wave", C.POINTER(C.c_float)), ("solar_rad", C.POINTER(C.c_float)),
    ]


class OrcDebug(C.Structure):
    _fields_ = [("perm", C.POINTER(C.c_int16)), ("split", C.POINTER(C.c_int16)),
                ("ties", C.POINTER(C.c_int16))]


NATIVE_PATH = os.path.join(HERE, "_build", "liboracle_native.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def use_native():
    """Load the -O3 -march=native build (made here, on the host that runs
    it) instead of the portable one: the timed CPU baseline.  Call before
    any other use of the oracle in the process."""
    global LIB_PATH
    if _lib is not None:
        raise RuntimeError("oracle already loaded")
    subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
    LIB_PATH = NATIVE_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_cirsrtfg_wave.restype = C.c_int
        L.orc_cirsrtfg_wave_mt.restype = C.c_int
        L.orc_det_expf_c.restype = C.c_float
        L.orc_det_expf_c.argtypes = [C.c_float]
        L.orc_planck_wave.restype = C.c_float
        L.orc_planck_wave.argtypes = [C.c_int, C.c_float, C.c_float]
        L.orc_planckg_wave.restype = C.c_float
        L.orc_planckg_wave.argtypes = [C.c_int, C.c_float, C.c_float]
        L.orc_locate.restype = C.c_int
        L.orc_locate.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_float]
        L.orc_calc_phiret.restype = C.c_float
        L.orc_calc_phiret_diag.restype = C.c_float
        L.orc_dinvertm_chol.restype = C.c_int
        _lib = L
    return _lib


def tables_struct(kt, cia=None, para=None, e3=None, solar=None):
    t = OrcTables()
    if solar is not None:
        t.solar_npt = len(solar.wave)
        t.solar_wave, t.solar_rad = _abi.fptr(solar.wave), _abi.fptr(solar.rad)
    if e3 is not None:
        t.e3_tran, t.e3_e3 = _abi.dptr(e3.tran), _abi.dptr(e3.e3)
    if para is None and cia is not None:
        para = getattr(cia, "para", None)
    if para is not None:
        t.has_para, t.ipara, t.dnu2 = 1, para.ipara, para.dnu2
        t.para_temps, t.para_fp = _abi.fptr(para.temps), _abi.fptr(para.fp)
        t.kh2h2, t.kh2he, t.kcia5 = _abi.fptr(para.kh2h2), _abi.fptr(para.kh2he), _abi.fptr(para.kcia5)
    t.ntab, t.np, t.nt, t.ng = kt.ntab, kt.np_, kt.nt, kt.ng
    t.lnp, t.tk, t.delg = _abi.fptr(kt.lnp), _abi.fptr(kt.tk), _abi.fptr(kt.delg)
    t.vmin, t.delv, t.nbin = _abi.fptr(kt.vmin), _abi.fptr(kt.delv), _abi.iptr(kt.nbin)
    t.data = _abi.fptr(kt.data)
    if kt.vcen is not None:
        t.npoint, t.vcen = len(kt.vcen), _abi.fptr(kt.vcen)
    if cia is not None:
        t.has_cia, t.dnu = 1, cia.dnu
        t.cia_temps = _abi.dptr(cia.temps)
        t.kcia = _abi.fptr(cia.kcia)
    t._keep = (kt, cia, para, e3, solar)
    return t


def cirsrtfg_wave(kt, cia, job, precision=ORC_MIXED, debug=False, nthreads=1, e3=None, solar=None):
    """Run the oracle forward model.  Returns (calcout, gradients, gradtsurf)
    as float64 arrays, plus (perm, split) debug arrays when requested.  e3 is
    e3interp's table (a synth.E3Table), needed by IMOD 18 paths; solar the
    stellar spectrum (a synth.StellarSpectrum) of iform 1 and 4."""
    L = lib()
    t = tables_struct(kt, cia, e3=e3, solar=solar)
    s = job.as_struct()
    n1, n2, n3 = job.out_shapes()
    out = np.zeros(n1), np.zeros(n2), np.zeros(n3)
    dbg = None
    perm = split = ties = None
    if debug and job.ngas > 1:
        npass = job.ngas - 1
        perm = np.full((job.nwave, job.nlayer, npass, kt.ng * kt.ng), -1, np.int16)
        split = np.full((job.nwave, job.nlayer, npass, kt.ng), -1, np.int16)
        ties = np.full((job.nwave, job.nlayer, npass), -1, np.int16)
        p16 = C.POINTER(C.c_int16)
        dbg = OrcDebug(perm.ctypes.data_as(p16), split.ctypes.data_as(p16), ties.ctypes.data_as(p16))
    dp = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in out]
    if nthreads > 1:
        st = L.orc_cirsrtfg_wave_mt(C.byref(t), C.byref(s), precision, dp[0], dp[1], dp[2], nthreads,
                                    C.byref(dbg) if dbg is not None else None)
    else:
        st = L.orc_cirsrtfg_wave(C.byref(t), C.byref(s), precision, dp[0], dp[1], dp[2],
                                 C.byref(dbg) if dbg is not None else None)
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    if debug:
        return out, (perm, split, ties)
    return out


def det_expf(x):
    L = lib()
    x = np.asarray(x, np.float32).ravel()
    return np.array([L.orc_det_expf_c(float(v)) for v in x], np.float32)


def sort2g(values):
    L = lib()
    a = np.ascontiguousarray(values, np.float32).copy()
    ib = np.zeros(a.size, np.int32)
    L.orc_sort2g(C.c_int(a.size), _abi.fptr(a), _abi.iptr(ib))
    return a, ib


def rankg(gw, weight, cont, grad):
    """rankg on one element set; grad shape (nparam, nloop)."""
    L = lib()
    gw = np.ascontiguousarray(gw, np.float32)
    weight = np.ascontiguousarray(weight, np.float32)
    cont = np.ascontiguousarray(cont, np.float32)
    grad = np.ascontiguousarray(grad, np.float32)
    nparam, nloop = grad.shape
    ng = gw.size
    k_g = np.zeros(ng, np.float32)
    dkdq = np.zeros((nparam, ng), np.float32)
    perm = np.zeros(nloop, np.int16)
    split = np.zeros(ng, np.int16)
    st = L.orc_rankg(C.c_int(nparam), _abi.fptr(gw), C.c_int(ng), C.c_int(nloop), _abi.fptr(weight),
                     _abi.fptr(cont), _abi.fptr(grad), _abi.fptr(k_g), _abi.fptr(dkdq),
                     perm.ctypes.data_as(C.POINTER(C.c_int16)), split.ctypes.data_as(C.POINTER(C.c_int16)))
    return st, k_g, dkdq, perm, split


class OrcTrace(C.Structure):
    _fields_ = [("n", C.c_int), ("phi", C.c_float * 64), ("verdict", C.c_int * 64), ("alambda", C.c_float * 64)]


def forward_state(kt, cia, case, x, precision=ORC_MIXED, nthreads=1, e3=None, solar=None):
    """Spectrum yn[ny] and K^T [nx, ny] of a retrieval case at state x."""
    L = lib()
    t = tables_struct(kt, cia, e3=e3, solar=solar)
    s = case.as_struct()
    x = np.ascontiguousarray(x, np.float32)
    yn = np.zeros(case.ny, np.float32)
    kk = np.zeros((case.nx, case.ny), np.float32)
    st = L.orc_forward_state(C.byref(t), C.byref(s), _abi.fptr(x), precision, nthreads, _abi.fptr(yn),
                             _abi.fptr(kk))
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    return yn, kk


def retrieve(kt, cia, case, kiter=10, phlimit=0.1, dchisq_stop=0.0, precision=ORC_MIXED, nthreads=1, e3=None,
             solar=None):
    """coreret restatement on one case: (result dict, trace dict)."""
    L = lib()
    t = tables_struct(kt, cia, e3=e3, solar=solar)
    s = case.as_struct()
    o = _abi.RtbRetrievalOpts(kiter, phlimit, dchisq_stop, 0)
    x = np.zeros(case.nx, np.float32)
    yn = np.zeros(case.ny, np.float32)
    r = _abi.RtbRetrievalResult()
    r.x, r.yn = _abi.fptr(x), _abi.fptr(yn)
    tr = OrcTrace()
    st = L.orc_retrieve(C.byref(t), C.byref(s), C.byref(o), precision, nthreads, C.byref(r), C.byref(tr))
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    res = {k: getattr(r, k) for k in _abi.RESULT_KEYS}
    res["x"], res["yn"] = x, yn
    trace = {"phi": np.array(tr.phi[:tr.n], np.float32), "verdict": np.array(tr.verdict[:tr.n]),
             "alambda": np.array(tr.alambda[:tr.n], np.float32)}
    return res, trace


def gain_matrix(kk, sei, sai):
    """calc_gain_matrix (diagonal Se): kk [nx, ny] (Fortran kk(ny, nx)).
    Returns (dd [nx, ny], aa [nx, nx]) as Fortran-ordered float64 arrays."""
    L = lib()
    kk = np.ascontiguousarray(kk, np.float32)
    nx, ny = kk.shape
    sai = np.asfortranarray(sai, np.float64)
    sei = np.ascontiguousarray(sei, np.float64)
    dd = np.zeros((nx, ny), order="F")
    aa = np.zeros((nx, nx), order="F")
    dp = C.POINTER(C.c_double)
    L.orc_calc_gain_matrix_diag(nx, ny, nx, ny, _abi.fptr(kk), sai.ctypes.data_as(dp), sei.ctypes.data_as(dp),
                                dd.ctypes.data_as(dp), aa.ctypes.data_as(dp), None)
    return dd, aa


def calcnextxn(xa, xn, y, yn, dd, aa):
    L = lib()
    dp = C.POINTER(C.c_double)
    dd = np.asfortranarray(dd, np.float64)
    aa = np.asfortranarray(aa, np.float64)
    nx, ny = dd.shape
    xa, xn, y, yn = (np.ascontiguousarray(a, np.float32) for a in (xa, xn, y, yn))
    x_out = np.zeros(nx, np.float32)
    L.orc_calcnextxn(nx, ny, nx, _abi.fptr(xa), _abi.fptr(xn), _abi.fptr(y), _abi.fptr(yn),
                     dd.ctypes.data_as(dp), aa.ctypes.data_as(dp), _abi.fptr(x_out))
    return x_out


def newton_step(kk, sei, sai, xa, xn, y, yn):
    """calc_gain_matrix (diagonal Se, dense D and AA) + calcnextxn for one
    retrieval: kk [nx, ny] (Fortran kk(ny, nx)), sei [ny], sai [nx, nx]."""
    L = lib()
    kk = np.ascontiguousarray(kk, np.float32)
    nx, ny = kk.shape
    sai = np.asfortranarray(sai, np.float64)
    sei = np.ascontiguousarray(sei, np.float64)
    dd = np.zeros((nx, ny), order="F")
    aa = np.zeros((nx, nx), order="F")
    dp = C.POINTER(C.c_double)
    L.orc_calc_gain_matrix_diag(nx, ny, nx, ny, _abi.fptr(kk), sai.ctypes.data_as(dp), sei.ctypes.data_as(dp),
                                dd.ctypes.data_as(dp), aa.ctypes.data_as(dp), None)
    x_out = np.zeros(nx, np.float32)
    f = lambda a: _abi.fptr(np.ascontiguousarray(a, np.float32))
    xa, xn, y, yn = (np.ascontiguousarray(a, np.float32) for a in (xa, xn, y, yn))
    L.orc_calcnextxn(nx, ny, nx, f(xa), f(xn), f(y), f(yn), dd.ctypes.data_as(dp), aa.ctypes.data_as(dp),
                     _abi.fptr(x_out))
    return x_out


def calc_phiret(y, yn, sei, xn, xa, sai):
    L = lib()
    dp = C.POINTER(C.c_double)
    y, yn, xn, xa = (np.ascontiguousarray(a, np.float32) for a in (y, yn, xn, xa))
    sei = np.ascontiguousarray(sei, np.float64)
    sai = np.asfortranarray(sai, np.float64)
    chisq = C.c_float(0.0)
    phi = L.orc_calc_phiret_diag(len(y), _abi.fptr(y), _abi.fptr(yn), sei.ctypes.data_as(dp), len(xn), len(xn),
                                 _abi.fptr(xn), _abi.fptr(xa), sai.ctypes.data_as(dp), C.byref(chisq))
    return np.float32(phi), np.float32(chisq.value)


def dinvertm(a):
    L = lib()
    dp = C.POINTER(C.c_double)
    a = np.asfortranarray(a, np.float64)
    out = np.zeros_like(a, order="F")
    ic = L.orc_dinvertm_chol(a.shape[0], a.shape[0], a.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return out, ic


def calc_serr(sx, se_diag, dd, aa):
    """calc_serr (diagonal Se): returns (st, sn, sm) [nx, nx] float32 (Fortran order)."""
    L = lib()
    dp = C.POINTER(C.c_double)
    dd = np.asfortranarray(dd, np.float64)
    aa = np.asfortranarray(aa, np.float64)
    nx, ny = dd.shape
    sx = np.asfortranarray(sx, np.float32)
    se = np.ascontiguousarray(se_diag, np.float32)
    out = [np.zeros((nx, nx), np.float32, order="F") for _ in range(3)]
    L.orc_calc_serr_diag(nx, ny, nx, _abi.fptr(sx), _abi.fptr(se), dd.ctypes.data_as(dp), aa.ctypes.data_as(dp),
                         _abi.fptr(out[0]), _abi.fptr(out[1]), _abi.fptr(out[2]))
    return tuple(out)


def layerg(prof, **opts):
    """The oracle's LAYERG + nadir ATMG path, same arguments and outputs as
    Context.layerg."""
    from radtrancode_b200.cirsradg import layer_call
    L = lib()
    st, out = layer_call(lambda p, o, r: L.orc_layerg(p, o, r), prof, **opts)
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    return out


def cirsconv_ex(vwave, y, fwhm, channels):
    """cirsconv.f:12-246 of one series onto ``channels`` (synth.Channels)."""
    L = lib()
    vwave = np.ascontiguousarray(vwave, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    ch = channels
    yout = np.zeros(len(ch.vconv), np.float32)
    nf = 0 if ch.vfwhm is None else len(ch.vfwhm)
    nfil = 0 if ch.vcen is None else len(ch.vcen)
    st = L.orc_cirsconv_ex(C.c_float(fwhm), len(vwave), _abi.fptr(vwave), _abi.fptr(y), len(ch.vconv),
                           _abi.fptr(ch.vconv), nf, _abi.fptr(ch.vfwhm), _abi.fptr(ch.xfwhm), nfil,
                           _abi.fptr(ch.vcen), _abi.iptr(ch.nsub), _abi.fptr(ch.vfil), _abi.fptr(ch.fil),
                           _abi.fptr(yout))
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    return yout


def cirsconv(vwave, y, fwhm, vconv):
    L = lib()
    vwave = np.ascontiguousarray(vwave, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    vconv = np.ascontiguousarray(vconv, np.float32)
    yout = np.zeros(len(vconv), np.float32)
    st = L.orc_cirsconv(len(vwave), _abi.fptr(vwave), _abi.fptr(y), C.c_float(fwhm), len(vconv), _abi.fptr(vconv),
                        _abi.fptr(yout))
    if st != 0:
        raise RuntimeError(f"oracle status {_abi.STATUS_NAMES.get(st, st)}")
    return yout

