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
    ]


class OrcDebug(C.Structure):
    _fields_ = [("perm", C.POINTER(C.c_int16)), ("split", C.POINTER(C.c_int16)),
                ("ties", C.POINTER(C.c_int16))]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


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


def tables_struct(kt, cia=None):
    t = OrcTables()
    t.ntab, t.np, t.nt, t.ng = kt.ntab, kt.np_, kt.nt, kt.ng
    t.lnp, t.tk, t.delg = _abi.fptr(kt.lnp), _abi.fptr(kt.tk), _abi.fptr(kt.delg)
    t.vmin, t.delv, t.nbin = _abi.fptr(kt.vmin), _abi.fptr(kt.delv), _abi.iptr(kt.nbin)
    t.data = _abi.fptr(kt.data)
    if cia is not None:
        t.has_cia, t.dnu = 1, cia.dnu
        t.cia_temps = _abi.dptr(cia.temps)
        t.kcia = _abi.fptr(cia.kcia)
    t._keep = (kt, cia)
    return t


def cirsrtfg_wave(kt, cia, job, precision=ORC_MIXED, debug=False, nthreads=1):
    """Run the oracle forward model.  Returns (calcout, gradients, gradtsurf)
    as float64 arrays, plus (perm, split) debug arrays when requested."""
    L = lib()
    t = tables_struct(kt, cia)
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
        st = L.orc_cirsrtfg_wave_mt(C.byref(t), C.byref(s), precision, dp[0], dp[1], dp[2], nthreads)
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
