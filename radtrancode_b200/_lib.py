"""Loader of the in-tree shared library libradtran_b200.so.

The library is the product: a missing or unloadable library is an error,
never a reason to fall back to another implementation.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libradtran_b200.so")
CSRC = os.path.join(HERE, "csrc")

_lib = None


def build(force: bool = False) -> str:
    """Compile the CUDA sources for sm_100a into the package directory."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", CSRC], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run radtrancode_b200._lib.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        dp = C.POINTER(C.c_double)
        L.rtb_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.rtb_create.restype = C.c_int
        L.rtb_destroy.argtypes = [vp]
        L.rtb_destroy.restype = None
        L.rtb_last_error.argtypes = [vp]
        L.rtb_last_error.restype = C.c_char_p
        L.rtb_version.restype = C.c_char_p
        L.rtb_set_ktables.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, fp, fp, fp, fp, fp, ip, fp]
        L.rtb_set_ktables.restype = C.c_int
        L.rtb_set_cia.argtypes = [vp, C.c_float, dp, fp]
        L.rtb_set_cia.restype = C.c_int
        L.rtb_cirsrtfg_wave.argtypes = [vp, C.POINTER(_abi.RtbAtm), fp, fp, fp]
        L.rtb_cirsrtfg_wave.restype = C.c_int
        L.rtb_cirsrtfg_wave_batch.argtypes = [vp, C.c_int, C.POINTER(_abi.RtbAtm), C.POINTER(fp), C.POINTER(fp),
                                              C.POINTER(fp)]
        L.rtb_cirsrtfg_wave_batch.restype = C.c_int
        L.rtb_get_fwd_stats.argtypes = [vp, C.POINTER(_abi.RtbFwdStats)]
        L.rtb_get_fwd_stats.restype = C.c_int
        L.rtb_set_debug.argtypes = [vp, C.c_int]
        L.rtb_set_debug.restype = C.c_int
        L.rtb_set_strict_ties.argtypes = [vp, C.c_int]
        L.rtb_set_strict_ties.restype = C.c_int
        L.rtb_fwd_prepare.argtypes = [vp, C.c_int, C.POINTER(_abi.RtbAtm)]
        L.rtb_fwd_prepare.restype = C.c_int
        L.rtb_fwd_launch.argtypes = [vp]
        L.rtb_fwd_launch.restype = C.c_int
        L.rtb_fwd_fetch.argtypes = [vp, C.POINTER(fp), C.POINTER(fp), C.POINTER(fp)]
        L.rtb_fwd_fetch.restype = C.c_int
        L.rtb_set_stream.argtypes = [vp, vp]
        L.rtb_set_stream.restype = C.c_int
        L.rtb_fwd_launch_static.argtypes = [vp]
        L.rtb_fwd_launch_static.restype = C.c_int
        L.rtb_set_newton_mode.argtypes = [vp, C.c_int, C.c_int]
        L.rtb_set_newton_mode.restype = C.c_int
        L.rtb_newton_step_batch.argtypes = [vp, C.c_int, C.c_int, C.c_int, fp, dp, dp, fp, fp, fp, fp, fp, ip, dp]
        L.rtb_newton_step_batch.restype = C.c_int
        L.rtb_calc_phiret_batch.argtypes = [vp, C.c_int, C.c_int, C.c_int, fp, fp, dp, fp, fp, dp, fp, fp]
        L.rtb_calc_phiret_batch.restype = C.c_int
        L.rtb_spd_inverse_batch.argtypes = [vp, C.c_int, C.c_int, dp, dp, ip]
        L.rtb_spd_inverse_batch.restype = C.c_int
        L.rtb_retrieve_batch.argtypes = [vp, C.c_int, C.POINTER(_abi.RtbRetrievalSpec),
                                         C.POINTER(_abi.RtbRetrievalOpts), C.POINTER(_abi.RtbRetrievalResult)]
        L.rtb_retrieve_batch.restype = C.c_int
        L.rtb_get_newton_stats.argtypes = [vp, C.POINTER(_abi.RtbNewtonStats)]
        L.rtb_get_newton_stats.restype = C.c_int
        L.rtb_fwd_set_schedule.argtypes = [vp, C.c_int, C.c_int]
        L.rtb_fwd_set_schedule.restype = C.c_int
        L.rtb_fwd_set_tile.argtypes = [vp, C.c_int]
        L.rtb_fwd_set_tile.restype = C.c_int
        L.rtb_fwd_autotune.argtypes = [vp, C.POINTER(_abi.RtbFwdTune)]
        L.rtb_fwd_autotune.restype = C.c_int
        L.rtb_fwd_use_graph.argtypes = [vp, C.c_int]
        L.rtb_fwd_use_graph.restype = C.c_int
        L.rtb_server_create.argtypes = [vp, C.c_size_t, C.POINTER(_abi.RtbRetrievalOpts), C.POINTER(vp)]
        L.rtb_server_create.restype = C.c_int
        L.rtb_server_destroy.argtypes = [vp]
        L.rtb_server_destroy.restype = None
        L.rtb_server_submit.argtypes = [vp, C.POINTER(_abi.RtbRetrievalSpec), C.POINTER(C.c_longlong)]
        L.rtb_server_submit.restype = C.c_int
        L.rtb_server_step.argtypes = [vp, ip, ip]
        L.rtb_server_step.restype = C.c_int
        L.rtb_server_poll.argtypes = [vp, C.c_longlong, ip, C.POINTER(_abi.RtbRetrievalResult)]
        L.rtb_server_poll.restype = C.c_int
        L.rtb_calc_gain_matrix.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, fp, dp, dp, dp, dp, ip]
        L.rtb_calc_gain_matrix.restype = C.c_int
        L.rtb_calcnextxn.argtypes = [vp, C.c_int, C.c_int, C.c_int, fp, fp, fp, fp, dp, dp, fp]
        L.rtb_calcnextxn.restype = C.c_int
        L.rtb_cirsradg_wave.argtypes = [vp, C.POINTER(_abi.RtbAtm), C.c_int, ip, fp, fp, fp, C.c_int, C.c_int,
                                        C.c_int]
        L.rtb_cirsradg_wave.restype = C.c_int
        L.rtb_calc_serr.argtypes = [vp, C.c_int, C.c_int, C.c_int, fp, fp, dp, dp, fp, fp, fp]
        L.rtb_calc_serr.restype = C.c_int
        L.rtb_cirsconv.argtypes = [vp, C.c_int, fp, C.c_int, fp, C.c_float, C.c_int, fp, fp]
        L.rtb_cirsconv.restype = C.c_int
        L.rtb_cirsconv_ex.argtypes = [vp, C.c_float, C.c_int, fp, C.c_int, fp, C.POINTER(_abi.RtbConv), fp]
        L.rtb_cirsconv_ex.restype = C.c_int
        L.rtb_read_fwh.argtypes = [C.c_char_p, ip, fp, fp, C.c_int]
        L.rtb_read_fwh.restype = C.c_int
        L.rtb_read_fil.argtypes = [C.c_char_p, ip, ip, fp, ip, fp, fp, C.c_int, C.c_int]
        L.rtb_read_fil.restype = C.c_int
        L.rtb_set_para_cia.argtypes = [vp, C.c_float, C.c_int, fp, fp, fp, fp, fp]
        L.rtb_set_para_cia.restype = C.c_int
        L.rtb_load_para_cia.argtypes = [vp, C.c_char_p, C.c_float, C.c_int]
        L.rtb_load_para_cia.restype = C.c_int
        L.rtb_set_e3_table.argtypes = [vp, C.c_int, dp, dp]
        L.rtb_set_e3_table.restype = C.c_int
        L.rtb_load_e3_table.argtypes = [vp, C.c_char_p]
        L.rtb_load_e3_table.restype = C.c_int
        L.rtb_set_stellar_spectrum.argtypes = [vp, C.c_int, fp, fp]
        L.rtb_set_stellar_spectrum.restype = C.c_int
        L.rtb_load_stellar_spectrum.argtypes = [vp, C.c_char_p, C.c_int]
        L.rtb_load_stellar_spectrum.restype = C.c_int
        L.rtb_set_ktable_ids.argtypes = [vp, C.c_int, ip, ip]
        L.rtb_set_ktable_ids.restype = C.c_int
        L.rtb_set_ktable_centres.argtypes = [vp, C.c_int, fp]
        L.rtb_set_ktable_centres.restype = C.c_int
        L.rtb_layerg.argtypes = [vp, C.POINTER(_abi.RtbProfile), C.POINTER(_abi.RtbLayerOpts),
                                 C.POINTER(_abi.RtbLayers)]
        L.rtb_layerg.restype = C.c_int
        L.rtb_kta_header.argtypes = [C.c_char_p, ip, ip, ip, ip, fp, fp, ip, ip]
        L.rtb_kta_header.restype = C.c_int
        L.rtb_load_ktables.argtypes = [vp, C.c_int, C.POINTER(C.c_char_p), ip, ip]
        L.rtb_load_ktables.restype = C.c_int
        L.rtb_load_cia.argtypes = [vp, C.c_char_p, C.c_float]
        L.rtb_load_cia.restype = C.c_int
        p16 = C.POINTER(C.c_int16)
        L.rtb_get_debug_bins.argtypes = [vp, p16, C.c_size_t, p16, C.c_size_t]
        L.rtb_get_debug_bins.restype = C.c_int
        _lib = L
    return _lib


# every symbol include/radtran_b200.h declares
EXPORTED = [
    "rtb_create", "rtb_destroy", "rtb_last_error", "rtb_version", "rtb_set_ktables", "rtb_set_cia",
    "rtb_cirsrtfg_wave", "rtb_cirsrtfg_wave_batch", "rtb_get_fwd_stats", "rtb_set_debug",
    "rtb_get_debug_bins", "rtb_set_strict_ties", "rtb_fwd_prepare", "rtb_fwd_launch", "rtb_fwd_fetch",
    "rtb_set_stream", "rtb_fwd_launch_static", "rtb_set_newton_mode", "rtb_newton_step_batch",
    "rtb_calc_phiret_batch", "rtb_spd_inverse_batch", "rtb_retrieve_batch", "rtb_get_newton_stats",
    "rtb_fwd_set_schedule", "rtb_fwd_set_tile", "rtb_fwd_autotune", "rtb_fwd_use_graph", "rtb_server_create", "rtb_server_destroy",
    "rtb_server_submit", "rtb_server_step", "rtb_server_poll", "rtb_calc_gain_matrix", "rtb_calcnextxn",
    "rtb_cirsradg_wave", "rtb_kta_header", "rtb_load_ktables", "rtb_load_cia",
    "rtb_calc_serr", "rtb_cirsconv", "rtb_cirsconv_ex", "rtb_read_fwh", "rtb_read_fil",
    "rtb_layerg", "rtb_set_ktable_centres", "rtb_set_ktable_ids",
    "rtb_set_para_cia", "rtb_load_para_cia", "rtb_set_e3_table", "rtb_load_e3_table",
    "rtb_set_stellar_spectrum", "rtb_load_stellar_spectrum",
]
