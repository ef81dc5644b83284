"""Python face of the B200 CIRSRADG forward model (C ABI in
include/radtran_b200.h).

``Context`` mirrors the reference's call sequence: ``read_klist`` (k-table
residency) -> ``ciaread`` (CIA table) -> ``cirsrtfg_wave`` (all wavenumbers
of one forward + Jacobian call, radtran/cirsradg/cirsrtfg_wave.f:1-3), with
the same argument meaning and output packing.  Errors are raised as
``RtbError`` carrying the status code and the library's message, where the
reference would STOP.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi, _lib


class RtbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _file_status(st, path):
    if st != _abi.RTB_OK:
        raise RtbError(st, f"cannot read {path}")


def read_fwh(path):
    """A .fwh file (cirsrtfg_wave.f:191-196): (vfwhm, xfwhm)."""
    L = _lib.lib()
    n = C.c_int(0)
    _file_status(L.rtb_read_fwh(os.fsencode(path), C.byref(n), None, None, 0), path)
    v, x = np.zeros(n.value, np.float32), np.zeros(n.value, np.float32)
    _file_status(L.rtb_read_fwh(os.fsencode(path), C.byref(n), _abi.fptr(v), _abi.fptr(x), len(v)), path)
    return v, x


def read_fil(path):
    """A .fil file (cirsconv.f:185-196): (vcen, nsub, vfil, fil)."""
    L = _lib.lib()
    nf, npt = C.c_int(0), C.c_int(0)
    _file_status(L.rtb_read_fil(os.fsencode(path), C.byref(nf), C.byref(npt), None, None, None, None, 0, 0), path)
    vc, ns = np.zeros(nf.value, np.float32), np.zeros(nf.value, np.int32)
    vf, fl = np.zeros(npt.value, np.float32), np.zeros(npt.value, np.float32)
    _file_status(L.rtb_read_fil(os.fsencode(path), C.byref(nf), C.byref(npt), _abi.fptr(vc), _abi.iptr(ns),
                                _abi.fptr(vf), _abi.fptr(fl), len(vc), len(vf)), path)
    return vc, ns, vf, fl


def layer_call(fn, prof, *, nlay, laytyp=1, layint=1, layht=None, layang=0.0, base=None, angle=0.0, botlay=1,
               ipzen=0):
    """Run a layering function with the rtb_layerg arguments (``fn(prof_struct,
    opts_struct, out_struct) -> status``) and return its outputs as arrays."""
    o = _abi.RtbLayerOpts()
    o.nlay, o.laytyp, o.layint = nlay, laytyp, layint
    o.layht = float(prof.h[0] if layht is None else layht)
    o.layang = float(layang)
    b = None if base is None else np.ascontiguousarray(base, np.float32)
    o.base = _abi.fptr(b)
    o.angle, o.botlay, o.ipzen = float(angle), botlay, ipzen
    npro, nvmr = prof.npro, prof.vmr.shape[1]
    out = {k: np.zeros(nlay, np.float32) for k in ("baseh", "delh", "basep", "baset", "press", "temp", "totam",
                                                   "laysf", "scale", "emtemp")}
    out["layinc"] = np.zeros(nlay, np.int32)
    for k, n in (("amount", nvmr), ("pp", nvmr), ("dte", npro), ("dam", npro), ("dco", npro)):
        out[k] = np.zeros((nlay, n), np.float32, order="F")
    ints = {k: np.zeros(1, np.int32) for k in ("npath", "nlayin", "imod")}
    r = _abi.RtbLayers()
    r.ld_lay, r.ld_con = nlay, 0
    for k, v in out.items():
        setattr(r, k, _abi.iptr(v) if v.dtype == np.int32 else _abi.fptr(v))
    for k, v in ints.items():
        setattr(r, k, _abi.iptr(v))
    ps = prof.as_struct()
    st = fn(C.byref(ps), C.byref(o), C.byref(r))
    out.update({k: int(v[0]) for k, v in ints.items()})
    out["nlay"] = nlay
    return st, out


class Context:
    """One device context (one CUDA device, one host thread at a time)."""

    def __init__(self, device: int = 0):
        self._L = _lib.lib()
        h = C.c_void_p()
        st = self._L.rtb_create(device, C.byref(h))
        if st != 0:
            raise RtbError(st, f"rtb_create(device={device}) failed: no usable CUDA device")
        self._h = h
        self.device = device
        self.tables = None

    def close(self):
        if getattr(self, "_h", None):
            self._L.rtb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != 0:
            raise RtbError(st, self._L.rtb_last_error(self._h).decode())

    # -- resident tables --------------------------------------------------
    def set_ktables(self, kt):
        """read_klist equivalent: upload the run's k-tables once."""
        self._check(self._L.rtb_set_ktables(
            self._h, kt.ntab, kt.np_, kt.nt, kt.ng, _abi.fptr(kt.lnp), _abi.fptr(kt.tk), _abi.fptr(kt.delg),
            _abi.fptr(kt.vmin), _abi.fptr(kt.delv), _abi.iptr(kt.nbin), _abi.fptr(kt.data)))
        ids = np.array([g[0] for g in kt.gases], np.int32)
        isos = np.array([g[1] for g in kt.gases], np.int32)
        self._check(self._L.rtb_set_ktable_ids(self._h, kt.ntab, _abi.iptr(ids), _abi.iptr(isos)))
        if kt.vcen is not None:     # irregular grid: the first table's centres
            self._check(self._L.rtb_set_ktable_centres(self._h, len(kt.vcen), _abi.fptr(kt.vcen)))
        self.tables = kt

    def load_ktables(self, paths):
        """read_klist equivalent from .kta files; returns [(idgas, isogas)]."""
        n = len(paths)
        arr = (C.c_char_p * n)(*[os.fsencode(p) for p in paths])
        ids = np.zeros(n, np.int32)
        isos = np.zeros(n, np.int32)
        self._check(self._L.rtb_load_ktables(self._h, n, arr, _abi.iptr(ids), _abi.iptr(isos)))
        return list(zip(ids.tolist(), isos.tolist()))

    def load_cia(self, path, dnu=1.0):
        """ciaread equivalent from a CIA .tab file."""
        self._check(self._L.rtb_load_cia(self._h, os.fsencode(path), float(dnu)))

    def set_para_cia(self, para):
        """fpread_all's one-time table read (a synth.ParaCIATable)."""
        self._check(self._L.rtb_set_para_cia(self._h, float(para.dnu2), int(para.ipara), _abi.fptr(para.temps),
                                             _abi.fptr(para.fp), _abi.fptr(para.kh2h2), _abi.fptr(para.kh2he),
                                             _abi.fptr(para.kcia5)))

    def load_para_cia(self, path, dnu2=1.0, ipara=24):
        """fpread_all equivalent from the table file."""
        self._check(self._L.rtb_load_para_cia(self._h, os.fsencode(path), float(dnu2), int(ipara)))

    def set_e3_table(self, e3):
        """e3interp's one-time table read (a synth.E3Table: 1001 transmissions
        and E3 values), needed by IMOD 18 paths."""
        self._check(self._L.rtb_set_e3_table(self._h, len(e3.tran), _abi.dptr(e3.tran), _abi.dptr(e3.e3)))

    def load_e3_table(self, path):
        """e3interp's read of the e3tab.dat text file."""
        self._check(self._L.rtb_load_e3_table(self._h, os.fsencode(path)))

    def set_stellar_spectrum(self, ss):
        """init_solar_wave's table (a synth.StellarSpectrum), used by iform 1
        and 4."""
        self._check(self._L.rtb_set_stellar_spectrum(self._h, len(ss.wave), _abi.fptr(ss.wave), _abi.fptr(ss.rad)))

    def load_stellar_spectrum(self, path, ispace=0):
        """init_solar_wave's read of the stellar spectrum file."""
        self._check(self._L.rtb_load_stellar_spectrum(self._h, os.fsencode(path), int(ispace)))

    def set_cia(self, cia):
        """ciaread's one-time table read."""
        self._check(self._L.rtb_set_cia(self._h, float(cia.dnu), _abi.dptr(cia.temps), _abi.fptr(cia.kcia)))

    def set_strict_ties(self, on: bool):
        self._check(self._L.rtb_set_strict_ties(self._h, int(bool(on))))

    def set_debug(self, on: bool):
        self._check(self._L.rtb_set_debug(self._h, int(bool(on))))

    # -- forward model ------------------------------------------------------
    def cirsrtfg_wave(self, job):
        """Forward model + Jacobian of one job.  Returns (calcout, gradients,
        gradtsurf) as float32 arrays packed as cirsrtfg_wave.f:425-446."""
        n1, n2, n3 = job.out_shapes()
        calcout = np.zeros(n1, np.float32)
        grads = np.zeros(n2, np.float32)
        gts = np.zeros(n3, np.float32)
        s = job.as_struct()
        self._check(self._L.rtb_cirsrtfg_wave(self._h, C.byref(s), _abi.fptr(calcout), _abi.fptr(grads),
                                              _abi.fptr(gts)))
        return calcout, grads, gts

    def cirsconv(self, vwave, y, fwhm, vconv):
        """cirsconv of series y [nser, nwave] to channels vconv: [nser, nconv]."""
        vwave = np.ascontiguousarray(vwave, np.float32)
        vconv = np.ascontiguousarray(vconv, np.float32)
        y = np.ascontiguousarray(np.atleast_2d(y), np.float32)
        out = np.zeros((y.shape[0], len(vconv)), np.float32)
        self._check(self._L.rtb_cirsconv(self._h, len(vwave), _abi.fptr(vwave), y.shape[0], _abi.fptr(y),
                                         float(fwhm), len(vconv), _abi.fptr(vconv), _abi.fptr(out)))
        return out

    def cirsconv_ex(self, vwave, y, fwhm, channels):
        """cirsconv of series y [nser, nwave] with any FWHM (> 0 with an
        optional width table, 0, < 0 with filter functions) onto
        ``channels`` (a ``synth.Channels``): [nser, nconv]."""
        vwave = np.ascontiguousarray(vwave, np.float32)
        y = np.ascontiguousarray(np.atleast_2d(y), np.float32)
        cs = channels.as_struct()
        out = np.zeros((y.shape[0], len(channels.vconv)), np.float32)
        self._check(self._L.rtb_cirsconv_ex(self._h, float(fwhm), len(vwave), _abi.fptr(vwave), y.shape[0],
                                            _abi.fptr(y), C.byref(cs), _abi.fptr(out)))
        return out

    def layerg(self, prof, **opts):
        """LAYERG + the nadir path of ATMG on the device (rtb_layerg): the
        layers, gradient matrices and path of a ``synth.Profile``."""
        st, out = layer_call(lambda p, o, r: self._L.rtb_layerg(self._h, p, o, r), prof, **opts)
        self._check(st)
        return out

    def cirsradg_wave(self, job, isw):
        """rtb_cirsradg_wave on a one-wavenumber job: (output [npath],
        gtsurf [npath], doutputdq [npath, nlayer, nparam])."""
        assert job.nwave == 1
        isw = np.ascontiguousarray(isw, np.int32)
        npath, nparam = job.npath, job.nparam
        out = np.zeros(npath, np.float32)
        gts = np.zeros(npath, np.float32)
        dq = np.zeros((npath, job.nlayer, nparam), np.float32, order="F")
        s = job.as_struct()
        self._check(self._L.rtb_cirsradg_wave(self._h, C.byref(s), len(isw), _abi.iptr(isw), _abi.fptr(out),
                                              _abi.fptr(gts), _abi.fptr(dq), npath, job.nlayer, nparam))
        return out, gts, dq

    def cirsrtfg_wave_batch(self, jobs, outs=None):
        """Batched forward model: one launch for all jobs.  Returns a list of
        (calcout, gradients, gradtsurf)."""
        n = len(jobs)
        structs = (_abi.RtbAtm * n)()
        keep = []
        if outs is None:
            outs = []
            for j in jobs:
                a, b, c = j.out_shapes()
                outs.append((np.zeros(a, np.float32), np.zeros(b, np.float32), np.zeros(c, np.float32)))
        fp = C.POINTER(C.c_float)
        p1, p2, p3 = (fp * n)(), (fp * n)(), (fp * n)()
        for i, j in enumerate(jobs):
            s = j.as_struct()
            keep.append(s)
            structs[i] = s
            p1[i], p2[i], p3[i] = _abi.fptr(outs[i][0]), _abi.fptr(outs[i][1]), _abi.fptr(outs[i][2])
        self._check(self._L.rtb_cirsrtfg_wave_batch(self._h, n, structs, p1, p2, p3))
        return outs

    # -- resident batch: prepare once, launch many times ------------------
    def prepare(self, jobs):
        n = len(jobs)
        structs = (_abi.RtbAtm * n)()
        self._prepared_keep = []
        for i, j in enumerate(jobs):
            s = j.as_struct()
            self._prepared_keep.append(s)
            structs[i] = s
        self._check(self._L.rtb_fwd_prepare(self._h, n, structs))
        self._prepared_jobs = list(jobs)

    def launch(self):
        self._check(self._L.rtb_fwd_launch(self._h))

    def set_schedule(self, schedule, blocks_per_sm=0):
        self._check(self._L.rtb_fwd_set_schedule(self._h, schedule, blocks_per_sm))

    def set_tile(self, warps=0):
        """Warps per block of the resident batch's launches (2, 4, 8; 0 = the default 8)."""
        self._check(self._L.rtb_fwd_set_tile(self._h, warps))

    def autotune(self) -> dict:
        t = _abi.RtbFwdTune()
        self._check(self._L.rtb_fwd_autotune(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def use_graph(self, on=True):
        self._check(self._L.rtb_fwd_use_graph(self._h, 1 if on else 0))

    def launch_static(self):
        """rtb_fwd_launch_static: the same launch with its scratch taken from
        the library's fixed per-device array, allocating nothing."""
        self._check(self._L.rtb_fwd_launch_static(self._h))

    def fetch(self):
        jobs = self._prepared_jobs
        n = len(jobs)
        outs = []
        fp = C.POINTER(C.c_float)
        p1, p2, p3 = (fp * n)(), (fp * n)(), (fp * n)()
        for i, j in enumerate(jobs):
            a, b, c = j.out_shapes()
            o = (np.zeros(a, np.float32), np.zeros(b, np.float32), np.zeros(c, np.float32))
            outs.append(o)
            p1[i], p2[i], p3[i] = _abi.fptr(o[0]), _abi.fptr(o[1]), _abi.fptr(o[2])
        self._check(self._L.rtb_fwd_fetch(self._h, p1, p2, p3))
        return outs

    # -- optimal-estimation Newton step and retrieval ----------------------
    def set_newton_mode(self, hessian=0, refine=1):
        """hessian 0: K^T Se^-1 K on tensor cores + `refine` refinement
        steps; 1: all FP64."""
        self._check(self._L.rtb_set_newton_mode(self._h, hessian, refine))

    def newton_step_batch(self, kk, sei, sai, xa, xn, y, yn):
        """calc_gain_matrix + calcnextxn for a batch: kk [nret, nx, ny],
        sei [nret, ny], sai [nret, nx, nx], xa/xn [nret, nx], y/yn [nret, ny].
        Returns (x_out [nret, nx], nonpd [nret], resid [nret])."""
        kk = np.ascontiguousarray(kk, np.float32)
        nret, nx, ny = kk.shape
        f32 = lambda a: np.ascontiguousarray(a, np.float32)
        f64 = lambda a: np.ascontiguousarray(a, np.float64)
        sei, sai, xa, xn, y, yn = f64(sei), f64(sai), f32(xa), f32(xn), f32(y), f32(yn)
        x_out = np.zeros((nret, nx), np.float32)
        nonpd = np.zeros(nret, np.int32)
        resid = np.zeros(nret, np.float64)
        self._check(self._L.rtb_newton_step_batch(
            self._h, nret, nx, ny, _abi.fptr(kk), _abi.dptr(sei), _abi.dptr(sai), _abi.fptr(xa), _abi.fptr(xn),
            _abi.fptr(y), _abi.fptr(yn), _abi.fptr(x_out), _abi.iptr(nonpd), _abi.dptr(resid)))
        return x_out, nonpd, resid

    def newton_stats(self) -> dict:
        s = _abi.RtbNewtonStats()
        self._check(self._L.rtb_get_newton_stats(self._h, C.byref(s)))
        return {"retrievals": s.retrievals, "ms_kernel": s.ms_kernel}

    def calc_gain_matrix(self, kk, sxi, sei):
        """calc_gain_matrix for one retrieval: kk [nx, ny] (Fortran kk(ny, nx)),
        sxi [nx, nx] (Sa^-1), sei [ny] (diagonal of Se^-1).  Returns
        (dd [nx, ny], aa [nx, nx], nonpd)."""
        kk = np.ascontiguousarray(kk, np.float32)
        nx, ny = kk.shape
        sxi = np.asfortranarray(sxi, np.float64)
        sei = np.ascontiguousarray(sei, np.float64)
        dd = np.zeros((nx, ny), np.float64, order="F")
        aa = np.zeros((nx, nx), np.float64, order="F")
        nonpd = C.c_int()
        self._check(self._L.rtb_calc_gain_matrix(self._h, nx, ny, nx, ny, _abi.fptr(kk), _abi.dptr(sxi),
                                                 _abi.dptr(sei), _abi.dptr(dd), _abi.dptr(aa), C.byref(nonpd)))
        return dd, aa, nonpd.value

    def calc_serr(self, sx, se_diag, dd, aa):
        """calc_serr: (st, sn, sm) [nx, nx] float32 from Sa, diag(Se), D, AA."""
        dd = np.asfortranarray(dd, np.float64)
        aa = np.asfortranarray(aa, np.float64)
        nx, ny = dd.shape
        sx = np.asfortranarray(sx, np.float32)
        se = np.ascontiguousarray(se_diag, np.float32)
        out = [np.zeros((nx, nx), np.float32, order="F") for _ in range(3)]
        self._check(self._L.rtb_calc_serr(self._h, nx, ny, nx, _abi.fptr(sx), _abi.fptr(se), _abi.dptr(dd),
                                          _abi.dptr(aa), _abi.fptr(out[0]), _abi.fptr(out[1]), _abi.fptr(out[2])))
        return tuple(out)

    def calcnextxn(self, x0, xn, y, yn, dd, aa):
        f32 = lambda a: np.ascontiguousarray(a, np.float32)
        x0, xn, y, yn = f32(x0), f32(xn), f32(y), f32(yn)
        dd = np.asfortranarray(dd, np.float64)
        aa = np.asfortranarray(aa, np.float64)
        nx, ny = dd.shape
        x_out = np.zeros(nx, np.float32)
        self._check(self._L.rtb_calcnextxn(self._h, nx, ny, nx, _abi.fptr(x0), _abi.fptr(xn), _abi.fptr(y),
                                           _abi.fptr(yn), _abi.dptr(dd), _abi.dptr(aa), _abi.fptr(x_out)))
        return x_out

    def calc_phiret_batch(self, y, yn, sei, xn, xa, sai):
        f32 = lambda a: np.ascontiguousarray(a, np.float32)
        f64 = lambda a: np.ascontiguousarray(a, np.float64)
        y, yn, sei, xn, xa, sai = f32(y), f32(yn), f64(sei), f32(xn), f32(xa), f64(sai)
        nret, ny = y.shape
        nx = xn.shape[1]
        phi = np.zeros(nret, np.float32)
        chisq = np.zeros(nret, np.float32)
        self._check(self._L.rtb_calc_phiret_batch(
            self._h, nret, nx, ny, _abi.fptr(y), _abi.fptr(yn), _abi.dptr(sei), _abi.fptr(xn), _abi.fptr(xa),
            _abi.dptr(sai), _abi.fptr(phi), _abi.fptr(chisq)))
        return phi, chisq

    def spd_inverse_batch(self, a):
        a = np.ascontiguousarray(a, np.float64)
        nret, n, _ = a.shape
        out = np.zeros_like(a)
        nonpd = np.zeros(nret, np.int32)
        self._check(self._L.rtb_spd_inverse_batch(self._h, nret, n, _abi.dptr(a), _abi.dptr(out),
                                                  _abi.iptr(nonpd)))
        return out, nonpd

    def retrieve_batch(self, cases, kiter=10, phlimit=0.1, dchisq_stop=0.0, max_batch=0):
        """rtb_retrieve_batch on synth.RetrievalCase objects; one result
        dict per case (x, yn, phi, chisq, alambda, iterations, forwards,
        converged, nonpd, ms)."""
        n = len(cases)
        specs = (_abi.RtbRetrievalSpec * n)()
        res = (_abi.RtbRetrievalResult * n)()
        keep, outs = [], []
        for i, c in enumerate(cases):
            s = c.as_struct()
            keep.append(s)
            specs[i] = s
            x = np.zeros(c.nx, np.float32)
            yn = np.zeros(c.ny, np.float32)
            outs.append((x, yn))
            res[i].x, res[i].yn = _abi.fptr(x), _abi.fptr(yn)
        o = _abi.RtbRetrievalOpts(kiter, phlimit, dchisq_stop, max_batch)
        self._check(self._L.rtb_retrieve_batch(self._h, n, specs, C.byref(o), res))
        out = []
        for i in range(n):
            d = {k: getattr(res[i], k) for k in _abi.RESULT_KEYS}
            d["x"], d["yn"] = outs[i]
            out.append(d)
        return out

    def set_stream(self, handle):
        """Issue the context's work on a caller-owned cudaStream_t (int handle,
        e.g. torch.cuda.Stream().cuda_stream); None restores the own stream."""
        self._check(self._L.rtb_set_stream(self._h, C.c_void_p(handle) if handle else None))

    def stats(self) -> dict:
        s = _abi.RtbFwdStats()
        self._check(self._L.rtb_get_fwd_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def debug_bins(self, job):
        npass = max(job.ngas - 1, 1)
        ng = self.tables.ng
        perm = np.full((job.nwave, job.nlayer, npass, ng * ng), -1, np.int16)
        split = np.full((job.nwave, job.nlayer, npass, ng), -1, np.int16)
        p16 = C.POINTER(C.c_int16)
        self._check(self._L.rtb_get_debug_bins(self._h, perm.ctypes.data_as(p16), perm.size,
                                               split.ctypes.data_as(p16), split.size))
        return perm, split


class Server:
    """Continuous-batching retrieval server (rtb_server_*): submit requests
    at any time, call step() to run rounds, poll() for finished results."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int, kiter=10, phlimit=0.1, dchisq_stop=0.0):
        self._ctx = ctx
        self._L = ctx._L
        o = _abi.RtbRetrievalOpts(kiter, phlimit, dchisq_stop, 0)
        h = C.c_void_p()
        ctx._check(self._L.rtb_server_create(ctx._h, hbm_budget_bytes, C.byref(o), C.byref(h)))
        self._h = h
        self._cases = {}

    def close(self):
        if self._h:
            self._L.rtb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, case) -> int:
        s = case.as_struct()
        rid = C.c_longlong()
        self._ctx._check(self._L.rtb_server_submit(self._h, C.byref(s), C.byref(rid)))
        self._cases[rid.value] = case
        return rid.value

    def step(self):
        a, q = C.c_int(), C.c_int()
        self._ctx._check(self._L.rtb_server_step(self._h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def poll(self, rid):
        case = self._cases[rid]
        r = _abi.RtbRetrievalResult()
        x = np.zeros(case.nx, np.float32)
        yn = np.zeros(case.ny, np.float32)
        r.x, r.yn = _abi.fptr(x), _abi.fptr(yn)
        done = C.c_int()
        self._ctx._check(self._L.rtb_server_poll(self._h, rid, C.byref(done), C.byref(r)))
        if not done.value:
            return None
        del self._cases[rid]
        d = {k: getattr(r, k) for k in _abi.RESULT_KEYS}
        d["x"], d["yn"] = x, yn
        return d

