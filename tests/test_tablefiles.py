"""The reference's table formats: .kta headers read without a device (CPU),
and whole runs loaded from .kta and CIA .tab files against the same tables
handed over in memory (GPU)."""
import ctypes as C
import os

import numpy as np
import pytest

from radtrancode_b200 import _lib, synth
from tests.helpers import JAC_TOL, RAD_TOL, jac_err, rad_err
from tests.tablefiles import write_cia_tab, write_kta


def _header(path):
    L = _lib.lib()
    ip = lambda: C.c_int()
    np_, nt, ng, npt, ida, iso = ip(), ip(), ip(), ip(), ip(), ip()
    vmin, delv = C.c_float(), C.c_float()
    st = L.rtb_kta_header(os.fsencode(path), C.byref(np_), C.byref(nt), C.byref(ng), C.byref(npt),
                          C.byref(vmin), C.byref(delv), C.byref(ida), C.byref(iso))
    return st, (np_.value, nt.value, ng.value, npt.value, vmin.value, delv.value, ida.value, iso.value)


def test_kta_header(tmp_path):
    _lib.build()
    kt, _, _ = synth.config1()
    p = str(tmp_path / "ch4.kta")
    write_kta(p, kt, 0, 6, 0)
    st, h = _header(p)
    assert st == 0
    assert h == (kt.np_, kt.nt, kt.ng, int(kt.nbin[0]), float(kt.vmin[0]), float(kt.delv[0]), 6, 0)


def test_kta_t2_header_and_short_files(tmp_path):
    _lib.build()
    kt = synth.make_ktables([synth.CH4], np_=12, nt=9, ng=10, nbin=4, t2=True)
    p = str(tmp_path / "t2.kta")
    write_kta(p, kt, 0, 6, 0)                        # TEMP2(NP, |NT|) tables
    st, h = _header(p)
    assert st == 0 and h[:3] == (12, -9, 10)
    q = str(tmp_path / "short.kta")
    open(q, "wb").write(open(p, "rb").read()[:20])
    assert _header(q)[0] == 1                        # RTB_ERR_ARG
    assert _header(str(tmp_path / "missing.kta"))[0] == 1


@pytest.mark.gpu
def test_run_from_files_matches_in_memory_tables(ctx, tmp_path):
    kt, cia, job = synth.config2(nwave=24, nlayer=60, nbin=24)
    paths = []
    for i, gas in enumerate(kt.gases):
        p = str(tmp_path / f"gas{i}.kta")
        write_kta(p, kt, i, gas[0], gas[1])
        paths.append(p)
    ctab = str(tmp_path / "cia.tab")
    write_cia_tab(ctab, cia)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, gt0 = ctx.cirsrtfg_wave(job)
    ids = ctx.load_ktables(paths)
    ctx.load_cia(ctab, cia.dnu)
    assert ids == [tuple(g) for g in kt.gases]
    c, g, gt = ctx.cirsrtfg_wave(job)
    assert rad_err(c, c0) <= RAD_TOL
    assert jac_err(g, g0, job.nv) <= JAC_TOL
    ctx.set_ktables(kt)                  # leave the session context as the other tests expect


@pytest.mark.gpu
def test_run_from_t2_files_matches_in_memory_tables(ctx, tmp_path):
    """.kta files with TEMP2(NP, |NT|) temperatures (read_khead.f:86-93) give
    the run of the same tables handed over in memory."""
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, nbin=12, seed=5, t2=True)
    cia = synth.make_cia(5)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=6, nwave=12)
    paths = []
    for i, gas in enumerate(kt.gases):
        p = str(tmp_path / f"t2gas{i}.kta")
        write_kta(p, kt, i, gas[0], gas[1])
        paths.append(p)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, _ = ctx.cirsrtfg_wave(job)
    ctx.load_ktables(paths)
    c, g, _ = ctx.cirsrtfg_wave(job)
    assert rad_err(c, c0) <= RAD_TOL
    assert jac_err(g, g0, job.nv) <= JAC_TOL


@pytest.mark.gpu
def test_run_from_irregular_files_matches_in_memory_tables(ctx, tmp_path):
    """.kta files on an irregular grid (DELV = 0, VCEN records,
    read_khead.f:100-103): the loader hands the first file's centres to
    rtb_set_ktable_centres and the run is the in-memory one."""
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, nbin=14, seed=8, irregular=0.0)
    cia = synth.make_cia(8)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=9, nwave=8)
    job.vwave = (600.0 + 0.4 * (np.arange(8) + 1) + 0.11).astype(np.float32)
    paths = []
    for i, gas in enumerate(kt.gases):
        p = str(tmp_path / f"irr{i}.kta")
        write_kta(p, kt, i, gas[0], gas[1])
        paths.append(p)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, _ = ctx.cirsrtfg_wave(job)
    ctx.load_ktables(paths)
    c, g, _ = ctx.cirsrtfg_wave(job)
    assert rad_err(c, c0) <= RAD_TOL
    assert jac_err(g, g0, job.nv) <= JAC_TOL

