"""CPU tests of the oracle (the C++ restatement in oracle/): known-answer
tests, finite differences, invariants and the committed golden fixtures."""
import hashlib
import os

import numpy as np
import pytest

from radtrancode_b200 import synth
from tests.helpers import jac_err, rad_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
# the reference's data directory (raddata/) of the checkout named by RADTRAN_REFERENCE,
# else of the default checkout; the tests that read it skip where it is absent
RADDATA = os.path.join(os.environ.get("RADTRAN_REFERENCE", "/root/reference"), "raddata")


def _golden_input_digest(kt, cia, job):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.input_digest(kt, cia, job), mg


# ---------------------------------------------------------------- det exp
def test_detexp_matches_golden_bits(oracle):
    g = np.load(os.path.join(GOLDEN, "detexp.npz"))
    y = oracle.det_expf(g["x"])
    assert np.array_equal(y.view(np.uint32), g["y"].view(np.uint32))


def test_detexp_is_correctly_rounded_almost_everywhere(oracle):
    x = np.random.default_rng(3).uniform(-30.0, 30.0, 20000).astype(np.float32)
    y = oracle.det_expf(x)
    ref = np.exp(x.astype(np.float64)).astype(np.float32)
    ulps = np.abs(y.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    assert (ulps == 0).mean() > 0.9999


# ---------------------------------------------------------------- locate
def test_locate_endpoint_snapping(oracle):
    import ctypes as C
    xx = np.array([1.0, 2.0, 3.0, 4.0], np.float32)
    p = xx.ctypes.data_as(C.POINTER(C.c_float))
    L = oracle.lib()
    assert L.orc_locate(p, 4, 1.0) == 1          # x == xx(1) -> 1
    assert L.orc_locate(p, 4, 4.0) == 3          # x == xx(n) -> n-1
    assert L.orc_locate(p, 4, 2.5) == 2
    assert L.orc_locate(p, 4, 0.5) == 0          # below range
    assert L.orc_locate(p, 4, 9.0) == 4          # above range
    xd = xx[::-1].copy()
    pd = xd.ctypes.data_as(C.POINTER(C.c_float))
    assert L.orc_locate(pd, 4, 2.5) == 2         # decreasing table


# ---------------------------------------------------------------- heapsort
def _nr_heapsort_py(ra):
    """Independent pure-Python restatement of sort2g.f for small arrays."""
    ra = [None] + list(ra)
    ib = [None] + list(range(len(ra) - 1))
    n = len(ra) - 1
    L, IR = n // 2 + 1, n
    while True:
        if L > 1:
            L -= 1
            rra, irb = ra[L], ib[L]
        else:
            rra, irb = ra[IR], ib[IR]
            ra[IR], ib[IR] = ra[1], ib[1]
            IR -= 1
            if IR == 1:
                ra[1], ib[1] = rra, irb
                return ra[1:], ib[1:]
        i, j = L, L + L
        while j <= IR:
            if j < IR and ra[j] < ra[j + 1]:
                j += 1
            if rra < ra[j]:
                ra[i], ib[i] = ra[j], ib[j]
                i, j = j, j + j
            else:
                j = IR + 1
        ra[i], ib[i] = rra, irb


@pytest.mark.parametrize("n,levels", [(2, 2), (7, 3), (50, 5), (400, 40), (400, 400)])
def test_sort2g_matches_python_heapsort_with_ties(oracle, n, levels):
    rng = np.random.default_rng(n + levels)
    a = rng.integers(0, levels, n).astype(np.float32)
    s, ib = oracle.sort2g(a)
    s_py, ib_py = _nr_heapsort_py(a.tolist())
    assert np.array_equal(s, np.array(s_py, np.float32))
    assert np.array_equal(ib, np.array(ib_py))
    assert np.all(np.diff(s) >= 0)


# ---------------------------------------------------------------- rankg
def test_rankg_conserves_weighted_k_and_is_monotone(oracle):
    ng = 20
    _, delg = synth.gauss_legendre_01(ng)
    rng = np.random.default_rng(11)
    k1 = np.sort(rng.lognormal(0, 2, ng)).astype(np.float32)
    k2 = np.sort(rng.lognormal(-1, 2, ng)).astype(np.float32)
    cont = (k1[:, None] + k2[None, :]).astype(np.float32).ravel()
    weight = (delg[:, None] * delg[None, :]).astype(np.float32).ravel()
    grad = np.stack([np.repeat(k1, ng), np.tile(k2, ng)]).astype(np.float32)
    st, k_g, dkdq, perm, split = oracle.rankg(delg, weight, cont, grad)
    assert st == 0
    assert np.all(np.diff(k_g) >= 0)
    lhs = float(np.sum(k_g.astype(np.float64) * delg))
    rhs = float(np.sum(cont.astype(np.float64) * weight))
    assert abs(lhs - rhs) / rhs < 1e-5
    assert sorted(perm.tolist()) == list(range(ng * ng))
    closed = split[split >= 0]
    assert closed.size >= ng - 1 and np.all(np.diff(closed) > 0)


# ---------------------------------------------------------------- forward KATs
def test_golden_fixtures_reproduced(oracle):
    for name, (kt, cia, job) in [("c1", synth.config1()), ("c2s", synth.config2(nwave=8, nlayer=30, nbin=8))]:
        g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        dig, _ = _golden_input_digest(kt, cia, job)
        assert str(g["input_sha256"]) == dig, f"{name}: synthetic generator changed"
        (c, gr, gt), (perm, split, ties) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
        assert np.array_equal(c, g["calcout"]) and np.array_equal(gr, g["gradients"])
        c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
        assert np.array_equal(c64, g["calcout64"]) and np.array_equal(g64, g["gradients64"])
        if perm is not None:
            assert hashlib.sha256(perm.tobytes()).hexdigest() == str(g["perm_sha256"])
            assert np.array_equal(split, g["split"])


def _isothermal(job, T):
    job.temp[:] = T
    job.emtemp[:job.nlayer, 0] = T
    return job


def test_isothermal_atmosphere_radiates_planck(oracle):
    kt, cia, job = synth.config2(nwave=6, nlayer=24, nbin=6)
    job = _isothermal(job, 150.0)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    v = job.vwave.astype(np.float64)
    c1, c2 = float(np.float32(1.1911e-12)), float(np.float32(1.439))
    # every g-ordinate radiates B(T); the quadrature weights (REAL) sum to 1 +- 1 ulp
    B = c1 * v ** 3 / np.expm1(c2 * v / 150.0) * float(np.sum(kt.delg.astype(np.float64)))
    assert np.max(np.abs(c64 - B) / B) < 1e-12
    G = g64.reshape(job.nv, -1)
    L = job.nlayer
    # gas-scale columns vanish for an isothermal atmosphere over a B(T) surface
    assert np.max(np.abs(G[L:])) < 1e-12 * np.max(np.abs(G[:L]))


def test_zero_table_gas_leaves_result_unchanged(oracle):
    kt, cia, job1 = synth.config2(nwave=6, nlayer=20, nbin=6)
    kt_z = synth.KTables(kt.np_, kt.nt, kt.ng, kt.lnp, kt.tk, kt.g_ord, kt.delg, kt.vmin, kt.delv, kt.nbin,
                         kt.data.copy(), kt.gases)
    kt_z.table(1)[:] = 0.0     # C2H6 table all zero: get_kg.f:228-250 zero probe, noverlapg skip branch
    kt_1 = synth.KTables(kt.np_, kt.nt, kt.ng, kt.lnp, kt.tk, kt.g_ord, kt.delg, kt.vmin[:1], kt.delv[:1],
                         kt.nbin[:1], kt.table(0).ravel().copy(), kt.gases[:1])
    job_a = synth.make_job(kt_z, [synth.CH4, synth.C2H6], nlayer=20, seed=5, nwave=6)
    job_b = synth.make_job(kt_1, [synth.CH4], nlayer=20, seed=5, nwave=6)
    ca, ga, _ = oracle.cirsrtfg_wave(kt_z, cia, job_a, oracle.ORC_MIXED)
    cb, gb, _ = oracle.cirsrtfg_wave(kt_1, cia, job_b, oracle.ORC_MIXED)
    assert np.array_equal(ca, cb)
    Ga = ga.reshape(job_a.nv, -1)
    Gb = gb.reshape(job_b.nv, -1)
    assert np.array_equal(Ga[:job_b.nv], Gb)       # T columns and the CH4 scale


def test_mixed_precision_agrees_with_fp64(oracle):
    kt, cia, job = synth.config2(nwave=10, nlayer=40, nbin=10)
    c, g, gt = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED)
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) < 1e-5
    assert jac_err(g, g64, job.nv) < 1e-4


def test_t2_tables_in_both_precisions(oracle):
    """NT < 0 tables (TEMP2, get_kg.f:143-169): the two precisions agree, and
    a table whose every pressure row carries the same grid gives the run of
    the single-grid table (the two interpolations are the same function)."""
    import dataclasses
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, nbin=10, seed=3, t2=True)
    cia = synth.make_cia(3)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=4, nwave=10)
    c, g, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) < 1e-5
    assert jac_err(g, g64, job.nv) < 1e-4
    grid = np.linspace(70.0, 200.0, 15).astype(np.float32)
    kts = dataclasses.replace(kt, nt=15, tk=grid)
    ktr = dataclasses.replace(kt, nt=-15, tk=np.repeat(grid, 20))     # TEMP2(i, j) = grid(j)
    a = oracle.cirsrtfg_wave(kts, cia, job, oracle.ORC_FP64)
    b = oracle.cirsrtfg_wave(ktr, cia, job, oracle.ORC_FP64)
    assert rad_err(b[0], a[0]) < 1e-12 and jac_err(b[1], a[1], job.nv) < 1e-11


def test_finite_difference_jacobian_fp64(oracle):
    """Analytic dR/dx of the FP64 oracle against central differences of its
    own forward model (temperature of chosen levels, gas scale factors)."""
    kt, cia, job = synth.config2(nwave=4, nlayer=20, nbin=4)
    absorbers = synth.ABSORBERS_C2
    base_T = job.temp.astype(np.float64).copy()
    c0, g0, gts0 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    G = g0.reshape(job.nv, -1)
    L = job.nlayer

    def run(T=None, xscale=None):
        j = synth.make_job(kt, absorbers, nlayer=L, seed=1003, nwave=4, vmr_perturb=0.3,
                           temp=base_T if T is None else T, xscale=xscale)
        j.delh[:] = job.delh           # layer thickness held fixed, as the analytic gradient assumes
        return oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64)[0]

    for lev in (0, 7, 19):
        h = 2e-3
        Tp = base_T.copy(); Tp[lev] += h
        Tm = base_T.copy(); Tm[lev] -= h
        # the layer arrays are REAL: divide by the step that survives float32 rounding
        h2 = float(np.float32(Tp[lev])) - float(np.float32(Tm[lev]))
        fd = (run(T=Tp) - run(T=Tm)) / h2
        ana = G[lev].copy()
        if lev == 0:
            # with TSURF <= 0 the surface radiates B(T) of the bottom layer; the
            # reference returns that dependence separately as gradtsurf
            # (cirsradg_wave.f:993-1006), not inside the layer gradient
            ana = ana + gts0
        scale = np.max(np.abs(ana))
        # piecewise-linear table interpolation and the rank rebinning have kinks:
        # the check is at the Jacobian acceptance level
        assert np.max(np.abs(fd - ana)) / scale < 1e-3, lev
    for a in range(len(absorbers)):
        h = 1e-4
        xp = np.zeros(len(absorbers)); xp[a] = h
        fd = (run(xscale=xp) - run(xscale=-xp)) / (2 * h)
        scale = np.max(np.abs(G[L + a]))
        assert np.max(np.abs(fd - G[L + a])) / scale < 1e-3, a


def test_unsupported_options_are_reported(oracle):
    kt, cia, job = synth.config1()
    job.imod[0] = 15       # multiple scattering STOPs in the reference
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        oracle.cirsrtfg_wave(kt, cia, job)


# ---------------------------------------------------------------- real CIA data
ISOTEST = os.path.join(RADDATA, "isotest.tab")


def read_cia_tab(path):
    """gfortran sequential unformatted file of ciaread.f:77-98: record 1 =
    25 DOUBLE temperatures, record 2 = REAL kcia(9, 25, 1501)."""
    raw = open(path, "rb").read()
    n1 = np.frombuffer(raw[0:4], np.int32)[0]
    temps = np.frombuffer(raw[4:4 + n1], np.float64).copy()
    o = 4 + n1 + 4
    n2 = np.frombuffer(raw[o:o + 4], np.int32)[0]
    kcia = np.frombuffer(raw[o + 4:o + 4 + n2], np.float32).copy()
    return temps, kcia


@pytest.mark.skipif(not os.path.exists(ISOTEST), reason="reference data not mounted")
def test_real_cia_table_isotest(oracle):
    temps, kcia = read_cia_tab(ISOTEST)
    assert temps.size == 25 and kcia.size == 9 * 25 * 1501
    assert np.all(np.diff(temps) > 0) and np.all(np.isfinite(kcia))
    kt, _, job = synth.config1()
    cia = synth.CIATable(1.0, temps, kcia)
    c, g, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    c0, _, _ = oracle.cirsrtfg_wave(kt, None, job, oracle.ORC_FP64)
    assert np.all(np.isfinite(c)) and np.all(c > 0)
    assert np.any(c != c0)     # the H2-H2/H2-He continuum changes the spectrum


def test_para_h2_jacobian_by_finite_differences(oracle):
    """The FP64 oracle's para-H2 fraction derivative (nparacon_all.f DH2DFP,
    DHEDFP through DFP and xmap) against central differences of its own
    radiance in the layer's para fraction; the coefficients are linear in the
    fraction within a bracket, so the two agree closely away from the
    bracket edges."""
    kt, cia, _ = synth.config2(nwave=4, nlayer=20, nbin=4)
    cia.para = synth.make_para_cia(7)
    job0 = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=20, seed=82, nwave=4)
    fp = cia.para.fp
    mid = 0.5 * (fp[4:15] + fp[5:16])                    # bracket centres
    hfp = np.resize(mid, 20).astype(np.float32)
    job = synth.with_para_h2(job0, hfp)
    c, g, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    G = g.reshape(job.nv, job.nwave)
    h = 1e-3
    for lay in (2, 9, 15):
        jp = synth.with_para_h2(job0, hfp + h * (np.arange(20) == lay))
        jm = synth.with_para_h2(job0, hfp - h * (np.arange(20) == lay))
        cp, _, _ = oracle.cirsrtfg_wave(kt, cia, jp, oracle.ORC_FP64)
        cm, _, _ = oracle.cirsrtfg_wave(kt, cia, jm, oracle.ORC_FP64)
        fd = (cp - cm) / (2 * h)
        an = G[job.nv - job.npro + lay]
        assert np.max(np.abs(fd - an)) <= 2e-3 * np.max(np.abs(an)) + 1e-30, lay


def _imod18(job, tsurf=0.0, emissivity=1.0):
    job.imod[:] = 18
    job.tsurf = tsurf
    job.vem = np.array([1.0, 1e4], np.float32)
    job.emissivity = np.array([emissivity, emissivity], np.float32)
    return job


def test_imod18_isothermal_hemisphere_radiates_pi_planck(oracle):
    """IMOD 18 (cirsradg_wave.f:1116-1225): over a black surface at the
    atmosphere's temperature the E3 differences telescope to E3(0) = 1/2, so
    the hemispherical flux is pi B(T) whatever the optical depths; with
    iform = 3 it is that flux times 4 pi ((radius1 + radextra) 1e5)^2 1e-18
    (cirsradg_wave.f:1136-1152)."""
    import dataclasses
    e3 = synth.make_e3_table()
    kt, cia, job = synth.config2(nwave=6, nlayer=24, nbin=6)
    job = _imod18(_isothermal(job, 150.0), tsurf=150.0)
    c64, _, gt = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=e3)
    v = job.vwave.astype(np.float64)
    c1, c2 = float(np.float32(1.1911e-12)), float(np.float32(1.439))
    pi = float(np.float32(np.pi))
    B = c1 * v ** 3 / np.expm1(c2 * v / 150.0) * float(np.sum(kt.delg.astype(np.float64)))
    assert np.max(np.abs(c64 - pi * B) / B) < 1e-12
    assert np.all(gt > 0)
    j3 = dataclasses.replace(job, iform=3, radius1=71492.0, radextra=25.0)
    c3, _, _ = oracle.cirsrtfg_wave(kt, cia, j3, oracle.ORC_FP64, e3=e3)
    r = (71492.0 + 25.0) * 1e5           # the FP64 oracle forms the factor in double
    xfac = 4.0 * pi * r * r * float(np.float32(1e-18))
    assert np.max(np.abs(c3 / c64 - xfac)) < 1e-12 * xfac


def test_imod18_jacobian_by_finite_differences(oracle):
    """The FP64 oracle's IMOD 18 Jacobian (the E3-gradient recurrence of
    cirsradg_wave.f:1176-1195) against central differences of its own
    hemispherical flux, with no surface term (TSURF = 0).  The analytic
    E3 gradient interpolates e3interp's central-difference table, not the
    slope of the interpolant, hence the looser bound than the IMOD 3 check."""
    e3 = synth.make_e3_table()
    kt, cia, job = synth.config2(nwave=4, nlayer=20, nbin=4)
    absorbers = synth.ABSORBERS_C2
    base_T = job.temp.astype(np.float64).copy()
    job = _imod18(job)
    _, g0, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=e3)
    G = g0.reshape(job.nv, -1)
    L = job.nlayer

    def run(T=None, xscale=None):
        j = synth.make_job(kt, absorbers, nlayer=L, seed=1003, nwave=4, vmr_perturb=0.3,
                           temp=base_T if T is None else T, xscale=xscale)
        j.delh[:] = job.delh
        return oracle.cirsrtfg_wave(kt, cia, _imod18(j), oracle.ORC_FP64, e3=e3)[0]

    for lev in (0, 7, 19):
        Tp = base_T.copy(); Tp[lev] += 2e-3
        Tm = base_T.copy(); Tm[lev] -= 2e-3
        h2 = float(np.float32(Tp[lev])) - float(np.float32(Tm[lev]))
        fd = (run(T=Tp) - run(T=Tm)) / h2
        assert np.max(np.abs(fd - G[lev])) / np.max(np.abs(G[lev])) < 5e-3, lev
    for a in range(len(absorbers)):
        xp = np.zeros(len(absorbers)); xp[a] = 1e-4
        fd = (run(xscale=xp) - run(xscale=-xp)) / 2e-4
        assert np.max(np.abs(fd - G[L + a])) / np.max(np.abs(G[L + a])) < 5e-3, a


def test_imod18_needs_the_e3_table(oracle):
    kt, cia, job = synth.config2(nwave=2, nlayer=10, nbin=2)
    job = _imod18(job)
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)


E3TAB = os.path.join(RADDATA, "e3tab.dat")


@pytest.mark.skipif(not os.path.exists(E3TAB), reason="reference data not mounted")
def test_real_e3_table(oracle):
    """The reference's own e3tab.dat (read as e3interp.f:36-45 reads it): the
    synthetic table the GPU tests use agrees with it to 5e-5 at transmissions
    >= 0.1 (below that the file's entries drift from E3 by up to a few tens
    of per cent), and the oracle's IMOD 18 run on it keeps the
    pi B identity of a black isothermal hemisphere."""
    lines = open(E3TAB).read().splitlines()
    n = int(lines[0])
    rec = np.array([[float(x) for x in ln.split()] for ln in lines[2:2 + n]])
    real = synth.E3Table(rec[:, 0].copy(), rec[:, 1].copy(), rec[:, 2].copy())
    syn = synth.make_e3_table()
    assert n == 1001 and real.tran[-1] == 1.0 and real.e3[-1] == 0.5
    assert np.max(np.abs(real.tran - syn.tran)) < 1e-9
    ok = syn.tran >= 0.1
    assert np.max(np.abs(real.e3[ok] - syn.e3[ok]) / syn.e3[ok]) < 5e-5
    kt, cia, job = synth.config2(nwave=4, nlayer=20, nbin=4)
    job = _imod18(_isothermal(job, 150.0), tsurf=150.0)
    c_real, _, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=real)
    c_syn, _, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=syn)
    assert np.max(np.abs(c_real - c_syn) / c_syn) < 1e-12


def test_dust_jacobian_by_finite_differences(oracle):
    """Dust continuum (cirsradg_wave.f:550-575: taucon += xsec * cont,
    dtaucondq(ngas+1+k) = xsec; DCO maps it to the levels): the FP64
    oracle's derivative in the scale of each dust profile against central
    differences of its own radiance, and a dusty spectrum darker than the
    clear one."""
    kt, cia, job = synth.config2(nwave=4, nlayer=30, nbin=4)
    jd = synth.with_dust(job, 2, seed=3)
    c, g, _ = oracle.cirsrtfg_wave(kt, cia, jd, oracle.ORC_FP64)
    c0, _, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert np.all(c < c0)
    G = g.reshape(jd.nv, -1)
    h = 1e-3
    for k in range(2):
        jp = synth.with_dust(job, 2, seed=3)
        jp.cont[k] *= 1 + h
        jm = synth.with_dust(job, 2, seed=3)
        jm.cont[k] *= 1 - h
        fd = (oracle.cirsrtfg_wave(kt, cia, jp, oracle.ORC_FP64)[0] -
              oracle.cirsrtfg_wave(kt, cia, jm, oracle.ORC_FP64)[0]) / (2 * h)
        an = G[job.nv + k]
        assert np.max(np.abs(fd - an)) <= 1e-4 * np.max(np.abs(an)), k


def test_nlte_emission_temperatures(oracle):
    """calc_nlte_t (inlte 1, 2): with A = 0 the source function is B(T)
    itself (T_nlte = invplanck(planck(T)) to rounding), so the spectrum is
    the LTE one; a finite A lowers the upper layers' source function and
    the spectrum darkens; inlte = 2 at these pressures (f >= 0.99) changes
    it by under 1 %.  k1 outside 1e-20 .. 1e-3 is refused."""
    import dataclasses
    kt, cia, job = synth.config2(nwave=4, nlayer=30, nbin=4)
    c0, g0, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    ca, ga, _ = oracle.cirsrtfg_wave(kt, cia, dataclasses.replace(job, inlte=1, nlte_k1=1e-10, nlte_A=0.0),
                                     oracle.ORC_FP64)
    assert rad_err(ca, c0) < 1e-6 and jac_err(ga, g0, job.nv) < 1e-5
    cb, _, _ = oracle.cirsrtfg_wave(kt, cia, dataclasses.replace(job, inlte=1, nlte_k1=1e-10, nlte_A=5e5),
                                    oracle.ORC_FP64)
    assert np.all(cb < c0)
    cc, _, _ = oracle.cirsrtfg_wave(kt, cia, dataclasses.replace(job, inlte=2), oracle.ORC_FP64)
    assert np.all(cc <= c0) and np.max(np.abs(cc - c0) / c0) < 1e-2
    with pytest.raises(RuntimeError, match="ARG"):
        oracle.cirsrtfg_wave(kt, cia, dataclasses.replace(job, inlte=1, nlte_k1=1e-2, nlte_A=1.0), oracle.ORC_FP64)


def _read_stellar(path):
    """init_solar_wave.f:22-78: '#' comment lines, the wavespace, the
    stellar radius, then WAVE RAD records."""
    rows = [ln.split() for ln in open(path).read().splitlines() if ln.strip() and not ln.startswith("#")]
    ispace, solrad = int(rows[0][0]), float(rows[1][0])
    rec = np.array([[float(a), float(b)] for a, b in rows[2:]], np.float32)
    return ispace, synth.StellarSpectrum(solrad, rec[:, 0].copy(), rec[:, 1].copy())


def test_stellar_flux_ratio_and_transmission(oracle):
    """iform 1 (cirsradg_wave.f:913-929): the IMOD 3 flux times
    pi 4 pi (R 1e5)^2, over get_solar_wave(v, -1); iform 4 (:861-879): the
    IMOD 0 transmission times get_solar_wave(v, dist), the star's power
    over 4 pi (dist AU)^2; without a stellar spectrum iform 1 keeps the
    total flux and iform 4 the transmission.  Checked against numpy's
    linear interpolation of the table."""
    import dataclasses
    kt, cia, job = synth.config2(nwave=4, nlayer=30, nbin=4)
    ss = synth.make_stellar_spectrum(500.0, 800.0, descending=True)
    v = job.vwave.astype(np.float64)
    xs = np.interp(v, ss.wave[::-1].astype(np.float64), ss.rad[::-1].astype(np.float64))
    pi = float(np.float32(np.pi))
    c0, g0, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    j1 = dataclasses.replace(job, iform=1, radius1=71492.0, radextra=10.0)
    c1, g1, _ = oracle.cirsrtfg_wave(kt, cia, j1, oracle.ORC_FP64, solar=ss)
    area = pi * 4.0 * pi * ((71492.0 + 10.0) * 1e5) ** 2
    assert np.max(np.abs(c1 * xs / area / c0 - 1.0)) < 1e-6
    assert jac_err(g1 * np.tile(xs, job.nv) / area, g0, job.nv) < 1e-6
    c1n, _, _ = oracle.cirsrtfg_wave(kt, cia, j1, oracle.ORC_FP64)
    assert np.max(np.abs(c1n / area / c0 - 1.0)) < 1e-6
    j4 = dataclasses.replace(job, iform=4, dist=5.2)
    j4.imod[:] = 0
    j0 = dataclasses.replace(job)
    j0.imod = np.zeros_like(job.imod)
    t0, _, _ = oracle.cirsrtfg_wave(kt, cia, j0, oracle.ORC_FP64)
    t4, _, _ = oracle.cirsrtfg_wave(kt, cia, j4, oracle.ORC_FP64, solar=ss)
    sph = 4.0 * pi * (5.2 * 1.49598e13) ** 2
    assert np.max(np.abs(t4 * sph / xs / t0 - 1.0)) < 1e-5


STELLAR = os.path.join(RADDATA, "upsAnd.dat")


@pytest.mark.skipif(not os.path.exists(STELLAR), reason="reference data not mounted")
def test_real_stellar_spectrum_file(oracle):
    """The reference's upsAnd.dat (wavelength space, 0.465-0.97 um) read as
    init_solar_wave reads it; the oracle's iform 4 transmission at 0.8 um
    is the IMOD 0 transmission times the file's interpolated luminosity
    over 4 pi (dist AU)^2."""
    import dataclasses
    ispace, ss = _read_stellar(STELLAR)
    assert ispace == 1 and ss.solrad > 0 and len(ss.wave) > 10 and np.all(ss.rad > 0)
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, vmin=12500.0, delv=0.4, nbin=4, seed=2)
    cia = synth.make_cia(2)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=30, seed=3, nwave=4)
    lam = (1e4 / job.vwave.astype(np.float64)).astype(np.float32)
    assert ss.wave.min() < lam.min() and lam.max() < ss.wave.max()
    j0 = dataclasses.replace(job, ispace=1, vwave=lam, imod=np.zeros_like(job.imod))
    j4 = dataclasses.replace(j0, iform=4, dist=3.0)
    t0, _, _ = oracle.cirsrtfg_wave(kt, None, j0, oracle.ORC_FP64)
    t4, _, _ = oracle.cirsrtfg_wave(kt, None, j4, oracle.ORC_FP64, solar=ss)
    xs = np.interp(lam.astype(np.float64), ss.wave.astype(np.float64), ss.rad.astype(np.float64))
    pi = float(np.float32(np.pi))
    sph = 4.0 * pi * (3.0 * 1.49598e13) ** 2
    assert np.all(t0 > 0) and np.max(np.abs(t4 * sph / xs / t0 - 1.0)) < 1e-5


def test_rayleigh_venus_and_air(oracle):
    """IRAY 2 (rayleighv.f, C / lambda^4 per wavenumber) and 3 (rayleigha.f,
    air at each layer's P and T): the two precisions agree, the scattering
    optical depth dims the spectrum against IRAY 0, and IRAY 4 (rayleighls,
    whose layer fractions the reference leaves unset for absent gases) is
    refused."""
    import dataclasses
    kt, cia, job = synth.config2(nwave=4, nlayer=30, nbin=4)
    c0, _, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    for iray in (2, 3):
        j = dataclasses.replace(job, iray=iray)
        cm, gm, _ = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_MIXED)
        c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64)
        assert rad_err(cm, c64) < 1e-5 and jac_err(gm, g64, j.nv) < 1e-4
        assert np.all(c64 <= c0) and np.any(c64 < c0)
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        oracle.cirsrtfg_wave(kt, cia, dataclasses.replace(job, iray=4), oracle.ORC_FP64)
