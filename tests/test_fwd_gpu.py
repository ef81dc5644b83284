"""GPU parity tests of the forward model + Jacobian against the oracle.

Every comparison runs the CUDA kernels through the C ABI (radtrancode_b200
Context -> libradtran_b200.so) and the oracle on the same seeded inputs.
Tolerances: tests/helpers.py."""
import copy
import dataclasses
import os

import numpy as np
import pytest

from radtrancode_b200 import synth
from tests.helpers import JAC_TOL, RAD_TOL, assignment, jac_err, rad_err

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _run(ctx, kt, cia, job):
    ctx.set_ktables(kt)
    if cia is not None:
        ctx.set_cia(cia)
    return ctx.cirsrtfg_wave(job)


def test_config1_against_fp64_oracle_and_golden(ctx, oracle):
    kt, cia, job = synth.config1()
    c, g, gt = _run(ctx, kt, cia, job)
    gold = np.load(os.path.join(GOLDEN, "c1.npz"))
    assert rad_err(c, gold["calcout64"]) <= RAD_TOL
    assert jac_err(g, gold["gradients64"], job.nv) <= JAC_TOL
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    assert np.max(np.abs(gt - gt64)) <= RAD_TOL * np.max(np.abs(gt64))


@pytest.mark.parametrize("strict", [False, True])
def test_config2_small_bins_bit_exact(ctx, oracle, strict):
    """Integer g-bin assignment of every sorted overlap pass identical to the
    mixed-precision oracle (the reference's REAL/DOUBLE semantics)."""
    kt, cia, job = synth.config2(nwave=16, nlayer=60, nbin=16)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_strict_ties(strict)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(job)
        perm, split = ctx.debug_bins(job)
        st = ctx.stats()
    finally:
        ctx.set_debug(False)
        ctx.set_strict_ties(False)
    (c0, g0, gt0), (operm, osplit, oties) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    assert st["sort_passes"] == int((operm[..., 0] >= 0).sum())
    assert st["tie_passes"] == int((oties > 0).sum())
    a_gpu = assignment(perm, split, kt.ng)
    a_orc = assignment(operm, osplit, kt.ng)
    assert np.array_equal(a_gpu, a_orc)
    assert np.array_equal(split, osplit)
    if strict:
        # every pass with a tie took the reference heapsort: the whole order matches
        assert np.array_equal(perm, operm)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL


@pytest.mark.parametrize("ng", [2, 5, 10, 13, 21, 22])
def test_other_ng_bins_bit_exact_every_tile(ctx, oracle, ng):
    """NG other than 20 runs the generic kernel instance: merge levels with an
    unpaired last run (odd NG), a last level shorter than its pair, the
    largest NG; g-bins identical to the mixed oracle under every tile."""
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=ng, vmin=600.0, delv=0.4, nbin=8, seed=70 + ng)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=71 + ng, nwave=8, vmr_perturb=0.3)
    cia = synth.make_cia(70 + ng)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    (c0, g0, gt0), (operm, osplit, oties) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    a_orc = assignment(operm, osplit, kt.ng)
    ctx.set_debug(True)
    try:
        for tile in (8, 4, 2):
            ctx.set_tile(tile)
            c, g, gt = ctx.cirsrtfg_wave(job)
            perm, split = ctx.debug_bins(job)
            assert ctx.stats()["sort_passes"] == int((operm[..., 0] >= 0).sum())
            assert np.array_equal(assignment(perm, split, kt.ng), a_orc)
            assert np.array_equal(split, osplit)
            assert rad_err(c, c64) <= RAD_TOL
            assert jac_err(g, g64, job.nv) <= JAC_TOL
    finally:
        ctx.set_debug(False)
        ctx.set_tile(0)


def test_k_distribution_not_monotone_in_g_takes_the_reference_heapsort(ctx, oracle):
    """A table whose k values are not sorted in g (the g axis of one gas
    permuted): its rows are not sorted, so those passes skip the merge and take
    the reference heapsort in-kernel; the whole sorted order is the oracle's."""
    kt, cia, job = synth.config2(nwave=8, nlayer=40, nbin=8)
    perm_g = np.random.default_rng(5).permutation(kt.ng)
    t = kt.table(1)                      # C2H6
    t[...] = t[..., perm_g]
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(job)
        perm, split = ctx.debug_bins(job)
        st = ctx.stats()
    finally:
        ctx.set_debug(False)
    (c0, g0, gt0), (operm, osplit, oties) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    assert st["exact_passes"] > 0
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    assert np.array_equal(split, osplit)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL


def test_config2_golden_fixture(ctx):
    kt, cia, job = synth.config2(nwave=8, nlayer=30, nbin=8)
    c, g, gt = _run(ctx, kt, cia, job)
    gold = np.load(os.path.join(GOLDEN, "c2s.npz"))
    assert rad_err(c, gold["calcout64"]) <= RAD_TOL
    assert jac_err(g, gold["gradients64"], job.nv) <= JAC_TOL


def test_fortran_leading_dimensions(ctx, oracle):
    """Arrays dimensioned MAXLAY x MAXGAS etc. as the COMMON blocks hold them."""
    kt, cia, _ = synth.config2(nwave=6, nlayer=30, nbin=6)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=30, seed=9, nwave=6, ld_lay=400)
    c, g, gt = _run(ctx, kt, cia, job)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL


@pytest.mark.parametrize("variant", ["tsurf", "rayleigh", "slant", "imod0", "imod1", "limb", "two_paths",
                                     "no_cia"])
def test_path_variants(ctx, oracle, variant):
    kt, cia, _ = synth.config2(nwave=5, nlayer=24, nbin=5)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=24, seed=21, nwave=5)
    use_cia = cia
    if variant == "tsurf":
        job.tsurf = 175.0
        job.vem = np.array([500.0, 1500.0], np.float32)
        job.emissivity = np.array([0.9, 0.7], np.float32)
    elif variant == "rayleigh":
        job.iray = 1
    elif variant == "slant":
        job.scale[:job.nlayer, 0] = 1.7
    elif variant in ("imod0", "imod1"):
        job.imod[0] = int(variant[-1])
    elif variant == "limb":
        # path goes down then up again: the bottom of the path is not the deepest layer
        L = job.nlayer
        half = np.arange(L, L // 2, -1)
        job.layinc[:, 0] = 0
        path = np.concatenate([half, half[::-1]])
        job.layinc[:path.size, 0] = path
        job.nlayin[0] = path.size
        job.emtemp[:path.size, 0] = job.temp[path - 1]
        job.scale[:path.size, 0] = 1.0
    elif variant == "two_paths":
        j2 = copy.deepcopy(job)
        L = job.nlayer
        lay = np.zeros((L, 2), np.int32, order="F")
        lay[:, 0] = job.layinc[:L, 0]
        lay[:, 1] = job.layinc[:L, 0]
        sc = np.zeros((L, 2), np.float32, order="F")
        sc[:, 0] = 1.0
        sc[:, 1] = 2.0
        em = np.zeros((L, 2), np.float32, order="F")
        em[:, 0] = job.emtemp[:L, 0]
        em[:, 1] = job.emtemp[:L, 0]
        j2.npath, j2.layinc, j2.scale, j2.emtemp = 2, lay, sc, em
        j2.nlayin = np.array([L, L], np.int32)
        j2.imod = np.array([3, 3], np.int32)
        job = j2
    elif variant == "no_cia":
        use_cia = None
    if use_cia is None:
        # a fresh context: the device context keeps a CIA table once loaded
        from radtrancode_b200 import cirsradg
        with cirsradg.Context(0) as c2:
            c2.set_ktables(kt)
            c, g, gt = c2.cirsrtfg_wave(job)
    else:
        c, g, gt = _run(ctx, kt, use_cia, job)
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, use_cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.npath * job.nv) <= JAC_TOL
    if variant == "tsurf":
        assert np.max(np.abs(gt - gt64)) <= RAD_TOL * np.max(np.abs(gt64))


def test_unsupported_options_raise(ctx):
    from radtrancode_b200 import cirsradg
    kt, cia, job = synth.config1()
    ctx.set_ktables(kt)
    j = copy.deepcopy(job)
    j.imod[0] = 15
    with pytest.raises(cirsradg.RtbError, match="UNSUPPORTED"):
        ctx.cirsrtfg_wave(j)
    j = copy.deepcopy(job)
    j.vem = np.array([1250.0, 1300.0], np.float32)   # interpem.f range error
    with pytest.raises(cirsradg.RtbError, match="RANGE"):
        ctx.cirsrtfg_wave(j)


def test_full_size_config2_properties(ctx):
    """Full config-2 size (120 layers, 4 absorbers, 2000 wavenumbers), where
    the oracle is too slow to run in a test: size-independent properties --
    finite positive radiance bounded by the Planck envelope of the profile,
    determinism, and agreement with the same spectrum computed in pieces."""
    kt, cia, job = synth.config2()
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, gt = ctx.cirsrtfg_wave(job)
    c2, g2, gt2 = ctx.cirsrtfg_wave(job)
    assert np.array_equal(c, c2) and np.array_equal(g, g2)
    assert np.all(np.isfinite(c)) and np.all(c > 0) and np.all(np.isfinite(g))
    v = job.vwave.astype(np.float64)
    c1_, c2_ = 1.1911e-12, 1.439
    Bmin = c1_ * v ** 3 / np.expm1(c2_ * v / job.temp.min())
    Bmax = c1_ * v ** 3 / np.expm1(c2_ * v / job.temp.max())
    assert np.all(c >= 0.999 * Bmin) and np.all(c <= 1.001 * Bmax)
    # the same wavenumbers in two halves give identical results (no cross-wavenumber state)
    j1 = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=0, nwave=1000, vmr_perturb=0.3)
    j2 = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=120, seed=1003, iw0=1000, nwave=1000, vmr_perturb=0.3)
    ca, ga, _ = ctx.cirsrtfg_wave(j1)
    cb, gb, _ = ctx.cirsrtfg_wave(j2)
    assert np.array_equal(np.concatenate([ca, cb]), c)
    G = g.reshape(job.nv, -1)
    assert np.array_equal(np.concatenate([ga.reshape(job.nv, -1), gb.reshape(job.nv, -1)], axis=1), G)


def _off_grid(job, kt, shift):
    """The job moved between the k-table points: vwave = vmin + delv (i + shift)."""
    j = copy.deepcopy(job)
    j.vwave = (kt.vmin[0] + kt.delv[0] * (np.arange(j.nwave) + shift)).astype(np.float32)
    return j


@pytest.mark.parametrize("shift", [0.37, 0.93])
def test_noncoincident_wavenumbers(ctx, oracle, shift):
    """get_kg.f:380-438 + rankk.f: two table points weighted and rank-rebinned.
    Radiance and Jacobian within tolerance of the FP64 oracle; the g-bins of
    the overlap passes built on those k values bit-exact with the mixed
    oracle."""
    kt, cia, job = synth.config2(nwave=12, nlayer=40, nbin=16)
    j = _off_grid(job, kt, shift)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(j)
        perm, split = ctx.debug_bins(j)
    finally:
        ctx.set_debug(False)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, j.nv) <= JAC_TOL
    (cm, gm, _), (operm, osplit, _) = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_MIXED, debug=True)
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    assert np.array_equal(split, osplit)
    # the coincident spectrum differs: the branch was taken
    c0, _, _ = ctx.cirsrtfg_wave(job)
    assert not np.array_equal(c0, c)


def test_cirsradg_wave_compat_matches_cirsrtfg_wave(ctx):
    """The per-wavenumber form (cirsradg_wave's output and doutputdq): its
    radiance is the whole-spectrum call's bit for bit, and map2pro + map2xvec
    of its doutputdq (done here in FP64) give the whole-spectrum Jacobian."""
    import dataclasses
    kt, cia, job = synth.config2(nwave=6, nlayer=40, nbin=8)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, gt = ctx.cirsrtfg_wave(job)
    G = g.reshape(job.nv, job.nwave).astype(np.float64)
    L, ngas = job.nlayer, job.ngas
    isw = [2, 3, 4, 5, ngas]                      # the absorbers and T: the parameters xmap touches
    lay = job.layinc[:L, 0] - 1
    scale = np.maximum(np.max(np.abs(G), axis=1), 1e-300)
    for iw in (0, 3, 5):
        j1 = dataclasses.replace(job, nwave=1, vwave=job.vwave[iw:iw + 1].copy())
        out, gts, dq = ctx.cirsradg_wave(j1, isw)
        assert out[0] == c[iw] and gts[0] == gt[iw]
        assert not dq[:, :, [0, 1]].any()          # H2, He: not in isw
        Gh = np.zeros(job.nv)
        for k in isw:
            M = (job.dte if k == ngas else job.dam).astype(np.float64)
            per_level = dq[0, :L, k].astype(np.float64) @ M[lay, :]
            Gh += job.xmap[:, k, :].astype(np.float64) @ per_level
        assert np.all(np.abs(Gh - G[:, iw]) <= 1e-5 * scale)


def test_cirsconv_fwhm_matches_oracle(ctx, oracle):
    """cirsconv.f with FWHM > 0 on the device (natural cubic spline, 20-point
    trapezoid per channel) against the oracle's restatement, on the radiance,
    d/dtsurf and every Jacobian row of a spectrum computed at FWHM = 0, with
    channels that need both end extrapolations and a series holding a NaN;
    1e-6 of each series' largest value."""
    kt, cia, job = synth.config2(nwave=200, nlayer=40, nbin=200)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, gt = ctx.cirsrtfg_wave(job)
    series = np.vstack([c[None], gt[None], g.reshape(job.nv, job.nwave)])
    series[3, 57] = np.nan
    fwhm = 2.5
    vconv = (job.vwave[0] + 0.3 + np.arange(0, 78, 1.0)).astype(np.float32)
    got = ctx.cirsconv(job.vwave, series, fwhm, vconv)
    for s in range(series.shape[0]):
        ref = oracle.cirsconv(job.vwave, series[s], fwhm, vconv)
        scale = max(np.max(np.abs(ref)), 1e-30)
        assert np.max(np.abs(got[s] - ref)) <= 1e-6 * scale, s
    same = ctx.cirsconv(job.vwave, series[:1], 0.0, job.vwave)
    assert np.array_equal(same[0], series[0])


@pytest.mark.parametrize("shift", [0.0, 0.13])
def test_pressure_dependent_temperature_grid(ctx, oracle, shift):
    """k-tables with one temperature grid per pressure (NT < 0, TEMP2;
    get_kg.f:143-169, 355-365, 413-423), on table wavenumbers and between
    them: radiance and Jacobian within tolerance of the FP64 oracle, g-bins
    bit-exact with the mixed oracle, and the k values differ from those of a
    single grid."""
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, nbin=16, seed=1002, t2=True)
    assert kt.nt == -15 and kt.tk.shape == (20 * 15,)
    cia = synth.make_cia(1002)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=77, nwave=12, vmr_perturb=0.3)
    j = _off_grid(job, kt, shift) if shift else job
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(j)
        perm, split = ctx.debug_bins(j)
    finally:
        ctx.set_debug(False)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, j.nv) <= JAC_TOL
    (cm, gm, _), (operm, osplit, _) = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_MIXED, debug=True)
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    assert np.array_equal(split, osplit)
    # the same k values read through the first pressure row's grid give another spectrum
    import dataclasses
    kt1 = dataclasses.replace(kt, nt=15, tk=np.ascontiguousarray(kt.tk[::20]))
    ctx.set_ktables(kt1)
    c1, _, _ = ctx.cirsrtfg_wave(j)
    assert not np.array_equal(c1, c)


def test_tables_covering_part_of_the_spectrum(ctx, oracle):
    """A table covers the calculation wavenumbers FINDLOC finds inside
    [VMIN, VMIN + (NPOINT-1) DELV] (read_klist.f:250-265); elsewhere its gas
    has no table (lun = -99, zero k; read_klist.f:341-351), including the
    last wavenumber of a grid shifted past the table's end.  Radiance and
    Jacobian within tolerance of the FP64 oracle; an uncovered gas's scale
    derivative is zero there and not elsewhere."""
    import dataclasses
    kt, cia, _ = synth.config2(nwave=40, nlayer=30, nbin=40)
    ktc = dataclasses.replace(kt, vmin=np.array([600.0, 604.0, 596.0, 600.0], np.float32))
    job = synth.make_job(ktc, synth.ABSORBERS_C2, nlayer=30, seed=31, nwave=40)
    ctx.set_ktables(ktc)
    ctx.set_cia(cia)
    c, g, _ = ctx.cirsrtfg_wave(job)
    c64, g64, _ = oracle.cirsrtfg_wave(ktc, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    G = g.reshape(job.nv, job.nwave)
    L = job.nlayer
    assert np.all(G[L + 1, :10] == 0) and np.all(G[L + 1, 10:] != 0)     # the C2H6 table starts at 604
    assert np.all(G[L + 2, 30:] == 0) and np.all(G[L + 2, :30] != 0)     # the C2H2 table ends at 611.6
    j = copy.deepcopy(job)
    j.vwave = j.vwave + np.float32(0.15)      # the last wavenumber is past the CH4 / NH3 tables' end
    c, g, _ = ctx.cirsrtfg_wave(j)
    c64, g64, _ = oracle.cirsrtfg_wave(ktc, cia, j, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, j.nv) <= JAC_TOL
    assert g.reshape(j.nv, j.nwave)[L + 3, -1] == 0


@pytest.mark.parametrize("delv", [-1.0, 0.0])
def test_irregular_wavenumber_grid(ctx, oracle, delv):
    """k-tables on an irregular grid (DELV <= 0, centres VCEN): DELV < 0
    snaps each wavenumber to the centre nearest in per cent (coincident),
    DELV = 0 weights the centre at or below it and the next by FRACK
    (read_klist.f:266-310, get_kg.f:209-279, 391-393).  Radiance and
    Jacobian within tolerance of the FP64 oracle, g-bins bit-exact with the
    mixed oracle."""
    kt = synth.make_ktables(synth.ABSORBERS_C2, np_=20, nt=15, ng=20, nbin=24, seed=41, irregular=delv)
    cia = synth.make_cia(41)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=40, seed=42, nwave=16)
    job.vwave = (600.0 + 0.4 * (np.arange(16) + 1) + 0.07).astype(np.float32)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(job)
        perm, split = ctx.debug_bins(job)
    finally:
        ctx.set_debug(False)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    (cm, gm, _), (operm, osplit, _) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    assert np.array_equal(split, osplit)
    # below the first centre there is no record at or below the wavenumber (read_klist.f:314-318)
    if delv == 0.0:
        from radtrancode_b200 import cirsradg
        j = copy.deepcopy(job)
        j.vwave = (j.vwave - np.float32(2.0)).astype(np.float32)
        with pytest.raises(cirsradg.RtbError, match="RANGE"):
            ctx.cirsrtfg_wave(j)



def test_several_tables_per_gas(ctx):
    """RTB_KTAB_BY_ID (read_klist.f:247-351): a gas served by several tables
    takes, per wavenumber, the first listed table covering it.  Every table
    split into two overlapping halves gives the run of the whole tables bit
    for bit; of two tables covering the same wavenumbers the first listed
    wins."""
    import dataclasses
    kt, cia, _ = synth.config2(nwave=40, nlayer=30, nbin=40)
    job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=30, seed=51, nwave=40)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, gt0 = ctx.cirsrtfg_wave(job)
    n = kt.ntab
    lo = [kt.table(i)[:22] for i in range(n)]
    hi = [kt.table(i)[18:] for i in range(n)]
    split = dataclasses.replace(
        kt, vmin=np.concatenate([kt.vmin, kt.vmin + np.float32(18) * kt.delv]).astype(np.float32),
        delv=np.concatenate([kt.delv, kt.delv]), nbin=np.full(2 * n, 22, np.int32),
        data=np.concatenate([a.ravel() for a in lo + hi]), gases=list(kt.gases) * 2)
    jb = copy.deepcopy(job)
    jb.ktab = np.full(job.ngas, -1, np.int32)
    jb.ktab[2:] = -2                                   # RTB_KTAB_BY_ID
    ctx.set_ktables(split)
    c, g, gt = ctx.cirsrtfg_wave(jb)
    assert np.array_equal(c, c0) and np.array_equal(g, g0) and np.array_equal(gt, gt0)
    # two whole tables for CH4: the first listed serves it
    twice = dataclasses.replace(
        kt, vmin=np.concatenate([kt.vmin, kt.vmin[:1]]), delv=np.concatenate([kt.delv, kt.delv[:1]]),
        nbin=np.concatenate([kt.nbin, kt.nbin[:1]]),
        data=np.concatenate([kt.data, (kt.table(0) * np.float32(3.0)).ravel()]), gases=list(kt.gases) + [kt.gases[0]])
    ctx.set_ktables(twice)
    c1, _, _ = ctx.cirsrtfg_wave(jb)
    assert np.array_equal(c1, c0)
    j3 = copy.deepcopy(job)
    j3.ktab = job.ktab.copy()
    j3.ktab[2] = n                                     # the tripled CH4 table
    c3, _, _ = ctx.cirsrtfg_wave(j3)
    assert not np.array_equal(c3, c0)
    flipped = dataclasses.replace(
        twice, vmin=twice.vmin[::-1].copy(), delv=twice.delv[::-1].copy(), nbin=twice.nbin[::-1].copy(),
        data=np.concatenate([twice.table(i).ravel() for i in range(n, -1, -1)]), gases=twice.gases[::-1])
    ctx.set_ktables(flipped)
    c4, _, _ = ctx.cirsrtfg_wave(jb)
    assert np.array_equal(c4, c3)
    ctx.set_ktables(kt)


def _para_case(nlayer=30, nwave=12):
    kt, cia, _ = synth.config2(nwave=nwave, nlayer=nlayer, nbin=nwave)
    para = synth.make_para_cia(7)
    job0 = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=nlayer, seed=81, nwave=nwave)
    rng = np.random.default_rng(3)
    hfp = rng.uniform(0.3, 0.9, nlayer)
    hfp[[3, 17]] = -1.0         # fpara < 0: the last tabulated fraction, no para derivative
    hfp[5] = 1.2                # above the table: the last bracket with f = 1
    hfp[8] = 0.1                # below it: the first bracket with f = 0
    return kt, cia, para, synth.with_para_h2(job0, hfp)


def test_para_h2_cia(ctx, oracle):
    """flagh2p = 1 (cirsradg_wave.f:634-661): the para-H2 CIA of
    nparacon_all / fpread_all replaces nciacon, and the para-H2 fraction of
    every level is a state element (DFP).  Radiance and Jacobian within
    tolerance of the FP64 oracle, the g-bins bit-exact with the mixed oracle;
    the para columns vanish for the fpara < 0 layers and not elsewhere."""
    kt, cia, para, job = _para_case()
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_para_cia(para)
    ctx.set_debug(True)
    try:
        c, g, gt = ctx.cirsrtfg_wave(job)
        perm, split = ctx.debug_bins(job)
    finally:
        ctx.set_debug(False)
    cia.para = para
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    (cm, gm, _), (operm, osplit, _) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    G = g.reshape(job.nv, job.nwave)
    rows = G[job.nv - job.npro:]
    zero = np.all(rows == 0, axis=1)
    assert zero[3] and zero[17] and not zero[[0, 1, 5, 8, 20]].any()
    del cia.para
    c0, _, _ = ctx.cirsrtfg_wave(dataclasses.replace(job, flagh2p=0, ld_param=job.ngas + 1,
                                                     xmap=np.asfortranarray(job.xmap[:, :job.ngas + 1, :]),
                                                     nv=job.nv, ld_v=job.nv))
    assert not np.array_equal(c0, c)


def test_para_h2_table_file(ctx, tmp_path):
    """The para-H2 table read from the unformatted file fpread_all reads
    (five framed records) gives the in-memory table's run bit for bit."""
    kt, cia, para, job = _para_case(nlayer=20, nwave=6)
    path = tmp_path / "para.tab"
    with open(path, "wb") as fh:
        for rec in (para.temps, para.fp, para.kh2h2, para.kh2he, para.kcia5):
            b = np.asarray(rec, np.float32).tobytes()
            n = np.array([len(b)], np.int32).tobytes()
            fh.write(n + b + n)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_para_cia(para)
    a = ctx.cirsrtfg_wave(job)
    ctx.load_para_cia(str(path), para.dnu2, para.ipara)
    b = ctx.cirsrtfg_wave(job)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def _emission_case(case):
    kt, cia, _ = synth.config2(nwave=5, nlayer=24, nbin=5)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=24, seed=23, nwave=5)
    job.vem = np.array([500.0, 1500.0], np.float32)
    job.emissivity = np.array([0.9, 0.7], np.float32)
    if case.startswith("imod18"):
        job.imod[:] = 18
    if case in ("imod18_surface", "imod18_iform3", "imod3_iform3"):
        job.tsurf = 175.0
    if case.endswith("iform3"):
        job.iform, job.radius1, job.radextra = 3, 71492.0, 40.0
    if case == "paths_18_and_3":
        L = job.nlayer
        lay = np.zeros((L, 2), np.int32, order="F")
        lay[:, 0] = lay[:, 1] = job.layinc[:L, 0]
        sc = np.ones((L, 2), np.float32, order="F")
        sc[:, 1] = 1.5
        em = np.zeros((L, 2), np.float32, order="F")
        em[:, 0] = em[:, 1] = job.emtemp[:L, 0]
        job = dataclasses.replace(job, npath=2, layinc=lay, scale=sc, emtemp=em, nlayin=np.array([L, L], np.int32),
                                  imod=np.array([18, 3], np.int32), tsurf=160.0)
    return kt, cia, job


@pytest.mark.parametrize("case", ["imod18", "imod18_surface", "imod18_iform3", "imod3_iform3", "paths_18_and_3"])
def test_hemispherical_emission_and_total_flux(ctx, oracle, case):
    """IMOD 18 (cirsradg_wave.f:1116-1225: the flux integrated over the
    hemisphere through e3interp's E3 table; the Jacobian by the E3-gradient
    recurrence, evaluated on the device as one backward sum) and iform = 3
    (the total flux of the planet, cirsradg_wave.f:913-929 and 1136-1152):
    radiance, Jacobian and surface-temperature gradient within tolerance of
    the FP64 oracle."""
    e3 = synth.make_e3_table()
    kt, cia, job = _emission_case(case)
    ctx.set_e3_table(e3)
    c, g, gt = _run(ctx, kt, cia, job)
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=e3)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.npath * job.nv) <= JAC_TOL
    if job.tsurf > 0:
        assert np.max(np.abs(gt - gt64)) <= RAD_TOL * np.max(np.abs(gt64))
    if case.endswith("iform3"):
        base = dataclasses.replace(job, iform=0)
        c0, _, _ = ctx.cirsrtfg_wave(base)
        assert np.max(c / c0) > 100.0


def test_e3_table_file_and_missing_table(tmp_path):
    """The E3 table read from e3interp's text file gives the in-memory
    table's run bit for bit; an IMOD 18 path without a table is refused."""
    from radtrancode_b200 import cirsradg
    e3 = synth.make_e3_table()
    path = tmp_path / "e3tab.dat"
    synth.write_e3_table(path, e3)
    kt, cia, job = _emission_case("imod18_surface")
    with cirsradg.Context(0) as c2:
        c2.set_ktables(kt)
        c2.set_cia(cia)
        with pytest.raises(cirsradg.RtbError, match="E3"):
            c2.cirsrtfg_wave(job)
        c2.set_e3_table(e3)
        a = c2.cirsrtfg_wave(job)
        c2.load_e3_table(str(path))
        b = c2.cirsrtfg_wave(job)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_dust_continuum(ctx, oracle):
    """Dust (cirsradg_wave.f:550-575) with two types whose profile scales are
    state elements (DCO): radiance and Jacobian within tolerance of the FP64
    oracle; in a batch beside dust-free spectra each gets its own result."""
    kt, cia, _ = synth.config2(nwave=6, nlayer=30, nbin=6)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=30, seed=31, nwave=6)
    jd = synth.with_dust(job, 2, seed=4)
    c, g, gt = _run(ctx, kt, cia, jd)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, jd, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, jd.nv) <= JAC_TOL
    assert np.all(g.reshape(jd.nv, -1)[job.nv:] != 0)
    c0, g0, _ = ctx.cirsrtfg_wave(job)
    outs = ctx.cirsrtfg_wave_batch([job, jd, job])
    assert np.array_equal(outs[1][0], c) and np.array_equal(outs[1][1], g)
    assert np.array_equal(outs[0][0], c0) and np.array_equal(outs[2][1], g0)


@pytest.mark.parametrize("case", ["inlte1", "inlte2", "inlte1_imod18"])
def test_nlte_emission_temperatures(ctx, oracle, case):
    """Non-LTE emission temperatures (calc_nlte_t.f, cirsradg_wave.f:933-935
    and 1156-1158) on IMOD 3 and IMOD 18 paths: radiance, Jacobian and
    surface gradient within tolerance of the FP64 oracle."""
    e3 = synth.make_e3_table()
    kt, cia, _ = synth.config2(nwave=5, nlayer=30, nbin=5)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=30, seed=37, nwave=5)
    job.tsurf = 170.0
    if case.startswith("inlte1"):
        job = dataclasses.replace(job, inlte=1, nlte_k1=1e-10, nlte_A=5e5)
    else:
        job = dataclasses.replace(job, inlte=2)
    if case.endswith("imod18"):
        job.imod[:] = 18
    ctx.set_e3_table(e3)
    c, g, gt = _run(ctx, kt, cia, job)
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=e3)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    assert np.max(np.abs(gt - gt64)) <= RAD_TOL * np.max(np.abs(gt64))


@pytest.mark.parametrize("case", ["iform1_imod3", "iform1_imod18", "iform4_imod0", "iform1_no_star"])
def test_stellar_spectrum_forms(ctx, oracle, case):
    """iform 1 (planet flux over the star's, cirsradg_wave.f:913-929 and
    1136-1152) and iform 4 (IMOD 0 transmission times the star's flux at
    dist, :861-879) with init_solar_wave's table, and iform 1 without one:
    radiance and Jacobian within tolerance of the FP64 oracle."""
    from radtrancode_b200 import cirsradg
    e3 = synth.make_e3_table()
    ss = synth.make_stellar_spectrum(550.0, 700.0, npt=301, descending=case == "iform4_imod0")
    kt, cia, _ = synth.config2(nwave=5, nlayer=30, nbin=5)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=30, seed=41, nwave=5)
    job.tsurf = 165.0
    if case.startswith("iform1"):
        job = dataclasses.replace(job, iform=1, radius1=71492.0, radextra=20.0)
    else:
        job = dataclasses.replace(job, iform=4, dist=5.2, imod=np.zeros_like(job.imod))
    if case == "iform1_imod18":
        job.imod[:] = 18
    with cirsradg.Context(0) as c2:
        c2.set_ktables(kt)
        c2.set_cia(cia)
        c2.set_e3_table(e3)
        if case != "iform1_no_star":
            c2.set_stellar_spectrum(ss)
        c, g, gt = c2.cirsrtfg_wave(job)
    star = None if case == "iform1_no_star" else ss
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, e3=e3, solar=star)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL


def test_stellar_spectrum_file(tmp_path):
    """The stellar spectrum read from init_solar_wave's text file gives the
    in-memory table's run bit for bit; a file in the other wavespace is
    refused."""
    from radtrancode_b200 import cirsradg
    ss = synth.make_stellar_spectrum(550.0, 700.0, npt=301)
    path = tmp_path / "star.dat"
    synth.write_stellar_file(path, ss, ispace=0)
    kt, cia, _ = synth.config2(nwave=5, nlayer=30, nbin=5)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=30, seed=43, nwave=5)
    job = dataclasses.replace(job, iform=1, radius1=71492.0)
    with cirsradg.Context(0) as c2:
        c2.set_ktables(kt)
        c2.set_cia(cia)
        c2.set_stellar_spectrum(ss)
        a = c2.cirsrtfg_wave(job)
        c2.load_stellar_spectrum(str(path), 0)
        b = c2.cirsrtfg_wave(job)
        with pytest.raises(cirsradg.RtbError, match="wavespace"):
            c2.load_stellar_spectrum(str(path), 1)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def _many_paths(npath=10, nlayer=24, nwave=5):
    """npath paths over one atmosphere: nadir-like paths at growing air
    masses (IMOD 3 through the column, 0 and 1 through its upper half, in
    turn) and every fourth a limb path down to
    a tangent layer and up again (cirsradg_wave.f:983-988 skips its
    surface term)."""
    kt, cia, _ = synth.config2(nwave=nwave, nlayer=nlayer, nbin=nwave)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=nlayer, seed=51, nwave=nwave)
    L = nlayer
    ld = 2 * L
    lay = np.zeros((ld, npath), np.int32, order="F")
    sc = np.zeros((ld, npath), np.float32, order="F")
    em = np.ones((ld, npath), np.float32, order="F")
    nl = np.zeros(npath, np.int32)
    imod = np.zeros(npath, np.int32)
    for p in range(npath):
        if p % 4 == 3:
            tang = 4 + p // 4
            half = np.arange(L, tang - 1, -1)
            path = np.concatenate([half, half[::-1]])
            imod[p] = 3
        else:
            imod[p] = (3, 0, 1)[p % 3]
            # transmission and absorption paths through the upper half only: over
            # the whole column 1 - A falls below 1e-13, where even the FP64
            # oracle's 1 - (1 - T) loses digits
            path = job.layinc[:L, 0].copy() if imod[p] == 3 else job.layinc[:L // 2, 0].copy()
        n = path.size
        lay[:n, p] = path
        sc[:n, p] = 1.0 + 0.15 * p
        em[:n, p] = job.temp[path - 1]
        nl[p] = n
    pad = lambda a, fill: np.asfortranarray(np.concatenate([a[:L], np.full((ld - L,) + a.shape[1:], fill, a.dtype)]))
    job = dataclasses.replace(job, npath=npath, ld_lay=ld, layinc=lay, scale=sc, emtemp=em, nlayin=nl, imod=imod,
                              press=job.press, temp=job.temp, delh=job.delh, pp=pad(job.pp, 0),
                              amount=pad(job.amount, 0), dte=pad(job.dte, 0), dam=pad(job.dam, 0))
    job.tsurf = 160.0
    return kt, cia, job


def test_many_paths_in_groups(ctx, oracle):
    """A spectrum of 10 paths (limb sets run many tangent paths per
    spectrum; the device takes them in groups of four): every path's
    radiance, Jacobian and surface gradient within tolerance of the FP64
    oracle, and the same result alone and in a batch beside a one-path
    spectrum."""
    kt, cia, job = _many_paths()
    c, g, gt = _run(ctx, kt, cia, job)
    c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.npath * job.nv) <= JAC_TOL
    assert np.max(np.abs(gt - gt64)) <= RAD_TOL * np.max(np.abs(gt64))
    one = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=24, seed=52, nwave=5)
    c1, g1, _ = ctx.cirsrtfg_wave(one)
    outs = ctx.cirsrtfg_wave_batch([one, job, one])
    assert np.array_equal(outs[1][0], c) and np.array_equal(outs[1][1], g) and np.array_equal(outs[1][2], gt)
    assert np.array_equal(outs[0][0], c1) and np.array_equal(outs[2][1], g1)


@pytest.mark.parametrize("iray", [2, 3])
def test_rayleigh_venus_and_air(ctx, oracle, iray):
    """IRAY 2 (Venus, per wavenumber on the host) and 3 (air at each
    layer's P and T, on the device): radiance and Jacobian within tolerance
    of the FP64 oracle, and in a batch beside IRAY 1 and 0 spectra each gets
    its own result."""
    kt, cia, _ = synth.config2(nwave=6, nlayer=30, nbin=6)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=30, seed=61, nwave=6)
    j = dataclasses.replace(job, iray=iray)
    c, g, _ = _run(ctx, kt, cia, j)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, j.nv) <= JAC_TOL
    j1 = dataclasses.replace(job, iray=1)
    outs = ctx.cirsrtfg_wave_batch([j1, j, job])
    assert np.array_equal(outs[1][0], c) and np.array_equal(outs[1][1], g)
    assert np.array_equal(outs[0][0], ctx.cirsrtfg_wave(j1)[0]) and np.array_equal(outs[2][0], ctx.cirsrtfg_wave(job)[0])
