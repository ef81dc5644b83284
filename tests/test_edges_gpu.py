"""Edge cases of the device forward model: the largest NG the device takes
(bit-exact g-bins at NG = 22) and the first one it refuses, a gas whose
k-table is all zero (the reference's skip branches, get_kg.f:228-250 and
noverlapg.f:88-108), one-wavenumber spectra, the smallest emission path, and
empty or malformed calls."""
import copy

import numpy as np
import pytest

from radtrancode_b200 import cirsradg, synth
from tests.helpers import JAC_TOL, RAD_TOL, assignment, jac_err, rad_err

pytestmark = pytest.mark.gpu


def _tables_ng(ng, seed=77, nbin=6):
    return synth.make_ktables(synth.ABSORBERS_C2[:3], np_=20, nt=15, ng=ng, vmin=600.0, delv=0.4, nbin=nbin,
                              seed=seed)


def test_largest_device_ng_bins_bit_exact(ctx, oracle):
    kt = _tables_ng(22)
    cia = synth.make_cia(1)
    job = synth.make_job(kt, synth.ABSORBERS_C2[:3], nlayer=30, seed=78, nwave=6, vmr_perturb=0.3)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_debug(True)
    try:
        c, g, _ = ctx.cirsrtfg_wave(job)
        perm, split = ctx.debug_bins(job)
    finally:
        ctx.set_debug(False)
    (cm, gm, _), (operm, osplit, _) = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_MIXED, debug=True)
    assert np.array_equal(assignment(perm, split, kt.ng), assignment(operm, osplit, kt.ng))
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL


def test_ng_beyond_device_range_is_refused(ctx):
    kt = _tables_ng(23)
    job = synth.make_job(kt, synth.ABSORBERS_C2[:3], nlayer=10, seed=79, nwave=2)
    ctx.set_ktables(kt)
    with pytest.raises(cirsradg.RtbError, match="UNSUPPORTED"):
        ctx.cirsrtfg_wave(job)


def test_zero_table_gas_matches_the_gas_left_out(ctx):
    kt, cia, _ = synth.config2(nwave=6, nlayer=20, nbin=6)
    kt_z = copy.deepcopy(kt)
    kt_z.table(1)[:] = 0.0
    kt_1 = synth.KTables(kt.np_, kt.nt, kt.ng, kt.lnp, kt.tk, kt.g_ord, kt.delg, kt.vmin[:1], kt.delv[:1],
                         kt.nbin[:1], kt.table(0).ravel().copy(), kt.gases[:1])
    job_a = synth.make_job(kt_z, [synth.CH4, synth.C2H6], nlayer=20, seed=5, nwave=6)
    job_b = synth.make_job(kt_1, [synth.CH4], nlayer=20, seed=5, nwave=6)
    ctx.set_cia(cia)
    ctx.set_ktables(kt_z)
    ca, ga, _ = ctx.cirsrtfg_wave(job_a)
    ctx.set_ktables(kt_1)
    cb, gb, _ = ctx.cirsrtfg_wave(job_b)
    assert np.array_equal(ca, cb)
    assert np.array_equal(ga.reshape(job_a.nv, -1)[:job_b.nv], gb.reshape(job_b.nv, -1))


def test_one_wavenumber_and_two_layer_spectra(ctx, oracle):
    kt, cia, _ = synth.config2(nwave=4, nlayer=20, nbin=4)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    for nlayer, nwave in ((2, 1), (2, 4), (20, 1)):
        job = synth.make_job(kt, synth.ABSORBERS_C2, nlayer=nlayer, seed=80 + nlayer, nwave=nwave,
                             vmr_perturb=0.3)
        c, g, _ = ctx.cirsrtfg_wave(job)
        c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
        assert rad_err(c, c64) <= RAD_TOL
        assert jac_err(g, g64, job.nv) <= JAC_TOL


def test_empty_and_malformed_calls(ctx):
    kt, cia, job = synth.config1()
    ctx.set_ktables(kt)
    with pytest.raises(cirsradg.RtbError, match="ARG"):
        ctx.cirsrtfg_wave_batch([])
    j = copy.deepcopy(job)
    j.nwave = 0
    with pytest.raises(cirsradg.RtbError, match="ARG"):
        ctx.cirsrtfg_wave(j)
    j = copy.deepcopy(job)
    j.layinc[0, 0] = job.nlayer + 1                      # a path through a layer that does not exist
    with pytest.raises(cirsradg.RtbError, match="LIMIT"):
        ctx.cirsrtfg_wave(j)


def test_largest_profile_and_its_limit(ctx, oracle):
    """200 layers, each its own profile level: NPRO = MAXPRO of arrdef.f,
    the largest profile the reference holds, against the FP64 oracle; one
    level more is refused with RTB_ERR_LIMIT (check_limits.f)."""
    kt, cia, _ = synth.config2(nwave=2, nlayer=20, nbin=2)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    job = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=200, seed=88, nwave=2)
    assert job.npro == 200
    c, g, _ = ctx.cirsrtfg_wave(job)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64, nthreads=2)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    big = synth.make_job(kt, [synth.CH4, synth.NH3], nlayer=201, seed=89, nwave=1)
    with pytest.raises(cirsradg.RtbError, match="LIMIT"):
        ctx.cirsrtfg_wave(big)


def test_ngascon_switches_refused_or_zero(ctx):
    """The NGASCON gate (ngascon.f:132-318 via cirsradg_wave.f:590-611).
    A /GASCONDEF/ switch whose gas is in the atmosphere would add a gas
    continuum the library does not compute: refused, naming the switch.  A
    switch whose gas is absent contributes nothing in the reference either:
    the spectrum is bit-identical to the all-off run."""
    kt, cia, job = synth.config2(nwave=4, nlayer=20, nbin=4)   # CH4 (6), C2H6 (27), C2H2 (26), NH3 (11)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, t0 = ctx.cirsrtfg_wave(job)
    refused = {(0, 1, 0, 0, 0): "ICH4", (0, 0, 1, 0, 0): "INH3", (0, 0, 0, 0, 1): "iuvscat bit 1",
               (0, 0, 0, 0, 4): "iuvscat bit 4", (0, 0, 0, 0, 8): "iuvscat bit 8", (0, 0, 0, 0, 32): "iuvscat bit 32"}
    for sw, name in refused.items():
        j = copy.deepcopy(job)
        j.gascon = sw
        with pytest.raises(cirsradg.RtbError, match="UNSUPPORTED") as e:
            ctx.cirsrtfg_wave(j)
        assert name in str(e.value)
    # switches of absent gases (H2O, O3, PH3, C4H2, CO, GeH4, H2O UV, C3H8), and CH4 of another isotope
    for sw in ((1, 0, 0, 0, 0), (2, 0, 0, 0, 0), (0, 0, 0, 1, 0), (0, 0, 0, 0, 2 | 16 | 64 | 128 | 256 | 512)):
        j = copy.deepcopy(job)
        j.gascon = sw
        c, g, t = ctx.cirsrtfg_wave(j)
        assert np.array_equal(c, c0) and np.array_equal(g, g0) and np.array_equal(t, t0)
    j = copy.deepcopy(job)
    j.isogas = job.isogas.copy()
    j.isogas[list(job.idgas).index(6)] = 2            # 13CH4: ICH4 applies to isotopes 0 and 1 only
    j.gascon = (0, 1, 0, 0, 0)
    c, g, t = ctx.cirsrtfg_wave(j)
    j.gascon = (0, 0, 0, 0, 0)
    c2, g2, t2 = ctx.cirsrtfg_wave(j)
    assert np.array_equal(c, c2) and np.array_equal(g, g2)
