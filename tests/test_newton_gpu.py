"""GPU parity tests of the Newton step, the cost function, the SPD inverse
and the retrieval loop against the oracle (oracle/newton_oracle.cpp,
oracle/coreret_oracle.cpp), all through the C ABI.

Tolerances (stated per result):
  Newton step  max_i |x_gpu - x_ref| <= tol * max_i |x_ref - xa| + 4 ulp(x_ref),
               tol = 1e-3 on tensor cores with one refinement step, 1e-6 all-FP64
  phi, chisq   relative 1e-6 (FP64 sums, REAL result)
  Sa^-1        relative to max |Sa^-1|: 1e-10
  retrieval    same number of iterations, forward evaluations and stop rule as
               the oracle; |x_gpu - x_ref| <= 1e-3 prior sigma; phi relative 1e-3
"""
import numpy as np
import pytest

from radtrancode_b200 import synth

pytestmark = pytest.mark.gpu

TOL_STEP = {0: 1e-3, 1: 1e-6}


def _case(oracle, kt, cia, absorbers, nlayer, seed, nwave=None, nthreads=1):
    case = synth.make_retrieval(kt, absorbers, nlayer=nlayer, seed=seed, nwave=nwave)
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=nthreads)
    return synth.observe(case, y_true, seed=seed + 1)


@pytest.fixture(scope="module")
def c1(oracle):
    kt, cia, _ = synth.config1()
    return kt, cia, [_case(oracle, kt, cia, [synth.CH4], 40, s) for s in (5, 7, 9)]


@pytest.fixture(scope="module")
def c2s(oracle):
    kt, cia, _ = synth.config2()
    return kt, cia, [_case(oracle, kt, cia, synth.ABSORBERS_C2, 120, 21, nwave=300, nthreads=8)]


def _newton_inputs(oracle, kt, cia, cases, shift):
    rows = []
    for i, case in enumerate(cases):
        xn = case.x_true.copy()
        xn[:case.job.nlayer] += np.float32(shift * (i + 1))
        yn, kk = oracle.forward_state(kt, cia, case, xn, nthreads=8)
        sai, ic = oracle.dinvertm(case.sa)
        rows.append((kk, case.sei, sai, case.xa, xn, case.y, yn))
    return [np.stack(a) for a in zip(*rows)]


def _ulp(x):
    return np.spacing(np.abs(x).astype(np.float32))


@pytest.mark.parametrize("hess", [0, 1])
@pytest.mark.parametrize("which", ["c1", "c2s"])
def test_newton_step_matches_reference_algebra(ctx, oracle, c1, c2s, hess, which):
    kt, cia, cases = c1 if which == "c1" else c2s
    kk, sei, sai, xa, xn, y, yn = _newton_inputs(oracle, kt, cia, cases, 2.0)
    ref = np.stack([oracle.newton_step(*a) for a in zip(kk, sei, sai, xa, xn, y, yn)])
    ctx.set_newton_mode(hess, 1)
    try:
        x, nonpd, resid = ctx.newton_step_batch(kk, sei, sai, xa, xn, y, yn)
    finally:
        ctx.set_newton_mode(0, 1)
    assert not nonpd.any()
    for r in range(len(ref)):
        step = np.max(np.abs(ref[r] - xa[r]))
        assert np.all(np.abs(x[r] - ref[r]) <= TOL_STEP[hess] * step + 4 * _ulp(ref[r])), r
    assert np.all(resid < (1e-4 if hess == 0 else 1e-10))


def test_drop_in_gain_matrix_and_calcnextxn(ctx, oracle, c1, c2s):
    """The reference's interface (D and AA returned, then calcnextxn) against
    the oracle's dense restatement; FP64 throughout, so 1e-9 of the largest
    entry for D and AA and REAL rounding for x_out."""
    for kt, cia, cases in (c1, c2s):
        kk, sei, sai, xa, xn, y, yn = _newton_inputs(oracle, kt, cia, cases[:1], 2.0)
        dd, aa, nonpd = ctx.calc_gain_matrix(kk[0], sai[0], sei[0])
        dd_r, aa_r = oracle.gain_matrix(kk[0], sei[0], sai[0])
        assert nonpd == 0
        assert np.max(np.abs(dd - dd_r)) <= 1e-9 * np.max(np.abs(dd_r))
        assert np.max(np.abs(aa - aa_r)) <= 1e-9 * np.max(np.abs(aa_r))
        x = ctx.calcnextxn(xa[0], xn[0], y[0], yn[0], dd, aa)
        x_r = oracle.calcnextxn(xa[0], xn[0], y[0], yn[0], dd_r, aa_r)
        step = np.max(np.abs(x_r - xa[0]))
        assert np.all(np.abs(x - x_r) <= 1e-6 * step + 2 * _ulp(x_r))


def test_calc_serr_matches_oracle(ctx, oracle, c2s):
    """Final error covariances (calc_serr.f) from the device D and AA, against
    the oracle's restatement on the same D and AA: REAL outputs within 1e-5 of
    the largest entry."""
    kt, cia, cases = c2s
    kk, sei, sai, xa, xn, y, yn = _newton_inputs(oracle, kt, cia, cases[:1], 2.0)
    dd, aa, _ = ctx.calc_gain_matrix(kk[0], sai[0], sei[0])
    sx = cases[0].sa.astype(np.float32)
    se = (1.0 / sei[0]).astype(np.float32)
    got = ctx.calc_serr(sx, se, dd, aa)
    ref = oracle.calc_serr(sx, se, dd, aa)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) <= 1e-5 * np.max(np.abs(r))
    st, sn, sm = got
    assert np.allclose(st, sn + sm, rtol=1e-5, atol=1e-5 * np.max(np.abs(st)))


def test_refinement_reduces_residual(ctx, oracle, c2s):
    kt, cia, cases = c2s
    args = _newton_inputs(oracle, kt, cia, cases, 1.0)
    res = []
    try:
        for refine in (0, 1, 2):
            ctx.set_newton_mode(0, refine)
            res.append(ctx.newton_step_batch(*args)[2][0])
    finally:
        ctx.set_newton_mode(0, 1)
    assert res[1] < res[0] and res[2] < res[1]


def test_phiret_matches_oracle(ctx, oracle, c1):
    kt, cia, cases = c1
    kk, sei, sai, xa, xn, y, yn = _newton_inputs(oracle, kt, cia, cases, 0.5)
    phi, chisq = ctx.calc_phiret_batch(y, yn, sei, xn, xa, sai)
    for r in range(len(phi)):
        p, c = oracle.calc_phiret(y[r], yn[r], sei[r], xn[r], xa[r], sai[r])
        assert abs(phi[r] - p) <= 1e-6 * abs(p)
        assert abs(chisq[r] - c) <= 1e-6 * abs(c)


def test_spd_inverse_matches_dinvertm(ctx, oracle, c2s):
    _, _, cases = c2s
    sa = np.stack([cases[0].sa, cases[0].sa * 2.0])
    inv, nonpd = ctx.spd_inverse_batch(sa)
    assert not nonpd.any()
    for r in range(2):
        ref, ic = oracle.dinvertm(sa[r])
        assert ic == 0
        assert np.max(np.abs(inv[r] - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_spd_inverse_flags_non_positive_pivot(ctx):
    a = np.diag([1.0, -2.0, 3.0])[None]
    inv, nonpd = ctx.spd_inverse_batch(a)
    assert nonpd[0] == 1
    assert np.isfinite(inv).all()


@pytest.mark.parametrize("hess", [1, 0])
def test_retrieve_batch_matches_oracle(ctx, oracle, c1, hess):
    kt, cia, cases = c1
    cases = [c for c in cases]
    far = synth.make_retrieval(kt, [synth.CH4], nlayer=40, seed=9)
    far.y = cases[2].y
    far.x0 = far.xa.copy()
    far.x0[-1] = 8.0                     # rejections on the way (coreret.f:1060-1064)
    cases.append(far)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_newton_mode(hess, 1)
    try:
        got = ctx.retrieve_batch(cases, kiter=10, phlimit=0.1)
    finally:
        ctx.set_newton_mode(0, 1)
    for case, g in zip(cases, got):
        ref, tr = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1)
        assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"],
                                                                   ref["forwards"])
        sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
        assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
        assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]


def test_retrieve_scale_model_2_and_gas_profile_match_oracle(ctx, oracle):
    """A linear (model 2) scale of CH4 and a log-vmr layer profile of NH3
    (model 0 for a gas) beside the temperatures: same iterations, forward
    evaluations and stop rule as the oracle's coreret loop, states within
    1e-3 prior sigma, cost within 1e-3."""
    kt, cia, _ = synth.config2()
    case = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=40, seed=41, nwave=120, scale_model=[2],
                                profile=[1])
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    synth.observe(case, y_true, seed=42)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ref, tr = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    for hess in (1, 0):
        ctx.set_newton_mode(hess, 1)
        try:
            g = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
        finally:
            ctx.set_newton_mode(0, 1)
        assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"],
                                                                   ref["forwards"])
        assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
        assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]


def test_level_state_retrieval_relayers_every_state(ctx, oracle):
    """The level-state model: the temperatures of 41 profile levels and two
    log gas scales, every evaluated state re-layered into 40 Curtis-Godson
    layers on a 20-degree path (rtb_layerg inside the loop, as gsetrad +
    subpathg re-layer the .prf each iteration).  Same iterations, forward
    evaluations and stop rule as the oracle's coreret loop over its own
    layering, states within 1e-3 prior sigma, cost within 1e-3; the same
    result alone and beside a second retrieval."""
    kt, cia, _ = synth.config2()
    cases = []
    for seed in (61, 71):
        case = synth.make_level_retrieval(kt, [synth.CH4, synth.NH3], npro=41, nlay=40, seed=seed, nwave=120,
                                          angle=20.0)
        y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
        synth.observe(case, y_true, seed=seed + 1)
        cases.append(case)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    both = ctx.retrieve_batch(cases, kiter=10, phlimit=0.1)
    alone = ctx.retrieve_batch(cases[:1], kiter=10, phlimit=0.1)[0]
    for case, g in zip(cases, both):
        ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
        assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"],
                                                                   ref["forwards"])
        sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
        assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
        assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]
    assert np.array_equal(alone["x"], both[0]["x"]) and alone["phi"] == both[0]["phi"]


def test_retrieve_batch_result_independent_of_batch(ctx, c1):
    kt, cia, cases = c1
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    together = ctx.retrieve_batch(cases, kiter=10)
    for case, t in zip(cases, together):
        alone = ctx.retrieve_batch([case], kiter=10)[0]
        assert np.array_equal(alone["x"], t["x"])
        assert np.array_equal(alone["yn"], t["yn"])
        assert (alone["phi"], alone["iterations"]) == (t["phi"], t["iterations"])


def _triangles(vc, a=1.6, b=0.7):
    pts = [c + np.array([-a, -b, 0.0, b, a], np.float32) for c in vc]
    return synth.Channels(vconv=vc, vcen=vc.copy(), nsub=np.full(len(vc), 5, np.int32),
                          vfil=np.concatenate(pts).astype(np.float32),
                          fil=np.tile(np.array([0.0, 0.5, 1.0, 0.5, 0.0], np.float32), len(vc)))


@pytest.mark.parametrize("mode", ["fwhm", "filter", "level_fwhm"])
def test_retrieval_on_convolved_channels(ctx, oracle, mode):
    """Retrievals measured on instrument channels (FWHM > 0, cirsconv's
    spline-interpolated boxcar; FWHM < 0, filter functions): every evaluated
    spectrum and Jacobian row is convolved on the device (cirsrtfg_wave.f:
    520-560) before the cost and the Newton step.  Same iterations, forward
    evaluations and stop rule as the oracle's coreret loop over the cirsconv
    of its own forward model, states within 1e-3 prior sigma, cost within
    1e-3; beside a calculation-grid retrieval in one batch, each gets the
    result it gets alone."""
    kt, cia, _ = synth.config2()
    if mode == "level_fwhm":
        base = synth.make_level_retrieval(kt, [synth.CH4, synth.NH3], npro=31, nlay=30, seed=91, nwave=300)
    else:
        base = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=30, seed=81, nwave=300)
    vc = (base.job.vwave[0] + 2.1 + np.arange(0, 112, 0.8)).astype(np.float32)
    fwhm, ch = (-1.0, _triangles(vc)) if mode == "filter" else (1.6, synth.Channels(vconv=vc))
    case = synth.with_channels(base, fwhm, ch)
    assert case.ny == len(vc) and case.ny > case.nx
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    synth.observe(case, y_true, seed=82)
    y_plain, _ = oracle.forward_state(kt, cia, base, base.x_true, nthreads=8)
    synth.observe(base, y_plain, seed=83)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    both = ctx.retrieve_batch([case, base], kiter=10, phlimit=0.1)
    alone = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
    ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
    g = both[0]
    assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"], ref["forwards"])
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
    assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]
    assert g["yn"].shape == (case.ny,)
    assert np.array_equal(alone["x"], g["x"]) and alone["phi"] == g["phi"]
    ref_b, _ = oracle.retrieve(kt, cia, base, kiter=10, phlimit=0.1, nthreads=8)
    assert np.all(np.abs(both[1]["x"] - ref_b["x"]) <= 1e-3 * np.sqrt(np.diag(base.sa)).astype(np.float32))


def test_retrieval_with_dust_background(ctx, oracle):
    """A layer-state retrieval through a fixed dust background (two dust
    types, their xmap columns zero): same iterations, forward evaluations
    and stop rule as the oracle's coreret loop, states within 1e-3 prior
    sigma, cost within 1e-3."""
    import dataclasses
    kt, cia, _ = synth.config2()
    case = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=30, seed=95, nwave=150)
    case = dataclasses.replace(case, job=synth.with_dust(case.job, 2, seed=5, state=False))
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    synth.observe(case, y_true, seed=96)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    g = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
    ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
    assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"], ref["forwards"])
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
    assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]


@pytest.mark.parametrize("mode", ["three_paths", "two_paths_channels"])
def test_retrieval_over_several_paths(ctx, oracle, mode):
    """One footprint seen along several paths at once (air masses 1, 1.4,
    2; y holds one spectrum per path, path after path, as cirsrtfg_wave
    packs them), on the calculation grid or on channels: same iterations,
    forward evaluations and stop rule as the oracle's coreret loop, states
    within 1e-3 prior sigma, cost within 1e-3."""
    kt, cia, _ = synth.config2()
    case = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=30, seed=61, nwave=150)
    if mode == "two_paths_channels":
        vc = (case.job.vwave[0] + 2.1 + np.arange(0, 55, 0.8)).astype(np.float32)
        case = synth.with_channels(case, 1.6, synth.Channels(vconv=vc))
        case = synth.with_paths(case, [1.0, 1.8])
    else:
        case = synth.with_paths(case, [1.0, 1.4, 2.0])
    assert case.ny == case.job.npath * case.job.nconv
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    synth.observe(case, y_true, seed=62)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    g = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
    ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
    assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"], ref["forwards"])
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
    assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]
    assert g["yn"].shape == (case.ny,)


def test_retrieval_of_total_planet_flux(ctx, oracle):
    """A retrieval on the hemispherically integrated total flux of the planet
    (IMOD 18 with iform 3, the extended kernel in the loop): same
    iterations, forward evaluations and stop rule as the oracle's coreret
    loop, states within 1e-3 prior sigma, cost within 1e-3."""
    import dataclasses
    kt, cia, _ = synth.config2()
    e3 = synth.make_e3_table()
    case = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=30, seed=61, nwave=150)
    job = dataclasses.replace(case.job, imod=np.full_like(case.job.imod, 18), iform=3, radius1=71492.0)
    noise = 2e-7                       # fluxes near 5e-4 (x 1e-18 of W (cm-1)-1)
    case = dataclasses.replace(case, job=job, sei=np.full(case.ny, 1.0 / noise ** 2))
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8, e3=e3)
    synth.observe(case, y_true, seed=62, noise=noise)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    ctx.set_e3_table(e3)
    g = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
    ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8, e3=e3)
    assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"], ref["forwards"])
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
    assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]


def test_retrieval_of_dust_scales(ctx, oracle):
    """Two dust types whose column profiles are retrieved as log scales
    beside the temperatures and gas scales (model 3 on an aerosol,
    subprofretg.f:735-750; their Jacobian through DCO): same iterations,
    forward evaluations and stop rule as the oracle's coreret loop, states
    within 1e-3 prior sigma, cost within 1e-3."""
    kt, cia, _ = synth.config2()
    base = synth.make_retrieval(kt, [synth.CH4, synth.NH3], nlayer=30, seed=61, nwave=150)
    case = synth.with_dust_scales(base, 2, seed=7)
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    synth.observe(case, y_true, seed=62)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    g = ctx.retrieve_batch([case], kiter=10, phlimit=0.1)[0]
    ref, _ = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1, nthreads=8)
    assert (g["converged"], g["iterations"], g["forwards"]) == (ref["converged"], ref["iterations"], ref["forwards"])
    sig = np.sqrt(np.diag(case.sa)).astype(np.float32)
    assert np.all(np.abs(g["x"] - ref["x"]) <= 1e-3 * sig)
    assert abs(g["phi"] - ref["phi"]) <= 1e-3 * ref["phi"]
