"""Layering (f1): LAYERG (radtran/path/layerg.f:146-458) and the nadir
thermal path of ATMG (radtran/path/atmg.f:250-373).  CPU: the oracle's
restatement against the physics it must satisfy and against itself across
layer types.  GPU: rtb_layerg against the oracle, and a level profile taken
through the device layering into the forward model against the FP64 oracle
forward model at the radiance and Jacobian tolerances."""
import numpy as np
import pytest

from radtrancode_b200 import synth
from tests.helpers import JAC_TOL, RAD_TOL, jac_err, rad_err

FLOATS = ("baseh", "delh", "basep", "baset", "press", "temp", "totam", "laysf", "amount", "pp", "dte", "dam", "dco",
          "scale", "emtemp")


def _profile(npro=81, seed=7):
    return synth.make_profile(synth.ABSORBERS_C2, npro=npro, seed=seed)


# ---------------------------------------------------------------- CPU

@pytest.mark.parametrize("layint", [0, 1])
def test_oracle_layers_conserve_the_column(oracle, layint):
    """Per layer: the temperature weights DTE sum to 1, the amount weights
    DAM sum to the layer column, a gas's amount over the column is its mixing
    ratio; over the layers the column is the hydrostatic one within 0.5 %."""
    prof = _profile()
    lay = oracle.layerg(prof, nlay=60, laytyp=1, layint=layint)
    assert np.max(np.abs(lay["dte"].sum(1) - 1.0)) < 1e-5
    assert np.max(np.abs(lay["dam"].sum(1) / lay["totam"] - 1.0)) < 1e-5
    assert np.max(np.abs(lay["amount"][:, 1] / lay["totam"] - synth.VMR[synth.HE])) < 1e-6
    col = (prof.p[0] - prof.p[-1]) / synth.BAR_TO_ATM * 1e5 / (synth.MMW * synth.AMU * synth.GRAV) * 1e-4
    assert abs(lay["totam"].sum() / col - 1.0) < 5e-3
    assert np.all(np.diff(lay["baseh"]) > 0) and np.all(np.diff(lay["press"]) < 0)
    # the nadir path: top layer first, every layer once, scale ~ 1
    assert lay["nlayin"] == 60 and lay["imod"] == 3 and lay["npath"] == 1
    assert lay["layinc"].tolist() == list(range(60, 0, -1))
    assert np.allclose(lay["scale"], 1.0, atol=5e-3)
    assert np.array_equal(lay["emtemp"], lay["temp"][::-1])


def test_oracle_layer_types_agree(oracle):
    """Given the base heights (LAYTYP 5) or base pressures (LAYTYP 4) of an
    equal-log-pressure layering, the layers are those of LAYTYP 1; every type
    gives increasing bases from LAYHT."""
    prof = _profile()
    ref = oracle.layerg(prof, nlay=40, laytyp=1, layint=1)
    same = oracle.layerg(prof, nlay=40, laytyp=5, layint=1, base=ref["baseh"])
    for k in FLOATS:
        assert np.array_equal(same[k], ref[k]), k
    byp = oracle.layerg(prof, nlay=40, laytyp=4, layint=1, base=ref["basep"])
    assert np.allclose(byp["baseh"], ref["baseh"], rtol=0, atol=2e-3)
    for t in (0, 2, 3):
        lay = oracle.layerg(prof, nlay=40, laytyp=t, layint=1, layht=2.0)
        assert abs(lay["baseh"][0] - 2.0) < 1e-3 and np.all(np.diff(lay["baseh"]) > 0), t


def test_oracle_slant_and_upward_paths(oracle):
    """A slant nadir path scales each layer by about 1/cos(angle) (slightly
    less, the planet being round); a path looking up (angle > 90) takes the
    layers bottom first."""
    prof = _profile()
    lay = oracle.layerg(prof, nlay=30, laytyp=1, layint=1, angle=50.0)
    assert np.all(np.abs(lay["scale"] / (1 / np.cos(np.deg2rad(50.0))) - 1) < 5e-3)
    up = oracle.layerg(prof, nlay=30, laytyp=1, layint=1, angle=130.0, botlay=3)
    assert up["nlayin"] == 28 and up["layinc"][:28].tolist() == list(range(1, 29))


# ---------------------------------------------------------------- GPU

CASES = [dict(laytyp=1, layint=1), dict(laytyp=1, layint=0), dict(laytyp=0, layint=1),
         dict(laytyp=2, layint=1, layht=3.0), dict(laytyp=3, layint=1, layang=30.0),
         dict(laytyp=1, layint=1, angle=55.0, botlay=4), dict(laytyp=1, layint=1, angle=140.0, botlay=2),
         dict(laytyp=1, layint=1, angle=40.0, ipzen=1)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_layerg_matches_oracle(ctx, oracle, case):
    """rtb_layerg against the oracle, bit for bit: the device does the
    layering in the reference's REAL arithmetic and order, and the
    transcendental set-up scalars come from the same C library."""
    prof = _profile()
    opts = dict(nlay=70, **CASES[case])
    got = ctx.layerg(prof, **opts)
    ref = oracle.layerg(prof, **opts)
    for k in ("npath", "nlayin", "imod"):
        assert got[k] == ref[k], k
    n = ref["nlayin"]
    assert np.array_equal(got["layinc"][:n], ref["layinc"][:n])
    for k in FLOATS:
        a, b = got[k], ref[k]
        if k in ("scale", "emtemp"):
            a, b = a[:n], b[:n]
        assert np.array_equal(a, b), (k, float(np.max(np.abs(a - b))))


@pytest.mark.gpu
def test_profile_to_radiance_through_device_layers(ctx, oracle):
    """A 121-level profile layered on the device into 120 layers, then the
    forward model with the Jacobian over the 121 level temperatures and the
    four gas scales (mapped through DTE / DAM): radiance within 1e-4 and
    Jacobian within 1e-3 of the FP64 oracle forward model on the same layers,
    and the device-layered spectrum equal to the oracle-layered one."""
    kt, cia, _ = synth.config2(nwave=300, nlayer=40, nbin=300)
    prof = synth.make_profile(synth.ABSORBERS_C2, npro=121, seed=11)
    lay = ctx.layerg(prof, nlay=120, laytyp=1, layint=1, angle=25.0)
    job = synth.job_from_layers(kt, prof, lay)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, _ = ctx.cirsrtfg_wave(job)
    c64, g64, _ = oracle.cirsrtfg_wave(kt, cia, job, oracle.ORC_FP64)
    assert rad_err(c, c64) <= RAD_TOL
    assert jac_err(g, g64, job.nv) <= JAC_TOL
    job_o = synth.job_from_layers(kt, prof, oracle.layerg(prof, nlay=120, laytyp=1, layint=1, angle=25.0))
    co, go, _ = ctx.cirsrtfg_wave(job_o)
    assert np.array_equal(c, co) and np.array_equal(g, go)
