"""rtb_fwd_launch_static: the forward launch whose per-block scratch comes
from the library's fixed per-device array instead of the context.

Checked against the ordinary entry point (rtb_cirsrtfg_wave) on the same
batch, on two calls in a row, within the parity tolerances of
tests/helpers.py.  The 200-layer case has more wavenumbers than the static
array holds block slots, so it also runs the reduced grid."""
import numpy as np
import pytest

from radtrancode_b200 import cirsradg, synth
from tests.helpers import JAC_TOL, RAD_TOL, jac_err, rad_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nwave,nlayer", [(64, 120), (1000, 200)])
def test_static_scratch_matches_rtb_cirsrtfg_wave(ctx, nwave, nlayer):
    kt, cia, job = synth.config2(nwave=nwave, nlayer=nlayer, nbin=nwave)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c_ref, g_ref, gt_ref = ctx.cirsrtfg_wave(job)
    ctx.prepare([job])
    for _ in range(2):
        ctx.launch_static()
        (c, g, gt), = ctx.fetch()
        assert rad_err(c, c_ref) <= RAD_TOL
        assert jac_err(g, g_ref, job.nv) <= JAC_TOL
        assert np.max(np.abs(gt - gt_ref)) <= RAD_TOL * np.max(np.abs(gt_ref))
        assert ctx.stats()["cells"] == nwave * nlayer


def test_static_scratch_needs_a_prepared_batch():
    with cirsradg.Context(0) as c:
        with pytest.raises(cirsradg.RtbError) as e:
            c.launch_static()
        assert e.value.status == 1
