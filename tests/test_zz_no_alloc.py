"""rtb_fwd_launch_static: the forward launch whose per-block scratch comes
from the library's fixed per-device array instead of the context.

Checked against the ordinary entry point (rtb_cirsrtfg_wave) on the same
batch, on two calls in a row, within the parity tolerances of
tests/helpers.py.  The 200-layer case has more blocks than the static array
holds slots: the test checks that it runs on fewer blocks than the ordinary
launch (the reduced grid), under the static schedule and the two dynamic
ones (which pull items from a counter and, longest first, from an order)."""
import numpy as np
import pytest

from radtrancode_b200 import cirsradg, synth
from tests.helpers import JAC_TOL, RAD_TOL, jac_err, rad_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nwave,nlayer,reduced", [(64, 120, False), (1000, 200, True)])
def test_static_scratch_matches_rtb_cirsrtfg_wave(ctx, nwave, nlayer, reduced):
    kt, cia, job = synth.config2(nwave=nwave, nlayer=nlayer, nbin=nwave)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c_ref, g_ref, gt_ref = ctx.cirsrtfg_wave(job)
    ctx.prepare([job])
    ctx.set_tile(4)          # 740 blocks of the ordinary launch against the static array's 349 slots of 96 KB
    ctx.launch()
    ctx.fetch()
    full_grid = ctx.stats()["grid"]
    try:
        for sched in ((0, 1, 2) if reduced else (0,)):
            ctx.set_schedule(sched, 0)
            for _ in range(2):
                ctx.launch_static()
                (c, g, gt), = ctx.fetch()
                st = ctx.stats()
                assert rad_err(c, c_ref) <= RAD_TOL
                assert jac_err(g, g_ref, job.nv) <= JAC_TOL
                assert np.max(np.abs(gt - gt_ref)) <= RAD_TOL * np.max(np.abs(gt_ref))
                assert st["cells"] == nwave * nlayer
                assert ((0 < st["grid"] < full_grid) if reduced else (st["grid"] == full_grid)), (st["grid"], full_grid)
    finally:
        ctx.set_tile(0)
        ctx.set_schedule(0, 0)


def test_static_scratch_needs_a_prepared_batch():
    with cirsradg.Context(0) as c:
        with pytest.raises(cirsradg.RtbError) as e:
            c.launch_static()
        assert e.value.status == 1
