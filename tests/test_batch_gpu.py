"""GPU tests of the batched forward model on uneven spectra (the
persistent-launch form): every tile (warps per block), schedule and
occupancy, the autotuner and the CUDA-graph replay give the same bits as one
rtb_cirsrtfg_wave call per spectrum, a re-prepared batch of the tuned shape
starts with the tuned configuration, and the batch agrees with the FP64
oracle within the parity tolerances."""
import os

import numpy as np
import pytest

from radtrancode_b200 import synth
from tests.helpers import JAC_TOL, RAD_TOL, jac_err, rad_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven():
    kt, cia, _ = synth.config2()
    jobs = synth.config3_jobs(kt, 24, seed=1003)
    return kt, cia, jobs


def _same(outs, singles):
    for (c, g, gt), (c1, g1, gt1) in zip(outs, singles):
        assert np.array_equal(c, c1) and np.array_equal(g, g1) and np.array_equal(gt, gt1)


def test_schedules_graph_and_autotune_are_bit_identical(ctx, uneven):
    kt, cia, jobs = uneven
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    singles = [ctx.cirsrtfg_wave(j) for j in jobs]
    ctx.prepare(jobs)
    try:
        for tile in (4, 2, 8):
            ctx.set_tile(tile)
            for sched in (0, 1, 2):
                for occ in (0, 1):
                    ctx.set_schedule(sched, occ)
                    ctx.launch()
                    _same(ctx.fetch(), singles)
        ctx.set_tile(0)
        ctx.use_graph(True)
        for _ in range(3):                       # capture, then two replays
            ctx.launch()
            _same(ctx.fetch(), singles)
        tune = ctx.autotune()
        assert tune["candidates"] >= 9 and tune["ms"] > 0 and tune["warps"] in (2, 4, 8)
        ctx.launch()
        _same(ctx.fetch(), singles)
        assert ctx.stats()["cells"] == sum(j.nlayer * j.nwave for j in jobs)
        # a batch of the same shape starts with the tuned tile: the launch's grid is the tuned one
        grid_tuned = ctx.stats()["grid"]
        ctx.use_graph(False)
        ctx.prepare(jobs[::-1])
        ctx.launch()
        _same(ctx.fetch()[::-1], singles)
        assert ctx.stats()["grid"] == grid_tuned
    finally:
        ctx.use_graph(False)
        ctx.set_tile(0)
        ctx.set_schedule(0, 0)


def test_uneven_batch_against_fp64_oracle(ctx, oracle, uneven):
    """Every spectrum of the 24-spectrum uneven batch (one persistent launch)
    against the FP64 oracle."""
    kt, cia, jobs = uneven
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    outs = ctx.cirsrtfg_wave_batch(jobs)
    worst_r = worst_j = 0.0
    for j, (c, g, gt) in zip(jobs, outs):
        c64, g64, gt64 = oracle.cirsrtfg_wave(kt, cia, j, oracle.ORC_FP64, nthreads=os.cpu_count() or 1)
        worst_r = max(worst_r, rad_err(c, c64))
        worst_j = max(worst_j, jac_err(g, g64, j.nv))
        assert rad_err(c, c64) <= RAD_TOL
        assert jac_err(g, g64, j.nv) <= JAC_TOL
    print(f"uneven batch of {len(jobs)}: radiance {worst_r:.2e}, Jacobian {worst_j:.2e}")
