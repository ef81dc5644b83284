"""GPU tests of the continuous-batching retrieval server (rtb_server_*):
a request's result is the same alone and in a mix of requests of other
sizes arriving at other times (bit for bit: every request's arithmetic is
independent of the batch it shares), admission respects the HBM budget,
and the server agrees with the batched entry point."""
import numpy as np
import pytest

from radtrancode_b200 import cirsradg, synth

pytestmark = pytest.mark.gpu


def _case(oracle, kt, cia, absorbers, nlayer, seed, nwave=None, iw0=0, theta=0.0):
    case = synth.make_retrieval(kt, absorbers, nlayer=nlayer, seed=seed, nwave=nwave, iw0=iw0, theta_deg=theta)
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true, nthreads=8)
    return synth.observe(case, y_true, seed=seed + 1)


@pytest.fixture(scope="module")
def mix(oracle):
    kt, cia, _ = synth.config2()
    cases = [
        _case(oracle, kt, cia, [synth.CH4], 40, 31, nwave=240, iw0=100),
        _case(oracle, kt, cia, synth.ABSORBERS_C2[:2], 60, 33, nwave=400, iw0=700, theta=35.0),
        _case(oracle, kt, cia, synth.ABSORBERS_C2, 90, 35, nwave=300, iw0=1200, theta=60.0),
        _case(oracle, kt, cia, synth.ABSORBERS_C2[1:3], 50, 37, nwave=220, iw0=40),
    ]
    return kt, cia, cases


def _run_alone(ctx, case, budget=1 << 30):
    with cirsradg.Server(ctx, budget, kiter=8) as srv:
        rid = srv.submit(case)
        while True:
            srv.step()
            r = srv.poll(rid)
            if r is not None:
                return r


def _equal(a, b):
    assert np.array_equal(a["x"], b["x"])
    assert np.array_equal(a["yn"], b["yn"])
    for k in ("phi", "chisq", "alambda", "iterations", "forwards", "converged"):
        assert a[k] == b[k], k


def test_result_same_alone_and_in_mix(ctx, mix):
    kt, cia, cases = mix
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    alone = [_run_alone(ctx, c) for c in cases]
    # the mix: requests arrive at different rounds, and a 500 kB budget
    # (about the two largest requests' device state) makes some wait
    got = {}
    waited = False
    with cirsradg.Server(ctx, 500_000, kiter=8) as srv:
        order = [2, 0, 3, 1]
        ids = {}
        for step in range(200):
            if step < len(order):
                ids[srv.submit(cases[order[step]])] = order[step]
            active, queued = srv.step()
            waited |= queued > 0
            for rid in list(ids):
                r = srv.poll(rid)
                if r is not None:
                    got[ids.pop(rid)] = r
            if not ids and step >= len(order):
                break
    assert waited and len(got) == len(cases)
    for i in range(len(cases)):
        _equal(got[i], alone[i])


def test_server_matches_batched_entry_point(ctx, mix):
    kt, cia, cases = mix
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    batch = ctx.retrieve_batch(cases, kiter=8)
    for c, b in zip(cases, batch):
        _equal(_run_alone(ctx, c), b)


def test_request_larger_than_budget_is_refused(ctx, mix):
    kt, cia, cases = mix
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    with cirsradg.Server(ctx, 64 * 1024, kiter=8) as srv:
        with pytest.raises(cirsradg.RtbError) as e:
            srv.submit(cases[2])
        assert e.value.status == 9        # RTB_ERR_BUDGET
