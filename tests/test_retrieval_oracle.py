"""CPU tests of the retrieval-loop restatement (oracle/coreret_oracle.cpp)
and of the algebra the device Newton step relies on."""
import numpy as np
import pytest

from radtrancode_b200 import synth


@pytest.fixture(scope="module")
def c1_case(oracle):
    kt, cia, _ = synth.config1()
    case = synth.make_retrieval(kt, [synth.CH4], nlayer=40, seed=5)
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true)
    synth.observe(case, y_true, seed=6)
    return kt, cia, case


def test_newton_step_without_gain_matrix_equals_reference_algebra(oracle, c1_case):
    """xa + C^-1 K'Se^-1 (y - yn + K (xn - xa)) (the device formulation)
    equals calc_gain_matrix + calcnextxn: xa + D (y - yn) - AA (xa - xn)."""
    kt, cia, case = c1_case
    xn = case.x_true + np.float32(0.3)
    yn, kk = oracle.forward_state(kt, cia, case, xn)
    sai, ic = oracle.dinvertm(case.sa)
    assert ic == 0
    x_ref = oracle.newton_step(kk, case.sei, sai, case.xa, xn, case.y, yn)
    K = kk.astype(np.float64).T                        # ny x nx
    C = K.T @ (case.sei[:, None] * K) + sai
    d = (xn - case.xa).astype(np.float64)
    r = K.T @ (case.sei * ((case.y - yn).astype(np.float64) + K @ d))
    x_new = case.xa + np.linalg.solve(C, r).astype(np.float32)
    step = np.max(np.abs(x_ref - case.xa))
    assert np.max(np.abs(x_new - x_ref)) <= 1e-5 * step + 1e-4


def test_retrieval_converges_and_fits(oracle, c1_case):
    kt, cia, case = c1_case
    res, tr = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1)
    assert res["converged"] == 1
    assert res["forwards"] == 1 + int(np.sum(tr["verdict"] > 0))
    # accepted costs decrease monotonically (coreret.f:979)
    acc = tr["phi"][tr["verdict"] == 1]
    assert np.all(np.diff(acc) <= 0)
    assert res["chisq"] / case.ny < 2.0
    # the log scale of CH4 is retrieved well inside its prior width (0.5)
    assert abs(res["x"][-1] - case.x_true[-1]) < 0.1


def test_rejection_raises_brake(oracle):
    """A first guess far from the data: rejected steps multiply alambda by
    10 (coreret.f:1060-1064), accepted ones by 0.3."""
    kt, cia, _ = synth.config1()
    case = synth.make_retrieval(kt, [synth.CH4], nlayer=40, seed=9)
    y_true, _ = oracle.forward_state(kt, cia, case, case.x_true)
    synth.observe(case, y_true, seed=10)
    case.x0 = case.xa.copy()
    case.x0[-1] = 8.0                                     # CH4 x 3000
    res, tr = oracle.retrieve(kt, cia, case, kiter=10, phlimit=0.1)
    assert np.any(tr["verdict"] == 2)
    lam = 1.0
    for v, a in zip(tr["verdict"], tr["alambda"]):
        if v == 1 and a != np.float32(lam):
            break                                         # converged on this accepted step (brake kept)
        lam = np.float32(lam * (0.3 if v == 1 else 10.0))
        assert a == lam
    assert res["phi"] <= tr["phi"][tr["verdict"] == 1].min() + 1e-6
