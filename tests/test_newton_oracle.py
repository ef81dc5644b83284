"""CPU tests of the Newton-step restatement (oracle/newton_oracle.cpp)."""
import ctypes as C

import numpy as np

D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)


def _spd(n, rng):
    a = rng.standard_normal((n, n))
    return a @ a.T + n * np.eye(n)


def _d(a):
    return np.asfortranarray(a, np.float64)


def _f(a):
    return np.asfortranarray(a, np.float32)


def test_dinvertm_cholesky_inverse(oracle):
    rng = np.random.default_rng(0)
    A = _d(_spd(30, rng))
    Ai = np.zeros_like(A, order="F")
    ic = oracle.lib().orc_dinvertm_chol(30, 30, A.ctypes.data_as(D), Ai.ctypes.data_as(D))
    assert ic == 0
    assert np.allclose(A @ Ai, np.eye(30), atol=1e-10)


def test_dinvertm_flags_non_positive_definite(oracle):
    A = _d(np.diag([1.0, -2.0, 3.0]))
    Ai = np.zeros_like(A, order="F")
    ic = oracle.lib().orc_dinvertm_chol(3, 3, A.ctypes.data_as(D), Ai.ctypes.data_as(D))
    assert ic == 1          # dcholdc sets p(i)=1 and continues; the A*Ainv check fails


def _problem(nx, ny, seed):
    rng = np.random.default_rng(seed)
    K = _f(rng.standard_normal((ny, nx)))
    sa = _spd(nx, rng) / nx
    sai = np.linalg.inv(sa)
    se_diag = rng.uniform(0.5, 2.0, ny)
    x_true = rng.standard_normal(nx)
    xa = np.zeros(nx, np.float32)
    y = (K.astype(np.float64) @ x_true).astype(np.float32)
    return K, _d(sa), _d(sai), se_diag, xa, y


def test_gain_matrix_linear_map_estimate(oracle):
    """One Newton step of a linear forward model equals the closed-form MAP
    estimate xa + (K'Se^-1K + Sa^-1)^-1 K'Se^-1 (y - K xa)."""
    nx, ny = 12, 40
    K, sa, sai, se_diag, xa, y = _problem(nx, ny, 1)
    se = _f(np.diag(se_diag))
    sei = _d(np.diag(1.0 / se_diag))
    dd = np.zeros((nx, ny), order="F")
    aa = np.zeros((nx, nx), order="F")
    ic = C.c_int(-1)
    L = oracle.lib()
    L.orc_calc_gain_matrix(nx, ny, nx, ny, K.ctypes.data_as(F), _f(sa).ctypes.data_as(F), sai.ctypes.data_as(D),
                           se.ctypes.data_as(F), sei.ctypes.data_as(D), dd.ctypes.data_as(D), aa.ctypes.data_as(D),
                           C.byref(ic))
    assert ic.value == 0
    xn = xa.copy()
    yn = (K.astype(np.float64) @ xn.astype(np.float64)).astype(np.float32)
    x_out = np.zeros(nx, np.float32)
    L.orc_calcnextxn(nx, ny, nx, xa.ctypes.data_as(F), xn.ctypes.data_as(F), y.ctypes.data_as(F),
                     yn.ctypes.data_as(F), dd.ctypes.data_as(D), aa.ctypes.data_as(D), x_out.ctypes.data_as(F))
    Kd = K.astype(np.float64)
    A = Kd.T @ np.diag(1 / se_diag) @ Kd + sai
    x_map = np.linalg.solve(A, Kd.T @ np.diag(1 / se_diag) @ (y - Kd @ xa))
    assert np.allclose(x_out, x_map, rtol=1e-5, atol=1e-5)
    assert np.allclose(aa, np.asarray(dd) @ Kd, atol=1e-12)


def test_diagonal_gain_matrix_is_bitwise_dense(oracle):
    nx, ny = 9, 33
    K, sa, sai, se_diag, xa, y = _problem(nx, ny, 2)
    se = _f(np.diag(se_diag))
    sei = _d(np.diag(1.0 / se_diag))
    L = oracle.lib()
    out = []
    for diag in (False, True):
        dd = np.zeros((nx, ny), order="F")
        aa = np.zeros((nx, nx), order="F")
        ic = C.c_int(-1)
        if diag:
            sed = np.ascontiguousarray(1.0 / se_diag)
            L.orc_calc_gain_matrix_diag(nx, ny, nx, ny, K.ctypes.data_as(F), sai.ctypes.data_as(D),
                                        sed.ctypes.data_as(D), dd.ctypes.data_as(D), aa.ctypes.data_as(D),
                                        C.byref(ic))
        else:
            L.orc_calc_gain_matrix(nx, ny, nx, ny, K.ctypes.data_as(F), _f(sa).ctypes.data_as(F),
                                   sai.ctypes.data_as(D), se.ctypes.data_as(F), sei.ctypes.data_as(D),
                                   dd.ctypes.data_as(D), aa.ctypes.data_as(D), C.byref(ic))
        out.append((dd, aa))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_phiret_dense_and_diagonal_agree(oracle):
    nx, ny = 7, 25
    rng = np.random.default_rng(4)
    y = rng.standard_normal(ny).astype(np.float32)
    yn = rng.standard_normal(ny).astype(np.float32)
    xn = rng.standard_normal(nx).astype(np.float32)
    xa = rng.standard_normal(nx).astype(np.float32)
    sai = _d(_spd(nx, rng))
    sed = rng.uniform(0.5, 2, ny)
    sei = _d(np.diag(sed))
    L = oracle.lib()
    c1, c2 = C.c_float(), C.c_float()
    p1 = L.orc_calc_phiret(ny, ny, y.ctypes.data_as(F), yn.ctypes.data_as(F), sei.ctypes.data_as(D), nx, nx,
                           xn.ctypes.data_as(F), xa.ctypes.data_as(F), sai.ctypes.data_as(D), C.byref(c1))
    sedc = np.ascontiguousarray(sed)
    p2 = L.orc_calc_phiret_diag(ny, y.ctypes.data_as(F), yn.ctypes.data_as(F), sedc.ctypes.data_as(D), nx, nx,
                                xn.ctypes.data_as(F), xa.ctypes.data_as(F), sai.ctypes.data_as(D), C.byref(c2))
    assert p1 == p2 and c1.value == c2.value
    r = (yn.astype(np.float64) - y)
    dx = (xn.astype(np.float64) - xa)
    assert np.isclose(p1, r @ (sed * r) + dx @ sai @ dx, rtol=1e-6)
