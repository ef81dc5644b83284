"""Shared comparison helpers of the parity tests.

Tolerances (stated per result, as the acceptance criteria require):
  radiance   max_w |R - R_ref| / |R_ref|                       <= 1e-4
  Jacobian   max_{w,iv} |K - K_ref| / max_w |K_ref(:, iv)|     <= 1e-3
             (column-normalised: each state element's row of the
             Jacobian is scaled by its own largest magnitude); reported
             beside it, element-wise |K - K_ref| / |K_ref| over the entries
             with |K_ref| >= 1e-3 of their row's largest magnitude
  g-bins     the element -> g-bin assignment of every sorted overlap
             pass identical (integer, bit-exact).
"""
import numpy as np

RAD_TOL = 1e-4
JAC_TOL = 1e-3


def rad_err(c, c_ref):
    c = np.asarray(c, np.float64)
    c_ref = np.asarray(c_ref, np.float64)
    return float(np.max(np.abs(c - c_ref) / np.abs(c_ref)))


def jac_err(g, g_ref, nv):
    G = np.asarray(g, np.float64).reshape(nv, -1)
    R = np.asarray(g_ref, np.float64).reshape(nv, -1)
    scale = np.max(np.abs(R), axis=1, keepdims=True)
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(G - R) / scale))


def jac_err_elementwise(g, g_ref, nv, floor=1e-3):
    """Element-wise relative Jacobian error over the entries whose magnitude
    is at least `floor` times their state element's largest one."""
    G = np.asarray(g, np.float64).reshape(nv, -1)
    R = np.asarray(g_ref, np.float64).reshape(nv, -1)
    scale = np.max(np.abs(R), axis=1, keepdims=True)
    big = (np.abs(R) >= floor * scale) & (scale > 0)
    if not big.any():
        return 0.0
    return float(np.max(np.abs(G - R)[big] / np.abs(R)[big]))


def assignment_fast(perm, split, ng, chunk=8192):
    """Vectorised form of `assignment` for large captures: an element's bin
    is the number of recorded split positions strictly before its sorted
    position (splits are increasing; -1 marks a bin never closed)."""
    nloop = perm.shape[-1]
    P = perm.reshape(-1, nloop)
    S = split.reshape(-1, ng).astype(np.int32)
    out = np.full(P.shape, -1, np.int8)
    pos = np.arange(nloop, dtype=np.int32)
    for r0 in range(0, P.shape[0], chunk):
        p = P[r0:r0 + chunk].astype(np.int64)
        s = S[r0:r0 + chunk]
        valid = p[:, 0] >= 0
        s = np.where(s >= 0, s, np.int32(1 << 20))
        pos_bin = np.zeros(p.shape, np.int8)
        for b in range(ng):
            pos_bin += (s[:, b:b + 1] < pos[None, :]).astype(np.int8)
        blk = np.full(p.shape, -1, np.int8)
        rows = np.nonzero(valid)[0]
        tmp = blk[rows]
        np.put_along_axis(tmp, p[rows], pos_bin[rows], axis=1)
        blk[rows] = tmp
        out[r0:r0 + chunk] = blk
    return out.reshape(perm.shape)


def assignment(perm, split, ng):
    """element -> g-bin (bin of the element's sorted position) for every
    recorded pass; -1 rows for passes that did not sort."""
    nloop = perm.shape[-1]
    P = perm.reshape(-1, nloop)
    S = split.reshape(-1, ng)
    out = np.full(P.shape, -1, np.int32)
    for r in range(P.shape[0]):
        if P[r, 0] < 0:
            continue
        pos_bin = np.zeros(nloop, np.int32)
        b = 0
        for pos in range(nloop):
            pos_bin[pos] = b
            if b < ng and S[r, b] == pos:
                b += 1
        out[r, P[r]] = pos_bin
    return out.reshape(perm.shape)
