"""Writers of the reference's table files, for the loader tests.

write_kta follows the record layout of radtran/radtran/calc_fnktablec.f:
304-367 (direct access, 4-byte records): IREC0, NPOINT, VMIN, DELV, FWHM,
NP, NT, NG, IDGAS, ISOGAS, G_ORD(NG), DEL_G(NG), two spare records,
PRESS(NP) in atm, TEMP(NT) -- or for NT < 0 TEMP2(NP, |NT|) with the
temperature index fastest (read_khead.f:87-93) -- and VCEN(NPOINT) when
DELV <= 0, then the k values (x 1e20) from record IREC0, bin by bin with g
fastest.  write_cia_tab writes the two sequential
unformatted records that ciaread.f:77-98 reads."""
import numpy as np


def write_kta(path, kt, i, idgas, isogas):
    ng, np_, nt = kt.ng, kt.np_, kt.nt
    ntk = nt if nt > 0 else np_ * -nt
    nvc = int(kt.nbin[i]) if not kt.delv[i] > 0 else 0      # VCEN(NPOINT) of an irregular grid
    irec0 = 11 + 2 * ng + 2 + np_ + ntk + nvc + 2
    head = np.zeros(irec0 - 1, np.int32)
    f = head.view(np.float32)
    head[0], head[1] = irec0, int(kt.nbin[i])
    f[2], f[3], f[4] = kt.vmin[i], kt.delv[i], 0.0
    head[5], head[6], head[7], head[8], head[9] = np_, nt, ng, idgas, isogas
    f[10:10 + ng] = kt.g_ord
    f[10 + ng:10 + 2 * ng] = kt.delg
    o = 10 + 2 * ng + 2
    f[o:o + np_] = np.exp(kt.lnp.astype(np.float64)).astype(np.float32)
    if nt > 0:
        f[o + np_:o + np_ + nt] = kt.tk
    else:   # TEMP2(I, J) records, J fastest
        f[o + np_:o + np_ + ntk] = kt.tk.reshape(-nt, np_).T.ravel()
    if nvc:
        f[o + np_ + ntk:o + np_ + ntk + nvc] = kt.vcen
    with open(path, "wb") as fh:
        fh.write(head.tobytes())
        fh.write(np.ascontiguousarray(kt.table(i), np.float32).tobytes())


def write_cia_tab(path, cia):
    temps = np.asarray(cia.temps, np.float64)
    kcia = np.asarray(cia.kcia, np.float32)
    with open(path, "wb") as fh:
        for rec in (temps.tobytes(), kcia.tobytes()):
            n = np.array([len(rec)], np.int32).tobytes()
            fh.write(n + rec + n)
