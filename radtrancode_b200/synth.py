"""Seeded synthetic workloads for the correlated-k gradient forward model.

The reference measures on no public dataset; these generators build the
workloads its own thermal-emission retrievals run on (a nadir giant-planet
atmosphere, k-tables in .kta record order, a CIA table of the ciaread
format) with the shapes and value distributions fixed by the configurations:

* ``config1``: 40 layers, H2/He + CH4, 100 wavenumbers 1200-1350 cm-1,
  k-table 20 P x 10 T x 20 g, NX = 41.
* ``config2``: 120 layers, H2/He + CH4, C2H6, C2H2, NH3, 2000 wavenumbers
  600-1400 cm-1, k-tables 20 P x 15 T x 20 g, NX = 124.
* ``config3``: batches of uneven spectra drawn around config 2.

Arrays use the Fortran layouts of the reference's COMMON blocks (column
major, leading dimensions recorded in the job) so they can be handed to the
C ABI (include/radtran_b200.h) unchanged.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _abi

BAR_TO_ATM = 0.986923
AMU = 1.66053907e-27
KB = 1.380649e-23
GRAV = 24.79          # m s-2 (Jupiter)
MMW = 2.3             # mean molecular weight, amu

# (HITRAN-style local id, isotope) of the gases of the configurations
H2, HE, CH4, C2H6, C2H2, NH3 = (39, 0), (40, 0), (6, 0), (27, 0), (26, 0), (11, 0)
ABSORBERS_C2 = [CH4, C2H6, C2H2, NH3]
VMR = {H2: 0.86, HE: 0.136, CH4: 2e-3, C2H6: 4e-6, C2H2: 1e-7, NH3: 1e-4}


def gauss_legendre_01(ng: int):
    """Gauss-Legendre ordinates and weights on [0, 1] (sum of weights = 1)."""
    x, w = np.polynomial.legendre.leggauss(ng)
    return ((x + 1.0) * 0.5).astype(np.float32), (w * 0.5).astype(np.float32)


@dataclasses.dataclass
class KTables:
    """k-tables of a run, laid out as rtb_set_ktables expects."""
    np_: int
    nt: int
    ng: int
    lnp: np.ndarray        # (np,) float32, ln(p / atm)
    tk: np.ndarray         # (nt,) float32; NT < 0: TEMP2 (np, |nt|) column-major, one grid per pressure
    g_ord: np.ndarray      # (ng,) float32
    delg: np.ndarray       # (ng,) float32
    vmin: np.ndarray       # (ntab,) float32
    delv: np.ndarray       # (ntab,) float32
    nbin: np.ndarray       # (ntab,) int32
    data: np.ndarray       # concatenated float32 records
    gases: list            # (id, iso) of each table
    vcen: np.ndarray | None = None   # irregular grid (delv <= 0): the centres, (nbin,) float32

    @property
    def ntab(self) -> int:
        return len(self.gases)

    def table(self, i: int) -> np.ndarray:
        """Table i as an array [nbin, np, |nt|, ng] (a view)."""
        nt = abs(self.nt)
        n = self.np_ * nt * self.ng
        off = int(sum(int(self.nbin[k]) for k in range(i))) * n
        return self.data[off: off + int(self.nbin[i]) * n].reshape(int(self.nbin[i]), self.np_, nt, self.ng)


@dataclasses.dataclass
class CIATable:
    dnu: float
    temps: np.ndarray      # (25,) float64
    kcia: np.ndarray       # float32, Fortran (9, 25, 1501) flattened in Fortran order


@dataclasses.dataclass
class ParaCIATable:
    """The para-H2 CIA table of fpread_all (rtb_set_para_cia layout)."""
    dnu2: float
    ipara: int
    temps: np.ndarray      # (25,) float32
    fp: np.ndarray         # (ipara,) float32
    kh2h2: np.ndarray      # float32, Fortran (ipara, 25, 1501) flattened
    kh2he: np.ndarray
    kcia5: np.ndarray      # float32, Fortran (5, 25, 1501) flattened


@dataclasses.dataclass
class E3Table:
    """e3interp's table (rtb_set_e3_table layout): the third exponential
    integral E3(tau) at the 1001 transmissions tran = i/1000, tau = -ln(tran)."""
    tau: np.ndarray        # (1001,) float64
    tran: np.ndarray
    e3: np.ndarray


@dataclasses.dataclass
class StellarSpectrum:
    """The stellar spectrum of init_solar_wave (/solardat/): the star's
    radius and its total power spectrum rad at the points wave."""
    solrad: float
    wave: np.ndarray       # float32, monotonic
    rad: np.ndarray        # float32


def make_stellar_spectrum(v0, v1, npt=400, teff=5800.0, solrad=6.96e10, descending=False) -> StellarSpectrum:
    """A blackbody star of temperature teff and radius solrad (cm): total
    power 4 pi^2 R^2 B(v, teff) at npt wavenumbers spanning [v0, v1],
    in descending order if asked (interp.f handles both)."""
    v = np.linspace(v0, v1, npt)
    b = 1.1911e-12 * v ** 3 / np.expm1(1.439 * v / teff)
    rad = 4.0 * np.pi ** 2 * solrad ** 2 * b
    if descending:
        v, rad = v[::-1].copy(), rad[::-1].copy()
    return StellarSpectrum(float(solrad), v.astype(np.float32), rad.astype(np.float32))


def write_stellar_file(path, ss: StellarSpectrum, ispace=0):
    """The text file init_solar_wave.f reads: comment lines, the wavespace,
    the stellar radius, then WAVE RAD records (9 significant digits: the
    REAL values read back exactly)."""
    with open(path, "w") as fh:
        fh.write("# synthetic stellar spectrum\n# wavespace, radius, then wave rad\n")
        fh.write(f"{ispace}\n{ss.solrad:.9e}\n")
        for w, r in zip(ss.wave, ss.rad):
            fh.write(f"{float(w):.9e} {float(r):.9e}\n")


def make_e3_table() -> E3Table:
    """E3 of the e3tab.dat layout: tran(i) = REAL(i/1000), tau = -ln(tran)
    (1e36 standing for tran = 0, where E3 = 0), E3(0) = 1/2."""
    from scipy.special import expn
    tran = (np.arange(1001) / 1000.0).astype(np.float32).astype(np.float64)
    pos = tran > 0
    tau = np.full(1001, 1e36)
    tau[pos] = -np.log(tran[pos])
    e3 = np.zeros(1001)
    e3[pos] = expn(3, tau[pos])
    e3[-1], tau[-1] = 0.5, 0.0
    return E3Table(tau, tran, e3)


def write_e3_table(path, e3: E3Table):
    """The text file e3interp.f reads: the count, a header line, then one
    TAU TRAN E3 record per line (17 significant digits: the doubles read
    back exactly)."""
    with open(path, "w") as fh:
        fh.write(f"{len(e3.tran):8d}\n      tau        trans        e3\n")
        for a, b, c in zip(e3.tau, e3.tran, e3.e3):
            fh.write(f" {a:.16e} {b:.16e} {c:.16e}\n")


def make_para_cia(seed=0, dnu2=1.0, ipara=24) -> ParaCIATable:
    """Smooth lognormal H2-H2 / H2-He coefficients that grow with the para-H2
    fraction (fp = 0.25 .. 1.0 evenly, as nparacon_all.f assumes), plus
    H2-CH4 and CH4-CH4 among the five further pairs (the N2 pairs zero)."""
    rng = np.random.default_rng(seed)
    temps = np.linspace(40.0, 400.0, _abi.CIA_NUMT)
    fp = np.linspace(0.25, 1.0, ipara)
    v = np.arange(_abi.CIA_NUMWN, dtype=np.float64) * dnu2
    vv = np.maximum(v, 1.0)

    def band(amp, v0, s, gam):
        shape = np.exp(-0.5 * (np.log(vv / v0) / s) ** 2)
        shape[v == 0] = 0.0
        return amp * shape[None, :] * (temps[:, None] / 150.0) ** gam

    h2 = band(2e-8, 500.0, 0.6, -0.5)
    he = band(0.8e-8, 700.0, 0.7, -0.3)
    tilt = 1.0 + 0.05 * rng.standard_normal()
    kh2h2 = np.stack([h2 * (0.7 + 0.9 * f * tilt) for f in fp])          # (ipara, 25, 1501)
    kh2he = np.stack([he * (0.9 + 0.3 * f) for f in fp])
    k5 = np.zeros((5, _abi.CIA_NUMT, _abi.CIA_NUMWN))
    k5[3] = band(3e-9, 900.0, 0.5, -0.4)          # CH4-CH4
    k5[4] = band(5e-9, 650.0, 0.6, -0.2)          # H2-CH4
    f32 = lambda a: np.asarray(a, np.float32).ravel(order="F")
    return ParaCIATable(float(dnu2), int(ipara), temps.astype(np.float32), fp.astype(np.float32),
                        f32(np.transpose(kh2h2, (0, 1, 2))), f32(kh2he), f32(k5))


def make_ktables(gases, *, np_=20, nt=15, ng=20, vmin=600.0, delv=0.4, nbin=2000, seed=0,
                 p_top_bar=1e-4, p_bot_bar=10.0, t_min=70.0, t_max=200.0, sigma=2.0,
                 median=1e-22, t2=False, irregular=None) -> KTables:
    """Lognormal k-tables, monotone in g, stored x1e20 (cm2 x 1e20).  t2:
    a pressure-dependent temperature grid (NT < 0, TEMP2(NP, |NT|)): row i
    spans [t_min, t_max] shifted by up to +/-15 K and stretched with
    pressure."""
    rng = np.random.default_rng(seed)
    p_atm = np.geomspace(p_top_bar, p_bot_bar, np_) * BAR_TO_ATM
    lnp = np.log(p_atm.astype(np.float32).astype(np.float64)).astype(np.float32)
    if t2:
        f = np.linspace(0.0, 1.0, np_)[:, None]
        grid = t_min - 15.0 + 30.0 * f + (t_max - t_min) * (0.9 + 0.2 * f) * np.linspace(0.0, 1.0, nt)[None, :]
        tk = np.asfortranarray(grid.astype(np.float32)).ravel(order="F")
    else:
        tk = np.linspace(t_min, t_max, nt).astype(np.float32)
    g_ord, delg = gauss_legendre_01(ng)
    mu = np.log(median * 1e20)
    tabs = []
    for _ in gases:
        z = rng.standard_normal((nbin, np_, nt, ng))
        z.sort(axis=-1)
        tabs.append(np.exp(mu + sigma * z).astype(np.float32).ravel())
    data = np.concatenate(tabs) if tabs else np.zeros(0, np.float32)
    n = len(gases)
    vcen = None
    if irregular is not None:
        # an irregular grid: DELV = irregular (0 or -1), centres vmin + delv * (i + a seeded jitter of +/-0.3)
        vcen = (vmin + delv * (np.arange(nbin) + rng.uniform(-0.3, 0.3, nbin))).astype(np.float32)
        delv = float(irregular)
    return KTables(np_, -nt if t2 else nt, ng, lnp, tk, g_ord, delg,
                   np.full(n, vmin, np.float32), np.full(n, delv, np.float32),
                   np.full(n, nbin, np.int32), data, list(gases), vcen)


def make_cia(seed=0, dnu=1.0) -> CIATable:
    """Smooth lognormal H2-H2 and H2-He CIA (pairs 1, 2; others zero)."""
    temps = np.linspace(40.0, 400.0, _abi.CIA_NUMT)
    v = np.arange(_abi.CIA_NUMWN, dtype=np.float64) * dnu
    k = np.zeros((_abi.CIA_NUMPAIRS, _abi.CIA_NUMT, _abi.CIA_NUMWN), np.float64)
    vv = np.maximum(v, 1.0)
    for pair, (amp, v0, s, gam) in enumerate([(2e-8, 500.0, 0.6, -0.5), (0.8e-8, 700.0, 0.7, -0.3)]):
        shape = np.exp(-0.5 * (np.log(vv / v0) / s) ** 2)
        shape[v == 0] = 0.0
        k[pair] = amp * shape[None, :] * (temps[:, None] / 150.0) ** gam
    return CIATable(float(dnu), temps.astype(np.float64), k.astype(np.float32).ravel(order="F"))


@dataclasses.dataclass
class Channels:
    """Instrument channels of cirsconv (the rtb_conv structure): centres,
    optionally a channel-dependent width table (.fwh, FWHM > 0) or filter
    functions (.fil, FWHM < 0; filter k has nsub[k] points)."""
    vconv: np.ndarray
    vfwhm: np.ndarray | None = None
    xfwhm: np.ndarray | None = None
    vcen: np.ndarray | None = None
    nsub: np.ndarray | None = None
    vfil: np.ndarray | None = None
    fil: np.ndarray | None = None

    def __post_init__(self):
        self.vconv = np.ascontiguousarray(self.vconv, np.float32)
        for k in ("vfwhm", "xfwhm", "vcen", "vfil", "fil"):
            v = getattr(self, k)
            if v is not None:
                setattr(self, k, np.ascontiguousarray(v, np.float32))
        if self.nsub is not None:
            self.nsub = np.ascontiguousarray(self.nsub, np.int32)

    def as_struct(self) -> _abi.RtbConv:
        s = _abi.RtbConv()
        f, i = _abi.fptr, _abi.iptr
        s.nconv, s.vconv = len(self.vconv), f(self.vconv)
        if self.vfwhm is not None:
            s.nfwhm, s.vfwhm, s.xfwhm = len(self.vfwhm), f(self.vfwhm), f(self.xfwhm)
        if self.vcen is not None:
            s.nfil, s.vcen, s.nsub, s.vfil, s.fil = len(self.vcen), f(self.vcen), i(self.nsub), f(self.vfil), f(self.fil)
        s._keep = self
        return s


@dataclasses.dataclass
class Job:
    """One cirsrtfg_wave call in the reference's Fortran array layout."""
    nlayer: int
    ngas: int
    npath: int
    npro: int
    nv: int
    nwave: int
    ld_lay: int
    ld_v: int
    ld_param: int
    press: np.ndarray
    temp: np.ndarray
    delh: np.ndarray
    pp: np.ndarray          # (ld_lay, ngas) F
    amount: np.ndarray      # (ld_lay, ngas) F
    idgas: np.ndarray
    isogas: np.ndarray
    ktab: np.ndarray
    nlayin: np.ndarray
    imod: np.ndarray
    layinc: np.ndarray      # (ld_lay, npath) F, 1-based
    scale: np.ndarray       # (ld_lay, npath) F
    emtemp: np.ndarray
    dte: np.ndarray         # (ld_lay, npro) F
    dam: np.ndarray
    xmap: np.ndarray        # (ld_v, ld_param, npro) F
    vwave: np.ndarray
    vem: np.ndarray
    emissivity: np.ndarray
    inormal: int = 0
    iray: int = 0
    itype: int = 11
    ispace: int = 0
    tsurf: float = 0.0
    iform: int = 0
    flagh2p: int = 0
    hfp: np.ndarray | None = None    # (nlayer) para-H2 fractions, flagh2p = 1
    dfp: np.ndarray | None = None    # (ld_lay, npro) F
    fwhm: float = 0.0
    radius1: float = 0.0             # km, planet radius (iform = 3 total flux)
    radextra: float = 0.0            # km, correction to radius1
    inlte: int = 0                   # non-LTE emission temperatures (calc_nlte_t.f): 0, 1 or 2
    nlte_k1: float = 0.0             # inlte = 1: collisional rate and Einstein A
    nlte_A: float = 0.0
    dist: float = 0.0                # AU, distance from the star (iform = 4)
    gascon: tuple = (0, 0, 0, 0, 0)  # /GASCONDEF/ switches IH2O, ICH4, INH3, IO3, iuvscat (ngascon.f)
    conv: "Channels | None" = None   # instrument channels (None: FWHM = 0, nconv = nwave)
    ncont: int = 0                   # dust types
    cont: np.ndarray | None = None   # (ncont, nlayer) F, dust particles / cm2 per layer
    xsec_ext: np.ndarray | None = None   # (ncont, nwave) F, extinction x-section at vwave (cm2)
    dco: np.ndarray | None = None    # (ld_lay, npro) F, d(layer dust)/d(level dust)
    # bookkeeping for the synthetic state vector (not part of the ABI)
    vmr: np.ndarray | None = None
    ncol: np.ndarray | None = None
    xscale: np.ndarray | None = None

    @property
    def nparam(self) -> int:
        return self.ngas + 1 + self.ncont + (1 if self.flagh2p else 0)

    def as_struct(self) -> _abi.RtbAtm:
        s = _abi.RtbAtm()
        s.nlayer, s.ngas, s.ncont, s.npath = self.nlayer, self.ngas, self.ncont, self.npath
        s.npro, s.nv, s.nwave = self.npro, self.nv, self.nwave
        s.ld_lay, s.ld_con, s.ld_v, s.ld_param = self.ld_lay, max(self.ncont, 1), self.ld_v, self.ld_param
        f, i = _abi.fptr, _abi.iptr
        s.press, s.temp, s.delh = f(self.press), f(self.temp), f(self.delh)
        s.pp, s.amount, s.cont = f(self.pp), f(self.amount), None
        s.idgas, s.isogas, s.ktab = i(self.idgas), i(self.isogas), i(self.ktab)
        s.nlayin, s.imod, s.layinc = i(self.nlayin), i(self.imod), i(self.layinc)
        s.scale, s.emtemp = f(self.scale), f(self.emtemp)
        s.dte, s.dam, s.dco, s.dfp = f(self.dte), f(self.dam), None, None
        s.xmap = f(self.xmap)
        s.vwave, s.xsec_ext = f(self.vwave), None
        if self.ncont:
            s.cont, s.xsec_ext, s.dco = f(self.cont), f(self.xsec_ext), f(self.dco)
        s.inormal, s.iray, s.itype, s.ispace = self.inormal, self.iray, self.itype, self.ispace
        s.flagh2p, s.ilbl, s.inlte, s.iform = self.flagh2p, 0, self.inlte, self.iform
        s.nlte_k1, s.nlte_A = float(self.nlte_k1), float(self.nlte_A)
        s.dist = float(self.dist)
        s.ih2o, s.ich4, s.inh3, s.io3, s.iuvscat = (int(x) for x in self.gascon)
        if self.flagh2p:
            s.hfp, s.dfp = f(self.hfp), f(self.dfp)
        s.tsurf, s.fwhm = float(self.tsurf), float(self.fwhm)
        s.radius1, s.radextra = float(self.radius1), float(self.radextra)
        s.nem, s.vem, s.emissivity = len(self.vem), f(self.vem), f(self.emissivity)
        if self.conv is not None:
            cs = self.conv.as_struct()
            s.conv = C.pointer(cs)
            s._keep_conv = cs
        s._keep = self   # keep the arrays alive with the struct
        return s

    @property
    def nconv(self) -> int:
        return self.nwave if self.conv is None else len(self.conv.vconv)

    def out_shapes(self):
        nc = self.nconv
        return (self.npath * nc,), (self.npath * self.nv * nc,), (self.npath * nc,)


def _levels(nlayer):
    p_lev = np.geomspace(10.0, 1e-4, nlayer + 1) * 1e5      # Pa, bottom first
    p_lay = np.sqrt(p_lev[:-1] * p_lev[1:])
    return p_lev, p_lay


def temperature_profile(p_pa, rng, noise=3.0):
    """Smooth 110-170 K profile in ln p (tanh) plus seeded N(0, noise) K."""
    x = np.log(p_pa / 1e5)            # ln(p / bar): +2.3 at 10 bar, -9.2 at 1e-4 bar
    t = 140.0 + 30.0 * np.tanh((x + 2.0) / 2.5)
    return t + noise * rng.standard_normal(p_pa.shape)


def make_job(tables: KTables, absorbers, *, nlayer, seed, iw0=0, nwave=None, theta_deg=0.0,
             vmr_perturb=0.0, ld_lay=None, temp=None, xscale=None) -> Job:
    """Nadir thermal-emission job on `nlayer` layers (10 -> 1e-4 bar).

    State vector (NX = nlayer + len(absorbers)): model-0 temperature at each
    level (xmap = 1) and one model-3 scale factor per absorber
    (xmap = vmr * exp(x), nemesis/subprofretg.f:735-741)."""
    rng = np.random.default_rng(seed)
    L = int(nlayer)
    ld = int(ld_lay or L)
    p_lev, p_lay = _levels(L)
    t_default = temperature_profile(p_lay, rng)     # always drawn: keeps the seeded stream aligned
    temp = t_default if temp is None else np.asarray(temp, np.float64)
    gases = [H2, HE] + list(absorbers)
    ng_ = len(gases)
    ncol = (p_lev[:-1] - p_lev[1:]) / (MMW * AMU * GRAV) * 1e-4          # molecules cm-2
    H = KB * temp / (MMW * AMU * GRAV) / 1e3                                # km
    delh = H * np.log(p_lev[:-1] / p_lev[1:])
    vmr = np.zeros((L, ng_))
    for k, g in enumerate(gases):
        prof = np.full(L, VMR[g])
        if vmr_perturb > 0 and k >= 2:
            prof = prof * np.exp(vmr_perturb * rng.standard_normal(L))
        vmr[:, k] = prof
    if xscale is None:
        xscale = np.zeros(len(absorbers))
    xscale = np.asarray(xscale, np.float64)
    vmr_eff = vmr.copy()
    vmr_eff[:, 2:] *= np.exp(xscale)[None, :]
    press_atm = (p_lay / 1e5 * BAR_TO_ATM).astype(np.float32)

    def fa(shape):
        return np.zeros(shape, np.float32, order="F")

    pp = fa((ld, ng_))
    amount = fa((ld, ng_))
    pp[:L] = (vmr_eff * press_atm[:, None].astype(np.float64)).astype(np.float32)
    amount[:L] = (vmr_eff * ncol[:, None]).astype(np.float32)
    tab_of = {g: i for i, g in enumerate(tables.gases)}
    ktab = np.array([tab_of.get(g, -1) for g in gases], np.int32)
    nbin = int(tables.nbin[0])
    if nwave is None:
        nwave = nbin - iw0
    vwave = (tables.vmin[0] + tables.delv[0] * np.arange(iw0, iw0 + nwave, dtype=np.float32)).astype(np.float32)
    layinc = np.zeros((ld, 1), np.int32, order="F")
    layinc[:L, 0] = np.arange(L, 0, -1)          # top layer first (atmg.f:348-352)
    scale = fa((ld, 1))
    scale[:L, 0] = np.float32(1.0 / np.cos(np.deg2rad(theta_deg)))
    emtemp = fa((ld, 1))
    emtemp[:L, 0] = temp.astype(np.float32)[layinc[:L, 0] - 1]
    npro = L
    dte = fa((ld, npro))
    dam = fa((ld, npro))
    idx = np.arange(L)
    dte[idx, idx] = 1.0
    dam[idx, idx] = ncol.astype(np.float32)
    nparam = ng_ + 1
    nv = L + len(absorbers)
    xmap = np.zeros((nv, nparam, npro), np.float32, order="F")
    xmap[idx, ng_, idx] = 1.0                                  # temperature, model 0
    for a in range(len(absorbers)):
        xmap[L + a, 2 + a, :] = (vmr[:, 2 + a] * np.exp(xscale[a])).astype(np.float32)
    return Job(nlayer=L, ngas=ng_, npath=1, npro=npro, nv=nv, nwave=int(nwave), ld_lay=ld, ld_v=nv,
               ld_param=nparam, press=np.ascontiguousarray(press_atm), temp=temp.astype(np.float32),
               delh=delh.astype(np.float32), pp=pp, amount=amount,
               idgas=np.array([g[0] for g in gases], np.int32), isogas=np.array([g[1] for g in gases], np.int32),
               ktab=ktab, nlayin=np.array([L], np.int32), imod=np.array([3], np.int32), layinc=layinc,
               scale=scale, emtemp=emtemp, dte=dte, dam=dam, xmap=xmap, vwave=vwave,
               vem=np.array([0.0, 1e5], np.float32), emissivity=np.array([1.0, 1.0], np.float32),
               vmr=vmr, ncol=ncol, xscale=xscale)


@dataclasses.dataclass
class Profile:
    """A .prf-style level profile (the rtb_profile structure): heights (km,
    ascending), pressures (atm), temperatures (K) and volume mixing ratios
    [npro, nvmr] of `gases` ([H2, He] + absorbers)."""
    h: np.ndarray
    p: np.ndarray
    t: np.ndarray
    vmr: np.ndarray
    gases: list
    molwt: float = MMW
    radius: float = 71492.0          # km (Jupiter)

    @property
    def npro(self):
        return len(self.h)

    def as_struct(self) -> _abi.RtbProfile:
        s = _abi.RtbProfile()
        f = _abi.fptr
        s.npro, s.nvmr, s.ndust, s.ld_pro, s.ld_con = self.npro, self.vmr.shape[1], 0, self.npro, 0
        s.h, s.p, s.t, s.vmr, s.dust = f(self.h), f(self.p), f(self.t), f(self.vmr), None
        s.molwt, s.radius = float(self.molwt), float(self.radius)
        s._keep = self
        return s


def make_profile(absorbers, *, npro, seed, vmr_perturb=0.3, p_bot_bar=10.0, p_top_bar=1e-4) -> Profile:
    """Level profile of the synthetic atmosphere: pressures log-spaced from
    p_bot to p_top, the smooth seeded T(p) of the layer jobs, hydrostatic
    heights from 0 km at the bottom, and seeded log-normal perturbations of
    the absorbers' mixing ratios."""
    rng = np.random.default_rng(seed)
    p_pa = np.geomspace(p_bot_bar, p_top_bar, npro) * 1e5
    t = temperature_profile(p_pa, rng)
    hs = KB * 0.5 * (t[1:] + t[:-1]) / (MMW * AMU * GRAV) / 1e3              # km
    h = np.concatenate([[0.0], np.cumsum(hs * np.log(p_pa[:-1] / p_pa[1:]))])
    gases = [H2, HE] + list(absorbers)
    vmr = np.zeros((npro, len(gases)))
    for k, g in enumerate(gases):
        prof = np.full(npro, VMR[g])
        if vmr_perturb > 0 and k >= 2:
            prof = prof * np.exp(vmr_perturb * rng.standard_normal(npro))
        vmr[:, k] = prof
    return Profile(h=h.astype(np.float32), p=(p_pa / 1e5 * BAR_TO_ATM).astype(np.float32),
                   t=t.astype(np.float32), vmr=np.asfortranarray(vmr, np.float32), gases=gases)


def job_from_layers(tables: KTables, prof: Profile, lay: dict, *, iw0=0, nwave=None) -> Job:
    """The forward-model job of a layered profile (rtb_layerg / oracle
    layerg outputs in `lay`): layers, the nadir path and the gradient
    matrices, with a state of temperature at every profile level (model 0)
    and one model-3 scale factor per absorber, mapped through DTE / DAM
    (map2pro.f)."""
    L = int(lay["nlay"])
    npro = prof.npro
    gases = prof.gases
    ng_ = len(gases)
    tab_of = {g: i for i, g in enumerate(tables.gases)}
    ktab = np.array([tab_of.get(g, -1) for g in gases], np.int32)
    nbin = int(tables.nbin[0])
    if nwave is None:
        nwave = nbin - iw0
    vwave = (tables.vmin[0] + tables.delv[0] * np.arange(iw0, iw0 + nwave, dtype=np.float32)).astype(np.float32)
    nl = int(lay["nlayin"])

    def col(a, n):
        out = np.zeros((L, 1), np.float32, order="F")
        out[:n, 0] = a[:n]
        return out

    nabs = ng_ - 2
    nparam = ng_ + 1
    nv = npro + nabs
    xmap = np.zeros((nv, nparam, npro), np.float32, order="F")
    idx = np.arange(npro)
    xmap[idx, ng_, idx] = 1.0
    for a in range(nabs):
        xmap[npro + a, 2 + a, :] = prof.vmr[:, 2 + a]
    return Job(nlayer=L, ngas=ng_, npath=1, npro=npro, nv=nv, nwave=int(nwave), ld_lay=L, ld_v=nv,
               ld_param=nparam, press=lay["press"].copy(), temp=lay["temp"].copy(), delh=lay["delh"].copy(),
               pp=np.asfortranarray(lay["pp"]), amount=np.asfortranarray(lay["amount"]),
               idgas=np.array([g[0] for g in gases], np.int32), isogas=np.array([g[1] for g in gases], np.int32),
               ktab=ktab, nlayin=np.array([nl], np.int32), imod=np.array([int(lay["imod"])], np.int32),
               layinc=col(lay["layinc"].astype(np.int32), nl).astype(np.int32), scale=col(lay["scale"], nl),
               emtemp=col(lay["emtemp"], nl), dte=np.asfortranarray(lay["dte"]),
               dam=np.asfortranarray(lay["dam"]), xmap=xmap, vwave=vwave,
               vem=np.array([0.0, 1e5], np.float32), emissivity=np.array([1.0, 1.0], np.float32))


def with_para_h2(job: Job, hfp) -> Job:
    """The job with the para-H2 CIA (flagh2p = 1): layer para fractions hfp,
    DFP the identity on the layers, and one more state element per layer,
    the para fraction of that level (model 0: xmap 1), after the others."""
    L, npro, nv0 = job.nlayer, job.npro, job.nv
    nparam = job.ngas + 2
    nv = nv0 + npro
    xmap = np.zeros((nv, nparam, npro), np.float32, order="F")
    xmap[:nv0, :job.ngas + 1, :] = job.xmap[:nv0, :job.ngas + 1, :]
    idx = np.arange(npro)
    xmap[nv0 + idx, job.ngas + 1, idx] = 1.0
    dfp = np.zeros((job.ld_lay, npro), np.float32, order="F")
    dfp[np.arange(L), np.arange(L)] = 1.0
    return dataclasses.replace(job, nv=nv, ld_v=nv, ld_param=nparam, xmap=xmap, flagh2p=1,
                               hfp=np.ascontiguousarray(hfp, np.float32), dfp=dfp)


def with_dust(job: Job, ncont=2, seed=0, tau=0.4, state=True) -> Job:
    """The job with ncont dust types (cirsradg_wave.f:550-575): layer
    columns cont(k, l) following a Gaussian in ln p around a seeded level,
    scaled to a total vertical optical depth near `tau`; smooth extinction
    cross sections at vwave; DCO the identity on the layers; and (state)
    one state element per dust type, the scale of its whole profile (xmap =
    the column of each level), after the others.  state=False: a fixed
    dust background, its xmap columns zero."""
    assert not job.flagh2p
    rng = np.random.default_rng(seed)
    L, npro, nv0 = job.nlayer, job.npro, job.nv
    lnp = np.log(job.press[:L].astype(np.float64))
    v = job.vwave.astype(np.float64)
    xs = np.zeros((ncont, job.nwave))
    cont = np.zeros((ncont, L))
    for k in range(ncont):
        x0 = 1e-12 * (1.0 + k) * (1.0 + 0.3 * np.sin(v / (40.0 + 25.0 * k) + rng.uniform(0, 6)))
        xs[k] = x0
        shape = np.exp(-0.5 * ((lnp - rng.uniform(lnp.min() + 1, lnp.max() - 1)) / 0.8) ** 2)
        cont[k] = shape / shape.sum() * tau / float(np.mean(x0)) / ncont
    nparam = job.ngas + 1 + ncont
    nv = nv0 + (ncont if state else 0)
    xmap = np.zeros((nv, nparam, npro), np.float32, order="F")
    xmap[:nv0, :job.ngas + 1, :] = job.xmap[:nv0, :job.ngas + 1, :]
    for k in range(ncont if state else 0):
        xmap[nv0 + k, job.ngas + 1 + k, :L] = cont[k].astype(np.float32)
    dco = np.zeros((job.ld_lay, npro), np.float32, order="F")
    dco[np.arange(L), np.arange(L)] = 1.0
    return dataclasses.replace(job, nv=nv, ld_v=nv, ld_param=nparam, xmap=xmap, ncont=ncont,
                               cont=np.asfortranarray(cont.astype(np.float32)),
                               xsec_ext=np.asfortranarray(xs.astype(np.float32)), dco=dco)


def config1(seed=1001):
    tables = make_ktables([CH4], np_=20, nt=10, ng=20, vmin=1200.0, delv=1.5, nbin=100, seed=seed)
    job = make_job(tables, [CH4], nlayer=40, seed=seed + 1)
    return tables, make_cia(seed), job


def config2(seed=1002, nwave=None, nlayer=120, nbin=2000):
    tables = make_ktables(ABSORBERS_C2, np_=20, nt=15, ng=20, vmin=600.0, delv=0.4, nbin=nbin, seed=seed)
    job = make_job(tables, ABSORBERS_C2, nlayer=nlayer, seed=seed + 1, nwave=nwave, vmr_perturb=0.3)
    return tables, make_cia(seed), job


def config3_jobs(tables: KTables, nspec: int, seed=1003):
    """Uneven batch: W ~ U[200, 2000] contiguous window of the config-2 grid,
    L ~ U[40, 120], 1-4 absorbers from the config-2 set, theta ~ U[0, 70] deg."""
    rng = np.random.default_rng(seed)
    nbin = int(tables.nbin[0])
    jobs = []
    for s in range(nspec):
        w = int(rng.integers(200, min(2000, nbin) + 1))
        iw0 = int(rng.integers(0, nbin - w + 1))
        L = int(rng.integers(40, 121))
        na = int(rng.integers(1, 5))
        absorbers = [ABSORBERS_C2[i] for i in sorted(rng.choice(4, size=na, replace=False))]
        theta = float(rng.uniform(0.0, 70.0))
        jobs.append(make_job(tables, absorbers, nlayer=L, seed=int(rng.integers(1 << 30)), iw0=iw0,
                             nwave=w, theta_deg=theta, vmr_perturb=0.3))
    return jobs


# --------------------------------------------------------------------- retrievals
@dataclasses.dataclass
class RetrievalCase:
    """One optimal-estimation retrieval of the layer-state model
    (rtb_retrieval_spec): x[l] = T of layer l, x[nlayer + a] = ln scale of
    gas scale_gas[a].  `job` is the atmosphere at scale factor 1."""
    job: Job
    scale_gas: np.ndarray      # int32 [nscale]
    xa: np.ndarray             # float32 [nx]
    sa: np.ndarray             # float64 [nx, nx]
    sei: np.ndarray            # float64 [ny]
    x_true: np.ndarray         # float32 [nx]
    y: np.ndarray | None = None
    x0: np.ndarray | None = None
    scale_model: np.ndarray | None = None   # int32 [nscale], 3 (log) or 2 (linear); None = all 3
    prof_gas: np.ndarray | None = None      # int32 [nprof] gases retrieved as log-vmr layer profiles
    prof: "Profile | None" = None           # level-state model: the profile re-layered every state
    lopts: dict | None = None               # its layering (rtb_layer_opts fields)
    dust_type: np.ndarray | None = None     # int32 [ndust] dust types whose column is scaled (log), last in x

    @property
    def nx(self):
        return self.job.nv

    @property
    def ny(self):
        return self.job.npath * self.job.nconv

    def as_struct(self):
        s = _abi.RtbRetrievalSpec()
        atm = self.job.as_struct()
        s.atm = C.pointer(atm)
        s.nscale = len(self.scale_gas)
        s.scale_gas = _abi.iptr(self.scale_gas)
        s.y = _abi.fptr(self.y)
        s.sei = _abi.dptr(self.sei)
        s.sa = _abi.dptr(self.sa)
        s.xa = _abi.fptr(self.xa)
        s.x0 = _abi.fptr(self.x0)
        s.scale_model = _abi.iptr(self.scale_model)
        pg = self.prof_gas if self.prof_gas is not None else np.zeros(0, np.int32)
        s.nprof = len(pg)
        s.prof_gas = _abi.iptr(pg) if len(pg) else None
        keep = [self, atm, pg]
        if self.prof is not None:
            ps = self.prof.as_struct()
            o = _abi.RtbLayerOpts()
            lo = dict(laytyp=1, layint=1, layht=float(self.prof.h[0]), layang=0.0, angle=0.0, botlay=1, ipzen=0)
            lo.update(self.lopts or {})
            base = lo.pop("base", None)
            for k, v in lo.items():
                setattr(o, k, v)
            if base is not None:
                base = np.ascontiguousarray(base, np.float32)
                o.base = _abi.fptr(base)
            s.prof, s.lopts = C.pointer(ps), C.pointer(o)
            keep += [ps, o, base]
        if self.dust_type is not None and len(self.dust_type):
            dt = np.ascontiguousarray(self.dust_type, np.int32)
            s.ndust, s.dust_type = len(dt), _abi.iptr(dt)
            keep.append(dt)
        s._keep = keep
        return s


def with_dust_scales(case: RetrievalCase, ncont=2, seed=0, sig=0.5) -> RetrievalCase:
    """The layer-state case through ncont dust types (with_dust) whose column
    profiles are scaled, log scale a priori 0 with sigma `sig` each, last in
    the state vector; the true scales a seeded draw."""
    rng = np.random.default_rng(seed)
    j = with_dust(case.job, ncont, seed=seed, state=False)
    nv0, L = j.nv, j.nlayer
    nv = nv0 + ncont
    xmap = np.zeros((nv, j.nparam, j.npro), np.float32, order="F")
    xmap[:nv0] = j.xmap
    for k in range(ncont):
        xmap[nv0 + k, j.ngas + 1 + k, :L] = j.cont[k]
    job = dataclasses.replace(j, nv=nv, ld_v=nv, xmap=xmap)
    sa = np.zeros((nv, nv))
    sa[:nv0, :nv0] = case.sa
    sa[nv0:, nv0:] = np.eye(ncont) * sig * sig
    xa = np.concatenate([case.xa, np.zeros(ncont, np.float32)]).astype(np.float32)
    x_true = np.concatenate([case.x_true, rng.normal(0.0, sig, ncont)]).astype(np.float32)
    return dataclasses.replace(case, job=job, sa=sa, xa=xa, x_true=x_true, y=None,
                               dust_type=np.arange(ncont, dtype=np.int32))


def prior_covariance(p_lay, n_scale, sig_t=3.0, sig_scale=0.5, clen=1.5):
    """Sa: temperature block with exponential correlation in ln p,
    sqrt(sx_ii sx_jj) exp(-|ln p_i - ln p_j| / clen) (the form of
    nemesis/readapriori.f:239-246), 3 K; uncorrelated log scales, 50 %."""
    lnp = np.log(p_lay)
    L = len(p_lay)
    sa = np.zeros((L + n_scale, L + n_scale))
    sa[:L, :L] = sig_t * sig_t * np.exp(-np.abs(lnp[:, None] - lnp[None, :]) / clen)
    sa[L:, L:] = np.eye(n_scale) * sig_scale * sig_scale
    return sa


def make_retrieval(tables: KTables, absorbers, *, nlayer, seed, iw0=0, nwave=None, theta_deg=0.0,
                   noise=1e-9, vmr_perturb=0.3, scale_model=None, profile=()) -> RetrievalCase:
    """Retrieval case with a priori = smooth T profile and unit gas scales;
    the true state is a seeded draw from Sa.  The measurement y is set by
    the caller (forward model at x_true plus noise, see `observe`).
    scale_model: per scaled absorber 3 (log scale, a priori 0) or 2 (linear
    scale, a priori 1); profile: indices into `absorbers` retrieved as
    log-vmr layer profiles (a priori the job's vmr, 50 %, correlated over
    1.5 scale heights) instead of a scale."""
    rng = np.random.default_rng(seed)
    p_lev, p_lay = _levels(nlayer)
    t_prior = temperature_profile(p_lay, rng, noise=0.0)
    job = make_job(tables, absorbers, nlayer=nlayer, seed=seed + 1, iw0=iw0, nwave=nwave, theta_deg=theta_deg,
                   vmr_perturb=vmr_perturb, temp=t_prior)
    L = nlayer
    prof = [int(a) for a in profile]
    scaled = [a for a in range(len(absorbers)) if a not in prof]
    ns, npf = len(scaled), len(prof)
    sm = np.array(scale_model if scale_model is not None else [3] * ns, np.int32)
    nv = L + ns + npf * L
    xmap = np.zeros((nv, job.nparam, L), np.float32, order="F")
    idx = np.arange(L)
    xmap[idx, job.ngas, idx] = 1.0
    for k, a in enumerate(scaled):
        xmap[L + k, 2 + a, :] = job.vmr[:, 2 + a].astype(np.float32)
    for k, a in enumerate(prof):
        xmap[L + ns + k * L + idx, 2 + a, idx] = job.vmr[:, 2 + a].astype(np.float32)
    job = dataclasses.replace(job, nv=nv, ld_v=nv, xmap=xmap)
    xa = np.concatenate([t_prior, np.where(sm == 2, 1.0, 0.0)] +
                        [np.log(job.vmr[:, 2 + a]) for a in prof]).astype(np.float32)
    sa = np.zeros((nv, nv))
    sa[:L + ns, :L + ns] = prior_covariance(p_lay, ns)
    lnp = np.log(p_lay)
    for k in range(npf):
        o = L + ns + k * L
        sa[o:o + L, o:o + L] = 0.25 * np.exp(-np.abs(lnp[:, None] - lnp[None, :]) / 1.5)
    x_true = (xa + np.linalg.cholesky(sa) @ rng.standard_normal(nv)).astype(np.float32)
    for k in range(ns):
        if sm[k] == 2:
            x_true[L + k] = max(x_true[L + k], np.float32(0.05))
    sei = np.full(job.nwave, 1.0 / (noise * noise))
    return RetrievalCase(job=job, scale_gas=np.array([2 + a for a in scaled], np.int32), xa=xa, sa=sa, sei=sei,
                         x_true=x_true, scale_model=sm if scale_model is not None else None,
                         prof_gas=np.array([2 + a for a in prof], np.int32) if npf else None)


def make_level_retrieval(tables: KTables, absorbers, *, npro, nlay, seed, iw0=0, nwave=None, angle=0.0,
                         noise=1e-9, scale_model=None) -> RetrievalCase:
    """Retrieval case of the level-state model: the state is the temperature
    of each of the npro profile levels plus one scale factor per absorber
    (model 3, or 2 where scale_model says so); every state is re-layered
    into nlay equal-log-pressure Curtis-Godson layers viewed at `angle`.  A
    priori: the smooth T(p) and unit scales; the true state a seeded draw
    from Sa.  The profile's heights stay those of the a priori (the
    reference re-integrates them only when hydrostatic adjustment is on)."""
    rng = np.random.default_rng(seed)
    prof = make_profile(absorbers, npro=npro, seed=seed + 1)
    p_pa = prof.p.astype(np.float64) / BAR_TO_ATM * 1e5
    t_prior = temperature_profile(p_pa, rng, noise=0.0)
    prior = dataclasses.replace(prof, t=t_prior.astype(np.float32))
    ns = len(absorbers)
    sm = np.array(scale_model if scale_model is not None else [3] * ns, np.int32)
    nv = npro + ns
    job = make_job(tables, absorbers, nlayer=nlay, seed=seed + 2, iw0=iw0, nwave=nwave)
    job = dataclasses.replace(job, nv=nv, ld_v=nv, npro=1, xmap=np.zeros((nv, job.nparam, 1), np.float32, order="F"))
    xa = np.concatenate([t_prior, np.where(sm == 2, 1.0, 0.0)]).astype(np.float32)
    sa = prior_covariance(p_pa, ns)
    x_true = (xa + np.linalg.cholesky(sa) @ rng.standard_normal(nv)).astype(np.float32)
    for k in range(ns):
        if sm[k] == 2:
            x_true[npro + k] = max(x_true[npro + k], np.float32(0.05))
    sei = np.full(job.nwave, 1.0 / (noise * noise))
    return RetrievalCase(job=job, scale_gas=np.arange(2, 2 + ns, dtype=np.int32), xa=xa, sa=sa, sei=sei,
                         x_true=x_true, scale_model=sm if scale_model is not None else None, prof=prior,
                         lopts=dict(nlay=nlay, laytyp=1, layint=1, angle=float(angle)))


def with_channels(case: RetrievalCase, fwhm, channels: Channels, noise=1e-9) -> RetrievalCase:
    """The case measured on instrument channels: the atmosphere convolves
    its spectrum and Jacobian with cirsconv (FWHM, channels), and y, Se are
    on the channels."""
    job = dataclasses.replace(case.job, fwhm=float(fwhm), conv=channels)
    return dataclasses.replace(case, job=job, y=None, sei=np.full(job.nconv, 1.0 / (noise * noise)))


def with_paths(case: RetrievalCase, airmass, noise=1e-9) -> RetrievalCase:
    """The case measured along several paths at once (emission angles of one
    footprint): the job's path repeated with its scale factors times each
    airmass; y holds one spectrum per path, path after path."""
    j = case.job
    npth = len(airmass)
    lay = np.zeros((j.ld_lay, npth), np.int32, order="F")
    sc = np.zeros((j.ld_lay, npth), np.float32, order="F")
    em = np.zeros((j.ld_lay, npth), np.float32, order="F")
    for p, f in enumerate(airmass):
        lay[:, p] = j.layinc[:, 0]
        sc[:, p] = j.scale[:, 0] * np.float32(f)
        em[:, p] = j.emtemp[:, 0]
    job = dataclasses.replace(j, npath=npth, layinc=lay, scale=sc, emtemp=em,
                              nlayin=np.full(npth, j.nlayin[0], np.int32), imod=np.full(npth, j.imod[0], np.int32))
    return dataclasses.replace(case, job=job, y=None, sei=np.full(npth * job.nconv, 1.0 / (noise * noise)))


def observe(case: RetrievalCase, spectrum, seed, noise=1e-9):
    """y = F(x_true) + N(0, noise) with F evaluated by the caller."""
    rng = np.random.default_rng(seed)
    case.y = (np.asarray(spectrum, np.float64) + noise * rng.standard_normal(case.ny)).astype(np.float32)
    return case



def job_at_state(case: RetrievalCase, x) -> Job:
    """The case's atmosphere at state x, by the mapping rtb_retrieve_batch
    applies: temp = x[:nlayer] (emtemp along the path), amount, pp and the
    gas's xmap rows times exp(x[nlayer + a]) in float32."""
    j = case.job
    L = j.nlayer
    x = np.asarray(x, np.float32)
    amount, pp, xmap = j.amount.copy(order="F"), j.pp.copy(order="F"), j.xmap.copy(order="F")
    for a, g in enumerate(case.scale_gas):
        f = np.float32(np.exp(np.float64(x[L + a])))
        amount[:L, g] = amount[:L, g] * f
        pp[:L, g] = pp[:L, g] * f
        xmap[:, g, :] = xmap[:, g, :] * f
    temp = x[:L].copy()
    emtemp = j.emtemp.copy(order="F")
    emtemp[:L, 0] = temp[j.layinc[:L, 0] - 1]
    return dataclasses.replace(j, temp=temp, amount=amount, pp=pp, xmap=xmap, emtemp=emtemp)
