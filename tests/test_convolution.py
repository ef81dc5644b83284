"""Instrument convolution (radtran/cirsrad/cirsconv.f:12-246) as
cirsrtfg_wave applies it (cirsrtfg_wave.f:448-516): the .fwh / .fil text
readers and the oracle's restatement (CPU); the device convolution against
the oracle, alone and inside rtb_cirsrtfg_wave (GPU)."""
import numpy as np
import pytest

from radtrancode_b200 import _lib, cirsradg, synth
from radtrancode_b200.synth import Channels


def _series(nw=200, v0=600.0, dv=0.4, seed=0):
    rng = np.random.default_rng(seed)
    vw = (v0 + dv * np.arange(nw)).astype(np.float32)
    y = (1.0 + 0.3 * np.sin(vw / 7.0) + 0.05 * rng.standard_normal(nw)).astype(np.float32)
    return vw, y


def _filters(vc, half=(3.0, 1.0), seed=1):
    """Triangular filter functions, one per channel, 5 points each, plus a
    second (flat) filter for the first channel listed last, which wins."""
    rng = np.random.default_rng(seed)
    pts, vals = [], []
    cen = list(vc)
    for c in vc:
        a, b = half
        pts.append(c + np.array([-a, -b, 0.0, b, a], np.float32))
        vals.append(np.array([0.0, 0.5, 1.0, 0.5, 0.0], np.float32) * (1.0 + 0.1 * rng.random()))
    cen.append(vc[0])
    pts.append(vc[0] + np.array([-9.0, 9.0], np.float32))
    vals.append(np.array([1.0, 1.0], np.float32))
    nsub = [len(p) for p in pts]
    return Channels(vconv=vc, vcen=np.array(cen, np.float32), nsub=np.array(nsub),
                    vfil=np.concatenate(pts), fil=np.concatenate(vals))


# ---------------------------------------------------------------- CPU

def test_read_fwh_and_fil(tmp_path):
    _lib.build()
    p = tmp_path / "run.fwh"
    p.write_text("3   ! number of points\n 600.0, 2.5\n700.0 3.0d0 extra\n\n  800.0\n 3.5\n")
    v, x = cirsradg.read_fwh(p)
    assert v.tolist() == [600.0, 700.0, 800.0] and x.tolist() == [2.5, 3.0, 3.5]
    q = tmp_path / "run.fil"
    q.write_text("2\n650.0\n3\n649.0 0.0\n650.0 1.0\n651.0 0.0\n660.5 centre\n2\n659.0 1.0\n662.0 1.0\n")
    vc, ns, vf, fl = cirsradg.read_fil(q)
    assert vc.tolist() == [650.0, 660.5] and ns.tolist() == [3, 2]
    assert vf.tolist() == [649.0, 650.0, 651.0, 659.0, 662.0] and fl.tolist() == [0.0, 1.0, 0.0, 1.0, 1.0]
    L = _lib.lib()
    import ctypes as C
    n = C.c_int()
    small = np.zeros(2, np.float32)
    from radtrancode_b200 import _abi
    assert L.rtb_read_fwh(str(p).encode(), C.byref(n), _abi.fptr(small), _abi.fptr(small.copy()), 2) == 2
    bad = tmp_path / "bad.fil"
    bad.write_text("1\n650.0\n3\n649.0 0.0\n")
    with pytest.raises(cirsradg.RtbError):
        cirsradg.read_fil(bad)


def test_oracle_conv_modes(oracle):
    vw, y = _series()
    vc = (vw[0] + 5.0 + np.arange(0, 70, 1.5)).astype(np.float32)
    plain = oracle.cirsconv(vw, y, 2.5, vc)
    # a width table that is 2.5 everywhere gives the plain result bit for bit
    ch = Channels(vconv=vc, vfwhm=np.array([500.0, 900.0], np.float32), xfwhm=np.array([2.5, 2.5], np.float32))
    assert np.array_equal(oracle.cirsconv_ex(vw, y, 2.5, ch), plain)
    # a wider bin at one end changes only the channels there; the sum is still divided by FWHM
    ch = Channels(vconv=vc, vfwhm=np.array([vc[0], vc[-1]], np.float32), xfwhm=np.array([5.0, 2.5], np.float32))
    varw = oracle.cirsconv_ex(vw, y, 2.5, ch)
    assert varw[0] == pytest.approx(2.0 * np.mean(y[(vw > vc[0] - 2.5) & (vw < vc[0] + 2.5)]), rel=0.05)
    assert varw[-1] == plain[-1]
    # filters: the filter-weighted mean, within float rounding of a float64 restatement
    chf = _filters(vc)
    got = oracle.cirsconv_ex(vw, y, -1.0, chf)
    dv = np.diff(vw.astype(np.float64))
    for i, c in enumerate(vc):
        k = i if i > 0 else len(vc)          # channel 0: the filter listed last wins
        o = int(np.sum(chf.nsub[:k]))
        w = np.interp(vw, chf.vfil[o:o + chf.nsub[k]], chf.fil[o:o + chf.nsub[k]], left=0.0, right=0.0)
        if k == len(vc):
            w = np.where((vw >= chf.vfil[o]) & (vw <= chf.vfil[o + 1]), 1.0, 0.0)
        ref = np.sum(w[:-1] * y[:-1] * dv) / np.sum(w[:-1] * dv)
        assert got[i] == pytest.approx(ref, rel=1e-6), i
    # one calculated point: 1 (cirsconv.f:45-54); FWHM = 0: a copy
    assert oracle.cirsconv_ex(vw[:1], y[:1], 2.0, Channels(vconv=vw[:1])).tolist() == [1.0]
    assert np.array_equal(oracle.cirsconv_ex(vw, y, 0.0, Channels(vconv=vw[:50])), y[:50])


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_cirsconv_ex_matches_oracle(ctx, oracle):
    """Device cirsconv against the oracle on one spectrum's radiance,
    d/dtsurf and Jacobian rows: a width table (FWHM > 0) within 1e-6 of each
    series' largest value, as the fixed-width case; filter channels
    (FWHM < 0) bit for bit."""
    kt, cia, job = synth.config2(nwave=200, nlayer=40, nbin=200)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, gt = ctx.cirsrtfg_wave(job)
    series = np.vstack([c[None], gt[None], g.reshape(job.nv, job.nwave)])
    vc = (job.vwave[0] + 1.3 + np.arange(0, 76, 1.0)).astype(np.float32)
    chw = Channels(vconv=vc, vfwhm=np.array([vc[0], vc[40], vc[-1]], np.float32),
                   xfwhm=np.array([1.5, 4.0, 2.0], np.float32))
    got = ctx.cirsconv_ex(job.vwave, series, 2.5, chw)
    for s in range(series.shape[0]):
        ref = oracle.cirsconv_ex(job.vwave, series[s], 2.5, chw)
        assert np.max(np.abs(got[s] - ref)) <= 1e-6 * max(np.max(np.abs(ref)), 1e-30), s
    chf = _filters(vc[2:-2])
    got = ctx.cirsconv_ex(job.vwave, series, -1.0, chf)
    for s in range(series.shape[0]):
        assert np.array_equal(got[s], oracle.cirsconv_ex(job.vwave, series[s], -1.0, chf)), s
    one = ctx.cirsconv_ex(job.vwave[:1], series[:3, :1], 2.0, Channels(vconv=job.vwave[:1]))
    assert one.tolist() == [[1.0], [1.0], [1.0]]
    nofil = Channels(vconv=np.array([vc[0], vc[0] + 0.37], np.float32), vcen=chf.vcen, nsub=chf.nsub,
                     vfil=chf.vfil, fil=chf.fil)
    with pytest.raises(cirsradg.RtbError):
        ctx.cirsconv_ex(job.vwave, series, -1.0, nofil)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fwhm", "table", "filter", "copy"])
def test_cirsrtfg_wave_convolves_outputs(ctx, oracle, mode):
    """rtb_cirsrtfg_wave with channels: every output (radiance, d/dtsurf, each
    Jacobian row) is the oracle's cirsconv of the calculation-grid output, and
    is packed with nconv (cirsrtfg_wave.f:448-516).  A batch that mixes
    convolved and calculation-grid spectra gives the same as one call each."""
    kt, cia, job = synth.config2(nwave=160, nlayer=40, nbin=200)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c0, g0, gt0 = ctx.cirsrtfg_wave(job)
    vc = (job.vwave[0] + 2.1 + np.arange(0, 58, 1.2)).astype(np.float32)
    if mode == "fwhm":
        fwhm, ch = 1.8, Channels(vconv=vc)
    elif mode == "table":
        fwhm, ch = 1.8, Channels(vconv=vc, vfwhm=np.array([vc[0], vc[-1]], np.float32),
                                 xfwhm=np.array([1.2, 3.0], np.float32))
    elif mode == "filter":
        fwhm, ch = -1.0, _filters(vc[3:-3], half=(2.0, 0.8))
    else:
        fwhm, ch = 0.0, Channels(vconv=job.vwave[:90])
    import dataclasses
    jc = dataclasses.replace(job, fwhm=fwhm, conv=ch)
    c, g, gt = ctx.cirsrtfg_wave(jc)
    nc = len(ch.vconv)
    assert c.shape == (nc,) and g.shape == (job.nv * nc,)
    g0r = g0.reshape(job.nv, job.nwave)
    exact = mode in ("filter", "copy")
    for s, (got, src) in enumerate([(c, c0), (gt, gt0)] + [(g[iv * nc:(iv + 1) * nc], g0r[iv])
                                                            for iv in range(job.nv)]):
        ref = oracle.cirsconv_ex(job.vwave, src, fwhm, ch)
        if exact:
            assert np.array_equal(got, ref), s
        else:
            assert np.max(np.abs(got - ref)) <= 1e-6 * max(np.max(np.abs(ref)), 1e-30), s
    outs = ctx.cirsrtfg_wave_batch([job, jc, job])
    assert np.array_equal(outs[1][0], c) and np.array_equal(outs[1][1], g) and np.array_equal(outs[1][2], gt)
    assert np.array_equal(outs[0][0], c0) and np.array_equal(outs[2][1], g0)
