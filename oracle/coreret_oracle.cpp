/*
 * coreret_oracle.cpp -- ORACLE (test infrastructure only; see oracle.h).
 *
 * Restatement of the retrieval loop of nemesis/coreret.f:520-1106 for the
 * layer-state model of rtb_retrieve_batch (include/radtran_b200.h):
 * temperatures per layer (model 0, nemesis/subprofretg.f:638-651) and log
 * gas scale factors (model 3, subprofretg.f:735-750, X1 = XREF*EXP(XN)).
 * Each step uses the oracle's own forward model (orc_cirsrtfg_wave) and the
 * reference's dense Newton algebra (orc_calc_gain_matrix_diag, which forms
 * D and AA, then orc_calcnextxn and orc_calc_phiret_diag).
 */
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

// compact copy of the atmosphere at scale factor 1 and its state layout
struct Work {
    rtb_atm a{};
    int L = 0, NV = 0, nparam = 0, NW = 0, NP = 1;   /* NP paths: y and K hold them path after path */
    /* the measurement's channels (cirsrtfg_wave.f:520-560 convolves the
     * spectrum and every Jacobian row onto them); NY = nconv, or NW */
    int NY = 0;
    float fwhm = 0.0f;
    const rtb_conv* cv = nullptr;
    std::vector<float> temp, pp, amount, emtemp, xmap, pp0, amount0, xmap0;
    std::vector<float> press, delh, scale, dte, dam, dco, vwave;
    std::vector<int> dust;              /* dust types whose column is scaled (model 3 on an aerosol) */
    std::vector<float> cont, cont0;     /* [nlayer][ncont] */
    std::vector<int> layinc, idgas, isogas, ktab, nlayin, imod, sg, sm, pg;
    std::vector<float> vmr0;   /* [nprof][L] pp / press of the profiled gases */
    /* level-state model: L counts the profile's levels (the state's temperatures) */
    bool level = false;
    rtb_profile pr{};
    rtb_layer_opts lo{};
    std::vector<float> ph, pp_atm, pt, pvmr0, pvmr, lbase;
};

int setup_level(const rtb_retrieval_spec& s, Work& w) {
    const rtb_atm& t = *s.atm;
    const rtb_profile& P = *s.prof;
    const int G = t.ngas, NPRO = P.npro, NV = t.nv, NW = t.nwave, NL = s.lopts->nlay;
    if (P.nvmr != G || P.ndust != 0 || NV != NPRO + s.nscale + s.nprof * NPRO) return RTB_ERR_UNSUPPORTED;
    w.level = true;
    w.L = NPRO;
    w.NV = NV;
    w.NW = NW;
    w.nparam = G + 1;
    w.sg.assign(s.scale_gas, s.scale_gas + s.nscale);
    w.sm.assign(s.nscale, 3);
    if (s.scale_model) w.sm.assign(s.scale_model, s.scale_model + s.nscale);
    w.pg.assign(s.prof_gas, s.prof_gas + s.nprof);
    const int ldp = P.ld_pro > 0 ? P.ld_pro : NPRO;
    w.ph.assign(P.h, P.h + NPRO);
    w.pp_atm.assign(P.p, P.p + NPRO);
    w.pt.assign(P.t, P.t + NPRO);
    w.pvmr0.resize((size_t)G * NPRO);
    for (int g = 0; g < G; ++g)
        for (int l = 0; l < NPRO; ++l) w.pvmr0[l + (size_t)NPRO * g] = P.vmr[l + (size_t)ldp * g];
    w.pvmr = w.pvmr0;
    w.pr = P;
    w.pr.ld_pro = NPRO;
    w.pr.h = w.ph.data();
    w.pr.p = w.pp_atm.data();
    w.pr.t = w.pt.data();
    w.pr.vmr = w.pvmr.data();
    w.lo = *s.lopts;
    if (w.lo.laytyp >= 4 && w.lo.base) w.lbase.assign(w.lo.base, w.lo.base + NL);
    w.lo.base = w.lbase.empty() ? nullptr : w.lbase.data();
    w.press.assign(NL, 0.0f);
    w.temp.assign(NL, 0.0f);
    w.delh.assign(NL, 0.0f);
    w.pp.assign((size_t)NL * G, 0.0f);
    w.amount.assign((size_t)NL * G, 0.0f);
    w.dte.assign((size_t)NL * NPRO, 0.0f);
    w.dam.assign((size_t)NL * NPRO, 0.0f);
    w.scale.assign(NL, 0.0f);
    w.emtemp.assign(NL, 0.0f);
    w.layinc.assign(NL, 0);
    w.nlayin.assign(1, 0);
    w.imod.assign(1, 3);
    w.xmap.assign((size_t)NV * w.nparam * NPRO, 0.0f);
    w.vwave.assign(t.vwave, t.vwave + NW);
    w.idgas.assign(t.idgas, t.idgas + G);
    w.isogas.assign(t.isogas, t.isogas + G);
    w.ktab.assign(t.ktab, t.ktab + G);
    w.a = t;
    w.a.nlayer = NL;
    w.a.npath = 1;
    w.a.npro = NPRO;
    w.a.ld_lay = NL;
    w.a.ld_v = NV;
    w.a.ld_param = w.nparam;
    w.a.press = w.press.data();
    w.a.temp = w.temp.data();
    w.a.delh = w.delh.data();
    w.a.pp = w.pp.data();
    w.a.amount = w.amount.data();
    w.a.idgas = w.idgas.data();
    w.a.isogas = w.isogas.data();
    w.a.ktab = w.ktab.data();
    w.a.nlayin = w.nlayin.data();
    w.a.imod = w.imod.data();
    w.a.layinc = w.layinc.data();
    w.a.scale = w.scale.data();
    w.a.emtemp = w.emtemp.data();
    w.a.dte = w.dte.data();
    w.a.dam = w.dam.data();
    w.a.dco = nullptr;
    w.a.dfp = nullptr;
    w.a.xmap = w.xmap.data();
    w.a.vwave = w.vwave.data();
    w.a.conv = nullptr;
    return RTB_OK;
}

/* subprofretg.f models 0 / 2 / 3 on every level of the profile, then
 * LAYERG + ATMG (the oracle's own, orc_layerg) */
int at_level_state(Work& w, const float* x) {
    const int NPRO = w.L, NV = w.NV, np_ = w.nparam, G = w.a.ngas;
    for (int l = 0; l < NPRO; ++l) w.pt[l] = x[l];
    w.pvmr = w.pvmr0;
    std::fill(w.xmap.begin(), w.xmap.end(), 0.0f);
    for (int l = 0; l < NPRO; ++l) w.xmap[l + (size_t)NV * (G + (size_t)np_ * l)] = 1.0f;     /* XMAP = 1.0 */
    const int ns = (int)w.sg.size();
    for (int a = 0; a < ns; ++a) {
        const int g = w.sg[a];
        const bool lin = w.sm[a] == 2;
        const float f = lin ? x[NPRO + a] : expf(x[NPRO + a]);
        for (int l = 0; l < NPRO; ++l) {
            const float xref = w.pvmr0[l + (size_t)NPRO * g];
            const float x1 = xref * f;                     /* X1(J) = XREF(J)*EXP(XN) or XREF(J)*XN */
            w.pvmr[l + (size_t)NPRO * g] = x1;
            w.xmap[(NPRO + a) + (size_t)NV * (g + (size_t)np_ * l)] = lin ? xref : x1;
        }
    }
    for (size_t p = 0; p < w.pg.size(); ++p) {
        const int g = w.pg[p];
        const int base = NPRO + ns + (int)p * NPRO;
        for (int l = 0; l < NPRO; ++l) {
            const float v = expf(x[base + l]);
            w.pvmr[l + (size_t)NPRO * g] = v;
            w.xmap[(base + l) + (size_t)NV * (g + (size_t)np_ * l)] = v;
        }
    }
    rtb_layers out;
    std::memset(&out, 0, sizeof out);
    int npath = 0;
    out.ld_lay = w.a.nlayer;
    out.delh = w.delh.data();
    out.press = w.press.data();
    out.temp = w.temp.data();
    out.amount = w.amount.data();
    out.pp = w.pp.data();
    out.dte = w.dte.data();
    out.dam = w.dam.data();
    out.npath = &npath;
    out.nlayin = w.nlayin.data();
    out.imod = w.imod.data();
    out.layinc = w.layinc.data();
    out.scale = w.scale.data();
    out.emtemp = w.emtemp.data();
    return orc_layerg(&w.pr, &w.lo, &out);
}

int setup_layers(const rtb_retrieval_spec& s, Work& w) {
    const rtb_atm& t = *s.atm;
    if (t.npath < 1 || t.npro != t.nlayer || t.nv != t.nlayer + s.nscale + s.nprof * t.nlayer + s.ndust ||
        t.ncont < 0 || s.ndust < 0 || (s.ndust > 0 && (!s.dust_type || t.ncont == 0 || !t.dco)))
        return RTB_ERR_UNSUPPORTED;
    for (int p = 0; p < t.npath; ++p)
        if (t.nlayin[p] > t.nlayer) return RTB_ERR_UNSUPPORTED;
    const int L = t.nlayer, G = t.ngas, NV = t.nv, NW = t.nwave;
    const int ldl = t.ld_lay > 0 ? t.ld_lay : RTB_MAXLAY;
    const int ldv = t.ld_v > 0 ? t.ld_v : RTB_MAXV;
    const int ldp = t.ld_param > 0 ? t.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    w.L = L;
    w.NV = NV;
    w.NW = NW;
    w.nparam = G + 1 + t.ncont;   /* dust: a fixed background, its columns of xmap zero */
    w.sg.assign(s.scale_gas, s.scale_gas + s.nscale);
    w.sm.assign(s.nscale, 3);
    if (s.scale_model) w.sm.assign(s.scale_model, s.scale_model + s.nscale);
    w.pg.assign(s.prof_gas, s.prof_gas + s.nprof);
    auto col = [&](const float* p, int n, std::vector<float>& v) {
        v.resize((size_t)L * n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < L; ++i) v[i + (size_t)L * j] = p[i + (size_t)ldl * j];
    };
    col(t.press, 1, w.press);
    col(t.temp, 1, w.temp);
    col(t.delh, 1, w.delh);
    col(t.pp, G, w.pp0);
    col(t.amount, G, w.amount0);
    w.NP = t.npath;
    col(t.scale, w.NP, w.scale);
    col(t.emtemp, w.NP, w.emtemp);
    col(t.dte, L, w.dte);
    col(t.dam, L, w.dam);
    if (t.ncont > 0 && t.dco) col(t.dco, L, w.dco);
    if (t.ncont > 0) {   /* a working copy of the dust columns, scaled per state */
        const int ldc = t.ld_con > 0 ? t.ld_con : RTB_MAXCON;
        w.cont0.resize((size_t)t.ncont * L);
        for (int l = 0; l < L; ++l)
            for (int k = 0; k < t.ncont; ++k) w.cont0[k + (size_t)t.ncont * l] = t.cont[k + (size_t)ldc * l];
        w.cont = w.cont0;
        w.dust.assign(s.dust_type, s.dust_type + s.ndust);
    }
    w.pp = w.pp0;
    w.amount = w.amount0;
    w.layinc.resize((size_t)L * w.NP);
    for (int p = 0; p < w.NP; ++p)
        for (int i = 0; i < L; ++i) w.layinc[i + (size_t)L * p] = t.layinc[i + (size_t)ldl * p];
    w.xmap0.resize((size_t)NV * w.nparam * L);
    for (int k = 0; k < L; ++k)
        for (int j = 0; j < w.nparam; ++j)
            for (int i = 0; i < NV; ++i)
                w.xmap0[i + (size_t)NV * (j + (size_t)w.nparam * k)] = t.xmap[i + (size_t)ldv * (j + (size_t)ldp * k)];
    w.xmap = w.xmap0;
    w.vmr0.resize((size_t)s.nprof * L);
    for (int p = 0; p < s.nprof; ++p)
        for (int l = 0; l < L; ++l) w.vmr0[(size_t)p * L + l] = w.pp0[l + (size_t)L * s.prof_gas[p]] / w.press[l];
    w.vwave.assign(t.vwave, t.vwave + NW);
    w.idgas.assign(t.idgas, t.idgas + G);
    w.isogas.assign(t.isogas, t.isogas + G);
    w.ktab.assign(t.ktab, t.ktab + G);
    w.nlayin.assign(t.nlayin, t.nlayin + w.NP);
    w.imod.assign(t.imod, t.imod + w.NP);
    w.a = t;
    w.a.ld_lay = L;
    w.a.ld_v = NV;
    w.a.ld_param = w.nparam;
    w.a.press = w.press.data();
    w.a.temp = w.temp.data();
    w.a.delh = w.delh.data();
    w.a.pp = w.pp.data();
    w.a.amount = w.amount.data();
    w.a.idgas = w.idgas.data();
    w.a.isogas = w.isogas.data();
    w.a.ktab = w.ktab.data();
    w.a.nlayin = w.nlayin.data();
    w.a.imod = w.imod.data();
    w.a.layinc = w.layinc.data();
    w.a.scale = w.scale.data();
    w.a.emtemp = w.emtemp.data();
    w.a.dte = w.dte.data();
    w.a.dam = w.dam.data();
    w.a.dco = w.dco.empty() ? nullptr : w.dco.data();   /* xsec_ext: the caller's array */
    if (t.ncont > 0) {
        w.a.cont = w.cont.data();
        w.a.ld_con = t.ncont;
    }
    w.a.dfp = nullptr;
    w.a.xmap = w.xmap.data();
    w.a.vwave = w.vwave.data();
    return RTB_OK;
}

void at_state(Work& w, const float* x) {
    if (w.level) return;   /* forward() re-layers through at_level_state */
    const int L = w.L;
    for (int l = 0; l < L; ++l) w.temp[l] = x[l];
    for (int p = 0; p < w.NP; ++p)
        for (int j = 0; j < w.nlayin[p]; ++j) w.emtemp[j + (size_t)L * p] = w.temp[w.layinc[j + (size_t)L * p] - 1];
    const int ns = (int)w.sg.size();
    for (int a = 0; a < ns; ++a) {
        const int g = w.sg[a];
        const bool lin = w.sm[a] == 2;                   /* model 2: X1 = XREF*XN (subprofretg.f:725-733) */
        const float f = lin ? x[L + a] : expf(x[L + a]); /* model 3: REAL EXP of subprofretg.f:746 */
        for (int l = 0; l < L; ++l) {
            w.amount[l + (size_t)L * g] = w.amount0[l + (size_t)L * g] * f;
            w.pp[l + (size_t)L * g] = w.pp0[l + (size_t)L * g] * f;
        }
        for (int k = 0; k < L; ++k)
            for (int i = 0; i < w.NV; ++i) {
                const size_t idx = i + (size_t)w.NV * (g + (size_t)w.nparam * k);
                w.xmap[idx] = lin ? w.xmap0[idx] : w.xmap0[idx] * f;
            }
    }
    /* model 0 for a gas: X1(I) = EXP(XN(I)), XMAP(I, IPAR, I) = X1(I) (subprofretg.f:638-651) */
    for (size_t p = 0; p < w.pg.size(); ++p) {
        const int g = w.pg[p];
        const int base = L + ns + (int)p * L;
        for (int l = 0; l < L; ++l) {
            const float v = expf(x[base + l]);
            const float f = v / w.vmr0[p * L + l];
            w.amount[l + (size_t)L * g] = w.amount0[l + (size_t)L * g] * f;
            w.pp[l + (size_t)L * g] = w.pp0[l + (size_t)L * g] * f;
            for (int k = 0; k < L; ++k)
                w.xmap[(base + l) + (size_t)w.NV * (g + (size_t)w.nparam * k)] = k == l ? v : 0.0f;
        }
    }
    /* dust scales: model 3 on the type's column profile (subprofretg.f:735-750) */
    const int NC = w.a.ncont;
    const int dbase = L + ns + (int)w.pg.size() * L;
    for (size_t d = 0; d < w.dust.size(); ++d) {
        const int k = w.dust[d];
        const float f = expf(x[dbase + (int)d]);
        for (int l = 0; l < L; ++l) w.cont[k + (size_t)NC * l] = w.cont0[k + (size_t)NC * l] * f;
        const int q = w.a.ngas + 1 + k;
        for (int lev = 0; lev < L; ++lev)
            for (int i = 0; i < w.NV; ++i) {
                const size_t idx = i + (size_t)w.NV * (q + (size_t)w.nparam * lev);
                w.xmap[idx] = w.xmap0[idx] * f;
            }
    }
}

int setup(const rtb_retrieval_spec& s, Work& w) {
    const int r = s.prof ? setup_level(s, w) : setup_layers(s, w);
    if (r) return r;
    const rtb_atm& t = *s.atm;
    w.NY = w.NW;
    if (t.conv && t.conv->nconv > 0) {
        w.fwhm = t.fwhm;
        w.cv = t.conv;
        w.NY = t.conv->nconv;
    } else if (t.fwhm != 0.0f) {
        return RTB_ERR_ARG;
    }
    w.NY *= w.NP;   /* the measurement: every path's spectrum, path after path */
    w.a.fwhm = 0.0f;
    w.a.conv = nullptr;
    return w.NV < w.NY ? RTB_OK : RTB_ERR_UNSUPPORTED;
}

/* forwardavfovX stand-in: spectrum and kk (ny, nx) REAL at state x */
int forward(const orc_tables* tab, Work& w, const float* x, int precision, int nthreads, std::vector<float>& yn,
            std::vector<float>& kk) {
    if (w.level) {
        const int r = at_level_state(w, x);
        if (r) return r;
    } else {
        at_state(w, x);
    }
    const int NP = w.NP, NW = w.NW, NV = w.NV;
    std::vector<double> c((size_t)NP * NW), g((size_t)NP * NV * NW);   /* [path][wave], [path][iv][wave] */
    const int r = orc_cirsrtfg_wave_mt(tab, &w.a, precision, c.data(), g.data(), nullptr, nthreads, nullptr);
    if (r) return r;
    /* per path: the spectrum and the Jacobian rows, cirsconv'd onto the channels when there are any */
    const int ny1 = w.NY / NP;
    yn.resize(w.NY);
    kk.resize((size_t)NV * w.NY);   /* kk[iv * NY + p * ny1 + i] */
    std::vector<float> src(NW), dst(ny1);
    auto conv1 = [&](const std::vector<float>& in, std::vector<float>& out) {
        if (!w.cv) {
            std::copy(in.begin(), in.begin() + ny1, out.begin());
            return 0;
        }
        const rtb_conv& v = *w.cv;
        return orc_cirsconv_ex(w.fwhm, NW, w.vwave.data(), in.data(), v.nconv, v.vconv, v.nfwhm, v.vfwhm, v.xfwhm,
                               v.nfil, v.vcen, v.nsub, v.vfil, v.fil, out.data());
    };
    for (int p = 0; p < NP; ++p) {
        for (int i = 0; i < NW; ++i) src[i] = (float)c[(size_t)p * NW + i];
        int e = conv1(src, dst);
        if (e) return e;
        std::copy(dst.begin(), dst.end(), yn.begin() + (size_t)p * ny1);
        for (int iv = 0; iv < NV; ++iv) {
            for (int i = 0; i < NW; ++i) src[i] = (float)g[((size_t)p * NV + iv) * NW + i];
            e = conv1(src, dst);
            if (e) return e;
            std::copy(dst.begin(), dst.end(), kk.begin() + (size_t)iv * w.NY + (size_t)p * ny1);
        }
    }
    return RTB_OK;
}

}  // namespace

extern "C" {

int orc_forward_state(const orc_tables* tab, const rtb_retrieval_spec* s, const float* x, int precision,
                      int nthreads, float* yn, float* kk) {
    Work w;
    int r = setup(*s, w);
    if (r) return r;
    std::vector<float> y, k;
    r = forward(tab, w, x, precision, nthreads, y, k);
    if (r) return r;
    if (yn) std::memcpy(yn, y.data(), y.size() * 4);
    if (kk) std::memcpy(kk, k.data(), k.size() * 4);
    return RTB_OK;
}

int orc_retrieve(const orc_tables* tab, const rtb_retrieval_spec* s, const rtb_retrieval_opts* o, int precision,
                 int nthreads, rtb_retrieval_result* res, orc_retrieval_trace* tr) {
    Work w;
    int r = setup(*s, w);
    if (r) return r;
    const int nx = w.NV, ny = w.NY, L = w.L;
    std::vector<float> xa(s->xa, s->xa + nx), xn(nx), xn1(nx), x_out(nx);
    for (int i = 0; i < nx; ++i) xn[i] = s->x0 ? s->x0[i] : s->xa[i];
    std::vector<double> sai((size_t)nx * nx), dd((size_t)nx * ny), aa((size_t)nx * nx);
    /* sa is symmetric: row-major equals the column-major (mx, mx) of the reference */
    orc_dinvertm_chol(nx, nx, s->sa, sai.data());
    std::vector<float> yn, kk, yn1, kk1;
    int forwards = 0;
    r = forward(tab, w, xn.data(), precision, nthreads, yn, kk);
    if (r) return r;
    forwards++;
    orc_calc_gain_matrix_diag(nx, ny, nx, ny, kk.data(), sai.data(), s->sei, dd.data(), aa.data(), nullptr);
    float chisq = 0.0f;
    float phi = orc_calc_phiret_diag(ny, s->y, yn.data(), s->sei, nx, nx, xn.data(), xa.data(), sai.data(), &chisq);
    float ophi = phi, ochisq = chisq, alambda = 1.0f;
    int converged = 0, iter = 0;
    if (tr) tr->n = 0;
    for (iter = 1; iter <= o->kiter; ++iter) {
        orc_calcnextxn(nx, ny, nx, xa.data(), xn.data(), s->y, yn.data(), dd.data(), aa.data(), x_out.data());
        bool ok = true;
        for (int i = 0; i < nx && ok; ++i) {
            xn1[i] = xn[i] + (x_out[i] - xn[i]) / (1.0f + alambda);
            if (std::isnan(xn1[i])) {
                alambda = alambda * 10.0f;
                if (alambda > 1e10f) alambda = 1e10f;
                ok = false;
            } else if (i >= L && !(i < L + s->nscale && s->scale_model && s->scale_model[i - L] == 2) &&
                       (xn1[i] > 85.0f || xn1[i] < -85.0f)) {   /* lx = 1: models 3 and gas model 0 */
                alambda = 1e10f;
                ok = false;
            }
        }
        /* subprofretg ierr = 1: a vmr gone negative (model-2 scale < 0), coreret.f:683-700 */
        for (int a = 0; a < s->nscale && ok; ++a)
            if (s->scale_model && s->scale_model[a] == 2 && xn1[L + a] < 0.0f) {
                alambda = alambda * 10.0f;
                if (alambda > 1e10f) alambda = 1e10f;
                ok = false;
            }
        for (int i = 0; i < L && ok; ++i)
            if (xn1[i] < 1.0f) {
                alambda = alambda * 10.0f;
                if (alambda > 1e10f) alambda = 1e10f;
                ok = false;
            }
        float phi1 = 0.0f, chisq1 = 0.0f;
        int verdict = 0;   /* 0 rejected before the forward model, 1 accepted, 2 rejected */
        bool stop = false;
        if (ok) {
            r = forward(tab, w, xn1.data(), precision, nthreads, yn1, kk1);
            if (r) return r;
            forwards++;
            phi1 = orc_calc_phiret_diag(ny, s->y, yn1.data(), s->sei, nx, nx, xn1.data(), xa.data(), sai.data(),
                                        &chisq1);
            const float tphi = 100.0f * (ophi - phi1) / ophi;
            const float abstphi = std::fabs(tphi);
            if (phi1 <= ophi) {
                verdict = 1;
                xn = xn1;
                yn = yn1;
                kk = kk1;
                phi = phi1;
                orc_calc_gain_matrix_diag(nx, ny, nx, ny, kk.data(), sai.data(), s->sei, dd.data(), aa.data(),
                                          nullptr);
                const float dchi = std::fabs(ochisq - chisq1);
                chisq = chisq1;
                if (tphi >= 0.0f && tphi <= o->phlimit && alambda < 1.0f) {
                    converged = 1;
                    stop = true;
                } else {
                    ophi = phi1;
                    alambda = alambda * 0.3f;
                }
                if (!stop && o->dchisq_stop > 0.0f && dchi < o->dchisq_stop) {
                    converged = 3;
                    stop = true;
                }
                ochisq = chisq1;
            } else if (iter >= 5 && abstphi <= o->phlimit) {
                if (alambda < 0.1f) {
                    alambda = alambda * 10.0f;
                    verdict = 2;
                } else {
                    verdict = 1;
                    xn = xn1;
                    yn = yn1;
                    kk = kk1;
                    phi = phi1;
                    chisq = chisq1;
                    converged = 2;
                    stop = true;
                }
            } else {
                verdict = 2;
                alambda = alambda * 10.0f;
                if (alambda > 1e10f) alambda = 1e10f;
            }
        }
        if (tr && tr->n < ORC_TRACE_MAX) {
            tr->phi[tr->n] = ok ? phi1 : 0.0f;
            tr->verdict[tr->n] = verdict;
            tr->alambda[tr->n] = alambda;
            tr->n++;
        }
        if (stop) break;
    }
    if (iter > o->kiter) iter = o->kiter;
    if (res->x) std::memcpy(res->x, xn.data(), nx * 4);
    if (res->yn) std::memcpy(res->yn, yn.data(), ny * 4);
    res->phi = phi;
    res->chisq = chisq;
    res->alambda = alambda;
    res->iterations = iter;
    res->forwards = forwards;
    res->converged = converged;
    res->nonpd = 0;
    res->ms = 0.0;
    return RTB_OK;
}

}  // extern "C"
