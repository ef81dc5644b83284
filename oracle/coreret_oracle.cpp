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
    int L = 0, NV = 0, nparam = 0, NW = 0;
    std::vector<float> temp, pp, amount, emtemp, xmap, pp0, amount0, xmap0;
    std::vector<float> press, delh, scale, dte, dam, vwave;
    std::vector<int> layinc, idgas, isogas, ktab, nlayin, imod, sg, sm, pg;
    std::vector<float> vmr0;   /* [nprof][L] pp / press of the profiled gases */
};

int setup(const rtb_retrieval_spec& s, Work& w) {
    const rtb_atm& t = *s.atm;
    if (t.npath != 1 || t.npro != t.nlayer || t.nv != t.nlayer + s.nscale + s.nprof * t.nlayer || t.ncont != 0)
        return RTB_ERR_UNSUPPORTED;
    const int L = t.nlayer, G = t.ngas, NV = t.nv, NW = t.nwave;
    const int ldl = t.ld_lay > 0 ? t.ld_lay : RTB_MAXLAY;
    const int ldv = t.ld_v > 0 ? t.ld_v : RTB_MAXV;
    const int ldp = t.ld_param > 0 ? t.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    w.L = L;
    w.NV = NV;
    w.NW = NW;
    w.nparam = G + 1;
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
    col(t.scale, 1, w.scale);
    col(t.emtemp, 1, w.emtemp);
    col(t.dte, L, w.dte);
    col(t.dam, L, w.dam);
    w.pp = w.pp0;
    w.amount = w.amount0;
    w.layinc.resize(L);
    for (int i = 0; i < L; ++i) w.layinc[i] = t.layinc[i];
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
    w.nlayin.assign(t.nlayin, t.nlayin + 1);
    w.imod.assign(t.imod, t.imod + 1);
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
    w.a.dco = nullptr;
    w.a.dfp = nullptr;
    w.a.xmap = w.xmap.data();
    w.a.vwave = w.vwave.data();
    return RTB_OK;
}

void at_state(Work& w, const float* x) {
    const int L = w.L;
    for (int l = 0; l < L; ++l) w.temp[l] = x[l];
    for (int j = 0; j < w.nlayin[0]; ++j) w.emtemp[j] = w.temp[w.layinc[j] - 1];
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
}

/* forwardavfovX stand-in: spectrum and kk (ny, nx) REAL at state x */
int forward(const orc_tables* tab, Work& w, const float* x, int precision, int nthreads, std::vector<float>& yn,
            std::vector<float>& kk) {
    at_state(w, x);
    std::vector<double> c(w.NW), g((size_t)w.NV * w.NW);
    const int r = orc_cirsrtfg_wave_mt(tab, &w.a, precision, c.data(), g.data(), nullptr, nthreads);
    if (r) return r;
    yn.resize(w.NW);
    kk.resize((size_t)w.NV * w.NW);
    for (int i = 0; i < w.NW; ++i) yn[i] = (float)c[i];
    for (size_t i = 0; i < g.size(); ++i) kk[i] = (float)g[i];   /* gradients(iv*ny + iw) = kk(iw, iv) */
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
    const int nx = w.NV, ny = w.NW, L = w.L;
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
