// retrieval.cu -- host side of the optimal-estimation Newton step and of the
// retrieval loop: rtb_newton_step_batch, rtb_calc_phiret_batch,
// rtb_spd_inverse_batch and rtb_retrieve_batch (include/radtran_b200.h).
//
// The loop restates the Levenberg-Marquardt control of nemesis/coreret.f:
// 578-1106 for the layer-state model (model 0 temperatures, model 3 gas
// scales, nemesis/subprofretg.f:638-651 and :735-741).  Everything sizeable
// stays on the device between rounds: K and the spectrum of the current and
// of the trial state (two buffers per retrieval, swapped on acceptance),
// y, Se^-1, Sa^-1.  The host keeps the scalar control (alambda, phi) and the
// state vectors, which it needs to lay out the trial atmosphere for the
// forward model's set-up.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"
#include "newton.h"

namespace rtb {

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

int64_t al4(int64_t n) { return (n + 3) & ~(int64_t)3; }

template <class T>
cudaError_t h2d(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
    cudaError_t e = b.ensure(v.size() * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    return v.empty() ? cudaSuccess : cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

// ---------------------------------------------------------------- the layer-state model
// Compact working copy of one retrieval's atmosphere (leading dimensions
// shrunk to the sizes), re-laid for every trial state.
struct AtmWork {
    rtb_atm a{};
    int nparam = 0;
    std::vector<float> press, temp, delh, pp, amount, cont, scale, emtemp, dte, dam, dco, xmap, vwave, xsec;
    std::vector<int> idgas, isogas, ktab, nlayin, imod, layinc;
    std::vector<float> pp0, amount0, xmap0;   // at scale factor 1
    std::vector<int> scale_gas;
};

int build_work(rtb_context* c, const rtb_retrieval_spec& s, AtmWork& w) {
    const rtb_atm& t = *s.atm;
    const int L = t.nlayer, G = t.ngas, NC = t.ncont, NP = t.npath, NPRO = t.npro, NV = t.nv, NW = t.nwave;
    const int ldl = t.ld_lay > 0 ? t.ld_lay : RTB_MAXLAY;
    const int ldc = t.ld_con > 0 ? t.ld_con : RTB_MAXCON;
    const int ldv = t.ld_v > 0 ? t.ld_v : RTB_MAXV;
    const int ldp = t.ld_param > 0 ? t.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    const int nparam = G + 1 + NC;
    if (NP != 1) return fail(c, RTB_ERR_UNSUPPORTED, "retrieval atmosphere must have one path (npath=%d)", NP);
    if (NPRO != L) return fail(c, RTB_ERR_UNSUPPORTED, "layer-state model needs npro == nlayer");
    if (NV != L + s.nscale) return fail(c, RTB_ERR_ARG, "nv=%d but nlayer + nscale = %d", NV, L + s.nscale);
    if (NV > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "state size %d > %d", NV, kNewtonMaxNx);
    if (NV >= NW) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d >= ny=%d (calc_gain_matrix nx<ny branch only)", NV, NW);
    if (!t.press || !t.temp || !t.delh || !t.pp || !t.amount || !t.idgas || !t.isogas || !t.ktab || !t.nlayin ||
        !t.imod || !t.layinc || !t.scale || !t.emtemp || !t.dte || !t.dam || !t.xmap || !t.vwave)
        return fail(c, RTB_ERR_ARG, "NULL input array in retrieval atmosphere");
    if (ldl < L || ldv < NV || ldp < nparam) return fail(c, RTB_ERR_ARG, "leading dimension smaller than size");
    if (NC > 0 && (!t.cont || !t.xsec_ext || !t.dco)) return fail(c, RTB_ERR_ARG, "dust arrays missing");
    for (int a = 0; a < s.nscale; ++a)
        if (!s.scale_gas || s.scale_gas[a] < 0 || s.scale_gas[a] >= G)
            return fail(c, RTB_ERR_ARG, "scale_gas[%d] outside 0..ngas-1", a);
    w.nparam = nparam;
    w.scale_gas.assign(s.scale_gas, s.scale_gas + s.nscale);
    auto lay1 = [&](const float* p, std::vector<float>& v) { v.assign(p, p + L); };
    auto lay2 = [&](const float* p, int ncols, std::vector<float>& v) {
        v.resize((size_t)L * ncols);
        for (int j = 0; j < ncols; ++j)
            for (int i = 0; i < L; ++i) v[i + (size_t)L * j] = p[i + (size_t)ldl * j];
    };
    lay1(t.press, w.press);
    lay1(t.temp, w.temp);
    lay1(t.delh, w.delh);
    lay2(t.pp, G, w.pp0);
    lay2(t.amount, G, w.amount0);
    w.pp = w.pp0;
    w.amount = w.amount0;
    if (NC > 0) {
        w.cont.resize((size_t)NC * L);
        for (int j = 0; j < L; ++j)
            for (int i = 0; i < NC; ++i) w.cont[i + (size_t)NC * j] = t.cont[i + (size_t)ldc * j];
        lay2(t.dco, NPRO, w.dco);
        w.xsec.assign(t.xsec_ext, t.xsec_ext + (size_t)NC * NW);
    }
    lay2(t.scale, NP, w.scale);
    lay2(t.emtemp, NP, w.emtemp);
    lay2(t.dte, NPRO, w.dte);
    lay2(t.dam, NPRO, w.dam);
    w.layinc.resize((size_t)L * NP);
    for (int j = 0; j < NP; ++j)
        for (int i = 0; i < L; ++i) w.layinc[i + (size_t)L * j] = t.layinc[i + (size_t)ldl * j];
    w.xmap0.resize((size_t)NV * nparam * NPRO);
    for (int k = 0; k < NPRO; ++k)
        for (int j = 0; j < nparam; ++j)
            for (int i = 0; i < NV; ++i)
                w.xmap0[i + (size_t)NV * (j + (size_t)nparam * k)] = t.xmap[i + (size_t)ldv * (j + (size_t)ldp * k)];
    w.xmap = w.xmap0;
    w.vwave.assign(t.vwave, t.vwave + NW);
    w.idgas.assign(t.idgas, t.idgas + G);
    w.isogas.assign(t.isogas, t.isogas + G);
    w.ktab.assign(t.ktab, t.ktab + G);
    w.nlayin.assign(t.nlayin, t.nlayin + NP);
    w.imod.assign(t.imod, t.imod + NP);
    rtb_atm& a = w.a;
    a = t;
    a.ld_lay = L;
    a.ld_con = NC > 0 ? NC : 1;
    a.ld_v = NV;
    a.ld_param = nparam;
    a.press = w.press.data();
    a.temp = w.temp.data();
    a.delh = w.delh.data();
    a.pp = w.pp.data();
    a.amount = w.amount.data();
    a.cont = NC > 0 ? w.cont.data() : nullptr;
    a.idgas = w.idgas.data();
    a.isogas = w.isogas.data();
    a.ktab = w.ktab.data();
    a.nlayin = w.nlayin.data();
    a.imod = w.imod.data();
    a.layinc = w.layinc.data();
    a.scale = w.scale.data();
    a.emtemp = w.emtemp.data();
    a.dte = w.dte.data();
    a.dam = w.dam.data();
    a.dco = NC > 0 ? w.dco.data() : nullptr;
    a.dfp = nullptr;
    a.xmap = w.xmap.data();
    a.vwave = w.vwave.data();
    a.xsec_ext = NC > 0 ? w.xsec.data() : nullptr;
    return RTB_OK;
}

// lay the atmosphere out at state x: temp = x[l]; amount, pp and the gas's
// xmap entries scaled by exp(x[L + a]) in REAL arithmetic (subprofretg.f:
// 746-750 computes X1 = XREF*EXP(XN)); emtemp follows temp along the path
void set_state(AtmWork& w, const float* x) {
    const int L = w.a.nlayer, NV = w.a.nv, NPRO = w.a.npro, nparam = w.nparam;
    for (int l = 0; l < L; ++l) w.temp[l] = x[l];
    const int nl = w.nlayin[0];
    for (int j = 0; j < nl; ++j) w.emtemp[j] = w.temp[w.layinc[j] - 1];
    for (size_t a = 0; a < w.scale_gas.size(); ++a) {
        const int g = w.scale_gas[a];
        const float f = expf(x[L + a]);
        for (int l = 0; l < L; ++l) {
            w.amount[l + (size_t)L * g] = w.amount0[l + (size_t)L * g] * f;
            w.pp[l + (size_t)L * g] = w.pp0[l + (size_t)L * g] * f;
        }
        for (int k = 0; k < NPRO; ++k)
            for (int i = 0; i < NV; ++i) {
                const size_t idx = i + (size_t)NV * (g + (size_t)nparam * k);
                w.xmap[idx] = w.xmap0[idx] * f;
            }
    }
}

// ---------------------------------------------------------------- one resident group
struct Ret {
    int nx = 0, ny = 0, nlayer = 0;
    // device offsets: floats into f32 (K pair), ysl (spectra), xsl (states); doubles into f64
    int64_t k_off = 0, yn_off = 0, y_off = 0, x_off = 0, sei_off = 0, sai_off = 0, sa_off = 0, work_off = 0;
    int cur = 0;                      // which K / yn buffer holds the current state
    std::vector<float> xa, xn, xn1, x_out;
    float phi = 0, ophi = 0, chisq = 0, ochisq = 0, alambda = 1.0f;
    int iter = 0, forwards = 0, converged = 0, done = 0, nonpd = 0, need_newton = 1, trial = 0;
    double t_done = 0;
    AtmWork w;
};

struct Group {
    std::vector<Ret> r;
    DevBuf kbuf, ybuf, gts, xbuf, f64, nt_desc, phi_desc, small;
    int64_t nk = 0, ny_tot = 0, nxs = 0, n64 = 0;
};

int newton_round(rtb_context* c, Group& G, const std::vector<int>& ids, cudaStream_t st) {
    if (ids.empty()) return RTB_OK;
    std::vector<NewtonDev> desc;
    float* K = (float*)G.kbuf.p;
    float* Y = (float*)G.ybuf.p;
    float* X = (float*)G.xbuf.p;
    double* D = (double*)G.f64.p;
    for (int i : ids) {
        const Ret& R = G.r[i];
        NewtonDev d;
        d.nx = R.nx;
        d.ny = R.ny;
        d.kt = K + R.k_off + (int64_t)R.cur * R.nx * R.ny;
        d.y = Y + R.y_off;
        d.yn = Y + R.yn_off + (int64_t)R.cur * al4(R.ny);
        d.sei = D + R.sei_off;
        d.sai = D + R.sai_off;
        d.xa = X + R.x_off;
        d.xn = X + R.x_off + al4(R.nx);
        d.x_out = X + R.x_off + 3 * al4(R.nx);
        d.work = D + R.work_off;
        desc.push_back(d);
    }
    CUDA_TRY(c, h2d(G.nt_desc, desc, st));
    unsigned* status = (unsigned*)G.small.p;
    CUDA_TRY(c, launch_newton_step((const NewtonDev*)G.nt_desc.p, (int)ids.size(), c->newton_hess, c->newton_refine,
                                   status, nullptr, st));
    return RTB_OK;
}

int phi_round(rtb_context* c, Group& G, const std::vector<int>& ids, bool trial, cudaStream_t st) {
    if (ids.empty()) return RTB_OK;
    std::vector<PhiDev> desc;
    float* Y = (float*)G.ybuf.p;
    float* X = (float*)G.xbuf.p;
    double* D = (double*)G.f64.p;
    for (int i : ids) {
        const Ret& R = G.r[i];
        PhiDev d;
        d.nx = R.nx;
        d.ny = R.ny;
        d.y = Y + R.y_off;
        d.yn = Y + R.yn_off + (int64_t)(trial ? 1 - R.cur : R.cur) * al4(R.ny);
        d.sei = D + R.sei_off;
        d.sai = D + R.sai_off;
        d.xn = X + R.x_off + (trial ? 2 : 1) * al4(R.nx);
        d.xa = X + R.x_off;
        desc.push_back(d);
    }
    CUDA_TRY(c, h2d(G.phi_desc, desc, st));
    float* ph = (float*)((char*)G.small.p + 4 * (size_t)G.r.size());
    CUDA_TRY(c, launch_phi((const PhiDev*)G.phi_desc.p, (int)ids.size(), ph, ph + G.r.size(), st));
    return RTB_OK;
}

// forward + Jacobian of the listed retrievals at xn (trial=false, into the
// current buffers) or xn1 (trial=true, into the other buffers)
int forward_round(rtb_context* c, Group& G, const std::vector<int>& ids, bool trial) {
    if (ids.empty()) return RTB_OK;
    std::vector<rtb_atm> atms;
    std::vector<int64_t> oo, jo;
    for (int i : ids) {
        Ret& R = G.r[i];
        set_state(R.w, trial ? R.xn1.data() : R.xn.data());
        atms.push_back(R.w.a);
        const int b = trial ? 1 - R.cur : R.cur;
        oo.push_back(R.yn_off + (int64_t)b * al4(R.ny));
        jo.push_back(R.k_off + (int64_t)b * R.nx * R.ny);
        R.forwards++;
    }
    OutPlace pl;
    pl.calcout = (float*)G.ybuf.p;
    pl.gradtsurf = (float*)G.gts.p;
    pl.gradients = (float*)G.kbuf.p;
    pl.out_off = oo.data();
    pl.jac_off = jo.data();
    int r = prepare_ex(c, (int)ids.size(), atms.data(), &pl);
    if (r) return r;
    r = launch(c);
    if (r) return r;
    return RTB_OK;
}

int upload_states(rtb_context* c, Group& G, cudaStream_t st) {
    std::vector<float> xs((size_t)G.nxs, 0.0f);
    for (const Ret& R : G.r) {
        const int64_t s = al4(R.nx);
        std::copy(R.xa.begin(), R.xa.end(), xs.begin() + R.x_off);
        std::copy(R.xn.begin(), R.xn.end(), xs.begin() + R.x_off + s);
        std::copy(R.xn1.begin(), R.xn1.end(), xs.begin() + R.x_off + 2 * s);
    }
    CUDA_TRY(c, cudaMemcpyAsync(G.xbuf.p, xs.data(), xs.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));   // xs is a local
    return RTB_OK;
}

int check_status(rtb_context* c, cudaStream_t st) {
    CUDA_TRY(c, cudaStreamSynchronize(st));
    unsigned long long diag[8];
    CUDA_TRY(c, cudaMemcpy(diag, c->d_diag.p, 64, cudaMemcpyDeviceToHost));
    if ((unsigned)(diag[0] & 0xffffffffu) & kStGord)
        return fail(c, RTB_ERR_GORD, "g-ordinate walk ran past NG (rankg.f:118-147)");
    return RTB_OK;
}

// coreret.f:621-700: next trial state, or a rejection before the forward model
bool make_trial(Ret& R) {
    const int nx = R.nx;
    R.xn1.resize(nx);
    for (int i = 0; i < nx; ++i) {
        const float step = (R.x_out[i] - R.xn[i]) / (1.0f + R.alambda);
        R.xn1[i] = R.xn[i] + step;
        if (std::isnan(R.xn1[i])) {                          // :641-649
            R.alambda = std::min(R.alambda * 10.0f, 1e10f);
            return false;
        }
        if (i >= R.nlayer && (R.xn1[i] > 85.0f || R.xn1[i] < -85.0f)) {   // :651-666, lx = 1 for model 3
            R.alambda = 1e10f;
            return false;
        }
    }
    for (int i = 0; i < R.nlayer; ++i)                       // :757-766, model-0 temperature
        if (R.xn1[i] < 1.0f) {
            R.alambda = std::min(R.alambda * 10.0f, 1e10f);
            return false;
        }
    return true;
}

// coreret.f:957-1062 for one evaluated trial state
void decide(Ret& R, float phi, float chisq, const rtb_retrieval_opts& o, double t) {
    const float tphi = 100.0f * (R.ophi - phi) / R.ophi;
    const float abstphi = std::fabs(tphi);
    auto accept = [&]() {
        R.cur = 1 - R.cur;
        R.xn = R.xn1;
        R.phi = phi;
        R.chisq = chisq;
        R.need_newton = 1;
    };
    if (phi <= R.ophi) {
        accept();
        const float dchi = std::fabs(R.ochisq - chisq);
        if (tphi >= 0.0f && tphi <= o.phlimit && R.alambda < 1.0f) {
            R.converged = 1;
            R.done = 1;
        } else {
            R.ophi = phi;
            R.alambda = R.alambda * 0.3f;
        }
        if (!R.done && o.dchisq_stop > 0.0f && dchi < o.dchisq_stop) {
            R.converged = 3;
            R.done = 1;
        }
        R.ochisq = chisq;
    } else if (R.iter >= 5 && abstphi <= o.phlimit) {
        if (R.alambda < 0.1f) {
            R.alambda = R.alambda * 10.0f;
        } else {
            accept();
            R.converged = 2;
            R.done = 1;
        }
    } else {
        R.alambda = std::min(R.alambda * 10.0f, 1e10f);
    }
    if (R.done) R.t_done = t;
}

int run_group(rtb_context* c, const rtb_retrieval_spec* specs, int n, const rtb_retrieval_opts& o,
              rtb_retrieval_result* res, double t0) {
    const cudaStream_t st = stream_of(c);
    Group G;
    G.r.resize(n);
    // ---- layout
    int64_t nk = 0, nys = 0, nxs = 0, n64 = 0;
    for (int i = 0; i < n; ++i) {
        Ret& R = G.r[i];
        const rtb_retrieval_spec& s = specs[i];
        if (!s.atm || !s.y || !s.sei || !s.sa || !s.xa) return fail(c, RTB_ERR_ARG, "retrieval %d: NULL input", i);
        int e = build_work(c, s, R.w);
        if (e) return e;
        R.nlayer = s.atm->nlayer;
        R.nx = s.atm->nv;
        R.ny = s.atm->nwave;
        R.k_off = nk;
        nk += 2 * (int64_t)R.nx * R.ny;
        R.y_off = nys;
        R.yn_off = nys + al4(R.ny);
        nys += 3 * al4(R.ny);
        R.x_off = nxs;
        nxs += 4 * al4(R.nx);
        R.sei_off = n64;
        n64 += al4(R.ny);
        R.sai_off = n64;
        n64 += (int64_t)R.nx * R.nx;
        R.sa_off = n64;
        n64 += (int64_t)R.nx * R.nx;
        R.work_off = n64;
        n64 += al4(R.ny);
        R.xa.assign(s.xa, s.xa + R.nx);
        R.xn.assign(s.x0 ? s.x0 : s.xa, (s.x0 ? s.x0 : s.xa) + R.nx);
        R.xn1 = R.xn;
        R.x_out = R.xn;
    }
    G.nk = nk;
    G.ny_tot = nys;
    G.nxs = nxs;
    G.n64 = n64;
    CUDA_TRY(c, G.kbuf.ensure((size_t)nk * 4));
    CUDA_TRY(c, G.ybuf.ensure((size_t)nys * 4));
    CUDA_TRY(c, G.gts.ensure((size_t)nys * 4));
    CUDA_TRY(c, G.xbuf.ensure((size_t)nxs * 4));
    CUDA_TRY(c, G.f64.ensure((size_t)n64 * 8));
    CUDA_TRY(c, G.small.ensure((size_t)12 * n + 64));
    // ---- resident inputs: y, Se^-1, Sa (-> Sa^-1 on the device)
    {
        std::vector<float> ys((size_t)nys, 0.0f);
        std::vector<double> ds((size_t)n64, 0.0);
        for (int i = 0; i < n; ++i) {
            const Ret& R = G.r[i];
            std::copy(specs[i].y, specs[i].y + R.ny, ys.begin() + R.y_off);
            std::copy(specs[i].sei, specs[i].sei + R.ny, ds.begin() + R.sei_off);
            std::copy(specs[i].sa, specs[i].sa + (size_t)R.nx * R.nx, ds.begin() + R.sa_off);
        }
        CUDA_TRY(c, cudaMemcpyAsync(G.ybuf.p, ys.data(), ys.size() * 4, cudaMemcpyHostToDevice, st));
        CUDA_TRY(c, cudaMemcpyAsync(G.f64.p, ds.data(), ds.size() * 8, cudaMemcpyHostToDevice, st));
        double* D = (double*)G.f64.p;
        for (int i = 0; i < n; ++i) {   // one launch per distinct nx would also do; inversion is one-time
            const Ret& R = G.r[i];
            CUDA_TRY(c, launch_spd_inverse(D + R.sa_off, D + R.sai_off, R.nx, 0, 1, nullptr, st));
        }
        CUDA_TRY(c, cudaStreamSynchronize(st));
    }
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    std::vector<float> ph(2 * (size_t)n);
    // ---- initial forward model and cost (coreret.f:520-557)
    {
        int e = upload_states(c, G, st);
        if (e) return e;
        e = forward_round(c, G, all, false);
        if (e) return e;
        e = check_status(c, st);
        if (e) return e;
        e = phi_round(c, G, all, false, st);
        if (e) return e;
        CUDA_TRY(c, cudaMemcpyAsync(ph.data(), (char*)G.small.p + 4 * (size_t)n, 8 * (size_t)n,
                                    cudaMemcpyDeviceToHost, st));
        CUDA_TRY(c, cudaStreamSynchronize(st));
        for (int i = 0; i < n; ++i) {
            Ret& R = G.r[i];
            R.phi = R.ophi = ph[i];
            R.chisq = R.ochisq = ph[n + i];
            R.alambda = 1.0f;
        }
    }
    // ---- iterations (coreret.f:591-1106)
    for (;;) {
        std::vector<int> act;
        for (int i = 0; i < n; ++i)
            if (!G.r[i].done) act.push_back(i);
        if (act.empty()) break;
        std::vector<int> nt;
        for (int i : act)
            if (G.r[i].need_newton) nt.push_back(i);
        if (!nt.empty()) {
            int e = upload_states(c, G, st);
            if (e) return e;
            e = newton_round(c, G, nt, st);
            if (e) return e;
            std::vector<float> xs((size_t)G.nxs);
            std::vector<unsigned> sts(n);
            CUDA_TRY(c, cudaMemcpyAsync(xs.data(), G.xbuf.p, xs.size() * 4, cudaMemcpyDeviceToHost, st));
            CUDA_TRY(c, cudaMemcpyAsync(sts.data(), G.small.p, 4 * nt.size(), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(c, cudaStreamSynchronize(st));
            for (size_t k = 0; k < nt.size(); ++k) {
                Ret& R = G.r[nt[k]];
                const float* xo = xs.data() + R.x_off + 3 * al4(R.nx);
                R.x_out.assign(xo, xo + R.nx);
                if (sts[k] & kNtNonPd) R.nonpd = 1;
                R.need_newton = 0;
            }
        }
        std::vector<int> fw;
        for (int i : act) {
            Ret& R = G.r[i];
            R.iter++;
            if (make_trial(R)) {
                fw.push_back(i);
            } else if (R.iter >= o.kiter) {
                R.done = 1;
                R.t_done = now_ms() - t0;
            }
        }
        if (!fw.empty()) {
            int e = upload_states(c, G, st);
            if (e) return e;
            e = forward_round(c, G, fw, true);
            if (e) return e;
            e = check_status(c, st);
            if (e) return e;
            e = phi_round(c, G, fw, true, st);
            if (e) return e;
            CUDA_TRY(c, cudaMemcpyAsync(ph.data(), (char*)G.small.p + 4 * (size_t)n, 8 * (size_t)n,
                                        cudaMemcpyDeviceToHost, st));
            CUDA_TRY(c, cudaStreamSynchronize(st));
            const double t = now_ms() - t0;
            for (size_t k = 0; k < fw.size(); ++k) {
                Ret& R = G.r[fw[k]];
                decide(R, ph[k], ph[n + k], o, t);
                if (!R.done && R.iter >= o.kiter) {
                    R.done = 1;
                    R.t_done = t;
                }
            }
        }
    }
    // ---- results: state, spectrum of the current buffers
    std::vector<float> ys((size_t)G.ny_tot);
    CUDA_TRY(c, cudaMemcpyAsync(ys.data(), G.ybuf.p, ys.size() * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        const Ret& R = G.r[i];
        rtb_retrieval_result& o2 = res[i];
        if (o2.x) std::copy(R.xn.begin(), R.xn.end(), o2.x);
        if (o2.yn) {
            const float* y = ys.data() + R.yn_off + (int64_t)R.cur * al4(R.ny);
            std::copy(y, y + R.ny, o2.yn);
        }
        o2.phi = R.phi;
        o2.chisq = R.chisq;
        o2.alambda = R.alambda;
        o2.iterations = R.iter;
        o2.forwards = R.forwards;
        o2.converged = R.converged;
        o2.nonpd = R.nonpd;
        o2.ms = R.t_done;
    }
    G.kbuf.release();
    G.ybuf.release();
    G.gts.release();
    G.xbuf.release();
    G.f64.release();
    G.nt_desc.release();
    G.phi_desc.release();
    G.small.release();
    return RTB_OK;
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" {

int rtb_set_newton_mode(rtb_context* c, int hessian, int refine) {
    if (!c) return RTB_ERR_ARG;
    if (!(hessian == RTB_HESS_TC || hessian == RTB_HESS_FP64) || refine < 0 || refine > 8)
        return fail(c, RTB_ERR_ARG, "newton mode: hessian %d refine %d", hessian, refine);
    c->newton_hess = hessian;
    c->newton_refine = refine;
    return RTB_OK;
}

int rtb_newton_step_batch(rtb_context* c, int nret, int nx, int ny, const float* kk, const double* sei,
                          const double* sai, const float* xa, const float* xn, const float* y, const float* yn,
                          float* x_out, int* nonpd, double* resid) {
    if (!c) return RTB_ERR_ARG;
    if (nret <= 0 || nx <= 0 || ny <= 0 || !kk || !sei || !sai || !xa || !xn || !y || !yn || !x_out)
        return fail(c, RTB_ERR_ARG, "newton step: bad arguments");
    if (nx > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d > %d", nx, kNewtonMaxNx);
    if (nx >= ny) return fail(c, RTB_ERR_UNSUPPORTED, "nx >= ny (calc_gain_matrix nx<ny branch only)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const int64_t nxa = al4(nx), nya = al4(ny);
    // f32: kk | y | yn | xa | xn | x_out ; f64: sei | sai | work
    const int64_t o_y = (int64_t)nret * nx * ny, o_yn = o_y + nret * nya, o_xa = o_yn + nret * nya;
    const int64_t o_xn = o_xa + nret * nxa, o_xo = o_xn + nret * nxa, n32 = o_xo + nret * nxa;
    const int64_t o_sai = nret * nya, o_w = o_sai + (int64_t)nret * nx * nx, n64 = o_w + nret * nya;
    CUDA_TRY(c, c->d_nt32.ensure((size_t)n32 * 4));
    CUDA_TRY(c, c->d_nt64.ensure((size_t)n64 * 8));
    CUDA_TRY(c, c->d_ntsmall.ensure((size_t)12 * nret + 64));
    float* F = (float*)c->d_nt32.p;
    double* D = (double*)c->d_nt64.p;
    CUDA_TRY(c, cudaMemcpyAsync(F, kk, (size_t)nret * nx * ny * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(F + o_y, nya * 4, y, ny * 4, ny * 4, nret, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(F + o_yn, nya * 4, yn, ny * 4, ny * 4, nret, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(F + o_xa, nxa * 4, xa, nx * 4, nx * 4, nret, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(F + o_xn, nxa * 4, xn, nx * 4, nx * 4, nret, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(D, nya * 8, sei, ny * 8, ny * 8, nret, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(D + o_sai, sai, (size_t)nret * nx * nx * 8, cudaMemcpyHostToDevice, st));
    std::vector<NewtonDev> desc(nret);
    for (int r = 0; r < nret; ++r) {
        NewtonDev& d = desc[r];
        d.nx = nx;
        d.ny = ny;
        d.kt = F + (int64_t)r * nx * ny;
        d.y = F + o_y + r * nya;
        d.yn = F + o_yn + r * nya;
        d.xa = F + o_xa + r * nxa;
        d.xn = F + o_xn + r * nxa;
        d.x_out = F + o_xo + r * nxa;
        d.sei = D + r * nya;
        d.sai = D + o_sai + (int64_t)r * nx * nx;
        d.work = D + o_w + r * nya;
    }
    CUDA_TRY(c, h2d(c->d_ntdesc, desc, st));
    unsigned* status = (unsigned*)c->d_ntsmall.p;
    double* dres = (double*)((char*)c->d_ntsmall.p + ((4 * (size_t)nret + 15) & ~(size_t)15));
    CUDA_TRY(c, cudaEventRecord(c->ev0, st));
    CUDA_TRY(c, launch_newton_step((const NewtonDev*)c->d_ntdesc.p, nret, c->newton_hess, c->newton_refine, status,
                                   resid ? dres : nullptr, st));
    CUDA_TRY(c, cudaEventRecord(c->ev1, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(x_out, nx * 4, F + o_xo, nxa * 4, nx * 4, nret, cudaMemcpyDeviceToHost, st));
    std::vector<unsigned> sts(nret);
    CUDA_TRY(c, cudaMemcpyAsync(sts.data(), status, 4 * (size_t)nret, cudaMemcpyDeviceToHost, st));
    if (resid) CUDA_TRY(c, cudaMemcpyAsync(resid, dres, 8 * (size_t)nret, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    if (nonpd)
        for (int r = 0; r < nret; ++r) nonpd[r] = (sts[r] & kNtNonPd) ? 1 : 0;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->newton_stats.retrievals = nret;
    c->newton_stats.ms_kernel = ms;
    return RTB_OK;
}

int rtb_get_newton_stats(const rtb_context* c, rtb_newton_stats* out) {
    if (!c || !out) return RTB_ERR_ARG;
    *out = c->newton_stats;
    return RTB_OK;
}

int rtb_calc_phiret_batch(rtb_context* c, int nret, int nx, int ny, const float* y, const float* yn,
                          const double* sei, const float* xn, const float* xa, const double* sai, float* phi,
                          float* chisq) {
    if (!c) return RTB_ERR_ARG;
    if (nret <= 0 || nx <= 0 || ny <= 0 || !y || !yn || !sei || !xn || !xa || !sai || !phi)
        return fail(c, RTB_ERR_ARG, "calc_phiret: bad arguments");
    if (nx > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d > %d", nx, kNewtonMaxNx);
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const int64_t o_yn = (int64_t)nret * ny, o_xn = 2 * o_yn, o_xa = o_xn + (int64_t)nret * nx,
                  n32 = o_xa + (int64_t)nret * nx, o_sai = (int64_t)nret * ny,
                  n64 = o_sai + (int64_t)nret * nx * nx;
    CUDA_TRY(c, c->d_nt32.ensure((size_t)n32 * 4));
    CUDA_TRY(c, c->d_nt64.ensure((size_t)n64 * 8));
    CUDA_TRY(c, c->d_ntsmall.ensure((size_t)12 * nret + 64));
    float* F = (float*)c->d_nt32.p;
    double* D = (double*)c->d_nt64.p;
    CUDA_TRY(c, cudaMemcpyAsync(F, y, (size_t)nret * ny * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(F + o_yn, yn, (size_t)nret * ny * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(F + o_xn, xn, (size_t)nret * nx * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(F + o_xa, xa, (size_t)nret * nx * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(D, sei, (size_t)nret * ny * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(D + o_sai, sai, (size_t)nret * nx * nx * 8, cudaMemcpyHostToDevice, st));
    std::vector<PhiDev> desc(nret);
    for (int r = 0; r < nret; ++r) {
        PhiDev& d = desc[r];
        d.nx = nx;
        d.ny = ny;
        d.y = F + (int64_t)r * ny;
        d.yn = F + o_yn + (int64_t)r * ny;
        d.xn = F + o_xn + (int64_t)r * nx;
        d.xa = F + o_xa + (int64_t)r * nx;
        d.sei = D + (int64_t)r * ny;
        d.sai = D + o_sai + (int64_t)r * nx * nx;
    }
    CUDA_TRY(c, h2d(c->d_ntdesc, desc, st));
    float* out = (float*)c->d_ntsmall.p;
    CUDA_TRY(c, launch_phi((const PhiDev*)c->d_ntdesc.p, nret, out, out + nret, st));
    CUDA_TRY(c, cudaMemcpyAsync(phi, out, 4 * (size_t)nret, cudaMemcpyDeviceToHost, st));
    if (chisq) CUDA_TRY(c, cudaMemcpyAsync(chisq, out + nret, 4 * (size_t)nret, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    return RTB_OK;
}

int rtb_spd_inverse_batch(rtb_context* c, int nret, int n, const double* a, double* ainv, int* nonpd) {
    if (!c) return RTB_ERR_ARG;
    if (nret <= 0 || n <= 0 || !a || !ainv) return fail(c, RTB_ERR_ARG, "spd inverse: bad arguments");
    if (n > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "n=%d > %d", n, kNewtonMaxNx);
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const size_t nn = (size_t)n * n;
    CUDA_TRY(c, c->d_nt64.ensure(2 * nn * nret * 8));
    CUDA_TRY(c, c->d_ntsmall.ensure((size_t)4 * nret + 64));
    double* D = (double*)c->d_nt64.p;
    CUDA_TRY(c, cudaMemcpyAsync(D, a, nn * nret * 8, cudaMemcpyHostToDevice, st));
    unsigned* status = (unsigned*)c->d_ntsmall.p;
    CUDA_TRY(c, launch_spd_inverse(D, D + nn * nret, n, (int64_t)nn, nret, status, st));
    CUDA_TRY(c, cudaMemcpyAsync(ainv, D + nn * nret, nn * nret * 8, cudaMemcpyDeviceToHost, st));
    std::vector<unsigned> sts(nret);
    CUDA_TRY(c, cudaMemcpyAsync(sts.data(), status, 4 * (size_t)nret, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    if (nonpd)
        for (int r = 0; r < nret; ++r) nonpd[r] = (sts[r] & kNtNonPd) ? 1 : 0;
    return RTB_OK;
}

int rtb_retrieve_batch(rtb_context* c, int nret, const rtb_retrieval_spec* specs, const rtb_retrieval_opts* opts,
                       rtb_retrieval_result* results) {
    if (!c) return RTB_ERR_ARG;
    if (nret <= 0 || !specs || !results) return fail(c, RTB_ERR_ARG, "retrieve: bad arguments");
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    rtb_retrieval_opts o{10, 0.1f, 0.0f, 0};
    if (opts) o = *opts;
    if (o.kiter < 1) return fail(c, RTB_ERR_ARG, "kiter < 1");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const double t0 = now_ms();
    const int chunk = o.max_batch > 0 ? o.max_batch : nret;
    for (int s = 0; s < nret; s += chunk) {
        const int n = std::min(chunk, nret - s);
        const int r = run_group(c, specs + s, n, o, results + s, t0);
        if (r) return r;
    }
    return RTB_OK;
}

}  // extern "C"
