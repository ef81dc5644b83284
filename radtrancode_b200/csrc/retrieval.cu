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
#include <deque>
#include <map>
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
    std::vector<int> scale_gas, scale_model, prof_gas, dust_type;
    std::vector<float> cont0;                 // dust columns at scale 1 [nlayer][ncont]
    std::vector<float> vmr0;                  // [nprof][L] pp0 / press of the profiled gases
    // the level-state model: the profile (levels) and its layering
    bool level = false;
    int npro = 0;
    rtb_profile pr{};
    rtb_layer_opts lo{};
    std::vector<float> ph, pp_atm, pt, pvmr0, pvmr, lbase;   // h, p, t [npro]; vmr [ngas][npro]
    // the measurement's channels: the forward model's spectrum and Jacobian
    // rows convolved by cirsconv onto them (cirsrtfg_wave.f:520-560)
    ConvSpec conv;
    bool has_conv = false;
    int ny = 0;                 // measurement points: npath x (nconv, or nwave without channels)
    int npath = 1;              // paths of the layer-state model, measured one after the other
};

// the channels of a retrieval's atmosphere (FWHM and rtb_conv as
// rtb_cirsrtfg_wave takes them) and the size of its measurement vector
int work_channels(rtb_context* c, const rtb_atm& t, AtmWork& w) {
    w.has_conv = false;
    w.ny = t.nwave;
    if (t.fwhm == 0.0f && !t.conv) return RTB_OK;
    const int r = conv_check(c, t.fwhm, t.nwave, t.vwave, t.conv, w.conv);
    if (r) return r;
    if (!w.conv.vconv.empty()) {
        w.has_conv = true;
        w.ny = (int)w.conv.vconv.size();
    }
    return RTB_OK;
}

int build_level_work(rtb_context* c, const rtb_retrieval_spec& s, AtmWork& w);

int build_work(rtb_context* c, const rtb_retrieval_spec& s, AtmWork& w) {
    if (s.prof) return build_level_work(c, s, w);
    const rtb_atm& t = *s.atm;
    const int L = t.nlayer, G = t.ngas, NC = t.ncont, NP = t.npath, NPRO = t.npro, NV = t.nv, NW = t.nwave;
    const int ldl = t.ld_lay > 0 ? t.ld_lay : RTB_MAXLAY;
    const int ldc = t.ld_con > 0 ? t.ld_con : RTB_MAXCON;
    const int ldv = t.ld_v > 0 ? t.ld_v : RTB_MAXV;
    const int ldp = t.ld_param > 0 ? t.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    const int nparam = G + 1 + NC;
    if (NP < 1 || NP > RTB_MAXPAT || !t.nlayin) return fail(c, RTB_ERR_ARG, "retrieval atmosphere: npath=%d", NP);
    for (int p = 0; p < NP; ++p)
        if (t.nlayin[p] < 1 || t.nlayin[p] > L)
            return fail(c, RTB_ERR_UNSUPPORTED, "retrieval path %d has %d positions (1..nlayer=%d)", p, t.nlayin[p], L);
    if (!t.vwave) return fail(c, RTB_ERR_ARG, "NULL input array in retrieval atmosphere");
    if (const int r = work_channels(c, t, w)) return r;
    w.npath = NP;
    w.ny *= NP;   // y: every path's spectrum, path after path
    if (NPRO != L) return fail(c, RTB_ERR_UNSUPPORTED, "layer-state model needs npro == nlayer");
    if (s.nprof < 0 || (s.nprof > 0 && !s.prof_gas)) return fail(c, RTB_ERR_ARG, "nprof/prof_gas");
    if (s.ndust < 0 || (s.ndust > 0 && (!s.dust_type || NC == 0 || !t.dco)))
        return fail(c, RTB_ERR_ARG, "ndust/dust_type (dust scales need ncont > 0 and dco)");
    for (int d = 0; d < s.ndust; ++d)
        if (s.dust_type[d] < 0 || s.dust_type[d] >= NC) return fail(c, RTB_ERR_ARG, "dust_type[%d] outside 0..ncont-1", d);
    if (NV != L + s.nscale + s.nprof * L + s.ndust)
        return fail(c, RTB_ERR_ARG, "nv=%d but nlayer + nscale + nprof*nlayer + ndust = %d", NV,
                    L + s.nscale + s.nprof * L + s.ndust);
    if (NV > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "state size %d > %d", NV, kNewtonMaxNx);
    if (NV >= w.ny) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d >= ny=%d (calc_gain_matrix nx<ny branch only)", NV, w.ny);
    if (!t.press || !t.temp || !t.delh || !t.pp || !t.amount || !t.idgas || !t.isogas || !t.ktab || !t.nlayin ||
        !t.imod || !t.layinc || !t.scale || !t.emtemp || !t.dte || !t.dam || !t.xmap || !t.vwave)
        return fail(c, RTB_ERR_ARG, "NULL input array in retrieval atmosphere");
    if (ldl < L || ldv < NV || ldp < nparam) return fail(c, RTB_ERR_ARG, "leading dimension smaller than size");
    if (NC > 0 && (!t.cont || !t.xsec_ext || !t.dco)) return fail(c, RTB_ERR_ARG, "dust arrays missing");
    for (int a = 0; a < s.nscale; ++a)
        if (!s.scale_gas || s.scale_gas[a] < 0 || s.scale_gas[a] >= G)
            return fail(c, RTB_ERR_ARG, "scale_gas[%d] outside 0..ngas-1", a);
    for (int a = 0; a < s.nscale; ++a)
        if (s.scale_model && !(s.scale_model[a] == 2 || s.scale_model[a] == 3))
            return fail(c, RTB_ERR_UNSUPPORTED, "scale_model[%d]=%d (models 2 and 3 only)", a, s.scale_model[a]);
    for (int p = 0; p < s.nprof; ++p) {
        if (s.prof_gas[p] < 0 || s.prof_gas[p] >= G) return fail(c, RTB_ERR_ARG, "prof_gas[%d] outside gases", p);
        for (int a = 0; a < s.nscale; ++a)
            if (s.scale_gas[a] == s.prof_gas[p]) return fail(c, RTB_ERR_ARG, "gas %d both scaled and profiled", s.prof_gas[p]);
    }
    w.nparam = nparam;
    w.scale_gas.assign(s.scale_gas, s.scale_gas + s.nscale);
    w.scale_model.assign(s.nscale, 3);
    if (s.scale_model) w.scale_model.assign(s.scale_model, s.scale_model + s.nscale);
    w.prof_gas.assign(s.prof_gas, s.prof_gas + s.nprof);
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
        w.cont0 = w.cont;
        w.dust_type.assign(s.dust_type, s.dust_type + s.ndust);
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
    w.vmr0.resize((size_t)s.nprof * L);
    for (int p = 0; p < s.nprof; ++p)
        for (int l = 0; l < L; ++l) w.vmr0[(size_t)p * L + l] = w.pp0[l + (size_t)L * s.prof_gas[p]] / w.press[l];
    w.vwave.assign(t.vwave, t.vwave + NW);
    w.idgas.assign(t.idgas, t.idgas + G);
    w.isogas.assign(t.isogas, t.isogas + G);
    w.ktab.assign(t.ktab, t.ktab + G);
    w.nlayin.assign(t.nlayin, t.nlayin + NP);
    w.imod.assign(t.imod, t.imod + NP);
    rtb_atm& a = w.a;
    a = t;
    a.fwhm = 0.0f;      // the engine convolves the raw outputs itself
    a.conv = nullptr;
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
int set_level_state(rtb_context* c, AtmWork& w, const float* x);

int set_state(rtb_context* c, AtmWork& w, const float* x) {
    if (w.level) return set_level_state(c, w, x);
    const int L = w.a.nlayer, NV = w.a.nv, NPRO = w.a.npro, nparam = w.nparam;
    for (int l = 0; l < L; ++l) w.temp[l] = x[l];
    for (int p = 0; p < w.npath; ++p)
        for (int j = 0; j < w.nlayin[p]; ++j) w.emtemp[j + (size_t)L * p] = w.temp[w.layinc[j + (size_t)L * p] - 1];
    const int ns = (int)w.scale_gas.size();
    for (int a = 0; a < ns; ++a) {
        const int g = w.scale_gas[a];
        const bool lin = w.scale_model[a] == 2;
        const float f = lin ? x[L + a] : expf(x[L + a]);
        for (int l = 0; l < L; ++l) {
            w.amount[l + (size_t)L * g] = w.amount0[l + (size_t)L * g] * f;
            w.pp[l + (size_t)L * g] = w.pp0[l + (size_t)L * g] * f;
        }
        for (int k = 0; k < NPRO; ++k)
            for (int i = 0; i < NV; ++i) {
                const size_t idx = i + (size_t)NV * (g + (size_t)nparam * k);
                w.xmap[idx] = lin ? w.xmap0[idx] : w.xmap0[idx] * f;
            }
    }
    // model-0 gas profiles: vmr = EXP(XN) per layer, xmap = vmr on its own level
    for (size_t p = 0; p < w.prof_gas.size(); ++p) {
        const int g = w.prof_gas[p];
        const int base = L + ns + (int)p * L;
        for (int l = 0; l < L; ++l) {
            const float v = expf(x[base + l]);
            const float f = v / w.vmr0[p * L + l];
            w.amount[l + (size_t)L * g] = w.amount0[l + (size_t)L * g] * f;
            w.pp[l + (size_t)L * g] = w.pp0[l + (size_t)L * g] * f;
            for (int k = 0; k < NPRO; ++k) w.xmap[(base + l) + (size_t)NV * (g + (size_t)nparam * k)] = k == l ? v : 0.0f;
        }
    }
    // dust scales: model 3 on the type's column profile (subprofretg.f:735-750)
    const int NC = w.a.ncont;
    const int dbase = L + ns + (int)w.prof_gas.size() * L;
    for (size_t d = 0; d < w.dust_type.size(); ++d) {
        const int k = w.dust_type[d];
        const float f = expf(x[dbase + (int)d]);
        for (int l = 0; l < L; ++l) w.cont[k + (size_t)NC * l] = w.cont0[k + (size_t)NC * l] * f;
        const int q = w.a.ngas + 1 + k;
        for (int lev = 0; lev < NPRO; ++lev)
            for (int i = 0; i < NV; ++i) {
                const size_t idx = i + (size_t)NV * (q + (size_t)nparam * lev);
                w.xmap[idx] = w.xmap0[idx] * f;
            }
    }
    return RTB_OK;
}

// ---------------------------------------------------------------- the level-state model
int build_level_work(rtb_context* c, const rtb_retrieval_spec& s, AtmWork& w) {
    const rtb_atm& t = *s.atm;
    const rtb_profile& P = *s.prof;
    const int G = t.ngas, NPRO = P.npro, NV = t.nv, NW = t.nwave;
    if (!s.lopts) return fail(c, RTB_ERR_ARG, "level-state retrieval without layering options");
    const rtb_layer_opts& o = *s.lopts;
    if (P.nvmr != G) return fail(c, RTB_ERR_ARG, "profile has %d gases, the atmosphere %d", P.nvmr, G);
    if (P.ndust != 0 || t.ncont != 0) return fail(c, RTB_ERR_UNSUPPORTED, "level-state retrieval with dust");
    if (NPRO < 2 || NPRO > RTB_MAXPRO || !P.h || !P.p || !P.t || (G > 0 && !P.vmr))
        return fail(c, RTB_ERR_ARG, "level profile arrays");
    if (s.nprof < 0 || (s.nprof > 0 && !s.prof_gas)) return fail(c, RTB_ERR_ARG, "nprof/prof_gas");
    if (NV != NPRO + s.nscale + s.nprof * NPRO)
        return fail(c, RTB_ERR_ARG, "nv=%d but npro + nscale + nprof*npro = %d", NV, NPRO + s.nscale + s.nprof * NPRO);
    if (NV > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "state size %d > %d", NV, kNewtonMaxNx);
    if (!t.vwave) return fail(c, RTB_ERR_ARG, "NULL input array in retrieval atmosphere");
    if (const int r = work_channels(c, t, w)) return r;
    if (NV >= w.ny) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d >= ny=%d (calc_gain_matrix nx<ny branch only)", NV, w.ny);
    if (o.nlay < 1 || o.nlay > RTB_MAXLAY) return fail(c, RTB_ERR_LIMIT, "layering: nlay %d", o.nlay);
    if (!t.idgas || !t.isogas || !t.ktab || !t.vwave) return fail(c, RTB_ERR_ARG, "NULL input array in retrieval atmosphere");
    for (int a = 0; a < s.nscale; ++a) {
        if (!s.scale_gas || s.scale_gas[a] < 0 || s.scale_gas[a] >= G)
            return fail(c, RTB_ERR_ARG, "scale_gas[%d] outside 0..ngas-1", a);
        if (s.scale_model && !(s.scale_model[a] == 2 || s.scale_model[a] == 3))
            return fail(c, RTB_ERR_UNSUPPORTED, "scale_model[%d]=%d (models 2 and 3 only)", a, s.scale_model[a]);
    }
    for (int p = 0; p < s.nprof; ++p) {
        if (s.prof_gas[p] < 0 || s.prof_gas[p] >= G) return fail(c, RTB_ERR_ARG, "prof_gas[%d] outside gases", p);
        for (int a = 0; a < s.nscale; ++a)
            if (s.scale_gas[a] == s.prof_gas[p]) return fail(c, RTB_ERR_ARG, "gas %d both scaled and profiled", s.prof_gas[p]);
    }
    const int L = o.nlay, nparam = G + 1;
    w.level = true;
    w.npro = NPRO;
    w.nparam = nparam;
    w.scale_gas.assign(s.scale_gas, s.scale_gas + s.nscale);
    w.scale_model.assign(s.nscale, 3);
    if (s.scale_model) w.scale_model.assign(s.scale_model, s.scale_model + s.nscale);
    w.prof_gas.assign(s.prof_gas, s.prof_gas + s.nprof);
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
    w.pr.ld_con = 0;
    w.pr.h = w.ph.data();
    w.pr.p = w.pp_atm.data();
    w.pr.t = w.pt.data();
    w.pr.vmr = w.pvmr.data();
    w.pr.dust = nullptr;
    w.lo = o;
    if (o.laytyp >= 4 && o.base) w.lbase.assign(o.base, o.base + L);
    w.lo.base = w.lbase.empty() ? nullptr : w.lbase.data();
    // layer, path and gradient arrays, written by every re-layering
    w.press.assign(L, 0.0f);
    w.temp.assign(L, 0.0f);
    w.delh.assign(L, 0.0f);
    w.pp.assign((size_t)L * G, 0.0f);
    w.amount.assign((size_t)L * G, 0.0f);
    w.dte.assign((size_t)L * NPRO, 0.0f);
    w.dam.assign((size_t)L * NPRO, 0.0f);
    w.scale.assign(L, 0.0f);
    w.emtemp.assign(L, 0.0f);
    w.layinc.assign(L, 0);
    w.nlayin.assign(1, 0);
    w.imod.assign(1, 3);
    w.xmap.assign((size_t)NV * nparam * NPRO, 0.0f);
    w.vwave.assign(t.vwave, t.vwave + NW);
    w.idgas.assign(t.idgas, t.idgas + G);
    w.isogas.assign(t.isogas, t.isogas + G);
    w.ktab.assign(t.ktab, t.ktab + G);
    rtb_atm& a = w.a;
    a = t;
    a.fwhm = 0.0f;      // the engine convolves the raw outputs itself
    a.conv = nullptr;
    a.nlayer = L;
    a.ncont = 0;
    a.npath = 1;
    a.npro = NPRO;
    a.ld_lay = L;
    a.ld_con = 1;
    a.ld_v = NV;
    a.ld_param = nparam;
    a.press = w.press.data();
    a.temp = w.temp.data();
    a.delh = w.delh.data();
    a.pp = w.pp.data();
    a.amount = w.amount.data();
    a.cont = nullptr;
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
    a.dco = nullptr;
    a.dfp = nullptr;
    a.xmap = w.xmap.data();
    a.vwave = w.vwave.data();
    a.xsec_ext = nullptr;
    a.conv = nullptr;
    return RTB_OK;
}

// the profile at state x (subprofretg.f:638-651, 725-750 on every level), then
// its layers, gradient matrices and path (layerg + atmg on the device)
int set_level_state(rtb_context* c, AtmWork& w, const float* x) {
    const int NPRO = w.npro, NV = w.a.nv, nparam = w.nparam, G = w.a.ngas;
    for (int l = 0; l < NPRO; ++l) w.pt[l] = x[l];
    w.pvmr = w.pvmr0;
    std::fill(w.xmap.begin(), w.xmap.end(), 0.0f);
    for (int l = 0; l < NPRO; ++l) w.xmap[l + (size_t)NV * (G + (size_t)nparam * l)] = 1.0f;
    const int ns = (int)w.scale_gas.size();
    for (int a = 0; a < ns; ++a) {
        const int g = w.scale_gas[a];
        const bool lin = w.scale_model[a] == 2;
        const float f = lin ? x[NPRO + a] : expf(x[NPRO + a]);
        for (int l = 0; l < NPRO; ++l) {
            const float ref = w.pvmr0[l + (size_t)NPRO * g];
            const float v = ref * f;
            w.pvmr[l + (size_t)NPRO * g] = v;
            w.xmap[(NPRO + a) + (size_t)NV * (g + (size_t)nparam * l)] = lin ? ref : v;
        }
    }
    for (size_t p = 0; p < w.prof_gas.size(); ++p) {
        const int g = w.prof_gas[p];
        const int base = NPRO + ns + (int)p * NPRO;
        for (int l = 0; l < NPRO; ++l) {
            const float v = expf(x[base + l]);
            w.pvmr[l + (size_t)NPRO * g] = v;
            w.xmap[(base + l) + (size_t)NV * (g + (size_t)nparam * l)] = v;
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
    return rtb_layerg(c, &w.pr, &w.lo, &out);
}

// ---------------------------------------------------------------- the retrieval engine
// One retrieval in flight.  Device memory: a block of the engine's arena
// (K of the current and the trial state, y and the two spectra, Se^-1,
// Sa^-1, Sa and the Newton scratch) and a row of the state area (xa, xn,
// xn1, x_out).
struct Slot {
    long long id = 0;
    int nx = 0, ny = 0, nlayer = 0;
    std::vector<unsigned char> kind;  // per state element: 0 T, 1 log variable (lx = 1), 2 linear scale
    size_t bytes = 0, off = 0;        // arena block
    int xrow = -1;                    // row of the state area
    int phase = 0;                    // 0: first forward model pending; 1: iterating
    int cur = 0;                      // which K / spectrum buffer holds the current state
    std::vector<float> xa, xn, xn1, x_out, y;
    std::vector<double> sei, sa;
    float phi = 0, ophi = 0, chisq = 0, ochisq = 0, alambda = 1.0f;
    int iter = 0, forwards = 0, converged = 0, done = 0, nonpd = 0, need_newton = 1;
    double t_submit = 0, t_done = 0;
    rtb_retrieval_result res{};
    AtmWork w;
    int nraw = 0;                     // calculation points of the raw outputs (channels or several paths)
    int np = 1;                       // paths measured one after the other
    // arena layout (element offsets from the block start)
    int64_t k_elems() const { return 2 * (int64_t)nx * ny; }
    int64_t y_elems() const { return 3 * al4(ny); }
};

size_t slot_core_bytes(int nx, int ny) {
    const size_t f = (size_t)(2 * (int64_t)nx * ny + 3 * al4(ny)) * 4;
    const size_t d = (size_t)(al4(ny) + 2 * (int64_t)nx * nx) * 8;
    return (((f + 7) & ~(size_t)7) + d + 255) & ~(size_t)255;
}

// K and the spectra of two states, y, Se^-1, Sa^-1 and Sa;
// with channels or several paths, after them the forward model's own
// outputs for the state being evaluated, [np][nraw] then [np][nx][nraw],
// and with both, the convolved Jacobian [np][nx][ny / np] before its rows
// are laid into K
int64_t raw_floats(int nx, int ny, int nraw, int np, bool conv) {
    int64_t f = al4((int64_t)np * nraw) + (int64_t)np * nx * nraw;
    if (conv && np > 1) f = al4(f) + (int64_t)nx * ny;
    return f;
}

size_t slot_bytes(int nx, int ny, int nraw, int np, bool conv) {
    return slot_core_bytes(nx, ny) + (((size_t)raw_floats(nx, ny, nraw, np, conv) * 4 + 255) & ~(size_t)255);
}

// the arena block of one retrieval, from its specification alone
size_t spec_bytes(const rtb_retrieval_spec& sp) {
    const rtb_atm& t = *sp.atm;
    const int np = sp.prof ? 1 : std::max(t.npath, 1);
    const bool conv = t.conv && t.conv->nconv > 0;
    const int ny = np * (conv ? t.conv->nconv : t.nwave);
    return (conv || np > 1) ? slot_bytes(t.nv, ny, t.nwave, np, conv) : slot_core_bytes(t.nv, ny);
}

// coreret.f:621-700 and :757-766: the next trial state, or its rejection
// before the forward model (NaN, log variable out of range, T < 1)
bool make_trial(Slot& R) {
    const int nx = R.nx;
    R.xn1.resize(nx);
    for (int i = 0; i < nx; ++i) {
        const float step = (R.x_out[i] - R.xn[i]) / (1.0f + R.alambda);
        R.xn1[i] = R.xn[i] + step;
        if (std::isnan(R.xn1[i])) {                          // :641-649
            R.alambda = std::min(R.alambda * 10.0f, 1e10f);
            return false;
        }
        if (R.kind[i] == 1 && (R.xn1[i] > 85.0f || R.xn1[i] < -85.0f)) {   // :651-666, log variables (lx = 1)
            R.alambda = 1e10f;
            return false;
        }
    }
    for (int i = 0; i < nx; ++i)                             // :683-700, a vmr gone negative (model 2)
        if (R.kind[i] == 2 && R.xn1[i] < 0.0f) {
            R.alambda = std::min(R.alambda * 10.0f, 1e10f);
            return false;
        }
    for (int i = 0; i < R.nlayer; ++i)                       // model-0 temperature
        if (R.xn1[i] < 1.0f) {
            R.alambda = std::min(R.alambda * 10.0f, 1e10f);
            return false;
        }
    return true;
}

// coreret.f:957-1062 for one evaluated trial state (REAL arithmetic)
void decide(Slot& R, float phi, float chisq, const rtb_retrieval_opts& o) {
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
        if (!R.done && o.dchisq_stop > 0.0f && dchi < o.dchisq_stop) {   // the optional early exit
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
}

constexpr int kXRow = 4 * kNewtonMaxNx;   // floats per state-area row: xa | xn | xn1 | x_out

struct Engine {
    rtb_context* c = nullptr;
    rtb_retrieval_opts o{10, 0.1f, 0.0f, 0};
    size_t budget = 0;
    DevBuf arena, xarea, nt_desc, phi_desc, small;
    std::map<size_t, size_t> free_list;   // offset -> size
    std::vector<int> free_rows;
    int rows = 0;
    std::deque<Slot*> queue;
    std::vector<Slot*> active;
    std::map<long long, Slot*> finished;
    long long next_id = 1;
    double t0 = 0;
    ~Engine() {
        for (Slot* s : queue) delete s;
        for (Slot* s : active) delete s;
        for (auto& kv : finished) delete kv.second;
        arena.release();
        xarea.release();
        nt_desc.release();
        phi_desc.release();
        small.release();
    }

    float* F() const { return (float*)arena.p; }
    float* K(const Slot& s, int b) const { return F() + s.off / 4 + (int64_t)b * s.nx * s.ny; }
    float* Yb(const Slot& s) const { return F() + s.off / 4 + s.k_elems(); }          // y
    float* Yn(const Slot& s, int b) const { return Yb(s) + (1 + b) * al4(s.ny); }     // spectrum b
    double* Db(const Slot& s) const {
        const size_t f = (size_t)(s.k_elems() + s.y_elems()) * 4;
        return (double*)((char*)arena.p + s.off + ((f + 7) & ~(size_t)7));
    }
    double* Sei(const Slot& s) const { return Db(s); }
    double* Sai(const Slot& s) const { return Db(s) + al4(s.ny); }
    double* Sa(const Slot& s) const { return Sai(s) + (int64_t)s.nx * s.nx; }
    float* Raw(const Slot& s) const { return F() + (s.off + slot_core_bytes(s.nx, s.ny)) / 4; }
    float* X(const Slot& s, int part) const { return (float*)xarea.p + (int64_t)s.xrow * kXRow + part * kNewtonMaxNx; }

    int init(rtb_context* ctx, const rtb_retrieval_opts& opts, size_t bytes) {
        c = ctx;
        o = opts;
        budget = bytes;
        CUDA_TRY(c, arena.ensure(budget));
        free_list.clear();
        free_list[0] = budget;
        t0 = now_ms();
        return RTB_OK;
    }

    bool alloc(size_t n, size_t& off) {
        for (auto it = free_list.begin(); it != free_list.end(); ++it)
            if (it->second >= n) {
                off = it->first;
                const size_t rest = it->second - n;
                free_list.erase(it);
                if (rest) free_list[off + n] = rest;
                return true;
            }
        return false;
    }

    void release(size_t off, size_t n) {
        auto it = free_list.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_list.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_list.erase(nx);
        }
        if (it != free_list.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_list.erase(it);
            }
        }
    }

    int submit(const rtb_retrieval_spec& sp, long long* id) {
        if (!sp.atm || !sp.y || !sp.sei || !sp.sa || !sp.xa) return fail(c, RTB_ERR_ARG, "retrieval: NULL input");
        Slot* s = new Slot;
        int e = build_work(c, sp, s->w);
        if (e) {
            delete s;
            return e;
        }
        s->nlayer = sp.prof ? sp.prof->npro : sp.atm->nlayer;   // the temperature elements of x
        s->nx = sp.atm->nv;
        s->kind.assign(s->nx, 1);
        for (int l = 0; l < s->nlayer; ++l) s->kind[l] = 0;
        for (int a = 0; a < sp.nscale; ++a) s->kind[s->nlayer + a] = (sp.scale_model && sp.scale_model[a] == 2) ? 2 : 1;
        s->ny = s->w.ny;
        s->np = s->w.level ? 1 : s->w.npath;
        const bool raw = s->w.has_conv || s->np > 1;
        s->nraw = raw ? sp.atm->nwave : 0;
        s->bytes = raw ? slot_bytes(s->nx, s->ny, s->nraw, s->np, s->w.has_conv) : slot_core_bytes(s->nx, s->ny);
        if (s->bytes > budget) {
            const size_t need = s->bytes;
            delete s;
            return fail(c, RTB_ERR_BUDGET, "retrieval needs %zu B, budget %zu B", need, budget);
        }
        s->xa.assign(sp.xa, sp.xa + s->nx);
        const float* x0 = sp.x0 ? sp.x0 : sp.xa;
        s->xn.assign(x0, x0 + s->nx);
        s->xn1 = s->xn;
        s->x_out = s->xn;
        s->y.assign(sp.y, sp.y + s->ny);
        s->sei.assign(sp.sei, sp.sei + s->ny);
        s->sa.assign(sp.sa, sp.sa + (size_t)s->nx * s->nx);
        s->id = next_id++;
        s->t_submit = now_ms();
        queue.push_back(s);
        if (id) *id = s->id;
        return RTB_OK;
    }

    // admit queued retrievals, first come first served, while the arena has room
    int admit(cudaStream_t st) {
        std::vector<Slot*> adm;
        while (!queue.empty()) {
            if (o.max_batch > 0 && (int)(active.size() + adm.size()) >= o.max_batch) break;
            Slot* s = queue.front();
            size_t off;
            if (!alloc(s->bytes, off)) break;
            s->off = off;
            queue.pop_front();
            adm.push_back(s);
        }
        if (adm.empty()) return RTB_OK;
        // state-area rows (grow: the whole area is re-uploaded every round)
        for (Slot* s : adm) {
            if (free_rows.empty()) free_rows.push_back(rows++);
            s->xrow = free_rows.back();
            free_rows.pop_back();
        }
        CUDA_TRY(c, xarea.ensure((size_t)rows * kXRow * 4));
        for (Slot* s : adm) {
            CUDA_TRY(c, cudaMemcpyAsync(Yb(*s), s->y.data(), (size_t)s->ny * 4, cudaMemcpyHostToDevice, st));
            CUDA_TRY(c, cudaMemcpyAsync(Sei(*s), s->sei.data(), (size_t)s->ny * 8, cudaMemcpyHostToDevice, st));
            CUDA_TRY(c, cudaMemcpyAsync(Sa(*s), s->sa.data(), (size_t)s->nx * s->nx * 8, cudaMemcpyHostToDevice, st));
            CUDA_TRY(c, launch_spd_inverse(Sa(*s), Sai(*s), s->nx, 0, 1, nullptr, st));
            active.push_back(s);
        }
        CUDA_TRY(c, cudaStreamSynchronize(st));   // host copies of y/sei/sa stay alive until here
        return RTB_OK;
    }

    int upload_x(cudaStream_t st) {
        std::vector<float> xs((size_t)rows * kXRow, 0.0f);
        for (const Slot* s : active) {
            float* r = xs.data() + (size_t)s->xrow * kXRow;
            std::copy(s->xa.begin(), s->xa.end(), r);
            std::copy(s->xn.begin(), s->xn.end(), r + kNewtonMaxNx);
            std::copy(s->xn1.begin(), s->xn1.end(), r + 2 * kNewtonMaxNx);
        }
        CUDA_TRY(c, cudaMemcpyAsync(xarea.p, xs.data(), xs.size() * 4, cudaMemcpyHostToDevice, st));
        CUDA_TRY(c, cudaStreamSynchronize(st));
        return RTB_OK;
    }

    int newton(const std::vector<Slot*>& v, cudaStream_t st) {
        std::vector<NewtonDev> desc;
        for (const Slot* s : v) {
            NewtonDev d;
            d.nx = s->nx;
            d.ny = s->ny;
            d.kt = K(*s, s->cur);
            d.y = Yb(*s);
            d.yn = Yn(*s, s->cur);
            d.sei = Sei(*s);
            d.sai = Sai(*s);
            d.xa = X(*s, 0);
            d.xn = X(*s, 1);
            d.x_out = X(*s, 3);
            desc.push_back(d);
        }
        CUDA_TRY(c, h2d(nt_desc, desc, st));
        CUDA_TRY(c, small.ensure(12 * v.size() + 64));
        CUDA_TRY(c, launch_newton_step((const NewtonDev*)nt_desc.p, (int)v.size(), c->newton_hess, c->newton_refine,
                                       (unsigned*)small.p, nullptr, st));
        std::vector<float> xs((size_t)rows * kXRow);
        std::vector<unsigned> sts(v.size());
        CUDA_TRY(c, cudaMemcpyAsync(xs.data(), xarea.p, xs.size() * 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(c, cudaMemcpyAsync(sts.data(), small.p, 4 * v.size(), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(c, cudaStreamSynchronize(st));
        for (size_t k = 0; k < v.size(); ++k)
            if (sts[k] & kNtTimeout) return fail(c, RTB_ERR_CUDA, "Newton step: the tensor-core pipeline timed out");
        for (size_t k = 0; k < v.size(); ++k) {
            Slot& s = *v[k];
            const float* xo = xs.data() + (size_t)s.xrow * kXRow + 3 * kNewtonMaxNx;
            s.x_out.assign(xo, xo + s.nx);
            if (sts[k] & kNtNonPd) s.nonpd = 1;
            s.need_newton = 0;
        }
        return RTB_OK;
    }

    // forward model of each listed retrieval (the first at xn into the
    // current buffers, later ones at xn1 into the other buffers), then phi
    int forward_phi(const std::vector<Slot*>& v, std::vector<float>& ph, cudaStream_t st) {
        std::vector<rtb_atm> atms;
        std::vector<int64_t> oo, jo;
        for (Slot* s : v) {
            const bool first = s->phase == 0;
            const int rs = set_state(c, s->w, first ? s->xn.data() : s->xn1.data());
            if (rs) return rs;
            atms.push_back(s->w.a);
            const int b = first ? s->cur : 1 - s->cur;
            if (s->nraw) {   // own outputs, convolved and / or laid out below into Yn and K
                oo.push_back(Raw(*s) - F());
                jo.push_back(Raw(*s) + al4((int64_t)s->np * s->nraw) - F());
            } else {
                oo.push_back(Yn(*s, b) - F());
                jo.push_back(K(*s, b) - F());
            }
            s->forwards++;
        }
        OutPlace pl;
        pl.calcout = F();
        pl.gradtsurf = nullptr;
        pl.gradients = F();
        pl.out_off = oo.data();
        pl.jac_off = jo.data();
        int r = prepare_ex(c, (int)v.size(), atms.data(), &pl);
        if (r) return r;
        r = launch(c);
        if (r) return r;
        for (const Slot* s : v) {
            if (!s->nraw) continue;
            const int b = s->phase == 0 ? s->cur : 1 - s->cur;
            const int np = s->np, ny1 = s->ny / np;
            float* ro = Raw(*s);
            float* rj = ro + al4((int64_t)np * s->nraw);
            float* kb = K(*s, b);
            if (s->w.has_conv && np == 1) {   // straight onto the channels: K's rows are the series
                const ConvSeg seg[2] = {{ro, 1, Yn(*s, b)}, {rj, s->nx, kb}};
                r = conv_run(c, s->w.conv, 2, seg, st);
                if (r) return r;
                continue;
            }
            // y_p follows y_{p-1}; K's row iv holds path 0's ny1 points, then path 1's, ...
            const float* jrow = rj;   // [np][nx][ny1] after the convolution, else the raw [np][nx][nraw]
            if (s->w.has_conv) {
                float* tmp = rj + al4((int64_t)np * s->nx * s->nraw);
                const ConvSeg seg[2] = {{ro, np, Yn(*s, b)}, {rj, np * s->nx, tmp}};
                r = conv_run(c, s->w.conv, 2, seg, st);
                if (r) return r;
                jrow = tmp;
            } else {
                CUDA_TRY(c, cudaMemcpyAsync(Yn(*s, b), ro, (size_t)np * s->nraw * 4, cudaMemcpyDeviceToDevice, st));
            }
            for (int p = 0; p < np; ++p)
                CUDA_TRY(c, cudaMemcpy2DAsync(kb + (size_t)p * ny1, (size_t)s->ny * 4, jrow + (size_t)p * s->nx * ny1,
                                              (size_t)ny1 * 4, (size_t)ny1 * 4, s->nx, cudaMemcpyDeviceToDevice, st));
        }
        CUDA_TRY(c, cudaStreamSynchronize(st));
        unsigned long long diag[8];
        CUDA_TRY(c, cudaMemcpy(diag, c->d_diag.p, 64, cudaMemcpyDeviceToHost));
        if ((unsigned)(diag[0] & 0xffffffffu) & kStGord)
            return fail(c, RTB_ERR_GORD, "g-ordinate walk ran past NG (rankg.f:118-147)");
        std::vector<PhiDev> desc;
        for (const Slot* s : v) {
            const bool first = s->phase == 0;
            PhiDev d;
            d.nx = s->nx;
            d.ny = s->ny;
            d.y = Yb(*s);
            d.yn = Yn(*s, first ? s->cur : 1 - s->cur);
            d.sei = Sei(*s);
            d.sai = Sai(*s);
            d.xn = X(*s, first ? 1 : 2);
            d.xa = X(*s, 0);
            desc.push_back(d);
        }
        CUDA_TRY(c, h2d(phi_desc, desc, st));
        CUDA_TRY(c, small.ensure(12 * v.size() + 64));
        float* out = (float*)small.p;
        CUDA_TRY(c, launch_phi((const PhiDev*)phi_desc.p, (int)v.size(), out, out + v.size(), st));
        ph.resize(2 * v.size());
        CUDA_TRY(c, cudaMemcpyAsync(ph.data(), out, 8 * v.size(), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(c, cudaStreamSynchronize(st));
        return RTB_OK;
    }

    void finish(Slot* s) {
        s->done = 1;
        s->t_done = now_ms();
        rtb_retrieval_result& r = s->res;
        r.phi = s->phi;
        r.chisq = s->chisq;
        r.alambda = s->alambda;
        r.iterations = s->iter;
        r.forwards = s->forwards;
        r.converged = s->converged;
        r.nonpd = s->nonpd;
        r.ms = s->t_done - s->t_submit;
    }

    // one round: admissions, Newton steps, trial states, one batched
    // forward+Jacobian launch, the costs, the coreret decisions, retirements
    int round() {
        const cudaStream_t st = stream_of(c);
        int e = admit(st);
        if (e) return e;
        if (active.empty()) return RTB_OK;
        std::vector<Slot*> nt;
        for (Slot* s : active)
            if (s->phase == 1 && s->need_newton) nt.push_back(s);
        if (!nt.empty()) {
            e = upload_x(st);
            if (e) return e;
            e = newton(nt, st);
            if (e) return e;
        }
        std::vector<Slot*> fw;
        for (Slot* s : active) {
            if (s->phase == 0) {
                fw.push_back(s);
                continue;
            }
            s->iter++;
            if (make_trial(*s)) fw.push_back(s);
            else if (s->iter >= o.kiter) finish(s);
        }
        if (!fw.empty()) {
            e = upload_x(st);
            if (e) return e;
            std::vector<float> ph;
            e = forward_phi(fw, ph, st);
            if (e) return e;
            const size_t n = fw.size();
            for (size_t k = 0; k < n; ++k) {
                Slot& s = *fw[k];
                if (s.phase == 0) {                 // coreret.f:554-582
                    s.phi = s.ophi = ph[k];
                    s.chisq = s.ochisq = ph[n + k];
                    s.alambda = 1.0f;
                    s.phase = 1;
                    s.need_newton = 1;
                    continue;
                }
                decide(s, ph[k], ph[n + k], o);
                if (s.done) finish(&s);
                else if (s.iter >= o.kiter) finish(&s);
            }
        }
        // retire
        std::vector<Slot*> keep;
        for (Slot* s : active) {
            if (!s->done) {
                keep.push_back(s);
                continue;
            }
            s->res.x = nullptr;
            s->res.yn = nullptr;
            // the result spectrum stays readable until the slot's block is released here
            s->y.resize(s->ny);
            CUDA_TRY(c, cudaMemcpy(s->y.data(), Yn(*s, s->cur), (size_t)s->ny * 4, cudaMemcpyDeviceToHost));
            release(s->off, s->bytes);
            free_rows.push_back(s->xrow);
            finished[s->id] = s;
        }
        active.swap(keep);
        return RTB_OK;
    }

    // copy a finished retrieval's result out (x, yn into the caller's buffers)
    int take(long long id, rtb_retrieval_result* out, bool erase) {
        auto it = finished.find(id);
        if (it == finished.end()) return 0;
        Slot* s = it->second;
        float* x = out->x;
        float* yn = out->yn;
        *out = s->res;
        out->x = x;
        out->yn = yn;
        if (x) std::copy(s->xn.begin(), s->xn.end(), x);
        if (yn) std::copy(s->y.begin(), s->y.end(), yn);
        if (erase) {
            delete s;
            finished.erase(it);
        }
        return 1;
    }
};

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
    const int64_t o_sai = nret * nya, n64 = o_sai + (int64_t)nret * nx * nx;
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
    for (int r = 0; r < nret; ++r)
        if (sts[r] & kNtTimeout) return fail(c, RTB_ERR_CUDA, "Newton step: the tensor-core pipeline timed out");
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
    // arena: every retrieval resident at once, or the max_batch largest
    std::vector<size_t> sz(nret);
    for (int i = 0; i < nret; ++i) {
        if (!specs[i].atm) return fail(c, RTB_ERR_ARG, "retrieval %d: NULL atmosphere", i);
        sz[i] = spec_bytes(specs[i]);
    }
    std::sort(sz.begin(), sz.end(), std::greater<size_t>());
    const int m = o.max_batch > 0 ? std::min(o.max_batch, nret) : nret;
    size_t need = 0;
    for (int i = 0; i < m; ++i) need += sz[i];
    Engine E;
    int r = E.init(c, o, need);
    if (r) return r;
    std::vector<long long> ids(nret);
    for (int i = 0; i < nret; ++i) {
        r = E.submit(specs[i], &ids[i]);
        if (r) return r;
    }
    while (!E.queue.empty() || !E.active.empty()) {
        r = E.round();
        if (r) return r;
    }
    for (int i = 0; i < nret; ++i) E.take(ids[i], &results[i], true);
    return RTB_OK;
}

struct rtb_server {
    rtb::Engine E;
};

int rtb_server_create(rtb_context* c, size_t hbm_budget_bytes, const rtb_retrieval_opts* opts, rtb_server** out) {
    if (!c || !out) return RTB_ERR_ARG;
    *out = nullptr;
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    if (hbm_budget_bytes < 4096) return fail(c, RTB_ERR_ARG, "budget of %zu B", hbm_budget_bytes);
    rtb_retrieval_opts o{10, 0.1f, 0.0f, 0};
    if (opts) o = *opts;
    if (o.kiter < 1) return fail(c, RTB_ERR_ARG, "kiter < 1");
    CUDA_TRY(c, cudaSetDevice(c->device));
    rtb_server* s = new rtb_server;
    const int r = s->E.init(c, o, hbm_budget_bytes);
    if (r) {
        delete s;
        return r;
    }
    *out = s;
    return RTB_OK;
}

void rtb_server_destroy(rtb_server* s) {
    if (!s) return;
    cudaSetDevice(s->E.c->device);
    cudaStreamSynchronize(stream_of(s->E.c));
    delete s;
}

int rtb_server_submit(rtb_server* s, const rtb_retrieval_spec* spec, long long* id) {
    if (!s || !spec) return RTB_ERR_ARG;
    return s->E.submit(*spec, id);
}

int rtb_server_step(rtb_server* s, int* active, int* queued) {
    if (!s) return RTB_ERR_ARG;
    CUDA_TRY(s->E.c, cudaSetDevice(s->E.c->device));
    const int r = s->E.round();
    if (active) *active = (int)s->E.active.size();
    if (queued) *queued = (int)s->E.queue.size();
    return r;
}

int rtb_server_poll(rtb_server* s, long long id, int* done, rtb_retrieval_result* result) {
    if (!s || !done || !result) return RTB_ERR_ARG;
    *done = s->E.take(id, result, true);
    return RTB_OK;
}

}  // extern "C"
