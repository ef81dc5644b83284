// host.cu -- C ABI (include/radtran_b200.h), device residency and the host
// side of the forward model: validation (check_limits.f), the discrete
// set-up the reference does per wavenumber and per layer (get_kg.f record
// choice and P/T location, ciaread/nciacon constants, isw selection of
// cirsrtfg_wave.f:301-313) and the sparse composition of map2pro and
// map2xvec.  No compute path runs on the CPU: the forward model itself is
// fwd_kernel.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context.h"

using namespace rtb;

namespace rtb {

int fail(rtb_context* c, int code, const char* fmt, ...) {
    static std::mutex mu;   // batch packing reports from several host threads
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) {
        std::lock_guard<std::mutex> lk(mu);
        c->err = buf;
    }
    return code;
}

}  // namespace rtb

namespace {

// LOCATE (radtran/scatter/locate.f:1-28), 1-based
int locate_f(const float* xx, int n, float x) {
    int jl = 0, ju = n + 1;
    while (ju - jl > 1) {
        const int jm = (ju + jl) / 2;
        if ((xx[n - 1] >= xx[0]) == (x >= xx[jm - 1])) jl = jm; else ju = jm;
    }
    if (x == xx[0]) return 1;
    if (x == xx[n - 1]) return n - 1;
    return jl;
}

// FINDLOC (radtran/cirsrad/findloc.f:13-100): the 1-based index range
// [I1, I2] of the calculation grid x that a table spanning [y1, y2] covers;
// 0, 0 when the table lies wholly outside it
void findloc_f(const float* x, int nx, float y1, float y2, int& I1, int& I2) {
    float xbot, xtop;
    int Ibot, Itop;
    if (x[0] < x[nx - 1]) {
        xbot = x[0];
        xtop = x[nx - 1];
        Ibot = 1;
        Itop = nx;
    } else {
        xbot = x[nx - 1];
        xtop = x[0];
        Ibot = nx;
        Itop = 1;
    }
    if ((y1 < xbot && y2 < xbot) || (y1 > xtop && y2 > xtop)) {
        I1 = 0;
        I2 = 0;
        return;
    }
    auto end = [&](float y, int& I, int& exact) {
        if (y <= xbot) {
            I = Ibot;
            exact = 1;
        } else if (y >= xtop) {
            I = Itop;
            exact = 1;
        } else {
            const int it = locate_f(x, nx, y);
            I = it;
            exact = 0;
            for (int i = it; i <= it + 1; ++i)
                if (std::fabs(y - x[i - 1]) < 1.e-5f) {
                    I = i;
                    exact = 1;
                }
        }
    };
    int f1 = 0, f2 = 0;
    end(y1, I1, f1);
    end(y2, I2, f2);
    if (y1 < y2) {
        if (f1 == 0) I1 = I1 + 1;
    } else {
        if (f2 == 0) I2 = I2 + 1;
    }
}

// PINDEX (radtran/radtran/read_ktable.f:201-226); clamps x1 in place, 1-based
int pindex_f(const float* x, int nx, float& x1) {
    if (x1 > x[nx - 1]) x1 = x[nx - 1];
    if (x1 < x[0]) x1 = x[0];
    int j = 0;
    for (int i = 1; i <= nx - 1; ++i) {
        if (x1 >= x[i - 1]) j = i; else break;
    }
    return j;
}

// PINDEX on an ascending grid: the loop above stops at the first point above
// x1, so its result is the number of the first nx-1 points <= x1, found here
// by bisection (the same index)
int pindex_ascending(const float* x, int nx, float& x1) {
    if (x1 > x[nx - 1]) x1 = x[nx - 1];
    if (x1 < x[0]) x1 = x[0];
    return (int)(std::upper_bound(x, x + nx - 1, x1) - x);
}

// RAYLEIGHJ (radtran/scatter/rayleighj.f) with faniso(0) = 1
// RAYLEIGHV (radtran/scatter/rayleighv.f:1-12): Venus, C / lambda^4
float rayleighv_f(float v) {
    const float C = 8.8E-28f;
    float lambda = 10000.0f / v;
    const float l2 = lambda * lambda;
    lambda = l2 * l2;
    return C / lambda;
}

float rayleighj_f(float v) {
    const float AH2 = 13.58E-5f, BH2 = 7.52E-3f, AHe = 3.48E-5f, BHe = 2.30E-3f;
    const float pi = 3.1415927f, fH2 = 0.864f, k = 1.37971e-23f, P0 = 1.013e5f, T0 = 273.15f;
    const float lambda = 1e-2f / v;
    float x = 1.0f / (lambda * 1e6f);
    const float nH2 = AH2 * (1.0f + BH2 * x * x);
    const float nHe = AHe * (1.0f + BHe * x * x);
    const float nAir = fH2 * nH2 + (1 - fH2) * nHe;
    const float delta = 0.0f;
    const float temp = 32 * (pi * pi * pi) * (nAir * nAir);
    const float N0 = P0 / (k * T0);
    x = N0 * lambda * lambda;
    const float faniso = (6.0f + 3.0f * delta) / (6.0f - 7.0f * delta);
    return temp * 1e4f * faniso / (3 * (x * x));
}

// planck_wave / planckg_wave (radtran/radtran/planck_wave.f, planckg_wave.f)
void planck_host(int ispace, float v, float T, float& B, float& dB) {
    const double c1 = (double)1.1911e-12f, c2 = (double)1.439f;
    double y;
    if (ispace == 0) y = v; else y = 1e4 / v;
    if (y == 0.0) { B = 0; dB = 0; return; }
    const double x = c2 * y / T;
    const double a = ispace == 0 ? c1 * y * y * y : c1 * y * y * y * y * y / 1e4;
    const double em1 = std::expm1(x);
    B = (float)(a / em1);
    dB = (float)(a / em1 * (x / T) * (em1 + 1.0) / em1);
}

// INTERPEM (radtran/cirsrad/interpem.f)
int interpem_f(int nem, const float* vem, const float* em, float v, float& out) {
    if (nem <= 0) { out = 1.0f; return RTB_OK; }
    if (v < vem[0] || v > vem[nem - 1]) return RTB_ERR_RANGE;
    float x = 0.0f;
    for (int i = 0; i < nem - 1; ++i)
        if (v >= vem[i] && v < vem[i + 1]) {
            const float f = (v - vem[i]) / (vem[i + 1] - vem[i]);
            x = (1 - f) * em[i] + f * em[i + 1];
        }
    if (v == vem[nem - 1]) x = em[nem - 1];
    out = x;
    return RTB_OK;
}

// host staging of one batch

struct Dims {
    int ld_lay, ld_con, ld_v, ld_param;
};

}  // namespace

namespace rtb {

// INTERP (radtran/rtm_util/interp.f:1-17): the first point past xin (the
// order of the table either way), then the segment before it
float interp_f(const float* x, const float* y, int n, float xin) {
    int i = 1;
    if (x[0] < x[n - 1]) {
        while (i <= n && !(x[i - 1] > xin)) ++i;
    } else {
        while (i <= n && !(x[i - 1] < xin)) ++i;
    }
    if (i > n) i = n;
    if (i == 1) i = 2;
    return y[i - 2] + (y[i - 1] - y[i - 2]) * (xin - x[i - 2]) / (x[i - 1] - x[i - 2]);
}

// GET_SOLAR_WAVE (radtran/cirsrad/get_solar_wave.f:17-39): zero outside the
// table; dist > 0 spreads the star's power over the sphere of radius dist AU
float get_solar_wave_f(const rtb_context* c, float x, float dist) {
    const float* w = c->solar_wave.data();
    const int n = (int)c->solar_wave.size();
    float y = interp_f(w, c->solar_rad.data(), n, x);
    if (w[0] < w[n - 1]) {
        if (x < w[0]) y = 0.0f;
        if (x > w[n - 1]) y = 0.0f;
    } else {
        if (x > w[0]) y = 0.0f;
        if (x < w[n - 1]) y = 0.0f;
    }
    if (dist > 0.0f) {
        const float PI = 3.1415927f, AU = 1.49598e13f;   // constdef.f:11
        const float d = dist * AU;
        const float area = 4.0f * PI * (d * d);
        return y / area;
    }
    return y;
}

// The NGASCON gate (radtran/radtran/ngascon.f:132-318): the first switch of
// /GASCONDEF/ that would give a gas of the atmosphere a continuum, as a
// message, or null when every gas's NGASCON term is the reference's zero.
// IH2O = 2 is refused too: that branch leaves ABSORB unassigned.
const char* gascon_refusal(const rtb_atm& a) {
    static thread_local char msg[160];
    struct Uv { int bit, id; const char* name; };
    static const Uv uv[] = {{1, 11, "NH3"}, {2, 28, "PH3"}, {4, 26, "C2H2"}, {8, 27, "C2H6"}, {16, 30, "C4H2"},
                            {32, 6, "CH4"}, {64, 5, "CO"}, {128, 33, "GeH4"}, {256, 1, "H2O"}, {512, 34, "C3H8"}};
    for (int k = 0; k < a.ngas; ++k) {
        const int id = a.idgas[k], iso = a.isogas[k];
        const bool iso01 = iso == 0 || iso == 1;
        const char* sw = nullptr;
        if (id == 1 && a.ih2o != 0) sw = a.ih2o == 1 ? "IH2O=1 (CKD H2O continuum)" : "IH2O!=0,1";
        else if (id == 6 && iso01 && a.ich4 != 0) sw = "ICH4 (Karkoschka CH4 continuum)";
        else if (id == 11 && iso01 && a.inh3 != 0) sw = "INH3 (Lutz-Owen NH3 continuum)";
        else if (id == 3 && iso01 && a.io3 != 0) sw = "IO3 (Serdyuchenko O3 cross sections)";
        if (!sw && a.iuvscat > 0)
            for (const Uv& u : uv)
                if (id == u.id && (a.iuvscat & u.bit)) {
                    snprintf(msg, sizeof msg, "ngascon: iuvscat bit %d (%s UV cross sections) for gas %d (id %d): "
                             "gas continua are not implemented", u.bit, u.name, k + 1, id);
                    return msg;
                }
        if (sw) {
            snprintf(msg, sizeof msg, "ngascon: %s for gas %d (id %d, iso %d): gas continua are not implemented",
                     sw, k + 1, id, iso);
            return msg;
        }
    }
    return nullptr;
}

int pack_spectrum(rtb_context* c, const rtb_atm& a, Staging& st) {
    Dims d;
    d.ld_lay = a.ld_lay > 0 ? a.ld_lay : RTB_MAXLAY;
    d.ld_con = a.ld_con > 0 ? a.ld_con : RTB_MAXCON;
    d.ld_v = a.ld_v > 0 ? a.ld_v : RTB_MAXV;
    d.ld_param = a.ld_param > 0 ? a.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    // ---- limits and supported options (check_limits.f:1-74) ----
    if (a.nlayer <= 0 || a.ngas <= 0 || a.npath <= 0 || a.nwave <= 0 || a.nv < 0 || a.npro <= 0)
        return fail(c, RTB_ERR_ARG, "non-positive size (nlayer=%d ngas=%d npath=%d nwave=%d npro=%d)", a.nlayer,
                    a.ngas, a.npath, a.nwave, a.npro);
    if (!a.press || !a.temp || !a.delh || !a.pp || !a.amount || !a.idgas || !a.isogas || !a.ktab || !a.nlayin ||
        !a.imod || !a.layinc || !a.scale || !a.emtemp || !a.dte || !a.dam || !a.xmap || !a.vwave)
        return fail(c, RTB_ERR_ARG, "NULL input array");
    if (a.nlayer > d.ld_lay || a.nlayer > RTB_MAXLAY || a.npath > RTB_MAXPAT || a.ngas > RTB_MAXGAS ||
        a.ncont > RTB_MAXCON || a.npro > RTB_MAXPRO || a.nv > d.ld_v || a.nv > RTB_MAXV)
        return fail(c, RTB_ERR_LIMIT, "array limit exceeded (check_limits.f)");
    if (a.flagh2p != 0 && a.flagh2p != 1) return fail(c, RTB_ERR_ARG, "flagh2p=%d", a.flagh2p);
    if (a.flagh2p == 1 && (!c->has_para || !a.hfp))
        return fail(c, RTB_ERR_ARG, "flagh2p=1 needs the para-H2 CIA table (rtb_set_para_cia) and hfp");
    if (a.ilbl != 0) return fail(c, RTB_ERR_UNSUPPORTED, "ILBL != 0 (line-by-line tables) not implemented");
    if (!(a.inlte == 0 || a.inlte == 1 || a.inlte == 2))
        return fail(c, RTB_ERR_UNSUPPORTED, "inlte=%d (calc_nlte_t.f knows 0, 1, 2)", a.inlte);
    if (a.inlte == 1 && !(a.nlte_k1 >= 1.0e-20f && a.nlte_k1 <= 1.0e-3f))   // calc_nlte_t.f:17-20
        return fail(c, RTB_ERR_ARG, "calc_nlte_t: k1=%g out of range", (double)a.nlte_k1);
    if (a.iform < 0 || a.iform > 4) return fail(c, RTB_ERR_UNSUPPORTED, "iform=%d", a.iform);
    if (a.iray > 3)   // rayleighls reads the layer fractions of gases the atmosphere may not hold
        return fail(c, RTB_ERR_UNSUPPORTED, "iray=%d (Jovian 1, Venus 2 and air 3 only)", a.iray);
    if (a.ncont > 0 && (!a.cont || !a.xsec_ext || !a.dco)) return fail(c, RTB_ERR_ARG, "dust arrays missing");
    const int ng = c->ng;
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    bool n2co2 = false;
    for (int k = 0; k < a.ngas; ++k) {
        const int id = a.idgas[k];
        if (id == 91 || id == 48 || id == 80)
            return fail(c, RTB_ERR_UNSUPPORTED, "gas id %d needs the H-/electron continuum", id);
        if (a.ktab[k] >= c->ntab) return fail(c, RTB_ERR_ARG, "ktab[%d]=%d >= ntab", k, a.ktab[k]);
        if (a.ktab[k] == RTB_KTAB_BY_ID && c->tab_id.empty())
            return fail(c, RTB_ERR_ARG, "ktab[%d] = RTB_KTAB_BY_ID but the tables' gas ids are unknown", k);
        if (id == 22 || id == 2) n2co2 = true;
    }
    if (const char* why = gascon_refusal(a)) return fail(c, RTB_ERR_UNSUPPORTED, "%s", why);
    int nlmax = 0;
    for (int ip = 0; ip < a.npath; ++ip) {
        const int m = a.imod[ip];
        if (!(m == 0 || m == 1 || m == 3 || m == 18))
            return fail(c, RTB_ERR_UNSUPPORTED, "IMOD=%d not implemented", m);
        if (m == 18 && !c->has_e3) return fail(c, RTB_ERR_ARG, "IMOD 18 needs the E3 table (rtb_set_e3_table)");
        if (m == 18 && a.tsurf < 0.0f) return fail(c, RTB_ERR_UNSUPPORTED, "IMOD 18 with TSURF < 0");
        const int nl = a.nlayin[ip];
        if (nl > d.ld_lay || nl > 2 * RTB_MAXPAT) return fail(c, RTB_ERR_LIMIT, "nlayin exceeds maxinc");
        if (nl < (m == 3 ? 2 : 1)) return fail(c, RTB_ERR_UNSUPPORTED, "path with %d layers", nl);
        for (int j = 0; j < nl; ++j) {
            const int l = a.layinc[j + (size_t)d.ld_lay * ip];
            if (l < 1 || l > a.nlayer) return fail(c, RTB_ERR_LIMIT, "layinc exceeds nlayer");
        }
        nlmax = std::max(nlmax, nl);
    }
    const int nparam = a.ngas + 1 + a.ncont + (a.flagh2p == 1 ? 1 : 0);   // cirsradg_wave.f:375-376
    // ---- the nonzero xmap entries per (parameter, level), and isw: the
    // parameters that have any (cirsrtfg_wave.f:301-313), in one pass ----
    std::vector<int> isw;
    std::vector<int> xm_off((size_t)nparam * a.npro + 1);
    std::vector<std::pair<int, float>> xm_e;
    xm_e.reserve((size_t)4 * a.nv);
    for (int ip = 0; ip < nparam; ++ip) {
        const size_t e0 = xm_e.size();
        for (int lev = 0; lev < a.npro; ++lev) {
            xm_off[(size_t)ip * a.npro + lev] = (int)xm_e.size();
            const float* col = a.xmap + (size_t)d.ld_v * (ip + (size_t)d.ld_param * lev);
            for (int iv = 0; iv < a.nv; ++iv)
                if (col[iv] != 0.0f) xm_e.push_back({iv, col[iv]});
        }
        if (xm_e.size() > e0) isw.push_back(ip);
    }
    xm_off[(size_t)nparam * a.npro] = (int)xm_e.size();
    if ((int)isw.size() > kMaxSw)
        return fail(c, RTB_ERR_UNSUPPORTED, "%d active gradient parameters (device limit %d)", (int)isw.size(), kMaxSw);
    SpecDev S;
    memset(&S, 0, sizeof S);
    S.nlayer = a.nlayer;
    S.ngas = a.ngas;
    S.npath = a.npath;
    S.nwave = a.nwave;
    S.nv = a.nv;
    S.ncont = a.ncont;
    S.nsw = (int)isw.size();
    S.nlmax = nlmax;
    S.sw_T = -1;
    S.ispace = a.ispace;
    S.inormal = a.inormal;
    S.iray = (a.iray > 0 && a.itype != 0) ? a.iray : 0;   // 1 Jovian, 2 Venus, 3 air (cirsradg_wave.f:663-680)
    S.has_cia = c->has_cia;
    S.tsurf_pos = a.tsurf > 0.0f ? 1 : 0;
    // iform 3: total spectral flux of the planet, x 1e-18 (cirsradg_wave.f:913-929, 1136-1152)
    S.xfac3 = 1.0f;
    S.xfac18 = 1.0f;
    if (a.iform == 1 || a.iform == 3) {
        const float PI = 3.1415927f;   // constdef.f:11
        const float r = (a.radius1 + a.radextra) * 1e5f;
        S.xfac3 = 1.0f * PI * 4.0f * PI * (r * r);
        S.xfac18 = 1.0f * 4.0f * PI * (r * r);
        if (a.iform == 3) {
            S.xfac3 = S.xfac3 * 1e-18f;
            S.xfac18 = S.xfac18 * 1e-18f;
        }
        st.any_ext = true;
    }
    // a stellar spectrum (iread = 999): iform 1 divides the planet's flux by
    // get_solar_wave(v, -1), iform 4 multiplies IMOD 0 by get_solar_wave(v, dist)
    S.wmode = 0;
    S.wf_off = (int64_t)st.wfac.size();
    if (!c->solar_wave.empty() && (a.iform == 1 || a.iform == 4)) {
        S.wmode = a.iform == 1 ? 1 : 2;
        const float dist = a.iform == 1 ? -1.0f : a.dist;
        for (int iw = 0; iw < a.nwave; ++iw) st.wfac.push_back(get_solar_wave_f(c, a.vwave[iw], dist));
        st.any_ext = true;
    }
    for (int ip = 0; ip < a.npath; ++ip)
        if (a.imod[ip] == 18) st.any_ext = true;
    for (int s = 0; s < kMaxSw; ++s) { S.isw[s] = -1; S.col_of_param[s] = -1; }
    for (int cc = 0; cc < kMaxCols; ++cc) S.col_gas[cc] = -1;
    int ncol = 0;
    for (int s = 0; s < S.nsw; ++s) {
        S.isw[s] = isw[s];
        if (isw[s] <= a.ngas) {   // a gas amount or the temperature: tracked through the overlap
            if (ncol >= kMaxCols) return fail(c, RTB_ERR_UNSUPPORTED, "too many tracked gradient columns");
            S.col_gas[ncol] = isw[s];
            S.col_of_param[s] = ncol;
            ++ncol;
        }
        if (isw[s] == a.ngas) S.sw_T = s;
    }
    S.ncol = ncol;
    S.para = a.flagh2p == 1 ? 1 : 0;
    S.sw_para = -1;
    for (int s = 0; s < S.nsw; ++s)
        if (S.para && isw[s] == a.ngas + 1 + a.ncont) S.sw_para = s;
    if (S.sw_para >= 0 && !a.dfp) return fail(c, RTB_ERR_ARG, "para-H2 fraction in xmap without dfp");
    S.para_off = (int64_t)st.para_lay.size();
    S.paraw_off = (int64_t)st.para_wave.size();
    // non-LTE emission temperatures (cirsradg_wave.f:933-935): the layer pressures
    S.inlte = a.inlte;
    S.nlte_k1 = a.nlte_k1;
    S.nlte_A = a.nlte_A;
    S.lp_off = (int64_t)st.lpress.size();
    if (a.inlte != 0 || S.iray == 3) {   // also rayleigha's P of each layer
        st.lpress.insert(st.lpress.end(), a.press, a.press + a.nlayer);
        st.any_ext = true;
    }
    S.lt_off = (int64_t)st.ltemp.size();
    if (S.iray == 3) st.ltemp.insert(st.ltemp.end(), a.temp, a.temp + a.nlayer);
    // ---- per-layer set-up ----
    S.lay_off = (int64_t)st.lay.size();
    S.lg_off = (int64_t)st.amo.size();
    S.lc_off = (int64_t)st.cont.size();
    const int np = c->np, nt = c->nt;
    const float pmax = c->lnp[np - 1], pmin = c->lnp[0];
    const float tmax = nt > 0 ? c->tk[nt - 1] : 0.0f, tmin = nt > 0 ? c->tk[0] : 0.0f;
    for (int l = 0; l < a.nlayer; ++l) {
        LayerDev L;
        memset(&L, 0, sizeof L);
        // get_kg.f:117-141
        float P1 = (float)std::log((double)a.press[l]);
        if (P1 < pmin) P1 = pmin;
        if (P1 > pmax) P1 = pmax;
        int cp = locate_f(c->lnp.data(), np, P1);
        if (cp < 1) cp = 1;
        if (cp >= np) cp = np - 1;
        L.v = (P1 - c->lnp[cp - 1]) / (c->lnp[cp] - c->lnp[cp - 1]);
        if (nt < 0) {
            // one temperature grid per pressure, TEMP2(NP, |NT|) (get_kg.f:143-169): the
            // bracket and weight at pressure cp, then at cp + 1
            const int nx = -nt;
            float TN[RTB_MAXK];
            int ct[2];
            float uu[2], du[2];
            for (int r = 0; r < 2; ++r) {
                for (int i = 0; i < nx; ++i) TN[i] = c->tk[(cp - 1 + r) + (size_t)np * i];
                float T1 = a.temp[l];
                if (T1 < TN[0]) T1 = TN[0];
                if (T1 > TN[nx - 1]) T1 = TN[nx - 1];
                int cc = locate_f(TN, nx, T1);
                if (cc < 1) cc = 1;
                if (cc >= nx) cc = nx - 1;
                uu[r] = (T1 - TN[cc - 1]) / (TN[cc] - TN[cc - 1]);
                du[r] = 1.0f / (TN[cc] - TN[cc - 1]);
                ct[r] = cc;
            }
            L.u = uu[0];
            L.dudt = du[0];
            L.u2 = uu[1];
            L.dudt2 = du[1];
            L.ioff[0] = (nx * ng * (cp - 1)) + (ng * (ct[0] - 1));
            L.ioff[1] = (nx * ng * cp) + (ng * (ct[1] - 1));
            L.ioff[2] = (nx * ng * cp) + (ng * ct[1]);
            L.ioff[3] = (nx * ng * (cp - 1)) + (ng * ct[0]);
        } else {
            float T1 = a.temp[l];
            if (T1 < tmin) T1 = tmin;
            if (T1 > tmax) T1 = tmax;
            int ct = locate_f(c->tk.data(), nt, T1);
            if (ct < 1) ct = 1;
            if (ct >= nt) ct = nt - 1;
            L.u = (T1 - c->tk[ct - 1]) / (c->tk[ct] - c->tk[ct - 1]);
            L.dudt = 1.0f / (c->tk[ct] - c->tk[ct - 1]);
            L.ioff[0] = (nt * ng * (cp - 1)) + (ng * (ct - 1));
            L.ioff[1] = (nt * ng * cp) + (ng * (ct - 1));
            L.ioff[2] = (nt * ng * cp) + (ng * ct);
            L.ioff[3] = (nt * ng * (cp - 1)) + (ng * ct);
        }
        // utotl (cirsradg_wave.f:418-426)
        float u = 0.0f;
        for (int k = 0; k < a.ngas; ++k) u = u + a.amount[l + (size_t)d.ld_lay * k];
        L.utotl = u * 1.e-20f;
        // nciacon.f:113-177 constants
        float qh2 = 0, qhe = 0, qn2 = 0, qch4 = 0, qco2 = 0;
        for (int i = 0; i < 5; ++i) L.iabs[i] = -1;
        const float p = a.press[l], T = a.temp[l];
        for (int i = 0; i < a.ngas; ++i) {
            const int id = a.idgas[i], iso = a.isogas[i];
            const float ppi = a.pp[l + (size_t)d.ld_lay * i];
            if (id == 39 && (iso == 0 || iso == 1)) { qh2 = ppi / p; L.iabs[0] = i; }
            if (id == 40) { qhe = ppi / p; L.iabs[1] = i; }
            if (id == 22) { qn2 = ppi / p; L.iabs[2] = i; }
            if (id == 6 && (iso == 0 || iso == 1)) { qch4 = (ppi / p); L.iabs[3] = i; }
            if (id == 2) { qco2 = ppi / p; L.iabs[4] = i; }
        }
        L.q[0] = qh2; L.q[1] = qhe; L.q[2] = qn2; L.q[3] = qch4; L.q[4] = qco2;
        const float xlen = a.delh[l];
        const float AMAGAT = 2.68675E19f, MODBOLTZA = 10.0f * 1.37947E-23f / 1.013f;
        float tau;
        if (xlen == 0.0f) {
            float XP1 = 0, height = 0;
            for (int i = 0; i < a.ngas; ++i) {
                const float ppi = a.pp[l + (size_t)d.ld_lay * i];
                if (ppi > XP1) { height = a.amount[l + (size_t)d.ld_lay * i] * MODBOLTZA * T / ppi; XP1 = ppi; }
            }
            const float aa = p / 1.0f, bb = 273.15f / T;
            tau = (aa * aa) * (bb * bb) * height;
        } else {
            const float height = xlen * 1e5f;
            float XP1 = -1, TOTAM = 0;
            for (int i = 0; i < a.ngas; ++i) {
                const float ppi = a.pp[l + (size_t)d.ld_lay * i];
                if (ppi > XP1 && ppi > 0) { TOTAM = a.amount[l + (size_t)d.ld_lay * i] * p / ppi; XP1 = ppi; }
            }
            const float amag1 = (TOTAM / height) / AMAGAT;
            tau = height * (amag1 * amag1);
        }
        L.cia_tau = tau;
        if (S.para) {
            // fpread_all.f:178-219 (PINDEX clamps the temperature) and the para
            // fraction bracket of nparacon_all.f:234-253
            ParaLayDev PL;
            const float* tk2 = c->para_tk.data();
            float temp1;
            if (T > tk2[RTB_CIA_NUMT - 1]) temp1 = tk2[RTB_CIA_NUMT - 1]; else temp1 = T;
            if (T < tk2[0]) temp1 = tk2[0]; else temp1 = T;
            const int ct = pindex_f(tk2, RTB_CIA_NUMT, temp1);
            PL.ct = ct - 1;
            PL.u = (temp1 - tk2[ct - 1]) / (tk2[ct] - tk2[ct - 1]);
            PL.dudt = 1.0f / (tk2[ct] - tk2[ct - 1]);
            const float fpara = a.hfp[l];
            const int kpara = c->ipara;
            if (fpara < 0.0f) {
                PL.neg = 1;
                PL.j0 = kpara - 1;
                PL.f = 0.0f;
            } else {
                PL.neg = 0;
                const float x1 = 1.0f + (fpara - 0.25f) / c->para_deltaf;
                int j = (int)x1;
                float f = x1 - (float)j;
                if (j < 1) {
                    j = 1;
                    f = 0.0f;
                } else if (j > kpara - 2) {
                    j = kpara - 2;
                    f = 1.0f;
                }
                PL.j0 = j - 1;
                PL.f = f;
            }
            st.para_lay.push_back(PL);
            st.any_para = true;
        }
        if (c->has_cia) {
            // ciaread.f:133-157 (the second test overwrites the first; pindex clamps)
            const float* tk1 = c->cia_tk.data();
            float temp1;
            if (T > tk1[RTB_CIA_NUMT - 1]) temp1 = tk1[RTB_CIA_NUMT - 1]; else temp1 = T;
            if (T < tk1[0]) temp1 = tk1[0]; else temp1 = T;
            const int ctc = pindex_f(tk1, RTB_CIA_NUMT, temp1);
            L.cia_ct = ctc - 1;
            L.cia_u = (temp1 - tk1[ctc - 1]) / (tk1[ctc] - tk1[ctc - 1]);
            L.cia_dudt = 1.0f / (tk1[ctc] - tk1[ctc - 1]);
        } else {
            L.cia_ct = -1;
        }
        st.lay.push_back(L);
        for (int k = 0; k < a.ngas; ++k) st.amo.push_back(a.amount[l + (size_t)d.ld_lay * k] * 1.0e-20f);
        for (int k = 0; k < a.ncont; ++k) st.cont.push_back(a.cont[k + (size_t)d.ld_con * l]);
    }
    // ---- per-wavenumber set-up ----
    S.wave_off = (int64_t)st.wave.size();
    S.wg_off = (int64_t)st.wg_slice.size();
    S.wc_off = (int64_t)st.xsec.size();
    std::vector<float> vvk1;
    if (c->has_cia) {
        vvk1.resize(RTB_CIA_NUMWN);
        for (int i = 0; i < RTB_CIA_NUMWN; ++i) vvk1[i] = (float)i * c->dnu;
    }
    // the table of every (gas, calculation wavenumber), read_klist.f:247-351: the
    // gas's tables in load order (its own ktab, or with RTB_KTAB_BY_ID every table
    // of its gas and isotope ids); a regular table takes the wavenumbers FINDLOC
    // places inside its range that no earlier table took, an irregular one every
    // wavenumber; what no table takes has none (lun = -99, zero k)
    std::vector<int> wtab((size_t)a.ngas * a.nwave, -1);
    for (int k = 0; k < a.ngas; ++k) {
        int* wt = wtab.data() + (size_t)k * a.nwave;
        for (int t = 0; t < c->ntab; ++t) {
            const bool serves = a.ktab[k] == RTB_KTAB_BY_ID
                                    ? (c->tab_id[t] == a.idgas[k] && c->tab_iso[t] == a.isogas[k])
                                    : t == a.ktab[k];
            if (!serves) continue;
            if (!(c->delv[t] > 0.0f)) {
                for (int iw = 0; iw < a.nwave; ++iw) wt[iw] = t;
                continue;
            }
            const float xmax = c->vmin[t] + (float)(c->nbin[t] - 1) * c->delv[t];
            int i1 = 0, i2 = 0;
            findloc_f(a.vwave, a.nwave, c->vmin[t], xmax, i1, i2);
            if (i1 == 0 || i2 == 0) continue;
            for (int iw = i1 - 1; iw <= i2 - 1 && iw < a.nwave; ++iw)
                if (wt[iw] < 0) wt[iw] = t;
        }
    }
    auto grow = [](auto& v, size_t extra) {
        if (v.capacity() < v.size() + extra) v.reserve(std::max(v.size() + extra, 2 * v.capacity()));
    };
    grow(st.wave, a.nwave);
    grow(st.wg_slice, (size_t)a.nwave * a.ngas);
    grow(st.wg_w2, (size_t)a.nwave * a.ngas);
    grow(st.wg_w1, (size_t)a.nwave * a.ngas);
    grow(st.xsec, (size_t)a.nwave * a.ncont);
    for (int iw = 0; iw < a.nwave; ++iw) {
        WaveDev W;
        memset(&W, 0, sizeof W);
        const float vwave = a.vwave[iw];
        W.vwave = vwave;
        float esurf;
        if (interpem_f(a.nem, a.vem, a.emissivity, vwave, esurf))
            return fail(c, RTB_ERR_RANGE, "surface emissivity table does not cover %g (interpem.f)", vwave);
        const float vv = a.ispace == 1 ? 1e4f / vwave : vwave;
        if (n2co2 && vv >= 3900.0f)
            return fail(c, RTB_ERR_UNSUPPORTED, "N2/CO2 near-IR CIA (co2cia/n2n2cia/n2h2cia) not implemented");
        W.cia_cv = -1;
        if (c->has_cia && !(vv > vvk1[RTB_CIA_NUMWN - 1] || vv < vvk1[0])) {
            float vvc = vv;
            const int cv = pindex_ascending(vvk1.data(), RTB_CIA_NUMWN, vvc);   // vvk1(i) = (i-1)*dnu
            W.cia_cv = cv - 1;
            W.cia_t = (vv - vvk1[cv - 1]) / (vvk1[cv] - vvk1[cv - 1]);
        }
        if (S.para) {
            // fpread_all.f:160-205: the wavenumber bracket on vvk2(i) = (i-1)*dnu2; the
            // reference reads no table outside it (its outputs are then undefined)
            const float top = (float)(RTB_CIA_NUMWN - 1) * c->dnu2;
            if (vv > top || vv < 0.0f)
                return fail(c, RTB_ERR_RANGE, "wavenumber %g outside the para-H2 CIA table (0..%g)", vv, top);
            std::vector<float>& vk2 = c->para_vk;
            float vvc = vv;
            const int cv = pindex_ascending(vk2.data(), RTB_CIA_NUMWN, vvc);
            ParaWaveDev PW;
            PW.cv = cv - 1;
            PW.t = (vv - vk2[cv - 1]) / (vk2[cv] - vk2[cv - 1]);
            st.para_wave.push_back(PW);
        }
        W.xray = S.iray ? (S.iray == 2 ? rayleighv_f(vv) : rayleighj_f(vv)) * 1E20f : 0.0f;   // air (3): per layer
        if (a.tsurf > 0.0f) {
            float B, dB;
            planck_host(a.ispace, vwave, a.tsurf, B, dB);
            W.radground_s = esurf * B;
            W.gradground_s = esurf * dB;
        }
        st.wave.push_back(W);
        // irregular grid (delv <= 0, shared by every table): the centre of this
        // wavenumber, nearest in per cent (delv < 0) or nearest at or below it
        // with FRACK (delv = 0), read_klist.f:266-310
        int irr_ipo = 0;
        float irr_frack = 1.0f;
        if (!c->vcen.empty()) {
            const int npoint = (int)c->vcen.size();
            const float delv0 = c->delv[0];
            float maxdx1 = 1e10f;
            for (int ipo = 1; ipo <= npoint; ++ipo) {
                const float xc = c->vcen[ipo - 1];
                const float dx = 100.0f * std::fabs((vwave - xc) / xc);
                if (delv0 == 0.0f) {
                    if (dx < maxdx1 && xc <= vwave) {
                        irr_ipo = ipo;
                        irr_frack = ipo < npoint ? 1.0f - (vwave - xc) / (c->vcen[ipo] - xc) : 1.0f;
                        maxdx1 = dx;
                    }
                } else if (dx < maxdx1) {
                    irr_ipo = ipo;
                    irr_frack = 1.0f;
                    maxdx1 = dx;
                }
            }
            if (irr_ipo == 0)
                return fail(c, RTB_ERR_RANGE, "no k-table centre at or below %g (read_klist.f:314-318)", vwave);
        }
        // table record choice (get_kg.f:189-275)
        for (int k = 0; k < a.ngas; ++k) {
            const int itab = wtab[(size_t)k * a.nwave + iw];
            int64_t slice = -1;
            float w2 = -1.0f;                  // < 0: coincident wavenumber
            float w1 = -1.0f;                  // irregular grid: the lower record's weight FRACK
            if (itab >= 0 && !(c->delv[itab] > 0.0f)) {
                if (c->vcen.empty()) return fail(c, RTB_ERR_ARG, "irregular k-tables without centres (rtb_set_ktable_centres)");
                const int n1 = irr_ipo - 1;
                const bool coinc = c->delv[itab] < 0.0f;          // get_kg.f:266-279
                if (!coinc) {
                    if (irr_ipo == (int)c->vcen.size())
                        return fail(c, RTB_ERR_RANGE, "wavenumber %g above the last k-table centre", vwave);
                    w1 = irr_frack;                                // get_kg.f:391-393
                    w2 = 1.0f - irr_frack;
                    st.any_noncoinc = true;
                    st.any_w1 = true;
                }
                const int need = coinc ? n1 : n1 + 1;
                if (need >= c->nbin[itab]) return fail(c, RTB_ERR_RANGE, "k-table %d has no record %d", itab, need);
                if (c->nonzero[itab][n1]) slice = c->tab_off[itab] + (int64_t)n1 * np * std::abs(nt) * ng;
            } else if (itab >= 0) {
                const float vmin = c->vmin[itab], delv = c->delv[itab];
                float eps;
                if (delv >= 0.0001f) eps = 0.02f * delv; else eps = 0.25f * delv;
                const int n1 = (int)(((double)vwave + (double)eps - (double)vmin) / (double)delv);
                const float tmp = vmin + delv * (float)n1;
                const float frac = std::fabs((float)((double)vwave - (double)tmp));
                const bool coinc = frac < eps;
                // between two table points: weight of the upper one (get_kg.f:380-395)
                if (!coinc) {
                    w2 = (vwave - tmp) / delv;
                    if (w2 > 1.0f) w2 = 1.0f;
                    if (w2 < 0.0f) w2 = 0.0f;
                    st.any_noncoinc = true;
                }
                const int need = coinc ? n1 : n1 + 1;
                if (n1 < 0 || need >= c->nbin[itab])
                    return fail(c, RTB_ERR_RANGE, "wavenumber %g outside k-table %d", vwave, itab);
                if (c->nonzero[itab][n1])
                    slice = c->tab_off[itab] + (int64_t)n1 * np * std::abs(nt) * ng;
            }
            st.wg_slice.push_back(slice);
            st.wg_w2.push_back(w2);
            st.wg_w1.push_back(w1);
        }
        for (int k = 0; k < a.ncont; ++k) st.xsec.push_back(a.xsec_ext[k + (size_t)a.ncont * iw]);
    }
    // ---- paths ----
    S.path_off = (int64_t)st.p_layinc.size();
    std::vector<char> nonlimb(a.npath, 0);
    for (int ip = 0; ip < a.npath; ++ip) {
        const int nl = a.nlayin[ip];
        for (int j = 0; j < nlmax; ++j) {
            if (j < nl) {
                st.p_layinc.push_back(a.layinc[j + (size_t)d.ld_lay * ip] - 1);
                st.p_scale.push_back(a.scale[j + (size_t)d.ld_lay * ip]);
                st.p_emtemp.push_back(a.emtemp[j + (size_t)d.ld_lay * ip]);
            } else {
                st.p_layinc.push_back(0);
                st.p_scale.push_back(0.0f);
                st.p_emtemp.push_back(1.0f);
            }
        }
        if (a.imod[ip] == 3) {   // limb test of cirsradg_wave.f:983-988
            const int j1 = (int)(0.5f * (float)nl);
            const float p1 = a.press[a.layinc[(j1 - 1) + (size_t)d.ld_lay * ip] - 1];
            const float p2 = a.press[a.layinc[(nl - 1) + (size_t)d.ld_lay * ip] - 1];
            if (p2 > p1) nonlimb[ip] = 1;
        }
    }
    // ---- map2pro o map2xvec: sparse (s, j) -> iv per path ----
    S.map_off = (int64_t)st.map_colptr.size();
    {
        const int nsw = S.nsw, nv = a.nv, npro = a.npro;
        // levels with a nonzero d(layer)/d(level) entry, per layer, in level
        // order, for each of dam, dte, dco (two passes down the columns)
        const float* mats[4] = {a.dam, a.dte, a.dco, a.flagh2p == 1 ? a.dfp : nullptr};
        std::vector<std::pair<int, float>> nzl[4];
        std::vector<int> nzl_ptr[4];
        for (int q = 0; q < 4; ++q) {
            if (!mats[q]) continue;
            std::vector<int>& ptr = nzl_ptr[q];
            ptr.assign(a.nlayer + 1, 0);
            for (int lev = 0; lev < npro; ++lev) {
                const float* col = mats[q] + (size_t)d.ld_lay * lev;
                for (int lay = 0; lay < a.nlayer; ++lay)
                    if (col[lay] != 0.0f) ++ptr[lay + 1];
            }
            for (int lay = 0; lay < a.nlayer; ++lay) ptr[lay + 1] += ptr[lay];
            nzl[q].resize(ptr[a.nlayer]);
            std::vector<int> at(ptr.begin(), ptr.end() - 1);
            for (int lev = 0; lev < npro; ++lev) {
                const float* col = mats[q] + (size_t)d.ld_lay * lev;
                for (int lay = 0; lay < a.nlayer; ++lay)
                    if (col[lay] != 0.0f) nzl[q][at[lay]++] = {lev, col[lay]};
            }
        }
        // Each (iv, j, s) entry sums m * xmap over levels in ascending order,
        // as a dense accumulation over (s, j, lev) would; the entries are then
        // ordered by iv (stable, so rows stay ascending within a column).
        std::vector<double> acc(nv, 0.0);
        std::vector<uint8_t> hit(nv, 0);
        std::vector<int> ivs, trip_iv, trip_r, cnt(nv + 1);
        std::vector<float> trip_v;
        ivs.reserve(nv);
        for (int ip = 0; ip < a.npath; ++ip) {
            const int nl = a.nlayin[ip];
            trip_iv.clear();
            trip_r.clear();
            trip_v.clear();
            for (int j = 0; j < nl; ++j) {
                const int lay = a.layinc[j + (size_t)d.ld_lay * ip] - 1;
                for (int s = 0; s < nsw; ++s) {
                    const int k = isw[s];
                    const int q = k < a.ngas ? 0 : (k == a.ngas ? 1 : (k < a.ngas + 1 + a.ncont ? 2 : 3));
                    if (!mats[q]) continue;
                    for (int e = nzl_ptr[q][lay]; e < nzl_ptr[q][lay + 1]; ++e) {
                        const int lev = nzl[q][e].first;
                        const double m = (double)nzl[q][e].second;
                        const size_t key = (size_t)k * npro + lev;
                        for (int xe = xm_off[key]; xe < xm_off[key + 1]; ++xe) {
                            const auto& x = xm_e[xe];
                            if (!hit[x.first]) {
                                hit[x.first] = 1;
                                ivs.push_back(x.first);
                            }
                            acc[x.first] += m * (double)x.second;
                        }
                    }
                    for (int iv : ivs) {
                        trip_iv.push_back(iv);
                        trip_r.push_back(j * nsw + s);
                        trip_v.push_back((float)acc[iv]);
                        acc[iv] = 0.0;
                        hit[iv] = 0;
                    }
                    ivs.clear();
                }
            }
            std::fill(cnt.begin(), cnt.end(), 0);
            for (int iv : trip_iv) ++cnt[iv + 1];
            for (int iv = 0; iv < nv; ++iv) cnt[iv + 1] += cnt[iv];
            const int base = (int)st.map_row.size();
            for (int iv = 0; iv < nv; ++iv) st.map_colptr.push_back(base + cnt[iv]);
            st.map_colptr.push_back(base + cnt[nv]);
            st.map_row.resize(base + trip_iv.size());
            st.map_val.resize(base + trip_iv.size());
            for (size_t t = 0; t < trip_iv.size(); ++t) {
                const int at = base + cnt[trip_iv[t]]++;
                st.map_row[at] = trip_r[t];
                st.map_val[at] = trip_v[t];
            }
        }
    }
    S.out_off = st.n_out;
    S.jac_off = st.n_jac;
    st.n_out += (int64_t)a.npath * a.nwave;
    st.n_jac += (int64_t)a.npath * a.nv * a.nwave;
    // The device takes up to kMaxPathDev paths per spectrum.  A spectrum with
    // more (limb sets of many tangent paths, up to MAXPAT) is launched as
    // groups of kMaxPathDev paths over the same layers, wavenumbers and
    // state map; each group writes its paths' slots of the spectrum's
    // outputs, which stay contiguous in path order.
    const int ngrp = (a.npath + kMaxPathDev - 1) / kMaxPathDev;
    for (int gi = 0; gi < ngrp; ++gi) {
        SpecDev G = S;
        const int p0 = gi * kMaxPathDev;
        G.npath = std::min(kMaxPathDev, a.npath - p0);
        G.nonlimb_mask = 0;
        for (int ip = 0; ip < kMaxPathDev; ++ip) {
            G.nlayin[ip] = ip < G.npath ? a.nlayin[p0 + ip] : 0;
            G.imod[ip] = ip < G.npath ? a.imod[p0 + ip] : 0;
            if (ip < G.npath && nonlimb[p0 + ip]) G.nonlimb_mask |= 1 << ip;
        }
        G.path_off = S.path_off + (int64_t)p0 * nlmax;
        G.map_off = S.map_off + (int64_t)p0 * (a.nv + 1);
        G.out_off = S.out_off + (int64_t)p0 * a.nwave;
        G.jac_off = S.jac_off + (int64_t)p0 * a.nv * a.nwave;
        st.item_start.push_back(st.item_start.back() + a.nwave);
        st.spec.push_back(G);
    }
    st.nsub.push_back(ngrp);
    st.Lmax = std::max(st.Lmax, a.nlayer);
    st.nsw_max = std::max(st.nsw_max, S.nsw);
    st.ncol_max = std::max(st.ncol_max, S.ncol);
    st.nlmax_max = std::max(st.nlmax_max, nlmax);
    st.npath_max = std::max(st.npath_max, std::min(a.npath, kMaxPathDev));
    st.ngas_max = std::max(st.ngas_max, a.ngas);
    return RTB_OK;
}

template <class T>
void append_vec(std::vector<T>& d, const std::vector<T>& s) {
    d.insert(d.end(), s.begin(), s.end());
}

// concatenate a privately packed staging onto dst, rebasing its offsets
void append_staging(Staging& dst, const Staging& src) {
    const int64_t lay = dst.lay.size(), amo = dst.amo.size(), cont = dst.cont.size(), wave = dst.wave.size();
    const int64_t wg = dst.wg_slice.size(), xsec = dst.xsec.size(), path = dst.p_layinc.size();
    const int64_t colptr = dst.map_colptr.size(), rows = dst.map_row.size(), items = dst.item_start.back();
    for (SpecDev S : src.spec) {
        S.lay_off += lay;
        S.lg_off += amo;
        S.lc_off += cont;
        S.wave_off += wave;
        S.wg_off += wg;
        S.wc_off += xsec;
        S.path_off += path;
        S.map_off += colptr;
        S.para_off += (int64_t)dst.para_lay.size();
        S.paraw_off += (int64_t)dst.para_wave.size();
        S.lp_off += (int64_t)dst.lpress.size();
        S.lt_off += (int64_t)dst.ltemp.size();
        S.wf_off += (int64_t)dst.wfac.size();
        S.out_off += dst.n_out;
        S.jac_off += dst.n_jac;
        dst.spec.push_back(S);
    }
    for (size_t i = 1; i < src.item_start.size(); ++i) dst.item_start.push_back(src.item_start[i] + items);
    append_vec(dst.lay, src.lay);
    append_vec(dst.amo, src.amo);
    append_vec(dst.wave, src.wave);
    append_vec(dst.wg_slice, src.wg_slice);
    append_vec(dst.wg_w2, src.wg_w2);
    append_vec(dst.wg_w1, src.wg_w1);
    append_vec(dst.xsec, src.xsec);
    append_vec(dst.cont, src.cont);
    append_vec(dst.p_layinc, src.p_layinc);
    append_vec(dst.p_scale, src.p_scale);
    append_vec(dst.p_emtemp, src.p_emtemp);
    append_vec(dst.map_row, src.map_row);
    append_vec(dst.map_val, src.map_val);
    for (int v : src.map_colptr) dst.map_colptr.push_back(v + (int)rows);
    append_vec(dst.para_lay, src.para_lay);
    append_vec(dst.lpress, src.lpress);
    append_vec(dst.ltemp, src.ltemp);
    append_vec(dst.nsub, src.nsub);
    append_vec(dst.wfac, src.wfac);
    append_vec(dst.para_wave, src.para_wave);
    dst.Lmax = std::max(dst.Lmax, src.Lmax);
    dst.nsw_max = std::max(dst.nsw_max, src.nsw_max);
    dst.ncol_max = std::max(dst.ncol_max, src.ncol_max);
    dst.nlmax_max = std::max(dst.nlmax_max, src.nlmax_max);
    dst.npath_max = std::max(dst.npath_max, src.npath_max);
    dst.ngas_max = std::max(dst.ngas_max, src.ngas_max);
    dst.any_noncoinc = dst.any_noncoinc || src.any_noncoinc;
    dst.any_w1 = dst.any_w1 || src.any_w1;
    dst.any_para = dst.any_para || src.any_para;
    dst.any_ext = dst.any_ext || src.any_ext;
    dst.n_out += src.n_out;
    dst.n_jac += src.n_jac;
}

// pack a batch: contiguous ranges of spectra on host threads, each into its
// own staging, concatenated in order (the same result as packing one by one)
int pack_batch(rtb_context* c, int nspec, const rtb_atm* atms, Staging& st) {
    st.item_start.assign(1, 0);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nthr = std::min<int>(std::min<unsigned>(hw, 32u), nspec / 4);
    if (nthr <= 1) {
        for (int s = 0; s < nspec; ++s) {
            const int r = pack_spectrum(c, atms[s], st);
            if (r) return r;
        }
        return RTB_OK;
    }
    std::vector<Staging> part(nthr);
    std::vector<int> status(nthr, RTB_OK);
    std::vector<std::thread> th;
    for (int t = 0; t < nthr; ++t)
        th.emplace_back([&, t]() {
            const int s0 = (int)((int64_t)nspec * t / nthr), s1 = (int)((int64_t)nspec * (t + 1) / nthr);
            Staging& p = part[t];
            p.item_start.assign(1, 0);
            for (int s = s0; s < s1 && status[t] == RTB_OK; ++s) status[t] = pack_spectrum(c, atms[s], p);
        });
    for (auto& x : th) x.join();
    for (int t = 0; t < nthr; ++t)
        if (status[t]) return status[t];
    // room for every part first, so that the concatenation copies each byte once
    auto total = [&](auto member) {
        size_t n = 0;
        for (const Staging& p : part) n += (p.*member).size();
        return n;
    };
    st.spec.reserve(total(&Staging::spec));
    st.item_start.reserve(total(&Staging::item_start) + 1);
    st.lay.reserve(total(&Staging::lay));
    st.amo.reserve(total(&Staging::amo));
    st.wave.reserve(total(&Staging::wave));
    st.wg_slice.reserve(total(&Staging::wg_slice));
    st.wg_w2.reserve(total(&Staging::wg_w2));
    st.wg_w1.reserve(total(&Staging::wg_w1));
    st.xsec.reserve(total(&Staging::xsec));
    st.cont.reserve(total(&Staging::cont));
    st.p_layinc.reserve(total(&Staging::p_layinc));
    st.p_scale.reserve(total(&Staging::p_scale));
    st.p_emtemp.reserve(total(&Staging::p_emtemp));
    st.map_row.reserve(total(&Staging::map_row));
    st.map_val.reserve(total(&Staging::map_val));
    st.map_colptr.reserve(total(&Staging::map_colptr));
    st.para_lay.reserve(total(&Staging::para_lay));
    st.lpress.reserve(total(&Staging::lpress));
    st.ltemp.reserve(total(&Staging::ltemp));
    st.wfac.reserve(total(&Staging::wfac));
    st.para_wave.reserve(total(&Staging::para_wave));
    for (int t = 0; t < nthr; ++t) append_staging(st, part[t]);
    return RTB_OK;
}

template <class T>
size_t bytes_of(const std::vector<T>& v) {
    return v.size() * sizeof(T);
}

cudaStream_t stream_of(rtb_context* c) { return c->user_stream ? c->user_stream : c->stream; }

// pack + upload a batch; the device copy stays resident until the next prepare
int prepare_ex(rtb_context* c, int nspec, const rtb_atm* atms, const OutPlace* place) {
    if (!c || nspec <= 0 || !atms) return fail(c, RTB_ERR_ARG, "bad batch arguments");
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    if (c->ng > 22 || c->ng < 2) return fail(c, RTB_ERR_UNSUPPORTED, "NG=%d outside the device range 2..22", c->ng);
    CUDA_TRY(c, cudaSetDevice(c->device));
    c->prepared = 0;
    // instrument convolution of each spectrum's outputs (cirsrtfg_wave.f:448-516)
    std::vector<ConvSpec> convs(nspec);
    int any_conv = 0;
    for (int s = 0; s < nspec; ++s) {
        const int r = conv_check(c, atms[s].fwhm, atms[s].nwave, atms[s].vwave, atms[s].conv, convs[s]);
        if (r) return r;
        if (!convs[s].vconv.empty()) any_conv = 1;
    }
    if (any_conv && place)
        return fail(c, RTB_ERR_UNSUPPORTED, "instrument convolution of a batch written to caller arrays");
    Staging st;
    const int r0 = pack_batch(c, nspec, atms, st);
    if (r0) return r0;
    int smem_max = 0;
    CUDA_TRY(c, cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const bool t2 = c->nt < 0, ext = st.any_para || st.any_ext;
    int bpsm_all = 0;
    for (int w : {2, 4, 8}) {
        const int sm_w = fwd_smem_bytes(c->ng, st.nsw_max, st.ncol_max, st.nlmax_max, st.npath_max, w);
        c->bpsm_w[w] =
            (sm_w <= smem_max && fwd_tile_warps(t2, ext, w) == w) ? fwd_blocks_per_sm(sm_w, t2, ext, w, c->ng) : 0;
        bpsm_all = std::max(bpsm_all, c->bpsm_w[w]);
    }
    const int smem = fwd_smem_bytes(c->ng, st.nsw_max, st.ncol_max, st.nlmax_max, st.npath_max, kWarps);
    if (smem > smem_max)
        return fail(c, RTB_ERR_UNSUPPORTED, "spectrum needs %d B of shared memory (device %d)", smem, smem_max);
    if (c->bpsm_w[kWarps] <= 0) return fail(c, RTB_ERR_CUDA, "forward kernel cannot be resident (smem %d B)", smem);
    // first device spectrum of each caller spectrum (path groups follow it)
    std::vector<int> first(nspec + 1, 0);
    for (int sp = 0; sp < nspec; ++sp) first[sp + 1] = first[sp] + st.nsub[sp];
    if (place)
        for (int sp = 0; sp < nspec; ++sp)
            for (int k = first[sp]; k < first[sp + 1]; ++k) {
                const int p0 = (k - first[sp]) * kMaxPathDev;
                st.spec[k].out_off = place->out_off[sp] + (int64_t)p0 * atms[sp].nwave;
                st.spec[k].jac_off = place->jac_off[sp] + (int64_t)p0 * atms[sp].nv * atms[sp].nwave;
            }
    struct Seg {
        const void* src;
        size_t n;
        size_t off;
    };
    std::vector<Seg> segs;
    size_t off = 0;
    auto add = [&](const void* p, size_t n) {
        off = (off + 255) & ~(size_t)255;
        segs.push_back({p, n, off});
        off += n;
        return segs.size() - 1;
    };
    const size_t i_spec = add(st.spec.data(), bytes_of(st.spec));
    const size_t i_item = add(st.item_start.data(), bytes_of(st.item_start));
    const size_t i_lay = add(st.lay.data(), bytes_of(st.lay));
    const size_t i_amo = add(st.amo.data(), bytes_of(st.amo));
    const size_t i_wave = add(st.wave.data(), bytes_of(st.wave));
    const size_t i_wg = add(st.wg_slice.data(), bytes_of(st.wg_slice));
    const size_t i_w2 = add(st.wg_w2.data(), st.any_noncoinc ? bytes_of(st.wg_w2) : 0);
    const size_t i_w1 = add(st.wg_w1.data(), st.any_w1 ? bytes_of(st.wg_w1) : 0);
    const size_t i_xsec = add(st.xsec.data(), bytes_of(st.xsec));
    const size_t i_cont = add(st.cont.data(), bytes_of(st.cont));
    const size_t i_pl = add(st.p_layinc.data(), bytes_of(st.p_layinc));
    const size_t i_ps = add(st.p_scale.data(), bytes_of(st.p_scale));
    const size_t i_pe = add(st.p_emtemp.data(), bytes_of(st.p_emtemp));
    const size_t i_mc = add(st.map_colptr.data(), bytes_of(st.map_colptr));
    const size_t i_mr = add(st.map_row.data(), bytes_of(st.map_row));
    const size_t i_mv = add(st.map_val.data(), bytes_of(st.map_val));
    const size_t i_parl = add(st.para_lay.data(), bytes_of(st.para_lay));
    const size_t i_parw = add(st.para_wave.data(), bytes_of(st.para_wave));
    const size_t i_lp = add(st.lpress.data(), bytes_of(st.lpress));
    const size_t i_lt = add(st.ltemp.data(), bytes_of(st.ltemp));
    const size_t i_wf = add(st.wfac.data(), bytes_of(st.wfac));
    const size_t in_bytes = off + 256;
    CUDA_TRY(c, c->h_in.ensure(in_bytes));
    CUDA_TRY(c, c->d_in.ensure(in_bytes));
    for (const auto& sg : segs)
        if (sg.n) memcpy((char*)c->h_in.p + sg.off, sg.src, sg.n);
    const cudaStream_t strm = stream_of(c);
    CUDA_TRY(c, cudaMemcpyAsync(c->d_in.p, c->h_in.p, off, cudaMemcpyHostToDevice, strm));
    const size_t out_bytes = place ? 0 : (size_t)(2 * st.n_out + st.n_jac) * sizeof(float);
    if (!place) {
        CUDA_TRY(c, c->d_out.ensure(out_bytes));
        CUDA_TRY(c, c->h_out.ensure(out_bytes));
    }
    CUDA_TRY(c, c->d_diag.ensure(64));
    auto dp = [&](size_t i) { return (const void*)((const char*)c->d_in.p + segs[i].off); };
    BatchDev& B = c->B;
    memset(&B, 0, sizeof B);
    B.nspec = (int)st.spec.size();   // device spectra: path groups of the caller's spectra
    B.nitems = st.item_start.back();
    B.item_start = (const int64_t*)dp(i_item);
    B.spec = (const SpecDev*)dp(i_spec);
    B.lay = (const LayerDev*)dp(i_lay);
    B.amo = (const float*)dp(i_amo);
    B.wave = (const WaveDev*)dp(i_wave);
    B.wg_slice = (const int64_t*)dp(i_wg);
    B.wg_w2 = st.any_noncoinc ? (const float*)dp(i_w2) : nullptr;
    B.wg_w1 = st.any_w1 ? (const float*)dp(i_w1) : nullptr;
    B.xsec = (const float*)dp(i_xsec);
    B.cont = (const float*)dp(i_cont);
    B.p_layinc = (const int*)dp(i_pl);
    B.p_scale = (const float*)dp(i_ps);
    B.p_emtemp = (const float*)dp(i_pe);
    B.map_colptr = (const int*)dp(i_mc);
    B.map_row = (const int*)dp(i_mr);
    B.map_val = (const float*)dp(i_mv);
    B.ktab_raw = (const float*)c->d_raw.p;
    B.ktab_log = (const float*)c->d_log.p;
    B.np = c->np;
    B.nt = std::abs(c->nt);
    B.t2 = c->nt < 0 ? 1 : 0;
    B.ng = c->ng;
    B.delg = (const float*)c->d_delg.p;
    B.g_ord = (const double*)c->d_gord.p;
    B.kcia = (const float*)c->d_kcia.p;
    B.e3tab = c->has_e3 ? (const double*)c->d_e3.p : nullptr;
    B.para = st.any_para ? 1 : 0;
    B.ext = (st.any_para || st.any_ext) ? 1 : 0;
    if (st.any_para) {
        const size_t nk = (size_t)c->ipara * RTB_CIA_NUMT * RTB_CIA_NUMWN;
        B.ipara = c->ipara;
        B.para_deltaf = c->para_deltaf;
        B.kh2h2 = (const float*)c->d_kpara.p;
        B.kh2he = B.kh2h2 + nk;
        B.kcia5 = B.kh2he + nk;
        B.para_lay = (const ParaLayDev*)dp(i_parl);
        B.para_wave = (const ParaWaveDev*)dp(i_parw);
    }
    B.lay_press = st.lpress.empty() ? nullptr : (const float*)dp(i_lp);
    B.lay_temp = st.ltemp.empty() ? nullptr : (const float*)dp(i_lt);
    B.wave_fac = st.wfac.empty() ? nullptr : (const float*)dp(i_wf);
    if (place) {
        B.calcout = place->calcout;
        B.gradtsurf = place->gradtsurf;
        B.gradients = place->gradients;
    } else {
        float* dout = (float*)c->d_out.p;
        B.calcout = dout;
        B.gradtsurf = dout + st.n_out;
        B.gradients = dout + 2 * st.n_out;
    }
    B.status = (unsigned*)c->d_diag.p;
    B.counters = (unsigned long long*)((char*)c->d_diag.p + 8);
    B.strict_ties = c->strict_ties;
    if (c->debug) {
        const rtb_atm& a0 = atms[0];
        const size_t npass = a0.ngas > 1 ? a0.ngas - 1 : 1;
        c->dbg_perm_n = (size_t)a0.nwave * a0.nlayer * npass * c->ng * c->ng;
        c->dbg_split_n = (size_t)a0.nwave * a0.nlayer * npass * c->ng;
        CUDA_TRY(c, c->d_dbg_perm.ensure(c->dbg_perm_n * 2));
        CUDA_TRY(c, c->d_dbg_split.ensure(c->dbg_split_n * 2));
        CUDA_TRY(c, cudaMemsetAsync(c->d_dbg_perm.p, 0xff, c->dbg_perm_n * 2, strm));
        CUDA_TRY(c, cudaMemsetAsync(c->d_dbg_split.p, 0xff, c->dbg_split_n * 2, strm));
        B.dbg_perm = (int16_t*)c->d_dbg_perm.p;
        B.dbg_split = (int16_t*)c->d_dbg_split.p;
    }
    // the scratch holds a slot for every block of the largest grid any tile launches
    int64_t grid = (int64_t)c->nsm * bpsm_all;
    if (grid > B.nitems) grid = B.nitems;
    c->grid = (int)grid;
    c->tile_eff = kWarps;
    c->bpsm_max = c->bpsm_w[kWarps];
    // one scratch slot per CTA: tau[Lmax][ng] + dtau[Lmax][nsw][ng]
    B.cell_Lmax = st.Lmax;
    B.cell_slot = (int64_t)st.Lmax * c->ng * (1 + st.nsw_max);
    B.nc_off = B.cell_slot;
    if (st.any_noncoinc) B.cell_slot += (int64_t)st.Lmax * st.ngas_max * kMaxNg * 2;
    B.cell_slot = (B.cell_slot + 63) & ~(int64_t)63;
    CUDA_TRY(c, c->d_cells.ensure((size_t)grid * B.cell_slot * sizeof(float)));
    B.cell_scratch = (float*)c->d_cells.p;
    c->Lmax = st.Lmax;
    c->nsw_max = st.nsw_max;
    c->ncol_max = st.ncol_max;
    c->nlmax_max = st.nlmax_max;
    c->npath_max = st.npath_max;
    c->spec_host.clear();
    for (int s = 0; s < nspec; ++s) c->spec_host.push_back(st.spec[first[s]]);   // outputs start at path 0
    c->spec_conv = std::move(convs);
    c->any_conv = any_conv;
    c->spec_npath.clear();
    c->spec_nv.clear();
    c->spec_nwave.clear();
    c->spec_nlayer.clear();
    c->cells = 0;
    c->spec_cost.clear();
    for (int s = 0; s < nspec; ++s) {
        c->spec_npath.push_back(atms[s].npath);
        c->spec_nv.push_back(atms[s].nv);
        c->spec_nwave.push_back(atms[s].nwave);
        c->spec_nlayer.push_back(atms[s].nlayer);
        c->cells += (long long)atms[s].nlayer * atms[s].nwave;
        // cost model of one item (wavenumber): layers x (1 + sorting overlap passes) x gradient columns
        int nabs = 0;
        for (int k = 0; k < atms[s].ngas; ++k)
            nabs += (atms[s].ktab[k] >= 0 || atms[s].ktab[k] == RTB_KTAB_BY_ID) ? 1 : 0;
        for (int k = first[s]; k < first[s + 1]; ++k)   // per device spectrum, as item_start_host
            c->spec_cost.push_back((float)atms[s].nlayer * (1.0f + 4.0f * std::max(nabs - 1, 0)) *
                                   (2.0f + st.spec[k].nsw));
    }
    c->item_start_host = st.item_start;
    c->order_ready = 0;
    c->n_out = st.n_out;
    c->n_jac = st.n_jac;
    c->in_bytes = off;
    c->out_bytes = out_bytes;
    c->placed = place ? 1 : 0;
    c->prepared = 1;
    // a batch of a shape tuned before starts with that tile and schedule;
    // any other batch with the caller's own choices (or the defaults)
    c->shape = {(st.Lmax + 19) / 20, st.ngas_max};
    const auto tn = c->tuned.find(c->shape);
    if (tn != c->tuned.end()) {
        c->tile = tn->second[0];
        c->sched = tn->second[1];
        c->occ = tn->second[2];
    } else {
        c->tile = c->tile_user;
        c->sched = c->sched_user;
        c->occ = c->occ_user;
    }
    return apply_schedule(c);
}

void drop_graph(rtb_context* c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
}

// grid, work counter and issue order of the resident batch from (sched, occ)
int apply_schedule(rtb_context* c) {
    drop_graph(c);
    BatchDev& B = c->B;
    const int w = fwd_tile_warps(B.t2, B.ext, c->tile);
    c->tile_eff = c->bpsm_w[w] > 0 ? w : kWarps;
    c->bpsm_max = c->bpsm_w[c->tile_eff];
    const int b = c->occ > 0 ? std::min(c->occ, c->bpsm_max) : c->bpsm_max;
    int64_t grid = (int64_t)c->nsm * b;
    if (grid > B.nitems) grid = B.nitems;
    c->grid = (int)std::max<int64_t>(grid, 1);
    B.work_next = c->sched >= 1 ? (unsigned long long*)((char*)c->d_diag.p + 48) : nullptr;
    B.item_order = nullptr;
    if (c->sched == 2) {
        if (!c->order_ready) {
            // longest-processing-time first: spectra by decreasing item cost, items of a spectrum together
            const int nspec = (int)c->spec_cost.size();
            std::vector<int> sp(nspec);
            for (int i = 0; i < nspec; ++i) sp[i] = i;
            std::stable_sort(sp.begin(), sp.end(), [&](int a, int b2) { return c->spec_cost[a] > c->spec_cost[b2]; });
            std::vector<int> order;
            order.reserve((size_t)B.nitems);
            for (int s : sp)
                for (int64_t it = c->item_start_host[s]; it < c->item_start_host[s + 1]; ++it) order.push_back((int)it);
            CUDA_TRY(c, c->d_order.ensure(order.size() * sizeof(int)));
            CUDA_TRY(c, cudaMemcpy(c->d_order.p, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
            c->order_ready = 1;
        }
        B.item_order = (const int*)c->d_order.p;
    }
    return RTB_OK;
}

int prepare(rtb_context* c, int nspec, const rtb_atm* atms) { return prepare_ex(c, nspec, atms, nullptr); }

int launch(rtb_context* c) {
    if (!c || !c->prepared) return fail(c, RTB_ERR_ARG, "no prepared batch (rtb_fwd_prepare)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t strm = stream_of(c);
    if (c->use_graph) {
        if (!c->gexec) {
            // one launch of the resident batch (status clear + forward kernel) as a graph
            cudaGraph_t g = nullptr;
            CUDA_TRY(c, cudaStreamBeginCapture(strm, cudaStreamCaptureModeRelaxed));
            cudaError_t e = cudaMemsetAsync(c->d_diag.p, 0, 64, strm);
            if (e == cudaSuccess)
                e = launch_fwd(c->B, c->nsw_max, c->ncol_max, c->nlmax_max, c->npath_max, c->grid, c->tile_eff, strm);
            const cudaError_t e2 = cudaStreamEndCapture(strm, &g);
            if (e != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return fail(c, RTB_ERR_CUDA, "graph capture of the forward launch failed: %s",
                            cudaGetErrorString(e != cudaSuccess ? e : e2));
            }
            c->graph = g;
            CUDA_TRY(c, cudaGraphInstantiate(&c->gexec, g, 0));
        }
        CUDA_TRY(c, cudaEventRecord(c->ev0, strm));
        CUDA_TRY(c, cudaGraphLaunch(c->gexec, strm));
        CUDA_TRY(c, cudaEventRecord(c->ev1, strm));
        c->launched_grid = c->grid;
        return RTB_OK;
    }
    CUDA_TRY(c, cudaMemsetAsync(c->d_diag.p, 0, 64, strm));
    CUDA_TRY(c, cudaEventRecord(c->ev0, strm));
    CUDA_TRY(c, launch_fwd(c->B, c->nsw_max, c->ncol_max, c->nlmax_max, c->npath_max, c->grid, c->tile_eff, strm));
    CUDA_TRY(c, cudaEventRecord(c->ev1, strm));
    c->launched_grid = c->grid;
    return RTB_OK;
}

// cirsrtfg_wave.f:448-516: the radiance, d/dtsurf and every Jacobian row of a
// spectrum with channels, convolved on the device from the batch's outputs
int fetch_convolved(rtb_context* c, cudaStream_t strm, float* const* calcout, float* const* gradients,
                    float* const* gradtsurf) {
    size_t need = 0;
    for (size_t s = 0; s < c->spec_host.size(); ++s)
        need = std::max(need, (size_t)c->spec_npath[s] * (2 + c->spec_nv[s]) * c->spec_conv[s].vconv.size());
    CUDA_TRY(c, c->d_convout.ensure(need * sizeof(float) + 16));
    const float* d = (const float*)c->d_out.p;
    float* o = (float*)c->d_convout.p;
    for (size_t s = 0; s < c->spec_host.size(); ++s) {
        const ConvSpec& cs = c->spec_conv[s];
        if (cs.vconv.empty()) continue;
        const SpecDev& S = c->spec_host[s];
        const int np = c->spec_npath[s], nv = c->spec_nv[s];
        const size_t nc = cs.vconv.size();
        const bool want_gt = gradtsurf && gradtsurf[s];
        const ConvSeg seg[3] = {{d + S.out_off, np, o},
                                {d + c->n_out + S.out_off, want_gt ? np : 0, o + np * nc},
                                {d + 2 * c->n_out + S.jac_off, np * nv, o + 2 * np * nc}};
        const int r = conv_run(c, cs, 3, seg, strm);
        if (r) return r;
        if (calcout && calcout[s])
            CUDA_TRY(c, cudaMemcpyAsync(calcout[s], o, np * nc * sizeof(float), cudaMemcpyDeviceToHost, strm));
        if (want_gt)
            CUDA_TRY(c, cudaMemcpyAsync(gradtsurf[s], o + np * nc, np * nc * sizeof(float), cudaMemcpyDeviceToHost,
                                        strm));
        if (gradients && gradients[s])
            CUDA_TRY(c, cudaMemcpyAsync(gradients[s], o + 2 * np * nc, (size_t)np * nv * nc * sizeof(float),
                                        cudaMemcpyDeviceToHost, strm));
        CUDA_TRY(c, cudaStreamSynchronize(strm));
    }
    return RTB_OK;
}

int fetch(rtb_context* c, float* const* calcout, float* const* gradients, float* const* gradtsurf) {
    if (!c || !c->prepared) return fail(c, RTB_ERR_ARG, "no prepared batch (rtb_fwd_prepare)");
    if (c->placed) return fail(c, RTB_ERR_ARG, "the resident batch belongs to the retrieval engine");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t strm = stream_of(c);
    CUDA_TRY(c, cudaMemcpyAsync(c->h_out.p, c->d_out.p, c->out_bytes, cudaMemcpyDeviceToHost, strm));
    unsigned long long diag[8];
    CUDA_TRY(c, cudaMemcpyAsync(diag, c->d_diag.p, 64, cudaMemcpyDeviceToHost, strm));
    CUDA_TRY(c, cudaStreamSynchronize(strm));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const unsigned status = (unsigned)(diag[0] & 0xffffffffu);
    c->stats.cells = c->cells;
    c->stats.sort_passes = (long long)diag[1];
    c->stats.tie_passes = (long long)diag[2];
    c->stats.exact_passes = (long long)diag[3];
    c->stats.irregular_passes = (long long)diag[4];
    c->stats.block_passes = (long long)diag[5];
    c->stats.ms_kernel = ms;
    c->stats.grid = c->launched_grid;
    c->stats.h2d_bytes = (long long)c->in_bytes;
    c->stats.d2h_bytes = (long long)c->out_bytes;
    if (status & kStGord) return fail(c, RTB_ERR_GORD, "g-ordinate walk ran past NG (rankg.f:118-147)");
    const float* h = (const float*)c->h_out.p;
    auto copy_out = [&](size_t s0, size_t s1) {
        for (size_t s = s0; s < s1; ++s) {
            if (c->any_conv && !c->spec_conv[s].vconv.empty()) continue;
            const SpecDev& S = c->spec_host[s];
            const size_t no = (size_t)c->spec_npath[s] * c->spec_nwave[s];
            const size_t nj = (size_t)c->spec_npath[s] * c->spec_nv[s] * c->spec_nwave[s];
            if (calcout && calcout[s]) memcpy(calcout[s], h + S.out_off, no * sizeof(float));
            if (gradtsurf && gradtsurf[s]) memcpy(gradtsurf[s], h + c->n_out + S.out_off, no * sizeof(float));
            if (gradients && gradients[s]) memcpy(gradients[s], h + 2 * c->n_out + S.jac_off, nj * sizeof(float));
        }
    };
    // a large batch is copied out by several host threads (spectrum ranges)
    const size_t nspec = c->spec_host.size();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nthr = (int)std::min<size_t>(std::min<unsigned>(hw, 16u), nspec / 8);
    if (nthr <= 1 || c->out_bytes < ((size_t)64 << 20)) {
        copy_out(0, nspec);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nthr; ++t)
            th.emplace_back(copy_out, nspec * t / nthr, nspec * (t + 1) / nthr);
        for (auto& x : th) x.join();
    }
    return c->any_conv ? fetch_convolved(c, strm, calcout, gradients, gradtsurf) : RTB_OK;
}

int run_batch(rtb_context* c, int nspec, const rtb_atm* atms, float* const* calcout, float* const* gradients,
              float* const* gradtsurf) {
    int r = prepare(c, nspec, atms);
    if (r) return r;
    r = launch(c);
    if (r) return r;
    return fetch(c, calcout, gradients, gradtsurf);
}

// Scratch of rtb_fwd_launch_static: one fixed array per device, part of the
// library's device image, so that the call never goes to the allocator.  The
// kernel writes every entry of a slot before it reads it, so nothing here has
// to start at zero.
static __device__ __align__(256) float g_fwd_static_scratch[RTB_STATIC_SCRATCH_BYTES / sizeof(float)];

constexpr int kMaxStaticDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kMaxStaticDevices] = {};

// device address of g_fwd_static_scratch on c->device (current), looked up
// once per device and kept for the process
int static_scratch_addr(rtb_context* c, float** out) {
    if (c->device >= kMaxStaticDevices)
        return fail(c, RTB_ERR_LIMIT, "static scratch supports devices 0..%d", kMaxStaticDevices - 1);
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[c->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_fwd_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(c, RTB_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed on device %d: %s", c->device,
                        cudaGetErrorString(e));
        g_static_addr[c->device] = p;
    }
    *out = (float*)g_static_addr[c->device];
    return RTB_OK;
}

int launch_static(rtb_context* c) {
    if (!c || !c->prepared) return fail(c, RTB_ERR_ARG, "no prepared batch (rtb_fwd_prepare)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    float* base = nullptr;
    const int r = static_scratch_addr(c, &base);
    if (r) return r;
    const size_t slot_bytes = (size_t)c->B.cell_slot * sizeof(float);
    const size_t nslot = (size_t)RTB_STATIC_SCRATCH_BYTES / slot_bytes;
    if (nslot < 1)
        return fail(c, RTB_ERR_LIMIT,
                    "forward scratch slot of %zu B (tau and dtau/dq of %d layers x NG %d, and the parked k of "
                    "off-grid wavenumbers) exceeds the static scratch of %u B",
                    slot_bytes, c->Lmax, c->ng, (unsigned)RTB_STATIC_SCRATCH_BYTES);
    const int grid = nslot < (size_t)c->grid ? (int)nslot : c->grid;
    BatchDev B = c->B;
    B.cell_scratch = base;
    const cudaStream_t strm = stream_of(c);
    CUDA_TRY(c, cudaMemsetAsync(c->d_diag.p, 0, 64, strm));
    CUDA_TRY(c, cudaEventRecord(c->ev0, strm));
    CUDA_TRY(c, launch_fwd(B, c->nsw_max, c->ncol_max, c->nlmax_max, c->npath_max, grid, c->tile_eff, strm));
    CUDA_TRY(c, cudaEventRecord(c->ev1, strm));
    c->launched_grid = grid;
    return RTB_OK;
}

}  // namespace rtb

extern "C" {

const char* rtb_version(void) { return "radtrancode_b200 0.1 (sm_100a)"; }

int rtb_create(int device, rtb_context** out) {
    if (!out) return RTB_ERR_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= device || device < 0) return RTB_ERR_CUDA;
    rtb_context* c = new rtb_context();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return RTB_ERR_CUDA; }
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        delete c;
        return RTB_ERR_CUDA;
    }
    *out = c;
    return RTB_OK;
}

void rtb_destroy(rtb_context* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->d_raw.release();
    c->d_log.release();
    c->d_delg.release();
    c->d_gord.release();
    c->d_kcia.release();
    c->d_in.release();
    c->d_out.release();
    c->d_diag.release();
    c->d_cells.release();
    c->d_dbg_perm.release();
    c->d_dbg_split.release();
    drop_graph(c);
    c->d_order.release();
    c->d_dq.release();
    c->d_conv.release();
    c->d_convout.release();
    c->d_layer.release();
    c->d_kpara.release();
    c->d_e3.release();
    c->d_nt32.release();
    c->d_nt64.release();
    c->d_ntsmall.release();
    c->d_ntdesc.release();
    c->h_in.release();
    c->h_out.release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* rtb_last_error(const rtb_context* c) { return c ? c->err.c_str() : "no context"; }

int rtb_set_ktable_ids(rtb_context* c, int ntab, const int* idgas, const int* isogas) {
    if (!c) return RTB_ERR_ARG;
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    if (ntab != c->ntab || !idgas || !isogas) return fail(c, RTB_ERR_ARG, "ids of %d tables, %d loaded", ntab, c->ntab);
    c->tab_id.assign(idgas, idgas + ntab);
    c->tab_iso.assign(isogas, isogas + ntab);
    return RTB_OK;
}

int rtb_set_ktable_centres(rtb_context* c, int npoint, const float* vcen) {
    if (!c) return RTB_ERR_ARG;
    if (c->ntab <= 0) return fail(c, RTB_ERR_NOTABLE, "no k-tables loaded");
    if (c->delv[0] > 0.0f) return fail(c, RTB_ERR_ARG, "k-table centres are for irregular grids (DELV <= 0)");
    if (!vcen || npoint != c->nbin[0]) return fail(c, RTB_ERR_ARG, "centres: npoint %d, the first table has %d", npoint, c->nbin[0]);
    for (int t = 0; t < c->ntab; ++t)
        if (c->nbin[t] < npoint)
            return fail(c, RTB_ERR_UNSUPPORTED, "k-table %d has %d records, fewer than the %d centres", t, c->nbin[t],
                        npoint);
    for (int i = 0; i < npoint; ++i)
        if (!(vcen[i] != 0.0f)) return fail(c, RTB_ERR_ARG, "k-table centre %d is zero", i);
    c->vcen.assign(vcen, vcen + npoint);
    return RTB_OK;
}

int rtb_set_ktables(rtb_context* c, int ntab, int np, int nt, int ng, const float* lnp, const float* tk,
                    const float* delg, const float* vmin, const float* delv, const int* nbin, const float* data) {
    if (!c) return RTB_ERR_ARG;
    if (ntab <= 0 || np < 2 || std::abs(nt) < 2 || ng < 1 || !lnp || !tk || !delg || !vmin || !delv || !nbin ||
        !data)
        return fail(c, RTB_ERR_ARG, "bad k-table arguments");
    if (np > RTB_MAXK || std::abs(nt) > RTB_MAXK || ng > RTB_MAXG || ntab > RTB_MAXGAS)
        return fail(c, RTB_ERR_LIMIT, "k-table grid exceeds MAXK/MAXG");
    if (ng > kMaxNg) return fail(c, RTB_ERR_UNSUPPORTED, "NG=%d > %d", ng, kMaxNg);
    // the FP64 cumulative-weight scan is exact in any order when every
    // product delg(i)*delg(j) >= 2^-28 and the total stays below 2
    double sdelg = 0.0;
    for (int i = 0; i < ng; ++i) {
        if (!(delg[i] >= 6.103515625e-05f)) return fail(c, RTB_ERR_UNSUPPORTED, "delg below 2^-14");
        sdelg += delg[i];
    }
    if (sdelg > 1.5) return fail(c, RTB_ERR_UNSUPPORTED, "sum of delg > 1.5");
    // an irregular grid (DELV <= 0) is one DELV for every table (read_klist.f:147-158)
    for (int t = 0; t < ntab; ++t)
        if ((!(delv[t] > 0.0f) || !(delv[0] > 0.0f)) && delv[t] != delv[0])
            return fail(c, RTB_ERR_ARG, "k-table %d: DELV %g differs from the first table's %g (read_klist.f:147-158)", t,
                        (double)delv[t], (double)delv[0]);
    CUDA_TRY(c, cudaSetDevice(c->device));
    c->ntab = 0;
    c->np = np;
    c->nt = nt;
    c->ng = ng;
    c->lnp.assign(lnp, lnp + np);
    c->tk.assign(tk, tk + (nt > 0 ? (size_t)nt : (size_t)np * -nt));   // TEMP(NT) or TEMP2(NP, |NT|)
    c->vcen.clear();
    c->tab_id.clear();
    c->tab_iso.clear();
    c->delg.assign(delg, delg + ng);
    c->g_ord.assign(ng + 1, 0.0);
    for (int i = 0; i < ng; ++i) c->g_ord[i + 1] = c->g_ord[i] + (double)delg[i];
    if (c->g_ord[ng] < 1.0) c->g_ord[ng] = 1.0;
    c->vmin.assign(vmin, vmin + ntab);
    c->delv.assign(delv, delv + ntab);
    c->nbin.assign(nbin, nbin + ntab);
    c->tab_off.assign(ntab, 0);
    c->nonzero.assign(ntab, {});
    const int64_t slice = (int64_t)np * std::abs(nt) * ng;
    int64_t total = 0;
    for (int t = 0; t < ntab; ++t) {
        if (nbin[t] <= 0) return fail(c, RTB_ERR_ARG, "table %d has no bins", t);
        c->tab_off[t] = total;
        total += (int64_t)nbin[t] * slice;
    }
    std::vector<float> lg((size_t)total);
    for (int t = 0; t < ntab; ++t) {
        c->nonzero[t].assign(nbin[t], 0);
        for (int b = 0; b < nbin[t]; ++b) {
            const float* s = data + c->tab_off[t] + (int64_t)b * slice;
            uint8_t any = 0;
            for (int64_t i = 0; i < slice; ++i)
                if (s[i] > 0.0f) { any = 1; break; }
            c->nonzero[t][b] = any;
        }
    }
    for (int64_t i = 0; i < total; ++i) lg[i] = (float)std::log((double)data[i]);
    CUDA_TRY(c, c->d_raw.ensure((size_t)total * 4));
    CUDA_TRY(c, c->d_log.ensure((size_t)total * 4));
    CUDA_TRY(c, c->d_delg.ensure(4 * 64));
    CUDA_TRY(c, c->d_gord.ensure(8 * 64));
    CUDA_TRY(c, cudaMemcpy(c->d_raw.p, data, (size_t)total * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(c->d_log.p, lg.data(), (size_t)total * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(c->d_delg.p, delg, (size_t)ng * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(c->d_gord.p, c->g_ord.data(), (size_t)(ng + 1) * 8, cudaMemcpyHostToDevice));
    c->ntab = ntab;
    return RTB_OK;
}

int rtb_set_cia(rtb_context* c, float dnu, const double* temps, const float* kcia) {
    if (!c) return RTB_ERR_ARG;
    if (!temps || !kcia || !(dnu > 0.0f)) return fail(c, RTB_ERR_ARG, "bad CIA arguments");
    CUDA_TRY(c, cudaSetDevice(c->device));
    c->dnu = dnu;
    c->cia_tk.resize(RTB_CIA_NUMT);
    for (int i = 0; i < RTB_CIA_NUMT; ++i) c->cia_tk[i] = (float)temps[i];
    const size_t n = (size_t)RTB_CIA_NUMPAIRS * RTB_CIA_NUMT * RTB_CIA_NUMWN;
    CUDA_TRY(c, c->d_kcia.ensure(n * 4));
    CUDA_TRY(c, cudaMemcpy(c->d_kcia.p, kcia, n * 4, cudaMemcpyHostToDevice));
    c->has_cia = 1;
    return RTB_OK;
}

int rtb_set_e3_table(rtb_context* c, int n, const double* tran, const double* e3) {
    if (!c) return RTB_ERR_ARG;
    constexpr int kMtab = 1001;   // e3interp.f: PARAMETER (mtab=1001)
    if (n != kMtab || !tran || !e3) return fail(c, RTB_ERR_ARG, "E3 table: %d points (e3interp.f holds 1001)", n);
    if (tran[kMtab - 1] != 1.0) return fail(c, RTB_ERR_ARG, "E3 table: the last transmission must be 1");
    std::vector<double> t(3 * kMtab);
    const double dtrans = (double)(1.0f / (float)(kMtab - 1));   // REAL 1.0/float(mtab-1) into DOUBLE
    for (int i = 0; i < kMtab; ++i) {
        t[i] = tran[i];
        t[kMtab + i] = e3[i];
    }
    double* eg = t.data() + 2 * kMtab;   // egrad (e3interp.f:36-40)
    eg[0] = (e3[1] - e3[0]) / dtrans;
    eg[kMtab - 1] = (e3[kMtab - 1] - e3[kMtab - 2]) / dtrans;
    for (int i = 1; i < kMtab - 1; ++i) eg[i] = 0.5 * (e3[i + 1] - e3[i - 1]) / dtrans;
    CUDA_TRY(c, cudaSetDevice(c->device));
    CUDA_TRY(c, c->d_e3.ensure(t.size() * 8));
    CUDA_TRY(c, cudaMemcpy(c->d_e3.p, t.data(), t.size() * 8, cudaMemcpyHostToDevice));
    c->has_e3 = 1;
    return RTB_OK;
}

int rtb_set_stellar_spectrum(rtb_context* c, int npt, const float* wave, const float* rad) {
    if (!c) return RTB_ERR_ARG;
    if (npt < 2 || !wave || !rad) return fail(c, RTB_ERR_ARG, "stellar spectrum: %d points", npt);
    for (int i = 0; i < npt; ++i)
        if (!std::isfinite(wave[i]) || !std::isfinite(rad[i]))
            return fail(c, RTB_ERR_ARG, "stellar spectrum: point %d not finite", i);
    c->solar_wave.assign(wave, wave + npt);
    c->solar_rad.assign(rad, rad + npt);
    return RTB_OK;
}

int rtb_set_para_cia(rtb_context* c, float dnu2, int ipara, const float* temps, const float* fp, const float* kh2h2,
                     const float* kh2he, const float* kcia5) {
    if (!c) return RTB_ERR_ARG;
    if (!(dnu2 > 0.0f) || (ipara != 12 && ipara != 24) || !temps || !fp || !kh2h2 || !kh2he || !kcia5)
        return fail(c, RTB_ERR_ARG, "bad para-H2 CIA arguments (ipara 12 or 24)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const size_t nk = (size_t)ipara * RTB_CIA_NUMT * RTB_CIA_NUMWN, n5 = (size_t)5 * RTB_CIA_NUMT * RTB_CIA_NUMWN;
    CUDA_TRY(c, c->d_kpara.ensure((2 * nk + n5) * 4));
    float* d = (float*)c->d_kpara.p;
    CUDA_TRY(c, cudaMemcpy(d, kh2h2, nk * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(d + nk, kh2he, nk * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(d + 2 * nk, kcia5, n5 * 4, cudaMemcpyHostToDevice));
    c->para_tk.assign(temps, temps + RTB_CIA_NUMT);
    c->para_fp.assign(fp, fp + ipara);
    c->para_deltaf = fp[1] - fp[0];   // fpread_all.f:197
    c->para_vk.resize(RTB_CIA_NUMWN);
    for (int i = 0; i < RTB_CIA_NUMWN; ++i) c->para_vk[i] = (float)i * dnu2;
    c->ipara = ipara;
    c->dnu2 = dnu2;
    c->has_para = 1;
    return RTB_OK;
}

int rtb_cirsrtfg_wave(rtb_context* c, const rtb_atm* atm, float* calcout, float* gradients, float* gradtsurf) {
    if (!c || !atm || !calcout || !gradients) return fail(c, RTB_ERR_ARG, "NULL argument");
    return run_batch(c, 1, atm, &calcout, &gradients, &gradtsurf);
}

int rtb_cirsrtfg_wave_batch(rtb_context* c, int nspec, const rtb_atm* atms, float* const* calcout,
                            float* const* gradients, float* const* gradtsurf) {
    return run_batch(c, nspec, atms, calcout, gradients, gradtsurf);
}

int rtb_fwd_prepare(rtb_context* c, int nspec, const rtb_atm* atms) { return prepare(c, nspec, atms); }

int rtb_fwd_launch(rtb_context* c) { return launch(c); }

int rtb_fwd_fetch(rtb_context* c, float* const* calcout, float* const* gradients, float* const* gradtsurf) {
    return fetch(c, calcout, gradients, gradtsurf);
}

int rtb_set_stream(rtb_context* c, void* stream) {
    if (!c) return RTB_ERR_ARG;
    c->user_stream = (cudaStream_t)stream;
    return RTB_OK;
}

int rtb_get_fwd_stats(const rtb_context* c, rtb_fwd_stats* out) {
    if (!c || !out) return RTB_ERR_ARG;
    *out = c->stats;
    return RTB_OK;
}

int rtb_set_debug(rtb_context* c, int on) {
    if (!c) return RTB_ERR_ARG;
    c->debug = on ? 1 : 0;
    return RTB_OK;
}

int rtb_set_strict_ties(rtb_context* c, int on) {
    if (!c) return RTB_ERR_ARG;
    c->strict_ties = on ? 1 : 0;
    return RTB_OK;
}

int rtb_fwd_launch_static(rtb_context* c) { return launch_static(c); }

int rtb_fwd_set_schedule(rtb_context* c, int schedule, int blocks_per_sm) {
    if (!c) return RTB_ERR_ARG;
    if (schedule < 0 || schedule > 2 || blocks_per_sm < 0)
        return fail(c, RTB_ERR_ARG, "schedule %d, blocks_per_sm %d", schedule, blocks_per_sm);
    c->sched = c->sched_user = schedule;
    c->occ = c->occ_user = blocks_per_sm;
    if (!c->prepared) return RTB_OK;
    CUDA_TRY(c, cudaSetDevice(c->device));
    return apply_schedule(c);
}

int rtb_fwd_set_tile(rtb_context* c, int warps) {
    if (!c) return RTB_ERR_ARG;
    if (!(warps == 0 || warps == 2 || warps == 4 || warps == 8))
        return fail(c, RTB_ERR_ARG, "tile of %d warps per block (2, 4 or 8)", warps);
    c->tile = c->tile_user = warps ? warps : kTileDefault;
    if (!c->prepared) return RTB_OK;
    CUDA_TRY(c, cudaSetDevice(c->device));
    return apply_schedule(c);
}

int rtb_fwd_autotune(rtb_context* c, rtb_fwd_tune* out) {
    if (!c || !c->prepared) return fail(c, RTB_ERR_ARG, "no prepared batch (rtb_fwd_prepare)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t strm = stream_of(c);
    const int keep_graph = c->use_graph;
    c->use_graph = 0;
    float best = 3.4e38f;
    int best_w = kWarps, best_s = 0, best_b = c->bpsm_w[kWarps], n = 0;
    for (int w : {4, 8, 2}) {
        if (fwd_tile_warps(c->B.t2, c->B.ext, w) != w || c->bpsm_w[w] <= 0) continue;
        const int bmax = c->bpsm_w[w];
        for (int sch = 0; sch <= 2; ++sch)
            for (int b = bmax; b >= 1 && b >= bmax - 2; --b) {
                c->tile = w;
                c->sched = sch;
                c->occ = b;
                int r = apply_schedule(c);
                if (r) return r;
                float ms = 0.0f;
                for (int rep = 0; rep < 2; ++rep) {   // the second launch is timed
                    r = launch(c);
                    if (r) return r;
                    CUDA_TRY(c, cudaStreamSynchronize(strm));
                    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
                }
                ++n;
                if (ms < best) {
                    best = ms;
                    best_w = w;
                    best_s = sch;
                    best_b = b;
                }
            }
    }
    c->tile = best_w;
    c->sched = best_s;
    c->occ = best_b;
    c->use_graph = keep_graph;
    c->tuned[c->shape] = {best_w, best_s, best_b};
    const int r = apply_schedule(c);
    if (r) return r;
    if (out) {
        out->schedule = best_s;
        out->blocks_per_sm = best_b;
        out->ms = best;
        out->candidates = n;
        out->warps = best_w;
    }
    return RTB_OK;
}

int rtb_fwd_use_graph(rtb_context* c, int on) {
    if (!c) return RTB_ERR_ARG;
    c->use_graph = on ? 1 : 0;
    drop_graph(c);
    return RTB_OK;
}

int rtb_cirsradg_wave(rtb_context* c, const rtb_atm* atm, int nsw, const int* isw, float* output, float* gtsurf,
                      float* doutputdq, int ld_pat, int ld_lay, int ld_param) {
    if (!c) return RTB_ERR_ARG;
    if (!atm || atm->nwave != 1 || nsw < 0 || nsw > kMaxSw || (nsw > 0 && !isw) || !output || !doutputdq)
        return fail(c, RTB_ERR_ARG, "cirsradg_wave: bad arguments (one wavenumber, 0 <= nsw <= %d)", kMaxSw);
    const rtb_atm& a0 = *atm;
    const int nparam = a0.ngas + 1 + a0.ncont;
    if (ld_pat < a0.npath || ld_lay < a0.nlayer || ld_param < nparam)
        return fail(c, RTB_ERR_ARG, "cirsradg_wave: doutputdq leading dimensions too small");
    if (a0.npath > kMaxPathDev)   // its per-path derivatives are captured for one path group only
        return fail(c, RTB_ERR_UNSUPPORTED, "cirsradg_wave: more than %d paths", kMaxPathDev);
    for (int s = 0; s < nsw; ++s)
        if (isw[s] < 0 || isw[s] >= nparam || (s > 0 && isw[s] <= isw[s - 1]))
            return fail(c, RTB_ERR_ARG, "cirsradg_wave: isw must increase within 0..%d", nparam - 1);
    // a one-element state that selects exactly the isw parameters, so that
    // the set-up derives the same isw (cirsrtfg_wave.f:301-313); its mapped
    // Jacobian is not used
    const int ldl = a0.ld_lay > 0 ? a0.ld_lay : RTB_MAXLAY;
    std::vector<float> xm(nparam, 0.0f), zl(ldl, 0.0f);
    for (int s = 0; s < nsw; ++s) xm[isw[s]] = 1.0f;
    rtb_atm a = a0;
    a.fwhm = 0.0f;   // cirsradg_wave returns the calculation-grid values
    a.conv = nullptr;
    a.nv = 1;
    a.npro = 1;
    a.ld_v = 1;
    a.ld_param = nparam;
    a.xmap = xm.data();
    a.dte = zl.data();
    a.dam = zl.data();
    a.dco = a0.ncont > 0 ? zl.data() : nullptr;
    int r = prepare(c, 1, &a);
    if (r) return r;
    const int64_t stride = (int64_t)c->nlmax_max * c->nsw_max;
    CUDA_TRY(c, c->d_dq.ensure((size_t)a.npath * stride * sizeof(float) + 16));
    drop_graph(c);
    c->B.dq_out = (float*)c->d_dq.p;
    c->B.dq_stride = stride;
    c->B.dq_npath = a.npath;
    r = launch(c);
    c->B.dq_out = nullptr;
    if (r) return r;
    std::vector<float> co(a.npath), gr(a.npath), gt(a.npath), dq((size_t)a.npath * stride);
    float* pc = co.data();
    float* pg = gr.data();
    float* pt = gt.data();
    r = fetch(c, &pc, &pg, &pt);
    if (r) return r;
    CUDA_TRY(c, cudaMemcpy(dq.data(), c->d_dq.p, dq.size() * sizeof(float), cudaMemcpyDeviceToHost));
    // cirsradg_wave.f:1240-1267: zero, then the isw columns of the path's layers
    for (int ip = 0; ip < a.npath; ++ip) {
        output[ip] = co[ip];
        if (gtsurf) gtsurf[ip] = gt[ip];
        for (int k = 0; k < nparam; ++k)
            for (int j = 0; j < ld_lay; ++j) doutputdq[ip + (size_t)ld_pat * (j + (size_t)ld_lay * k)] = 0.0f;
        for (int j = 0; j < a.nlayin[ip]; ++j)
            for (int s = 0; s < nsw; ++s)
                doutputdq[ip + (size_t)ld_pat * (j + (size_t)ld_lay * isw[s])] = dq[ip * stride + j * nsw + s];
    }
    return RTB_OK;
}

int rtb_get_debug_bins(const rtb_context* c, int16_t* perm, size_t n_perm, int16_t* split, size_t n_split) {
    if (!c || !c->debug) return RTB_ERR_ARG;
    if (perm) {
        if (n_perm < c->dbg_perm_n) return RTB_ERR_ARG;
        if (cudaMemcpy(perm, c->d_dbg_perm.p, c->dbg_perm_n * 2, cudaMemcpyDeviceToHost) != cudaSuccess)
            return RTB_ERR_CUDA;
    }
    if (split) {
        if (n_split < c->dbg_split_n) return RTB_ERR_ARG;
        if (cudaMemcpy(split, c->d_dbg_split.p, c->dbg_split_n * 2, cudaMemcpyDeviceToHost) != cudaSuccess)
            return RTB_ERR_CUDA;
    }
    return RTB_OK;
}

}  // extern "C"
