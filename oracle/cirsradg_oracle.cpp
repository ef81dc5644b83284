/*
 * cirsradg_oracle.cpp -- ORACLE (test infrastructure only; see oracle.h).
 *
 * Line-by-line CPU restatement of the reference's correlated-k gradient
 * forward model.  Each function names the Fortran file:line it follows
 * (paths relative to the reference repository root).  Written in templated
 * C++: R = float reproduces the reference's REAL arithmetic (DOUBLE
 * PRECISION variables stay double), R = double promotes everything.
 *
 * Build with -ffp-contract=off so that no multiply-add is fused: gfortran
 * -O2 on x86-64 evaluates every REAL expression as separate IEEE operations
 * left to right, and this file spells each expression in that order.
 */
#include "oracle.h"
#include "detexp.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int kMaxG = RTB_MAXG;
/* 0: the reference heapsort (default).  1: stable sort by key, ties in
 * element order -- used by the oracle tests to show which passes depend on
 * the heapsort's order of tied keys. */
int g_sort_mode = 0;

template <class R> struct Prec;
template <> struct Prec<float> {
    static float EXP(float x) { return orc_det_expf(x); }
    static float LOG(float x) { return (float)std::log((double)x); }
    static bool isnan_(float x) { return x != x; }
};
template <> struct Prec<double> {
    static double EXP(double x) { return std::exp(x); }
    static double LOG(double x) { return std::log(x); }
    static bool isnan_(double x) { return x != x; }
};

/* LOCATE: radtran/scatter/locate.f:1-28 (the copy linked into cirsradg;
 * scatter.a precedes libfrecipes.a on the link line). 1-based result. */
template <class R>
int locate(const R* xx, int n, R x) {
    int jl = 0, ju = n + 1;
    while (ju - jl > 1) {
        int jm = (ju + jl) / 2;
        if ((xx[n - 1] >= xx[0]) == (x >= xx[jm - 1])) jl = jm; else ju = jm;
    }
    if (x == xx[0]) return 1;
    if (x == xx[n - 1]) return n - 1;
    return jl;
}

/* FINDLOC: radtran/cirsrad/findloc.f:13-100.  The 1-based range [I1, I2] of
 * the grid x inside [y1, y2] (0, 0 when disjoint), the ends snapped to grid
 * points within 1e-5. */
void findloc(const float* x, int nx, float y1, float y2, int& I1, int& I2) {
    const bool up = x[0] < x[nx - 1];
    const float xbot = up ? x[0] : x[nx - 1], xtop = up ? x[nx - 1] : x[0];
    const int Ibot = up ? 1 : nx, Itop = up ? nx : 1;
    if ((y1 < xbot && y2 < xbot) || (y1 > xtop && y2 > xtop)) {
        I1 = I2 = 0;
        return;
    }
    int I1f, I2f;
    const float ys[2] = {y1, y2};
    int* Is[2] = {&I1, &I2};
    int* fs[2] = {&I1f, &I2f};
    for (int e = 0; e < 2; ++e) {
        const float y = ys[e];
        if (y <= xbot) { *Is[e] = Ibot; *fs[e] = 1; }
        else if (y >= xtop) { *Is[e] = Itop; *fs[e] = 1; }
        else {
            const int it = locate<float>(x, nx, y);
            *Is[e] = it;
            *fs[e] = 0;
            for (int I = it; I <= it + 1; ++I)
                if (std::fabs(y - x[I - 1]) < 1.e-5f) { *Is[e] = I; *fs[e] = 1; }
        }
    }
    if (y1 < y2) { if (I1f == 0) I1 = I1 + 1; }
    else { if (I2f == 0) I2 = I2 + 1; }
}

/* SORT2G: radtran/cirsradg/sort2g.f:1-52, Numerical Recipes heapsort that
 * carries an integer index.  ra/ib are 0-based storage of RA(1..N)/IB(1..N).
 * N < 2 is not reached by the reference path (NG >= 2 checked by caller). */
template <class R>
void sort2g(int n, R* ra0, int* ib0) {
    if (n < 2) return;
    R* RA = ra0 - 1;
    int* IB = ib0 - 1;
    int L = n / 2 + 1, IR = n;
    R RRA;
    int IRB;
    for (;;) {
        if (L > 1) {
            L = L - 1;
            RRA = RA[L];
            IRB = IB[L];
        } else {
            RRA = RA[IR];
            IRB = IB[IR];
            RA[IR] = RA[1];
            IB[IR] = IB[1];
            IR = IR - 1;
            if (IR == 1) {
                RA[1] = RRA;
                IB[1] = IRB;
                return;
            }
        }
        int I = L, J = L + L;
        while (J <= IR) {
            if (J < IR) {
                if (RA[J] < RA[J + 1]) J = J + 1;
            }
            if (RRA < RA[J]) {
                RA[I] = RA[J];
                IB[I] = IB[J];
                I = J;
                J = J + J;
            } else {
                J = IR + 1;
            }
        }
        RA[I] = RRA;
        IB[I] = IRB;
    }
}

/* RANKG: radtran/cirsradg/rankg.f:59-152.  grad is [nparam][nloop]
 * (column iparam of grad(maxrank, maxgas+1)); dkdq is [nparam][ng].
 * Cumulative g (g_ord, gdist), sum and frac are DOUBLE PRECISION.
 * perm/split: optional debug capture of the assignment. */
template <class R>
int rankg(int nparam, const R* gw, int ng, int nloop, R* weight, R* cont, R* grad,
          R* k_g, R* dkdq, int16_t* perm, int16_t* split, int16_t* ties = nullptr) {
    double g_ord[kMaxG + 2];
    g_ord[0] = 0.0;
    for (int i = 0; i < ng; ++i) g_ord[i + 1] = g_ord[i] + (double)gw[i];
    if (g_ord[ng] < 1.0) g_ord[ng] = 1.0;                 /* rankg.f:65-67 */

    std::vector<int> ico(nloop);
    for (int i = 0; i < nloop; ++i) ico[i] = i + 1;
    if (g_sort_mode == 0) {
        sort2g<R>(nloop, cont, ico.data());
    } else {
        std::stable_sort(ico.begin(), ico.end(), [&](int a, int b) { return cont[a - 1] < cont[b - 1]; });
        std::vector<R> c2(nloop);
        for (int i = 0; i < nloop; ++i) c2[i] = cont[ico[i] - 1];
        for (int i = 0; i < nloop; ++i) cont[i] = c2[i];
    }

    std::vector<R> tmp(nloop);
    for (int i = 0; i < nloop; ++i) tmp[i] = weight[ico[i] - 1];
    for (int i = 0; i < nloop; ++i) weight[i] = tmp[i];
    for (int p = 0; p < nparam; ++p) {
        R* g = grad + (size_t)p * nloop;
        for (int i = 0; i < nloop; ++i) tmp[i] = g[ico[i] - 1];
        for (int i = 0; i < nloop; ++i) g[i] = tmp[i];
    }
    if (perm) for (int i = 0; i < nloop; ++i) perm[i] = (int16_t)(ico[i] - 1);
    if (ties) {
        int n = 0;
        for (int i = 1; i < nloop; ++i) n += (cont[i] == cont[i - 1]);
        *ties = (int16_t)n;
    }
    if (split) for (int b = 0; b < ng; ++b) split[b] = -1;

    std::vector<double> gdist(nloop + 1);
    gdist[0] = 0.0;
    gdist[1] = (double)weight[0];
    for (int i = 2; i <= nloop; ++i) gdist[i] = (double)weight[i - 1] + gdist[i - 1];

    for (int i = 0; i < ng; ++i) {
        k_g[i] = 0;
        for (int p = 0; p < nparam; ++p) dkdq[(size_t)p * ng + i] = 0;
    }
    int ig = 1;
    double sum = 0.0;
    for (int I = 1; I <= nloop; ++I) {
        const R c = cont[I - 1], w = weight[I - 1];
        if (ig > ng) return RTB_ERR_GORD;  /* reference reads g_ord(ng+2): undefined */
        if (gdist[I] < g_ord[ig]) {
            k_g[ig - 1] = k_g[ig - 1] + c * w;
            for (int p = 0; p < nparam; ++p)
                dkdq[(size_t)p * ng + ig - 1] =
                    dkdq[(size_t)p * ng + ig - 1] + grad[(size_t)p * nloop + I - 1] * w;
            sum = sum + (double)w;
        } else {
            const double frac = (g_ord[ig] - gdist[I - 1]) / (gdist[I] - gdist[I - 1]);
            const R sf = (R)frac;
            k_g[ig - 1] = k_g[ig - 1] + sf * c * w;
            for (int p = 0; p < nparam; ++p)
                dkdq[(size_t)p * ng + ig - 1] =
                    dkdq[(size_t)p * ng + ig - 1] + sf * grad[(size_t)p * nloop + I - 1] * w;
            sum = sum + frac * (double)w;
            k_g[ig - 1] = k_g[ig - 1] / (R)sum;
            for (int p = 0; p < nparam; ++p)
                dkdq[(size_t)p * ng + ig - 1] = dkdq[(size_t)p * ng + ig - 1] / (R)sum;
            if (split) split[ig - 1] = (int16_t)(I - 1);
            ig = ig + 1;
            sum = (1.0 - frac) * (double)w;
            if (ig <= ng) {  /* the reference writes k_g(ng+1) of a MAXG array: unused */
                const R sr = (R)(1.0 - frac);
                k_g[ig - 1] = sr * c * w;
                for (int p = 0; p < nparam; ++p)
                    dkdq[(size_t)p * ng + ig - 1] = sr * grad[(size_t)p * nloop + I - 1] * w;
            }
        }
    }
    if (ig == ng) {
        k_g[ig - 1] = k_g[ig - 1] / (R)sum;
        for (int p = 0; p < nparam; ++p)
            dkdq[(size_t)p * ng + ig - 1] = dkdq[(size_t)p * ng + ig - 1] / (R)sum;
    }
    return RTB_OK;
}

/* RANKK: radtran/cirsradg/rankk.f:34-117 -- REAL g_ord/gdist/sum/frac,
 * `<=` test and the ig <= ng guards.  Used by the non-coincident branch of
 * get_kg (get_kg.f:380-438). */
template <class R>
void rankk(const R* gw, int ng, R* cont, R* dcont, R* weight, int nloop, R* k_g, R* dkdt) {
    R g_ord[kMaxG + 2];
    g_ord[0] = 0;
    for (int i = 0; i < ng; ++i) g_ord[i + 1] = g_ord[i] + gw[i];
    if (g_ord[ng] < (R)1.0) g_ord[ng] = (R)1.0;
    std::vector<int> ico(nloop);
    for (int i = 0; i < nloop; ++i) ico[i] = i + 1;
    sort2g<R>(nloop, cont, ico.data());
    std::vector<R> tmp(nloop);
    for (int i = 0; i < nloop; ++i) tmp[i] = weight[ico[i] - 1];
    for (int i = 0; i < nloop; ++i) weight[i] = tmp[i];
    for (int i = 0; i < nloop; ++i) tmp[i] = dcont[ico[i] - 1];
    for (int i = 0; i < nloop; ++i) dcont[i] = tmp[i];
    std::vector<R> gdist(nloop + 1);
    gdist[0] = 0;
    gdist[1] = weight[0];
    for (int i = 2; i <= nloop; ++i) gdist[i] = weight[i - 1] + gdist[i - 1];
    for (int i = 0; i < ng; ++i) { k_g[i] = 0; dkdt[i] = 0; }
    int ig = 1;
    R sum = 0;
    for (int I = 1; I <= nloop; ++I) {
        if (ig <= ng && gdist[I] <= g_ord[ig]) {
            k_g[ig - 1] = k_g[ig - 1] + cont[I - 1] * weight[I - 1];
            dkdt[ig - 1] = dkdt[ig - 1] + dcont[I - 1] * weight[I - 1];
            sum = sum + weight[I - 1];
        } else {
            /* with ig > ng the reference reads g_ord(ng+2) and writes
             * k_g(ng+1); those slots are never used afterwards */
            if (ig > ng) continue;
            const R frac = (g_ord[ig] - gdist[I - 1]) / (gdist[I] - gdist[I - 1]);
            k_g[ig - 1] = k_g[ig - 1] + frac * cont[I - 1] * weight[I - 1];
            dkdt[ig - 1] = dkdt[ig - 1] + frac * dcont[I - 1] * weight[I - 1];
            sum = sum + frac * weight[I - 1];
            k_g[ig - 1] = k_g[ig - 1] / sum;
            dkdt[ig - 1] = dkdt[ig - 1] / sum;
            ig = ig + 1;
            if (ig <= ng) {
                sum = ((R)1.0 - frac) * weight[I - 1];
                k_g[ig - 1] = ((R)1.0 - frac) * cont[I - 1] * weight[I - 1];
                dkdt[ig - 1] = ((R)1.0 - frac) * dcont[I - 1] * weight[I - 1];
            }
        }
    }
    if (ig == ng) {
        k_g[ig - 1] = k_g[ig - 1] / sum;
        dkdt[ig - 1] = dkdt[ig - 1] / sum;
    }
}

/* NOVERLAPG: radtran/cirsradg/noverlapg.f:64-198.
 * k_gn/dkgndt: [ngas][ng]; amount[ngas]; outputs k_g[ng], dkdq[ngas+1][ng]
 * (column-major dkdq(maxg, maxgas+1) restricted to its first ngas+1 columns).
 * dbg_perm/dbg_split: per pass (igas-1) records, may be NULL. */
template <class R>
int noverlapg(const R* delg, int ng, int ngas, const R* amount, const R* k_gn, const R* dkgndt,
              R* k_g, R* dkdq, int16_t* dbg_perm, int16_t* dbg_split, int16_t* dbg_ties) {
    const int nrank = ng * ng;
    std::vector<R> contri(nrank), weight(nrank), grad((size_t)(ngas + 1) * nrank);
    R k_g1[kMaxG], k_g2[kMaxG], dk1dT[kMaxG], dk2dT[kMaxG];
    auto DK = [&](int i, int col) -> R& { return dkdq[(size_t)col * ng + i]; }; /* col 0-based */
    for (int igas = 1; igas <= ngas - 1; ++igas) {
        int16_t* pperm = dbg_perm ? dbg_perm + (size_t)(igas - 1) * nrank : nullptr;
        int16_t* psplit = dbg_split ? dbg_split + (size_t)(igas - 1) * ng : nullptr;
        if (pperm) for (int i = 0; i < nrank; ++i) pperm[i] = -1;
        if (psplit) for (int i = 0; i < ng; ++i) psplit[i] = -1;
        int16_t* pties = dbg_ties ? dbg_ties + (igas - 1) : nullptr;
        if (pties) *pties = -1;
        int nloop = 0;
        if (igas == 1) {
            const R a1 = amount[igas - 1], a2 = amount[igas];
            for (int i = 0; i < ng; ++i) {
                k_g1[i] = k_gn[(size_t)(igas - 1) * ng + i];
                k_g2[i] = k_gn[(size_t)igas * ng + i];
                dk1dT[i] = dkgndt[(size_t)(igas - 1) * ng + i];
                dk2dT[i] = dkgndt[(size_t)igas * ng + i];
            }
            if (k_g1[ng - 1] == 0) {                          /* noverlapg.f:88-97 */
                for (int i = 0; i < ng; ++i) {
                    k_g[i] = k_g2[i] * a2;
                    DK(i, igas - 1) = 0;
                    DK(i, igas) = k_g2[i];
                    DK(i, igas + 1) = dk2dT[i] * a2;
                }
                continue;
            }
            if (k_g2[ng - 1] == 0) {                          /* noverlapg.f:99-108 */
                for (int i = 0; i < ng; ++i) {
                    k_g[i] = k_g1[i] * a1;
                    DK(i, igas - 1) = k_g1[i];
                    DK(i, igas) = 0;
                    DK(i, igas + 1) = dk1dT[i] * a1;
                }
                continue;
            }
            for (int i = 0; i < ng; ++i)
                for (int j = 0; j < ng; ++j) {
                    weight[nloop] = delg[i] * delg[j];
                    contri[nloop] = k_g1[i] * a1 + k_g2[j] * a2;
                    grad[(size_t)(igas - 1) * nrank + nloop] = k_g1[i];
                    grad[(size_t)igas * nrank + nloop] = k_g2[j];
                    grad[(size_t)(igas + 1) * nrank + nloop] = dk1dT[i] * a1 + dk2dT[j] * a2;
                    ++nloop;
                }
        } else {
            const R a2 = amount[igas];
            for (int i = 0; i < ng; ++i) {
                k_g1[i] = k_g[i];
                k_g2[i] = k_gn[(size_t)igas * ng + i];
                dk1dT[i] = DK(i, igas);           /* dkdq(i, igas+1): dK/dT of the sum */
                dk2dT[i] = dkgndt[(size_t)igas * ng + i];
            }
            if (k_g1[ng - 1] == 0) {                          /* noverlapg.f:152-162 */
                for (int i = 0; i < ng; ++i) {
                    k_g[i] = k_g2[i] * a2;
                    for (int jg = 1; jg <= igas; ++jg) DK(i, jg - 1) = 0;
                    DK(i, igas) = k_g2[i];
                    DK(i, igas + 1) = dk2dT[i] * a2;
                }
                continue;
            }
            if (k_g2[ng - 1] == 0) {                          /* noverlapg.f:164-173 */
                for (int i = 0; i < ng; ++i) {
                    k_g[i] = k_g1[i];
                    DK(i, igas) = 0;
                    DK(i, igas + 1) = dk1dT[i];
                }
                continue;
            }
            for (int i = 0; i < ng; ++i)
                for (int j = 0; j < ng; ++j) {
                    weight[nloop] = delg[i] * delg[j];
                    contri[nloop] = k_g1[i] + k_g2[j] * a2;
                    for (int jg = 1; jg <= igas; ++jg)
                        grad[(size_t)(jg - 1) * nrank + nloop] = DK(i, jg - 1);
                    grad[(size_t)igas * nrank + nloop] = k_g2[j];
                    grad[(size_t)(igas + 1) * nrank + nloop] = dk1dT[i] + dk2dT[j] * a2;
                    ++nloop;
                }
        }
        int st = rankg<R>(igas + 2, delg, ng, nloop, weight.data(), contri.data(), grad.data(),
                          k_g, dkdq, pperm, psplit, pties);
        if (st) return st;
    }
    return RTB_OK;
}

/* Per-layer position in the k-table grid: get_kg.f:117-171 (NT > 0, and
 * NT < 0 with one temperature grid per pressure, TEMP2(NP, |NT|)). */
template <class R>
struct LayerK {
    int ioff[4];
    R u, v, dudt;
    R u2, dudt2;   /* NT < 0: the temperature weight at pressure cp + 1 */
};

template <class R>
void layer_prep(const orc_tables& t, const R* p, const R* tt, float press, float temp, LayerK<R>& L) {
    const int np = t.np, nt = t.nt, ng = t.ng;
    R P1 = Prec<R>::LOG((R)press);
    if (P1 < p[0]) P1 = p[0];
    if (P1 > p[np - 1]) P1 = p[np - 1];
    int cp = locate<R>(p, np, P1);
    if (cp < 1) cp = 1;
    if (cp >= np) cp = np - 1;
    L.v = (P1 - p[cp - 1]) / (p[cp] - p[cp - 1]);
    if (nt < 0) {                                   /* get_kg.f:143-169 */
        const int nx = -nt;
        R TN[RTB_MAXK];
        int ct[2];
        R u[2], du[2];
        for (int r = 0; r < 2; ++r) {
            for (int i = 0; i < nx; ++i) TN[i] = tt[(cp - 1 + r) + (size_t)np * i];
            R T1 = (R)temp;
            if (T1 < TN[0]) T1 = TN[0];
            if (T1 > TN[nx - 1]) T1 = TN[nx - 1];
            int c = locate<R>(TN, nx, T1);
            if (c < 1) c = 1;
            if (c >= nx) c = nx - 1;
            u[r] = (T1 - TN[c - 1]) / (TN[c] - TN[c - 1]);
            du[r] = (R)1.0 / (TN[c] - TN[c - 1]);
            ct[r] = c;
        }
        L.u = u[0];
        L.dudt = du[0];
        L.u2 = u[1];
        L.dudt2 = du[1];
        L.ioff[0] = (nx * ng * (cp - 1)) + (ng * (ct[0] - 1));
        L.ioff[1] = (nx * ng * cp) + (ng * (ct[1] - 1));
        L.ioff[2] = (nx * ng * cp) + (ng * ct[1]);
        L.ioff[3] = (nx * ng * (cp - 1)) + (ng * ct[0]);
        return;
    }
    L.u2 = 0;
    L.dudt2 = 0;
    const R tmax = tt[nt - 1], tmin = tt[0];
    R T1 = (R)temp;
    if (T1 < tmin) T1 = tmin;
    if (T1 > tmax) T1 = tmax;
    int ct = locate<R>(tt, nt, T1);
    if (ct < 1) ct = 1;
    if (ct >= nt) ct = nt - 1;
    L.u = (T1 - tt[ct - 1]) / (tt[ct] - tt[ct - 1]);
    L.dudt = (R)1.0 / (tt[ct] - tt[ct - 1]);
    L.ioff[0] = (nt * ng * (cp - 1)) + (ng * (ct - 1));
    L.ioff[1] = (nt * ng * cp) + (ng * (ct - 1));
    L.ioff[2] = (nt * ng * cp) + (ng * ct);
    L.ioff[3] = (nt * ng * (cp - 1)) + (ng * ct);
}

/* Table record selection of get_kg.f:189-275 for one (wavenumber, table).
 * Shared by both precisions (the choice is discrete).  Returns the 0-based
 * bin n1 and whether the wavenumber is coincident; weight2 for the
 * non-coincident branch. */
struct BinSel {
    int n1;
    bool coinc;
    float w2;
    bool zero;  /* KTEST == 0: all-zero slice (get_kg.f:228-250) */
    bool irr;   /* irregular grid: the two weights are FRACK and 1 - FRACK */
    float w1;
};

/* Irregular grid (delv <= 0, read_klist.f:266-310): the centre nearest in
 * per cent (delv < 0, snapped, coincident), or nearest at or below the
 * wavenumber (delv = 0, weighted with the next centre by FRACK). */
int select_bin_irregular(const orc_tables& t, int itab, float vwave, BinSel& b) {
    const float delv = t.delv[itab];
    if (!t.vcen || t.npoint < 1) return RTB_ERR_UNSUPPORTED;
    const int npoint = t.npoint;
    int ipo_m = 0;
    float maxdx1 = 1e10f, frack = 1.0f;
    for (int ipo = 1; ipo <= npoint; ++ipo) {
        const float xc = t.vcen[ipo - 1];
        const float dx = 100.0f * std::fabs((vwave - xc) / xc);
        if (delv == 0.0f) {
            if (dx < maxdx1 && xc <= vwave) {
                ipo_m = ipo;
                if (ipo < npoint) {
                    const float dxx = t.vcen[ipo] - xc;
                    frack = 1.0f - (vwave - xc) / dxx;
                } else {
                    frack = 1.0f;
                }
                maxdx1 = dx;
            }
        } else if (dx < maxdx1) {
            ipo_m = ipo;
            frack = 1.0f;
            maxdx1 = dx;
        }
    }
    if (ipo_m == 0) return RTB_ERR_RANGE;          /* 'Match not found' STOP */
    b.n1 = ipo_m - 1;
    b.coinc = delv < 0.0f;                         /* get_kg.f:266-279 */
    b.irr = true;
    b.w1 = frack;                                  /* get_kg.f:391-393 */
    b.w2 = 1.0f - frack;
    const int need = b.coinc ? b.n1 : b.n1 + 1;
    if (need >= t.nbin[itab] || (!b.coinc && ipo_m == npoint)) return RTB_ERR_RANGE;
    return RTB_OK;
}

int select_bin(const orc_tables& t, int itab, float vwave, BinSel& b) {
    const float vmin = t.vmin[itab], delv = t.delv[itab];
    b.irr = false;
    b.w1 = 0.0f;
    if (!(delv > 0.0f)) {
        const int r = select_bin_irregular(t, itab, vwave, b);
        if (r) return r;
        size_t off = 0;
        for (int k = 0; k < itab; ++k) off += (size_t)t.nbin[k] * t.np * std::abs(t.nt) * t.ng;
        const size_t ntab = (size_t)t.np * std::abs(t.nt) * t.ng;
        const float* s = t.data + off + (size_t)b.n1 * ntab;
        bool any = false;
        for (size_t i = 0; i < ntab; ++i) if (s[i] > 0.0f) { any = true; break; }
        b.zero = !any;
        return RTB_OK;
    }
    float eps;
    if (delv >= 0.0001f) eps = 0.02f * delv; else eps = 0.25f * delv;
    const int n1 = (int)(((double)vwave + (double)eps - (double)vmin) / (double)delv);
    const float tmp = vmin + delv * (float)n1;
    const float frac = std::fabs((float)((double)vwave - (double)tmp));
    b.n1 = n1;
    b.coinc = frac < eps;
    float w2 = (vwave - tmp) / delv;
    if (w2 > 1.0f) w2 = 1.0f;
    if (w2 < 0.0f) w2 = 0.0f;
    b.w2 = w2;
    const int need = b.coinc ? n1 : n1 + 1;
    if (n1 < 0 || need >= t.nbin[itab]) return RTB_ERR_RANGE;
    /* zero probe over the slice at n1 */
    size_t off = 0;
    for (int k = 0; k < itab; ++k) off += (size_t)t.nbin[k] * t.np * std::abs(t.nt) * t.ng;
    const size_t ntab = (size_t)t.np * std::abs(t.nt) * t.ng;
    const float* s = t.data + off + (size_t)n1 * ntab;
    bool any = false;
    for (size_t i = 0; i < ntab; ++i) if (s[i] > 0.0f) { any = true; break; }
    b.zero = !any;
    return RTB_OK;
}

const float* table_slice(const orc_tables& t, int itab, int n1) {
    size_t off = 0;
    for (int k = 0; k < itab; ++k) off += (size_t)t.nbin[k] * t.np * std::abs(t.nt) * t.ng;
    return t.data + off + (size_t)n1 * t.np * std::abs(t.nt) * t.ng;
}

/* GET_KG interpolation for one layer of one gas: get_kg.f:306-471. */
template <class R>
void get_kg_layer(const orc_tables& t, const BinSel& b, const float* tab1, const float* tab2,
                  const LayerK<R>& L, const R* delg, R* kout, R* dkout) {
    const int ng = t.ng;
    R k_g[kMaxG], dkdt[kMaxG];
    const R U = L.u, V = L.v, DUDT = L.dudt, U2 = L.u2, DUDT2 = L.dudt2;
    const int I1 = L.ioff[0], I2 = L.ioff[1], I3 = L.ioff[2], I4 = L.ioff[3];
    const bool t2 = t.nt < 0;
    /* get_kg.f:355-365 / 413-423: X and dX/dT of the four corners */
    auto interp = [&](R Y1, R Y2, R Y3, R Y4, R& X, R& DXDT) {
        const R a = (R)1.0 - V, bb = (R)1.0 - U;
        if (t2) {
            const R X1 = bb * Y1 + U * Y4;
            const R X2 = ((R)1.0 - U2) * Y2 + U2 * Y3;
            X = a * X1 + V * X2;
            DXDT = a * (-Y1 + Y4) * DUDT + V * (-Y2 + Y3) * DUDT2;
        } else {
            X = a * bb * Y1 + V * bb * Y2 + V * U * Y3 + a * U * Y4;
            DXDT = (-(a * Y1) - V * Y2 + V * Y3 + a * Y4) * DUDT;
        }
    };
    if (b.coinc) {
        R Y1 = tab1[I1], Y2 = tab1[I2], Y3 = tab1[I3], Y4 = tab1[I4];
        bool KLOG = !((Y1 <= 0) || (Y2 <= 0) || (Y3 <= 0) || (Y4 <= 0));
        for (int i = 0; i < ng; ++i) {
            Y1 = tab1[I1 + i]; Y2 = tab1[I2 + i]; Y3 = tab1[I3 + i]; Y4 = tab1[I4 + i];
            if (KLOG) {
                Y1 = Prec<R>::LOG(Y1); Y2 = Prec<R>::LOG(Y2);
                Y3 = Prec<R>::LOG(Y3); Y4 = Prec<R>::LOG(Y4);
            }
            R X, DXDT;
            interp(Y1, Y2, Y3, Y4, X, DXDT);
            if (KLOG) {
                k_g[i] = Prec<R>::EXP(X);
                dkdt[i] = Prec<R>::EXP(X) * DXDT;
            } else {
                k_g[i] = X;
                dkdt[i] = DXDT;
            }
        }
    } else {
        const R w[2] = {b.irr ? (R)b.w1 : (R)1.0f - (R)b.w2, (R)b.w2};
        R cont[2 * kMaxG], dcont[2 * kMaxG], fac[2 * kMaxG];
        int count = 0;
        for (int loop = 0; loop < 2; ++loop) {
            const float* tb = loop == 0 ? tab1 : tab2;
            for (int i = 0; i < ng; ++i) {
                const R Y1 = tb[I1 + i], Y2 = tb[I2 + i], Y3 = tb[I3 + i], Y4 = tb[I4 + i];
                R X, DXDT;
                interp(Y1, Y2, Y3, Y4, X, DXDT);
                cont[count] = X;
                dcont[count] = DXDT;
                fac[count] = delg[i] * w[loop];
                ++count;
            }
        }
        rankk<R>(delg, ng, cont, dcont, fac, count, k_g, dkdt);
    }
    for (int i = 0; i < ng; ++i) {                               /* get_kg.f:443-471 */
        kout[i] = Prec<R>::isnan_(k_g[i]) ? (R)1e-37f : k_g[i];
        dkout[i] = Prec<R>::isnan_(dkdt[i]) ? (R)1e-37f : dkdt[i];
    }
}

/* PINDEX: radtran/radtran/read_ktable.f:201-226 (clamps x1 in place). */
template <class R>
int pindex(const R* x, int nx, R& x1) {
    if (x1 > x[nx - 1]) x1 = x[nx - 1];
    if (x1 < x[0]) x1 = x[0];
    int j = 0;
    for (int i = 1; i <= nx - 1; ++i) {
        if (x1 >= x[i - 1]) j = i; else break;
    }
    return j;
}

/* CIAREAD: radtran/radtran/ciaread.f:108-198.  alpha/dalpha[9]. */
template <class R>
void ciaread(const orc_tables& t, R vv, R temp, R* alpha, R* dalpha) {
    const int NWN = RTB_CIA_NUMWN, NT = RTB_CIA_NUMT, NP = RTB_CIA_NUMPAIRS;
    R vvk1_first = 0, vvk1_last = (R)((float)(NWN - 1) * t.dnu);
    for (int i = 0; i < NP; ++i) { alpha[i] = 0; dalpha[i] = 0; }
    if (vv > vvk1_last || vv < vvk1_first) return;
    R tempk1[RTB_CIA_NUMT];
    for (int i = 0; i < NT; ++i) tempk1[i] = (R)(float)t.cia_temps[i];
    R temp1;
    if (temp > tempk1[NT - 1]) temp1 = tempk1[NT - 1]; else temp1 = temp;
    if (temp < tempk1[0]) temp1 = tempk1[0]; else temp1 = temp;     /* overwrites: ciaread.f:133-157 */
    /* vvk1(i) = (i-1)*dnu1 as REAL; pindex on that grid */
    std::vector<R> vvk1(NWN);
    for (int i = 0; i < NWN; ++i) vvk1[i] = (R)((float)i * t.dnu);
    R vvc = vv;
    const int cv = pindex<R>(vvk1.data(), NWN, vvc);
    const int ct = pindex<R>(tempk1, NT, temp1);
    for (int i = 0; i < NP; ++i) {
        const R abs11 = t.kcia[i + NP * (ct - 1) + NP * NT * (cv - 1)];
        const R abs12 = t.kcia[i + NP * (ct - 1) + NP * NT * cv];
        const R abs22 = t.kcia[i + NP * ct + NP * NT * cv];
        const R abs21 = t.kcia[i + NP * ct + NP * NT * (cv - 1)];
        const R tt = (vv - vvk1[cv - 1]) / (vvk1[cv] - vvk1[cv - 1]);
        const R u = (temp1 - tempk1[ct - 1]) / (tempk1[ct] - tempk1[ct - 1]);
        const R dudt = (R)1.0 / (tempk1[ct] - tempk1[ct - 1]);
        alpha[i] = ((R)1.0 - tt) * ((R)1.0 - u) * abs11 + tt * ((R)1.0 - u) * abs12 +
                   tt * u * abs22 + ((R)1.0 - tt) * u * abs21;
        dalpha[i] = (-((R)1.0 - tt) * abs11 - tt * abs12 + tt * abs22 + ((R)1.0 - tt) * abs21) * dudt;
    }
}

/* INTERP: radtran/rtm_util/interp.f:1-17 (the first point past xin, then
 * the segment before it) */
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

/* GET_SOLAR_WAVE: radtran/cirsrad/get_solar_wave.f:17-39 */
float get_solar_wave(const orc_tables& t, float x, float dist) {
    const float* w = t.solar_wave;
    const int n = t.solar_npt;
    float y = interp_f(w, t.solar_rad, n, x);
    if (w[0] < w[n - 1]) {
        if (x < w[0]) y = 0.0f;
        if (x > w[n - 1]) y = 0.0f;
    } else {
        if (x > w[0]) y = 0.0f;
        if (x < w[n - 1]) y = 0.0f;
    }
    if (dist > 0.0f) {
        const float PI = 3.1415927f, AU = 1.49598e13f;   /* constdef.f:11 */
        const float d = dist * AU;
        const float area = 4.0f * PI * (d * d);
        return y / area;
    }
    return y;
}

/* E3INTERP: radtran/radtran/e3interp.f:14-75 on the table held in t (1001
 * points; egrad formed as the reference forms it at its read) */
void e3interp(const orc_tables& t, double xtrans, double& e3out, double& de3out) {
    const int mtab = 1001;
    const double dtrans = 1.0f / (float)(mtab - 1);
    auto egrad = [&](int i) {   /* 1-based */
        if (i == 1) return (t.e3_e3[1] - t.e3_e3[0]) / dtrans;
        if (i == mtab) return (t.e3_e3[mtab - 1] - t.e3_e3[mtab - 2]) / dtrans;
        return 0.5 * (t.e3_e3[i] - t.e3_e3[i - 2]) / dtrans;
    };
    if (xtrans < 0 || std::isnan(xtrans)) {
        e3out = 0.;
        de3out = 0.;
        return;
    }
    int j = 1 + (int)(xtrans / dtrans);
    if (j >= mtab) j = mtab - 1;
    double f = (xtrans - t.e3_tran[j - 1]) / dtrans;
    if (f > 1.0) f = 1.0;
    e3out = (1.0 - f) * t.e3_e3[j - 1] + f * t.e3_e3[j];
    de3out = (1.0 - f) * egrad(j) + f * egrad(j + 1);
}

/* FPREAD_ALL: radtran/radtran/fpread_all.f:160-266, the table held in t:
 * every para fraction's H2-H2 and H2-He coefficient and d/dT, and the five
 * further pairs, at (vv, temp).  Returns false outside the wavenumber range,
 * where the reference computes nothing. */
template <class R>
bool fpread_all(const orc_tables& t, R vv, R temp, R* absh2, R* abshe, R* dah2dT, R* dahedT, R& deltaf, R* abs5,
                R* dabs5dT) {
    const int NWN = RTB_CIA_NUMWN, NT = RTB_CIA_NUMT, KP = t.ipara;
    std::vector<R> vvk2(NWN);
    for (int i = 0; i < NWN; ++i) vvk2[i] = (R)((float)i * t.dnu2);
    if (vv > vvk2[NWN - 1] || vv < vvk2[0]) return false;
    R tempk2[RTB_CIA_NUMT];
    for (int i = 0; i < NT; ++i) tempk2[i] = (R)t.para_temps[i];
    R temp1;
    if (temp > tempk2[NT - 1]) temp1 = tempk2[NT - 1]; else temp1 = temp;
    if (temp < tempk2[0]) temp1 = tempk2[0]; else temp1 = temp;    /* overwrites (fpread_all.f:178-195) */
    deltaf = (R)t.para_fp[1] - (R)t.para_fp[0];
    R vvc = vv;
    const int cv = pindex<R>(vvk2.data(), NWN, vvc);
    const int ct = pindex<R>(tempk2, NT, temp1);
    const R tt = (vv - vvk2[cv - 1]) / (vvk2[cv] - vvk2[cv - 1]);
    const R u = (temp1 - tempk2[ct - 1]) / (tempk2[ct] - tempk2[ct - 1]);
    const R dudt = (R)1.0 / (tempk2[ct] - tempk2[ct - 1]);
    auto at = [&](const float* k, int n, int i, int c_t, int c_v) {
        return (R)k[i + (size_t)n * ((c_t - 1) + (size_t)NT * (c_v - 1))];
    };
    for (int i = 0; i < KP; ++i) {
        const float* tabs[2] = {t.kh2h2, t.kh2he};
        R* outv[2] = {absh2, abshe};
        R* outd[2] = {dah2dT, dahedT};
        for (int q = 0; q < 2; ++q) {
            const R a11 = at(tabs[q], KP, i, ct, cv), a12 = at(tabs[q], KP, i, ct, cv + 1);
            const R a22 = at(tabs[q], KP, i, ct + 1, cv + 1), a21 = at(tabs[q], KP, i, ct + 1, cv);
            outv[q][i] = ((R)1.0 - tt) * ((R)1.0 - u) * a11 + tt * ((R)1.0 - u) * a12 + tt * u * a22 +
                         ((R)1.0 - tt) * u * a21;
            const R d = -((R)1.0 - tt) * a11 - tt * a12 + tt * a22 + ((R)1.0 - tt) * a21;
            outd[q][i] = d * dudt;
        }
    }
    for (int i = 0; i < 5; ++i) {
        const R a11 = at(t.kcia5, 5, i, ct, cv), a12 = at(t.kcia5, 5, i, ct, cv + 1);
        const R a22 = at(t.kcia5, 5, i, ct + 1, cv + 1), a21 = at(t.kcia5, 5, i, ct + 1, cv);
        abs5[i] = ((R)1.0 - tt) * ((R)1.0 - u) * a11 + tt * ((R)1.0 - u) * a12 + tt * u * a22 + ((R)1.0 - tt) * u * a21;
        dabs5dT[i] = (-((R)1.0 - tt) * a11 - tt * a12 + tt * a22 + ((R)1.0 - tt) * a21) * dudt;
    }
    return true;
}

/* NPARACON_ALL: radtran/radtran/nparacon_all.f:88-336.  dabsorb[6] is the
 * derivative with the para-H2 fraction.  Returns false outside the table. */
template <class R>
bool nparacon_all(const orc_tables& t, R v0, R p, R temp, int ngas, const int* idgas, const int* isogas,
                  const R* amount, const R* pp, R fpara, R xlen, R& absorb, int* iabs, R* dabsorb) {
    R qh2 = 0, qhe = 0, qn2 = 0, qch4 = 0, qco2 = 0;
    for (int i = 0; i < 5; ++i) { iabs[i] = 0; dabsorb[i] = 0; }
    dabsorb[5] = 0; dabsorb[6] = 0;
    for (int i = 0; i < ngas; ++i) {
        const int id = idgas[i], iso = isogas[i];
        if (id == 39 && (iso == 0 || iso == 1)) { qh2 = pp[i] / p; iabs[0] = i + 1; }
        if (id == 40) { qhe = pp[i] / p; iabs[1] = i + 1; }
        if (id == 22) { qn2 = pp[i] / p; iabs[2] = i + 1; }
        if (id == 6 && (iso == 0 || iso == 1)) { qch4 = (pp[i] / p); iabs[3] = i + 1; }
        if (id == 2) { qco2 = pp[i] / p; iabs[4] = i + 1; }
    }
    const R AMAGAT = (R)2.68675E19f;
    const R MODBOLTZA = (R)(10.0f * 1.37947E-23f / 1.013f);
    R tau;
    if (xlen == 0) {
        R XP1 = 0, height = 0;
        for (int i = 0; i < ngas; ++i)
            if (pp[i] > XP1) { height = amount[i] * MODBOLTZA * temp / pp[i]; XP1 = pp[i]; }
        const R a = p / (R)1.0, b = (R)273.15f / temp;
        tau = (a * a) * (b * b) * height;
    } else {
        const R height = xlen * (R)1e5f;
        R XP1 = -1, TOTAM = 0;
        for (int i = 0; i < ngas; ++i)
            if (pp[i] > XP1 && pp[i] > 0) { TOTAM = amount[i] * p / pp[i]; XP1 = pp[i]; }
        const R amag1 = (TOTAM / height) / AMAGAT;
        tau = height * (amag1 * amag1);
    }
    const int KP = t.ipara;
    std::vector<R> h2(KP), he(KP), dh2(KP), dhe(KP);
    R deltaf = 0, alpha[5], dalpha[5];
    if (!fpread_all<R>(t, v0, temp, h2.data(), he.data(), dh2.data(), dhe.data(), deltaf, alpha, dalpha)) return false;
    R AH2H2, AH2HE, DH2DT, DHEDT, DH2DFP, DHEDFP;
    if (fpara < 0) {
        AH2H2 = h2[KP - 1];
        AH2HE = he[KP - 1];
        DH2DT = dh2[KP - 1];
        DHEDT = dhe[KP - 1];
        DH2DFP = 0;
        DHEDFP = 0;
    } else {
        const R x1 = (R)1.0 + (fpara - (R)0.25) / deltaf;
        int j = (int)x1;
        R f = x1 - (R)j;
        if (j < 1) { j = 1; f = 0; }
        else if (j > KP - 2) { j = KP - 2; f = 1; }
        AH2H2 = ((R)1.0 - f) * h2[j - 1] + f * h2[j];
        AH2HE = ((R)1.0 - f) * he[j - 1] + f * he[j];
        DH2DT = ((R)1.0 - f) * dh2[j - 1] + f * dh2[j];
        DHEDT = ((R)1.0 - f) * dhe[j - 1] + f * dhe[j];
        DH2DFP = (h2[j] - h2[j - 1]) / deltaf;
        DHEDFP = (he[j] - he[j - 1]) / deltaf;
    }
    R sum = AH2H2 * qh2 * qh2 + AH2HE * qh2 * qhe;
    dabsorb[0] = ((R)2 * qh2 * AH2H2 + qhe * AH2HE);
    dabsorb[1] = qh2 * AH2HE;
    dabsorb[5] = (DH2DT * qh2 * qh2 + DHEDT * qh2 * qhe);
    dabsorb[6] = (DH2DFP * qh2 * qh2 + DHEDFP * qh2 * qhe);
    sum = sum + (alpha[0] * qh2 * qn2);
    dabsorb[0] = dabsorb[0] + qn2 * alpha[0];
    dabsorb[2] = dabsorb[2] + qh2 * alpha[0];
    dabsorb[5] = dabsorb[5] + qh2 * qn2 * dalpha[0];
    sum = sum + (alpha[1] * qn2 * qch4);
    dabsorb[2] = dabsorb[2] + qch4 * alpha[1];
    dabsorb[3] = dabsorb[3] + qn2 * alpha[1];
    dabsorb[5] = dabsorb[5] + qn2 * qch4 * dalpha[1];
    sum = sum + (alpha[2] * qn2 * qn2);
    dabsorb[2] = dabsorb[2] + (R)2 * qn2 * alpha[2];
    dabsorb[5] = dabsorb[5] + qn2 * qn2 * dalpha[2];
    sum = sum + (alpha[3] * qch4 * qch4);
    dabsorb[3] = dabsorb[3] + (R)2 * qch4 * alpha[3];
    dabsorb[5] = dabsorb[5] + qch4 * qch4 * dalpha[3];
    sum = sum + (alpha[4] * qh2 * qch4);
    dabsorb[0] = dabsorb[0] + qch4 * alpha[4];
    dabsorb[3] = dabsorb[3] + qh2 * alpha[4];
    dabsorb[5] = dabsorb[5] + qh2 * qch4 * dalpha[4];
    const R z = 0;   /* co2cia, n2n2cia, n2h2cia: zero below 3900 cm-1 */
    sum = sum + z * qco2 * qco2;
    dabsorb[4] = dabsorb[4] + (R)2 * qco2 * z;
    sum = sum + z * qn2 * qn2;
    dabsorb[2] = dabsorb[2] + (R)2 * qn2 * z;
    sum = sum + z * qn2 * qh2;
    dabsorb[2] = dabsorb[2] + qh2 * z;
    dabsorb[0] = dabsorb[0] + qn2 * z;
    absorb = sum * tau;
    for (int i = 0; i < 7; ++i) dabsorb[i] = dabsorb[i] * tau;
    return true;
}

/* NCIACON: radtran/radtran/nciacon.f:84-310 (the three NIR add-ons co2cia,
 * n2n2cia, n2h2cia are zero below 3900 cm-1; the caller rejects N2/CO2
 * runs above that). iabs[5] are 1-based gas numbers (0 = absent). */
template <class R>
void nciacon(const orc_tables& t, R v0, R p, R temp, int inormal, int ngas, const int* idgas,
             const int* isogas, const R* amount, const R* pp, R xlen, R& absorb, int* iabs,
             R* dabsorb) {
    R qh2 = 0, qhe = 0, qn2 = 0, qch4 = 0, qco2 = 0;
    for (int i = 0; i < 5; ++i) { iabs[i] = 0; dabsorb[i] = 0; }
    dabsorb[5] = 0; dabsorb[6] = 0;
    for (int i = 0; i < ngas; ++i) {
        const int id = idgas[i], iso = isogas[i];
        if (id == 39 && (iso == 0 || iso == 1)) { qh2 = pp[i] / p; iabs[0] = i + 1; }
        if (id == 40) { qhe = pp[i] / p; iabs[1] = i + 1; }
        if (id == 22) { qn2 = pp[i] / p; iabs[2] = i + 1; }
        if (id == 6 && (iso == 0 || iso == 1)) { qch4 = (pp[i] / p); iabs[3] = i + 1; }
        if (id == 2) { qco2 = pp[i] / p; iabs[4] = i + 1; }
    }
    const R AMAGAT = (R)2.68675E19f;
    const R MODBOLTZA = (R)(10.0f * 1.37947E-23f / 1.013f);
    R tau;
    if (xlen == 0) {
        R XP1 = 0, height = 0;
        for (int i = 0; i < ngas; ++i)
            if (pp[i] > XP1) { height = amount[i] * MODBOLTZA * temp / pp[i]; XP1 = pp[i]; }
        const R P0 = 1.0f, T0 = 273.15f;
        const R a = p / P0, b = T0 / temp;
        tau = (a * a) * (b * b) * height;
    } else {
        const R height = xlen * (R)1e5f;
        R XP1 = -1, TOTAM = 0;
        for (int i = 0; i < ngas; ++i)
            if (pp[i] > XP1 && pp[i] > 0) { TOTAM = amount[i] * p / pp[i]; XP1 = pp[i]; }
        const R amag1 = (TOTAM / height) / AMAGAT;
        tau = height * (amag1 * amag1);
    }
    R alpha[9], da[9];
    ciaread<R>(t, v0, temp, alpha, da);
    R sum = 0;
    if (inormal == 0) {
        sum = sum + (alpha[0] * qh2 * qh2) + (alpha[1] * qh2 * qhe);
        dabsorb[0] = dabsorb[0] + (R)2 * qh2 * alpha[0] + qhe * alpha[1];
        dabsorb[1] = dabsorb[1] + qh2 * alpha[1];
        dabsorb[5] = dabsorb[5] + qh2 * qh2 * da[0] + qh2 * qhe * da[1];
    } else {
        sum = sum + (alpha[2] * qh2 * qh2) + (alpha[3] * qh2 * qhe);
        dabsorb[0] = dabsorb[0] + (R)2 * qh2 * alpha[2] + qhe * alpha[3];
        dabsorb[1] = dabsorb[1] + qh2 * alpha[3];
        dabsorb[5] = dabsorb[5] + qh2 * qh2 * da[2] + qh2 * qhe * da[3];
    }
    sum = sum + (alpha[4] * qh2 * qn2);
    dabsorb[0] = dabsorb[0] + qn2 * alpha[4];
    dabsorb[2] = dabsorb[2] + qh2 * alpha[4];
    dabsorb[5] = dabsorb[5] + qh2 * qn2 * da[4];
    sum = sum + (alpha[5] * qn2 * qch4);
    dabsorb[2] = dabsorb[2] + qch4 * alpha[5];
    dabsorb[3] = dabsorb[3] + qn2 * alpha[5];
    dabsorb[5] = dabsorb[5] + qn2 * qch4 * da[5];
    sum = sum + (alpha[6] * qn2 * qn2);
    dabsorb[2] = dabsorb[2] + (R)2 * qn2 * alpha[6];
    dabsorb[5] = dabsorb[5] + qn2 * qn2 * da[6];
    sum = sum + (alpha[7] * qch4 * qch4);
    dabsorb[3] = dabsorb[3] + (R)2 * qch4 * alpha[7];
    dabsorb[5] = dabsorb[5] + qch4 * qch4 * da[7];
    sum = sum + (alpha[8] * qh2 * qch4);
    dabsorb[0] = dabsorb[0] + qch4 * alpha[8];
    dabsorb[3] = dabsorb[3] + qh2 * alpha[8];
    dabsorb[5] = dabsorb[5] + qh2 * qch4 * da[8];
    /* co2cia / n2n2cia / n2h2cia: zero below 3900 cm-1 -> adding exact zeros */
    const R z = 0;
    sum = sum + z * qco2 * qco2;
    dabsorb[4] = dabsorb[4] + (R)2 * qco2 * z;
    sum = sum + z * qn2 * qn2;
    dabsorb[2] = dabsorb[2] + (R)2 * qn2 * z;
    sum = sum + z * qn2 * qh2;
    dabsorb[2] = dabsorb[2] + qh2 * z;
    dabsorb[0] = dabsorb[0] + qn2 * z;
    absorb = sum * tau;
    for (int i = 0; i < 7; ++i) dabsorb[i] = dabsorb[i] * tau;
}

/* PLANCK_WAVE / PLANCKG_WAVE: radtran/radtran/planck_wave.f:1-42,
 * planckg_wave.f:1-40.  c1, c2 are REAL literals stored in DOUBLE
 * parameters; integer powers of the REAL y follow gfortran's expansion. */
const double kC1 = (double)1.1911e-12f, kC2 = (double)1.439f;

template <class R> R planck_wave(int ispace, R v, R T);
template <> float planck_wave<float>(int ispace, float v, float T) {
    float y;
    double a;
    if (ispace == 0) { y = v; float y2 = y * y; a = kC1 * (double)(y2 * y); }
    else { y = 1e4f / v; float y2 = y * y; float y4 = y2 * y2; a = kC1 * (double)(y4 * y) / 1e4; }
    if (y == 0.0f) return 0.0f;
    const double tmp = kC2 * (double)y / (double)T;
    const double b = std::exp(tmp) - 1.;
    return (float)(a / b);
}
template <> double planck_wave<double>(int ispace, double v, double T) {
    double y, a;
    if (ispace == 0) { y = v; a = kC1 * (y * y * y); }
    else { y = 1e4 / v; a = kC1 * (y * y * y * y * y) / 1e4; }
    if (y == 0.0) return 0.0;
    return a / std::expm1(kC2 * y / T);
}
template <class R> R planckg_wave(int ispace, R v, R T);
template <> float planckg_wave<float>(int ispace, float v, float T) {
    float y;
    double A;
    const float T2 = T * T;
    if (ispace == 0) { y = v; float y2 = y * y; A = kC1 * kC2 * (double)(y2 * y2) / (double)T2; }
    else {
        y = 1e4f / v; float y2 = y * y; float y3 = y2 * y;
        A = kC1 * kC2 * (double)(y3 * y3) * (double)1e-4f / (double)T2;
    }
    const double tmp = kC2 * (double)y / (double)T;
    const double e = std::exp(tmp);
    const double bot = (e - 1.0) * (e - 1.0);
    const double top = e * A;
    return (float)(top / bot);
}
template <> double planckg_wave<double>(int ispace, double v, double T) {
    double y, A;
    if (ispace == 0) { y = v; A = kC1 * kC2 * (y * y * y * y) / (T * T); }
    else { y = 1e4 / v; A = kC1 * kC2 * (y * y * y * y * y * y) * 1e-4 / (T * T); }
    const double tmp = kC2 * y / T;
    const double em1 = std::expm1(tmp);
    return std::exp(tmp) * A / (em1 * em1);
}

/* INVPLANCK_WAVE: radtran/radtran/invplanck_wave.f:1-30 (DOUBLE inside,
 * REAL result) */
template <class R> R invplanck_wave(int iwave, R v, R B) {
    double t;
    if (B == (R)0 || v == (R)0) t = 0.0;
    else {
        const double dv = (double)v, v2 = dv * dv, v4 = v2 * v2;   /* dble(v)**3, **5 as products */
        if (iwave == 0) t = kC2 * dv / std::log((kC1 * (v2 * dv)) / (double)B + 1.0);
        else t = kC2 * (double)1.0e4f / dv / std::log((kC1 * (double)1.0e16f) / ((double)B * (v4 * dv)) + 1.0);
    }
    return (R)t;
}

/* CALC_NLTE_T: radtran/radtran/calc_nlte_t.f:1-45.  cirsradg_wave.f:933-935
 * passes the wavenumber index as its IWAVE, so planck_wave and
 * invplanck_wave there always take their IWAVE != 0 branch */
template <class R> R calc_nlte_t(R T, R p, R v, int inlte, R k1, R A) {
    R f;
    if (inlte == 1) {
        const R kboltz = (R)1.380658e-23f;
        const R ntot = (p * (R)101325.f / (kboltz * T)) * (R)1.0e-6f;
        f = (k1 * ntot) / (A + k1 * ntot);
    } else if (inlte == 2) {
        f = p * (R)1.0e6f / ((R)1.0 + p * (R)1.0e6f);
    } else {
        return T;
    }
    const R B = planck_wave<R>(1, v, T);
    return invplanck_wave<R>(1, v, B * f);
}

/* DPEXP: radtran/radtran/dpexp.f */
template <class R>
R dpexp(R x) {
    R y = std::max(x, (R)-500.0f);
    if (y >= (R)88.7f) y = (R)88.7f;
    return (R)std::exp((double)y);
}

/* INTERPEM: radtran/cirsrad/interpem.f:1-37 */
float interpem(int nem, const float* vem, const float* em, float v, int* err) {
    if (nem <= 0) return 1.0f;
    if (v < vem[0] || v > vem[nem - 1]) { *err = RTB_ERR_RANGE; return 0.0f; }
    float x = 0.0f;
    for (int i = 0; i < nem - 1; ++i)
        if (v >= vem[i] && v < vem[i + 1]) {
            const float f = (v - vem[i]) / (vem[i + 1] - vem[i]);
            x = (1 - f) * em[i] + f * em[i + 1];
        }
    if (v == vem[nem - 1]) x = em[nem - 1];
    return x;
}

/* RAYLEIGHJ: radtran/scatter/rayleighj.f:1-35 with faniso(0) = 1
 * (radtran/scatter/rayleigha.f:55-63). */
/* RAYLEIGHV: radtran/scatter/rayleighv.f:1-12 (Venus, C / lambda^4) */
float rayleighv(float v) {
    const float C = 8.8E-28f;
    float lambda = 10000.0f / v;
    const float l2 = lambda * lambda;   /* lambda**4 as gfortran expands it */
    lambda = l2 * l2;
    return C / lambda;
}

/* RAYLEIGHA: radtran/scatter/rayleigha.f:1-38 (air at the layer's P, T) */
float rayleigha(float v, float P, float T) {
    const float c1 = 8342.12f, c2 = 2406030.0f, c3 = 15997.0f, delta = 0.035f, pi = 3.1415927f, k = 1.37971e-23f;
    float lambda = 1e4f / v;
    const float nu2 = 1.0f / (lambda * lambda);
    float m1 = c1 + c2 / (130.0f - nu2) + c3 / (38.9f - nu2);
    m1 = m1 * 1e-8f;
    const float P1 = P * 1.013e5f, T1 = T - 273.15f;
    const float xcorr = P1 * (1.0f + P1 * (61.3f - T1) * 1E-10f) / (96095.4f * (1.0f + 0.003661f * T1));
    m1 = m1 * xcorr;
    const float Ns = P1 / (k * T);
    lambda = lambda * 1e-6f;
    const float x = Ns * lambda * lambda;
    const float mm = m1 * (m1 + 2.0f);
    const float temp = 8.0f * (pi * pi * pi) * (mm * mm);
    const float faniso = (6.0f + 3.0f * delta) / (6.0f - 7.0f * delta);
    return temp * 1e4f * faniso / (3.0f * (x * x));
}

float rayleighj(float v) {
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

/* Column accessors for Fortran arrays with leading dimensions. */
struct Dims {
    int ld_lay, ld_con, ld_v, ld_param;
};

Dims dims_of(const rtb_atm& a) {
    Dims d;
    d.ld_lay = a.ld_lay > 0 ? a.ld_lay : RTB_MAXLAY;
    d.ld_con = a.ld_con > 0 ? a.ld_con : RTB_MAXCON;
    d.ld_v = a.ld_v > 0 ? a.ld_v : RTB_MAXV;
    d.ld_param = a.ld_param > 0 ? a.ld_param : (RTB_MAXGAS + 2 + RTB_MAXCON);
    return d;
}

int validate(const orc_tables& t, const rtb_atm& a, const Dims& d) {
    if (a.nlayer <= 0 || a.ngas <= 0 || a.npath <= 0 || a.nwave <= 0 || a.nv < 0 || a.npro <= 0)
        return RTB_ERR_ARG;
    if (a.nlayer > d.ld_lay || a.nlayer > RTB_MAXLAY || a.npath > RTB_MAXPAT ||
        a.ngas > RTB_MAXGAS || a.ncont > RTB_MAXCON || a.npro > RTB_MAXPRO || a.nv > d.ld_v)
        return RTB_ERR_LIMIT;
    if (t.ng > RTB_MAXG || t.np > RTB_MAXK || std::abs(t.nt) > RTB_MAXK) return RTB_ERR_LIMIT;
    if (t.ng < 2 || std::abs(t.nt) < 2) return RTB_ERR_UNSUPPORTED;
    if ((a.flagh2p == 1 && (!t.has_para || !a.hfp)) || (a.flagh2p != 0 && a.flagh2p != 1) || a.ilbl != 0 ||
        !(a.inlte == 0 || a.inlte == 1 || a.inlte == 2) || a.fwhm != 0.0f)
        return RTB_ERR_UNSUPPORTED;
    if (a.iform < 0 || a.iform > 4) return RTB_ERR_UNSUPPORTED;
    if (t.solar_npt == 1 || (t.solar_npt > 1 && (!t.solar_wave || !t.solar_rad))) return RTB_ERR_ARG;
    if (a.inlte == 1 && !(a.nlte_k1 >= 1.0e-20f && a.nlte_k1 <= 1.0e-3f)) return RTB_ERR_ARG;   /* calc_nlte_t.f:17-20 */
    if (a.ncont < 0 || (a.ncont > 0 && (!a.cont || !a.xsec_ext))) return RTB_ERR_ARG;
    if (a.iray > 3) return RTB_ERR_UNSUPPORTED;   /* rayleighls reads FRAC of gases it may not have */
    for (int k = 0; k < a.ngas; ++k) {
        if (a.idgas[k] == 91 || a.idgas[k] == 48 || a.idgas[k] == 80) return RTB_ERR_UNSUPPORTED;
        if (a.ktab[k] >= t.ntab) return RTB_ERR_ARG;
    }
    for (int ip = 0; ip < a.npath; ++ip) {
        const int m = a.imod[ip];
        if (!(m == 0 || m == 1 || m == 3 || m == 18)) return RTB_ERR_UNSUPPORTED;
        if (m == 18 && (!t.e3_tran || !t.e3_e3 || a.tsurf < 0.0f)) return RTB_ERR_UNSUPPORTED;
        if (a.nlayin[ip] > d.ld_lay || a.nlayin[ip] > 2 * RTB_MAXPAT) return RTB_ERR_LIMIT;
        if (a.nlayin[ip] < (m == 3 ? 2 : 1)) return RTB_ERR_UNSUPPORTED;
        for (int j = 0; j < a.nlayin[ip]; ++j) {
            const int l = a.layinc[j + (size_t)d.ld_lay * ip];
            if (l < 1 || l > a.nlayer) return RTB_ERR_LIMIT;
        }
    }
    bool n2co2 = false;
    for (int k = 0; k < a.ngas; ++k) if (a.idgas[k] == 22 || a.idgas[k] == 2) n2co2 = true;
    if (n2co2)
        for (int w = 0; w < a.nwave; ++w) {
            const float vv = a.ispace == 1 ? 1e4f / a.vwave[w] : a.vwave[w];
            if (vv >= 3900.0f) return RTB_ERR_UNSUPPORTED;
        }
    return RTB_OK;
}

/* Per-wavenumber work of cirsradg_wave (cirsradg_wave.f:333-1290) for the
 * IMOD 0/1/3 paths, followed by map2pro + map2xvec and packing
 * (cirsrtfg_wave.f:397-446).  All scratch is owned by the Work object. */
template <class R>
struct Work {
    std::vector<R> kout, dkout;              /* [ngas][nlayer][ng] */
    std::vector<R> taucon, utotl;
    std::vector<R> dtaucondq;                /* [nlayer][nparam] */
    std::vector<R> kl_g;                     /* [nlayer][ng] */
    std::vector<R> dkdql;                    /* [nlayer][ngas+1][ng] */
    std::vector<R> dcoutdq;                  /* [npath][ng][nlaymax][nparam] */
    std::vector<R> corkout, tempgtsurf;      /* [npath][ng] */
    std::vector<R> bb, dbdt;                 /* [npath][nlaymax] */
    std::vector<R> doutputdq;                /* [npath][nlaymax][nparam] */
    std::vector<R> doutmoddq;                /* [npath][nparam][npro] */
};

template <class R>
int one_wave(const orc_tables& t, const rtb_atm& a, const Dims& d, const std::vector<LayerK<R>>& LK,
             const std::vector<int>& isw, int iw, Work<R>& W, double* calcout, double* gradients,
             double* gradtsurf, const orc_debug* dbg) {
    const int nlayer = a.nlayer, ngas = a.ngas, ng = t.ng, ncont = a.ncont, npath = a.npath;
    const int nparam = ngas + 1 + ncont + (a.flagh2p == 1 ? 1 : 0);   /* cirsradg_wave.f:375-376 */
    const int nsw = (int)isw.size();
    const float vwave = a.vwave[iw];
    float vv = vwave;
    int err = 0;
    const float esurf = interpem(a.nem, a.vem, a.emissivity, vwave, &err);
    if (err) return err;
    if (a.ispace == 1) vv = 1e4f / vwave;
    std::vector<R> delg(ng);
    for (int i = 0; i < ng; ++i) delg[i] = (R)t.delg[i];

    /* utotl: cirsradg_wave.f:418-426 */
    for (int i = 0; i < nlayer; ++i) {
        R u = 0;
        for (int j = 0; j < ngas; ++j) u = u + (R)a.amount[i + (size_t)d.ld_lay * j];
        W.utotl[i] = u * (R)1.e-20f;
    }
    /* get_kg: cirsradg_wave.f:502-506 */
    for (int k = 0; k < ngas; ++k) {
        R* ko = &W.kout[(size_t)k * nlayer * ng];
        R* dko = &W.dkout[(size_t)k * nlayer * ng];
        const int itab = a.ktab[k];
        BinSel bs{};
        bool zero = itab < 0;
        if (!zero && t.delv[itab] > 0.0f) {   /* a wavenumber the table does not cover: no table
                                                  (read_klist.f:250-265, 341-351) */
            const float xmax = t.vmin[itab] + (float)(t.nbin[itab] - 1) * t.delv[itab];
            int i1 = 0, i2 = 0;
            findloc(a.vwave, a.nwave, t.vmin[itab], xmax, i1, i2);
            zero = i1 == 0 || i2 == 0 || iw + 1 < i1 || iw + 1 > i2;
        }
        if (!zero) {
            int st = select_bin(t, itab, vwave, bs);
            if (st) return st;
            zero = bs.zero;
        }
        if (zero) {
            std::fill(ko, ko + (size_t)nlayer * ng, (R)0);
            std::fill(dko, dko + (size_t)nlayer * ng, (R)0);
            continue;
        }
        const float* tab1 = table_slice(t, itab, bs.n1);
        const float* tab2 = bs.coinc ? nullptr : table_slice(t, itab, bs.n1 + 1);
        for (int l = 0; l < nlayer; ++l)
            get_kg_layer<R>(t, bs, tab1, tab2, LK[l], delg.data(), ko + (size_t)l * ng, dko + (size_t)l * ng);
    }
    /* :663-680: Jovian (1) or Venus (2) per wavenumber; air (3) per layer below */
    const float xray = (a.iray > 0 && a.itype != 0) ? (a.iray == 2 ? rayleighv(vv) : rayleighj(vv)) * 1E20f : 0.0f;
    std::vector<R> amo(ngas), kgn((size_t)ngas * ng), dkgn((size_t)ngas * ng), aam(ngas), ppp(ngas);
    std::vector<R> k_g(ng), dkdq((size_t)(ngas + 1) * ng);
    /* layer loop: cirsradg_wave.f:510-760 */
    for (int j = 0; j < nlayer; ++j) {
        R taucon = 0;
        R* dtc = &W.dtaucondq[(size_t)j * nparam];
        for (int k = 0; k < nparam; ++k) dtc[k] = 0;
        const R p = (R)a.press[j], tt = (R)a.temp[j];
        for (int k = 0; k < ncont; ++k) {                       /* dust :550-575 */
            const R tau = (R)a.xsec_ext[k + (size_t)ncont * iw];
            taucon = taucon + tau * (R)a.cont[k + (size_t)d.ld_con * j];
            dtc[ngas + 1 + k] = tau;
        }
        /* ngascon (:590-611): every continuum flag off -> 0.0 */
        for (int k = 0; k < ngas; ++k) taucon = taucon + (R)0;
        for (int ii = 0; ii < ngas; ++ii) {
            aam[ii] = (R)a.amount[j + (size_t)d.ld_lay * ii];
            ppp[ii] = (R)a.pp[j + (size_t)d.ld_lay * ii];
        }
        R avgcontmp = 0;
        int iabs[5];
        R dabs[7];
        if (a.flagh2p == 1) {                                    /* :634-637 */
            if (!nparacon_all<R>(t, (R)vv, p, tt, ngas, a.idgas, a.isogas, aam.data(), ppp.data(), (R)a.hfp[j],
                                 (R)a.delh[j], avgcontmp, iabs, dabs))
                return RTB_ERR_RANGE;
        } else if (t.has_cia) {
            nciacon<R>(t, (R)vv, p, tt, a.inormal, ngas, a.idgas, a.isogas, aam.data(), ppp.data(),
                       (R)a.delh[j], avgcontmp, iabs, dabs);
        } else {
            avgcontmp = 0;
            for (int i = 0; i < 5; ++i) iabs[i] = 0;
            for (int i = 0; i < 7; ++i) dabs[i] = 0;
        }
        taucon = taucon + avgcontmp;
        for (int ii = 0; ii < 5; ++ii) {
            const int k = iabs[ii];
            if (k > 0) dtc[k - 1] = dtc[k - 1] + dabs[ii] / (W.utotl[j] * (R)1.0e20f);
        }
        dtc[ngas] = dtc[ngas] + dabs[5];
        if (a.flagh2p == 1) dtc[nparam - 1] = dtc[nparam - 1] + dabs[6];   /* :659-661 */
        if (a.iray > 0 && a.itype != 0) {                        /* :663-691 */
            const float xr = a.iray == 3 ? rayleigha(vv, a.press[j], a.temp[j]) * 1E20f : xray;
            const R av = W.utotl[j] * (R)xr;
            taucon = taucon + av;
            for (int k = 0; k < ngas; ++k) dtc[k] = dtc[k] + (R)xr * (R)1.0e-20f;
        }
        W.taucon[j] = taucon;
        /* gather and overlap: :703-753 */
        for (int k = 0; k < ngas; ++k) {
            amo[k] = (R)a.amount[j + (size_t)d.ld_lay * k] * (R)1.0e-20f;
            for (int l = 0; l < ng; ++l) {
                kgn[(size_t)k * ng + l] = W.kout[((size_t)k * nlayer + j) * ng + l];
                dkgn[(size_t)k * ng + l] = W.dkout[((size_t)k * nlayer + j) * ng + l];
            }
        }
        int16_t* pp_ = nullptr;
        int16_t* ps_ = nullptr;
        int16_t* pt_ = nullptr;
        if (dbg && ngas > 1) {
            const size_t rec = ((size_t)iw * nlayer + j) * (ngas - 1);
            if (dbg->perm) pp_ = dbg->perm + rec * ng * ng;
            if (dbg->split) ps_ = dbg->split + rec * ng;
            if (dbg->ties) pt_ = dbg->ties + rec;
        }
        if (ngas == 1) {
            /* noverlapg's pass loop is empty for one gas: k_g keeps its prior
             * contents in the reference; defined here as the gas itself. */
            for (int l = 0; l < ng; ++l) {
                k_g[l] = kgn[l] * amo[0];
                dkdq[l] = kgn[l];
                dkdq[(size_t)ng + l] = dkgn[l] * amo[0];
            }
        } else {
            int st = noverlapg<R>(delg.data(), ng, ngas, amo.data(), kgn.data(), dkgn.data(), k_g.data(),
                                  dkdq.data(), pp_, ps_, pt_);
            if (st) return st;
        }
        for (int l = 0; l < ng; ++l) {
            W.kl_g[(size_t)j * ng + l] = k_g[l];
            for (int k = 0; k < ngas; ++k)
                W.dkdql[((size_t)j * (ngas + 1) + k) * ng + l] = dkdq[(size_t)k * ng + l] * (R)1.0e-20f;
            W.dkdql[((size_t)j * (ngas + 1) + ngas) * ng + l] = dkdq[(size_t)ngas * ng + l];
        }
    }

    /* g loop: cirsradg_wave.f:776-1035 */
    const int nlmax = *std::max_element(a.nlayin, a.nlayin + npath);
    std::vector<R> tautmp(nlayer), dtautmpdq((size_t)nlayer * nparam), taus(nlmax),
        dtaudq((size_t)nlmax * nparam), dtolddq((size_t)nlmax * nparam), dtrdq((size_t)nlmax * nparam);
    auto DC = [&](int ip, int ig, int j, int k) -> R& {
        return W.dcoutdq[(((size_t)ip * ng + ig) * nlmax + j) * nparam + k];
    };
    for (int ig = 0; ig < ng; ++ig) {
        for (int j = 0; j < nlayer; ++j) {
            tautmp[j] = W.taucon[j] + W.kl_g[(size_t)j * ng + ig];
            for (int k = 0; k < nparam; ++k) dtautmpdq[(size_t)j * nparam + k] = W.dtaucondq[(size_t)j * nparam + k];
            for (int k = 0; k < ngas + 1; ++k)
                dtautmpdq[(size_t)j * nparam + k] =
                    dtautmpdq[(size_t)j * nparam + k] + W.dkdql[((size_t)j * (ngas + 1) + k) * ng + ig];
        }
        for (int ip = 0; ip < npath; ++ip) {
            const int nlays = a.nlayin[ip];
            R& cork = W.corkout[(size_t)ip * ng + ig];
            cork = 0;
            W.tempgtsurf[(size_t)ip * ng + ig] = 0;
            for (int j = 0; j < nlays; ++j)
                for (int k = 0; k < nparam; ++k) DC(ip, ig, j, k) = 0;
            for (int j = 0; j < nlays; ++j) {
                const int l = a.layinc[j + (size_t)d.ld_lay * ip] - 1;
                const R sc = (R)a.scale[j + (size_t)d.ld_lay * ip];
                taus[j] = tautmp[l] * sc;
                for (int k = 0; k < nparam; ++k) dtaudq[(size_t)j * nparam + k] = dtautmpdq[(size_t)l * nparam + k] * sc;
            }
            const int im = a.imod[ip];
            if (im == 0 || im == 1) {
                for (int j = 0; j < nlays; ++j) cork = cork + taus[j];
                const R tmp = cork;
                if (im == 0) {
                    cork = dpexp<R>(-tmp);
                    R xfac = 1;   /* iform 4 with a stellar spectrum: x the star's flux (:861-867) */
                    if (t.solar_npt > 0 && a.iform == 4) xfac = (R)get_solar_wave(t, vwave, a.dist);
                    for (int j = 0; j < nlays; ++j)
                        for (int k1 = 0; k1 < nsw; ++k1) {
                            const int k = isw[k1];
                            DC(ip, ig, j, k) = -tmp * cork * dtaudq[(size_t)j * nparam + k] * xfac;
                        }
                    cork = cork * xfac;
                } else {
                    cork = (R)1. - dpexp<R>(-tmp);
                    for (int j = 0; j < nlays; ++j)
                        for (int k1 = 0; k1 < nsw; ++k1) {
                            const int k = isw[k1];
                            DC(ip, ig, j, k) = tmp * ((R)1 - cork) * dtaudq[(size_t)j * nparam + k];
                        }
                }
            } else if (im == 18) {  /* hemispherically integrated emission: :1116-1225 */
                const R PI = (R)3.1415927f;
                R xfac = 1;   /* :1136-1152 */
                if (a.iform == 1 || a.iform == 3) {
                    const R rr = ((R)a.radius1 + (R)a.radextra) * (R)1e5f;
                    xfac = xfac * (R)4. * PI * (rr * rr);
                }
                if (t.solar_npt > 0 && a.iform == 1) xfac = xfac / (R)get_solar_wave(t, vwave, -1.0f);
                if (a.iform == 3) xfac = xfac * (R)1e-18f;
                double trold = 1., e3old = 0.5;
                std::vector<R> de3olddq((size_t)nlays * nparam, 0), de3dq((size_t)nlays * nparam, 0);
                for (int j = 0; j < nlays; ++j)
                    for (int k = 0; k < nparam; ++k) {
                        dtolddq[(size_t)j * nparam + k] = 0;
                        dtrdq[(size_t)j * nparam + k] = 0;
                    }
                const R bsurf = a.tsurf > 0.0f ? planck_wave<R>(a.ispace, (R)vwave, (R)a.tsurf) : (R)0;
                const R gsurf = a.tsurf > 0.0f ? planckg_wave<R>(a.ispace, (R)vwave, (R)a.tsurf) : (R)0;
                for (int j = 0; j < nlays; ++j) {
                    if (ig == 0) {   /* calc_nlte_t at the layer's pressure (:933-935, :1156-1158) */
                        const R Tn = calc_nlte_t<R>((R)a.emtemp[j + (size_t)d.ld_lay * ip],
                                                    (R)a.press[a.layinc[j + (size_t)d.ld_lay * ip] - 1], (R)vwave,
                                                    a.inlte, (R)a.nlte_k1, (R)a.nlte_A);
                        W.bb[(size_t)ip * nlmax + j] = planck_wave<R>(a.ispace, (R)vwave, Tn);
                        W.dbdt[(size_t)ip * nlmax + j] = planckg_wave<R>(a.ispace, (R)vwave, Tn);
                    }
                    const R bbj = W.bb[(size_t)ip * nlmax + j];
                    const double tlayer = std::exp(-(double)taus[j]);
                    const double tr = trold * tlayer;
                    double e3new, e3grad;
                    e3interp(t, tr, e3new, e3grad);
                    cork = cork + xfac * (R)2.0 * PI * (R)(e3old - e3new) * bbj;
                    for (int k1 = 0; k1 < nsw; ++k1) {
                        const int k = isw[k1];
                        for (int j1 = 0; j1 <= j; ++j1) {
                            R& dtr = dtrdq[(size_t)j1 * nparam + k];
                            if (j1 < j) dtr = dtolddq[(size_t)j1 * nparam + k] * (R)tlayer;
                            else dtr = -dtaudq[(size_t)j1 * nparam + k] * (R)tr;
                            de3dq[(size_t)j1 * nparam + k] = (R)e3grad * dtr;
                            DC(ip, ig, j1, k) = DC(ip, ig, j1, k) + bbj * xfac * (R)2.0 * PI *
                                                (de3olddq[(size_t)j1 * nparam + k] - de3dq[(size_t)j1 * nparam + k]);
                        }
                        if (k == ngas)
                            DC(ip, ig, j, k) = DC(ip, ig, j, k) + xfac * (R)2.0 * PI * (R)(e3old - e3new) *
                                                                      W.dbdt[(size_t)ip * nlmax + j];
                    }
                    e3old = e3new;
                    trold = tr;
                    for (int j1 = 0; j1 <= j; ++j1)
                        for (int k1 = 0; k1 < nsw; ++k1) {
                            const int k = isw[k1];
                            dtolddq[(size_t)j1 * nparam + k] = dtrdq[(size_t)j1 * nparam + k];
                            de3olddq[(size_t)j1 * nparam + k] = de3dq[(size_t)j1 * nparam + k];
                        }
                }
                /* the surface, without its derivative (:1196-1205) */
                cork = cork + xfac * (R)2.0 * PI * (R)e3old * ((R)esurf * bsurf);
                W.tempgtsurf[(size_t)ip * ng + ig] = xfac * (R)2.0 * PI * (R)e3old * (R)esurf * gsurf;
            } else {  /* IMOD = 3: :896-1035 */
                double trold = 1., taud = 0.0;
                for (int j = 0; j < nlays; ++j)
                    for (int k = 0; k < nparam; ++k) {
                        dtolddq[(size_t)j * nparam + k] = 0;
                        dtrdq[(size_t)j * nparam + k] = 0;
                    }
                R xfac = 1.;   /* :913-929: the total flux of the planet, over the star's (iform 1), x 1e-18 (iform 3) */
                if (a.iform == 1 || a.iform == 3) {
                    const R PI = (R)3.1415927f;
                    const R rr = ((R)a.radius1 + (R)a.radextra) * (R)1e5f;
                    xfac = xfac * PI * (R)4. * PI * (rr * rr);
                }
                if (t.solar_npt > 0 && a.iform == 1) xfac = xfac / (R)get_solar_wave(t, vwave, -1.0f);
                if (a.iform == 3) xfac = xfac * (R)1e-18f;
                for (int j = 0; j < nlays; ++j) {
                    if (ig == 0) {   /* calc_nlte_t at the layer's pressure (:933-935, :1156-1158) */
                        const R Tn = calc_nlte_t<R>((R)a.emtemp[j + (size_t)d.ld_lay * ip],
                                                    (R)a.press[a.layinc[j + (size_t)d.ld_lay * ip] - 1], (R)vwave,
                                                    a.inlte, (R)a.nlte_k1, (R)a.nlte_A);
                        W.bb[(size_t)ip * nlmax + j] = planck_wave<R>(a.ispace, (R)vwave, Tn);
                        W.dbdt[(size_t)ip * nlmax + j] = planckg_wave<R>(a.ispace, (R)vwave, Tn);
                    }
                    const R bbj = W.bb[(size_t)ip * nlmax + j];
                    const double tlayer = std::exp(-(double)taus[j]);
                    taud = taud + (double)taus[j];
                    const double tr = trold * tlayer;
                    cork = cork + xfac * (R)(trold - tr) * bbj;
                    for (int k1 = 0; k1 < nsw; ++k1) {
                        const int k = isw[k1];
                        for (int j1 = 0; j1 <= j; ++j1) {
                            R& dtr = dtrdq[(size_t)j1 * nparam + k];
                            if (j1 < j) dtr = dtolddq[(size_t)j1 * nparam + k] * (R)tlayer;
                            else dtr = -dtaudq[(size_t)j1 * nparam + k] * (R)(tlayer * trold);
                            DC(ip, ig, j1, k) = DC(ip, ig, j1, k) +
                                                xfac * bbj * (dtolddq[(size_t)j1 * nparam + k] - dtr);
                        }
                        if (k == ngas)  /* temperature column ngas+1 (1-based) */
                            DC(ip, ig, j, k) = DC(ip, ig, j, k) + xfac * (R)(trold - tr) * W.dbdt[(size_t)ip * nlmax + j];
                    }
                    trold = tr;
                    for (int j1 = 0; j1 <= j; ++j1)
                        for (int k1 = 0; k1 < nsw; ++k1) {
                            const int k = isw[k1];
                            dtolddq[(size_t)j1 * nparam + k] = dtrdq[(size_t)j1 * nparam + k];
                        }
                }
                /* limb test and surface term: :991-1025 */
                const int j1 = (int)(0.5f * (float)nlays);
                const float p1 = a.press[a.layinc[(j1 - 1) + (size_t)d.ld_lay * ip] - 1];
                const float p2 = a.press[a.layinc[(nlays - 1) + (size_t)d.ld_lay * ip] - 1];
                if (p2 > p1) {
                    R radground, gradground;
                    if (a.tsurf <= 0.0f) {
                        radground = W.bb[(size_t)ip * nlmax + nlays - 1];
                        gradground = W.dbdt[(size_t)ip * nlmax + nlays - 1];
                    } else {
                        radground = (R)esurf * planck_wave<R>(a.ispace, (R)vwave, (R)a.tsurf);
                        gradground = (R)esurf * planckg_wave<R>(a.ispace, (R)vwave, (R)a.tsurf);
                    }
                    cork = cork + xfac * (R)trold * radground;
                    W.tempgtsurf[(size_t)ip * ng + ig] = xfac * (R)trold * gradground;
                    for (int j = 0; j < nlays; ++j)
                        for (int k1 = 0; k1 < nsw; ++k1) {
                            const int k = isw[k1];
                            DC(ip, ig, j, k) = DC(ip, ig, j, k) + xfac * radground * dtolddq[(size_t)j * nparam + k];
                        }
                }
            }
        }
    }
    /* g quadrature: :1240-1286 */
    std::vector<R> output(npath), gtsurf(npath);
    for (int ip = 0; ip < npath; ++ip) {
        output[ip] = 0;
        gtsurf[ip] = 0;
        for (int j = 0; j < nlmax; ++j)
            for (int k = 0; k < nparam; ++k) W.doutputdq[((size_t)ip * nlmax + j) * nparam + k] = 0;
        const int nlay1 = a.nlayin[ip];
        for (int ig = 0; ig < ng; ++ig) {
            output[ip] = output[ip] + W.corkout[(size_t)ip * ng + ig] * delg[ig];
            gtsurf[ip] = gtsurf[ip] + W.tempgtsurf[(size_t)ip * ng + ig] * delg[ig];
            for (int j = 0; j < nlay1; ++j)
                for (int k1 = 0; k1 < nsw; ++k1) {
                    const int k = isw[k1];
                    R& o = W.doutputdq[((size_t)ip * nlmax + j) * nparam + k];
                    o = o + DC(ip, ig, j, k) * delg[ig];
                }
        }
    }
    /* map2pro: radtran/cirsradg/map2pro.f:49-82 */
    const int npro = a.npro;
    for (int ip = 0; ip < npath; ++ip)
        for (int k = 0; k < nparam; ++k)
            for (int jj = 0; jj < npro; ++jj) {
                R s = 0;
                const int nlay1 = a.nlayin[ip];
                for (int j = 0; j < nlay1; ++j) {
                    const int lay = a.layinc[j + (size_t)d.ld_lay * ip] - 1;
                    const R dq = W.doutputdq[((size_t)ip * nlmax + j) * nparam + k];
                    const float* M;
                    if (k < ngas) M = a.dam;
                    else if (k == ngas) M = a.dte;
                    else if (k < ngas + 1 + ncont) M = a.dco;
                    else M = a.dfp;                                   /* para-H2 fraction */
                    if (!M) continue;
                    s = s + dq * (R)M[lay + (size_t)d.ld_lay * jj];
                }
                W.doutmoddq[((size_t)ip * nparam + k) * npro + jj] = s;
            }
    /* map2xvec: radtran/cirsradg/map2xvec.f:41-55; packing cirsrtfg_wave.f:425-446 */
    const int nwave = a.nwave, nv = a.nv;
    for (int ip = 0; ip < npath; ++ip) {
        calcout[(size_t)nwave * ip + iw] = (double)output[ip];
        if (gradtsurf) gradtsurf[(size_t)nwave * ip + iw] = (double)gtsurf[ip];
        for (int iv = 0; iv < nv; ++iv) {
            R s = 0;
            for (int ipar = 0; ipar < nparam; ++ipar)
                for (int ipro = 0; ipro < npro; ++ipro)
                    s = s + W.doutmoddq[((size_t)ip * nparam + ipar) * npro + ipro] *
                                (R)a.xmap[iv + (size_t)d.ld_v * (ipar + (size_t)d.ld_param * ipro)];
            gradients[(size_t)nwave * nv * ip + (size_t)nwave * iv + iw] = (double)s;
        }
    }
    return RTB_OK;
}

template <class R>
int run(const orc_tables& t, const rtb_atm& a, double* calcout, double* gradients, double* gradtsurf,
        const orc_debug* dbg, int nthreads) {
    const Dims d = dims_of(a);
    int st = validate(t, a, d);
    if (st) return st;
    const int nparam = a.ngas + 1 + a.ncont + (a.flagh2p == 1 ? 1 : 0);
    /* nsw / isw: cirsrtfg_wave.f:301-313 */
    std::vector<int> isw;
    for (int ip = 0; ip < nparam; ++ip) {
        bool on = false;
        for (int iv = 0; iv < a.nv && !on; ++iv)
            for (int ipro = 0; ipro < a.npro; ++ipro)
                if (a.xmap[iv + (size_t)d.ld_v * (ip + (size_t)d.ld_param * ipro)] != 0.0f) { on = true; break; }
        if (on) isw.push_back(ip);
    }
    const size_t ntk = t.nt < 0 ? (size_t)t.np * -t.nt : (size_t)t.nt;   /* TEMP2(NP, |NT|) or TEMP(NT) */
    std::vector<R> p(t.np), tt(ntk);
    for (int i = 0; i < t.np; ++i) p[i] = (R)t.lnp[i];
    for (size_t i = 0; i < ntk; ++i) tt[i] = (R)t.tk[i];
    std::vector<LayerK<R>> LK(a.nlayer);
    for (int l = 0; l < a.nlayer; ++l) layer_prep<R>(t, p.data(), tt.data(), a.press[l], a.temp[l], LK[l]);

    auto make_work = [&](Work<R>& W) {
        const int ng = t.ng, nl = a.nlayer, npath = a.npath;
        const int nlmax = *std::max_element(a.nlayin, a.nlayin + npath);
        W.kout.resize((size_t)a.ngas * nl * ng);
        W.dkout.resize((size_t)a.ngas * nl * ng);
        W.taucon.resize(nl);
        W.utotl.resize(nl);
        W.dtaucondq.resize((size_t)nl * nparam);
        W.kl_g.resize((size_t)nl * ng);
        W.dkdql.resize((size_t)nl * (a.ngas + 1) * ng);
        W.dcoutdq.resize((size_t)npath * ng * nlmax * nparam);
        W.corkout.resize((size_t)npath * ng);
        W.tempgtsurf.resize((size_t)npath * ng);
        W.bb.resize((size_t)npath * nlmax);
        W.dbdt.resize((size_t)npath * nlmax);
        W.doutputdq.resize((size_t)npath * nlmax * nparam);
        W.doutmoddq.resize((size_t)npath * nparam * a.npro);
    };
    if (nthreads <= 1) {
        Work<R> W;
        make_work(W);
        for (int iw = 0; iw < a.nwave; ++iw) {
            st = one_wave<R>(t, a, d, LK, isw, iw, W, calcout, gradients, gradtsurf, dbg);
            if (st) return st;
        }
        return RTB_OK;
    }
    std::vector<int> stat(nthreads, RTB_OK);
    std::vector<std::thread> th;
    for (int tid = 0; tid < nthreads; ++tid)
        th.emplace_back([&, tid]() {
            Work<R> W;
            make_work(W);
            for (int iw = tid; iw < a.nwave; iw += nthreads) {
                // debug records are per (wavenumber, layer, pass): the threads write disjoint ones
                int s = one_wave<R>(t, a, d, LK, isw, iw, W, calcout, gradients, gradtsurf, dbg);
                if (s) { stat[tid] = s; return; }
            }
        });
    for (auto& x : th) x.join();
    for (int s : stat) if (s) return s;
    return RTB_OK;
}

}  // namespace

extern "C" {

int orc_cirsrtfg_wave(const orc_tables* tab, const rtb_atm* atm, int precision, double* calcout,
                      double* gradients, double* gradtsurf, const orc_debug* dbg) {
    if (!tab || !atm || !calcout || !gradients) return RTB_ERR_ARG;
    if (precision == ORC_MIXED) return run<float>(*tab, *atm, calcout, gradients, gradtsurf, dbg, 1);
    return run<double>(*tab, *atm, calcout, gradients, gradtsurf, nullptr, 1);
}

int orc_cirsrtfg_wave_mt(const orc_tables* tab, const rtb_atm* atm, int precision, double* calcout,
                         double* gradients, double* gradtsurf, int nthreads, const orc_debug* dbg) {
    if (!tab || !atm || !calcout || !gradients) return RTB_ERR_ARG;
    if (precision == ORC_MIXED) return run<float>(*tab, *atm, calcout, gradients, gradtsurf, dbg, nthreads);
    return run<double>(*tab, *atm, calcout, gradients, gradtsurf, nullptr, nthreads);
}

float orc_det_expf_c(float x) { return orc_det_expf(x); }

void orc_set_sort_mode(int mode) { g_sort_mode = mode; }

int orc_locate(const float* xx, int n, float x) { return locate<float>(xx, n, x); }

void orc_sort2g(int n, float* ra, int* ib) {
    std::vector<int> ico(n);
    for (int i = 0; i < n; ++i) ico[i] = i + 1;
    sort2g<float>(n, ra, ico.data());
    for (int i = 0; i < n; ++i) ib[i] = ico[i] - 1;
}

int orc_rankg(int nparam, const float* gw, int ng, int nloop, const float* weight, const float* cont,
              const float* grad, float* k_g, float* dkdq, int16_t* perm, int16_t* split) {
    std::vector<float> w(weight, weight + nloop), c(cont, cont + nloop), g(grad, grad + (size_t)nparam * nloop);
    return rankg<float>(nparam, gw, ng, nloop, w.data(), c.data(), g.data(), k_g, dkdq, perm, split);
}

float orc_planck_wave(int ispace, float v, float t) { return planck_wave<float>(ispace, v, t); }
float orc_planckg_wave(int ispace, float v, float t) { return planckg_wave<float>(ispace, v, t); }

}  // extern "C"
