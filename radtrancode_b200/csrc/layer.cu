// layer.cu -- atmospheric layering on the device: LAYERG
// (radtran/path/layerg.f:146-458) and the nadir thermal path of ATMG
// (radtran/path/atmg.f:250-373, 509-560), the set-up subpathg runs before
// every forward call of a retrieval (the .prf -> layers step).
//
// One warp (block) per layer.  For a Curtis-Godson layer the lanes first
// evaluate the 101 Simpson points side by side into shared memory (the
// bracket search and every interpolation); then each lane owns one
// accumulator -- lane 0 the layer totals (TOTAM, TEMP, PRESS) and the
// gradient rows DTE, DAM, DCO, the next lanes the amount and partial
// pressure of one gas each, the rest one dust type each -- and sums it over
// the points in the reference's order, so every sum rounds as the
// reference's does; the REAL
// arithmetic is written with explicitly rounded intrinsics (no contraction
// into FMA) so that it rounds as the reference's does.  The few
// transcendental scalars of the set-up (SIN/COS of the two angles, ASIN of
// IPZEN 1, ALOG/EXP of the equal-log-pressure grid) are evaluated once on
// the host with the C library, as the reference's build evaluates them: the
// geometry takes differences of nearly equal squares in REAL
// (sqrt((R + h)^2 - sin^2 a Z^2) at R ~ 7e4 km), where one ulp of SIN moves
// a scale factor by 1e-3.  Everything the device computes is then IEEE-exact
// arithmetic in the reference's order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"

namespace rtb {

namespace {

constexpr int kNint = 101;                              // layerg.f:44

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

// first point beyond XIN in the table's direction (N if none, 2 if the
// first): the search of VERINT / VERINTG
__device__ int above_dev(const float* X, int N, float XIN) {
    int I = N;
    if (X[0] < X[N - 1]) {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] > XIN) { I = k; break; }
    } else {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] < XIN) { I = k; break; }
    }
    return I == 1 ? 2 : I;
}

// the same bracket on a non-decreasing grid with x[0] < x[N-1], by bisection:
// the first point above XIN is the upper bound
__device__ int above_sorted(const float* X, int N, float XIN) {
    int lo = 0, hi = N;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (X[mid] > XIN) hi = mid; else lo = mid + 1;
    }
    int I = lo + 1;
    if (I > N) I = N;
    return I == 1 ? 2 : I;
}

// VERINT (radtran/path/verint.f:29-46) at a known bracket I
__device__ float verint_at(const float* X, const float* Y, int I, float XIN) {
    float y = fa(Y[I - 2], fd(fm(fs(Y[I - 1], Y[I - 2]), fs(XIN, X[I - 2])), fs(X[I - 1], X[I - 2])));
    if (X[I - 2] == X[I - 1]) y = Y[I - 1];
    if (isnan(y)) y = Y[I - 1];
    return y;
}

__device__ float verint_dev(const float* X, const float* Y, int N, float XIN) {
    return verint_at(X, Y, above_dev(X, N, XIN), XIN);
}

// VERINTG (radtran/path/verintg.f) at a known bracket I: F and the value
__device__ float verintg_f(const float* X, int I, float XIN) {
    return fd(fs(XIN, X[I - 2]), fs(X[I - 1], X[I - 2]));
}
__device__ float verintg_y(const float* Y, int I, float F) {
    return fa(fm(fs(1.0f, F), Y[I - 2]), fm(F, Y[I - 1]));
}

struct LayGeom {
    float layht, sin2a, cosa, z0, pbot, lnpbot, smax;
};

struct LayArgs {
    int npro, nvmr, ndust, nlay, laytyp, layint, botlay, surface;
    int hsorted;                                   // h ascending: the height bracket by bisection
    const float *h, *p, *t, *vmr, *dust;          // vmr [nvmr][npro], dust [ndust][npro]
    const float* bases_h;                          // [nlay] layer base heights (layerg.f:164-224, on the host)
    float molwt, radius;
    LayGeom g;
    float sin2, cosz, zpath;                       // the path's geometry (atmg.f:290-292)
    // outputs, compact: [nlay] scalars, amount/pp [nvmr][nlay], cont [nlay][ndust], dte/dam/dco [npro][nlay]
    float *baseh, *delh, *basep, *baset, *press, *temp, *totam, *laysf;
    float *amount, *pp, *cont, *dte, *dam, *dco;
    int* layinc;
    float *scale, *emtemp;
    int* status;
};

// distance along a path from its start to height b (atmg.f:357-362 / layerg.f:236-240)
__device__ float path_s(float radius, float b, float sin2, float z, float cosz) {
    float stmp = fs(fm(fa(radius, b), fa(radius, b)), fm(sin2, fm(z, z)));
    if (stmp < 0.0f) stmp = 0.0f;
    return fs(__fsqrt_rn(stmp), fm(z, cosz));
}

// shared memory of one layer's Curtis-Godson pass: the 101 points' bracket,
// P, T, DUDS and F, every gas's and dust's value at them, and the layer's
// three gradient rows
constexpr int kPointArrays = 8;   // per point: bracket, DUDS*W, T*DUDS*W, P*DUDS*W, the two DTE/DAM and DCO terms

size_t layer_smem_bytes(int nvmr, int ndust, int npro) {
    const int nq = 1 + nvmr + ndust;
    return (size_t)(kPointArrays + 2 * nvmr + ndust) * kNint * 4 + (size_t)3 * npro * 4 + (size_t)(2 + nq) * npro * 4;
}

// the Curtis-Godson layer (layerg.f:315-422) in three phases: the lanes
// evaluate the 101 points side by side (bracket search and interpolations,
// the costly part); then each lane sums its own quantity over the points in
// the reference's order, reading them from shared memory; then the lanes
// normalise the gradient rows together
__device__ void curtis_godson(const LayArgs& A, int i, float S0, float S1, float laysf, float* sm, float& PRESS_o,
                              float& TEMP_o, float& TOTAM_o, bool& bad) {
    const int lane = threadIdx.x, NPRO = A.npro, NLAY = A.nlay, NV = A.nvmr, ND = A.ndust;
    const int nq = 1 + NV + ND;
    const LayGeom& g = A.g;
    int* pI = (int*)sm;
    float* dw = sm + kNint;                 // DUDS*W(K)
    float* tw = dw + kNint;                 // TNOW*DUDS*W(K)
    float* pw = tw + kNint;                 // PNOW*DUDS*W(K)
    float* a0 = pw + kNint;                 // (1-F)*DUDS*W(K), F*DUDS*W(K): DTE and DAM
    float* a1 = a0 + kNint;
    float* c0 = a1 + kNint;                 // the same times XMOLWT / AVOGAD: DCO
    float* c1 = c0 + kNint;
    float* gw = c1 + kNint;                 // per gas VMR1*DUDS*W(K) [NV][kNint], VMR1*PNOW*DUDS*W(K) [NV][kNint]
    float* gw2 = gw + (size_t)NV * kNint;
    float* dwc = gw2 + (size_t)NV * kNint;  // per dust DNOW*(XMOLWT/AVOGAD)*DUDS*W(K) [ND][kNint]
    float* rows = dwc + (size_t)ND * kNint; // dte, dam, dco [NPRO] each
    float* prof = rows + (size_t)3 * NPRO;  // h, p, t, every gas, every dust [NPRO] each
    for (int k = lane; k < (2 + nq) * NPRO; k += 32) prof[k] = A.h[k];
    for (int jj = lane; jj < 3 * NPRO; jj += 32) rows[jj] = 0.0f;
    __syncwarp();
    const float* H = prof;
    const float* Pp = prof + NPRO;
    const float* Tp = prof + 2 * NPRO;
    const float* Yp = prof + 3 * NPRO;
    const float modboltz = 1.013E4f / 1.37947E-23f;  // constdef.f:8-9
    const float mw_av = fd(A.molwt, 6.022045E23f);   // XMOLWT / AVOGAD
    const float DELS = fd(fs(S1, S0), (float)(kNint - 1));
    // every point's terms, side by side (layerg.f:335-400 less the sums)
    for (int K = lane + 1; K <= kNint; K += 32) {
        const float S = fa(S0, fm((float)(K - 1), DELS));
        const float u = fa(S, fm(g.z0, g.cosa));
        const float HEIGHT = fs(__fsqrt_rn(fa(fm(u, u), fm(g.sin2a, fm(g.z0, g.z0)))), A.radius);
        const int I = A.hsorted ? above_sorted(H, NPRO, HEIGHT) : above_dev(H, NPRO, HEIGHT);
        const float PNOW = verint_at(H, Pp, I, HEIGHT);
        const float TNOW = verint_at(H, Tp, I, HEIGHT);
        const float DUDS = fd(fm(modboltz, PNOW), TNOW);
        const float F = verintg_f(H, I, HEIGHT);
        const float WK = (K == 1 || K == kNint) ? 1.0f : ((K & 1) == 0 ? 4.0f : 2.0f);
        const int k = K - 1;
        pI[k] = I;
        dw[k] = fm(DUDS, WK);
        tw[k] = fm(fm(TNOW, DUDS), WK);
        pw[k] = fm(fm(PNOW, DUDS), WK);
        const float b0 = fm(fm(fs(1.0f, F), DUDS), WK), b1 = fm(fm(F, DUDS), WK);
        a0[k] = b0;
        a1[k] = b1;
        c0[k] = fd(fm(b0, A.molwt), 6.022045E23f);
        c1[k] = fd(fm(b1, A.molwt), 6.022045E23f);
        for (int q = 0; q < NV; ++q) {
            const float v = verint_at(H, Yp + (size_t)q * NPRO, I, HEIGHT);
            gw[(size_t)q * kNint + k] = fm(fm(v, DUDS), WK);
            gw2[(size_t)q * kNint + k] = fm(fm(fm(v, PNOW), DUDS), WK);
        }
        for (int q = 0; q < ND; ++q) {
            const float d = verint_at(H, Yp + (size_t)(NV + q) * NPRO, I, HEIGHT);
            dwc[(size_t)q * kNint + k] = fm(fm(fm(d, mw_av), DUDS), WK);
        }
    }
    __syncwarp();
    // the sums, each on one lane in the reference's order; TOTAM on every lane
    float TOTAM = 0.0f;
    for (int k = 0; k < kNint; ++k) TOTAM = fa(TOTAM, dw[k]);
    float* dte = rows;
    float* dam = rows + NPRO;
    float* dco = rows + 2 * NPRO;
    for (int q = lane; q < nq; q += 32) {
        if (q == 0) {
            float TEMP = 0.0f, PRESS = 0.0f;
            for (int k = 0; k < kNint; ++k) {
                const int JJ = pI[k] - 1;
                TEMP = fa(TEMP, tw[k]);
                dte[JJ - 1] = fa(dte[JJ - 1], a0[k]);
                dte[JJ] = fa(dte[JJ], a1[k]);
                PRESS = fa(PRESS, pw[k]);
                dco[JJ - 1] = fa(dco[JJ - 1], c0[k]);
                dco[JJ] = fa(dco[JJ], c1[k]);
                dam[JJ - 1] = fa(dam[JJ - 1], a0[k]);
                dam[JJ] = fa(dam[JJ], a1[k]);
            }
            // normalisation (layerg.f:403-422) and the vertical path (:430-447)
            TEMP_o = fd(TEMP, TOTAM);
            PRESS_o = fd(PRESS, TOTAM);
            TOTAM_o = fd(fd(fm(TOTAM, DELS), 3.0f), laysf);
            bad = bad || PRESS_o < 0.0f || TEMP_o < 0.0f || TOTAM_o < 0.0f;
        } else if (q - 1 < NV) {
            const int gas = q - 1;
            float ACC = 0.0f, ACC2 = 0.0f;
            for (int k = 0; k < kNint; ++k) {
                ACC = fa(ACC, gw[(size_t)gas * kNint + k]);
                ACC2 = fa(ACC2, gw2[(size_t)gas * kNint + k]);
            }
            const float amount = fd(fd(fm(ACC, DELS), 3.0f), laysf);
            const float pp = fd(ACC2, TOTAM);
            A.amount[(size_t)gas * NLAY + i] = amount;
            A.pp[(size_t)gas * NLAY + i] = pp;
            bad = bad || amount < 0.0f || pp < 0.0f;
        } else {
            const int dst = q - 1 - NV;
            float ACC = 0.0f;
            for (int k = 0; k < kNint; ++k) ACC = fa(ACC, dwc[(size_t)dst * kNint + k]);
            const float cont = fd(fd(fm(ACC, DELS), 3.0f), laysf);
            A.cont[(size_t)i * ND + dst] = cont;
            bad = bad || cont < 0.0f;
        }
    }
    __syncwarp();
    for (int jj = lane; jj < NPRO; jj += 32) {
        A.dte[(size_t)jj * NLAY + i] = fd(dte[jj], TOTAM);
        A.dam[(size_t)jj * NLAY + i] = fd(fd(fm(dam[jj], DELS), 3.0f), laysf);
        A.dco[(size_t)jj * NLAY + i] = fd(fd(fm(dco[jj], DELS), 3.0f), laysf);
    }
}

__global__ void __launch_bounds__(32) layerg_kernel(LayArgs A) {
    extern __shared__ __align__(16) float lsm[];
    const int lane = threadIdx.x;
    const int L = blockIdx.x + 1;   // 1-based layer
    if (L > A.nlay) return;
    const int i = L - 1, NPRO = A.npro, NLAY = A.nlay;
    const float* H = A.h;
    const float* P = A.p;
    const float* T = A.t;
    const LayGeom& g = A.g;
    const float radius = A.radius;
    const float bh = A.bases_h[L - 1];
    const float bh1 = L < NLAY ? A.bases_h[L] : 0.0f;
    const float htop = H[NPRO - 1];
    const float S0 = path_s(radius, bh, g.sin2a, g.z0, g.cosa);
    const float S1 = L < NLAY ? path_s(radius, bh1, g.sin2a, g.z0, g.cosa) : g.smax;
    const float laysf = fd(fs(S1, S0), L < NLAY ? fs(bh1, bh) : fs(htop, bh));
    bool bad = false;
    float temp_layer = 0.0f;
    if (A.layint == 1) {
        float PRESS = 0.0f, TEMP = 0.0f, TOTAM = 0.0f;
        curtis_godson(A, i, S0, S1, laysf, lsm, PRESS, TEMP, TOTAM, bad);
        if (lane == 0) {
            A.press[i] = PRESS;
            A.temp[i] = TEMP;
            A.totam[i] = TOTAM;
            temp_layer = TEMP;
        }
    } else {
        // layer-centre values (layerg.f:264-313): one point, every lane one quantity
        const int nq = 1 + A.nvmr + A.ndust;
        const float modboltz = 1.013E4f / 1.37947E-23f;  // constdef.f:8-9
        for (int jj = lane; jj < NPRO; jj += 32) {
            A.dte[(size_t)jj * NLAY + i] = 0.0f;
            A.dam[(size_t)jj * NLAY + i] = 0.0f;
            A.dco[(size_t)jj * NLAY + i] = 0.0f;
        }
        __syncwarp();
        const float S = fm(0.5f, fa(S0, S1));
        const float u = fa(S, fm(g.z0, g.cosa));
        const float HEIGHT = fs(__fsqrt_rn(fa(fm(u, u), fm(g.sin2a, fm(g.z0, g.z0)))), radius);
        const int I = A.hsorted ? above_sorted(H, NPRO, HEIGHT) : above_dev(H, NPRO, HEIGHT);
        const float F = verintg_f(H, I, HEIGHT);
        const float PRESS = verint_at(H, P, I, HEIGHT);
        const float TEMP = verintg_y(T, I, F);
        const float TOTAM = fm(fd(fm(modboltz, PRESS), TEMP), fs(S1, S0));
        for (int q = lane; q < nq; q += 32) {
            const int gas = q - 1, dst = q - 1 - A.nvmr;
            if (q == 0) {
                const int JJ = I - 1;
                float* dte = A.dte + i;
                float* dam = A.dam + i;
                float* dco = A.dco + i;
                dte[(size_t)(JJ - 1) * NLAY] = fs(1.0f, F);
                dte[(size_t)JJ * NLAY] = F;
                // DCO(I,JJ) = (1-F) * TOTAM * XMOLWT / AVOGAD, likewise F; then / LAYSF
                dco[(size_t)(JJ - 1) * NLAY] = fd(fd(fm(fm(fs(1.0f, F), TOTAM), A.molwt), 6.022045E23f), laysf);
                dco[(size_t)JJ * NLAY] = fd(fd(fm(fm(F, TOTAM), A.molwt), 6.022045E23f), laysf);
                dam[(size_t)(JJ - 1) * NLAY] = fd(fm(fs(1.0f, F), TOTAM), laysf);
                dam[(size_t)JJ * NLAY] = fd(fm(F, TOTAM), laysf);
                const float tot = fd(TOTAM, laysf);
                A.press[i] = PRESS;
                A.temp[i] = TEMP;
                A.totam[i] = tot;
                temp_layer = TEMP;
                bad = bad || PRESS < 0.0f || TEMP < 0.0f || tot < 0.0f;
            } else if (gas < A.nvmr) {
                const float v = verintg_y(A.vmr + (size_t)gas * NPRO, I, F);
                const float amount = fd(fm(v, TOTAM), laysf);
                const float pp = fm(v, PRESS);
                A.amount[(size_t)gas * NLAY + i] = amount;
                A.pp[(size_t)gas * NLAY + i] = pp;
                bad = bad || amount < 0.0f || pp < 0.0f;
            } else {
                const float v = verintg_y(A.dust + (size_t)dst * NPRO, I, F);
                const float cont = fd(fd(fm(fm(v, TOTAM), A.molwt), 6.022045E23f), laysf);
                A.cont[(size_t)i * A.ndust + dst] = cont;
                bad = bad || cont < 0.0f;
            }
        }
    }
    if (lane == 0) {
        A.laysf[i] = laysf;
        A.baseh[i] = bh;
        A.delh[i] = L < NLAY ? fs(bh1, bh) : fs(htop, bh);
        const int Ib = A.hsorted ? above_sorted(H, NPRO, bh) : above_dev(H, NPRO, bh);
        A.basep[i] = verint_at(H, P, Ib, bh);
        A.baset[i] = verint_at(H, T, Ib, bh);
    }
    if (bad) atomicOr(A.status, 1);
    // the path entry of this layer (atmg.f:328-373): position I holds layer LOC
    if (lane == 0) {
        const int I = A.surface ? L : NLAY - L + 1;
        const int nuse = NLAY - A.botlay + 1;
        if (I <= nuse) {
            const int LOC = L;
            const float s0 = path_s(radius, bh, A.sin2, A.zpath, A.cosz);
            float sf;
            if (LOC == NLAY) {
                const float s1 = path_s(radius, htop, A.sin2, A.zpath, A.cosz);
                sf = fd(fs(s1, s0), fs(htop, bh));
            } else {
                const float s1 = path_s(radius, bh1, A.sin2, A.zpath, A.cosz);
                sf = fd(fs(s1, s0), fs(bh1, bh));
            }
            A.layinc[I - 1] = LOC;
            A.scale[I - 1] = sf;
            A.emtemp[I - 1] = temp_layer;
        }
    }
}

// VERINT on the host, for the set-up scalars below (same arithmetic as the device's)
float verint_host(const float* X, const float* Y, int N, float XIN) {
    int I = N;
    if (X[0] < X[N - 1]) {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] > XIN) { I = k; break; }
    } else {
        for (int k = 1; k <= N; ++k)
            if (X[k - 1] < XIN) { I = k; break; }
    }
    if (I == 1) I = 2;
    float y = Y[I - 2] + (Y[I - 1] - Y[I - 2]) * (XIN - X[I - 2]) / (X[I - 1] - X[I - 2]);
    if (X[I - 2] == X[I - 1]) y = Y[I - 1];
    if (std::isnan(y)) y = Y[I - 1];
    return y;
}

size_t al16(size_t n) { return (n + 15) & ~(size_t)15; }

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" int rtb_layerg(rtb_context* c, const rtb_profile* pr, const rtb_layer_opts* o, rtb_layers* out) {
    if (!c) return RTB_ERR_ARG;
    if (!pr || !o || !out) return fail(c, RTB_ERR_ARG, "layerg: NULL argument");
    const int npro = pr->npro, nvmr = pr->nvmr, ndust = pr->ndust, nlay = o->nlay;
    if (npro < 2 || npro > RTB_MAXPRO || nvmr < 0 || nvmr > RTB_MAXGAS || ndust < 0 || ndust > RTB_MAXCON)
        return fail(c, RTB_ERR_LIMIT, "layerg: npro %d, nvmr %d, ndust %d outside 2..%d, 0..%d, 0..%d", npro, nvmr,
                    ndust, RTB_MAXPRO, RTB_MAXGAS, RTB_MAXCON);
    if (nlay < 1 || nlay > RTB_MAXLAY) return fail(c, RTB_ERR_LIMIT, "layerg: NLAY > MAXLAY (layerg.f:128-134)");
    if (!pr->h || !pr->p || !pr->t || (nvmr > 0 && !pr->vmr) || (ndust > 0 && !pr->dust))
        return fail(c, RTB_ERR_ARG, "layerg: profile arrays missing");
    if (o->laytyp < 0 || o->laytyp > 5) return fail(c, RTB_ERR_UNSUPPORTED, "layerg: LAYTYP %d", o->laytyp);
    if ((o->laytyp == 4 || o->laytyp == 5) && !o->base) return fail(c, RTB_ERR_ARG, "layerg: LAYTYP 4/5 need base");
    if (o->layint != 0 && o->layint != 1) return fail(c, RTB_ERR_UNSUPPORTED, "layerg: LAYINT %d", o->layint);
    if (o->botlay < 1 || o->botlay > nlay) return fail(c, RTB_ERR_ARG, "atmg: botlay %d outside 1..%d", o->botlay, nlay);
    if (o->ipzen != 0 && o->ipzen != 1)
        return fail(c, RTB_ERR_UNSUPPORTED, "atmg: ipzen %d (near-limb paths) not supported", o->ipzen);
    const int ldp = pr->ld_pro > 0 ? pr->ld_pro : npro, ldc = pr->ld_con > 0 ? pr->ld_con : ndust;
    const int LDL = out->ld_lay > 0 ? out->ld_lay : nlay, LDC = out->ld_con > 0 ? out->ld_con : ndust;
    if (ldp < npro || (ndust > 0 && ldc < ndust) || LDL < nlay || (ndust > 0 && LDC < ndust))
        return fail(c, RTB_ERR_ARG, "layerg: leading dimension below the size");
    // compact inputs: h, p, t, vmr [nvmr][npro], dust [ndust][npro], base
    std::vector<float> in;
    in.insert(in.end(), pr->h, pr->h + npro);
    in.insert(in.end(), pr->p, pr->p + npro);
    in.insert(in.end(), pr->t, pr->t + npro);
    for (int g = 0; g < nvmr; ++g) in.insert(in.end(), pr->vmr + (size_t)ldp * g, pr->vmr + (size_t)ldp * g + npro);
    for (int d = 0; d < ndust; ++d)
        for (int m = 0; m < npro; ++m) in.push_back(pr->dust[d + (size_t)ldc * m]);
    // the set-up scalars (layerg.f:146-161), on the host (see the file header)
    const float* H = pr->h;
    const float* P = pr->p;
    const float dtr = 3.1415926f / 180.0f, radius = pr->radius, htop = H[npro - 1];
    LayGeom g;
    g.layht = o->layht < H[0] ? H[0] : o->layht;    // layerg.f:95-103
    const float sa = std::sin(dtr * o->layang);
    g.sin2a = sa * sa;
    g.cosa = std::cos(dtr * o->layang);
    g.z0 = radius + g.layht;
    g.pbot = verint_host(H, P, npro, g.layht);
    g.lnpbot = std::log(g.pbot);
    g.smax = std::sqrt((radius + htop) * (radius + htop) - (g.sin2a * (g.z0 * g.z0))) - g.cosa * g.z0;
    // the layers' base heights (layerg.f:164-224): nlay scalars of the set-up
    std::vector<float> bases_h(nlay);
    const float lnptop = std::log(P[npro - 1]);
    for (int I = 1; I <= nlay; ++I) {
        float v = 0.0f;
        switch (o->laytyp) {
            case 0: v = verint_host(P, H, npro, g.pbot + (float)(I - 1) * (P[npro - 1] - g.pbot) / (float)nlay); break;
            case 1:
                v = verint_host(P, H, npro, std::exp(g.lnpbot + (float)(I - 1) * (lnptop - g.lnpbot) / (float)nlay));
                break;
            case 2: v = g.layht + (float)(I - 1) * (htop - g.layht) / (float)nlay; break;
            case 3: {
                const float s = (float)(I - 1) * g.smax / (float)nlay;
                v = std::sqrt(g.sin2a * (g.z0 * g.z0) + (s + g.cosa * g.z0) * (s + g.cosa * g.z0)) - radius;
                break;
            }
            case 4: v = verint_host(P, H, npro, o->base[I - 1]); break;
            default: v = o->base[I - 1];
        }
        bases_h[I - 1] = v;
    }
    in.insert(in.end(), bases_h.begin(), bases_h.end());
    // the path (atmg.f:142-147, 250-292): the bottom layer's base height, the angle
    const float bb = bases_h[o->botlay - 1];
    const bool surface = o->angle > 90.0f;
    float angle = surface ? 180 - o->angle : o->angle;
    if (o->ipzen == 1) angle = (1.0f / dtr) * std::asin(radius * std::sin(dtr * angle) / (radius + bb));
    // compact outputs
    const size_t n_sc = (size_t)nlay * 8, n_gas = (size_t)nvmr * nlay * 2, n_dust = (size_t)nlay * ndust;
    const size_t n_grad = (size_t)npro * nlay * 3, n_path = (size_t)nlay * 3;
    const size_t n_out = n_sc + n_gas + n_dust + n_grad + n_path;
    const size_t b_in = al16(in.size() * 4), b_out = al16(n_out * 4);
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    CUDA_TRY(c, c->d_layer.ensure(b_in + b_out + 16));
    char* base = (char*)c->d_layer.p;
    float* din = (float*)base;
    float* dout = (float*)(base + b_in);
    int* dstatus = (int*)(base + b_in + b_out);
    LayArgs A;
    std::memset(&A, 0, sizeof A);
    A.npro = npro;
    A.nvmr = nvmr;
    A.ndust = ndust;
    A.nlay = nlay;
    A.laytyp = o->laytyp;
    A.layint = o->layint;
    A.botlay = o->botlay;
    A.surface = surface ? 1 : 0;
    A.hsorted = pr->h[0] < pr->h[npro - 1] ? 1 : 0;
    for (int k = 1; k < npro && A.hsorted; ++k)
        if (!(pr->h[k] >= pr->h[k - 1])) A.hsorted = 0;
    A.h = din;
    A.p = din + npro;
    A.t = din + 2 * npro;
    A.vmr = din + 3 * npro;
    A.dust = A.vmr + (size_t)nvmr * npro;
    A.bases_h = A.dust + (size_t)ndust * npro;
    A.molwt = pr->molwt;
    A.radius = pr->radius;
    A.g = g;
    const float s2 = std::sin(dtr * angle);
    A.sin2 = s2 * s2;
    A.cosz = std::cos(dtr * angle);
    A.zpath = radius + bb;
    float* q = dout;
    float** sc[8] = {&A.baseh, &A.delh, &A.basep, &A.baset, &A.press, &A.temp, &A.totam, &A.laysf};
    for (int k = 0; k < 8; ++k, q += nlay) *sc[k] = q;
    A.amount = q;
    q += (size_t)nvmr * nlay;
    A.pp = q;
    q += (size_t)nvmr * nlay;
    A.cont = q;
    q += n_dust;
    A.dte = q;
    q += (size_t)npro * nlay;
    A.dam = q;
    q += (size_t)npro * nlay;
    A.dco = q;
    q += (size_t)npro * nlay;
    A.layinc = (int*)q;
    q += nlay;
    A.scale = q;
    q += nlay;
    A.emtemp = q;
    A.status = dstatus;
    CUDA_TRY(c, cudaMemcpyAsync(din, in.data(), in.size() * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemsetAsync(A.status, 0, 4, st));
    CUDA_TRY(c, cudaMemsetAsync(A.layinc, 0, (size_t)nlay * 3 * 4, st));
    const size_t lsm = layer_smem_bytes(nvmr, ndust, npro);
    CUDA_TRY(c, cudaFuncSetAttribute(layerg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm));
    layerg_kernel<<<nlay, 32, lsm, st>>>(A);
    CUDA_TRY(c, cudaGetLastError());
    std::vector<float> h(n_out);
    int status = 0;
    CUDA_TRY(c, cudaMemcpyAsync(h.data(), dout, n_out * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(&status, A.status, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    if (status) return fail(c, RTB_ERR_RANGE, "layerg: layer properties gone negative (layerg.f:460-495)");
    // scatter into the caller's arrays with their leading dimensions
    const float* r = h.data();
    float* dst1[8] = {out->baseh, out->delh, out->basep, out->baset, out->press, out->temp, out->totam, out->laysf};
    for (int k = 0; k < 8; ++k, r += nlay)
        if (dst1[k]) std::memcpy(dst1[k], r, (size_t)nlay * 4);
    for (int k = 0; k < 2; ++k) {
        float* d = k == 0 ? out->amount : out->pp;
        for (int g = 0; g < nvmr; ++g, r += nlay)
            if (d) std::memcpy(d + (size_t)LDL * g, r, (size_t)nlay * 4);
    }
    for (int l = 0; l < nlay; ++l, r += ndust)
        if (out->cont && ndust) std::memcpy(out->cont + (size_t)LDC * l, r, (size_t)ndust * 4);
    float* dst2[3] = {out->dte, out->dam, out->dco};
    for (int k = 0; k < 3; ++k)
        for (int m = 0; m < npro; ++m, r += nlay)
            if (dst2[k]) std::memcpy(dst2[k] + (size_t)LDL * m, r, (size_t)nlay * 4);
    const int nuse = nlay - o->botlay + 1;
    if (out->layinc) std::memcpy(out->layinc, r, (size_t)nuse * 4);
    r += nlay;
    if (out->scale) std::memcpy(out->scale, r, (size_t)nuse * 4);
    r += nlay;
    if (out->emtemp) std::memcpy(out->emtemp, r, (size_t)nuse * 4);
    if (out->npath) *out->npath = 1;
    if (out->nlayin) *out->nlayin = nuse;
    if (out->imod) *out->imod = 3;
    return RTB_OK;
}
