/*
 * layer_oracle.cpp -- ORACLE (test infrastructure only): CPU restatement of
 * LAYERG (radtran/path/layerg.f:146-458) and of the nadir thermal path of
 * ATMG (radtran/path/atmg.f:250-373, 509-560), in the reference's REAL
 * arithmetic and evaluation order, with VERINT (radtran/path/verint.f:29-46)
 * and VERINTG (radtran/path/verintg.f).  Only tests/ use it, as the checker
 * of rtb_layerg.
 */
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

const float kDtr = 3.1415926f / 180.0f;                 /* layerg.f:49 */
const float kModBoltz = 1.013E4f / 1.37947E-23f;        /* constdef.f:8-9 */
const float kAvogad = 6.022045E23f;                     /* constdef.f:10 */
const int kNint = 101;                                  /* layerg.f:44 */

/* first point beyond XIN in the table's direction (N if none, 2 if the first) */
int above(const float* X, int N, float XIN) {
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

float verint(const float* X, const float* Y, int N, float XIN) {
    const int I = above(X, N, XIN);
    float YOUT = Y[I - 2] + (Y[I - 1] - Y[I - 2]) * (XIN - X[I - 2]) / (X[I - 1] - X[I - 2]);
    if (X[I - 2] == X[I - 1]) YOUT = Y[I - 1];
    if (std::isnan(YOUT)) YOUT = Y[I - 1];
    return YOUT;
}

/* VERINTG: value, J (1-based lower point) and F */
float verintg(const float* X, const float* Y, int N, float XIN, int& J, float& F) {
    const int I = above(X, N, XIN);
    J = I - 1;
    F = (XIN - X[I - 2]) / (X[I - 1] - X[I - 2]);
    return (1.0f - F) * Y[I - 2] + F * Y[I - 1];
}

}  // namespace

extern "C" int orc_layerg(const rtb_profile* pr, const rtb_layer_opts* o, rtb_layers* out) {
    const int NPRO = pr->npro, NVMR = pr->nvmr, NDUST = pr->ndust, NLAY = o->nlay;
    const int ldp = pr->ld_pro > 0 ? pr->ld_pro : NPRO, ldc = pr->ld_con > 0 ? pr->ld_con : NDUST;
    const int LDL = out->ld_lay > 0 ? out->ld_lay : NLAY, LDC = out->ld_con > 0 ? out->ld_con : NDUST;
    const float *H = pr->h, *P = pr->p, *T = pr->t;
    const float RADIUS = pr->radius, XMOLWT = pr->molwt;
    float LAYHT = o->layht;
    if (LAYHT < H[0]) LAYHT = H[0];                     /* layerg.f:95-103 */
    float W[kNint];
    for (int I = 1; I <= kNint; ++I) W[I - 1] = (I == 2 * (I / 2)) ? 4.0f : 2.0f;
    W[0] = 1.0f;
    W[kNint - 1] = 1.0f;
    const float sa = std::sin(kDtr * o->layang);
    const float SIN2A = sa * sa;
    const float COSA = std::cos(kDtr * o->layang);
    const float Z0 = RADIUS + LAYHT;
    const float PBOT = verint(H, P, NPRO, LAYHT);
    const float LNPBOT = std::log(PBOT);
    const float SMAX = std::sqrt((RADIUS + H[NPRO - 1]) * (RADIUS + H[NPRO - 1]) - (SIN2A * (Z0 * Z0))) - COSA * Z0;
    std::vector<float> BASEH(NLAY);
    for (int I = 1; I <= NLAY; ++I) {
        float v = 0.0f;
        switch (o->laytyp) {
            case 0: {
                const float PNOW = PBOT + (float)(I - 1) * (P[NPRO - 1] - PBOT) / (float)NLAY;
                v = verint(P, H, NPRO, PNOW);
                break;
            }
            case 1: {
                float LNPNOW = std::log(P[NPRO - 1]);
                LNPNOW = LNPBOT + (float)(I - 1) * (LNPNOW - LNPBOT) / (float)NLAY;
                v = verint(P, H, NPRO, std::exp(LNPNOW));
                break;
            }
            case 2: v = LAYHT + (float)(I - 1) * (H[NPRO - 1] - LAYHT) / (float)NLAY; break;
            case 3: {
                const float S = (float)(I - 1) * SMAX / (float)NLAY;
                v = std::sqrt(SIN2A * (Z0 * Z0) + (S + COSA * Z0) * (S + COSA * Z0)) - RADIUS;
                break;
            }
            case 4: v = verint(P, H, NPRO, o->base[I - 1]); break;
            case 5: v = o->base[I - 1]; break;
            default: return RTB_ERR_UNSUPPORTED;
        }
        BASEH[I - 1] = v;
    }
    std::vector<float> D(NPRO), TL(NLAY);
    for (int L = 1; L <= NLAY; ++L) {
        const int i = L - 1;
        const float bh = BASEH[i];
        if (out->baseh) out->baseh[i] = bh;
        if (out->delh) out->delh[i] = L < NLAY ? BASEH[i + 1] - bh : H[NPRO - 1] - bh;
        if (out->basep) out->basep[i] = verint(H, P, NPRO, bh);
        if (out->baset) out->baset[i] = verint(H, T, NPRO, bh);
        float STMP = (RADIUS + bh) * (RADIUS + bh) - SIN2A * (Z0 * Z0);
        if (STMP < 0) STMP = 0;
        const float S0 = std::sqrt(STMP) - Z0 * COSA;
        float S1, LAYSF;
        if (L < NLAY) {
            S1 = std::sqrt((RADIUS + BASEH[i + 1]) * (RADIUS + BASEH[i + 1]) - SIN2A * (Z0 * Z0)) - Z0 * COSA;
            LAYSF = (S1 - S0) / (BASEH[i + 1] - bh);
        } else {
            S1 = SMAX;
            LAYSF = (S1 - S0) / (H[NPRO - 1] - bh);
        }
        float PRESS = 0, TEMP = 0, TOTAM = 0;
        std::vector<float> DTE(NPRO, 0.0f), DAM(NPRO, 0.0f), DCO(NPRO, 0.0f);
        std::vector<float> AMOUNT(NVMR, 0.0f), PP(NVMR, 0.0f), CONT(NDUST, 0.0f);
        if (o->layint == 0) {
            const float S = 0.5f * (S0 + S1);
            const float HEIGHT = std::sqrt((S + Z0 * COSA) * (S + Z0 * COSA) + SIN2A * (Z0 * Z0)) - RADIUS;
            int JJ = 0;
            float F = 0;
            PRESS = verint(H, P, NPRO, HEIGHT);
            TEMP = verintg(H, T, NPRO, HEIGHT, JJ, F);
            DTE[JJ - 1] = DTE[JJ - 1] + (1 - F);
            DTE[JJ] = DTE[JJ] + F;
            for (int J = 0; J < NDUST; ++J) {
                for (int M = 0; M < NPRO; ++M) D[M] = pr->dust[J + (size_t)ldc * M];
                CONT[J] = verintg(H, D.data(), NPRO, HEIGHT, JJ, F);
            }
            DCO[JJ - 1] = DCO[JJ - 1] + (1.0f - F);
            DCO[JJ] = DCO[JJ] + F;
            const float DUDS = kModBoltz * PRESS / TEMP;
            TOTAM = DUDS * (S1 - S0);
            for (int J = 0; J < NDUST; ++J) CONT[J] = CONT[J] * TOTAM * XMOLWT / kAvogad;
            for (int JJ2 = 0; JJ2 < NPRO; ++JJ2) DCO[JJ2] = DCO[JJ2] * TOTAM * XMOLWT / kAvogad;
            for (int J = 0; J < NVMR; ++J) {
                const float VMR1 = verintg(H, pr->vmr + (size_t)ldp * J, NPRO, HEIGHT, JJ, F);
                AMOUNT[J] = AMOUNT[J] + VMR1 * TOTAM;
                PP[J] = PP[J] + VMR1 * PRESS;
            }
            DAM[JJ - 1] = DAM[JJ - 1] + (1.0f - F) * TOTAM;
            DAM[JJ] = DAM[JJ] + F * TOTAM;
        } else if (o->layint == 1) {
            const float DELS = (S1 - S0) / (float)(kNint - 1);
            for (int K = 1; K <= kNint; ++K) {
                const float S = S0 + (float)(K - 1) * DELS;
                const float HEIGHT = std::sqrt((S + Z0 * COSA) * (S + Z0 * COSA) + SIN2A * (Z0 * Z0)) - RADIUS;
                const float PNOW = verint(H, P, NPRO, HEIGHT);
                const float TNOW = verint(H, T, NPRO, HEIGHT);
                int JJ = 0;
                float F = 0;
                verintg(H, H, NPRO, HEIGHT, JJ, F);     /* the level and fraction of the FPH2I call */
                const float DUDS = kModBoltz * PNOW / TNOW;
                const float WK = W[K - 1];
                TOTAM = TOTAM + DUDS * WK;
                TEMP = TEMP + TNOW * DUDS * WK;
                DTE[JJ - 1] = DTE[JJ - 1] + (1 - F) * DUDS * WK;
                DTE[JJ] = DTE[JJ] + F * DUDS * WK;
                PRESS = PRESS + PNOW * DUDS * WK;
                for (int J = 0; J < NDUST; ++J) {
                    for (int M = 0; M < NPRO; ++M) D[M] = pr->dust[J + (size_t)ldc * M];
                    const float DNOW = verint(H, D.data(), NPRO, HEIGHT);
                    CONT[J] = CONT[J] + DNOW * (XMOLWT / kAvogad) * DUDS * WK;
                }
                DCO[JJ - 1] = DCO[JJ - 1] + (1 - F) * DUDS * WK * XMOLWT / kAvogad;
                DCO[JJ] = DCO[JJ] + F * DUDS * WK * XMOLWT / kAvogad;
                for (int J = 0; J < NVMR; ++J) {
                    const float VMR1 = verint(H, pr->vmr + (size_t)ldp * J, NPRO, HEIGHT);
                    AMOUNT[J] = AMOUNT[J] + VMR1 * DUDS * WK;
                    PP[J] = PP[J] + VMR1 * PNOW * DUDS * WK;
                }
                DAM[JJ - 1] = DAM[JJ - 1] + (1 - F) * DUDS * WK;
                DAM[JJ] = DAM[JJ] + F * DUDS * WK;
            }
            TEMP = TEMP / TOTAM;
            PRESS = PRESS / TOTAM;
            for (int JJ = 0; JJ < NPRO; ++JJ) DTE[JJ] = DTE[JJ] / TOTAM;
            for (int J = 0; J < NVMR; ++J) {
                AMOUNT[J] = AMOUNT[J] * DELS / 3.0f;
                PP[J] = PP[J] / TOTAM;
            }
            for (int JJ = 0; JJ < NPRO; ++JJ) DAM[JJ] = DAM[JJ] * DELS / 3.0f;
            TOTAM = TOTAM * DELS / 3.0f;
            for (int J = 0; J < NDUST; ++J) CONT[J] = CONT[J] * DELS / 3.0f;
            for (int JJ = 0; JJ < NPRO; ++JJ) DCO[JJ] = DCO[JJ] * DELS / 3.0f;
        } else {
            return RTB_ERR_UNSUPPORTED;
        }
        /* back to a vertical path (layerg.f:434-447) */
        TOTAM = TOTAM / LAYSF;
        for (int J = 0; J < NVMR; ++J) AMOUNT[J] = AMOUNT[J] / LAYSF;
        for (int JJ = 0; JJ < NPRO; ++JJ) DAM[JJ] = DAM[JJ] / LAYSF;
        for (int J = 0; J < NDUST; ++J) CONT[J] = CONT[J] / LAYSF;
        for (int JJ = 0; JJ < NPRO; ++JJ) DCO[JJ] = DCO[JJ] / LAYSF;
        bool bad = PRESS < 0.0f || TEMP < 0.0f || TOTAM < 0.0f;
        for (int J = 0; J < NVMR; ++J) bad = bad || AMOUNT[J] < 0.0f || PP[J] < 0.0f;
        for (int J = 0; J < NDUST; ++J) bad = bad || CONT[J] < 0.0f;
        if (bad) return RTB_ERR_RANGE;
        TL[i] = TEMP;
        if (out->press) out->press[i] = PRESS;
        if (out->temp) out->temp[i] = TEMP;
        if (out->totam) out->totam[i] = TOTAM;
        if (out->laysf) out->laysf[i] = LAYSF;
        for (int J = 0; J < NVMR; ++J) {
            if (out->amount) out->amount[i + (size_t)LDL * J] = AMOUNT[J];
            if (out->pp) out->pp[i + (size_t)LDL * J] = PP[J];
        }
        for (int J = 0; J < NDUST; ++J)
            if (out->cont) out->cont[J + (size_t)LDC * i] = CONT[J];
        for (int JJ = 0; JJ < NPRO; ++JJ) {
            if (out->dte) out->dte[i + (size_t)LDL * JJ] = DTE[JJ];
            if (out->dam) out->dam[i + (size_t)LDL * JJ] = DAM[JJ];
            if (out->dco) out->dco[i + (size_t)LDL * JJ] = DCO[JJ];
        }
    }
    /* ATMG nadir thermal path: one path (IMOD 3), layers botlay..nlay */
    float ANGLE = o->angle;
    const bool SURFACE = ANGLE > 90.0f;                  /* atmg.f:142-147 */
    if (SURFACE) ANGLE = 180 - ANGLE;
    const int BOTLAY = o->botlay;
    if (BOTLAY < 1 || BOTLAY > NLAY) return RTB_ERR_ARG;
    if (o->ipzen == 1) {                                 /* atmg.f:253-257 */
        const float z = RADIUS + BASEH[BOTLAY - 1];
        ANGLE = (1.0f / kDtr) * std::asin(RADIUS * std::sin(kDtr * ANGLE) / z);
    } else if (o->ipzen != 0) {
        return RTB_ERR_UNSUPPORTED;
    }
    const float s2 = std::sin(kDtr * ANGLE);
    const float SIN2 = s2 * s2, COS = std::cos(kDtr * ANGLE);
    const float Z = RADIUS + BASEH[BOTLAY - 1];
    const int NUSE = NLAY - BOTLAY + 1;
    for (int I = 1; I <= NUSE; ++I) {
        const int LOC = SURFACE ? I : NLAY - I + 1;      /* atmg.f:328-350 */
        const float b = BASEH[LOC - 1];
        float STMP = (RADIUS + b) * (RADIUS + b) - SIN2 * (Z * Z);
        if (STMP < 0) STMP = 0;
        const float S0 = std::sqrt(STMP) - Z * COS;
        float SF;
        if (LOC == NLAY) {
            const float S1 = std::sqrt((RADIUS + H[NPRO - 1]) * (RADIUS + H[NPRO - 1]) - SIN2 * (Z * Z)) - Z * COS;
            SF = (S1 - S0) / (H[NPRO - 1] - b);
        } else {
            const float S1 = std::sqrt((RADIUS + BASEH[LOC]) * (RADIUS + BASEH[LOC]) - SIN2 * (Z * Z)) - Z * COS;
            SF = (S1 - S0) / (BASEH[LOC] - b);
        }
        if (out->layinc) out->layinc[I - 1] = LOC;
        if (out->scale) out->scale[I - 1] = SF;
        if (out->emtemp) out->emtemp[I - 1] = TL[LOC - 1];
    }
    if (out->npath) *out->npath = 1;
    if (out->nlayin) *out->nlayin = NUSE;
    if (out->imod) *out->imod = 3;
    return RTB_OK;
}
