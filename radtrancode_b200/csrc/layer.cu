// layer.cu -- atmospheric layering on the device: LAYERG
// (radtran/path/layerg.f:146-458) and the nadir thermal path of ATMG
// (radtran/path/atmg.f:250-373, 509-560), the set-up subpathg runs before
// every forward call of a retrieval (the .prf -> layers step).
//
// One warp per layer.  The warp's lanes share the layer's accumulators: lane
// role 0 the layer totals (TOTAM, TEMP, PRESS) and the gradient rows DTE,
// DAM, DCO; roles 1..nvmr the amount and partial pressure of one gas; the
// rest one dust type each.  Every role walks the 101 Simpson points itself,
// so each accumulator is summed in the reference's order; the REAL
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

constexpr int kLayWarps = 4;
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
    const float *h, *p, *t, *vmr, *dust, *base;   // vmr [nvmr][npro], dust [ndust][npro]
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

// base height of layer I (1-based), layerg.f:164-224
__device__ float base_height(const LayArgs& A, int I) {
    const int NPRO = A.npro;
    const float* H = A.h;
    const float* P = A.p;
    const LayGeom& g = A.g;
    const float fi = (float)(I - 1), fn = (float)A.nlay;
    switch (A.laytyp) {
        case 0: {
            const float pnow = fa(g.pbot, fd(fm(fi, fs(P[NPRO - 1], g.pbot)), fn));
            return verint_dev(P, H, NPRO, pnow);
        }
        case 2: return fa(g.layht, fd(fm(fi, fs(H[NPRO - 1], g.layht)), fn));
        case 3: {
            const float s = fd(fm(fi, g.smax), fn);
            const float u = fa(s, fm(g.cosa, g.z0));
            return fs(__fsqrt_rn(fa(fm(g.sin2a, fm(g.z0, g.z0)), fm(u, u))), A.radius);
        }
        case 1:   // base pressures exp(ln p) from the host (layerg.f:174-181)
        case 4: return verint_dev(P, H, NPRO, A.base[I - 1]);
        default: return A.base[I - 1];
    }
}

// distance along a path from its start to height b (atmg.f:357-362 / layerg.f:236-240)
__device__ float path_s(float radius, float b, float sin2, float z, float cosz) {
    float stmp = fs(fm(fa(radius, b), fa(radius, b)), fm(sin2, fm(z, z)));
    if (stmp < 0.0f) stmp = 0.0f;
    return fs(__fsqrt_rn(stmp), fm(z, cosz));
}

__global__ void __launch_bounds__(32 * kLayWarps) layerg_kernel(LayArgs A) {
    const int lane = threadIdx.x & 31;
    const int L = blockIdx.x * kLayWarps + (threadIdx.x >> 5) + 1;   // 1-based layer
    if (L > A.nlay) return;
    const int i = L - 1, NPRO = A.npro, NLAY = A.nlay;
    const float* H = A.h;
    const float* P = A.p;
    const float* T = A.t;
    const LayGeom& g = A.g;
    const float radius = A.radius;
    const float bh = base_height(A, L);
    const float bh1 = L < NLAY ? base_height(A, L + 1) : 0.0f;
    const float htop = H[NPRO - 1];
    const float S0 = path_s(radius, bh, g.sin2a, g.z0, g.cosa);
    const float S1 = L < NLAY ? path_s(radius, bh1, g.sin2a, g.z0, g.cosa) : g.smax;
    const float laysf = fd(fs(S1, S0), L < NLAY ? fs(bh1, bh) : fs(htop, bh));
    // zero this layer's gradient rows
    for (int jj = lane; jj < NPRO; jj += 32) {
        A.dte[(size_t)jj * NLAY + i] = 0.0f;
        A.dam[(size_t)jj * NLAY + i] = 0.0f;
        A.dco[(size_t)jj * NLAY + i] = 0.0f;
    }
    __syncwarp();
    const int nq = 1 + A.nvmr + A.ndust;
    const float mw_av = fd(A.molwt, 6.022045E23f);   // XMOLWT / AVOGAD
    const float modboltz = 1.013E4f / 1.37947E-23f;  // constdef.f:8-9
    bool bad = false;
    float temp_layer = 0.0f;
    for (int q = lane; q < nq; q += 32) {
        const int gas = q - 1, dst = q - 1 - A.nvmr;
        const float* Y = q == 0 ? T : (gas < A.nvmr ? A.vmr + (size_t)gas * NPRO : A.dust + (size_t)dst * NPRO);
        float TOTAM = 0.0f, TEMP = 0.0f, PRESS = 0.0f, ACC = 0.0f, ACC2 = 0.0f;
        float* dte = A.dte + i;
        float* dam = A.dam + i;
        float* dco = A.dco + i;
        if (A.layint == 0) {
            // layer-centre values (layerg.f:264-313)
            const float S = fm(0.5f, fa(S0, S1));
            const float u = fa(S, fm(g.z0, g.cosa));
            const float HEIGHT = fs(__fsqrt_rn(fa(fm(u, u), fm(g.sin2a, fm(g.z0, g.z0)))), radius);
            const int I = above_dev(H, NPRO, HEIGHT);
            const float F = verintg_f(H, I, HEIGHT);
            PRESS = verint_at(H, P, I, HEIGHT);
            TEMP = verintg_y(T, I, F);
            TOTAM = fm(fd(fm(modboltz, PRESS), TEMP), fs(S1, S0));
            if (q == 0) {
                const int JJ = I - 1;
                dte[(size_t)(JJ - 1) * NLAY] = fa(dte[(size_t)(JJ - 1) * NLAY], fs(1.0f, F));
                dte[(size_t)JJ * NLAY] = fa(dte[(size_t)JJ * NLAY], F);
                // DCO(I,JJ) = (1-F) * TOTAM * XMOLWT / AVOGAD, likewise F
                dco[(size_t)(JJ - 1) * NLAY] = fd(fm(fm(fs(1.0f, F), TOTAM), A.molwt), 6.022045E23f);
                dco[(size_t)JJ * NLAY] = fd(fm(fm(F, TOTAM), A.molwt), 6.022045E23f);
                dam[(size_t)(JJ - 1) * NLAY] = fm(fs(1.0f, F), TOTAM);
                dam[(size_t)JJ * NLAY] = fm(F, TOTAM);
            } else if (gas < A.nvmr) {
                const float v = verintg_y(Y, I, F);
                ACC = fm(v, TOTAM);
                ACC2 = fm(v, PRESS);
            } else {
                ACC = fd(fm(fm(verintg_y(Y, I, F), TOTAM), A.molwt), 6.022045E23f);
            }
        } else {
            // Curtis-Godson path (layerg.f:315-402)
            const float DELS = fd(fs(S1, S0), (float)(kNint - 1));
            for (int K = 1; K <= kNint; ++K) {
                const float S = fa(S0, fm((float)(K - 1), DELS));
                const float u = fa(S, fm(g.z0, g.cosa));
                const float HEIGHT = fs(__fsqrt_rn(fa(fm(u, u), fm(g.sin2a, fm(g.z0, g.z0)))), radius);
                const int I = above_dev(H, NPRO, HEIGHT);
                const float PNOW = verint_at(H, P, I, HEIGHT);
                const float TNOW = verint_at(H, T, I, HEIGHT);
                const float DUDS = fd(fm(modboltz, PNOW), TNOW);
                const float WK = (K == 1 || K == kNint) ? 1.0f : ((K & 1) == 0 ? 4.0f : 2.0f);
                const float dw = fm(DUDS, WK);
                TOTAM = fa(TOTAM, dw);
                if (q == 0) {
                    const float F = verintg_f(H, I, HEIGHT);
                    const int JJ = I - 1;
                    const float a0 = fm(fm(fs(1.0f, F), DUDS), WK), a1 = fm(fm(F, DUDS), WK);
                    TEMP = fa(TEMP, fm(fm(TNOW, DUDS), WK));
                    dte[(size_t)(JJ - 1) * NLAY] = fa(dte[(size_t)(JJ - 1) * NLAY], a0);
                    dte[(size_t)JJ * NLAY] = fa(dte[(size_t)JJ * NLAY], a1);
                    PRESS = fa(PRESS, fm(fm(PNOW, DUDS), WK));
                    dco[(size_t)(JJ - 1) * NLAY] = fa(dco[(size_t)(JJ - 1) * NLAY], fd(fm(a0, A.molwt), 6.022045E23f));
                    dco[(size_t)JJ * NLAY] = fa(dco[(size_t)JJ * NLAY], fd(fm(a1, A.molwt), 6.022045E23f));
                    dam[(size_t)(JJ - 1) * NLAY] = fa(dam[(size_t)(JJ - 1) * NLAY], a0);
                    dam[(size_t)JJ * NLAY] = fa(dam[(size_t)JJ * NLAY], a1);
                } else if (gas < A.nvmr) {
                    const float v = verint_at(H, Y, I, HEIGHT);
                    ACC = fa(ACC, fm(fm(v, DUDS), WK));
                    ACC2 = fa(ACC2, fm(fm(fm(v, PNOW), DUDS), WK));
                } else {
                    const float d = verint_at(H, Y, I, HEIGHT);
                    ACC = fa(ACC, fm(fm(fm(d, mw_av), DUDS), WK));
                }
            }
            // normalisation (layerg.f:403-422)
            if (q == 0) {
                TEMP = fd(TEMP, TOTAM);
                PRESS = fd(PRESS, TOTAM);
                for (int jj = 0; jj < NPRO; ++jj) {
                    dte[(size_t)jj * NLAY] = fd(dte[(size_t)jj * NLAY], TOTAM);
                    dam[(size_t)jj * NLAY] = fd(fm(dam[(size_t)jj * NLAY], DELS), 3.0f);
                    dco[(size_t)jj * NLAY] = fd(fm(dco[(size_t)jj * NLAY], DELS), 3.0f);
                }
            } else if (gas < A.nvmr) {
                ACC = fd(fm(ACC, DELS), 3.0f);
                ACC2 = fd(ACC2, TOTAM);
            } else {
                ACC = fd(fm(ACC, DELS), 3.0f);
            }
            TOTAM = fd(fm(TOTAM, DELS), 3.0f);
        }
        // back to a vertical path (layerg.f:430-447) and the range check (:449-495)
        TOTAM = fd(TOTAM, laysf);
        if (q == 0) {
            for (int jj = 0; jj < NPRO; ++jj) {
                dam[(size_t)jj * NLAY] = fd(dam[(size_t)jj * NLAY], laysf);
                dco[(size_t)jj * NLAY] = fd(dco[(size_t)jj * NLAY], laysf);
            }
            A.press[i] = PRESS;
            A.temp[i] = TEMP;
            A.totam[i] = TOTAM;
            A.laysf[i] = laysf;
            A.baseh[i] = bh;
            A.delh[i] = L < NLAY ? fs(bh1, bh) : fs(htop, bh);
            A.basep[i] = verint_dev(H, P, NPRO, bh);
            A.baset[i] = verint_dev(H, T, NPRO, bh);
            bad = bad || PRESS < 0.0f || TEMP < 0.0f || TOTAM < 0.0f;
            temp_layer = TEMP;
        } else if (gas < A.nvmr) {
            ACC = fd(ACC, laysf);
            A.amount[(size_t)gas * NLAY + i] = ACC;
            A.pp[(size_t)gas * NLAY + i] = ACC2;
            bad = bad || ACC < 0.0f || ACC2 < 0.0f;
        } else {
            ACC = fd(ACC, laysf);
            A.cont[(size_t)i * A.ndust + dst] = ACC;
            bad = bad || ACC < 0.0f;
        }
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
    std::vector<float> bases;
    if (o->laytyp == 1) {   // equal log pressure (layerg.f:174-181): the base pressures
        const float lnptop = std::log(P[npro - 1]);
        for (int I = 1; I <= nlay; ++I)
            bases.push_back(std::exp(g.lnpbot + (float)(I - 1) * (lnptop - g.lnpbot) / (float)nlay));
    } else if (o->laytyp >= 4) {
        bases.assign(o->base, o->base + nlay);
    }
    in.insert(in.end(), bases.begin(), bases.end());
    // the path (atmg.f:142-147, 250-292): the bottom layer's base height, the angle
    const int bl = o->botlay;
    float bb = 0.0f;
    switch (o->laytyp) {
        case 0: bb = verint_host(P, H, npro, g.pbot + (float)(bl - 1) * (P[npro - 1] - g.pbot) / (float)nlay); break;
        case 1:
        case 4: bb = verint_host(P, H, npro, bases[bl - 1]); break;
        case 2: bb = g.layht + (float)(bl - 1) * (htop - g.layht) / (float)nlay; break;
        case 3: {
            const float s = (float)(bl - 1) * g.smax / (float)nlay;
            bb = std::sqrt(g.sin2a * (g.z0 * g.z0) + (s + g.cosa * g.z0) * (s + g.cosa * g.z0)) - radius;
            break;
        }
        default: bb = bases[bl - 1];
    }
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
    A.h = din;
    A.p = din + npro;
    A.t = din + 2 * npro;
    A.vmr = din + 3 * npro;
    A.dust = A.vmr + (size_t)nvmr * npro;
    A.base = A.dust + (size_t)ndust * npro;
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
    layerg_kernel<<<(nlay + kLayWarps - 1) / kLayWarps, 32 * kLayWarps, 0, st>>>(A);
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
