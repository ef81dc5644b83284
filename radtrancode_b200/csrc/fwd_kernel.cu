// fwd_kernel.cu -- B200 forward model + analytic Jacobian of the correlated-k
// thermal-emission path (radtran/cirsradg/cirsradg_wave.f, IMOD 0/1/3) fused
// with map2pro/map2xvec (radtran/cirsradg/map2pro.f, map2xvec.f).
//
// One CTA (8 warps) owns one (spectrum, wavenumber) work item at a time and
// loops over items grid-stride (persistent).  Stages:
//   A  per layer (one warp each): k-table interpolation of every gas
//      (get_kg.f:306-378), continuum optical depth and its derivatives
//      (nciacon.f, dust, Rayleigh: cirsradg_wave.f:510-691) and the random
//      overlap of the gas k-distributions (noverlapg.f/rankg.f) with a
//      warp-wide bitonic sort of the NG*NG combinations, an exact FP64 scan
//      of the weights and one lane per g-bin for the rebinning sums.
//      Results (tau and dtau/dq per g) stay in shared memory.
//   B  per path (one warp, one lane per g): Planck, transmissions, radiance
//      and dR/dtau of every layer by a suffix sum, which replaces the
//      O(L^2) recurrence of cirsradg_wave.f:954-978 by O(L) exact algebra.
//   C  g-quadrature of the layer Jacobian (cirsradg_wave.f:1240-1286).
//   D  layer -> state vector through a precomputed sparse map
//      (map2pro o map2xvec), written in the packing of cirsrtfg_wave.f:425-446.
//
// Bit-exactness of the g-bin assignment: every operation that feeds a sort
// key or a bin boundary is an explicitly rounded IEEE operation in the
// reference's order (no FMA contraction); the cumulative weights are FP64
// sums of FP32 products >= 2^-28, which are exact in any order; tied keys
// whose order could move a bin boundary take the reference's heapsort
// (sort2g.f) in-kernel.
#include <cuda_runtime.h>
#include <stdint.h>

#include "detexp.cuh"
#include "rtb_common.h"

namespace rtb {

namespace {

constexpr int kE = 16;               // sort elements per lane (NG*NG <= 512)
constexpr int kN = 32 * kE;

__device__ __forceinline__ unsigned long long shfl_xor64(unsigned long long v, int m) {
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    lo = __shfl_xor_sync(0xffffffffu, lo, m);
    hi = __shfl_xor_sync(0xffffffffu, hi, m);
    return ((unsigned long long)hi << 32) | lo;
}

// order-preserving map of a float onto uint32 (-0 folded onto +0 first)
__device__ __forceinline__ unsigned fkey(float f) {
    unsigned u = __float_as_uint(__fadd_rn(f, 0.0f));
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(unsigned k) {
    unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// Warp bitonic sort of 32*kE packed (key, index) words; element lane*kE + r
// lives in v[r]; ascending.
__device__ __forceinline__ void warp_bitonic(unsigned long long (&v)[kE], int lane) {
#pragma unroll
    for (int k = 2; k <= kN; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= kE) {
                const int lm = j / kE;
                const bool lower = (lane & lm) == 0;
#pragma unroll
                for (int r = 0; r < kE; ++r) {
                    const unsigned long long o = shfl_xor64(v[r], lm);
                    const int idx = lane * kE + r;
                    const bool up = (idx & k) == 0;
                    const bool keep_min = (up == lower);
                    const unsigned long long mn = v[r] < o ? v[r] : o;
                    const unsigned long long mx = v[r] < o ? o : v[r];
                    v[r] = keep_min ? mn : mx;
                }
            } else {
#pragma unroll
                for (int r = 0; r < kE; ++r) {
                    const int p = r ^ j;
                    if (p > r) {
                        const int idx = lane * kE + r;
                        const bool up = (idx & k) == 0;
                        const unsigned long long a = v[r], b = v[p];
                        const bool sw = up ? (a > b) : (a < b);
                        v[r] = sw ? b : a;
                        v[p] = sw ? a : b;
                    }
                }
            }
        }
    }
}

// NR heapsort of radtran/cirsradg/sort2g.f:1-52 on shared memory (one thread);
// ra/ib hold RA(1..n)/IB(1..n) at ra[0..n-1].
__device__ void heapsort_sort2g(int n, float* ra0, short* ib0) {
    if (n < 2) return;
    float* RA = ra0 - 1;
    short* IB = ib0 - 1;
    int L = n / 2 + 1, IR = n;
    float RRA;
    short IRB;
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

// Shared-memory layout (bytes), identical on host and device.
struct Layout {
    int warp_bytes;       // per-warp scratch of stage A
    int off_gord;         // double[kMaxNg+1]
    int off_delg;         // float[kMaxNg]
    int off_tau;          // float[Lmax][ng]
    int off_dtau;         // float[Lmax][nsw][ng]
    int off_region;       // aliased: per-warp scratch (A) / path arrays (B-D)
    int path_bytes;       // per path in the region
    int total;
};

__host__ __device__ inline int align8(int x) { return (x + 7) & ~7; }

// per-warp scratch sub-offsets
struct WarpOff {
    int splitfrac, keys, idx, k1, k2, dk1, dk2, kg, colA, colB, splitpos, total;
};
__host__ __device__ inline WarpOff warp_off(int ncol) {
    WarpOff w;
    int o = 0;
    w.splitfrac = o; o += 8 * kMaxNg;
    w.keys = o; o += 4 * kN;
    w.idx = o; o += 2 * kN;
    w.k1 = o; o += 4 * kMaxNg;
    w.k2 = o; o += 4 * kMaxNg;
    w.dk1 = o; o += 4 * kMaxNg;
    w.dk2 = o; o += 4 * kMaxNg;
    w.kg = o; o += 4 * kMaxNg;
    w.colA = o; o += 4 * kMaxNg * (ncol > 0 ? ncol : 1);
    w.colB = o; o += 4 * kMaxNg * (ncol > 0 ? ncol : 1);
    w.splitpos = o; o += 4 * kMaxNg;
    w.total = align8(o);
    return w;
}
// per-path sub-offsets inside the region (stages B-D)
struct PathOff {
    int drdt, trd, bb, dbdt, dq, rad, gts, total;
};
__host__ __device__ inline PathOff path_off(int nlmax, int ng, int nsw) {
    PathOff p;
    int o = 0;
    p.drdt = o; o += 4 * nlmax * ng;
    p.trd = o; o += 4 * nlmax * ng;
    p.bb = o; o += 4 * nlmax;
    p.dbdt = o; o += 4 * nlmax;
    p.dq = o; o += 4 * nlmax * (nsw > 0 ? nsw : 1);
    p.rad = o; o += 4 * kMaxNg;
    p.gts = o; o += 4 * kMaxNg;
    p.total = align8(o);
    return p;
}

__host__ __device__ inline Layout make_layout(int ng, int Lmax, int nsw, int ncol, int nlmax, int npath) {
    Layout Lo;
    Lo.warp_bytes = warp_off(ncol).total;
    int o = 0;
    Lo.off_gord = o; o += 8 * (kMaxNg + 1);
    Lo.off_delg = o; o += 4 * kMaxNg;
    o = align8(o);
    Lo.off_tau = o; o += 4 * Lmax * ng;
    Lo.off_dtau = o; o += 4 * Lmax * (nsw > 0 ? nsw : 1) * ng;
    o = align8(o);
    Lo.off_region = o;
    Lo.path_bytes = path_off(nlmax, ng, nsw).total;
    const int a = kWarps * Lo.warp_bytes, b = npath * Lo.path_bytes;
    o += a > b ? a : b;
    Lo.total = o;
    return Lo;
}

// per-warp accumulation of diagnostics, flushed once per work item
struct Diag {
    unsigned long long sort_passes, tie_passes, exact_passes, irregular;
};

// ---------------------------------------------------------------------------
// get_kg for one gas at one layer: lane g < ng returns k(g), dk/dT(g)
// (get_kg.f:320-378 coincident branch, NaN -> 1e-37 at :443-471).
__device__ __forceinline__ void get_kg_lane(const BatchDev& B, int64_t slice, const LayerDev& L, int lane,
                                            float& k, float& dk) {
    k = 0.0f;
    dk = 0.0f;
    if (slice < 0) return;
    const float* raw = B.ktab_raw + slice;
    const float y10 = __ldg(raw + L.ioff[0]), y20 = __ldg(raw + L.ioff[1]);
    const float y30 = __ldg(raw + L.ioff[2]), y40 = __ldg(raw + L.ioff[3]);
    const bool klog = !((y10 <= 0.0f) || (y20 <= 0.0f) || (y30 <= 0.0f) || (y40 <= 0.0f));
    if (lane >= B.ng) return;
    const float* t = klog ? (B.ktab_log + slice) : raw;
    const float Y1 = __ldg(t + L.ioff[0] + lane), Y2 = __ldg(t + L.ioff[1] + lane);
    const float Y3 = __ldg(t + L.ioff[2] + lane), Y4 = __ldg(t + L.ioff[3] + lane);
    const float U = L.u, V = L.v;
    const float a = __fsub_rn(1.0f, V), b = __fsub_rn(1.0f, U);
    float X = __fmul_rn(__fmul_rn(a, b), Y1);
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(V, b), Y2));
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(V, U), Y3));
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(a, U), Y4));
    float D = -__fmul_rn(a, Y1);
    D = __fsub_rn(D, __fmul_rn(V, Y2));
    D = __fadd_rn(D, __fmul_rn(V, Y3));
    D = __fadd_rn(D, __fmul_rn(a, Y4));
    const float DXDT = __fmul_rn(D, L.dudt);
    if (klog) {
        const float e = det_expf(X);
        k = e;
        dk = __fmul_rn(e, DXDT);
    } else {
        k = X;
        dk = DXDT;
    }
    if (k != k) k = 1e-37f;
    if (dk != dk) dk = 1e-37f;
}

// continuum optical depth of one layer and its active derivatives
// (cirsradg_wave.f:526-691 with nciacon.f:84-310 / ciaread.f:108-198).
// Every lane computes the same scalars.
__device__ __forceinline__ float continuum(const BatchDev& B, const SpecDev& S, const LayerDev& L, const WaveDev& W,
                                           int64_t iw_glob, int64_t il_glob, float (&dtc)[kMaxSw]) {
#pragma unroll
    for (int s = 0; s < kMaxSw; ++s) dtc[s] = 0.0f;
    float taucon = 0.0f;
    for (int k = 0; k < S.ncont; ++k) {
        const float tau = B.xsec[iw_glob * S.ncont + k];
        taucon = __fadd_rn(taucon, __fmul_rn(tau, B.cont[il_glob * S.ncont + k]));
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s < S.nsw && S.isw[s] == S.ngas + 1 + k) dtc[s] = tau;
    }
    float absorb = 0.0f, dab[7] = {0, 0, 0, 0, 0, 0, 0};
    if (S.has_cia) {
        float alpha[9], da[9];
#pragma unroll
        for (int p = 0; p < 9; ++p) { alpha[p] = 0.0f; da[p] = 0.0f; }
        if (W.cia_cv >= 0) {
            const float t = W.cia_t, u = L.cia_u;
            const float omt = __fsub_rn(1.0f, t), omu = __fsub_rn(1.0f, u);
            const float* kc = B.kcia;
            const int64_t b11 = 9 * ((int64_t)L.cia_ct + 25 * (int64_t)W.cia_cv);
            const int64_t b12 = 9 * ((int64_t)L.cia_ct + 25 * ((int64_t)W.cia_cv + 1));
            const int64_t b22 = 9 * ((int64_t)L.cia_ct + 1 + 25 * ((int64_t)W.cia_cv + 1));
            const int64_t b21 = 9 * ((int64_t)L.cia_ct + 1 + 25 * (int64_t)W.cia_cv);
#pragma unroll
            for (int p = 0; p < 9; ++p) {
                const float a11 = __ldg(kc + b11 + p), a12 = __ldg(kc + b12 + p);
                const float a22 = __ldg(kc + b22 + p), a21 = __ldg(kc + b21 + p);
                float x = __fmul_rn(__fmul_rn(omt, omu), a11);
                x = __fadd_rn(x, __fmul_rn(__fmul_rn(t, omu), a12));
                x = __fadd_rn(x, __fmul_rn(__fmul_rn(t, u), a22));
                x = __fadd_rn(x, __fmul_rn(__fmul_rn(omt, u), a21));
                float d = -__fmul_rn(omt, a11);
                d = __fsub_rn(d, __fmul_rn(t, a12));
                d = __fadd_rn(d, __fmul_rn(t, a22));
                d = __fadd_rn(d, __fmul_rn(omt, a21));
                alpha[p] = x;
                da[p] = __fmul_rn(d, L.cia_dudt);
            }
        }
        const float qh2 = L.q[0], qhe = L.q[1], qn2 = L.q[2], qch4 = L.q[3], qco2 = L.q[4];
        float sum = 0.0f;
        const int o = S.inormal == 0 ? 0 : 2;
        sum = __fadd_rn(__fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[o], qh2), qh2)),
                        __fmul_rn(__fmul_rn(alpha[o + 1], qh2), qhe));
        dab[0] = __fadd_rn(__fadd_rn(dab[0], __fmul_rn(__fmul_rn(2.0f, qh2), alpha[o])), __fmul_rn(qhe, alpha[o + 1]));
        dab[1] = __fadd_rn(dab[1], __fmul_rn(qh2, alpha[o + 1]));
        dab[5] = __fadd_rn(__fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qh2), da[o])),
                           __fmul_rn(__fmul_rn(qh2, qhe), da[o + 1]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[4], qh2), qn2));
        dab[0] = __fadd_rn(dab[0], __fmul_rn(qn2, alpha[4]));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(qh2, alpha[4]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qn2), da[4]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[5], qn2), qch4));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(qch4, alpha[5]));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(qn2, alpha[5]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qn2, qch4), da[5]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[6], qn2), qn2));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(__fmul_rn(2.0f, qn2), alpha[6]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qn2, qn2), da[6]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[7], qch4), qch4));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(__fmul_rn(2.0f, qch4), alpha[7]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qch4, qch4), da[7]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(alpha[8], qh2), qch4));
        dab[0] = __fadd_rn(dab[0], __fmul_rn(qch4, alpha[8]));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(qh2, alpha[8]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qch4), da[8]));
        // co2cia / n2n2cia / n2h2cia are zero below 3900 cm-1 (host-checked)
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qco2), qco2));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qn2), qn2));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qn2), qh2));
        absorb = __fmul_rn(sum, L.cia_tau);
#pragma unroll
        for (int i = 0; i < 7; ++i) dab[i] = __fmul_rn(dab[i], L.cia_tau);
    }
    taucon = __fadd_rn(taucon, absorb);
    const float den = __fmul_rn(L.utotl, 1.0e20f);
    for (int ii = 0; ii < 5; ++ii) {
        const int k = L.iabs[ii];
        if (k < 0) continue;
        const float add = __fdiv_rn(dab[ii], den);
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s < S.nsw && S.isw[s] == k) dtc[s] = __fadd_rn(dtc[s], add);
    }
#pragma unroll
    for (int s = 0; s < kMaxSw; ++s)
        if (s == S.sw_T) dtc[s] = __fadd_rn(dtc[s], dab[5]);
    if (S.iray) {
        const float av = __fmul_rn(L.utotl, W.xray);
        taucon = __fadd_rn(taucon, av);
        const float add = __fmul_rn(W.xray, 1.0e-20f);
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s < S.nsw && S.isw[s] < S.ngas) dtc[s] = __fadd_rn(dtc[s], add);
    }
    return taucon;
}

// ---------------------------------------------------------------------------
// One overlap pass with sorting (noverlapg.f:110-147/175-190 + rankg.f).
// Inputs in the warp scratch: k1[i], k2[j], dk1[i], dk2[j] and the previous
// columns colP[c][i].  Outputs: new k_g in kg[], new columns in colN[c][].
struct PassCtx {
    int ng, nloop, ncol, first, igas;   // igas: 0-based index of the gas being added
    float a1, a2;
};

__device__ __forceinline__ float elem_grad(const PassCtx& P, const SpecDev& S, int c, int i, int j,
                                           const float* k1, const float* k2, const float* dk1, const float* dk2,
                                           const float* colP) {
    const int g = S.col_gas[c];
    if (g == S.ngas) {   // temperature column
        if (P.first) return __fadd_rn(__fmul_rn(dk1[i], P.a1), __fmul_rn(dk2[j], P.a2));
        return __fadd_rn(dk1[i], __fmul_rn(dk2[j], P.a2));
    }
    if (g == P.igas) return k2[j];
    if (P.first) return g == 0 ? k1[i] : 0.0f;
    return colP[c * kMaxNg + i];
}

__device__ void sort_pass(const BatchDev& B, const SpecDev& S, const PassCtx& P, char* wsm, const WarpOff& wo,
                          const double* g_ord, const float* delg, int lane, Diag& dg, float* colP, float* colN,
                          int16_t* dbg_perm, int16_t* dbg_split) {
    float* keys_s = (float*)(wsm + wo.keys);
    short* idx_s = (short*)(wsm + wo.idx);
    const float* k1 = (const float*)(wsm + wo.k1);
    const float* k2 = (const float*)(wsm + wo.k2);
    const float* dk1 = (const float*)(wsm + wo.dk1);
    const float* dk2 = (const float*)(wsm + wo.dk2);
    float* kg = (float*)(wsm + wo.kg);
    double* splitfrac = (double*)(wsm + wo.splitfrac);
    int* splitpos = (int*)(wsm + wo.splitpos);
    const int ng = P.ng, nloop = P.nloop;

    auto key_of = [&](int e) -> float {
        const int i = e / ng, j = e - (e / ng) * ng;
        return P.first ? __fadd_rn(__fmul_rn(k1[i], P.a1), __fmul_rn(k2[j], P.a2))
                       : __fadd_rn(k1[i], __fmul_rn(k2[j], P.a2));
    };

    // fast path: bitonic sort of (key, element) -> stable order of ties
    unsigned long long v[kE];
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        const int e = lane * kE + r;
        const float key = e < nloop ? key_of(e) : __int_as_float(0x7f800000);
        v[r] = ((unsigned long long)fkey(key) << 32) | (unsigned)e;
    }
    warp_bitonic(v, lane);
    float kr[kE];
    int ir[kE];
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        kr[r] = funkey((unsigned)(v[r] >> 32));
        ir[r] = (int)(v[r] & 0xffffffffu);
    }

    bool exact = false;
    double gd[kE], gprev0;
    int cc[kE], cprev0;
    bool irregular = false, gerr = false;
    for (int attempt = 0; attempt < 2; ++attempt) {
        // FP64 cumulative weights (exact in any order) and bin counts
        double run = 0.0;
#pragma unroll
        for (int r = 0; r < kE; ++r) {
            const int p = lane * kE + r;
            float w = 0.0f;
            if (p < nloop) {
                const int e = ir[r], i = e / ng, j = e - (e / ng) * ng;
                w = __fmul_rn(delg[i], delg[j]);
            }
            run = __dadd_rn(run, (double)w);
            gd[r] = run;
        }
        double incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl = __dadd_rn(incl, t);
        }
        const double base = __dsub_rn(incl, run);   // exact (all partial sums are exact)
        gprev0 = base;
#pragma unroll
        for (int r = 0; r < kE; ++r) gd[r] = __dadd_rn(gd[r], base);
        // c(p) = #{b in 1..ng : g_ord[b] <= gdist(p)}
#pragma unroll
        for (int r = 0; r < kE; ++r) {
            int lo = 0, hi = ng;   // count in [0, ng]
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (g_ord[mid] <= gd[r]) lo = mid; else hi = mid - 1;
            }
            cc[r] = lo;
        }
        cprev0 = __shfl_up_sync(0xffffffffu, cc[kE - 1], 1);
        if (lane == 0) cprev0 = 0;
        const float kprev0 = __shfl_up_sync(0xffffffffu, kr[kE - 1], 1);
        const float knext0 = __shfl_down_sync(0xffffffffu, kr[0], 1);
        bool risky = false, anytie = false, nan = false;
        irregular = false;
        gerr = false;
#pragma unroll
        for (int r = 0; r < kE; ++r) {
            const int p = lane * kE + r;
            if (p >= nloop) continue;
            const int cp = r == 0 ? cprev0 : cc[r - 1];
            const float kp = r == 0 ? kprev0 : kr[r - 1];
            const float kn = r == kE - 1 ? knext0 : kr[r + 1];
            const bool tl = p >= 1 && kr[r] == kp;
            const bool tr = p + 1 < nloop && kr[r] == kn;
            const bool split = cc[r] > cp;
            if (split && (tl || tr)) risky = true;
            anytie |= tl;
            nan |= (kr[r] != kr[r]);
            if (cc[r] - cp >= 2) irregular = true;
            if (cp >= ng) gerr = true;
        }
        risky = __any_sync(0xffffffffu, risky);
        anytie = __any_sync(0xffffffffu, anytie);
        nan = __any_sync(0xffffffffu, nan);
        irregular = __any_sync(0xffffffffu, irregular);
        gerr = __any_sync(0xffffffffu, gerr);
        if (attempt == 0) {
            dg.sort_passes += (lane == 0);
            dg.tie_passes += (lane == 0 && anytie);
        }
        if (exact || !(risky || nan || (B.strict_ties && anytie))) break;
        // exact path: the reference heapsort on the elements in nloop order
        exact = true;
        dg.exact_passes += (lane == 0);
        for (int e = lane; e < nloop; e += 32) {
            keys_s[e] = key_of(e);
            idx_s[e] = (short)(e + 1);
        }
        __syncwarp();
        if (lane == 0) heapsort_sort2g(nloop, keys_s, idx_s);
        __syncwarp();
#pragma unroll
        for (int r = 0; r < kE; ++r) {
            const int p = lane * kE + r;
            kr[r] = p < nloop ? keys_s[p] : __int_as_float(0x7f800000);
            ir[r] = p < nloop ? (int)idx_s[p] - 1 : p;
        }
        __syncwarp();
    }
    if (gerr) atomicOr(B.status, kStGord);

    // publish the sorted sequence
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        const int p = lane * kE + r;
        if (p < nloop) {
            keys_s[p] = kr[r];
            idx_s[p] = (short)ir[r];
        }
    }
    if (lane < kMaxNg) splitpos[lane] = -1;
    __syncwarp();
    if (dbg_perm) {
        for (int p = lane; p < nloop; p += 32) dbg_perm[p] = idx_s[p];
    }

    if (irregular) {
        // sequential rankg walk (rankg.f:118-152) by lane 0
        dg.irregular += (lane == 0);
        if (lane == 0) {
            for (int b = 0; b < ng; ++b) {
                kg[b] = 0.0f;
                for (int c = 0; c < P.ncol; ++c) colN[c * kMaxNg + b] = 0.0f;
            }
            int ig = 0;
            double sum = 0.0, gprev = 0.0;
            for (int p = 0; p < nloop; ++p) {
                const int e = idx_s[p], i = e / ng, j = e - (e / ng) * ng;
                const float c = keys_s[p];
                const float w = __fmul_rn(delg[i], delg[j]);
                const double gcur = __dadd_rn(gprev, (double)w);
                if (ig >= ng) { atomicOr(B.status, kStGord); break; }
                if (gcur < g_ord[ig + 1]) {
                    kg[ig] = __fadd_rn(kg[ig], __fmul_rn(c, w));
                    for (int cc2 = 0; cc2 < P.ncol; ++cc2)
                        colN[cc2 * kMaxNg + ig] = __fadd_rn(colN[cc2 * kMaxNg + ig],
                            __fmul_rn(elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP), w));
                    sum = __dadd_rn(sum, (double)w);
                } else {
                    const double frac = __ddiv_rn(__dsub_rn(g_ord[ig + 1], gprev), __dsub_rn(gcur, gprev));
                    const float sf = __double2float_rn(frac);
                    kg[ig] = __fadd_rn(kg[ig], __fmul_rn(__fmul_rn(sf, c), w));
                    for (int cc2 = 0; cc2 < P.ncol; ++cc2)
                        colN[cc2 * kMaxNg + ig] = __fadd_rn(colN[cc2 * kMaxNg + ig],
                            __fmul_rn(__fmul_rn(sf, elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP)), w));
                    sum = __dadd_rn(sum, __dmul_rn(frac, (double)w));
                    const float fs = __double2float_rn(sum);
                    kg[ig] = __fdiv_rn(kg[ig], fs);
                    for (int cc2 = 0; cc2 < P.ncol; ++cc2)
                        colN[cc2 * kMaxNg + ig] = __fdiv_rn(colN[cc2 * kMaxNg + ig], fs);
                    if (dbg_split) dbg_split[ig] = (int16_t)p;
                    ig = ig + 1;
                    sum = __dmul_rn(__dsub_rn(1.0, frac), (double)w);
                    if (ig < ng) {
                        const float sr = __double2float_rn(__dsub_rn(1.0, frac));
                        kg[ig] = __fmul_rn(__fmul_rn(sr, c), w);
                        for (int cc2 = 0; cc2 < P.ncol; ++cc2)
                            colN[cc2 * kMaxNg + ig] =
                                __fmul_rn(__fmul_rn(sr, elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP)), w);
                    }
                }
                gprev = gcur;
            }
            if (ig == ng - 1) {
                const float fs = __double2float_rn(sum);
                kg[ig] = __fdiv_rn(kg[ig], fs);
                for (int cc2 = 0; cc2 < P.ncol; ++cc2) colN[cc2 * kMaxNg + ig] = __fdiv_rn(colN[cc2 * kMaxNg + ig], fs);
            }
        }
        __syncwarp();
        return;
    }

    // regular walk: publish split positions and fractions
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        const int p = lane * kE + r;
        if (p >= nloop) continue;
        const int cp = r == 0 ? cprev0 : cc[r - 1];
        if (cc[r] > cp) {
            const double gp = r == 0 ? gprev0 : gd[r - 1];
            splitpos[cp] = p;
            splitfrac[cp] = __ddiv_rn(__dsub_rn(g_ord[cp + 1], gp), __dsub_rn(gd[r], gp));
        }
    }
    // c_last = c(nloop-1)
    const int last_lane = (nloop - 1) / kE, last_r = (nloop - 1) - ((nloop - 1) / kE) * kE;
    int my_last = 0;
#pragma unroll
    for (int r = 0; r < kE; ++r)
        if (r == last_r) my_last = cc[r];
    const int c_last = __shfl_sync(0xffffffffu, my_last, last_lane);
    __syncwarp();
    if (dbg_split && lane < ng) dbg_split[lane] = (short)splitpos[lane];

    // one lane per bin: sums in the reference's order (rankg.f:118-146)
    const int b = lane;
    if (b < ng) {
        float k = 0.0f;
        float cs[kMaxCols];
#pragma unroll
        for (int c = 0; c < kMaxCols; ++c) cs[c] = 0.0f;
#define RTB_FOR_COL(c2) _Pragma("unroll") for (int c2 = 0; c2 < kMaxCols; ++c2) if (c2 < P.ncol)
        if (b <= c_last && (b < ng)) {
            double sum = 0.0;
            int p = 0;
            if (b > 0) {
                const int s = splitpos[b - 1];
                const double frac = splitfrac[b - 1];
                const int e = idx_s[s], i = e / ng, j = e - (e / ng) * ng;
                const float c = keys_s[s], w = __fmul_rn(delg[i], delg[j]);
                const float sr = __double2float_rn(__dsub_rn(1.0, frac));
                k = __fmul_rn(__fmul_rn(sr, c), w);
                RTB_FOR_COL(cc2)
                    cs[cc2] = __fmul_rn(__fmul_rn(sr, elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP)), w);
                sum = __dmul_rn(__dsub_rn(1.0, frac), (double)w);
                p = s + 1;
            }
            const bool closes = b < c_last;
            const int pend = closes ? splitpos[b] : nloop;   // exclusive end of whole elements
            for (; p < pend; ++p) {
                const int e = idx_s[p], i = e / ng, j = e - (e / ng) * ng;
                const float c = keys_s[p], w = __fmul_rn(delg[i], delg[j]);
                k = __fadd_rn(k, __fmul_rn(c, w));
                RTB_FOR_COL(cc2)
                    cs[cc2] = __fadd_rn(cs[cc2], __fmul_rn(elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP), w));
                sum = __dadd_rn(sum, (double)w);
            }
            if (closes) {
                const int s = splitpos[b];
                const double frac = splitfrac[b];
                const int e = idx_s[s], i = e / ng, j = e - (e / ng) * ng;
                const float c = keys_s[s], w = __fmul_rn(delg[i], delg[j]);
                const float sf = __double2float_rn(frac);
                k = __fadd_rn(k, __fmul_rn(__fmul_rn(sf, c), w));
                RTB_FOR_COL(cc2)
                    cs[cc2] = __fadd_rn(cs[cc2], __fmul_rn(__fmul_rn(sf, elem_grad(P, S, cc2, i, j, k1, k2, dk1, dk2, colP)), w));
                sum = __dadd_rn(sum, __dmul_rn(frac, (double)w));
                const float fs = __double2float_rn(sum);
                k = __fdiv_rn(k, fs);
                RTB_FOR_COL(cc2) cs[cc2] = __fdiv_rn(cs[cc2], fs);
            } else if (b == ng - 1) {
                const float fs = __double2float_rn(sum);
                k = __fdiv_rn(k, fs);
                RTB_FOR_COL(cc2) cs[cc2] = __fdiv_rn(cs[cc2], fs);
            }
        }
        kg[b] = k;
        RTB_FOR_COL(cc2) colN[cc2 * kMaxNg + b] = cs[cc2];
#undef RTB_FOR_COL
    }
    __syncwarp();
}

// Planck function and its temperature derivative in FP32
// (planck_wave.f / planckg_wave.f; c1, c2 as the reference's REAL literals).
__device__ __forceinline__ void planck_fp32(int ispace, float vwave, float T, float& B, float& dBdT) {
    const float c1 = 1.1911e-12f, c2 = 1.439f;
    float y, a;
    if (ispace == 0) { y = vwave; a = c1 * y * y * y; }
    else { y = 1e4f / vwave; a = c1 * y * y * y * y * y / 1e4f; }
    if (y == 0.0f) { B = 0.0f; dBdT = 0.0f; return; }
    const float x = c2 * y / T;
    const float em1 = expm1f(x);
    B = a / em1;
    // dB/dT = B * (x/T) * e^x/(e^x-1)
    dBdT = B * (x / T) * ((em1 + 1.0f) / em1);
}

}  // namespace

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 2)
fwd_kernel(BatchDev B, int Lmax, int nsw_max, int ncol_max, int nlmax_max, int npath_max) {
    extern __shared__ __align__(16) char smem[];
    const Layout Lo = make_layout(B.ng, Lmax, nsw_max, ncol_max, nlmax_max, npath_max);
    const WarpOff wo = warp_off(ncol_max);
    const PathOff po = path_off(nlmax_max, B.ng, nsw_max);
    double* g_ord = (double*)(smem + Lo.off_gord);
    float* delg = (float*)(smem + Lo.off_delg);
    float* tau_s = (float*)(smem + Lo.off_tau);
    float* dtau_s = (float*)(smem + Lo.off_dtau);
    char* region = smem + Lo.off_region;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ng = B.ng;
    for (int i = tid; i <= ng; i += kThreads) g_ord[i] = B.g_ord[i];
    for (int i = tid; i < ng; i += kThreads) delg[i] = B.delg[i];
    Diag dg{0, 0, 0, 0};
    __syncthreads();

    for (int64_t item = blockIdx.x; item < B.nitems; item += gridDim.x) {
        // locate the spectrum of this item
        int lo = 0, hi = B.nspec - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (B.item_start[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int sidx = lo;
        __shared__ SpecDev S_sh;
        {
            const int* src = (const int*)(B.spec + sidx);
            int* dst = (int*)&S_sh;
            for (int i = tid; i < (int)(sizeof(SpecDev) / sizeof(int)); i += kThreads) dst[i] = src[i];
        }
        __syncthreads();
        const SpecDev& S = S_sh;
        const int iw = (int)(item - B.item_start[sidx]);
        const int64_t iw_glob = S.wave_off + iw;
        const WaveDev W = B.wave[iw_glob];
        const int nsw = S.nsw, ncol = S.ncol;

        // ---------------- stage A: layers --------------------------------
        char* wsm = region + warp * Lo.warp_bytes;
        float* colA = (float*)(wsm + wo.colA);
        float* colB = (float*)(wsm + wo.colB);
        float* k1s = (float*)(wsm + wo.k1);
        float* k2s = (float*)(wsm + wo.k2);
        float* dk1s = (float*)(wsm + wo.dk1);
        float* dk2s = (float*)(wsm + wo.dk2);
        float* kgs = (float*)(wsm + wo.kg);
        for (int l = warp; l < S.nlayer; l += kWarps) {
            const int64_t il_glob = S.lay_off + l;
            const LayerDev L = B.lay[il_glob];
            float dtc[kMaxSw];
            const float taucon = continuum(B, S, L, W, iw_glob, il_glob, dtc);
            const float* amo = B.amo + S.lg_off + (int64_t)l * S.ngas;
            const int64_t* slices = B.wg_slice + S.wg_off + (int64_t)iw * S.ngas;
            float* colP = colA;
            float* colN = colB;
            float kgv;   // lane value of the running k-distribution
            if (S.ngas == 1) {
                float k0, d0;
                get_kg_lane(B, slices[0], L, lane, k0, d0);
                const float a0 = amo[0];
                kgv = __fmul_rn(k0, a0);
                if (lane < ng)
                    for (int c = 0; c < ncol; ++c)
                        colN[c * kMaxNg + lane] = S.col_gas[c] == S.ngas ? __fmul_rn(d0, a0) : k0;
                float* t = colP; colP = colN; colN = t;
            } else {
                float k1v, d1v;
                get_kg_lane(B, slices[0], L, lane, k1v, d1v);
                kgv = 0.0f;
                for (int ig = 1; ig < S.ngas; ++ig) {
                    const bool first = ig == 1;
                    float k2v, d2v;
                    get_kg_lane(B, slices[ig], L, lane, k2v, d2v);
                    const float a2 = amo[ig];
                    const float a1 = first ? amo[0] : 1.0f;
                    const float k1e = first ? k1v : kgv;
                    const bool z1 = __shfl_sync(0xffffffffu, k1e, ng - 1) == 0.0f;
                    const bool z2 = __shfl_sync(0xffffffffu, k2v, ng - 1) == 0.0f;
                    int16_t* dp = nullptr;
                    int16_t* dsp = nullptr;
                    if (B.dbg_perm && sidx == 0) {
                        const int64_t rec = ((int64_t)iw * S.nlayer + l) * (S.ngas - 1) + (ig - 1);
                        dp = B.dbg_perm + rec * ng * ng;
                        dsp = B.dbg_split + rec * ng;
                        for (int p = lane; p < ng * ng; p += 32) dp[p] = -1;
                        if (lane < ng) dsp[lane] = -1;
                    }
                    if (z1) {                       // noverlapg.f:88-97 / :152-162
                        if (lane < ng) {
                            for (int c = 0; c < ncol; ++c) {
                                const int g = S.col_gas[c];
                                float v;
                                if (g == S.ngas) v = __fmul_rn(d2v, a2);
                                else if (g == ig) v = k2v;
                                else if (g < ig) v = 0.0f;
                                else v = colP[c * kMaxNg + lane];
                                colN[c * kMaxNg + lane] = v;
                            }
                        }
                        kgv = __fmul_rn(k2v, a2);
                    } else if (z2) {                // noverlapg.f:99-108 / :164-173
                        if (lane < ng) {
                            for (int c = 0; c < ncol; ++c) {
                                const int g = S.col_gas[c];
                                float v;
                                if (first) {
                                    if (g == S.ngas) v = __fmul_rn(d1v, a1);
                                    else if (g == 0) v = k1v;
                                    else if (g == 1) v = 0.0f;
                                    else v = 0.0f;
                                } else {
                                    if (g == ig) v = 0.0f;
                                    else v = colP[c * kMaxNg + lane];   // T column unchanged, earlier gases kept
                                }
                                colN[c * kMaxNg + lane] = v;
                            }
                        }
                        kgv = first ? __fmul_rn(k1v, a1) : kgv;
                    } else {
                        // stage the operands for arbitrary-lane access
                        if (lane < ng) {
                            k1s[lane] = k1e;
                            k2s[lane] = k2v;
                            float d1e = d1v;
                            if (!first) {
                                d1e = 0.0f;
                                for (int c = 0; c < ncol; ++c)
                                    if (S.col_gas[c] == S.ngas) d1e = colP[c * kMaxNg + lane];
                            }
                            dk1s[lane] = d1e;
                            dk2s[lane] = d2v;
                        }
                        __syncwarp();
                        PassCtx P;
                        P.ng = ng; P.nloop = ng * ng; P.ncol = ncol; P.first = first; P.igas = ig;
                        P.a1 = a1; P.a2 = a2;
                        sort_pass(B, S, P, wsm, wo, g_ord, delg, lane, dg, colP, colN, dp, dsp);
                        kgv = lane < ng ? kgs[lane] : 0.0f;
                    }
                    __syncwarp();
                    float* t = colP; colP = colN; colN = t;
                    __syncwarp();
                }
            }
            // tau and dtau/dq per g (cirsradg_wave.f:744-790)
            if (lane < ng) {
                tau_s[l * ng + lane] = __fadd_rn(taucon, kgv);
#pragma unroll
                for (int s = 0; s < kMaxSw; ++s) {
                    if (s >= nsw) continue;
                    const int c = S.col_of_param[s];
                    float v = dtc[s];
                    if (c >= 0) {
                        const float col = colP[c * kMaxNg + lane];
                        const float dkdql = S.col_gas[c] == S.ngas ? col : __fmul_rn(col, 1.0e-20f);
                        v = __fadd_rn(v, dkdql);
                    }
                    dtau_s[((size_t)l * nsw + s) * ng + lane] = v;
                }
            }
            __syncwarp();
        }
        __syncthreads();

        // ---------------- stage B: paths ---------------------------------
        for (int p = warp; p < S.npath; p += kWarps) {
            char* ps = region + p * Lo.path_bytes;
            float* drdt = (float*)(ps + po.drdt);
            float* trd = (float*)(ps + po.trd);
            float* bb = (float*)(ps + po.bb);
            float* dbdt = (float*)(ps + po.dbdt);
            float* rad = (float*)(ps + po.rad);
            float* gts = (float*)(ps + po.gts);
            const int nlays = S.nlayin[p], im = S.imod[p];
            const int* layinc = B.p_layinc + S.path_off + (int64_t)p * S.nlmax;
            const float* scale = B.p_scale + S.path_off + (int64_t)p * S.nlmax;
            const float* emt = B.p_emtemp + S.path_off + (int64_t)p * S.nlmax;
            if (im == 3) {
                for (int j = lane; j < nlays; j += 32) planck_fp32(S.ispace, W.vwave, emt[j], bb[j], dbdt[j]);
            }
            __syncwarp();
            if (lane < ng) {
                const int g = lane;
                if (im == 3) {
                    float tr = 1.0f, R = 0.0f;
                    for (int j = 0; j < nlays; ++j) {
                        const float tau = tau_s[layinc[j] * ng + g] * scale[j];
                        const float td = -expm1f(-tau) * tr;
                        const float trn = tr * expf(-tau);
                        R = fmaf(bb[j], td, R);
                        drdt[j * ng + g] = trn;     // transmission to the top of layer j's bottom
                        trd[j * ng + g] = td;
                        tr = trn;
                    }
                    // surface term unless the path is a limb path (cirsradg_wave.f:991-1025)
                    float Ssum = 0.0f, gt = 0.0f;
                    if ((S.nonlimb_mask >> p) & 1) {
                        const float rg = S.tsurf_pos ? W.radground_s : bb[nlays - 1];
                        const float gg = S.tsurf_pos ? W.gradground_s : dbdt[nlays - 1];
                        R = fmaf(rg, tr, R);
                        gt = tr * gg;
                        Ssum = rg * tr;
                    }
                    for (int j = nlays - 1; j >= 0; --j) {
                        const float trj = drdt[j * ng + g];
                        drdt[j * ng + g] = bb[j] * trj - Ssum;   // dR/dtau_j
                        Ssum = fmaf(bb[j], trd[j * ng + g], Ssum);
                    }
                    rad[g] = R;
                    gts[g] = gt;
                } else {
                    float tsum = 0.0f;
                    for (int j = 0; j < nlays; ++j) tsum = tsum + tau_s[layinc[j] * ng + g] * scale[j];
                    float y = fmaxf(-tsum, -500.0f);
                    if (y >= 88.7f) y = 88.7f;
                    const float e = (float)exp((double)y);
                    float out, dr;
                    // IMOD 0: dcoutdq = -tau*T*dtau/dq; IMOD 1: tau*(1-A)*dtau/dq with
                    // 1-A formed as T itself (no cancellation when T < 2^-25)
                    if (im == 0) { out = e; dr = -tsum * e; }
                    else { out = 1.0f - e; dr = tsum * e; }
                    for (int j = 0; j < nlays; ++j) { drdt[j * ng + g] = dr; trd[j * ng + g] = 0.0f; }
                    rad[g] = out;
                    gts[g] = 0.0f;
                }
            }
        }
        __syncthreads();

        // ---------------- stage C: g-quadrature of dR/dq -----------------
        for (int p = 0; p < S.npath; ++p) {
            char* ps = region + p * Lo.path_bytes;
            const float* drdt = (const float*)(ps + po.drdt);
            const float* trd = (const float*)(ps + po.trd);
            const float* dbdt = (const float*)(ps + po.dbdt);
            float* dq = (float*)(ps + po.dq);
            const int nlays = S.nlayin[p];
            const int* layinc = B.p_layinc + S.path_off + (int64_t)p * S.nlmax;
            const float* scale = B.p_scale + S.path_off + (int64_t)p * S.nlmax;
            const bool em = S.imod[p] == 3;
            for (int t = tid; t < nlays * nsw; t += kThreads) {
                const int j = t / nsw, s = t - (t / nsw) * nsw;
                const int l = layinc[j];
                const float sc = scale[j];
                const float* dt = dtau_s + ((size_t)l * nsw + s) * ng;
                const float* dr = drdt + j * ng;
                float acc = 0.0f;
                if (em && s == S.sw_T) {
                    const float dB = dbdt[j];
                    const float* td = trd + j * ng;
                    for (int g = 0; g < ng; ++g)
                        acc = fmaf(delg[g], fmaf(dr[g], dt[g] * sc, td[g] * dB), acc);
                } else {
                    for (int g = 0; g < ng; ++g) acc = fmaf(delg[g], dr[g] * (dt[g] * sc), acc);
                }
                dq[j * nsw + s] = acc;
            }
        }
        __syncthreads();

        // ---------------- stage D: map to the state vector ---------------
        for (int p = 0; p < S.npath; ++p) {
            char* ps = region + p * Lo.path_bytes;
            const float* dq = (const float*)(ps + po.dq);
            const int* cp = B.map_colptr + S.map_off + (int64_t)p * (S.nv + 1);
            for (int iv = tid; iv < S.nv; iv += kThreads) {
                float acc = 0.0f;
                for (int e = cp[iv]; e < cp[iv + 1]; ++e) acc = fmaf(dq[B.map_row[e]], B.map_val[e], acc);
                B.gradients[S.jac_off + ((int64_t)p * S.nv + iv) * S.nwave + iw] = acc;
            }
            if (tid == 0) {
                const float* rad = (const float*)(ps + po.rad);
                const float* gts = (const float*)(ps + po.gts);
                float o = 0.0f, gt = 0.0f;
                for (int g = 0; g < ng; ++g) {
                    o = fmaf(rad[g], delg[g], o);
                    gt = fmaf(gts[g], delg[g], gt);
                }
                B.calcout[S.out_off + (int64_t)p * S.nwave + iw] = o;
                if (B.gradtsurf) B.gradtsurf[S.out_off + (int64_t)p * S.nwave + iw] = gt;
            }
        }
        __syncthreads();
    }
    if (lane == 0) {
        if (dg.sort_passes) atomicAdd(B.counters + 0, dg.sort_passes);
        if (dg.tie_passes) atomicAdd(B.counters + 1, dg.tie_passes);
        if (dg.exact_passes) atomicAdd(B.counters + 2, dg.exact_passes);
        if (dg.irregular) atomicAdd(B.counters + 3, dg.irregular);
    }
}

// host-side helpers exported to host.cu
int fwd_smem_bytes(int ng, int Lmax, int nsw, int ncol, int nlmax, int npath) {
    return make_layout(ng, Lmax, nsw, ncol, nlmax, npath).total;
}

cudaError_t launch_fwd(const BatchDev& B, int Lmax, int nsw, int ncol, int nlmax, int npath, int grid,
                       cudaStream_t st) {
    const int smem = fwd_smem_bytes(B.ng, Lmax, nsw, ncol, nlmax, npath);
    cudaError_t e = cudaFuncSetAttribute(fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    fwd_kernel<<<grid, kThreads, smem, st>>>(B, Lmax, nsw, ncol, nlmax, npath);
    return cudaGetLastError();
}

}  // namespace rtb
