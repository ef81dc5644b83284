// fwd_kernel.cu -- B200 forward model + analytic Jacobian of the correlated-k
// thermal-emission path (radtran/cirsradg/cirsradg_wave.f, IMOD 0/1/3) fused
// with map2pro/map2xvec (radtran/cirsradg/map2pro.f, map2xvec.f).
//
// One CTA (8 warps) owns one (spectrum, wavenumber) work item at a time and
// loops over items grid-stride (persistent grid, one scratch slot per CTA).
//   A  per layer (one warp each): k-table interpolation of every gas
//      (get_kg.f:306-378), continuum optical depth and its derivatives
//      (nciacon.f, dust, Rayleigh: cirsradg_wave.f:510-691) and the random
//      overlap of the gas k-distributions (noverlapg.f/rankg.f).  The NG*NG
//      combined keys k1(i)*a1 + k2(j)*a2 form NG sorted rows when both
//      distributions are monotone in g (every k-distribution is), so they are
//      sorted by a stable warp merge sort of those rows; otherwise by a warp
//      bitonic network.  The FP64 cumulative weights come from a warp scan
//      (exact in any order), and the rebinning sums of rankg.f:118-146 run as
//      (bin, column) tasks in the reference's order.  tau and dtau/dq per g
//      go to the CTA's scratch slot (L2-resident).
//   B  per path (one warp, one lane per g): Planck, transmissions, radiance
//      and dR/dtau of every layer by a suffix sum, which replaces the O(L^2)
//      recurrence of cirsradg_wave.f:954-978 by O(L) exact algebra.
//   C  g-quadrature of the layer Jacobian (cirsradg_wave.f:1240-1286).
//   D  layer -> state vector through a precomputed sparse map
//      (map2pro o map2xvec), packed as cirsrtfg_wave.f:425-446.
//
// Bit-exactness of the g-bin assignment: every operation that feeds a sort
// key or a bin boundary is an explicitly rounded IEEE operation in the
// reference's order (no FMA contraction); the cumulative weights are FP64
// sums of FP32 products >= 2^-28, exact in any order; a pass whose bin
// boundaries fall inside a run of tied keys (where the reference's unstable
// heapsort order decides the bins) takes that heapsort (sort2g.f) in-kernel.
#include <cuda_runtime.h>
#include <stdint.h>

#include "detexp.cuh"
#include "rtb_common.h"

namespace rtb {

namespace {

constexpr int kN = 484;              // largest NG*NG (NG <= 22)
constexpr unsigned kFull = 0xffffffffu;
// order-preserving map of a float onto uint32 (-0 folded onto +0 first)
__device__ __forceinline__ unsigned fkey(float f) {
    unsigned u = __float_as_uint(__fadd_rn(f, 0.0f));
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(unsigned k) {
    unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// NR heapsort of radtran/cirsradg/sort2g.f:1-52 on shared memory (one thread);
// ra/ib hold RA(1..n)/IB(1..n) at ra[0..n-1].
__device__ __noinline__ void heapsort_sort2g(int n, float* ra0, unsigned short* ib0) {
    if (n < 2) return;
    float* RA = ra0 - 1;
    unsigned short* IB = ib0 - 1;
    int L = n / 2 + 1, IR = n;
    float RRA;
    unsigned short IRB;
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

// The same heapsort on 64-bit words (float bits of RA << 32 | IB), one thread:
// the comparisons are the float comparisons of sort2g.f (RA(J) < RA(J+1),
// RRA < RA(J)), so the words end in exactly the order of heapsort_sort2g.
// RA and IB move as one word, and the sift-down loads the four grandchildren
// while it compares the two children, so that no shared-memory load is on
// the critical path of a level.
__device__ __forceinline__ float wkey(unsigned long long w) { return __uint_as_float((unsigned)(w >> 32)); }
__device__ __noinline__ void heapsort_words(int n, unsigned long long* W0) {
    if (n < 2) return;
    unsigned long long* W = W0 - 1;            // W[1..n]
    int L = n / 2 + 1, IR = n;
    for (;;) {
        unsigned long long R;
        if (L > 1) {
            L = L - 1;
            R = W[L];
        } else {
            R = W[IR];
            W[IR] = W[1];
            IR = IR - 1;
            if (IR == 1) {
                W[1] = R;
                return;
            }
        }
        const float kR = wkey(R);
        int I = L, J = L + L;
        if (J <= IR) {
            unsigned long long c0 = W[J], c1 = W[J < IR ? J + 1 : J];
            for (;;) {
                // grandchildren of J and J + 1 (clamped into 1..IR; used only when in range)
                const int G = J + J;
                const unsigned long long g0 = W[G <= IR ? G : IR], g1 = W[G + 1 <= IR ? G + 1 : IR];
                const unsigned long long g2 = W[G + 2 <= IR ? G + 2 : IR], g3 = W[G + 3 <= IR ? G + 3 : IR];
                int Jc = J;
                unsigned long long c = c0;
                if (J < IR && wkey(c0) < wkey(c1)) {
                    Jc = J + 1;
                    c = c1;
                }
                if (!(kR < wkey(c))) break;
                W[I] = c;
                I = Jc;
                J = Jc + Jc;
                if (J > IR) break;
                c0 = Jc == G / 2 ? g0 : g2;
                c1 = Jc == G / 2 ? g1 : g3;
            }
        }
        W[I] = R;
    }
}

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }

// bytes of one element buffer: the NG rows of 64-bit words with a sentinel
// word on either side of each and one sentinel pair after the last (the
// merge's layout), or the gradient-column tables (6 NG float4), whichever is
// larger, for NG up to 22
constexpr int kNgDev = 22;
constexpr int kGradScratch = 96 * kNgDev;
constexpr int kMergeWords = kN + 2 * kNgDev + 2;
constexpr int kElemBuf = ((8 * kMergeWords > kGradScratch ? 8 * kMergeWords : kGradScratch) + 15) & ~15;
// per-warp scratch sub-offsets (bytes).  bufA and bufB hold the (key,
// element) words of a pass and the merge's levels in turn; the one not
// holding the sorted words then takes the FP64 cumulative weights and the
// gradient-column tables.
struct WarpOff {
    int bufA, bufB, splitfrac, k1, k2, dk1, dk2, kg, splitpos, colA, colB, total;
};
__host__ __device__ inline WarpOff warp_off(int ncol) {
    WarpOff w;
    int o = 0;
    const int nc = ncol > 0 ? ncol : 1;
    // 8 B words (the element buffers); the free one also holds the FP64
    // cumulative weights and, later, the gradient-column tables and partials
    w.bufA = o; o += kElemBuf;
    w.bufB = o; o += kElemBuf;
    w.splitfrac = o; o += 8 * kMaxNg;
    w.k1 = o; o += 4 * kMaxNg;
    w.k2 = o; o += 4 * kMaxNg;
    w.dk1 = o; o += 4 * kMaxNg;
    w.dk2 = o; o += 4 * kMaxNg;
    w.kg = o; o += 4 * kMaxNg;
    w.splitpos = o; o += 4 * kMaxNg;
    w.colA = o; o += 4 * kMaxNg * nc;
    w.colB = o; o += 4 * kMaxNg * nc;
    w.total = align16(o);
    return w;
}
// per-path sub-offsets (stages B-D)
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
    p.total = align16(o);
    return p;
}

constexpr int kMergeLevels = 5;   // merge levels of NG <= 32 rows

struct Layout {
    int warp_bytes, path_bytes, off_gord, off_delg, off_wtab, off_mtab, off_region, total;
};
__host__ __device__ inline Layout make_layout(int ng, int nsw, int ncol, int nlmax, int npath, int warps) {
    Layout Lo;
    Lo.warp_bytes = warp_off(ncol).total;
    Lo.path_bytes = path_off(nlmax, ng, nsw).total;
    int o = 0;
    Lo.off_gord = o; o += 8 * (kMaxNg + 3);
    Lo.off_delg = o; o += 4 * kMaxNg;
    Lo.off_wtab = o; o += 4 * 33 * kNgDev;       // element weights w(i, j) at 33 i + j (rows spread over the banks)
    Lo.off_mtab = o; o += 2 * kMergeLevels * 33;  // lanes' merge ranges
    o = align16(o);
    Lo.off_region = o;
    const int a = warps * Lo.warp_bytes, b = npath * Lo.path_bytes;
    o += a > b ? a : b;
    Lo.total = o;
    return Lo;
}

struct Diag {
    unsigned long long sort_passes, tie_passes, exact_passes, irregular, block_passes;
};

// ---------------------------------------------------------------------------
// get_kg for one gas at one layer: lane g < ng returns k(g), dk/dT(g)
// (get_kg.f:320-378 coincident branch, NaN -> 1e-37 at :443-471).
// RANKK (radtran/cirsradg/rankk.f:34-117) on one thread: REAL cumulative
// ordinates and distribution summed in the reference's order, the `<=` test,
// the split fraction and the ig <= ng guards.  cont/dcont/weight are sorted
// and permuted in place (sort2g heapsort); ico is scratch.
__device__ void rankk_lane(int ng, const float* gw, int nloop, float* cont, float* dcont, float* weight,
                                        unsigned short* ico, float* tmp, float* k_g, float* dkdt) {
    float g_ord[kMaxNg + 1];
    g_ord[0] = 0.0f;
    for (int i = 0; i < ng; ++i) g_ord[i + 1] = __fadd_rn(g_ord[i], gw[i]);
    if (g_ord[ng] < 1.0f) g_ord[ng] = 1.0f;
    for (int i = 0; i < nloop; ++i) ico[i] = (unsigned short)i;
    heapsort_sort2g(nloop, cont, ico);
    for (int i = 0; i < nloop; ++i) tmp[i] = weight[ico[i]];
    for (int i = 0; i < nloop; ++i) weight[i] = tmp[i];
    for (int i = 0; i < nloop; ++i) tmp[i] = dcont[ico[i]];
    for (int i = 0; i < nloop; ++i) dcont[i] = tmp[i];
    // gdist(I) in tmp[I], I = 0..nloop
    tmp[0] = 0.0f;
    tmp[1] = weight[0];
    for (int i = 2; i <= nloop; ++i) tmp[i] = __fadd_rn(weight[i - 1], tmp[i - 1]);
    for (int i = 0; i < ng; ++i) {
        k_g[i] = 0.0f;
        dkdt[i] = 0.0f;
    }
    int ig = 1;
    float sum = 0.0f;
    for (int I = 1; I <= nloop; ++I) {
        const float c = cont[I - 1], dc = dcont[I - 1], w = weight[I - 1];
        if (ig <= ng && tmp[I] <= g_ord[ig]) {
            k_g[ig - 1] = __fadd_rn(k_g[ig - 1], __fmul_rn(c, w));
            dkdt[ig - 1] = __fadd_rn(dkdt[ig - 1], __fmul_rn(dc, w));
            sum = __fadd_rn(sum, w);
        } else {
            if (ig > ng) continue;      // the reference writes past NG here; those slots are never read
            const float frac = __fdiv_rn(__fsub_rn(g_ord[ig], tmp[I - 1]), __fsub_rn(tmp[I], tmp[I - 1]));
            k_g[ig - 1] = __fadd_rn(k_g[ig - 1], __fmul_rn(__fmul_rn(frac, c), w));
            dkdt[ig - 1] = __fadd_rn(dkdt[ig - 1], __fmul_rn(__fmul_rn(frac, dc), w));
            sum = __fadd_rn(sum, __fmul_rn(frac, w));
            k_g[ig - 1] = __fdiv_rn(k_g[ig - 1], sum);
            dkdt[ig - 1] = __fdiv_rn(dkdt[ig - 1], sum);
            ig = ig + 1;
            if (ig <= ng) {
                const float rest = __fsub_rn(1.0f, frac);
                sum = __fmul_rn(rest, w);
                k_g[ig - 1] = __fmul_rn(__fmul_rn(rest, c), w);
                dkdt[ig - 1] = __fmul_rn(__fmul_rn(rest, dc), w);
            }
        }
    }
    if (ig == ng) {
        k_g[ig - 1] = __fdiv_rn(k_g[ig - 1], sum);
        dkdt[ig - 1] = __fdiv_rn(dkdt[ig - 1], sum);
    }
}

// X and dX/dT of the four (P, T) corners of one g (get_kg.f:355-365 and
// 413-423): bilinear in (ln p, T) for a table with one temperature grid; for
// TEMP2 tables (NT < 0) linear in T along each pressure row with its own
// weight, then linear in ln p
template <bool t2>
__device__ __forceinline__ void corners(const LayerDev& L, float Y1, float Y2, float Y3, float Y4, float& X,
                                        float& DXDT) {
    const float U = L.u, V = L.v;
    const float a = __fsub_rn(1.0f, V), b = __fsub_rn(1.0f, U);
    if (t2) {
        const float X1 = __fadd_rn(__fmul_rn(b, Y1), __fmul_rn(U, Y4));
        const float X2 = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, L.u2), Y2), __fmul_rn(L.u2, Y3));
        X = __fadd_rn(__fmul_rn(a, X1), __fmul_rn(V, X2));
        DXDT = __fadd_rn(__fmul_rn(__fmul_rn(a, __fadd_rn(-Y1, Y4)), L.dudt),
                         __fmul_rn(__fmul_rn(V, __fadd_rn(-Y2, Y3)), L.dudt2));
        return;
    }
    X = __fmul_rn(__fmul_rn(a, b), Y1);
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(V, b), Y2));
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(V, U), Y3));
    X = __fadd_rn(X, __fmul_rn(__fmul_rn(a, U), Y4));
    float D = -__fmul_rn(a, Y1);
    D = __fsub_rn(D, __fmul_rn(V, Y2));
    D = __fadd_rn(D, __fmul_rn(V, Y3));
    D = __fadd_rn(D, __fmul_rn(a, Y4));
    DXDT = __fmul_rn(D, L.dudt);
}

// linear interpolation of one g of one table slice (no logarithms: the
// non-coincident branch of get_kg.f:396-420)
template <bool t2>
__device__ __forceinline__ void interp_lin(const float* t, const LayerDev& L, int g, float& X, float& DXDT) {
    const float Y1 = __ldg(t + L.ioff[0] + g), Y2 = __ldg(t + L.ioff[1] + g);
    const float Y3 = __ldg(t + L.ioff[2] + g), Y4 = __ldg(t + L.ioff[3] + g);
    corners<t2>(L, Y1, Y2, Y3, Y4, X, DXDT);
}

// get_kg for a wavenumber between two table points (get_kg.f:380-438):
// 2 NG linearly interpolated values, weighted (1 - w2) delg and w2 delg,
// rank-rebinned by rankk on lane 0.  scr: per-warp shared scratch of at least
// 8 * kMaxNg floats + 2 * kMaxNg shorts.  Called by the whole warp.
template <bool t2>
__device__ void get_kg_lane_nc(const BatchDev& B, int64_t slice, float w1, float w2, const LayerDev& L, int lane,
                               float* scr,
                               float& k, float& dk) {
    const int ng = B.ng;
    float* cont = scr;
    float* dcont = scr + 2 * kMaxNg;
    float* fac = scr + 4 * kMaxNg;
    float* tmp = scr + 6 * kMaxNg;                  // 2 ng + 1 entries
    float* kg = scr + 8 * kMaxNg + 2;
    float* dkg = kg + kMaxNg;
    unsigned short* ico = (unsigned short*)(dkg + kMaxNg);
    k = 0.0f;
    dk = 0.0f;
    if (slice < 0) return;
    if (lane < ng) {
        const int64_t step = (int64_t)B.np * B.nt * ng;
        for (int loop = 0; loop < 2; ++loop) {
            float X, D;
            interp_lin<t2>(B.ktab_raw + slice + loop * step, L, lane, X, D);
            cont[loop * ng + lane] = X;
            dcont[loop * ng + lane] = D;
            fac[loop * ng + lane] = __fmul_rn(B.delg[lane], loop ? w2 : w1);
        }
    }
    __syncwarp();
    if (lane == 0) rankk_lane(ng, B.delg, 2 * ng, cont, dcont, fac, ico, tmp, kg, dkg);
    __syncwarp();
    if (lane < ng) {
        k = kg[lane];
        dk = dkg[lane];
        if (k != k) k = 1e-37f;
        if (dk != dk) dk = 1e-37f;
    }
    __syncwarp();
}

template <bool t2, int NGC>
__device__ __forceinline__ void get_kg_lane(const BatchDev& B, int64_t slice, const LayerDev& L, int lane,
                                            float& k, float& dk) {
    k = 0.0f;
    dk = 0.0f;
    if (slice < 0) return;
    const float* raw = B.ktab_raw + slice;
    const float y10 = __ldg(raw + L.ioff[0]), y20 = __ldg(raw + L.ioff[1]);
    const float y30 = __ldg(raw + L.ioff[2]), y40 = __ldg(raw + L.ioff[3]);
    const bool klog = !((y10 <= 0.0f) || (y20 <= 0.0f) || (y30 <= 0.0f) || (y40 <= 0.0f));
    if (lane >= (NGC ? NGC : B.ng)) return;
    const float* t = klog ? (B.ktab_log + slice) : raw;
    const float Y1 = __ldg(t + L.ioff[0] + lane), Y2 = __ldg(t + L.ioff[1] + lane);
    const float Y3 = __ldg(t + L.ioff[2] + lane), Y4 = __ldg(t + L.ioff[3] + lane);
    float X, DXDT;
    corners<t2>(L, Y1, Y2, Y3, Y4, X, DXDT);
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

// E3INTERP (radtran/radtran/e3interp.f:42-75) on the table tabtran | tabe3 |
// egrad (1001 points each): E3 and dE3/dtrans of a transmission, DOUBLE
__device__ __forceinline__ void e3interp_dev(const double* tab, double x, double& e3, double& de3) {
    constexpr int mtab = 1001;
    if (x < 0.0 || x != x) {
        e3 = 0.0;
        de3 = 0.0;
        return;
    }
    const double dtrans = (double)(1.0f / 1000.0f);
    int j = 1 + (int)(x / dtrans);
    if (j >= mtab) j = mtab - 1;
    double f = (x - tab[j - 1]) / dtrans;
    if (f > 1.0) f = 1.0;
    const double* te3 = tab + mtab;
    const double* eg = tab + 2 * mtab;
    e3 = __dadd_rn(__dmul_rn(1.0 - f, te3[j - 1]), __dmul_rn(f, te3[j]));
    de3 = __dadd_rn(__dmul_rn(1.0 - f, eg[j - 1]), __dmul_rn(f, eg[j]));
}

// calc_nlte_t.f:1-45, the emission temperature of a layer at pressure p (atm)
// outside LTE: B(T_nlte) = f B(T) with f = k1 N / (A + k1 N), N the number
// density (inlte = 1), or f = 1e6 p / (1 + 1e6 p) (inlte = 2).  Its IWAVE is
// the wavenumber index in cirsradg_wave.f:933-935, never 0, so planck_wave
// and invplanck_wave take their wavelength branch (y = 1e4 / v) there.
// DOUBLE inside as those two are; REAL factors as calc_nlte_t forms them.
__device__ __noinline__ float nlte_temp(int inlte, float T, float p, float v, float k1, float A) {
    float f;
    if (inlte == 1) {
        const float ntot = __fmul_rn(__fdiv_rn(__fmul_rn(p, 101325.0f), __fmul_rn(1.380658e-23f, T)), 1.0e-6f);
        f = __fdiv_rn(__fmul_rn(k1, ntot), __fadd_rn(A, __fmul_rn(k1, ntot)));
    } else if (inlte == 2) {
        const float x = __fmul_rn(p, 1.0e6f);
        f = __fdiv_rn(x, __fadd_rn(1.0f, x));
    } else {
        return T;
    }
    const double c1 = (double)1.1911e-12f, c2 = (double)1.439f;
    const float y = __fdiv_rn(1e4f, v);
    if (y == 0.0f) return 0.0f;                  // planck_wave = 0, then invplanck_wave(B = 0) = 0
    const float y2 = __fmul_rn(y, y), y4 = __fmul_rn(y2, y2);
    const double a = c1 * (double)__fmul_rn(y4, y) / 1e4;
    const float Bt = __double2float_rn(a / (exp(c2 * (double)y / (double)T) - 1.0));
    const float Bf = __fmul_rn(Bt, f);
    if (Bf == 0.0f || v == 0.0f) return 0.0f;
    const double dv = (double)v, v2 = dv * dv, v4 = v2 * v2;
    return __double2float_rn(c2 * (double)1.0e4f / dv / log((c1 * (double)1.0e16f) / ((double)Bf * (v4 * dv)) + 1.0));
}

// iform = 3 on an IMOD 3 path (cirsradg_wave.f:913-929): the total flux of the
// planet, every term of lane g's radiance and derivatives times x.  Out of
// line, as is path_imod18: the common paths' code stays as compact as it was.
__device__ __noinline__ void scale_path(float x, int nlays, int ng, int g, float* drdt, float* trd, float* rad,
                                        float* gts) {
    rad[g] *= x;
    gts[g] *= x;
    for (int j = 0; j < nlays; ++j) {
        drdt[j * ng + g] *= x;
        trd[j * ng + g] *= x;
    }
}

// IMOD 18, hemispherically integrated emission (cirsradg_wave.f:1116-1225), on
// g-ordinate g of one path:
// R = c sum_j B_j (E3(T_{j-1}) - E3(T_j)) + c E3(T_N) e_s B_s with the vertical
// transmissions T_j in DOUBLE and E3 from e3interp's table, c = 2 pi xfac;
// dR/dtau_j = c (B_j G_j + sum_{m>j} B_m (G_m - G_{m-1})), G_m = E3'(T_m) T_m
// (the reference leaves the surface term out of the derivative).  drdt
// receives dR/dtau_j, trd the factor of dB/dT in the temperature column.
__device__ __noinline__ void path_imod18(const double* e3tab, float xfac18, int nlays, int ng, int g,
                                         const int* layinc, const float* scale, const float* tau_s,
                                         const float* bb, float radground_s, float gradground_s, float* drdt,
                                         float* trd, float* rad, float* gts) {
    const float c = __fmul_rn(__fmul_rn(xfac18, 2.0f), 3.1415927f);
    double tr = 1.0, e3o = 0.5;
    float R = 0.0f;
    for (int j = 0; j < nlays; ++j) {
        const float tau = tau_s[layinc[j] * ng + g] * scale[j];
        tr = tr * exp(-(double)tau);
        double e3n, e3g;
        e3interp_dev(e3tab, tr, e3n, e3g);
        const float d = __double2float_rn(e3o - e3n);
        R = __fadd_rn(R, __fmul_rn(__fmul_rn(c, d), bb[j]));
        trd[j * ng + g] = __fmul_rn(c, d);
        drdt[j * ng + g] = __double2float_rn(e3g) * __double2float_rn(tr);   // G_j
        e3o = e3n;
    }
    const float e3l = __double2float_rn(e3o);
    R = __fadd_rn(R, __fmul_rn(__fmul_rn(c, e3l), radground_s));
    float Ssum = 0.0f;
    for (int j = nlays - 1; j >= 0; --j) {
        const float Gj = drdt[j * ng + g];
        drdt[j * ng + g] = c * fmaf(bb[j], Gj, Ssum);
        if (j > 0) Ssum = fmaf(bb[j], Gj - drdt[(j - 1) * ng + g], Ssum);
    }
    rad[g] = R;
    gts[g] = __fmul_rn(__fmul_rn(c, e3l), gradground_s);
}

// bilinear (wavenumber, temperature) value of one CIA table entry and its
// d/dT (ciaread.f:178-196, fpread_all.f:220-266): REAL, in the reference's
// order; the four corners are at b + stride * (ct + 25 cv) and neighbours
__device__ __forceinline__ void cia_bilinear(const float* kc, int64_t e, int64_t stride, int ct, int cv, float t,
                                             float u, float dudt, float& x, float& dx) {
    const float omt = __fsub_rn(1.0f, t), omu = __fsub_rn(1.0f, u);
    const float a11 = __ldg(kc + e + stride * ((int64_t)ct + 25 * (int64_t)cv));
    const float a12 = __ldg(kc + e + stride * ((int64_t)ct + 25 * ((int64_t)cv + 1)));
    const float a22 = __ldg(kc + e + stride * ((int64_t)ct + 1 + 25 * ((int64_t)cv + 1)));
    const float a21 = __ldg(kc + e + stride * ((int64_t)ct + 1 + 25 * (int64_t)cv));
    x = __fmul_rn(__fmul_rn(omt, omu), a11);
    x = __fadd_rn(x, __fmul_rn(__fmul_rn(t, omu), a12));
    x = __fadd_rn(x, __fmul_rn(__fmul_rn(t, u), a22));
    x = __fadd_rn(x, __fmul_rn(__fmul_rn(omt, u), a21));
    float d = -__fmul_rn(omt, a11);
    d = __fsub_rn(d, __fmul_rn(t, a12));
    d = __fadd_rn(d, __fmul_rn(t, a22));
    d = __fadd_rn(d, __fmul_rn(omt, a21));
    dx = __fmul_rn(d, dudt);
}

// RAYLEIGHA (radtran/scatter/rayleigha.f:1-38): the Rayleigh cross section of
// air at pressure P (atm) and temperature T, REAL arithmetic in its order
__device__ __noinline__ float rayleigha_dev(float v, float P, float T) {
    const float c1 = 8342.12f, c2 = 2406030.0f, c3 = 15997.0f, delta = 0.035f, pi = 3.1415927f, k = 1.37971e-23f;
    float lambda = __fdiv_rn(1e4f, v);
    const float nu2 = __fdiv_rn(1.0f, __fmul_rn(lambda, lambda));
    float m1 = __fadd_rn(__fadd_rn(c1, __fdiv_rn(c2, __fsub_rn(130.0f, nu2))), __fdiv_rn(c3, __fsub_rn(38.9f, nu2)));
    m1 = __fmul_rn(m1, 1e-8f);
    const float P1 = __fmul_rn(P, 1.013e5f), T1 = __fsub_rn(T, 273.15f);
    const float num = __fmul_rn(P1, __fadd_rn(1.0f, __fmul_rn(__fmul_rn(P1, __fsub_rn(61.3f, T1)), 1E-10f)));
    const float xcorr = __fdiv_rn(num, __fmul_rn(96095.4f, __fadd_rn(1.0f, __fmul_rn(0.003661f, T1))));
    m1 = __fmul_rn(m1, xcorr);
    const float Ns = __fdiv_rn(P1, __fmul_rn(k, T));
    lambda = __fmul_rn(lambda, 1e-6f);
    const float x = __fmul_rn(__fmul_rn(Ns, lambda), lambda);
    const float mm = __fmul_rn(m1, __fadd_rn(m1, 2.0f));
    const float temp = __fmul_rn(__fmul_rn(8.0f, __fmul_rn(__fmul_rn(pi, pi), pi)), __fmul_rn(mm, mm));
    const float faniso = __fdiv_rn(__fadd_rn(6.0f, __fmul_rn(3.0f, delta)), __fsub_rn(6.0f, __fmul_rn(7.0f, delta)));
    return __fdiv_rn(__fmul_rn(__fmul_rn(temp, 1e4f), faniso), __fmul_rn(3.0f, __fmul_rn(x, x)));
}

// continuum optical depth of one layer and its active derivatives
// (cirsradg_wave.f:526-691 with nciacon.f:84-310 / ciaread.f:108-198, or for
// flagh2p = 1 nparacon_all.f:160-336 / fpread_all.f:195-266).  Lanes 0..8
// interpolate one CIA table entry each; the sums run on every lane.
template <bool para>
__device__ __forceinline__ float continuum(const BatchDev& B, const SpecDev& S, const LayerDev& L, const WaveDev& W,
                                           int64_t iw_glob, int64_t il_glob, int lane, float (&dtc)[kMaxSw]) {
#pragma unroll
    for (int s = 0; s < kMaxSw; ++s) dtc[s] = 0.0f;
    float taucon = 0.0f;
    for (int k = 0; k < S.ncont; ++k) {
        // this spectrum's [nwave][ncont] and [nlayer][ncont] blocks: the
        // batch's spectra need not share ncont
        const float tau = B.xsec[S.wc_off + (iw_glob - S.wave_off) * S.ncont + k];
        taucon = __fadd_rn(taucon, __fmul_rn(tau, B.cont[S.lc_off + (il_glob - S.lay_off) * S.ncont + k]));
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s < S.nsw && S.isw[s] == S.ngas + 1 + k) dtc[s] = tau;
    }
    float absorb = 0.0f, dab[7] = {0, 0, 0, 0, 0, 0, 0};
    if (para && S.para) {
        // lanes 0, 1: H2-H2 at the para entries j0, j0+1; 2, 3: H2-He; 4..8: the
        // five further pairs of kcia5
        const ParaLayDev PL = B.para_lay[S.para_off + (il_glob - S.lay_off)];
        const ParaWaveDev PW = B.para_wave[S.paraw_off + (iw_glob - S.wave_off)];
        float my_a = 0.0f, my_d = 0.0f;
        if (lane < 9) {
            if (lane < 4) {
                const int e = PL.j0 + ((lane & 1) && !PL.neg ? 1 : 0);
                cia_bilinear(lane < 2 ? B.kh2h2 : B.kh2he, e, B.ipara, PL.ct, PW.cv, PW.t, PL.u, PL.dudt, my_a, my_d);
            } else {
                cia_bilinear(B.kcia5, lane - 4, 5, PL.ct, PW.cv, PW.t, PL.u, PL.dudt, my_a, my_d);
            }
        }
        float v[9], dv[9];
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            v[p] = __shfl_sync(kFull, my_a, p);
            dv[p] = __shfl_sync(kFull, my_d, p);
        }
        float ah2h2, ah2he, dh2dt, dhedt, dh2dfp = 0.0f, dhedfp = 0.0f;
        if (PL.neg) {
            ah2h2 = v[0];
            ah2he = v[2];
            dh2dt = dv[0];
            dhedt = dv[2];
        } else {
            const float f = PL.f, omf = __fsub_rn(1.0f, PL.f);
            ah2h2 = __fadd_rn(__fmul_rn(omf, v[0]), __fmul_rn(f, v[1]));
            ah2he = __fadd_rn(__fmul_rn(omf, v[2]), __fmul_rn(f, v[3]));
            dh2dt = __fadd_rn(__fmul_rn(omf, dv[0]), __fmul_rn(f, dv[1]));
            dhedt = __fadd_rn(__fmul_rn(omf, dv[2]), __fmul_rn(f, dv[3]));
            dh2dfp = __fdiv_rn(__fsub_rn(v[1], v[0]), B.para_deltaf);
            dhedfp = __fdiv_rn(__fsub_rn(v[3], v[2]), B.para_deltaf);
        }
        const float qh2 = L.q[0], qhe = L.q[1], qn2 = L.q[2], qch4 = L.q[3], qco2 = L.q[4];
        float sum = __fadd_rn(__fmul_rn(__fmul_rn(ah2h2, qh2), qh2), __fmul_rn(__fmul_rn(ah2he, qh2), qhe));
        dab[0] = __fadd_rn(__fmul_rn(__fmul_rn(2.0f, qh2), ah2h2), __fmul_rn(qhe, ah2he));
        dab[1] = __fmul_rn(qh2, ah2he);
        dab[5] = __fadd_rn(__fmul_rn(__fmul_rn(dh2dt, qh2), qh2), __fmul_rn(__fmul_rn(dhedt, qh2), qhe));
        dab[6] = __fadd_rn(__fmul_rn(__fmul_rn(dh2dfp, qh2), qh2), __fmul_rn(__fmul_rn(dhedfp, qh2), qhe));
        // H2-N2, N2-CH4, N2-N2, CH4-CH4, H2-CH4 (nparacon_all.f:262-318)
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(v[4], qh2), qn2));
        dab[0] = __fadd_rn(dab[0], __fmul_rn(qn2, v[4]));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(qh2, v[4]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qn2), dv[4]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(v[5], qn2), qch4));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(qch4, v[5]));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(qn2, v[5]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qn2, qch4), dv[5]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(v[6], qn2), qn2));
        dab[2] = __fadd_rn(dab[2], __fmul_rn(__fmul_rn(2.0f, qn2), v[6]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qn2, qn2), dv[6]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(v[7], qch4), qch4));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(__fmul_rn(2.0f, qch4), v[7]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qch4, qch4), dv[7]));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(v[8], qh2), qch4));
        dab[0] = __fadd_rn(dab[0], __fmul_rn(qch4, v[8]));
        dab[3] = __fadd_rn(dab[3], __fmul_rn(qh2, v[8]));
        dab[5] = __fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qch4), dv[8]));
        // co2cia / n2n2cia / n2h2cia are zero below 3900 cm-1 (host-checked)
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qco2), qco2));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qn2), qn2));
        sum = __fadd_rn(sum, __fmul_rn(__fmul_rn(0.0f, qn2), qh2));
        absorb = __fmul_rn(sum, L.cia_tau);
#pragma unroll
        for (int i = 0; i < 7; ++i) dab[i] = __fmul_rn(dab[i], L.cia_tau);
    } else if (S.has_cia) {
        float my_a = 0.0f, my_d = 0.0f;
        if (W.cia_cv >= 0 && lane < 9) {
            const int p = lane;
            const float t = W.cia_t, u = L.cia_u;
            const float omt = __fsub_rn(1.0f, t), omu = __fsub_rn(1.0f, u);
            const float* kc = B.kcia;
            const int64_t b11 = 9 * ((int64_t)L.cia_ct + 25 * (int64_t)W.cia_cv);
            const int64_t b12 = 9 * ((int64_t)L.cia_ct + 25 * ((int64_t)W.cia_cv + 1));
            const int64_t b22 = 9 * ((int64_t)L.cia_ct + 1 + 25 * ((int64_t)W.cia_cv + 1));
            const int64_t b21 = 9 * ((int64_t)L.cia_ct + 1 + 25 * (int64_t)W.cia_cv);
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
            my_a = x;
            my_d = __fmul_rn(d, L.cia_dudt);
        }
        float alpha[9], da[9];
#pragma unroll
        for (int p = 0; p < 9; ++p) {
            alpha[p] = __shfl_sync(kFull, my_a, p);
            da[p] = __shfl_sync(kFull, my_d, p);
        }
        const float qh2 = L.q[0], qhe = L.q[1], qn2 = L.q[2], qch4 = L.q[3], qco2 = L.q[4];
        float sum = 0.0f;
        const bool eq = S.inormal == 0;
        const float ao = eq ? alpha[0] : alpha[2], ao1 = eq ? alpha[1] : alpha[3];
        const float dao = eq ? da[0] : da[2], dao1 = eq ? da[1] : da[3];
        sum = __fadd_rn(__fadd_rn(sum, __fmul_rn(__fmul_rn(ao, qh2), qh2)), __fmul_rn(__fmul_rn(ao1, qh2), qhe));
        dab[0] = __fadd_rn(__fadd_rn(dab[0], __fmul_rn(__fmul_rn(2.0f, qh2), ao)), __fmul_rn(qhe, ao1));
        dab[1] = __fadd_rn(dab[1], __fmul_rn(qh2, ao1));
        dab[5] = __fadd_rn(__fadd_rn(dab[5], __fmul_rn(__fmul_rn(qh2, qh2), dao)), __fmul_rn(__fmul_rn(qh2, qhe), dao1));
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
#pragma unroll
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
    if (para) {   // the para-H2 fraction (cirsradg_wave.f:659-661)
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s == S.sw_para) dtc[s] = __fadd_rn(dtc[s], dab[6]);
    }
    if (S.iray) {
        float xr = W.xray;
        if (para && S.iray == 3) {   // air: rayleigha at this layer's P and T (cirsradg_wave.f:668-669)
            const int64_t l = il_glob - S.lay_off;
            const float vv = S.ispace ? __fdiv_rn(1e4f, W.vwave) : W.vwave;
            xr = __fmul_rn(rayleigha_dev(vv, B.lay_press[S.lp_off + l], B.lay_temp[S.lt_off + l]), 1E20f);
        }
        const float av = __fmul_rn(L.utotl, xr);
        taucon = __fadd_rn(taucon, av);
        const float add = __fmul_rn(xr, 1.0e-20f);
#pragma unroll
        for (int s = 0; s < kMaxSw; ++s)
            if (s < S.nsw && S.isw[s] < S.ngas) dtc[s] = __fadd_rn(dtc[s], add);
    }
    return taucon;
}

// ---------------------------------------------------------------------------
// One overlap pass with sorting (noverlapg.f:110-147/175-190 + rankg.f).
// Warp scratch holds k1[i], k2[j], dk1[i], dk2[j] and the previous gradient
// columns colP[c][i]; the pass writes the new distribution to kg[] and the
// new columns to colN[c][].  An element (i, j) travels as the 64-bit word
// fkey(key) << 32 | i << 5 | j: its low half orders like the reference's
// element number i*ng + j, so word order is the stable key order.
struct PassCtx {
    int ng, nloop, ncol, first, igas;
    float a1, a2;
};

struct WarpPtr {
    unsigned long long *bufA, *bufB;
    const short* mtab;       // lanes' merge output ranges (merge_lane_start), per CTA
    float *k1, *k2, *dk1, *dk2, *kg;
    double* splitfrac;
    int* splitpos;
};

__device__ __forceinline__ float key_of(const PassCtx& P, const WarpPtr& wp, int i, int j) {
    return P.first ? __fadd_rn(__fmul_rn(wp.k1[i], P.a1), __fmul_rn(wp.k2[j], P.a2))
                   : __fadd_rn(wp.k1[i], __fmul_rn(wp.k2[j], P.a2));
}

__device__ __forceinline__ unsigned long long pack(float key, int i, int j) {
    return ((unsigned long long)fkey(key) << 32) | (unsigned)((i << 5) | j);
}

__device__ __forceinline__ unsigned hi32(unsigned long long w) { return (unsigned)(w >> 32); }

// Merge of A = ki[a0, a1) and B = ki[b0, b1) into ko[s, e) (e - s elements):
// the front half smallest-first from the start, the back half largest-first
// from the end, as two independent chains.  Only the key halves are
// compared: every element of A precedes every element of B, so on equal keys
// A's word comes first (the stable order).  No bounds are checked: past a
// side's end of the range lies the next word of its run (which follows every
// word of the other side still in the range: the ranges end at a merge-path
// split) or the run's sentinel (key ~0 after a run, 0 before it, keys no word
// holds since NaN keys never reach the merge).
__device__ __forceinline__ void merge_seg(const unsigned long long* ki, unsigned long long* ko, int s, int e,
                                          int a0, int a1, int b0, int b1) {
    const int len = e - s, nb = len >> 1;
    int fa = a0, fb = b0, ba = a1, bb = b1;
    unsigned long long xa = ki[fa], yb = ki[fb], xA = ki[ba - 1], yB = ki[bb - 1];
#pragma unroll 1
    for (int t = 0; t < nb; ++t) {
        const bool ta = hi32(xa) <= hi32(yb), tA = hi32(xA) > hi32(yB);
        ko[s + t] = ta ? xa : yb;
        ko[e - 1 - t] = tA ? xA : yB;
        fa += ta;
        fb += !ta;
        ba -= tA;
        bb -= !tA;
        const unsigned long long nv = ki[ta ? fa : fb];
        const unsigned long long nv2 = ki[tA ? ba - 1 : bb - 1];
        xa = ta ? nv : xa;
        yb = ta ? yb : nv;
        xA = tA ? nv2 : xA;
        yB = tA ? yB : nv2;
    }
    if (len & 1) ko[s + nb] = hi32(xa) <= hi32(yb) ? xa : yb;   // the middle word
}

// Output ranges of the lanes at each merge level, for NG rows (run = NG <<
// level): pair p of runs (start st_p) is served by lanes [L_p, L_p+1),
// L_p = floor(32 st_p / n), which split it evenly.  No lane's range crosses
// a pair boundary, so every lane runs a single two-ended merge per level (7
// steps for NG = 20).  The table mtab[level * 33 + lane] holds the lane's
// first output position (n past the last level, and at lane 32).
__device__ __forceinline__ int merge_lane_start(int ng, int level, int l) {
    const int n = ng * ng, run = ng << level;
    if (run >= n || l >= 32) return n;
    const int two = run << 1, npairs = (n + two - 1) / two;
    int p = 0;
    while (p + 1 < npairs && (32 * (p + 1) * two) / n <= l) ++p;
    const int st = p * two, sz = min(two, n - st);
    const int lp = (32 * st) / n, lq = p + 1 < npairs ? (32 * (p + 1) * two) / n : 32;
    return st + ((l - lp) * sz) / (lq - lp);
}

// Stable merge sort of ng sorted rows of ng words.  Layout of every level:
// run r of length `run` (the last one may be shorter) at r * (run + 2) + 1,
// the word 0 before it and ~0 after it, and right after the last run's ~0 a
// further pair 0, ~0 (the empty right run of an unpaired last run).  The rows start
// in buffer `start` in that layout (run = ng); the result is one run at
// offset 1 of the returned buffer.  At each level every lane merges the
// output range mtab gives it (inside one pair of runs): one merge-path
// search finds the split of its first position, the next lane's search gives
// the split of its last (a pair's end needs none).  A level whose every pair
// is already in order (left run's last word below the right run's first) is
// copied instead; in the overlap passes of typical k-distributions that holds
// for about one level in four.  Within a merge every word of the left run has
// a smaller element part than every word of the right run, so comparing
// whole words is the stable merge.
template <int NGC>
__device__ int merge_rows(const WarpPtr& wp, const short* mtab, int ng_run, int lane, int start) {
    const int ng = NGC ? NGC : ng_run;
    const int n = ng * ng;
    int cur = start;
    int level = 0;
    for (int run = ng; run < n; run <<= 1, ++level) {
        const unsigned long long* ki = cur ? wp.bufB : wp.bufA;
        unsigned long long* ko = cur ? wp.bufA : wp.bufB;
        const int two = run << 1, sin = run + 2, sout = two + 2;
        const int sh = level + 1;               // two = ng << sh, n / two = ng >> sh
        const int nout = (ng + (1 << sh) - 1) >> sh;   // runs after this level
        bool inorder = true;                    // pair `lane` already in order
        if (lane * two + run < n) inorder = ki[2 * lane * sin + run] < ki[(2 * lane + 1) * sin + 1];
        const bool copy = __all_sync(kFull, inorder);
        if (lane < nout) {                      // the output runs' sentinels
            ko[lane * sout] = 0ull;
            ko[lane * sout + 1 + min(two, n - lane * two)] = ~0ull;
        }
        if (lane == 0) {
            const int last = (nout - 1) * sout + 2 + (n - (nout - 1) * two);
            ko[last] = 0ull;
            ko[last + 1] = ~0ull;
        }
        const int s = mtab[level * 33 + lane], e = mtab[level * 33 + lane + 1];
        const int p = (s / ng) >> sh, ms = p * two;
        const int m = min(run, n - ms), ny = max(0, min(run, n - ms - run));
        const int kk = s - ms;
        const int abase = 2 * p * sin + 1, bbase = ny > 0 ? abase + sin : abase + m + 2;
        const int obase = p * sout + 1 - ms;
        if (copy) {
#pragma unroll 1
            for (int k = s; k < e; ++k) {
                const int o = k - ms;
                ko[obase + k] = ki[o < m ? abase + o : bbase + (o - m)];
            }
        } else {
            int as = 0;                         // split of s: words taken from the pair's left run
            if (s < n) {
                const unsigned* kh = (const unsigned*)ki + 1;   // the key halves
                int lo = max(0, kk - ny), hi = min(kk, m);
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (kh[2 * (abase + mid)] <= kh[2 * (bbase + kk - mid - 1)]) lo = mid + 1; else hi = mid;
                }
                as = lo;
            }
            const int as_next = __shfl_down_sync(kFull, as, 1);
            if (s < e) {
                int ae = m, be = ny;
                if (e < ms + m + ny) {          // ends inside the pair: the next lane's split
                    ae = as_next;
                    be = (e - ms) - as_next;
                }
                merge_seg(ki, ko, obase + s, obase + e, abase + as, abase + ae, bbase + (kk - as), bbase + be);
            }
        }
        __syncwarp();
        cur ^= 1;
    }
    return cur;
}

// gradient value of tracked column c for element (i, j) (noverlapg.f:125-127,
// 184-187); used by the sequential (irregular) walk only
__device__ __forceinline__ float elem_grad(const PassCtx& P, int gcol, int c, int i, int j, const WarpPtr& wp,
                                           const float* colP, int ngas) {
    if (gcol == ngas) {
        if (P.first) return __fadd_rn(__fmul_rn(wp.dk1[i], P.a1), __fmul_rn(wp.dk2[j], P.a2));
        return __fadd_rn(wp.dk1[i], __fmul_rn(wp.dk2[j], P.a2));
    }
    if (gcol == P.igas) return wp.k2[j];
    if (P.first) return gcol == 0 ? wp.k1[i] : 0.0f;
    if (gcol > P.igas) return 0.0f;
    return colP[c * kMaxNg + i];
}

// Gradient columns of one sorted pass.  They feed the Jacobian alone (never a
// sort key), so they need not follow the reference's summation order.  Every
// column is v_c(i, j) = U[i][c] + V[j][c] (T: dk1(i)[a1] + dk2(j) a2; earlier
// gas: u(i); added gas: k2(j)).  column_tables writes U and V for the columns
// a pass can make non-zero (slots 0..nz-1: slot k holds column
// (cm >> 3k) & 7; a column of a gas not yet added is zero and not computed):
// rows of 8 values and a pad (48 B apart, spread over the banks), U rows then
// V rows.  One slot per iteration, kept rolled (the kernel is bound by its
// instruction cache).
__device__ __forceinline__ void column_tables(const SpecDev& S, const PassCtx& P, const WarpPtr& wp,
                                              const float* colP, float4* UV, unsigned cm, int nz,
                                              int ng, int lane) {
    if (lane < ng) {
        const int x = lane;
        float* Ur = (float*)(UV + 3 * x);
        float* Vr = (float*)(UV + 3 * ng + 3 * x);
#pragma unroll 1
        for (int k = 0; k < kMaxCols; ++k) {
            float u = 0.0f, v = 0.0f;
            if (k < nz) {
                const int c = (cm >> (3 * k)) & 7;
                const int gcol = S.col_gas[c];
                if (gcol == S.ngas) {
                    u = P.first ? wp.dk1[x] * P.a1 : wp.dk1[x];
                    v = wp.dk2[x] * P.a2;
                } else if (gcol == P.igas) {
                    v = wp.k2[x];
                } else if (gcol < P.igas) {
                    if (!P.first) u = colP[c * kMaxNg + x];
                    else if (gcol == 0) u = wp.k1[x];
                }
            }
            Ur[k] = u;
            Vr[k] = v;
        }
    }
}

// k(g) and the gradient columns of one sorted pass, one lane per bin
// (rankg.f:118-146).  k: the split remainder, the whole elements and the
// split fraction, then / sngl(sum), every operation rounded as in the
// reference.  The gradient columns take the same walk: bin b of column c is
// the sum of share * w * v_c over the bin's elements (split elements shared
// f : 1 - f), divided by the same normalisation.  NCV: the slots computed per
// element (4, 5 or 8, at least nz).
template <int NCV>
__device__ __forceinline__ void bins_and_columns(const PassCtx& P, const WarpPtr& wp, const unsigned long long* A,
                                                 const float4* UV, const float* wtab, float* colN,
                                                 unsigned cm, int nz, int ng, int nloop,
                                                 int c_last, int lane) {
    if (lane >= ng) return;
    const int bb = lane;
    float acc = 0.0f, nf = 0.0f;            // nf == 0: bin never reached
    float gc[NCV];
#pragma unroll
    for (int c = 0; c < NCV; ++c) gc[c] = 0.0f;
    auto add_columns = [&](unsigned q, float sw) {   // sw: share x weight of element q
        const int i = q >> 5, j = q & 31;
        float uu[8], vv[8];
        const float4 u0 = UV[3 * i], v0 = UV[3 * ng + 3 * j];
        uu[0] = u0.x; uu[1] = u0.y; uu[2] = u0.z; uu[3] = u0.w;
        vv[0] = v0.x; vv[1] = v0.y; vv[2] = v0.z; vv[3] = v0.w;
        if (NCV == 5) {
            uu[4] = ((const float*)(UV + 3 * i + 1))[0];
            vv[4] = ((const float*)(UV + 3 * ng + 3 * j + 1))[0];
        } else if (NCV == 8) {
            const float4 u1 = UV[3 * i + 1], v1 = UV[3 * ng + 3 * j + 1];
            uu[4] = u1.x; uu[5] = u1.y; uu[6] = u1.z; uu[7] = u1.w;
            vv[4] = v1.x; vv[5] = v1.y; vv[6] = v1.z; vv[7] = v1.w;
        }
#pragma unroll
        for (int c = 0; c < NCV; ++c) gc[c] = fmaf(sw, uu[c] + vv[c], gc[c]);
    };
    if (bb <= c_last) {
        double sum = 0.0;
        int p = 0;
        if (bb > 0) {
            const int s = wp.splitpos[bb - 1];
            const double frac = wp.splitfrac[bb - 1];
            const unsigned long long word = A[s];
            const unsigned q = (unsigned)word & 0xffffu;
            const float w = wtab[q + (q >> 5)];
            const float sr = __double2float_rn(__dsub_rn(1.0, frac));
            acc = __fmul_rn(__fmul_rn(sr, funkey((unsigned)(word >> 32))), w);
            sum = __dmul_rn(__dsub_rn(1.0, frac), (double)w);
            add_columns(q, __fmul_rn(sr, w));
            p = s + 1;
        }
        const bool closes = bb < c_last;
        const int pend = closes ? wp.splitpos[bb] : nloop;
#pragma unroll 1
        for (; p < pend; ++p) {
            const unsigned long long word = A[p];
            const unsigned q = (unsigned)word & 0xffffu;
            const float w = wtab[q + (q >> 5)];
            acc = __fadd_rn(acc, __fmul_rn(funkey((unsigned)(word >> 32)), w));
            sum = __dadd_rn(sum, (double)w);
            add_columns(q, w);
        }
        nf = 1.0f;
        if (closes) {
            const int s = wp.splitpos[bb];
            const double frac = wp.splitfrac[bb];
            const unsigned long long word = A[s];
            const unsigned q = (unsigned)word & 0xffffu;
            const float w = wtab[q + (q >> 5)];
            const float sf = __double2float_rn(frac);
            acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(sf, funkey((unsigned)(word >> 32))), w));
            sum = __dadd_rn(sum, __dmul_rn(frac, (double)w));
            add_columns(q, __fmul_rn(sf, w));
            nf = __double2float_rn(sum);
            acc = __fdiv_rn(acc, nf);
        } else if (bb == ng - 1) {
            nf = __double2float_rn(sum);
            acc = __fdiv_rn(acc, nf);
        }
    }
    wp.kg[bb] = acc;
#pragma unroll
    for (int c = 0; c < kMaxCols; ++c)
        if (c < P.ncol) colN[c * kMaxNg + bb] = 0.0f;
#pragma unroll
    for (int k = 0; k < NCV; ++k)
        if (k < nz) colN[((cm >> (3 * k)) & 7) * kMaxNg + bb] = nf != 0.0f ? gc[k] / nf : 0.0f;
}

template <int NGC>
__device__ void sort_pass(const BatchDev& B, const SpecDev& S, const PassCtx& P, const WarpPtr& wp,
                          const double* g_ord, const float* wtab, int lane, Diag& dg, const float* colP,
                          float* colN, int16_t* dbg_perm, int16_t* dbg_split) {
    // NGC > 0: the run's NG as a compile-time constant (NGC = P.ng)
    const int ng = NGC ? NGC : P.ng, nloop = NGC ? NGC * NGC : P.nloop;
    // ---- sort --------------------------------------------------------------
    // The words of row i, k1(i)[*a1] + k2(j)*a2 over j, are sorted when k2 is
    // monotone and a2 >= 0.  If every row's first word exceeds the last word
    // of the row before it (and the rows are in order), row-major order is
    // already the sorted order; otherwise the rows are merged.  Other inputs
    // (and any NaN key) take the reference heapsort.
    bool monoB = P.a2 >= 0.0f && (!P.first || P.a1 >= 0.0f);
    if (lane + 1 < ng) monoB = monoB && (wp.k2[lane] <= wp.k2[lane + 1]);
    monoB = __all_sync(kFull, monoB);
    const unsigned long long* A = wp.bufA;
    if (monoB) {
        // row-major words: contiguous in bufA, and in bufB in the merge's
        // layout (row i at i (ng + 2) + 1 between sentinels)
        unsigned long long* W = wp.bufA;
        unsigned long long* Wg = wp.bufB;
        bool finite = true;                         // no NaN key
        {
            int i = lane / ng, j = lane - (lane / ng) * ng;
#pragma unroll 1
            for (int e = lane; e < nloop; e += 32) {
                const float kv = key_of(P, wp, i, j);
                finite = finite && kv == kv;
                const unsigned long long w = pack(kv, i, j);
                W[e] = w;
                Wg[e + 2 * i + 1] = w;
                j += 32;
                while (j >= ng) { j -= ng; ++i; }
            }
            if (lane <= ng) {
                Wg[lane * (ng + 2)] = 0ull;
                Wg[lane * (ng + 2) + (lane < ng ? ng + 1 : 1)] = ~0ull;
            }
        }
        monoB = __all_sync(kFull, finite);
        __syncwarp();
        bool disjoint = true;
        if (lane + 1 < ng) disjoint = W[(lane + 1) * ng] > W[lane * ng + ng - 1];
        disjoint = __all_sync(kFull, disjoint);
        if (monoB && disjoint) {
            dg.block_passes += (lane == 0);
        } else if (monoB) {
            A = (merge_rows<NGC>(wp, wp.mtab, ng, lane, 1) ? wp.bufB : wp.bufA) + 1;
        }
    }
    // inputs whose rows are not sorted (a k-distribution not monotone in g)
    // or that hold a NaN key take the reference heapsort below
    const bool need_exact = !monoB;

    // ---- cumulative weights, bin boundaries, tie checks --------------------
    // Each lane takes a chunk of consecutive sorted positions: the FP64 prefix
    // of the weights inside its chunk into scratch, and a warp scan of the
    // chunk totals (every partial sum is exact, so any order gives the
    // reference's values); then one lane per g boundary finds its split
    // position (the first position whose cumulative weight reaches
    // g_ord(b+1), rankg.f:119-129) and forms the split fraction.
    const int ch = (nloop + 31) >> 5;
    const int p0 = min(lane * ch, nloop), p1 = min(p0 + ch, nloop);
    bool exact = false, irregular = false, gerr = false;
    int c_last = 0;
    // the reference heapsort on the elements in nloop order (sort2g.f); its
    // scratch lives in the buffer not holding A, its result replaces A
    auto heapsort_pass = [&]() {
        __syncwarp();
        unsigned long long* Aw = (A >= wp.bufB) ? wp.bufB : wp.bufA;
#pragma unroll 1
        for (int e = lane; e < nloop; e += 32) {
            const int i = e / ng, j = e - i * ng;
            Aw[e] = ((unsigned long long)__float_as_uint(key_of(P, wp, i, j)) << 32) | (unsigned)e;
        }
        __syncwarp();
        if (lane == 0) heapsort_words(nloop, Aw);
        __syncwarp();
#pragma unroll 1
        for (int p = lane; p < nloop; p += 32) {
            const unsigned long long w = Aw[p];
            const int e = (int)(unsigned)w;
            const int i = e / ng, j = e - i * ng;
            Aw[p] = pack(wkey(w), i, j);
        }
        __syncwarp();
        A = Aw;
        exact = true;
        dg.exact_passes += (lane == 0);
    };
    if (need_exact) heapsort_pass();
    double* gd = nullptr;
    for (int attempt = 0; attempt < 2; ++attempt) {
        gd = (double*)((A >= wp.bufB) ? wp.bufA : wp.bufB);   // free buffer
        double run = 0.0;
        unsigned kbp = p0 >= 1 && p0 < p1 ? (unsigned)(A[p0 - 1] >> 32) : 0u;
        bool anytie = false;
#pragma unroll 1
        for (int p = p0; p < p1; ++p) {
            const unsigned long long word = A[p];
            const unsigned q = (unsigned)word & 0xffffu;
            const unsigned kb = (unsigned)(word >> 32);
            run = __dadd_rn(run, (double)wtab[q + (q >> 5)]);
            gd[p] = run;
            anytie |= (p >= 1 && kb == kbp);         // fkey folds -0 onto +0
            kbp = kb;
        }
        double incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl = __dadd_rn(incl, t);
        }
        const double base = __dsub_rn(incl, run);   // exact: every partial sum is exact
        __syncwarp();
        // boundary b = lane: the lane L whose chunk the prefix reaches g_ord(b+1)
        // in (a search over the lanes' totals), then the position inside it
        const double gb = lane < ng ? g_ord[lane + 1] : 0.0;
        int L = 0;
#pragma unroll
        for (int st = 16; st >= 1; st >>= 1) {
            const double v = __shfl_sync(kFull, incl, L + st - 1);
            if (v < gb) L += st;
        }
        const double tot = __shfl_sync(kFull, incl, 31);
        const double bL = __shfl_sync(kFull, base, L);
        int sp = nloop;
        bool risky = false;
        if (lane < ng) {
            const int c0 = min(L * ch, nloop);
            if (tot >= gb) {
                int lo = c0, hi = min(c0 + ch, nloop);
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (__dadd_rn(gd[mid], bL) >= gb) hi = mid; else lo = mid + 1;
                }
                sp = lo;
            }
            if (sp < nloop) {
                const unsigned long long word = A[sp];
                const unsigned q = (unsigned)word & 0xffffu;
                const unsigned kb = (unsigned)(word >> 32);
                const double gprev = sp > c0 ? __dadd_rn(gd[sp - 1], bL) : bL;
                wp.splitpos[lane] = sp;
                wp.splitfrac[lane] = __ddiv_rn(__dsub_rn(gb, gprev), (double)wtab[q + (q >> 5)]);
                const bool tl = sp >= 1 && kb == (unsigned)(A[sp - 1] >> 32);
                const bool tr = sp + 1 < nloop && kb == (unsigned)(A[sp + 1] >> 32);
                risky = tl || tr;
            } else {
                wp.splitpos[lane] = -1;
            }
        }
        // one element crossing two boundaries: equal split positions
        const int sp_next = __shfl_down_sync(kFull, sp, 1);
        irregular = __any_sync(kFull, lane + 1 < ng && sp < nloop && sp == sp_next);
        c_last = __popc(__ballot_sync(kFull, lane < ng && sp < nloop));
        const int sp_last = __shfl_sync(kFull, sp, ng - 1);
        gerr = c_last == ng && sp_last < nloop - 1;    // elements left after the last boundary
        risky = __any_sync(kFull, risky);
        anytie = __any_sync(kFull, anytie);
        if (attempt == 0) {
            dg.sort_passes += (lane == 0);
            dg.tie_passes += (lane == 0 && anytie);
        }
        if (exact || !(risky || (B.strict_ties && anytie))) break;
        heapsort_pass();
    }
    if (gerr) atomicOr(B.status, kStGord);
    __syncwarp();
    if (dbg_perm) {
#pragma unroll 1
        for (int p = lane; p < nloop; p += 32) {
            const unsigned q = (unsigned)A[p] & 0xffffu;
            dbg_perm[p] = (int16_t)((q >> 5) * ng + (q & 31));
        }
        if (lane < ng && !irregular) dbg_split[lane] = (int16_t)wp.splitpos[lane];
    }

    if (irregular) {
        const int ncol = P.ncol;
        // sequential rankg walk (rankg.f:118-152) by lane 0
        dg.irregular += (lane == 0);
        if (lane == 0) {
#pragma unroll 1
            for (int bb = 0; bb < ng; ++bb) {
                wp.kg[bb] = 0.0f;
                for (int c = 0; c < ncol; ++c) colN[c * kMaxNg + bb] = 0.0f;
            }
            int ig = 0;
            double sum = 0.0, gprev = 0.0;
#pragma unroll 1
            for (int p = 0; p < nloop; ++p) {
                const unsigned long long word = A[p];
                const unsigned q = (unsigned)word & 0xffffu;
                const int i = q >> 5, j = q & 31;
                const float cval = funkey((unsigned)(word >> 32));
                const float w = wtab[q + (q >> 5)];
                const double gcur = __dadd_rn(gprev, (double)w);
                if (ig >= ng) { atomicOr(B.status, kStGord); break; }
                if (gcur < g_ord[ig + 1]) {
                    wp.kg[ig] = __fadd_rn(wp.kg[ig], __fmul_rn(cval, w));
                    for (int c = 0; c < ncol; ++c)
                        colN[c * kMaxNg + ig] = __fadd_rn(colN[c * kMaxNg + ig],
                            __fmul_rn(elem_grad(P, S.col_gas[c], c, i, j, wp, colP, S.ngas), w));
                    sum = __dadd_rn(sum, (double)w);
                } else {
                    const double frac = __ddiv_rn(__dsub_rn(g_ord[ig + 1], gprev), __dsub_rn(gcur, gprev));
                    const float sf = __double2float_rn(frac);
                    wp.kg[ig] = __fadd_rn(wp.kg[ig], __fmul_rn(__fmul_rn(sf, cval), w));
                    for (int c = 0; c < ncol; ++c)
                        colN[c * kMaxNg + ig] = __fadd_rn(colN[c * kMaxNg + ig],
                            __fmul_rn(__fmul_rn(sf, elem_grad(P, S.col_gas[c], c, i, j, wp, colP, S.ngas)), w));
                    sum = __dadd_rn(sum, __dmul_rn(frac, (double)w));
                    const float fs = __double2float_rn(sum);
                    wp.kg[ig] = __fdiv_rn(wp.kg[ig], fs);
                    for (int c = 0; c < ncol; ++c) colN[c * kMaxNg + ig] = __fdiv_rn(colN[c * kMaxNg + ig], fs);
                    if (dbg_split) dbg_split[ig] = (int16_t)p;
                    ig = ig + 1;
                    sum = __dmul_rn(__dsub_rn(1.0, frac), (double)w);
                    if (ig < ng) {
                        const float sr = __double2float_rn(__dsub_rn(1.0, frac));
                        wp.kg[ig] = __fmul_rn(__fmul_rn(sr, cval), w);
                        for (int c = 0; c < ncol; ++c)
                            colN[c * kMaxNg + ig] =
                                __fmul_rn(__fmul_rn(sr, elem_grad(P, S.col_gas[c], c, i, j, wp, colP, S.ngas)), w);
                    }
                }
                gprev = gcur;
            }
            if (ig == ng - 1) {
                const float fs = __double2float_rn(sum);
                wp.kg[ig] = __fdiv_rn(wp.kg[ig], fs);
                for (int c = 0; c < ncol; ++c) colN[c * kMaxNg + ig] = __fdiv_rn(colN[c * kMaxNg + ig], fs);
            }
        }
        __syncwarp();
        return;
    }

    // ---- k(g) and gradient columns -------------------------------------------
    // A column of a gas not yet added (gas index above igas) is zero in this
    // pass; the others are computed, their arithmetic specialised on how many
    // there are.  Their tables go to the free buffer (the prefix is done with).
    unsigned cm = 0;                            // slot k holds column (cm >> 3k) & 7
    int nz = 0;
#pragma unroll
    for (int c = 0; c < kMaxCols; ++c) {
        if (c < P.ncol) {
            const int g = S.col_gas[c];
            if (g == S.ngas || g <= P.igas) {
                cm |= (unsigned)c << (3 * nz);
                ++nz;
            }
        }
    }
    float4* UV = (float4*)gd;
    __syncwarp();
    column_tables(S, P, wp, colP, UV, cm, nz, ng, lane);
    __syncwarp();
    if (nz <= 4) bins_and_columns<4>(P, wp, A, UV, wtab, colN, cm, nz, ng, nloop, c_last, lane);
    else if (nz == 5) bins_and_columns<5>(P, wp, A, UV, wtab, colN, cm, nz, ng, nloop, c_last, lane);
    else bins_and_columns<8>(P, wp, A, UV, wtab, colN, cm, nz, ng, nloop, c_last, lane);
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
    dBdT = B * (x / T) * ((em1 + 1.0f) / em1);
}

}  // namespace

// ---------------------------------------------------------------------------
// t2: the run's k-tables carry one temperature grid per pressure (NT < 0);
// ext: some spectrum takes the para-H2 CIA (flagh2p = 1), an IMOD 18 path or
// iform = 3.  Template arguments, so that the usual kernel carries no trace
// of either.  WARPS: warps per CTA, the layers of one (spectrum, wavenumber)
// item worked on at once -- the tile shape the autotuner chooses; the
// residency bound keeps 20 warps per SM at 96 registers.  NGC: NG as a
// compile-time constant (the overlap's sizes, offsets and loop bounds fold),
// or 0 for an NG read at run time
template <bool t2, bool ext, int WARPS, int NGC>
__global__ void __launch_bounds__(WARPS * 32, 20 / WARPS)
fwd_kernel(BatchDev B, int nsw_max, int ncol_max, int nlmax_max, int npath_max) {
    constexpr int kThreads = WARPS * 32;
    constexpr int kWarps = WARPS;
    extern __shared__ __align__(16) char smem[];
    __shared__ SpecDev S_sh;
    const Layout Lo = make_layout(B.ng, nsw_max, ncol_max, nlmax_max, npath_max, WARPS);
    const WarpOff wo = warp_off(ncol_max);
    const PathOff po = path_off(nlmax_max, B.ng, nsw_max);
    double* g_ord = (double*)(smem + Lo.off_gord);
    float* delg = (float*)(smem + Lo.off_delg);
    float* wtab = (float*)(smem + Lo.off_wtab);   // w(i, j) = delg(i) delg(j) at 33 i + j: the overlap's element weights, read with q + (q >> 5) for q = i << 5 | j
    char* region = smem + Lo.off_region;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ng = NGC ? NGC : B.ng;   // NGC > 0: the instance for NG = NGC (== B.ng)
    // per-CTA scratch slot in global memory (L2-resident): tau[l][g], dtau[l][s][g]
    float* tau_s = B.cell_scratch + (int64_t)blockIdx.x * B.cell_slot;
    float* dtau_s = tau_s + (int64_t)B.cell_Lmax * ng;
    for (int i = tid; i <= ng + 2; i += kThreads) g_ord[i] = i <= ng ? B.g_ord[i] : __longlong_as_double(0x7ff0000000000000ll);
    for (int i = tid; i < ng; i += kThreads) delg[i] = B.delg[i];
    for (int q = tid; q < ng * 32; q += kThreads) {
        const int j = q & 31;
        wtab[q + (q >> 5)] = j < ng ? __fmul_rn(B.delg[q >> 5], B.delg[j]) : 0.0f;
    }
    short* mtab = (short*)(smem + Lo.off_mtab);
    for (int i = tid; i < kMergeLevels * 33; i += kThreads) mtab[i] = (short)merge_lane_start(ng, i / 33, i % 33);
    Diag dg{0, 0, 0, 0, 0};
    __syncthreads();

    char* wsm = region + warp * Lo.warp_bytes;
    WarpPtr wp;
    wp.bufA = (unsigned long long*)(wsm + wo.bufA);
    wp.bufB = (unsigned long long*)(wsm + wo.bufB);
    wp.mtab = mtab;
    wp.k1 = (float*)(wsm + wo.k1);
    wp.k2 = (float*)(wsm + wo.k2);
    wp.dk1 = (float*)(wsm + wo.dk1);
    wp.dk2 = (float*)(wsm + wo.dk2);
    wp.kg = (float*)(wsm + wo.kg);
    wp.splitfrac = (double*)(wsm + wo.splitfrac);
    wp.splitpos = (int*)(wsm + wo.splitpos);
    float* colA = (float*)(wsm + wo.colA);
    float* colB = (float*)(wsm + wo.colB);

    __shared__ long long s_next;
    int64_t k_static = blockIdx.x;
    for (;;) {
        // next work item: grid-stride, or pulled from the launch's counter
        // (dynamic schedule); item_order maps the issue order to items
        int64_t k;
        if (B.work_next) {
            if (tid == 0) s_next = (long long)atomicAdd(B.work_next, 1ull);
            __syncthreads();
            k = s_next;
        } else {
            k = k_static;
            k_static += gridDim.x;
        }
        if (k >= B.nitems) break;
        const int64_t item = B.item_order ? (int64_t)B.item_order[k] : k;
        // locate the spectrum of this item
        int lo = 0, hi = B.nspec - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (B.item_start[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int sidx = lo;
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

        // ---------------- stage A0: non-coincident gases -----------------
        // k-distributions of gases whose wavenumber falls between two table
        // points (rankk on lane 0), parked per (layer, gas) in the slot for
        // stage A; each warp handles the layers it takes in stage A
        if (B.wg_w2) {
            const float* w2s = B.wg_w2 + S.wg_off + (int64_t)iw * S.ngas;
            const int64_t* slices = B.wg_slice + S.wg_off + (int64_t)iw * S.ngas;
            for (int l = warp; l < S.nlayer; l += kWarps) {
                const LayerDev L = B.lay[S.lay_off + l];
                float* ncw = tau_s + B.nc_off + ((int64_t)l * S.ngas) * kMaxNg * 2;
                for (int g = 0; g < S.ngas; ++g)
                    if (w2s[g] >= 0.0f) {
                        float kv, dv;
                        const float w1 = B.wg_w1 ? B.wg_w1[S.wg_off + (int64_t)iw * S.ngas + g]
                                                 : __fsub_rn(1.0f, w2s[g]);
                        get_kg_lane_nc<t2>(B, slices[g], w1, w2s[g], L, lane, (float*)wp.bufA, kv, dv);
                        if (lane < ng) {
                            ncw[(g * kMaxNg + lane) * 2] = kv;
                            ncw[(g * kMaxNg + lane) * 2 + 1] = dv;
                        }
                    }
            }
        }
        // ---------------- stage A: layers --------------------------------
        for (int l = warp; l < S.nlayer; l += kWarps) {
            const int64_t il_glob = S.lay_off + l;
            const LayerDev L = B.lay[il_glob];
            float dtc[kMaxSw];
            const float taucon = continuum<ext>(B, S, L, W, iw_glob, il_glob, lane, dtc);
            const float* amo = B.amo + S.lg_off + (int64_t)l * S.ngas;
            const int64_t* slices = B.wg_slice + S.wg_off + (int64_t)iw * S.ngas;
            const float* w2s = B.wg_w2 ? B.wg_w2 + S.wg_off + (int64_t)iw * S.ngas : nullptr;
            const float* ncw = w2s ? tau_s + B.nc_off + ((int64_t)l * S.ngas) * kMaxNg * 2 : nullptr;
            auto get_kg = [&](int g, float& kv, float& dv) {
                if (w2s && w2s[g] >= 0.0f) {
                    kv = lane < ng ? ncw[(g * kMaxNg + lane) * 2] : 0.0f;
                    dv = lane < ng ? ncw[(g * kMaxNg + lane) * 2 + 1] : 0.0f;
                } else {
                    get_kg_lane<t2, NGC>(B, slices[g], L, lane, kv, dv);
                }
            };
            float* colP = colA;
            float* colN = colB;
            float kgv;
            if (S.ngas == 1) {
                float k0, d0;
                get_kg(0, k0, d0);
                const float a0 = amo[0];
                kgv = __fmul_rn(k0, a0);
                if (lane < ng)
                    for (int c = 0; c < ncol; ++c)
                        colN[c * kMaxNg + lane] = S.col_gas[c] == S.ngas ? __fmul_rn(d0, a0) : k0;
                float* t = colP; colP = colN; colN = t;
            } else {
                float k1v, d1v;
                get_kg(0, k1v, d1v);
                kgv = 0.0f;
                for (int ig = 1; ig < S.ngas; ++ig) {
                    const bool first = ig == 1;
                    float k2v, d2v;
                    get_kg(ig, k2v, d2v);
                    const float a2 = amo[ig];
                    const float a1 = first ? amo[0] : 1.0f;
                    const float k1e = first ? k1v : kgv;
                    const bool z1 = __shfl_sync(kFull, k1e, ng - 1) == 0.0f;
                    const bool z2 = __shfl_sync(kFull, k2v, ng - 1) == 0.0f;
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
                                    else v = 0.0f;
                                } else {
                                    if (g == ig) v = 0.0f;
                                    else v = colP[c * kMaxNg + lane];
                                }
                                colN[c * kMaxNg + lane] = v;
                            }
                        }
                        kgv = first ? __fmul_rn(k1v, a1) : kgv;
                    } else {
                        if (lane < ng) {
                            wp.k1[lane] = k1e;
                            wp.k2[lane] = k2v;
                            float d1e = d1v;
                            if (!first) {
                                d1e = 0.0f;
                                for (int c = 0; c < ncol; ++c)
                                    if (S.col_gas[c] == S.ngas) d1e = colP[c * kMaxNg + lane];
                            }
                            wp.dk1[lane] = d1e;
                            wp.dk2[lane] = d2v;
                        }
                        __syncwarp();
                        PassCtx P;
                        P.ng = ng; P.nloop = ng * ng; P.ncol = ncol; P.first = first; P.igas = ig;
                        P.a1 = a1; P.a2 = a2;
                        sort_pass<NGC>(B, S, P, wp, g_ord, wtab, lane, dg, colP, colN, dp, dsp);
                        kgv = lane < ng ? wp.kg[lane] : 0.0f;
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
            if (im == 3 || (ext && im == 18)) {
                for (int j = lane; j < nlays; j += 32) {
                    float Tn = emt[j];
                    if (ext && S.inlte)
                        Tn = nlte_temp(S.inlte, Tn, B.lay_press[S.lp_off + layinc[j]], W.vwave, S.nlte_k1, S.nlte_A);
                    planck_fp32(S.ispace, W.vwave, Tn, bb[j], dbdt[j]);
                }
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
                        drdt[j * ng + g] = trn;
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
                    if (ext) {   // iform 1 (over the star's flux at v) and 3 (cirsradg_wave.f:913-929)
                        float x = S.xfac3;
                        if (S.wmode == 1) x = __fdiv_rn(x, B.wave_fac[S.wf_off + iw]);
                        if (x != 1.0f) scale_path(x, nlays, ng, g, drdt, trd, rad, gts);
                    }
                } else if (ext && im == 18) {
                    const float x18 = S.wmode == 1 ? __fdiv_rn(S.xfac18, B.wave_fac[S.wf_off + iw]) : S.xfac18;
                    path_imod18(B.e3tab, x18, nlays, ng, g, layinc, scale, tau_s, bb, W.radground_s,
                                W.gradground_s, drdt, trd, rad, gts);
                } else {
                    float tsum = 0.0f;
                    for (int j = 0; j < nlays; ++j) tsum = tsum + tau_s[layinc[j] * ng + g] * scale[j];
                    float y = fmaxf(-tsum, -500.0f);
                    if (y >= 88.7f) y = 88.7f;
                    const float e = (float)exp((double)y);
                    // IMOD 0: dcoutdq = -tau*T*dtau/dq; IMOD 1: tau*(1-A)*dtau/dq with
                    // 1-A formed as T itself (no cancellation when T < 2^-25)
                    float out, dr;
                    if (im == 0) { out = e; dr = -tsum * e; }
                    else { out = 1.0f - e; dr = tsum * e; }
                    if (ext && im == 0 && S.wmode == 2) {   // iform 4: times the star's flux (cirsradg_wave.f:861-879)
                        const float x = B.wave_fac[S.wf_off + iw];
                        out = out * x;
                        dr = dr * x;
                    }
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
            const bool em = S.imod[p] == 3 || (ext && S.imod[p] == 18);
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
                    for (int g = 0; g < ng; ++g) acc = fmaf(delg[g], fmaf(dr[g], dt[g] * sc, td[g] * dB), acc);
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
            if (B.dq_out) {
                float* o = B.dq_out + ((S.wave_off + iw) * B.dq_npath + p) * B.dq_stride;
                for (int t = tid; t < S.nlayin[p] * nsw; t += kThreads) o[t] = dq[t];
            }
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
        if (dg.block_passes) atomicAdd(B.counters + 4, dg.block_passes);
    }
}

// host-side helpers exported to host.cu
int fwd_smem_bytes(int ng, int nsw, int ncol, int nlmax, int npath, int warps) {
    return make_layout(ng, nsw, ncol, nlmax, npath, warps).total;
}

namespace {
using FwdKern = void (*)(BatchDev, int, int, int, int);
// the instance of a launch: t2 and ext as the batch needs them; a tile other
// than kWarps, and NG = 20 as a constant, exist for the usual instance only
// (one temperature grid, no extended options)
constexpr int kNgConst = 20;
FwdKern fwd_instance(bool t2, bool ext, int warps, int ng) {
    if (ext) return t2 ? fwd_kernel<true, true, kWarps, 0> : fwd_kernel<false, true, kWarps, 0>;
    if (t2) return fwd_kernel<true, false, kWarps, 0>;
    const bool c20 = ng == kNgConst;
    switch (warps) {
    case 2: return c20 ? fwd_kernel<false, false, 2, kNgConst> : fwd_kernel<false, false, 2, 0>;
    case 8: return c20 ? fwd_kernel<false, false, 8, kNgConst> : fwd_kernel<false, false, 8, 0>;
    default: return c20 ? fwd_kernel<false, false, kWarps, kNgConst> : fwd_kernel<false, false, kWarps, 0>;
    }
}
}  // namespace

int fwd_tile_warps(bool t2, bool ext, int warps) {
    return (ext || t2 || (warps != 2 && warps != 8)) ? kWarps : warps;
}

int fwd_blocks_per_sm(int smem, bool t2, bool ext, int warps, int ng) {
    const int w = fwd_tile_warps(t2, ext, warps);
    const FwdKern k = fwd_instance(t2, ext, w, ng);
    int n = 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, w * 32, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_fwd(const BatchDev& B, int nsw, int ncol, int nlmax, int npath, int grid, int warps,
                       cudaStream_t st) {
    const int w = fwd_tile_warps(B.t2, B.ext, warps);
    const int smem = fwd_smem_bytes(B.ng, nsw, ncol, nlmax, npath, w);
    const FwdKern kern = fwd_instance(B.t2, B.ext, w, B.ng);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, w * 32, smem, st>>>(B, nsw, ncol, nlmax, npath);
    return cudaGetLastError();
}

}  // namespace rtb
