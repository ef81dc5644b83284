// conv.cu -- instrument convolution of calculated spectra on the device.
//
// Reference: radtran/cirsrad/cirsconv.f:12-246 as cirsrtfg_wave.f:448-516
// applies it to the radiance, d/dtsurf and every Jacobian row:
//   * one calculated point and FWHM != 0 (:45-54): the output is 1;
//   * FWHM > 0 (:64-160): a natural cubic spline through the calculated
//     points (CSPLINE rtm_util/cspline.f, read by CSPLINT rtm_util/csplint.f)
//     averaged at 20 equally spaced points across each channel's square bin,
//     trapezoid sum in DOUBLE PRECISION; the bin width may vary by channel
//     (the .fwh table read by VERINT radtran/path/verint.f, :147-150);
//   * FWHM = 0 (:162-169): a copy of the first nconv points;
//   * FWHM < 0 (:171-239): each channel's filter function from the .fil file,
//     linearly interpolated (INTERP rtm_util/interp.f) onto the calculated
//     points, and the filter-weighted mean of the series.
// One block per series.  For FWHM > 0 the first warp compacts the
// extrapolated, NaN-free knot list (ballots), the block computes each row's
// terms of the spline's tridiagonal system side by side, one thread runs the
// recurrence and the back substitution (sequential by nature), and the
// block's threads fill the channels; the knots sit in shared memory.  REAL
// arithmetic is written with explicitly rounded intrinsics so that it rounds
// as the reference's does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "context.h"

namespace rtb {

namespace {

constexpr int kConvThreads = 128;
constexpr int kNstep = 20;   // cirsconv.f: PARAMETER (nstep=20)
constexpr size_t kConvSmemMax = 200 * 1024;

__device__ float csplint_dev(const float* XA, const float* YA, const float* Y2A, int N, float X) {
    int klo = 1, khi = N;
    while (khi - klo > 1) {
        const int k = (khi + klo) / 2;
        if (XA[k - 1] > X) khi = k; else klo = k;
    }
    const double H = (double)__fsub_rn(XA[khi - 1], XA[klo - 1]);
    const double A = __ddiv_rn((double)__fsub_rn(XA[khi - 1], X), H);
    const double B = __ddiv_rn((double)__fsub_rn(X, XA[klo - 1]), H);
    const double a3 = __dsub_rn(__dmul_rn(__dmul_rn(A, A), A), A);
    const double b3 = __dsub_rn(__dmul_rn(__dmul_rn(B, B), B), B);
    double y1 = __dadd_rn(__dmul_rn(A, (double)YA[klo - 1]), __dmul_rn(B, (double)YA[khi - 1]));
    const double c = __dadd_rn(__dmul_rn(a3, (double)Y2A[klo - 1]), __dmul_rn(b3, (double)Y2A[khi - 1]));
    y1 = __dadd_rn(y1, __ddiv_rn(__dmul_rn(c, __dmul_rn(H, H)), 6.0));
    return fabs(y1) > 1.00E-37 ? __double2float_rn(y1) : 1.00E-37f;
}

// INTERP (rtm_util/interp.f) and VERINT (radtran/path/verint.f): the first
// point beyond XIN in the table's direction (the last point if none, the
// second if it is the first), then the REAL line through it and the point
// before.  VERINT also returns Y(I) for a vertical segment or a NaN.
__device__ float interp_dev(const float* X, const float* Y, int N, float XIN, bool verint) {
    int I = 1;
    if (X[0] < X[N - 1]) {
        while (I <= N && !(X[I - 1] > XIN)) ++I;
    } else {
        while (I <= N && !(X[I - 1] < XIN)) ++I;
    }
    if (I > N) I = N;
    if (I == 1) I = 2;
    const float t = __fdiv_rn(__fmul_rn(__fsub_rn(Y[I - 1], Y[I - 2]), __fsub_rn(XIN, X[I - 2])),
                              __fsub_rn(X[I - 1], X[I - 2]));
    float y = __fadd_rn(Y[I - 2], t);
    if (verint) {
        if (X[I - 2] == X[I - 1]) y = Y[I - 1];
        if (isnan(y)) y = Y[I - 1];
    }
    return y;
}

// Scratch of one series: knots xc, yc, then y2 and u (which first hold each
// knot's sig and right-hand side, cirsspline's terms that do not depend on
// the recurrence), and a flag per knot for a repeated abscissa.
__host__ __device__ inline size_t conv_scratch_floats(int nwave) { return (size_t)4 * (nwave + 2) + (nwave + 2 + 3) / 4; }

template <bool kShared>
__global__ void __launch_bounds__(kConvThreads)
cirsconv_kernel(int nwave, const float* __restrict__ vwave, const float* __restrict__ y, float fwhm, int nconv,
                const float* __restrict__ vconv, int nfwhm, const float* __restrict__ vfwhm,
                const float* __restrict__ xfwhm, float* __restrict__ yout, float* __restrict__ scr) {
    extern __shared__ __align__(16) float csm[];
    __shared__ int s_nc;
    const int s = blockIdx.x;
    const float* ys = y + (int64_t)s * nwave;
    const int cap = nwave + 2;
    float* xc = kShared ? csm : scr + (int64_t)s * conv_scratch_floats(nwave);
    float* yc = xc + cap;
    float* y2 = yc + cap;
    float* u = y2 + cap;
    unsigned char* dup = (unsigned char*)(u + cap);
    const float half = __fdiv_rn(fwhm, 2.0f);
    if (threadIdx.x < 32) {
        // the knots: extrapolated end points (cirsconv.f:77-104) around the
        // calculated points, NaNs dropped (:107-132); warp 0 compacts them
        const int lane = threadIdx.x;
        int nc = 0;
        if (vconv[0] < __fadd_rn(vwave[0], half)) {
            const float x = __fsub_rn(vconv[0], fwhm);
            const float sl = __fdiv_rn(__fsub_rn(ys[1], ys[0]), __fsub_rn(vwave[1], vwave[0]));
            const float v = __fadd_rn(ys[0], __fmul_rn(sl, __fsub_rn(x, vwave[0])));
            if (!isnan(v)) {
                if (lane == 0) {
                    xc[0] = x;
                    yc[0] = v;
                }
                nc = 1;
            }
        }
        for (int b = 0; b < nwave; b += 32) {
            const int i = b + lane;
            const float yi = i < nwave ? ys[i] : 0.0f;
            const bool ok = i < nwave && !isnan(yi);
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int at = nc + __popc(m & ((1u << lane) - 1u));
                xc[at] = vwave[i];
                yc[at] = yi;
            }
            nc += __popc(m);
        }
        if (vconv[nconv - 1] > __fsub_rn(vwave[nwave - 1], half)) {
            const float x = __fadd_rn(vconv[nconv - 1], fwhm);
            const float sl = __fdiv_rn(__fsub_rn(ys[nwave - 1], ys[nwave - 2]),
                                       __fsub_rn(vwave[nwave - 1], vwave[nwave - 2]));
            const float v = __fadd_rn(ys[nwave - 1], __fmul_rn(sl, __fsub_rn(x, vwave[nwave - 1])));
            if (!isnan(v)) {
                if (lane == 0) {
                    xc[nc] = x;
                    yc[nc] = v;
                }
                ++nc;
            }
        }
        if (lane == 0) s_nc = nc;
    }
    __syncthreads();
    const int nc = s_nc;
    // CSPLINE with natural ends (YP1, YPN > .99E30): the terms of each row
    // that do not depend on the recurrence, side by side
    for (int i = 1 + threadIdx.x; i < nc - 1; i += kConvThreads) {
        const float sig = __fdiv_rn(__fsub_rn(xc[i], xc[i - 1]), __fsub_rn(xc[i + 1], xc[i - 1]));
        y2[i] = sig;
        if (xc[i - 1] == xc[i] || xc[i] == xc[i + 1]) {
            dup[i] = 1;
            u[i] = 0.0f;
        } else {
            dup[i] = 0;
            const float d1 = __fdiv_rn(__fsub_rn(yc[i + 1], yc[i]), __fsub_rn(xc[i + 1], xc[i]));
            const float d0 = __fdiv_rn(__fsub_rn(yc[i], yc[i - 1]), __fsub_rn(xc[i], xc[i - 1]));
            u[i] = __fdiv_rn(__fmul_rn(6.0f, __fsub_rn(d1, d0)), __fsub_rn(xc[i + 1], xc[i - 1]));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // the recurrence and the back substitution (cspline.f), one thread
        // (each row's precomputed terms are read one step ahead, off the chain)
        float y2p = 0.0f, up = 0.0f;
        y2[0] = 0.0f;
        u[0] = 0.0f;
        float sig_n = 0.0f, t_n = 0.0f;
        unsigned char d_n = 0;
        if (nc > 2) {
            sig_n = y2[1];
            t_n = u[1];
            d_n = dup[1];
        }
        for (int i = 1; i < nc - 1; ++i) {
            const float sig = sig_n, t = t_n;
            const unsigned char dd = d_n;
            if (i + 1 < nc - 1) {
                sig_n = y2[i + 1];
                t_n = u[i + 1];
                d_n = dup[i + 1];
            }
            const float p = __fadd_rn(__fmul_rn(sig, y2p), 2.0f);
            y2p = __fdiv_rn(__fsub_rn(sig, 1.0f), p);
            up = dd ? up : __fdiv_rn(__fsub_rn(t, __fmul_rn(sig, up)), p);
            y2[i] = y2p;
            u[i] = up;
        }
        if (nc >= 2) {
            float nxt = __fdiv_rn(__fsub_rn(0.0f, __fmul_rn(0.0f, u[nc - 2])), __fadd_rn(__fmul_rn(0.0f, y2[nc - 2]), 1.0f));
            y2[nc - 1] = nxt;
            float yk = y2[nc - 2], uk = u[nc - 2];
            for (int k = nc - 2; k >= 0; --k) {
                const float ycur = yk, ucur = uk;
                if (k > 0) {
                    yk = y2[k - 1];
                    uk = u[k - 1];
                }
                nxt = __fadd_rn(__fmul_rn(ycur, nxt), ucur);
                y2[k] = nxt;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nconv; i += kConvThreads) {
        // the channel's bin width: FWHM, or the .fwh table at the channel (cirsconv.f:147-150)
        const float yfwhm = nfwhm > 0 ? interp_dev(vfwhm, xfwhm, nfwhm, vconv[i], true) : fwhm;
        const float hw = __fdiv_rn(yfwhm, 2.0f);
        const float x1 = __fsub_rn(vconv[i], hw), x2 = __fadd_rn(vconv[i], hw);
        const float delx = __fdiv_rn(__fsub_rn(x2, x1), (float)(kNstep - 1));
        const double hd = (double)__fdiv_rn(delx, 2.0f);
        double sum = 0.0, yold = 0.0;
        for (int j = 1; j <= kNstep; ++j) {
            const float xi = __fadd_rn(x1, __fmul_rn((float)(j - 1), delx));
            const double yi = nc >= 2 ? (double)csplint_dev(xc, yc, y2, nc, xi) : 0.0;
            if (j > 1) sum = __dadd_rn(sum, __dmul_rn(__dadd_rn(yi, yold), hd));
            yold = yi;
        }
        // the sum is divided by FWHM itself, not the channel's width (cirsconv.f:159)
        yout[(int64_t)s * nconv + i] = __double2float_rn(__ddiv_rn(sum, (double)fwhm));
    }
}

// FWHM < 0: ytmp of cirsconv.f:205-213 for every (channel, calculated point),
// the channel's filter interpolated where the point lies inside it, else 0
__global__ void __launch_bounds__(kConvThreads)
filter_weights_kernel(int nwave, const float* __restrict__ vwave, const int* __restrict__ fil_of,
                      const int* __restrict__ fil_off, const float* __restrict__ vfil, const float* __restrict__ fil,
                      float* __restrict__ w, int* __restrict__ span) {
    __shared__ int s_lo, s_hi;
    const int i = blockIdx.x;
    const int k = fil_of[i];
    const float* X = vfil + fil_off[k];
    const float* Y = fil + fil_off[k];
    const int n = fil_off[k + 1] - fil_off[k];
    if (threadIdx.x == 0) {
        s_lo = nwave;
        s_hi = -1;
    }
    __syncthreads();
    int lo = nwave, hi = -1;
    for (int j = threadIdx.x; j < nwave; j += kConvThreads) {
        const float v = vwave[j];
        const float yt = (v >= X[0] && v <= X[n - 1]) ? interp_dev(X, Y, n, v, false) : 0.0f;
        w[(int64_t)i * nwave + j] = yt;
        if (yt != 0.0f) {
            lo = min(lo, j);
            hi = max(hi, j);
        }
    }
    atomicMin(&s_lo, lo);
    atomicMax(&s_hi, hi);
    __syncthreads();
    if (threadIdx.x == 0) {   // the points where the channel's weight is not zero
        span[2 * i] = s_lo;
        span[2 * i + 1] = s_hi;
    }
}

// FWHM < 0: the filter-weighted mean (cirsconv.f:220-237, xnorm true): DOUBLE
// sums of the REAL products ytmp*y*delv and ytmp*delv over the points below
// the last one where ytmp is not zero
__global__ void __launch_bounds__(kConvThreads)
filter_conv_kernel(int nwave, int nconv, const float* __restrict__ vwave, const float* __restrict__ y,
                   const float* __restrict__ w, const int* __restrict__ span, float* __restrict__ yout) {
    const int s = blockIdx.x;
    const float* ys = y + (int64_t)s * nwave;
    for (int i = threadIdx.x; i < nconv; i += kConvThreads) {
        const float* wi = w + (int64_t)i * nwave;
        double sum = 0.0, sumf = 0.0;
        // outside [lo, hi] every weight is zero and adds nothing
        const int lo = span[2 * i], hi = min(span[2 * i + 1], nwave - 2);
        for (int j = lo; j <= hi; ++j) {
            const float yt = wi[j];
            if (yt != 0.0f) {
                const float delv = __fsub_rn(vwave[j + 1], vwave[j]);
                sum = __dadd_rn(sum, (double)__fmul_rn(__fmul_rn(yt, ys[j]), delv));
                sumf = __dadd_rn(sumf, (double)__fmul_rn(yt, delv));
            }
        }
        yout[(int64_t)s * nconv + i] = __double2float_rn(__ddiv_rn(sum, sumf));
    }
}

__global__ void fill_kernel(float* p, int64_t n, float v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

size_t align16(size_t n) { return (n + 15) & ~(size_t)15; }

}  // namespace

int conv_check(rtb_context* c, float fwhm, int nwave, const float* vwave, const rtb_conv* cv, ConvSpec& out) {
    out = ConvSpec();
    out.fwhm = fwhm;
    if (!cv) {
        if (fwhm != 0.0f) return fail(c, RTB_ERR_ARG, "cirsconv: FWHM != 0 needs the channel list (rtb_conv)");
        return RTB_OK;
    }
    if (nwave <= 0 || !vwave) return fail(c, RTB_ERR_ARG, "cirsconv: no calculated points");
    if (cv->nconv <= 0 || !cv->vconv) return fail(c, RTB_ERR_ARG, "cirsconv: no channels (nconv, vconv)");
    out.vwave.assign(vwave, vwave + nwave);
    out.vconv.assign(cv->vconv, cv->vconv + cv->nconv);
    if (nwave == 1 && fwhm != 0.0f) {   // cirsconv.f:45-54 resets nconv to 1
        if (cv->nconv != 1) return fail(c, RTB_ERR_ARG, "cirsconv: one calculated point gives one channel (nconv=1)");
        return RTB_OK;
    }
    if (fwhm == 0.0f) {
        if (cv->nconv > nwave) return fail(c, RTB_ERR_ARG, "cirsconv: FWHM = 0 copies, so nconv <= nwave");
        return RTB_OK;
    }
    if (fwhm > 0.0f) {
        if (cv->nfwhm != 0) {
            if (cv->nfwhm < 2 || !cv->vfwhm || !cv->xfwhm)
                return fail(c, RTB_ERR_ARG, "cirsconv: a FWHM table needs at least two points");
            out.vfwhm.assign(cv->vfwhm, cv->vfwhm + cv->nfwhm);
            out.xfwhm.assign(cv->xfwhm, cv->xfwhm + cv->nfwhm);
        }
        return RTB_OK;
    }
    // FWHM < 0: filter channels
    if (cv->nfil <= 0 || !cv->vcen || !cv->nsub || !cv->vfil || !cv->fil)
        return fail(c, RTB_ERR_ARG, "cirsconv: FWHM < 0 needs the filter functions (nfil, vcen, nsub, vfil, fil)");
    out.fil_off.assign(1, 0);
    for (int k = 0; k < cv->nfil; ++k) {
        if (cv->nsub[k] < 2) return fail(c, RTB_ERR_ARG, "cirsconv: filter %d has fewer than two points", k);
        out.fil_off.push_back(out.fil_off.back() + cv->nsub[k]);
    }
    out.vfil.assign(cv->vfil, cv->vfil + out.fil_off.back());
    out.fil.assign(cv->fil, cv->fil + out.fil_off.back());
    out.fil_of.assign(cv->nconv, -1);
    for (int i = 0; i < cv->nconv; ++i) {
        // the last filter centred within 1e-5 of the channel (cirsconv.f:197-202)
        for (int k = 0; k < cv->nfil; ++k)
            if (std::fabs(cv->vcen[k] - cv->vconv[i]) < 0.00001f) out.fil_of[i] = k;
        if (out.fil_of[i] < 0)
            return fail(c, RTB_ERR_ARG, "cirsconv: no filter function centred on channel %d (%g)", i,
                        (double)cv->vconv[i]);
    }
    return RTB_OK;
}

int conv_run(rtb_context* c, const ConvSpec& cs, int nseg, const ConvSeg* seg, cudaStream_t st) {
    const int nwave = (int)cs.vwave.size(), nconv = (int)cs.vconv.size();
    int nser_max = 0;
    for (int q = 0; q < nseg; ++q) nser_max = std::max(nser_max, seg[q].nser);
    if (nser_max == 0) return RTB_OK;
    if (nwave == 1 && cs.fwhm != 0.0f) {
        for (int q = 0; q < nseg; ++q)
            if (seg[q].nser > 0) {
                fill_kernel<<<1, 128, 0, st>>>(seg[q].yout, seg[q].nser, 1.0f);
                CUDA_TRY(c, cudaGetLastError());
            }
        return RTB_OK;
    }
    if (cs.fwhm == 0.0f) {
        for (int q = 0; q < nseg; ++q)
            if (seg[q].nser > 0)
                CUDA_TRY(c, cudaMemcpy2DAsync(seg[q].yout, (size_t)nconv * 4, seg[q].y, (size_t)nwave * 4,
                                              (size_t)nconv * 4, seg[q].nser, cudaMemcpyDeviceToDevice, st));
        return RTB_OK;
    }
    // one upload of the channel description, then the scratch
    std::vector<char>& blob = c->h_conv;
    blob.clear();
    auto put = [&](const void* p, size_t n) {
        const size_t o = align16(blob.size());
        blob.resize(o + align16(n));
        if (n) std::memcpy(blob.data() + o, p, n);
        return o;
    };
    const size_t o_vw = put(cs.vwave.data(), nwave * 4), o_vc = put(cs.vconv.data(), nconv * 4);
    const size_t o_vf = put(cs.vfwhm.data(), cs.vfwhm.size() * 4), o_xf = put(cs.xfwhm.data(), cs.xfwhm.size() * 4);
    const size_t o_fo = put(cs.fil_of.data(), cs.fil_of.size() * 4), o_ff = put(cs.fil_off.data(), cs.fil_off.size() * 4);
    const size_t o_pv = put(cs.vfil.data(), cs.vfil.size() * 4), o_pf = put(cs.fil.data(), cs.fil.size() * 4);
    const size_t o_scr = align16(blob.size());
    // FWHM > 0: spline knots in shared memory when they fit, else in this scratch
    const size_t knot_bytes = conv_scratch_floats(nwave) * 4;
    const bool knots_shared = knot_bytes <= kConvSmemMax;
    const size_t n_scr = cs.fwhm > 0.0f ? (knots_shared ? 0 : (size_t)nser_max * knot_bytes)
                                        : (size_t)nconv * nwave * 4 + (size_t)nconv * 8;
    CUDA_TRY(c, c->d_conv.ensure(o_scr + n_scr + 16));
    char* d = (char*)c->d_conv.p;
    CUDA_TRY(c, cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, st));
    const float* dvw = (const float*)(d + o_vw);
    const float* dvc = (const float*)(d + o_vc);
    float* dscr = (float*)(d + o_scr);
    if (cs.fwhm > 0.0f) {
        if (knots_shared)
            CUDA_TRY(c, cudaFuncSetAttribute(cirsconv_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)knot_bytes));
        for (int q = 0; q < nseg; ++q)
            if (seg[q].nser > 0) {
                if (knots_shared)
                    cirsconv_kernel<true><<<seg[q].nser, kConvThreads, knot_bytes, st>>>(
                        nwave, dvw, seg[q].y, cs.fwhm, nconv, dvc, (int)cs.vfwhm.size(), (const float*)(d + o_vf),
                        (const float*)(d + o_xf), seg[q].yout, dscr);
                else
                    cirsconv_kernel<false><<<seg[q].nser, kConvThreads, 0, st>>>(
                        nwave, dvw, seg[q].y, cs.fwhm, nconv, dvc, (int)cs.vfwhm.size(), (const float*)(d + o_vf),
                        (const float*)(d + o_xf), seg[q].yout, dscr);
                CUDA_TRY(c, cudaGetLastError());
            }
        return RTB_OK;
    }
    int* dspan = (int*)(dscr + (size_t)nconv * nwave);
    filter_weights_kernel<<<nconv, kConvThreads, 0, st>>>(nwave, dvw, (const int*)(d + o_fo), (const int*)(d + o_ff),
                                                          (const float*)(d + o_pv), (const float*)(d + o_pf), dscr,
                                                          dspan);
    CUDA_TRY(c, cudaGetLastError());
    for (int q = 0; q < nseg; ++q)
        if (seg[q].nser > 0) {
            filter_conv_kernel<<<seg[q].nser, kConvThreads, 0, st>>>(nwave, nconv, dvw, seg[q].y, dscr, dspan,
                                                                     seg[q].yout);
            CUDA_TRY(c, cudaGetLastError());
        }
    return RTB_OK;
}

}  // namespace rtb

using namespace rtb;

extern "C" int rtb_cirsconv_ex(rtb_context* c, float fwhm, int nwave, const float* vwave, int nser, const float* y,
                               const rtb_conv* conv, float* yout) {
    if (!c) return RTB_ERR_ARG;
    if (nwave <= 0 || nser <= 0 || !vwave || !y || !conv || !yout) return fail(c, RTB_ERR_ARG, "cirsconv: bad arguments");
    ConvSpec cs;
    const int r = conv_check(c, fwhm, nwave, vwave, conv, cs);
    if (r) return r;
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const int nconv = conv->nconv;
    const size_t ny = (size_t)nser * nwave, no = (size_t)nser * nconv;
    CUDA_TRY(c, c->d_nt32.ensure((ny + no) * sizeof(float) + 64));
    float* dy = (float*)c->d_nt32.p;
    float* dout = dy + ((ny + 3) & ~(size_t)3);
    CUDA_TRY(c, cudaMemcpyAsync(dy, y, ny * 4, cudaMemcpyHostToDevice, st));
    const ConvSeg seg{dy, nser, dout};
    const int r2 = conv_run(c, cs, 1, &seg, st);
    if (r2) return r2;
    CUDA_TRY(c, cudaMemcpyAsync(yout, dout, no * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    return RTB_OK;
}

extern "C" int rtb_cirsconv(rtb_context* c, int nwave, const float* vwave, int nser, const float* y, float fwhm,
                            int nconv, const float* vconv, float* yout) {
    if (!c) return RTB_ERR_ARG;
    if (fwhm < 0.0f)
        return fail(c, RTB_ERR_UNSUPPORTED, "cirsconv: FWHM < 0 takes the filter functions (rtb_cirsconv_ex)");
    if (fwhm == 0.0f && nconv != nwave) return fail(c, RTB_ERR_ARG, "cirsconv: FWHM = 0 needs nconv == nwave");
    rtb_conv cv;
    std::memset(&cv, 0, sizeof cv);
    cv.nconv = nconv;
    cv.vconv = vconv;
    return rtb_cirsconv_ex(c, fwhm, nwave, vwave, nser, y, &cv, yout);
}
