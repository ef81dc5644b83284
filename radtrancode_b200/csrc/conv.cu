// conv.cu -- instrument convolution of calculated spectra on the device.
//
// Reference: radtran/cirsrad/cirsconv.f:12-160 (FWHM > 0: a natural cubic
// spline through the calculated points, CSPLINE rtm_util/cspline.f, read by
// CSPLINT rtm_util/csplint.f at 20 equally spaced points across each
// channel's square bin, trapezoid sum in DOUBLE PRECISION; FWHM = 0: a copy)
// as cirsrtfg_wave.f:448-516 applies it to the radiance, d/dtsurf and every
// Jacobian row.  One block per series: thread 0 builds the extrapolated,
// NaN-free knot list and solves the spline's tridiagonal system (a sequential
// recurrence), then the block's threads fill the channels.  REAL arithmetic
// is written with explicitly rounded intrinsics so that it rounds as the
// reference's does.
#include <cuda_runtime.h>

#include "context.h"

namespace rtb {

namespace {

constexpr int kConvThreads = 128;
constexpr int kNstep = 20;   // cirsconv.f: PARAMETER (nstep=20)

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

__global__ void __launch_bounds__(kConvThreads)
cirsconv_kernel(int nwave, const float* __restrict__ vwave, const float* __restrict__ y, float fwhm, int nconv,
                const float* __restrict__ vconv, float* __restrict__ yout, float* __restrict__ scr) {
    __shared__ int s_nc;
    const int s = blockIdx.x;
    const float* ys = y + (int64_t)s * nwave;
    const int cap = nwave + 2;
    float* xc = scr + (int64_t)s * 4 * cap;
    float* yc = xc + cap;
    float* y2 = yc + cap;
    float* u = y2 + cap;
    if (threadIdx.x == 0) {
        const float half = __fdiv_rn(fwhm, 2.0f);
        int nc = 0;
        // extrapolated end points (cirsconv.f:77-104), then the points, NaNs dropped (:107-132)
        const bool lo = vconv[0] < __fadd_rn(vwave[0], half);
        const bool hi = vconv[nconv - 1] > __fsub_rn(vwave[nwave - 1], half);
        if (lo) {
            const float x = __fsub_rn(vconv[0], fwhm);
            const float sl = __fdiv_rn(__fsub_rn(ys[1], ys[0]), __fsub_rn(vwave[1], vwave[0]));
            const float v = __fadd_rn(ys[0], __fmul_rn(sl, __fsub_rn(x, vwave[0])));
            if (!isnan(v)) {
                xc[nc] = x;
                yc[nc] = v;
                ++nc;
            }
        }
        for (int i = 0; i < nwave; ++i)
            if (!isnan(ys[i])) {
                xc[nc] = vwave[i];
                yc[nc] = ys[i];
                ++nc;
            }
        if (hi) {
            const float x = __fadd_rn(vconv[nconv - 1], fwhm);
            const float sl = __fdiv_rn(__fsub_rn(ys[nwave - 1], ys[nwave - 2]),
                                       __fsub_rn(vwave[nwave - 1], vwave[nwave - 2]));
            const float v = __fadd_rn(ys[nwave - 1], __fmul_rn(sl, __fsub_rn(x, vwave[nwave - 1])));
            if (!isnan(v)) {
                xc[nc] = x;
                yc[nc] = v;
                ++nc;
            }
        }
        // CSPLINE with natural ends (YP1, YPN > .99E30)
        y2[0] = 0.0f;
        u[0] = 0.0f;
        for (int i = 1; i < nc - 1; ++i) {
            const float sig = __fdiv_rn(__fsub_rn(xc[i], xc[i - 1]), __fsub_rn(xc[i + 1], xc[i - 1]));
            const float p = __fadd_rn(__fmul_rn(sig, y2[i - 1]), 2.0f);
            y2[i] = __fdiv_rn(__fsub_rn(sig, 1.0f), p);
            if (xc[i - 1] == xc[i] || xc[i] == xc[i + 1]) {
                u[i] = u[i - 1];
                continue;
            }
            const float d1 = __fdiv_rn(__fsub_rn(yc[i + 1], yc[i]), __fsub_rn(xc[i + 1], xc[i]));
            const float d0 = __fdiv_rn(__fsub_rn(yc[i], yc[i - 1]), __fsub_rn(xc[i], xc[i - 1]));
            const float t = __fdiv_rn(__fmul_rn(6.0f, __fsub_rn(d1, d0)), __fsub_rn(xc[i + 1], xc[i - 1]));
            u[i] = __fdiv_rn(__fsub_rn(t, __fmul_rn(sig, u[i - 1])), p);
        }
        if (nc >= 2) {
            y2[nc - 1] = __fdiv_rn(__fsub_rn(0.0f, __fmul_rn(0.0f, u[nc - 2])),
                                   __fadd_rn(__fmul_rn(0.0f, y2[nc - 2]), 1.0f));
            for (int k = nc - 2; k >= 0; --k) y2[k] = __fadd_rn(__fmul_rn(y2[k], y2[k + 1]), u[k]);
        }
        s_nc = nc;
    }
    __syncthreads();
    const int nc = s_nc;
    for (int i = threadIdx.x; i < nconv; i += kConvThreads) {
        const float half = __fdiv_rn(fwhm, 2.0f);
        const float x1 = __fsub_rn(vconv[i], half), x2 = __fadd_rn(vconv[i], half);
        const float delx = __fdiv_rn(__fsub_rn(x2, x1), (float)(kNstep - 1));
        const double hd = (double)__fdiv_rn(delx, 2.0f);
        double sum = 0.0, yold = 0.0;
        for (int j = 1; j <= kNstep; ++j) {
            const float xi = __fadd_rn(x1, __fmul_rn((float)(j - 1), delx));
            const double yi = nc >= 2 ? (double)csplint_dev(xc, yc, y2, nc, xi) : 0.0;
            if (j > 1) sum = __dadd_rn(sum, __dmul_rn(__dadd_rn(yi, yold), hd));
            yold = yi;
        }
        yout[(int64_t)s * nconv + i] = __double2float_rn(__ddiv_rn(sum, (double)fwhm));
    }
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" int rtb_cirsconv(rtb_context* c, int nwave, const float* vwave, int nser, const float* y, float fwhm,
                            int nconv, const float* vconv, float* yout) {
    if (!c) return RTB_ERR_ARG;
    if (nwave <= 0 || nser <= 0 || nconv <= 0 || !vwave || !y || !vconv || !yout)
        return fail(c, RTB_ERR_ARG, "cirsconv: bad arguments");
    if (fwhm == 0.0f) {   // cirsconv.f:141-147: the outputs are the inputs
        if (nconv != nwave) return fail(c, RTB_ERR_ARG, "cirsconv: FWHM = 0 needs nconv == nwave");
        for (size_t i = 0; i < (size_t)nser * nwave; ++i) yout[i] = y[i];
        return RTB_OK;
    }
    if (fwhm < 0.0f) return fail(c, RTB_ERR_UNSUPPORTED, "cirsconv: FWHM < 0 (filter-file channels) not implemented");
    if (nwave < 2) return fail(c, RTB_ERR_ARG, "cirsconv: FWHM > 0 needs at least two calculated points");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const size_t ny = (size_t)nser * nwave, no = (size_t)nser * nconv, ns = (size_t)nser * 4 * (nwave + 2);
    CUDA_TRY(c, c->d_nt32.ensure((nwave + nconv + ny + no + ns) * sizeof(float) + 64));
    float* dv = (float*)c->d_nt32.p;
    float* dc = dv + nwave;
    float* dy = dc + nconv;
    float* dout = dy + ny;
    float* dscr = dout + no;
    CUDA_TRY(c, cudaMemcpyAsync(dv, vwave, (size_t)nwave * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dc, vconv, (size_t)nconv * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dy, y, ny * 4, cudaMemcpyHostToDevice, st));
    cirsconv_kernel<<<nser, kConvThreads, 0, st>>>(nwave, dv, dy, fwhm, nconv, dc, dout, dscr);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(yout, dout, no * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    return RTB_OK;
}
