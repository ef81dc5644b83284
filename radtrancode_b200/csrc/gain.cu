// gain.cu -- drop-in calc_gain_matrix, calcnextxn and calc_serr on the device.
//
// Reference: nemesis/calc_gain_matrix.f:123-163 (nx < ny branch: C = K^T Se^-1 K
// + Sa^-1, A = C^-1 by dinvertm jmod=2, D = A K^T Se^-1, AA = D K) and
// nemesis/calcnextxn.f:64-104 (x_out = x0 + D (y - yn) - AA (x0 - xn)) and
// nemesis/calc_serr.f (Sm = D Se D^T, Sn = (AA - I) Sa (AA - I)^T, St = Sn + Sm).  The
// reference works in DOUBLE PRECISION on promoted REAL inputs; so do these
// kernels (FP64 on the CUDA cores; the sizes are small: 2 NX^2 NY flops per
// product).  The fused batched step (newton.cu) is the fast path; these
// entry points exist for callers that keep the reference's D / AA interface.
#include <cuda_runtime.h>

#include <vector>

#include "context.h"
#include "newton.h"

namespace rtb {

namespace {

constexpr int kT = 16;   // output tile edge, and k chunk

// C(m, n) = scale_n(n) * sum_k A(m, k) B(k, n) scale_k(k) + add(m, n)
// A(m, k) = A[m * am + k * ak], B(k, n) = B[k * bk + n * bn],
// C(m, n) = C[m * cm + n * cn], add(m, n) = add[m * dm + n * dn].
template <class TA, class TB>
__global__ void __launch_bounds__(kT * kT)
tile_gemm(int M, int N, int K, const TA* __restrict__ A, int64_t am, int64_t ak, const TB* __restrict__ B,
          int64_t bk, int64_t bn, const double* __restrict__ scale_k, const double* __restrict__ scale_n,
          const double* __restrict__ add, int64_t dm, int64_t dn, double* __restrict__ C, int64_t cm, int64_t cn) {
    __shared__ double As[kT][kT + 1];
    __shared__ double Bs[kT][kT + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int m = blockIdx.y * kT + ty, n = blockIdx.x * kT + tx;
    double acc = 0.0;
    for (int k0 = 0; k0 < K; k0 += kT) {
        const int ka = k0 + tx, kb = k0 + ty;
        const int mA = blockIdx.y * kT + ty, nB = blockIdx.x * kT + tx;
        double a = 0.0, b = 0.0;
        if (mA < M && ka < K) {
            a = (double)A[mA * am + ka * ak];
            if (scale_k) a *= scale_k[ka];
        }
        if (kb < K && nB < N) b = (double)B[kb * bk + nB * bn];
        As[ty][tx] = a;
        Bs[ty][tx] = b;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kT; ++k) acc = fma(As[ty][k], Bs[k][tx], acc);
        __syncthreads();
    }
    if (m < M && n < N) {
        if (scale_n) acc *= scale_n[n];
        if (add) acc += add[m * dm + n * dn];
        C[m * cm + n * cn] = acc;
    }
}

// x_out(a) = x0(a) + sngl(D(a,:) (y - yn) - AA(a,:) (x0 - xn)), differences
// in REAL (calcnextxn.f:84-104); one warp per state element.
__global__ void __launch_bounds__(256)
nextxn_kernel(int nx, int ny, const double* __restrict__ dd, int64_t ldx, const double* __restrict__ aa,
              const float* __restrict__ x0, const float* __restrict__ xn, const float* __restrict__ y,
              const float* __restrict__ yn, float* __restrict__ x_out) {
    const int lane = threadIdx.x & 31;
    const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (a >= nx) return;
    double x2 = 0.0, x1 = 0.0;
    for (int i = lane; i < ny; i += 32) x2 = fma(dd[a + ldx * i], (double)(y[i] - yn[i]), x2);
    for (int b = lane; b < nx; b += 32) x1 = fma(aa[a + ldx * b], (double)(x0[b] - xn[b]), x1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x2 += __shfl_xor_sync(0xffffffffu, x2, o);
        x1 += __shfl_xor_sync(0xffffffffu, x1, o);
    }
    if (lane == 0) x_out[a] = x0[a] + (float)(x2 - x1);
}

// E = aa - I, aa(ldx, nx) column-major -> E row-major [nx][nx]
__global__ void aa_minus_identity(int nx, const double* __restrict__ aa, int64_t ldx, double* __restrict__ E) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * nx) return;
    const int a = e / nx, b = e - a * nx;
    E[e] = aa[a + ldx * b] - (a == b ? 1.0 : 0.0);
}

template <class TA, class TB>
cudaError_t gemm(int M, int N, int K, const TA* A, int64_t am, int64_t ak, const TB* B, int64_t bk, int64_t bn,
                 const double* sk, const double* sn, const double* add, int64_t dm, int64_t dn, double* C,
                 int64_t cm, int64_t cn, cudaStream_t st) {
    const dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT), block(kT, kT);
    tile_gemm<TA, TB><<<grid, block, 0, st>>>(M, N, K, A, am, ak, B, bk, bn, sk, sn, add, dm, dn, C, cm, cn);
    return cudaGetLastError();
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" {

int rtb_calc_gain_matrix(rtb_context* c, int nx, int ny, int ldx, int ldy, const float* kk, const double* sxi,
                         const double* sei, double* dd, double* aa, int* nonpd) {
    if (!c) return RTB_ERR_ARG;
    if (nx <= 0 || ny <= 0 || ldx < nx || ldy < ny || !kk || !sxi || !sei || !dd || !aa)
        return fail(c, RTB_ERR_ARG, "calc_gain_matrix: bad arguments");
    if (nx > kNewtonMaxNx) return fail(c, RTB_ERR_UNSUPPORTED, "nx=%d > %d", nx, kNewtonMaxNx);
    if (nx >= ny) return fail(c, RTB_ERR_UNSUPPORTED, "nx >= ny (calc_gain_matrix.f:86-121 branch not implemented)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const size_t nn = (size_t)nx * nx, nd = (size_t)nx * ny;
    // f32: K^T [nx][ny]; f64: Sa^-1 [nx][nx] | sei [ny] | C | C^-1 | D [nx][ny] (row-major) | AA | status
    CUDA_TRY(c, c->d_nt32.ensure(nd * 4));
    CUDA_TRY(c, c->d_nt64.ensure((4 * nn + ny + nd + 8) * 8));
    float* kt = (float*)c->d_nt32.p;
    double* sai = (double*)c->d_nt64.p;
    double* se = sai + nn;
    double* C = se + ny;
    double* Ci = C + nn;
    double* D = Ci + nn;
    double* AA = D + nd;
    unsigned* status = (unsigned*)(AA + nn);
    // kk(ldy, nx) column-major: column j (over i) is row j of K^T
    CUDA_TRY(c, cudaMemcpy2DAsync(kt, (size_t)ny * 4, kk, (size_t)ldy * 4, (size_t)ny * 4, nx,
                                  cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpy2DAsync(sai, (size_t)nx * 8, sxi, (size_t)ldx * 8, (size_t)nx * 8, nx,
                                  cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(se, sei, (size_t)ny * 8, cudaMemcpyHostToDevice, st));
    // C(a, b) = sum_i K(i, a) Se^-1(i) K(i, b) + Sa^-1(a, b)   (Sa^-1 stored column-major = (b, a) row-major)
    CUDA_TRY(c, (gemm<float, float>(nx, nx, ny, kt, ny, 1, kt, 1, ny, se, nullptr, sai, 1, nx, C, nx, 1, st)));
    CUDA_TRY(c, launch_spd_inverse(C, Ci, nx, 0, 1, status, st));
    // D(a, i) = Se^-1(i) sum_b C^-1(a, b) K(i, b)
    CUDA_TRY(c, (gemm<double, float>(nx, ny, nx, Ci, nx, 1, kt, ny, 1, nullptr, se, nullptr, 0, 0, D, ny, 1, st)));
    // AA(a, b) = sum_i D(a, i) K(i, b)
    CUDA_TRY(c, (gemm<double, float>(nx, nx, ny, D, ny, 1, kt, 1, ny, nullptr, nullptr, nullptr, 0, 0, AA, nx, 1,
                                     st)));
    // back to the caller's dd(ldx, ny) and aa(ldx, nx), column-major
    std::vector<double> hd(nd), ha(nn);
    unsigned hs = 0;
    CUDA_TRY(c, cudaMemcpyAsync(hd.data(), D, nd * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(ha.data(), AA, nn * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(&hs, status, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    for (int a = 0; a < nx; ++a) {
        for (int i = 0; i < ny; ++i) dd[a + (size_t)ldx * i] = hd[(size_t)a * ny + i];
        for (int b = 0; b < nx; ++b) aa[a + (size_t)ldx * b] = ha[(size_t)a * nx + b];
    }
    if (nonpd) *nonpd = (hs & kNtNonPd) ? 1 : 0;
    return RTB_OK;
}

int rtb_calc_serr(rtb_context* c, int nx, int ny, int ldx, const float* sx, const float* se, const double* dd,
                  const double* aa, float* st, float* sn, float* sm) {
    if (!c) return RTB_ERR_ARG;
    if (nx <= 0 || ny <= 0 || ldx < nx || !sx || !se || !dd || !aa || !st || !sn || !sm)
        return fail(c, RTB_ERR_ARG, "calc_serr: bad arguments");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st_ = stream_of(c);
    const size_t nn = (size_t)nx * nx, ndl = (size_t)ldx * ny, nal = (size_t)ldx * nx;
    // f64: D (ldx, ny) | AA (ldx, nx) | se [ny] | Sa [nx][nx] col-major | E | C | Sm | Sn | St
    CUDA_TRY(c, c->d_nt64.ensure((ndl + nal + ny + 6 * nn) * 8));
    double* D = (double*)c->d_nt64.p;
    double* AA = D + ndl;
    double* sed = AA + nal;
    double* sxd = sed + ny;
    double* E = sxd + nn;
    double* Cm = E + nn;
    double* Sm = Cm + nn;
    double* Sn = Sm + nn;
    double* St = Sn + nn;
    std::vector<double> h_se(se, se + ny), h_sx(nn);
    for (int j = 0; j < nx; ++j)
        for (int i = 0; i < nx; ++i) h_sx[i + (size_t)nx * j] = (double)sx[i + (size_t)ldx * j];
    CUDA_TRY(c, cudaMemcpyAsync(D, dd, ndl * 8, cudaMemcpyHostToDevice, st_));
    CUDA_TRY(c, cudaMemcpyAsync(AA, aa, nal * 8, cudaMemcpyHostToDevice, st_));
    CUDA_TRY(c, cudaMemcpyAsync(sed, h_se.data(), (size_t)ny * 8, cudaMemcpyHostToDevice, st_));
    CUDA_TRY(c, cudaMemcpyAsync(sxd, h_sx.data(), nn * 8, cudaMemcpyHostToDevice, st_));
    // Sm(a, b) = sum_i D(a, i) Se(i) D(b, i)
    CUDA_TRY(c, (gemm<double, double>(nx, nx, ny, D, 1, ldx, D, ldx, 1, sed, nullptr, nullptr, 0, 0, Sm, nx, 1,
                                      st_)));
    aa_minus_identity<<<(int)((nn + 255) / 256), 256, 0, st_>>>(nx, AA, ldx, E);
    CUDA_TRY(c, cudaGetLastError());
    // C = E Sa, Sn = C E^T, St = C E^T + Sm
    CUDA_TRY(c, (gemm<double, double>(nx, nx, nx, E, nx, 1, sxd, 1, nx, nullptr, nullptr, nullptr, 0, 0, Cm, nx, 1,
                                      st_)));
    CUDA_TRY(c, (gemm<double, double>(nx, nx, nx, Cm, nx, 1, E, 1, nx, nullptr, nullptr, nullptr, 0, 0, Sn, nx, 1,
                                      st_)));
    CUDA_TRY(c, (gemm<double, double>(nx, nx, nx, Cm, nx, 1, E, 1, nx, nullptr, nullptr, Sm, nx, 1, St, nx, 1,
                                      st_)));
    std::vector<double> h((size_t)3 * nn);
    CUDA_TRY(c, cudaMemcpyAsync(h.data(), Sm, 3 * nn * 8, cudaMemcpyDeviceToHost, st_));
    CUDA_TRY(c, cudaStreamSynchronize(st_));
    // REAL outputs (ldx, nx), column-major (calc_serr.f sngl copies)
    for (int a = 0; a < nx; ++a)
        for (int b = 0; b < nx; ++b) {
            const size_t k = (size_t)a * nx + b, o = a + (size_t)ldx * b;
            sm[o] = (float)h[k];
            sn[o] = (float)h[nn + k];
            st[o] = (float)h[2 * nn + k];
        }
    return RTB_OK;
}

int rtb_calcnextxn(rtb_context* c, int nx, int ny, int ldx, const float* x0, const float* xn, const float* y,
                   const float* yn, const double* dd, const double* aa, float* x_out) {
    if (!c) return RTB_ERR_ARG;
    if (nx <= 0 || ny <= 0 || ldx < nx || !x0 || !xn || !y || !yn || !dd || !aa || !x_out)
        return fail(c, RTB_ERR_ARG, "calcnextxn: bad arguments");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const cudaStream_t st = stream_of(c);
    const size_t nd = (size_t)ldx * ny, na = (size_t)ldx * nx;
    CUDA_TRY(c, c->d_nt64.ensure((nd + na) * 8));
    CUDA_TRY(c, c->d_nt32.ensure((size_t)(3 * nx + 2 * ny) * 4));
    double* D = (double*)c->d_nt64.p;
    double* AA = D + nd;
    float* f = (float*)c->d_nt32.p;
    float *dx0 = f, *dxn = f + nx, *dxo = f + 2 * nx, *dy = f + 3 * nx, *dyn = dy + ny;
    CUDA_TRY(c, cudaMemcpyAsync(D, dd, nd * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(AA, aa, na * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dx0, x0, (size_t)nx * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dxn, xn, (size_t)nx * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dy, y, (size_t)ny * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(dyn, yn, (size_t)ny * 4, cudaMemcpyHostToDevice, st));
    nextxn_kernel<<<(nx + 7) / 8, 256, 0, st>>>(nx, ny, D, ldx, AA, dx0, dxn, dy, dyn, dxo);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(x_out, dxo, (size_t)nx * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    return RTB_OK;
}

}  // extern "C"
