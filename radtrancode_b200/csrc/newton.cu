// newton.cu -- batched optimal-estimation Newton step (one block per retrieval).
//
// Reference: nemesis/calc_gain_matrix.f:123-163 (nx < ny branch), the
// Cholesky inverse of radtran/matrices/dinvertm.f:114-141 with dcholdc.f and
// dcholsl.f, nemesis/calcnextxn.f:64-104 and nemesis/calc_phiret.f:49-102.
//
// With C = K^T Se^-1 K + Sa^-1 and a diagonal Se the reference's
//     x_out = xa + D (y - yn) - AA (xa - xn),   D = C^-1 K^T Se^-1,  AA = D K
// equals
//     x_out = xa + C^-1 K^T Se^-1 (y - yn + K (xn - xa)),
// so neither D (NX x NY) nor AA is formed.  Per retrieval:
//   1. N = K^T Se^-1 K.  Default: tensor cores.  K~ = Se^-1/2 K is split into
//      bf16 hi + lo parts; three m16n8k16 MMAs per tile (hi*hi + hi*lo +
//      lo*hi) accumulate in FP32, about 2^-17 relative error per product.
//      Alternative: FP64 on the CUDA cores (the all-FP64 solve).
//   2. C = N + Sa^-1 in FP64 shared memory; Cholesky in FP64 with the
//      reference's non-positive-pivot rule (pivot 1, continue).
//   3. rhs = K^T Se^-1 (y - yn + K d) with FP64 accumulation of the FP32 K.
//   4. dx = C^-1 rhs, then `refine` steps dx += C^-1 (rhs - C_exact dx) where
//      C_exact applies K^T Se^-1 K through K in FP64 (never through N).
//   5. x_out = xa + (float)dx.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "newton.h"

namespace rtb {

namespace {

constexpr int kNt = 256;                  // threads per block (8 warps)
constexpr int kNw = kNt / 32;
constexpr int kNp = kNewtonMaxNx;         // padded state size of the tensor-core tile
constexpr int kKc = 32;                   // wavenumbers per staged chunk
constexpr int kLds = kKc + 8;             // bf16 row stride of a staging tile (80 B: conflict-free fragments)
constexpr int kStageMma = 2 * kNp * kLds * 2 + kKc * 4;
constexpr int kStageF64 = kKc * kNp * 8 + kKc * 8;

__host__ __device__ constexpr int region_bytes(int nx) {
    return ((nx * nx * 8 > (kStageMma > kStageF64 ? kStageMma : kStageF64)
                 ? nx * nx * 8
                 : (kStageMma > kStageF64 ? kStageMma : kStageF64)) + 15) & ~15;
}
// region (staging aliased with C) + d, rhs, dx, res (kNp doubles each)
__host__ __device__ constexpr int newton_smem(int nx) { return region_bytes(nx) + 8 * 4 * kNp; }

__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (unsigned)__bfloat16_as_ushort(a) | ((unsigned)__bfloat16_as_ushort(b) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// C (nx x nx, row-major FP64) = K~^T K~ + Sa^-1 with the tensor-core split.
// Warp w owns output rows 32*(w>>1).. and columns 64*(w&1).. of the 128x128 tile.
__device__ void hessian_mma(const NewtonDev& R, char* sm, double* C) {
    __nv_bfloat16* Xh = (__nv_bfloat16*)sm;
    __nv_bfloat16* Xl = Xh + kNp * kLds;
    float* sc = (float*)(Xl + kNp * kLds);
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int m0 = (warp >> 1) * 32, n0 = (warp & 1) * 64;
    float acc[2][8][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    const int srow = tid >> 1, scol = (tid & 1) * 16;   // staging: row, 16 consecutive wavenumbers
    const float* krow = R.kt + (int64_t)srow * ny;
    for (int k0 = 0; k0 < ny; k0 += kKc) {
        __syncthreads();
        if (tid < kKc) sc[tid] = k0 + tid < ny ? (float)sqrt(R.sei[k0 + tid]) : 0.0f;
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 16; u += 2) {
            const int nu = k0 + scol + u;
            float v0 = 0.0f, v1 = 0.0f;
            if (srow < nx) {
                if (nu < ny) v0 = krow[nu] * sc[scol + u];
                if (nu + 1 < ny) v1 = krow[nu + 1] * sc[scol + u + 1];
            }
            const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
            const __nv_bfloat16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
            const __nv_bfloat16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
            *(unsigned*)&Xh[srow * kLds + scol + u] = pack_bf16(h0, h1);
            *(unsigned*)&Xl[srow * kLds + scol + u] = pack_bf16(l0, l1);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kKc; kk += 16) {
            const int c0 = kk + 2 * t4;
            unsigned ah[2][4], al[2][4];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int row = m0 + a * 16 + g;
                ah[a][0] = *(const unsigned*)&Xh[row * kLds + c0];
                ah[a][1] = *(const unsigned*)&Xh[(row + 8) * kLds + c0];
                ah[a][2] = *(const unsigned*)&Xh[row * kLds + c0 + 8];
                ah[a][3] = *(const unsigned*)&Xh[(row + 8) * kLds + c0 + 8];
                al[a][0] = *(const unsigned*)&Xl[row * kLds + c0];
                al[a][1] = *(const unsigned*)&Xl[(row + 8) * kLds + c0];
                al[a][2] = *(const unsigned*)&Xl[row * kLds + c0 + 8];
                al[a][3] = *(const unsigned*)&Xl[(row + 8) * kLds + c0 + 8];
            }
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const int col = n0 + b * 8 + g;     // B(k, n) = X(n, k): column-major B from the row tile
                const unsigned bh[2] = {*(const unsigned*)&Xh[col * kLds + c0],
                                        *(const unsigned*)&Xh[col * kLds + c0 + 8]};
                const unsigned bl[2] = {*(const unsigned*)&Xl[col * kLds + c0],
                                        *(const unsigned*)&Xl[col * kLds + c0 + 8]};
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    mma_bf16(acc[a][b], ah[a], bh);
                    mma_bf16(acc[a][b], ah[a], bl);
                    mma_bf16(acc[a][b], al[a], bh);
                }
            }
        }
    }
    __syncthreads();   // the staging tiles are dead: C overwrites them
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + a * 16 + g + 8 * h, col = n0 + b * 8 + 2 * t4;
                if (row < nx) {
                    if (col < nx) C[row * nx + col] = (double)acc[a][b][2 * h] + R.sai[row * nx + col];
                    if (col + 1 < nx)
                        C[row * nx + col + 1] = (double)acc[a][b][2 * h + 1] + R.sai[row * nx + col + 1];
                }
            }
    __syncthreads();
}

// C = K^T Se^-1 K + Sa^-1 in FP64 on the CUDA cores; thread (ti, tj) owns an 8x8 tile
__device__ void hessian_f64(const NewtonDev& R, char* sm, double* C) {
    double* Kt = (double*)sm;          // [kKc][kNp]
    double* se = Kt + kKc * kNp;       // [kKc]
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, ti = tid >> 4, tj = tid & 15;
    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
    for (int k0 = 0; k0 < ny; k0 += kKc) {
        __syncthreads();
        for (int e = tid; e < kNp * kKc; e += kNt) {
            const int i = e / kKc, k = e - i * kKc, nu = k0 + k;
            Kt[k * kNp + i] = (i < nx && nu < ny) ? (double)R.kt[(int64_t)i * ny + nu] : 0.0;
        }
        if (tid < kKc) se[tid] = k0 + tid < ny ? R.sei[k0 + tid] : 0.0;
        __syncthreads();
        for (int k = 0; k < kKc; ++k) {
            double a[8], b[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) a[r] = Kt[k * kNp + ti * 8 + r];
#pragma unroll
            for (int c = 0; c < 8; ++c) b[c] = Kt[k * kNp + tj * 8 + c] * se[k];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int row = ti * 8 + r, col = tj * 8 + c;
            if (row < nx && col < nx) C[row * nx + col] = acc[r][c] + R.sai[row * nx + col];
        }
    __syncthreads();
}

// In-place Cholesky C = L L^T (lower triangle, row-major, stride n).
// A pivot <= 0 becomes 1 and the factorisation goes on (dcholdc.f:69-84);
// a NaN pivot propagates as in the reference (sqrt of NaN).
__device__ bool cholesky(double* C, int n) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool bad = false;
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            const double v = C[k * n + k];
            if (v <= 0.0) {
                C[k * n + k] = 1.0;
                bad = true;
            } else {
                C[k * n + k] = sqrt(v);
            }
        }
        __syncthreads();
        const double p = C[k * n + k];
        for (int i = k + 1 + tid; i < n; i += kNt) C[i * n + k] = C[i * n + k] / p;
        __syncthreads();
        for (int i = k + 1 + warp; i < n; i += kNw) {
            const double lik = C[i * n + k];
            for (int j = k + 1 + lane; j <= i; j += 32) C[i * n + j] -= lik * C[j * n + k];
        }
        __syncthreads();
    }
    return bad;
}

// Solve L L^T x = b in place in v (one warp; L from cholesky)
__device__ void chol_solve_warp(const double* L, int n, double* v) {
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < n; ++j) {
        __syncwarp();
        const double zj = v[j] / L[j * n + j];
        __syncwarp();
        if (lane == 0) v[j] = zj;
        for (int i = j + 1 + lane; i < n; i += 32) v[i] -= L[i * n + j] * zj;
    }
    for (int j = n - 1; j >= 0; --j) {
        __syncwarp();
        const double zj = v[j] / L[j * n + j];
        __syncwarp();
        if (lane == 0) v[j] = zj;
        for (int i = lane; i < j; i += 32) v[i] -= L[j * n + i] * zj;
    }
    __syncwarp();
}

// out = (K^T Se^-1 K + Sa^-1) x, K applied in FP64 from FP32 (work: ny doubles)
__device__ void apply_c_exact(const NewtonDev& R, const double* x, double* out) {
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int nu = tid; nu < ny; nu += kNt) {
        double s = 0.0;
        for (int i = 0; i < nx; ++i) s = fma((double)R.kt[(int64_t)i * ny + nu], x[i], s);
        R.work[nu] = s * R.sei[nu];
    }
    __syncthreads();
    for (int i = warp; i < nx; i += kNw) {
        const float* krow = R.kt + (int64_t)i * ny;
        double s = 0.0;
        for (int nu = lane; nu < ny; nu += 32) s = fma((double)krow[nu], R.work[nu], s);
        for (int j = lane; j < nx; j += 32) s = fma(R.sai[i * nx + j], x[j], s);
        s = warp_sum(s);
        if (lane == 0) out[i] = s;
    }
    __syncthreads();
}

template <int kHess>
__global__ void __launch_bounds__(kNt, 1)
newton_step_kernel(const NewtonDev* __restrict__ rets, int refine, unsigned* __restrict__ status,
                   double* __restrict__ resid) {
    extern __shared__ __align__(16) char smem[];
    const NewtonDev R = rets[blockIdx.x];
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* C = (double*)smem;
    double* d = (double*)(smem + region_bytes(kNp));
    double* rhs = d + kNp;
    double* dx = rhs + kNp;
    double* res = dx + kNp;
    if (kHess == 0) hessian_mma(R, smem, C); else hessian_f64(R, smem, C);
    // d = xn - xa (REAL difference, calcnextxn.f:84-86 with the sign folded in)
    for (int i = tid; i < kNp; i += kNt) d[i] = i < nx ? (double)(R.xn[i] - R.xa[i]) : 0.0;
    __syncthreads();
    // work = Se^-1 ((y - yn) + K d), (y - yn) REAL as calcnextxn.f:92
    for (int nu = tid; nu < ny; nu += kNt) {
        double s = 0.0;
        for (int i = 0; i < nx; ++i) s = fma((double)R.kt[(int64_t)i * ny + nu], d[i], s);
        R.work[nu] = ((double)(R.y[nu] - R.yn[nu]) + s) * R.sei[nu];
    }
    __syncthreads();
    for (int i = warp; i < nx; i += kNw) {
        const float* krow = R.kt + (int64_t)i * ny;
        double s = 0.0;
        for (int nu = lane; nu < ny; nu += 32) s = fma((double)krow[nu], R.work[nu], s);
        s = warp_sum(s);
        if (lane == 0) rhs[i] = s;
    }
    __syncthreads();
    const bool bad = cholesky(C, nx);
    if (tid == 0 && status) status[blockIdx.x] = bad ? kNtNonPd : 0u;
    for (int i = tid; i < nx; i += kNt) dx[i] = rhs[i];
    __syncthreads();
    if (warp == 0) chol_solve_warp(C, nx, dx);
    __syncthreads();
    const int nsteps = refine + (resid ? 1 : 0);
    for (int it = 0; it < nsteps; ++it) {
        apply_c_exact(R, dx, res);
        for (int i = tid; i < nx; i += kNt) res[i] = rhs[i] - res[i];
        __syncthreads();
        if (it == refine) {            // residual of the final dx (no further update)
            if (warp == 0) {
                double rr = 0.0, bb = 0.0;
                for (int i = lane; i < nx; i += 32) {
                    rr += res[i] * res[i];
                    bb += rhs[i] * rhs[i];
                }
                rr = warp_sum(rr);
                bb = warp_sum(bb);
                if (lane == 0) resid[blockIdx.x] = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
            }
            break;
        }
        if (warp == 0) chol_solve_warp(C, nx, res);
        __syncthreads();
        for (int i = tid; i < nx; i += kNt) dx[i] += res[i];
        __syncthreads();
    }
    for (int i = tid; i < nx; i += kNt) R.x_out[i] = R.xa[i] + (float)dx[i];   // calcnextxn.f:104
}

// phi = (yn-y)^T Se^-1 (yn-y) + (xn-xa)^T Sa^-1 (xn-xa), chisq = first term (calc_phiret.f:49-102)
__global__ void __launch_bounds__(kNt)
phi_kernel(const PhiDev* __restrict__ rets, float* __restrict__ phi, float* __restrict__ chisq) {
    __shared__ double red[kNw];
    __shared__ double bx[kNp];
    const PhiDev R = rets[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double s = 0.0;
    for (int nu = tid; nu < R.ny; nu += kNt) {
        const double b = (double)(R.yn[nu] - R.y[nu]);
        s += b * (R.sei[nu] * b);
    }
    s = warp_sum(s);
    if (lane == 0) red[warp] = s;
    for (int i = tid; i < R.nx; i += kNt) bx[i] = (double)(R.xn[i] - R.xa[i]);
    __syncthreads();
    double p1 = 0.0;
    for (int w = 0; w < kNw; ++w) p1 += red[w];
    __syncthreads();
    double t = 0.0;
    for (int i = warp; i < R.nx; i += kNw) {
        double a = 0.0;
        for (int j = lane; j < R.nx; j += 32) a += R.sai[i * R.nx + j] * bx[j];
        t += bx[i] * warp_sum(a);
    }
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (tid == 0) {
        double p2 = 0.0;
        for (int w = 0; w < kNw; ++w) p2 += red[w];
        phi[blockIdx.x] = (float)(p1 + p2);
        chisq[blockIdx.x] = (float)p1;
    }
}

// Ainv = A^-1 for SPD A (dinvertm.f jmod=2): Cholesky, then one identity
// column per warp through the two triangular solves.
__global__ void __launch_bounds__(kNt, 1)
spd_inverse_kernel(const double* __restrict__ A, double* __restrict__ Ainv, int n, int64_t stride,
                   unsigned* __restrict__ status) {
    extern __shared__ __align__(16) char smem[];
    double* L = (double*)smem;
    double* cols = L + n * n;          // [kNw][kNp]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double* a = A + (int64_t)blockIdx.x * stride;
    double* ai = Ainv + (int64_t)blockIdx.x * stride;
    for (int e = tid; e < n * n; e += kNt) L[e] = a[e];
    __syncthreads();
    const bool bad = cholesky(L, n);
    if (tid == 0 && status) status[blockIdx.x] = bad ? kNtNonPd : 0u;
    double* v = cols + warp * kNp;
    for (int j = warp; j < n; j += kNw) {
        for (int i = lane; i < n; i += 32) v[i] = i == j ? 1.0 : 0.0;
        chol_solve_warp(L, n, v);
        for (int i = lane; i < n; i += 32) ai[i * n + j] = v[i];
        __syncwarp();
    }
}

}  // namespace

cudaError_t launch_newton_step(const NewtonDev* d_ret, int nret, int hessian, int refine, unsigned* d_status,
                               double* d_resid, cudaStream_t st) {
    if (nret <= 0) return cudaSuccess;
    const int smem = newton_smem(kNp);
    cudaError_t e;
    if (hessian == 0) {
        e = cudaFuncSetAttribute(newton_step_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        newton_step_kernel<0><<<nret, kNt, smem, st>>>(d_ret, refine, d_status, d_resid);
    } else {
        e = cudaFuncSetAttribute(newton_step_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        newton_step_kernel<1><<<nret, kNt, smem, st>>>(d_ret, refine, d_status, d_resid);
    }
    return cudaGetLastError();
}

cudaError_t launch_phi(const PhiDev* d_ret, int nret, float* d_phi, float* d_chisq, cudaStream_t st) {
    if (nret <= 0) return cudaSuccess;
    phi_kernel<<<nret, kNt, 0, st>>>(d_ret, d_phi, d_chisq);
    return cudaGetLastError();
}

cudaError_t launch_spd_inverse(const double* d_a, double* d_ainv, int n, int64_t stride, int nret,
                               unsigned* d_status, cudaStream_t st) {
    if (nret <= 0) return cudaSuccess;
    const int smem = n * n * 8 + kNw * kNp * 8;
    cudaError_t e = cudaFuncSetAttribute(spd_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    spd_inverse_kernel<<<nret, kNt, smem, st>>>(d_a, d_ainv, n, stride, d_status);
    return cudaGetLastError();
}

}  // namespace rtb
