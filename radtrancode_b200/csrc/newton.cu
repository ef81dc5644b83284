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
//   1. One pass over K in chunks of 64 wavenumbers (K read from HBM once):
//      a. N = K^T Se^-1 K on the 5th-generation tensor cores.  K~ = Se^-1/2 K
//         is split into bf16 hi + lo parts, written to shared memory in the
//         128-byte-swizzled K-major layout, and one elected thread issues
//         three tcgen05.mma (hi*hi + hi*lo + lo*hi, M = N = 128, K = 16 each)
//         per 16 wavenumbers into one FP32 accumulator in tensor memory
//         (128 lanes x 128 columns).  About 2^-17 relative error per product.
//         Two staging buffers: the chunk after next waits on the mbarrier the
//         MMAs of a chunk commit to.
//      b. the right-hand side rhs = K^T Se^-1 (y - yn + K d) on the CUDA
//         cores from the same registers, FP64 accumulation of the FP32 K.
//      (Alternative: N in FP64 on the CUDA cores, the all-FP64 solve.)
//   2. C = N + Sa^-1 in FP64 shared memory; Cholesky in FP64 with the
//      reference's non-positive-pivot rule (pivot 1, continue).
//   3. dx = C^-1 rhs, then `refine` steps dx += C^-1 (rhs - C_exact dx) where
//      C_exact applies K^T Se^-1 K through K in FP64 (never through N), one
//      more pass over K per step.
//   4. x_out = xa + (float)dx.
#include <cuda_runtime.h>
#include <stdint.h>

#include "newton.h"

namespace rtb {

namespace {

constexpr int kNt = 256;                  // threads per block (8 warps)
constexpr int kNw = kNt / 32;
constexpr int kNp = kNewtonMaxNx;         // padded state size: the MMA's M and N
constexpr int kKc = 64;                   // wavenumbers per chunk (one 128-byte bf16 row of the staging tile)
constexpr int kTile = kNp * kKc * 2;      // bytes of one bf16 staging tile (16 KB)
constexpr int kStage = 2 * kTile;         // hi + lo
constexpr int kStaging = 2 * kStage + 1024;   // two stages, 1024-byte alignment slack
constexpr int kStageF64 = 32 * kNp * 8 + 32 * 8;   // hessian_f64: 32 wavenumbers of K in FP64

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
// C (nx x nx FP64) aliased with the staging buffers of the pass over K
__host__ __device__ constexpr int region_bytes(int nx) {
    return (cmax(nx * nx * 8, cmax(kStaging, kStageF64)) + 15) & ~15;
}
// region + d, rhs, dx, res (kNp doubles each) + the pass's per-warp column
// partials [kNw][kKc] and the chunk's Se^-1 (dy + K d) [kKc] + 2 mbarriers +
// the tensor-memory address
constexpr int kTailBytes = 8 * 4 * kNp + 8 * kNw * kKc + 8 * kKc + 16 + 16;
__host__ __device__ constexpr int newton_smem(int nx) { return region_bytes(nx) + kTailBytes; }

constexpr unsigned kWaitLimit = 1u << 22;

// ---------------------------------------------------------------- tcgen05 / mbarrier primitives
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 64 bf16 (128 B) with 8-row groups 1024 B apart; the tile starts on a
// 1024-byte boundary (base offset 0), k-slices advance the start by 32 B
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused by swizzled K-major): 16 B
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                  // descriptor version of sm_100
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}
// instruction descriptor of kind::f16: FP32 accumulator, A and B bf16, both
// K-major, M = 128, N = 128, dense
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kNp >> 3) << 17) |
                            ((uint32_t)(kNp >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// bounded wait for the phase with parity `phase` to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// bf16 round-to-nearest-even of a finite float, as its 16 bits
__device__ __forceinline__ unsigned bf16_bits(float x) {
    const unsigned u = __float_as_uint(x);
    return (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
}

struct PassSm {
    double* colp;     // [kNw][kKc] per-warp column partials
    double* wch;      // [kKc] Se^-1 (dy + K v) of the chunk
    uint32_t stage0;  // shared address of the first staging stage (1024-aligned)
    uint32_t bar0;    // shared address of the two mbarriers
    uint32_t tmem;    // accumulator address in tensor memory
};

// One pass over K (nx x ny, FP32, row iv = dR/dx_iv) in chunks of kKc
// wavenumbers.  Thread t owns 8 consecutive wavenumbers (t & 7) of the rows
// t/8 + 32 r (r = 0..3).  For every chunk:
//   w(nu) = Se^-1(nu) (dy(nu) + sum_i K(i, nu) v(i))        (dy = y - yn, REAL, or 0)
//   out(i) += sum_nu K(i, nu) w(nu)                           (FP64 accumulation)
// and with kTc the chunk's K~ = Se^-1/2 K goes to shared memory as bf16
// hi/lo for the tensor-core product N += K~ K~^T.  v and out hold kNp
// entries (zero beyond nx).  Returns false if an mbarrier wait gave up.
template <bool kTc>
__device__ bool k_pass(const NewtonDev& R, const double* v, bool with_dy, double* out, const PassSm& P) {
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g8 = tid & 7, rb = tid >> 3;
    double vr[4], acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < 4; ++r) vr[r] = v[rb + 32 * r];
    float x[4][8];
    auto load = [&](int c) {
        const int nu0 = c * kKc + 8 * g8;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int row = rb + 32 * r;
            const float* src = R.kt + (int64_t)row * ny + nu0;
            if (row < nx && nu0 + 8 <= ny && (((uintptr_t)src) & 15) == 0) {
                const float4 a = __ldg((const float4*)src), b = __ldg((const float4*)src + 1);
                x[r][0] = a.x; x[r][1] = a.y; x[r][2] = a.z; x[r][3] = a.w;
                x[r][4] = b.x; x[r][5] = b.y; x[r][6] = b.z; x[r][7] = b.w;
            } else {
#pragma unroll
                for (int e = 0; e < 8; ++e) x[r][e] = (row < nx && nu0 + e < ny) ? __ldg(src + e) : 0.0f;
            }
        }
    };
    const int nchunk = (ny + kKc - 1) / kKc;
    bool ok = true;
    uint32_t phase[2] = {0u, 0u};
    load(0);
    for (int c = 0; c < nchunk; ++c) {
        const int nu0 = c * kKc + 8 * g8;
        // column partials over this thread's 4 rows, then over the warp's 4 row groups
        double cp[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            double s = 0.0;
#pragma unroll
            for (int r = 0; r < 4; ++r) s = fma((double)x[r][e], vr[r], s);
            s += __shfl_xor_sync(0xffffffffu, s, 8);
            s += __shfl_xor_sync(0xffffffffu, s, 16);
            cp[e] = s;
        }
        if (lane < 8) {
#pragma unroll
            for (int e = 0; e < 8; ++e) P.colp[warp * kKc + 8 * g8 + e] = cp[e];
        }
        const int s = c & 1;
        if (kTc && c >= 2) {   // stage s is free once the MMAs of chunk c - 2 are complete
            if (tid == 0 && !mbar_wait(P.bar0 + 8 * s, phase[s])) ok = false;
            phase[s] ^= 1u;
        }
        __syncthreads();
        if (tid < kKc) {
            const int nu = c * kKc + tid;
            double w = 0.0;
            if (nu < ny) {
                double cs = 0.0;
#pragma unroll
                for (int w8 = 0; w8 < kNw; ++w8) cs += P.colp[w8 * kKc + tid];
                const double dy = with_dy ? (double)(R.y[nu] - R.yn[nu]) : 0.0;   // REAL difference (calcnextxn.f:92)
                w = (dy + cs) * R.sei[nu];
            }
            P.wch[tid] = w;
        }
        if (kTc) {
            float sc[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) sc[e] = nu0 + e < ny ? (float)sqrt(R.sei[nu0 + e]) : 0.0f;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = rb + 32 * r;
                unsigned hi[4], lo[4];
#pragma unroll
                for (int e = 0; e < 8; e += 2) {
                    const float a = x[r][e] * sc[e], b = x[r][e + 1] * sc[e + 1];
                    const unsigned ha = bf16_bits(a), hb = bf16_bits(b);
                    const float ra = a - __uint_as_float(ha << 16), rb2 = b - __uint_as_float(hb << 16);
                    hi[e / 2] = ha | (hb << 16);
                    lo[e / 2] = bf16_bits(ra) | (bf16_bits(rb2) << 16);
                }
                // row `row`, 16-byte chunk g8, XOR-swizzled by row & 7
                const uint32_t off = (uint32_t)(row * 128 + ((g8 ^ (row & 7)) << 4));
                const uint32_t a_hi = P.stage0 + s * kStage + off, a_lo = a_hi + kTile;
                asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(a_hi), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]),
                             "r"(hi[3])
                             : "memory");
                asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(a_lo), "r"(lo[0]), "r"(lo[1]), "r"(lo[2]),
                             "r"(lo[3])
                             : "memory");
            }
            fence_async_smem();   // the generic-proxy writes become visible to the tensor core
        }
        __syncthreads();
        if (kTc && tid == 0) {
            tc_fence_after();
            const uint32_t hi = P.stage0 + s * kStage, lo = hi + kTile;
#pragma unroll
            for (int k = 0; k < kKc / 16; ++k) {
                const uint64_t dh = sw128_desc(hi + 32 * k), dl = sw128_desc(lo + 32 * k);
                umma_bf16(P.tmem, dh, dh, (c > 0 || k > 0) ? 1u : 0u);
                umma_bf16(P.tmem, dh, dl, 1u);
                umma_bf16(P.tmem, dl, dh, 1u);
            }
            umma_commit(P.bar0 + 8 * s);
        }
        // this chunk's share of K^T w
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            double a = acc[r];
#pragma unroll
            for (int e = 0; e < 8; ++e) a = fma((double)x[r][e], P.wch[8 * g8 + e], a);
            acc[r] = a;
        }
        if (c + 1 < nchunk) load(c + 1);
    }
    if (kTc && tid == 0) {
        // the last commit completes after every MMA of the pass; should it not
        // arrive in time, wait once more (bounded) before tensor memory is freed
        const int sl = (nchunk - 1) & 1;
        if (!mbar_wait(P.bar0 + 8 * sl, phase[sl])) {
            ok = false;
            mbar_wait(P.bar0 + 8 * sl, phase[sl]);
        }
    }
    // rows: sum over the 8 threads of a row (lanes differing in bits 0..2)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        double a = acc[r];
        a += __shfl_xor_sync(0xffffffffu, a, 1);
        a += __shfl_xor_sync(0xffffffffu, a, 2);
        a += __shfl_xor_sync(0xffffffffu, a, 4);
        if (g8 == 0) out[rb + 32 * r] = a;
    }
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// C (nx x nx, row-major FP64) = N + Sa^-1 from the tensor-memory accumulator:
// warp w reads lanes 32 (w & 3).. and columns 64 (w >> 2)..
__device__ void c_from_tmem(const NewtonDev& R, uint32_t tmem, double* C) {
    const int nx = R.nx, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = 32 * (warp & 3) + lane, c0 = 64 * (warp >> 2);
    tc_fence_after();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(c0 + 16 * q), v);
        if (row < nx) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int col = c0 + 16 * q + i;
                if (col < nx) C[row * nx + col] = (double)v[i] + R.sai[row * nx + col];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
}

// C = K^T Se^-1 K + Sa^-1 in FP64 on the CUDA cores; thread (ti, tj) owns an 8x8 tile
__device__ void hessian_f64(const NewtonDev& R, char* sm, double* C) {
    constexpr int kc = 32;
    double* Kt = (double*)sm;          // [kc][kNp]
    double* se = Kt + kc * kNp;        // [kc]
    const int nx = R.nx, ny = R.ny;
    const int tid = threadIdx.x, ti = tid >> 4, tj = tid & 15;
    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
    for (int k0 = 0; k0 < ny; k0 += kc) {
        __syncthreads();
        for (int e = tid; e < kNp * kc; e += kNt) {
            const int i = e / kc, k = e - i * kc, nu = k0 + k;
            Kt[k * kNp + i] = (i < nx && nu < ny) ? (double)R.kt[(int64_t)i * ny + nu] : 0.0;
        }
        if (tid < kc) se[tid] = k0 + tid < ny ? R.sei[k0 + tid] : 0.0;
        __syncthreads();
        for (int k = 0; k < kc; ++k) {
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

// out = (K^T Se^-1 K + Sa^-1) x, K applied in FP64 from FP32: one pass over K
__device__ void apply_c_exact(const NewtonDev& R, const double* x, double* out, const PassSm& P) {
    const int nx = R.nx;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    k_pass<false>(R, x, false, out, P);
    for (int i = warp; i < nx; i += kNw) {
        double s = 0.0;
        for (int j = lane; j < nx; j += 32) s = fma(R.sai[i * nx + j], x[j], s);
        s = warp_sum(s);
        if (lane == 0) out[i] += s;
    }
    __syncthreads();
}

template <int kHess>
__global__ void __launch_bounds__(kNt, 1)
newton_step_kernel(const NewtonDev* __restrict__ rets, int refine, unsigned* __restrict__ status,
                   double* __restrict__ resid) {
    extern __shared__ __align__(16) char smem[];
    const NewtonDev R = rets[blockIdx.x];
    const int nx = R.nx;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* C = (double*)smem;
    double* d = (double*)(smem + region_bytes(kNp));
    double* rhs = d + kNp;
    double* dx = rhs + kNp;
    double* res = dx + kNp;
    PassSm P;
    P.colp = res + kNp;
    P.wch = P.colp + kNw * kKc;
    uint64_t* bars = (uint64_t*)(P.wch + kKc);
    uint32_t* tslot = (uint32_t*)(bars + 2);
    P.stage0 = (smem_u32(smem) + 1023u) & ~1023u;
    P.bar0 = smem_u32(bars);
    P.tmem = 0;
    if (kHess == 0) {
        if (tid == 0) {
            mbar_init(P.bar0, 1);
            mbar_init(P.bar0 + 8, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        if (warp == 0) {   // 128 FP32 columns of tensor memory for the 128 x 128 accumulator
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                         "r"(kNp));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        tc_fence_before();
    }
    // d = xn - xa (REAL difference, calcnextxn.f:84-86 with the sign folded in)
    for (int i = tid; i < kNp; i += kNt) d[i] = i < nx ? (double)(R.xn[i] - R.xa[i]) : 0.0;
    __syncthreads();
    if (kHess == 0) {
        tc_fence_after();
        P.tmem = *tslot;
        const bool ok = k_pass<true>(R, d, true, rhs, P);   // N in tensor memory, rhs = K^T Se^-1 (y - yn + K d)
        if (ok) c_from_tmem(R, P.tmem, C);
        if (warp == 0) {
            tc_fence_after();
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(P.tmem), "r"(kNp));
        }
        if (!ok) {
            if (tid == 0 && status) status[blockIdx.x] = kNtTimeout;
            return;
        }
    } else {
        hessian_f64(R, smem, C);
        k_pass<false>(R, d, true, rhs, P);
    }
    const bool bad = cholesky(C, nx);
    if (tid == 0 && status) status[blockIdx.x] = bad ? kNtNonPd : 0u;
    // padded entries stay 0: the passes over K read all kNp of them
    for (int i = tid; i < kNp; i += kNt) dx[i] = i < nx ? rhs[i] : 0.0;
    __syncthreads();
    if (warp == 0) chol_solve_warp(C, nx, dx);
    __syncthreads();
    const int nsteps = refine + (resid ? 1 : 0);
    for (int it = 0; it < nsteps; ++it) {
        apply_c_exact(R, dx, res, P);
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
