// newton.h -- device descriptors and launchers of the optimal-estimation
// Newton step (newton.cu), shared with the host side (retrieval.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rtb {

constexpr int kNewtonMaxNx = 128;   // state size handled by one block (NX=124 at full size)

// status bits of one retrieval's step
constexpr unsigned kNtNonPd = 1u;   // a Cholesky pivot was <= 0 and was replaced by 1 (dcholdc.f:69-84)
constexpr unsigned kNtTimeout = 2u; // a wait on the tensor-core pipeline gave up: x_out was not written

// one retrieval's Newton step: every pointer is device memory
struct NewtonDev {
    int nx, ny;
    const float* kt;      // [nx][ny] K^T: row iv = dR/dx_iv over the spectrum (the gradients packing)
    const float* y;       // [ny] measurement
    const float* yn;      // [ny] spectrum at xn
    const double* sei;    // [ny] diagonal of Se^-1
    const double* sai;    // [nx][nx] Sa^-1 (symmetric)
    const float* xa;      // [nx] a priori
    const float* xn;      // [nx] current state
    float* x_out;         // [nx] out: xa + C^-1 K^T Se^-1 (y - yn + K (xn - xa))
};

// chi^2 and cost of one retrieval (calc_phiret.f), every pointer device memory
struct PhiDev {
    int nx, ny;
    const float* y;
    const float* yn;
    const double* sei;
    const double* sai;
    const float* xn;
    const float* xa;
};

// hessian: 0 = K^T Se^-1 K on tensor cores (bf16 hi/lo split, FP32
// accumulation) + `refine` steps of iterative refinement in FP64;
// 1 = K^T Se^-1 K in FP64 on the CUDA cores (the all-FP64 solve).
// resid (may be null): per retrieval ||rhs - C dx|| / ||rhs|| after the
// last refinement step, with C applied exactly in FP64.
cudaError_t launch_newton_step(const NewtonDev* d_ret, int nret, int hessian, int refine, unsigned* d_status,
                               double* d_resid, cudaStream_t st);
// phi (REAL, as the reference function) and chisq per retrieval
cudaError_t launch_phi(const PhiDev* d_ret, int nret, float* d_phi, float* d_chisq, cudaStream_t st);
// Sa^-1 from Sa (FP64 Cholesky inverse, dinvertm.f jmod=2) for nret
// matrices [n][n] at a[r*stride], written to ainv[r*stride]
cudaError_t launch_spd_inverse(const double* d_a, double* d_ainv, int n, int64_t stride, int nret,
                               unsigned* d_status, cudaStream_t st);

}  // namespace rtb
