// Residual norms of a solution: r = b - A x with A the matrix as assembled.  After a
// solve has balanced the values in place (A~ = B A B, paso/src/SystemMatrix.cpp:263-312)
// the kernel undoes the scaling on the fly: (A x)_i = (1/bv_i) sum_j a~_ij x_j / bv_j.
#pragma once

#include "rg_internal.cuh"

namespace rg {
namespace residual {

constexpr int kThreads = 256;
constexpr int kLpr = 8;                                  // lanes per CSR row
constexpr int kRowsPerBlock = kThreads / kLpr;
constexpr int kMaxBlocks = 148 * 8;                      // grid cap (multiple of the SM count)

// grid for n rows (<= kMaxBlocks)
inline int grid(int64_t n) { return grid_for(n, kRowsPerBlock, 8); }

namespace {  // internal linkage: the kernel may be compiled into several translation units

// out[0] = sum r_i^2, out[1] = max |r_i|; rb is the reduction scratch (partials of
// gridDim.x * 2 doubles and a zeroed counter)
__global__ void __launch_bounds__(kThreads) k_residual_norms(int64_t n, const int32_t* __restrict__ ptr,
                                                             const int32_t* __restrict__ idx,
                                                             const double* __restrict__ val,
                                                             const double* __restrict__ bv,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ x, ReduceBuf rb,
                                                             double* __restrict__ out)
{
    const int lane = threadIdx.x & (kLpr - 1);
    const int64_t groups = (int64_t)gridDim.x * blockDim.x / kLpr;
    const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;
    const int64_t wg0 = g0 & ~(int64_t)(32 / kLpr - 1);
    double v[2] = {0.0, 0.0};
    for (int64_t gb = wg0; gb < n; gb += groups) {
        const int64_t row = gb + (g0 - wg0);
        double acc = 0.0;
        if (row < n)
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) {
                const int32_t j = idx[k];
                acc = fma(val[k], bv ? x[j] / bv[j] : x[j], acc);
            }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row < n && lane == 0) {
            const double r = b[row] - (bv ? acc / bv[row] : acc);
            v[0] += r * r;
            v[1] = fmax(v[1], fabs(r));
        }
    }
    double t[2];
    if (grid_reduce<2, 2u>(v, rb, t) && threadIdx.x == 0) {
        out[0] = t[0];
        out[1] = t[1];
    }
}

}  // namespace
}  // namespace residual
}  // namespace rg
