// paso CSR operations on the device: SpMV (ypAx), the Dirichlet constraint of
// LinearPDE.insertConstraint, nullifyRowsAndCols, balancing, the Jacobi diagonal and
// the structured band copy used by the fast inner solver.
//
// CSR rows hold <= 27 entries, so a row is handled by a group of 8 lanes (4 rows per
// warp): the lanes of a group read consecutive entries, a warp reads 4 consecutive
// rows = one contiguous stretch of val/idx, and the row sum is a 3-step shuffle.
#include "rg_internal.cuh"

namespace rg {

namespace {

constexpr int kLpr = 8;  // lanes per CSR row

// paso SparseMatrix_MatrixVector_CSR_OFFSET0 semantics
// (paso/src/SparseMatrix_MatrixVector.cpp:243-266): y = beta*y (y = 0 when beta == 0),
// then y += alpha*A*x when alpha != 0.
__global__ void __launch_bounds__(256) k_spmv64(int64_t n, const int32_t* __restrict__ ptr,
                                                const int32_t* __restrict__ idx,
                                                const double* __restrict__ val, double alpha,
                                                const double* __restrict__ x, double beta,
                                                double* __restrict__ y)
{
    const int lane = threadIdx.x & (kLpr - 1);
    const int64_t groups = (int64_t)gridDim.x * blockDim.x / kLpr;
    const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;
    // trip count uniform per warp: rows are visited in warp-sized batches
    const int64_t warp_g0 = g0 & ~(int64_t)(32 / kLpr - 1);
    for (int64_t gb = warp_g0; gb < n; gb += groups) {
        const int64_t row = gb + (g0 - warp_g0);
        double s = 0.0;
        if (row < n && fabs(alpha) > 0) {
            const int32_t k1 = ptr[row + 1];
            for (int32_t k = ptr[row] + lane; k < k1; k += kLpr) s = fma(val[k], x[idx[k]], s);
        }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (row < n && lane == 0) {
            double o = fabs(beta) > 0 ? (beta != 1.0 ? y[row] * beta : y[row]) : 0.0;
            if (fabs(alpha) > 0) o += alpha * s;
            y[row] = o;
        }
    }
}

// insertConstraint (escriptcore/py_src/linearPDEs.py:2084-2112) fused per row:
//   rhs_i -= sum_j a_ij u_j,  u_j = r_j if q_j > 0 else 0     (ypAx with the unbalanced A)
//   a_ij  = (i == j) if q_i > 0 or q_j > 0                     (SparseMatrix.h:494-509)
//   rhs_i = r_i if q_i > 0                                     (copyWithMask)
// Row i's update reads only row i's original values, so one pass suffices.
__global__ void __launch_bounds__(256) k_insert_constraint(int64_t n, const int32_t* __restrict__ ptr,
                                                           const int32_t* __restrict__ idx,
                                                           double* __restrict__ val,
                                                           double* __restrict__ rhs,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ r,
                                                           int rhs_only)
{
    const int lane = threadIdx.x & (kLpr - 1);
    const int64_t groups = (int64_t)gridDim.x * blockDim.x / kLpr;
    const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;
    const int64_t warp_g0 = g0 & ~(int64_t)(32 / kLpr - 1);
    for (int64_t gb = warp_g0; gb < n; gb += groups) {
        const int64_t row = gb + (g0 - warp_g0);
        double s = 0.0;
        const bool valid = row < n;
        const bool qi = valid && q[row] > 0.0;
        if (valid && !rhs_only && val) {
            const int32_t k1 = ptr[row + 1];
            for (int32_t k = ptr[row] + lane; k < k1; k += kLpr) {
                const int32_t j = idx[k];
                const bool qj = q[j] > 0.0;
                const double a = val[k];
                if (qj && r) s = fma(a, r[j], s);
                if (qi || qj) val[k] = (j == row) ? 1.0 : 0.0;
            }
        }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (valid && lane == 0 && rhs) {
            if (qi)
                rhs[row] = r ? r[row] : 0.0;
            else if (!rhs_only && val)
                rhs[row] = rhs[row] + (-1.0) * s;
        }
    }
}

// SystemMatrix::nullifyRowsAndCols (paso/src/SystemMatrix.h:544-605, SparseMatrix.h:494-509)
__global__ void __launch_bounds__(256) k_nullify(int64_t n, const int32_t* __restrict__ ptr,
                                                 const int32_t* __restrict__ idx,
                                                 double* __restrict__ val,
                                                 const double* __restrict__ mr,
                                                 const double* __restrict__ mc, double diag)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool qi = mr[i] > 0.0;
    for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
        const int32_t j = idx[k];
        if (qi || mc[j] > 0.0) val[k] = (j == i) ? diag : 0.0;
    }
}

// balance, step 1 (paso/src/SystemMatrix.cpp:263-290): bv_i = sqrt(1/max_j |a_ij|), or 1
__global__ void __launch_bounds__(256) k_row_balance(int64_t n, const int32_t* __restrict__ ptr,
                                                     const double* __restrict__ val,
                                                     double* __restrict__ bv)
{
    const int lane = threadIdx.x & (kLpr - 1);
    const int64_t groups = (int64_t)gridDim.x * blockDim.x / kLpr;
    const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;
    const int64_t warp_g0 = g0 & ~(int64_t)(32 / kLpr - 1);
    for (int64_t gb = warp_g0; gb < n; gb += groups) {
        const int64_t row = gb + (g0 - warp_g0);
        double m = 0.0;
        if (row < n)
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) m = fmax(m, fabs(val[k]));
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (row < n && lane == 0) bv[row] = m > 0 ? sqrt(1. / m) : 1.;
    }
}

// balance, step 2 (SparseMatrix::applyDiagonal_CSR_OFFSET0, paso/src/SparseMatrix.cpp:361-385)
// a_ij *= bv_i*bv_j, followed by the Jacobi data of the balanced matrix
// (SparseMatrix::invMain, paso/src/SparseMatrix.cpp:387-435): dinv_i = 1/a~_ii; a zero or
// missing diagonal sets *bad.  With band != null the balanced row is also copied into the
// tile-major FP32 band layout: band[((i/256)*nbands + b)*256 + i%256],
// b = (dx+1) + 3(dy+1) (+ 9(dz+1)); with band64 != null the same in FP64.
__global__ void __launch_bounds__(256) k_apply_balance(int64_t n, int nbands, int dim, int64_t NN0, int64_t NN1,
                                                       const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx,
                                                       double* __restrict__ val,
                                                       const double* __restrict__ bv, int scale,
                                                       double* __restrict__ dinv,
                                                       float* __restrict__ dinv32,
                                                       float* __restrict__ band, double* __restrict__ band64,
                                                       int* bad)
{
    const int lane = threadIdx.x & (kLpr - 1);
    const int64_t groups = (int64_t)gridDim.x * blockDim.x / kLpr;
    const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;
    const int64_t warp_g0 = g0 & ~(int64_t)(32 / kLpr - 1);
    const int64_t plane = NN0 * NN1;
    for (int64_t gb = warp_g0; gb < n; gb += groups) {
        const int64_t row = gb + (g0 - warp_g0);
        double dg = 0.0;
        int found = 0;
        if (row < n) {
            const double bi = bv[row];
            const int64_t xi = row % NN0, yi = (row / NN0) % NN1, zi = row / plane;
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) {
                const int32_t j = idx[k];
                double a = val[k];
                if (scale) {
                    a *= bi * bv[j];
                    val[k] = a;
                }
                if (j == row) {
                    dg = a;
                    found = 1;
                }
                if (band || band64) {
                    const int64_t xj = j % NN0, yj = (j / NN0) % NN1, zj = j / plane;
                    int b = (int)(xj - xi + 1) + 3 * (int)(yj - yi + 1);
                    if (dim == 3) b += 9 * (int)(zj - zi + 1);
                    const size_t o = ((size_t)(row >> 8) * nbands + b) * 256 + (row & 255);
                    if (band) band[o] = (float)a;
                    if (band64) band64[o] = a;
                }
            }
        }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) {
            dg += __shfl_xor_sync(0xffffffffu, dg, o);
            found += __shfl_xor_sync(0xffffffffu, found, o);
        }
        if (row < n && lane == 0) {
            if (!found || !(fabs(dg) > 0.)) {
                atomicOr(bad, 1);
                dinv[row] = 0.0;
                if (dinv32) dinv32[row] = 0.f;
            } else {
                dinv[row] = 1. / dg;
                if (dinv32) dinv32[row] = (float)(1. / dg);
            }
        }
    }
}

}  // namespace

int launch_spmv64(const Domain* d, const double* val, double alpha, const double* x, double beta,
                  double* y)
{
    const int grid = grid_for(d->n, 256 / kLpr, 16);
    RG_TIMED(T_SPMV, (k_spmv64<<<grid, 256, 0, stream()>>>(d->n, d->ptr, d->idx, val, alpha, x, beta, y)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_insert_constraint(Matrix* m, double* rhs, const double* q, const double* r, int rhs_only)
{
    const Domain* d = m->dom;
    const int grid = grid_for(d->n, 256 / kLpr, 16);
    RG_TIMED(T_CONSTRAINT, (k_insert_constraint<<<grid, 256, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, rhs, q, r, rhs_only)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_nullify(Matrix* m, const double* mr, const double* mc, double diag)
{
    const Domain* d = m->dom;
    RG_TIMED(T_CONSTRAINT, (k_nullify<<<(int)((d->n + 255) / 256), 256, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, mr, mc, diag)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_balance(Matrix* m, int scale, int* d_bad, bool want_band, bool want_band64)
{
    const Domain* d = m->dom;
    const int grid = grid_for(d->n, 256 / kLpr, 16);
    if (scale) {
        RG_TIMED(T_BALANCE, (k_row_balance<<<grid, 256, 0, stream()>>>(d->n, d->ptr, m->val, m->bv)));
        RG_CHECK_LAUNCH();
    }
    if (want_band) RG_CHECK_CUDA(cudaMemsetAsync(m->band32, 0, sizeof(float) * d->nbands * d->npad, stream()));
    if (want_band64) RG_CHECK_CUDA(cudaMemsetAsync(m->band64, 0, sizeof(double) * d->nbands * d->npad, stream()));
    RG_TIMED(T_BALANCE, (k_apply_balance<<<grid, 256, 0, stream()>>>(d->n, d->nbands, d->dim, d->nn[0], d->nn[1], d->ptr, d->idx, m->val,
                                                m->bv, scale, m->dinv, m->dinv32,
                                                want_band ? m->band32 : nullptr,
                                                want_band64 ? m->band64 : nullptr, d_bad)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

}  // namespace rg
