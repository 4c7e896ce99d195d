// PDE systems (block size NB = numEq = numComp, 2 or 3) on the node pattern:
//  * assembly of the interior terms, DefaultAssembler3D::assemblePDESystem
//    (ripley/src/DefaultAssembler3D.cpp:3630-5751) and DefaultAssembler2D::assemblePDESystem
//    (ripley/src/DefaultAssembler2D.cpp:1186-1980), into block CSR values
//    val[k NB^2 + ir + NB ic] (column-major blocks, RipleyDomain.cpp:1508-1518);
//  * insertConstraint per component (linearPDEs.py:2084-2112 with
//    SparseMatrix::nullifyRowsAndCols_CSR, paso/src/SparseMatrix.h:513-535);
//  * the block SpMV (paso/src/SparseMatrix_MatrixVector.cpp, blocked branches);
//  * paso's Solver + PCG with the block Jacobi preconditioner: balance per scalar row
//    (SystemMatrix.cpp:263-312, SparseMatrix.cpp:266-282, 361-385), inverses of the main
//    diagonal blocks (SparseMatrix.cpp:387-435, BlockOps.h:99-160), the PCG with residual
//    smoothing (PCG.cpp:62-367) and the outer dual-norm loop (Solver.cpp:46-330), in FP64.
// Vectors keep the NB components of a node together: u[node NB + comp].
#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "rg_internal.cuh"

namespace rg {

struct SysWorkspace {
    int64_t N = 0;  // scalar unknowns = nodes * NB
    double *r = nullptr, *x = nullptr, *rs = nullptr, *x2 = nullptr, *q = nullptr, *z = nullptr,
           *p = nullptr, *bb = nullptr;
    double* partials = nullptr;
    unsigned* counter = nullptr;
    void* s = nullptr;   // device scalars (BScal)
    void* hs = nullptr;  // pinned host copy
    int* bad = nullptr;
};

namespace sys {
namespace {

constexpr int kThreads = 256;
constexpr int kLpr = 8;
constexpr int kRows = 128;  // assembly threads per CTA

struct BScal {
    double tau, tau_next, delta, alpha, beta, gamma1, gamma2, norm, tol, n2, nm;
    long long iter, maxit;
    int done, status;
};
enum { ST_RUN = 0, ST_CONV = 1, ST_MAXIT = 3, ST_BREAK = 4 };

__device__ __forceinline__ int64_t gtid() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

// 8 lanes per scalar row (node NB + ir); every lane of a warp runs the same trips
#define RG_SROW_LOOP(N)                                                                 \
    const int lane = threadIdx.x & (kLpr - 1);                                          \
    const int64_t groups_ = (int64_t)gridDim.x * blockDim.x / kLpr;                     \
    const int64_t g0_ = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;        \
    const int64_t wg0_ = g0_ & ~(int64_t)(32 / kLpr - 1);                               \
    for (int64_t gb_ = wg0_; gb_ < (N); gb_ += groups_)                                 \
        if (const int64_t row = gb_ + (g0_ - wg0_); true)

__device__ __forceinline__ double group_sum(double s)
{
#pragma unroll
    for (int o = kLpr / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// sum_k sum_ic val[k NB^2 + ir + NB ic] x[idx[k] NB + ic] over this lane's entries of the
// node's row
template <int NB>
__device__ __forceinline__ double brow_dot(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                           const double* __restrict__ val, const double* __restrict__ x,
                                           int64_t node, int ir, int lane)
{
    double acc = 0.0;
    for (int32_t k = ptr[node] + lane; k < ptr[node + 1]; k += kLpr) {
        const int64_t c = (int64_t)idx[k] * NB;
        const double* v = val + (int64_t)k * NB * NB + ir;
#pragma unroll
        for (int ic = 0; ic < NB; ++ic) acc = fma(v[NB * ic], x[c + ic], acc);
    }
    return acc;
}

// ------------------------------------------------------------------ assembly
struct CoefArg {
    const double* p;
    int kind;
};

struct SysArgs {
    CoefArg c[6];
    Q1Tables t;
    int64_t NE0, NE1, NE2, NN0, NN1, NN2, n;
    const int32_t* ptr;
    double* val;
    double* rhs;
};

// data point of element e at point q (SIZE values)
template <int SIZE, int NQ>
__device__ __forceinline__ const double* cptr(const CoefArg& c, int64_t e, int q)
{
    if (c.kind == RG_COEF_EXPANDED) return c.p + ((size_t)e * NQ + q) * SIZE;
    if (c.kind == RG_COEF_PER_ELEMENT) return c.p + (size_t)e * SIZE;
    return c.p;
}

// Row R (local node) of the element block (equation k, component m):
//   em[c] = sum_q W (A_kimj G_Ri G_cj + B_kim G_Ri N_c + C_kmj N_R G_cj + D_km N_R N_c)
//   f     = sum_q W (X_ki G_Ri + Y_k N_R)   (for m == 0)
// layouts A[k + NB (i + DIM (m + NB j))], B[k + NB (i + DIM m)], C[k + NB (m + NB j)],
// D[k + NB m], X[k + NB i], Y[k]
template <int DIM, int NB, int NQ, int R>
__device__ __forceinline__ void element_row(const SysArgs& a, int64_t e, int k, int m, double (&em)[1 << DIM],
                                            double& f)
{
    constexpr int NK = 1 << DIM;
    constexpr int SA = NB * DIM * NB * DIM, SB = NB * DIM * NB, SC = NB * NB * DIM, SD = NB * NB;
    constexpr int SX = NB * DIM, SY = NB;
    const CoefArg& A = a.c[0];
    const CoefArg& B = a.c[1];
    const CoefArg& C = a.c[2];
    const CoefArg& D = a.c[3];
    const CoefArg& X = a.c[4];
    const CoefArg& Y = a.c[5];
#pragma unroll
    for (int c = 0; c < NK; ++c) em[c] = 0.0;
    f = 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const double NR = a.t.N[q][R];
        double s[DIM], t0 = 0.0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) s[j] = 0.0;
        if (A.kind) {
            const double* ap = cptr<SA, NQ>(A, e, q);
#pragma unroll
            for (int j = 0; j < DIM; ++j)
#pragma unroll
                for (int i = 0; i < DIM; ++i)
                    s[j] = fma(__ldg(ap + k + NB * (i + DIM * (m + NB * j))), a.t.G[q][R][i], s[j]);
        }
        if (C.kind) {
            const double* cp = cptr<SC, NQ>(C, e, q);
#pragma unroll
            for (int j = 0; j < DIM; ++j) s[j] = fma(__ldg(cp + k + NB * (m + NB * j)), NR, s[j]);
        }
        if (B.kind) {
            const double* bp = cptr<SB, NQ>(B, e, q);
#pragma unroll
            for (int i = 0; i < DIM; ++i) t0 = fma(__ldg(bp + k + NB * (i + DIM * m)), a.t.G[q][R][i], t0);
        }
        if (D.kind) t0 = fma(__ldg(cptr<SD, NQ>(D, e, q) + k + NB * m), NR, t0);
#pragma unroll
        for (int c = 0; c < NK; ++c) {
            double v = t0 * a.t.N[q][c];
#pragma unroll
            for (int j = 0; j < DIM; ++j) v = fma(s[j], a.t.G[q][c][j], v);
            em[c] = fma(a.t.W, v, em[c]);
        }
        if (m == 0) {
            double fq = 0.0;
            if (Y.kind) fq = __ldg(cptr<SY, NQ>(Y, e, q) + k) * NR;
            if (X.kind) {
                const double* xp = cptr<SX, NQ>(X, e, q);
#pragma unroll
                for (int i = 0; i < DIM; ++i) fq = fma(__ldg(xp + k + NB * i), a.t.G[q][R][i], fq);
            }
            f = fma(a.t.W, fq, f);
        }
    }
}

template <int DIM>
__host__ __device__ constexpr int band_of(int sx, int sy, int sz, int c)
{
    return DIM == 3 ? (sx + (c & 1)) + 3 * (sy + ((c >> 1) & 1)) + 9 * (sz + ((c >> 2) & 1))
                    : (sx + (c & 1)) + 3 * (sy + ((c >> 1) & 1));
}

template <int DIM, int NB, int NQ, int SX, int SY, int SZ>
__device__ __forceinline__ void add_element(const SysArgs& a, int64_t x, int64_t y, int64_t z, int k, int m,
                                            double (&acc)[DIM == 3 ? 27 : 9], double& facc)
{
    constexpr int NK = 1 << DIM;
    const int64_t ex = x - 1 + SX, ey = y - 1 + SY, ez = z - 1 + SZ;
    if (ex < 0 || ex >= a.NE0 || ey < 0 || ey >= a.NE1) return;
    if (DIM == 3 && (ez < 0 || ez >= a.NE2)) return;
    const int64_t e = ex + a.NE0 * ey + (DIM == 3 ? a.NE0 * a.NE1 * ez : 0);
    constexpr int R = (1 - SX) + 2 * (1 - SY) + (DIM == 3 ? 4 * (1 - SZ) : 0);
    double em[NK], f;
    element_row<DIM, NB, NQ, R>(a, e, k, m, em, f);
#pragma unroll
    for (int c = 0; c < NK; ++c) acc[band_of<DIM>(SX, SY, SZ, c)] += em[c];
    facc += f;
}

// one thread per (node, equation k, component m): the node's block row entries (k, m) over
// its <= 27 (9) neighbours, gathered from the adjacent elements; no atomics.  NQ = 2^DIM
// Gauss points, or 1 (the element centre with weight = volume) for coefficients on
// ReducedFunction (assemblePDESystemReduced, DefaultAssembler3D.cpp:6466-6876,
// DefaultAssembler2D.cpp assemblePDESystemReduced)
template <int DIM, int NB, int NQ>
__global__ void __launch_bounds__(kRows) k_assemble_sys(const __grid_constant__ SysArgs a)
{
    constexpr int NBD = DIM == 3 ? 27 : 9;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= a.n * NB * NB) return;
    const int64_t i = tid / (NB * NB);
    const int cm = (int)(tid % (NB * NB));
    const int k = cm % NB, m = cm / NB;
    double acc[NBD];
#pragma unroll
    for (int b = 0; b < NBD; ++b) acc[b] = 0.0;
    double facc = 0.0;
    const int64_t x = i % a.NN0, y = (i / a.NN0) % a.NN1, z = DIM == 3 ? i / (a.NN0 * a.NN1) : 0;
    add_element<DIM, NB, NQ, 0, 0, 0>(a, x, y, z, k, m, acc, facc);
    add_element<DIM, NB, NQ, 1, 0, 0>(a, x, y, z, k, m, acc, facc);
    add_element<DIM, NB, NQ, 0, 1, 0>(a, x, y, z, k, m, acc, facc);
    add_element<DIM, NB, NQ, 1, 1, 0>(a, x, y, z, k, m, acc, facc);
    if (DIM == 3) {
        add_element<DIM, NB, NQ, 0, 0, 1>(a, x, y, z, k, m, acc, facc);
        add_element<DIM, NB, NQ, 1, 0, 1>(a, x, y, z, k, m, acc, facc);
        add_element<DIM, NB, NQ, 0, 1, 1>(a, x, y, z, k, m, acc, facc);
        add_element<DIM, NB, NQ, 1, 1, 1>(a, x, y, z, k, m, acc, facc);
    }
    if (a.rhs && m == 0) a.rhs[i * NB + k] += facc;
    if (!a.val) return;
    int64_t kk = a.ptr[i];
#pragma unroll
    for (int b = 0; b < NBD; ++b) {
        const int bx = b % 3 - 1, by = (b / 3) % 3 - 1, bz = DIM == 3 ? b / 9 - 1 : 0;
        const bool in = x + bx >= 0 && x + bx < a.NN0 && y + by >= 0 && y + by < a.NN1 &&
                        (DIM == 2 || (z + bz >= 0 && z + bz < a.NN2));
        if (in) {
            a.val[kk * NB * NB + k + NB * m] += acc[b];
            ++kk;
        }
    }
}

// ------------------------------------------------------------------ constraint, SpMV, nullify
template <int NB>
__global__ void __launch_bounds__(kThreads) k_constraint_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                             const int32_t* __restrict__ idx,
                                                             double* __restrict__ val, double* __restrict__ rhs,
                                                             const double* __restrict__ q,
                                                             const double* __restrict__ r, int rhs_only)
{
    const int64_t N = nodes * NB;
    RG_SROW_LOOP(N)
    {
        double s = 0.0;
        const bool valid = row < N;
        const int64_t node = row / NB;
        const int ir = (int)(row % NB);
        const bool qi = valid && q[row] > 0.0;
        if (valid && !rhs_only)
            for (int32_t k = ptr[node] + lane; k < ptr[node + 1]; k += kLpr) {
                const int64_t c = (int64_t)idx[k] * NB;
#pragma unroll
                for (int ic = 0; ic < NB; ++ic) {
                    const int64_t icol = c + ic;
                    const bool qj = q[icol] > 0.0;
                    double* v = val + (int64_t)k * NB * NB + ir + NB * ic;
                    if (qj && r) s = fma(*v, r[icol], s);
                    if (qi || qj) *v = (icol == row) ? 1.0 : 0.0;
                }
            }
        s = group_sum(s);
        if (valid && lane == 0 && rhs) {
            if (qi)
                rhs[row] = r ? r[row] : 0.0;
            else if (!rhs_only)
                rhs[row] -= s;
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(kThreads) k_nullify_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                          const int32_t* __restrict__ idx, double* __restrict__ val,
                                                          const double* __restrict__ mr,
                                                          const double* __restrict__ mc, double diag)
{
    const int64_t N = nodes * NB;
    RG_SROW_LOOP(N)
    {
        if (row < N) {
            const int64_t node = row / NB;
            const int ir = (int)(row % NB);
            const bool qi = mr[row] > 0.0;
            for (int32_t k = ptr[node] + lane; k < ptr[node + 1]; k += kLpr) {
                const int64_t c = (int64_t)idx[k] * NB;
#pragma unroll
                for (int ic = 0; ic < NB; ++ic)
                    if (qi || mc[c + ic] > 0.0) val[(int64_t)k * NB * NB + ir + NB * ic] = (c + ic == row) ? diag : 0.0;
            }
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(kThreads) k_spmv_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx,
                                                       const double* __restrict__ val, double alpha,
                                                       const double* __restrict__ x, double beta,
                                                       double* __restrict__ y)
{
    const int64_t N = nodes * NB;
    RG_SROW_LOOP(N)
    {
        double acc = row < N ? brow_dot<NB>(ptr, idx, val, x, row / NB, (int)(row % NB), lane) : 0.0;
        acc = group_sum(acc);
        if (row < N && lane == 0) y[row] = (beta == 0.0 ? 0.0 : beta * y[row]) + alpha * acc;
    }
}

// ------------------------------------------------------------------ balance and block Jacobi
template <int NB>
__global__ void __launch_bounds__(kThreads) k_balance_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                          const double* __restrict__ val, double* __restrict__ bv)
{
    const int64_t N = nodes * NB;
    RG_SROW_LOOP(N)
    {
        double m = 0.0;
        if (row < N) {
            const int64_t node = row / NB;
            const int ir = (int)(row % NB);
            for (int32_t k = ptr[node] + lane; k < ptr[node + 1]; k += kLpr)
#pragma unroll
                for (int ic = 0; ic < NB; ++ic) m = fmax(m, fabs(val[(int64_t)k * NB * NB + ir + NB * ic]));
        }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (row < N && lane == 0) bv[row] = m > 0.0 ? sqrt(1.0 / m) : 1.0;
    }
}

template <int NB>
__device__ bool invert_block(const double* A, double* inv)
{
    if (NB == 2) {
        double D = A[0] * A[3] - A[2] * A[1];
        if (!(fabs(D) > 0.0)) return false;
        D = 1.0 / D;
        inv[0] = A[3] * D;
        inv[1] = -A[1] * D;
        inv[2] = -A[2] * D;
        inv[3] = A[0] * D;
        return true;
    }
    const double A11 = A[0], A21 = A[1], A31 = A[2], A12 = A[3], A22 = A[4], A32 = A[5];
    const double A13 = A[6], A23 = A[7], A33 = A[8];
    double D = A11 * (A22 * A33 - A23 * A32) + A12 * (A31 * A23 - A21 * A33) + A13 * (A21 * A32 - A31 * A22);
    if (!(fabs(D) > 0.0)) return false;
    D = 1.0 / D;
    inv[0] = (A22 * A33 - A23 * A32) * D;
    inv[1] = (A31 * A23 - A21 * A33) * D;
    inv[2] = (A21 * A32 - A31 * A22) * D;
    inv[3] = (A13 * A32 - A12 * A33) * D;
    inv[4] = (A11 * A33 - A31 * A13) * D;
    inv[5] = (A12 * A31 - A11 * A32) * D;
    inv[6] = (A12 * A23 - A13 * A22) * D;
    inv[7] = (A13 * A21 - A11 * A23) * D;
    inv[8] = (A11 * A22 - A12 * A21) * D;
    return true;
}

// val *= bv_row bv_col (scale != 0) and the inverses of the main diagonal blocks; one group
// of 8 lanes per node; *bad set when a diagonal block is missing or singular
template <int NB>
__global__ void __launch_bounds__(kThreads) k_apply_balance_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                                const int32_t* __restrict__ idx,
                                                                double* __restrict__ val,
                                                                const double* __restrict__ bv, int scale,
                                                                double* __restrict__ dinv, int* bad)
{
    RG_SROW_LOOP(nodes)
    {
        int found = 0;
        if (row < nodes) {
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) {
                const int64_t j = idx[k];
                double* v = val + (int64_t)k * NB * NB;
                if (scale)
#pragma unroll
                    for (int ic = 0; ic < NB; ++ic)
#pragma unroll
                        for (int ir = 0; ir < NB; ++ir) v[ir + NB * ic] *= bv[row * NB + ir] * bv[j * NB + ic];
                if (j == row) {
                    found = 1;
                    double blk[NB * NB];
#pragma unroll
                    for (int t = 0; t < NB * NB; ++t) blk[t] = v[t];
                    if (!invert_block<NB>(blk, dinv + row * NB * NB)) atomicOr(bad, 1);
                }
            }
        }
#pragma unroll
        for (int o = kLpr / 2; o > 0; o >>= 1) found += __shfl_xor_sync(0xffffffffu, found, o);
        if (row < nodes && lane == 0 && !found) atomicOr(bad, 1);
    }
}

// out = Dinv in per node (x = D^-1 b, BlockOps_solveAll)
template <int NB>
__global__ void k_block_jacobi(int64_t nodes, const double* __restrict__ dinv, const double* __restrict__ in,
                               double* __restrict__ out)
{
    for (int64_t i = gtid(); i < nodes; i += gstride()) {
        double b[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) b[c] = in[i * NB + c];
#pragma unroll
        for (int ir = 0; ir < NB; ++ir) {
            double s = 0.0;
#pragma unroll
            for (int ic = 0; ic < NB; ++ic) s = fma(dinv[i * NB * NB + ir + NB * ic], b[ic], s);
            out[i * NB + ir] = s;
        }
    }
}

// ------------------------------------------------------------------ paso PCG on blocks
__global__ void __launch_bounds__(kThreads) k_scale_norms(int64_t n, const double* __restrict__ a,
                                                          const double* __restrict__ b, double* __restrict__ out,
                                                          ReduceBuf rb, BScal* s)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const double o = a[i] * b[i];
        out[i] = o;
        v[0] += o * o;
        v[1] = fmax(v[1], fabs(o));
    }
    double t[2];
    if (grid_reduce<2, 2u>(v, rb, t) && threadIdx.x == 0) {
        s->n2 = t[0];
        s->nm = t[1];
    }
}

__global__ void k_mul(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ o)
{
    for (int64_t i = gtid(); i < n; i += gstride()) o[i] = a[i] * b[i];
}

template <int NB>
__global__ void __launch_bounds__(kThreads) k_residual_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                           const int32_t* __restrict__ idx,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ bb, double* __restrict__ r,
                                                           ReduceBuf rb, BScal* s)
{
    const int64_t N = nodes * NB;
    double v[2] = {0.0, 0.0};
    RG_SROW_LOOP(N)
    {
        double acc = row < N ? brow_dot<NB>(ptr, idx, val, x, row / NB, (int)(row % NB), lane) : 0.0;
        acc = group_sum(acc);
        if (row < N && lane == 0) {
            const double o = bb[row] - acc;
            r[row] = o;
            v[0] += o * o;
            v[1] = fmax(v[1], fabs(o));
        }
    }
    double t[2];
    if (grid_reduce<2, 2u>(v, rb, t) && threadIdx.x == 0) {
        s->n2 = t[0];
        s->nm = t[1];
    }
}

// PCG.cpp:102-131: rs = r, x2 = x, z = Dinv r, p = z, tau = z.r
template <int NB>
__global__ void __launch_bounds__(kThreads) k_init_sys(int64_t nodes, const double* __restrict__ r,
                                                       const double* __restrict__ x, const double* __restrict__ dinv,
                                                       double* __restrict__ rs, double* __restrict__ x2,
                                                       double* __restrict__ p, double* __restrict__ z, ReduceBuf rb,
                                                       BScal* s, double tol, long long maxit)
{
    double v[1] = {0.0};
    for (int64_t i = gtid(); i < nodes; i += gstride()) {
        double rr[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            rr[c] = r[i * NB + c];
            rs[i * NB + c] = rr[c];
            x2[i * NB + c] = x[i * NB + c];
        }
#pragma unroll
        for (int ir = 0; ir < NB; ++ir) {
            double zz = 0.0;
#pragma unroll
            for (int ic = 0; ic < NB; ++ic) zz = fma(dinv[i * NB * NB + ir + NB * ic], rr[ic], zz);
            z[i * NB + ir] = zz;
            p[i * NB + ir] = zz;
            v[0] += zz * rr[ir];
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->tau = t[0];
        s->iter = 0;
        s->maxit = maxit;
        s->tol = tol;
        s->done = 0;
        s->status = ST_RUN;
        s->norm = 0.0;
    }
}

// q = A p, delta = p.q, alpha = tau/delta (PCG.cpp:223-262)
template <int NB>
__global__ void __launch_bounds__(kThreads) k_pcg_spmv_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                           const int32_t* __restrict__ idx,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ p, double* __restrict__ q,
                                                           ReduceBuf rb, BScal* s)
{
    if (s->done) return;
    const int64_t N = nodes * NB;
    double v[1] = {0.0};
    RG_SROW_LOOP(N)
    {
        double acc = row < N ? brow_dot<NB>(ptr, idx, val, p, row / NB, (int)(row % NB), lane) : 0.0;
        acc = group_sum(acc);
        if (row < N && lane == 0) {
            q[row] = acc;
            v[0] += acc * p[row];
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->delta = t[0];
        s->alpha = s->tau / t[0];
        if (fabs(t[0]) <= 0.0) {
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// r -= alpha q; smoothing sums; x2 += alpha p; z = Dinv r; tau_next = z.r (PCG.cpp:263-306)
template <int NB>
__global__ void __launch_bounds__(kThreads) k_update1_sys(int64_t nodes, double* __restrict__ r,
                                                          const double* __restrict__ q,
                                                          const double* __restrict__ rs, double* __restrict__ x2,
                                                          const double* __restrict__ p,
                                                          const double* __restrict__ dinv, double* __restrict__ z,
                                                          ReduceBuf rb, BScal* s)
{
    if (s->done) return;
    const double alpha = s->alpha;
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = gtid(); i < nodes; i += gstride()) {
        double rr[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            const int64_t o = i * NB + c;
            const double rn = r[o] - alpha * q[o];
            r[o] = rn;
            rr[c] = rn;
            const double d = rn - rs[o];
            v[0] += d * d;
            v[1] += d * rs[o];
            x2[o] += alpha * p[o];
        }
#pragma unroll
        for (int ir = 0; ir < NB; ++ir) {
            double zz = 0.0;
#pragma unroll
            for (int ic = 0; ic < NB; ++ic) zz = fma(dinv[i * NB * NB + ir + NB * ic], rr[ic], zz);
            z[i * NB + ir] = zz;
            v[2] += zz * rr[ir];
        }
    }
    double t[3];
    if (grid_reduce<3>(v, rb, t) && threadIdx.x == 0) {
        const double g1 = (fabs(t[0]) <= 0.0) ? 0.0 : -t[1] / t[0];
        s->gamma1 = g1;
        s->gamma2 = 1.0 - g1;
        s->tau_next = t[2];
        s->beta = t[2] / s->tau;
    }
}

// One more sweep of the block Jacobi smoother used as preconditioner when sweeps > 1
// (Preconditioner_LocalSmoother_solve, paso/src/Smoother.cpp:161-184): t = b - A z here,
// then z += Dinv t in k_sys_sweep_update.  mode 1 (inside the PCG loop) skips finished
// solves.
template <int NB>
__global__ void __launch_bounds__(kThreads) k_sys_sweep_resid(int64_t nodes, const int32_t* __restrict__ ptr,
                                                              const int32_t* __restrict__ idx,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ b,
                                                              const double* __restrict__ z,
                                                              double* __restrict__ t, const BScal* s, int mode)
{
    if (mode == 1 && s->done) return;
    const int64_t N = nodes * NB;
    RG_SROW_LOOP(N)
    {
        double acc = row < N ? brow_dot<NB>(ptr, idx, val, z, row / NB, (int)(row % NB), lane) : 0.0;
        acc = group_sum(acc);
        if (row < N && lane == 0) t[row] = b[row] - acc;
    }
}

// z += Dinv t per node.  mode 0: that alone; mode 1 (the last sweep inside the PCG loop):
// tau_next = z.b and beta = tau_next/tau; mode 2 (the last sweep of the PCG start): tau = z.b
// and p = z.
template <int NB>
__global__ void __launch_bounds__(kThreads) k_sys_sweep_update(int64_t nodes, const double* __restrict__ dinv,
                                                               const double* __restrict__ t,
                                                               const double* __restrict__ b,
                                                               double* __restrict__ z, double* __restrict__ p,
                                                               ReduceBuf rb, BScal* s, int mode)
{
    if (mode == 1 && s->done) return;
    double v[1] = {0.0};
    for (int64_t i = gtid(); i < nodes; i += gstride()) {
        double tt[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) tt[c] = t[i * NB + c];
#pragma unroll
        for (int ir = 0; ir < NB; ++ir) {
            double dz = 0.0;
#pragma unroll
            for (int ic = 0; ic < NB; ++ic) dz = fma(dinv[i * NB * NB + ir + NB * ic], tt[ic], dz);
            const double zz = z[i * NB + ir] + dz;
            z[i * NB + ir] = zz;
            if (mode == 2) p[i * NB + ir] = zz;
            v[0] += zz * b[i * NB + ir];
        }
    }
    if (mode == 0) return;
    double r[1];
    if (grid_reduce<1>(v, rb, r) && threadIdx.x == 0) {
        if (mode == 1) {
            s->tau_next = r[0];
            s->beta = r[0] / s->tau;
        } else {
            s->tau = r[0];
        }
    }
}

// rs, x smoothing; stopping tests (PCG.cpp:307-347); p = z + beta p (PCG.cpp:193-218)
__global__ void __launch_bounds__(kThreads) k_update2_sys(int64_t n, double* __restrict__ rs,
                                                          const double* __restrict__ r, double* __restrict__ x,
                                                          const double* __restrict__ x2,
                                                          const double* __restrict__ z, double* __restrict__ p,
                                                          ReduceBuf rb, BScal* s)
{
    if (s->done) return;
    const double g1 = s->gamma1, g2 = s->gamma2, beta = s->beta;
    double v[1] = {0.0};
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const double a = g2 * rs[i] + g1 * r[i];
        rs[i] = a;
        x[i] = g2 * x[i] + g1 * x2[i];
        p[i] = z[i] + beta * p[i];
        v[0] += a * a;
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        const long long it = s->iter + 1;
        s->iter = it;
        const double norm = sqrt(t[0]);
        s->norm = norm;
        if (it > s->maxit) {
            s->status = ST_MAXIT;
            s->done = 1;
        } else if (fabs(s->tau) <= 0.0) {
            s->status = ST_BREAK;
            s->done = 1;
        } else if (norm <= s->tol) {
            s->status = ST_CONV;
            s->done = 1;
        }
        s->tau = s->tau_next;
    }
}

// ------------------------------------------------------------------ host side
SysWorkspace* ensure_ws(Matrix* m)
{
    if (m->sws) return m->sws;
    SysWorkspace* w = new SysWorkspace();
    const int64_t N = m->dom->n * m->nb;
    w->N = N;
    cudaError_t e = cudaSuccess;
    double** v[] = {&w->r, &w->x, &w->rs, &w->x2, &w->q, &w->z, &w->p, &w->bb};
    for (double** pp : v)
        if (e == cudaSuccess) e = cudaMalloc((void**)pp, sizeof(double) * (N ? N : 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&w->partials, sizeof(double) * 4 * kNumSMs * 64);
    if (e == cudaSuccess) e = cudaMalloc((void**)&w->counter, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&w->s, sizeof(BScal));
    if (e == cudaSuccess) e = cudaMalloc((void**)&w->bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&w->hs, sizeof(BScal));
    if (e == cudaSuccess) e = cudaMemsetAsync(w->counter, 0, sizeof(unsigned), stream());
    m->sws = w;
    if (e != cudaSuccess) {
        set_error(std::string("system solver workspace: ") + cudaGetErrorString(e));
        return nullptr;
    }
    return w;
}

ReduceBuf rbuf(SysWorkspace* w) { return ReduceBuf{w->partials, w->counter}; }

int read_s(SysWorkspace* w)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(w->hs, w->s, sizeof(BScal), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    return RG_OK;
}

template <int NB>
int prepare_sys(Matrix* m, SysWorkspace* w)
{
    const Domain* d = m->dom;
    if (m->balanced && m->solver_ready) return RG_OK;
    if (!m->dinv) RG_CHECK_CUDA(cudaMalloc((void**)&m->dinv, sizeof(double) * d->n * NB * NB));
    const int grid = grid_for(d->n * NB, kThreads / kLpr, 16);
    if (!m->balanced) {
        RG_TIMED(T_BALANCE, (k_balance_sys<NB><<<grid, kThreads, 0, stream()>>>(d->n, d->ptr, m->val, m->bv)));
        RG_CHECK_LAUNCH();
    }
    RG_CHECK_CUDA(cudaMemsetAsync(w->bad, 0, sizeof(int), stream()));
    RG_TIMED(T_BALANCE, (k_apply_balance_sys<NB><<<grid_for(d->n, kThreads / kLpr, 16), kThreads, 0, stream()>>>(
                            d->n, d->ptr, d->idx, m->val, m->bv, m->balanced ? 0 : 1, m->dinv, w->bad)));
    RG_CHECK_LAUNCH();
    int bad = 0;
    RG_CHECK_CUDA(cudaMemcpyAsync(&bad, w->bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    m->balanced = true;
    if (bad) {
        set_error("SparseMatrix::invMain: non-regular main diagonal block.");
        return RG_INVALID_ARG;
    }
    m->solver_ready = true;
    return RG_OK;
}

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// paso::Solver (Solver.cpp:46-330) with Solver_PCG on the block matrix
template <int NB>
int solve_sys(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag)
{
    const double t0 = now_s();
    rg_diag dg{};
    const double EPS = 2.220446049250313e-16;
    RG_REQUIRE(o->method == RG_METHOD_PCG && o->preconditioner == RG_PRECOND_JACOBI,
               "solver: only PCG with the Jacobi preconditioner is implemented");
    RG_REQUIRE(o->tolerance >= 100. * EPS, "Solver: Tolerance is too small.");
    RG_REQUIRE(o->tolerance <= 1., "Solver: Tolerance must be less than one.");
    if (o->precision != RG_PREC_FP64 || o->initial_guess) {
        set_error("solver: PDE systems are solved by the paso algorithm in FP64");
        return RG_NOT_SUPPORTED;
    }
    SysWorkspace* w = ensure_ws(m);
    if (!w) return RG_CUDA_ERROR;
    int rc = prepare_sys<NB>(m, w);
    if (rc) return rc;
    const Domain* d = m->dom;
    const int64_t nodes = d->n, N = w->N;
    BScal* s = static_cast<BScal*>(w->s);
    BScal* hs = static_cast<BScal*>(w->hs);
    const int gv = grid_for(N, kThreads, 8);
    const int gn = grid_for(nodes, kThreads, 8);
    const int gr = grid_for(N, kThreads / kLpr, 8);
    // sweeps - 1 more block Jacobi sweeps on z (the preconditioned b), t in the spare buffer q
    auto sweeps = [&](const double* b, double* z, double* p, int last_mode) {
        for (int k = 1; k < o->sweeps; ++k) {
            const int mode = k == o->sweeps - 1 ? last_mode : 0;
            RG_TIMED(T_PASO_UPDATE1, (k_sys_sweep_resid<NB><<<gr, kThreads, 0, stream()>>>(
                                         nodes, d->ptr, d->idx, m->val, b, z, w->q, s, mode)));
            RG_TIMED(T_PASO_UPDATE1, (k_sys_sweep_update<NB><<<gn, kThreads, 0, stream()>>>(
                                         nodes, m->dinv, w->q, b, z, p, rbuf(w), s, mode)));
        }
    };
    dg.set_up_time = now_s() - t0;
    RG_TIMED(T_NORMS, (k_scale_norms<<<gv, kThreads, 0, stream()>>>(N, m->bv, rhs, w->bb, rbuf(w), s)));
    RG_CHECK_LAUNCH();
    if ((rc = read_s(w))) return rc;
    const double n2b = std::sqrt(hs->n2), nmb = hs->nm;
    dg.rhs_norm = n2b;
    int status = RG_OK;
    const double tn = now_s();
    if (std::isnan(n2b) || std::isnan(nmb)) {
        set_error("Solver: Matrix or right hand side contains undefined values.");
        status = RG_NAN;
    } else if (n2b <= 0.) {
        RG_CHECK_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * N, stream()));
        dg.converged = 1;
    } else {
        // initial guess: block Jacobi of the balanced rhs (Solver.cpp:181)
        RG_TIMED(T_VECTOR, (k_block_jacobi<NB><<<gn, kThreads, 0, stream()>>>(nodes, m->dinv, w->bb, w->x)));
        sweeps(w->bb, w->x, nullptr, 0);
        RG_CHECK_LAUNCH();
        long long totIter = 1;
        double last2 = n2b, lastm = nmb;
        bool first = true;
        for (;;) {
            RG_TIMED(T_RESIDUAL, (k_residual_sys<NB><<<gr, kThreads, 0, stream()>>>(
                                     nodes, d->ptr, d->idx, m->val, w->x, w->bb, w->r, rbuf(w), s)));
            RG_CHECK_LAUNCH();
            if ((rc = read_s(w))) return rc;
            const double n2r = std::sqrt(hs->n2), nmr = hs->nm;
            dg.residual_norm = n2r;
            dg.residual_max = nmr;
            dg.num_outer++;
            if (o->verbose) printf("Solver: Step %lld: l2/lmax-norm of residual is %g/%g\n", totIter, n2r, nmr);
            if (std::isnan(n2r)) {
                set_error("Solver: Matrix or right hand side contains undefined values.");
                status = RG_NAN;
                break;
            }
            if (!first && n2r >= last2 && nmr >= lastm) {
                set_error("Solver: No improvement during iteration. Iterative solver gives up.");
                status = RG_DIVERGENCE;
                break;
            }
            first = false;
            if (!(n2r > o->tolerance * n2b || nmr > o->tolerance * nmb)) {
                dg.converged = 1;
                break;
            }
            const double tol = o->tolerance * std::fmin(n2b, 0.1 * n2r / nmr * nmb);
            last2 = n2r;
            lastm = nmr;
            const long long cnt = o->iter_max - totIter;
            RG_TIMED(T_VECTOR, (k_init_sys<NB><<<gn, kThreads, 0, stream()>>>(nodes, w->r, w->x, m->dinv, w->rs,
                                                                             w->x2, w->p, w->z, rbuf(w), s, tol,
                                                                             cnt)));
            sweeps(w->r, w->z, w->p, 2);  // the first v = prec(r): p and tau
            RG_CHECK_LAUNCH();
            // iterations in chunks between polls of the done flag
            const int chunk = 16;
            long long launched = 0;
            for (;;) {
                for (int c = 0; c < chunk; ++c) {
                    RG_TIMED(T_PASO_SPMV, (k_pcg_spmv_sys<NB><<<gr, kThreads, 0, stream()>>>(
                                              nodes, d->ptr, d->idx, m->val, w->p, w->q, rbuf(w), s)));
                    RG_TIMED(T_PASO_UPDATE1, (k_update1_sys<NB><<<gn, kThreads, 0, stream()>>>(
                                                 nodes, w->r, w->q, w->rs, w->x2, w->p, m->dinv, w->z, rbuf(w), s)));
                    sweeps(w->r, w->z, nullptr, 1);
                    RG_TIMED(T_PASO_UPDATE2, (k_update2_sys<<<gv, kThreads, 0, stream()>>>(
                                                 N, w->rs, w->r, w->x, w->x2, w->z, w->p, rbuf(w), s)));
                }
                RG_CHECK_LAUNCH();
                launched += chunk;
                if ((rc = read_s(w))) return rc;
                if (hs->done) break;
                if (launched > cnt + 2 * chunk + 8) {
                    set_error("PCG iteration loop did not terminate");
                    return RG_TIMEOUT;
                }
            }
            const long long it = hs->iter;
            totIter += it;
            if (hs->status == ST_CONV) continue;
            if (hs->status == ST_BREAK && it > 1) continue;
            if (hs->status == ST_MAXIT) {
                set_error("Solver: maximum number of iteration steps reached.\nReturned solution does not fulfil stopping criterion.");
                status = RG_MAXITER;
            } else {
                set_error("Solver: fatal break down in iterative solver.");
                status = RG_BREAKDOWN;
            }
            break;
        }
        dg.num_iter = totIter;
        if (status == RG_OK || status == RG_MAXITER) {
            RG_TIMED(T_VECTOR, (k_mul<<<gv, kThreads, 0, stream()>>>(N, m->bv, w->x, x)));
            RG_CHECK_LAUNCH();
        }
    }
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    dg.net_time = now_s() - tn;
    dg.time = now_s() - t0;
    if (diag) *diag = dg;
    if ((status == RG_MAXITER || status == RG_DIVERGENCE) && o->accept_convergence_failure) status = RG_OK;
    return status;
}

// norms of b - A x with A as assembled (the balancing undone on the fly), per scalar row
template <int NB>
__global__ void __launch_bounds__(kThreads) k_true_residual_sys(int64_t nodes, const int32_t* __restrict__ ptr,
                                                                const int32_t* __restrict__ idx,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ bv,
                                                                const double* __restrict__ b,
                                                                const double* __restrict__ x, ReduceBuf rb,
                                                                BScal* s)
{
    const int64_t N = nodes * NB;
    double v[2] = {0.0, 0.0};
    RG_SROW_LOOP(N)
    {
        double acc = 0.0;
        if (row < N) {
            const int64_t node = row / NB;
            const int ir = (int)(row % NB);
            for (int32_t k = ptr[node] + lane; k < ptr[node + 1]; k += kLpr) {
                const int64_t c = (int64_t)idx[k] * NB;
#pragma unroll
                for (int ic = 0; ic < NB; ++ic) {
                    const double xv = bv ? x[c + ic] / bv[c + ic] : x[c + ic];
                    acc = fma(val[(int64_t)k * NB * NB + ir + NB * ic], xv, acc);
                }
            }
        }
        acc = group_sum(acc);
        if (row < N && lane == 0) {
            const double r = b[row] - (bv ? acc / bv[row] : acc);
            v[0] += r * r;
            v[1] = fmax(v[1], fabs(r));
        }
    }
    double t[2];
    if (grid_reduce<2, 2u>(v, rb, t) && threadIdx.x == 0) {
        s->n2 = t[0];
        s->nm = t[1];
    }
}

}  // namespace
}  // namespace sys

// ------------------------------------------------------------------ entry points between units
int residual_norms_system(Matrix* m, const double* b, const double* x, double* l2, double* linf)
{
    SysWorkspace* w = sys::ensure_ws(m);
    if (!w) return RG_CUDA_ERROR;
    const Domain* d = m->dom;
    const int grid = grid_for(d->n * m->nb, sys::kThreads / sys::kLpr, 8);
    const double* bv = m->balanced ? m->bv : nullptr;
    sys::BScal* s = static_cast<sys::BScal*>(w->s);
    if (m->nb == 2)
        RG_TIMED(T_NORMS, (sys::k_true_residual_sys<2><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, bv, b, x, sys::rbuf(w), s)));
    else
        RG_TIMED(T_NORMS, (sys::k_true_residual_sys<3><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, bv, b, x, sys::rbuf(w), s)));
    RG_CHECK_LAUNCH();
    int rc = sys::read_s(w);
    if (rc) return rc;
    const sys::BScal* hs = static_cast<const sys::BScal*>(w->hs);
    if (l2) *l2 = std::sqrt(hs->n2);
    if (linf) *linf = hs->nm;
    return RG_OK;
}

int assemble_system_impl(const Domain* d, int nb, double* val, double* rhs, const rg_coef* c[6], bool reduced)
{
    sys::SysArgs a;
    bool addS = false, addF = false;
    for (int j = 0; j < 6; ++j) {
        a.c[j].p = (c[j] && c[j]->kind != RG_COEF_EMPTY) ? c[j]->ptr : nullptr;
        a.c[j].kind = (c[j] && c[j]->ptr) ? c[j]->kind : RG_COEF_EMPTY;
        if (a.c[j].kind) (j < 4 ? addS : addF) = true;
    }
    a.t = reduced ? d->q1r : d->q1;
    a.NE0 = d->ne[0];
    a.NE1 = d->ne[1];
    a.NE2 = d->ne[2];
    a.NN0 = d->nn[0];
    a.NN1 = d->nn[1];
    a.NN2 = d->nn[2];
    a.n = d->n;
    a.ptr = d->ptr;
    a.val = addS ? val : nullptr;
    a.rhs = addF ? rhs : nullptr;
    if (!a.val && !a.rhs) return RG_OK;
    const int64_t threads = d->n * nb * nb;
    const int grid = (int)((threads + sys::kRows - 1) / sys::kRows);
#define RG_SYS_ASM(DIM, NB, NQ) \
    RG_TIMED(T_ASSEMBLE, (sys::k_assemble_sys<DIM, NB, NQ><<<grid, sys::kRows, 0, stream()>>>(a)))
    if (d->dim == 3 && nb == 2) {
        if (reduced) RG_SYS_ASM(3, 2, 1); else RG_SYS_ASM(3, 2, 8);
    } else if (d->dim == 3) {
        if (reduced) RG_SYS_ASM(3, 3, 1); else RG_SYS_ASM(3, 3, 8);
    } else if (nb == 2) {
        if (reduced) RG_SYS_ASM(2, 2, 1); else RG_SYS_ASM(2, 2, 4);
    } else {
        if (reduced) RG_SYS_ASM(2, 3, 1); else RG_SYS_ASM(2, 3, 4);
    }
#undef RG_SYS_ASM
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_system_constraint(Matrix* m, double* rhs, const double* q, const double* r, int rhs_only)
{
    const Domain* d = m->dom;
    const int grid = grid_for(d->n * m->nb, sys::kThreads / sys::kLpr, 16);
    if (m->nb == 2)
        RG_TIMED(T_CONSTRAINT, (sys::k_constraint_sys<2><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, rhs, q, r, rhs_only)));
    else
        RG_TIMED(T_CONSTRAINT, (sys::k_constraint_sys<3><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, rhs, q, r, rhs_only)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_system_nullify(Matrix* m, const double* mr, const double* mc, double diag)
{
    const Domain* d = m->dom;
    const int grid = grid_for(d->n * m->nb, sys::kThreads / sys::kLpr, 16);
    if (m->nb == 2)
        RG_TIMED(T_CONSTRAINT, (sys::k_nullify_sys<2><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, mr, mc, diag)));
    else
        RG_TIMED(T_CONSTRAINT, (sys::k_nullify_sys<3><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, mr, mc, diag)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_system_spmv(const Matrix* m, double alpha, const double* x, double beta, double* y)
{
    const Domain* d = m->dom;
    const int grid = grid_for(d->n * m->nb, sys::kThreads / sys::kLpr, 16);
    if (m->nb == 2)
        RG_TIMED(T_SPMV, (sys::k_spmv_sys<2><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, alpha, x, beta, y)));
    else
        RG_TIMED(T_SPMV, (sys::k_spmv_sys<3><<<grid, sys::kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, alpha, x, beta, y)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int solve_system(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag)
{
    return m->nb == 2 ? sys::solve_sys<2>(m, rhs, x, o, diag) : sys::solve_sys<3>(m, rhs, x, o, diag);
}

void free_system_workspace(Matrix* m)
{
    SysWorkspace* w = m->sws;
    if (!w) return;
    double* v[] = {w->r, w->x, w->rs, w->x2, w->q, w->z, w->p, w->bb, w->partials};
    for (double* p : v) cudaFree(p);
    cudaFree(w->counter);
    cudaFree(w->s);
    cudaFree(w->bad);
    cudaFreeHost(w->hs);
    delete w;
    m->sws = nullptr;
}

}  // namespace rg
