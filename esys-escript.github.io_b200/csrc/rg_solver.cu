// paso Solver() + Solver_PCG on the device.
//
//  * RG_MODE_PASO: the reference algorithm (paso/src/Solver.cpp:46-330 and
//    paso/src/PCG.cpp:62-367): in-place balancing, Jacobi initial guess, PCG with the
//    minimal-residual smoothing sequence (rs, x2, gamma_1/2) stopping on the smoothed
//    residual, and the outer loop's dual l2/lmax test on the true residual.
//  * RG_MODE_STANDARD: the same outer loop around textbook Jacobi-PCG (no smoothing).
//  * RG_PREC_FP32_REFINE: FP32 Jacobi-PCG on the band copy of the balanced matrix with
//    FP64 residual replacement: the solution is accumulated in FP64, and every time the
//    recursive FP32 residual has dropped by `inner_tolerance` the true residual is
//    recomputed in FP64 on the CSR values, tested with paso's dual-norm criterion and
//    written back into the FP32 recurrence (the Krylov direction is kept, no restart).
//    One FP32 iteration is one kernel (k_f32_cg, the one-reduction recurrence of
//    Chronopoulos and Gear).
//
// One FP64 PCG iteration is three kernels: a pure SpMV of the search direction with its
// p.q reduction, an elementwise update with the iteration's reductions, and an
// elementwise kernel that forms the next search direction (in paso mode it also does
// the smoothing step).  Scalars (alpha, beta, tau, ...) live in device memory: the last
// CTA of each reduction kernel finishes the sum in a fixed order, sets the next step's
// scalars and a `done` flag, so the host polls `done` once per chunk of iterations and
// kernels queued after convergence return at once.  Elementwise kernels use 16-byte
// vector accesses; matrix data is loaded with streaming (evict-first) hints so that the
// solver vectors stay resident in the 126 MB L2.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "rg_bulk.cuh"
#include "rg_internal.cuh"

namespace rg {
using namespace bulk;

namespace {

constexpr int kLpr = 8;  // lanes per CSR row
constexpr int kThreads = 256;

struct Scal {
    double tau, tau_next;      // paso: tau = v.r of this and of the next iteration
    double delta, alpha, beta;
    double gamma1, gamma2;
    double norm, tol;          // stopping norm and its limit
    double rho;                // textbook PCG: r.z
    double n2, nm;             // norms from norm kernels
    long long iter, maxit;
    long long pk;              // FP32 path: parity counter of the two search-direction buffers
    double best;               // FP32 path: smallest recursive residual norm of the segment
    int since;                 // iterations since `best` last dropped by 5%
    int done, status;
};

enum { ST_RUN = 0, ST_CONV = 1, ST_MAXIT = 3, ST_BREAK = 4 };

}  // namespace

struct Workspace {
    int64_t n = 0;
    double *r = nullptr, *x = nullptr, *rs = nullptr, *x2 = nullptr, *q = nullptr, *z = nullptr;
    double* p = nullptr;
    double* bb = nullptr;  // balanced rhs
    float* d32 = nullptr;                // FP32 path: correction accumulated over a segment
    float4* v4[2] = {nullptr, nullptr};  // FP32 iteration state {u, D^-1 A u, D^-1 A p_prev, p_prev}
    double* partials = nullptr;
    unsigned* counter = nullptr;
    Scal* s = nullptr;   // device scalars
    Scal* hs = nullptr;  // pinned host copy
    int* bad = nullptr;
    int grid_rows = 0;   // CSR row-group kernels
    int grid_vec = 0;    // elementwise kernels
    // solves run on a private stream (ordered after and before the caller's stream) so
    // that chunks of iterations can be captured and replayed as CUDA graphs
    cudaStream_t priv = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaEvent_t poll_ev[2] = {nullptr, nullptr};
    Scal* hpoll = nullptr;                   // 2 pinned slots for pipelined polling
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
    int graph_chunk[3] = {0, 0, 0};
    int graph_sweeps[3] = {0, 0, 0};  // Jacobi sweeps the captured iterations apply
    bool graph_coef[3] = {false, false, false};  // the captured FP32 iterations' operator
    long long graph_launches[3][T_COUNT] = {};
    int sweeps = 1;  // Jacobi sweeps of the current paso solve (Smoother.cpp:100-128)
    bool band64 = false;              // paso FP64 SpMV on the FP64 band copy (RG_LAYOUT_BAND)
    bool graph_band64[3] = {false, false, false};
    int spmv_cfg = -1;   // FP32 iteration pipeline of the band operator (kSpmvCfg; -1: not tuned)
    int coef_cfg = -1;   // the same for the element-coefficient operator (kCoefCfg)
    bool coef_op = false;  // the current FP32 solve evaluates the operator from the coefficients
    int grid_upd32 = 0;  // kept for rg_solver_config: the FP32 iteration has no separate update kernel
    double spmv_us[2][2] = {};   // tuner's time per launch of each configuration [coef_op][cfg]
};

namespace {

template <typename T>
int dalloc(T** p, size_t count)
{
    RG_CHECK_CUDA(cudaMalloc((void**)p, sizeof(T) * (count ? count : 1)));
    return RG_OK;
}

int ensure_workspace(Matrix* m, bool fp32)
{
    const int64_t n = m->dom->n;
    if (!m->ws) {
        // the solver vectors of a destroyed matrix on this grid: the captured iteration graphs
        // named that matrix's arrays and were dropped; the SpMV pipeline is tuned again
        std::lock_guard<std::mutex> lock(pool_mutex());
        if (m->dom->spare_ws) {
            m->ws = m->dom->spare_ws;
            m->dom->spare_ws = nullptr;
            m->ws->spmv_cfg = -1;
            m->ws->coef_cfg = -1;
            m->ws->grid_upd32 = 0;
        }
    }
    if (!m->ws) {
        Workspace* w = new Workspace();
        m->ws = w;
        w->n = n;
        w->grid_rows = grid_for(n, kThreads / kLpr, 8);
        w->grid_vec = grid_for((n + 3) / 4, kThreads, 8);
        int rc;
        if ((rc = dalloc(&w->r, n)) || (rc = dalloc(&w->x, n)) || (rc = dalloc(&w->rs, n)) ||
            (rc = dalloc(&w->x2, n)) || (rc = dalloc(&w->q, n)) || (rc = dalloc(&w->z, n)) ||
            (rc = dalloc(&w->p, n)) || (rc = dalloc(&w->bb, n)) ||
            (rc = dalloc(&w->partials, (size_t)4 * kNumSMs * 64)) || (rc = dalloc(&w->counter, 1)) ||
            (rc = dalloc(&w->s, 1)) || (rc = dalloc(&w->bad, 1)))
            return rc;
        RG_CHECK_CUDA(cudaMallocHost((void**)&w->hs, sizeof(Scal)));
        RG_CHECK_CUDA(cudaMallocHost((void**)&w->hpoll, 2 * sizeof(Scal)));
        RG_CHECK_CUDA(cudaStreamCreateWithFlags(&w->priv, cudaStreamNonBlocking));
        RG_CHECK_CUDA(cudaEventCreateWithFlags(&w->ev_in, cudaEventDisableTiming));
        RG_CHECK_CUDA(cudaEventCreateWithFlags(&w->ev_out, cudaEventDisableTiming));
        RG_CHECK_CUDA(cudaEventCreateWithFlags(&w->poll_ev[0], cudaEventDisableTiming));
        RG_CHECK_CUDA(cudaEventCreateWithFlags(&w->poll_ev[1], cudaEventDisableTiming));
        RG_CHECK_CUDA(cudaMemsetAsync(w->counter, 0, sizeof(unsigned), stream()));
    }
    Workspace* w = m->ws;
    if (fp32 && !w->d32) {
        int rc;
        if ((rc = dalloc(&w->d32, n)) || (rc = dalloc(&w->v4[0], n)) || (rc = dalloc(&w->v4[1], n))) return rc;
    }
    return RG_OK;
}

// ------------------------------------------------------------------ access helpers
__device__ __forceinline__ int64_t gtid() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

__device__ __forceinline__ double2 ld2(const double* p, int64_t v) { return reinterpret_cast<const double2*>(p)[v]; }
__device__ __forceinline__ void st2(double* p, int64_t v, double2 a) { reinterpret_cast<double2*>(p)[v] = a; }

// CSR row-group loop: each group of kLpr lanes owns one row per trip; the trip count is
// uniform over a warp so the shuffles stay converged.
#define RG_ROW_LOOP(n)                                                                  \
    const int lane = threadIdx.x & (kLpr - 1);                                          \
    const int64_t groups_ = (int64_t)gridDim.x * blockDim.x / kLpr;                     \
    const int64_t g0_ = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLpr;        \
    const int64_t wg0_ = g0_ & ~(int64_t)(32 / kLpr - 1);                               \
    for (int64_t gb_ = wg0_; gb_ < (n); gb_ += groups_)                                 \
        if (const int64_t row = gb_ + (g0_ - wg0_); true)

__device__ __forceinline__ double group_sum(double s)
{
#pragma unroll
    for (int o = kLpr / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// sum_k val[k]*x[idx[k]] over this lane's entries of CSR row `row`; all loads of a
// 32-entry chunk are issued before the multiply-adds.  Matrix data streams (evict-first).
__device__ __forceinline__ double csr_row_dot(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                              const double* __restrict__ val, const double* __restrict__ x,
                                              int64_t row, int lane)
{
    const int32_t k0 = __ldg(ptr + row), k1 = __ldg(ptr + row + 1);
    double acc = 0.0;
    for (int32_t kb = k0 + lane; kb < k1; kb += 4 * kLpr) {
        int32_t j[4];
        double a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int32_t k = kb + u * kLpr;
            const bool ok = k < k1;
            j[u] = ok ? __ldcs(idx + k) : (int32_t)row;
            a[u] = ok ? __ldcs(val + k) : 0.0;
        }
        double xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) xv[u] = __ldg(x + j[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) acc = fma(a[u], xv[u], acc);
    }
    return acc;
}

// ------------------------------------------------------------------ common kernels
// out = a .* b, with ||out||_2^2 and ||out||_inf into s->n2, s->nm.  b is the caller's
// right hand side, whose alignment is unknown, so the accesses are scalar.
__global__ void __launch_bounds__(kThreads) k_scale_norms(int64_t n, const double* __restrict__ a,
                                                          const double* __restrict__ b,
                                                          double* __restrict__ out, ReduceBuf rb, Scal* s)
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

// r = bb - A x (paso MatrixVector_CSR_OFFSET0(-1, x, 1, r)) with l2^2 / max norms of r
__global__ void __launch_bounds__(kThreads) k_residual(int64_t n, const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx,
                                                       const double* __restrict__ val,
                                                       const double* __restrict__ x,
                                                       const double* __restrict__ bb,
                                                       double* __restrict__ r, ReduceBuf rb, Scal* s)
{
    double v[2] = {0.0, 0.0};
    RG_ROW_LOOP(n)
    {
        double acc = row < n ? csr_row_dot(ptr, idx, val, x, row, lane) : 0.0;
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            const double o = bb[row] + (-1.0) * acc;
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

// One step of Chebyshev smoothing with the Jacobi preconditioner on the balanced system
// (the semi-iterative method for D^-1 A with eigenvalues in [a, b]):
//   d = c_d d + c_r D^-1 (bb - A x),  y = x + d
// (step 0: c_d = 0, c_r = 1/theta).  It damps the error components of D^-1 A in [a, b]
// uniformly, the rough part of a guess that dominates its residual.
__global__ void __launch_bounds__(kThreads) k_cheb_step(int64_t n, const int32_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        const double* __restrict__ dinv,
                                                        const double* __restrict__ x,
                                                        const double* __restrict__ bb, double c_d, double c_r,
                                                        double* __restrict__ d, double* __restrict__ y)
{
    RG_ROW_LOOP(n)
    {
        double acc = row < n ? csr_row_dot(ptr, idx, val, x, row, lane) : 0.0;
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            const double dn = c_d * (c_d != 0.0 ? d[row] : 0.0) + c_r * dinv[row] * (bb[row] - acc);
            d[row] = dn;
            y[row] = x[row] + dn;
        }
    }
}

// Gershgorin bound of the spectrum of D^-1 A: max over rows of sum_j |a_ij| / a_ii
__global__ void __launch_bounds__(kThreads) k_gershgorin(int64_t n, const int32_t* __restrict__ ptr,
                                                         const double* __restrict__ val,
                                                         const double* __restrict__ dinv, ReduceBuf rb,
                                                         double* __restrict__ out)
{
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = 0.0;
        if (row < n)
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) acc += fabs(val[k]);
        acc = group_sum(acc);
        if (row < n && lane == 0) v[0] = fmax(v[0], acc * fabs(dinv[row]));
    }
    double t[1];
    if (grid_reduce<1, 1u>(v, rb, t) && threadIdx.x == 0) *out = t[0];
}

__global__ void k_mul(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out)
{
    for (int64_t i = gtid(); i < n; i += gstride()) out[i] = a[i] * b[i];
}

__global__ void k_div(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out)
{
    for (int64_t i = gtid(); i < n; i += gstride()) out[i] = a[i] / b[i];
}

// ------------------------------------------------------------------ paso PCG (FP64, CSR)
// PCG.cpp:102-131 initialisation, the first v = prec(r), tau = v.r and p = v
__global__ void __launch_bounds__(kThreads) k_paso_init(int64_t n, const double* __restrict__ r,
                                                        const double* __restrict__ x,
                                                        const double* __restrict__ dinv,
                                                        double* __restrict__ rs, double* __restrict__ x2,
                                                        double* __restrict__ p, double* __restrict__ z,
                                                        ReduceBuf rb, Scal* s, double tol, long long maxit)
{
    double v[1] = {0.0};
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const double ri = r[i];
        rs[i] = ri;
        x2[i] = x[i];
        const double zi = ri * dinv[i];
        z[i] = zi;
        p[i] = zi;
        v[0] += zi * ri;
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

// v = A*p (PCG.cpp:223), delta = p.v, alpha = tau/delta; breakdown on delta == 0 (228-262)
__global__ void __launch_bounds__(kThreads) k_paso_spmv(int64_t n, const int32_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        const double* __restrict__ p,
                                                        double* __restrict__ q, ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = row < n ? csr_row_dot(ptr, idx, val, p, row, lane) : 0.0;
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            q[row] = acc;
            v[0] += acc * p[row];
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->delta = t[0];
        s->alpha = s->tau / t[0];
        if (fabs(t[0]) <= 0.0) {  // breakFlag
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// One more sweep of the Jacobi smoother used as preconditioner when sweeps > 1
// (Preconditioner_LocalSmoother_solve, paso/src/Smoother.cpp:161-184: b_new = b - A x,
// x += D^-1 b_new): zout = zin + dinv (b - A zin).  mode 0: that alone; mode 1 (the last
// sweep inside the PCG loop): tau_next = zout.b and beta = tau_next/tau; mode 2 (the last
// sweep of the PCG start): tau = zout.b and p = zout.
__global__ void __launch_bounds__(kThreads) k_jacobi_sweep(int64_t n, const int32_t* __restrict__ ptr,
                                                           const int32_t* __restrict__ idx,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ dinv,
                                                           const double* __restrict__ b,
                                                           const double* __restrict__ zin,
                                                           double* __restrict__ zout, double* __restrict__ p,
                                                           ReduceBuf rb, Scal* s, int mode)
{
    if (mode == 1 && s->done) return;
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = row < n ? csr_row_dot(ptr, idx, val, zin, row, lane) : 0.0;
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            const double bi = b[row];
            const double db = dinv[row] * (bi - acc);
            const double zi = zin[row] + db;
            zout[row] = zi;
            if (mode == 2) p[row] = zi;
            v[0] += zi * bi;
        }
    }
    if (mode == 0) return;
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        if (mode == 1) {
            s->tau_next = t[0];
            s->beta = t[0] / s->tau;
        } else {
            s->tau = t[0];
        }
    }
}

// r -= alpha*v; d = r - rs; sum d^2 and d.rs (PCG.cpp:263-306); x2 += alpha*p; the next
// iteration's v = prec(r) and tau = v.r, so that beta = tau_next/tau is known before
// the smoothing kernel
__global__ void __launch_bounds__(kThreads) k_paso_update1(int64_t n, double* __restrict__ r,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ rs,
                                                           double* __restrict__ x2,
                                                           const double* __restrict__ p,
                                                           const double* __restrict__ dinv,
                                                           double* __restrict__ z, ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double alpha = s->alpha;
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t nv = n >> 1;
    for (int64_t k = gtid(); k < nv; k += gstride()) {
        const double2 r0 = ld2(r, k), q0 = ld2(q, k), rs0 = ld2(rs, k), x20 = ld2(x2, k);
        const double2 p0 = ld2(p, k), di = ld2(dinv, k);
        const double ra = r0.x - alpha * q0.x, rb2 = r0.y - alpha * q0.y;
        st2(r, k, make_double2(ra, rb2));
        const double da = ra - rs0.x, db = rb2 - rs0.y;
        v[0] += da * da + db * db;
        v[1] += da * rs0.x + db * rs0.y;
        st2(x2, k, make_double2(x20.x + alpha * p0.x, x20.y + alpha * p0.y));
        const double za = ra * di.x, zb = rb2 * di.y;
        st2(z, k, make_double2(za, zb));
        v[2] += za * ra + zb * rb2;
    }
    if ((n & 1) && gtid() == 0) {
        const int64_t i = n - 1;
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double d = ri - rs[i];
        v[0] += d * d;
        v[1] += d * rs[i];
        x2[i] += alpha * p[i];
        const double zi = ri * dinv[i];
        z[i] = zi;
        v[2] += zi * ri;
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

// rs = g2 rs + g1 r; x = g2 x + g1 x2; sum rs^2; stopping tests (PCG.cpp:307-347); then
// the next search direction p = v + beta p (PCG.cpp:193-218)
__global__ void __launch_bounds__(kThreads) k_paso_update2(int64_t n, double* __restrict__ rs,
                                                           const double* __restrict__ r,
                                                           double* __restrict__ x,
                                                           const double* __restrict__ x2,
                                                           const double* __restrict__ z,
                                                           double* __restrict__ p, ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double g1 = s->gamma1, g2 = s->gamma2, beta = s->beta;
    double v[1] = {0.0};
    const int64_t nv = n >> 1;
    for (int64_t k = gtid(); k < nv; k += gstride()) {
        const double2 rs0 = ld2(rs, k), r0 = ld2(r, k), x0 = ld2(x, k), x20 = ld2(x2, k);
        const double2 z0 = ld2(z, k), p0 = ld2(p, k);
        const double a = g2 * rs0.x + g1 * r0.x, b = g2 * rs0.y + g1 * r0.y;
        st2(rs, k, make_double2(a, b));
        st2(x, k, make_double2(g2 * x0.x + g1 * x20.x, g2 * x0.y + g1 * x20.y));
        st2(p, k, make_double2(z0.x + beta * p0.x, z0.y + beta * p0.y));
        v[0] += a * a + b * b;
    }
    if ((n & 1) && gtid() == 0) {
        const int64_t i = n - 1;
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
        const bool conv = norm <= s->tol;
        const bool maxf = it > s->maxit;
        const bool brk = fabs(s->tau) <= 0.0;
        if (maxf) {
            s->status = ST_MAXIT;
            s->done = 1;
        } else if (brk) {
            s->status = ST_BREAK;
            s->done = 1;
        } else if (conv) {
            s->status = ST_CONV;
            s->done = 1;
        }
        s->tau = s->tau_next;
    }
}

// ------------------------------------------------------------------ textbook PCG, FP64 CSR
__global__ void __launch_bounds__(kThreads) k_std_init(int64_t n, const double* __restrict__ r,
                                                       const double* __restrict__ dinv,
                                                       double* __restrict__ z, double* __restrict__ p,
                                                       ReduceBuf rb, Scal* s, double tol, long long maxit)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const double ri = r[i];
        const double zi = ri * dinv[i];
        z[i] = zi;
        p[i] = zi;
        v[0] += zi * ri;
        v[1] += ri * ri;
    }
    double t[2];
    if (grid_reduce<2>(v, rb, t) && threadIdx.x == 0) {
        s->rho = t[0];
        s->norm = sqrt(t[1]);
        s->iter = 0;
        s->maxit = maxit;
        s->tol = tol;
        s->status = ST_RUN;
        s->done = (s->norm <= tol) ? 1 : 0;
        if (s->done) s->status = ST_CONV;
    }
}

__global__ void __launch_bounds__(kThreads) k_std_spmv(int64_t n, const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx,
                                                       const double* __restrict__ val,
                                                       const double* __restrict__ p,
                                                       double* __restrict__ q, ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = row < n ? csr_row_dot(ptr, idx, val, p, row, lane) : 0.0;
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            q[row] = acc;
            v[0] += acc * p[row];
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->delta = t[0];
        s->alpha = s->rho / t[0];
        if (!(fabs(t[0]) > 0.0)) {
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// x += alpha p; r -= alpha q; z = dinv r; rho_next = r.z, ||r||^2; stopping tests; beta
__global__ void __launch_bounds__(kThreads) k_std_update(int64_t n, double* __restrict__ x,
                                                         double* __restrict__ r,
                                                         const double* __restrict__ q,
                                                         const double* __restrict__ p,
                                                         const double* __restrict__ dinv,
                                                         double* __restrict__ z, ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double alpha = s->alpha;
    double v[2] = {0.0, 0.0};
    const int64_t nv = n >> 1;
    for (int64_t k = gtid(); k < nv; k += gstride()) {
        const double2 x0 = ld2(x, k), r0 = ld2(r, k), q0 = ld2(q, k), p0 = ld2(p, k), di = ld2(dinv, k);
        st2(x, k, make_double2(x0.x + alpha * p0.x, x0.y + alpha * p0.y));
        const double ra = r0.x - alpha * q0.x, rb2 = r0.y - alpha * q0.y;
        st2(r, k, make_double2(ra, rb2));
        const double za = ra * di.x, zb = rb2 * di.y;
        st2(z, k, make_double2(za, zb));
        v[0] += za * ra + zb * rb2;
        v[1] += ra * ra + rb2 * rb2;
    }
    if ((n & 1) && gtid() == 0) {
        const int64_t i = n - 1;
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double zi = ri * dinv[i];
        z[i] = zi;
        v[0] += zi * ri;
        v[1] += ri * ri;
    }
    double t[2];
    if (grid_reduce<2>(v, rb, t) && threadIdx.x == 0) {
        const long long it = s->iter + 1;
        s->iter = it;
        const double norm = sqrt(t[1]);
        s->norm = norm;
        s->beta = t[0] / s->rho;
        const bool brk = !(fabs(t[0]) > 0.0);
        s->rho = t[0];
        if (norm <= s->tol) {
            s->status = ST_CONV;
            s->done = 1;
        } else if (it >= s->maxit) {
            s->status = ST_MAXIT;
            s->done = 1;
        } else if (brk) {
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_std_pupdate(int64_t n, const double* __restrict__ z,
                                                          double* __restrict__ p, const Scal* s)
{
    if (s->done) return;
    const double beta = s->beta;
    const int64_t nv = n >> 1;
    for (int64_t k = gtid(); k < nv; k += gstride()) {
        const double2 z0 = ld2(z, k), p0 = ld2(p, k);
        st2(p, k, make_double2(z0.x + beta * p0.x, z0.y + beta * p0.y));
    }
    if ((n & 1) && gtid() == 0) p[n - 1] = z[n - 1] + beta * p[n - 1];
}

// ------------------------------------------------------------------ FP32 PCG on the band copy
// Tile-major band layout: rows are grouped in tiles of kTile; tile T's coefficients are
// band[(T*NB + b)*kTile + t] for row T*kTile + t and band b (neighbour i + off_b; 0 where
// there is none, and in padding rows), so one tile's whole matrix slice is one contiguous
// NB*kTile*4-byte block.  One FP32 PCG iteration is one kernel (k_f32_cg below).
constexpr int kTile = 256;
constexpr int kConsumerWarps = kTile / 32;
enum { ST_TIMEOUT = 6 };

// Limits of the bounded waits of the warp-specialised kernels below, read once per CTA.
// polls = 0 keeps the default limit; withhold != 0 makes the producer issue no copies, so
// that every consumer wait runs out without any copy in flight (the test of the timeout
// path sets both through rg_test_wait_limit).
struct WaitCtl {
    int polls;
    int withhold;
};
__device__ WaitCtl g_wait_ctl = {0, 0};

// A CTA whose wait gave up records the timeout; status codes are ordered so that the
// most severe one wins when several CTAs report at once (ST_TIMEOUT > ST_BREAK > ...).
__device__ __forceinline__ void report_status(Scal* s, int st)
{
    atomicMax(&s->status, st);
    s->done = 1;
}

struct TmaBandArgs {
    int off[27];   // column offset of band b
    int goff[9];   // column offset of stencil column g = (dy,dz) at dx = -1
    int64_t n;
    int64_t halo;  // largest |offset|
};

// k_cheb_step on the FP32 band copy (tile-major, absent neighbours hold 0): the same step
// with the balanced matrix rounded to FP32, x, d and y in FP64.  One thread per row; the
// band values of a tile are read coalesced band by band.
template <int NB>
__global__ void __launch_bounds__(kThreads) k_cheb_step_band(const __grid_constant__ TmaBandArgs ta,
                                                             const float* __restrict__ band,
                                                             const double* __restrict__ dinv,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ bb, double c_d, double c_r,
                                                             double* __restrict__ d, double* __restrict__ y)
{
    const int64_t n = ta.n;
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const float* bt = band + (i >> 8) * (int64_t)NB * 256 + (i & 255);
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int64_t j = i + ta.off[b];
            const int64_t jc = j < 0 ? 0 : (j >= n ? n - 1 : j);
            acc = fma((double)__ldg(bt + b * 256), __ldg(x + jc), acc);
        }
        const double dn = c_d * (c_d != 0.0 ? d[i] : 0.0) + c_r * dinv[i] * (bb[i] - acc);
        d[i] = dn;
        y[i] = x[i] + dn;
    }
}

// The FP64 band kernels of the paso PCG (RG_LAYOUT_BAND), warp-specialised and persistent
// like k_f32_cg: lane 0 of warp kConsumerWarps streams, per tile, the tile's FP64 band
// block (one bulk copy, L2 evict-first) and, for interior tiles, the NG windows of x its
// stencil columns span (kTile+4 values from a 16-byte aligned start) into a kStages ring;
// consumer warps compute row i0 + t from shared memory.  Tiles near the two ends read x with
// clamped loads.  The bands are summed in column order.
//   SWEEP = false: v = A x, delta = x.v; mode 0: alpha = tau/delta, breakdown on delta == 0
//                  (PCG.cpp:223-262), i.e. k_paso_spmv; mode 1: alpha = rho/delta, i.e.
//                  k_std_spmv (RG_MODE_STANDARD).
//   SWEEP = true:  one Jacobi sweep out = x + dinv (b - A x) with k_jacobi_sweep's modes.
// All waits are bounded: on timeout the kernel records ST_TIMEOUT and returns.
constexpr int kWin64 = kTile + 4;

template <int NB, int kStages>
constexpr size_t band64_smem()
{
    return sizeof(double) * (size_t)kStages * (NB * kTile + (NB / 3) * kWin64);
}

template <int NB, int kStages, bool SWEEP>
__global__ void __launch_bounds__(kTile + 32, 1) k_band64_bulk(const double* __restrict__ band,
                                                               const __grid_constant__ TmaBandArgs ta,
                                                               const double* __restrict__ x,
                                                               double* __restrict__ out,
                                                               const double* __restrict__ dinv,
                                                               const double* __restrict__ b,
                                                               double* __restrict__ pout, ReduceBuf rb, Scal* s,
                                                               int mode)
{
    constexpr int NG = NB / 3;
    constexpr int kBand = NB * kTile;
    constexpr int kStage = kBand + NG * kWin64;
    extern __shared__ __align__(128) double smem64[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
    __shared__ int bad;
    if (SWEEP ? (mode == 1 && s->done) : s->done) return;
    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int64_t n = ta.n;
    const int64_t ntiles = (n + kTile - 1) / kTile;
    const int64_t my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    if (t == 0) {
        for (int k = 0; k < kStages; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], kConsumerWarps);
        }
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto interior = [&](int64_t i0) { return i0 - ta.halo - 8 >= 0 && i0 + kTile + ta.halo + 8 <= n; };

    double v[1] = {0.0};
    int64_t issued = 0;
    const WaitCtl wc = g_wait_ctl;
    const int polls = wc.polls > 0 ? wc.polls : kDefaultPolls;
    if (warp == kConsumerWarps) {
        // ---------------- producer
        if ((t & 31) == 0 && !wc.withhold) {
            const uint64_t pol = evict_first_policy();
            for (int64_t k = 0; k < my_tiles; ++k, issued = k) {
                const int st = (int)(k % kStages);
                if (k >= kStages && !mbar_wait(&empty[st], (uint32_t)(((k / kStages) - 1) & 1), polls)) {
                    bad = 1;
                    break;
                }
                const int64_t tile = blockIdx.x + k * gridDim.x;
                const int64_t i0 = tile * kTile;
                double* dst = smem64 + (size_t)st * kStage;
                const bool in = interior(i0);
                mbar_expect_tx(&full[st], (kBand + (in ? NG * kWin64 : 0)) * 8);
                bulk_g2s_hint(dst, band + (size_t)tile * kBand, kBand * 8, &full[st], pol);
                if (in)
                    for (int g = 0; g < NG; ++g) {
                        const int64_t a = (i0 + ta.goff[g]) & ~(int64_t)1;
                        bulk_g2s(dst + kBand + g * kWin64, x + a, kWin64 * 8, &full[st]);
                    }
            }
        }
    } else {
        // ---------------- consumers: row i0 + t of every tile
        for (int64_t k = 0; k < my_tiles; ++k) {
            const int st = (int)(k % kStages);
            if (!mbar_wait(&full[st], (uint32_t)((k / kStages) & 1), polls)) {
                bad = 1;
                break;
            }
            const double* bs = smem64 + (size_t)st * kStage;
            const int64_t i0 = (blockIdx.x + k * gridDim.x) * (int64_t)kTile;
            const int64_t i = i0 + t;
            double acc = 0.0, xi = 0.0;
            if (interior(i0)) {
                const double* xw = bs + kBand;
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    const int base = (int)((i0 + ta.goff[g]) & 1) + t + g * kWin64;
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const double xj = xw[base + m];
                        acc = fma(bs[(3 * g + m) * kTile + t], xj, acc);
                        if (3 * g + m == NB / 2) xi = xj;
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    const int64_t j = min(max(i + ta.off[c], (int64_t)0), n - 1);
                    const double xj = __ldg(x + j);
                    acc = fma(bs[c * kTile + t], xj, acc);
                    if (c == NB / 2) xi = xj;
                }
            }
            __syncwarp();
            if ((t & 31) == 0) mbar_arrive(&empty[st]);
            if (i < n) {
                if (SWEEP) {
                    const double bi = b[i];
                    const double zi = xi + dinv[i] * (bi - acc);
                    out[i] = zi;
                    if (mode == 2) pout[i] = zi;
                    v[0] += zi * bi;
                } else {
                    out[i] = acc;
                    v[0] += acc * xi;
                }
            }
        }
    }
    __syncthreads();
    if (bad) {
        // let the copies this CTA issued land (bounded) before its shared memory is released
        if (warp == kConsumerWarps && (t & 31) == 0)
            for (int64_t k = issued > kStages ? issued - kStages : 0; k < issued; ++k)
                for (int tries = 0; tries < (1 << 20) && !mbar_try_wait(&full[k % kStages], (uint32_t)((k / kStages) & 1));
                     ++tries) {
                }
        if (t == 0) report_status(s, ST_TIMEOUT);
        // the CTA still takes its turn in the grid reduction (with nothing to add), so the
        // reduction counter ends the launch at zero for the kernels that follow
        v[0] = 0.0;
    }
    if (SWEEP && mode == 0) return;
    double tt[1];
    if (grid_reduce<1>(v, rb, tt) && threadIdx.x == 0) {
        if (!SWEEP && mode == 0) {
            s->delta = tt[0];
            s->alpha = s->tau / tt[0];
            if (fabs(tt[0]) <= 0.0) {  // breakFlag
                s->iter += 1;
                report_status(s, ST_BREAK);
            }
        } else if (!SWEEP) {
            s->delta = tt[0];
            s->alpha = s->rho / tt[0];
            if (!(fabs(tt[0]) > 0.0)) {
                s->iter += 1;
                report_status(s, ST_BREAK);
            }
        } else if (mode == 1) {
            s->tau_next = tt[0];
            s->beta = tt[0] / s->tau;
        } else {
            s->tau = tt[0];
        }
    }
}

// stages of the FP64 band ring: 3 x 74 KB (27 bands) or 8 x 24 KB (9 bands), one CTA per SM
template <int NB>
constexpr int band64_stages() { return NB == 27 ? 3 : 8; }

// ------------------------------------------------------------------ FP32 PCG, one kernel per iteration
// Jacobi-PCG in the one-reduction form of Chronopoulos and Gear ("s-step iterative methods
// for symmetric linear systems", J. Comput. Appl. Math. 25, 1989): besides the search
// direction p the recurrences carry s = A p and w = A u (u = D^-1 r, the preconditioned
// residual), so that the SpMV of an iteration is applied to u_{i+1}, which every tile can
// form itself from the previous vectors:
//     p_i = u_i + b_i p_{i-1}          s_i = w_i + b_i s_{i-1}          d += a_i p_i
//     u_{i+1} = u_i - a_i D^-1 s_i     w_{i+1} = A u_{i+1}
// and all scalars of the next iteration come from ONE grid reduction over the rows:
//     g = r.u = sum diag u^2,  |r|^2 = sum (diag u)^2,  u.w,  u.s,  p.w,  p.s
//     b_{i+1} = g_{i+1} / g_i,
//     a_{i+1} = g_{i+1} / (p_{i+1}.A p_{i+1})  with  p_{i+1}.s_{i+1} = u.w + b (u.s + p.w) + b^2 p.s
// (the expansion of p.Ap gives the step length from the stored vectors instead of the
// orthogonality relations of the original recurrence for a).  D^-1 s and D^-1 w are stored,
// so that u_{i+1} at a neighbour needs no diagonal there; the diagonal comes from the band.
// (The pipelined variant of Ghysels and Vanroose, whose SpMV input is complete before the
// iteration, was measured too: its auxiliary recurrences drift too far in FP32 for the FP64
// refinement, which then stalls.)
//
// Per row the vector state is one float4 {u, D^-1 w, D^-1 s_prev, p_prev}, double-buffered
// by the parity counter s->pk: every tile reads the previous state in the windows its stencil
// spans (one window per stencil plane when its rows overlap, i.e. x-lines shorter than about
// a tile, else one per stencil column), bulk-copied into shared memory with the tile's band
// block by a producer warp (one bulk copy each, the band with an L2 evict-first policy), and
// writes its own rows' new state.  All waits are bounded.  A
// consumer thread forms u_{i+1} once per stencil column, at its own dx = 0 position, and takes
// the dx = -1 / +1 values from the neighbouring lanes (warp shuffles; lanes 0 and 31 form their
// outer neighbour themselves): 9 state loads per row instead of 27.  Per row the kernel moves
// the 108 band bytes, 16 bytes of state in and out and the correction d (8 bytes): 148 B, in
// one launch with one reduction.
//
// mode 0: iteration.  mode 1/2: start of a segment (fresh / continuing direction): u was just
// seeded from the FP64 residual; both A u and A p_prev are formed from the windows (no
// recurrence), d is not touched, and the reduction sets the first a, b (b = 0 when fresh;
// when continuing, b divides by r.u of the residual the kept direction came from).
constexpr int kMaxWin = 9;

struct CgArgs {
    int bpos[27];          // shared-memory float4 index of band b's neighbour for consumer row 0
    int off[27];           // column offset of band b
    int woff[kMaxWin];     // row offset of window w's first row relative to the tile's first row
    int nwin, wlen;        // windows per tile and rows per window
    int64_t n;
    int64_t lo, hi;        // a tile is interior when i0 + lo >= 0 and i0 + hi <= n
    // element-coefficient operator (RG_LAYOUT_COEF): khat windows and the Q1 table
    int kwoff[4];          // khat window offsets (multiples of 4: 16-byte aligned starts)
    int nkw, kwlen;        // khat windows per tile and floats per window (a multiple of 4)
    int kpos[8];           // shared-memory float index of corner element j = a + 2b + 4c for row 0
    int kdelta[8];         // khat offset of corner element j: a + NN0 b + NN0 NN1 c
    float T[8];            // Q1 stiffness entry for nodes differing in x (bit 0), y (1), z (2)
};

// u_{i+1} at a neighbour from its state: u - a (D^-1 w + b D^-1 s_prev)
__device__ __forceinline__ float next_u(float4 v, float alpha, float beta)
{
    return fmaf(-alpha, fmaf(beta, v.z, v.y), v.x);
}

// A row of the element-coefficient operator from the kappa of the 2^dim elements around the
// node, kv[a + 2b + 4c] for the element whose upper corner is the node + (a, b, c).  The
// neighbour at offset o lies in element (a, b, c) when o_x is a - 1 or a (likewise y, z), so its
// coefficient is T[|o|] times the sum of kappa over the elements with a in A(o_x), b in A(o_y),
// c in A(o_z), where A(-1) = {0}, A(1) = {1}, A(0) = {0, 1}.  CoefRow keeps the sums over a
// (sx[o_x + 1][b][c]); coef_at adds the y and z sums and the table entry for band b =
// (o_x+1) + 3 (o_y+1) + 9 (o_z+1).
struct CoefRow {
    float sx[3][2][2];
};

template <int NB>
__device__ __forceinline__ void coef_row(const float (&kv)[8], CoefRow& r)
{
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < (NB == 27 ? 2 : 1); ++c) {
            const float k0 = kv[0 + 2 * b + 4 * c], k1 = kv[1 + 2 * b + 4 * c];
            r.sx[0][b][c] = k0;
            r.sx[1][b][c] = k0 + k1;
            r.sx[2][b][c] = k1;
        }
}

// the sum of kappa over the elements shared by the node and its neighbour of band b
template <int NB>
__device__ __forceinline__ float ksum_at(const CoefRow& r, int b)
{
    const int x = b % 3, y = (b / 3) % 3, z = b / 9;
    auto ysum = [&](int c) {
        return y == 0 ? r.sx[x][0][c] : (y == 2 ? r.sx[x][1][c] : r.sx[x][0][c] + r.sx[x][1][c]);
    };
    if (NB == 27) return z == 0 ? ysum(0) : (z == 2 ? ysum(1) : ysum(0) + ysum(1));
    return ysum(0);
}

// the Q1 table class of band b: which coordinates differ (bit 0 x, 1 y, 2 z)
__host__ __device__ constexpr int band_class(int b) { return (b % 3 != 1) + 2 * ((b / 3) % 3 != 1) + 4 * (b / 9 != 1); }

template <int NB>
__device__ __forceinline__ float coef_at(const CoefRow& r, const float (&T)[8], int b)
{
    return T[NB == 27 ? band_class(b) : (band_class(b) & 3)] * ksum_at<NB>(r, b);
}

// The scalars of the next FP32 iteration from the six sums of one (the grid reduction's result,
// thread 0 of the last CTA): a, b, r.u and the stopping test.
__device__ void cg_scalars(Scal* s, const double* tt, int mode)
{
    // s->rho holds r.u of the current u, s->tau that of the u the kept direction was
    // formed from: a continuing segment start replaces the current u, so its b divides
    // by the older one
    const double g = tt[0];
    const double beta_n = mode == 1 ? 0.0 : g / (mode == 2 ? s->tau : s->rho);
    const double pap = tt[2] + beta_n * (tt[3] + tt[4]) + beta_n * beta_n * tt[5];
    s->beta = beta_n;
    s->alpha = g / pap;
    if (mode == 0) s->tau = s->rho;
    s->rho = g;
    s->pk += 1;
    const double norm = sqrt(tt[1]);
    s->norm = norm;
    if (mode == 0) {
        const long long it = s->iter + 1;
        s->iter = it;
        // the FP32 recurrence has stagnated when no new minimum (5% below the best)
        // appeared for 200 iterations: end the segment so that the FP64 residual is
        // recomputed and fed back
        if (norm < 0.95 * s->best) {
            s->best = norm;
            s->since = 0;
        } else {
            s->since += 1;
        }
        if (norm <= s->tol || s->since > 200) {
            report_status(s, ST_CONV);
        } else if (it >= s->maxit) {
            report_status(s, ST_MAXIT);
        } else if (!(g > 0.0) || !(pap > 0.0)) {
            report_status(s, ST_BREAK);
        }
    } else if (!(g > 0.0) || !(pap > 0.0)) {
        atomicMax(&s->status, (int)ST_BREAK);  // read by the host after the start pass
    }
}

// Fused FP32 PCG iteration, two operators:
//   COEF = false: the tile's band block (FP32 copy of the balanced matrix) is bulk-copied with
//                 the state windows; the diagonal is its centre band.
//   COEF = true:  the operator is evaluated from the element coefficients (unbalanced A; the
//                 Jacobi-preconditioned iteration is the same for any symmetric diagonal scaling
//                 of the matrix, so the balancing is applied only where the FP64 refinement
//                 hands residuals and corrections over): windows of khat replace the band
//                 block (4 instead of 108 bytes per row).  Rows of nodes fixed by the constraint
//                 are identity rows, solved exactly by the seed; their state stays zero, so
//                 their columns drop out of every other row without a mask.
template <int NB, int kStages, int kCtas, bool COEF>
__global__ void __launch_bounds__(kTile + 32, kCtas) k_f32_cg(const float* __restrict__ band,
                                                              const __grid_constant__ CgArgs ca,
                                                              const float4* V0, const float4* V1,
                                                              float4* W0, float4* W1,
                                                              float* __restrict__ d, ReduceBuf rb, Scal* s, int mode)
{
    constexpr int kCenter = NB / 2;
    constexpr int NG = NB / 3;
    constexpr int NK = NB == 27 ? 8 : 4;  // elements around a node
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
    __shared__ int bad;
    if (mode == 0 && s->done) return;
    const float alpha = mode == 0 ? (float)s->alpha : 0.f;
    const float beta = mode == 0 ? (float)s->beta : 0.f;
    const bool odd = (s->pk & 1) != 0;
    const float4* __restrict__ vin = odd ? V1 : V0;   // state of this iteration
    float4* __restrict__ vout = odd ? W0 : W1;        // state of the next one
    const int t = threadIdx.x;
    const int lane = t & 31;
    const int warp = t >> 5;
    const int eoff = lane == 0 ? -1 : (lane == 31 ? 1 : 0);  // the outer x-neighbour of warp edge lanes
    const int64_t n = ca.n;
    const int64_t ntiles = (n + kTile - 1) / kTile;
    const int64_t my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    // tile k of this CTA; on the band operator odd iterations walk the tiles backwards, so that
    // the state rows the previous launch wrote last, the likeliest to be still in L2, are read
    // first (measured at 128^3: 58.4 -> 55.4 us per launch; the coefficient operator, whose
    // launch is not bound by memory, gained nothing and spilled registers with it)
    const bool back = !COEF && odd;
    const int64_t tbase = back ? ntiles - 1 - blockIdx.x : (int64_t)blockIdx.x;
    const int64_t tstep = back ? -(int64_t)gridDim.x : (int64_t)gridDim.x;
    auto tile_of = [&](int64_t k) { return tbase + k * tstep; };
    const int kmat = COEF ? ca.nkw * ca.kwlen : NB * kTile;  // floats of the operator's part of a stage
    const int stage_floats = kmat + 4 * ca.nwin * ca.wlen;
    if (t == 0) {
        for (int k = 0; k < kStages; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], kConsumerWarps);
        }
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto interior = [&](int64_t i0) { return i0 + ca.lo >= 0 && i0 + ca.hi <= n; };

    // sums: g = r.u, |r|^2, u.w, u.s, p.w, p.s (u, w of the next iteration; p, s of this one)
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int64_t issued = 0;
    const WaitCtl wc = g_wait_ctl;
    const int polls = wc.polls > 0 ? wc.polls : kDefaultPolls;
    if (warp == kConsumerWarps) {
        // ---------------- producer: operator data and state windows of each tile
        if (lane == 0 && !wc.withhold) {
            const uint64_t pol = evict_first_policy();
            const uint32_t wbytes = (uint32_t)ca.wlen * 16u;
            for (int64_t k = 0; k < my_tiles; ++k, issued = k) {
                const int st = (int)(k % kStages);
                if (k >= kStages && !mbar_wait(&empty[st], (uint32_t)(((k / kStages) - 1) & 1), polls)) {
                    bad = 1;
                    break;
                }
                const int64_t tile = tile_of(k);
                const int64_t i0 = tile * kTile;
                float* dst = smem + (size_t)st * stage_floats;
                const bool in = interior(i0);
                mbar_expect_tx(&full[st], (uint32_t)kmat * 4u + (in ? (uint32_t)ca.nwin * wbytes : 0u));
                if (COEF) {
                    // khat is padded: every tile's windows are in range
                    for (int w = 0; w < ca.nkw; ++w)
                        bulk_g2s(dst + w * ca.kwlen, band + (i0 + ca.kwoff[w]), (uint32_t)ca.kwlen * 4u, &full[st]);
                } else {
                    bulk_g2s_hint(dst, band + (size_t)tile * NB * kTile, NB * kTile * 4, &full[st], pol);
                }
                if (in)
                    for (int w = 0; w < ca.nwin; ++w)
                        bulk_g2s(dst + kmat + 4 * w * ca.wlen, vin + (i0 + ca.woff[w]), wbytes, &full[st]);
            }
        }
    } else {
        // ---------------- consumers: row i0 + t of every tile
        for (int k = 0; k < (int)my_tiles; ++k) {  // (32-bit tile count: cheaper stage arithmetic)
            const int st = k % kStages;
            const int64_t i0 = tile_of(k) * (int64_t)kTile;
            const int64_t i = i0 + t;
            // the correction is only read and written by this row: load it while the stage fills
            const float dold = (mode == 0 && i < n) ? __ldcs(d + i) : 0.f;
            if (!mbar_wait(&full[st], (uint32_t)((k / kStages) & 1), polls)) {
                bad = 1;
                break;
            }
            const float* bs = smem + st * stage_floats;
            const float4* win = reinterpret_cast<const float4*>(bs + kmat);
            // this row's coefficients: formed from the element values (COEF), or read from the
            // band block where they are used
            CoefRow cr;
            bool fixed = false;
            if constexpr (COEF) {
                float kv[8];
#pragma unroll
                for (int j = 0; j < NK; ++j) kv[j] = bs[ca.kpos[j] + t];
                fixed = (__float_as_uint(kv[0]) >> 31) != 0;
#pragma unroll
                for (int j = 0; j < NK; ++j) kv[j] = fabsf(kv[j]);
#pragma unroll
                for (int j = NK; j < 8; ++j) kv[j] = 0.f;
                coef_row<NB>(kv, cr);
            }
            auto coefb = [&](int b) -> float {
                if constexpr (COEF)
                    return coef_at<NB>(cr, ca.T, b);
                else
                    return bs[b * kTile + t];
            };
            float acc_u = 0.f, acc_p = 0.f;
            float4 c = make_float4(0.f, 0.f, 0.f, 0.f);  // this row's state
            if (interior(i0) && mode == 0) {
                // (a row's products are summed in band order: summing them per Q1 table class
                // and scaling once was measured to cost ~7% more iterations at 128^3, from the
                // FP32 cancellation of a Laplacian row's nearly zero sum)
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    // u_{i+1} at this lane's dx = 0 neighbour of stencil column g; dx = -1 / +1
                    // from the lanes beside it; lanes 0 / 31 form that outer value themselves
                    const int pc = ca.bpos[3 * g + 1] + t;
                    const float4 vc = win[pc];
                    const float uc = next_u(vc, alpha, beta);
                    float ue = 0.f;
                    if (lane == 0 || lane == 31) ue = next_u(win[pc + eoff], alpha, beta);
                    const float up = __shfl_up_sync(0xffffffffu, uc, 1);
                    const float dn = __shfl_down_sync(0xffffffffu, uc, 1);
                    const float ul = lane == 0 ? ue : up;
                    const float ur = lane == 31 ? ue : dn;
                    acc_u = fmaf(coefb(3 * g), ul, acc_u);
                    acc_u = fmaf(coefb(3 * g + 1), uc, acc_u);
                    acc_u = fmaf(coefb(3 * g + 2), ur, acc_u);
                    if (3 * g + 1 == kCenter) c = vc;
                }
            } else {
                const bool in = interior(i0);
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    float4 nb;
                    if (in) {
                        nb = win[ca.bpos[b] + t];
                    } else {
                        const int64_t j = min(max(i + ca.off[b], (int64_t)0), n - 1);
                        nb = __ldg(vin + j);
                    }
                    if (mode == 0) {
                        acc_u = fmaf(coefb(b), next_u(nb, alpha, beta), acc_u);
                    } else {
                        acc_u = fmaf(coefb(b), nb.x, acc_u);
                        acc_p = fmaf(coefb(b), nb.w, acc_p);
                    }
                    if (b == kCenter) c = nb;
                }
            }
            float diag = coefb(kCenter);
            if (COEF && fixed) {  // identity row: solved by the seed, state stays zero
                acc_u = 0.f;
                acc_p = 0.f;
                diag = 1.f;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            if (i < n) {
                float un, spn, pn;
                if (mode == 0) {
                    pn = fmaf(beta, c.w, c.x);      // p_i = u_i + beta p_{i-1}
                    spn = fmaf(beta, c.z, c.y);     // D^-1 s_i = D^-1 w_i + beta D^-1 s_{i-1}
                    un = fmaf(-alpha, spn, c.x);    // u_{i+1}, as next_u forms it
                    d[i] = fmaf(alpha, pn, dold);   // d += alpha p_i
                } else {
                    pn = c.w;                       // the kept direction (0 when fresh)
                    spn = __fdividef(acc_p, diag);  // D^-1 A p, formed afresh
                    un = c.x;
                }
                const float w = acc_u;              // (A u_{i+1})_i
                vout[i] = make_float4(un, __fdividef(w, diag), spn, pn);
                const double du = un, dd = diag, ds = (double)spn * dd;
                v[0] += dd * du * du;
                // the segment's stopping norm: |r| of the balanced residual (band copy); for the
                // unbalanced coefficient operator r.u = r.D^-1 r (= v[0], copied after the
                // reduction), which paso's balancing leaves unchanged and which is |B r|^2 when
                // the balance vector is D^-1/2 (diagonally dominant rows)
                if (!COEF) v[1] += (dd * du) * (dd * du);
                v[2] += du * (double)w;
                v[3] += du * ds;
                v[4] += (double)pn * (double)w;
                v[5] += (double)pn * ds;
            }
        }
    }
    __syncthreads();
    if (bad) {
        // let the copies this CTA issued land (bounded) before its shared memory is released
        if (warp == kConsumerWarps && lane == 0)
            for (int64_t k = issued > kStages ? issued - kStages : 0; k < issued; ++k)
                for (int tries = 0; tries < (1 << 20) && !mbar_try_wait(&full[k % kStages], (uint32_t)((k / kStages) & 1));
                     ++tries) {
                }
        if (t == 0) report_status(s, ST_TIMEOUT);
        // the CTA still takes its turn in the grid reduction (with nothing to add)
#pragma unroll
        for (int j = 0; j < 6; ++j) v[j] = 0.0;
    }
    double tt[6];
    if (grid_reduce<6>(v, rb, tt) && threadIdx.x == 0) {
        if (COEF) tt[1] = tt[0];
        cg_scalars(s, tt, mode);
    }
}

// The element-coefficient operator's seed: the balanced FP64 residual is unbalanced (r =
// r64 / bv, scaled by inv_scale); fixed nodes get their exact correction d = r (identity
// rows) and a zero state; free rows u = r / diag (z, p, d = 0 when fresh).
template <int NB>
__global__ void __launch_bounds__(kThreads) k_f32_cg_seed_coef(const __grid_constant__ CgArgs ca,
                                                               const double* __restrict__ r64,
                                                               const double* __restrict__ bv,
                                                               const float* __restrict__ khat, float4* V0,
                                                               float4* V1,
                                                               float* __restrict__ d, int fresh, const Scal* s,
                                                               double inv_scale)
{
    constexpr int NK = NB == 27 ? 8 : 4;
    float4* __restrict__ v = (s->pk & 1) ? V1 : V0;
    const int64_t n = ca.n;
    for (int64_t i = gtid(); i < n; i += gstride()) {
        float kv[8];
#pragma unroll
        for (int j = 0; j < NK; ++j) kv[j] = khat[i + ca.kdelta[j]];
        const bool fixed = (__float_as_uint(kv[0]) >> 31) != 0;
#pragma unroll
        for (int j = 0; j < NK; ++j) kv[j] = fabsf(kv[j]);
#pragma unroll
        for (int j = NK; j < 8; ++j) kv[j] = 0.f;
        CoefRow cr;
        coef_row<NB>(kv, cr);
        const float r = (float)(r64[i] / bv[i] * inv_scale);
        float4 c = v[i];
        if (fixed) {
            c = make_float4(0.f, 0.f, 0.f, 0.f);
            d[i] = r;
        } else {
            c.x = r / coef_at<NB>(cr, ca.T, NB / 2);
            if (fresh) {
                c.y = 0.f;
                c.z = 0.f;
                c.w = 0.f;
                d[i] = 0.f;
            }
        }
        v[i] = c;
    }
}

// zb_i = bv_i x_i, 0 on the nodes the constraint fixes (the sign bit of khat): the vector
// k_cheb_step_coef gathers
__global__ void k_mask_scale(int64_t n, const float* __restrict__ khat, const double* __restrict__ bv,
                             const double* __restrict__ x, double* __restrict__ zb)
{
    for (int64_t i = gtid(); i < n; i += gstride())
        zb[i] = (__float_as_uint(khat[i]) >> 31) ? 0.0 : bv[i] * x[i];
}

// k_cheb_step on the element-coefficient operator (when the FP32 solve evaluates its operator
// from the coefficients there is no band copy): the balanced operator is bv_i sum_j a_ij bv_j
// x_j with a_ij from kappa (FP32 coefficients, FP64 vectors); rows and columns of fixed nodes
// (the sign bit of khat) are those of the identity.  The neighbours' bv_j x_j come masked in
// zx (k_mask_scale, then each step's zy for the next): one gathered load per neighbour.
template <int NB>
__global__ void __launch_bounds__(kThreads) k_cheb_step_coef(const __grid_constant__ CgArgs ca,
                                                             const float* __restrict__ khat,
                                                             const double* __restrict__ bv,
                                                             const double* __restrict__ dinv,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ zx,
                                                             const double* __restrict__ bb, double c_d, double c_r,
                                                             double* __restrict__ d, double* __restrict__ y,
                                                             double* __restrict__ zy)
{
    constexpr int NK = NB == 27 ? 8 : 4;
    const int64_t n = ca.n;
    for (int64_t i = gtid(); i < n; i += gstride()) {
        float kv[8];
#pragma unroll
        for (int j = 0; j < NK; ++j) kv[j] = __ldg(khat + i + ca.kdelta[j]);
        const bool fixed = (__float_as_uint(kv[0]) >> 31) != 0;
#pragma unroll
        for (int j = 0; j < NK; ++j) kv[j] = fabsf(kv[j]);
#pragma unroll
        for (int j = NK; j < 8; ++j) kv[j] = 0.f;
        CoefRow cr;
        coef_row<NB>(kv, cr);
        double acc;
        if (fixed) {
            acc = x[i];
        } else {
            acc = 0.0;
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const float c = coef_at<NB>(cr, ca.T, b);
                const int64_t j = min(max(i + ca.off[b], (int64_t)0), n - 1);
                if (c != 0.f) acc = fma((double)c, __ldg(zx + j), acc);
            }
            acc *= bv[i];
        }
        const double dn = c_d * (c_d != 0.0 ? d[i] : 0.0) + c_r * dinv[i] * (bb[i] - acc);
        d[i] = dn;
        const double yi = x[i] + dn;
        y[i] = yi;
        zy[i] = fixed ? 0.0 : bv[i] * yi;
    }
}

// x64 += scale * d32 / bv (the element-coefficient operator's correction is unbalanced); d32 = 0
__global__ void k_fold_correction_unbalance(int64_t n, double* __restrict__ x, float* __restrict__ d,
                                            const double* __restrict__ bv, double scale)
{
    for (int64_t i = gtid(); i < n; i += gstride()) {
        x[i] += scale * (double)d[i] / bv[i];
        d[i] = 0.f;
    }
}

// u = D^-1 (r64 / scale) into the current state (p_prev = 0 and d = 0 when fresh): the start
// of a segment of k_f32_cg
__global__ void __launch_bounds__(kThreads) k_f32_cg_seed(int64_t n, const double* __restrict__ r64,
                                                          const float* __restrict__ dinv32, float4* V0, float4* V1,
                                                          float* __restrict__ d, int fresh, const Scal* s,
                                                          double inv_scale)
{
    float4* __restrict__ v = (s->pk & 1) ? V1 : V0;
    for (int64_t i = gtid(); i < n; i += gstride()) {
        float4 c = v[i];
        c.x = (float)(r64[i] * inv_scale) * dinv32[i];
        if (fresh) {
            c.y = 0.f;
            c.z = 0.f;
            c.w = 0.f;
            d[i] = 0.f;
        }
        v[i] = c;
    }
}

// x64 += scale * d32; d32 = 0
__global__ void k_fold_correction(int64_t n, double* __restrict__ x, float* __restrict__ d, double scale)
{
    for (int64_t i = gtid(); i < n; i += gstride()) {
        x[i] += scale * (double)d[i];
        d[i] = 0.f;
    }
}

// ------------------------------------------------------------------ host helpers
double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int read_scal(Workspace* w)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(w->hs, w->s, sizeof(Scal), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    return RG_OK;
}

// set device scalars from the host (stream-ordered)
int write_scal_fields(Workspace* w, double tol, long long maxit, long long iter0)
{
    Scal h = *w->hs;
    h.tol = tol;
    h.maxit = maxit;
    h.iter = iter0;
    h.best = h.norm;
    h.since = 0;
    h.done = 0;
    h.status = ST_RUN;
    *w->hs = h;
    RG_CHECK_CUDA(cudaMemcpyAsync(w->s, w->hs, sizeof(Scal), cudaMemcpyHostToDevice, stream()));
    return RG_OK;
}

ReduceBuf rbuf(Workspace* w) { return ReduceBuf{w->partials, w->counter}; }

// iterations per host poll: about 1 ms of device work, at least 4
int chunk_for(int64_t n, int64_t bytes_per_row)
{
    const double iter_s = (double)n * bytes_per_row / 5.0e12 + 8e-6;
    int c = (int)(1e-3 / iter_s);
    return c < 4 ? 4 : (c > 256 ? 256 : c);
}

using IterFn = int (*)(Matrix*);

bool graphs_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("RG_GRAPHS");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1 && !timers_on();
}

// runs PCG iterations until the device flags done.  Chunks of `chunk` iterations are
// captured once per (matrix, kind) as a CUDA graph and replayed; the done flag of chunk
// k is read while chunk k+1 is already queued, so the device never waits for the host.
// Kernels of a chunk that follow convergence return at once.  With kernel timers on the
// steps are launched directly (events cannot be timed inside a replayed graph).
int run_until_done(Matrix* m, int kind, IterFn step, int chunk, long long cap, long long* iters,
                   int* status)
{
    Workspace* w = m->ws;
    long long launched = 0;
    if (!graphs_enabled()) {
        for (;;) {
            for (int c = 0; c < chunk; ++c) {
                int rc = step(m);
                if (rc) return rc;
            }
            launched += chunk;
            int rc = read_scal(w);
            if (rc) return rc;
            if (w->hs->done) break;
            if (launched > cap + 2 * chunk + 8) {
                set_error("PCG iteration loop did not terminate");
                return RG_TIMEOUT;
            }
        }
        *iters = w->hs->iter;
        *status = w->hs->status;
        return RG_OK;
    }
    if (!w->graph[kind] || w->graph_chunk[kind] != chunk || w->graph_sweeps[kind] != w->sweeps ||
        w->graph_band64[kind] != w->band64 || w->graph_coef[kind] != w->coef_op) {
        if (w->graph[kind]) cudaGraphExecDestroy(w->graph[kind]);
        w->graph[kind] = nullptr;
        long long before[T_COUNT], after[T_COUNT];
        timers_snapshot(before);
        RG_CHECK_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
        int rc = RG_OK;
        for (int c = 0; c < chunk && rc == RG_OK; ++c) rc = step(m);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream(), &g);
        if (rc) return rc;
        if (e != cudaSuccess) {
            set_error(std::string("graph capture: ") + cudaGetErrorString(e));
            return RG_CUDA_ERROR;
        }
        e = cudaGraphInstantiate(&w->graph[kind], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
            return RG_CUDA_ERROR;
        }
        w->graph_chunk[kind] = chunk;
        w->graph_sweeps[kind] = w->sweeps;
        w->graph_band64[kind] = w->band64;
        w->graph_coef[kind] = w->coef_op;
        timers_snapshot(after);
        long long undo[T_COUNT];
        for (int k = 0; k < T_COUNT; ++k) {
            w->graph_launches[kind][k] = after[k] - before[k];
            undo[k] = before[k] - after[k];
        }
        timers_add(undo, 1);  // captured launches are counted when replayed
    }
    int k = 0;
    const Scal* last = nullptr;
    for (;;) {
        RG_CHECK_CUDA(cudaGraphLaunch(w->graph[kind], stream()));
        timers_add(w->graph_launches[kind], 1);
        RG_CHECK_CUDA(cudaMemcpyAsync(&w->hpoll[k & 1], w->s, sizeof(Scal), cudaMemcpyDeviceToHost, stream()));
        RG_CHECK_CUDA(cudaEventRecord(w->poll_ev[k & 1], stream()));
        launched += chunk;
        if (k >= 1) {
            RG_CHECK_CUDA(cudaEventSynchronize(w->poll_ev[(k - 1) & 1]));
            if (w->hpoll[(k - 1) & 1].done) {
                last = &w->hpoll[k & 1];
                break;
            }
        }
        if (launched > cap + 3 * chunk + 8) {
            RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
            set_error("PCG iteration loop did not terminate");
            return RG_TIMEOUT;
        }
        ++k;
    }
    RG_CHECK_CUDA(cudaEventSynchronize(w->poll_ev[k & 1]));
    *w->hs = *last;
    *iters = last->iter;
    *status = last->status;
    return RG_OK;
}

// sweeps - 1 more Jacobi sweeps on the preconditioned vector z (of b), alternating between
// z and `spare`; returns the buffer that holds the result.  mode of the last sweep as in
// k_jacobi_sweep.
TmaBandArgs band_offsets(const Domain* d)
{
    TmaBandArgs ta{};
    for (int b = 0; b < d->nbands; ++b) {
        ta.off[b] = (int)d->band_off[b];
        ta.halo = std::max<int64_t>(ta.halo, std::abs(d->band_off[b]));
    }
    for (int g = 0; g < d->nbands / 3; ++g) ta.goff[g] = (int)d->band_off[3 * g];  // dx = -1 member
    ta.n = d->n;
    return ta;
}

int sm_count();

// FP64 band kernel (SpMV or Jacobi sweep) over all tiles, one CTA per SM.  The vector x that
// is bulk-copied is always a solver workspace array (cudaMalloc: 256-byte aligned).  Launch
// errors are picked up by the caller's RG_CHECK_LAUNCH.
template <bool SWEEP>
void launch_band64(Matrix* m, const double* x, double* out, const double* b, double* pout, int mode)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    const TmaBandArgs ta = band_offsets(d);
    const int64_t ntiles = (d->n + kTile - 1) / kTile;
    const int grid = (int)std::min<int64_t>(ntiles, sm_count());
    const int kind = SWEEP ? T_PASO_UPDATE1 : (mode == 1 ? T_STD_SPMV : T_PASO_SPMV);
    if (d->nbands == 27) {
        constexpr int S = band64_stages<27>();
        RG_TIMED(kind, (k_band64_bulk<27, S, SWEEP><<<grid, kTile + 32, band64_smem<27, S>(), stream()>>>(
                           m->band64, ta, x, out, m->dinv, b, pout, rbuf(w), w->s, mode)));
    } else {
        constexpr int S = band64_stages<9>();
        RG_TIMED(kind, (k_band64_bulk<9, S, SWEEP><<<grid, kTile + 32, band64_smem<9, S>(), stream()>>>(
                           m->band64, ta, x, out, m->dinv, b, pout, rbuf(w), w->s, mode)));
    }
}

double* jacobi_sweeps(Matrix* m, const double* b, double* z, double* spare, double* p, int last_mode)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    double* src = z;
    double* dst = spare;
    const bool band = w->band64 && m->band64;
    for (int k = 1; k < w->sweeps; ++k) {
        const int mode = k == w->sweeps - 1 ? last_mode : 0;
        if (band)
            launch_band64<true>(m, src, dst, b, p, mode);
        else
            RG_TIMED(T_PASO_UPDATE1, (k_jacobi_sweep<<<w->grid_rows, kThreads, 0, stream()>>>(
                                         d->n, d->ptr, d->idx, m->val, m->dinv, b, src, dst, p, rbuf(w), w->s, mode)));
        std::swap(src, dst);
    }
    return src;
}

int paso_step(Matrix* m)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    if (w->band64 && m->band64) {
        launch_band64<false>(m, w->p, w->q, nullptr, nullptr, 0);
    } else {
        RG_TIMED(T_PASO_SPMV, (k_paso_spmv<<<w->grid_rows, kThreads, 0, stream()>>>(
                                  d->n, d->ptr, d->idx, m->val, w->p, w->q, rbuf(w), w->s)));
    }
    RG_TIMED(T_PASO_UPDATE1, (k_paso_update1<<<w->grid_vec, kThreads, 0, stream()>>>(
                                 d->n, w->r, w->q, w->rs, w->x2, w->p, m->dinv, w->z, rbuf(w), w->s)));
    // v = prec(r) with more than one Jacobi sweep: q (free after update1) is the spare buffer
    const double* v = jacobi_sweeps(m, w->r, w->z, w->q, nullptr, 1);
    RG_TIMED(T_PASO_UPDATE2, (k_paso_update2<<<w->grid_vec, kThreads, 0, stream()>>>(
                                 d->n, w->rs, w->r, w->x, w->x2, v, w->p, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int std_step(Matrix* m)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    if (w->band64 && m->band64)
        launch_band64<false>(m, w->p, w->q, nullptr, nullptr, 1);
    else
        RG_TIMED(T_STD_SPMV, (k_std_spmv<<<w->grid_rows, kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val,
                                                                                  w->p, w->q, rbuf(w), w->s)));
    RG_TIMED(T_STD_UPDATE, (k_std_update<<<w->grid_vec, kThreads, 0, stream()>>>(d->n, w->x, w->r, w->q, w->p,
                                                                                 m->dinv, w->z, rbuf(w), w->s)));
    RG_TIMED(T_VECTOR, (k_std_pupdate<<<w->grid_vec, kThreads, 0, stream()>>>(d->n, w->z, w->p, w->s)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int sm_count()
{
    static int count = 0;
    if (!count) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = kNumSMs;
    }
    return count;
}

// configurations of the FP32 iteration pipeline: (stages, CTAs per SM), for the band operator
// and for the element-coefficient operator (whose stages are a quarter of the size)
constexpr int kSpmvCfg[2][2] = {{3, 1}, {2, 2}};
constexpr int kCoefCfg[2][2] = {{3, 2}, {2, 2}};

// Window geometry of k_f32_cg for a domain: one window per stencil plane (dz) covering the
// rows [i0 - NN0 - 1, i0 + kTile + NN0 + 1) when that is shorter than three windows of
// kTile + 2 rows (x-lines shorter than about a tile), else one window per stencil column
// (dy, dz) of kTile + 2 rows; bpos[b] locates band b's neighbour of consumer row 0 in shared
// memory (float4 elements).
CgArgs cg_args(const Domain* d)
{
    CgArgs ca{};
    const int64_t nn0 = d->nn[0], nn01 = d->nn[0] * d->nn[1];
    const bool three = d->dim == 3;
    const bool merged = 2 * nn0 + kTile + 2 <= 3 * (kTile + 2);
    const int planes = three ? 3 : 1;
    int64_t nominal[kMaxWin];
    int64_t len;
    if (merged) {
        ca.nwin = planes;
        len = kTile + 2 * nn0 + 2;
        for (int z = 0; z < planes; ++z) nominal[z] = (three ? (z - 1) * nn01 : 0) - nn0 - 1;
    } else {
        ca.nwin = 3 * planes;
        len = kTile + 2;
        for (int z = 0; z < planes; ++z)
            for (int y = 0; y < 3; ++y) nominal[3 * z + y] = (three ? (z - 1) * nn01 : 0) + (y - 1) * nn0 - 1;
    }
    ca.wlen = (int)len;  // the state is 16 bytes per row: every window start is 16-byte aligned
    int64_t lo = 0, hi = 0;
    for (int w = 0; w < ca.nwin; ++w) {
        ca.woff[w] = (int)nominal[w];
        lo = std::min<int64_t>(lo, nominal[w]);
        hi = std::max<int64_t>(hi, nominal[w] + ca.wlen);
    }
    ca.lo = lo;
    ca.hi = hi;
    for (int b = 0; b < d->nbands; ++b) {
        const int dy = (b / 3) % 3, dz = three ? b / 9 : 0;  // 0..2
        const int w = merged ? dz : 3 * dz + dy;
        ca.off[b] = (int)d->band_off[b];
        ca.bpos[b] = w * ca.wlen + (int)(d->band_off[b] - ca.woff[w]);
    }
    ca.n = d->n;
    // element-coefficient operator: khat windows hold the elements around the tile's rows,
    // corner j = a + 2b + 4c at node offset a + NN0 b + NN0 NN1 c (all >= 0): one window per
    // element plane (c) when NN0 is short, else one per (b, c); starts rounded down to 4 floats
    const int nk = three ? 8 : 4;
    const bool kmerged = nn0 + kTile + 1 <= 2 * (kTile + 1);
    int64_t knom[4];
    int64_t klen;
    if (kmerged) {
        ca.nkw = three ? 2 : 1;
        klen = kTile + nn0 + 1;
        for (int c = 0; c < ca.nkw; ++c) knom[c] = c * nn01;
    } else {
        ca.nkw = three ? 4 : 2;
        klen = kTile + 1;
        for (int w = 0; w < ca.nkw; ++w) knom[w] = (w & 1) * nn0 + (w >> 1) * nn01;
    }
    ca.kwlen = (int)((klen + 3 + 3) & ~(int64_t)3);
    for (int w = 0; w < ca.nkw; ++w) ca.kwoff[w] = (int)(knom[w] - (knom[w] & 3));
    for (int j = 0; j < 8; ++j) {
        const int a = j & 1, b = (j >> 1) & 1, c = j >> 2;
        const int64_t delta = j < nk ? a + nn0 * b + nn01 * c : 0;
        ca.kdelta[j] = (int)delta;
        const int w = j < nk ? (kmerged ? c : b + 2 * c) : 0;
        ca.kpos[j] = w * ca.kwlen + (int)(delta - ca.kwoff[w]);
    }
    // Q1 stiffness of the reference box (exact 1D integrals; the 2-point Gauss rule of the
    // assembly is exact for them): per axis K = 1/h (same node) or -1/h, M = h/3 or h/6
    for (int cls = 0; cls < 8; ++cls) {
        double k1[3], m1[3];
        for (int ax = 0; ax < 3; ++ax) {
            const bool diff = (cls >> ax) & 1;
            const double h = d->dx[ax];
            k1[ax] = (diff ? -1.0 : 1.0) / h;
            m1[ax] = diff ? h / 6.0 : h / 3.0;
        }
        const double t = three ? k1[0] * m1[1] * m1[2] + m1[0] * k1[1] * m1[2] + m1[0] * m1[1] * k1[2]
                               : k1[0] * m1[1] + m1[0] * k1[1];
        ca.T[cls] = (float)t;
    }
    return ca;
}

size_t cg_smem(const Domain* d, const CgArgs& ca, int stages, bool coef)
{
    const size_t mat = coef ? (size_t)ca.nkw * ca.kwlen : (size_t)d->nbands * kTile;
    return sizeof(float) * (size_t)stages * (mat + 4 * (size_t)ca.nwin * ca.wlen);
}

// largest dynamic shared memory a launch of `kernel` may ask for: the device's opt-in limit
// per CTA less the kernel's static shared memory
int max_dyn_smem(const void* kernel, int* out)
{
    int dev = 0, optin = 0;
    RG_CHECK_CUDA(cudaGetDevice(&dev));
    RG_CHECK_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    RG_CHECK_CUDA(cudaFuncGetAttributes(&fa, kernel));
    *out = optin - (int)fa.sharedSizeBytes;
    return RG_OK;
}

template <int NB, int S, int CPS, bool COEF>
int cg_attribute()
{
    int lim = 0;
    int rc = max_dyn_smem((const void*)k_f32_cg<NB, S, CPS, COEF>, &lim);
    if (rc) return rc;
    RG_CHECK_CUDA(
        cudaFuncSetAttribute(k_f32_cg<NB, S, CPS, COEF>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    return RG_OK;
}

int tma_attributes()
{
    static bool done = false;
    if (!done) {
        int rc;
        if ((rc = cg_attribute<27, 3, 1, false>()) || (rc = cg_attribute<27, 2, 2, false>()) ||
            (rc = cg_attribute<9, 3, 1, false>()) || (rc = cg_attribute<9, 2, 2, false>()) ||
            (rc = cg_attribute<27, 3, 2, true>()) || (rc = cg_attribute<27, 2, 2, true>()) ||
            (rc = cg_attribute<9, 3, 2, true>()) || (rc = cg_attribute<9, 2, 2, true>()))
            return rc;
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_band64_bulk<27, band64_stages<27>(), false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)band64_smem<27, band64_stages<27>()>()));
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_band64_bulk<27, band64_stages<27>(), true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)band64_smem<27, band64_stages<27>()>()));
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_band64_bulk<9, band64_stages<9>(), false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)band64_smem<9, band64_stages<9>()>()));
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_band64_bulk<9, band64_stages<9>(), true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)band64_smem<9, band64_stages<9>()>()));
        done = true;
    }
    return RG_OK;
}

template <int NB, int S, int CPS, bool COEF>
const void* cg_kernel() { return (const void*)k_f32_cg<NB, S, CPS, COEF>; }

const void* cg_kernel_for(int nb, int cfg, bool coef)
{
    if (coef) {
        if (nb == 27) return cfg == 0 ? cg_kernel<27, 3, 2, true>() : cg_kernel<27, 2, 2, true>();
        return cfg == 0 ? cg_kernel<9, 3, 2, true>() : cg_kernel<9, 2, 2, true>();
    }
    if (nb == 27) return cfg == 0 ? cg_kernel<27, 3, 1, false>() : cg_kernel<27, 2, 2, false>();
    return cfg == 0 ? cg_kernel<9, 3, 1, false>() : cg_kernel<9, 2, 2, false>();
}

// (stages, CTAs per SM) of configuration cfg of an operator
const int* cg_cfg(int cfg, bool coef) { return coef ? kCoefCfg[cfg] : kSpmvCfg[cfg]; }

// whether configuration cfg reaches its CTAs per SM with this domain's windows
bool cg_config_fits(const Domain* d, int cfg, bool coef)
{
    const void* kern = cg_kernel_for(d->nbands, cfg, coef);
    const size_t smem = cg_smem(d, cg_args(d), cg_cfg(cfg, coef)[0], coef);
    int lim = 0;
    if (max_dyn_smem(kern, &lim) != RG_OK || smem > (size_t)lim) return false;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kTile + 32, smem) != cudaSuccess) return false;
    return blocks >= cg_cfg(cfg, coef)[1];
}

// one launch of the fused FP32 iteration (mode 0) or of a segment start (mode 1, 2) with the
// workspace's current operator (band copy, or element coefficients when w->coef_op)
template <int NB, int S, int CPS, bool COEF>
void launch_cg_k(Matrix* m, const CgArgs& ca, int grid, size_t smem, int mode)
{
    Workspace* w = m->ws;
    const float* op = COEF ? m->coef.khat : m->band32;
    RG_TIMED(T_F32_SPMV, (k_f32_cg<NB, S, CPS, COEF><<<grid, kTile + 32, smem, stream()>>>(
                             op, ca, w->v4[0], w->v4[1], w->v4[0], w->v4[1], w->d32, rbuf(w), w->s, mode)));
}

template <int NB>
int launch_cg(Matrix* m, int cfg, int mode)
{
    const Domain* d = m->dom;
    const bool coef = m->ws->coef_op;
    const CgArgs ca = cg_args(d);
    const int* sc = cg_cfg(cfg, coef);
    const int64_t ntiles = (d->n + kTile - 1) / kTile;
    const int grid = (int)std::min<int64_t>(ntiles, (int64_t)sm_count() * sc[1]);
    const size_t smem = cg_smem(d, ca, sc[0], coef);
    if (coef) {
        if (cfg == 0)
            launch_cg_k<NB, 3, 2, true>(m, ca, grid, smem, mode);
        else
            launch_cg_k<NB, 2, 2, true>(m, ca, grid, smem, mode);
    } else {
        if (cfg == 0)
            launch_cg_k<NB, 3, 1, false>(m, ca, grid, smem, mode);
        else
            launch_cg_k<NB, 2, 2, false>(m, ca, grid, smem, mode);
    }
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_spmv_cfg(Matrix* m, int cfg, int mode = 0)
{
    return m->dom->nbands == 27 ? launch_cg<27>(m, cfg, mode) : launch_cg<9>(m, cfg, mode);
}

// the tuned configuration of the workspace's current operator
int& cfg_slot(Workspace* w) { return w->coef_op ? w->coef_cfg : w->spmv_cfg; }

// a start state for the tuner's timed launches: u varies from row to row (A applied to a
// constant is ~0 on the rows of a Laplacian, which would end the iterations at once)
__global__ void k_fill_state(int64_t n, float4* __restrict__ v0, float4* __restrict__ v1, float* __restrict__ d)
{
    for (int64_t i = gtid(); i < n; i += gstride()) {
        const float u = 1.f + 0.5f * (float)((i * 2654435761ull >> 7) & 1023) / 1024.f;
        v0[i] = make_float4(u, 0.f, 0.f, 0.f);
        v1[i] = make_float4(u, 0.f, 0.f, 0.f);
        d[i] = 0.f;
    }
}

// Picks the faster iteration pipeline for this matrix once per workspace: a few timed
// iterations of each configuration that fits, from a varying state u, before the first FP32
// segment seeds the recursion (which overwrites what these launches wrote).
int tune_spmv(Matrix* m)
{
    Workspace* w = m->ws;
    int& slot = cfg_slot(w);
    if (slot >= 0) return RG_OK;
    const bool coef = w->coef_op;
    bool fits[2] = {cg_config_fits(m->dom, 0, coef), cg_config_fits(m->dom, 1, coef)};
    if (!fits[0] && !fits[1]) {
        set_error("FP32 iteration: no pipeline configuration fits the shared memory of one SM");
        return RG_NOT_SUPPORTED;
    }
    if (m->force_spmv >= 0 && !fits[m->force_spmv]) {
        set_error("rg_solver_set_config: that configuration does not fit this grid's windows");
        return RG_INVALID_ARG;
    }
    const int fallback = fits[1] ? 1 : 0;
    if (timers_on()) {  // keep the timed launch counts clean: no tuning launches
        slot = m->force_spmv >= 0 ? m->force_spmv : fallback;
        return RG_OK;
    }
    double* us = w->spmv_us[coef ? 1 : 0];
    us[0] = us[1] = 0.0;
    int rc = RG_OK;
    cudaEvent_t e0, e1;
    RG_CHECK_CUDA(cudaEventCreate(&e0));
    RG_CHECK_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_cfg = fallback;
    for (int cfg = 0; cfg < 2 && rc == RG_OK; ++cfg) {
        if (!fits[cfg]) continue;
        k_fill_state<<<w->grid_vec, kThreads, 0, stream()>>>(w->n, w->v4[0], w->v4[1], w->d32);
        RG_CHECK_LAUNCH();
        w->hs->alpha = 0.0;
        w->hs->beta = 0.0;
        w->hs->rho = 1.0;
        w->hs->tau = 1.0;
        w->hs->pk = 0;
        w->hs->norm = 1.0;
        if ((rc = write_scal_fields(w, 0.0, 1LL << 40, 0))) break;  // done = 0, no iteration cap
        for (int k = 0; k < 2 && rc == RG_OK; ++k) rc = launch_spmv_cfg(m, cfg);
        RG_CHECK_CUDA(cudaEventRecord(e0, stream()));
        for (int k = 0; k < 8 && rc == RG_OK; ++k) rc = launch_spmv_cfg(m, cfg);
        RG_CHECK_CUDA(cudaEventRecord(e1, stream()));
        RG_CHECK_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        us[cfg] = 1e3 * ms / 8;
        if (rc == RG_OK && ms < best) {
            best = ms;
            best_cfg = cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    slot = m->force_spmv >= 0 ? m->force_spmv : best_cfg;
    w->grid_upd32 = 0;  // the iteration has no separate update kernel
    return RG_OK;
}

int f32_step(Matrix* m)
{
    Workspace* w = m->ws;
    const int cfg = cfg_slot(w);
    return launch_spmv_cfg(m, cfg < 0 ? 0 : cfg, 0);
}

// balance (first solve only) and the preconditioner data (paso Solver.cpp:98,177)
int prepare(Matrix* m, bool want_band, bool want_band64)
{
    Domain* d = m->dom;
    Workspace* w = m->ws;
    // a band copy is written once a solve reads it and kept current from then on; arrays
    // adopted from a destroyed matrix are not written until then
    if (want_band && !m->band32) RG_CHECK_CUDA(cudaMalloc((void**)&m->band32, sizeof(float) * d->nbands * d->npad));
    if (want_band && !m->dinv32) RG_CHECK_CUDA(cudaMalloc((void**)&m->dinv32, sizeof(float) * d->n));
    if (want_band64 && !m->band64)
        RG_CHECK_CUDA(cudaMalloc((void**)&m->band64, sizeof(double) * d->nbands * d->npad));
    if ((want_band && !m->band32_ok) || (want_band64 && !m->band64_ok)) m->solver_ready = false;
    want_band = want_band || m->band32_ok;
    want_band64 = want_band64 || m->band64_ok;
    if (want_band || want_band64) {
        int rc = tma_attributes();
        if (rc) return rc;
    }
    if (m->balanced && m->solver_ready) return RG_OK;
    if (!m->dinv) RG_CHECK_CUDA(cudaMalloc((void**)&m->dinv, sizeof(double) * d->n));
    RG_CHECK_CUDA(cudaMemsetAsync(w->bad, 0, sizeof(int), stream()));
    int rc = launch_balance(m, m->balanced ? 0 : 1, w->bad, want_band, want_band64);
    if (rc) return rc;
    int bad = 0;
    RG_CHECK_CUDA(cudaMemcpyAsync(&bad, w->bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    m->balanced = true;
    if (bad) {
        set_error("SparseMatrix::invMain: non-regular main diagonal block.");
        return RG_INVALID_ARG;
    }
    m->solver_ready = true;
    m->band32_ok = want_band;
    m->band64_ok = want_band64;
    return RG_OK;
}

struct OuterState {
    double n2b, nmb;
    double last2, lastm;
    long long totIter;
};

// r = B b - A x and the paso dual-norm test (Solver.cpp:190-248).  Returns RG_OK with
// *conv set, or an error status (NaN, divergence).
int outer_residual(Matrix* m, const rg_solver_opts* o, OuterState& st, rg_diag& dg, bool* conv,
                   double* n2r, double* nmr, bool first)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    RG_TIMED(T_RESIDUAL, (k_residual<<<w->grid_rows, kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, w->x,
                                                                              w->bb, w->r, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    int rc = read_scal(w);
    if (rc) return rc;
    *n2r = std::sqrt(w->hs->n2);
    *nmr = w->hs->nm;
    dg.residual_norm = *n2r;
    dg.residual_max = *nmr;
    dg.num_outer++;
    if (o->verbose) printf("Solver: Step %lld: l2/lmax-norm of residual is %g/%g", st.totIter, *n2r, *nmr);
    if (std::isnan(*n2r)) {
        if (o->verbose) printf("\n");
        set_error("Solver: Matrix or right hand side contains undefined values.");
        return RG_NAN;
    }
    if (!first && *n2r >= st.last2 && *nmr >= st.lastm) {
        if (o->verbose) printf(" divergence!\n");
        set_error("Solver: No improvement during iteration. Iterative solver gives up.");
        return RG_DIVERGENCE;
    }
    *conv = !(*n2r > o->tolerance * st.n2b || *nmr > o->tolerance * st.nmb);
    if (*conv) {
        if (o->verbose) printf(" convergence!\n");
        dg.converged = 1;
    }
    return RG_OK;
}

int status_from(int st, long long it, const rg_solver_opts* o, long long totIter, bool* restart)
{
    *restart = false;
    if (st == ST_CONV) {
        *restart = true;
        return RG_OK;
    }
    if (st == ST_MAXIT) {
        if (o->verbose) printf("Solver: Maximum number of iterations reached.\n");
        set_error("Solver: maximum number of iteration steps reached.\nReturned solution does not fulfil stopping criterion.");
        return RG_MAXITER;
    }
    if (st == ST_TIMEOUT) {
        set_error("solver: a bounded device wait of the band SpMV pipeline gave up");
        return RG_TIMEOUT;
    }
    if (st == ST_BREAK) {
        if (it <= 1) {
            if (o->verbose) printf("Solver: Uncurable break down!\n");
            set_error("Solver: fatal break down in iterative solver.");
            return RG_BREAKDOWN;
        }
        if (o->verbose) printf("Solver: Breakdown at iter %lld. Restarting ...\n", totIter);
        *restart = true;
        return RG_OK;
    }
    return RG_OK;
}

// paso Solver() outer loop around the paso or the textbook FP64 PCG
int solve_fp64(Matrix* m, const rg_solver_opts* o, bool paso, OuterState& st, rg_diag& dg)
{
    Workspace* w = m->ws;
    const int64_t n = m->dom->n;
    const int chunk = chunk_for(n, paso ? 12 * 27 + 160 : 12 * 27 + 112);
    bool first = true;
    for (;;) {
        const long long cnt = o->iter_max - st.totIter;
        bool conv = false;
        double n2r = 0, nmr = 0;
        int rc = outer_residual(m, o, st, dg, &conv, &n2r, &nmr, first);
        first = false;
        if (rc || conv) return rc;
        const double tol = o->tolerance * std::fmin(st.n2b, 0.1 * n2r / nmr * st.nmb);
        if (o->verbose) printf(" (new tolerance = %g).\n", tol);
        st.last2 = n2r;
        st.lastm = nmr;
        long long it = 0;
        int dst = ST_RUN;
        if (paso) {
            RG_TIMED(T_VECTOR, (k_paso_init<<<w->grid_rows, kThreads, 0, stream()>>>(
                                   n, w->r, w->x, m->dinv, w->rs, w->x2, w->p, w->z, rbuf(w), w->s, tol, cnt)));
            RG_CHECK_LAUNCH();
            jacobi_sweeps(m, w->r, w->z, w->q, w->p, 2);  // the first v = prec(r): p and tau
            RG_CHECK_LAUNCH();
            if ((rc = run_until_done(m, 0, paso_step, chunk, cnt, &it, &dst))) return rc;
        } else {
            RG_TIMED(T_VECTOR, (k_std_init<<<w->grid_rows, kThreads, 0, stream()>>>(
                                   n, w->r, m->dinv, w->z, w->p, rbuf(w), w->s, tol, cnt > 0 ? cnt : 1)));
            RG_CHECK_LAUNCH();
            if ((rc = run_until_done(m, 1, std_step, chunk, cnt, &it, &dst))) return rc;
        }
        st.totIter += it;
        bool restart = false;
        rc = status_from(dst, it, o, st.totIter, &restart);
        if (rc || !restart) return rc;
    }
}

// FP32 PCG with FP64 residual replacement
int solve_f32(Matrix* m, const rg_solver_opts* o, OuterState& st, rg_diag& dg)
{
    Workspace* w = m->ws;
    const int64_t n = m->dom->n;
    const int eg = grid_for(n, kThreads, 8);
    const int chunk = chunk_for(n, w->coef_op ? 4 + 40 : 4 * 27 + 40);  // bytes per row of an iteration
    // segment reduction factor: 1e-2 keeps the FP32 recurrence within a few ulps of the
    // true residual (smaller factors let it drift and cost iterations)
    const double seg = std::fmin(std::fmax(o->inner_tolerance > 0 ? o->inner_tolerance : 1e-2, 1e-4), 0.5);
    const double scale = st.nmb;  // fixed FP32 scaling of the recurrence
    bool conv = false;
    double n2r = 0, nmr = 0;
    int rc = outer_residual(m, o, st, dg, &conv, &n2r, &nmr, true);
    if (rc || conv) return rc;
    if ((rc = tune_spmv(m))) return rc;
    bool first = true;
    long long done_iters = 0;
    for (;;) {
        // (re)seed the FP32 recurrence from the FP64 residual, keeping the search direction
        // after the first time; the start pass forms A u and A p and the first step length
        if (w->coef_op) {
            const CgArgs ca = cg_args(m->dom);
            if (m->dom->nbands == 27)
                RG_TIMED(T_VECTOR, (k_f32_cg_seed_coef<27><<<eg, kThreads, 0, stream()>>>(
                                       ca, w->r, m->bv, m->coef.khat, w->v4[0], w->v4[1], w->d32, first ? 1 : 0, w->s,
                                       1.0 / scale)));
            else
                RG_TIMED(T_VECTOR, (k_f32_cg_seed_coef<9><<<eg, kThreads, 0, stream()>>>(
                                       ca, w->r, m->bv, m->coef.khat, w->v4[0], w->v4[1], w->d32, first ? 1 : 0, w->s,
                                       1.0 / scale)));
        } else {
            RG_TIMED(T_VECTOR, (k_f32_cg_seed<<<eg, kThreads, 0, stream()>>>(n, w->r, m->dinv32, w->v4[0], w->v4[1],
                                                                             w->d32, first ? 1 : 0, w->s, 1.0 / scale)));
        }
        RG_CHECK_LAUNCH();
        w->hs->status = ST_RUN;
        RG_CHECK_CUDA(cudaMemcpyAsync(&w->s->status, &w->hs->status, sizeof(int), cudaMemcpyHostToDevice, stream()));
        const int cfg = cfg_slot(w);
        if ((rc = launch_spmv_cfg(m, cfg < 0 ? 0 : cfg, first ? 1 : 2))) return rc;
        if ((rc = read_scal(w))) return rc;
        if (w->hs->status == ST_BREAK || w->hs->status == ST_TIMEOUT) {
            bool restart = false;
            return status_from(w->hs->status, 0, o, st.totIter, &restart);
        }
        const double norm0 = w->hs->norm;  // ||r32||
        // stop this segment when the recursive residual has dropped by `seg`, or below
        // what the dual-norm test needs (with a margin for the FP32 recurrence)
        const double need = 0.5 * o->tolerance * std::fmin(st.n2b, 0.1 * n2r / nmr * st.nmb) / scale;
        const double tol = std::fmax(need, seg * norm0);
        const long long cap = o->iter_max - st.totIter;
        if ((rc = write_scal_fields(w, tol, cap > 0 ? cap : 1, 0))) return rc;
        long long it = 0;
        int dst = ST_RUN;
        if ((rc = run_until_done(m, 2, f32_step, chunk, cap, &it, &dst))) return rc;
        st.totIter += it;
        done_iters += it;
        if (dst == ST_TIMEOUT) {
            bool restart = false;
            return status_from(dst, it, o, st.totIter, &restart);
        }
        // fold the FP32 correction into x and test the FP64 true residual
        if (w->coef_op)
            RG_TIMED(T_VECTOR, (k_fold_correction_unbalance<<<eg, kThreads, 0, stream()>>>(n, w->x, w->d32, m->bv,
                                                                                          scale)));
        else
            RG_TIMED(T_VECTOR, (k_fold_correction<<<eg, kThreads, 0, stream()>>>(n, w->x, w->d32, scale)));
        RG_CHECK_LAUNCH();
        st.last2 = n2r;
        st.lastm = nmr;
        rc = outer_residual(m, o, st, dg, &conv, &n2r, &nmr, false);
        if (rc == RG_DIVERGENCE) {
            // the FP32 corrections stopped reducing the FP64 residual (rounding the values of
            // a badly conditioned matrix to FP32 bounds what refinement can reach): finish
            // with FP64 PCG from the current x
            if (o->verbose) printf("Solver: FP32 refinement stalled; continuing in FP64.\n");
            set_error("");
            dg.fp64_fallback = 1;
            return solve_fp64(m, o, false, st, dg);
        }
        if (rc || conv) return rc;
        if (o->verbose) printf(" (FP32 segment of %lld iterations).\n", it);
        bool restart = false;
        rc = status_from(dst, it, o, st.totIter, &restart);
        if (rc) return rc;
        if (dst == ST_BREAK) first = true;  // restart the recurrence after a breakdown
        else first = false;
        (void)done_iters;
    }
}

}  // namespace

int solver_config(const Matrix* m, int* spmv_cfg, int* update_grid, double* spmv_us)
{
    if (spmv_us)
        for (int c = 0; c < 2; ++c) spmv_us[c] = m->ws ? m->ws->spmv_us[m->ws->coef_op ? 1 : 0][c] : 0.0;
    if (spmv_cfg) *spmv_cfg = m->ws ? (m->ws->coef_op ? m->ws->coef_cfg : m->ws->spmv_cfg) : -1;
    if (update_grid) *update_grid = m->ws ? m->ws->grid_upd32 : 0;
    return RG_OK;
}

int solver_set_config(Matrix* m, int spmv_cfg)
{
    if (spmv_cfg < -1 || spmv_cfg > 1) {
        set_error("rg_solver_set_config: spmv_config must be -1, 0 or 1");
        return RG_INVALID_ARG;
    }
    m->force_spmv = spmv_cfg;
    if (m->ws) m->ws->spmv_cfg = m->ws->coef_cfg = -1;  // re-tune (and apply) at the next FP32 solve
    return RG_OK;
}

int set_wait_control(int polls, int withhold)
{
    if (polls < 0) {
        set_error("rg_test_wait_limit: max_polls must be >= 0");
        return RG_INVALID_ARG;
    }
    const WaitCtl c = {polls, withhold ? 1 : 0};
    // no solver kernel may be running while the limits change
    RG_CHECK_CUDA(cudaDeviceSynchronize());
    RG_CHECK_CUDA(cudaMemcpyToSymbol(g_wait_ctl, &c, sizeof(c)));
    return RG_OK;
}

int solver_prepare(Matrix* m, bool band)
{
    int rc = ensure_workspace(m, band);
    if (rc) return rc;
    return prepare(m, band, false);
}

std::mutex& pool_mutex()
{
    static std::mutex mu;
    return mu;
}

void release_workspace(Matrix* m)
{
    Workspace* w = m->ws;
    if (!w) return;
    {
        std::lock_guard<std::mutex> lock(pool_mutex());
        if (!m->dom->spare_ws) {
            for (int k = 0; k < 3; ++k) {
                if (w->graph[k]) cudaGraphExecDestroy(w->graph[k]);
                w->graph[k] = nullptr;
                w->graph_chunk[k] = 0;
                w->graph_sweeps[k] = 0;
            }
            m->dom->spare_ws = w;
            m->ws = nullptr;
            return;
        }
    }
    free_workspace(m);
}

void free_domain_workspace(Domain* d)
{
    Matrix tmp;
    tmp.dom = d;
    {
        std::lock_guard<std::mutex> lock(pool_mutex());
        tmp.ws = d->spare_ws;
        d->spare_ws = nullptr;
    }
    free_workspace(&tmp);
}

void free_workspace(Matrix* m)
{
    Workspace* w = m->ws;
    if (!w) return;
    double* dd[] = {w->r, w->x, w->rs, w->x2, w->q, w->z, w->p, w->bb, w->partials};
    for (double* p : dd) cudaFree(p);
    cudaFree(w->d32);
    cudaFree(w->v4[0]);
    cudaFree(w->v4[1]);
    cudaFree(w->counter);
    cudaFree(w->s);
    cudaFree(w->bad);
    cudaFreeHost(w->hs);
    cudaFreeHost(w->hpoll);
    for (int k = 0; k < 3; ++k)
        if (w->graph[k]) cudaGraphExecDestroy(w->graph[k]);
    if (w->ev_in) cudaEventDestroy(w->ev_in);
    if (w->ev_out) cudaEventDestroy(w->ev_out);
    for (int k = 0; k < 2; ++k)
        if (w->poll_ev[k]) cudaEventDestroy(w->poll_ev[k]);
    if (w->priv) cudaStreamDestroy(w->priv);
    delete w;
    m->ws = nullptr;
}

namespace {
int solve_impl(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag,
               double t_start);

// runs the solve on the workspace's private stream, ordered after the caller's pending
// work and before the caller's later work
struct PrivateStream {
    cudaStream_t caller;
    Workspace* w;
    bool ok = false;
    PrivateStream(Workspace* ws) : caller(stream()), w(ws)
    {
        if (cudaEventRecord(w->ev_in, caller) != cudaSuccess) return;
        if (cudaStreamWaitEvent(w->priv, w->ev_in, 0) != cudaSuccess) return;
        set_stream(w->priv);
        ok = true;
    }
    ~PrivateStream()
    {
        if (!ok) return;
        cudaEventRecord(w->ev_out, w->priv);
        cudaStreamWaitEvent(caller, w->ev_out, 0);
        set_stream(caller);
    }
};
}  // namespace

int solve(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag)
{
    const double t_start = now_s();
    const bool fp32 = o->precision == RG_PREC_FP32_REFINE;
    int rc = ensure_workspace(m, fp32);
    if (rc) return rc;
    PrivateStream ps(m->ws);
    if (!ps.ok) {
        set_error("solver: cannot order the private stream after the caller's stream");
        return RG_CUDA_ERROR;
    }
    return solve_impl(m, rhs, x, o, diag, t_start);
}

namespace {
int solve_impl(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag,
               double t_start)
{
    rg_diag dg{};
    Domain* d = m->dom;
    const int64_t n = d->n;
    const double EPS = 2.220446049250313e-16;
    RG_REQUIRE(o->method == RG_METHOD_PCG, "solver: only PCG is implemented");
    RG_REQUIRE(o->preconditioner == RG_PRECOND_JACOBI, "solver: only the Jacobi preconditioner is implemented");
    RG_REQUIRE(o->tolerance >= 100. * EPS, "Solver: Tolerance is too small.");
    RG_REQUIRE(o->tolerance <= 1., "Solver: Tolerance must be less than one.");
    RG_REQUIRE(o->guess_sweeps >= 0 && o->guess_sweeps <= 1000, "solver: guess_sweeps must be in [0, 1000]");
    const bool fp32 = o->precision == RG_PREC_FP32_REFINE;
    const bool paso = o->mode == RG_MODE_PASO && !fp32;
    if (o->sweeps > 1 && !paso) {
        set_error("solver: Jacobi with more than one sweep runs in paso mode with FP64 (RG_MODE_PASO, "
                  "RG_PREC_FP64)");
        return RG_NOT_SUPPORTED;
    }
    RG_REQUIRE(!(paso && o->initial_guess), "solver: paso mode ignores initial guesses; use RG_MODE_STANDARD");
    int rc = ensure_workspace(m, fp32);
    if (rc) return rc;
    Workspace* w = m->ws;
    // every grid reduction leaves the counter at zero; clearing it here as well keeps one
    // solve independent of anything an earlier, interrupted one left behind
    RG_CHECK_CUDA(cudaMemsetAsync(w->counter, 0, sizeof(unsigned), stream()));
    const bool band64 = !fp32 && o->layout == RG_LAYOUT_BAND;
    if (!fp32 && o->layout == RG_LAYOUT_COEF) {
        set_error("solver: RG_LAYOUT_COEF evaluates the FP32 inner operator; FP64 solves use RG_LAYOUT_CSR or "
                  "RG_LAYOUT_BAND");
        return RG_NOT_SUPPORTED;
    }
    // the FP32 iterations evaluate the operator from the element coefficients when asked and
    // when the matrix's values are what the coefficient record describes; else the band copy
    bool coef = false;
    if (fp32 && o->layout == RG_LAYOUT_COEF && (rc = coef_usable(m, &coef))) return rc;
    if ((rc = prepare(m, fp32 && !coef, band64))) return rc;
    if (coef && (rc = tma_attributes())) return rc;
    w->band64 = band64;
    w->coef_op = coef;
    dg.inner_operator = coef ? 1 : 0;
    const double t_setup = now_s();
    dg.set_up_time = t_setup - t_start;

    // r = B b and its norms (Solver.cpp:104-130)
    RG_TIMED(T_NORMS, (k_scale_norms<<<w->grid_vec, kThreads, 0, stream()>>>(n, m->bv, rhs, w->bb, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    if ((rc = read_scal(w))) return rc;
    OuterState st;
    st.n2b = std::sqrt(w->hs->n2);
    st.nmb = w->hs->nm;
    st.last2 = st.n2b;
    st.lastm = st.nmb;
    st.totIter = 1;
    dg.rhs_norm = st.n2b;
    int status = RG_OK;
    const int eg = grid_for(n, kThreads, 8);
    if (std::isnan(st.n2b) || std::isnan(st.nmb)) {
        set_error("Solver: Matrix or right hand side contains undefined values.");
        status = RG_NAN;
    } else if (st.n2b <= 0.) {
        RG_CHECK_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream()));
        dg.converged = 1;
        if (o->verbose) printf("right hand side is identical to zero.\n");
    } else {
        if (o->verbose)
            printf("Solver: l2/lmax-norm of right hand side is %g/%g.\n"
                   "Solver: l2/lmax-stopping criterion is %g/%g.\n"
                   "Solver: Iterative method is PCG.\n",
                   st.n2b, st.nmb, st.n2b * o->tolerance, st.nmb * o->tolerance);
        // initial guess: Jacobi of B b in paso (Solver.cpp:181); x0 / B or 0 otherwise
        if (paso) {
            RG_TIMED(T_VECTOR, (k_mul<<<eg, kThreads, 0, stream()>>>(n, m->dinv, w->bb, w->x)));
            RG_CHECK_LAUNCH();
            w->sweeps = o->sweeps > 1 ? o->sweeps : 1;
            const double* x0 = jacobi_sweeps(m, w->bb, w->x, w->q, nullptr, 0);
            if (x0 != w->x)
                RG_CHECK_CUDA(cudaMemcpyAsync(w->x, x0, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream()));
        } else if (o->initial_guess) {
            RG_TIMED(T_VECTOR, (k_div<<<eg, kThreads, 0, stream()>>>(n, o->initial_guess, m->bv, w->x)));
            RG_CHECK_LAUNCH();
            // Chebyshev smoothing removes the guess's rough error (which dominates its residual)
            // and keeps its smooth part, which is what PCG is slow to find: eigenvalues of
            // D^-1 A in [lmax/30, lmax], lmax from Gershgorin
            if (o->guess_sweeps > 0) {
                const Domain* dm = m->dom;
                RG_TIMED(T_NORMS, (k_gershgorin<<<w->grid_rows, kThreads, 0, stream()>>>(n, dm->ptr, m->val, m->dinv,
                                                                                      rbuf(w), &w->s->tau_next)));
                RG_CHECK_LAUNCH();
                if ((rc = read_scal(w))) return rc;
                const double lmax = w->hs->tau_next, lmin = lmax / 30.0;
                const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
                double rho = 1.0 / sigma;
                for (int k = 0; k < o->guess_sweeps; ++k) {
                    const double* src = (k & 1) ? w->x2 : w->x;
                    double* dst = (k & 1) ? w->x : w->x2;
                    double c_d = 0.0, c_r = 1.0 / theta;
                    if (k > 0) {
                        const double rho_n = 1.0 / (2.0 * sigma - rho);
                        c_d = rho_n * rho;
                        c_r = 2.0 * rho_n / delta;
                        rho = rho_n;
                    }
                    if (w->coef_op) {
                        // the operator from the element coefficients (no band copy on this path);
                        // the masked bv x of the source ping-pongs between p and q
                        const CgArgs ca = cg_args(dm);
                        double* zs = (k & 1) ? w->q : w->p;
                        double* zd = (k & 1) ? w->p : w->q;
                        if (k == 0) {
                            RG_TIMED(T_VECTOR, (k_mask_scale<<<eg, kThreads, 0, stream()>>>(n, m->coef.khat, m->bv, src,
                                                                                            zs)));
                            RG_CHECK_LAUNCH();
                        }
                        if (dm->nbands == 27)
                            RG_TIMED(T_VECTOR, (k_cheb_step_coef<27><<<eg, kThreads, 0, stream()>>>(
                                                   ca, m->coef.khat, m->bv, m->dinv, src, zs, w->bb, c_d, c_r, w->z,
                                                   dst, zd)));
                        else
                            RG_TIMED(T_VECTOR, (k_cheb_step_coef<9><<<eg, kThreads, 0, stream()>>>(
                                                   ca, m->coef.khat, m->bv, m->dinv, src, zs, w->bb, c_d, c_r, w->z,
                                                   dst, zd)));
                    } else if (m->band32 && m->band32_ok) {
                        // the FP32 band copy streams a third of the bytes of the FP64 CSR
                        TmaBandArgs ta{};
                        for (int b = 0; b < dm->nbands; ++b) ta.off[b] = (int)dm->band_off[b];
                        ta.n = n;
                        if (dm->nbands == 27)
                            RG_TIMED(T_VECTOR, (k_cheb_step_band<27><<<eg, kThreads, 0, stream()>>>(
                                                   ta, m->band32, m->dinv, src, w->bb, c_d, c_r, w->z, dst)));
                        else
                            RG_TIMED(T_VECTOR, (k_cheb_step_band<9><<<eg, kThreads, 0, stream()>>>(
                                                   ta, m->band32, m->dinv, src, w->bb, c_d, c_r, w->z, dst)));
                    } else {
                        RG_TIMED(T_VECTOR, (k_cheb_step<<<w->grid_rows, kThreads, 0, stream()>>>(
                                               n, dm->ptr, dm->idx, m->val, m->dinv, src, w->bb, c_d, c_r, w->z, dst)));
                    }
                    RG_CHECK_LAUNCH();
                }
                if (o->guess_sweeps & 1)
                    RG_CHECK_CUDA(
                        cudaMemcpyAsync(w->x, w->x2, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream()));
            }
            // a guess whose residual exceeds the right hand side's is worse than zero: drop it
            // (the residual kernel of the outer test: r = B b - A x with its norms)
            RG_TIMED(T_NORMS, (k_residual<<<w->grid_rows, kThreads, 0, stream()>>>(
                                  n, m->dom->ptr, m->dom->idx, m->val, w->x, w->bb, w->r, rbuf(w), w->s)));
            RG_CHECK_LAUNCH();
            if ((rc = read_scal(w))) return rc;
            const double r0 = std::sqrt(w->hs->n2);
            dg.guess_residual = r0;
            if (!(r0 <= st.n2b)) {
                RG_CHECK_CUDA(cudaMemsetAsync(w->x, 0, sizeof(double) * n, stream()));
                dg.guess_rejected = 1;
                if (o->verbose) printf("Solver: initial guess rejected (residual %g > %g).\n", r0, st.n2b);
            }
        } else {
            RG_CHECK_CUDA(cudaMemsetAsync(w->x, 0, sizeof(double) * n, stream()));
        }
        RG_CHECK_LAUNCH();
        const double t_net = now_s();
        status = fp32 ? solve_f32(m, o, st, dg) : solve_fp64(m, o, paso, st, dg);
        dg.net_time = now_s() - t_net;
        dg.num_iter = st.totIter;
        if (status == RG_OK || status == RG_MAXITER) {
            // x = B x (Solver.cpp:326)
            RG_TIMED(T_VECTOR, (k_mul<<<eg, kThreads, 0, stream()>>>(n, m->bv, w->x, x)));
            RG_CHECK_LAUNCH();
        }
    }
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    dg.time = now_s() - t_start;
    if (diag) *diag = dg;
    if ((status == RG_MAXITER || status == RG_DIVERGENCE) && o->accept_convergence_failure) {
        if (o->verbose) printf("paso: failed convergence error has been canceled as requested.\n");
        status = RG_OK;
    }
    return status;
}

}  // namespace

}  // namespace rg
