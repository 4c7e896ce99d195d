// paso Solver() + Solver_PCG on the device.
//
//  * RG_MODE_PASO: the reference algorithm (paso/src/Solver.cpp:46-330 and
//    paso/src/PCG.cpp:62-367): in-place balancing, Jacobi initial guess, PCG with the
//    minimal-residual smoothing sequence (rs, x2, gamma_1/2) stopping on the smoothed
//    residual, and the outer loop's dual l2/lmax test on the true residual.
//  * RG_MODE_STANDARD: the same outer loop around textbook Jacobi-PCG (no smoothing).
//  * RG_PREC_FP32_REFINE: the outer loop stays FP64 (true residual on the FP64 CSR
//    values, solution update, norms), the inner Jacobi-PCG runs on the FP32 band copy
//    with FP32 vectors and FP64 dot products.
//
// One PCG iteration is two or three kernels.  Scalars (alpha, beta, tau, ...) live in
// device memory: every reduction is finished by the last CTA of its kernel, which
// also sets the next step's scalars and a `done` flag, so the host only polls `done`
// once per chunk of iterations and kernels queued after convergence return at once.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "rg_internal.cuh"

namespace rg {

namespace {

constexpr int kLpr = 8;     // lanes per CSR row
constexpr int kThreads = 256;

struct Scal {
    double tau, tau_next, tau_old;  // paso: tau = v.r
    double delta, alpha, beta;
    double gamma1, gamma2;
    double norm, tol;               // stopping norm and its limit
    double rho, rho_next;           // textbook PCG
    double n2, nm;                  // norms from norm kernels
    long long iter, maxit;
    int done, status, pidx, pad;
};

enum { ST_RUN = 0, ST_CONV = 1, ST_MAXIT = 3, ST_BREAK = 4 };

}  // namespace

struct Workspace {
    int64_t n = 0;
    double *r = nullptr, *x = nullptr, *rs = nullptr, *x2 = nullptr, *q = nullptr, *z = nullptr;
    double* p[2] = {nullptr, nullptr};
    double *bb = nullptr;  // balanced rhs
    float *r32 = nullptr, *d32 = nullptr, *q32 = nullptr, *z32 = nullptr;
    float* p32[2] = {nullptr, nullptr};
    double* partials = nullptr;
    unsigned* counter = nullptr;
    Scal* s = nullptr;        // device scalars
    Scal* hs = nullptr;       // pinned host copy
    int* bad = nullptr;
    int grid = 0;
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
        Workspace* w = new Workspace();
        m->ws = w;
        w->n = n;
        w->grid = grid_for(n, kThreads / kLpr, 8);
        int rc;
        if ((rc = dalloc(&w->r, n)) || (rc = dalloc(&w->x, n)) || (rc = dalloc(&w->rs, n)) ||
            (rc = dalloc(&w->x2, n)) || (rc = dalloc(&w->q, n)) || (rc = dalloc(&w->z, n)) ||
            (rc = dalloc(&w->p[0], n)) || (rc = dalloc(&w->p[1], n)) || (rc = dalloc(&w->bb, n)) ||
            (rc = dalloc(&w->partials, (size_t)4 * kNumSMs * 64)) || (rc = dalloc(&w->counter, 1)) ||
            (rc = dalloc(&w->s, 1)) || (rc = dalloc(&w->bad, 1)))
            return rc;
        RG_CHECK_CUDA(cudaMallocHost((void**)&w->hs, sizeof(Scal)));
        RG_CHECK_CUDA(cudaMemsetAsync(w->counter, 0, sizeof(unsigned), stream()));
    }
    Workspace* w = m->ws;
    if (fp32 && !w->r32) {
        int rc;
        if ((rc = dalloc(&w->r32, n)) || (rc = dalloc(&w->d32, n)) || (rc = dalloc(&w->q32, n)) ||
            (rc = dalloc(&w->z32, n)) || (rc = dalloc(&w->p32[0], n)) || (rc = dalloc(&w->p32[1], n)))
            return rc;
    }
    return RG_OK;
}

// ------------------------------------------------------------------ common kernels
// row-group iteration helper: each group of kLpr lanes owns one row per trip; the trip
// count is uniform over a warp so shuffles stay converged.
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

// out = a .* b (out may be b), returns ||out||_2^2 and ||out||_inf in s->n2, s->nm
__global__ void __launch_bounds__(kThreads) k_scale_norms(int64_t n, const double* __restrict__ a,
                                                          const double* b, double* out, ReduceBuf rb,
                                                          Scal* s)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
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

// r = bb - A x (bb the balanced rhs) with the l2^2 / max norms of r
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
        double acc = 0.0;
        if (row < n)
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) acc = fma(val[k], x[idx[k]], acc);
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

__global__ void k_mul(int64_t n, const double* __restrict__ a, const double* b, double* out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

__global__ void k_div(int64_t n, const double* a, const double* __restrict__ b, double* out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] / b[i];
}

// ------------------------------------------------------------------ paso PCG (FP64, CSR)
// PCG.cpp:102-131 initialisation + the first v = prec(r), tau = v.r
__global__ void __launch_bounds__(kThreads) k_paso_init(int64_t n, const double* __restrict__ r,
                                                        const double* __restrict__ x,
                                                        const double* __restrict__ dinv,
                                                        double* rs, double* x2, double* p0,
                                                        double* z, ReduceBuf rb, Scal* s,
                                                        double tol, long long maxit)
{
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = r[i];
        rs[i] = ri;
        x2[i] = x[i];
        p0[i] = 0.0;
        const double zi = ri * dinv[i];
        z[i] = zi;
        v[0] += zi * ri;
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->tau = 0.0;
        s->tau_next = t[0];
        s->iter = 0;
        s->maxit = maxit;
        s->tol = tol;
        s->done = 0;
        s->status = ST_RUN;
        s->pidx = 0;
        s->norm = 0.0;
    }
}

// p = v + beta*p (PCG.cpp:193-218) evaluated per column on the fly, v = A*p (223),
// delta = p.v (228-260), alpha = tau/delta, breakdown on delta == 0
__global__ void __launch_bounds__(kThreads) k_paso_spmv(int64_t n, const int32_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        const double* __restrict__ z,
                                                        double* pa, double* pb, double* __restrict__ q,
                                                        ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double tau = s->tau_next;
    const bool first = s->iter == 0;
    const double beta = first ? 0.0 : tau / s->tau;
    const double* __restrict__ pold = s->pidx ? pb : pa;
    double* __restrict__ pnew = s->pidx ? pa : pb;
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = 0.0;
        if (row < n) {
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) {
                const int32_t j = idx[k];
                const double pj = first ? z[j] : z[j] + beta * pold[j];
                acc = fma(val[k], pj, acc);
            }
        }
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            const double pi = first ? z[row] : z[row] + beta * pold[row];
            pnew[row] = pi;
            q[row] = acc;
            v[0] += acc * pi;
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->tau_old = s->tau;
        s->tau = tau;
        s->beta = beta;
        s->delta = t[0];
        s->alpha = tau / t[0];
        if (fabs(t[0]) <= 0.0) {  // breakFlag (PCG.cpp:262)
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// r -= alpha*v; d = r - rs; sum d^2, d.rs (PCG.cpp:263-306); x2 += alpha*p; and the next
// iteration's v = prec(r), tau = v.r
__global__ void __launch_bounds__(kThreads) k_paso_update1(int64_t n, double* __restrict__ r,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ rs,
                                                           double* __restrict__ x2,
                                                           const double* pa, const double* pb,
                                                           const double* __restrict__ dinv,
                                                           double* __restrict__ z, ReduceBuf rb,
                                                           Scal* s)
{
    if (s->done) return;
    const double alpha = s->alpha;
    const double* __restrict__ pnew = s->pidx ? pa : pb;
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double rsi = rs[i];
        const double d = ri - rsi;
        v[0] += d * d;
        v[1] += d * rsi;
        x2[i] += alpha * pnew[i];
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
    }
}

// rs = g2 rs + g1 r; x = g2 x + g1 x2; sum rs^2; stopping tests (PCG.cpp:307-347)
__global__ void __launch_bounds__(kThreads) k_paso_update2(int64_t n, double* __restrict__ rs,
                                                           const double* __restrict__ r,
                                                           double* __restrict__ x,
                                                           const double* __restrict__ x2,
                                                           ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double g1 = s->gamma1, g2 = s->gamma2;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double rsi = g2 * rs[i] + g1 * r[i];
        rs[i] = rsi;
        x[i] = g2 * x[i] + g1 * x2[i];
        v[0] += rsi * rsi;
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
        s->pidx ^= 1;
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
    }
}

// ------------------------------------------------------------------ textbook PCG, FP64 CSR
__global__ void __launch_bounds__(kThreads) k_std_init(int64_t n, const double* __restrict__ r,
                                                       const double* __restrict__ dinv,
                                                       double* z, double* p0, ReduceBuf rb,
                                                       Scal* s, double tol, long long maxit)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = r[i];
        const double zi = ri * dinv[i];
        z[i] = zi;
        p0[i] = 0.0;
        v[0] += zi * ri;
        v[1] += ri * ri;
    }
    double t[2];
    if (grid_reduce<2>(v, rb, t) && threadIdx.x == 0) {
        s->rho = 0.0;
        s->rho_next = t[0];
        s->norm = sqrt(t[1]);
        s->iter = 0;
        s->maxit = maxit;
        s->tol = tol;
        s->pidx = 0;
        s->status = ST_RUN;
        s->done = (s->norm <= tol) ? 1 : 0;
        if (s->done) s->status = ST_CONV;
    }
}

__global__ void __launch_bounds__(kThreads) k_std_spmv(int64_t n, const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx,
                                                       const double* __restrict__ val,
                                                       const double* __restrict__ z, double* pa,
                                                       double* pb, double* __restrict__ q,
                                                       ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double rho = s->rho_next;
    const bool first = s->iter == 0;
    const double beta = first ? 0.0 : rho / s->rho;
    const double* __restrict__ pold = s->pidx ? pb : pa;
    double* __restrict__ pnew = s->pidx ? pa : pb;
    double v[1] = {0.0};
    RG_ROW_LOOP(n)
    {
        double acc = 0.0;
        if (row < n)
            for (int32_t k = ptr[row] + lane; k < ptr[row + 1]; k += kLpr) {
                const int32_t j = idx[k];
                acc = fma(val[k], first ? z[j] : z[j] + beta * pold[j], acc);
            }
        acc = group_sum(acc);
        if (row < n && lane == 0) {
            const double pi = first ? z[row] : z[row] + beta * pold[row];
            pnew[row] = pi;
            q[row] = acc;
            v[0] += acc * pi;
        }
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->rho = rho;
        s->delta = t[0];
        s->alpha = rho / t[0];
        if (!(fabs(t[0]) > 0.0)) {
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_std_update(int64_t n, double* __restrict__ x,
                                                         double* __restrict__ r,
                                                         const double* __restrict__ q,
                                                         const double* pa, const double* pb,
                                                         const double* __restrict__ dinv,
                                                         double* __restrict__ z, ReduceBuf rb,
                                                         Scal* s)
{
    if (s->done) return;
    const double alpha = s->alpha;
    const double* __restrict__ pnew = s->pidx ? pa : pb;
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * pnew[i];
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
        s->rho_next = t[0];
        const double norm = sqrt(t[1]);
        s->norm = norm;
        s->pidx ^= 1;
        if (norm <= s->tol) {
            s->status = ST_CONV;
            s->done = 1;
        } else if (it >= s->maxit) {
            s->status = ST_MAXIT;
            s->done = 1;
        } else if (!(fabs(t[0]) > 0.0)) {
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// ------------------------------------------------------------------ textbook PCG, FP32 band
// The band copy stores row i's coefficient to neighbour i+off_b at band[b*n + i] (0 where
// the neighbour does not exist), so a thread per row reads every band coalesced; column
// indices are clamped into range, where the matching band value is 0.
struct BandOffsets {
    int off[27];
};

__global__ void __launch_bounds__(kThreads) k_f32_init(int64_t n, const double* __restrict__ r64,
                                                       const float* __restrict__ dinv32,
                                                       float* r32, float* z32, float* d32,
                                                       float* p0, ReduceBuf rb, Scal* s,
                                                       double inv_scale, double rel_tol,
                                                       long long maxit)
{
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float ri = (float)(r64[i] * inv_scale);
        r32[i] = ri;
        const float zi = ri * dinv32[i];
        z32[i] = zi;
        d32[i] = 0.f;
        p0[i] = 0.f;
        v[0] += (double)zi * (double)ri;
        v[1] += (double)ri * (double)ri;
    }
    double t[2];
    if (grid_reduce<2>(v, rb, t) && threadIdx.x == 0) {
        s->rho = 0.0;
        s->rho_next = t[0];
        s->norm = sqrt(t[1]);
        s->tol = rel_tol * sqrt(t[1]);
        s->iter = 0;
        s->maxit = maxit;
        s->pidx = 0;
        s->status = ST_RUN;
        s->done = 0;
    }
}

template <int NB>
__global__ void __launch_bounds__(kThreads) k_f32_spmv(int64_t n, const float* __restrict__ band,
                                                       const __grid_constant__ BandOffsets bo,
                                                       const float* __restrict__ z, float* pa,
                                                       float* pb, float* __restrict__ q,
                                                       ReduceBuf rb, Scal* s)
{
    if (s->done) return;
    const double rho = s->rho_next;
    const bool first = s->iter == 0;
    const float beta = first ? 0.f : (float)(rho / s->rho);
    const float* __restrict__ pold = s->pidx ? pb : pa;
    float* __restrict__ pnew = s->pidx ? pa : pb;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float acc = 0.f;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            int64_t j = i + bo.off[b];
            j = j < 0 ? 0 : (j >= n ? n - 1 : j);
            const float pj = first ? z[j] : fmaf(beta, pold[j], z[j]);
            acc = fmaf(band[(size_t)b * n + i], pj, acc);
        }
        const float pi = first ? z[i] : fmaf(beta, pold[i], z[i]);
        pnew[i] = pi;
        q[i] = acc;
        v[0] += (double)acc * (double)pi;
    }
    double t[1];
    if (grid_reduce<1>(v, rb, t) && threadIdx.x == 0) {
        s->rho = rho;
        s->delta = t[0];
        s->alpha = rho / t[0];
        if (!(fabs(t[0]) > 0.0)) {
            s->iter += 1;
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_f32_update(int64_t n, float* __restrict__ d,
                                                         float* __restrict__ r,
                                                         const float* __restrict__ q,
                                                         const float* pa, const float* pb,
                                                         const float* __restrict__ dinv,
                                                         float* __restrict__ z, ReduceBuf rb,
                                                         Scal* s)
{
    if (s->done) return;
    const float alpha = (float)s->alpha;
    const float* __restrict__ pnew = s->pidx ? pa : pb;
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        d[i] = fmaf(alpha, pnew[i], d[i]);
        const float ri = fmaf(-alpha, q[i], r[i]);
        r[i] = ri;
        const float zi = ri * dinv[i];
        z[i] = zi;
        v[0] += (double)zi * (double)ri;
        v[1] += (double)ri * (double)ri;
    }
    double t[2];
    if (grid_reduce<2>(v, rb, t) && threadIdx.x == 0) {
        const long long it = s->iter + 1;
        s->iter = it;
        s->rho_next = t[0];
        const double norm = sqrt(t[1]);
        s->norm = norm;
        s->pidx ^= 1;
        if (norm <= s->tol) {
            s->status = ST_CONV;
            s->done = 1;
        } else if (it >= s->maxit) {
            s->status = ST_MAXIT;
            s->done = 1;
        } else if (!(fabs(t[0]) > 0.0)) {
            s->status = ST_BREAK;
            s->done = 1;
        }
    }
}

// x64 += scale * d32
__global__ void k_add_correction(int64_t n, double* __restrict__ x, const float* __restrict__ d,
                                 double scale)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] += scale * (double)d[i];
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

ReduceBuf rbuf(Workspace* w) { return ReduceBuf{w->partials, w->counter}; }

// iterations per host poll: about 1 ms of device work, at least 4
int chunk_for(int64_t n, int64_t bytes_per_row)
{
    const double iter_s = (double)n * bytes_per_row / 5.0e12 + 6e-6;
    int c = (int)(1e-3 / iter_s);
    return c < 4 ? 4 : (c > 256 ? 256 : c);
}

// runs PCG iterations until the device flags done; returns iterations and status
using IterFn = int (*)(Matrix*, int);
int run_until_done(Matrix* m, IterFn step, int chunk, long long cap, long long* iters, int* status)
{
    Workspace* w = m->ws;
    long long launched = 0;
    for (;;) {
        for (int c = 0; c < chunk; ++c) {
            int rc = step(m, c);
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

int paso_step(Matrix* m, int)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    RG_TIMED(T_PASO_SPMV, (k_paso_spmv<<<w->grid, kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, w->z, w->p[0], w->p[1],
                                                   w->q, rbuf(w), w->s)));
    RG_TIMED(T_PASO_UPDATE1, (k_paso_update1<<<w->grid, kThreads, 0, stream()>>>(d->n, w->r, w->q, w->rs, w->x2, w->p[0], w->p[1],
                                                      m->dinv, w->z, rbuf(w), w->s)));
    RG_TIMED(T_PASO_UPDATE2, (k_paso_update2<<<w->grid, kThreads, 0, stream()>>>(d->n, w->rs, w->r, w->x, w->x2, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int std_step(Matrix* m, int)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    RG_TIMED(T_STD_SPMV, (k_std_spmv<<<w->grid, kThreads, 0, stream()>>>(d->n, d->ptr, d->idx, m->val, w->z, w->p[0], w->p[1],
                                                  w->q, rbuf(w), w->s)));
    RG_TIMED(T_STD_UPDATE, (k_std_update<<<w->grid, kThreads, 0, stream()>>>(d->n, w->x, w->r, w->q, w->p[0], w->p[1], m->dinv,
                                                    w->z, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int f32_step(Matrix* m, int)
{
    Workspace* w = m->ws;
    const Domain* d = m->dom;
    const int grid = grid_for(d->n, kThreads, 8);
    BandOffsets bo;
    for (int b = 0; b < d->nbands; ++b) bo.off[b] = (int)d->band_off[b];
    if (d->nbands == 27)
        RG_TIMED(T_F32_SPMV, (k_f32_spmv<27><<<grid, kThreads, 0, stream()>>>(d->n, m->band32, bo, w->z32, w->p32[0], w->p32[1],
                                                       w->q32, rbuf(w), w->s)));
    else
        RG_TIMED(T_F32_SPMV, (k_f32_spmv<9><<<grid, kThreads, 0, stream()>>>(d->n, m->band32, bo, w->z32, w->p32[0], w->p32[1],
                                                      w->q32, rbuf(w), w->s)));
    RG_TIMED(T_F32_UPDATE, (k_f32_update<<<grid, kThreads, 0, stream()>>>(d->n, w->d32, w->r32, w->q32, w->p32[0], w->p32[1],
                                                 m->dinv32, w->z32, rbuf(w), w->s)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

// balance (first solve only) and the preconditioner data (paso Solver.cpp:98,177)
int prepare(Matrix* m, bool want_band)
{
    Domain* d = m->dom;
    Workspace* w = m->ws;
    const bool need_band = want_band && !m->band32;
    if (need_band) {
        RG_CHECK_CUDA(cudaMalloc((void**)&m->band32, sizeof(float) * d->nbands * d->n));
        if (!m->dinv32) RG_CHECK_CUDA(cudaMalloc((void**)&m->dinv32, sizeof(float) * d->n));
        m->solver_ready = false;
    }
    if (m->balanced && m->solver_ready) return RG_OK;
    if (!m->dinv) RG_CHECK_CUDA(cudaMalloc((void**)&m->dinv, sizeof(double) * d->n));
    RG_CHECK_CUDA(cudaMemsetAsync(w->bad, 0, sizeof(int), stream()));
    int rc = launch_balance(m, m->balanced ? 0 : 1, w->bad, m->band32 != nullptr);
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
    return RG_OK;
}

}  // namespace

void free_workspace(Matrix* m)
{
    Workspace* w = m->ws;
    if (!w) return;
    double* dd[] = {w->r, w->x, w->rs, w->x2, w->q, w->z, w->p[0], w->p[1], w->bb, w->partials};
    for (double* p : dd) cudaFree(p);
    float* ff[] = {w->r32, w->d32, w->q32, w->z32, w->p32[0], w->p32[1]};
    for (float* p : ff) cudaFree(p);
    cudaFree(w->counter);
    cudaFree(w->s);
    cudaFree(w->bad);
    cudaFreeHost(w->hs);
    delete w;
    m->ws = nullptr;
}

int solve(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag)
{
    const double t_start = now_s();
    rg_diag dg{};
    Domain* d = m->dom;
    const int64_t n = d->n;
    const double EPS = 2.220446049250313e-16;
    RG_REQUIRE(o->method == RG_METHOD_PCG, "solver: only PCG is implemented");
    RG_REQUIRE(o->preconditioner == RG_PRECOND_JACOBI, "solver: only the Jacobi preconditioner is implemented");
    RG_REQUIRE(o->tolerance >= 100. * EPS, "Solver: Tolerance is too small.");
    RG_REQUIRE(o->tolerance <= 1., "Solver: Tolerance must be less than one.");
    if (o->sweeps > 1) {
        set_error("solver: Jacobi with more than one sweep is not implemented on the GPU");
        return RG_NOT_SUPPORTED;
    }
    const bool fp32 = o->precision == RG_PREC_FP32_REFINE;
    const bool paso = o->mode == RG_MODE_PASO && !fp32;
    RG_REQUIRE(!(paso && o->initial_guess), "solver: paso mode ignores initial guesses; use RG_MODE_STANDARD");
    int rc = ensure_workspace(m, fp32);
    if (rc) return rc;
    Workspace* w = m->ws;
    if ((rc = prepare(m, fp32))) return rc;
    const double t_setup = now_s();
    dg.set_up_time = t_setup - t_start;
    const int grid = w->grid;
    const ReduceBuf rb = rbuf(w);
    const double tolerance = o->tolerance;

    // r = B b and its norms (Solver.cpp:104-130)
    RG_TIMED(T_NORMS, (k_scale_norms<<<grid, kThreads, 0, stream()>>>(n, m->bv, rhs, w->bb, rb, w->s)));
    RG_CHECK_LAUNCH();
    if ((rc = read_scal(w))) return rc;
    const double n2b = std::sqrt(w->hs->n2), nmb = w->hs->nm;
    dg.rhs_norm = n2b;
    int status = RG_OK;
    if (std::isnan(n2b) || std::isnan(nmb)) {
        set_error("Solver: Matrix or right hand side contains undefined values.");
        status = RG_NAN;
    } else if (n2b <= 0.) {
        RG_CHECK_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream()));
        dg.converged = 1;
        if (o->verbose) printf("right hand side is identical to zero.\n");
    } else {
        if (o->verbose)
            printf("Solver: l2/lmax-norm of right hand side is %g/%g.\n"
                   "Solver: l2/lmax-stopping criterion is %g/%g.\n"
                   "Solver: Iterative method is PCG.\n",
                   n2b, nmb, n2b * tolerance, nmb * tolerance);
        // initial guess: Jacobi of B b in paso (Solver.cpp:181); x0 / B or 0 otherwise
        const int eg = grid_for(n, kThreads, 8);
        if (paso) {
            RG_TIMED(T_VECTOR, (k_mul<<<eg, kThreads, 0, stream()>>>(n, m->dinv, w->bb, w->x)));
        } else if (o->initial_guess) {
            RG_TIMED(T_VECTOR, (k_div<<<eg, kThreads, 0, stream()>>>(n, o->initial_guess, m->bv, w->x)));
        } else {
            RG_CHECK_CUDA(cudaMemsetAsync(w->x, 0, sizeof(double) * n, stream()));
        }
        RG_CHECK_LAUNCH();
        const double t_net = now_s();
        long long totIter = 1;
        double last2 = n2b, lastm = nmb;
        bool fin = false;
        const int chunk_paso = chunk_for(n, 12 * 27 + 152);
        const int chunk_std = chunk_for(n, 12 * 27 + 96);
        const int chunk_f32 = chunk_for(n, 4 * 27 + 48);
        while (!fin) {
            long long cnt = o->iter_max - totIter;
            fin = true;
            // r = B b - A x, norms (Solver.cpp:190-224)
            RG_TIMED(T_RESIDUAL, (k_residual<<<grid, kThreads, 0, stream()>>>(n, d->ptr, d->idx, m->val, w->x, w->bb, w->r, rb, w->s)));
            RG_CHECK_LAUNCH();
            if ((rc = read_scal(w))) return rc;
            const double n2r = std::sqrt(w->hs->n2), nmr = w->hs->nm;
            dg.residual_norm = n2r;
            dg.residual_max = nmr;
            dg.num_outer++;
            if (o->verbose) printf("Solver: Step %lld: l2/lmax-norm of residual is %g/%g", totIter, n2r, nmr);
            if (std::isnan(n2r)) {
                set_error("Solver: Matrix or right hand side contains undefined values.");
                status = RG_NAN;
                break;
            }
            if (totIter > 1 && n2r >= last2 && nmr >= lastm) {
                if (o->verbose) printf(" divergence!\n");
                set_error("Solver: No improvement during iteration. Iterative solver gives up.");
                status = RG_DIVERGENCE;
                break;
            }
            if (!(n2r > tolerance * n2b || nmr > tolerance * nmb)) {
                if (o->verbose) printf(" convergence!\n");
                dg.converged = 1;
                break;
            }
            double tol = tolerance * std::fmin(n2b, 0.1 * n2r / nmr * nmb);
            if (o->verbose) printf(" (new tolerance = %g).\n", tol);
            last2 = n2r;
            lastm = nmr;
            long long it = 0;
            int st = ST_RUN;
            if (paso) {
                RG_TIMED(T_VECTOR, (k_paso_init<<<grid, kThreads, 0, stream()>>>(n, w->r, w->x, m->dinv, w->rs, w->x2, w->p[0], w->z,
                                                            rb, w->s, tol, cnt)));
                RG_CHECK_LAUNCH();
                if ((rc = run_until_done(m, paso_step, chunk_paso, cnt, &it, &st))) return rc;
            } else if (!fp32) {
                RG_TIMED(T_VECTOR, (k_std_init<<<grid, kThreads, 0, stream()>>>(n, w->r, m->dinv, w->z, w->p[0], rb, w->s, tol,
                                                           cnt > 0 ? cnt : 1)));
                RG_CHECK_LAUNCH();
                if ((rc = run_until_done(m, std_step, chunk_std, cnt, &it, &st))) return rc;
            } else {
                // FP32 inner solve of A d = r / s, relative reduction eta
                const double need = tol / n2r;
                const double eta = std::fmax(need, o->inner_tolerance > 0 ? o->inner_tolerance : 1e-5);
                const double scale = nmr;
                RG_TIMED(T_VECTOR, (k_f32_init<<<grid_for(n, kThreads, 8), kThreads, 0, stream()>>>(
                    n, w->r, m->dinv32, w->r32, w->z32, w->d32, w->p32[0], rb, w->s, 1.0 / scale, eta,
                    cnt > 0 ? cnt : 1)));
                RG_CHECK_LAUNCH();
                if ((rc = run_until_done(m, f32_step, chunk_f32, cnt, &it, &st))) return rc;
                RG_TIMED(T_VECTOR, (k_add_correction<<<grid_for(n, kThreads, 8), kThreads, 0, stream()>>>(n, w->x, w->d32, scale)));
                RG_CHECK_LAUNCH();
                if (st == ST_CONV || st == ST_MAXIT) {
                    // a converged or exhausted inner solve still improves x; the outer
                    // residual decides
                }
            }
            totIter += it;
            if (st == ST_CONV) {
                fin = false;
            } else if (st == ST_MAXIT) {
                if (o->verbose) printf("Solver: Maximum number of iterations reached.\n");
                set_error("Solver: maximum number of iteration steps reached.\nReturned solution does not fulfil stopping criterion.");
                status = RG_MAXITER;
                break;
            } else if (st == ST_BREAK) {
                if (it <= 1) {
                    if (o->verbose) printf("Solver: Uncurable break down!\n");
                    set_error("Solver: fatal break down in iterative solver.");
                    status = RG_BREAKDOWN;
                    break;
                }
                if (o->verbose) printf("Solver: Breakdown at iter %lld. Restarting ...\n", totIter);
                fin = false;
            }
        }
        dg.net_time = now_s() - t_net;
        dg.num_iter = totIter;
        // x = B x (Solver.cpp:326)
        RG_TIMED(T_VECTOR, (k_mul<<<eg, kThreads, 0, stream()>>>(n, m->bv, w->x, x)));
        RG_CHECK_LAUNCH();
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

}  // namespace rg
