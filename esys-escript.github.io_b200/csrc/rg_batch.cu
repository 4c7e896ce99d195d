// Batched solves: many Brick/Rectangle systems of different sizes, each with R right hand
// sides, solved together by PCG + Jacobi with FP32 inner iterations and FP64 iterative
// refinement (the per-system algorithm of rg_solve's FP32_REFINE precision; paso's
// Solver.cpp/PCG.cpp outer test per right hand side).
//
// Layout.  The systems' FP32 27-band (9 in 2D) copies stay where rg_solve's preparation put
// them (tile-major: 256 rows x nbands per tile).  The batch numbers all tiles of all systems
// consecutively; every kernel walks that tile list (grid-stride, persistent CTAs), so one
// launch advances every system by one step.  Vectors hold the R right hand sides of a row
// next to each other ([row][R], rows of a system padded to a multiple of 256): one matrix
// read serves all R right hand sides.
//
// One inner iteration is three launches: q = A p with the p.q partial sums (the last CTA
// of each system reduces them in a fixed order and sets alpha), the x/r update with r.z and
// r.r (last CTA: beta, convergence, stagnation), and p = z + beta p.  Chunks of iterations
// are captured as a CUDA graph and replayed until no right hand side is active; then one
// FP64 pass folds the FP32 corrections into x, recomputes r = B b - A x from the balanced
// FP64 CSR values and the host applies paso's dual-norm test per right hand side.
//
// The autotuner times the three kernels for a few grid sizes (CTAs per SM) on the batch
// itself and picks the fastest; the chunk length follows from the measured iteration time.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rg_internal.cuh"

namespace rg {
namespace batch {

constexpr int kTile = 256;
constexpr int kMaxBands = 27;

struct Inst {
    int64_t n;            // rows (nodes)
    int64_t tile0;        // first batch tile
    int64_t ntiles;
    int64_t voff;         // first batch row (multiple of kTile)
    int nbands;
    int64_t off[kMaxBands];
    const float* band;    // [ntiles][nbands][256]
    const float* dinv32;
    const int32_t* ptr;   // FP64 CSR (balanced values)
    const int32_t* idx;
    const double* val;
    const double* bv;     // balance vector
    int64_t nunits;       // work units of the iteration kernels (current tile-group size)
};

// A work unit of the iteration kernels: up to `group` consecutive tiles of one system (the
// autotuned tile-group size); one partial sum per unit.  .x system, .y first batch tile,
// .z tiles, .w the unit's index within its system.
using Unit = int4;

// per right hand side state (device); host reads and writes it between segments
struct Rhs {
    double rz, pq, alpha, beta;
    double norm;          // ||r32||_2 of the recursion
    double target;        // segment ends when norm <= target
    double best;
    double inv_scale;     // r32 = r64 * inv_scale
    double n2r, nmr;      // FP64 residual norms (outer pass)
    double n2b, nmb;      // balanced right hand side norms
    double need, seg;     // segment target = max(need, seg * ||r32|| at the seed)
    int active;           // iterating in the current segment
    int since;            // iterations without a new 5% minimum
    int iters;            // inner iterations, all segments
    int breakdown;        // rz or pq was not positive
    int fresh;            // host: start the search direction afresh at the next seed
    int pad;
};

// a segment also ends when the recursion makes no new 5% minimum for this many iterations
constexpr int kStagnation = 200;

struct Batch {
    int ninst = 0, R = 0, dim = 3;
    int64_t ntiles = 0, rows = 0;
    std::vector<Inst> h_inst;
    std::vector<Matrix*> mats;
    Inst* d_inst = nullptr;
    int* d_tile_inst = nullptr;
    Unit* d_units = nullptr;      // iteration work units (capacity ntiles)
    int64_t nunits = 0;
    int group = 4;                // tiles per work unit
    int* d_inst_active = nullptr;
    int* d_nactive = nullptr;     // number of active right hand sides
    int* h_nactive = nullptr;     // pinned
    Rhs* d_rhs = nullptr;
    std::vector<Rhs> h_rhs;
    unsigned* d_cnt = nullptr;    // per system tickets
    double* d_part = nullptr;     // [ntiles][2R]
    float *p = nullptr, *q = nullptr, *r32 = nullptr, *d32 = nullptr;
    double *x64 = nullptr, *bb64 = nullptr, *r64 = nullptr;
    double** d_user = nullptr;  // per system user pointers (rhs or x)
    cudaStream_t priv = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // tuning
    int grid_spmv = 0, grid_upd = 0, chunk = 16;
    int spmv_kind = 0;    // 0: one row per thread (k_b_spmv); 1: two rows per thread (k_b_spmv2)
    int force_kind = -1;  // SpMV kernel fixed by the caller (-1: the tuner's choice)
    bool tuned = false;
    cudaGraphExec_t graph = nullptr;
    int graph_chunk = 0;
    long long graph_launches[T_COUNT] = {};
    double tuned_iter_us = 0;
    int maxit = 100000;
};

// ------------------------------------------------------------------ device helpers
template <int R>
struct Vec;
template <>
struct Vec<1> {
    __device__ static void ld(const float* p, float (&v)[1]) { v[0] = *p; }
    __device__ static void st(float* p, const float (&v)[1]) { *p = v[0]; }
};
template <>
struct Vec<2> {
    __device__ static void ld(const float* p, float (&v)[2])
    {
        const float2 a = *reinterpret_cast<const float2*>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
    __device__ static void st(float* p, const float (&v)[2]) { *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]); }
};
template <>
struct Vec<4> {
    __device__ static void ld(const float* p, float (&v)[4])
    {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
    __device__ static void st(float* p, const float (&v)[4])
    {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <>
struct Vec<8> {
    __device__ static void ld(const float* p, float (&v)[8])
    {
        const float4 a = reinterpret_cast<const float4*>(p)[0];
        const float4 b = reinterpret_cast<const float4*>(p)[1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
        v[4] = b.x;
        v[5] = b.y;
        v[6] = b.z;
        v[7] = b.w;
    }
    __device__ static void st(float* p, const float (&v)[8])
    {
        reinterpret_cast<float4*>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4*>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
};

// block-wide sums of NV values (NT threads); thread 0 writes them to out[0..NV)
template <int NV, int NT = kTile>
__device__ void block_sum_to(double (&v)[NV], double* out)
{
    __shared__ double sh[NT / 32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    warp_sum<NV>(v);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[wid][j] = v[j];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double a = 0.0;
            for (int w = 0; w < NT / 32; ++w) a += sh[w][j];
            out[j] = a;
        }
    __syncthreads();
}

// Ticket of system i: true in the CTA that wrote the last of the system's `count` partials
// (slots first..first+count-1), which then reduces them in a fixed order into tot[0..NV).
template <int NV, int NT = kTile>
__device__ bool last_reduce(int i, int64_t first, int64_t count, unsigned* cnt, const double* part, int stride,
                            double (&tot)[NV])
{
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&cnt[i], 1u) == (unsigned)(count - 1);
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) a[j] = 0.0;
    for (int64_t t = threadIdx.x; t < count; t += NT)
#pragma unroll
        for (int j = 0; j < NV; ++j) a[j] += __ldcg(part + (first + t) * stride + j);
    __shared__ double res[NV];
    block_sum_to<NV, NT>(a, res);
#pragma unroll
    for (int j = 0; j < NV; ++j) tot[j] = res[j];
    if (threadIdx.x == 0) cnt[i] = 0u;
    return true;
}

template <int NV>
__device__ bool last_tile_reduce(const Inst& I, int i, unsigned* cnt, const double* part, int stride,
                                 double (&tot)[NV])
{
    return last_reduce<NV>(i, I.tile0, I.ntiles, cnt, part, stride, tot);
}


// ------------------------------------------------------------------ inner iteration kernels
// q = A p for every row of every active system, and the p.q partial sums.  A warp holds 32
// consecutive rows, so of the three columns dx = -1, 0, +1 of a stencil line only dx = 0 is
// loaded: the other two come from the neighbouring lanes (lanes 0 and 31 load their outer
// value), a third of the vector traffic of one load per band.
template <int R, int NB>
__global__ void __launch_bounds__(kTile, 3) k_b_spmv(const Inst* __restrict__ insts, const Unit* __restrict__ units,
                                                  int64_t nunits, const int* __restrict__ inst_active,
                                                  const float* __restrict__ p, float* __restrict__ q,
                                                  double* __restrict__ part, unsigned* __restrict__ cnt,
                                                  Rhs* __restrict__ st)
{
    constexpr int NL = NB / 3;  // stencil lines (dy, dz)
    const int lane = threadIdx.x & 31;
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const int i = un.x;
        if (!inst_active[i]) continue;
        const Inst& I = insts[i];
        const int64_t n = I.n;
        int64_t off[NL];
#pragma unroll
        for (int g = 0; g < NL; ++g) off[g] = I.off[3 * g + 1];
        const float* pv = p + I.voff * R;
        float vf[R];  // per-thread partial over the unit's rows (at most 8 terms)
#pragma unroll
        for (int r = 0; r < R; ++r) vf[r] = 0.f;
        for (int k = 0; k < un.z; ++k) {
            const int64_t lt = un.y + k - I.tile0;
            const int64_t row = lt * kTile + threadIdx.x;
            float acc[R], self[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = self[r] = 0.f;
            const float* bt = I.band + lt * NB * kTile + threadIdx.x;
#pragma unroll
            for (int g = 0; g < NL; ++g) {
                const float am = __ldcs(bt + (3 * g) * kTile);
                const float a0 = __ldcs(bt + (3 * g + 1) * kTile);
                const float ap = __ldcs(bt + (3 * g + 2) * kTile);
                const int64_t c = row + off[g];
                const int64_t j = c < 0 ? 0 : (c >= n ? n - 1 : c);  // absent neighbours have a == 0
                float w[R], lv[R], rv[R];
                Vec<R>::ld(pv + j * R, w);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    lv[r] = __shfl_up_sync(0xffffffffu, w[r], 1);
                    rv[r] = __shfl_down_sync(0xffffffffu, w[r], 1);
                }
                if (lane == 0) {
                    const int64_t jl = c - 1 < 0 ? 0 : (c - 1 >= n ? n - 1 : c - 1);
                    Vec<R>::ld(pv + jl * R, lv);
                }
                if (lane == 31) {
                    const int64_t jr = c + 1 < 0 ? 0 : (c + 1 >= n ? n - 1 : c + 1);
                    Vec<R>::ld(pv + jr * R, rv);
                }
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] = fmaf(am, lv[r], fmaf(a0, w[r], fmaf(ap, rv[r], acc[r])));
                if (g == NL / 2)
#pragma unroll
                    for (int r = 0; r < R; ++r) self[r] = w[r];
            }
            if (row < n) {
                Vec<R>::st(q + (I.voff + row) * R, acc);
#pragma unroll
                for (int r = 0; r < R; ++r) vf[r] = fmaf(self[r], acc[r], vf[r]);
            }
        }
        double v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = vf[r];
        block_sum_to<R>(v, part + u * 2 * R);
        double tot[R];
        if (last_reduce<R>(i, u - un.w, I.nunits, cnt, part, 2 * R, tot) && threadIdx.x < R) {
            Rhs& s = st[i * R + threadIdx.x];
            if (s.active) {
                const double pq = tot[threadIdx.x];
                s.pq = pq;
                if (!(pq > 0.0)) {
                    s.breakdown = 1;
                    s.alpha = 0.0;
                } else {
                    s.alpha = s.rz / pq;
                }
            }
        }
    }
}

// The same product with two consecutive rows per thread (kTile/2 threads per tile): a
// thread loads p at its two rows, the outer neighbours come from the adjacent lanes, so a
// stencil line costs one shuffle per right hand side and direction for two rows instead
// of one (the shuffles share the load/store pipe with the loads).
constexpr int kPairThreads = kTile / 2;

template <int R, int NB>
__global__ void __launch_bounds__(kPairThreads, 4)
    k_b_spmv2(const Inst* __restrict__ insts, const Unit* __restrict__ units, int64_t nunits,
              const int* __restrict__ inst_active, const float* __restrict__ p, float* __restrict__ q,
              double* __restrict__ part, unsigned* __restrict__ cnt, Rhs* __restrict__ st)
{
    constexpr int NL = NB / 3;
    const int lane = threadIdx.x & 31;
    const int t2 = 2 * threadIdx.x;  // the thread's first row within the tile
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const int i = un.x;
        if (!inst_active[i]) continue;
        const Inst& I = insts[i];
        const int64_t n = I.n;
        int off[NL];
#pragma unroll
        for (int g = 0; g < NL; ++g) off[g] = (int)I.off[3 * g + 1];
        const float* pv = p + I.voff * R;
        float vf[R];
#pragma unroll
        for (int r = 0; r < R; ++r) vf[r] = 0.f;
        for (int k = 0; k < un.z; ++k) {
            const int64_t lt = un.y + k - I.tile0;
            const int64_t row = lt * kTile + t2;
            float acc0[R], acc1[R], self0[R], self1[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc0[r] = acc1[r] = self0[r] = self1[r] = 0.f;
            const float* bt = I.band + lt * NB * kTile + t2;
#pragma unroll
            for (int g = 0; g < NL; ++g) {
                const float2 am = __ldcs(reinterpret_cast<const float2*>(bt + (3 * g) * kTile));
                const float2 a0 = __ldcs(reinterpret_cast<const float2*>(bt + (3 * g + 1) * kTile));
                const float2 ap = __ldcs(reinterpret_cast<const float2*>(bt + (3 * g + 2) * kTile));
                const int64_t c = row + off[g];  // the first row's centre column
                const int64_t j0 = c < 0 ? 0 : (c >= n ? n - 1 : c);
                const int64_t j1 = c + 1 < 0 ? 0 : (c + 1 >= n ? n - 1 : c + 1);
                float w0[R], w1[R], lv[R], rv[R];
                Vec<R>::ld(pv + j0 * R, w0);
                Vec<R>::ld(pv + j1 * R, w1);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    lv[r] = __shfl_up_sync(0xffffffffu, w1[r], 1);    // column c - 1
                    rv[r] = __shfl_down_sync(0xffffffffu, w0[r], 1);  // column c + 2
                }
                if (lane == 0) {
                    const int64_t jl = c - 1 < 0 ? 0 : (c - 1 >= n ? n - 1 : c - 1);
                    Vec<R>::ld(pv + jl * R, lv);
                }
                if (lane == 31) {
                    const int64_t jr = c + 2 < 0 ? 0 : (c + 2 >= n ? n - 1 : c + 2);
                    Vec<R>::ld(pv + jr * R, rv);
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    acc0[r] = fmaf(am.x, lv[r], fmaf(a0.x, w0[r], fmaf(ap.x, w1[r], acc0[r])));
                    acc1[r] = fmaf(am.y, w0[r], fmaf(a0.y, w1[r], fmaf(ap.y, rv[r], acc1[r])));
                }
                if (g == NL / 2)
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        self0[r] = w0[r];
                        self1[r] = w1[r];
                    }
            }
            if (row < n) {
                Vec<R>::st(q + (I.voff + row) * R, acc0);
#pragma unroll
                for (int r = 0; r < R; ++r) vf[r] = fmaf(self0[r], acc0[r], vf[r]);
            }
            if (row + 1 < n) {
                Vec<R>::st(q + (I.voff + row + 1) * R, acc1);
#pragma unroll
                for (int r = 0; r < R; ++r) vf[r] = fmaf(self1[r], acc1[r], vf[r]);
            }
        }
        double v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = vf[r];
        block_sum_to<R, kPairThreads>(v, part + u * 2 * R);
        double tot[R];
        if (last_reduce<R, kPairThreads>(i, u - un.w, I.nunits, cnt, part, 2 * R, tot) && threadIdx.x < R) {
            Rhs& s = st[i * R + threadIdx.x];
            if (s.active) {
                const double pq = tot[threadIdx.x];
                s.pq = pq;
                if (!(pq > 0.0)) {
                    s.breakdown = 1;
                    s.alpha = 0.0;
                } else {
                    s.alpha = s.rz / pq;
                }
            }
        }
    }
}

// d += alpha p, r -= alpha q, z = dinv r; partial r.z and r.r; the last CTA of a system
// sets beta and pauses right hand sides that met their segment target or stagnated
template <int R>
__global__ void __launch_bounds__(kTile, 3) k_b_update(const Inst* __restrict__ insts, const Unit* __restrict__ units,
                                                    int64_t nunits, int* __restrict__ inst_active,
                                                    const float* __restrict__ p, const float* __restrict__ q,
                                                    float* __restrict__ r32, float* __restrict__ d32,
                                                    double* __restrict__ part, unsigned* __restrict__ cnt,
                                                    Rhs* __restrict__ st, int* __restrict__ nactive, int maxit)
{
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const int i = un.x;
        if (!inst_active[i]) continue;
        const Inst& I = insts[i];
        __shared__ float alpha[8];
        __shared__ int act[8];
        if (threadIdx.x < R) {
            const Rhs& s = st[i * R + threadIdx.x];
            act[threadIdx.x] = s.active && !s.breakdown;
            alpha[threadIdx.x] = (float)s.alpha;
        }
        __syncthreads();
        float vf[2 * R];  // per-thread partials over the unit's rows (at most 8 terms)
#pragma unroll
        for (int r = 0; r < 2 * R; ++r) vf[r] = 0.f;
        for (int k = 0; k < un.z; ++k) {
            const int64_t row = (un.y + k - I.tile0) * kTile + threadIdx.x;
            if (row < I.n) {
                const int64_t o = (I.voff + row) * R;
                float pv[R], qv[R], rv[R], dv[R];
                Vec<R>::ld(p + o, pv);
                Vec<R>::ld(q + o, qv);
                Vec<R>::ld(r32 + o, rv);
                Vec<R>::ld(d32 + o, dv);
                const float di = I.dinv32[row];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (act[r]) {
                        dv[r] = fmaf(alpha[r], pv[r], dv[r]);
                        rv[r] = fmaf(-alpha[r], qv[r], rv[r]);
                    }
                    const float z = di * rv[r];
                    vf[r] = fmaf(rv[r], z, vf[r]);
                    vf[R + r] = fmaf(rv[r], rv[r], vf[R + r]);
                }
                Vec<R>::st(r32 + o, rv);
                Vec<R>::st(d32 + o, dv);
            }
        }
        double v[2 * R];
#pragma unroll
        for (int r = 0; r < 2 * R; ++r) v[r] = vf[r];
        block_sum_to<2 * R>(v, part + u * 2 * R);
        double tot[2 * R];
        if (last_reduce<2 * R>(i, u - un.w, I.nunits, cnt, part, 2 * R, tot)) {
            __shared__ int any;
            if (threadIdx.x == 0) any = 0;
            __syncthreads();
            if (threadIdx.x < R) {
                Rhs& s = st[i * R + threadIdx.x];
                if (s.active) {
                    const double rz = tot[threadIdx.x];
                    const double nrm = sqrt(tot[R + threadIdx.x]);
                    s.iters += 1;
                    bool stop = false;
                    if (s.breakdown || !(rz > 0.0) || !(nrm == nrm)) {
                        s.breakdown = 1;
                        stop = true;
                    } else {
                        s.beta = rz / s.rz;
                        s.rz = rz;
                        s.norm = nrm;
                        if (nrm < 0.95 * s.best) {
                            s.best = nrm;
                            s.since = 0;
                        } else {
                            s.since += 1;
                        }
                        stop = nrm <= s.target || s.since > kStagnation || s.iters >= maxit;
                    }
                    if (stop) {
                        s.active = 0;
                        atomicSub(nactive, 1);
                    } else {
                        atomicOr(&any, 1);
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) inst_active[i] = any;
        }
        __syncthreads();
    }
}

// p = dinv r + beta p for the active right hand sides
template <int R>
__global__ void __launch_bounds__(kTile) k_b_pupdate(const Inst* __restrict__ insts, const Unit* __restrict__ units,
                                                     int64_t nunits, const int* __restrict__ inst_active,
                                                     float* __restrict__ p, const float* __restrict__ r32,
                                                     const Rhs* __restrict__ st)
{
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit un = units[u];
        const int i = un.x;
        if (!inst_active[i]) continue;
        const Inst& I = insts[i];
        __shared__ float beta[8];
        __shared__ int act[8];
        if (threadIdx.x < R) {
            const Rhs& s = st[i * R + threadIdx.x];
            act[threadIdx.x] = s.active;
            beta[threadIdx.x] = (float)s.beta;
        }
        __syncthreads();
        for (int k = 0; k < un.z; ++k) {
            const int64_t row = (un.y + k - I.tile0) * kTile + threadIdx.x;
            if (row < I.n) {
                const int64_t o = (I.voff + row) * R;
                float pv[R], rv[R];
                Vec<R>::ld(p + o, pv);
                Vec<R>::ld(r32 + o, rv);
                const float di = I.dinv32[row];
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (act[r]) pv[r] = fmaf(beta[r], pv[r], di * rv[r]);
                Vec<R>::st(p + o, pv);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ segment and outer kernels
// seed the FP32 recursion of every right hand side that is still running from the FP64
// residual: r32 = r64 / scale, d = 0 (p = 0 for a fresh start); last CTA: rz, norm, target,
// active, and beta for the search direction (k_b_pupdate follows): 0 when fresh, else
// rescaled to the new residual, beta' = beta rz'/rz, so the Krylov space is kept
template <int R>
__global__ void __launch_bounds__(kTile) k_b_seed(const Inst* __restrict__ insts, const int* __restrict__ tile_inst,
                                                  int64_t ntiles, int* __restrict__ inst_active,
                                                  const double* __restrict__ r64, float* __restrict__ r32,
                                                  float* __restrict__ d32, float* __restrict__ p,
                                                  double* __restrict__ part, unsigned* __restrict__ cnt,
                                                  Rhs* __restrict__ st, int* __restrict__ nactive)
{
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tile_inst[t];
        const Inst& I = insts[i];
        __shared__ float isc[8];
        __shared__ int run[8], fresh[8];
        if (threadIdx.x < R) {
            const Rhs& s = st[i * R + threadIdx.x];
            run[threadIdx.x] = s.active;  // host marks the right hand sides to run
            fresh[threadIdx.x] = s.fresh;
            isc[threadIdx.x] = (float)s.inv_scale;
        }
        __syncthreads();
        const int64_t row = (t - I.tile0) * kTile + threadIdx.x;
        double v[2 * R];
#pragma unroll
        for (int r = 0; r < 2 * R; ++r) v[r] = 0.0;
        if (row < I.n) {
            const int64_t o = (I.voff + row) * R;
            float rv[R], dv[R], pv[R];
            const float di = I.dinv32[row];
            Vec<R>::ld(p + o, pv);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                rv[r] = run[r] ? (float)(r64[o + r] * (double)isc[r]) : 0.f;
                dv[r] = 0.f;
                if (!run[r] || fresh[r]) pv[r] = 0.f;
                v[r] = (double)rv[r] * (di * rv[r]);
                v[R + r] = (double)rv[r] * rv[r];
            }
            Vec<R>::st(r32 + o, rv);
            Vec<R>::st(d32 + o, dv);
            Vec<R>::st(p + o, pv);
        }
        block_sum_to<2 * R>(v, part + t * 2 * R);
        double tot[2 * R];
        if (last_tile_reduce<2 * R>(I, i, cnt, part, 2 * R, tot)) {
            __shared__ int any;
            if (threadIdx.x == 0) any = 0;
            __syncthreads();
            if (threadIdx.x < R) {
                Rhs& s = st[i * R + threadIdx.x];
                if (s.active) {
                    const double rz = tot[threadIdx.x];
                    s.beta = (s.fresh || !(s.rz > 0.0)) ? 0.0 : s.beta * (rz / s.rz);
                    s.rz = rz;
                    s.norm = sqrt(tot[R + threadIdx.x]);
                    s.best = s.norm;
                    s.since = 0;
                    s.breakdown = 0;
                    s.target = fmax(s.need, s.seg * s.norm);
                    s.alpha = 0.0;
                    if (s.norm > s.target && s.rz > 0.0) {
                        atomicAdd(nactive, 1);
                        atomicOr(&any, 1);
                    } else {
                        s.active = 0;
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) inst_active[i] = any;
        }
    }
}

// x64 += d32 / inv_scale (all rows of all systems)
template <int R>
__global__ void __launch_bounds__(kTile) k_b_add_correction(const Inst* __restrict__ insts,
                                                            const int* __restrict__ tile_inst, int64_t ntiles,
                                                            const float* __restrict__ d32, double* __restrict__ x64,
                                                            const Rhs* __restrict__ st)
{
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tile_inst[t];
        const Inst& I = insts[i];
        const int64_t row = (t - I.tile0) * kTile + threadIdx.x;
        if (row < I.n) {
            const int64_t o = (I.voff + row) * R;
#pragma unroll
            for (int r = 0; r < R; ++r) x64[o + r] += (double)d32[o + r] / st[i * R + r].inv_scale;
        }
    }
}

// r64 = bb - A x64 with the balanced FP64 CSR (8 lanes per row), norms per right hand side
template <int R>
__global__ void __launch_bounds__(kTile) k_b_residual(const Inst* __restrict__ insts,
                                                      const int* __restrict__ tile_inst, int64_t ntiles,
                                                      const double* __restrict__ x64, const double* __restrict__ bb,
                                                      double* __restrict__ r64, double* __restrict__ part,
                                                      unsigned* __restrict__ cnt, Rhs* __restrict__ st)
{
    constexpr int kL = 8;
    const int lane = threadIdx.x & (kL - 1);
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tile_inst[t];
        const Inst& I = insts[i];
        double v[2 * R];
#pragma unroll
        for (int r = 0; r < 2 * R; ++r) v[r] = 0.0;
        // 256 rows per tile, 32 rows per pass of the block
        for (int pass = 0; pass < kTile / (kTile / kL); ++pass) {
            const int64_t row = (t - I.tile0) * kTile + pass * (kTile / kL) + threadIdx.x / kL;
            double acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.0;
            if (row < I.n) {
                for (int32_t k = I.ptr[row] + lane; k < I.ptr[row + 1]; k += kL) {
                    const double a = I.val[k];
                    const double* xj = x64 + (I.voff + I.idx[k]) * R;
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] = fma(a, xj[r], acc[r]);
                }
            }
#pragma unroll
            for (int o = kL / 2; o > 0; o >>= 1)
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
            if (row < I.n && lane == 0) {
                const int64_t o = (I.voff + row) * R;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const double rr = bb[o + r] - acc[r];
                    r64[o + r] = rr;
                    v[r] += rr * rr;
                    v[R + r] = fmax(v[R + r], fabs(rr));
                }
            }
        }
        // block: sums of v[0..R), maxima of v[R..2R)
        __shared__ double sh[kTile / 32][2 * R];
        const int wl = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
                v[R + r] = fmax(v[R + r], __shfl_xor_sync(0xffffffffu, v[R + r], o));
            }
        if (wl == 0)
#pragma unroll
            for (int r = 0; r < 2 * R; ++r) sh[wid][r] = v[r];
        __syncthreads();
        if (threadIdx.x < 2 * R) {
            double a = sh[0][threadIdx.x];
            for (int w = 1; w < kTile / 32; ++w)
                a = threadIdx.x < R ? a + sh[w][threadIdx.x] : fmax(a, sh[w][threadIdx.x]);
            part[t * 2 * R + threadIdx.x] = a;
        }
        __syncthreads();
        __shared__ bool last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) last = atomicAdd(&cnt[i], 1u) == (unsigned)(I.ntiles - 1);
        __syncthreads();
        if (last) {
            __threadfence();
            if (threadIdx.x < 2 * R) {
                double a = 0.0;
                for (int64_t k = 0; k < I.ntiles; ++k) {
                    const double pv = __ldcg(part + (I.tile0 + k) * 2 * R + threadIdx.x);
                    a = threadIdx.x < R ? a + pv : fmax(a, pv);
                }
                Rhs& s = st[i * R + (threadIdx.x % R)];
                if (threadIdx.x < R) s.n2r = sqrt(a);
                else s.nmr = a;
            }
            if (threadIdx.x == 0) cnt[i] = 0u;
        }
        __syncthreads();
    }
}

// bb = B rhs (balanced, interleaved) from the callers' per-system column-major arrays, and
// the norms of bb per right hand side (written into n2b/nmb through the residual kernel's
// reduction scheme: r64 = bb, x = 0)
template <int R>
__global__ void __launch_bounds__(kTile) k_b_gather(const Inst* __restrict__ insts, const int* __restrict__ tile_inst,
                                                    int64_t ntiles, const double* const* __restrict__ user,
                                                    double* __restrict__ bb, double* __restrict__ x64,
                                                    double* __restrict__ r64)
{
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tile_inst[t];
        const Inst& I = insts[i];
        const int64_t row = (t - I.tile0) * kTile + threadIdx.x;
        if (row < I.n) {
            const int64_t o = (I.voff + row) * R;
            const double b = I.bv[row];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double v = b * user[i][r * I.n + row];
                bb[o + r] = v;
                r64[o + r] = v;
                x64[o + r] = 0.0;
            }
        }
    }
}

// x_user = B x64 (unbalanced), column-major per system
template <int R>
__global__ void __launch_bounds__(kTile) k_b_scatter(const Inst* __restrict__ insts, const int* __restrict__ tile_inst,
                                                     int64_t ntiles, const double* __restrict__ x64,
                                                     double* const* __restrict__ user)
{
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tile_inst[t];
        const Inst& I = insts[i];
        const int64_t row = (t - I.tile0) * kTile + threadIdx.x;
        if (row < I.n) {
            const int64_t o = (I.voff + row) * R;
            const double b = I.bv[row];
#pragma unroll
            for (int r = 0; r < R; ++r) user[i][r * I.n + row] = b * x64[o + r];
        }
    }
}

__global__ void k_b_fill(double* __restrict__ p, int64_t n, double v)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// ------------------------------------------------------------------ host side
double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

bool graphs_wanted()
{
    const char* e = std::getenv("RG_GRAPHS");
    return !(e && e[0] == '0') && !timers_on();
}

template <int R>
int iter_step(Batch* b)
{
    const int nb = b->dim == 3 ? 27 : 9;
#define RG_B_SPMV(KERNEL, NBANDS, THREADS)                                                               \
    RG_TIMED(T_BATCH_SPMV, (KERNEL<<<b->grid_spmv, THREADS, 0, stream()>>>(                                 \
                               b->d_inst, b->d_units, b->nunits, b->d_inst_active, b->p, b->q, b->d_part, \
                               b->d_cnt, b->d_rhs)))
    if (b->spmv_kind == 1) {
        if (nb == 27) RG_B_SPMV((k_b_spmv2<R, 27>), 27, kPairThreads);
        else RG_B_SPMV((k_b_spmv2<R, 9>), 9, kPairThreads);
    } else {
        if (nb == 27) RG_B_SPMV((k_b_spmv<R, 27>), 27, kTile);
        else RG_B_SPMV((k_b_spmv<R, 9>), 9, kTile);
    }
#undef RG_B_SPMV
    RG_CHECK_LAUNCH();
    RG_TIMED(T_BATCH_UPDATE, (k_b_update<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                 b->d_inst, b->d_units, b->nunits, b->d_inst_active, b->p, b->q, b->r32, b->d32,
                                 b->d_part, b->d_cnt, b->d_rhs, b->d_nactive, b->maxit)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_BATCH_UPDATE, (k_b_pupdate<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                 b->d_inst, b->d_units, b->nunits, b->d_inst_active, b->p, b->r32, b->d_rhs)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

}  // namespace batch
}  // namespace rg

namespace rg {
namespace batch {

template <int R>
int launch_seed(Batch* b)
{
    RG_TIMED(T_BATCH_OUTER, (k_b_seed<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                b->d_inst, b->d_tile_inst, b->ntiles, b->d_inst_active, b->r64, b->r32, b->d32, b->p,
                                b->d_part, b->d_cnt, b->d_rhs, b->d_nactive)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_BATCH_UPDATE, (k_b_pupdate<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                 b->d_inst, b->d_units, b->nunits, b->d_inst_active, b->p, b->r32, b->d_rhs)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

template <int R>
int launch_outer(Batch* b)
{
    RG_TIMED(T_BATCH_OUTER, (k_b_add_correction<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                b->d_inst, b->d_tile_inst, b->ntiles, b->d32, b->x64, b->d_rhs)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_BATCH_OUTER, (k_b_residual<R><<<b->grid_upd, kTile, 0, stream()>>>(
                                b->d_inst, b->d_tile_inst, b->ntiles, b->x64, b->bb64, b->r64, b->d_part, b->d_cnt,
                                b->d_rhs)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int step(Batch* b)
{
    switch (b->R) {
    case 1: return iter_step<1>(b);
    case 2: return iter_step<2>(b);
    case 4: return iter_step<4>(b);
    default: return iter_step<8>(b);
    }
}

int seed(Batch* b)
{
    RG_CHECK_CUDA(cudaMemsetAsync(b->d_nactive, 0, sizeof(int), stream()));
    switch (b->R) {
    case 1: return launch_seed<1>(b);
    case 2: return launch_seed<2>(b);
    case 4: return launch_seed<4>(b);
    default: return launch_seed<8>(b);
    }
}

int outer(Batch* b)
{
    switch (b->R) {
    case 1: return launch_outer<1>(b);
    case 2: return launch_outer<2>(b);
    case 4: return launch_outer<4>(b);
    default: return launch_outer<8>(b);
    }
}

int gather(Batch* b, const double* const* rhs)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(b->d_user, rhs, sizeof(double*) * b->ninst, cudaMemcpyHostToDevice, stream()));
    const int g = grid_for(b->ntiles, 1, 8);
    switch (b->R) {
    case 1: k_b_gather<1><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, (const double* const*)b->d_user, b->bb64, b->x64, b->r64); break;
    case 2: k_b_gather<2><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, (const double* const*)b->d_user, b->bb64, b->x64, b->r64); break;
    case 4: k_b_gather<4><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, (const double* const*)b->d_user, b->bb64, b->x64, b->r64); break;
    default: k_b_gather<8><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, (const double* const*)b->d_user, b->bb64, b->x64, b->r64); break;
    }
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int scatter(Batch* b, double* const* x)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(b->d_user, x, sizeof(double*) * b->ninst, cudaMemcpyHostToDevice, stream()));
    const int g = grid_for(b->ntiles, 1, 8);
    double* const* u = b->d_user;
    switch (b->R) {
    case 1: k_b_scatter<1><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, b->x64, u); break;
    case 2: k_b_scatter<2><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, b->x64, u); break;
    case 4: k_b_scatter<4><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, b->x64, u); break;
    default: k_b_scatter<8><<<g, kTile, 0, stream()>>>(b->d_inst, b->d_tile_inst, b->ntiles, b->x64, u); break;
    }
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int read_rhs(Batch* b)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(b->h_rhs.data(), b->d_rhs, sizeof(Rhs) * b->h_rhs.size(), cudaMemcpyDeviceToHost,
                                  stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    return RG_OK;
}

int write_rhs(Batch* b)
{
    RG_CHECK_CUDA(cudaMemcpyAsync(b->d_rhs, b->h_rhs.data(), sizeof(Rhs) * b->h_rhs.size(), cudaMemcpyHostToDevice,
                                  stream()));
    return RG_OK;
}

// iterations until no right hand side is active (or the cap); graph replays of `chunk`
int run_segment(Batch* b, long long cap, long long* launched_iters)
{
    long long it = 0;
    const bool use_graph = graphs_wanted();
    if (use_graph && (!b->graph || b->graph_chunk != b->chunk)) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        long long before[T_COUNT], after[T_COUNT];
        timers_snapshot(before);
        RG_CHECK_CUDA(cudaStreamBeginCapture(stream(), cudaStreamCaptureModeThreadLocal));
        int rc = RG_OK;
        for (int c = 0; c < b->chunk && rc == RG_OK; ++c) rc = step(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream(), &g);
        if (rc) return rc;
        if (e != cudaSuccess) {
            set_error(std::string("batch graph capture: ") + cudaGetErrorString(e));
            return RG_CUDA_ERROR;
        }
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error(std::string("batch graph instantiate: ") + cudaGetErrorString(e));
            return RG_CUDA_ERROR;
        }
        b->graph_chunk = b->chunk;
        timers_snapshot(after);
        long long undo[T_COUNT];
        for (int k = 0; k < T_COUNT; ++k) {
            b->graph_launches[k] = after[k] - before[k];
            undo[k] = before[k] - after[k];
        }
        timers_add(undo, 1);
    }
    for (;;) {
        if (use_graph) {
            RG_CHECK_CUDA(cudaGraphLaunch(b->graph, stream()));
            timers_add(b->graph_launches, 1);
        } else {
            for (int c = 0; c < b->chunk; ++c) {
                int rc = step(b);
                if (rc) return rc;
            }
        }
        it += b->chunk;
        RG_CHECK_CUDA(cudaMemcpyAsync(b->h_nactive, b->d_nactive, sizeof(int), cudaMemcpyDeviceToHost, stream()));
        RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
        if (*b->h_nactive <= 0) break;
        if (it > cap + 2 * b->chunk) {
            set_error("batched PCG loop did not terminate");
            return RG_TIMEOUT;
        }
    }
    *launched_iters = it;
    return RG_OK;
}

// time `iters` iterations of the three kernels at the current grid sizes (ms per iteration)
int time_iters(Batch* b, int iters, double* ms)
{
    cudaEvent_t e0, e1;
    RG_CHECK_CUDA(cudaEventCreate(&e0));
    RG_CHECK_CUDA(cudaEventCreate(&e1));
    RG_CHECK_CUDA(cudaEventRecord(e0, stream()));
    int rc = RG_OK;
    for (int k = 0; k < iters && rc == RG_OK; ++k) rc = step(b);
    RG_CHECK_CUDA(cudaEventRecord(e1, stream()));
    RG_CHECK_CUDA(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / iters;
    return rc;
}

// every right hand side active from r = 1 with a target it never reaches (tuning only)
int seed_all_active(Batch* b)
{
    for (auto& s : b->h_rhs) {
        std::memset(&s, 0, sizeof(s));
        s.active = 1;
        s.fresh = 1;
        s.inv_scale = 1.0;
    }
    int rc = write_rhs(b);
    if (rc) return rc;
    k_b_fill<<<grid_for(b->rows * b->R, kTile, 8), kTile, 0, stream()>>>(b->r64, b->rows * b->R, 1.0);
    RG_CHECK_LAUNCH();
    return seed(b);
}

// work units of `group` consecutive tiles per system (the last unit of a system may be short)
int set_group(Batch* b, int group)
{
    std::vector<Unit> units;
    for (int i = 0; i < b->ninst; ++i) {
        Inst& I = b->h_inst[i];
        int w = 0;
        for (int64_t t = 0; t < I.ntiles; t += group, ++w)
            units.push_back(make_int4(i, (int)(I.tile0 + t), (int)std::min<int64_t>(group, I.ntiles - t), w));
        I.nunits = w;
    }
    b->nunits = (int64_t)units.size();
    b->group = group;
    RG_CHECK_CUDA(cudaMemcpyAsync(b->d_units, units.data(), sizeof(Unit) * units.size(), cudaMemcpyHostToDevice,
                                  stream()));
    RG_CHECK_CUDA(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), sizeof(Inst) * b->ninst, cudaMemcpyHostToDevice,
                                  stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));  // the host vectors go out of scope
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return RG_OK;
}

int tune(Batch* b)
{
    // candidates: tiles per work unit x CTAs per SM, the same grid for the three kernels
    // first, then the update kernels' grid on its own
    int rc;
    const int groups[] = {1, 2, 4, 8};
    const int cands[] = {2, 4, 8, 16};
    const int saved_maxit = b->maxit;
    b->maxit = 1 << 30;
    double best = 1e30;
    int best_g = 4, best_s = 8, best_u = 8, best_k = 0;
    for (int kind : {0, 1}) {
        if (b->force_kind >= 0 && kind != b->force_kind) continue;
        b->spmv_kind = kind;
        for (int g : groups) {
            if ((rc = set_group(b, g))) return rc;
            for (int c : cands) {
                if (c > 2 && (int64_t)c * kNumSMs > b->nunits) break;
                b->grid_spmv = b->grid_upd = kNumSMs * c;
                if ((rc = seed_all_active(b))) return rc;
                double ms;
                if ((rc = time_iters(b, 2, &ms))) return rc;  // warm
                if ((rc = time_iters(b, 6, &ms))) return rc;
                if (ms < best) {
                    best = ms;
                    best_g = g;
                    best_s = best_u = c;
                    best_k = kind;
                }
            }
        }
    }
    b->spmv_kind = best_k;
    if ((rc = set_group(b, best_g))) return rc;
    for (int c : cands) {
        if (c == best_s || (c > 2 && (int64_t)c * kNumSMs > b->nunits)) continue;
        b->grid_spmv = kNumSMs * best_s;
        b->grid_upd = kNumSMs * c;
        if ((rc = seed_all_active(b))) return rc;
        double ms;
        if ((rc = time_iters(b, 2, &ms))) return rc;
        if ((rc = time_iters(b, 6, &ms))) return rc;
        if (ms < best) {
            best = ms;
            best_u = c;
        }
    }
    b->grid_spmv = kNumSMs * best_s;
    b->grid_upd = kNumSMs * best_u;
    if ((rc = seed_all_active(b))) return rc;
    double ms;
    if ((rc = time_iters(b, 6, &ms))) return rc;
    b->tuned_iter_us = ms * 1e3;
    // about 2 ms of work per graph replay between polls, 4..64 iterations
    b->chunk = (int)std::min(64.0, std::max(4.0, 2.0 / std::max(ms, 1e-3)));
    b->maxit = saved_maxit;
    b->tuned = true;
    return RG_OK;
}

void destroy(Batch* b)
{
    if (!b) return;
    cudaFree(b->d_inst);
    cudaFree(b->d_tile_inst);
    cudaFree(b->d_units);
    cudaFree(b->d_inst_active);
    cudaFree(b->d_nactive);
    cudaFreeHost(b->h_nactive);
    cudaFree(b->d_rhs);
    cudaFree(b->d_cnt);
    cudaFree(b->d_part);
    cudaFree(b->p);
    cudaFree(b->q);
    cudaFree(b->r32);
    cudaFree(b->d32);
    cudaFree(b->x64);
    cudaFree(b->bb64);
    cudaFree(b->r64);
    cudaFree(b->d_user);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->priv) cudaStreamDestroy(b->priv);
    if (b->ev_in) cudaEventDestroy(b->ev_in);
    if (b->ev_out) cudaEventDestroy(b->ev_out);
    delete b;
}

}  // namespace batch
}  // namespace rg

struct rg_batch {
    rg::batch::Batch b;
};

using namespace rg;
using namespace rg::batch;

namespace {

struct OnPrivate {
    cudaStream_t caller;
    Batch* b;
    OnPrivate(Batch* bb) : caller(stream()), b(bb)
    {
        cudaEventRecord(b->ev_in, caller);
        cudaStreamWaitEvent(b->priv, b->ev_in, 0);
        set_stream(b->priv);
    }
    ~OnPrivate()
    {
        cudaEventRecord(b->ev_out, b->priv);
        cudaStreamWaitEvent(caller, b->ev_out, 0);
        set_stream(caller);
    }
};

}  // namespace

extern "C" {

int rg_batch_create(rg_matrix* const* mats, int ninst, int nrhs, rg_batch** out)
{
    RG_REQUIRE(mats && out && ninst > 0, "rg_batch_create: invalid argument");
    RG_REQUIRE(nrhs == 1 || nrhs == 2 || nrhs == 4 || nrhs == 8, "rg_batch_create: nrhs must be 1, 2, 4 or 8");
    *out = nullptr;
    rg_batch* h = new rg_batch();
    Batch* b = &h->b;
    b->ninst = ninst;
    b->R = nrhs;
    int rc = RG_OK;
    auto fail = [&](int code) {
        destroy(b);
        return code;
    };
    for (int i = 0; i < ninst; ++i) {
        if (!mats[i]) {
            set_error("rg_batch_create: NULL matrix");
            return fail(RG_INVALID_ARG);
        }
        Matrix* m = &mats[i]->m;
        const Domain* d = m->dom;
        if (m->nb != 1) {
            set_error("rg_batch_create: PDE systems (block size > 1) are not supported in batches");
            return fail(RG_NOT_SUPPORTED);
        }
        if (i == 0) b->dim = d->dim;
        if (d->dim != b->dim) {
            set_error("rg_batch_create: all systems must have the same dimension");
            return fail(RG_INVALID_ARG);
        }
        if ((rc = solver_prepare(m, true))) return fail(rc);
        Inst I{};
        I.n = d->n;
        I.tile0 = b->ntiles;
        I.ntiles = (d->n + kTile - 1) / kTile;
        I.voff = b->rows;
        I.nbands = d->nbands;
        for (int k = 0; k < d->nbands; ++k) I.off[k] = d->band_off[k];
        I.band = m->band32;
        I.dinv32 = m->dinv32;
        I.ptr = d->ptr;
        I.idx = d->idx;
        I.val = m->val;
        I.bv = m->bv;
        b->h_inst.push_back(I);
        b->mats.push_back(m);
        b->ntiles += I.ntiles;
        b->rows += I.ntiles * kTile;
    }
    const size_t nv = (size_t)b->rows * b->R;
    std::vector<int> tile_inst((size_t)b->ntiles);
    for (int i = 0; i < ninst; ++i)
        for (int64_t t = 0; t < b->h_inst[i].ntiles; ++t) tile_inst[(size_t)(b->h_inst[i].tile0 + t)] = i;
    b->h_rhs.assign((size_t)ninst * b->R, Rhs{});
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 1);
    };
    A((void**)&b->d_inst, sizeof(Inst) * ninst);
    A((void**)&b->d_tile_inst, sizeof(int) * b->ntiles);
    A((void**)&b->d_units, sizeof(Unit) * b->ntiles);
    A((void**)&b->d_inst_active, sizeof(int) * ninst);
    A((void**)&b->d_nactive, sizeof(int));
    A((void**)&b->d_rhs, sizeof(Rhs) * b->h_rhs.size());
    A((void**)&b->d_cnt, sizeof(unsigned) * ninst);
    A((void**)&b->d_part, sizeof(double) * b->ntiles * 2 * b->R);
    A((void**)&b->p, sizeof(float) * nv);
    A((void**)&b->q, sizeof(float) * nv);
    A((void**)&b->r32, sizeof(float) * nv);
    A((void**)&b->d32, sizeof(float) * nv);
    A((void**)&b->x64, sizeof(double) * nv);
    A((void**)&b->bb64, sizeof(double) * nv);
    A((void**)&b->r64, sizeof(double) * nv);
    A((void**)&b->d_user, sizeof(double*) * ninst);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_nactive, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->priv, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        set_error(std::string("rg_batch_create: ") + cudaGetErrorString(e));
        return fail(RG_CUDA_ERROR);
    }
    {
        OnPrivate on(b);
        e = cudaMemcpyAsync(b->d_inst, b->h_inst.data(), sizeof(Inst) * ninst, cudaMemcpyHostToDevice, stream());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->d_tile_inst, tile_inst.data(), sizeof(int) * b->ntiles, cudaMemcpyHostToDevice,
                                stream());
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_cnt, 0, sizeof(unsigned) * ninst, stream());
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_inst_active, 0, sizeof(int) * ninst, stream());
        // padding rows stay zero in every vector
        float* fv[] = {b->p, b->q, b->r32, b->d32};
        for (float* v : fv)
            if (e == cudaSuccess) e = cudaMemsetAsync(v, 0, sizeof(float) * nv, stream());
        double* dv[] = {b->x64, b->bb64, b->r64};
        for (double* v : dv)
            if (e == cudaSuccess) e = cudaMemsetAsync(v, 0, sizeof(double) * nv, stream());
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    }
    if (e != cudaSuccess) {
        set_error(std::string("rg_batch_create: ") + cudaGetErrorString(e));
        return fail(RG_CUDA_ERROR);
    }
    {
        OnPrivate on(b);
        rc = set_group(b, 4);
        if (rc) return fail(rc);
    }
    b->grid_spmv = b->grid_upd = grid_for(b->nunits, 1, 8);
    *out = h;
    return RG_OK;
}

int rg_batch_destroy(rg_batch* h)
{
    if (h) destroy(&h->b);
    return RG_OK;
}

int rg_batch_info(const rg_batch* h, int64_t* rows, int64_t* tiles, int* group, int* grid_spmv, int* grid_update,
                  int* chunk, double* iter_us, int* spmv_kernel)
{
    RG_REQUIRE(h, "rg_batch_info: NULL batch");
    const Batch* b = &h->b;
    if (rows) *rows = b->rows;
    if (tiles) *tiles = b->ntiles;
    if (group) *group = b->group;
    if (grid_spmv) *grid_spmv = b->grid_spmv;
    if (grid_update) *grid_update = b->grid_upd;
    if (chunk) *chunk = b->chunk;
    if (iter_us) *iter_us = b->tuned_iter_us;
    if (spmv_kernel) *spmv_kernel = b->spmv_kind;
    return RG_OK;
}

int rg_batch_set_spmv(rg_batch* h, int spmv_kernel)
{
    RG_REQUIRE(h, "rg_batch_set_spmv: NULL batch");
    RG_REQUIRE(spmv_kernel >= -1 && spmv_kernel <= 1, "rg_batch_set_spmv: spmv_kernel must be -1, 0 or 1");
    h->b.force_kind = spmv_kernel;
    h->b.tuned = false;  // the next solve (or rg_batch_tune) tunes within the choice
    return RG_OK;
}

int rg_batch_tune(rg_batch* h)
{
    RG_REQUIRE(h, "rg_batch_tune: NULL batch");
    Batch* b = &h->b;
    OnPrivate on(b);
    int rc = tune(b);
    if (rc) return rc;
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    return RG_OK;
}

int rg_batch_solve(rg_batch* h, const double* const* rhs, double* const* x, const rg_solver_opts* opts,
                   rg_diag* diag)
{
    RG_REQUIRE(h && rhs && x, "rg_batch_solve: NULL argument");
    Batch* b = &h->b;
    rg_solver_opts def;
    rg_solver_opts_default(&def);
    const rg_solver_opts* o = opts ? opts : &def;
    const double EPS = 2.220446049250313e-16;
    RG_REQUIRE(o->method == RG_METHOD_PCG && o->preconditioner == RG_PRECOND_JACOBI,
               "rg_batch_solve: only PCG with the Jacobi preconditioner is implemented");
    RG_REQUIRE(o->tolerance >= 100. * EPS && o->tolerance <= 1., "rg_batch_solve: tolerance out of range");
    RG_REQUIRE(o->initial_guess == nullptr, "rg_batch_solve: initial guesses are not supported for batches");
    for (int i = 0; i < b->ninst; ++i)
        RG_REQUIRE(b->mats[i]->balanced && b->mats[i]->solver_ready && b->mats[i]->band32 && b->mats[i]->band32_ok,
                   "rg_batch_solve: a system's values changed after rg_batch_create (recreate the batch)");
    const double t0 = now_s();
    OnPrivate on(b);
    int rc;
    if (!b->tuned && (rc = tune(b))) return rc;
    b->maxit = (int)std::min<int64_t>(o->iter_max, 1 << 30);
    const double seg = std::fmin(std::fmax(o->inner_tolerance > 0 ? o->inner_tolerance : 1e-2, 1e-4), 0.5);
    const int R = b->R, nr = b->ninst * R;
    // norms of B b: the residual pass with x = 0 and no correction
    for (auto& s : b->h_rhs) {
        std::memset(&s, 0, sizeof(s));
        s.inv_scale = 1.0;
    }
    if ((rc = write_rhs(b))) return rc;
    RG_CHECK_CUDA(cudaMemsetAsync(b->d32, 0, sizeof(float) * b->rows * R, stream()));
    if ((rc = gather(b, rhs))) return rc;
    if ((rc = outer(b))) return rc;
    if ((rc = read_rhs(b))) return rc;
    std::vector<int> status(nr, RG_OK);
    std::vector<char> done(nr, 0);
    std::vector<double> last2(nr), lastm(nr);
    std::vector<int> worse(nr, 0);  // consecutive outer steps without improvement
    for (int k = 0; k < nr; ++k) {
        Rhs& s = b->h_rhs[k];
        const double n2r = s.n2r, nmr = s.nmr;
        std::memset(&s, 0, sizeof(s));
        s.n2b = n2r;
        s.nmb = nmr;
        s.n2r = n2r;
        s.nmr = nmr;
        s.inv_scale = nmr > 0 ? 1.0 / nmr : 1.0;
        s.fresh = 1;
        if (std::isnan(n2r) || std::isnan(nmr)) {
            status[k] = RG_NAN;
            done[k] = 1;
        } else if (n2r <= 0.0) {
            done[k] = 1;  // x = 0
        }
        last2[k] = n2r;
        lastm[k] = nmr;
    }
    long long outer_steps = 0;
    for (;;) {
        int running = 0;
        for (int k = 0; k < nr; ++k) {
            Rhs& s = b->h_rhs[k];
            s.active = done[k] ? 0 : 1;
            if (!done[k]) {
                ++running;
                s.need = 0.5 * o->tolerance * std::fmin(s.n2b, 0.1 * s.n2r / s.nmr * s.nmb) * s.inv_scale;
                s.seg = seg;
            }
        }
        if (!running) break;
        if ((rc = write_rhs(b))) return rc;
        if ((rc = seed(b))) return rc;
        long long it = 0;
        int64_t maxleft = 0;
        for (int k = 0; k < nr; ++k)
            if (!done[k]) maxleft = std::max<int64_t>(maxleft, o->iter_max - b->h_rhs[k].iters);
        if ((rc = run_segment(b, maxleft, &it))) return rc;
        if ((rc = outer(b))) return rc;
        if ((rc = read_rhs(b))) return rc;
        ++outer_steps;
        for (int k = 0; k < nr; ++k) {
            if (done[k]) continue;
            Rhs& s = b->h_rhs[k];
            if (std::isnan(s.n2r)) {
                status[k] = RG_NAN;
                done[k] = 1;
                continue;
            }
            const bool conv = !(s.n2r > o->tolerance * s.n2b || s.nmr > o->tolerance * s.nmb);
            if (conv) {
                done[k] = 1;
                continue;
            }
            if (s.iters >= o->iter_max) {
                status[k] = RG_MAXITER;
                done[k] = 1;
                continue;
            }
            // paso's divergence test (no improvement in either norm), given three segments:
            // the CG residual is not monotone, and a segment can end on stagnation
            if (s.n2r >= last2[k] && s.nmr >= lastm[k]) {
                if (++worse[k] >= 3) {
                    status[k] = RG_DIVERGENCE;
                    done[k] = 1;
                    continue;
                }
            } else {
                worse[k] = 0;
                last2[k] = s.n2r;
                lastm[k] = s.nmr;
            }
            // a breakdown restarts the search direction
            s.fresh = s.breakdown ? 1 : 0;
        }
    }
    if ((rc = scatter(b, x))) return rc;
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    const double t1 = now_s();
    int worst = RG_OK;
    for (int k = 0; k < nr; ++k) {
        const Rhs& s = b->h_rhs[k];
        if (diag) {
            rg_diag& d = diag[k];
            std::memset(&d, 0, sizeof(d));
            d.num_iter = s.iters;
            d.num_outer = outer_steps;
            d.residual_norm = s.n2r;
            d.residual_max = s.nmr;
            d.rhs_norm = s.n2b;
            d.converged = status[k] == RG_OK;
            d.time = t1 - t0;
            d.net_time = t1 - t0;
        }
        if (status[k] != RG_OK && !(o->accept_convergence_failure &&
                                    (status[k] == RG_MAXITER || status[k] == RG_DIVERGENCE)))
            worst = worst == RG_OK ? status[k] : worst;
    }
    if (worst != RG_OK) set_error("rg_batch_solve: at least one right hand side did not converge (see the diagnostics)");
    return worst;
}

}  // extern "C"
