// Internal declarations shared by the ripley_gpu translation units.
#pragma once
#include <mutex>

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/ripley_gpu.h"

namespace rg {

// ---------------------------------------------------------------- error plumbing
void set_error(const std::string& msg);
void set_stream(cudaStream_t s);
const std::string& last_error();
cudaStream_t stream();

#define RG_CHECK_CUDA(call)                                                          \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            ::rg::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));      \
            return RG_CUDA_ERROR;                                                    \
        }                                                                            \
    } while (0)

#define RG_CHECK_LAUNCH() RG_CHECK_CUDA(cudaGetLastError())

#define RG_REQUIRE(cond, msg)                                                        \
    do {                                                                             \
        if (!(cond)) {                                                               \
            ::rg::set_error(msg);                                                    \
            return RG_INVALID_ARG;                                                   \
        }                                                                            \
    } while (0)

constexpr int kNumSMs = 148;  // B200; grids are sized as multiples of this

// ---------------------------------------------------------------- Q1 tables
// Reference-element data for one domain spacing, passed to kernels by value.
// N[q][k]: shape function k at Gauss point q; G[q][k][d]: its physical gradient;
// W: quadrature weight (equal for all points).  Local node k / point q: bit d is the
// offset along axis d (x fastest).
struct Q1Tables {
    double N[8][8];
    double G[8][8][3];
    double W;
    double Wf[3];  // face quadrature weight for faces normal to axis d
};
void build_q1_tables(int dim, const double dx[3], Q1Tables* t);
void build_q1_reduced_tables(int dim, const double dx[3], Q1Tables* t);

// ---------------------------------------------------------------- handles
struct Workspace;
struct Domain {
    int dim;
    int64_t ne[3], nn[3];  // unused axes hold 1
    double x0[3], x1[3], dx[3];
    int64_t n, nnz;
    int32_t* ptr = nullptr;  // device CSR pattern
    int32_t* idx = nullptr;
    int nbands;              // 27 (3D) or 9 (2D)
    int64_t npad;            // band stride: n rounded up to a multiple of 256
    int64_t band_off[27];    // column offset of band b: dx + NN0*dy + NN0*NN1*dz
    Q1Tables q1;
    Q1Tables q1r;            // 1-point rule of the reduced-order assembly
    int refs = 1;                   // the caller's handle + one per live matrix (rg_capi.cu)
    Workspace* spare_ws = nullptr;  // solver vectors of a destroyed matrix, kept for the next one
    // the value arrays of a destroyed block-size-1 matrix, kept for the next one
    struct Spare {
        double *val = nullptr, *bv = nullptr, *dinv = nullptr, *band64 = nullptr;
        float *band32 = nullptr, *dinv32 = nullptr;
    } spare;
};

struct Workspace;        // solver vectors, allocated lazily (rg_solver.cu)
struct SysWorkspace;     // vectors of the block (PDE system) solver (rg_system.cu)
struct ResidualScratch;  // reduction scratch of rg_residual_norms (rg_residual.cu)

// What the values of a scalar matrix were built from, so that the FP32 inner solve can
// evaluate the operator from the element coefficients instead of streaming stored values
// (RG_LAYOUT_COEF, rg_coef.cu).  Representable: the sum of interior assemblies with A = kappa I
// per element (CONSTANT, PER_ELEMENT, or EXPANDED with the same value at every Gauss point)
// and no B, C, D, followed by at most insertConstraint.  khat is node-indexed: khat[i] =
// kappa of the element whose upper corner is node i (0 where there is no such element), with
// the sign bit set on nodes the constraint fixes; it holds n + NN0 NN1 + NN0 + kCoefPad floats
// so that every element a node touches (i + {0,1} + NN0 {0,1} + NN0 NN1 {0,1}) is in range.
constexpr int64_t kCoefPad = 1024;
struct CoefRecord {
    int state = 0;              // 0: values are zero, 1: khat describes them, -1: not representable
    bool constrained = false;   // a constraint was recorded (a later assembly is not representable)
    float* khat = nullptr;
    int* bad = nullptr;         // set on the device when an element's A is not kappa I with kappa >= 0
};

struct Matrix {
    Domain* dom;
    int nb = 1;                // block size (numEq = numComp of a PDE system; 1 = scalar)
    double* val = nullptr;     // nnz * nb^2 FP64 CSR values (paso mainBlock->val), blocks
                               // column-major: val[k nb^2 + ir + nb ic]
    double* bv = nullptr;      // balance vector
    bool balanced = false;
    // solver data derived from the balanced values (paso's preconditioner data)
    bool solver_ready = false;
    bool band32_ok = false, band64_ok = false;  // band copies hold the current balanced values
    double* dinv = nullptr;    // 1 / balanced diagonal
    float* band32 = nullptr;   // [nbands][npad] FP32 copy of the balanced matrix
    double* band64 = nullptr;  // the same layout in FP64 (paso in FP64 with RG_LAYOUT_BAND)
    int force_spmv = -1;       // FP32 SpMV configuration fixed by the caller (-1: tuned)
    float* dinv32 = nullptr;
    Workspace* ws = nullptr;
    ResidualScratch* rs = nullptr;
    SysWorkspace* sws = nullptr;
    CoefRecord coef;
};

// ---------------------------------------------------------------- deterministic reductions
// Every block writes NV partial sums; the last block to finish (atomic ticket) sums
// the partials in a fixed order, so results do not depend on block scheduling.
struct ReduceBuf {
    double* partials;     // gridDim.x * NV doubles
    unsigned* counter;    // zero between launches
};

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV])
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
}

template <int NV>
__device__ __forceinline__ void warp_max(double (&v)[NV])
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = fmax(v[j], __shfl_xor_sync(0xffffffffu, v[j], o));
}

// Reduces v over the grid.  ISMAX selects which components are max-reductions
// (bit j set) instead of sums.  Returns true in the (single) last block, where
// `out` holds the grid totals for every thread of that block.
template <int NV, unsigned ISMAX = 0u>
__device__ bool grid_reduce(double (&v)[NV], ReduceBuf rb, double (&out)[NV])
{
    __shared__ double sh[32][NV];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    double s[NV], m[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) { s[j] = v[j]; m[j] = v[j]; }
    warp_sum<NV>(s);
    warp_max<NV>(m);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[wid][j] = ((ISMAX >> j) & 1u) ? m[j] : s[j];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double a = sh[0][j];
            for (int w = 1; w < nw; ++w) a = ((ISMAX >> j) & 1u) ? fmax(a, sh[w][j]) : a + sh[w][j];
            rb.partials[(size_t)blockIdx.x * NV + j] = a;
        }
        __threadfence();
        const unsigned t = atomicAdd(rb.counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    // fixed-order pass over the block partials
    double a[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) a[j] = 0.0;  // sums, and maxima of values >= 0
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double pv = __ldcg(rb.partials + (size_t)b * NV + j);
            a[j] = ((ISMAX >> j) & 1u) ? fmax(a[j], pv) : a[j] + pv;
        }
    double s2[NV], m2[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) { s2[j] = a[j]; m2[j] = a[j]; }
    warp_sum<NV>(s2);
    warp_max<NV>(m2);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[wid][j] = ((ISMAX >> j) & 1u) ? m2[j] : s2[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double r = sh[0][j];
        for (int w = 1; w < nw; ++w) r = ((ISMAX >> j) & 1u) ? fmax(r, sh[w][j]) : r + sh[w][j];
        out[j] = r;
    }
    if (threadIdx.x == 0) *rb.counter = 0u;
    return true;
}

// grid sized to a multiple of the SM count, capped by the work
inline int grid_for(int64_t work_items, int items_per_block, int blocks_per_sm = 8)
{
    int64_t g = (work_items + items_per_block - 1) / items_per_block;
    const int64_t cap = (int64_t)kNumSMs * blocks_per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// ---------------------------------------------------------------- kernel timers
// Optional CUDA-event timing of every library kernel launch, grouped by kind, and a
// launch counter that is always on.  Events are recorded on the launching stream.
enum TimerKind {
    T_PATTERN = 0, T_ASSEMBLE, T_BOUNDARY, T_CONSTRAINT, T_SPMV, T_BALANCE, T_NORMS, T_RESIDUAL,
    T_PASO_SPMV, T_PASO_UPDATE1, T_PASO_UPDATE2, T_STD_SPMV, T_STD_UPDATE, T_F32_SPMV,
    T_F32_UPDATE, T_VECTOR, T_BATCH_SPMV, T_BATCH_UPDATE, T_BATCH_OUTER, T_WS_CONV, T_WS_WGRAD, T_WS_OPS, T_COUNT
};
void timer_begin(int kind);
void timer_end(int kind);
void timers_collect();  // folds finished event pairs into the totals (syncs the events)
bool timers_on();
void timers_snapshot(long long out[T_COUNT]);  // launch counters
void timers_add(const long long delta[T_COUNT], long long times);

#define RG_TIMED(kind, launch) \
    do {                       \
        ::rg::timer_begin(kind); \
        launch;                \
        ::rg::timer_end(kind); \
    } while (0)

// ---------------------------------------------------------------- entry points between units
int launch_pattern(Domain* d);
int assemble_single_impl(const Domain* d, double* val, double* rhs, const rg_coef* c[6], bool reduced);
int assemble_boundary_impl(const Domain* d, int nb, bool reduced, double* val, double* rhs, const rg_coef* dc,
                           const rg_coef* yc);
int launch_interpolate(const Domain* d, const double* nodal, int ncomp, double* out, int reduced);
int launch_insert_constraint(Matrix* m, double* rhs, const double* q, const double* r, int rhs_only);
int launch_nullify(Matrix* m, const double* mr, const double* mc, double diag);
int launch_spmv64(const Domain* d, const double* val, double alpha, const double* x, double beta,
                  double* y);
// balance in place (scale=1) and/or derive dinv (+dinv32, + the FP32 band copy when
// want_band) from the current values; *d_bad is set when a diagonal is zero or missing
int launch_balance(Matrix* m, int scale, int* d_bad, bool want_band, bool want_band64);
int solve(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag);
// balance the matrix in place (first time) and build its solver data, the FP32 band copy
// included when `band` (what rg_solve does before iterating)
int solver_prepare(Matrix* m, bool band);
// the FP32 path's tuned configuration (see rg_solver_config)
int solver_config(const Matrix* m, int* spmv_cfg, int* update_grid, double* spmv_us);
// fixes the FP32 SpMV configuration (-1: tune at the next FP32 solve)
int solver_set_config(Matrix* m, int spmv_cfg);
// poll limit of the band kernels' bounded waits (0: default) and whether their producer
// withholds its copies (rg_test_wait_limit)
int set_wait_control(int polls, int withhold);
namespace ws {
// the same test hook for the persistent convolution (ws_conv.cu)
int set_conv_wait_control(int polls, int withhold);
}  // namespace ws
void free_workspace(Matrix* m);
// hands the matrix's solver vectors to its domain for the next matrix there (one is kept; a
// further one is freed), instead of freeing them: a fresh matrix on the same grid then
// solves without device and pinned host allocations
void release_workspace(Matrix* m);
void free_domain_workspace(Domain* d);
std::mutex& pool_mutex();  // guards the domains' spare workspaces and arrays
// PDE systems (rg_system.cu): block size m->nb in {2, 3}
int assemble_system_impl(const Domain* d, int nb, double* val, double* rhs, const rg_coef* c[6], bool reduced);
int launch_system_constraint(Matrix* m, double* rhs, const double* q, const double* r, int rhs_only);
int launch_system_nullify(Matrix* m, const double* mr, const double* mc, double diag);
int launch_system_spmv(const Matrix* m, double alpha, const double* x, double beta, double* y);
int solve_system(Matrix* m, const double* rhs, double* x, const rg_solver_opts* o, rg_diag* diag);
int residual_norms_system(Matrix* m, const double* b, const double* x, double* l2, double* linf);
void free_system_workspace(Matrix* m);
void free_residual_scratch(Matrix* m);
// coefficient record of a scalar matrix (rg_coef.cu)
void coef_reset(Matrix* m);                                                // values zeroed
void coef_invalidate(Matrix* m);                                           // values no longer representable
int coef_on_assemble(Matrix* m, const rg_coef* c[6], bool reduced);        // before an interior assembly
int coef_on_constraint(Matrix* m, const double* q);                        // insertConstraint (not rhs_only)
// whether the record describes the values (reads the device flag: synchronises the stream)
int coef_usable(Matrix* m, bool* usable);
void free_coef(Matrix* m);

}  // namespace rg

struct rg_domain { rg::Domain d; };
struct rg_matrix { rg::Matrix m; };
