// extern "C" entry points of libripley_gpu.so (declared in include/ripley_gpu.h).
// Handles own their device memory; errors are reported as status codes plus a
// thread-local message, never as C++ exceptions across the ABI.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "rg_internal.cuh"

namespace rg {

namespace {
thread_local std::string g_error;
thread_local cudaStream_t g_stream = nullptr;
}  // namespace

void set_error(const std::string& msg) { g_error = msg; }
const std::string& last_error() { return g_error; }
cudaStream_t stream() { return g_stream; }
void set_stream(cudaStream_t s) { g_stream = s; }

}  // namespace rg

using namespace rg;

#define RG_GUARD_BEGIN try {
#define RG_GUARD_END                                      \
    }                                                     \
    catch (const std::bad_alloc&)                         \
    {                                                     \
        set_error("host allocation failed");              \
        return RG_INVALID_ARG;                            \
    }                                                     \
    catch (...)                                           \
    {                                                     \
        set_error("unexpected C++ exception");            \
        return RG_INVALID_ARG;                            \
    }

namespace {

bool coef_ok(const rg_coef* c)
{
    if (!c || c->kind == RG_COEF_EMPTY) return true;
    if (c->kind < RG_COEF_EMPTY || c->kind > RG_COEF_PER_ELEMENT) return false;
    return c->ptr != nullptr;
}

void free_domain(Domain* d)
{
    free_domain_workspace(d);
    {
        Domain::Spare& sp = d->spare;
        if (sp.val) cudaFree(sp.val);
        if (sp.bv) cudaFree(sp.bv);
        if (sp.dinv) cudaFree(sp.dinv);
        if (sp.band32) cudaFree(sp.band32);
        if (sp.dinv32) cudaFree(sp.dinv32);
        if (sp.band64) cudaFree(sp.band64);
        sp = Domain::Spare();
    }
    if (d->ptr) cudaFree(d->ptr);
    if (d->idx) cudaFree(d->idx);
    d->ptr = nullptr;
    d->idx = nullptr;
}

void free_matrix(Matrix* m)
{
    free_coef(m);
    release_workspace(m);
    free_residual_scratch(m);
    free_system_workspace(m);
    if (m->nb == 1 && m->val) {
        // keep the arrays for the next matrix on this domain (one set)
        std::lock_guard<std::mutex> lock(pool_mutex());
        Domain::Spare& sp = m->dom->spare;
        if (!sp.val) {
            sp.val = m->val;
            sp.bv = m->bv;
            sp.dinv = m->dinv;
            sp.band32 = m->band32;
            sp.dinv32 = m->dinv32;
            sp.band64 = m->band64;
            m->val = m->bv = m->dinv = m->band64 = nullptr;
            m->band32 = m->dinv32 = nullptr;
        }
    }
    if (m->band64) cudaFree(m->band64);
    m->band64 = nullptr;
    if (m->val) cudaFree(m->val);
    if (m->bv) cudaFree(m->bv);
    if (m->dinv) cudaFree(m->dinv);
    if (m->band32) cudaFree(m->band32);
    if (m->dinv32) cudaFree(m->dinv32);
    m->val = m->bv = m->dinv = nullptr;
    m->band32 = m->dinv32 = nullptr;
}

int require_unbalanced(const Matrix* m, const char* what)
{
    if (m->balanced) {
        set_error(std::string(what) +
                  ": the matrix was balanced in place by a solve; reset it before changing values");
        return RG_INVALID_ARG;
    }
    return RG_OK;
}

}  // namespace

extern "C" {

int rg_version(void) { return 100; }

int rg_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return RG_INVALID_ARG;
    const std::string& e = last_error();
    const size_t k = e.size() < len - 1 ? e.size() : len - 1;
    memcpy(buf, e.data(), k);
    buf[k] = '\0';
    return RG_OK;
}

int rg_set_stream(void* s)
{
    set_stream(static_cast<cudaStream_t>(s));
    return RG_OK;
}

// ------------------------------------------------------------------ domain
int rg_domain_create(int dim, const int64_t ne[3], const double x0[3], const double x1[3],
                     rg_domain** out)
{
    RG_REQUIRE(out, "rg_domain_create: out is NULL");
    *out = nullptr;
    RG_REQUIRE(dim == 2 || dim == 3, "rg_domain_create: dim must be 2 or 3");
    RG_REQUIRE(ne && x0 && x1, "rg_domain_create: NULL argument");
    for (int k = 0; k < dim; ++k) {
        RG_REQUIRE(ne[k] > 0, "Number of elements in each spatial dimension must be positive");
        RG_REQUIRE(x1[k] > x0[k], "rg_domain_create: every axis needs x1 > x0");
    }
    RG_GUARD_BEGIN
    rg_domain* h = new rg_domain();
    Domain& d = h->d;
    d.dim = dim;
    int64_t n = 1, nnz = 1;
    for (int k = 0; k < 3; ++k) {
        d.ne[k] = k < dim ? ne[k] : 1;
        d.nn[k] = k < dim ? ne[k] + 1 : 1;
        d.x0[k] = k < dim ? x0[k] : 0.0;
        d.x1[k] = k < dim ? x1[k] : 1.0;
        d.dx[k] = k < dim ? (x1[k] - x0[k]) / (double)ne[k] : 1.0;
        if (k < dim) {
            n *= d.nn[k];
            nnz *= 3 * d.nn[k] - 2;
        }
    }
    if (nnz > 2147483647LL || n > 2147483647LL) {
        delete h;
        set_error("The number of elements has overflowed the 32-bit index range");
        return RG_INVALID_ARG;
    }
    d.n = n;
    d.nnz = nnz;
    d.npad = (n + 255) / 256 * 256;  // whole 256-row tiles of the band SpMV
    d.nbands = dim == 3 ? 27 : 9;
    for (int b = 0; b < d.nbands; ++b) {
        const int bx = b % 3 - 1, by = (b / 3) % 3 - 1, bz = dim == 3 ? b / 9 - 1 : 0;
        d.band_off[b] = bx + d.nn[0] * by + d.nn[0] * d.nn[1] * bz;
    }
    build_q1_tables(dim, d.dx, &d.q1);
    build_q1_reduced_tables(dim, d.dx, &d.q1r);
    cudaError_t e1 = cudaMalloc((void**)&d.ptr, sizeof(int32_t) * (n + 1));
    cudaError_t e2 = e1 == cudaSuccess ? cudaMalloc((void**)&d.idx, sizeof(int32_t) * nnz) : e1;
    if (e2 != cudaSuccess) {
        free_domain(&d);
        delete h;
        set_error(std::string("rg_domain_create: ") + cudaGetErrorString(e2));
        return RG_CUDA_ERROR;
    }
    int rc = launch_pattern(&d);
    if (rc == RG_OK) {
        cudaError_t e = cudaStreamSynchronize(stream());
        if (e != cudaSuccess) {
            set_error(std::string("rg_domain_create: ") + cudaGetErrorString(e));
            rc = RG_CUDA_ERROR;
        }
    }
    if (rc) {
        free_domain(&d);
        delete h;
        return rc;
    }
    *out = h;
    return RG_OK;
    RG_GUARD_END
}

// drops one reference to the domain; the last one frees it (matrices keep their domain
// alive, so destroying a domain before its matrices is safe)
static void release_domain(Domain* d)
{
    bool last;
    {
        std::lock_guard<std::mutex> lock(pool_mutex());
        last = --d->refs == 0;
    }
    if (last) {
        cudaStreamSynchronize(stream());
        free_domain(d);
        delete reinterpret_cast<rg_domain*>(d);  // Domain is rg_domain's only member
    }
}

int rg_domain_destroy(rg_domain* dom)
{
    if (!dom) return RG_OK;
    release_domain(&dom->d);
    return RG_OK;
}

int rg_domain_info(const rg_domain* dom, int64_t* n, int64_t* nnz, int64_t nn[3], int64_t ne[3],
                   double dx[3])
{
    RG_REQUIRE(dom, "rg_domain_info: NULL domain");
    const Domain& d = dom->d;
    if (n) *n = d.n;
    if (nnz) *nnz = d.nnz;
    for (int k = 0; k < 3; ++k) {
        if (nn) nn[k] = d.nn[k];
        if (ne) ne[k] = d.ne[k];
        if (dx) dx[k] = d.dx[k];
    }
    return RG_OK;
}

int rg_pattern(const rg_domain* dom, const int32_t** ptr, const int32_t** idx, int64_t* n,
               int64_t* nnz)
{
    RG_REQUIRE(dom, "rg_pattern: NULL domain");
    if (ptr) *ptr = dom->d.ptr;
    if (idx) *idx = dom->d.idx;
    if (n) *n = dom->d.n;
    if (nnz) *nnz = dom->d.nnz;
    return RG_OK;
}

int rg_pattern_to_host(const rg_domain* dom, int32_t* ptr_host, int32_t* idx_host)
{
    RG_REQUIRE(dom, "rg_pattern_to_host: NULL domain");
    const Domain& d = dom->d;
    if (ptr_host)
        RG_CHECK_CUDA(cudaMemcpyAsync(ptr_host, d.ptr, sizeof(int32_t) * (d.n + 1), cudaMemcpyDeviceToHost,
                                      stream()));
    if (idx_host)
        RG_CHECK_CUDA(cudaMemcpyAsync(idx_host, d.idx, sizeof(int32_t) * d.nnz, cudaMemcpyDeviceToHost,
                                      stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    return RG_OK;
}

// ------------------------------------------------------------------ matrix
int rg_matrix_create(rg_domain* dom, rg_matrix** out)
{
    RG_REQUIRE(out, "rg_matrix_create: out is NULL");
    *out = nullptr;
    RG_REQUIRE(dom, "rg_matrix_create: NULL domain");
    RG_GUARD_BEGIN
    rg_matrix* h = new rg_matrix();
    Matrix& m = h->m;
    m.dom = &dom->d;
    {
        // the arrays of a destroyed matrix on this domain, when there are some
        std::lock_guard<std::mutex> lock(pool_mutex());
        Domain::Spare& sp = dom->d.spare;
        if (sp.val) {
            m.val = sp.val;
            m.bv = sp.bv;
            m.dinv = sp.dinv;
            m.band32 = sp.band32;
            m.dinv32 = sp.dinv32;
            m.band64 = sp.band64;
            sp = Domain::Spare();
        }
    }
    cudaError_t e = cudaSuccess;
    if (!m.val) e = cudaMalloc((void**)&m.val, sizeof(double) * dom->d.nnz);
    if (e == cudaSuccess && !m.bv) e = cudaMalloc((void**)&m.bv, sizeof(double) * dom->d.n);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.val, 0, sizeof(double) * dom->d.nnz, stream());
    if (e != cudaSuccess) {
        free_matrix(&m);
        delete h;
        set_error(std::string("rg_matrix_create: ") + cudaGetErrorString(e));
        return RG_CUDA_ERROR;
    }
    {
        std::lock_guard<std::mutex> lock(pool_mutex());
        ++dom->d.refs;  // the matrix keeps its domain alive
    }
    *out = h;
    return RG_OK;
    RG_GUARD_END
}

int rg_matrix_create_system(rg_domain* dom, int block_size, rg_matrix** out)
{
    RG_REQUIRE(out, "rg_matrix_create_system: out is NULL");
    *out = nullptr;
    RG_REQUIRE(dom, "rg_matrix_create_system: NULL domain");
    if (block_size == 1) return rg_matrix_create(dom, out);
    if (block_size != 2 && block_size != 3) {
        set_error("rg_matrix_create_system: block sizes 1, 2 and 3 are supported");
        return RG_NOT_SUPPORTED;
    }
    RG_GUARD_BEGIN
    rg_matrix* h = new rg_matrix();
    Matrix& m = h->m;
    m.dom = &dom->d;
    m.nb = block_size;
    const size_t nv = (size_t)dom->d.nnz * block_size * block_size;
    cudaError_t e = cudaMalloc((void**)&m.val, sizeof(double) * nv);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m.bv, sizeof(double) * dom->d.n * block_size);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.val, 0, sizeof(double) * nv, stream());
    if (e != cudaSuccess) {
        free_matrix(&m);
        delete h;
        set_error(std::string("rg_matrix_create_system: ") + cudaGetErrorString(e));
        return RG_CUDA_ERROR;
    }
    {
        std::lock_guard<std::mutex> lock(pool_mutex());
        ++dom->d.refs;  // the matrix keeps its domain alive
    }
    *out = h;
    return RG_OK;
    RG_GUARD_END
}

int rg_matrix_block_size(const rg_matrix* mat, int* block_size)
{
    RG_REQUIRE(mat && block_size, "rg_matrix_block_size: NULL argument");
    *block_size = mat->m.nb;
    return RG_OK;
}

int rg_matrix_destroy(rg_matrix* mat)
{
    if (!mat) return RG_OK;
    cudaStreamSynchronize(stream());
    Domain* d = mat->m.dom;
    free_matrix(&mat->m);
    delete mat;
    release_domain(d);
    return RG_OK;
}

int rg_matrix_reset(rg_matrix* mat)
{
    RG_REQUIRE(mat, "rg_matrix_reset: NULL matrix");
    Matrix& m = mat->m;
    RG_CHECK_CUDA(cudaMemsetAsync(m.val, 0, sizeof(double) * m.dom->nnz * m.nb * m.nb, stream()));
    m.balanced = false;
    m.solver_ready = false;
    coef_reset(&m);
    return RG_OK;
}

int rg_matrix_values(rg_matrix* mat, double** val)
{
    RG_REQUIRE(mat && val, "rg_matrix_values: NULL argument");
    *val = mat->m.val;
    return RG_OK;
}

int rg_matrix_is_balanced(const rg_matrix* mat, int* balanced)
{
    RG_REQUIRE(mat && balanced, "rg_matrix_is_balanced: NULL argument");
    *balanced = mat->m.balanced ? 1 : 0;
    return RG_OK;
}

int rg_matrix_balance_vector(rg_matrix* mat, const double** bv)
{
    RG_REQUIRE(mat && bv, "rg_matrix_balance_vector: NULL argument");
    RG_REQUIRE(mat->m.balanced, "rg_matrix_balance_vector: matrix is not balanced");
    *bv = mat->m.bv;
    return RG_OK;
}

// ------------------------------------------------------------------ assembly
int rg_assemble_single(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                       const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y)
{
    RG_REQUIRE(mat, "rg_assemble_single: a matrix handle is required (it names the domain)");
    if (mat->m.nb != 1) {
        set_error("rg_assemble_single: the matrix is a PDE system; use rg_assemble_system");
        return RG_INVALID_ARG;
    }
    const rg_coef* c[6] = {A, B, C, D, X, Y};
    for (int j = 0; j < 6; ++j) RG_REQUIRE(coef_ok(c[j]), "rg_assemble_single: invalid coefficient");
    const bool addS = (A && A->kind) || (B && B->kind) || (C && C->kind) || (D && D->kind);
    if (addS) {
        int rc = require_unbalanced(&mat->m, "rg_assemble_single");
        if (rc) return rc;
        mat->m.solver_ready = false;
        if ((rc = coef_on_assemble(&mat->m, c, false))) return rc;
    }
    return assemble_single_impl(mat->m.dom, mat->m.val, rhs, c, false);
}

int rg_assemble_single_reduced(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                               const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y)
{
    RG_REQUIRE(mat, "rg_assemble_single_reduced: a matrix handle is required (it names the domain)");
    if (mat->m.nb != 1) {
        set_error("rg_assemble_single_reduced: the matrix is a PDE system; use rg_assemble_system_reduced");
        return RG_INVALID_ARG;
    }
    const rg_coef* c[6] = {A, B, C, D, X, Y};
    for (int j = 0; j < 6; ++j) RG_REQUIRE(coef_ok(c[j]), "rg_assemble_single_reduced: invalid coefficient");
    const bool addS = (A && A->kind) || (B && B->kind) || (C && C->kind) || (D && D->kind);
    if (addS) {
        int rc = require_unbalanced(&mat->m, "rg_assemble_single_reduced");
        if (rc) return rc;
        mat->m.solver_ready = false;
        if ((rc = coef_on_assemble(&mat->m, c, true))) return rc;
    }
    return assemble_single_impl(mat->m.dom, mat->m.val, rhs, c, true);
}

int rg_assemble_system(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                       const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y)
{
    RG_REQUIRE(mat, "rg_assemble_system: a matrix handle is required (it names the domain and block size)");
    const rg_coef* c[6] = {A, B, C, D, X, Y};
    for (int j = 0; j < 6; ++j) RG_REQUIRE(coef_ok(c[j]), "rg_assemble_system: invalid coefficient");
    const bool addS = (A && A->kind) || (B && B->kind) || (C && C->kind) || (D && D->kind);
    if (addS) {
        int rc = require_unbalanced(&mat->m, "rg_assemble_system");
        if (rc) return rc;
        mat->m.solver_ready = false;
        if ((rc = coef_on_assemble(&mat->m, c, false))) return rc;
    }
    if (mat->m.nb == 1) return assemble_single_impl(mat->m.dom, mat->m.val, rhs, c, false);
    return assemble_system_impl(mat->m.dom, mat->m.nb, mat->m.val, rhs, c, false);
}

int rg_assemble_system_reduced(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                               const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y)
{
    RG_REQUIRE(mat, "rg_assemble_system_reduced: a matrix handle is required (it names the domain and block size)");
    const rg_coef* c[6] = {A, B, C, D, X, Y};
    for (int j = 0; j < 6; ++j) RG_REQUIRE(coef_ok(c[j]), "rg_assemble_system_reduced: invalid coefficient");
    const bool addS = (A && A->kind) || (B && B->kind) || (C && C->kind) || (D && D->kind);
    if (addS) {
        int rc = require_unbalanced(&mat->m, "rg_assemble_system_reduced");
        if (rc) return rc;
        mat->m.solver_ready = false;
        if ((rc = coef_on_assemble(&mat->m, c, true))) return rc;
    }
    if (mat->m.nb == 1) return assemble_single_impl(mat->m.dom, mat->m.val, rhs, c, true);
    return assemble_system_impl(mat->m.dom, mat->m.nb, mat->m.val, rhs, c, true);
}

static int assemble_boundary_any(rg_matrix* mat, double* rhs, const rg_coef* d, const rg_coef* y, bool reduced,
                                 const char* who)
{
    if (!mat) {
        set_error(std::string(who) + ": a matrix handle is required");
        return RG_INVALID_ARG;
    }
    if (!coef_ok(d) || !coef_ok(y)) {
        set_error(std::string(who) + ": invalid coefficient");
        return RG_INVALID_ARG;
    }
    if (d && d->kind) {
        int rc = require_unbalanced(&mat->m, who);
        if (rc) return rc;
        mat->m.solver_ready = false;
        coef_invalidate(&mat->m);  // face terms are not part of the coefficient operator
    }
    return assemble_boundary_impl(mat->m.dom, mat->m.nb, reduced, mat->m.val, rhs, d, y);
}

int rg_assemble_boundary(rg_matrix* mat, double* rhs, const rg_coef* d, const rg_coef* y)
{
    return assemble_boundary_any(mat, rhs, d, y, false, "rg_assemble_boundary");
}

int rg_assemble_boundary_reduced(rg_matrix* mat, double* rhs, const rg_coef* d, const rg_coef* y)
{
    return assemble_boundary_any(mat, rhs, d, y, true, "rg_assemble_boundary_reduced");
}

int rg_insert_constraint(rg_matrix* mat, double* rhs, const double* q, const double* r, int rhs_only)
{
    RG_REQUIRE(mat && q, "rg_insert_constraint: NULL matrix or mask");
    if (!rhs_only) {
        int rc = require_unbalanced(&mat->m, "rg_insert_constraint");
        if (rc) return rc;
        mat->m.solver_ready = false;
        if ((rc = coef_on_constraint(&mat->m, q))) return rc;
    }
    if (mat->m.nb != 1) return launch_system_constraint(&mat->m, rhs, q, r, rhs_only);
    return launch_insert_constraint(&mat->m, rhs, q, r, rhs_only);
}

int rg_nullify_rows_and_cols(rg_matrix* mat, const double* mask_row, const double* mask_col,
                             double main_diagonal_value)
{
    RG_REQUIRE(mat && mask_row && mask_col, "rg_nullify_rows_and_cols: NULL argument");
    int rc = require_unbalanced(&mat->m, "rg_nullify_rows_and_cols");
    if (rc) return rc;
    mat->m.solver_ready = false;
    coef_invalidate(&mat->m);
    if (mat->m.nb != 1) return launch_system_nullify(&mat->m, mask_row, mask_col, main_diagonal_value);
    return launch_nullify(&mat->m, mask_row, mask_col, main_diagonal_value);
}

int rg_spmv(rg_matrix* mat, double alpha, const double* x, double beta, double* y)
{
    RG_REQUIRE(mat && x && y, "rg_spmv: NULL argument");
    RG_REQUIRE(!mat->m.balanced, "MatrixVector: balanced matrix is not supported.");
    if (mat->m.nb != 1) return launch_system_spmv(&mat->m, alpha, x, beta, y);
    return launch_spmv64(mat->m.dom, mat->m.val, alpha, x, beta, y);
}

int rg_interpolate_nodes(const rg_domain* dom, const double* nodal, int ncomp, double* out, int reduced)
{
    RG_REQUIRE(dom && nodal && out && ncomp > 0, "rg_interpolate_nodes: invalid argument");
    return launch_interpolate(&dom->d, nodal, ncomp, out, reduced);
}

int rg_save_mm(rg_matrix* mat, const char* path)
{
    RG_REQUIRE(mat && path, "rg_save_mm: NULL argument");
    RG_GUARD_BEGIN
    const Domain& d = *mat->m.dom;
    const int nb = mat->m.nb;
    std::vector<int32_t> ptr(d.n + 1), idx(d.nnz);
    std::vector<double> val((size_t)d.nnz * nb * nb);
    RG_CHECK_CUDA(cudaMemcpyAsync(ptr.data(), d.ptr, sizeof(int32_t) * (d.n + 1), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaMemcpyAsync(idx.data(), d.idx, sizeof(int32_t) * d.nnz, cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaMemcpyAsync(val.data(), mat->m.val, sizeof(double) * val.size(), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    FILE* f = fopen(path, "w");
    if (!f) {
        set_error(std::string("rg_save_mm: cannot open ") + path);
        return RG_INVALID_ARG;
    }
    // SparseMatrix<double>::saveMM (paso/src/SparseMatrix.cpp:180-240): banner, size line, then
    // per node pair (i, j) of the pattern its block entries (ir, ic), row-block index outer, as
    // scalar coordinates (i nb + ir, j nb + ic), 1-based, values with 15 significant digits
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(f, "%lld %lld %lld\n", (long long)d.n * nb, (long long)d.n * nb, (long long)d.nnz * nb * nb);
    for (int64_t i = 0; i < d.n; ++i)
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
            for (int ir = 0; ir < nb; ++ir)
                for (int ic = 0; ic < nb; ++ic)
                    fprintf(f, "%lld %lld %.15g\n", (long long)(i * nb + ir + 1), (long long)idx[k] * nb + ic + 1,
                            val[(size_t)k * nb * nb + ir + nb * ic]);
    fclose(f);
    return RG_OK;
    RG_GUARD_END
}

// ------------------------------------------------------------------ solver
void rg_solver_opts_default(rg_solver_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->method = RG_METHOD_PCG;
    o->preconditioner = RG_PRECOND_JACOBI;
    o->tolerance = 1e-8;
    o->iter_max = 100000;
    o->sweeps = 1;
    o->mode = RG_MODE_PASO;
    o->precision = RG_PREC_FP64;
    o->layout = RG_LAYOUT_CSR;
    o->inner_tolerance = 1e-2;
}

int rg_solver_config(const rg_matrix* mat, int* spmv_config, int* update_grid, double* spmv_us)
{
    RG_REQUIRE(mat, "rg_solver_config: NULL matrix");
    return rg::solver_config(&mat->m, spmv_config, update_grid, spmv_us);
}

int rg_solver_set_config(rg_matrix* mat, int spmv_config)
{
    RG_REQUIRE(mat, "rg_solver_set_config: NULL matrix");
    return rg::solver_set_config(&mat->m, spmv_config);
}

int rg_test_wait_limit(int max_polls, int withhold_copies)
{
    const int rc = rg::set_wait_control(max_polls, withhold_copies);
    if (rc) return rc;
    return rg::ws::set_conv_wait_control(max_polls, withhold_copies);
}

int rg_solve(rg_matrix* mat, const double* rhs, double* x, const rg_solver_opts* opts, rg_diag* diag)
{
    RG_REQUIRE(mat && rhs && x, "rg_solve: NULL argument");
    rg_solver_opts o;
    if (opts)
        o = *opts;
    else
        rg_solver_opts_default(&o);
    RG_GUARD_BEGIN
    if (mat->m.nb != 1) return rg::solve_system(&mat->m, rhs, x, &o, diag);
    return rg::solve(&mat->m, rhs, x, &o, diag);
    RG_GUARD_END
}

}  // extern "C"
