// The coefficient record of a scalar matrix: what its values were assembled from, kept so
// that the FP32 inner PCG can evaluate the operator from the element coefficients on the fly
// (RG_LAYOUT_COEF) instead of streaming a stored copy of the values.
//
// A matrix assembled by DefaultAssembler3D/2D::assemblePDESingle (ripley/src/
// DefaultAssembler3D.cpp:152-2226, DefaultAssembler2D.cpp:151-597) from A = kappa_e I per
// element with no B, C, D has a_ij = sum over the elements e holding nodes i and j of
// kappa_e T(l_i, l_j), T the Q1 stiffness of the reference box (the Gauss rule integrates it
// exactly); insertConstraint (escriptcore/py_src/linearPDEs.py:2084-2112) then zeroes the rows
// and columns of the fixed nodes and puts 1 on their diagonal.  Both steps are recorded here:
// the element values into the node-indexed array khat (element with upper corner at node i),
// the fixed nodes as the sign bit of khat at that node.  Anything else that changes the values
// (B, C, D, reduced-order or face terms, nullifyRowsAndCols, an assembly after a constraint)
// marks the record as not representable, and the solver then uses the stored values.
#include "rg_internal.cuh"

namespace rg {
namespace {

int64_t khat_size(const Domain* d) { return d->n + d->nn[0] * d->nn[1] + d->nn[0] + kCoefPad; }

// kappa of every element from A (escript layout: A[i + dim j + dim^2 q + dim^2 Q e], Q = 2^dim
// Gauss points when EXPANDED; PER_ELEMENT drops q; CONSTANT also drops e); *bad = 1 where A is
// not kappa I with the same kappa >= 0 at every point.  khat[upper corner of e] += kappa.
__global__ void k_coef_record(int dim, int64_t ne0, int64_t ne1, int64_t nel, int64_t nn0, int64_t nn01,
                              const double* __restrict__ A, int kind, float* __restrict__ khat, int* __restrict__ bad)
{
    const int dd = dim * dim;
    const int npts = kind == RG_COEF_EXPANDED ? (1 << dim) : 1;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        const double* a = A + (kind == RG_COEF_CONSTANT ? 0 : e * dd * npts);
        const double k = a[0];
        bool ok = k >= 0.0;
        for (int q = 0; q < npts; ++q)
            for (int i = 0; i < dim; ++i)
                for (int j = 0; j < dim; ++j) ok = ok && a[q * dd + i + dim * j] == (i == j ? k : 0.0);
        if (!ok) *bad = 1;
        const int64_t ex = e % ne0, ey = (e / ne0) % ne1, ez = e / (ne0 * ne1);
        const int64_t node = (ex + 1) + nn0 * (ey + 1) + (dim == 3 ? nn01 * (ez + 1) : 0);
        khat[node] += (float)k;
    }
}

// the nodes insertConstraint fixes (q > 0) get the sign bit of khat
__global__ void k_coef_mask(int64_t n, const double* __restrict__ q, float* __restrict__ khat)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (q[i] > 0.0) khat[i] = -fabsf(khat[i]);
}

// khat zeroed (state 0 -> the record starts)
int coef_begin(Matrix* m)
{
    CoefRecord& c = m->coef;
    const Domain* d = m->dom;
    if (!c.khat) RG_CHECK_CUDA(cudaMalloc((void**)&c.khat, sizeof(float) * khat_size(d)));
    if (!c.bad) RG_CHECK_CUDA(cudaMalloc((void**)&c.bad, sizeof(int)));
    RG_CHECK_CUDA(cudaMemsetAsync(c.khat, 0, sizeof(float) * khat_size(d), stream()));
    RG_CHECK_CUDA(cudaMemsetAsync(c.bad, 0, sizeof(int), stream()));
    c.state = 1;
    return RG_OK;
}

}  // namespace

void coef_reset(Matrix* m)
{
    m->coef.state = 0;
    m->coef.constrained = false;
}

void coef_invalidate(Matrix* m) { m->coef.state = -1; }

int coef_on_assemble(Matrix* m, const rg_coef* c[6], bool reduced)
{
    CoefRecord& r = m->coef;
    const bool A = c[0] && c[0]->kind, others = (c[1] && c[1]->kind) || (c[2] && c[2]->kind) || (c[3] && c[3]->kind);
    if (!A && !others) return RG_OK;  // right hand side only: the values do not change
    if (m->nb != 1 || reduced || others || r.constrained || r.state < 0) {
        coef_invalidate(m);
        return RG_OK;
    }
    if (r.state == 0) {
        int rc = coef_begin(m);
        if (rc) return rc;
    }
    const Domain* d = m->dom;
    const int64_t nel = d->ne[0] * d->ne[1] * d->ne[2];
    const int grid = grid_for(nel, 256, 8);
    k_coef_record<<<grid, 256, 0, stream()>>>(d->dim, d->ne[0], d->ne[1], nel, d->nn[0], d->nn[0] * d->nn[1],
                                              static_cast<const double*>(c[0]->ptr), c[0]->kind, r.khat, r.bad);
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int coef_on_constraint(Matrix* m, const double* q)
{
    CoefRecord& r = m->coef;
    if (m->nb != 1 || r.state < 0) {
        coef_invalidate(m);
        return RG_OK;
    }
    if (r.state == 0) {
        int rc = coef_begin(m);
        if (rc) return rc;
    }
    const Domain* d = m->dom;
    k_coef_mask<<<grid_for(d->n, 256, 8), 256, 0, stream()>>>(d->n, q, r.khat);
    RG_CHECK_LAUNCH();
    r.constrained = true;
    return RG_OK;
}

int coef_usable(Matrix* m, bool* usable)
{
    CoefRecord& r = m->coef;
    *usable = false;
    if (m->nb != 1 || r.state != 1) return RG_OK;
    int bad = 1;
    RG_CHECK_CUDA(cudaMemcpyAsync(&bad, r.bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    if (bad) {
        coef_invalidate(m);
        return RG_OK;
    }
    *usable = true;
    return RG_OK;
}

void free_coef(Matrix* m)
{
    if (m->coef.khat) cudaFree(m->coef.khat);
    if (m->coef.bad) cudaFree(m->coef.bad);
    m->coef = CoefRecord();
}

}  // namespace rg
