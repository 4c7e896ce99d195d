// rg_residual_norms: norms of b - A x for a solution x (LinearPDE.getResidual,
// escriptcore/py_src/linearPDEs.py, measured in the l2 and max norms that paso's stopping
// test uses).  The reduction scratch lives with the matrix and is allocated on first use.
#include <cmath>

#include "rg_residual.cuh"

namespace rg {

struct ResidualScratch {
    double* partials = nullptr;  // residual::kMaxBlocks * 2 doubles
    unsigned* counter = nullptr;
    double* out = nullptr;       // 2 doubles
};

void free_residual_scratch(Matrix* m)
{
    if (!m->rs) return;
    cudaFree(m->rs->partials);
    cudaFree(m->rs->counter);
    cudaFree(m->rs->out);
    delete m->rs;
    m->rs = nullptr;
}

int ensure_residual_scratch(Matrix* m)
{
    if (m->rs) return RG_OK;
    ResidualScratch* s = new ResidualScratch();
    m->rs = s;
    RG_CHECK_CUDA(cudaMalloc((void**)&s->partials, sizeof(double) * residual::kMaxBlocks * 2));
    RG_CHECK_CUDA(cudaMalloc((void**)&s->counter, sizeof(unsigned)));
    RG_CHECK_CUDA(cudaMalloc((void**)&s->out, sizeof(double) * 2));
    RG_CHECK_CUDA(cudaMemsetAsync(s->counter, 0, sizeof(unsigned), stream()));
    return RG_OK;
}

}  // namespace rg

using namespace rg;

extern "C" int rg_residual_norms(rg_matrix* mat, const double* rhs, const double* x, double* l2_host,
                                 double* linf_host)
{
    RG_REQUIRE(mat && rhs && x, "rg_residual_norms: NULL argument");
    Matrix* m = &mat->m;
    if (m->nb != 1) return residual_norms_system(m, rhs, x, l2_host, linf_host);
    const Domain* d = m->dom;
    int rc = ensure_residual_scratch(m);
    if (rc) return rc;
    const int grid = residual::grid(d->n);
    RG_TIMED(T_NORMS, (residual::k_residual_norms<<<grid, residual::kThreads, 0, stream()>>>(
                          d->n, d->ptr, d->idx, m->val, m->balanced ? m->bv : nullptr, rhs, x,
                          ReduceBuf{m->rs->partials, m->rs->counter}, m->rs->out)));
    RG_CHECK_LAUNCH();
    double h[2];
    RG_CHECK_CUDA(cudaMemcpyAsync(h, m->rs->out, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    if (l2_host) *l2_host = std::sqrt(h[0]);
    if (linf_host) *linf_host = h[1];
    return RG_OK;
}
