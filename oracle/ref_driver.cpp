// Driver that links the reference's own hot-path sources, compiled in place from
// the esys-escript tree by oracle/Makefile (target ref), into oracle/_ref/libripley_ref.so:
//
//   ripley/src/DefaultAssembler2D.cpp, ripley/src/DefaultAssembler3D.cpp
//   paso/src/Solver.cpp, paso/src/PCG.cpp, paso/src/SparseMatrix_MatrixVector.cpp
//
// TEST INFRASTRUCTURE ONLY (checker and CPU baseline).  This file supplies the
// pieces those sources call into that live in files which need boost/MPI and are
// not compiled: the element scatter of Brick/Rectangle::addToMatrixAndRHS +
// RipleyDomain::addToPasoMatrix (Brick.cpp:3238-3265, RipleyDomain.cpp:1488-1614),
// SystemMatrix::balance/applyBalance (SystemMatrix.cpp:223-312) and the Jacobi
// smoother (Smoother.cpp:100-128, SparseMatrix.cpp:387-435, Pattern.cpp:139-164).
#include <ripley/DefaultAssembler2D.h>
#include <ripley/DefaultAssembler3D.h>

#include <paso/paso_shim.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace escript {
double gettime()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace escript

namespace ripley {

template <>
void ShimDomain::addToMatrixAndRHS<double>(escript::AbstractSystemMatrix* S, escript::Data& F,
                                           const std::vector<double>& EM_S,
                                           const std::vector<double>& EM_F, bool addS,
                                           bool addF, index_t firstNode, int nEq, int nComp) const
{
    // element arrays EM_S[INDEX4(ieq, icomp, r, c, nEq, nComp, nk)], EM_F[INDEX2(ieq, r, nEq)];
    // block entries val[k nEq^2 + ieq + nEq icomp] (RipleyDomain.cpp:1508-1518)
    const int nk = dim == 3 ? 8 : 4;
    index_t rows[8];
    for (int k = 0; k < nk; ++k)
        rows[k] = firstNode + (k & 1) + ((k >> 1) & 1) * m_NN[0] +
                  ((k >> 2) & 1) * m_NN[0] * m_NN[1];
    if (addF) {
        double* F_p = F.getSampleDataRW(0, 0.0);
        for (int k = 0; k < nk; ++k)
            if (rows[k] < numDOF)
                for (int e = 0; e < nEq; ++e) F_p[rows[k] * nEq + e] += EM_F[e + nEq * k];
    }
    if (addS && S && S->val) {
        for (int r = 0; r < nk; ++r) {
            const index_t row = rows[r];
            for (int c = 0; c < nk; ++c) {
                const index_t col = rows[c];
                for (index_t k = S->ptr[row]; k < S->ptr[row + 1]; ++k)
                    if (S->idx[k] == col) {
                        for (int ic = 0; ic < nComp; ++ic)
                            for (int ie = 0; ie < nEq; ++ie)
                                S->val[k * nEq * nComp + ie + nEq * ic] +=
                                    EM_S[ie + nEq * (ic + nComp * (r + nk * c))];
                        break;
                    }
            }
        }
    }
}

template <>
void ShimDomain::addToMatrixAndRHS<cplx_t>(escript::AbstractSystemMatrix*, escript::Data&,
                                           const std::vector<cplx_t>&,
                                           const std::vector<cplx_t>&, bool, bool, index_t,
                                           int, int) const
{
    throw std::runtime_error("complex assembly is not part of the oracle");
}

}  // namespace ripley

namespace paso {

template <>
void SystemMatrix<double>::balance()
{
    // SystemMatrix::balance (SystemMatrix.cpp:263-312) with SparseMatrix::maxAbsRow and
    // applyDiagonal (SparseMatrix.cpp:266-282, 361-385): one factor per scalar row
    if (is_balanced) return;
    const dim_t nodes = mainBlock->numRows;
    const dim_t nb = row_block_size;
    const index_t* ptr = mainBlock->pattern->ptr;
    const index_t* idx = mainBlock->pattern->index;
    double* val = mainBlock->val;
    balance_vector.assign(nodes * nb, 0.0);
#pragma omp parallel for
    for (dim_t i = 0; i < nodes; ++i)
        for (dim_t ir = 0; ir < nb; ++ir) {
            double fac = 0.;
            for (index_t k = ptr[i]; k < ptr[i + 1]; ++k)
                for (dim_t ic = 0; ic < nb; ++ic) fac = std::max(fac, std::abs(val[k * nb * nb + ir + nb * ic]));
            balance_vector[i * nb + ir] = fac > 0 ? std::sqrt(1. / fac) : 1.;
        }
#pragma omp parallel for
    for (dim_t i = 0; i < nodes; ++i)
        for (dim_t ir = 0; ir < nb; ++ir)
            for (index_t k = ptr[i]; k < ptr[i + 1]; ++k)
                for (dim_t ic = 0; ic < nb; ++ic)
                    val[k * nb * nb + ir + nb * ic] *= balance_vector[i * nb + ir] * balance_vector[idx[k] * nb + ic];
    is_balanced = true;
}

template <>
void SystemMatrix<double>::applyBalance(double* x_out, const double* x, bool) const
{
    if (!is_balanced) return;
    const dim_t n = getTotalNumRows();
#pragma omp parallel for
    for (dim_t i = 0; i < n; ++i) x_out[i] = x[i] * balance_vector[i];
}

template <>
void SystemMatrix<double>::applyBalanceInPlace(double* x, bool) const
{
    if (!is_balanced) return;
    const dim_t n = getTotalNumRows();
#pragma omp parallel for
    for (dim_t i = 0; i < n; ++i) x[i] *= balance_vector[i];
}

namespace {
// BlockOps_invM_2 / _3 (BlockOps.h:99-160): inverse of a column-major block
bool invert_block(dim_t nb, const double* A, double* inv)
{
    if (nb == 1) {
        if (!(std::abs(A[0]) > 0.)) return false;
        inv[0] = 1. / A[0];
        return true;
    }
    if (nb == 2) {
        double D = A[0] * A[3] - A[2] * A[1];
        if (!(std::abs(D) > 0)) return false;
        D = 1. / D;
        inv[0] = A[3] * D;
        inv[1] = -A[1] * D;
        inv[2] = -A[2] * D;
        inv[3] = A[0] * D;
        return true;
    }
    const double A11 = A[0], A21 = A[1], A31 = A[2], A12 = A[3], A22 = A[4], A32 = A[5];
    const double A13 = A[6], A23 = A[7], A33 = A[8];
    double D = A11 * (A22 * A33 - A23 * A32) + A12 * (A31 * A23 - A21 * A33) + A13 * (A21 * A32 - A31 * A22);
    if (!(std::abs(D) > 0)) return false;
    D = 1. / D;
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
}  // namespace

template <>
void SystemMatrix<double>::setPreconditioner(Options* options)
{
    // SparseMatrix::invMain (SparseMatrix.cpp:387-435) via the diagonal pointer
    // (Pattern.cpp:139-164): inverses of the main diagonal blocks
    sweeps = options->sweeps;
    if (!dinv.empty()) return;
    const dim_t nodes = mainBlock->numRows;
    const dim_t nb = row_block_size;
    const index_t* ptr = mainBlock->pattern->ptr;
    const index_t* idx = mainBlock->pattern->index;
    dinv.assign(nodes * nb * nb, 0.0);
    bool failed = false;
    for (dim_t i = 0; i < nodes; ++i) {
        const index_t* lo = idx + ptr[i];
        const index_t* hi = idx + ptr[i + 1];
        const index_t* w = std::lower_bound(lo, hi, i);
        if (w == hi || *w != i) { failed = true; continue; }
        if (!invert_block(nb, mainBlock->val + (w - idx) * nb * nb, &dinv[i * nb * nb])) failed = true;
    }
    if (failed) throw PasoException("SparseMatrix::invMain: non-regular main diagonal block.");
}

template <>
void SystemMatrix<double>::solvePreconditioner(double* x, double* b)
{
    // Preconditioner_Smoother_solve (Smoother.cpp:100-128): x = D^-1 b, then sweeps-1
    // corrections x += D^-1 (b - A x) (BlockOps_solveAll: block products)
    const dim_t nodes = mainBlock->numRows;
    const dim_t nb = row_block_size;
    const dim_t n = nodes * nb;
    auto apply = [&](const double* in, double* out, bool add) {
        for (dim_t i = 0; i < nodes; ++i)
            for (dim_t ir = 0; ir < nb; ++ir) {
                double s = 0.0;
                for (dim_t ic = 0; ic < nb; ++ic) s += dinv[i * nb * nb + ir + nb * ic] * in[i * nb + ic];
                out[i * nb + ir] = add ? out[i * nb + ir] + s : s;
            }
    };
    apply(b, x, false);
    std::vector<double> bn;
    for (int s = 1; s < sweeps; ++s) {
        bn.assign(b, b + n);
        SparseMatrix_MatrixVector_CSR_OFFSET0(-1., mainBlock, x, 1., bn.data());
        apply(bn.data(), x, true);
    }
}

template <>
void SystemMatrix<double>::MatrixVector_CSR_OFFSET0(double alpha, const double* in, double beta,
                                                    double* out) const
{
    SparseMatrix_MatrixVector_CSR_OFFSET0(alpha, mainBlock, in, beta, out);
}

}  // namespace paso

namespace {
char g_err[512];

escript::Data make_coef(const double* p, int kind, int dpsize, int nq)
{
    // kinds: 0 empty, 1 constant, 2 expanded
    if (!p || kind == 0) return escript::Data();
    return escript::Data(const_cast<double*>(p), dpsize, nq, kind == 2);
}

struct Geometry {
    ripley::ShimDomain dom;
    ripley::dim_t NE[3], NN[3];
    double dx[3];
};

void make_geometry(Geometry& g, int dim, const int64_t ne[3], const double dx[3])
{
    g.dom.dim = dim;
    for (int d = 0; d < 3; ++d) {
        g.NE[d] = d < dim ? (ripley::dim_t)ne[d] : 1;
        g.NN[d] = d < dim ? g.NE[d] + 1 : 1;
        g.dx[d] = d < dim ? dx[d] : 1.0;
        g.dom.m_NN[d] = g.NN[d];
    }
    g.dom.numDOF = g.NN[0] * g.NN[1] * (dim == 3 ? g.NN[2] : 1);
    ripley::index_t counts[6];
    if (dim == 2) {
        counts[0] = counts[1] = g.NE[1];
        counts[2] = counts[3] = g.NE[0];
        counts[4] = counts[5] = 0;
    } else {
        counts[0] = counts[1] = g.NE[1] * g.NE[2];
        counts[2] = counts[3] = g.NE[0] * g.NE[2];
        counts[4] = counts[5] = g.NE[0] * g.NE[1];
    }
    ripley::index_t off = 0;
    for (int f = 0; f < 2 * dim; ++f) {
        g.dom.m_faceOffset[f] = off;
        off += counts[f];
    }
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err; }

void ref_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

// interior terms; kinds[6]/coefs[6] for A,B,C,D,X,Y (0 empty, 1 constant, 2 expanded)
int ref_assemble(int dim, const int64_t ne[3], const double dx[3], const int32_t* ptr,
                 const int32_t* idx, double* val, double* rhs, const int* kinds,
                 const double* const* coefs)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        const int nq = 1 << dim;
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        escript::Data rhsD(rhs, 1, 1, true);
        escript::Data A = make_coef(coefs[0], kinds[0], dim * dim, nq);
        escript::Data B = make_coef(coefs[1], kinds[1], dim, nq);
        escript::Data C = make_coef(coefs[2], kinds[2], dim, nq);
        escript::Data D = make_coef(coefs[3], kinds[3], 1, nq);
        escript::Data X = make_coef(coefs[4], kinds[4], dim, nq);
        escript::Data Y = make_coef(coefs[5], kinds[5], 1, nq);
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESingle(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESingle(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// the reduced-order interior terms (coefficients on ReducedFunction: one data point per
// element), DefaultAssembler{2,3}D::assemblePDESingleReduced
int ref_assemble_reduced(int dim, const int64_t ne[3], const double dx[3], const int32_t* ptr,
                         const int32_t* idx, double* val, double* rhs, const int* kinds,
                         const double* const* coefs)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        escript::Data rhsD(rhs, 1, 1, true);
        escript::Data A = make_coef(coefs[0], kinds[0], dim * dim, 1);
        escript::Data B = make_coef(coefs[1], kinds[1], dim, 1);
        escript::Data C = make_coef(coefs[2], kinds[2], dim, 1);
        escript::Data D = make_coef(coefs[3], kinds[3], 1, 1);
        escript::Data X = make_coef(coefs[4], kinds[4], dim, 1);
        escript::Data Y = make_coef(coefs[5], kinds[5], 1, 1);
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESingleReduced(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESingleReduced(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// PDE systems: DefaultAssembler{2,3}D::assemblePDESystem with block size nb; coefficient data
// point sizes A nb^2 dim^2, B/C nb^2 dim, D nb^2, X nb dim, Y nb
int ref_assemble_system(int dim, const int64_t ne[3], const double dx[3], int nb, const int32_t* ptr,
                        const int32_t* idx, double* val, double* rhs, const int* kinds,
                        const double* const* coefs)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        const int nq = 1 << dim;
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        S.nb = nb;
        escript::Data rhsD(rhs, nb, 1, true);
        escript::Data A = make_coef(coefs[0], kinds[0], nb * nb * dim * dim, nq);
        escript::Data B = make_coef(coefs[1], kinds[1], nb * nb * dim, nq);
        escript::Data C = make_coef(coefs[2], kinds[2], nb * nb * dim, nq);
        escript::Data D = make_coef(coefs[3], kinds[3], nb * nb, nq);
        escript::Data X = make_coef(coefs[4], kinds[4], nb * dim, nq);
        escript::Data Y = make_coef(coefs[5], kinds[5], nb, nq);
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESystem(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESystem(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// boundary terms d, y on the faces (FunctionOnBoundary layout)
int ref_assemble_boundary(int dim, const int64_t ne[3], const double dx[3], const int32_t* ptr,
                          const int32_t* idx, double* val, double* rhs, int dkind,
                          const double* d, int ykind, const double* y)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        const int nq = 1 << (dim - 1);
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        escript::Data rhsD(rhs, 1, 1, true);
        escript::Data dD = make_coef(d, dkind, 1, nq);
        escript::Data yD = make_coef(y, ykind, 1, nq);
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDEBoundarySingle(val ? &S : nullptr, rhsD, dD, yD);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDEBoundarySingle(val ? &S : nullptr, rhsD, dD, yD);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// face terms in general form: block size nb and, with `reduced`, ReducedFunctionOnBoundary
// (one data point per face element): assemblePDEBoundarySingle / SingleReduced / System /
// SystemReduced of DefaultAssembler{2,3}D
int ref_assemble_boundary_ex(int dim, const int64_t ne[3], const double dx[3], int nb, int reduced,
                             const int32_t* ptr, const int32_t* idx, double* val, double* rhs, int dkind,
                             const double* d, int ykind, const double* y)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        const int nq = reduced ? 1 : 1 << (dim - 1);
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        S.nb = nb;
        escript::Data rhsD(rhs, nb, 1, true);
        escript::Data dD = make_coef(d, dkind, nb * nb, nq);
        escript::Data yD = make_coef(y, ykind, nb, nq);
        escript::AbstractSystemMatrix* M = val ? &S : nullptr;
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            if (nb == 1 && !reduced) a.assemblePDEBoundarySingle(M, rhsD, dD, yD);
            else if (nb == 1) a.assemblePDEBoundarySingleReduced(M, rhsD, dD, yD);
            else if (!reduced) a.assemblePDEBoundarySystem(M, rhsD, dD, yD);
            else a.assemblePDEBoundarySystemReduced(M, rhsD, dD, yD);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            if (nb == 1 && !reduced) a.assemblePDEBoundarySingle(M, rhsD, dD, yD);
            else if (nb == 1) a.assemblePDEBoundarySingleReduced(M, rhsD, dD, yD);
            else if (!reduced) a.assemblePDEBoundarySystem(M, rhsD, dD, yD);
            else a.assemblePDEBoundarySystemReduced(M, rhsD, dD, yD);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// assemblePDESystemReduced: the system terms on ReducedFunction (one data point per element)
int ref_assemble_system_reduced(int dim, const int64_t ne[3], const double dx[3], int nb, const int32_t* ptr,
                                const int32_t* idx, double* val, double* rhs, const int* kinds,
                                const double* const* coefs)
{
    try {
        Geometry g;
        make_geometry(g, dim, ne, dx);
        escript::AbstractSystemMatrix S;
        S.ptr = ptr;
        S.idx = idx;
        S.val = val;
        S.nb = nb;
        escript::Data rhsD(rhs, nb, 1, true);
        escript::Data A = make_coef(coefs[0], kinds[0], nb * nb * dim * dim, 1);
        escript::Data B = make_coef(coefs[1], kinds[1], nb * nb * dim, 1);
        escript::Data C = make_coef(coefs[2], kinds[2], nb * nb * dim, 1);
        escript::Data D = make_coef(coefs[3], kinds[3], nb * nb, 1);
        escript::Data X = make_coef(coefs[4], kinds[4], nb * dim, 1);
        escript::Data Y = make_coef(coefs[5], kinds[5], nb, 1);
        if (dim == 3) {
            ripley::DefaultAssembler3D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESystemReduced(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        } else {
            ripley::DefaultAssembler2D<double> a(&g.dom, g.dx, g.NE, g.NN);
            a.assemblePDESystemReduced(val ? &S : nullptr, rhsD, A, B, C, D, X, Y);
        }
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return 1;
    }
    return 0;
}

// paso::Solver with PCG + Jacobi on a CSR matrix (balanced in place).
// Returns the paso SolverResult, or -1 when a PasoException was thrown.
int ref_solve(int64_t n, int32_t* ptr, int32_t* idx, double* val, double* b, double* x,
              double tol, int64_t iter_max, int sweeps, int verbose, int64_t* num_iter,
              double* residual_norm, int* converged, double* seconds)
{
    try {
        auto A = std::make_shared<paso::SystemMatrix<double>>();
        A->mainBlock = std::make_shared<paso::SparseMatrix<double>>();
        A->mainBlock->numRows = A->mainBlock->numCols = (paso::dim_t)n;
        A->mainBlock->pattern = std::make_shared<paso::Pattern>();
        A->mainBlock->pattern->ptr = ptr;
        A->mainBlock->pattern->index = idx;
        A->mainBlock->pattern->numOutput = A->mainBlock->pattern->numInput = (paso::dim_t)n;
        A->mainBlock->val = val;
        paso::Options o;
        o.tolerance = tol;
        o.iter_max = (paso::dim_t)iter_max;
        o.sweeps = sweeps;
        o.verbose = verbose != 0;
        paso::Performance pp;
        const double t0 = escript::gettime();
        paso::SolverResult res = paso::Solver(A, x, b, &o, &pp);
        if (seconds) *seconds = escript::gettime() - t0;
        *num_iter = o.num_iter;
        *residual_norm = o.residual_norm;
        *converged = o.converged ? 1 : 0;
        return (int)res;
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return -1;
    }
}

// paso::Solver with PCG + (block) Jacobi on a block CSR matrix with block size nb
int ref_solve_block(int64_t nodes, int nb, int32_t* ptr, int32_t* idx, double* val, double* b, double* x,
                    double tol, int64_t iter_max, int sweeps, int64_t* num_iter, double* residual_norm,
                    int* converged)
{
    try {
        auto A = std::make_shared<paso::SystemMatrix<double>>();
        A->row_block_size = A->col_block_size = nb;
        A->mainBlock = std::make_shared<paso::SparseMatrix<double>>();
        A->mainBlock->numRows = A->mainBlock->numCols = (paso::dim_t)nodes;
        A->mainBlock->row_block_size = A->mainBlock->col_block_size = nb;
        A->mainBlock->block_size = nb * nb;
        A->mainBlock->pattern = std::make_shared<paso::Pattern>();
        A->mainBlock->pattern->ptr = ptr;
        A->mainBlock->pattern->index = idx;
        A->mainBlock->pattern->numOutput = A->mainBlock->pattern->numInput = (paso::dim_t)nodes;
        A->mainBlock->val = val;
        paso::Options o;
        o.tolerance = tol;
        o.iter_max = (paso::dim_t)iter_max;
        o.sweeps = sweeps;
        paso::Performance pp;
        paso::SolverResult res = paso::Solver(A, x, b, &o, &pp);
        *num_iter = o.num_iter;
        *residual_norm = o.residual_norm;
        *converged = o.converged ? 1 : 0;
        return (int)res;
    } catch (const std::exception& e) {
        snprintf(g_err, sizeof(g_err), "%s", e.what());
        return -1;
    }
}

// the reference CSR SpMV: out = alpha*A*in + beta*out
void ref_spmv(int64_t n, int32_t* ptr, int32_t* idx, double* val, double alpha,
              const double* in, double beta, double* out)
{
    auto M = std::make_shared<paso::SparseMatrix<double>>();
    M->numRows = M->numCols = (paso::dim_t)n;
    M->pattern = std::make_shared<paso::Pattern>();
    M->pattern->ptr = ptr;
    M->pattern->index = idx;
    M->val = val;
    paso::SparseMatrix_MatrixVector_CSR_OFFSET0(alpha, M, in, beta, out);
}

}  // extern "C"
