/*
 * CPU oracle for the ripley Q1 assembly + paso PCG/Jacobi path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links this code;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
 * and only as the checker or the timed CPU baseline.
 *
 * This is a plain-C restatement of the reference algorithms.  Each function
 * names the reference file:line it follows (paths are relative to the
 * esys-escript source tree).  Parity of the restatement is pinned against the
 * reference's own DefaultAssembler2D/3D.cpp, PCG.cpp and Solver.cpp compiled
 * from their sources (oracle/build_ref.sh -> oracle/_ref/) and against the
 * reference test suite's known-answer problems (tests/test_oracle.py).
 */
#ifndef RIPLEY_ORACLE_H
#define RIPLEY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* coefficient kinds (escript Data storage of a coefficient on Function) */
enum { RO_EMPTY = 0, RO_CONSTANT = 1, RO_EXPANDED = 2, RO_PER_ELEMENT = 3 };

typedef struct {
    const double* p;   /* NULL when kind == RO_EMPTY */
    int kind;
} ro_coef;

/* solver status codes (paso SolverResult, paso/src/Paso.h) */
enum { RO_OK = 0, RO_MAXITER = 3, RO_BREAKDOWN = 4, RO_NAN = 5, RO_DIVERGENCE = 7,
       RO_INPUT_ERROR = 1 };

typedef struct {
    double tolerance;   /* SolverBuddy default 1e-8 (escriptcore/src/SolverOptions.cpp:48) */
    int64_t iter_max;   /* SolverBuddy default 100000 */
    int sweeps;         /* Jacobi sweeps, SolverBuddy default 1 */
    int verbose;
} ro_opts;

typedef struct {
    int64_t num_iter;
    int64_t num_outer;
    double residual_norm;
    int converged;
} ro_diag;

/* number of stored entries of the single-rank ripley pattern */
int64_t ro_pattern_nnz(int dim, const int64_t nn[3]);
/* CSR pattern of Brick/Rectangle::getConnections(false) (Brick.cpp:3000-3061) */
void ro_pattern(int dim, const int64_t nn[3], int32_t* ptr, int32_t* idx);

/* DefaultAssembler{2,3}D::assemblePDESingle + addToMatrixAndRHS + addToPasoMatrix.
   val/rhs are accumulated into (caller zeroes them); either may be NULL. */
void ro_assemble_single(int dim, const int64_t ne[3], const double dx[3],
                        const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                        ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y);

/* DefaultAssembler{2,3}D::assemblePDESingleReduced: the same terms with the 1-point
   (element centre) rule; coefficients constant or one value set per element. */
void ro_assemble_single_reduced(int dim, const int64_t ne[3], const double dx[3],
                                const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                                ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y);

/* DefaultAssembler{2,3}D::assemblePDEBoundarySingle (face terms d, y), 2x2 (2) Gauss
   per face.  d, y are given per face element in ripley face order. */
void ro_assemble_boundary(int dim, const int64_t ne[3], const double dx[3],
                          const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                          ro_coef d, ro_coef y);

/* The face terms for block size nb (1..3; d[k + nb m], y[k] per data point) and, with
   `reduced`, on ReducedFunctionOnBoundary (one data point per face element, 1-point rule):
   assemblePDEBoundarySystem / assemblePDEBoundarySingleReduced /
   assemblePDEBoundarySystemReduced. */
void ro_assemble_boundary_ex(int dim, const int64_t ne[3], const double dx[3], int nb, int reduced,
                             const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                             ro_coef d, ro_coef y);

/* node -> Function (2^dim Gauss points) interpolation, Brick.cpp:3355-3391 */
void ro_interpolate_nodes(int dim, const int64_t ne[3], const double* nodal, int ncomp,
                          double* out);

/* paso CSR SpMV  out = alpha*A*in + beta*out (SparseMatrix_MatrixVector.cpp:191-264) */
void ro_spmv(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
             double alpha, const double* in, double beta, double* out);

/* LinearPDE.insertConstraint (linearPDEs.py:2084-2112): rhs -= A*u_r; nullify rows and
   columns with q>0 (SparseMatrix.h:494-509); rhs[q>0] = r */
void ro_insert_constraint(int64_t n, const int32_t* ptr, const int32_t* idx, double* val,
                          double* rhs, const double* q, const double* r);

/* paso::Solver with PCG + Jacobi (Solver.cpp:46-330, PCG.cpp:62-367).
   Balances val in place (SystemMatrix.cpp:263-312), writes the balance vector to bv.
   Returns an RO_* status. */
int ro_solve_paso(int64_t n, const int32_t* ptr, const int32_t* idx, double* val,
                  const double* b, double* x, double* bv, const ro_opts* opts, ro_diag* diag);

/* plain textbook Jacobi-PCG on an unbalanced matrix with ||r||_2 <= rtol ||b||_2 */
int ro_solve_cg(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
                const double* b, double* x, double rtol, int64_t iter_max, ro_diag* diag);

/* PDE systems with block size nb (1..3): block CSR values val[k nb^2 + ir + nb ic] on the
   node pattern, vectors u[node nb + comp].  Coefficient data points: A (nb, dim, nb, dim),
   B (nb, dim, nb), C (nb, nb, dim), D (nb, nb), X (nb, dim), Y (nb), first index fastest. */
void ro_assemble_system(int dim, const int64_t ne[3], const double dx[3], int nb,
                        const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                        ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y);
/* assemblePDESystemReduced: the system terms with the 1-point rule (ReducedFunction) */
void ro_assemble_system_reduced(int dim, const int64_t ne[3], const double dx[3], int nb,
                                const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                                ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y);
void ro_spmv_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, const double* val,
                   double alpha, const double* x, double beta, double* y);
void ro_insert_constraint_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx,
                                double* val, double* rhs, const double* q, const double* r);
int ro_solve_paso_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, double* val,
                        const double* b, double* x, double* bv, const ro_opts* opts, ro_diag* diag);

#ifdef __cplusplus
}
#endif
#endif
