// Force-included (-include) stand-in for the paso headers that the reference's
// PCG.cpp, Solver.cpp and SparseMatrix_MatrixVector.cpp pull in.  It defines the
// include guards of the real headers so that their bodies are skipped, and
// declares only the types, fields and functions those three files use.  The
// member functions of SystemMatrix (balance, Jacobi preconditioner, SpMV) are
// implemented in oracle/ref_driver.cpp.
#pragma once
#define __PASO_H__
#define __PASO_SOLVER_H__
#define __PASO_SYSTEMMATRIX_H__
#define __PASO_OPTIONS_H__
#define __PASO_SPARSEMATRIX_H__
#include <escript/DataTypes.h>
#include <cmath>
#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
namespace escript {
double gettime();
}
namespace paso {
typedef escript::DataTypes::index_t index_t;
typedef escript::DataTypes::dim_t dim_t;
typedef escript::DataTypes::cplx_t cplx_t;
typedef escript::DataTypes::real_t real_t;
#define PASO_ONE (double)(1.0)
#define PASO_ZERO (double)(0.0)
#define TOLERANCE_FOR_SCALARS (double)(0.)
enum { MATRIX_FORMAT_DEFAULT = 1, MATRIX_FORMAT_CSC = 2, MATRIX_FORMAT_BLK1 = 4,
       MATRIX_FORMAT_OFFSET1 = 8, MATRIX_FORMAT_TRILINOS_CRS = 16, MATRIX_FORMAT_DIAGONAL_BLOCK = 32 };
enum { PASO_DEFAULT = 0, PASO_PASO = 21, PASO_PCG = 10, PASO_BICGSTAB = 6, PASO_TFQMR = 16,
       PASO_MINRES = 17, PASO_PRES20 = 4, PASO_GMRES = 3, PASO_NONLINEAR_GMRES = 18, PASO_JACOBI = 20 };
enum SolverResult { NoError = 0, MaxIterReached, InputError, MemoryError, Breakdown,
                    NegativeNormError, Divergence };
struct PasoException : public std::runtime_error {
    explicit PasoException(const std::string& s) : std::runtime_error(s) {}
};
struct Performance {};
enum { PERFORMANCE_ALL = 0, PERFORMANCE_SOLVER, PERFORMANCE_PRECONDITIONER_INIT,
       PERFORMANCE_PRECONDITIONER, PERFORMANCE_MVM, PERFORMANCE_ASSEMBLAGE };
inline void Performance_startMonitor(Performance*, int) {}
inline void Performance_stopMonitor(Performance*, int) {}
struct MPIInfo { int size = 1; int rank = 0; int comm = 0; };
typedef std::shared_ptr<MPIInfo> JMPI;
struct Options {
    int method = PASO_PCG, package = PASO_PASO, preconditioner = PASO_JACOBI;
    bool symmetric = false, verbose = false, converged = false;
    double tolerance = 1e-8;
    dim_t iter_max = 100000, sweeps = 1, truncation = 20, restart = 0;
    dim_t num_iter = 0, num_level = 0, num_inner_iter = 0;
    double time = 0, set_up_time = 0, net_time = 0, residual_norm = 0;
    static int getSolver(int method, int, bool, const JMPI&) { return method; }
};
struct Pattern {
    index_t* ptr = nullptr;
    index_t* index = nullptr;
    dim_t numOutput = 0;
    dim_t numInput = 0;
    bool isEmpty() const { return ptr == nullptr && index == nullptr; }
};
template <class T>
struct SparseMatrix {
    int type = MATRIX_FORMAT_DEFAULT;
    dim_t numRows = 0, numCols = 0;
    dim_t row_block_size = 1, col_block_size = 1, block_size = 1;
    std::shared_ptr<Pattern> pattern;
    T* val = nullptr;
};
template <class T> using SparseMatrix_ptr = std::shared_ptr<SparseMatrix<T>>;
template <class T> using const_SparseMatrix_ptr = std::shared_ptr<const SparseMatrix<T>>;
void SparseMatrix_MatrixVector_CSC_OFFSET0(double alpha, const_SparseMatrix_ptr<double> A,
                                           const double* in, double beta, double* out);
void SparseMatrix_MatrixVector_CSC_OFFSET1(double alpha, const_SparseMatrix_ptr<double> A,
                                           const double* in, double beta, double* out);
void SparseMatrix_MatrixVector_CSR_OFFSET0(double alpha, const_SparseMatrix_ptr<double> A,
                                           const double* in, double beta, double* out);
void SparseMatrix_MatrixVector_CSR_OFFSET0_DIAG(double alpha, const_SparseMatrix_ptr<double> A,
                                                const double* in, double beta, double* out);
void SparseMatrix_MatrixVector_CSR_OFFSET0_stripe(double alpha, dim_t nRows, dim_t row_block_size,
        dim_t col_block_size, const index_t* ptr, const index_t* index, const double* val,
        const double* in, double beta, double* out);
template <typename T>
void SparseMatrix_MatrixVector_CSR_OFFSET1(double alpha, const_SparseMatrix_ptr<T> A,
                                           const T* in, double beta, T* out);

/* The single-rank system matrix: main block only, balance vector and a Jacobi
   preconditioner.  Member functions live in ref_driver.cpp. */
template <class T>
class SystemMatrix {
public:
    int type = MATRIX_FORMAT_DEFAULT;
    dim_t row_block_size = 1, col_block_size = 1;
    JMPI mpi_info = std::make_shared<MPIInfo>();
    SparseMatrix_ptr<T> mainBlock;
    std::vector<double> balance_vector;
    std::vector<double> dinv;
    bool is_balanced = false;
    int sweeps = 1;
    dim_t getTotalNumRows() const { return mainBlock->numRows * row_block_size; }
    dim_t getTotalNumCols() const { return mainBlock->numCols * col_block_size; }
    dim_t getGlobalNumRows() const { return mainBlock->numRows * row_block_size; }
    dim_t getGlobalNumCols() const { return mainBlock->numCols * col_block_size; }
    void balance();
    void applyBalance(T* x_out, const T* x, bool RHS) const;
    void applyBalanceInPlace(T* x, bool RHS) const;
    void setPreconditioner(Options* options);
    void solvePreconditioner(T* x, T* b);
    void freePreconditioner() { dinv.clear(); }
    void MatrixVector_CSR_OFFSET0(double alpha, const T* in, double beta, T* out) const;
};
template <class T> using SystemMatrix_ptr = std::shared_ptr<SystemMatrix<T>>;

struct Function {};
struct LinearSystem : public Function {
    LinearSystem(SystemMatrix_ptr<double>, double*, Options*) {}
};
SolverResult Solver(SystemMatrix_ptr<double>, double*, double*, Options*, Performance*);
SolverResult Solver(SystemMatrix_ptr<cplx_t>, cplx_t*, cplx_t*, Options*, Performance*);
void Solver_free(SystemMatrix<double>*);
void Solver_free(SystemMatrix<cplx_t>*);
SolverResult Solver_PCG(SystemMatrix_ptr<double> A, double* B, double* X, dim_t* iter,
                        double* tolerance, Performance* pp);
/* Krylov methods other than PCG are outside the oracle; they report InputError. */
inline SolverResult Solver_BiCGStab(SystemMatrix_ptr<double>, double*, double*, dim_t*, double*, Performance*) { return InputError; }
inline SolverResult Solver_TFQMR(SystemMatrix_ptr<double>, double*, double*, dim_t*, double*, Performance*) { return InputError; }
inline SolverResult Solver_MINRES(SystemMatrix_ptr<double>, double*, double*, dim_t*, double*, Performance*) { return InputError; }
inline SolverResult Solver_GMRES(SystemMatrix_ptr<double>, double*, double*, dim_t*, double*, dim_t, dim_t, Performance*) { return InputError; }
inline SolverResult Solver_NewtonGMRES(Function*, double*, Options*, Performance*) { return InputError; }
}  // namespace paso
