/*
 * ripley_gpu — B200 (sm_100a) implementation of the ripley Q1 assembly and
 * paso PCG/Jacobi solve path of esys-escript, behind a plain C ABI.
 *
 * Every entry point returns an int status (RG_OK on success) and never throws.
 * rg_last_error() returns the message of the last failure on the calling thread.
 * Pointers are DEVICE pointers unless the name says _host.  Work is ordered on
 * the stream set by rg_set_stream (default: the legacy default stream); calls
 * are not thread-safe per handle.
 *
 * The reference interfaces replaced (paths relative to the esys-escript tree):
 *   ripley::Brick / ripley::Rectangle construction     ripley/src/ripleycpp.cpp:151-238, 521-546
 *   RipleyDomain::getPasoMatrixPattern / Pattern       ripley/src/Brick.cpp:2546-2747, 3000-3061
 *   RipleyDomain::newSystemMatrix (paso SystemMatrix)   ripley/src/RipleyDomain.cpp:950-1022
 *   AbstractAssembler::assemblePDESingle               ripley/src/AbstractAssembler.h:33-63
 *   DefaultAssembler{2,3}D::assemblePDESingle          ripley/src/DefaultAssembler3D.cpp:152-2226
 *   DefaultAssembler{2,3}D::assemblePDEBoundarySingle  ripley/src/DefaultAssembler3D.cpp:2232-2888
 *   LinearPDE.insertConstraint                         escriptcore/py_src/linearPDEs.py:2084-2112
 *   AbstractSystemMatrix::nullifyRowsAndCols           paso/src/SystemMatrix.h:544-605
 *   AbstractSystemMatrix::ypAx                         paso/src/SystemMatrix.h:643-666
 *   AbstractSystemMatrix::setToSolution -> paso solve  paso/src/SystemMatrix.h:614-641,
 *                                                      paso/src/Solver.cpp:46-330, PCG.cpp:62-367
 *   AbstractSystemMatrix::saveMM                       paso/src/SystemMatrix.h:70-80
 *   Brick::interpolateNodesOnElements                  ripley/src/Brick.cpp:3315-3398
 */
#ifndef RIPLEY_GPU_H
#define RIPLEY_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (paso SolverResult + PasoException classes, paso/src/solve.cpp:119-142) */
#define RG_OK 0
#define RG_INVALID_ARG 1   /* ValueError / PasoException on bad input                       */
#define RG_CUDA_ERROR 2    /* a CUDA runtime call failed                                    */
#define RG_MAXITER 3       /* "maximum number of iteration steps reached"                   */
#define RG_BREAKDOWN 4     /* "fatal break down in iterative solver"                        */
#define RG_NAN 5           /* "Matrix or right hand side contains undefined values"        */
#define RG_TIMEOUT 6       /* a bounded device wait gave up (persistent kernels)            */
#define RG_DIVERGENCE 7    /* "No improvement during iteration. Iterative solver gives up." */
#define RG_NOT_SUPPORTED 8 /* option combination this library does not implement            */

typedef struct rg_domain rg_domain;
typedef struct rg_matrix rg_matrix;

/* ---- library ------------------------------------------------------------------------- */
int rg_version(void);
/* copies the last error message (NUL-terminated, truncated to len) */
int rg_last_error(char* buf, size_t len);
/* cudaStream_t used for all following calls from this thread (NULL = default stream) */
int rg_set_stream(void* stream);

/* ---- domain: ripley::Rectangle (dim 2) / ripley::Brick (dim 3), one rank -------------- */
/* ne: elements per axis; x0/x1: coordinate range per axis (Brick(n0,n1,n2,l0,l1,l2) with
   l = (x0, x1) tuples).  The CSR pattern is built on the device at creation. */
int rg_domain_create(int dim, const int64_t ne[3], const double x0[3], const double x1[3],
                     rg_domain** out);
/* Frees the domain; its matrices (and batches) must be destroyed first.  Solver vectors of
   a destroyed matrix are kept by the domain for the next matrix on it and freed here. */
int rg_domain_destroy(rg_domain* dom);
/* n: DOF count (= nodes); nnz: pattern entries; nn/ne: nodes/elements per axis; dx: spacing */
int rg_domain_info(const rg_domain* dom, int64_t* n, int64_t* nnz, int64_t nn[3],
                   int64_t ne[3], double dx[3]);
/* device CSR pattern (int32, offset 0, rows sorted): Brick::getConnections +
   paso::Pattern.  Pointers stay owned by the domain. */
int rg_pattern(const rg_domain* dom, const int32_t** ptr, const int32_t** idx, int64_t* n,
               int64_t* nnz);
/* host copy of the pattern; ptr_host has n+1 entries, idx_host nnz */
int rg_pattern_to_host(const rg_domain* dom, int32_t* ptr_host, int32_t* idx_host);

/* ---- coefficients (escript::Data on Function / FunctionOnBoundary) -------------------- */
#define RG_COEF_EMPTY 0       /* coefficient not set                                      */
#define RG_COEF_CONSTANT 1    /* one data point for every element (DataConstant)          */
#define RG_COEF_EXPANDED 2    /* one data point per quadrature point (DataExpanded)       */
#define RG_COEF_PER_ELEMENT 3 /* one data point per element, same at its quadrature points */
typedef struct {
    const double* ptr; /* device pointer; layout as escript: A[i + d*j + d*d*q + d*d*Q*e],
                          B/C/X[i + d*q + d*Q*e], D/Y[q + Q*e] (Q = 2^dim quadrature
                          points, q x-fastest); PER_ELEMENT drops the q index          */
    int kind;
} rg_coef;

/* ---- system matrix: paso::SystemMatrix<double>, block size 1 -------------------------- */
int rg_matrix_create(rg_domain* dom, rg_matrix** out); /* values zeroed */
int rg_matrix_destroy(rg_matrix* mat);
/* A PDE system's matrix (numEq = numComp = block_size, 1..3; paso block CSR on the node
   pattern, SystemMatrix.h:403-492): values val[k bs^2 + ir + bs ic] for pattern entry k,
   equation ir, component ic (column-major blocks); vectors hold a node's components
   together, u[node bs + comp].  Solved by the paso algorithm in FP64 with block Jacobi. */
int rg_matrix_create_system(rg_domain* dom, int block_size, rg_matrix** out);
int rg_matrix_block_size(const rg_matrix* mat, int* block_size);
/* AbstractSystemMatrix::resetValues: zero the values, drop balancing and solver data */
int rg_matrix_reset(rg_matrix* mat);
/* device pointer to the nnz CSR values (FP64), in the domain's pattern order */
int rg_matrix_values(rg_matrix* mat, double** val);
/* 1 when the values have been balanced in place by a solve (paso keeps them so) */
int rg_matrix_is_balanced(const rg_matrix* mat, int* balanced);
/* device pointer to the balance vector (n entries); valid when balanced */
int rg_matrix_balance_vector(rg_matrix* mat, const double** bv);

/* assemblePDESingle: adds the interior terms of
     -(A_ij u_,j + B_i u)_,i + C_j u_,j + D u = -X_i,i + Y
   into mat (may be NULL) and rhs (n doubles, may be NULL).  Any coefficient may be NULL
   or RG_COEF_EMPTY. */
int rg_assemble_single(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                       const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y);
/* assemblePDESingleReduced (ripley/src/DefaultAssembler3D.cpp:2891-3271,
   DefaultAssembler2D.cpp:842-1010): the same terms for coefficients on ReducedFunction
   (A_reduced ... Y_reduced), integrated with the 1-point rule at the element centre.
   Coefficients are CONSTANT, or EXPANDED / PER_ELEMENT with one value set per element. */
int rg_assemble_single_reduced(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                               const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y);
/* assemblePDESystem (ripley/src/DefaultAssembler3D.cpp:3630-5751, DefaultAssembler2D.cpp:
   1186-1980): the interior terms of a PDE system into a matrix of rg_matrix_create_system.
   Coefficient data points, first index fastest: A (bs, dim, bs, dim), B (bs, dim, bs),
   C (bs, bs, dim), D (bs, bs), X (bs, dim), Y (bs); rhs has n bs entries. */
int rg_assemble_system(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                       const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y);
/* assemblePDESystemReduced (ripley/src/DefaultAssembler3D.cpp:6466-6876, DefaultAssembler2D
   assemblePDESystemReduced): the terms of rg_assemble_system for coefficients on
   ReducedFunction, 1-point rule at the element centre (one data point per element).  For a
   matrix of block size 1 this is rg_assemble_single_reduced. */
int rg_assemble_system_reduced(rg_matrix* mat, double* rhs, const rg_coef* A, const rg_coef* B,
                               const rg_coef* C, const rg_coef* D, const rg_coef* X, const rg_coef* Y);
/* assemblePDEBoundarySingle / assemblePDEBoundarySystem (DefaultAssembler3D.cpp:2232-2888,
   5753-6464): adds the face terms d (matrix) and y (rhs).  d/y are on FunctionOnBoundary:
   faces left,right,bottom,top(,front,back), face elements lower in-face axis fastest,
   2^(dim-1) Gauss points per face element.  For a matrix of block size bs the data points
   are d (bs, bs) = d[k + bs m] and y (bs); rhs has n bs entries. */
int rg_assemble_boundary(rg_matrix* mat, double* rhs, const rg_coef* d, const rg_coef* y);
/* assemblePDEBoundarySingleReduced / assemblePDEBoundarySystemReduced (DefaultAssembler3D.cpp:
   3274-3628, 6878-7255): the face terms for d_reduced / y_reduced on
   ReducedFunctionOnBoundary, one data point per face element, 1-point rule at the face
   centre. */
int rg_assemble_boundary_reduced(rg_matrix* mat, double* rhs, const rg_coef* d, const rg_coef* y);

/* LinearPDE.insertConstraint(rhs_only=0): rhs -= A*u with u = r on q>0 else 0; rows and
   columns with q>0 nullified with 1 on the diagonal; rhs[q>0] = r.  r may be NULL (= 0).
   With rhs_only=1 only rhs[q>0] = r is applied, as the reference does. */
int rg_insert_constraint(rg_matrix* mat, double* rhs, const double* q, const double* r,
                         int rhs_only);
/* SystemMatrix::nullifyRowsAndCols(mask_row, mask_col, main_diagonal_value) */
int rg_nullify_rows_and_cols(rg_matrix* mat, const double* mask_row, const double* mask_col,
                             double main_diagonal_value);
/* ypAx / MatrixVector: y = alpha*A*x + beta*y on the unbalanced matrix (paso throws for a
   balanced matrix: RG_INVALID_ARG here) */
int rg_spmv(rg_matrix* mat, double alpha, const double* x, double beta, double* y);
/* Brick/Rectangle::interpolateNodesOnElements: nodal (n x ncomp) -> Function
   (NE x Q x ncomp), or ReducedFunction (element mean) when reduced != 0 */
int rg_interpolate_nodes(const rg_domain* dom, const double* nodal, int ncomp, double* out,
                         int reduced);
/* norms of rhs - A*x with A the matrix as assembled (also after a solve balanced it in
   place), like Lsup/L2 of LinearPDE.getResidual (escriptcore/py_src/linearPDEs.py).  The
   reduction scratch is allocated with the matrix on first use. */
int rg_residual_norms(rg_matrix* mat, const double* rhs, const double* x, double* l2_host,
                      double* linf_host);
/* The same residual norms computed without any device allocation: the reduction scratch
   is a fixed static device array (18,976 bytes, at most 1184 CTAs' partial sums) that every
   GPU loading the library holds until exit.  No counterpart in the reference: it is for
   callers that cannot let a library call cudaMalloc (a host whose own pool owns the
   device memory, or a latency-critical loop that cannot absorb the implicit
   synchronisation of cudaMalloc/cudaFree).  All calls share the array: calls that overlap
   on the GPU race and must be serialised.  The first call on a device looks up the array's
   address (make it before any stream capture); a call whose device work fails forgets it,
   so a call after cudaDeviceReset looks it up again.  The reduction grid is capped at 1184
   CTAs for any size, so every size fits the array; should that cap ever exceed it, the call
   returns RG_INVALID_ARG instead of writing past the array.  PDE systems (block size > 1):
   RG_NOT_SUPPORTED. */
int rg_residual_norms_noalloc(rg_matrix* mat, const double* rhs, const double* x,
                              double* l2_host, double* linf_host);
/* SystemMatrix::saveMM (paso/src/SystemMatrix.h:70-80 -> SparseMatrix<double>::saveMM,
   paso/src/SparseMatrix.cpp:180-240): MatrixMarket coordinate real general, 1-based, the
   values as they are now (balanced in place after a solve, as in paso), entries in paso's
   order: node rows, their pattern entries, then block row and block column. */
int rg_save_mm(rg_matrix* mat, const char* path);

/* ---- solver: SolverBuddy subset + paso Options (escriptcore/src/SolverOptions.cpp:40-70) */
#define RG_METHOD_PCG 10          /* SolverOptions.PCG                                       */
#define RG_PRECOND_JACOBI 20      /* SolverOptions.JACOBI                                    */
#define RG_MODE_PASO 0            /* paso Solver(): balance, Jacobi initial guess, smoothed
                                     residual PCG, dual-norm outer test (Solver.cpp:186-322)*/
#define RG_MODE_STANDARD 1        /* textbook Jacobi-PCG on the balanced system, same outer
                                     dual-norm test, optional initial guess               */
#define RG_PREC_FP64 0            /* all FP64                                                */
#define RG_PREC_FP32_REFINE 1     /* FP32 inner PCG, FP64 residual/update/stop test         */
#define RG_LAYOUT_CSR 0           /* inner SpMV on the paso CSR values                       */
#define RG_LAYOUT_BAND 1          /* SpMV on a 27-band (9 in 2D) structured copy: FP32_REFINE
                                     always; FP64 solves (paso or standard mode) with this
                                     layout stream an FP64 band copy (8 bytes per coefficient
                                     against the CSR's 12).  Scalar PDEs only: systems
                                     (block size 2, 3) always use the block CSR            */
#define RG_LAYOUT_COEF 2          /* FP32_REFINE only: the FP32 inner PCG evaluates the operator
                                     from the element coefficients instead of streaming stored
                                     values (4 bytes per row instead of 108), when the matrix's
                                     values are what the library recorded while building them:
                                     interior assemblies of A = kappa I per element (CONSTANT,
                                     PER_ELEMENT, or EXPANDED with one value per element) with
                                     no B, C, D, then insertConstraint.  Otherwise (other
                                     coefficients, face terms, nullifyRowsAndCols, reduced
                                     order) the band copy is used (rg_diag.inner_operator).
                                     Values changed through rg_matrix_values' pointer are not
                                     seen: the FP64 outer residual then stops improving and
                                     the solve finishes in FP64 (rg_diag.fp64_fallback), so
                                     results stay correct.  FP64 solves: RG_NOT_SUPPORTED. */

typedef struct {
    int method;                 /* RG_METHOD_PCG                                            */
    int preconditioner;         /* RG_PRECOND_JACOBI                                        */
    double tolerance;           /* relative tolerance, default 1e-8                         */
    int64_t iter_max;           /* default 100000                                           */
    int sweeps;                 /* Jacobi sweeps, default 1 (> 1: paso mode, FP64)          */
    int verbose;                /* print per-step residuals like paso                       */
    int accept_convergence_failure;
    int mode;                   /* RG_MODE_*                                                */
    int precision;              /* RG_PREC_*                                                */
    int layout;                 /* RG_LAYOUT_*                                              */
    double inner_tolerance;     /* FP32_REFINE: reduction of the FP32 recursive residual    
                                   between FP64 residual replacements (default 1e-2)      */
    const double* initial_guess;/* STANDARD mode only: device x0 (unbalanced units) or NULL;
                                   dropped for zero when ||B(b - A x0)|| > ||B b||          */
    int guess_sweeps;           /* Chebyshev smoothing steps (Jacobi-preconditioned, on the
                                   upper 29/30 of the Gershgorin range) applied to
                                   initial_guess before that test; default 0               */
} rg_solver_opts;

typedef struct {
    int64_t num_iter;           /* total inner iterations (SolverBuddy num_iter)            */
    int64_t num_outer;          /* outer residual steps                                     */
    double residual_norm;       /* last l2 norm of the balanced true residual               */
    double residual_max;        /* last max norm of the balanced true residual              */
    double rhs_norm;            /* l2 norm of the balanced right hand side                  */
    int converged;
    double time;                /* seconds, whole solve (SolverBuddy time)                  */
    double set_up_time;         /* balancing + preconditioner                               */
    double net_time;            /* iterations                                               */
    double guess_residual;      /* l2 norm of the balanced residual of the initial guess    */
    int guess_rejected;         /* 1: the guess's residual exceeded the right hand side's
                                   and the solve started from zero instead                  */
    int fp64_fallback;          /* FP32_REFINE: 1 when the FP32 corrections stopped reducing
                                   the FP64 residual and the solve finished in FP64 PCG     */
    int inner_operator;         /* FP32_REFINE: the operator of the FP32 iterations, 1 = the
                                   element coefficients (RG_LAYOUT_COEF), 0 = the band copy */
} rg_diag;

void rg_solver_opts_default(rg_solver_opts* opts);
/* setToSolution: x (n doubles) = A^-1 rhs.  rhs is not modified.  The matrix is
   balanced in place on the first solve, as paso does; later solves reuse it. */
int rg_solve(rg_matrix* mat, const double* rhs, double* x, const rg_solver_opts* opts,
             rg_diag* diag);


/* The FP32 path's configuration chosen at the matrix's first FP32_REFINE solve (no reference
   counterpart; diagnostics and tests), for the inner operator of the matrix's latest solve:
   spmv_config 0/1 = the pipeline of the fused FP32 PCG iteration (one kernel per iteration:
   operator product, vector updates and one reduction) with 3 stages x 1 CTA per SM / 2 stages
   x 2 CTAs per SM on the band copy, 3 stages x 2 CTAs per SM / 2 stages x 2 CTAs per SM on the
   element coefficients (-1: not tuned yet); update_grid: 0 (the iteration has no separate
   vector-update kernel); spmv_us (NULL or 2 entries): the tuner's time per iteration of each
   configuration, 0 where not timed (a configuration whose shared memory does not fit the
   grid's windows is not timed).  Any output pointer may be NULL. */
int rg_solver_config(const rg_matrix* mat, int* spmv_config, int* update_grid, double* spmv_us);

/* Fixes the FP32 iteration configuration used from the next FP32_REFINE solve on (-1 restores
   the tuner's choice; a configuration that does not fit the grid makes that solve return
   RG_INVALID_ARG).  The tuner still times every configuration that fits, so rg_solver_config
   reports them. */
int rg_solver_set_config(rg_matrix* mat, int spmv_config);

/* Test hook for the timeout path of the warp-specialised kernels (no reference counterpart;
   paso has no device waits).  max_polls > 0 caps the polls of each bounded wait of the band
   kernels (FP32_REFINE, and FP64 with RG_LAYOUT_BAND) and of the persistent convolution of
   rg_ws_conv3; 0 restores the default limit.  withhold_copies != 0 makes their producers
   issue no copies, so every wait runs out with nothing in flight: a solve then returns
   RG_TIMEOUT, a convolution sets its device error flag, and the matrix, its domain and the
   library stay usable.  Applies to all matrices on the current device from the next launch
   on; it waits for the device to be idle first.  Not for use in production code. */
int rg_test_wait_limit(int max_polls, int withhold_copies);

/* ---- batched solves (no reference counterpart: many independent systems at once) ------- */
/* A batch holds assembled matrices of the same dimension (any sizes) that are solved
   together, each with nrhs right hand sides (1, 2, 4 or 8), by PCG + Jacobi with FP32 inner
   iterations and FP64 refinement: paso's dual-norm stopping test per right hand side.  The
   matrices are balanced and prepared at creation; they must not change while the batch
   lives.  Every kernel launch advances all systems; chunks of iterations replay as CUDA
   graphs; grid sizes and the chunk length come from rg_batch_tune (run by the first solve
   when not called). */
typedef struct rg_batch rg_batch;
int rg_batch_create(rg_matrix* const* mats, int nsystems, int nrhs, rg_batch** out);
int rg_batch_destroy(rg_batch* batch);
int rg_batch_tune(rg_batch* batch);
/* rows: padded batch rows; tiles: 256-row tiles; group: tiles per work unit of the
   iteration kernels; grids in CTAs; iter_us: measured time of one iteration of all systems
   at the tuned configuration; spmv_kernel: 0 = one row per thread, 1 = two rows per thread.
   Any output pointer may be NULL. */
int rg_batch_info(const rg_batch* batch, int64_t* rows, int64_t* tiles, int* group, int* grid_spmv,
                  int* grid_update, int* chunk, double* iter_us, int* spmv_kernel);
/* Restricts the tuner to one SpMV kernel (0 or 1 as in rg_batch_info; -1: either, the
   default); the next solve or rg_batch_tune re-tunes. */
int rg_batch_set_spmv(rg_batch* batch, int spmv_kernel);
/* rhs[i], x[i]: device arrays of n_i * nrhs doubles for system i, right hand side k at
   offset k * n_i.  opts: tolerance, iter_max, inner_tolerance, accept_convergence_failure
   (NULL: defaults).  diag: nsystems * nrhs entries (system-major) or NULL. */
int rg_batch_solve(rg_batch* batch, const double* const* rhs, double* const* x, const rg_solver_opts* opts,
                   rg_diag* diag);

/* ---- instrumentation ------------------------------------------------------------------ */
/* Every kernel launch of the library is counted per kind; with timers enabled each launch
   is also bracketed by CUDA events on its stream.  rg_timers_read folds finished events
   into the totals (it waits for them).  Kinds are 0..rg_timers_count()-1. */
int rg_timers_enable(int on);
int rg_timers_reset(void);
int rg_timers_count(void);
const char* rg_timer_name(int kind);
int rg_timers_read(int kind, int64_t* launches, int64_t* timed, double* total_ms);

/* ---- warm-start network: tensor-core 3x3x3 convolutions (bf16, fp32 accumulation) ------ */
/* bf16 channels-last activations with one zero slice before and after every sample along
   depth: element (n, d, h, w, c) at ptr[(((n*(d_+2) + 1 + d)*h_ + h)*w_ + w)*c_ + c]. */
typedef struct {
    void* ptr;
    int n, d, h, w, c;
} rg_act;
/* y = act(conv3x3x3(x, weights) + bias) with zero padding.  weights: bf16 [27][c_out][c_in],
   tap = kw + 3 kh + 9 kd.  relu != 0 applies max(0, .); mask (shape of y) zeroes the
   outputs where mask <= 0 (ReLU derivative of the layer below, for data gradients).
   x->c a multiple of 16; y->c one of 16, 32, 48, 64, 80, 112, 128; spatial sizes must tile
   into 128-position boxes.  *err_dev is set non-zero when a bounded device wait gave up. */
int rg_ws_conv3(const rg_act* x, const void* weights, const float* bias, rg_act* y, int relu,
                const rg_act* mask, int* err_dev);
/* Weight gradient of rg_ws_conv3: dw[tap][c_out][c_in] (fp32) = sum over positions p of
   g(p, c_out) x(p + offset(tap), c_in), g the gradient at the conv output (after the ReLU
   mask).  Split over position tiles; the splits' partial sums go to `partials`
   (partials_floats floats; more lets more CTAs run) and are added in a fixed order, so the
   result is deterministic.  accumulate != 0 adds into dw.  Spatial sizes must tile into
   64-position boxes.  Data gradients are rg_ws_conv3 of g with rg_ws_weights_bf16's
   flipped weights and the mask of the layer below. */
int rg_ws_conv3_wgrad(const rg_act* x, const rg_act* g, float* dw, float* partials,
                      int64_t partials_floats, int accumulate, int* err_dev);

/* Memory-bound layers of the network (all on the library stream, bf16 activations). */
/* out = 2x2x2 average of in (out spatial sizes are half of in's) */
int rg_ws_avgpool(const rg_act* in, rg_act* out);
/* din = (dout upsampled / 8 [+ dskip channels skip_off..]) where in > 0, else 0; dskip may be
   NULL (the gradient reaching a pooled tensor's skip connection) */
int rg_ws_avgpool_bwd(const rg_act* dout, const rg_act* in, const rg_act* dskip, int skip_off,
                      rg_act* din);
/* out = concat(nearest-upsample-2x(a), b) along channels */
int rg_ws_upcat(const rg_act* a, const rg_act* b, rg_act* out);
/* da = sum over each parent's 8 children of dcat's first da->c channels, zero where the
   upsampled tensor a <= 0 (its ReLU derivative; a may be NULL) */
int rg_ws_upcat_bwd(const rg_act* dcat, const rg_act* a, rg_act* da);
/* 1x1x1 output head: out[pos] = b[0] + sum_c w[c] x(pos, c); out fp32 [n][d][h][w] */
int rg_ws_head(const rg_act* x, const float* w, const float* b, float* out);
/* dx(pos, c) = w[c] dout[pos] where x(pos, c) > 0, else 0 */
int rg_ws_head_bwd_x(const rg_act* x, const float* w, const float* dout, rg_act* dx);
/* out[c] (+)= sum over positions of v(pos, c) [* dout[pos] when dout != NULL]; bias gradients
   (dout NULL) and the head's weight gradient.  work: 592 * v->c floats, v->c <= 128 */
int rg_ws_colsum(const rg_act* v, const float* dout, float* out, float* work, int accumulate);
/* *loss_dev = mean (out - target)^2 (fp64), dout = its gradient, *dsum_dev = sum of dout
   (may be NULL); work: 1184 doubles */
int rg_ws_mse(const float* out, const float* target, int64_t count, float* dout, double* loss_dev,
              float* dsum_dev, double* work);
/* as rg_ws_mse on an (n, d, h, w) grid with a gradient term: loss = (sum e_i^2 + lambda sum over
   face-adjacent cell pairs (e_i - e_j)^2) / count, e = out - target */
int rg_ws_h1_loss(const float* out, const float* target, int n, int d, int h, int w, float lambda, float* dout,
                  double* loss_dev, float* dsum_dev, double* work);
/* Adam step `step` (>= 1, bias-corrected) on fp32 master weights */
int rg_ws_adam(float* w, const float* g, float* m, float* v, int64_t count, float lr, float beta1,
               float beta2, float eps, int step);
/* fp32 weights [27][c_out][c_in] -> bf16 forward copy (same layout) and/or bf16 data-gradient
   copy [27][c_in][c_out] with taps reversed (tap' = 26 - tap); either output may be NULL */
int rg_ws_weights_bf16(const float* w, void* w_fwd, void* w_dgrad, int c_out, int c_in);
/* Glue between the PDE's fields and the network.  Fields are fp32 per element of a fine
   grid (x fastest, samples consecutive); the network grid is the fine grid coarsened by an
   integer factor.  rg_ws_field_stats writes 4 floats per sample: mu = mean log kappa,
   sY = max |Y|, kappa_g = exp(mu), u_unit = 10 sY h_net^2 / kappa_g (work: 128 * nsamples
   doubles).  The network sees (log kappa - mu, Y / sY) averaged over each of its cells and
   the cell centre's (z, y, x) in the unit cube (channels 0..4, x->c >= 5; others zero), and
   predicts u / u_unit per cell. */
int rg_ws_field_stats(const float* kappa, const float* y, int nsamples, int64_t per_sample, double h_net,
                      float* stats, double* work);
int rg_ws_pack_input(const float* kappa, const float* y, int factor, rg_act* x, const float* stats);
/* The per-element fields the network reads, from the PDE's coefficient arrays (device
   pointers): kappa[e] = A[e a_stride] (A's first entry: a_stride 9 for A per element, 72
   for A on the Gauss points, whose first point is taken), y[e] = mean of Y[e y_points ..
   e y_points + y_points - 1]; fp32 outputs, nel elements. */
int rg_ws_element_fields(const double* A, int a_stride, const double* Y, int y_points, int64_t nel, float* kappa,
                         float* y);
/* training target per network cell: mean of the nodal solution u (fp64, (f d+1)(f h+1)(f w+1)
   nodes per sample) over the cell, in units of u_unit */
int rg_ws_nodes_to_cells(const double* u, int factor, int nsamples, int d, int h, int w, const float* stats,
                         float* target);
/* initial guess on nd x nh x nw nodes per sample: trilinear interpolation of the cell values
   (cell centres, clamped at the faces) times u_unit; 0 where q > 0 (q may be NULL) */
int rg_ws_cells_to_nodes(const float* cells, int nsamples, int d, int h, int w, const float* stats, int nd, int nh,
                         int nw, const double* q, double* u);

#ifdef __cplusplus
}
#endif
#endif /* RIPLEY_GPU_H */
