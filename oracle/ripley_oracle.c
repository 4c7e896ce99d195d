/*
 * CPU oracle for the ripley Q1 assembly + paso PCG/Jacobi path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
 * baseline.  The product library never links or calls this file.
 *
 * Element matrices are written from the Q1 / 2x2(x2)-Gauss definition
 * (shape functions, their gradients at the Gauss points, quadrature weights),
 * not from the reference's closed-form expansions; the scatter, Dirichlet,
 * balancing and solver steps restate the reference algorithms in the order the
 * reference performs them.  Citations are file:line in the esys-escript tree.
 */
#include "ripley_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* pattern: Brick::getConnections(false) Brick.cpp:3000-3061,
            Rectangle::getConnections Rectangle.cpp:2035-2086                 */
/* ------------------------------------------------------------------------- */

int64_t ro_pattern_nnz(int dim, const int64_t nn[3])
{
    /* every axis contributes 3 neighbours per node except the two end nodes (2) */
    int64_t s = 1;
    for (int d = 0; d < dim; ++d) s *= 3 * nn[d] - 2;
    return s;
}

void ro_pattern(int dim, const int64_t nn[3], int32_t* ptr, int32_t* idx)
{
    const int64_t N0 = nn[0], N1 = nn[1], N2 = dim == 3 ? nn[2] : 1;
    int64_t k = 0, row = 0;
    ptr[0] = 0;
    for (int64_t z = 0; z < N2; ++z)
        for (int64_t y = 0; y < N1; ++y)
            for (int64_t x = 0; x < N0; ++x, ++row) {
                for (int64_t i2 = z - 1; i2 <= z + 1; ++i2) {
                    if (dim == 3 && (i2 < 0 || i2 >= N2)) continue;
                    if (dim == 2 && i2 != z) continue;
                    for (int64_t i1 = y - 1; i1 <= y + 1; ++i1) {
                        if (i1 < 0 || i1 >= N1) continue;
                        for (int64_t i0 = x - 1; i0 <= x + 1; ++i0) {
                            if (i0 < 0 || i0 >= N0) continue;
                            idx[k++] = (int32_t)(i0 + N0 * i1 + N0 * N1 * i2);
                        }
                    }
                }
                ptr[row + 1] = (int32_t)k;
            }
}

/* ------------------------------------------------------------------------- */
/* Q1 reference element and 2^dim Gauss rule                                  */
/* local node k: bit d of k is the node's offset along axis d                 */
/* (Brick.cpp:3243-3251, Rectangle.cpp addToMatrixAndRHS); quadrature point q */
/* likewise, x fastest (Brick.cpp:3375-3384), at (1 -/+ 1/sqrt(3))/2.         */
/* ------------------------------------------------------------------------- */

typedef struct {
    int dim, nk, nq;
    double N[8][8];     /* N[q][k]     shape function value */
    double G[8][8][3];  /* G[q][k][d]  physical gradient     */
    double W;           /* quadrature weight (all points equal) */
} q1_tab;

static void q1_build(int dim, const double dx[3], q1_tab* t)
{
    const double g[2] = {0.5 - sqrt(3.0) / 6.0, 0.5 + sqrt(3.0) / 6.0};
    t->dim = dim;
    t->nk = 1 << dim;
    t->nq = 1 << dim;
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= dx[d];
    t->W = vol / t->nq;
    for (int q = 0; q < t->nq; ++q) {
        double xi[3];
        for (int d = 0; d < dim; ++d) xi[d] = g[(q >> d) & 1];
        for (int k = 0; k < t->nk; ++k) {
            double f[3], df[3];
            for (int d = 0; d < dim; ++d) {
                const int b = (k >> d) & 1;
                f[d] = b ? xi[d] : 1.0 - xi[d];
                df[d] = (b ? 1.0 : -1.0) / dx[d];
            }
            double v = 1.0;
            for (int d = 0; d < dim; ++d) v *= f[d];
            t->N[q][k] = v;
            for (int d = 0; d < dim; ++d) {
                double gd = df[d];
                for (int e = 0; e < dim; ++e)
                    if (e != d) gd *= f[e];
                t->G[q][k][d] = gd;
            }
        }
    }
}

/* The 1-point rule of the reduced-order assembly (assemblePDESingleReduced,
   DefaultAssembler3D.cpp:2891-3271, DefaultAssembler2D.cpp:842-1010): the element centre
   with weight = element volume. */
static void q1_build_reduced(int dim, const double dx[3], q1_tab* t)
{
    t->dim = dim;
    t->nk = 1 << dim;
    t->nq = 1;
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= dx[d];
    t->W = vol;
    for (int k = 0; k < t->nk; ++k) {
        t->N[0][k] = 1.0 / t->nk;
        for (int d = 0; d < dim; ++d) {
            double gd = (((k >> d) & 1) ? 1.0 : -1.0) / dx[d];
            for (int e = 0; e < dim; ++e)
                if (e != d) gd *= 0.5;
            t->G[0][k][d] = gd;
        }
    }
}

/* value of component c of a coefficient at quadrature point q of element e */
static inline double coef_at(ro_coef a, int size, int nq, int64_t e, int c, int q)
{
    switch (a.kind) {
    case RO_CONSTANT: return a.p[c];
    case RO_PER_ELEMENT: return a.p[(int64_t)size * e + c];
    case RO_EXPANDED: return a.p[(int64_t)size * nq * e + (int64_t)size * q + c];
    default: return 0.0;
    }
}

/* Element matrix EM_S[r + nk*c] and vector EM_F[r] of
      -(A_ij u_,j + B_i u)_,i + C_j u_,j + D u = -X_i,i + Y
   i.e. EM_S = sum_q W (A_ij G_ri G_cj + B_i G_ri N_c + C_j N_r G_cj + D N_r N_c),
        EM_F = sum_q W (X_i G_ri + Y N_r)
   Coefficient layouts follow escript: A[i + dim*j (+ dim^2*q)], B/C/X[i (+dim*q)],
   D/Y[q] (DefaultAssembler3D.cpp:260-331, 1851-1860, 2168-2176). */
static void element_single(const q1_tab* t, int64_t e, ro_coef A, ro_coef B, ro_coef C,
                           ro_coef D, ro_coef X, ro_coef Y, double* EM_S, double* EM_F)
{
    const int dim = t->dim, nk = t->nk, nq = t->nq;
    memset(EM_S, 0, sizeof(double) * 64);
    memset(EM_F, 0, sizeof(double) * 8);
    for (int q = 0; q < nq; ++q) {
        double a[9] = {0}, b[3] = {0}, c[3] = {0}, dq = 0.0, xq[3] = {0}, yq = 0.0;
        if (A.kind) for (int m = 0; m < dim * dim; ++m) a[m] = coef_at(A, dim * dim, nq, e, m, q);
        if (B.kind) for (int m = 0; m < dim; ++m) b[m] = coef_at(B, dim, nq, e, m, q);
        if (C.kind) for (int m = 0; m < dim; ++m) c[m] = coef_at(C, dim, nq, e, m, q);
        if (D.kind) dq = coef_at(D, 1, nq, e, 0, q);
        if (X.kind) for (int m = 0; m < dim; ++m) xq[m] = coef_at(X, dim, nq, e, m, q);
        if (Y.kind) yq = coef_at(Y, 1, nq, e, 0, q);
        for (int r = 0; r < nk; ++r) {
            const double* Gr = t->G[q][r];
            const double Nr = t->N[q][r];
            /* row vector a^T-contracted with grad phi_r: s_j = sum_i A_ij G_ri */
            double s[3] = {0, 0, 0};
            double bg = 0.0;
            for (int j = 0; j < dim; ++j)
                for (int i = 0; i < dim; ++i) s[j] += a[i + dim * j] * Gr[i];
            for (int i = 0; i < dim; ++i) bg += b[i] * Gr[i];
            for (int cc = 0; cc < nk; ++cc) {
                const double* Gc = t->G[q][cc];
                const double Nc = t->N[q][cc];
                double v = 0.0;
                for (int j = 0; j < dim; ++j) v += (s[j] + Nr * c[j]) * Gc[j];
                v += bg * Nc + dq * Nr * Nc;
                EM_S[r + nk * cc] += t->W * v;
            }
            double f = yq * Nr;
            for (int i = 0; i < dim; ++i) f += xq[i] * Gr[i];
            EM_F[r] += t->W * f;
        }
    }
}

/* addToPasoMatrix (RipleyDomain.cpp:1488-1614), CSR branch, block size 1: for every
   (row, col) pair of the element a linear search of the row's column list. */
static void scatter(int nk, const int64_t* nodes, const int32_t* ptr, const int32_t* idx,
                    double* val, double* rhs, const double* EM_S, const double* EM_F,
                    int addS, int addF)
{
    if (addF && rhs)
        for (int r = 0; r < nk; ++r) rhs[nodes[r]] += EM_F[r];
    if (addS && val)
        for (int r = 0; r < nk; ++r) {
            const int64_t row = nodes[r];
            for (int c = 0; c < nk; ++c) {
                const int32_t col = (int32_t)nodes[c];
                for (int64_t k = ptr[row]; k < ptr[row + 1]; ++k)
                    if (idx[k] == col) { val[k] += EM_S[r + nk * c]; break; }
            }
        }
}

/* DefaultAssembler3D::assemblePDESingle (DefaultAssembler3D.cpp:152-2226) and the 2D
   analogue (DefaultAssembler2D.cpp:151-597): two colours of z-slabs (y-rows in 2D),
   elements in k2,k1,k0 order inside a colour; element node order as in
   Brick::addToMatrixAndRHS (Brick.cpp:3238-3265). */
static void assemble_with(const q1_tab* tp, int dim, const int64_t ne[3], const int32_t* ptr,
                          const int32_t* idx, double* val, double* rhs, ro_coef A, ro_coef B,
                          ro_coef C, ro_coef D, ro_coef X, ro_coef Y);

void ro_assemble_single(int dim, const int64_t ne[3], const double dx[3],
                        const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                        ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y)
{
    q1_tab t;
    q1_build(dim, dx, &t);
    assemble_with(&t, dim, ne, ptr, idx, val, rhs, A, B, C, D, X, Y);
}

/* DefaultAssembler3D::assemblePDESingleReduced (DefaultAssembler3D.cpp:2891-3271) and
   DefaultAssembler2D::assemblePDESingleReduced (DefaultAssembler2D.cpp:842-1010): the same
   element formula with the 1-point rule; coefficients on ReducedFunction (one value set
   per element, or constant). */
void ro_assemble_single_reduced(int dim, const int64_t ne[3], const double dx[3],
                                const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                                ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y)
{
    q1_tab t;
    q1_build_reduced(dim, dx, &t);
    assemble_with(&t, dim, ne, ptr, idx, val, rhs, A, B, C, D, X, Y);
}

static void assemble_with(const q1_tab* tp, int dim, const int64_t ne[3], const int32_t* ptr,
                          const int32_t* idx, double* val, double* rhs, ro_coef A, ro_coef B,
                          ro_coef C, ro_coef D, ro_coef X, ro_coef Y)
{
    const q1_tab t = *tp;
    const int addS = A.kind || B.kind || C.kind || D.kind;
    const int addF = X.kind || Y.kind;
    if (!addS && !addF) return;
    const int64_t NE0 = ne[0], NE1 = ne[1], NE2 = dim == 3 ? ne[2] : 1;
    const int64_t NN0 = NE0 + 1, NN1 = NE1 + 1;
    const int64_t outer = dim == 3 ? NE2 : NE1;
    for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
        for (int64_t ko = colour; ko < outer; ko += 2) {
            double EM_S[64], EM_F[8];
            int64_t nodes[8];
            const int64_t k1lo = dim == 3 ? 0 : ko, k1hi = dim == 3 ? NE1 : ko + 1;
            const int64_t k2 = dim == 3 ? ko : 0;
            for (int64_t k1 = k1lo; k1 < k1hi; ++k1)
                for (int64_t k0 = 0; k0 < NE0; ++k0) {
                    const int64_t e = k0 + NE0 * k1 + NE0 * NE1 * k2;
                    element_single(&t, e, A, B, C, D, X, Y, EM_S, EM_F);
                    const int64_t first = k0 + NN0 * k1 + NN0 * NN1 * k2;
                    for (int k = 0; k < t.nk; ++k)
                        nodes[k] = first + (k & 1) + ((k >> 1) & 1) * NN0 +
                                   ((k >> 2) & 1) * NN0 * NN1;
                    scatter(t.nk, nodes, ptr, idx, val, rhs, EM_S, EM_F, addS, addF);
                }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* boundary terms d, y: DefaultAssembler3D::assemblePDEBoundarySingle          */
/* (DefaultAssembler3D.cpp:2232-2888), DefaultAssembler2D.cpp:600-1010.        */
/* Faces in ripley order left,right,bottom,top,front,back (x=0,x=L0,y=0,...);   */
/* face element f within face numbered with the lower in-face axis fastest     */
/* (Brick.cpp:1399-1480); face data offset of face i = sum of earlier counts.  */
/* Face Gauss points: 2 per in-face axis, lower in-face axis fastest.          */
/* ------------------------------------------------------------------------- */

void ro_assemble_boundary(int dim, const int64_t ne[3], const double dx[3],
                          const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                          ro_coef d, ro_coef y)
{
    const int addS = d.kind != RO_EMPTY, addF = y.kind != RO_EMPTY;
    if (!addS && !addF) return;
    const double g[2] = {0.5 - sqrt(3.0) / 6.0, 0.5 + sqrt(3.0) / 6.0};
    const int nk = 1 << dim;
    const int nqf = 1 << (dim - 1);
    const int64_t NE[3] = {ne[0], ne[1], dim == 3 ? ne[2] : 1};
    const int64_t NN0 = NE[0] + 1, NN1 = NE[1] + 1;
    int64_t offset = 0;
    for (int face = 0; face < 2 * dim; ++face) {
        const int ax = face / 2, side = face % 2;
        /* in-face axes, lower first */
        int fa[2] = {-1, -1}, nf = 0;
        for (int a = 0; a < dim; ++a)
            if (a != ax) fa[nf++] = a;
        const int64_t n_a = NE[fa[0]], n_b = dim == 3 ? NE[fa[1]] : 1;
        double area = 1.0;
        for (int i = 0; i < nf; ++i) area *= dx[fa[i]];
        const double W = area / nqf;
        /* face shape-function values on the face Gauss points, for the nk element
           nodes (nodes off the face are zero) */
        double Nf[4][8];
        for (int q = 0; q < nqf; ++q)
            for (int k = 0; k < nk; ++k) {
                if (((k >> ax) & 1) != side) { Nf[q][k] = 0.0; continue; }
                double v = 1.0;
                for (int i = 0; i < nf; ++i) {
                    const double xi = g[(q >> i) & 1];
                    v *= ((k >> fa[i]) & 1) ? xi : 1.0 - xi;
                }
                Nf[q][k] = v;
            }
        for (int colour = 0; colour < 2; ++colour) {
            const int64_t outer = dim == 3 ? n_b : n_a;
#pragma omp parallel for schedule(static)
            for (int64_t ko = colour; ko < outer; ko += 2) {
                double EM_S[64], EM_F[8];
                int64_t nodes[8];
                const int64_t alo = dim == 3 ? 0 : ko, ahi = dim == 3 ? n_a : ko + 1;
                const int64_t kb = dim == 3 ? ko : 0;
                for (int64_t ka = alo; ka < ahi; ++ka) {
                    const int64_t f = offset + ka + n_a * kb;
                    const int64_t floc = ka + n_a * kb;
                    int64_t k[3] = {0, 0, 0};
                    k[ax] = side ? NE[ax] - 1 : 0;
                    k[fa[0]] = ka;
                    if (dim == 3) k[fa[1]] = kb;
                    memset(EM_S, 0, sizeof(EM_S));
                    memset(EM_F, 0, sizeof(EM_F));
                    for (int q = 0; q < nqf; ++q) {
                        const double dq = addS ? coef_at(d, 1, nqf, f, 0, q) : 0.0;
                        const double yq = addF ? coef_at(y, 1, nqf, f, 0, q) : 0.0;
                        for (int r = 0; r < nk; ++r) {
                            if (Nf[q][r] == 0.0) continue;
                            EM_F[r] += W * yq * Nf[q][r];
                            for (int c = 0; c < nk; ++c)
                                EM_S[r + nk * c] += W * dq * Nf[q][r] * Nf[q][c];
                        }
                    }
                    (void)floc;
                    const int64_t first = k[0] + NN0 * k[1] + NN0 * NN1 * k[2];
                    for (int m = 0; m < nk; ++m)
                        nodes[m] = first + (m & 1) + ((m >> 1) & 1) * NN0 +
                                   ((m >> 2) & 1) * NN0 * NN1;
                    scatter(nk, nodes, ptr, idx, val, rhs, EM_S, EM_F, addS, addF);
                }
            }
        }
        offset += n_a * n_b;
    }
}

/* The face terms in general form: block size nb (assemblePDEBoundarySystem,
   DefaultAssembler3D.cpp:5753-6464; EM_S[k + nb (m + nb (r + nk c))] from
   d[k + nb m] per data point, EM_F[k + nb r] from y[k]) and, with `reduced`, the 1-point
   rule at the face centre with weight = face area (assemblePDEBoundarySingleReduced,
   DefaultAssembler3D.cpp:3274-3628, assemblePDEBoundarySystemReduced, 6878-7255: d, y have
   one data point per face element). */
void ro_assemble_boundary_ex(int dim, const int64_t ne[3], const double dx[3], int nb, int reduced,
                             const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                             ro_coef d, ro_coef y)
{
    const int addS = d.kind != RO_EMPTY, addF = y.kind != RO_EMPTY;
    if (!addS && !addF) return;
    const double g2[2] = {0.5 - sqrt(3.0) / 6.0, 0.5 + sqrt(3.0) / 6.0};
    const double g1[2] = {0.5, 0.5};
    const double* g = reduced ? g1 : g2;
    const int nk = 1 << dim;
    const int nqf = reduced ? 1 : 1 << (dim - 1);
    const int bs = nb * nb;
    const int64_t NE[3] = {ne[0], ne[1], dim == 3 ? ne[2] : 1};
    const int64_t NN0 = NE[0] + 1, NN1 = NE[1] + 1;
    int64_t offset = 0;
    for (int face = 0; face < 2 * dim; ++face) {
        const int ax = face / 2, side = face % 2;
        int fa[2] = {-1, -1}, nf = 0;
        for (int a = 0; a < dim; ++a)
            if (a != ax) fa[nf++] = a;
        const int64_t n_a = NE[fa[0]], n_b = dim == 3 ? NE[fa[1]] : 1;
        double area = 1.0;
        for (int i = 0; i < nf; ++i) area *= dx[fa[i]];
        const double W = area / nqf;
        double Nf[4][8];
        for (int q = 0; q < nqf; ++q)
            for (int k = 0; k < nk; ++k) {
                if (((k >> ax) & 1) != side) { Nf[q][k] = 0.0; continue; }
                double v = 1.0;
                for (int i = 0; i < nf; ++i) {
                    const double xi = g[(q >> i) & 1];
                    v *= ((k >> fa[i]) & 1) ? xi : 1.0 - xi;
                }
                Nf[q][k] = v;
            }
        for (int colour = 0; colour < 2; ++colour) {
            const int64_t outer = dim == 3 ? n_b : n_a;
#pragma omp parallel for schedule(static)
            for (int64_t ko = colour; ko < outer; ko += 2) {
                double EM_S[9 * 64], EM_F[3 * 8];
                int64_t nodes[8];
                const int64_t alo = dim == 3 ? 0 : ko, ahi = dim == 3 ? n_a : ko + 1;
                const int64_t kb = dim == 3 ? ko : 0;
                for (int64_t ka = alo; ka < ahi; ++ka) {
                    const int64_t f = offset + ka + n_a * kb;
                    int64_t k[3] = {0, 0, 0};
                    k[ax] = side ? NE[ax] - 1 : 0;
                    k[fa[0]] = ka;
                    if (dim == 3) k[fa[1]] = kb;
                    memset(EM_S, 0, sizeof(double) * (size_t)(bs * nk * nk));
                    memset(EM_F, 0, sizeof(double) * (size_t)(nb * nk));
                    for (int q = 0; q < nqf; ++q)
                        for (int kk = 0; kk < nb; ++kk) {
                            const double yq = addF ? coef_at(y, nb, nqf, f, kk, q) : 0.0;
                            for (int r = 0; r < nk; ++r) {
                                if (Nf[q][r] == 0.0) continue;
                                EM_F[kk + nb * r] += W * yq * Nf[q][r];
                                for (int m = 0; m < nb && addS; ++m) {
                                    const double dq = coef_at(d, bs, nqf, f, kk + nb * m, q);
                                    for (int c = 0; c < nk; ++c)
                                        EM_S[kk + nb * (m + nb * (r + nk * c))] += W * dq * Nf[q][r] * Nf[q][c];
                                }
                            }
                        }
                    const int64_t first = k[0] + NN0 * k[1] + NN0 * NN1 * k[2];
                    for (int m = 0; m < nk; ++m)
                        nodes[m] = first + (m & 1) + ((m >> 1) & 1) * NN0 + ((m >> 2) & 1) * NN0 * NN1;
                    if (addF && rhs)
                        for (int r = 0; r < nk; ++r)
                            for (int ir = 0; ir < nb; ++ir) rhs[nodes[r] * nb + ir] += EM_F[ir + nb * r];
                    if (addS && val)
                        for (int r = 0; r < nk; ++r)
                            for (int c = 0; c < nk; ++c) {
                                if (Nf[0][r] == 0.0 || Nf[0][c] == 0.0) continue;
                                for (int64_t kk = ptr[nodes[r]]; kk < ptr[nodes[r] + 1]; ++kk)
                                    if (idx[kk] == nodes[c]) {
                                        for (int ic = 0; ic < nb; ++ic)
                                            for (int ir = 0; ir < nb; ++ir)
                                                val[kk * bs + ir + nb * ic] += EM_S[ir + nb * (ic + nb * (r + nk * c))];
                                        break;
                                    }
                            }
                }
            }
        }
        offset += n_a * n_b;
    }
}

/* ------------------------------------------------------------------------- */
/* Brick::interpolateNodesOnElementsWorker (Brick.cpp:3355-3391) and the       */
/* Rectangle analogue: trilinear (bilinear) interpolation to the Gauss points. */
/* ------------------------------------------------------------------------- */

void ro_interpolate_nodes(int dim, const int64_t ne[3], const double* nodal, int ncomp,
                          double* out)
{
    q1_tab t;
    const double dx1[3] = {1.0, 1.0, 1.0};
    q1_build(dim, dx1, &t);
    const int64_t NE0 = ne[0], NE1 = ne[1], NE2 = dim == 3 ? ne[2] : 1;
    const int64_t NN0 = NE0 + 1, NN1 = NE1 + 1;
#pragma omp parallel for schedule(static)
    for (int64_t k2 = 0; k2 < NE2; ++k2)
        for (int64_t k1 = 0; k1 < NE1; ++k1)
            for (int64_t k0 = 0; k0 < NE0; ++k0) {
                const int64_t e = k0 + NE0 * k1 + NE0 * NE1 * k2;
                const int64_t first = k0 + NN0 * k1 + NN0 * NN1 * k2;
                for (int c = 0; c < ncomp; ++c)
                    for (int q = 0; q < t.nq; ++q) {
                        double v = 0.0;
                        for (int k = 0; k < t.nk; ++k) {
                            const int64_t node = first + (k & 1) + ((k >> 1) & 1) * NN0 +
                                                 ((k >> 2) & 1) * NN0 * NN1;
                            v += t.N[q][k] * nodal[node * ncomp + c];
                        }
                        out[(e * t.nq + q) * ncomp + c] = v;
                    }
            }
}

/* ------------------------------------------------------------------------- */
/* paso SpMV and vector kernels                                               */
/* ------------------------------------------------------------------------- */

void ro_spmv(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
             double alpha, const double* in, double beta, double* out)
{
    /* SparseMatrix_MatrixVector_CSR_OFFSET0_stripe (SparseMatrix_MatrixVector.cpp:243-266) */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double o = fabs(beta) > 0 ? (beta != 1.0 ? out[i] * beta : out[i]) : 0.0;
        if (fabs(alpha) > 0) {
            double reg = 0.0;
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) reg += val[k] * in[idx[k]];
            o += alpha * reg;
        }
        out[i] = o;
    }
}

void ro_insert_constraint(int64_t n, const int32_t* ptr, const int32_t* idx, double* val,
                          double* rhs, const double* q, const double* r)
{
    double* u = (double*)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) u[i] = (q[i] > 0 && r) ? r[i] : 0.0;
    if (val && rhs) ro_spmv(n, ptr, idx, val, -1.0, u, 1.0, rhs);
    if (val) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int64_t j = idx[k];
                if (q[j] > 0. || q[i] > 0.) val[k] = (i == j) ? 1.0 : 0.0;
            }
    }
    if (rhs)
        for (int64_t i = 0; i < n; ++i)
            if (q[i] > 0) rhs[i] = r ? r[i] : 0.0;
    free(u);
}

/* static row stripes as paso's OpenMP loops use (PCG.cpp:86-96): thread p owns
   [len*p + min(p,rest), len*(p+1) + min(p+1,rest)).  Partial sums are combined in
   thread order, which equals the reference at one thread. */
static int nthreads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define STRIPE_BEGIN(n, np, p) ((n) / (np) * (p) + ((p) < (n) % (np) ? (p) : (n) % (np)))

static double dot(int64_t n, const double* a, const double* b)
{
    const int np = nthreads();
    double part[256];
    const int npp = np > 256 ? 256 : np;
#pragma omp parallel for schedule(static) num_threads(npp)
    for (int p = 0; p < npp; ++p) {
        double s = 0.0;
        for (int64_t i = STRIPE_BEGIN(n, npp, p); i < STRIPE_BEGIN(n, npp, p + 1); ++i)
            s += a[i] * b[i];
        part[p] = s;
    }
    double s = 0.0;
    for (int p = 0; p < npp; ++p) s += part[p];
    return s;
}

static void norms(int64_t n, const double* r, double* l2sq, double* linf)
{
    double s = 0.0, m = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) reduction(max : m)
    for (int64_t i = 0; i < n; ++i) {
        s += r[i] * r[i];
        const double a = fabs(r[i]);
        if (a > m) m = a;
    }
    *l2sq = s;
    *linf = m;
}

/* Jacobi smoother, sweeps >= 1 (Smoother.cpp:100-128, BlockOps.h:219-225) */
static void jacobi(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
                   const double* dinv, int sweeps, const double* b, double* x, double* tmp)
{
    for (int64_t i = 0; i < n; ++i) x[i] = b[i] * dinv[i];
    for (int s = 1; s < sweeps; ++s) {
        memcpy(tmp, b, sizeof(double) * (size_t)n);
        ro_spmv(n, ptr, idx, val, -1.0, x, 1.0, tmp);
        for (int64_t i = 0; i < n; ++i) x[i] += tmp[i] * dinv[i];
    }
}

/* Solver_PCG (PCG.cpp:62-367): PCG with minimal-residual smoothing.  r and x are
   updated in place; *iter in: max iterations, out: iterations done; *tol in:
   tolerance on the smoothed residual, out: its final norm. */
static int pcg(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
               const double* dinv, int sweeps, double* r, double* x, int64_t* iter,
               double* tol)
{
    double* rs = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* v = (double*)malloc(sizeof(double) * (size_t)n);
    double* x2 = (double*)malloc(sizeof(double) * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    const int64_t maxit = *iter;
    const double tolv = *tol;
    for (int64_t i = 0; i < n; ++i) { rs[i] = r[i]; x2[i] = x[i]; p[i] = 0; v[i] = 0; }
    int64_t num_iter = 0;
    double tau = 0.0, tau_old, norm_of_residual = 0.0;
    int converge = 0, maxflag = 0, brk = 0;
    while (!(converge || maxflag || brk)) {
        ++num_iter;
        jacobi(n, ptr, idx, val, dinv, sweeps, r, v, tmp);
        const double sum1 = dot(n, v, r);
        tau_old = tau;
        tau = sum1;
        if (num_iter == 1) {
            for (int64_t i = 0; i < n; ++i) p[i] = v[i];
        } else {
            const double beta = tau / tau_old;
            for (int64_t i = 0; i < n; ++i) p[i] = v[i] + beta * p[i];
        }
        ro_spmv(n, ptr, idx, val, 1.0, p, 0.0, v);
        const double delta = dot(n, v, p);
        const double alpha = tau / delta;
        brk = fabs(delta) <= 0.0;
        if (!brk) {
            double s3 = 0.0, s4 = 0.0;
            {
                const int np = nthreads() > 256 ? 256 : nthreads();
                double p3[256], p4[256];
#pragma omp parallel for schedule(static) num_threads(np)
                for (int t = 0; t < np; ++t) {
                    double a3 = 0.0, a4 = 0.0;
                    for (int64_t i = STRIPE_BEGIN(n, np, t); i < STRIPE_BEGIN(n, np, t + 1); ++i) {
                        r[i] -= alpha * v[i];
                        const double d = r[i] - rs[i];
                        a3 += d * d;
                        a4 += d * rs[i];
                    }
                    p3[t] = a3;
                    p4[t] = a4;
                }
                for (int t = 0; t < np; ++t) { s3 += p3[t]; s4 += p4[t]; }
            }
            const double gamma_1 = (fabs(s3) <= 0.0) ? 0.0 : -s4 / s3;
            const double gamma_2 = 1.0 - gamma_1;
            double s5 = 0.0;
            {
                const int np = nthreads() > 256 ? 256 : nthreads();
                double p5[256];
#pragma omp parallel for schedule(static) num_threads(np)
                for (int t = 0; t < np; ++t) {
                    double a5 = 0.0;
                    for (int64_t i = STRIPE_BEGIN(n, np, t); i < STRIPE_BEGIN(n, np, t + 1); ++i) {
                        rs[i] = gamma_2 * rs[i] + gamma_1 * r[i];
                        x2[i] += alpha * p[i];
                        x[i] = gamma_2 * x[i] + gamma_1 * x2[i];
                        a5 += rs[i] * rs[i];
                    }
                    p5[t] = a5;
                }
                for (int t = 0; t < np; ++t) s5 += p5[t];
            }
            norm_of_residual = sqrt(s5);
            converge = norm_of_residual <= tolv;
            maxflag = num_iter > maxit;
            brk = fabs(tau) <= 0.0;
        }
    }
    free(rs); free(p); free(v); free(x2); free(tmp);
    *iter = num_iter;
    *tol = norm_of_residual;
    if (maxflag) return RO_MAXITER;
    if (brk) return RO_BREAKDOWN;
    return RO_OK;
}

/* paso::Solver (Solver.cpp:46-330) for PCG + Jacobi */
int ro_solve_paso(int64_t n, const int32_t* ptr, const int32_t* idx, double* val,
                  const double* b, double* x, double* bv, const ro_opts* opts, ro_diag* diag)
{
    const double EPS = 2.220446049250313e-16;
    const double tolerance = opts->tolerance;
    memset(diag, 0, sizeof(*diag));
    if (tolerance < 100. * EPS || tolerance > 1.) return RO_INPUT_ERROR;
    /* balance (SystemMatrix.cpp:263-312): bv_i = 1/sqrt(max_j |a_ij|) or 1 */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double fac = 0.0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) fac = fmax(fac, fabs(val[k]));
        bv[i] = fac > 0 ? sqrt(1. / fac) : 1.0;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k) val[k] *= bv[i] * bv[idx[k]];
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* dinv = (double*)malloc(sizeof(double) * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] * bv[i];
    double n2b, nmb;
    norms(n, r, &n2b, &nmb);
    n2b = sqrt(n2b);
    int err = RO_OK;
    if (isnan(n2b) || isnan(nmb)) {
        err = RO_NAN;
    } else if (n2b <= 0.) {
        for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
    } else {
        /* Jacobi on the balanced main diagonal (SparseMatrix.cpp:387-435) */
        for (int64_t i = 0; i < n; ++i) {
            double a = 0.0;
            int found = 0;
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (idx[k] == i) { a = val[k]; found = 1; break; }
            if (!found || !(fabs(a) > 0.)) { err = RO_INPUT_ERROR; break; }
            dinv[i] = 1. / a;
        }
        if (err == RO_OK) {
            jacobi(n, ptr, idx, val, dinv, opts->sweeps, r, x, tmp);
            int64_t totIter = 1;
            int fin = 0;
            double last2 = n2b, lastm = nmb;
            while (!fin) {
                int64_t cnt = opts->iter_max - totIter;
                fin = 1;
                if (totIter > 1)
                    for (int64_t i = 0; i < n; ++i) r[i] = b[i] * bv[i];
                ro_spmv(n, ptr, idx, val, -1., x, 1., r);
                double n2r, nmr;
                norms(n, r, &n2r, &nmr);
                n2r = sqrt(n2r);
                diag->residual_norm = n2r;
                diag->num_outer++;
                if (opts->verbose)
                    printf("Solver: Step %lld: l2/lmax-norm of residual is %g/%g\n",
                           (long long)totIter, n2r, nmr);
                if (totIter > 1 && n2r >= last2 && nmr >= lastm) {
                    err = RO_DIVERGENCE;
                    break;
                }
                if (n2r > tolerance * n2b || nmr > tolerance * nmb) {
                    double tol = tolerance * fmin(n2b, 0.1 * n2r / nmr * nmb);
                    last2 = n2r;
                    lastm = nmr;
                    int st = pcg(n, ptr, idx, val, dinv, opts->sweeps, r, x, &cnt, &tol);
                    totIter += cnt;
                    if (st == RO_OK) {
                        fin = 0;
                    } else if (st == RO_BREAKDOWN && cnt > 1) {
                        fin = 0;
                    } else {
                        err = st;
                        break;
                    }
                } else {
                    diag->converged = 1;
                }
            }
            diag->num_iter = totIter;
            for (int64_t i = 0; i < n; ++i) x[i] *= bv[i];
        }
    }
    free(r); free(dinv); free(tmp);
    return err;
}

/* textbook Jacobi-PCG, used by tests as an independent solution check */
int ro_solve_cg(int64_t n, const int32_t* ptr, const int32_t* idx, const double* val,
                const double* b, double* x, double rtol, int64_t iter_max, ro_diag* diag)
{
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    double* dinv = (double*)malloc(sizeof(double) * (size_t)n);
    memset(diag, 0, sizeof(*diag));
    for (int64_t i = 0; i < n; ++i) {
        double a = 1.0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            if (idx[k] == i) a = val[k];
        dinv[i] = 1.0 / a;
    }
    memcpy(r, b, sizeof(double) * (size_t)n);
    ro_spmv(n, ptr, idx, val, -1.0, x, 1.0, r);
    const double nb = sqrt(dot(n, b, b));
    for (int64_t i = 0; i < n; ++i) { z[i] = dinv[i] * r[i]; p[i] = z[i]; }
    double rho = dot(n, r, z);
    int64_t it = 0;
    double nr = sqrt(dot(n, r, r));
    int st = RO_OK;
    while (nr > rtol * nb) {
        if (it >= iter_max) { st = RO_MAXITER; break; }
        ro_spmv(n, ptr, idx, val, 1.0, p, 0.0, q);
        const double alpha = rho / dot(n, p, q);
        for (int64_t i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; z[i] = dinv[i] * r[i]; }
        const double rho_new = dot(n, r, z);
        const double beta = rho_new / rho;
        rho = rho_new;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        nr = sqrt(dot(n, r, r));
        ++it;
    }
    diag->num_iter = it;
    diag->residual_norm = nr;
    diag->converged = st == RO_OK;
    free(r); free(z); free(p); free(q); free(dinv);
    return st;
}

/* ------------------------------------------------------------------------- */
/* PDE systems: block size nb = numEq = numComp (paso block CSR, MATRIX_FORMAT  */
/* DEFAULT, blocks up to 3 without LAPACK: SystemMatrix.h:403-492).  A block   */
/* of pattern entry k is val[k nb^2 + ir + nb ic] (column-major, SparseMatrix  */
/* layout used by addToPasoMatrix, RipleyDomain.cpp:1508-1518); vectors hold   */
/* the nb components of a node together: u[node nb + comp].                   */
/* ------------------------------------------------------------------------- */

/* DefaultAssembler3D::assemblePDESystem (DefaultAssembler3D.cpp:3630-5751) and the 2D
   analogue: per equation k and component m
     EM_S[k + nb (m + nb (r + nk c))] = sum_q W (A_kimj G_ri G_cj + B_kim G_ri N_c
                                                 + C_kmj N_r G_cj + D_km N_r N_c)
     EM_F[k + nb r] = sum_q W (X_ki G_ri + Y_k N_r)
   with A[k + nb (i + dim (m + nb j))], B[k + nb (i + dim m)], C[k + nb (m + nb j)],
   D[k + nb m], X[k + nb i], Y[k] per data point (DefaultAssembler3D.cpp:3748-3777, ...). */
static void element_system(const q1_tab* t, int nb, int64_t e, ro_coef A, ro_coef B, ro_coef C,
                           ro_coef D, ro_coef X, ro_coef Y, double* EM_S, double* EM_F)
{
    const int dim = t->dim, nk = t->nk, nq = t->nq;
    const int sA = nb * dim * nb * dim, sB = nb * dim * nb, sC = nb * nb * dim, sD = nb * nb;
    const int sX = nb * dim, sY = nb;
    memset(EM_S, 0, sizeof(double) * (size_t)(nb * nb * nk * nk));
    memset(EM_F, 0, sizeof(double) * (size_t)(nb * nk));
    for (int q = 0; q < nq; ++q)
        for (int k = 0; k < nb; ++k) {
            for (int m = 0; m < nb; ++m) {
                double a[9] = {0}, b[3] = {0}, c[3] = {0}, dq = 0.0;
                for (int i = 0; i < dim; ++i)
                    for (int j = 0; j < dim; ++j)
                        if (A.kind) a[i + dim * j] = coef_at(A, sA, nq, e, k + nb * (i + dim * (m + nb * j)), q);
                for (int i = 0; i < dim; ++i) {
                    if (B.kind) b[i] = coef_at(B, sB, nq, e, k + nb * (i + dim * m), q);
                    if (C.kind) c[i] = coef_at(C, sC, nq, e, k + nb * (m + nb * i), q);
                }
                if (D.kind) dq = coef_at(D, sD, nq, e, k + nb * m, q);
                for (int r = 0; r < nk; ++r) {
                    const double* Gr = t->G[q][r];
                    const double Nr = t->N[q][r];
                    double s[3] = {0, 0, 0};
                    double bg = 0.0;
                    for (int j = 0; j < dim; ++j)
                        for (int i = 0; i < dim; ++i) s[j] += a[i + dim * j] * Gr[i];
                    for (int i = 0; i < dim; ++i) bg += b[i] * Gr[i];
                    for (int cc = 0; cc < nk; ++cc) {
                        const double* Gc = t->G[q][cc];
                        const double Nc = t->N[q][cc];
                        double v = 0.0;
                        for (int j = 0; j < dim; ++j) v += (s[j] + Nr * c[j]) * Gc[j];
                        v += bg * Nc + dq * Nr * Nc;
                        EM_S[k + nb * (m + nb * (r + nk * cc))] += t->W * v;
                    }
                }
            }
            double xq[3] = {0}, yq = 0.0;
            for (int i = 0; i < dim; ++i)
                if (X.kind) xq[i] = coef_at(X, sX, nq, e, k + nb * i, q);
            if (Y.kind) yq = coef_at(Y, sY, nq, e, k, q);
            for (int r = 0; r < nk; ++r) {
                double f = yq * t->N[q][r];
                for (int i = 0; i < dim; ++i) f += xq[i] * t->G[q][r][i];
                EM_F[k + nb * r] += t->W * f;
            }
        }
}

static void system_with(const q1_tab* tp, int dim, const int64_t ne[3], int nb, const int32_t* ptr,
                        const int32_t* idx, double* val, double* rhs, ro_coef A, ro_coef B, ro_coef C,
                        ro_coef D, ro_coef X, ro_coef Y);

void ro_assemble_system(int dim, const int64_t ne[3], const double dx[3], int nb,
                        const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                        ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y)
{
    q1_tab t;
    q1_build(dim, dx, &t);
    system_with(&t, dim, ne, nb, ptr, idx, val, rhs, A, B, C, D, X, Y);
}

/* DefaultAssembler3D::assemblePDESystemReduced (DefaultAssembler3D.cpp:6466-6876) and
   DefaultAssembler2D::assemblePDESystemReduced: the system terms with the 1-point rule */
void ro_assemble_system_reduced(int dim, const int64_t ne[3], const double dx[3], int nb,
                                const int32_t* ptr, const int32_t* idx, double* val, double* rhs,
                                ro_coef A, ro_coef B, ro_coef C, ro_coef D, ro_coef X, ro_coef Y)
{
    q1_tab t;
    q1_build_reduced(dim, dx, &t);
    system_with(&t, dim, ne, nb, ptr, idx, val, rhs, A, B, C, D, X, Y);
}

static void system_with(const q1_tab* tp, int dim, const int64_t ne[3], int nb, const int32_t* ptr,
                        const int32_t* idx, double* val, double* rhs, ro_coef A, ro_coef B, ro_coef C,
                        ro_coef D, ro_coef X, ro_coef Y)
{
    const q1_tab t = *tp;
    const int addS = A.kind || B.kind || C.kind || D.kind;
    const int addF = X.kind || Y.kind;
    if (!addS && !addF) return;
    const int64_t NE0 = ne[0], NE1 = ne[1], NE2 = dim == 3 ? ne[2] : 1;
    const int64_t NN0 = NE0 + 1, NN1 = NE1 + 1;
    const int nk = t.nk, bs = nb * nb;
    const int64_t outer = dim == 3 ? NE2 : NE1;
    for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
        for (int64_t ko = colour; ko < outer; ko += 2) {
            double EM_S[9 * 64], EM_F[3 * 8];
            int64_t nodes[8];
            const int64_t k1lo = dim == 3 ? 0 : ko, k1hi = dim == 3 ? NE1 : ko + 1;
            const int64_t k2 = dim == 3 ? ko : 0;
            for (int64_t k1 = k1lo; k1 < k1hi; ++k1)
                for (int64_t k0 = 0; k0 < NE0; ++k0) {
                    const int64_t e = k0 + NE0 * k1 + NE0 * NE1 * k2;
                    element_system(&t, nb, e, A, B, C, D, X, Y, EM_S, EM_F);
                    const int64_t first = k0 + NN0 * k1 + NN0 * NN1 * k2;
                    for (int k = 0; k < nk; ++k)
                        nodes[k] = first + (k & 1) + ((k >> 1) & 1) * NN0 + ((k >> 2) & 1) * NN0 * NN1;
                    if (addF && rhs)
                        for (int r = 0; r < nk; ++r)
                            for (int ir = 0; ir < nb; ++ir) rhs[nodes[r] * nb + ir] += EM_F[ir + nb * r];
                    if (addS && val)
                        for (int r = 0; r < nk; ++r)
                            for (int c = 0; c < nk; ++c)
                                for (int64_t kk = ptr[nodes[r]]; kk < ptr[nodes[r] + 1]; ++kk)
                                    if (idx[kk] == nodes[c]) {
                                        for (int ic = 0; ic < nb; ++ic)
                                            for (int ir = 0; ir < nb; ++ir)
                                                val[kk * bs + ir + nb * ic] +=
                                                    EM_S[ir + nb * (ic + nb * (r + nk * c))];
                                        break;
                                    }
                }
        }
    }
}

/* y = alpha A x + beta y for a block CSR matrix (SparseMatrix_MatrixVector.cpp, blocked
   branches) */
void ro_spmv_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, const double* val,
                   double alpha, const double* x, double beta, double* y)
{
    const int bs = nb * nb;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nodes; ++i)
        for (int ir = 0; ir < nb; ++ir) {
            double s = 0.0;
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                for (int ic = 0; ic < nb; ++ic) s += val[k * bs + ir + nb * ic] * x[(int64_t)idx[k] * nb + ic];
            y[i * nb + ir] = (beta == 0.0 ? 0.0 : beta * y[i * nb + ir]) + alpha * s;
        }
}

/* insertConstraint for systems (linearPDEs.py:2084-2112 with
   SparseMatrix::nullifyRowsAndCols_CSR, SparseMatrix.h:513-535): q, r per component */
void ro_insert_constraint_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx,
                                double* val, double* rhs, const double* q, const double* r)
{
    const int64_t n = nodes * nb;
    const int bs = nb * nb;
    double* u = (double*)calloc((size_t)n, sizeof(double));
    if (r)
        for (int64_t i = 0; i < n; ++i) u[i] = q[i] > 0 ? r[i] : 0.0;
    ro_spmv_block(nodes, nb, ptr, idx, val, -1.0, u, 1.0, rhs);
    for (int64_t i = 0; i < nodes; ++i)
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            for (int ir = 0; ir < nb; ++ir)
                for (int ic = 0; ic < nb; ++ic) {
                    const int64_t irow = i * nb + ir, icol = (int64_t)idx[k] * nb + ic;
                    if (q[icol] > 0. || q[irow] > 0.) val[k * bs + ir + nb * ic] = irow == icol ? 1.0 : 0.0;
                }
    for (int64_t i = 0; i < n; ++i)
        if (q[i] > 0) rhs[i] = r ? r[i] : 0.0;
    free(u);
}

/* block Jacobi: x = D^-1 b with the inverses of the main diagonal blocks (SparseMatrix::
   invMain with BlockOps_invM_2/3, BlockOps_solveAll; Smoother.cpp:100-128) */
static void jacobi_block(int64_t nodes, int nb, const double* dinv, const double* b, double* x)
{
    const int bs = nb * nb;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nodes; ++i)
        for (int ir = 0; ir < nb; ++ir) {
            double s = 0.0;
            for (int ic = 0; ic < nb; ++ic) s += dinv[i * bs + ir + nb * ic] * b[i * nb + ic];
            x[i * nb + ir] = s;
        }
}

static int invert_block(int nb, const double* A, double* inv)
{
    if (nb == 1) {
        if (!(fabs(A[0]) > 0.)) return 1;
        inv[0] = 1. / A[0];
        return 0;
    }
    if (nb == 2) {
        const double A11 = A[0], A21 = A[1], A12 = A[2], A22 = A[3];
        double D = A11 * A22 - A12 * A21;
        if (!(fabs(D) > 0)) return 1;
        D = 1. / D;
        inv[0] = A22 * D;
        inv[1] = -A21 * D;
        inv[2] = -A12 * D;
        inv[3] = A11 * D;
        return 0;
    }
    const double A11 = A[0], A21 = A[1], A31 = A[2], A12 = A[3], A22 = A[4], A32 = A[5];
    const double A13 = A[6], A23 = A[7], A33 = A[8];
    double D = A11 * (A22 * A33 - A23 * A32) + A12 * (A31 * A23 - A21 * A33) + A13 * (A21 * A32 - A31 * A22);
    if (!(fabs(D) > 0)) return 1;
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
    return 0;
}

/* the block Jacobi smoother with `sweeps` sweeps (Smoother.cpp:161-184): x = D^-1 b, then
   sweeps-1 times x += D^-1 (b - A x) with D the main diagonal blocks */
static void prec_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, const double* val,
                       const double* dinv, int sweeps, const double* b, double* x)
{
    jacobi_block(nodes, nb, dinv, b, x);
    if (sweeps <= 1) return;
    const int64_t n = nodes * nb;
    double* t = (double*)malloc(sizeof(double) * (size_t)n);
    double* c = (double*)malloc(sizeof(double) * (size_t)n);
    for (int s = 1; s < sweeps; ++s) {
        memcpy(t, b, sizeof(double) * (size_t)n);
        ro_spmv_block(nodes, nb, ptr, idx, val, -1.0, x, 1.0, t);
        jacobi_block(nodes, nb, dinv, t, c);
        for (int64_t i = 0; i < n; ++i) x[i] += c[i];
    }
    free(t);
    free(c);
}

/* Solver_PCG (PCG.cpp:62-367) on a block matrix */
static int pcg_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, const double* val,
                     const double* dinv, int sweeps, double* r, double* x, int64_t* iter, double* tol)
{
    const int64_t n = nodes * nb;
    double* rs = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* v = (double*)malloc(sizeof(double) * (size_t)n);
    double* x2 = (double*)malloc(sizeof(double) * (size_t)n);
    const int64_t maxit = *iter;
    const double tolv = *tol;
    for (int64_t i = 0; i < n; ++i) { rs[i] = r[i]; x2[i] = x[i]; p[i] = 0; v[i] = 0; }
    int64_t num_iter = 0;
    double tau = 0.0, tau_old, norm_of_residual = 0.0;
    int converge = 0, maxflag = 0, brk = 0;
    while (!(converge || maxflag || brk)) {
        ++num_iter;
        prec_block(nodes, nb, ptr, idx, val, dinv, sweeps, r, v);
        const double sum1 = dot(n, v, r);
        tau_old = tau;
        tau = sum1;
        if (num_iter == 1) {
            for (int64_t i = 0; i < n; ++i) p[i] = v[i];
        } else {
            const double beta = tau / tau_old;
            for (int64_t i = 0; i < n; ++i) p[i] = v[i] + beta * p[i];
        }
        ro_spmv_block(nodes, nb, ptr, idx, val, 1.0, p, 0.0, v);
        const double delta = dot(n, v, p);
        const double alpha = tau / delta;
        brk = fabs(delta) <= 0.0;
        if (!brk) {
            double s3 = 0.0, s4 = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                r[i] -= alpha * v[i];
                const double d = r[i] - rs[i];
                s3 += d * d;
                s4 += d * rs[i];
            }
            const double gamma_1 = (fabs(s3) <= 0.0) ? 0.0 : -s4 / s3;
            const double gamma_2 = 1.0 - gamma_1;
            double s5 = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                rs[i] = gamma_2 * rs[i] + gamma_1 * r[i];
                x2[i] += alpha * p[i];
                x[i] = gamma_2 * x[i] + gamma_1 * x2[i];
                s5 += rs[i] * rs[i];
            }
            norm_of_residual = sqrt(s5);
            converge = norm_of_residual <= tolv;
            maxflag = num_iter > maxit;
            brk = fabs(tau) <= 0.0;
        }
    }
    free(rs); free(p); free(v); free(x2);
    *iter = num_iter;
    *tol = norm_of_residual;
    if (maxflag) return RO_MAXITER;
    if (brk) return RO_BREAKDOWN;
    return RO_OK;
}

/* paso::Solver (Solver.cpp:46-330), PCG + block Jacobi (opts->sweeps), block matrix balanced
   in place per scalar row (SparseMatrix::maxAbsRow_CSR_OFFSET0 and applyDiagonal). */
int ro_solve_paso_block(int64_t nodes, int nb, const int32_t* ptr, const int32_t* idx, double* val,
                        const double* b, double* x, double* bv, const ro_opts* opts, ro_diag* diag)
{
    const double EPS = 2.220446049250313e-16;
    const double tolerance = opts->tolerance;
    const int64_t n = nodes * nb;
    const int bs = nb * nb;
    memset(diag, 0, sizeof(*diag));
    if (tolerance < 100. * EPS || tolerance > 1.) return RO_INPUT_ERROR;
    if (nb < 1 || nb > 3) return RO_INPUT_ERROR;
    for (int64_t i = 0; i < nodes; ++i)
        for (int ir = 0; ir < nb; ++ir) {
            double fac = 0.0;
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                for (int ic = 0; ic < nb; ++ic) fac = fmax(fac, fabs(val[k * bs + ir + nb * ic]));
            bv[i * nb + ir] = fac > 0 ? sqrt(1. / fac) : 1.0;
        }
    for (int64_t i = 0; i < nodes; ++i)
        for (int ir = 0; ir < nb; ++ir)
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                for (int ic = 0; ic < nb; ++ic)
                    val[k * bs + ir + nb * ic] *= bv[i * nb + ir] * bv[(int64_t)idx[k] * nb + ic];
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* dinv = (double*)malloc(sizeof(double) * (size_t)(nodes * bs));
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] * bv[i];
    double n2b, nmb;
    norms(n, r, &n2b, &nmb);
    n2b = sqrt(n2b);
    int err = RO_OK;
    if (isnan(n2b) || isnan(nmb)) {
        err = RO_NAN;
    } else if (n2b <= 0.) {
        for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
    } else {
        for (int64_t i = 0; i < nodes && err == RO_OK; ++i) {
            int64_t kd = -1;
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (idx[k] == i) { kd = k; break; }
            if (kd < 0 || invert_block(nb, val + kd * bs, dinv + i * bs)) err = RO_INPUT_ERROR;
        }
        if (err == RO_OK) {
            prec_block(nodes, nb, ptr, idx, val, dinv, opts->sweeps, r, x);
            int64_t totIter = 1;
            int fin = 0;
            double last2 = n2b, lastm = nmb;
            while (!fin) {
                int64_t cnt = opts->iter_max - totIter;
                fin = 1;
                if (totIter > 1)
                    for (int64_t i = 0; i < n; ++i) r[i] = b[i] * bv[i];
                ro_spmv_block(nodes, nb, ptr, idx, val, -1., x, 1., r);
                double n2r, nmr;
                norms(n, r, &n2r, &nmr);
                n2r = sqrt(n2r);
                diag->residual_norm = n2r;
                diag->num_outer++;
                if (totIter > 1 && n2r >= last2 && nmr >= lastm) {
                    err = RO_DIVERGENCE;
                    break;
                }
                if (n2r > tolerance * n2b || nmr > tolerance * nmb) {
                    double tol = tolerance * fmin(n2b, 0.1 * n2r / nmr * nmb);
                    last2 = n2r;
                    lastm = nmr;
                    int st = pcg_block(nodes, nb, ptr, idx, val, dinv, opts->sweeps, r, x, &cnt, &tol);
                    totIter += cnt;
                    if (st == RO_OK) {
                        fin = 0;
                    } else if (st == RO_BREAKDOWN && cnt > 1) {
                        fin = 0;
                    } else {
                        err = st;
                        break;
                    }
                } else {
                    diag->converged = 1;
                }
            }
            diag->num_iter = totIter;
            for (int64_t i = 0; i < n; ++i) x[i] *= bv[i];
        }
    }
    free(r); free(dinv);
    return err;
}
