// CSR pattern, Q1 element assembly (interior and boundary) and node -> Gauss point
// interpolation for ripley Rectangle/Brick domains on one B200.
//
// Design: assembly is node-centric.  One thread owns one matrix row (node) and
// sums the rows of its <= 2^dim adjacent element matrices in registers, so the
// scatter needs no atomics and the FP64 result is deterministic.  The element-matrix
// rows are computed from the Q1 shape-function gradients at the Gauss points (the
// same quantities DefaultAssembler{2,3}D.cpp expands in closed form,
// ripley/src/DefaultAssembler3D.cpp:152-2226).  Rows of a CTA are contiguous in the
// CSR arrays, so each CTA stages its rows in shared memory and writes them back with
// coalesced stores.
#include <cmath>
#include <cstring>

#include "rg_internal.cuh"

namespace rg {

// the 1-point rule of assemblePDESingleReduced (DefaultAssembler3D.cpp:2891-3271,
// DefaultAssembler2D.cpp:842-1010): element centre, weight = element volume; N = 2^-dim,
// dN_k/dx_d = +-(1/dx_d) 2^-(dim-1)
void build_q1_reduced_tables(int dim, const double dx[3], Q1Tables* t)
{
    build_q1_tables(dim, dx, t);  // face weights and zeroed tables
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= dx[d];
    t->W = vol;
    const int nk = 1 << dim;
    for (int k = 0; k < nk; ++k) {
        t->N[0][k] = 1.0 / nk;
        for (int d = 0; d < dim; ++d) {
            double g = (((k >> d) & 1) ? 1.0 : -1.0) / dx[d];
            for (int e = 0; e < dim; ++e)
                if (e != d) g *= 0.5;
            t->G[0][k][d] = g;
        }
    }
}

void build_q1_tables(int dim, const double dx[3], Q1Tables* t)
{
    const double g[2] = {0.5 - std::sqrt(3.0) / 6.0, 0.5 + std::sqrt(3.0) / 6.0};
    const int nk = 1 << dim, nq = 1 << dim;
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= dx[d];
    t->W = vol / nq;
    for (int d = 0; d < 3; ++d) {
        double a = 1.0;
        for (int e = 0; e < dim; ++e)
            if (e != d) a *= dx[e];
        t->Wf[d] = a / (1 << (dim - 1));
    }
    for (int q = 0; q < 8; ++q)
        for (int k = 0; k < 8; ++k) {
            t->N[q][k] = 0.0;
            for (int d = 0; d < 3; ++d) t->G[q][k][d] = 0.0;
        }
    for (int q = 0; q < nq; ++q) {
        double xi[3];
        for (int d = 0; d < dim; ++d) xi[d] = g[(q >> d) & 1];
        for (int k = 0; k < nk; ++k) {
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

namespace {

constexpr int kRowsPerCta = 128;

// ------------------------------------------------------------------ pattern
// Row i of Brick::getConnections(false) (ripley/src/Brick.cpp:3000-3061): the <=27
// in-range neighbours in ascending id order.  Row starts follow in closed form:
// along an axis with N nodes, node k has c(k) = 3 - [k==0] - [k==N-1] neighbours and
// sum_{k'<k} c(k') = 3k - [k>0].
struct PatternArgs {
    int dim;
    int64_t N0, N1, N2, n, nnz;
    int32_t* ptr;
    int32_t* idx;
};

__device__ __forceinline__ int64_t axis_count(int64_t k, int64_t N) { return 3 - (k == 0) - (k == N - 1); }
__device__ __forceinline__ int64_t axis_prefix(int64_t k) { return 3 * k - (k > 0); }

__device__ __forceinline__ int64_t row_start(const PatternArgs& a, int64_t x, int64_t y, int64_t z)
{
    const int64_t Cx = 3 * a.N0 - 2, Cy = 3 * a.N1 - 2;
    const int64_t cx = axis_count(x, a.N0), cy = axis_count(y, a.N1);
    if (a.dim == 2) return Cx * axis_prefix(y) + cy * axis_prefix(x);
    const int64_t cz = axis_count(z, a.N2);
    return Cx * Cy * axis_prefix(z) + cz * Cx * axis_prefix(y) + cz * cy * axis_prefix(x);
}

__global__ void __launch_bounds__(kRowsPerCta) k_pattern(const __grid_constant__ PatternArgs a)
{
    __shared__ int32_t stage[kRowsPerCta * 27];
    const int64_t row0 = (int64_t)blockIdx.x * kRowsPerCta;
    const int64_t row1 = min(row0 + kRowsPerCta, a.n);
    const int64_t i = row0 + threadIdx.x;
    const int64_t plane = a.N0 * a.N1;
    const int64_t z0 = row0 / plane, y0 = (row0 % plane) / a.N0, x0 = row0 % a.N0;
    const int64_t base = row_start(a, x0, y0, z0);
    if (i < a.n) {
        const int64_t z = i / plane, y = (i % plane) / a.N0, x = i % a.N0;
        const int64_t s = row_start(a, x, y, z);
        a.ptr[i] = (int32_t)s;
        if (i == a.n - 1) a.ptr[a.n] = (int32_t)a.nnz;
        int64_t k = s - base;
        const int zl = a.dim == 3 ? -1 : 0, zh = a.dim == 3 ? 1 : 0;
        for (int dz = zl; dz <= zh; ++dz) {
            if (z + dz < 0 || z + dz >= a.N2) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                if (y + dy < 0 || y + dy >= a.N1) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    if (x + dx < 0 || x + dx >= a.N0) continue;
                    stage[k++] = (int32_t)(i + dx + a.N0 * dy + plane * dz);
                }
            }
        }
    }
    __syncthreads();
    // rows [row0, row1) occupy idx[base, end) contiguously
    const int64_t zl = (row1 - 1) / plane, yl = ((row1 - 1) % plane) / a.N0, xl = (row1 - 1) % a.N0;
    const int64_t end = row_start(a, xl, yl, zl) + (a.dim == 3 ? axis_count(zl, a.N2) : 1) *
                                                      axis_count(yl, a.N1) * axis_count(xl, a.N0);
    for (int64_t t = threadIdx.x; t < end - base; t += kRowsPerCta) a.idx[base + t] = stage[t];
}

// ------------------------------------------------------------------ interior assembly
struct CoefArg {
    const double* p;
    int kind;
};

// Element-matrix tables integrated over the Gauss points, for operator coefficients that
// are constant over an element (CONSTANT or PER_ELEMENT):
//   SA[i][j][R][c] = sum_q W G_qRi G_qcj,  SB[i][R][c] = sum_q W G_qRi N_qc,
//   SC[j][R][c] = sum_q W N_qR G_qcj,      M[R][c] = sum_q W N_qR N_qc,
// so a row of the element matrix costs one multiply-add per table entry instead of a sum
// over the Gauss points.
struct UniTables {
    double SA[3][3][8][8];
    double SB[3][8][8];
    double SC[3][8][8];
    double M[8][8];
};

struct AsmArgs {
    CoefArg c[6];  // A B C D X Y
    Q1Tables t;
    UniTables u;
    int64_t NE0, NE1, NE2, NN0, NN1, NN2, n;
    const int32_t* ptr;
    double* val;
    double* rhs;
};

// coefficient data point of element e at Gauss point q (SIZE values)
template <int SIZE, int NQ>
__device__ __forceinline__ const double* coef_ptr(const CoefArg& c, int64_t e, int q)
{
    if (c.kind == RG_COEF_EXPANDED) return c.p + ((size_t)e * NQ + q) * SIZE;
    if (c.kind == RG_COEF_PER_ELEMENT) return c.p + (size_t)e * SIZE;
    return c.p;
}

// Row R of the element matrix and vector of element e:
//   em[c] = sum_q W (A_ij G_Ri G_cj + B_i G_Ri N_c + C_j N_R G_cj + D N_R N_c)
//   f     = sum_q W (X_i G_Ri + Y N_R)
// UNI: A, B, C, D are constant over the element, em comes from the integrated tables.
template <int DIM, int NQ, int R, bool UNI>
__device__ __forceinline__ void element_row(const AsmArgs& a, int64_t e, double (&em)[1 << DIM],
                                            double& f)
{
    if constexpr (UNI) {
        constexpr int NK = 1 << DIM;
        const CoefArg& A = a.c[0];
        const CoefArg& B = a.c[1];
        const CoefArg& C = a.c[2];
        const CoefArg& D = a.c[3];
        const CoefArg& X = a.c[4];
        const CoefArg& Y = a.c[5];
#pragma unroll
        for (int c = 0; c < NK; ++c) em[c] = 0.0;
        if (A.kind) {
            const double* ap = coef_ptr<DIM * DIM, 1>(A, e, 0);
#pragma unroll
            for (int j = 0; j < DIM; ++j)
#pragma unroll
                for (int i = 0; i < DIM; ++i) {
                    const double aij = __ldg(ap + i + DIM * j);
#pragma unroll
                    for (int c = 0; c < NK; ++c) em[c] = fma(aij, a.u.SA[i][j][R][c], em[c]);
                }
        }
        if (B.kind) {
            const double* bp = coef_ptr<DIM, 1>(B, e, 0);
#pragma unroll
            for (int i = 0; i < DIM; ++i) {
                const double bi = __ldg(bp + i);
#pragma unroll
                for (int c = 0; c < NK; ++c) em[c] = fma(bi, a.u.SB[i][R][c], em[c]);
            }
        }
        if (C.kind) {
            const double* cp = coef_ptr<DIM, 1>(C, e, 0);
#pragma unroll
            for (int j = 0; j < DIM; ++j) {
                const double cj = __ldg(cp + j);
#pragma unroll
                for (int c = 0; c < NK; ++c) em[c] = fma(cj, a.u.SC[j][R][c], em[c]);
            }
        }
        if (D.kind) {
            const double dd = __ldg(coef_ptr<1, 1>(D, e, 0));
#pragma unroll
            for (int c = 0; c < NK; ++c) em[c] = fma(dd, a.u.M[R][c], em[c]);
        }
        f = 0.0;
        if (X.kind || Y.kind) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                double fq = 0.0;
                if (Y.kind) fq = __ldg(coef_ptr<1, NQ>(Y, e, q)) * a.t.N[q][R];
                if (X.kind) {
                    const double* xp = coef_ptr<DIM, NQ>(X, e, q);
#pragma unroll
                    for (int i = 0; i < DIM; ++i) fq = fma(__ldg(xp + i), a.t.G[q][R][i], fq);
                }
                f = fma(a.t.W, fq, f);
            }
        }
        return;
    }
    constexpr int NK = 1 << DIM, D2 = DIM * DIM;
    const CoefArg& A = a.c[0];
    const CoefArg& B = a.c[1];
    const CoefArg& C = a.c[2];
    const CoefArg& D = a.c[3];
    const CoefArg& X = a.c[4];
    const CoefArg& Y = a.c[5];
#pragma unroll
    for (int c = 0; c < NK; ++c) em[c] = 0.0;
    f = 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const double NR = a.t.N[q][R];
        double s[DIM];
#pragma unroll
        for (int j = 0; j < DIM; ++j) s[j] = 0.0;
        double t0 = 0.0;
        if (A.kind) {
            const double* ap = coef_ptr<D2, NQ>(A, e, q);
#pragma unroll
            for (int j = 0; j < DIM; ++j)
#pragma unroll
                for (int i = 0; i < DIM; ++i) s[j] = fma(__ldg(ap + i + DIM * j), a.t.G[q][R][i], s[j]);
        }
        if (C.kind) {
            const double* cp = coef_ptr<DIM, NQ>(C, e, q);
#pragma unroll
            for (int j = 0; j < DIM; ++j) s[j] = fma(__ldg(cp + j), NR, s[j]);
        }
        if (B.kind) {
            const double* bp = coef_ptr<DIM, NQ>(B, e, q);
#pragma unroll
            for (int i = 0; i < DIM; ++i) t0 = fma(__ldg(bp + i), a.t.G[q][R][i], t0);
        }
        if (D.kind) t0 = fma(__ldg(coef_ptr<1, NQ>(D, e, q)), NR, t0);
#pragma unroll
        for (int c = 0; c < NK; ++c) {
            double v = t0 * a.t.N[q][c];
#pragma unroll
            for (int j = 0; j < DIM; ++j) v = fma(s[j], a.t.G[q][c][j], v);
            em[c] = fma(a.t.W, v, em[c]);
        }
        double fq = 0.0;
        if (Y.kind) fq = __ldg(coef_ptr<1, NQ>(Y, e, q)) * NR;
        if (X.kind) {
            const double* xp = coef_ptr<DIM, NQ>(X, e, q);
#pragma unroll
            for (int i = 0; i < DIM; ++i) fq = fma(__ldg(xp + i), a.t.G[q][R][i], fq);
        }
        f = fma(a.t.W, fq, f);
    }
}

// band index of the neighbour reached from a node through element offset (sx,sy,sz)
// (element = node - 1 + s per axis) and the element's local node c
template <int DIM>
__host__ __device__ constexpr int band_of(int sx, int sy, int sz, int c)
{
    return DIM == 3 ? (sx + (c & 1)) + 3 * (sy + ((c >> 1) & 1)) + 9 * (sz + ((c >> 2) & 1))
                    : (sx + (c & 1)) + 3 * (sy + ((c >> 1) & 1));
}

template <int DIM, int NQ, bool UNI, int SX, int SY, int SZ>
__device__ __forceinline__ void add_element(const AsmArgs& a, int64_t x, int64_t y, int64_t z,
                                            double (&acc)[DIM == 3 ? 27 : 9], double& facc)
{
    constexpr int NK = 1 << DIM;
    const int64_t ex = x - 1 + SX, ey = y - 1 + SY, ez = z - 1 + SZ;
    if (ex < 0 || ex >= a.NE0 || ey < 0 || ey >= a.NE1) return;
    if (DIM == 3 && (ez < 0 || ez >= a.NE2)) return;
    const int64_t e = ex + a.NE0 * ey + (DIM == 3 ? a.NE0 * a.NE1 * ez : 0);
    constexpr int R = (1 - SX) + 2 * (1 - SY) + (DIM == 3 ? 4 * (1 - SZ) : 0);
    double em[NK], f;
    element_row<DIM, NQ, R, UNI>(a, e, em, f);
#pragma unroll
    for (int c = 0; c < NK; ++c) acc[band_of<DIM>(SX, SY, SZ, c)] += em[c];
    facc += f;
}

// NQ = 2^DIM Gauss points (assemblePDESingle) or 1, the element centre
// (assemblePDESingleReduced); the tables in `a.t` hold the matching rule
template <int DIM, int NQ, bool UNI>
__global__ void __launch_bounds__(kRowsPerCta) k_assemble(const __grid_constant__ AsmArgs a)
{
    constexpr int NB = DIM == 3 ? 27 : 9;
    __shared__ double stage[kRowsPerCta * NB];
    const int64_t row0 = (int64_t)blockIdx.x * kRowsPerCta;
    const int64_t row1 = min(row0 + kRowsPerCta, a.n);
    const int64_t i = row0 + threadIdx.x;
    double acc[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) acc[b] = 0.0;
    double facc = 0.0;
    int64_t x = 0, y = 0, z = 0;
    if (i < a.n) {
        x = i % a.NN0;
        y = (i / a.NN0) % a.NN1;
        z = DIM == 3 ? i / (a.NN0 * a.NN1) : 0;
        add_element<DIM, NQ, UNI, 0, 0, 0>(a, x, y, z, acc, facc);
        add_element<DIM, NQ, UNI, 1, 0, 0>(a, x, y, z, acc, facc);
        add_element<DIM, NQ, UNI, 0, 1, 0>(a, x, y, z, acc, facc);
        add_element<DIM, NQ, UNI, 1, 1, 0>(a, x, y, z, acc, facc);
        if (DIM == 3) {
            add_element<DIM, NQ, UNI, 0, 0, 1>(a, x, y, z, acc, facc);
            add_element<DIM, NQ, UNI, 1, 0, 1>(a, x, y, z, acc, facc);
            add_element<DIM, NQ, UNI, 0, 1, 1>(a, x, y, z, acc, facc);
            add_element<DIM, NQ, UNI, 1, 1, 1>(a, x, y, z, acc, facc);
        }
        if (a.rhs) a.rhs[i] += facc;
    }
    if (!a.val) return;  // uniform across the CTA
    const int64_t base = a.ptr[row0];
    if (i < a.n) {
        int64_t k = a.ptr[i] - base;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int bx = b % 3 - 1, by = (b / 3) % 3 - 1, bz = DIM == 3 ? b / 9 - 1 : 0;
            const bool in = x + bx >= 0 && x + bx < a.NN0 && y + by >= 0 && y + by < a.NN1 &&
                            (DIM == 2 || (z + bz >= 0 && z + bz < a.NN2));
            if (in) stage[k++] = acc[b];
        }
    }
    __syncthreads();
    const int64_t end = a.ptr[row1];
    for (int64_t t = threadIdx.x; t < end - base; t += kRowsPerCta) a.val[base + t] += stage[t];
}

// ------------------------------------------------------------------ boundary assembly
// DefaultAssembler3D::assemblePDEBoundarySingle (ripley/src/DefaultAssembler3D.cpp:2232-2888):
// face terms d (matrix) and y (rhs) on FunctionOnBoundary.  Face f of axis ax, side s:
// faces ordered left,right,bottom,top,front,back; face element (ka,kb) over the lower
// and upper in-face axes has index offset_f + ka + NEa*kb; its Gauss points are
// q = qa + 2*qb.  One thread per (node, equation k, component m); threads of nodes off the
// boundary exit at once.  The same kernel covers
//   * PDE systems, block size NBLK (assemblePDEBoundarySystem, DefaultAssembler3D.cpp:
//     5753-6464): d[k + NBLK m] and y[k] per data point, blocks val[e NBLK^2 + k + NBLK m];
//   * ReducedFunctionOnBoundary (assemblePDEBoundarySingleReduced, 3274-3628, and
//     ...SystemReduced, 6878-7255): one data point per face element, the 1-point rule at the
//     face centre with weight = face area.
struct BndArgs {
    CoefArg d, y;
    double g[2];  // 1D Gauss points
    double Wf[3];
    int64_t NE[3], NN[3], n;
    int64_t face_off[6];
    int dim;
    const int32_t* ptr;
    double* val;
    double* rhs;
};

template <int DIM, int NBLK, bool RED>
__global__ void __launch_bounds__(128) k_assemble_boundary(const __grid_constant__ BndArgs a)
{
    constexpr int NB = DIM == 3 ? 27 : 9;
    constexpr int NQF = RED ? 1 : 1 << (DIM - 1);
    constexpr int BS = NBLK * NBLK;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i = tid / BS;
    const int km = (int)(tid % BS);
    const int k = km % NBLK, m = km / NBLK;
    if (i >= a.n) return;
    int64_t c3[3];
    c3[0] = i % a.NN[0];
    c3[1] = (i / a.NN[0]) % a.NN[1];
    c3[2] = DIM == 3 ? i / (a.NN[0] * a.NN[1]) : 0;
    bool on = false;
#pragma unroll
    for (int ax = 0; ax < DIM; ++ax) on |= (c3[ax] == 0) || (c3[ax] == a.NN[ax] - 1);
    if (!on) return;
    const bool with_y = a.y.kind && m == 0;
    double acc[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) acc[b] = 0.0;
    double facc = 0.0;
#pragma unroll
    for (int face = 0; face < 2 * DIM; ++face) {
        const int ax = face / 2, side = face % 2;
        if (c3[ax] != (side ? a.NN[ax] - 1 : 0)) continue;
        const int fa0 = ax == 0 ? 1 : 0;
        const int fa1 = DIM == 3 ? (ax == 2 ? 1 : 2) : 0;
        const int64_t u = c3[fa0], v = DIM == 3 ? c3[fa1] : 0;
        const int64_t na = a.NE[fa0], nb = DIM == 3 ? a.NE[fa1] : 1;
        for (int sb = 0; sb < (DIM == 3 ? 2 : 1); ++sb)
            for (int sa = 0; sa < 2; ++sa) {
                const int64_t ka = u - 1 + sa, kb = DIM == 3 ? v - 1 + sb : 0;
                if (ka < 0 || ka >= na || kb < 0 || kb >= nb) continue;
                const int64_t fe = a.face_off[face] + ka + na * kb;
                const int r = (1 - sa) + (DIM == 3 ? 2 * (1 - sb) : 0);  // face-local node
                for (int q = 0; q < NQF; ++q) {
                    const double xa = RED ? 0.5 : a.g[q & 1], xb = RED ? 0.5 : a.g[(q >> 1) & 1];
                    double Nf[4];
                    for (int kk = 0; kk < (DIM == 3 ? 4 : 2); ++kk) {
                        double w = (kk & 1) ? xa : 1.0 - xa;
                        if (DIM == 3) w *= ((kk >> 1) & 1) ? xb : 1.0 - xb;
                        Nf[kk] = w;
                    }
                    const double Wf = RED ? a.Wf[ax] * (1 << (DIM - 1)) : a.Wf[ax];
                    if (with_y) {
                        const double* yp = a.y.kind == RG_COEF_EXPANDED ? a.y.p + (fe * NQF + q) * NBLK
                                         : a.y.kind == RG_COEF_PER_ELEMENT ? a.y.p + fe * NBLK : a.y.p;
                        facc = fma(Wf, __ldg(yp + k) * Nf[r], facc);
                    }
                    if (a.d.kind) {
                        const double* dp = a.d.kind == RG_COEF_EXPANDED ? a.d.p + (fe * NQF + q) * BS
                                         : a.d.kind == RG_COEF_PER_ELEMENT ? a.d.p + fe * BS : a.d.p;
                        const double dr = __ldg(dp + k + NBLK * m) * Nf[r];
                        for (int kk = 0; kk < (DIM == 3 ? 4 : 2); ++kk) {
                            int off[3] = {0, 0, 0};
                            off[fa0] = (int)(ka + (kk & 1) - u);
                            if (DIM == 3) off[fa1] = (int)(kb + ((kk >> 1) & 1) - v);
                            const int b = (off[0] + 1) + 3 * (off[1] + 1) + (DIM == 3 ? 9 * (off[2] + 1) : 0);
                            acc[b] = fma(Wf, dr * Nf[kk], acc[b]);
                        }
                    }
                }
            }
    }
    if (a.rhs && with_y) a.rhs[i * NBLK + k] += facc;
    if (a.val && a.d.kind) {
        int64_t e = a.ptr[i];
        for (int b = 0; b < NB; ++b) {
            const int bx = b % 3 - 1, by = (b / 3) % 3 - 1, bz = DIM == 3 ? b / 9 - 1 : 0;
            const bool in = c3[0] + bx >= 0 && c3[0] + bx < a.NN[0] && c3[1] + by >= 0 &&
                            c3[1] + by < a.NN[1] &&
                            (DIM == 2 || (c3[2] + bz >= 0 && c3[2] + bz < a.NN[2]));
            if (in) {
                a.val[e * BS + k + NBLK * m] += acc[b];
                ++e;
            }
        }
    }
}

// ------------------------------------------------------------------ interpolation
// Brick::interpolateNodesOnElementsWorker (ripley/src/Brick.cpp:3315-3398): Q1 values
// at the Gauss points, or the mean of the element's nodes for ReducedFunction.
struct InterpArgs {
    Q1Tables t;
    int dim, ncomp, reduced;
    int64_t NE0, NE1, NE2, NN0, NN1, nel;
    const double* nodal;
    double* out;
};

__global__ void k_interpolate(const __grid_constant__ InterpArgs a)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.nel) return;
    const int nk = 1 << a.dim;
    const int64_t k0 = e % a.NE0, k1 = (e / a.NE0) % a.NE1, k2 = a.dim == 3 ? e / (a.NE0 * a.NE1) : 0;
    const int64_t first = k0 + a.NN0 * k1 + a.NN0 * a.NN1 * k2;
    int64_t node[8];
    for (int k = 0; k < nk; ++k)
        node[k] = first + (k & 1) + ((k >> 1) & 1) * a.NN0 + ((k >> 2) & 1) * a.NN0 * a.NN1;
    for (int c = 0; c < a.ncomp; ++c) {
        if (a.reduced) {
            // summation order of the reference: z fastest, then y, then x
            double s = 0.0;
            for (int bx = 0; bx < 2; ++bx)
                for (int by = 0; by < 2; ++by)
                    for (int bz = 0; bz < (a.dim == 3 ? 2 : 1); ++bz)
                        s += a.nodal[node[bx + 2 * by + 4 * bz] * a.ncomp + c];
            a.out[e * a.ncomp + c] = s / nk;
        } else {
            for (int q = 0; q < nk; ++q) {
                double v = 0.0;
                for (int k = 0; k < nk; ++k) v = fma(a.t.N[q][k], a.nodal[node[k] * a.ncomp + c], v);
                a.out[(e * nk + q) * a.ncomp + c] = v;
            }
        }
    }
}

}  // namespace

int launch_pattern(Domain* d)
{
    PatternArgs a;
    a.dim = d->dim;
    a.N0 = d->nn[0];
    a.N1 = d->nn[1];
    a.N2 = d->nn[2];
    a.n = d->n;
    a.nnz = d->nnz;
    a.ptr = d->ptr;
    a.idx = d->idx;
    const int grid = (int)((d->n + kRowsPerCta - 1) / kRowsPerCta);
    RG_TIMED(T_PATTERN, (k_pattern<<<grid, kRowsPerCta, 0, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int assemble_single_impl(const Domain* d, double* val, double* rhs, const rg_coef* c[6], bool reduced)
{
    AsmArgs a;
    bool addS = false, addF = false;
    for (int j = 0; j < 6; ++j) {
        a.c[j].p = (c[j] && c[j]->kind != RG_COEF_EMPTY) ? c[j]->ptr : nullptr;
        a.c[j].kind = (c[j] && c[j]->ptr) ? c[j]->kind : RG_COEF_EMPTY;
        if (a.c[j].kind) (j < 4 ? addS : addF) = true;
    }
    a.t = reduced ? d->q1r : d->q1;
    // operator coefficients constant over each element: integrated element tables
    bool uni = !reduced;
    for (int j = 0; j < 4; ++j) uni = uni && a.c[j].kind != RG_COEF_EXPANDED;
    if (uni) {
        const int nk = 1 << d->dim, nq = nk, dim = d->dim;
        const Q1Tables& t = a.t;
        std::memset(&a.u, 0, sizeof(a.u));
        for (int r = 0; r < nk; ++r)
            for (int c = 0; c < nk; ++c)
                for (int q = 0; q < nq; ++q) {
                    a.u.M[r][c] += t.W * t.N[q][r] * t.N[q][c];
                    for (int i = 0; i < dim; ++i) {
                        a.u.SB[i][r][c] += t.W * t.G[q][r][i] * t.N[q][c];
                        a.u.SC[i][r][c] += t.W * t.N[q][r] * t.G[q][c][i];
                        for (int j = 0; j < dim; ++j) a.u.SA[i][j][r][c] += t.W * t.G[q][r][i] * t.G[q][c][j];
                    }
                }
    }
    a.NE0 = d->ne[0];
    a.NE1 = d->ne[1];
    a.NE2 = d->ne[2];
    a.NN0 = d->nn[0];
    a.NN1 = d->nn[1];
    a.NN2 = d->nn[2];
    a.n = d->n;
    a.ptr = d->ptr;
    a.val = addS ? val : nullptr;
    a.rhs = addF ? rhs : nullptr;
    if (!a.val && !a.rhs) return RG_OK;
    const int grid = (int)((d->n + kRowsPerCta - 1) / kRowsPerCta);
    if (d->dim == 3 && !reduced && uni)
        RG_TIMED(T_ASSEMBLE, (k_assemble<3, 8, true><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    else if (d->dim == 3 && !reduced)
        RG_TIMED(T_ASSEMBLE, (k_assemble<3, 8, false><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    else if (d->dim == 3)
        RG_TIMED(T_ASSEMBLE, (k_assemble<3, 1, false><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    else if (!reduced && uni)
        RG_TIMED(T_ASSEMBLE, (k_assemble<2, 4, true><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    else if (!reduced)
        RG_TIMED(T_ASSEMBLE, (k_assemble<2, 4, false><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    else
        RG_TIMED(T_ASSEMBLE, (k_assemble<2, 1, false><<<grid, kRowsPerCta, 0, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

template <int DIM, bool RED>
void launch_boundary(const BndArgs& a, int nb, int grid)
{
    if (nb == 1)
        RG_TIMED(T_BOUNDARY, (k_assemble_boundary<DIM, 1, RED><<<grid, 128, 0, stream()>>>(a)));
    else if (nb == 2)
        RG_TIMED(T_BOUNDARY, (k_assemble_boundary<DIM, 2, RED><<<grid, 128, 0, stream()>>>(a)));
    else
        RG_TIMED(T_BOUNDARY, (k_assemble_boundary<DIM, 3, RED><<<grid, 128, 0, stream()>>>(a)));
}

int assemble_boundary_impl(const Domain* d, int nb, bool reduced, double* val, double* rhs, const rg_coef* dc,
                           const rg_coef* yc)
{
    BndArgs a;
    a.d.p = (dc && dc->kind) ? dc->ptr : nullptr;
    a.d.kind = (dc && dc->ptr) ? dc->kind : RG_COEF_EMPTY;
    a.y.p = (yc && yc->kind) ? yc->ptr : nullptr;
    a.y.kind = (yc && yc->ptr) ? yc->kind : RG_COEF_EMPTY;
    if (!a.d.kind) val = nullptr;
    if (!a.y.kind) rhs = nullptr;
    if (!val && !rhs) return RG_OK;
    a.g[0] = 0.5 - std::sqrt(3.0) / 6.0;
    a.g[1] = 0.5 + std::sqrt(3.0) / 6.0;
    for (int k = 0; k < 3; ++k) {
        a.Wf[k] = d->q1.Wf[k];
        a.NE[k] = d->ne[k];
        a.NN[k] = d->nn[k];
    }
    a.n = d->n;
    a.dim = d->dim;
    int64_t counts[6] = {0, 0, 0, 0, 0, 0};
    if (d->dim == 2) {
        counts[0] = counts[1] = d->ne[1];
        counts[2] = counts[3] = d->ne[0];
    } else {
        counts[0] = counts[1] = d->ne[1] * d->ne[2];
        counts[2] = counts[3] = d->ne[0] * d->ne[2];
        counts[4] = counts[5] = d->ne[0] * d->ne[1];
    }
    int64_t off = 0;
    for (int f = 0; f < 6; ++f) {
        a.face_off[f] = off;
        off += counts[f];
    }
    a.ptr = d->ptr;
    a.val = val;
    a.rhs = rhs;
    const int grid = (int)((d->n * nb * nb + 127) / 128);
    if (d->dim == 3 && !reduced)
        launch_boundary<3, false>(a, nb, grid);
    else if (d->dim == 3)
        launch_boundary<3, true>(a, nb, grid);
    else if (!reduced)
        launch_boundary<2, false>(a, nb, grid);
    else
        launch_boundary<2, true>(a, nb, grid);
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int launch_interpolate(const Domain* d, const double* nodal, int ncomp, double* out, int reduced)
{
    InterpArgs a;
    a.t = d->q1;
    a.dim = d->dim;
    a.ncomp = ncomp;
    a.reduced = reduced;
    a.NE0 = d->ne[0];
    a.NE1 = d->ne[1];
    a.NE2 = d->ne[2];
    a.NN0 = d->nn[0];
    a.NN1 = d->nn[1];
    a.nel = d->ne[0] * d->ne[1] * d->ne[2];
    a.nodal = nodal;
    a.out = out;
    const int grid = (int)((a.nel + 127) / 128);
    RG_TIMED(T_VECTOR, (k_interpolate<<<grid, 128, 0, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

}  // namespace rg
