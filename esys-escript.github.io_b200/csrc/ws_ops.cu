// Memory-bound operators of the warm-start network (everything but the 3x3x3 convolutions):
// 2x2x2 average pooling, nearest-neighbour upsampling fused with channel concatenation,
// their backward passes with the ReLU masks of the tensors they read, the 1x1x1 output
// head, bias gradients, the mean-squared-error loss, the Adam update with bf16 weight
// refresh (forward and flipped/transposed data-gradient layouts), and the packing of
// (log kappa, Y) into the network input.  Activations use the layout of rg_act.
#include <algorithm>
#include <cuda_bf16.h>

#include "rg_internal.cuh"

namespace rg {
namespace ws {
namespace {

struct Act {
    __nv_bfloat16* p;
    int n, d, h, w, c;
    __host__ __device__ size_t at(int nn, int dd, int hh, int ww) const
    {
        return ((((size_t)nn * (d + 2) + 1 + dd) * h + hh) * w + ww) * c;
    }
    __host__ __device__ size_t positions() const { return (size_t)n * d * h * w; }
    // position index -> (n, d, h, w)
    __host__ __device__ void coords(size_t pos, int& nn, int& dd, int& hh, int& ww) const
    {
        ww = (int)(pos % w);
        pos /= w;
        hh = (int)(pos % h);
        pos /= h;
        dd = (int)(pos % d);
        nn = (int)(pos / d);
    }
};

inline Act act(const rg_act* a) { return Act{static_cast<__nv_bfloat16*>(a->ptr), a->n, a->d, a->h, a->w, a->c}; }

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ __nv_bfloat16 tobf(float v) { return __float2bfloat16_rn(v); }

#define RG_GRID_LOOP(i, count) \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (count); i += (size_t)gridDim.x * blockDim.x)

// out(n, d, h, w, c) = mean of in(n, 2d+i, 2h+j, 2w+k, c)
__global__ void k_avgpool(Act in, Act out)
{
    RG_GRID_LOOP(i, out.positions() * out.c)
    {
        const int c = (int)(i % out.c);
        int n, d, h, w;
        out.coords(i / out.c, n, d, h, w);
        float s = 0.f;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int e = 0; e < 2; ++e) s += bf(in.p[in.at(n, 2 * d + a, 2 * h + b, 2 * w + e) + c]);
        out.p[out.at(n, d, h, w) + c] = tobf(0.125f * s);
    }
}

// din(child) = [dskip(child, skip_off + c)] + dout(parent)/8, times (in(child) > 0)
__global__ void k_avgpool_bwd(Act dout, Act in, Act dskip, int skip_off, Act din)
{
    RG_GRID_LOOP(i, din.positions() * din.c)
    {
        const int c = (int)(i % din.c);
        int n, d, h, w;
        din.coords(i / din.c, n, d, h, w);
        float g = 0.125f * bf(dout.p[dout.at(n, d >> 1, h >> 1, w >> 1) + c]);
        if (dskip.p) g += bf(dskip.p[dskip.at(n, d, h, w) + skip_off + c]);
        if (!(bf(in.p[in.at(n, d, h, w) + c]) > 0.f)) g = 0.f;
        din.p[din.at(n, d, h, w) + c] = tobf(g);
    }
}

// out = cat(up2(a), b) along channels: out(.., c) = a(parent, c) for c < a.c, b(.., c - a.c)
__global__ void k_upcat(Act a, Act b, Act out)
{
    RG_GRID_LOOP(i, out.positions() * out.c)
    {
        const int c = (int)(i % out.c);
        int n, d, h, w;
        out.coords(i / out.c, n, d, h, w);
        const float v = c < a.c ? bf(a.p[a.at(n, d >> 1, h >> 1, w >> 1) + c]) : bf(b.p[b.at(n, d, h, w) + c - a.c]);
        out.p[out.at(n, d, h, w) + c] = tobf(v);
    }
}

// da(parent, c) = sum over the 8 children of dcat(child, c), c < da.c, where a(parent, c) > 0
__global__ void k_upcat_bwd(Act dcat, Act a, Act da)
{
    RG_GRID_LOOP(i, da.positions() * da.c)
    {
        const int c = (int)(i % da.c);
        int n, d, h, w;
        da.coords(i / da.c, n, d, h, w);
        float s = 0.f;
        for (int x = 0; x < 2; ++x)
            for (int y = 0; y < 2; ++y)
                for (int z = 0; z < 2; ++z) s += bf(dcat.p[dcat.at(n, 2 * d + x, 2 * h + y, 2 * w + z) + c]);
        if (a.p && !(bf(a.p[a.at(n, d, h, w) + c]) > 0.f)) s = 0.f;
        da.p[da.at(n, d, h, w) + c] = tobf(s);
    }
}

// out(pos) = sum_c w[c] x(pos, c) + b   (fp32 output, dense [n][d][h][w])
__global__ void k_head(Act x, const float* __restrict__ w, const float* __restrict__ b, float* __restrict__ out)
{
    RG_GRID_LOOP(i, x.positions())
    {
        int n, d, h, ww;
        x.coords(i, n, d, h, ww);
        const __nv_bfloat16* xp = x.p + x.at(n, d, h, ww);
        float s = b[0];
        for (int c = 0; c < x.c; ++c) s = fmaf(w[c], bf(xp[c]), s);
        out[i] = s;
    }
}

// dx(pos, c) = w[c] dout(pos) where x(pos, c) > 0
__global__ void k_head_bwd_x(Act x, const float* __restrict__ w, const float* __restrict__ dout, Act dx)
{
    RG_GRID_LOOP(i, x.positions() * x.c)
    {
        const int c = (int)(i % x.c);
        const size_t pos = i / x.c;
        int n, d, h, ww;
        x.coords(pos, n, d, h, ww);
        const size_t o = x.at(n, d, h, ww) + c;
        dx.p[o] = tobf(bf(x.p[o]) > 0.f ? w[c] * dout[pos] : 0.f);
    }
}

// per-CTA partial sums over positions of v(pos, c) (optionally times dout(pos)); one
// partial row of `cols` floats per CTA, summed in a fixed order by k_colsum_finish
template <bool WITH_DOUT>
__global__ void k_colsum(Act v, const float* __restrict__ dout, float* __restrict__ part, int cols)
{
    extern __shared__ float acc[];  // blockDim.x * cols
    for (int c = 0; c < cols; ++c) acc[threadIdx.x * cols + c] = 0.f;
    for (size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x; pos < v.positions();
         pos += (size_t)gridDim.x * blockDim.x) {
        int n, d, h, w;
        v.coords(pos, n, d, h, w);
        const __nv_bfloat16* vp = v.p + v.at(n, d, h, w);
        const float s = WITH_DOUT ? dout[pos] : 1.f;
        for (int c = 0; c < cols; ++c) acc[threadIdx.x * cols + c] += s * bf(vp[c]);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < cols; c += blockDim.x) {
        float s = 0.f;
        for (int t = 0; t < (int)blockDim.x; ++t) s += acc[t * cols + c];
        part[(size_t)blockIdx.x * cols + c] = s;
    }
}

__global__ void k_colsum_finish(const float* __restrict__ part, int nblocks, int cols, float* __restrict__ out,
                                int accumulate)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * cols + c];
        out[c] = accumulate ? out[c] + s : s;
    }
}

// loss partials: sum (out - t)^2 and sum dout; dout = 2 (out - t) / count
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ t, size_t count, float* __restrict__ dout,
                      double* __restrict__ part)
{
    __shared__ double sh[2][256];
    double s = 0.0, g = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const float e = out[i] - t[i];
        const float de = 2.f * e / (float)count;
        dout[i] = de;
        s += (double)e * e;
        g += de;
    }
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = g;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sh[0][0];
        part[2 * blockIdx.x + 1] = sh[1][0];
    }
}

__global__ void k_mse_finish(const double* __restrict__ part, int nblocks, size_t count, double* __restrict__ loss,
                             float* __restrict__ dsum)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0, g = 0.0;
        for (int b = 0; b < nblocks; ++b) {
            s += part[2 * b];
            g += part[2 * b + 1];
        }
        *loss = s / (double)count;
        if (dsum) *dsum = (float)g;
    }
}

// loss = (sum_i e_i^2 + lambda sum over neighbouring cell pairs (e_i - e_j)^2) / count with
// e = out - t on a (n, d, h, w) grid: the squared error plus a discrete gradient (H1
// seminorm) term, which weighs the rough error that dominates a guess's residual.
// dout_i = (2 e_i + 2 lambda sum_{j adjacent to i} (e_i - e_j)) / count.
__global__ void k_h1_loss(const float* __restrict__ out, const float* __restrict__ t, int n, int d_, int h_, int w_,
                          float lambda, float* __restrict__ dout, double* __restrict__ part)
{
    __shared__ double sh[2][256];
    const size_t count = (size_t)n * d_ * h_ * w_;
    const float inv = 1.f / (float)count;
    double s = 0.0, g = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % w_), y = (int)((i / w_) % h_), z = (int)((i / ((size_t)w_ * h_)) % d_);
        const float e = out[i] - t[i];
        float lap = 0.f, pairs = 0.f;
        const size_t sy = (size_t)w_, sz = (size_t)w_ * h_;
        if (x > 0) lap += e - (out[i - 1] - t[i - 1]);
        if (x + 1 < w_) {
            const float f = e - (out[i + 1] - t[i + 1]);
            lap += f;
            pairs += f * f;
        }
        if (y > 0) lap += e - (out[i - sy] - t[i - sy]);
        if (y + 1 < h_) {
            const float f = e - (out[i + sy] - t[i + sy]);
            lap += f;
            pairs += f * f;
        }
        if (z > 0) lap += e - (out[i - sz] - t[i - sz]);
        if (z + 1 < d_) {
            const float f = e - (out[i + sz] - t[i + sz]);
            lap += f;
            pairs += f * f;
        }
        const float de = (2.f * e + 2.f * lambda * lap) * inv;
        dout[i] = de;
        s += (double)e * e + (double)lambda * pairs;
        g += 2.0 * e * inv;
    }
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = g;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sh[0][0];
        part[2 * blockIdx.x + 1] = sh[1][0];
    }
}

// Adam on fp32 master weights (bias-corrected), grads fp32
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t count, float lr, float b1, float b2, float eps, float c1, float c2)
{
    RG_GRID_LOOP(i, count)
    {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// fp32 [27][cout][cin] -> bf16 forward weights (same layout) and data-gradient weights
// [27][cin][cout] with the taps flipped (tap' = 26 - tap)
__global__ void k_weights_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                               __nv_bfloat16* __restrict__ wd, int cout, int cin)
{
    RG_GRID_LOOP(i, (size_t)27 * cout * cin)
    {
        const int ci = (int)(i % cin), co = (int)((i / cin) % cout), tap = (int)(i / ((size_t)cin * cout));
        const __nv_bfloat16 b = tobf(w[i]);
        if (wf) wf[i] = b;
        if (wd) wd[((size_t)(26 - tap) * cin + ci) * cout + co] = b;
    }
}

// ---- glue between the PDE's fields and the network (per sample n) --------------------
// stats[4n..4n+3] = {mu = mean log kappa, sY = max |Y| (1 if Y == 0), kappa_g = exp(mu),
// u_unit = 10 sY h^2 / kappa_g}: the network sees log kappa - mu and Y / sY and predicts
// u / u_unit (the solution scales with Y h^2 / kappa).  Fields are fp32 per element of the
// fine grid (fd, fh, fw), x fastest.
constexpr int kStatBlocks = 64;

// the network's per-element inputs from the PDE's coefficient arrays: kappa_e = A's first
// entry of element e (a_stride doubles per element: 9 for A per element, 72 for A expanded
// to the Gauss points, whose first point is read), y_e = mean of Y's y_points values
__global__ void k_element_fields(const double* __restrict__ A, int a_stride, const double* __restrict__ Y,
                                 int y_points, size_t nel, float* __restrict__ kappa, float* __restrict__ y)
{
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
        kappa[e] = (float)__ldcs(A + e * a_stride);
        double s = 0.0;
        for (int q = 0; q < y_points; ++q) s += __ldcs(Y + e * y_points + q);
        y[e] = (float)(s / y_points);
    }
}

__global__ void k_field_stats(const float* __restrict__ kappa, const float* __restrict__ y, size_t per_sample,
                              double* __restrict__ part)
{
    __shared__ double sh[2][256];
    const int n = blockIdx.y;
    double s = 0.0, m = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < per_sample; i += (size_t)gridDim.x * blockDim.x) {
        s += log((double)kappa[n * per_sample + i]);
        m = fmax(m, fabs((double)y[n * per_sample + i]));
    }
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * ((size_t)n * gridDim.x + blockIdx.x)] = sh[0][0];
        part[2 * ((size_t)n * gridDim.x + blockIdx.x) + 1] = sh[1][0];
    }
}

__global__ void k_field_stats_finish(const double* __restrict__ part, int nblocks, size_t per_sample, int nsamples,
                                     double h, float* __restrict__ stats)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nsamples) return;
    double s = 0.0, m = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        s += part[2 * ((size_t)n * nblocks + b)];
        m = fmax(m, part[2 * ((size_t)n * nblocks + b) + 1]);
    }
    const double mu = s / (double)per_sample;
    const double sy = m > 0.0 ? m : 1.0;
    const double kg = exp(mu);
    stats[4 * n + 0] = (float)mu;
    stats[4 * n + 1] = (float)sy;
    stats[4 * n + 2] = (float)kg;
    stats[4 * n + 3] = (float)(10.0 * sy * h * h / kg);
}

// network input: channel 0 = log kappa - mu, 1 = Y / sY (each the mean over the network
// cell's f^3 fine elements), 2..4 = the cell centre's (z, y, x) in the unit cube, others 0
__global__ void k_pack_input(const float* __restrict__ kappa, const float* __restrict__ y, int f, Act x,
                             const float* __restrict__ stats)
{
    const int fd = x.d * f, fh = x.h * f, fw = x.w * f;
    const float inv = 1.f / (float)(f * f * f);
    RG_GRID_LOOP(pos, x.positions())
    {
        int n, d, h, w;
        x.coords(pos, n, d, h, w);
        float lk = 0.f, yy = 0.f;
        for (int a = 0; a < f; ++a)
            for (int b = 0; b < f; ++b)
                for (int c = 0; c < f; ++c) {
                    const size_t e = (((size_t)n * fd + d * f + a) * fh + h * f + b) * fw + w * f + c;
                    lk += logf(kappa[e]);
                    yy += y[e];
                }
        __nv_bfloat16* xp = x.p + x.at(n, d, h, w);
        xp[0] = tobf(lk * inv - stats[4 * n]);
        xp[1] = tobf(yy * inv / stats[4 * n + 1]);
        // the cell centre's position in the unit cube: convolutions with zero padding cannot
        // tell the Dirichlet face (z = 1) from the others without it
        if (x.c > 4) {
            xp[2] = tobf(((float)d + 0.5f) / (float)x.d);
            xp[3] = tobf(((float)h + 0.5f) / (float)x.h);
            xp[4] = tobf(((float)w + 0.5f) / (float)x.w);
        }
        for (int c = 5; c < x.c; ++c) xp[c] = tobf(0.f);
    }
}

// training target: the solution's mean over each network cell (f^3 fine elements, 8 nodes
// each) in units of u_unit; nodes (fd+1)(fh+1)(fw+1) per sample, x fastest
__global__ void k_nodes_to_cells(const double* __restrict__ u, int f, int nsamples, int d_, int h_, int w_,
                                 const float* __restrict__ stats, float* __restrict__ t)
{
    const int fd = d_ * f, fh = h_ * f, fw = w_ * f;
    const size_t nodes = (size_t)(fd + 1) * (fh + 1) * (fw + 1);
    const size_t count = (size_t)nsamples * d_ * h_ * w_;
    RG_GRID_LOOP(i, count)
    {
        const int w = (int)(i % w_), h = (int)((i / w_) % h_), d = (int)((i / ((size_t)w_ * h_)) % d_);
        const int n = (int)(i / ((size_t)w_ * h_ * d_));
        const double* un = u + n * nodes;
        double s = 0.0;
        for (int a = 0; a <= f; ++a)
            for (int b = 0; b <= f; ++b)
                for (int c = 0; c <= f; ++c) {
                    // trapezoid weights over the block's nodes = mean of the elements' node means
                    const double wt = (a == 0 || a == f ? 0.5 : 1.0) * (b == 0 || b == f ? 0.5 : 1.0) *
                                      (c == 0 || c == f ? 0.5 : 1.0);
                    s += wt * un[((size_t)(d * f + a) * (fh + 1) + h * f + b) * (fw + 1) + w * f + c];
                }
        t[i] = (float)(s / ((double)f * f * f) / (double)stats[4 * n + 3]);
    }
}

// initial guess on the nodes of the fine grid (nd, nh, nw nodes per sample) from the
// network's cell values: trilinear between cell centres, clamped at the faces, times
// u_unit; zero where q > 0 (Dirichlet nodes)
__global__ void k_cells_to_nodes(const float* __restrict__ cells, int nsamples, int d_, int h_, int w_,
                                 const float* __restrict__ stats, int nd, int nh, int nw,
                                 const double* __restrict__ q, double* __restrict__ u)
{
    const size_t per = (size_t)nd * nh * nw;
    RG_GRID_LOOP(i, (size_t)nsamples * per)
    {
        const int n = (int)(i / per);
        const size_t r = i % per;
        const int x = (int)(r % nw), y = (int)((r / nw) % nh), z = (int)(r / ((size_t)nw * nh));
        double v = 0.0;
        if (!(q && q[i] > 0.0)) {
            float sx = (float)x * w_ / (float)(nw - 1) - 0.5f, sy = (float)y * h_ / (float)(nh - 1) - 0.5f,
                  sz = (float)z * d_ / (float)(nd - 1) - 0.5f;
            sx = fminf(fmaxf(sx, 0.f), (float)(w_ - 1));
            sy = fminf(fmaxf(sy, 0.f), (float)(h_ - 1));
            sz = fminf(fmaxf(sz, 0.f), (float)(d_ - 1));
            const int x0 = min((int)sx, w_ - 1), y0 = min((int)sy, h_ - 1), z0 = min((int)sz, d_ - 1);
            const int x1 = min(x0 + 1, w_ - 1), y1 = min(y0 + 1, h_ - 1), z1 = min(z0 + 1, d_ - 1);
            const float tx = sx - x0, ty = sy - y0, tz = sz - z0;
            const float* c = cells + (size_t)n * d_ * h_ * w_;
            auto at = [&](int zz, int yy, int xx) { return c[((size_t)zz * h_ + yy) * w_ + xx]; };
            const float c00 = at(z0, y0, x0) * (1 - tx) + at(z0, y0, x1) * tx;
            const float c01 = at(z0, y1, x0) * (1 - tx) + at(z0, y1, x1) * tx;
            const float c10 = at(z1, y0, x0) * (1 - tx) + at(z1, y0, x1) * tx;
            const float c11 = at(z1, y1, x0) * (1 - tx) + at(z1, y1, x1) * tx;
            const float c0 = c00 * (1 - ty) + c01 * ty, c1 = c10 * (1 - ty) + c11 * ty;
            v = (double)(c0 * (1 - tz) + c1 * tz) * (double)stats[4 * n + 3];
        }
        u[i] = v;
    }
}

int grid_elems(size_t count) { return (int)((count + 255) / 256 < (size_t)kNumSMs * 16 ? (count + 255) / 256 : kNumSMs * 16); }

}  // namespace
}  // namespace ws
}  // namespace rg

using namespace rg;
using namespace rg::ws;

#define RG_ACT_OK(a, name) RG_REQUIRE((a) && (a)->ptr && (a)->n > 0 && (a)->c > 0, name ": invalid activation")

extern "C" {

int rg_ws_avgpool(const rg_act* in, rg_act* out)
{
    RG_ACT_OK(in, "rg_ws_avgpool");
    RG_ACT_OK(out, "rg_ws_avgpool");
    RG_REQUIRE(out->d * 2 == in->d && out->h * 2 == in->h && out->w * 2 == in->w && out->c == in->c && out->n == in->n,
               "rg_ws_avgpool: out must be in halved");
    const Act o = act(out);
    RG_TIMED(T_WS_OPS, (k_avgpool<<<grid_elems(o.positions() * o.c), 256, 0, stream()>>>(act(in), o)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_avgpool_bwd(const rg_act* dout, const rg_act* in, const rg_act* dskip, int skip_off, rg_act* din)
{
    RG_ACT_OK(dout, "rg_ws_avgpool_bwd");
    RG_ACT_OK(in, "rg_ws_avgpool_bwd");
    RG_ACT_OK(din, "rg_ws_avgpool_bwd");
    RG_REQUIRE(dout->d * 2 == din->d && din->c == dout->c && in->c == din->c, "rg_ws_avgpool_bwd: shape mismatch");
    RG_REQUIRE(!dskip || (dskip->d == din->d && skip_off + din->c <= dskip->c), "rg_ws_avgpool_bwd: skip shape");
    const Act di = act(din);
    const Act ds = dskip ? act(dskip) : Act{nullptr, 0, 0, 0, 0, 0};
    RG_TIMED(T_WS_OPS, (k_avgpool_bwd<<<grid_elems(di.positions() * di.c), 256, 0, stream()>>>(act(dout), act(in), ds, skip_off, di)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_upcat(const rg_act* a, const rg_act* b, rg_act* out)
{
    RG_ACT_OK(a, "rg_ws_upcat");
    RG_ACT_OK(b, "rg_ws_upcat");
    RG_ACT_OK(out, "rg_ws_upcat");
    RG_REQUIRE(a->d * 2 == out->d && b->d == out->d && out->c == a->c + b->c, "rg_ws_upcat: shape mismatch");
    const Act o = act(out);
    RG_TIMED(T_WS_OPS, (k_upcat<<<grid_elems(o.positions() * o.c), 256, 0, stream()>>>(act(a), act(b), o)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_upcat_bwd(const rg_act* dcat, const rg_act* a, rg_act* da)
{
    RG_ACT_OK(dcat, "rg_ws_upcat_bwd");
    RG_ACT_OK(da, "rg_ws_upcat_bwd");
    RG_REQUIRE(da->d * 2 == dcat->d && da->h * 2 == dcat->h && da->w * 2 == dcat->w && da->c <= dcat->c &&
                   da->n == dcat->n,
               "rg_ws_upcat_bwd: shape mismatch");
    RG_REQUIRE(!a || (a->c == da->c && a->d == da->d && a->h == da->h && a->w == da->w && a->n == da->n),
               "rg_ws_upcat_bwd: mask shape must equal da's");
    const Act d = act(da);
    const Act am = a ? act(a) : Act{nullptr, 0, 0, 0, 0, 0};
    RG_TIMED(T_WS_OPS, (k_upcat_bwd<<<grid_elems(d.positions() * d.c), 256, 0, stream()>>>(act(dcat), am, d)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_head(const rg_act* x, const float* w, const float* b, float* out)
{
    RG_ACT_OK(x, "rg_ws_head");
    RG_REQUIRE(w && b && out, "rg_ws_head: NULL argument");
    const Act xa = act(x);
    RG_TIMED(T_WS_OPS, (k_head<<<grid_elems(xa.positions()), 256, 0, stream()>>>(xa, w, b, out)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

// column sums over positions: out[c] (+)= sum_pos v(pos, c) [* dout(pos)]; work holds
// kNumSMs*4 * v->c floats
int rg_ws_colsum(const rg_act* v, const float* dout, float* out, float* work, int accumulate)
{
    RG_ACT_OK(v, "rg_ws_colsum");
    RG_REQUIRE(out && work && v->c <= 128, "rg_ws_colsum: invalid argument");
    const Act va = act(v);
    const int blocks = kNumSMs * 4, threads = 64;
    const size_t sm = sizeof(float) * threads * v->c;
    if (dout)
        RG_TIMED(T_WS_OPS, (k_colsum<true><<<blocks, threads, sm, stream()>>>(va, dout, work, v->c)));
    else
        RG_TIMED(T_WS_OPS, (k_colsum<false><<<blocks, threads, sm, stream()>>>(va, nullptr, work, v->c)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_WS_OPS, (k_colsum_finish<<<1, 128, 0, stream()>>>(work, blocks, v->c, out, accumulate)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_head_bwd_x(const rg_act* x, const float* w, const float* dout, rg_act* dx)
{
    RG_ACT_OK(x, "rg_ws_head_bwd_x");
    RG_ACT_OK(dx, "rg_ws_head_bwd_x");
    RG_REQUIRE(w && dout && dx->c == x->c, "rg_ws_head_bwd_x: invalid argument");
    const Act xa = act(x);
    RG_TIMED(T_WS_OPS, (k_head_bwd_x<<<grid_elems(xa.positions() * xa.c), 256, 0, stream()>>>(xa, w, dout, act(dx))));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

// loss_dev (double) = mean (out - t)^2; dout = d loss / d out; *dsum_dev = sum of dout (the
// head's bias gradient) when not NULL; work: 2 * kNumSMs*4 doubles
int rg_ws_mse(const float* out, const float* target, int64_t count, float* dout, double* loss_dev, float* dsum_dev,
              double* work)
{
    RG_REQUIRE(out && target && dout && loss_dev && work && count > 0, "rg_ws_mse: invalid argument");
    const int blocks = kNumSMs * 4;
    RG_TIMED(T_WS_OPS, (k_mse<<<blocks, 256, 0, stream()>>>(out, target, (size_t)count, dout, work)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_WS_OPS, (k_mse_finish<<<1, 32, 0, stream()>>>(work, blocks, (size_t)count, loss_dev, dsum_dev)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_h1_loss(const float* out, const float* target, int n, int d, int h, int w, float lambda, float* dout,
                  double* loss_dev, float* dsum_dev, double* work)
{
    RG_REQUIRE(out && target && dout && loss_dev && work && n > 0 && d > 0 && h > 0 && w > 0 && lambda >= 0.f,
               "rg_ws_h1_loss: invalid argument");
    const int blocks = kNumSMs * 4;
    const size_t count = (size_t)n * d * h * w;
    RG_TIMED(T_WS_OPS, (k_h1_loss<<<blocks, 256, 0, stream()>>>(out, target, n, d, h, w, lambda, dout, work)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_WS_OPS, (k_mse_finish<<<1, 32, 0, stream()>>>(work, blocks, count, loss_dev, dsum_dev)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_adam(float* w, const float* g, float* m, float* v, int64_t count, float lr, float beta1, float beta2,
               float eps, int step)
{
    RG_REQUIRE(w && g && m && v && count > 0 && step > 0, "rg_ws_adam: invalid argument");
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    RG_TIMED(T_WS_OPS, (k_adam<<<grid_elems((size_t)count), 256, 0, stream()>>>(w, g, m, v, (size_t)count, lr, beta1, beta2, eps, c1, c2)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_weights_bf16(const float* w, void* w_fwd, void* w_dgrad, int cout, int cin)
{
    RG_REQUIRE(w && (w_fwd || w_dgrad) && cout > 0 && cin > 0, "rg_ws_weights_bf16: invalid argument");
    RG_TIMED(T_WS_OPS, (k_weights_bf16<<<grid_elems((size_t)27 * cout * cin), 256, 0, stream()>>>(
        w, static_cast<__nv_bfloat16*>(w_fwd), static_cast<__nv_bfloat16*>(w_dgrad), cout, cin)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

// per-sample normalisation of the fields (fine grid fd x fh x fw elements, h = the network
// grid's cell size); stats: 4 floats per sample, work: 2 * 64 * nsamples doubles
int rg_ws_field_stats(const float* kappa, const float* y, int nsamples, int64_t per_sample, double h_net,
                      float* stats, double* work)
{
    RG_REQUIRE(kappa && y && stats && work && nsamples > 0 && per_sample > 0 && h_net > 0,
               "rg_ws_field_stats: invalid argument");
    RG_TIMED(T_WS_OPS, (k_field_stats<<<dim3(kStatBlocks, nsamples), 256, 0, stream()>>>(kappa, y, (size_t)per_sample, work)));
    RG_CHECK_LAUNCH();
    RG_TIMED(T_WS_OPS, (k_field_stats_finish<<<(nsamples + 63) / 64, 64, 0, stream()>>>(work, kStatBlocks, (size_t)per_sample, nsamples,
                                                                     h_net, stats)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_element_fields(const double* A, int a_stride, const double* Y, int y_points, int64_t nel, float* kappa,
                         float* y)
{
    RG_REQUIRE(A && Y && kappa && y && a_stride >= 1 && y_points >= 1 && nel > 0,
               "rg_ws_element_fields: invalid argument");
    const int grid = (int)std::min<int64_t>((nel + 255) / 256, 148 * 8);
    RG_TIMED(T_WS_OPS, (k_element_fields<<<grid, 256, 0, stream()>>>(A, a_stride, Y, y_points, (size_t)nel, kappa, y)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_pack_input(const float* kappa, const float* y, int factor, rg_act* x, const float* stats)
{
    RG_ACT_OK(x, "rg_ws_pack_input");
    RG_REQUIRE(kappa && y && stats && x->c >= 5 && factor >= 1, "rg_ws_pack_input: invalid argument");
    const Act xa = act(x);
    RG_TIMED(T_WS_OPS, (k_pack_input<<<grid_elems(xa.positions()), 256, 0, stream()>>>(kappa, y, factor, xa, stats)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_nodes_to_cells(const double* u, int factor, int nsamples, int d, int h, int w, const float* stats,
                         float* target)
{
    RG_REQUIRE(u && stats && target && factor >= 1 && nsamples > 0 && d > 0 && h > 0 && w > 0,
               "rg_ws_nodes_to_cells: invalid argument");
    RG_TIMED(T_WS_OPS, (k_nodes_to_cells<<<grid_elems((size_t)nsamples * d * h * w), 256, 0, stream()>>>(u, factor, nsamples, d, h, w,
                                                                                   stats, target)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

int rg_ws_cells_to_nodes(const float* cells, int nsamples, int d, int h, int w, const float* stats, int nd, int nh,
                         int nw, const double* q, double* u)
{
    RG_REQUIRE(cells && stats && u && nsamples > 0 && d > 0 && h > 0 && w > 0 && nd > 1 && nh > 1 && nw > 1,
               "rg_ws_cells_to_nodes: invalid argument");
    RG_TIMED(T_WS_OPS, (k_cells_to_nodes<<<grid_elems((size_t)nsamples * nd * nh * nw), 256, 0, stream()>>>(cells, nsamples, d, h, w,
                                                                                      stats, nd, nh, nw, q, u)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

}  // extern "C"
