// rg_residual_norms_noalloc: the residual-norm reduction of rg_residual_norms with its
// scratch in a fixed, statically allocated device array instead of memory the library
// allocates.  It exists for callers that cannot let a library call cudaMalloc: hosts
// that hand all device memory to their own pool or caching allocator (a cudaMalloc behind
// its back can fail or fragment that budget), and latency-critical loops in which the
// implicit device synchronisation of cudaMalloc/cudaFree is not acceptable.
//
// Limits and sharing:
//  * the scratch holds the partial sums of at most kMaxPartialBlocks CTAs, the result
//    and the reduction counter: (2 * 1184 + 4) doubles = 18,976 bytes, held by every GPU
//    that loads the library until the process exits;
//  * all calls share that array and it keeps the last call's contents; the counter is
//    cleared at the start of every call.  Calls that overlap on the GPU (different
//    streams or threads at the same time) race on the array and must be serialised by
//    the caller;
//  * the first call on a device looks up the array's device address with the device
//    current (cudaGetSymbolAddress) and caches it; make that first call before any
//    stream capture.  The cached address does not survive cudaDeviceReset: a call whose
//    device work fails drops it, so the next call looks it up again.
//
// The reduction grid of k_residual_norms is capped at residual::kMaxBlocks CTAs for every
// size, so the array always holds enough partial sums; the size check below guards that
// invariant should the cap ever change.
#include <cmath>
#include <mutex>

#include "rg_residual.cuh"

namespace rg {
namespace {

constexpr int kMaxPartialBlocks = residual::kMaxBlocks;          // 1184 CTAs
static_assert(residual::kMaxBlocks >= kNumSMs * 8,
              "the residual grid (grid_for caps it at kNumSMs * 8 CTAs) must fit the static scratch");
constexpr int kScratchDoubles = 2 * kMaxPartialBlocks + 4;       // partials, result, counter
constexpr int kOutSlot = 2 * kMaxPartialBlocks;                  // 2 doubles
constexpr int kCounterSlot = 2 * kMaxPartialBlocks + 2;          // an unsigned in a double slot

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// device address of the scratch on the current device, looked up once per device
int scratch_address(double** out)
{
    int dev = 0;
    RG_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("rg_residual_norms_noalloc: device ordinal out of range");
        return RG_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error(std::string("rg_residual_norms_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return RG_CUDA_ERROR;
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return RG_OK;
}

// forgets the current device's address after failed device work (e.g. after a device reset)
void drop_address()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_addr[dev] = nullptr;
}

// the reduction on the static scratch: clear the counter, launch, read the two results
int norms_with_scratch(Matrix* m, double* scratch, int grid, const double* rhs, const double* x, double* l2_host,
                       double* linf_host)
{
    const Domain* d = m->dom;
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + kCounterSlot);
    double* out = scratch + kOutSlot;
    RG_CHECK_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), stream()));
    RG_TIMED(T_NORMS, (residual::k_residual_norms<<<grid, residual::kThreads, 0, stream()>>>(
                          d->n, d->ptr, d->idx, m->val, m->balanced ? m->bv : nullptr, rhs, x,
                          ReduceBuf{scratch, counter}, out)));
    RG_CHECK_LAUNCH();
    double h[2];
    RG_CHECK_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    RG_CHECK_CUDA(cudaStreamSynchronize(stream()));
    if (l2_host) *l2_host = std::sqrt(h[0]);
    if (linf_host) *linf_host = h[1];
    return RG_OK;
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" int rg_residual_norms_noalloc(rg_matrix* mat, const double* rhs, const double* x, double* l2_host,
                                         double* linf_host)
{
    RG_REQUIRE(mat && rhs && x, "rg_residual_norms_noalloc: NULL argument");
    if (mat->m.nb != 1) {
        set_error("rg_residual_norms_noalloc: PDE systems are not supported (use rg_residual_norms)");
        return RG_NOT_SUPPORTED;
    }
    Matrix* m = &mat->m;
    const Domain* d = m->dom;
    const int grid = residual::grid(d->n);
    if (grid > kMaxPartialBlocks) {
        set_error("rg_residual_norms_noalloc: the reduction needs " + std::to_string(grid) +
                  " partial sums but the static scratch holds " + std::to_string(kMaxPartialBlocks));
        return RG_INVALID_ARG;
    }
    double* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    rc = norms_with_scratch(m, scratch, grid, rhs, x, l2_host, linf_host);
    if (rc == RG_CUDA_ERROR) drop_address();
    return rc;
}
