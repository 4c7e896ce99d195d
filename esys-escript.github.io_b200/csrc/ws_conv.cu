// 3x3x3 convolutions of the warm-start network on the 5th-generation tensor cores
// (tcgen05 UMMA, bf16 operands, fp32 accumulators in tensor memory).
//
// Activations are bf16, channels-last, with one zero slice before and after every
// sample along depth: x[z][h][w][c] with z = n*(D+2) + 1 + d, so a 3x3x3 stencil never
// crosses into the neighbouring sample, and the W/H borders are the zero fill of the TMA
// loads.
//
// Forward (and data-gradient) convolution as an implicit GEMM: one CTA computes a tile of
// 128 output positions (a BW x BH x BZ box) x Cout channels.  K runs over the 27 taps x
// Cin/16 channel chunks; for each (tap, chunk) the producer warp loads with TMA the input
// box shifted by the tap (128 positions x 16 channels, 32-byte swizzle) and the tap's
// 16-channel weight slice (Cout x 16), the MMA warp issues one 128 x Cout x 16 UMMA into
// tensor memory and releases the stage through tcgen05.commit, and four epilogue warps
// read the accumulator (one TMEM lane = one output position per thread), add the bias,
// apply ReLU and/or the ReLU mask of the layer below (data gradient), and store bf16.
#include <cuda.h>

#include <algorithm>
#include <string>

#include "rg_internal.cuh"
#include "ws_conv.cuh"

namespace rg {
namespace ws {

constexpr int kStages = 8;
constexpr int kConvThreads = 192;  // warp 0 TMA, warp 1 MMA + TMEM, warps 2-5 epilogue
constexpr int kATile = 128 * 32;   // 128 positions x 16 bf16

struct ConvArgs {
    CUtensorMap xmap;  // input: dims (Cin, W, H, Z), box (16, BW, BH, BZ), 32B swizzle
    CUtensorMap wmap;  // weights [27][Cout][Cin]: dims (Cin, 27*Cout), box (16, Cout), 32B swizzle
    const float* bias;          // Cout or null
    __nv_bfloat16* out;         // [Z][H][W][Cout]
    const __nv_bfloat16* mask;  // [Z][H][W][Cout] or null: out *= (mask > 0)
    int W, H, D, Cin;
    int BW, BH, BZ;
    int tiles_w, tiles_h, tiles_z;
    int relu;
    int* err;
};

template <int COUT>
struct ConvSmem {
    static constexpr int kB = COUT * 32;
    static constexpr int kBPad = (kB + 1023) / 1024 * 1024;
    static constexpr int kStage = kATile + kBPad;
    static constexpr int kBytes = kStages * kStage + 1024;  // + alignment slack
};

template <int COUT>
__global__ void __launch_bounds__(kConvThreads) k_conv3(const __grid_constant__ ConvArgs a)
{
    using S = ConvSmem<COUT>;
    constexpr int kTmemCols = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : (COUT <= 128 ? 128 : 256));
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full;
    __shared__ uint32_t tmem_slot;
    __shared__ int bad;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // tile coordinates
    int tile = blockIdx.x;
    const int tw = tile % a.tiles_w;
    tile /= a.tiles_w;
    const int th = tile % a.tiles_h;
    const int tz = tile / a.tiles_h;
    const int per_sample = a.D / a.BZ;
    const int w0 = tw * a.BW, h0 = th * a.BH;
    const int z0 = (tz / per_sample) * (a.D + 2) + 1 + (tz % per_sample) * a.BZ;
    const int chunks = a.Cin / 16;
    const int ksteps = 27 * chunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&acc_full, 1);
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- producer
        for (int k = 0; k < ksteps; ++k) {
            const int s = k % kStages;
            if (k >= kStages && !mbar_wait(&empty[s], (uint32_t)(((k / kStages) - 1) & 1))) {
                bad = 1;
                break;
            }
            const int tap = k / chunks, c = k % chunks;
            const int kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
            uint8_t* st = smem + s * S::kStage;
            mbar_expect_tx(&full[s], kATile + S::kB);
            tma_load_4d(st, &a.xmap, c * 16, w0 + kw - 1, h0 + kh - 1, z0 + kd - 1, &full[s]);
            tma_load_2d(st + kATile, &a.wmap, c * 16, tap * COUT, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        constexpr uint32_t idesc = idesc_bf16(COUT, 0, 0);
        bool ok = true;
        for (int k = 0; k < ksteps; ++k) {
            const int s = k % kStages;
            if (!mbar_wait(&full[s], (uint32_t)((k / kStages) & 1))) {
                bad = 1;
                ok = false;
                break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * S::kStage;
            const uint64_t ad = smem_desc(st, 16, 256, LAYOUT_SW32);
            const uint64_t bd = smem_desc(st + kATile, 16, 256, LAYOUT_SW32);
            umma_f16(tmem, ad, bd, idesc, k > 0 ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&acc_full);
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM lane quarter (warp % 4) -> 32 output positions
        const int q = warp & 3;
        const int m = 32 * q + lane;
        // one decision per warp: the TMEM loads below are warp-collective
        const bool ready = __all_sync(0xffffffffu, mbar_wait(&acc_full, 0));
        tc_fence_after();
        if (!ready) {
            bad = 1;
        } else {
            const int w = w0 + m % a.BW;
            const int h = h0 + (m / a.BW) % a.BH;
            const int z = z0 + m / (a.BW * a.BH);
            const size_t row = ((size_t)z * a.H + h) * a.W + w;
            __nv_bfloat16* o = a.out + row * COUT;
            const __nv_bfloat16* mk = a.mask ? a.mask + row * COUT : nullptr;
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                __align__(16) __nv_bfloat16 ob[16];
                __align__(16) __nv_bfloat16 mb[16];
                if (mk) {
                    *reinterpret_cast<uint4*>(mb) = *reinterpret_cast<const uint4*>(mk + c0);
                    *reinterpret_cast<uint4*>(mb + 8) = *reinterpret_cast<const uint4*>(mk + c0 + 8);
                }
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float x = v[i] + (a.bias ? a.bias[c0 + i] : 0.f);
                    if (a.relu) x = fmaxf(x, 0.f);
                    if (mk && !(__bfloat162float(mb[i]) > 0.f)) x = 0.f;
                    ob[i] = __float2bfloat16_rn(x);
                }
                *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(ob);
                *reinterpret_cast<uint4*>(o + c0 + 8) = *reinterpret_cast<const uint4*>(ob + 8);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
    if (bad && threadIdx.x == 0) atomicOr(a.err, 1);
}

// ------------------------------------------------------------------ box-reuse forward convolution
// The same convolution for grids whose tiles are 8 (w) x 16 (h) x 2 (z) output positions and
// Cout <= 64.  A GEMM row is an output position, w fastest, so one 256-byte atom of the
// 32-byte-swizzled K-major operand is one h-row of 8 positions.  A tap's h and z shifts then
// move the operand by whole atoms: the A operand of tap (kw, kh, kd) for output slice zz is
// 16 consecutive atoms of an input box that the producer loads once per 16-channel chunk and
// per kw (8 x 18 x 4 positions: the tile plus its h and z halo), starting at atom
// kh + 18 (kd + zz).  Per chunk: 3 TMA boxes (55 KB) and the chunk's 27 weight slices instead
// of 27 shifted 4 KB boxes per 128 positions, and 54 UMMAs (two 128 x Cout accumulators in
// tensor memory, one per output z slice).
constexpr int kBoxW = 8, kBoxH = 16, kBoxZ = 2;
constexpr int kBoxRows = kBoxW * (kBoxH + 2) * (kBoxZ + 2);  // 576 input positions per kw box
constexpr int kBoxBytes = kBoxRows * 32;                      // 18 KB
constexpr int kBoxA = 3 * kBoxBytes;                          // the three kw boxes

template <int COUT, int S>
struct BoxSmem {
    static constexpr int kB = 27 * COUT * 32;  // the chunk's weight slices of every tap
    static constexpr int kStage = (kBoxA + kB + 1023) / 1024 * 1024;
    static constexpr int kBytes = S * kStage + 1024;  // + alignment slack
};

template <int COUT, int S>
__global__ void __launch_bounds__(kConvThreads) k_conv3_box(const __grid_constant__ ConvArgs a)
{
    using M = BoxSmem<COUT, S>;
    constexpr int kAcc = kBoxZ * COUT;  // TMEM columns: one accumulator per output z slice
    constexpr int kTmemCols = kAcc <= 32 ? 32 : (kAcc <= 64 ? 64 : (kAcc <= 128 ? 128 : 256));
    static_assert(kAcc <= 256, "the accumulators must fit 256 TMEM columns");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], acc_full;
    __shared__ uint32_t tmem_slot;
    __shared__ int bad;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int tile = blockIdx.x;
    const int tw = tile % a.tiles_w;
    tile /= a.tiles_w;
    const int th = tile % a.tiles_h;
    const int tz = tile / a.tiles_h;
    const int per_sample = a.D / kBoxZ;
    const int w0 = tw * kBoxW, h0 = th * kBoxH;
    const int z0 = (tz / per_sample) * (a.D + 2) + 1 + (tz % per_sample) * kBoxZ;
    const int chunks = a.Cin / 16;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&acc_full, 1);
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------- producer: per chunk the three kw boxes and the 27 weight slices
        for (int k = 0; k < chunks; ++k) {
            const int s = k % S;
            if (k >= S && !mbar_wait(&empty[s], (uint32_t)(((k / S) - 1) & 1))) {
                bad = 1;
                break;
            }
            uint8_t* st = smem + s * M::kStage;
            mbar_expect_tx(&full[s], kBoxA + M::kB);
            for (int kw = 0; kw < 3; ++kw)
                tma_load_4d(st + kw * kBoxBytes, &a.xmap, k * 16, w0 + kw - 1, h0 - 1, z0 - 1, &full[s]);
            for (int t = 0; t < 27; ++t) tma_load_2d(st + kBoxA + t * COUT * 32, &a.wmap, k * 16, t * COUT, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        constexpr uint32_t idesc = idesc_bf16(COUT, 0, 0);
        bool ok = true;
        for (int k = 0; k < chunks; ++k) {
            const int s = k % S;
            if (!mbar_wait(&full[s], (uint32_t)((k / S) & 1))) {
                bad = 1;
                ok = false;
                break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * M::kStage;
            // the output slices' accumulations alternate: consecutive UMMAs are independent; the
            // descriptors are the stage's plus constant offsets (the loops unroll), so that the
            // one issuing thread spends a few instructions per UMMA
            const uint64_t ad0 = smem_desc(st, 16, 256, LAYOUT_SW32);
            const uint64_t bd0 = smem_desc(st + kBoxA, 16, 256, LAYOUT_SW32);
#pragma unroll
            for (int t = 0; t < 27; ++t)
#pragma unroll
                for (int zz = 0; zz < kBoxZ; ++zz) {
                    const int kw = t % 3, kh = (t / 3) % 3, kd = t / 9;
                    const uint64_t ad = desc_add(ad0, kw * kBoxBytes + (kh + (kBoxH + 2) * (kd + zz)) * 256);
                    const uint64_t bd = desc_add(bd0, t * COUT * 32);
                    umma_f16(tmem + (uint32_t)(zz * COUT), ad, bd, idesc, (k > 0 || t > 0) ? 1u : 0u);
                }
            umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&acc_full);
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM lane quarter (warp % 4) -> 32 output positions
        const int q = warp & 3;
        const int m = 32 * q + lane;  // GEMM row: w = m % 8, h = m / 8
        const bool ready = __all_sync(0xffffffffu, mbar_wait(&acc_full, 0));
        tc_fence_after();
        if (!ready) {
            bad = 1;
        } else {
            const int w = w0 + (m % kBoxW);
            const int h = h0 + m / kBoxW;
#pragma unroll 1
            for (int zz = 0; zz < kBoxZ; ++zz) {
                const size_t row = ((size_t)(z0 + zz) * a.H + h) * a.W + w;
                __nv_bfloat16* o = a.out + row * COUT;
                const __nv_bfloat16* mk = a.mask ? a.mask + row * COUT : nullptr;
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16) {
                    float v[16];
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(zz * COUT + c0), v);
                    __align__(16) __nv_bfloat16 ob[16];
                    __align__(16) __nv_bfloat16 mb[16];
                    if (mk) {
                        *reinterpret_cast<uint4*>(mb) = *reinterpret_cast<const uint4*>(mk + c0);
                        *reinterpret_cast<uint4*>(mb + 8) = *reinterpret_cast<const uint4*>(mk + c0 + 8);
                    }
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        float x = v[i] + (a.bias ? a.bias[c0 + i] : 0.f);
                        if (a.relu) x = fmaxf(x, 0.f);
                        if (mk && !(__bfloat162float(mb[i]) > 0.f)) x = 0.f;
                        ob[i] = __float2bfloat16_rn(x);
                    }
                    *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(ob);
                    *reinterpret_cast<uint4*>(o + c0 + 8) = *reinterpret_cast<const uint4*>(ob + 8);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
    if (bad && threadIdx.x == 0) atomicOr(a.err, 1);
}

// ------------------------------------------------------------------ persistent box-reuse forward convolution
// k_conv3_box's tiles and operands, with each CTA walking tiles blockIdx.x, + gridDim.x, ...:
// the weights of every 16-channel chunk are loaded once and stay in shared memory, the input
// boxes of consecutive (tile, chunk) steps stream through an S-stage ring, and the
// accumulators of consecutive tiles alternate between two TMEM buffers, so that the box loads
// of the next tile, its UMMAs and the epilogue of the previous tile overlap (k_conv3_box runs
// the three one after the other, once per CTA).  Every wait is bounded; a wait that runs out
// sets the error flag and the CTA stops.
// test hook of the persistent convolution's bounded waits (rg_test_wait_limit): a poll limit
// (0: the default) and a switch that makes the producer issue no copies
struct ConvWaitCtl {
    int polls;
    int withhold;
};
__device__ ConvWaitCtl g_conv_wait = {0, 0};

template <int COUT>
struct BoxPSmem {
    static constexpr int kB = 27 * COUT * 32;                 // one chunk's weight slices
    static constexpr int kBPad = (kB + 1023) / 1024 * 1024;
    static constexpr int bytes(int chunks, int stages) { return chunks * kBPad + stages * kBoxA + 1024; }
};

template <int COUT, int S>
__global__ void __launch_bounds__(kConvThreads) k_conv3_boxp(const __grid_constant__ ConvArgs a)
{
    using M = BoxPSmem<COUT>;
    constexpr int kAcc = kBoxZ * COUT;  // TMEM columns of one tile (one accumulator per output z slice)
    constexpr int kTmemCols =
        2 * kAcc <= 32 ? 32 : (2 * kAcc <= 64 ? 64 : (2 * kAcc <= 128 ? 128 : (2 * kAcc <= 256 ? 256 : 512)));
    static_assert(2 * kAcc <= 512, "two tiles' accumulators must fit the 512 TMEM columns");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], wfull, acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int bad;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunks = a.Cin / 16;
    const ConvWaitCtl wc = g_conv_wait;
    const int polls = wc.polls > 0 ? wc.polls : 1 << 22;
    const int ntiles = a.tiles_w * a.tiles_h * a.tiles_z;
    const int per_sample = a.D / kBoxZ;
    uint8_t* wsm = smem;                             // chunks x kBPad: the weights
    uint8_t* ring = smem + chunks * M::kBPad;        // S x kBoxA: the input boxes
    // origin of tile `tile`: first output w, h and the row z of its first output slice
    auto origin = [&](int tile, int& w0, int& h0, int& z0) {
        const int tw = tile % a.tiles_w;
        tile /= a.tiles_w;
        const int th = tile % a.tiles_h;
        const int tz = tile / a.tiles_h;
        w0 = tw * kBoxW;
        h0 = th * kBoxH;
        z0 = (tz / per_sample) * (a.D + 2) + 1 + (tz % per_sample) * kBoxZ;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&wfull, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);  // the four epilogue warps
        }
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0 && !wc.withhold) {
        // ---------------- producer: the weights once, then per (tile, chunk) the three kw boxes
        mbar_expect_tx(&wfull, (uint32_t)(chunks * M::kB));
        for (int k = 0; k < chunks; ++k)
            for (int t = 0; t < 27; ++t)
                tma_load_2d(wsm + k * M::kBPad + t * COUT * 32, &a.wmap, k * 16, t * COUT, &wfull);
        int it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            int w0, h0, z0;
            origin(tile, w0, h0, z0);
            for (int k = 0; k < chunks; ++k, ++it) {
                const int s = it % S;
                if (it >= S && !mbar_wait(&empty[s], (uint32_t)(((it / S) - 1) & 1), polls)) {
                    ok = false;
                    break;
                }
                uint8_t* st = ring + s * kBoxA;
                mbar_expect_tx(&full[s], kBoxA);
                for (int kw = 0; kw < 3; ++kw)
                    tma_load_4d(st + kw * kBoxBytes, &a.xmap, k * 16, w0 + kw - 1, h0 - 1, z0 - 1, &full[s]);
            }
        }
        if (!ok) bad = 1;
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: tile j accumulates into TMEM buffer j & 1
        constexpr uint32_t idesc = idesc_bf16(COUT, 0, 0);
        bool ok = mbar_wait(&wfull, 0, polls);
        int it = 0, j = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++j) {
            const int b = j & 1;
            // the epilogue has read out what tile j - 2 left in this buffer
            if (j >= 2 && !mbar_wait(&acc_empty[b], (uint32_t)(((j >> 1) - 1) & 1), polls)) {
                ok = false;
                break;
            }
            tc_fence_after();
            for (int k = 0; k < chunks; ++k, ++it) {
                const int s = it % S;
                if (!mbar_wait(&full[s], (uint32_t)((it / S) & 1), polls)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint8_t* st = ring + s * kBoxA;
                const uint8_t* wk = wsm + k * M::kBPad;
                // the output slices' accumulations alternate: consecutive UMMAs are independent;
                // descriptors are the stage's plus constant offsets (the loops unroll): the
                // issuing thread, not the tensor pipe, set the pace with descriptors built per UMMA
                const uint64_t ad0 = smem_desc(st, 16, 256, LAYOUT_SW32);
                const uint64_t bd0 = smem_desc(wk, 16, 256, LAYOUT_SW32);
                const uint32_t d0 = tmem + (uint32_t)(b * kAcc);
#pragma unroll
                for (int t = 0; t < 27; ++t)
#pragma unroll
                    for (int zz = 0; zz < kBoxZ; ++zz) {
                        const int kw = t % 3, kh = (t / 3) % 3, kd = t / 9;
                        const uint64_t ad = desc_add(ad0, kw * kBoxBytes + (kh + (kBoxH + 2) * (kd + zz)) * 256);
                        const uint64_t bd = desc_add(bd0, t * COUT * 32);
                        umma_f16(d0 + (uint32_t)(zz * COUT), ad, bd, idesc, (k > 0 || t > 0) ? 1u : 0u);
                    }
                umma_commit(&empty[s]);  // the stage is free once these UMMAs have read it
            }
            if (!ok) break;
            umma_commit(&acc_full[b]);   // tile j's accumulators are complete
        }
        if (!ok) bad = 1;
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM lane quarter (warp % 4) -> 32 output positions
        const int q = warp & 3;
        const int m = 32 * q + lane;  // GEMM row: w = m % 8, h = m / 8
        int j = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++j) {
            const int b = j & 1;
            const bool ready = __all_sync(0xffffffffu, mbar_wait(&acc_full[b], (uint32_t)((j >> 1) & 1), polls));
            if (!ready) {
                bad = 1;
                break;
            }
            tc_fence_after();
            int w0, h0, z0;
            origin(tile, w0, h0, z0);
            const int w = w0 + (m % kBoxW);
            const int h = h0 + m / kBoxW;
#pragma unroll 1
            for (int zz = 0; zz < kBoxZ; ++zz) {
                const size_t row = ((size_t)(z0 + zz) * a.H + h) * a.W + w;
                __nv_bfloat16* o = a.out + row * COUT;
                const __nv_bfloat16* mk = a.mask ? a.mask + row * COUT : nullptr;
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16) {
                    float v[16];
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * kAcc + zz * COUT + c0), v);
                    __align__(16) __nv_bfloat16 ob[16];
                    __align__(16) __nv_bfloat16 mb[16];
                    if (mk) {
                        *reinterpret_cast<uint4*>(mb) = *reinterpret_cast<const uint4*>(mk + c0);
                        *reinterpret_cast<uint4*>(mb + 8) = *reinterpret_cast<const uint4*>(mk + c0 + 8);
                    }
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        float x = v[i] + (a.bias ? a.bias[c0 + i] : 0.f);
                        if (a.relu) x = fmaxf(x, 0.f);
                        if (mk && !(__bfloat162float(mb[i]) > 0.f)) x = 0.f;
                        ob[i] = __float2bfloat16_rn(x);
                    }
                    *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(ob);
                    *reinterpret_cast<uint4*>(o + c0 + 8) = *reinterpret_cast<const uint4*>(ob + 8);
                }
            }
            // this warp's lanes of buffer b are read: the MMA issuer may overwrite them
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
    if (bad && threadIdx.x == 0) atomicOr(a.err, 1);
}

// ------------------------------------------------------------------ weight gradient
// dW[tap][co][ci] = sum_pos X[pos + off(tap)][ci] * G[pos][co] as a GEMM with
//   M = 128 rows = 8 (tap, 16-channel chunk) pairs x 16 channels,  N = Cout,  K = positions.
// Both operands are M/N-major with 32-byte swizzle: for each pair the producer loads the
// input box shifted by the pair's tap (kWgKP positions x 16 channels) and for each
// 16-channel group of Cout the gradient box (kWgKP positions x 16 channels).  A CTA
// accumulates the positions of its K split in TMEM and writes its 128 x Cout partial sums;
// k_wgrad_reduce adds the splits in a fixed order into dW (fp32, [27][Cout][Cin]).
constexpr int kWgKP = 64;                  // positions per stage (4 UMMAs of K = 16)
constexpr int kWgStages = 3;
constexpr int kWgA = 8 * kWgKP * 32;       // 16 KB

struct WgradArgs {
    CUtensorMap xmap;  // input activations, box (16, BW, BH, BZ) with BW*BH*BZ = kWgKP
    CUtensorMap gmap;  // output gradient (Cout channels), same box
    float* partials;   // [ksplit][mtiles*128][Cout]
    int W, H, D, Cin, npairs;
    int BW, BH, BZ, tiles_w, tiles_h, tiles_z;
    int ptiles, ksplit, mtiles;
    int* err;
};

template <int COUT>
struct WgSmem {
    static constexpr int kB = (COUT / 16) * kWgKP * 32;
    static constexpr int kStage = kWgA + (kB + 1023) / 1024 * 1024;
    static constexpr int kBytes = kWgStages * kStage + 1024;
};

template <int COUT>
__global__ void __launch_bounds__(kConvThreads) k_wgrad(const __grid_constant__ WgradArgs a)
{
    using S = WgSmem<COUT>;
    constexpr int kTmemCols = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : (COUT <= 128 ? 128 : 256));
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kWgStages], empty[kWgStages], acc_full;
    __shared__ uint32_t tmem_slot;
    __shared__ int bad;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x % a.mtiles;
    const int ks = blockIdx.x / a.mtiles;
    // this split's position tiles
    const int per = (a.ptiles + a.ksplit - 1) / a.ksplit;
    const int pt0 = ks * per;
    const int pt1 = min(a.ptiles, pt0 + per);
    const int nk = pt1 > pt0 ? pt1 - pt0 : 0;
    const int per_sample = a.D / a.BZ;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kWgStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&acc_full, 1);
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0) {
        for (int k = 0; k < nk; ++k) {
            const int s = k % kWgStages;
            if (k >= kWgStages && !mbar_wait(&empty[s], (uint32_t)(((k / kWgStages) - 1) & 1))) {
                bad = 1;
                break;
            }
            int t = pt0 + k;
            const int tw = t % a.tiles_w;
            t /= a.tiles_w;
            const int th = t % a.tiles_h;
            const int tz = t / a.tiles_h;
            const int w0 = tw * a.BW, h0 = th * a.BH;
            const int z0 = (tz / per_sample) * (a.D + 2) + 1 + (tz % per_sample) * a.BZ;
            uint8_t* st = smem + s * S::kStage;
            mbar_expect_tx(&full[s], kWgA + S::kB);
            for (int p = 0; p < 8; ++p) {
                // pairs past the end re-load the last pair; their rows are discarded
                const int pair = min(mt * 8 + p, a.npairs - 1);
                const int chunks = a.Cin / 16;
                const int tap = pair / chunks, c = pair % chunks;
                const int kw = tap % 3, kh = (tap / 3) % 3, kd = tap / 9;
                tma_load_4d(st + p * kWgKP * 32, &a.xmap, c * 16, w0 + kw - 1, h0 + kh - 1, z0 + kd - 1, &full[s]);
            }
            for (int g = 0; g < COUT / 16; ++g)
                tma_load_4d(st + kWgA + g * kWgKP * 32, &a.gmap, g * 16, w0, h0, z0, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(COUT, 1, 1);
        bool ok = true;
        for (int k = 0; k < nk; ++k) {
            const int s = k % kWgStages;
            if (!mbar_wait(&full[s], (uint32_t)((k / kWgStages) & 1))) {
                bad = 1;
                ok = false;
                break;
            }
            tc_fence_after();
            const uint8_t* st = smem + s * S::kStage;
#pragma unroll
            for (int j = 0; j < kWgKP / 16; ++j) {
                // K slice j: 16 positions = 2 groups of 8 rows of 32 B
                const uint64_t ad = smem_desc(st + j * 512, kWgKP * 32, 256, LAYOUT_SW32);
                const uint64_t bd = smem_desc(st + kWgA + j * 512, kWgKP * 32, 256, LAYOUT_SW32);
                umma_f16(tmem, ad, bd, idesc, (k > 0 || j > 0) ? 1u : 0u);
            }
            umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&acc_full);
    } else if (warp >= 2) {
        const int q = warp & 3;
        const int m = 32 * q + lane;
        const bool ready = nk == 0 || __all_sync(0xffffffffu, mbar_wait(&acc_full, 0));
        tc_fence_after();
        float* dst = a.partials + ((size_t)ks * a.mtiles * 128 + (size_t)mt * 128 + m) * COUT;
        if (!ready) {
            bad = 1;
        } else if (nk == 0) {
            for (int c = 0; c < COUT; ++c) dst[c] = 0.f;
        } else {
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4*>(dst + c0 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
    if (bad && threadIdx.x == 0) atomicOr(a.err, 1);
}

// dW[tap][co][ci] = sum over splits (fixed order) of partials[split][pair*16 + ci%16][co]
__global__ void k_wgrad_reduce(const float* __restrict__ partials, float* __restrict__ dw, int ksplit, int mtiles,
                               int cout, int cin, int accumulate)
{
    const int total = 27 * cout * cin;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        const int ci = idx % cin, co = (idx / cin) % cout, tap = idx / (cin * cout);
        const int row = (tap * (cin / 16) + ci / 16) * 16 + ci % 16;
        float s = 0.f;
        for (int k = 0; k < ksplit; ++k) s += partials[((size_t)k * mtiles * 128 + row) * cout + co];
        dw[idx] = accumulate ? dw[idx] + s : s;
    }
}

// ------------------------------------------------------------------ host side
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_fn(EncodeTiled* out)
{
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) {
            set_error("cuTensorMapEncodeTiled is not available from the driver");
            return RG_CUDA_ERROR;
        }
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    *out = fn;
    return RG_OK;
}

// activation map: dims (C, W, H, Z) with box (16, bw, bh, bz), 32-byte swizzle
// box of 16 channels x (bw, bh, bz) positions, bw * bh * bz == positions
int make_act_map(CUtensorMap* map, const void* base, int C, int W, int H, int Z, int bw, int bh, int bz,
                 int positions)
{
    EncodeTiled enc;
    int rc = encode_fn(&enc);
    if (rc) return rc;
    RG_REQUIRE(C % 16 == 0 && bw * bh * bz == positions,
               "activation map: C must be a multiple of 16 and the box must hold the kernel's positions");
    RG_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, "activation map: base must be 16-byte aligned");
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Z};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {16, (cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)bz};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (activations) failed with code " + std::to_string((int)r));
        return RG_CUDA_ERROR;
    }
    return RG_OK;
}

// activation map with the box-reuse kernel's input box (16, 8, 18, 4), 32-byte swizzle
int make_box_map(CUtensorMap* map, const void* base, int C, int W, int H, int Z)
{
    EncodeTiled enc;
    int rc = encode_fn(&enc);
    if (rc) return rc;
    RG_REQUIRE(C % 16 == 0, "activation map: C must be a multiple of 16");
    RG_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, "activation map: base must be 16-byte aligned");
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)Z};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {16, (cuuint32_t)kBoxW, (cuuint32_t)(kBoxH + 2), (cuuint32_t)(kBoxZ + 2)};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (activation box) failed with code " + std::to_string((int)r));
        return RG_CUDA_ERROR;
    }
    return RG_OK;
}

// weight map: [rows][K] bf16 (K contiguous), box (16, box_rows), 32-byte swizzle
int make_weight_map(CUtensorMap* map, const void* base, int K, int rows, int box_rows)
{
    EncodeTiled enc;
    int rc = encode_fn(&enc);
    if (rc) return rc;
    RG_REQUIRE(K % 16 == 0 && box_rows <= 256, "weight map: K must be a multiple of 16");
    RG_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, "weight map: base must be 16-byte aligned");
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    cuuint32_t box[2] = {16, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (weights) failed with code " + std::to_string((int)r));
        return RG_CUDA_ERROR;
    }
    return RG_OK;
}

// 128-position box for a W x H slice grid
void tile_box(int W, int H, int D, int* bw, int* bh, int* bz)
{
    *bw = W >= 128 ? 128 : W;
    *bh = 128 / *bw;
    if (*bh > H) *bh = H;
    *bz = 128 / (*bw * *bh);
    (void)D;
}

template <int COUT>
int launch_conv3(ConvArgs& a, int ntiles)
{
    static bool attr = false;
    if (!attr) {
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_conv3<COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           ConvSmem<COUT>::kBytes));
        attr = true;
    }
    RG_TIMED(T_WS_CONV, (k_conv3<COUT><<<ntiles, kConvThreads, ConvSmem<COUT>::kBytes, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

template <int COUT, int S>
int launch_conv3_box(ConvArgs& a, int ntiles)
{
    static bool attr = false;
    if (!attr) {
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_conv3_box<COUT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           BoxSmem<COUT, S>::kBytes));
        attr = true;
    }
    RG_TIMED(T_WS_CONV, (k_conv3_box<COUT, S><<<ntiles, kConvThreads, BoxSmem<COUT, S>::kBytes, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

template <int COUT>
int launch_conv3_box_any(ConvArgs& a, int ntiles)
{
    // one stage when there is one chunk (several CTAs per SM overlap instead), else two
    return a.Cin == 16 ? launch_conv3_box<COUT, 1>(a, ntiles) : launch_conv3_box<COUT, 2>(a, ntiles);
}

int set_conv_wait_control(int polls, int withhold)
{
    const ConvWaitCtl c = {polls, withhold ? 1 : 0};
    RG_CHECK_CUDA(cudaDeviceSynchronize());  // no convolution may be running while it changes
    RG_CHECK_CUDA(cudaMemcpyToSymbol(g_conv_wait, &c, sizeof(c)));
    return RG_OK;
}

// stages of the persistent kernel's input-box ring
constexpr int kBoxPStages = 2;

// whether the persistent kernel's shared memory (all weights resident) fits one CTA
bool boxp_fits(int cout, int cin)
{
    const int chunks = cin / 16;
    int b = 0;
    switch (cout) {
    case 16: b = BoxPSmem<16>::bytes(chunks, kBoxPStages); break;
    case 32: b = BoxPSmem<32>::bytes(chunks, kBoxPStages); break;
    case 48: b = BoxPSmem<48>::bytes(chunks, kBoxPStages); break;
    case 64: b = BoxPSmem<64>::bytes(chunks, kBoxPStages); break;
    default: return false;
    }
    return b <= 227 * 1024;
}

template <int COUT>
int launch_conv3_boxp(ConvArgs& a, int ntiles)
{
    constexpr int S = kBoxPStages;
    const int bytes = BoxPSmem<COUT>::bytes(a.Cin / 16, S);
    // host-side setup once per shared-memory size (the launches of a network come back to back)
    static int attr = 0, last_bytes = -1, slots = 0;
    if (bytes > attr) {
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_conv3_boxp<COUT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr = bytes;
    }
    if (bytes != last_bytes) {
        int per_sm = 0, dev = 0, sms = 0;
        RG_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3_boxp<COUT, S>, kConvThreads, bytes));
        RG_CHECK_CUDA(cudaGetDevice(&dev));
        RG_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        slots = std::max(per_sm, 1) * sms;
        last_bytes = bytes;
    }
    const int grid = std::min(ntiles, slots);
    RG_TIMED(T_WS_CONV, (k_conv3_boxp<COUT, S><<<grid, kConvThreads, bytes, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

template <int COUT>
int launch_wgrad(WgradArgs& a, int grid)
{
    static bool attr = false;
    if (!attr) {
        RG_CHECK_CUDA(cudaFuncSetAttribute(k_wgrad<COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           WgSmem<COUT>::kBytes));
        attr = true;
    }
    RG_TIMED(T_WS_WGRAD, (k_wgrad<COUT><<<grid, kConvThreads, WgSmem<COUT>::kBytes, stream()>>>(a)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}

// 64-position box for the weight gradient's K slices
void wg_box(int W, int H, int* bw, int* bh, int* bz)
{
    *bw = W >= 64 ? 64 : W;
    *bh = 64 / *bw;
    if (*bh > H) *bh = H;
    *bz = 64 / (*bw * *bh);
}

}  // namespace ws
}  // namespace rg

using namespace rg;

extern "C" int rg_ws_conv3(const rg_act* x, const void* weights, const float* bias, rg_act* y, int relu,
                           const rg_act* mask, int* err_dev)
{
    RG_REQUIRE(x && weights && y && err_dev, "rg_ws_conv3: NULL argument");
    RG_REQUIRE(x->n == y->n && x->d == y->d && x->h == y->h && x->w == y->w, "rg_ws_conv3: x and y shapes differ");
    RG_REQUIRE(x->c % 16 == 0 && x->c <= 256, "rg_ws_conv3: input channels must be a multiple of 16");
    const int cout = y->c;
    RG_REQUIRE(cout == 16 || cout == 32 || cout == 48 || cout == 64 || cout == 80 || cout == 112 || cout == 128,
               "rg_ws_conv3: output channels must be 16, 32, 48, 64, 80, 112 or 128");
    RG_REQUIRE(!mask || (mask->c == cout && mask->n == y->n && mask->d == y->d && mask->h == y->h && mask->w == y->w),
               "rg_ws_conv3: mask shape must equal the output shape");
    ws::ConvArgs a;
    const int Z = x->n * (x->d + 2);
    if (x->w % ws::kBoxW == 0 && x->h % ws::kBoxH == 0 && x->d % ws::kBoxZ == 0 && cout <= 64) {
        // box-reuse kernel: 8 x 16 x 2 output tiles, the input box loaded once per kw and chunk
        int rc = ws::make_box_map(&a.xmap, x->ptr, x->c, x->w, x->h, Z);
        if (rc) return rc;
        rc = ws::make_weight_map(&a.wmap, weights, x->c, 27 * cout, cout);
        if (rc) return rc;
        a.bias = bias;
        a.out = static_cast<__nv_bfloat16*>(y->ptr);
        a.mask = mask ? static_cast<const __nv_bfloat16*>(mask->ptr) : nullptr;
        a.W = x->w;
        a.H = x->h;
        a.D = x->d;
        a.Cin = x->c;
        a.BW = ws::kBoxW;
        a.BH = ws::kBoxH;
        a.BZ = ws::kBoxZ;
        a.tiles_w = x->w / ws::kBoxW;
        a.tiles_h = x->h / ws::kBoxH;
        a.tiles_z = x->n * x->d / ws::kBoxZ;
        a.relu = relu;
        a.err = err_dev;
        const int ntiles = a.tiles_w * a.tiles_h * a.tiles_z;
        if (ws::boxp_fits(cout, x->c)) {
            // persistent: weights resident, box loads, UMMAs and epilogues of consecutive tiles overlap
            switch (cout) {
            case 16: return ws::launch_conv3_boxp<16>(a, ntiles);
            case 32: return ws::launch_conv3_boxp<32>(a, ntiles);
            case 48: return ws::launch_conv3_boxp<48>(a, ntiles);
            default: return ws::launch_conv3_boxp<64>(a, ntiles);
            }
        }
        switch (cout) {
        case 16: return ws::launch_conv3_box_any<16>(a, ntiles);
        case 32: return ws::launch_conv3_box_any<32>(a, ntiles);
        case 48: return ws::launch_conv3_box_any<48>(a, ntiles);
        default: return ws::launch_conv3_box_any<64>(a, ntiles);
        }
    }
    int bw, bh, bz;
    ws::tile_box(x->w, x->h, x->d, &bw, &bh, &bz);
    RG_REQUIRE(x->w % bw == 0 && x->h % bh == 0 && x->d % bz == 0 && bw * bh * bz == 128,
               "rg_ws_conv3: spatial sizes must tile into 128-position boxes");
    int rc = ws::make_act_map(&a.xmap, x->ptr, x->c, x->w, x->h, Z, bw, bh, bz, 128);
    if (rc) return rc;
    rc = ws::make_weight_map(&a.wmap, weights, x->c, 27 * cout, cout);
    if (rc) return rc;
    a.bias = bias;
    a.out = static_cast<__nv_bfloat16*>(y->ptr);
    a.mask = mask ? static_cast<const __nv_bfloat16*>(mask->ptr) : nullptr;
    a.W = x->w;
    a.H = x->h;
    a.D = x->d;
    a.Cin = x->c;
    a.BW = bw;
    a.BH = bh;
    a.BZ = bz;
    a.tiles_w = x->w / bw;
    a.tiles_h = x->h / bh;
    a.tiles_z = x->n * x->d / bz;
    a.relu = relu;
    a.err = err_dev;
    const int ntiles = a.tiles_w * a.tiles_h * a.tiles_z;
    switch (cout) {
    case 16: return ws::launch_conv3<16>(a, ntiles);
    case 32: return ws::launch_conv3<32>(a, ntiles);
    case 48: return ws::launch_conv3<48>(a, ntiles);
    case 64: return ws::launch_conv3<64>(a, ntiles);
    case 80: return ws::launch_conv3<80>(a, ntiles);
    case 112: return ws::launch_conv3<112>(a, ntiles);
    default: return ws::launch_conv3<128>(a, ntiles);
    }
}

extern "C" int rg_ws_conv3_wgrad(const rg_act* x, const rg_act* g, float* dw, float* partials,
                                 int64_t partials_floats, int accumulate, int* err_dev)
{
    RG_REQUIRE(x && g && dw && partials && err_dev, "rg_ws_conv3_wgrad: NULL argument");
    RG_REQUIRE(x->n == g->n && x->d == g->d && x->h == g->h && x->w == g->w, "rg_ws_conv3_wgrad: x and g shapes differ");
    RG_REQUIRE(x->c % 16 == 0 && x->c <= 256, "rg_ws_conv3_wgrad: input channels must be a multiple of 16");
    const int cout = g->c;
    RG_REQUIRE(cout == 16 || cout == 32 || cout == 48 || cout == 64 || cout == 80 || cout == 112 || cout == 128,
               "rg_ws_conv3_wgrad: gradient channels must be 16, 32, 48, 64, 80, 112 or 128");
    int bw, bh, bz;
    ws::wg_box(x->w, x->h, &bw, &bh, &bz);
    RG_REQUIRE(x->w % bw == 0 && x->h % bh == 0 && x->d % bz == 0 && bw * bh * bz == ws::kWgKP,
               "rg_ws_conv3_wgrad: spatial sizes must tile into 64-position boxes");
    ws::WgradArgs a;
    const int Z = x->n * (x->d + 2);
    int rc = ws::make_act_map(&a.xmap, x->ptr, x->c, x->w, x->h, Z, bw, bh, bz, ws::kWgKP);
    if (rc) return rc;
    rc = ws::make_act_map(&a.gmap, g->ptr, cout, g->w, g->h, Z, bw, bh, bz, ws::kWgKP);
    if (rc) return rc;
    a.W = x->w;
    a.H = x->h;
    a.D = x->d;
    a.Cin = x->c;
    a.npairs = 27 * (x->c / 16);
    a.BW = bw;
    a.BH = bh;
    a.BZ = bz;
    a.tiles_w = x->w / bw;
    a.tiles_h = x->h / bh;
    a.tiles_z = x->n * x->d / bz;
    a.ptiles = a.tiles_w * a.tiles_h * a.tiles_z;
    a.mtiles = (a.npairs + 7) / 8;
    // about four CTAs per SM in total
    int ksplit = (4 * kNumSMs + a.mtiles - 1) / a.mtiles;
    if (ksplit > a.ptiles) ksplit = a.ptiles;
    const int64_t need = (int64_t)ksplit * a.mtiles * 128 * cout;
    if (need > partials_floats) {
        ksplit = (int)(partials_floats / ((int64_t)a.mtiles * 128 * cout));
        RG_REQUIRE(ksplit >= 1, "rg_ws_conv3_wgrad: partials buffer too small");
    }
    a.ksplit = ksplit;
    a.partials = partials;
    a.err = err_dev;
    const int grid = a.mtiles * ksplit;
    switch (cout) {
    case 16: rc = ws::launch_wgrad<16>(a, grid); break;
    case 32: rc = ws::launch_wgrad<32>(a, grid); break;
    case 48: rc = ws::launch_wgrad<48>(a, grid); break;
    case 64: rc = ws::launch_wgrad<64>(a, grid); break;
    case 80: rc = ws::launch_wgrad<80>(a, grid); break;
    case 112: rc = ws::launch_wgrad<112>(a, grid); break;
    default: rc = ws::launch_wgrad<128>(a, grid); break;
    }
    if (rc) return rc;
    const int total = 27 * cout * x->c;
    RG_TIMED(T_WS_WGRAD, (ws::k_wgrad_reduce<<<(total + 255) / 256, 256, 0, stream()>>>(partials, dw, ksplit, a.mtiles, cout, x->c,
                                                                 accumulate)));
    RG_CHECK_LAUNCH();
    return RG_OK;
}
