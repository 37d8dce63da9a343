// Fused inference of one surrogate network on sm_100a: every layer of a
// 128-row tile of queries in one persistent kernel, activations kept on
// the SM between layers.
//
//   H_0 = X (128 x 64 bf16), H_l = relu(H_{l-1} W_l^T + b_l) (128 x 512),
//   Y = (H_{L-2} W_{L-1}^T + b_{L-1}) * sd + mean (the nout real columns, FP32)
//
// Shared memory holds the tile's activations as eight K-major 128 x 64
// bf16 blocks in the 128-byte swizzle layout (the A operand of the next
// layer's MMAs, 128 KB) and a 3-stage ring of 256 x 64 weight tiles (the B
// operand, 32 KB each). Tensor memory holds one layer's 128 x 512 FP32
// accumulator (all 512 columns, as two N = 256 halves). 18 warps:
//   - warp 0, one lane: TMA producer -- the X tile into activation block 0
//     once the previous tile's last MMAs have read the activations, and the
//     weight tiles of every layer, half and K block in order;
//   - warp 1, one lane: MMA issuer -- per layer and half, tcgen05.mma
//     (M 128, N 256, K 16) over the layer's K blocks, then tcgen05.commit
//     to the epilogue. A half starts once the previous layer's epilogue has
//     read that half of tensor memory, and each K block once its
//     activation block is written, so the next layer's first half runs
//     under the second half of the previous epilogue;
//   - warps 2..17: epilogue -- four warps per tensor-memory lane quarter
//     (with two, the next layer's MMAs waited on the epilogue: 4 % slower);
//     a thread owns one tile row. Hidden layers: the four warps of a quarter
//     take every fourth 64-column block in K order (bias + ReLU, bf16,
//     written straight into the activation block in the swizzled layout)
//     and signal each finished block and each tensor-memory half read.
//     Last layer: bias and the output denormalisation (y = v * sd + mean)
//     into the caller's FP32 rows.
// The weights (about 1.9 MB per network) stream from L2 for every tile; no
// activation leaves the SM. Every mbarrier wait is bounded; a wait that
// runs out sets bit 0 of *status and the kernel finishes without hanging.
// Operand loads use only this GPU's own memory and no multicast.
#pragma once

#include "mlp_tc.cuh"

namespace fdtd {
namespace mlp {

constexpr int kFusedWidth = 512;                              // hidden width: 8 K blocks
constexpr int kFusedHalf = 256;                               // MMA N, tensor-memory columns per half
constexpr int kFusedStages = 3;
constexpr int kFusedMaxLayers = 8;
constexpr int kFusedBlockBytes = kTileM * kTileK * 2;         // one 128 x 64 activation block: 16 KB
constexpr int kFusedHBytes = kFusedWidth / kTileK * kFusedBlockBytes;  // 128 KB
constexpr int kFusedBBytes = kFusedHalf * kTileK * 2;         // one 256 x 64 weight tile: 32 KB
constexpr int kFusedEpiWarps = 16;                            // four per tensor-memory lane quarter
constexpr int kFusedThreads = 64 + 32 * kFusedEpiWarps;        // warp 0 TMA, warp 1 MMA, the rest epilogue
constexpr int kEpiPar = kFusedEpiWarps / 4;                    // epilogue warps sharing a lane quarter

struct FusedMaps {
    CUtensorMap x;                     // bf16 [M][64], boxes 64 x 128
    CUtensorMap w[kFusedMaxLayers];    // bf16 [N_l][K_l], boxes 64 x 256
};

struct FusedArgs {
    int M;                             // rows, a multiple of 128
    int L;                             // layers
    int nkb[kFusedMaxLayers];          // K blocks of layer l (1 for the input layer, 8 after)
    int nhalf[kFusedMaxLayers];        // N halves of layer l (2 hidden, 1 for the 256-wide output)
    const float* bias[kFusedMaxLayers];
    int valid;                         // rows of the caller's output (the rest are padding)
    int nout;                          // output columns written
    const float* omean;                // [nout] output denormalisation: y = v * osd + omean
    const float* osd;
    float* y;                          // [valid][nout] FP32, the caller's buffer
    int* status;                       // bit 0: a wait ran out
};

constexpr size_t fused_smem_bytes() { return 1024 + kFusedHBytes + kFusedStages * kFusedBBytes + 256; }

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 lanes x 32 bits, 32 consecutive columns (one wait for 32 columns)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

__global__ void __launch_bounds__(kFusedThreads, 1) k_mlp_fused(const __grid_constant__ FusedMaps maps, const FusedArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* sH = smem;
    unsigned char* sB = smem + kFusedHBytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kFusedStages * kFusedBBytes);
    uint64_t* empty = full + kFusedStages;
    uint64_t* xfull = empty + kFusedStages;  // the tile's X landed in block 0
    uint64_t* hfree = xfull + 1;             // the tile's last MMAs have read the activations
    uint64_t* accf = hfree + 1;              // a layer's MMAs are complete
    uint64_t* hblk = accf + 1;               // [8] activation block written (one warp per lane quarter)
    uint64_t* tfree = hblk + 8;              // [2] tensor-memory half read by the epilogue (every epilogue warp)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tfree + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = g.M / kTileM;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(2 * kFusedHalf)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kFusedStages; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        bar_init(xfull, 1);
        bar_init(hfree, 1);
        bar_init(accf, 1);
        for (int b = 0; b < 8; ++b) bar_init(&hblk[b], 4);  // one warp of each lane quarter
        bar_init(&tfree[0], kFusedEpiWarps);
        bar_init(&tfree[1], kFusedEpiWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int kbg = 0, it = 0;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
                if (it >= 1 && !(ok = bar_wait(hfree, (it - 1) & 1))) break;
                bar_expect_tx(xfull, kFusedBlockBytes);
                tma_load_2d(sH, &maps.x, 0, t * kTileM, xfull);
                for (int l = 0; l < g.L && ok; ++l)
                    for (int h = 0; h < g.nhalf[l] && ok; ++h)
                        for (int kb = 0; kb < g.nkb[l]; ++kb, ++kbg) {
                            const int s = kbg % kFusedStages;
                            if (kbg >= kFusedStages && !(ok = bar_wait(&empty[s], ((kbg / kFusedStages) - 1) & 1)))
                                break;
                            bar_expect_tx(&full[s], kFusedBBytes);
                            tma_load_2d(sB + s * kFusedBBytes, &maps.w[l], kb * kTileK, h * kFusedHalf, &full[s]);
                        }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = idesc_bf16<kFusedHalf>();
            int kbg = 0, it = 0, seq = 0;  // seq: layers issued so far (all tiles)
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
                if (!(ok = bar_wait(xfull, it & 1))) break;
                for (int l = 0; l < g.L && ok; ++l, ++seq) {
                    const int hseq = it * (g.L - 1) + (l - 1);  // the hidden epilogue that wrote this layer's input
                    for (int h = 0; h < g.nhalf[l] && ok; ++h) {
                        // the previous layer's epilogue has read this tensor-memory half
                        if (seq >= 1 && !(ok = bar_wait(&tfree[h], (seq - 1) & 1))) break;
                        tc_fence_after();
                        for (int kb = 0; kb < g.nkb[l]; ++kb, ++kbg) {
                            // the activation block this K step reads is written
                            if (l >= 1 && h == 0 && !(ok = bar_wait(&hblk[kb], hseq & 1))) break;
                            const int s = kbg % kFusedStages;
                            if (!(ok = bar_wait(&full[s], (kbg / kFusedStages) & 1))) break;
                            tc_fence_after();
                            const uint64_t da = sw128_desc(su32(sH + kb * kFusedBlockBytes));
                            const uint64_t db = sw128_desc(su32(sB + s * kFusedBBytes));
#pragma unroll
                            for (int kk = 0; kk < kTileK / 16; ++kk)
                                mma_bf16(tmem + h * kFusedHalf, da + 2 * kk, db + 2 * kk, idesc, (kb | kk) != 0);
                            mma_commit(&empty[s]);
                        }
                    }
                    if (!ok) break;
                    mma_commit(accf);
                    if (l == g.L - 1) mma_commit(hfree);
                }
            }
        }
    } else {  // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31; parity (w - 2) / 4
        const int quarter = warp & 3, par = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        const uint32_t ta = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
        auto arrive = [&](uint64_t* b) {
            __syncwarp();
            if (lane == 0) bar_arrive(b);
        };
        constexpr int bph = kFusedHalf / kTileK;  // activation blocks per tensor-memory half
        int seq = 0;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            for (int l = 0; l < g.L; ++l, ++seq) {
                if (!__all_sync(0xffffffffu, bar_wait(accf, seq & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const float* bias = g.bias[l];
                if (l < g.L - 1) {
                    // blocks par, par + kEpiPar, ...: 64 columns, row `row` = 128 bytes,
                    // 16-byte chunks swizzled by row % 8
                    const int nb = g.nhalf[l] * kFusedHalf / kTileK, sw = row & 7;
                    for (int kb = par; kb < nb; kb += kEpiPar) {
                        unsigned char* blk = sH + kb * kFusedBlockBytes + row * 128;
#pragma unroll 1
                        for (int c = kb * kTileK; c < (kb + 1) * kTileK; c += 32) {
                            float v[32];
                            tmem_ld32(ta + c, v);
                            uint32_t pk[16];
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const float4 b = ldg4(bias + c + 4 * q);
                                const __nv_bfloat162 lo = __floats2bfloat162_rn(fmaxf(v[4 * q] + b.x, 0.0f),
                                                                                fmaxf(v[4 * q + 1] + b.y, 0.0f));
                                const __nv_bfloat162 hi = __floats2bfloat162_rn(fmaxf(v[4 * q + 2] + b.z, 0.0f),
                                                                                fmaxf(v[4 * q + 3] + b.w, 0.0f));
                                pk[2 * q] = *reinterpret_cast<const uint32_t*>(&lo);
                                pk[2 * q + 1] = *reinterpret_cast<const uint32_t*>(&hi);
                            }
                            const int ch = (c % kTileK) / 8;  // 32 columns = 4 chunks of 16 bytes
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                                *reinterpret_cast<uint4*>(blk + (((ch + q) ^ sw) << 4)) =
                                    make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
                        }
                        fence_async_shared();  // the generic-proxy writes become visible to the MMAs
                        tc_fence_before();
                        arrive(&hblk[kb]);
                        // this warp's last block in a tensor-memory half: that half is read
                        if (kb + kEpiPar >= nb || (kb / bph) != ((kb + kEpiPar) / bph)) arrive(&tfree[kb / bph]);
                    }
                    if (nb <= bph) arrive(&tfree[1]);  // a 256-wide layer leaves half 1 untouched
                } else {
                    const int N = g.nhalf[l] * kFusedHalf, c0 = par * (N / kEpiPar), c1 = c0 + N / kEpiPar;
                    const int m = t * kTileM + row;
                    float* o = g.y + static_cast<size_t>(m) * g.nout;
                    const int ce = min(c1, g.nout);
#pragma unroll 1
                    for (int c = c0; c < c1; c += 32) {
                        float v[32];
                        tmem_ld32(ta + c, v);  // every lane takes part in the collective load
                        if (m < g.valid) {
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (c + j < ce) o[c + j] = (v[j] + bias[c + j]) * g.osd[c + j] + g.omean[c + j];
                        }
                    }
                    tc_fence_before();
                    arrive(&tfree[0]);
                    arrive(&tfree[1]);
                }
            }
        }
    }
    if (!ok && lane == 0) atomicOr(g.status, 1);
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kFusedHalf)
                     : "memory");
}

}  // namespace mlp
}  // namespace fdtd
