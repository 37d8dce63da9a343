// Tensor-core GEMM for the surrogate network on sm_100a (5th-generation
// tensor cores, tcgen05):
//
//   D[M, N] = A[M, K] . B[N, K]^T      A, B bf16, row-major (K contiguous),
//                                      D accumulated in FP32 in tensor memory
//
// followed by a fused epilogue (bias, ReLU, ReLU-gradient mask, bf16 or FP32
// stores, optionally also the transposed bf16 result that the backward pass
// reads as its next operand).
//
// A persistent CTA of 192 threads per SM walks 128 x BN output tiles:
//   - warp 0, one lane: TMA producer. Each K block of 64 elements of A
//     (128 rows) and B (BN rows) lands in a shared-memory stage (a 4-stage
//     ring) through cp.async.bulk.tensor with the 128-byte swizzle,
//     completing on the stage's "full" mbarrier;
//   - warp 1, one lane: MMA issuer. Four tcgen05.mma (K = 16 each) per stage
//     read both operands from shared memory through matrix descriptors and
//     accumulate into one of two 128 x BN FP32 tiles in tensor memory;
//     tcgen05.commit frees the stage ("empty") once they complete and hands
//     the finished accumulator to the epilogue;
//   - warps 2..5: epilogue. Each reads its quarter of the accumulator rows
//     with tcgen05.ld, stores, and hands the accumulator back, while the MMA
//     warp already fills the other one.
// Tensor memory (2 BN columns) is allocated and released by warp 1. Every
// mbarrier wait is bounded; a wait that runs out sets bit 0 of *status and
// the kernel finishes without hanging.
//
// Operand loads use only this GPU's own memory and no multicast.
#pragma once

#include <cstdint>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace fdtd {
namespace mlp {

constexpr int kTileM = 128;  // rows per CTA (one tcgen05.mma M)
constexpr int kTileK = 64;   // K elements per stage: 128 bytes of bf16, one swizzle atom row
constexpr int kStages = 4;
constexpr int kGemmThreads = 192;  // warp 0 TMA, warp 1 MMA, warps 2..5 epilogue
constexpr long long kSpin = 1LL << 24;

enum Epilogue : int {
    kEpiF32 = 0,         // out_f32[m][n] = acc
    kEpiBiasReluT = 1,   // h = relu(acc + bias[n]) -> out_bf16[m][n] and outT_bf16[n][m]
    kEpiBiasF32 = 2,     // out_f32[m][n] = acc + bias[n]
    kEpiReluGradT = 3,   // g = acc * (mask_bf16[m][n] > 0) -> out_bf16[m][n] and outT_bf16[n][m]
    kEpiBiasRelu = 4,    // h = relu(acc + bias[n]) -> out_bf16[m][n]
};

struct GemmArgs {
    int M, N, K;
    const float* bias;             // [N] (bias epilogues)
    const __nv_bfloat16* mask;     // [M][ldm] (ReLU-gradient epilogue)
    int ldm;
    void* out;                     // [M][ldo] bf16 or FP32
    int ldo;
    __nv_bfloat16* outT;           // [N][ldt] (transposing epilogues)
    int ldt;
    int* status;                   // bit 0: a wait ran out
};

// shared memory: stages of A (128 x 64 bf16 = 16 KB) and B (BN x 64 bf16),
// 1024-byte aligned for the 128-byte swizzle, then the mbarriers (stage
// full / empty, accumulator full / empty) and the tensor-memory address slot
template <int BN>
constexpr size_t gemm_smem_bytes() {
    return 1024 + kStages * (kTileM * kTileK * 2 + BN * kTileK * 2) + 256;
}

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false when it ran out
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
    for (long long i = 0; i < kSpin; ++i)
        if (bar_try(b, parity)) return true;
    return false;
}

// 2D tiled TMA load: box (x = K offset, y = row offset) of the tensor map
// into shared memory, completing on mbarrier b
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(b))
        : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile in the 128-byte
// swizzle layout: rows of 128 bytes, 8-row groups 1024 bytes apart (stride
// byte offset), leading byte offset 16 (unused by this layout), descriptor
// version 1, base offset 0 (1024-byte aligned tiles), layout 2 = 128-byte
// swizzle. The K = 16 sub-blocks of one 64-wide stage start 32 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr & 0x3FFFF) >> 4);     // start address
    d |= static_cast<uint64_t>(16 >> 4) << 16;              // leading byte offset
    d |= static_cast<uint64_t>(1024 >> 4) << 32;            // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;                    // version
    d |= static_cast<uint64_t>(2) << 61;                    // 128-byte swizzle
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, bf16 A and B, both
// K-major, M = 128, N = BN
template <int BN>
__device__ __forceinline__ constexpr uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(BN >> 3) << 17) |
           (static_cast<uint32_t>(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 bits, 16 consecutive columns: thread t of the warp gets lane
// (warp's lane base + t), columns col .. col+15
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Epilogue of one accumulator tile row: this thread's row m of the tile
// starting at column n0, read from tensor memory at taddr (the warp's lane
// quarter, the tile's first column).
template <int BN, int EPI>
__device__ __forceinline__ void epilogue_row(const GemmArgs& g, uint32_t taddr, int m, int n0) {
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
        float v[16];
        tmem_ld16(taddr + c, v);
        const int n = n0 + c;
        if constexpr (EPI == kEpiF32 || EPI == kEpiBiasF32) {
            if constexpr (EPI == kEpiBiasF32) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += g.bias[n + j];
            }
            float4* o = reinterpret_cast<float4*>(static_cast<float*>(g.out) + static_cast<size_t>(m) * g.ldo + n);
#pragma unroll
            for (int j = 0; j < 4; ++j) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else {
            if constexpr (EPI == kEpiBiasReluT || EPI == kEpiBiasRelu) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + g.bias[n + j], 0.0f);
            } else {  // ReLU gradient: pass where the forward activation was positive
                const uint4* mk = reinterpret_cast<const uint4*>(g.mask + static_cast<size_t>(m) * g.ldm + n);
                const uint4 q0 = mk[0], q1 = mk[1];
                const __nv_bfloat16* h0 = reinterpret_cast<const __nv_bfloat16*>(&q0);
                const __nv_bfloat16* h1 = reinterpret_cast<const __nv_bfloat16*>(&q1);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (!(__bfloat162float(h0[j]) > 0.0f)) v[j] = 0.0f;
                    if (!(__bfloat162float(h1[j]) > 0.0f)) v[8 + j] = 0.0f;
                }
            }
            __nv_bfloat16 b[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) b[j] = __float2bfloat16_rn(v[j]);
            uint4* o = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(g.out) + static_cast<size_t>(m) * g.ldo + n);
            o[0] = *reinterpret_cast<const uint4*>(&b[0]);
            o[1] = *reinterpret_cast<const uint4*>(&b[8]);
            if constexpr (EPI == kEpiBiasReluT || EPI == kEpiReluGradT) {
#pragma unroll
                for (int j = 0; j < 16; ++j) g.outT[static_cast<size_t>(n + j) * g.ldt + m] = b[j];
            }
        }
    }
}

__device__ __forceinline__ void bar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}

// Persistent GEMM: CTA b computes tiles b, b + gridDim.x, ... (tile t =
// row block t / (N / BN), column block t % (N / BN), so the column blocks of
// one row block run together and share that block of A in L2). Six warps:
// warp 0 (one lane) loads stages with TMA, warp 1 (one lane) issues the
// MMAs, warps 2..5 run the epilogue. Two accumulators in tensor memory
// (2 BN columns) let the epilogue of one tile overlap the MMAs of the next:
// "tfull[a]" (MMA commit) hands accumulator a to the epilogue warps,
// "tempty[a]" (one arrival per epilogue warp) hands it back.
template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_tn(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, const GemmArgs g) {
    static_assert(BN == 64 || BN == 128, "tile width");  // 128 x 256 tiles measured slower
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    constexpr int kABytes = kTileM * kTileK * 2, kBBytes = BN * kTileK * 2;
    unsigned char* sA = smem;
    unsigned char* sB = smem + kStages * kABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kStages * kBBytes);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntn = g.N / BN, ntiles = (g.M / kTileM) * ntn, nk = g.K / kTileK;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(2 * BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            bar_init(&tfull[a], 1);
            bar_init(&tempty[a], 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int kbg = 0;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const int m0 = (t / ntn) * kTileM, n0 = (t % ntn) * BN;
                for (int kb = 0; kb < nk; ++kb, ++kbg) {
                    const int s = kbg % kStages;
                    if (kbg >= kStages && !(ok = bar_wait(&empty[s], ((kbg / kStages) - 1) & 1))) break;
                    bar_expect_tx(&full[s], kABytes + kBBytes);
                    tma_load_2d(sA + s * kABytes, &mapA, kb * kTileK, m0, &full[s]);
                    tma_load_2d(sB + s * kBBytes, &mapB, kb * kTileK, n0, &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = idesc_bf16<BN>();
            int kbg = 0, it = 0;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
                const int a = it & 1;
                if (it >= 2 && !(ok = bar_wait(&tempty[a], ((it >> 1) - 1) & 1))) break;
                tc_fence_after();
                const uint32_t d = tmem + a * BN;
                for (int kb = 0; kb < nk; ++kb, ++kbg) {
                    const int s = kbg % kStages;
                    if (!(ok = bar_wait(&full[s], (kbg / kStages) & 1))) break;
                    tc_fence_after();
                    const uint64_t da = sw128_desc(su32(sA + s * kABytes)), db = sw128_desc(su32(sB + s * kBBytes));
#pragma unroll
                    for (int kk = 0; kk < kTileK / 16; ++kk)  // +32 bytes per K = 16 step: +2 in the address field
                        mma_bf16(d, da + 2 * kk, db + 2 * kk, idesc, (kb | kk) != 0);
                    mma_commit(&empty[s]);
                }
                if (!ok) break;
                mma_commit(&tfull[a]);
            }
        }
    } else {  // epilogue warps: warp w reads tensor-memory lanes 32 (w % 4) .. + 31
        const int quarter = warp & 3;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
            const int a = it & 1;
            const bool w = __all_sync(0xffffffffu, bar_wait(&tfull[a], (it >> 1) & 1));
            if (!w) {
                ok = false;
                break;
            }
            tc_fence_after();
            const int m = (t / ntn) * kTileM + quarter * 32 + lane, n0 = (t % ntn) * BN;
            epilogue_row<BN, EPI>(g, tmem + a * BN + (static_cast<uint32_t>(quarter * 32) << 16), m, n0);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&tempty[a]);
        }
    }
    if (!ok && lane == 0) atomicOr(g.status, 1);
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN) : "memory");
}

}  // namespace mlp
}  // namespace fdtd
