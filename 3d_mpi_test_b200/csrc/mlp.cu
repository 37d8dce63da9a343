// Surrogate network on the device: tensor-core GEMMs (mlp_tc.cuh) plus the
// small kernels around them (input packing and normalisation, loss gradient,
// bias gradients, Adam, bf16 weight copies), forward, backward and training
// loop, and batched inference.
//
// Layout: every activation is kept as bf16 [rows][features] and, where the
// backward pass needs it as a GEMM operand with the batch as the reduction
// axis, also as its transpose [features][rows]; the transposed copy is
// written by the producing GEMM's epilogue. Weights: FP32 masters
// [N][K] (zero padding to the tile sizes), bf16 copies W [N][K] and
// W^T [K][N] refreshed after every update.
//
// A training step is captured once as a CUDA graph: the step counter, the
// learning-rate schedule and the minibatch indices live in device memory.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "fdtd_solver.hpp"
#include "mlp.hpp"
#include "mlp_fused.cuh"
#include "mlp_tc.cuh"

namespace fdtd {
namespace mlp {
namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw SolverError{-3, std::string(what) + ": " + cudaGetErrorString(e)};
}
[[noreturn]] void bad(const std::string& m) { throw SolverError{-5, m}; }

int round_up(int x, int m) { return (x + m - 1) / m * m; }

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "driver entry point");
        if (q != cudaDriverEntryPointSuccess || !p) throw SolverError{-3, "cuTensorMapEncodeTiled is unavailable"};
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// bf16 [rows][cols] row-major as a TMA tensor map: boxes of 64 columns
// (128 bytes) x box_rows rows, 128-byte swizzle (the layout the MMA
// descriptors of k_gemm_tn expect)
CUtensorMap bf16_map(const void* base, int rows, int cols, int box_rows) {
    if (reinterpret_cast<uintptr_t>(base) % 16) bad("GEMM operand not 16-byte aligned");
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kTileK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                                 es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw SolverError{-3, "tensor map encoding failed"};
    return m;
}

// one GEMM with fixed operands, ready to launch (also inside a graph)
struct Plan {
    CUtensorMap a, b;
    GemmArgs g;  // g.M may be lowered (to a multiple of 128) before a launch
    int bn = 128, epi = 0;
};

template <int BN, int EPI>
void set_attr() {
    ck(cudaFuncSetAttribute(k_gemm_tn<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(gemm_smem_bytes<BN>())),
       "GEMM shared-memory attribute");
}

template <int BN>
void set_attrs() {
    set_attr<BN, kEpiF32>();
    set_attr<BN, kEpiBiasReluT>();
    set_attr<BN, kEpiBiasF32>();
    set_attr<BN, kEpiReluGradT>();
    set_attr<BN, kEpiBiasRelu>();
}

void validate(int epi, int M, int N, int K, const void* A, const void* B, const float* bias, const void* mask,
              const void* out, const void* outT) {
    if (M <= 0 || N <= 0 || K <= 0 || M % kTileM || N % 64 || K % kTileK)
        bad("GEMM sizes: M must be a multiple of 128, N and K of 64");
    if (epi < 0 || epi > 4) bad("unknown GEMM epilogue");
    if (!A || !B || !out) bad("null GEMM operand");
    if ((epi == kEpiBiasReluT || epi == kEpiBiasF32 || epi == kEpiBiasRelu) && !bias) bad("epilogue needs a bias");
    if (epi == kEpiReluGradT && !mask) bad("epilogue needs a mask");
    if ((epi == kEpiBiasReluT || epi == kEpiReluGradT) && !outT) bad("epilogue needs a transposed output");
}

Plan make_plan(int epi, int M, int N, int K, const void* A, const void* B, const float* bias, const void* mask,
               int ldm, void* out, int ldo, void* outT, int ldt, int* status) {
    validate(epi, M, N, K, A, B, bias, mask, out, outT);
    static bool attrs = false;
    if (!attrs) {
        set_attrs<64>();
        set_attrs<128>();
        attrs = true;
    }
    Plan p;
    p.bn = (N % 128 == 0) ? 128 : 64;
    p.epi = epi;
    p.a = bf16_map(A, M, K, kTileM);
    p.b = bf16_map(B, N, K, p.bn);
    p.g = GemmArgs{M, N, K, bias, static_cast<const __nv_bfloat16*>(mask), ldm, out, ldo,
                   static_cast<__nv_bfloat16*>(outT), ldt, status};
    return p;
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "SM count");
    }
    return n;
}

// persistent launch: one CTA per SM, at most one per tile
template <int BN>
void launch_bn(const Plan& p, cudaStream_t s) {
    const size_t smem = gemm_smem_bytes<BN>();
    const int tiles = (p.g.M / kTileM) * (p.g.N / BN);
    const dim3 grid(std::min(tiles, sm_count())), blk(kGemmThreads);
    switch (p.epi) {
        case kEpiF32: k_gemm_tn<BN, kEpiF32><<<grid, blk, smem, s>>>(p.a, p.b, p.g); break;
        case kEpiBiasReluT: k_gemm_tn<BN, kEpiBiasReluT><<<grid, blk, smem, s>>>(p.a, p.b, p.g); break;
        case kEpiBiasF32: k_gemm_tn<BN, kEpiBiasF32><<<grid, blk, smem, s>>>(p.a, p.b, p.g); break;
        case kEpiReluGradT: k_gemm_tn<BN, kEpiReluGradT><<<grid, blk, smem, s>>>(p.a, p.b, p.g); break;
        default: k_gemm_tn<BN, kEpiBiasRelu><<<grid, blk, smem, s>>>(p.a, p.b, p.g); break;
    }
    ck(cudaGetLastError(), "GEMM launch");
}

void launch(const Plan& p, cudaStream_t s) {
    if (p.bn == 128) launch_bn<128>(p, s);
    else launch_bn<64>(p, s);
}

// ------------------------------------------------------------ small kernels
// rows r < B of the minibatch (rows past `valid` are zero): normalised
// inputs as bf16 [B][K0] and [K0][B]; row source idx[row0 + r] (or
// row0 + r without idx); row0 = *step * B when `step` is given
__global__ void k_pack(const float* __restrict__ X, int nin, const int* __restrict__ idx, const int* __restrict__ step,
                       int row0, int valid, int B, const float* __restrict__ mean, const float* __restrict__ istd,
                       __nv_bfloat16* __restrict__ Xb, int K0, __nv_bfloat16* __restrict__ XbT) {
    const int r = blockIdx.x * blockDim.y + threadIdx.y;
    const int c = threadIdx.x;
    if (r >= B || c >= K0) return;
    const int base = step ? *step * B : row0;
    float v = 0.0f;
    if (c < nin && r < valid) {
        const int src = idx ? idx[base + r] : base + r;
        v = (X[static_cast<size_t>(src) * nin + c] - mean[c]) * istd[c];
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    Xb[static_cast<size_t>(r) * K0 + c] = b;
    if (XbT) XbT[static_cast<size_t>(c) * B + r] = b;
}

// loss gradient of the mean squared error over the nout real outputs:
// dY = 2 (Y - T) / (B nout) as bf16 [B][NO] and [NO][B]; the sum of squared
// errors / (B nout) is added to loss[*step]
__global__ void k_loss(const float* __restrict__ Y, int NO, const float* __restrict__ T, int nout,
                       const int* __restrict__ idx, const int* __restrict__ step, int B, __nv_bfloat16* __restrict__ dY,
                       __nv_bfloat16* __restrict__ dYT, float* __restrict__ loss) {
    const int r = blockIdx.x;
    const int base = step ? *step * B : 0;
    const int src = idx ? idx[base + r] : base + r;
    const float scale = 2.0f / (static_cast<float>(B) * nout);
    float sq = 0.0f;
    for (int c = threadIdx.x; c < NO; c += blockDim.x) {
        float g = 0.0f;
        if (c < nout) {
            const float d = Y[static_cast<size_t>(r) * NO + c] - T[static_cast<size_t>(src) * nout + c];
            sq += d * d;
            g = scale * d;
        }
        const __nv_bfloat16 b = __float2bfloat16_rn(g);
        dY[static_cast<size_t>(r) * NO + c] = b;
        dYT[static_cast<size_t>(c) * B + r] = b;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += part[w];
        atomicAdd(loss + (step ? *step : 0), s / (static_cast<float>(B) * nout));
    }
}

// db[n] = sum over the batch of dZ^T[n][:]
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dZT, int N, int B, float* __restrict__ db) {
    const int n = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (n >= N) return;
    float s = 0.0f;
    for (int b = lane; b < B; b += 32) s += __bfloat162float(dZT[static_cast<size_t>(n) * B + b]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) db[n] = s;
}

// Adam (Kingma & Ba 2015) with bias correction and decoupled weight decay
// wd (Loshchilov & Hutter 2019); step t = *step + 1 and the learning rate
// lr[*step] are read from device memory
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, const float* __restrict__ lr, const int* __restrict__ step, float wd) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    constexpr float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int t = *step + 1;
    const float c1 = 1.0f / (1.0f - powf(b1, static_cast<float>(t)));
    const float c2 = 1.0f / (1.0f - powf(b2, static_cast<float>(t)));
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr[*step] * ((mi * c1) / (sqrtf(vi * c2) + eps) + wd * w[i]);
}

// bf16 copies W [N][K] and W^T [K][N] of an FP32 master
__global__ void k_cast(const float* __restrict__ W, int N, int K, __nv_bfloat16* __restrict__ Wb,
                       __nv_bfloat16* __restrict__ WTb) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<size_t>(N) * K) return;
    const int n = static_cast<int>(i / K), k = static_cast<int>(i % K);
    const __nv_bfloat16 b = __float2bfloat16_rn(W[i]);
    Wb[i] = b;
    WTb[static_cast<size_t>(k) * N + n] = b;
}

__global__ void k_next_step(int* step) { *step += 1; }

// one thread per output element of F [n][np + 2 nrec] (RayFeatures in
// mlp.hpp); d2 - d1 is formed as 4 hs hr / (d1 + d2), free of cancellation
__global__ void k_ray_features(const float* __restrict__ P, long long n, int np, int chs, int chr, int crange,
                               int nrec, float* __restrict__ F) {
    const int nf = np + 2 * nrec;
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * nf) return;
    const long long r = t / nf;
    const int c = static_cast<int>(t - r * nf);
    const float* p = P + r * np;
    float v;
    if (c < np) {
        v = p[c];
    } else {
        const int k = (c - np) % nrec;
        const float hs = p[chs], hr = p[chr];
        const float rk = p[crange] * static_cast<float>(k + 1) / static_cast<float>(nrec);
        const float a = rk * rk + (hs - hr) * (hs - hr), b = rk * rk + (hs + hr) * (hs + hr);
        v = (c - np < nrec) ? logf(4.0f * hs * hr) - logf(sqrtf(a) + sqrtf(b)) : 10.0f * log10f(b / a);
    }
    F[t] = v;
}

// one warp per query: mean over `members` predictions Y [members][n][nout]
// and the root mean square over the outputs of their standard deviation
__global__ void k_ensemble_stats(const float* __restrict__ Y, int members, int n, int nout, float* __restrict__ mean,
                                 float* __restrict__ spread) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const size_t plane = static_cast<size_t>(n) * nout;
    float var = 0.0f;
    for (int c = lane; c < nout; c += 32) {
        const size_t o = static_cast<size_t>(row) * nout + c;
        float s = 0.0f;
        for (int m = 0; m < members; ++m) s += Y[m * plane + o];
        const float mu = s / members;
        float q = 0.0f;
        for (int m = 0; m < members; ++m) {
            const float d = Y[m * plane + o] - mu;
            q += d * d;
        }
        mean[o] = mu;
        var += q / members;
    }
    for (int k = 16; k > 0; k >>= 1) var += __shfl_xor_sync(0xffffffffu, var, k);
    if (lane == 0) spread[row] = sqrtf(var / nout);
}

// denormalised outputs of the first `valid` rows: out [valid][nout]
__global__ void k_denorm(const float* __restrict__ Y, int NO, int valid, int nout, const float* __restrict__ mean,
                         const float* __restrict__ sd, float* __restrict__ out) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<size_t>(valid) * nout) return;
    const int r = static_cast<int>(i / nout), c = static_cast<int>(i % nout);
    out[i] = Y[static_cast<size_t>(r) * NO + c] * sd[c] + mean[c];
}

struct Buf {
    void* p = nullptr;
    Buf() = default;
    explicit Buf(size_t bytes) {  // zeroed and complete before any stream uses it
        ck(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc");
        ck(cudaMemset(p, 0, bytes ? bytes : 16), "cudaMemset");
        ck(cudaDeviceSynchronize(), "cudaMemset");
    }
    Buf(Buf&& o) noexcept : p(o.p) { o.p = nullptr; }
    Buf& operator=(Buf&& o) noexcept {
        std::swap(p, o.p);
        return *this;
    }
    ~Buf() {
        if (p) cudaFree(p);
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

}  // namespace

void gemm(int device, int epi, int M, int N, int K, const void* A, const void* B, const float* bias, const void* mask,
          void* out, void* outT, void* stream) {
    validate(epi, M, N, K, A, B, bias, mask, out, outT);
    ck(cudaSetDevice(device), "cudaSetDevice");
    Buf status(sizeof(int));
    const Plan p = make_plan(epi, M, N, K, A, B, bias, mask, N, out, N, outT, M, status.as<int>());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    launch(p, s);
    ck(cudaStreamSynchronize(s), "GEMM");
    int st = 0;
    ck(cudaMemcpy(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost), "GEMM status");
    if (st) throw SolverError{-7, "a GEMM pipeline wait ran out"};
}

// ----------------------------------------------------------------- network
class NetImpl {
   public:
    NetImpl(int device, int n_in, int width, int hidden, int n_out, int batch, uint64_t seed)
        : dev_(device), nin_(n_in), nout_(n_out), width_(width), hidden_(hidden), B_(batch) {
        if (n_in < 1 || n_out < 1 || hidden < 1 || width < 128 || width % 128 || batch < 128 || batch % 128)
            bad("network: need n_in, n_out, hidden >= 1, width and batch multiples of 128");
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, dev_), "device properties");
        if (prop.major != 10) throw SolverError{-3, "the tensor-core kernels target sm_100a (B200)"};
        ck(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreate(&e0_), "event");
        ck(cudaEventCreate(&e1_), "event");
        K0_ = round_up(nin_, kTileK);
        NO_ = round_up(nout_, 128);
        L_ = hidden_ + 1;
        for (int l = 0; l < L_; ++l) {
            Kp_.push_back(l == 0 ? K0_ : width_);
            Np_.push_back(l == L_ - 1 ? NO_ : width_);
            Kr_.push_back(l == 0 ? nin_ : width_);
            Nr_.push_back(l == L_ - 1 ? nout_ : width_);
        }
        for (int l = 0; l < L_; ++l) {
            const size_t nw = static_cast<size_t>(Np_[l]) * Kp_[l];
            W_.emplace_back(nw * 4); mW_.emplace_back(nw * 4); vW_.emplace_back(nw * 4); dW_.emplace_back(nw * 4);
            b_.emplace_back(Np_[l] * 4); mb_.emplace_back(Np_[l] * 4); vb_.emplace_back(Np_[l] * 4); db_.emplace_back(Np_[l] * 4);
            Wb_.emplace_back(nw * 2); WTb_.emplace_back(nw * 2);
        }
        status_ = Buf(sizeof(int));
        step_ = Buf(sizeof(int));
        norm_ = Buf(sizeof(float) * 2 * (nin_ + nout_));
        std::vector<float> nrm(2 * (nin_ + nout_), 0.0f);
        for (int c = 0; c < nin_; ++c) nrm[nin_ + c] = 1.0f;              // input 1/std
        for (int c = 0; c < nout_; ++c) nrm[2 * nin_ + nout_ + c] = 1.0f;  // output std
        upload_norm(nrm);
        init_params(seed);
        // training activations
        X0_ = Buf(static_cast<size_t>(B_) * K0_ * 2);
        X0T_ = Buf(static_cast<size_t>(B_) * K0_ * 2);
        for (int l = 0; l < L_; ++l) {
            H_.emplace_back(static_cast<size_t>(B_) * Np_[l] * 2);
            HT_.emplace_back(static_cast<size_t>(B_) * Np_[l] * 2);
            dZ_.emplace_back(static_cast<size_t>(B_) * Np_[l] * 2);
            dZT_.emplace_back(static_cast<size_t>(B_) * Np_[l] * 2);
        }
        Y_ = Buf(static_cast<size_t>(B_) * NO_ * 4);
        build_train_plans();
    }

    ~NetImpl() {
        cudaSetDevice(dev_);
        if (graph_) cudaGraphExecDestroy(graph_);
        if (e0_) cudaEventDestroy(e0_);
        if (e1_) cudaEventDestroy(e1_);
        if (s_) cudaStreamDestroy(s_);
    }

    // every transfer is ordered on the network's stream (non-blocking with
    // respect to the legacy stream)
    void up(void* dst, const void* src, size_t bytes) const {
        ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s_), "upload");
    }
    void down(void* dst, const void* src, size_t bytes) const {
        ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s_), "download");
        ck(cudaStreamSynchronize(s_), "download");
    }
    void clear(void* dst, size_t bytes) const { ck(cudaMemsetAsync(dst, 0, bytes, s_), "memset"); }

    int n_params() const {
        int n = 0;
        for (int l = 0; l < L_; ++l) n += Nr_[l] * Kr_[l] + Nr_[l];
        return n;
    }

    void get_params(float* out) const {
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        size_t o = 0;
        for (int l = 0; l < L_; ++l) {
            std::vector<float> w(static_cast<size_t>(Np_[l]) * Kp_[l]), b(Np_[l]);
            down(w.data(), W_[l].p, w.size() * 4);
            down(b.data(), b_[l].p, b.size() * 4);
            for (int n = 0; n < Nr_[l]; ++n)
                for (int k = 0; k < Kr_[l]; ++k) out[o++] = w[static_cast<size_t>(n) * Kp_[l] + k];
            for (int n = 0; n < Nr_[l]; ++n) out[o++] = b[n];
        }
    }

    void set_params(const float* in) {
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        size_t o = 0;
        for (int l = 0; l < L_; ++l) {
            std::vector<float> w(static_cast<size_t>(Np_[l]) * Kp_[l], 0.0f), b(Np_[l], 0.0f);
            for (int n = 0; n < Nr_[l]; ++n)
                for (int k = 0; k < Kr_[l]; ++k) w[static_cast<size_t>(n) * Kp_[l] + k] = in[o++];
            for (int n = 0; n < Nr_[l]; ++n) b[n] = in[o++];
            up(W_[l].p, w.data(), w.size() * 4);
            up(b_[l].p, b.data(), b.size() * 4);
            clear(mW_[l].p, w.size() * 4);
            clear(vW_[l].p, w.size() * 4);
            clear(mb_[l].p, b.size() * 4);
            clear(vb_[l].p, b.size() * 4);
        }
        refresh_bf16();
        ck(cudaStreamSynchronize(s_), "params");
    }

    void set_data(const float* X, const float* T, int n) {
        if (n < 1) bad("no training data");
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        std::vector<float> nrm(2 * (nin_ + nout_));
        auto stats = [&](const float* A, int cols, int c, float& mean, float& sd) {
            double s = 0, q = 0;
            for (int r = 0; r < n; ++r) s += A[static_cast<size_t>(r) * cols + c];
            mean = static_cast<float>(s / n);
            for (int r = 0; r < n; ++r) {
                const double d = A[static_cast<size_t>(r) * cols + c] - mean;
                q += d * d;
            }
            sd = static_cast<float>(std::sqrt(q / n));
            if (!(sd > 1e-12f)) sd = 1.0f;
        };
        for (int c = 0; c < nin_; ++c) {
            float m, sd;
            stats(X, nin_, c, m, sd);
            nrm[c] = m;
            nrm[nin_ + c] = 1.0f / sd;
        }
        for (int c = 0; c < nout_; ++c) {
            float m, sd;
            stats(T, nout_, c, m, sd);
            nrm[2 * nin_ + c] = m;
            nrm[2 * nin_ + nout_ + c] = sd;
        }
        upload_norm(nrm);
        // targets are stored normalised; inputs raw (normalised when packed)
        std::vector<float> Tn(static_cast<size_t>(n) * nout_);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < nout_; ++c)
                Tn[static_cast<size_t>(r) * nout_ + c] =
                    (T[static_cast<size_t>(r) * nout_ + c] - nrm[2 * nin_ + c]) / nrm[2 * nin_ + nout_ + c];
        Xd_ = Buf(sizeof(float) * n * nin_);
        Td_ = Buf(sizeof(float) * n * nout_);
        up(Xd_.p, X, sizeof(float) * n * nin_);
        up(Td_.p, Tn.data(), sizeof(float) * n * nout_);
        ck(cudaStreamSynchronize(s_), "data");
        n_data_ = n;
    }

    void get_normalization(float* im, float* is, float* om, float* os) const {
        for (int c = 0; c < nin_; ++c) { im[c] = norm_h_[c]; is[c] = 1.0f / norm_h_[nin_ + c]; }
        for (int c = 0; c < nout_; ++c) { om[c] = norm_h_[2 * nin_ + c]; os[c] = norm_h_[2 * nin_ + nout_ + c]; }
    }
    void set_normalization(const float* im, const float* is, const float* om, const float* os) {
        std::vector<float> nrm(2 * (nin_ + nout_));
        for (int c = 0; c < nin_; ++c) {
            if (!(is[c] > 0)) bad("input standard deviations must be positive");
            nrm[c] = im[c];
            nrm[nin_ + c] = 1.0f / is[c];
        }
        for (int c = 0; c < nout_; ++c) {
            if (!(os[c] > 0)) bad("output standard deviations must be positive");
            nrm[2 * nin_ + c] = om[c];
            nrm[2 * nin_ + nout_ + c] = os[c];
        }
        upload_norm(nrm);
    }

    double train(int steps, float lr0, float lr1, uint64_t seed, int report, float wd) {
        if (!(wd >= 0.0f)) bad("weight decay must be >= 0");
        wd_ = wd;
        if (!n_data_) bad("set_data first");
        if (steps < 1) bad("steps must be positive");
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        // minibatch rows: shuffled passes over the data
        std::mt19937_64 rng(seed);
        std::vector<int> idx(static_cast<size_t>(steps) * B_), perm(n_data_);
        std::iota(perm.begin(), perm.end(), 0);
        size_t pos = perm.size();
        for (size_t i = 0; i < idx.size(); ++i) {
            if (pos == perm.size()) {
                std::shuffle(perm.begin(), perm.end(), rng);
                pos = 0;
            }
            idx[i] = perm[pos++];
        }
        // cosine learning-rate schedule lr0 -> lr1
        std::vector<float> lr(steps);
        for (int t = 0; t < steps; ++t)
            lr[t] = lr1 + 0.5f * (lr0 - lr1) * (1.0f + std::cos(3.14159265358979f * t / std::max(1, steps - 1)));
        idx_ = Buf(sizeof(int) * idx.size());
        lr_ = Buf(sizeof(float) * steps);
        loss_ = Buf(sizeof(float) * steps);
        up(idx_.p, idx.data(), sizeof(int) * idx.size());
        up(lr_.p, lr.data(), sizeof(float) * steps);
        clear(step_.p, sizeof(int));
        clear(status_.p, sizeof(int));
        // the step graph reads the index / schedule / loss buffers by pointer
        if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
        cudaGraph_t g;
        ck(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal), "capture");
        enqueue_step(idx_.as<int>(), step_.as<int>(), true);
        ck(cudaStreamEndCapture(s_, &g), "capture");
        ck(cudaGraphInstantiate(&graph_, g, 0), "graph");
        cudaGraphDestroy(g);
        ck(cudaEventRecord(e0_, s_), "event");
        for (int t = 0; t < steps; ++t) {
            ck(cudaGraphLaunch(graph_, s_), "graph launch");
            launches_ += per_step_;
        }
        ck(cudaEventRecord(e1_, s_), "event");
        ck(cudaStreamSynchronize(s_), "training");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, e0_, e1_), "event");
        last_ms_ = ms;
        check_status();
        std::vector<float> lh(steps);
        down(lh.data(), loss_.p, sizeof(float) * steps);
        const int k = std::max(1, std::min(report, steps));
        double s = 0;
        for (int t = steps - k; t < steps; ++t) s += lh[t];
        return s / k;
    }

    double gradients(float* grad) {
        if (n_data_ < B_) bad("gradients need at least one batch of data");
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        loss_ = Buf(sizeof(float));
        clear(status_.p, sizeof(int));
        enqueue_step(nullptr, nullptr, false);
        ck(cudaStreamSynchronize(s_), "gradients");
        check_status();
        size_t o = 0;
        for (int l = 0; l < L_; ++l) {
            std::vector<float> w(static_cast<size_t>(Np_[l]) * Kp_[l]), b(Np_[l]);
            down(w.data(), dW_[l].p, w.size() * 4);
            down(b.data(), db_[l].p, b.size() * 4);
            for (int n = 0; n < Nr_[l]; ++n)
                for (int k = 0; k < Kr_[l]; ++k) grad[o++] = w[static_cast<size_t>(n) * Kp_[l] + k];
            for (int n = 0; n < Nr_[l]; ++n) grad[o++] = b[n];
        }
        float loss = 0;
        down(&loss, loss_.p, sizeof(float));
        return loss;
    }

    void predict(const float* X, int n, float* Y) {
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        Buf xd(sizeof(float) * static_cast<size_t>(std::max(n, 1)) * nin_), yd(sizeof(float) * static_cast<size_t>(std::max(n, 1)) * nout_);
        ck(cudaMemcpyAsync(xd.p, X, sizeof(float) * static_cast<size_t>(n) * nin_, cudaMemcpyHostToDevice, s_), "inputs");
        predict_device(xd.as<float>(), n, yd.as<float>(), s_);
        ck(cudaMemcpyAsync(Y, yd.p, sizeof(float) * static_cast<size_t>(n) * nout_, cudaMemcpyDeviceToHost, s_), "outputs");
        ck(cudaStreamSynchronize(s_), "predict");
    }

    void predict_device(const float* X, int n, float* Y, cudaStream_t s) {
        if (n < 0) bad("negative query count");
        if (n == 0) return;
        ck(cudaSetDevice(dev_), "cudaSetDevice");
        ensure_infer();
        ck(cudaMemsetAsync(status_.p, 0, sizeof(int), s), "status");
        ck(cudaEventRecord(e0_, s), "event");
        if (use_fused_ && fused_ok_) {
            // per pass: pack + one fused launch that writes the denormalised rows
            for (int r0 = 0; r0 < n; r0 += kFusedChunk) {
                const int valid = std::min(kFusedChunk, n - r0);
                const int rows = round_up(valid, kTileM);
                const dim3 blk(K0_, std::max(1, 256 / K0_));
                k_pack<<<(rows + blk.y - 1) / blk.y, blk, 0, s>>>(X, nin_, nullptr, nullptr, r0, valid, rows, norm(0),
                                                                 norm(1), fX_.as<__nv_bfloat16>(), K0_, nullptr);
                ck(cudaGetLastError(), "pack");
                FusedArgs a = fargs_;
                a.M = rows;
                a.valid = valid;
                a.y = Y + static_cast<size_t>(r0) * nout_;
                k_mlp_fused<<<std::min(rows / kTileM, sm_count()), kFusedThreads, fused_smem_bytes(), s>>>(fmaps_, a);
                ck(cudaGetLastError(), "fused inference");
                launches_ += 2;
            }
        } else {
            for (int r0 = 0; r0 < n; r0 += kChunk) {
                const int valid = std::min(kChunk, n - r0);
                const int rows = round_up(valid, kTileM);
                const dim3 blk(K0_, std::max(1, 256 / K0_));
                k_pack<<<(rows + blk.y - 1) / blk.y, blk, 0, s>>>(X, nin_, nullptr, nullptr, r0, valid, rows, norm(0),
                                                                 norm(1), iX_.as<__nv_bfloat16>(), K0_, nullptr);
                ck(cudaGetLastError(), "pack");
                ++launches_;
                for (int l = 0; l < L_; ++l) {
                    Plan p = infer_[l];
                    p.g.M = rows;
                    launch(p, s);
                    ++launches_;
                }
                const size_t cnt = static_cast<size_t>(valid) * nout_;
                k_denorm<<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, s>>>(iY_.as<float>(), NO_, valid, nout_, norm(2),
                                                                                   norm(3), Y + static_cast<size_t>(r0) * nout_);
                ck(cudaGetLastError(), "denorm");
                ++launches_;
            }
        }
        ck(cudaEventRecord(e1_, s), "event");
        ck(cudaStreamSynchronize(s), "predict");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, e0_, e1_), "event");
        last_ms_ = ms;
        check_status();
    }

    long long launches() const { return launches_; }
    // returns whether the fused kernel serves this network's shapes
    bool set_fused(bool on) {
        ensure_infer();
        use_fused_ = on;
        return fused_ok_;
    }
    double last_ms() const { return last_ms_; }
    int n_in() const { return nin_; }
    int n_out() const { return nout_; }
    int device() const { return dev_; }

   private:
    static constexpr int kChunk = 65536;  // inference rows per pass

    const float* norm(int part) const {  // 0 in mean, 1 in 1/std, 2 out mean, 3 out std
        const int off[4] = {0, nin_, 2 * nin_, 2 * nin_ + nout_};
        return norm_.as<float>() + off[part];
    }
    void upload_norm(const std::vector<float>& nrm) {
        norm_h_ = nrm;
        up(norm_.p, nrm.data(), sizeof(float) * nrm.size());
        ck(cudaStreamSynchronize(s_), "normalisation");
    }
    void check_status() {
        int st = 0;
        down(&st, status_.p, sizeof(int));
        if (st) throw SolverError{-7, "a GEMM pipeline wait ran out"};
    }

    // He-uniform weights (bound sqrt(6 / fan_in)), zero biases; padding zero
    void init_params(uint64_t seed) {
        std::mt19937_64 rng(seed);
        for (int l = 0; l < L_; ++l) {
            std::vector<float> w(static_cast<size_t>(Np_[l]) * Kp_[l], 0.0f);
            const float a = std::sqrt(6.0f / Kr_[l]);
            std::uniform_real_distribution<float> u(-a, a);
            for (int n = 0; n < Nr_[l]; ++n)
                for (int k = 0; k < Kr_[l]; ++k) w[static_cast<size_t>(n) * Kp_[l] + k] = u(rng);
            up(W_[l].p, w.data(), w.size() * 4);
        }
        refresh_bf16();
        ck(cudaStreamSynchronize(s_), "init");
    }

    void refresh_bf16() {
        for (int l = 0; l < L_; ++l) {
            const size_t nw = static_cast<size_t>(Np_[l]) * Kp_[l];
            k_cast<<<static_cast<unsigned>((nw + 255) / 256), 256, 0, s_>>>(W_[l].as<float>(), Np_[l], Kp_[l],
                                                                            Wb_[l].as<__nv_bfloat16>(),
                                                                            WTb_[l].as<__nv_bfloat16>());
            ck(cudaGetLastError(), "cast");
        }
    }

    void build_train_plans() {
        int* st = status_.as<int>();
        for (int l = 0; l < L_; ++l) {
            const void* in = l == 0 ? X0_.p : H_[l - 1].p;
            const void* inT = l == 0 ? X0T_.p : HT_[l - 1].p;
            if (l < L_ - 1)
                fwd_.push_back(make_plan(kEpiBiasReluT, B_, Np_[l], Kp_[l], in, Wb_[l].p, b_[l].as<float>(), nullptr, 0,
                                         H_[l].p, Np_[l], HT_[l].p, B_, st));
            else
                fwd_.push_back(make_plan(kEpiBiasF32, B_, Np_[l], Kp_[l], in, Wb_[l].p, b_[l].as<float>(), nullptr, 0,
                                         Y_.p, Np_[l], nullptr, 0, st));
            // dW_l = dZ_l^T . X_l  (M = N_l, N = K_l, reduction over the batch)
            wgrad_.push_back(make_plan(kEpiF32, Np_[l], Kp_[l], B_, dZT_[l].p, inT, nullptr, nullptr, 0, dW_[l].p,
                                       Kp_[l], nullptr, 0, st));
            // dZ_{l-1} = (dZ_l . W_l) masked by the ReLU of layer l-1
            if (l > 0)
                dgrad_.push_back(make_plan(kEpiReluGradT, B_, Kp_[l], Np_[l], dZ_[l].p, WTb_[l].p, nullptr, H_[l - 1].p,
                                           Kp_[l], dZ_[l - 1].p, Kp_[l], dZT_[l - 1].p, B_, st));
            else
                dgrad_.push_back(Plan{});
        }
    }

    void ensure_infer() {
        if (!infer_.empty()) return;
        iX_ = Buf(static_cast<size_t>(kChunk) * K0_ * 2);
        iH_[0] = Buf(static_cast<size_t>(kChunk) * width_ * 2);
        iH_[1] = Buf(static_cast<size_t>(kChunk) * width_ * 2);
        iY_ = Buf(static_cast<size_t>(kChunk) * NO_ * 4);
        int* st = status_.as<int>();
        for (int l = 0; l < L_; ++l) {
            const void* in = l == 0 ? iX_.p : iH_[(l - 1) & 1].p;
            if (l < L_ - 1)
                infer_.push_back(make_plan(kEpiBiasRelu, kChunk, Np_[l], Kp_[l], in, Wb_[l].p, b_[l].as<float>(),
                                           nullptr, 0, iH_[l & 1].p, Np_[l], nullptr, 0, st));
            else
                infer_.push_back(make_plan(kEpiBiasF32, kChunk, Np_[l], Kp_[l], in, Wb_[l].p, b_[l].as<float>(), nullptr,
                                           0, iY_.p, Np_[l], nullptr, 0, st));
        }
        fused_ok_ = L_ >= 2 && L_ <= kFusedMaxLayers && K0_ == kTileK && NO_ == kFusedHalf;
        for (int l = 0; l < L_ && fused_ok_; ++l) {
            if (l < L_ - 1 && Np_[l] != kFusedWidth) fused_ok_ = false;
            if (l > 0 && Kp_[l] != kFusedWidth) fused_ok_ = false;
        }
        if (!fused_ok_) return;
        static bool attr = false;
        if (!attr) {
            ck(cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(fused_smem_bytes())),
               "fused inference shared-memory attribute");
            attr = true;
        }
        fX_ = Buf(static_cast<size_t>(kFusedChunk) * K0_ * 2);
        fmaps_.x = bf16_map(fX_.p, kFusedChunk, K0_, kTileM);
        fargs_.L = L_;
        for (int l = 0; l < L_; ++l) {
            fmaps_.w[l] = bf16_map(Wb_[l].p, Np_[l], Kp_[l], kFusedHalf);
            fargs_.nkb[l] = Kp_[l] / kTileK;
            fargs_.nhalf[l] = Np_[l] / kFusedHalf;
            fargs_.bias[l] = b_[l].as<float>();
        }
        fargs_.nout = nout_;
        fargs_.omean = norm(2);
        fargs_.osd = norm(3);
        fargs_.status = st;
    }

    // one training step: minibatch rows from idx (by the device step
    // counter) or rows 0 .. B-1; `update` adds Adam and the step increment
    void enqueue_step(const int* idx, const int* step, bool update) {
        int n = 0;
        const dim3 pb(K0_, std::max(1, 256 / K0_));
        k_pack<<<(B_ + pb.y - 1) / pb.y, pb, 0, s_>>>(Xd_.as<float>(), nin_, idx, step, 0, B_, B_, norm(0), norm(1),
                                                      X0_.as<__nv_bfloat16>(), K0_, X0T_.as<__nv_bfloat16>());
        ck(cudaGetLastError(), "pack");
        ++n;
        for (int l = 0; l < L_; ++l) { launch(fwd_[l], s_); ++n; }
        k_loss<<<B_, 256, 0, s_>>>(Y_.as<float>(), NO_, Td_.as<float>(), nout_, idx, step, B_,
                                   dZ_[L_ - 1].as<__nv_bfloat16>(), dZT_[L_ - 1].as<__nv_bfloat16>(), loss_.as<float>());
        ck(cudaGetLastError(), "loss");
        ++n;
        for (int l = L_ - 1; l >= 0; --l) {
            launch(wgrad_[l], s_);
            k_bias_grad<<<(Np_[l] + 7) / 8, 256, 0, s_>>>(dZT_[l].as<__nv_bfloat16>(), Np_[l], B_, db_[l].as<float>());
            ck(cudaGetLastError(), "bias gradient");
            n += 2;
            if (l > 0) { launch(dgrad_[l], s_); ++n; }
        }
        if (update) {
            for (int l = 0; l < L_; ++l) {
                const size_t nw = static_cast<size_t>(Np_[l]) * Kp_[l];
                k_adam<<<static_cast<unsigned>((nw + 255) / 256), 256, 0, s_>>>(
                    W_[l].as<float>(), dW_[l].as<float>(), mW_[l].as<float>(), vW_[l].as<float>(), nw, lr_.as<float>(), step,
                    wd_);
                k_adam<<<(Np_[l] + 255) / 256, 256, 0, s_>>>(b_[l].as<float>(), db_[l].as<float>(), mb_[l].as<float>(),
                                                              vb_[l].as<float>(), Np_[l], lr_.as<float>(), step, 0.0f);
                ck(cudaGetLastError(), "adam");
                n += 2;
            }
            refresh_bf16();
            n += L_;
            k_next_step<<<1, 1, 0, s_>>>(step_.as<int>());
            ck(cudaGetLastError(), "step");
            ++n;
        }
        per_step_ = n;
    }

    int dev_, nin_, nout_, width_, hidden_, B_;
    int K0_ = 0, NO_ = 0, L_ = 0;
    std::vector<int> Kp_, Np_, Kr_, Nr_;
    std::vector<Buf> W_, mW_, vW_, dW_, b_, mb_, vb_, db_, Wb_, WTb_;
    std::vector<Buf> H_, HT_, dZ_, dZT_;
    Buf X0_, X0T_, Y_, status_, step_, norm_, Xd_, Td_, idx_, lr_, loss_;
    Buf iX_, iH_[2], iY_;
    // fused inference (one persistent kernel for all layers) where the
    // shapes fit it: 64 inputs, hidden layers of 512, 256 outputs
    bool fused_ok_ = false, use_fused_ = true;
    static constexpr int kFusedChunk = 1 << 18;  // fused inference rows per pass
    Buf fX_;
    FusedMaps fmaps_{};
    FusedArgs fargs_{};
    std::vector<float> norm_h_;
    std::vector<Plan> fwd_, wgrad_, dgrad_, infer_;
    int n_data_ = 0;
    cudaStream_t s_ = nullptr;
    cudaEvent_t e0_ = nullptr, e1_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int per_step_ = 0;
    float wd_ = 0.0f;
    long long launches_ = 0;
    double last_ms_ = 0;
};

Net::Net(int device, int n_in, int width, int hidden, int n_out, int batch, uint64_t seed)
    : impl_(new NetImpl(device, n_in, width, hidden, n_out, batch, seed)) {}
Net::~Net() = default;
int Net::n_params() const { return impl_->n_params(); }
void Net::get_params(float* out) const { impl_->get_params(out); }
void Net::set_params(const float* in) { impl_->set_params(in); }
void Net::set_data(const float* X, const float* T, int n) { impl_->set_data(X, T, n); }
void Net::get_normalization(float* a, float* b, float* c, float* d) const { impl_->get_normalization(a, b, c, d); }
void Net::set_normalization(const float* a, const float* b, const float* c, const float* d) {
    impl_->set_normalization(a, b, c, d);
}
double Net::train(int steps, float lr, float lr_final, uint64_t seed, int report, float weight_decay) {
    return impl_->train(steps, lr, lr_final, seed, report, weight_decay);
}
double Net::gradients(float* grad) { return impl_->gradients(grad); }
void Net::predict(const float* X, int n, float* Y) { impl_->predict(X, n, Y); }
void Net::predict_device(const float* X, int n, float* Y, void* stream) {
    impl_->predict_device(X, n, Y, static_cast<cudaStream_t>(stream));
}
long long Net::launches() const { return impl_->launches(); }
bool Net::set_fused(bool on) { return impl_->set_fused(on); }
int Net::n_in() const { return impl_->n_in(); }
int Net::n_out() const { return impl_->n_out(); }
int Net::device() const { return impl_->device(); }

void RayFeatures::validate() const {
    if (n_par < 1 || n_rec < 1 || col_hs < 0 || col_hs >= n_par || col_hr < 0 || col_hr >= n_par || col_range < 0 ||
        col_range >= n_par)
        bad("ray features: need n_par, n_rec >= 1 and the height and range columns inside the row");
}

static void launch_ray_features(const RayFeatures& g, const float* P, int n, float* F, cudaStream_t s) {
    const long long total = static_cast<long long>(n) * g.n_out();
    if (total == 0) return;
    k_ray_features<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(P, n, g.n_par, g.col_hs, g.col_hr,
                                                                              g.col_range, g.n_rec, F);
    ck(cudaGetLastError(), "ray features");
}

void ray_features(const RayFeatures& g, const float* P, int n, float* F, void* stream) {
    g.validate();
    if (n < 0) bad("ray features: n >= 0");
    launch_ray_features(g, P, n, F, static_cast<cudaStream_t>(stream));
}

// mean and disagreement of the members over host rows X [n][nx]; with g,
// X holds query rows and the networks read their ray features
static void ensemble_run(Net* const* nets, int members, const RayFeatures* g, const float* X, int n, float* mean,
                         float* spread) {
    if (members < 1 || !nets || n < 0) bad("ensemble: need at least one network and n >= 0");
    const int nin = nets[0]->n_in(), nout = nets[0]->n_out(), dev = nets[0]->device();
    for (int m = 0; m < members; ++m)
        if (!nets[m] || nets[m]->n_in() != nin || nets[m]->n_out() != nout || nets[m]->device() != dev)
            bad("ensemble members must share inputs, outputs and device");
    if (g) {
        g->validate();
        if (g->n_out() != nin) bad("ensemble: the networks' inputs are not the query rows' ray features");
    }
    const int nx = g ? g->n_par : nin;
    if (n == 0) return;
    ck(cudaSetDevice(dev), "cudaSetDevice");
    const int chunk = std::min(n, 1 << 18);
    Buf xd(sizeof(float) * static_cast<size_t>(chunk) * nin), yd(sizeof(float) * static_cast<size_t>(chunk) * nout * members),
        md(sizeof(float) * static_cast<size_t>(chunk) * nout), sd(sizeof(float) * chunk),
        pd(g ? sizeof(float) * static_cast<size_t>(chunk) * nx : 0);
    cudaStream_t s;
    ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    try {
        for (int r0 = 0; r0 < n; r0 += chunk) {
            const int c = std::min(chunk, n - r0);
            ck(cudaMemcpyAsync(g ? pd.p : xd.p, X + static_cast<size_t>(r0) * nx, sizeof(float) * c * nx,
                               cudaMemcpyHostToDevice, s), "inputs");
            if (g) launch_ray_features(*g, pd.as<float>(), c, xd.as<float>(), s);
            for (int m = 0; m < members; ++m)
                nets[m]->predict_device(xd.as<float>(), c, yd.as<float>() + static_cast<size_t>(m) * c * nout, s);
            k_ensemble_stats<<<(c + 7) / 8, 256, 0, s>>>(yd.as<float>(), members, c, nout, md.as<float>(), sd.as<float>());
            ck(cudaGetLastError(), "ensemble statistics");
            ck(cudaMemcpyAsync(mean + static_cast<size_t>(r0) * nout, md.p, sizeof(float) * c * nout,
                               cudaMemcpyDeviceToHost, s), "outputs");
            ck(cudaMemcpyAsync(spread + r0, sd.p, sizeof(float) * c, cudaMemcpyDeviceToHost, s), "outputs");
            ck(cudaStreamSynchronize(s), "ensemble");
        }
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
}

void ensemble_predict(Net* const* nets, int members, const float* X, int n, float* mean, float* spread) {
    ensemble_run(nets, members, nullptr, X, n, mean, spread);
}

void ensemble_predict_rays(Net* const* nets, int members, const RayFeatures& g, const float* P, int n, float* mean,
                           float* spread) {
    ensemble_run(nets, members, &g, P, n, mean, spread);
}
double Net::last_device_ms() const { return impl_->last_ms(); }

}  // namespace mlp
}  // namespace fdtd
