// Host side of the surrogate network: a ReLU MLP with bf16 weights and
// activations, FP32 accumulation (tcgen05 tensor cores) and FP32 master
// weights trained by Adam, all on one device.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

namespace fdtd {
namespace mlp {

// D = A . B^T on the device (all pointers device memory): A [M][K] and
// B [N][K] bf16 row-major; epi selects the epilogue (mlp_tc.cuh Epilogue);
// out [M][N] bf16 or FP32; outT [N][M] bf16 for the transposing epilogues;
// bias [N] FP32; mask [M][N] bf16. M a multiple of 128, N and K of 64.
void gemm(int device, int epi, int M, int N, int K, const void* A, const void* B, const float* bias, const void* mask,
          void* out, void* outT, void* stream);

class NetImpl;

class Net {
   public:
    // n_in inputs, `hidden` ReLU layers of `width` units, n_out linear
    // outputs; batch: training minibatch rows (a multiple of 128)
    Net(int device, int n_in, int width, int hidden, int n_out, int batch, uint64_t seed);
    ~Net();
    Net(const Net&) = delete;
    Net& operator=(const Net&) = delete;

    int n_params() const;
    // FP32 master parameters, layer by layer: W [N][K] (unpadded) then b [N]
    void get_params(float* out) const;
    void set_params(const float* in);
    // training data (host, row-major): X [n][n_in], T [n][n_out]; input and
    // target normalisation (mean / standard deviation per column) is taken
    // from this data
    void set_data(const float* X, const float* T, int n);
    void get_normalization(float* in_mean, float* in_std, float* out_mean, float* out_std) const;
    void set_normalization(const float* in_mean, const float* in_std, const float* out_mean, const float* out_std);
    // Adam steps on shuffled minibatches (decoupled weight decay on the
    // weights); returns the mean loss (normalised MSE) of the last `report`
    // steps
    double train(int steps, float lr, float lr_final, uint64_t seed, int report, float weight_decay);
    // One forward + backward on the first `batch` rows of the data without
    // an update: loss and the gradients of every parameter (same order as
    // get_params)
    double gradients(float* grad);
    // predictions for host inputs X [n][n_in] -> Y [n][n_out] (denormalised)
    void predict(const float* X, int n, float* Y);
    // the same on device buffers (X [n][n_in], Y [n][n_out] FP32) on a stream
    void predict_device(const float* X, int n, float* Y, void* stream);
    long long launches() const;
    // inference by one fused kernel for all layers (default, where the
    // shapes fit it) or by one GEMM per layer; returns whether the fused
    // kernel serves this network
    bool set_fused(bool on);
    double last_device_ms() const;
    int n_in() const;
    int n_out() const;
    int device() const;

   private:
    std::unique_ptr<NetImpl> impl_;
};

// Answer of an ensemble of networks with the same inputs and outputs on one
// device, for host inputs X [n][n_in]: the members' mean [n][n_out] and
// their disagreement [n] (root mean square over the outputs of the standard
// deviation across members), host buffers. The reduction runs on the
// device, so only the mean and the disagreement cross back to the host.
void ensemble_predict(Net* const* nets, int members, const float* X, int n, float* mean, float* spread);

// Ray-geometry inputs of excess-attenuation queries. A query row P [n_par]
// holds the source height, receiver height and farthest range at columns
// col_hs, col_hr, col_range; its network input row is P followed, per
// receiver k < n_rec at range r_k = range (k + 1) / n_rec, by
// ln(d2 - d1) and then, for every k, 20 log10(d2 / d1), with the direct
// and ground-reflected path lengths d1 = |(r_k, hs - hr)| and
// d2 = |(r_k, hs + hr)| (flat-ground image source).
struct RayFeatures {
    int n_par, col_hs, col_hr, col_range, n_rec;
    int n_out() const { return n_par + 2 * n_rec; }
    void validate() const;
};
// F [n][g.n_out()] from P [n][g.n_par], device buffers, on a stream
void ray_features(const RayFeatures& g, const float* P, int n, float* F, void* stream);
// ensemble_predict of host query rows P [n][g.n_par]: the rows cross to the
// device as they are and the networks (n_in == g.n_out()) read their ray
// features, formed there
void ensemble_predict_rays(Net* const* nets, int members, const RayFeatures& g, const float* P, int n, float* mean,
                           float* spread);

}  // namespace mlp
}  // namespace fdtd
