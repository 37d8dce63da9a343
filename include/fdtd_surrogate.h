/*
 * fdtd_surrogate.h -- C ABI of the surrogate network that maps ground,
 * geometry, terrain and wind parameters to excess-attenuation spectra,
 * trained on solves of the FDTD path (fdtd_b200.h). No counterpart in the
 * reference repository, which only runs the solver.
 *
 * The network is a ReLU MLP: n_in inputs, `hidden` layers of `width`
 * units, n_out linear outputs. Weights and activations are bf16, products
 * accumulate in FP32 on the sm_100a tensor cores (tcgen05, operands staged
 * by TMA, accumulators in tensor memory), and the FP32 master weights are
 * trained with Adam on the device. Inputs are normalised by per-column mean
 * and standard deviation and outputs denormalised likewise (taken from the
 * training data). Status codes and fdtd_last_error() are those of
 * fdtd_b200.h; FDTD_ERR_TIMEOUT reports a tensor-core pipeline wait that
 * ran out (the kernels never hang).
 */
#ifndef FDTD_SURROGATE_H
#define FDTD_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

/* GEMM epilogues of fdtd_tc_gemm */
#define FDTD_EPI_F32 0            /* out = A B^T (FP32) */
#define FDTD_EPI_BIAS_RELU_T 1    /* out = relu(A B^T + bias) (bf16), outT = its transpose */
#define FDTD_EPI_BIAS_F32 2       /* out = A B^T + bias (FP32) */
#define FDTD_EPI_RELU_GRAD_T 3    /* out = A B^T where mask > 0, else 0 (bf16), outT = transpose */
#define FDTD_EPI_BIAS_RELU 4      /* out = relu(A B^T + bias) (bf16) */

/* One tensor-core GEMM on device buffers: A [M][K] and B [N][K] bf16
 * row-major, out [M][N], outT [N][M], bias [N] FP32, mask [M][N] bf16.
 * M a multiple of 128, N and K multiples of 64, pointers 16-byte aligned.
 * stream: a cudaStream_t (NULL: legacy stream); synchronises it. */
int fdtd_tc_gemm(int device, int epilogue, int M, int N, int K, const void *A, const void *B, const float *bias,
                 const void *mask, void *out, void *outT, void *stream);

typedef struct fdtd_net fdtd_net;

/* batch: training minibatch rows, a multiple of 128; width a multiple of 128 */
int fdtd_net_create(int device, int n_in, int width, int hidden, int n_out, int batch, unsigned long long seed,
                    fdtd_net **out);
int fdtd_net_destroy(fdtd_net *h);

/* FP32 master parameters, layer by layer: W [N][K] then b [N] */
int fdtd_net_n_params(const fdtd_net *h, int *n);
int fdtd_net_get_params(const fdtd_net *h, float *out);
int fdtd_net_set_params(fdtd_net *h, const float *in);

/* training data on the host: X [n][n_in], T [n][n_out]; sets the
 * normalisation from it */
int fdtd_net_set_data(fdtd_net *h, const float *X, const float *T, int n);
int fdtd_net_get_normalization(const fdtd_net *h, float *in_mean, float *in_std, float *out_mean, float *out_std);
int fdtd_net_set_normalization(fdtd_net *h, const float *in_mean, const float *in_std, const float *out_mean,
                               const float *out_std);

/* steps Adam updates on shuffled minibatches (cosine learning rate lr ->
 * lr_final, decoupled weight decay on the weights, minibatch order from
 * seed); *loss = mean normalised MSE of the last `report` steps */
int fdtd_net_train(fdtd_net *h, int steps, float lr, float lr_final, float weight_decay, unsigned long long seed,
                   int report, double *loss);

/* forward + backward on the first `batch` data rows without an update:
 * gradients of every parameter (fdtd_net_get_params order) and the loss */
int fdtd_net_gradients(fdtd_net *h, float *grad, double *loss);

/* predictions: X [n][n_in] -> Y [n][n_out], host buffers */
int fdtd_net_predict(fdtd_net *h, const float *X, int n, float *Y);
/* the same on device buffers, on a cudaStream_t (synchronises it) */
int fdtd_net_predict_device(fdtd_net *h, const float *X, int n, float *Y, void *stream);

/* answer of an ensemble of networks (same n_in, n_out and device): the
 * members' mean [n][n_out] and their disagreement [n] -- the root mean
 * square over the outputs of the standard deviation across members --
 * for host inputs X [n][n_in]; the reduction runs on the device */
int fdtd_net_ensemble_predict(fdtd_net *const *nets, int members, const float *X, int n, float *mean,
                              float *spread);

/* Ray-geometry network inputs of excess-attenuation queries, formed on the
 * device. A query row P [n_par] holds the source height, the receiver
 * height and the farthest range at columns col_hs, col_hr, col_range. Its
 * network input row [n_par + 2 n_rec] is P, then ln(d2 - d1) for every
 * receiver k < n_rec at range r_k = range (k + 1) / n_rec, then
 * 20 log10(d2 / d1) for every k, with d1 = |(r_k, hs - hr)| the direct and
 * d2 = |(r_k, hs + hr)| the ground-reflected path (flat-ground image
 * source). F [n][n_par + 2 n_rec] from P [n][n_par], device buffers, on a
 * cudaStream_t (not synchronised). */
int fdtd_ray_features(const float *P, int n, int n_par, int col_hs, int col_hr, int col_range, int n_rec, float *F,
                      void *stream);
/* fdtd_net_ensemble_predict of host query rows P [n][n_par]: the rows cross
 * to the device as they are and the members (n_in = n_par + 2 n_rec) read
 * their ray features, formed there */
int fdtd_net_ensemble_predict_rays(fdtd_net *const *nets, int members, const float *P, int n, int n_par, int col_hs,
                                   int col_hr, int col_range, int n_rec, float *mean, float *spread);

/* Inference path: on != 0 one fused persistent kernel for all layers
 * (activations stay in shared and tensor memory; the default where the
 * shapes fit it: 64 padded inputs, hidden layers of 512, 256 padded
 * outputs), on = 0 one tensor-core GEMM per layer. served (may be NULL)
 * receives whether the fused kernel serves this network. */
int fdtd_net_set_fused(fdtd_net *h, int on, int *served);

/* kernel launches so far and device milliseconds of the last train /
 * predict call */
int fdtd_net_info(const fdtd_net *h, long long *launches, double *last_ms);

#ifdef __cplusplus
}
#endif

#endif
