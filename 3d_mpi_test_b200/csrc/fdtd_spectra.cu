// Receiver spectra on the GPU: the reference's post-processing
// (airpore::get_FFT_y1, airpore.cpp:966-1011, and FFT / FFT_output,
// FFT.cpp:15-120) for a batch of receiver traces, plus third-octave band
// levels and excess attenuation built on it.
//
// The transform is the reference's radix-2 decimation-in-time FFT run stage
// by stage with one thread per butterfly. Its twiddle factors are generated
// on the host by the reference's own recurrence (start at 1, advance by the
// stage root, next root by the half-angle formulas) and every butterfly is
// evaluated with explicitly rounded FP64 operations in the reference's
// order, so the GPU result equals the reference's FFT bit for bit.
#include <cmath>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fdtd_solver.hpp"

namespace fdtd {
namespace {

// bit-reversal permutation of the zero-padded traces: traces [nrec][nt] ->
// re/im [nrec][n] (airpore.cpp:1004-1005 padding, FFT.cpp:27-43 reversal)
__global__ void k_fft_load(const double* __restrict__ tr, int nt, int m, double* re, double* im) {
    const long n = 1L << m;
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int r = blockIdx.y;
    const long rev = static_cast<long>(__brevll(static_cast<unsigned long long>(i)) >> (64 - m));
    re[r * n + rev] = i < nt ? tr[static_cast<long>(r) * nt + i] : 0.0;
    im[r * n + rev] = 0.0;
}

// one butterfly stage (FFT.cpp:46-72): pair p of stage `half`
__global__ void k_fft_stage(double* re, double* im, int m, long half, const double2* __restrict__ tw) {
    const long n = 1L << m;
    const long p = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (p >= n / 2) return;
    const long a = p % half, i = (p / half) * 2 * half + a, b = i + half;
    double* x = re + blockIdx.y * n;
    double* y = im + blockIdx.y * n;
    const double2 w = tw[half - 1 + a];  // stage twiddles are stored from offset half - 1
    const double t1 = __dsub_rn(__dmul_rn(w.x, x[b]), __dmul_rn(w.y, y[b]));
    const double t2 = __dadd_rn(__dmul_rn(w.x, y[b]), __dmul_rn(w.y, x[b]));
    const double xi = x[i], yi = y[i];
    x[b] = __dsub_rn(xi, t1);
    y[b] = __dsub_rn(yi, t2);
    x[i] = __dadd_rn(xi, t1);
    y[i] = __dadd_rn(yi, t2);
}

// |X_k| of the forward transform scaled by 1/n (FFT.cpp:75-80 scaling,
// FFT_output's abs) for bins k in [k0, k0 + nk)
__global__ void k_fft_mag(const double* re, const double* im, int m, long k0, long nk, double* mag) {
    const long n = 1L << m;
    const long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (k >= nk) return;
    const long src = blockIdx.y * n + k0 + k;
    const double x = __ddiv_rn(re[src], static_cast<double>(n)), y = __ddiv_rn(im[src], static_cast<double>(n));
    mag[blockIdx.y * nk + k] = hypot(x, y);
}

// forward scaling by 1/n (FFT.cpp:75-80), in place
__global__ void k_fft_scale(double* re, double* im, int m) {
    const long n = 1L << m;
    const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    re[blockIdx.y * n + i] = __ddiv_rn(re[blockIdx.y * n + i], static_cast<double>(n));
    im[blockIdx.y * n + i] = __ddiv_rn(im[blockIdx.y * n + i], static_cast<double>(n));
}

// twiddles of every stage in the reference's recurrence: stage with span
// 2*half stores its half factors at [half - 1, 2*half - 1) (FFT.cpp:46-72)
std::vector<double2> twiddles(int m) {
    const long n = 1L << m;
    std::vector<double2> tw(n > 1 ? n - 1 : 1);
    double c1 = -1.0, c2 = 0.0;
    for (long half = 1; half < n; half *= 2) {
        double u1 = 1.0, u2 = 0.0;
        for (long a = 0; a < half; ++a) {
            tw[half - 1 + a] = make_double2(u1, u2);
            const double z = u1 * c1 - u2 * c2;
            u2 = u1 * c2 + u2 * c1;
            u1 = z;
        }
        c2 = -std::sqrt((1.0 - c1) / 2.0);  // forward transform (dir = 1)
        c1 = std::sqrt((1.0 + c1) / 2.0);
    }
    return tw;
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t bytes) {
        if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) throw SolverError{-3, "cudaMalloc failed for the spectrum buffers"};
    }
    ~DevBuf() { cudaFree(p); }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw SolverError{-3, std::string(what) + ": " + cudaGetErrorString(e)};
}

}  // namespace

// Runs the transform of every trace on the device; then either copies the
// 1/n-scaled complex spectra (re, im [nrec][n]) or the magnitudes of bins
// [k0, k0 + nk) (mag [nrec][nk]) to the host.
static void run_fft(int device, const double* traces, int nrec, int nt, int m, long k0, long nk, double* mag,
                    double* re_out, double* im_out) {
    if (nrec < 1 || nt < 1 || m < 1 || m > 24) throw SolverError{-5, "spectrum: need nrec >= 1, nt >= 1, 1 <= fft_m <= 24"};
    const long n = 1L << m;
    if (mag && (k0 < 0 || nk < 1 || k0 + nk > n / 2 + 1))
        throw SolverError{-5, "spectrum: bin range outside 0 .. 2^(fft_m-1)"};
    ck(cudaSetDevice(device), "cudaSetDevice");
    cudaStream_t s;
    ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        const std::vector<double2> tw = twiddles(m);
        DevBuf dtr(sizeof(double) * nrec * static_cast<size_t>(nt)), dre(sizeof(double) * nrec * n),
            dim(sizeof(double) * nrec * n), dtw(sizeof(double2) * tw.size()),
            dmag(mag ? sizeof(double) * nrec * nk : 1);
        ck(cudaMemcpyAsync(dtr.p, traces, sizeof(double) * nrec * static_cast<size_t>(nt), cudaMemcpyHostToDevice, s),
           "trace upload");
        ck(cudaMemcpyAsync(dtw.p, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice, s), "twiddle upload");
        const int T = 256;
        k_fft_load<<<dim3((n + T - 1) / T, nrec), T, 0, s>>>(dtr.as<double>(), nt, m, dre.as<double>(), dim.as<double>());
        for (long half = 1; half < n; half *= 2)
            k_fft_stage<<<dim3((n / 2 + T - 1) / T, nrec), T, 0, s>>>(dre.as<double>(), dim.as<double>(), m, half,
                                                                      dtw.as<double2>());
        if (mag) {
            k_fft_mag<<<dim3((nk + T - 1) / T, nrec), T, 0, s>>>(dre.as<double>(), dim.as<double>(), m, k0, nk,
                                                                  dmag.as<double>());
            ck(cudaGetLastError(), "spectrum kernels");
            ck(cudaMemcpyAsync(mag, dmag.p, sizeof(double) * nrec * nk, cudaMemcpyDeviceToHost, s), "spectrum download");
        } else {
            k_fft_scale<<<dim3((n + T - 1) / T, nrec), T, 0, s>>>(dre.as<double>(), dim.as<double>(), m);
            ck(cudaGetLastError(), "spectrum kernels");
            ck(cudaMemcpyAsync(re_out, dre.p, sizeof(double) * nrec * n, cudaMemcpyDeviceToHost, s), "spectrum download");
            ck(cudaMemcpyAsync(im_out, dim.p, sizeof(double) * nrec * n, cudaMemcpyDeviceToHost, s), "spectrum download");
        }
        ck(cudaStreamSynchronize(s), "spectrum");
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
}

// 1/n-scaled forward FFT of each zero-padded trace, complex [nrec][n]
void fft_forward(int device, const double* traces, int nrec, int nt, int m, double* re, double* im) {
    run_fft(device, traces, nrec, nt, m, 0, 0, nullptr, re, im);
}

// magnitudes |X_k| (k = k0 .. k0+nk-1) of the zero-padded, 1/n-scaled
// forward FFT of each trace; traces [nrec][nt], mag [nrec][nk] (host)
void spectrum_bins(int device, const double* traces, int nrec, int nt, int m, long k0, long nk, double* mag) {
    run_fft(device, traces, nrec, nt, m, k0, nk, mag, nullptr, nullptr);
}

// Band levels 10 log10(sum |X_k|^2) over the FFT bins whose frequency
// k / (dt 2^m) lies in [fc 2^(-1/6), fc 2^(1/6)) (third-octave bands); a
// band without bins gets -inf. levels [nrec][nband].
void band_levels(int device, const double* traces, int nrec, int nt, int m, double dt, int nband, const double* fc,
                 double* levels) {
    if (nband < 1 || !(dt > 0)) throw SolverError{-5, "band levels: need nband >= 1 and dt > 0"};
    if (m < 1 || m > 24) throw SolverError{-5, "spectrum: need 1 <= fft_m <= 24"};
    const long n = 1L << m;
    const double df = 1.0 / (dt * static_cast<double>(n));
    const double e = std::pow(2.0, 1.0 / 6.0);
    double flo = 1e300, fhi = 0.0;
    for (int b = 0; b < nband; ++b) {
        if (!(fc[b] > 0)) throw SolverError{-5, "band levels: centre frequencies must be positive"};
        flo = std::min(flo, fc[b] / e);
        fhi = std::max(fhi, fc[b] * e);
    }
    const long kmax = n / 2;
    const long k0 = std::min(kmax, static_cast<long>(std::ceil(flo / df)));
    const long k1 = std::min(kmax, static_cast<long>(std::ceil(fhi / df)));  // exclusive
    const long nk = std::max(1L, k1 - k0);
    std::vector<double> mag(static_cast<size_t>(nrec) * nk);
    spectrum_bins(device, traces, nrec, nt, m, k0, nk, mag.data());
    for (int r = 0; r < nrec; ++r)
        for (int b = 0; b < nband; ++b) {
            const double lo = fc[b] / e, hi = fc[b] * e;
            double sum = 0.0;
            for (long k = 0; k < nk; ++k) {
                const double f = static_cast<double>(k0 + k) * df;
                if (f >= lo && f < hi) sum += mag[r * nk + k] * mag[r * nk + k];
            }
            levels[static_cast<size_t>(r) * nband + b] = 10.0 * std::log10(sum);
        }
}

}  // namespace fdtd
