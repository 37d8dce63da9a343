// fdtd_fb_step_noalloc: one forward-backward step of a rigid-walled air box
// on caller-owned device buffers, with no device allocation of any kind.
//
// Who needs it: code that cannot call cudaMalloc -- a host that hands the
// library pre-allocated buffers from its own memory pool, code running
// while another component owns all allocation, or a caller that must not
// trigger the implicit device synchronisation cudaMalloc/cudaFree perform.
// The handle-based entry points (fdtd_create ...) allocate their own state;
// this one only uses the buffers it is given plus a fixed scratch area
// compiled into the library.
//
// Scratch: the step kernels read per-axis derivative factors, PML side
// flags and two step counters plus a status word from global memory. Here
// they live in g_noalloc_scratch, a file-scope __device__ array of
// kNoAllocScratchBytes (128 KiB) that every GPU loading the library holds
// until the process exits. It bounds each axis to kNoAllocMaxAxis nodes.
// All calls share the array and it keeps the last call's contents: each
// call rewrites the factors and zeroes the counters and status word, so
// calls that overlap on the GPU (different streams, or host threads on one
// device) race on it and must be serialised by the caller.
#include <atomic>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/fdtd_b200.h"
#include "fdtd_device.cuh"

namespace fdtd {
void set_last_error(const char* msg);  // fdtd_capi.cpp
}

namespace {

constexpr int kNoAllocMaxAxis = 4096;
constexpr size_t kNoAllocScratchBytes = 128 * 1024;

// layout (bytes): [0, 3*4096*8) factors x|y|z as R, then 3*4096 int8 side
// flags (all zero: no PML), then 2 step counters + 1 status word
constexpr size_t kFactorBytes = 3 * kNoAllocMaxAxis * sizeof(double);
constexpr size_t kSideBytes = 3 * kNoAllocMaxAxis;
constexpr size_t kCounterOff = kFactorBytes + kSideBytes;
static_assert(kCounterOff + 4 * sizeof(int) <= kNoAllocScratchBytes, "scratch layout");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array per device, resolved once per device
// with that device current (a host-side name of a __device__ symbol is not
// a device address).
std::atomic<unsigned char*> g_scratch_ptr[64] = {};

// per-thread host staging for the axis factors (no heap allocation per call)
thread_local double tl_fac64[3 * kNoAllocMaxAxis];
thread_local float tl_fac32[3 * kNoAllocMaxAxis];

int fail(int code, const char* msg) {
    fdtd::set_last_error(msg);
    return code;
}

int resolve_scratch(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 64) return fail(FDTD_ERR_ARG, "device ordinal out of range");
    unsigned char* p = g_scratch_ptr[dev].load();
    if (!p) {
        void* sym = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&sym, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
        p = static_cast<unsigned char*>(sym);
        g_scratch_ptr[dev].store(p);
    }
    *out = p;
    return FDTD_OK;
}

// x_over_X * rdx for one axis (calculation_2D.cpp:416-433 with zero cross metrics)
template <typename R>
void factors(const double* a, int n, double d, R* f) {
    const double rd = 1.0 / d;
    for (int q = 0; q < kNoAllocMaxAxis; ++q) f[q] = R(0);
    for (int q = 1; q < n - 1; ++q) f[q] = static_cast<R>(rd / ((a[q + 1] - a[q - 1]) * rd * 0.5));
}

template <typename R>
R* staging();
template <>
double* staging<double>() { return tl_fac64; }
template <>
float* staging<float>() { return tl_fac32; }

template <typename R>
int step(int NI, int NJ, int NK, const double* X, const double* Y, const double* Z, double dx, double dy, double dz,
         double dt, double gamma, double P0, double c0, const void* u_in, const void* v_in, const void* w_in,
         const void* p_in, void* u_out, void* v_out, void* w_out, void* p_out, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
    unsigned char* base = nullptr;
    int rc = resolve_scratch(dev, &base);
    if (rc != FDTD_OK) return rc;
    // host staging is pageable; cudaMemcpyAsync copies it out before returning
    R* fac = staging<R>();
    factors<R>(X, NI, dx, fac);
    factors<R>(Y, NJ, dy, fac + kNoAllocMaxAxis);
    factors<R>(Z, NK, dz, fac + 2 * kNoAllocMaxAxis);
    R* dfac = reinterpret_cast<R*>(base);
    int8_t* side = reinterpret_cast<int8_t*>(base + kFactorBytes);
    int* counters = reinterpret_cast<int*>(base + kCounterOff);
    e = cudaMemcpyAsync(dfac, fac, 3 * kNoAllocMaxAxis * sizeof(R), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(side, 0, kSideBytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 3 * sizeof(int), st);  // counters + status start at 0
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));

    fdtd::Dev<R> d{};
    d.NI = NI; d.NJ = NJ; d.NG = NK; d.NJP = NJ;  // caller rows are unpadded
    d.porous = 0; d.gAir0 = 0; d.gOff = 0; d.Kair = NK;
    d.rigid_south = 1; d.tdbc = 0; d.fbvp = 0;
    d.axA = dfac; d.ayA = dfac + kNoAllocMaxAxis; d.azG = dfac + 2 * kNoAllocMaxAxis;
    d.axP = d.axA; d.ayP = d.ayA;
    d.dt = R(dt); d.gP0dt = R(gamma * P0 * dt); d.gdt = R(gamma * dt);
    const double Aav = c0 * c0 / gamma / P0;  // airpore.cpp:177
    d.Aavdt = R(Aav * dt); d.Aav = R(Aav); d.gP0 = R(gamma * P0);
    d.sdI = side; d.sdJ = side + kNoAllocMaxAxis; d.sdK = side + 2 * kNoAllocMaxAxis;
    d.pml_y_time = 0;
    for (auto& s : d.sl) s.ni = 0;
    d.mask = nullptr;
    d.nrec = 0;
    d.counters = counters;
    d.status = counters + 2;
    const dim3 blk(32, 8, 1), grd((NJ + 31) / 32, (NI + 7) / 8, NK);
    // pressure pass: p_out from the old state
    fdtd::Dev<R> dp = d;
    dp.u_in = static_cast<const R*>(u_in); dp.v_in = static_cast<const R*>(v_in); dp.w_in = static_cast<const R*>(w_in);
    dp.pold = static_cast<const R*>(p_in); dp.p_in = dp.pold;
    dp.p_out = static_cast<R*>(p_out);
    fdtd::k_pressure<R, false><<<grd, blk, 0, st>>>(dp, 1);
    // velocity pass: old velocity, new pressure
    fdtd::Dev<R> dv = d;
    dv.u_in = dp.u_in; dv.v_in = dp.v_in; dv.w_in = dp.w_in;
    dv.p_in = static_cast<const R*>(p_out); dv.pold = dp.pold;
    dv.u_out = static_cast<R*>(u_out); dv.v_out = static_cast<R*>(v_out); dv.w_out = static_cast<R*>(w_out);
    fdtd::k_velocity<R, false><<<grd, blk, 0, st>>>(dv, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
    int status = 0;
    e = cudaMemcpyAsync(&status, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
    if (status & 1) return fail(FDTD_ERR_NONFINITE, "pressure became non-finite");
    return FDTD_OK;
}

}  // namespace

extern "C" int fdtd_fb_step_noalloc(int precision, int NI, int NJ, int NK, const double* X, const double* Y,
                                    const double* Z, double dx, double dy, double dz, double dt, double gamma,
                                    double P0, double c0, const void* u_in, const void* v_in, const void* w_in,
                                    const void* p_in, void* u_out, void* v_out, void* w_out, void* p_out,
                                    void* stream) {
    if (!X || !Y || !Z || !u_in || !v_in || !w_in || !p_in || !u_out || !v_out || !w_out || !p_out)
        return fail(FDTD_ERR_ARG, "null pointer argument");
    if (NI < 3 || NJ < 5 || NK < 3) return fail(FDTD_ERR_ARG, "grid needs at least 3 x 5 x 3 nodes");
    if (NI > kNoAllocMaxAxis || NJ > kNoAllocMaxAxis || NK > kNoAllocMaxAxis)
        return fail(FDTD_ERR_ARG, "fdtd_fb_step_noalloc: each axis is limited to 4096 nodes (fixed 128 KiB scratch)");
    if (!(dt > 0) || !(dx > 0) || !(dy > 0) || !(dz > 0) || !(gamma > 0) || !(P0 > 0) || !(c0 > 0))
        return fail(FDTD_ERR_ARG, "non-positive physical parameter");
    if (precision == FDTD_F64 || precision == FDTD_F32) {
        // face nodes read their inward neighbour and the velocity pass reads
        // the old pressure, so an output that shares memory with any input
        // (or another output) would be read after other threads wrote it
        const size_t bytes = static_cast<size_t>(NI) * NJ * NK * (precision == FDTD_F64 ? 8 : 4);
        const void* in[4] = {u_in, v_in, w_in, p_in};
        const void* out[4] = {u_out, v_out, w_out, p_out};
        auto overlap = [bytes](const void* a, const void* b) {
            const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
            return x < y + bytes && y < x + bytes;
        };
        for (int o = 0; o < 4; ++o) {
            for (int q = 0; q < 4; ++q)
                if (overlap(out[o], in[q])) return fail(FDTD_ERR_ARG, "output buffer overlaps an input buffer");
            for (int q = o + 1; q < 4; ++q)
                if (overlap(out[o], out[q])) return fail(FDTD_ERR_ARG, "two output buffers overlap");
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == FDTD_F64)
        return step<double>(NI, NJ, NK, X, Y, Z, dx, dy, dz, dt, gamma, P0, c0, u_in, v_in, w_in, p_in, u_out, v_out,
                            w_out, p_out, st);
    if (precision == FDTD_F32)
        return step<float>(NI, NJ, NK, X, Y, Z, dx, dy, dz, dt, gamma, P0, c0, u_in, v_in, w_in, p_in, u_out, v_out,
                           w_out, p_out, st);
    return fail(FDTD_ERR_ARG, "precision must be FDTD_F64 or FDTD_F32");
}
