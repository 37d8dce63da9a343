// Row marching kernel (one launch = one FB_p_v step of a whole domain) and
// its batched form for ensembles, instantiated for float (2- and 4-column
// vectors) and double (2-column vectors).
#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R, bool XF>
static const void* march_ptr_xf(int VW, bool wind) {
    if constexpr (sizeof(R) == 4) {
        if (VW == 4) return wind ? reinterpret_cast<const void*>(k_march<R, true, 4, XF>)
                                 : reinterpret_cast<const void*>(k_march<R, false, 4, XF>);
    }
    return wind ? reinterpret_cast<const void*>(k_march<R, true, 2, XF>)
                : reinterpret_cast<const void*>(k_march<R, false, 2, XF>);
}

template <typename R>
const void* march_kernel_ptr(int VW, bool wind, bool xf) {
    return xf ? march_ptr_xf<R, true>(VW, wind) : march_ptr_xf<R, false>(VW, wind);
}

template <typename R, bool XF>
static void run_march_xf(int VW, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
                         const MarchTiling& t, int par) {
    if constexpr (sizeof(R) == 4) {
        if (VW == 4) {
            if (wind) k_march<R, true, 4, XF><<<grd, blk, smem, s>>>(d, t, par);
            else k_march<R, false, 4, XF><<<grd, blk, smem, s>>>(d, t, par);
            return;
        }
    }
    if (wind) k_march<R, true, 2, XF><<<grd, blk, smem, s>>>(d, t, par);
    else k_march<R, false, 2, XF><<<grd, blk, smem, s>>>(d, t, par);
}

template <typename R>
void run_march(int VW, bool wind, bool xf, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const Dev<R>& d,
               const MarchTiling& t, int par) {
    if (xf) run_march_xf<R, true>(VW, wind, grd, blk, smem, s, d, t, par);
    else run_march_xf<R, false>(VW, wind, grd, blk, smem, s, d, t, par);
}

template <typename R, bool XF>
static const void* batch_ptr_xf(int VW, bool wind) {
    if constexpr (sizeof(R) == 4) {
        if (VW == 4) return wind ? reinterpret_cast<const void*>(k_march_batch<R, true, 4, XF>)
                                 : reinterpret_cast<const void*>(k_march_batch<R, false, 4, XF>);
    }
    return wind ? reinterpret_cast<const void*>(k_march_batch<R, true, 2, XF>)
                : reinterpret_cast<const void*>(k_march_batch<R, false, 2, XF>);
}

template <typename R>
const void* march_batch_kernel_ptr(int VW, bool wind, bool xf) {
    return xf ? batch_ptr_xf<R, true>(VW, wind) : batch_ptr_xf<R, false>(VW, wind);
}

template <typename R, bool XF>
static void run_batch_xf(int VW, bool wind, dim3 grd, dim3 blk, size_t smem, cudaStream_t s, const BatchWork* work,
                         const BatchEntry<R>* entries, int nm, int phase) {
    if constexpr (sizeof(R) == 4) {
        if (VW == 4) {
            if (wind) k_march_batch<R, true, 4, XF><<<grd, blk, smem, s>>>(work, entries, nm, phase);
            else k_march_batch<R, false, 4, XF><<<grd, blk, smem, s>>>(work, entries, nm, phase);
            return;
        }
    }
    if (wind) k_march_batch<R, true, 2, XF><<<grd, blk, smem, s>>>(work, entries, nm, phase);
    else k_march_batch<R, false, 2, XF><<<grd, blk, smem, s>>>(work, entries, nm, phase);
}

template <typename R>
void run_march_batch(int VW, bool wind, bool xf, dim3 grd, dim3 blk, size_t smem, cudaStream_t s,
                     const BatchWork* work, const BatchEntry<R>* entries, int nm, int phase) {
    if (xf) run_batch_xf<R, true>(VW, wind, grd, blk, smem, s, work, entries, nm, phase);
    else run_batch_xf<R, false>(VW, wind, grd, blk, smem, s, work, entries, nm, phase);
}

#define FDTD_INST(R)                                                                                            \
    template const void* march_kernel_ptr<R>(int, bool, bool);                                                 \
    template void run_march<R>(int, bool, bool, dim3, dim3, size_t, cudaStream_t, const Dev<R>&,              \
                               const MarchTiling&, int);                                                       \
    template const void* march_batch_kernel_ptr<R>(int, bool, bool);                                           \
    template void run_march_batch<R>(int, bool, bool, dim3, dim3, size_t, cudaStream_t, const BatchWork*,      \
                                     const BatchEntry<R>*, int, int);
FDTD_INST(float)
FDTD_INST(double)
#undef FDTD_INST

}  // namespace fdtd
