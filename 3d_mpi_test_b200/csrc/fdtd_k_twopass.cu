// Two-pass kernels (pressure pass, velocity pass), the moving-frame row
// shift and the impedance-ground update, instantiated for float and double.
#include "fdtd_kernels.hpp"

namespace fdtd {

template <typename R>
void run_two_pass(bool pressure, bool wind, dim3 grd, dim3 blk, cudaStream_t s, const Dev<R>& d, int code) {
    if (pressure) {
        if (wind) k_pressure<R, true><<<grd, blk, 0, s>>>(d, code);
        else k_pressure<R, false><<<grd, blk, 0, s>>>(d, code);
    } else {
        if (wind) k_velocity<R, true><<<grd, blk, 0, s>>>(d, code);
        else k_velocity<R, false><<<grd, blk, 0, s>>>(d, code);
    }
}

template <typename R>
void run_shift_rows(cudaStream_t s, R* a, int rows, int nj, int sh, int lead, int tempJ, int J, int west_copy) {
    k_shift_rows<R><<<(rows + 127) / 128, 128, 0, s>>>(a, rows, nj, sh, lead, tempJ, J, west_copy);
}

template <typename R>
void run_ground_tdbc(cudaStream_t s, const Dev<R>& d, const GroundC& gc, int par) {
    const dim3 blk(32, 8, 1);
    const dim3 grd((d.NJ - 2 + 31) / 32, (d.NI - 2 + 7) / 8, 1);
    k_ground_tdbc<R><<<grd, blk, 0, s>>>(d, gc, par);
}

template void run_two_pass<float>(bool, bool, dim3, dim3, cudaStream_t, const Dev<float>&, int);
template void run_two_pass<double>(bool, bool, dim3, dim3, cudaStream_t, const Dev<double>&, int);
template void run_shift_rows<float>(cudaStream_t, float*, int, int, int, int, int, int, int);
template void run_shift_rows<double>(cudaStream_t, double*, int, int, int, int, int, int, int);
template void run_ground_tdbc<float>(cudaStream_t, const Dev<float>&, const GroundC&, int);
template void run_ground_tdbc<double>(cudaStream_t, const Dev<double>&, const GroundC&, int);

}  // namespace fdtd
