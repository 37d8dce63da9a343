// Two-pass kernels (pressure pass, velocity pass) and the moving-frame row
// shift, instantiated for float and double.
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

template void run_two_pass<float>(bool, bool, dim3, dim3, cudaStream_t, const Dev<float>&, int);
template void run_two_pass<double>(bool, bool, dim3, dim3, cudaStream_t, const Dev<double>&, int);
template void run_shift_rows<float>(cudaStream_t, float*, int, int, int, int, int, int, int);
template void run_shift_rows<double>(cudaStream_t, double*, int, int, int, int, int, int, int);

}  // namespace fdtd
