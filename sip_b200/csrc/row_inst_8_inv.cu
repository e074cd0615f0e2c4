// Runtime-radix row kernels, at most 8 points per thread, INVERSE direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_8_inv(int io) { return runtime_row_kernel<8, false>(io); }

}  // namespace sipfft
