// Runtime-radix row kernels, at most 8 points per thread, FORWARD direction.
#include "row_fft_inst.cuh"

namespace sipfft {

const void *runtime_row_kernel_8_fwd(int io) { return runtime_row_kernel<8, true>(io); }

}  // namespace sipfft
