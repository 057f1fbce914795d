// fft_reg64b.cu -- the FP64 register forms of the PME line transforms
// (fft_reg.cuh), second half of the size table.
#include "fft_reg.cuh"

namespace atvb {

bool fftr_launch_64b(int pass, int idx, const ItemList& il, const SysParams* sp,
                     cudaStream_t s) {
    return fftr::launch_half_b<false>(pass, idx, il, sp, s);
}

} // namespace atvb
