// fft_reg32a.cu -- the FP32 (mixed-precision) register forms of the PME line transforms
// (fft_reg.cuh), first half of the size table.
#include "fft_reg.cuh"

namespace atvb {

bool fftr_launch_32a(int pass, int idx, const ItemList& il, const SysParams* sp,
                     cudaStream_t s) {
    return fftr::launch_half_a<true>(pass, idx, il, sp, s);
}

} // namespace atvb
