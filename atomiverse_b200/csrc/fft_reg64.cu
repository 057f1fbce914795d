// fft_reg64.cu -- the FP64 register forms of the PME line transforms
// (fft_reg.cuh), and the size table the engine consults.
#include "fft_reg.cuh"

namespace atvb {

void launch_fft_reg32(int pass, int idx, const ItemList& il, const SysParams* sp,
                      cudaStream_t s);

int fft_reg_index(int n) {
    switch (n) {
#define ATVB_FFTR_IDX(i, len, a, b)                                                     \
    case len: return i;
        ATVB_FFTR_SIZES(ATVB_FFTR_IDX)
#undef ATVB_FFTR_IDX
    default: return -1;
    }
}

int fft_reg_lines(int idx, bool mixed) {
    switch (idx) {
#define ATVB_FFTR_LINES(i, len, a, b)                                                   \
    case i: return mixed ? fftr::Shape<a, b>::zlines<true>() : fftr::Shape<a, b>::zlines<false>();
        ATVB_FFTR_SIZES(ATVB_FFTR_LINES)
#undef ATVB_FFTR_LINES
    default: return 1;
    }
}

int fft_reg_cols(bool mixed) { return mixed ? fftr::cols<true>() : fftr::cols<false>(); }

void launch_fft_reg(int pass, int idx, bool mixed, const ItemList& il, const SysParams* sp,
                    cudaStream_t s) {
    if (il.n == 0)
        return;
    if (mixed)
        launch_fft_reg32(pass, idx, il, sp, s);
    else
        fftr::launch_any<false>(pass, idx, il, sp, s);
}

} // namespace atvb
