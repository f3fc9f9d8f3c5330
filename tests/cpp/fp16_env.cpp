// Prints how the C++ drop-in resolves the reference's fp16 storage switch
// (APXCHOL_SPTRSV_FP16, cuda.h:186-205): the tri-state, whether fp16 is
// selected, and the precision setup() picks by default.
#include <cstdio>

#include "apxb200.hpp"

int main() {
    std::printf("%d %d %d\n", apxb::cuda_sptrsv::fp16_env_tristate(), apxb::cuda_sptrsv::fp16_resolved() ? 1 : 0,
                apxb::cuda_sptrsv::default_precision());
    return 0;
}
