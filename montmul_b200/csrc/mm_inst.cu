// Kernel instantiations of one transform length, n = 2^MM_M (the build compiles this file once
// per length so the lengths compile in parallel).
#include "mm_kernels.cuh"

#ifndef MM_M
#error "compile with -DMM_M=<log2 n>"
#endif

namespace mm {

#define MM_CAT2(a, b) a##b
#define MM_CAT(a, b) MM_CAT2(a, b)

KernelSet MM_CAT(kernels_m, MM_M)() {
    constexpr int NT = threads_for(MM_M);
    return KernelSet{step_kernel<MM_M, NT>, mul_kernel<MM_M, NT>, setup_kernel<MM_M, NT>, transform_kernel<MM_M, NT>, NT,
                     smem_bytes<MM_M>()};
}

}  // namespace mm
