// Kernel instantiations of one transform length, n = 2^MM_M (the build compiles this file once
// per length so the lengths compile in parallel).
#include "mm_kernels.cuh"

#ifndef MM_M
#error "compile with -DMM_M=<log2 n>"
#endif

namespace mm {

#define MM_CAT2(a, b) a##b
#define MM_CAT(a, b) MM_CAT2(a, b)

template <int M, int NTA>
struct AltStep {
    static StepFn fn() { return step_kernel<M, NTA, alt_min_blocks_for(M)>; }
};
template <int M>
struct AltStep<M, 0> {
    static StepFn fn() { return nullptr; }
};

KernelSet MM_CAT(kernels_m, MM_M)() {
    constexpr int NT = threads_for(MM_M), NTA = alt_threads_for(MM_M);
    return KernelSet{step_kernel<MM_M, NT>, AltStep<MM_M, NTA>::fn(), NTA, mul_kernel<MM_M, NT>, setup_kernel<MM_M, NT>,
                     transform_kernel<MM_M, NT>, NT,
                     smem_bytes<MM_M>()};
}

}  // namespace mm
