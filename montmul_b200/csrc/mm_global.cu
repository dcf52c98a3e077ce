// Kernel instantiations of global mode (one set for every length 2^12 .. 2^23; the length is a
// kernel argument).
#include "mm_global.cuh"

namespace mm {

GlobalKernels global_kernels() {
    constexpr int NT = 256;
    return GlobalKernels{gstep_kernel<NT>, gmul_kernel<NT>, gsetup_kernel<NT>, NT, kGlobalSmem};
}

}  // namespace mm
