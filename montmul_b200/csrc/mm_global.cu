// Kernel instantiations of global mode (one set for every length 2^12 .. 2^23; the length is a
// kernel argument).
#include "mm_global.cuh"

namespace mm {

GlobalKernels global_kernels() {
    constexpr int NT = 256;
    return GlobalKernels{gstep_kernel<NT>, gmul_kernel<NT>, gsetup_kernel<NT>, NT, kGlobalSmem};
}

// Exercises the bounded wait's failure path: one thread arms an mbarrier for a 16-byte copy that
// is never issued (nothing is in flight), so the wait gives up after `limit_ns`, and the time-out
// is recorded in *err as a late bulk copy would be. Launched with one block of 32 threads.
__global__ void wait_check_kernel(uint32_t* err, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        mbar_expect(&bar, 16);
        if (!mbar_wait(&bar, 0, limit_ns)) *err = kErrTimeout;
    }
}

int launch_wait_check(uint32_t* err, uint64_t limit_ns, void* stream) {
    wait_check_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(err, limit_ns);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace mm
