// Kernel instantiations of cluster mode (L = 32768 and 65536) and their launch.
#include "mm_cluster.cuh"

namespace mm {

namespace {

template <int M>
cudaError_t launch_cluster_m(const SlotArgs& a, uint32_t slots, uint32_t bits, cudaStream_t s) {
    constexpr int C = 1 << (M - kChunkLog);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * slots, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = kClusterSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, cluster_step_kernel<M>, a, 0u, bits);
}

template <int M>
cudaError_t configure_cluster_m() {
    return cudaFuncSetAttribute((const void*)cluster_step_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kClusterSmem);
}

}  // namespace

static_assert(kMaxClusterLogN - kChunkLog <= 3, "clusters of at most 8 blocks");

int cluster_configure() {
    cudaError_t e = configure_cluster_m<14>();
    if (e == cudaSuccess) e = configure_cluster_m<15>();
    return (int)e;
}

int cluster_launch(int m, const SlotArgs& a, uint32_t slots, uint32_t bits, void* stream) {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (m == 14) return (int)launch_cluster_m<14>(a, slots, bits, s);
    if (m == 15) return (int)launch_cluster_m<15>(a, slots, bits, s);
    return (int)cudaErrorInvalidValue;
}

}  // namespace mm
