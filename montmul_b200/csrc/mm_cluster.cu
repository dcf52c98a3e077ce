// Kernel instantiations of cluster mode with 8,192-element chunks (L = 32768 and 65536) and the
// launch of every cluster kernel. The 4,096-element-chunk kernel (L = 32768, two blocks per SM,
// 64 registers) lives in mm_cluster_half.cu: its non-inlined passes are compiled there for 64
// registers, leaving these kernels' copies their 128.
#include "mm_cluster.cuh"

namespace mm {


static_assert(kMaxClusterLogN - kChunkLog <= 3, "clusters of at most 8 blocks");
static_assert(kClusterPairChunkLog == kChunkLog - 1, "the second chunk size is the default's half");

int cluster_configure() {
    cudaError_t e = configure_cluster_m<14, kChunkLog>();
    if (e == cudaSuccess) e = configure_cluster_m<15, kChunkLog>();
    if (e == cudaSuccess) e = cluster_half_chunk_configure();
    return (int)e;
}

int cluster_launch(int m, int chunk_log, const SlotArgs& a, uint32_t slots, uint32_t bits, void* stream) {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (chunk_log == kChunkLog) {
        if (m == 14) return (int)launch_cluster_m<14, kChunkLog>(a, slots, bits, s);
        if (m == 15) return (int)launch_cluster_m<15, kChunkLog>(a, slots, bits, s);
    } else if (chunk_log == kClusterPairChunkLog && m == 14) {
        return (int)cluster_half_chunk_launch(a, slots, bits, s);
    }
    return (int)cudaErrorInvalidValue;
}

}  // namespace mm
