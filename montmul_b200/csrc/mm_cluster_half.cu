// Cluster mode at L = 32768 with 4,096-element chunks: a cluster of 4 blocks of 512 threads per
// slot, two blocks per SM (64 registers per thread). A translation unit of its own, so that the
// non-inlined passes it shares with the 8,192-element kernels (mm_cluster.cu, 128 registers) are
// compiled separately for each register budget.
#include "mm_cluster.cuh"

namespace mm {

cudaError_t cluster_half_chunk_configure() { return configure_cluster_m<14, kClusterPairChunkLog>(); }

cudaError_t cluster_half_chunk_launch(const SlotArgs& a, uint32_t slots, uint32_t bits, cudaStream_t s) {
    return launch_cluster_m<14, kClusterPairChunkLog>(a, slots, bits, s);
}

}  // namespace mm
