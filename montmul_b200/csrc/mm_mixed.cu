// The mixed-length persistent launch: slots of several batches (each batch one transform length)
// run in one launch whose blocks take work items from device counters. One item = every step
// (up to `bits`) of one slot, so a worker stays on a slot until it is done with it and then
// takes the next item; the host orders the items longest first, which bounds the tail of the
// launch by the cost of one of the shortest items.
//
// One block per SM: 512 threads and 192 KiB of dynamic shared memory, launched as clusters of two
// blocks. Each pair first takes the cluster items (L = 32768 batches in cluster mode: the pair
// on one slot, the vector in the two blocks' shared memory, mm_cluster.cuh). Each block then
// takes the wide items (L = 16384 in shared mode: all 512 threads and all of the shared memory on one
// slot), then splits into two groups of 256 threads, each with its own 96 KiB and hardware
// barrier, which take the other items independently: lengths with n <= 4096 with the whole
// vector in shared memory, longer ones (and batches tuned to it) in global mode. There is no
// counterpart in the reference, whose launches each cover one batch of one length
// (montmul/src/gpu/mod.rs:119-158).
#include "mm_cluster.cuh"

namespace mm {

// One slot of a shared-mode batch; one function per length keeps each length's register
// allocation separate from the dispatch.
template <int M>
__device__ __noinline__ void mixed_shared(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem,
                                          uint64_t* sc) {
    step_slot<M, kMixedThreads>(a, slot, bits, smem, sc);
}

__device__ __noinline__ void mixed_wide(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem,
                                        uint64_t* sc) {
    step_slot<kWideLogN, kWideThreads>(a, slot, bits, smem, sc);
}

__device__ __noinline__ void mixed_pair(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem,
                                        uint64_t* sc, ClusterCarry* cc) {
    cl_step_slot<kPairLogN, kWideThreads, kMixedCluster>(a, slot, bits, smem, sc, cc);
}

// gsync / gsync_or (mm_ntt.cuh) give a block at most two groups, and treat a group of 512 or
// more threads as the whole block.
static_assert(kMixedGroups == 2 && kWideThreads == 512, "group barriers: two workers, one wide group");
static_assert(kWideThreads == kClusterThreads && kMixedSmem == kClusterSmem &&
                  (1 << (kPairLogN - kChunkLog)) == kMixedCluster,
              "a block pair holds one cluster item");

constexpr int kGroupScratch = CarryScratch<kMixedThreads>::words;
constexpr int kScratchWords = cmax(kMixedGroups * kGroupScratch, CarryScratch<kWideThreads>::words);

__device__ __forceinline__ uint32_t item_steps(const uint4& it, const MixedDesc& d, uint32_t bits) {
    return it.z ? it.z : (d.bits ? d.bits : bits);
}

__global__ void __launch_bounds__(kMixedBlockThreads, 1)
    mixed_step_kernel(const MixedDesc* __restrict__ descs, MixedLists l, uint32_t bits) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[kScratchWords];
    __shared__ uint64_t bars[kMixedGroups][2];
    __shared__ uint32_t next[kMixedGroups];
    __shared__ uint32_t pair_next;
    __shared__ ClusterCarry cc;
    // Cluster items: the block pair on one slot. Block 0 of the pair takes the item and hands its
    // index to block 1, so both leave the loop together.
    const cgx::cluster_group cl = cgx::this_cluster();
    const uint32_t pair_count = *l.pair_count;
    while (pair_count) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) {
            const uint32_t i = atomicAdd(&l.counter[2], 1u);
            for (int d = 0; d < kMixedCluster; ++d) *cl.map_shared_rank(&pair_next, d) = i;
        }
        cl.sync();
        const uint32_t i = pair_next;
        cl.sync();   // every thread of the pair has read the index before it is replaced
        if (i >= pair_count) break;
        const uint4 it = l.pair[i];
        const MixedDesc& d = descs[it.x];
        SlotArgs a = d.g.a;
        a.tab2 = d.ctab2;
        a.tab1 = d.ctab1;
        mixed_pair(a, it.y, item_steps(it, d, bits), smem_raw, sc, &cc);
    }
    // Wide items: the whole block on one slot.
    const uint32_t wide_count = *l.wide_count;
    while (wide_count) {
        if (threadIdx.x == 0) next[0] = atomicAdd(&l.counter[1], 1u);
        __syncthreads();
        const uint32_t i = next[0];
        __syncthreads();   // every thread has read `next` before thread 0 takes the next item
        if (i >= wide_count) break;
        const uint4 it = l.wide[i];
        const MixedDesc& d = descs[it.x];
        mixed_wide(d.g.a, it.y, item_steps(it, d, bits), smem_raw, sc);
    }
    // The other items: two groups, each on its own slots with its own half of the memory.
    const int grp = threadIdx.x / kMixedThreads;
    unsigned char* gsm = smem_raw + grp * kMixedGroupSmem;
    uint64_t* gsc = sc + grp * kGroupScratch;
    const TileSmem sm{gsm, bars[grp]};
    tile_init<kMixedThreads>(sm);
    uint32_t par = 0;
    const uint32_t count = *l.count;
    for (;;) {
        if (gtid<kMixedThreads>() == 0) next[grp] = atomicAdd(&l.counter[0], 1u);
        gsync<kMixedThreads>();
        const uint32_t i = next[grp];
        gsync<kMixedThreads>();   // the group has read `next` before its thread 0 takes the next item
        if (i >= count) break;
        const uint4 it = l.items[i];
        const MixedDesc& d = descs[it.x];
        const uint32_t steps = item_steps(it, d, bits);
        if (d.global) {
            if (!gstep_slot<kMixedThreads>(d.g, it.y, steps, sm, gsc, par)) break;
            continue;
        }
        switch (d.g.m) {
            case 2: mixed_shared<2>(d.g.a, it.y, steps, gsm, gsc); break;
            case 3: mixed_shared<3>(d.g.a, it.y, steps, gsm, gsc); break;
            case 4: mixed_shared<4>(d.g.a, it.y, steps, gsm, gsc); break;
            case 5: mixed_shared<5>(d.g.a, it.y, steps, gsm, gsc); break;
            case 6: mixed_shared<6>(d.g.a, it.y, steps, gsm, gsc); break;
            case 7: mixed_shared<7>(d.g.a, it.y, steps, gsm, gsc); break;
            case 8: mixed_shared<8>(d.g.a, it.y, steps, gsm, gsc); break;
            case 9: mixed_shared<9>(d.g.a, it.y, steps, gsm, gsc); break;
            case 10: mixed_shared<10>(d.g.a, it.y, steps, gsm, gsc); break;
            case 11: mixed_shared<11>(d.g.a, it.y, steps, gsm, gsc); break;
            case 12: mixed_shared<12>(d.g.a, it.y, steps, gsm, gsc); break;
            default: break;   // the host never builds such a descriptor
        }
    }
}

MixedFn mixed_kernel() { return mixed_step_kernel; }

int mixed_launch(int grid, const MixedDesc* descs, const MixedLists& l, uint32_t bits, void* stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(kMixedBlockThreads, 1, 1);
    cfg.dynamicSmemBytes = kMixedSmem;
    cfg.stream = static_cast<cudaStream_t>(stream);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kMixedCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, mixed_step_kernel, descs, l, bits);
}

int mixed_clusters(int* clusters) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kMixedCluster, 1, 1);
    cfg.blockDim = dim3(kMixedBlockThreads, 1, 1);
    cfg.dynamicSmemBytes = kMixedSmem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kMixedCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaOccupancyMaxActiveClusters(clusters, (const void*)mixed_step_kernel, &cfg);
}

}  // namespace mm
