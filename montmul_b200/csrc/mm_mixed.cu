// The mixed-length persistent launch: slots of several batches (each batch one transform length)
// run in one launch whose blocks take work items from a device counter. One item = every step
// (up to `bits`) of one slot, so a block stays on a slot until it is done with it and then
// takes the next item; the host orders the items longest first, which bounds the tail of the
// launch by the cost of one of the shortest items.
//
// Every block has 256 threads and 96 KiB of dynamic shared memory (two blocks per SM): lengths
// with n <= 4096 run with the whole vector in shared memory, longer ones in global mode. There
// is no counterpart in the reference, whose launches each cover one batch of one length
// (montmul/src/gpu/mod.rs:119-158).
#include "mm_global.cuh"

namespace mm {

// One slot of a shared-mode batch; one function per length keeps each length's register
// allocation separate from the dispatch.
template <int M>
__device__ __noinline__ void mixed_shared(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem_raw,
                                          uint64_t* sc) {
    step_slot<M, kMixedThreads>(a, slot, bits, smem_raw, sc);
}

__global__ void __launch_bounds__(kMixedThreads, 2)
    mixed_step_kernel(const MixedDesc* __restrict__ descs, const uint4* __restrict__ items,
                      const uint32_t* __restrict__ count_ptr, uint32_t* counter, uint32_t bits) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[CarryScratch<kMixedThreads>::words];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t next;
    const TileSmem sm{smem_raw, bars};
    tile_init(sm);
    uint32_t par = 0;
    const uint32_t count = *count_ptr;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t i = next;
        __syncthreads();   // every thread has read `next` before thread 0 takes the next item
        if (i >= count) break;
        const uint4 it = items[i];
        const MixedDesc& d = descs[it.x];
        const uint32_t steps = it.z ? it.z : (d.bits ? d.bits : bits);
        if (d.global) {
            if (!gstep_slot<kMixedThreads>(d.g, it.y, steps, sm, sc, par)) break;
            continue;
        }
        switch (d.g.m) {
            case 2: mixed_shared<2>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 3: mixed_shared<3>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 4: mixed_shared<4>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 5: mixed_shared<5>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 6: mixed_shared<6>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 7: mixed_shared<7>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 8: mixed_shared<8>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 9: mixed_shared<9>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 10: mixed_shared<10>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 11: mixed_shared<11>(d.g.a, it.y, steps, smem_raw, sc); break;
            case 12: mixed_shared<12>(d.g.a, it.y, steps, smem_raw, sc); break;
            default: break;   // the host never builds such a descriptor
        }
    }
}

MixedFn mixed_kernel() { return mixed_step_kernel; }

}  // namespace mm
