// Host-visible interface between the backend (mm_backend.cu) and the per-length kernel
// instantiations (mm_inst.cu, compiled once per log2 n): the kernel argument block and the
// table of kernel entry points of one length.
#pragma once
#include <vector_types.h>

#include "mm_common.h"

namespace mm {

// Per-batch device state, structure of arrays over slots.
struct SlotArgs {
    uint32_t* x;          // slots x k limbs, Montgomery form in [0, 2N)
    uint32_t* tbuf;       // slots x 2n limbs: T of the step in flight
    const F2* c2;         // slots x 2n: F(N') in fused-pass order, then A | B
    const F1* c1;
    const uint32_t* exp;  // slots x ew words, most significant bit first
    const uint32_t* nbits;
    uint32_t* pos;
    uint32_t* err;        // set to 1 when a carry that must vanish does not
    const F2K* tab2;      // this length's tables (mm_common.h layout; M61 twiddles in Karatsuba form)
    const F1* tab1;
    uint32_t ew;
    uint32_t base;
    uint32_t bare;        // 1: each step stops after T = c x^2 (x unchanged), as run_bare
    uint32_t k;           // limbs per value (n with the wraparound path; k0 <= n without)
    uint32_t plain;       // 1: REDC without the wraparound path (constants F(N') | F(N))
};

typedef void (*StepFn)(SlotArgs, uint32_t, uint32_t, const uint2*);
typedef void (*MulFn)(SlotArgs, uint32_t, uint32_t, uint32_t, F2*, F1*);
typedef void (*SetupFn)(const uint32_t*, const uint32_t*, F2*, F1*, const F2K*, const F1*, F2, F1, uint32_t,
                        const uint32_t*, uint32_t, int);
typedef void (*TransformFn)(F2*, F1*, const F2K*, const F1*, uint32_t, int);

struct KernelSet {
    StepFn step;
    StepFn step_alt;         // the alternative block shape of this length's step (nullptr: none)
    int threads_alt;
    MulFn mul;
    SetupFn setup;
    TransformFn transform;   // the Transform trait's forward / inverse (shared memory)
    int threads;   // block size
    int smem;      // dynamic shared memory per block
};

// Global mode (kMaxSharedLogN < m <= kMaxGlobalLogN, or forced from m = 12): the same slot
// state plus a per-slot work vector of n elements (F2 then F1 arrays, swizzled order).
struct GArgs {
    SlotArgs a;
    F2* w2;   // slots x n
    F1* w1;
    int m;    // log2 n
};
typedef void (*GStepFn)(GArgs, uint32_t, uint32_t);
typedef void (*GMulFn)(GArgs, uint32_t, uint32_t, uint32_t, F2*, F1*);
typedef void (*GSetupFn)(GArgs, const uint32_t*, const uint32_t*, F2*, F1*, F2, F1, uint32_t, const uint32_t*);   // k, plain in g.a
struct GlobalKernels {
    GStepFn step;
    GMulFn mul;
    GSetupFn setup;
    int threads;
    int smem;
};
constexpr int kMinGlobalLogN = 12;   // smallest length the global kernels accept (one tile per half)
GlobalKernels global_kernels();       // mm_global.cu
// Cluster mode (mm_cluster.cu): L = 32768 and 65536, one thread-block cluster of n / 2^chunk_log
// blocks per slot, 2^chunk_log elements in each: chunk_log 13 (one block per SM) at both
// lengths, or 12 (two blocks per SM) at L = 32768. cluster_configure sets the kernels' shared-
// memory opt-in on the current device; cluster_launch runs `bits` steps on every slot of a batch.
constexpr int kMinClusterLogN = 14;
constexpr int kMaxClusterLogN = 15;
constexpr int kClusterChunkLog = 13;        // the default chunk
constexpr int kClusterPairChunkLog = 12;    // the two-blocks-per-SM chunk, at L = 32768
int cluster_configure();
int cluster_launch(int m, int chunk_log, const SlotArgs& a, uint32_t slots, uint32_t bits, void* stream);
// Enqueues wait_check_kernel (mm_global.cuh) on a stream; non-zero if the launch failed.
int launch_wait_check(uint32_t* err, uint64_t limit_ns, void* stream);   // mm_global.cu

// The mixed-length persistent launch (mm_mixed.cu): one descriptor per batch, one work item
// (descriptor index, slot) per slot. Each block first takes "wide" items (L = 16384 in shared
// mode, the whole block on one slot with the vector in all of its shared memory), then splits
// into groups of kMixedThreads threads that take the other items, each group with its own
// 96 KiB of shared memory; both lists are taken from device counters in list order.
struct MixedDesc {
    GArgs g;        // the batch's slot state (w2 / w1 unused in shared mode)
    int global;     // 1: global mode; 0: the vector in shared memory
    uint32_t bits;  // steps per item of this batch in this launch (0: the launch's `bits`)
    const F2K* ctab2;   // cluster items: the shared-layout tables of the batch's length
    const F1* ctab1;
};
constexpr int kMixedThreads = 256;        // one group: the threads on one slot
constexpr int kMixedGroups = 2;           // groups per block (gsync has barriers for two)
constexpr int kMixedBlockThreads = kMixedThreads * kMixedGroups;
constexpr int kMaxMixedSharedLogN = 12;   // 96 KiB per group, as global mode's tiles
constexpr int kMixedGroupSmem = 24 << kMaxMixedSharedLogN;
constexpr int kMixedSmem = kMixedGroups * kMixedGroupSmem;
constexpr int kWideLogN = kMaxSharedLogN;  // n = 8192: 24 n bytes = all of a block's shared memory
constexpr int kWideThreads = kMixedBlockThreads;
static_assert(kMixedSmem == (24 << kWideLogN), "one wide vector fills the groups' shared memory");
// Items: (descriptor, slot, steps, unused); steps 0 takes the descriptor's, then the launch's.
// The item counts are read from device memory, so one captured launch serves any lists.
// counter[0] counts the group items taken, counter[1] the wide items, counter[2] the cluster
// items. The launch is a cluster launch of block pairs (kMixedCluster): each pair first takes
// cluster items (L = 32768 batches in cluster mode, the pair on one slot, mm_cluster.cuh), then
// its blocks go on independently.
constexpr int kMixedCluster = 2;
constexpr int kPairLogN = 14;
struct MixedLists {
    const uint4* items;
    const uint32_t* count;
    const uint4* wide;
    const uint32_t* wide_count;
    uint32_t* counter;
    const uint4* pair;            // cluster items (L = 32768 in cluster mode): a block pair each
    const uint32_t* pair_count;
};
typedef void (*MixedFn)(const MixedDesc*, MixedLists, uint32_t);
MixedFn mixed_kernel();               // mm_mixed.cu
// The mixed launch on a stream: a cluster launch of `grid` blocks (pairs), grid a multiple of
// kMixedCluster; returns a cudaError_t value. mixed_clusters gives the pairs that fit at once.
int mixed_launch(int grid, const MixedDesc* descs, const MixedLists& l, uint32_t bits, void* stream);
int mixed_clusters(int* clusters);

// Threads per block for transform length 2^m: one radix-8 group per thread up to 256 threads;
// n = 8192 (one block per SM, all of its shared memory) takes 512, which hide more latency.
// n = 4096 takes 512 too: one radix-8 group per thread per pass, 64 registers, two blocks and 32
// warps per SM, measured 5% faster than 256 threads with 128 registers. At the other lengths the
// spills that 64 registers force cost more than the extra warps gain (measured 15-40% slower).
constexpr int threads_for(int m) {
    return m >= kWideLogN || m == 12 ? 512 : (m - 3 <= 5 ? 32 : (m - 3 >= 8 ? 256 : (1 << (m - 3))));
}

// The alternative step-kernel shape a schedule may select per length (threads, minimum blocks per
// SM; 0 threads: none): the runner-up of the shapes measured at full occupancy, 4,096 <= L <= 16,384.
constexpr int alt_threads_for(int m) { return m == 11 ? 256 : (m == 12 ? 256 : (m == 13 ? 1024 : 0)); }
constexpr int alt_min_blocks_for(int m) { return m == 11 ? 4 : (m == 12 ? 2 : 1); }

// Defined in mm_inst.cu for each m in [kMinLogN, kMaxSharedLogN].
#define MM_DECLARE_KERNELS(M) KernelSet kernels_m##M();
MM_DECLARE_KERNELS(2) MM_DECLARE_KERNELS(3) MM_DECLARE_KERNELS(4) MM_DECLARE_KERNELS(5)
MM_DECLARE_KERNELS(6) MM_DECLARE_KERNELS(7) MM_DECLARE_KERNELS(8) MM_DECLARE_KERNELS(9)
MM_DECLARE_KERNELS(10) MM_DECLARE_KERNELS(11) MM_DECLARE_KERNELS(12) MM_DECLARE_KERNELS(13)
#undef MM_DECLARE_KERNELS

}  // namespace mm
