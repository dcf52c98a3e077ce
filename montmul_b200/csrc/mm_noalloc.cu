// mm_b200_mul_noalloc: a·b·R^-1 mod N for one modulus of an existing batch, on device buffers
// the caller owns, with every intermediate kept in a fixed static device array instead of
// memory allocated per call or per batch.
//
// It serves callers that cannot allocate device memory when they multiply: services whose
// device memory is owned by their own pool allocator and may not grow behind its back, and
// latency-critical loops that cannot afford the device-wide synchronization cudaFree implies.
//
// The scratch (kNoAllocScratchBytes = 256 KiB: the 2n product limbs and the n-element spectrum
// of the second operand at the largest length this library builds, n = 8192) is a file-scope
// __device__ array, so every GPU that loads the library holds it until the process exits. All
// calls share it: calls that overlap on the GPU (two streams, or two host threads) race on it
// and must be serialized by the caller. Every call overwrites the parts it reads, so nothing is
// carried over from the previous call.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/montmul_b200.h"
#include "mm_kernels.cuh"

namespace mm {

constexpr size_t kNoAllocScratchBytes = 256u << 10;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Bytes of scratch a length-2^(m+1) product needs: T (2n u32) then the spectrum (n F2, n F1).
constexpr size_t noalloc_bytes(int m) { return (size_t)(8 + 24) << m; }
static_assert(noalloc_bytes(kMaxSharedLogN) <= kNoAllocScratchBytes, "scratch too small");

template <int M, int NT>
__global__ void __launch_bounds__(NT) mul_noalloc_kernel(const uint32_t* a, const uint32_t* b, uint32_t* out,
                                                          const F2* cc2, const F1* cc1, const F2K* tab2,
                                                          const F1* tab1, unsigned char* scratch, uint32_t* err) {
    constexpr int N = 1 << M;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * N);
    __shared__ uint64_t sc[CarryScratch<NT>::words];
    uint32_t* tl = reinterpret_cast<uint32_t*>(scratch);                 // 2n limbs
    F2* spec2 = reinterpret_cast<F2*>(scratch + 8 * (size_t)N);          // n elements, 16 B aligned
    F1* spec1 = reinterpret_cast<F1*>(scratch + 24 * (size_t)N);
    fwd_limbs<M, NT>(b, N, s2, s1, tab2, tab1);
    fused_mid<M, NT, false>(b, N, s2, s1, tab2, tab1, SpecStoreOp<M>{spec2, spec1});
    __syncthreads();
    fwd_limbs<M, NT>(a, N, s2, s1, tab2, tab1);
    fused_mid<M, NT, false>(a, N, s2, s1, tab2, tab1, SpecMulOp<M>{spec2, spec1});
    inv_to_natural<M, NT, false>(s2, s1, tab2, tab1);
    bool ok = carry_product<M, NT>(s2, s1, tl, sc) == 0;
    ok &= redc_wrap<M, NT>(s2, s1, tl, out, cc2, cc1, tab2, tab1, sc);
    if (threadIdx.x == 0 && err) *err = ok ? 0u : 1u;
}

typedef void (*NoAllocFn)(const uint32_t*, const uint32_t*, uint32_t*, const F2*, const F1*, const F2K*, const F1*,
                          unsigned char*, uint32_t*);

template <int M> NoAllocFn noalloc_fn() { return mul_noalloc_kernel<M, threads_for(M)>; }

static NoAllocFn noalloc_kernel(int m) {
    switch (m) {
        case 2: return noalloc_fn<2>();
        case 3: return noalloc_fn<3>();
        case 4: return noalloc_fn<4>();
        case 5: return noalloc_fn<5>();
        case 6: return noalloc_fn<6>();
        case 7: return noalloc_fn<7>();
        case 8: return noalloc_fn<8>();
        case 9: return noalloc_fn<9>();
        case 10: return noalloc_fn<10>();
        case 11: return noalloc_fn<11>();
        case 12: return noalloc_fn<12>();
        case 13: return noalloc_fn<13>();
        default: return nullptr;
    }
}

// Device address of the static scratch and the kernels' shared-memory opt-in, once per device.
struct NoAllocDevice {
    unsigned char* scratch = nullptr;
};
static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

static int noalloc_setup(int device, unsigned char** scratch, std::string& msg) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[device];
    if (!d.scratch) {
        // In host code the array's name is only a stand-in; its device address comes from the
        // runtime, with this device current.
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            msg = std::string("mul_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return MM_ERR_CUDA;
        }
        for (int m = kMinLogN; m <= kMaxSharedLogN; ++m) {
            e = cudaFuncSetAttribute((const void*)noalloc_kernel(m), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     smem_bytes_host(m));
            if (e != cudaSuccess) {
                msg = std::string("mul_noalloc: cudaFuncSetAttribute: ") + cudaGetErrorString(e);
                return MM_ERR_CUDA;
            }
        }
        d.scratch = static_cast<unsigned char*>(p);
    }
    *scratch = d.scratch;
    return MM_OK;
}

}  // namespace mm

// Defined in mm_backend.cu: the batch fields this entry point reads, and the error message slot.
extern "C++" int mm_batch_view(const mm_b200_batch* b, int* device, int* m, const mm::F2** c2, const mm::F1** c1,
                               const mm::F2K** tab2, const mm::F1** tab1, size_t* slots);
extern "C++" int mm_set_error(int code, const std::string& msg);
extern "C++" int mm_batch_plain(const mm_b200_batch* b);

extern "C" int mm_b200_mul_noalloc(const mm_b200_batch* b, size_t slot, const uint32_t* d_a, const uint32_t* d_b,
                                   uint32_t* d_out, uint32_t* d_err, void* stream) {
    using namespace mm;
    int device = 0, m = 0;
    const F2* c2 = nullptr;
    const F2K* tab2 = nullptr;
    const F1 *c1 = nullptr, *tab1 = nullptr;
    size_t slots = 0;
    if (!b || !d_a || !d_b || !d_out) return mm_set_error(MM_ERR_ARG, "mul_noalloc: null argument");
    if (mm_batch_plain(b)) return mm_set_error(MM_ERR_UNSUPPORTED, "mul_noalloc: needs the wraparound path (k = L/2)");
    if (int rc = mm_batch_view(b, &device, &m, &c2, &c1, &tab2, &tab1, &slots)) return rc;
    if (slot >= slots) return mm_set_error(MM_ERR_ARG, "mul_noalloc: bad slot");
    if (device < 0 || device >= kNoAllocMaxDevices) return mm_set_error(MM_ERR_ARG, "mul_noalloc: device ordinal too large");
    if (noalloc_bytes(m) > kNoAllocScratchBytes)
        return mm_set_error(MM_ERR_ARG, "mul_noalloc: transform length " + std::to_string(2ull << m) + " needs " +
                                            std::to_string(noalloc_bytes(m)) + " bytes of scratch; the static scratch holds " +
                                            std::to_string(kNoAllocScratchBytes));
    NoAllocFn fn = noalloc_kernel(m);
    if (!fn) return mm_set_error(MM_ERR_UNSUPPORTED, "mul_noalloc: transform length not built");
    // The batch's device becomes current for the call; the caller's current device is restored
    // on every return path.
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return mm_set_error(MM_ERR_CUDA, std::string("mul_noalloc: ") + cudaGetErrorString(e));
    struct Restore {
        int dev, cur;
        ~Restore() { if (cur != dev) cudaSetDevice(dev); }
    } restore{prev, prev};
    if (device != prev) {
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return mm_set_error(MM_ERR_CUDA, std::string("mul_noalloc: ") + cudaGetErrorString(e));
        restore.cur = device;
    }
    unsigned char* scratch = nullptr;
    std::string msg;
    int rc = noalloc_setup(device, &scratch, msg);
    if (rc) return mm_set_error(rc, msg);
    const size_t n = (size_t)1 << m;
    fn<<<1, threads_for(m), smem_bytes_host(m), static_cast<cudaStream_t>(stream)>>>(
        d_a, d_b, d_out, c2 + slot * 2 * n, c1 + slot * 2 * n, tab2, tab1, scratch, d_err);
    e = cudaGetLastError();
    if (e != cudaSuccess) return mm_set_error(MM_ERR_CUDA, std::string("mul_noalloc: launch: ") + cudaGetErrorString(e));
    return MM_OK;
}
