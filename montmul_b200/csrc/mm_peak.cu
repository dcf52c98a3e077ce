// Integer roofline probe: the peak rate of "butterfly pairs" (one radix-2 butterfly, a GF(p^2)
// product plus an add and a sub, in both GF(M31^2) and GF(M61^2)) with the kernels' own field
// arithmetic (the lazy Karatsuba product and folded add/sub for M61, canonical M31), from
// independent register-resident chains on every SM. The fused step's
// algorithmic work is counted in the same unit, so achieved / peak is its integer-pipe
// roofline fraction.
#include <cuda_runtime.h>

#include "../../include/montmul_b200.h"
#include "mm_field.cuh"

namespace mm {

constexpr int kPeakChains = 4;

__global__ void __launch_bounds__(256) bfly_peak_kernel(int iters, F2* out2, F1* out1) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    F2 u2[kPeakChains], v2[kPeakChains];
    F1 u1[kPeakChains], v1[kPeakChains];
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) {
        u2[c] = f2(t * 7919ull + c, t + 17ull * c + 1);
        v2[c] = f2(t * 104729ull + 3 * c, 5ull + c);
        u1[c] = f1(t * 31u + c, t + 5u * c + 1);
        v1[c] = f1(t * 131u + 3u * c, 7u + c);
    }
    const uint64_t wr = 0x123456789abcdefull & P2, wi = 0x0fedcba987654321ull & P2;
    F2K w2;
    w2.re = wr; w2.im = wi; w2.s = (wr + wi) % P2; w2.d = (wi + P2 - wr) % P2;
    const F1 w1 = f1(0x12345678u, 0x7654321u);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kPeakChains; ++c) {
            const F2 m2 = lkmul(v2[c], w2);
            v2[c] = lcfold(lcsub<2>(u2[c], m2));
            u2[c] = lcfold(lcadd(u2[c], m2));
            const F1 m1 = cmul(v1[c], w1);
            v1[c] = csub(u1[c], m1);
            u1[c] = cadd(u1[c], m1);
        }
    }
    F2 s2 = f2(0, 0);
    F1 s1 = f1(0, 0);
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) {
        s2 = cadd(s2, cadd(lccanon(u2[c]), lccanon(v2[c])));
        s1 = cadd(s1, cadd(u1[c], v1[c]));
    }
    out2[t] = s2;
    out1[t] = s1;
}

}  // namespace mm

extern "C" int mm_b200_bfly_peak(int device, int iters, double* pairs_per_s, double* ms_out) {
    using namespace mm;
    if (!pairs_per_s || iters <= 0) return MM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MM_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return MM_ERR_CUDA;
    const int threads = 256, blocks = sms * 8;
    F2* o2 = nullptr;
    F1* o1 = nullptr;
    if (cudaMalloc(&o2, sizeof(F2) * threads * blocks) != cudaSuccess) return MM_ERR_CUDA;
    if (cudaMalloc(&o1, sizeof(F1) * threads * blocks) != cudaSuccess) { cudaFree(o2); return MM_ERR_CUDA; }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bfly_peak_kernel<<<blocks, threads>>>(iters / 8 + 1, o2, o1);   // warm-up
    cudaEventRecord(a);
    bfly_peak_kernel<<<blocks, threads>>>(iters, o2, o1);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(o2);
    cudaFree(o1);
    if (e != cudaSuccess) return MM_ERR_CUDA;
    *pairs_per_s = (double)threads * blocks * iters * kPeakChains / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return MM_OK;
}
