// The Transform trait of the reference (montmul/src/transform.rs:22-46), as its Gpu backend
// implements it (gpu/mod.rs:286-319): buffers of `count` vectors of L/2 elements in GF(M31^2) x
// GF(M61^2), batched forward (weight by zeta^j, DIF), inverse (DIT, unweight by zeta^-j / n)
// and pointwise products with per-vector scales. Lengths up to L = 16,384 transform one vector
// per block in shared memory; longer ones in global mode (passes over device memory plus
// bulk-copied shared-memory tiles).
//
// On the device a vector keeps the kernels' element order (element j at swz(j), a permutation
// within aligned 16-element blocks); the host applies and removes it on upload and download, so
// mm_b200_t_download_raw returns the reference's element order.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/montmul_b200.h"
#include "mm_global.cuh"
#include "mm_host.hpp"

using namespace mm;

// Defined in mm_backend.cu.
extern "C++" int mm_set_error(int code, const std::string& msg);
extern "C++" int mm_device_tables(mm_b200_device* dev, int m, bool global, const F2K** t2, const F1** t1,
                                  KernelSet* ks, GlobalKernels* gk);
extern "C++" int mm_device_ordinal(const mm_b200_device* dev);

struct mm_b200_tbuf {
    mm_b200_device* dev = nullptr;
    size_t len = 0, count = 0, n = 0;
    F2* d2 = nullptr;
    F1* d1 = nullptr;
};

namespace {

#define TK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return mm_set_error(MM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int swz_host(int e) { return swz_c(e); }

int log2_len(size_t len) {
    int l = 0;
    while (((size_t)1 << l) < len) ++l;
    return ((size_t)1 << l) == len ? l : -1;
}

// out = scale a b per element (cpu.rs:395-407): canonical GF(p^2) products; the scale of vector
// v is scales[v] (reduced mod M31 for the M31 part), or 1.
__global__ void pointwise_kernel(F2* o2, F1* o1, const F2* a2, const F1* a1, const F2* b2, const F1* b1,
                                 const uint32_t* scales, int logn, size_t total) {
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        F2 x = cmul(a2[e], b2[e]);
        F1 y = cmul(a1[e], b1[e]);
        const uint32_t c = scales ? scales[e >> logn] : 1u;
        if (c != 1) {
            x = cmul_r((uint64_t)c, x);
            y = cmul_r(c % P1, y);
        }
        o2[e] = x;
        o1[e] = y;
    }
}

int check_buf(const mm_b200_tbuf* b, size_t len, size_t count, const char* what) {
    if (!b) return mm_set_error(MM_ERR_ARG, std::string(what) + ": null buffer");
    if (b->len != len || b->count < count)
        return mm_set_error(MM_ERR_ARG, std::string(what) + ": buffer holds " + std::to_string(b->count) +
                                            " vectors of length " + std::to_string(b->len));
    return MM_OK;
}

int transform(mm_b200_tbuf* b, size_t len, size_t count, bool inverse) {
    const char* what = inverse ? "t_inverse" : "t_forward";
    int rc = check_buf(b, len, count, what);
    if (rc || count == 0) return rc;
    const int m = log2_len(len) - 1;
    TK(cudaSetDevice(mm_device_ordinal(b->dev)));
    const bool global = m > kMaxSharedLogN;
    const F2K* t2 = nullptr;
    const F1* t1 = nullptr;
    KernelSet ks{};
    GlobalKernels gk{};
    rc = mm_device_tables(b->dev, m, global, &t2, &t1, &ks, &gk);
    if (rc) return rc;
    uint32_t* d_err = nullptr;
    if (global) {
        TK(cudaFuncSetAttribute((const void*)gtransform_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGlobalSmem));
        TK(cudaMalloc(&d_err, 4));
        TK(cudaMemset(d_err, 0, 4));
    }
    for (size_t v0 = 0; v0 < count; v0 += 65535) {
        const unsigned grid = (unsigned)std::min<size_t>(65535, count - v0);
        if (global)
            gtransform_kernel<256><<<grid, 256, kGlobalSmem>>>(b->d2, b->d1, t2, t1, m, (uint32_t)v0, inverse ? 1 : 0, d_err);
        else
            ks.transform<<<grid, ks.threads, ks.smem>>>(b->d2, b->d1, t2, t1, (uint32_t)v0, inverse ? 1 : 0);
        TK(cudaGetLastError());
    }
    TK(cudaDeviceSynchronize());
    if (global) {
        uint32_t err = 0;
        TK(cudaMemcpy(&err, d_err, 4, cudaMemcpyDeviceToHost));
        TK(cudaFree(d_err));
        if (err) return mm_set_error(MM_ERR_CUDA, std::string(what) + ": a bulk copy did not complete within its time limit");
    }
    return MM_OK;
}

}  // namespace

extern "C" {

int mm_b200_t_upload(mm_b200_device* dev, const uint32_t* coeffs, size_t len, size_t count, mm_b200_tbuf** out) {
    if (!dev || !out || (!coeffs && count)) return mm_set_error(MM_ERR_ARG, "t_upload: null argument");
    const int l = log2_len(len);
    if (l < 3 || l > kMaxGlobalLogN + 1) return mm_set_error(MM_ERR_ARG, "t_upload: length must be a power of two in 8 .. 2^24");
    const size_t n = len / 2;
    TK(cudaSetDevice(mm_device_ordinal(dev)));
    // upload (cpu.rs:349-358): coefficient j in the real part of element j, j + n in the imaginary
    // part, as field values (mod M31, and as they are for M61).
    std::vector<F2> h2(count * n);
    std::vector<F1> h1(count * n);
    for (size_t v = 0; v < count; ++v) {
        const uint32_t* c = coeffs + v * len;
        for (size_t j = 0; j < n; ++j) {
            const size_t at = v * n + (size_t)swz_host((int)j);
            h2[at] = F2{c[j], c[j + n]};
            h1[at] = F1{c[j] % P1, c[j + n] % P1};
        }
    }
    std::unique_ptr<mm_b200_tbuf> b(new mm_b200_tbuf());
    b->dev = dev;
    b->len = len;
    b->count = count;
    b->n = n;
    TK(cudaMalloc(&b->d2, std::max<size_t>(1, count * n) * sizeof(F2)));
    TK(cudaMalloc(&b->d1, std::max<size_t>(1, count * n) * sizeof(F1)));
    if (count) {
        TK(cudaMemcpy(b->d2, h2.data(), count * n * sizeof(F2), cudaMemcpyHostToDevice));
        TK(cudaMemcpy(b->d1, h1.data(), count * n * sizeof(F1), cudaMemcpyHostToDevice));
    }
    *out = b.release();
    return MM_OK;
}

int mm_b200_t_download_raw(const mm_b200_tbuf* b, uint32_t* f1, uint64_t* f2) {
    if (!b || (!f1 && !f2)) return mm_set_error(MM_ERR_ARG, "t_download_raw: null argument");
    TK(cudaSetDevice(mm_device_ordinal(b->dev)));
    const size_t total = b->count * b->n;
    std::vector<F2> h2(total);
    std::vector<F1> h1(total);
    if (total) {
        TK(cudaMemcpy(h2.data(), b->d2, total * sizeof(F2), cudaMemcpyDeviceToHost));
        TK(cudaMemcpy(h1.data(), b->d1, total * sizeof(F1), cudaMemcpyDeviceToHost));
    }
    for (size_t v = 0; v < b->count; ++v)
        for (size_t j = 0; j < b->n; ++j) {
            const size_t at = v * b->n + (size_t)swz_host((int)j), to = v * b->n + j;
            if (f2) {
                f2[2 * to] = h2[at].re;
                f2[2 * to + 1] = h2[at].im;
            }
            if (f1) {
                f1[2 * to] = h1[at].re;
                f1[2 * to + 1] = h1[at].im;
            }
        }
    return MM_OK;
}

int mm_b200_t_forward(mm_b200_tbuf* b, size_t len, size_t count) { return transform(b, len, count, false); }
int mm_b200_t_inverse(mm_b200_tbuf* b, size_t len, size_t count) { return transform(b, len, count, true); }

int mm_b200_t_pointwise(mm_b200_tbuf* out, const mm_b200_tbuf* a, const mm_b200_tbuf* bb, const uint32_t* scales,
                        size_t len, size_t count) {
    int rc = check_buf(out, len, count, "t_pointwise");
    if (!rc) rc = check_buf(a, len, count, "t_pointwise");
    if (!rc) rc = check_buf(bb, len, count, "t_pointwise");
    if (rc || count == 0) return rc;
    TK(cudaSetDevice(mm_device_ordinal(out->dev)));
    uint32_t* d_sc = nullptr;
    if (scales) {
        TK(cudaMalloc(&d_sc, count * 4));
        TK(cudaMemcpy(d_sc, scales, count * 4, cudaMemcpyHostToDevice));
    }
    const size_t total = count * out->n;
    const int logn = log2_len(out->n);
    const unsigned grid = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
    pointwise_kernel<<<grid, 256>>>(out->d2, out->d1, a->d2, a->d1, bb->d2, bb->d1, d_sc, logn, total);
    TK(cudaGetLastError());
    TK(cudaDeviceSynchronize());
    if (d_sc) TK(cudaFree(d_sc));
    return MM_OK;
}

int mm_b200_t_load_forward(mm_b200_device* dev, const uint32_t* limbs, size_t k, size_t len, size_t count,
                           mm_b200_tbuf** out) {
    if (!dev || !out || (!limbs && count && k)) return mm_set_error(MM_ERR_ARG, "t_load_forward: null argument");
    if (k > len) return mm_set_error(MM_ERR_ARG, "t_load_forward: more limbs than coefficients");
    std::vector<uint32_t> padded(count * len, 0u);
    for (size_t v = 0; v < count; ++v) std::memcpy(padded.data() + v * len, limbs + v * k, k * 4);
    int rc = mm_b200_t_upload(dev, padded.data(), len, count, out);
    if (rc) return rc;
    rc = mm_b200_t_forward(*out, len, count);
    if (rc) {
        mm_b200_t_free(*out);
        *out = nullptr;
    }
    return rc;
}

size_t mm_b200_t_count(const mm_b200_tbuf* b) { return b ? b->count : 0; }
size_t mm_b200_t_len(const mm_b200_tbuf* b) { return b ? b->len : 0; }

void mm_b200_t_free(mm_b200_tbuf* b) {
    if (!b) return;
    cudaSetDevice(mm_device_ordinal(b->dev));
    cudaFree(b->d2);
    cudaFree(b->d1);
    delete b;
}

}  // extern "C"
