// C-ABI implementation of the B200 backend (include/montmul_b200.h): device and batch state,
// host-side caches of x and exponents (as gpu/mod.rs:161-176, 238-270 of the reference), the
// launch of the fused step kernels, and error reporting by status code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/montmul_b200.h"
#include "mm_host.hpp"
#include "mm_abi.h"

using namespace mm;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define MM_CK(call)                                                                            \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(MM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool kernel_set(int m, KernelSet& ks) {
    switch (m) {
        case 2: ks = kernels_m2(); return true;
        case 3: ks = kernels_m3(); return true;
        case 4: ks = kernels_m4(); return true;
        case 5: ks = kernels_m5(); return true;
        case 6: ks = kernels_m6(); return true;
        case 7: ks = kernels_m7(); return true;
        case 8: ks = kernels_m8(); return true;
        case 9: ks = kernels_m9(); return true;
        case 10: ks = kernels_m10(); return true;
        case 11: ks = kernels_m11(); return true;
        case 12: ks = kernels_m12(); return true;
        case 13: ks = kernels_m13(); return true;
        default: return false;
    }
}

struct DevTables {
    F2K* t2 = nullptr;
    F1* t1 = nullptr;
    F2 inv8h2;
    F1 inv8h1;
};

int log2_exact(size_t v) {
    int l = 0;
    while (((size_t)1 << l) < v) ++l;
    return ((size_t)1 << l) == v ? l : -1;
}

}  // namespace

struct mm_b200_device {
    int device = 0;
    int sms = 0;
    int max_smem = 0;
    int max_launch_steps = 512;
    bool force_global = false;
    bool wrap = true;          // GpuOptions::wraparound (k = L/2); off: k = k0 and the plain REDC
    bool global_configured = false;
    bool mixed_configured = false;
    bool cluster_configured = false;
    std::string name;
    std::mutex mu;
    std::map<int, DevTables> tables;
    std::map<int, bool> configured;
};

struct mm_b200_batch {
    mm_b200_device* dev = nullptr;
    int m = 0;
    size_t k = 0, n = 0, slots = 0;
    uint32_t base = 3;
    KernelSet ks{};
    StepFn step_fn = nullptr;  // the step kernel of the schedule's block shape (ks.step or ks.step_alt)
    int step_threads = 0;
    bool global = false;       // vector in HBM, tiles through shared memory (mm_global.cuh)
    bool cluster = false;      // global batch stepped in cluster mode (mm_cluster.cuh)
    int cluster_chunk_log = kClusterChunkLog;   // elements per block of the cluster: 2^13 or 2^12
    const DevTables* ctab = nullptr;   // shared-layout tables of a cluster-mode length
    bool plain = false;        // REDC without the wraparound path (k may be below L/2)
    GlobalKernels gk{};
    F2* d_w2 = nullptr;        // global mode: slots x n work elements
    F1* d_w1 = nullptr;
    const DevTables* gtab = nullptr;   // global-mode tables (global batches)
    mm_b200_schedule sched{0, 0, 0.0, 0};
    uint32_t* d_stage = nullptr;       // refill staging: device words and pinned host words
    size_t stage_cap = 0;
    uint32_t* h_stage = nullptr;
    cudaEvent_t stage_copied = nullptr;   // the last host-to-device copy out of h_stage
    size_t hstage_cap = 0;
    cudaStream_t stream = nullptr;
    uint32_t* d_x = nullptr;
    uint32_t* d_t = nullptr;
    F2* d_c2 = nullptr;
    F1* d_c1 = nullptr;
    uint32_t* d_exp = nullptr;
    uint32_t* d_nbits = nullptr;
    uint32_t* d_pos = nullptr;
    uint32_t* d_err = nullptr;
    F2* d_spec2 = nullptr;
    F1* d_spec1 = nullptr;
    size_t ew = 0, exp_cap = 0;
    const DevTables* tab = nullptr;
    uint32_t* host_x = nullptr;    // pinned, slots x k
    size_t host_x_len = 0;
    uint32_t* host_exp = nullptr;  // pinned staging of the exponent words, nbits and pos
    size_t host_exp_cap = 0;
    bool host_x_valid = true;
    bool device_x_stale = false;
    std::vector<std::vector<uint32_t>> exps;
    std::vector<uint32_t> nbits, pos;
    bool exp_dirty = false;
    uint64_t launches = 0;
    uint2* d_items = nullptr;          // run_items: the list on the device and its pinned staging
    uint2* h_items = nullptr;
    cudaEvent_t items_copied = nullptr;   // the staging may be rewritten once this has passed
};

namespace {

// Tables of length 2^(m+1) in the layout of the shared-memory kernels or of global mode.
int ensure_tables(mm_b200_device* dev, int m, bool global, const DevTables** out) {
    std::lock_guard<std::mutex> lock(dev->mu);
    const int key = global ? 100 + m : m;
    auto it = dev->tables.find(key);
    if (it == dev->tables.end()) {
        std::vector<F2K> t2 = host::karatsuba_form(global ? host::gen_global_length_tables<F2>(m) : host::gen_length_tables<F2>(m));
        std::vector<F1> t1 = global ? host::gen_global_length_tables<F1>(m) : host::gen_length_tables<F1>(m);
        DevTables d;
        MM_CK(cudaMalloc(&d.t2, t2.size() * sizeof(F2K)));
        MM_CK(cudaMalloc(&d.t1, t1.size() * sizeof(F1)));
        MM_CK(cudaMemcpy(d.t2, t2.data(), t2.size() * sizeof(F2K), cudaMemcpyHostToDevice));
        MM_CK(cudaMemcpy(d.t1, t1.data(), t1.size() * sizeof(F1), cudaMemcpyHostToDevice));
        d.inv8h2 = host::inv8h<F2>(m);
        d.inv8h1 = host::inv8h<F1>(m);
        it = dev->tables.emplace(key, d).first;
    }
    if (global && !dev->global_configured) {
        const GlobalKernels gk = global_kernels();
        MM_CK(cudaFuncSetAttribute((const void*)gk.step, cudaFuncAttributeMaxDynamicSharedMemorySize, gk.smem));
        MM_CK(cudaFuncSetAttribute((const void*)gk.mul, cudaFuncAttributeMaxDynamicSharedMemorySize, gk.smem));
        MM_CK(cudaFuncSetAttribute((const void*)gk.setup, cudaFuncAttributeMaxDynamicSharedMemorySize, gk.smem));
        MM_CK(cudaFuncSetAttribute((const void*)gk.step, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
        dev->global_configured = true;
    }
    if (!global && m <= kMaxSharedLogN && !dev->configured[m]) {
        KernelSet ks;
        kernel_set(m, ks);
        MM_CK(cudaFuncSetAttribute((const void*)ks.step, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
        MM_CK(cudaFuncSetAttribute((const void*)ks.mul, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
        MM_CK(cudaFuncSetAttribute((const void*)ks.setup, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
        MM_CK(cudaFuncSetAttribute((const void*)ks.transform, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
        MM_CK(cudaFuncSetAttribute((const void*)ks.step, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
        if (ks.step_alt) {
            MM_CK(cudaFuncSetAttribute((const void*)ks.step_alt, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
            MM_CK(cudaFuncSetAttribute((const void*)ks.step_alt, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       cudaSharedmemCarveoutMaxShared));
        }
        dev->configured[m] = true;
    }
    *out = &it->second;
    return MM_OK;
}

GArgs global_args(const mm_b200_batch* b);

SlotArgs slot_args(const mm_b200_batch* b) {
    SlotArgs a;
    a.x = b->d_x;
    a.tbuf = b->d_t;
    a.c2 = b->d_c2;
    a.c1 = b->d_c1;
    a.exp = b->d_exp;
    a.nbits = b->d_nbits;
    a.pos = b->d_pos;
    a.err = b->d_err;
    a.tab2 = b->tab->t2;
    a.tab1 = b->tab->t1;
    a.ew = (uint32_t)b->ew;
    a.base = b->base;
    a.bare = 0;
    a.k = (uint32_t)b->k;
    a.plain = b->plain ? 1 : 0;
    return a;
}

// Requires the batch's global-mode tables (a global batch, or ensure_global_buffers).
GArgs global_args(const mm_b200_batch* b) {
    GArgs g;
    g.a = slot_args(b);
    g.a.tab2 = b->gtab->t2;
    g.a.tab1 = b->gtab->t1;
    g.w2 = b->d_w2;
    g.w1 = b->d_w1;
    g.m = b->m;
    return g;
}

int pull_x(mm_b200_batch* b) {
    if (b->host_x_valid) return MM_OK;
    MM_CK(cudaMemcpyAsync(b->host_x, b->d_x, b->host_x_len * 4, cudaMemcpyDeviceToHost, b->stream));
    MM_CK(cudaStreamSynchronize(b->stream));
    b->host_x_valid = true;
    return MM_OK;
}

// Uploads host-side changes (loaded values, exponents) before a launch (gpu/mod.rs:161-176).
int push(mm_b200_batch* b) {
    if (b->device_x_stale) {
        MM_CK(cudaMemcpyAsync(b->d_x, b->host_x, b->host_x_len * 4, cudaMemcpyHostToDevice, b->stream));
        b->device_x_stale = false;
    }
    if (b->exp_dirty) {
        size_t ew = 1;
        for (auto& e : b->exps) ew = std::max(ew, e.size());
        // The staging buffer may still feed a copy of the previous push.
        MM_CK(cudaStreamSynchronize(b->stream));
        const size_t need = b->slots * (ew + 2);
        if (need > b->host_exp_cap) {
            if (b->host_exp) MM_CK(cudaFreeHost(b->host_exp));
            b->host_exp = nullptr;
            MM_CK(cudaMallocHost(&b->host_exp, need * 4));
            b->host_exp_cap = need;
        }
        uint32_t* words = b->host_exp;
        std::memset(words, 0, b->slots * ew * 4);
        for (size_t i = 0; i < b->slots; ++i)
            std::copy(b->exps[i].begin(), b->exps[i].end(), words + i * ew);
        std::memcpy(words + b->slots * ew, b->nbits.data(), b->slots * 4);
        std::memcpy(words + b->slots * (ew + 1), b->pos.data(), b->slots * 4);
        if (ew > b->exp_cap) {
            if (b->d_exp) MM_CK(cudaFree(b->d_exp));
            MM_CK(cudaMalloc(&b->d_exp, b->slots * ew * 4));
            b->exp_cap = ew;
        }
        b->ew = ew;
        MM_CK(cudaMemcpyAsync(b->d_exp, words, b->slots * ew * 4, cudaMemcpyHostToDevice, b->stream));
        MM_CK(cudaMemcpyAsync(b->d_nbits, words + b->slots * ew, b->slots * 4, cudaMemcpyHostToDevice, b->stream));
        MM_CK(cudaMemcpyAsync(b->d_pos, words + b->slots * (ew + 1), b->slots * 4, cudaMemcpyHostToDevice, b->stream));
        b->exp_dirty = false;
    }
    return MM_OK;
}

// Names the first slot whose error word is set, after clearing the words (gpu/mod.rs:178-184).
int check_err(mm_b200_batch* b, const char* what) {
    std::vector<uint32_t> err(b->slots);
    MM_CK(cudaMemcpyAsync(err.data(), b->d_err, b->slots * 4, cudaMemcpyDeviceToHost, b->stream));
    MM_CK(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < b->slots; ++i) {
        if (err[i]) {
            MM_CK(cudaMemsetAsync(b->d_err, 0, b->slots * 4, b->stream));
            MM_CK(cudaStreamSynchronize(b->stream));
            if (err[i] == 2)
                return fail(MM_ERR_CUDA, std::string(what) + ": a bulk copy of slot " + std::to_string(i) +
                                             " did not complete within its time limit");
            return fail(MM_ERR_CARRY, std::string(what) + ": carry out of a product that must fit, slot " + std::to_string(i));
        }
    }
    return MM_OK;
}

int launch_steps(mm_b200_batch* b, size_t bits, bool bare = false) {
    size_t most = 0;
    for (size_t i = 0; i < b->slots; ++i) most = std::max(most, (size_t)(b->nbits[i] - b->pos[i]));
    size_t left = std::min(bits, most);
    if (left == 0) return MM_OK;
    int rc = push(b);
    if (rc) return rc;
    SlotArgs a = slot_args(b);
    a.bare = bare ? 1 : 0;
    GArgs g{};
    if (b->global) {
        g = global_args(b);
        g.a.bare = a.bare;
    }
    const size_t chunk = (size_t)std::max(1, b->sched.launch_steps > 0 ? b->sched.launch_steps : b->dev->max_launch_steps);
    while (left > 0) {
        const uint32_t s = (uint32_t)std::min(left, chunk);
        if (b->cluster) {
            SlotArgs c = a;
            c.tab2 = b->ctab->t2;
            c.tab1 = b->ctab->t1;
            const int e = cluster_launch(b->m, b->cluster_chunk_log, c, (uint32_t)b->slots, s, b->stream);
            if (e) return fail(MM_ERR_CUDA, std::string("cluster launch: ") + cudaGetErrorString((cudaError_t)e));
        } else if (b->global) {
            b->gk.step<<<(unsigned)b->slots, b->gk.threads, b->gk.smem, b->stream>>>(g, 0, s);
        } else {
            b->step_fn<<<(unsigned)b->slots, b->step_threads, b->ks.smem, b->stream>>>(a, 0, s, nullptr);
        }
        MM_CK(cudaGetLastError());
        ++b->launches;
        for (size_t i = 0; i < b->slots; ++i) b->pos[i] += std::min<uint32_t>(s, b->nbits[i] - b->pos[i]);
        left -= s;
    }
    if (!bare) b->host_x_valid = false;
    return MM_OK;
}

// Global-mode work vectors and tables for a batch created in shared mode (a schedule switch).
int ensure_global_buffers(mm_b200_batch* b) {
    if (b->m < kMinGlobalLogN) return fail(MM_ERR_UNSUPPORTED, "global mode needs L >= 8192");
    if (!b->gtab) {
        const DevTables* t = nullptr;
        int rc = ensure_tables(b->dev, b->m, true, &t);
        if (rc) return rc;
        b->gtab = t;
    }
    if (!b->d_w2) {
        MM_CK(cudaMalloc(&b->d_w2, b->slots * b->n * sizeof(F2)));
        MM_CK(cudaMalloc(&b->d_w1, b->slots * b->n * sizeof(F1)));
    }
    return MM_OK;
}

// Cluster mode of a global batch: the shared-layout tables of its length and the kernels' shared
// memory opt-in (once per device).
int ensure_cluster(mm_b200_batch* b) {
    if (!b->ctab) {
        const DevTables* t = nullptr;
        int rc = ensure_tables(b->dev, b->m, false, &t);
        if (rc) return rc;
        b->ctab = t;
    }
    std::lock_guard<std::mutex> lock(b->dev->mu);
    if (!b->dev->cluster_configured) {
        const int e = cluster_configure();
        if (e) return fail(MM_ERR_CUDA, std::string("cluster mode: ") + cudaGetErrorString((cudaError_t)e));
        b->dev->cluster_configured = true;
    }
    return MM_OK;
}

// Staging words for a refill: pinned host and device buffers of at least `words` u32. Waits
// for the batch's stream first, since an earlier copy may still read the pinned buffer.
int ensure_stage(mm_b200_batch* b, size_t words) {
    if (!b->stage_copied) MM_CK(cudaEventCreateWithFlags(&b->stage_copied, cudaEventDisableTiming));
    if (words <= b->stage_cap && words <= b->hstage_cap) {
        // The pinned words may be rewritten once the last copy out of them has passed; device
        // work that still reads the device staging is ordered before the next copy by the stream.
        MM_CK(cudaEventSynchronize(b->stage_copied));
        return MM_OK;
    }
    MM_CK(cudaStreamSynchronize(b->stream));
    if (words > b->stage_cap) {
        if (b->d_stage) MM_CK(cudaFree(b->d_stage));
        b->d_stage = nullptr;
        MM_CK(cudaMalloc(&b->d_stage, words * 4));
        b->stage_cap = words;
    }
    if (words > b->hstage_cap) {
        if (b->h_stage) MM_CK(cudaFreeHost(b->h_stage));
        b->h_stage = nullptr;
        MM_CK(cudaMallocHost(&b->h_stage, words * 4));
        b->hstage_cap = words;
    }
    return MM_OK;
}

// Widens the device exponent rows to `ew` words per slot, keeping every row.
int grow_exponents(mm_b200_batch* b, size_t ew) {
    uint32_t* nd = nullptr;
    MM_CK(cudaMalloc(&nd, b->slots * ew * 4));
    MM_CK(cudaMemsetAsync(nd, 0, b->slots * ew * 4, b->stream));
    MM_CK(cudaMemcpy2DAsync(nd, ew * 4, b->d_exp, b->ew * 4, b->ew * 4, b->slots, cudaMemcpyDeviceToDevice, b->stream));
    MM_CK(cudaStreamSynchronize(b->stream));
    MM_CK(cudaFree(b->d_exp));
    b->d_exp = nd;
    b->exp_cap = ew;
    b->ew = ew;
    return MM_OK;
}

// Refill scatter: stage = [slot ids | nbits | x rows (k) | exponent rows (ew_in)], one block per
// row; exponent rows are zero-padded to the batch's row stride ew_out.
__global__ void scatter_rows_kernel(const uint32_t* __restrict__ stage, uint32_t count, uint32_t k, uint32_t ew_in,
                                    uint32_t ew_out, uint32_t* x, uint32_t* exp, uint32_t* nbits, uint32_t* pos) {
    const uint32_t r = blockIdx.x;
    const size_t slot = stage[r];
    const uint32_t* xs = stage + 2 * (size_t)count + (size_t)r * k;
    const uint32_t* es = stage + 2 * (size_t)count + (size_t)count * k + (size_t)r * ew_in;
    if (x)
        for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) x[slot * k + j] = xs[j];
    if (exp) {
        for (uint32_t j = threadIdx.x; j < ew_out; j += blockDim.x) exp[slot * ew_out + j] = j < ew_in ? es[j] : 0u;
        if (threadIdx.x == 0) {
            nbits[slot] = stage[count + r];
            pos[slot] = 0;
        }
    }
}

// Refill gather: x rows of the slots listed in stage[0 .. count) into out (count x k).
__global__ void gather_rows_kernel(const uint32_t* __restrict__ ids, uint32_t k, const uint32_t* __restrict__ x,
                                   uint32_t* out) {
    const uint32_t r = blockIdx.x;
    const size_t slot = ids[r];
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) out[(size_t)r * k + j] = x[slot * k + j];
}

int check_slot_list(const mm_b200_batch* b, size_t count, const size_t* slots, const char* what) {
    if (!slots && count) return fail(MM_ERR_ARG, std::string(what) + ": null slot list");
    if (count > 0xffffffffu) return fail(MM_ERR_ARG, std::string(what) + ": too many slots");
    for (size_t r = 0; r < count; ++r)
        if (slots[r] >= b->slots) return fail(MM_ERR_ARG, std::string(what) + ": bad slot " + std::to_string(slots[r]));
    return MM_OK;
}

}  // namespace

// Accessors for entry points defined in other translation units.
int mm_set_error(int code, const std::string& msg) { return fail(code, msg); }

int mm_device_ordinal(const mm_b200_device* dev) { return dev ? dev->device : 0; }

// The tables and kernels of length 2^(m+1) in one mode, for the Transform trait.
int mm_device_tables(mm_b200_device* dev, int m, bool global, const F2K** t2, const F1** t1, KernelSet* ks,
                     GlobalKernels* gk) {
    const DevTables* t = nullptr;
    int rc = ensure_tables(dev, m, global, &t);
    if (rc) return rc;
    *t2 = t->t2;
    *t1 = t->t1;
    if (global) {
        *gk = global_kernels();
    } else {
        kernel_set(m, *ks);
    }
    return MM_OK;
}

int mm_batch_plain(const mm_b200_batch* b) { return b && b->plain ? 1 : 0; }

int mm_batch_view(const mm_b200_batch* b, int* device, int* m, const F2** c2, const F1** c1, const F2K** tab2,
                  const F1** tab1, size_t* slots) {
    *device = b->dev->device;
    *m = b->m;
    *c2 = b->d_c2;
    *c1 = b->d_c1;
    *tab2 = b->tab->t2;
    *tab1 = b->tab->t1;
    *slots = b->slots;
    return MM_OK;
}

extern "C" {

const char* mm_b200_last_error(void) { return g_err.c_str(); }

int mm_b200_open(const mm_b200_options* opts, mm_b200_device** out) {
    if (!out) return fail(MM_ERR_ARG, "null output pointer");
    mm_b200_options o{0, 0, 1, 0};
    if (opts) o = *opts;
    if (!host::check_fixed_roots()) return fail(MM_ERR_UNSUPPORTED, "field roots differ from the ones the kernels assume");
    int count = 0;
    MM_CK(cudaGetDeviceCount(&count));
    if (o.device < 0 || o.device >= count) return fail(MM_ERR_ARG, "no CUDA device " + std::to_string(o.device));
    MM_CK(cudaSetDevice(o.device));
    cudaDeviceProp prop;
    MM_CK(cudaGetDeviceProperties(&prop, o.device));
    auto* d = new mm_b200_device();
    d->device = o.device;
    d->sms = prop.multiProcessorCount;
    d->max_smem = (int)prop.sharedMemPerBlockOptin;
    d->name = prop.name;
    if (o.max_launch_steps > 0) d->max_launch_steps = o.max_launch_steps;
    d->force_global = o.force_global != 0;
    d->wrap = o.wraparound != 0;
    *out = d;
    return MM_OK;
}

void mm_b200_close(mm_b200_device* dev) {
    if (!dev) return;
    cudaSetDevice(dev->device);
    for (auto& kv : dev->tables) {
        cudaFree(kv.second.t2);
        cudaFree(kv.second.t1);
    }
    delete dev;
}

int mm_b200_sm_count(const mm_b200_device* dev) { return dev ? dev->sms : 0; }
int mm_b200_max_dyn_smem(const mm_b200_device* dev) { return dev ? dev->max_smem : 0; }
const char* mm_b200_device_name(const mm_b200_device* dev) { return dev ? dev->name.c_str() : ""; }

size_t mm_b200_free_memory(mm_b200_device* dev) {
    if (!dev) return 0;
    cudaSetDevice(dev->device);
    size_t free_b = 0, total = 0;
    if (cudaMemGetInfo(&free_b, &total) != cudaSuccess) return 0;
    return free_b;
}

void mm_b200_coefficient_bound(uint64_t out[2]) {
    unsigned __int128 q = (unsigned __int128)P1 * P2;
    out[0] = (uint64_t)q;
    out[1] = (uint64_t)(q >> 64);
}

size_t mm_b200_supported_lengths(size_t* out, size_t cap) {
    size_t cnt = 0;
    for (int m = kMinLogN; m <= kMaxGlobalLogN; ++m) {
        if (out && cnt < cap) out[cnt] = (size_t)2 << m;
        ++cnt;
    }
    return cnt;
}

int mm_b200_full_k(const mm_b200_device* dev) { return dev && !dev->wrap ? 0 : 1; }

size_t mm_b200_batch_bytes(size_t slots, size_t len, size_t exp_words) {
    const size_t n = len / 2;
    // x (4n), T (8n), constants F(N') and A|B (2n elements of 24 B), exponent words, nbits,
    // pos and err, per slot; plus mul's spectrum scratch (24n) and this length's tables. Global
    // mode (n > 8192) adds the per-slot work vector (24n).
    const int m = log2_exact(n);
    const bool global = m > kMaxSharedLogN;
    const size_t per_slot = 4 * n + 8 * n + 48 * n + (global ? 24 * n : 0) + 4 * exp_words + 12;
    const size_t tabs = m < kMinLogN ? 0 : (size_t)(global ? glt_size(m) : lt_size(m)) * (sizeof(F2K) + sizeof(F1));
    return slots * per_slot + 24 * n + tabs;
}

int mm_b200_create(mm_b200_device* dev, size_t k, size_t len, uint32_t base, size_t slots, const uint32_t* n,
                   const uint32_t* nprime, const uint32_t* two_n, mm_b200_batch** out) {
    (void)two_n;
    if (!dev || !out || !n || !nprime) return fail(MM_ERR_ARG, "null argument");
    if (slots == 0) return fail(MM_ERR_ARG, "empty batch");
    const int m = log2_exact(len / 2);
    if (len < 8 || m < kMinLogN || ((size_t)2 << m) != len) return fail(MM_ERR_ARG, "transform length must be a power of two >= 8");
    if (m > kMaxGlobalLogN) return fail(MM_ERR_UNSUPPORTED, "transform length " + std::to_string(len) + " exceeds the largest supported (2^24)");
    const bool global = m > kMaxSharedLogN || (dev->force_global && m >= kMinGlobalLogN);
    if (dev->wrap && k != len / 2) return fail(MM_ERR_ARG, "wraparound needs k = L/2");
    if (k == 0 || k > len / 2) return fail(MM_ERR_ARG, "k must be in 1 .. L/2");
    if (base < 1 || base > 4) return fail(MM_ERR_ARG, "base must be in 1..4 (lazy range)");
    MM_CK(cudaSetDevice(dev->device));
    // batch_bytes counts global mode's work vectors from n > 8192 on; forced global mode below
    // that adds them here.
    const size_t forced = global && m <= kMaxSharedLogN ? 24 * slots * k : 0;
    const size_t need = mm_b200_batch_bytes(slots, len, 1) + 8 * slots * k + forced + ((size_t)64 << 20);
    const size_t freeb = mm_b200_free_memory(dev);
    if (need > freeb) return fail(MM_ERR_OOM, "batch needs " + std::to_string(need) + " bytes, " + std::to_string(freeb) + " free");
    // Shared-mode tables for every length that has them (mul_noalloc and schedule switches read
    // them), global-mode tables for a global batch.
    const DevTables *stab = nullptr, *gtab = nullptr;
    int rc = MM_OK;
    if (m <= kMaxSharedLogN) rc = ensure_tables(dev, m, false, &stab);
    if (!rc && global) rc = ensure_tables(dev, m, true, &gtab);
    if (rc) return rc;
    const DevTables* tab = stab ? stab : gtab;
    // On a failure below, everything allocated so far is released with the batch.
    std::unique_ptr<mm_b200_batch, void (*)(mm_b200_batch*)> b(new mm_b200_batch(), mm_b200_destroy);
    b->dev = dev;
    b->m = m;
    b->k = k;
    b->n = len / 2;
    b->slots = slots;
    b->base = base;
    b->tab = tab;
    b->global = global;
    b->plain = !dev->wrap;
    b->sched.global = global ? 1 : 0;
    b->gk = global_kernels();
    b->sched.threads = global ? b->gk.threads : (m <= kMaxSharedLogN ? threads_for(m) : 0);
    b->gtab = gtab;
    if (m <= kMaxSharedLogN) {
        kernel_set(m, b->ks);
        b->step_fn = b->ks.step;
        b->step_threads = b->ks.threads;
    }
    MM_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    const size_t nn = b->n;
    MM_CK(cudaMalloc(&b->d_x, slots * k * 4));
    MM_CK(cudaMalloc(&b->d_t, slots * 2 * nn * 4));
    MM_CK(cudaMalloc(&b->d_c2, slots * 2 * nn * sizeof(F2)));
    MM_CK(cudaMalloc(&b->d_c1, slots * 2 * nn * sizeof(F1)));
    MM_CK(cudaMalloc(&b->d_exp, slots * 4));
    b->exp_cap = 1;
    b->ew = 1;
    MM_CK(cudaMalloc(&b->d_nbits, slots * 4));
    MM_CK(cudaMalloc(&b->d_pos, slots * 4));
    MM_CK(cudaMalloc(&b->d_err, slots * 4));
    MM_CK(cudaMalloc(&b->d_spec2, nn * sizeof(F2)));
    MM_CK(cudaMalloc(&b->d_spec1, nn * sizeof(F1)));
    if (global) {
        MM_CK(cudaMalloc(&b->d_w2, slots * nn * sizeof(F2)));
        MM_CK(cudaMalloc(&b->d_w1, slots * nn * sizeof(F1)));
    }
    MM_CK(cudaMemsetAsync(b->d_x, 0, slots * k * 4, b->stream));
    MM_CK(cudaMemsetAsync(b->d_exp, 0, slots * 4, b->stream));
    MM_CK(cudaMemsetAsync(b->d_nbits, 0, slots * 4, b->stream));
    MM_CK(cudaMemsetAsync(b->d_pos, 0, slots * 4, b->stream));
    MM_CK(cudaMemsetAsync(b->d_err, 0, slots * 4, b->stream));
    // Per-slot constants from N and N' on the device.
    uint32_t *d_n = nullptr, *d_np = nullptr;
    MM_CK(cudaMalloc(&d_n, slots * k * 4));
    MM_CK(cudaMalloc(&d_np, slots * k * 4));
    MM_CK(cudaMemcpyAsync(d_n, n, slots * k * 4, cudaMemcpyHostToDevice, b->stream));
    MM_CK(cudaMemcpyAsync(d_np, nprime, slots * k * 4, cudaMemcpyHostToDevice, b->stream));
    for (size_t first = 0; first < slots; first += 65535) {
        const unsigned grid = (unsigned)std::min<size_t>(65535, slots - first);
        if (global)
            b->gk.setup<<<grid, b->gk.threads, b->gk.smem, b->stream>>>(global_args(b.get()), d_n, d_np, b->d_c2, b->d_c1,
                                                                       gtab->inv8h2, gtab->inv8h1, (uint32_t)first, nullptr);
        else
            b->ks.setup<<<grid, b->ks.threads, b->ks.smem, b->stream>>>(d_n, d_np, b->d_c2, b->d_c1, tab->t2, tab->t1,
                                                                       tab->inv8h2, tab->inv8h1, (uint32_t)first, nullptr,
                                                                       (uint32_t)k, b->plain ? 1 : 0);
        MM_CK(cudaGetLastError());
        ++b->launches;
    }
    MM_CK(cudaStreamSynchronize(b->stream));
    MM_CK(cudaFree(d_n));
    MM_CK(cudaFree(d_np));
    rc = check_err(b.get(), "create");
    if (rc) return rc;
    MM_CK(cudaMallocHost(&b->host_x, slots * k * 4));
    b->host_x_len = slots * k;
    std::memset(b->host_x, 0, slots * k * 4);
    b->host_x_valid = true;
    b->device_x_stale = false;
    b->exps.assign(slots, std::vector<uint32_t>());
    b->nbits.assign(slots, 0);
    b->pos.assign(slots, 0);
    *out = b.release();
    return MM_OK;
}

int mm_b200_load(mm_b200_batch* b, size_t i, const uint32_t* limbs) {
    if (!b || !limbs || i >= b->slots) return fail(MM_ERR_ARG, "load: bad slot");
    int rc = pull_x(b);
    if (rc) return rc;
    std::memcpy(b->host_x + i * b->k, limbs, b->k * 4);
    b->device_x_stale = true;
    return MM_OK;
}

int mm_b200_load_all(mm_b200_batch* b, const uint32_t* limbs) {
    if (!b || !limbs) return fail(MM_ERR_ARG, "load_all: null argument");
    // The pinned buffer may still feed the upload of a previous push.
    MM_CK(cudaStreamSynchronize(b->stream));
    std::memcpy(b->host_x, limbs, b->host_x_len * 4);
    b->host_x_valid = true;
    b->device_x_stale = true;
    return MM_OK;
}

int mm_b200_set_exponent(mm_b200_batch* b, size_t i, const uint32_t* words, size_t nwords, size_t nbits) {
    if (!b || i >= b->slots) return fail(MM_ERR_ARG, "set_exponent: bad slot");
    if (nbits > 32 * nwords || nbits > 0xffffffffu || (nwords && !words)) return fail(MM_ERR_ARG, "set_exponent: nbits exceeds the words");
    b->exps[i].assign(words, words + nwords);
    b->nbits[i] = (uint32_t)nbits;
    b->pos[i] = 0;
    b->exp_dirty = true;
    return MM_OK;
}

int mm_b200_set_exponents(mm_b200_batch* b, const uint32_t* words, size_t ew, const uint32_t* nbits) {
    if (!b || (!words && ew) || !nbits) return fail(MM_ERR_ARG, "set_exponents: null argument");
    for (size_t i = 0; i < b->slots; ++i) {
        if (nbits[i] > 32 * ew) return fail(MM_ERR_ARG, "set_exponents: nbits exceeds the words");
        b->exps[i].assign(words + i * ew, words + (i + 1) * ew);
        b->nbits[i] = nbits[i];
        b->pos[i] = 0;
    }
    b->exp_dirty = true;
    return MM_OK;
}

int mm_b200_run_async(mm_b200_batch* b, size_t bits) {
    if (!b) return fail(MM_ERR_ARG, "run: null batch");
    MM_CK(cudaSetDevice(b->dev->device));
    return launch_steps(b, bits);
}

int mm_b200_push(mm_b200_batch* b) {
    if (!b) return fail(MM_ERR_ARG, "push: null batch");
    MM_CK(cudaSetDevice(b->dev->device));
    return push(b);
}

int mm_b200_sync(mm_b200_batch* b) {
    if (!b) return fail(MM_ERR_ARG, "sync: null batch");
    MM_CK(cudaStreamSynchronize(b->stream));
    return check_err(b, "run");
}

int mm_b200_run_bare(mm_b200_batch* b, size_t bits) {
    if (!b) return fail(MM_ERR_ARG, "run_bare: null batch");
    MM_CK(cudaSetDevice(b->dev->device));
    int rc = launch_steps(b, bits, true);
    if (rc) return rc;
    return mm_b200_sync(b);
}

int mm_b200_run(mm_b200_batch* b, size_t bits) {
    int rc = mm_b200_run_async(b, bits);
    if (rc) return rc;
    return mm_b200_sync(b);
}

int mm_b200_mul(mm_b200_batch* b, size_t out, size_t a, size_t bb) {
    if (!b || out >= b->slots || a >= b->slots || bb >= b->slots) return fail(MM_ERR_ARG, "mul: bad slot");
    MM_CK(cudaSetDevice(b->dev->device));
    int rc = push(b);
    if (rc) return rc;
    if (b->global)
        b->gk.mul<<<1, b->gk.threads, b->gk.smem, b->stream>>>(global_args(b), (uint32_t)out, (uint32_t)a, (uint32_t)bb,
                                                              b->d_spec2, b->d_spec1);
    else
        b->ks.mul<<<1, b->ks.threads, b->ks.smem, b->stream>>>(slot_args(b), (uint32_t)out, (uint32_t)a, (uint32_t)bb,
                                                              b->d_spec2, b->d_spec1);
    MM_CK(cudaGetLastError());
    ++b->launches;
    MM_CK(cudaStreamSynchronize(b->stream));
    b->host_x_valid = false;
    return check_err(b, "mul");
}

int mm_b200_run_items_async(mm_b200_batch* b, size_t count, const size_t* slots, const uint32_t* steps) {
    if (!b || (count && (!slots || !steps))) return fail(MM_ERR_ARG, "run_items: null argument");
    if (b->global || b->cluster) return fail(MM_ERR_UNSUPPORTED, "run_items: shared-memory lengths only (L <= 16384)");
    if (count == 0) return MM_OK;
    int rc = check_slot_list(b, count, slots, "run_items");
    if (rc) return rc;
    std::vector<char> seen(b->slots, 0);
    for (size_t i = 0; i < count; ++i) {
        if (seen[slots[i]]) return fail(MM_ERR_ARG, "run_items: slot listed twice");
        if (steps[i] == 0) return fail(MM_ERR_ARG, "run_items: a step budget must be at least 1");
        seen[slots[i]] = 1;
    }
    MM_CK(cudaSetDevice(b->dev->device));
    rc = push(b);
    if (rc) return rc;
    if (!b->d_items) {
        MM_CK(cudaMalloc(&b->d_items, b->slots * sizeof(uint2)));
        MM_CK(cudaMallocHost(&b->h_items, b->slots * sizeof(uint2)));
        MM_CK(cudaEventCreateWithFlags(&b->items_copied, cudaEventDisableTiming));
    } else {
        MM_CK(cudaEventSynchronize(b->items_copied));   // the previous list has left the staging
    }
    for (size_t i = 0; i < count; ++i) b->h_items[i] = make_uint2((unsigned)slots[i], steps[i]);
    MM_CK(cudaMemcpyAsync(b->d_items, b->h_items, count * sizeof(uint2), cudaMemcpyHostToDevice, b->stream));
    MM_CK(cudaEventRecord(b->items_copied, b->stream));
    SlotArgs a = slot_args(b);
    for (size_t first = 0; first < count; first += 65535) {
        const unsigned grid = (unsigned)std::min<size_t>(65535, count - first);
        b->step_fn<<<grid, b->step_threads, b->ks.smem, b->stream>>>(a, 0, 0, b->d_items + first);
        MM_CK(cudaGetLastError());
        ++b->launches;
    }
    for (size_t i = 0; i < count; ++i) {
        const size_t s = slots[i];
        b->pos[s] += std::min<uint32_t>(steps[i], b->nbits[s] - b->pos[s]);
    }
    b->host_x_valid = false;
    return MM_OK;
}

int mm_b200_busy(const mm_b200_batch* b) {
    if (!b) return 0;
    if (cudaSetDevice(b->dev->device) != cudaSuccess) return 0;
    const cudaError_t e = cudaStreamQuery(b->stream);
    return e == cudaErrorNotReady ? 1 : 0;
}

int mm_b200_blocks_per_sm(const mm_b200_batch* b) {
    if (!b) return 0;
    int per = 0;
    if (b->cluster || b->global) return b->cluster ? 1 : 2;
    if (cudaSetDevice(b->dev->device) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, b->step_fn, b->step_threads, b->ks.smem) != cudaSuccess) return 0;
    return per;
}

int mm_b200_wait_check(mm_b200_batch* b, uint64_t limit_ns) {
    if (!b) return fail(MM_ERR_ARG, "null batch");
    if (limit_ns < 1000 || limit_ns > 1000000000ull) return fail(MM_ERR_ARG, "wait_check: limit must be 1 us .. 1 s");
    MM_CK(cudaSetDevice(b->dev->device));
    if (launch_wait_check(b->d_err, limit_ns, b->stream)) return fail(MM_ERR_CUDA, "wait_check: launch failed");
    return check_err(b, "wait_check");
}

int mm_b200_read(mm_b200_batch* b, size_t i, uint32_t* limbs) {
    if (!b || !limbs || i >= b->slots) return fail(MM_ERR_ARG, "read: bad slot");
    int rc = pull_x(b);
    if (rc) return rc;
    std::memcpy(limbs, b->host_x + i * b->k, b->k * 4);
    return MM_OK;
}

int mm_b200_read_all(mm_b200_batch* b, uint32_t* limbs) {
    if (!b || !limbs) return fail(MM_ERR_ARG, "read_all: null argument");
    int rc = pull_x(b);
    if (rc) return rc;
    std::memcpy(limbs, b->host_x, b->host_x_len * 4);
    return MM_OK;
}

size_t mm_b200_remaining(const mm_b200_batch* b, size_t i) {
    if (!b || i >= b->slots) return 0;
    return b->nbits[i] - b->pos[i];
}

size_t mm_b200_slots(const mm_b200_batch* b) { return b ? b->slots : 0; }

void* mm_b200_stream(mm_b200_batch* b) { return b ? (void*)b->stream : nullptr; }

uint64_t mm_b200_launches(const mm_b200_batch* b) { return b ? b->launches : 0; }

void mm_b200_destroy(mm_b200_batch* b) {
    if (!b) return;
    cudaSetDevice(b->dev->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaFree(b->d_x);
    cudaFree(b->d_t);
    cudaFree(b->d_c2);
    cudaFree(b->d_c1);
    cudaFree(b->d_exp);
    cudaFree(b->d_nbits);
    cudaFree(b->d_pos);
    cudaFree(b->d_err);
    cudaFree(b->d_spec2);
    cudaFree(b->d_spec1);
    cudaFree(b->d_w2);
    cudaFree(b->d_w1);
    cudaFree(b->d_stage);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    if (b->stage_copied) cudaEventDestroy(b->stage_copied);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->host_x) cudaFreeHost(b->host_x);
    if (b->host_exp) cudaFreeHost(b->host_exp);
    if (b->d_items) cudaFree(b->d_items);
    if (b->h_items) cudaFreeHost(b->h_items);
    if (b->items_copied) cudaEventDestroy(b->items_copied);
    delete b;
}

int mm_b200_set_schedule(mm_b200_batch* b, const mm_b200_schedule* sc) {
    if (!b || !sc) return fail(MM_ERR_ARG, "set_schedule: null argument");
    if (sc->launch_steps < 0 || sc->step_ns < 0) return fail(MM_ERR_ARG, "set_schedule: negative value");
    if (sc->global < 0 || sc->global > 2) return fail(MM_ERR_ARG, "set_schedule: mode must be 0, 1 or 2");
    MM_CK(cudaSetDevice(b->dev->device));
    const bool global = sc->global != 0;
    const bool cluster = sc->global == 2;
    if (!global && b->m > kMaxSharedLogN) return fail(MM_ERR_UNSUPPORTED, "set_schedule: L > 16384 runs in global mode only");
    if (cluster && (b->m < kMinClusterLogN || b->m > kMaxClusterLogN))
        return fail(MM_ERR_UNSUPPORTED, "set_schedule: cluster mode runs L = 32768 and 65536 only");
    if (cluster && b->plain) return fail(MM_ERR_UNSUPPORTED, "set_schedule: cluster mode needs the wraparound path");
    // Cluster mode: threads per SM picks the chunk, 512 (one 8,192-element block) or, at
    // L = 32768, 1024 (two 4,096-element blocks of 512 threads).
    int chunk_log = kClusterChunkLog;
    if (cluster && sc->threads != 0 && sc->threads != 512) {
        if (sc->threads != 1024 || b->m != kMinClusterLogN)
            return fail(MM_ERR_UNSUPPORTED, "set_schedule: cluster mode runs 512 threads per SM"
                                            " (1024 at L = 32768: two blocks per SM)");
        chunk_log = kClusterPairChunkLog;
    }
    StepFn fn = b->ks.step;
    int threads = b->ks.threads;
    if (!global && sc->threads != 0 && sc->threads != b->ks.threads) {
        if (!b->ks.step_alt || sc->threads != b->ks.threads_alt)
            return fail(MM_ERR_UNSUPPORTED, "set_schedule: L = " + std::to_string(2 * b->n) + " runs " +
                                                std::to_string(b->ks.threads) +
                                                (b->ks.step_alt ? " or " + std::to_string(b->ks.threads_alt) : std::string()) +
                                                " threads per block");
        fn = b->ks.step_alt;
        threads = b->ks.threads_alt;
    }
    if (global) {
        int rc = ensure_global_buffers(b);
        if (rc) return rc;
    }
    if (cluster) {
        int rc = ensure_cluster(b);
        if (rc) return rc;
    }
    b->global = global;
    b->cluster = cluster;
    b->cluster_chunk_log = chunk_log;
    if (!global) {
        b->step_fn = fn;
        b->step_threads = threads;
    }
    b->sched = *sc;
    b->sched.global = cluster ? 2 : (global ? 1 : 0);
    b->sched.threads = global ? (cluster ? (chunk_log == kClusterChunkLog ? 512 : 1024) : b->gk.threads) : threads;
    return MM_OK;
}

int mm_b200_get_schedule(const mm_b200_batch* b, mm_b200_schedule* sc) {
    if (!b || !sc) return fail(MM_ERR_ARG, "get_schedule: null argument");
    *sc = b->sched;
    return MM_OK;
}

int mm_b200_set_moduli(mm_b200_batch* b, size_t count, const size_t* slots, const uint32_t* n, const uint32_t* nprime) {
    if (!b || ((!n || !nprime) && count)) return fail(MM_ERR_ARG, "set_moduli: null argument");
    int rc = check_slot_list(b, count, slots, "set_moduli");
    if (rc || count == 0) return rc;
    MM_CK(cudaSetDevice(b->dev->device));
    const size_t k = b->k;
    rc = ensure_stage(b, count * (1 + 2 * k));
    if (rc) return rc;
    uint32_t* h = b->h_stage;
    for (size_t r = 0; r < count; ++r) h[r] = (uint32_t)slots[r];
    std::memcpy(h + count, n, count * k * 4);
    std::memcpy(h + count + count * k, nprime, count * k * 4);
    MM_CK(cudaMemcpyAsync(b->d_stage, h, count * (1 + 2 * k) * 4, cudaMemcpyHostToDevice, b->stream));
    MM_CK(cudaEventRecord(b->stage_copied, b->stream));
    const DevTables* tab = b->global ? b->gtab : b->tab;
    for (size_t c0 = 0; c0 < count; c0 += 65535) {
        const unsigned grid = (unsigned)std::min<size_t>(65535, count - c0);
        const uint32_t* ids = b->d_stage + c0;
        const uint32_t* nl = b->d_stage + count + c0 * k;
        const uint32_t* npl = b->d_stage + count + count * k + c0 * k;
        if (b->global)
            b->gk.setup<<<grid, b->gk.threads, b->gk.smem, b->stream>>>(global_args(b), nl, npl, b->d_c2, b->d_c1,
                                                                       tab->inv8h2, tab->inv8h1, 0, ids);
        else
            b->ks.setup<<<grid, b->ks.threads, b->ks.smem, b->stream>>>(nl, npl, b->d_c2, b->d_c1, tab->t2, tab->t1,
                                                                       tab->inv8h2, tab->inv8h1, 0, ids, (uint32_t)k,
                                                                       b->plain ? 1 : 0);
        MM_CK(cudaGetLastError());
        ++b->launches;
    }
    return MM_OK;
}

int mm_b200_write_slots(mm_b200_batch* b, size_t count, const size_t* slots, const uint32_t* x, const uint32_t* words,
                        size_t ew, const uint32_t* nbits) {
    if (!b) return fail(MM_ERR_ARG, "write_slots: null batch");
    int rc = check_slot_list(b, count, slots, "write_slots");
    if (rc || count == 0) return rc;
    if (words && (!nbits || ew == 0)) return fail(MM_ERR_ARG, "write_slots: exponents need ew > 0 and nbits");
    if (words)
        for (size_t r = 0; r < count; ++r)
            if (nbits[r] > 32 * ew) return fail(MM_ERR_ARG, "write_slots: nbits exceeds the words");
    MM_CK(cudaSetDevice(b->dev->device));
    // Earlier host-side loads and exponents reach the device first.
    rc = push(b);
    if (rc) return rc;
    if (words && ew > b->ew) {
        rc = grow_exponents(b, ew);
        if (rc) return rc;
    }
    const size_t k = b->k, ewi = words ? ew : 0;
    const size_t total = count * (2 + k + ewi);
    rc = ensure_stage(b, total);
    if (rc) return rc;
    uint32_t* h = b->h_stage;
    for (size_t r = 0; r < count; ++r) {
        h[r] = (uint32_t)slots[r];
        h[count + r] = words ? nbits[r] : 0;
    }
    if (x) std::memcpy(h + 2 * count, x, count * k * 4);
    if (words) std::memcpy(h + 2 * count + count * k, words, count * ew * 4);
    MM_CK(cudaMemcpyAsync(b->d_stage, h, total * 4, cudaMemcpyHostToDevice, b->stream));
    MM_CK(cudaEventRecord(b->stage_copied, b->stream));
    scatter_rows_kernel<<<(unsigned)count, 128, 0, b->stream>>>(b->d_stage, (uint32_t)count, (uint32_t)k, (uint32_t)ewi,
                                                                (uint32_t)b->ew, x ? b->d_x : nullptr,
                                                                words ? b->d_exp : nullptr, b->d_nbits, b->d_pos);
    MM_CK(cudaGetLastError());
    for (size_t r = 0; r < count; ++r) {
        const size_t i = slots[r];
        if (x && b->host_x_valid) std::memcpy(b->host_x + i * k, x + r * k, k * 4);
        if (words) {
            b->exps[i].assign(words + r * ew, words + (r + 1) * ew);
            b->nbits[i] = nbits[r];
            b->pos[i] = 0;
        }
    }
    return MM_OK;
}

int mm_b200_read_slots(mm_b200_batch* b, size_t count, const size_t* slots, uint32_t* x) {
    if (!b || (!x && count)) return fail(MM_ERR_ARG, "read_slots: null argument");
    int rc = check_slot_list(b, count, slots, "read_slots");
    if (rc || count == 0) return rc;
    const size_t k = b->k;
    if (b->host_x_valid) {
        for (size_t r = 0; r < count; ++r) std::memcpy(x + r * k, b->host_x + slots[r] * k, k * 4);
        return MM_OK;
    }
    MM_CK(cudaSetDevice(b->dev->device));
    rc = ensure_stage(b, count * (1 + k));
    if (rc) return rc;
    uint32_t* h = b->h_stage;
    for (size_t r = 0; r < count; ++r) h[r] = (uint32_t)slots[r];
    MM_CK(cudaMemcpyAsync(b->d_stage, h, count * 4, cudaMemcpyHostToDevice, b->stream));
    MM_CK(cudaEventRecord(b->stage_copied, b->stream));
    gather_rows_kernel<<<(unsigned)count, 128, 0, b->stream>>>(b->d_stage, (uint32_t)k, b->d_x, b->d_stage + count);
    MM_CK(cudaGetLastError());
    MM_CK(cudaMemcpyAsync(h + count, b->d_stage + count, count * k * 4, cudaMemcpyDeviceToHost, b->stream));
    MM_CK(cudaStreamSynchronize(b->stream));
    std::memcpy(x, h + count, count * k * 4);
    return MM_OK;
}

}  // extern "C"

// ---- the mixed-length plan ----
struct mm_b200_plan {
    mm_b200_device* dev = nullptr;
    std::vector<mm_b200_batch*> batches;
    std::vector<char> wide;           // per batch: 1 its slots are in d_wide, 2 in d_pair (its kind at creation)
    std::vector<cudaEvent_t> ready;   // per batch: its stream's work before a launch
    cudaEvent_t done = nullptr;       // the plan's last launch
    cudaStream_t stream = nullptr;
    size_t quantum = 0;
    int grid = 0;
    MixedDesc* d_descs = nullptr;
    MixedDesc* h_descs = nullptr;     // pinned copy of what the device holds
    // Every slot (plan_run, plan_run_each): the group items longest first, then the wide items.
    uint4* d_items = nullptr;
    uint4* d_wide = nullptr;
    uint4* d_pair = nullptr;           // cluster items (a block pair on one slot)
    uint32_t count = 0;                // slots of all batches
    // [0], [1], [2]: counts of d_items, d_wide and d_pair; [3], [4], [5]: counts of
    // plan_run_items' three lists.
    uint32_t* d_count = nullptr;
    uint4* d_tick = nullptr;           // plan_run_items' lists: group items at 0, wide at `count`, pairs at 2 `count`
    uint4* h_tick = nullptr;           // pinned staging of those lists (+ their counts)
    cudaGraph_t graph_items = nullptr;
    cudaGraphExec_t exec_items = nullptr;
    uint32_t* d_counter = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphExec_t exec_each = nullptr;   // the launch with per-batch step budgets
    cudaGraph_t graph_each = nullptr;
    uint64_t launches = 0, graph_launches = 0;
};

namespace {

// Relative cost of one slot-step of a batch: the schedule's measured time, else the transform
// work n log2 n (global mode pays about a fifth more in memory traffic).
double step_cost(const mm_b200_batch* b, bool global) {
    if (b->sched.step_ns > 0) return b->sched.step_ns;
    const double n = (double)b->n;
    return n * (double)b->m * (global ? 1.2 : 1.0);
}

MixedDesc mixed_desc(const mm_b200_batch* b, bool global, uint32_t bits) {
    MixedDesc d{};
    d.bits = bits;
    if (global) d.g = global_args(b);
    else {
        d.g.a = slot_args(b);
        d.g.w2 = nullptr;
        d.g.w1 = nullptr;
        d.g.m = b->m;
    }
    d.global = global ? 1 : 0;
    d.ctab2 = b->ctab ? b->ctab->t2 : nullptr;
    d.ctab1 = b->ctab ? b->ctab->t1 : nullptr;
    return d;
}

// A batch whose slots run as wide items (a whole block each, the vector in shared memory).
bool plan_wide(const mm_b200_batch* b) { return !b->global && b->m == kWideLogN; }
// A batch whose slots run in global mode inside the mixed launch.
bool plan_global(const mm_b200_batch* b) { return b->global || b->m > kWideLogN; }
// A batch whose slots run as cluster items (a block pair each, mm_cluster.cuh): L = 32768 in
// cluster mode.
bool plan_pair(const mm_b200_batch* b) { return b->cluster && b->m == kPairLogN && b->ctab && !b->plain; }
int plan_kind(const mm_b200_batch* b) { return plan_pair(b) ? 2 : (plan_wide(b) ? 1 : 0); }

// The counter reset and one persistent launch over lists `items` (count at count[0]), `wide`
// (count at count[1]) and `pair` (count at count[2]).
cudaError_t plan_launch(mm_b200_plan* p, const uint4* items, const uint4* wide, const uint4* pair, const uint32_t* count,
                        uint32_t bits) {
    cudaError_t e = cudaMemsetAsync(p->d_counter, 0, 3 * sizeof(uint32_t), p->stream);
    if (e != cudaSuccess) return e;
    const MixedLists l{items, count, wide, count + 1, p->d_counter, pair, count + 2};
    return (cudaError_t)mixed_launch(p->grid, p->d_descs, l, bits, p->stream);
}

// Descriptor of batch i for plan_run and plan_run_each, whose item lists were built at creation:
// a batch keeps the kind it had then. A wide batch runs in shared mode on whole blocks whatever
// its schedule says now; any other batch of L = 16384 (tuned to global mode at creation) runs
// in global mode on a worker, whose 96 KiB cannot hold its vector. The per-slot constants are
// the same in both modes, so the results do not depend on the mode.
MixedDesc plan_desc(const mm_b200_plan* p, size_t i, uint32_t bits) {
    const mm_b200_batch* b = p->batches[i];
    return mixed_desc(b, p->wide[i] != 1 && (plan_global(b) || b->m == kWideLogN), bits);
}

// One launch of `bits` steps over every slot.
int plan_enqueue(mm_b200_plan* p, uint32_t bits) {
    MM_CK(plan_launch(p, p->d_items, p->d_wide, p->d_pair, p->d_count, bits));
    return MM_OK;
}

}  // namespace

extern "C" {

int mm_b200_plan_create(mm_b200_batch* const* batches, size_t count, size_t quantum, mm_b200_plan** out) {
    if (!batches || !out || count == 0) return fail(MM_ERR_ARG, "plan_create: no batches");
    if (quantum == 0 || quantum > 0xffffffffu) return fail(MM_ERR_ARG, "plan_create: quantum must be in 1 .. 2^32 - 1");
    mm_b200_device* dev = batches[0] ? batches[0]->dev : nullptr;
    size_t total = 0;
    for (size_t i = 0; i < count; ++i) {
        if (!batches[i]) return fail(MM_ERR_ARG, "plan_create: null batch");
        if (batches[i]->dev != dev) return fail(MM_ERR_ARG, "plan_create: batches on different devices");
        total += batches[i]->slots;
    }
    if (total > 0xffffffffu) return fail(MM_ERR_ARG, "plan_create: too many slots");
    MM_CK(cudaSetDevice(dev->device));
    for (size_t i = 0; i < count; ++i) {
        if (plan_global(batches[i])) {
            int rc = ensure_global_buffers(batches[i]);
            if (rc) return rc;
        }
    }
    std::unique_ptr<mm_b200_plan, void (*)(mm_b200_plan*)> p(new mm_b200_plan(), mm_b200_plan_destroy);
    p->dev = dev;
    p->batches.assign(batches, batches + count);
    p->wide.assign(count, 0);
    for (size_t i = 0; i < count; ++i) p->wide[i] = (char)plan_kind(batches[i]);
    p->quantum = quantum;
    p->count = (uint32_t)total;
    MM_CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    MM_CK(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming));
    p->ready.assign(count, nullptr);
    for (auto& e : p->ready) MM_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    {
        std::lock_guard<std::mutex> lock(dev->mu);
        if (!dev->mixed_configured) {
            MM_CK(cudaFuncSetAttribute((const void*)mixed_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, kMixedSmem));
            MM_CK(cudaFuncSetAttribute((const void*)mixed_kernel(), cudaFuncAttributePreferredSharedMemoryCarveout,
                                       cudaSharedmemCarveoutMaxShared));
            dev->mixed_configured = true;
        }
    }
    // Block pairs that fit on the device at once (the launch is a cluster launch of pairs).
    int pairs = 0;
    {
        const int e = mixed_clusters(&pairs);
        if (e) return fail(MM_ERR_CUDA, std::string("plan_create: ") + cudaGetErrorString((cudaError_t)e));
    }
    if (pairs < 1) return fail(MM_ERR_CUDA, "plan_create: the mixed launch fits no block pair on the device");
    p->grid = pairs * kMixedCluster;
    // Group items longest first (by cost per step; every slot of a batch has the same), then by
    // batch and slot; wide and cluster items by batch and slot.
    std::vector<std::pair<double, uint4>> items;
    std::vector<uint4> wide, pair;
    items.reserve(total);
    for (size_t i = 0; i < count; ++i) {
        const double c = step_cost(batches[i], plan_global(batches[i]));
        for (size_t s = 0; s < batches[i]->slots; ++s) {
            const uint4 it = make_uint4((unsigned)i, (unsigned)s, 0u, 0u);
            if (p->wide[i] == 2) pair.push_back(it);
            else if (p->wide[i] == 1) wide.push_back(it);
            else items.push_back({c, it});
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<uint4> it(total);
    for (size_t i = 0; i < items.size(); ++i) it[i] = items[i].second;
    std::copy(wide.begin(), wide.end(), it.begin() + items.size());
    std::copy(pair.begin(), pair.end(), it.begin() + items.size() + wide.size());
    MM_CK(cudaMalloc(&p->d_items, total * sizeof(uint4)));
    MM_CK(cudaMemcpy(p->d_items, it.data(), total * sizeof(uint4), cudaMemcpyHostToDevice));
    p->d_wide = p->d_items + items.size();
    p->d_pair = p->d_wide + wide.size();
    MM_CK(cudaMalloc(&p->d_count, 6 * sizeof(uint32_t)));
    const uint32_t counts[6] = {(uint32_t)items.size(), (uint32_t)wide.size(), (uint32_t)pair.size(), 0, 0, 0};
    MM_CK(cudaMemcpy(p->d_count, counts, sizeof(counts), cudaMemcpyHostToDevice));
    MM_CK(cudaMalloc(&p->d_descs, count * sizeof(MixedDesc)));
    MM_CK(cudaMallocHost(&p->h_descs, count * sizeof(MixedDesc)));
    std::memset(p->h_descs, 0, count * sizeof(MixedDesc));
    MM_CK(cudaMalloc(&p->d_counter, 3 * sizeof(uint32_t)));
    *out = p.release();
    return MM_OK;
}

int mm_b200_plan_run_async(mm_b200_plan* p, size_t bits) {
    if (!p) return fail(MM_ERR_ARG, "plan_run: null plan");
    MM_CK(cudaSetDevice(p->dev->device));
    size_t most = 0;
    for (auto* b : p->batches)
        for (size_t i = 0; i < b->slots; ++i) most = std::max(most, (size_t)(b->nbits[i] - b->pos[i]));
    size_t left = std::min(bits, most);
    if (left == 0) return MM_OK;
    const size_t nb = p->batches.size();
    for (size_t i = 0; i < nb; ++i) {
        mm_b200_batch* b = p->batches[i];
        int rc = push(b);
        if (rc) return rc;
        MM_CK(cudaEventRecord(p->ready[i], b->stream));
        MM_CK(cudaStreamWaitEvent(p->stream, p->ready[i], 0));
    }
    // Descriptors follow the batches' buffers (exponent rows can be reallocated and restrided).
    std::vector<MixedDesc> d(nb);
    for (size_t i = 0; i < nb; ++i) d[i] = plan_desc(p, i, 0);
    if (std::memcmp(d.data(), p->h_descs, nb * sizeof(MixedDesc)) != 0) {
        MM_CK(cudaStreamSynchronize(p->stream));   // the pinned copy may still feed the last upload
        std::memcpy(p->h_descs, d.data(), nb * sizeof(MixedDesc));
        MM_CK(cudaMemcpyAsync(p->d_descs, p->h_descs, nb * sizeof(MixedDesc), cudaMemcpyHostToDevice, p->stream));
    }
    while (left > 0) {
        const size_t s = std::min(left, p->quantum);
        if (s == p->quantum) {
            if (!p->exec) {
                MM_CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
                int rc = plan_enqueue(p, (uint32_t)s);
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(p->stream, &g);
                if (rc) return rc;
                if (e != cudaSuccess) return fail(MM_ERR_CUDA, std::string("plan capture: ") + cudaGetErrorString(e));
                p->graph = g;
                MM_CK(cudaGraphInstantiate(&p->exec, p->graph, 0));
            }
            MM_CK(cudaGraphLaunch(p->exec, p->stream));
            ++p->graph_launches;
        } else {
            int rc = plan_enqueue(p, (uint32_t)s);
            if (rc) return rc;
        }
        ++p->launches;
        for (auto* b : p->batches) {
            for (size_t i = 0; i < b->slots; ++i) b->pos[i] += std::min<uint32_t>((uint32_t)s, b->nbits[i] - b->pos[i]);
        }
        left -= s;
    }
    MM_CK(cudaEventRecord(p->done, p->stream));
    for (auto* b : p->batches) {
        MM_CK(cudaStreamWaitEvent(b->stream, p->done, 0));
        b->host_x_valid = false;
    }
    return MM_OK;
}

int mm_b200_plan_run_each_async(mm_b200_plan* p, const size_t* steps) {
    if (!p || !steps) return fail(MM_ERR_ARG, "plan_run_each: null argument");
    MM_CK(cudaSetDevice(p->dev->device));
    const size_t nb = p->batches.size();
    bool any = false;
    for (size_t i = 0; i < nb; ++i) {
        if (steps[i] > 0xffffffffu) return fail(MM_ERR_ARG, "plan_run_each: steps must be below 2^32");
        const mm_b200_batch* b = p->batches[i];
        for (size_t s = 0; steps[i] && s < b->slots && !any; ++s) any = b->pos[s] < b->nbits[s];
    }
    if (!any) return MM_OK;
    for (size_t i = 0; i < nb; ++i) {
        mm_b200_batch* b = p->batches[i];
        int rc = push(b);
        if (rc) return rc;
        MM_CK(cudaEventRecord(p->ready[i], b->stream));
        MM_CK(cudaStreamWaitEvent(p->stream, p->ready[i], 0));
    }
    // The launch's own `bits` is 0, so a batch whose budget is 0 runs no step.
    std::vector<MixedDesc> d(nb);
    for (size_t i = 0; i < nb; ++i) d[i] = plan_desc(p, i, (uint32_t)steps[i]);
    if (std::memcmp(d.data(), p->h_descs, nb * sizeof(MixedDesc)) != 0) {
        MM_CK(cudaStreamSynchronize(p->stream));
        std::memcpy(p->h_descs, d.data(), nb * sizeof(MixedDesc));
        MM_CK(cudaMemcpyAsync(p->d_descs, p->h_descs, nb * sizeof(MixedDesc), cudaMemcpyHostToDevice, p->stream));
    }
    if (!p->exec_each) {
        MM_CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
        int rc = plan_enqueue(p, 0);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(p->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(MM_ERR_CUDA, std::string("plan capture: ") + cudaGetErrorString(e));
        p->graph_each = g;
        MM_CK(cudaGraphInstantiate(&p->exec_each, p->graph_each, 0));
    }
    MM_CK(cudaGraphLaunch(p->exec_each, p->stream));
    ++p->graph_launches;
    ++p->launches;
    for (size_t i = 0; i < nb; ++i) {
        mm_b200_batch* b = p->batches[i];
        for (size_t s = 0; s < b->slots; ++s)
            b->pos[s] += (uint32_t)std::min<size_t>(steps[i], (size_t)(b->nbits[s] - b->pos[s]));
    }
    MM_CK(cudaEventRecord(p->done, p->stream));
    for (auto* b : p->batches) {
        MM_CK(cudaStreamWaitEvent(b->stream, p->done, 0));
        b->host_x_valid = false;
    }
    return MM_OK;
}

int mm_b200_plan_run_items(mm_b200_plan* p, size_t count, const uint32_t* batch, const uint32_t* slot,
                           const uint32_t* steps) {
    if (!p || (count && (!batch || !slot || !steps))) return fail(MM_ERR_ARG, "plan_run_items: null argument");
    if (count == 0) return MM_OK;
    if (count > p->count) return fail(MM_ERR_ARG, "plan_run_items: more items than the plan's slots");
    MM_CK(cudaSetDevice(p->dev->device));
    const size_t nb = p->batches.size();
    // Each slot at most once per launch: two blocks must not step one slot at the same time.
    std::vector<std::vector<bool>> seen(nb);
    for (size_t i = 0; i < count; ++i) {
        if (batch[i] >= nb || slot[i] >= p->batches[batch[i]]->slots)
            return fail(MM_ERR_ARG, "plan_run_items: bad item " + std::to_string(i));
        auto& s = seen[batch[i]];
        if (s.empty()) s.assign(p->batches[batch[i]]->slots, false);
        if (s[slot[i]]) return fail(MM_ERR_ARG, "plan_run_items: slot listed twice");
        s[slot[i]] = true;
    }
    for (size_t i = 0; i < nb; ++i) {
        mm_b200_batch* b = p->batches[i];
        int rc = push(b);
        if (rc) return rc;
        MM_CK(cudaEventRecord(p->ready[i], b->stream));
        MM_CK(cudaStreamWaitEvent(p->stream, p->ready[i], 0));
    }
    std::vector<MixedDesc> d(nb);
    for (size_t i = 0; i < nb; ++i) d[i] = mixed_desc(p->batches[i], plan_global(p->batches[i]), 0);
    // The pinned list and descriptors may still feed the previous launch's uploads.
    MM_CK(cudaStreamSynchronize(p->stream));
    if (std::memcmp(d.data(), p->h_descs, nb * sizeof(MixedDesc)) != 0) {
        std::memcpy(p->h_descs, d.data(), nb * sizeof(MixedDesc));
        MM_CK(cudaMemcpyAsync(p->d_descs, p->h_descs, nb * sizeof(MixedDesc), cudaMemcpyHostToDevice, p->stream));
    }
    const size_t cap = p->count;
    if (!p->d_tick) {
        MM_CK(cudaMalloc(&p->d_tick, 3 * cap * sizeof(uint4)));
        MM_CK(cudaMallocHost(&p->h_tick, (3 * cap + 1) * sizeof(uint4)));
    }
    // The list splits into group items at 0, wide items at cap and cluster items at 2 cap, each
    // in list order; a batch keeps the kind it has now.
    size_t ng = 0, nw = 0, np = 0;
    for (size_t i = 0; i < count; ++i) {
        const uint4 it = make_uint4(batch[i], slot[i], steps[i], 0u);
        const int kind = plan_kind(p->batches[batch[i]]);
        if (kind == 2) p->h_tick[2 * cap + np++] = it;
        else if (kind == 1) p->h_tick[cap + nw++] = it;
        else p->h_tick[ng++] = it;
    }
    uint32_t* hc = reinterpret_cast<uint32_t*>(p->h_tick + 3 * cap);
    hc[0] = (uint32_t)ng;
    hc[1] = (uint32_t)nw;
    hc[2] = (uint32_t)np;
    if (ng) MM_CK(cudaMemcpyAsync(p->d_tick, p->h_tick, ng * sizeof(uint4), cudaMemcpyHostToDevice, p->stream));
    if (nw)
        MM_CK(cudaMemcpyAsync(p->d_tick + cap, p->h_tick + cap, nw * sizeof(uint4), cudaMemcpyHostToDevice, p->stream));
    if (np)
        MM_CK(cudaMemcpyAsync(p->d_tick + 2 * cap, p->h_tick + 2 * cap, np * sizeof(uint4), cudaMemcpyHostToDevice,
                              p->stream));
    MM_CK(cudaMemcpyAsync(p->d_count + 3, hc, 3 * sizeof(uint32_t), cudaMemcpyHostToDevice, p->stream));
    if (!p->exec_items) {
        MM_CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e0 = plan_launch(p, p->d_tick, p->d_tick + cap, p->d_tick + 2 * cap, p->d_count + 3, 0);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(p->stream, &g);
        if (e0 != cudaSuccess) return fail(MM_ERR_CUDA, std::string("plan capture: ") + cudaGetErrorString(e0));
        if (e != cudaSuccess) return fail(MM_ERR_CUDA, std::string("plan capture: ") + cudaGetErrorString(e));
        p->graph_items = g;
        MM_CK(cudaGraphInstantiate(&p->exec_items, p->graph_items, 0));
    }
    MM_CK(cudaGraphLaunch(p->exec_items, p->stream));
    ++p->graph_launches;
    ++p->launches;
    for (size_t i = 0; i < count; ++i) {
        mm_b200_batch* b = p->batches[batch[i]];
        const size_t s = slot[i];
        b->pos[s] += std::min<uint32_t>(steps[i], b->nbits[s] - b->pos[s]);
    }
    MM_CK(cudaEventRecord(p->done, p->stream));
    for (auto* b : p->batches) {
        MM_CK(cudaStreamWaitEvent(b->stream, p->done, 0));
        b->host_x_valid = false;
    }
    return mm_b200_plan_sync(p);
}

int mm_b200_plan_blocks(const mm_b200_plan* p) { return p ? p->grid * kMixedGroups : 0; }

int mm_b200_plan_wide_blocks(const mm_b200_plan* p) { return p ? p->grid : 0; }

int mm_b200_plan_batch_wide(const mm_b200_plan* p, size_t i) {
    return p && i < p->batches.size() && plan_wide(p->batches[i]) ? 1 : 0;
}

int mm_b200_plan_run_each(mm_b200_plan* p, const size_t* steps) {
    int rc = mm_b200_plan_run_each_async(p, steps);
    if (rc) return rc;
    return mm_b200_plan_sync(p);
}

int mm_b200_plan_sync(mm_b200_plan* p) {
    if (!p) return fail(MM_ERR_ARG, "plan_sync: null plan");
    MM_CK(cudaSetDevice(p->dev->device));
    MM_CK(cudaStreamSynchronize(p->stream));
    for (auto* b : p->batches) {
        int rc = check_err(b, "run");
        if (rc) return rc;
    }
    return MM_OK;
}

int mm_b200_plan_run(mm_b200_plan* p, size_t bits) {
    int rc = mm_b200_plan_run_async(p, bits);
    if (rc) return rc;
    return mm_b200_plan_sync(p);
}

void* mm_b200_plan_stream(mm_b200_plan* p) { return p ? (void*)p->stream : nullptr; }
uint64_t mm_b200_plan_launches(const mm_b200_plan* p) { return p ? p->launches : 0; }
uint64_t mm_b200_plan_graph_launches(const mm_b200_plan* p) { return p ? p->graph_launches : 0; }

void mm_b200_plan_destroy(mm_b200_plan* p) {
    if (!p) return;
    if (p->dev) cudaSetDevice(p->dev->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->exec_each) cudaGraphExecDestroy(p->exec_each);
    if (p->graph_each) cudaGraphDestroy(p->graph_each);
    cudaFree(p->d_items);
    cudaFree(p->d_count);
    cudaFree(p->d_tick);
    if (p->h_tick) cudaFreeHost(p->h_tick);
    if (p->exec_items) cudaGraphExecDestroy(p->exec_items);
    if (p->graph_items) cudaGraphDestroy(p->graph_items);
    cudaFree(p->d_descs);
    cudaFree(p->d_counter);
    if (p->h_descs) cudaFreeHost(p->h_descs);
    for (auto e : p->ready)
        if (e) cudaEventDestroy(e);
    if (p->done) cudaEventDestroy(p->done);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

}  // extern "C"
