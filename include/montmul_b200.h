/* montmul_b200 — C ABI of the B200 backend for MontMul's batched Montgomery step
 * x <- x^2 c R^-1 mod N (and a b R^-1 mod N) over many independent odd moduli.
 *
 * The ABI mirrors the reference's backend contract, the `Limits` and `Backend` traits of
 * montmul/src/transform.rs:11-20 and 61-77, as implemented by the CUDA backend `Gpu`
 * (montmul/src/gpu/mod.rs:321-398). The caller (the host API `ModBatch`, batch.rs:53-184)
 * keeps the big-integer work — N' = -N^-1 mod R, Montgomery conversion, is_one — and passes
 * plain little-endian 32-bit limb arrays.
 *
 * Conventions (the reference panics where this ABI returns a status):
 *   - every call that can fail returns an int status (MM_OK = 0); mm_b200_last_error() then
 *     describes it with the reference's wording ("batch needs ... bytes", "carry out of a
 *     product that must fit, slot i");
 *   - the backend copies every input; the caller owns its buffers;
 *   - one batch is used by one host thread at a time (the trait's &mut State).
 * The wraparound path is on by default (k = L/2, GpuOptions::wraparound, gpu/mod.rs:36-44);
 * mm_b200_options.wraparound = 0 selects the plain REDC with k = k0 (Cpu::default).
 */
#ifndef MONTMUL_B200_H
#define MONTMUL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MM_OK = 0,
    MM_ERR_ARG = 1,          /* bad argument (index, size, unsupported length, ...) */
    MM_ERR_OOM = 2,          /* batch does not fit in device memory (message names the bytes) */
    MM_ERR_CARRY = 3,        /* a carry that must vanish did not (message names the slot) */
    MM_ERR_CUDA = 4,         /* CUDA runtime error (message carries the runtime's text), or a
                                device copy that did not complete within its time limit */
    MM_ERR_UNSUPPORTED = 5   /* a configuration this build does not run */
};

typedef struct mm_b200_device mm_b200_device; /* `Gpu` (gpu/mod.rs:47-54): one CUDA device */
typedef struct mm_b200_batch mm_b200_batch;   /* `GpuState` (gpu/mod.rs:237-258): one batch */

/* `GpuOptions` (gpu/mod.rs:28-45). Lengths L <= 16384 run with the whole vector in shared
 * memory; longer ones (up to 2^24) keep it in device memory and stream 2,048-element tiles
 * through shared memory ("global mode"). force_global selects global mode from L = 8192 on
 * (the reference's force_global). max_launch_steps bounds the steps of one kernel launch (the
 * reference bounds launches by time, max_launch_ms); 0 selects the default. */
typedef struct {
    int device;
    int force_global;
    int wraparound;          /* 1 (default): k = L/2 and the wraparound REDC; 0: k = k0, plain REDC */
    int max_launch_steps;
} mm_b200_options;

/* Message of the last failing call on this host thread ("" if none). */
const char *mm_b200_last_error(void);

/* Gpu::with_options (gpu/mod.rs:62-67). */
int mm_b200_open(const mm_b200_options *opts, mm_b200_device **out);
void mm_b200_close(mm_b200_device *dev);
/* Gpu::sm_count / free_memory / max_dyn_smem / device_name (gpu/mod.rs:83-99). */
int mm_b200_sm_count(const mm_b200_device *dev);
size_t mm_b200_free_memory(mm_b200_device *dev);
int mm_b200_max_dyn_smem(const mm_b200_device *dev);
const char *mm_b200_device_name(const mm_b200_device *dev);

/* Limits (transform.rs:11-20): Q = M31 * M61 as two 64-bit halves (lo, hi); the supported
 * transform lengths L ascending (returns their number, writes at most cap); full_k. */
void mm_b200_coefficient_bound(uint64_t out[2]);
size_t mm_b200_supported_lengths(size_t *out, size_t cap);
int mm_b200_full_k(const mm_b200_device *dev);

/* Device bytes a batch of `slots` slots at length `len` takes (Gpu::create's check,
 * gpu/mod.rs:332, with this backend's buffers). */
size_t mm_b200_batch_bytes(size_t slots, size_t len, size_t exp_words);

/* Backend::create (transform.rs:64; gpu/mod.rs:325-370). n, nprime, two_n: slots x k limbs,
 * row-major (BatchSetup, transform.rs:49-59). k must equal len / 2. */
int mm_b200_create(mm_b200_device *dev, size_t k, size_t len, uint32_t base, size_t slots,
                   const uint32_t *n, const uint32_t *nprime, const uint32_t *two_n,
                   mm_b200_batch **out);
/* Backend::load (transform.rs:65-66): k limbs of a Montgomery-form value in [0, 2N). */
int mm_b200_load(mm_b200_batch *b, size_t i, const uint32_t *limbs);
/* All slots at once: slots x k limbs. */
int mm_b200_load_all(mm_b200_batch *b, const uint32_t *limbs);
/* Backend::set_exponent (transform.rs:67-68): MSB-first words; resets the slot's position. */
int mm_b200_set_exponent(mm_b200_batch *b, size_t i, const uint32_t *words, size_t nwords, size_t nbits);
/* All slots at once: slots x ew words and slots bit counts. */
int mm_b200_set_exponents(mm_b200_batch *b, const uint32_t *words, size_t ew, const uint32_t *nbits);
/* Backend::run (transform.rs:69-70): up to `bits` steps on every slot with bits left. */
int mm_b200_run(mm_b200_batch *b, size_t bits);
/* Gpu::run_bare (gpu/mod.rs:109-111): like run, but each step stops after the squaring
 * T = c x^2 and leaves x unchanged; it times the squaring alone for the overhead ratio
 * (score.rs:140-159). Positions advance as in run. */
int mm_b200_run_bare(mm_b200_batch *b, size_t bits);
/* Backend::mul (transform.rs:71-72): slot out <- a b R^-1, slots sharing a modulus. */
int mm_b200_mul(mm_b200_batch *b, size_t out, size_t a, size_t bb);
/* Backend::read (transform.rs:73-74): k limbs in [0, 2N). */
int mm_b200_read(mm_b200_batch *b, size_t i, uint32_t *limbs);
int mm_b200_read_all(mm_b200_batch *b, uint32_t *limbs);
/* Backend::remaining (transform.rs:75-76). */
size_t mm_b200_remaining(const mm_b200_batch *b, size_t i);
size_t mm_b200_slots(const mm_b200_batch *b);
void mm_b200_destroy(mm_b200_batch *b);

/* Asynchronous form of run for timing: enqueues the launches on the batch's stream and
 * returns; mm_b200_sync waits and performs run's error check. mm_b200_stream is the
 * cudaStream_t the batch launches on. */
int mm_b200_run_async(mm_b200_batch *b, size_t bits);
/* Uploads pending loads and exponents now (run does this itself before its first launch). */
int mm_b200_push(mm_b200_batch *b);
int mm_b200_sync(mm_b200_batch *b);
void *mm_b200_stream(mm_b200_batch *b);
/* Kernel launches issued by this batch so far (for launch accounting). */
uint64_t mm_b200_launches(const mm_b200_batch *b);

/* Serving launches (no counterpart in the reference): run_items_async enqueues, on the batch's
 * stream, one launch of the uniform step kernel over an explicit list, slot slots[i] running up
 * to steps[i] steps (each slot at most once, steps[i] >= 1), and returns; mm_b200_sync waits and
 * reports errors as run does. Lists of several batches on their own streams run on the device
 * at the same time. Shared-memory lengths only (L <= 16384). blocks_per_sm: blocks of the
 * batch's step kernel that one SM holds at once (0 on an error). */
int mm_b200_run_items_async(mm_b200_batch *b, size_t count, const size_t *slots, const uint32_t *steps);
int mm_b200_blocks_per_sm(const mm_b200_batch *b);
/* 1 while work enqueued on the batch's stream is still running, 0 once it has finished (then
 * mm_b200_sync returns at once with the error check): lets a loop service whichever batch is
 * done while the others run. */
int mm_b200_busy(const mm_b200_batch *b);

/* Failure path of the bounded waits (no counterpart in the reference): every wait of a kernel on
 * a bulk copy gives up after a time limit (100 ms in the step kernels), sets the slot's error
 * word to 2, and the call reports MM_ERR_CUDA "... did not complete within its time limit" with
 * the context still usable (the reference's error-word check, gpu/mod.rs:179-184). This runs
 * that wait once on the batch's stream against an mbarrier armed for a copy that is never
 * issued, with a limit of limit_ns (1 us .. 1 s), and returns what run would after a late copy:
 * MM_ERR_CUDA naming slot 0. The batch's state is not changed. */
int mm_b200_wait_check(mm_b200_batch *b, uint64_t limit_ns);

/* a b R^-1 mod N (lazy, in [0, 2N)) for slot `slot`'s modulus N, without allocating: no
 * counterpart in the reference. For callers that cannot allocate device memory at the point of
 * the call: services whose device memory belongs to their own pool allocator, and loops that
 * cannot afford cudaFree's implicit device synchronization. d_a, d_b (inputs) and d_out (output)
 * are device buffers of k limbs the caller owns; d_err (optional) receives 0, or 1 when a carry
 * that must vanish did not. The work is enqueued on `stream` (a cudaStream_t; NULL is the
 * legacy default stream) and the call returns without waiting. The kernel reads the slot's
 * per-batch constants, so work still queued on the batch's own stream that writes them
 * (mm_b200_set_moduli) must be complete first: call mm_b200_sync(b), or make `stream` wait on
 * an event recorded on mm_b200_stream(b). The batch's device is made current for the call and
 * the caller's current device is restored before it returns. Intermediates live in a static
 * 256 KiB device array that every GPU loading this library holds until exit; lengths needing
 * more scratch (the global-mode lengths, L >= 32768) are rejected with MM_ERR_ARG. The first
 * call on each device looks up that array's device address and sets kernel attributes, so make
 * it before any stream capture. All calls share the array: calls that overlap on the GPU race
 * and must be serialized by the caller. */
int mm_b200_mul_noalloc(const mm_b200_batch *b, size_t slot, const uint32_t *d_a, const uint32_t *d_b,
                        uint32_t *d_out, uint32_t *d_err, void *stream);

/* ---- The Transform trait (transform.rs:22-46; the Gpu backend's impl, gpu/mod.rs:286-319) ----
 * A buffer holds `count` vectors of length len = L, each L/2 elements of GF(M31^2) x GF(M61^2):
 * coefficient j in the real part of element j, coefficient j + L/2 in the imaginary part.
 * t_upload copies coefficients in (upload); t_download_raw writes the elements as
 * count x L/2 x (re, im) field values in the reference's element order (download_raw; the CRT
 * to exact coefficients, download, is host arithmetic on these). t_forward weights by zeta^j and
 * runs the DIF (natural in, bit-reversed out); t_inverse runs the DIT and unweights by
 * zeta^-j / n; t_pointwise sets out = scale a b per element, scales[v] for vector v (NULL: 1).
 * t_load_forward uploads k limbs per vector, zero-padded to len, and forward-transforms them
 * (load_forward). Results are canonical field values, bit-identical to the reference's Cpu. */
typedef struct mm_b200_tbuf mm_b200_tbuf;
int mm_b200_t_upload(mm_b200_device *dev, const uint32_t *coeffs, size_t len, size_t count, mm_b200_tbuf **out);
int mm_b200_t_download_raw(const mm_b200_tbuf *b, uint32_t *f1, uint64_t *f2);
int mm_b200_t_forward(mm_b200_tbuf *b, size_t len, size_t count);
int mm_b200_t_inverse(mm_b200_tbuf *b, size_t len, size_t count);
int mm_b200_t_pointwise(mm_b200_tbuf *out, const mm_b200_tbuf *a, const mm_b200_tbuf *b, const uint32_t *scales,
                        size_t len, size_t count);
int mm_b200_t_load_forward(mm_b200_device *dev, const uint32_t *limbs, size_t k, size_t len, size_t count,
                           mm_b200_tbuf **out);
size_t mm_b200_t_count(const mm_b200_tbuf *b);
size_t mm_b200_t_len(const mm_b200_tbuf *b);
void mm_b200_t_free(mm_b200_tbuf *b);

/* ---- Schedules (no counterpart in the reference, whose planner fixes them: gpu/plan.rs:26-60) ----
 * global: the mode. 0 runs the batch with the whole vector in shared memory (L <= 16384), 1 in
 * global mode (L >= 8192), 2 in cluster mode (L = 32768 and 65536: a thread-block cluster of
 * L / 16384 blocks per slot with the vector in the cluster's shared memory). All modes compute
 * the same per-slot constants, so a batch may switch at any time. launch_steps: steps per kernel
 * launch of run (0: the device default). step_ns: the measured time of one slot-step at full
 * occupancy, which orders the items of a mixed launch (0: a model of the transform work).
 * threads: threads per block of the shared-memory step kernel (0: the length's default; L = 4096,
 * 8192 and 16384 also build one alternative shape); in cluster mode, threads per SM (0 or 512:
 * one 512-thread block of 8192 elements per SM; 1024 at L = 32768: two 512-thread blocks of 4096
 * elements per SM, a cluster of 4). get_schedule reports the shape in use. The autotuner
 * (montmul_b200.tune) measures these per length and caches them. */
typedef struct {
    int global;
    int launch_steps;
    double step_ns;
    int threads;
} mm_b200_schedule;
int mm_b200_set_schedule(mm_b200_batch *b, const mm_b200_schedule *s);
int mm_b200_get_schedule(const mm_b200_batch *b, mm_b200_schedule *s);

/* ---- In-place refill (no counterpart in the reference): a serving loop replaces finished
 * slots while the others keep their state on the device. ----
 * set_moduli: new moduli for `count` slots (N and N' rows of k limbs, row r for slots[r]); their
 * per-slot constants are recomputed on the device. write_slots: x rows (k limbs, Montgomery
 * form in [0, 2N)) and exponents (ew words per row, MSB first, nbits[r] bits) for the listed
 * slots, positions reset to 0; x or words may be NULL to keep that part. read_slots: x rows of
 * the listed slots. All three order themselves after earlier work on the batch, including
 * mixed launches that cover it. */
int mm_b200_set_moduli(mm_b200_batch *b, size_t count, const size_t *slots, const uint32_t *n, const uint32_t *nprime);
int mm_b200_write_slots(mm_b200_batch *b, size_t count, const size_t *slots, const uint32_t *x, const uint32_t *words,
                        size_t ew, const uint32_t *nbits);
int mm_b200_read_slots(mm_b200_batch *b, size_t count, const size_t *slots, uint32_t *x);

/* ---- Mixed-length persistent launch (no counterpart in the reference) ----
 * A plan covers every slot of `count` batches on one device, of any lengths. plan_run runs up
 * to `bits` steps on every slot with bits left, like run on each batch, but in persistent
 * launches (one 512-thread block per SM) that take (batch, slot) items from device work queues;
 * each launch covers `quantum` steps and is replayed from a CUDA graph. A block first takes
 * "wide" items (L = 16384 batches in shared mode: the whole block and all its shared memory on
 * one slot), then splits into two 256-thread workers that take the other items longest first:
 * L <= 8192 with the vector in shared memory, longer lengths and batches tuned to global mode in
 * global mode. The batches must outlive the plan; plan_sync performs run's error check on every
 * batch. */
typedef struct mm_b200_plan mm_b200_plan;
int mm_b200_plan_create(mm_b200_batch *const *batches, size_t count, size_t quantum, mm_b200_plan **out);
int mm_b200_plan_run_async(mm_b200_plan *p, size_t bits);
int mm_b200_plan_sync(mm_b200_plan *p);
int mm_b200_plan_run(mm_b200_plan *p, size_t bits);
/* One launch in which the slots of batch i (in creation order) run up to steps[i] steps each;
 * a serving loop gives each length a budget that takes about the same time, so blocks holding
 * short lengths do not idle while the longest items finish. */
int mm_b200_plan_run_each_async(mm_b200_plan *p, const size_t *steps);
int mm_b200_plan_run_each(mm_b200_plan *p, const size_t *steps);
/* One launch over an explicit work list, taken in list order: item i runs up to steps[i]
 * (>= 1) steps of slot slot[i] of batch batch[i]; each slot at most once. The wide items of the
 * list run first, then the others, each kind in list order. A scheduler orders the list longest
 * first and sizes the budgets so the plan's workers finish together. Waits for the launch and
 * checks errors, as plan_run. */
int mm_b200_plan_run_items(mm_b200_plan *p, size_t count, const uint32_t *batch, const uint32_t *slot,
                           const uint32_t *steps);
/* Workers of the plan's launch that take items other than wide ones (two per block), the
 * blocks (each takes wide items one at a time), and whether batch i's items are wide. */
int mm_b200_plan_blocks(const mm_b200_plan *p);
int mm_b200_plan_wide_blocks(const mm_b200_plan *p);
int mm_b200_plan_batch_wide(const mm_b200_plan *p, size_t i);
void *mm_b200_plan_stream(mm_b200_plan *p);
/* Kernel launches of the plan so far, and how many of them were graph replays. */
uint64_t mm_b200_plan_launches(const mm_b200_plan *p);
uint64_t mm_b200_plan_graph_launches(const mm_b200_plan *p);
void mm_b200_plan_destroy(mm_b200_plan *p);

/* Integer roofline probe (no counterpart in the reference, whose roofline is not measured):
 * the peak rate of butterfly pairs (a GF(p^2) product, an add and a sub in both fields) of the
 * kernels' arithmetic from register-resident chains on every SM of `device`; `iters` chain
 * steps per thread. Writes pairs per second and the timed kernel's milliseconds. */
int mm_b200_bfly_peak(int device, int iters, double *pairs_per_s, double *ms);

#ifdef __cplusplus
}
#endif
#endif
