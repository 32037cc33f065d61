/*
 * polymul.h -- C ABI of the B200 exact negacyclic multiplier
 *
 *     c = a * b  mod (X^n + 1, q)     n a power of two, 2 <= n <= 65536,
 *                                      q odd, up to 896 bits.
 *
 * Coefficients are little-endian 64-bit limbs, `coef_limbs` per coefficient,
 * row-major n x coef_limbs, each value in [0, q).  For the reference's point
 * (N x 28 x u32, fherma.h:27-42) that is n x 14 u64 -- the same bytes.
 *
 * Every entry point returns a pm_status; on failure pm_last_error() gives a
 * message for the calling thread.  No entry point throws, and none takes or
 * returns a framework type: plain pointers, sizes and a CUDA stream handle.
 *
 * The reference's drop-in boundary is three C++ functions (fherma.h:44-46);
 * fherma_polymul.h declares those, implemented on top of this header.
 */
#ifndef POLYMUL_H
#define POLYMUL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pm_plan pm_plan;
/* A cudaStream_t; NULL means the legacy default stream. */
typedef struct CUstream_st* pm_stream;

enum pm_status {
    PM_OK = 0,
    PM_ERR_INVALID = 1,     /* bad argument: n not a power of two, even q, short buffers, ... */
    PM_ERR_UNSUPPORTED = 2, /* outside coverage: n > 65536, q wider than 896 bits, ... */
    PM_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    PM_ERR_NO_MEMORY = 4,   /* device or pinned host allocation failed */
    PM_ERR_TIMEOUT = 5,     /* a bounded wait ran out */
    PM_ERR_BUSY = 6         /* admission refused: no slot or device memory free */
};

/* Residue conversion and CRT implementation.  With neither PM_CONVERT_TENSOR nor
 * PM_CONVERT_SIMT a plan takes the tensor-core path whenever coef_limbs is even (16-byte
 * coefficient rows, which its tensor maps need; the FHERMA point's 14 limbs are), else
 * the plain method; pm_plan_info.convert says which one it runs. */
enum pm_flags {
    PM_CONVERT_DEFAULT = 0, /* the tensor path where the plan allows it, else the plain method */
    PM_CONVERT_TENSOR = 1,  /* exact INT8 digit contractions on the tcgen05 tensor cores */
    PM_CONVERT_SIMT = 8,    /* scalar CUDA-core conversion and CRT (the plain method) */
    /* For a q of the special form 2^k - delta (k >= 80, delta < 2^32, e.g. the FHERMA modulus
     * 2^868 - 11993087; the family the reference's quartic backend targets,
     * quartic/host_setup.h:41-110), reduce the CRT sum by folding 2^k = delta instead of by the
     * general Barrett division.  Same results; ignored for other q.  Measured no faster on
     * B200 (the CRT kernel is bound by latency, not by this step), so it is not the default. */
    PM_SPECIAL_FORM = 2,
    /* The reference's wide backend for comparison (solve.cu): the NTT taken modulo q itself,
     * each butterfly a W-word Montgomery multiplication, no residues and no CRT.  Needs a
     * prime q = 1 (mod 2n) (the FHERMA modulus 2^868 - 11993087 is one at n <= 32768);
     * PM_ERR_UNSUPPORTED otherwise.  Same results as the RNS method, several times slower. */
    PM_WIDE_NTT = 4,
    /* The reference's quartic factorization (its best backend, quartic/host_setup.h:41-110,
     * quartic/solve.cu) for q = B^4 - delta with B = 2^(bits(q)/4), 0 < delta < 2^28, q of
     * 772..896 bits, a multiple of 4 (the FHERMA modulus 2^868 - 11993087 is one): each coefficient split in
     * four parts of bits(q)/4 bits, the product taken in Z[X, Y] / (X^n + 1, Y^4 - delta)
     * modulo 16 primes in which delta is a fourth power, each at the four roots of
     * Y^4 = delta (64 residue planes), then interpolated and recombined with
     * Y = B mod q.  Tensor path only, coef_limbs = 14, 64 <= n; PM_ERR_UNSUPPORTED when
     * 16 primes below 2^30 do not cover n (1 + 3 delta) B^2 four times over. */
    PM_QUARTIC = 16
};

typedef struct {
    uint32_t n;
    uint32_t q_bits;
    uint32_t coef_limbs;
    uint32_t primes;          /* RNS basis size for (n, q) */
    uint32_t convert;         /* PM_CONVERT_TENSOR or PM_CONVERT_SIMT: the path the plan runs (0 for PM_WIDE_NTT) */
    uint32_t reserved;
    size_t workspace_bytes;   /* device scratch one product needs (residue planes) */
} pm_plan_info;

/*
 * Build a plan: choose the prime basis, upload CRT constants, allocate the
 * plan's own device workspace and pinned staging.  Untimed set-up.
 * Replaces fherma_init (fherma.h:44; rns/solve.cu:581-720, rns/host_setup.h:61-126),
 * widened from q = 2^868 - c to any odd q and from n <= 32768 to n <= 65536.
 * q: q_limbs little-endian u64 words.  coef_limbs >= ceil(bits(q) / 64).
 */
int pm_plan_create(pm_plan** plan, uint32_t n, const uint64_t* q, uint32_t q_limbs, uint32_t coef_limbs,
                   uint32_t flags);

int pm_plan_get_info(const pm_plan* plan, pm_plan_info* info);

/* Launch shapes of a plan (see pm_plan_autotune). */
typedef struct {
    uint32_t row_radix;         /* radix of the row NTT register passes: 4, 8 or 16 (16: rows of >= 1024
                                   values in the persistent kernel; other rows then use 8) */
    uint32_t conv_ctas_per_sm;  /* persistent CTAs of the tensor conversion per SM, 1..8 */
    uint32_t crt_ctas_per_sm;   /* persistent CTAs of the tensor CRT per SM, 1..4 */
    uint32_t group;             /* products per launch group in batched calls (0: up to ~2 GB of residues and
                                   128 products; at most 256) */
    uint32_t row_persistent;    /* 1: rows of >= 1024 values by the persistent kernel that stages a row's
                                   twiddles once per group and prefetches rows; 0: one CTA per row */
    uint32_t conv_whole_basis;  /* tensor conversion: 1 (the default) takes each coefficient tile through all
                                   primes at once (weights of the whole basis resident, 2 CTAs per SM;
                                   conv_ctas_per_sm unused); 0 runs it once per group of 16 primes */
    double us_per_product;      /* device time the autotuner measured (-1: taken from its cache) */
} pm_tuning;

/*
 * Time candidate launch shapes on a synthetic batch of this plan's products
 * (allocates temporary device memory; set-up time, not a hot-path call) and
 * keep the fastest.  Results are cached per (n, bits(q), coef_limbs, flags)
 * for the process.  Results of the products never depend on the tuning.
 */
int pm_plan_autotune(pm_plan* plan, uint32_t reps, pm_tuning* chosen);
/* Apply launch shapes directly (us_per_product is ignored). */
int pm_plan_set_tuning(pm_plan* plan, const pm_tuning* tuning);

/* Replaces fherma_free (fherma.h:46; rns/solve.cu:854). */
int pm_plan_destroy(pm_plan* plan);

/*
 * One product on device memory, asynchronous on `stream`.  a, b, c are device
 * pointers (n x coef_limbs u64); c may alias neither a nor b.  workspace is a
 * device buffer of info.workspace_bytes, or NULL to use the plan's own (then
 * calls on one plan must not overlap).  Replaces the device half of fherma_run
 * (rns/solve.cu:504-578, launch_rns).
 * Pointers must be device, managed or pinned memory, 8-byte aligned; on the
 * tensor path a, b and workspace 16-byte aligned (cudaMalloc gives 256):
 * otherwise PM_ERR_INVALID, before anything runs.  The call runs on the
 * current device, which must be the one the plan was created on, and device
 * pointers must be that device's memory: otherwise PM_ERR_INVALID too.  The
 * same holds for pm_multiply_batch and pm_multiply_noalloc.
 */
int pm_multiply(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, void* workspace,
                pm_stream stream);

/*
 * A batch of `count` products of one plan, stored back to back: a, b, c are
 * device arrays [count][n][coef_limbs].  The library runs them in launch
 * groups (one launch per pass covers a group; by default up to ~2 GB of residue
 * planes, 128 products at n = 32768, or the autotuner's choice).  workspace: a
 * device buffer of workspace_bytes (at least one product's worth; a smaller
 * buffer than a group needs shrinks the group, see pm_batch_workspace_size), or
 * NULL to use a plan-owned buffer that the first call allocates.  Asynchronous
 * on `stream`.
 */
int pm_multiply_batch(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count,
                      void* workspace, size_t workspace_bytes, pm_stream stream);
/* Workspace bytes pm_multiply_batch uses for `count` products at its preferred group size. */
int pm_batch_workspace_size(const pm_plan* plan, uint32_t count, size_t* bytes);

/*
 * One product on host memory, synchronous: copy in, multiply, copy out.
 * Pinned (page-locked) buffers are copied directly; pageable ones are staged
 * through the plan's pinned buffers.  Runs on the plan's device whichever
 * device is current (and leaves the caller's current device as it was).
 * Replaces fherma_run (fherma.h:45; rns/solve.cu:721-853).
 */
int pm_multiply_host(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c);

/*
 * pm_multiply_host in two halves, so that the caller can do its own work
 * while the GPU runs (the drop-in fherma_run allocates its output tensor
 * there).  begin copies a and b in -- host threads stage pageable pieces
 * while earlier pieces cross the link -- and queues the kernels and the copy
 * back; a and b may be reused when it returns.  end copies the product into
 * c piece by piece as the pieces land and returns the call's status (a wait
 * that timed out on the device: PM_ERR_TIMEOUT).  One product per plan may be
 * open at a time (PM_ERR_BUSY otherwise); every begin needs its end.  Same
 * role as the reference's overlapped input pipeline and output allocation in
 * fherma_run (rns/solve.cu:729-803, input_pipeline.h:12-54).
 */
int pm_multiply_host_begin(pm_plan* plan, const uint64_t* a, const uint64_t* b);
int pm_multiply_host_end(pm_plan* plan, uint64_t* c);

/*
 * One product, like pm_multiply, but the call allocates nothing: no
 * cudaMalloc, no cudaFree, no allocating library routine.  Its residue
 * scratch is a 4 MiB array built into the library (one per GPU), so it serves
 * plans whose workspace_bytes fit in 4 MiB (n <= 8192 for an 868-bit q) and
 * refuses larger ones with PM_ERR_UNSUPPORTED.  For callers that cannot
 * allocate device memory when they multiply.  All calls on a device share the
 * array: calls that overlap on the GPU race.  The first call on each device
 * (and the first after a cudaDeviceReset, whose new context holds the array at
 * a new address) looks the array's address up (cudaGetSymbolAddress); make
 * that first call before any stream capture.  This entry point has no counterpart in the
 * reference, which always multiplies in buffers it allocated in fherma_init.
 */
int pm_multiply_noalloc(const pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, pm_stream stream);

/*
 * `count` products on host memory, stored back to back ([count][n][coef_limbs]
 * u64 each), synchronous.  The batch is cut into groups that rotate over three
 * streams, so the copies in of one group, the kernels of another and the
 * copies out of a third overlap.  Pinned buffers are copied directly; pageable
 * ones are staged through pinned memory by the calling thread.  Runs on the
 * plan's device, like pm_multiply_host.  No counterpart in the reference (one
 * product per fherma_run).
 */
int pm_multiply_host_batch(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count);

/*
 * Host-only (no GPU needed): the RNS basis a plan for (n, q_bits) would use.
 * Writes up to `capacity` primes (descending, p = 1 mod 2^17, p < 2^30) and
 * sets *count.  Mirrors rns::setup's prime search (rns/host_setup.h:67-83).
 */
int pm_basis_query(uint32_t n, uint32_t q_bits, uint32_t* primes, uint32_t capacity, uint32_t* count);

/* ------------------------------------------------------------------------
 * Uneven batches: `count` products of different n (256..65536) and different
 * odd q, all on the tensor path, run as one CUDA graph of persistent kernels
 * over flat work tables (conversion items ordered by prime group, row items per
 * ring size, CRT items per width).  The batch owns packed device buffers:
 * product z's a, b, c start offsets[z] u64 words into the buffers returned by
 * pm_batch_buffers, each n_z x coef_limbs.  No counterpart in the reference.
 * ------------------------------------------------------------------------ */
typedef struct pm_batch pm_batch;
/* q[z] points to q_limbs[z] u64 words; coef_limbs is shared and even. */
int pm_batch_create(pm_batch** batch, uint32_t count, const uint32_t* n, const uint64_t* const* q,
                    const uint32_t* q_limbs, uint32_t coef_limbs);
int pm_batch_buffers(pm_batch* batch, uint64_t** a, uint64_t** b, uint64_t** c, uint64_t* offsets);
/* Copy all products' a and b in (host or device arrays in the batch's packing:
   product z at offsets[z] u64 words), or all c out; asynchronous on `stream`. */
int pm_batch_copy_in(pm_batch* batch, const uint64_t* a, const uint64_t* b, pm_stream stream);
int pm_batch_copy_out(pm_batch* batch, uint64_t* c, pm_stream stream);
/* One graph launch, asynchronous on `stream`. */
int pm_batch_run(pm_batch* batch, pm_stream stream);
/* After the stream is idle: PM_ERR_TIMEOUT if a kernel's bounded wait ran out. */
int pm_batch_check(pm_batch* batch);
/*
 * Re-time the batch graph under candidate launch shapes (row-pass radix per
 * ring size, persistent grid sizes of the conversion and CRT phases), keep the
 * fastest and re-capture; *us_per_run gets its device time.  Set-up time, not a
 * hot-path call; results never depend on it.
 */
int pm_batch_autotune(pm_batch* batch, uint32_t reps, double* us_per_run);
int pm_batch_destroy(pm_batch* batch);

/* ------------------------------------------------------------------------
 * Serving: products submitted one by one from host threads, admitted onto the
 * GPU as stream slots and device memory free up (continuous batching).  No
 * counterpart in the reference (a single-threaded caller, one product per
 * fherma_run, main.cpp:173-205).
 * ------------------------------------------------------------------------ */
typedef struct pm_server pm_server;

typedef struct {
    uint32_t slots;              /* groups in flight at once, one stream each, 1..64 */
    uint32_t max_group;          /* same-plan requests merged into one launch (0 = 8) */
    uint32_t flags;              /* PM_CONVERT_* for the server's plans */
    uint32_t reserved;
    size_t device_budget_bytes;  /* arena for the a, b, c and workspaces of in-flight
                                    groups (0 = a quarter of the free device memory) */
} pm_server_config;

typedef struct {
    uint64_t submitted, completed, failed, groups;
    uint32_t peak_inflight, peak_group;
    size_t arena_bytes, arena_used;
    double p50_us, p99_us, mean_us, max_us;  /* submission-to-completion latency */
    double products_per_s;                   /* completed / (last completion - first submission) */
} pm_server_stats;

/* Allocates the device arena once; creates the worker thread and streams. */
int pm_server_create(pm_server** server, const pm_server_config* config);
/*
 * Queue c = a*b mod (X^n+1, q); a, b, c are host buffers of n x coef_limbs u64
 * that must stay valid until pm_server_wait returns for the ticket.  Pinned
 * buffers let copies overlap; pageable ones work but serialize the worker.
 * Plans (tables) are created on first use of an (n, q) and stay resident.
 * PM_ERR_BUSY if one product needs more than the whole arena.
 */
int pm_server_submit(pm_server* server, uint32_t n, const uint64_t* q, uint32_t q_limbs, uint32_t coef_limbs,
                     const uint64_t* a, const uint64_t* b, uint64_t* c, uint64_t* ticket);
/* Bounded wait for one ticket: PM_OK, PM_ERR_TIMEOUT, or the request's failure. */
int pm_server_wait(pm_server* server, uint64_t ticket, uint32_t timeout_ms);
/* Bounded wait until nothing is queued or in flight. */
int pm_server_drain(pm_server* server, uint32_t timeout_ms);
int pm_server_get_stats(pm_server* server, pm_server_stats* stats);
int pm_server_reset_stats(pm_server* server);
/* Finishes queued work, then releases the arena, streams and plans. */
int pm_server_destroy(pm_server* server);

const char* pm_status_string(int status);
/* Message of the last failure on the calling thread ("" if none). */
const char* pm_last_error(void);
/* Number of kernel launches the library issued on this process so far. */
uint64_t pm_kernel_launch_count(void);

/*
 * Diagnostic (no counterpart in the reference): runs the library's bounded
 * mbarrier wait on a barrier that nothing arrives at, with a limit of limit_us
 * (1 .. 2e6) instead of the kernels' 1 s.  *timed_out = 1 when the wait gave up,
 * *waited_ns = how long it waited.  Shows that a device wait that cannot finish
 * ends with an error status and leaves the CUDA context usable.
 */
int pm_selftest_bounded_wait(uint32_t limit_us, uint32_t* timed_out, uint64_t* waited_ns);

/*
 * Kernel timing for measurement runs.  pm_profile_enable(capacity) makes the
 * library record a CUDA event before and after each kernel it launches, on the
 * launching stream, for up to `capacity` launches (0 switches it off and drops
 * pending records).  pm_profile_read synchronizes those events and returns,
 * per kernel name, the launch count and summed device milliseconds; names stay
 * valid for the life of the process.  Plays the role of the reference's
 * FHERMA_PROFILE stage events (rns/solve.cu:474-486, 819-835).
 */
int pm_profile_enable(uint32_t capacity);
int pm_profile_read(const char** names, uint64_t* launches, double* total_ms, uint32_t capacity, uint32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* POLYMUL_H */
