// Internal types shared by the host translation units of libpolymul.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_math.h"
#include "pm_common.cuh"

namespace pm {

struct Failure : std::runtime_error {
    int status;
    Failure(int s, std::string m);
};

void cuda_check(cudaError_t e, const char* what);
int fail(int status, const std::string& message);
void count_launches(uint64_t k);

// Records a CUDA event pair around the launches in its scope while
// pm_profile_enable is on; a no-op otherwise.
struct ProfileScope {
    cudaStream_t stream;
    long index = -1;
    ProfileScope(const char* name, cudaStream_t st);
    ~ProfileScope();
};
int profile_enable(uint32_t capacity);
int profile_read(const char** names, uint64_t* launches, double* total_ms, uint32_t capacity, uint32_t* count);

// Device-resident prime basis shared by every plan on one GPU.
struct DeviceBasis {
    int device = 0;
    std::vector<uint32_t> primes;   // kPMax primes, descending
    std::vector<uint32_t> inv1;     // [kPMax] psi^-brev(1): the inverse twiddle of the last column stage
    PrimeConst* d_pc = nullptr;     // [kPMax]
    uint2* d_tw_fwd = nullptr;      // [kPMax][kNMax] psi^brev(k)   (value, Shoup)
    uint2* d_tw_inv = nullptr;      // [kPMax][kNMax] psi^-brev(k)
    uint2* d_conv_pow = nullptr;    // [kPMax][kPowWords] 2^(32k) mod p
    // tensor-core conversion table (built on first tensor plan)
    uint8_t* d_conv_weights = nullptr;
    ~DeviceBasis();
};

DeviceBasis& basis_for_device(int device);
PrimeConst prime_const(uint32_t p);
// Psi_rev[k] = psi^brev(k) and psi^-brev(k) (value, Shoup), k < kNMax, psi of order 2 kNMax mod p
void twiddle_tables(uint32_t p, uint2* fwd, uint2* inv);
std::vector<uint32_t> make_primes();
unsigned basis_size(const std::vector<uint32_t>& primes, unsigned n, unsigned qbits);

// One stage of the host-batch pipeline: a stream with its own device buffers
// (a, b, c and the residue workspace of a group) and pinned staging.
struct PipelineSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    void* d_buf = nullptr;
    void* h_buf = nullptr;
    bool pending = false;
    ~PipelineSlot();
};

// The single-product host-buffer call (host_call.cu): pinned staging, device
// copies of a, b, c, a host copy pool and the events of the product's pieces.
class CopyPool;
struct HostCall {
    cudaStream_t stream = nullptr;  // the plan's stream
    cudaStream_t side = nullptr;    // converts a while b is on the link
    cudaEvent_t a_in = nullptr, a_converted = nullptr;
    void* d_io = nullptr;           // a, b, c on the device
    void* h_stage = nullptr;        // pinned a, b, c and the error word
    std::vector<cudaEvent_t> out_ready;
    std::unique_ptr<CopyPool> pool;
    std::atomic<uint8_t> ready[64];  // input piece k staged
    bool pending = false;           // between multiply_host_begin and multiply_host_end
    uint8_t* direct_out = nullptr;  // pinned caller output the product lands in directly, or null
    ~HostCall();
};

// Largest launch group by default, and the largest a caller may set.
constexpr uint32_t kMaxDefaultGroup = 128;
constexpr uint32_t kMaxGroup = 256;

// Launch shapes the autotuner chooses per plan (defaults apply until it runs).
struct Tuning {
    int row_radix_log = 4;   // K2 register-pass radix: 2, 3 or 4 (radix 4, 8, 16; 16 in the persistent kernel)
    int conv_ctas_per_sm = 3;  // K1T persistent CTAs per SM (up to four fit; three measured fastest)
    int crt_ctas_per_sm = 2;   // K3T persistent CTAs per SM
    bool row_persistent = true;  // K2 as the persistent, prefetching kernel (rows of C >= 1024)
    bool conv_whole_basis = true;  // tensor conversion: one pass of a tile over every prime (K1W) or per group (K1T)
    uint32_t group = 0;        // products per launch group in batches (0: up to ~2 GB of residues, <= 128)
    bool tuned = false;
};

// Tables of the direct wide-modulus NTT (PM_WIDE_NTT, wide.cu).
struct WideTables {
    uint32_t* d_q = nullptr;      // [W]
    uint32_t* d_r2 = nullptr;     // [W] R^2 mod q, R = 2^(32W)
    uint32_t* d_ninv = nullptr;   // [W] n^-1 mod q
    uint32_t* d_tw_fwd = nullptr; // [n][W] psi^brev(k) R mod q
    uint32_t* d_tw_inv = nullptr; // [n][W] psi^-brev(k) R mod q
    uint32_t qinv = 0;            // -q^-1 mod 2^32
    ~WideTables();
};

// Tables of the quartic factorization (PM_QUARTIC, quartic.cu): q = B^4 - delta.
struct QuarticTables {
    uint32_t bbits = 0;            // B = 2^bbits
    uint32_t primes[16] = {};
    PrimeConst* d_pc = nullptr;    // [64] plane 4i + j: prime i
    uint2* d_tw_fwd = nullptr;     // [64][kNMax] psi_i^brev(k), plane 4i + j: prime i's table
    uint2* d_tw_inv = nullptr;
    uint8_t* d_conv = nullptr;     // [4][64 rows][128 B] conversion weights (channel evaluation folded in)
    uint8_t* d_crt = nullptr;      // [2][160 rows][128 B] CRT weights (components and quotient groups)
    uint2* d_mix = nullptr;        // [16] iota_i^-1; then [4][16] scale of component m, prime i
    uint32_t* d_ktab = nullptr;    // [4][33][W] k (-P 2^(bbits m)) mod q
    int fix_count = 0;             // straddling bytes at the part boundaries
    int fix_byte[3] = {}, fix_shift[3] = {};
    ~QuarticTables();
};

// Everything one (n, q) product needs on the device.
struct PlanCore {
    int device = 0;
    int sms = 148;           // streaming multiprocessors of the plan's device
    uint32_t n = 0, logn = 0, logR = 0, logC = 0;
    uint32_t P = 0;          // basis size
    uint32_t qbits = 0;
    uint32_t W = 0;          // q words rounded up to a multiple of 4 (kernel template width)
    uint32_t coef_limbs = 0, stride = 0;  // u64 limbs and u32 words per coefficient
    uint32_t flags = 0;
    Words q;
    uint64_t mu_q = 0;
    uint32_t delta = 0;      // q = 2^qbits - delta, delta < 2^32, PM_SPECIAL_FORM asked: folding reduction; else 0
    DeviceBasis* basis = nullptr;
    uint32_t* d_mq = nullptr;      // [P][W] (P_total/p_i) mod q
    uint32_t* d_consts = nullptr;  // q[W], (-P_total mod q)[W]
    uint32_t* d_ktab = nullptr;    // [2P+1][W] k (-P_total mod q) mod q: the CRT's quotient correction by table
    uint2* d_scale = nullptr;      // [2P] s_i = 2^32 n^-1 (P_total/p_i)^-1 mod p_i, then s_i psi_i^-brev(1)
    uint32_t* d_work = nullptr;    // [2][P][n] residue planes (plan-owned workspace)
    void* d_batch_work = nullptr;  // residue planes for a group of products (pm_multiply_batch)
    uint32_t batch_work_group = 0;
    size_t workspace_bytes = 0;
    size_t io_bytes = 0;           // bytes of one polynomial
    std::unique_ptr<HostCall> host;  // the host-buffer call's buffers and copy threads (first use)
    cudaStream_t stream = nullptr;
    // tensor path constants
    uint8_t* d_crt_weights = nullptr;
    uint64_t* d_kfrac = nullptr;   // [2P+1] floor(2^64 (k (-P_total mod q) mod q) / q)
    uint32_t* d_err = nullptr;     // set by a kernel whose bounded wait ran out
    uint32_t tensor_k_crt = 0;

    std::unique_ptr<WideTables> wide;  // set for PM_WIDE_NTT plans
    std::unique_ptr<QuarticTables> quartic;  // set for PM_QUARTIC plans

    // Per-plane tables the kernels index by residue plane: the device basis for the RNS
    // method, the plan's own for the quartic factorization (a plane per prime and channel).
    const PrimeConst* plane_pc() const;
    const uint2* plane_fwd() const;
    const uint2* plane_inv() const;
    const uint8_t* conv_weights() const;

    Tuning tune;
    std::unique_ptr<PipelineSlot> pipe[3];
    uint32_t pipe_group = 0;

    bool tables_only = false;      // set-up for a batch: no own workspace or stream

    void init(uint32_t n, const uint64_t* q64, uint32_t q_limbs, uint32_t coef_limbs, uint32_t flags);
    void init_tables_only(uint32_t n, const uint64_t* q64, uint32_t q_limbs, uint32_t coef_limbs, uint32_t flags);
    void ensure_batch_workspace(uint32_t group);
    void ensure_pipeline(uint32_t group);
    ~PlanCore();
};

void launch_simt(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                 uint32_t count, cudaStream_t st);
uint32_t group_size(const PlanCore& s);
void launch_rows(const PlanCore& s, uint32_t* work, uint32_t count, cudaStream_t st);
void check_device_errors(const PlanCore& s);
// Device-pointer arguments a kernel may touch: reachable from the device (not
// pageable host memory), 8-byte aligned (u64 coefficients; the kernels move 8
// and 16 bytes at a time), and 16-byte aligned on the tensor path (tensor maps
// of a, b and the residue workspace).  Throws PM_ERR_INVALID otherwise.
void check_device_pointers(const PlanCore& s, const void* a, const void* b, const void* c, const void* workspace);
// Calls on device pointers run on the caller's current device, which must be the
// plan's: its tables, twiddles, error word and workspace live there.  Throws
// PM_ERR_INVALID otherwise (nothing is launched).
void require_plan_device(const PlanCore& s);
// Host-buffer calls make the plan's device current for their duration and put
// the caller's device back afterwards.
struct DeviceScope {
    int previous = -1;
    explicit DeviceScope(int device);
    ~DeviceScope();
};
void launch_batch(const PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count,
                  uint32_t group, void* workspace, cudaStream_t st);
void launch_product(const PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, void* workspace,
                    cudaStream_t st);
void multiply_host(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c);
// the same call in two halves: begin stages a, b and queues everything on the plan's
// stream; end copies the product out (direct_out: a pinned c the product may land in)
void multiply_host_begin(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* direct_out = nullptr);
void multiply_host_end(PlanCore& s, uint64_t* c);
void multiply_host_batch(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count);

// direct wide-modulus NTT (wide.cu)
void wide_init(PlanCore& s);
size_t wide_workspace_bytes(const PlanCore& s);
void launch_wide(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                 uint32_t count, cudaStream_t st);

// tensor-core conversion / CRT (tensor.cu)
void tensor_init(PlanCore& s);
void tensor_release(PlanCore& s);

// quartic factorization (quartic.cu)
void quartic_init(PlanCore& s);
void launch_quartic(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                    uint32_t count, cudaStream_t st);
// The single-product host call's split: conversion of one polynomial (K1W plans only:
// conversion_splits), then the row and CRT kernels once both are converted.
bool conversion_splits(const PlanCore& s);
void launch_tensor_convert_poly(const PlanCore& s, const uint32_t* x, int poly, uint32_t* work, cudaStream_t st);
void launch_tensor_after_conversion(const PlanCore& s, uint32_t* c, uint32_t* work, uint32_t count, cudaStream_t st);
void launch_tensor(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                   uint32_t count, cudaStream_t st);

}  // namespace pm

// The C ABI's opaque plan handle.
struct pm_plan {
    pm::PlanCore core;
};
