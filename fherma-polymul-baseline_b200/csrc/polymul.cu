// Host side of the multiplier: the per-device prime basis, plans, the launch
// sequence of one product, and the C ABI declared in include/polymul.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/polymul.h"
#include "host_math.h"
#include "pm_device.cuh"
#include "pm_internal.h"
#include "rows_persistent.cuh"

namespace pm {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};

Failure::Failure(int s, std::string m) : std::runtime_error(m), status(s) {}

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Failure(PM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void count_launches(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// kernel timing (pm_profile_*)
// ---------------------------------------------------------------------------
namespace {
struct ProfileRecord {
    const char* name;
    cudaEvent_t start, stop;
};
std::mutex g_prof_mutex;
std::atomic<bool> g_prof_on{false};
std::vector<cudaEvent_t> g_prof_pool;
std::vector<ProfileRecord> g_prof_pending;
size_t g_prof_used = 0;
struct ProfileTotal {
    const char* name;
    uint64_t launches;
    double ms;
};
std::vector<ProfileTotal> g_prof_totals;
}  // namespace

ProfileScope::ProfileScope(const char* name, cudaStream_t st) : stream(st) {
    if (!g_prof_on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    if (g_prof_used + 2 > g_prof_pool.size()) return;
    ProfileRecord r{name, g_prof_pool[g_prof_used], g_prof_pool[g_prof_used + 1]};
    g_prof_used += 2;
    if (cudaEventRecord(r.start, st) != cudaSuccess) return;
    g_prof_pending.push_back(r);
    index = long(g_prof_pending.size()) - 1;
}

ProfileScope::~ProfileScope() {
    if (index < 0) return;
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    if (size_t(index) < g_prof_pending.size()) cudaEventRecord(g_prof_pending[index].stop, stream);
}

int profile_enable(uint32_t capacity) {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    g_prof_on = false;
    for (auto& r : g_prof_pending) {
        cudaEventSynchronize(r.stop);
    }
    for (auto e : g_prof_pool) cudaEventDestroy(e);
    g_prof_pool.clear();
    g_prof_pending.clear();
    g_prof_totals.clear();
    g_prof_used = 0;
    if (!capacity) return PM_OK;
    g_prof_pool.resize(2 * size_t(capacity));
    for (auto& e : g_prof_pool)
        if (cudaEventCreate(&e) != cudaSuccess) {
            g_prof_pool.clear();
            return fail(PM_ERR_CUDA, "cannot create profiling events");
        }
    g_prof_on = true;
    return PM_OK;
}

int profile_read(const char** names, uint64_t* launches, double* total_ms, uint32_t capacity, uint32_t* count) {
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    for (auto& r : g_prof_pending) {
        float ms = 0;
        if (cudaEventSynchronize(r.stop) != cudaSuccess || cudaEventElapsedTime(&ms, r.start, r.stop) != cudaSuccess)
            return fail(PM_ERR_CUDA, "profiling event failed");
        bool found = false;
        for (auto& t : g_prof_totals)
            if (t.name == r.name) {
                ++t.launches;
                t.ms += ms;
                found = true;
            }
        if (!found) g_prof_totals.push_back({r.name, 1, ms});
    }
    g_prof_pending.clear();
    g_prof_used = 0;
    *count = uint32_t(g_prof_totals.size());
    for (uint32_t i = 0; i < capacity && i < g_prof_totals.size(); ++i) {
        names[i] = g_prof_totals[i].name;
        launches[i] = g_prof_totals[i].launches;
        total_ms[i] = g_prof_totals[i].ms;
    }
    return PM_OK;
}

int fail(int status, const std::string& message) {
    g_last_error = message;
    return status;
}

// ---------------------------------------------------------------------------
// The prime basis: primes p = 1 mod 2^17 below 2^30, descending, with
// psi-merged bit-reversed twiddle tables of length 65536 per prime.  The table
// of a smaller ring n is the length-n prefix of the same table, so one copy
// per device serves every plan (the reference builds per-n tables,
// rns/host_setup.h:108-124).
// ---------------------------------------------------------------------------
namespace {
std::mutex g_basis_mutex;
std::vector<std::unique_ptr<DeviceBasis>> g_basis;  // index = device ordinal
}  // namespace

std::vector<uint32_t> make_primes() {
    std::vector<uint32_t> primes;
    const uint32_t order = 1u << (kLogNMax + 1);
    for (uint64_t cand = (uint64_t(1) << 30) - order + 1; primes.size() < unsigned(kPMax); cand -= order) {
        if (cand <= (uint64_t(1) << 29)) throw Failure(PM_ERR_UNSUPPORTED, "prime search ran below 2^29");
        if (is_prime32(uint32_t(cand))) primes.push_back(uint32_t(cand));
    }
    return primes;
}

namespace {
// psi of multiplicative order exactly 2 * 65536
uint32_t root_of_unity(uint32_t p) {
    const uint64_t order = uint64_t(2) << kLogNMax;
    for (uint32_t g = 2; g < 1000000; ++g) {
        const uint32_t root = powmod(g, (p - 1) / order, p);
        if (powmod(root, order / 2, p) == p - 1) return root;
    }
    throw Failure(PM_ERR_UNSUPPORTED, "no root of unity of order 2^17");
}
}  // namespace

PrimeConst prime_const(uint32_t p) {
    PrimeConst c{};
    c.p = p;
    c.two_p = 2 * p;
    c.mu = uint32_t((uint64_t(1) << 61) / p);
    uint32_t pinv = p;  // p^-1 mod 2^32 by Newton: p * p = 1 mod 8, each step doubles the bits
    for (int it = 0; it < 5; ++it) pinv *= 2u - p * pinv;
    c.pinv = pinv;
    c.recip = uint64_t(((unsigned __int128)1 << 64) / p);
    return c;
}

// Psi_rev[k] = psi^brev(k) and its inverse, with Shoup companions, k < 65536.
void twiddle_tables(uint32_t p, uint2* fwd, uint2* inv) {
    std::vector<uint32_t> ppow(kNMax), ipow(kNMax);
    const uint32_t psi = root_of_unity(p), ipsi = powmod(psi, p - 2, p);
    ppow[0] = ipow[0] = 1;
    for (int e = 1; e < kNMax; ++e) {
        ppow[e] = mulmod(ppow[e - 1], psi, p);
        ipow[e] = mulmod(ipow[e - 1], ipsi, p);
    }
    for (int k = 0; k < kNMax; ++k) {
        const uint32_t e = bit_reverse(uint32_t(k), kLogNMax);
        fwd[k] = make_uint2(ppow[e], shoup_of(ppow[e], p));
        inv[k] = make_uint2(ipow[e], shoup_of(ipow[e], p));
    }
}

DeviceBasis::~DeviceBasis() {
    cudaSetDevice(device);
    cudaFree(d_pc);
    cudaFree(d_tw_fwd);
    cudaFree(d_tw_inv);
    cudaFree(d_conv_pow);
}

DeviceBasis& basis_for_device(int device) {
    std::lock_guard<std::mutex> lock(g_basis_mutex);
    if (device < 0) throw Failure(PM_ERR_INVALID, "bad device ordinal");
    if (g_basis.size() <= size_t(device)) g_basis.resize(device + 1);
    if (g_basis[device]) return *g_basis[device];
    auto B = std::make_unique<DeviceBasis>();
    B->device = device;
    B->primes = make_primes();
    const size_t P = B->primes.size();
    std::vector<PrimeConst> pc(P);
    std::vector<uint2> fwd(P * kNMax), inv(P * kNMax), pow(P * kPowWords);
    B->inv1.assign(P, 0);
    auto fill = [&](size_t begin, size_t end) {
        for (size_t i = begin; i < end; ++i) {
            const uint32_t p = B->primes[i];
            twiddle_tables(p, fwd.data() + i * kNMax, inv.data() + i * kNMax);
            uint32_t w = 1;
            const uint32_t base = uint32_t((uint64_t(1) << 32) % p);
            for (int k = 0; k < kPowWords; ++k) {
                pow[i * kPowWords + k] = make_uint2(w, shoup_of(w, p));
                w = mulmod(w, base, p);
            }
            pc[i] = prime_const(p);
            B->inv1[i] = inv[i * kNMax + 1].x;
        }
    };
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt == 0 ? 1 : (nt > 16 ? 16 : nt);
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) pool.emplace_back(fill, P * t / nt, P * (t + 1) / nt);
    for (auto& th : pool) th.join();

    int previous = 0;
    cuda_check(cudaGetDevice(&previous), "cudaGetDevice");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaMalloc(&B->d_pc, P * sizeof(PrimeConst)), "allocate prime constants");
    cuda_check(cudaMalloc(&B->d_tw_fwd, fwd.size() * sizeof(uint2)), "allocate forward twiddles");
    cuda_check(cudaMalloc(&B->d_tw_inv, inv.size() * sizeof(uint2)), "allocate inverse twiddles");
    cuda_check(cudaMalloc(&B->d_conv_pow, pow.size() * sizeof(uint2)), "allocate limb powers");
    cuda_check(cudaMemcpy(B->d_pc, pc.data(), P * sizeof(PrimeConst), cudaMemcpyHostToDevice), "upload primes");
    cuda_check(cudaMemcpy(B->d_tw_fwd, fwd.data(), fwd.size() * sizeof(uint2), cudaMemcpyHostToDevice),
               "upload forward twiddles");
    cuda_check(cudaMemcpy(B->d_tw_inv, inv.data(), inv.size() * sizeof(uint2), cudaMemcpyHostToDevice),
               "upload inverse twiddles");
    cuda_check(cudaMemcpy(B->d_conv_pow, pow.data(), pow.size() * sizeof(uint2), cudaMemcpyHostToDevice),
               "upload limb powers");
    cuda_check(cudaSetDevice(previous), "cudaSetDevice");
    g_basis[device] = std::move(B);
    return *g_basis[device];
}

// Smallest prefix of the basis with product above 2^(2*bits(q) + 2 + log2 n):
// the negacyclic coefficients lie in (-n(q-1)^2, n(q-1)^2), and a quarter of
// the CRT range is what the nearest-quotient correction needs
// (rns/host_setup.h:81-83 checks P > 4N(q-1)^2 the same way).
unsigned basis_size(const std::vector<uint32_t>& primes, unsigned n, unsigned qbits) {
    unsigned logn = 0;
    while ((1u << logn) < n) ++logn;
    const unsigned need = 2 * qbits + 2 + logn + 1;  // bit_length(P) >= need  <=>  P > 2^(need-1)
    Words P{1};
    for (unsigned i = 0; i < primes.size(); ++i) {
        P = multiply_small(P, primes[i]);
        if (bit_length(P) >= need) return i + 1;
    }
    throw Failure(PM_ERR_UNSUPPORTED, "q too wide for the prime basis");
}

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------
PlanCore::~PlanCore() {
    int previous = 0;
    cudaGetDevice(&previous);
    cudaSetDevice(device);
    cudaFree(d_mq);
    cudaFree(d_consts);
    cudaFree(d_ktab);
    cudaFree(d_scale);
    for (auto& sl : pipe) sl.reset();
    tensor_release(*this);
    wide.reset();
    cudaFree(d_err);
    cudaFree(d_work);
    cudaFree(d_batch_work);
    host.reset();
    if (stream) cudaStreamDestroy(stream);
    cudaSetDevice(previous);
}

void PlanCore::init(uint32_t n_, const uint64_t* q64, uint32_t q_limbs, uint32_t coef_limbs_, uint32_t flags_) {
    if (!q64 || q_limbs == 0) throw Failure(PM_ERR_INVALID, "q is missing");
    if (n_ < 2 || (n_ & (n_ - 1))) throw Failure(PM_ERR_INVALID, "n must be a power of two >= 2");
    if (n_ > uint32_t(kNMax)) throw Failure(PM_ERR_UNSUPPORTED, "n above 65536");
    if (flags_ & ~uint32_t(PM_CONVERT_TENSOR | PM_CONVERT_SIMT | PM_SPECIAL_FORM | PM_WIDE_NTT | PM_QUARTIC))
        throw Failure(PM_ERR_INVALID, "unknown flags");
    if ((flags_ & PM_QUARTIC) && (flags_ & (PM_CONVERT_SIMT | PM_WIDE_NTT)))
        throw Failure(PM_ERR_INVALID, "PM_QUARTIC runs on the tensor path only");
    if ((flags_ & PM_CONVERT_TENSOR) && (flags_ & PM_CONVERT_SIMT))
        throw Failure(PM_ERR_INVALID, "PM_CONVERT_TENSOR and PM_CONVERT_SIMT exclude each other");
    // no path asked for: the tensor path wherever its 16-byte coefficient rows exist
    if (!(flags_ & (PM_CONVERT_TENSOR | PM_CONVERT_SIMT | PM_WIDE_NTT)) && coef_limbs_ % 2 == 0)
        flags_ |= PM_CONVERT_TENSOR;
    q.assign(2 * q_limbs, 0);
    for (uint32_t i = 0; i < q_limbs; ++i) {
        q[2 * i] = uint32_t(q64[i]);
        q[2 * i + 1] = uint32_t(q64[i] >> 32);
    }
    trim(q);
    qbits = bit_length(q);
    if (qbits < 2 || !(q[0] & 1)) throw Failure(PM_ERR_INVALID, "q must be odd and at least 3");
    if (qbits > 32u * kWMax) throw Failure(PM_ERR_UNSUPPORTED, "q wider than 896 bits");
    const uint32_t qwords = (qbits + 31) / 32;
    if (uint64_t(coef_limbs_) * 64 < qbits) throw Failure(PM_ERR_INVALID, "coef_limbs too small for q");
    if (coef_limbs_ > 64) throw Failure(PM_ERR_UNSUPPORTED, "coef_limbs above 64");
    n = n_;
    logn = 0;
    while ((1u << logn) < n) ++logn;
    // rows of the R x C view: 32 for the SIMT path (column stages across warp
    // lanes), 16 for the tensor path (column stages in registers)
    const uint32_t maxlogR = (flags_ & PM_CONVERT_TENSOR) ? 4 : 5;
    logR = logn < maxlogR ? logn : maxlogR;
    logC = logn - logR;
    coef_limbs = coef_limbs_;
    stride = 2 * coef_limbs;
    W = (qwords + 3) / 4 * 4;
    if (W < 4) W = 4;
    flags = flags_;
    cuda_check(cudaGetDevice(&device), "cudaGetDevice");
    basis = &basis_for_device(device);
    P = basis_size(basis->primes, n, qbits);

    // CRT constants: (P_total / p_i) mod q, (-P_total) mod q,
    // scale = 2^32 n^-1 (P/p_i)^-1 mod p_i (2^32 undoes the Montgomery product of K2)
    Words total{1};
    for (unsigned i = 0; i < P; ++i) total = multiply_small(total, basis->primes[i]);
    std::vector<uint32_t> mq(size_t(P) * W, 0), consts(2 * size_t(W), 0);
    std::vector<uint2> scale(2 * size_t(P));
    for (unsigned i = 0; i < P; ++i) {
        const uint32_t p = basis->primes[i];
        Words m = total;
        if (divide_small(m, p)) throw Failure(PM_ERR_UNSUPPORTED, "basis product not divisible");
        const Words mmod = padded(mod(m, q), W);
        std::copy(mmod.begin(), mmod.end(), mq.begin() + size_t(i) * W);
        const uint32_t minv = powmod(mod_small(m, p), p - 2, p);
        const uint32_t ninv = powmod(n % p, p - 2, p);
        const uint32_t r32 = uint32_t((uint64_t(1) << 32) % p);
        const uint32_t s = mulmod(mulmod(minv, ninv, p), r32, p);
        scale[i] = make_uint2(s, shoup_of(s, p));
        const uint32_t sw = mulmod(s, basis->inv1[i], p);  // the tensor CRT folds s_i into its last stage
        scale[P + i] = make_uint2(sw, shoup_of(sw, p));
    }
    const Words qpad = padded(q, W);
    Words pmod = mod(total, q);
    const Words pneg = padded(compare(pmod, Words{}) == 0 ? Words{} : subtract(q, pmod), W);
    std::copy(qpad.begin(), qpad.end(), consts.begin());
    std::copy(pneg.begin(), pneg.end(), consts.begin() + W);
    // k (-P mod q) mod q for every nearest quotient k the CRT can meet: k <= sum t_i / p_i + 1/2
    // with digits t_i < 2 p_i, so k <= 2P
    std::vector<uint32_t> ktab(size_t(2 * P + 1) * W, 0);
    for (unsigned k = 1; k <= 2 * P; ++k) {
        const Words row = padded(mod(multiply_small(pneg, k), q), W);
        std::copy(row.begin(), row.end(), ktab.begin() + size_t(k) * W);
    }
    // mu_q = floor(2^(qbits + 62) / q)
    Words quo;
    Words num(((qbits + 62) / 32) + 1, 0);
    num[(qbits + 62) / 32] = 1u << ((qbits + 62) % 32);
    divmod(num, q, &quo, nullptr);
    quo.resize(2, 0);
    mu_q = (uint64_t(quo[1]) << 32) | quo[0];
    // special form q = 2^qbits - delta, delta < 2^32 (on request): the CRT folds 2^qbits = delta
    delta = 0;
    if (qbits >= 80 && (flags & PM_SPECIAL_FORM)) {
        Words top(qbits / 32 + 1, 0);
        top[qbits / 32] = 1u << (qbits % 32);
        const Words d = subtract(top, q);
        if (bit_length(d) <= 32) delta = d.empty() ? 0u : d[0];
    }

    if (flags & PM_QUARTIC) quartic_init(*this);  // 64 planes (16 primes x 4 channels), its own tables
    workspace_bytes = size_t(2) * P * n * sizeof(uint32_t);
    if (flags & PM_WIDE_NTT) {
        wide_init(*this);
        workspace_bytes = std::max(workspace_bytes, wide_workspace_bytes(*this));
    }
    io_bytes = size_t(n) * coef_limbs * sizeof(uint64_t);
    cuda_check(cudaMalloc(&d_mq, mq.size() * 4), "allocate CRT rows");
    cuda_check(cudaMalloc(&d_consts, consts.size() * 4), "allocate q constants");
    cuda_check(cudaMalloc(&d_scale, scale.size() * sizeof(uint2)), "allocate CRT scales");
    cuda_check(cudaMemcpy(d_mq, mq.data(), mq.size() * 4, cudaMemcpyHostToDevice), "upload CRT rows");
    cuda_check(cudaMemcpy(d_consts, consts.data(), consts.size() * 4, cudaMemcpyHostToDevice), "upload q");
    cuda_check(cudaMalloc(&d_ktab, ktab.size() * 4), "allocate CRT correction table");
    cuda_check(cudaMemcpy(d_ktab, ktab.data(), ktab.size() * 4, cudaMemcpyHostToDevice), "upload CRT correction table");
    cuda_check(cudaMemcpy(d_scale, scale.data(), scale.size() * sizeof(uint2), cudaMemcpyHostToDevice),
               "upload CRT scales");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    if (sms <= 0) sms = 148;
    cuda_check(cudaMalloc(&d_err, sizeof(uint32_t)), "allocate error word");
    cuda_check(cudaMemset(d_err, 0, sizeof(uint32_t)), "clear error word");
    if ((flags & PM_CONVERT_TENSOR) && !quartic) tensor_init(*this);
    if (tables_only) return;
    cuda_check(cudaMalloc(&d_work, workspace_bytes), "allocate residue workspace");
    cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "create plan stream");
}

void PlanCore::init_tables_only(uint32_t n_, const uint64_t* q64, uint32_t q_limbs, uint32_t coef_limbs_,
                                uint32_t flags_) {
    tables_only = true;
    init(n_, q64, q_limbs, coef_limbs_, flags_);
}

void PlanCore::ensure_batch_workspace(uint32_t group) {
    if (batch_work_group >= group) return;
    cuda_check(cudaStreamSynchronize(stream), "drain plan stream");
    cudaFree(d_batch_work);
    d_batch_work = nullptr;
    batch_work_group = 0;
    cuda_check(cudaMalloc(&d_batch_work, workspace_bytes * group), "allocate batch workspace");
    batch_work_group = group;
}

// ---------------------------------------------------------------------------
// launch sequence of one product: K1 -> K2 -> K3 on one stream
// ---------------------------------------------------------------------------
namespace {
struct Batch {
    uint32_t count;     // products in this launch
    size_t io_bstride;  // words between consecutive products' a (b, c)
    size_t ws_bstride;  // words between consecutive products' residue planes
};

template <int W>
void launch_k1(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* work, const Batch& bt,
               cudaStream_t st) {
    const int G = s.logC >= 3 ? 8 : (1 << s.logC);
    const int groups = s.P >= 32 ? 4 : (s.P >= 16 ? 2 : 1);
    const int ppc = int((s.P + groups - 1) / groups);
    dim3 grid((1u << s.logC) / G, 2 * bt.count, (s.P + ppc - 1) / ppc), block((1u << s.logR) * G);
    const size_t smem = size_t(ppc) * W * sizeof(uint2);
    k1_convert_cols<W><<<grid, block, smem, st>>>(a, b, work, s.basis->d_pc, s.basis->d_conv_pow, s.basis->d_tw_fwd,
                                                  int(s.n), int(s.logR), int(s.logC), int(s.P), int(s.stride), ppc,
                                                  bt.io_bstride, bt.ws_bstride);
}

template <int W>
void launch_k3(const PlanCore& s, const uint32_t* work, uint32_t* c, const Batch& bt, cudaStream_t st) {
    const int G = s.logC >= 3 ? 8 : (1 << s.logC);
    const int RG = (1 << s.logR) * G;
    dim3 grid((1u << s.logC) / G, bt.count), block(RG);
    const size_t smem = (size_t(s.P) * W + size_t(s.P) * RG) * 4;
    if (smem > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(k3_cols_crt<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "raise K3 shared memory");
    k3_cols_crt<W><<<grid, block, smem, st>>>(work, c, s.basis->d_pc, s.basis->d_tw_inv, s.d_scale, s.d_mq,
                                              s.d_consts, s.d_ktab, s.mu_q, int(s.qbits), s.delta, int(s.n),
                                              int(s.logR),
                                              int(s.logC),
                                              int(s.P), int(s.stride), bt.io_bstride, bt.ws_bstride);
}

template <int LOGC, int KP>
void launch_k2_fixed(const PlanCore& s, uint32_t* work, const Batch& bt, cudaStream_t st) {
    constexpr int C = 1 << LOGC, T = C / 8;
    if constexpr (LOGC >= 10) {
        // bulk copies need 16-byte aligned rows (n, C and the product stride are multiples of 4 words)
        if (s.tune.row_persistent && (reinterpret_cast<uintptr_t>(work) & 15) == 0 && (bt.ws_bstride & 3) == 0) {
            const size_t smem = k2p_smem_bytes(LOGC);
            cuda_check(cudaFuncSetAttribute(k2p_rows<LOGC, KP, PlanRowWork>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(smem)),
                       "raise K2P shared memory");
            const int64_t items = int64_t(s.P) << s.logR;
            const int64_t total = items * bt.count;
            const int ctas = int(std::min<int64_t>(total, int64_t(s.sms) * k2p_min_blocks(LOGC)));
            const PlanRowWork w{work, bt.ws_bstride, int(s.n), int(s.logR), int(s.logC), int(s.P), int(bt.count)};
            k2p_rows<LOGC, KP, PlanRowWork><<<ctas, k2p_threads(LOGC, KP), smem, st>>>(
                w, s.plane_pc(), s.plane_fwd(), s.plane_inv(), int(s.logR), s.d_err);
            return;
        }
    }
    if constexpr (KP == 4) {  // radix-16 passes exist in the persistent kernel only
        launch_k2_fixed<LOGC, 3>(s, work, bt, st);
    } else {
        int rows = T >= 128 ? 1 : 128 / T;
        const int R = 1 << s.logR;
        if (rows > R) rows = R;
        const size_t smem = size_t(rows) * 24 * C;  // 2C uint2 twiddles + 2C words of data per row
        if (smem > 48 * 1024)
            cuda_check(cudaFuncSetAttribute(k2_rows<LOGC, KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                       "raise K2 shared memory");
        dim3 grid(R / rows, s.P, bt.count), block(rows * T);
        k2_rows<LOGC, KP><<<grid, block, smem, st>>>(work, s.plane_pc(), s.plane_fwd(), s.plane_inv(),
                                                     int(s.n), int(s.logR), int(s.P), bt.ws_bstride);
    }
}

template <int LOGC>
void launch_k2_radix(const PlanCore& s, uint32_t* work, const Batch& bt, cudaStream_t st) {
    if (s.tune.row_radix_log == 2)
        launch_k2_fixed<LOGC, 2>(s, work, bt, st);
    else if (LOGC >= 10 && s.tune.row_radix_log == 4)
        launch_k2_fixed<LOGC, LOGC >= 10 ? 4 : 3>(s, work, bt, st);
    else
        launch_k2_fixed<LOGC, 3>(s, work, bt, st);
}

void launch_k2(const PlanCore& s, uint32_t* work, const Batch& bt, cudaStream_t st) {
    switch (s.logC) {
        case 12: return launch_k2_radix<12>(s, work, bt, st);
        case 3: return launch_k2_fixed<3, 3>(s, work, bt, st);
        case 4: return launch_k2_radix<4>(s, work, bt, st);
        case 5: return launch_k2_radix<5>(s, work, bt, st);
        case 6: return launch_k2_radix<6>(s, work, bt, st);
        case 7: return launch_k2_radix<7>(s, work, bt, st);
        case 8: return launch_k2_radix<8>(s, work, bt, st);
        case 9: return launch_k2_radix<9>(s, work, bt, st);
        case 10: return launch_k2_radix<10>(s, work, bt, st);
        case 11: return launch_k2_radix<11>(s, work, bt, st);
        default: {
            const int R = 1 << s.logR;
            dim3 grid((R + 31) / 32, s.P, bt.count), block(R < 32 ? R : 32);
            k2_rows_small<<<grid, block, 0, st>>>(work, s.plane_pc(), s.plane_fwd(), s.plane_inv(),
                                                 int(s.n), int(s.logR), int(s.logC), int(s.P), bt.ws_bstride);
        }
    }
}

#define PM_DISPATCH_W(W_, CALL)                                          \
    switch (W_) {                                                       \
        case 4: CALL(4); break;                                         \
        case 8: CALL(8); break;                                         \
        case 12: CALL(12); break;                                       \
        case 16: CALL(16); break;                                       \
        case 20: CALL(20); break;                                       \
        case 24: CALL(24); break;                                       \
        case 28: CALL(28); break;                                       \
        default: throw Failure(PM_ERR_UNSUPPORTED, "unsupported width"); \
    }
}  // namespace

void launch_rows(const PlanCore& s, uint32_t* work, uint32_t count, cudaStream_t st) {
    launch_k2(s, work, Batch{count, size_t(s.n) * s.stride, s.workspace_bytes / 4}, st);
}

void launch_simt(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                 uint32_t count, cudaStream_t st) {
    const Batch bt{count, size_t(s.n) * s.stride, s.workspace_bytes / 4};
    {
        ProfileScope prof("k1_convert_cols", st);
#define PM_K1(W) launch_k1<W>(s, a, b, work, bt, st)
        PM_DISPATCH_W(s.W, PM_K1)
#undef PM_K1
    }
    {
        ProfileScope prof("k2_rows", st);
        launch_k2(s, work, bt, st);
    }
    {
        ProfileScope prof("k3_cols_crt", st);
#define PM_K3(W) launch_k3<W>(s, work, c, bt, st)
        PM_DISPATCH_W(s.W, PM_K3)
#undef PM_K3
    }
    cuda_check(cudaGetLastError(), "launch product kernels");
    count_launches(3);
}

void check_device_pointers(const PlanCore& s, const void* a, const void* b, const void* c, const void* workspace) {
    const void* ptrs[4] = {a, b, c, workspace};
    const char* names[4] = {"a", "b", "c", "workspace"};
    for (int i = 0; i < 4; ++i) {
        if (!ptrs[i]) continue;
        const uintptr_t addr = reinterpret_cast<uintptr_t>(ptrs[i]);
        // tensor path: tensor maps over a, b and the workspace; wide NTT: 16-byte workspace loads
        const bool tensor = (s.flags & PM_CONVERT_TENSOR) != 0;
        const uintptr_t need = (tensor && i != 2) || (s.wide && i == 3) ? 16 : 8;
        if (addr % need)
            throw Failure(PM_ERR_INVALID, std::string(names[i]) + " must be " + std::to_string(need) +
                                              "-byte aligned");
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ptrs[i]) != cudaSuccess) {
            cudaGetLastError();
            throw Failure(PM_ERR_INVALID, std::string(names[i]) + " is not a pointer the device can use");
        }
        if (at.type == cudaMemoryTypeUnregistered)
            throw Failure(PM_ERR_INVALID, std::string(names[i]) +
                                              " is pageable host memory: pass device, managed or pinned memory");
        if (at.type == cudaMemoryTypeDevice && at.device != s.device)
            throw Failure(PM_ERR_INVALID, std::string(names[i]) + " is memory of device " + std::to_string(at.device) +
                                              ", the plan belongs to device " + std::to_string(s.device));
    }
}

void require_plan_device(const PlanCore& s) {
    int device = -1;
    cuda_check(cudaGetDevice(&device), "cudaGetDevice");
    if (device != s.device)
        throw Failure(PM_ERR_INVALID, "the current device is " + std::to_string(device) + ", the plan belongs to device " +
                                          std::to_string(s.device) + ": make the plan's device current first");
}

DeviceScope::DeviceScope(int device) {
    cuda_check(cudaGetDevice(&previous), "cudaGetDevice");
    if (previous != device) cuda_check(cudaSetDevice(device), "cudaSetDevice");
}

DeviceScope::~DeviceScope() {
    int now = -1;
    if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous) cudaSetDevice(previous);
}

const PrimeConst* PlanCore::plane_pc() const { return quartic ? quartic->d_pc : basis->d_pc; }
const uint2* PlanCore::plane_fwd() const { return quartic ? quartic->d_tw_fwd : basis->d_tw_fwd; }
const uint2* PlanCore::plane_inv() const { return quartic ? quartic->d_tw_inv : basis->d_tw_inv; }
const uint8_t* PlanCore::conv_weights() const { return quartic ? quartic->d_conv : basis->d_conv_weights; }

// A kernel that gave up a bounded wait records it in the plan's error word.
void check_device_errors(const PlanCore& s) {
    if (!s.d_err) return;
    uint32_t err = 0;
    cuda_check(cudaMemcpy(&err, s.d_err, sizeof err, cudaMemcpyDeviceToHost), "read error word");
    if (err) {
        cudaMemset(s.d_err, 0, sizeof err);
        throw Failure(PM_ERR_TIMEOUT, "a tensor-core wait timed out; results of that call are invalid");
    }
}

// Products per launch group when the plan is not tuned: residue planes of up
// to about 2 GB (128 products at N=32768).  Larger groups measured faster on
// B200 although their planes no longer fit in L2: each persistent kernel
// amortizes its per-CTA set-up (twiddle staging, CRT weights) and its tail over
// more items (at N=32768, 128 products a group ran 2% faster than 64, 256 no
// faster than 128), and the row kernel's DRAM traffic stays at its algorithmic
// bytes.
uint32_t group_size(const PlanCore& s) {
    if (s.tune.group) return s.tune.group;
    const size_t budget = size_t(2) << 30;
    size_t g = budget / s.workspace_bytes;
    if (g < 1) g = 1;
    if (g > kMaxDefaultGroup) g = kMaxDefaultGroup;
    return uint32_t(g);
}

void launch_batch(const PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count,
                  uint32_t group, void* workspace, cudaStream_t st) {
    uint32_t* work = static_cast<uint32_t*>(workspace);
    const size_t io_words = size_t(s.n) * s.stride;
    for (uint32_t z = 0; z < count; z += group) {
        const uint32_t g = count - z < group ? count - z : group;
        const uint32_t* a32 = reinterpret_cast<const uint32_t*>(a) + z * io_words;
        const uint32_t* b32 = reinterpret_cast<const uint32_t*>(b) + z * io_words;
        uint32_t* c32 = reinterpret_cast<uint32_t*>(c) + z * io_words;
        if (s.wide)
            launch_wide(s, a32, b32, c32, work, g, st);
        else if (s.quartic)
            launch_quartic(s, a32, b32, c32, work, g, st);
        else if (s.flags & PM_CONVERT_TENSOR)
            launch_tensor(s, a32, b32, c32, work, g, st);
        else
            launch_simt(s, a32, b32, c32, work, g, st);
    }
}

void launch_product(const PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, void* workspace,
                    cudaStream_t st) {
    launch_batch(s, a, b, c, 1, 1, workspace ? workspace : s.d_work, st);
}

// ---------------------------------------------------------------------------
// host batches: chunks of `group` products rotate over three slots, each with
// its own stream, device buffers and workspace, so one slot's H2D, another's
// kernels and a third's D2H run at the same time.  Pageable buffers are staged
// through the slot's pinned memory by the calling thread.
// ---------------------------------------------------------------------------
PipelineSlot::~PipelineSlot() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_buf);
    cudaFreeHost(h_buf);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
}

void PlanCore::ensure_pipeline(uint32_t group) {
    if (pipe_group >= group && pipe[0]) return;
    for (auto& sl : pipe) sl.reset();
    pipe_group = 0;
    for (auto& sl : pipe) {
        sl = std::make_unique<PipelineSlot>();
        cuda_check(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking), "pipeline stream");
        cuda_check(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming), "pipeline event");
        cuda_check(cudaMalloc(&sl->d_buf, size_t(group) * (3 * io_bytes + workspace_bytes)), "pipeline buffers");
        cuda_check(cudaMallocHost(&sl->h_buf, size_t(group) * 3 * io_bytes), "pipeline staging");
        sl->pending = false;
    }
    pipe_group = group;
}

void multiply_host_batch(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count) {
    if (!count) return;
    // Chunks of at most kHostChunk products: the copies, not the kernels, bound
    // this call (a chunk's kernels take a fraction of its H2D time).  Each copy
    // costs the link a few microseconds on top of its bytes, so the steady state
    // moves 16 products a chunk (N = 32768: 98% of the measured both-directions
    // PCIe bound, against 91% with chunks of 4; 32 and 64 measured lower), and
    // the ramp below keeps the fill and drain short.
    constexpr uint32_t kHostChunk = 16;
    uint32_t g = std::min(group_size(s), kHostChunk);
    if (g > count) g = count;
    s.ensure_pipeline(g);
    auto pinned = [](const void* p) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    const bool pa = pinned(a), pb = pinned(b), pc = pinned(c);
    const size_t io = s.io_bytes;
    struct Out {
        uint8_t* dst;
        const uint8_t* staged;
        size_t bytes;
    };
    Out outs[3] = {};
    const uint8_t* A = reinterpret_cast<const uint8_t*>(a);
    const uint8_t* B = reinterpret_cast<const uint8_t*>(b);
    uint8_t* Cc = reinterpret_cast<uint8_t*>(c);
    // chunk sizes ramp 1, 2, .. up to g and back down at the end: the first H2D and the
    // last D2H, which nothing overlaps, move one product instead of g
    std::vector<uint32_t> chunks, tail;
    {
        uint32_t left = count;
        for (uint32_t sz = 1; sz < g && left > 2 * g; sz *= 2) {
            chunks.push_back(sz);
            left -= sz;
        }
        for (uint32_t sz = 1; sz < g && left > g + sz; sz *= 2) {
            tail.push_back(sz);
            left -= sz;
        }
        while (left) {
            const uint32_t sz = left < g ? left : g;
            chunks.push_back(sz);
            left -= sz;
        }
        chunks.insert(chunks.end(), tail.rbegin(), tail.rend());
    }
    uint32_t k = 0, z = 0;
    for (const uint32_t cnt : chunks) {
        PipelineSlot& sl = *s.pipe[k % 3];
        const size_t bytes = size_t(cnt) * io;
        if (sl.pending) {  // the slot's previous chunk must be out before its buffers are reused
            cuda_check(cudaEventSynchronize(sl.done), "pipeline chunk");
            Out& o = outs[k % 3];
            if (o.staged) std::memcpy(o.dst, o.staged, o.bytes);
            sl.pending = false;
        }
        uint8_t* dev = static_cast<uint8_t*>(sl.d_buf);
        uint8_t* stage = static_cast<uint8_t*>(sl.h_buf);
        uint8_t *da = dev, *db = dev + size_t(g) * io, *dc = dev + 2 * size_t(g) * io;
        void* ws = dev + 3 * size_t(g) * io;
        const void* sa = A + size_t(z) * io;
        const void* sb = B + size_t(z) * io;
        if (!pa) {
            std::memcpy(stage, sa, bytes);
            sa = stage;
        }
        if (!pb) {
            std::memcpy(stage + size_t(g) * io, sb, bytes);
            sb = stage + size_t(g) * io;
        }
        cuda_check(cudaMemcpyAsync(da, sa, bytes, cudaMemcpyHostToDevice, sl.stream), "batch a to device");
        cuda_check(cudaMemcpyAsync(db, sb, bytes, cudaMemcpyHostToDevice, sl.stream), "batch b to device");
        launch_batch(s, reinterpret_cast<const uint64_t*>(da), reinterpret_cast<const uint64_t*>(db),
                     reinterpret_cast<uint64_t*>(dc), cnt, g, ws, sl.stream);
        uint8_t* out = Cc + size_t(z) * io;
        uint8_t* land = pc ? out : stage + 2 * size_t(g) * io;
        cuda_check(cudaMemcpyAsync(land, dc, bytes, cudaMemcpyDeviceToHost, sl.stream), "batch c to host");
        cuda_check(cudaEventRecord(sl.done, sl.stream), "pipeline event");
        outs[k % 3] = Out{out, pc ? nullptr : land, bytes};
        sl.pending = true;
        z += cnt;
        ++k;
    }
    for (int i = 0; i < 3; ++i) {
        PipelineSlot& sl = *s.pipe[i];
        if (!sl.pending) continue;
        cuda_check(cudaEventSynchronize(sl.done), "pipeline drain");
        if (outs[i].staged) std::memcpy(outs[i].dst, outs[i].staged, outs[i].bytes);
        sl.pending = false;
    }
    check_device_errors(s);
}

}  // namespace pm

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using pm::fail;
using pm::Failure;

#define PM_GUARD(body)                                                   \
    try {                                                                \
        body;                                                            \
        return PM_OK;                                                    \
    } catch (const Failure& f) {                                         \
        return fail(f.status, f.what());                                 \
    } catch (const std::bad_alloc&) {                                    \
        return fail(PM_ERR_NO_MEMORY, "host allocation failed");         \
    } catch (const std::exception& e) {                                  \
        return fail(PM_ERR_INVALID, e.what());                           \
    }

extern "C" int pm_plan_create(pm_plan** plan, uint32_t n, const uint64_t* q, uint32_t q_limbs, uint32_t coef_limbs,
                              uint32_t flags) {
    if (!plan) return fail(PM_ERR_INVALID, "plan pointer is NULL");
    *plan = nullptr;
    PM_GUARD({
        auto p = std::make_unique<pm_plan>();
        p->core.init(n, q, q_limbs, coef_limbs, flags);
        *plan = p.release();
    })
}

extern "C" int pm_plan_get_info(const pm_plan* plan, pm_plan_info* info) {
    if (!plan || !info) return fail(PM_ERR_INVALID, "NULL argument");
    const auto& s = plan->core;
    info->n = s.n;
    info->q_bits = s.qbits;
    info->coef_limbs = s.coef_limbs;
    info->primes = s.P;
    info->convert = s.wide ? 0u : ((s.flags & PM_CONVERT_TENSOR) ? uint32_t(PM_CONVERT_TENSOR) : uint32_t(PM_CONVERT_SIMT));
    info->reserved = 0;
    info->workspace_bytes = s.workspace_bytes;
    return PM_OK;
}

extern "C" int pm_plan_destroy(pm_plan* plan) {
    if (!plan) return PM_OK;
    PM_GUARD({
        cudaStreamSynchronize(plan->core.stream);
        delete plan;
    })
}

extern "C" int pm_multiply(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, void* workspace,
                           pm_stream stream) {
    if (!plan || !a || !b || !c) return fail(PM_ERR_INVALID, "NULL argument");
    PM_GUARD({
        pm::require_plan_device(plan->core);
        pm::check_device_pointers(plan->core, a, b, c, workspace);
        pm::launch_product(plan->core, a, b, c, workspace, reinterpret_cast<cudaStream_t>(stream));
    })
}

extern "C" int pm_batch_workspace_size(const pm_plan* plan, uint32_t count, size_t* bytes) {
    if (!plan || !bytes) return fail(PM_ERR_INVALID, "NULL argument");
    const uint32_t g = pm::group_size(plan->core);
    *bytes = plan->core.workspace_bytes * (count < g ? (count ? count : 1) : g);
    return PM_OK;
}

extern "C" int pm_multiply_batch(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c, uint32_t count,
                                 void* workspace, size_t workspace_bytes, pm_stream stream) {
    if (!plan || !a || !b || !c) return fail(PM_ERR_INVALID, "NULL argument");
    if (count == 0) return PM_OK;
    PM_GUARD({
        auto& s = plan->core;
        pm::require_plan_device(s);
        pm::check_device_pointers(s, a, b, c, workspace);
        uint32_t g = pm::group_size(s);
        if (g > count) g = count;
        if (workspace) {
            const size_t fit = workspace_bytes / s.workspace_bytes;
            if (fit == 0) throw Failure(PM_ERR_INVALID, "workspace smaller than one product needs");
            if (fit < g) g = uint32_t(fit);
        } else {
            s.ensure_batch_workspace(g);
            workspace = s.d_batch_work;
        }
        pm::launch_batch(s, a, b, c, count, g, workspace, reinterpret_cast<cudaStream_t>(stream));
    })
}

extern "C" int pm_multiply_host_batch(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c,
                                      uint32_t count) {
    if (!plan || !a || !b || !c) return fail(PM_ERR_INVALID, "NULL argument");
    PM_GUARD({
        pm::DeviceScope on(plan->core.device);
        pm::multiply_host_batch(plan->core, a, b, c, count);
    })
}

extern "C" int pm_multiply_host(pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c) {
    if (!plan || !a || !b || !c) return fail(PM_ERR_INVALID, "NULL argument");
    PM_GUARD({
        pm::DeviceScope on(plan->core.device);
        pm::multiply_host(plan->core, a, b, c);
    })
}

extern "C" int pm_multiply_host_begin(pm_plan* plan, const uint64_t* a, const uint64_t* b) {
    if (!plan || !a || !b) return fail(PM_ERR_INVALID, "NULL argument");
    PM_GUARD({
        pm::DeviceScope on(plan->core.device);
        pm::multiply_host_begin(plan->core, a, b);
    })
}

extern "C" int pm_multiply_host_end(pm_plan* plan, uint64_t* c) {
    if (!plan || !c) return fail(PM_ERR_INVALID, "NULL argument");
    PM_GUARD({
        pm::DeviceScope on(plan->core.device);
        pm::multiply_host_end(plan->core, c);
    })
}

extern "C" int pm_basis_query(uint32_t n, uint32_t q_bits, uint32_t* primes, uint32_t capacity, uint32_t* count) {
    if (!count) return fail(PM_ERR_INVALID, "count pointer is NULL");
    *count = 0;
    if (n < 2 || (n & (n - 1))) return fail(PM_ERR_INVALID, "n must be a power of two >= 2");
    if (n > uint32_t(pm::kNMax)) return fail(PM_ERR_UNSUPPORTED, "n above 65536");
    if (q_bits < 2 || q_bits > 32u * pm::kWMax) return fail(PM_ERR_UNSUPPORTED, "q_bits outside [2, 896]");
    PM_GUARD({
        static const std::vector<uint32_t> all = pm::make_primes();
        const unsigned k = pm::basis_size(all, n, q_bits);
        *count = k;
        for (unsigned i = 0; i < k && i < capacity; ++i) primes[i] = all[i];
    })
}

extern "C" const char* pm_status_string(int status) {
    switch (status) {
        case PM_OK: return "ok";
        case PM_ERR_INVALID: return "invalid argument";
        case PM_ERR_UNSUPPORTED: return "unsupported parameters";
        case PM_ERR_CUDA: return "CUDA error";
        case PM_ERR_NO_MEMORY: return "out of memory";
        case PM_ERR_TIMEOUT: return "timed out";
        case PM_ERR_BUSY: return "busy";
        default: return "unknown status";
    }
}

extern "C" const char* pm_last_error(void) { return pm::g_last_error.c_str(); }

extern "C" uint64_t pm_kernel_launch_count(void) { return pm::g_launches.load(); }

extern "C" int pm_profile_enable(uint32_t capacity) { return pm::profile_enable(capacity); }

extern "C" int pm_profile_read(const char** names, uint64_t* launches, double* total_ms, uint32_t capacity,
                               uint32_t* count) {
    if (!count || (capacity && (!names || !launches || !total_ms))) return fail(PM_ERR_INVALID, "NULL argument");
    return pm::profile_read(names, launches, total_ms, capacity, count);
}
