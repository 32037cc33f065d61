// The single-product host-buffer call (pm_multiply_host, the fherma_run of the
// drop-in), pipelined.
//
// The caller's a, b, c are usually pageable (the harness's std::vector
// tensors), which the GPU cannot read: every byte goes through pinned staging.
// Done serially that is two host copies of 3.7 MB, an H2D of 7.3 MB, the
// kernels, a D2H of 3.7 MB and a host copy of 3.7 MB, one after the other.
// Here:
//   - the inputs are cut into pieces; a small pool of host threads copies
//     piece k into pinned staging (non-temporal stores) and queues its H2D at
//     once, so staging, the PCIe transfer and the other threads' copies
//     overlap (the reference gets the same overlap from its copy pool and
//     4-chunk input pipeline, host_copy_pool.h, input_pipeline.h:12-54,
//     rns/solve.cu:731-761);
//   - a's conversion starts on a side stream as soon as a's copies are queued,
//     so it runs while b is still on the link; b's conversion, the row and the
//     CRT kernels follow on the plan's stream; the product comes back in
//     pieces, each with an event, and the pool copies piece k out as soon as
//     its event fires, while later pieces are still on the link;
//   - the call is split (begin / end) so that a caller can do its own work --
//     the drop-in allocates the output tensor -- while the GPU runs.
// Pinned caller buffers skip the staging: their pieces are copied directly.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <immintrin.h>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/polymul.h"
#include "pm_internal.h"

namespace pm {

namespace {

// dst 32-byte aligned, bytes a multiple of 32: 256-bit loads, streaming stores
__attribute__((target("avx2"))) void stream_copy_avx2(void* dst, const void* src, size_t bytes) {
    auto* d = static_cast<__m256i*>(dst);
    auto* s = static_cast<const __m256i*>(src);
    const size_t n = bytes / 32;
    size_t k = 0;
    for (; k + 4 <= n; k += 4) {
        const __m256i x0 = _mm256_loadu_si256(s + k), x1 = _mm256_loadu_si256(s + k + 1);
        const __m256i x2 = _mm256_loadu_si256(s + k + 2), x3 = _mm256_loadu_si256(s + k + 3);
        _mm256_stream_si256(d + k, x0);
        _mm256_stream_si256(d + k + 1, x1);
        _mm256_stream_si256(d + k + 2, x2);
        _mm256_stream_si256(d + k + 3, x3);
    }
    for (; k < n; ++k) _mm256_stream_si256(d + k, _mm256_loadu_si256(s + k));
    _mm_sfence();
}

bool have_avx2() {
    static const bool yes = __builtin_cpu_supports("avx2");
    return yes;
}

// Copy that does not pull the destination into the cache when it can.
void host_copy(void* dst, const void* src, size_t bytes) {
    const uintptr_t d = reinterpret_cast<uintptr_t>(dst);
    if (have_avx2() && bytes >= 4096) {
        const size_t head = (32 - (d & 31)) & 31;
        if (head) std::memcpy(dst, src, head);
        const size_t body = (bytes - head) & ~size_t(31);
        stream_copy_avx2(static_cast<uint8_t*>(dst) + head, static_cast<const uint8_t*>(src) + head, body);
        const size_t tail = bytes - head - body;
        if (tail) std::memcpy(static_cast<uint8_t*>(dst) + head + body, static_cast<const uint8_t*>(src) + head + body, tail);
        return;
    }
    std::memcpy(dst, src, bytes);
}

bool is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

}  // namespace

// How long an idle copy thread spins before it sleeps: PM_HOST_SPIN_US (microseconds,
// read once), 20000 by default.  A caller that leaves longer gaps between products finds
// the threads asleep and waits for them to wake: a harness that writes one case's 3.7 MB
// result and reads the next case's 7.3 MB between calls spends a few milliseconds there,
// and with a 2 ms spin its calls took 15 us longer at N = 32768.  The spin costs the
// pool's threads that long of CPU time after each call; 0 makes them sleep at once.
static long spin_us() {
    static const long us = [] {
        const char* e = std::getenv("PM_HOST_SPIN_US");
        if (!e || !*e) return 20000L;
        char* end = nullptr;
        const long v = std::strtol(e, &end, 10);
        return (end && *end == 0 && v >= 0 && v <= 10000000L) ? v : 20000L;
    }();
    return us;
}

// Persistent host threads that run the pieces of one job; the calling thread
// takes pieces too.  Idle workers spin for a short while (back-to-back calls
// find them awake), then sleep on a condition variable.
class CopyPool {
public:
    explicit CopyPool(int threads) {
        for (int t = 0; t < threads; ++t) workers_.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lock(m_);
            stop_ = true;
            ++generation_;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    int threads() const { return int(workers_.size()); }

    // Runs f(k) for k in [0, pieces) on the workers and the caller; returns when
    // all are done and no worker is still inside the job.  The first exception a
    // piece throws is rethrown here.
    void run(int pieces, const std::function<void(int)>& f) {
        {
            std::lock_guard<std::mutex> lock(m_);
            job_ = &f;
            pieces_ = pieces;
            next_.store(0);
            done_.store(0);
            error_ = nullptr;
            generation_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        work(&f, pieces);
        while (done_.load(std::memory_order_acquire) < pieces) _mm_pause();
        // no worker joins from here on (they join under the lock while job_ is set); the ones
        // that joined find no piece left and leave before the next job resets the counters
        {
            std::lock_guard<std::mutex> lock(m_);
            job_ = nullptr;
        }
        while (active_.load(std::memory_order_acquire) > 0) _mm_pause();
        if (error_) std::rethrow_exception(error_);
    }

    // The same job without the caller: returns at once; finish() waits for it.
    void start(int pieces, const std::function<void(int)>& f) {
        {
            std::lock_guard<std::mutex> lock(m_);
            job_ = &f;
            pieces_ = pieces;
            next_.store(0);
            done_.store(0);
            error_ = nullptr;
            generation_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        started_ = pieces;
        job_started_ = &f;
    }
    // The caller takes one piece of the started job, if one is left; false when none is.
    bool help() {
        const int pieces = started_;
        const int k = next_.fetch_add(1);
        if (k >= pieces) return false;
        try {
            (*job_started_)(k);
        } catch (...) {
            std::lock_guard<std::mutex> lock(m_);
            if (!error_) error_ = std::current_exception();
        }
        done_.fetch_add(1, std::memory_order_release);
        return true;
    }
    void finish() {
        const int pieces = started_;
        started_ = 0;
        while (done_.load(std::memory_order_acquire) < pieces) _mm_pause();
        {
            std::lock_guard<std::mutex> lock(m_);
            job_ = nullptr;
        }
        while (active_.load(std::memory_order_acquire) > 0) _mm_pause();
        if (error_) std::rethrow_exception(error_);
    }

private:
    void work(const std::function<void(int)>* f, int pieces) {
        for (int k = next_.fetch_add(1); k < pieces; k = next_.fetch_add(1)) {
            try {
                (*f)(k);
            } catch (...) {
                std::lock_guard<std::mutex> lock(m_);
                if (!error_) error_ = std::current_exception();
            }
            done_.fetch_add(1, std::memory_order_release);
        }
    }
    void loop() {
        uint64_t seen = 0;
        while (true) {
            // spinning a while keeps the threads awake from one half of a product to the next
            // (the GPU's part lasts a few hundred microseconds) and between back-to-back calls
            const auto spin_until = std::chrono::steady_clock::now() + std::chrono::microseconds(spin_us());
            while (generation_.load(std::memory_order_acquire) == seen && std::chrono::steady_clock::now() < spin_until)
                _mm_pause();
            std::unique_lock<std::mutex> lock(m_);
            cv_.wait(lock, [&] { return generation_.load() != seen; });
            seen = generation_.load();
            if (stop_) return;
            if (!job_) continue;  // that job is over already
            const std::function<void(int)>* f = job_;
            const int pieces = pieces_;
            active_.fetch_add(1, std::memory_order_acq_rel);
            lock.unlock();
            work(f, pieces);
            active_.fetch_sub(1, std::memory_order_acq_rel);
        }
    }

    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_;
    std::atomic<uint64_t> generation_{0};
    const std::function<void(int)>* job_ = nullptr;
    int pieces_ = 0;
    std::atomic<int> next_{0}, done_{0}, active_{0};
    std::exception_ptr error_;
    bool stop_ = false;
    int started_ = 0;
    const std::function<void(int)>* job_started_ = nullptr;
};

namespace {
// Every copy the link makes costs about 3.7 us of its time on top of the bytes (B200,
// PCIe 5: 7.3 MB in 16 copies took 196 us against 139 us in one), so the host threads
// work in small units while the link gets few copies.  A staged input goes in copy
// groups of kGroupUnits units (one round of the threads); the first polynomial's groups
// grow geometrically (1/16, 1/8, 1/4, then the remaining 9/16) so that the link starts
// after a small first round instead of a quarter of the bytes -- the threads stage about
// twice as fast as the link moves -- and the second polynomial, staged while the first is
// on the link, goes in two halves.
constexpr int kGroupUnits = 9;  // staging units per H2D copy
constexpr int kMaxGroups = 6;   // H2D copies of the staged inputs (4 + 2)
constexpr int kOutPieces = 4;   // D2H copies of the product: 1/2, 1/4, 1/8, 1/8 of it, the last
                                // one's copy-out (after everything else) short
static_assert(kMaxGroups * kGroupUnits <= 64 && kOutPieces <= 64, "one ready flag per unit");

// D2H piece k of the product: offset and length
void out_piece(size_t io, int k, size_t* off, size_t* len) {
    const auto cut = [](size_t x) { return x & ~size_t(63); };
    const size_t b1 = cut(io / 2), b2 = b1 + cut(io / 4), b3 = b2 + cut(io / 8);
    const size_t bound[kOutPieces + 1] = {0, b1, b2, b3, io};
    *off = bound[k];
    *len = bound[k + 1] - bound[k];
}

// the H2D copies of the staged inputs: polynomial, byte offset and length of each
struct InGroups {
    int count = 0;
    int poly[kMaxGroups];
    size_t off[kMaxGroups], len[kMaxGroups];
    void add(int p, size_t o, size_t l) {
        poly[count] = p;
        off[count] = o;
        len[count] = l;
        ++count;
    }
};

InGroups input_groups(size_t io, bool pinned_a, bool pinned_b) {
    InGroups g;
    const auto cut = [](size_t x) { return x & ~size_t(63); };
    bool first = true;
    for (int poly = 0; poly < 2; ++poly) {
        if (poly == 0 ? pinned_a : pinned_b) continue;
        if (first) {
            size_t o = 0;
            for (int d = 16; d >= 4; d /= 2) {
                const size_t l = std::min(io - o, cut(io / size_t(d)));
                if (l) g.add(poly, o, l);
                o += l;
            }
            if (io > o) g.add(poly, o, io - o);
            first = false;
        } else {
            const size_t h = std::min(io, cut(io / 2 + 63));
            g.add(poly, 0, h);
            if (io > h) g.add(poly, h, io - h);
        }
    }
    return g;
}

int pool_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    int t = hw ? int(hw / 2) : 4;
    if (t > 8) t = 8;
    if (t < 1) t = 1;
    return t;
}

// piece k of `bytes` cut into `pieces` runs of 64-byte multiples
void piece(size_t bytes, int pieces, int k, size_t* off, size_t* len) {
    const size_t unit = ((bytes + pieces - 1) / pieces + 63) & ~size_t(63);
    *off = std::min(bytes, unit * size_t(k));
    *len = std::min(bytes, *off + unit) - *off;
}
}  // namespace

HostCall::~HostCall() {
    if (stream) cudaStreamSynchronize(stream);
    if (side) {
        cudaStreamSynchronize(side);
        cudaStreamDestroy(side);
    }
    if (a_in) cudaEventDestroy(a_in);
    if (a_converted) cudaEventDestroy(a_converted);
    for (auto& e : out_ready)
        if (e) cudaEventDestroy(e);
    cudaFree(d_io);
    cudaFreeHost(h_stage);
}

void multiply_host_begin(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* direct_out) {
    if (!s.host) s.host = std::make_unique<HostCall>();
    HostCall& h = *s.host;
    if (h.pending) throw Failure(PM_ERR_BUSY, "a host-buffer product of this plan is still open: end it first");
    if (!h.d_io) {
        h.stream = s.stream;
        cuda_check(cudaMalloc(&h.d_io, 3 * s.io_bytes), "allocate plan I/O buffers");
        // staging for a, b, c, then one word the device error flag is copied into
        cuda_check(cudaMallocHost(&h.h_stage, 3 * s.io_bytes + 64), "allocate pinned staging");
        h.out_ready.assign(kOutPieces, nullptr);
        for (auto& e : h.out_ready) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "output events");
        cuda_check(cudaStreamCreateWithFlags(&h.side, cudaStreamNonBlocking), "conversion stream");
        cuda_check(cudaEventCreateWithFlags(&h.a_in, cudaEventDisableTiming), "input event");
        cuda_check(cudaEventCreateWithFlags(&h.a_converted, cudaEventDisableTiming), "conversion event");
    }
    if (!h.pool) h.pool = std::make_unique<CopyPool>(pool_threads());
    const size_t io = s.io_bytes;
    uint8_t* dev = static_cast<uint8_t*>(h.d_io);
    uint8_t* stage = static_cast<uint8_t*>(h.h_stage);
    const uint8_t* src[2] = {reinterpret_cast<const uint8_t*>(a), reinterpret_cast<const uint8_t*>(b)};
    const bool pinned[2] = {is_pinned(a), is_pinned(b)};
    // Where the plan converts one polynomial at a time, a's conversion runs on the side
    // stream as soon as a's copies are queued, while b is still on the link.
    const bool split = conversion_splits(s);
    uint32_t* work = s.d_work;
    bool a_aside = false;
    auto convert_a_aside = [&]() {
        cuda_check(cudaEventRecord(h.a_in, h.stream), "input event");
        cuda_check(cudaStreamWaitEvent(h.side, h.a_in, 0), "conversion stream wait");
        launch_tensor_convert_poly(s, reinterpret_cast<const uint32_t*>(dev), 0, work, h.side);
        cuda_check(cudaEventRecord(h.a_converted, h.side), "conversion event");
        a_aside = true;
    };
    // pinned inputs go straight to the link in one copy each
    for (int poly = 0; poly < 2; ++poly)
        if (pinned[poly]) {
            cuda_check(cudaMemcpyAsync(dev + poly * io, src[poly], io, cudaMemcpyHostToDevice, h.stream), "copy in");
            if (split && poly == 0) convert_a_aside();
        }
    // pageable inputs: the pool's threads stage the units (in index order, as they take
    // them) while this thread queues each copy group as soon as its units are staged -- one
    // thread talks to the runtime, so the copies enter the stream without contending
    const InGroups g = input_groups(io, pinned[0], pinned[1]);
    if (g.count) {
        const int nu = g.count * kGroupUnits;
        for (int k = 0; k < nu; ++k) h.ready[k].store(0, std::memory_order_relaxed);
        const std::function<void(int)> stage_unit = [&](int k) {
            const int grp = k / kGroupUnits, poly = g.poly[grp];
            size_t off, len;
            piece(g.len[grp], kGroupUnits, k % kGroupUnits, &off, &len);
            off += g.off[grp];
            if (len) host_copy(stage + poly * io + off, src[poly] + off, len);
            h.ready[k].store(1, std::memory_order_release);
        };
        h.pool->start(nu, stage_unit);
        try {
            for (int grp = 0; grp < g.count; ++grp) {
                // stage units too while this copy's are not all ready (the workers may be waking)
                for (int k = grp * kGroupUnits; k < (grp + 1) * kGroupUnits; ++k)
                    while (!h.ready[k].load(std::memory_order_acquire))
                        if (!h.pool->help()) _mm_pause();
                const size_t off = g.off[grp];
                uint8_t* dst = dev + g.poly[grp] * io + off;
                cuda_check(cudaMemcpyAsync(dst, stage + g.poly[grp] * io + off, g.len[grp], cudaMemcpyHostToDevice,
                                           h.stream),
                           "copy in");
                if (split && !a_aside && g.poly[grp] == 0 && (grp + 1 == g.count || g.poly[grp + 1] != 0))
                    convert_a_aside();
            }
        } catch (...) {
            try {
                h.pool->finish();
            } catch (...) {
            }
            throw;
        }
        h.pool->finish();
    }
    if (a_aside) {
        launch_tensor_convert_poly(s, reinterpret_cast<const uint32_t*>(dev + io), 1, work, h.stream);
        cuda_check(cudaStreamWaitEvent(h.stream, h.a_converted, 0), "conversion wait");
        launch_tensor_after_conversion(s, reinterpret_cast<uint32_t*>(dev + 2 * io), work, 1, h.stream);
    } else {
        launch_product(s, reinterpret_cast<const uint64_t*>(dev), reinterpret_cast<const uint64_t*>(dev + io),
                       reinterpret_cast<uint64_t*>(dev + 2 * io), nullptr, h.stream);
    }
    // a pinned output takes the product directly; otherwise it lands in the staging
    h.direct_out = direct_out && is_pinned(direct_out) ? reinterpret_cast<uint8_t*>(direct_out) : nullptr;
    uint8_t* land = h.direct_out ? h.direct_out : stage + 2 * io;
    if (h.direct_out) {  // nothing to copy out afterwards: one transfer
        cuda_check(cudaMemcpyAsync(land, dev + 2 * io, io, cudaMemcpyDeviceToHost, h.stream), "copy out");
    } else {
        for (int k = 0; k < kOutPieces; ++k) {
            size_t off, len;
            out_piece(io, k, &off, &len);
            if (len)
                cuda_check(cudaMemcpyAsync(land + off, dev + 2 * io + off, len, cudaMemcpyDeviceToHost, h.stream),
                           "copy out");
            cuda_check(cudaEventRecord(h.out_ready[k], h.stream), "output event");
        }
    }
    // the error word rides on the same stream: no second round trip after the product
    cuda_check(cudaMemcpyAsync(stage + 3 * io, s.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, h.stream),
               "read error word");
    h.pending = true;
}

void multiply_host_end(PlanCore& s, uint64_t* c) {
    if (!s.host || !s.host->pending) throw Failure(PM_ERR_INVALID, "no host-buffer product of this plan is open");
    HostCall& h = *s.host;
    h.pending = false;
    const size_t io = s.io_bytes;
    uint8_t* stage = static_cast<uint8_t*>(h.h_stage);
    uint8_t* dst = reinterpret_cast<uint8_t*>(c);
    if (h.direct_out && h.direct_out != dst)
        throw Failure(PM_ERR_INVALID, "the product was directed to another output buffer at the start of the call");
    // each product piece leaves the staging as soon as it has landed: this thread polls the
    // pieces' events in order (a blocking wait can sleep for longer than a piece takes) and
    // flags them; the pool's threads copy the units of flagged pieces out
    if (!h.direct_out) {
        for (int k = 0; k < kOutPieces; ++k) h.ready[k].store(0, std::memory_order_relaxed);
        const std::function<void(int)> copy_unit = [&](int k) {  // unit k % 9 of piece k / 9
            const int pc = k / kGroupUnits;
            size_t poff, plen, off, len;
            out_piece(io, pc, &poff, &plen);
            piece(plen, kGroupUnits, k % kGroupUnits, &off, &len);
            if (!len) return;
            while (!h.ready[pc].load(std::memory_order_acquire)) _mm_pause();
            host_copy(dst + poff + off, stage + 2 * io + poff + off, len);
        };
        h.pool->start(kOutPieces * kGroupUnits, copy_unit);
        try {
            const auto give_up = std::chrono::steady_clock::now() + std::chrono::seconds(60);
            for (int k = 0; k < kOutPieces; ++k) {
                cudaError_t e;
                while ((e = cudaEventQuery(h.out_ready[k])) == cudaErrorNotReady) {
                    if (std::chrono::steady_clock::now() > give_up)
                        throw Failure(PM_ERR_TIMEOUT, "the product did not come back within 60 s");
                    _mm_pause();
                }
                cuda_check(e, "product");
                h.ready[k].store(1, std::memory_order_release);
            }
        } catch (...) {
            for (int k = 0; k < kOutPieces; ++k) h.ready[k].store(1, std::memory_order_release);  // release the copiers
            try {
                h.pool->finish();
            } catch (...) {
            }
            throw;
        }
        while (h.pool->help()) {
        }
        h.pool->finish();
    }
    cuda_check(cudaStreamSynchronize(h.stream), "product");
    uint32_t herr = 0;
    std::memcpy(&herr, stage + 3 * io, sizeof herr);
    if (herr) check_device_errors(s);
}

void multiply_host(PlanCore& s, const uint64_t* a, const uint64_t* b, uint64_t* c) {
    multiply_host_begin(s, a, b, c);
    multiply_host_end(s, c);
}

}  // namespace pm
