// Serving loop: products arrive one by one (host buffers) and are admitted
// onto the GPU as stream slots and device memory free up.
//
//  - Device memory: one arena allocated at creation; an admitted group of
//    requests takes one contiguous region (a, b, c and residue workspace of
//    every product in it) from a first-fit free list and returns it when the
//    group completes -- admission is by free arena bytes, and no device
//    allocation happens per request.
//  - Concurrency: each in-flight group owns a stream; groups on different
//    streams overlap on the GPU (copies of one, kernels of another).
//  - Batching: requests at the head of the queue that share a plan are
//    admitted together (up to max_group) and run as one batched launch.
//  - Tables: plans (prime basis views, CRT constants, twiddle tables on the
//    device) are cached by (n, q, coef_limbs, flags) and stay resident.
//  - Waits are bounded: pm_server_wait gives up after its timeout with
//    PM_ERR_TIMEOUT; a request that can never fit the arena is refused at
//    submission with PM_ERR_BUSY.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/polymul.h"
#include "pm_internal.h"

namespace pm {
namespace {

using Clock = std::chrono::steady_clock;

// First-fit allocator over [0, size) with 256-byte granularity.
class Arena {
   public:
    explicit Arena(size_t size) : size_(size) { free_[0] = size; }
    bool take(size_t bytes, size_t* offset) {
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *offset = it->first;
            const size_t rest = it->second - bytes, at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void give(size_t offset, size_t bytes) {
        bytes = round(bytes);
        used_ -= bytes;
        auto it = free_.emplace(offset, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t used() const { return used_; }
    size_t size() const { return size_; }

   private:
    static size_t round(size_t b) { return (b + 255) & ~size_t(255); }
    size_t size_, used_ = 0;
    std::map<size_t, size_t> free_;  // offset -> length
};

struct Request {
    uint64_t ticket;
    PlanCore* plan;
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* c;
    Clock::time_point arrived;
    int status = PM_OK;
    bool done = false;
};

struct Group {
    std::vector<std::shared_ptr<Request>> reqs;
    PlanCore* plan = nullptr;
    size_t offset = 0, bytes = 0;
    int slot = -1;
    cudaEvent_t done = nullptr;
};

size_t group_bytes(const PlanCore& p, size_t count) { return count * (3 * p.io_bytes + p.workspace_bytes); }

}  // namespace

struct Server {
    pm_server_config cfg{};
    int device = 0;
    void* arena_base = nullptr;
    std::unique_ptr<Arena> arena;
    std::vector<cudaStream_t> streams;
    std::vector<bool> slot_busy;
    std::vector<cudaEvent_t> events;  // one per slot
    std::map<std::vector<uint8_t>, std::unique_ptr<PlanCore>> plans;

    std::mutex mu;
    std::condition_variable wake, finished;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> live;
    std::vector<Group> inflight;
    uint64_t next_ticket = 1;
    bool stopping = false;
    std::thread worker;

    // statistics
    std::vector<double> latencies_us;
    uint64_t submitted = 0, completed = 0, failed = 0, groups = 0;
    uint32_t peak_inflight = 0, peak_group = 0;
    Clock::time_point first_submit{}, last_done{};

    ~Server() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stopping = true;
        }
        wake.notify_all();
        if (worker.joinable()) worker.join();
        cudaSetDevice(device);
        for (auto& g : inflight) cudaEventSynchronize(g.done);
        for (auto s : streams) cudaStreamDestroy(s);
        for (auto e : events) cudaEventDestroy(e);
        plans.clear();
        cudaFree(arena_base);
    }

    PlanCore* plan_for(uint32_t n, const uint64_t* q, uint32_t q_limbs, uint32_t limbs) {
        std::vector<uint8_t> key(16 + size_t(q_limbs) * 8);
        const uint32_t head[4] = {n, q_limbs, limbs, cfg.flags};
        std::memcpy(key.data(), head, 16);
        std::memcpy(key.data() + 16, q, size_t(q_limbs) * 8);
        auto it = plans.find(key);
        if (it != plans.end()) return it->second.get();
        auto p = std::make_unique<PlanCore>();
        p->init(n, q, q_limbs, limbs, cfg.flags);
        PlanCore* raw = p.get();
        plans.emplace(std::move(key), std::move(p));
        return raw;
    }

    // Admit from the head of the queue while a slot and arena space are free.
    // Called with mu held.
    void admit() {
        while (!pending.empty()) {
            int slot = -1;
            for (size_t i = 0; i < slot_busy.size(); ++i)
                if (!slot_busy[i]) {
                    slot = int(i);
                    break;
                }
            if (slot < 0) return;
            PlanCore* plan = pending.front()->plan;
            size_t count = 1;
            while (count < pending.size() && count < cfg.max_group && pending[count]->plan == plan) ++count;
            size_t offset = 0;
            while (count > 0 && !arena->take(group_bytes(*plan, count), &offset)) --count;
            if (count == 0) return;  // head-of-line waits for memory; FIFO order is kept
            Group g;
            g.plan = plan;
            g.offset = offset;
            g.bytes = group_bytes(*plan, count);
            g.slot = slot;
            g.done = events[slot];
            for (size_t k = 0; k < count; ++k) {
                g.reqs.push_back(pending.front());
                pending.pop_front();
            }
            slot_busy[slot] = true;
            issue(g);
            inflight.push_back(std::move(g));
            peak_inflight = std::max<uint32_t>(peak_inflight, uint32_t(inflight.size()));
            peak_group = std::max<uint32_t>(peak_group, uint32_t(count));
            ++groups;
        }
    }

    void issue(Group& g) {
        const PlanCore& p = *g.plan;
        const size_t io = p.io_bytes, count = g.reqs.size();
        uint8_t* base = static_cast<uint8_t*>(arena_base) + g.offset;
        uint8_t* da = base;
        uint8_t* db = base + count * io;
        uint8_t* dc = base + 2 * count * io;
        void* ws = base + 3 * count * io;
        cudaStream_t st = streams[g.slot];
        int status = PM_OK;
        try {
            for (size_t k = 0; k < count; ++k) {
                cuda_check(cudaMemcpyAsync(da + k * io, g.reqs[k]->a, io, cudaMemcpyHostToDevice, st), "request a");
                cuda_check(cudaMemcpyAsync(db + k * io, g.reqs[k]->b, io, cudaMemcpyHostToDevice, st), "request b");
            }
            launch_batch(p, reinterpret_cast<const uint64_t*>(da), reinterpret_cast<const uint64_t*>(db),
                         reinterpret_cast<uint64_t*>(dc), uint32_t(count), uint32_t(count), ws, st);
            for (size_t k = 0; k < count; ++k)
                cuda_check(cudaMemcpyAsync(g.reqs[k]->c, dc + k * io, io, cudaMemcpyDeviceToHost, st), "request c");
        } catch (const Failure& f) {
            status = f.status;
        }
        if (status != PM_OK)
            for (auto& r : g.reqs) r->status = status;
        cudaEventRecord(g.done, st);
    }

    // Retire finished groups.  Called with mu held.
    bool retire() {
        bool any = false;
        for (size_t i = 0; i < inflight.size();) {
            Group& g = inflight[i];
            const cudaError_t e = cudaEventQuery(g.done);
            if (e == cudaErrorNotReady) {
                ++i;
                continue;
            }
            const auto now = Clock::now();
            for (auto& r : g.reqs) {
                if (e != cudaSuccess && r->status == PM_OK) r->status = PM_ERR_CUDA;
                r->done = true;
                if (r->status == PM_OK) {
                    ++completed;
                    latencies_us.push_back(std::chrono::duration<double, std::micro>(now - r->arrived).count());
                } else {
                    ++failed;
                }
            }
            last_done = now;
            arena->give(g.offset, g.bytes);
            slot_busy[g.slot] = false;
            inflight.erase(inflight.begin() + i);
            any = true;
        }
        return any;
    }

    void run() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(mu);
        while (true) {
            if (stopping && pending.empty() && inflight.empty()) return;
            const bool freed = retire();
            admit();
            if (freed) finished.notify_all();
            if (inflight.empty() && pending.empty()) {
                wake.wait_for(lock, std::chrono::milliseconds(50));
            } else {
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                lock.lock();
            }
        }
    }
};

}  // namespace pm

struct pm_server {
    pm::Server s;
};

using pm::fail;
using pm::Failure;

#define PM_SGUARD(...)                                           \
    try {                                                        \
        __VA_ARGS__;                                             \
        return PM_OK;                                            \
    } catch (const Failure& f) {                                 \
        return fail(f.status, f.what());                         \
    } catch (const std::bad_alloc&) {                            \
        return fail(PM_ERR_NO_MEMORY, "host allocation failed"); \
    } catch (const std::exception& e) {                          \
        return fail(PM_ERR_INVALID, e.what());                   \
    }

extern "C" int pm_server_create(pm_server** out, const pm_server_config* cfg) {
    if (!out || !cfg) return fail(PM_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (cfg->slots == 0 || cfg->slots > 64) return fail(PM_ERR_INVALID, "slots must be in [1, 64]");
    if (cfg->flags & ~uint32_t(PM_CONVERT_TENSOR | PM_CONVERT_SIMT)) return fail(PM_ERR_INVALID, "unknown flags");
    PM_SGUARD({
        auto srv = std::make_unique<pm_server>();
        pm::Server& s = srv->s;
        s.cfg = *cfg;
        if (!s.cfg.max_group) s.cfg.max_group = 8;
        pm::cuda_check(cudaGetDevice(&s.device), "cudaGetDevice");
        size_t budget = cfg->device_budget_bytes;
        if (!budget) {
            size_t free_b = 0, total_b = 0;
            pm::cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            budget = free_b / 4;
        }
        pm::cuda_check(cudaMalloc(&s.arena_base, budget), "allocate serving arena");
        s.arena = std::make_unique<pm::Arena>(budget);
        s.streams.resize(cfg->slots);
        s.events.resize(cfg->slots);
        s.slot_busy.assign(cfg->slots, false);
        for (uint32_t i = 0; i < cfg->slots; ++i) {
            pm::cuda_check(cudaStreamCreateWithFlags(&s.streams[i], cudaStreamNonBlocking), "serving stream");
            pm::cuda_check(cudaEventCreateWithFlags(&s.events[i], cudaEventDisableTiming), "serving event");
        }
        s.worker = std::thread([&s] { s.run(); });
        *out = srv.release();
    })
}

extern "C" int pm_server_submit(pm_server* srv, uint32_t n, const uint64_t* q, uint32_t q_limbs,
                                uint32_t coef_limbs, const uint64_t* a, const uint64_t* b, uint64_t* c,
                                uint64_t* ticket) {
    if (!srv || !q || !a || !b || !c || !ticket) return fail(PM_ERR_INVALID, "NULL argument");
    pm::Server& s = srv->s;
    PM_SGUARD({
        std::lock_guard<std::mutex> lock(s.mu);
        pm::cuda_check(cudaSetDevice(s.device), "cudaSetDevice");
        pm::PlanCore* plan = s.plan_for(n, q, q_limbs, coef_limbs);
        if (pm::group_bytes(*plan, 1) > s.arena->size())
            throw Failure(PM_ERR_BUSY, "request needs more device memory than the serving arena holds");
        auto r = std::make_shared<pm::Request>();
        r->ticket = s.next_ticket++;
        r->plan = plan;
        r->a = a;
        r->b = b;
        r->c = c;
        r->arrived = pm::Clock::now();
        if (s.submitted++ == 0) s.first_submit = r->arrived;
        s.pending.push_back(r);
        s.live[r->ticket] = r;
        *ticket = r->ticket;
        s.wake.notify_all();
    })
}

extern "C" int pm_server_wait(pm_server* srv, uint64_t ticket, uint32_t timeout_ms) {
    if (!srv) return fail(PM_ERR_INVALID, "NULL server");
    pm::Server& s = srv->s;
    std::unique_lock<std::mutex> lock(s.mu);
    auto it = s.live.find(ticket);
    if (it == s.live.end()) return fail(PM_ERR_INVALID, "unknown or already collected ticket");
    auto r = it->second;
    if (!s.finished.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return r->done; }))
        return fail(PM_ERR_TIMEOUT, "request not finished within the timeout");
    s.live.erase(ticket);
    if (r->status != PM_OK) return fail(r->status, "request failed on the device");
    return PM_OK;
}

extern "C" int pm_server_drain(pm_server* srv, uint32_t timeout_ms) {
    if (!srv) return fail(PM_ERR_INVALID, "NULL server");
    pm::Server& s = srv->s;
    std::unique_lock<std::mutex> lock(s.mu);
    if (!s.finished.wait_for(lock, std::chrono::milliseconds(timeout_ms),
                             [&] { return s.pending.empty() && s.inflight.empty(); }))
        return fail(PM_ERR_TIMEOUT, "server not drained within the timeout");
    return PM_OK;
}

extern "C" int pm_server_get_stats(pm_server* srv, pm_server_stats* st) {
    if (!srv || !st) return fail(PM_ERR_INVALID, "NULL argument");
    pm::Server& s = srv->s;
    std::lock_guard<std::mutex> lock(s.mu);
    std::memset(st, 0, sizeof *st);
    st->submitted = s.submitted;
    st->completed = s.completed;
    st->failed = s.failed;
    st->groups = s.groups;
    st->peak_inflight = s.peak_inflight;
    st->peak_group = s.peak_group;
    st->arena_bytes = s.arena->size();
    st->arena_used = s.arena->used();
    std::vector<double> l = s.latencies_us;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) { return l[std::min(l.size() - 1, size_t(q * double(l.size() - 1) + 0.5))]; };
        st->p50_us = pct(0.50);
        st->p99_us = pct(0.99);
        st->max_us = l.back();
        double sum = 0;
        for (double x : l) sum += x;
        st->mean_us = sum / double(l.size());
        const double span = std::chrono::duration<double>(s.last_done - s.first_submit).count();
        st->products_per_s = span > 0 ? double(s.completed) / span : 0.0;
    }
    return PM_OK;
}

extern "C" int pm_server_reset_stats(pm_server* srv) {
    if (!srv) return fail(PM_ERR_INVALID, "NULL server");
    pm::Server& s = srv->s;
    std::lock_guard<std::mutex> lock(s.mu);
    s.latencies_us.clear();
    s.submitted = s.completed = s.failed = s.groups = 0;
    s.peak_inflight = s.peak_group = 0;
    return PM_OK;
}

extern "C" int pm_server_destroy(pm_server* srv) {
    delete srv;
    return PM_OK;
}
