// fherma_init / fherma_run / fherma_free on top of the C ABI (include/polymul.h).
// Status codes become std::runtime_error, as the reference's check() does
// (rns/solve.cu:421-423).
#include <condition_variable>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

#include "../../include/fherma_polymul.h"
#include "../../include/polymul.h"

namespace {

// The output tensor of the next fherma_run, allocated and zero-filled by a helper
// thread while the GPU works on the current product: filling 3.7 MB of fresh
// std::vector storage takes a core over a hundred microseconds, which the call
// then does not spend.  take() hands over the prepared vector (or, if the helper
// has not finished, allocates one itself) and asks for the next.
class SpareOutput {
public:
    explicit SpareOutput(size_t words) : words_(words), worker_([this] { loop(); }) {}
    ~SpareOutput() {
        {
            std::lock_guard<std::mutex> lock(m_);
            stop_ = true;
        }
        cv_.notify_all();
        worker_.join();
    }
    std::vector<uint32_t> take() {
        std::vector<uint32_t> v;
        {
            std::lock_guard<std::mutex> lock(m_);
            if (ready_) {
                v.swap(spare_);
                ready_ = false;
            }
            want_ = true;
        }
        cv_.notify_all();
        if (v.size() != words_) v.assign(words_, 0u);
        return v;
    }

private:
    void loop() {
        std::unique_lock<std::mutex> lock(m_);
        while (true) {
            cv_.wait(lock, [&] { return stop_ || (want_ && !ready_); });
            if (stop_) return;
            want_ = false;
            lock.unlock();
            std::vector<uint32_t> v;
            try {
                v.assign(words_, 0u);
            } catch (...) {  // out of memory here: take() allocates on the caller's thread instead
                v.clear();
            }
            lock.lock();
            if (v.size() == words_) {
                spare_.swap(v);
                ready_ = true;
            }
        }
    }
    const size_t words_;
    std::mutex m_;
    std::condition_variable cv_;
    std::vector<uint32_t> spare_;
    bool ready_ = false, want_ = true, stop_ = false;
    std::thread worker_;  // last: starts once the members above exist
};

struct State {
    pm_plan* plan = nullptr;
    uint32_t n = 0, words = 0;
    std::unique_ptr<SpareOutput> spare;
    ~State() {
        spare.reset();
        pm_plan_destroy(plan);
    }
};

[[noreturn]] void raise(int status, const char* what) {
    throw std::runtime_error(std::string(what) + ": " + pm_status_string(status) + " (" + pm_last_error() + ")");
}

unsigned bit_length(const std::vector<uint32_t>& w) {
    for (size_t i = w.size(); i--;)
        if (w[i]) return unsigned(i * 32 + 32 - __builtin_clz(w[i]));
    return 0;
}

}  // namespace

void* fherma_init(const fherma::Point& p) {
    if (p.L == 0 || p.q.data.size() != p.L) throw std::runtime_error("fherma_init: q must hold L words");
    if (p.L % 2) throw std::runtime_error("fherma_init: L must be even (coefficients are read as 64-bit limbs)");
    if (p.N < 2 || (p.N & (p.N - 1)) || p.N > 65536)
        throw std::runtime_error("fherma_init: N must be a power of two in [2, 65536]");
    const unsigned bits = bit_length(p.q.data);
    if (p.W && bits > p.W) throw std::runtime_error("fherma_init: q is wider than W bits");
    std::vector<uint64_t> q64(p.L / 2);
    for (uint32_t i = 0; i < p.L / 2; ++i) q64[i] = uint64_t(p.q.data[2 * i]) | (uint64_t(p.q.data[2 * i + 1]) << 32);
    auto s = std::make_unique<State>();
    s->n = p.N;
    s->words = p.L;
    const uint32_t limbs = p.L / 2;
    // the tensor-core conversion reads 16-byte coefficient rows (even limb counts)
    const uint32_t flags = (limbs % 2 == 0) ? PM_CONVERT_TENSOR : PM_CONVERT_SIMT;
    const int st = pm_plan_create(&s->plan, p.N, q64.data(), limbs, limbs, flags);
    if (st != PM_OK) raise(st, "fherma_init");
    s->spare = std::make_unique<SpareOutput>(size_t(p.N) * p.L);
    return s.release();
}

fherma::Outputs fherma_run(void* state, const fherma::Inputs& in) {
    if (!state) throw std::runtime_error("fherma_run: no state");
    auto& s = *static_cast<State*>(state);
    const size_t words = size_t(s.n) * s.words;
    if (in.a.data.size() != words || in.b.data.size() != words)
        throw std::runtime_error("fherma_run: inputs must be N x L words");
    // inputs staged and everything queued; the output tensor is taken while the GPU runs
    int st = pm_multiply_host_begin(s.plan, reinterpret_cast<const uint64_t*>(in.a.data.data()),
                                    reinterpret_cast<const uint64_t*>(in.b.data.data()));
    if (st != PM_OK) raise(st, "fherma_run");
    fherma::Outputs out;
    try {
        out.c.shape = {int64_t(s.n), int64_t(s.words)};
        out.c.data = s.spare->take();
    } catch (...) {
        std::vector<uint32_t> sink(words);  // the open product still needs somewhere to land
        pm_multiply_host_end(s.plan, reinterpret_cast<uint64_t*>(sink.data()));
        throw;
    }
    st = pm_multiply_host_end(s.plan, reinterpret_cast<uint64_t*>(out.c.data.data()));
    if (st != PM_OK) raise(st, "fherma_run");
    return out;
}

void fherma_free(void* state) { delete static_cast<State*>(state); }
