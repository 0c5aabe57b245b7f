// Host side of the frames' transfer encoding (include/xpgi.h, "Transfer encoding"): uint32 pixels to one byte each
// plus (index, value) exceptions, on a pool of host threads. The work is a streaming read of the frames, so the pool
// splits a run into slices of kSlice pixels handed out in order; each slice records which of its kBlock-pixel
// blocks hold an exception, and the calling thread lists those blocks' exceptions afterwards, in pixel order.
#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "xpgi.h"
#include "xpgi_internal.h"

namespace {

constexpr int64_t kBlock = 4096;                 // pixels per exception flag
constexpr int64_t kSlice = 256 * kBlock;         // pixels per work item (4 MB of frames)

// one block: the byte codes, and whether any pixel needs an exception (written so that the compiler vectorises it)
__attribute__((target_clones("avx2", "default")))
uint32_t pack_block(const uint32_t* __restrict__ s, uint8_t* __restrict__ d, int64_t m) {
    uint32_t esc = 0;
    for (int64_t i = 0; i < m; ++i) {
        const uint32_t v = s[i];
        const uint32_t flagged = v == 0xFFFFFFFFu;
        const uint32_t big = v >= XI_PACK_ESCAPE;
        d[i] = (uint8_t)(big ? (flagged ? XI_PACK_FLAGGED : XI_PACK_ESCAPE) : v);
        esc |= big & (flagged ^ 1u);
    }
    return esc;
}

// a block's codes go through a cache-resident buffer to the plane with streaming stores: the plane is read next by
// the copy engine, not by this core, so its cache lines are not fetched first (32-byte aligned, whole blocks only)
__attribute__((target("avx2"))) void stream_copy(uint8_t* __restrict__ d, const uint8_t* __restrict__ s, int64_t m) {
    for (int64_t i = 0; i < m; i += 32)
        _mm256_stream_si256(reinterpret_cast<__m256i*>(d + i),
                            _mm256_load_si256(reinterpret_cast<const __m256i*>(s + i)));
}

bool have_avx2() {
    static const bool ok = __builtin_cpu_supports("avx2");
    return ok;
}

class Pool {
public:
    // runs f(item) for item in [0, n_items) on up to `threads` threads (the caller among them)
    template <class F>
    void run(int64_t n_items, int threads, F&& f) {
        std::lock_guard<std::mutex> call(call_mu_);
        const int want = std::max(1, std::min<int>(threads, (int)std::min<int64_t>(n_items, 256)));
        grow(want - 1);
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = [&f](int64_t i) { f(i); };
            next_.store(0);
            n_items_ = n_items;
            helpers_ = want - 1;
            busy_ = want - 1;
            ++gen_;
        }
        cv_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return busy_ == 0; });
        job_ = nullptr;
    }

    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }

private:
    void drain() {
        for (;;) {
            const int64_t i = next_.fetch_add(1);
            if (i >= n_items_) return;
            job_(i);
        }
    }

    void grow(int n) {
        while ((int)th_.size() < n) {
            const int id = (int)th_.size();
            th_.emplace_back([this, id] { loop(id); });
        }
    }

    void loop(int id) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || (gen_ != seen && id < helpers_); });
                if (stop_) return;
                seen = gen_;
            }
            drain();
            std::lock_guard<std::mutex> lk(mu_);
            if (--busy_ == 0) done_cv_.notify_all();
        }
    }

    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    std::vector<std::thread> th_;
    std::function<void(int64_t)> job_;
    std::atomic<int64_t> next_{0};
    int64_t n_items_ = 0;
    int helpers_ = 0, busy_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

Pool& pool() {
    static Pool* p = new Pool();          // never destroyed: its threads may outlive static destruction order
    return *p;
}

int default_threads() {
    // the packing is bound by the host's memory bandwidth well before every core is busy: leave cores to the
    // threads that launch the kernels and issue the raw copies
    const unsigned hc = std::thread::hardware_concurrency();
    return hc > 5 ? (int)hc - 4 : 1;
}

}  // namespace

extern "C" int xi_pack_u8(const uint32_t* src, int64_t n, uint8_t* plane, uint32_t* exc, int64_t exc_cap,
                          int threads, int64_t* n_exc) {
    if (!n_exc || n < 0 || exc_cap < 0 || (n && (!src || !plane)) || (exc_cap && !exc))
        return xi_fail(XI_E_ARG, "xi_pack_u8: null pointer or negative size");
    if (n > XI_PACK_MAX_PIXELS) return xi_fail(XI_E_LIMIT, "xi_pack_u8: more than XI_PACK_MAX_PIXELS pixels");
    *n_exc = 0;
    if (n == 0) return XI_OK;
    if (threads <= 0) threads = default_threads();
    const int64_t n_blocks = (n + kBlock - 1) / kBlock;
    std::vector<uint8_t> flag((size_t)n_blocks, 0);
    const int64_t n_items = (n + kSlice - 1) / kSlice;
    pool().run(n_items, threads, [&](int64_t it) {
        const int64_t a = it * kSlice, b = std::min(n, a + kSlice);
        alignas(64) uint8_t buf[kBlock];
        const bool stream = have_avx2() && ((uintptr_t)plane & 31) == 0;
        for (int64_t p = a; p < b; p += kBlock) {
            const int64_t m = std::min(kBlock, b - p);
            if (stream && m == kBlock) {
                flag[(size_t)(p / kBlock)] = (uint8_t)pack_block(src + p, buf, m);
                stream_copy(plane + p, buf, m);
            } else {
                flag[(size_t)(p / kBlock)] = (uint8_t)pack_block(src + p, plane + p, m);
            }
        }
        _mm_sfence();                     // the streaming stores are visible before the call returns
    });
    int64_t k = 0;
    for (int64_t blk = 0; blk < n_blocks; ++blk) {
        if (!flag[(size_t)blk]) continue;
        const int64_t a = blk * kBlock, b = std::min(n, a + kBlock);
        for (int64_t i = a; i < b; ++i) {
            const uint32_t v = src[i];
            if (v < XI_PACK_ESCAPE || v == 0xFFFFFFFFu) continue;
            if (k == exc_cap) {
                *n_exc = k;
                return xi_fail(XI_E_LIMIT, "xi_pack_u8: more exceptions than exc_cap");
            }
            exc[2 * k] = (uint32_t)i;
            exc[2 * k + 1] = v;
            ++k;
        }
    }
    *n_exc = k;
    return XI_OK;
}
