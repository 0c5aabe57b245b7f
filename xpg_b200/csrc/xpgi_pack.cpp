// Host-side codecs of the library, on a pool of host threads: the frames' transfer encoding (include/xpgi.h,
// "Transfer encoding": uint32 pixels to one byte each plus (index, value) exceptions), the LZ4 stage of
// bitshuffle-LZ4 chunks, and the INTEGRATE.HKL records. The transfer encoding: The work is a streaming read of the frames, so the pool
// splits a run into slices of kSlice pixels handed out in order; each slice records which of its kBlock-pixel
// blocks hold an exception, and the calling thread lists those blocks' exceptions afterwards, in pixel order.
#include <immintrin.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <string>
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

// ---- bitshuffle-LZ4 chunks: the LZ4 stage ----------------------------------------------------------------------
// Chunk layout (HDF5 filter 32008): 8-byte big-endian uncompressed size, 4-byte big-endian block size (0: 8192), then
// per block a 4-byte big-endian compressed size and an LZ4 block; a last partial block's n % 8 elements follow as
// they are. The block headers are walked once on the calling thread, then the blocks decompress on the pool.
namespace {

uint64_t be(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v = (v << 8) | p[i];
    return v;
}

// one LZ4 block (the published block format) into exactly n_out bytes; false on a malformed block
bool lz4_block(const uint8_t* src, int64_t n, uint8_t* dst, int64_t n_out) {
    int64_t ip = 0, op = 0;
    for (;;) {
        if (ip >= n) return false;
        const unsigned token = src[ip++];
        int64_t lit = token >> 4;
        if (lit == 15) {
            unsigned b;
            do {
                if (ip >= n) return false;
                b = src[ip++];
                lit += b;
            } while (b == 255);
        }
        if (lit > n - ip || lit > n_out - op) return false;
        memcpy(dst + op, src + ip, (size_t)lit);
        ip += lit;
        op += lit;
        if (ip == n) break;                          // the last sequence: literals only
        if (n - ip < 2) return false;
        const int64_t off = (int64_t)src[ip] | ((int64_t)src[ip + 1] << 8);
        ip += 2;
        int64_t ml = token & 15;
        if (ml == 15) {
            unsigned b;
            do {
                if (ip >= n) return false;
                b = src[ip++];
                ml += b;
            } while (b == 255);
        }
        ml += 4;
        if (off == 0 || off > op || ml > n_out - op) return false;
        uint8_t* d = dst + op;
        for (int64_t k = 0; k < ml;) {               // pieces of at most `off` bytes never overlap their source
            const int64_t c = std::min(off, ml - k);
            memcpy(d + k, d + k - off, (size_t)c);
            k += c;
        }
        op += ml;
    }
    return op == n_out;
}

struct Lz4Block {
    int64_t src, csize, dst, bytes;
};

}  // namespace

extern "C" int xi_bslz4_lz4_stage(const uint8_t* chunk, int64_t chunk_bytes, int esize, uint8_t* out, int64_t out_bytes,
                                  int threads, int64_t* n_bytes, int64_t* block_elems) {
    if (!chunk || !out || !n_bytes || !block_elems || chunk_bytes < 0 || out_bytes < 0)
        return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: null pointer or negative size");
    if (esize != 2 && esize != 4) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: element size must be 2 or 4");
    if (chunk_bytes < 12) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: chunk shorter than its header");
    const uint64_t total = be(chunk, 8);
    const uint64_t bsize = be(chunk + 8, 4) ? be(chunk + 8, 4) : 8192;
    if (total % (uint64_t)esize || total > (uint64_t)out_bytes)
        return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: uncompressed size is not a whole frame of this buffer");
    const int64_t n = (int64_t)(total / esize);
    int64_t belem = (int64_t)(bsize / esize);
    belem -= belem % 8;
    if (belem <= 0) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: block smaller than 8 elements");
    std::vector<Lz4Block> blocks;
    blocks.reserve((size_t)(n / belem + 1));
    int64_t pos = 12, done = 0;
    while (done < n) {
        const int64_t m = std::min(belem, n - done), m8 = m - m % 8;
        if (m8) {
            if (chunk_bytes - pos < 4) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: truncated block header");
            const int64_t c = (int64_t)be(chunk + pos, 4);
            pos += 4;
            if (c > chunk_bytes - pos) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: block beyond the chunk");
            blocks.push_back({pos, c, done * esize, m8 * esize});
            pos += c;
        }
        if (m8 < m) {
            const int64_t r = (m - m8) * esize;
            if (r > chunk_bytes - pos) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: truncated trailing elements");
            memcpy(out + (done + m8) * esize, chunk + pos, (size_t)r);
            pos += r;
        }
        done += m;
    }
    std::atomic<int> bad{0};
    if (!blocks.empty()) {
        pool().run((int64_t)blocks.size(), threads <= 0 ? default_threads() : threads, [&](int64_t i) {
            const Lz4Block& b = blocks[(size_t)i];
            if (!lz4_block(chunk + b.src, b.csize, out + b.dst, b.bytes)) bad.store(1);
        });
    }
    if (bad.load()) return xi_fail(XI_E_ARG, "xi_bslz4_lz4_stage: malformed LZ4 block");
    *n_bytes = (int64_t)total;
    *block_elems = belem;
    return XI_OK;
}

// ---- INTEGRATE.HKL data records ---------------------------------------------------------------------------------
// Rows are formatted in chunks on the pool (C's printf conversions %.3E / %.1f / %.5f / %.2f round exactly as the
// Python format specifications of the same names), then concatenated in row order.
#include <stdio.h>
#include <string>

namespace {

void hkl_line(const XiHklRows* r, int64_t i, std::string& s) {
    char line[512];
    auto fmt = [&](char* buf, size_t cap) {
        return snprintf(buf, cap,
                        " %lld %lld %lld %.3E %.3E %.1f %.1f %.1f %.5f %.5f %lld 0 %.1f %.1f %.1f %.2f %.2f %.2f %.2f "
                        "0.00 1\n",
                        (long long)r->hkl[3 * i], (long long)r->hkl[3 * i + 1], (long long)r->hkl[3 * i + 2], r->I[i],
                        r->sig[i], r->x[i], r->y[i], r->zc[i], r->rlp[i], r->peak[i], (long long)r->corr[i], r->xo[i],
                        r->yo[i], r->zo[i], r->alf0, r->bet0, r->alf1[i], r->bet1[i]);
    };
    const int n = fmt(line, sizeof line);
    if (n < 0) return;
    if ((size_t)n < sizeof line) {
        s.append(line, (size_t)n);
    } else {                                        // a huge value: format again at its length
        std::vector<char> big((size_t)n + 1);
        fmt(big.data(), big.size());
        s.append(big.data(), (size_t)n);
    }
}

}  // namespace

extern "C" int xi_format_integrate_hkl(const XiHklRows* r, char* out, int64_t cap, int threads, int64_t* n_bytes) {
    if (!r || !n_bytes || r->n < 0 || cap < 0 || (cap && !out))
        return xi_fail(XI_E_ARG, "xi_format_integrate_hkl: null pointer or negative size");
    if (r->n && (!r->hkl || !r->I || !r->sig || !r->x || !r->y || !r->zc || !r->rlp || !r->peak || !r->corr ||
                 !r->xo || !r->yo || !r->zo || !r->alf1 || !r->bet1))
        return xi_fail(XI_E_ARG, "xi_format_integrate_hkl: null column");
    const int64_t per = 4096;
    const int64_t n_items = (r->n + per - 1) / per;
    std::vector<std::string> parts((size_t)n_items);
    if (n_items)
        pool().run(n_items, threads <= 0 ? default_threads() : threads, [&](int64_t it) {
            std::string& s = parts[(size_t)it];
            s.reserve((size_t)per * 128);
            const int64_t a = it * per, b = std::min(r->n, a + per);
            for (int64_t i = a; i < b; ++i) hkl_line(r, i, s);
        });
    int64_t total = 0;
    for (const auto& s : parts) total += (int64_t)s.size();
    *n_bytes = total;
    if (total > cap) return xi_fail(XI_E_LIMIT, "xi_format_integrate_hkl: buffer too small (size in *n_bytes)");
    int64_t o = 0;
    for (const auto& s : parts) {
        memcpy(out + o, s.data(), s.size());
        o += (int64_t)s.size();
    }
    return XI_OK;
}
