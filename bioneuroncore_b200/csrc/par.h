// par.h -- host loops on all cores, for the builder and the exporter.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

namespace bnc {

// Runs f(begin, end) over [0, n) in contiguous chunks on up to hardware_concurrency
// threads (one chunk per thread); small ranges run inline.  Used for loops whose
// iterations write disjoint outputs, so the result does not depend on the split.
template <typename F>
void parallel_for(size_t n, F&& f, size_t min_chunk = 1 << 16) {
    unsigned T = std::thread::hardware_concurrency();
    if (T == 0) T = 1;
    T = std::min<unsigned>(T, 32u);
    const size_t chunks = std::min<size_t>(T, (n + min_chunk - 1) / min_chunk);
    if (chunks <= 1) { f((size_t)0, n); return; }
    const size_t per = (n + chunks - 1) / chunks;
    std::vector<std::thread> th;
    th.reserve(chunks);
    for (size_t c = 0; c < chunks; c++) {
        const size_t b = c * per, e = std::min(n, b + per);
        if (b < e) th.emplace_back([&f, b, e]() { f(b, e); });
    }
    for (auto& t : th) t.join();
}

// The lowest index at which a parallel loop found an error (UINT64_MAX: none).
struct FirstError {
    std::atomic<uint64_t> at{UINT64_MAX};
    void note(uint64_t i) {
        uint64_t cur = at.load();
        while (i < cur && !at.compare_exchange_weak(cur, i)) {}
    }
    bool any() const { return at.load() != UINT64_MAX; }
};

}  // namespace bnc
