// pw_host.h -- host-side helpers shared by the engine, the native formatters
// and the record reader.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

// f(begin, end) over [0, n) in up to 32 contiguous chunks of at least
// min_chunk elements, one host thread each (the caller's thread alone when
// one chunk covers n).
template <typename F>
static void parallel_for(int64_t n, F&& f, int64_t min_chunk = 1 << 15) {
    const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
    const int T = (int)std::min<int64_t>(std::min<int64_t>(hw, 32), std::max<int64_t>(1, n / min_chunk));
    if (T <= 1) {
        f((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(T);
    for (int k = 0; k < T; ++k) th.emplace_back([&, k] { f(n * k / T, n * (k + 1) / T); });
    for (auto& t : th) t.join();
}

// Stable order of n uint64 keys (LSD radix, 16 bits a pass, skipping the
// digits in which every key agrees); keys travel with their indices.
static std::vector<uint32_t> radix_order(std::vector<uint64_t> key) {
    const size_t n = key.size();
    uint64_t differ = 0;
    for (size_t k = 0; k < n; ++k) differ |= key[k] ^ key[0];
    std::vector<uint32_t> idx(n), tmp(n);
    for (size_t k = 0; k < n; ++k) idx[k] = (uint32_t)k;
    std::vector<uint64_t> ktmp(n);
    std::vector<uint32_t> cnt(65537);
    for (int shift = 0; shift < 64 && n > 0; shift += 16) {
        if (((differ >> shift) & 0xffff) == 0) continue;
        std::fill(cnt.begin(), cnt.end(), 0u);
        for (size_t k = 0; k < n; ++k) cnt[((key[k] >> shift) & 0xffff) + 1]++;
        for (int d = 0; d < 65536; ++d) cnt[d + 1] += cnt[d];
        for (size_t k = 0; k < n; ++k) {
            const uint32_t pos = cnt[(key[k] >> shift) & 0xffff]++;
            tmp[pos] = idx[k];
            ktmp[pos] = key[k];
        }
        idx.swap(tmp);
        key.swap(ktmp);
    }
    return idx;
}
