// pw_plan.h -- host-side queue planning of the chained 16-bit score sweep
// (score16_chain_kernel).  Plain C++, no CUDA: the plan is a pure function of
// the items' shapes, so it is tested and timed without a GPU.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace pw {

struct PlanEntry {
    int32_t item;   // index of the source item (in the order given)
    int32_t chain;  // chain index, -1 for a whole item
    int32_t strip;  // strip index in the chain, -1 for a whole item
    int32_t pred;   // queue index of the chain's previous strip, -1 if none
};

struct ChainPlan {
    std::vector<PlanEntry> queue;
    std::vector<int64_t> chain_xm4;  // per chain: its column count (ring row length / 32)
};

// Items (already ordered longest first) have nstr[k] strips of xm4[k]
// columns.  Items whose cost nstr * xm4 reaches permille/1000 of the mean
// per-warp load become chains of one-strip entries; the rest stay whole.
// The queue comes from a list-scheduling simulation of `warps` equally fast
// warps, time counted in columns of one strip: a warp that frees up takes the
// next strip of the chain that became ready first (its predecessor started at
// least `lead` columns ago; ties go to the longer chain), else the next whole
// item, else the chain strip that becomes ready first.  Every strip is queued
// after its predecessor.
inline void plan_chain_queue(const std::vector<int>& nstr, const std::vector<int64_t>& xm4, int warps,
                             int64_t permille, int lead, ChainPlan& out) {
    const int n = (int)nstr.size();
    out.queue.clear();
    out.chain_xm4.clear();
    warps = std::max(1, warps);
    double total = 0;
    for (int k = 0; k < n; ++k) total += (double)xm4[k] * nstr[k];
    const double thr = total / warps * (double)permille / 1000.0;
    std::vector<int32_t> chain_item, whole;
    for (int k = 0; k < n; ++k) {
        if (nstr[k] >= 2 && (double)xm4[k] * nstr[k] >= thr)
            chain_item.push_back(k);
        else
            whole.push_back(k);
    }
    const int nc = (int)chain_item.size();
    out.chain_xm4.resize(nc);
    std::vector<int32_t> next(nc, 0), last_q(nc, -1);
    size_t n_sub = whole.size();
    for (int c = 0; c < nc; ++c) {
        out.chain_xm4[c] = xm4[chain_item[c]];
        n_sub += (size_t)nstr[chain_item[c]];
    }
    out.queue.reserve(n_sub);
    // min-heaps on int64 keys: warps by free time; ready chains by
    // (ready time << 24 | chain), chain < 2^24
    std::vector<int64_t> freew((size_t)warps, 0);
    std::vector<int64_t> ready;
    ready.reserve(nc);
    for (int c = 0; c < nc; ++c) ready.push_back((int64_t)c);  // ready at 0, chain order
    std::make_heap(ready.begin(), ready.end(), std::greater<int64_t>());
    size_t wnext = 0;
    int open = nc;
    while (open > 0) {
        std::pop_heap(freew.begin(), freew.end(), std::greater<int64_t>());
        const int64_t t = freew.back();
        int64_t done;
        const bool take_chain = (ready.front() >> 24) <= t || wnext >= whole.size();
        if (take_chain) {
            std::pop_heap(ready.begin(), ready.end(), std::greater<int64_t>());
            const int64_t key = ready.back();
            ready.pop_back();
            const int c = (int)(key & 0xffffff);
            const int64_t start = std::max(t, key >> 24);
            out.queue.push_back(PlanEntry{chain_item[c], c, next[c], last_q[c]});
            last_q[c] = (int32_t)out.queue.size() - 1;
            done = start + out.chain_xm4[c];
            if (++next[c] < nstr[chain_item[c]]) {
                ready.push_back(((start + lead) << 24) | c);
                std::push_heap(ready.begin(), ready.end(), std::greater<int64_t>());
            } else {
                --open;
            }
        } else {
            const int k = whole[wnext++];
            out.queue.push_back(PlanEntry{k, -1, -1, -1});
            done = t + xm4[k] * nstr[k];
        }
        freew.back() = done;
        std::push_heap(freew.begin(), freew.end(), std::greater<int64_t>());
    }
    // the chains are all queued: the remaining whole items follow, longest first
    for (; wnext < whole.size(); ++wnext) out.queue.push_back(PlanEntry{whole[wnext], -1, -1, -1});
}

}  // namespace pw
