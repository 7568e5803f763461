// pw_band16.cuh -- the band score sweep of two long pairs at once, 16x2.
//
// Two explicit pairs that share their query and whose targets have the same
// length (a pair and the pair with the target's reverse complement, as the
// long-DNA workload lists them) run as one band sweep with each cell's two H
// values in the low and high 16-bit halves of one register: the query
// residues (the steps) are shared, the profile word of a row holds the two
// targets' scores, and every DPX add-max (__viaddmax_s16x2) advances both
// pairs.  Everything else is band_kernel<false, 4>: 256-row bands chained
// across warps, the pair maxima, and per pair the tile form's checkpoints and
// tile maxima, written as int32 for each pair separately -- except that a band
// lags the band above by one 32-column block, with progress published every
// 16 steps (half as many chains run as in the 32-bit form, so the chains'
// length bounds the sweep).
//
// 16-bit halves hold H exactly while every value stays at or below
// 32767 - highest (no add can then wrap); a pair whose maximum passes that
// limit is reported in `over` and swept again on 32-bit lanes by the host.
#pragma once
#include "pw_band.cuh"

namespace pw {

struct BandPair2 {
    int32_t q;            // the shared query
    int32_t t[2];         // targets of the low and high halves (same length)
    int32_t nbands;
    int64_t slot[2];      // pair-list indices (maxima)
    int64_t ck[2];        // int offsets of the pairs' checkpoints
    int64_t tm[2];        // int offsets of the pairs' tile maxima
};

struct BandArgs2 {
    const int4* entries;  // per queue entry: (pair, band, queue index of the band above, 0)
    const BandPair2* pairs;
    int n_entries;
    int* counter;
    int* progress;        // per entry: columns of the bottom row stored (kChainDone when finished)
    int2* run_max;        // per entry: running maxima of the two pairs' bands so far
    int* abort_flag;
    float* max_out;       // pair maxima, indexed by BandPair2.slot
    int* over;            // per pair-list index: 1 when its maximum passed the 16-bit limit
    int* ck;              // checkpoints and tile maxima
    int limit;            // 32767 - highest substitution score
    unsigned long long wait_ns;
};

__device__ __forceinline__ int lo16(uint32_t v) { return (int)(int16_t)(v & 0xffffu); }
__device__ __forceinline__ int hi16(uint32_t v) { return (int)(int16_t)(v >> 16); }
__device__ __forceinline__ uint32_t pack16(int a, int b) {
    return ((uint32_t)(uint16_t)a) | ((uint32_t)(uint16_t)b << 16);
}

__global__ void __launch_bounds__(128, 6) band16_kernel(KernelArgs A, BandArgs2 B) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int alpha1 = A.P.alpha + 1;
    // [lane][alpha1] -> 8 rows x (score of target 0 | score of target 1 << 16)
    const int prof_bytes = kWarp * alpha1 * kWarpRows * 4;
    uint4* prof = (uint4*)(smem + wib * prof_bytes);
    const uint32_t gap2 = pack16(A.P.gap_i, A.P.gap_i);
    const uint32_t neg2 = 0x80008000u;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(B.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= B.n_entries) break;
        const int4 en = B.entries[it];
        const BandPair2 BP = B.pairs[en.x];
        const int band = en.y, pred = en.z;
        const int lq = A.q.len[BP.q], lt = A.t.len[BP.t[0]];
        const int nbands = BP.nbands;
        const uint8_t* qg = A.q.codes + A.q.code_off[BP.q];
        const uint8_t* tr0 = A.t.codes + A.t.code_off[BP.t[0]];
        const uint8_t* tr1 = A.t.codes + A.t.code_off[BP.t[1]];
        const int64_t nsteps = (int64_t)lq + kWarp - 1;
        const int yb = band * kBandRows;
        __syncwarp();
        for (int idx = lane; idx < kWarp * alpha1; idx += kWarp) {
            const int ll = idx / alpha1, a = idx % alpha1;
            uint32_t w[kWarpRows];
#pragma unroll
            for (int r = 0; r < kWarpRows; ++r) {
                const int y = yb + ll * kWarpRows + r;
                const int s0 = y < lt ? A.cmat_i8[a * A.P.dim + tr0[y]] : -128;
                const int s1 = y < lt ? A.cmat_i8[a * A.P.dim + tr1[y]] : -128;
                w[r] = pack16(s0, s1);
            }
            prof[2 * idx] = make_uint4(w[0], w[1], w[2], w[3]);
            prof[2 * idx + 1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
        __syncwarp();
        const bool has_up = band > 0;
        const bool store_bnd = band + 1 < nbands;
        const int ntiles = tile_count(lq);
        const int64_t col0 = tile_col_offset(lq, lt) + ((int64_t)band * ntiles) * kBandRows + lane * kWarpRows;
        int* ck0 = B.ck + BP.ck[0];
        int* ck1 = B.ck + BP.ck[1];
        int* tmax0 = B.ck + BP.tm[0] + (int64_t)band * ntiles;
        int* tmax1 = B.ck + BP.tm[1] + (int64_t)band * ntiles;
        const int* prog_in = B.progress + pred;
        int* prog_out = B.progress + it;
        uint32_t Hl[kWarpRows];
#pragma unroll
        for (int r = 0; r < kWarpRows; ++r) Hl[r] = 0u;
        uint32_t up_h = 0u, bt_h = 0u, mx = 0u, tm = 0u;
        int avail = 0;
        bool ok = true;
        // the row above, 32 columns at a time (both pairs' values packed)
        uint32_t cur = 0u;
        auto fetch = [&](int64_t c) -> uint32_t {
            if (c >= lq) return 0u;
            return pack16(__ldcg(ck0 + (int64_t)(band - 1) * lq + c), __ldcg(ck1 + (int64_t)(band - 1) * lq + c));
        };
        for (int64_t s = 0; s < nsteps; ++s) {
            if (has_up && (s & 31) == 0) {
                // only this block of the row above is waited for (one block
                // of lag between bands; fetching the next block too would
                // double it, and the chains' length is what bounds this sweep)
                const int need = (int)(s + 32 < (int64_t)lq ? s + 32 : (int64_t)lq);
                if (avail < need) {
                    avail = chain_wait(prog_in, need, B.abort_flag, B.wait_ns);
                    if (avail < 0) {
                        ok = false;
                        break;
                    }
                }
                cur = fetch(s + lane);
            }
            const int x = (int)s - lane;
            const bool active = x >= 0 && x < lq;
            uint32_t above = 0u;
            if (has_up) above = __shfl_sync(0xffffffffu, cur, (int)(s & 31));
            uint32_t rh = __shfl_up_sync(0xffffffffu, bt_h, 1);
            if (lane == 0) rh = (has_up && active) ? above : 0u;
            const uint32_t dg_h = x == 0 ? 0u : up_h;
            up_h = rh;
            if (active) {
                const int a = __ldg(qg + x);
                const uint4 p0 = prof[2 * (lane * alpha1 + a)], p1 = prof[2 * (lane * alpha1 + a) + 1];
                const uint32_t sc[kWarpRows] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
                uint32_t up = up_h, diag = dg_h;
#pragma unroll
                for (int r = 0; r < kWarpRows; ++r) {
                    const uint32_t left = Hl[r];
                    uint32_t h = __viaddmax_s16x2(diag, sc[r], neg2);
                    h = __viaddmax_s16x2(left, gap2, h);
                    h = __viaddmax_s16x2_relu(up, gap2, h);
                    diag = left;
                    Hl[r] = h;
                    up = h;
                }
                tm = __vimax3_s16x2(tm, __vimax3_s16x2(Hl[0], Hl[1], Hl[2]),
                                    __vimax3_s16x2(Hl[3], Hl[4], __vimax3_s16x2(Hl[5], Hl[6], Hl[7])));
                bt_h = up;
                if (((x + 1) & (kTileW - 1)) == 0 || x + 1 == lq) {
                    atomicMax(tmax0 + x / kTileW, lo16(tm));
                    atomicMax(tmax1 + x / kTileW, hi16(tm));
                    mx = __vimax_s16x2_relu(mx, tm);
                    tm = 0u;
                }
                if (((x + 1) & (kTileW - 1)) == 0 && x + 1 < lq) {
                    const int64_t o = col0 + (int64_t)((x + 1) / kTileW) * kBandRows;
                    __stcg((int4*)(ck0 + o), make_int4(lo16(Hl[0]), lo16(Hl[1]), lo16(Hl[2]), lo16(Hl[3])));
                    __stcg((int4*)(ck0 + o) + 1, make_int4(lo16(Hl[4]), lo16(Hl[5]), lo16(Hl[6]), lo16(Hl[7])));
                    __stcg((int4*)(ck1 + o), make_int4(hi16(Hl[0]), hi16(Hl[1]), hi16(Hl[2]), hi16(Hl[3])));
                    __stcg((int4*)(ck1 + o) + 1, make_int4(hi16(Hl[4]), hi16(Hl[5]), hi16(Hl[6]), hi16(Hl[7])));
                }
                if (lane == kWarp - 1 && store_bnd) {
                    __stcg(ck0 + (int64_t)band * lq + x, lo16(bt_h));
                    __stcg(ck1 + (int64_t)band * lq + x, hi16(bt_h));
                }
            } else {
                bt_h = 0u;  // not started (x < 0): the left boundary
            }
            // progress every 16 steps
            if (store_bnd && lane == kWarp - 1 && ((s + 1) & 15) == 0 && s >= kWarp - 1)
                st_release_gpu(prog_out, (int)(s - (kWarp - 2)));
        }
        if (!ok) break;
        if (store_bnd && lane == kWarp - 1) st_release_gpu(prog_out, lq);
        int m0 = __reduce_max_sync(0xffffffffu, lo16(mx)), m1 = __reduce_max_sync(0xffffffffu, hi16(mx));
        if (has_up) {
            if (chain_wait(prog_in, kChainDone, B.abort_flag, B.wait_ns) < 0) break;
            const int2 pm = __ldcg(&B.run_max[pred]);
            m0 = max(m0, pm.x);
            m1 = max(m1, pm.y);
        }
        if (store_bnd) {
            if (lane == 0) __stcg(&B.run_max[it], make_int2(m0, m1));
            chain_publish(prog_out, kChainDone);
        } else if (lane == 0) {
            B.max_out[BP.slot[0]] = (float)m0;
            B.max_out[BP.slot[1]] = (float)m1;
            B.over[BP.slot[0]] = m0 > B.limit ? 1 : 0;
            B.over[BP.slot[1]] = m1 > B.limit ? 1 : 0;
        }
    }
}

}  // namespace pw
