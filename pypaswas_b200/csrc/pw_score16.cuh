// pw_score16.cuh -- the 16-bit score sweep: two pairs per lane.
//
// Pair maxima only (the engine's first phase).  Every 32-bit register holds
// the same DP cell of two different pairs as signed 16-bit halves, and the
// recurrences run on the DPX 16x2 instructions (__viaddmax_s16x2 and friends),
// which update two cells per instruction at the rate of one 32-bit update.
// A warp aligns two "strip" sequences (low and high halves) against up to 32
// "lane" sequences, one per lane.  Both halves of a lane read the same lane
// residue, so the strip profile stores ready-made 16x2 score pairs: one
// 128-bit shared-memory load yields the scores of four strip rows for both
// strip sequences.  Which input set provides the strips and which the lanes
// is chosen per run by the host (pair maxima are symmetric in the two
// sequences, so either orientation gives the same maxima).
//
// Overflow: with every score in [-127, 127], no 16-bit operation can exceed
// 32767 while all cell values stay below kOvf16 (32640 = 32767 - 127).  A pair
// whose maximum reaches kOvf16 is reported as NaN and recomputed by the 32-bit
// sweep.
#pragma once
#include "pw_kernels.cuh"

namespace pw {

constexpr int kOvf16 = 32767 - 127;
constexpr uint32_t kNeg16x2 = 0xC000C000u;  // -16384 in both halves (boundary of the gap chains)

__device__ __forceinline__ uint32_t pack16(int v) { return ((uint32_t)v & 0xffffu) * 0x00010001u; }
__device__ __forceinline__ uint32_t pack16x2(int lo, int hi) {
    return ((uint32_t)lo & 0xffffu) | ((uint32_t)hi << 16);
}

struct Score16Args {
    const WorkItem* items;   // target = strip A, index = strip B (or -1), first/lanes index the lane order
    int n_items;
    int* counter;
    const uint8_t* lane_codes;   // compact lane-alphabet codes, 16-aligned, pad-coded tail
    const int64_t* lane_off;
    const int32_t* lane_len;
    const int32_t* lane_order;   // sorted position -> lane sequence
    const uint8_t* strip_res;    // strip residues as matrix indices, 16-aligned
    const int64_t* strip_off;
    const int32_t* strip_len;
    const int8_t* cmat;          // [(alpha + 1) * dim] scores lane residue x strip residue
    int alpha1, dim;
    int gap, ext, ge;
    float* pair_max;
    int64_t stride_strip, stride_lane;  // pair_max[strip * stride_strip + lane * stride_lane]
    uint4* bnd_pool;
    int64_t bnd_slot;            // uint4 elements per warp slot (xmax4 * 32)
    // multi-strip launch with chains (score16_chain_kernel): per queue entry
    // (chain, strip, queue index of the chain's previous strip); strip -1 marks
    // a whole item swept by one warp with its boundary in bnd_pool
    const int4* chain;
    const int64_t* ring_off;     // per chain: its two boundary rows (xm4 * 32 uint4 each) in `ring`
    uint4* ring;
    int* progress;               // per queue entry: columns whose boundary row is written (kChainDone when finished)
    uint32_t* run_max;           // per queue entry x 32 lanes: running 16x2 maximum of the chain so far
    int pad_code;                // lane code of the padding residue
    int* abort_flag;             // set when a wait runs out of time; every waiting warp then gives up
    int n_chain_items;           // host-side bookkeeping: entries of the chained launch
    int item_base;               // chained launch: first queue entry of this launch (entries [item_base, n_items))
    int* ovf_count;              // pairs reported as NaN (16-bit limit reached)
    unsigned long long wait_ns;  // bound of one chain wait
    // grid form of a one-strip class launch (no item list): item `it` is lane
    // group it / grid_n_strips (grid_lane_step lanes from the sorted position
    // it / grid_n_strips * grid_lane_step) against strip pair
    // grid_strips[it % grid_n_strips] (x: strip A, y: strip B or -1)
    const int2* grid_strips;     // null: items come from `items`
    int grid_n_strips;
    int grid_lane_step;          // 32, or 64 for the dual-lane form
    int grid_n_lane;             // lane sequences in the sorted order
};

// Profile of strip rows [y0, y0 + S): for row group g (4 rows) and lane
// residue a, one uint4 holds the 16x2 scores of the 4 rows, strip A in the low
// halves and strip B in the high halves.  Rows past a strip's end get -128.
// Affine sweeps store score + gap_open in the halves (see sweep16).
template <int S>
__device__ __forceinline__ void build_profile16(uint4* prof, const int8_t* cmat, const uint8_t* ra,
                                                const uint8_t* rb, int y0, int la, int lb, int alpha1, int dim,
                                                int shift, int lane) {
    const int n = (S / 4) * alpha1;
    for (int idx = lane; idx < n; idx += kWarp) {
        const int g = idx / alpha1, a = idx % alpha1;
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = y0 + 4 * g + k;
            const int sa = y < la ? (int)cmat[a * dim + ra[y]] : -128;
            const int sb = y < lb ? (int)cmat[a * dim + rb[y]] : -128;
            w[k] = pack16x2(sa + shift, sb + shift);
        }
        prof[idx] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Dual-lane form: one strip sequence against two lane sequences per lane (the
// lanes' own group in the low halves, the next 32-lane group in the high
// halves).  The halves then read different lane residues, so the profile
// holds plain 16-bit scores, [row group][lane residue] -> 4 rows in a uint2,
// and the sweep interleaves the two residues' words with byte permutes.
template <int S>
__device__ __forceinline__ void build_profile16_dual(uint2* prof, const int8_t* cmat, const uint8_t* ra, int y0,
                                                     int la, int alpha1, int dim, int shift, int lane) {
    const int n = (S / 4) * alpha1;
    for (int idx = lane; idx < n; idx += kWarp) {
        const int g = idx / alpha1, a = idx % alpha1;
        int v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = y0 + 4 * g + k;
            v[k] = (y < la ? (int)cmat[a * dim + ra[y]] : -128) + shift;
        }
        prof[idx] = make_uint2(pack16x2(v[0], v[1]), pack16x2(v[2], v[3]));
    }
}

// The 16x2 scores of rows 4g .. 4g + 3: profile entries `ia` (low halves) and
// `ib` (high halves; the dual-lane form only).
template <bool DL>
__device__ __forceinline__ void fetch16(const void* prof, int ia, int ib, uint32_t (&sc)[4]) {
    if constexpr (!DL) {
        const uint4 w = ((const uint4*)prof)[ia];
        sc[0] = w.x;
        sc[1] = w.y;
        sc[2] = w.z;
        sc[3] = w.w;
    } else {
        const uint2 lo = ((const uint2*)prof)[ia], hi = ((const uint2*)prof)[ib];
        sc[0] = __byte_perm(lo.x, hi.x, 0x5410);
        sc[1] = __byte_perm(lo.x, hi.x, 0x7632);
        sc[2] = __byte_perm(lo.y, hi.y, 0x5410);
        sc[3] = __byte_perm(lo.y, hi.y, 0x7632);
    }
}

template <bool DL>
__host__ __device__ constexpr int prof_entry_bytes() { return DL ? (int)sizeof(uint2) : (int)sizeof(uint4); }

// Bytes of the four warps' profiles of a 128-thread block, rounded to 16.
template <int S, bool DL>
__host__ __device__ constexpr int chain_profile_bytes(int alpha1) {
    return (4 * (S / 4) * alpha1 * prof_entry_bytes<DL>() + 15) & ~15;
}

// This warp's profile in shared memory (typed offsets keep the address a
// 32-bit shared-window computation).
template <int S, bool DL>
__device__ __forceinline__ void* warp_profile(unsigned char* smem, int wib, int alpha1) {
    if constexpr (DL) return (uint2*)smem + wib * ((S / 4) * alpha1);
    else return (uint4*)smem + wib * ((S / 4) * alpha1);
}

// One lane, two pairs (strip A / strip B against the lane sequence).
//   linear: H = max(diag + s, left + gap, up + gap, 0)                 3 DPX / row
//   affine: carries Mg = M + gap_open (gap_open = gap + ext):
//     M  = max(Bdiag + s, 0)          Mg = M + ge  (profile holds s + ge,
//     so Mg = max(Bdiag + (s + ge), ge) in one instruction)
//     Y  = max(Yup + ext, Mg_up)      strip-axis gap chain
//     X  = max(Xleft + ext, Mg_left)  sweep-axis gap chain
//     B  = max(Mg - ge, Y, X)          as max(M, Y, X)                 5 DPX / row
//
// Dual-lane form (DL): the high halves sweep a second lane sequence (qc2,
// lq42) against the same strip; the column loop runs to the longer of the two
// and a sequence past its end reads padding codes (pad4), which cannot raise
// its maximum.
template <int S, bool AFFINE, bool DL>
__device__ __forceinline__ void sweep16(const uint8_t* qc, int lq4, const uint8_t* qc2, int lq42, uint32_t pad4,
                                        const void* prof, int alpha1, int gap, int ext, int ge, bool has_up,
                                        bool has_down, uint4* bnd, uint32_t& mx) {
    const uint32_t g2 = pack16(gap), e2 = pack16(ext), ge2 = pack16(ge), nge2 = pack16(-ge);
    auto word = [&](const uint8_t* q, int lim, int x4) -> uint32_t {
        return !DL || x4 < lim ? *(const uint32_t*)(q + x4) : pad4;
    };
    const int lqa = lq4;  // the low halves' own columns
    if constexpr (DL) lq4 = lq4 > lq42 ? lq4 : lq42;
    if constexpr (!AFFINE) {
        uint32_t H[S];
#pragma unroll
        for (int r = 0; r < S; ++r) H[r] = 0;
        uint32_t hb_prev = 0;
        // the code word of the next 4 columns and the boundary value of the
        // next column are loaded one step ahead (their latency hides behind a
        // column of arithmetic)
        uint32_t cw_next = lq4 > 0 ? word(qc, lqa, 0) : 0u;
        uint32_t cw2_next = DL && lq4 > 0 ? word(qc2, lq42, 0) : 0u;
        uint32_t up_next = has_up && lq4 > 0 ? bnd[0].x : 0u;
        for (int x4 = 0; x4 < lq4; x4 += 4) {
            const uint32_t cw = cw_next, cw2 = cw2_next;
            if (x4 + 4 < lq4) {
                cw_next = word(qc, lqa, x4 + 4);
                if constexpr (DL) cw2_next = word(qc2, lq42, x4 + 4);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const int a2 = DL ? (cw2 >> (8 * j)) & 0xff : 0;
                uint32_t up = up_next;
                if (has_up && x + 1 < lq4) up_next = bnd[(int64_t)(x + 1) * kWarp].x;
                uint32_t diag = hb_prev;
                hb_prev = up;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    uint32_t sc[4];
                    fetch16<DL>(prof, g * alpha1 + a, g * alpha1 + a2, sc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t left = H[r];
                        uint32_t t = __viaddmax_s16x2(diag, sc[k], kNeg16x2);   // diag + s
                        t = __viaddmax_s16x2(left, g2, t);                      // max(left + gap, .)
                        const uint32_t h = __viaddmax_s16x2_relu(up, g2, t);    // max(up + gap, ., 0)
                        diag = left;
                        H[r] = h;
                        up = h;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = __vimax3_s16x2(mx, H[r], H[r + 1]);
                if (has_down) bnd[(int64_t)x * kWarp].x = H[S - 1];
            }
        }
    } else {
        // Zl[r] = max(X + ext, M + gap_open) of the previous column: exactly
        // this column's X (the sweep-axis gap chain), one row array instead of
        // two (X and M + gap_open); M = 0 and X = -inf left of the matrix
        uint32_t Zl[S], Bl[S];
#pragma unroll
        for (int r = 0; r < S; ++r) {
            Zl[r] = ge2;
            Bl[r] = 0;
        }
        uint32_t bb_prev = 0;
        uint32_t cw_next = lq4 > 0 ? word(qc, lqa, 0) : 0u;
        uint32_t cw2_next = DL && lq4 > 0 ? word(qc2, lq42, 0) : 0u;
        uint4 v_next = has_up && lq4 > 0 ? bnd[0] : make_uint4(ge2, kNeg16x2, 0u, 0u);
        uint4 v_next2 = has_up && lq4 > 1 ? bnd[kWarp] : make_uint4(ge2, kNeg16x2, 0u, 0u);
        for (int x4 = 0; x4 < lq4; x4 += 4) {
            const uint32_t cw = cw_next, cw2 = cw2_next;
            if (x4 + 4 < lq4) {
                cw_next = word(qc, lqa, x4 + 4);
                if constexpr (DL) cw2_next = word(qc2, lq42, x4 + 4);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const int a2 = DL ? (cw2 >> (8 * j)) & 0xff : 0;
                const uint4 v = v_next;
                v_next = v_next2;
                if (has_up && x + 2 < lq4) v_next2 = bnd[(int64_t)(x + 2) * kWarp];
                uint32_t mgup = v.x, yup = v.y, bup = v.z;
                uint32_t bdiag = bb_prev;
                bb_prev = bup;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    uint32_t sc[4];
                    fetch16<DL>(prof, g * alpha1 + a, g * alpha1 + a2, sc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t mg = __viaddmax_s16x2(bdiag, sc[k], ge2);   // M + ge
                        const uint32_t y = __viaddmax_s16x2(yup, e2, mgup);
                        const uint32_t xg = Zl[r];
                        const uint32_t bst = __vimax3_s16x2(__viaddmax_s16x2(mg, nge2, kNeg16x2), y, xg);
                        Zl[r] = __viaddmax_s16x2(xg, e2, mg);
                        bdiag = Bl[r];
                        Bl[r] = bst;
                        mgup = mg;
                        yup = y;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = __vimax3_s16x2(mx, Bl[r], Bl[r + 1]);
                if (has_down) bnd[(int64_t)x * kWarp] = make_uint4(mgup, yup, Bl[S - 1], 0u);
            }
        }
    }
}

// ------------------------------------------------------------ chained strips
// A multi-strip item (two strip sequences against 32 lane sequences) is cut
// into one item per 32-row strip.  Strip s of a chain runs on whichever warp
// takes it, a few columns behind strip s - 1: it reads the boundary row that
// strip s - 1 writes into the chain's ring slot (two rows, alternating), as
// far as strip s - 1 has published its progress.  So one long item no longer
// runs on a single warp from its first row to its last.
//
// Ordering: the writer stores its boundary values, every lane fences
// (fence.acq_rel.gpu), the warp synchronises, and lane 0 publishes the column
// count with st.release.gpu; readers poll with ld.acquire.gpu and read the
// ring with ld.global.cg (L2, never a stale L1 line).  A ring row is
// rewritten by strip s + 2 only after strip s + 1 has published progress past
// those columns, i.e. after it has read them.
//
// Progress: entries are handed out in queue order and a strip waits only for
// its predecessor, which is queued before it and so was taken by a warp that
// is running; every wait therefore ends.  Each wait is nevertheless bounded:
// after the launch's wait limit (kChainWaitNs unless the host sets another)
// without progress, or when another warp has given up, the
// warp sets abort_flag and stops, and the host reports the launch as failed.
// Only the longest items are chained (the host plans the queue so that a
// strip is handed out about when its predecessor is kChainLead columns
// ahead); the others run whole on one warp, as in score16_kernel.
constexpr int kChainDone = 1 << 30;
// A strip publishes its progress every kChainPublish columns (one fence per
// lane each time); its successor starts once kChainLead columns are out and
// afterwards asks for kChainNeed columns beyond its current block, so that in
// the steady state it runs a publish period or more behind and its polls
// find the columns already there.
constexpr int kChainPublish = 32;
constexpr int kChainLead = 64;
constexpr int kChainNeed = 40;
// Default bound of one wait (PW_TUNE_WAIT_NS overrides it per launch).
constexpr unsigned long long kChainWaitNs = 2000000000ull;
// Columns of the ring row above that the affine chained sweep keeps in
// flight: each lane copies its own 16-byte entry into a per-warp shared-memory
// ring with cp.async, kPre - 1 columns ahead of the column it computes (within
// the kChainNeed columns the chain wait guarantees).
constexpr int kPre = 8;
static_assert(kPre - 1 < kChainNeed - 4, "prefetched columns must be published");

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Warp-uniform wait until *flag >= need.  Returns the smallest value the lanes
// saw (>= need), or -1 when the wait gave up after limit_ns without success or
// because another warp had given up (abort_flag is then set).
__device__ __forceinline__ int chain_wait(const int* flag, int need, int* abort_flag, unsigned long long limit_ns) {
    int v = ld_acquire_gpu(flag);
    if (__all_sync(0xffffffffu, v >= need)) return __reduce_min_sync(0xffffffffu, v);
    const unsigned long long t0 = global_ns();
    unsigned ns = 32;
    for (;;) {
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
        v = ld_acquire_gpu(flag);
        if (__all_sync(0xffffffffu, v >= need)) return __reduce_min_sync(0xffffffffu, v);
        const bool give_up = ld_acquire_gpu(abort_flag) != 0 || global_ns() - t0 > limit_ns;
        if (__any_sync(0xffffffffu, give_up)) {
            if ((threadIdx.x & 31) == 0) atomicExch(abort_flag, 1);
            return -1;
        }
    }
}

// Publishes `v` as the item's progress after this warp's boundary stores.
__device__ __forceinline__ void chain_publish(int* flag, int v) {
    fence_acq_rel_gpu();
    __syncwarp();
    if ((threadIdx.x & 31) == 0) st_release_gpu(flag, v);
}

// sweep16 for one strip of a chain.  The column loop runs to the warp's
// longest lane (xm4, warp-uniform); a lane past its own sequence sweeps
// padding-code columns, which cannot raise its maximum.  Returns false when a
// wait gave up.
template <int S, bool AFFINE, bool DL>
__device__ __forceinline__ bool sweep16_chain(const uint8_t* qc, int lq4, const uint8_t* qc2, int lq42, int xm4,
                                              uint32_t pad4, const void* prof, int alpha1, int gap, int ext, int ge,
                                              bool has_up, bool has_down, const uint4* ring_in, uint4* ring_out,
                                              const int* prog_in, int* prog_out, int* abort_flag,
                                              unsigned long long wait_ns, uint4* pre, uint32_t& mx) {
    const uint32_t g2 = pack16(gap), e2 = pack16(ext), ge2 = pack16(ge), nge2 = pack16(-ge);
    int avail = 0;  // columns of the predecessor known to be published
    auto need_cols = [&](int upto) -> bool {  // columns [0, upto) of ring_in readable
        if (!has_up || avail >= upto) return true;
        avail = chain_wait(prog_in, upto, abort_flag, wait_ns);
        return avail >= 0;
    };
    auto code_word = [&](int x4) -> uint32_t { return x4 < lq4 ? *(const uint32_t*)(qc + x4) : pad4; };
    auto code_word2 = [&](int x4) -> uint32_t { return DL && x4 < lq42 ? *(const uint32_t*)(qc2 + x4) : pad4; };
    if (!need_cols(min(kChainLead, xm4))) return false;
    if constexpr (!AFFINE) {
        uint32_t H[S];
#pragma unroll
        for (int r = 0; r < S; ++r) H[r] = 0;
        uint32_t hb_prev = 0;
        uint32_t cw_next = xm4 > 0 ? code_word(0) : pad4;
        uint32_t cw2_next = DL && xm4 > 0 ? code_word2(0) : pad4;
        uint32_t up_next = has_up && xm4 > 0 ? __ldcg(&ring_in[0]).x : 0u;
        for (int x4 = 0; x4 < xm4; x4 += 4) {
            if (!need_cols(min(x4 + kChainNeed, xm4))) return false;
            const uint32_t cw = cw_next, cw2 = cw2_next;
            if (x4 + 4 < xm4) {
                cw_next = code_word(x4 + 4);
                if constexpr (DL) cw2_next = code_word2(x4 + 4);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const int a2 = DL ? (cw2 >> (8 * j)) & 0xff : 0;
                uint32_t up = up_next;
                if (has_up && x + 1 < xm4) up_next = __ldcg(&ring_in[(int64_t)(x + 1) * kWarp]).x;
                uint32_t diag = hb_prev;
                hb_prev = up;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    uint32_t sc[4];
                    fetch16<DL>(prof, g * alpha1 + a, g * alpha1 + a2, sc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t left = H[r];
                        uint32_t t = __viaddmax_s16x2(diag, sc[k], kNeg16x2);
                        t = __viaddmax_s16x2(left, g2, t);
                        const uint32_t h = __viaddmax_s16x2_relu(up, g2, t);
                        diag = left;
                        H[r] = h;
                        up = h;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = __vimax3_s16x2(mx, H[r], H[r + 1]);
                if (has_down) __stcg(&ring_out[(int64_t)x * kWarp], make_uint4(H[S - 1], 0u, 0u, 0u));
            }
            if (has_down && (((x4 + 4) % kChainPublish) == 0 || x4 + 4 >= xm4)) chain_publish(prog_out, x4 + 4);
        }
    } else {
        uint32_t Zl[S], Bl[S];  // as in sweep16
#pragma unroll
        for (int r = 0; r < S; ++r) {
            Zl[r] = ge2;
            Bl[r] = 0;
        }
        uint32_t bb_prev = 0;
        uint32_t cw_next = xm4 > 0 ? code_word(0) : pad4;
        uint32_t cw2_next = DL && xm4 > 0 ? code_word2(0) : pad4;
        // this lane's entries of the ring row above: slot k % kPre holds column k
        uint4* my = pre + (threadIdx.x & 31);
        if (has_up) {
#pragma unroll
            for (int k = 0; k < kPre - 1; ++k) {
                if (k < xm4) cp_async16(&my[k * kWarp], &ring_in[(int64_t)k * kWarp]);
                cp_async_commit();
            }
        }
        for (int x4 = 0; x4 < xm4; x4 += 4) {
            if (!need_cols(min(x4 + kChainNeed, xm4))) {
                cp_async_wait<0>();  // no copy outlives the sweep
                return false;
            }
            const uint32_t cw = cw_next, cw2 = cw2_next;
            if (x4 + 4 < xm4) {
                cw_next = code_word(x4 + 4);
                if constexpr (DL) cw2_next = code_word2(x4 + 4);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const int a2 = DL ? (cw2 >> (8 * j)) & 0xff : 0;
                uint4 v = make_uint4(ge2, kNeg16x2, 0u, 0u);
                if (has_up) {
                    const int xn = x + kPre - 1;  // its slot held column x - 1, already read
                    if (xn < xm4) cp_async16(&my[(xn % kPre) * kWarp], &ring_in[(int64_t)xn * kWarp]);
                    cp_async_commit();
                    cp_async_wait<kPre - 1>();  // column x's copy has landed
                    v = my[(x % kPre) * kWarp];
                }
                uint32_t mgup = v.x, yup = v.y, bup = v.z;
                uint32_t bdiag = bb_prev;
                bb_prev = bup;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    uint32_t sc[4];
                    fetch16<DL>(prof, g * alpha1 + a, g * alpha1 + a2, sc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t mg = __viaddmax_s16x2(bdiag, sc[k], ge2);
                        const uint32_t y = __viaddmax_s16x2(yup, e2, mgup);
                        const uint32_t xg = Zl[r];
                        const uint32_t bst = __vimax3_s16x2(__viaddmax_s16x2(mg, nge2, kNeg16x2), y, xg);
                        Zl[r] = __viaddmax_s16x2(xg, e2, mg);
                        bdiag = Bl[r];
                        Bl[r] = bst;
                        mgup = mg;
                        yup = y;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = __vimax3_s16x2(mx, Bl[r], Bl[r + 1]);
                if (has_down) __stcg(&ring_out[(int64_t)x * kWarp], make_uint4(mgup, yup, Bl[S - 1], 0u));
            }
            if (has_down && (((x4 + 4) % kChainPublish) == 0 || x4 + 4 >= xm4)) chain_publish(prog_out, x4 + 4);
        }
        cp_async_wait<0>();
    }
    return true;
}

// One item's lanes.  Strip-pair form: strip A (W.target) in the low halves,
// strip B (W.index, or none) in the high halves, one lane sequence per lane.
// Dual-lane form (DL): strip W.target in both halves, the lane sequences of
// sorted positions W.first + lane (low) and W.first + 32 + lane (high, the
// first W.lanes_hi lanes).
struct Lanes16 {
    bool active;        // the low half's lane sequence exists
    int p, p2;          // lane sequences of the low / high halves
    const uint8_t* qc;  // their codes
    const uint8_t* qc2;
    int lq4, lq42;      // their lengths rounded up to 4 (0: padding only)
};

template <bool DL>
__device__ __forceinline__ Lanes16 item_lanes(const Score16Args& A, const WorkItem& W, int lane) {
    Lanes16 L;
    L.active = lane < W.lanes;
    L.p = L.active ? A.lane_order[W.first + lane] : 0;
    L.qc = A.lane_codes + A.lane_off[L.p];
    L.lq4 = L.active ? (A.lane_len[L.p] + 3) & ~3 : 0;
    const bool hi = DL && lane < W.lanes_hi;
    L.p2 = hi ? A.lane_order[W.first + kWarp + lane] : -1;
    L.qc2 = hi ? A.lane_codes + A.lane_off[L.p2] : L.qc;
    L.lq42 = hi ? (A.lane_len[L.p2] + 3) & ~3 : 0;
    return L;
}

// Work item `it` of a grid-form launch (see Score16Args::grid_strips).
template <int S, bool DL>
__device__ __forceinline__ WorkItem grid_item(const Score16Args& A, int it) {
    const int g = it / A.grid_n_strips, p = it - g * A.grid_n_strips;
    const int2 sp = A.grid_strips[p];
    WorkItem W;
    W.target = sp.x;
    W.index = sp.y;
    W.first = g * A.grid_lane_step;
    W.lanes = min(kWarp, A.grid_n_lane - W.first);
    W.lanes_hi = DL ? max(0, min(kWarp, A.grid_n_lane - W.first - kWarp)) : 0;
    W.xmax = A.lane_len[A.lane_order[W.first]];
    W.S = S;
    W.orient = 0;
    W.dir_base = 0;
    W.pair_base = 0;
    return W;
}

// Writes a lane's two pair maxima (NaN where the 16-bit limit was reached).
template <bool DL>
__device__ __forceinline__ void store_max16(const Score16Args& A, const WorkItem& W, const Lanes16& L, uint32_t mx) {
    const int sa = W.target;
    const int s_hi = DL ? (L.p2 >= 0 ? sa : -1) : W.index;
    const int p_hi = DL ? L.p2 : L.p;
    const int ma = (int)(int16_t)(mx & 0xffffu), mb = (int)(int16_t)(mx >> 16);
    A.pair_max[(int64_t)sa * A.stride_strip + (int64_t)L.p * A.stride_lane] =
        ma >= kOvf16 ? __int_as_float(0x7fc00000) : (float)ma;
    if (s_hi >= 0)
        A.pair_max[(int64_t)s_hi * A.stride_strip + (int64_t)p_hi * A.stride_lane] =
            mb >= kOvf16 ? __int_as_float(0x7fc00000) : (float)mb;
    if (ma >= kOvf16 || (s_hi >= 0 && mb >= kOvf16)) atomicAdd(A.ovf_count, 1);
}

template <int S, bool DL>
__device__ __forceinline__ void build_item_profile(void* prof, const Score16Args& A, const uint8_t* ra,
                                                   const uint8_t* rb, int y0, int la, int lb, int shift, int lane) {
    if constexpr (DL)
        build_profile16_dual<S>((uint2*)prof, A.cmat, ra, y0, la, A.alpha1, A.dim, shift, lane);
    else
        build_profile16<S>((uint4*)prof, A.cmat, ra, rb, y0, la, lb, A.alpha1, A.dim, shift, lane);
}

template <int S, bool AFFINE, bool DL>
__global__ void __launch_bounds__(128, 3) score16_chain_kernel(Score16Args A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    void* prof = warp_profile<S, DL>(smem, wib, A.alpha1);
    // after the four warps' profiles: each warp's prefetch ring (affine)
    uint4* pre = (uint4*)(smem + chain_profile_bytes<S, DL>(A.alpha1)) + wib * kPre * kWarp;
    const int shift = AFFINE ? A.ge : 0;
    const uint32_t pad4 = (uint32_t)A.pad_code * 0x01010101u;
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    uint4* bnd = A.bnd_pool + warp_global * A.bnd_slot + lane;
    for (;;) {
        int it = 0;
        if (lane == 0) it = A.item_base + atomicAdd(A.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const WorkItem W = A.items[it];
        const int4 ci = A.chain[it];
        const int c = ci.x, s = ci.y, pred = ci.z;
        const int sa = W.target, sb = DL ? -1 : W.index;
        const int la = A.strip_len[sa];
        const int lb = sb >= 0 ? A.strip_len[sb] : 0;
        const int ls = la > lb ? la : lb;
        const int nstrips = (ls + S - 1) / S;
        const Lanes16 L = item_lanes<DL>(A, W, lane);
        const uint8_t* ra = A.strip_res + A.strip_off[sa];
        const uint8_t* rb = A.strip_res + A.strip_off[sb >= 0 ? sb : sa];
        uint32_t mx = 0;
        bool finished = true;
        if (s < 0) {
            // a whole item on this warp, strip after strip
            for (int st = 0; st < nstrips; ++st) {
                __syncwarp();
                build_item_profile<S, DL>(prof, A, ra, rb, st * S, la, lb, shift, lane);
                __syncwarp();
                if (L.active)
                    sweep16<S, AFFINE, DL>(L.qc, L.lq4, L.qc2, L.lq42, pad4, prof, A.alpha1, A.gap, A.ext, A.ge,
                                           st > 0, st + 1 < nstrips, bnd, mx);
            }
        } else {
            const int xm4 = (W.xmax + 3) & ~3;
            const int64_t row = (int64_t)xm4 * kWarp;
            const uint4* ring_in = A.ring + A.ring_off[c] + ((s + 1) & 1) * row + lane;
            uint4* ring_out = A.ring + A.ring_off[c] + (s & 1) * row + lane;
            __syncwarp();
            build_item_profile<S, DL>(prof, A, ra, rb, s * S, la, lb, shift, lane);
            __syncwarp();
            const bool has_down = s + 1 < nstrips;
            if (!sweep16_chain<S, AFFINE, DL>(L.qc, L.lq4, L.qc2, L.lq42, xm4, pad4, prof, A.alpha1, A.gap, A.ext,
                                              A.ge, s > 0, has_down, ring_in, ring_out,
                                              s > 0 ? A.progress + pred : nullptr, A.progress + it, A.abort_flag,
                                              A.wait_ns, pre, mx))
                break;
            if (s > 0) {
                // the predecessor's running maximum is final once it has finished
                if (chain_wait(A.progress + pred, kChainDone, A.abort_flag, A.wait_ns) < 0) break;
                mx = __vmaxs2(mx, __ldcg(&A.run_max[(int64_t)pred * kWarp + lane]));
            }
            if (has_down) {
                __stcg(&A.run_max[(int64_t)it * kWarp + lane], mx);
                chain_publish(A.progress + it, kChainDone);
                finished = false;
            }
        }
        if (finished && L.active) store_max16<DL>(A, W, L, mx);
    }
}

template <int S, bool AFFINE, bool MULTI, bool DL>
__global__ void __launch_bounds__(128) score16_kernel(Score16Args A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    void* prof = warp_profile<S, DL>(smem, wib, A.alpha1);
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    uint4* bnd = MULTI ? A.bnd_pool + warp_global * A.bnd_slot + lane : nullptr;
    const int shift = AFFINE ? A.ge : 0;
    const uint32_t pad4 = (uint32_t)A.pad_code * 0x01010101u;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(A.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const WorkItem W = A.grid_strips ? grid_item<S, DL>(A, it) : A.items[it];
        const int sa = W.target, sb = DL ? -1 : W.index;
        const int la = A.strip_len[sa];
        const int lb = sb >= 0 ? A.strip_len[sb] : 0;
        const Lanes16 L = item_lanes<DL>(A, W, lane);
        const uint8_t* ra = A.strip_res + A.strip_off[sa];
        const uint8_t* rb = A.strip_res + A.strip_off[sb >= 0 ? sb : sa];
        const int ls = la > lb ? la : lb;
        const int nstrips = MULTI ? (ls + S - 1) / S : 1;
        uint32_t mx = 0;
        for (int s = 0; s < nstrips; ++s) {
            const int y0 = s * S;
            __syncwarp();
            build_item_profile<S, DL>(prof, A, ra, rb, y0, la, lb, shift, lane);
            __syncwarp();
            if (L.active)
                sweep16<S, AFFINE, DL>(L.qc, L.lq4, L.qc2, L.lq42, pad4, prof, A.alpha1, A.gap, A.ext, A.ge, s > 0,
                                       s + 1 < nstrips, bnd, mx);
        }
        if (L.active) store_max16<DL>(A, W, L, mx);
    }
}

}  // namespace pw
