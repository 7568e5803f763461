// pw_band.cuh -- one pair per warp, its 256-row bands chained across warps.
//
// The 32 lanes of a warp share one (query, target) pair: lane l owns target
// rows [y0 + 8l, y0 + 8l + 8) of a 256-row band and the warp walks the query
// columns as a skewed wavefront (lane l works on column s - l at step s).  The
// values lane l needs from the row above its slice -- computed one step
// earlier by lane l - 1 -- arrive through __shfl_up_sync; lane 0 reads them
// from the boundary row that the band above stored (lane 31's bottom row).
//
// Each band is a queue entry of its own, so the bands of one long pair run on
// different warps at the same time, each a publish period or more behind the
// band above: the band's lane 31 stores its bottom row into the pair's ring
// (two rows, alternating by band parity) and publishes every 32 steps how many
// columns are stored (st.release.gpu, by the storing thread itself); the band
// below polls that count (ld.acquire.gpu, bounded wait) and reads the ring
// with ld.global.cg, 32 columns per coalesced warp load, one block ahead (it
// waits for 64 columns at each 32-step block).  A ring row is rewritten by
// band b + 2 only after band b + 1 has published progress past those columns,
// which it does only after it has read them.  In the queue every band comes after the band
// above it: band-major when there are many pairs, otherwise planned like the
// chained strips (pw_plan.h) so that the bands of a few long pairs pipeline.
//
// DIRS = 0: pair maxima only (the score sweep of long pairs).
// DIRS = 1: the direction sweep of traced pairs: per cell the code of the
// reference's classification (direction, stop flag, candidate flag) and the
// pair's candidate list, exactly as the strip sweep computes them; 4-bit cell
// codes are stored [band][step][lane][8 rows] (warp_layout_offset), one 4-byte
// word per lane and step: a warp stores 128 contiguous bytes.
// DIRS = 2 (linear gap): the same sweep storing each cell's 16-bit H at the
// same positions (16 bytes per lane and step, 512 contiguous bytes a warp) and
// the candidate list; codes are derived from H on read (PairView::code).
// DIRS = 3 (linear gap): the checkpoint sweep of the tile form (pw_tiles.cuh):
// the candidate list as DIRS 1 finds it, no cell codes; instead every band's
// bottom row is kept (in place of the two-row ring) and every lane stores its
// 8 rows' H at the last column of each kTileW-column tile, from which any
// 256 x kTileW tile's codes are recomputed later.
// DIRS = 4 (linear gap): the score sweep of DIRS 0 that also keeps the tile
// form's checkpoints (as DIRS 3) and each tile's maximum H, so that traced
// pairs need no second sweep: only the tiles that reach a pair's threshold
// are recomputed for its candidates (pw_tiles.cuh).
#pragma once
#include "pw_kernels.cuh"
#include "pw_score16.cuh"

namespace pw {

constexpr int kWarpRows = 8;                   // rows per lane
constexpr int kBandRows = kWarpRows * kWarp;   // 256 rows per band
constexpr int kBandLead = 128;                 // planning lead between bands (steps)
constexpr int kTileW = 128;                    // tile form: columns of a checkpointed tile

static_assert(kBandRows == 256 && kWarpRows == 8, "warp_layout_offset (pw_kernels.cuh) assumes 8 x 32 rows");

// Bytes of a pair's 4-bit cell codes in the band layout (8 rows of a lane per
// 4-byte word), or of its 16-bit H values (hstore: four times as many).
__host__ __device__ __forceinline__ int64_t warp_code_bytes(int lq, int lt, bool hstore = false) {
    const int64_t bands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
    const int64_t cells = bands * ((int64_t)lq + kWarp - 1) * kWarp * kWarpRows;
    return hstore ? cells * 2 : cells / 2;
}

// Tile form: ints of a pair's checkpoints -- the bottom rows of its bands but
// the last ((nbands - 1) x lq), then per band and tile the 256 H values of the
// tile's last column (nbands x ntiles x 256; tile ntiles - 1's are not read).
__host__ __device__ __forceinline__ int tile_count(int lq) { return lq > 0 ? (lq + kTileW - 1) / kTileW : 1; }
__host__ __device__ __forceinline__ int64_t tile_col_offset(int lq, int lt) {  // 4-int aligned
    const int64_t bands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
    return ((bands - 1) * (int64_t)lq + 3) & ~(int64_t)3;
}
__host__ __device__ __forceinline__ int64_t tile_checkpoint_ints(int lq, int lt) {  // a multiple of 4
    const int64_t bands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
    return tile_col_offset(lq, lt) + bands * tile_count(lq) * (int64_t)kBandRows;
}

struct BandPair {
    int32_t q, t;        // query / target index (reference orientation)
    int32_t nbands;
    int32_t meta_item;   // DIRS: value for PairMeta.item (the pair's work item in the wave)
    int64_t ring_off;    // int4 offset of the pair's two boundary rows (2 x lq)
    int64_t dir_base;    // DIRS 1, 2: byte offset of the pair's cell codes; 3: int offset of its checkpoints
    int64_t slot;        // DIRS: pair slot (metas, candidates); score sweep: pair_max index
};

struct BandArgs {
    const int4* entries;  // per queue entry: (pair, band, queue index of the band above, 0)
    const BandPair* pairs;
    int n_entries;
    int* counter;
    int4* ring;
    int* progress;        // per entry: columns of the bottom row stored (kChainDone when finished)
    int* run_max;         // per entry: running maximum of the pair's bands so far
    int* abort_flag;
    float* max_out;       // score sweep: pair maxima, indexed by BandPair.slot
    int* ck;              // DIRS 3, 4: checkpoints (tile_checkpoint_ints per pair, at BandPair.dir_base);
                          // DIRS 4: tile maxima (bands x tiles per pair, at BandPair.ring_off)
    unsigned long long wait_ns;  // bound of one wait for the band above
};

// Byte k of w as a signed int: one prmt whose selector copies byte k into the
// low byte and replicates its sign bit over the three others (PTX prmt.b32,
// default mode: the msb of a selector nibble replicates the byte's sign).
template <int K>
__device__ __forceinline__ int sbyte(uint32_t w) {
    constexpr uint32_t sel = K | ((8u | K) << 4) | ((8u | K) << 8) | ((8u | K) << 12);
    int d;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(d) : "r"(w), "n"(sel));
    return d;
}

// Score of row r (0..7) of a lane's profile word pair (r a constant once the
// row loop is unrolled).
__device__ __forceinline__ int prof_score(uint2 pw, int r) {
    switch (r) {
        case 0: return sbyte<0>(pw.x);
        case 1: return sbyte<1>(pw.x);
        case 2: return sbyte<2>(pw.x);
        case 3: return sbyte<3>(pw.x);
        case 4: return sbyte<0>(pw.y);
        case 5: return sbyte<1>(pw.y);
        case 6: return sbyte<2>(pw.y);
        default: return sbyte<3>(pw.y);
    }
}

template <bool AFFINE, int DIRS>
__global__ void __launch_bounds__(128, AFFINE ? 5 : 8) band_kernel(KernelArgs A, BandArgs B) {
    static_assert(DIRS < 2 || !AFFINE, "H store and tile form: linear gap only");
    constexpr bool MAXIMA = DIRS == 0 || DIRS == 4;  // pair maxima, no trace
    constexpr bool CKPT = DIRS == 3 || DIRS == 4;    // tile-form checkpoints
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int alpha1 = A.P.alpha + 1;
    const int prof_bytes = ((kWarp * alpha1 * kWarpRows) + 15) & ~15;
    uint2* prof = (uint2*)(smem + wib * prof_bytes);  // [lane][alpha1] -> 8 int8 scores of that lane's rows
    const int gap = A.P.gap_i, ext = A.P.ext_i, ge = A.P.ge_i;
    const int neg = kNeg;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(B.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= B.n_entries) break;
        const int4 en = B.entries[it];
        const BandPair BP = B.pairs[en.x];
        const int band = en.y, pred = en.z;
        const int q = BP.q, t = BP.t;
        const int lq = A.q.len[q], lt = A.t.len[t];
        const int nbands = BP.nbands;
        int thr = 0;
        Cand* cand = nullptr;
        int cap = 0;
        int* ncand = nullptr;
        uint8_t* codes = nullptr;
        if constexpr (!MAXIMA) {
            // threshold of the pair (default_main.cu:609, SmithWatermanCuda.py:269-275)
            const float maxf = A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip];
            const int mn = lq < lt ? lq : lt;
            const float pos = (float)(A.P.highest * (double)mn * A.P.filter_factor);
            const float thf = fmaxf(__fmul_rn(A.P.lower_limit, maxf), pos);
            thr = (int)fminf(fmaxf(ceilf(thf), -1.0e9f), 1.0e9f);
            if (band == 0 && lane == 0) {
                PairMeta& pm = A.metas[BP.slot];
                pm.query = q;
                pm.target = t;
                pm.item = BP.meta_item;
                pm.lane = 0;
                pm.thr_f = thf;
                pm.thr_i = thr;
                pm.max_f = maxf;
            }
            cand = A.cands + A.cand_base[BP.slot];
            cap = A.cand_cap[BP.slot];
            ncand = A.n_cand + BP.slot;
            if constexpr (DIRS != 3) codes = A.codes + BP.dir_base;
        }
        const uint8_t* qg = A.q.codes + A.q.code_off[q];
        const uint8_t* tres = A.t.codes + A.t.code_off[t];
        const int64_t nsteps = (int64_t)lq + kWarp - 1;
        const int yb = band * kBandRows;
        __syncwarp();
        for (int idx = lane; idx < kWarp * alpha1; idx += kWarp) {
            const int ll = idx / alpha1, a = idx % alpha1;
            uint32_t w0 = 0, w1 = 0;
#pragma unroll
            for (int r = 0; r < kWarpRows; ++r) {
                const int y = yb + ll * kWarpRows + r;
                const int8_t sc = y < lt ? A.cmat_i8[a * A.P.dim + tres[y]] : (int8_t)-128;
                if (r < 4)
                    w0 |= (uint32_t)(uint8_t)sc << (8 * r);
                else
                    w1 |= (uint32_t)(uint8_t)sc << (8 * (r - 4));
            }
            prof[idx] = make_uint2(w0, w1);
        }
        __syncwarp();
        const bool has_up = band > 0;
        const bool store_bnd = band + 1 < nbands;
        const int4* ring_in = nullptr;
        int4* ring_out = nullptr;
        const int* ck_in = nullptr;  // DIRS 3, 4: the bottom row of the band above, this band's, its tile columns
        int* ck_out = nullptr;
        int* ck_col = nullptr;
        int* tmax = nullptr;  // DIRS 4: this band's tile maxima
        if constexpr (CKPT) {
            int* ckp = B.ck + BP.dir_base;
            if constexpr (DIRS == 4) tmax = B.ck + BP.ring_off + (int64_t)band * tile_count(lq);
            if (has_up) ck_in = ckp + (int64_t)(band - 1) * lq;
            if (store_bnd) ck_out = ckp + (int64_t)band * lq;
            ck_col = ckp + tile_col_offset(lq, lt) + ((int64_t)band * tile_count(lq)) * kBandRows + lane * kWarpRows;
        } else {
            ring_in = B.ring + BP.ring_off + (int64_t)((band + 1) & 1) * lq;
            ring_out = B.ring + BP.ring_off + (int64_t)(band & 1) * lq;
        }
        const int* prog_in = B.progress + pred;
        int* prog_out = B.progress + it;
        const int ymine = yb + lane * kWarpRows;
        const bool ypos = ymine > 0;       // this lane's first row is not row 0
        const int rows_left = lt - ymine;  // rows r < rows_left of this lane lie inside the target
        int Hl[kWarpRows], Ml[kWarpRows], Jl[kWarpRows], Bl[kWarpRows];
#pragma unroll
        for (int r = 0; r < kWarpRows; ++r) {
            Hl[r] = 0;
            Ml[r] = 0;
            Jl[r] = neg;
            Bl[r] = 0;
        }
        int up_h = 0, up_m = 0, up_i = neg, up_b = 0;
        int dg_h = 0, dg_m = 0, dg_b = 0;
        int bt_h = 0, bt_m = 0, bt_i = neg, bt_b = 0;
        int mx = 0;
        int tm = 0;  // DIRS 4: the lane's maximum in its current tile
        int avail = 0;
        bool ok = true;
        // the row above, 32 columns at a time: lane k holds column 32j + k of
        // the current block (cur) and of the next one (nxt), loaded with one
        // coalesced read a block ahead; lane 0 takes column s by a shuffle
        // (linear gap: the H values only)
        int4 cur = make_int4(0, 0, 0, 0), nxt = make_int4(0, 0, 0, 0);
        auto fetch = [&](int64_t c) -> int4 {
            if (c >= lq) return make_int4(0, 0, 0, 0);
            if constexpr (CKPT) return make_int4(__ldcg(ck_in + c), 0, 0, 0);
            if constexpr (AFFINE) return __ldcg(&ring_in[c]);
            return make_int4(__ldcg((const int*)&ring_in[c]), 0, 0, 0);
        };
        for (int64_t s = 0; s < nsteps; ++s) {
            if (has_up && (s & 31) == 0) {
                // this block and the next one must be stored by the band above
                const int need = (int)(s + 64 < (int64_t)lq ? s + 64 : (int64_t)lq);
                if (avail < need) {
                    avail = chain_wait(prog_in, need, B.abort_flag, B.wait_ns);
                    if (avail < 0) {
                        ok = false;
                        break;
                    }
                }
                cur = s == 0 ? fetch(s + lane) : nxt;
                nxt = fetch(s + 32 + lane);
            }
            const int x = (int)s - lane;
            const bool active = x >= 0 && x < lq;
            int rh = 0, rm = 0, ri = neg, rb = 0;
            int4 above = make_int4(0, 0, 0, 0);
            if (has_up) {
                above.x = __shfl_sync(0xffffffffu, cur.x, (int)(s & 31));
                if constexpr (AFFINE) {
                    above.y = __shfl_sync(0xffffffffu, cur.y, (int)(s & 31));
                    above.z = __shfl_sync(0xffffffffu, cur.z, (int)(s & 31));
                }
            }
            if constexpr (AFFINE) {
                rm = __shfl_up_sync(0xffffffffu, bt_m, 1);
                ri = __shfl_up_sync(0xffffffffu, bt_i, 1);
                rb = __shfl_up_sync(0xffffffffu, bt_b, 1);
            } else {
                rh = __shfl_up_sync(0xffffffffu, bt_h, 1);
            }
            if (lane == 0) {
                if (has_up && active) {
                    const int4 v = above;
                    rh = v.x;
                    rm = v.x;
                    ri = v.y;
                    rb = v.z;
                } else {
                    rh = 0;
                    rm = 0;
                    ri = neg;
                    rb = 0;
                }
            }
            dg_h = x == 0 ? 0 : up_h;
            dg_m = x == 0 ? 0 : up_m;
            dg_b = x == 0 ? 0 : up_b;
            up_h = rh;
            up_m = rm;
            up_i = ri;
            up_b = rb;
            if (active) {
                const int a = __ldg(qg + x);
                const uint2 pw = prof[lane * alpha1 + a];
                const bool xin = x > 0;
                uint32_t w0 = 0;  // the lane's 8 rows as 4-bit codes
                if constexpr (!AFFINE) {
                    int up = up_h, diag = dg_h;
                    int Hold[kWarpRows];  // the left neighbours (previous column), for the candidate test
#pragma unroll
                    for (int r = 0; r < kWarpRows; ++r) Hold[r] = Hl[r];
                    // the stop flag needs a cell inside the matrix: x > 0 and y > 0
                    const bool stop_ok0 = xin && ypos, stop_ok = xin;
#pragma unroll
                    for (int r = 0; r < kWarpRows; ++r) {
                        const int sc = prof_score(pw, r);
                        const int left = Hl[r];
                        int h = addmax(left, gap, diag + sc);
                        h = addmax_relu(up, gap, h);
                        if constexpr (DIRS == 1) {
                            // the reference's classification (LEFT > UP > UL, NO at
                            // 0), shifted into the row's nibble; the stop flag on a
                            // UL cell inside the matrix whose diagonal is 0
                            const uint32_t sh = 4 * r;
                            uint32_t code = h == left + gap ? (kLeft << sh) : (h == up + gap ? (kUp << sh) : (kUL << sh));
                            const bool stop = (r > 0 ? stop_ok : stop_ok0) && diag == 0 && code == (kUL << sh);
                            code = stop ? code | (kStopFlag << sh) : code;
                            w0 |= h > 0 ? code : 0u;
                        }
                        diag = left;
                        Hl[r] = h;
                        up = h;
                    }
                    if constexpr (DIRS == 4)
                        tm = max3(tm, max3(Hl[0], Hl[1], Hl[2]), max3(Hl[3], Hl[4], max3(Hl[5], Hl[6], Hl[7])));
                    else if constexpr (DIRS == 0)
                        mx = max3(mx, max3(Hl[0], Hl[1], Hl[2]), max3(Hl[3], Hl[4], max3(Hl[5], Hl[6], Hl[7])));
                    if constexpr (!MAXIMA) {
                        // candidates: UL cells inside the matrix at or above the
                        // threshold -- rare, so one test of the step's maximum
                        const int smax = max(max3(Hl[0], Hl[1], Hl[2]), max3(Hl[3], Hl[4], max3(Hl[5], Hl[6], Hl[7])));
                        if (smax >= thr) {
#pragma unroll
                            for (int r = 0; r < kWarpRows; ++r) {
                                const int h = Hl[r], upv = r > 0 ? Hl[r - 1] : up_h;
                                if (h < thr || h <= 0 || r >= rows_left || h == Hold[r] + gap || h == upv + gap)
                                    continue;
                                if constexpr (DIRS == 1) w0 |= kCand << (4 * r);
                                const int k = atomicAdd(ncand, 1);
                                if (k < cap) {
                                    Cand cc;
                                    cc.x = x;
                                    cc.y = ymine + r;
                                    cc.score_i = h;
                                    cc.score_f = (float)h;
                                    cand[k] = cc;
                                }
                            }
                        }
                    }
                    bt_h = up;
                    if constexpr (DIRS == 4) {
                        // the lane's maximum over a tile's columns, into the tile's maximum
                        if (((x + 1) & (kTileW - 1)) == 0 || x + 1 == lq) {
                            atomicMax(tmax + x / kTileW, tm);
                            mx = max(mx, tm);
                            tm = 0;
                        }
                    }
                    if constexpr (CKPT) {
                        // the lane's rows at the last column of a tile: the next tile's left boundary
                        if (((x + 1) & (kTileW - 1)) == 0 && x + 1 < lq) {
                            int4* d = (int4*)(ck_col + (int64_t)((x + 1) / kTileW) * kBandRows);
                            __stcg(d, make_int4(Hl[0], Hl[1], Hl[2], Hl[3]));
                            __stcg(d + 1, make_int4(Hl[4], Hl[5], Hl[6], Hl[7]));
                        }
                    }
                    if constexpr (DIRS == 2) {
                        uint4 hv;
                        hv.x = __byte_perm(Hl[0], Hl[1], 0x5410);
                        hv.y = __byte_perm(Hl[2], Hl[3], 0x5410);
                        hv.z = __byte_perm(Hl[4], Hl[5], 0x5410);
                        hv.w = __byte_perm(Hl[6], Hl[7], 0x5410);
                        *(uint4*)(codes + ((band * nsteps + s) * kWarp + lane) * kWarpRows * 2) = hv;
                    }
                } else {
                    int mup = up_m, iup = up_i, bdiag = dg_b, mdiag = dg_m;
#pragma unroll
                    for (int r = 0; r < kWarpRows; ++r) {
                        const int sc = prof_score(pw, r);
                        const int m = addmax_relu(bdiag, sc, neg);
                        const int i = addmax(iup, ext, mup + ge);
                        const int jj = addmax(Jl[r], ext, Ml[r] + ge);
                        const int b = max3(m, i, jj);
                        if constexpr (!MAXIMA) {
                            uint32_t code = b == m ? kUL : (b == i ? kUp : kLeft);
                            code = b > 0 ? code : kNo;
                            const bool main_src = code == kUL;
                            const bool stop = main_src && xin && (r > 0 || ypos) && mdiag == 0;
                            code |= stop ? kStopFlag : 0u;
                            w0 |= code << (4 * r);
                        } else {
                            mx = max(mx, b);
                        }
                        bdiag = Bl[r];
                        mdiag = Ml[r];
                        Ml[r] = m;
                        Jl[r] = jj;
                        Bl[r] = b;
                        mup = m;
                        iup = i;
                    }
                    bt_m = mup;
                    bt_i = iup;
                    bt_b = Bl[kWarpRows - 1];
                    if constexpr (!MAXIMA) {
                        // candidates: MAIN-source cells (b == m > 0) inside the
                        // matrix with m at or above the threshold -- rare, so one
                        // test of the step's maximum of m
                        const int smax = max(max3(Ml[0], Ml[1], Ml[2]), max3(Ml[3], Ml[4], max3(Ml[5], Ml[6], Ml[7])));
                        if (smax >= thr) {
#pragma unroll
                            for (int r = 0; r < kWarpRows; ++r) {
                                const int m = Ml[r];
                                if (m < thr || Bl[r] != m || m <= 0 || r >= rows_left) continue;
                                w0 |= kCand << (4 * r);
                                const int k = atomicAdd(ncand, 1);
                                if (k < cap) {
                                    Cand cc;
                                    cc.x = x;
                                    cc.y = ymine + r;
                                    cc.score_i = m;
                                    cc.score_f = (float)m;
                                    cand[k] = cc;
                                }
                            }
                        }
                    }
                }
                if constexpr (DIRS == 1)
                    *(uint32_t*)(codes + ((band * nsteps + s) * kWarp + lane) * kWarpRows / 2) = w0;
                if (lane == kWarp - 1 && store_bnd) {
                    if constexpr (CKPT)
                        __stcg(ck_out + x, bt_h);
                    else
                        __stcg(&ring_out[x], make_int4(AFFINE ? bt_m : bt_h, bt_i, bt_b, 0));
                }
            } else {
                // not started (x < 0): hand the left-boundary values down
                bt_h = 0;
                bt_m = 0;
                bt_i = neg;
                bt_b = 0;
            }
            // lane 31 stored columns 0 .. s - 31 of the bottom row
            if (store_bnd && lane == kWarp - 1 && ((s + 1) & 31) == 0 && s >= kWarp - 1)
                st_release_gpu(prog_out, (int)(s - (kWarp - 2)));
        }
        if (!ok) break;
        if (store_bnd && lane == kWarp - 1) st_release_gpu(prog_out, lq);
        // pair maximum (score sweep) / candidate count (direction sweep)
        if constexpr (MAXIMA) mx = __reduce_max_sync(0xffffffffu, mx);
        if (has_up) {
            // the band above has finished: its running maximum and its candidates are final
            if (chain_wait(prog_in, kChainDone, B.abort_flag, B.wait_ns) < 0) break;
            if constexpr (MAXIMA) mx = max(mx, __ldcg(&B.run_max[pred]));
        }
        if (store_bnd) {
            if constexpr (MAXIMA)
                if (lane == 0) __stcg(&B.run_max[it], mx);
            chain_publish(prog_out, kChainDone);
        } else if (lane == 0) {
            if constexpr (!MAXIMA)
                A.metas[BP.slot].n_cand = atomicAdd(ncand, 0);
            else
                B.max_out[BP.slot] = (float)mx;
        }
    }
}

}  // namespace pw
