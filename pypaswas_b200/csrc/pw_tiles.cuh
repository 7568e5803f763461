// pw_tiles.cuh -- the tile form of the long-pair traceback (linear gap).
//
// The band direction sweep of a long pair stores a 4-bit code for every cell
// (a 30 kb x 30 kb pair: 450 MB), and the walks then follow their paths one
// dependent global load a step.  The tile form stores no cell codes: the
// checkpoint sweep (band_kernel<false, 3>) finds the candidates and keeps
// every band's bottom row and, per band, the H column at every kTileW-th
// column.  From those, one warp recomputes the codes of any 256 x kTileW tile
// into shared memory -- the same codes, bit for bit, as the direction sweep
// (same recurrence, same boundary values, same classification) -- and the
// covering chains, the walks and the column operations read them there.
//
// One warp per pair (collect, walk) or per hit (operations); every lane runs
// the same path in step, so a tile miss is recomputed by the whole warp.  The
// walk follows up to 32 steps by the codes alone and then checks the cells'
// marks (one load per lane): a walk never revisits its own cells, so the
// first marked cell of the batch is where the reference's walk stops.  Marks
// are one bit per cell, bit y * lq + x of the pair's plane.
#pragma once
#include "pw_band.cuh"

namespace pw {

// A traced long pair in the tile form.
struct TilePair {
    int32_t q, t;     // query / target index (reference orientation)
    int32_t slot;     // pair slot of the wave (metas, candidates, starting points)
    int32_t pad;
    int64_t ck;       // int offset of the pair's checkpoints (tile_checkpoint_ints)
    int64_t marks;    // uint32 offset of the pair's mark plane
    int64_t tm;       // checkpoints of the score sweep (band_kernel<false, 4>): int offset of the tile maxima
    int64_t scratch;  // byte offset of the pair's walk scratch (lq + lt bytes)
};

// Where a tile sweep puts the candidates it finds (the pair's slot).
struct CandSink {
    Cand* cand;
    int cap;
    int* n;
};

struct TileArgs {
    const TilePair* pairs;
    int n_pairs;
    const int* ck;
    uint32_t* marks;
    const int32_t* slot_tile;  // per pair slot: index into pairs, -1 for the other pairs
    // the walk writes its hits' column operations itself when ops is set:
    // reserved from ops_total in ops (offsets relative to ops, the host adds
    // the base), spelled in walk order into the pair's scratch first
    char* scratch;
    char* ops;
    unsigned long long* ops_total;
    unsigned long long* ops_bound;  // tile_collect_kernel: sum of starts x (lq + lt) over the pairs
};

// The cached tile holds H, int32, column-major with a one-cell border:
// column c = x - x0 + 1 (c = 0: the left boundary, column x0 - 1), row
// r = y - yb + 1 (r = 0: the row above the band); kTileRows values a column.
constexpr int kTileRows = kBandRows + 1;
constexpr int kTileCells = (kTileW + 1) * kTileRows;

__host__ __device__ __forceinline__ int tile_smem_bytes(int alpha1) {
    return ((kTileCells * 4 + 15) & ~15) + ((kWarp * alpha1 * kWarpRows + 15) & ~15) + kTileW;
}

// One warp's view of a pair in the tile form, with its one cached tile.
struct TileView {
    const int* ckp;         // the pair's checkpoints
    int64_t col_off;        // tile columns' offset in ckp
    int ntiles, lq, lt, thr, gap, alpha1, dim;
    const uint8_t* qg;      // query codes (compact)
    const uint8_t* tres;    // target residues (matrix index)
    const int8_t* cmat;
    int* hs;                // shared: the cached tile's H with its border
    uint2* prof;            // shared: [lane][alpha1] scores of the lane's 8 rows in the cached band
    uint8_t* qc;            // shared: the query codes of the tile's columns
    int band, tile, prof_band, x0, yb;
    int xmax_c, ymax_c;     // the cached tile's computed extent (its cells up to these coordinates)
    uint32_t* mark_plane;   // the pair's mark bits

    __device__ __forceinline__ uint32_t* mark_word(int x, int y) const {
        return mark_plane + (((int64_t)y * lq + x) >> 5);
    }
    __device__ __forceinline__ uint32_t mark_bit(int x, int y) const {
        return 1u << ((((int64_t)y * lq + x)) & 31);
    }
    __device__ __forceinline__ bool marked(int x, int y) const { return (__ldcg(mark_word(x, y)) & mark_bit(x, y)) != 0; }
    __device__ __forceinline__ void mark(int x, int y) const { atomicOr(mark_word(x, y), mark_bit(x, y)); }
    __device__ __forceinline__ void unmark(int x, int y) const { atomicAnd(mark_word(x, y), ~mark_bit(x, y)); }

    __device__ void load(int b, int j, int xneed, int yneed) {
        load_h<false>(b, j, CandSink{nullptr, 0, nullptr}, xneed, yneed);
    }

    // Recomputes the H values of tile (band b, tile j) and its border, as far
    // as cell (xneed, yneed): the columns up to xneed and the lanes up to
    // yneed's (a walk only moves up and left, so it needs no more of the
    // tile); every lane of the warp calls it.  CANDS: the whole tile, and its
    // candidates into the sink, with the band sweep's test (UL cells inside
    // the matrix at or above the threshold).
    template <bool CANDS>
    __device__ void load_h(int b, int j, CandSink sink, int xneed, int yneed) {
        const int lane = threadIdx.x & 31;
        __syncwarp();
        yb = b * kBandRows;
        x0 = j * kTileW;
        if (prof_band != b) {
            for (int idx = lane; idx < kWarp * alpha1; idx += kWarp) {
                const int ll = idx / alpha1, a = idx % alpha1;
                uint32_t w0 = 0, w1 = 0;
#pragma unroll
                for (int r = 0; r < kWarpRows; ++r) {
                    const int y = yb + ll * kWarpRows + r;
                    const int8_t sc = y < lt ? cmat[a * dim + tres[y]] : (int8_t)-128;
                    if (r < 4)
                        w0 |= (uint32_t)(uint8_t)sc << (8 * r);
                    else
                        w1 |= (uint32_t)(uint8_t)sc << (8 * (r - 4));
                }
                prof[idx] = make_uint2(w0, w1);
            }
            prof_band = b;
        }
        const int ncol = min(min(kTileW, lq - x0), xneed - x0 + 1);
        const int lanes_need = min(kWarp - 1, (yneed - yb) >> 3);
        // border row (r = 0): the row above, columns x0 - 1 .. x0 + ncol - 1; 0 above band 0 and left of column 0
        for (int k = lane; k <= ncol; k += kWarp) {
            const int xx = x0 - 1 + k;
            hs[k * kTileRows] = (b > 0 && xx >= 0) ? __ldcg(ckp + (int64_t)(b - 1) * lq + xx) : 0;
        }
        for (int k = lane; k < ncol; k += kWarp) qc[k] = qg[x0 + k];
        // border column (c = 0): the checkpointed last column of tile j - 1
        int Hl[kWarpRows];
        if (j > 0) {
            const int4* src = (const int4*)(ckp + col_off + ((int64_t)b * ntiles + j) * kBandRows + lane * kWarpRows);
            const int4 v0 = __ldcg(src), v1 = __ldcg(src + 1);
            Hl[0] = v0.x; Hl[1] = v0.y; Hl[2] = v0.z; Hl[3] = v0.w;
            Hl[4] = v1.x; Hl[5] = v1.y; Hl[6] = v1.z; Hl[7] = v1.w;
        } else {
#pragma unroll
            for (int r = 0; r < kWarpRows; ++r) Hl[r] = 0;
        }
#pragma unroll
        for (int r = 0; r < kWarpRows; ++r) hs[1 + lane * kWarpRows + r] = Hl[r];
        __syncwarp();
        // the skewed wavefront of band_kernel over the tile's columns; a lane
        // that has not started hands down its left boundary's bottom value
        const int ymine = yb + lane * kWarpRows;
        const int rows_left = lt - ymine;
        int bt_h = Hl[kWarpRows - 1];
        int up_h = lane == 0 ? hs[0] : 0;  // lane 0: the corner, its first cell's diagonal
        const int nsteps = ncol + lanes_need;
        // the shared-memory reads of a step (its scores; lane 0: the row
        // above) are issued one step ahead, off the recurrence's path
        auto fetch_pw = [&](int c) -> uint2 {
            return (c >= 0 && c < ncol) ? prof[lane * alpha1 + qc[c]] : make_uint2(0u, 0u);
        };
        auto fetch_top = [&](int c) -> int { return (b > 0 && c >= 0 && c < ncol) ? hs[(c + 1) * kTileRows] : 0; };
        uint2 pw_n = fetch_pw(-lane);
        int top_n = lane == 0 ? fetch_top(0) : 0;
        for (int s = 0; s < nsteps; ++s) {
            const int xl = s - lane;
            const int x = x0 + xl;
            const bool active = xl >= 0 && xl < ncol;
            const uint2 pw = pw_n;
            const int top = top_n;
            pw_n = fetch_pw(xl + 1);
            if (lane == 0) top_n = fetch_top(xl + 1);
            int rh = __shfl_up_sync(0xffffffffu, bt_h, 1);
            if (lane == 0) rh = top;
            const int dg_h = x == 0 ? 0 : up_h;
            up_h = rh;
            if (active) {
                int up = up_h, diag = dg_h;
                int Hold[kWarpRows];
                if constexpr (CANDS) {
#pragma unroll
                    for (int r = 0; r < kWarpRows; ++r) Hold[r] = Hl[r];
                }
#pragma unroll
                for (int r = 0; r < kWarpRows; ++r) {
                    const int sc = prof_score(pw, r);
                    const int left = Hl[r];
                    int h = addmax(left, gap, diag + sc);
                    h = addmax_relu(up, gap, h);
                    diag = left;
                    Hl[r] = h;
                    up = h;
                }
                if constexpr (CANDS) {
                    const int smax = max(max3(Hl[0], Hl[1], Hl[2]), max3(Hl[3], Hl[4], max3(Hl[5], Hl[6], Hl[7])));
                    if (smax >= thr) {
#pragma unroll
                        for (int r = 0; r < kWarpRows; ++r) {
                            const int h = Hl[r], upv = r > 0 ? Hl[r - 1] : up_h;
                            if (h < thr || h <= 0 || r >= rows_left || h == Hold[r] + gap || h == upv + gap) continue;
                            const int k = atomicAdd(sink.n, 1);
                            if (k < sink.cap) {
                                Cand cc;
                                cc.x = x;
                                cc.y = ymine + r;
                                cc.score_i = h;
                                cc.score_f = (float)h;
                                sink.cand[k] = cc;
                            }
                        }
                    }
                }
                bt_h = up;
                int* dst = hs + (xl + 1) * kTileRows + 1 + lane * kWarpRows;
#pragma unroll
                for (int r = 0; r < kWarpRows; ++r) dst[r] = Hl[r];
            } else if (xl < 0) {
                bt_h = Hl[kWarpRows - 1];
            }
        }
        band = b;
        tile = j;
        xmax_c = x0 + ncol - 1;
        ymax_c = yb + (lanes_need + 1) * kWarpRows - 1;
        __syncwarp();
    }

    // The 4-bit code of cell (x, y), derived from the cached H values exactly
    // as the direction sweep classifies it (LEFT when the left neighbour plus
    // the gap reaches H, else UP, else UL; NO where H is 0; the stop flag on a
    // UL cell inside the matrix with a zero diagonal neighbour, the candidate
    // flag on a UL cell at or above the pair's threshold); kNo outside the
    // matrix.  Uniform across the warp.
    __device__ __forceinline__ uint32_t code(int x, int y) {
        if (x < 0 || y < 0 || x >= lq || y >= lt) return kNo;
        const int b = y >> 8, j = x / kTileW;
        if (b != band || j != tile || x > xmax_c || y > ymax_c) {
            // a miss, or a cell past the cached extent (the covering chains of
            // several candidates reuse a tile): recompute far enough for both
            const bool same = b == band && j == tile;
            load(b, j, same ? max(x, xmax_c) : x, same ? max(y, ymax_c) : y);
        }
        const int* c = hs + (x - x0 + 1) * kTileRows + (y - yb + 1);
        const int h = c[0], l = c[-kTileRows], u = c[-1], d = c[-kTileRows - 1];
        if (h <= 0) return kNo;
        if (h == l + gap) return kLeft;
        if (h == u + gap) return kUp;
        uint32_t cd = kUL;
        if (x > 0 && y > 0 && d == 0) cd |= kStopFlag;
        if (h >= thr) cd |= kCand;
        return cd;
    }
};

__device__ __forceinline__ TileView tile_view(const KernelArgs& A, const TileArgs& T, const TilePair& tp, int thr,
                                              unsigned char* smem) {
    TileView v;
    v.lq = A.q.len[tp.q];
    v.lt = A.t.len[tp.t];
    v.ckp = T.ck + tp.ck;
    v.col_off = tile_col_offset(v.lq, v.lt);
    v.ntiles = tile_count(v.lq);
    v.thr = thr;
    v.gap = A.P.gap_i;
    v.alpha1 = A.P.alpha + 1;
    v.dim = A.P.dim;
    v.qg = A.q.codes + A.q.code_off[tp.q];
    v.tres = A.t.codes + A.t.code_off[tp.t];
    v.cmat = A.cmat_i8;
    v.hs = (int*)smem;
    v.prof = (uint2*)(smem + ((kTileCells * 4 + 15) & ~15));
    v.qc = (uint8_t*)v.prof + ((kWarp * v.alpha1 * kWarpRows + 15) & ~15);
    v.x0 = 0;
    v.yb = 0;
    v.band = -1;
    v.xmax_c = -1;
    v.ymax_c = -1;
    v.tile = -1;
    v.prof_band = -1;
    v.mark_plane = T.marks + tp.marks;
    return v;
}

// collect_kernel for the pairs of the tile form: the covering chains, the
// uncovered candidates in walk order, their count.  One warp per pair.
__global__ void __launch_bounds__(32) tile_collect_kernel(KernelArgs A, TraceArgs TA, TileArgs T) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x;
    const TilePair tp = T.pairs[blockIdx.x];
    const int p = tp.slot;
    const PairMeta pm = TA.metas[p];
    Cand* cl = TA.cands + TA.cand_base[p];
    const int n = pm.n_cand;
    TileView v = tile_view(A, T, tp, pm.thr_i, smem);
    // marking chains: the nearest candidate up a candidate's chain is covered
    // (a lone candidate has no other candidate to cover)
    for (int k = 0; k < n && n > 1; ++k) {
        int x = cl[k].x - 1, y = cl[k].y - 1;
        while (x >= 0 && y >= 0) {
            const uint32_t cd = v.code(x, y);
            const int d = cd & 3;
            if (cd & kCand) {
                if (lane == 0) v.mark(x, y);  // covered
                break;
            }
            if (d == kNo) break;
            if (d == kUL) {
                --x;
                --y;
            } else if (d == kUp) {
                --y;
            } else {
                --x;
            }
        }
    }
    __syncwarp();
    if (lane != 0) return;
    // the uncovered candidates (covered marks cleared again), ordered for the
    // walk: ascending score, then emission order (a stable sort)
    int m = 0;
    for (int k = 0; k < n; ++k) {
        const Cand cc = cl[k];
        if (v.marked(cc.x, cc.y))
            v.unmark(cc.x, cc.y);
        else
            cl[m++] = cc;
    }
    for (int k = 1; k < m; ++k) {
        const Cand key = cl[k];
        const uint64_t ek = emission_key(key.x, key.y);
        int j = k - 1;
        while (j >= 0) {
            const Cand o = cl[j];
            const bool after = o.score_f > key.score_f || (o.score_f == key.score_f && emission_key(o.x, o.y) > ek);
            if (!after) break;
            cl[j + 1] = o;
            --j;
        }
        cl[j + 1] = key;
    }
    TA.n_starts[p] = m;
    if (T.ops_bound) atomicAdd(T.ops_bound, (unsigned long long)m * (unsigned long long)(v.lq + v.lt));
}

// walk_kernel for the pairs of the tile form.  One warp per pair; the walks
// of a pair run in order, as the reference's (their marks stop later walks).
__global__ void __launch_bounds__(32) tile_walk_kernel(KernelArgs A, TraceArgs TA, TileArgs T) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x;
    const TilePair tp = T.pairs[blockIdx.x];
    const int p = tp.slot;
    const PairMeta pm = TA.metas[p];
    const Cand* cl = TA.cands + TA.cand_base[p];
    const int m = TA.n_starts[p];
    TileView v = tile_view(A, T, tp, pm.thr_i, smem);
    const uint8_t* qs = TA.q.raw + TA.q.raw_off[pm.query];
    const uint8_t* ts = TA.t.raw + TA.t.raw_off[pm.target];
    const bool same_id = TA.q.key[pm.query] == TA.t.key[pm.target];
    char* scr = T.ops ? T.scratch + tp.scratch : nullptr;
    for (int k = 0; k < m; ++k) {
        if (TA.allowed && !TA.allowed[TA.start_off[p] + k]) continue;
        const Cand st = cl[k];
        int x = st.x, y = st.y;
        // walk_direction of the starting cell
        int dir;
        {
            const bool mk = v.marked(x, y);
            const uint32_t cd = v.code(x, y);
            const int d = cd & 3;
            dir = mk ? kInAlignment : ((d == kUL && (cd & kStopFlag)) ? kStopDir : d);
        }
        bool show = true;
        if (same_id) {  // SmithWaterman.py:752-755
            dir = kStopDir;
            show = false;
        }
        if ((double)st.score_f < A.P.host_minimum) show = false;  // :758-759
        int s_start = x + 1, t_start = y + 1, ncols = 0, mt = 0, mm = 0;
        bool go = show && x >= 0 && y >= 0 && dir != kStopDir && dir != 32;  // :761
        while (go) {
            // up to 32 steps by the codes alone; lane i keeps step i
            int sx = 0, sy = 0, sd = kNo, n = 0;
            bool end = false;
            int cx = x, cy = y;
            for (int i = 0; i < kWarp; ++i) {
                if (cx < 0 || cy < 0) {
                    end = true;
                    break;
                }
                const uint32_t cd = v.code(cx, cy);
                const int d = cd & 3;
                const int dd = (d == kUL && (cd & kStopFlag)) ? kStopDir : d;
                if (lane == i) {
                    sx = cx;
                    sy = cy;
                    sd = dd;
                }
                ++n;
                if (dd == kStopDir || dd == kNo) {  // the walk ends at this cell
                    end = true;
                    break;
                }
                if (dd == kUL) {
                    --cx;
                    --cy;
                } else if (dd == kLeft) {
                    --cx;
                } else {
                    --cy;
                }
            }
            // the first marked cell of the batch ends the walk there (IN_ALIGNMENT)
            const unsigned hit_mark = __ballot_sync(0xffffffffu, lane < n && v.marked(sx, sy));
            const int f = hit_mark ? __ffs(hit_mark) - 1 : n;
            if (lane < (hit_mark ? f + 1 : n)) v.mark(sx, sy);
            const bool proc = lane < f;
            const bool dg = proc && (sd == kUL || sd == kStopDir);
            if (T.ops) {  // the batch's columns in walk order (a prefix of the lanes)
                const bool col = proc && sd != kNo;
                if (col) scr[ncols + lane] = dg ? 'M' : (sd == kLeft ? 'I' : 'D');
            }
            const unsigned n_dg = __popc(__ballot_sync(0xffffffffu, dg));
            const unsigned n_mt = __popc(__ballot_sync(0xffffffffu, dg && same_residue(ts[sy], qs[sx])));
            const unsigned n_l = __popc(__ballot_sync(0xffffffffu, proc && sd == kLeft));
            const unsigned n_u = __popc(__ballot_sync(0xffffffffu, proc && sd == kUp));
            mt += (int)n_mt;
            mm += (int)(n_dg - n_mt);
            ncols += (int)(n_dg + n_l + n_u);
            s_start -= (int)(n_dg + n_l);
            t_start -= (int)(n_dg + n_u);
            __syncwarp();
            if (hit_mark) {
                show = false;
                go = false;
            } else if (end) {
                go = false;
            } else {
                x = cx;
                y = cy;
            }
        }
        __syncwarp();
        int h = 0;
        int64_t ops_off = 0;
        if (show && lane == 0) {
            h = atomicAdd(TA.hit_count, 1);
            if (h < TA.max_hits)
                ops_off = T.ops ? (int64_t)atomicAdd(T.ops_total, (unsigned long long)ncols)
                                : (int64_t)atomicAdd(TA.ops_total, (unsigned long long)ncols);
        }
        if (show && T.ops) {
            // the operations in alignment order: the scratch reversed
            h = __shfl_sync(0xffffffffu, h, 0);
            ops_off = __shfl_sync(0xffffffffu, ops_off, 0);
            if (h < TA.max_hits)
                for (int i = lane; i < ncols; i += kWarp) T.ops[ops_off + ncols - 1 - i] = scr[i];
        }
        if (show && lane == 0) {
            if (h < TA.max_hits) {
                DevHit o;
                o.pair = p;
                o.query = pm.query;
                o.target = pm.target;
                o.s_start = s_start;
                o.s_end = st.x;
                o.t_start = t_start;
                o.t_end = st.y;
                o.score = st.score_f;
                o.matches = mt;
                o.mismatches = mm;
                o.n_cols = ncols;
                o.end_x = st.x;
                o.end_y = st.y;
                o.ops_offset = ops_off;
                TA.hits[h] = o;
            }
        }
        __syncwarp();
    }
}

// ops_kernel for the hits of tile-form pairs: one warp per hit of the wave
// (hits of the other pairs return at once).
__global__ void __launch_bounds__(32) tile_ops_kernel(KernelArgs A, TraceArgs TA, TileArgs T, const DevHit* hits) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x;
    const DevHit H = hits[blockIdx.x];
    const int ti = T.slot_tile[H.pair];
    if (ti < 0) return;
    const TilePair tp = T.pairs[ti];
    TileView v = tile_view(A, T, tp, TA.metas[H.pair].thr_i, smem);
    int x = H.end_x, y = H.end_y;
    char* o = TA.ops + H.ops_offset;
    char mine = 0;
    for (int k = 0; k < H.n_cols; ++k) {
        const int d = v.code(x, y) & 3;
        char op;
        if (d == kLeft) {
            op = 'I';
            --x;
        } else if (d == kUp) {
            op = 'D';
            --y;
        } else {
            op = 'M';
            --x;
            --y;
        }
        if (lane == (k & 31)) mine = op;
        if ((k & 31) == 31 || k + 1 == H.n_cols) {
            // the batch of up to 32 operations, one byte a lane
            if (lane <= (k & 31)) o[H.n_cols - 1 - (k - (k & 31) + lane)] = mine;
            __syncwarp();
        }
    }
}

// ---- candidates from the score sweep's checkpoints (band_kernel<false, 4>)

// The candidate threshold of a pair (default_main.cu:609,
// SmithWatermanCuda.py:269-275), as band_kernel computes it.
__device__ __forceinline__ float tile_pair_threshold(const KernelArgs& A, int q, int t, int lq, int lt, float* maxf) {
    *maxf = A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip];
    const int mn = lq < lt ? lq : lt;
    const float pos = (float)(A.P.highest * (double)mn * A.P.filter_factor);
    return fmaxf(__fmul_rn(A.P.lower_limit, *maxf), pos);
}

// One block per pair of `list`: the pair's record (threshold, maximum) and
// the tiles whose maximum reaches the threshold, appended to sel as
// (list index, band * tiles + tile).
__global__ void tile_select_kernel(KernelArgs A, TileArgs T, const TilePair* list, int2* sel, int* sel_count,
                                   int sel_cap) {
    const TilePair tp = list[blockIdx.x];
    const int lq = A.q.len[tp.q], lt = A.t.len[tp.t];
    float maxf;
    const float thf = tile_pair_threshold(A, tp.q, tp.t, lq, lt, &maxf);
    const int thr = (int)fminf(fmaxf(ceilf(thf), -1.0e9f), 1.0e9f);
    if (threadIdx.x == 0) {
        PairMeta pm;
        pm.query = tp.q;
        pm.target = tp.t;
        pm.item = 0;
        pm.lane = 0;
        pm.n_cand = 0;
        pm.thr_i = thr;
        pm.thr_f = thf;
        pm.max_f = maxf;
        A.metas[tp.slot] = pm;
    }
    const int nbands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
    const int n = nbands * tile_count(lq);
    const int* tmx = T.ck + tp.tm;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (tmx[i] >= thr) {
            const int k = atomicAdd(sel_count, 1);
            if (k < sel_cap) sel[k] = make_int2((int)blockIdx.x, i);
        }
}

// One warp a block, persistent: each selected tile recomputed from the
// checkpoints, its candidates into the pair's slot.
__global__ void __launch_bounds__(32) tile_cand_kernel(KernelArgs A, TileArgs T, const TilePair* list,
                                                       const int2* sel, const int* sel_count, int* counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x;
    const int total = *sel_count;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= total) break;
        const int2 en = sel[it];
        const TilePair tp = list[en.x];
        TileView v = tile_view(A, T, tp, A.metas[tp.slot].thr_i, smem);
        const int b = en.y / v.ntiles, j = en.y % v.ntiles;
        v.load_h<true>(b, j, CandSink{A.cands + A.cand_base[tp.slot], A.cand_cap[tp.slot], A.n_cand + tp.slot},
                       v.lq - 1, b * kBandRows + kBandRows - 1);
    }
}

// The candidate counts of `list`'s pairs into their records.
__global__ void tile_cand_count_kernel(KernelArgs A, const TilePair* list, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = list[i].slot;
    A.metas[p].n_cand = A.n_cand[p];
}

// After a walk that wrote the tile-form hits' operations into their own
// buffer: those hits' offsets move past the other hits' operations (base).
__global__ void tile_ops_rebase_kernel(TileArgs T, DevHit* hits, int n_hits, int64_t base) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_hits) return;
    if (T.slot_tile[hits[h].pair] >= 0) hits[h].ops_offset += base;
}

}  // namespace pw
