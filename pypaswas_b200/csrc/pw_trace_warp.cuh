// pw_trace_warp.cuh -- direction sweep with one warp per pair.
//
// Used for traced pairs whose target is longer than one register strip: the
// per-lane strip sweep would give each such pair to a single lane, and a few
// thousand traced pairs cannot fill the GPU that way.  Here the 32 lanes of a
// warp share one pair: lane l owns target rows [y0 + 8l, y0 + 8l + 8) of a
// 256-row band and the warp walks the query columns as a skewed wavefront
// (lane l works on column s - l at step s).  The values lane l needs from the
// row above its slice -- computed one step earlier by lane l - 1 -- arrive
// through __shfl_up_sync; lane 0 reads them from the band boundary row that
// lane 31 stored for the previous band.
//
// Per cell it computes exactly what sweep_dirs computes (same recurrence, same
// classification, same candidate rule); only the order differs, and every cell
// still sees its up, left and diagonal neighbours.
//
// Cell codes are stored as [band][step][lane][8 rows]: one 8-byte store per
// lane and step, so every warp step writes 256 contiguous bytes.
#pragma once
#include "pw_kernels.cuh"

namespace pw {

constexpr int kWarpRows = 8;                   // rows per lane
constexpr int kBandRows = kWarpRows * kWarp;   // 256 rows per band

static_assert(kBandRows == 256 && kWarpRows == 8, "warp_layout_offset (pw_kernels.cuh) assumes 8 x 32 rows");

__host__ __device__ __forceinline__ int64_t warp_code_bytes(int lq, int lt) {
    const int64_t bands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
    return bands * ((int64_t)lq + kWarp - 1) * kWarp * kWarpRows;
}

// One item = one pair: W.first = query, W.target = target, W.pair_base = slot.
// Shared memory per warp: the lane profiles (32 x alpha1 x 8 scores, int8) and
// the query codes (padded to a multiple of 16).
template <bool AFFINE>
__global__ void __launch_bounds__(128) dir_warp_kernel(KernelArgs A, int qmax16) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int alpha1 = A.P.alpha + 1;
    const int prof_bytes = ((kWarp * alpha1 * kWarpRows) + 15) & ~15;
    unsigned char* wsm = smem + wib * (prof_bytes + qmax16);
    uint2* prof = (uint2*)wsm;              // [lane][alpha1] -> 8 int8 scores of that lane's rows
    uint8_t* qsm = wsm + prof_bytes;         // query codes
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    int4* bnd = (int4*)A.bnd_pool + warp_global * A.bnd_slot_elems;  // band boundary row: (H|M, I, B, -)
    const int gap = A.P.gap_i, ext = A.P.ext_i, ge = A.P.ge_i;
    const int neg = kNeg;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(A.item_counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const WorkItem W = A.items[it];
        const int q = W.first, t = W.target;
        const int lq = A.q.len[q], lt = A.t.len[t];
        const int64_t pslot = W.pair_base;
        // threshold of the pair (default_main.cu:609, SmithWatermanCuda.py:269-275)
        const float maxf = A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip];
        const int mn = lq < lt ? lq : lt;
        const float pos = (float)(A.P.highest * (double)mn * A.P.filter_factor);
        const float thf = fmaxf(__fmul_rn(A.P.lower_limit, maxf), pos);
        const int thr = (int)fminf(fmaxf(ceilf(thf), -1.0e9f), 1.0e9f);
        if (lane == 0) {
            PairMeta& pm = A.metas[pslot];
            pm.query = q;
            pm.target = t;
            pm.item = W.index;
            pm.lane = 0;
            pm.thr_f = thf;
            pm.thr_i = thr;
            pm.max_f = maxf;
        }
        Cand* cand = A.cands + A.cand_base[pslot];
        const int cap = A.cand_cap[pslot];
        int* ncand = A.n_cand + pslot;
        // query codes into shared memory
        const uint8_t* qg = A.q.codes + A.q.code_off[q];
        const int lq16 = (lq + 15) & ~15;
        for (int k = lane * 16; k < lq16; k += kWarp * 16) *(uint4*)(qsm + k) = *(const uint4*)(qg + k);
        const uint8_t* tres = A.t.codes + A.t.code_off[t];
        uint8_t* codes = A.codes + W.dir_base;
        const int64_t nsteps = (int64_t)lq + kWarp - 1;
        const int nbands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
        for (int band = 0; band < nbands; ++band) {
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
            const int ymine = yb + lane * kWarpRows;
            // per-row state of column x - 1
            int Hl[kWarpRows], Ml[kWarpRows], Jl[kWarpRows], Bl[kWarpRows];
#pragma unroll
            for (int r = 0; r < kWarpRows; ++r) {
                Hl[r] = 0;
                Ml[r] = 0;
                Jl[r] = neg;
                Bl[r] = 0;
            }
            // values of the row above this lane's slice: column x (up) and x - 1 (diag)
            int up_h = 0, up_m = 0, up_i = neg, up_b = 0;
            int dg_h = 0, dg_m = 0, dg_b = 0;
            // this lane's bottom row at its last column (handed to lane + 1)
            int bt_h = 0, bt_m = 0, bt_i = neg, bt_b = 0;
            for (int64_t s = 0; s < nsteps; ++s) {
                const int x = (int)s - lane;
                const bool active = x >= 0 && x < lq;
                // what lane - 1 computed at step s - 1 (its column x)
                int rh = 0, rm = 0, ri = neg, rb = 0;
                if constexpr (AFFINE) {
                    rm = __shfl_up_sync(0xffffffffu, bt_m, 1);
                    ri = __shfl_up_sync(0xffffffffu, bt_i, 1);
                    rb = __shfl_up_sync(0xffffffffu, bt_b, 1);
                } else {
                    rh = __shfl_up_sync(0xffffffffu, bt_h, 1);
                }
                if (lane == 0) {
                    if (has_up && active) {
                        const int4 v = bnd[x];
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
                // x == 0: the diagonal comes from the left boundary
                dg_h = x == 0 ? 0 : up_h;
                dg_m = x == 0 ? 0 : up_m;
                dg_b = x == 0 ? 0 : up_b;
                up_h = rh;
                up_m = rm;
                up_i = ri;
                up_b = rb;
                if (active) {
                    const int a = qsm[x];
                    const uint2 pw = prof[lane * alpha1 + a];
                    const bool xin = x > 0;
                    uint32_t w0 = 0, w1 = 0;
                    if constexpr (!AFFINE) {
                        int up = up_h, diag = dg_h;
#pragma unroll
                        for (int r = 0; r < kWarpRows; ++r) {
                            const int sc = (int)(int8_t)(uint8_t)((r < 4 ? pw.x : pw.y) >> (8 * (r & 3)));
                            const int left = Hl[r];
                            const int ls = left + gap, us = up + gap, ds = diag + sc;
                            int h = addmax(left, gap, ds);
                            h = addmax_relu(up, gap, h);
                            uint32_t code = h == ls ? kLeft : (h == us ? kUp : kUL);
                            code = h > 0 ? code : kNo;
                            const int y = ymine + r;
                            const bool ul = code == kUL;
                            const bool yin = y > 0;
                            const bool stop = ul && xin && yin && diag == 0;
                            code |= stop ? kStopFlag : 0u;
                            if (ul && h >= thr && y < lt) {
                                code |= kCand;
                                const int k = atomicAdd(ncand, 1);
                                if (k < cap) {
                                    Cand cc;
                                    cc.x = x;
                                    cc.y = y;
                                    cc.score_i = h;
                                    cc.score_f = (float)h;
                                    cand[k] = cc;
                                }
                            }
                            if (r < 4)
                                w0 |= code << (8 * r);
                            else
                                w1 |= code << (8 * (r - 4));
                            diag = left;
                            Hl[r] = h;
                            up = h;
                        }
                        bt_h = up;
                    } else {
                        int mup = up_m, iup = up_i, bdiag = dg_b, mdiag = dg_m;
#pragma unroll
                        for (int r = 0; r < kWarpRows; ++r) {
                            const int sc = (int)(int8_t)(uint8_t)((r < 4 ? pw.x : pw.y) >> (8 * (r & 3)));
                            const int m = addmax_relu(bdiag, sc, neg);
                            const int i = addmax(iup, ext, mup + ge);
                            const int jj = addmax(Jl[r], ext, Ml[r] + ge);
                            const int b = max3(m, i, jj);
                            uint32_t code = b == m ? kUL : (b == i ? kUp : kLeft);
                            code = b > 0 ? code : kNo;
                            const int y = ymine + r;
                            const bool main_src = code == kUL;
                            const bool yin = y > 0;
                            const bool stop = main_src && xin && yin && mdiag == 0;
                            code |= stop ? kStopFlag : 0u;
                            if (main_src && m >= thr && y < lt) {
                                code |= kCand;
                                const int k = atomicAdd(ncand, 1);
                                if (k < cap) {
                                    Cand cc;
                                    cc.x = x;
                                    cc.y = y;
                                    cc.score_i = m;
                                    cc.score_f = (float)m;
                                    cand[k] = cc;
                                }
                            }
                            if (r < 4)
                                w0 |= code << (8 * r);
                            else
                                w1 |= code << (8 * (r - 4));
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
                    }
                    *(uint2*)(codes + ((band * nsteps + s) * kWarp + lane) * kWarpRows) = make_uint2(w0, w1);
                    if (lane == kWarp - 1 && store_bnd) bnd[x] = make_int4(AFFINE ? bt_m : bt_h, bt_i, bt_b, 0);
                } else {
                    // not started (x < 0): hand the left-boundary values down
                    bt_h = 0;
                    bt_m = 0;
                    bt_i = neg;
                    bt_b = 0;
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            const int n = atomicAdd(ncand, 0);
            A.metas[pslot].n_cand = n;
        }
    }
}

}  // namespace pw
