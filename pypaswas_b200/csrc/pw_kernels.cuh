// pw_kernels.cuh -- the engine's kernels.
//
//   score_kernel     pair maxima (calculateScore / calculateScoreAffineGap,
//                    default_main.cu:130-303 / 317-561, max chain :169-180,297)
//   dir_kernel       the same sweep again for pairs whose maximum reached
//                    MINIMUM_SCORE, writing one code byte per cell (direction,
//                    stop flag, candidate flag) and the pair's candidate list
//   collect_kernel   starting points (traceback / tracebackAffineGap,
//                    default_main.cu:566-714 / 802-909): a candidate is a start
//                    unless another candidate's marking chain reaches it
//   walk_kernel      the host walk of SmithWaterman._print_alignments
//                    (SmithWaterman.py:699-838), one thread per pair
//   ops_kernel       writes the column operations of every kept hit
#pragma once
#include <type_traits>

#include "pw_device.cuh"

namespace pw {

// ------------------------------------------------------------------ profile
// Strip profile: for strip rows [y0, y0+S) and compact query residue a,
// word (g, a) packs the scores of rows y0+4g .. y0+4g+3 (int8 each; rows past
// the target end get the padding score).  fp32 path: one float4 per (g, a).
template <typename T, int S>
__device__ __forceinline__ void build_profile(void* prof, const int8_t* cmat_i8, const float* cmat_f,
                                              const uint8_t* tres, int y0, int lt, int alpha1, int dim,
                                              int lane) {
    const int n = (S / 4) * alpha1;
    for (int idx = lane; idx < n; idx += kWarp) {
        const int g = idx / alpha1, a = idx % alpha1;
        if constexpr (sizeof(T) == 4 && T(0.5f) == T(0)) {  // int path
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int y = y0 + 4 * g + k;
                const int8_t s = y < lt ? cmat_i8[a * dim + tres[y]] : (int8_t)-128;
                w |= (uint32_t)(uint8_t)s << (8 * k);
            }
            ((uint32_t*)prof)[idx] = w;
        } else {
            float4 w;
            float* wp = &w.x;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int y = y0 + 4 * g + k;
                wp[k] = y < lt ? cmat_f[a * dim + tres[y]] : -1.0e30f;
            }
            ((float4*)prof)[idx] = w;
        }
    }
}

template <typename T>
struct Prof4 {
    T s[4];
};

template <typename T>
__device__ __forceinline__ Prof4<T> load_prof(const void* prof, int g, int alpha1, int a) {
    Prof4<T> p;
    if constexpr (T(0.5f) == T(0)) {
        const uint32_t w = ((const uint32_t*)prof)[g * alpha1 + a];
#pragma unroll
        for (int k = 0; k < 4; ++k) p.s[k] = sext_byte(w, k);
    } else {
        const float4 w = ((const float4*)prof)[g * alpha1 + a];
        p.s[0] = w.x;
        p.s[1] = w.y;
        p.s[2] = w.z;
        p.s[3] = w.w;
    }
    return p;
}

template <typename T>
__device__ __forceinline__ T relu_addmax(T a, T b, T c) {  // max(a + b, c, 0)
    if constexpr (T(0.5f) == T(0))
        return addmax_relu(a, b, c);
    else
        return fmaxf(fmaxf(a + b, c), 0.0f);
}

template <typename T>
__device__ __forceinline__ T negT() {
    if constexpr (T(0.5f) == T(0))
        return (T)kNeg;
    else
        return (T)-1.0e10f;
}

// Boundary element handed from one strip to the next (row y0 + S - 1).
template <typename T>
struct Bnd {
    T m, i, b, pad;
};

// Per-lane context of one (query, target) pair.
struct LaneCtx {
    const uint8_t* qc;  // compact query codes, padded to a multiple of 4 with the pad code
    int lq, lq4;        // length and length rounded up to 4
    int lt;
    int y0;
    bool has_up, has_down;
};

// ------------------------------------------------------------ score sweeps
template <typename T, int S, bool AFFINE>
__device__ __forceinline__ void sweep_score(const LaneCtx& c, const void* prof, int alpha1, T gap, T ext, T ge,
                                            Bnd<T>* bnd, T& mx) {
    if constexpr (!AFFINE) {
        T H[S];
#pragma unroll
        for (int r = 0; r < S; ++r) H[r] = 0;
        T hb_prev = 0;
        for (int x4 = 0; x4 < c.lq4; x4 += 4) {
            const uint32_t cw = *(const uint32_t*)(c.qc + x4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                T up = c.has_up ? bnd[(int64_t)x * kWarp].m : T(0);
                T diag = hb_prev;
                hb_prev = up;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const Prof4<T> p = load_prof<T>(prof, g, alpha1, a);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const T left = H[r];
                        T h = addmax(left, gap, diag + p.s[k]);
                        h = relu_addmax(up, gap, h);
                        diag = left;
                        H[r] = h;
                        up = h;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = max3(mx, H[r], H[r + 1]);
                if (c.has_down) bnd[(int64_t)x * kWarp].m = H[S - 1];
            }
        }
    } else {
        T Ml[S], Jl[S], Bl[S];
        const T neg = negT<T>();
#pragma unroll
        for (int r = 0; r < S; ++r) {
            Ml[r] = 0;
            Jl[r] = neg;
            Bl[r] = 0;
        }
        T bb_prev = 0;
        for (int x4 = 0; x4 < c.lq4; x4 += 4) {
            const uint32_t cw = *(const uint32_t*)(c.qc + x4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                T mup = 0, iup = neg, bup = 0;
                if (c.has_up) {
                    const Bnd<T> b = bnd[(int64_t)x * kWarp];
                    mup = b.m;
                    iup = b.i;
                    bup = b.b;
                }
                T bdiag = bb_prev;
                bb_prev = bup;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const Prof4<T> p = load_prof<T>(prof, g, alpha1, a);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const T m = relu_addmax(bdiag, p.s[k], neg);
                        const T i = addmax(iup, ext, mup + ge);
                        const T jj = addmax(Jl[r], ext, Ml[r] + ge);
                        const T b = max3(m, i, jj);
                        bdiag = Bl[r];
                        Ml[r] = m;
                        Jl[r] = jj;
                        Bl[r] = b;
                        mup = m;
                        iup = i;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = max3(mx, Bl[r], Bl[r + 1]);
                if (c.has_down) {
                    Bnd<T> b;
                    b.m = mup;
                    b.i = iup;
                    b.b = Bl[S - 1];
                    b.pad = 0;
                    bnd[(int64_t)x * kWarp] = b;
                }
            }
        }
    }
}

// --------------------------------------------------------- direction sweeps
// Same recurrence as sweep_score; additionally classifies every cell like the
// reference and records starting-point candidates.
//   linear (default_main.cu:259-271): direction LEFT if H == left+gap, else UP
//     if H == up+gap, else UPPER_LEFT; NO when H == 0.  Stop flag: UPPER_LEFT
//     with a zero diagonal predecessor inside the matrix (:632-659).
//     Candidate: UPPER_LEFT and H >= threshold (:609).
//   affine (:467-526): best B = max(M, I, J); source MAIN if B == M, else I if
//     B == I, else J; NO when B == 0.  Stop flag: MAIN with M(x-1, y-1) == 0
//     inside the matrix (:724-751).  Candidate: MAIN and M >= threshold (:850).
// TRANS: the strip sequence is the query (the reference's x axis) and the
// lanes sweep targets (its y axis), so the reference's LEFT neighbour is the
// previous strip row and its UP neighbour the previous column; likewise the
// affine I matrix (gaps along y) is the per-row chain and J the column chain.
template <typename T, int S, bool AFFINE, bool TRANS = false>
__device__ __forceinline__ void sweep_dirs(const LaneCtx& c, const void* prof, int alpha1, T gap, T ext, T ge,
                                           Bnd<T>* bnd, uint8_t* codes, int lane, int xmax4, T thr, Cand* cand,
                                           int cand_cap, int& n_cand) {
    uint2* out = (uint2*)codes;  // 4-bit cell codes: 16 rows of a lane in 8 bytes
    if constexpr (!AFFINE) {
        T H[S];
#pragma unroll
        for (int r = 0; r < S; ++r) H[r] = 0;
        T hb_prev = 0;
        for (int x4 = 0; x4 < c.lq4; x4 += 4) {
            const uint32_t cw = *(const uint32_t*)(c.qc + x4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const bool xin = x > 0;
                T up = c.has_up ? bnd[(int64_t)x * kWarp].m : T(0);
                T diag = hb_prev;
                hb_prev = up;
                uint32_t words[S / 8];
#pragma unroll
                for (int q = 0; q < S / 8; ++q) words[q] = 0;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const Prof4<T> p = load_prof<T>(prof, g, alpha1, a);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const T left = H[r];
                        const T ls = left + gap, us = up + gap, ds = diag + p.s[k];
                        T h = addmax(left, gap, ds);
                        h = relu_addmax(up, gap, h);
                        uint32_t code = TRANS ? (h == us ? kLeft : (h == ls ? kUp : kUL))
                                              : (h == ls ? kLeft : (h == us ? kUp : kUL));
                        code = h > T(0) ? code : kNo;
                        const bool ul = code == kUL;
                        const bool yin = (r > 0) || c.has_up;
                        const bool stop = ul && xin && yin && diag == T(0);
                        const bool cnd = ul && h >= thr;
                        code |= stop ? kStopFlag : 0u;
                        if (cnd) {
                            const int y = c.y0 + r;
                            if (x < c.lq && y < c.lt) {
                                code |= kCand;
                                if (n_cand < cand_cap) {
                                    Cand cc;
                                    cc.x = TRANS ? y : x;
                                    cc.y = TRANS ? x : y;
                                    cc.score_i = (int32_t)h;
                                    cc.score_f = (float)h;
                                    cand[n_cand] = cc;
                                }
                                ++n_cand;
                            }
                        }
                        words[r / 8] |= code << (4 * (r % 8));
                        diag = left;
                        H[r] = h;
                        up = h;
                    }
                }
#pragma unroll
                for (int q = 0; q < S / 16; ++q)
                    out[((int64_t)x * (S / 16) + q) * kWarp + lane] = make_uint2(words[2 * q], words[2 * q + 1]);
                if (c.has_down) bnd[(int64_t)x * kWarp].m = H[S - 1];
            }
        }
    } else {
        T Ml[S], Jl[S], Bl[S];
        const T neg = negT<T>();
#pragma unroll
        for (int r = 0; r < S; ++r) {
            Ml[r] = 0;
            Jl[r] = neg;
            Bl[r] = 0;
        }
        T bb_prev = 0, bm_prev = 0;
        for (int x4 = 0; x4 < c.lq4; x4 += 4) {
            const uint32_t cw = *(const uint32_t*)(c.qc + x4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cw >> (8 * j)) & 0xff;
                const bool xin = x > 0;
                T mup = 0, iup = neg, bup = 0;
                if (c.has_up) {
                    const Bnd<T> b = bnd[(int64_t)x * kWarp];
                    mup = b.m;
                    iup = b.i;
                    bup = b.b;
                }
                T bdiag = bb_prev, mdiag = bm_prev;
                bb_prev = bup;
                bm_prev = mup;
                uint32_t words[S / 8];
#pragma unroll
                for (int q = 0; q < S / 8; ++q) words[q] = 0;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const Prof4<T> p = load_prof<T>(prof, g, alpha1, a);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const T m = relu_addmax(bdiag, p.s[k], neg);
                        const T i = addmax(iup, ext, mup + ge);
                        const T jj = addmax(Jl[r], ext, Ml[r] + ge);
                        const T b = max3(m, i, jj);
                        uint32_t code = b == m ? kUL : (b == (TRANS ? jj : i) ? kUp : kLeft);
                        code = b > T(0) ? code : kNo;
                        const bool main_src = code == kUL;
                        const bool yin = (r > 0) || c.has_up;
                        const bool stop = main_src && xin && yin && mdiag == T(0);
                        const bool cnd = main_src && m >= thr;
                        code |= stop ? kStopFlag : 0u;
                        if (cnd) {
                            const int y = c.y0 + r;
                            if (x < c.lq && y < c.lt) {
                                code |= kCand;
                                if (n_cand < cand_cap) {
                                    Cand cc;
                                    cc.x = TRANS ? y : x;
                                    cc.y = TRANS ? x : y;
                                    cc.score_i = (int32_t)m;
                                    cc.score_f = (float)m;
                                    cand[n_cand] = cc;
                                }
                                ++n_cand;
                            }
                        }
                        words[r / 8] |= code << (4 * (r % 8));
                        bdiag = Bl[r];
                        mdiag = Ml[r];
                        Ml[r] = m;
                        Jl[r] = jj;
                        Bl[r] = b;
                        mup = m;
                        iup = i;
                    }
                }
#pragma unroll
                for (int q = 0; q < S / 16; ++q)
                    out[((int64_t)x * (S / 16) + q) * kWarp + lane] = make_uint2(words[2 * q], words[2 * q + 1]);
                if (c.has_down) {
                    Bnd<T> b;
                    b.m = mup;
                    b.i = iup;
                    b.b = Bl[S - 1];
                    b.pad = 0;
                    bnd[(int64_t)x * kWarp] = b;
                }
            }
        }
    }
    (void)xmax4;
}

// Direction sweep of linear-gap integer pairs that stores H instead of cell
// codes: every cell's 16-bit score (all traced maxima are below 2^15), 16 rows
// of a lane in 32 bytes at the cells' code positions, [strip][x][r / 16][lane]
// [16 rows], so that a warp stores 1 KB contiguous per 16 rows and column.  The
// code of a cell (direction, stop flag, candidate flag) is derived on read
// from the cell and its left, upper and diagonal neighbours (PairView::code):
// the collect and walk kernels read only the cells on their paths.  The
// candidate list is written here, as sweep_dirs writes it.
template <int S, bool TRANS = false>
__device__ __forceinline__ void sweep_hstore(const LaneCtx& c, const void* prof, int alpha1, int gap,
                                             Bnd<int>* bnd, uint8_t* hs, int lane, int thr, Cand* cand,
                                             int cand_cap, int& n_cand) {
    uint4* out = (uint4*)hs;
    const int16_t* hv = (const int16_t*)hs;
    int H[S];
#pragma unroll
    for (int r = 0; r < S; ++r) H[r] = 0;
    int hb_prev = 0;
    // the code word of the next four columns is loaded four columns ahead
    uint32_t cw = 0, cw_next = c.lq4 > 0 ? *(const uint32_t*)c.qc : 0u;
    // one column per iteration (a compact loop body: the fully unrolled
    // four-column form stalled on instruction fetch)
#pragma unroll 1
    for (int x = 0; x < c.lq4; ++x) {
        if ((x & 3) == 0) {
            cw = cw_next;
            if (x + 4 < c.lq4) cw_next = *(const uint32_t*)(c.qc + x + 4);
        }
        const int a = (cw >> (8 * (x & 3))) & 0xff;
        const int up0 = c.has_up ? bnd[(int64_t)x * kWarp].m : 0;
        int up = up0;
        int diag = hb_prev;
        hb_prev = up0;
#pragma unroll
        for (int g = 0; g < S / 4; ++g) {
            const Prof4<int> p = load_prof<int>(prof, g, alpha1, a);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int r = 4 * g + k;
                const int left = H[r];
                int h = addmax(left, gap, diag + p.s[k]);
                h = relu_addmax(up, gap, h);
                diag = left;
                H[r] = h;
                up = h;
            }
        }
#pragma unroll
        for (int q = 0; q < S / 16; ++q) {
            uint32_t w[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = __byte_perm(H[16 * q + 2 * k], H[16 * q + 2 * k + 1], 0x5410);
            uint4* o = out + (((int64_t)x * (S / 16) + q) * kWarp + lane) * 2;
            o[0] = make_uint4(w[0], w[1], w[2], w[3]);
            o[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
        if (c.has_down) bnd[(int64_t)x * kWarp].m = H[S - 1];
        // candidates (rare: cells reaching the pair's threshold): a UL cell,
        // i.e. neither gap source reaches h (in either orientation), inside
        // the matrix; the left neighbours come back from the column stored
        // one iteration earlier by this thread
        int cm = 0;
#pragma unroll
        for (int r = 0; r < S; r += 2) cm = max3(cm, H[r], H[r + 1]);
        if (cm >= thr) {
#pragma unroll
            for (int r = 0; r < S; ++r) {  // unrolled: H stays in registers
                const int h = H[r];
                const int y = c.y0 + r;
                if (h < thr || h <= 0 || x >= c.lq || y >= c.lt) continue;
                const int left = x > 0 ? (int)hv[(((int64_t)(x - 1) * (S / 16) + r / 16) * kWarp + lane) * 16 + r % 16]
                                       : 0;
                const int upv = r > 0 ? H[r - 1] : up0;
                if (h == left + gap || h == upv + gap) continue;
                if (n_cand < cand_cap) {
                    Cand cc;
                    cc.x = TRANS ? y : x;
                    cc.y = TRANS ? x : y;
                    cc.score_i = h;
                    cc.score_f = (float)h;
                    cand[n_cand] = cc;
                }
                ++n_cand;
            }
        }
    }
}

// Sequences on the device.
struct SeqSet {
    const uint8_t* codes;    // query: compact codes / target: matrix residue index
    const int64_t* code_off; // 16-byte aligned offsets into codes
    const uint8_t* raw;      // upper-cased residues as given
    const int64_t* raw_off;
    const int32_t* len;
    const int32_t* key;      // id equality key
};

struct KernelArgs {
    const WorkItem* items;
    int n_items;
    int* item_counter;
    SeqSet q, t;
    const int32_t* q_order;  // sorted position -> query index
    const int8_t* cmat_i8;   // [(alpha+1) * dim]
    const float* cmat_f;
    ScoreParams P;
    float* pair_max;         // [nq * nt]
    int nt;
    int64_t pm_lane, pm_strip;  // pair_max index = lane * pm_lane + strip * pm_strip
    void* bnd_pool;
    int64_t bnd_slot_elems;  // elements per warp slot (xmax4 * 32)
    // phase 2
    uint8_t* codes;
    PairMeta* metas;
    Cand* cands;
    const int64_t* cand_base;  // per pair slot: first candidate
    const int32_t* cand_cap;   // per pair slot: capacity
    int32_t* n_cand;           // per pair slot: candidates found (may exceed the capacity)
};

template <typename T>
__device__ __forceinline__ T from_f(float v) {
    if constexpr (T(0.5f) == T(0))
        return (T)v;
    else
        return v;
}

// Persistent kernel over work items: one warp per item, dynamic scheduling.
// PHASE 1 writes pair maxima; PHASE 2 writes cell codes and candidates;
// PHASE 3 writes 16-bit H values and candidates (sweep_hstore).
template <typename T, int S, bool AFFINE, bool MULTI, int PHASE, bool TRANS = false>
__global__ void __launch_bounds__(128) sweep_kernel(KernelArgs A) {
    static_assert(PHASE != 3 || (std::is_same<T, int>::value && !AFFINE), "H store: linear gap, int lanes");
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int alpha1 = A.P.alpha + 1;
    const int prof_bytes = (S / 4) * alpha1 * (int)(T(0.5f) == T(0) ? 4 : 16);
    void* prof = smem + wib * ((prof_bytes + 15) & ~15);
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    Bnd<T>* bnd_slot = MULTI ? (Bnd<T>*)A.bnd_pool + warp_global * A.bnd_slot_elems + lane : nullptr;
    const T gap = A.P.is_float ? from_f<T>(A.P.gap_f) : (T)A.P.gap_i;
    const T ext = A.P.is_float ? from_f<T>(A.P.ext_f) : (T)A.P.ext_i;
    const T ge = A.P.is_float ? from_f<T>(A.P.ge_f) : (T)A.P.ge_i;

    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(A.item_counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const WorkItem W = A.items[it];
        const int t = W.target;
        const int lt = A.t.len[t];
        const bool active = lane < W.lanes;
        const int q = active ? A.q_order[W.first + lane] : 0;
        LaneCtx c;
        c.qc = A.q.codes + A.q.code_off[q];
        c.lq = active ? A.q.len[q] : 0;
        c.lq4 = (c.lq + 3) & ~3;
        c.lt = lt;
        const uint8_t* tres = A.t.codes + A.t.code_off[t];
        const int nstrips = MULTI ? (lt + S - 1) / S : 1;
        T mx = 0;
        // phase 2 per-pair state
        T thr = 0;
        int n_cand = 0;
        Cand* cand = nullptr;
        int cap = 0;
        int64_t pslot = W.pair_base + lane;
        if (PHASE >= 2 && active) {
            const float maxf = A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip];
            const int mn = c.lq < lt ? c.lq : lt;
            // maxPossibleScore, SmithWatermanCuda.py:269-275 (double, stored as fp32)
            const float pos = (float)(A.P.highest * (double)mn * A.P.filter_factor);
            const float llm = __fmul_rn(A.P.lower_limit, maxf);
            const float thf = fmaxf(llm, pos);
            if constexpr (T(0.5f) == T(0)) {
                float tc = ceilf(thf);
                tc = fminf(fmaxf(tc, -1.0e9f), 1.0e9f);
                thr = (T)tc;
            } else {
                thr = thf;
            }
            cand = A.cands + A.cand_base[pslot];
            cap = A.cand_cap[pslot];
            PairMeta& pm = A.metas[pslot];
            pm.query = TRANS ? t : q;
            pm.target = TRANS ? q : t;
            pm.item = W.index;
            pm.lane = lane;
            pm.thr_f = thf;
            pm.thr_i = (int32_t)(T(0.5f) == T(0) ? (float)thr : 0.0f);
            pm.max_f = maxf;
        }
        const int xmax4 = (W.xmax + 3) & ~3;
        for (int s = 0; s < nstrips; ++s) {
            c.y0 = s * S;
            c.has_up = s > 0;
            c.has_down = s + 1 < nstrips;
            __syncwarp();
            build_profile<T, S>(prof, A.cmat_i8, A.cmat_f, tres, c.y0, lt, alpha1, A.P.dim, lane);
            __syncwarp();
            if (active) {
                if constexpr (PHASE == 1) {
                    sweep_score<T, S, AFFINE>(c, prof, alpha1, gap, ext, ge, bnd_slot, mx);
                } else if constexpr (PHASE == 2) {
                    uint8_t* codes = A.codes + W.dir_base + (int64_t)s * xmax4 * S * kWarp / 2;
                    sweep_dirs<T, S, AFFINE, TRANS>(c, prof, alpha1, gap, ext, ge, bnd_slot, codes, lane, xmax4,
                                                    thr, cand, cap, n_cand);
                } else {
                    uint8_t* hs = A.codes + W.dir_base + (int64_t)s * xmax4 * S * kWarp * 2;
                    sweep_hstore<S, TRANS>(c, prof, alpha1, (int)gap, (Bnd<int>*)bnd_slot, hs, lane, (int)thr,
                                           cand, cap, n_cand);
                }
            }
        }
        if (active) {
            if constexpr (PHASE == 1)
                A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip] = (float)mx;
            else {
                A.metas[pslot].n_cand = n_cand;
                A.n_cand[pslot] = n_cand;
            }
        }
    }
}

// ------------------------------------------------------------ traceback side
struct TraceArgs {
    const PairMeta* metas;
    int n_pairs;
    const WorkItem* items;
    uint8_t* codes;          // 4-bit cell codes of the wave, or 16-bit H values (hstore)
    int hstore;              // linear integer sweeps: the wave holds H, codes are derived on read
    uint8_t* marks;          // one bit per cell of the wave (zeroed per wave): covered, then visited
    Cand* cands;
    const int64_t* cand_base;
    int32_t* n_starts;       // per pair: starting points (after collect)
    SeqSet q, t;
    ScoreParams P;
    const uint8_t* allowed;  // per start (packed order, see gather_kernel): walk it; null = all
    const int64_t* start_off; // per pair: first packed start index
    DevHit* hits;
    int* hit_count;
    int max_hits;
    char* ops;
    unsigned long long* ops_total;  // column operations reserved so far (walk_kernel assigns ops offsets)
    const int32_t* slot_tile;       // per pair slot: >= 0 for pairs of the tile form (pw_tiles.cuh), which
                                    // these kernels leave to the tile kernels; null: none
};

// Offset of cell (x, y) in the layout of the band direction sweep
// (pw_band.cuh): [band of 256 rows][step][lane][8 rows], step = x + lane.
__host__ __device__ __forceinline__ int64_t warp_layout_offset(int x, int y, int lq) {
    const int band = y >> 8, l = (y & 255) >> 3, r = y & 7;
    const int64_t nsteps = (int64_t)lq + 31;
    return ((band * nsteps + x + l) * 32 + l) * 8 + r;
}

// A traced pair's cells.  Each cell has a 4-bit code (direction, stop flag,
// candidate flag; two cells per byte, the even index in the low nibble) and a
// 1-bit mark in a separate plane: collect_kernel marks covered candidates there
// (and clears them again), walk_kernel marks the cells it visits
// (IN_ALIGNMENT).  The cell index is the item's own: the strip or band layout.
struct PairView {
    uint8_t* base;      // the item's cell codes (4 bits a cell), or its 16-bit H values (hstore)
    uint8_t* marks;     // the wave's mark plane
    int64_t cell0;      // the item's first cell in the wave
    int S, lane, xmax4, lq, lt;
    int layout;  // 0: strip sweep, targets as strips; 1: strip sweep, queries as strips; 2: warp sweep
    bool hstore;        // base holds H; codes are derived on read
    int gap, thr;       // hstore: the linear gap and the pair's integer candidate threshold
    // cell (x, y) in the reference's coordinates (x: query, y: target)
    __device__ __forceinline__ int64_t index(int x, int y) const {
        if (layout == 2) return warp_layout_offset(x, y, lq);
        return layout == 1 ? cell_offset_rt(S, y, x, lane, xmax4) : cell_offset_rt(S, x, y, lane, xmax4);
    }
    // H of a cell; 0 left of and above the matrix (the sweeps' boundary)
    __device__ __forceinline__ int hval(int x, int y) const {
        return (x < 0 || y < 0) ? 0 : (int)((const int16_t*)base)[index(x, y)];
    }
    __device__ __forceinline__ uint32_t code(int x, int y) const {
        if (!hstore) {
            const int64_t i = index(x, y);
            return (base[i >> 1] >> ((i & 1) * 4)) & 15u;
        }
        // the classification of sweep_dirs from the stored H values: LEFT
        // when the left neighbour plus the gap reaches H, else UP when the
        // upper one does, else UL; NO where H is 0; a UL cell inside the
        // matrix with a zero diagonal neighbour carries the stop flag, one
        // reaching the pair's threshold the candidate flag
        // the four loads are issued together (one memory round trip a cell)
        const int h = hval(x, y), l = hval(x - 1, y), u = hval(x, y - 1), d = hval(x - 1, y - 1);
        if (h <= 0) return kNo;
        if (h == l + gap) return kLeft;
        if (h == u + gap) return kUp;
        uint32_t cd = kUL;
        if (x > 0 && y > 0 && d == 0) cd |= kStopFlag;
        if (h >= thr && x < lq && y < lt) cd |= kCand;
        return cd;
    }
    // Starts fetching cell (x, y)'s code (or H values) and mark into L2: the
    // walks follow one path a dependent load at a time, mostly along the
    // diagonal, so the cells a few steps ahead are requested early.  A hint
    // only: cells outside the matrix are skipped.
    __device__ __forceinline__ void prefetch(int x, int y) const {
        if (x < 1 || y < 1) return;
        const int64_t i = index(x, y);
        const uint8_t* c = hstore ? base + 2 * i : base + (i >> 1);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(c));
        if (hstore) asm volatile("prefetch.global.L2 [%0];" ::"l"(base + 2 * index(x - 1, y)));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(marks + ((cell0 + i) >> 3)));
    }
    __device__ __forceinline__ bool marked(int x, int y) const {
        const int64_t i = cell0 + index(x, y);
        return (marks[i >> 3] >> (i & 7)) & 1u;
    }
    __device__ __forceinline__ void mark(int x, int y) const {
        const int64_t i = cell0 + index(x, y);
        marks[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
    __device__ __forceinline__ void unmark(int x, int y) const {
        const int64_t i = cell0 + index(x, y);
        marks[i >> 3] &= (uint8_t)~(1u << (i & 7));
    }
};

// Diagonal steps a path walk requests ahead (PairView::prefetch).
constexpr int kWalkAhead = 8;

__device__ __forceinline__ PairView pair_view(const TraceArgs& A, const PairMeta& pm) {
    PairView v;
    const WorkItem W = A.items[pm.item];
    v.base = A.codes + W.dir_base;
    v.marks = A.marks;
    v.hstore = A.hstore != 0;
    v.cell0 = v.hstore ? W.dir_base / 2 : W.dir_base * 2;
    v.gap = A.P.gap_i;
    v.thr = pm.thr_i;
    v.S = W.S;
    v.lane = pm.lane;
    v.xmax4 = (W.xmax + 3) & ~3;
    v.lq = A.q.len[pm.query];
    v.lt = A.t.len[pm.target];
    v.layout = W.orient;
    return v;
}

// Emission rank of a starting point inside its pair: the reference's reverse
// sweep emits by block anti-diagonal descending, block x descending, cell
// anti-diagonal descending inside the 8x8 block, then linear thread index
// (thread y ascending).  Smaller key = emitted earlier.
__host__ __device__ __forceinline__ uint64_t emission_key(int x, int y) {
    const uint32_t bx = (uint32_t)x >> 3, by = (uint32_t)y >> 3;
    const uint32_t d = bx + by, i = (x & 7) + (y & 7), ty = y & 7;
    // descending fields are stored complemented
    return ((uint64_t)(0xFFFFFu - d) << 40) | ((uint64_t)(0xFFFFFu - bx) << 20) |
           ((uint64_t)(15u - i) << 4) | ty;
}

template <bool AFFINE>
__global__ void collect_kernel(TraceArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_pairs) return;
    if (A.slot_tile && A.slot_tile[p] >= 0) return;
    const PairMeta pm = A.metas[p];
    Cand* cl = A.cands + A.cand_base[p];
    const int n = pm.n_cand;
    PairView v = pair_view(A, pm);
    // marking chains: the nearest candidate up a candidate's chain is covered
    for (int k = 0; k < n; ++k) {
        int x = cl[k].x - 1, y = cl[k].y - 1;
        while (x >= 0 && y >= 0) {
            v.prefetch(x - kWalkAhead, y - kWalkAhead);
            const uint32_t cd = v.code(x, y);
            const int d = cd & 3;
            if (cd & kCand) {
                v.mark(x, y);  // covered
                break;
            }
            if (AFFINE) {
                if (d != kUL) break;
                --x;
                --y;
            } else {
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
    }
    // keep uncovered candidates (clearing the covered marks, so that the
    // plane holds only the walk's marks afterwards), then order them for the
    // walk: ascending score, then emission order (SmithWaterman.py:699 is a
    // stable sort)
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
            const bool after = o.score_f > key.score_f ||
                               (o.score_f == key.score_f && emission_key(o.x, o.y) > ek);
            if (!after) break;
            cl[j + 1] = o;
            --j;
        }
        cl[j + 1] = key;
    }
    A.n_starts[p] = m;
}

// Affine stop rule: a MAIN cell with a zero diagonal predecessor becomes STOP
// only if it is marked, i.e. a candidate lies on its diagonal run of MAIN cells
// (itself or further down-right).
__device__ __forceinline__ bool run_has_candidate(const PairView& v, int x, int y) {
    while (x < v.lq && y < v.lt) {
        const uint32_t cd = v.code(x, y);
        if (cd & kCand) return true;
        if ((cd & 3) != kUL) return false;
        ++x;
        ++y;
    }
    return false;
}

constexpr int kStopDir = 64, kInAlignment = 96;

template <bool AFFINE>
__device__ __forceinline__ int walk_direction(const PairView& v, int x, int y) {
    if (v.marked(x, y)) return kInAlignment;
    const uint32_t cd = v.code(x, y);
    const int d = cd & 3;
    if (d == kUL && (cd & kStopFlag)) {
        if (!AFFINE || run_has_candidate(v, x, y)) return kStopDir;
    }
    return d;  // 0: never written in the reference's zero-copy buffer
}

__device__ __forceinline__ bool same_residue(uint8_t a, uint8_t b) {
    // str.lower() equality of single characters (SmithWaterman.py:771)
    const bool la = (a >= 'A' && a <= 'Z') || (a >= 'a' && a <= 'z');
    return la ? ((a | 0x20) == (b | 0x20)) : a == b;
}

template <bool AFFINE>
__global__ void walk_kernel(TraceArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_pairs) return;
    if (A.slot_tile && A.slot_tile[p] >= 0) return;
    const PairMeta pm = A.metas[p];
    const Cand* cl = A.cands + A.cand_base[p];
    const int m = A.n_starts[p];
    PairView v = pair_view(A, pm);
    const uint8_t* qs = A.q.raw + A.q.raw_off[pm.query];
    const uint8_t* ts = A.t.raw + A.t.raw_off[pm.target];
    const bool same_id = A.q.key[pm.query] == A.t.key[pm.target];
    for (int k = 0; k < m; ++k) {
        if (A.allowed && !A.allowed[A.start_off[p] + k]) continue;
        const Cand st = cl[k];
        int x = st.x, y = st.y;
        int dir = walk_direction<AFFINE>(v, x, y);
        bool show = true;
        if (same_id) {  // SmithWaterman.py:752-755
            dir = kStopDir;
            show = false;
        }
        if ((double)st.score_f < A.P.host_minimum) show = false;  // :758-759
        int s_start = x + 1, t_start = y + 1, ncols = 0, mt = 0, mm = 0;
        // Affine stop rule: whether a candidate lies on the cell's diagonal
        // run of MAIN cells (run_has_candidate).  Along a diagonal stretch of
        // the walk it follows from the cell the walk came from (-1: unknown,
        // after a gap move), so the run is scanned only when that is unknown.
        int run_next = -1;
        while (show && x >= 0 && y >= 0 && dir != kStopDir && dir != 32) {  // :761
            v.prefetch(x - kWalkAhead, y - kWalkAhead);
            const uint32_t cd = v.code(x, y);
            const int d = cd & 3;
            int run_here = (cd & kCand) ? 1 : (d != kUL ? 0 : run_next);
            if (v.marked(x, y)) {
                dir = kInAlignment;
            } else if (d == kUL && (cd & kStopFlag)) {
                if (AFFINE && run_here < 0) run_here = run_has_candidate(v, x + 1, y + 1) ? 1 : 0;
                dir = (!AFFINE || run_here) ? kStopDir : kUL;
            } else {
                dir = d;
            }
            run_next = dir == kUL ? run_here : -1;
            v.mark(x, y);  // IN_ALIGNMENT
            if (dir == kInAlignment) {
                show = false;
            } else if (dir == kUL || dir == kStopDir) {
                if (same_residue(ts[y], qs[x]))
                    ++mt;
                else
                    ++mm;
                --s_start;
                --t_start;
                ++ncols;
                if (dir == kUL) {
                    --x;
                    --y;
                }
            } else if (dir == kLeft) {
                --s_start;
                ++ncols;
                --x;
            } else if (dir == kUp) {
                --t_start;
                ++ncols;
                --y;
            } else {
                x = -1;
            }
        }
        if (show) {
            const int h = atomicAdd(A.hit_count, 1);
            if (h < A.max_hits) {
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
                o.ops_offset = (int64_t)atomicAdd(A.ops_total, (unsigned long long)ncols);
                A.hits[h] = o;
            }
        }
    }
}

// Translation units that only need the score sweep define PW_SCORE_SWEEP_ONLY
// so that these non-template kernels are emitted once, by engine.cu.
#ifndef PW_SCORE_SWEEP_ONLY
// Column operations of each hit, in alignment order: 'M' both residues,
// 'I' query residue against a gap, 'D' target residue against a gap.
__global__ void ops_kernel(TraceArgs A, const DevHit* hits, int n_hits) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_hits) return;
    const DevHit H = hits[h];
    if (A.slot_tile && A.slot_tile[H.pair] >= 0) return;
    const PairMeta pm = A.metas[H.pair];
    PairView v = pair_view(A, pm);
    int x = H.end_x, y = H.end_y;
    char* o = A.ops + H.ops_offset;
    for (int k = 0; k < H.n_cols; ++k) {
        v.prefetch(x - kWalkAhead, y - kWalkAhead);
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
        o[H.n_cols - 1 - k] = op;
    }
}

// Packs every pair's ordered starting points into one array (pair slot, cell,
// score) so that the host reads only what exists.
// One starting point as the host orders and reports it (StartingPoint of
// default_main.cu:66-76 with the pair resolved to query / target indices).
struct StartRec {
    int32_t query, target, x, y;
    float score;
    float max_score, pos_score;
};

// Starting points of every pair, packed by start_off (an exclusive scan of
// n_starts), with the pair's maximum and maxPossibleScore
// (fp32(highest * min(len_q, len_t) * filter_factor) in double,
// SmithWatermanCuda.py:269-275).
__global__ void gather_kernel(TraceArgs A, StartRec* out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_pairs) return;
    const Cand* cl = A.cands + A.cand_base[p];
    const int m = A.n_starts[p];
    const int64_t o = A.start_off[p];
    const PairMeta pm = A.metas[p];
    const int lq = A.q.len[pm.query], lt = A.t.len[pm.target];
    const float pos = (float)(A.P.highest * (double)(lq < lt ? lq : lt) * A.P.filter_factor);
    for (int k = 0; k < m; ++k) {
        StartRec s;
        s.query = pm.query;
        s.target = pm.target;
        s.x = cl[k].x;
        s.y = cl[k].y;
        s.score = cl[k].score_f;
        s.max_score = pm.max_f;
        s.pos_score = pos;
        out[o + k] = s;
    }
}

// Integer issue-rate probe for the roofline denominator: independent chains
// of the DPX add-max used by the recurrences (one __viaddmax_s32 = one add +
// one max).  Each thread runs 8 independent chains; the result is stored so
// that nothing is optimised away.
__global__ void int_peak_kernel(int iters, int seed, int* sink) {
    int a0 = threadIdx.x + seed, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
        a7 = a0 + 7;
    const int b = seed & 7, c = -seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = __viaddmax_s32(a0, b, c);
            a1 = __viaddmax_s32(a1, b, c);
            a2 = __viaddmax_s32(a2, b, c);
            a3 = __viaddmax_s32(a3, b, c);
            a4 = __viaddmax_s32(a4, b, c);
            a5 = __viaddmax_s32(a5, b, c);
            a6 = __viaddmax_s32(a6, b, c);
            a7 = __viaddmax_s32(a7, b, c);
        }
    }
    const int r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x7fffffff) sink[0] = r;
}

// Same probe on the 16x2 form (one instruction = two adds and two maxima).
__global__ void int_peak16_kernel(int iters, int seed, int* sink) {
    unsigned a0 = threadIdx.x + seed, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5,
             a6 = a0 + 6, a7 = a0 + 7;
    const unsigned b = (unsigned)(seed & 7) * 0x10001u, c = 0xC000C000u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = __viaddmax_s16x2(a0, b, c);
            a1 = __viaddmax_s16x2(a1, b, c);
            a2 = __viaddmax_s16x2(a2, b, c);
            a3 = __viaddmax_s16x2(a3, b, c);
            a4 = __viaddmax_s16x2(a4, b, c);
            a5 = __viaddmax_s16x2(a5, b, c);
            a6 = __viaddmax_s16x2(a6, b, c);
            a7 = __viaddmax_s16x2(a7, b, c);
        }
    }
    const unsigned r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x7fffffffu) sink[0] = (int)r;
}

// Passing pairs per query (target-major pair indices k = t * nq + sp from the
// pruning selection; pairs of targets marked in skip are left out).
__global__ void query_count_kernel(const int64_t* sel, int64_t n, int nq, const int32_t* q_order,
                                   const uint8_t* skip, int32_t* count) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = sel[j];
        const int t = (int)(k / nq);
        if (!skip[t]) atomicAdd(&count[q_order[k - (int64_t)t * nq]], 1);
    }
}

// Sum over queries of ceil(count / per_item) * per_item * len: the lane slots
// of the transposed orientation's groups, in units of one shortest target.
__global__ void group_bound_kernel(const int32_t* count, int nq, const int32_t* q_len, int per_item,
                                   unsigned long long* sum) {
    unsigned long long acc = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        if (count[q] > 0)
            acc += (unsigned long long)((count[q] + per_item - 1) / per_item) * per_item * (unsigned long long)q_len[q];
    if (acc) atomicAdd(sum, acc);
}

// Candidate slots of a wave's pairs: pair p owns [p * cap, (p + 1) * cap).
__global__ void cand_slot_kernel(int64_t* cand_base, int32_t* cand_cap, int64_t n_pairs, int cap) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs; p += (int64_t)gridDim.x * blockDim.x) {
        cand_base[p] = p * cap;
        cand_cap[p] = cap;
    }
}

// Pairs whose candidate count exceeds their slot (*count += such pairs).
__global__ void cand_overflow_kernel(const int32_t* n_cand, const int32_t* cand_cap, int64_t n_pairs,
                                     unsigned long long* count) {
    unsigned long long k = 0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs; p += (int64_t)gridDim.x * blockDim.x)
        k += n_cand[p] > cand_cap[p] ? 1 : 0;
    if (k) atomicAdd(count, k);
}

// Pruning of the traced pairs on the device (the host then reads only the
// pairs that pass).  Pair k = t * nq + sp (target-major, sp the query's sorted
// position) passes when its maximum reaches MINIMUM_SCORE and
// max(LOWER_LIMIT_SCORE * max, maxPossibleScore) -- the starting-point
// threshold of default_main.cu:596,609, maxPossibleScore =
// highest * min(len) * filter_factor in double precision, stored as fp32 as
// the reference's host does (SmithWatermanCuda._set_max_possible_score,
// SmithWatermanCuda.py:268-274) -- so that no pair without a starting point
// is swept.  flags[k] = pass; counts[0] += pairs
// reaching MINIMUM_SCORE, counts[1] += passing pairs.
__global__ void prune_kernel(const float* pair_max, const int32_t* q_order, const int32_t* q_len,
                             const int32_t* t_len, int nq, int nt, float minimum, double highest,
                             double filter_factor, float lower_limit, const uint8_t* q_trace, uint8_t* flags,
                             unsigned long long* counts) {
    const int64_t n = (int64_t)nq * nt;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long n_min = 0, n_pass = 0;
    unsigned pass_max = 0;  // largest maximum of a passing pair (counts[3])
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t k = base + threadIdx.x;
        bool m = false, pass = false;
        if (k < n) {
            const int t = (int)(k / nq), sp = (int)(k - (int64_t)t * nq);
            const int q = q_order[sp];
            const float mx = pair_max[(int64_t)q * nt + t];
            m = mx >= minimum;
            if (m) {
                const int mn = min(q_len[q], t_len[t]);
                const float pos = (float)(highest * (double)mn * filter_factor);
                const float llm = __fmul_rn(lower_limit, mx);
                // q_trace (null: every query): queries whose hits are wanted
                pass = mx >= fmaxf(llm, pos) && (q_trace == nullptr || q_trace[q] != 0);
                if (pass) pass_max = max(pass_max, __float2uint_rz(fminf(fmaxf(mx, 0.0f), 4.0e9f)));
            }
            flags[k] = pass ? 1 : 0;
        }
        const unsigned bm = __ballot_sync(0xffffffffu, m), bp = __ballot_sync(0xffffffffu, pass);
        if ((threadIdx.x & 31) == 0) {
            n_min += __popc(bm);
            n_pass += __popc(bp);
        }
    }
    pass_max = __reduce_max_sync(0xffffffffu, pass_max);
    if ((threadIdx.x & 31) == 0 && (n_min | n_pass)) {
        atomicAdd(&counts[0], n_min);
        atomicAdd(&counts[1], n_pass);
        atomicMax(&counts[3], (unsigned long long)pass_max);
    }
}

#endif  // PW_SCORE_SWEEP_ONLY

}  // namespace pw
