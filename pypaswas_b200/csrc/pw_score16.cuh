// pw_score16.cuh -- the 16-bit score sweep: two pairs per lane.
//
// Pair maxima only (the engine's first phase).  Every 32-bit register holds
// the same DP cell of two different pairs as signed 16-bit halves, and the
// recurrences run on the DPX 16x2 instructions (__viaddmax_s16x2 and friends),
// which update two cells per instruction at the rate of one 32-bit update.
// A warp aligns one "strip" sequence against up to 64 "lane" sequences: lane l
// carries lane sequences l and l + 32 of its work item (similar lengths, the
// lane list is sorted by length).  Which input set provides the strips and
// which the lanes is chosen per run by the host (pair maxima are symmetric in
// the two sequences, so either orientation gives the same maxima).
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

__device__ __forceinline__ uint32_t prmt_sign(uint32_t a, uint32_t b, uint32_t sel) {
#ifdef __CUDA_ARCH__
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
#else
    // PTX prmt, default mode: selector nibble n picks byte (n & 7) of {b, a};
    // with bit 3 set it replicates that byte's sign bit instead.
    const uint64_t v = ((uint64_t)b << 32) | a;
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) {
        const uint32_t n = (sel >> (4 * i)) & 0xf;
        uint32_t byte = (uint32_t)(v >> (8 * (n & 7))) & 0xff;
        if (n & 8) byte = (byte & 0x80) ? 0xff : 0;
        r |= byte << (8 * i);
    }
    return r;
#endif
}

// Scores of strip row k for the two pairs, as signed 16-bit halves: low half
// from pair A's profile word wa, high half from pair B's word wb.
__device__ __forceinline__ uint32_t pair_scores(uint32_t wa, uint32_t wb, int k) {
    const uint32_t sel = (uint32_t)k | ((8u | k) << 4) | ((4u + k) << 8) | ((12u + k) << 12);
    return prmt_sign(wa, wb, sel);
}

__device__ __forceinline__ uint32_t pack16(int v) { return ((uint32_t)v & 0xffffu) * 0x00010001u; }

struct Score16Args {
    const WorkItem* items;   // target = strip sequence, first/lanes index the lane order
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
};

template <int S, bool AFFINE>
__device__ __forceinline__ void sweep16(const uint8_t* qa, const uint8_t* qb, int lq4a, int lq4b, uint32_t pad4,
                                        const uint32_t* prof, int alpha1, int gap, int ext, int ge, bool has_up,
                                        bool has_down, uint4* bnd, uint32_t& mx) {
    const int lq4 = lq4a > lq4b ? lq4a : lq4b;
    const uint32_t g2 = pack16(gap), e2 = pack16(ext), ge2 = pack16(ge);
    if constexpr (!AFFINE) {
        uint32_t H[S];
#pragma unroll
        for (int r = 0; r < S; ++r) H[r] = 0;
        uint32_t hb_prev = 0;
        for (int x4 = 0; x4 < lq4; x4 += 4) {
            const uint32_t cwa = x4 < lq4a ? *(const uint32_t*)(qa + x4) : pad4;
            const uint32_t cwb = x4 < lq4b ? *(const uint32_t*)(qb + x4) : pad4;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cwa >> (8 * j)) & 0xff, b = (cwb >> (8 * j)) & 0xff;
                uint32_t up = has_up ? bnd[(int64_t)x * kWarp].x : 0u;
                uint32_t diag = hb_prev;
                hb_prev = up;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const uint32_t wa = prof[g * alpha1 + a], wb = prof[g * alpha1 + b];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t s = pair_scores(wa, wb, k);
                        const uint32_t left = H[r];
                        uint32_t t = __viaddmax_s16x2(diag, s, kNeg16x2);       // diag + s
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
        // strip-axis gap chain carried down the column (scalar), sweep-axis gap
        // chain and best score kept per row (arrays); see sweep_score
        uint32_t Ml[S], Xl[S], Bl[S];
#pragma unroll
        for (int r = 0; r < S; ++r) {
            Ml[r] = 0;
            Xl[r] = kNeg16x2;
            Bl[r] = 0;
        }
        uint32_t bb_prev = 0;
        for (int x4 = 0; x4 < lq4; x4 += 4) {
            const uint32_t cwa = x4 < lq4a ? *(const uint32_t*)(qa + x4) : pad4;
            const uint32_t cwb = x4 < lq4b ? *(const uint32_t*)(qb + x4) : pad4;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int x = x4 + j;
                const int a = (cwa >> (8 * j)) & 0xff, b = (cwb >> (8 * j)) & 0xff;
                uint32_t mup = 0, yup = kNeg16x2, bup = 0;
                if (has_up) {
                    const uint4 v = bnd[(int64_t)x * kWarp];
                    mup = v.x;
                    yup = v.y;
                    bup = v.z;
                }
                uint32_t bdiag = bb_prev;
                bb_prev = bup;
#pragma unroll
                for (int g = 0; g < S / 4; ++g) {
                    const uint32_t wa = prof[g * alpha1 + a], wb = prof[g * alpha1 + b];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int r = 4 * g + k;
                        const uint32_t s = pair_scores(wa, wb, k);
                        const uint32_t m = __viaddmax_s16x2_relu(bdiag, s, kNeg16x2);
                        const uint32_t y = __viaddmax_s16x2(yup, e2, __viaddmax_s16x2(mup, ge2, kNeg16x2));
                        const uint32_t xg = __viaddmax_s16x2(Xl[r], e2, __viaddmax_s16x2(Ml[r], ge2, kNeg16x2));
                        const uint32_t bst = __vimax3_s16x2(m, y, xg);
                        bdiag = Bl[r];
                        Ml[r] = m;
                        Xl[r] = xg;
                        Bl[r] = bst;
                        mup = m;
                        yup = y;
                    }
                }
#pragma unroll
                for (int r = 0; r < S; r += 2) mx = __vimax3_s16x2(mx, Bl[r], Bl[r + 1]);
                if (has_down) bnd[(int64_t)x * kWarp] = make_uint4(mup, yup, Bl[S - 1], 0u);
            }
        }
    }
}

template <int S, bool AFFINE, bool MULTI>
__global__ void __launch_bounds__(128) score16_kernel(Score16Args A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int prof_bytes = ((S / 4) * A.alpha1 * 4 + 15) & ~15;
    uint32_t* prof = (uint32_t*)(smem + wib * prof_bytes);
    const int64_t warp_global = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    uint4* bnd = MULTI ? A.bnd_pool + warp_global * A.bnd_slot + lane : nullptr;
    const uint32_t pad = (uint32_t)(A.alpha1 - 1);
    const uint32_t pad4 = pad * 0x01010101u;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(A.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= A.n_items) break;
        const WorkItem W = A.items[it];
        const int st = W.target;
        const int ls = A.strip_len[st];
        const bool has_a = lane < W.lanes, has_b = lane + kWarp < W.lanes;
        const int pa = has_a ? A.lane_order[W.first + lane] : 0;
        const int pb = has_b ? A.lane_order[W.first + lane + kWarp] : 0;
        const uint8_t* qa = A.lane_codes + A.lane_off[pa];
        const uint8_t* qb = A.lane_codes + A.lane_off[pb];
        const int lq4a = has_a ? (A.lane_len[pa] + 3) & ~3 : 0;
        const int lq4b = has_b ? (A.lane_len[pb] + 3) & ~3 : 0;
        const uint8_t* sres = A.strip_res + A.strip_off[st];
        const int nstrips = MULTI ? (ls + S - 1) / S : 1;
        uint32_t mx = 0;
        for (int s = 0; s < nstrips; ++s) {
            const int y0 = s * S;
            __syncwarp();
            build_profile<int, S>(prof, A.cmat, nullptr, sres, y0, ls, A.alpha1, A.dim, lane);
            __syncwarp();
            if (has_a)
                sweep16<S, AFFINE>(qa, qb, lq4a, lq4b, pad4, prof, A.alpha1, A.gap, A.ext, A.ge, s > 0,
                                   s + 1 < nstrips, bnd, mx);
        }
        const int ma = (int)(int16_t)(mx & 0xffffu), mb = (int)(int16_t)(mx >> 16);
        if (has_a)
            A.pair_max[(int64_t)st * A.stride_strip + (int64_t)pa * A.stride_lane] =
                ma >= kOvf16 ? __int_as_float(0x7fc00000) : (float)ma;
        if (has_b)
            A.pair_max[(int64_t)st * A.stride_strip + (int64_t)pb * A.stride_lane] =
                mb >= kOvf16 ? __int_as_float(0x7fc00000) : (float)mb;
    }
}

}  // namespace pw
