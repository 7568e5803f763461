// pw_finish.cuh -- hit order and alignment strings on the device.
//
// The walk leaves its hits (DevHit) and their column operations ('M', 'I',
// 'D' per alignment column) in device memory, appended across memory waves.
// These kernels put the hits in the order the reference's HitList has them
// and spell out the three alignment strings of every hit, so that the host
// receives the final records in two copies.
//
// Order (SmithWaterman._print_alignments appends in the pinned emission
// order of the starting points and HitList sorts by score,
// SmithWaterman.py:699): score ascending; then block anti-diagonal
// descending, block x descending, target, query, cell anti-diagonal
// descending, row ascending; then walk order.  The key is packed into three
// 64-bit words (scores are >= 0, so their fp32 bits order like the values)
// and sorted by three stable radix passes, least significant word first,
// starting from the walk order, which gives the last tie-break.
#pragma once
#include "../../include/paswas_b200.h"
#include "pw_device.cuh"

namespace pw {

__global__ void hit_key_kernel(const DevHit* h, int64_t n, uint64_t* ka, uint64_t* kb, uint64_t* kc, int32_t* idx) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const DevHit d = h[k];
        const uint32_t sb = __float_as_uint(d.score);
        const uint32_t diag = (uint32_t)((d.end_x >> 3) + (d.end_y >> 3));
        const uint32_t small = (uint32_t)((d.end_x & 7) + (d.end_y & 7));
        ka[k] = ((uint64_t)sb << 32) | (0xFFFFFFFFu - diag);
        kb[k] = ((uint64_t)(0xFFFFFFFFu - (uint32_t)(d.end_x >> 3)) << 32) | (uint32_t)d.target;
        kc[k] = ((uint64_t)(uint32_t)d.query << 32) | ((uint64_t)(0xFFu - small) << 8) | (uint32_t)(d.end_y & 7);
        idx[k] = (int32_t)k;
    }
}

__global__ void gather_key_kernel(const uint64_t* src, const int32_t* idx, int64_t n, uint64_t* dst) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[idx[k]];
}

// String bytes of the hit at each sorted position (three strings of n_cols).
__global__ void hit_len_kernel(const DevHit* h, const int32_t* idx, int64_t n, int64_t* len) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        len[k] = 3 * (int64_t)h[idx[k]].n_cols;
}

// The hit records in order and their strings: sequence_match (query residue
// or '-'), alignment ('|' for equal residues -- letters compared without
// case -- '.' for a mismatch, ' ' in a gap) and target_match, one column per
// operation, as SmithWaterman._print_alignments spells them
// (SmithWaterman.py:765-815).
// Hits longer than kWarpStringCols columns get only their record here; a
// warp spells their strings (hit_strings_warp_kernel).
constexpr int kWarpStringCols = 512;

__global__ void hit_out_kernel(const DevHit* h, const int32_t* idx, const int64_t* soff, int64_t n, const char* ops,
                               const uint8_t* q_raw, const int64_t* q_off, const uint8_t* t_raw,
                               const int64_t* t_off, pw_hit* out, char* str) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const DevHit d = h[idx[k]];
        pw_hit o;
        o.query = d.query;
        o.target = d.target;
        o.s_start = d.s_start;
        o.s_end = d.s_end;
        o.t_start = d.t_start;
        o.t_end = d.t_end;
        o.score = d.score;
        o.matches = d.matches;
        o.mismatches = d.mismatches;
        o.n_cols = d.n_cols;
        o.str_offset = soff[k];
        out[k] = o;
        if (d.n_cols > kWarpStringCols) continue;
        char* sq = str + o.str_offset;
        char* al = sq + d.n_cols;
        char* tg = al + d.n_cols;
        const uint8_t* qs = q_raw + q_off[d.query];
        const uint8_t* ts = t_raw + t_off[d.target];
        const char* op = ops + d.ops_offset;
        int x = d.s_start, y = d.t_start;
        for (int i = 0; i < d.n_cols; ++i) {
            const char c = op[i];
            if (c == 'M') {
                const uint8_t ca = ts[y], cb = qs[x];
                const bool la = (ca >= 'A' && ca <= 'Z') || (ca >= 'a' && ca <= 'z');
                const bool eq = la ? ((ca | 0x20) == (cb | 0x20)) : ca == cb;
                sq[i] = (char)cb;
                tg[i] = (char)ca;
                al[i] = eq ? '|' : '.';
                ++x;
                ++y;
            } else if (c == 'I') {
                sq[i] = (char)qs[x];
                tg[i] = '-';
                al[i] = ' ';
                ++x;
            } else {
                sq[i] = '-';
                tg[i] = (char)ts[y];
                al[i] = ' ';
                ++y;
            }
        }
    }
}

// The strings of the long hits, one warp per hit and 32 columns per step:
// the query / target position of every column is the starting position plus
// an exclusive warp scan of the columns that consume a query residue ('M',
// 'I') or a target residue ('M', 'D'); the characters are those of
// hit_out_kernel.
__global__ void hit_strings_warp_kernel(const DevHit* h, const int32_t* idx, const int64_t* soff, int64_t n,
                                        const char* ops, const uint8_t* q_raw, const int64_t* q_off,
                                        const uint8_t* t_raw, const int64_t* t_off, char* str) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp; k < n; k += warps) {
        {
            const DevHit d = h[idx[k]];
            if (d.n_cols <= kWarpStringCols) continue;
            char* sq = str + soff[k];
            char* al = sq + d.n_cols;
            char* tg = al + d.n_cols;
            const uint8_t* qs = q_raw + q_off[d.query];
            const uint8_t* ts = t_raw + t_off[d.target];
            const char* op = ops + d.ops_offset;
            int x = d.s_start, y = d.t_start;
            for (int c0 = 0; c0 < d.n_cols; c0 += 32) {
                const int i = c0 + lane;
                const bool act = i < d.n_cols;
                const char c = act ? op[i] : 'M';
                const int dx = act && c != 'D' ? 1 : 0, dy = act && c != 'I' ? 1 : 0;
                int sx = dx, sy = dy;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int tx = __shfl_up_sync(0xffffffffu, sx, off), ty = __shfl_up_sync(0xffffffffu, sy, off);
                    if (lane >= off) {
                        sx += tx;
                        sy += ty;
                    }
                }
                if (act) {
                    const int px = x + sx - dx, py = y + sy - dy;
                    if (c == 'M') {
                        const uint8_t ca = ts[py], cb = qs[px];
                        const bool la = (ca >= 'A' && ca <= 'Z') || (ca >= 'a' && ca <= 'z');
                        const bool eq = la ? ((ca | 0x20) == (cb | 0x20)) : ca == cb;
                        sq[i] = (char)cb;
                        tg[i] = (char)ca;
                        al[i] = eq ? '|' : '.';
                    } else if (c == 'I') {
                        sq[i] = (char)qs[px];
                        tg[i] = '-';
                        al[i] = ' ';
                    } else {
                        sq[i] = '-';
                        tg[i] = (char)ts[py];
                        al[i] = ' ';
                    }
                }
                x += __shfl_sync(0xffffffffu, sx, 31);
                y += __shfl_sync(0xffffffffu, sy, 31);
            }
        }
    }
}

}  // namespace pw
