// pw_device.cuh -- device-side data layout and per-lane DP sweeps of the B200
// Smith-Waterman engine.
//
// Work decomposition ("inter-sequence" batching): one warp aligns one target
// against up to 32 queries, one query per lane.  The target is the strip axis:
// a lane keeps S consecutive target rows of its DP column in registers and
// sweeps the query positions (the reference's x axis) one column at a time.
// Target rows are processed in strips of S; the last row of a strip is handed
// to the next strip through a per-warp boundary buffer.  Substitution scores
// come from a per-warp strip profile in shared memory: for 4 consecutive target
// rows and one query residue, one 32-bit word holds the 4 scores (int8 each),
// so one shared-memory load feeds 4 cells.
//
// Arithmetic: the reference computes in fp32 (pyPaSWAS/Core/cuda/default_main.cu);
// when every score and penalty is an integer the engine computes in int32 and
// is bit-identical (all values are integers < 2^24, so fp32 adds and compares
// are exact).  Otherwise it computes in fp32 with the reference's operation
// order.  DPX instructions (__viaddmax_s32, __vimax3_s32, ...) carry the
// integer recurrence.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pw {

constexpr int kWarp = 32;
constexpr int kCandCap = 64;          // candidates stored per pair before overflow
constexpr int kNeg = -(1 << 28);       // stands in for AFFINE_GAP_INIT (-1e10f) in int32

// direction codes of the 4-bit cell code (bits 0-1)
constexpr uint8_t kNo = 0, kUL = 1, kUp = 2, kLeft = 3;
// flag bits of the cell code
constexpr uint8_t kStopFlag = 1u << 2;  // UL/MAIN cell whose diagonal predecessor is 0 (in matrix)
constexpr uint8_t kCand = 1u << 3;      // starting-point candidate (score >= threshold)
// (covered candidates and the walk's IN_ALIGNMENT marks are bits of a
// separate plane, see PairView in pw_kernels.cuh)

// Scoring constants shared by all kernels.
struct ScoreParams {
    int affine;
    int is_float;          // 0: int32 path, 1: fp32 path
    int gap_i, ext_i, ge_i;   // gap, ext, gap+ext as integers (int path)
    float gap_f, ext_f, ge_f; // as fp32 (ge_f = fl(gap + ext), folded like the reference)
    float lower_limit;
    float minimum_score;
    double host_minimum;
    double highest, filter_factor;
    int alpha;             // compact query alphabet size
    int dim;               // full matrix dimension (target residue range)
};

// One unit of phase-1 / phase-2 work: a target against up to 32 queries.
struct WorkItem {
    int32_t target;
    int32_t first;         // index into the sorted query order of lane 0
    int32_t lanes;         // number of queries (<= 32)
    int32_t xmax;          // longest query of the group (lane 0, sorted)
    int32_t index;         // position of the item in its wave (phase 2); 16-bit sweep: second strip
    int32_t S;             // strip height of the item's sweep
    int32_t orient;        // 0: targets are the strips, queries the lanes; 1: the reverse
    int32_t lanes_hi;      // 16-bit dual-lane sweep: lanes of the second group (sorted positions first + 32 ...)
    int64_t dir_base;      // byte offset of the group's cell codes (phase 2)
    int64_t pair_base;     // index of lane 0's per-pair slot (phase 2)
};

struct Cand {
    int32_t x, y;
    int32_t score_i;       // int path score
    float score_f;         // fp32 score (both paths)
};

struct PairMeta {          // phase-2 per-pair record
    int32_t query, target;
    int32_t item;          // work item index
    int32_t lane;
    int32_t n_cand;        // may exceed kCandCap (overflow)
    int32_t thr_i;         // integer candidate threshold (int path)
    float thr_f;           // fp32 candidate threshold
    float max_f;
};

struct DevHit {
    int32_t pair;          // phase-2 pair slot of the walk
    int32_t query, target;
    int32_t s_start, s_end, t_start, t_end;
    float score;
    int32_t matches, mismatches, n_cols;
    int32_t end_x, end_y;  // starting point of the walk (alignment end)
    int64_t ops_offset;
};

// Index of cell (x, y) of lane `lane` inside a group's code block.
// Layout: [strip][x][chunk of 16 rows][lane][16 cells]; cells are 4-bit codes,
// so one 8-byte store per lane and chunk makes each warp store a contiguous
// 256 bytes (the byte of cell i is i / 2).
template <int S>
__host__ __device__ __forceinline__ int64_t cell_offset(int x, int y, int lane, int xmax) {
    const int strip = y / S, r = y % S;
    return ((((int64_t)strip * xmax + x) * (S / 16) + r / 16) * kWarp + lane) * 16 + (r % 16);
}

__host__ __device__ __forceinline__ int64_t cell_offset_rt(int S, int x, int y, int lane, int xmax) {
    const int strip = y / S, r = y % S;
    return ((((int64_t)strip * xmax + x) * (S / 16) + r / 16) * kWarp + lane) * 16 + (r % 16);
}

// ---------------------------------------------------------------- arithmetic
__device__ __forceinline__ int sext_byte(uint32_t w, int k) {
    // sign-extend byte k of w
    return (int)(int8_t)(uint8_t)(w >> (8 * k));
}
__device__ __forceinline__ int addmax(int a, int b, int c) { return __viaddmax_s32(a, b, c); }
__device__ __forceinline__ int addmax_relu(int a, int b, int c) { return __viaddmax_s32_relu(a, b, c); }
__device__ __forceinline__ int max3(int a, int b, int c) { return __vimax3_s32(a, b, c); }
__device__ __forceinline__ float addmax(float a, float b, float c) { return fmaxf(a + b, c); }
__device__ __forceinline__ float max3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

}  // namespace pw
