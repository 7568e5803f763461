// engine.cu -- C ABI (include/paswas_b200.h) and host orchestration of the
// B200 Smith-Waterman engine.
//
// pw_align runs the reference's path in three device phases:
//   1. score   -- every (query, target) pair, pair maxima only
//   2. trace   -- pairs whose maximum reached MINIMUM_SCORE: cell codes and
//                 starting-point candidates, then starting points (collect)
//   3. walk    -- the host walk of the reference on the device, then the
//                 column operations of each kept hit
// The host only builds work lists, sizes memory waves and formats results.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <map>
#include <atomic>
#include <numeric>
#include <queue>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/paswas_b200.h"
#include "pw_kernels.cuh"
#include "pw_score16.cuh"
#include "pw_band.cuh"
#include "pw_tiles.cuh"
#include "pw_band16.cuh"
#include "pw_plan.h"
#include "pw_finish.cuh"
#include "pw_host.h"

using namespace pw;

#ifndef PW_LAUNCH
#define PW_LAUNCH(kern, grid, block, smem, stream, ...) kern<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__)
#endif

static double wall_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Host-phase timing on stderr when the environment sets PW_HOST_TRACE
// (diagnostics of the host orchestration between kernels; off by default).
struct HostTrace {
    bool on;
    double t;
    HostTrace() : on(std::getenv("PW_HOST_TRACE") != nullptr), t(wall_ms()) {}
    void mark(const char* what) {
        if (!on) return;
        const double n = wall_ms();
        std::fprintf(stderr, "[pw host] %-34s %10.3f ms\n", what, n - t);
        t = n;
    }
};


// Host array in page-locked memory when the driver grants it (faster device
// copies of large results such as the pair maxima), else in ordinary memory.
template <typename T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    bool pinned = false;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { release(); }
    void release() {
        if (p) {
            if (pinned)
                cudaFreeHost(p);
            else
                free(p);
        }
        p = nullptr;
        n = cap = 0;
    }
    bool resize(size_t m) {  // contents are not kept
        if (m > cap) {
            release();
            const size_t want = std::max<size_t>(m, 1);
            pinned = cudaMallocHost((void**)&p, want * sizeof(T)) == cudaSuccess;
            if (!pinned) {
                cudaGetLastError();
                p = (T*)malloc(want * sizeof(T));
                if (!p) return false;
            }
            cap = want;
        }
        n = m;
        return true;
    }
    bool resize_keep(size_t m) {  // contents [0, min(n, m)) are kept; capacity grows by half
        if (m > cap) {
            const size_t want = std::max<size_t>(m, cap + cap / 2);
            T* q = nullptr;
            bool pin = cudaMallocHost((void**)&q, want * sizeof(T)) == cudaSuccess;
            if (!pin) {
                cudaGetLastError();
                q = (T*)malloc(want * sizeof(T));
                if (!q) return false;
            }
            if (n) std::memcpy(q, p, n * sizeof(T));
            const size_t keep = n;
            release();
            p = q;
            pinned = pin;
            cap = want;
            n = keep;
        }
        n = m;
        return true;
    }
    void clear() { n = 0; }
    bool empty() const { return n == 0; }
    void fill(T v) { std::fill(p, p + n, v); }
    size_t size() const { return n; }
    T* data() { return p; }
    const T* data() const { return p; }
    T& operator[](size_t i) { return p[i]; }
    const T& operator[](size_t i) const { return p[i]; }
};

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Stream-ordered growth (cudaFreeAsync / cudaMallocAsync on the engine's
    // stream, from the device's memory pool, which keeps freed blocks): unlike
    // cudaFree, nothing here synchronises the device, so a growing buffer
    // never stalls other engines (the serving loop's workers).  Grows by half
    // again (small buffers double) so that slightly larger calls reuse it.
    cudaError_t reserve(cudaStream_t st, size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) {
            cudaError_t e = cudaFreeAsync(p, st);
            if (e != cudaSuccess) return e;
            p = nullptr;
            bytes = 0;
        }
        size_t want = n ? n : 16;
        want = want < (1u << 20) ? 2 * want : want + want / 2;
        cudaError_t e = cudaMallocAsync(&p, want, st);
        if (e == cudaErrorMemoryAllocation) {  // retry at the exact size
            cudaGetLastError();
            want = n ? n : 16;
            e = cudaMallocAsync(&p, want, st);
        }
        if (e == cudaSuccess) bytes = want;
        else p = nullptr;
        return e;
    }
    // Growth that keeps the first `used` bytes (stream-ordered copy into the
    // new block), for buffers appended to across memory waves.
    cudaError_t grow_keep(cudaStream_t st, size_t used, size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        size_t want = std::max<size_t>(n, bytes + bytes / 2);
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, want, st);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            want = n;
            e = cudaMallocAsync(&q, want, st);
        }
        if (e != cudaSuccess) return e;
        if (p && used && (e = cudaMemcpyAsync(q, p, used, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
        if (p && (e = cudaFreeAsync(p, st)) != cudaSuccess) return e;
        p = q;
        bytes = want;
        return cudaSuccess;
    }
    template <typename T>
    T* as() const { return (T*)p; }
};

struct HostSeqs {
    std::vector<uint8_t> raw;
    std::vector<int64_t> off;
    std::vector<int32_t> key;
    int32_t n = 0;
    bool set = false;
};

struct Prepared {
    int alpha = 0;               // distinct query residues
    int alpha_t = 0;             // distinct target residues
    bool int_path = true;
    bool s16_q = false;          // 16-bit sweep possible with queries on the lanes
    bool s16_t = false;          // ... with targets on the lanes
    std::vector<int32_t> order;  // query indices by length, longest first
    std::vector<int32_t> order_t;  // target indices by length, longest first
    std::vector<int32_t> qlen, tlen;
    int64_t maxlq = 0, maxlt = 0;
    float maxabs = 0.0f;         // largest |score| over the query residues' rows
    bool q_int8 = true;          // query rows: integers in [-127, 127]
    bool t_int8 = true;          // transposed target rows: the same
};


}  // namespace

struct pw_engine {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string err;
    // scoring
    bool scoring_set = false;
    std::vector<float> matrix;
    int dim = 0, char_offset = 0;
    float gap = 0, ext = 0, lower_limit = 0, minimum_score = 0;
    int affine = 0;
    double host_minimum = 0, highest = 0, filter_factor = 0;
    // sequences
    HostSeqs Q, T;
    // device buffers
    DevBuf q_codes, q_code_off, q_raw, q_raw_off, q_len, q_key, q_order;
    DevBuf t_codes, t_code_off, t_raw, t_raw_off, t_len, t_key;
    DevBuf q_res, t_ccodes, t_order, cmat_t8, cmat_tf;  // the other orientation's encodings
    DevBuf cmat_i8, cmat_f, pair_max, items, items_alt, counter, bnd_pool, q_order2;
    DevBuf band_pairs, band_entries, band_prog, band_max, band_ring, band_out;  // band sweep (pw_band.cuh)
    DevBuf tile_ck, tile_marks, tile_pairs, slot_tile;                        // tile form (pw_tiles.cuh)
    DevBuf tile_pairs_alt, tile_sel, tile_cnt, tile_acc, tile_scratch, tile_ops;
    DevBuf band_over;                                                         // band16_kernel: pairs past 16 bits
    // explicit pairs: the score sweep's tile-form checkpoints (band_kernel<false, 4>)
    DevBuf p1_ck;
    bool p1_tiles = false;
    int64_t p1_free = 0;
    double p1_free_t = -1.0;
    std::vector<int64_t> p1_ck_off, p1_tm_off;           // per listed pair
    std::unordered_map<int64_t, int32_t> p1_index;        // query * nt + target -> listed pair
    DevBuf scan_tmp;  // CUB scan / select scratch
    DevBuf prune_flags, prune_cnt, prune_sel, t_skip, q_count;  // phase-2 pruning on the device
    // hits and column operations of all memory waves, then their order and strings
    DevBuf acc_hits, acc_ops, fk_a, fk_b, fk_c, fk_t, fk_g, fi_a, fi_b, f_len, f_soff, f_out, f_str;
    HostBuf<int64_t> h_sel;
    HostBuf<int32_t> h_ptq, h_p2order;  // phase-2 pair lists (kept across calls: no page faults, no zero fill)
    HostBuf<uint8_t> h_qc, h_qres;      // query encodings staged for upload (page-locked, kept across calls)
    HostBuf<uint8_t> h_stage;           // page-locked staging of the other per-set uploads (Staged)
    int64_t free_mem = 0;    // free device memory plus this engine's kept wave buffers, as last queried
    double free_mem_t = -1;  // wall_ms() of that query
    DevBuf chain_items, chain_info, chain_prog, chain_max, chain_ring_off, chain_ring, chain_abort, p1_items, p1_grid;
    // plan of the 16-bit score phase (work items, classes, chain queue), kept
    // on the device and reused while inputs, scoring, flags and tuning stay
    struct {
        bool valid = false;
        int64_t qg = 0, tg = 0, sg = 0, tune = 0, share = 0, dual_mode = 0;
        uint32_t flags = 0;
        bool trans = false, chained = false, dual = false;
        int begin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int xm_multi = 4;
        int n_chain_items = 0;
        // grid form: one-strip classes as strip-pair lists (p1_grid) x lane groups
        bool grid = false;
        int gbegin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int n_groups = 0;
    } p1;
    DevBuf codes, marks, metas, cands, cands_alt, cand_base, cand_cap, n_cand, n_starts, start_off, starts, hits,
        hit_count, ops, allowed;
    // prepared (device-resident) inputs
    Prepared pr;
    int64_t q_gen = 1, t_gen = 1, s_gen = 1;      // inputs: queries, targets, scoring
    int64_t prep_q[2] = {0, 0}, prep_t[2] = {0, 0};  // (sequence gen, scoring gen) last prepared
    int64_t wave_limit = 0;                          // cell-code bytes per memory wave (0: automatic)
    std::vector<int32_t> pair_q, pair_t;             // pw_set_pairs: explicit (query, target) pairs
    bool q_trace_set = false;                        // pw_set_query_trace: a mask is on the device
    DevBuf q_trace;                                  // per query: 1 traced, 0 maxima only
    int64_t tune[16] = {};                           // pw_set_tuning values (0: automatic)
    // results
    HostBuf<float> h_pair_max;
    bool pm_stale = false;  // h_pair_max lags the device maxima (copied on pw_get_pair_max)
    HostBuf<pw_hit> h_hits;
    HostBuf<char> h_strings;
    HostBuf<StartRec> h_starts;
    int64_t launches = 0;
    int64_t h2d = 0, d2h = 0;  // bytes copied by the current pw_align
    int32_t reuse = 0;         // PW_REUSE_* bits of the current pw_align
    std::vector<int4> h_chain_info;  // the chained queue's (chain, strip, pred) entries, host copy
    DevBuf stall_buf;          // PW_TUNE_STALL_TEST: the queue with one entry re-pointed at a silent flag
};

// Resident-block budget of this engine's persistent kernels: all SMs' worth,
// or the share set with PW_TUNE_GRID_SHARE (thousandths), so that the kernels
// of several engines (the serving loop's workers) can be resident together.
static int grid_cap(const pw_engine* e, int per_sm) {
    const int64_t share = e->tune[PW_TUNE_GRID_SHARE];
    const int64_t full = (int64_t)e->sm_count * std::max(1, per_sm);
    if (share <= 0 || share >= 1000) return (int)full;
    return (int)std::max<int64_t>(1, full * share / 1000);
}

// Bound of one chain or band wait (PW_TUNE_WAIT_NS, else kChainWaitNs).
static unsigned long long wait_limit(const pw_engine* e) {
    const int64_t v = e->tune[PW_TUNE_WAIT_NS];
    return v > 0 ? (unsigned long long)v : kChainWaitNs;
}

static int fail(pw_engine* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    return code;
}

static int cuda_fail(pw_engine* e, cudaError_t c, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(c);
    int code = (c == cudaErrorMemoryAllocation) ? PW_ERR_NOMEM : PW_ERR_KERNEL;
    return fail(e, code, m);
}

// Host <-> device copies on the engine's stream, counted for pw_run_info.
static cudaError_t copy_h2d(pw_engine* e, void* dst, const void* src, size_t n) {
    e->h2d += (int64_t)n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, e->stream);
}

static cudaError_t copy_d2h(pw_engine* e, void* dst, const void* src, size_t n) {
    e->d2h += (int64_t)n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, e->stream);
}

#define PW_CUDA(call, what)                                   \
    do {                                                      \
        cudaError_t _c = (call);                              \
        if (_c != cudaSuccess) return cuda_fail(e, _c, what); \
    } while (0)

extern "C" int pw_create(int device, pw_engine** out) {
    if (!out) return PW_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return PW_ERR_DEVICE;
    if (device < 0 || device >= n) return PW_ERR_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PW_ERR_DEVICE;
    if (prop.major < 10) return PW_ERR_DEVICE;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return PW_ERR_DEVICE;
    pw_engine* e = new pw_engine();
    e->device = device;
    e->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return PW_ERR_DEVICE;
    }
    for (auto& ev : e->ev) cudaEventCreate(&ev);
    // keep freed blocks in the device's pool for reuse (stream-ordered growth)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = e;
    return PW_OK;
}

extern "C" void pw_destroy(pw_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (auto& ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

extern "C" const char* pw_last_error(pw_engine* e) { return e ? e->err.c_str() : "no engine"; }

extern "C" int pw_device_free_memory(pw_engine* e, int64_t* free_bytes, int64_t* total_bytes) {
    if (!e) return PW_ERR_ARG;
    cudaSetDevice(e->device);
    size_t f = 0, t = 0;
    PW_CUDA(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
    if (free_bytes) *free_bytes = (int64_t)f;
    if (total_bytes) *total_bytes = (int64_t)t;
    return PW_OK;
}

extern "C" int pw_set_scoring(pw_engine* e, const float* matrix, int dim, int char_offset, float gap, float ext,
                              int affine, float lower_limit, float minimum_score, double host_minimum,
                              double highest, double filter_factor) {
    if (!e) return PW_ERR_ARG;
    if (!matrix || dim <= 0 || dim > 256) return fail(e, PW_ERR_ARG, "scoring matrix dimension must be 1..256");
    if (char_offset < 0 || char_offset + dim > 256) return fail(e, PW_ERR_ARG, "char_offset + dim exceeds 256");
    if (!(gap <= 0.0f) || (affine && !(ext <= 0.0f)))
        return fail(e, PW_ERR_ARG, "gap penalties must be <= 0");
    for (int i = 0; i < dim * dim; ++i)
        if (!std::isfinite(matrix[i])) return fail(e, PW_ERR_ARG, "scoring matrix holds a non-finite value");
    e->matrix.assign(matrix, matrix + (size_t)dim * dim);
    e->dim = dim;
    e->char_offset = char_offset;
    e->gap = gap;
    e->ext = affine ? ext : 0.0f;
    e->affine = affine ? 1 : 0;
    e->lower_limit = lower_limit;
    e->minimum_score = minimum_score;
    e->host_minimum = host_minimum;
    e->highest = highest;
    e->filter_factor = filter_factor;
    e->scoring_set = true;
    e->s_gen++;
    return PW_OK;
}

// The residues as the engine keeps them: ASCII letters upper-cased (the
// reference upper-cases every sequence before its kernels see it), on host
// threads.  Returns whether dst already held exactly that.
static bool copy_upper(std::vector<uint8_t>& dst, const uint8_t* src, int64_t n) {
    const bool same_size = (int64_t)dst.size() == n;
    std::atomic<bool> differ{!same_size};
    if (!same_size) dst.resize((size_t)n);
    parallel_for(n, [&](int64_t i0, int64_t i1) {
        uint8_t* d = dst.data();
        bool diff = false;
        for (int64_t i = i0; i < i1; ++i) {
            const uint8_t c = src[i];
            const uint8_t u = (uint8_t)(c - (((uint8_t)(c - 'a') < 26u) ? 32 : 0));
            diff |= d[i] != u;
            d[i] = u;
        }
        if (diff) differ.store(true, std::memory_order_relaxed);
    }, (int64_t)1 << 22);
    return !differ.load();
}

static int set_seqs(pw_engine* e, HostSeqs& S, const uint8_t* residues, const int64_t* offsets, int32_t n,
                    const int32_t* id_keys) {
    if (!e) return PW_ERR_ARG;
    if (n < 0 || (n > 0 && (!offsets || !id_keys))) return fail(e, PW_ERR_ARG, "bad sequence arguments");
    if (n > 0 && offsets[0] != 0) return fail(e, PW_ERR_ARG, "offsets must start at 0");
    for (int32_t i = 0; i < n; ++i) {
        const int64_t len = offsets[i + 1] - offsets[i];
        if (len < 0) return fail(e, PW_ERR_ARG, "offsets must be non-decreasing");
        if (len > (1 << 24)) return fail(e, PW_ERR_ARG, "sequence longer than 16M residues");
    }
    const int64_t total = n > 0 ? offsets[n] : 0;
    if (total > 0 && !residues) return fail(e, PW_ERR_ARG, "residues missing");
    // the same set again (a resident database handed in once more): keep the
    // device copy
    const bool same_raw = copy_upper(S.raw, residues, total);
    if (S.set && S.n == n && same_raw && S.off.size() == (size_t)(n > 0 ? n + 1 : 1) &&
        (n == 0 || (std::memcmp(S.off.data(), offsets, (size_t)(n + 1) * sizeof(int64_t)) == 0 &&
                    std::memcmp(S.key.data(), id_keys, (size_t)n * sizeof(int32_t)) == 0)))
        return PW_OK;
    S.off.assign(offsets, offsets + (n > 0 ? n + 1 : 0));
    if (n == 0) S.off.assign(1, 0);
    S.key.assign(id_keys, id_keys + n);
    S.n = n;
    S.set = true;
    (&S == &e->Q ? e->q_gen : e->t_gen)++;
    return PW_OK;
}

extern "C" int pw_set_queries(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                              const int32_t* id_keys) {
    if (e) e->q_trace_set = false;  // a trace mask belongs to one pw_set_queries
    return set_seqs(e, e->Q, residues, offsets, n, id_keys);
}

extern "C" int pw_set_targets(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                              const int32_t* id_keys) {
    return set_seqs(e, e->T, residues, offsets, n, id_keys);
}

namespace {

// Strip classes: one-strip sweeps of 16, 32, 48 (linear) and 64 (linear)
// rows, and multi-strip items of 32-row strips; the 16-bit score sweep also
// has one-strip classes of 24 and 40 (linear) rows (its strips need a
// multiple of 4 rows, the cell-code layout of the other sweeps 16).
enum SClass { kS16 = 0, kS32 = 1, kS64 = 2, kS32Multi = 3, kS48 = 4, kS24 = 5, kS40 = 6, kNumClasses = 7 };

int class_S(int c) {
    switch (c) {
        case kS16: return 16;
        case kS24: return 24;
        case kS40: return 40;
        case kS48: return 48;
        case kS64: return 64;
        default: return 32;
    }
}

int pick_class(int lt, bool affine) {
    if (lt <= 16) return kS16;
    if (lt <= 32) return kS32;
    if (!affine && lt <= 48) return kS48;
    if (!affine && lt <= 64) return kS64;
    return kS32Multi;
}

// The 16-bit score sweep's class of a strip pair whose longer strip has lt rows.
int pick_class16(int lt, bool affine) {
    if (lt > 16 && lt <= 24) return kS24;
    if (!affine && lt > 32 && lt <= 40) return kS40;
    return pick_class(lt, affine);
}

int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

template <typename T, int S, bool AFF, bool MULTI, int PH, bool TR>
cudaError_t launch_sweep(pw_engine* e, KernelArgs A, int* counter) {
    auto kern = sweep_kernel<T, S, AFF, MULTI, PH, TR>;
    const int alpha1 = A.P.alpha + 1;
    const int prof_bytes = ((S / 4) * alpha1 * (std::is_integral<T>::value ? 4 : 16) + 15) & ~15;
    const int smem = 4 * prof_bytes;
    if (smem > 48 * 1024) {
        cudaError_t c = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (c != cudaSuccess) return c;
    }
    int per_sm = 0;
    cudaError_t c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
    if (c != cudaSuccess) return c;
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 16) per_sm = 16;
    int grid = grid_cap(e, per_sm);
    const int need = (A.n_items + 3) / 4;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    A.item_counter = counter;
    PW_LAUNCH(kern, grid, 128, smem, e->stream, A);
    e->launches++;
    return cudaGetLastError();
}

template <typename T, int PH, bool TR>
cudaError_t launch_class_o(pw_engine* e, int cls, bool affine, const KernelArgs& A, int* counter) {
    if constexpr (PH == 3) {  // H store: linear gap, int lanes only
        switch (cls) {
            case kS16: return launch_sweep<int, 16, false, false, 3, TR>(e, A, counter);
            case kS32: return launch_sweep<int, 32, false, false, 3, TR>(e, A, counter);
            case kS48: return launch_sweep<int, 48, false, false, 3, TR>(e, A, counter);
            case kS64: return launch_sweep<int, 64, false, false, 3, TR>(e, A, counter);
            default: return launch_sweep<int, 32, false, true, 3, TR>(e, A, counter);
        }
    } else {
        if (affine) {
            switch (cls) {
                case kS16: return launch_sweep<T, 16, true, false, PH, TR>(e, A, counter);
                case kS32: return launch_sweep<T, 32, true, false, PH, TR>(e, A, counter);
                default: return launch_sweep<T, 32, true, true, PH, TR>(e, A, counter);
            }
        }
        switch (cls) {
            case kS16: return launch_sweep<T, 16, false, false, PH, TR>(e, A, counter);
            case kS32: return launch_sweep<T, 32, false, false, PH, TR>(e, A, counter);
            case kS48: return launch_sweep<T, 48, false, false, PH, TR>(e, A, counter);
            case kS64: return launch_sweep<T, 64, false, false, PH, TR>(e, A, counter);
            default: return launch_sweep<T, 32, false, true, PH, TR>(e, A, counter);
        }
    }
}

// Phase 1 never needs the transposed form (maxima are orientation-free).
template <typename T, int PH>
cudaError_t launch_class(pw_engine* e, int cls, bool affine, const KernelArgs& A, int* counter, bool trans) {
    if (PH >= 2 && trans) return launch_class_o<T, PH, true>(e, cls, affine, A, counter);
    return launch_class_o<T, PH, false>(e, cls, affine, A, counter);
}

}  // namespace

template <typename HT>
static cudaError_t upload(pw_engine* e, DevBuf& b, const HostBuf<HT>& v) {
    cudaError_t c = b.reserve(e->stream, std::max<size_t>(v.size() * sizeof(HT), 16));
    if (c != cudaSuccess) return c;
    if (v.empty()) return cudaSuccess;
    return copy_h2d(e, b.p, v.data(), v.size() * sizeof(HT));
}

template <typename HT>
static cudaError_t upload(pw_engine* e, DevBuf& b, const std::vector<HT>& v) {
    cudaError_t c = b.reserve(e->stream, std::max<size_t>(v.size() * sizeof(HT), 16));
    if (c != cudaSuccess) return c;
    if (v.empty()) return cudaSuccess;
    return copy_h2d(e, b.p, v.data(), v.size() * sizeof(HT));
}

static cudaError_t download(pw_engine* e, HostBuf<float>& v, const void* src, size_t n) {
    if (!v.resize(n)) return cudaErrorMemoryAllocation;
    if (!n) return cudaSuccess;
    cudaError_t c = copy_d2h(e, v.data(), src, n * sizeof(float));
    if (c != cudaSuccess) return c;
    return cudaStreamSynchronize(e->stream);
}

// Brings the host copy of the pair maxima up to date (the batched sweeps
// leave them on the device, where pruning and the trace kernels read them).
static int sync_pair_max(pw_engine* e, const float* dev) {
    if (!e->pm_stale) return PW_OK;
    cudaError_t c;
    if ((c = download(e, e->h_pair_max, dev, e->h_pair_max.size())) != cudaSuccess ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "copy pair maxima");
    e->pm_stale = false;
    return PW_OK;
}

template <typename HT>
static cudaError_t download(pw_engine* e, std::vector<HT>& v, const void* src, size_t n) {
    v.resize(n);
    if (!n) return cudaSuccess;
    cudaError_t c = copy_d2h(e, v.data(), src, n * sizeof(HT));
    if (c != cudaSuccess) return c;
    return cudaStreamSynchronize(e->stream);
}

// The uploads of one sequence set, gathered into the engine's page-locked
// staging buffer and copied asynchronously (a pageable source makes every
// cudaMemcpyAsync a synchronous staged copy of its own); the caller
// synchronises the stream before the staging buffer is reused.
struct Staged {
    struct Item {
        DevBuf* dst;
        const void* src;
        size_t bytes;
    };
    std::vector<Item> items;
    template <typename V>
    void add(DevBuf& b, const V& v) {
        items.push_back({&b, v.data(), v.size() * sizeof(v[0])});
    }
    cudaError_t run(pw_engine* e) {
        size_t total = 0;
        for (const Item& it : items) total += (it.bytes + 15) & ~(size_t)15;
        if (!e->h_stage.resize(std::max<size_t>(total, 16))) return cudaErrorMemoryAllocation;
        size_t off = 0;
        for (const Item& it : items) {
            cudaError_t c = it.dst->reserve(e->stream, std::max<size_t>(it.bytes, 16));
            if (c != cudaSuccess) return c;
            if (it.bytes) {
                std::memcpy(e->h_stage.data() + off, it.src, it.bytes);
                if ((c = copy_h2d(e, it.dst->p, e->h_stage.data() + off, it.bytes)) != cudaSuccess) return c;
            }
            off += (it.bytes + 15) & ~(size_t)15;
        }
        return cudaSuccess;
    }
};

// The byte values present in data[0, n), ascending (chunks marked on host
// threads, without branches).  The compact alphabets number them in this
// order; any numbering gives the same scores.
static std::vector<int> present_bytes(const uint8_t* data, int64_t n) {
    std::vector<std::vector<uint8_t>> marks;
    std::mutex mu;
    parallel_for(n, [&](int64_t b0, int64_t b1) {
        std::vector<uint8_t> m(256, 0);
        for (int64_t k = b0; k < b1; ++k) m[data[k]] = 1;
        std::lock_guard<std::mutex> g(mu);
        marks.push_back(std::move(m));
    }, (int64_t)1 << 20);
    std::vector<int> out;
    for (int c = 0; c < 256; ++c) {
        bool any = false;
        for (auto& m : marks) any = any || m[c];
        if (any) out.push_back(c);
    }
    return out;
}

// Builds the device copies of the sequences, the compact query alphabet and the
// compact substitution matrices.  Targets and queries are prepared separately
// and cached: a target database stays resident on the device while query sets
// come and go, and nothing is uploaded again while the sequences and the
// scoring model are unchanged.
static int prepare_targets(pw_engine* e) {
    if (e->prep_t[0] == e->t_gen && e->prep_t[1] == e->s_gen) {
        e->reuse |= PW_REUSE_TARGETS;
        return PW_OK;
    }
    const HostSeqs& T = e->T;
    const int off = e->char_offset, dim = e->dim;
    Prepared& pr = e->pr;
    // the byte values present (host threads)
    const std::vector<int> present = present_bytes(T.raw.data(), (int64_t)T.raw.size());
    {
        // the first invalid residue of the input is reported
        int64_t bad_at = INT64_MAX;
        int bad = -1;
        for (int c : present)
            if (c == 0 || c < off || c >= off + dim) {
                const int64_t at = (int64_t)(std::find(T.raw.begin(), T.raw.end(), (uint8_t)c) - T.raw.begin());
                if (at < bad_at) {
                    bad_at = at;
                    bad = c;
                }
            }
        if (bad >= 0)
            return fail(e, PW_ERR_ARG, "target residue outside the scoring matrix: code " + std::to_string(bad));
    }
    pr.tlen.assign(T.n, 0);
    pr.maxlt = 0;
    for (int32_t i = 0; i < T.n; ++i)
        pr.maxlt = std::max<int64_t>(pr.maxlt, pr.tlen[i] = (int32_t)(T.off[i + 1] - T.off[i]));
    // targets: matrix residue index, each sequence 16-byte aligned
    std::vector<int64_t> tco(T.n + 1, 0);
    int64_t pos = 0;
    for (int32_t i = 0; i < T.n; ++i) {
        tco[i] = pos;
        pos += align_up(std::max<int64_t>(pr.tlen[i], 1), 16);
    }
    tco[T.n] = pos;
    // the transposed orientation: targets on the lanes in a compact target
    // alphabet, with the matrix transposed to [target residue][query residue]
    int tmap[256];
    for (int i = 0; i < 256; ++i) tmap[i] = -1;
    std::vector<int> talpha;
    for (int c : present) {
        tmap[c] = (int)talpha.size();
        talpha.push_back(c);
    }
    pr.alpha_t = (int)talpha.size();
    std::vector<uint8_t> tc((size_t)std::max<int64_t>(pos, 16), 0);
    std::vector<uint8_t> tcc(tc.size(), (uint8_t)pr.alpha_t);
    parallel_for(T.n, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            const uint8_t* r = T.raw.data() + T.off[i];
            for (int32_t k = 0; k < pr.tlen[i]; ++k) {
                tc[tco[i] + k] = (uint8_t)(r[k] - off);
                tcc[tco[i] + k] = (uint8_t)tmap[r[k]];
            }
        }
    }, (int64_t)64);
    {
        std::vector<uint64_t> key((size_t)T.n);
        for (int32_t i = 0; i < T.n; ++i) key[i] = (uint64_t)(pr.maxlt - pr.tlen[i]);
        const std::vector<uint32_t> o = radix_order(std::move(key));
        pr.order_t.assign(o.begin(), o.end());
    }
    std::vector<int8_t> cmt8((size_t)(pr.alpha_t + 1) * dim, (int8_t)-128);
    std::vector<float> cmtf((size_t)(pr.alpha_t + 1) * dim, -1.0e30f);
    bool t_int8 = pr.alpha_t <= 250;
    for (int b = 0; b < pr.alpha_t; ++b)
        for (int j = 0; j < dim; ++j) {
            const float v = e->matrix[(size_t)j * dim + (talpha[b] - off)];
            if (std::floor(v) != v || v < -127.0f || v > 127.0f) t_int8 = false;
            cmt8[(size_t)b * dim + j] = (int8_t)(t_int8 ? v : 0);
            cmtf[(size_t)b * dim + j] = v;
        }
    pr.t_int8 = t_int8;
    cudaError_t c;
    Staged st;
    st.add(e->t_codes, tc);
    st.add(e->t_code_off, tco);
    st.add(e->t_raw, T.raw);
    st.add(e->t_raw_off, T.off);
    st.add(e->t_len, pr.tlen);
    st.add(e->t_key, T.key);
    st.add(e->t_ccodes, tcc);
    st.add(e->t_order, pr.order_t);
    st.add(e->cmat_t8, cmt8);
    st.add(e->cmat_tf, cmtf);
    if ((c = st.run(e)) != cudaSuccess || (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "upload targets");
    e->prep_t[0] = e->t_gen;
    e->prep_t[1] = e->s_gen;
    return PW_OK;
}

static int prepare_queries(pw_engine* e) {
    if (e->prep_q[0] == e->q_gen && e->prep_q[1] == e->s_gen) {
        e->reuse |= PW_REUSE_QUERIES;
        return PW_OK;
    }
    const HostSeqs& Q = e->Q;
    const int off = e->char_offset, dim = e->dim;
    Prepared& pr = e->pr;
    // residues must index the matrix (default_main.cu:234 reads matrix[c - offset];
    // the first invalid one of the input is reported); the compact alphabet
    // numbers the residues present in byte order
    int map[256];
    for (int i = 0; i < 256; ++i) map[i] = -1;
    std::vector<int> alphabet;
    const std::vector<int> present = present_bytes(Q.raw.data(), (int64_t)Q.raw.size());
    {
        int64_t bad_at = INT64_MAX;
        int bad = -1;
        for (int c : present)
            if (c == 0 || c < off || c >= off + dim) {
                const int64_t at = (int64_t)(std::find(Q.raw.begin(), Q.raw.end(), (uint8_t)c) - Q.raw.begin());
                if (at < bad_at) {
                    bad_at = at;
                    bad = c;
                }
            }
        if (bad >= 0)
            return fail(e, PW_ERR_ARG, "query residue outside the scoring matrix: code " + std::to_string(bad));
    }
    for (int c : present) {
        map[c] = (int)alphabet.size();
        alphabet.push_back(c);
    }
    if (alphabet.size() > 250) return fail(e, PW_ERR_ARG, "too many distinct query residues");
    pr.alpha = (int)alphabet.size();
    const int alpha1 = pr.alpha + 1;
    // scores of the used rows: all integers in the int8 range?
    bool q_int8 = true;
    float maxabs = 0.0f;
    for (int a = 0; a < pr.alpha; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = e->matrix[(size_t)(alphabet[a] - off) * dim + j];
            if (std::floor(v) != v || v < -127.0f || v > 127.0f) q_int8 = false;
            maxabs = std::max(maxabs, std::fabs(v));
        }
    pr.q_int8 = q_int8;
    pr.maxabs = maxabs;
    pr.qlen.assign(Q.n, 0);
    pr.maxlq = 0;
    for (int32_t i = 0; i < Q.n; ++i)
        pr.maxlq = std::max<int64_t>(pr.maxlq, pr.qlen[i] = (int32_t)(Q.off[i + 1] - Q.off[i]));
    std::vector<int8_t> cm8((size_t)alpha1 * dim, (int8_t)-128);
    std::vector<float> cmf((size_t)alpha1 * dim, -1.0e30f);
    for (int a = 0; a < pr.alpha; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = e->matrix[(size_t)(alphabet[a] - off) * dim + j];
            cmf[(size_t)a * dim + j] = v;
            cm8[(size_t)a * dim + j] = q_int8 ? (int8_t)v : 0;
        }
    // queries: compact codes, each sequence 16-byte aligned and padded to a
    // multiple of 4 with the pad code
    std::vector<int64_t> qco(Q.n + 1, 0);
    int64_t pos = 0;
    for (int32_t i = 0; i < Q.n; ++i) {
        qco[i] = pos;
        pos += align_up(std::max<int64_t>(pr.qlen[i], 1), 16);
    }
    qco[Q.n] = pos;
    // the transposed orientation: queries as strips (matrix residue indices)
    HostBuf<uint8_t>& qc = e->h_qc;
    HostBuf<uint8_t>& qres = e->h_qres;
    if (!qc.resize((size_t)std::max<int64_t>(pos, 16)) || !qres.resize((size_t)std::max<int64_t>(pos, 16)))
        return fail(e, PW_ERR_NOMEM, "host memory for the query encodings");
    parallel_for(Q.n, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            const uint8_t* r = Q.raw.data() + Q.off[i];
            uint8_t* d = qc.data() + qco[i];
            uint8_t* d2 = qres.data() + qco[i];
            const int64_t L = pr.qlen[i], end = qco[i + 1] - qco[i];
            for (int64_t k = 0; k < L; ++k) {
                d[k] = (uint8_t)map[r[k]];
                d2[k] = (uint8_t)(r[k] - off);
            }
            for (int64_t k = L; k < end; ++k) {
                d[k] = (uint8_t)pr.alpha;
                d2[k] = 0;
            }
        }
    }, (int64_t)1 << 14);
    for (size_t k = (size_t)pos; k < qc.size(); ++k) {
        qc.data()[k] = (uint8_t)pr.alpha;
        qres.data()[k] = 0;
    }
    // a stable sort by length, longest first
    {
        std::vector<uint64_t> key((size_t)Q.n);
        for (int32_t i = 0; i < Q.n; ++i) key[i] = (uint64_t)(pr.maxlq - pr.qlen[i]);
        const std::vector<uint32_t> o = radix_order(std::move(key));
        pr.order.assign(o.begin(), o.end());
    }
    cudaError_t c;
    // the encodings are page-locked already; the rest goes through the staging buffer
    if ((c = upload(e, e->q_codes, qc)) != cudaSuccess || (c = upload(e, e->q_res, qres)) != cudaSuccess)
        return cuda_fail(e, c, "upload query encodings");
    Staged st;
    st.add(e->q_code_off, qco);
    st.add(e->q_raw, Q.raw);
    st.add(e->q_raw_off, Q.off);
    st.add(e->q_len, pr.qlen);
    st.add(e->q_key, Q.key);
    st.add(e->q_order, pr.order);
    st.add(e->cmat_i8, cm8);
    st.add(e->cmat_f, cmf);
    if ((c = st.run(e)) != cudaSuccess || (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "upload queries");
    e->prep_q[0] = e->q_gen;
    e->prep_q[1] = e->s_gen;
    return PW_OK;
}

static int prepare(pw_engine* e) {
    int rc = prepare_targets(e);
    if (rc != PW_OK) return rc;
    if ((rc = prepare_queries(e)) != PW_OK) return rc;
    Prepared& pr = e->pr;
    // integer path: every used score and penalty is an integer, scores fit int8,
    // and no DP value can reach 2^24 (where fp32 stops being exact)
    bool ints = pr.q_int8 && std::floor(e->gap) == e->gap && std::floor(e->ext) == e->ext;
    if ((double)pr.maxabs * (double)std::min(pr.maxlq, pr.maxlt) + std::fabs(e->gap) + std::fabs(e->ext) >=
        16777216.0)
        ints = false;
    if (std::fabs(e->gap) > 1.0e6f || std::fabs(e->ext) > 1.0e6f) ints = false;
    pr.int_path = ints;
    // 16-bit halves hold every cell while the maximum stays below 32640; gap
    // chains must stay well inside the negative half-range
    const bool gaps16 = std::fabs(e->gap) + std::fabs(e->ext) < 8192.0f;
    pr.s16_q = ints && gaps16;
    pr.s16_t = ints && gaps16 && pr.t_int8;
    cudaError_t c;
    if ((c = e->counter.reserve(e->stream, 64 * sizeof(int))) != cudaSuccess) return cuda_fail(e, c, "alloc counter");
    return PW_OK;
}

static KernelArgs base_args(pw_engine* e) {
    KernelArgs A;
    memset(&A, 0, sizeof(A));
    const Prepared& pr = e->pr;
    ScoreParams& P = A.P;
    P.affine = e->affine;
    P.is_float = pr.int_path ? 0 : 1;
    P.gap_i = (int)e->gap;
    P.ext_i = (int)e->ext;
    P.ge_i = (int)e->gap + (int)e->ext;
    P.gap_f = e->gap;
    P.ext_f = e->ext;
    P.ge_f = e->gap + e->ext;
    P.lower_limit = e->lower_limit;
    P.minimum_score = e->minimum_score;
    P.host_minimum = e->host_minimum;
    P.highest = e->highest;
    P.filter_factor = e->filter_factor;
    P.alpha = pr.alpha;
    P.dim = e->dim;
    A.q = SeqSet{e->q_codes.as<uint8_t>(), e->q_code_off.as<int64_t>(), e->q_raw.as<uint8_t>(),
                 e->q_raw_off.as<int64_t>(), e->q_len.as<int32_t>(), e->q_key.as<int32_t>()};
    A.t = SeqSet{e->t_codes.as<uint8_t>(), e->t_code_off.as<int64_t>(), e->t_raw.as<uint8_t>(),
                 e->t_raw_off.as<int64_t>(), e->t_len.as<int32_t>(), e->t_key.as<int32_t>()};
    A.q_order = e->q_order.as<int32_t>();
    A.cmat_i8 = e->cmat_i8.as<int8_t>();
    A.cmat_f = e->cmat_f.as<float>();
    A.nt = e->T.n;
    A.pm_lane = e->T.n;
    A.pm_strip = 1;
    A.pair_max = e->pair_max.as<float>();
    return A;
}

// Launches a sweep phase over items already sorted by strip class and uploaded
// as one array; class c covers [cls_begin[c], cls_begin[c + 1]).  Each class
// gets its own work counter, so there is no host synchronisation in between.
// Kernel time per launch is accumulated into *kernel_ms after the phase.
template <int PH>
static int run_phase(pw_engine* e, KernelArgs A, const WorkItem* dev_items, const int (&cls_begin)[kNumClasses + 1],
                     int xmax_multi4, double* kernel_ms, int* n_launch, bool trans = false) {
    cudaError_t c;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
    if (cls_begin[kS32Multi + 1] > cls_begin[kS32Multi]) {
        // one boundary slot per resident warp (at most 16 blocks of 4 warps per SM)
        const int64_t slot = (int64_t)xmax_multi4 * kWarp;
        const int64_t warps = (int64_t)e->sm_count * 16 * 4;
        const size_t elem = e->pr.int_path ? sizeof(Bnd<int>) : sizeof(Bnd<float>);
        c = e->bnd_pool.reserve(e->stream, (size_t)(slot * warps) * elem);
        if (c != cudaSuccess) return cuda_fail(e, c, "alloc boundary pool");
        A.bnd_pool = e->bnd_pool.p;
        A.bnd_slot_elems = slot;
    }
    if ((c = cudaMemsetAsync(e->counter.p, 0, kNumClasses * sizeof(int), e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "reset counters");
    for (int cls = 0; cls < kNumClasses; ++cls) {
        const int n = cls_begin[cls + 1] - cls_begin[cls];
        if (n <= 0) continue;
        A.items = dev_items + cls_begin[cls];
        A.n_items = n;
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, e->stream);
        if constexpr (PH == 3)
            c = launch_class<int, 3>(e, cls, false, A, e->counter.as<int>() + cls, trans);
        else
            c = e->pr.int_path ? launch_class<int, PH>(e, cls, e->affine, A, e->counter.as<int>() + cls, trans)
                               : launch_class<float, PH>(e, cls, e->affine, A, e->counter.as<int>() + cls, trans);
        cudaEventRecord(b, e->stream);
        evs.push_back({a, b});
        if (c != cudaSuccess) return cuda_fail(e, c, "sweep kernel launch");
        if (n_launch) ++*n_launch;
    }
    if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "sweep kernel");
    for (auto& ab : evs) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ab.first, ab.second);
        if (kernel_ms) *kernel_ms += ms;
        cudaEventDestroy(ab.first);
        cudaEventDestroy(ab.second);
    }
    return PW_OK;
}

// Sorts items by strip class (stable; a counting sort) and returns the class
// boundaries.
static void order_by_class(std::vector<WorkItem>& items, std::vector<int>& cls, int (&begin)[kNumClasses + 1]) {
    for (int c = 0; c <= kNumClasses; ++c) begin[c] = 0;
    for (int c : cls) begin[c + 1]++;
    for (int c = 0; c < kNumClasses; ++c) begin[c + 1] += begin[c];
    int pos[kNumClasses + 1];
    for (int c = 0; c <= kNumClasses; ++c) pos[c] = begin[c];
    std::vector<WorkItem> it2(items.size());
    std::vector<int> c2(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        const int p = pos[cls[k]]++;
        it2[p] = items[k];
        c2[p] = cls[k];
    }
    items.swap(it2);
    cls.swap(c2);
}

// Phase-1 work items above which the one-strip classes take the grid form
// (strip-pair lists, items formed on the device) instead of an item list.
constexpr int64_t kGridItems = (int64_t)1 << 18;

// Order of items by strip class ascending, then cost descending, ties in
// their current order (what a stable sort by cost followed by a stable sort
// by class gives): an LSD radix sort of (class, ~cost) keys, 16 bits a pass,
// skipping the digits in which every key agrees.  Linear in the item count:
// millions of work items (short reads) are ordered in milliseconds.
static std::vector<uint32_t> class_cost_order(const std::vector<int>& cls, const std::vector<int64_t>& cost) {
    constexpr uint64_t kCostMask = ((uint64_t)1 << 48) - 1;
    std::vector<uint64_t> key(cls.size());
    for (size_t k = 0; k < key.size(); ++k) {
        const uint64_t c = std::min<uint64_t>((uint64_t)std::max<int64_t>(cost[k], 0), kCostMask);
        key[k] = ((uint64_t)cls[k] << 48) | (kCostMask - c);
    }
    return radix_order(std::move(key));
}


// ------------------------------------------------------------ 16-bit phase 1
template <int S, bool AFF, bool MULTI, bool DL>
static cudaError_t launch_s16(pw_engine* e, Score16Args A) {
    auto kern = score16_kernel<S, AFF, MULTI, DL>;
    const int smem = 4 * (S / 4) * A.alpha1 * prof_entry_bytes<DL>();
    if (smem > 48 * 1024) {
        cudaError_t c = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (c != cudaSuccess) return c;
    }
    int per_sm = 0;
    cudaError_t c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
    if (c != cudaSuccess) return c;
    per_sm = std::max(1, std::min(per_sm, 16));
    int grid = std::min(grid_cap(e, per_sm), (A.n_items + 3) / 4);
    PW_LAUNCH(kern, std::max(grid, 1), 128, smem, e->stream, A);
    e->launches++;
    return cudaGetLastError();
}

template <bool DL>
static cudaError_t launch_s16_class(pw_engine* e, int cls, bool affine, const Score16Args& A) {
    if (affine) {
        if (cls == kS16) return launch_s16<16, true, false, DL>(e, A);
        if (cls == kS24) return launch_s16<24, true, false, DL>(e, A);
        if (cls == kS32) return launch_s16<32, true, false, DL>(e, A);
        return launch_s16<32, true, true, DL>(e, A);
    }
    if (cls == kS16) return launch_s16<16, false, false, DL>(e, A);
    if (cls == kS24) return launch_s16<24, false, false, DL>(e, A);
    if (cls == kS32) return launch_s16<32, false, false, DL>(e, A);
    if (cls == kS40) return launch_s16<40, false, false, DL>(e, A);
    if (cls == kS48) return launch_s16<48, false, false, DL>(e, A);
    if (cls == kS64) return launch_s16<64, false, false, DL>(e, A);
    return launch_s16<32, false, true, DL>(e, A);
}

// Plans the multi-strip launch.  Items whose sweep cost (columns x strips)
// reaches `min_permille`/1000 of the mean per-warp load are cut into chains of
// one-strip entries (score16_chain_kernel); the others stay whole.  The queue
// order comes from a list-scheduling simulation of `warps` equally fast warps:
// a free warp takes the next strip of the largest chain whose predecessor is
// at least kChainLead columns ahead, else the next whole item (longest first),
// else the strip that becomes ready first.  Every strip is queued after its
// predecessor, which is what the kernel's waits rely on.
static int setup_chains(pw_engine* e, const std::vector<WorkItem>& items, int i0, int i1,
                        const std::vector<int32_t>& strip_len, int warps, int* n_entries) {
    const int n = i1 - i0;
    std::vector<int> nstr(n);
    std::vector<int64_t> xm4(n);
    for (int k = 0; k < n; ++k) {
        const WorkItem& W = items[i0 + k];
        const int ls = std::max(strip_len[W.target], W.index >= 0 ? strip_len[W.index] : 0);
        nstr[k] = (ls + 31) / 32;
        xm4[k] = align_up(W.xmax, 4);
    }
    const int64_t permille = e->tune[PW_TUNE_CHAIN_MIN] > 0 ? e->tune[PW_TUNE_CHAIN_MIN] : 500;
    ChainPlan plan;
    plan_chain_queue(nstr, xm4, warps, permille, kChainLead, plan);
    std::vector<WorkItem> q(plan.queue.size());
    std::vector<int4> info(plan.queue.size());
    for (size_t k = 0; k < plan.queue.size(); ++k) {
        const PlanEntry& p = plan.queue[k];
        q[k] = items[i0 + p.item];
        info[k] = make_int4(p.chain, p.strip, p.pred, 0);
    }
    std::vector<int64_t> ring_off(std::max<size_t>(plan.chain_xm4.size(), 1), 0);
    int64_t ring_elems = 0;
    for (size_t c = 0; c < plan.chain_xm4.size(); ++c) {
        ring_off[c] = ring_elems;
        ring_elems += 2 * plan.chain_xm4[c] * kWarp;
    }
    cudaError_t c;
    if ((c = upload(e, e->chain_items, q)) != cudaSuccess) return cuda_fail(e, c, "upload chain items");
    if ((c = upload(e, e->chain_info, info)) != cudaSuccess) return cuda_fail(e, c, "upload chain info");
    e->h_chain_info = info;
    if ((c = upload(e, e->chain_ring_off, ring_off)) != cudaSuccess) return cuda_fail(e, c, "upload ring offsets");
    // one progress flag per entry, plus one that no entry ever sets (PW_TUNE_STALL_TEST)
    if ((c = e->chain_prog.reserve(e->stream, (q.size() + 1) * sizeof(int))) != cudaSuccess)
        return cuda_fail(e, c, "alloc chain progress");
    if ((c = e->chain_max.reserve(e->stream, q.size() * kWarp * sizeof(uint32_t))) != cudaSuccess)
        return cuda_fail(e, c, "alloc chain maxima");
    if ((c = e->chain_ring.reserve(e->stream, (size_t)std::max<int64_t>(ring_elems, 1) * sizeof(uint4))) != cudaSuccess)
        return cuda_fail(e, c, "alloc chain ring");
    if ((c = e->chain_abort.reserve(e->stream, sizeof(int))) != cudaSuccess) return cuda_fail(e, c, "alloc chain status");
    *n_entries = (int)q.size();
    return PW_OK;
}

template <int S, bool AFF, bool DL>
static cudaError_t launch_s16_chain(pw_engine* e, Score16Args A) {
    auto kern = score16_chain_kernel<S, AFF, DL>;
    // the four warps' profiles, then (affine) their prefetch rings of the row above
    const int smem = chain_profile_bytes<S, DL>(A.alpha1) + (AFF ? 4 * kPre * kWarp * (int)sizeof(uint4) : 0);
    if (smem > 48 * 1024) {
        cudaError_t c = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (c != cudaSuccess) return c;
    }
    int per_sm = 0;
    cudaError_t c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
    if (c != cudaSuccess) return c;
    per_sm = std::max(1, std::min(per_sm, 16));
    const int grid = std::max(1, std::min(grid_cap(e, per_sm), (A.n_items - A.item_base + 3) / 4));
    PW_LAUNCH(kern, grid, 128, smem, e->stream, A);
    e->launches++;
    return cudaGetLastError();
}

// Cell-slot cost of an orientation: strips are paired in length order (one
// pair per 16x2 register), lanes grouped 32 at a time in length order; every
// work item pays its longer strip times its longest lane for all 64 slots.
static double orientation_cost(const std::vector<int32_t>& strip_len, const std::vector<int32_t>& strip_order,
                               const std::vector<int32_t>& lane_len, const std::vector<int32_t>& lane_order) {
    double lane_groups = 0;
    for (size_t g = 0; g < lane_order.size(); g += kWarp) lane_groups += lane_len[lane_order[g]];
    double strips = 0;
    for (size_t i = 0; i < strip_order.size(); i += 2) strips += strip_len[strip_order[i]];
    return strips * lane_groups * 2 * kWarp;
}

// Cell-slot cost of the dual-lane form: every strip alone, against lane
// groups taken 64 at a time (two 32-lane groups in the low and high halves).
static double dual_cost(const std::vector<int32_t>& strip_len, const std::vector<int32_t>& lane_len,
                        const std::vector<int32_t>& lane_order) {
    double lane_pairs = 0;
    for (size_t g = 0; g < lane_order.size(); g += 2 * kWarp) lane_pairs += lane_len[lane_order[g]];
    double strips = 0;
    for (int32_t l : strip_len) strips += l;
    return strips * lane_pairs * 2 * kWarp;
}

// Relative cost of a dual-lane cell slot: its profile fetch interleaves two
// residues' words (two 64-bit shared loads and four byte permutes per four
// rows instead of one 128-bit load).
constexpr double kDualSlotCost = 1.15;

// Pair maxima with the 16-bit dual-pair sweep.  Returns the device time of
// the sweep launches in *kernel_ms.  Pairs whose maximum could overflow
// 16-bit halves come back as NaN; they are recomputed by the 32-bit sweep.
static int phase1_s16(pw_engine* e, const KernelArgs& A32, pw_run_info& inf, uint32_t flags) {
    const Prepared& pr = e->pr;
    const int nq = e->Q.n, nt = e->T.n;
    auto& P1 = e->p1;
    const uint32_t pflags = flags & PW_FLAG_NO_CHAIN;
    const bool reuse = !(flags & PW_FLAG_REPLAN) && P1.valid && P1.qg == e->q_gen && P1.tg == e->t_gen &&
                       P1.sg == e->s_gen &&
                       P1.flags == pflags && P1.tune == e->tune[PW_TUNE_CHAIN_MIN] &&
                       P1.share == e->tune[PW_TUNE_GRID_SHARE] && P1.dual_mode == e->tune[PW_TUNE_DUAL];
    cudaError_t c;
    if (reuse) e->reuse |= PW_REUSE_PLAN;
    if (!reuse) {
        const double t_plan = wall_ms();
        P1.valid = false;
        // four forms: targets or queries as strips, strip pairs or dual lanes
        // (PW_TUNE_DUAL: 1 always dual lanes, 2 never, else the cheaper form)
        bool trans = false, dual = false;
        {
            const int64_t dm = e->tune[PW_TUNE_DUAL];
            double best = -1;
            for (int o = 0; o < 2; ++o) {
                if (o == 1 ? !pr.s16_t : !pr.s16_q) continue;
                const bool tr = o == 1;
                const auto& sl = tr ? pr.qlen : pr.tlen;
                const auto& so = tr ? pr.order : pr.order_t;
                const auto& ll = tr ? pr.tlen : pr.qlen;
                const auto& lo = tr ? pr.order_t : pr.order;
                for (int d = 0; d < 2; ++d) {
                    if ((d == 1 && dm == 2) || (d == 0 && dm == 1)) continue;
                    const double cst = d ? dual_cost(sl, ll, lo) * kDualSlotCost : orientation_cost(sl, so, ll, lo);
                    if (best < 0 || cst < best) {
                        best = cst;
                        trans = tr;
                        dual = d == 1;
                    }
                }
            }
        }
        const std::vector<int32_t>& strip_len = trans ? pr.qlen : pr.tlen;
        const std::vector<int32_t>& strip_order = trans ? pr.order : pr.order_t;
        const std::vector<int32_t>& lane_len = trans ? pr.tlen : pr.qlen;
        const std::vector<int32_t>& lane_order = trans ? pr.order_t : pr.order;
        const int n_strip = trans ? nq : nt, n_lane = trans ? nt : nq;
        std::vector<WorkItem> items;
        std::vector<int> cls;
        std::vector<int64_t> cost;
        const int strip_step = dual ? 1 : 2, lane_step = dual ? 2 * kWarp : kWarp;
        // Many items (short reads against a few targets): the one-strip
        // classes go as strip-pair lists, their items formed on the device
        // (grid_item), lane groups longest first; the chained class keeps its
        // explicit queue.
        const int64_t n_groups = (n_lane + lane_step - 1) / lane_step;
        const int64_t n_pairs_s = (n_strip + strip_step - 1) / strip_step;
        if (n_pairs_s * n_groups > (int64_t)INT32_MAX) return fail(e, PW_ERR_CAPACITY, "too many work items");
        const bool grid = n_pairs_s * n_groups > kGridItems;
        std::vector<int2> gstrips[kNumClasses];
        for (int i = 0; i < n_strip; i += strip_step) {
            const int sa = strip_order[i], sb = !dual && i + 1 < n_strip ? strip_order[i + 1] : -1;
            const int ls = std::max(strip_len[sa], sb >= 0 ? strip_len[sb] : 0);
            if (grid) {
                const int k = pick_class16(ls, e->affine);
                if (k != kS32Multi) {
                    gstrips[k].push_back(make_int2(sa, sb));
                    continue;
                }
            }
            for (int g = 0; g < n_lane; g += lane_step) {
                WorkItem w;
                memset(&w, 0, sizeof(w));
                w.target = sa;
                w.index = sb;
                w.first = g;
                w.lanes = std::min(kWarp, n_lane - g);
                w.lanes_hi = dual ? std::max(0, std::min(kWarp, n_lane - g - kWarp)) : 0;
                w.xmax = lane_len[lane_order[g]];
                const int k = pick_class16(ls, e->affine);
                w.S = class_S(k);
                items.push_back(w);
                cls.push_back(k);
                cost.push_back((int64_t)w.xmax * ls);
            }
        }
        // largest cost first within each strip class (dynamic scheduling tail)
        const std::vector<uint32_t> idx = class_cost_order(cls, cost);
        std::vector<WorkItem> it2(items.size());
        std::vector<int> c2(items.size());
        for (size_t k = 0; k < idx.size(); ++k) {
            it2[k] = items[idx[k]];
            c2[k] = cls[idx[k]];
        }
        int begin[kNumClasses + 1];
        for (int k = 0; k <= kNumClasses; ++k) begin[k] = 0;
        for (int k : c2) begin[k + 1]++;
        for (int k = 0; k < kNumClasses; ++k) begin[k + 1] += begin[k];
        if ((c = upload(e, e->p1_items, it2)) != cudaSuccess) return cuda_fail(e, c, "upload items");
        {
            std::vector<int2> gs;
            for (int k = 0; k < kNumClasses; ++k) {
                P1.gbegin[k] = (int)gs.size();
                gs.insert(gs.end(), gstrips[k].begin(), gstrips[k].end());
            }
            P1.gbegin[kNumClasses] = (int)gs.size();
            if ((c = upload(e, e->p1_grid, gs)) != cudaSuccess) return cuda_fail(e, c, "upload strip pairs");
            P1.grid = grid;
            P1.n_groups = (int)n_groups;
        }
        int xm = 4;
        for (int k = begin[kS32Multi]; k < begin[kS32Multi + 1]; ++k) xm = std::max(xm, (int)align_up(it2[k].xmax, 4));
        P1.chained = !(flags & PW_FLAG_NO_CHAIN) && begin[kS32Multi + 1] > begin[kS32Multi];
        P1.n_chain_items = 0;
        if (P1.chained) {
            int per_sm = 0;
            const int a1 = (trans ? pr.alpha_t : pr.alpha) + 1;
            const int smem = (dual ? chain_profile_bytes<32, true>(a1) : chain_profile_bytes<32, false>(a1)) +
                             (e->affine ? 4 * kPre * kWarp * (int)sizeof(uint4) : 0);
            auto kern = e->affine ? (dual ? score16_chain_kernel<32, true, true> : score16_chain_kernel<32, true, false>)
                                  : (dual ? score16_chain_kernel<32, false, true> : score16_chain_kernel<32, false, false>);
            if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if ((c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem)) != cudaSuccess)
                return cuda_fail(e, c, "occupancy");
            const int rc = setup_chains(e, it2, begin[kS32Multi], begin[kS32Multi + 1], strip_len,
                                        grid_cap(e, std::max(1, std::min(per_sm, 16))) * 4, &P1.n_chain_items);
            if (rc != PW_OK) return rc;
        }
        P1.trans = trans;
        P1.dual = dual;
        P1.dual_mode = e->tune[PW_TUNE_DUAL];
        for (int k = 0; k <= kNumClasses; ++k) P1.begin[k] = begin[k];
        P1.xm_multi = xm;
        P1.qg = e->q_gen;
        P1.tg = e->t_gen;
        P1.sg = e->s_gen;
        P1.flags = pflags;
        P1.tune = e->tune[PW_TUNE_CHAIN_MIN];
        P1.share = e->tune[PW_TUNE_GRID_SHARE];
        P1.valid = true;
        inf.setup_ms += wall_ms() - t_plan;
        HostTrace ht;
        ht.t = t_plan;
        ht.mark("phase-1 plan (rebuilt)");
    }
    const bool trans = P1.trans;
    const bool chained = P1.chained;
    const bool dual = P1.dual;
    const int* begin = P1.begin;
    inf.orientation = trans ? 1 : 0;
    inf.dual_lanes = dual ? 1 : 0;
    Score16Args S;
    memset(&S, 0, sizeof(S));
    S.lane_codes = trans ? e->t_ccodes.as<uint8_t>() : e->q_codes.as<uint8_t>();
    S.lane_off = trans ? e->t_code_off.as<int64_t>() : e->q_code_off.as<int64_t>();
    S.lane_len = trans ? e->t_len.as<int32_t>() : e->q_len.as<int32_t>();
    S.lane_order = trans ? e->t_order.as<int32_t>() : e->q_order.as<int32_t>();
    S.strip_res = trans ? e->q_res.as<uint8_t>() : e->t_codes.as<uint8_t>();
    S.strip_off = trans ? e->q_code_off.as<int64_t>() : e->t_code_off.as<int64_t>();
    S.strip_len = trans ? e->q_len.as<int32_t>() : e->t_len.as<int32_t>();
    S.cmat = trans ? e->cmat_t8.as<int8_t>() : e->cmat_i8.as<int8_t>();
    S.alpha1 = (trans ? pr.alpha_t : pr.alpha) + 1;
    S.dim = e->dim;
    S.gap = (int)e->gap;
    S.ext = (int)e->ext;
    S.ge = S.gap + S.ext;
    S.pair_max = A32.pair_max;
    S.stride_strip = trans ? nt : 1;
    S.stride_lane = trans ? 1 : nt;
    S.pad_code = S.alpha1 - 1;
    S.wait_ns = wait_limit(e);
    if (begin[kS32Multi + 1] > begin[kS32Multi]) {
        const int64_t slot = (int64_t)P1.xm_multi * kWarp;
        if ((c = e->bnd_pool.reserve(e->stream, (size_t)slot * e->sm_count * 16 * 4 * sizeof(uint4))) != cudaSuccess)
            return cuda_fail(e, c, "alloc boundary pool");
        S.bnd_pool = e->bnd_pool.as<uint4>();
        S.bnd_slot = slot;
    }
    if ((c = cudaMemsetAsync(e->counter.p, 0, 16 * sizeof(int), e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "reset counters");
    S.ovf_count = e->counter.as<int>() + 8;
    if (chained) {
        S.chain = e->chain_info.as<int4>();
        S.ring_off = e->chain_ring_off.as<int64_t>();
        S.ring = e->chain_ring.as<uint4>();
        S.progress = e->chain_prog.as<int>();
        S.run_max = e->chain_max.as<uint32_t>();
        S.abort_flag = e->chain_abort.as<int>();
        S.n_chain_items = P1.n_chain_items;
        if (e->tune[PW_TUNE_STALL_TEST]) {
            // one entry with a predecessor waits on the spare flag instead
            e->tune[PW_TUNE_STALL_TEST] = 0;
            std::vector<int4> info = e->h_chain_info;
            for (int4& v : info)
                if (v.y > 0) {
                    v.z = P1.n_chain_items;
                    break;
                }
            if ((c = upload(e, e->stall_buf, info)) != cudaSuccess) return cuda_fail(e, c, "upload stalled queue");
            S.chain = e->stall_buf.as<int4>();
        }
        if ((c = cudaMemsetAsync(e->chain_prog.p, 0, (size_t)(P1.n_chain_items + 1) * sizeof(int), e->stream)) !=
                cudaSuccess ||
            (c = cudaMemsetAsync(e->chain_abort.p, 0, sizeof(int), e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "clear chain state");
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    for (int k = 0; k < kNumClasses; ++k) {
        const int n = begin[k + 1] - begin[k];
        if (n <= 0) continue;
        if (k == kS32Multi && chained) {
            // the queue in consecutive segments, one launch each (PW_TUNE_SEGMENT):
            // every strip's predecessor is in the same or an earlier segment
            S.items = e->chain_items.as<WorkItem>();
            S.counter = e->counter.as<int>() + k;
            const int total = S.n_chain_items;
            const int seg = e->tune[PW_TUNE_SEGMENT] > 0 ? (int)std::min<int64_t>(e->tune[PW_TUNE_SEGMENT], total)
                                                          : total;
            for (int base = 0; base < total; base += std::max(seg, 1)) {
                S.item_base = base;
                S.n_items = std::min(total, base + std::max(seg, 1));
                if (base > 0 && (c = cudaMemsetAsync(S.counter, 0, sizeof(int), e->stream)) != cudaSuccess)
                    return cuda_fail(e, c, "reset counter");
                c = e->affine ? (dual ? launch_s16_chain<32, true, true>(e, S) : launch_s16_chain<32, true, false>(e, S))
                              : (dual ? launch_s16_chain<32, false, true>(e, S) : launch_s16_chain<32, false, false>(e, S));
                if (c != cudaSuccess) return cuda_fail(e, c, "score16 chain launch");
                inf.score_launches++;
            }
            continue;
        }
        S.items = e->p1_items.as<WorkItem>() + begin[k];
        S.n_items = n;
        S.counter = e->counter.as<int>() + k;
        S.grid_strips = nullptr;
        c = dual ? launch_s16_class<true>(e, k, e->affine, S) : launch_s16_class<false>(e, k, e->affine, S);
        if (c != cudaSuccess) return cuda_fail(e, c, "score16 launch");
        inf.score_launches++;
    }
    for (int k = 0; P1.grid && k < kNumClasses; ++k) {
        const int np_ = P1.gbegin[k + 1] - P1.gbegin[k];
        if (np_ <= 0 || k == kS32Multi) continue;
        S.items = nullptr;
        S.grid_strips = e->p1_grid.as<int2>() + P1.gbegin[k];
        S.grid_n_strips = np_;
        S.grid_lane_step = dual ? 2 * kWarp : kWarp;
        S.grid_n_lane = trans ? nt : nq;
        S.n_items = (int)((int64_t)np_ * P1.n_groups);
        S.counter = e->counter.as<int>() + k;
        c = dual ? launch_s16_class<true>(e, k, e->affine, S) : launch_s16_class<false>(e, k, e->affine, S);
        if (c != cudaSuccess) return cuda_fail(e, c, "score16 launch");
        inf.score_launches++;
    }
    cudaEventRecord(b, e->stream);
    int status[2] = {0, 0};  // overflow count, chain abort flag
    if ((c = copy_d2h(e, &status[0], S.ovf_count, sizeof(int))) != cudaSuccess ||
        (chained &&
         (c = copy_d2h(e, &status[1], e->chain_abort.p, sizeof(int))) !=
             cudaSuccess) ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "read score status");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    inf.score_kernel_ms += ms;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (status[1]) return fail(e, PW_ERR_KERNEL, "chained score sweep: a strip waited too long for its predecessor");
    // the maxima stay on the device (pruning reads them there); the host
    // copy is needed only to find the pairs that reached the 16-bit limit
    e->pm_stale = true;
    if (status[0] > 0) {
        const int rc = sync_pair_max(e, A32.pair_max);
        if (rc != PW_OK) return rc;
    }

    // pairs that reached the 16-bit limit: the 32-bit sweep, per target
    std::vector<std::vector<int32_t>> ovf(nt);
    int64_t n_ovf = 0;
    for (int sp = 0; sp < nq && status[0] > 0; ++sp) {
        const int q = pr.order[sp];
        for (int t = 0; t < nt; ++t)
            if (std::isnan(e->h_pair_max[(size_t)q * nt + t])) {
                ovf[t].push_back(q);
                ++n_ovf;
            }
    }
    inf.overflow_pairs = n_ovf;
    if (n_ovf == 0) return PW_OK;
    std::vector<int32_t> order2;
    std::vector<WorkItem> its;
    std::vector<int> cl;
    for (int t = 0; t < nt; ++t)
        for (size_t g = 0; g < ovf[t].size(); g += kWarp) {
            WorkItem w;
            memset(&w, 0, sizeof(w));
            w.target = t;
            w.first = (int32_t)order2.size();
            w.lanes = (int32_t)std::min<size_t>(kWarp, ovf[t].size() - g);
            for (int l = 0; l < w.lanes; ++l) order2.push_back(ovf[t][g + l]);
            w.xmax = pr.qlen[order2[w.first]];
            const int k = pick_class(pr.tlen[t], e->affine);
            w.S = class_S(k);
            its.push_back(w);
            cl.push_back(k);
        }
    int bg[kNumClasses + 1];
    order_by_class(its, cl, bg);
    int xm = 4;
    for (int k = bg[kS32Multi]; k < bg[kS32Multi + 1]; ++k) xm = std::max(xm, (int)align_up(its[k].xmax, 4));
    if ((c = upload(e, e->q_order2, order2)) != cudaSuccess) return cuda_fail(e, c, "upload order");
    if ((c = upload(e, e->items, its)) != cudaSuccess) return cuda_fail(e, c, "upload items");
    KernelArgs A = A32;
    A.q_order = e->q_order2.as<int32_t>();
    int rc = run_phase<1>(e, A, e->items.as<WorkItem>(), bg, xm, &inf.score_kernel_ms, &inf.score_launches);
    if (rc != PW_OK) return rc;
    e->pm_stale = true;
    return PW_OK;
}


// Orders the n accumulated hits (acc_hits / acc_ops) as the reference's
// HitList and spells their strings on the device; the records land in
// h_hits / h_strings.
static cudaError_t finish_hits(pw_engine* e, int64_t n, int64_t* str_bytes) {
    *str_bytes = 0;
    e->h_hits.clear();
    e->h_strings.clear();
    if (n <= 0) return cudaSuccess;
    if (n > (int64_t)INT32_MAX) return cudaErrorInvalidValue;
    cudaError_t c;
    const size_t k8 = (size_t)n * sizeof(uint64_t), k4 = (size_t)n * sizeof(int32_t);
    if ((c = e->fk_a.reserve(e->stream, k8)) != cudaSuccess || (c = e->fk_b.reserve(e->stream, k8)) != cudaSuccess ||
        (c = e->fk_c.reserve(e->stream, k8)) != cudaSuccess || (c = e->fk_t.reserve(e->stream, k8)) != cudaSuccess ||
        (c = e->fk_g.reserve(e->stream, k8)) != cudaSuccess || (c = e->fi_a.reserve(e->stream, k4)) != cudaSuccess ||
        (c = e->fi_b.reserve(e->stream, k4)) != cudaSuccess || (c = e->f_len.reserve(e->stream, k8)) != cudaSuccess ||
        (c = e->f_soff.reserve(e->stream, k8)) != cudaSuccess)
        return c;
    const DevHit* h = e->acc_hits.as<DevHit>();
    uint64_t *ka = e->fk_a.as<uint64_t>(), *kb = e->fk_b.as<uint64_t>(), *kc = e->fk_c.as<uint64_t>();
    uint64_t *kt = e->fk_t.as<uint64_t>(), *kg = e->fk_g.as<uint64_t>();
    int32_t *ia = e->fi_a.as<int32_t>(), *ib = e->fi_b.as<int32_t>();
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)e->sm_count * 16));
    PW_LAUNCH(hit_key_kernel, grid, 256, 0, e->stream, h, n, ka, kb, kc, ia);
    size_t tmp = 0;
    if ((c = cub::DeviceRadixSort::SortPairs(nullptr, tmp, kc, kt, ia, ib, (int)n, 0, 64, e->stream)) != cudaSuccess ||
        (c = e->scan_tmp.reserve(e->stream, std::max<size_t>(tmp, 16))) != cudaSuccess)
        return c;
    tmp = e->scan_tmp.bytes;
    // three stable passes, least significant word first
    if ((c = cub::DeviceRadixSort::SortPairs(e->scan_tmp.p, tmp, kc, kt, ia, ib, (int)n, 0, 64, e->stream)) !=
        cudaSuccess)
        return c;
    PW_LAUNCH(gather_key_kernel, grid, 256, 0, e->stream, kb, ib, n, kg);
    tmp = e->scan_tmp.bytes;
    if ((c = cub::DeviceRadixSort::SortPairs(e->scan_tmp.p, tmp, kg, kt, ib, ia, (int)n, 0, 64, e->stream)) !=
        cudaSuccess)
        return c;
    PW_LAUNCH(gather_key_kernel, grid, 256, 0, e->stream, ka, ia, n, kg);
    tmp = e->scan_tmp.bytes;
    if ((c = cub::DeviceRadixSort::SortPairs(e->scan_tmp.p, tmp, kg, kt, ia, ib, (int)n, 0, 64, e->stream)) !=
        cudaSuccess)
        return c;
    // string offsets in the final order
    int64_t *len = e->f_len.as<int64_t>(), *soff = e->f_soff.as<int64_t>();
    PW_LAUNCH(hit_len_kernel, grid, 256, 0, e->stream, h, ib, n, len);
    size_t stmp = 0;
    if ((c = cub::DeviceScan::ExclusiveSum(nullptr, stmp, len, soff, (int64_t)n, e->stream)) != cudaSuccess) return c;
    if (stmp > e->scan_tmp.bytes && (c = e->scan_tmp.reserve(e->stream, stmp)) != cudaSuccess) return c;
    stmp = e->scan_tmp.bytes;
    if ((c = cub::DeviceScan::ExclusiveSum(e->scan_tmp.p, stmp, len, soff, (int64_t)n, e->stream)) != cudaSuccess)
        return c;
    int64_t tail[2] = {0, 0};
    if ((c = copy_d2h(e, &tail[0], soff + n - 1, sizeof(int64_t))) !=
            cudaSuccess ||
        (c = copy_d2h(e, &tail[1], len + n - 1, sizeof(int64_t))) !=
            cudaSuccess ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return c;
    const int64_t total = tail[0] + tail[1];
    if ((c = e->f_out.reserve(e->stream, (size_t)n * sizeof(pw_hit))) != cudaSuccess ||
        (c = e->f_str.reserve(e->stream, (size_t)std::max<int64_t>(total, 16))) != cudaSuccess)
        return c;
    PW_LAUNCH(hit_out_kernel, grid, 256, 0, e->stream, h, ib, soff, n, e->acc_ops.as<char>(), e->q_raw.as<uint8_t>(),
              e->q_raw_off.as<int64_t>(), e->t_raw.as<uint8_t>(), e->t_raw_off.as<int64_t>(), e->f_out.as<pw_hit>(),
              e->f_str.as<char>());
    {
        const int wgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, (int64_t)e->sm_count * 16));
        PW_LAUNCH(hit_strings_warp_kernel, wgrid, 128, 0, e->stream, h, ib, soff, n, e->acc_ops.as<char>(),
                  e->q_raw.as<uint8_t>(), e->q_raw_off.as<int64_t>(), e->t_raw.as<uint8_t>(),
                  e->t_raw_off.as<int64_t>(), e->f_str.as<char>());
    }
    e->launches += 6;  // this library's kernels (the CUB sorts and scan are not counted)
    if ((c = cudaGetLastError()) != cudaSuccess) return c;
    if (!e->h_hits.resize((size_t)n) || !e->h_strings.resize((size_t)total)) return cudaErrorMemoryAllocation;
    if ((c = copy_d2h(e, e->h_hits.data(), e->f_out.p, (size_t)n * sizeof(pw_hit))) != cudaSuccess ||
        (total > 0 && (c = copy_d2h(e, e->h_strings.data(), e->f_str.p, (size_t)total)) != cudaSuccess) ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return c;
    *str_bytes = total;
    return cudaSuccess;
}

// Queue entries (pair, band, queue index of the band above) of band chains:
// pair k has nbands[k] bands of steps[k] steps, pairs in priority order.
static std::vector<int4> band_queue(const std::vector<int>& nbands, const std::vector<int64_t>& steps, int warps) {
    std::vector<int4> entries;
    if ((int64_t)nbands.size() * 2 >= warps) {
        // many pairs: band-major order (every band 0, then every band 1, ...,
        // longest pairs first within a band); a band's predecessor was handed
        // out at least a whole band generation earlier, so nobody waits long
        int maxb = 0;
        for (int nb : nbands) maxb = std::max(maxb, nb);
        std::vector<int32_t> last(nbands.size(), -1);
        for (int b = 0; b < maxb; ++b)
            for (size_t k = 0; k < nbands.size(); ++k)
                if (b < nbands[k]) {
                    entries.push_back(make_int4((int)k, b, last[k], 0));
                    last[k] = (int32_t)entries.size() - 1;
                }
    } else {
        // few (long) pairs: a list-scheduling plan pipelines each pair's bands
        ChainPlan plan;
        plan_chain_queue(nbands, steps, warps, 1, kBandLead, plan);
        entries.resize(plan.queue.size());
        for (size_t k = 0; k < plan.queue.size(); ++k) {
            const PlanEntry& p = plan.queue[k];
            entries[k] = make_int4(p.item, p.chain >= 0 ? p.strip : 0, p.pred, 0);
        }
    }
    return entries;
}

// Launches band_kernel over `pairs` (one warp per band, the bands of a pair
// chained across warps, pw_band.cuh).  DIRS 1: the direction sweep of traced
// pairs (cell codes), 2: the same storing H (linear gap), 3: the checkpoint
// sweep of the tile form (linear gap, checkpoints into tile_ck); 0: pair
// maxima into band_max (indexed by BandPair.slot).
template <int DIRS>
static int run_band_phase(pw_engine* e, KernelArgs A, std::vector<BandPair>& pairs, double* kernel_ms,
                          int* n_launch) {
    if (pairs.empty()) return PW_OK;
    const int prof_bytes = (int)align_up((int64_t)kWarp * (A.P.alpha + 1) * kWarpRows, 16);
    const int smem = 4 * prof_bytes;
    auto kern = band_kernel<false, DIRS>;
    if constexpr (DIRS < 2)
        if (e->affine) kern = band_kernel<true, DIRS>;
    cudaError_t c;
    if (smem > 48 * 1024 &&
        (c = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
        return cuda_fail(e, c, "band sweep smem");
    int per_sm = 0;
    if ((c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem)) != cudaSuccess)
        return cuda_fail(e, c, "occupancy");
    per_sm = std::max(1, std::min(per_sm, 16));
    const int warps = grid_cap(e, per_sm) * 4;
    // queue: the bands of each pair form a chain (pw_plan.h), longest pairs first
    std::vector<int> order(pairs.size());
    std::iota(order.begin(), order.end(), 0);
    std::vector<int64_t> steps(pairs.size());
    for (size_t k = 0; k < pairs.size(); ++k) {
        pairs[k].nbands = std::max(1, pairs[k].nbands);
        steps[k] = (int64_t)e->pr.qlen[pairs[k].q] + kWarp - 1;
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return steps[x] * pairs[x].nbands > steps[y] * pairs[y].nbands;
    });
    std::vector<BandPair> sorted(pairs.size());
    std::vector<int> nstr(pairs.size());
    std::vector<int64_t> xm(pairs.size());
    int64_t ring_elems = 0;
    for (size_t k = 0; k < order.size(); ++k) {
        sorted[k] = pairs[order[k]];
        nstr[k] = sorted[k].nbands;
        xm[k] = steps[order[k]];
        if constexpr (DIRS < 3) {  // DIRS 4 keeps its tile-maxima offset there
            sorted[k].ring_off = ring_elems;
            if (sorted[k].nbands > 1) ring_elems += 2 * (int64_t)e->pr.qlen[sorted[k].q];
        }
    }
    std::vector<int4> entries = band_queue(nstr, xm, warps);
    const size_t n = entries.size();
    if (e->tune[PW_TUNE_STALL_TEST]) {
        // one band below another waits on the spare flag (index n) instead
        for (int4& v : entries)
            if (v.y > 0) {
                e->tune[PW_TUNE_STALL_TEST] = 0;
                v.z = (int)n;
                break;
            }
    }
    if ((c = upload(e, e->band_pairs, sorted)) != cudaSuccess) return cuda_fail(e, c, "upload band pairs");
    if ((c = upload(e, e->band_entries, entries)) != cudaSuccess) return cuda_fail(e, c, "upload band queue");
    if ((c = e->band_prog.reserve(e->stream, (n + 1) * sizeof(int))) != cudaSuccess ||
        (c = e->band_max.reserve(e->stream, n * sizeof(int))) != cudaSuccess ||
        (c = e->band_ring.reserve(e->stream, (size_t)std::max<int64_t>(ring_elems, 1) * sizeof(int4))) != cudaSuccess ||
        (c = e->chain_abort.reserve(e->stream, sizeof(int))) != cudaSuccess)
        return cuda_fail(e, c, "alloc band state");
    if ((c = cudaMemsetAsync(e->band_prog.p, 0, (n + 1) * sizeof(int), e->stream)) != cudaSuccess ||
        (c = cudaMemsetAsync(e->chain_abort.p, 0, sizeof(int), e->stream)) != cudaSuccess ||
        (c = cudaMemsetAsync(e->counter.as<int>() + kNumClasses, 0, sizeof(int), e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "reset band state");
    BandArgs B;
    memset(&B, 0, sizeof(B));
    B.entries = e->band_entries.as<int4>();
    B.pairs = e->band_pairs.as<BandPair>();
    B.n_entries = (int)n;
    B.counter = e->counter.as<int>() + kNumClasses;
    B.ring = e->band_ring.as<int4>();
    B.progress = e->band_prog.as<int>();
    B.run_max = e->band_max.as<int>();
    B.abort_flag = e->chain_abort.as<int>();
    B.max_out = e->band_out.as<float>();
    B.ck = DIRS == 3 ? e->tile_ck.as<int>() : DIRS == 4 ? e->p1_ck.as<int>() : nullptr;
    B.wait_ns = wait_limit(e);
    const int grid = std::max(1, std::min(grid_cap(e, per_sm), (int)((n + 3) / 4)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    PW_LAUNCH(kern, grid, 128, smem, e->stream, A, B);
    e->launches++;
    cudaEventRecord(b, e->stream);
    if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "band sweep launch");
    int aborted = 0;
    if ((c = copy_d2h(e, &aborted, e->chain_abort.p, sizeof(int))) != cudaSuccess ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "band sweep");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (kernel_ms) *kernel_ms += ms;
    if (n_launch) ++*n_launch;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (aborted) return fail(e, PW_ERR_KERNEL, "band sweep: a band waited too long for the band above");
    return PW_OK;
}

// Launches band16_kernel over `pairs` (two explicit pairs a chain, 16x2;
// pw_band16.cuh): maxima into band_out by pair-list index, the pairs past the
// 16-bit limit flagged in band_over, checkpoints and tile maxima into p1_ck.
static int run_band16_phase(pw_engine* e, KernelArgs A, const std::vector<BandPair2>& pairs, int limit,
                            double* kernel_ms, int* n_launch) {
    if (pairs.empty()) return PW_OK;
    const int smem = 4 * kWarp * (A.P.alpha + 1) * kWarpRows * 4;
    cudaError_t c;
    if (smem > 48 * 1024 &&
        (c = cudaFuncSetAttribute(band16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
        return cuda_fail(e, c, "band sweep smem");
    int per_sm = 0;
    if ((c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band16_kernel, 128, smem)) != cudaSuccess)
        return cuda_fail(e, c, "occupancy");
    per_sm = std::max(1, std::min(per_sm, 16));
    const int warps = grid_cap(e, per_sm) * 4;
    std::vector<int> order(pairs.size());
    std::iota(order.begin(), order.end(), 0);
    std::vector<int64_t> steps(pairs.size());
    for (size_t k = 0; k < pairs.size(); ++k) steps[k] = (int64_t)e->pr.qlen[pairs[k].q] + kWarp - 1;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return steps[x] * pairs[x].nbands > steps[y] * pairs[y].nbands;
    });
    std::vector<BandPair2> sorted(pairs.size());
    std::vector<int> nstr(pairs.size());
    std::vector<int64_t> xm(pairs.size());
    for (size_t k = 0; k < order.size(); ++k) {
        sorted[k] = pairs[order[k]];
        nstr[k] = std::max(1, sorted[k].nbands);
        xm[k] = steps[order[k]];
    }
    const std::vector<int4> entries = band_queue(nstr, xm, warps);
    const size_t n = entries.size();
    if ((c = upload(e, e->band_pairs, sorted)) != cudaSuccess) return cuda_fail(e, c, "upload band pairs");
    if ((c = upload(e, e->band_entries, entries)) != cudaSuccess) return cuda_fail(e, c, "upload band queue");
    if ((c = e->band_prog.reserve(e->stream, (n + 1) * sizeof(int))) != cudaSuccess ||
        (c = e->band_max.reserve(e->stream, n * sizeof(int2))) != cudaSuccess ||
        (c = e->chain_abort.reserve(e->stream, sizeof(int))) != cudaSuccess)
        return cuda_fail(e, c, "alloc band state");
    if ((c = cudaMemsetAsync(e->band_prog.p, 0, (n + 1) * sizeof(int), e->stream)) != cudaSuccess ||
        (c = cudaMemsetAsync(e->chain_abort.p, 0, sizeof(int), e->stream)) != cudaSuccess ||
        (c = cudaMemsetAsync(e->counter.as<int>() + kNumClasses, 0, sizeof(int), e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "reset band state");
    BandArgs2 B;
    memset(&B, 0, sizeof(B));
    B.entries = e->band_entries.as<int4>();
    B.pairs = e->band_pairs.as<BandPair2>();
    B.n_entries = (int)n;
    B.counter = e->counter.as<int>() + kNumClasses;
    B.progress = e->band_prog.as<int>();
    B.run_max = e->band_max.as<int2>();
    B.abort_flag = e->chain_abort.as<int>();
    B.max_out = e->band_out.as<float>();
    B.over = e->band_over.as<int>();
    B.ck = e->p1_ck.as<int>();
    B.limit = limit;
    B.wait_ns = wait_limit(e);
    const int grid = std::max(1, std::min(grid_cap(e, per_sm), (int)((n + 3) / 4)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    PW_LAUNCH(band16_kernel, grid, 128, smem, e->stream, A, B);
    e->launches++;
    cudaEventRecord(b, e->stream);
    if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "band sweep launch");
    int aborted = 0;
    if ((c = copy_d2h(e, &aborted, e->chain_abort.p, sizeof(int))) != cudaSuccess ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "band sweep");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (kernel_ms) *kernel_ms += ms;
    if (n_launch) ++*n_launch;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (aborted) return fail(e, PW_ERR_KERNEL, "band sweep: a band waited too long for the band above");
    return PW_OK;
}

// Candidates of tile-form pairs whose checkpoints the score sweep kept
// (band_kernel<false, 4>): the pairs' records and the tiles that reach their
// thresholds (tile_select_kernel), those tiles recomputed with the
// candidate test (tile_cand_kernel), the counts into the records.
static int run_tile_cands(pw_engine* e, KernelArgs A, TileArgs T, const TilePair* dev_list,
                          const std::vector<TilePair>& list, double* kernel_ms, int* n_launch) {
    if (list.empty()) return PW_OK;
    int64_t tiles = 0;
    for (const TilePair& tp : list) {
        const int lq = e->pr.qlen[tp.q], lt = e->pr.tlen[tp.t];
        tiles += (int64_t)(lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1) * tile_count(lq);
    }
    if (tiles > INT32_MAX) return fail(e, PW_ERR_CAPACITY, "tile form: too many tiles in one wave");
    cudaError_t c;
    const int tsmem = tile_smem_bytes(A.P.alpha + 1);
    if ((c = e->tile_sel.reserve(e->stream, (size_t)std::max<int64_t>(tiles, 1) * sizeof(int2))) != cudaSuccess ||
        (c = e->tile_cnt.reserve(e->stream, 4 * sizeof(int))) != cudaSuccess ||
        (c = cudaMemsetAsync(e->tile_cnt.p, 0, 4 * sizeof(int), e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "tile selection");
    if (tsmem > 48 * 1024 &&
        (c = cudaFuncSetAttribute(tile_cand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem)) != cudaSuccess)
        return cuda_fail(e, c, "tile kernels smem");
    int* cnt = e->tile_cnt.as<int>();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    const int n = (int)list.size();
    PW_LAUNCH(tile_select_kernel, n, 256, 0, e->stream, A, T, dev_list, e->tile_sel.as<int2>(), cnt, (int)tiles);
    PW_LAUNCH(tile_cand_kernel, e->sm_count, kWarp, tsmem, e->stream, A, T, dev_list,
              (const int2*)e->tile_sel.as<int2>(), (const int*)cnt, cnt + 1);
    PW_LAUNCH(tile_cand_count_kernel, (n + 127) / 128, 128, 0, e->stream, A, dev_list, n);
    e->launches += 3;
    cudaEventRecord(b, e->stream);
    if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "tile candidates launch");
    if ((c = cudaEventSynchronize(b)) != cudaSuccess) return cuda_fail(e, c, "tile candidates");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (kernel_ms) *kernel_ms += ms;
    if (n_launch) *n_launch += 3;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return PW_OK;
}

// The phase-2 warp items as band pairs.
static std::vector<BandPair> band_pairs_of(pw_engine* e, const std::vector<WorkItem>& items) {
    std::vector<BandPair> v(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        const WorkItem& W = items[k];
        BandPair& p = v[k];
        memset(&p, 0, sizeof(p));
        p.q = W.first;
        p.t = W.target;
        const int lt = e->pr.tlen[W.target];
        p.nbands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
        p.meta_item = W.index;
        p.dir_base = W.dir_base;
        p.slot = W.pair_base;
    }
    return v;
}

static int emit_key_less(const StartRec& a, const StartRec& b) {
    auto k = [](const StartRec& r) {
        return std::make_tuple(-(int64_t)((r.x >> 3) + (r.y >> 3)), -(int64_t)(r.x >> 3), r.target, r.query,
                               -(int64_t)((r.x & 7) + (r.y & 7)), (int64_t)(r.y & 7));
    };
    return k(a) < k(b);
}


extern "C" int pw_align(pw_engine* e, uint32_t flags, int64_t start_cap, pw_run_info* info) {
    if (!e) return PW_ERR_ARG;
    const double t_call = wall_ms();
    if (!e->scoring_set) return fail(e, PW_ERR_STATE, "pw_set_scoring was not called");
    if (!e->Q.set || !e->T.set) return fail(e, PW_ERR_STATE, "queries and targets must be set");
    if (cudaSetDevice(e->device) != cudaSuccess) return fail(e, PW_ERR_DEVICE, "cudaSetDevice failed");
    e->err.clear();
    e->h_hits.clear();
    e->h_strings.clear();
    e->h_starts.clear();
    e->launches = 0;
    e->h2d = e->d2h = 0;
    e->reuse = 0;
    pw_run_info inf;
    memset(&inf, 0, sizeof(inf));
    const int nq = e->Q.n, nt = e->T.n;
    if (!e->h_pair_max.resize((size_t)nq * nt)) return fail(e, PW_ERR_NOMEM, "host pair maxima");
    e->pm_stale = false;
    e->p1_tiles = false;
    inf.pairs = (int64_t)nq * nt;
    int64_t sumq = 0, sumt = 0;
    for (int i = 0; i < nq; ++i) sumq += e->Q.off[i + 1] - e->Q.off[i];
    for (int i = 0; i < nt; ++i) sumt += e->T.off[i + 1] - e->T.off[i];
    inf.cells = sumq * sumt;
    bool pair_mode = !e->pair_q.empty();
    if (pair_mode) {
        inf.pairs = (int64_t)e->pair_q.size();
        inf.cells = 0;
        for (size_t k = 0; k < e->pair_q.size(); ++k) {
            if (e->pair_q[k] < 0 || e->pair_q[k] >= nq || e->pair_t[k] < 0 || e->pair_t[k] >= nt)
                return fail(e, PW_ERR_ARG, "pair list index outside the query or target list");
            inf.cells += (e->Q.off[e->pair_q[k] + 1] - e->Q.off[e->pair_q[k]]) *
                         (e->T.off[e->pair_t[k] + 1] - e->T.off[e->pair_t[k]]);
        }
    }
    if (nq == 0 || nt == 0) {
        inf.h2d_bytes = e->h2d;
        inf.d2h_bytes = e->d2h;
        inf.reuse = e->reuse;
        if (info) *info = inf;
        return PW_OK;
    }
    HostTrace ht0;
    int rc = prepare(e);
    if (rc != PW_OK) return rc;
    ht0.mark("prepare (encodings, uploads)");
    const Prepared& pr = e->pr;
    const std::vector<int32_t>& qlen = pr.qlen;
    const std::vector<int32_t>& tlen = pr.tlen;
    cudaError_t c;
    if ((c = e->pair_max.reserve(e->stream, (size_t)nq * nt * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, c, "alloc pair maxima");
    KernelArgs A = base_args(e);
    const bool plain = (flags & PW_FLAG_PLAIN) != 0;
    if (e->tune[PW_TUNE_LANES] == 32) flags |= PW_FLAG_INT32;  // the tuned lane width

    // ---------------------------------------------------------- phase 1
    // All-vs-all calls too small for the inter-sequence sweeps to give every
    // SM a warp (a few long sequences, e.g. one query against one target and
    // its reverse complement) are swept band by band like explicit pairs.
    std::vector<int32_t> auto_q, auto_t;
    if (!pair_mode && pr.int_path && !plain && !(flags & PW_FLAG_INT32) &&
        (int64_t)((nq + 1) / 2) * ((nt + kWarp - 1) / kWarp) < e->sm_count &&
        (int64_t)((nt + 1) / 2) * ((nq + kWarp - 1) / kWarp) < e->sm_count && inf.cells >= (int64_t)1 << 24) {
        for (int q = 0; q < nq; ++q)
            for (int t = 0; t < nt; ++t) {
                auto_q.push_back(q);
                auto_t.push_back(t);
            }
    }
    const std::vector<int32_t>& list_q = pair_mode ? e->pair_q : auto_q;
    const std::vector<int32_t>& list_t = pair_mode ? e->pair_t : auto_t;
    const bool band1 = !list_q.empty() && pr.int_path && !plain;
    const bool plain_band = plain && pr.int_path;
    const bool use_s16 = !band1 && !plain && (pr.s16_q || pr.s16_t) && !(flags & PW_FLAG_INT32);
    if (band1) {
        // explicit pairs: one warp per 256-row band, bands chained (pw_band.cuh)
        const size_t np = list_q.size();
        std::vector<BandPair> bp(np);
        for (size_t k = 0; k < np; ++k) {
            memset(&bp[k], 0, sizeof(BandPair));
            bp[k].q = list_q[k];
            bp[k].t = list_t[k];
            const int lt = tlen[bp[k].t];
            bp[k].nbands = lt > 0 ? (lt + kBandRows - 1) / kBandRows : 1;
            bp[k].slot = (int64_t)k;
        }
        if ((c = e->band_out.reserve(e->stream, np * sizeof(float))) != cudaSuccess)
            return cuda_fail(e, c, "alloc band maxima");
        // linear integer scoring: the sweep also keeps the tile form's
        // checkpoints and tile maxima (band_kernel<false, 4>), so that the
        // traced pairs need no second sweep -- when they take at most 35% of
        // the free device memory
        bool p1ck = !e->affine && e->tune[PW_TUNE_TILE_TRACE] != 1;
        if (p1ck) {
            e->p1_ck_off.assign(np, 0);
            e->p1_tm_off.assign(np, 0);
            int64_t ck = 0, tm = 0;
            for (size_t k = 0; k < np; ++k) {
                const int lq = qlen[bp[k].q], lt = tlen[bp[k].t];
                e->p1_ck_off[k] = ck;
                ck += tile_checkpoint_ints(lq, lt);
                e->p1_tm_off[k] = tm;
                tm += (int64_t)bp[k].nbands * tile_count(lq);
            }
            // the driver's free-memory query can be held for tens of
            // milliseconds by tools polling the GPU: read at most every 10 s
            const double now = wall_ms();
            if (e->p1_free_t < 0 || now - e->p1_free_t > 10000.0) {
                size_t free_b = 0, total_b = 0;
                cudaMemGetInfo(&free_b, &total_b);
                e->p1_free = (int64_t)free_b + (int64_t)e->p1_ck.bytes;
                e->p1_free_t = now;
            }
            const int64_t bytes = (ck + tm) * (int64_t)sizeof(int);
            p1ck = (double)bytes <= 0.35 * (double)e->p1_free;
            if (p1ck && e->p1_ck.reserve(e->stream, (size_t)bytes) != cudaSuccess) {
                cudaGetLastError();  // no room after all: the traced pairs get the checkpoint sweep
                p1ck = false;
            }
            if (p1ck) {
                if ((c = cudaMemsetAsync(e->p1_ck.as<int>() + ck, 0, (size_t)tm * sizeof(int), e->stream)) != cudaSuccess)
                    return cuda_fail(e, c, "reset tile maxima");
                e->p1_index.clear();
                for (size_t k = 0; k < np; ++k) {
                    e->p1_tm_off[k] += ck;
                    bp[k].dir_base = e->p1_ck_off[k];
                    bp[k].ring_off = e->p1_tm_off[k];
                    e->p1_index.emplace((int64_t)bp[k].q * nt + bp[k].t, (int32_t)k);
                }
            }
        }
        cudaEventRecord(e->ev[0], e->stream);
        if (p1ck) {
            // pairs that share their query and their target's length go two to
            // a 16x2 sweep (pw_band16.cuh); the others, and pairs whose maximum
            // passes the 16-bit limit, run on 32-bit lanes
            const int limit = 32767 - (int)std::ceil(A.P.highest);
            std::vector<BandPair2> bp2;
            std::vector<BandPair> bp1;
            if (!(flags & PW_FLAG_INT32) && limit > 0) {
                std::map<std::pair<int32_t, int32_t>, size_t> open;
                std::vector<char> paired(np, 0);
                for (size_t k = 0; k < np; ++k) {
                    const auto key = std::make_pair(bp[k].q, tlen[bp[k].t]);
                    const auto f = open.find(key);
                    if (f == open.end()) {
                        open.emplace(key, k);
                        continue;
                    }
                    const size_t j = f->second;
                    open.erase(f);
                    BandPair2 p2;
                    memset(&p2, 0, sizeof(p2));
                    p2.q = bp[j].q;
                    p2.t[0] = bp[j].t;
                    p2.t[1] = bp[k].t;
                    p2.nbands = bp[j].nbands;
                    p2.slot[0] = (int64_t)j;
                    p2.slot[1] = (int64_t)k;
                    p2.ck[0] = bp[j].dir_base;
                    p2.ck[1] = bp[k].dir_base;
                    p2.tm[0] = bp[j].ring_off;
                    p2.tm[1] = bp[k].ring_off;
                    bp2.push_back(p2);
                    paired[j] = paired[k] = 1;
                    inf.paired_cells += 2 * (int64_t)qlen[bp[j].q] * tlen[bp[j].t];
                }
                for (size_t k = 0; k < np; ++k)
                    if (!paired[k]) bp1.push_back(bp[k]);
            } else {
                bp1 = bp;
            }
            if (!bp2.empty()) {
                if ((c = e->band_over.reserve(e->stream, np * sizeof(int))) != cudaSuccess ||
                    (c = cudaMemsetAsync(e->band_over.p, 0, np * sizeof(int), e->stream)) != cudaSuccess)
                    return cuda_fail(e, c, "alloc band flags");
                rc = run_band16_phase(e, A, bp2, limit, &inf.score_kernel_ms, &inf.score_launches);
                if (rc != PW_OK) return rc;
                std::vector<int32_t> over;
                if ((c = download(e, over, e->band_over.p, np)) != cudaSuccess) return cuda_fail(e, c, "copy band flags");
                for (size_t k = 0; k < np; ++k) {
                    if (!over[k]) continue;
                    const int lq = qlen[bp[k].q];
                    if ((c = cudaMemsetAsync(e->p1_ck.as<int>() + bp[k].ring_off, 0,
                                             (size_t)bp[k].nbands * tile_count(lq) * sizeof(int), e->stream)) != cudaSuccess)
                        return cuda_fail(e, c, "reset tile maxima");
                    bp1.push_back(bp[k]);
                    inf.overflow_pairs++;
                    inf.paired_cells -= (int64_t)qlen[bp[k].q] * tlen[bp[k].t];
                }
            }
            rc = run_band_phase<4>(e, A, bp1, &inf.score_kernel_ms, &inf.score_launches);
        } else {
            rc = run_band_phase<0>(e, A, bp, &inf.score_kernel_ms, &inf.score_launches);
        }
        if (rc != PW_OK) return rc;
        e->p1_tiles = p1ck;
        cudaEventRecord(e->ev[1], e->stream);
        std::vector<float> bm;
        if ((c = download(e, bm, e->band_out.p, np)) != cudaSuccess) return cuda_fail(e, c, "copy pair maxima");
        e->h_pair_max.fill(-1.0f);
        for (size_t k = 0; k < np; ++k) e->h_pair_max[(size_t)list_q[k] * nt + list_t[k]] = bm[k];
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
        inf.score_ms = ms;
        inf.score_path = 2;
    } else if (plain_band) {
        // the unbatched form: one launch per (query, target) pair, as the
        // reference launches one pair's kernels at a time, each pair on the
        // single-pair wavefront kernel (a warp per 256-row band, the bands of
        // a long pair chained across warps)
        inf.score_path = 3;
        if ((c = e->band_out.reserve(e->stream, sizeof(float))) != cudaSuccess)
            return cuda_fail(e, c, "alloc band maxima");
        e->h_pair_max.fill(-1.0f);
        cudaEventRecord(e->ev[0], e->stream);
        const size_t np = pair_mode ? e->pair_q.size() : (size_t)nq * nt;
        for (size_t k = 0; k < np; ++k) {
            const int q = pair_mode ? e->pair_q[k] : (int)(k / nt);
            const int t = pair_mode ? e->pair_t[k] : (int)(k % nt);
            std::vector<BandPair> bp(1);
            memset(&bp[0], 0, sizeof(BandPair));
            bp[0].q = q;
            bp[0].t = t;
            bp[0].nbands = tlen[t] > 0 ? (tlen[t] + kBandRows - 1) / kBandRows : 1;
            rc = run_band_phase<0>(e, A, bp, &inf.score_kernel_ms, &inf.score_launches);
            if (rc != PW_OK) return rc;
            float m = 0.0f;
            if ((c = copy_d2h(e, &m, e->band_out.p, sizeof(float))) != cudaSuccess ||
                (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "copy pair maximum");
            e->h_pair_max[(size_t)q * nt + t] = m;
        }
        cudaEventRecord(e->ev[1], e->stream);
        cudaStreamSynchronize(e->stream);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
        inf.score_ms = ms;
    } else if (use_s16) {
        cudaEventRecord(e->ev[0], e->stream);
        rc = phase1_s16(e, A, inf, flags);
        if (rc != PW_OK) return rc;
        cudaEventRecord(e->ev[1], e->stream);
        cudaStreamSynchronize(e->stream);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
        inf.score_ms = ms;
        ht0.mark("score phase (16-bit, wall)");
    } else {
        inf.score_path = 1;
    // items: one target against 32 consecutive queries of the length order
        std::vector<WorkItem> items;
        std::vector<int> cls;
        for (int t = 0; t < nt; ++t)
            for (int g = 0; g < nq; g += (plain ? 1 : kWarp)) {
                WorkItem w;
                memset(&w, 0, sizeof(w));
                w.target = t;
                w.first = g;
                w.lanes = plain ? 1 : std::min(kWarp, nq - g);
                w.xmax = qlen[pr.order[g]];
                const int k = pick_class(tlen[t], e->affine);
                w.S = class_S(k);
                items.push_back(w);
                cls.push_back(k);
            }
        // largest work first inside each class (dynamic scheduling tail)
        std::vector<int64_t> cost(items.size());
        for (size_t k = 0; k < items.size(); ++k) cost[k] = (int64_t)items[k].xmax * tlen[items[k].target];
        const std::vector<uint32_t> idx = class_cost_order(cls, cost);
        std::vector<WorkItem> it2(items.size());
        std::vector<int> c2(items.size());
        for (size_t k = 0; k < idx.size(); ++k) {
            it2[k] = items[idx[k]];
            c2[k] = cls[idx[k]];
        }
        int begin[kNumClasses + 1];
        for (int k = 0; k <= kNumClasses; ++k) begin[k] = 0;
        for (int k : c2) begin[k + 1]++;
        for (int k = 0; k < kNumClasses; ++k) begin[k + 1] += begin[k];
        int xm = 4;
        for (int k = begin[kS32Multi]; k < begin[kS32Multi + 1]; ++k) xm = std::max(xm, (int)align_up(it2[k].xmax, 4));
        if ((c = upload(e, e->items, it2)) != cudaSuccess) return cuda_fail(e, c, "upload items");
        cudaEventRecord(e->ev[0], e->stream);
        if (plain) {
            // the unbatched form: one launch per (query, target) pair
            for (size_t k = 0; k < it2.size(); ++k) {
                int b1[kNumClasses + 1];
                for (int q = 0; q <= kNumClasses; ++q) b1[q] = (q > c2[k]) ? 1 : 0;
                rc = run_phase<1>(e, A, e->items.as<WorkItem>() + k, b1, xm, &inf.score_kernel_ms,
                                  &inf.score_launches);
                if (rc != PW_OK) return rc;
            }
        } else {
            rc = run_phase<1>(e, A, e->items.as<WorkItem>(), begin, xm, &inf.score_kernel_ms, &inf.score_launches);
            if (rc != PW_OK) return rc;
        }
        cudaEventRecord(e->ev[1], e->stream);
        if ((c = cudaEventSynchronize(e->ev[1])) != cudaSuccess) return cuda_fail(e, c, "score sweep");
        e->pm_stale = true;
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
        inf.score_ms = ms;
    }
    if ((band1 || plain_band) && !pair_mode) {
        // the band sweep wrote host maxima only: the trace kernels read them on the device
        if ((c = copy_h2d(e, A.pair_max, e->h_pair_max.data(), e->h_pair_max.size() * sizeof(float))) != cudaSuccess ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "upload pair maxima");
    }
    if (pair_mode) {
        // pairs outside the list get -1: below MINIMUM_SCORE, never traced
        if (const int r = sync_pair_max(e, A.pair_max)) return r;
        std::vector<uint8_t> listed((size_t)nq * nt, 0);
        for (size_t k = 0; k < e->pair_q.size(); ++k) listed[(size_t)e->pair_q[k] * nt + e->pair_t[k]] = 1;
        for (size_t k = 0; k < listed.size(); ++k)
            if (!listed[k]) e->h_pair_max[k] = -1.0f;
        if ((c = copy_h2d(e, A.pair_max, e->h_pair_max.data(), e->h_pair_max.size() * sizeof(float))) != cudaSuccess ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "upload pair maxima");
    }
    if (flags & PW_FLAG_SCORE_ONLY) {
        inf.kernel_launches = (int32_t)e->launches;
        inf.total_ms = wall_ms() - t_call;
        inf.h2d_bytes = e->h2d;
        inf.d2h_bytes = e->d2h;
        inf.reuse = e->reuse;
        if (info) *info = inf;
        return PW_OK;
    }

    // ---------------------------------------------------------- phase 2
    const double t_setup = wall_ms();
    HostTrace ht;
    // Pairs that can yield a starting point, per target in query length order,
    // 32 per work item.  The reference traces every pair whose maximum reaches
    // MINIMUM_SCORE (default_main.cu:596), but a starting point also needs a
    // cell with H >= max(LOWER_LIMIT_SCORE * max, maxPossibleScore) (:609) and
    // no cell exceeds the pair maximum, so a pair whose maximum is below that
    // threshold has no starting point and contributes nothing: it is skipped.
    // passing pairs per target, query length order: pt_q[pt_off[t] .. pt_off[t + 1])
    std::vector<int64_t> pt_off((size_t)nt + 1, 0);
    HostBuf<int32_t>& pt_q = e->h_ptq;
    pt_q.clear();
    int64_t min_pass = 0, n_pass = 0, max_pass = 0;
    {
        // the test runs on the device over the resident maxima (prune_kernel);
        // the passing pairs come back as a target-major list of pair indices
        const int64_t npairs = (int64_t)nq * nt;
        unsigned long long cnt[4] = {0, 0, 0, 0};
        if ((c = e->prune_flags.reserve(e->stream, (size_t)std::max<int64_t>(npairs, 16))) != cudaSuccess ||
            (c = e->prune_cnt.reserve(e->stream, 4 * sizeof(unsigned long long))) != cudaSuccess ||
            (c = cudaMemsetAsync(e->prune_cnt.p, 0, 4 * sizeof(unsigned long long), e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "alloc pruning flags");
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((npairs + 255) / 256, (int64_t)e->sm_count * 16));
        PW_LAUNCH(prune_kernel, grid, 256, 0, e->stream, (const float*)A.pair_max, e->q_order.as<int32_t>(),
                  e->q_len.as<int32_t>(), e->t_len.as<int32_t>(), nq, nt, e->minimum_score, e->highest,
                  e->filter_factor, e->lower_limit,
                  e->q_trace_set ? (const uint8_t*)e->q_trace.as<uint8_t>() : (const uint8_t*)nullptr,
                  e->prune_flags.as<uint8_t>(), e->prune_cnt.as<unsigned long long>());
        e->launches++;
        if ((c = cudaGetLastError()) != cudaSuccess ||
            (c = copy_d2h(e, cnt, e->prune_cnt.p, sizeof(cnt))) != cudaSuccess ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "prune pairs");
        min_pass = (int64_t)cnt[0];
        n_pass = (int64_t)cnt[1];
        max_pass = (int64_t)cnt[3];
        ht.mark("prune kernel + counts");
        if (n_pass > 0) {
            int64_t* d_count = e->prune_cnt.as<int64_t>() + 2;
            thrust::counting_iterator<int64_t> ids(0);
            size_t tmp_bytes = 0;
            if ((c = cub::DeviceSelect::Flagged(nullptr, tmp_bytes, ids, e->prune_flags.as<uint8_t>(), (int64_t*)nullptr,
                                                d_count, npairs, e->stream)) != cudaSuccess ||
                (c = e->scan_tmp.reserve(e->stream, std::max<size_t>(tmp_bytes, 16))) != cudaSuccess ||
                (c = e->prune_sel.reserve(e->stream, (size_t)n_pass * sizeof(int64_t))) != cudaSuccess ||
                (c = cub::DeviceSelect::Flagged(e->scan_tmp.p, tmp_bytes, ids, e->prune_flags.as<uint8_t>(),
                                                e->prune_sel.as<int64_t>(), d_count, npairs, e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "select passing pairs");
            if (!e->h_sel.resize((size_t)n_pass)) return fail(e, PW_ERR_NOMEM, "host memory for the passing pairs");
            if ((c = copy_d2h(e, e->h_sel.data(), e->prune_sel.p, (size_t)n_pass * sizeof(int64_t))) != cudaSuccess ||
                (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "copy passing pairs");
            const int64_t* sel = e->h_sel.data();
            for (int t = 0; t <= nt; ++t) pt_off[t] = std::lower_bound(sel, sel + n_pass, (int64_t)t * nq) - sel;
            if (!pt_q.resize((size_t)n_pass)) return fail(e, PW_ERR_NOMEM, "host memory for the passing pairs");
            std::mutex mu;
            parallel_for(n_pass, [&](int64_t j0, int64_t j1) {
                int64_t tc = 0;
                for (int64_t j = j0; j < j1; ++j) {
                    const int t = (int)(sel[j] / nq);
                    const int q = pr.order[(size_t)(sel[j] - (int64_t)t * nq)];
                    pt_q[j] = q;
                    tc += (int64_t)qlen[q] * tlen[t];
                }
                std::lock_guard<std::mutex> g(mu);
                inf.traced_cells += tc;
            }, (int64_t)1 << 16);
        }
        ht.mark("passing pairs to per-target lists");
    }
    auto span_n = [&](int t) -> int64_t { return pt_off[t + 1] - pt_off[t]; };
    // Traced pairs with targets longer than one register strip go to the
    // one-warp-per-pair sweep (pw_band.cuh); the others are grouped 32 to
    // a warp, one pair per lane, in the orientation where they cluster
    // (slot cost = strip length x longest lane x 32 per item).
    const bool warp_ok = pr.int_path;
    std::vector<std::pair<int32_t, int32_t>> warp_pairs;  // (query, target)
    std::vector<char> t_warp((size_t)nt, 0);              // targets whose pairs went to the warp sweep
    if (warp_ok) {
        // short targets stay on the strip sweep only when there are enough of
        // them to give every SM a full warp: a few strip items run one lane per
        // pair, latency bound, far longer than the same pairs one per warp
        int64_t n_short = 0;
        for (int t = 0; t < nt; ++t)
            if (tlen[t] <= 64) n_short += span_n(t);
        // (the unbatched form sweeps every traced pair alone on a warp)
        const bool all_warp = plain || n_short < (int64_t)kWarp * e->sm_count;
        for (int t = 0; t < nt; ++t) {
            if (tlen[t] <= 64 && !all_warp) continue;
            for (int64_t j = pt_off[t]; j < pt_off[t + 1]; ++j) warp_pairs.push_back({pt_q[j], t});
            t_warp[t] = 1;
        }
    }
    auto live_n = [&](int t) -> int64_t { return t_warp[t] ? 0 : span_n(t); };
    ht.mark("warp-sweep routing");
    // Linear integer scoring whose traced maxima all stay below 2^15, with
    // most traced cells on the strip sweep: the direction sweeps store each
    // cell's 16-bit H (four times the bytes of a 4-bit code, a few
    // instructions a cell instead of the classification); collect and walk
    // derive the codes of the cells they visit.  Long pairs (the one-warp
    // band sweep) keep the codes: their multi-kilobase walks read one code
    // per step instead of up to four H values, and their cells fit fewer
    // memory waves.
    int64_t warp_cells = 0;
    for (const auto& wp : warp_pairs) warp_cells += (int64_t)qlen[wp.first] * tlen[wp.second];
    // Long pairs of linear integer scoring take the tile form (pw_tiles.cuh):
    // no cell codes at all, so the strip sweep's items decide the store alone.
    const int64_t store_mode = e->tune[PW_TUNE_TRACE_STORE];
    const bool tile_form = pr.int_path && !e->affine && e->tune[PW_TUNE_TILE_TRACE] != 1 && !warp_pairs.empty();
    const bool hstore = pr.int_path && !e->affine && max_pass < 32767 && store_mode != 1 &&
                        (store_mode == 2 || (tile_form ? inf.traced_cells > warp_cells
                                                       : inf.traced_cells - warp_cells >= warp_cells));
    inf.trace_store = hstore ? 1 : 0;
    inf.tile_pairs = tile_form ? (int32_t)warp_pairs.size() : 0;
    // the traced long pairs' checkpoints and tile maxima from the score sweep
    const bool p1ck = tile_form && e->p1_tiles;
    const int per_item = plain ? 1 : kWarp;
    double cost_t = 0, cost_q = 0;
    for (int t = 0; t < nt; ++t)
        for (int64_t g = 0; g < live_n(t); g += per_item) cost_t += (double)tlen[t] * qlen[pt_q[pt_off[t] + g]] * per_item;
    // the transposed orientation (queries as strips) can only win if even a
    // lower bound of its slot cost -- every query's groups paying the
    // shortest target -- is below the cost of the direct one; the per-query
    // group counts of that bound are summed on the device
    bool trans2 = false;
    std::vector<std::vector<int32_t>> pass_q;  // per query: passing targets, length order (when needed)
    if (n_pass > 0 && cost_t > 0) {
        int tmin = INT32_MAX;
        for (int t = 0; t < nt; ++t) tmin = std::min(tmin, std::max(tlen[t], 1));
        std::vector<uint8_t> skip(t_warp.begin(), t_warp.end());
        unsigned long long lb_units = 0;  // sum over queries of ceil(k / per_item) * per_item * len
        if ((c = upload(e, e->t_skip, skip)) != cudaSuccess ||
            (c = e->q_count.reserve(e->stream, (size_t)nq * sizeof(int32_t))) != cudaSuccess ||
            (c = cudaMemsetAsync(e->q_count.p, 0, (size_t)nq * sizeof(int32_t), e->stream)) != cudaSuccess ||
            (c = cudaMemsetAsync(e->prune_cnt.p, 0, sizeof(unsigned long long), e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "query counts");
        const int g1 = (int)std::max<int64_t>(1, std::min<int64_t>((n_pass + 255) / 256, (int64_t)e->sm_count * 16));
        PW_LAUNCH(query_count_kernel, g1, 256, 0, e->stream, (const int64_t*)e->prune_sel.as<int64_t>(), n_pass, nq,
                  e->q_order.as<int32_t>(), e->t_skip.as<uint8_t>(), e->q_count.as<int32_t>());
        const int g2 = (int)std::max<int64_t>(1, std::min<int64_t>((nq + 255) / 256, (int64_t)e->sm_count * 16));
        PW_LAUNCH(group_bound_kernel, g2, 256, 0, e->stream, (const int32_t*)e->q_count.as<int32_t>(), nq,
                  e->q_len.as<int32_t>(), per_item, e->prune_cnt.as<unsigned long long>());
        e->launches += 2;
        if ((c = cudaGetLastError()) != cudaSuccess ||
            (c = copy_d2h(e, &lb_units, e->prune_cnt.p, sizeof(lb_units))) !=
                cudaSuccess ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "query counts");
        const double lb_q = (double)lb_units * tmin;
        if (lb_q < cost_t) {
            pass_q.resize(nq);
            std::vector<int32_t> rank_t(nt);
            for (int k = 0; k < nt; ++k) rank_t[pr.order_t[k]] = k;
            for (int t = 0; t < nt; ++t)
                for (int64_t j = pt_off[t]; j < pt_off[t] + live_n(t); ++j) pass_q[pt_q[j]].push_back(t);
            for (int q = 0; q < nq; ++q)
                std::stable_sort(pass_q[q].begin(), pass_q[q].end(),
                                 [&](int a, int b) { return rank_t[a] < rank_t[b]; });
            for (int q = 0; q < nq; ++q)
                for (size_t g = 0; g < pass_q[q].size(); g += per_item)
                    cost_q += (double)qlen[q] * tlen[pass_q[q][g]] * per_item;
            trans2 = cost_q < cost_t;
        }
    }
    ht.mark("phase-2 orientation");
    const int n_strip = trans2 ? nq : nt;
    // per strip: its pairs and items at offsets from prefix sums, filled by host threads
    std::vector<int64_t> s_pairs((size_t)n_strip + 1, 0), s_items((size_t)n_strip + 1, 0);
    for (int st = 0; st < n_strip; ++st) {
        const int64_t np_ = trans2 ? (int64_t)pass_q[st].size() : live_n(st);
        s_pairs[st + 1] = s_pairs[st] + np_;
        s_items[st + 1] = s_items[st] + (np_ + per_item - 1) / per_item;
    }
    HostBuf<int32_t>& p2_order = e->h_p2order;
    if (!p2_order.resize((size_t)s_pairs[n_strip])) return fail(e, PW_ERR_NOMEM, "host memory for the phase-2 order");
    std::vector<WorkItem> items2((size_t)s_items[n_strip]);
    std::vector<int> cls2((size_t)s_items[n_strip]);
    std::vector<int64_t> bytes2((size_t)s_items[n_strip]);
    parallel_for(n_strip, [&](int64_t s0, int64_t s1) {
        for (int64_t st = s0; st < s1; ++st) {
            const int32_t* pass = trans2 ? pass_q[st].data() : pt_q.data() + pt_off[st];
            const int64_t np_ = s_pairs[st + 1] - s_pairs[st];
            const int ls = trans2 ? qlen[st] : tlen[st];
            const int k = pick_class(ls, e->affine);
            const int S = class_S(k);
            const int64_t strips = std::max<int64_t>((ls + S - 1) / S, 1);
            int64_t it = s_items[st];
            for (int64_t g = 0; g < np_; g += per_item, ++it) {
                WorkItem w;
                memset(&w, 0, sizeof(w));
                w.target = (int32_t)st;
                w.first = (int32_t)(s_pairs[st] + g);
                w.lanes = (int32_t)std::min<int64_t>(per_item, np_ - g);
                std::memcpy(p2_order.data() + w.first, pass + g, (size_t)w.lanes * sizeof(int32_t));
                w.xmax = trans2 ? tlen[pass[g]] : qlen[pass[g]];
                w.orient = trans2 ? 1 : 0;
                w.S = S;
                items2[it] = w;
                cls2[it] = k;
                const int64_t cells = strips * S * align_up(std::max(w.xmax, 1), 4) * kWarp;
                bytes2[it] = hstore ? cells * 2 : cells / 2;  // 16-bit H or 4-bit codes
            }
        }
    }, std::max<int64_t>(1, (int64_t)n_strip * ((int64_t)1 << 15) / std::max<int64_t>(s_pairs[n_strip], 1)));
    // warp items: longest first (dynamic scheduling tail)
    std::stable_sort(warp_pairs.begin(), warp_pairs.end(), [&](const std::pair<int32_t, int32_t>& a,
                                                               const std::pair<int32_t, int32_t>& b) {
        return (int64_t)qlen[a.first] * tlen[a.second] > (int64_t)qlen[b.first] * tlen[b.second];
    });
    int qmax_warp = 1;
    inf.warp_pairs = (int64_t)warp_pairs.size();
    for (const auto& wp : warp_pairs) {
        WorkItem w;
        memset(&w, 0, sizeof(w));
        w.target = wp.second;
        w.first = wp.first;
        w.lanes = 1;
        w.xmax = qlen[wp.first];
        w.orient = 2;
        w.S = kWarpRows;
        items2.push_back(w);
        cls2.push_back(kNumClasses);  // marks a warp item
        // tile form: checkpoints and the mark plane; else cell codes (or H)
        // (the score sweep's checkpoints, when it kept them, are not the wave's)
        bytes2.push_back(tile_form ? (p1ck ? 0 : tile_checkpoint_ints(qlen[wp.first], tlen[wp.second]) * 4) +
                                         align_up(((int64_t)qlen[wp.first] * tlen[wp.second] + 31) / 32 * 4, 16)
                                   : align_up(warp_code_bytes(qlen[wp.first], tlen[wp.second], hstore), 16));
        qmax_warp = std::max(qmax_warp, qlen[wp.first]);
    }
    ht.mark("phase-2 work items");
    inf.traced_pairs = n_pass;
    inf.minimum_pairs = min_pass;
    inf.trace_orientation = trans2 ? 1 : 0;
    if (items2.empty()) {
        inf.kernel_launches = (int32_t)e->launches;
        inf.total_ms = wall_ms() - t_call;
        inf.h2d_bytes = e->h2d;
        inf.d2h_bytes = e->d2h;
        inf.reuse = e->reuse;
        if (info) *info = inf;
        return PW_OK;
    }
    if ((c = upload(e, e->q_order2, p2_order)) != cudaSuccess) return cuda_fail(e, c, "upload phase-2 order");
    A.q_order = e->q_order2.as<int32_t>();
    if (trans2) {
        // lanes sweep targets (compact target codes), strips are queries
        A.q = SeqSet{e->t_ccodes.as<uint8_t>(), e->t_code_off.as<int64_t>(), e->t_raw.as<uint8_t>(),
                     e->t_raw_off.as<int64_t>(), e->t_len.as<int32_t>(), e->t_key.as<int32_t>()};
        A.t = SeqSet{e->q_res.as<uint8_t>(), e->q_code_off.as<int64_t>(), e->q_raw.as<uint8_t>(),
                     e->q_raw_off.as<int64_t>(), e->q_len.as<int32_t>(), e->q_key.as<int32_t>()};
        A.cmat_i8 = e->cmat_t8.as<int8_t>();
        A.cmat_f = e->cmat_tf.as<float>();
        A.P.alpha = pr.alpha_t;
        A.pm_lane = 1;
        A.pm_strip = nt;
    }
    const KernelArgs Aref = base_args(e);  // reference-oriented sets for the trace kernels

    // memory waves: the cell codes of one wave must fit the budget (set by
    // pw_set_wave_limit); the automatic budget, 55% of the free memory plus
    // the buffers kept from the previous call, also counts each pair's
    // candidate slot and bookkeeping
    int64_t budget = e->wave_limit;
    const bool auto_budget = budget <= 0;
    if (auto_budget) {
        // the free-memory query goes to the driver, which tools polling the
        // GPU (nvidia-smi) can hold for tens of milliseconds: it is refreshed
        // at most every 10 s (the budget is a fraction of it, and an allocation
        // that still fails is reported)
        const double now = wall_ms();
        if (e->free_mem_t < 0 || now - e->free_mem_t > 10000.0) {
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            e->free_mem = (int64_t)free_b + (int64_t)(e->codes.bytes + e->marks.bytes + e->cands.bytes +
                                                      e->metas.bytes);
            e->free_mem_t = now;
        }
        const int64_t kept = (int64_t)(e->codes.bytes + e->marks.bytes + e->cands.bytes + e->metas.bytes);
        budget = std::min<int64_t>((int64_t)(std::max<int64_t>(e->free_mem - kept, 0) * 0.55) + kept,
                                   (int64_t)100 << 30);
    }
    const int64_t pair_bytes = auto_budget ? (int64_t)(kCandCap * sizeof(Cand) + sizeof(PairMeta)) + 64 : 0;
    std::vector<std::pair<size_t, size_t>> waves;
    {
        size_t i0 = 0;
        int64_t acc = 0;
        for (size_t i = 0; i < items2.size(); ++i) {
            const bool tile_item = tile_form && cls2[i] == kNumClasses;  // its marks are in bytes2
            const int64_t b = bytes2[i] + (tile_item ? 0 : bytes2[i] / (hstore ? 16 : 4)) + items2[i].lanes * pair_bytes;
            if (acc > 0 && (acc + b > budget || plain)) {
                waves.push_back({i0, i});
                i0 = i;
                acc = 0;
            }
            acc += b;
        }
        waves.push_back({i0, items2.size()});
    }
    inf.waves = (int32_t)waves.size();

    double trace_ms = 0, walk_ms = 0;
    int64_t total_starts = 0;
    int64_t acc_n = 0, acc_ops = 0;  // hits and operation bytes accumulated over the waves
    inf.setup_ms += wall_ms() - t_setup;
    for (size_t wv = 0; wv < waves.size(); ++wv) {
        const size_t i0 = waves[wv].first, i1 = waves[wv].second;
        std::vector<WorkItem> wi(items2.begin() + i0, items2.begin() + i1);
        std::vector<int> wc(cls2.begin() + i0, cls2.begin() + i1);
        int64_t dir_off = 0, n_pairs = 0;
        int64_t ck_ints = 0, mark_words = 0, scratch_bytes = 0;  // tile form: checkpoints, mark planes, walk scratch
        std::vector<TilePair> tps;
        for (size_t k = 0; k < wi.size(); ++k) {
            wi[k].index = (int32_t)k;
            wi[k].pair_base = n_pairs;
            if (tile_form && wc[k] == kNumClasses) {
                TilePair tp;
                memset(&tp, 0, sizeof(tp));
                const int lq_ = qlen[wi[k].first], lt_ = tlen[wi[k].target];
                tp.q = wi[k].first;
                tp.t = wi[k].target;
                tp.slot = (int32_t)n_pairs;
                tp.marks = mark_words;
                tp.scratch = scratch_bytes;
                scratch_bytes += align_up((int64_t)lq_ + lt_ + 32, 16);
                if (p1ck) {
                    const auto f = e->p1_index.find((int64_t)tp.q * nt + tp.t);
                    if (f == e->p1_index.end()) return fail(e, PW_ERR_STATE, "traced pair without checkpoints");
                    tp.ck = e->p1_ck_off[f->second];
                    tp.tm = e->p1_tm_off[f->second];
                } else {
                    tp.ck = ck_ints;
                    wi[k].dir_base = ck_ints;  // band_kernel<false, 3>: the pair's checkpoints
                    ck_ints += tile_checkpoint_ints(lq_, lt_);
                }
                tps.push_back(tp);
                mark_words += align_up(((int64_t)lq_ * lt_ + 31) / 32, 4);
            } else {
                wi[k].dir_base = dir_off;
                dir_off += bytes2[i0 + k];
            }
            n_pairs += wi[k].lanes;
        }
        std::vector<WorkItem> by_index = wi;  // trace kernels index items by wave position
        std::vector<WorkItem> ww;              // one-warp-per-pair items
        {
            std::vector<WorkItem> ws;
            std::vector<int> wsc;
            for (size_t k = 0; k < wi.size(); ++k) {
                if (wc[k] == kNumClasses) {
                    ww.push_back(wi[k]);
                } else {
                    ws.push_back(wi[k]);
                    wsc.push_back(wc[k]);
                }
            }
            wi.swap(ws);
            wc.swap(wsc);
        }
        int begin[kNumClasses + 1];
        order_by_class(wi, wc, begin);
        int xm = 4;
        for (int k = begin[kS32Multi]; k < begin[kS32Multi + 1]; ++k) xm = std::max(xm, (int)align_up(wi[k].xmax, 4));
        if ((c = e->codes.reserve(e->stream, (size_t)dir_off)) != cudaSuccess) return cuda_fail(e, c, "alloc cell codes");
        // one mark bit per cell (two cells per code byte, half a cell per H
        // byte), zeroed for the wave
        const size_t mark_bytes = (size_t)(dir_off / (hstore ? 16 : 4) + 16);
        if ((c = e->marks.reserve(e->stream, mark_bytes)) != cudaSuccess ||
            (c = cudaMemsetAsync(e->marks.p, 0, mark_bytes, e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "alloc cell marks");
        const int n_tile = (int)tps.size();
        if (n_tile > 0) {
            std::vector<int32_t> slot_tile((size_t)n_pairs, -1);
            for (int k = 0; k < n_tile; ++k) slot_tile[tps[k].slot] = k;
            if ((!p1ck && (c = e->tile_ck.reserve(e->stream, (size_t)ck_ints * sizeof(int))) != cudaSuccess) ||
                (c = e->tile_scratch.reserve(e->stream, (size_t)scratch_bytes)) != cudaSuccess ||
                (c = e->tile_acc.reserve(e->stream, 4 * sizeof(unsigned long long))) != cudaSuccess ||
                (c = cudaMemsetAsync(e->tile_acc.p, 0, 4 * sizeof(unsigned long long), e->stream)) != cudaSuccess ||
                (c = e->tile_marks.reserve(e->stream, (size_t)mark_words * 4)) != cudaSuccess ||
                (c = cudaMemsetAsync(e->tile_marks.p, 0, (size_t)mark_words * 4, e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "alloc tile-form checkpoints");
            if ((c = upload(e, e->tile_pairs, tps)) != cudaSuccess || (c = upload(e, e->slot_tile, slot_tile)) != cudaSuccess)
                return cuda_fail(e, c, "upload tile pairs");
        }
        TileArgs TT;
        memset(&TT, 0, sizeof(TT));
        TT.pairs = n_tile > 0 ? e->tile_pairs.as<TilePair>() : nullptr;
        TT.n_pairs = n_tile;
        TT.ck = n_tile == 0 ? nullptr : p1ck ? e->p1_ck.as<int>() : e->tile_ck.as<int>();
        TT.marks = n_tile > 0 ? e->tile_marks.as<uint32_t>() : nullptr;
        TT.slot_tile = n_tile > 0 ? e->slot_tile.as<int32_t>() : nullptr;
        TT.scratch = n_tile > 0 ? e->tile_scratch.as<char>() : nullptr;
        TT.ops_bound = n_tile > 0 ? e->tile_acc.as<unsigned long long>() : nullptr;
        TT.ops_total = n_tile > 0 ? e->tile_acc.as<unsigned long long>() + 1 : nullptr;
        const int tsmem = tile_smem_bytes(Aref.P.alpha + 1);
        if (n_tile > 0 && tsmem > 48 * 1024) {
            if ((c = cudaFuncSetAttribute(tile_collect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem)) != cudaSuccess ||
                (c = cudaFuncSetAttribute(tile_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem)) != cudaSuccess ||
                (c = cudaFuncSetAttribute(tile_ops_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem)) != cudaSuccess)
                return cuda_fail(e, c, "tile kernels smem");
        }
        if ((c = e->metas.reserve(e->stream, n_pairs * sizeof(PairMeta))) != cudaSuccess) return cuda_fail(e, c, "alloc metas");
        if ((c = e->n_cand.reserve(e->stream, n_pairs * sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, c, "alloc");
        if ((c = e->n_starts.reserve(e->stream, n_pairs * sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, c, "alloc");
        // every pair starts with a slot of kCandCap candidates, filled on the
        // device (PW_TUNE_CAND_SLOT: another capacity); pairs that outgrow it
        // are swept again with an exact slot
        const int64_t slot_tune = e->tune[PW_TUNE_CAND_SLOT];
        const int cap0 = slot_tune > 0 ? (int)std::min<int64_t>(slot_tune, (int64_t)1 << 20) : kCandCap;
        int64_t cand_total = n_pairs * cap0;
        if ((c = e->cand_base.reserve(e->stream, (size_t)std::max<int64_t>(n_pairs, 2) * sizeof(int64_t))) != cudaSuccess ||
            (c = e->cand_cap.reserve(e->stream, (size_t)std::max<int64_t>(n_pairs, 4) * sizeof(int32_t))) != cudaSuccess)
            return cuda_fail(e, c, "alloc candidate slots");
        const int gslot = (int)std::max<int64_t>(1, std::min<int64_t>((n_pairs + 255) / 256, (int64_t)e->sm_count * 16));
        PW_LAUNCH(cand_slot_kernel, gslot, 256, 0, e->stream, e->cand_base.as<int64_t>(), e->cand_cap.as<int32_t>(),
                  n_pairs, cap0);
        e->launches++;
        if ((c = e->cands.reserve(e->stream, cand_total * sizeof(Cand))) != cudaSuccess) return cuda_fail(e, c, "alloc cands");
        if ((c = upload(e, e->items, wi)) != cudaSuccess) return cuda_fail(e, c, "upload items");
        ht.mark("wave buffers");
        A.codes = e->codes.as<uint8_t>();
        A.metas = e->metas.as<PairMeta>();
        A.cands = e->cands.as<Cand>();
        A.cand_base = e->cand_base.as<int64_t>();
        A.cand_cap = e->cand_cap.as<int32_t>();
        A.n_cand = e->n_cand.as<int32_t>();
        KernelArgs Aw = Aref;  // the warp sweep runs in the reference orientation
        Aw.codes = A.codes;
        Aw.metas = A.metas;
        Aw.cands = A.cands;
        Aw.cand_base = A.cand_base;
        Aw.cand_cap = A.cand_cap;
        Aw.n_cand = A.n_cand;
        cudaEventRecord(e->ev[0], e->stream);
        if ((c = cudaMemsetAsync(A.n_cand, 0, n_pairs * sizeof(int32_t), e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "reset candidate counts");
        if (!wi.empty()) {
            rc = hstore ? run_phase<3>(e, A, e->items.as<WorkItem>(), begin, xm, &inf.trace_kernel_ms,
                                       &inf.trace_launches, trans2)
                        : run_phase<2>(e, A, e->items.as<WorkItem>(), begin, xm, &inf.trace_kernel_ms,
                                       &inf.trace_launches, trans2);
            if (rc != PW_OK) return rc;
        }
        {
            std::vector<BandPair> bp = band_pairs_of(e, ww);
            rc = p1ck ? run_tile_cands(e, Aw, TT, TT.pairs, tps, &inf.trace_kernel_ms, &inf.trace_launches)
                 : tile_form ? run_band_phase<3>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches)
                 : hstore  ? run_band_phase<2>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches)
                           : run_band_phase<1>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches);
            if (rc != PW_OK) return rc;
        }
        // candidate overflow: pairs with more candidates than their slot get an
        // exact slot past the regular ones, and their items are swept again
        // (counted on the device; the host reads the per-pair counts only then)
        unsigned long long n_over = 0;
        if ((c = e->prune_cnt.reserve(e->stream, 4 * sizeof(unsigned long long))) != cudaSuccess ||
            (c = cudaMemsetAsync(e->prune_cnt.p, 0, sizeof(unsigned long long), e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "candidate overflow count");
        PW_LAUNCH(cand_overflow_kernel, gslot, 256, 0, e->stream, (const int32_t*)A.n_cand, (const int32_t*)A.cand_cap,
                  n_pairs, e->prune_cnt.as<unsigned long long>());
        e->launches++;
        if ((c = copy_d2h(e, &n_over, e->prune_cnt.p, sizeof(n_over))) !=
                cudaSuccess ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "candidate overflow count");
        ht.mark("direction sweep");
        std::vector<int32_t> ncand;
        std::vector<int64_t> cbase;
        std::vector<int32_t> ccap;
        std::vector<char> over;  // pairs that outgrew their slot
        int64_t extra = 0;
        if (n_over > 0) {
            over.assign((size_t)n_pairs, 0);
            if ((c = download(e, ncand, A.n_cand, (size_t)n_pairs)) != cudaSuccess ||
                (c = download(e, cbase, A.cand_base, (size_t)n_pairs)) != cudaSuccess ||
                (c = download(e, ccap, A.cand_cap, (size_t)n_pairs)) != cudaSuccess)
                return cuda_fail(e, c, "copy");
            for (int64_t p = 0; p < n_pairs; ++p) {
                if (ncand[p] > ccap[p]) {
                    over[p] = 1;
                    inf.cand_overflow_pairs++;
                    cbase[p] = cand_total + extra;
                    ccap[p] = ncand[p];
                    extra += ncand[p];
                }
            }
        }
        if (extra > 0) {
            DevBuf& nb = e->cands_alt;
            if ((c = nb.reserve(e->stream, (cand_total + extra) * sizeof(Cand))) != cudaSuccess)
                return cuda_fail(e, c, "alloc cands");
            c = cudaMemcpyAsync(nb.p, e->cands.p, cand_total * sizeof(Cand), cudaMemcpyDeviceToDevice, e->stream);
            if (c != cudaSuccess) return cuda_fail(e, c, "copy cands");
            std::swap(e->cands.p, nb.p);
            std::swap(e->cands.bytes, nb.bytes);
            cand_total += extra;
            if ((c = upload(e, e->cand_base, cbase)) != cudaSuccess) return cuda_fail(e, c, "upload cand base");
            if ((c = upload(e, e->cand_cap, ccap)) != cudaSuccess) return cuda_fail(e, c, "upload cand cap");
            A.cands = e->cands.as<Cand>();
            Aw.cands = A.cands;
            std::vector<WorkItem> ri, rw;
            std::vector<int> rcl;
            for (size_t k = 0; k < wi.size(); ++k) {
                bool ov = false;
                for (int l = 0; l < wi[k].lanes; ++l)
                    if (over[wi[k].pair_base + l]) ov = true;
                if (ov) {
                    ri.push_back(wi[k]);
                    rcl.push_back(wc[k]);
                }
            }
            for (const WorkItem& w : ww)
                if (over[w.pair_base]) rw.push_back(w);
            // the warp sweep counts with atomics from zero; the strip sweep
            // overwrites its counts, and the other pairs' counts are no longer read
            if ((c = cudaMemsetAsync(A.n_cand, 0, n_pairs * sizeof(int32_t), e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "reset candidate counts");
            if (!ri.empty()) {
                int rb[kNumClasses + 1];
                order_by_class(ri, rcl, rb);
                if ((c = upload(e, e->items_alt, ri)) != cudaSuccess) return cuda_fail(e, c, "upload items");
                rc = hstore ? run_phase<3>(e, A, e->items_alt.as<WorkItem>(), rb, xm, &inf.trace_kernel_ms,
                                           &inf.trace_launches, trans2)
                            : run_phase<2>(e, A, e->items_alt.as<WorkItem>(), rb, xm, &inf.trace_kernel_ms,
                                           &inf.trace_launches, trans2);
                if (rc != PW_OK) return rc;
            }
            if (!rw.empty()) {
                std::vector<BandPair> bp = band_pairs_of(e, rw);
                std::vector<TilePair> rt;  // the overflowing tile-form pairs
                if (p1ck) {
                    for (const TilePair& tp : tps)
                        if (over[tp.slot]) rt.push_back(tp);
                    if ((c = upload(e, e->tile_pairs_alt, rt)) != cudaSuccess) return cuda_fail(e, c, "upload tile pairs");
                }
                rc = p1ck ? run_tile_cands(e, Aw, TT, e->tile_pairs_alt.as<TilePair>(), rt, &inf.trace_kernel_ms,
                                           &inf.trace_launches)
                     : tile_form ? run_band_phase<3>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches)
                     : hstore  ? run_band_phase<2>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches)
                               : run_band_phase<1>(e, Aw, bp, &inf.trace_kernel_ms, &inf.trace_launches);
                if (rc != PW_OK) return rc;
            }
        }

        // starting points
        if ((c = upload(e, e->items, by_index)) != cudaSuccess) return cuda_fail(e, c, "upload items");
        ht.mark("candidate overflow");
        TraceArgs TA;
        memset(&TA, 0, sizeof(TA));
        TA.metas = A.metas;
        TA.n_pairs = (int)n_pairs;
        TA.items = e->items.as<WorkItem>();
        TA.codes = A.codes;
        TA.hstore = hstore ? 1 : 0;
        TA.marks = e->marks.as<uint8_t>();
        TA.cands = A.cands;
        TA.cand_base = A.cand_base;
        TA.n_starts = e->n_starts.as<int32_t>();
        TA.q = Aref.q;
        TA.t = Aref.t;
        TA.P = Aref.P;
        TA.slot_tile = TT.slot_tile;
        const int tb = 128;
        const int gb = (int)((n_pairs + tb - 1) / tb);
        if (e->affine)
            PW_LAUNCH(collect_kernel<true>, gb, tb, 0, e->stream, TA);
        else
            PW_LAUNCH(collect_kernel<false>, gb, tb, 0, e->stream, TA);
        e->launches++;
        if (n_tile > 0) {
            PW_LAUNCH(tile_collect_kernel, n_tile, kWarp, tsmem, e->stream, Aw, TA, TT);
            e->launches++;
        }
        if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "collect launch");
        // packed start offsets: exclusive scan of the per-pair counts on the device
        {
            size_t tmp = 0;
            cub::DeviceScan::ExclusiveScan(nullptr, tmp, TA.n_starts, (int64_t*)nullptr, cub::Sum(), (int64_t)0,
                                           (int)n_pairs, e->stream);
            if ((c = e->start_off.reserve(e->stream, (size_t)(n_pairs + 1) * sizeof(int64_t))) != cudaSuccess ||
                (c = e->scan_tmp.reserve(e->stream, std::max<size_t>(tmp, 16))) != cudaSuccess)
                return cuda_fail(e, c, "alloc start offsets");
            tmp = e->scan_tmp.bytes;
            if ((c = cub::DeviceScan::ExclusiveScan(e->scan_tmp.p, tmp, TA.n_starts, e->start_off.as<int64_t>(),
                                                    cub::Sum(), (int64_t)0, (int)n_pairs, e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "scan start counts");
        }
        cudaEventRecord(e->ev[2], e->stream);
        int64_t last_off = 0;
        int32_t last_n = 0;
        unsigned long long tile_bound = 0;  // tile form: bytes of operations its walks can reserve at most
        if ((c = copy_d2h(e, &last_off, e->start_off.as<int64_t>() + n_pairs - 1, sizeof(int64_t))) != cudaSuccess ||
            (c = copy_d2h(e, &last_n, TA.n_starts + n_pairs - 1, sizeof(int32_t))) != cudaSuccess ||
            (n_tile > 0 && (c = copy_d2h(e, &tile_bound, TT.ops_bound, sizeof(tile_bound))) != cudaSuccess) ||
            (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
            return cuda_fail(e, c, "collect");
        // the tile walks spell their hits' operations themselves unless that
        // bound is large (more than 1 GiB); else tile_ops_kernel walks the
        // hits again
        TT.ops = nullptr;
        if (n_tile > 0 && tile_bound <= (1ull << 30)) {
            if ((c = e->tile_ops.reserve(e->stream, (size_t)std::max<unsigned long long>(tile_bound, 16))) != cudaSuccess)
                return cuda_fail(e, c, "alloc tile operations");
            TT.ops = e->tile_ops.as<char>();
        }
        const int64_t wave_starts = last_off + last_n;
        TA.start_off = e->start_off.as<int64_t>();
        const size_t first_rec = e->h_starts.size();
        if (wave_starts > 0) {
            if ((c = e->starts.reserve(e->stream, wave_starts * sizeof(StartRec))) != cudaSuccess) return cuda_fail(e, c, "alloc");
            PW_LAUNCH(gather_kernel, gb, tb, 0, e->stream, TA, e->starts.as<StartRec>());
            e->launches++;
            if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "gather launch");
            if (!e->h_starts.resize_keep(first_rec + (size_t)wave_starts))
                return fail(e, PW_ERR_NOMEM, "host memory for the starting points");
            if ((c = copy_d2h(e, e->h_starts.data() + first_rec, e->starts.p, wave_starts * sizeof(StartRec))) != cudaSuccess ||
                (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
                return cuda_fail(e, c, "copy starts");
        }
        total_starts += wave_starts;
        ht.mark("starting points");
        TA.allowed = nullptr;
        if (start_cap >= 0 && total_starts >= start_cap) {
            if (waves.size() > 1)
                return fail(e, PW_ERR_CAPACITY, "starting-point cap reached with more than one memory wave");
            // walk only the first start_cap starting points in emission order
            // (SmithWaterman.py:683-685)
            std::vector<int64_t> idx(wave_starts);
            std::iota(idx.begin(), idx.end(), 0);
            std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
                return emit_key_less(e->h_starts[first_rec + a], e->h_starts[first_rec + b]);
            });
            std::vector<uint8_t> allow((size_t)wave_starts, 0);
            for (int64_t k = 0; k < start_cap && k < wave_starts; ++k) allow[idx[k]] = 1;
            if ((c = upload(e, e->allowed, allow)) != cudaSuccess) return cuda_fail(e, c, "upload allowed");
            TA.allowed = e->allowed.as<uint8_t>();
            inf.truncated = 1;
        }

        // walk; the hits go straight into the accumulated hit array, and each
        // reserves its column operations at an absolute offset of the
        // accumulated operations (ops_total starts at the bytes used so far)
        if (wave_starts > 0) {
            if ((c = e->acc_hits.grow_keep(e->stream, (size_t)acc_n * sizeof(DevHit),
                                           (size_t)(acc_n + wave_starts) * sizeof(DevHit))) != cudaSuccess)
                return cuda_fail(e, c, "alloc hits");
            if ((c = e->hit_count.reserve(e->stream, 16)) != cudaSuccess) return cuda_fail(e, c, "alloc");
            const unsigned long long init[2] = {0ull, (unsigned long long)acc_ops};
            if ((c = copy_h2d(e, e->hit_count.p, init, sizeof(init))) !=
                cudaSuccess)
                return cuda_fail(e, c, "reset hit count");
            TA.hits = e->acc_hits.as<DevHit>() + acc_n;
            TA.hit_count = e->hit_count.as<int>();
            TA.ops_total = (unsigned long long*)(e->hit_count.as<char>() + 8);
            TA.max_hits = (int)wave_starts;
            if (e->affine)
                PW_LAUNCH(walk_kernel<true>, gb, tb, 0, e->stream, TA);
            else
                PW_LAUNCH(walk_kernel<false>, gb, tb, 0, e->stream, TA);
            e->launches++;
            if (n_tile > 0) {
                PW_LAUNCH(tile_walk_kernel, n_tile, kWarp, tsmem, e->stream, Aw, TA, TT);
                e->launches++;
            }
            if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "walk launch");
            std::vector<int64_t> cnt;
            if ((c = download(e, cnt, TA.hit_count, 2)) != cudaSuccess) return cuda_fail(e, c, "walk");
            const int nh = (int)std::min<int64_t>((int32_t)(cnt[0] & 0xffffffff), wave_starts);
            unsigned long long tile_ops_n = 0;
            if (TT.ops && (c = copy_d2h(e, &tile_ops_n, TT.ops_total, sizeof(tile_ops_n))) != cudaSuccess)
                return cuda_fail(e, c, "walk");
            if (TT.ops && (c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "walk");
            const int64_t strip_end = cnt[1];
            const int64_t ops_end = strip_end + (int64_t)tile_ops_n;
            if (nh) {
                // column operations of the kept hits
                if ((c = e->acc_ops.grow_keep(e->stream, (size_t)acc_ops, (size_t)std::max<int64_t>(ops_end, 16))) !=
                    cudaSuccess)
                    return cuda_fail(e, c, "alloc ops");
                TA.ops = e->acc_ops.as<char>();
                PW_LAUNCH(ops_kernel, (nh + 127) / 128, 128, 0, e->stream, TA, TA.hits, nh);
                e->launches++;
                if (n_tile > 0 && TT.ops) {
                    // the tile walks' operations go after the others
                    PW_LAUNCH(tile_ops_rebase_kernel, (nh + 127) / 128, 128, 0, e->stream, TT, TA.hits, nh, strip_end);
                    e->launches++;
                    if (tile_ops_n > 0 &&
                        (c = cudaMemcpyAsync(e->acc_ops.as<char>() + strip_end, TT.ops, (size_t)tile_ops_n,
                                             cudaMemcpyDeviceToDevice, e->stream)) != cudaSuccess)
                        return cuda_fail(e, c, "copy tile operations");
                } else if (n_tile > 0) {
                    PW_LAUNCH(tile_ops_kernel, nh, kWarp, tsmem, e->stream, Aw, TA, TT, (const DevHit*)TA.hits);
                    e->launches++;
                }
                if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "ops launch");
                acc_n += nh;
                acc_ops = ops_end;
            }
        }
        cudaEventRecord(e->ev[3], e->stream);
        cudaStreamSynchronize(e->stream);
        ht.mark("walk");
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, e->ev[0], e->ev[2]);
        cudaEventElapsedTime(&t2, e->ev[2], e->ev[3]);
        trace_ms += t1;
        walk_ms += t2;
    }

    // hits in the reference's HitList order and their strings, on the device
    // (pw_finish.cuh), then both to the host
    const double t_finish = wall_ms();
    int64_t str_bytes = 0;
    if ((c = finish_hits(e, acc_n, &str_bytes)) != cudaSuccess) return cuda_fail(e, c, "order hits");
    ht.mark("hit order + strings");
    inf.starting_points = total_starts;
    inf.hits = (int64_t)e->h_hits.size();
    inf.string_bytes = str_bytes;
    inf.trace_ms = trace_ms;
    inf.walk_ms = walk_ms;
    inf.kernel_launches = (int32_t)e->launches;
    inf.finish_ms = wall_ms() - t_finish;
    inf.total_ms = wall_ms() - t_call;
    inf.h2d_bytes = e->h2d;
    inf.d2h_bytes = e->d2h;
    inf.reuse = e->reuse;
    if (info) *info = inf;
    return PW_OK;
}

extern "C" int pw_set_query_trace(pw_engine* e, const uint8_t* mask, int32_t n) {
    if (!e) return PW_ERR_ARG;
    if (n == 0) {
        e->q_trace_set = false;
        return PW_OK;
    }
    if (!mask || n != e->Q.n) return fail(e, PW_ERR_ARG, "the trace mask needs one byte per query");
    if (cudaSetDevice(e->device) != cudaSuccess) return fail(e, PW_ERR_DEVICE, "cudaSetDevice failed");
    cudaError_t c;
    if ((c = e->q_trace.reserve(e->stream, (size_t)std::max(n, 16))) != cudaSuccess ||
        (c = copy_h2d(e, e->q_trace.p, mask, (size_t)n)) != cudaSuccess ||
        (c = cudaStreamSynchronize(e->stream)) != cudaSuccess)
        return cuda_fail(e, c, "upload trace mask");
    e->q_trace_set = true;
    return PW_OK;
}

extern "C" int pw_set_pairs(pw_engine* e, const int32_t* query_idx, const int32_t* target_idx, int64_t n) {
    if (!e) return PW_ERR_ARG;
    if (n < 0 || (n > 0 && (!query_idx || !target_idx))) return fail(e, PW_ERR_ARG, "bad pair list");
    e->pair_q.assign(query_idx, query_idx + n);
    e->pair_t.assign(target_idx, target_idx + n);
    return PW_OK;
}

extern "C" int pw_set_tuning(pw_engine* e, int key, int64_t value) {
    if (!e) return PW_ERR_ARG;
    if (key < 0 || key > PW_TUNE_TILE_TRACE || value < 0)
        return fail(e, PW_ERR_ARG, "unknown tuning key or negative value");
    e->tune[key] = value;
    return PW_OK;
}

extern "C" int pw_set_wave_limit(pw_engine* e, int64_t bytes) {
    if (!e) return PW_ERR_ARG;
    if (bytes < 0) return fail(e, PW_ERR_ARG, "wave limit must be >= 0");
    e->wave_limit = bytes;
    return PW_OK;
}

extern "C" int pw_get_pair_max(pw_engine* e, float* out, int64_t n) {
    if (!e || !out) return PW_ERR_ARG;
    if (n < (int64_t)e->h_pair_max.size()) return fail(e, PW_ERR_ARG, "output too small");
    if (e->pm_stale) {
        if (cudaSetDevice(e->device) != cudaSuccess) return fail(e, PW_ERR_DEVICE, "cudaSetDevice failed");
        const int rc = sync_pair_max(e, e->pair_max.as<float>());
        if (rc != PW_OK) return rc;
    }
    std::memcpy(out, e->h_pair_max.data(), e->h_pair_max.size() * sizeof(float));
    return PW_OK;
}

extern "C" int pw_get_hits_view(pw_engine* e, const pw_hit** hits, int64_t* n_hits, const char** strbuf,
                                int64_t* strbuf_bytes) {
    if (!e || !hits || !n_hits || !strbuf || !strbuf_bytes) return PW_ERR_ARG;
    *hits = e->h_hits.empty() ? nullptr : e->h_hits.data();
    *n_hits = (int64_t)e->h_hits.size();
    *strbuf = e->h_strings.empty() ? nullptr : (const char*)e->h_strings.data();
    *strbuf_bytes = (int64_t)e->h_strings.size();
    return PW_OK;
}

extern "C" int pw_get_hits(pw_engine* e, pw_hit* hits, int64_t max_hits, char* strbuf, int64_t strbuf_bytes) {
    if (!e) return PW_ERR_ARG;
    if (max_hits < (int64_t)e->h_hits.size() || (strbuf && strbuf_bytes < (int64_t)e->h_strings.size()))
        return fail(e, PW_ERR_ARG, "output buffers too small");
    if (!e->h_hits.empty()) {
        if (!hits) return fail(e, PW_ERR_ARG, "no hit buffer");
        std::memcpy(hits, e->h_hits.data(), e->h_hits.size() * sizeof(pw_hit));
    }
    if (strbuf && !e->h_strings.empty()) std::memcpy(strbuf, e->h_strings.data(), e->h_strings.size());
    return PW_OK;
}

extern "C" int pw_get_starting_points(pw_engine* e, void* out36, int64_t max_points, int64_t* n_points) {
    if (!e) return PW_ERR_ARG;
    // emission order: block anti-diagonal descending, block x descending,
    // target, query, cell anti-diagonal descending, thread y ascending
    std::vector<StartRec> s(e->h_starts.data(), e->h_starts.data() + e->h_starts.size());
    std::stable_sort(s.begin(), s.end(), [](const StartRec& a, const StartRec& b) {
        auto k = [](const StartRec& r) {
            return std::make_tuple(-(int64_t)((r.x >> 3) + (r.y >> 3)), -(int64_t)(r.x >> 3), r.target, r.query,
                                   -(int64_t)((r.x & 7) + (r.y & 7)), (int64_t)(r.y & 7));
        };
        return k(a) < k(b);
    });
    if (n_points) *n_points = (int64_t)s.size();
    if (!out36) return PW_OK;
    const int64_t n = std::min<int64_t>(max_points, (int64_t)s.size());
    for (int64_t i = 0; i < n; ++i) {
        uint32_t u[6] = {(uint32_t)s[i].query, (uint32_t)s[i].target, (uint32_t)(s[i].x >> 3),
                         (uint32_t)(s[i].y >> 3), (uint32_t)(s[i].x & 7), (uint32_t)(s[i].y & 7)};
        float f[3] = {s[i].score, s[i].max_score, s[i].pos_score};
        std::memcpy((char*)out36 + 36 * i, u, 24);
        std::memcpy((char*)out36 + 36 * i + 24, f, 12);
    }
    return PW_OK;
}

extern "C" int pw_last_launch_count(pw_engine* e, int64_t* n) {
    if (!e || !n) return PW_ERR_ARG;
    *n = e->launches;
    return PW_OK;
}

extern "C" int pw_measure_int_peak(pw_engine* e, double* ops32, double* ops16x2, double* ms_out) {
    if (!e || !ops32) return PW_ERR_ARG;
    cudaSetDevice(e->device);
    cudaError_t c;
    if ((c = e->counter.reserve(e->stream, 64 * sizeof(int))) != cudaSuccess) return cuda_fail(e, c, "alloc");
    const int threads = 256, blocks = e->sm_count * 8, iters = 4096;
    const double instr = (double)blocks * threads * iters * 16.0 * 8.0;
    float ms = 0, ms16 = 0;
    // warm-up, then the timed launches
    PW_LAUNCH(int_peak_kernel, blocks, threads, 0, e->stream, 64, 1, e->counter.as<int>());
    cudaEventRecord(e->ev[0], e->stream);
    PW_LAUNCH(int_peak_kernel, blocks, threads, 0, e->stream, iters, 3, e->counter.as<int>());
    cudaEventRecord(e->ev[1], e->stream);
    PW_LAUNCH(int_peak16_kernel, blocks, threads, 0, e->stream, 64, 1, e->counter.as<int>());
    cudaEventRecord(e->ev[2], e->stream);
    PW_LAUNCH(int_peak16_kernel, blocks, threads, 0, e->stream, iters, 3, e->counter.as<int>());
    cudaEventRecord(e->ev[3], e->stream);
    if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "int peak probe");
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    cudaEventElapsedTime(&ms16, e->ev[2], e->ev[3]);
    *ops32 = ms > 0 ? 2.0 * instr / (ms * 1e-3) : 0.0;            // add + max
    if (ops16x2) *ops16x2 = ms16 > 0 ? 4.0 * instr / (ms16 * 1e-3) : 0.0;  // two adds + two maxima
    if (ms_out) *ms_out = ms + ms16;
    return PW_OK;
}
