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

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/paswas_b200.h"
#include "pw_kernels.cuh"

using namespace pw;

#ifndef PW_LAUNCH
#define PW_LAUNCH(kern, grid, block, smem, stream, ...) kern<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__)
#endif

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
    cudaError_t reserve(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        size_t want = n ? n : 16;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) bytes = want;
        return e;
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

struct StartRec {  // one starting point (emission order sortable)
    int32_t query, target, x, y;
    float score;
    float max_score, pos_score;
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
    DevBuf cmat_i8, cmat_f, pair_max, items, counter, bnd_pool;
    DevBuf codes, metas, cands, cand_base, cand_cap, n_starts, hits, hit_count, ops, allowed;
    // results
    std::vector<float> h_pair_max;
    std::vector<pw_hit> h_hits;
    std::vector<char> h_strings;
    std::vector<StartRec> h_starts;
    int64_t launches = 0;
};

static int fail(pw_engine* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    return code;
}

static int cuda_fail(pw_engine* e, cudaError_t c, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(c);
    int code = (c == cudaErrorMemoryAllocation) ? PW_ERR_NOMEM : PW_ERR_KERNEL;
    return fail(e, code, m);
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
    return PW_OK;
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
    S.raw.assign(residues, residues + total);
    S.off.assign(offsets, offsets + (n > 0 ? n + 1 : 0));
    if (n == 0) S.off.assign(1, 0);
    S.key.assign(id_keys, id_keys + n);
    S.n = n;
    S.set = true;
    return PW_OK;
}

extern "C" int pw_set_queries(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                              const int32_t* id_keys) {
    return set_seqs(e, e->Q, residues, offsets, n, id_keys);
}

extern "C" int pw_set_targets(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                              const int32_t* id_keys) {
    return set_seqs(e, e->T, residues, offsets, n, id_keys);
}

namespace {

enum SClass { kS16 = 0, kS32 = 1, kS64 = 2, kS32Multi = 3, kNumClasses = 4 };

int class_S(int c) { return c == kS16 ? 16 : (c == kS64 ? 64 : 32); }

int pick_class(int lt, bool affine) {
    if (lt <= 16) return kS16;
    if (lt <= 32) return kS32;
    if (!affine && lt <= 64) return kS64;
    return kS32Multi;
}

template <typename T, int S, bool AFF, bool MULTI, int PH>
cudaError_t launch_sweep(pw_engine* e, KernelArgs A, int n_items) {
    auto kern = sweep_kernel<T, S, AFF, MULTI, PH>;
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
    int grid = e->sm_count * per_sm;
    const int need = (n_items + 3) / 4;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    c = cudaMemsetAsync(A.item_counter, 0, sizeof(int), e->stream);
    if (c != cudaSuccess) return c;
    PW_LAUNCH(kern, grid, 128, smem, e->stream, A);
    e->launches++;
    return cudaGetLastError();
}

template <typename T, int PH>
cudaError_t launch_class(pw_engine* e, int cls, bool affine, KernelArgs A, int n_items) {
    if (affine) {
        switch (cls) {
            case kS16: return launch_sweep<T, 16, true, false, PH>(e, A, n_items);
            case kS32: return launch_sweep<T, 32, true, false, PH>(e, A, n_items);
            default: return launch_sweep<T, 32, true, true, PH>(e, A, n_items);
        }
    }
    switch (cls) {
        case kS16: return launch_sweep<T, 16, false, false, PH>(e, A, n_items);
        case kS32: return launch_sweep<T, 32, false, false, PH>(e, A, n_items);
        case kS64: return launch_sweep<T, 64, false, false, PH>(e, A, n_items);
        default: return launch_sweep<T, 32, false, true, PH>(e, A, n_items);
    }
}

int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct Prepared {
    int alpha = 0;
    bool int_path = true;
    std::vector<int32_t> order;  // sorted position -> query
    int xmax_all4 = 0;
};

}  // namespace

template <typename HT>
static cudaError_t upload(pw_engine* e, DevBuf& b, const std::vector<HT>& v) {
    cudaError_t c = b.reserve(std::max<size_t>(v.size() * sizeof(HT), 16));
    if (c != cudaSuccess) return c;
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(HT), cudaMemcpyHostToDevice, e->stream);
}

// Builds device sequence sets, the compact query alphabet and the compact
// substitution matrix.
static int prepare(pw_engine* e, Prepared& pr, KernelArgs& A) {
    const HostSeqs& Q = e->Q;
    const HostSeqs& T = e->T;
    const int off = e->char_offset, dim = e->dim;
    // residues must index the matrix (default_main.cu:234 reads matrix[c - offset])
    int map[256];
    for (int i = 0; i < 256; ++i) map[i] = -1;
    std::vector<int> alphabet;
    for (uint8_t c : Q.raw) {
        if (map[c] >= 0) continue;
        if (c == 0 || (int)c < off || (int)c >= off + dim)
            return fail(e, PW_ERR_ARG, "query residue outside the scoring matrix: code " + std::to_string(c));
        map[c] = (int)alphabet.size();
        alphabet.push_back(c);
    }
    for (uint8_t c : T.raw)
        if (c == 0 || (int)c < off || (int)c >= off + dim)
            return fail(e, PW_ERR_ARG, "target residue outside the scoring matrix: code " + std::to_string(c));
    if (alphabet.size() > 250) return fail(e, PW_ERR_ARG, "too many distinct query residues");
    pr.alpha = (int)alphabet.size();
    const int alpha1 = pr.alpha + 1;

    // integer path: every used score and penalty is an integer, scores fit int8,
    // and no DP value can reach 2^24 (where fp32 stops being exact)
    bool ints = std::floor(e->gap) == e->gap && std::floor(e->ext) == e->ext;
    float maxabs = 0.0f;
    for (int a = 0; a < pr.alpha; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = e->matrix[(size_t)(alphabet[a] - off) * dim + j];
            if (std::floor(v) != v || v < -127.0f || v > 127.0f) ints = false;
            maxabs = std::max(maxabs, std::fabs(v));
        }
    int64_t maxlen = 0;
    for (int32_t i = 0; i < Q.n; ++i) maxlen = std::max<int64_t>(maxlen, Q.off[i + 1] - Q.off[i]);
    int64_t maxlt = 0;
    for (int32_t i = 0; i < T.n; ++i) maxlt = std::max<int64_t>(maxlt, T.off[i + 1] - T.off[i]);
    if ((double)maxabs * (double)std::min(maxlen, maxlt) + std::fabs(e->gap) + std::fabs(e->ext) >= 16777216.0)
        ints = false;
    if (std::fabs(e->gap) > 1.0e6f || std::fabs(e->ext) > 1.0e6f) ints = false;
    pr.int_path = ints;

    std::vector<int8_t> cm8((size_t)alpha1 * dim, (int8_t)-128);
    std::vector<float> cmf((size_t)alpha1 * dim, -1.0e30f);
    for (int a = 0; a < pr.alpha; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = e->matrix[(size_t)(alphabet[a] - off) * dim + j];
            cmf[(size_t)a * dim + j] = v;
            cm8[(size_t)a * dim + j] = ints ? (int8_t)v : 0;
        }

    // queries: compact codes, each sequence 16-byte aligned and padded to a
    // multiple of 4 with the pad code
    std::vector<int64_t> qco(Q.n + 1, 0);
    std::vector<int32_t> qlen(Q.n);
    int64_t pos = 0;
    for (int32_t i = 0; i < Q.n; ++i) {
        qlen[i] = (int32_t)(Q.off[i + 1] - Q.off[i]);
        qco[i] = pos;
        pos += align_up(std::max<int64_t>(qlen[i], 1), 16);
    }
    qco[Q.n] = pos;
    std::vector<uint8_t> qc((size_t)std::max<int64_t>(pos, 16), (uint8_t)pr.alpha);
    for (int32_t i = 0; i < Q.n; ++i)
        for (int32_t k = 0; k < qlen[i]; ++k) qc[qco[i] + k] = (uint8_t)map[Q.raw[Q.off[i] + k]];
    // targets: matrix residue index
    std::vector<int64_t> tco(T.n + 1, 0);
    std::vector<int32_t> tlen(T.n);
    pos = 0;
    for (int32_t i = 0; i < T.n; ++i) {
        tlen[i] = (int32_t)(T.off[i + 1] - T.off[i]);
        tco[i] = pos;
        pos += align_up(std::max<int64_t>(tlen[i], 1), 16);
    }
    tco[T.n] = pos;
    std::vector<uint8_t> tc((size_t)std::max<int64_t>(pos, 16), 0);
    for (int32_t i = 0; i < T.n; ++i)
        for (int32_t k = 0; k < tlen[i]; ++k) tc[tco[i] + k] = (uint8_t)(T.raw[T.off[i] + k] - off);

    pr.order.resize(Q.n);
    std::iota(pr.order.begin(), pr.order.end(), 0);
    std::stable_sort(pr.order.begin(), pr.order.end(), [&](int a, int b) { return qlen[a] > qlen[b]; });
    pr.xmax_all4 = Q.n ? (int)align_up(std::max(qlen[pr.order[0]], 1), 4) : 4;

    cudaError_t c;
#define UP(buf, vec)                                      \
    if ((c = upload(e, buf, vec)) != cudaSuccess) return cuda_fail(e, c, "upload " #buf);
    UP(e->q_codes, qc);
    UP(e->q_code_off, qco);
    UP(e->q_raw, Q.raw);
    UP(e->q_raw_off, Q.off);
    UP(e->q_len, qlen);
    UP(e->q_key, Q.key);
    UP(e->q_order, pr.order);
    UP(e->t_codes, tc);
    UP(e->t_code_off, tco);
    UP(e->t_raw, T.raw);
    UP(e->t_raw_off, T.off);
    UP(e->t_len, tlen);
    UP(e->t_key, T.key);
    UP(e->cmat_i8, cm8);
    UP(e->cmat_f, cmf);
#undef UP
    if ((c = e->counter.reserve(64)) != cudaSuccess) return cuda_fail(e, c, "alloc counter");

    ScoreParams& P = A.P;
    P.affine = e->affine;
    P.is_float = ints ? 0 : 1;
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
    P.dim = dim;
    A.q = SeqSet{e->q_codes.as<uint8_t>(), e->q_code_off.as<int64_t>(), e->q_raw.as<uint8_t>(),
                 e->q_raw_off.as<int64_t>(), e->q_len.as<int32_t>(), e->q_key.as<int32_t>()};
    A.t = SeqSet{e->t_codes.as<uint8_t>(), e->t_code_off.as<int64_t>(), e->t_raw.as<uint8_t>(),
                 e->t_raw_off.as<int64_t>(), e->t_len.as<int32_t>(), e->t_key.as<int32_t>()};
    A.q_order = e->q_order.as<int32_t>();
    A.cmat_i8 = e->cmat_i8.as<int8_t>();
    A.cmat_f = e->cmat_f.as<float>();
    A.item_counter = e->counter.as<int>();
    A.nt = T.n;
    return PW_OK;
}

// Launches one phase over a list of work items grouped by strip class.
template <int PH>
static int run_items(pw_engine* e, const Prepared& pr, KernelArgs A, const std::vector<WorkItem> (&by_class)[kNumClasses],
                     DevBuf& item_buf, int64_t item_base_offset) {
    (void)item_base_offset;
    int xmax_multi = 4;
    for (const WorkItem& w : by_class[kS32Multi]) xmax_multi = std::max(xmax_multi, (int)align_up(w.xmax, 4));
    for (int cls = 0; cls < kNumClasses; ++cls) {
        const std::vector<WorkItem>& its = by_class[cls];
        if (its.empty()) continue;
        cudaError_t c = upload(e, item_buf, its);
        if (c != cudaSuccess) return cuda_fail(e, c, "upload items");
        A.items = item_buf.as<WorkItem>();
        A.n_items = (int)its.size();
        if (cls == kS32Multi) {
            // one boundary slot per resident warp
            const int64_t slot = (int64_t)xmax_multi * kWarp;
            const int64_t warps = (int64_t)e->sm_count * 16 * 4;
            const size_t elem = pr.int_path ? sizeof(Bnd<int>) : sizeof(Bnd<float>);
            c = e->bnd_pool.reserve((size_t)(slot * warps) * elem);
            if (c != cudaSuccess) return cuda_fail(e, c, "alloc boundary pool");
            A.bnd_pool = e->bnd_pool.p;
            A.bnd_slot_elems = slot;
        }
        c = pr.int_path ? launch_class<int, PH>(e, cls, e->affine, A, A.n_items)
                        : launch_class<float, PH>(e, cls, e->affine, A, A.n_items);
        if (c != cudaSuccess) return cuda_fail(e, c, "sweep kernel launch");
        // items buffer is reused by the next class: wait for this launch
        c = cudaStreamSynchronize(e->stream);
        if (c != cudaSuccess) return cuda_fail(e, c, "sweep kernel");
    }
    return PW_OK;
}

static void build_items(const std::vector<std::vector<int32_t>>& per_target_sorted_pos, const std::vector<int32_t>& order,
                        const std::vector<int32_t>& qlen, const std::vector<int32_t>& tlen, bool affine,
                        std::vector<WorkItem> (&by_class)[kNumClasses], std::vector<int32_t>* pair_query) {
    for (auto& v : by_class) v.clear();
    (void)order;
    for (size_t t = 0; t < per_target_sorted_pos.size(); ++t) {
        const std::vector<int32_t>& pos = per_target_sorted_pos[t];
        for (size_t g = 0; g < pos.size(); g += kWarp) {
            WorkItem w;
            w.target = (int32_t)t;
            w.first = (int32_t)g;  // caller rewrites for phase 2
            w.lanes = (int32_t)std::min<size_t>(kWarp, pos.size() - g);
            w.xmax = qlen[order[pos[g]]];
            w.dir_base = 0;
            w.pair_base = 0;
            const int cls = pick_class(tlen[t], affine);
            w.S = class_S(cls);
            w.index = 0;
            by_class[cls].push_back(w);
        }
    }
    (void)pair_query;
}

extern "C" int pw_align(pw_engine* e, uint32_t flags, int64_t start_cap, pw_run_info* info) {
    if (!e) return PW_ERR_ARG;
    if (!e->scoring_set) return fail(e, PW_ERR_STATE, "pw_set_scoring was not called");
    if (!e->Q.set || !e->T.set) return fail(e, PW_ERR_STATE, "queries and targets must be set");
    if (cudaSetDevice(e->device) != cudaSuccess) return fail(e, PW_ERR_DEVICE, "cudaSetDevice failed");
    e->err.clear();
    e->h_hits.clear();
    e->h_strings.clear();
    e->h_starts.clear();
    e->launches = 0;
    pw_run_info inf;
    memset(&inf, 0, sizeof(inf));
    const int nq = e->Q.n, nt = e->T.n;
    e->h_pair_max.assign((size_t)nq * nt, 0.0f);
    inf.pairs = (int64_t)nq * nt;
    std::vector<int32_t> qlen(nq), tlen(nt);
    int64_t sumq = 0, sumt = 0;
    for (int i = 0; i < nq; ++i) sumq += (qlen[i] = (int32_t)(e->Q.off[i + 1] - e->Q.off[i]));
    for (int i = 0; i < nt; ++i) sumt += (tlen[i] = (int32_t)(e->T.off[i + 1] - e->T.off[i]));
    inf.cells = sumq * sumt;
    if (nq == 0 || nt == 0) {
        if (info) *info = inf;
        return PW_OK;
    }
    KernelArgs A;
    memset(&A, 0, sizeof(A));
    Prepared pr;
    int rc = prepare(e, pr, A);
    if (rc != PW_OK) return rc;
    cudaError_t c;
    if ((c = e->pair_max.reserve((size_t)nq * nt * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, c, "alloc pair maxima");
    A.pair_max = e->pair_max.as<float>();

    // ---------------------------------------------------------- phase 1
    std::vector<std::vector<int32_t>> all_pos(nt);
    for (int t = 0; t < nt; ++t) {
        all_pos[t].resize(nq);
        std::iota(all_pos[t].begin(), all_pos[t].end(), 0);
    }
    std::vector<WorkItem> by_class[kNumClasses];
    build_items(all_pos, pr.order, qlen, tlen, e->affine, by_class, nullptr);
    for (auto& v : by_class)  // largest work first
        std::stable_sort(v.begin(), v.end(), [&](const WorkItem& a, const WorkItem& b) {
            return (int64_t)a.xmax * tlen[a.target] > (int64_t)b.xmax * tlen[b.target];
        });
    cudaEventRecord(e->ev[0], e->stream);
    rc = run_items<1>(e, pr, A, by_class, e->items, 0);
    if (rc != PW_OK) return rc;
    cudaEventRecord(e->ev[1], e->stream);
    c = cudaMemcpyAsync(e->h_pair_max.data(), A.pair_max, (size_t)nq * nt * sizeof(float), cudaMemcpyDeviceToHost,
                        e->stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "copy pair maxima");
    if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "score phase");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    inf.score_ms = ms;

    if (flags & PW_FLAG_SCORE_ONLY) {
        inf.kernel_launches = (int32_t)e->launches;
        if (info) *info = inf;
        return PW_OK;
    }

    // ---------------------------------------------------------- phase 2
    // pairs whose maximum reaches MINIMUM_SCORE (default_main.cu:596), per
    // target in sorted query order
    std::vector<std::vector<int32_t>> pass_pos(nt);
    int64_t n_pass = 0;
    for (int t = 0; t < nt; ++t)
        for (int sp = 0; sp < nq; ++sp) {
            const int q = pr.order[sp];
            if (e->h_pair_max[(size_t)q * nt + t] >= e->minimum_score) {
                pass_pos[t].push_back(sp);
                ++n_pass;
            }
        }
    inf.traced_pairs = n_pass;
    if (n_pass == 0) {
        inf.kernel_launches = (int32_t)e->launches;
        if (info) *info = inf;
        return PW_OK;
    }
    // work items over passing pairs; `first` indexes a per-item list of sorted
    // positions, so phase 2 gets its own query order array
    std::vector<int32_t> p2_order;
    std::vector<WorkItem> items2;
    std::vector<int32_t> items2_cls, items2_S;  // strip class and height per item
    for (int t = 0; t < nt; ++t) {
        const std::vector<int32_t>& pos = pass_pos[t];
        for (size_t g = 0; g < pos.size(); g += kWarp) {
            WorkItem w;
            w.target = t;
            w.first = (int32_t)p2_order.size();
            w.lanes = (int32_t)std::min<size_t>(kWarp, pos.size() - g);
            for (int l = 0; l < w.lanes; ++l) p2_order.push_back(pr.order[pos[g + l]]);
            w.xmax = qlen[p2_order[w.first]];
            w.dir_base = 0;
            w.pair_base = 0;
            const int cls = pick_class(tlen[t], e->affine);
            w.S = class_S(cls);
            w.index = 0;
            items2.push_back(w);
            items2_cls.push_back(cls);
            items2_S.push_back(class_S(cls));
        }
    }
    if ((c = upload(e, e->q_order, p2_order)) != cudaSuccess) return cuda_fail(e, c, "upload phase-2 order");
    A.q_order = e->q_order.as<int32_t>();

    // memory waves: cell codes of one wave must fit the budget
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    int64_t budget = (int64_t)(free_b * 0.5);
    budget = std::min<int64_t>(budget, (int64_t)48 << 30);
    std::vector<int64_t> item_bytes(items2.size());
    for (size_t i = 0; i < items2.size(); ++i) {
        const int S = items2_S[i];
        const int64_t strips = (tlen[items2[i].target] + S - 1) / S;
        item_bytes[i] = std::max<int64_t>(strips, 1) * S * align_up(items2[i].xmax, 4) * kWarp;
    }
    std::vector<std::pair<size_t, size_t>> waves;
    {
        size_t i0 = 0;
        int64_t acc = 0;
        for (size_t i = 0; i < items2.size(); ++i) {
            if (acc > 0 && acc + item_bytes[i] > budget) {
                waves.push_back({i0, i});
                i0 = i;
                acc = 0;
            }
            acc += item_bytes[i];
        }
        waves.push_back({i0, items2.size()});
    }
    if (waves.size() > 1 && start_cap >= 0 && (int64_t)start_cap < n_pass * 1000)
        ;  // the cap is checked per wave below

    double trace_ms = 0, walk_ms = 0;
    int64_t total_starts = 0;
    std::vector<DevHit> all_hits;
    std::vector<char> all_ops;
    std::vector<int64_t> all_ops_base;

    for (size_t wv = 0; wv < waves.size(); ++wv) {
        const size_t i0 = waves[wv].first, i1 = waves[wv].second;
        std::vector<WorkItem> wave_items(items2.begin() + i0, items2.begin() + i1);
        int64_t dir_off = 0, pair_off = 0;
        for (size_t k = 0; k < wave_items.size(); ++k) {
            wave_items[k].index = (int32_t)k;
            wave_items[k].dir_base = dir_off;
            wave_items[k].pair_base = pair_off;
            dir_off += item_bytes[i0 + k];
            pair_off += wave_items[k].lanes;
        }
        const int64_t n_pairs = pair_off;
        if ((c = e->codes.reserve((size_t)dir_off)) != cudaSuccess) return cuda_fail(e, c, "alloc cell codes");
        if ((c = e->metas.reserve(n_pairs * sizeof(PairMeta))) != cudaSuccess) return cuda_fail(e, c, "alloc metas");
        std::vector<int32_t> cbase(n_pairs), ccap(n_pairs, kCandCap);
        for (int64_t p = 0; p < n_pairs; ++p) cbase[p] = (int32_t)(p * kCandCap);
        int64_t cand_total = n_pairs * kCandCap;
        if ((c = e->cands.reserve(cand_total * sizeof(Cand))) != cudaSuccess) return cuda_fail(e, c, "alloc cands");
        if ((c = upload(e, e->cand_base, cbase)) != cudaSuccess) return cuda_fail(e, c, "upload cand base");
        if ((c = upload(e, e->cand_cap, ccap)) != cudaSuccess) return cuda_fail(e, c, "upload cand cap");
        A.codes = e->codes.as<uint8_t>();
        A.metas = e->metas.as<PairMeta>();
        A.cands = e->cands.as<Cand>();
        A.cand_base = e->cand_base.as<int32_t>();
        A.cand_cap = e->cand_cap.as<int32_t>();

        // phase 2 by class; the items buffer holds the whole wave, classes are
        // launched over contiguous sub-ranges
        std::vector<WorkItem> wave_by_class[kNumClasses];
        std::vector<int32_t> wave_cls(items2_cls.begin() + i0, items2_cls.begin() + i1);
        cudaEventRecord(e->ev[0], e->stream);
        for (int pass = 0; pass < 2; ++pass) {
            for (auto& v : wave_by_class) v.clear();
            for (size_t k = 0; k < wave_items.size(); ++k) wave_by_class[wave_cls[k]].push_back(wave_items[k]);
            rc = run_items<2>(e, pr, A, wave_by_class, e->items, 0);
            if (rc != PW_OK) return rc;
            // candidate overflow: give overflowing items exact capacities and
            // sweep them again (their codes and lists are rewritten)
            std::vector<PairMeta> metas(n_pairs);
            c = cudaMemcpy(metas.data(), A.metas, n_pairs * sizeof(PairMeta), cudaMemcpyDeviceToHost);
            if (c != cudaSuccess) return cuda_fail(e, c, "copy metas");
            bool overflow = false;
            for (int64_t p = 0; p < n_pairs; ++p)
                if (metas[p].n_cand > ccap[p]) overflow = true;
            if (!overflow) break;
            if (pass == 1) return fail(e, PW_ERR_KERNEL, "candidate list overflow after resize");
            std::vector<WorkItem> redo;
            std::vector<int32_t> redo_cls;
            int64_t pos = 0;
            for (int64_t p = 0; p < n_pairs; ++p) {
                cbase[p] = (int32_t)pos;
                ccap[p] = std::max<int32_t>(kCandCap, metas[p].n_cand);
                pos += ccap[p];
            }
            if (pos > INT32_MAX) return fail(e, PW_ERR_CAPACITY, "too many starting-point candidates");
            for (size_t k = 0; k < wave_items.size(); ++k) {
                bool ov = false;
                for (int l = 0; l < wave_items[k].lanes; ++l) {
                    const int64_t p = wave_items[k].pair_base + l;
                    if (metas[p].n_cand > kCandCap) ov = true;
                }
                if (ov) {
                    redo.push_back(wave_items[k]);
                    redo_cls.push_back(wave_cls[k]);
                }
            }
            // keep the non-overflowing lists where they are: copy them over
            std::vector<Cand> old_c((size_t)n_pairs * kCandCap);
            c = cudaMemcpy(old_c.data(), A.cands, old_c.size() * sizeof(Cand), cudaMemcpyDeviceToHost);
            if (c != cudaSuccess) return cuda_fail(e, c, "copy cands");
            std::vector<Cand> new_c((size_t)pos);
            for (int64_t p = 0; p < n_pairs; ++p)
                for (int k = 0; k < std::min<int>(metas[p].n_cand, kCandCap); ++k)
                    new_c[cbase[p] + k] = old_c[(size_t)p * kCandCap + k];
            if ((c = upload(e, e->cands, new_c)) != cudaSuccess) return cuda_fail(e, c, "upload cands");
            if ((c = upload(e, e->cand_base, cbase)) != cudaSuccess) return cuda_fail(e, c, "upload cand base");
            if ((c = upload(e, e->cand_cap, ccap)) != cudaSuccess) return cuda_fail(e, c, "upload cand cap");
            A.cands = e->cands.as<Cand>();
            A.cand_base = e->cand_base.as<int32_t>();
            A.cand_cap = e->cand_cap.as<int32_t>();
            wave_items = redo;
            wave_cls = redo_cls;
        }
        cudaEventRecord(e->ev[1], e->stream);

        // collect starting points
        std::vector<WorkItem> wave_items_all(items2.begin() + i0, items2.begin() + i1);
        {
            int64_t d = 0, p = 0;
            for (size_t k = 0; k < wave_items_all.size(); ++k) {
                wave_items_all[k].index = (int32_t)k;
                wave_items_all[k].dir_base = d;
                wave_items_all[k].pair_base = p;
                d += item_bytes[i0 + k];
                p += wave_items_all[k].lanes;
            }
        }
        if ((c = upload(e, e->items, wave_items_all)) != cudaSuccess) return cuda_fail(e, c, "upload items");
        if ((c = e->n_starts.reserve(n_pairs * sizeof(int32_t))) != cudaSuccess) return cuda_fail(e, c, "alloc");
        TraceArgs TA;
        memset(&TA, 0, sizeof(TA));
        TA.metas = A.metas;
        TA.n_pairs = (int)n_pairs;
        TA.items = e->items.as<WorkItem>();
        TA.codes = A.codes;
        TA.cands = A.cands;
        TA.cand_base = A.cand_base;
        TA.n_starts = e->n_starts.as<int32_t>();
        TA.q = A.q;
        TA.t = A.t;
        TA.P = A.P;
        const int tb = 128;
        const int gb = (int)((n_pairs + tb - 1) / tb);
        if (e->affine)
            PW_LAUNCH(collect_kernel<true>, gb, tb, 0, e->stream, TA);
        else
            PW_LAUNCH(collect_kernel<false>, gb, tb, 0, e->stream, TA);
        e->launches++;
        if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "collect launch");
        cudaEventRecord(e->ev[2], e->stream);

        // starting points to the host (emission order records, start cap)
        std::vector<int32_t> ns(n_pairs);
        std::vector<PairMeta> metas(n_pairs);
        c = cudaMemcpyAsync(ns.data(), TA.n_starts, n_pairs * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream);
        if (c != cudaSuccess) return cuda_fail(e, c, "copy n_starts");
        c = cudaMemcpyAsync(metas.data(), A.metas, n_pairs * sizeof(PairMeta), cudaMemcpyDeviceToHost, e->stream);
        if (c != cudaSuccess) return cuda_fail(e, c, "copy metas");
        const int64_t cand_slots = (int64_t)cbase.back() + ccap.back();
        std::vector<Cand> hc((size_t)cand_slots);
        c = cudaMemcpyAsync(hc.data(), A.cands, hc.size() * sizeof(Cand), cudaMemcpyDeviceToHost, e->stream);
        if (c != cudaSuccess) return cuda_fail(e, c, "copy starts");
        if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "collect");
        int64_t wave_starts = 0;
        for (int64_t p = 0; p < n_pairs; ++p) {
            wave_starts += ns[p];
            const PairMeta& pm = metas[p];
            const int mn = std::min(qlen[pm.query], tlen[pm.target]);
            const float pos = (float)(e->highest * (double)mn * e->filter_factor);
            for (int k = 0; k < ns[p]; ++k) {
                const Cand& cc = hc[cbase[p] + k];
                e->h_starts.push_back(StartRec{pm.query, pm.target, cc.x, cc.y, cc.score_f, pm.max_f, pos});
            }
        }
        total_starts += wave_starts;
        const uint8_t* allowed_dev = nullptr;
        if (start_cap >= 0 && total_starts >= start_cap) {
            if (waves.size() > 1)
                return fail(e, PW_ERR_CAPACITY, "starting-point cap reached with more than one memory wave");
            // walk only the first start_cap starting points in emission order
            std::vector<int64_t> idx(e->h_starts.size());
            std::iota(idx.begin(), idx.end(), 0);
            std::vector<int64_t> slot_of(e->h_starts.size());
            {
                int64_t s = 0;
                for (int64_t p = 0; p < n_pairs; ++p)
                    for (int k = 0; k < ns[p]; ++k) slot_of[s++] = cbase[p] + k;
            }
            auto key = [&](const StartRec& r) {
                return std::make_tuple(-(int64_t)((r.x >> 3) + (r.y >> 3)), -(int64_t)(r.x >> 3), r.target, r.query,
                                       -(int64_t)((r.x & 7) + (r.y & 7)), (int64_t)(r.y & 7));
            };
            std::stable_sort(idx.begin(), idx.end(),
                             [&](int64_t a, int64_t b) { return key(e->h_starts[a]) < key(e->h_starts[b]); });
            std::vector<uint8_t> allow((size_t)cand_slots, 0);
            for (int64_t k = 0; k < start_cap && k < (int64_t)idx.size(); ++k) allow[slot_of[idx[k]]] = 1;
            if ((c = upload(e, e->allowed, allow)) != cudaSuccess) return cuda_fail(e, c, "upload allowed");
            allowed_dev = e->allowed.as<uint8_t>();
            inf.truncated = 1;
        }

        // walk
        const int64_t max_hits = std::max<int64_t>(wave_starts, 1);
        if ((c = e->hits.reserve(max_hits * sizeof(DevHit))) != cudaSuccess) return cuda_fail(e, c, "alloc hits");
        if ((c = e->hit_count.reserve(16)) != cudaSuccess) return cuda_fail(e, c, "alloc");
        cudaMemsetAsync(e->hit_count.p, 0, sizeof(int), e->stream);
        TA.allowed = allowed_dev;
        TA.hits = e->hits.as<DevHit>();
        TA.hit_count = e->hit_count.as<int>();
        TA.max_hits = (int)max_hits;
        if (e->affine)
            PW_LAUNCH(walk_kernel<true>, gb, tb, 0, e->stream, TA);
        else
            PW_LAUNCH(walk_kernel<false>, gb, tb, 0, e->stream, TA);
        e->launches++;
        if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "walk launch");
        int nh = 0;
        c = cudaMemcpyAsync(&nh, TA.hit_count, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
        if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "walk");
        nh = (int)std::min<int64_t>(nh, max_hits);
        std::vector<DevHit> hh(nh);
        if (nh) {
            c = cudaMemcpy(hh.data(), TA.hits, nh * sizeof(DevHit), cudaMemcpyDeviceToHost);
            if (c != cudaSuccess) return cuda_fail(e, c, "copy hits");
        }
        // column operations
        int64_t ops_total = 0;
        for (int k = 0; k < nh; ++k) {
            hh[k].ops_offset = ops_total;
            ops_total += hh[k].n_cols;
        }
        if (nh) {
            if ((c = upload(e, e->hits, hh)) != cudaSuccess) return cuda_fail(e, c, "upload hits");
            if ((c = e->ops.reserve(std::max<int64_t>(ops_total, 16))) != cudaSuccess) return cuda_fail(e, c, "alloc ops");
            TA.ops = e->ops.as<char>();
            PW_LAUNCH(ops_kernel, (nh + 127) / 128, 128, 0, e->stream, TA, e->hits.as<DevHit>(), nh);
            e->launches++;
            if ((c = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, c, "ops launch");
            std::vector<char> ops((size_t)ops_total);
            if (ops_total) {
                c = cudaMemcpyAsync(ops.data(), TA.ops, ops_total, cudaMemcpyDeviceToHost, e->stream);
                if (c != cudaSuccess) return cuda_fail(e, c, "copy ops");
            }
            cudaEventRecord(e->ev[3], e->stream);
            if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return cuda_fail(e, c, "ops");
            const int64_t base = (int64_t)all_ops.size();
            for (int k = 0; k < nh; ++k) hh[k].ops_offset += base;
            all_ops.insert(all_ops.end(), ops.begin(), ops.end());
            all_hits.insert(all_hits.end(), hh.begin(), hh.end());
        } else {
            cudaEventRecord(e->ev[3], e->stream);
            cudaStreamSynchronize(e->stream);
        }
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, e->ev[0], e->ev[2]);
        cudaEventElapsedTime(&t2, e->ev[2], e->ev[3]);
        trace_ms += t1;
        walk_ms += t2;
    }

    // hits in the reference's HitList order: ascending score, then the pinned
    // emission order of their starting points (SmithWaterman.py:699)
    std::vector<int64_t> ord(all_hits.size());
    std::iota(ord.begin(), ord.end(), 0);
    auto hkey = [&](const DevHit& h) {
        return std::make_tuple(h.score, -(int64_t)((h.end_x >> 3) + (h.end_y >> 3)), -(int64_t)(h.end_x >> 3),
                               h.target, h.query, -(int64_t)((h.end_x & 7) + (h.end_y & 7)), (int64_t)(h.end_y & 7));
    };
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int64_t a, int64_t b) { return hkey(all_hits[a]) < hkey(all_hits[b]); });
    int64_t str_bytes = 0;
    e->h_hits.resize(all_hits.size());
    for (size_t k = 0; k < ord.size(); ++k) {
        const DevHit& d = all_hits[ord[k]];
        pw_hit& h = e->h_hits[k];
        h.query = d.query;
        h.target = d.target;
        h.s_start = d.s_start;
        h.s_end = d.s_end;
        h.t_start = d.t_start;
        h.t_end = d.t_end;
        h.score = d.score;
        h.matches = d.matches;
        h.mismatches = d.mismatches;
        h.n_cols = d.n_cols;
        h.str_offset = str_bytes;
        str_bytes += 3 * (int64_t)d.n_cols;
    }
    // alignment strings from the column operations
    e->h_strings.resize((size_t)str_bytes);
    for (size_t k = 0; k < ord.size(); ++k) {
        const DevHit& d = all_hits[ord[k]];
        const pw_hit& h = e->h_hits[k];
        char* sq = e->h_strings.data() + h.str_offset;
        char* al = sq + h.n_cols;
        char* tg = al + h.n_cols;
        const uint8_t* qs = e->Q.raw.data() + e->Q.off[d.query];
        const uint8_t* ts = e->T.raw.data() + e->T.off[d.target];
        int x = d.s_start, y = d.t_start;
        const char* ops = all_ops.data() + d.ops_offset;
        for (int i = 0; i < d.n_cols; ++i) {
            const char op = ops[i];
            if (op == 'M') {
                const uint8_t a = ts[y], b = qs[x];
                const bool la = (a >= 'A' && a <= 'Z') || (a >= 'a' && a <= 'z');
                const bool eq = la ? ((a | 0x20) == (b | 0x20)) : a == b;
                sq[i] = (char)b;
                tg[i] = (char)a;
                al[i] = eq ? '|' : '.';
                ++x;
                ++y;
            } else if (op == 'I') {
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
    inf.starting_points = total_starts;
    inf.hits = (int64_t)e->h_hits.size();
    inf.string_bytes = str_bytes;
    inf.trace_ms = trace_ms;
    inf.walk_ms = walk_ms;
    inf.kernel_launches = (int32_t)e->launches;
    if (info) *info = inf;
    return PW_OK;
}

extern "C" int pw_get_pair_max(pw_engine* e, float* out, int64_t n) {
    if (!e || !out) return PW_ERR_ARG;
    if (n < (int64_t)e->h_pair_max.size()) return fail(e, PW_ERR_ARG, "output too small");
    std::memcpy(out, e->h_pair_max.data(), e->h_pair_max.size() * sizeof(float));
    return PW_OK;
}

extern "C" int pw_get_hits(pw_engine* e, pw_hit* hits, int64_t max_hits, char* strbuf, int64_t strbuf_bytes) {
    if (!e) return PW_ERR_ARG;
    if (max_hits < (int64_t)e->h_hits.size() || strbuf_bytes < (int64_t)e->h_strings.size())
        return fail(e, PW_ERR_ARG, "output buffers too small");
    if (!e->h_hits.empty()) std::memcpy(hits, e->h_hits.data(), e->h_hits.size() * sizeof(pw_hit));
    if (!e->h_strings.empty()) std::memcpy(strbuf, e->h_strings.data(), e->h_strings.size());
    return PW_OK;
}

extern "C" int pw_get_starting_points(pw_engine* e, void* out36, int64_t max_points, int64_t* n_points) {
    if (!e) return PW_ERR_ARG;
    // emission order: block anti-diagonal descending, block x descending,
    // target, query, cell anti-diagonal descending, thread y ascending
    std::vector<StartRec> s = e->h_starts;
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
