// noalloc.cu -- pair maxima for callers that cannot allocate device memory.
//
// pw_score_max_noalloc() computes the same pair maxima as pw_align() with
// PW_FLAG_SCORE_ONLY, but it never calls cudaMalloc / cudaFree and creates no
// engine, stream or event.  All device working memory -- the staged sequences,
// the compact substitution matrix, the work list and counters, the strip
// boundary rows of long targets and the result array -- lives in one
// file-scope __device__ array of kNoAllocScratchBytes.  The array is part of
// the library image, so every GPU that loads the library holds it until the
// process exits.
//
// Sharing rules: every call reuses the same array and leaves its contents
// behind; the parts that must start at zero (the work counters) are cleared by
// each call.  Two calls whose GPU work overlaps (from different host threads,
// or on different streams) race on the array and corrupt each other's
// results; calls are serialised by a host mutex inside this library, but
// callers that enqueue other work touching the results must keep it ordered
// after the call returns.  Work runs on the legacy default stream and the call
// returns when the results are in the caller's buffer.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current and caches it; make that
// first call before any stream capture is active on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/paswas_b200.h"
#define PW_SCORE_SWEEP_ONLY
#include "pw_kernels.cuh"

using namespace pw;

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;  // 64 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch per device, looked up once per device
void* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;
// host staging area with the device layout (static, so the call allocates nothing)
alignas(256) unsigned char g_stage[kNoAllocScratchBytes];

int report(char* err, int32_t err_bytes, int code, const char* fmt, ...) {
    if (err && err_bytes > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, (size_t)err_bytes, fmt, ap);
        va_end(ap);
    }
    return code;
}

int class_of(int lt, bool affine) {
    if (lt <= 16) return 0;
    if (lt <= 32) return 1;
    if (!affine && lt <= 64) return 2;
    return 3;
}
int S_of(int cls) { return cls == 0 ? 16 : (cls == 2 ? 64 : 32); }

size_t align_to(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Makes `device` current for the lifetime of the guard and gives the caller
// back the device that was current before, on every return path.
struct DeviceGuard {
    int previous = -1;
    bool switched = false;
    cudaError_t enter(int device) {
        cudaError_t c = cudaGetDevice(&previous);
        if (c != cudaSuccess) return c;
        if (previous == device) return cudaSuccess;
        c = cudaSetDevice(device);
        switched = c == cudaSuccess;
        return c;
    }
    ~DeviceGuard() {
        if (switched) cudaSetDevice(previous);
    }
};

// Score-sweep variant: the same per-lane sweep as sweep_kernel's first phase
// (sweep_score / build_profile), with the work counter and boundary rows in
// the caller-free scratch array.
template <typename T, int S, bool AFFINE, bool MULTI>
__global__ void __launch_bounds__(128) noalloc_score_kernel(KernelArgs A) {
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
        for (int s = 0; s < nstrips; ++s) {
            c.y0 = s * S;
            c.has_up = s > 0;
            c.has_down = s + 1 < nstrips;
            __syncwarp();
            build_profile<T, S>(prof, A.cmat_i8, A.cmat_f, tres, c.y0, lt, alpha1, A.P.dim, lane);
            __syncwarp();
            if (active) sweep_score<T, S, AFFINE>(c, prof, alpha1, gap, ext, ge, bnd_slot, mx);
        }
        if (active) A.pair_max[(int64_t)q * A.pm_lane + (int64_t)t * A.pm_strip] = (float)mx;
    }
}

template <typename T, int S, bool AFF, bool MULTI>
cudaError_t launch_variant(const KernelArgs& A, int max_blocks) {
    auto kern = noalloc_score_kernel<T, S, AFF, MULTI>;
    const int alpha1 = A.P.alpha + 1;
    const int prof_bytes = ((S / 4) * alpha1 * (std::is_integral<T>::value ? 4 : 16) + 15) & ~15;
    const int smem = 4 * prof_bytes;
    if (smem > 48 * 1024) {
        cudaError_t c = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (c != cudaSuccess) return c;
    }
    int dev = 0, sms = 1, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
    if (c != cudaSuccess) return c;
    int grid = std::max(1, std::min(sms * std::max(per_sm, 1), max_blocks));
    grid = std::min(grid, (A.n_items + 3) / 4);
    kern<<<std::max(grid, 1), 128, smem, 0>>>(A);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cls(int cls, bool affine, const KernelArgs& A, int max_blocks) {
    if (affine) {
        if (cls == 0) return launch_variant<T, 16, true, false>(A, max_blocks);
        if (cls == 1) return launch_variant<T, 32, true, false>(A, max_blocks);
        return launch_variant<T, 32, true, true>(A, max_blocks);
    }
    if (cls == 0) return launch_variant<T, 16, false, false>(A, max_blocks);
    if (cls == 1) return launch_variant<T, 32, false, false>(A, max_blocks);
    if (cls == 2) return launch_variant<T, 64, false, false>(A, max_blocks);
    return launch_variant<T, 32, false, true>(A, max_blocks);
}

}  // namespace

extern "C" int pw_score_max_noalloc(int device, const float* matrix, int dim, int char_offset, float gap, float ext,
                                    int affine, const uint8_t* q_res, const int64_t* q_off, int32_t nq,
                                    const uint8_t* t_res, const int64_t* t_off, int32_t nt, float* pair_max,
                                    char* err, int32_t err_bytes) {
    if (err && err_bytes > 0) err[0] = 0;
    if (device < 0 || device >= kMaxDevices) return report(err, err_bytes, PW_ERR_DEVICE, "bad device %d", device);
    if (!matrix || dim <= 0 || dim > 256 || char_offset < 0 || char_offset + dim > 256)
        return report(err, err_bytes, PW_ERR_ARG, "bad scoring matrix");
    if (!(gap <= 0.0f) || (affine && !(ext <= 0.0f)))
        return report(err, err_bytes, PW_ERR_ARG, "gap penalties must be <= 0");
    if (!affine) ext = 0.0f;
    if (nq < 0 || nt < 0 || (nq && (!q_off || !q_res)) || (nt && (!t_off || !t_res)) ||
        (nq && nt && !pair_max))
        return report(err, err_bytes, PW_ERR_ARG, "bad sequence or output arguments");
    if (nq == 0 || nt == 0) return PW_OK;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    DeviceGuard guard;  // the caller's current device is restored on return
    if (guard.enter(device) != cudaSuccess)
        return report(err, err_bytes, PW_ERR_DEVICE, "cudaSetDevice(%d) failed", device);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t c = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (c != cudaSuccess || !p)
            return report(err, err_bytes, PW_ERR_DEVICE, "cudaGetSymbolAddress: %s", cudaGetErrorString(c));
        g_scratch_addr[device] = p;
    }
    unsigned char* dev_base = (unsigned char*)g_scratch_addr[device];
    const bool aff = affine != 0;

    // ---- validate residues and build the compact query alphabet
    int map[256];
    for (int i = 0; i < 256; ++i) map[i] = -1;
    int alphabet[256];
    int alpha = 0;
    int64_t qtot = q_off[nq], ttot = t_off[nt];
    if (q_off[0] != 0 || t_off[0] != 0) return report(err, err_bytes, PW_ERR_ARG, "offsets must start at 0");
    for (int64_t k = 0; k < qtot; ++k) {
        const uint8_t c = q_res[k];
        if (map[c] >= 0) continue;
        if (c == 0 || (int)c < char_offset || (int)c >= char_offset + dim)
            return report(err, err_bytes, PW_ERR_ARG, "query residue %d outside the scoring matrix", (int)c);
        map[c] = alpha;
        alphabet[alpha++] = c;
    }
    for (int64_t k = 0; k < ttot; ++k) {
        const uint8_t c = t_res[k];
        if (c == 0 || (int)c < char_offset || (int)c >= char_offset + dim)
            return report(err, err_bytes, PW_ERR_ARG, "target residue %d outside the scoring matrix", (int)c);
    }
    if (alpha > 250) return report(err, err_bytes, PW_ERR_ARG, "too many distinct query residues");
    const int alpha1 = alpha + 1;
    bool ints = std::floor(gap) == gap && std::floor(ext) == ext && std::fabs(gap) <= 1e6f && std::fabs(ext) <= 1e6f;
    float maxabs = 0;
    for (int a = 0; a < alpha; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = matrix[(size_t)(alphabet[a] - char_offset) * dim + j];
            if (!std::isfinite(v)) return report(err, err_bytes, PW_ERR_ARG, "non-finite score");
            if (std::floor(v) != v || v < -127.0f || v > 127.0f) ints = false;
            maxabs = std::max(maxabs, std::fabs(v));
        }
    int maxlq = 0, maxlt = 0;
    for (int32_t i = 0; i < nq; ++i) {
        const int64_t l = q_off[i + 1] - q_off[i];
        if (l < 0 || l > (1 << 24)) return report(err, err_bytes, PW_ERR_ARG, "bad query offsets");
        maxlq = std::max(maxlq, (int)l);
    }
    for (int32_t i = 0; i < nt; ++i) {
        const int64_t l = t_off[i + 1] - t_off[i];
        if (l < 0 || l > (1 << 24)) return report(err, err_bytes, PW_ERR_ARG, "bad target offsets");
        maxlt = std::max(maxlt, (int)l);
    }
    if ((double)maxabs * std::min(maxlq, maxlt) + std::fabs(gap) + std::fabs(ext) >= 16777216.0) ints = false;

    // ---- layout of the scratch array (all offsets 256-byte aligned)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_to(off + bytes, 256);
        return o;
    };
    int64_t qcode_bytes = 0, tcode_bytes = 0;
    for (int32_t i = 0; i < nq; ++i) qcode_bytes += (int64_t)align_to(std::max<int64_t>(q_off[i + 1] - q_off[i], 1), 16);
    for (int32_t i = 0; i < nt; ++i) tcode_bytes += (int64_t)align_to(std::max<int64_t>(t_off[i + 1] - t_off[i], 1), 16);
    int64_t n_items = 0;
    for (int32_t t = 0; t < nt; ++t) n_items += (nq + kWarp - 1) / kWarp;
    const size_t o_counter = take(256);
    const size_t o_cm8 = take((size_t)alpha1 * dim);
    const size_t o_cmf = take((size_t)alpha1 * dim * sizeof(float));
    const size_t o_qc = take((size_t)qcode_bytes);
    const size_t o_qco = take((size_t)nq * sizeof(int64_t));
    const size_t o_qlen = take((size_t)nq * sizeof(int32_t));
    const size_t o_qord = take((size_t)nq * sizeof(int32_t));
    const size_t o_tc = take((size_t)tcode_bytes);
    const size_t o_tco = take((size_t)nt * sizeof(int64_t));
    const size_t o_tlen = take((size_t)nt * sizeof(int32_t));
    const size_t o_items = take((size_t)n_items * sizeof(WorkItem));
    const size_t o_pm = take((size_t)nq * nt * sizeof(float));
    const size_t staged = off;
    if (staged > kNoAllocScratchBytes)
        return report(err, err_bytes, PW_ERR_CAPACITY,
                      "input needs %zu bytes of device scratch; the no-allocation limit is %zu bytes", staged,
                      kNoAllocScratchBytes);
    // boundary rows of long targets: one slot per resident warp, as many warps
    // as the remaining scratch holds
    const int xmax4 = (int)align_to(std::max(maxlq, 1), 4);
    const size_t slot_bytes = (size_t)xmax4 * kWarp * (ints ? sizeof(Bnd<int>) : sizeof(Bnd<float>));
    const size_t o_bnd = align_to(staged, 256);
    const size_t bnd_room = kNoAllocScratchBytes > o_bnd ? kNoAllocScratchBytes - o_bnd : 0;
    const int max_warps = (int)std::min<size_t>(bnd_room / slot_bytes, (size_t)1 << 20);
    bool need_multi = false;
    for (int32_t t = 0; t < nt; ++t) need_multi |= class_of((int)(t_off[t + 1] - t_off[t]), aff) == 3;
    if (need_multi && max_warps < 4)
        return report(err, err_bytes, PW_ERR_CAPACITY,
                      "queries of %d residues leave no room for boundary rows within the %zu-byte limit", maxlq,
                      kNoAllocScratchBytes);

    // ---- stage everything on the host with the device layout
    unsigned char* h = g_stage;
    memset(h, 0, staged);  // counters start at zero
    int8_t* cm8 = (int8_t*)(h + o_cm8);
    float* cmf = (float*)(h + o_cmf);
    for (int a = 0; a < alpha1; ++a)
        for (int j = 0; j < dim; ++j) {
            const float v = a < alpha ? matrix[(size_t)(alphabet[a] - char_offset) * dim + j] : -1.0e30f;
            cmf[(size_t)a * dim + j] = v;
            cm8[(size_t)a * dim + j] = a < alpha ? (ints ? (int8_t)v : 0) : (int8_t)-128;
        }
    int64_t* qco = (int64_t*)(h + o_qco);
    int32_t* qlen = (int32_t*)(h + o_qlen);
    int32_t* qord = (int32_t*)(h + o_qord);
    uint8_t* qc = h + o_qc;
    int64_t pos = 0;
    for (int32_t i = 0; i < nq; ++i) {
        qlen[i] = (int32_t)(q_off[i + 1] - q_off[i]);
        qco[i] = pos;
        const int64_t span = (int64_t)align_to(std::max(qlen[i], 1), 16);
        memset(qc + pos, alpha, (size_t)span);
        for (int32_t k = 0; k < qlen[i]; ++k) qc[pos + k] = (uint8_t)map[q_res[q_off[i] + k]];
        pos += span;
        qord[i] = i;
    }
    std::stable_sort(qord, qord + nq, [&](int a, int b) { return qlen[a] > qlen[b]; });
    int64_t* tco = (int64_t*)(h + o_tco);
    int32_t* tlen = (int32_t*)(h + o_tlen);
    uint8_t* tc = h + o_tc;
    pos = 0;
    for (int32_t i = 0; i < nt; ++i) {
        tlen[i] = (int32_t)(t_off[i + 1] - t_off[i]);
        tco[i] = pos;
        for (int32_t k = 0; k < tlen[i]; ++k) tc[pos + k] = (uint8_t)(t_res[t_off[i] + k] - char_offset);
        pos += (int64_t)align_to(std::max(tlen[i], 1), 16);
    }
    // work items grouped by strip class: one target against 32 queries
    WorkItem* items = (WorkItem*)(h + o_items);
    int cls_begin[5] = {0, 0, 0, 0, 0};
    int64_t k = 0;
    for (int cls = 0; cls < 4; ++cls) {
        cls_begin[cls] = (int)k;
        for (int32_t t = 0; t < nt; ++t) {
            if (class_of(tlen[t], aff) != cls) continue;
            for (int g = 0; g < nq; g += kWarp) {
                WorkItem w;
                memset(&w, 0, sizeof(w));
                w.target = t;
                w.first = g;
                w.lanes = std::min(kWarp, nq - g);
                w.xmax = qlen[qord[g]];
                w.S = S_of(cls);
                items[k++] = w;
            }
        }
    }
    cls_begin[4] = (int)k;

    cudaError_t c = cudaMemcpy(dev_base, h, staged, cudaMemcpyHostToDevice);
    if (c != cudaSuccess) return report(err, err_bytes, PW_ERR_KERNEL, "staging copy: %s", cudaGetErrorString(c));
    c = cudaMemset(dev_base + o_counter, 0, 256);
    if (c != cudaSuccess) return report(err, err_bytes, PW_ERR_KERNEL, "counter reset: %s", cudaGetErrorString(c));

    KernelArgs A;
    memset(&A, 0, sizeof(A));
    A.P.affine = aff;
    A.P.is_float = ints ? 0 : 1;
    A.P.gap_i = (int)gap;
    A.P.ext_i = aff ? (int)ext : 0;
    A.P.ge_i = A.P.gap_i + A.P.ext_i;
    A.P.gap_f = gap;
    A.P.ext_f = aff ? ext : 0.0f;
    A.P.ge_f = gap + A.P.ext_f;
    A.P.alpha = alpha;
    A.P.dim = dim;
    A.q = SeqSet{dev_base + o_qc, (const int64_t*)(dev_base + o_qco), nullptr, nullptr,
                 (const int32_t*)(dev_base + o_qlen), nullptr};
    A.t = SeqSet{dev_base + o_tc, (const int64_t*)(dev_base + o_tco), nullptr, nullptr,
                 (const int32_t*)(dev_base + o_tlen), nullptr};
    A.q_order = (const int32_t*)(dev_base + o_qord);
    A.cmat_i8 = (const int8_t*)(dev_base + o_cm8);
    A.cmat_f = (const float*)(dev_base + o_cmf);
    A.pair_max = (float*)(dev_base + o_pm);
    A.nt = nt;
    A.pm_lane = nt;
    A.pm_strip = 1;
    A.bnd_pool = dev_base + o_bnd;
    A.bnd_slot_elems = (int64_t)xmax4 * kWarp;
    for (int cls = 0; cls < 4; ++cls) {
        const int n = cls_begin[cls + 1] - cls_begin[cls];
        if (n <= 0) continue;
        A.items = (const WorkItem*)(dev_base + o_items) + cls_begin[cls];
        A.n_items = n;
        A.item_counter = (int*)(dev_base + o_counter) + cls;
        const int max_blocks = cls == 3 ? max_warps / 4 : (1 << 20);
        c = ints ? launch_cls<int>(cls, aff, A, max_blocks) : launch_cls<float>(cls, aff, A, max_blocks);
        if (c != cudaSuccess) return report(err, err_bytes, PW_ERR_KERNEL, "launch: %s", cudaGetErrorString(c));
    }
    c = cudaMemcpy(pair_max, dev_base + o_pm, (size_t)nq * nt * sizeof(float), cudaMemcpyDeviceToHost);
    if (c != cudaSuccess) return report(err, err_bytes, PW_ERR_KERNEL, "result copy: %s", cudaGetErrorString(c));
    return PW_OK;
}
