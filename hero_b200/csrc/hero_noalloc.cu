// hero_noalloc.cu -- banded DP over caller-owned device buffers, with no allocation.
//
// Some callers cannot allocate device memory themselves: code running inside a
// host framework whose allocator owns the GPU (a plugin handed device buffers
// by its host, a pool that forbids stray cudaMalloc calls while a graph or a
// fixed memory plan is live).  hero_align_segments_noalloc serves them: the
// caller passes every input and output in device memory it already owns, and
// the only working memory is the fixed array below, which lives in the
// library's module for as long as the process has it loaded.
//
// Limits: a segment may have at most kNoallocMaxSide bases on either side
// (after setSequences puts the longer side on the rows), and at most
// kNoallocThreads segments are in flight at once.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hero_gpu.h"
#include "hero_internal.cuh"

namespace hero {
namespace {

constexpr int kNoallocMaxSide = 128;
constexpr int kNoallocThreads = 8192;
// 32-thread blocks: 256 of them, so every one of a B200's 148 SMs gets work
constexpr int kNoallocBlock = 32;
constexpr int kNoallocStrips = (kNoallocMaxSide + kStripW - 1) / kStripW;
// per thread: traceback codes (u16 per strip row), the boundary column and the
// base codes of the segment's two sides; all interleaved by thread
constexpr size_t kNoallocTbBytes = size_t(kNoallocThreads) * kNoallocMaxSide * kNoallocStrips * 2;
constexpr size_t kNoallocBndBytes = size_t(kNoallocThreads) * 3 * (kNoallocMaxSide + 1) * 4;
constexpr size_t kNoallocCodeBytes = size_t(kNoallocThreads) * 2 * kNoallocMaxSide;
constexpr size_t kNoallocScratchBytes =
    kNoallocTbBytes + kNoallocBndBytes + kNoallocCodeBytes;  // 48.2 MB

// The fixed working array (every call shares it; its contents are never read
// before being written within a call, so nothing needs clearing) and the
// per-call status word (cleared by each call before its launch).
__device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocScratchBytes];
__device__ int g_noalloc_status;

struct NoallocScratch {
    uint16_t *tb;
    int32_t *bnd;
    uint64_t t;
    __device__ __forceinline__ void tb_set(int32_t s, int32_t i, uint32_t bits) {
        tb[(uint64_t(s) * kNoallocMaxSide + uint64_t(i - 1)) * kNoallocThreads + t] = uint16_t(bits);
    }
    __device__ __forceinline__ uint32_t tb_get(int32_t s, int32_t i) const {
        return tb[(uint64_t(s) * kNoallocMaxSide + uint64_t(i - 1)) * kNoallocThreads + t];
    }
    __device__ __forceinline__ int32_t &b(int32_t st, int32_t i) {
        return bnd[(uint64_t(st) * (kNoallocMaxSide + 1) + uint64_t(i)) * kNoallocThreads + t];
    }
};

// A read view over ASCII bases in caller memory: codes are derived on the fly.
struct AsciiView {
    const uint8_t *base;
    int32_t dir;
    uint8_t x;
    __device__ __forceinline__ uint8_t at(int32_t i) const {
        return uint8_t(base_code(base[int64_t(dir) * i]) ^ x);
    }
};

template <bool AFFINE>
__global__ void __launch_bounds__(kNoallocBlock)
    k_dp_noalloc(uint8_t *scratch, const uint8_t *subj, const uint64_t *subj_off, uint64_t n_subj,
                 const uint8_t *query, const uint64_t *query_off, uint64_t n_query,
                 uint64_t n_seg, const uint32_t *seg_subject, const uint8_t *seg_orient,
                 const uint32_t *seg_query, const int32_t *s0v, const int32_t *s1v,
                 const int32_t *q0v, const int32_t *q1v, const uint8_t *seg_flags,
                 const int64_t *band, const uint64_t *ops_off, uint8_t *ops, int32_t *nops) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    NoallocScratch sc{reinterpret_cast<uint16_t *>(scratch),
                      reinterpret_cast<int32_t *>(scratch + kNoallocTbBytes), t};
    for (uint64_t i = t; i < n_seg; i += kNoallocThreads) {
        const uint32_t si = seg_subject[i], qi = seg_query[i];
        const int32_t s0 = s0v[i], s1 = s1v[i], q0 = q0v[i], q1 = q1v[i];
        const int64_t ls_read = si < n_subj ? int64_t(subj_off[si + 1] - subj_off[si]) : -1;
        const int64_t lq_read = qi < n_query ? int64_t(query_off[qi + 1] - query_off[qi]) : -1;
        const int32_t ls = s1 - s0, lq = q1 - q0;
        // the output slot: ops_off must not decrease (a decreasing pair would
        // wrap the unsigned capacity and pass the size test below)
        const uint64_t o0 = ops_off[i], o1 = ops_off[i + 1];
        const uint64_t cap = o1 >= o0 ? o1 - o0 : 0;
        if (ls_read < 0 || lq_read < 0 || s0 < 0 || ls < 1 || s1 > ls_read || q0 < 0 || lq < 1 ||
            q1 > lq_read || ls > kNoallocMaxSide || lq > kNoallocMaxSide || o1 < o0 ||
            cap < uint64_t(ls + lq)) {
            nops[i] = -1;
            atomicExch(&g_noalloc_status, 1);
            continue;
        }
        // the codes of both sides as setSequences lays them out (longer side on
        // the rows), converted from the caller's ASCII into this thread's slots
        const uint8_t orient = seg_orient[i] & 1u;
        const uint8_t *sb = subj + subj_off[si];
        AsciiView sv = orient ? AsciiView{sb + (ls_read - 1 - s0), -1, 2} : AsciiView{sb + s0, 1, 0};
        AsciiView qv{query + query_off[qi] + q0, 1, 0};
        uint8_t *rowc = scratch + kNoallocTbBytes + kNoallocBndBytes + t;
        uint8_t *colc = rowc + uint64_t(kNoallocThreads) * kNoallocMaxSide;
        const bool rev = lq > ls;
        const int32_t R = rev ? lq : ls, C = rev ? ls : lq;
        for (int32_t k = 0; k < R; k++) rowc[uint64_t(k) * kNoallocThreads] = rev ? qv.at(k) : sv.at(k);
        for (int32_t k = 0; k < C; k++) colc[uint64_t(k) * kNoallocThreads] = rev ? sv.at(k) : qv.at(k);
        const int64_t b = band[i] > 65535 ? 65535 : (band[i] < 0 ? 0 : band[i]);
        SegView w;
        w.row_base = rowc;
        w.col_base = colc;
        w.row_dir = kNoallocThreads;
        w.col_dir = kNoallocThreads;
        w.row_xor = 0;
        w.col_xor = 0;
        w.R = R;
        w.C = C;
        w.band = b > int64_t(R - C) ? b : int64_t(R - C);  // setBand, then widened (BandAligner.cpp:59-62)
        w.right = (seg_flags[i] & DPF_RIGHT) != 0;
        w.left = (seg_flags[i] & DPF_LEFT) != 0;
        w.reversed = rev;  // ops are reported in the original orientation
        dp_fill<kStripW, AFFINE>(w, sc);
        uint8_t *out = ops + ops_off[i];
        int32_t k = 0;
        auto emit = [&](uint8_t op) { out[cap - 1 - k++] = op; };
        DpSum sum;
        const int32_t n = dp_traceback<kStripW>(w, sc, emit, sum);
        for (int32_t m = 0; m < n; m++) out[m] = out[cap - n + m];  // to the front
        nops[i] = n;
    }
}

// the array's device address per device, looked up on the first call made on
// that device; only a successful lookup is kept, so a call that failed (for
// instance one made while its stream was being captured) is retried by the next
void *g_scratch_ptr[64];
std::mutex g_scratch_mu;

void *scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) == cudaSuccess) g_scratch_ptr[dev] = p;
        else (void)cudaGetLastError();  // a failed lookup leaves no error behind for the caller
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace hero

using namespace hero;

extern "C" int hero_align_segments_noalloc(int affine, const uint8_t *subj, const uint64_t *subj_off,
                                           uint64_t n_subj, const uint8_t *query,
                                           const uint64_t *query_off, uint64_t n_query,
                                           uint64_t n_seg, const uint32_t *seg_subject,
                                           const uint8_t *seg_orient, const uint32_t *seg_query,
                                           const int32_t *s0, const int32_t *s1, const int32_t *q0,
                                           const int32_t *q1, const uint8_t *seg_flags,
                                           const int64_t *band, int32_t max_side,
                                           const uint64_t *ops_off, uint8_t *ops, int32_t *nops,
                                           void *stream) {
    if (max_side < 1 || max_side > kNoallocMaxSide) return HERO_E_INPUT;
    if (n_seg == 0) return HERO_OK;
    if (!subj || !subj_off || !query || !query_off || !seg_subject || !seg_orient || !seg_query ||
        !s0 || !s1 || !q0 || !q1 || !seg_flags || !band || !ops_off || !ops || !nops)
        return HERO_E_INPUT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HERO_E_CUDA;
    // the array's device address, with this device current (looked up once)
    void *scratch = scratch_address(dev);
    if (!scratch) return HERO_E_CUDA;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int zero = 0;
    if (cudaMemcpyToSymbolAsync(g_noalloc_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice,
                                st) != cudaSuccess)
        return HERO_E_CUDA;
    const unsigned grid = kNoallocThreads / kNoallocBlock;
    uint8_t *scr = reinterpret_cast<uint8_t *>(scratch);
    if (affine) {
        k_dp_noalloc<true><<<grid, kNoallocBlock, 0, st>>>(
            scr, subj, subj_off, n_subj, query, query_off, n_query, n_seg, seg_subject, seg_orient,
            seg_query, s0, s1, q0, q1, seg_flags, band, ops_off, ops, nops);
    } else {
        k_dp_noalloc<false><<<grid, kNoallocBlock, 0, st>>>(
            scr, subj, subj_off, n_subj, query, query_off, n_query, n_seg, seg_subject, seg_orient,
            seg_query, s0, s1, q0, q1, seg_flags, band, ops_off, ops, nops);
    }
    if (cudaGetLastError() != cudaSuccess) return HERO_E_CUDA;
    int status = 0;
    if (cudaMemcpyFromSymbolAsync(&status, g_noalloc_status, sizeof(int), 0,
                                  cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return HERO_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HERO_E_CUDA;
    return status ? HERO_E_INPUT : HERO_OK;
}
