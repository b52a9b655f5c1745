// hero_kernels.cu -- sm_100a kernels of the HERO read-correction path.
//
// Stage map (reference function -> kernel):
//   QueryDataset::qualityFilter / setGcContent        k_codes, k_read_flags
//   HashTableLongKey::insertQueryDataset              k_key_count, k_key_emit,
//                                                     k_table_insert/fill/finalize
//   SubjectReadAligner::searchHashTable2 (+ sort)     k_probe, k_sort_hits
//   processOneSubjectRead2 chaining + getAlignment2
//   segment layout                                    k_chain
//   BandAligner::calculateAlignment                   k_dp_hist/scatter, k_dp
//   AlignmentRecord scoring + early exits             k_assemble
//   SubjectRead::addAlignment                         k_dedupe
//   SubjectRead::updateQueryCoverage                  k_vote
//   QueryRead::callConsensus + coverage statistics    k_consensus
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "hero_internal.cuh"

namespace hero {

namespace {

std::atomic<uint64_t> g_launches{0};
inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }

constexpr uint32_t kEmptyOwner = 0xffffffffu;

inline unsigned grid_1d(uint64_t n, unsigned block, unsigned cap = 148u * 64u) {
    uint64_t g = (n + block - 1) / block;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return unsigned(g);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
template <class T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
// exclusive prefix over lanes; *total receives the warp total
template <class T>
__device__ __forceinline__ T warp_exclusive(T v, T *total) {
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (int(lane_id()) >= o) x += y;
    }
    *total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// ---------------------------------------------------------------------------
// reads
// ---------------------------------------------------------------------------
__global__ void k_codes(const uint8_t *raw, uint64_t n, uint8_t *code) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x)
        code[i] = base_code(raw[i]);
}

// QueryDataset::qualityFilter (QueryDataset.cpp:60-75), the good-read tests of
// QueryDataset.cpp:226 (query) and SubjectDataset.cpp:157-162 (subject), and
// QueryRead::setGcContent (QueryRead.cpp:73-81)
__global__ void k_read_flags(const uint8_t *code, const uint64_t *off, uint64_t n, uint32_t *len,
                             uint8_t *gq, uint8_t *gs, double *gc, int32_t l) {
    for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
         r += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t b = off[r], L = off[r + 1] - b;
        uint64_t cnt[4] = {0, 0, 0, 0};
        bool valid = true;
        uint64_t ngc = 0;
        for (uint64_t i = 0; i < L; i++) {
            const uint8_t c = code[b + i];
            if (c >= 4) {
                valid = false;
            } else {
                cnt[c]++;
                ngc += (c & 1u);  // C (1) or G (3)
            }
        }
        bool qf = valid;
        if (qf) {
            const uint64_t thr = uint64_t(__dmul_rn(double(L), 0.8));
            if (cnt[0] >= thr || cnt[1] >= thr || cnt[2] >= thr || cnt[3] >= thr) qf = false;
        }
        const uint64_t lu = uint16_t(l);  // the reference compares with a UINT16 copy
        len[r] = uint32_t(L);
        if (gq) gq[r] = (L > lu && qf) ? 1 : 0;
        if (gs) gs[r] = (L < lu || qf) ? 1 : 0;
        if (gc) gc[r] = __ddiv_rn(double(ngc), double(L));
    }
}

// ---------------------------------------------------------------------------
// exclusive scan (u32 counts -> u64 offsets, n+1 entries)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

template <class T>
__global__ void k_scan_tile(const T *in, uint64_t n, uint64_t *out, uint64_t *tile_sums) {
    __shared__ uint64_t warp_tot[kScanThreads / 32];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    uint64_t loc[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint64_t idx = base + j;
        const uint64_t v = idx < n ? uint64_t(in[idx]) : 0;
        loc[j] = s;
        s += v;
    }
    uint64_t tot;
    uint64_t ex = warp_exclusive<uint64_t>(s, &tot);
    if (lane_id() == 0) warp_tot[threadIdx.x >> 5] = tot;
    __syncthreads();
    uint64_t wpre = 0, btot = 0;
    for (int w = 0; w < kScanThreads / 32; w++) {
        if (w < int(threadIdx.x >> 5)) wpre += warp_tot[w];
        btot += warp_tot[w];
    }
    ex += wpre;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint64_t idx = base + j;
        if (idx < n) out[idx] = ex + loc[j];
    }
    if (threadIdx.x == 0) {
        tile_sums[blockIdx.x] = btot;
        if (blockIdx.x == gridDim.x - 1) out[n] = btot;
    }
}

__global__ void k_scan_add(uint64_t *out, uint64_t n, const uint64_t *tile_prefix) {
    const uint64_t add = tile_prefix[blockIdx.x];
    if (add == 0) return;
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile;
    for (uint64_t i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        const uint64_t idx = base + i;
        if (idx < n) out[idx] += add;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] += add;
}

size_t scan_levels_bytes(uint64_t n) {
    size_t b = 0;
    uint64_t m = n;
    while (true) {
        const uint64_t nt = (m + kScanTile - 1) / kScanTile;
        b += (nt + 1) * 2 * sizeof(uint64_t);
        if (nt <= 1) break;
        m = nt;
    }
    return b + 256;
}

template <class T>
void scan_rec(const T *in, uint64_t *out, uint64_t n, uint64_t *tmp, cudaStream_t st) {
    if (n == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint64_t), st);
        return;
    }
    const uint64_t nt = (n + kScanTile - 1) / kScanTile;
    uint64_t *sums = tmp;
    uint64_t *pref = tmp + (nt + 1);
    counted();
    k_scan_tile<T><<<unsigned(nt), kScanThreads, 0, st>>>(in, n, out, sums);
    if (nt > 1) {
        scan_rec<uint64_t>(sums, pref, nt, tmp + 2 * (nt + 1), st);
        counted();
        k_scan_add<<<unsigned(nt), kScanThreads, 0, st>>>(out, n, pref);
    }
}

// ---------------------------------------------------------------------------
// k-mer table (HashTableLongKey.cpp:41-68, 250-342)
// ---------------------------------------------------------------------------
__global__ void k_key_count(ReadsView q, int32_t k, uint32_t *count) {
    for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < q.n;
         r += uint64_t(gridDim.x) * blockDim.x)
        count[r] = q.good[r] ? uint32_t(query_key_count(q.len[r], k)) : 0u;
}

__global__ void k_key_emit(ReadsView q, int32_t k, const uint64_t *key_off, uint64_t *klo,
                           uint64_t *khi, uint64_t *kval) {
    for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < q.n;
         r += uint64_t(gridDim.x) * blockDim.x) {
        if (!q.good[r]) continue;
        const int64_t L = q.len[r];
        const int32_t nk = query_key_count(L, k);
        const uint8_t *c = q.code + q.off[r];
        uint64_t e = key_off[r];
        const uint32_t tag = uid_tag(q.uid[r]);
        for (int32_t i = 0; i < nk; i++, e++) {
            const int64_t pos = query_key_pos(L, k, i);
            Kmer m{0, 0};
            for (int32_t t = 0; t < k; t++) kmer_push(m, c[pos + t] & 3u, k);
            if (q.job) kmer_tag(m, q.job[r], k);
            klo[e] = m.lo;
            khi[e] = m.hi;
            kval[e] = table_value(r, tag, pos);
        }
    }
}

__global__ void k_table_insert(const uint64_t *klo, const uint64_t *khi, uint64_t nkeys,
                               uint32_t *owner, uint32_t *count, uint32_t *slot_of,
                               uint64_t mask) {
    for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < nkeys;
         e += uint64_t(gridDim.x) * blockDim.x) {
        const Kmer m{klo[e], khi[e]};
        uint64_t h = kmer_hash(m) & mask;
        for (uint64_t it = 0; it <= mask; it++) {
            const uint32_t prev = atomicCAS(&owner[h], kEmptyOwner, uint32_t(e));
            if (prev == kEmptyOwner || (klo[prev] == m.lo && khi[prev] == m.hi)) {
                slot_of[e] = uint32_t(h);
                atomicAdd(&count[h], 1u);
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

__global__ void k_table_fill(const uint64_t *kval, uint64_t nkeys, const uint32_t *slot_of,
                             const uint64_t *start, uint32_t *fill, uint64_t *vals) {
    for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < nkeys;
         e += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t s = slot_of[e];
        const uint64_t p = start[s] + atomicAdd(&fill[s], 1u);
        vals[p] = kval[e];
    }
}

__global__ void k_table_finalize(const uint64_t *klo, const uint64_t *khi, const uint32_t *owner,
                                 const uint32_t *count, const uint64_t *start, uint64_t nslots,
                                 Slot *slots) {
    for (uint64_t h = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < nslots;
         h += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t o = owner[h];
        Slot s;
        s.pad = 0;
        if (o != kEmptyOwner) {
            s.lo = klo[o];
            s.hi = khi[o];
            s.start = uint32_t(start[h]);
            s.count = count[h];
        } else {
            s.lo = 0;
            s.hi = 0;
            s.start = 0;
            s.count = 0;
        }
        slots[h] = s;
    }
}

// exact multimap lookup (HashTableLongKey::getListOfReads, HashTableLongKey.cpp:79-99)
__device__ __forceinline__ bool table_find(const TableView &t, const Kmer &m, uint32_t &start,
                                           uint32_t &count) {
    uint64_t h = kmer_hash(m) & t.mask;
    for (uint64_t it = 0; it <= t.mask; it++) {
        const uint4 a = __ldg(reinterpret_cast<const uint4 *>(&t.slots[h]));
        const uint4 b = __ldg(reinterpret_cast<const uint4 *>(&t.slots[h]) + 1);
        const uint32_t cnt = b.y;
        if (cnt == 0) return false;
        const uint64_t lo = (uint64_t(a.y) << 32) | a.x, hi = (uint64_t(a.w) << 32) | a.z;
        if (lo == m.lo && hi == m.hi) {
            start = b.x;
            count = cnt;
            return true;
        }
        h = (h + 1) & t.mask;
    }
    return false;
}

// ---------------------------------------------------------------------------
// seeding: SubjectReadAligner::searchHashTable2 (SubjectReadAligner.cpp:444-491)
// Count pass: one warp per subject read; lane f takes the contiguous windows
// [fa, fb), so both k-mers roll one base per window (the forward window at f
// and the reverse-complement window at L-k-f are the same bases).  It probes
// the table for each window and orientation, counts the hits of each
// (subject, orientation) and leaves the slot it found (start, count) in the
// window cache, indexed by the window's base in the batch: 2 entries a base.
// Emit pass: the same warps read the cache (lanes interleaved, so the reads
// are coalesced) and write the hits without probing the table again.
// ---------------------------------------------------------------------------
constexpr int kProbeWarps = 8;

__global__ void __launch_bounds__(kProbeWarps * 32)
    k_probe_count(ReadsView subj, uint64_t nsub, ReadsView q, TableView t, int32_t k, uint2 *wcache,
                  uint32_t *seg_hits, unsigned long long *counters) {
    const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
    const uint64_t warps = uint64_t(gridDim.x) * kProbeWarps;
    const uint64_t base0 = subj.off[0];
    unsigned long long probes = 0, nhits = 0;
    for (uint64_t s = uint64_t(blockIdx.x) * kProbeWarps + wib; s < nsub; s += warps) {
        const int32_t L = int32_t(subj.len[s]);
        const int64_t su = subj.uid[s];
        const uint32_t stag = uid_tag(su);
        const uint8_t *c = subj.code + subj.off[s];
        uint2 *wc = wcache + 2 * (subj.off[s] - base0);
        uint32_t c0 = 0, c1 = 0;
        if (subj.good[s] && L >= k) {
            const int32_t P = L - k + 1;
            if (lane == 0) probes += 2ull * uint64_t(P);
            // nbad counts the non-ACGT bases in the window
            const int32_t fa = int32_t(int64_t(P) * lane / 32), fb = int32_t(int64_t(P) * (lane + 1) / 32);
            Kmer fr{0, 0}, rr{0, 0};
            int32_t nbad = 0;
            if (fa < fb)
                for (int32_t i = 0; i < k - 1; i++) {
                    const uint8_t x = c[fa + i];
                    nbad += x >= 4;
                    kmer_push(fr, x & 3u, k);
                    kmer_push_front(rr, (x & 3u) ^ 2u, k);
                }
            for (int32_t f = fa; f < fb; f++) {
                const uint8_t x = c[f + k - 1];
                nbad += x >= 4;
                if (f > fa) nbad -= c[f - 1] >= 4;
                kmer_push(fr, x & 3u, k);
                kmer_push_front(rr, (x & 3u) ^ 2u, k);
                uint2 found[2] = {make_uint2(0, 0), make_uint2(0, 0)};
                if (!nbad) {
                    Kmer fm = fr, rm = rr;
                    if (subj.job) {
                        kmer_tag(fm, subj.job[s], k);
                        kmer_tag(rm, subj.job[s], k);
                    }
                    for (int o = 0; o < 2; o++) {
                        uint32_t st = 0, cnt = 0;
                        if (!table_find(t, o ? rm : fm, st, cnt)) continue;
                        found[o] = make_uint2(st, cnt);
                        for (uint32_t e = 0; e < cnt; e++) {
                            const uint64_t v = __ldg(&t.vals[st + e]);
                            // self hit (SubjectReadAligner.cpp:463-465): ids compared
                            // only where their folds agree
                            if (value_tag(v) == stag && __ldg(&q.uid[value_query(v)]) == su) continue;
                            if (o) {
                                c1++;
                            } else {
                                c0++;
                            }
                        }
                    }
                }
                reinterpret_cast<uint4 *>(wc)[f] = make_uint4(found[0].x, found[0].y, found[1].x, found[1].y);
            }
        }
        c0 = warp_sum(c0);
        c1 = warp_sum(c1);
        if (lane == 0) {
            seg_hits[2 * s] = c0;
            seg_hits[2 * s + 1] = c1;
            nhits += c0 + c1;
        }
    }
    if (lane == 0) {
        atomicAdd(&counters[C_PROBES], probes);
        atomicAdd(&counters[C_HITS], nhits);
    }
}

__global__ void __launch_bounds__(kProbeWarps * 32)
    k_probe_emit(ReadsView subj, uint64_t nsub, ReadsView q, TableView t, int32_t k, bool aln,
                 const uint2 *wcache, const uint64_t *hit_off, uint64_t *hits) {
    __shared__ uint32_t fill[kProbeWarps][2];
    const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
    const uint64_t warps = uint64_t(gridDim.x) * kProbeWarps;
    const uint64_t base0 = subj.off[0];
    for (uint64_t s = uint64_t(blockIdx.x) * kProbeWarps + wib; s < nsub; s += warps) {
        const int32_t L = int32_t(subj.len[s]);
        if (lane == 0) {
            fill[wib][0] = 0;
            fill[wib][1] = 0;
        }
        __syncwarp();
        if (subj.good[s] && L >= k) {
            const int64_t su = subj.uid[s];
            const uint32_t stag = uid_tag(su);
            const uint64_t o0 = hit_off[2 * s], o1 = hit_off[2 * s + 1];
            const uint4 *wc = reinterpret_cast<const uint4 *>(wcache + 2 * (subj.off[s] - base0));
            const int32_t P = L - k + 1;
            for (int32_t f = int32_t(lane); f < P; f += 32) {
                const uint4 w = wc[f];
                for (int o = 0; o < 2; o++) {
                    const uint32_t st = o ? w.z : w.x, cnt = o ? w.w : w.y;
                    for (uint32_t e = 0; e < cnt; e++) {
                        const uint64_t v = __ldg(&t.vals[st + e]);
                        const uint32_t qq = value_query(v);
                        if (value_tag(v) == stag && __ldg(&q.uid[qq]) == su) continue;
                        const uint32_t slot = atomicAdd(&fill[wib][o], 1u);
                        const int32_t lq = (aln && o) ? int32_t(__ldg(&q.len[qq])) : 0;
                        hits[(o ? o1 : o0) + slot] = seed_hit(aln, o, qq, value_pos(v), f, L, lq, k);
                    }
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// per-segment sort of hits by (query, posQ, posS) (SubjectRead::sortKeyPosition)
// Bitonic network in its all-ascending form (mirror step + half cleaners), so
// positions past n behave as +infinity and need no storage.
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256, kSortSmem = 4096;

__device__ __forceinline__ void cmpx(uint64_t *a, uint64_t lo, uint64_t hi) {
    const uint64_t x = a[lo], y = a[hi];
    if (y < x) {
        a[lo] = y;
        a[hi] = x;
    }
}

__device__ void bitonic(uint64_t *a, uint64_t n, uint64_t N) {
    for (uint64_t k = 2; k <= N; k <<= 1) {
        const uint64_t half = k >> 1;
        for (uint64_t i = threadIdx.x; i < N / 2; i += blockDim.x) {
            const uint64_t blk = i / half, off = i % half;
            const uint64_t lo = blk * k + off, hi = blk * k + k - 1 - off;
            if (hi < n) cmpx(a, lo, hi);
        }
        __syncthreads();
        for (uint64_t j = half >> 1; j >= 1; j >>= 1) {
            for (uint64_t i = threadIdx.x; i < N / 2; i += blockDim.x) {
                const uint64_t blk = i / j, off = i % j;
                const uint64_t lo = blk * 2 * j + off, hi = lo + j;
                if (hi < n) cmpx(a, lo, hi);
            }
            __syncthreads();
        }
    }
}

// The same network run by one warp on up to kWarpSort hits in shared memory,
// with power-of-two index arithmetic (segments hold ~100 hits).
constexpr int kWarpSort = 512;

__device__ __forceinline__ void bitonic_warp(uint64_t *a, uint32_t n, uint32_t lgN) {
    const uint32_t lane = threadIdx.x & 31u, N = 1u << lgN;
    for (uint32_t lk = 1; lk <= lgN; lk++) {
        const uint32_t k = 1u << lk, hm = (k >> 1) - 1u;
        for (uint32_t i = lane; i < N / 2; i += 32u) {  // mirror step of stage k
            const uint32_t base = (i >> (lk - 1)) << lk, off = i & hm;
            const uint32_t lo = base + off, hi = base + k - 1u - off;
            if (hi < n) cmpx(a, lo, hi);
        }
        __syncwarp();
        for (uint32_t lj = lk - 1; lj-- > 0;) {  // half cleaners, j = 2^lj
            const uint32_t jm = (1u << lj) - 1u;
            for (uint32_t i = lane; i < N / 2; i += 32u) {
                const uint32_t lo = ((i >> lj) << (lj + 1)) + (i & jm), hi = lo + (1u << lj);
                if (hi < n) cmpx(a, lo, hi);
            }
            __syncwarp();
        }
    }
}

// small segments: one warp each, in shared memory
__global__ void __launch_bounds__(kSortThreads)
    k_sort_hits_warp(uint64_t nseg, const uint64_t *hit_off, uint64_t *hits) {
    __shared__ uint64_t sm[kSortThreads / 32][kWarpSort];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    for (uint64_t seg = uint64_t(blockIdx.x) * (kSortThreads / 32) + wib; seg < nseg;
         seg += uint64_t(gridDim.x) * (kSortThreads / 32)) {
        const uint64_t b = hit_off[seg], n = hit_off[seg + 1] - b;
        if (n < 2 || n > uint64_t(kWarpSort)) continue;
        uint32_t lgN = 0;
        while ((1u << lgN) < uint32_t(n)) lgN++;
        uint64_t *a = sm[wib];
        for (uint32_t i = lane; i < uint32_t(n); i += 32u) a[i] = hits[b + i];
        __syncwarp();
        bitonic_warp(a, uint32_t(n), lgN);
        for (uint32_t i = lane; i < uint32_t(n); i += 32u) hits[b + i] = a[i];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kSortThreads)
    k_sort_hits(uint64_t nseg, const uint64_t *hit_off, uint64_t *hits) {
    __shared__ uint64_t sm[kSortSmem];
    for (uint64_t seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
        const uint64_t b = hit_off[seg], n = hit_off[seg + 1] - b;
        if (n <= uint64_t(kWarpSort)) continue;  // sorted by k_sort_hits_warp
        uint64_t N = 1;
        while (N < n) N <<= 1;
        if (n <= uint64_t(kSortSmem)) {
            for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) sm[i] = hits[b + i];
            __syncthreads();
            bitonic(sm, n, N);
            for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) hits[b + i] = sm[i];
            __syncthreads();
        } else {
            bitonic(hits + b, n, N);
        }
    }
}

// ---------------------------------------------------------------------------
// chaining + record layout: processOneSubjectRead2 (SubjectReadAligner.cpp:805-852)
// One warp per (subject, orientation); lane g takes query groups g, g+32, ...
// ---------------------------------------------------------------------------
struct CountDp {
    uint32_t n = 0;
    HERO_HD void begin(int64_t, int64_t, int64_t) {}
    HERO_HD void position(int64_t) {}
    HERO_HD void run(uint8_t, int64_t) {}
    HERO_HD void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) { n++; }
    HERO_HD bool check(int64_t, int64_t) { return true; }
    HERO_HD void finish() {}
};

struct EmitDp {
    DpSeg *out;
    uint32_t subj, query, orient;
    uint32_t orient_shift;  // the subject's orientation (-c), or the query's (alignment output)
    uint32_t n = 0;
    int32_t maxr = 0, maxc = 0;
    HERO_HD void begin(int64_t, int64_t, int64_t) {}
    HERO_HD void position(int64_t) {}
    HERO_HD void run(uint8_t, int64_t) {}
    HERO_HD void dp(int64_t s0, int64_t s1, int64_t q0, int64_t q1, uint32_t flags, int64_t band) {
        DpSeg g;
        g.subj = subj;
        g.query = query;
        g.s0 = uint16_t(s0);
        g.s1 = uint16_t(s1);
        g.q0 = uint16_t(q0);
        g.q1 = uint16_t(q1);
        // any band >= 65535 covers every cell of a segment of reads below 65536 bases
        g.band = int32_t(band > 65535 ? 65535 : band);
        g.flags = flags | (orient << orient_shift);
        g.pad = 0;
        out[n++] = g;
        const int32_t ls = int32_t(s1 - s0), lq = int32_t(q1 - q0);
        const int32_t r = ls > lq ? ls : lq, c = ls > lq ? lq : ls;
        if (r > maxr) maxr = r;
        if (c > maxc) maxc = c;
    }
    HERO_HD bool check(int64_t, int64_t) { return true; }
    HERO_HD void finish() {}
};

__global__ void __launch_bounds__(256)
    k_chain(Params p, uint64_t nseg, ReadsView subj, ReadsView q, const uint64_t *hit_off,
            const uint64_t *hits, ChainScratch sc, uint32_t *seg_chain_start,
            uint32_t *seg_chain_count, ChainArrays ch, uint32_t *keys, DpSeg *segs,
            uint64_t cap_chains, uint64_t cap_keys, uint64_t cap_segs,
            unsigned long long *counters) {
    const uint32_t lane = lane_id();
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    unsigned long long nchains_all = 0;
    int32_t maxr = 0, maxc = 0;
    for (uint64_t seg = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); seg < nseg;
         seg += warps) {
        const uint64_t base = hit_off[seg], n = hit_off[seg + 1] - base;
        const uint32_t s = uint32_t(seg >> 1), orient = uint32_t(seg & 1);
        if (n == 0) {
            if (lane == 0) {
                seg_chain_start[seg] = 0;
                seg_chain_count[seg] = 0;
            }
            continue;
        }
        const uint64_t *H = hits + base;
        // group starts (a group = hits of one query read)
        uint32_t ng = 0;
        for (uint64_t c0 = 0; c0 < n; c0 += 32) {
            const uint64_t i = c0 + lane;
            const bool flag = i < n && (i == 0 || hit_q(H[i]) != hit_q(H[i - 1]));
            const uint32_t m = __ballot_sync(0xffffffffu, flag);
            if (flag) sc.grp[base + ng + __popc(m & ((1u << lane) - 1u))] = uint32_t(i);
            ng += __popc(m);
        }
        __syncwarp();
        const int32_t Ls = int32_t(subj.len[s]);
        // pass A: chain every group, keep the results in the scratch
        uint32_t tk = 0, tkeys = 0, tdp = 0;
        for (uint32_t g = lane; g < ng; g += 32) {
            const uint32_t gs = sc.grp[base + g];
            const uint32_t ge = (g + 1 < ng) ? sc.grp[base + g + 1] : uint32_t(n);
            const int32_t gn = int32_t(ge - gs);
            const uint64_t off = base + gs;
            const uint64_t *G = H + gs;
            auto hit = [G](int32_t h) { return G[h]; };
            const int32_t nch = chain_group(p, hit, gn, sc.chain_of + off, sc.first + off, sc.last + off);
            const int64_t best = chain_key_lengths(p, hit, gn, sc.chain_of + off, nch, sc.kl + off, sc.prev + off);
            // bucket the keys by chain, in order
            for (int32_t c = 0; c < nch; c++) sc.size[off + c] = 0;
            for (int32_t h = 0; h < gn; h++) sc.size[off + sc.chain_of[off + h]]++;
            int32_t run = 0;
            for (int32_t c = 0; c < nch; c++) {
                sc.coff[off + c] = run;
                sc.prev[off + c] = run;
                run += sc.size[off + c];
            }
            for (int32_t h = 0; h < gn; h++) {
                const uint32_t c = sc.chain_of[off + h];
                sc.ckeys[off + sc.prev[off + c]++] = h;
            }
            const uint32_t qid = hit_q(G[0]);
            const int64_t Lq = q.len[qid];
            uint32_t kept = 0, nkeys = 0, ndp = 0;
            for (int32_t c = 0; c < nch; c++) {
                if (sc.kl[off + c] != best) continue;
                kept++;
                nkeys += uint32_t(sc.size[off + c]);
                const int32_t *ck = sc.ckeys + off + sc.coff[off + c];
                auto key = [G, ck](int32_t i) { return G[ck[i]]; };
                CountDp cv;
                walk_chain(p, Lq, Ls, key, sc.size[off + c], cv);
                ndp += cv.n;
            }
            sc.g_nch[off] = nch;
            sc.g_best[off] = best;
            sc.g_kept[off] = kept;
            sc.g_keys[off] = nkeys;
            sc.g_dp[off] = ndp;
            tk += kept;
            tkeys += nkeys;
            tdp += ndp;
            nchains_all += uint64_t(nch);
        }
        tk = warp_sum(tk);
        tkeys = warp_sum(tkeys);
        tdp = warp_sum(tdp);
        unsigned long long cs = 0, ks = 0, ds = 0;
        int overflow = 0;
        if (lane == 0) {
            cs = atomicAdd(&counters[C_NC], (unsigned long long)tk);
            ks = atomicAdd(&counters[C_NK], (unsigned long long)tkeys);
            ds = atomicAdd(&counters[C_ND], (unsigned long long)tdp);
            if (cs + tk > cap_chains || ks + tkeys > cap_keys || ds + tdp > cap_segs) {
                overflow = 1;
                atomicAdd(&counters[C_OVERFLOW], 1ull);
                atomicAdd(&counters[C_OVERFLOW_ALL], 1ull);
            }
            seg_chain_start[seg] = overflow ? 0u : uint32_t(cs);
            seg_chain_count[seg] = overflow ? 0u : tk;
        }
        overflow = __shfl_sync(0xffffffffu, overflow, 0);
        if (overflow) continue;
        cs = __shfl_sync(0xffffffffu, cs, 0);
        ks = __shfl_sync(0xffffffffu, ks, 0);
        ds = __shfl_sync(0xffffffffu, ds, 0);
        // pass B: emit chains, keys and DP segments in (query, chain) order
        for (uint32_t g0 = 0; g0 < ng; g0 += 32) {
            const uint32_t g = g0 + lane;
            const bool has = g < ng;
            uint32_t gs = 0, gk = 0, gkeys = 0, gdp = 0;
            if (has) {
                gs = sc.grp[base + g];
                gk = sc.g_kept[base + gs];
                gkeys = sc.g_keys[base + gs];
                gdp = sc.g_dp[base + gs];
            }
            uint32_t tot_c, tot_k, tot_d;
            const uint32_t ec = warp_exclusive<uint32_t>(gk, &tot_c);
            const uint32_t ek = warp_exclusive<uint32_t>(gkeys, &tot_k);
            const uint32_t ed = warp_exclusive<uint32_t>(gdp, &tot_d);
            if (has) {
                const uint32_t ge = (g + 1 < ng) ? sc.grp[base + g + 1] : uint32_t(n);
                const uint64_t off = base + gs;
                const uint64_t *G = H + gs;
                const uint32_t qid = hit_q(G[0]);
                const int64_t Lq = q.len[qid];
                const int32_t nch = sc.g_nch[off];
                const int64_t best = sc.g_best[off];
                (void)ge;
                uint64_t ci = cs + ec, ki = ks + ek, di = ds + ed;
                for (int32_t c = 0; c < nch; c++) {
                    if (sc.kl[off + c] != best) continue;
                    const int32_t sz = sc.size[off + c];
                    const int32_t *ck = sc.ckeys + off + sc.coff[off + c];
                    for (int32_t i = 0; i < sz; i++) {
                        const uint64_t x = G[ck[i]];
                        keys[ki + i] = (uint32_t(hit_posQ(x)) << 16) | uint32_t(hit_posS(x));
                    }
                    auto key = [G, ck](int32_t i) { return G[ck[i]]; };
                    EmitDp ev;
                    ev.out = segs + di;
                    ev.subj = s;
                    ev.query = qid;
                    ev.orient = orient;
                    ev.orient_shift = p.aln ? kSegQrcShift : kSegOrientShift;
                    walk_chain(p, Lq, Ls, key, sz, ev);
                    if (ev.maxr > maxr) maxr = ev.maxr;
                    if (ev.maxc > maxc) maxc = ev.maxc;
                    ch.subj[ci] = s;
                    ch.query[ci] = qid;
                    ch.key_off[ci] = uint32_t(ki);
                    ch.seg_off[ci] = uint32_t(di);
                    ch.nkeys[ci] = uint16_t(sz);
                    ch.nseg[ci] = uint16_t(ev.n);
                    ch.orient[ci] = uint8_t(orient);
                    ch.status[ci] = CH_NONE;
                    ch.win[ci] = 0;
                    ci++;
                    ki += uint32_t(sz);
                    di += ev.n;
                }
            }
            cs += tot_c;
            ks += tot_k;
            ds += tot_d;
        }
    }
    nchains_all = warp_sum(nchains_all);
    maxr = warp_max(maxr);
    maxc = warp_max(maxc);
    if (lane == 0) {
        atomicAdd(&counters[C_CHAINS], nchains_all);
        atomicMax(&counters[C_MAXR], (unsigned long long)maxr);
        atomicMax(&counters[C_MAXC], (unsigned long long)maxc);
    }
}

// ---------------------------------------------------------------------------
// banded DP (BandAligner.cpp:56-419), one thread per segment
// ---------------------------------------------------------------------------
struct DevScratch {
    uint16_t *tb;
    int32_t *bnd;
    uint64_t T;
    int32_t rmax;
    uint64_t t;
    __device__ __forceinline__ void tb_set(int32_t s, int32_t i, uint32_t bits) {
        tb[(uint64_t(s) * uint64_t(rmax) + uint64_t(i - 1)) * T + t] = uint16_t(bits);
    }
    __device__ __forceinline__ uint32_t tb_get(int32_t s, int32_t i) const {
        return tb[(uint64_t(s) * uint64_t(rmax) + uint64_t(i - 1)) * T + t];
    }
    __device__ __forceinline__ int32_t &b(int32_t st, int32_t i) {
        return bnd[(uint64_t(st) * uint64_t(rmax + 1) + uint64_t(i)) * T + t];
    }
};

struct OpsWriter {
    uint32_t *base;
    int32_t p;
    uint32_t acc = 0;
    __device__ __forceinline__ void operator()(uint8_t op) {
        p--;
        acc |= uint32_t(op) << (2 * (p & 15));
        if ((p & 15) == 0) {
            base[p >> 4] = acc;
            acc = 0;
        }
    }
    __device__ __forceinline__ void flush() {
        if (p & 15) base[p >> 4] = acc;
    }
};

// (strips, align-left column, rows): a warp of the wavefront kernel takes
// segments with equal strips, so they are grouped first; the align-left column
// (1 + position of column C in the last strip, 0 when not aligned left) and the
// row count keep the warps uniform
__device__ __forceinline__ uint32_t shape_key(const DpSeg &g) {
    const int32_t ls = g.s1 - g.s0, lq = g.q1 - g.q0;
    const int32_t r = ls > lq ? ls : lq, c = ls > lq ? lq : ls;
    int32_t nst = (c + kStripW - 1) / kStripW;
    if (nst > 63) nst = 63;
    const uint32_t wl = (g.flags & DPF_LEFT) ? 1u + uint32_t((c - 1) % kStripW) : 0u;
    return (uint32_t(nst) << kShapeStripShift) | (wl << 10) | uint32_t(r > 1023 ? 1023 : r);
}

// Counting sort by shape.  Segments of a chain mostly share a few shapes, so
// the lanes of a warp with equal keys (__match_any_sync) add their count with
// one atomic by the lowest of them; in the scatter each lane then takes its
// rank among them.  The order inside a bin is free: every segment writes its
// results to its own slot.
__global__ void k_dp_hist(const DpSeg *segs, uint64_t nd, uint32_t *bins) {
    const uint32_t lane = lane_id();
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) & ~uint64_t(31); b < nd;
         b += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = b + lane;
        const uint32_t key = i < nd ? shape_key(segs[i]) : 0xffffffffu;
        const uint32_t same = __match_any_sync(0xffffffffu, key);
        if (i < nd && lane == uint32_t(__ffs(int(same))) - 1u) atomicAdd(&bins[key], uint32_t(__popc(same)));
    }
}

__global__ void k_dp_scatter(const DpSeg *segs, uint64_t nd, uint32_t *cursor,
                             const uint64_t *bin_off, uint32_t *perm) {
    const uint32_t lane = lane_id();
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) & ~uint64_t(31); b < nd;
         b += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = b + lane;
        const uint32_t key = i < nd ? shape_key(segs[i]) : 0xffffffffu;
        const uint32_t same = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = uint32_t(__ffs(int(same))) - 1u;
        uint32_t base = 0;
        if (i < nd && lane == leader) base = atomicAdd(&cursor[key], uint32_t(__popc(same)));
        base = __shfl_sync(0xffffffffu, base, int(leader));
        if (i < nd) perm[bin_off[key] + base + __popc(same & ((1u << lane) - 1u))] = uint32_t(i);
    }
}

constexpr int kDpThreads = 128;

template <bool AFFINE>
__global__ void __launch_bounds__(kDpThreads) k_dp(DpLaunch a) {
    const uint64_t T = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    DevScratch sc{a.tb, a.bnd, T, a.rmax, t};
    for (uint64_t idx = t; idx < a.nd; idx += T) {
        const uint32_t si = a.perm ? a.perm[idx] : uint32_t(idx);
        const DpSeg g = a.segs[si];
        const SegView v = dpseg_view(g, a.scode, a.soff, a.slen, a.qcode, a.qoff);
        dp_fill<kStripW, AFFINE>(v, sc);
        OpsWriter w{a.ops + uint64_t(si) * a.stride, int32_t(a.stride * 16u)};
        DpSum sum;
        dp_traceback<kStripW>(v, sc, w, sum);
        w.flush();
        a.sums[si] = sum;
        if (a.cells) {
            const uint64_t cl = band_cells(v.R, v.C, v.band);
            a.cells[si] = uint32_t(cl > 0xffffffffull ? 0xffffffffull : cl);
        }
    }
}

// ---------------------------------------------------------------------------
// banded DP as a warp wavefront.  Segments are sorted by (strips, rows); a
// warp takes S = 32 / G segments that all have G strips of kStripW columns.
// Lane (g, s) owns strip s of segment g and computes row i = t - s + 1 at step
// t: the states of its strip's last column go to lane s+1 by __shfl_up_sync,
// which uses them as its left boundary one step later (and as its diagonal one
// step after that), so no boundary column is ever stored.  Each lane writes
// its 2-bit codes of a row to shared memory; lane s = 0 of every group then
// traces its segment back from there.
// ---------------------------------------------------------------------------
// warps per block of k_dp_wave: 4 (default) or 2; blocks per SM are set so that
// every thread keeps 128 registers
constexpr int kWaveWarps = 4;
// warps per SM the register budget is set for, by register tier: 16 (128
// registers a thread), 12 (168: the affine pair rows spill less) or 8 (up to
// 255: no spills, at two warps a scheduler).  A scheduler's 16K registers are
// shared by its warps, so 9-11 warps a SM allow no more than 12 do.
constexpr int kWaveSmWarps(int tier) { return tier == 2 ? 8 : (tier == 1 ? 12 : 16); }
constexpr int kWaveRegBlocks(int warps, int tier) {
    return kWaveSmWarps(tier) / warps > 0 ? kWaveSmWarps(tier) / warps : 1;
}
// register tier of a regs_per_thread value (0 = the default 128)
inline int wave_reg_tier(int32_t regs) { return regs > 168 ? 2 : (regs > 128 ? 1 : 0); }

constexpr int kTaskQueue = 127;  // tasks[127]: next task to hand out

// segments of n strips run as 16-bit pairs (n <= 32; bit 32 does not exist)
__device__ __forceinline__ bool pair_strips(uint32_t mask, int n) {
    return n < 32 && ((mask >> n) & 1u) != 0u;
}

__global__ void k_dp_tasks(const uint64_t *bin_off, uint64_t *tasks, uint32_t pair_mask) {
    // tasks[n] (n = 1..33): first task of segments with n strips; tasks[34+n]:
    // first sorted segment with n strips; tasks[68+n]: one past the last.
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint64_t t = 0;
    for (int n = 1; n <= 32; n++) {
        const uint64_t b = bin_off[uint32_t(n) << kShapeStripShift];
        const uint64_t e = bin_off[uint32_t(n + 1) << kShapeStripShift];
        tasks[n] = t;
        tasks[34 + n] = b;
        tasks[68 + n] = e;
        const uint64_t S = uint64_t(32 / n) * (pair_strips(pair_mask, n) ? 2u : 1u);  // segments a task
        t += (e - b + S - 1) / S;
    }
    tasks[33] = t;
    tasks[0] = bin_off[uint32_t(33) << kShapeStripShift];  // first segment for the per-thread kernel
    tasks[kTaskQueue] = 0;  // work queue head of k_dp_wave
}

// the wavefront over one warp's segments; FULL / LEFT are warp-uniform.  The
// wavefront paths are separate functions so that each gets its own register
// allocation (inlined into one kernel body they spill)
template <bool AFFINE, bool FULL, bool LEFT>
__device__ __noinline__ void wave_fill(const SegView v, bool active, int32_t R, int32_t Rw,
                                          int G, int s, int lane, int32_t wlast, uint16_t *tb) {
    const int32_t j0 = s * kStripW;
    uint8_t bc[kStripW];
    int32_t uf[kStripW], ux[kStripW], uy[kStripW];
    Cell3 prev{0, 0, 0};
    uint8_t ch = 0;
    if (active) {
        dp_strip_init<kStripW, AFFINE>(v, j0, bc, uf, ux, uy);
        prev = dp_row0<AFFINE>(v, j0);  // diagonal of row 1: (0, j0)
        if (R >= 1) ch = v.row(1);
    }
    Cell3 pub{kNEG, kNEG, kNEG};
    for (int32_t t = 0; t < Rw + G - 1; t++) {
        Cell3 in;
        in.f = __shfl_up_sync(0xffffffffu, pub.f, 1);
        in.x = __shfl_up_sync(0xffffffffu, pub.x, 1);
        in.y = __shfl_up_sync(0xffffffffu, pub.y, 1);
        const int32_t i = t - s + 1;
        if (active && i >= 1 && i <= R) {
            const uint8_t a = ch;
            if (i < R) ch = v.row(i + 1);  // next row's base, loaded a step early
            Cell3 left = (s == 0) ? dp_col0<AFFINE>(v, i) : in;
            const Cell3 dg = (s == 0) ? dp_col0<AFFINE>(v, i - 1) : prev;
            const Cell3 lb = left;
            const uint32_t bits = dp_strip_row<kStripW, AFFINE, FULL, LEFT>(v, i, j0, a, bc, uf, ux,
                                                                             uy, left, dg, wlast);
            tb[size_t(i - 1) * 32u + lane] = uint16_t(bits);
            pub = left;
            prev = lb;
        }
    }
}

// the wavefront over one warp's whole-band segments (dp_whole_row); LEFT: the
// warp's segments align left with column C at position wl of their last strip;
// tab is the lane's strip table in shared memory
template <bool AFFINE, bool LEFT>
__device__ __noinline__ void wave_whole(const SegView v, bool active, int32_t R, int32_t Rw,
                                        int G, int s, int lane, int32_t wl, uint16_t *tb,
                                        int32_t *tab) {
    const int32_t j0 = s * kStripW;
    int32_t f[kStripW], x[kStripW], m[kStripW], c0[3];
    int32_t pm = 0;
    const uint8_t *rp = v.row_base;
    uint32_t ch = 0;
    if (active) {
        dp_whole_table<kStripW>(v, j0, tab);
        dp_whole_init<AFFINE, kStripW>(v, j0, f, x, m, pm);
        dp_whole_col0<AFFINE>(v, c0);
        ch = (rp[0] ^ v.row_xor) & 3u;
    }
    const bool holds_c = LEFT && s == G - 1;
    int32_t pf = kNEG, py = kNEG, pmv = kNEG;  // FM, IY, M published to lane s+1
    uint16_t *tp = tb + lane;
#pragma unroll 1
    for (int32_t t = 0; t < Rw + G - 1; t++) {
        const int32_t inf = __shfl_up_sync(0xffffffffu, pf, 1);
        const int32_t iny = AFFINE ? __shfl_up_sync(0xffffffffu, py, 1) : 0;
        const int32_t inm = __shfl_up_sync(0xffffffffu, pmv, 1);
        const int32_t i = t - s + 1;
        if (active && uint32_t(i - 1) < uint32_t(R)) {
            const uint32_t a = ch;
            if (i < R) {
                rp += v.row_dir;
                ch = (rp[0] ^ v.row_xor) & 3u;  // next row's base, loaded a step early
            }
            const int32_t c0f = i * c0[0] + c0[1];
            int32_t lf = s == 0 ? c0f : inf;
            int32_t ly = s == 0 ? i * c0[0] + c0[2] : iny;
            const int4 s0 = reinterpret_cast<const int4 *>(tab + a * kStripW)[0];
            const int4 s1 = reinterpret_cast<const int4 *>(tab + a * kStripW)[1];
            const int32_t sc[kStripW] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
            const uint32_t diag = uint32_t(tab[4 * kStripW + a]);
            if (LEFT) dp_whole_left<AFFINE, kStripW>(wl, holds_c, f, x);
            const uint32_t bits = dp_whole_row<AFFINE, kStripW>(sc, diag, f, x, m, lf, ly, pm);
            *tp = uint16_t(bits);
            tp += 32;
            pf = lf;
            py = ly;
            pmv = AFFINE ? m[kStripW - 1] : f[kStripW - 1];
            pm = s == 0 ? c0f : inm;
        }
    }
}


// Per-warp shared memory of k_dp_wave: the lanes' strip tables (32 x
// tab_stride words: kTabWords, or kTabWords2 when pairs run), then rmax rows of
// traceback codes, 32 lanes wide (16 bits a lane for single segments, 32 for
// pairs: tb_bytes per lane-row).
__host__ __device__ constexpr uint32_t tab_stride(uint32_t tb_bytes) {
    return tb_bytes == 4u ? uint32_t(kTabWords2) : uint32_t(kTabWords);
}

// codes of one segment of a group: a 16-bit word per (row, strip), or one half
// of a pair's 32-bit word
struct SmemCodes {
    const uint16_t *tb;
    int base;
    __device__ __forceinline__ uint32_t tb_get(int32_t st, int32_t i) const {
        return tb[size_t(i - 1) * 32u + base + st];
    }
};
struct SmemCodesPair {
    const uint32_t *tb;
    int base, shift;
    __device__ __forceinline__ uint32_t tb_get(int32_t st, int32_t i) const {
        return (tb[size_t(i - 1) * 32u + base + st] >> shift) & 0xffffu;
    }
};

// Traceback of the group's segment.  When the ops fit in the group's strip
// tables in shared memory (free once the fill is done), every lane of the group
// walks a chunk of rows (dp_walk_span) from a guessed start; a start is right
// once it equals the end of the lane before, and each round makes at least one
// more lane right (mostly one round in all).  The verified chunks then write
// their ops at their offsets.  Otherwise lane s = 0 walks the whole path.  Then
// the segment's DpSum, its reference cells and its ops go out.
template <class Codes>
__device__ __forceinline__ void group_traceback(const DpLaunch &a, const Codes &sc,
                                                const SegView &v, bool active, uint32_t si,
                                                int G, int g, int s, uint32_t *stage,
                                                uint32_t stage_words) {
    const bool staged = a.stride <= stage_words;
    const bool chunk = pair_strips(a.chunk_mask, G);  // bit G of the mask
    int32_t n = 0;
    if (staged && !chunk) {
        if (active && s == 0) {
            OpsWriter w{stage, int32_t(a.stride * 16u)};
            n = dp_walk<kStripW>(v, sc, w);
            w.flush();
        }
        n = __shfl_sync(0xffffffffu, n, (g * G) & 31);
    } else if (staged) {
        if (active)
            for (uint32_t k = uint32_t(s); k < a.stride; k += uint32_t(G)) stage[k] = 0u;
        int32_t rtop = 0, rbot = 0, c = 0, e = 0, cnt = 0;
        if (active) {
            dp_chunk_rows(v.R, G, s, rtop, rbot);
            c = s == 0 ? v.C : dp_chunk_guess(v, rtop);
        }
        const uint32_t gbits = G >= 32 ? 0xffffffffu : (1u << G) - 1u;
        bool todo = active;
        for (int round = 0; round <= 32; round++) {  // at most G rounds
            if (todo) {
                int32_t jj = c;
                cnt = dp_walk_span<kStripW>(sc, rtop, jj, rbot);
                e = jj;
            }
            const int32_t pe = __shfl_up_sync(0xffffffffu, e, 1);
            const bool wrong = active && s > 0 && c != pe;
            const uint32_t gm = (__ballot_sync(0xffffffffu, wrong) >> (g * G)) & gbits;
            if (!__any_sync(0xffffffffu, gm != 0u)) break;
            // lanes from the first wrong one on start again where the lane
            // before them ended (right for the first wrong lane, whose
            // predecessor is right; a good guess for the rest)
            const int32_t f = gm ? __ffs(int(gm)) - 1 : G;
            todo = active && s >= f;
            if (todo) c = pe;
        }
        int32_t before = cnt;  // ops of the lanes before this one (exclusive scan)
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, before, d);
            if (s >= d) before += y;
        }
        n = __shfl_sync(0xffffffffu, before, (g * G + G - 1) & 31);  // the group's total
        before -= cnt;
        __syncwarp();  // stage zeroed
        if (active && cnt > 0) {
            struct Put {
                uint32_t *stage;
                int32_t p;
                int32_t q;
                uint32_t acc;
                __device__ __forceinline__ void operator()(uint32_t op) {
                    p--;
                    if ((p >> 4) != q) {
                        atomicOr(stage + q, acc);
                        acc = 0u;
                        q = p >> 4;
                    }
                    acc |= op << (2 * (p & 15));
                }
            };
            const int32_t p0 = int32_t(a.stride * 16u) - before;
            Put put{stage, p0, (p0 - 1) >> 4, 0u};
            dp_walk_span_ops<kStripW>(sc, dp_op_lut(v), rtop, c, rbot, put);
            atomicOr(stage + put.q, put.acc);
        }
    } else if (active && s == 0) {
        uint32_t *words = a.ops + uint64_t(si) * a.stride;
        OpsWriter w{words, int32_t(a.stride * 16u)};
        n = dp_walk<kStripW>(v, sc, w);
        w.flush();
    }
    __syncwarp();
    if (active && s == 0) {
        DpSum sum;
        ops_summary(staged ? stage : a.ops + uint64_t(si) * a.stride, a.stride * 16u - uint32_t(n),
                    uint32_t(n), sum);
        a.sums[si] = sum;
        if (a.cells) {
            const uint64_t cl = band_cells(v.R, v.C, v.band);
            a.cells[si] = uint32_t(cl > 0xffffffffull ? 0xffffffffull : cl);
        }
    }
    if (staged && active) {  // the group's lanes copy the ops out together
        uint32_t *out = a.ops + uint64_t(si) * a.stride;
        for (uint32_t k = ((a.stride * 16u - uint32_t(n)) >> 4) + uint32_t(s); k < a.stride;
             k += uint32_t(G))
            out[k] = stage[k];
    }
    __syncwarp();
}

__device__ __forceinline__ SegView seg_view(const DpLaunch &a, uint32_t si) {
    return dpseg_view(a.segs[si], a.scode, a.soff, a.slen, a.qcode, a.qoff);
}

// One task of single segments: group g (G lanes) takes the sorted segment
// first + g * step, if below end.
template <bool AFFINE>
__device__ __forceinline__ void task_single(const DpLaunch a, uint64_t first, uint64_t step,
                                         uint64_t end, int G, int lane, uint16_t *tb,
                                         uint32_t *tabs) {
    const int S = 32 / G, g = lane / G, s = lane % G;
    const bool active = g < S && first + uint64_t(g) * step < end;
    uint32_t si = 0;
    SegView v{};
    int32_t R = 0;
    if (active) {
        si = a.perm[first + uint64_t(g) * step];
        v = seg_view(a, si);
        R = v.R;
    }
    const int32_t Rw = warp_max(R);
    const int32_t j0 = s * kStripW;
    const bool full = !active || dp_strip_full(v, j0, kStripW);
    const int32_t wlast = active ? dp_strip_wlast(v, j0, kStripW) : -1;
    const bool wfull = __all_sync(0xffffffffu, full);
    const bool wleft = __any_sync(0xffffffffu, wlast >= 0);
    // whole-band fast path: every segment of the warp inside its band and all
    // with the same align-left column (the shape key makes it so)
    const int32_t wl = active ? dp_left_col<kStripW>(v) : -2;
    const int32_t wl0 = warp_max(wl);
    const bool whole =
        a.whole && __all_sync(0xffffffffu, !active || (dp_whole_band(v) && wl == wl0));
    const uint32_t TS = tab_stride(a.tb_bytes);
    int32_t *tab = reinterpret_cast<int32_t *>(tabs + size_t(lane) * TS);
    if (whole) {
        if (wl0 >= 0) {
            wave_whole<AFFINE, true>(v, active, R, Rw, G, s, lane, wl0, tb, tab);
        } else {
            wave_whole<AFFINE, false>(v, active, R, Rw, G, s, lane, -1, tb, tab);
        }
    } else if (wfull) {
        if (wleft) {
            wave_fill<AFFINE, true, true>(v, active, R, Rw, G, s, lane, wlast, tb);
        } else {
            wave_fill<AFFINE, true, false>(v, active, R, Rw, G, s, lane, wlast, tb);
        }
    } else {
        if (wleft) {
            wave_fill<AFFINE, false, true>(v, active, R, Rw, G, s, lane, wlast, tb);
        } else {
            wave_fill<AFFINE, false, false>(v, active, R, Rw, G, s, lane, wlast, tb);
        }
    }
    __syncwarp();
    group_traceback(a, SmemCodes{tb, g * G}, v, active, si, G, g, s,
                    tabs + size_t(g) * G * TS, uint32_t(G) * TS);
}

// ---------------------------------------------------------------------------
// Row bases staged by the bulk copy engine.  Before a pair task's fill, each
// group's leader lane copies the bases of its two segments' rows (contiguous
// bytes of one read each, forward or reversed) from global memory into shared
// memory with one cp.async.bulk each; the copies complete on the warp's
// mbarrier, whose phase the whole warp waits for.  The staging space is the
// rows of the warp's traceback-code area that the task leaves unused (rows
// Rw .. rmax - 1), so it costs no shared memory; a task without room, or a
// wait that runs out (bounded: it sets a counter and the rows are read from
// global memory as without staging), keeps the global row pointers.  Copies
// start on 16-byte boundaries and move whole 16-byte units: a span is widened
// to them (the code buffers hold 16 bytes past their last base).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
    uint64_t state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state)
                 : "r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    (void)state;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// global -> shared, `bytes` (a multiple of 16) from a 16-byte aligned source
// to a 16-byte aligned destination, completing on `bar`
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
constexpr uint32_t kStageSpins = 1u << 22;  // try_wait rounds before a staging wait gives up

// the 16-byte units covering rows 1..R of a segment: first unit's address, bytes
__device__ __forceinline__ void row_span(const SegView &v, uintptr_t &lo, uint32_t &bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(v.row_base);
    const uintptr_t b = a + uintptr_t(intptr_t(v.row_dir) * intptr_t(v.R - 1));
    const uintptr_t first = a < b ? a : b, last = a < b ? b : a;
    lo = first & ~uintptr_t(15);
    bytes = uint32_t(((last + 1 - lo) + 15) & ~uintptr_t(15));
}

struct StageState {
    uint64_t *bar;     // the warp's mbarrier
    uint32_t phase;    // parity of the barrier's next phase
    bool on;           // off after a wait ran out (its copy may still land)
    uint32_t staged;   // tasks staged by this warp
};

// Points va / vb (the fill's copies) at staged rows when the warp's copies fit
// in `room` bytes at `space`; every lane of the warp calls it.
__device__ __forceinline__ void stage_rows(const DpLaunch &a, SegView &va, SegView &vb, bool active,
                                           bool has_b, int G, int g, int s, int lane,
                                           uint8_t *space, uint32_t room, StageState &st) {
    if (!st.on) return;
    const bool lead = active && s == 0;
    uintptr_t loa = 0, lob = 0;
    uint32_t na = 0, nb = 0;
    if (lead && va.R > 0) {
        row_span(va, loa, na);
        if (has_b) row_span(vb, lob, nb);
    }
    // exclusive scan of the leaders' bytes: each group's place in the space
    const uint32_t need = na + nb;
    uint32_t incl = need;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0u || total > room) return;  // warp-uniform
    const uint32_t off = incl - need;
    if (lane == 0) mbar_expect(st.bar, total);
    __syncwarp();
    // the space was last read by this warp's generic loads; order those
    // before the copy engine's writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lead) {
        bulk_g2s(space + off, reinterpret_cast<const void *>(loa), na, st.bar);
        if (nb) bulk_g2s(space + off + na, reinterpret_cast<const void *>(lob), nb, st.bar);
    }
    bool done = false;
    for (uint32_t k = 0; k < kStageSpins && !done; k++) done = mbar_try_wait(st.bar, st.phase);
    done = __all_sync(0xffffffffu, done);
    if (!done) {  // keep the global rows; this warp stages no more
        st.on = false;
        if (lane == 0 && a.staged) atomicAdd(a.staged + 1, 1ull);
        return;
    }
    st.phase ^= 1u;
    st.staged++;
    // the group's rows in shared memory, at the same offsets from their units
    const int lead_lane = (g * G) & 31;
    const uint32_t goff = __shfl_sync(0xffffffffu, off, lead_lane);
    const uint32_t gna = __shfl_sync(0xffffffffu, na, lead_lane);
    const unsigned long long gloa = __shfl_sync(0xffffffffu, (unsigned long long)loa, lead_lane);
    const unsigned long long glob = __shfl_sync(0xffffffffu, (unsigned long long)lob, lead_lane);
    if (active && va.R > 0) {
        const uint8_t *ra = space + goff + (reinterpret_cast<uintptr_t>(va.row_base) - uintptr_t(gloa));
        const uint8_t *rb = has_b ? space + goff + gna + (reinterpret_cast<uintptr_t>(vb.row_base) - uintptr_t(glob))
                                  : ra;
        va.row_base = ra;
        vb.row_base = rb;
    }
}

// the wavefront over one warp's pairs of whole-band segments (dp_pair_row,
// tagged 16-bit halves): group lanes hold segment A in the low halves and B in
// the high halves
template <bool AFFINE, bool LEFT>
__device__ __noinline__ void wave_pair(const SegView va, const SegView vb, bool active, int32_t R,
                                       int32_t Rw, int G, int s, int lane, int32_t wl,
                                       uint32_t *tb, uint32_t *tab) {
    const int32_t j0 = s * kStripW;
    uint32_t f[kStripW], x[kStripW], m[kStripW];
    uint32_t pm = 0, c0f = 0, c0y = 0, mul = 0;
    const uint8_t *rpa = va.row_base, *rpb = vb.row_base;
    uint32_t cha = 0, chb = 0;
    if (active) {
        dp_pair_table<AFFINE, kStripW>(va, vb, j0, tab);
        dp_pair_init<AFFINE, kStripW>(va, vb, j0, f, x, m, pm);
        dp_pair_col0<AFFINE>(va, vb, c0f, c0y, mul);
        cha = (rpa[0] ^ va.row_xor) & 3u;
        chb = (rpb[0] ^ vb.row_xor) & 3u;
    }
    // column 0's clean M is its FM without the FM tag
    constexpr uint32_t c0tag = AFFINE ? 0x00010001u * uint32_t(PairTags<AFFINE>::diag) : 0u;
    const bool holds_c = LEFT && s == G - 1;
    const uint32_t pad = pack2s(kPairPad);
    uint32_t pf = pad, py = pad, pmv = pad;  // FM (global F), IY, M published to lane s+1
    uint32_t *tp = tb + lane;
    const uint16_t *sc16 = reinterpret_cast<const uint16_t *>(tab);
#pragma unroll 1
    for (int32_t t = 0; t < Rw + G - 1; t++) {
        const uint32_t inf = __shfl_up_sync(0xffffffffu, pf, 1);
        const uint32_t iny = AFFINE ? __shfl_up_sync(0xffffffffu, py, 1) : 0u;
        const uint32_t inm = AFFINE ? __shfl_up_sync(0xffffffffu, pmv, 1) : inf;
        const int32_t i = t - s + 1;
        if (active && uint32_t(i - 1) < uint32_t(R)) {
            const uint32_t ba = cha, bb = chb;
            if (i < R) {  // next row's bases, loaded a step early
                rpa += va.row_dir;
                rpb += vb.row_dir;
                cha = (rpa[0] ^ va.row_xor) & 3u;
                chb = (rpb[0] ^ vb.row_xor) & 3u;
            }
            uint32_t lf = s == 0 ? c0f : inf;
            uint32_t ly = s == 0 ? c0y : iny;
            const uint4 A = reinterpret_cast<const uint4 *>(sc16 + ba * kStripW)[0];
            const uint4 B = reinterpret_cast<const uint4 *>(sc16 + (4u + bb) * kStripW)[0];
            const uint32_t sc[kStripW] = {__byte_perm(A.x, B.x, 0x5410), __byte_perm(A.x, B.x, 0x7632),
                                          __byte_perm(A.y, B.y, 0x5410), __byte_perm(A.y, B.y, 0x7632),
                                          __byte_perm(A.z, B.z, 0x5410), __byte_perm(A.z, B.z, 0x7632),
                                          __byte_perm(A.w, B.w, 0x5410), __byte_perm(A.w, B.w, 0x7632)};
            if (LEFT) dp_pair_left<AFFINE, kStripW>(wl, holds_c, f, x);
            const uint32_t eq = tab[32 + ba] | tab[36 + bb];
            const uint32_t bits = dp_pair_row<AFFINE, kStripW>(sc, eq, f, x, m, lf, ly, pm);
            *tp = bits;
            tp += 32;
            pf = lf;
            py = ly;
            pmv = AFFINE ? m[kStripW - 1] : lf;
            pm = s == 0 ? c0f - c0tag : inm;
            c0f = add2(c0f, mul);
            c0y = add2(c0y, mul);
        }
    }
}

// One task of pairs: group g takes the sorted segments first + 2g (A, low
// halves) and first + 2g + 1 (B, high halves).  Warps whose pairs are not all
// whole-band (or too long for 16-bit scores) run their A segments, then their
// B segments, as two tasks of single segments.
template <bool AFFINE>
__device__ __forceinline__ void task_pair(const DpLaunch a, uint64_t first, uint64_t end, int G,
                                          int lane, uint32_t *tb, uint32_t *tabs, StageState &stg) {
    const int S = 32 / G, g = lane / G, s = lane % G;
    const uint64_t ia = first + 2u * uint64_t(g), ib = ia + 1u;
    const bool active = g < S && ia < end;
    const bool has_b = active && ib < end;
    uint32_t sa = 0, sb = 0;
    SegView va{}, vb{};
    int32_t R = 0;
    bool ok = true;
    int32_t wl = -2;
    if (active) {
        sa = a.perm[ia];
        va = seg_view(a, sa);
        sb = has_b ? a.perm[ib] : sa;
        vb = has_b ? seg_view(a, sb) : va;
        R = va.R;
        wl = dp_left_col<kStripW>(va);
        ok = dp_whole_band(va) && dp_whole_band(vb) && va.R == vb.R &&
             dp_left_col<kStripW>(vb) == wl && va.R + va.C <= kPairMaxSide &&
             vb.R + vb.C <= kPairMaxSide;
    }
    const int32_t wl0 = warp_max(wl);
    if (!(a.whole && __all_sync(0xffffffffu, !active || (ok && wl == wl0)))) {
        uint16_t *tb16 = reinterpret_cast<uint16_t *>(tb);
        task_single<AFFINE>(a, first, 2, end, G, lane, tb16, tabs);
        task_single<AFFINE>(a, first + 1, 2, end, G, lane, tb16, tabs);
        return;
    }
    const int32_t Rw = warp_max(R);
    const uint32_t TS = kTabWords2;
    uint32_t *tab = tabs + size_t(lane) * TS;
    // the fill reads its row bases through copies of the views, staged in the
    // code rows this task leaves free when they fit
    SegView fa = va, fb = vb;
    {
        uint8_t *space = reinterpret_cast<uint8_t *>(tb + size_t(Rw) * 32u);
        const uint32_t room = (a.rmax > Rw ? uint32_t(a.rmax - Rw) * 32u * 4u : 0u) + a.stage_extra;
        stage_rows(a, fa, fb, active, has_b, G, g, s, lane, space, room, stg);
    }
    if (wl0 >= 0) {
        wave_pair<AFFINE, true>(fa, fb, active, R, Rw, G, s, lane, wl0, tb, tab);
    } else {
        wave_pair<AFFINE, false>(fa, fb, active, R, Rw, G, s, lane, -1, tb, tab);
    }
    __syncwarp();
    if (a.pair_cells) {  // the cells this warp computed as pairs
        unsigned long long pc = 0;
        if (active && s == 0)
            pc = band_cells(va.R, va.C, va.band) + (has_b ? band_cells(vb.R, vb.C, vb.band) : 0ull);
        pc = warp_sum(pc);
        if (lane == 0 && pc) atomicAdd(a.pair_cells, pc);
    }
    uint32_t *stage = tabs + size_t(g) * G * TS;
    group_traceback(a, SmemCodesPair{tb, g * G, 0}, va, active, sa, G, g, s, stage,
                    uint32_t(G) * TS);
    group_traceback(a, SmemCodesPair{tb, g * G, 16}, vb, has_b, sb, G, g, s, stage,
                    uint32_t(G) * TS);
}

template <bool AFFINE, int WARPS, int TIER>
__global__ void __launch_bounds__(WARPS * 32, kWaveRegBlocks(WARPS, TIER))
    k_dp_wave(DpLaunch a, uint64_t *tasks) {
    extern __shared__ int4 wave_smem[];
    const int lane = int(threadIdx.x & 31u), wib = int(threadIdx.x >> 5);
    const uint32_t TS = tab_stride(a.tb_bytes);
    uint32_t *tabs = reinterpret_cast<uint32_t *>(wave_smem) + size_t(wib) * 32u * TS;
    // a warp's code area: rmax rows, then stage_extra bytes of staging space
    const size_t code_area = size_t(a.rmax) * 32u * a.tb_bytes + a.stage_extra;
    uint8_t *tbw = reinterpret_cast<uint8_t *>(wave_smem) + size_t(WARPS) * 32u * TS * 4u +
                   size_t(wib) * code_area;
    // the warps' mbarriers for staged rows: 16 bytes each, after every code area
    uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<uint8_t *>(wave_smem) +
                                                 size_t(WARPS) * 32u * TS * 4u +
                                                 size_t(WARPS) * code_area) +
                    2u * size_t(wib);
    StageState stg{bar, 0u, a.tb_bytes == 4u, 0u};  // pairs only (4-byte code rows)
    if (stg.on && lane == 0) mbar_init(bar);
    __syncwarp();
    // a persistent grid fed by a work queue: each warp takes the next task, the
    // largest shapes first (tasks are sorted by strips, then rows)
    const uint64_t ntask = tasks[33];
    for (;;) {
        unsigned long long q = 0;
        if (lane == 0) q = atomicAdd(reinterpret_cast<unsigned long long *>(tasks + kTaskQueue), 1ull);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= ntask) break;
        const uint64_t task = ntask - 1 - q;
        int G = 1;
        while (G < 32 && tasks[G + 1] <= task) G++;
        const bool pair = pair_strips(a.pair_mask, G);
        const uint64_t per = uint64_t(32 / G) * (pair ? 2u : 1u);  // segments per task
        const uint64_t first = tasks[34 + G] + (task - tasks[G]) * per;
        const uint64_t end = tasks[68 + G];
        if (pair) {
            task_pair<AFFINE>(a, first, end, G, lane, reinterpret_cast<uint32_t *>(tbw), tabs, stg);
        } else {
            task_single<AFFINE>(a, first, 1, end, G, lane, reinterpret_cast<uint16_t *>(tbw), tabs);
        }
    }
    if (a.tb_bytes == 4u) {
        if (!stg.on) {  // a copy whose wait ran out: give it its time before the block ends
            bool done = false;
            for (uint32_t k = 0; k < kStageSpins && !done; k++) done = mbar_try_wait(bar, stg.phase);
        }
        if (lane == 0 && a.staged && stg.staged) atomicAdd(a.staged, (unsigned long long)stg.staged);
    }
}

// per-thread kernel for the segments wider than 32 strips (after the wavefront ranges)
template <bool AFFINE>
__global__ void __launch_bounds__(kDpThreads) k_dp_wide(DpLaunch a, const uint64_t *tasks) {
    const uint64_t T = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    DevScratch sc{a.tb, a.bnd, T, a.rmax, t};
    for (uint64_t idx = tasks[0] + t; idx < a.nd; idx += T) {
        const uint32_t si = a.perm[idx];
        const DpSeg g = a.segs[si];
        const SegView v = dpseg_view(g, a.scode, a.soff, a.slen, a.qcode, a.qoff);
        dp_fill<kStripW, AFFINE>(v, sc);
        OpsWriter w{a.ops + uint64_t(si) * a.stride, int32_t(a.stride * 16u)};
        DpSum sum;
        dp_traceback<kStripW>(v, sc, w, sum);
        w.flush();
        a.sums[si] = sum;
        if (a.cells) {
            const uint64_t cl = band_cells(v.R, v.C, v.band);
            a.cells[si] = uint32_t(cl > 0xffffffffull ? 0xffffffffull : cl);
        }
    }
}

// ---------------------------------------------------------------------------
// records: AlignmentRecord scoring with getAlignment2's early exits
// ---------------------------------------------------------------------------
struct AsmVisitor {
    const DpSum *sums;
    const uint32_t *cells;
    RecState st;
    uint32_t used = 0;
    unsigned long long cells_used = 0;
    bool built = false;
    HERO_HD void begin(int64_t, int64_t, int64_t) { built = true; }
    HERO_HD void position(int64_t) {}
    HERO_HD void run(uint8_t t, int64_t c) { st.add(t, c); }
    HERO_HD void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        st.add_piece(sums[used]);
        if (cells) cells_used += cells[used];
        used++;
    }
    HERO_HD bool check(int64_t m, int64_t i) { return st.good_counts(m, i); }
    HERO_HD void finish() {}
};

struct KeyAt {
    const uint32_t *k;
    HERO_HD uint64_t operator()(int32_t i) const { return hit_pack(0, k[i] >> 16, k[i] & 0xffffu); }
};

__global__ void k_assemble(Params p, uint64_t nc, ChainArrays ch, const uint32_t *keys,
                           ReadsView subj, ReadsView q, const DpSum *sums, const uint32_t *cells,
                           unsigned long long *counters) {
    unsigned long long built = 0, acc = 0, used = 0, ncells = 0, nall = 0;
    for (uint64_t ci = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; ci < nc;
         ci += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t s = ch.subj[ci], qid = ch.query[ci];
        AsmVisitor v;
        v.sums = sums + ch.seg_off[ci];
        v.cells = cells ? cells + ch.seg_off[ci] : nullptr;
        KeyAt ka{keys + ch.key_off[ci]};
        const bool ok = walk_chain(p, int64_t(q.len[qid]), int64_t(subj.len[s]), ka,
                                   int32_t(ch.nkeys[ci]), v);
        uint8_t status = CH_NONE;
        double rate = 0, len = 0;
        if (v.built) {
            built++;
            status = CH_REJECTED;
            if (ok && v.st.good_rates(p, rate, len)) {
                status = CH_ACCEPTED;
                acc++;
            }
        }
        ch.status[ci] = status;
        ch.rate[ci] = rate;
        ch.len[ci] = len;
        used += v.used;
        ncells += v.cells_used;
        if (cells)
            for (uint32_t k = 0; k < ch.nseg[ci]; k++) nall += cells[ch.seg_off[ci] + k];
    }
    built = warp_sum(built);
    acc = warp_sum(acc);
    used = warp_sum(used);
    ncells = warp_sum(ncells);
    nall = warp_sum(nall);
    if (lane_id() == 0) {
        atomicAdd(&counters[C_BUILT], built);
        atomicAdd(&counters[C_ACCEPTED], acc);
        atomicAdd(&counters[C_DP_REF], used);
        atomicAdd(&counters[C_CELLS], ncells);
        atomicAdd(&counters[C_CELLS_ALL], nall);
    }
}

// SubjectRead::addAlignment (SubjectRead.cpp:25-79): one record per (subject,
// query); forward chains arrive before reverse-complement chains.
__global__ void k_dedupe(uint64_t nsub, const uint32_t *seg_chain_start,
                         const uint32_t *seg_chain_count, ChainArrays ch, uint32_t *winners,
                         unsigned long long *counters) {
    unsigned long long kept = 0;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nsub;
         s += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t i = seg_chain_start[2 * s], ie = i + seg_chain_count[2 * s];
        uint32_t j = seg_chain_start[2 * s + 1], je = j + seg_chain_count[2 * s + 1];
        while (i < ie || j < je) {
            const uint32_t qi = i < ie ? ch.query[i] : 0xffffffffu;
            const uint32_t qj = j < je ? ch.query[j] : 0xffffffffu;
            const uint32_t qq = qi < qj ? qi : qj;
            int64_t best = -1;
            auto consider = [&](uint32_t c) {
                if (ch.status[c] != CH_ACCEPTED) return;
                if (best < 0 || record_better(ch.rate[c], ch.len[c], ch.rate[best], ch.len[best]))
                    best = c;
            };
            while (i < ie && ch.query[i] == qq) consider(i++);
            while (j < je && ch.query[j] == qq) consider(j++);
            if (best >= 0) {
                ch.win[best] = 1;
                winners[atomicAdd(&counters[C_WIN], 1ull)] = uint32_t(best);
                kept++;
            }
        }
    }
    kept = warp_sum(kept);
    if (lane_id() == 0) atomicAdd(&counters[C_KEPT], kept);
}

// ---------------------------------------------------------------------------
// alignment output (HERO without -c): SubjectRead::addAlignment's list keyed by
// the query's uniqueId (list_add), then the batch's .aln text
// (SubjectReadAligner::writeToFile, SubjectRead::writeAlignment,
// AlignmentRecord::getCigar).  The text is cut into units -- per subject its
// header ">id\n", its records in list order and its closing "\n" -- that one
// kernel sizes, a scan places and another writes, one thread per unit.
// ---------------------------------------------------------------------------
// the list slots of a subject: its forward chains' range, then its reverse range
struct ChainSlots {
    uint32_t *a;
    uint32_t s0, n0, s1;
    __device__ __forceinline__ uint32_t slot(uint32_t i) const { return i < n0 ? s0 + i : s1 + (i - n0); }
    __device__ __forceinline__ uint32_t get(uint32_t i) const { return a[slot(i)]; }
    __device__ __forceinline__ void set(uint32_t i, uint32_t v) { a[slot(i)] = v; }
};

// one thread per subject: its accepted records in arrival order (forward
// chains, then reverse-complement chains, each in (query, chain) order)
__global__ void k_aln_list(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                           ChainArrays ch, ReadsView q, uint32_t *alist, uint32_t *alist_n,
                           unsigned long long *counters) {
    unsigned long long kept = 0;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nsub;
         s += uint64_t(gridDim.x) * blockDim.x) {
        ChainSlots L{alist, cstart[2 * s], ccount[2 * s], cstart[2 * s + 1]};
        auto key = [&](uint32_t c) { return uint64_t(q.uid[ch.query[c]]); };
        auto better = [&](uint32_t a, uint32_t b) {
            return record_better(ch.rate[a], ch.len[a], ch.rate[b], ch.len[b]);
        };
        uint32_t n = 0;
        uint64_t largest = 0;
        for (int o = 0; o < 2; o++) {
            const uint32_t b = cstart[2 * s + o], e = b + ccount[2 * s + o];
            for (uint32_t c = b; c < e; c++)
                if (ch.status[c] == CH_ACCEPTED) n = list_add(L, n, largest, c, key, better);
        }
        alist_n[s] = n;
        kept += n;
    }
    kept = warp_sum(kept);
    if (lane_id() == 0) atomicAdd(&counters[C_KEPT], kept);
}

// --mapping, one thread per subject (SubjectReadAligner.cpp:556-561): its
// accepted records in arrival order kept as SubjectRead::addAlignment keeps
// them in consensus mode (keyed by the query's inner id, list_add), then
// chooseQueryWithBestAlignment (SubjectRead.cpp:463-500, map_choose) picks the
// records that vote; they become the batch's winners for k_vote.
__global__ void k_map_choose(Params p, uint64_t nsub, const uint32_t *cstart,
                             const uint32_t *ccount, ChainArrays ch, const uint32_t *keys,
                             ReadsView subj, ReadsView q, const DpSum *sums, uint32_t *alist,
                             uint32_t *winners, unsigned long long *counters) {
    unsigned long long kept = 0;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nsub;
         s += uint64_t(gridDim.x) * blockDim.x) {
        ChainSlots L{alist, cstart[2 * s], ccount[2 * s], cstart[2 * s + 1]};
        auto key = [&](uint32_t c) { return uint64_t(ch.query[c]); };
        auto better = [&](uint32_t a, uint32_t b) {
            return record_better(ch.rate[a], ch.len[a], ch.rate[b], ch.len[b]);
        };
        uint32_t n = 0;
        uint64_t largest = 0;
        for (int o = 0; o < 2; o++) {
            const uint32_t b = cstart[2 * s + o], e = b + ccount[2 * s + o];
            for (uint32_t c = b; c < e; c++)
                if (ch.status[c] == CH_ACCEPTED) n = list_add(L, n, largest, c, key, better);
        }
        const int64_t Ls = subj.len[s];
        // one walk per listed record: map_choose asks covers(i), then subs(i)
        int64_t walked = -1;
        bool cov = false;
        int64_t sub = 0;
        auto walk = [&](uint32_t i) {
            if (int64_t(i) == walked) return;
            const uint32_t c = L.get(i);
            const DpSum *sm = sums + ch.seg_off[c];
            auto piece = [sm](uint32_t k) { return sm[k]; };
            CoverWalk<decltype(piece)> w{piece};
            walk_chain(p, int64_t(q.len[ch.query[c]]), Ls, KeyAt{keys + ch.key_off[c]},
                       int32_t(ch.nkeys[c]), w);
            cov = w.covers(Ls);
            sub = w.subs;
            walked = int64_t(i);
        };
        auto covers = [&](uint32_t i) {
            walk(i);
            return cov;
        };
        auto subs = [&](uint32_t i) {
            walk(i);
            return sub;
        };
        uint32_t n_keep = 0;
        const int32_t best = map_choose(n, Ls, covers, subs, &n_keep);
        for (uint32_t i = 0; i < n_keep; i++) {
            const uint32_t c = L.get(n_keep == 1 && best >= 0 ? uint32_t(best) : i);
            ch.win[c] = 1;
            winners[atomicAdd(&counters[C_WIN], 1ull)] = c;
        }
        kept += n_keep;
    }
    kept = warp_sum(kept);
    if (lane_id() == 0) atomicAdd(&counters[C_KEPT], kept);
}

// --mapping: QueryDataset::getCoverageAndWriteResults (QueryDataset.cpp:560-599)
// -- per query base the sum of its four vote counts (no self vote), counted
// into hist[min(sum, bins - 1)]; the largest sum goes to *maxc.  One warp per read.
__global__ void k_map_hist(ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint64_t bins,
                           unsigned long long *hist, unsigned long long *maxc) {
    const uint32_t lane = lane_id();
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    unsigned long long mx = 0;
    for (uint64_t r = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < q.n;
         r += warps) {
        const uint64_t b = q.off[r];
        const uint32_t Lr = q.len[r];
        int32_t carry = 0;  // match-run votes entering the current chunk
        for (uint32_t c0 = 0; c0 < Lr; c0 += 32) {
            const uint32_t i = c0 + lane;
            const int32_t d = i < Lr ? mdiff[b + i] : 0;
            int32_t tot;
            const int32_t run = carry + warp_exclusive<int32_t>(d, &tot) + d;
            carry += tot;
            if (i < Lr) {
                const uint64_t sum = uint64_t(cov[(b + i) * 4]) + cov[(b + i) * 4 + 1] +
                                     cov[(b + i) * 4 + 2] + cov[(b + i) * 4 + 3] + uint64_t(run);
                atomicAdd(&hist[sum < bins ? sum : bins - 1], 1ull);
                mx = sum > mx ? sum : mx;
            }
        }
    }
    mx = warp_max(mx);
    if (lane == 0) atomicMax(maxc, mx);
}

// one thread per subject: its units (rec_off = exclusive scan of alist_n)
__global__ void k_aln_units(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                            const uint32_t *alist, const uint32_t *alist_n,
                            const uint64_t *rec_off, ReadsView subj, uint32_t *unit,
                            uint32_t *ulen) {
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nsub;
         s += uint64_t(gridDim.x) * blockDim.x) {
        const ChainSlots L{const_cast<uint32_t *>(alist), cstart[2 * s], ccount[2 * s],
                           cstart[2 * s + 1]};
        const uint64_t u0 = rec_off[s] + 2 * s;
        const uint32_t n = alist_n[s];
        unit[u0] = kUnitSubject | uint32_t(s);
        ulen[u0] = 2u + dec_len_signed(subj.uid[s]);
        for (uint32_t i = 0; i < n; i++) unit[u0 + 1 + i] = L.get(i);
        unit[u0 + 1 + n] = kUnitEnd;
        ulen[u0 + 1 + n] = 1u;
    }
}

// the DP pieces of a chain: ops of segment seg0 + piece, packed 2 bits a step at
// the end of the segment's stride words
struct DevPieces {
    const uint32_t *ops;
    uint32_t stride;
    const DpSum *sums;
    uint32_t seg0;
    template <class F>
    __device__ void each(uint32_t piece, F f) const {
        const uint32_t si = seg0 + piece;
        const DpSum sm = sums[si];
        const uint32_t P = uint32_t(sm.tot[0]) + sm.tot[1] + sm.tot[2] + sm.tot[3];
        const uint32_t *w = ops + uint64_t(si) * stride;
        const uint32_t end = stride * 16u;
        for (uint32_t pos = end - P; pos < end; pos++) f(uint8_t((w[pos >> 4] >> (2 * (pos & 15u))) & 3u));
    }
};

struct AlnRec {
    AlnText<DevPieces> t;
    KeyAt ka;
    int32_t nkeys;
    int64_t Ls;
    uint64_t key;
    uint32_t orient;
};

__device__ __forceinline__ AlnRec aln_rec(uint32_t c, ChainArrays ch, const uint32_t *keys,
                                          ReadsView subj, ReadsView q, const uint32_t *ops,
                                          uint32_t stride, const DpSum *sums) {
    const uint32_t s = ch.subj[c], qid = ch.query[c];
    AlnRec r{AlnText<DevPieces>{DevPieces{ops, stride, sums, ch.seg_off[c]}, q.code + q.off[qid],
                                int32_t(q.len[qid]), ch.orient[c] != 0},
             KeyAt{keys + ch.key_off[c]}, int32_t(ch.nkeys[c]), int64_t(subj.len[s]),
             uint64_t(q.uid[qid]), uint32_t(ch.orient[c])};
    return r;
}

// one thread per unit: text length of each record (and of its prefix and CIGAR)
__global__ void k_aln_size(Params p, uint64_t nunit, const uint32_t *unit, ChainArrays ch,
                           const uint32_t *keys, ReadsView subj, ReadsView q, const uint32_t *ops,
                           uint32_t stride, const DpSum *sums, uint32_t *ulen, uint32_t *upre,
                           uint32_t *ucig) {
    for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < nunit;
         u += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = unit[u];
        if (c & kUnitSubject) continue;
        AlnRec r = aln_rec(c, ch, keys, subj, q, ops, stride, sums);
        walk_chain(p, int64_t(r.t.Lq), r.Ls, r.ka, r.nkeys, r.t);
        const uint32_t pre = aln_prefix_len(r.key, r.orient, r.t.pos);
        upre[u] = pre;
        ucig[u] = r.t.cig_len;
        ulen[u] = pre + r.t.cig_len + 1u + r.t.ins_len + 1u;
    }
}

// one thread per unit: the text at its offset
__global__ void k_aln_write(Params p, uint64_t nunit, const uint32_t *unit, const uint64_t *uoff,
                            ChainArrays ch, const uint32_t *keys, ReadsView subj, ReadsView q,
                            const uint32_t *ops, uint32_t stride, const DpSum *sums,
                            const uint32_t *upre, const uint32_t *ucig, char *text) {
    for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < nunit;
         u += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = unit[u];
        char *o = text + uoff[u];
        if (c == kUnitEnd) {
            *o = '\n';
            continue;
        }
        if (c & kUnitSubject) {
            *o++ = '>';
            o = dec_put_signed(o, subj.uid[c & ~kUnitSubject]);
            *o = '\n';
            continue;
        }
        AlnRec r = aln_rec(c, ch, keys, subj, q, ops, stride, sums);
        r.t.cig = o + upre[u];
        r.t.ins = r.t.cig + ucig[u] + 1;
        walk_chain(p, int64_t(r.t.Lq), r.Ls, r.ka, r.nkeys, r.t);
        o = dec_put(o, r.key);
        *o++ = ',';
        o = dec_put(o, r.orient);
        *o++ = ',';
        o = dec_put_signed(o, r.t.pos);
        *o = ',';
        *r.t.cig = ',';
        *r.t.ins = ',';
    }
}

// SubjectRead::updateQueryCoverage (SubjectRead.cpp:208-330): M votes the
// query's own base, a mismatch votes the subject base, I/D only move.  Runs of
// M are kept open across pieces and land as two difference-array updates.
struct VoteVisitor {
    const uint8_t *sc;  // subject codes (forward)
    int32_t Ls, orient;
    int32_t Lq;
    uint32_t *cov;      // query's rows of the mismatch-vote matrix
    int32_t *md;        // query's match-run difference array
    const uint32_t *ops;
    uint32_t stride;
    const DpSum *sums;
    uint32_t seg;       // segment index of the next DP piece
    int64_t ps = 0, pq = 0;
    int64_t open = -1;  // start of the open match run
    unsigned long long anomalies = 0;

    __device__ __forceinline__ uint8_t subj_code(int64_t i) const {
        return orient ? uint8_t(sc[Ls - 1 - i] ^ 2u) : sc[i];
    }
    __device__ __forceinline__ void close() {
        if (open < 0) return;
        int64_t e = pq;
        if (e > Lq) {  // match votes past the read (the reference reads out of range)
            anomalies += uint64_t(e - (open > Lq ? open : Lq));
            e = Lq;
        }
        if (open < e) {
            atomicAdd(&md[open], 1);
            if (e < Lq) atomicAdd(&md[e], -1);
        }
        open = -1;
    }
    __device__ __forceinline__ void match(int64_t c) {
        if (open < 0) open = pq;
        pq += c;
        ps += c;
    }
    __device__ __forceinline__ void mismatch() {
        close();
        const uint8_t code = (ps >= 0 && ps < Ls) ? subj_code(ps) : uint8_t(kBad);
        if (pq < 0 || pq >= Lq || code >= 4) {
            anomalies++;
        } else {
            atomicAdd(&cov[pq * 4 + code], 1u);
        }
        pq++;
        ps++;
    }
    __device__ void begin(int64_t, int64_t, int64_t) {}
    __device__ void position(int64_t p) {
        ps = p;
        pq = 0;
    }
    __device__ void run(uint8_t t, int64_t c) {
        if (t == OP_M) {
            match(c);
        } else {
            close();
            if (t == OP_I) {
                pq += c;
            } else {
                ps += c;
            }
        }
    }
    __device__ void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        const DpSum s = sums[seg];
        const uint32_t P = uint32_t(s.tot[0]) + s.tot[1] + s.tot[2] + s.tot[3];
        if (s.tot[OP_M] == P) {  // one match run
            match(P);
        } else {
            // ops a word (16) at a time: match stretches advance at once, the
            // other ops are found by their non-zero 2-bit fields (OP_M is 0)
            const uint32_t *w = ops + uint64_t(seg) * stride;
            const uint32_t end = stride * 16u;
            for (uint32_t pos = end - P; pos < end;) {
                const uint32_t f0 = pos & 15u, nf = 16u - f0;  // fields left in this word
                const uint32_t word = w[pos >> 4] >> (2 * f0);
                uint32_t nm = (word | (word >> 1)) & 0x55555555u;
                uint32_t done = 0;
                while (nm) {
                    const uint32_t b = uint32_t(__ffs(int(nm))) - 1u, fi = b >> 1;
                    if (fi > done) match(int64_t(fi - done));
                    const uint32_t op = (word >> b) & 3u;
                    if (op == OP_X) {
                        mismatch();
                    } else {
                        close();
                        if (op == OP_I) {
                            pq++;
                        } else {
                            ps++;
                        }
                    }
                    done = fi + 1u;
                    nm &= nm - 1u;
                }
                if (nf > done) match(int64_t(nf - done));
                pos += nf;
            }
        }
        seg++;
    }
    __device__ bool check(int64_t, int64_t) { return true; }
    __device__ void finish() { close(); }
};

// Winners sorted by chain shape (DP pieces, keys) before the votes: a warp then
// walks chains of one shape, and its lanes stay together (a counting sort over
// kWinBins shapes; order inside a shape is free, votes commute).
constexpr uint32_t kWinBins = 512;

__device__ __forceinline__ uint32_t win_key(const ChainArrays &ch, uint32_t c) {
    const uint32_t ns = ch.nseg[c], nk = ch.nkeys[c];
    return ((ns < 31u ? ns : 31u) << 4) | (nk < 15u ? nk : 15u);
}

__global__ void k_win_hist(const unsigned long long *counters, ChainArrays ch,
                           const uint32_t *winners, uint32_t *bins) {
    __shared__ uint32_t h[kWinBins];
    for (uint32_t i = threadIdx.x; i < kWinBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint64_t nw = counters[C_WIN];
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nw;
         i += uint64_t(gridDim.x) * blockDim.x)
        atomicAdd(&h[win_key(ch, winners[i])], 1u);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kWinBins; i += blockDim.x)
        if (h[i]) atomicAdd(&bins[i], h[i]);
}

// bins -> first slot of each shape (exclusive scan); cursors start at zero
__global__ void k_win_offsets(const uint32_t *bins, uint32_t *off, uint32_t *cursor) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t i = 0; i < kWinBins; i++) {
            off[i] = t;
            t += bins[i];
            cursor[i] = 0;
        }
    }
}

__global__ void k_win_scatter(const unsigned long long *counters, ChainArrays ch,
                              const uint32_t *winners, const uint32_t *off, uint32_t *cursor,
                              uint32_t *sorted) {
    const uint32_t lane = lane_id();
    const uint64_t nw = counters[C_WIN];
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) & ~uint64_t(31); b < nw;
         b += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = b + lane;
        const uint32_t w = i < nw ? winners[i] : 0u;
        const uint32_t key = i < nw ? win_key(ch, w) : 0xffffffffu;
        const uint32_t same = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = uint32_t(__ffs(int(same))) - 1u;
        uint32_t base = 0;
        if (i < nw && lane == leader) base = atomicAdd(&cursor[key], uint32_t(__popc(same)));
        base = __shfl_sync(0xffffffffu, base, int(leader));
        if (i < nw) sorted[off[key] + base + __popc(same & ((1u << lane) - 1u))] = w;
    }
}

__global__ void k_vote(Params p, const unsigned long long *counters_in, ChainArrays ch,
                       const uint32_t *winners, const uint32_t *keys, ReadsView subj, ReadsView q,
                       const uint32_t *ops, uint32_t stride, const DpSum *sums, uint32_t *cov,
                       int32_t *mdiff, unsigned long long *counters) {
    unsigned long long anomalies = 0;
    const uint64_t nw = counters_in[C_WIN];
    for (uint64_t wi = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; wi < nw;
         wi += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t ci = winners[wi];
        const uint32_t s = ch.subj[ci], qid = ch.query[ci];
        VoteVisitor v;
        v.sc = subj.code + subj.off[s];
        v.Ls = int32_t(subj.len[s]);
        v.orient = ch.orient[ci];
        v.Lq = int32_t(q.len[qid]);
        v.cov = cov + q.off[qid] * 4;
        v.md = mdiff + q.off[qid];
        v.ops = ops;
        v.stride = stride;
        v.sums = sums;
        v.seg = ch.seg_off[ci];
        KeyAt ka{keys + ch.key_off[ci]};
        walk_chain(p, v.Lq, v.Ls, ka, int32_t(ch.nkeys[ci]), v);
        anomalies += v.anomalies;
    }
    anomalies = warp_sum(anomalies);
    if (lane_id() == 0 && anomalies) atomicAdd(&counters[C_ANOMALY], anomalies);
}

// --merge: per kept record, the subject bases past its end voted into the
// query's overhang matrix (SubjectRead::updateQueryCoverageConsiderMerging,
// SubjectRead.cpp:332-462; QueryRead::updateExtraCoverageMatrix,
// QueryRead.cpp:352-369).  A second, light walk of each winner (positions and
// DP totals only); k_vote is unchanged.
__global__ void k_vote_overhang(Params p, const unsigned long long *counters_in, ChainArrays ch,
                                const uint32_t *winners, const uint32_t *keys, ReadsView subj,
                                ReadsView q, const DpSum *sums, uint32_t *ext) {
    const uint64_t nw = counters_in[C_WIN];
    for (uint64_t wi = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; wi < nw;
         wi += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t ci = winners[wi];
        const uint32_t s = ch.subj[ci], qid = ch.query[ci];
        const DpSum *sm = sums + ch.seg_off[ci];
        auto piece = [sm](uint32_t i) { return sm[i]; };
        OverhangWalk<decltype(piece)> w{piece};
        const int64_t Ls = subj.len[s];
        walk_chain(p, int64_t(q.len[qid]), Ls, KeyAt{keys + ch.key_off[ci]}, int32_t(ch.nkeys[ci]), w);
        if (!w.other) continue;
        const uint8_t *sc = subj.code + subj.off[s];
        const bool rc = ch.orient[ci] != 0;
        uint32_t *m = ext + uint64_t(qid) * (kOverhang * 4);
        for (int64_t i = 0; i < kOverhang && w.ps + i < Ls; i++) {
            const int64_t x = w.ps + i;
            const uint8_t code = rc ? uint8_t(sc[Ls - 1 - x] ^ 2u) : sc[x];
            if (code < 4) atomicAdd(&m[i * 4 + code], 1u);
        }
    }
}

// --merge after the consensus: QueryDataset::mergePairedReads (QueryDataset.cpp:
// 539-558) -> merge_pair on reads (2p, 2p+1), one thread per pair; the merged
// read is written from the pair's first base in `merged` (a copy of the
// corrected reads), its length to merged_len[p] (0: not merged)
__global__ void k_merge_pairs(uint64_t npairs, const uint64_t *off, const uint8_t *corrected,
                              const uint32_t *ext, uint8_t *merged, uint32_t *merged_len) {
    for (uint64_t pr = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; pr < npairs;
         pr += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t a = off[2 * pr], b = off[2 * pr + 1], e = off[2 * pr + 2];
        merged_len[pr] = merge_pair(reinterpret_cast<const char *>(corrected + a), int(b - a),
                                    reinterpret_cast<const char *>(corrected + b), int(e - b),
                                    ext + 2 * pr * (kOverhang * 4),
                                    ext + (2 * pr + 1) * (kOverhang * 4),
                                    reinterpret_cast<char *>(merged + a));
    }
}

// ---------------------------------------------------------------------------
// consensus: QueryRead::callConsensus + calculateCoverageStatistic
// (QueryRead.cpp:148-212); one warp per query read
// ---------------------------------------------------------------------------
constexpr uint32_t kConsWarps = 8, kConsSmem = 1024;  // column sums of reads up to 1024 bases

__global__ void __launch_bounds__(kConsWarps * 32)
    k_consensus(Params p, ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint8_t *out,
                uint32_t *colsum, uint32_t *imin, uint32_t *imed, uint32_t *imax, double *mis) {
    __shared__ uint32_t sums[kConsWarps][kConsSmem];
    const uint32_t lane = lane_id();
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t r = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < q.n;
         r += warps) {
        if (!q.good[r]) {
            if (lane == 0) {
                imin[r] = 0;
                imed[r] = 0;
                imax[r] = 0;
                mis[r] = 0;
            }
            continue;
        }
        const uint64_t b = q.off[r];
        const uint32_t L = q.len[r];
        // the read's column sums, in shared memory when they fit
        uint32_t *cs = L <= kConsSmem ? sums[threadIdx.x >> 5] : colsum + b;
        uint32_t changed = 0, mn = 0xffffffffu, mx = 0;
        int32_t carry = 0;  // match-run coverage entering the current chunk
        for (uint32_t c0 = 0; c0 < L; c0 += 32) {
            const uint32_t i = c0 + lane;
            const int32_t d = i < L ? mdiff[b + i] : 0;
            int32_t tot;
            const int32_t run = carry + warp_exclusive<int32_t>(d, &tot) + d;
            carry += tot;
            if (i < L) {
                const uint8_t own = q.code[b + i];
                uint32_t c[4];
                for (int j = 0; j < 4; j++) c[j] = cov[(b + i) * 4 + j];
                c[own] += uint32_t(run) + 1u;  // match votes + the read's own vote
                const int32_t id = column_consensus(c, p.thr);
                uint8_t nb = own;
                if (id >= 0) {
                    if (uint8_t(id) != own) changed++;
                    nb = uint8_t(id);
                }
                out[b + i] = uint8_t(code_base(nb));
                const uint32_t sm = c[0] + c[1] + c[2] + c[3];
                cs[i] = sm;
                mn = sm < mn ? sm : mn;
                mx = sm > mx ? sm : mx;
            }
        }
        changed = warp_sum(changed);
        mn = warp_min(mn);
        mx = warp_max(mx);
        __syncwarp();
        // median of the column sums (QueryRead.cpp:204-211: the sorted sums'
        // middle one, or the mean of the middle two): the p-th smallest value by
        // a binary search over [mn, mx] -- the smallest v with more than p sums
        // at or below it, each count one pass over the sums and a warp sum
        const uint32_t p_hi = L / 2, p_lo = (L % 2 == 0) ? L / 2 - 1 : (L - 1) / 2;
        auto count_le = [&](uint32_t v) {
            uint32_t c = 0;
            for (uint32_t i = lane; i < L; i += 32) c += cs[i] <= v;
            return warp_sum(c);
        };
        auto select = [&](uint32_t p, uint32_t lo, uint32_t hi) {
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (count_le(mid) > p) {
                    hi = mid;
                } else {
                    lo = mid + 1;
                }
            }
            return lo;
        };
        const uint32_t v_lo = select(p_lo, mn, mx);
        const uint32_t v_hi = (p_hi == p_lo || count_le(v_lo) > p_hi) ? v_lo : select(p_hi, v_lo, mx);
        if (lane == 0) {
            imin[r] = mn;
            imax[r] = mx;
            imed[r] = (L % 2 == 0) ? (v_hi + v_lo) / 2u : v_lo;
            mis[r] = __ddiv_rn(double(changed), double(L));
        }
    }
}

__global__ void k_expand_votes(ReadsView q, const uint32_t *cov, const int32_t *mdiff,
                               uint32_t *out) {
    const uint32_t lane = lane_id();
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t r = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < q.n;
         r += warps) {
        const uint64_t b = q.off[r];
        const uint32_t L = q.len[r];
        int32_t carry = 0;
        for (uint32_t c0 = 0; c0 < L; c0 += 32) {
            const uint32_t i = c0 + lane;
            const int32_t d = i < L ? mdiff[b + i] : 0;
            int32_t tot;
            const int32_t run = carry + warp_exclusive<int32_t>(d, &tot) + d;
            carry += tot;
            if (i < L) {
                const uint8_t own = q.code[b + i];
                for (int j = 0; j < 4; j++) {
                    uint32_t v = cov[(b + i) * 4 + j];
                    if (j == own) v += uint32_t(run);
                    out[(b + i) * 4 + j] = v;
                }
            }
        }
    }
}

// device timestamp (ns) for timing kernels inside a replayed graph
__global__ void k_stamp(unsigned long long *out) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *out = t;
}

// order-independent 64-bit fingerprint of a read set (bytes, offsets, ids)
__global__ void k_fingerprint(const uint8_t *raw, uint64_t nb, const uint64_t *off,
                              const int64_t *uid, uint64_t n, unsigned long long *out) {
    unsigned long long h = 0;
    const uint64_t T = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (uint64_t w = t0; w * 8 < nb; w += T) {
        uint64_t x = 0;
        for (int b = 0; b < 8 && w * 8 + b < nb; b++) x |= uint64_t(raw[w * 8 + b]) << (8 * b);
        h += mix64(x ^ (w * 0x9e3779b97f4a7c15ull));
    }
    for (uint64_t i = t0; i < n; i += T) {
        h += mix64(off[i + 1] ^ 0x5bd1e995ull ^ (i << 20));
        h += mix64(uint64_t(uid[i]) ^ 0xc2b2ae3d27d4eb4full ^ (i << 1));
    }
    h = warp_sum(h);
    if (lane_id() == 0) atomicAdd(out, h);
}

__global__ void k_unpack_ops(const uint32_t *ops, uint32_t stride, const DpSum *sums, uint64_t nd,
                             const uint64_t *out_off, uint8_t *out, int32_t *nops) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nd;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const DpSum s = sums[i];
        const uint32_t P = uint32_t(s.tot[0]) + s.tot[1] + s.tot[2] + s.tot[3];
        const uint32_t *w = ops + i * stride;
        const uint32_t first = stride * 16u - P;
        const uint64_t cap = out_off[i + 1] - out_off[i];
        for (uint32_t t = 0; t < P && t < cap; t++) {
            const uint32_t pos = first + t;
            out[out_off[i] + t] = uint8_t((w[pos >> 4] >> (2 * (pos & 15))) & 3u);
        }
        nops[i] = int32_t(P);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_prep_reads(const uint8_t *raw, uint64_t nbases, uint8_t *code, const uint64_t *off,
                       uint64_t n, uint32_t *len, uint8_t *good_query, uint8_t *good_subject,
                       double *gc, int32_t l, cudaStream_t st) {
    if (nbases) {
        counted();
        k_codes<<<grid_1d(nbases, 256), 256, 0, st>>>(raw, nbases, code);
    }
    if (n) {
        counted();
        k_read_flags<<<grid_1d(n, 128), 128, 0, st>>>(code, off, n, len, good_query, good_subject, gc, l);
    }
}

size_t scan_tmp_bytes(uint64_t n) { return scan_levels_bytes(n); }

uint64_t kernel_launches() { return g_launches.load(std::memory_order_relaxed); }

void launch_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, void *tmp, cudaStream_t st) {
    scan_rec<uint32_t>(in, out, n, reinterpret_cast<uint64_t *>(tmp), st);
}

void launch_key_count(ReadsView q, int32_t k, uint32_t *count, cudaStream_t st) {
    if (q.n) {
        counted();
        k_key_count<<<grid_1d(q.n, 256), 256, 0, st>>>(q, k, count);
    }
}
void launch_key_emit(ReadsView q, int32_t k, const uint64_t *key_off, uint64_t *klo,
                     uint64_t *khi, uint64_t *kval, cudaStream_t st) {
    if (q.n) {
        counted();
        k_key_emit<<<grid_1d(q.n, 128), 128, 0, st>>>(q, k, key_off, klo, khi, kval);
    }
}
void launch_table_insert(const uint64_t *klo, const uint64_t *khi, uint64_t nkeys,
                         uint32_t *owner, uint32_t *count, uint32_t *slot_of, uint64_t mask,
                         cudaStream_t st) {
    if (nkeys) {
        counted();
        k_table_insert<<<grid_1d(nkeys, 256), 256, 0, st>>>(klo, khi, nkeys, owner, count, slot_of, mask);
    }
}
void launch_table_fill(const uint64_t *kval, uint64_t nkeys, const uint32_t *slot_of,
                       const uint64_t *start, uint32_t *fill, uint64_t *vals, cudaStream_t st) {
    if (nkeys) {
        counted();
        k_table_fill<<<grid_1d(nkeys, 256), 256, 0, st>>>(kval, nkeys, slot_of, start, fill, vals);
    }
}
void launch_table_finalize(const uint64_t *klo, const uint64_t *khi, const uint32_t *owner,
                           const uint32_t *count, const uint64_t *start, uint64_t nslots,
                           Slot *slots, cudaStream_t st) {
    counted();
    k_table_finalize<<<grid_1d(nslots, 256), 256, 0, st>>>(klo, khi, owner, count, start, nslots, slots);
}

void launch_probe(bool emit, bool aln, ReadsView subj, uint64_t nsub, ReadsView q, TableView t, int32_t k,
                  uint2 *wcache, uint32_t *seg_hits, const uint64_t *hit_off, uint64_t *hits,
                  unsigned long long *counters, cudaStream_t st) {
    if (!nsub) return;
    const unsigned g = grid_1d(nsub, kProbeWarps, 148u * 16u);
    counted();
    if (emit) {
        k_probe_emit<<<g, kProbeWarps * 32, 0, st>>>(subj, nsub, q, t, k, aln, wcache, hit_off, hits);
    } else {
        k_probe_count<<<g, kProbeWarps * 32, 0, st>>>(subj, nsub, q, t, k, wcache, seg_hits, counters);
    }
}

void launch_sort_hits(uint64_t nseg, const uint64_t *hit_off, uint64_t *hits, cudaStream_t st) {
    if (!nseg) return;
    const unsigned g = unsigned(nseg < 148u * 16u ? nseg : 148u * 16u);
    counted();
    k_sort_hits_warp<<<grid_1d(nseg, kSortThreads / 32, 148u * 8u), kSortThreads, 0, st>>>(
        nseg, hit_off, hits);
    counted();
    k_sort_hits<<<g, kSortThreads, 0, st>>>(nseg, hit_off, hits);
}

void launch_chain(const Params &p, uint64_t nseg, ReadsView subj, ReadsView q,
                  const uint64_t *hit_off, const uint64_t *hits, ChainScratch sc,
                  uint32_t *seg_chain_start, uint32_t *seg_chain_count, ChainArrays ch,
                  uint32_t *keys, DpSeg *segs, uint64_t cap_chains, uint64_t cap_keys,
                  uint64_t cap_segs, unsigned long long *counters, cudaStream_t st) {
    if (!nseg) return;
    counted();
    k_chain<<<grid_1d(nseg, 8, 148u * 16u), 256, 0, st>>>(p, nseg, subj, q, hit_off, hits, sc,
                                                        seg_chain_start, seg_chain_count, ch, keys,
                                                        segs, cap_chains, cap_keys, cap_segs,
                                                        counters);
}

void launch_dp_sort(const DpSeg *segs, uint64_t nd, uint32_t *bins, uint32_t *perm,
                    uint64_t *bin_off, void *scan_tmp, cudaStream_t st) {
    cudaMemsetAsync(bins, 0, sizeof(uint32_t) * kDpBins, st);
    if (!nd) return;
    counted();
    k_dp_hist<<<grid_1d(nd, 256), 256, 0, st>>>(segs, nd, bins);
    launch_scan_u32(bins, bin_off, kDpBins, scan_tmp, st);
    cudaMemsetAsync(bins, 0, sizeof(uint32_t) * kDpBins, st);
    counted();
    k_dp_scatter<<<grid_1d(nd, 256), 256, 0, st>>>(segs, nd, bins, bin_off, perm);
}

uint64_t dp_threads(int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return uint64_t(sms) * 8u * kDpThreads;
}

// shared memory of a wavefront block: per warp, the lanes' strip tables and
// rmax rows of 2-bit codes (32 lanes x 16 bits, or x 32 bits for pairs)
static size_t wave_smem(int32_t rmax, uint32_t tb_bytes, int warps, uint32_t stage_extra = 0) {
    // + the staging space and a 16-byte mbarrier slot per warp (staged row bases)
    return size_t(warps) *
           (32u * tab_stride(tb_bytes) * 4u + size_t(rmax) * 32u * tb_bytes + stage_extra + 16u);
}

// Staging space a warp can have past its code rows without costing a block an
// SM: the shared memory the register budget's block count leaves unused (a
// multiple of 16 bytes, at most 16 KB; 0 when shared memory already limits).
static uint32_t wave_stage_extra(int dev, int32_t rmax, uint32_t tb_bytes, int warps, int tier) {
    if (tb_bytes != 4u) return 0u;  // only the pair tasks stage
    int smem_sm = 0, reserved = 0;
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0u;
    }
    const size_t blocks = size_t(kWaveRegBlocks(warps, tier));
    const size_t per_block = size_t(smem_sm) / blocks;
    const size_t base = wave_smem(rmax, tb_bytes, warps) + size_t(reserved);
    if (per_block <= base) return 0u;
    const size_t extra = ((per_block - base) / size_t(warps)) & ~size_t(15);
    return uint32_t(extra < 16384u ? extra : 16384u);
}

bool dp_wave_fits(int32_t rmax) { return wave_smem(rmax, 2, kWaveWarps) <= 200u * 1024u; }

void launch_dp(const DpLaunch &a_in, const uint64_t *bin_off, uint64_t *tasks, int32_t cmax,
               cudaStream_t st) {
    if (!a_in.nd) return;
    DpLaunch a = a_in;
    if (a.warps != 1 && a.warps != 2) a.warps = 4;
    // pairs need 32-bit code rows; without the room none run
    if (wave_smem(a.rmax, 4, a.warps) > 200u * 1024u) a.pair_mask = 0;
    a.tb_bytes = a.pair_mask ? 4u : 2u;
    if (!dp_wave_fits(a.rmax)) {  // rows too long for the shared-memory codes
        const unsigned g = unsigned(a.threads / kDpThreads);
        counted();
        if (a.affine) {
            k_dp<true><<<g, kDpThreads, 0, st>>>(a);
        } else {
            k_dp<false><<<g, kDpThreads, 0, st>>>(a);
        }
        return;
    }
    counted();
    k_dp_tasks<<<1, 32, 0, st>>>(bin_off, tasks, a.pair_mask);
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // a persistent grid: twice the blocks that fit for registers (the work queue
    // stops the extra ones at once)
    const int tier = (a.warps == 1 || wave_reg_tier(a.regs) < 2) ? wave_reg_tier(a.regs) : 1;
    a.stage_extra = wave_stage_extra(dev, a.rmax, a.tb_bytes, a.warps, tier);
    const size_t smem = wave_smem(a.rmax, a.tb_bytes, a.warps, a.stage_extra);
    const unsigned g = unsigned(sms) * unsigned(2 * kWaveRegBlocks(a.warps, tier));
    // the opt-in is set once per size increase (never while a graph is being captured
    // for a size not seen before: the eager round that precedes a capture sets it)
    // (per device, and shared by the host threads of every context in the process)
    constexpr int kOptDevices = 64;
    static std::mutex opt_mu;
    static size_t opted[kOptDevices][2][3][3] = {};
    const int ai = a.affine ? 1 : 0, wi = a.warps == 1 ? 0 : (a.warps == 2 ? 1 : 2), ri = tier;
    using WaveFn = void (*)(DpLaunch, uint64_t *);
    // the 255-register tier is built for 1-warp blocks only (the tuning
    // table refuses it with larger blocks); their slots take tier 1
    const WaveFn fns[2][3][3] = {
        {{k_dp_wave<false, 1, 0>, k_dp_wave<false, 1, 1>, k_dp_wave<false, 1, 2>},
         {k_dp_wave<false, 2, 0>, k_dp_wave<false, 2, 1>, k_dp_wave<false, 2, 1>},
         {k_dp_wave<false, 4, 0>, k_dp_wave<false, 4, 1>, k_dp_wave<false, 4, 1>}},
        {{k_dp_wave<true, 1, 0>, k_dp_wave<true, 1, 1>, k_dp_wave<true, 1, 2>},
         {k_dp_wave<true, 2, 0>, k_dp_wave<true, 2, 1>, k_dp_wave<true, 2, 1>},
         {k_dp_wave<true, 4, 0>, k_dp_wave<true, 4, 1>, k_dp_wave<true, 4, 1>}}};
    const WaveFn fn = fns[ai][wi][ri];
    if (smem > 48u * 1024u) {
        std::lock_guard<std::mutex> lock(opt_mu);
        if (dev >= kOptDevices || smem > opted[dev][ai][wi][ri]) {
            cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (dev < kOptDevices) opted[dev][ai][wi][ri] = smem;
        }
    }
    counted();
    fn<<<g, unsigned(32 * a.warps), smem, st>>>(a, tasks);
    if (cmax > 32 * kStripW) {
        const unsigned gw = unsigned(a.threads / kDpThreads);
        counted();
        if (a.affine) {
            k_dp_wide<true><<<gw, kDpThreads, 0, st>>>(a, tasks);
        } else {
            k_dp_wide<false><<<gw, kDpThreads, 0, st>>>(a, tasks);
        }
    }
}

void launch_assemble(const Params &p, uint64_t nc, ChainArrays ch, const uint32_t *keys,
                     ReadsView subj, ReadsView q, const DpSum *sums, const uint32_t *cells,
                     unsigned long long *counters, cudaStream_t st) {
    if (nc) {
        counted();
        k_assemble<<<grid_1d(nc, 128), 128, 0, st>>>(p, nc, ch, keys, subj, q, sums, cells, counters);
    }
}

void launch_dedupe(uint64_t nsub, const uint32_t *seg_chain_start,
                   const uint32_t *seg_chain_count, ChainArrays ch, uint32_t *winners,
                   unsigned long long *counters, cudaStream_t st) {
    if (nsub) {
        counted();
        k_dedupe<<<grid_1d(nsub, 128), 128, 0, st>>>(nsub, seg_chain_start, seg_chain_count, ch,
                                                     winners, counters);
    }
}

void launch_map_choose(const Params &p, uint64_t nsub, const uint32_t *cstart,
                       const uint32_t *ccount, ChainArrays ch, const uint32_t *keys,
                       ReadsView subj, ReadsView q, const DpSum *sums, uint32_t *alist,
                       uint32_t *winners, unsigned long long *counters, cudaStream_t st) {
    if (!nsub) return;
    counted();
    k_map_choose<<<grid_1d(nsub, 128), 128, 0, st>>>(p, nsub, cstart, ccount, ch, keys, subj, q,
                                                     sums, alist, winners, counters);
}

void launch_map_hist(ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint64_t bins,
                     unsigned long long *hist, unsigned long long *maxc, cudaStream_t st) {
    if (!q.n) return;
    counted();
    k_map_hist<<<grid_1d(q.n * 32, 256), 256, 0, st>>>(q, cov, mdiff, bins, hist, maxc);
}

void launch_aln_list(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                     ChainArrays ch, ReadsView q, uint32_t *alist, uint32_t *alist_n,
                     unsigned long long *counters, cudaStream_t st) {
    if (!nsub) return;
    counted();
    k_aln_list<<<grid_1d(nsub, 128), 128, 0, st>>>(nsub, cstart, ccount, ch, q, alist, alist_n,
                                                   counters);
}

void launch_aln_units(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                      const uint32_t *alist, const uint32_t *alist_n, const uint64_t *rec_off,
                      ReadsView subj, uint32_t *unit, uint32_t *ulen, cudaStream_t st) {
    if (!nsub) return;
    counted();
    k_aln_units<<<grid_1d(nsub, 128), 128, 0, st>>>(nsub, cstart, ccount, alist, alist_n, rec_off,
                                                    subj, unit, ulen);
}

void launch_aln_size(const Params &p, uint64_t nunit, const uint32_t *unit, ChainArrays ch,
                     const uint32_t *keys, ReadsView subj, ReadsView q, const uint32_t *ops,
                     uint32_t stride, const DpSum *sums, uint32_t *ulen, uint32_t *upre,
                     uint32_t *ucig, cudaStream_t st) {
    if (!nunit) return;
    counted();
    k_aln_size<<<grid_1d(nunit, 128), 128, 0, st>>>(p, nunit, unit, ch, keys, subj, q, ops, stride,
                                                    sums, ulen, upre, ucig);
}

void launch_aln_write(const Params &p, uint64_t nunit, const uint32_t *unit, const uint64_t *uoff,
                      ChainArrays ch, const uint32_t *keys, ReadsView subj, ReadsView q,
                      const uint32_t *ops, uint32_t stride, const DpSum *sums,
                      const uint32_t *upre, const uint32_t *ucig, char *text, cudaStream_t st) {
    if (!nunit) return;
    counted();
    k_aln_write<<<grid_1d(nunit, 128), 128, 0, st>>>(p, nunit, unit, uoff, ch, keys, subj, q, ops,
                                                     stride, sums, upre, ucig, text);
}

void launch_vote(const Params &p, uint64_t max_winners, ChainArrays ch, const uint32_t *winners,
                 uint32_t *sorted, uint32_t *win_bins, const uint32_t *keys, ReadsView subj,
                 ReadsView q, const uint32_t *ops, uint32_t stride, const DpSum *sums,
                 uint32_t *cov, int32_t *mdiff, unsigned long long *counters, cudaStream_t st) {
    if (!max_winners) return;
    uint32_t *bins = win_bins, *off = win_bins + kWinBins, *cursor = win_bins + 2 * kWinBins;
    cudaMemsetAsync(bins, 0, kWinBins * sizeof(uint32_t), st);
    const unsigned g = grid_1d(max_winners, 256, 148u * 8u);
    counted();
    k_win_hist<<<g, 256, 0, st>>>(counters, ch, winners, bins);
    counted();
    k_win_offsets<<<1, 32, 0, st>>>(bins, off, cursor);
    counted();
    k_win_scatter<<<g, 256, 0, st>>>(counters, ch, winners, off, cursor, sorted);
    counted();
    k_vote<<<grid_1d(max_winners, 128), 128, 0, st>>>(p, counters, ch, sorted, keys, subj, q, ops,
                                                      stride, sums, cov, mdiff, counters);
}

void launch_vote_overhang(const Params &p, uint64_t max_winners, ChainArrays ch,
                          const uint32_t *winners, const uint32_t *keys, ReadsView subj,
                          ReadsView q, const DpSum *sums, uint32_t *ext,
                          const unsigned long long *counters, cudaStream_t st) {
    if (!max_winners) return;
    counted();
    k_vote_overhang<<<grid_1d(max_winners, 128), 128, 0, st>>>(p, counters, ch, winners, keys, subj,
                                                               q, sums, ext);
}

void launch_merge_pairs(uint64_t npairs, const uint64_t *off, const uint8_t *corrected,
                        const uint32_t *ext, uint8_t *merged, uint32_t *merged_len,
                        cudaStream_t st) {
    if (!npairs) return;
    counted();
    k_merge_pairs<<<grid_1d(npairs, 128), 128, 0, st>>>(npairs, off, corrected, ext, merged,
                                                        merged_len);
}

void launch_consensus(const Params &p, ReadsView q, const uint32_t *cov, const int32_t *mdiff,
                      uint8_t *out, uint32_t *colsum, uint32_t *imin, uint32_t *imed,
                      uint32_t *imax, double *mis, cudaStream_t st) {
    if (q.n) {
        counted();
        k_consensus<<<grid_1d(q.n, 8, 148u * 32u), 256, 0, st>>>(p, q, cov, mdiff, out, colsum,
                                                                 imin, imed, imax, mis);
    }
}

void launch_expand_votes(ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint32_t *out,
                         cudaStream_t st) {
    if (q.n) {
        counted();
        k_expand_votes<<<grid_1d(q.n, 8, 148u * 32u), 256, 0, st>>>(q, cov, mdiff, out);
    }
}

void launch_fingerprint(const uint8_t *raw, uint64_t nb, const uint64_t *off, const int64_t *uid,
                        uint64_t n, unsigned long long *out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, 8, st);
    counted();
    k_fingerprint<<<grid_1d(std::max<uint64_t>(nb / 8, n), 256, 148u * 8u), 256, 0, st>>>(
        raw, nb, off, uid, n, out);
}

void launch_stamp(unsigned long long *out, cudaStream_t st) {
    counted();
    k_stamp<<<1, 1, 0, st>>>(out);
}

void launch_unpack_ops(const uint32_t *ops, uint32_t stride, const DpSum *sums, uint64_t nd,
                       const uint64_t *out_off, uint8_t *out, int32_t *nops, cudaStream_t st) {
    if (nd) {
        counted();
        k_unpack_ops<<<grid_1d(nd, 128), 128, 0, st>>>(ops, stride, sums, nd, out_off, out, nops);
    }
}

}  // namespace hero
