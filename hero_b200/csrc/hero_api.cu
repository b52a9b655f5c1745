// hero_api.cu -- host engine behind the C ABI declared in include/hero_gpu.h.
//
// One context = one device, one stream, one query set, its k-mer table and
// its vote matrix.  Subject reads stream through in batches; every stage of a
// batch runs as its own kernel (the plain one-launch-per-stage form).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hero_gpu.h"
#include "hero_internal.cuh"

using namespace hero;

namespace {

struct DBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool external = false;  // caller-owned memory: never freed or grown here
    bool pooled = false;    // allocated stream-ordered (freed the same way)
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

}  // namespace

struct hero_ctx {
    hero_params P{};
    Params p{};
    int dev = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::string err;
    size_t bytes = 0, bytes_peak = 0;
    std::vector<DBuf *> all;

    // query set
    uint64_t nq = 0, nqb = 0;
    DBuf q_raw, q_code, q_off, q_len, q_uid, q_good, q_sgood, q_gc;
    DBuf q_job;            // job of each query read (jobs served together)
    bool tagged = false;   // q_job holds the reads' jobs
    bool have_queries = false, have_index = false;
    // k-mer table
    DBuf t_slots, t_vals;
    uint64_t t_mask = 0, t_keys = 0;
    // vote matrix + consensus outputs
    DBuf cov, mdiff, out_seq, colsum, o_imin, o_imed, o_imax, o_mis;
    // subject batch (when not aligning the query set against itself)
    DBuf s_raw, s_code, s_off, s_len, s_uid, s_good;
    // batch buffers
    DBuf seg_hits, hit_off, hits, seg_cstart, seg_ccount;
    DBuf cs_grp, cs_chain_of, cs_first, cs_last, cs_prev, cs_size, cs_coff, cs_ckeys, cs_kl,
        cs_gnch, cs_gbest, cs_gkept, cs_gkeys, cs_gdp;
    DBuf ch_subj, ch_query, ch_key_off, ch_seg_off, ch_nkeys, ch_nseg, ch_orient, ch_status,
        ch_win, ch_rate, ch_len;
    DBuf keys, segs, sums, cells, ops, perm, bins, bin_off, tb, bnd, dp_tasks, winners;
    DBuf win_sorted, win_bins;  // winners sorted by chain shape, and the sort's bins
    DBuf scan_tmp, counters;
    // alignment output: record lists, text units and the batch's text
    DBuf a_list, a_n, a_roff, a_unit, a_len, a_pre, a_cig, a_uoff, a_text;
    // --merge: overhang votes per query read, merged pairs
    DBuf q_ext, m_seq, m_len;
    bool merge = false;
    bool mapping = false;  // --mapping: chosen records vote; coverage histogram
    std::vector<uint64_t> q_off_h;  // host copy of the query offsets (sizes of subject batches)
    void *vote_ext = nullptr;       // caller-owned vote state (hero_set_vote_buffer), or NULL
    uint64_t vote_ext_bytes = 0;
    DBuf wcache;                    // per batch: the table slot each probe window found
    DBuf map_hist, map_max;
    bool consensus_done = false;  // out_seq holds the consensus of the current votes
    std::vector<uint8_t> aln_host;  // .aln text of every subject aligned since the last take
    // index build temporaries (kept between builds)
    DBuf x_cnt, x_koff, x_klo, x_khi, x_kval, x_owner, x_count, x_slot_of, x_start, x_fill, x_tmp;
    uint64_t dp_T = 0;

    hero_stats stats{};
    unsigned long long ctr[C_COUNT] = {};

    // batched form: per-batch sizes of the last eager round, and its graph
    struct BatchPlan {
        uint64_t H, NC, ND;
        int32_t rmax, cmax;
    };
    std::vector<BatchPlan> plan;
    uint64_t plan_nkeys = 0, plan_fp = 0, qfp = 0;
    bool plan_ok = false, capturing = false;
    size_t batch_idx = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    DBuf stamps;  // DP kernel start/stop times per batch (ns), written inside the graph
    DBuf fp;
    std::vector<hero_dp_tuning> tuning;  // DP kernel shapes per class of batch

    hero_ctx() {
        DBuf *list[] = {&q_raw, &q_code, &q_off, &q_len, &q_uid, &q_good, &q_sgood, &q_gc,
                        &t_slots, &t_vals, &cov, &mdiff, &out_seq, &colsum, &o_imin, &o_imed, &o_imax,
                        &o_mis, &s_raw, &s_code, &s_off, &s_len, &s_uid, &s_good, &seg_hits,
                        &hit_off, &hits, &seg_cstart, &seg_ccount, &cs_grp, &cs_chain_of,
                        &cs_first, &cs_last, &cs_prev, &cs_size, &cs_coff, &cs_ckeys, &cs_kl,
                        &cs_gnch, &cs_gbest, &cs_gkept, &cs_gkeys, &cs_gdp, &ch_subj, &ch_query,
                        &ch_key_off, &ch_seg_off, &ch_nkeys, &ch_nseg, &ch_orient, &ch_status,
                        &ch_win, &ch_rate, &ch_len, &keys, &segs, &sums, &cells, &ops, &perm,
                        &bins, &bin_off, &tb, &bnd, &dp_tasks, &winners, &scan_tmp, &counters, &x_cnt, &x_koff,
                        &x_klo, &x_khi, &x_kval, &x_owner, &x_count, &x_slot_of, &x_start,
                        &x_fill, &x_tmp, &q_job, &win_sorted, &win_bins, &a_list, &a_n,
                        &a_roff, &a_unit, &a_len, &a_pre, &a_cig, &a_uoff, &a_text, &q_ext,
                        &m_seq, &m_len, &map_hist, &map_max, &wcache};
        for (DBuf *b : list) all.push_back(b);
    }

    int fail(int code, const std::string &m) {
        err = m;
        return code;
    }
    int cuda(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return HERO_OK;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return HERO_E_CUDA;
    }
    int check_launch(const char *what) {
        cudaError_t e = cudaGetLastError();
        return cuda(e, what);
    }
    // Buffers are allocated and freed stream-ordered on the context's stream
    // (the device's default memory pool, which returns freed memory to the
    // device at the stream's next synchronisation): growing one waits for no
    // other stream, so contexts that run side by side -- the serving workers --
    // do not stall each other's launches the way cudaFree's device-wide
    // synchronisation does.  Inside a stream capture (no growth is expected
    // there: sizes come from the eager round's plan) the plain calls are used.
    void release(DBuf &b) {
        if (b.p && !b.external) {
            if (b.pooled) cudaFreeAsync(b.p, st);
            else cudaFree(b.p);
            bytes -= b.cap;
        }
        b.p = nullptr;
        b.cap = 0;
        b.external = false;
        b.pooled = false;
    }
    // grows a device buffer to at least `need` bytes (contents are not kept)
    int ensure(DBuf &b, size_t need, const char *what) {
        if (need == 0) need = 16;
        if (b.cap >= need) return HERO_OK;
        if (b.external) return fail(HERO_E_INPUT, std::string("caller's buffer too small for ") + what);
        const auto t0 = std::chrono::steady_clock::now();
        release(b);
        size_t want = need + need / 4 + 256;
        if (P.device_memory_budget && bytes + want > P.device_memory_budget) {
            want = need;
            if (bytes + want > P.device_memory_budget)
                return fail(HERO_E_OOM, std::string("device memory budget exceeded at ") + what);
        }
        const bool pooled = !capturing && st;
        cudaError_t e = pooled ? cudaMallocAsync(&b.p, want, st) : cudaMalloc(&b.p, want);
        if (e != cudaSuccess && pooled) {
            // memory freed on other streams may still wait in the pool: settle
            // this stream and try once more
            cudaGetLastError();
            cudaStreamSynchronize(st);
            e = cudaMallocAsync(&b.p, want, st);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return fail(HERO_E_OOM, std::string("device allocation failed for ") + what + ": " +
                                        cudaGetErrorString(e));
        }
        b.cap = want;
        b.pooled = pooled;
        bytes += want;
        bytes_peak = std::max(bytes_peak, bytes);
        stats.buffer_allocs++;
        stats.ms_alloc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return HERO_OK;
    }
    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }
    ~hero_ctx() {
        drop_graph();
        release(fp);
        release(stamps);
        for (DBuf *b : all) release(*b);
        if (own_stream && st) cudaStreamDestroy(st);
    }
};

template <class T>
static T *P_(DBuf &b) {
    return reinterpret_cast<T *>(b.p);
}

#define HERO_TRY(x)                 \
    do {                            \
        int _r = (x);               \
        if (_r != HERO_OK) return _r; \
    } while (0)

static const uint32_t *job_tags(hero_ctx *c) { return c->tagged ? P_<uint32_t>(c->q_job) : nullptr; }

static ReadsView query_view(hero_ctx *c) {
    return ReadsView{P_<uint8_t>(c->q_code), P_<uint64_t>(c->q_off), P_<uint32_t>(c->q_len),
                     P_<int64_t>(c->q_uid), P_<uint8_t>(c->q_good), c->nq, job_tags(c)};
}

// kernel shape of a DP launch from the tuning table (first class covering rmax)
static void apply_tuning(const hero_ctx *c, DpLaunch &a) {
    for (const hero_dp_tuning &t : c->tuning)
        if (a.rmax <= t.rows_max) {
            a.warps = (t.warps_per_block == 1 || t.warps_per_block == 2) ? t.warps_per_block : 4;
            a.regs = (t.regs_per_thread == 168 || t.regs_per_thread == 255) ? t.regs_per_thread : 128;
            a.pair_mask = t.pair_strips;
            a.chunk_mask = t.chunk_strips;
            return;
        }
}

static double elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return double(ms);
}

extern "C" int hero_device_init(int32_t device) {
    if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
        cudaGetLastError();
        return HERO_E_CUDA;
    }
    return HERO_OK;
}

extern "C" void hero_default_params(hero_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->k = 39;
    p->min_overlap = 40;
    p->aligner = HERO_ALIGNER_GLOBAL;
    p->device = 0;
    p->max_mismatch_rate = 1.0;
    p->max_indel_rate = 1.0;
    p->consensus_threshold = 0.6;
}

extern "C" int hero_create(const hero_params *p, hero_ctx **out) {
    if (!p || !out) return HERO_E_INPUT;
    *out = nullptr;
    if (p->k < 1 || p->k > 63) return HERO_E_INPUT;
    if (p->flags & ~(HERO_FLAG_ALIGNMENT_OUTPUT | HERO_FLAG_MERGE_PAIRS | HERO_FLAG_MAPPING))
        return HERO_E_INPUT;
    if ((p->flags & HERO_FLAG_ALIGNMENT_OUTPUT) && (p->flags & (HERO_FLAG_MERGE_PAIRS | HERO_FLAG_MAPPING)))
        return HERO_E_INPUT;  // --merge and --mapping are parts of the consensus mode
    if ((p->flags & HERO_FLAG_MERGE_PAIRS) && (p->flags & HERO_FLAG_MAPPING))
        return HERO_E_INPUT;  // the reference writes the mapping histogram instead
    hero_ctx *c = new hero_ctx();
    c->P = *p;
    c->p.k = p->k;
    c->p.l = p->min_overlap;
    c->p.affine = p->aligner == HERO_ALIGNER_AFFINE ? 1 : 0;
    c->p.mis_rate = p->max_mismatch_rate;
    c->p.indel_rate = p->max_indel_rate;
    c->p.thr = p->consensus_threshold;
    c->p.aln = (p->flags & HERO_FLAG_ALIGNMENT_OUTPUT) ? 1 : 0;
    c->merge = (p->flags & HERO_FLAG_MERGE_PAIRS) != 0;
    c->mapping = (p->flags & HERO_FLAG_MAPPING) != 0;
    c->dev = p->device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        delete c;
        return HERO_E_CUDA;
    }
    if (cudaSetDevice(c->dev) != cudaSuccess) {
        delete c;
        return HERO_E_CUDA;
    }
    if (p->stream) {
        c->st = reinterpret_cast<cudaStream_t>(p->stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return HERO_E_CUDA;
        }
        c->own_stream = true;
    }
    c->dp_T = dp_threads(c->dev);
    if (c->ensure(c->counters, sizeof(unsigned long long) * C_COUNT, "counters")) {
        delete c;
        return HERO_E_OOM;
    }
    // running totals and the overflow flag start at zero (recycled device memory
    // holds whatever its last owner left there)
    if (cudaMemset(c->counters.p, 0, sizeof(unsigned long long) * C_COUNT) != cudaSuccess) {
        hero_destroy(c);
        return HERO_E_CUDA;
    }
    *out = c;
    return HERO_OK;
}

extern "C" void hero_destroy(hero_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->dev);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    delete ctx;
}

extern "C" const char *hero_last_error(const hero_ctx *ctx) {
    return ctx ? ctx->err.c_str() : "no context";
}

// uploads reads and derives codes, lengths and good flags on the device
static int upload_reads(hero_ctx *c, const uint8_t *seq, const uint64_t *off, const int64_t *uid,
                        uint64_t n, DBuf &raw, DBuf &code, DBuf &doff, DBuf &len, DBuf &duid,
                        DBuf *gq, DBuf *gs, DBuf *gc) {
    const uint64_t nb = n ? off[n] : 0;
    HERO_TRY(c->ensure(raw, nb, "reads"));
    // 16 bytes past the last base: the DP's bulk copies of a segment's rows
    // round their end up to 16 bytes
    HERO_TRY(c->ensure(code, nb + 16, "codes"));
    HERO_TRY(c->ensure(doff, (n + 1) * 8, "offsets"));
    HERO_TRY(c->ensure(len, n * 4, "lengths"));
    HERO_TRY(c->ensure(duid, n * 8, "ids"));
    if (gq) HERO_TRY(c->ensure(*gq, n, "good"));
    if (gs) HERO_TRY(c->ensure(*gs, n, "good"));
    if (gc) HERO_TRY(c->ensure(*gc, n * 8, "gc"));
    if (n == 0) {
        const uint64_t z = 0;
        return c->cuda(cudaMemcpy(doff.p, &z, 8, cudaMemcpyHostToDevice), "upload");
    }
    HERO_TRY(c->cuda(cudaMemcpyAsync(raw.p, seq, nb, cudaMemcpyHostToDevice, c->st), "upload"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(doff.p, off, (n + 1) * 8, cudaMemcpyHostToDevice, c->st), "upload"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(duid.p, uid, n * 8, cudaMemcpyHostToDevice, c->st), "upload"));
    launch_prep_reads(P_<uint8_t>(raw), nb, P_<uint8_t>(code), P_<uint64_t>(doff), n,
                      P_<uint32_t>(len), gq ? P_<uint8_t>(*gq) : nullptr,
                      gs ? P_<uint8_t>(*gs) : nullptr, gc ? P_<double>(*gc) : nullptr, c->p.l, c->st);
    return c->check_launch("prep reads");
}

static int validate_reads(hero_ctx *c, const uint8_t *seq, const uint64_t *off, const int64_t *uid,
                          uint64_t n) {
    if (n && (!seq || !off || !uid)) return c->fail(HERO_E_INPUT, "null read buffer");
    if (n >= 0xffffffffull) return c->fail(HERO_E_INPUT, "too many reads");
    if (!off) return HERO_OK;
    if (off[0] != 0) return c->fail(HERO_E_INPUT, "offsets must start at 0");
    for (uint64_t i = 0; i < n; i++) {
        if (off[i + 1] < off[i]) return c->fail(HERO_E_INPUT, "offsets must not decrease");
        if (off[i + 1] - off[i] > 32767) return c->fail(HERO_E_INPUT, "reads longer than 32767 bases");
    }
    return HERO_OK;
}

extern "C" int hero_set_queries(hero_ctx *c, const uint8_t *seq, const uint64_t *off,
                                const int64_t *uid, uint64_t n) {
    if (!c) return HERO_E_INPUT;
    cudaSetDevice(c->dev);
    HERO_TRY(validate_reads(c, seq, off, uid, n));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c->st);
    c->nq = n;
    c->nqb = n ? off[n] : 0;
    c->q_off_h.assign(off, off + (n ? n + 1 : 0));
    c->have_index = false;
    c->consensus_done = false;
    c->tagged = false;
    HERO_TRY(upload_reads(c, seq, n ? off : nullptr, uid, n, c->q_raw, c->q_code, c->q_off,
                          c->q_len, c->q_uid, &c->q_good, &c->q_sgood, &c->q_gc));
    HERO_TRY(c->ensure(c->fp, 8, "fingerprint"));
    launch_fingerprint(P_<uint8_t>(c->q_raw), c->nqb, P_<uint64_t>(c->q_off), P_<int64_t>(c->q_uid), n,
                       P_<unsigned long long>(c->fp), c->st);
    if (c->vote_ext) {  // the caller's buffer: mismatch votes, then match-run differences
        if (c->vote_ext_bytes < c->nqb * 20) return c->fail(HERO_E_INPUT, "vote buffer smaller than 20 bytes a query base");
        c->release(c->cov);
        c->release(c->mdiff);
        c->cov = DBuf{c->vote_ext, size_t(c->nqb * 16), true};
        c->mdiff = DBuf{static_cast<uint8_t *>(c->vote_ext) + c->nqb * 16, size_t(c->nqb * 4), true};
    }
    HERO_TRY(c->ensure(c->cov, c->nqb * 16, "vote matrix"));
    HERO_TRY(c->ensure(c->mdiff, c->nqb * 4, "vote matrix"));
    HERO_TRY(c->cuda(cudaMemsetAsync(c->cov.p, 0, c->nqb * 16, c->st), "memset"));
    HERO_TRY(c->cuda(cudaMemsetAsync(c->mdiff.p, 0, c->nqb * 4, c->st), "memset"));
    if (c->merge) {
        HERO_TRY(c->ensure(c->q_ext, n * kOverhang * 16, "overhang votes"));
        if (n) HERO_TRY(c->cuda(cudaMemsetAsync(c->q_ext.p, 0, n * kOverhang * 16, c->st), "memset"));
    }
    cudaEventRecord(e1, c->st);
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "set queries"));
    c->stats.ms_upload += elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->stats.queries = n;
    unsigned long long fpv = 0;
    HERO_TRY(c->cuda(cudaMemcpy(&fpv, c->fp.p, 8, cudaMemcpyDeviceToHost), "fingerprint"));
    c->qfp = fpv ^ (uint64_t(n) * 0x9e3779b97f4a7c15ull) ^ c->nqb;
    if (c->qfp != c->plan_fp) c->plan_ok = false;
    std::vector<uint8_t> g(n);
    if (n) HERO_TRY(c->cuda(cudaMemcpy(g.data(), c->q_good.p, n, cudaMemcpyDeviceToHost), "good flags"));
    uint64_t ng = 0;
    for (uint8_t x : g) ng += x;
    c->stats.good_queries = ng;
    c->have_queries = true;
    return HERO_OK;
}

// the first fault of a tuning table, or nullptr
static const char *dp_tuning_fault(const hero_dp_tuning *t, uint32_t n) {
    if (n && !t) return "null tuning table";
    for (uint32_t i = 0; i < n; i++)
        if (t[i].warps_per_block != 1 && t[i].warps_per_block != 2 && t[i].warps_per_block != 4)
            return "warps_per_block must be 1, 2 or 4";
        else if (t[i].regs_per_thread != 0 && t[i].regs_per_thread != 128 && t[i].regs_per_thread != 168 &&
                 !(t[i].regs_per_thread == 255 && t[i].warps_per_block == 1))
            return "regs_per_thread must be 0, 128 or 168 (or 255 with 1-warp blocks)";
    return nullptr;
}

extern "C" int hero_dp_tuning_check(const hero_dp_tuning *t, uint32_t n) {
    return dp_tuning_fault(t, n) ? HERO_E_INPUT : HERO_OK;
}

extern "C" int hero_set_dp_tuning(hero_ctx *c, const hero_dp_tuning *t, uint32_t n) {
    if (!c) return HERO_E_INPUT;
    if (const char *f = dp_tuning_fault(t, n)) return c->fail(HERO_E_INPUT, f);
    c->tuning.assign(t, t + n);
    c->plan_ok = false;  // a captured round keeps the shapes it was captured with
    return HERO_OK;
}

extern "C" int hero_set_query_jobs(hero_ctx *c, const uint32_t *job, uint64_t n) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (n != c->nq) return c->fail(HERO_E_INPUT, "one job per query read");
    if (n && !job) return c->fail(HERO_E_INPUT, "null job buffer");
    cudaSetDevice(c->dev);
    const int bits = kmer_job_bits(c->p.k);
    uint64_t h = 0x51ed270b27a4f3b1ull;
    for (uint64_t i = 0; i < n; i++) {
        if (bits < 32 && (job[i] >> bits) != 0)
            return c->fail(HERO_E_INPUT, "job index does not fit beside the k-mer in a key");
        h = mix64(h ^ (uint64_t(job[i]) + i));
    }
    HERO_TRY(c->ensure(c->q_job, n * 4, "jobs"));
    if (n)
        HERO_TRY(c->cuda(cudaMemcpy(c->q_job.p, job, n * 4, cudaMemcpyHostToDevice), "upload jobs"));
    c->tagged = true;
    c->have_index = false;
    c->qfp ^= h;  // the graph of a round is keyed on the tagged read set
    if (c->qfp != c->plan_fp) c->plan_ok = false;
    return HERO_OK;
}

extern "C" int hero_build_index(hero_ctx *c) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    cudaSetDevice(c->dev);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (!c->capturing) cudaEventRecord(e0, c->st);
    const uint64_t n = c->nq;
    ReadsView q = query_view(c);
    DBuf &cnt = c->x_cnt, &koff = c->x_koff, &klo = c->x_klo, &khi = c->x_khi, &kval = c->x_kval,
         &owner = c->x_owner, &count = c->x_count, &slot_of = c->x_slot_of, &start = c->x_start,
         &fill = c->x_fill, &tmp = c->x_tmp;
    int r = HERO_OK;
    do {
        if ((r = c->ensure(cnt, n * 4 + 4, "key counts"))) break;
        if ((r = c->ensure(koff, (n + 1) * 8, "key offsets"))) break;
        if ((r = c->ensure(tmp, scan_tmp_bytes(n + 1), "scan"))) break;
        if ((r = c->check_launch("index: before"))) break;
        launch_key_count(q, c->p.k, P_<uint32_t>(cnt), c->st);
        if ((r = c->check_launch("index: key count"))) break;
        launch_scan_u32(P_<uint32_t>(cnt), P_<uint64_t>(koff), n, tmp.p, c->st);
        if ((r = c->check_launch("index: key scan"))) break;
        uint64_t nkeys = 0;
        if (c->capturing) {
            nkeys = c->plan_nkeys;
        } else {
            if ((r = c->cuda(cudaMemcpyAsync(&nkeys, P_<uint64_t>(koff) + n, 8, cudaMemcpyDeviceToHost, c->st), "keys"))) break;
            if ((r = c->cuda(cudaStreamSynchronize(c->st), "keys"))) break;
            c->plan_nkeys = nkeys;
        }
        uint64_t slots = 1024;
        while (slots < 2 * nkeys) slots <<= 1;
        c->t_keys = nkeys;
        c->t_mask = slots - 1;
        if ((r = c->ensure(klo, nkeys * 8, "keys"))) break;
        if ((r = c->ensure(khi, nkeys * 8, "keys"))) break;
        if ((r = c->ensure(kval, nkeys * 8, "keys"))) break;
        if ((r = c->ensure(slot_of, nkeys * 4, "keys"))) break;
        if ((r = c->ensure(owner, slots * 4, "table"))) break;
        if ((r = c->ensure(count, slots * 4, "table"))) break;
        if ((r = c->ensure(fill, slots * 4, "table"))) break;
        if ((r = c->ensure(start, (slots + 1) * 8, "table"))) break;
        if ((r = c->ensure(c->t_slots, slots * sizeof(Slot), "table"))) break;
        if ((r = c->ensure(c->t_vals, nkeys * 8, "table values"))) break;
        if ((r = c->ensure(tmp, scan_tmp_bytes(slots + 1), "scan"))) break;
        launch_key_emit(q, c->p.k, P_<uint64_t>(koff), P_<uint64_t>(klo), P_<uint64_t>(khi),
                        P_<uint64_t>(kval), c->st);
        if ((r = c->check_launch("index: key emit"))) break;
        if ((r = c->cuda(cudaMemsetAsync(owner.p, 0xff, slots * 4, c->st), "index: memset"))) break;
        if ((r = c->cuda(cudaMemsetAsync(count.p, 0, slots * 4, c->st), "index: memset"))) break;
        if ((r = c->cuda(cudaMemsetAsync(fill.p, 0, slots * 4, c->st), "index: memset"))) break;
        launch_table_insert(P_<uint64_t>(klo), P_<uint64_t>(khi), nkeys, P_<uint32_t>(owner),
                            P_<uint32_t>(count), P_<uint32_t>(slot_of), c->t_mask, c->st);
        launch_scan_u32(P_<uint32_t>(count), P_<uint64_t>(start), slots, tmp.p, c->st);
        launch_table_fill(P_<uint64_t>(kval), nkeys, P_<uint32_t>(slot_of), P_<uint64_t>(start),
                          P_<uint32_t>(fill), P_<uint64_t>(c->t_vals), c->st);
        launch_table_finalize(P_<uint64_t>(klo), P_<uint64_t>(khi), P_<uint32_t>(owner),
                              P_<uint32_t>(count), P_<uint64_t>(start), slots,
                              P_<Slot>(c->t_slots), c->st);
        if ((r = c->check_launch("index"))) break;
        if (!c->capturing) {
            cudaEventRecord(e1, c->st);
            if ((r = c->cuda(cudaStreamSynchronize(c->st), "index"))) break;
            c->stats.ms_index += elapsed(e0, e1);
        }
        c->stats.index_keys = nkeys;
        c->stats.index_slots = slots;
        c->have_index = true;
    } while (0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return r;
}

// Alignment output of one batch (after the records are scored): the kept
// records per subject (SubjectRead::addAlignment by query uniqueId), the text
// units, their sizes, a scan, the text; appended to the context's host text.
static int aln_batch(hero_ctx *c, ReadsView subj, uint64_t nsub, ReadsView q,
                     const ChainArrays &ch, uint64_t NC, uint32_t stride) {
    unsigned long long *ctr = P_<unsigned long long>(c->counters);
    if (NC >= uint64_t(kUnitChainLimit) || nsub >= uint64_t(kUnitChainLimit))
        return c->fail(HERO_E_INPUT, "too many chains or subjects in a batch");
    HERO_TRY(c->ensure(c->a_list, std::max<uint64_t>(NC, 1) * 4, "alignment lists"));
    HERO_TRY(c->ensure(c->a_n, nsub * 4 + 4, "alignment lists"));
    HERO_TRY(c->ensure(c->a_roff, (nsub + 1) * 8, "alignment lists"));
    launch_aln_list(nsub, P_<uint32_t>(c->seg_cstart), P_<uint32_t>(c->seg_ccount), ch, q,
                    P_<uint32_t>(c->a_list), P_<uint32_t>(c->a_n), ctr, c->st);
    launch_scan_u32(P_<uint32_t>(c->a_n), P_<uint64_t>(c->a_roff), nsub, c->scan_tmp.p, c->st);
    HERO_TRY(c->check_launch("alignment lists"));
    uint64_t R = 0;
    HERO_TRY(c->cuda(cudaMemcpyAsync(&R, P_<uint64_t>(c->a_roff) + nsub, 8, cudaMemcpyDeviceToHost, c->st), "alignment lists"));
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "alignment lists"));
    const uint64_t U = R + 2 * nsub;  // units: header, records, closing newline per subject
    HERO_TRY(c->ensure(c->a_unit, U * 4, "alignment text"));
    HERO_TRY(c->ensure(c->a_len, U * 4, "alignment text"));
    HERO_TRY(c->ensure(c->a_pre, U * 4, "alignment text"));
    HERO_TRY(c->ensure(c->a_cig, U * 4, "alignment text"));
    HERO_TRY(c->ensure(c->a_uoff, (U + 1) * 8, "alignment text"));
    HERO_TRY(c->ensure(c->scan_tmp, scan_tmp_bytes(std::max<uint64_t>(U + 1, std::max<uint64_t>(2 * nsub + 1, kDpBins + 1))), "scan"));
    launch_aln_units(nsub, P_<uint32_t>(c->seg_cstart), P_<uint32_t>(c->seg_ccount),
                     P_<uint32_t>(c->a_list), P_<uint32_t>(c->a_n), P_<uint64_t>(c->a_roff), subj,
                     P_<uint32_t>(c->a_unit), P_<uint32_t>(c->a_len), c->st);
    launch_aln_size(c->p, U, P_<uint32_t>(c->a_unit), ch, P_<uint32_t>(c->keys), subj, q,
                    P_<uint32_t>(c->ops), stride, P_<DpSum>(c->sums), P_<uint32_t>(c->a_len),
                    P_<uint32_t>(c->a_pre), P_<uint32_t>(c->a_cig), c->st);
    launch_scan_u32(P_<uint32_t>(c->a_len), P_<uint64_t>(c->a_uoff), U, c->scan_tmp.p, c->st);
    HERO_TRY(c->check_launch("alignment text"));
    uint64_t B = 0;
    HERO_TRY(c->cuda(cudaMemcpyAsync(&B, P_<uint64_t>(c->a_uoff) + U, 8, cudaMemcpyDeviceToHost, c->st), "alignment text"));
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "alignment text"));
    HERO_TRY(c->ensure(c->a_text, B, "alignment text"));
    launch_aln_write(c->p, U, P_<uint32_t>(c->a_unit), P_<uint64_t>(c->a_uoff), ch,
                     P_<uint32_t>(c->keys), subj, q, P_<uint32_t>(c->ops), stride,
                     P_<DpSum>(c->sums), P_<uint32_t>(c->a_pre), P_<uint32_t>(c->a_cig),
                     P_<char>(c->a_text), c->st);
    HERO_TRY(c->check_launch("alignment text"));
    const size_t o = c->aln_host.size();
    c->aln_host.resize(o + B);
    if (B)
        HERO_TRY(c->cuda(cudaMemcpyAsync(c->aln_host.data() + o, c->a_text.p, B, cudaMemcpyDeviceToHost, c->st), "alignment text"));
    return c->cuda(cudaStreamSynchronize(c->st), "alignment text");
}

// runs every stage for subjects [0, nsub) of the given reads
static int align_batch(hero_ctx *c, ReadsView subj, uint64_t nsub, uint64_t nbases, double ms[6]) {
    const uint64_t nseg = 2 * nsub;
    ReadsView q = query_view(c);
    TableView t{P_<Slot>(c->t_slots), P_<uint64_t>(c->t_vals), c->t_mask};
    unsigned long long *ctr = P_<unsigned long long>(c->counters);
    const bool cap = c->capturing;
    hero_ctx::BatchPlan &bp = c->plan[c->batch_idx];
    cudaEvent_t ev[7];
    for (auto &e : ev) cudaEventCreate(&e);
    auto rec = [&](int k) {
        if (!cap) cudaEventRecord(ev[k], c->st);
    };
    int r = HERO_OK;
    do {
        rec(0);
        if ((r = c->ensure(c->seg_hits, nseg * 4 + 4, "segments"))) break;
        if ((r = c->ensure(c->hit_off, (nseg + 1) * 8, "segments"))) break;
        if ((r = c->ensure(c->seg_cstart, nseg * 4 + 4, "segments"))) break;
        if ((r = c->ensure(c->seg_ccount, nseg * 4 + 4, "segments"))) break;
        if ((r = c->ensure(c->scan_tmp, scan_tmp_bytes(std::max<uint64_t>(nseg + 1, kDpBins + 1)), "scan"))) break;
        // zero the per-batch counters that size buffers (keep the running totals)
        if ((r = c->cuda(cudaMemsetAsync(ctr + C_NC, 0, sizeof(unsigned long long) * (C_MAXC - C_NC + 1), c->st), "batch: counters"))) break;
        static_assert(C_WIN == C_OVERFLOW + 1, "overflow flag and winner count are cleared together");
        if ((r = c->cuda(cudaMemsetAsync(ctr + C_OVERFLOW, 0, 2 * sizeof(unsigned long long), c->st), "batch: counters"))) break;
        // the count pass leaves the slot of every window (2 x 8 bytes a subject base) for the emit pass
        if ((r = c->ensure(c->wcache, std::max<uint64_t>(nbases, 1) * 16, "probe windows"))) break;
        uint2 *wc = P_<uint2>(c->wcache);
        launch_probe(false, c->p.aln != 0, subj, nsub, q, t, c->p.k, wc, P_<uint32_t>(c->seg_hits), nullptr, nullptr, ctr, c->st);
        launch_scan_u32(P_<uint32_t>(c->seg_hits), P_<uint64_t>(c->hit_off), nseg, c->scan_tmp.p, c->st);
        uint64_t H = 0;
        if (cap) {
            H = bp.H;
        } else {
            if ((r = c->cuda(cudaMemcpyAsync(&H, P_<uint64_t>(c->hit_off) + nseg, 8, cudaMemcpyDeviceToHost, c->st), "hits"))) break;
            if ((r = c->cuda(cudaStreamSynchronize(c->st), "probe count"))) break;
            bp.H = H;
        }
        const uint64_t Hc = std::max<uint64_t>(H, 1);
        if ((r = c->ensure(c->hits, Hc * 8, "hits"))) break;
        launch_probe(true, c->p.aln != 0, subj, nsub, q, t, c->p.k, wc, nullptr, P_<uint64_t>(c->hit_off), P_<uint64_t>(c->hits), ctr, c->st);
        launch_sort_hits(nseg, P_<uint64_t>(c->hit_off), P_<uint64_t>(c->hits), c->st);
        if ((r = c->check_launch("seed"))) break;
        rec(1);
        // chain scratch and outputs (bounds: chains <= hits, keys <= hits, DP <= 2 hits)
        struct {
            DBuf *b;
            size_t per;
        } hb[] = {{&c->cs_grp, 4},     {&c->cs_chain_of, 4}, {&c->cs_first, 4}, {&c->cs_last, 4},
                  {&c->cs_prev, 4},    {&c->cs_size, 4},     {&c->cs_coff, 4},  {&c->cs_ckeys, 4},
                  {&c->cs_kl, 8},      {&c->cs_gnch, 4},     {&c->cs_gbest, 8}, {&c->cs_gkept, 4},
                  {&c->cs_gkeys, 4},   {&c->cs_gdp, 4},      {&c->ch_subj, 4},  {&c->ch_query, 4},
                  {&c->ch_key_off, 4}, {&c->ch_seg_off, 4},  {&c->ch_nkeys, 2}, {&c->ch_nseg, 2},
                  {&c->ch_orient, 1},  {&c->ch_status, 1},   {&c->ch_win, 1},   {&c->ch_rate, 8},
                  {&c->ch_len, 8},     {&c->keys, 4}};
        for (auto &x : hb)
            if ((r = c->ensure(*x.b, Hc * x.per, "chains"))) break;
        if (r) break;
        if ((r = c->ensure(c->segs, 2 * Hc * sizeof(DpSeg), "DP segments"))) break;
        ChainScratch sc{P_<uint32_t>(c->cs_grp),  P_<uint32_t>(c->cs_chain_of), P_<int32_t>(c->cs_first),
                        P_<int32_t>(c->cs_last),  P_<int32_t>(c->cs_prev),      P_<int32_t>(c->cs_size),
                        P_<int32_t>(c->cs_coff),  P_<int32_t>(c->cs_ckeys),     P_<int64_t>(c->cs_kl),
                        P_<int32_t>(c->cs_gnch),  P_<int64_t>(c->cs_gbest),     P_<uint32_t>(c->cs_gkept),
                        P_<uint32_t>(c->cs_gkeys), P_<uint32_t>(c->cs_gdp)};
        ChainArrays ch{P_<uint32_t>(c->ch_subj),   P_<uint32_t>(c->ch_query), P_<uint32_t>(c->ch_key_off),
                       P_<uint32_t>(c->ch_seg_off), P_<uint16_t>(c->ch_nkeys), P_<uint16_t>(c->ch_nseg),
                       P_<uint8_t>(c->ch_orient),  P_<uint8_t>(c->ch_status), P_<uint8_t>(c->ch_win),
                       P_<double>(c->ch_rate),     P_<double>(c->ch_len)};
        launch_chain(c->p, nseg, subj, q, P_<uint64_t>(c->hit_off), P_<uint64_t>(c->hits), sc,
                     P_<uint32_t>(c->seg_cstart), P_<uint32_t>(c->seg_ccount), ch,
                     P_<uint32_t>(c->keys), P_<DpSeg>(c->segs), Hc, Hc, 2 * Hc, ctr, c->st);
        if ((r = c->check_launch("chain"))) break;
        if (!cap) {
            unsigned long long h_ctr[C_COUNT];
            if ((r = c->cuda(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, c->st), "counters"))) break;
            if ((r = c->cuda(cudaStreamSynchronize(c->st), "chain"))) break;
            if (h_ctr[C_OVERFLOW]) {
                r = c->fail(HERO_E_STATE, "chain buffer overflow");
                break;
            }
            bp.NC = h_ctr[C_NC];
            bp.ND = h_ctr[C_ND];
            bp.rmax = int32_t(std::max<unsigned long long>(h_ctr[C_MAXR], 1));
            bp.cmax = int32_t(std::max<unsigned long long>(h_ctr[C_MAXC], 1));
        }
        rec(2);
        const uint64_t NC = bp.NC, ND = bp.ND;
        const int32_t rmax = bp.rmax, cmax = bp.cmax;
        const uint32_t stride = uint32_t((rmax + cmax + 15) / 16);
        const uint64_t NDc = std::max<uint64_t>(ND, 1);
        if ((r = c->ensure(c->sums, NDc * sizeof(DpSum), "DP sums"))) break;
        if ((r = c->ensure(c->cells, NDc * 4, "DP cells"))) break;
        if ((r = c->ensure(c->perm, NDc * 4, "DP order"))) break;
        if ((r = c->ensure(c->ops, NDc * stride * 4, "DP ops"))) break;
        if ((r = c->ensure(c->bins, kDpBins * 4, "DP bins"))) break;
        if ((r = c->ensure(c->bin_off, (kDpBins + 1) * 8, "DP bins"))) break;
        const int32_t nst = (cmax + kStripW - 1) / kStripW;
        if ((r = c->ensure(c->dp_tasks, 128 * 8, "DP tasks"))) break;
        if (dp_needs_scratch(rmax, cmax)) {
            if ((r = c->ensure(c->tb, size_t(c->dp_T) * size_t(rmax) * size_t(nst) * 2, "DP traceback scratch"))) break;
            if ((r = c->ensure(c->bnd, size_t(c->dp_T) * size_t(rmax + 1) * 3 * 4, "DP boundary scratch"))) break;
        }
        launch_dp_sort(P_<DpSeg>(c->segs), ND, P_<uint32_t>(c->bins), P_<uint32_t>(c->perm),
                       P_<uint64_t>(c->bin_off), c->scan_tmp.p, c->st);
        rec(3);
        if (cap) launch_stamp(P_<unsigned long long>(c->stamps) + 2 * c->batch_idx, c->st);
        DpLaunch a{P_<DpSeg>(c->segs), P_<uint32_t>(c->perm), ND, subj.code, subj.off, subj.len,
                   q.code, q.off, P_<uint32_t>(c->ops), stride, P_<DpSum>(c->sums),
                   P_<uint32_t>(c->cells), P_<uint16_t>(c->tb), P_<int32_t>(c->bnd), c->dp_T, rmax,
                   c->p.affine, 1,  // reads with a non-ACGT base never reach the DP
                   0u, 0u, kStripsAll, 4, ctr + C_CELLS_PAIR};
        a.staged = ctr + C_STAGED;
        apply_tuning(c, a);
        launch_dp(a, P_<uint64_t>(c->bin_off), P_<uint64_t>(c->dp_tasks), cmax, c->st);
        if ((r = c->check_launch("dp"))) break;
        rec(4);
        if (cap) launch_stamp(P_<unsigned long long>(c->stamps) + 2 * c->batch_idx + 1, c->st);
        launch_assemble(c->p, NC, ch, P_<uint32_t>(c->keys), subj, q, P_<DpSum>(c->sums),
                        P_<uint32_t>(c->cells), ctr, c->st);
        if (c->p.aln) {
            rec(5);
            if ((r = aln_batch(c, subj, nsub, q, ch, NC, stride))) break;
        } else {
            if ((r = c->ensure(c->winners, std::max<uint64_t>(NC, 1) * 4, "winners"))) break;
            if ((r = c->ensure(c->win_sorted, std::max<uint64_t>(NC, 1) * 4, "winners"))) break;
            if ((r = c->ensure(c->win_bins, kWinScratch * 4, "winners"))) break;
            if (c->mapping) {
                if ((r = c->ensure(c->a_list, std::max<uint64_t>(NC, 1) * 4, "mapping lists"))) break;
                launch_map_choose(c->p, nsub, P_<uint32_t>(c->seg_cstart), P_<uint32_t>(c->seg_ccount),
                                  ch, P_<uint32_t>(c->keys), subj, q, P_<DpSum>(c->sums),
                                  P_<uint32_t>(c->a_list), P_<uint32_t>(c->winners), ctr, c->st);
            } else {
                launch_dedupe(nsub, P_<uint32_t>(c->seg_cstart), P_<uint32_t>(c->seg_ccount), ch,
                              P_<uint32_t>(c->winners), ctr, c->st);
            }
            rec(5);
            launch_vote(c->p, NC, ch, P_<uint32_t>(c->winners), P_<uint32_t>(c->win_sorted),
                        P_<uint32_t>(c->win_bins), P_<uint32_t>(c->keys), subj, q,
                        P_<uint32_t>(c->ops), stride, P_<DpSum>(c->sums), P_<uint32_t>(c->cov),
                        P_<int32_t>(c->mdiff), ctr, c->st);
            if (c->merge)
                launch_vote_overhang(c->p, NC, ch, P_<uint32_t>(c->winners), P_<uint32_t>(c->keys),
                                     subj, q, P_<DpSum>(c->sums), P_<uint32_t>(c->q_ext), ctr, c->st);
        }
        if ((r = c->check_launch("record/vote"))) break;
        if (cap) break;
        rec(6);
        if ((r = c->cuda(cudaStreamSynchronize(c->st), "batch"))) break;
        ms[0] += elapsed(ev[0], ev[1]);
        ms[1] += elapsed(ev[1], ev[2]);
        ms[2] += elapsed(ev[2], ev[4]);
        ms[3] += elapsed(ev[4], ev[5]);
        ms[4] += elapsed(ev[5], ev[6]);
        ms[5] += elapsed(ev[3], ev[4]);
        c->stats.dp_segments += ND;
        c->stats.chains_kept += NC;
    } while (0);
    for (auto &e : ev) cudaEventDestroy(e);
    return r;
}

// off_h: host offsets of the n reads (n + 1 entries), for the batch sizes
static int align_reads(hero_ctx *c, const ReadsView &all, uint64_t n, const uint64_t *off_h) {
    c->consensus_done = false;
    const auto wall0 = std::chrono::steady_clock::now();
    uint64_t B = c->P.subject_batch ? c->P.subject_batch : 131072;
    double ms[6] = {0, 0, 0, 0, 0, 0};
    const size_t nbatch = size_t((n + B - 1) / B);
    if (!c->capturing) c->plan.assign(nbatch, hero_ctx::BatchPlan{0, 0, 0, 1, 1});
    if (c->plan.size() != nbatch) return c->fail(HERO_E_STATE, "plan does not match the reads");
    for (uint64_t b = 0; b < n; b += B) {
        const uint64_t nb = std::min(B, n - b);
        c->batch_idx = size_t(b / B);
        // a batch is a window of the read arrays: shift the per-read pointers
        ReadsView v{all.code, all.off + b,  all.len + b, all.uid + b, all.good + b,
                    nb,       all.job ? all.job + b : nullptr};
        HERO_TRY(align_batch(c, v, nb, off_h[b + nb] - off_h[b], ms));
    }
    if (c->capturing) return HERO_OK;
    c->stats.subjects += n;
    c->stats.ms_seed += ms[0];
    c->stats.ms_chain += ms[1];
    c->stats.ms_dp += ms[2];
    c->stats.ms_record += ms[3];
    c->stats.ms_vote += ms[4];
    c->stats.ms_dp_kernel += ms[5];
    unsigned long long h[C_COUNT];
    HERO_TRY(c->cuda(cudaMemcpy(h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost), "counters"));
    for (int i = 0; i < C_COUNT; i++) c->ctr[i] = h[i];
    c->stats.ms_align_wall +=
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
    return HERO_OK;
}

extern "C" int hero_align_self(hero_ctx *c) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_index) return c->fail(HERO_E_STATE, "index not built");
    cudaSetDevice(c->dev);
    ReadsView v{P_<uint8_t>(c->q_code), P_<uint64_t>(c->q_off), P_<uint32_t>(c->q_len),
                P_<int64_t>(c->q_uid), P_<uint8_t>(c->q_sgood), c->nq, job_tags(c)};
    return align_reads(c, v, c->nq, c->q_off_h.data());
}

extern "C" int hero_align_self_range(hero_ctx *c, uint64_t first, uint64_t count) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_index) return c->fail(HERO_E_STATE, "index not built");
    if (first > c->nq || count > c->nq - first) return c->fail(HERO_E_INPUT, "range outside the query set");
    if (count == 0) return HERO_OK;
    cudaSetDevice(c->dev);
    const uint32_t *job = job_tags(c);
    ReadsView v{P_<uint8_t>(c->q_code), P_<uint64_t>(c->q_off) + first, P_<uint32_t>(c->q_len) + first,
                P_<int64_t>(c->q_uid) + first, P_<uint8_t>(c->q_sgood) + first, count,
                job ? job + first : nullptr};
    return align_reads(c, v, count, c->q_off_h.data() + first);
}

extern "C" int hero_votes_words(hero_ctx *c, uint64_t *words) {
    if (!c || !words) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    *words = c->nqb * 5;
    return HERO_OK;
}

extern "C" int hero_votes_save(hero_ctx *c, void *dst) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->merge) return c->fail(HERO_E_STATE, "the overhang votes of --merge are not part of the exchanged state");
    if (!c->nqb) return HERO_OK;
    if (!dst) return c->fail(HERO_E_INPUT, "null vote buffer");
    cudaSetDevice(c->dev);
    uint8_t *d = static_cast<uint8_t *>(dst);
    HERO_TRY(c->cuda(cudaMemcpyAsync(d, c->cov.p, c->nqb * 16, cudaMemcpyDeviceToDevice, c->st), "votes save"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(d + c->nqb * 16, c->mdiff.p, c->nqb * 4, cudaMemcpyDeviceToDevice, c->st), "votes save"));
    return c->cuda(cudaStreamSynchronize(c->st), "votes save");
}

extern "C" int hero_votes_load(hero_ctx *c, const void *src) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->merge) return c->fail(HERO_E_STATE, "the overhang votes of --merge are not part of the exchanged state");
    if (!c->nqb) return HERO_OK;
    if (!src) return c->fail(HERO_E_INPUT, "null vote buffer");
    cudaSetDevice(c->dev);
    const uint8_t *s = static_cast<const uint8_t *>(src);
    c->consensus_done = false;
    HERO_TRY(c->cuda(cudaMemcpyAsync(c->cov.p, s, c->nqb * 16, cudaMemcpyDeviceToDevice, c->st), "votes load"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(c->mdiff.p, s + c->nqb * 16, c->nqb * 4, cudaMemcpyDeviceToDevice, c->st), "votes load"));
    return c->cuda(cudaStreamSynchronize(c->st), "votes load");
}

extern "C" int hero_set_vote_buffer(hero_ctx *c, void *dev_ptr, uint64_t bytes) {
    if (!c) return HERO_E_INPUT;
    if (c->merge) return c->fail(HERO_E_STATE, "the overhang votes of --merge are not part of the exchanged state");
    if (dev_ptr && (reinterpret_cast<uintptr_t>(dev_ptr) & 255u))
        return c->fail(HERO_E_INPUT, "vote buffer not 256-byte aligned");
    c->vote_ext = dev_ptr;
    c->vote_ext_bytes = dev_ptr ? bytes : 0;
    if (!dev_ptr) {  // back to the context's own buffers at the next hero_set_queries
        if (c->cov.external) c->release(c->cov);
        if (c->mdiff.external) c->release(c->mdiff);
        c->have_queries = false;
        c->have_index = false;
    }
    return HERO_OK;
}

extern "C" int hero_consensus_range(hero_ctx *c, uint64_t first, uint64_t count, uint8_t *seq_out,
                                    uint32_t *imin, uint32_t *imed, uint32_t *imax,
                                    double *mismatch_rate, double *gc_content, uint8_t *good_out) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->p.aln) return c->fail(HERO_E_STATE, "an alignment-output context has no consensus");
    if (first > c->nq || count > c->nq - first) return c->fail(HERO_E_INPUT, "range outside the query set");
    if (count == 0) return HERO_OK;
    cudaSetDevice(c->dev);
    const uint64_t n = c->nq, nb = c->nqb;
    HERO_TRY(c->ensure(c->out_seq, nb, "consensus"));
    HERO_TRY(c->ensure(c->colsum, nb * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imin, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imed, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imax, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_mis, n * 8, "consensus"));
    const uint64_t b0 = c->q_off_h[first], b1 = c->q_off_h[first + count];
    uint8_t *os = P_<uint8_t>(c->out_seq);
    if (b1 > b0)
        HERO_TRY(c->cuda(cudaMemcpyAsync(os + b0, P_<uint8_t>(c->q_raw) + b0, b1 - b0, cudaMemcpyDeviceToDevice, c->st), "consensus"));
    // the reads of the range: per-read arrays shifted, bases and votes absolute
    ReadsView v = query_view(c);
    v.off += first;
    v.len += first;
    v.uid += first;
    v.good += first;
    v.n = count;
    v.job = nullptr;
    launch_consensus(c->p, v, P_<uint32_t>(c->cov), P_<int32_t>(c->mdiff), os, P_<uint32_t>(c->colsum),
                     P_<uint32_t>(c->o_imin) + first, P_<uint32_t>(c->o_imed) + first,
                     P_<uint32_t>(c->o_imax) + first, P_<double>(c->o_mis) + first, c->st);
    HERO_TRY(c->check_launch("consensus"));
    auto d2h = [&](void *dst, const void *src, size_t bytes) {
        return dst && bytes ? c->cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st), "consensus") : HERO_OK;
    };
    HERO_TRY(d2h(seq_out, os + b0, b1 - b0));
    HERO_TRY(d2h(imin, P_<uint32_t>(c->o_imin) + first, count * 4));
    HERO_TRY(d2h(imed, P_<uint32_t>(c->o_imed) + first, count * 4));
    HERO_TRY(d2h(imax, P_<uint32_t>(c->o_imax) + first, count * 4));
    HERO_TRY(d2h(mismatch_rate, P_<double>(c->o_mis) + first, count * 8));
    HERO_TRY(d2h(gc_content, P_<double>(c->q_gc) + first, count * 8));
    HERO_TRY(d2h(good_out, P_<uint8_t>(c->q_good) + first, count));
    return c->cuda(cudaStreamSynchronize(c->st), "consensus");
}

extern "C" int hero_align_subjects(hero_ctx *c, const uint8_t *seq, const uint64_t *off,
                                   const int64_t *uid, uint64_t n) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_index) return c->fail(HERO_E_STATE, "index not built");
    cudaSetDevice(c->dev);
    HERO_TRY(validate_reads(c, seq, off, uid, n));
    if (n == 0) return HERO_OK;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c->st);
    HERO_TRY(upload_reads(c, seq, off, uid, n, c->s_raw, c->s_code, c->s_off, c->s_len, c->s_uid,
                          nullptr, &c->s_good, nullptr));
    cudaEventRecord(e1, c->st);
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "upload subjects"));
    c->stats.ms_upload += elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ReadsView v{P_<uint8_t>(c->s_code), P_<uint64_t>(c->s_off), P_<uint32_t>(c->s_len),
                P_<int64_t>(c->s_uid), P_<uint8_t>(c->s_good), n};
    return align_reads(c, v, n, off);
}

extern "C" int hero_consensus(hero_ctx *c, uint8_t *seq_out, uint32_t *imin, uint32_t *imed,
                              uint32_t *imax, double *mismatch_rate, double *gc_content,
                              uint8_t *good_out) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->p.aln) return c->fail(HERO_E_STATE, "an alignment-output context has no consensus");
    cudaSetDevice(c->dev);
    const uint64_t n = c->nq, nb = c->nqb;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    HERO_TRY(c->ensure(c->out_seq, nb, "consensus"));
    HERO_TRY(c->ensure(c->colsum, nb * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imin, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imed, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imax, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_mis, n * 8, "consensus"));
    cudaEventRecord(e0, c->st);
    if (nb) cudaMemcpyAsync(c->out_seq.p, c->q_raw.p, nb, cudaMemcpyDeviceToDevice, c->st);
    launch_consensus(c->p, query_view(c), P_<uint32_t>(c->cov), P_<int32_t>(c->mdiff),
                     P_<uint8_t>(c->out_seq),
                     P_<uint32_t>(c->colsum), P_<uint32_t>(c->o_imin), P_<uint32_t>(c->o_imed),
                     P_<uint32_t>(c->o_imax), P_<double>(c->o_mis), c->st);
    HERO_TRY(c->check_launch("consensus"));
    cudaEventRecord(e1, c->st);
    if (seq_out && nb) cudaMemcpyAsync(seq_out, c->out_seq.p, nb, cudaMemcpyDeviceToHost, c->st);
    if (imin && n) cudaMemcpyAsync(imin, c->o_imin.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (imed && n) cudaMemcpyAsync(imed, c->o_imed.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (imax && n) cudaMemcpyAsync(imax, c->o_imax.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (mismatch_rate && n) cudaMemcpyAsync(mismatch_rate, c->o_mis.p, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (gc_content && n) cudaMemcpyAsync(gc_content, c->q_gc.p, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (good_out && n) cudaMemcpyAsync(good_out, c->q_good.p, n, cudaMemcpyDeviceToHost, c->st);
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "consensus"));
    c->consensus_done = true;
    c->stats.ms_consensus += elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return HERO_OK;
}

extern "C" int hero_reset_votes(hero_ctx *c) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    cudaSetDevice(c->dev);
    c->consensus_done = false;
    if (c->nqb) HERO_TRY(c->cuda(cudaMemsetAsync(c->cov.p, 0, c->nqb * 16, c->st), "reset votes"));
    if (c->nqb) HERO_TRY(c->cuda(cudaMemsetAsync(c->mdiff.p, 0, c->nqb * 4, c->st), "reset votes"));
    if (c->merge && c->nq)
        HERO_TRY(c->cuda(cudaMemsetAsync(c->q_ext.p, 0, c->nq * kOverhang * 16, c->st), "reset votes"));
    return c->cuda(cudaStreamSynchronize(c->st), "reset votes");
}

// consensus kernel of a round; results stay on the device until hero_fetch
static int consensus_device(hero_ctx *c) {
    const uint64_t n = c->nq, nb = c->nqb;
    HERO_TRY(c->ensure(c->out_seq, nb, "consensus"));
    HERO_TRY(c->ensure(c->colsum, nb * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imin, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imed, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_imax, n * 4, "consensus"));
    HERO_TRY(c->ensure(c->o_mis, n * 8, "consensus"));
    if (nb) cudaMemcpyAsync(c->out_seq.p, c->q_raw.p, nb, cudaMemcpyDeviceToDevice, c->st);
    launch_consensus(c->p, query_view(c), P_<uint32_t>(c->cov), P_<int32_t>(c->mdiff),
                     P_<uint8_t>(c->out_seq), P_<uint32_t>(c->colsum), P_<uint32_t>(c->o_imin),
                     P_<uint32_t>(c->o_imed), P_<uint32_t>(c->o_imax), P_<double>(c->o_mis), c->st);
    c->consensus_done = true;
    return c->check_launch("consensus");
}

// reset + index + align (queries as subjects) + consensus, enqueued on the stream
static int round_body(hero_ctx *c) {
    if (c->nqb) {
        HERO_TRY(c->cuda(cudaMemsetAsync(c->cov.p, 0, c->nqb * 16, c->st), "round: clear votes"));
        HERO_TRY(c->cuda(cudaMemsetAsync(c->mdiff.p, 0, c->nqb * 4, c->st), "round: clear votes"));
    }
    if (c->merge && c->nq)
        HERO_TRY(c->cuda(cudaMemsetAsync(c->q_ext.p, 0, c->nq * kOverhang * 16, c->st), "round: clear votes"));
    HERO_TRY(hero_build_index(c));
    ReadsView v{P_<uint8_t>(c->q_code), P_<uint64_t>(c->q_off), P_<uint32_t>(c->q_len),
                P_<int64_t>(c->q_uid), P_<uint8_t>(c->q_sgood), c->nq, job_tags(c)};
    HERO_TRY(align_reads(c, v, c->nq, c->q_off_h.data()));
    return consensus_device(c);
}

extern "C" int hero_round(hero_ctx *c, uint32_t flags) {
    if (!c) return HERO_E_INPUT;
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->p.aln) return c->fail(HERO_E_STATE, "rounds are correction rounds (consensus mode)");
    cudaSetDevice(c->dev);
    const bool graph = (flags & HERO_ROUND_GRAPH) != 0;
    if (graph && c->gexec && c->plan_ok && c->plan_fp == c->qfp) {
        // the device checks of the eager path, read after the replay: buffers are
        // sized from the plan, so a batch that outgrew it would raise the
        // lifetime overflow count (the per-batch flag is cleared by every batch)
        unsigned long long before[C_COUNT], after[C_COUNT];
        HERO_TRY(c->cuda(cudaMemcpyAsync(before, c->counters.p, sizeof(before), cudaMemcpyDeviceToHost, c->st),
                         "graph round: counters"));
        HERO_TRY(c->cuda(cudaGraphLaunch(c->gexec, c->st), "graph launch"));
        HERO_TRY(c->cuda(cudaMemcpyAsync(after, c->counters.p, sizeof(after), cudaMemcpyDeviceToHost, c->st),
                         "graph round: counters"));
        HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "graph round"));
        for (int i = 0; i < C_COUNT; i++) c->ctr[i] = after[i];
        if (after[C_OVERFLOW_ALL] != before[C_OVERFLOW_ALL]) {
            c->plan_ok = false;  // the next round runs eagerly and re-plans
            return c->fail(HERO_E_STATE, "graph round: chain buffer overflow (plan outgrown)");
        }
        std::vector<unsigned long long> t(2 * c->plan.size());
        HERO_TRY(c->cuda(cudaMemcpy(t.data(), c->stamps.p, t.size() * 8, cudaMemcpyDeviceToHost),
                         "graph stamps"));
        for (size_t b = 0; b < c->plan.size(); b++) {
            c->stats.ms_dp_kernel += double(t[2 * b + 1] - t[2 * b]) * 1e-6;
            c->stats.dp_segments += c->plan[b].ND;
            c->stats.chains_kept += c->plan[b].NC;
        }
        c->stats.subjects += c->nq;
        c->stats.graph_rounds++;
        c->consensus_done = true;
        return HERO_OK;
    }
    // eager round: runs the work and records the per-batch plan
    HERO_TRY(round_body(c));
    HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "round"));
    c->plan_fp = c->qfp;
    c->plan_ok = true;
    if (!graph) return HERO_OK;
    // capture the same round (every size from the plan, no host syncs)
    c->drop_graph();
    HERO_TRY(c->ensure(c->stamps, 16 * c->plan.size(), "stamps"));
    c->capturing = true;
    cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
    int r = e == cudaSuccess ? round_body(c) : c->cuda(e, "begin capture");
    cudaGraph_t g = nullptr;
    cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(c->st, &g) : cudaSuccess;
    c->capturing = false;
    if (r != HERO_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e2 != cudaSuccess) return c->cuda(e2, "end capture");
    c->graph = g;
    HERO_TRY(c->cuda(cudaGraphInstantiate(&c->gexec, c->graph, 0), "graph instantiate"));
    return HERO_OK;
}

extern "C" int hero_fetch(hero_ctx *c, uint8_t *seq_out, uint32_t *imin, uint32_t *imed,
                          uint32_t *imax, double *mismatch_rate, double *gc_content,
                          uint8_t *good_out) {
    if (!c) return HERO_E_INPUT;
    if (!c->consensus_done) return c->fail(HERO_E_STATE, "no consensus to fetch");
    cudaSetDevice(c->dev);
    const uint64_t n = c->nq, nb = c->nqb;
    if (seq_out && nb) cudaMemcpyAsync(seq_out, c->out_seq.p, nb, cudaMemcpyDeviceToHost, c->st);
    if (imin && n) cudaMemcpyAsync(imin, c->o_imin.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (imed && n) cudaMemcpyAsync(imed, c->o_imed.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (imax && n) cudaMemcpyAsync(imax, c->o_imax.p, n * 4, cudaMemcpyDeviceToHost, c->st);
    if (mismatch_rate && n) cudaMemcpyAsync(mismatch_rate, c->o_mis.p, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (gc_content && n) cudaMemcpyAsync(gc_content, c->q_gc.p, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (good_out && n) cudaMemcpyAsync(good_out, c->q_good.p, n, cudaMemcpyDeviceToHost, c->st);
    return c->cuda(cudaStreamSynchronize(c->st), "fetch");
}

extern "C" int hero_merge_pairs(hero_ctx *c, uint8_t *seq_out, uint32_t *merged_len) {
    if (!c) return HERO_E_INPUT;
    if (!c->merge) return c->fail(HERO_E_STATE, "the context was not created with HERO_FLAG_MERGE_PAIRS");
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    if (c->nq % 2) return c->fail(HERO_E_INPUT, "an odd number of reads cannot be paired");
    if (!c->consensus_done) return c->fail(HERO_E_STATE, "no consensus of the current votes yet");
    if (c->nq && (!seq_out || !merged_len)) return c->fail(HERO_E_INPUT, "null output buffer");
    cudaSetDevice(c->dev);
    const uint64_t np = c->nq / 2;
    if (!np) return HERO_OK;
    HERO_TRY(c->ensure(c->m_seq, c->nqb, "merged reads"));
    HERO_TRY(c->ensure(c->m_len, np * 4, "merged reads"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(c->m_seq.p, c->out_seq.p, c->nqb, cudaMemcpyDeviceToDevice, c->st), "merge"));
    launch_merge_pairs(np, P_<uint64_t>(c->q_off), P_<uint8_t>(c->out_seq), P_<uint32_t>(c->q_ext),
                       P_<uint8_t>(c->m_seq), P_<uint32_t>(c->m_len), c->st);
    HERO_TRY(c->check_launch("merge"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(seq_out, c->m_seq.p, c->nqb, cudaMemcpyDeviceToHost, c->st), "merge"));
    HERO_TRY(c->cuda(cudaMemcpyAsync(merged_len, c->m_len.p, np * 4, cudaMemcpyDeviceToHost, c->st), "merge"));
    return c->cuda(cudaStreamSynchronize(c->st), "merge");
}

extern "C" int hero_mapping_histogram(hero_ctx *c, uint64_t *hist, uint64_t cap, uint64_t *n_bins) {
    if (!c || !n_bins || (cap && !hist)) return HERO_E_INPUT;
    if (!c->mapping) return c->fail(HERO_E_STATE, "the context was not created with HERO_FLAG_MAPPING");
    if (!c->have_queries) return c->fail(HERO_E_STATE, "no query set");
    cudaSetDevice(c->dev);
    const ReadsView q = query_view(c);
    uint64_t bins = 1u << 16;
    unsigned long long maxc = 0;
    for (int pass = 0; pass < 2; pass++) {  // a second pass only when a sum exceeds the bins
        HERO_TRY(c->ensure(c->map_hist, bins * 8, "mapping histogram"));
        HERO_TRY(c->ensure(c->map_max, 8, "mapping histogram"));
        HERO_TRY(c->cuda(cudaMemsetAsync(c->map_hist.p, 0, bins * 8, c->st), "mapping histogram"));
        HERO_TRY(c->cuda(cudaMemsetAsync(c->map_max.p, 0, 8, c->st), "mapping histogram"));
        launch_map_hist(q, P_<uint32_t>(c->cov), P_<int32_t>(c->mdiff), bins,
                        P_<unsigned long long>(c->map_hist), P_<unsigned long long>(c->map_max), c->st);
        HERO_TRY(c->check_launch("mapping histogram"));
        HERO_TRY(c->cuda(cudaMemcpyAsync(&maxc, c->map_max.p, 8, cudaMemcpyDeviceToHost, c->st), "mapping histogram"));
        HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "mapping histogram"));
        if (maxc < bins) break;
        bins = maxc + 1;
    }
    *n_bins = c->nqb ? uint64_t(maxc) + 1 : 0;
    const uint64_t m = std::min<uint64_t>(cap, *n_bins);
    if (m) {
        HERO_TRY(c->cuda(cudaMemcpyAsync(hist, c->map_hist.p, m * 8, cudaMemcpyDeviceToHost, c->st), "mapping histogram"));
        HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "mapping histogram"));
    }
    return HERO_OK;
}

extern "C" int hero_get_overhang(hero_ctx *c, uint32_t *out) {
    if (!c || !out) return HERO_E_INPUT;
    if (!c->merge) return c->fail(HERO_E_STATE, "the context was not created with HERO_FLAG_MERGE_PAIRS");
    if (!c->nq) return HERO_OK;
    cudaSetDevice(c->dev);
    HERO_TRY(c->cuda(cudaMemcpyAsync(out, c->q_ext.p, c->nq * kOverhang * 16, cudaMemcpyDeviceToHost, c->st), "overhang"));
    return c->cuda(cudaStreamSynchronize(c->st), "overhang");
}

extern "C" int hero_alignments_size(hero_ctx *c, uint64_t *bytes) {
    if (!c || !bytes) return HERO_E_INPUT;
    if (!c->p.aln) return c->fail(HERO_E_STATE, "not an alignment-output context");
    *bytes = c->aln_host.size();
    return HERO_OK;
}

extern "C" int hero_alignments_take(hero_ctx *c, uint8_t *out, uint64_t cap) {
    if (!c) return HERO_E_INPUT;
    if (!c->p.aln) return c->fail(HERO_E_STATE, "not an alignment-output context");
    const uint64_t n = c->aln_host.size();
    if (cap < n || (n && !out)) return c->fail(HERO_E_INPUT, "output buffer too small");
    if (n) std::memcpy(out, c->aln_host.data(), n);
    std::vector<uint8_t>().swap(c->aln_host);
    return HERO_OK;
}

extern "C" int hero_get_votes(hero_ctx *c, uint32_t *cov) {
    if (!c || !cov) return HERO_E_INPUT;
    cudaSetDevice(c->dev);
    if (!c->nqb) return HERO_OK;
    DBuf tmp;
    int r = c->ensure(tmp, c->nqb * 16, "votes");
    if (r == HERO_OK) {
        launch_expand_votes(query_view(c), P_<uint32_t>(c->cov), P_<int32_t>(c->mdiff),
                            P_<uint32_t>(tmp), c->st);
        r = c->check_launch("votes");
        if (r == HERO_OK)
            r = c->cuda(cudaMemcpyAsync(cov, tmp.p, c->nqb * 16, cudaMemcpyDeviceToHost, c->st), "votes");
        if (r == HERO_OK) r = c->cuda(cudaStreamSynchronize(c->st), "votes");
    }
    c->release(tmp);
    return r;
}

extern "C" int hero_get_stats(hero_ctx *c, hero_stats *out) {
    if (!c || !out) return HERO_E_INPUT;
    cudaSetDevice(c->dev);
    if (c->counters.p) {  // device counters also advance inside graph rounds
        unsigned long long h[C_COUNT];
        HERO_TRY(c->cuda(cudaStreamSynchronize(c->st), "stats"));
        HERO_TRY(c->cuda(cudaMemcpy(h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost), "stats"));
        for (int i = 0; i < C_COUNT; i++) c->ctr[i] = h[i];
    }
    hero_stats s = c->stats;
    s.probes = c->ctr[C_PROBES];
    s.hits = c->ctr[C_HITS];
    s.chains = c->ctr[C_CHAINS];
    s.records_built = c->ctr[C_BUILT];
    s.records_accepted = c->ctr[C_ACCEPTED];
    s.records_kept = c->ctr[C_KEPT];
    s.dp_segments_ref = c->ctr[C_DP_REF];
    s.dp_cells = c->ctr[C_CELLS];
    s.dp_cells_computed = c->ctr[C_CELLS_ALL];
    s.dp_cells_pairs = c->ctr[C_CELLS_PAIR];
    s.dp_tasks_staged = c->ctr[C_STAGED];
    s.dp_stage_timeouts = c->ctr[C_STAGE_FAIL];
    s.dp_rows_max = c->ctr[C_MAXR];
    s.vote_anomalies = c->ctr[C_ANOMALY];
    s.device_bytes_peak = c->bytes_peak;
    s.kernel_launches = kernel_launches();
    *out = s;
    return HERO_OK;
}

extern "C" int hero_align_segments(hero_ctx *c, int affine, const uint8_t *subj,
                                   const uint64_t *subj_off, uint64_t n_subj,
                                   const uint8_t *query, const uint64_t *query_off,
                                   uint64_t n_query, uint64_t n_seg, const uint32_t *seg_subject,
                                   const uint8_t *seg_orient, const uint32_t *seg_query,
                                   const int32_t *s0, const int32_t *s1, const int32_t *q0,
                                   const int32_t *q1, const uint8_t *seg_flags,
                                   const int64_t *band, const uint64_t *ops_off, uint8_t *ops,
                                   int32_t *nops) {
    if (!c) return HERO_E_INPUT;
    cudaSetDevice(c->dev);
    if (n_seg == 0) return HERO_OK;
    std::vector<int64_t> no_uid(std::max(n_subj, n_query), 0);
    HERO_TRY(validate_reads(c, subj, subj_off, no_uid.data(), n_subj));
    HERO_TRY(validate_reads(c, query, query_off, no_uid.data(), n_query));
    std::vector<DpSeg> h(n_seg);
    int32_t rmax = 1, cmax = 1;
    for (uint64_t i = 0; i < n_seg; i++) {
        if (seg_subject[i] >= n_subj || seg_query[i] >= n_query)
            return c->fail(HERO_E_INPUT, "segment read index out of range");
        const int64_t ls_read = int64_t(subj_off[seg_subject[i] + 1] - subj_off[seg_subject[i]]);
        const int64_t lq_read = int64_t(query_off[seg_query[i] + 1] - query_off[seg_query[i]]);
        if (s0[i] < 0 || s1[i] <= s0[i] || s1[i] > ls_read || q0[i] < 0 || q1[i] <= q0[i] ||
            q1[i] > lq_read)
            return c->fail(HERO_E_INPUT, "segment range out of the read");
        if (ops_off[i + 1] - ops_off[i] < uint64_t((s1[i] - s0[i]) + (q1[i] - q0[i])))
            return c->fail(HERO_E_INPUT, "ops capacity too small");
        DpSeg g;
        g.subj = seg_subject[i];
        g.query = seg_query[i];
        g.s0 = uint16_t(s0[i]);
        g.s1 = uint16_t(s1[i]);
        g.q0 = uint16_t(q0[i]);
        g.q1 = uint16_t(q1[i]);
        g.band = int32_t(band[i] > 65535 ? 65535 : (band[i] < 0 ? 0 : band[i]));
        g.flags = (seg_flags[i] & 3u) | (uint32_t(seg_orient[i] & 1u) << kSegOrientShift);
        g.pad = 0;
        h[i] = g;
        const int32_t ls = s1[i] - s0[i], lq = q1[i] - q0[i];
        rmax = std::max(rmax, std::max(ls, lq));
        cmax = std::max(cmax, std::min(ls, lq));
    }
    const uint32_t stride = uint32_t((rmax + cmax + 15) / 16);
    // the whole-band rows score only A/C/G/T; other bases take the general rows
    bool acgt = true;
    for (const auto &rd : {std::make_pair(subj, subj_off[n_subj]), std::make_pair(query, query_off[n_query])})
        for (uint64_t k = 0; k < rd.second && acgt; k++) acgt = base_code(rd.first[k]) < 4;
    DBuf sraw, scode, soff, slen, suid, qraw, qcode, qoff, qlen, quid, dsegs, dsums, dops, dtb, dbnd,
        doo, dout, dn, dperm, dbins, dbinoff, dtasks, dtmp;
    auto cleanup = [&]() {
        for (DBuf *b : {&sraw, &scode, &soff, &slen, &suid, &qraw, &qcode, &qoff, &qlen, &quid,
                        &dsegs, &dsums, &dops, &dtb, &dbnd, &doo, &dout, &dn, &dperm, &dbins,
                        &dbinoff, &dtasks, &dtmp})
            c->release(*b);
    };
    int r = HERO_OK;
    do {
        if ((r = upload_reads(c, subj, subj_off, no_uid.data(), n_subj, sraw, scode, soff, slen, suid,
                              nullptr, nullptr, nullptr)))
            break;
        if ((r = upload_reads(c, query, query_off, no_uid.data(), n_query, qraw, qcode, qoff, qlen,
                              quid, nullptr, nullptr, nullptr)))
            break;
        const int32_t nst = (cmax + kStripW - 1) / kStripW;
        if ((r = c->ensure(dsegs, n_seg * sizeof(DpSeg), "segments"))) break;
        if ((r = c->ensure(dsums, n_seg * sizeof(DpSum), "segments"))) break;
        if ((r = c->ensure(dops, n_seg * stride * 4, "segments"))) break;
        if (dp_needs_scratch(rmax, cmax)) {
            if ((r = c->ensure(dtb, size_t(c->dp_T) * rmax * nst * 2, "scratch"))) break;
            if ((r = c->ensure(dbnd, size_t(c->dp_T) * (rmax + 1) * 3 * 4, "scratch"))) break;
        }
        if ((r = c->ensure(dperm, n_seg * 4, "order"))) break;
        if ((r = c->ensure(dbins, kDpBins * 4, "bins"))) break;
        if ((r = c->ensure(dbinoff, (kDpBins + 1) * 8, "bins"))) break;
        if ((r = c->ensure(dtasks, 128 * 8, "tasks"))) break;
        if ((r = c->ensure(dtmp, scan_tmp_bytes(kDpBins + 1), "scan"))) break;
        if ((r = c->ensure(doo, (n_seg + 1) * 8, "ops"))) break;
        if ((r = c->ensure(dout, ops_off[n_seg], "ops"))) break;
        if ((r = c->ensure(dn, n_seg * 4, "ops"))) break;
        cudaMemcpyAsync(dsegs.p, h.data(), n_seg * sizeof(DpSeg), cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(doo.p, ops_off, (n_seg + 1) * 8, cudaMemcpyHostToDevice, c->st);
        launch_dp_sort(P_<DpSeg>(dsegs), n_seg, P_<uint32_t>(dbins), P_<uint32_t>(dperm),
                       P_<uint64_t>(dbinoff), dtmp.p, c->st);
        DpLaunch a{P_<DpSeg>(dsegs), P_<uint32_t>(dperm), n_seg, P_<uint8_t>(scode), P_<uint64_t>(soff),
                   P_<uint32_t>(slen), P_<uint8_t>(qcode), P_<uint64_t>(qoff), P_<uint32_t>(dops),
                   stride, P_<DpSum>(dsums), nullptr, P_<uint16_t>(dtb), P_<int32_t>(dbnd),
                   c->dp_T, rmax, affine ? 1 : 0, acgt ? 1 : 0, 0u, 0u, kStripsAll, 4};
        apply_tuning(c, a);
        launch_dp(a, P_<uint64_t>(dbinoff), P_<uint64_t>(dtasks), cmax, c->st);
        launch_unpack_ops(P_<uint32_t>(dops), stride, P_<DpSum>(dsums), n_seg, P_<uint64_t>(doo),
                          P_<uint8_t>(dout), P_<int32_t>(dn), c->st);
        if ((r = c->check_launch("align segments"))) break;
        cudaMemcpyAsync(ops, dout.p, ops_off[n_seg], cudaMemcpyDeviceToHost, c->st);
        cudaMemcpyAsync(nops, dn.p, n_seg * 4, cudaMemcpyDeviceToHost, c->st);
        r = c->cuda(cudaStreamSynchronize(c->st), "align segments");
    } while (0);
    cleanup();
    return r;
}
