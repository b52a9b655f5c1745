// hero_server.cu -- serving form: many independent correction jobs on one GPU.
//
// The reference corrects one read set per process (main.cpp:36-104).  A server
// runs a stream of such jobs with continuous batching.  Two worker threads,
// each owning a context with its own stream, run correction rounds; a worker
// that is free admits the oldest queued jobs that fit in the device-memory
// budget left by the rounds already in flight.  So while one round's kernels
// run, the other worker gathers and uploads the next round's reads, and it
// downloads its results while the next round runs: host work and copies
// overlap device work.  The device phases themselves pass a gate (may_compute):
// a small round may run beside a large one, so a job arriving during a long
// round is not held up for all of it, while two small or two large rounds take
// the device in turn.  Inside a round the admitted jobs' reads are concatenated
// into one query set whose reads carry their job (hero_set_query_jobs), so one
// set of launches -- index build, seeding, chaining, DP, votes, consensus --
// serves every job of the round, and a job's k-mers only ever meet its own
// reads: each job's output is the output it gets alone.  A round's results
// stay in one host block that its jobs share, each job reading its own slice,
// until every job of the round is released.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <sys/mman.h>

#include <cuda_runtime.h>

#include "../../include/hero_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

// Host array left uninitialised (results are written over it by the device
// copy; zero-filling GBs first would cost as much as the copy).  Arrays of 2 MB
// and more sit on 2 MB-aligned memory advised for huge pages: the first touch
// of a GB-sized array -- the driver's copy of a round's results, a job's reads
// copied in at submission -- then takes 512x fewer page faults.
template <class T>
struct HostArray {
    static constexpr size_t kHuge = size_t(2) << 20;
    T *p = nullptr;
    size_t n = 0;
    HostArray() = default;
    HostArray(const HostArray &) = delete;
    HostArray &operator=(const HostArray &) = delete;
    HostArray(HostArray &&o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    HostArray &operator=(HostArray &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~HostArray() { release(); }
    void release() {
        std::free(p);
        p = nullptr;
        n = 0;
    }
    bool alloc(size_t k) {
        release();
        if (!k) return true;
        const size_t b = k * sizeof(T);
        void *q = nullptr;
        if (b >= kHuge) {
            const size_t rb = (b + kHuge - 1) & ~(kHuge - 1);
            if (posix_memalign(&q, kHuge, rb) != 0) return false;
            madvise(q, rb, MADV_HUGEPAGE);  // advice only: without it the array still works
        } else if (!(q = std::malloc(b))) {
            return false;
        }
        p = static_cast<T *>(q);
        n = k;
        return true;
    }
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
    T *data() const { return p; }
    T &operator[](size_t i) const { return p[i]; }
    T back() const { return p[n - 1]; }
};

// One round's results, shared by its jobs: each job reads its own slice, so a
// round's output is never split or copied before a caller fetches it.
struct RoundOut {
    HostArray<uint8_t> seq, good;
    HostArray<uint32_t> imin, imed, imax;
    HostArray<double> mis, gc;
};

struct Job {
    uint64_t id = 0;
    int32_t state = HERO_JOB_QUEUED, status = HERO_OK;
    std::string err;
    HostArray<uint8_t> seq;   // freed when the job's round ends
    HostArray<uint64_t> off;
    HostArray<int64_t> uid;
    uint64_t bases = 0;
    uint64_t bytes = 0;  // admission estimate
    // results: a slice of the round's output (reads [out_read, +n), bases [out_base, +bases))
    std::shared_ptr<const RoundOut> out;
    uint64_t out_read = 0, out_base = 0;
    uint64_t round = 0;
    uint32_t round_jobs = 0;
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    uint64_t n() const { return uid.size(); }
};

// memcpy spread over a few threads (a round's reads and results are up to GBs)
void copy_parallel(void *dst, const void *src, size_t bytes) {
    constexpr size_t kChunk = size_t(16) << 20;
    const size_t nt = std::min<size_t>(8, (bytes + kChunk - 1) / kChunk);
    if (nt <= 1) {
        if (bytes) std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (size_t t = 0; t < nt; t++) {
        const size_t a = t * per, b = std::min(bytes, a + per);
        if (a < b)
            th.emplace_back([=] { std::memcpy(static_cast<uint8_t *>(dst) + a, static_cast<const uint8_t *>(src) + a, b - a); });
    }
    for (auto &x : th) x.join();
}

}  // namespace

// Round policy defaults, measured on the serving stream (jobs of 0.2-30 Mbp and
// of 10 Mbp-1.6 Gbp): rounds of up to ~8 Mbp beyond their first job, and 64 Mbp
// as the line between small and large rounds for the device-phase gate (two
// device phases side by side lost 3-18 % against taking turns; a small round
// still runs beside a large one, so it is not held up for all of it).
constexpr uint64_t kRoundBasesDefault = 8000000;
constexpr uint64_t kOverlapBasesDefault = 64000000;

// rounds that may be in flight at once (one context and worker thread each)
#ifndef HERO_SERVE_WORKERS
#define HERO_SERVE_WORKERS 2
#endif
constexpr int kServeWorkers = HERO_SERVE_WORKERS;

struct hero_server {
    hero_params p{};
    hero_ctx *ctx[kServeWorkers] = {};
    uint64_t round_bytes = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Job> jobs;
    std::thread worker[kServeWorkers];
    bool stop = false;
    uint64_t next_id = 1, rounds = 0, submitted = 0, done = 0, failed = 0, bases_done = 0;
    uint64_t max_jobs = 0;   // jobs a key can tell apart (k-mer bits leave room for the job)
    uint64_t cap_jobs = 0;   // jobs per round after a round ran out of memory (0: no cap)
    std::vector<hero_dp_tuning> tuning;  // DP kernel shapes to apply before the next round
    uint64_t tuning_gen = 0;             // bumped by every hero_server_set_dp_tuning
    uint64_t in_flight_bytes = 0;        // admission estimates of the rounds running
    int in_flight = 0;                   // rounds running
    bool exclusive = false;              // the queue head needs the device to itself
    double busy_ms = 0, busy_since = 0;  // time with at least one round in flight
    uint64_t overlapped_rounds = 0;      // rounds that started while another ran
    // round policy (hero_server_set_round_policy)
    uint64_t round_bases_max = kRoundBasesDefault;      // bases a round admits beyond its first job
    uint64_t overlap_bases_max = kOverlapBasesDefault;  // small / large line of the device-phase gate
    uint64_t running_bases[kServeWorkers] = {};         // bases of each worker's round in flight
    uint64_t computing[kServeWorkers] = {};             // bases of each worker's round in its device phase
    uint64_t overlapped_compute = 0;                    // device phases started beside another
    std::condition_variable cv_gate;
    double ms_stage_in = 0, ms_round_calls = 0, ms_stage_out = 0;  // worker wall time, all rounds
    hero_stats ctx_stats[kServeWorkers] = {};  // each worker context's statistics after its last round

    // The device phase of a round (index, seeding, alignment, votes, consensus)
    // may start beside another only if one of the two rounds is within the
    // overlap limit and the other above it: two small rounds or two large ones
    // run their device phases one after the other (side by side they only share
    // the SMs and the L2, and lose against running in turn), while a small round
    // beside a large one is not held up for the whole large round.  Uploads and
    // downloads are outside the gate: they overlap the other round's device phase.
    bool may_compute(int w, uint64_t bases) const {
        for (int v = 0; v < kServeWorkers; v++) {
            if (v == w || !computing[v] || !overlap_bases_max) continue;
            if ((bases <= overlap_bases_max) == (computing[v] <= overlap_bases_max)) return false;
        }
        return true;
    }
    bool large_running() const {  // a round above the overlap limit is in flight
        for (int v = 0; v < kServeWorkers; v++)
            if (running_bases[v] > overlap_bases_max) return true;
        return false;
    }
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    }
    void run(int w);
    void run_round(int w, std::vector<uint64_t> ids, uint64_t bytes);
    void round_begin(uint64_t bytes);  // with mu held
    void round_end(uint64_t bytes);    // with mu held
};

void hero_server::round_begin(uint64_t bytes) {
    if (in_flight == 0) busy_since = now_ms();
    else overlapped_rounds++;
    in_flight++;
    in_flight_bytes += bytes;
}

void hero_server::round_end(uint64_t bytes) {
    in_flight--;
    in_flight_bytes -= bytes;
    if (in_flight == 0) busy_ms += now_ms() - busy_since;
}

extern "C" uint64_t hero_job_bytes(uint64_t bases, uint64_t reads, int32_t k) {
    // per base: read copies and codes (2), vote matrix (16 + 4), corrected bases (1);
    // per read: offsets, lengths, ids, flags, GC, job, statistics and index
    // temporaries (~70); per k-mer key (one every k bases, plus a tail key per
    // read): table slots at <= 4 per key plus build temporaries (~260).  Device
    // buffers grow with 25 % slack.
    const uint64_t kk = k > 0 ? uint64_t(k) : 39u;
    const uint64_t keys = bases / kk + reads;
    const uint64_t raw = 24u * bases + 70u * reads + 260u * keys;
    return raw + raw / 4 + 4096u;
}

extern "C" uint64_t hero_round_admit(const uint64_t *bytes, uint64_t n_queued, uint64_t round_bytes) {
    if (n_queued == 0) return 0;
    uint64_t sum = 0, n = 0;
    while (n < n_queued && (n == 0 || sum + bytes[n] <= round_bytes)) sum += bytes[n++];
    return n;
}

void hero_server::run(int w) {
    uint64_t my_tuning_gen = 0;
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        // admissible: the queue head fits the budget the running rounds leave
        // (a head that needs the device to itself waits for every round to end)
        auto admissible = [&] {
            if (queue.empty()) return false;
            if (in_flight == 0) return true;
            if (exclusive) return false;
            const Job &head = jobs[queue.front()];
            if (in_flight_bytes + head.bytes > round_bytes) return false;
            return true;
        };
        cv_work.wait(lk, [&] { return stop || admissible(); });
        if (stop) break;
        const uint64_t room = in_flight == 0 ? round_bytes : round_bytes - in_flight_bytes;
        std::vector<uint64_t> sizes;
        for (uint64_t id : queue) sizes.push_back(jobs[id].bytes);
        uint64_t take = hero_round_admit(sizes.data(), sizes.size(), room);
        take = std::min(take, max_jobs);
        if (cap_jobs) take = std::min(take, cap_jobs);
        // bases beyond the first job: the round limit, and beside a large
        // round the overlap limit (the round must stay small)
        uint64_t cap_bases = round_bases_max ? round_bases_max : ~0ull;
        if (in_flight && overlap_bases_max && large_running()) cap_bases = std::min(cap_bases, overlap_bases_max);
        {
            uint64_t nb = 0, t = 0;
            for (uint64_t id : queue) {
                if (t >= take) break;
                const uint64_t jb = jobs[id].bases;
                if (t > 0 && nb + jb > cap_bases) break;
                nb += jb;
                t++;
            }
            take = t;
        }
        std::vector<uint64_t> ids(queue.begin(), queue.begin() + long(take));
        queue.erase(queue.begin(), queue.begin() + long(take));
        exclusive = false;
        uint64_t bytes = 0, bases = 0;
        const double t = now_ms();
        for (uint64_t id : ids) {
            jobs[id].state = HERO_JOB_RUNNING;
            jobs[id].start_ms = t;
            bytes += jobs[id].bytes;
            bases += jobs[id].bases;
        }
        round_begin(bytes);
        running_bases[w] = bases;
        std::vector<hero_dp_tuning> tun;
        const bool retune = tuning_gen != my_tuning_gen;
        if (retune) {
            tun = tuning;
            my_tuning_gen = tuning_gen;
        }
        lk.unlock();
        cv_work.notify_all();  // the other worker may admit what is left
        if (retune) hero_set_dp_tuning(ctx[w], tun.data(), uint32_t(tun.size()));
        run_round(w, ids, bytes);
        lk.lock();
        running_bases[w] = 0;
        cv_done.notify_all();
        cv_work.notify_all();
    }
    // jobs still queued at shutdown fail (the first worker to get here fails them)
    for (uint64_t id : queue) {
        Job &j = jobs[id];
        j.err = "server stopped";
        j.status = HERO_E_STATE;
        j.state = HERO_JOB_FAILED;
        failed++;
    }
    queue.clear();
    cv_done.notify_all();
}

// One round over the given jobs on worker w's context (the worker owns it; job
// inputs are not touched by other threads while the job is running).
void hero_server::run_round(int w, std::vector<uint64_t> ids, uint64_t round_est) {
    hero_ctx *ctx = this->ctx[w];
    std::vector<Job *> js;
    {
        std::lock_guard<std::mutex> g(mu);
        for (uint64_t id : ids) js.push_back(&jobs[id]);
    }
    // jobs in order of their longest read: subject batches then hold reads of
    // similar length (a job's reads only meet its own), so each batch's DP
    // launch is shaped for its own segments rather than the round's longest
    auto longest = [](const Job *j) {
        uint64_t m = 0;
        for (size_t i = 0; i + 1 < j->off.size(); i++) m = std::max(m, j->off[i + 1] - j->off[i]);
        return m;
    };
    std::vector<std::pair<uint64_t, size_t>> order;
    for (size_t t = 0; t < js.size(); t++) order.push_back({longest(js[t]), t});
    std::stable_sort(order.begin(), order.end());
    {
        std::vector<Job *> js2;
        std::vector<uint64_t> ids2;
        for (const auto &o : order) {
            js2.push_back(js[o.second]);
            ids2.push_back(ids[o.second]);
        }
        js.swap(js2);
        ids.swap(ids2);
    }
    uint64_t n = 0, nb = 0;
    for (Job *j : js) {
        n += j->n();
        nb += j->bases;
    }
    // one job: its own buffers go up as they are; several: concatenated
    // (reads | offsets | ids | job tags), each read carrying its job
    HostArray<uint8_t> cat_seq;
    HostArray<uint64_t> cat_off;
    HostArray<int64_t> cat_uid;
    HostArray<uint32_t> cat_tag;
    const uint8_t *seq = js[0]->seq.data();
    const uint64_t *off = js[0]->off.data();
    const int64_t *uid = js[0]->uid.data();
    const double t_in = now_ms();
    bool host_ok = true;
    if (js.size() > 1) {
        host_ok = cat_seq.alloc(nb) && cat_off.alloc(n + 1) && cat_uid.alloc(n) && cat_tag.alloc(n);
    }
    if (js.size() > 1 && host_ok) {
        uint64_t r = 0, b = 0;
        cat_off.p[0] = 0;
        for (size_t t = 0; t < js.size(); t++) {
            const Job &j = *js[t];
            copy_parallel(cat_seq.data() + b, j.seq.data(), j.bases);
            for (uint64_t i = 0; i < j.n(); i++) {
                cat_off.p[r + i + 1] = b + j.off[i + 1];
                cat_uid.p[r + i] = j.uid[i];
                cat_tag.p[r + i] = uint32_t(t);
            }
            r += j.n();
            b += j.bases;
        }
        seq = cat_seq.data();
        off = cat_off.data();
        uid = cat_uid.data();
    }
    auto out = std::make_shared<RoundOut>();
    host_ok = host_ok && out->seq.alloc(nb) && out->good.alloc(n) && out->imin.alloc(n) &&
              out->imed.alloc(n) && out->imax.alloc(n) && out->mis.alloc(n) && out->gc.alloc(n);
    const double t_calls = now_ms();
    int st = host_ok ? hero_set_queries(ctx, seq, off, uid, n) : HERO_E_OOM;
    if (st == HERO_OK && js.size() > 1) st = hero_set_query_jobs(ctx, cat_tag.data(), n);
    if (st == HERO_OK) {
        {  // the device phase, through the gate
            std::unique_lock<std::mutex> lk(mu);
            cv_gate.wait(lk, [&] { return may_compute(w, nb); });
            for (int v = 0; v < kServeWorkers; v++)
                if (v != w && computing[v]) {
                    overlapped_compute++;
                    break;
                }
            computing[w] = nb;
        }
        st = hero_build_index(ctx);
        if (st == HERO_OK) st = hero_align_self(ctx);
        // results stay on the device until the fetch below, outside the gate
        if (st == HERO_OK) st = hero_consensus(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        {
            std::lock_guard<std::mutex> g(mu);
            computing[w] = 0;
        }
        cv_gate.notify_all();
    }
    if (st == HERO_OK)
        st = hero_fetch(ctx, out->seq.data(), out->imin.data(), out->imed.data(), out->imax.data(),
                        out->mis.data(), out->gc.data(), out->good.data());
    const double t_out = now_ms();
    const std::string err = st == HERO_OK ? std::string()
                            : host_ok ? std::string(hero_last_error(ctx))
                                      : std::string("host memory for the round's reads or results not available");
    if (st == HERO_OK) {  // each job's slice of the round's output (nobody reads a running job)
        uint64_t r = 0, b = 0;
        for (Job *j : js) {
            j->out = out;
            j->out_read = r;
            j->out_base = b;
            r += j->n();
            b += j->bases;
        }
    }
    hero_stats cs{};
    const bool have_cs = hero_get_stats(ctx, &cs) == HERO_OK;
    const double t_done = now_ms();
    std::lock_guard<std::mutex> g(mu);
    if (have_cs) ctx_stats[w] = cs;
    ms_stage_in += t_calls - t_in;
    ms_round_calls += t_out - t_calls;
    ms_stage_out += t_done - t_out;
    if (st == HERO_E_OOM && (js.size() > 1 || in_flight > 1)) {
        // the estimate was short, or another round held the memory: requeue the
        // jobs in order, then admit half as many (one job: with the device to itself)
        for (size_t t = js.size(); t-- > 0;) {
            js[t]->state = HERO_JOB_QUEUED;
            queue.push_front(ids[t]);
        }
        if (js.size() > 1) cap_jobs = js.size() / 2;
        else exclusive = true;
        round_end(round_est);
        return;
    }
    if (st == HERO_OK && cap_jobs) cap_jobs *= 2;
    rounds++;
    const double t_end = now_ms();
    round_end(round_est);
    for (Job *j : js) {
        const uint64_t jb = j->bases;
        j->round = rounds;
        j->round_jobs = uint32_t(js.size());
        j->done_ms = t_end;
        if (st == HERO_OK) {
            j->state = HERO_JOB_DONE;
            done++;
            bases_done += jb;
        } else {
            j->err = err;
            j->status = st;
            j->state = HERO_JOB_FAILED;
            failed++;
        }
        // the reads are no longer needed (offsets and ids stay for the job's info)
        j->seq.release();
    }
}

extern "C" int hero_server_create(const hero_params *p, uint64_t round_bytes, hero_server **out) {
    if (!p || !out) return HERO_E_INPUT;
    *out = nullptr;
    hero_server *s = new hero_server();
    s->p = *p;
    s->p.stream = nullptr;  // every worker context creates its own stream
    s->t0 = Clock::now();
    for (int w = 0; w < kServeWorkers; w++) {
        const int st = hero_create(&s->p, &s->ctx[w]);
        if (st != HERO_OK) {
            for (int v = 0; v < w; v++) hero_destroy(s->ctx[v]);
            delete s;
            return st;
        }
    }
    if (round_bytes == 0) {
        // per-batch working set of each worker (hits, chains, DP segments of one
        // subject batch)
        const uint64_t reserve = 12ull << 30;
        uint64_t budget = p->device_memory_budget;
        if (!budget) {
            size_t fr = 0, tot = 0;
            cudaSetDevice(p->device);
            if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
                for (int w = 0; w < kServeWorkers; w++) hero_destroy(s->ctx[w]);
                delete s;
                return HERO_E_CUDA;
            }
            budget = uint64_t(double(fr) * 0.8);
        }
        const uint64_t res = kServeWorkers * reserve;
        round_bytes = budget > 2 * res ? budget - res : budget / 2;
    }
    s->round_bytes = round_bytes;
    // job tags share a 128-bit key with the 2k k-mer bits (hero_set_query_jobs)
    const int free_bits = 2 * p->k <= 64 ? 32 : std::min(32, 128 - 2 * p->k);
    s->max_jobs = free_bits >= 32 ? 0xffffffffull : (1ull << free_bits);
    for (int w = 0; w < kServeWorkers; w++) s->worker[w] = std::thread([s, w] { s->run(w); });
    *out = s;
    return HERO_OK;
}

extern "C" void hero_server_destroy(hero_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (int w = 0; w < kServeWorkers; w++)
        if (s->worker[w].joinable()) s->worker[w].join();
    for (int w = 0; w < kServeWorkers; w++) hero_destroy(s->ctx[w]);
    delete s;
}

extern "C" int hero_server_set_round_policy(hero_server *s, uint64_t round_bases_max,
                                            uint64_t overlap_bases_max) {
    if (!s) return HERO_E_INPUT;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->round_bases_max = round_bases_max;
        s->overlap_bases_max = overlap_bases_max;
    }
    s->cv_work.notify_all();
    return HERO_OK;
}

extern "C" int hero_server_set_dp_tuning(hero_server *s, const hero_dp_tuning *t, uint32_t n) {
    if (!s || hero_dp_tuning_check(t, n) != HERO_OK) return HERO_E_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    s->tuning.assign(t, t + n);
    s->tuning_gen++;
    return HERO_OK;
}

extern "C" int hero_job_submit(hero_server *s, const uint8_t *seq, const uint64_t *off,
                               const int64_t *uid, uint64_t n, uint64_t *job_id) {
    if (!s || !job_id || (n && (!seq || !off || !uid))) return HERO_E_INPUT;
    if (n && off[0] != 0) return HERO_E_INPUT;
    for (uint64_t i = 0; i < n; i++)
        if (off[i + 1] < off[i] || off[i + 1] - off[i] > 32767) return HERO_E_INPUT;
    Job j;
    const uint64_t nb = n ? off[n] : 0;
    if (!j.seq.alloc(nb) || !j.off.alloc(n + 1) || !j.uid.alloc(n)) return HERO_E_OOM;
    copy_parallel(j.seq.data(), seq, nb);
    if (n) {
        copy_parallel(j.off.data(), off, (n + 1) * sizeof(uint64_t));
        copy_parallel(j.uid.data(), uid, n * sizeof(int64_t));
    } else {
        j.off[0] = 0;
    }
    j.bases = nb;
    j.bytes = hero_job_bytes(nb, n, s->p.k);
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return HERO_E_STATE;
    j.id = s->next_id++;
    j.submit_ms = s->now_ms();
    *job_id = j.id;
    s->submitted++;
    if (n == 0) {  // nothing to correct
        j.state = HERO_JOB_DONE;
        j.start_ms = j.done_ms = j.submit_ms;
        s->done++;
        s->jobs.emplace(j.id, std::move(j));
        s->cv_done.notify_all();
        return HERO_OK;
    }
    const uint64_t id = j.id;
    s->jobs.emplace(id, std::move(j));
    s->queue.push_back(id);
    s->cv_work.notify_one();
    return HERO_OK;
}

static void fill_info(const Job &j, hero_job_info *info) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->state = j.state;
    info->status = j.status;
    info->round = j.round;
    info->round_jobs = j.round_jobs;
    info->bases = j.off.empty() ? 0 : j.off.back();
    info->reads = j.n();
    info->submit_ms = j.submit_ms;
    info->start_ms = j.start_ms;
    info->done_ms = j.done_ms;
}

extern "C" int hero_job_poll(hero_server *s, uint64_t job_id, hero_job_info *info) {
    if (!s) return HERO_E_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return HERO_E_INPUT;
    fill_info(it->second, info);
    return HERO_OK;
}

extern "C" int hero_job_wait(hero_server *s, uint64_t job_id, int64_t timeout_ms,
                             hero_job_info *info) {
    if (!s) return HERO_E_INPUT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto finished = [&] {
        auto it = s->jobs.find(job_id);
        return it == s->jobs.end() || it->second.state == HERO_JOB_DONE ||
               it->second.state == HERO_JOB_FAILED;
    };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, finished);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished)) {
        auto it = s->jobs.find(job_id);
        if (it != s->jobs.end()) fill_info(it->second, info);
        return HERO_E_TIMEOUT;
    }
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return HERO_E_INPUT;
    fill_info(it->second, info);
    return HERO_OK;
}

extern "C" int hero_job_result(hero_server *s, uint64_t job_id, uint8_t *seq_out, uint32_t *imin,
                               uint32_t *imed, uint32_t *imax, double *mismatch_rate,
                               double *gc_content, uint8_t *good_out) {
    if (!s) return HERO_E_INPUT;
    std::shared_ptr<const RoundOut> out;
    uint64_t r = 0, b = 0, n = 0, nb = 0;
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->jobs.find(job_id);
        if (it == s->jobs.end()) return HERO_E_INPUT;
        const Job &j = it->second;
        if (j.state == HERO_JOB_FAILED) return j.status;
        if (j.state != HERO_JOB_DONE) return HERO_E_STATE;
        out = j.out;
        r = j.out_read;
        b = j.out_base;
        n = j.n();
        nb = j.off.empty() ? 0 : j.off.back();
    }
    if (!out || n == 0) return HERO_OK;  // a job without reads has no output
    // the copy runs outside the lock (the shared slice outlives a concurrent release)
    auto put = [](auto *dst, const auto &a, uint64_t at, uint64_t k) {
        if (dst && k) std::memcpy(dst, a.data() + at, k * sizeof(a.data()[0]));
    };
    put(seq_out, out->seq, b, nb);
    put(imin, out->imin, r, n);
    put(imed, out->imed, r, n);
    put(imax, out->imax, r, n);
    put(mismatch_rate, out->mis, r, n);
    put(gc_content, out->gc, r, n);
    put(good_out, out->good, r, n);
    return HERO_OK;
}

extern "C" const char *hero_job_error(hero_server *s, uint64_t job_id) {
    if (!s) return "";
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(job_id);
    // the worker writes err before it marks the job failed and never after, so
    // the string is stable from then until hero_job_release frees the job
    if (it == s->jobs.end() || it->second.state != HERO_JOB_FAILED) return "";
    return it->second.err.c_str();
}

extern "C" int hero_job_release(hero_server *s, uint64_t job_id) {
    if (!s) return HERO_E_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return HERO_E_INPUT;
    if (it->second.state != HERO_JOB_DONE && it->second.state != HERO_JOB_FAILED)
        return HERO_E_STATE;
    s->jobs.erase(it);
    return HERO_OK;
}

extern "C" int hero_server_get_stats(hero_server *s, hero_server_stats *out) {
    if (!s || !out) return HERO_E_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    out->jobs_submitted = s->submitted;
    out->jobs_done = s->done;
    out->jobs_failed = s->failed;
    out->rounds = s->rounds;
    out->bases_done = s->bases_done;
    out->round_bytes_budget = s->round_bytes;
    out->busy_ms = s->busy_ms + (s->in_flight ? s->now_ms() - s->busy_since : 0.0);
    out->uptime_ms = s->now_ms();
    out->overlapped_rounds = s->overlapped_rounds;
    out->overlapped_compute = s->overlapped_compute;
    out->ms_stage_in = s->ms_stage_in;
    out->ms_round_calls = s->ms_round_calls;
    out->ms_stage_out = s->ms_stage_out;
    out->buffer_allocs = 0;
    out->ms_alloc = 0;
    for (int w = 0; w < kServeWorkers; w++) {
        out->buffer_allocs += s->ctx_stats[w].buffer_allocs;
        out->ms_alloc += s->ctx_stats[w].ms_alloc;
    }
    return HERO_OK;
}

extern "C" int hero_server_worker_stats(hero_server *s, int32_t worker, hero_stats *out) {
    if (!s || !out || worker < 0) return HERO_E_INPUT;
    if (worker >= kServeWorkers) return HERO_E_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    *out = s->ctx_stats[worker];
    return HERO_OK;
}

extern "C" int32_t hero_server_workers(void) { return kServeWorkers; }
