// hero_server.cu -- serving form: many independent correction jobs on one GPU.
//
// The reference corrects one read set per process (main.cpp:36-104).  A server
// runs a stream of such jobs with continuous batching.  Two worker threads,
// each owning a context with its own stream, run correction rounds; a worker
// that is free admits the oldest queued jobs that fit in the device-memory
// budget left by the rounds already in flight.  So while one round's kernels
// run, the other worker concatenates and uploads the next round's reads and
// starts it: rounds overlap on the device (their launches share the SMs), host
// preparation overlaps device work, and a job that arrives while a long round
// runs is admitted as soon as a worker and memory are free instead of waiting
// for that round.  Inside a round the admitted jobs' reads are concatenated
// into one query set whose reads carry their job (hero_set_query_jobs), so one
// set of launches -- index build, seeding, chaining, DP, votes, consensus --
// serves every job of the round, and a job's k-mers only ever meet its own
// reads: each job's output is the output it gets alone.  Results are split
// back per job and kept until released.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/hero_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    int32_t state = HERO_JOB_QUEUED, status = HERO_OK;
    std::string err;
    std::vector<uint8_t> seq;
    std::vector<uint64_t> off;
    std::vector<int64_t> uid;
    uint64_t bytes = 0;  // admission estimate
    // results
    std::vector<uint8_t> out_seq, good;
    std::vector<uint32_t> imin, imed, imax;
    std::vector<double> mis, gc;
    uint64_t round = 0;
    uint32_t round_jobs = 0;
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    uint64_t n() const { return uid.size(); }
};

// Host memory a worker stages a round in: page-locked, so the uploads and
// downloads run at the link's speed, and reused from round to round (grown,
// never shrunk).
struct Staging {
    uint8_t *p = nullptr;
    size_t cap = 0;
    bool ensure(size_t need) {
        if (need <= cap) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = need + need / 4 + 4096;
        if (cudaHostAlloc(reinterpret_cast<void **>(&p), want, cudaHostAllocDefault) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        cap = want;
        return true;
    }
    ~Staging() {
        if (p) cudaFreeHost(p);
    }
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

// rounds that may be in flight at once (one context and worker thread each)
constexpr int kServeWorkers = 2;

struct hero_server {
    hero_params p{};
    hero_ctx *ctx[kServeWorkers] = {};
    Staging stage[kServeWorkers];  // each worker's round inputs and outputs
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
            return in_flight_bytes + jobs[queue.front()].bytes <= round_bytes;
        };
        cv_work.wait(lk, [&] { return stop || admissible(); });
        if (stop) break;
        const uint64_t room = in_flight == 0 ? round_bytes : round_bytes - in_flight_bytes;
        std::vector<uint64_t> sizes;
        for (uint64_t id : queue) sizes.push_back(jobs[id].bytes);
        uint64_t take = hero_round_admit(sizes.data(), sizes.size(), room);
        take = std::min(take, max_jobs);
        if (cap_jobs) take = std::min(take, cap_jobs);
        std::vector<uint64_t> ids(queue.begin(), queue.begin() + long(take));
        queue.erase(queue.begin(), queue.begin() + long(take));
        exclusive = false;
        uint64_t bytes = 0;
        const double t = now_ms();
        for (uint64_t id : ids) {
            jobs[id].state = HERO_JOB_RUNNING;
            jobs[id].start_ms = t;
            bytes += jobs[id].bytes;
        }
        round_begin(bytes);
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
        nb += j->seq.size();
    }
    // the round's reads and results staged in the worker's page-locked
    // buffer: reads | offsets | ids | job tags, then corrected bases | good |
    // imin | imed | imax | mismatch rate | GC
    Staging &sg = stage[w];
    const size_t off_at = (nb + 7) & ~size_t(7);
    const size_t in_bytes = off_at + 8 * (n + 1) + 8 * n + 4 * n;
    const size_t out_at = (in_bytes + 255) & ~size_t(255);
    const size_t out_bytes = nb + n + 12 * n + 16 * n + 64;
    int st = sg.ensure(out_at + out_bytes) ? HERO_OK : HERO_E_OOM;
    uint8_t *seq = sg.p;
    uint64_t *off = reinterpret_cast<uint64_t *>(sg.p + off_at);
    int64_t *uid = reinterpret_cast<int64_t *>(off + n + 1);
    uint32_t *tag = reinterpret_cast<uint32_t *>(uid + n);
    uint8_t *o_seq = sg.p + out_at;
    uint8_t *o_good = o_seq + nb;
    // 8-byte alignment for the doubles: after the bytes, round up
    uint8_t *o_u32 = o_good + n;
    while (reinterpret_cast<uintptr_t>(o_u32) & 7u) o_u32++;
    uint32_t *o_imin = reinterpret_cast<uint32_t *>(o_u32), *o_imed = o_imin + n, *o_imax = o_imed + n;
    uint8_t *o_d = reinterpret_cast<uint8_t *>(o_imax + n);
    while (reinterpret_cast<uintptr_t>(o_d) & 7u) o_d++;
    double *o_mis = reinterpret_cast<double *>(o_d), *o_gc = o_mis + n;
    if (st == HERO_OK) {
        uint64_t r = 0, b = 0;
        off[0] = 0;
        for (size_t t = 0; t < js.size(); t++) {
            const Job &j = *js[t];
            copy_parallel(seq + b, j.seq.data(), j.seq.size());
            for (uint64_t i = 0; i < j.n(); i++) {
                off[r + i + 1] = b + j.off[i + 1];
                uid[r + i] = j.uid[i];
                tag[r + i] = uint32_t(t);
            }
            r += j.n();
            b += j.seq.size();
        }
        st = hero_set_queries(ctx, seq, off, uid, n);
        if (st == HERO_OK && js.size() > 1) st = hero_set_query_jobs(ctx, tag, n);
        if (st == HERO_OK) st = hero_build_index(ctx);
        if (st == HERO_OK) st = hero_align_self(ctx);
        if (st == HERO_OK) st = hero_consensus(ctx, o_seq, o_imin, o_imed, o_imax, o_mis, o_gc, o_good);
    }
    const std::string err = st == HERO_OK ? std::string()
                            : (sg.p ? std::string(hero_last_error(ctx))
                                    : std::string("page-locked staging memory not available"));
    if (st == HERO_OK) {  // results into the jobs, before the lock (nobody reads a running job)
        uint64_t r = 0, b = 0;
        for (Job *j : js) {
            const uint64_t jn = j->n(), jb = j->seq.size();
            j->out_seq.resize(jb);
            copy_parallel(j->out_seq.data(), o_seq + b, jb);
            j->good.assign(o_good + r, o_good + r + jn);
            j->imin.assign(o_imin + r, o_imin + r + jn);
            j->imed.assign(o_imed + r, o_imed + r + jn);
            j->imax.assign(o_imax + r, o_imax + r + jn);
            j->mis.assign(o_mis + r, o_mis + r + jn);
            j->gc.assign(o_gc + r, o_gc + r + jn);
            r += jn;
            b += jb;
        }
    }
    std::lock_guard<std::mutex> g(mu);
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
        const uint64_t jb = j->seq.size();
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
        // inputs are no longer needed
        std::vector<uint8_t>().swap(j->seq);
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

extern "C" int hero_server_set_dp_tuning(hero_server *s, const hero_dp_tuning *t, uint32_t n) {
    if (!s || (n && !t)) return HERO_E_INPUT;
    for (uint32_t i = 0; i < n; i++)
        if ((t[i].warps_per_block != 1 && t[i].warps_per_block != 2 && t[i].warps_per_block != 4) ||
            (t[i].regs_per_thread != 0 && t[i].regs_per_thread != 128 && t[i].regs_per_thread != 168))
            return HERO_E_INPUT;
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
    j.seq.assign(seq, seq + nb);
    j.off.assign(off, off + n + 1);
    if (!n) j.off.assign(1, 0);
    j.uid.assign(uid, uid + n);
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
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return HERO_E_INPUT;
    const Job &j = it->second;
    if (j.state == HERO_JOB_FAILED) return j.status;
    if (j.state != HERO_JOB_DONE) return HERO_E_STATE;
    auto put = [](auto *dst, const auto &v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    put(seq_out, j.out_seq);
    put(imin, j.imin);
    put(imed, j.imed);
    put(imax, j.imax);
    put(mismatch_rate, j.mis);
    put(gc_content, j.gc);
    put(good_out, j.good);
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
    return HERO_OK;
}
