/*
 * hero_gpu.h -- C ABI of the B200 read-correction path (HERO consensus mode,
 * its alignment output and paired-read merging).
 *
 * The reference (guo-xuan/Hero) has no plugin or FFI layer: its hot path is a
 * set of C++ classes driven from main.cpp.  These entry points replace the
 * calls main.cpp makes on those classes, one for one:
 *
 *   hero_create           Config statics read by the aligner
 *                         (Config.h:88-145; SubjectReadAligner.cpp:10-22)
 *   hero_set_queries      QueryDataset::buildDataset / loadDatasetParallel
 *                         (QueryDataset.cpp:89-244; main.cpp:36-50) -- reads
 *                         already parsed on the host, uploaded once
 *   hero_build_index      HashTableMethod::createHashTables + insertQueryDataset
 *                         (HashTableLongKey.cpp:41-68, 250-306; main.cpp:60-66)
 *   hero_align_subjects   SubjectReadAligner::start over one chunk of subject
 *                         reads (SubjectReadAligner.cpp:493-645); votes accumulate
 *   hero_align_self       the same with the query set as the subject set (HERO is
 *                         run with -q X -s X for correction)
 *   hero_reset_votes      QueryRead::initilizeCoverageMatrix (QueryRead.cpp:100-115)
 *   hero_consensus        QueryDataset::callConsensus (QueryDataset.cpp:393-412)
 *                         plus the fields QueryDataset::writeQueryOut prints
 *                         (QueryDataset.cpp:414-537)
 *   hero_round            one whole correction round (plain, or the batched
 *                         form replayed as a CUDA graph); hero_fetch its results
 *   hero_get_stats        the per-phase timers the reference prints
 *                         (SubjectReadAligner.cpp:635-640) and work counters
 *   hero_alignments_size / _take
 *                         SubjectReadAligner::writeToFile of HERO run without -c
 *                         (SubjectReadAligner.cpp:854-906; HERO_FLAG_ALIGNMENT_OUTPUT)
 *   hero_merge_pairs      QueryDataset::mergePairedReads of --merge
 *                         (QueryDataset.cpp:539-558; HERO_FLAG_MERGE_PAIRS)
 *   hero_align_self_range, hero_set_vote_buffer, hero_consensus_range
 *                         one correction split across devices by subject reads
 *                         (SubjectReadAligner::start's chunks on several GPUs),
 *                         each owner's slice of the votes reduced to it
 *                         (hero_votes_save / _load: the whole state instead)
 *   hero_mapping_histogram
 *                         the coverage histogram of -c --mapping
 *                         (QueryDataset::getCoverageAndWriteResults,
 *                         QueryDataset.cpp:560-600; HERO_FLAG_MAPPING)
 *   hero_server_*, hero_job_*
 *                         serving: independent correction jobs (one main.cpp
 *                         run each) with continuous batching on one device
 *
 * Conventions: plain pointers and sizes only; host buffers belong to the
 * caller and are only read during the call.  Every call returns 0 or a
 * negative HERO_E_* code; hero_last_error() gives the message.  A context is
 * bound to one CUDA device and one stream and is not re-entrant.
 */
#ifndef HERO_GPU_H_
#define HERO_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HERO_OK 0
#define HERO_E_INPUT (-1)   /* bad argument or read set */
#define HERO_E_OOM (-2)     /* device memory budget exceeded */
#define HERO_E_CUDA (-3)    /* CUDA runtime error */
#define HERO_E_STATE (-4)   /* call out of order (e.g. align before index) */
#define HERO_E_TIMEOUT (-5) /* a bounded device wait gave up */

#define HERO_ALIGNER_AFFINE 0 /* BandAligner::IAFFINE, flag -a a */
#define HERO_ALIGNER_GLOBAL 1 /* BandAligner::IGLOBAL, default */

typedef struct hero_ctx hero_ctx;

/* Alignment-output mode: HERO run without -c.  The aligner keeps one record per
 * (subject, query uniqueId) and writes them as the .aln file
 * (SubjectReadAligner::writeToFile, SubjectReadAligner.cpp:854-906); the
 * reverse-complement pass aligns the query's reverse complement to the forward
 * subject (SubjectReadAligner.cpp:199-210, 477-481).  No votes, no consensus:
 * hero_align_subjects / hero_align_self append each subject's text, and
 * hero_alignments_size / hero_alignments_take return it. */
#define HERO_FLAG_ALIGNMENT_OUTPUT 1u

/* --merge (consensus mode only): the votes also fill each query read's
 * overhang matrix -- the subject bases past the end of every kept record of
 * more than one CIGAR entry, 20 columns (SubjectRead::
 * updateQueryCoverageConsiderMerging, SubjectRead.cpp:332-462) -- and after the
 * consensus hero_merge_pairs merges reads (2i, 2i+1) as
 * QueryDataset::mergePairedReads does (QueryDataset.cpp:539-558). */
#define HERO_FLAG_MERGE_PAIRS 2u

/* --mapping (with -c): per subject, of the records SubjectRead::addAlignment
 * keeps, only those SubjectRead::chooseQueryWithBestAlignment keeps vote
 * (SubjectRead.cpp:463-500; SubjectReadAligner.cpp:556-561): no record that
 * covers the whole subject -- none; exactly one -- all of the subject's
 * records; two or more -- the covering one with the fewest substitutions.
 * hero_mapping_histogram then gives QueryDataset::getCoverageAndWriteResults'
 * histogram (QueryDataset.cpp:560-599).  Reads keep HERO's own limit of this
 * path, shorter than 32768 bases. */
#define HERO_FLAG_MAPPING 4u

typedef struct {
    int32_t k;              /* k-mer length, 1..63 (Config::iKmer, -k; default 39) */
    int32_t min_overlap;    /* Config::minimumOverlapLength, -l (default 40) */
    int32_t aligner;        /* HERO_ALIGNER_GLOBAL or HERO_ALIGNER_AFFINE (-a) */
    int32_t device;         /* CUDA device ordinal */
    double max_mismatch_rate; /* Config::dMaxMismatchRate = atof(-m)/100 (default 1) */
    double max_indel_rate;    /* Config::dMaxIndelRate = atof(-i)/100 (default 1) */
    double consensus_threshold; /* Config::dMinFrequencyCallConsensus, -c (default 0.6) */
    uint64_t device_memory_budget; /* bytes this context may hold; 0 = no limit */
    uint32_t subject_batch; /* subject reads per device batch; 0 = default */
    uint32_t flags;         /* HERO_FLAG_* (0 = consensus mode, -c) */
    void *stream;           /* cudaStream_t to run on; NULL = a private stream */
} hero_params;

typedef struct {
    uint64_t queries, good_queries, index_keys, index_slots;
    uint64_t subjects, probes, hits, chains, chains_kept;
    uint64_t records_built, records_accepted, records_kept;
    uint64_t dp_segments;      /* DP segments computed on the device */
    uint64_t dp_segments_ref;  /* of those, the ones the reference would compute */
    uint64_t dp_cells;         /* band cells of the reference's loop bounds, ref segments */
    uint64_t vote_anomalies;   /* votes outside a read (reference: undefined behaviour) */
    uint64_t device_bytes_peak;
    uint64_t kernel_launches;  /* kernels this process launched through the library */
    double ms_upload, ms_index, ms_seed, ms_chain, ms_dp, ms_record, ms_vote, ms_consensus;
    double ms_dp_kernel;       /* device time of the DP kernels alone */
    double ms_align_wall;      /* host wall time inside the align calls */
    uint64_t graph_rounds;     /* rounds replayed from a CUDA graph */
    uint64_t dp_cells_computed; /* band cells of every DP segment computed on the device */
    uint64_t dp_rows_max;      /* longest DP side (the row count of a segment) seen so far;
                                  the key of hero_dp_tuning classes */
    uint64_t dp_cells_pairs;   /* of dp_cells_computed, the cells computed as 16-bit pairs */
    uint64_t buffer_allocs;    /* device buffers grown (allocated stream-ordered) */
    double ms_alloc;           /* host time spent growing device buffers */
    uint64_t dp_tasks_staged;  /* DP wavefront tasks whose row bases the bulk copy engine
                                  staged in shared memory */
    uint64_t dp_stage_timeouts; /* staging waits that ran out (those rows were read from
                                   global memory instead; results are unaffected) */
} hero_stats;

/* Returns the default parameters of the reference's Config. */
void hero_default_params(hero_params *p);
/* Creates the CUDA context of a device ahead of the first context (the first
 * CUDA call of a process pays it, often a second or more): a caller may run it
 * on a thread of its own while it parses its input.  HERO_OK, or HERO_E_CUDA
 * when the device cannot be opened.  Thread-safe; later calls return at once. */
int hero_device_init(int32_t device);

int hero_create(const hero_params *p, hero_ctx **out);
void hero_destroy(hero_ctx *ctx);
const char *hero_last_error(const hero_ctx *ctx);

/* Query reads: seq holds the concatenated bases (uppercase ASCII, as
 * QueryDataset stores them after toupper), read i is seq[off[i]..off[i+1]);
 * uid[i] = atoi(read name).  Replaces any previous query set and resets votes. */
int hero_set_queries(hero_ctx *ctx, const uint8_t *seq, const uint64_t *off, const int64_t *uid,
                     uint64_t n);

int hero_build_index(hero_ctx *ctx);

/* One chunk of subject reads (same layout).  May be called repeatedly; the
 * votes of every chunk accumulate, as SubjectReadAligner::start streams chunks. */
int hero_align_subjects(hero_ctx *ctx, const uint8_t *seq, const uint64_t *off,
                        const int64_t *uid, uint64_t n);

/* The query set itself as the subject set, without a second upload. */
int hero_align_self(hero_ctx *ctx);

/* The query reads [first, first + count) as the subject set: one shard of
 * hero_align_self, for a correction split across devices by subject reads
 * (each device aligns its range against the whole query table; the votes of
 * all ranges add up to hero_align_self's). */
int hero_align_self_range(hero_ctx *ctx, uint64_t first, uint64_t count);

/* Vote state for the exchange between contexts that aligned different subject
 * reads against the same query set: hero_votes_words gives its size in 32-bit
 * words (5 per query base: mismatch votes [bases][4], then the match-run
 * difference array [bases]); it is additive -- the element-wise sum of the
 * shards' states (integer addition mod 2^32) is the state of the whole run.
 * hero_votes_save copies it to, and hero_votes_load replaces it from, a
 * buffer in this context's device memory owned by the caller (e.g. the
 * buffer of an NCCL all-reduce); both return once the copy is done.  Contexts
 * created with HERO_FLAG_MERGE_PAIRS refuse both (HERO_E_STATE): their overhang
 * votes are not part of this state. */
int hero_votes_words(hero_ctx *ctx, uint64_t *words);
int hero_votes_save(hero_ctx *ctx, void *dev_dst);
int hero_votes_load(hero_ctx *ctx, const void *dev_src);

/* Keeps the vote state in caller-owned memory of this context's device, laid
 * out as hero_votes_words describes (bytes >= 20 per query base, 256-byte
 * aligned): from the next hero_set_queries on, the context votes there instead
 * of into its own buffers, so shards can add their states in place (one NCCL
 * reduce of each owner's slice to its owner, no copies).  The buffer must
 * outlive its use; NULL returns to the context's own buffers (the query set
 * must then be set again).  HERO_FLAG_MERGE_PAIRS contexts refuse it.  No
 * reference counterpart (HERO runs on one host). */
int hero_set_vote_buffer(hero_ctx *ctx, void *dev_ptr, uint64_t bytes);

/* QueryDataset::callConsensus (QueryDataset.cpp:393-412) for the query reads
 * [first, first + count) only, once their votes are complete (a shard that
 * owns those reads): outputs as hero_consensus's, holding just those reads
 * (seq_out from the range's first base). */
int hero_consensus_range(hero_ctx *ctx, uint64_t first, uint64_t count, uint8_t *seq_out,
                         uint32_t *imin, uint32_t *imed, uint32_t *imax, double *mismatch_rate,
                         double *gc_content, uint8_t *good_out);

/* Clears the vote matrix for a new correction of the same query set, as
 * QueryRead::initilizeCoverageMatrix zeroes it at load (QueryRead.cpp:100-115). */
int hero_reset_votes(hero_ctx *ctx);

/* Consensus over the accumulated votes.  seq_out has the query layout; bases of
 * reads that are not good are left untouched (the reference leaves them as
 * read).  Any output pointer may be NULL.  good_out[i] = 1 for a good read. */
int hero_consensus(hero_ctx *ctx, uint8_t *seq_out, uint32_t *imin, uint32_t *imed,
                   uint32_t *imax, double *mismatch_rate, double *gc_content,
                   uint8_t *good_out);

/* One correction round over the resident query set (main.cpp:60-104: table,
 * aligner with the query set as subjects, consensus); results stay on the
 * device until hero_fetch.  flags: HERO_ROUND_GRAPH = the batched form -- the
 * first round runs eagerly and records every batch's sizes, then the whole
 * round is captured as one CUDA graph; later rounds over the same reads (checked
 * by a device fingerprint taken in hero_set_queries) replay the graph, with no
 * host synchronisation inside the round.  0 = the plain form, one launch per
 * stage with host-sized buffers. */
#define HERO_ROUND_GRAPH 1u
int hero_round(hero_ctx *ctx, uint32_t flags);

/* Results of the last round, or of the last hero_consensus (whose NULL outputs
 * stay on the device until fetched here); same outputs as hero_consensus. */
int hero_fetch(hero_ctx *ctx, uint8_t *seq_out, uint32_t *imin, uint32_t *imed, uint32_t *imax,
               double *mismatch_rate, double *gc_content, uint8_t *good_out);

/* --merge, after hero_consensus (or hero_round): merges every pair of query
 * reads (2p, 2p+1) (QueryRead::mergingPairedReads, QueryRead.cpp:268-319).
 * seq_out has the query layout: pair p's merged read is written from the pair's
 * first base and merged_len[p] is its length; a pair that does not merge keeps
 * both corrected reads and merged_len[p] = 0.  An odd read count is refused. */
int hero_merge_pairs(hero_ctx *ctx, uint8_t *seq_out, uint32_t *merged_len);
/* --merge: the overhang votes, uint32 [query reads][20][4] (A,C,T,G). */
int hero_get_overhang(hero_ctx *ctx, uint32_t *out);

/* Alignment-output mode: bytes of .aln text held (every subject aligned since the
 * last take, in subject order: ">uniqueId\n", its records
 * "queryUniqueId,orientation,position,CIGAR,inserted bases," (AlignmentRecord::
 * getCigar, AlignmentRecord.cpp:102-149), "\n"). */
int hero_alignments_size(hero_ctx *ctx, uint64_t *bytes);
/* Copies the held text to out (cap >= hero_alignments_size) and drops it. */
int hero_alignments_take(hero_ctx *ctx, uint8_t *out, uint64_t cap);

/* Vote matrix before the self vote: uint32 [total query bases][4] (A,C,T,G). */
int hero_get_votes(hero_ctx *ctx, uint32_t *cov);

int hero_get_stats(hero_ctx *ctx, hero_stats *out);

/* Shapes of the banded-DP kernel per class of subject batch, chosen by the
 * project's autotuner (hero_b200/autotune.py: it times each candidate on a
 * sample of a workload and records the fastest per class in a JSON file that
 * the Python binding loads).  A batch whose longest DP side is at most
 * rows_max takes the first such class; batches no class covers, and contexts
 * without a table, use 4 warps a block, no pairs and row-chunk walks for every
 * strip count.  No reference counterpart (the reference has one CPU aligner). */
typedef struct {
    int32_t rows_max;          /* class bound on the longest DP side of a batch */
    int32_t warps_per_block;   /* 1, 2 or 4 */
    uint32_t pair_strips;      /* bit n: n-strip segments run as 16-bit pairs */
    uint32_t chunk_strips;     /* bit n: n-strip tracebacks walk in row chunks */
    int32_t regs_per_thread;   /* 0 or 128 (16 warps an SM), 168 (12 warps, fewer spills),
                                  or 255 with 1-warp blocks (8 warps, no spills) */
} hero_dp_tuning;

/* Replaces the context's tuning table (n = 0 clears it). */
int hero_set_dp_tuning(hero_ctx *ctx, const hero_dp_tuning *t, uint32_t n);
/* Checks a tuning table the way hero_set_dp_tuning and
 * hero_server_set_dp_tuning do (HERO_OK or HERO_E_INPUT), without a context. */
int hero_dp_tuning_check(const hero_dp_tuning *t, uint32_t n);

/* Aligns an explicit list of DP segments on the device (test and tooling entry
 * point).  subj/query: concatenated reads (same layout as above); per segment
 * the subject read index, its orientation (0 forward, 1 reverse complement),
 * the query read index, half-open ranges [s0,s1) and [q0,q1), flags (1 = align
 * right, 2 = align left) and the band the aligner holds before the call.
 * Outputs: ops (per-step codes 0=M 1=X 2=I 3=D, first to last) written at
 * ops_off[i] (caller sizes ops_off[i+1]-ops_off[i] >= (s1-s0)+(q1-q0)); nops[i]
 * receives the path length. */
int hero_align_segments(hero_ctx *ctx, int affine, const uint8_t *subj, const uint64_t *subj_off,
                        uint64_t n_subj, const uint8_t *query, const uint64_t *query_off,
                        uint64_t n_query, uint64_t n_seg, const uint32_t *seg_subject,
                        const uint8_t *seg_orient, const uint32_t *seg_query,
                        const int32_t *s0, const int32_t *s1, const int32_t *q0,
                        const int32_t *q1, const uint8_t *seg_flags, const int64_t *band,
                        const uint64_t *ops_off, uint8_t *ops, int32_t *nops);

/* Allocation-free form of hero_align_segments, for callers that cannot
 * allocate device memory (code inside a host framework that owns the GPU's
 * allocator, or a fixed memory plan that forbids new allocations).  It has no
 * counterpart in the reference.  Every pointer is caller-owned DEVICE memory:
 * the reads as uppercase ASCII with their offsets, the per-segment arrays of
 * hero_align_segments, ops_off/ops/nops for the results (ops per step, 0=M
 * 1=X 2=I 3=D, first to last, at ops_off[i]).  It needs no context, calls no
 * cudaMalloc/cudaFree and uses one fixed working array of about 48 MB that the
 * library keeps on every device where it has run, until the process exits.
 * Limits: max_side (the caller's bound on either side of any segment) must be
 * 1..128, else HERO_E_INPUT before any launch; a segment beyond 128 on a side,
 * outside its read, with too little ops room or with ops_off[i+1] < ops_off[i]
 * gets nops[i] = -1 and the call returns HERO_E_INPUT.  The first call on a
 * device looks up the working array's address: make it before any stream
 * capture (a lookup that fails is retried by the next call).  Calls share the array,
 * so calls that overlap on the GPU (other streams, other host threads) race;
 * the call runs on `stream` and returns after it has completed. */
int hero_align_segments_noalloc(int affine, const uint8_t *subj, const uint64_t *subj_off,
                                uint64_t n_subj, const uint8_t *query, const uint64_t *query_off,
                                uint64_t n_query, uint64_t n_seg, const uint32_t *seg_subject,
                                const uint8_t *seg_orient, const uint32_t *seg_query,
                                const int32_t *s0, const int32_t *s1, const int32_t *q0,
                                const int32_t *q1, const uint8_t *seg_flags, const int64_t *band,
                                int32_t max_side, const uint64_t *ops_off, uint8_t *ops,
                                int32_t *nops, void *stream);

/* --mapping: coverage histogram of the current votes (QueryDataset::
 * getCoverageAndWriteResults, QueryDataset.cpp:560-599).  hist[c] = the number
 * of query bases whose four vote counts sum to c (no self vote), for
 * c = 0 .. *n_bins - 1, where *n_bins is the largest sum + 1.  Copies
 * min(cap, *n_bins) entries (hist may be NULL with cap 0 to learn *n_bins).
 * The writer prints "COV\tFRE" and "c\thist[c]" for every c with hist[c] > 0.
 * Needs a context created with HERO_FLAG_MAPPING (else HERO_E_STATE). */
int hero_mapping_histogram(hero_ctx *ctx, uint64_t *hist, uint64_t cap, uint64_t *n_bins);

/* ------------------------------------------------------------------------
 * Serving: many independent correction jobs (each its own -q X -s X run)
 * corrected together.  No reference counterpart: HERO runs one job per
 * process.  These build on the single-job calls above.
 * ------------------------------------------------------------------------ */

/* Tags each read of the current query set with its job (job[i] for read i) so
 * that one round corrects several independent jobs: a read's k-mers only meet
 * reads of its own job, so every job's output equals its output alone.  The
 * job index must fit beside the k-mer in a 128-bit key (below 2^(128-2k), and
 * below 2^32).  Cleared by hero_set_queries; only the self alignment
 * (hero_align_self, hero_round) honours the tags. */
int hero_set_query_jobs(hero_ctx *ctx, const uint32_t *job, uint64_t n);

typedef struct hero_server hero_server;

#define HERO_JOB_QUEUED 0
#define HERO_JOB_RUNNING 1
#define HERO_JOB_DONE 2
#define HERO_JOB_FAILED 3

typedef struct {
    int32_t state;        /* HERO_JOB_* */
    int32_t status;       /* HERO_OK, or the error that failed the job */
    uint64_t round;       /* round that corrected the job (1-based; 0 = not yet) */
    uint32_t round_jobs;  /* jobs corrected in that round */
    uint32_t reserved;
    uint64_t bases, reads;
    double submit_ms, start_ms, done_ms; /* server clock (ms since creation) */
} hero_job_info;

typedef struct {
    uint64_t jobs_submitted, jobs_done, jobs_failed, rounds, bases_done;
    uint64_t round_bytes_budget; /* admission limit of one round (estimated device bytes) */
    double busy_ms;              /* wall time with at least one round in flight */
    double uptime_ms;
    uint64_t overlapped_rounds;  /* rounds started while another round ran */
    /* worker wall time summed over rounds: staging the round's reads (host
       copies), the round's library calls (upload, index, alignment, consensus
       and the download of results), and splitting results back to the jobs */
    double ms_stage_in, ms_round_calls, ms_stage_out;
    uint64_t buffer_allocs;      /* device buffers the workers' contexts have grown */
    double ms_alloc;             /* host time the workers spent growing them */
    uint64_t overlapped_compute; /* rounds whose device phase started beside another's */
} hero_server_stats;

/* A server owns two contexts on p->device, each with its own stream and worker
 * thread (continuous batching with overlapping rounds: one round's upload and
 * download run while the other round is on the device).  A free worker admits
 * the oldest queued jobs whose estimated device memory (hero_job_bytes) fits in
 * what the rounds in flight leave of round_bytes (0 = p->device_memory_budget,
 * or 80 % of the device's free memory at creation, minus each worker's
 * per-batch working set); a job larger than round_bytes runs in a round of its
 * own once no other round is in flight.  p->stream is ignored.  All jobs of a
 * server share p's parameters. */
int hero_server_create(const hero_params *p, uint64_t round_bytes, hero_server **out);
/* Stops the workers after the rounds in flight; jobs still queued fail. */
void hero_server_destroy(hero_server *s);

/* Copies a job's reads (layout of hero_set_queries) into the server and queues
 * it; thread-safe.  *job_id identifies it in the calls below. */
int hero_job_submit(hero_server *s, const uint8_t *seq, const uint64_t *off, const int64_t *uid,
                    uint64_t n, uint64_t *job_id);
int hero_job_poll(hero_server *s, uint64_t job_id, hero_job_info *info);
/* Waits until the job is done or failed, at most timeout_ms (< 0: no limit);
 * HERO_E_TIMEOUT when the limit passes first. */
int hero_job_wait(hero_server *s, uint64_t job_id, int64_t timeout_ms, hero_job_info *info);
/* Results of a done job (hero_consensus outputs, the job's own layout). */
int hero_job_result(hero_server *s, uint64_t job_id, uint8_t *seq_out, uint32_t *imin,
                    uint32_t *imed, uint32_t *imax, double *mismatch_rate, double *gc_content,
                    uint8_t *good_out);
/* Error message of a failed job ("" for a job that has not failed).  The
 * pointer stays valid until hero_job_release of that job; do not use it after. */
const char *hero_job_error(hero_server *s, uint64_t job_id);
/* Frees a finished job's results. */
int hero_job_release(hero_server *s, uint64_t job_id);
int hero_server_get_stats(hero_server *s, hero_server_stats *out);
/* Statistics of one worker's context (0 <= worker < hero_server_workers()),
 * as of the end of its last round: where the workers' time went, per stage. */
int hero_server_worker_stats(hero_server *s, int32_t worker, hero_stats *out);
int32_t hero_server_workers(void);

/* Round policy.  round_bases_max: the most bases a round admits beyond its
 * first job (0: as many as fit the memory budget).  overlap_bases_max: the
 * device phase of a round (index to consensus) starts beside another round's
 * only if one of the two has at most this many bases and the other more, and a
 * round admitted beside a larger one stays within it; two small rounds, or two
 * large ones, take the device in turn (0: device phases always overlap; 1: they
 * never do).  Uploads and downloads are not held: they overlap the other
 * round's device phase.  A round's device work is the same whether its jobs
 * run together or apart; side by side, two rounds only share the SMs and the
 * L2.  Defaults: 8,000,000 and 64,000,000. */
int hero_server_set_round_policy(hero_server *s, uint64_t round_bases_max,
                                 uint64_t overlap_bases_max);
/* DP kernel shapes (hero_set_dp_tuning) for the rounds the server runs next. */
int hero_server_set_dp_tuning(hero_server *s, const hero_dp_tuning *t, uint32_t n);

/* Admission estimate: device bytes a job of `bases` bases in `reads` reads adds
 * to a round (read copies, vote matrix, k-mer table, consensus outputs). */
uint64_t hero_job_bytes(uint64_t bases, uint64_t reads, int32_t k);
/* How many of the queued jobs (in order, sizes bytes[i]) the next round
 * admits under round_bytes: the longest prefix that fits, at least 1. */
uint64_t hero_round_admit(const uint64_t *bytes, uint64_t n_queued, uint64_t round_bytes);

#ifdef __cplusplus
}
#endif
#endif
