// hero_internal.cuh -- device data layout and kernel launchers of the B200 path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "hero_core.cuh"

namespace hero {

// open-addressed k-mer slot: one 32-byte sector per probe
struct __align__(32) Slot {
    uint64_t lo, hi;      // 2k-bit key
    uint32_t start;       // first value in the value array
    uint32_t count;       // number of values; 0 = empty slot
    uint64_t pad;
};

// one DP segment: BandAligner::setSequences arguments of one call
struct __align__(16) DpSeg {
    uint32_t subj;    // subject index within the batch
    uint32_t query;   // query inner id
    uint16_t s0, s1;  // subject range, subject orientation coordinates
    uint16_t q0, q1;  // query range
    int32_t band;     // band held by the aligner before the call
    uint32_t flags;   // DPF_RIGHT | DPF_LEFT | orient << 2 (subject reverse complement)
                      // | qrc << 3 (query reverse complement: alignment output)
    uint32_t pad;
};
constexpr uint32_t kSegOrientShift = 2;
constexpr uint32_t kSegQrcShift = 3;

// the BandAligner view of a DP segment; qoff has n+1 entries
HERO_HD SegView dpseg_view(const DpSeg &g, const uint8_t *scode, const uint64_t *soff,
                           const uint32_t *slen, const uint8_t *qcode, const uint64_t *qoff) {
    const uint32_t orient = (g.flags >> kSegOrientShift) & 1u;
    const bool qrc = ((g.flags >> kSegQrcShift) & 1u) != 0;
    const uint64_t qo = qoff[g.query];
    const int32_t Lq = qrc ? int32_t(qoff[g.query + 1] - qo) : 0;
    return make_view(scode + soff[g.subj], int32_t(slen[g.subj]), int32_t(orient), qcode + qo,
                     g.s0, g.s1, g.q0, g.q1, g.flags & 3u, g.band, Lq, qrc);
}

// reads resident on the device (queries, or one batch of subjects)
struct ReadsView {
    const uint8_t *code;  // base codes, A0 C1 T2 G3, other 4
    const uint64_t *off;  // n+1 offsets
    const uint32_t *len;
    const int64_t *uid;
    const uint8_t *good;
    uint64_t n;
    const uint32_t *job;  // job of each read when jobs share a table; NULL: one job
};

struct TableView {
    const Slot *slots;
    const uint64_t *vals;  // table_value: (query << 32) | (uid_tag << 16) | position
    uint64_t mask;
};

// device counters (uint64), indices
enum Counter : int {
    C_PROBES = 0,
    C_HITS,
    C_CHAINS,
    C_NC,           // chains kept (allocated)
    C_NK,           // chain keys
    C_ND,           // DP segments
    C_MAXR,
    C_MAXC,
    C_BUILT,
    C_ACCEPTED,
    C_KEPT,
    C_DP_REF,
    C_CELLS,
    C_CELLS_ALL,    // band cells of every segment computed
    C_ANOMALY,
    C_OVERFLOW,
    C_WIN,          // winners of the current batch (compacted list length)
    C_OVERFLOW_ALL, // overflows over the context's life (C_OVERFLOW is cleared per batch)
    C_CELLS_PAIR,   // band cells computed in 16-bit pairs (of C_CELLS_ALL's)
    C_STAGED,       // wavefront tasks whose row bases were staged by the bulk copy engine
    C_STAGE_FAIL,   // staging waits that ran out (the rows were read from global memory)
    C_COUNT
};

// per-batch chain outputs (structure of arrays)
struct ChainArrays {
    uint32_t *subj, *query, *key_off, *seg_off;
    uint16_t *nkeys, *nseg;
    uint8_t *orient, *status, *win;
    double *rate, *len;
};
enum : uint8_t { CH_NONE = 0, CH_REJECTED = 1, CH_ACCEPTED = 2 };

// scratch parallel to the hit array used by the chaining kernel
struct ChainScratch {
    uint32_t *grp;       // group starts
    uint32_t *chain_of;  // chain of each hit
    int32_t *first, *last, *prev, *size, *coff, *ckeys;
    int64_t *kl;
    int32_t *g_nch;
    int64_t *g_best;
    uint32_t *g_kept, *g_keys, *g_dp;
};

// kernels launched through the launchers below since the library was loaded
uint64_t kernel_launches();

// ---------------------------------------------------------------------------
// launchers (hero_kernels.cu); all asynchronous on `st`
// ---------------------------------------------------------------------------
void launch_prep_reads(const uint8_t *raw, uint64_t nbases, uint8_t *code, const uint64_t *off,
                       uint64_t n, uint32_t *len, uint8_t *good_query, uint8_t *good_subject,
                       double *gc, int32_t l, cudaStream_t st);
// exclusive scan of n uint32 counts into n+1 uint64 offsets; tmp sized by scan_tmp_bytes
size_t scan_tmp_bytes(uint64_t n);
void launch_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, void *tmp, cudaStream_t st);

void launch_key_count(ReadsView q, int32_t k, uint32_t *count, cudaStream_t st);
void launch_key_emit(ReadsView q, int32_t k, const uint64_t *key_off, uint64_t *klo,
                     uint64_t *khi, uint64_t *kval, cudaStream_t st);
void launch_table_insert(const uint64_t *klo, const uint64_t *khi, uint64_t nkeys,
                         uint32_t *owner, uint32_t *count, uint32_t *slot_of, uint64_t mask,
                         cudaStream_t st);
void launch_table_fill(const uint64_t *kval, uint64_t nkeys, const uint32_t *slot_of,
                       const uint64_t *start, uint32_t *fill, uint64_t *vals, cudaStream_t st);
void launch_table_finalize(const uint64_t *klo, const uint64_t *khi, const uint32_t *owner,
                           const uint32_t *count, const uint64_t *start, uint64_t nslots,
                           Slot *slots, cudaStream_t st);

// aln: the alignment output's positions (seed_hit)
void launch_probe(bool emit, bool aln, ReadsView subj, uint64_t nsub, ReadsView q, TableView t, int32_t k,
                  uint2 *wcache, uint32_t *seg_hits, const uint64_t *hit_off, uint64_t *hits,
                  unsigned long long *counters, cudaStream_t st);
void launch_map_choose(const Params &p, uint64_t nsub, const uint32_t *cstart,
                       const uint32_t *ccount, ChainArrays ch, const uint32_t *keys,
                       ReadsView subj, ReadsView q, const DpSum *sums, uint32_t *alist,
                       uint32_t *winners, unsigned long long *counters, cudaStream_t st);
void launch_map_hist(ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint64_t bins,
                     unsigned long long *hist, unsigned long long *maxc, cudaStream_t st);
void launch_sort_hits(uint64_t nseg, const uint64_t *hit_off, uint64_t *hits, cudaStream_t st);
void launch_chain(const Params &p, uint64_t nseg, ReadsView subj, ReadsView q,
                  const uint64_t *hit_off, const uint64_t *hits, ChainScratch sc,
                  uint32_t *seg_chain_start, uint32_t *seg_chain_count, ChainArrays ch,
                  uint32_t *keys, DpSeg *segs, uint64_t cap_chains, uint64_t cap_keys,
                  uint64_t cap_segs, unsigned long long *counters, cudaStream_t st);

// DP: shape sort then the strip kernel
void launch_dp_sort(const DpSeg *segs, uint64_t nd, uint32_t *bins, uint32_t *perm,
                    uint64_t *bin_off, void *scan_tmp, cudaStream_t st);
constexpr uint32_t kShapeStripShift = 14;  // shape key: strips << 14 | align-left column << 10 | rows
constexpr uint32_t kDpBins = 1u << 20;
struct DpLaunch {
    const DpSeg *segs;
    const uint32_t *perm;   // processing order; NULL = identity
    uint64_t nd;
    const uint8_t *scode;   // subject codes + offsets + lengths of the batch
    const uint64_t *soff;
    const uint32_t *slen;
    const uint8_t *qcode;
    const uint64_t *qoff;
    uint32_t *ops;          // packed ops, `stride` u32 words per segment
    uint32_t stride;
    DpSum *sums;
    uint32_t *cells;        // reference band cells per segment (may be NULL)
    uint16_t *tb;           // traceback scratch: threads * rmax * nstrips
    int32_t *bnd;           // boundary scratch: threads * 3 * (rmax + 1)
    uint64_t threads;       // resident threads the scratch is laid out for
    int32_t rmax;
    int32_t affine;
    int32_t whole;          // 1: every base is A/C/G/T, the whole-band rows may run
    uint32_t pair_mask;     // bit n: segments of n strips run as 16-bit pairs (affine)
    uint32_t tb_bytes;      // bytes of traceback codes per lane and row (set by launch_dp)
    uint32_t chunk_mask;    // bit n: tracebacks of n-strip segments walk in row chunks
    int32_t warps;          // warps per block of the wavefront kernel (1, 2 or 4)
    unsigned long long *pair_cells;  // += band cells of the segments run as 16-bit pairs (may be NULL)
    int32_t regs;           // registers a thread of the wavefront kernel: 128 (0 too) or 168
    unsigned long long *staged = nullptr;  // counters: C_STAGED, then C_STAGE_FAIL (may be NULL)
    uint32_t stage_extra = 0;  // bytes a warp's code area has past its rmax rows (set by launch_dp)
};
constexpr int kStripW = 8;
constexpr uint32_t kStripsAll = 0xfffffffeu;  // every strip count 1..31 (bit n: n strips)
// needs the shape sort (perm, bin_off); tasks: 128 uint64 of device scratch.
// The per-thread scratch (tb, bnd) is only used when dp_needs_scratch().
void launch_dp(const DpLaunch &a, const uint64_t *bin_off, uint64_t *tasks, int32_t cmax,
               cudaStream_t st);
bool dp_wave_fits(int32_t rmax);
inline bool dp_needs_scratch(int32_t rmax, int32_t cmax) {
    return !dp_wave_fits(rmax) || cmax > 32 * kStripW;
}
uint64_t dp_threads(int device);

void launch_assemble(const Params &p, uint64_t nc, ChainArrays ch, const uint32_t *keys,
                     ReadsView subj, ReadsView q, const DpSum *sums, const uint32_t *cells,
                     unsigned long long *counters, cudaStream_t st);
// winners (one per subject x query) are appended to `winners`; the count is
// counters[C_WIN]
void launch_dedupe(uint64_t nsub, const uint32_t *seg_chain_start,
                   const uint32_t *seg_chain_count, ChainArrays ch, uint32_t *winners,
                   unsigned long long *counters, cudaStream_t st);
// Votes.  A mismatch votes the subject base into cov[pos][4]; a run of matches
// votes the query's own base, recorded as +1/-1 at the run's ends in mdiff
// (a per-read difference array, summed by the consensus).
constexpr uint32_t kWinScratch = 3 * 512;  // uint32 bins, offsets and cursors of the winner sort
constexpr uint32_t kUnitSubject = 0x80000000u;  // header unit: kUnitSubject | subject
constexpr uint32_t kUnitEnd = 0xffffffffu;      // closing newline of a subject
constexpr uint32_t kUnitChainLimit = kUnitSubject;  // chains and subjects of a batch stay below
// alignment output (HERO without -c): per subject the list of kept records
// (alist: slots in the subject's chain ranges, alist_n: lengths), then the .aln
// text in units (unit: kUnitSubject | subject, a chain index, or the closing
// newline; sizes ulen, prefix and CIGAR lengths upre / ucig; offsets uoff)
void launch_aln_list(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                     ChainArrays ch, ReadsView q, uint32_t *alist, uint32_t *alist_n,
                     unsigned long long *counters, cudaStream_t st);
void launch_aln_units(uint64_t nsub, const uint32_t *cstart, const uint32_t *ccount,
                      const uint32_t *alist, const uint32_t *alist_n, const uint64_t *rec_off,
                      ReadsView subj, uint32_t *unit, uint32_t *ulen, cudaStream_t st);
void launch_aln_size(const Params &p, uint64_t nunit, const uint32_t *unit, ChainArrays ch,
                     const uint32_t *keys, ReadsView subj, ReadsView q, const uint32_t *ops,
                     uint32_t stride, const DpSum *sums, uint32_t *ulen, uint32_t *upre,
                     uint32_t *ucig, cudaStream_t st);
void launch_aln_write(const Params &p, uint64_t nunit, const uint32_t *unit, const uint64_t *uoff,
                      ChainArrays ch, const uint32_t *keys, ReadsView subj, ReadsView q,
                      const uint32_t *ops, uint32_t stride, const DpSum *sums,
                      const uint32_t *upre, const uint32_t *ucig, char *text, cudaStream_t st);
// --merge: overhang votes of the batch's winners (after launch_vote; ext is
// uint32 [query reads][kOverhang][4]), and the pair merge after the consensus
void launch_vote_overhang(const Params &p, uint64_t max_winners, ChainArrays ch,
                          const uint32_t *winners, const uint32_t *keys, ReadsView subj,
                          ReadsView q, const DpSum *sums, uint32_t *ext,
                          const unsigned long long *counters, cudaStream_t st);
void launch_merge_pairs(uint64_t npairs, const uint64_t *off, const uint8_t *corrected,
                        const uint32_t *ext, uint8_t *merged, uint32_t *merged_len,
                        cudaStream_t st);
void launch_vote(const Params &p, uint64_t max_winners, ChainArrays ch, const uint32_t *winners,
                 uint32_t *sorted, uint32_t *win_bins, const uint32_t *keys, ReadsView subj,
                 ReadsView q, const uint32_t *ops, uint32_t stride, const DpSum *sums,
                 uint32_t *cov, int32_t *mdiff, unsigned long long *counters, cudaStream_t st);
void launch_consensus(const Params &p, ReadsView q, const uint32_t *cov, const int32_t *mdiff,
                      uint8_t *out, uint32_t *colsum, uint32_t *imin, uint32_t *imed,
                      uint32_t *imax, double *mis, cudaStream_t st);
// full vote matrix (cov + match runs), as the reference's coverage matrix
void launch_expand_votes(ReadsView q, const uint32_t *cov, const int32_t *mdiff, uint32_t *out,
                         cudaStream_t st);
void launch_stamp(unsigned long long *out, cudaStream_t st);
void launch_fingerprint(const uint8_t *raw, uint64_t nb, const uint64_t *off, const int64_t *uid,
                        uint64_t n, unsigned long long *out, cudaStream_t st);
void launch_unpack_ops(const uint32_t *ops, uint32_t stride, const DpSum *sums, uint64_t nd,
                       const uint64_t *out_off, uint8_t *out, int32_t *nops, cudaStream_t st);

}  // namespace hero
