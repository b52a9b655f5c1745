/*
 * hero_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the HERO read-correction path (guo-xuan/Hero, consensus
 * mode `-c`, and the alignment-output mode that writes the .aln file).  Only
 * the test suite, the smoke check and the benchmark's CPU baseline use it, and
 * only as the checker: the product path never links or calls anything in
 * oracle/.
 *
 * Parity pin: the restatement is checked byte-for-byte against the reference
 * itself (oracle/_ref/hero_ref, built from the reference sources by
 * oracle/Makefile) on the seeded fixtures under tests/golden/.
 */
#ifndef HERO_ORACLE_H_
#define HERO_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t k;              /* Config::iKmer (default 39) */
    int32_t min_overlap;    /* Config::minimumOverlapLength, flag -l (default 40) */
    int32_t affine;         /* 1 = `-a a` (bandedAlignAffineGap), 0 = global */
    int32_t keep_segments;  /* 1 = keep every DP segment with its ops for inspection */
    double mis_rate;        /* Config::dMaxMismatchRate = atof(-m)/100 (default 1) */
    double indel_rate;      /* Config::dMaxIndelRate = atof(-i)/100 (default 1) */
    double consensus_thr;   /* Config::dMinFrequencyCallConsensus (default 0.6) */
    int32_t aln_mode;       /* 1 = alignment output (no -c): the .aln file, no votes */
    int32_t merge_pairs;    /* 1 = --merge: overhang votes, reads (2i, 2i+1) merged after
                               the consensus (an odd read count is refused) */
    int32_t mapping;        /* 1 = -c --mapping: per subject the best record covering it
                               (query uids are then the inner ids: pass 0..n-1) */
} hero_oracle_params;

typedef struct {
    uint64_t probes;            /* getListOfReads calls */
    uint64_t hits;              /* PairKeyPosition entries after self exclusion */
    uint64_t chains;            /* chains formed */
    uint64_t chains_kept;       /* chains that survive markTheBestPossibleAlignment */
    uint64_t records_built;     /* chains that pass the overlap test */
    uint64_t records_accepted;  /* records passing every isGoodAlignment test */
    uint64_t records_kept;      /* records left after SubjectRead::addAlignment */
    uint64_t dp_segments;       /* BandAligner::calculateAlignment calls */
    uint64_t dp_cells;          /* sum over calls of the band cells of the loop bounds */
} hero_oracle_stats;

/* Per-step op codes used by every op string of this API (original orientation:
 * I consumes the query only, D the subject only). */
enum { HERO_OP_M = 0, HERO_OP_X = 1, HERO_OP_I = 2, HERO_OP_D = 3 };

typedef struct hero_oracle_run_s hero_oracle_run;

/* Runs the whole path.  Reads are uppercase ASCII, concatenated; read i is
 * seq[off[i]:off[i+1]].  uid = atoi(read name).  Returns NULL on bad input. */
hero_oracle_run *hero_oracle_correct(const hero_oracle_params *p, int nthreads,
                                     uint64_t nq, const uint8_t *qseq, const uint64_t *qoff,
                                     const int64_t *quid,
                                     uint64_t ns, const uint8_t *sseq, const uint64_t *soff,
                                     const int64_t *suid);
void hero_oracle_free(hero_oracle_run *r);

void hero_oracle_stats_get(const hero_oracle_run *r, hero_oracle_stats *out);

/* Corrected reads (same layout as the query input), coverage statistics and
 * the .info columns.  Reads that are not good are returned unchanged with
 * zero statistics, as QueryDataset::callConsensus leaves them. */
void hero_oracle_consensus(const hero_oracle_run *r, uint8_t *seq_out, uint32_t *imin,
                           uint32_t *imed, uint32_t *imax, double *mismatch_rate,
                           double *gc, uint8_t *good);

/* The .aln file of the alignment-output mode (aln_mode = 1): per subject read,
 * ">id\n", its records as "query,orientation,position,CIGAR,inserted bases,",
 * then "\n" (SubjectReadAligner::writeToFile, SubjectRead::writeAlignment,
 * AlignmentRecord::getCigar). */
uint64_t hero_oracle_aln_size(const hero_oracle_run *r);
void hero_oracle_aln(const hero_oracle_run *r, uint8_t *out);

/* --merge: per read pair p (reads 2p, 2p+1), merged_len[p] = length of the
 * merged read (0: not merged); seq_out has the query layout with pair p's
 * merged read written from offset off[2p] (it fits in the pair's bases), else
 * both corrected reads.  hero_oracle_overhang: the overhang votes, uint32
 * [reads][20][4]. */
void hero_oracle_merged(const hero_oracle_run *r, uint8_t *seq_out, uint32_t *merged_len);
void hero_oracle_overhang(const hero_oracle_run *r, uint32_t *out);

/* --mapping: the coverage histogram file (QueryDataset::
 * getCoverageAndWriteResults): its length; copied to out when cap suffices. */
uint64_t hero_oracle_mapping_histogram(const hero_oracle_run *r, uint8_t *out, uint64_t cap);

/* Item checks: QueryRead::mergingPairedReads on one pair (extL / extR: 20x4
 * overhang votes; out: room for lenL + lenR; returns the merged length or 0),
 * and SubjectRead::addAlignment's list over n records in arrival order (keys =
 * query uniqueIds, rate sums, lengths; out: the kept record indices in list
 * order; returns their count). */
int hero_oracle_merge_pair(const uint8_t *left, int32_t lenL, const uint8_t *right, int32_t lenR,
                           const uint32_t *extL, const uint32_t *extR, uint8_t *out);
int32_t hero_oracle_record_list(uint32_t n, const uint64_t *key, const double *rate_sum,
                                const double *len, uint32_t *out);
/* QueryRead::callConsensus on n columns of counts [n][4] (A,C,T,G): the called
 * row per column, or -1. */
void hero_oracle_columns(uint64_t n, const uint32_t *counts, double thr, int32_t *out);
/* AlignmentRecord::calculateScore of a record given as nev events in order:
 * type (HERO_OP_*), count, and for a mismatch its letter; piece[i] = 0 for a
 * run outside the DP, else the number of the DP piece the step belongs to
 * (ignored here: the reference merges every equal neighbour).  out: mismatches,
 * indels, alignment length. */
/* Chaining of one query group: hits sorted by (posQ, posS); chain_of[h] = the
 * chain of hit h, kept[c] = 1 for the chains of the largest key length (room
 * for n); returns the number of chains. */
int32_t hero_oracle_chain(int32_t k, double indel_rate, uint32_t n, const int64_t *posQ,
                          const int64_t *posS, uint32_t *chain_of, uint8_t *kept);
/* getAlignment2 on one chain of keys (posQ, posS) between a query and a
 * subject (ASCII): the DP calls it makes, 6 values each (s0, s1, q0, q1,
 * flags 1 = align right / 2 = align left, band before the call; room for
 * cap), *pos_out the record's position, *status 0 = no record (overlap below
 * l), 1 = rejected, 2 = accepted.  Returns the number of DP calls. */
int32_t hero_oracle_chain_layout(int32_t k, int32_t l, int32_t affine, double mis_rate,
                                 double indel_rate, const uint8_t *qseq, int32_t Lq,
                                 const uint8_t *sseq, int32_t Ls, uint32_t nkeys,
                                 const int64_t *posQ, const int64_t *posS, int64_t *seg,
                                 int32_t cap, int64_t *pos_out, int32_t *status);
/* AlignmentRecord::getCigar of a record given as events (as for
 * hero_oracle_record_score; a mismatch is a single step named by the query's
 * base; qrc: the query's reverse complement is aligned).  Returns the text's
 * length, or -1 if cap is too small. */
int32_t hero_oracle_record_text(uint64_t key, uint32_t orient, int64_t pos, uint32_t nev,
                                const uint32_t *piece, const uint8_t *type, const int32_t *count,
                                const uint8_t *query, int32_t Lq, int32_t qrc, uint8_t *out,
                                int32_t cap);
/* Positions of the k-mers a query read of length L puts in the table. */
int32_t hero_oracle_key_positions(int64_t L, int64_t k, int64_t *out);
void hero_oracle_record_score(uint32_t nev, const uint32_t *piece, const uint8_t *type,
                              const int32_t *count, const uint8_t *letter, int64_t *out);

/* Vote matrix after every subject's votes and before the self vote:
 * uint32 [total query bases][4], column index (c>>1)&3 (A,C,T,G). */
void hero_oracle_votes(const hero_oracle_run *r, uint32_t *cov);

/* Kept records (one per subject x query), ordered by subject then query. */
uint64_t hero_oracle_num_records(const hero_oracle_run *r);
uint64_t hero_oracle_record_ops_total(const hero_oracle_run *r);
void hero_oracle_records(const hero_oracle_run *r, uint32_t *subject, uint32_t *query,
                         uint8_t *orient, int64_t *pos, double *rate_sum, double *align_len,
                         uint64_t *ops_off, uint8_t *ops);

/* Every DP segment (only with keep_segments=1), in call order per subject. */
uint64_t hero_oracle_num_segments(const hero_oracle_run *r);
uint64_t hero_oracle_segment_ops_total(const hero_oracle_run *r);
void hero_oracle_segments(const hero_oracle_run *r, uint32_t *subject, uint8_t *orient,
                          uint32_t *query, int32_t *s0, int32_t *s1, int32_t *q0, int32_t *q1,
                          uint8_t *flags, int64_t *band, uint64_t *ops_off, uint8_t *ops);

/* One BandAligner call on explicit segments (setSequences + setBand + flags +
 * calculateAlignment).  ops: per-step codes in original orientation; returns
 * the number of steps, or -1 if ops_cap is too small.  *band_used receives the
 * band after the call (it grows to the length difference). */
int hero_oracle_align(int affine, const uint8_t *subj, int32_t ls, const uint8_t *query,
                      int32_t lq, int64_t band, int align_right, int align_left,
                      uint8_t *ops, int32_t ops_cap, int64_t *band_used);

/* QueryDataset::qualityFilter (QueryDataset.cpp:60-75). */
int hero_oracle_quality_filter(const uint8_t *seq, uint64_t len);

#ifdef __cplusplus
}
#endif
#endif
