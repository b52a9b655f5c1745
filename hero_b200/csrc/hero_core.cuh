// hero_core.cuh -- per-item logic of the HERO read-correction path.
//
// Everything here works on one item (one k-mer, one chain, one DP segment,
// one record, one read column) and is written once as __host__ __device__
// code: the CUDA kernels in hero_kernels.cu call it per thread, and the host
// test harness compiles the same header with g++ to check it item by item.
//
// Reference semantics (guo-xuan/Hero, src/) are cited per function.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define HERO_HD __host__ __device__ __forceinline__
#else
#define HERO_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define HERO_DMUL(a, b) __dmul_rn((a), (b))
#define HERO_DDIV(a, b) __ddiv_rn((a), (b))
#define HERO_DADD(a, b) __dadd_rn((a), (b))
#define HERO_DSUB(a, b) __dsub_rn((a), (b))
#define HERO_ROUND(a) round(a)
#define HERO_FABS(a) fabs(a)
#else
#include <cmath>
#define HERO_DMUL(a, b) ((a) * (b))
#define HERO_DDIV(a, b) ((a) / (b))
#define HERO_DADD(a, b) ((a) + (b))
#define HERO_DSUB(a, b) ((a) - (b))
#define HERO_ROUND(a) std::round(a)
#define HERO_FABS(a) std::fabs(a)
#endif

namespace hero {

// ---------------------------------------------------------------------------
// constants
// ---------------------------------------------------------------------------
// BandAligner::setCost (BandAligner.cpp:528-542); sentinel -MAXDUL (BandAligner.h:18)
constexpr int kDX = -4, kDY = -4, kMISS = -4, kHIT = 1, kSX = 0, kEX = -1;
constexpr int kNEG = -100000;

// per-step alignment ops in original orientation (I consumes query only, D subject only)
enum : uint8_t { OP_M = 0, OP_X = 1, OP_I = 2, OP_D = 3 };

// base codes: (c >> 1) & 3 of the ASCII letter, as HERO indexes its coverage
// matrix (QueryRead.cpp:124-131): A=0 C=1 T=2 G=3; anything else is 4.
// The complement of an ACGT code is code ^ 2.
constexpr uint8_t kBad = 4;
HERO_HD uint8_t base_code(uint8_t c) {
    return (c == 'A' || c == 'C' || c == 'G' || c == 'T') ? uint8_t((c >> 1) & 3) : kBad;
}
HERO_HD char code_base(uint8_t c) {  // aDNA (QueryRead.cpp:11)
    return c == 0 ? 'A' : c == 1 ? 'C' : c == 2 ? 'T' : 'G';
}

struct Params {
    int32_t k;          // Config::iKmer
    int32_t l;          // Config::minimumOverlapLength
    int32_t affine;     // Config::iAlignerType == IAFFINE
    int32_t aln;        // !Config::bCallConsensus: alignment output (the .aln file)
    double mis_rate;    // Config::dMaxMismatchRate
    double indel_rate;  // Config::dMaxIndelRate
    double thr;         // Config::dMinFrequencyCallConsensus
};

// ---------------------------------------------------------------------------
// k-mer keys: the 2k-bit integer of the k-mer codes, first base most significant
// (hi holds the bits above 64).  Supports 1 <= k <= 63.
// ---------------------------------------------------------------------------
struct Kmer {
    uint64_t lo, hi;
};

HERO_HD void kmer_push(Kmer &m, uint32_t code, int k) {
    m.hi = (m.hi << 2) | (m.lo >> 62);
    m.lo = (m.lo << 2) | code;
    if (2 * k < 64) {
        m.lo &= (1ull << (2 * k)) - 1ull;
        m.hi = 0;
    } else if (2 * k == 64) {
        m.hi = 0;
    } else {
        m.hi &= (1ull << (2 * k - 64)) - 1ull;
    }
}

// Adds a base as the most significant of k digits (the reverse complement of a
// window rolls this way: the base entering the window goes on top, the base
// leaving it drops off the bottom).
HERO_HD void kmer_push_front(Kmer &m, uint32_t code, int k) {
    m.lo = (m.lo >> 2) | (m.hi << 62);
    m.hi >>= 2;
    const int b = 2 * (k - 1);
    if (b < 64) {
        m.lo |= uint64_t(code) << b;
    } else {
        m.hi |= uint64_t(code) << (b - 64);
    }
}

// Jobs served together share one k-mer table: a key carries its job above the
// 2k k-mer bits, so keys of different jobs never compare equal (job must fit
// in the 128 - 2k bits left: kmer_job_bits).
HERO_HD void kmer_tag(Kmer &m, uint32_t job, int k) {
    if (2 * k <= 64) {
        m.hi = job;
    } else if (job) {
        m.hi |= uint64_t(job) << (2 * k - 64);
    }
}
HERO_HD int kmer_job_bits(int k) { return 2 * k <= 64 ? 32 : (128 - 2 * k < 32 ? 128 - 2 * k : 32); }

HERO_HD uint64_t mix64(uint64_t z) {  // splitmix64 finalizer
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ull;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebull;
    z ^= z >> 31;
    return z;
}
HERO_HD uint64_t kmer_hash(const Kmer &m) { return mix64(m.lo ^ mix64(m.hi + 0x9e3779b97f4a7c15ull)); }

// Keys a good query read contributes (HashTableLongKey::insertQueryDataset,
// HashTableLongKey.cpp:279-289): positions 0, k, 2k, ... while <= L-k, then
// a tail key at L-k when the stride did not land on L.
HERO_HD int32_t query_key_count(int64_t L, int64_t k) {
    if (L < k) return 0;  // the reference throws on such a read (substr out of range)
    int64_t n = (L - k) / k + 1;
    return int32_t(n + (n * k < L ? 1 : 0));
}
HERO_HD int64_t query_key_pos(int64_t L, int64_t k, int32_t idx) {
    int64_t n = (L - k) / k + 1;
    return idx < n ? int64_t(idx) * k : L - k;
}

// hit: (query inner id, position on query, position on subject), ordered like
// comparePairKeyPosition (SubjectRead.cpp:157-173) when compared as u64
HERO_HD uint64_t hit_pack(uint32_t q, uint32_t posQ, uint32_t posS) {
    return (uint64_t(q) << 32) | (uint64_t(posQ) << 16) | uint64_t(posS);
}
HERO_HD uint32_t hit_q(uint64_t h) { return uint32_t(h >> 32); }

// A hit of subject window f (forward) against query position posQ, found in
// pass o (0 forward, 1 reverse complement) of a subject of length Ls.  With -c
// the reverse pass keeps positions on the reverse-complemented subject; the
// alignment-output mode flips them onto the forward subject and the query's
// reverse complement (SubjectReadAligner.cpp:477-481).
HERO_HD uint64_t seed_hit(bool aln, int o, uint32_t q, uint32_t posQ, int32_t f, int32_t Ls,
                          int32_t Lq, int32_t k) {
    if (o == 0) return hit_pack(q, posQ, uint32_t(f));
    if (aln) return hit_pack(q, uint32_t(Lq - (int32_t(posQ) + k)), uint32_t(f));
    return hit_pack(q, posQ, uint32_t(Ls - k - f));
}
// A k-mer table value: (query << 32) | (uid_tag << 16) | position.  Read
// positions are below 2^15, so the low word has room for a 16-bit fold of the
// query's uniqueId: the self-hit test (SubjectReadAligner.cpp:463-465) loads
// the query's id only when the folds agree.
HERO_HD uint32_t uid_tag(int64_t u) {
    const uint64_t x = uint64_t(u);
    return uint32_t((x ^ (x >> 16) ^ (x >> 32) ^ (x >> 48)) & 0xffffu);
}
HERO_HD uint64_t table_value(uint64_t q, uint32_t tag, int64_t pos) {
    return (q << 32) | (uint64_t(tag) << 16) | uint64_t(pos);
}
HERO_HD uint32_t value_query(uint64_t v) { return uint32_t(v >> 32); }
HERO_HD uint32_t value_tag(uint64_t v) { return uint32_t(v >> 16) & 0xffffu; }
HERO_HD uint32_t value_pos(uint64_t v) { return uint32_t(v) & 0xffffu; }
HERO_HD int32_t hit_posQ(uint64_t h) { return int32_t((h >> 16) & 0xffff); }
HERO_HD int32_t hit_posS(uint64_t h) { return int32_t(h & 0xffff); }

// ---------------------------------------------------------------------------
// chaining (SubjectReadAligner.cpp:391-408, 711-751, 805-852)
// ---------------------------------------------------------------------------
// isFromTheSameAlignment
HERO_HD bool same_alignment(const Params &p, int32_t addQ, int32_t addS, int32_t begQ,
                            int32_t begS, int32_t endQ, int32_t endS) {
    if (addS <= endS) return false;
    if (addQ <= endQ) return false;
    double lq = HERO_FABS(double(addQ - begQ));
    double ls = HERO_FABS(double(addS - begS));
    double total = (lq >= ls ? lq : ls);
    total = HERO_DADD(total, double(p.k));
    double diff = HERO_FABS(HERO_DSUB(lq, ls));
    if (HERO_DDIV(diff, total) > p.indel_rate) return false;
    return true;
}

// Greedy chain assignment of one query group (hits sorted by posQ, posS).
// chain_of[h] receives the chain index of each hit; first/last are scratch of
// the group's size.  Returns the number of chains.
template <class HitAt>
HERO_HD int32_t chain_group(const Params &p, const HitAt &hit, int32_t n, uint32_t *chain_of,
                            int32_t *first, int32_t *last) {
    int32_t nch = 0;
    for (int32_t h = 0; h < n; h++) {
        const uint64_t x = hit(h);
        const int32_t q = hit_posQ(x), s = hit_posS(x);
        int32_t c = 0;
        for (; c < nch; c++) {
            const uint64_t b = hit(first[c]), e = hit(last[c]);
            if (same_alignment(p, q, s, hit_posQ(b), hit_posS(b), hit_posQ(e), hit_posS(e))) break;
        }
        if (c == nch) {
            first[nch] = h;
            nch++;
        }
        last[c] = h;
        chain_of[h] = uint32_t(c);
    }
    return nch;
}

// calKeyLength of every chain of a group; kl must hold nch entries and prev
// nch scratch slots.  Returns the largest key length.
template <class HitAt>
HERO_HD int64_t chain_key_lengths(const Params &p, const HitAt &hit, int32_t n,
                                  const uint32_t *chain_of, int32_t nch, int64_t *kl,
                                  int32_t *prev) {
    for (int32_t c = 0; c < nch; c++) {
        kl[c] = 0;
        prev[c] = -1;
    }
    for (int32_t h = 0; h < n; h++) {
        const uint32_t c = chain_of[h];
        if (prev[c] >= 0) {
            const int32_t a = hit_posS(hit(prev[c])), b = hit_posS(hit(h));
            kl[c] += (a + p.k <= b) ? p.k : (b - a);
        }
        prev[c] = h;
    }
    int64_t best = 0;
    for (int32_t c = 0; c < nch; c++) {
        kl[c] += p.k;
        if (kl[c] > best) best = kl[c];
    }
    return best;
}

// ---------------------------------------------------------------------------
// record pieces: getAlignment2 (SubjectReadAligner.cpp:197-389)
// ---------------------------------------------------------------------------
enum : uint32_t { DPF_RIGHT = 1u, DPF_LEFT = 2u };

// Walks one chain the way getAlignment2 builds its record and calls the visitor:
//   v.begin(extra, maxMis, maxIndel) once the overlap test has passed
//   v.position(pos)
//   v.run(op, count)        CIGAR runs added by k-mer arithmetic (addCigar)
//   v.dp(s0, s1, q0, q1, flags, band)   one BandAligner call; band is the value the
//                                        aligner holds before the call
//   v.check(maxMis, maxIndel) -> bool   isGoodAlignment(m, i) early exit point
//   v.finish()              after the end piece (the rate test is the caller's)
// keys(i) returns (posQ, posS) of the i-th key of the chain as a hit word.
// Returns false when the chain yields no record (overlap test or early exit).
template <class KeyAt, class V>
HERO_HD bool walk_chain(const Params &p, int64_t Lq, int64_t Ls, const KeyAt &keys, int32_t n,
                        V &v) {
    const int64_t k = p.k;
    int64_t posQ = hit_posQ(keys(0)), posS = hit_posS(keys(0));
    int64_t ov = (posQ < posS ? posQ : posS);
    ov += (Lq - posQ < Ls - posS ? Lq - posQ : Ls - posS);
    if (ov < p.l) return false;
    const int64_t extra = int64_t(HERO_ROUND(HERO_DMUL(double(ov), p.indel_rate)));
    const int64_t maxMis = int64_t(HERO_ROUND(HERO_DMUL(double(ov), p.mis_rate)));
    const int64_t maxIndel = extra;
    v.begin(extra, maxMis, maxIndel);
    int64_t band = extra * 2;  // setBand; grows inside the aligner (BandAligner.cpp:59-62)
    auto dp = [&](int64_t s0, int64_t s1, int64_t q0, int64_t q1, uint32_t flags) {
        v.dp(s0, s1, q0, q1, flags, band);
        // setSequences puts the longer segment on the rows; the aligner then
        // widens its band to the length difference
        int64_t ls = s1 - s0, lq = q1 - q0;
        int64_t d = lq <= ls ? ls - lq : lq - ls;
        if (d > band) band = d;
    };
    if (posQ != 0 && posS != 0) {
        if (posQ < posS) {
            int64_t s0 = (posS - posQ - extra < 0 ? 0 : posS - posQ - extra);
            v.position(s0);
            dp(s0, posS, 0, posQ, DPF_RIGHT);
        } else if (posQ == posS) {
            v.position(0);
            dp(0, posS, 0, posQ, DPF_RIGHT);
        } else {
            int64_t q0 = (posQ - posS - extra < 0 ? 0 : posQ - posS - extra);
            v.position(0);
            if (posQ - posS - extra > 0) v.run(OP_I, posQ - posS - extra);
            dp(0, posS, q0, posQ, DPF_RIGHT);
        }
        v.run(OP_M, k);
    } else {
        if (posS == 0 && posQ == 0) {
            v.position(0);
        } else if (posS == 0) {
            v.position(0);
            v.run(OP_I, posQ);
        } else {
            v.position(posS);
        }
        v.run(OP_M, k);
    }
    if (!v.check(maxMis, maxIndel)) return false;
    for (int32_t i = 1; i < n; i++) {
        const int64_t cQ = hit_posQ(keys(i)), cS = hit_posS(keys(i));
        if (cQ - posQ == cS - posS && posS + k >= cS) {
            if (posS + k > cS) {
                v.run(OP_M, cS - posS);
            } else {
                v.run(OP_M, k);
            }
        } else {
            if (posS + k == cS) {
                if (cQ - posQ - k > 0) {
                    v.run(OP_I, cQ - posQ - k);
                    v.run(OP_M, k);
                } else {
                    v.run(OP_D, -cQ + posQ + k);
                    v.run(OP_M, cQ - posQ);
                }
            } else if (posS + k > cS) {
                if (cQ - posQ < cS - posS) {
                    v.run(OP_D, cS - posS - cQ + posQ);
                    v.run(OP_M, cQ - posQ);
                } else {
                    v.run(OP_I, cQ - posQ + posS - cS);
                    v.run(OP_M, cS - posS);
                }
            } else {
                if (posQ + k == cQ) {
                    v.run(OP_D, cS - posS - k);
                    v.run(OP_M, k);
                } else if (posQ + k > cQ) {
                    v.run(OP_D, cS - posS + posQ - cQ);
                    v.run(OP_M, k + posQ - cQ);
                } else {
                    dp(posS + k, cS, posQ + k, cQ, 0);
                    v.run(OP_M, k);
                }
            }
        }
        posQ = cQ;
        posS = cS;
        if (!v.check(maxMis, maxIndel)) return false;
    }
    posQ = hit_posQ(keys(n - 1)) + k;
    posS = hit_posS(keys(n - 1)) + k;
    if (posQ < Lq) {
        if (posS == Ls) {
            v.run(OP_I, Lq - posQ);
        } else if (Ls - posS < Lq - posQ) {
            int64_t qe = (Ls - posS + posQ + extra < Lq ? Ls - posS + posQ + extra : Lq);
            dp(posS, Ls, posQ, qe, DPF_LEFT);
            if (Ls - posS + posQ + extra < Lq) v.run(OP_I, Lq - (Ls - posS + posQ + extra));
        } else if (Ls - posS == Lq - posQ) {
            dp(posS, Ls, posQ, Lq, DPF_LEFT);
        } else {
            int64_t se = (posS + (Lq - posQ) + extra < Ls ? posS + (Lq - posQ) + extra : Ls);
            dp(posS, se, posQ, Lq, DPF_LEFT);
        }
    }
    v.finish();
    return true;
}

// ---------------------------------------------------------------------------
// record score: AlignmentRecord::addCigar + calculateScore (AlignmentRecord.cpp:35-100)
// Only the first and last runs are treated specially (leading/trailing I or D
// are not counted), so a record is summarised exactly by its first run, its
// last run and the totals of the runs strictly between them.  Mismatch runs
// with different letters are separate CIGAR entries in the reference but are
// never first-vs-interior ambiguous (they are not I/D), so they merge here.
// ---------------------------------------------------------------------------
struct DpSum {  // summary of one DP segment's op path (16 bytes)
    uint16_t tot[4];  // ops of each kind over the whole path
    uint16_t fc, lc;  // first / last run lengths
    uint8_t ft, lt;   // first / last run kinds
    uint8_t nruns;    // 1, or 2 meaning "two or more"
    uint8_t pad;
};

struct RecState {
    int32_t n = 0;  // runs so far: 0, 1, 2 (= two or more)
    uint8_t ft = 0, lt = 0;
    int64_t fc = 0, lc = 0;
    int64_t im = 0, ix = 0, iid = 0;  // interior totals

    HERO_HD void interior_add(uint8_t t, int64_t c) {
        if (t == OP_M) {
            im += c;
        } else if (t == OP_X) {
            ix += c;
        } else {
            iid += c;
        }
    }
    HERO_HD void add(uint8_t t, int64_t c) {
        if (n == 0) {
            ft = t;
            fc = c;
            n = 1;
        } else if (n == 1) {
            if (ft == t) {
                fc += c;
            } else {
                lt = t;
                lc = c;
                n = 2;
            }
        } else {
            if (lt == t) {
                lc += c;
            } else {
                interior_add(lt, lc);
                lt = t;
                lc = c;
            }
        }
    }
    HERO_HD void add_piece(const DpSum &s) {
        add(s.ft, s.fc);
        if (s.nruns >= 2) {
            if (n >= 2) interior_add(lt, lc);
            // interior runs of the piece: totals minus its first and last runs
            const int64_t fm = (s.ft == OP_M ? s.fc : 0) + (s.lt == OP_M ? s.lc : 0);
            const int64_t fx = (s.ft == OP_X ? s.fc : 0) + (s.lt == OP_X ? s.lc : 0);
            const int64_t fid = (s.ft >= OP_I ? s.fc : 0) + (s.lt >= OP_I ? s.lc : 0);
            im += int64_t(s.tot[OP_M]) - fm;
            ix += int64_t(s.tot[OP_X]) - fx;
            iid += int64_t(s.tot[OP_I]) + int64_t(s.tot[OP_D]) - fid;
            lt = s.lt;
            lc = s.lc;
            n = 2;
        }
    }
    // calculateScore: (mismatches, indels, alignment length)
    HERO_HD void score(int64_t &mis, int64_t &indel, int64_t &len) const {
        mis = ix;
        indel = iid;
        len = im + ix + iid;
        if (n >= 1 && ft != OP_I && ft != OP_D) {
            len += fc;
            if (ft == OP_X) mis += fc;
        }
        if (n >= 2 && lt != OP_I && lt != OP_D) {
            len += lc;
            if (lt == OP_X) mis += lc;
        }
    }
    // isGoodAlignment(maxMis, maxIndel) (AlignmentRecord.cpp:310-316)
    HERO_HD bool good_counts(int64_t maxMis, int64_t maxIndel) const {
        int64_t m, i, l;
        score(m, i, l);
        return !(m > maxMis || i > maxIndel);
    }
    // isGoodAlignment() rates and the dedupe keys (AlignmentRecord.cpp:92-99, 302-308)
    HERO_HD bool good_rates(const Params &p, double &rate_sum, double &len_out) const {
        int64_t m, i, l;
        score(m, i, l);
        double indel_rate = 100, mis_rate = 100;
        if (l != 0) {
            indel_rate = HERO_DDIV(double(i), double(l));
            mis_rate = HERO_DDIV(double(m), double(l));
        }
        rate_sum = HERO_DADD(indel_rate, mis_rate);
        len_out = double(l);
        return mis_rate <= p.mis_rate && indel_rate <= p.indel_rate;
    }
};

// SubjectRead::addAlignment (SubjectRead.cpp:25-79): a later record replaces the
// kept one only if it is strictly better: smaller rate sum, or equal rate sum
// and longer alignment.  Folding in arrival order keeps the earliest best.
HERO_HD bool record_better(double rs_new, double len_new, double rs_cur, double len_cur) {
    if (rs_cur < rs_new) return false;
    if (rs_cur == rs_new) return !(len_cur >= len_new);
    return true;
}

// SubjectRead::addAlignment (SubjectRead.cpp:25-79) as the list it keeps, for
// the alignment output, where the order of the list is the order of the .aln
// records.  Records are ids; key(id) is iQueryReadUniqueId (UINT64: the
// query's atoi(name)); better(a, b) is record_better of a over b.  A record
// equal in key to the last one competes with it; otherwise, if its key is not
// above the largest key seen, the list is scanned up to the first larger key
// for an equal one (which it may replace) and else appended; a key above the
// largest is appended.  list.get(i) / list.set(i, id) address slot i.
// Returns the new length.
template <class List, class Key, class Better>
HERO_HD uint32_t list_add(List &list, uint32_t n, uint64_t &largest, uint32_t id, const Key &key,
                          const Better &better) {
    const uint64_t k = key(id);
    if (n == 0) {
        largest = k;
        list.set(0, id);
        return 1;
    }
    const uint32_t last = list.get(n - 1);
    if (key(last) == k) {
        if (better(id, last)) list.set(n - 1, id);
        return n;
    }
    if (largest >= k) {
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t e = list.get(i);
            const uint64_t ke = key(e);
            if (ke > k) break;
            if (ke == k) {
                if (better(id, e)) list.set(i, id);
                return n;
            }
        }
        list.set(n, id);
        return n + 1;
    }
    largest = k;
    list.set(n, id);
    return n + 1;
}

// decimal text of integers, as ostream prints them
HERO_HD uint32_t dec_len(uint64_t v) {
    uint32_t n = 1;
    while (v >= 10) {
        v /= 10;
        n++;
    }
    return n;
}
HERO_HD uint32_t dec_len_signed(int64_t v) {
    return v < 0 ? 1u + dec_len(uint64_t(0) - uint64_t(v)) : dec_len(uint64_t(v));
}
HERO_HD char *dec_put(char *o, uint64_t v) {
    const uint32_t n = dec_len(v);
    for (uint32_t i = n; i > 0; i--) {
        o[i - 1] = char('0' + v % 10);
        v /= 10;
    }
    return o + n;
}
HERO_HD char *dec_put_signed(char *o, int64_t v) {
    if (v < 0) {
        *o++ = '-';
        return dec_put(o, uint64_t(0) - uint64_t(v));
    }
    return dec_put(o, uint64_t(v));
}

// Text of one alignment record, AlignmentRecord::getCigar (AlignmentRecord.cpp:
// 102-149) with storeOverhang off:  "id,orientation,position,CIGAR,inserted,".
// The CIGAR is the run-length form of the per-base types -- M, I, D, or the
// query's base at a mismatch (BandAligner.cpp:258-419) -- because
// AlignmentRecord::addCigar (AlignmentRecord.cpp:35-48) merges every equal
// neighbour, whichever piece it came from.  "inserted" holds the query bases
// of every I entry except the first and the last entry.  Driven by walk_chain
// through a piece source: src.each(piece, f) calls f(op) for the ops of DP
// piece `piece` in order.  Count mode (cig == nullptr) only sizes the text.
template <class Src>
struct AlnText {
    Src src;
    const uint8_t *qc;  // query codes, forward
    int32_t Lq;
    bool qrc;           // the query's reverse complement is aligned
    char *cig = nullptr, *ins = nullptr;  // write cursors (write mode)
    uint32_t cig_len = 0, ins_len = 0;
    uint32_t entries = 0, piece = 0;
    char t = 0;
    int64_t c = 0, q0 = 0, pq = 0;
    int64_t pos = 0;  // iPositionOfQueryOnSubject

    // the query's base letter at i (a position past the read, which only a record
    // that also votes past the read could reach, reads as N)
    HERO_HD char qbase(int64_t i) const {
        if (i < 0 || i >= Lq) return 'N';
        return code_base(qrc ? uint8_t((qc[Lq - 1 - i] ^ 2u) & 3u) : uint8_t(qc[i] & 3u));
    }
    HERO_HD void flush(bool last) {
        cig_len += dec_len(uint64_t(c)) + 1u;
        if (cig) {
            cig = dec_put(cig, uint64_t(c));
            *cig++ = t;
        }
        if (t == 'I' && entries != 1u && !last) {
            ins_len += uint32_t(c);
            if (ins)
                for (int64_t i = 0; i < c; i++) *ins++ = qbase(q0 + i);
        }
    }
    HERO_HD void add(char type, int64_t n) {  // AlignmentRecord::addCigar
        if (entries && type == t) {
            c += n;
        } else {
            if (entries) flush(false);
            t = type;
            c = n;
            q0 = pq;
            entries++;
        }
        if (type != 'D') pq += n;
    }
    HERO_HD void op(uint8_t o) {
        if (o == OP_M) {
            add('M', 1);
        } else if (o == OP_X) {
            add(qbase(pq), 1);
        } else {
            add(o == OP_I ? 'I' : 'D', 1);
        }
    }
    HERO_HD void begin(int64_t, int64_t, int64_t) {}
    HERO_HD void position(int64_t p) { pos = p; }
    HERO_HD void run(uint8_t o, int64_t n) { add(o == OP_M ? 'M' : o == OP_I ? 'I' : 'D', n); }
    HERO_HD void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        src.each(piece++, [this](uint8_t o) { op(o); });
    }
    HERO_HD bool check(int64_t, int64_t) { return true; }
    HERO_HD void finish() {
        if (entries) flush(true);  // the open entry is the last one
    }
};

// ---------------------------------------------------------------------------
// --merge: overhang votes and paired-read merging
// ---------------------------------------------------------------------------
constexpr int kOverhang = 20;  // QueryRead::iLength4ExtraMatrix (QueryRead.cpp:225)

// Where a kept record ends on its subject, and whether its CIGAR has more than
// one entry (SubjectRead::updateQueryCoverageConsiderMerging,
// SubjectRead.cpp:332-462, votes the subject bases past the record's end into
// the query's overhang matrix only then).  A CIGAR has a single entry exactly
// when every step is a match (I, D and mismatch letters differ from M), so the
// DP pieces' totals decide it: sums(piece) gives a piece's DpSum.
template <class Sums>
struct OverhangWalk {
    Sums sums;
    uint32_t piece = 0;
    int64_t ps = 0;
    bool other = false;
    HERO_HD void begin(int64_t, int64_t, int64_t) {}
    HERO_HD void position(int64_t p) { ps = p; }
    HERO_HD void run(uint8_t t, int64_t c) {
        if (t != OP_M) other = true;
        if (t != OP_I) ps += c;
    }
    HERO_HD void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        const DpSum s = sums(piece++);
        const uint32_t P = uint32_t(s.tot[0]) + s.tot[1] + s.tot[2] + s.tot[3];
        if (s.tot[OP_M] != P) other = true;
        ps += int64_t(s.tot[OP_M]) + s.tot[OP_X] + s.tot[OP_D];
    }
    HERO_HD bool check(int64_t, int64_t) { return true; }
    HERO_HD void finish() {}
};

// --mapping: what SubjectRead::chooseQueryWithBestAlignment (SubjectRead.cpp:
// 463-500) reads of a record.  AlignmentRecord::isSubjectCoveredByQuery
// (AlignmentRecord.cpp:343-370) needs the record's position on the subject,
// the kinds of its first and last CIGAR entries and the bases of every entry
// that is not an insertion; getAccuracy (AlignmentRecord.cpp:372-381) the
// mismatch bases.  Entry boundaries do not change either sum, so a walk over
// the record's runs and DP pieces gives them.
template <class Sums>
struct CoverWalk {
    Sums sums;
    uint32_t piece = 0;
    int64_t pos = 0, non_ins = 0, subs = 0;
    int32_t first = -1, last = -1;
    HERO_HD void begin(int64_t, int64_t, int64_t) {}
    HERO_HD void position(int64_t p) { pos = p; }
    HERO_HD void run(uint8_t t, int64_t c) {
        if (c <= 0) return;
        if (first < 0) first = t;
        last = t;
        if (t != OP_I) non_ins += c;
        if (t == OP_X) subs += c;
    }
    HERO_HD void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        const DpSum s = sums(piece++);
        const uint32_t P = uint32_t(s.tot[0]) + s.tot[1] + s.tot[2] + s.tot[3];
        if (P == 0) return;
        if (first < 0) first = s.ft;
        last = s.nruns >= 2 ? s.lt : s.ft;
        non_ins += int64_t(s.tot[OP_M]) + s.tot[OP_X] + s.tot[OP_D];
        subs += s.tot[OP_X];
    }
    HERO_HD bool check(int64_t, int64_t) { return true; }
    HERO_HD void finish() {}
    // isSubjectCoveredByQuery(Ls)
    HERO_HD bool covers(int64_t Ls) const {
        return first >= 0 && pos == 0 && first != OP_D && last != OP_D && non_ins >= Ls;
    }
};

// chooseQueryWithBestAlignment over a subject's record list (n records in list
// order; covers(i), subs(i) of each): how many of the list's records vote and
// which.  No covering record: none (-1 returned, *n_keep = 0).  Exactly one:
// the whole list keeps voting (the reference returns without touching the
// list; returns -1, *n_keep = n).  Two or more: the first covering record with
// the fewest substitutions, below the subject's length (returns its index,
// *n_keep = 1; none below the length: -1, *n_keep = 0, where the reference
// reports an error).
template <class Covers, class Subs>
HERO_HD int32_t map_choose(uint32_t n, int64_t Ls, const Covers &covers, const Subs &subs,
                           uint32_t *n_keep) {
    uint32_t qualified = 0;
    int32_t best = -1;
    double least = double(Ls);
    for (uint32_t i = 0; i < n; i++) {
        if (!covers(i)) continue;
        qualified++;
        const double d = double(subs(i));
        if (d < least) {
            least = d;
            best = int32_t(i);
        }
    }
    if (qualified == 0) {
        *n_keep = 0;
        return -1;
    }
    if (qualified == 1) {
        *n_keep = n;
        return -1;
    }
    *n_keep = best >= 0 ? 1u : 0u;
    return best;
}

// QueryRead::getComplementBase (QueryRead.cpp:375-382), on the ASCII letter:
// bit 2 set (C, G) flips C<->G, else A<->T by xor 0x15
HERO_HD char complement_char(char c) { return (c & 0x02) ? char(c ^ 0x04) : char(c ^ 0x15); }

// QueryRead::getExtendSequence (QueryRead.cpp:384-403): per overhang column the
// strictly largest count (the first of equal counts), as an aDNA letter; stops
// at a column without votes.  Returns the length (at most kOverhang).
HERO_HD int overhang_letters(const uint32_t *m, char *out) {
    int n = 0;
    for (int i = 0; i < kOverhang; i++) {
        int id = -1;
        uint32_t best = 0;
        for (int j = 0; j < 4; j++) {
            const uint32_t v = m[i * 4 + j];
            if (best < v) {
                best = v;
                id = j;
            }
        }
        if (best < 1) break;
        out[n++] = code_base(uint8_t(id));
    }
    return n;
}

// QueryRead::mergingPairedReads (QueryRead.cpp:268-319) for one pair after the
// consensus: left and right are the corrected reads (raw lengths lenL, lenR),
// extL / extR their overhang votes.  The first left offset at which the whole
// rest of the left read equals the right read's complement read backwards is
// the overlap; the pair merges if the overlap plus both extensions reach 40
// bases and both extensions agree with the other read.  The merged read -- the
// left read, then the right read's complement bases backwards from where the
// overlap leaves off -- goes to out (room for lenL + lenR); returns its length,
// or 0 when the pair does not merge.
HERO_HD uint32_t merge_pair(const char *left, int lenL, const char *right, int lenR,
                            const uint32_t *extL, const uint32_t *extR, char *out) {
    char seqL[kOverhang], seqR[kOverhang];
    const int nL = overhang_letters(extL, seqL);
    const int nR = overhang_letters(extR, seqR);
    for (int i = 0; i < nR; i++) seqR[i] = complement_char(seqR[i]);  // getExtendComplementSequence
    int pl = 0;
    bool match = true;
    for (; pl < lenL; pl++) {
        const int old = pl;
        int pr = lenR - 1;
        match = true;
        for (; pr >= 0 && pl < lenL; pr--, pl++) {
            if (left[pl] != complement_char(right[pr])) {
                match = false;
                break;
            }
        }
        pl = old;
        if (match) break;
    }
    if (!(match && pl < lenL)) return 0;
    if (nL + nR + (lenL - pl) < 40) return 0;
    int mism = 0;
    for (int a = lenR - lenL + pl - 1, j = 0; a >= 0 && j < nL; j++, a--)
        if (complement_char(right[a]) != seqL[j]) mism++;
    for (int a = pl - 1, j = 0; a >= 0 && j < nR; j++, a--)
        if (left[a] != seqR[j]) mism++;
    if (mism > 0) return 0;
    int n = 0;
    for (int i = 0; i < lenL; i++) out[n++] = left[i];
    for (int a = lenR - lenL + pl - 1; a >= 0; a--) out[n++] = complement_char(right[a]);
    return uint32_t(n);
}

// length of a record's "id,orientation,position," prefix
HERO_HD uint32_t aln_prefix_len(uint64_t key, uint32_t orient, int64_t pos) {
    return dec_len(key) + 1u + dec_len(orient) + 1u + dec_len_signed(pos) + 1u;
}

// ---------------------------------------------------------------------------
// banded DP: BandAligner::bandedAlign / bandedAlignAffineGap (BandAligner.cpp:56-239)
//
// The matrix is computed in vertical strips of W columns held in registers,
// row by row.  A cell outside the band is forced to the sentinel for every
// state: the reference guards exactly the neighbours that fall outside the
// band with -MAXDUL (BandAligner.cpp:72,86,180,189), real scores are always
// far above any sentinel-derived value, and the direction rules never pick a
// sentinel option over a real one, so every in-band value and direction
// matches.  Row 0 and column 0 always trace left / up.
// ---------------------------------------------------------------------------
struct SegView {  // a DP segment after setSequences (rows = longer side)
    const uint8_t *row_base;  // DP "subject" (rows)
    const uint8_t *col_base;  // DP "query" (columns)
    int32_t row_dir, col_dir;  // +1 forward, -1 reverse-complement walk
    uint8_t row_xor, col_xor;  // 2 for reverse complement
    int32_t R, C;
    int64_t band;     // after widening to R - C
    bool right, left, reversed;

    HERO_HD uint8_t row(int32_t i) const { return uint8_t(row_base[int64_t(row_dir) * (i - 1)] ^ row_xor); }
    HERO_HD uint8_t col(int32_t j) const { return uint8_t(col_base[int64_t(col_dir) * (j - 1)] ^ col_xor); }
};

// builds the view of segment [s0,s1) of the subject (orientation rc when
// orient=1) against [q0,q1) of the query (of the query's reverse complement
// when qrc, for the alignment output's reverse pass; Lq = query length), as
// BandAligner::setSequences does
HERO_HD SegView make_view(const uint8_t *subj, int32_t Ls, int32_t orient, const uint8_t *qry,
                          int32_t s0, int32_t s1, int32_t q0, int32_t q1, uint32_t flags,
                          int64_t band_in, int32_t Lq = 0, bool qrc = false) {
    SegView v;
    const uint8_t *sb;
    int32_t sdir;
    uint8_t sx;
    if (orient) {  // position p of the reverse complement is comp(fwd[Ls-1-p])
        sb = subj + (Ls - 1 - s0);
        sdir = -1;
        sx = 2;
    } else {
        sb = subj + s0;
        sdir = 1;
        sx = 0;
    }
    const uint8_t *qb = qrc ? qry + (Lq - 1 - q0) : qry + q0;
    const int32_t qdir = qrc ? -1 : 1;
    const uint8_t qx = qrc ? 2 : 0;
    const int32_t ls = s1 - s0, lq = q1 - q0;
    if (lq <= ls) {
        v.row_base = sb;
        v.row_dir = sdir;
        v.row_xor = sx;
        v.col_base = qb;
        v.col_dir = qdir;
        v.col_xor = qx;
        v.R = ls;
        v.C = lq;
        v.reversed = false;
    } else {
        v.row_base = qb;
        v.row_dir = qdir;
        v.row_xor = qx;
        v.col_base = sb;
        v.col_dir = sdir;
        v.col_xor = sx;
        v.R = lq;
        v.C = ls;
        v.reversed = true;
    }
    int64_t d = int64_t(v.R) - v.C;
    v.band = band_in > d ? band_in : d;
    v.right = (flags & DPF_RIGHT) != 0;
    v.left = (flags & DPF_LEFT) != 0;
    return v;
}

// Cells of the reference's loop bounds (BandAligner.cpp:63-66): the sum over
// rows i = 0..R of min(C, i + m) - max(0, i - m) + 1.  With m >= R - C (the
// aligner widens its band to the length difference) every row is non-empty,
// so the sum splits into two arithmetic series.
HERO_HD uint64_t band_cells(int32_t R, int32_t C, int64_t m) {
    const int64_t r = R, c = C;
    int64_t hi;  // sum of min(C, i + m)
    const int64_t t = (c - m < r) ? c - m : r;  // last row with i + m <= C
    if (t >= 0) {
        hi = (t + 1) * m + t * (t + 1) / 2 + (r - t) * c;
    } else {
        hi = (r + 1) * c;
    }
    const int64_t k = r - m;  // rows with i > m contribute i - m to the sum of max(0, i - m)
    const int64_t lo = k > 0 ? k * (k + 1) / 2 : 0;
    return uint64_t(hi - lo + r + 1);
}

HERO_HD bool in_band(int32_t i, int32_t j, int32_t C, int64_t m) {
    return j <= C && int64_t(j) >= int64_t(i) - m && int64_t(j) <= int64_t(i) + m;
}

// State of one DP cell: FM, IX, IY (the global aligner uses f only).
struct Cell3 {
    int32_t f, x, y;
};

// Column 0 (BandAligner.cpp:75-79 with j == 0; affine init BandAligner.cpp:150-164)
template <bool AFFINE>
HERO_HD Cell3 dp_col0(const SegView &v, int32_t i) {
    if (i == 0) return AFFINE ? Cell3{0, kDX - kEX, kDX - kEX} : Cell3{0, 0, 0};
    if (int64_t(i) > v.band) return Cell3{kNEG, kNEG, kNEG};
    if (AFFINE) {
        if (v.right) return Cell3{0, 0, kDY};
        const int32_t z = kDX - kEX + i * kEX;
        return Cell3{z, z, z};
    }
    const int32_t z = i * (v.right ? kSX : kDX);
    return Cell3{z, z, z};
}

// Row 0 (BandAligner.cpp:58-126 with i == 0; affine init BandAligner.cpp:165-171)
template <bool AFFINE>
HERO_HD Cell3 dp_row0(const SegView &v, int32_t j) {
    if (j == 0) return dp_col0<AFFINE>(v, 0);
    if (j > v.C || int64_t(j) > v.band) return Cell3{kNEG, kNEG, kNEG};
    const int32_t z = AFFINE ? kDX - kEX + j * kEX : kDY * j;
    return Cell3{z, z, z};
}

// One row i of a strip of W columns j0+1 .. j0+W.
//   u*[w]  : states of row i-1 on entry, of row i on exit
//   left   : states at (i, j0) on entry, at (i, j0+W) on exit
//   dg     : states at (i-1, j0)
// Returns the row's traceback codes, 2 bits per cell: 0 up, 1 left, 2 diagonal
// mismatch, 3 diagonal match (the match bit spares the traceback the bases).
// FULL: the band covers every cell of the strip up to column C; cells past C
//       are then computed as if inside the matrix -- no cell at or left of
//       column C ever reads them, so they only cost time.
// LEFT: column wlast (0-based in the strip) is column C of an align-left
//       segment, whose vertical moves cost sx (BandAligner.cpp:69-82,190-196).
template <int W, bool AFFINE, bool FULL, bool LEFT>
HERO_HD uint32_t dp_strip_row(const SegView &v, int32_t i, int32_t j0, uint8_t a,
                              const uint8_t (&bc)[W], int32_t (&uf)[W], int32_t (&ux)[W],
                              int32_t (&uy)[W], Cell3 &left, Cell3 dg, int32_t wlast) {
    uint32_t bits = 0;
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const int32_t j = j0 + w + 1;
        const bool in = FULL || in_band(i, j, v.C, v.band);
        const bool lastcol = LEFT && (w == wlast);
        Cell3 c;
        uint32_t code;
        if (AFFINE) {
            if (in) {
                // IY: gap along the row (BandAligner.cpp:180-188)
                const int32_t y0 = left.f + kDY, y1 = left.y + kEX;
                c.y = y0 >= y1 ? y0 : y1;
                // IX: gap down the column (BandAligner.cpp:189-201)
                const int32_t x0 = uf[w] + (lastcol ? kSX : kDX);
                const int32_t x1 = ux[w] + (lastcol ? kSX : kEX);
                c.x = x1 > x0 ? x1 : x0;
                // FM = max3(FM, IX, IY)(i-1, j-1) + s (BandAligner.cpp:203-207)
                int32_t mm = dg.f >= dg.x ? dg.f : dg.x;
                mm = mm >= dg.y ? mm : dg.y;
                const bool eq = a == bc[w];
                c.f = mm + (eq ? kHIT : kMISS);
                // BM1 (BandAligner.cpp:214-222)
                code = (c.f > c.x && c.f >= c.y) ? (2u | uint32_t(eq)) : (c.y > c.x ? 1u : 0u);
            } else {
                c = Cell3{kNEG, kNEG, kNEG};
                code = 0;
            }
            dg = Cell3{uf[w], ux[w], uy[w]};
            uf[w] = c.f;
            ux[w] = c.x;
            uy[w] = c.y;
        } else {
            if (in) {
                // BandAligner.cpp:66-110: up, left, diag; diag wins ties, then left
                const int32_t vu = uf[w] + (lastcol ? kSX : kDX);
                const int32_t vl = left.f + kDY;
                const bool eq = a == bc[w];
                const int32_t vd = dg.f + (eq ? kHIT : kMISS);
                if (vd >= vl && vd >= vu) {
                    c.f = vd;
                    code = 2u | uint32_t(eq);
                } else if (vl >= vu) {
                    c.f = vl;
                    code = 1;
                } else {
                    c.f = vu;
                    code = 0;
                }
            } else {
                c.f = kNEG;
                code = 0;
            }
            c.x = c.y = c.f;
            dg.f = uf[w];
            uf[w] = c.f;
        }
        left = c;
        bits |= code << (2 * w);
    }
    return bits;
}

// 0-based position of column C in the strip starting after j0 when the segment
// aligns left, else -1
HERO_HD int32_t dp_strip_wlast(const SegView &v, int32_t j0, int32_t W) {
    const int32_t w = v.C - j0 - 1;
    return (v.left && w >= 0 && w < W) ? w : -1;
}

// dispatch on the strip's band coverage and align-left column
template <int W, bool AFFINE>
HERO_HD uint32_t dp_strip_row_any(bool full, int32_t wlast, const SegView &v, int32_t i,
                                  int32_t j0, uint8_t a, const uint8_t (&bc)[W], int32_t (&uf)[W],
                                  int32_t (&ux)[W], int32_t (&uy)[W], Cell3 &left, Cell3 dg) {
    if (full) {
        if (wlast >= 0) return dp_strip_row<W, AFFINE, true, true>(v, i, j0, a, bc, uf, ux, uy, left, dg, wlast);
        return dp_strip_row<W, AFFINE, true, false>(v, i, j0, a, bc, uf, ux, uy, left, dg, wlast);
    }
    if (wlast >= 0) return dp_strip_row<W, AFFINE, false, true>(v, i, j0, a, bc, uf, ux, uy, left, dg, wlast);
    return dp_strip_row<W, AFFINE, false, false>(v, i, j0, a, bc, uf, ux, uy, left, dg, wlast);
}

// strip setup: column codes and row-0 states of columns j0+1 .. j0+W
template <int W, bool AFFINE>
HERO_HD void dp_strip_init(const SegView &v, int32_t j0, uint8_t (&bc)[W], int32_t (&uf)[W],
                           int32_t (&ux)[W], int32_t (&uy)[W]) {
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const int32_t j = j0 + w + 1;
        bc[w] = j <= v.C ? v.col(j) : uint8_t(7);
        const Cell3 r = dp_row0<AFFINE>(v, j);
        uf[w] = r.f;
        ux[w] = r.x;
        uy[w] = r.y;
    }
}

// a strip is FULL when the band covers every cell of its columns up to C:
// |i - j| <= m for rows 1..R and columns j0+1 .. min(j0+W, C)
HERO_HD bool dp_strip_full(const SegView &v, int32_t j0, int32_t W) {
    const int64_t jl = j0 + W < v.C ? j0 + W : v.C;
    if (jl < j0 + 1) return true;
    return v.band >= int64_t(v.R) - (j0 + 1) && v.band >= jl - 1;
}

// ---------------------------------------------------------------------------
// Whole-band rows.  When the band covers the whole matrix (m >= R >= C; every
// segment of a typical correction) no cell is outside the band and column 0
// never holds the sentinel, so a row of a strip is the bare recurrence.  The
// stored state per column is (FM, IX, M) with M = max3(FM, IX, IY): IY is only
// ever read through that maximum (as the next row's diagonal input) and by the
// cell to its right.  The score of each column against each row base and the
// diagonal codes (2 | match) come from a per-strip table built once per
// segment: kTabWords 32-bit words, score[base][w] then diag[base].
// The global aligner keeps FM alone (M = FM).
// ---------------------------------------------------------------------------
constexpr int kTabWords = 36;

HERO_HD int32_t add_max(int32_t a, int32_t b, int32_t c) {  // max(a + b, c)
#if defined(__CUDA_ARCH__)
    return __viaddmax_s32(a, b, c);
#else
    return a + b > c ? a + b : c;
#endif
}

HERO_HD int32_t max3(int32_t a, int32_t b, int32_t c) {
#if defined(__CUDA_ARCH__)
    return __vimax3_s32(a, b, c);
#else
    const int32_t m = a > b ? a : b;
    return m > c ? m : c;
#endif
}

HERO_HD bool dp_whole_band(const SegView &v) { return v.band >= int64_t(v.R); }

// 0-based column of C in the last strip of an align-left segment, else -1
template <int W>
HERO_HD int32_t dp_left_col(const SegView &v) { return v.left ? (v.C - 1) % W : -1; }

// table of the strip j0+1 .. j0+W (columns past C never match)
template <int W>
HERO_HD void dp_whole_table(const SegView &v, int32_t j0, int32_t *tab) {
    uint32_t dg[4] = {0, 0, 0, 0};
    for (int32_t w = 0; w < W; w++) {
        const int32_t j = j0 + w + 1;
        const uint32_t b = j <= v.C ? v.col(j) : 7u;
        for (uint32_t c = 0; c < 4; c++) {
            const bool eq = b == c;
            tab[c * W + w] = eq ? kHIT : kMISS;
            dg[c] |= (2u | uint32_t(eq)) << (2 * w);
        }
    }
    for (int c = 0; c < 4; c++) tab[4 * W + c] = int32_t(dg[c]);
}

// row-0 states of the strip and the M state at (0, j0)
template <bool AFFINE, int W>
HERO_HD void dp_whole_init(const SegView &v, int32_t j0, int32_t (&f)[W], int32_t (&x)[W],
                           int32_t (&m)[W], int32_t &pm) {
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const Cell3 r = dp_row0<AFFINE>(v, j0 + w + 1);
        f[w] = r.f;
        x[w] = r.x;
        m[w] = AFFINE ? max3(r.f, r.x, r.y) : r.f;
    }
    const Cell3 r = dp_row0<AFFINE>(v, j0);
    pm = AFFINE ? max3(r.f, r.x, r.y) : r.f;
}

// column-0 states of row i >= 1 (dp_col0 inside the band) as i * mul + add:
// FM (and M) = i * c0[0] + c0[1], IY = i * c0[0] + c0[2]
template <bool AFFINE>
HERO_HD void dp_whole_col0(const SegView &v, int32_t (&c0)[3]) {
    if (AFFINE) {
        c0[0] = v.right ? 0 : kEX;
        c0[1] = v.right ? 0 : kDX - kEX;
        c0[2] = v.right ? kDY : kDX - kEX;
    } else {
        c0[0] = v.right ? kSX : kDX;
        c0[1] = 0;
        c0[2] = 0;
    }
}

// One row of a whole-band strip.  lf, ly: FM, IY at (i, j0) on entry, at
// (i, j0 + W) on exit; dm: M at (i-1, j0); m: M of row i-1 on entry, row i on
// exit.  The align-left column C (vertical moves cost sx there,
// BandAligner.cpp:189-201) is handled by the caller: FM and IX of the row above
// at that column feed only its IX, so raising them by sx - dx and sx - ex before
// the row (dp_whole_left) makes the same recurrence give its value and code.
template <bool AFFINE, int W>
HERO_HD uint32_t dp_whole_row(const int32_t (&sc)[W], uint32_t diag, int32_t (&f)[W],
                              int32_t (&x)[W], int32_t (&m)[W], int32_t &lf, int32_t &ly,
                              int32_t dm) {
    uint32_t dmask = 0, lbits = 0;
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const int32_t dx = kDX;
        if (AFFINE) {
            const int32_t ex = kEX;
            // BandAligner.cpp:180-188: max(FM + dy, IY + ex) of the cell to the left,
            // with the add on FM off the IY chain (one dependent op per column)
            const int32_t yv = add_max(ly, kEX, lf + kDY);
            const int32_t xv = add_max(f[w], dx, x[w] + ex);  // BandAligner.cpp:189-201
            const int32_t fv = dm + sc[w];                    // BandAligner.cpp:203-207
            dm = m[w];
            m[w] = max3(fv, xv, yv);
            if (fv > xv && fv >= yv) dmask |= 3u << (2 * w);  // BM1, BandAligner.cpp:214-222
            if (yv > xv) lbits |= 1u << (2 * w);
            f[w] = fv;
            x[w] = xv;
            lf = fv;
            ly = yv;
        } else {
            const int32_t vu = f[w] + dx, vl = lf + kDY, vd = dm + sc[w];  // BandAligner.cpp:66-110
            dm = f[w];
            const int32_t fv = max3(vd, vl, vu);
            if (vd >= vl && vd >= vu) dmask |= 3u << (2 * w);
            if (vl >= vu) lbits |= 1u << (2 * w);
            f[w] = fv;
            lf = fv;
        }
    }
    return (dmask & diag) | (~dmask & lbits);
}

// Before a row: the lane holding column C of an align-left segment raises the
// row-above FM and IX of that column (wl, 0-based in the strip) so that the
// plain recurrence charges sx for the vertical moves there.  wl is the same for
// the whole warp; the switch costs a uniform branch per row.
template <bool AFFINE, int W>
HERO_HD void dp_whole_left(int32_t wl, bool holds_c, int32_t (&f)[W], int32_t (&x)[W]) {
    if (!holds_c) return;
    switch (wl) {
#define HERO_LEFT_CASE(w)                        \
    case w:                                      \
        if (w < W) {                             \
            f[w < W ? w : 0] += kSX - kDX;       \
            if (AFFINE) x[w < W ? w : 0] += kSX - kEX; \
        }                                        \
        break;
        HERO_LEFT_CASE(0)
        HERO_LEFT_CASE(1)
        HERO_LEFT_CASE(2)
        HERO_LEFT_CASE(3)
        HERO_LEFT_CASE(4)
        HERO_LEFT_CASE(5)
        HERO_LEFT_CASE(6)
        HERO_LEFT_CASE(7)
#undef HERO_LEFT_CASE
        default:
            break;
    }
}

// ---------------------------------------------------------------------------
// Whole-band rows of two segments at once, tagged.  Every state is held as
// 4v + tag in a signed 16-bit half of a 32-bit register (segment A low, B
// high), so one DPX instruction advances a cell of each segment.  The tag, in
// the two low bits, names the move a value stands for, in the order that breaks
// the reference's ties, so the 3-way max of a cell's tagged candidates is at
// once its value (bits 2..15) and its traceback move (bits 0..1):
//   affine: IX (up, tag 2) beats FM (diagonal, tag 1) beats IY (left, tag 0)
//           on equal values -- BM1 is diagonal iff FM > IX && FM >= IY, else
//           left iff IY > IX, else up (BandAligner.cpp:214-222);
//   global: diagonal (tag 2) beats left (tag 1) beats up (tag 0) -- diagonal
//           if >= both, else left if >= up (BandAligner.cpp:99-110).
// The recurrences keep the tags right by construction: the affine FM carries
// tag 1 (diagonal input M is stored clean, the score adds 4s + 1), IX tag 2
// (FM + 4dx + 1 and IX + 4ex), IY tag 0 (FM + 4dy - 1 and IY + 4ex); the
// global F and the affine M are stored clean (tag masked off) and each
// candidate adds its tag.  Per cell that leaves one mask for the move, one
// shift-add into the row's code word and one mask for the clean value.
// Two segments share a lane when they have the same rows, strips and
// align-left column (the shape key), so their wavefronts run in lockstep.
// Every real value of a whole-band matrix lies in [-4(R+C) - 3, R], so with
// R + C <= kPairMaxSide no half ever wraps; columns past C start at kPairPad
// and are never read by a real cell (only cells to their right read them).
// ---------------------------------------------------------------------------
constexpr int32_t kPairPad = -8192;
constexpr int32_t kPairMaxSide = 2000;  // R + C of a segment in a packed pair
constexpr int kTabWords2 = 40;          // per lane: int16 tagged scores [2][4][8], eq words [2][4]
constexpr uint32_t kTagMask2 = 0x00030003u;
constexpr uint32_t kLow2 = 0x55555555u;  // the low bit of every 2-bit field

HERO_HD uint32_t pack2(int32_t lo, int32_t hi) { return (uint32_t(lo) & 0xffffu) | (uint32_t(hi) << 16); }
HERO_HD uint32_t pack2s(int32_t v) { return pack2(v, v); }
HERO_HD int32_t half_lo(uint32_t v) { return int32_t(int16_t(uint16_t(v & 0xffffu))); }
HERO_HD int32_t half_hi(uint32_t v) { return int32_t(int16_t(uint16_t(v >> 16))); }

// per half: max(a + b, c)
HERO_HD uint32_t add_max2(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
    return __viaddmax_s16x2(a, b, c);
#else
    const int32_t l = int16_t(uint16_t(half_lo(a) + half_lo(b))), h = int16_t(uint16_t(half_hi(a) + half_hi(b)));
    return pack2(l > half_lo(c) ? l : half_lo(c), h > half_hi(c) ? h : half_hi(c));
#endif
}

// per half: a + b (the floor of the add-max is never reached)
HERO_HD uint32_t add2(uint32_t a, uint32_t b) { return add_max2(a, b, 0x80008000u); }

// per half: max(a, b, c)
HERO_HD uint32_t max3_2(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
    return __vimax3_s16x2(a, b, c);
#else
    const int32_t l = max3(half_lo(a), half_lo(b), half_lo(c));
    const int32_t h = max3(half_hi(a), half_hi(b), half_hi(c));
    return pack2(l, h);
#endif
}

// the tag a candidate of each move adds (see above)
template <bool AFFINE>
struct PairTags {
    static constexpr int32_t diag = AFFINE ? 1 : 2, left = AFFINE ? 0 : 1, up = AFFINE ? 2 : 0;
};

// Tables of strip j0+1 .. j0+W for segments A and B: the tagged diagonal
// increment 4s + tag per base (tab16[seg][base][w]; columns past C never
// match) and the match bits per base (words 32..: A's in the low 16 bits,
// B's in the high, bit 2w for column w).
template <bool AFFINE, int W>
HERO_HD void dp_pair_table(const SegView &va, const SegView &vb, int32_t j0, uint32_t *tab) {
    uint16_t *sc = reinterpret_cast<uint16_t *>(tab);
    for (int h = 0; h < 2; h++) {
        const SegView &v = h ? vb : va;
        uint32_t eq[4] = {0, 0, 0, 0};
        for (int32_t w = 0; w < W; w++) {
            const int32_t j = j0 + w + 1;
            const uint32_t b = j <= v.C ? v.col(j) : 7u;
            for (uint32_t c = 0; c < 4; c++) {
                const bool e = b == c;
                sc[(h * 4 + c) * W + w] = uint16_t(int16_t(4 * (e ? kHIT : kMISS) + PairTags<AFFINE>::diag));
                eq[c] |= uint32_t(e) << (2 * w);
            }
        }
        for (int c = 0; c < 4; c++) tab[32 + h * 4 + c] = eq[c] << (16 * h);
    }
}

// row-0 states of the strip (tagged) and the clean M (global: F) at (0, j0)
template <bool AFFINE, int W>
HERO_HD void dp_pair_init(const SegView &va, const SegView &vb, int32_t j0, uint32_t (&f)[W],
                          uint32_t (&x)[W], uint32_t (&m)[W], uint32_t &pm) {
    using T = PairTags<AFFINE>;
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const int32_t j = j0 + w + 1;
        int32_t fa = kPairPad, fb = kPairPad, xa = kPairPad, xb = kPairPad, ma = kPairPad, mb = kPairPad;
        if (j <= va.C) {
            const Cell3 r = dp_row0<AFFINE>(va, j);
            fa = AFFINE ? 4 * r.f + T::diag : 4 * r.f;
            xa = 4 * r.x + T::up;
            ma = 4 * (AFFINE ? max3(r.f, r.x, r.y) : r.f);
        }
        if (j <= vb.C) {
            const Cell3 r = dp_row0<AFFINE>(vb, j);
            fb = AFFINE ? 4 * r.f + T::diag : 4 * r.f;
            xb = 4 * r.x + T::up;
            mb = 4 * (AFFINE ? max3(r.f, r.x, r.y) : r.f);
        }
        f[w] = pack2(fa, fb);
        x[w] = pack2(xa, xb);
        m[w] = pack2(ma, mb);
    }
    const Cell3 a = dp_row0<AFFINE>(va, j0), b = dp_row0<AFFINE>(vb, j0);
    pm = AFFINE ? pack2(4 * max3(a.f, a.x, a.y), 4 * max3(b.f, b.x, b.y)) : pack2(4 * a.f, 4 * b.f);
}

// Column-0 states of a pair, row 1, tagged as the recurrences read them: lf
// (affine FM, tag 1; global F, clean), ly (affine IY, tag 0) and the per-row
// increment (dp_whole_col0: FM = i * c0[0] + c0[1], IY = i * c0[0] + c0[2]).
// The clean M (global: F) of column 0 is lf minus its tag: M = FM there.
template <bool AFFINE>
HERO_HD void dp_pair_col0(const SegView &va, const SegView &vb, uint32_t &c0f, uint32_t &c0y,
                          uint32_t &mul) {
    int32_t ca[3], cb[3];
    dp_whole_col0<AFFINE>(va, ca);
    dp_whole_col0<AFFINE>(vb, cb);
    const int32_t t = PairTags<AFFINE>::diag * int32_t(AFFINE);
    mul = pack2(4 * ca[0], 4 * cb[0]);
    c0f = pack2(4 * (ca[0] + ca[1]) + t, 4 * (cb[0] + cb[1]) + t);
    c0y = pack2(4 * (ca[0] + ca[2]), 4 * (cb[0] + cb[2]));
}

// One row of a pair (dp_whole_row on both halves, tagged).  Returns the
// traceback codes (0 up, 1 left, 2 diagonal mismatch, 3 diagonal match) of A
// in the low 16 bits and of B in the high 16 bits; eq holds the match bits of
// both rows' bases (dp_pair_table's words).
template <bool AFFINE, int W>
HERO_HD uint32_t dp_pair_row(const uint32_t (&sc)[W], uint32_t eq, uint32_t (&f)[W],
                             uint32_t (&x)[W], uint32_t (&m)[W], uint32_t &lf, uint32_t &ly,
                             uint32_t dm) {
    uint32_t acc = 0;
    if (AFFINE) {
        constexpr uint32_t DYT = (uint32_t(4 * kDY - 1) & 0xffffu) * 0x10001u;  // FM(tag 1) -> IY (tag 0)
        constexpr uint32_t DXT = (uint32_t(4 * kDX + 1) & 0xffffu) * 0x10001u;  // FM(tag 1) -> IX (tag 2)
        constexpr uint32_t EX4 = (uint32_t(4 * kEX) & 0xffffu) * 0x10001u;
#pragma unroll
        for (int32_t w = 0; w < W; w++) {
            const uint32_t yv = add_max2(ly, EX4, add2(lf, DYT));      // BandAligner.cpp:180-188
            const uint32_t xv = add_max2(f[w], DXT, add2(x[w], EX4));  // BandAligner.cpp:189-201
            const uint32_t fv = add2(dm, sc[w]);                       // BandAligner.cpp:203-207
            dm = m[w];
            const uint32_t mt = max3_2(fv, xv, yv);
            acc += (mt & kTagMask2) << (2 * w);
            m[w] = mt & ~kTagMask2;
            f[w] = fv;
            x[w] = xv;
            lf = fv;
            ly = yv;
        }
        // tags (2 up, 1 diagonal, 0 left) to codes: the low tag bit is the
        // diagonal bit, the match bit joins it there; tag 0 becomes left
        const uint32_t L = acc & kLow2;
        const uint32_t lft = ~(acc | (acc >> 1)) & kLow2;
        return (L << 1) | (L & eq) | lft;
    }
    constexpr uint32_t DX4 = (uint32_t(4 * kDX) & 0xffffu) * 0x10001u;      // up: tag 0
    constexpr uint32_t DYT = (uint32_t(4 * kDY + 1) & 0xffffu) * 0x10001u;  // left: tag 1
#pragma unroll
    for (int32_t w = 0; w < W; w++) {
        const uint32_t vd = add2(dm, sc[w]);  // diagonal, tag 2 (BandAligner.cpp:66-110)
        dm = f[w];
        const uint32_t mt = add_max2(lf, DYT, add_max2(f[w], DX4, vd));
        acc += (mt & kTagMask2) << (2 * w);
        f[w] = mt & ~kTagMask2;
        lf = f[w];
    }
    // tags (2 diagonal, 1 left, 0 up) are the codes; the match bit joins the diagonals
    return acc | ((acc >> 1) & eq);
}

// the align-left column of a pair (both segments share it): dp_whole_left on
// both halves, scaled by 4 (tags unchanged)
template <bool AFFINE, int W>
HERO_HD void dp_pair_left(int32_t wl, bool holds_c, uint32_t (&f)[W], uint32_t (&x)[W]) {
    if (!holds_c) return;
    constexpr uint32_t SD2 = (uint32_t(4 * (kSX - kDX)) & 0xffffu) * 0x10001u;
    constexpr uint32_t SE2 = (uint32_t(4 * (kSX - kEX)) & 0xffffu) * 0x10001u;
    switch (wl) {
#define HERO_PAIR_CASE(w)                                               \
    case w:                                                             \
        if (w < W) {                                                    \
            f[w < W ? w : 0] = add2(f[w < W ? w : 0], SD2);             \
            if (AFFINE) x[w < W ? w : 0] = add2(x[w < W ? w : 0], SE2); \
        }                                                               \
        break;
        HERO_PAIR_CASE(0)
        HERO_PAIR_CASE(1)
        HERO_PAIR_CASE(2)
        HERO_PAIR_CASE(3)
        HERO_PAIR_CASE(4)
        HERO_PAIR_CASE(5)
        HERO_PAIR_CASE(6)
        HERO_PAIR_CASE(7)
#undef HERO_PAIR_CASE
        default:
            break;
    }
}

// Whole-matrix fill by one thread, strip after strip.  Scratch provides
//   int32_t& b(int32_t state, int32_t row)          boundary column, state 0..2
//   void tb_set(int32_t strip, int32_t row, uint32_t bits)  traceback codes of a
//   uint32_t tb_get(int32_t strip, int32_t row)             row, 2 bits per cell
template <int W, bool AFFINE, class Scratch>
HERO_HD void dp_fill(const SegView &v, Scratch &sc) {
    const int32_t R = v.R, C = v.C;
    for (int32_t i = 0; i <= R; i++) {
        const Cell3 c = dp_col0<AFFINE>(v, i);
        sc.b(0, i) = c.f;
        sc.b(1, i) = c.x;
        sc.b(2, i) = c.y;
    }
    const int32_t nst = (C + W - 1) / W;
    for (int32_t s = 0; s < nst; s++) {
        const int32_t j0 = s * W;
        uint8_t bc[W];
        int32_t uf[W], ux[W], uy[W];
        dp_strip_init<W, AFFINE>(v, j0, bc, uf, ux, uy);
        const bool full = dp_strip_full(v, j0, W);
        const int32_t wlast = dp_strip_wlast(v, j0, W);
        Cell3 dg{sc.b(0, 0), sc.b(1, 0), sc.b(2, 0)};
        for (int32_t i = 1; i <= R; i++) {
            Cell3 left{sc.b(0, i), sc.b(1, i), sc.b(2, i)};
            const Cell3 lb = left;
            const uint8_t a = v.row(i);
            const uint32_t bits =
                dp_strip_row_any<W, AFFINE>(full, wlast, v, i, j0, a, bc, uf, ux, uy, left, dg);
            sc.tb_set(s, i, bits);
            sc.b(0, i) = left.f;
            sc.b(1, i) = left.x;
            sc.b(2, i) = left.y;
            dg = lb;
        }
        const Cell3 r0 = dp_row0<AFFINE>(v, j0 + W);
        sc.b(0, 0) = r0.f;
        sc.b(1, 0) = r0.x;
        sc.b(2, 0) = r0.y;
    }
}

// Op of each move code: up, left, diagonal mismatch, diagonal match (the
// rows hold the longer segment; reversed = the query is on the rows).
HERO_HD uint32_t dp_op_lut(const SegView &v) {
    return uint32_t(v.reversed ? OP_I : OP_D) | (uint32_t(v.reversed ? OP_D : OP_I) << 2) |
           (uint32_t(OP_X) << 4) | (uint32_t(OP_M) << 6);
}

// Traceback (BandAligner.cpp:114-125 / 227-238) from (R, C) to (0, 0).
// emit(op) receives ops last-to-first; returns the path length.
template <int W, class Scratch, class Emit>
HERO_HD int32_t dp_walk(const SegView &v, const Scratch &sc, Emit &emit) {
    int32_t i = v.R, j = v.C, n = 0;
    const uint32_t lut = dp_op_lut(v);
    while (i > 0 || j > 0) {
        // row 0 traces left, column 0 up; inside, the code names the move
        uint32_t code = i == 0 ? 1u : 0u;
        if (i > 0 && j > 0) {
            const uint32_t jj = uint32_t(j - 1);
            code = (sc.tb_get(int32_t(jj / W), i) >> (2 * (jj % W))) & 3u;
        }
        i -= code != 1u;
        j -= code != 0u;
        emit(uint8_t((lut >> (2 * code)) & 3u));
        n++;
    }
    return n;
}

// ---------------------------------------------------------------------------
// Traceback in row chunks, for the lanes of a wavefront group.  The path from
// (R, C) to (0, 0) visits every row; lane s of G takes the moves that start in
// rows (rbot, rtop] (the last chunk also takes the left moves along row 0).
// A lane starts from a guessed column, walks its chunk, and is right once its
// start equals the end of the lane before it (the true path enters row rtop
// there); lanes that are not get new guesses and walk again.  Moves are the
// ones dp_walk makes, so the concatenated chunks are its path exactly.
// ---------------------------------------------------------------------------
HERO_HD void dp_chunk_rows(int32_t R, int32_t G, int32_t s, int32_t &rtop, int32_t &rbot) {
    const int32_t h = (R + G - 1) / G;
    rtop = R - s * h > 0 ? R - s * h : 0;
    rbot = R - (s + 1) * h > 0 ? R - (s + 1) * h : 0;
}

// First guess of the column where the path meets row rtop.  An align-left
// segment climbs column C for free (vertical moves there cost sx), then runs
// diagonally to (0, 0): column min(rtop, C).  Otherwise the path runs
// diagonally from (R, C) (an align-right segment then climbs column 0).
HERO_HD int32_t dp_chunk_guess(const SegView &v, int32_t rtop) {
    if (v.left) return rtop < v.C ? rtop : v.C;
    const int32_t c = v.C - (v.R - rtop);
    return c > 0 ? c : 0;
}

// Walks from (i, j) while i > stop (column 0 moves up); with stop == 0 it also
// makes the left moves along row 0.  Returns the number of moves; j is left at
// the end column.
template <int W, class Scratch>
HERO_HD int32_t dp_walk_span(const Scratch &sc, int32_t i, int32_t &j, int32_t stop) {
    int32_t n = 0;
    while (i > stop) {
        uint32_t code = 0u;
        if (j > 0) {
            const uint32_t jj = uint32_t(j - 1);
            code = (sc.tb_get(int32_t(jj / W), i) >> (2 * (jj % W))) & 3u;
        }
        i -= code != 1u;
        j -= code != 0u;
        n++;
    }
    if (stop == 0) {
        n += j;
        j = 0;
    }
    return n;
}

// the same moves, handing each op to put() in walk order
template <int W, class Scratch, class Put>
HERO_HD void dp_walk_span_ops(const Scratch &sc, uint32_t lut, int32_t i, int32_t j, int32_t stop,
                              Put &put) {
    while (i > stop) {
        uint32_t code = 0u;
        if (j > 0) {
            const uint32_t jj = uint32_t(j - 1);
            code = (sc.tb_get(int32_t(jj / W), i) >> (2 * (jj % W))) & 3u;
        }
        i -= code != 1u;
        j -= code != 0u;
        put((lut >> (2 * code)) & 3u);
    }
    if (stop == 0)
        for (; j > 0; j--) put((lut >> 2) & 3u);
}

// DpSum of the ops at positions [first, first + P) of a packed op array (16
// ops per word, op at position p in word p / 16, bits 2 (p % 16)), by counting
// 2-bit fields a word at a time.
HERO_HD uint32_t ops_field(const uint32_t *w, uint32_t p) { return (w[p >> 4] >> (2 * (p & 15))) & 3u; }

HERO_HD uint32_t ops_mask(uint32_t lo, uint32_t hi) {  // 0x55.. pattern over fields lo..hi
    return 0x55555555u & (0xffffffffu << (2 * lo)) & (0xffffffffu >> (30 - 2 * hi));
}

HERO_HD int32_t popc32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}

// index of the lowest / highest set bit of x != 0
HERO_HD int32_t low_bit(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs(int(x)) - 1;
#else
    return __builtin_ctz(x);
#endif
}
HERO_HD int32_t high_bit(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return 31 - __clz(int(x));
#else
    return 31 - __builtin_clz(x);
#endif
}

// What the words k0 + s, k0 + s + G, ... of an op range [first, first + P)
// contribute to its DpSum: op counts of kinds 1..3, the first field that
// differs from the range's first op (fpos, ~0u: none) and one past the last
// field that differs from its last op (lpos, 0: none).  Parts of disjoint word
// sets merge (ops_part_merge), so G lanes can each take every G-th word.
struct OpsPart {
    int32_t c1, c2, c3;
    uint32_t fpos, lpos;
};

HERO_HD OpsPart ops_part(const uint32_t *w, uint32_t first, uint32_t P, uint32_t s, uint32_t G) {
    OpsPart r{0, 0, 0, ~0u, 0u};
    if (P == 0) return r;
    const uint32_t end = first + P, k0 = first >> 4, k1 = (end - 1) >> 4;
    const uint32_t f = ops_field(w, first) * 0x55555555u, l = ops_field(w, end - 1) * 0x55555555u;
    for (uint32_t k = k0 + s; k <= k1; k += G) {
        const uint32_t m = ops_mask(k == k0 ? (first & 15) : 0, k == k1 ? ((end - 1) & 15) : 15);
        const uint32_t x = w[k], xl = x & 0x55555555u, xh = (x >> 1) & 0x55555555u;
        r.c1 += popc32(xl & ~xh & m);
        r.c2 += popc32(xh & ~xl & m);
        r.c3 += popc32(xl & xh & m);
        const uint32_t yf = x ^ f, zf = (yf | (yf >> 1)) & m;
        if (zf && r.fpos == ~0u) r.fpos = (k << 4) + uint32_t(low_bit(zf) >> 1);  // words rise: the first is the least
        const uint32_t yl = x ^ l, zl = (yl | (yl >> 1)) & m;
        if (zl) r.lpos = (k << 4) + uint32_t(high_bit(zl) >> 1) + 1u;  // the last is the greatest
    }
    return r;
}

HERO_HD OpsPart ops_part_merge(OpsPart a, const OpsPart &b) {
    a.c1 += b.c1;
    a.c2 += b.c2;
    a.c3 += b.c3;
    a.fpos = b.fpos < a.fpos ? b.fpos : a.fpos;
    a.lpos = b.lpos > a.lpos ? b.lpos : a.lpos;
    return a;
}

// the DpSum of the range from the merged part of all its words
HERO_HD void ops_part_sum(const OpsPart &p, const uint32_t *w, uint32_t first, uint32_t P,
                          DpSum &sum) {
    const uint32_t end = first + P;
    sum.tot[0] = uint16_t(int32_t(P) - p.c1 - p.c2 - p.c3);
    sum.tot[1] = uint16_t(p.c1);
    sum.tot[2] = uint16_t(p.c2);
    sum.tot[3] = uint16_t(p.c3);
    // first run: fields equal to the first op, from `first` on; last run:
    // fields equal to the last op, backwards from end - 1
    const uint32_t fc = p.fpos == ~0u ? P : p.fpos - first;
    const uint32_t lc = p.lpos == 0u ? P : end - p.lpos;
    sum.ft = uint8_t(P ? ops_field(w, first) : 0u);
    sum.fc = uint16_t(fc);
    sum.lt = uint8_t(P ? ops_field(w, end - 1) : 0u);
    sum.lc = uint16_t(lc);
    sum.nruns = fc == P ? 1 : 2;
    sum.pad = 0;
}

HERO_HD void ops_summary(const uint32_t *w, uint32_t first, uint32_t P, DpSum &sum) {
    ops_part_sum(ops_part(w, first, P, 0, 1), w, first, P, sum);
}

// walk + per-op run tracking, for callers that emit ops one by one
template <int W, class Scratch, class Emit>
HERO_HD int32_t dp_traceback(const SegView &v, Scratch &sc, Emit &emit, DpSum &sum) {
    uint64_t tot = 0;  // four 16-bit op counters (path length < 65536)
    uint32_t cur = 0xffu, cc = 0, lt = 0, lc = 0;
    int32_t nr = 0;
    auto track = [&](uint8_t op) {
        emit(op);
        tot += 1ull << (16 * op);
        if (op == cur) {
            cc++;
        } else {
            if (cc > 0) {
                if (nr == 0) {
                    lt = cur;
                    lc = cc;
                }
                nr++;
            }
            cur = op;
            cc = 1;
        }
    };
    const int32_t nops = dp_walk<W>(v, sc, track);
    // the run open at the end of the walk is the first run of the path
    sum.ft = uint8_t(cur);
    sum.fc = uint16_t(cc);
    if (nr == 0) {
        sum.lt = uint8_t(cur);
        sum.lc = uint16_t(cc);
        sum.nruns = 1;
    } else {
        sum.lt = uint8_t(lt);
        sum.lc = uint16_t(lc);
        sum.nruns = 2;
    }
    sum.tot[0] = uint16_t(tot);
    sum.tot[1] = uint16_t(tot >> 16);
    sum.tot[2] = uint16_t(tot >> 32);
    sum.tot[3] = uint16_t(tot >> 48);
    sum.pad = 0;
    return nops;
}

// ---------------------------------------------------------------------------
// consensus of one column: QueryRead::callConsensus (QueryRead.cpp:148-180)
// c[] already includes the read's own vote.  Returns the new code, or -1 to
// keep the base.
// ---------------------------------------------------------------------------
// The reference divides every count by the sum and keeps the largest fraction
// and the one it replaced.  For sum > 0 the fractions compare as the counts do
// (two different counts differ by at least 1/sum, far above the rounding), so
// the scan runs on the counts and only the two kept fractions are divided, with
// the same operands and rounding.  With sum == 0 no fraction is ever larger.
HERO_HD int32_t column_consensus(const uint32_t c[4], double thr) {
    double sum = 0;
    for (int j = 0; j < 4; j++) sum = HERO_DADD(sum, double(c[j]));
    int32_t id = -1;
    uint32_t largest = 0, larger = 0;  // counts behind fLargest, fLarger
    for (int j = 0; j < 4; j++) {
        if (largest < c[j]) {
            larger = largest;
            largest = c[j];
            id = j;
        }
    }
    if (id < 0) return -1;  // no count above 0: the reference keeps id -1 too
    const double fLargest = HERO_DDIV(double(largest), sum);
    const double fLarger = HERO_DDIV(double(larger), sum);
    if (HERO_DSUB(fLargest, fLarger) >= thr) return id;
    return -1;
}

}  // namespace hero
