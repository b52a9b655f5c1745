/*
 * hero_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see hero_oracle.h).
 *
 * A plain CPU restatement of HERO's consensus-mode correction path
 * (guo-xuan/Hero, src/).  Each function names the reference lines it follows.
 * Scores are the reference's integer-valued doubles held in int (every value
 * is a small integer, so the arithmetic and every comparison are identical).
 */
#include "hero_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// BandAligner.h:18 and BandAligner::setCost (BandAligner.cpp:528-542)
const int MAXDUL = 100000;
const int DX = -4, DY = -4, MISS = -4, HIT = 1, UNOBSERVED = -1, SX = 0, EX = -1;
const int SI[3] = {-1, 0, -1};
const int SJ[3] = {0, -1, -1};
const char CWILD = 'N';
const char ADNA[4] = {'A', 'C', 'T', 'G'};  // QueryRead.cpp:11

struct Params {
    int64_t k, l;
    bool affine, keep_segments;
    bool aln;  // alignment output (no -c): SubjectReadAligner::writeToFile
    bool merge;  // --merge: overhang votes and paired-read merging
    bool mapping;  // --mapping: the best covering record per subject, a coverage histogram
    double mis_rate, indel_rate, thr;
};

// -------------------------------------------------------------------------
// BandAligner (BandAligner.cpp)
// -------------------------------------------------------------------------
struct Band {
    bool affine = false;
    int64_t m_band = 0;
    std::string subj, qry;       // cSubjectSeq / cQuerySeq
    int64_t s_start = 0, q_start = 0;
    bool reversed = false, right = false, left = false;
    std::vector<int> FM, IX, IY;
    std::vector<signed char> BM;
    std::vector<int> edit;
    int ei = 0;
    std::vector<char> ctype;      // vCigarType
    std::vector<int> ccount;      // vCigarCount
    uint64_t cells = 0;

    // setSequences (BandAligner.cpp:559-573); end is exclusive
    void setSequences(const std::string &S, int64_t s0, int64_t s1, const std::string &Q,
                      int64_t q0, int64_t q1) {
        if (q1 - q0 <= s1 - s0) {
            qry.assign(Q, q0, q1 > q0 ? q1 - q0 : 0);
            subj.assign(S, s0, s1 > s0 ? s1 - s0 : 0);
            reversed = false;
        } else {
            qry.assign(S, s0, s1 > s0 ? s1 - s0 : 0);
            subj.assign(Q, q0, q1 > q0 ? q1 - q0 : 0);
            reversed = true;
        }
        s_start = s0;
        q_start = q0;
        left = right = false;
    }

    void alloc(int R, int C) {
        size_t n = size_t(R + 1) * size_t(C + 1);
        if (FM.size() < n) {
            FM.resize(n);
            BM.resize(n);
            IX.resize(n);
            IY.resize(n);
        }
        if (edit.size() < size_t(R + C + 1)) edit.resize(R + C + 1);
    }

    // bandedAlign (BandAligner.cpp:56-126)
    void bandedAlign() {
        const int R = int(subj.size()), C = int(qry.size()), W = C + 1;
        alloc(R, C);
        FM[0] = 0;
        BM[0] = 0;
        int64_t id = R - C;
        if (id > m_band) m_band = id;
        for (int i = 0; i <= R; i++) {
            int64_t lm = 0 > i - m_band ? 0 : i - m_band;
            int64_t rm = C < i + m_band ? C : i + m_band;
            if (rm >= lm) cells += uint64_t(rm - lm + 1);
            for (int64_t j = lm; j <= rm; j++) {
                if (i == 0 && j == 0) continue;
                int v0 = -MAXDUL, v1 = -MAXDUL, v2 = -MAXDUL;
                if (i > 0 && j < i + m_band) {
                    v0 = FM[size_t(i - 1) * W + j];
                    if (j > 0 && j < C) {
                        v0 += DX;
                    } else if (j == 0 && right) {
                        v0 += SX;
                    } else if (j >= C && left) {
                        v0 += SX;
                    } else {
                        v0 += DX;
                    }
                }
                if (j > lm) v1 = DY + FM[size_t(i) * W + j - 1];
                if (i > 0 && j > 0) {
                    char a = subj[i - 1], b = qry[j - 1];
                    v2 = FM[size_t(i - 1) * W + j - 1] +
                         (a != b ? ((a == CWILD || b == CWILD) ? UNOBSERVED : MISS) : HIT);
                }
                size_t c = size_t(i) * W + j;
                if (v2 >= v1 && v2 >= v0) {
                    FM[c] = v2;
                    BM[c] = 2;
                } else if (v1 >= v0) {
                    FM[c] = v1;
                    BM[c] = 1;
                } else {
                    FM[c] = v0;
                    BM[c] = 0;
                }
            }
        }
        traceback(R, C);
    }

    // bandedAlignAffineGap (BandAligner.cpp:139-239); max3 (BandAligner.cpp:128-137)
    void bandedAlignAffineGap() {
        const int R = int(subj.size()), C = int(qry.size()), W = C + 1;
        alloc(R, C);
        FM[0] = 0;
        IX[0] = DX - EX;
        IY[0] = DX - EX;
        BM[0] = 0;
        int64_t id = R - C;
        if (id > m_band) m_band = id;
        int64_t rmax = R < m_band ? R : m_band;
        for (int64_t i = 1; i <= rmax; i++) {
            size_t c = size_t(i) * W, u = size_t(i - 1) * W;
            if (right) {
                IX[c] = FM[u] + SX;
                IY[c] = DY;
                FM[c] = IX[c];
            } else {
                IX[c] = IX[u] + EX;
                IY[c] = IX[c];
                FM[c] = IX[c];
            }
            BM[c] = 0;
        }
        int64_t cmax = C < m_band ? C : m_band;
        for (int64_t j = 1; j <= cmax; j++) {
            IY[j] = IY[j - 1] + EX;
            IX[j] = IY[j];
            FM[j] = IY[j];
            BM[j] = 1;
        }
        for (int i = 0; i <= R; i++) {  // cell count with the same bounds as bandedAlign
            int64_t lm = 0 > i - m_band ? 0 : i - m_band;
            int64_t rm = C < i + m_band ? C : i + m_band;
            if (rm >= lm) cells += uint64_t(rm - lm + 1);
        }
        for (int i = 1; i <= R; i++) {
            int64_t lm = 0 > i - m_band ? 0 : i - m_band;
            int64_t rm = C < i + m_band ? C : i + m_band;
            for (int64_t j = lm; j <= rm; j++) {
                if (j == 0) continue;
                size_t c = size_t(i) * W + j, u = size_t(i - 1) * W + j;
                if (j == lm) {
                    IY[c] = -MAXDUL;
                } else {
                    int t0 = FM[c - 1] + DY, t1 = IY[c - 1] + EX;
                    IY[c] = t0 >= t1 ? t0 : t1;
                }
                if (j == rm && i + m_band <= rm) {
                    IX[c] = -MAXDUL;
                } else if (left && j >= C) {
                    int t0 = FM[u] + SX, t1 = IX[u] + SX;
                    IX[c] = t1 > t0 ? t1 : t0;
                } else {
                    int t0 = FM[u] + DX, t1 = IX[u] + EX;
                    IX[c] = t1 > t0 ? t1 : t0;
                }
                int s = subj[i - 1] != qry[j - 1] ? MISS : HIT;
                int x = FM[u - 1] + s, y = IX[u - 1] + s, z = IY[u - 1] + s;
                FM[c] = (x >= y && x >= z) ? x : ((y >= x && y >= z) ? y : z);
                if (FM[c] > IX[c] && FM[c] >= IY[c]) {
                    BM[c] = 2;
                } else if (IY[c] > IX[c]) {
                    BM[c] = 1;
                } else {
                    BM[c] = 0;
                }
            }
        }
        traceback(R, C);
    }

    // traceback loop shared by both aligners (BandAligner.cpp:114-125, 227-238)
    void traceback(int R, int C) {
        const int W = C + 1;
        ei = R + C;
        int i = R, j = C;
        int id = BM[size_t(i) * W + j];
        while (true) {
            edit[--ei] = SJ[id] - SI[id];
            i += SI[id];
            j += SJ[id];
            id = BM[size_t(i) * W + j];
            if (i == 0 && j == 0) break;
        }
    }

    // calculateCigarAndPosition(Reversed) (BandAligner.cpp:258-419)
    void cigar() {
        ctype.clear();
        ccount.clear();
        const int editLen = int(subj.size() + qry.size());
        int si = 0, qi = 0;
        char cur = 0;
        int cnt = 0;
        const char on_minus = reversed ? 'D' : 'I';
        const char on_plus = reversed ? 'I' : 'D';
        for (int i = ei; i < editLen; i++) {
            char t;
            if (edit[i] == -1) {
                t = on_minus;
                qi++;
            } else if (edit[i] == 0) {
                if (qry[qi] == subj[si]) {
                    t = 'M';
                } else {
                    t = reversed ? subj[si] : qry[qi];
                    // a mismatch always opens a new entry (BandAligner.cpp:313-318)
                    if (i != ei) {
                        ccount.push_back(cnt);
                        ctype.push_back(cur);
                    }
                    cur = t;
                    cnt = 1;
                    qi++;
                    si++;
                    continue;
                }
                qi++;
                si++;
            } else {
                t = on_plus;
                si++;
            }
            if (i == ei) {
                cur = t;
                cnt = 1;
            } else if (t == cur) {
                cnt++;
            } else {
                ccount.push_back(cnt);
                ctype.push_back(cur);
                cur = t;
                cnt = 1;
            }
        }
        ccount.push_back(cnt);
        ctype.push_back(cur);
    }

    // calculateAlignment (BandAligner.cpp:241-256)
    void calculateAlignment() {
        if (affine) {
            bandedAlignAffineGap();
        } else {
            bandedAlign();
        }
        cigar();
    }

    // per-step ops in original orientation
    void steps(std::vector<uint8_t> &out) const {
        const int editLen = int(subj.size() + qry.size());
        int si = 0, qi = 0;
        for (int i = ei; i < editLen; i++) {
            if (edit[i] == -1) {
                out.push_back(reversed ? HERO_OP_D : HERO_OP_I);
                qi++;
            } else if (edit[i] == 0) {
                out.push_back(qry[qi] == subj[si] ? HERO_OP_M : HERO_OP_X);
                qi++;
                si++;
            } else {
                out.push_back(reversed ? HERO_OP_I : HERO_OP_D);
                si++;
            }
        }
    }
};

// -------------------------------------------------------------------------
// AlignmentRecord (AlignmentRecord.cpp)
// -------------------------------------------------------------------------
struct Record {
    uint32_t orient = 0;
    uint32_t query = 0;              // inner id of the query read
    uint64_t key = 0;                // iQueryReadUniqueId: inner id with -c, else atoi(name)
    int64_t pos = 0;                 // iPositionOfQueryOnSubject
    std::vector<char> type;
    std::vector<int> count;
    double nmis = 0, nindel = 0, len = 0, mis_rate = 100, indel_rate = 100;

    // addCigar (AlignmentRecord.cpp:35-48)
    void addCigar(int64_t c, char t) {
        int ci = int(c);
        if (!type.empty() && type.back() == t) {
            count.back() += ci;
        } else {
            count.push_back(ci);
            type.push_back(t);
        }
    }
    // addAlignment (AlignmentRecord.cpp:50-54)
    void addAlignment(const Band &b) {
        for (size_t i = 0; i < b.ctype.size(); i++) addCigar(b.ccount[i], b.ctype[i]);
    }
    static bool isID(char t) { return t == 'I' || t == 'D'; }
    // calculateScore (AlignmentRecord.cpp:56-100)
    void calculateScore() {
        nmis = nindel = len = 0;
        size_t n = type.size();
        if (n > 0) {
            if (!isID(type[0])) {
                if (type[0] == 'M') {
                    len += count[0];
                } else {
                    nmis += count[0];
                    len += count[0];
                }
            }
            for (size_t i = 1; i + 1 < n; i++) {
                if (type[i] == 'M') {
                    len += count[i];
                } else if (isID(type[i])) {
                    nindel += count[i];
                    len += count[i];
                } else {
                    nmis += count[i];
                    len += count[i];
                }
            }
        }
        if (n > 1 && !isID(type.back())) {
            if (type.back() == 'M') {
                len += count.back();
            } else {
                nmis += count.back();
                len += count.back();
            }
        }
        if (len == 0) {
            indel_rate = 100;
            mis_rate = 100;
        } else {
            indel_rate = nindel / len;
            mis_rate = nmis / len;
        }
    }
    // isGoodAlignment() (AlignmentRecord.cpp:302-308)
    bool goodRates(const Params &p) {
        calculateScore();
        return mis_rate <= p.mis_rate && indel_rate <= p.indel_rate;
    }
    // isGoodAlignment(maxMis, maxIndel) (AlignmentRecord.cpp:310-316)
    bool goodCounts(int64_t maxMis, int64_t maxIndel) {
        calculateScore();
        return !(nmis > maxMis || nindel > maxIndel);
    }
};

struct Key {  // PairKeyPosition (SubjectRead.h:57-66)
    uint32_t q;
    int64_t posS, posQ;
};

struct Segment {
    uint32_t subject, query;
    uint8_t orient, flags;
    int32_t s0, s1, q0, q1;
    int64_t band;
    std::vector<uint8_t> ops;
};

struct Reads {
    std::vector<std::string> seq;
    std::vector<int64_t> uid;
    std::vector<uint8_t> good;
};

// QueryDataset::qualityFilter (QueryDataset.cpp:60-75)
bool qualityFilter(const char *s, uint64_t n) {
    uint64_t cnt[4] = {0, 0, 0, 0};
    for (uint64_t i = 0; i < n; i++) {
        char c = s[i];
        if (c != 'A' && c != 'C' && c != 'G' && c != 'T') return false;
        cnt[(c >> 1) & 3]++;
    }
    uint64_t threshold = uint64_t(double(n) * .8);
    if (cnt[0] >= threshold || cnt[1] >= threshold || cnt[2] >= threshold ||
        cnt[3] >= threshold)
        return false;
    return true;
}

// SubjectRead::getReverseComplement (SubjectRead.cpp:131-141)
std::string revcomp(const std::string &s) {
    size_t n = s.size();
    std::string r(n, '0');
    for (size_t i = 0; i < n; i++) r[n - i - 1] = (s[i] & 0x02) ? (s[i] ^ 0x04) : (s[i] ^ 0x15);
    return r;
}

// k-mer table: exact multimap k-mer -> (inner id, position) in insertion order
// (HashTableLongKey::insertQueryDataset/insertQueryRead, HashTableLongKey.cpp:250-342;
// getListOfReads returns exactly this list for a present key, HashTableLongKey.cpp:79-99)
struct Table {
    std::unordered_map<std::string, std::vector<std::pair<uint32_t, int64_t>>> map;
    void build(const Reads &q, int64_t k) {
        for (size_t id = 0; id < q.seq.size(); id++) {
            if (!q.good[id]) continue;
            const std::string &s = q.seq[id];
            int64_t L = int64_t(s.size());
            int64_t i = 0;
            for (i = 0; i <= L - k; i += k) map[s.substr(i, k)].push_back({uint32_t(id), i});
            if (i < L) {
                i = L - k;
                map[s.substr(i, k)].push_back({uint32_t(id), i});
            }
        }
    }
};

struct Outputs {
    std::vector<Record> kept;                 // SubjectRead::vAlignment
    std::vector<std::pair<uint32_t, std::string>> aln;  // SubjectRead::sAlignment per subject
    std::vector<Segment> segments;
    hero_oracle_stats st{};
};

struct Corrector {
    Params p;
    const Reads &Q;
    const Reads &S;
    const Table &T;
    std::vector<uint32_t> *votes;  // per query: L*4 (atomic adds)
    std::vector<uint32_t> *extra = nullptr;  // --merge: per query 20*4 overhang votes
    std::vector<uint64_t> qoff;
    const std::vector<std::string> *qrc = nullptr;  // query reverse complements (alignment output)

    Corrector(const Params &p_, const Reads &q, const Reads &s, const Table &t,
              std::vector<uint32_t> *v, std::vector<uint64_t> off)
        : p(p_), Q(q), S(s), T(t), votes(v), qoff(std::move(off)) {}

    // isFromTheSameAlignment (SubjectReadAligner.cpp:391-408)
    bool sameAlignment(const Key &add, const Key &begin, const Key &end) const {
        if (add.posS <= end.posS) return false;
        if (add.posQ <= end.posQ) return false;
        double lq = std::fabs(double(add.posQ - begin.posQ));
        double ls = std::fabs(double(add.posS - begin.posS));
        double total = (lq >= ls ? lq : ls);
        total += double(p.k);
        double diff = std::fabs(lq - ls);
        if ((diff / total) > p.indel_rate) return false;
        return true;
    }

    // calKeyLength (SubjectReadAligner.cpp:711-727)
    int64_t keyLength(const std::vector<Key> &c) const {
        if (c.size() == 1) return p.k;
        int64_t len = 0;
        for (size_t i = 0; i + 1 < c.size(); i++) {
            if (c[i].posS + p.k <= c[i + 1].posS) {
                len += p.k;
            } else {
                len += c[i + 1].posS - c[i].posS;
            }
        }
        return len + p.k;
    }

    void recordSegment(Outputs &o, const Band &b, uint32_t subject, uint32_t orient,
                       uint32_t query, int64_t s0, int64_t s1, int64_t q0, int64_t q1,
                       int64_t band_before) {
        o.st.dp_segments++;
        if (!p.keep_segments) return;
        Segment sg;
        sg.subject = subject;
        sg.orient = uint8_t(orient);
        sg.query = query;
        sg.s0 = int32_t(s0);
        sg.s1 = int32_t(s1);
        sg.q0 = int32_t(q0);
        sg.q1 = int32_t(q1);
        sg.flags = uint8_t((b.right ? 1 : 0) | (b.left ? 2 : 0));
        sg.band = band_before;
        b.steps(sg.ops);
        o.segments.push_back(std::move(sg));
    }

    void runDP(Outputs &o, Band &b, uint32_t subject, uint32_t orient, uint32_t query, int64_t s0,
               int64_t s1, int64_t q0, int64_t q1) {
        int64_t before = b.m_band;
        uint64_t c0 = b.cells;
        b.calculateAlignment();
        o.st.dp_cells += b.cells - c0;
        recordSegment(o, b, subject, orient, query, s0, s1, q0, q1, before);
    }

    // getAlignment2 (SubjectReadAligner.cpp:197-389)
    bool getAlignment2(Outputs &o, Band &b, uint32_t subject, const std::string &Sseq,
                       uint32_t orient, const std::vector<Key> &keys, Record &rec) {
        // SubjectReadAligner.cpp:199-210: without -c the reverse-complement pass
        // aligns the query's reverse complement to the forward subject
        const std::string &Qs = (p.aln && orient == 1) ? (*qrc)[keys[0].q] : Q.seq[keys[0].q];
        const int64_t k = p.k;
        int64_t posQ = keys[0].posQ, posS = keys[0].posS;
        int64_t Lq = int64_t(Qs.size()), Ls = int64_t(Sseq.size());
        int64_t ov = (posQ < posS ? posQ : posS);
        ov += (Lq - posQ < Ls - posS ? Lq - posQ : Ls - posS);
        if (ov < p.l) return false;
        o.st.records_built++;
        int64_t extra = int64_t(std::round(double(ov) * p.indel_rate));
        int64_t maxMis = int64_t(std::round(double(ov) * p.mis_rate));
        int64_t maxIndel = extra;
        rec = Record();
        rec.orient = orient;
        rec.query = keys[0].q;
        // SubjectReadAligner.cpp:230-235 (UINT64 field)
        rec.key = p.aln ? uint64_t(Q.uid[keys[0].q]) : uint64_t(keys[0].q);
        b.m_band = extra * 2;  // setBand
        const uint32_t qid = keys[0].q;
        if (posQ != 0 && posS != 0) {
            int64_t s0, s1, q0, q1;
            if (posQ < posS) {
                s0 = (posS - posQ - extra < 0 ? 0 : posS - posQ - extra);
                s1 = posS;
                q0 = 0;
                q1 = posQ;
                rec.pos = s0;
            } else if (posQ == posS) {
                s0 = 0;
                s1 = posS;
                q0 = 0;
                q1 = posQ;
                rec.pos = 0;
            } else {
                s0 = 0;
                s1 = posS;
                q0 = (posQ - posS - extra < 0 ? 0 : posQ - posS - extra);
                q1 = posQ;
                rec.pos = 0;
                if (posQ - posS - extra > 0) rec.addCigar(posQ - posS - extra, 'I');
            }
            b.setSequences(Sseq, s0, s1, Qs, q0, q1);
            b.right = true;
            runDP(o, b, subject, orient, qid, s0, s1, q0, q1);
            rec.addAlignment(b);
            rec.addCigar(k, 'M');
        } else {
            if (posS == 0 && posQ == 0) {
                rec.pos = 0;
            } else if (posS == 0) {
                rec.pos = 0;
                rec.addCigar(posQ, 'I');
            } else {
                rec.pos = posS;
            }
            rec.addCigar(k, 'M');
        }
        if (!rec.goodCounts(maxMis, maxIndel)) return false;
        for (size_t i = 1; i < keys.size(); i++) {
            int64_t cQ = keys[i].posQ, cS = keys[i].posS;
            if (cQ - posQ == cS - posS && posS + k >= cS) {
                if (posS + k > cS) {
                    rec.addCigar(cS - posS, 'M');
                } else {
                    rec.addCigar(k, 'M');
                }
            } else {
                if (posS + k == cS) {
                    if (cQ - posQ - k > 0) {
                        rec.addCigar(cQ - posQ - k, 'I');
                        rec.addCigar(k, 'M');
                    } else {
                        rec.addCigar(-cQ + posQ + k, 'D');
                        rec.addCigar(cQ - posQ, 'M');
                    }
                } else if (posS + k > cS) {
                    if (cQ - posQ < cS - posS) {
                        rec.addCigar(cS - posS - cQ + posQ, 'D');
                        rec.addCigar(cQ - posQ, 'M');
                    } else {
                        rec.addCigar(cQ - posQ + posS - cS, 'I');
                        rec.addCigar(cS - posS, 'M');
                    }
                } else {
                    if (posQ + k == cQ) {
                        rec.addCigar(cS - posS - k, 'D');
                        rec.addCigar(k, 'M');
                    } else if (posQ + k > cQ) {
                        rec.addCigar(cS - posS + posQ - cQ, 'D');
                        rec.addCigar(k + posQ - cQ, 'M');
                    } else {
                        b.setSequences(Sseq, posS + k, cS, Qs, posQ + k, cQ);
                        runDP(o, b, subject, orient, qid, posS + k, cS, posQ + k, cQ);
                        rec.addAlignment(b);
                        rec.addCigar(k, 'M');
                    }
                }
            }
            posQ = cQ;
            posS = cS;
            if (!rec.goodCounts(maxMis, maxIndel)) return false;
        }
        posQ = keys.back().posQ + k;
        posS = keys.back().posS + k;
        if (posQ < Lq) {
            if (posS == Ls) {
                rec.addCigar(Lq - posQ, 'I');
            } else if (Ls - posS < Lq - posQ) {
                int64_t qe = (Ls - posS + posQ + extra < Lq ? Ls - posS + posQ + extra : Lq);
                b.setSequences(Sseq, posS, Ls, Qs, posQ, qe);
                b.left = true;
                runDP(o, b, subject, orient, qid, posS, Ls, posQ, qe);
                rec.addAlignment(b);
                if (Ls - posS + posQ + extra < Lq) rec.addCigar(Lq - (Ls - posS + posQ + extra), 'I');
            } else if (Ls - posS == Lq - posQ) {
                b.setSequences(Sseq, posS, Ls, Qs, posQ, Lq);
                b.left = true;
                runDP(o, b, subject, orient, qid, posS, Ls, posQ, Lq);
                rec.addAlignment(b);
            } else {
                int64_t se = (posS + (Lq - posQ) + extra < Ls ? posS + (Lq - posQ) + extra : Ls);
                b.setSequences(Sseq, posS, se, Qs, posQ, Lq);
                b.left = true;
                runDP(o, b, subject, orient, qid, posS, se, posQ, Lq);
                rec.addAlignment(b);
            }
        }
        if (!rec.goodRates(p)) return false;
        return true;
    }

    // SubjectRead::addAlignment (SubjectRead.cpp:25-79), without -v
    static void addAlignment(std::vector<Record> &v, uint64_t &largest, Record &&r) {
        auto better_in_place = [](Record &cur, Record &&r) {
            double a = cur.indel_rate + cur.mis_rate, b = r.indel_rate + r.mis_rate;
            if (a < b) return;
            if (a == b) {
                if (cur.len >= r.len) return;
                cur = std::move(r);
                return;
            }
            cur = std::move(r);
        };
        if (v.empty()) {
            largest = r.key;
            v.push_back(std::move(r));
            return;
        }
        if (v.back().key == r.key) {
            better_in_place(v.back(), std::move(r));
        } else if (largest >= r.key) {
            for (size_t i = 0; i < v.size(); i++) {
                if (v[i].key > r.key) break;
                if (v[i].key == r.key) {
                    better_in_place(v[i], std::move(r));
                    return;
                }
            }
            v.push_back(std::move(r));
        } else {
            largest = r.key;
            v.push_back(std::move(r));
        }
    }

    // QueryRead::updateCoveragematrix (QueryRead.cpp:124-146)
    void vote(uint32_t q, uint64_t pos, char c) {
        // the reference writes past the matrix here (undefined behaviour); never seen
        if (pos >= qoff[q + 1] - qoff[q]) return;
        uint32_t *m = &(*votes)[qoff[q] * 4];
#pragma omp atomic
        m[pos * 4 + ((c >> 1) & 3)]++;
    }

    // SubjectRead::updateQueryCoverage (SubjectRead.cpp:208-330): the first,
    // middle and last entries are walked with the same rule, so one loop.
    void applyVotes(const std::vector<Record> &recs, const std::string &fwd,
                    const std::string &rc) {
        for (const Record &r : recs) {
            const std::string &qs = Q.seq[r.query];
            uint64_t ps = uint64_t(r.pos), pq = 0;
            const std::string &ss = (r.orient == 0) ? fwd : rc;
            for (size_t j = 0; j < r.type.size(); j++) {
                char t = r.type[j];
                int c = r.count[j];
                if (t == 'I') {
                    pq += c;
                } else if (t == 'D') {
                    ps += c;
                } else if (t == 'M') {
                    for (int x = 0; x < c; x++) vote(r.query, pq + x, qs.at(pq + x));
                    pq += c;
                    ps += c;
                } else {
                    for (int x = 0; x < c; x++) {
                        vote(r.query, pq, ss.at(ps));
                        pq++;
                        ps++;
                    }
                }
            }
            // --merge: SubjectRead::updateQueryCoverageConsiderMerging
            // (SubjectRead.cpp:332-462) votes like the loop above, and a record of
            // more than one entry also votes the subject bases past its end into
            // the query's overhang matrix (QueryRead::updateExtraCoverageMatrix,
            // QueryRead.cpp:352-369: at most 20 columns)
            if (extra && r.type.size() > 1) {
                uint32_t *m = &(*extra)[size_t(r.query) * 80];
                for (int idx = 0; idx < 20 && ps < ss.size(); idx++, ps++) {
#pragma omp atomic
                    m[idx * 4 + ((ss[ps] >> 1) & 3)]++;
                }
            }
        }
    }

    // SubjectReadAligner::start loop body (SubjectReadAligner.cpp:523-562) for one subject
    // AlignmentRecord::isSubjectCoveredByQuery (AlignmentRecord.cpp:343-370)
    static bool coversSubject(const Record &r, int64_t Ls) {
        if (r.pos != 0) return false;
        int64_t len = 0;
        if (r.type.at(0) == 'D') return false;
        if (r.type.at(0) != 'I') len += r.count.at(0);
        if (r.type.size() > 1) {
            for (size_t i = 1; i < r.type.size() - 1; i++)
                if (r.type[i] != 'I') len += r.count[i];
            if (r.type.back() == 'D') return false;
            if (r.type.back() != 'I') len += r.count.back();
        }
        return len >= Ls;
    }

    // SubjectRead::chooseQueryWithBestAlignment (SubjectRead.cpp:463-500): no
    // record covering the subject clears the list; two or more keep the one of
    // fewest substitutions (AlignmentRecord::getAccuracy, AlignmentRecord.cpp:
    // 372-381; the first of equals in list order); exactly one keeps the list.
    static void chooseBest(std::vector<Record> &v, int64_t Ls) {
        if (v.empty()) return;
        std::vector<size_t> q;
        for (size_t i = 0; i < v.size(); i++)
            if (coversSubject(v[i], Ls)) q.push_back(i);
        if (q.empty()) {
            v.clear();
            return;
        }
        if (q.size() == 1) return;
        int64_t best = -1;
        double least = double(Ls);
        for (size_t i : q) {
            double subs = 0;
            for (size_t j = 0; j < v[i].type.size(); j++) {
                const char t = v[i].type[j];
                if (t != 'I' && t != 'D' && t != 'M') subs += v[i].count[j];
            }
            if (subs < least) {
                least = subs;
                best = int64_t(i);
            }
        }
        if (best < 0) {  // the reference prints an error and then indexes -1; kept empty here
            v.clear();
            return;
        }
        Record keep = std::move(v[size_t(best)]);
        v.clear();
        v.push_back(std::move(keep));
    }

    // AlignmentRecord::getCigar (AlignmentRecord.cpp:102-149), storeOverhang off:
    // id,orientation,position,CIGAR,inserted bases of the inner I entries,
    static void cigarText(const Record &r, const std::string &qs, std::string &t) {
        t += std::to_string(r.key);
        t += ',';
        t += std::to_string(r.orient);
        t += ',';
        t += std::to_string(r.pos);
        t += ',';
        for (size_t i = 0; i < r.type.size(); i++) {
            t += std::to_string(r.count[i]);
            t += r.type[i];
        }
        t += ',';
        size_t index = 0;
        for (size_t i = 0; i < r.type.size(); i++) {
            if (r.type[i] == 'I') {
                for (int j = 0; j < r.count[i]; j++) {
                    if (i != 0 && i != r.count.size() - 1) t += qs.at(index);
                    index++;
                }
                continue;
            }
            if (r.type[i] == 'D') continue;
            index += size_t(r.count[i]);
        }
        t += ',';
    }

    void processSubject(uint32_t s, Outputs &o, Band &b) {
        if (!S.good[s]) {
            // SubjectReadAligner::writeToFile (SubjectReadAligner.cpp:898-902): no alignment string
            if (p.aln) o.aln.push_back({s, ">" + std::to_string(S.uid[s]) + "\n\n"});
            return;
        }
        const std::string &fwd = S.seq[s];
        std::string rc = revcomp(fwd);
        std::vector<Record> vAlignment;
        uint64_t largest = 0;
        std::vector<Key> hits;
        std::vector<std::vector<Key>> chains;
        for (uint32_t orient = 0; orient < 2; orient++) {
            const std::string &seq = orient == 0 ? fwd : rc;
            // searchHashTable2 (SubjectReadAligner.cpp:444-491)
            hits.clear();
            int64_t end = int64_t(seq.size()) - p.k;
            for (int64_t i = 0; i <= end; i++) {
                o.st.probes++;
                auto it = T.map.find(seq.substr(i, p.k));
                if (it == T.map.end()) continue;
                for (auto &e : it->second) {
                    if (Q.uid[e.first] == S.uid[s]) continue;
                    if (p.aln && orient == 1) {
                        // SubjectReadAligner.cpp:477-481: positions flipped onto the
                        // forward subject and the query's reverse complement
                        const int64_t lq = int64_t(Q.seq[e.first].size());
                        hits.push_back(Key{e.first, int64_t(seq.size()) - (i + p.k),
                                           lq - (e.second + p.k)});
                        continue;
                    }
                    hits.push_back(Key{e.first, i, e.second});
                }
            }
            if (hits.empty()) continue;
            o.st.hits += hits.size();
            // sortKeyPosition (SubjectRead.cpp:157-177)
            std::sort(hits.begin(), hits.end(), [](const Key &a, const Key &c) {
                if (a.q != c.q) return a.q < c.q;
                if (a.posQ != c.posQ) return a.posQ < c.posQ;
                return a.posS < c.posS;
            });
            // processOneSubjectRead2 (SubjectReadAligner.cpp:805-852)
            size_t g0 = 0;
            for (size_t i = 0; i < hits.size(); i++) {
                if (i + 1 != hits.size() && hits[i].q == hits[i + 1].q) continue;
                chains.clear();
                for (size_t h = g0; h <= i; h++) {
                    bool added = false;
                    for (auto &c : chains) {
                        if (sameAlignment(hits[h], c.front(), c.back())) {
                            c.push_back(hits[h]);
                            added = true;
                            break;
                        }
                    }
                    if (!added) chains.push_back({hits[h]});
                }
                o.st.chains += chains.size();
                // markTheBestPossibleAlignment (SubjectReadAligner.cpp:729-751)
                int64_t best = 0;
                std::vector<int64_t> kl(chains.size());
                for (size_t c = 0; c < chains.size(); c++) {
                    kl[c] = keyLength(chains[c]);
                    if (kl[c] > best) best = kl[c];
                }
                for (size_t c = 0; c < chains.size(); c++) {
                    if (kl[c] != best) continue;
                    o.st.chains_kept++;
                    Record rec;
                    // processOneSubjectRead2 (SubjectReadAligner.cpp:808-812): without
                    // -c the subject stays forward in both passes
                    if (getAlignment2(o, b, s, p.aln ? fwd : seq, orient, chains[c], rec)) {
                        o.st.records_accepted++;
                        addAlignment(vAlignment, largest, std::move(rec));
                    }
                }
                g0 = i + 1;
            }
        }
        o.st.records_kept += vAlignment.size();
        if (p.aln) {
            // SubjectRead::writeAlignment (SubjectRead.cpp:179-193): records in list order
            std::string t = ">" + std::to_string(S.uid[s]) + "\n";
            for (const Record &r : vAlignment)
                cigarText(r, r.orient == 1 ? (*qrc)[r.query] : Q.seq[r.query], t);
            t += "\n";
            o.aln.push_back({s, std::move(t)});
        } else {
            if (p.mapping) chooseBest(vAlignment, int64_t(fwd.size()));
            applyVotes(vAlignment, fwd, rc);
        }
        std::sort(vAlignment.begin(), vAlignment.end(),
                  [](const Record &a, const Record &c) { return a.query < c.query; });
        for (auto &r : vAlignment) o.kept.push_back(std::move(r));
    }
};

}  // namespace

struct hero_oracle_run_s {
    Params p;
    Reads Q;
    std::vector<std::string> qrc;
    std::string aln;  // the .aln file (alignment output)
    std::vector<uint32_t> extra;    // --merge: overhang votes, 20*4 per query
    std::vector<uint32_t> merged_len;  // --merge: per pair, length of the merged read (0: not merged)
    std::vector<uint64_t> qoff;
    std::vector<uint32_t> votes;
    std::vector<uint32_t> subj_of_kept;
    std::vector<Record> kept;
    std::vector<Segment> segments;
    hero_oracle_stats st{};
    // consensus results
    std::vector<std::string> corrected;
    std::vector<uint32_t> imin, imed, imax;
    std::vector<double> mis, gc;
};

// QueryRead::callConsensus per column (QueryRead.cpp:151-177): fractions of the
// sum in column order, the largest and the one it replaced; the letter is
// called when their difference reaches the threshold.  Returns the column's
// row (A,C,T,G) or -1.
static int consensusColumn(const uint32_t *c, double thr) {
    int largest_id = -1;
    double fLargest = 0, fLarger = 0, sum = 0, f;
    for (int j = 0; j < 4; j++) sum += c[j];
    for (int j = 0; j < 4; j++) {
        f = double(c[j]) / sum;
        if (fLargest < f) {
            fLarger = fLargest;
            fLargest = f;
            largest_id = j;
        }
    }
    if (largest_id >= 0 && fLargest - fLarger >= thr) return largest_id;
    return -1;
}

// QueryRead::getComplementBase (QueryRead.cpp:375-382): C<->G by bit 2, A<->T by 0x15
static char complementBase(char c) { return (c & 0x02) ? char(c ^ 0x04) : char(c ^ 0x15); }

// QueryRead::getExtendSequence (QueryRead.cpp:384-403): per overhang column the
// strictly largest count (first of equals), aDNA letter; stop at a column of zeros
static std::string extendSequence(const uint32_t *m) {
    std::string out;
    for (int i = 0; i < 20; i++) {
        int id = -1;
        double largest = 0;
        for (int j = 0; j < 4; j++) {
            const double f = double(m[i * 4 + j]);
            if (largest < f) {
                largest = f;
                id = j;
            }
        }
        if (largest < 1) break;
        out.push_back(ADNA[id]);
    }
    return out;
}

// QueryDataset::mergePairedReads (QueryDataset.cpp:539-558) ->
// QueryRead::mergingPairedReads (QueryRead.cpp:268-319) on reads (2i, 2i+1), after
// the consensus.  isGoodRead() is always true (QueryRead.cpp:214-216), so every
// pair is tried.  The left read grows by the right read's complement bases; the
// right read becomes empty.
// one pair: merges right into left in place (right emptied); returns whether merged
static bool mergePair(std::string &left, std::string &right, int lenL, int lenR,
                      const uint32_t *extL, const uint32_t *extR) {
    {
        const std::string seqL = extendSequence(extL);
        std::string seqR = extendSequence(extR);
        for (char &c : seqR) c = complementBase(c);  // getExtendComplementSequence
        int pl = 0;
        bool match = true;
        for (; pl < lenL; pl++) {
            const int old = pl;
            int pr = lenR - 1;
            match = true;
            for (; pr >= 0 && pl < lenL; pr--, pl++) {
                if (left.at(size_t(pl)) != complementBase(right[size_t(pr)])) {
                    match = false;
                    break;
                }
            }
            pl = old;
            if (match) break;
        }
        if (!(match && pl < lenL)) return false;
        if (int(seqL.size() + seqR.size()) + (lenL - pl) < 40) return false;
        int mism = 0;
        for (int a = lenR - lenL + pl - 1, j = 0; a >= 0 && j < int(seqL.size()); j++, a--)
            if (complementBase(right[size_t(a)]) != seqL.at(size_t(j))) mism++;
        for (int a = pl - 1, j = 0; a >= 0 && j < int(seqR.size()); j++, a--)
            if (left.at(size_t(a)) != seqR.at(size_t(j))) mism++;
        if (mism > 0) return false;
        for (int a = lenR - lenL + pl - 1; a >= 0; a--) left.push_back(complementBase(right[size_t(a)]));
        right.clear();
        return true;
    }
}

static void mergePairs(hero_oracle_run_s &run) {
    const size_t n = run.corrected.size();
    run.merged_len.assign(n / 2, 0);
    for (size_t i = 0; i + 1 < n; i += 2) {
        if (mergePair(run.corrected[i], run.corrected[i + 1], int(run.Q.seq[i].size()),
                      int(run.Q.seq[i + 1].size()), &run.extra[i * 80], &run.extra[(i + 1) * 80]))
            run.merged_len[i / 2] = uint32_t(run.corrected[i].size());
    }
}

static void load(Reads &r, uint64_t n, const uint8_t *seq, const uint64_t *off,
                 const int64_t *uid) {
    r.seq.resize(n);
    r.uid.assign(uid, uid + n);
    r.good.resize(n);
    for (uint64_t i = 0; i < n; i++) {
        r.seq[i].assign(reinterpret_cast<const char *>(seq + off[i]), off[i + 1] - off[i]);
    }
}

extern "C" hero_oracle_run *hero_oracle_correct(const hero_oracle_params *pp, int nthreads,
                                                uint64_t nq, const uint8_t *qseq,
                                                const uint64_t *qoff, const int64_t *quid,
                                                uint64_t ns, const uint8_t *sseq,
                                                const uint64_t *soff, const int64_t *suid) {
    if (!pp || pp->k <= 0) return nullptr;
    // --merge pairs reads (i, i+1): with an odd count the reference reads past the end
    if (pp->merge_pairs && (nq % 2)) return nullptr;
    hero_oracle_run *run = new hero_oracle_run_s();
    Params &p = run->p;
    p.k = pp->k;
    p.l = pp->min_overlap;
    p.affine = pp->affine != 0;
    p.keep_segments = pp->keep_segments != 0;
    p.mis_rate = pp->mis_rate;
    p.indel_rate = pp->indel_rate;
    p.thr = pp->consensus_thr;
    p.aln = pp->aln_mode != 0;
    p.merge = pp->merge_pairs != 0;
    p.mapping = pp->mapping != 0;

    load(run->Q, nq, qseq, qoff, quid);
    Reads S;
    load(S, ns, sseq, soff, suid);
    run->qoff.assign(qoff, qoff + nq + 1);
    // QueryDataset.cpp:226: good iff len > l and qualityFilter
    for (uint64_t i = 0; i < nq; i++) {
        const std::string &s = run->Q.seq[i];
        run->Q.good[i] = (int64_t(s.size()) > p.l && qualityFilter(s.data(), s.size())) ? 1 : 0;
    }
    // SubjectDataset.cpp:157-162: good iff len < l or qualityFilter
    for (uint64_t i = 0; i < ns; i++) {
        const std::string &s = S.seq[i];
        S.good[i] = (int64_t(s.size()) < p.l || qualityFilter(s.data(), s.size())) ? 1 : 0;
    }
    Table T;
    T.build(run->Q, p.k);
    run->votes.assign(size_t(qoff[nq]) * 4, 0);

    int nt = nthreads > 0 ? nthreads : 1;
    std::vector<Outputs> outs(nt);
    std::vector<std::vector<uint32_t>> subj_ids(nt);
    Corrector cor(p, run->Q, S, T, &run->votes, run->qoff);
    if (p.merge) {
        run->extra.assign(size_t(nq) * 80, 0);
        cor.extra = &run->extra;
    }
    if (p.aln) {  // QueryRead::setSequence (QueryRead.cpp:36-43) without -c
        run->qrc.resize(nq);
        for (uint64_t i = 0; i < nq; i++) run->qrc[i] = revcomp(run->Q.seq[i]);
        cor.qrc = &run->qrc;
    }
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        Band b;
        b.affine = p.affine;
#pragma omp for schedule(dynamic, 64)
        for (int64_t s = 0; s < int64_t(ns); s++) {
            size_t before = outs[t].kept.size();
            cor.processSubject(uint32_t(s), outs[t], b);
            for (size_t i = before; i < outs[t].kept.size(); i++) subj_ids[t].push_back(uint32_t(s));
        }
    }
    // merge per-thread outputs in subject order
    std::vector<std::pair<uint32_t, std::pair<int, size_t>>> order;
    for (int t = 0; t < nt; t++) {
        for (size_t i = 0; i < outs[t].kept.size(); i++) order.push_back({subj_ids[t][i], {t, i}});
        hero_oracle_stats &a = run->st;
        const hero_oracle_stats &c = outs[t].st;
        a.probes += c.probes;
        a.hits += c.hits;
        a.chains += c.chains;
        a.chains_kept += c.chains_kept;
        a.records_built += c.records_built;
        a.records_accepted += c.records_accepted;
        a.records_kept += c.records_kept;
        a.dp_segments += c.dp_segments;
        a.dp_cells += c.dp_cells;
    }
    if (p.aln) {  // SubjectReadAligner::writeToFile (SubjectReadAligner.cpp:854-906): subject order
        std::vector<std::pair<uint32_t, std::pair<int, size_t>>> ao;
        for (int t = 0; t < nt; t++)
            for (size_t i = 0; i < outs[t].aln.size(); i++) ao.push_back({outs[t].aln[i].first, {t, i}});
        std::sort(ao.begin(), ao.end());
        for (auto &a : ao) run->aln += outs[a.second.first].aln[a.second.second].second;
    }
    std::stable_sort(order.begin(), order.end(), [&](const auto &a, const auto &b) {
        if (a.first != b.first) return a.first < b.first;
        return outs[a.second.first].kept[a.second.second].query <
               outs[b.second.first].kept[b.second.second].query;
    });
    for (auto &o : order) {
        run->subj_of_kept.push_back(o.first);
        run->kept.push_back(std::move(outs[o.second.first].kept[o.second.second]));
    }
    if (p.keep_segments) {
        std::vector<std::pair<uint32_t, std::pair<int, size_t>>> so;
        for (int t = 0; t < nt; t++)
            for (size_t i = 0; i < outs[t].segments.size(); i++)
                so.push_back({outs[t].segments[i].subject, {t, i}});
        std::stable_sort(so.begin(), so.end(),
                         [](const auto &a, const auto &b) { return a.first < b.first; });
        for (auto &o : so) run->segments.push_back(std::move(outs[o.second.first].segments[o.second.second]));
    }
    // QueryDataset::callConsensus (QueryDataset.cpp:393-412) -> QueryRead::callConsensus
    // (QueryRead.cpp:148-180) and calculateCoverageStatistic (QueryRead.cpp:192-212)
    run->corrected = run->Q.seq;
    run->imin.assign(nq, 0);
    run->imed.assign(nq, 0);
    run->imax.assign(nq, 0);
    run->mis.assign(nq, 0.0);
    run->gc.assign(nq, 0.0);
    std::vector<uint32_t> cov = run->votes;
    for (uint64_t q = 0; q < nq; q++) {
        const std::string &s = run->Q.seq[q];
        // QueryRead::setGcContent (QueryRead.cpp:73-81)
        double g = 0;
        for (char c : s)
            if (c == 'C' || c == 'G') g++;
        run->gc[q] = g / double(s.size());
        if (!run->Q.good[q]) continue;
        uint32_t *m = &cov[qoff[q] * 4];
        size_t L = s.size();
        for (size_t i = 0; i < L; i++) m[i * 4 + ((s[i] >> 1) & 3)]++;
        std::string &out = run->corrected[q];
        double changed = 0;
        for (size_t i = 0; i < L; i++) {
            const int largest_id = consensusColumn(&m[i * 4], p.thr);
            if (largest_id >= 0) {
                if (out[i] != ADNA[largest_id]) changed++;
                out[i] = ADNA[largest_id];
            }
        }
        run->mis[q] = changed / double(L);
        std::vector<uint32_t> sums(L);
        for (size_t i = 0; i < L; i++) {
            uint32_t sm = 0;
            for (int j = 0; j < 4; j++) sm += m[i * 4 + j];
            sums[i] = sm;
        }
        std::sort(sums.begin(), sums.end());
        run->imin[q] = sums[0];
        run->imax[q] = sums.back();
        if (L % 2 == 0) {
            run->imed[q] = (sums[L / 2] + sums[L / 2 - 1]) / 2;
        } else {
            run->imed[q] = sums[(L - 1) / 2];
        }
    }
    if (p.merge) mergePairs(*run);
    return run;
}

extern "C" void hero_oracle_free(hero_oracle_run *r) { delete r; }

extern "C" void hero_oracle_stats_get(const hero_oracle_run *r, hero_oracle_stats *out) {
    *out = r->st;
}

extern "C" void hero_oracle_consensus(const hero_oracle_run *r, uint8_t *seq_out, uint32_t *imin,
                                      uint32_t *imed, uint32_t *imax, double *mismatch_rate,
                                      double *gc, uint8_t *good) {
    for (size_t q = 0; q < r->corrected.size(); q++) {
        if (seq_out) std::memcpy(seq_out + r->qoff[q], r->corrected[q].data(), r->corrected[q].size());
        if (imin) imin[q] = r->imin[q];
        if (imed) imed[q] = r->imed[q];
        if (imax) imax[q] = r->imax[q];
        if (mismatch_rate) mismatch_rate[q] = r->mis[q];
        if (gc) gc[q] = r->gc[q];
        if (good) good[q] = r->Q.good[q];
    }
}

extern "C" void hero_oracle_merged(const hero_oracle_run *r, uint8_t *seq_out, uint32_t *merged_len) {
    for (size_t p = 0; p < r->merged_len.size(); p++) {
        merged_len[p] = r->merged_len[p];
        const std::string &a = r->corrected[2 * p], &b = r->corrected[2 * p + 1];
        uint8_t *o = seq_out + r->qoff[2 * p];
        std::memcpy(o, a.data(), a.size());
        if (!r->merged_len[p]) std::memcpy(seq_out + r->qoff[2 * p + 1], b.data(), b.size());
    }
}

extern "C" int hero_oracle_merge_pair(const uint8_t *left, int32_t lenL, const uint8_t *right,
                                      int32_t lenR, const uint32_t *extL, const uint32_t *extR,
                                      uint8_t *out) {
    std::string l(reinterpret_cast<const char *>(left), size_t(lenL));
    std::string r(reinterpret_cast<const char *>(right), size_t(lenR));
    if (!mergePair(l, r, lenL, lenR, extL, extR)) return 0;
    std::memcpy(out, l.data(), l.size());
    return int(l.size());
}

extern "C" void hero_oracle_record_score(uint32_t nev, const uint32_t *piece, const uint8_t *type,
                                         const int32_t *count, const uint8_t *letter,
                                         int64_t *out) {
    // AlignmentRecord::addCigar per event, then calculateScore
    Record r;
    for (uint32_t i = 0; i < nev; i++) {
        const char t = type[i] == HERO_OP_M   ? 'M'
                       : type[i] == HERO_OP_I ? 'I'
                       : type[i] == HERO_OP_D ? 'D'
                                              : char(letter[i]);
        (void)piece;
        r.addCigar(count[i], t);
    }
    r.calculateScore();
    out[0] = int64_t(r.nmis);
    out[1] = int64_t(r.nindel);
    out[2] = int64_t(r.len);
}

extern "C" int32_t hero_oracle_chain(int32_t k, double indel_rate, uint32_t n, const int64_t *posQ,
                                     const int64_t *posS, uint32_t *chain_of, uint8_t *kept) {
    // processOneSubjectRead2's chaining of one query group (hits sorted by posQ,
    // posS) and markTheBestPossibleAlignment
    Params p{};
    p.k = k;
    p.indel_rate = indel_rate;
    Reads none;
    Table t;
    Corrector cor(p, none, none, t, nullptr, {});
    std::vector<std::vector<Key>> chains;
    std::vector<std::vector<uint32_t>> ids;
    for (uint32_t h = 0; h < n; h++) {
        const Key x{0, posS[h], posQ[h]};
        size_t c = 0;
        for (; c < chains.size(); c++)
            if (cor.sameAlignment(x, chains[c].front(), chains[c].back())) break;
        if (c == chains.size()) {
            chains.push_back({});
            ids.push_back({});
        }
        chains[c].push_back(x);
        ids[c].push_back(h);
        chain_of[h] = uint32_t(c);
    }
    int64_t best = 0;
    std::vector<int64_t> kl(chains.size());
    for (size_t c = 0; c < chains.size(); c++) {
        kl[c] = cor.keyLength(chains[c]);
        if (kl[c] > best) best = kl[c];
    }
    for (size_t c = 0; c < chains.size(); c++) kept[c] = kl[c] == best ? 1 : 0;
    return int32_t(chains.size());
}

extern "C" int32_t hero_oracle_chain_layout(int32_t k, int32_t l, int32_t affine, double mis_rate,
                                            double indel_rate, const uint8_t *qseq, int32_t Lq,
                                            const uint8_t *sseq, int32_t Ls, uint32_t nkeys,
                                            const int64_t *posQ, const int64_t *posS, int64_t *seg,
                                            int32_t cap, int64_t *pos_out, int32_t *status) {
    // getAlignment2 on one chain: the DP calls it makes (s0, s1, q0, q1, flags,
    // band before the call), the record's position and its fate
    Params p{};
    p.k = k;
    p.l = l;
    p.affine = affine != 0;
    p.keep_segments = true;
    p.mis_rate = mis_rate;
    p.indel_rate = indel_rate;
    Reads Q;
    Q.seq.push_back(std::string(reinterpret_cast<const char *>(qseq), size_t(Lq)));
    Q.uid.push_back(1);
    Q.good.push_back(1);
    Table t;
    Corrector cor(p, Q, Q, t, nullptr, {});
    std::vector<Key> keys(nkeys);
    for (uint32_t i = 0; i < nkeys; i++) keys[i] = Key{0, posS[i], posQ[i]};
    Outputs o;
    Band b;
    b.affine = p.affine;
    Record rec;
    const std::string S(reinterpret_cast<const char *>(sseq), size_t(Ls));
    const uint64_t built0 = o.st.records_built;
    const bool ok = cor.getAlignment2(o, b, 0, S, 0, keys, rec);
    *status = o.st.records_built == built0 ? 0 : (ok ? 2 : 1);
    *pos_out = rec.pos;
    const int32_t n = int32_t(o.segments.size());
    for (int32_t i = 0; i < n && i < cap; i++) {
        const Segment &g = o.segments[size_t(i)];
        int64_t *x = seg + 6 * i;
        x[0] = g.s0;
        x[1] = g.s1;
        x[2] = g.q0;
        x[3] = g.q1;
        x[4] = g.flags;
        x[5] = g.band;
    }
    return n;
}

extern "C" int32_t hero_oracle_record_text(uint64_t key, uint32_t orient, int64_t pos, uint32_t nev,
                                           const uint32_t *piece, const uint8_t *type,
                                           const int32_t *count, const uint8_t *query, int32_t Lq,
                                           int32_t qrc, uint8_t *out, int32_t cap) {
    // the record as getAlignment2 builds it (addCigar per run and per step, a
    // mismatch named by the query's base there), then AlignmentRecord::getCigar
    std::string qs(reinterpret_cast<const char *>(query), size_t(Lq));
    if (qrc) qs = revcomp(qs);
    Record r;
    r.key = key;
    r.orient = orient;
    r.pos = pos;
    size_t pq = 0;
    for (uint32_t i = 0; i < nev; i++) {
        (void)piece;
        const uint8_t t = type[i];
        if (t == HERO_OP_X) {
            r.addCigar(count[i], qs.at(pq));
        } else {
            r.addCigar(count[i], t == HERO_OP_M ? 'M' : t == HERO_OP_I ? 'I' : 'D');
        }
        if (t != HERO_OP_D) pq += size_t(count[i]);
    }
    std::string text;
    Corrector::cigarText(r, qs, text);
    if (int32_t(text.size()) > cap) return -1;
    std::memcpy(out, text.data(), text.size());
    return int32_t(text.size());
}

// QueryDataset::getCoverageAndWriteResults (QueryDataset.cpp:560-599): per
// query base the sum of its four vote counts (no self vote), a histogram of
// those sums, "COV\tFRE" and one "coverage\tbases" line per non-empty bin
extern "C" uint64_t hero_oracle_mapping_histogram(const hero_oracle_run *r, uint8_t *out, uint64_t cap) {
    uint32_t maxc = 0;
    const size_t nb = r->votes.size() / 4;
    for (size_t i = 0; i < nb; i++) {
        const uint32_t c = r->votes[4 * i] + r->votes[4 * i + 1] + r->votes[4 * i + 2] + r->votes[4 * i + 3];
        if (c > maxc) maxc = c;
    }
    std::vector<uint32_t> hist(size_t(maxc) + 1, 0);
    for (size_t i = 0; i < nb; i++)
        hist[r->votes[4 * i] + r->votes[4 * i + 1] + r->votes[4 * i + 2] + r->votes[4 * i + 3]]++;
    std::string t = "COV\tFRE\n";
    for (size_t i = 0; i < hist.size(); i++)
        if (hist[i] > 0) t += std::to_string(i) + "\t" + std::to_string(hist[i]) + "\n";
    if (out && t.size() <= cap) std::memcpy(out, t.data(), t.size());
    return t.size();
}

extern "C" int32_t hero_oracle_key_positions(int64_t L, int64_t k, int64_t *out) {
    // HashTableLongKey::insertQueryDataset (HashTableLongKey.cpp:279-289): keys at
    // 0, k, 2k, ... while i <= L - k, then one at L - k if i < L
    int32_t n = 0;
    int64_t i = 0;
    for (i = 0; i <= L - k; i += k) out[n++] = i;
    if (i < L) out[n++] = L - k;
    return n;
}

extern "C" void hero_oracle_columns(uint64_t n, const uint32_t *counts, double thr, int32_t *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = consensusColumn(counts + 4 * i, thr);
}

extern "C" int32_t hero_oracle_record_list(uint32_t n, const uint64_t *key, const double *rate_sum,
                                           const double *len, uint32_t *out) {
    // SubjectRead::addAlignment's list over records 0..n-1 in arrival order
    std::vector<Record> v;
    uint64_t largest = 0;
    for (uint32_t i = 0; i < n; i++) {
        Record r;
        r.query = i;
        r.key = key[i];
        r.mis_rate = rate_sum[i];
        r.indel_rate = 0;
        r.len = len[i];
        Corrector::addAlignment(v, largest, std::move(r));
    }
    for (size_t i = 0; i < v.size(); i++) out[i] = v[i].query;
    return int32_t(v.size());
}

extern "C" void hero_oracle_overhang(const hero_oracle_run *r, uint32_t *out) {
    std::memcpy(out, r->extra.data(), r->extra.size() * sizeof(uint32_t));
}

extern "C" uint64_t hero_oracle_aln_size(const hero_oracle_run *r) { return r->aln.size(); }

extern "C" void hero_oracle_aln(const hero_oracle_run *r, uint8_t *out) {
    std::memcpy(out, r->aln.data(), r->aln.size());
}

extern "C" void hero_oracle_votes(const hero_oracle_run *r, uint32_t *cov) {
    std::memcpy(cov, r->votes.data(), r->votes.size() * sizeof(uint32_t));
}

static void expand(const Record &r, std::vector<uint8_t> &out) {
    for (size_t j = 0; j < r.type.size(); j++) {
        uint8_t op = r.type[j] == 'M' ? HERO_OP_M
                     : r.type[j] == 'I' ? HERO_OP_I
                     : r.type[j] == 'D' ? HERO_OP_D
                                        : HERO_OP_X;
        for (int c = 0; c < r.count[j]; c++) out.push_back(op);
    }
}

extern "C" uint64_t hero_oracle_num_records(const hero_oracle_run *r) { return r->kept.size(); }

extern "C" uint64_t hero_oracle_record_ops_total(const hero_oracle_run *r) {
    uint64_t t = 0;
    for (auto &k : r->kept)
        for (int c : k.count) t += uint64_t(c);
    return t;
}

extern "C" void hero_oracle_records(const hero_oracle_run *r, uint32_t *subject, uint32_t *query,
                                    uint8_t *orient, int64_t *pos, double *rate_sum,
                                    double *align_len, uint64_t *ops_off, uint8_t *ops) {
    uint64_t o = 0;
    std::vector<uint8_t> tmp;
    for (size_t i = 0; i < r->kept.size(); i++) {
        const Record &k = r->kept[i];
        subject[i] = r->subj_of_kept[i];
        query[i] = k.query;
        orient[i] = uint8_t(k.orient);
        pos[i] = k.pos;
        rate_sum[i] = k.indel_rate + k.mis_rate;
        align_len[i] = k.len;
        ops_off[i] = o;
        tmp.clear();
        expand(k, tmp);
        if (ops) std::memcpy(ops + o, tmp.data(), tmp.size());
        o += tmp.size();
    }
    ops_off[r->kept.size()] = o;
}

extern "C" uint64_t hero_oracle_num_segments(const hero_oracle_run *r) { return r->segments.size(); }

extern "C" uint64_t hero_oracle_segment_ops_total(const hero_oracle_run *r) {
    uint64_t t = 0;
    for (auto &s : r->segments) t += s.ops.size();
    return t;
}

extern "C" void hero_oracle_segments(const hero_oracle_run *r, uint32_t *subject, uint8_t *orient,
                                     uint32_t *query, int32_t *s0, int32_t *s1, int32_t *q0,
                                     int32_t *q1, uint8_t *flags, int64_t *band,
                                     uint64_t *ops_off, uint8_t *ops) {
    uint64_t o = 0;
    for (size_t i = 0; i < r->segments.size(); i++) {
        const Segment &s = r->segments[i];
        subject[i] = s.subject;
        orient[i] = s.orient;
        query[i] = s.query;
        s0[i] = s.s0;
        s1[i] = s.s1;
        q0[i] = s.q0;
        q1[i] = s.q1;
        flags[i] = s.flags;
        band[i] = s.band;
        ops_off[i] = o;
        if (ops) std::memcpy(ops + o, s.ops.data(), s.ops.size());
        o += s.ops.size();
    }
    ops_off[r->segments.size()] = o;
}

extern "C" int hero_oracle_align(int affine, const uint8_t *subj, int32_t ls, const uint8_t *query,
                                 int32_t lq, int64_t band, int align_right, int align_left,
                                 uint8_t *ops, int32_t ops_cap, int64_t *band_used) {
    Band b;
    b.affine = affine != 0;
    std::string S(reinterpret_cast<const char *>(subj), size_t(ls));
    std::string Q(reinterpret_cast<const char *>(query), size_t(lq));
    b.setSequences(S, 0, ls, Q, 0, lq);
    b.m_band = band;
    b.right = align_right != 0;
    b.left = align_left != 0;
    b.calculateAlignment();
    std::vector<uint8_t> st;
    b.steps(st);
    if (band_used) *band_used = b.m_band;
    if (int32_t(st.size()) > ops_cap) return -1;
    std::memcpy(ops, st.data(), st.size());
    return int(st.size());
}

extern "C" int hero_oracle_quality_filter(const uint8_t *seq, uint64_t len) {
    return qualityFilter(reinterpret_cast<const char *>(seq), len) ? 1 : 0;
}
