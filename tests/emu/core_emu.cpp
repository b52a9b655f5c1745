// core_emu.cpp -- TEST HARNESS ONLY.
//
// Compiles the device-side item logic (hero_b200/csrc/hero_core.cuh) with the
// host compiler and drives it through a plain sequential loop, so the per-item
// code (DP strips + traceback, chaining, record scoring, dedupe, votes,
// consensus) can be checked against the oracle on a machine without a GPU.
// It is never part of the product: the library has no CPU path.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../hero_b200/csrc/hero_core.cuh"

using namespace hero;

namespace {

template <int W>
struct HostScratch {
    int32_t R = 0, C = 0;
    std::vector<uint32_t> tbv;
    std::vector<int32_t> bv;
    void reset(int32_t r, int32_t c) {
        R = r;
        C = c;
        const int32_t nst = (c + W - 1) / W;
        tbv.assign(size_t(nst) * size_t(r + 1), 0xdeadbeefu);
        bv.assign(size_t(3) * size_t(r + 1), 0x7f7f7f7f);
    }
    void tb_set(int32_t s, int32_t i, uint32_t bits) { tbv[size_t(s) * (R + 1) + i] = bits; }
    uint32_t tb_get(int32_t s, int32_t i) const { return tbv[size_t(s) * (R + 1) + i]; }
    int32_t &b(int32_t st, int32_t i) { return bv[size_t(st) * (R + 1) + i]; }
};

template <int W>
int run_dp(const SegView &v, bool affine, std::vector<uint8_t> &ops, DpSum &sum) {
    HostScratch<W> sc;
    sc.reset(v.R, v.C);
    if (affine) {
        dp_fill<W, true>(v, sc);
    } else {
        dp_fill<W, false>(v, sc);
    }
    std::vector<uint8_t> rev;
    auto emit = [&](uint8_t op) { rev.push_back(op); };
    int n = dp_traceback<W>(v, sc, emit, sum);
    ops.assign(rev.rbegin(), rev.rend());
    return n;
}

struct Reads {
    std::vector<uint8_t> code;
    std::vector<uint64_t> off;
    std::vector<uint32_t> len;
    std::vector<int64_t> uid;
    std::vector<uint8_t> gq, gs;
    std::vector<double> gc;
};

void load(Reads &r, uint64_t n, const uint8_t *seq, const uint64_t *off, const int64_t *uid,
          int32_t l) {
    r.off.assign(off, off + n + 1);
    r.uid.assign(uid, uid + n);
    r.code.resize(off[n]);
    for (uint64_t i = 0; i < off[n]; i++) r.code[i] = base_code(seq[i]);
    r.len.resize(n);
    r.gq.resize(n);
    r.gs.resize(n);
    r.gc.resize(n);
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t L = off[i + 1] - off[i];
        uint64_t cnt[4] = {0, 0, 0, 0}, ngc = 0;
        bool valid = true;
        for (uint64_t j = 0; j < L; j++) {
            uint8_t c = r.code[off[i] + j];
            if (c >= 4) {
                valid = false;
            } else {
                cnt[c]++;
                ngc += c & 1;
            }
        }
        bool qf = valid;
        const uint64_t thr = uint64_t(double(L) * 0.8);
        if (qf && (cnt[0] >= thr || cnt[1] >= thr || cnt[2] >= thr || cnt[3] >= thr)) qf = false;
        const uint64_t lu = uint16_t(l);
        r.len[i] = uint32_t(L);
        r.gq[i] = (L > lu && qf) ? 1 : 0;
        r.gs[i] = (L < lu || qf) ? 1 : 0;
        r.gc[i] = double(ngc) / double(L);
    }
}

struct KeyHash {
    size_t operator()(const std::pair<uint64_t, uint64_t> &k) const {
        return size_t(kmer_hash(Kmer{k.first, k.second}));
    }
};

struct SegRec {
    int64_t s0, s1, q0, q1, band;
    uint32_t flags;
    std::vector<uint8_t> ops;
    DpSum sum;
};

struct Collect {
    std::vector<SegRec> *out;
    uint32_t n = 0;
    void begin(int64_t, int64_t, int64_t) {}
    void position(int64_t) {}
    void run(uint8_t, int64_t) {}
    void dp(int64_t s0, int64_t s1, int64_t q0, int64_t q1, uint32_t f, int64_t band) {
        SegRec r;
        r.s0 = s0;
        r.s1 = s1;
        r.q0 = q0;
        r.q1 = q1;
        r.flags = f;
        r.band = band > 65535 ? 65535 : band;
        out->push_back(r);
        n++;
    }
    bool check(int64_t, int64_t) { return true; }
    void finish() {}
};

struct Asm {
    const SegRec *segs;
    RecState st;
    uint32_t used = 0;
    bool built = false;
    void begin(int64_t, int64_t, int64_t) { built = true; }
    void position(int64_t) {}
    void run(uint8_t t, int64_t c) { st.add(t, c); }
    void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) { st.add_piece(segs[used++].sum); }
    bool check(int64_t m, int64_t i) { return st.good_counts(m, i); }
    void finish() {}
};

struct Vote {
    const uint8_t *sc;
    int64_t Ls;
    int orient;
    const uint8_t *qc;
    int64_t Lq;
    uint32_t *cov;
    const SegRec *segs;
    uint32_t used = 0;
    int64_t ps = 0, pq = 0;
    uint64_t anomalies = 0;
    uint8_t sub(int64_t i) const { return orient ? uint8_t(sc[Ls - 1 - i] ^ 2) : sc[i]; }
    void vote(int64_t pos, uint8_t code) {
        if (pos < 0 || pos >= Lq || code >= 4) {
            anomalies++;
            return;
        }
        cov[pos * 4 + code]++;
    }
    void one(uint8_t t) {
        if (t == OP_I) {
            pq++;
        } else if (t == OP_D) {
            ps++;
        } else if (t == OP_M) {
            vote(pq, pq < Lq ? qc[pq] : kBad);
            pq++;
            ps++;
        } else {
            vote(pq, (ps >= 0 && ps < Ls) ? sub(ps) : kBad);
            pq++;
            ps++;
        }
    }
    void begin(int64_t, int64_t, int64_t) {}
    void position(int64_t p) {
        ps = p;
        pq = 0;
    }
    void run(uint8_t t, int64_t c) {
        if (t == OP_I) {
            pq += c;
        } else if (t == OP_D) {
            ps += c;
        } else {
            for (int64_t x = 0; x < c; x++) one(t);
        }
    }
    void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {
        for (uint8_t op : segs[used].ops) one(op);
        used++;
    }
    bool check(int64_t, int64_t) { return true; }
    void finish() {}
};

}  // namespace

// test-harness instrumentation: rounds the chunked traceback of the last segment took
int g_chunk_rounds = 0;

extern "C" {
int emu_chunk_rounds() { return g_chunk_rounds; }

uint64_t emu_band_cells(int32_t R, int32_t C, int64_t m) { return band_cells(R, C, m); }

// rolling forward / reverse-complement k-mers (the probe kernel) against
// building each window from scratch; returns the first bad window or -1
int64_t emu_kmer_roll_check(const uint8_t *codes, int64_t n, int32_t k) {
    Kmer fr{0, 0}, rr{0, 0};
    for (int64_t i = 0; i + 1 < k && i < n; i++) {
        kmer_push(fr, codes[i] & 3u, k);
        kmer_push_front(rr, (codes[i] & 3u) ^ 2u, k);
    }
    for (int64_t f = 0; f + k <= n; f++) {
        kmer_push(fr, codes[f + k - 1] & 3u, k);
        kmer_push_front(rr, (codes[f + k - 1] & 3u) ^ 2u, k);
        Kmer fm{0, 0}, rm{0, 0};
        for (int32_t i = 0; i < k; i++) kmer_push(fm, codes[f + i] & 3u, k);
        for (int32_t i = k - 1; i >= 0; i--) kmer_push(rm, (codes[f + i] & 3u) ^ 2u, k);
        if (fm.lo != fr.lo || fm.hi != fr.hi || rm.lo != rr.lo || rm.hi != rr.hi) return f;
    }
    return -1;
}


// one DP segment through the core strip DP; same argument meaning as
// hero_oracle_align (segments given directly, orientation forward)
int emu_align(int affine, const uint8_t *subj, int32_t ls, const uint8_t *query, int32_t lq,
              int64_t band, int align_right, int align_left, int strip16, uint8_t *ops,
              int32_t cap) {
    std::vector<uint8_t> sc(ls), qc(lq);
    for (int i = 0; i < ls; i++) sc[i] = base_code(subj[i]);
    for (int i = 0; i < lq; i++) qc[i] = base_code(query[i]);
    uint32_t flags = (align_right ? DPF_RIGHT : 0) | (align_left ? DPF_LEFT : 0);
    SegView v = make_view(sc.data(), ls, 0, qc.data(), 0, ls, 0, lq, flags, band);
    std::vector<uint8_t> out;
    DpSum sum;
    int n = strip16 ? run_dp<16>(v, affine != 0, out, sum) : run_dp<8>(v, affine != 0, out, sum);
    if (n > cap) return -1;
    std::memcpy(ops, out.data(), out.size());
    return n;
}

// one DP segment through the warp-wavefront schedule of k_dp_wave: lane s owns
// strip s and computes row t - s + 1 at step t; the left boundary of a row is
// what lane s-1 published one step earlier.  Lanes are simulated in order.
extern "C++" {
// whole-band wavefront lanes (the kernel's wave_whole), stepped sequentially:
// at step t every lane reads what its left neighbour published at step t-1
template <bool AFFINE, bool LEFT>
void emu_whole(const SegView &v, int G, int32_t wl, std::vector<uint16_t> &tb) {
    constexpr int W = 8;
    struct Lane {
        int32_t f[W], x[W], m[W], c0[3], tab[kTabWords];
        int32_t pm, pf, py, pmv;
        const uint8_t *rp;
        uint32_t ch;
    };
    std::vector<Lane> L(G);
    for (int s = 0; s < G; s++) {
        Lane &x = L[s];
        dp_whole_table<W>(v, s * W, x.tab);
        dp_whole_init<AFFINE, W>(v, s * W, x.f, x.x, x.m, x.pm);
        dp_whole_col0<AFFINE>(v, x.c0);
        x.rp = v.row_base;
        x.ch = (x.rp[0] ^ v.row_xor) & 3u;
        x.pf = x.py = x.pmv = kNEG;
    }
    std::vector<int32_t> inf(G), iny(G), inm(G);
    for (int t = 0; t < v.R + G - 1; t++) {
        for (int s = 0; s < G; s++) {  // __shfl_up_sync
            inf[s] = s > 0 ? L[s - 1].pf : 0;
            iny[s] = s > 0 ? L[s - 1].py : 0;
            inm[s] = s > 0 ? L[s - 1].pmv : 0;
        }
        for (int s = 0; s < G; s++) {
            const int32_t i = t - s + 1;
            if (i < 1 || i > v.R) continue;
            Lane &x = L[s];
            const uint32_t a = x.ch;
            if (i < v.R) {
                x.rp += v.row_dir;
                x.ch = (x.rp[0] ^ v.row_xor) & 3u;
            }
            const int32_t c0f = i * x.c0[0] + x.c0[1];
            int32_t lf = s == 0 ? c0f : inf[s];
            int32_t ly = s == 0 ? i * x.c0[0] + x.c0[2] : iny[s];
            int32_t sc[W];
            for (int w = 0; w < W; w++) sc[w] = x.tab[a * W + w];
            const uint32_t diag = uint32_t(x.tab[4 * W + a]);
            if (LEFT) dp_whole_left<AFFINE, W>(wl, s == G - 1, x.f, x.x);
            const uint32_t bits = dp_whole_row<AFFINE, W>(sc, diag, x.f, x.x, x.m, lf, ly, x.pm);
            tb[size_t(i - 1) * 32 + s] = uint16_t(bits);
            x.pf = lf;
            x.py = ly;
            x.pmv = AFFINE ? x.m[W - 1] : x.f[W - 1];
            x.pm = s == 0 ? c0f : inm[s];
        }
    }
}

template <bool AFFINE>
void emu_whole_any(int wl, const SegView &v, int G, std::vector<uint16_t> &tb) {
    if (wl >= 0) {
        emu_whole<AFFINE, true>(v, G, wl, tb);
    } else {
        emu_whole<AFFINE, false>(v, G, -1, tb);
    }
}

// two segments of one shape as a tagged 16-bit pair (the kernel's wave_pair), lanes in turn
template <bool AFFINE, bool LEFT>
void emu_pair(const SegView &va, const SegView &vb, int G, int32_t wl, std::vector<uint32_t> &tb) {
    constexpr int W = 8;
    constexpr uint32_t c0tag = AFFINE ? 0x00010001u * uint32_t(PairTags<AFFINE>::diag) : 0u;
    struct Lane {
        uint32_t f[W], x[W], m[W], tab[kTabWords2];
        uint32_t pm, pf, py, pmv, c0f, c0y, mul;
        const uint8_t *rpa, *rpb;
        uint32_t cha, chb;
    };
    std::vector<Lane> L(G);
    for (int s = 0; s < G; s++) {
        Lane &x = L[s];
        dp_pair_table<AFFINE, W>(va, vb, s * W, x.tab);
        dp_pair_init<AFFINE, W>(va, vb, s * W, x.f, x.x, x.m, x.pm);
        dp_pair_col0<AFFINE>(va, vb, x.c0f, x.c0y, x.mul);
        x.rpa = va.row_base;
        x.rpb = vb.row_base;
        x.cha = (x.rpa[0] ^ va.row_xor) & 3u;
        x.chb = (x.rpb[0] ^ vb.row_xor) & 3u;
        x.pf = x.py = x.pmv = pack2s(kPairPad);
    }
    std::vector<uint32_t> inf(G), iny(G), inm(G);
    for (int t = 0; t < va.R + G - 1; t++) {
        for (int s = 0; s < G; s++) {
            inf[s] = s > 0 ? L[s - 1].pf : 0;
            iny[s] = s > 0 ? L[s - 1].py : 0;
            inm[s] = s > 0 ? L[s - 1].pmv : 0;
        }
        for (int s = 0; s < G; s++) {
            const int32_t i = t - s + 1;
            if (i < 1 || i > va.R) continue;
            Lane &x = L[s];
            const uint32_t ba = x.cha, bb = x.chb;
            if (i < va.R) {
                x.rpa += va.row_dir;
                x.rpb += vb.row_dir;
                x.cha = (x.rpa[0] ^ va.row_xor) & 3u;
                x.chb = (x.rpb[0] ^ vb.row_xor) & 3u;
            }
            uint32_t lf = s == 0 ? x.c0f : inf[s];
            uint32_t ly = s == 0 ? x.c0y : iny[s];
            const uint16_t *sc16 = reinterpret_cast<const uint16_t *>(x.tab);
            uint32_t sc[W];
            for (int w = 0; w < W; w++) sc[w] = uint32_t(sc16[ba * W + w]) | (uint32_t(sc16[(4 + bb) * W + w]) << 16);
            if (LEFT) dp_pair_left<AFFINE, W>(wl, s == G - 1, x.f, x.x);
            const uint32_t eq = x.tab[32 + ba] | x.tab[36 + bb];
            const uint32_t bits = dp_pair_row<AFFINE, W>(sc, eq, x.f, x.x, x.m, lf, ly, x.pm);
            tb[size_t(i - 1) * 32 + s] = bits;
            x.pf = lf;
            x.py = ly;
            x.pmv = AFFINE ? x.m[W - 1] : lf;
            x.pm = s == 0 ? x.c0f - c0tag : (AFFINE ? inm[s] : inf[s]);
            x.c0f = add2(x.c0f, x.mul);
            x.c0y = add2(x.c0y, x.mul);
        }
    }
}
}  // extern "C++"


// A pair of segments with equal lengths (same rows, strips and align-left
// column) through the 16-bit pair rows; each half's ops are walked and returned
// (ops_a / ops_b, capacity cap each).  Returns 0, or -1 if the pair does not
// qualify or a path does not fit.
int emu_align_pair(int affine, const uint8_t *sa, const uint8_t *qa, const uint8_t *sb,
                   const uint8_t *qb, int32_t ls, int32_t lq, int32_t lqb, int64_t band_a,
                   int64_t band_b, int flags_a, int flags_b, uint8_t *ops_a, int32_t *na,
                   uint8_t *ops_b, int32_t *nb, int32_t cap) {
    constexpr int W = 8;
    std::vector<uint8_t> sca(ls), qca(lq), scb(ls), qcb(lqb);
    for (int i = 0; i < ls; i++) {
        sca[i] = base_code(sa[i]);
        scb[i] = base_code(sb[i]);
    }
    for (int i = 0; i < lq; i++) qca[i] = base_code(qa[i]);
    for (int i = 0; i < lqb; i++) qcb[i] = base_code(qb[i]);
    const SegView va = make_view(sca.data(), ls, 0, qca.data(), 0, ls, 0, lq, uint32_t(flags_a), band_a);
    const SegView vb = make_view(scb.data(), ls, 0, qcb.data(), 0, ls, 0, lqb, uint32_t(flags_b), band_b);
    // the kernel's pairing rule: same rows, strips and align-left column
    if (!dp_whole_band(va) || !dp_whole_band(vb) || dp_left_col<W>(va) != dp_left_col<W>(vb) ||
        va.R != vb.R || (va.C + W - 1) / W != (vb.C + W - 1) / W || va.R + va.C > kPairMaxSide ||
        vb.R + vb.C > kPairMaxSide)
        return -1;
    const int G = (va.C + W - 1) / W;
    std::vector<uint32_t> tb(size_t(va.R) * 32, 0);
    const int32_t wl = dp_left_col<W>(va);
    if (affine) {
        if (wl >= 0) emu_pair<true, true>(va, vb, G, wl, tb);
        else emu_pair<true, false>(va, vb, G, -1, tb);
    } else {
        if (wl >= 0) emu_pair<false, true>(va, vb, G, wl, tb);
        else emu_pair<false, false>(va, vb, G, -1, tb);
    }
    for (int h = 0; h < 2; h++) {
        struct Codes {
            const uint32_t *tb;
            int shift;
            uint32_t tb_get(int32_t st, int32_t i) const { return (tb[size_t(i - 1) * 32 + st] >> shift) & 0xffffu; }
        } sc{tb.data(), 16 * h};
        std::vector<uint8_t> rev;
        auto emit = [&](uint8_t op) { rev.push_back(op); };
        const int n = dp_walk<W>(h ? vb : va, sc, emit);
        if (n > cap) return -1;
        uint8_t *out = h ? ops_b : ops_a;
        for (int k = 0; k < n; k++) out[k] = rev[size_t(n - 1 - k)];
        (h ? *nb : *na) = n;
    }
    return 0;
}

int emu_align_wave(int affine, const uint8_t *subj, int32_t ls, const uint8_t *query, int32_t lq,
                   int64_t band, int align_right, int align_left, uint8_t *ops, int32_t cap) {
    constexpr int W = 8;
    std::vector<uint8_t> scd(ls), qcd(lq);
    for (int i = 0; i < ls; i++) scd[i] = base_code(subj[i]);
    for (int i = 0; i < lq; i++) qcd[i] = base_code(query[i]);
    uint32_t flags = (align_right ? DPF_RIGHT : 0) | (align_left ? DPF_LEFT : 0);
    SegView v = make_view(scd.data(), ls, 0, qcd.data(), 0, ls, 0, lq, flags, band);
    const int G = (v.C + W - 1) / W;
    struct Lane {
        uint8_t bc[W];
        int32_t uf[W], ux[W], uy[W];
        bool full;
        int32_t wlast;
        Cell3 prev, pub;
    };
    std::vector<Lane> L(G);
    std::vector<uint16_t> tb(size_t(v.R) * 32, 0);
    for (int s = 0; s < G; s++) {
        if (affine) {
            dp_strip_init<W, true>(v, s * W, L[s].bc, L[s].uf, L[s].ux, L[s].uy);
            L[s].prev = dp_row0<true>(v, s * W);
        } else {
            dp_strip_init<W, false>(v, s * W, L[s].bc, L[s].uf, L[s].ux, L[s].uy);
            L[s].prev = dp_row0<false>(v, s * W);
        }
        L[s].full = dp_strip_full(v, s * W, W);
        L[s].wlast = dp_strip_wlast(v, s * W, W);
        L[s].pub = Cell3{kNEG, kNEG, kNEG};
    }
    if (dp_whole_band(v)) {  // the kernel's whole-band path
        if (affine) {
            emu_whole_any<true>(dp_left_col<W>(v), v, G, tb);
        } else {
            emu_whole_any<false>(dp_left_col<W>(v), v, G, tb);
        }
    }
    for (int t = 0; t < (dp_whole_band(v) ? 0 : v.R + G - 1); t++) {
        std::vector<Cell3> in(G);
        for (int s = 0; s < G; s++) in[s] = s > 0 ? L[s - 1].pub : Cell3{0, 0, 0};  // shfl_up
        for (int s = 0; s < G; s++) {
            const int i = t - s + 1;
            if (i < 1 || i > v.R) continue;
            Lane &x = L[s];
            Cell3 left, dg;
            if (affine) {
                left = s == 0 ? dp_col0<true>(v, i) : in[s];
                dg = s == 0 ? dp_col0<true>(v, i - 1) : x.prev;
            } else {
                left = s == 0 ? dp_col0<false>(v, i) : in[s];
                dg = s == 0 ? dp_col0<false>(v, i - 1) : x.prev;
            }
            const Cell3 lb = left;
            const uint8_t ch = v.row(i);
            uint32_t bits;
            if (affine) {
                bits = dp_strip_row_any<W, true>(x.full, x.wlast, v, i, s * W, ch, x.bc, x.uf, x.ux, x.uy, left, dg);
            } else {
                bits = dp_strip_row_any<W, false>(x.full, x.wlast, v, i, s * W, ch, x.bc, x.uf, x.ux, x.uy, left, dg);
            }
            tb[size_t(i - 1) * 32 + s] = uint16_t(bits);
            x.pub = left;
            x.prev = lb;
        }
    }
    struct Codes {
        const uint16_t *tb;
        uint32_t tb_get(int32_t st, int32_t i) const { return tb[size_t(i - 1) * 32 + st]; }
    } sc{tb.data()};
    // packed words written back to front, as the kernel's OpsWriter does
    const uint32_t words = uint32_t((v.R + v.C + 15) / 16);
    std::vector<uint32_t> wv(words + 1, 0);
    int32_t p = int32_t(words * 16);
    auto emit = [&](uint8_t op) {
        p--;
        wv[p >> 4] |= uint32_t(op) << (2 * (p & 15));
    };
    const int n = dp_walk<W>(v, sc, emit);
    {  // the kernel's chunked traceback (one chunk of rows per lane), lanes in turn
        const int32_t P = int32_t(words * 16);
        std::vector<int32_t> rtop(G), rbot(G), c(G), e(G), cnt(G);
        std::vector<char> todo(G, 1);
        for (int s = 0; s < G; s++) {
            dp_chunk_rows(v.R, G, s, rtop[s], rbot[s]);
            c[s] = s == 0 ? v.C : dp_chunk_guess(v, rtop[s]);
        }
        int f = 0;
        g_chunk_rounds = 0;
        for (int round = 0; round <= 32; round++) {
            g_chunk_rounds++;
            for (int s = 0; s < G; s++)
                if (todo[s]) {
                    int32_t jj = c[s];
                    cnt[s] = dp_walk_span<W>(sc, rtop[s], jj, rbot[s]);
                    e[s] = jj;
                }
            f = G;
            for (int s = 1; s < G; s++)
                if (c[s] != e[s - 1]) {
                    f = s;
                    break;
                }
            if (f == G) break;
            for (int s = 0; s < G; s++) {  // from the first wrong lane on: the previous end
                todo[s] = s >= f;
                if (todo[s]) c[s] = e[s - 1];
            }
        }
        if (f != G) return -6;
        std::vector<uint32_t> cw(words + 1, 0);
        int32_t Ps = P;
        const uint32_t lut = dp_op_lut(v);
        for (int s = 0; s < G; s++) {
            int32_t pp = Ps;
            auto put = [&](uint32_t op) {
                pp--;
                cw[pp >> 4] |= op << (2 * (pp & 15));
            };
            dp_walk_span_ops<W>(sc, lut, rtop[s], c[s], rbot[s], put);
            if (Ps - pp != cnt[s]) return -7;
            Ps -= cnt[s];
        }
        if (P - Ps != n) return -5;
        for (int32_t q = 0; q < n; q++)
            if (ops_field(cw.data(), uint32_t(P - n + q)) != ops_field(wv.data(), uint32_t(P - n + q)))
                return -5;
    }
    DpSum sum;
    ops_summary(wv.data(), words * 16 - uint32_t(n), uint32_t(n), sum);
    // cross-check the word-level summary against per-op counting
    uint32_t tot[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++) tot[ops_field(wv.data(), words * 16 - n + i)]++;
    for (int t = 0; t < 4; t++)
        if (tot[t] != sum.tot[t]) return -2;
    const uint32_t f0 = ops_field(wv.data(), words * 16 - n);
    uint32_t fc = 0;
    while (int(fc) < n && ops_field(wv.data(), words * 16 - n + fc) == f0) fc++;
    const uint32_t l0 = ops_field(wv.data(), words * 16 - 1);
    uint32_t lc = 0;
    while (int(lc) < n && ops_field(wv.data(), words * 16 - 1 - lc) == l0) lc++;
    if (sum.ft != f0 || sum.fc != fc || sum.lt != l0 || sum.lc != lc ||
        sum.nruns != (int(fc) == n ? 1 : 2))
        return -3;
    if (n > cap) return -1;
    for (int i = 0; i < n; i++) ops[i] = uint8_t(ops_field(wv.data(), words * 16 - n + i));
    return n;
}

// alignment output (no -c), sequentially, through the same core functions as
// the kernels: seed_hit, make_view with the query reverse complement,
// list_add, AlnText.  out receives the .aln text; returns its length, or -1 if
// cap is too small.
extern "C++" {
struct EmuPieces {
    const SegRec *segs;
    template <class F>
    void each(uint32_t piece, F f) const {
        for (uint8_t o : segs[piece].ops) f(o);
    }
};
}  // extern "C++"

int64_t emu_align_output(int32_t k, int32_t l, int32_t affine, double mis_rate, double indel_rate,
                         uint64_t nq, const uint8_t *qseq, const uint64_t *qoff,
                         const int64_t *quid, uint8_t *out, uint64_t cap) {
    Params p{k, l, affine, 1, mis_rate, indel_rate, 0.6};
    Reads Q;
    load(Q, nq, qseq, qoff, quid, l);
    std::unordered_map<std::pair<uint64_t, uint64_t>, std::vector<uint64_t>, KeyHash> table;
    for (uint64_t r = 0; r < nq; r++) {
        if (!Q.gq[r]) continue;
        const int64_t L = Q.len[r];
        const int32_t nk = query_key_count(L, k);
        for (int32_t i = 0; i < nk; i++) {
            const int64_t pos = query_key_pos(L, k, i);
            Kmer m{0, 0};
            for (int32_t t = 0; t < k; t++) kmer_push(m, Q.code[Q.off[r] + pos + t] & 3u, k);
            table[{m.lo, m.hi}].push_back((uint64_t(r) << 32) | uint64_t(pos));
        }
    }
    std::string text;
    for (uint64_t s = 0; s < nq; s++) {
        text += '>';
        text += std::to_string(Q.uid[s]);
        text += '\n';
        if (!Q.gs[s]) {
            text += '\n';
            continue;
        }
        const int32_t L = int32_t(Q.len[s]);
        const uint8_t *c = Q.code.data() + Q.off[s];
        std::vector<uint64_t> hits[2];
        if (L >= k) {
            for (int32_t f = 0; f + k <= L; f++) {
                Kmer fm{0, 0}, rm{0, 0};
                bool bad = false;
                for (int32_t i = 0; i < k; i++) {
                    bad |= c[f + i] >= 4;
                    kmer_push(fm, c[f + i] & 3u, k);
                }
                if (bad) continue;
                for (int32_t i = k - 1; i >= 0; i--) kmer_push(rm, (c[f + i] & 3u) ^ 2u, k);
                for (int o = 0; o < 2; o++) {
                    Kmer m = o ? rm : fm;
                    auto it = table.find({m.lo, m.hi});
                    if (it == table.end()) continue;
                    for (uint64_t v : it->second) {
                        uint32_t qq = uint32_t(v >> 32);
                        if (Q.uid[qq] == Q.uid[s]) continue;
                        hits[o].push_back(seed_hit(true, o, qq, uint32_t(v), f, L, int32_t(Q.len[qq]), k));
                    }
                }
            }
        }
        struct Cand {
            uint32_t q;
            int orient;
            std::vector<SegRec> segs;
            std::vector<uint64_t> keys;
            bool accepted;
            double rate, len;
        };
        std::vector<Cand> cands;
        for (int o = 0; o < 2; o++) {
            auto &H = hits[o];
            std::sort(H.begin(), H.end());
            size_t g0 = 0;
            for (size_t i = 0; i < H.size(); i++) {
                if (i + 1 != H.size() && hit_q(H[i]) == hit_q(H[i + 1])) continue;
                const int32_t gn = int32_t(i + 1 - g0);
                const uint64_t *G = H.data() + g0;
                auto hit = [G](int32_t h) { return G[h]; };
                std::vector<uint32_t> chain_of(gn);
                std::vector<int32_t> first(gn), last(gn), prev(gn);
                std::vector<int64_t> kl(gn);
                int32_t nch = chain_group(p, hit, gn, chain_of.data(), first.data(), last.data());
                int64_t best = chain_key_lengths(p, hit, gn, chain_of.data(), nch, kl.data(), prev.data());
                const uint32_t qid = hit_q(G[0]);
                const int32_t Lq = int32_t(Q.len[qid]);
                for (int32_t ch = 0; ch < nch; ch++) {
                    if (kl[ch] != best) continue;
                    Cand cd;
                    cd.q = qid;
                    cd.orient = o;
                    for (int32_t h = 0; h < gn; h++)
                        if (chain_of[h] == uint32_t(ch)) cd.keys.push_back(G[h]);
                    auto key = [&cd](int32_t t) { return cd.keys[t]; };
                    Collect col{&cd.segs};
                    walk_chain(p, Lq, L, key, int32_t(cd.keys.size()), col);
                    for (SegRec &sr : cd.segs) {
                        SegView v = make_view(c, L, 0, Q.code.data() + Q.off[qid], int32_t(sr.s0),
                                              int32_t(sr.s1), int32_t(sr.q0), int32_t(sr.q1),
                                              sr.flags, sr.band, Lq, o == 1);
                        run_dp<8>(v, affine != 0, sr.ops, sr.sum);
                    }
                    Asm as;
                    as.segs = cd.segs.data();
                    bool ok = walk_chain(p, Lq, L, key, int32_t(cd.keys.size()), as);
                    cd.accepted = as.built && ok && as.st.good_rates(p, cd.rate, cd.len);
                    cands.push_back(std::move(cd));
                }
                g0 = i + 1;
            }
        }
        struct Slots {
            std::vector<uint32_t> v;
            uint32_t get(uint32_t i) const { return v[i]; }
            void set(uint32_t i, uint32_t x) {
                if (i >= v.size()) v.resize(i + 1);
                v[i] = x;
            }
        } list;
        auto key = [&](uint32_t i) { return uint64_t(Q.uid[cands[i].q]); };
        auto better = [&](uint32_t a, uint32_t b) {
            return record_better(cands[a].rate, cands[a].len, cands[b].rate, cands[b].len);
        };
        uint32_t n = 0;
        uint64_t largest = 0;
        for (uint32_t i = 0; i < cands.size(); i++)
            if (cands[i].accepted) n = list_add(list, n, largest, i, key, better);
        for (uint32_t e = 0; e < n; e++) {
            const Cand &w = cands[list.get(e)];
            const int32_t Lq = int32_t(Q.len[w.q]);
            auto kk = [&w](int32_t t) { return w.keys[t]; };
            AlnText<EmuPieces> sz{EmuPieces{w.segs.data()}, Q.code.data() + Q.off[w.q], Lq, w.orient == 1};
            walk_chain(p, Lq, L, kk, int32_t(w.keys.size()), sz);
            const uint32_t pre = aln_prefix_len(key(list.get(e)), uint32_t(w.orient), sz.pos);
            std::string rec(pre + sz.cig_len + 1 + sz.ins_len + 1, '?');
            AlnText<EmuPieces> wr{EmuPieces{w.segs.data()}, Q.code.data() + Q.off[w.q], Lq, w.orient == 1};
            wr.cig = &rec[pre];
            wr.ins = wr.cig + sz.cig_len + 1;
            walk_chain(p, Lq, L, kk, int32_t(w.keys.size()), wr);
            char *o = &rec[0];
            o = dec_put(o, key(list.get(e)));
            *o++ = ',';
            o = dec_put(o, uint32_t(w.orient));
            *o++ = ',';
            o = dec_put_signed(o, wr.pos);
            *o = ',';
            *wr.cig = ',';
            *wr.ins = ',';
            text += rec;
        }
        text += '\n';
    }
    if (text.size() > cap) return -1;
    std::memcpy(out, text.data(), text.size());
    return int64_t(text.size());
}

// whole path, sequentially, through the core item functions
// ext: NULL, or the overhang votes of --merge (uint32 [reads][20][4], zeroed here)
int emu_correct_ext(int32_t k, int32_t l, int32_t affine, double mis_rate, double indel_rate,
                    double thr, uint64_t nq, const uint8_t *qseq, const uint64_t *qoff,
                    const int64_t *quid, uint8_t *out_seq, uint32_t *imin, uint32_t *imed,
                    uint32_t *imax, double *mis, double *gc, uint32_t *cov_out, uint64_t *counters,
                    uint32_t *ext) {
    Params p{k, l, affine, 0, mis_rate, indel_rate, thr};
    if (ext) std::memset(ext, 0, size_t(nq) * kOverhang * 4 * sizeof(uint32_t));
    Reads Q;
    load(Q, nq, qseq, qoff, quid, l);
    // table: exact multimap
    std::unordered_map<std::pair<uint64_t, uint64_t>, std::vector<uint64_t>, KeyHash> table;
    for (uint64_t r = 0; r < nq; r++) {
        if (!Q.gq[r]) continue;
        const int64_t L = Q.len[r];
        const int32_t nk = query_key_count(L, k);
        for (int32_t i = 0; i < nk; i++) {
            const int64_t pos = query_key_pos(L, k, i);
            Kmer m{0, 0};
            for (int32_t t = 0; t < k; t++) kmer_push(m, Q.code[Q.off[r] + pos + t] & 3u, k);
            table[{m.lo, m.hi}].push_back((uint64_t(r) << 32) | uint64_t(pos));
        }
    }
    std::vector<uint32_t> cov(Q.code.size() * 4, 0);
    uint64_t nhits = 0, nchains = 0, kept_total = 0, dpseg = 0, anomalies = 0;
    for (uint64_t s = 0; s < nq; s++) {  // subject set = query set
        if (!Q.gs[s]) continue;
        const int32_t L = int32_t(Q.len[s]);
        const uint8_t *c = Q.code.data() + Q.off[s];
        std::vector<uint64_t> hits[2];
        if (L >= k) {
            for (int32_t f = 0; f + k <= L; f++) {
                Kmer fm{0, 0}, rm{0, 0};
                bool bad = false;
                for (int32_t i = 0; i < k; i++) {
                    bad |= c[f + i] >= 4;
                    kmer_push(fm, c[f + i] & 3u, k);
                }
                if (bad) continue;
                for (int32_t i = k - 1; i >= 0; i--) kmer_push(rm, (c[f + i] & 3u) ^ 2u, k);
                for (int o = 0; o < 2; o++) {
                    Kmer m = o ? rm : fm;
                    auto it = table.find({m.lo, m.hi});
                    if (it == table.end()) continue;
                    for (uint64_t v : it->second) {
                        uint32_t qq = uint32_t(v >> 32);
                        if (Q.uid[qq] == Q.uid[s]) continue;
                        hits[o].push_back(hit_pack(qq, uint32_t(v), o ? uint32_t(L - k - f) : uint32_t(f)));
                    }
                }
            }
        }
        struct Cand {
            uint32_t q;
            int orient;
            std::vector<SegRec> segs;
            std::vector<uint64_t> keys;
            int status;
            double rate, len;
        };
        std::vector<Cand> cands;
        for (int o = 0; o < 2; o++) {
            auto &H = hits[o];
            std::sort(H.begin(), H.end());
            nhits += H.size();
            size_t g0 = 0;
            for (size_t i = 0; i < H.size(); i++) {
                if (i + 1 != H.size() && hit_q(H[i]) == hit_q(H[i + 1])) continue;
                const int32_t gn = int32_t(i + 1 - g0);
                const uint64_t *G = H.data() + g0;
                auto hit = [G](int32_t h) { return G[h]; };
                std::vector<uint32_t> chain_of(gn);
                std::vector<int32_t> first(gn), last(gn), prev(gn);
                std::vector<int64_t> kl(gn);
                int32_t nch = chain_group(p, hit, gn, chain_of.data(), first.data(), last.data());
                int64_t best = chain_key_lengths(p, hit, gn, chain_of.data(), nch, kl.data(), prev.data());
                nchains += nch;
                const uint32_t qid = hit_q(G[0]);
                for (int32_t ch = 0; ch < nch; ch++) {
                    if (kl[ch] != best) continue;
                    Cand cd;
                    cd.q = qid;
                    cd.orient = o;
                    for (int32_t h = 0; h < gn; h++)
                        if (chain_of[h] == uint32_t(ch)) cd.keys.push_back(G[h]);
                    auto key = [&cd](int32_t t) { return cd.keys[t]; };
                    Collect col{&cd.segs};
                    walk_chain(p, Q.len[qid], L, key, int32_t(cd.keys.size()), col);
                    for (SegRec &sr : cd.segs) {
                        SegView v = make_view(c, L, o, Q.code.data() + Q.off[qid], int32_t(sr.s0),
                                              int32_t(sr.s1), int32_t(sr.q0), int32_t(sr.q1),
                                              sr.flags, sr.band);
                        run_dp<8>(v, affine != 0, sr.ops, sr.sum);
                        dpseg++;
                    }
                    Asm as;
                    as.segs = cd.segs.data();
                    bool ok = walk_chain(p, Q.len[qid], L, key, int32_t(cd.keys.size()), as);
                    cd.status = 0;
                    cd.rate = 0;
                    cd.len = 0;
                    if (as.built) {
                        cd.status = 1;
                        if (ok && as.st.good_rates(p, cd.rate, cd.len)) cd.status = 2;
                    }
                    cands.push_back(std::move(cd));
                }
                g0 = i + 1;
            }
        }
        // dedupe: per query, forward chains then reverse-complement chains
        std::vector<size_t> order(cands.size());
        for (size_t i = 0; i < order.size(); i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t b) { return cands[a].q < cands[b].q; });
        for (size_t a = 0; a < order.size();) {
            size_t b = a;
            int64_t best = -1;
            while (b < order.size() && cands[order[b]].q == cands[order[a]].q) {
                const Cand &x = cands[order[b]];
                if (x.status == 2 &&
                    (best < 0 || record_better(x.rate, x.len, cands[best].rate, cands[best].len)))
                    best = int64_t(order[b]);
                b++;
            }
            if (best >= 0) {
                kept_total++;
                Cand &w = cands[best];
                Vote vt;
                vt.sc = c;
                vt.Ls = L;
                vt.orient = w.orient;
                vt.qc = Q.code.data() + Q.off[w.q];
                vt.Lq = Q.len[w.q];
                vt.cov = cov.data() + Q.off[w.q] * 4;
                vt.segs = w.segs.data();
                auto key = [&w](int32_t t) { return w.keys[t]; };
                walk_chain(p, vt.Lq, vt.Ls, key, int32_t(w.keys.size()), vt);
                anomalies += vt.anomalies;
                if (ext) {  // the device's overhang pass over the same record
                    const SegRec *sr = w.segs.data();
                    auto sums = [sr](uint32_t i) { return sr[i].sum; };
                    OverhangWalk<decltype(sums)> ow{sums};
                    walk_chain(p, vt.Lq, vt.Ls, key, int32_t(w.keys.size()), ow);
                    uint32_t *m = ext + size_t(w.q) * kOverhang * 4;
                    for (int64_t i = 0; ow.other && i < kOverhang && ow.ps + i < L; i++) {
                        const int64_t x = ow.ps + i;
                        const uint8_t code = w.orient ? uint8_t(c[L - 1 - x] ^ 2u) : c[x];
                        if (code < 4) m[i * 4 + code]++;
                    }
                }
            }
            a = b;
        }
    }
    if (cov_out) std::memcpy(cov_out, cov.data(), cov.size() * 4);
    // consensus
    for (uint64_t r = 0; r < nq; r++) {
        const uint64_t b = Q.off[r];
        const uint32_t L = Q.len[r];
        gc[r] = Q.gc[r];
        std::memcpy(out_seq + b, qseq + b, L);
        if (!Q.gq[r]) {
            imin[r] = imed[r] = imax[r] = 0;
            mis[r] = 0;
            continue;
        }
        uint32_t changed = 0;
        std::vector<uint32_t> sums(L);
        for (uint32_t i = 0; i < L; i++) {
            uint32_t cc[4];
            const uint8_t own = Q.code[b + i];
            for (int j = 0; j < 4; j++) cc[j] = cov[(b + i) * 4 + j] + (own == j ? 1 : 0);
            int32_t id = column_consensus(cc, thr);
            uint8_t nb = own;
            if (id >= 0) {
                if (uint8_t(id) != own) changed++;
                nb = uint8_t(id);
            }
            out_seq[b + i] = uint8_t(code_base(nb));
            sums[i] = cc[0] + cc[1] + cc[2] + cc[3];
        }
        std::sort(sums.begin(), sums.end());
        imin[r] = sums[0];
        imax[r] = sums.back();
        imed[r] = (L % 2 == 0) ? (sums[L / 2] + sums[L / 2 - 1]) / 2 : sums[(L - 1) / 2];
        mis[r] = double(changed) / double(L);
    }
    if (counters) {
        counters[0] = nhits;
        counters[1] = nchains;
        counters[2] = kept_total;
        counters[3] = dpseg;
        counters[4] = anomalies;
    }
    return 0;
}

int emu_correct(int32_t k, int32_t l, int32_t affine, double mis_rate, double indel_rate,
                double thr, uint64_t nq, const uint8_t *qseq, const uint64_t *qoff,
                const int64_t *quid, uint8_t *out_seq, uint32_t *imin, uint32_t *imed,
                uint32_t *imax, double *mis, double *gc, uint32_t *cov_out, uint64_t *counters) {
    return emu_correct_ext(k, l, affine, mis_rate, indel_rate, thr, nq, qseq, qoff, quid, out_seq,
                           imin, imed, imax, mis, gc, cov_out, counters, nullptr);
}

// item checks of the shared core: merge_pair on one pair, and list_add over
// records in arrival order (record_better as the comparison)
int emu_merge_pair(const uint8_t *left, int32_t lenL, const uint8_t *right, int32_t lenR,
                   const uint32_t *extL, const uint32_t *extR, uint8_t *out) {
    return int(merge_pair(reinterpret_cast<const char *>(left), lenL,
                          reinterpret_cast<const char *>(right), lenR, extL, extR,
                          reinterpret_cast<char *>(out)));
}

// ops_summary of the packed op range [first, first + P) of w against the
// fields read one by one (-1 when they differ), then against the parts of G
// lanes (each taking every G-th word) merged as the kernel's shuffle tree
// merges them, for G = 1..32 (the first G that differs, 0 when none does)
int32_t emu_ops_summary_groups(const uint32_t *w, uint32_t first, uint32_t P) {
    DpSum ref;
    ops_summary(w, first, P, ref);
    {
        auto field = [&](uint32_t p) { return (w[p >> 4] >> (2 * (p & 15))) & 3u; };
        uint32_t tot[4] = {0, 0, 0, 0};
        for (uint32_t q = first; q < first + P; q++) tot[field(q)]++;
        const uint32_t ft = field(first), lt = field(first + P - 1);
        uint32_t fc = 0, lc = 0;
        while (fc < P && field(first + fc) == ft) fc++;
        while (lc < P && field(first + P - 1 - lc) == lt) lc++;
        for (int k = 0; k < 4; k++)
            if (ref.tot[k] != tot[k]) return -1;
        if (ref.ft != ft || ref.fc != fc || ref.lt != lt || ref.lc != lc || ref.nruns != (fc == P ? 1 : 2))
            return -1;
    }
    for (uint32_t G = 1; G <= 32; G++) {
        std::vector<OpsPart> part(G);
        for (uint32_t s = 0; s < G; s++) part[s] = ops_part(w, first, P, s, G);
        for (uint32_t d = 1; d < G; d <<= 1) {
            const std::vector<OpsPart> old = part;  // a shuffle reads every lane's value before the step
            for (uint32_t s = 0; s + d < G; s++) part[s] = ops_part_merge(old[s], old[s + d]);
        }
        DpSum got;
        ops_part_sum(part[0], w, first, P, got);
        if (std::memcmp(&got, &ref, sizeof(DpSum)) != 0) return int32_t(G);
    }
    return 0;
}

// RecState over the same events: runs through add, the steps of each DP piece
// packed as the kernel packs ops (2 bits each, at the end of the words) and
// summarised by ops_summary for add_piece
void emu_record_score(uint32_t nev, const uint32_t *piece, const uint8_t *type,
                      const int32_t *count, const uint8_t *, int64_t *out) {
    RecState st;
    for (uint32_t i = 0; i < nev;) {
        if (piece[i] == 0) {
            st.add(type[i], count[i]);
            i++;
            continue;
        }
        uint32_t j = i;
        while (j < nev && piece[j] == piece[i]) j++;
        const uint32_t P = j - i, words = (P + 15) / 16 + 1, first = words * 16 - P;
        std::vector<uint32_t> w(words, 0);
        for (uint32_t k = 0; k < P; k++) {
            const uint32_t f = first + k;
            w[f >> 4] |= uint32_t(type[i + k]) << (2 * (f & 15));
        }
        DpSum sum;
        ops_summary(w.data(), first, P, sum);
        st.add_piece(sum);
        i = j;
    }
    st.score(out[0], out[1], out[2]);
}

int32_t emu_chain(int32_t k, double indel_rate, uint32_t n, const int64_t *posQ,
                  const int64_t *posS, uint32_t *chain_of, uint8_t *kept) {
    Params p{k, 0, 0, 0, 1.0, indel_rate, 0.6};
    std::vector<uint64_t> hits(n);
    for (uint32_t h = 0; h < n; h++) hits[h] = hit_pack(0, uint32_t(posQ[h]), uint32_t(posS[h]));
    auto hit = [&hits](int32_t h) { return hits[size_t(h)]; };
    std::vector<int32_t> first(n + 1), last(n + 1), prev(n + 1);
    std::vector<int64_t> kl(n + 1);
    const int32_t nch = chain_group(p, hit, int32_t(n), chain_of, first.data(), last.data());
    const int64_t best = chain_key_lengths(p, hit, int32_t(n), chain_of, nch, kl.data(), prev.data());
    for (int32_t c = 0; c < nch; c++) kept[c] = kl[size_t(c)] == best ? 1 : 0;
    return nch;
}

// walk_chain on one chain: every DP piece (Collect), each aligned (run_dp), then
// the record replayed with getAlignment2's exits (Asm): the pieces the
// reference computes (Asm::used), the position and the record's fate
int32_t emu_chain_layout(int32_t k, int32_t l, int32_t affine, double mis_rate, double indel_rate,
                         const uint8_t *qseq, int32_t Lq, const uint8_t *sseq, int32_t Ls,
                         uint32_t nkeys, const int64_t *posQ, const int64_t *posS, int64_t *seg,
                         int32_t cap, int64_t *pos_out, int32_t *status) {
    Params p{k, l, affine, 0, mis_rate, indel_rate, 0.6};
    std::vector<uint8_t> qc(static_cast<size_t>(Lq)), sc(static_cast<size_t>(Ls));
    for (int32_t i = 0; i < Lq; i++) qc[size_t(i)] = base_code(qseq[i]);
    for (int32_t i = 0; i < Ls; i++) sc[size_t(i)] = base_code(sseq[i]);
    std::vector<uint64_t> keys(nkeys);
    for (uint32_t i = 0; i < nkeys; i++) keys[i] = hit_pack(0, uint32_t(posQ[i]), uint32_t(posS[i]));
    auto key = [&keys](int32_t t) { return keys[size_t(t)]; };
    std::vector<SegRec> segs;
    Collect col{&segs};
    walk_chain(p, Lq, Ls, key, int32_t(nkeys), col);
    for (SegRec &sr : segs) {
        SegView v = make_view(sc.data(), Ls, 0, qc.data(), int32_t(sr.s0), int32_t(sr.s1),
                              int32_t(sr.q0), int32_t(sr.q1), sr.flags, sr.band);
        run_dp<8>(v, affine != 0, sr.ops, sr.sum);
    }
    Asm as;
    as.segs = segs.data();
    struct Pos {
        int64_t pos = 0;
        void begin(int64_t, int64_t, int64_t) {}
        void position(int64_t q) { pos = q; }
        void run(uint8_t, int64_t) {}
        void dp(int64_t, int64_t, int64_t, int64_t, uint32_t, int64_t) {}
        bool check(int64_t, int64_t) { return true; }
        void finish() {}
    } ps;
    walk_chain(p, Lq, Ls, key, int32_t(nkeys), ps);
    const bool ok = walk_chain(p, Lq, Ls, key, int32_t(nkeys), as);
    double rate = 0, len = 0;
    *status = !as.built ? 0 : (ok && as.st.good_rates(p, rate, len)) ? 2 : 1;
    *pos_out = ps.pos;
    const int32_t n = int32_t(as.used);
    for (int32_t i = 0; i < n && i < cap; i++) {
        const SegRec &g = segs[size_t(i)];
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

// AlnText driven by the same events: runs through run(), each DP piece through
// dp() with its steps from a vector source; sized, then written, as the kernels do
extern "C++" {
struct VecPieces {
    const std::vector<std::vector<uint8_t>> *p;
    template <class F>
    void each(uint32_t i, F f) const {
        for (uint8_t o : (*p)[i]) f(o);
    }
};
}  // extern "C++"

int32_t emu_record_text(uint64_t key, uint32_t orient, int64_t pos, uint32_t nev,
                        const uint32_t *piece, const uint8_t *type, const int32_t *count,
                        const uint8_t *query, int32_t Lq, int32_t qrc, uint8_t *out, int32_t cap) {
    std::vector<uint8_t> qc(static_cast<size_t>(Lq));
    for (int32_t i = 0; i < Lq; i++) qc[size_t(i)] = base_code(query[i]);
    std::vector<std::vector<uint8_t>> pieces;
    for (uint32_t i = 0; i < nev; i++) {
        if (!piece[i]) continue;
        if (i == 0 || piece[i - 1] != piece[i]) pieces.emplace_back();
        pieces.back().push_back(type[i]);
    }
    auto drive = [&](AlnText<VecPieces> &t) {
        t.position(pos);
        for (uint32_t i = 0; i < nev; i++) {
            if (!piece[i]) {
                t.run(type[i], count[i]);
            } else if (i == 0 || piece[i - 1] != piece[i]) {
                t.dp(0, 0, 0, 0, 0, 0);
            }
        }
        t.finish();
    };
    AlnText<VecPieces> sz{VecPieces{&pieces}, qc.data(), Lq, qrc != 0};
    drive(sz);
    const uint32_t pre = aln_prefix_len(key, orient, sz.pos);
    const uint32_t total = pre + sz.cig_len + 1 + sz.ins_len + 1;
    if (int32_t(total) > cap) return -1;
    AlnText<VecPieces> wr{VecPieces{&pieces}, qc.data(), Lq, qrc != 0};
    char *o = reinterpret_cast<char *>(out);
    wr.cig = o + pre;
    wr.ins = wr.cig + sz.cig_len + 1;
    drive(wr);
    o = dec_put(o, key);
    *o++ = ',';
    o = dec_put(o, orient);
    *o++ = ',';
    o = dec_put_signed(o, wr.pos);
    *o = ',';
    *wr.cig = ',';
    *wr.ins = ',';
    return int32_t(total);
}

int32_t emu_key_positions(int64_t L, int64_t k, int64_t *out) {
    const int32_t n = L >= k ? query_key_count(L, int32_t(k)) : 0;
    for (int32_t i = 0; i < n; i++) out[i] = query_key_pos(L, k, i);
    return n;
}

void emu_columns(uint64_t n, const uint32_t *counts, double thr, int32_t *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = column_consensus(counts + 4 * i, thr);
}

int32_t emu_record_list(uint32_t n, const uint64_t *key, const double *rate_sum, const double *len,
                        uint32_t *out) {
    struct Slots {
        uint32_t *o;
        uint32_t get(uint32_t i) const { return o[i]; }
        void set(uint32_t i, uint32_t x) { o[i] = x; }
    } list{out};
    auto k = [key](uint32_t i) { return key[i]; };
    auto better = [rate_sum, len](uint32_t a, uint32_t b) {
        return record_better(rate_sum[a], len[a], rate_sum[b], len[b]);
    };
    uint32_t m = 0;
    uint64_t largest = 0;
    for (uint32_t i = 0; i < n; i++) m = list_add(list, m, largest, i, k, better);
    return int32_t(m);
}

// --merge after the emulated correction: merge_pair on reads (2p, 2p+1) of the
// corrected reads.  merged_seq has the read layout (pair p's merged read from
// off[2p], else both corrected reads); merged_len[p] = 0 when not merged.
int emu_merge(int32_t k, int32_t l, int32_t affine, double mis_rate, double indel_rate, double thr,
              uint64_t nq, const uint8_t *qseq, const uint64_t *qoff, const int64_t *quid,
              uint8_t *corrected, uint8_t *merged_seq, uint32_t *merged_len, uint32_t *ext) {
    if (nq % 2) return -1;
    std::vector<uint32_t> imin(nq), imed(nq), imax(nq);
    std::vector<double> mis(nq), gc(nq);
    emu_correct_ext(k, l, affine, mis_rate, indel_rate, thr, nq, qseq, qoff, quid, corrected,
                    imin.data(), imed.data(), imax.data(), mis.data(), gc.data(), nullptr, nullptr,
                    ext);
    std::memcpy(merged_seq, corrected, qoff[nq]);
    for (uint64_t pr = 0; pr < nq / 2; pr++) {
        const uint64_t a = qoff[2 * pr], b = qoff[2 * pr + 1], e = qoff[2 * pr + 2];
        merged_len[pr] = merge_pair(reinterpret_cast<const char *>(corrected + a), int(b - a),
                                    reinterpret_cast<const char *>(corrected + b), int(e - b),
                                    ext + 2 * pr * kOverhang * 4, ext + (2 * pr + 1) * kOverhang * 4,
                                    reinterpret_cast<char *>(merged_seq + a));
    }
    return 0;
}
}
