// hero_host.cpp -- host side of the drop-in (see hero_host.h).
#include "hero_host.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <algorithm>
#include <string_view>
#include <thread>
#include <vector>

namespace herohost {

// ---------------------------------------------------------------------------
// Config::setConfig (Config.cpp:118-243); flags outside the consensus path are
// refused with a message instead of being silently ignored.
// ---------------------------------------------------------------------------
void Config::help() {
    std::cout << "Usage: hero_b200 -q <query[,query...]> -s <subject[,subject...]> [-c [thr]]\n"
                 "  -o/--out      output prefix (default: query) -> <out>.fasta, <out>.info with -c,\n"
                 "                else <out>.aln (every subject read's alignment records)\n"
                 "  -c [thr]      call the consensus (default threshold 0.6)\n"
                 "  --covinfo     write <out>.info (coverage min/median/max, rates)\n"
                 "  --merge       with -c: merge read pairs (2i, 2i+1) -> <out>_merged.fasta,\n"
                 "                <out>_unmerged.fasta instead of <out>.fasta\n"
                 "  --singleReads inputs are unpaired reads\n"
                 "  -k            k-mer length (default 39, at most 63)\n"
                 "  -m / -i       maximum mismatch / indel rate in percent (default 100)\n"
                 "  -l            minimum overlap length (default 40)\n"
                 "  -a a|g        affine or global aligner (default g)\n"
                 "  -t -y -z -f   accepted for compatibility (host threads, chunk sizes, table factor)\n"
                 "  --device N    CUDA device; --batch N subject reads per device batch\n";
}

bool Config::parse(int argc, char **argv) {
    auto split = [](const std::string &s, std::vector<std::string> &out) {
        std::stringstream ss(s);
        std::string item;
        while (std::getline(ss, item, ',')) out.push_back(item);
    };
    if (argc <= 1) {
        help();
        return false;
    }
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](std::string &v) -> bool {
            if (i + 1 >= argc) {
                std::cerr << "missing value after " << a << "\n";
                return false;
            }
            v = argv[++i];
            return true;
        };
        std::string v;
        if (a == "-h" || a == "--help") {
            help();
            return false;
        } else if (a == "-s" || a == "--subject") {
            if (!next(v)) return false;
            split(v, subject_files);
        } else if (a == "-q" || a == "--query") {
            if (!next(v)) return false;
            split(v, query_files);
        } else if (a == "-o" || a == "--out") {
            if (!next(v)) return false;
            out = v;
            // a trailing ".aln" is dropped (Config.cpp:213-221 intends this)
            if (out.size() >= 4 && out.compare(out.size() - 4, 4, ".aln") == 0)
                out = out.substr(0, out.size() - 4);
        } else if (a == "-k") {
            if (!next(v)) return false;
            k = std::atoi(v.c_str());
        } else if (a == "-m") {
            if (!next(v)) return false;
            mis_rate = std::atof(v.c_str()) / 100.0;
        } else if (a == "-i") {
            if (!next(v)) return false;
            indel_rate = std::atof(v.c_str()) / 100.0;
        } else if (a == "-l") {
            if (!next(v)) return false;
            min_overlap = std::atoi(v.c_str());
        } else if (a == "-t") {
            if (!next(v)) return false;
            threads = std::atoi(v.c_str());
        } else if (a == "-z") {
            if (!next(v)) return false;
            stream_chunk = std::strtoull(v.c_str(), nullptr, 10);
        } else if (a == "-y") {
            if (!next(v)) return false;
            query_chunk = std::strtoull(v.c_str(), nullptr, 10);
        } else if (a == "-f") {
            if (!next(v)) return false;  // table size factor: the device table sizes itself
        } else if (a == "-a") {
            if (!next(v)) return false;
            if (v == "a") affine = true;
            if (v == "g") affine = false;
        } else if (a == "-c") {
            consensus = true;
            if (i + 1 < argc && argv[i + 1][0] >= '0' && argv[i + 1][0] <= '9')
                consensus_thr = std::atof(argv[++i]);
        } else if (a == "--covinfo") {
            covinfo = true;
        } else if (a == "--singleReads") {
            single_reads = true;
        } else if (a == "--device") {
            if (!next(v)) return false;
            device = std::atoi(v.c_str());
        } else if (a == "--batch") {
            if (!next(v)) return false;
            subject_batch = uint32_t(std::strtoul(v.c_str(), nullptr, 10));
        } else if (a == "--merge") {
            merge = true;
        } else if (a == "--mapping") {
            mapping = true;
        } else if (a == "-v" || a == "--covfilter" ||
                   a == "--suffix" || a == "--size" || a == "--notification") {
            std::cerr << a << ": not part of the path this build replaces\n";
            return false;
        } else {
            std::cerr << "unknown flag " << a << "\n";
            help();
            return false;
        }
    }
    if (subject_files.empty() || query_files.empty()) {
        std::cerr << "missed -subject or -query input files!\n";
        return false;
    }
    if (k < 1 || k > 63) {
        std::cerr << "-k must be in 1..63\n";
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// read loading (QueryDataset.cpp:103-244): FASTQ = four lines per read, FASTA =
// header line then everything up to the next '>' with newlines removed; names
// lose a leading '>' or '@'; bases are upper-cased; id = atoi(name).
// ---------------------------------------------------------------------------
// host threads for parsing and formatting
static unsigned host_threads() {
    const unsigned t = std::thread::hardware_concurrency();
    return t ? (t > 64 ? 64 : t) : 4;
}

// runs fn(begin, end) over [0, n) in one contiguous piece per thread
template <class Fn>
static void parallel_ranges(uint64_t n, Fn fn) {
    const unsigned T = n < 4096 ? 1 : host_threads();
    if (T == 1) {
        fn(uint64_t(0), n);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++) {
        const uint64_t a = n * t / T, b = n * (t + 1) / T;
        th.emplace_back([=] { fn(a, b); });
    }
    for (std::thread &x : th) x.join();
}

// The file is mapped, not copied.  FASTQ: a record is four lines (the
// reference reads them with four getline calls, QueryDataset.cpp:246-391), so
// the threads count the line breaks of their slices, a scan numbers the lines,
// and record r is lines 4r..4r+3; FASTA: one pass from '>' to '>'.  Threads then
// parse the ids and copy the uppercased bases into place.
namespace {

struct Mapped {
    const char *d = nullptr;
    size_t n = 0;
    int fd = -1;
    ~Mapped() {
        if (d && n) munmap(const_cast<char *>(d), n);
        if (fd >= 0) close(fd);
    }
};

char upper_ascii(char c) { return (c >= 'a' && c <= 'z') ? char(c - 32) : c; }

}  // namespace

bool load_reads(const std::string &path, ReadSet &out, std::string *err) {
    Mapped m;
    m.fd = open(path.c_str(), O_RDONLY);
    if (m.fd < 0) {
        if (err) *err = "Unable to open file: " + path;
        return false;
    }
    struct stat st;
    if (fstat(m.fd, &st) != 0) {
        if (err) *err = "Unable to open file: " + path;
        return false;
    }
    m.n = size_t(st.st_size);
    if (m.n == 0) return true;
    void *mp = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (mp == MAP_FAILED) {
        m.n = 0;
        if (err) *err = "Unable to map file: " + path;
        return false;
    }
    m.d = static_cast<const char *>(mp);
    madvise(mp, m.n, MADV_SEQUENTIAL | MADV_WILLNEED);
    const char *d = m.d;
    const size_t n = m.n;
    const bool fasta = d[0] == '>';
    if (!fasta && d[0] != '@') {
        if (err) *err = "Unknown input file format: " + path;
        return false;
    }
    struct Rec {
        size_t name, nlen, seq, slen;  // spans in the file; FASTA sequences may hold newlines
    };
    std::vector<Rec> recs;
    if (!fasta) {
        // line starts, numbered across the slices of the threads
        const unsigned T = n < (1u << 20) ? 1 : host_threads();
        std::vector<uint64_t> cnt(T + 1, 0);
        auto slice = [&](unsigned t, size_t &a, size_t &b) {
            a = n * t / T;
            b = n * (t + 1) / T;
        };
        auto each_break = [&](size_t a, size_t b, auto fn) {
            const char *q = d + a;
            const char *e = d + b;
            while (q < e) {
                const void *h = std::memchr(q, '\n', size_t(e - q));
                if (!h) break;
                const char *x = static_cast<const char *>(h);
                fn(size_t(x - d));
                q = x + 1;
            }
        };
        auto run = [&](auto fn) {
            if (T == 1) {
                fn(0u);
                return;
            }
            std::vector<std::thread> th;
            for (unsigned t = 0; t < T; t++) th.emplace_back(fn, t);
            for (std::thread &x : th) x.join();
        };
        // a line starts at 0 and after every break that is not the last byte
        run([&](unsigned t) {
            size_t a, b;
            slice(t, a, b);
            uint64_t c = 0;
            each_break(a, b, [&](size_t i) { c += i + 1 < n; });
            cnt[t + 1] = c;
        });
        for (unsigned t = 0; t < T; t++) cnt[t + 1] += cnt[t];
        const uint64_t nlines = cnt[T] + 1;
        std::vector<uint64_t> ls(nlines + 1);
        ls[0] = 0;
        run([&](unsigned t) {
            size_t a, b;
            slice(t, a, b);
            uint64_t j = cnt[t] + 1;
            each_break(a, b, [&](size_t i) {
                if (i + 1 < n) ls[j++] = i + 1;
            });
        });
        // one past the end of the last line: its break, or the end of the file
        ls[nlines] = d[n - 1] == '\n' ? n : n + 1;
        auto span = [&](uint64_t j, size_t &b, size_t &len) {
            b = size_t(ls[j]);
            len = size_t(ls[j + 1]) - 1 - b;  // up to the break ending line j
        };
        recs.reserve(nlines / 4 + 1);
        for (uint64_t g = 0; g < nlines; g += 4) {
            size_t b0, n0, b1, n1;
            span(g, b0, n0);
            if (g + 1 >= nlines) {
                if (n0) {  // a lone header line at the end
                    if (err) *err = "truncated FASTQ record in " + path;
                    return false;
                }
                break;
            }
            span(g + 1, b1, n1);
            if (!n0 && !n1) continue;  // blank lines
            recs.push_back({b0, n0, b1, n1});
        }
    } else {
        size_t p = 0;
        recs.reserve(n / 256 + 16);
        while (p < n) {
            const void *q0 = std::memchr(d + p, '\n', n - p);
            const size_t e0 = q0 ? size_t(static_cast<const char *>(q0) - d) : n;
            const size_t b0 = p, n0 = e0 - p;
            p = e0 < n ? e0 + 1 : n;
            const void *q = p < n ? std::memchr(d + p, '>', n - p) : nullptr;
            const size_t e = q ? size_t(static_cast<const char *>(q) - d) : n;
            const size_t b = p;
            p = e < n ? e + 1 : n;
            if (!n0 && e == b) continue;  // blank trailing record
            recs.push_back({b0, n0, b, e - b});
        }
    }
    const uint64_t nr = recs.size(), base_reads = out.uid.size();
    const uint64_t base = out.seq.size();
    std::vector<uint64_t> len(nr);
    out.uid.resize(base_reads + nr);
    parallel_ranges(nr, [&](uint64_t a, uint64_t b) {
        char nm[64];
        std::string big;
        for (uint64_t r = a; r < b; r++) {
            const Rec &x = recs[r];
            size_t nb = x.name, nl = x.nlen;
            if (nl && (d[nb] == '>' || d[nb] == '@')) {
                nb++;
                nl--;
            }
            const char *s;
            if (nl < sizeof(nm)) {
                std::memcpy(nm, d + nb, nl);
                nm[nl] = 0;
                s = nm;
            } else {
                big.assign(d + nb, nl);
                s = big.c_str();
            }
            out.uid[base_reads + r] = int64_t(std::atoi(s));
            uint64_t l = x.slen;
            if (fasta) l -= uint64_t(std::count(d + x.seq, d + x.seq + x.slen, '\n'));
            len[r] = l;
        }
    });
    out.off.resize(base_reads + nr + 1);
    uint64_t tot = base;
    for (uint64_t r = 0; r < nr; r++) {
        tot += len[r];
        out.off[base_reads + r + 1] = tot;
    }
    out.seq.resize(tot);
    parallel_ranges(nr, [&](uint64_t a, uint64_t b) {
        for (uint64_t r = a; r < b; r++) {
            const Rec &x = recs[r];
            char *o = &out.seq[out.off[base_reads + r]];
            if (!fasta) {
                for (size_t i = 0; i < x.slen; i++) o[i] = upper_ascii(d[x.seq + i]);
                continue;
            }
            for (size_t i = 0; i < x.slen; i++) {
                const char c = d[x.seq + i];
                if (c == '\n') continue;
                *o++ = upper_ascii(c);
            }
        }
    });
    return true;
}

bool QueryDataset::build(const Config &c, std::string *err) {
    for (const std::string &path : c.query_files)
        if (!load_reads(path, reads, err)) return false;
    return true;
}

// QueryDataset::writeQueryOut (QueryDataset.cpp:414-537): records formatted by
// threads in contiguous pieces, appended in order.  A double prints as an
// ostream prints it by default (precision 6, the %g conversion).
bool QueryDataset::write(const Config &c, std::string *err) const {
    const uint64_t n = reads.n();
    if ((!c.single_reads || c.merge) && (n % 2)) {
        if (err) *err = "an odd number of reads needs --singleReads (the paired writer reads past the end)";
        return false;
    }
    const unsigned T = n < 4096 ? 1 : host_threads();
    std::vector<std::string> fa_parts(T), info_parts(T);
    auto piece = [&](unsigned t) {
        const uint64_t a = n * t / T, b = n * (t + 1) / T;
        std::string &fa = fa_parts[t], &fi = info_parts[t];
        fa.reserve(size_t(reads.off[b] - reads.off[a]) + size_t(b - a) * 24);
        char buf[160];
        for (uint64_t i = a; i < b; i++) {
            const uint64_t L = reads.off[i + 1] - reads.off[i];
            int k = std::snprintf(buf, sizeof(buf), ">%lld\n", static_cast<long long>(reads.uid[i]));
            fa.append(buf, size_t(k));
            fa.append(corrected.data() + reads.off[i], size_t(L));
            fa.push_back('\n');
            if (c.covinfo) {
                k = std::snprintf(buf, sizeof(buf), "%lld\t%u\t%u\t%u\t%llu\t%g\t%g\n",
                                  static_cast<long long>(reads.uid[i]), imin[i], imed[i], imax[i],
                                  static_cast<unsigned long long>(L), mismatch_rate[i], gc[i]);
                fi.append(buf, size_t(k));
            }
        }
    };
    if (T == 1) {
        piece(0);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < T; t++) th.emplace_back(piece, t);
        for (std::thread &x : th) x.join();
    }
    // both files are opened in append mode, as the reference does
    auto put = [&](const std::string &path, const std::vector<std::string> &parts) {
        std::FILE *f = std::fopen(path.c_str(), "ab");
        if (!f) return false;
        bool good = true;
        for (const std::string &x : parts)
            if (!x.empty() && std::fwrite(x.data(), 1, x.size(), f) != x.size()) good = false;
        return std::fclose(f) == 0 && good;
    };
    if (c.merge) {
        // QueryDataset::writeQueryOut with --merge (QueryDataset.cpp:417-459): a
        // merged pair goes to _merged.fasta as the left read's id and the merged
        // read, any other pair to _unmerged.fasta as both reads
        // (isGoodRead() is always true, QueryRead.cpp:214-216)
        std::string mg, um;
        char buf[32];
        for (uint64_t p = 0; 2 * p + 1 < n; p++) {
            const uint64_t a = reads.off[2 * p];
            if (merged_len[p]) {
                int k = std::snprintf(buf, sizeof(buf), ">%lld\n", static_cast<long long>(reads.uid[2 * p]));
                mg.append(buf, size_t(k));
                mg.append(merged.data() + a, merged_len[p]);
                mg.push_back('\n');
            } else {
                for (uint64_t r = 2 * p; r < 2 * p + 2; r++) {
                    int k = std::snprintf(buf, sizeof(buf), ">%lld\n", static_cast<long long>(reads.uid[r]));
                    um.append(buf, size_t(k));
                    um.append(merged.data() + reads.off[r], size_t(reads.off[r + 1] - reads.off[r]));
                    um.push_back('\n');
                }
            }
        }
        if (!put(c.out + "_merged.fasta", {mg}) || !put(c.out + "_unmerged.fasta", {um})) {
            if (err) *err = "cannot write " + c.out + "_merged.fasta / _unmerged.fasta";
            return false;
        }
    } else if (!put(c.out + ".fasta", fa_parts)) {
        if (err) *err = "cannot write " + c.out + ".fasta";
        return false;
    }
    if (c.covinfo && !put(c.out + ".info", info_parts)) {
        if (err) *err = "cannot write " + c.out + ".info";
        return false;
    }
    return true;
}

bool SubjectDataset::next(ReadSet &chunk, std::string *err) {
    chunk = ReadSet();
    // large chunks: the device batches internally; the result does not depend
    // on the chunking (votes commute)
    const uint64_t want = 4u << 20;
    while (chunk.n() < want) {
        if (!loaded || pos >= cur.n()) {
            if (file >= cfg.subject_files.size()) break;
            cur = ReadSet();
            if (!load_reads(cfg.subject_files[file++], cur, err)) return false;
            pos = 0;
            loaded = true;
            continue;
        }
        const uint64_t take = std::min<uint64_t>(want - chunk.n(), cur.n() - pos);
        const uint64_t b = cur.off[pos], e = cur.off[pos + take];
        chunk.seq.append(cur.seq, b, e - b);
        for (uint64_t i = 0; i < take; i++) {
            chunk.uid.push_back(cur.uid[pos + i]);
            chunk.off.push_back(chunk.off.back() + (cur.off[pos + i + 1] - cur.off[pos + i]));
        }
        pos += take;
    }
    return true;
}

static bool ok(hero_ctx *ctx, int rc, const char *what, std::string *err) {
    if (rc == HERO_OK) return true;
    if (err) *err = std::string(what) + ": " + (ctx ? hero_last_error(ctx) : "") +
                    " (status " + std::to_string(rc) + ")";
    return false;
}

bool HashTableGpu::createHashTables(const Config &c, QueryDataset *q, std::string *err) {
    dataSet = q;
    hero_params p;
    hero_default_params(&p);
    p.k = c.k;
    p.min_overlap = c.min_overlap;
    p.aligner = c.affine ? HERO_ALIGNER_AFFINE : HERO_ALIGNER_GLOBAL;
    p.max_mismatch_rate = c.mis_rate;
    p.max_indel_rate = c.indel_rate;
    p.consensus_threshold = c.consensus_thr;
    p.device = c.device;
    p.subject_batch = c.subject_batch;
    p.flags = !c.consensus ? HERO_FLAG_ALIGNMENT_OUTPUT
              : c.mapping  ? HERO_FLAG_MAPPING
              : c.merge    ? HERO_FLAG_MERGE_PAIRS
                           : 0u;
    if (!ok(nullptr, hero_create(&p, &ctx), "hero_create", err)) return false;
    const ReadSet &r = q->reads;
    return ok(ctx, hero_set_queries(ctx, reinterpret_cast<const uint8_t *>(r.seq.data()),
                                    r.off.data(), r.uid.data(), r.n()),
              "hero_set_queries", err);
}

bool HashTableGpu::insertQueryDataset(std::string *err) {
    return ok(ctx, hero_build_index(ctx), "hero_build_index", err);
}

HashTableGpu::~HashTableGpu() {
    if (ctx) hero_destroy(ctx);
}

// SubjectReadAligner::writeToFile (SubjectReadAligner.cpp:854-906): after each
// chunk the chunk's alignment text is appended to <out>.aln
static bool write_alignments(const Config &c, hero_ctx *ctx, std::string *err) {
    uint64_t n = 0;
    if (!ok(ctx, hero_alignments_size(ctx, &n), "hero_alignments_size", err)) return false;
    std::vector<uint8_t> buf(n ? n : 1);
    if (!ok(ctx, hero_alignments_take(ctx, buf.data(), n), "hero_alignments_take", err)) return false;
    const std::string path = c.out + ".aln";
    std::FILE *f = std::fopen(path.c_str(), "ab");
    if (!f) {
        if (err) *err = "Unable to open file: " + path;
        return false;
    }
    const bool good = std::fwrite(buf.data(), 1, n, f) == n;
    return (std::fclose(f) == 0) && good;
}

bool SubjectReadAligner::start(const Config &c, std::string *err) {
    using clk = std::chrono::steady_clock;
    if (c.subject_files == c.query_files) {  // -q X -s X: the resident query set
        const auto t0 = clk::now();
        const bool r = ok(table->ctx, hero_align_self(table->ctx), "hero_align_self", err);
        seconds_aligning += std::chrono::duration<double>(clk::now() - t0).count();
        return r && (c.consensus || write_alignments(c, table->ctx, err));
    }
    SubjectDataset sd(c);
    ReadSet chunk;
    while (true) {
        const auto t0 = clk::now();
        if (!sd.next(chunk, err)) return false;
        seconds_loading += std::chrono::duration<double>(clk::now() - t0).count();
        if (chunk.n() == 0) break;
        const auto t1 = clk::now();
        if (!ok(table->ctx, hero_align_subjects(table->ctx,
                                                reinterpret_cast<const uint8_t *>(chunk.seq.data()),
                                                chunk.off.data(), chunk.uid.data(), chunk.n()),
                "hero_align_subjects", err))
            return false;
        if (!c.consensus && !write_alignments(c, table->ctx, err)) return false;
        seconds_aligning += std::chrono::duration<double>(clk::now() - t1).count();
    }
    return true;
}

bool call_consensus(HashTableGpu &t, QueryDataset &q, std::string *err) {
    const uint64_t n = q.reads.n();
    q.corrected.assign(q.reads.seq.size(), 0);
    q.imin.assign(n, 0);
    q.imed.assign(n, 0);
    q.imax.assign(n, 0);
    q.mismatch_rate.assign(n, 0);
    q.gc.assign(n, 0);
    return ok(t.ctx, hero_consensus(t.ctx, reinterpret_cast<uint8_t *>(&q.corrected[0]),
                                    q.imin.data(), q.imed.data(), q.imax.data(),
                                    q.mismatch_rate.data(), q.gc.data(), nullptr),
              "hero_consensus", err);
}

bool merge_pairs(HashTableGpu &t, QueryDataset &q, std::string *err) {
    q.merged.assign(q.reads.seq.size(), 0);
    q.merged_len.assign(q.reads.n() / 2, 0);
    return ok(t.ctx, hero_merge_pairs(t.ctx, reinterpret_cast<uint8_t *>(&q.merged[0]),
                                      q.merged_len.data()),
              "hero_merge_pairs", err);
}

}  // namespace herohost

namespace herohost {

bool write_mapping(HashTableGpu &t, const Config &c, std::string *err) {
    uint64_t n = 0;
    if (hero_mapping_histogram(t.ctx, nullptr, 0, &n) != HERO_OK) {
        *err = hero_last_error(t.ctx);
        return false;
    }
    std::vector<uint64_t> hist(n);
    if (n && hero_mapping_histogram(t.ctx, hist.data(), n, &n) != HERO_OK) {
        *err = hero_last_error(t.ctx);
        return false;
    }
    // QueryDataset.cpp:589-596: the output name as given, opened for appending
    std::FILE *f = std::fopen(c.out.c_str(), "ab");
    if (!f) {
        *err = "cannot open " + c.out;
        return false;
    }
    std::fputs("COV\tFRE\n", f);
    for (uint64_t i = 0; i < n; i++)
        if (hist[i]) std::fprintf(f, "%llu\t%llu\n", (unsigned long long)i, (unsigned long long)hist[i]);
    const bool ok = std::fclose(f) == 0;
    if (!ok) *err = "cannot write " + c.out;
    return ok;
}

}  // namespace herohost
