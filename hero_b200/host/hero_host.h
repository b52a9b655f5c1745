// hero_host.h -- host side of the drop-in: HERO's driver classes over the C ABI.
//
// The classes keep the reference's names and roles (Config, QueryDataset,
// SubjectDataset, HashTableMethod/HashTableGpu, SubjectReadAligner) so the
// program reads like main.cpp; the work they hand to OpenMP in the reference
// goes to the device through include/hero_gpu.h.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "hero_gpu.h"

namespace herohost {

// Config::setConfig flags (Config.cpp:118-243) of the consensus path.
struct Config {
    std::vector<std::string> subject_files, query_files;
    std::string out = "query";
    int32_t k = 39, min_overlap = 40, threads = 1;
    double mis_rate = 1.0, indel_rate = 1.0, consensus_thr = 0.6;
    bool affine = false, consensus = false, covinfo = false, single_reads = false;
    bool merge = false;  // --merge: paired reads (2i, 2i+1) merged after the consensus
    bool mapping = false;  // --mapping: chosen records vote; the coverage histogram is written
    uint64_t stream_chunk = 400, query_chunk = 800;
    int device = 0;
    uint32_t subject_batch = 0;
    // returns false (after printing the reason) for bad or unsupported flags
    bool parse(int argc, char **argv);
    static void help();
};

// A read set as HERO holds it after loading: uppercase bases, atoi ids.
struct ReadSet {
    std::string seq;                 // concatenated bases
    std::vector<uint64_t> off{0};    // n+1 offsets
    std::vector<int64_t> uid;        // atoi(read name)
    uint64_t n() const { return uid.size(); }
};

// QueryDataset::loadDatasetParallel (QueryDataset.cpp:103-391) for well-formed
// FASTA/FASTQ; appends to `out`.  Returns false if a file cannot be read.
bool load_reads(const std::string &path, ReadSet &out, std::string *err);

class QueryDataset {
   public:
    ReadSet reads;
    // consensus results (QueryRead fields)
    std::string corrected;
    std::vector<uint32_t> imin, imed, imax;
    std::vector<double> mismatch_rate, gc;
    // --merge: per pair the merged read (from the pair's first base) and its length
    std::string merged;
    std::vector<uint32_t> merged_len;
    bool build(const Config &c, std::string *err);
    // QueryDataset::writeQueryOut (QueryDataset.cpp:414-537): append mode
    bool write(const Config &c, std::string *err) const;
};

// Streams subject reads in chunks (SubjectDataset::loadNextChunkParallel,
// SubjectDataset.cpp:45-179): whole files are read, then handed out in chunks.
class SubjectDataset {
   public:
    explicit SubjectDataset(const Config &c) : cfg(c) {}
    bool next(ReadSet &chunk, std::string *err);
   private:
    const Config &cfg;
    size_t file = 0;
    ReadSet cur;
    uint64_t pos = 0;
    bool loaded = false;
};

// HashTableMethod (HashTableMethod.h:13-40) backed by the device table.
class HashTableGpu {
   public:
    hero_ctx *ctx = nullptr;
    QueryDataset *dataSet = nullptr;
    bool createHashTables(const Config &c, QueryDataset *q, std::string *err);
    bool insertQueryDataset(std::string *err);
    ~HashTableGpu();
};

// SubjectReadAligner::start (SubjectReadAligner.cpp:493-645)
class SubjectReadAligner {
   public:
    explicit SubjectReadAligner(HashTableGpu *t) : table(t) {}
    bool start(const Config &c, std::string *err);
    double seconds_loading = 0, seconds_aligning = 0;
   private:
    HashTableGpu *table;
};

// QueryDataset::callConsensus (QueryDataset.cpp:393-412) on the device
bool call_consensus(HashTableGpu &t, QueryDataset &q, std::string *err);

// QueryDataset::mergePairedReads (QueryDataset.cpp:539-558) on the device (--merge)
bool merge_pairs(HashTableGpu &t, QueryDataset &q, std::string *err);

// QueryDataset::getCoverageAndWriteResults (QueryDataset.cpp:560-599): the
// coverage histogram of the votes, appended to the output name (--mapping)
bool write_mapping(HashTableGpu &t, const Config &c, std::string *err);

}  // namespace herohost
