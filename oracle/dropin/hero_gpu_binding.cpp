// hero_gpu_binding.cpp -- HERO's classes over the hero-b200 C ABI (see the header).
#include "hero_gpu_binding.h"

#include <cstdlib>
#include <iostream>

HashTableGpu *HashTableGpu::current = NULL;

static void die(hero_ctx *ctx, const char *what) {
    std::cout << "hero-b200: " << what << ": " << (ctx ? hero_last_error(ctx) : "") << std::endl;
    std::exit(1);
}

// the reads as the ABI takes them: concatenated bases, n+1 offsets, atoi ids
struct Packed {
    std::vector<uint8_t> seq;
    std::vector<uint64_t> off;
    std::vector<int64_t> uid;
};

HashTableGpu::HashTableGpu(QueryDataset *q) : ctx(NULL) {
    dataSet = q;
    hashTableSize = 0;
    vviHashTable = NULL;
    iBitOfReadId = 0;
    iMask = 0;
    hashKeyLength = Config::iKmer;
    numberOfHashCollision = 0;
    maxSingleHashCollision = 0;
    current = this;
}

HashTableGpu::~HashTableGpu() {
    if (ctx) hero_destroy(ctx);
    if (current == this) current = NULL;
}

bool HashTableGpu::createHashTables() {
    hero_params p;
    hero_default_params(&p);
    p.k = int32_t(Config::iKmer);
    p.min_overlap = int32_t(Config::minimumOverlapLength);
    p.aligner = Config::iAlignerType == BandAligner::IAFFINE ? HERO_ALIGNER_AFFINE : HERO_ALIGNER_GLOBAL;
    p.max_mismatch_rate = Config::dMaxMismatchRate;
    p.max_indel_rate = Config::dMaxIndelRate;
    p.consensus_threshold = Config::dMinFrequencyCallConsensus;
    if (hero_create(&p, &ctx) != HERO_OK) die(ctx, "hero_create");
    return true;
}

bool HashTableGpu::insertQueryDataset(QueryDataset *q) {
    Packed r;
    r.off.push_back(0);
    const vector<QueryRead *> &reads = *q->vQueryReads;
    for (size_t i = 0; i < reads.size(); i++) {
        const string &s = reads[i]->sReadSequence;
        r.seq.insert(r.seq.end(), s.begin(), s.end());
        r.off.push_back(r.seq.size());
        r.uid.push_back(reads[i]->iReadUniqueId);
    }
    if (hero_set_queries(ctx, r.seq.empty() ? NULL : &r.seq[0], &r.off[0],
                         r.uid.empty() ? NULL : &r.uid[0], r.uid.size()) != HERO_OK)
        die(ctx, "hero_set_queries");
    if (hero_build_index(ctx) != HERO_OK) die(ctx, "hero_build_index");
    return true;
}

vector<INT64> *HashTableGpu::getListOfReads(const string &, INT64, INT64) { return NULL; }
UINT64 HashTableGpu::getPrimeLargerThanNumber(UINT64 number) { return number; }
UINT64 HashTableGpu::hashFunction(const string &) { return 0; }
UINT64 HashTableGpu::hashFunction(const string &, INT64, INT64) { return 0; }
bool HashTableGpu::insertQueryRead(QueryRead *, string, INT64) { return false; }
bool HashTableGpu::isEmptyAt(INT64) { return true; }
void HashTableGpu::setHashTableSizeAndInitialize(INT64) {}

void HashTableGpu::callConsensus(QueryDataset *q) {
    hero_ctx *ctx = current ? current->ctx : NULL;
    if (!ctx) die(NULL, "no device table for the consensus");
    const vector<QueryRead *> &reads = *q->vQueryReads;
    const size_t n = reads.size();
    std::vector<uint64_t> off(n + 1, 0);
    for (size_t i = 0; i < n; i++) off[i + 1] = off[i] + reads[i]->sReadSequence.size();
    std::vector<uint8_t> seq(off[n] ? off[n] : 1);
    std::vector<uint32_t> imin(n + 1), imed(n + 1), imax(n + 1);
    std::vector<double> mis(n + 1);
    if (hero_consensus(ctx, &seq[0], &imin[0], &imed[0], &imax[0], &mis[0], NULL, NULL) != HERO_OK)
        die(ctx, "hero_consensus");
    for (size_t i = 0; i < n; i++) {
        QueryRead *r = reads[i];
        r->sReadSequence.assign(reinterpret_cast<const char *>(&seq[0]) + off[i], off[i + 1] - off[i]);
        r->iMin = imin[i];
        r->iMed = imed[i];
        r->iMax = imax[i];
        r->dActualMismatchRate = mis[i];
    }
}

bool SubjectReadAlignerGpu::start() {
    HashTableGpu *table = static_cast<HashTableGpu *>(hashTable);
    SubjectDataset *subjects = new SubjectDataset();
    while (subjects->loadNextChunkParallel(Config::numberOfThreads)) {
        Packed r;
        r.off.push_back(0);
        for (UINT64 i = 0; i < subjects->iCountSubjectRead; i++) {
            const SubjectRead *s = subjects->vpSubjectRead->at(i);
            r.seq.insert(r.seq.end(), s->sReadSequence.begin(), s->sReadSequence.end());
            r.off.push_back(r.seq.size());
            r.uid.push_back(s->iReadUniqueId);
        }
        if (!r.uid.empty() &&
            hero_align_subjects(table->ctx, r.seq.empty() ? NULL : &r.seq[0], &r.off[0], &r.uid[0],
                                r.uid.size()) != HERO_OK)
            die(table->ctx, "hero_align_subjects");
    }
    delete subjects;
    return true;
}
