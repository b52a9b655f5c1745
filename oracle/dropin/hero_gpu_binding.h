// hero_gpu_binding.h -- the drop-in binding a HERO maintainer adds: HERO's own
// classes (HashTableMethod, SubjectReadAligner, QueryDataset) served by the
// hero-b200 C ABI (include/hero_gpu.h).  Compiled into HERO itself by
// oracle/dropin/make_dropin.py (test infrastructure: it proves that the library
// drops into the unmodified reference program, beside main.cpp's three changed
// lines).  Written in the reference's C++ dialect (gnu++98).
#ifndef HERO_GPU_BINDING_H_
#define HERO_GPU_BINDING_H_

#include "HashTableMethod.h"
#include "QueryDataset.h"
#include "SubjectReadAligner.h"
#include "hero_gpu.h"

// HashTableMethod (HashTableMethod.h:13-40) backed by the device k-mer table.
// createHashTables/insertQueryDataset upload the query reads and build the
// table on the device; the host-side lookups of the interface are not used by
// the GPU aligner and answer "no list".
class HashTableGpu : public HashTableMethod {
   public:
    hero_ctx *ctx;
    explicit HashTableGpu(QueryDataset *q);
    ~HashTableGpu();
    bool createHashTables();
    bool insertQueryDataset(QueryDataset *q);
    vector<INT64> *getListOfReads(const string &sequence, INT64 start, INT64 length);
    UINT64 getPrimeLargerThanNumber(UINT64 number);
    UINT64 hashFunction(const string &subString);
    UINT64 hashFunction(const string &sequence, INT64 start, INT64 length);
    bool insertQueryRead(QueryRead *read, string subString, INT64 position);
    bool isEmptyAt(INT64 index);
    void setHashTableSizeAndInitialize(INT64 size);
    // QueryDataset::callConsensus (QueryDataset.cpp:393-412) through the ABI:
    // corrected bases and statistics back into the QueryReads
    static void callConsensus(QueryDataset *q);
    static HashTableGpu *current;  // the table the consensus reads the votes of
};

// SubjectReadAligner::start (SubjectReadAligner.cpp:493-645) through the ABI:
// the same SubjectDataset chunks, each aligned on the device and voted into the
// table's query set.
class SubjectReadAlignerGpu : public SubjectReadAligner {
   public:
    explicit SubjectReadAlignerGpu(HashTableMethod *table) : SubjectReadAligner(table) {}
    bool start();
};

#endif
