// host_parse.cpp -- TEST HARNESS ONLY.
//
// Runs the drop-in's read parser (herohost::load_reads, hero_b200/host/) on
// the files named on the command line, appending them into one read set as
// QueryDataset does with several query files, and prints the result for the
// test to compare: "ERR <message>" on a refusal, else one line per read
// "<id> <sequence>".
#include <cstdio>
#include <string>

#include "../../hero_b200/host/hero_host.h"

int main(int argc, char **argv) {
    herohost::ReadSet rs;
    std::string err;
    for (int i = 1; i < argc; i++) {
        if (!herohost::load_reads(argv[i], rs, &err)) {
            std::printf("ERR %s\n", err.c_str());
            return 0;
        }
    }
    for (uint64_t r = 0; r < rs.n(); r++) {
        std::printf("%lld ", static_cast<long long>(rs.uid[r]));
        std::fwrite(rs.seq.data() + rs.off[r], 1, rs.off[r + 1] - rs.off[r], stdout);
        std::printf("\n");
    }
    return 0;
}
