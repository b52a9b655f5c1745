// main.cpp -- drop-in replacement of HERO's driver (main.cpp:26-106 of the
// reference): same flags, same sequence, same .fasta/.info output with -c and
// the same .aln output without it.
#include <chrono>
#include <iostream>
#include <thread>

#include "hero_host.h"

using namespace herohost;

int main(int argc, char **argv) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto sec_since = [](clk::time_point a) {
        return std::chrono::duration<double>(clk::now() - a).count();
    };
    Config cfg;
    if (!cfg.parse(argc, argv)) {
        std::cout << "Please follow the above help information." << std::endl;
        return 1;
    }
    // the device's CUDA context is created while the queries are parsed
    struct Joined {
        std::thread t;
        ~Joined() {
            if (t.joinable()) t.join();
        }
    } device_init{std::thread([&cfg] { hero_device_init(cfg.device); })};
    std::string err;
    QueryDataset query;
    if (!query.build(cfg, &err)) {
        std::cerr << "Error: cannot build query dataset: " << err << std::endl;
        return 1;
    }
    if (query.reads.n() == 0) {
        std::cout << "Unfortunately all the query data are filtered out. " << std::endl
                  << "Further processing is aborted. " << std::endl;
        return 1;
    }
    device_init.t.join();
    const auto t1 = clk::now();
    HashTableGpu table;
    if (!table.createHashTables(cfg, &query, &err) || !table.insertQueryDataset(&err)) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    const auto t2 = clk::now();
    SubjectReadAligner aligner(&table);
    if (!aligner.start(cfg, &err)) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    const auto t3 = clk::now();
    if (cfg.consensus && cfg.mapping) {  // main.cpp:83-87: the histogram instead of reads
        if (!write_mapping(table, cfg, &err)) {
            std::cerr << "Error: " << err << std::endl;
            return 1;
        }
        std::cout << sec_since(t0) << " seconds (Total time used)" << std::endl;
        return 0;
    }
    if (cfg.consensus && !call_consensus(table, query, &err)) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    if (cfg.consensus && cfg.merge && !merge_pairs(table, query, &err)) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    const auto t4 = clk::now();
    if (cfg.consensus && !query.write(cfg, &err)) {
        std::cerr << "Error: " << err << std::endl;
        return 1;
    }
    const auto t5 = clk::now();
    auto sec = [](clk::time_point a, clk::time_point b) {
        return std::chrono::duration<double>(b - a).count();
    };
    hero_stats st;
    hero_get_stats(table.ctx, &st);
    std::cout << sec(t0, t1) << " seconds (Time for loading queries)" << std::endl
              << sec(t1, t2) << " seconds (Time for upload and k-mer table)" << std::endl
              << aligner.seconds_loading << " seconds (Time for loading subjects)" << std::endl
              << sec(t2, t3) << " seconds (Time for seeding, aligning and voting)" << std::endl
              << sec(t3, t4) << " seconds (Time for calling consensus)" << std::endl
              << sec(t4, t5) << " seconds (Time for writing results)" << std::endl
              << sec(t0, t5) << " seconds (Total time used)" << std::endl
              << st.dp_cells << " band cells, " << st.records_kept << " records" << std::endl;
    return 0;
}
