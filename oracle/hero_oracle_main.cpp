/*
 * hero_oracle_main.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Command-line front end of the CPU restatement: reads the same FASTA/FASTQ
 * files and the consensus-mode flags of the reference (Config::setConfig,
 * Config.cpp:118-243) and writes the same <out>.fasta / <out>.info
 * (QueryDataset::writeQueryOut, QueryDataset.cpp:414-537, --singleReads form).
 * Used only to pin the restatement against oracle/_ref/hero_ref.
 */
#include "hero_oracle.h"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

struct Set {
    std::string seq;
    std::vector<uint64_t> off{0};
    std::vector<int64_t> uid;
};

// Record reading for well-formed files, as QueryDataset::loadDatasetParallel
// (QueryDataset.cpp:103-244): FASTQ = 4 lines per read; FASTA = header line,
// then everything up to the next '>' with newlines removed.
static bool readSet(const std::string &path, Set &out) {
    std::ifstream f(path.c_str());
    if (!f.is_open()) return false;
    std::string first;
    std::getline(f, first);
    f.seekg(0, std::ios::beg);
    bool fasta = !first.empty() && first[0] == '>';
    std::string l0, l1, l2, l3;
    while (true) {
        if (fasta) {
            if (!std::getline(f, l0)) break;
            std::getline(f, l1, '>');
            std::string t;
            for (char c : l1)
                if (c != '\n') t.push_back(c);
            l1.swap(t);
            if (l0.empty() && l1.empty()) break;
        } else {
            if (!std::getline(f, l0)) break;
            if (!std::getline(f, l1)) break;
            std::getline(f, l2);
            std::getline(f, l3);
        }
        std::string name = (!l0.empty() && (l0[0] == '>' || l0[0] == '@')) ? l0.substr(1) : l0;
        for (char &c : l1) c = char(std::toupper(static_cast<unsigned char>(c)));
        out.uid.push_back(int64_t(std::atoi(name.c_str())));
        out.seq += l1;
        out.off.push_back(out.seq.size());
    }
    return true;
}

int main(int argc, char **argv) {
    std::string q, s, o = "query";
    hero_oracle_params p{39, 40, 0, 0, 1.0, 1.0, 0.6};
    int threads = 1;
    bool covinfo = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() { return std::string(i + 1 < argc ? argv[++i] : ""); };
        if (a == "-q" || a == "--query") q = next();
        else if (a == "-s" || a == "--subject") s = next();
        else if (a == "-o" || a == "--out") o = next();
        else if (a == "-k") p.k = std::atoi(next().c_str());
        else if (a == "-l") p.min_overlap = std::atoi(next().c_str());
        else if (a == "-m") p.mis_rate = std::atof(next().c_str()) / 100.0;
        else if (a == "-i") p.indel_rate = std::atof(next().c_str()) / 100.0;
        else if (a == "-t") threads = std::atoi(next().c_str());
        else if (a == "-a") p.affine = next() == "a" ? 1 : 0;
        else if (a == "-c") {
            if (i + 1 < argc && argv[i + 1][0] >= '0' && argv[i + 1][0] <= '9')
                p.consensus_thr = std::atof(argv[++i]);
        } else if (a == "--covinfo") covinfo = true;
        else if (a == "--singleReads") {
        } else if (a == "-z" || a == "-y") next();
        else {
            std::cerr << "unknown flag " << a << "\n";
            return 2;
        }
    }
    Set Q, S;
    if (!readSet(q, Q) || !readSet(s, S)) {
        std::cerr << "cannot read input\n";
        return 1;
    }
    uint64_t nq = Q.uid.size(), ns = S.uid.size();
    hero_oracle_run *r = hero_oracle_correct(
        &p, threads, nq, reinterpret_cast<const uint8_t *>(Q.seq.data()), Q.off.data(),
        Q.uid.data(), ns, reinterpret_cast<const uint8_t *>(S.seq.data()), S.off.data(),
        S.uid.data());
    if (!r) return 1;
    std::vector<uint8_t> out(Q.seq.size());
    std::vector<uint32_t> imin(nq), imed(nq), imax(nq);
    std::vector<double> mis(nq), gc(nq);
    hero_oracle_consensus(r, out.data(), imin.data(), imed.data(), imax.data(), mis.data(),
                          gc.data(), nullptr);
    {
        std::ofstream fa((o + ".fasta").c_str());
        for (uint64_t i = 0; i < nq; i++) {
            fa << ">" << Q.uid[i] << std::endl;
            fa.write(reinterpret_cast<const char *>(out.data() + Q.off[i]),
                     std::streamsize(Q.off[i + 1] - Q.off[i]));
            fa << std::endl;
        }
    }
    if (covinfo) {
        std::ofstream fi((o + ".info").c_str());
        for (uint64_t i = 0; i < nq; i++) {
            fi << Q.uid[i] << "\t" << imin[i] << "\t" << imed[i] << "\t" << imax[i] << "\t"
               << (Q.off[i + 1] - Q.off[i]) << "\t" << mis[i] << "\t" << gc[i] << std::endl;
        }
    }
    hero_oracle_stats st;
    hero_oracle_stats_get(r, &st);
    std::cout << "probes " << st.probes << " hits " << st.hits << " chains " << st.chains
              << " kept " << st.chains_kept << " built " << st.records_built << " accepted "
              << st.records_accepted << " records " << st.records_kept << " segments "
              << st.dp_segments << " cells " << st.dp_cells << std::endl;
    hero_oracle_free(r);
    return 0;
}
