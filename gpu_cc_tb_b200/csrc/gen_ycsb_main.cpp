// gen_ycsb -- drop-in for gCCTB's dataset generator (generation/gen_ycsb.cu:34-58).
//
//   gen_ycsb <ycsb_rownum> <ycsb_txcnt> <theta> <r_ratio> <path_to_dataset> [key=value ...]
//
// Writes a headerless array of 136-byte YCSBTx records. Defaults reproduce
// the reference's rules (up to 16 requests, repeated keys dropped, keys in
// [1, rownum-1], sorted by key); options: seed=N (default 141919810, the
// reference's SEED), dedup=drop|resample, key_base=0|1, threads=N.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/gcc_engine.h"

int main(int argc, char **argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s <ycsb_rownum> <ycsb_txcnt> <theta> <r_ratio> <path> [key=value ...]\n",
                     argv[0]);
        return 2;
    }
    int rownum = 0, txcnt = 0;
    float theta = 0.6f, rr = 0.9f;
    std::sscanf(argv[1], "%d", &rownum);
    std::sscanf(argv[2], "%d", &txcnt);
    std::sscanf(argv[3], "%f", &theta);
    std::sscanf(argv[4], "%f", &rr);
    uint64_t seed = 141919810;
    int dedup = GCC_DEDUP_DROP, key_base = 1, threads = 0;
    for (int i = 6; i < argc; ++i) {
        std::string kv(argv[i]);
        size_t eq = kv.find('=');
        if (eq == std::string::npos) continue;
        std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
        if (k == "seed") seed = std::strtoull(v.c_str(), nullptr, 10);
        else if (k == "dedup") dedup = v == "resample" ? GCC_DEDUP_RESAMPLE : GCC_DEDUP_DROP;
        else if (k == "key_base") key_base = std::atoi(v.c_str());
        else if (k == "threads") threads = std::atoi(v.c_str());
    }
    std::vector<gcc_ycsb_tx> txs((size_t)txcnt);
    // theta and r_ratio are parsed as float, like the reference (gen_ycsb.cu:39-40)
    int rc = gcc_gen_ycsb((uint64_t)rownum, (uint64_t)txcnt, (double)theta, (double)rr, seed, dedup,
                          key_base, threads, txs.data());
    if (rc) {
        std::fprintf(stderr, "gcc_gen_ycsb: %s (%d)\n", gcc_strerror(rc), rc);
        return 1;
    }
    std::cout << "GEN OK\n";
    FILE *f = std::fopen(argv[5], "wb");
    if (!f) { std::perror(argv[5]); return 1; }
    std::fwrite(txs.data(), sizeof(gcc_ycsb_tx), txs.size(), f);
    std::fclose(f);
    return 0;
}
