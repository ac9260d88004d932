// test_ycsb -- drop-in for gCCTB's benchmark driver (benchmark_cpu/ycsb.cu:81-302)
// over the engine's C ABI.
//
//   test_ycsb <dataset> <ycsb_rownum> <ycsb_txcnt> <cc_scheme> <warp_density>
//             <block_size> <batch_size> <debug_flag> [key=value ...]
//
// Positional arguments and their checks follow the reference
// (benchmark_cpu/ycsb.cu:89-98: warp_density > 5 or block_size > 32 exits
// with -1). It prints the reference's "TRY" line and result block and
// appends the 15-column CSV line to <dataset>.txt (include/runtime.cuh:
// 180-213). Options beyond the reference (defaults reproduce its setup):
//   layout=ref104|u64x11   row format (default ref104: 104-byte Item rows)
//   index=sorted|hash|direct  key -> row index (default sorted)
//   write=rowcopy|field    write semantics (default rowcopy)
//   fill_seed=N            row fields from seed N (default 0: zero fields)
//   device=N  spin_ms=N  backoff_ns=N
// Result files (headerless little-endian arrays, for parity tooling):
//   table_out=PATH       final rows, packed (104 or 88 bytes each)
//   digests_out=PATH     u64 read digest per transaction
//   commit_log_out=PATH  {u64 hi, u64 lo} serialization key per transaction
//   aborts_out=PATH      u32 aborted attempts per transaction
//   read_log_out=PATH    every read row image, txcnt x 16 slots of 112 / 96 B
// debug_flag=1 additionally re-executes the committed transactions in their
// recorded serialization order on the GPU and compares final table and read
// digests: prints GOOD or BAD (the reference's debug check prints GOOD/BAD
// after a conflict-graph cycle search, src/runtime.cu:129-158).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/gcc_engine.h"

static int die(const char *what, int rc) {
    std::fprintf(stderr, "%s: %s (%d)\n", what, gcc_strerror(rc), rc);
    return 1;
}

int main(int argc, char **argv) {
    if (argc < 9) {
        std::fprintf(stderr,
                     "usage: %s <dataset> <ycsb_rownum> <ycsb_txcnt> <cc_scheme> "
                     "<warp_density> <block_size> <batch_size> <debug_flag> [key=value ...]\n",
                     argv[0]);
        return 2;
    }
    int rownum = 0, txcnt = 0, wd = 0, bs = 0, batch = 0, debug = 0;
    std::sscanf(argv[2], "%d", &rownum);
    std::sscanf(argv[3], "%d", &txcnt);
    std::string cc_type(argv[4]);
    std::sscanf(argv[5], "%d", &wd);
    std::sscanf(argv[6], "%d", &bs);
    std::sscanf(argv[7], "%d", &batch);
    std::sscanf(argv[8], "%d", &debug);
    if (bs > 32 || wd > 5) return -1;

    gcc_table_desc desc{};
    desc.rows = (uint64_t)rownum;
    desc.layout = GCC_LAYOUT_REF104;
    desc.index_kind = GCC_INDEX_SORTED;
    desc.fill_seed = 0;
    desc.device = 0;
    desc.max_batch = batch;
    gcc_run_params rp{};
    rp.cc_scheme = argv[4];
    rp.warp_density = wd;
    rp.block_size = bs;
    rp.batch_size = batch;
    rp.write_mode = GCC_WRITE_ROWCOPY;
    rp.write_seed = 1;
    std::string table_out, digests_out, commit_out, aborts_out, readlog_out;
    for (int i = 9; i < argc; ++i) {
        std::string kv(argv[i]);
        size_t eq = kv.find('=');
        if (eq == std::string::npos) continue;
        std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
        if (k == "layout") desc.layout = v == "u64x11" ? GCC_LAYOUT_U64X11 : GCC_LAYOUT_REF104;
        else if (k == "index") desc.index_kind = v == "hash" ? GCC_INDEX_HASH : v == "direct" ? GCC_INDEX_DIRECT : GCC_INDEX_SORTED;
        else if (k == "write") rp.write_mode = v == "field" ? GCC_WRITE_FIELD : GCC_WRITE_ROWCOPY;
        else if (k == "fill_seed") desc.fill_seed = std::strtoull(v.c_str(), nullptr, 10);
        else if (k == "device") desc.device = std::atoi(v.c_str());
        else if (k == "spin_ms") rp.spin_limit_ns = std::strtoull(v.c_str(), nullptr, 10) * 1000000ull;
        else if (k == "backoff_ns") rp.backoff_ns = std::atoi(v.c_str());
        else if (k == "table_out") table_out = v;
        else if (k == "digests_out") digests_out = v;
        else if (k == "commit_log_out") commit_out = v;
        else if (k == "aborts_out") aborts_out = v;
        else if (k == "read_log_out") readlog_out = v;
    }
    if (!commit_out.empty()) rp.flags |= GCC_F_COMMIT_LOG;
    if (!readlog_out.empty()) rp.flags |= GCC_F_READ_LOG;
    std::cout << "TRY " << argv[4] << "," << wd << "," << bs << "," << batch << "\n";

    std::vector<gcc_ycsb_tx> txs((size_t)txcnt);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) { std::perror(argv[1]); return 1; }
    size_t got = std::fread(txs.data(), sizeof(gcc_ycsb_tx), (size_t)txcnt, f);
    std::fclose(f);
    if (got != (size_t)txcnt) {
        std::fprintf(stderr, "%s: %zu of %d records\n", argv[1], got, txcnt);
        return 1;
    }
    gcc_engine *e = nullptr;
    int rc = gcc_create(&desc, &e);
    if (rc) return die("gcc_create", rc);
    if ((rc = gcc_load_txs(e, txs.data(), txs.size()))) return die("gcc_load_txs", rc);
    gcc_result r{};
    if (debug) rp.flags |= GCC_F_COMMIT_LOG;
    int verdict = -1;
    if (debug) rc = gcc_run_checked(e, &rp, &r, &verdict);
    else rc = gcc_run(e, &rp, &r);
    if (rc) {
        gcc_destroy(e);
        return die("gcc_run", rc);
    }
    char line[512];
    gcc_format_line(&rp, &r, line, sizeof line);
    std::ofstream of(std::string(argv[1]) + ".txt", std::ios::out | std::ios::app);
    of << line << "\n";
    of.close();
    std::cout << cc_type << ",\n"
              << "valid_txn_bitoffset " << wd << ",\n"
              << "warp_cnt " << bs << ",\n"
              << "batch_size " << batch << ",\n"
              << "through " << (float)r.tx_per_s << ",\n"
              << "abort " << r.aborts << " avr " << (double)r.aborts / batch << ",\n"
              << "ts_d " << (float)r.ts_d << ",\n"
              << "wait_d " << (float)r.wait_d << ",\n"
              << "abort_d " << (float)r.abort_d << ",\n"
              << "mng_d " << (float)r.mng_d << ",\n"
              << "tot_d " << (float)r.tot_d << ",\n"
              << "idx_d " << (float)r.idx_d << ",\n"
              << "pre " << (float)r.pre_s << ",\n"
              << "proc " << (float)r.proc_s << ",\n"
              << "tot " << (float)r.tot_s << "\n";
    if (debug) std::cout << (verdict == 1 ? "GOOD" : "BAD") << "\n";
    // result files
    auto write_file = [&](const std::string &path, const void *data, size_t bytes) -> bool {
        FILE *o = std::fopen(path.c_str(), "wb");
        if (!o) { std::perror(path.c_str()); return false; }
        const bool ok = std::fwrite(data, 1, bytes, o) == bytes;
        std::fclose(o);
        return ok;
    };
    const uint64_t n = (uint64_t)txcnt;
    bool files_ok = true;
    if (!table_out.empty()) {
        std::vector<uint8_t> t((size_t)rownum * gcc_row_bytes(desc.layout));
        if ((rc = gcc_dump_table(e, t.data(), t.size()))) { gcc_destroy(e); return die("gcc_dump_table", rc); }
        files_ok &= write_file(table_out, t.data(), t.size());
    }
    if (!digests_out.empty()) {
        std::vector<uint64_t> d(n);
        if ((rc = gcc_get_digests(e, d.data(), n))) { gcc_destroy(e); return die("gcc_get_digests", rc); }
        files_ok &= write_file(digests_out, d.data(), d.size() * 8);
    }
    if (!commit_out.empty()) {
        std::vector<gcc_commit_rec> c(n);
        if ((rc = gcc_get_commit_log(e, c.data(), n))) { gcc_destroy(e); return die("gcc_get_commit_log", rc); }
        files_ok &= write_file(commit_out, c.data(), c.size() * sizeof(gcc_commit_rec));
    }
    if (!aborts_out.empty()) {
        std::vector<uint32_t> a(n);
        if ((rc = gcc_get_tx_aborts(e, a.data(), n))) { gcc_destroy(e); return die("gcc_get_tx_aborts", rc); }
        files_ok &= write_file(aborts_out, a.data(), a.size() * 4);
    }
    if (!readlog_out.empty()) {
        std::vector<uint8_t> l((size_t)n * 16 * gcc_row_stride(desc.layout));
        if ((rc = gcc_get_read_log(e, l.data(), l.size()))) { gcc_destroy(e); return die("gcc_get_read_log", rc); }
        files_ok &= write_file(readlog_out, l.data(), l.size());
    }
    gcc_destroy(e);
    return files_ok ? 0 : 1;
}
