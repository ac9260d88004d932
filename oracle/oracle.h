/*
 * oracle.h -- CPU oracle of the YCSB transaction path. TEST INFRASTRUCTURE:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it; the engine never does.
 *
 * It restates, on the CPU and independently of the engine's sources:
 *   - the table fill, field-write and read-digest formulas of the engine;
 *   - serial execution of YCSB transactions with gCCTB's per-op semantics
 *     (benchmark/ycsb.cu:51-106: reads copy the row into the transaction's
 *     `item`, writes store into the row);
 *   - GaccO's serial order (ascending tx index within a batch,
 *     include/gacco.cuh:156-175) and GPUTx's rank order (src/gputx.cu:5-38,
 *     include/gputx.cuh:252-294);
 *   - a commit-log replay checker for the non-deterministic schemes;
 *   - a conflict-graph acyclicity check over (tx, row, read/write, seq)
 *     events, with the edge rules of src/runtime.cu:23-127;
 *   - multi-threaded CPU executors (2PL no-wait, Silo, TicToc on
 *     std::atomic words) used as the timed CPU baseline.
 *
 * Parity status: the reference ships no golden vectors, fixtures or
 * known-answer tests for this path (no test directory; datasets are
 * generated and git-ignored). Parity of these restatements is therefore
 * anchored on the reference's code (file:line above) and on the format
 * checks in tests/; it is "parity unpinned" in the sense that no
 * reference-produced output vector exists to compare against.
 */
#ifndef GCC_ORACLE_H
#define GCC_ORACLE_H
#include <stdint.h>
#include "../include/gcc_engine.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Table after initialisation, rows packed at gcc_row_bytes(layout). */
int oracle_fill_table(uint64_t rows, int32_t layout, uint64_t seed, uint8_t *out);

/* Serial replay of `order` (n_order tx ids) over `table` (packed rows,
 * modified in place). digests[tx] receives each replayed tx's read digest;
 * read_log (optional) receives row images at slot (tx*16+op) of `stride`
 * bytes. Returns 0 or GCC_EKEY / GCC_EFORMAT. */
int oracle_replay(uint8_t *table, uint64_t rows, int32_t layout, const gcc_ycsb_tx *txs,
                  uint64_t n_tx, const uint32_t *order, uint64_t n_order, int32_t write_mode,
                  uint64_t write_seed, uint64_t *digests, uint8_t *read_log);

/* The same serial replay for variable-length transactions: tx t owns
 * reqs[tx_off[t] .. tx_off[t+1]) (at most 64). */
int oracle_replay_var(uint8_t *table, uint64_t rows, int32_t layout, const uint32_t *tx_off,
                      const gcc_ycsb_req *reqs, uint64_t n_tx, const uint32_t *order,
                      uint64_t n_order, int32_t write_mode, uint64_t write_seed,
                      uint64_t *digests);

/* The same with extended ops (gcc_engine.h GCC_OP_*) when ext_ops != 0:
 * requests with a negative `read` word apply their integer read-modify-write
 * or insert, read-modify-writes adding the row image they read to the
 * digest. */
int oracle_replay_var_ext(uint8_t *table, uint64_t rows, int32_t layout, const uint32_t *tx_off,
                          const gcc_ycsb_req *reqs, uint64_t n_tx, const uint32_t *order,
                          uint64_t n_order, int32_t write_mode, uint64_t write_seed,
                          uint64_t *digests, int32_t ext_ops);

/* GPUTx execution order: ranks per tx (reference rank function), and the
 * txs sorted by (rank, tx). */
int oracle_gputx_order(const gcc_ycsb_tx *txs, uint64_t n_tx, uint64_t rows, uint32_t *ranks,
                       uint32_t *order, uint32_t *max_rank);

/* Order txs by their commit records (hi, lo, tx). */
int oracle_commit_order(const gcc_commit_rec *log, uint64_t n_tx, uint32_t *order);

/* Conflict graph over events {tx, row, is_write, seq} sorted by seq:
 * returns 1 if acyclic (serializable), 0 if a cycle exists. */
typedef struct oracle_event {
    uint32_t tx;
    uint32_t row;
    uint32_t is_write;
    uint32_t pad;
    uint64_t seq;
} oracle_event;
int oracle_conflict_acyclic(const oracle_event *ev, uint64_t n_ev, uint64_t n_tx);

/* Multi-threaded CPU execution (baseline). scheme: "tpl_nw", "silo",
 * "tictoc". The table is modified in place, digests/commit log filled.
 * Returns 0 or an error; seconds/aborts report the run. */
int oracle_cpu_run(const char *scheme, uint8_t *table, uint64_t rows, int32_t layout,
                   const gcc_ycsb_tx *txs, uint64_t n_tx, int32_t write_mode,
                   uint64_t write_seed, int32_t threads, uint64_t *digests,
                   gcc_commit_rec *commit_log, double *seconds, uint64_t *aborts);

/* The same executors over variable-length transactions (CSR, at most 64
 * requests), with extended ops (ext_ops != 0) applied under the
 * transaction's exclusive access like the engine does. */
int oracle_cpu_run_var(const char *scheme, uint8_t *table, uint64_t rows, int32_t layout,
                       const uint32_t *tx_off, const gcc_ycsb_req *reqs, uint64_t n_tx,
                       int32_t write_mode, uint64_t write_seed, int32_t ext_ops, int32_t threads,
                       uint64_t *digests, gcc_commit_rec *commit_log, double *seconds,
                       uint64_t *aborts);

/* Independent restatement of the dataset generator (gen_ycsb semantics). */
int oracle_gen_ycsb(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                    uint64_t seed, int32_t dedup, int32_t key_base, gcc_ycsb_tx *out);

#ifdef __cplusplus
}
#endif
#endif
