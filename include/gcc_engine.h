/*
 * gcc_engine.h -- C ABI of the B200 transaction-execution engine.
 *
 * The engine executes YCSB transactions on one GPU under the concurrency
 * control (CC) schemes of the gCCTB testbed. Every entry point below takes
 * plain pointers and sizes and returns a status code (0 = ok, < 0 = error);
 * nothing calls exit() and every device-side wait is bounded.
 *
 * Reference interfaces replaced (paths inside the gCCTB project):
 *   - host driver `test_ycsb` main loop          benchmark_cpu/ycsb.cu:81-302
 *   - CC host base class (Init0/Init/ToGPU/Sync)  include/cc.cuh:18-56
 *   - device CC duck type (TxStart/Read/Write/TxEnd/Finalize)
 *                                                  include/cc.cuh:58-88
 *   - transaction kernel `ycsb`                   benchmark/ycsb.cu:21-111
 *   - row table + sorted index (Table_CPU::InitData/AddIndex/ToGPU,
 *     SortedArray_GPU::Find)                       include/table.cuh:61-130,
 *                                                  include/index.cuh:65-127
 *   - dataset generator `gen_ycsb`                 generation/gen_ycsb.cu:34-152
 *   - metrics report ExecInfo::Analyse            include/runtime.cuh:169-214
 *   - serializability check ExecInfo::Check       src/runtime.cu:129-158
 *
 * Threading: one engine is used by one host thread at a time. Separate
 * engines (on the same or different GPUs) are independent.
 */
#ifndef GCC_ENGINE_H
#define GCC_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GCC_OK 0
#define GCC_EINVAL (-1)    /* bad argument: unknown scheme, knob out of range */
#define GCC_ENOMEM (-2)    /* device or host allocation failed */
#define GCC_ECUDA (-3)     /* a CUDA runtime call failed */
#define GCC_ETIMEOUT (-4)  /* a bounded device-side wait ran out */
#define GCC_EFORMAT (-5)   /* malformed transaction record */
#define GCC_EKEY (-6)      /* a request key is not in the index */
#define GCC_EOVERFLOW (-7) /* timestamp space of a scheme exhausted */
#define GCC_ESTATE (-8)    /* call out of order (e.g. run before load) */
#define GCC_ENODEV (-9)    /* no CUDA device / wrong architecture */

/* ---- table layouts ----------------------------------------------------- */
/* 88-byte rows: uint64 key + 10 uint64 fields, stored at a 96-byte stride. */
#define GCC_LAYOUT_U64X11 0
/* 104-byte rows of gCCTB's `Item` (uint32 id + 10 x char[10],
 * include/ycsb.cuh:6-19), stored at a 112-byte stride. */
#define GCC_LAYOUT_REF104 1

/* ---- key -> row indexes ------------------------------------------------ */
#define GCC_INDEX_HASH 0   /* open addressing, one 32-byte bucket per probe */
#define GCC_INDEX_SORTED 1 /* sorted (key,row) array + binary search, the
                              reference's SortedArray_GPU (index.cuh:65-92) */
#define GCC_INDEX_DIRECT 2 /* key == row id */

/* ---- write semantics --------------------------------------------------- */
/* A write stores a fresh uint64 into one field; field and value are a pure
 * function of (write_seed, transaction id, op index). */
#define GCC_WRITE_FIELD 0
/* A write copies the transaction-local row buffer (the last row this
 * transaction read before the write in program order, zeros if none) over
 * the whole target row: gCCTB's `cc.Write(idx, w_idx, &item, row, sizeof
 * (Item))` (benchmark/ycsb.cu:84-97). */
#define GCC_WRITE_ROWCOPY 1

/* ---- run flags --------------------------------------------------------- */
#define GCC_F_COMMIT_LOG 1u /* record each tx's serialization key */
#define GCC_F_READ_LOG 2u   /* record every read row image (parity runs) */
#define GCC_F_NO_RESET 4u   /* keep CC metadata across batches where the
                               scheme allows it (tpl, silo, tictoc) */
#define GCC_F_RETRY_IMMEDIATE 8u /* retry an aborted transaction at once
                               instead of first waiting (up to 50 us) until
                               the row that made it abort looks free */
#define GCC_F_REQUEST_ORDER 256u /* tpl_nw, tpl_wd and to: retries that
                               visit their requests one at a time do so in
                               request order (the reference's order,
                               benchmark/ycsb.cu:60-98). Without it they take
                               every other request at once and the one that
                               failed in the previous attempt last, so that
                               contended row is locked (2PL) or held
                               uncommitted (TO) the shortest time; a starving
                               TO transaction (see starve_limit) and the
                               latch variants always go in request order.
                               Either way the same requests under the same
                               rule; only the order differs. */
#define GCC_F_EXT_OPS 64u   /* requests with a negative `read` word are
                               extended ops (GCC_OP_*); without this flag
                               every request with read <= 0 is a YCSB write */
#define GCC_F_QUEUE 128u    /* gcc_run / gcc_run_host: the batches go through
                               ONE persistent launch that takes positions in
                               batch order from a device queue, instead of one
                               launch per batch with a barrier between
                               batches (the reference's loop, benchmark_cpu/
                               ycsb.cu:262-285), so batch b+1's first
                               transactions fill the SMs that batch b's retry
                               tail leaves idle. gcc_run admits every batch at
                               once; gcc_run_host admits batch b when its
                               records have reached the device. The CC
                               metadata and the timestamp counter are reset
                               once per run, not per batch. Schemes whose
                               metadata stays valid across batches: tpl_nw,
                               tpl_wd, to, silo, tictoc and their slow_
                               variants; GCC_WRITE_FIELD only. */

/* ---- extended request ops ------------------------------------------------
 * A request whose `read` word is negative is an integer write op on the u64
 * key + 10 field layout (no counterpart in the reference's YCSB records,
 * whose `read` is 0 or 1): bits 28-30 opcode, 24-27 field f (0-9), 0-23
 * parameter v; write with GCC_OP_WORD. Read-modify-write ops return the row
 * they read in the transaction's digest, like a read; an insert does not.
 *   ADD    field f += v
 *   SUB    field f -= v (two's complement)
 *   STOCK  q = v & 0xFF, remote = v >> 8 & 1: field f = f >= q + 10 ? f - q
 *          : f - q + 91; f+1 += q; f+2 += 1; f+3 += remote   (f <= 6)
 *   PAY    field f -= v; f+1 += v; f+2 += 1                   (f <= 7)
 *   INSERT field 0 = transaction id, field 1 = v, fields 2-9 = a hash of
 *          (write_seed, transaction id, op index)
 * Enabled per run by GCC_F_EXT_OPS on variable-length transactions
 * (gcc_load_var_txs + gcc_run_batches / gcc_serve). Schemes: tpl_nw, tpl_wd,
 * to, silo, tictoc; layout GCC_LAYOUT_U64X11, write mode GCC_WRITE_FIELD. A
 * malformed op word ends the run with GCC_EFORMAT. */
#define GCC_OP_ADD 1
#define GCC_OP_SUB 2
#define GCC_OP_STOCK 3
#define GCC_OP_PAY 4
#define GCC_OP_INSERT 5
#define GCC_OP_WORD(op, field, v) \
    ((int32_t)(0x80000000u | ((uint32_t)(op) << 28) | ((uint32_t)(field) << 24) | ((uint32_t)(v) & 0xFFFFFFu)))

/* Dataset generator dedup modes (gen_ycsb drops repeated keys, which leaves
 * fewer than 16 requests; resample redraws until 16 distinct keys). */
#define GCC_DEDUP_DROP 0
#define GCC_DEDUP_RESAMPLE 1

/* One request of a gen_ycsb record: {int read; unsigned key;} (8 bytes). */
typedef struct gcc_ycsb_req {
    int32_t read;
    uint32_t key;
} gcc_ycsb_req;

/* One gen_ycsb record: {size_t request_cnt; YCSBReq requests[16];} = 136
 * bytes, little-endian, headerless array (include/ycsb.cuh:21-33). */
typedef struct gcc_ycsb_tx {
    uint64_t request_cnt;
    gcc_ycsb_req requests[16];
} gcc_ycsb_tx;

typedef struct gcc_table_desc {
    uint64_t rows;       /* number of rows (keys 0..rows-1) */
    int32_t layout;      /* GCC_LAYOUT_* */
    int32_t index_kind;  /* GCC_INDEX_* */
    uint64_t fill_seed;  /* fields uniform from this seed; 0 = zero fields */
    int32_t device;      /* CUDA device ordinal */
    int32_t max_batch;   /* largest batch_size a run may use (sizes scratch) */
} gcc_table_desc;

typedef struct gcc_run_params {
    const char *cc_scheme; /* tpl_nw tpl_wd to mvcc silo tictoc gacco gputx
                              slow_tpl_nw slow_tpl_wd slow_to slow_mvcc
                              slow_silo slow_tictoc (+ aliases slowto,
                              slowmvcc) */
    int32_t warp_density;  /* 2^wd threads per transaction, 0..5 */
    int32_t block_size;    /* warps per CTA, 1..32 */
    int32_t batch_size;    /* transactions per batch (gputx ranks all) */
    uint32_t flags;        /* GCC_F_* */
    int32_t write_mode;    /* GCC_WRITE_* */
    int32_t backoff_ns;    /* retry pause: after 8 failed attempts each retry
                              first sleeps a random 0..backoff_ns ns (0 means
                              512); -1 never sleeps (the reference retries at
                              once, benchmark/ycsb.cu:101, which lets two OCC
                              transactions with crossing read/write sets abort
                              each other indefinitely) */
    uint64_t write_seed;   /* seed of GCC_WRITE_FIELD values */
    uint64_t spin_limit_ns;/* bound of any single device wait; 0 = 4 s */
    int32_t starve_limit;  /* attempts after which a transaction counts as
                              starving: while one is, no new transaction is
                              started (for at most spin_limit_ns), and past 4x
                              this many attempts starving transactions retry
                              one at a time (0: 32; -1: never) */
    int32_t max_active;    /* cap on transactions in flight at once: the
                              persistent grid holds at most this many (rounded
                              up to whole CTAs); 0 = as many as the GPU holds.
                              Under heavy contention fewer in flight abort
                              less. With GCC_F_AUTOTUNE the tuner picks it. */
    int32_t ordered_after; /* 2PL and TO: failed attempts after which a retry
                              visits its requests one at a time instead of
                              all at once; 0 = 15 */
    int32_t reserved;
} gcc_run_params;

/* Fields 1-15 are the 15 columns of the reference's output line
 * (include/runtime.cuh:182-196); *_d are per-transaction averages in ms of
 * GPU clock, *_s are seconds of host-observed (CUDA event) time. */
typedef struct gcc_result {
    double tx_per_s;
    uint64_t committed;
    uint64_t aborts;
    double ts_d, wait_d, abort_d, mng_d, tot_d, idx_d;
    double pre_s, proc_s, tot_s;
    double lat_p50_us, lat_p99_us; /* per-tx first start -> commit */
    uint64_t rank_count;           /* gputx: number of ranks */
    uint64_t batches;              /* kernel batches launched */
    uint64_t kernel_launches;      /* engine kernels launched by the run */
    uint32_t max_attempts;         /* most attempts any one tx needed */
    uint32_t err_site;             /* where a bounded wait gave up (0: none) */
} gcc_result;

/* Serialization key of one committed transaction: replaying transactions in
 * ascending (hi, lo) order reproduces the run. */
typedef struct gcc_commit_rec {
    uint64_t hi;
    uint64_t lo;
} gcc_commit_rec;

typedef struct gcc_engine gcc_engine;

/* Library / device information. */
const char *gcc_version(void);
const char *gcc_strerror(int status);
int gcc_scheme_id(const char *cc_scheme); /* >= 0, or GCC_EINVAL */
uint32_t gcc_row_bytes(int32_t layout);   /* 88 or 104 */
uint32_t gcc_row_stride(int32_t layout);  /* 96 or 112 */

/* Dataset generation (host; gen_ycsb, generation/gen_ycsb.cu:34-152).
 * Keys are Zipfian (Gray et al. 1994) ranks: key_base 1 draws keys in
 * [1, rows-1] exactly like gen_ycsb; key_base 0 draws in [0, rows-1].
 * Deterministic in (seed, tx index); `threads` host threads (0 = all). */
int gcc_gen_ycsb(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                 uint64_t seed, int32_t dedup, int32_t key_base,
                 int32_t threads, gcc_ycsb_tx *out);

/* Variable-length transactions (no counterpart in the reference's 136-byte
 * format, which caps a transaction at 16 requests): transaction t owns
 * requests reqs[tx_off[t] .. tx_off[t+1]), 1..64 of them, distinct keys in
 * ascending order. The offsets are a pure function of (seed, tx) with
 * min_ops..max_ops requests per transaction; the requests follow gen_ycsb's
 * rules (Zipf keys, read probability, repeats redrawn, key order). */
int gcc_gen_ycsb_var_offsets(uint64_t n_tx, uint32_t min_ops, uint32_t max_ops,
                             uint64_t seed, uint32_t *tx_off /* n_tx + 1 */);
int gcc_gen_ycsb_var(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                     uint64_t seed, int32_t key_base, int32_t threads,
                     const uint32_t *tx_off, gcc_ycsb_req *reqs);

/* ---- Order-entry workload (integer; shape of the reference's TPC-C
 * new-order / payment path, benchmark/tpcc.cu:35-380 and
 * generation/gen_tpcc.cu:108-182, with money in integer cents instead of
 * floats and inserted rows at ids assigned at generation). Transactions are
 * variable-length requests with extended ops (GCC_OP_*), sorted by row id;
 * run them with GCC_F_EXT_OPS on an engine of `rows` rows with the direct
 * index, after gcc_oe_fill. Row groups and fields:
 *   warehouse w                 0 ytd cents, 1 tax bp
 *   district  w*D + d           0 ytd, 1 tax, 2 next_o_id
 *   customer  (w*D + d)*C + c   0 balance (signed), 1 ytd_payment,
 *                               2 payment_cnt, 3 discount bp
 *   item      i                 0 price cents (read only)
 *   stock     w*I + i           0 quantity, 1 ytd, 2 order_cnt, 3 remote_cnt
 *   inserts                     one slot per inserted row
 * new-order: read warehouse, district next_o_id += 1, read customer, per
 * line read item + STOCK update + insert order line, insert order (4 + 3 x
 * lines requests); payment: warehouse and district ytd += amount, customer
 * PAY, insert history (4 requests). */
typedef struct gcc_oe_desc {
    uint32_t warehouses;           /* W (64 in the serving workload) */
    uint32_t districts;            /* D per warehouse (10) */
    uint32_t customers;            /* C per district (3000) */
    uint32_t items;                /* I, also stock rows per warehouse (100000) */
    uint32_t new_order_pct;        /* share of new-order transactions (50) */
    uint32_t remote_line_permille; /* order lines from another warehouse (10) */
    uint32_t remote_customer_pct;  /* payments of another warehouse's customer (15) */
    uint32_t min_lines, max_lines; /* order lines per new-order (5, 15) */
} gcc_oe_desc;

typedef struct gcc_oe_layout {
    uint64_t warehouse, district, customer, item, stock, inserts; /* first rows */
    uint64_t rows;                                                /* total rows */
} gcc_oe_layout;

/* Request offsets of n_tx transactions (tx_off[n_tx + 1]) and the row
 * layout they need; pure functions of (desc, seed, transaction index). */
int gcc_oe_offsets(const gcc_oe_desc *d, uint64_t n_tx, uint64_t seed, uint32_t *tx_off,
                   gcc_oe_layout *layout);
/* The requests (reqs[tx_off[n_tx]]); kind[t] = 1 new-order, 2 payment
 * (optional). `threads` host threads (0 = all). */
int gcc_oe_gen(const gcc_oe_desc *d, uint64_t n_tx, uint64_t seed, int32_t threads,
               const uint32_t *tx_off, gcc_ycsb_req *reqs, uint8_t *kind);
/* Initial order-entry rows on the device (the engine's rows must be at least
 * layout.rows of the same desc; inserts area and unused fields zero):
 * warehouse ytd 30,000,000 and tax h % 2001; district ytd 3,000,000, tax
 * h % 2001, next_o_id 3001; customer balance -1000, ytd_payment 1000,
 * payment_cnt 1, discount h % 5001; item price 100 + h % 9901; stock
 * quantity 10 + h % 91; h = splitmix-based hash of (seed, row, field). */
int gcc_oe_fill(gcc_engine *e, const gcc_oe_desc *d, uint64_t seed);

/* Engine lifetime (Table_CPU::InitData + AddIndex + DB_CPU::ToGPU). */
int gcc_create(const gcc_table_desc *desc, gcc_engine **out);
void gcc_destroy(gcc_engine *e);

/* Upload n_tx gen_ycsb records from host memory (benchmark_cpu/ycsb.cu:
 * 120-148). Records are validated on the device (request_cnt <= 16). */
int gcc_load_txs(gcc_engine *e, const gcc_ycsb_tx *txs, uint64_t n_tx);

/* Execute every loaded transaction under one scheme (the batch loop of
 * benchmark_cpu/ycsb.cu:249-292). Synchronous. */
int gcc_run(gcc_engine *e, const gcc_run_params *p, gcc_result *out);

/* gcc_run plus a serializability check (the role of ExecInfo::Check,
 * src/runtime.cu:129-158, run on the GPU): the committed transactions are
 * executed again, one after another in their recorded serialization order,
 * from the table as it was before the run, by the deterministic ordered
 * executor; *verdict = 1 when that reproduces the run's final table and
 * every read digest, else 0. The engine is left in the run's final state. */
int gcc_run_checked(gcc_engine *e, const gcc_run_params *p, gcc_result *out,
                    int *verdict);

/* Reference output line (ExecInfo::Analyse CSV columns) for a result. */
int gcc_format_line(const gcc_run_params *p, const gcc_result *r, char *buf,
                    size_t buf_bytes);

/* ---- batched execution of variable-length transactions ------------------
 * Upload n_tx variable-length transactions (tx_off: n_tx + 1 offsets into
 * reqs; at most 64 requests each). They replace nothing loaded by
 * gcc_load_txs; digests, aborts and commit keys of gcc_run_batches are read
 * with the same getters (indexed by tx). */
int gcc_load_var_txs(gcc_engine *e, const uint32_t *tx_off, const gcc_ycsb_req *reqs,
                     uint64_t n_tx);

/* Modes of gcc_run_batches. */
#define GCC_BATCHES_SEQUENTIAL 0 /* one kernel launch per batch, batch after
                                    batch, metadata reset per batch (the
                                    reference's batch loop) */
#define GCC_BATCHES_QUEUE 1      /* one persistent kernel drains every batch
                                    from a device queue in admission order;
                                    no per-batch barrier (tpl_nw, tpl_wd, to,
                                    silo, tictoc) */
/* Extra run flags of gcc_run_batches. */
#define GCC_F_AUTOTUNE 16u /* choose warp_density / block_size / transactions
                              in flight / batch_size per batch class (size,
                              requests per tx) from measured runs */
#define GCC_F_GRAPH 32u    /* capture the whole run in a CUDA graph once and
                              replay it while the configuration is unchanged */

/* Run the loaded variable-length transactions split into n_batches batches
 * (batch b = transactions batch_off[b] .. batch_off[b+1]). Schemes: every
 * scheme but gacco and gputx (their ordering passes take 16-request records),
 * mvcc and slow_mvcc in sequential mode only; warp_density 2..5. With
 * GCC_F_AUTOTUNE the tuner picks per batch class warp_density, block_size,
 * the transactions in flight and the batch_size of the launches inside a
 * batch. Synchronous. */
int gcc_run_batches(gcc_engine *e, const gcc_run_params *p, const uint32_t *batch_off,
                    uint64_t n_batches, int32_t mode, gcc_result *out);

/* Per-batch configuration and kernel time of the last gcc_run_batches
 * (sequential mode; queue mode reports one entry for the whole run). */
int gcc_get_batch_stats(gcc_engine *e, int32_t *warp_density, int32_t *block_size,
                        double *kernel_ms, uint64_t n);

/* Transactions in flight (persistent grid x transactions per CTA) of each
 * entry of the last gcc_run_batches, entry for entry as gcc_get_batch_stats.
 * No counterpart in the reference (its grid covers the whole batch). */
int gcc_get_batch_active(gcc_engine *e, uint64_t *active, uint64_t n);

/* batch_size the autotuner chose for each batch of the last gcc_run_batches
 * (entry for entry as gcc_get_batch_stats): the batch ran in launches of at
 * most this many transactions, 0 = one launch for the whole batch (the
 * reference's batch_size knob, benchmark_cpu/ycsb.cu:262-271). */
int gcc_get_batch_split(gcc_engine *e, uint32_t *split, uint64_t n);

/* Results of the last run / current state (device -> host copies). */
int gcc_dump_table(gcc_engine *e, void *host_dst, uint64_t bytes); /* packed rows */
int gcc_upload_table(gcc_engine *e, const void *host_src, uint64_t bytes);
int gcc_get_digests(gcc_engine *e, uint64_t *dst, uint64_t n_tx);
int gcc_get_commit_log(gcc_engine *e, gcc_commit_rec *dst, uint64_t n_tx);
int gcc_get_tx_aborts(gcc_engine *e, uint32_t *dst, uint64_t n_tx);
/* Read log: n_tx * 16 slots of gcc_row_stride(layout) bytes (slot = tx*16 +
 * op), each holding the row image that read request read (row_bytes used). */
int gcc_get_read_log(gcc_engine *e, void *dst, uint64_t bytes);
/* Index probe for n keys (testing the index): rows[i] = row or UINT32_MAX. */
int gcc_index_lookup(gcc_engine *e, const uint32_t *keys, uint32_t *rows,
                     uint64_t n);

/* 2PL no-wait over caller-owned device buffers, allocating no device memory
 * (no counterpart in the reference). For callers that cannot call cudaMalloc:
 * code whose device memory belongs to another allocator (a framework's pool,
 * a pre-sized arena) or that runs on a latency-bound thread where
 * cudaMalloc's implicit device synchronisation is not acceptable. All
 * pointers are device pointers owned by the caller: `txs` (n_tx gen_ycsb
 * records, keys are row ids), `table` (rows x 96-byte rows of the u64x11
 * layout, updated in place), outputs `digests` (n_tx) and `tx_aborts`
 * (n_tx). Writes are GCC_WRITE_FIELD with `write_seed`. Scratch (a lock word
 * per row and the run counters) lives in a static device array of this
 * library: at most 1,048,576 rows (8 MiB), held by every GPU that loads the
 * library until exit; larger tables are rejected with GCC_EINVAL. Calls on a
 * device share that array and clear it before use, so calls that overlap on
 * the GPU race. The first call on a device looks up the array's address with
 * the device current; make it before any stream capture. The address belongs
 * to the device's primary context: after cudaDeviceReset the entry point
 * must not be called on that device again in the process. Runs on `stream`
 * (a cudaStream_t, may be null) and returns only after its kernel has
 * finished, on errors too; committed / aborts may be null. Retries follow
 * gcc_run's defaults (starvation control at 32 attempts). */
int gcc_run_tpl_nw_noalloc(const gcc_ycsb_tx *txs, uint64_t n_tx, void *table,
                           uint64_t rows, uint64_t *digests, uint32_t *tx_aborts,
                           uint64_t write_seed, void *stream, uint64_t *committed,
                           uint64_t *aborts);

/* gcc_run with the records coming from host memory: batch b's records are
 * copied on a copy stream while earlier batches execute, each batch waits
 * only for its own records, and (if host_digests is not null) each batch's
 * read digests are copied back while later batches execute. Results equal
 * gcc_load_txs + gcc_run + gcc_get_digests; use pinned host memory for the
 * copies to overlap. No counterpart in the reference (it reads the whole
 * dataset first, benchmark_cpu/ycsb.cu:120-124). */
int gcc_run_host(gcc_engine *e, const gcc_run_params *p, const gcc_ycsb_tx *host_txs,
                 uint64_t n_tx, uint64_t *host_digests, gcc_result *out);

/* Device-side timing of the last run's main kernels: total ms and number of
 * launches of the transaction kernel (for roofline accounting). */
int gcc_last_kernel_ms(gcc_engine *e, double *kernel_ms, uint64_t *launches);

/* L2 atomic throughput of `device` on the CC metadata's access pattern (no
 * counterpart in the reference): every SM issues 64-bit atomics to
 * pseudo-random words of a `words`-word array (a power of two, 1,024 ..
 * 16,777,216 words, i.e. at most 128 MiB, about the L2), 8 in flight per
 * thread; *atomics_per_s = atomics completed per second of the timed pass.
 * The denominator of the transaction kernel's L2 atomic rate (ncu
 * lts__t_requests_op_atom + _op_red). Allocates and frees its array. */
#define GCC_CALIB_ADD 0
#define GCC_CALIB_CAS 1
int gcc_l2_atomic_rate(int32_t device, uint64_t words, int32_t mode, double *atomics_per_s);

/* ---- Learned contention scheduling (no counterpart in the reference,
 * which runs every batch in transaction-index order with one launch,
 * benchmark_cpu/ycsb.cu:262-285). A small MLP (66 -> 128 -> 128 -> 1, BF16
 * weights, FP32 accumulation, sigmoid) predicts per transaction the
 * probability that it aborts at least once under plain ordering. Each
 * scheduled batch runs its predicted-safe transactions first at full
 * concurrency and defers the rest into a second sub-batch with a cap on
 * transactions in flight (and, for 2PL, no-wait or wait-die). The choice is
 * measured, with plain ordering as one of the choices: a batch runs its
 * first half under the incumbent choice and its second half under a
 * neighbouring one, and the faster becomes the incumbent; the comparisons
 * restart when the network's mean prediction shows the contention moved. Every explore_every-th batch first runs a probe of probe_rows
 * transactions with plain ordering at full concurrency: their abort outcomes
 * are the training labels (Adam on the GPU) and their abort rate the
 * yardstick. CC arithmetic and commit rules are untouched. Schemes: tpl_nw,
 * tpl_wd, silo, tictoc; 16-request records loaded with gcc_load_txs;
 * batch_size at most 1,048,576. */
#define GCC_SCHED_PLAIN 0   /* plain ordering every batch (same driver) */
#define GCC_SCHED_LEARNED 1
#define GCC_SCHED_FEAT_STRIDE 72 /* u16 per feature row (66 used) */

typedef struct gcc_sched gcc_sched;

typedef struct gcc_sched_params {
    int32_t mode;            /* GCC_SCHED_* */
    int32_t explore_every;   /* every n-th batch starts with a probe; 0 = 4 */
    int32_t probe_rows;      /* transactions of a probe; 0 = 4096 */
    int32_t train_steps;     /* Adam steps after each probe; 0 = 4, -1 = none */
    int32_t minibatch;       /* rows per step; 0 = 4096 */
    float lr;                /* Adam learning rate; 0 = 2e-3 */
    float defer_threshold;   /* predicted probability above which a
                                transaction is deferred; 0 = 0.2 */
    int32_t fixed_arm;       /* 0: the policy chooses; k > 0: every batch
                                runs arm k-1 of: plain ordering, deferral
                                with in-flight cap 2048, 1024, 512, 256, 128,
                                and for 2PL wait-die deferral at 1024, 512 */
    int32_t min_sched;       /* batches smaller than this run with plain
                                ordering and skip the predictor (few
                                transactions are in flight anyway, and the
                                scheduling pass would add its latency);
                                0 = 4096, -1 = schedule every batch */
    int32_t plan_threshold;  /* 2PL lock plans of scheduled batches (16-request
                                records): a request whose key's counter in the
                                frequency table is at least this is locked
                                after the others, one at a time, the hottest
                                last, so the hottest locks are held the
                                shortest time (counters are halved after
                                every batch and count every request, so a
                                key read or written k times per batch
                                settles near 2k); 0 = 1024, -1 = no plans */
    uint64_t seed;           /* initial weights (He-uniform from this seed) */
    int32_t plan_after;      /* attempts after which a planned transaction
                                locks as planned (before that, all at once);
                                0 = 1 (from its first retry), -1 = from its
                                first attempt */
    int32_t reserved;
} gcc_sched_params;

typedef struct gcc_sched_batch {
    uint32_t kind;           /* 0 plain mode, 1 scheduled */
    uint32_t bucket;         /* contention level: mean prediction x 4 */
    uint32_t arm;            /* the incumbent arm (0 = plain ordering) */
    uint32_t in_flight_cap;  /* cap of the deferred sub-batch (0 = none) */
    uint32_t wait_die;       /* deferred sub-batch ran 2PL wait-die */
    uint32_t probe;          /* transactions of the batch's probe */
    uint64_t deferred;       /* transactions in the deferred sub-batch */
    float pred_mean;         /* mean predicted abort probability (after the probe) */
    float label_mean;        /* probes: fraction that aborted */
    float loss;              /* probes: mean BCE of the predictions made
                                before training on the probe */
    uint32_t explored;       /* 1 + the arm the batch's second half ran to
                                compare it with the incumbent (0 = none) */
    double ms;               /* device time of the batch incl. scheduling */
    uint64_t committed, aborts;
} gcc_sched_batch;

typedef struct gcc_sched_result {
    gcc_result run;          /* totals over all batches, as gcc_run */
    uint64_t probed, deferred;
    double probe_tx_per_s;   /* committed / kernel time of the probes */
    double sched_tx_per_s;   /* the same over the non-probe parts */
    double probe_abort_rate; /* aborts / (aborts + committed) in probes */
    double sched_abort_rate; /* the same over the non-probe parts */
    double predict_ms, train_ms; /* device time of inference / training */
    double last_loss;        /* BCE of the last probe's predictions */
} gcc_sched_result;

int gcc_sched_create(gcc_engine *e, const gcc_sched_params *p, gcc_sched **out);
void gcc_sched_destroy(gcc_sched *s);
/* Run the loaded records in batches of rp->batch_size under the schedule
 * (rp->max_active, if set, caps the plain sub-batches too). Synchronous;
 * the engine's outputs (table, digests, commit log, tx aborts) are those of
 * the run. The frequency table, weights and policy statistics persist
 * across runs. */
int gcc_sched_run(gcc_sched *s, const gcc_run_params *rp, gcc_sched_result *out);
/* Per-batch records of the last run (n <= its batch count). */
int gcc_sched_batches(gcc_sched *s, gcc_sched_batch *dst, uint64_t n);
/* Features of loaded records first .. first+n-1 against the current
 * frequency table: n rows of GCC_SCHED_FEAT_STRIDE u16 (host). */
int gcc_sched_features(gcc_sched *s, uint64_t first, uint64_t n, uint16_t *dst);
/* 2PL lock plans of loaded records first .. first+n-1 against the current
 * frequency table and the scheduler's plan_threshold, as a scheduled batch
 * computes them (host, one u64 per record): bits 0-15 mark the requests
 * locked last, bits 16-19 count them (at most 11, the hottest), and nibble j
 * at bit 20 + 4j is the j-th of them in locking order (the request whose
 * key has the larger counter later; equal counters by ascending key).
 * GCC_EINVAL when plans are off (plan_threshold -1). */
int gcc_sched_lock_plans(gcc_sched *s, uint64_t first, uint64_t n, uint64_t *dst);
/* Count records first .. first+n-1 into the frequency table (after halving
 * it), as a run does after each batch; clear = 1 zeroes it first. */
int gcc_sched_observe(gcc_sched *s, uint64_t first, uint64_t n, int32_t clear);
/* The same two over the loaded variable-length transactions (requests past
 * the 16th count in the sketch, write and hot-key features alike). */
int gcc_sched_features_var(gcc_sched *s, uint64_t first, uint64_t n, uint16_t *dst);
int gcc_sched_observe_var(gcc_sched *s, uint64_t first, uint64_t n, int32_t clear);
/* Parameters: gcc_sched_param_count() FP32 values, layout W1[66][128],
 * b1[128], W2[128][128], b2[128], w3[128], b3. set rounds them to BF16 for
 * compute and resets Adam. */
uint64_t gcc_sched_param_count(void);
int gcc_sched_set_weights(gcc_sched *s, const float *w, uint64_t n);
int gcc_sched_get_weights(gcc_sched *s, float *w, uint64_t n);
/* Forward pass over n host feature rows -> p[n] (host). */
int gcc_sched_predict(gcc_sched *s, const uint16_t *feat, uint64_t n, float *p);
/* Gradient of the mean binary cross-entropy over n host rows with 0/1
 * labels -> grad[param_count] (host), *loss = the mean loss. */
int gcc_sched_gradient(gcc_sched *s, const uint16_t *feat, const uint8_t *labels, uint64_t n,
                       float *grad, double *loss);
/* steps Adam steps on minibatches of the given rows (cycling through them);
 * *loss = mean loss of the last step. */
int gcc_sched_train(gcc_sched *s, const uint16_t *feat, const uint8_t *labels, uint64_t n,
                    int32_t steps, double *loss);

/* ---- Serving (no counterpart in the reference, which runs a fixed dataset
 * in batches): the engine's loaded variable-length transactions arrive one
 * by one as a Poisson process of rate rate_tps; a host loop admits every
 * arrived transaction (at most the admission cap) as the next batch once
 * min_batch have arrived or the oldest has waited max_wait_us, runs it
 * through the scheduler `s` (GCC_SCHED_LEARNED: predictor, deferral, probes
 * and training; GCC_SCHED_PLAIN: plain ordering) and takes the time the
 * batch's commit is visible on the host as the commit time of all its
 * transactions. Table and CC state stay resident across batches (use
 * GCC_F_NO_RESET to keep the metadata too). Schemes: tpl_nw, tpl_wd, silo,
 * tictoc; warp_density 2..5. Synchronous; wall-clock paced. */
typedef struct gcc_serve_params {
    double rate_tps;        /* mean arrival rate, transactions / s */
    uint64_t seed;          /* arrival process */
    int32_t max_batch;      /* admission cap; 0 = what half the free device
                               memory holds at the scheduler's footprint */
    int32_t min_batch;      /* arrivals that start a batch at once (0 = 1) */
    double max_wait_us;     /* ... or the oldest's wait (0 = 200 us) */
} gcc_serve_params;

typedef struct gcc_serve_result {
    uint64_t committed, aborts, batches, admit_cap;
    double offered_tps;      /* arrivals / s of the generated process */
    double tx_per_s;         /* commits / s of wall time */
    double device_tx_per_s;  /* commits / s of device time (the batches) */
    double lat_p50_us, lat_p99_us, lat_max_us; /* arrival -> commit */
    double mean_batch;       /* transactions per batch */
    double busy_frac;        /* share of wall time spent in batches */
    double sched_abort_rate; /* aborts / (aborts + commits) outside probes */
    uint64_t kernel_launches;/* engine kernels launched by the run */
} gcc_serve_result;

int gcc_serve(gcc_sched *s, const gcc_run_params *rp, const gcc_serve_params *sp,
              gcc_serve_result *out);

#ifdef __cplusplus
}
#endif
#endif /* GCC_ENGINE_H */
