/* inspire_b200.h -- C ABI of the B200-native InsPIRe PIR server.
 *
 * Part 1 is the server half of the reference's C ABI (SoraSuegami/InsPIRe-GPU
 * src/capi.h:23-91), same names, same struct layouts, same flat array layouts
 * and the same return codes, so an FFI consumer that linked the reference's
 * GPU library links this one instead.  The client half of that header
 * (ipir_query_build, ipir_extract, packing, compression) stays in the
 * reference's CPU library and is not defined here.
 *
 * Part 2 holds additive entry points (prefix ipir_b200_) that the reference
 * does not have: explicit streams, a device-resident staged pipeline, stage
 * timers, precomp export, schedule autotuning, and the GPU primitives for
 * parity checks.  Part 3 (prefix ipir_serve_) is the continuous-batching
 * serving loop.  Part 4 splits one database over several GPUs by group
 * ranges (shards and a Horner owner).
 *
 * Values are residues mod the two 27-bit primes q0 = 94519297 and
 * q1 = 95293441 carried in u64 (u32 for GPU-side primitives).  One server
 * handle is single-threaded; distinct handles are independent.  No entry
 * point aborts the process: CUDA failures come back as error codes, with
 * the text in ipir_b200_last_error().
 */
#ifndef INSPIRE_B200_H
#define INSPIRE_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ===================================================== part 1: server half */

/* Opaque handle (reference src/capi.h:23). */
typedef struct ipir_server ipir_server;

/* Public parameters (reference src/capi.h:27-38). */
typedef struct {
    size_t n_entries;
    size_t entry_bytes;
    size_t db_rows;
    size_t db_cols;
    size_t n_packed;
    size_t interp_d;
    size_t num_cts;
    size_t ring_n;
    size_t d_eff;
    uint8_t seed[64];
} ipir_params;

/* Capability report (reference src/capi.h:40-45). */
typedef struct {
    size_t max_batch;
    size_t resident_bytes;
    size_t device_free_bytes;
    size_t num_cts;
} ipir_caps;

/* One query as views into caller-owned u64 arrays (reference src/capi.h:47-61):
 *   lwe_b_limb0/1     db_rows values (mod q0 / q1)
 *   ksk5_b, kskneg1_b d_eff*2*ring_n values, [digit][limb][coeff], coefficient form
 *   rgsw              4*d_eff*2*ring_n values,
 *                     [top_a | top_b | bot_a | bot_b][digit][limb][coeff], NTT form */
typedef struct {
    const uint64_t* lwe_b_limb0;
    const uint64_t* lwe_b_limb1;
    const uint64_t* ksk5_b;
    const uint64_t* kskneg1_b;
    const uint64_t* rgsw;
} ipir_query_view;

/* Build a server for one database generation (replaces reference
 * src/capi.h:76-80 / src/capi.cu:51-87).  db: db_rows*db_cols u16 values in
 * [0, 65535), row-major.  db_rows_or_zero == 0 picks db_rows = 32768.
 * crs_seed_or_null: 64-byte CRS seed or NULL for a fresh one.  Returns NULL
 * on error (bad geometry, CUDA failure, out of memory). */
ipir_server* ipir_server_create(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero,
                                size_t max_batch, const uint16_t* db, const uint8_t* crs_seed_or_null,
                                ipir_params* out_params);

/* Reference src/capi.h:82 / src/capi.cu:89-96. */
void ipir_server_caps(const ipir_server* srv, ipir_caps* out);

/* Answer count <= max_batch queries (reference src/capi.h:84-89 /
 * src/capi.cu:98-126).  out_resp: count*num_cts*4*ring_n u64,
 * [query][ct][a | b][limb][coeff], NTT form.  Returns 0 on success, 1 null
 * argument, 2 count > max_batch, 3 null view field (nothing written on 1-3),
 * 4 CUDA failure (the reference exits the process instead). */
int ipir_answer_batch(ipir_server* srv, const ipir_query_view* queries, size_t count, uint64_t* out_resp);

/* Reference src/capi.h:91. */
void ipir_server_destroy(ipir_server* srv);

/* ===================================================== part 2: additive */

/* Text of the calling thread's last failure ("" if none). */
const char* ipir_b200_last_error(void);

/* Geometry exactly as the reference's setup() (src/params.cpp:23-68) plus
 * this server's layout checks; seed left zero.  Returns 0, or nonzero when
 * the geometry is rejected (text in ipir_b200_last_error). */
int ipir_b200_setup(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero, ipir_params* out);

/* Run this handle's work on the caller's CUDA stream (cudaStream_t cast to
 * void*; NULL restores the handle's own stream). */
int ipir_b200_set_stream(ipir_server* srv, void* cuda_stream);

/* Device-resident pipeline split in three: stage copies count queries into
 * the device slots (async on the handle's stream); run launches the answer
 * kernels on the staged slots; fetch copies the responses (same layout as
 * ipir_answer_batch) to the host and synchronises.  Return codes as
 * ipir_answer_batch. */
int ipir_b200_stage_queries(ipir_server* srv, const ipir_query_view* queries, size_t count);
int ipir_b200_run(ipir_server* srv, size_t count);
int ipir_b200_fetch_responses(ipir_server* srv, size_t count, uint64_t* out_resp);
int ipir_b200_sync(ipir_server* srv);

/* Stage timers (CUDA events on the handle's stream), off by default.
 * stage_times writes up to n floats (ms) of the last run:
 * [qprep, matvec, collapse, finalize, horner]. */
int ipir_b200_enable_stage_timing(ipir_server* srv, int on);
int ipir_b200_stage_times(const ipir_server* srv, float* ms_out, size_t n);

/* Copy one group's precomputed tensors to the host (u32, NTT form, the
 * reference's per-group layouts, src/protocol.h:14-17):
 *   a [limb][N], d_plus / d_minus [limb][step<1023][digit][N],
 *   d_final [limb][digit][N].  Any pointer may be NULL. */
int ipir_b200_export_precomp(const ipir_server* srv, size_t group, uint32_t* a, uint32_t* d_plus,
                             uint32_t* d_minus, uint32_t* d_final);
/* Copy rows [row0, row0+nrows) of the encoded device DB to the host. */
int ipir_b200_export_db(const ipir_server* srv, size_t row0, size_t nrows, uint16_t* out);

/* Server checkpoints.  No counterpart in the reference, whose server state
 * lives only in device memory (a restart re-runs gpu_preprocess on the raw
 * DB).  save writes the handle's resident state -- the encoded DB, the
 * precomputed a, D (as the tensor pass's byte planes) and D_final tensors,
 * and the public parameters including the CRS seed -- to `path`, each
 * section with a checksum computed on the device: 0, 1 null argument,
 * 4 CUDA failure, 5 I/O error (text in ipir_b200_last_error).  load
 * restores it into a new handle on the current device without the raw DB
 * and without preprocessing; responses are bit-identical to the saved
 * handle's.  It returns NULL (text in ipir_b200_last_error) for a missing,
 * truncated or foreign file, a geometry setup() rejects, or a checksum
 * mismatch; the file is checked before any device memory is allocated.
 * Layout (little-endian): "IPIRB200", u32 version 1, u32 header bytes 256,
 * u64 n_entries, entry_bytes, db_rows, db_cols, n_packed, interp_d, num_cts,
 * 64 seed bytes, u64 section bytes[4] and checksums[4] (db, a, d byte
 * planes, d_final), zero padding to 256, then the sections. */
int ipir_b200_save_server(const ipir_server* srv, const char* path);
ipir_server* ipir_b200_load_server(const char* path, size_t max_batch, ipir_params* out_params);

/* GPU primitives on host buffers (current device), the kernels the server
 * runs.  ntt: in-place forward (inverse = 0) or inverse NTT of n polys of
 * 2048 residues; poly i is mod q_((i / limb_run) & 1).  decomp: n polys
 * [i][limb][2048] coefficient form -> [i][digit][limb][2048] (reference
 * src/ring.cpp:205-246, digits 1..2 of base 2^18). */
int ipir_b200_ntt(uint32_t* polys, size_t n, int limb_run, int inverse);
int ipir_b200_decomp(const uint32_t* in, uint32_t* out, size_t n);

/* Host SHAKE-256 and the CRS expand_seed of reference src/ring.cpp:252-279
 * (out: [limb][2048] u32). */
int ipir_b200_shake256(const uint8_t* in, size_t inlen, uint8_t* out, size_t outlen);
int ipir_b200_expand_seed(const uint8_t* seed64, const char* domain, uint64_t index, uint32_t* out);

/* Standalone exact mat-vec on the tensor cores (the DB pass of the answer,
 * reference src/gpu_online.cu:23-175 gpu_matvec_dual / _batched), on device
 * pointers: out[q][limb][c] = sum_i db[i][c] * (queries[q][limb][i] mod q_limb)
 * mod q_limb for q < count.  db: rows x cols u16 row-major; queries:
 * count x [2][rows] u64; out: count x [2][cols] u32.  rows a multiple of
 * 1024 (of 32768 above 32768), cols a multiple of 128.  Scratch (query byte
 * planes, K-chunk partials, tables) is allocated on the first call per
 * device and grown on demand; calls on one device must not overlap.
 * Enqueued on `stream`; with sync != 0 the call waits and reports a device
 * wait timeout as 5.  Returns 0, 1 null argument, 2 bad shape, 4 CUDA error. */
int ipir_b200_matvec(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries, size_t count,
                     uint32_t* out, void* stream, int sync);

/* Schedule of one ipir_b200_matvec_ex call.  Zero fields take the defaults. */
typedef struct {
    int path;             /* 0: tcgen05 int8 tensor cores (default), 1: CUDA cores (cols a multiple of 2048) */
    int queries_per_pass; /* queries sharing one DB pass: 1..32 (tensor cores, default 32), 1..4 (CUDA cores) */
    int kchunk_rows;      /* tensor cores: rows per exact s32 accumulation, a multiple of 1024 dividing rows and
                             <= 32768 (default: the largest that still gives every SM work) */
} ipir_matvec_opts;
/* ipir_b200_matvec with an explicit kernel schedule (opts may be NULL);
 * every schedule gives the same result.  No counterpart in the reference. */
int ipir_b200_matvec_ex(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries, size_t count,
                        uint32_t* out, void* stream, int sync, const ipir_matvec_opts* opts);

/* Same result as ipir_b200_matvec, for callers that may not allocate device
 * memory: processes whose device memory belongs to an allocator or pool they
 * must not bypass, or code that cannot afford cudaMalloc's implicit device
 * synchronisation.  No counterpart in the reference.  It allocates nothing:
 * its scratch (tables, error word, query byte planes) is a fixed ~2.7 MB
 * array in the library's device image, which every GPU that loads the
 * library keeps until the process exits.  Limits: rows a multiple of 1024
 * and <= 32768, count <= 8, cols a multiple of 128; larger shapes return 2
 * with the reason in ipir_b200_last_error().  The first call on a device
 * (and the first after a device reset, which gives the device a new
 * context) resolves the array's device address and writes the NTT tables
 * into it with a copy on `stream` that it waits for: make that first call
 * before any stream capture.  All calls share the one array, so calls whose
 * GPU work overlaps (other streams, other threads) race; serialise them.
 * The call synchronises `stream` only (the error word is read back on it)
 * and returns 0, 1 null argument, 2 shape beyond the limits, 4 CUDA error,
 * 5 device wait timeout. */
int ipir_b200_matvec_noalloc(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries,
                             size_t count, uint32_t* out, void* stream);

/* HornerEval (the reference's src/crypto.cpp:264-279, GPU form
 * src/gpu_online.cu:474-540) on caller data, through the server's Horner
 * kernels: acc = cts[L - 1]; for i = L - 2 .. 0: acc = ExtProd(rgsw, acc) +
 * cts[i]; out = acc.  rgsw: 4 * D_EFF * 2 * N u64
 * ([top_a|top_b|bot_a|bot_b][digit][limb][coeff], NTT form); cts: L * 4 * N
 * u64 ([ct][a|b][limb][coeff], NTT form); out: 4 * N u64.  L = 2 with
 * cts[0] = 0 is one ExtProd (src/crypto.cpp:219-257).  variant: 0 one CTA
 * per chain, 1 a 4-CTA cluster, 2 an 8-CTA cluster.  A parity primitive: it
 * allocates and synchronises.  Returns 0, 1 null argument or L = 0, 2 bad
 * variant or L > 4096, 4 CUDA error. */
int ipir_b200_horner_eval(const uint64_t* rgsw, const uint64_t* cts, size_t L, uint64_t* out, int variant);

/* Target of the library's device code as the CUDA runtime loaded it:
 * *out = cudaFuncAttributes.binaryVersion of its tensor-core mat-vec kernel
 * (100 for the sm_100a cubins this library is built from).  Returns 0, 1
 * null argument, 4 CUDA error.  No counterpart in the reference. */
int ipir_b200_kernel_binary_version(int* out);

/* Synthetic queries for load generation, written by a kernel on `stream`
 * (enqueued, not waited for) into the DEVICE buffer
 * out[count][2 db_rows + 6 * 2 * 2 * N] u64 in the flat query layout: word k
 * of query id = first_id + j is splitmix64(splitmix64(seed ^ id *
 * 0xd1b54a32d192ed03) ^ k) mod q_l (l: the word's limb), so any query can be
 * regenerated from its id.  Uniform residues, not encryptions: the server's
 * work does not depend on the values, and the reference's query() stays the
 * client for every correctness check.  No counterpart in the reference.
 * Returns 0, 1 null out, 2 db_rows not a positive multiple of N, 4 CUDA
 * error. */
int ipir_b200_synth_queries(size_t db_rows, uint64_t seed, uint64_t first_id, size_t count, uint64_t* out,
                            void* stream);

/* Synthetic database for benchmarks and tests: out[k] = splitmix64(seed ^ k)
 * mod 65535 for k < count, filled on all host threads. */
int ipir_b200_fill_db(uint16_t* out, size_t count, uint64_t seed);
/* Same values written by a kernel into device memory (enqueued on stream). */
int ipir_b200_fill_db_device(uint16_t* out, size_t count, uint64_t seed, void* stream);

/* Kernel schedule for one batch size: mat-vec on the tensor cores
 * (matvec_tc = 1) or the CUDA cores (0); queries per tensor-pass GEMM
 * (tp_pass); Horner on a 4-CTA cluster per chain (horner_cluster = 1), an
 * 8-CTA cluster (2) or one CTA per chain (0); tp_sms > 0 runs the tensor
 * pass on that many SMs at the same time as the tensor-core mat-vec on the
 * others (the two read disjoint data: the tensor pass is DRAM-bound, the
 * batched mat-vec tensor-core-bound), 0 runs them one after the other;
 * slice = 32 runs a batch of more than 32 queries as consecutive 32-query
 * pipelines (query prep to Horner), 0 as one pipeline; hchunks = 2..16
 * runs the tensor pass first and then the mat-vec and finalize in at most
 * that many group chunks (whole waves of mat-vec work) from the top group
 * down, each chunk's Horner steps on a second stream as soon as its packed
 * ciphertexts are final (databases whose response ciphertexts all chain
 * the same number of groups L = min(D, G), cluster Horner kernels, batches
 * of at most 32; the blocking and staged paths and the serving loop's lane
 * batches), 0 off; the default schedule uses 8 on such databases with
 * L >= 32 for batches of at most min(16, L / 16) queries.  Every schedule gives the same responses. */
typedef struct {
    int matvec_tc;
    int tp_pass;
    int horner_cluster;
    int tp_sms;
    int slice;
    int hchunks;
} ipir_serve_schedule;

/* Time the candidate schedules on this handle for batch sizes 1, 2, 4, ...
 * up to max_batch and keep the fastest for later calls (a second or so for
 * a 16 GB database).  No counterpart in the reference. */
int ipir_b200_autotune(ipir_server* srv);
/* The schedule the handle uses for `count` queries. */
int ipir_b200_get_schedule(const ipir_server* srv, size_t count, ipir_serve_schedule* out);
/* Pin the schedule the handle uses for `count` queries (tp_pass at most
 * the handle's tensor-pass capacity, min(max_batch, 32) or less for large
 * group counts): 0, 1 null argument, 2 out of range. */
int ipir_b200_set_schedule(ipir_server* srv, size_t count, const ipir_serve_schedule* sc);
/* Kernels launched by the handle's answer pipeline since create. */
int ipir_b200_launch_count(const ipir_server* srv, unsigned long long* out);

/* Wire formats on the GPU: the reference client library's packed query
 * (ipir_query_pack, 53-bit CRT-combined values), packed response
 * (ipir_response_pack) and compressed response (ipir_response_compress,
 * modulus switching to 28 / 20 bits), src/capi_client.cpp:156-385.
 * wire_sizes gives their per-query byte counts (as ipir_query_packed_bytes,
 * ipir_response_packed_bytes, ipir_response_compressed_bytes); any out
 * pointer may be NULL. */
#define IPIR_B200_RESP_FLAT 0
#define IPIR_B200_RESP_PACKED 1
#define IPIR_B200_RESP_COMPRESSED 2
int ipir_b200_wire_sizes(const ipir_params* params, size_t* query_packed, size_t* response_packed,
                         size_t* response_compressed);
/* ipir_answer_batch on packed queries: `packed` holds count queries back to
 * back (query_packed bytes each, as ipir_query_pack writes them); they cross
 * PCIe packed and are unpacked on the device.  The responses are written to
 * out back to back in resp_format: FLAT (ipir_response_u64s u64 each, the
 * ipir_answer_batch layout), PACKED (response_packed bytes each, identical to
 * ipir_response_pack of the flat response) or COMPRESSED (response_compressed
 * bytes each, identical to ipir_response_compress).  Returns 0, 1 null
 * argument, 2 count > max_batch, 3 unknown format, 4 CUDA failure. */
int ipir_b200_answer_wire(ipir_server* srv, const uint8_t* packed, size_t count, int resp_format, void* out);

/* ===================================================== part 3: serving loop
 *
 * Continuous batching over one or more resident databases: server handles
 * of any geometry, each created by ipir_server_create.  No counterpart in
 * the reference, whose batch entry point answers one caller-formed batch
 * per blocking call (src/capi.h:84-89).
 *
 * ipir_serve_submit copies one query for one database into a pinned request
 * slot and returns a ticket at once.  A worker thread admits waiting
 * requests, oldest first and up to max_batch at a time, into any free lane
 * of their database (per-batch device buffers with their own stream).  A
 * database's next batch starts as soon as its previous batch has finished
 * streaming the database and precomputed tensors, overlapping that batch's
 * Horner chains; requests that arrive meanwhile join it.  Lanes of
 * different databases run concurrently.  A lane batch replays the CUDA
 * graphs captured for its batch size at create.  With scan_segments > 1 a
 * database instead runs its DB and tensor passes as that many segments in
 * rotation, and waiting requests join at the next segment (the config
 * field says more).  All device and pinned memory is allocated at create,
 * with lanes sized to the HBM budget; submit, poll and wait allocate
 * nothing.  Each response is bit-identical to ipir_answer_batch on the same
 * query, whatever else shares its batch.
 *
 * The database handles must outlive the serving loop; while it runs, do not
 * autotune them.  The loop never touches a handle's own buffers or stream,
 * so a handle's blocking entry points stay usable from one other thread. */
typedef struct ipir_serve ipir_serve;

/* Zero fields take the defaults. */
typedef struct {
    size_t max_batch;        /* queries per lane batch (default 64) */
    size_t lanes_per_db;     /* concurrent batches per database (default 2) */
    size_t queue_slots;      /* pinned request slots (default 256) */
    size_t hbm_budget_bytes; /* device bytes for all lanes (default: free memory less 2 GiB);
                                over budget, max_batch halves, then lanes_per_db drops */
    int disable_graphs;      /* 1: launch the kernels directly instead of graph replays */
    int disable_autotune;    /* 1: default schedule instead of timing candidates at create */
    int overlap_db_passes;   /* 1: admit a batch on any free lane at once, even while the previous
                                batch of its database still streams the DB (default 0: wait for
                                that pass to end, overlapping only its Horner chains) */
    int scan_segments;       /* > 1 (a power of two <= 128): cyclic scan for each database whose
                                columns split into this many multiples of 128: its DB and tensor
                                passes run as that many segments in rotation on one lane of up to 32
                                queries, and waiting requests join at the next segment instead of
                                the next whole pass (default 0: lane batches); < 0: chosen per
                                database at create from its plain answer's device time (cyclic
                                scan from 2 ms, in the power of two of segments nearest to that
                                time in ms, 2 to 16; lane batches below) */
} ipir_serve_config;

typedef struct {
    uint64_t submitted;
    uint64_t completed;
    uint64_t failed;
    uint64_t batches;
    uint64_t batched_queries;
    uint64_t max_batch_seen;
    size_t queued;        /* admitted to no lane yet */
    size_t free_slots;    /* request slots free */
    double max_notice_ms; /* bound on the longest wait from a batch's end to the worker handling it */
} ipir_serve_counters;

/* NULL on error (text in ipir_b200_last_error).  cfg may be NULL. */
ipir_serve* ipir_serve_create(ipir_server* const* dbs, size_t n_dbs, const ipir_serve_config* cfg);
/* 0 queued (*ticket set), 1 null argument or bad db index, 3 null view
 * field, 4 the loop failed earlier (text in ipir_b200_last_error), 6 every
 * request slot is in use (collect tickets, then retry). */
int ipir_serve_submit(ipir_serve* sv, size_t db, const ipir_query_view* query, uint64_t* ticket);
/* Collect a ticket: 0 done (num_cts*4*ring_n u64 written to out_resp if not
 * NULL; *latency_ms = submit to response on the host, *queue_ms = submit to
 * the batch launch; either pointer may be NULL), 1 still pending, 2 unknown
 * or already collected ticket, 4 failed.  Every ticket must be collected
 * once: that frees its request slot. */
int ipir_serve_poll(ipir_serve* sv, uint64_t ticket, uint64_t* out_resp, double* latency_ms, double* queue_ms);
/* Same, blocking up to timeout_s; 5 when it is still pending then. */
int ipir_serve_wait(ipir_serve* sv, uint64_t ticket, double timeout_s, uint64_t* out_resp, double* latency_ms,
                    double* queue_ms);
int ipir_serve_stats(ipir_serve* sv, ipir_serve_counters* out);
/* Lanes, batch limit and schedule table (entries 1..min(sched_len-1,
 * max_batch) of sched) the loop chose for database db. */
int ipir_serve_db_info(ipir_serve* sv, size_t db, size_t* lanes, size_t* max_batch, ipir_serve_schedule* sched,
                       size_t sched_len);
/* Replace database `db` by its next generation `next` (a handle of the same
 * geometry on the same device, e.g. the refreshed DB preprocessed while the
 * loop kept serving the old one): admission to db pauses, its batches in
 * flight finish on the old generation, its graphs are re-captured for the
 * new one, and admission resumes; requests still queued at that point are
 * answered by the new generation.  Blocks until the switch is done; the old
 * handle is then no longer referenced and may be destroyed.  Returns 0,
 * 1 null argument or bad index, 2 geometry or device differs, 4 the loop
 * failed, 6 another swap of db is in progress. */
int ipir_serve_replace_db(ipir_serve* sv, size_t db, ipir_server* next);

/* One lane batch (in cyclic-scan mode: one group of requests admitted at
 * the same segment), for tracing. */
typedef struct {
    double t_issue_s;  /* steady (CLOCK_MONOTONIC) seconds when the batch was issued */
    float issue_ms;    /* host time to enqueue copies + graph replay (scan: admission, Horner and copies) */
    float device_ms;   /* device time of the batch, copies included (CUDA events; scan: admission to
                          response copy, the whole rotation) */
    float notice_ms;   /* bound on the delay from the batch's end to the worker handling it */
    uint16_t db, lane;
    uint32_t count;    /* queries in the batch */
    uint32_t failed;
} ipir_serve_batch_record;
/* Copies the most recent batches (up to max_records of the last 4096, oldest
 * first) into out; returns how many. */
size_t ipir_serve_trace(ipir_serve* sv, ipir_serve_batch_record* out, size_t max_records);
/* Waits for the batches on the device, fails requests not yet admitted,
 * frees everything. */
void ipir_serve_destroy(ipir_serve* sv);

/* ===================================================== part 4: group shards
 * One database split over several GPUs by contiguous group ranges (no
 * counterpart in the reference, which runs on one GPU: docs/ARCHITECTURE.md:32).
 * Each GPU holds a shard: its column slab of the encoded DB and its groups'
 * tensors; per batch it computes the b parts of its groups' packed
 * ciphertexts.  The caller gathers them (one collective, 2 N u32 per group
 * and query) to one GPU, whose Horner owner runs the chains.  The responses
 * equal ipir_answer_batch's on the whole database. */
typedef struct ipir_shard ipir_shard;
typedef struct ipir_horner ipir_horner;

/* Preprocesses groups [group_lo, group_hi) of the database
 * setup(n_entries, entry_bytes, db_rows_or_zero) on the current device; db is
 * the whole host DB (the encode mixes columns of several groups per row, so
 * it runs over full rows, chunk by chunk, and keeps the slab), crs_seed the
 * 64-byte CRS seed every shard shares (required).  out_params receives the
 * whole database's parameters.  NULL on failure (ipir_b200_last_error()). */
ipir_shard* ipir_b200_shard_create(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero, size_t max_batch,
                                   const uint16_t* db, const uint8_t* crs_seed, size_t group_lo, size_t group_hi,
                                   ipir_params* out_params);
/* The a parts of the shard's groups, host out[(group_hi - group_lo) * 2 * N]
 * u32 ([group][limb][coeff], NTT form), for the Horner owner's set-up. */
int ipir_b200_shard_export_a(const ipir_shard* shard, uint32_t* out);
/* The shard's part of a batch: mat-vec over its slab, tensor pass and
 * finalize of its groups for count <= max_batch queries (their LWE and KSK
 * parts are read, not their RGSW parts); writes the DEVICE buffer
 * out_packed_b[count][group_hi - group_lo][limb][N] u32 (b parts, NTT form).
 * Blocking.  Returns 0, 1 null argument, 2 count > max_batch, 3 null view
 * field, 4 CUDA error or device wait timeout. */
int ipir_b200_shard_pack(ipir_shard* shard, const ipir_query_view* queries, size_t count, uint32_t* out_packed_b);
/* For a database of several response ciphertexts, a shard whose groups
 * cover whole Horner chunks (group_lo a multiple of min(D, n_packed), and
 * group_hi one too or n_packed) answers its own ciphertexts with no
 * exchange: out_resp[count][its ciphertexts][a|b][limb][N] u64 (NTT form),
 * ciphertexts (group_lo / D_act) onward; a query's full response is the
 * shards' parts in group order.  Returns ipir_answer_batch's codes, or 6
 * when the range does not cover whole ciphertexts. */
int ipir_b200_shard_answer(ipir_shard* shard, const ipir_query_view* queries, size_t count, uint64_t* out_resp);
void ipir_b200_shard_destroy(ipir_shard* shard);

/* The Horner owner of a sharded database (params as ipir_b200_shard_create
 * returned them) on the current device; a_all: host [n_packed][limb][N] u32,
 * the shards' exported a parts in group order. */
ipir_horner* ipir_b200_horner_create(const ipir_params* params, const uint32_t* a_all, size_t max_batch);
/* Responses of count <= max_batch queries from the gathered b parts, DEVICE
 * packed_b[count][n_packed][limb][N] u32, and the queries' RGSW parts (only
 * those are read); out_resp as ipir_answer_batch's.  The work waits for what
 * `stream` (0: the legacy default stream) has enqueued, so packed_b may come
 * from a collective on that stream.  Blocking; returns 0, 1, 2, 3, 4 as
 * ipir_b200_shard_pack. */
int ipir_b200_horner_answer(ipir_horner* h, const uint32_t* packed_b, const ipir_query_view* queries, size_t count,
                            uint64_t* out_resp, void* stream);
void ipir_b200_horner_destroy(ipir_horner* h);

#ifdef __cplusplus
}
#endif
#endif /* INSPIRE_B200_H */
