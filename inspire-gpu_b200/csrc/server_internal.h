// server_internal.h -- server state shared by the per-handle entry points
// (server.cpp) and the serving loop (serve.cpp).  Not installed.
//
// A Server is one resident database: its preprocess output (Precomp), its
// derived geometry, one Lane of per-batch device scratch for the plain
// blocking entry points, and a schedule table (which mat-vec kernel, how
// many queries per tensor-pass GEMM, which Horner kernel) per batch size.
// The serving loop adds more Lanes over the same Precomp.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_util.h"
#include "inspire_b200.h"
#include "ipb_launch.h"

namespace ipb {

struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

[[noreturn]] void cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define IPB_CK(call)                                                            \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess) ::ipb::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

// Puts the calling thread's current device back on scope exit.  Entry points
// switch to their handle's device; a caller in a multi-GPU process keeps the
// device it had chosen, on error paths too.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    }
    ~DeviceRestore() {
        int cur = -1;
        if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev) cudaSetDevice(dev);
    }
    DeviceRestore(const DeviceRestore&) = delete;
    DeviceRestore& operator=(const DeviceRestore&) = delete;
};

// Device allocations freed together.
struct DevArena {
    std::vector<void*> ptrs;
    size_t bytes = 0;
    template <class T>
    T* alloc(size_t count) {
        void* p = nullptr;
        const size_t b = count * sizeof(T);
        IPB_CK(cudaMalloc(&p, b ? b : 16));
        ptrs.push_back(p);
        bytes += b;
        return static_cast<T*>(p);
    }
    void free_all() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
        bytes = 0;
    }
};

constexpr size_t kGroupStrideD = (size_t)2 * kSteps * kDeff * kN;  // u32 per group, D_plus / D_minus
constexpr size_t kGroupStrideF = (size_t)2 * kDeff * kN;
constexpr size_t kGroupStrideA = (size_t)2 * kN;
constexpr size_t kBlk = (size_t)kDeff * 2 * kN;                    // one KSK / RGSW part
constexpr size_t kKeyStride = 4 * kDeff * kN;                      // keys per query (u32)
constexpr size_t kRgswStride = 4 * kBlk;                           // rgsw32 per query (u32)

const DevTables& host_tables();
DevTables* upload_tables(DevArena& A, cudaStream_t s);

// Output of gpu_preprocess: the encoded DB and the precomputed tensors.
struct Precomp {
    Params pp{};
    int device = 0;
    DevArena arena;  // owns everything below
    DevTables* tables = nullptr;
    uint16_t* db = nullptr;
    uint32_t* pre_a = nullptr;
    uint8_t* pre_dt = nullptr;  // D_plus / D_minus as GEMM byte planes [l][i][g*4+a][4096]
    uint32_t* pre_df = nullptr;
    bool adopted = false;
    ~Precomp() {
        if (!adopted) {
            cudaSetDevice(device);
            arena.free_all();
        }
    }
};

// Kernel choices for one batch size.
struct Sched {
    int matvec_tc = 1;       // 1: tcgen05 int8 mat-vec, 0: CUDA-core mat-vec
    int tp_pass = 32;        // queries per tensor-pass GEMM (<= the lane's Gt capacity)
    int horner_cluster = 1;  // 1: 4-CTA cluster per chain, 2: 8-CTA cluster, 0: one CTA per chain
    int tp_sms = 0;          // > 0: tensor pass on this many SMs beside the tcgen05 mat-vec on the
                             // others (the lane's second stream); 0: tensor pass after the mat-vec
    int slice = 32;          // > 0: a batch larger than this runs as consecutive slices of this many
                             // queries, each its own pipeline (query prep .. Horner) on the lane's slots;
                             // 0: the whole batch in one pipeline
    int hchunks = 0;         // > 1: the tensor pass first, then the mat-vec and finalize in at most this
                             // many chunks of chain positions from the top down, each chunk's Horner steps
                             // on a second stream as soon as it is final (every ciphertext's chain of
                             // D_act groups, cluster Horner, tensor-core mat-vec, one slice); 0: off
};
constexpr int kMaxHChunks = 16;

// Queries per slice a batch is cut into (one DB pass of the tensor-core
// mat-vec serves at most this many) and the slices a batch of c needs.
constexpr size_t kSliceQueries = 32;
inline size_t slices_of(size_t c, const Sched& sc) {
    return sc.slice > 0 ? (c + (size_t)sc.slice - 1) / (size_t)sc.slice : 1;
}

// Per-batch device scratch for up to `cap` queries.
struct Lane {
    DevArena arena;
    size_t cap = 0;
    int gt_pass = 0;  // queries per tensor pass the key-table buffer holds
    uint64_t* qraw = nullptr;
    uint32_t* keys = nullptr;
    uint32_t* rgsw32 = nullptr;
    uint32_t* mvpart = nullptr;
    uint32_t* keyt = nullptr;    // per-pass key table the tensor-pass GEMM gathers its N operand from
    uint32_t* tp_out = nullptr;  // tensor-pass result [l][i][q][g]
    uint32_t* packed_b = nullptr;
    uint64_t* resp = nullptr;
    uint8_t* planes = nullptr;   // query byte planes for the tensor-core mat-vec
    int* d_err = nullptr;        // device error word (pipeline wait timeouts)
    unsigned* tiles = nullptr;   // work-item counters: [0] mat-vec, [1] tensor pass
    uint8_t* wire_in = nullptr;  // packed queries
    uint8_t* wire_out = nullptr; // packed or compressed responses
    uint32_t* codec_tmp = nullptr;  // coefficient-form responses for compression
    cudaStream_t aux = nullptr;     // second stream: the tensor pass beside the mat-vec
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t rgsw_ready = nullptr;  // RGSW parts staged and prepared on aux
    cudaStream_t hstream = nullptr;    // Horner chunks trailing the DB pass (Sched::hchunks)
    cudaEvent_t hjoin = nullptr;
    cudaEvent_t hev[kMaxHChunks] = {};  // chunk c's packed ciphertexts are final
    ~Lane() {
        for (auto& e : hev)
            if (e) cudaEventDestroy(e);
        if (hjoin) cudaEventDestroy(hjoin);
        if (hstream) cudaStreamDestroy(hstream);
        if (rgsw_ready) cudaEventDestroy(rgsw_ready);
        if (join) cudaEventDestroy(join);
        if (fork) cudaEventDestroy(fork);
        if (aux) cudaStreamDestroy(aux);
        arena.free_all();
    }
};

struct Server {
    Params pp{};
    int device = 0;
    size_t max_batch = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::shared_ptr<Precomp> pre;
    Lane lane;
    // geometry derived at setup
    size_t qstride = 0, mv_qstride = 0, pb_qstride = 0, resp_qstride = 0;
    size_t wire_q = 0, wire_r = 0, wire_c = 0;  // bytes per query: packed query, packed / compressed response
    int mv_chunks = 1;
    int num_sms = 148;
    int tc_kchunk_rows = 0, tc_kchunks = 1;
    // sched[c] for batch size c (index 0 unused); env overrides applied at setup
    std::vector<Sched> sched;
    bool tuned = false;
    size_t staged = 0;
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // 6 stage events per slice of the largest batch
    size_t timed_slices = 0;      // slices of the last batch run with stage timing
    float stage_ms[5] = {};
    size_t resident_bytes = 0;
    unsigned long long launches = 0;  // kernels launched through this handle's pipeline

    ~Server();
};

// Bytes of a lane of `cap` queries whose Gt holds `gt_pass` queries.
size_t lane_bytes(const Server& S, size_t cap, int gt_pass);
void alloc_lane(const Server& S, Lane& L, size_t cap, int gt_pass);
// Device buffers of a server's resident state (tables, DB, a, D byte planes,
// D_final) for P.pp, on P.device.
void alloc_precomp(Precomp& P, cudaStream_t s);
// A server handle over preprocessed (or restored) state.
Server* make_server(const Params& pp, std::shared_ptr<Precomp> pre, size_t max_batch);
void fill_params(const Params& pp, ipir_params* o);
// Pipeline phases: the DB-bound part (query prep, mat-vec, tensor pass,
// finalize) and the Horner chains.
constexpr int kPhaseDb = 1, kPhaseHorner = 2, kPhaseAll = 3;
// Enqueues the answer pipeline (the given phases) for `count` staged
// queries of lane L on stream st; returns the number of kernels launched.
// ev (6 stage events, used when all phases run) or null.
// ev holds n_ev events: 6 per slice (fewer than the batch's slices need: no
// stage events are recorded).
// db_done (optional): recorded once the DB-bound part is done (after the
// last finalize when the Horner chain trails the DB pass in chunks, else at
// the end), as an external event node under stream capture.
int run_pipeline(const Server& S, Lane& L, const Sched& sc, size_t count, cudaStream_t st, cudaEvent_t* ev,
                 int phases = kPhaseAll, size_t n_ev = 6, cudaEvent_t db_done = nullptr);
// Whether the pipeline for `count` queries under sc runs with the Horner
// chain trailing the DB pass in group chunks (then the DB and Horner phases
// cannot be run apart).
bool runs_chunked(const Server& S, const Sched& sc, size_t count);
// Device time (ms, best of three after one warm run) of one plain answer
// through the handle's own lane and schedule, on a stream of its own.
float time_plain_answer(Server& S);
// Cyclic-scan segment count the serving loop picks for a database whose
// plain answer takes `ms` (0: lane batches); see serve.cpp.
size_t auto_scan_segments(float ms);
// The DB-bound phase (query prep, mat-vec, tensor pass, finalize) of lane
// slots [q_off, q_off + count) on st: packed ciphertext b parts into
// L.packed_b.  lwe_ready: an event the mat-vec waits for (the key side runs
// first); qprep_parts: 3 keys and RGSW parts, 1 keys only.  Returns launches.
int run_db_phase(const Server& S, Lane& L, const Sched& sc, size_t q_off, size_t count, cudaStream_t st,
                 cudaEvent_t* ev, cudaEvent_t lwe_ready = nullptr, int qprep_parts = 3);
// H2D of parts [p0, p0 + np) (0, 1: LWE limbs, 2: KSK5, 3: KSK-1, 4: RGSW) of
// each query into the handle's lane, one copy per contiguous host run.
void stage_parts(const Server& S, const ipir_query_view* qs, size_t count, int p0, int np, cudaStream_t st);
// Waits for the work enqueued on st, then throws (and clears the word, on
// st) if a kernel's bounded wait ran out or a kernel stopped early.
void check_device_error(Lane& L, cudaStream_t st);
// Whether [g0, g1) covers whole Horner chunks (response ciphertexts).
bool shard_whole_cts(const Params& global, size_t g0, size_t g1);
// Geometry of the group shard [g0, g1) of a database (its column slab);
// for whole chunks its D and num_cts are those of its own ciphertexts.
Params shard_params(const Params& global, size_t g0, size_t g1);
// gpu_preprocess of the group shard [g0, g1) of the host DB db (global
// geometry): the encoded column slab and the shard's tensors.
std::shared_ptr<Precomp> run_preprocess_shard(const Params& global, const uint16_t* db, size_t g0, size_t g1);

// H2D of one flat query into query slot i of lane L.
void stage_query_flat(const Server& S, Lane& L, size_t i, const uint64_t* flat, cudaStream_t st);
// Schedule table (index = batch size, 0 unused) for a lane of `cap` queries
// whose Gt holds gt_pass: the handle's defaults (env overrides included).
std::vector<Sched> default_sched(const Server& S, size_t cap, int gt_pass);
// Measures candidate schedules per batch size on lane L; returns the table.
std::vector<Sched> autotune(const Server& S, Lane& L, cudaStream_t st);
// Sched for batch size c of the handle's own table.
const Sched& sched_for(const Server& S, size_t c);
// Queries per tensor-pass GEMM a lane of `cap` queries provisions Gt for.
int lane_gt_pass(const Server& S, size_t cap);

// Horner chains (variant sc.horner_cluster) of `count` queries whose
// packed ciphertexts, RGSW parts and responses start at the given pointers
// (per-query strides of S).
void enqueue_horner(const Server& S, const Sched& sc, const uint32_t* packed_b, const uint32_t* rgsw32,
                    uint64_t* resp, size_t count, int* err, cudaStream_t st);
// Query prep (keys, RGSW parts) of the flat queries in lane slots [s0, s0 + count).
void enqueue_qprep_slots(const Server& S, Lane& L, size_t s0, size_t count, cudaStream_t st);
// Lane query slots [s0, s0 + k).
struct SlotRun {
    size_t s0, k;
};
// One segment (seg of ns) of the cyclic scan for the queries in `runs`
// (their positions in this pass follow the order of runs): the tensor-core
// mat-vec over DB columns [seg C/ns, (seg + 1) C/ns) and the tensor pass
// over the (limb, slot) indices [seg 2N/ns, (seg + 1) 2N/ns), all groups,
// writing each query's mat-vec partials and tensor-pass rows under its own
// lane slot.  keys_pos: scratch for the keys in pass order (<= 32 queries).
// after_matvec (may be null) is recorded once the mat-vec is enqueued.
void enqueue_scan_segment(const Server& S, Lane& L, uint32_t* keys_pos, const std::vector<SlotRun>& runs, int seg,
                          int ns, cudaStream_t st, cudaEvent_t after_matvec);
// Finalize (all groups) of lane slots r after their ns segments: packed
// ciphertexts from the slots' mat-vec partials and tensor-pass rows.
void enqueue_scan_finalize(const Server& S, Lane& L, const SlotRun& r, cudaStream_t st);

}  // namespace ipb

// The C ABI handle (opaque in the public header).
struct ipir_server {
    ipb::Server* s;
};
