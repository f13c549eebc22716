// server.cpp -- host orchestration of the B200 InsPIRe server: preprocess,
// server context, answer pipeline, schedule autotuner, caps, and the C / C++
// entry points.
//
// Reference counterparts: src/gpu_protocol.cu (GpuServerCtx, gpu_preprocess,
// gpu_setup_server, answer_one, gpu_answer_batch, caps, free) and
// src/capi.cu (the C ABI server half).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "inspire_b200.h"
#include "inspire_b200.hpp"
#include "server_internal.h"

namespace ipb {

namespace {
thread_local std::string g_last_error;

uint32_t inv_mod_p(uint32_t d) {  // d^-1 mod 65535 (d a power of two)
    int64_t old_r = d, r = kP, old_s = 1, s = 0;
    while (r) {
        int64_t qq = old_r / r, t = r;
        r = old_r - qq * r; old_r = t;
        t = s; s = old_s - qq * s; old_s = t;
    }
    return (uint32_t)((old_s % (int64_t)kP + kP) % kP);
}
}  // namespace

[[noreturn]] void cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "CUDA error %d (%s) at %s:%d in %s", (int)e, cudaGetErrorString(e), file, line,
                  what);
    throw CudaFailure(buf);
}

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

const DevTables& host_tables() {
    static DevTables T;
    static std::once_flag once;
    std::call_once(once, [] { build_tables(T); });
    return T;
}

DevTables* upload_tables(DevArena& A, cudaStream_t s) {
    DevTables* d = A.alloc<DevTables>(1);
    IPB_CK(cudaMemcpyAsync(d, &host_tables(), sizeof(DevTables), cudaMemcpyHostToDevice, s));
    return d;
}

// gpu_preprocess (reference src/gpu_protocol.cu:535-817) on one stream.
void alloc_precomp(Precomp& P, cudaStream_t s) {
    const size_t R = P.pp.db_rows, C = P.pp.db_cols, G = P.pp.n_packed;
    DevArena& A = P.arena;
    P.tables = upload_tables(A, s);
    P.db = A.alloc<uint16_t>(R * C);
    P.pre_a = A.alloc<uint32_t>(G * kGroupStrideA);
    P.pre_dt = A.alloc<uint8_t>(tp_dt_bytes(G));
    P.pre_df = A.alloc<uint32_t>(G * kGroupStrideF);
}

// P.pp is the geometry P holds.  For a group shard (global != null), P.pp
// covers groups [g0, g0 + P.pp.n_packed) of the global database: the encode
// mixes the D_act column polynomials of each row block across groups, so it
// runs over full global rows (row chunks) and keeps the shard's column slab;
// every later stage is per group and runs on the slab alone.
static void preprocess_into(Precomp& P, const uint16_t* db_host, cudaStream_t s, const Params* global = nullptr,
                            size_t g0 = 0) {
    const Params& pp = P.pp;
    const size_t R = pp.db_rows, C = pp.db_cols, G = pp.n_packed;
    const Params& gp = global ? *global : pp;
    const size_t d_act = std::min(gp.D, gp.n_packed);
    const size_t Cg = gp.db_cols, col0 = g0 * kN;  // global width, first column of this slab
    alloc_precomp(P, s);

    DevArena tmp;
    try {
        // ---- encode (in-place inverse DFT over D_act column polys per row block)
        if (d_act <= 1) {
            IPB_CK(cudaMemcpy2DAsync(P.db, C * sizeof(uint16_t), db_host + col0, Cg * sizeof(uint16_t),
                                     C * sizeof(uint16_t), R, cudaMemcpyHostToDevice, s));
        } else if (global) {
            int logd = 0;
            while (((size_t)1 << logd) < d_act) ++logd;
            const int nlA = std::min(logd, 4), nlB = logd - nlA;
            const uint32_t dinv = inv_mod_p((uint32_t)d_act);
            const size_t row_bytes = Cg * sizeof(uint16_t);
            const size_t chunk_rows = std::max<size_t>(1, std::min<size_t>(R, (size_t)(256u << 20) / row_bytes));
            uint16_t* staging = tmp.alloc<uint16_t>(chunk_rows * Cg);
            uint16_t* enc = tmp.alloc<uint16_t>(chunk_rows * Cg);
            for (size_t r0 = 0; r0 < R; r0 += chunk_rows) {
                const size_t nr = std::min(chunk_rows, R - r0);
                IPB_CK(cudaMemcpyAsync(staging, db_host + r0 * Cg, nr * row_bytes, cudaMemcpyHostToDevice, s));
                IPB_CK(launch_encode_pass(staging, enc, nr, Cg, d_act, logd, 0, nlA, true, nlB == 0, dinv, s));
                if (nlB > 0)
                    IPB_CK(launch_encode_pass(nullptr, enc, nr, Cg, d_act, logd, nlA, nlB, false, true, dinv, s));
                IPB_CK(cudaMemcpy2DAsync(P.db + r0 * C, C * sizeof(uint16_t), enc + col0, row_bytes,
                                         C * sizeof(uint16_t), nr, cudaMemcpyDeviceToDevice, s));
            }
        } else {
            int logd = 0;
            while (((size_t)1 << logd) < d_act) ++logd;
            const int nlA = std::min(logd, 4), nlB = logd - nlA;
            const uint32_t dinv = inv_mod_p((uint32_t)d_act);
            const size_t row_bytes = C * sizeof(uint16_t);
            const size_t chunk_rows = std::max<size_t>(1, std::min<size_t>(R, (size_t)(256u << 20) / row_bytes));
            uint16_t* staging = tmp.alloc<uint16_t>(chunk_rows * C);
            for (size_t r0 = 0; r0 < R; r0 += chunk_rows) {
                const size_t nr = std::min(chunk_rows, R - r0);
                IPB_CK(cudaMemcpyAsync(staging, db_host + r0 * C, nr * row_bytes, cudaMemcpyHostToDevice, s));
                IPB_CK(launch_encode_pass(staging, P.db + r0 * C, nr, C, d_act, logd, 0, nlA, true, nlB == 0, dinv, s));
                if (nlB > 0)
                    IPB_CK(launch_encode_pass(nullptr, P.db + r0 * C, nr, C, d_act, logd, nlA, nlB, false, true, dinv, s));
            }
        }
        // ---- CRS polys a~_r = NTT(tau_{2N-1}(expand_seed("rlwe", r)))  (src/gpu_protocol.cu:569-582)
        const size_t n_r = R / kN;
        std::vector<uint32_t> h_crs(n_r * 2 * kN);
        {
            std::vector<uint32_t> a(2 * kN);
            for (size_t r = 0; r < n_r; ++r) {
                expand_seed(pp.seed, "rlwe", r, a.data());
                for (int l = 0; l < 2; ++l) {
                    const uint32_t q = l ? kQ1 : kQ0;
                    uint32_t* o = h_crs.data() + (r * 2 + l) * kN;
                    const uint32_t* in = a.data() + (size_t)l * kN;
                    o[0] = in[0];
                    for (size_t i = 1; i < (size_t)kN; ++i) o[i] = in[kN - i] ? q - in[kN - i] : 0;
                }
            }
        }
        uint32_t* crs = tmp.alloc<uint32_t>(n_r * 2 * kN);
        IPB_CK(cudaMemcpyAsync(crs, h_crs.data(), h_crs.size() * 4, cudaMemcpyHostToDevice, s));
        IPB_CK(launch_ntt_batch(crs, 2 * n_r, 1, false, P.tables, s));
        // ---- ExpandKSK_a sources: K5[j] = expand_seed("ksk", 5*100+j+1), Kn1[j] with (2N-1)*100+j+1
        //      layout [key][limb][digit][N], NTT form (src/gpu_protocol.cu:364-474)
        std::vector<uint32_t> h_k(2 * 2 * kDeff * kN);
        {
            std::vector<uint32_t> a(2 * kN);
            for (int key = 0; key < 2; ++key)
                for (int j = 0; j < kDeff; ++j) {
                    const uint64_t idx = key == 0 ? 5ull * 100 + j + 1 : (uint64_t)(2 * kN - 1) * 100 + j + 1;
                    expand_seed(pp.seed, "ksk", idx, a.data());
                    for (int l = 0; l < 2; ++l)
                        std::memcpy(h_k.data() + (((size_t)key * 2 + l) * kDeff + j) * kN, a.data() + (size_t)l * kN,
                                    kN * 4);
                }
        }
        uint32_t* kk = tmp.alloc<uint32_t>(h_k.size());
        IPB_CK(cudaMemcpyAsync(kk, h_k.data(), h_k.size() * 4, cudaMemcpyHostToDevice, s));
        IPB_CK(launch_ntt_batch(kk, 2 * 2 * kDeff, kDeff, false, P.tables, s));
        const uint32_t* k5 = kk;
        const uint32_t* kn1 = kk + 2 * kDeff * kN;
        // ---- per group: a-side -> column NTTs -> ring-embed gather; CollapseA in waves
        uint32_t* V = tmp.alloc<uint32_t>((size_t)2 * kN * kN);
        uint32_t* Tm = tmp.alloc<uint32_t>((size_t)2 * kN * kN);
        const size_t ap_gstride = (size_t)kHalf * 2 * 2 * kN;
        const size_t wave = std::min<size_t>(G, 64);
        uint32_t* a_post = tmp.alloc<uint32_t>(wave * ap_gstride);
        uint32_t* ends = tmp.alloc<uint32_t>(wave * 2 * 2 * kN);
        uint32_t* dp_w = tmp.alloc<uint32_t>(wave * kGroupStrideD);  // D in the reference layout, one wave
        uint32_t* dm_w = tmp.alloc<uint32_t>(wave * kGroupStrideD);
        for (size_t w0 = 0; w0 < G; w0 += wave) {
            const size_t nw = std::min(wave, G - w0);
            for (size_t g = w0; g < w0 + nw; ++g) {
                IPB_CK(launch_a_side(P.db, R, C, g, crs, P.tables, V, s));
                IPB_CK(launch_col_ntt(V, P.tables, Tm, s));
                IPB_CK(launch_embed_gather(Tm, a_post + (g - w0) * ap_gstride, s));
            }
            IPB_CK(launch_collapse_a(a_post, ap_gstride, k5, P.tables, dp_w, dm_w, ends, nw, s));
            IPB_CK(launch_dt_transpose(dp_w, dm_w, w0, nw, G, P.pre_dt, s));
            IPB_CK(launch_collapse_final(ends, kn1, P.tables, P.pre_df + w0 * kGroupStrideF,
                                         P.pre_a + w0 * kGroupStrideA, nw, s));
        }
        IPB_CK(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        tmp.free_all();
        throw;
    }
    tmp.free_all();
}

// --------------------------------------------------------------- server
Server::~Server() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    lane.arena.free_all();
    if (pre) {
        pre->adopted = false;  // Precomp frees the DB and tensors
        pre.reset();
    }
    if (own_stream) cudaStreamDestroy(own_stream);
}

static int pick_pow2_chunks(size_t target, size_t maxv) {
    size_t c = 1;
    while (c < target && c * 2 <= maxv) c *= 2;
    return (int)c;
}

size_t lane_bytes(const Server& S, size_t cap, int gt_pass) {
    const size_t R = S.pp.db_rows, G = S.pp.n_packed;
    return cap * S.qstride * 8 + cap * kKeyStride * 4 + cap * kRgswStride * 4 + cap * S.mv_qstride * 4 +
           tp_keyt_bytes(gt_pass) + (size_t)2 * kN * cap * G * 4 + cap * S.pb_qstride * 4 + cap * S.resp_qstride * 8 +
           mv_tc_planes_bytes(R, (int)cap) + sizeof(int) + 2 * sizeof(unsigned) + cap * S.wire_q +
           cap * std::max(S.wire_r, S.wire_c) + cap * S.pp.num_cts * 4 * kN * 4;
}

void alloc_lane(const Server& S, Lane& L, size_t cap, int gt_pass) {
    const size_t R = S.pp.db_rows, G = S.pp.n_packed;
    DevArena& A = L.arena;
    L.cap = cap;
    L.gt_pass = gt_pass;
    L.qraw = A.alloc<uint64_t>(cap * S.qstride);
    L.keys = A.alloc<uint32_t>(cap * kKeyStride);
    L.rgsw32 = A.alloc<uint32_t>(cap * kRgswStride);
    L.mvpart = A.alloc<uint32_t>(cap * S.mv_qstride);
    L.keyt = A.alloc<uint32_t>(tp_keyt_bytes(gt_pass) / 4);
    L.tp_out = A.alloc<uint32_t>((size_t)2 * kN * cap * G);
    L.packed_b = A.alloc<uint32_t>(cap * S.pb_qstride);
    L.resp = A.alloc<uint64_t>(cap * S.resp_qstride);
    L.planes = A.alloc<uint8_t>(mv_tc_planes_bytes(R, (int)cap));
    L.d_err = A.alloc<int>(1);
    L.tiles = A.alloc<unsigned>(2);
    L.wire_in = A.alloc<uint8_t>(cap * S.wire_q);
    L.wire_out = A.alloc<uint8_t>(cap * std::max(S.wire_r, S.wire_c));
    L.codec_tmp = A.alloc<uint32_t>(cap * S.pp.num_cts * 4 * kN);
    IPB_CK(cudaStreamCreateWithFlags(&L.aux, cudaStreamNonBlocking));
    IPB_CK(cudaEventCreateWithFlags(&L.fork, cudaEventDisableTiming));
    IPB_CK(cudaEventCreateWithFlags(&L.join, cudaEventDisableTiming));
    IPB_CK(cudaEventCreateWithFlags(&L.rgsw_ready, cudaEventDisableTiming));
    IPB_CK(cudaStreamCreateWithFlags(&L.hstream, cudaStreamNonBlocking));
    IPB_CK(cudaEventCreateWithFlags(&L.hjoin, cudaEventDisableTiming));
    for (auto& e : L.hev) IPB_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // Defined contents before any pipeline run (the autotuner runs on them).
    IPB_CK(cudaMemset(L.qraw, 0, cap * S.qstride * 8));
    IPB_CK(cudaMemset(L.planes, 0, mv_tc_planes_bytes(R, (int)cap)));
    IPB_CK(cudaMemset(L.d_err, 0, sizeof(int)));
    // The lanes run on non-blocking streams, which do not wait for the
    // legacy stream the memsets above went to.
    IPB_CK(cudaDeviceSynchronize());
}

Server* make_server(const Params& pp, std::shared_ptr<Precomp> pre, size_t max_batch) {
    if (max_batch == 0) throw std::invalid_argument("gpu_setup_server: max_batch must be >= 1");
    if (!pre || pre->adopted) throw std::invalid_argument("gpu_setup_server: preprocess data missing or adopted");
    auto S = std::make_unique<Server>();
    S->pp = pp;
    S->device = pre->device;
    IPB_CK(cudaSetDevice(S->device));
    S->max_batch = max_batch;
    IPB_CK(cudaStreamCreateWithFlags(&S->own_stream, cudaStreamNonBlocking));
    S->stream = S->own_stream;
    const size_t R = pp.db_rows, C = pp.db_cols, G = pp.n_packed;
    S->qstride = 2 * R + 6 * kBlk;
    const size_t tiles = C / 2048;
    S->mv_chunks = pick_pow2_chunks((592 + tiles - 1) / tiles, std::max<size_t>(1, R / 256));
    // <= 4096 rows per chunk keeps the staged query words (4 queries x 2
    // limbs x rows x 4 B) within 128 KB of shared memory.
    while (R / (size_t)S->mv_chunks > 4096) S->mv_chunks *= 2;
    IPB_CK(cudaDeviceGetAttribute(&S->num_sms, cudaDevAttrMultiProcessorCount, S->device));
    S->tc_kchunk_rows = matvec_tc_kchunk_rows(R, C, S->num_sms);
    S->tc_kchunks = (int)(R / (size_t)S->tc_kchunk_rows);
    S->mv_qstride = (size_t)std::max(S->mv_chunks, S->tc_kchunks) * 2 * C;
    S->pb_qstride = G * 2 * kN;
    S->resp_qstride = pp.num_cts * 4 * kN;
    S->wire_q = wire_query_bytes(R);
    S->wire_r = wire_response_bytes(pp.num_cts);
    S->wire_c = wire_compressed_bytes(pp.num_cts);
    const int gt_pass = lane_gt_pass(*S, max_batch);
    S->sched = default_sched(*S, max_batch, gt_pass);
    alloc_lane(*S, S->lane, max_batch, gt_pass);
    S->ev.assign(6 * ((max_batch + kSliceQueries - 1) / kSliceQueries), nullptr);
    for (auto& e : S->ev) IPB_CK(cudaEventCreate(&e));
    pre->adopted = true;
    S->resident_bytes = pre->arena.bytes + S->lane.arena.bytes;
    S->pre = std::move(pre);
    return S.release();
}

void stage_query_flat(const Server& S, Lane& L, size_t i, const uint64_t* flat, cudaStream_t st) {
    IPB_CK(cudaMemcpyAsync(L.qraw + i * S.qstride, flat, S.qstride * 8, cudaMemcpyHostToDevice, st));
}

// The five parts of each query land back to back in the lane's flat query
// buffer.  Parts that also sit back to back in host memory (a flat query, or
// a batch of them in one array, as the reference client's flattening lays
// them out) go in one copy: one cudaMemcpyAsync per contiguous run instead
// of five per query, which matters at 32 queries per batch.
static void stage_queries(Server* S, const ipir_query_view* qs, size_t count) {
    IPB_CK(cudaSetDevice(S->device));
    const size_t R = S->pp.db_rows;
    uint64_t* d = S->lane.qraw;
    const uint64_t* run = nullptr;  // host start of the pending run
    size_t run_len = 0;             // its length in u64
    auto part = [&](const uint64_t* src, size_t n) {
        if (run && src == run + run_len) {
            run_len += n;
            return;
        }
        if (run) IPB_CK(cudaMemcpyAsync(d, run, run_len * 8, cudaMemcpyHostToDevice, S->stream));
        d += run_len;
        run = src;
        run_len = n;
    };
    for (size_t i = 0; i < count; ++i) {
        const ipir_query_view& v = qs[i];
        part(v.lwe_b_limb0, R);
        part(v.lwe_b_limb1, R);
        part(v.ksk5_b, kBlk);
        part(v.kskneg1_b, kBlk);
        part(v.rgsw, 4 * kBlk);
    }
    if (run) IPB_CK(cudaMemcpyAsync(d, run, run_len * 8, cudaMemcpyHostToDevice, S->stream));
    S->staged = count;
}

// Host -> device copy of parts [p0, p0 + np) of every query (0, 1: the LWE
// limbs; 2, 3, 4: KSK5, KSK-1, RGSW) into their place in the lane's flat
// query buffer.  One 2-D copy when each query's parts are back to back in
// host memory at a constant stride between queries (a flat batch array),
// else one copy per host-contiguous run.
void stage_parts(const Server& S, const ipir_query_view* qs, size_t count, int p0, int np, cudaStream_t st) {
    const size_t R = S.pp.db_rows;
    const size_t len[5] = {R, R, kBlk, kBlk, 4 * kBlk};
    const size_t off[5] = {0, R, 2 * R, 2 * R + kBlk, 2 * R + 2 * kBlk};
    auto ptr = [&](size_t i, int p) -> const uint64_t* {
        const ipir_query_view& v = qs[i];
        return p == 0 ? v.lwe_b_limb0 : p == 1 ? v.lwe_b_limb1 : p == 2 ? v.ksk5_b : p == 3 ? v.kskneg1_b : v.rgsw;
    };
    size_t width = 0;
    for (int p = p0; p < p0 + np; ++p) width += len[p];
    bool strided = true;
    for (size_t i = 0; i < count && strided; ++i) {
        for (int p = p0 + 1; p < p0 + np; ++p) strided = strided && ptr(i, p) == ptr(i, p - 1) + len[p - 1];
        if (i > 0) strided = strided && ptr(i, p0) - ptr(i - 1, p0) == ptr(1, p0) - ptr(0, p0);
    }
    if (strided && count > 1 && ptr(1, p0) - ptr(0, p0) >= (ptrdiff_t)width) {
        IPB_CK(cudaMemcpy2DAsync(S.lane.qraw + off[p0], S.qstride * 8, ptr(0, p0), (ptr(1, p0) - ptr(0, p0)) * 8,
                                 width * 8, count, cudaMemcpyHostToDevice, st));
        return;
    }
    for (size_t i = 0; i < count; ++i) {
        uint64_t* d = S.lane.qraw + i * S.qstride + off[p0];
        const uint64_t* run = ptr(i, p0);
        size_t run_len = len[p0];
        for (int p = p0 + 1; p <= p0 + np; ++p) {
            if (p < p0 + np && ptr(i, p) == run + run_len) {
                run_len += len[p];
                continue;
            }
            IPB_CK(cudaMemcpyAsync(d, run, run_len * 8, cudaMemcpyHostToDevice, st));
            d += run_len;
            if (p < p0 + np) {
                run = ptr(i, p);
                run_len = len[p];
            }
        }
    }
}

const Sched& sched_for(const Server& S, size_t c) { return S.sched[std::min(c, S.sched.size() - 1)]; }

int lane_gt_pass(const Server& S, size_t cap) {
    return (int)std::min<size_t>(cap, (size_t)tp_pass_queries(S.pp.n_packed));
}

static bool chunked_ok(const Server& S, const Sched& sc, size_t count);

std::vector<Sched> default_sched(const Server& S, size_t cap, int gt_pass) {
    Sched def;
    def.tp_pass = gt_pass;
    if (const char* m = std::getenv("IPB_MATVEC")) def.matvec_tc = std::strcmp(m, "simt") != 0;
    if (const char* h = std::getenv("IPB_HORNER"))
        def.horner_cluster = std::strcmp(h, "cta") == 0 ? 0 : (std::strcmp(h, "cl8") == 0 ? 2 : 1);
    if (const char* t = std::getenv("IPB_TP_SMS"))
        def.tp_sms = def.matvec_tc ? std::max(0, std::min(std::atoi(t), S.num_sms - 1)) : 0;
    std::vector<Sched> out(cap + 1, def);
    // The Horner chain trails the DB pass in chunks by default where the
    // geometry allows it, the chain is long enough to matter (at least 32
    // groups per response ciphertext) and the batch has at most chain / 16
    // queries (at most 16): the hidden chain then outweighs the extra
    // launches.  Measured: 128 groups
    // 2-8 % faster from 1 to 16 queries; 32 groups 4.5 % faster at 1 query
    // and 1 % slower at 8; 8 groups 4-9 % slower.  IPB_HCHUNKS sets it for
    // every batch size.
    const size_t chain = std::min(S.pp.D, S.pp.n_packed);  // groups per response ciphertext
    for (size_t c = 1; c <= cap; ++c) {
        Sched probe = def;
        probe.hchunks = 8;
        if (chain >= 32 && c <= std::min<size_t>(16, chain / 16) && chunked_ok(S, probe, c)) out[c].hchunks = 8;
    }
    if (const char* h = std::getenv("IPB_HCHUNKS"))
        for (auto& sc : out) sc.hchunks = std::max(0, std::min(std::atoi(h), kMaxHChunks));
    return out;
}

// Query prep, mat-vec, tensor pass, finalize: the part that streams the DB
// and the precomputed tensors.
// lwe_ready (optional): the queries' LWE vectors arrive later than their
// key parts (copied on another stream, this event marks them); the key side
// (query prep, tensor pass) then runs first and the mat-vec after the event.
// The RGSW parts are then prepared on that other stream as well.
// q_off: the batch's first lane slot (slices of a batch larger than one DB
// pass run the whole phase on slots [q_off, q_off + count)); the tensor-pass
// rows (tp_out) and key table are shared by slices run one after the other.
// qprep_parts: 3 prepares keys and RGSW parts here, 1 the keys only (the
// RGSW parts are prepared elsewhere).
int run_db_phase(const Server& S, Lane& L, const Sched& sc, size_t q_off, size_t count, cudaStream_t st,
                 cudaEvent_t* ev, cudaEvent_t lwe_ready, int qprep_parts) {
    const Params& pp = S.pp;
    const Precomp& P = *S.pre;
    const size_t R = pp.db_rows, C = pp.db_cols, G = pp.n_packed;
    const int nq = (int)count;
    uint64_t* const qraw = L.qraw + q_off * S.qstride;
    uint32_t* const keys = L.keys + q_off * kKeyStride;
    uint32_t* const mvpart = L.mvpart + q_off * S.mv_qstride;
    uint8_t* const planes = L.planes + mv_tc_planes_offset(q_off, R);
    int launches = 0;
    if (ev) IPB_CK(cudaEventRecord(ev[0], st));
    IPB_CK(launch_qprep_parts(qraw, S.qstride, R, P.tables, keys, L.rgsw32 + q_off * kRgswStride, nq, qprep_parts,
                              st));
    ++launches;
    if (ev) IPB_CK(cudaEventRecord(ev[1], st));
    // Beside: the tensor pass (keys only) on sc.tp_sms SMs from the lane's
    // second stream while the mat-vec (DB only) runs on the other SMs; the
    // two persistent kernels take one CTA per SM each, so the split holds.
    const bool beside = sc.matvec_tc && sc.tp_sms > 0 && sc.tp_sms < S.num_sms;
    auto tensor_pass = [&](cudaStream_t ts, int sms) {
        for (size_t c0 = 0; c0 < count; c0 += (size_t)sc.tp_pass) {
            const int n = (int)std::min<size_t>((size_t)sc.tp_pass, count - c0);
            IPB_CK(launch_tensor_pass(P.pre_dt, G, keys + c0 * kKeyStride, kKeyStride, n, nq, (int)c0, L.keyt,
                                      L.tp_out, L.d_err, L.tiles + 1, sms, ts));
            launches += 2;  // key table + GEMM
        }
    };
    if (beside) {
        IPB_CK(cudaEventRecord(L.fork, st));
        IPB_CK(cudaStreamWaitEvent(L.aux, L.fork, 0));
        tensor_pass(L.aux, sc.tp_sms);
        IPB_CK(cudaEventRecord(L.join, L.aux));
    }
    if (lwe_ready && !beside) {
        tensor_pass(st, S.num_sms);
        IPB_CK(cudaStreamWaitEvent(st, lwe_ready, 0));
    }
    int mv_parts;
    if (sc.matvec_tc) {
        IPB_CK(launch_qplanes(qraw, S.qstride, R, P.tables, planes, nq, st));
        ++launches;
        for (size_t c0 = 0; c0 < count; c0 += 32) {
            const int n = (int)std::min<size_t>(32, count - c0);
            IPB_CK(launch_matvec_tc(P.db, R, C, planes + mv_tc_planes_offset(c0, R), n, P.tables,
                                    mvpart + c0 * S.mv_qstride, S.mv_qstride, L.d_err, L.tiles,
                                    beside ? S.num_sms - sc.tp_sms : S.num_sms, S.tc_kchunk_rows, st));
            ++launches;
        }
        mv_parts = S.tc_kchunks;
    } else {
        for (size_t c0 = 0; c0 < count; c0 += 4) {
            const int n = (int)std::min<size_t>(4, count - c0);
            IPB_CK(launch_matvec(P.db, R, C, S.mv_chunks, qraw + c0 * S.qstride, S.qstride, P.tables,
                                 mvpart + c0 * S.mv_qstride, S.mv_qstride, n, st));
            ++launches;
        }
        mv_parts = S.mv_chunks;
    }
    if (beside)
        IPB_CK(cudaStreamWaitEvent(st, L.join, 0));  // stage times: mat-vec = both, tensor pass = 0
    if (ev) IPB_CK(cudaEventRecord(ev[2], st));
    if (!beside && !lwe_ready) tensor_pass(st, S.num_sms);
    if (ev) IPB_CK(cudaEventRecord(ev[3], st));
    IPB_CK(launch_finalize(mvpart, S.mv_qstride, mv_parts, C, L.tp_out, P.pre_df, keys, kKeyStride, P.tables,
                           L.packed_b + q_off * S.pb_qstride, S.pb_qstride, G, nq, st));
    return launches + 1;
}

static int run_horner_phase(const Server& S, Lane& L, const Sched& sc, size_t q_off, size_t count, cudaStream_t st,
                            cudaEvent_t* ev) {
    if (ev) IPB_CK(cudaEventRecord(ev[4], st));
    enqueue_horner(S, sc, L.packed_b + q_off * S.pb_qstride, L.rgsw32 + q_off * kRgswStride,
                   L.resp + q_off * S.resp_qstride, count, L.d_err, st);
    if (ev) IPB_CK(cudaEventRecord(ev[5], st));
    return 1;
}

// Whether a batch of `count` can run with its Horner chunks trailing the DB
// pass (Sched::hchunks): every response ciphertext's chain of the same
// length (one ciphertext, or G a multiple of D), one slice, the tensor-core
// mat-vec and a cluster Horner kernel (those resume a chain from memory).
static bool chunked_ok(const Server& S, const Sched& sc, size_t count) {
    const size_t G = S.pp.n_packed, d_act = std::min(S.pp.D, G);
    // every response ciphertext's chain covers d_act >= 2 groups (no short last one)
    return sc.hchunks > 1 && sc.matvec_tc && sc.horner_cluster != 0 && sc.tp_sms == 0 &&
           G == S.pp.num_cts * d_act && d_act >= 2 && count <= kSliceQueries;
}

bool runs_chunked(const Server& S, const Sched& sc, size_t count) { return chunked_ok(S, sc, count); }

float time_plain_answer(Server& S) {
    IPB_CK(cudaSetDevice(S.device));
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    IPB_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float best = 1e30f;
    try {
        IPB_CK(cudaEventCreate(&e0));
        IPB_CK(cudaEventCreate(&e1));
        IPB_CK(cudaStreamSynchronize(S.stream));  // the lane's last use is done
        const Sched& sc = sched_for(S, 1);
        run_pipeline(S, S.lane, sc, 1, st, nullptr);  // warm
        for (int r = 0; r < 3; ++r) {
            IPB_CK(cudaEventRecord(e0, st));
            run_pipeline(S, S.lane, sc, 1, st, nullptr);
            IPB_CK(cudaEventRecord(e1, st));
            IPB_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            IPB_CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaStreamDestroy(st);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    return best;
}

size_t auto_scan_segments(float ms) {
    // A database whose plain answer takes at least 2 ms (IPB_SCAN_AUTO_MS
    // overrides the threshold) joins requests at segments of about 1 ms:
    // the power of two nearest to ms / 1 ms, 2 .. 16.  Measured: the 16 GB
    // database (about 4 ms) serves with a p99 of 1.6-1.7 plain answers in 4
    // segments at 3 and 5 times the plain rate, while 1 GB databases (0.4-0.5
    // ms) keep a lower median on lane batches (0.49 vs 0.67 ms).
    float threshold = 2.0f;
    if (const char* t = std::getenv("IPB_SCAN_AUTO_MS")) threshold = (float)std::atof(t);
    if (!(ms >= threshold)) return 0;
    size_t ns = 2;
    while (ns < 16 && (float)(2 * ns) <= ms * 1.41421356f) ns *= 2;
    return ns;
}

// An event record that becomes an external event node (observable outside
// the graph) when st is being captured.
static void record_outside(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    IPB_CK(cudaStreamIsCapturing(st, &cs));
    IPB_CK(cudaEventRecordWithFlags(e, st, cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0));
}

// Group chunks of the chunked pipeline, top chunk first, at most `cap`.  A
// chunk's Horner steps run beside the next chunk's DB pass, where the chain
// takes about 11 us per group (2.5 times its rate alone: its loads meet a
// saturated memory system) against the DB pass's 18 us per group at 16 GB,
// and the last chunk's steps follow the DB pass.  So the chunks are whole
// waves of mat-vec work items (floor(w x groups per wave) groups; a partial
// wave costs nearly a whole one, since the persistent mat-vec's last items
// set its end), one wave at the bottom and one wave more per chunk going
// up, at most four, the top chunk taking the rest: at 128 groups and 148
// SMs 37 + 37 + 27 + 18 + 9 (14 waves, as many as one unchunked pass).
static std::vector<size_t> chunk_sizes(size_t G, size_t ipg, int num_sms, size_t cap) {
    const double per_wave = (double)num_sms / (double)ipg;
    std::vector<size_t> up;  // bottom chunk first
    size_t rest = G;
    for (size_t w = 1; rest > 0 && up.size() + 1 < cap; w = std::min<size_t>(w + 1, 4)) {
        const size_t n = std::min(rest, std::max<size_t>(1, (size_t)((double)w * per_wave)));
        up.push_back(n);
        rest -= n;
    }
    if (rest > 0) up.push_back(rest);
    return std::vector<size_t>(up.rbegin(), up.rend());
}

// The plain pipeline with the Horner chain trailing the DB pass.  The
// tensor pass runs first for all groups; then the mat-vec and finalize run
// in chunks of groups (chunk_sizes) from the top group down, and as soon as
// a chunk's packed ciphertexts are final its Horner steps run on the lane's
// Horner stream, which resumes the chain from the accumulators of the
// previous chunk (kept in the lane's codec buffer, unused until the
// pipeline ends).  The chain consumes groups from the top (acc =
// packed[G - 1], then i = G - 2 .. 0), so it follows the DB pass instead of
// waiting for all of it.  Same kernels and the same arithmetic: identical
// responses.  The mat-vec keeps every SM: its tiles are handed out from a
// counter, so a Horner cluster that takes a few SMs first only shifts their
// tiles to the other CTAs (keeping SMs free for the clusters measured no
// faster).
// lwe_ready / rgsw_ready (optional): the blocking path's copies, on other
// streams, of the LWE vectors (the mat-vec waits) and of the prepared RGSW
// parts (the first Horner chunk waits).  qprep_parts as run_db_phase's.
static int run_chunked(const Server& S, Lane& L, const Sched& sc, size_t count, cudaStream_t st,
                       cudaEvent_t lwe_ready = nullptr, cudaEvent_t rgsw_ready = nullptr, int qprep_parts = 3,
                       cudaEvent_t db_done = nullptr) {
    const Params& pp = S.pp;
    const Precomp& P = *S.pre;
    const size_t R = pp.db_rows, C = pp.db_cols, G = pp.n_packed;
    const int nq = (int)count;
    int launches = 0;
    IPB_CK(launch_qprep_parts(L.qraw, S.qstride, R, P.tables, L.keys, L.rgsw32, nq, qprep_parts, st));
    ++launches;
    for (size_t c0 = 0; c0 < count; c0 += (size_t)sc.tp_pass) {
        const int n = (int)std::min<size_t>((size_t)sc.tp_pass, count - c0);
        IPB_CK(launch_tensor_pass(P.pre_dt, G, L.keys + c0 * kKeyStride, kKeyStride, n, nq, (int)c0, L.keyt,
                                  L.tp_out, L.d_err, L.tiles + 1, S.num_sms, st));
        launches += 2;
    }
    if (lwe_ready) IPB_CK(cudaStreamWaitEvent(st, lwe_ready, 0));
    IPB_CK(launch_qplanes(L.qraw, S.qstride, R, P.tables, L.planes, nq, st));
    ++launches;
    // Chunks are ranges [lo, hi) of chain positions, the same in every
    // response ciphertext (ciphertext t's groups t * d_act + [lo, hi)): one
    // mat-vec launch covers the range in all of them.
    const size_t nct = pp.num_cts, d_act = std::min(pp.D, G);
    const size_t ipg = (kN / (size_t)matvec_tc_item_cols()) * (size_t)S.tc_kchunks * nct;
    const std::vector<size_t> sizes =
        chunk_sizes(d_act, ipg, S.num_sms, std::min<size_t>((size_t)sc.hchunks, kMaxHChunks));
    IPB_CK(cudaEventRecord(L.hjoin, st));               // the Horner stream starts after this batch's prep
    IPB_CK(cudaStreamWaitEvent(L.hstream, L.hjoin, 0));
    if (rgsw_ready) IPB_CK(cudaStreamWaitEvent(L.hstream, rgsw_ready, 0));
    uint32_t* state = L.codec_tmp;
    size_t hi = d_act;
    for (size_t c = 0; c < sizes.size(); hi -= sizes[c], ++c) {
        const size_t lo = hi - sizes[c];
        IPB_CK(launch_matvec_tc_ranges(P.db, R, C, lo * kN, (hi - lo) * kN, (int)nct, d_act * kN, L.planes, nq,
                                       P.tables, L.mvpart, S.mv_qstride, nullptr, L.d_err, L.tiles, S.num_sms,
                                       S.tc_kchunk_rows, st));
        for (size_t t = 0; t < nct; ++t) {
            IPB_CK(launch_finalize_range(L.mvpart, S.mv_qstride, S.tc_kchunks, C, L.tp_out, nq, 0, P.pre_df, L.keys,
                                         kKeyStride, P.tables, L.packed_b, S.pb_qstride, G, t * d_act + lo, hi - lo,
                                         nq, st));
            ++launches;
        }
        IPB_CK(cudaEventRecord(L.hev[c], st));
        IPB_CK(cudaStreamWaitEvent(L.hstream, L.hev[c], 0));
        HornerRange hr;
        hr.i_first = c == 0 ? -1 : (long)hi - 1;
        hr.i_last = (long)lo;
        hr.state = state;
        if (sc.horner_cluster == 2)
            IPB_CK(launch_horner_cluster8(P.pre_a, L.packed_b, S.pb_qstride, L.rgsw32, P.tables, G, d_act, nct,
                                          L.resp, S.resp_qstride, nq, L.d_err, L.hstream, hr));
        else
            IPB_CK(launch_horner_cluster(P.pre_a, L.packed_b, S.pb_qstride, L.rgsw32, P.tables, G, d_act, nct,
                                         L.resp, S.resp_qstride, nq, L.d_err, L.hstream, hr));
        launches += 2;
    }
    if (db_done) record_outside(db_done, st);
    IPB_CK(cudaEventRecord(L.hjoin, L.hstream));
    IPB_CK(cudaStreamWaitEvent(st, L.hjoin, 0));
    return launches;
}

void enqueue_horner(const Server& S, const Sched& sc, const uint32_t* packed_b, const uint32_t* rgsw32,
                    uint64_t* resp, size_t count, int* err, cudaStream_t st) {
    const Params& pp = S.pp;
    const Precomp& P = *S.pre;
    const size_t G = pp.n_packed, d_act = std::min(pp.D, G);
    const int nq = (int)count;
    if (sc.horner_cluster == 2)
        IPB_CK(launch_horner_cluster8(P.pre_a, packed_b, S.pb_qstride, rgsw32, P.tables, G, d_act, pp.num_cts, resp,
                                      S.resp_qstride, nq, err, st));
    else if (sc.horner_cluster)
        IPB_CK(launch_horner_cluster(P.pre_a, packed_b, S.pb_qstride, rgsw32, P.tables, G, d_act, pp.num_cts, resp,
                                     S.resp_qstride, nq, err, st));
    else
        IPB_CK(launch_horner(P.pre_a, packed_b, S.pb_qstride, rgsw32, P.tables, G, d_act, pp.num_cts, resp,
                             S.resp_qstride, nq, st));
}

void enqueue_qprep_slots(const Server& S, Lane& L, size_t s0, size_t count, cudaStream_t st) {
    IPB_CK(launch_qprep(L.qraw + s0 * S.qstride, S.qstride, S.pp.db_rows, S.pre->tables, L.keys + s0 * kKeyStride,
                        L.rgsw32 + s0 * kRgswStride, (int)count, st));
}

void enqueue_scan_segment(const Server& S, Lane& L, uint32_t* keys_pos, const std::vector<SlotRun>& runs, int seg,
                          int ns, cudaStream_t st, cudaEvent_t after_matvec) {
    const Params& pp = S.pp;
    const Precomp& P = *S.pre;
    const size_t R = pp.db_rows, C = pp.db_cols, G = pp.n_packed;
    uint8_t qmap[32];
    size_t n = 0;
    for (const SlotRun& r : runs) {
        if (n + r.k > 32 || r.s0 + r.k > L.cap) throw std::invalid_argument("scan segment: 1..32 queries per pass");
        // positions n .. n + k - 1 of this segment's pass: query planes and keys
        IPB_CK(launch_qplanes(L.qraw + r.s0 * S.qstride, S.qstride, R, P.tables, L.planes + mv_tc_planes_offset(n, R),
                              (int)r.k, st));
        IPB_CK(cudaMemcpyAsync(keys_pos + n * kKeyStride, L.keys + r.s0 * kKeyStride, r.k * kKeyStride * 4,
                               cudaMemcpyDeviceToDevice, st));
        for (size_t i = 0; i < r.k; ++i) qmap[n + i] = (uint8_t)(r.s0 + i);
        n += r.k;
    }
    if (n == 0) throw std::invalid_argument("scan segment: no queries");
    if (ns < 1 || C % (128 * (size_t)ns) || (2 * kN) % (32 * ns)) throw std::invalid_argument("scan segment: bad split");
    const size_t c0 = C / ns * seg, c1 = c0 + C / ns;
    IPB_CK(launch_matvec_tc_range(P.db, R, C, c0, c1, L.planes, (int)n, P.tables, L.mvpart, S.mv_qstride, qmap,
                                  L.d_err, L.tiles, S.num_sms, S.tc_kchunk_rows, st));
    if (after_matvec) IPB_CK(cudaEventRecord(after_matvec, st));
    const int n_li = (int)(2 * kN) / ns, li0 = n_li * seg;
    for (size_t q0 = 0; q0 < n; q0 += (size_t)L.gt_pass) {
        const int k = (int)std::min<size_t>((size_t)L.gt_pass, n - q0);
        IPB_CK(launch_tensor_pass_slots(P.pre_dt, G, li0, n_li, keys_pos + q0 * kKeyStride, kKeyStride, k,
                                        (int)L.cap, (int)q0, qmap, L.keyt, L.tp_out, L.d_err, L.tiles + 1, S.num_sms,
                                        st));
    }
}

void enqueue_scan_finalize(const Server& S, Lane& L, const SlotRun& r, cudaStream_t st) {
    const Params& pp = S.pp;
    const Precomp& P = *S.pre;
    const size_t C = pp.db_cols, G = pp.n_packed;
    IPB_CK(launch_finalize_range(L.mvpart + r.s0 * S.mv_qstride, S.mv_qstride, S.tc_kchunks, C, L.tp_out, (int)L.cap,
                                 (int)r.s0, P.pre_df, L.keys + r.s0 * kKeyStride, kKeyStride, P.tables,
                                 L.packed_b + r.s0 * S.pb_qstride, S.pb_qstride, G, 0, G, (int)r.k, st));
}

int run_pipeline(const Server& S, Lane& L, const Sched& sc, size_t count, cudaStream_t st, cudaEvent_t* ev,
                 int phases, size_t n_ev, cudaEvent_t db_done) {
    if (count == 0) return 0;
    if (count > L.cap || sc.tp_pass < 1 || sc.tp_pass > L.gt_pass)
        throw std::invalid_argument("run_pipeline: batch exceeds the lane or its tensor-pass buffer");
    const size_t ns = slices_of(count, sc), slice = sc.slice > 0 ? (size_t)sc.slice : count;
    // Stage timing needs the stages one after the other: it times the
    // unchunked pipeline.
    if (phases == kPhaseAll && !ev && chunked_ok(S, sc, count))
        return run_chunked(S, L, sc, count, st, nullptr, nullptr, 3, db_done);
    if (phases != kPhaseAll || 6 * ns > n_ev) ev = nullptr;
    int launches = 0;
    // Slices run one after the other, each its own pipeline on its lane
    // slots: the DB and the tensors are read once per slice either way (one
    // mat-vec pass serves at most 32 queries), and a slice's Horner chains fit
    // the SMs in one wave.
    if (phases & kPhaseDb)
        for (size_t k = 0; k < ns; ++k) {
            const size_t q0 = k * slice;
            launches += run_db_phase(S, L, sc, q0, std::min(slice, count - q0), st, ev ? ev + 6 * k : nullptr);
            if ((phases & kPhaseHorner) && ns > 1)
                launches += run_horner_phase(S, L, sc, q0, std::min(slice, count - q0), st, ev ? ev + 6 * k : nullptr);
        }
    if ((phases & kPhaseHorner) && !((phases & kPhaseDb) && ns > 1))
        for (size_t k = 0; k < ns; ++k) {
            const size_t q0 = k * slice;
            launches += run_horner_phase(S, L, sc, q0, std::min(slice, count - q0), st, ev ? ev + 6 * k : nullptr);
        }
    if (db_done) record_outside(db_done, st);  // unchunked: at the end (slices interleave the phases)
    return launches;
}

static void run_pipeline(Server* S, size_t count) {
    IPB_CK(cudaSetDevice(S->device));
    const Sched& sc = sched_for(*S, count);
    S->timed_slices = S->timing ? slices_of(count, sc) : 0;
    S->launches += (unsigned long long)run_pipeline(*S, S->lane, sc, count, S->stream,
                                                    S->timing ? S->ev.data() : nullptr, kPhaseAll, S->ev.size());
}

// The blocking answer from host views: the KSK parts are copied first and
// the query prep and tensor pass (which need only them) start while the
// LWE vectors and then the RGSW parts cross PCIe on the lane's second
// stream; the mat-vec waits for the LWE vectors, the Horner chains for the
// RGSW parts (prepared on that stream).  Schedules that already run the
// tensor pass on the second stream stage everything first instead.
static void stage_and_run(Server* S, const ipir_query_view* qs, size_t count) {
    IPB_CK(cudaSetDevice(S->device));
    const Sched& sc = sched_for(*S, count);
    if (sc.tp_sms > 0 || S->timing) {
        stage_queries(S, qs, count);
        S->timed_slices = S->timing ? slices_of(count, sc) : 0;
        S->launches += (unsigned long long)run_pipeline(*S, S->lane, sc, count, S->stream,
                                                        S->timing ? S->ev.data() : nullptr, kPhaseAll, S->ev.size());
        return;
    }
    Lane& L = S->lane;
    IPB_CK(cudaEventRecord(L.fork, S->stream));  // the lane's buffers are free from here on
    IPB_CK(cudaStreamWaitEvent(L.aux, L.fork, 0));
    stage_parts(*S, qs, count, 2, 2, S->stream);  // KSK parts: needed first
    stage_parts(*S, qs, count, 0, 2, L.aux);      // LWE vectors: needed by the mat-vec
    IPB_CK(cudaEventRecord(L.join, L.aux));
    stage_parts(*S, qs, count, 4, 1, L.aux);      // RGSW parts: needed by the Horner chains
    IPB_CK(launch_qprep_parts(L.qraw, S->qstride, S->pp.db_rows, S->pre->tables, L.keys, L.rgsw32, (int)count, 2,
                              L.aux));
    IPB_CK(cudaEventRecord(L.rgsw_ready, L.aux));
    S->staged = count;
    S->launches += 1;
    if (chunked_ok(*S, sc, count)) {
        S->launches += (unsigned long long)run_chunked(*S, L, sc, count, S->stream, L.join, L.rgsw_ready, 1);
        return;
    }
    // The first slice's key side starts before the LWE vectors land; every
    // slice's RGSW parts were prepared on the second stream above.
    const size_t ns = slices_of(count, sc), slice = sc.slice > 0 ? (size_t)sc.slice : count;
    for (size_t k = 0; k < ns; ++k) {
        const size_t q0 = k * slice, n = std::min(slice, count - q0);
        S->launches += (unsigned long long)run_db_phase(*S, L, sc, q0, n, S->stream, nullptr,
                                                        k == 0 ? L.join : nullptr, 1);
        if (k == 0) IPB_CK(cudaStreamWaitEvent(S->stream, L.rgsw_ready, 0));
        S->launches += (unsigned long long)run_horner_phase(*S, L, sc, q0, n, S->stream, nullptr);
    }
}

// A kernel whose pipeline wait ran out of iterations leaves a code in the
// device error word; report it (the responses are then not valid).
void check_device_error(Lane& L, cudaStream_t st) {
    int e = 0;
    IPB_CK(cudaMemcpyAsync(&e, L.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    IPB_CK(cudaStreamSynchronize(st));
    if (e) {
        IPB_CK(cudaMemsetAsync(L.d_err, 0, sizeof(int), st));  // ordered before the next batch's kernels
        IPB_CK(cudaStreamSynchronize(st));
        throw std::runtime_error("device pipeline wait timed out (code " + std::to_string(e) + ")");
    }
}

// The error word is read first, once the batch has run: a batch whose
// kernels stopped early writes nothing into the caller's buffer.
static void fetch(Server* S, size_t count, uint64_t* out) {
    IPB_CK(cudaSetDevice(S->device));
    check_device_error(S->lane, S->stream);
    IPB_CK(cudaMemcpyAsync(out, S->lane.resp, count * S->resp_qstride * 8, cudaMemcpyDeviceToHost, S->stream));
    IPB_CK(cudaStreamSynchronize(S->stream));
    if (S->timing && S->timed_slices)  // stage times summed over the batch's slices
        for (int i = 0; i < 5; ++i) {
            S->stage_ms[i] = 0.f;
            for (size_t k = 0; k < S->timed_slices; ++k) {
                float t = 0.f;
                IPB_CK(cudaEventElapsedTime(&t, S->ev[6 * k + i], S->ev[6 * k + i + 1]));
                S->stage_ms[i] += t;
            }
        }
}

// ------------------------------------------------------------ schedule autotuner
// For batch sizes 1, 2, 4, ... up to the lane's capacity (and the capacity
// itself) time every candidate schedule end to end on the device -- mat-vec
// kernel (tcgen05 / CUDA-core; the CUDA-core kernel streams the DB once per
// 4 queries, so it is tried up to 8), queries per tensor-pass GEMM (the
// key-table capacity and its half: fewer queries per pass re-read the
// tensors but double-buffer the accumulators), Horner kernel (4-CTA
// cluster, 8-CTA cluster, single CTA) -- and keep the fastest; then, for the
// tensor-core mat-vec, the number of SMs (1/18 .. 8/18 of them) that run the
// tensor pass at the same time as the mat-vec, if that is faster still.
// Batches larger than 32 queries also try one pipeline for the whole batch
// against consecutive 32-query slices.  Sizes between two measured ones use
// the smaller's.
std::vector<Sched> autotune(const Server& S, Lane& L, cudaStream_t st) {
    IPB_CK(cudaSetDevice(S.device));
    std::vector<size_t> sizes;
    for (size_t b = 1; b <= L.cap; b *= 2) sizes.push_back(b);
    if (sizes.back() != L.cap) sizes.push_back(L.cap);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    IPB_CK(cudaEventCreate(&e0));
    IPB_CK(cudaEventCreate(&e1));
    std::vector<std::pair<size_t, Sched>> best;
    try {
        for (size_t b : sizes) {
            std::vector<Sched> cands;
            std::vector<int> passes{(int)std::min<size_t>(b, (size_t)L.gt_pass)};
            if (passes[0] >= 16) passes.push_back(passes[0] / 2);
            for (int mv : {1, 0}) {
                if (!mv && b > 8) continue;
                for (int p : passes)
                    for (int h : {1, 2, 0}) cands.push_back(Sched{mv, p, h});
            }
            // Batches larger than one slice: also the whole batch in one
            // pipeline (one query prep, finalize and Horner launch for all).
            if (b > kSliceQueries)
                for (size_t i = 0, n = cands.size(); i < n; ++i) {
                    Sched w = cands[i];
                    w.slice = 0;
                    cands.push_back(w);
                }
            auto time_of = [&](const Sched& c) {
                run_pipeline(S, L, c, b, st, nullptr);  // warm
                float ms = 1e30f;
                for (int r = 0; r < 2; ++r) {
                    IPB_CK(cudaEventRecord(e0, st));
                    run_pipeline(S, L, c, b, st, nullptr);
                    IPB_CK(cudaEventRecord(e1, st));
                    IPB_CK(cudaEventSynchronize(e1));
                    float t = 0;
                    IPB_CK(cudaEventElapsedTime(&t, e0, e1));
                    ms = std::min(ms, t);
                }
                return ms;
            };
            float best_ms = 1e30f;
            Sched pick = cands[0];
            for (const Sched& c : cands) {
                const float ms = time_of(c);
                if (ms < best_ms * 0.98f) {  // keep the earlier (default-ordered) choice on near ties
                    best_ms = ms;
                    pick = c;
                }
            }
            // Then the SM split for running the tensor pass beside the mat-vec.
            // Clocks drift under the power cap while candidates are timed, so
            // the best split must also beat the sequential schedule by 3 % in
            // an interleaved head-to-head of three rounds.
            if (pick.matvec_tc) {
                const Sched seq = pick;
                Sched split = seq;
                float split_ms = 1e30f;
                for (int k = 1; k <= 8; ++k) {
                    Sched c = seq;
                    c.tp_sms = S.num_sms * k / 18;  // 1/18 .. 8/18 of the SMs
                    if (c.tp_sms < 1) continue;
                    const float ms = time_of(c);
                    if (ms < split_ms) {
                        split_ms = ms;
                        split = c;
                    }
                }
                if (split.tp_sms > 0 && split_ms < best_ms * 0.98f) {
                    float a = 1e30f, b = 1e30f;
                    for (int r = 0; r < 3; ++r) {
                        a = std::min(a, time_of(seq));
                        b = std::min(b, time_of(split));
                    }
                    if (b < a * 0.97f) pick = split;
                }
            }
            // Then the Horner chain trailing the DB pass in chunks (at most 8,
            // the schedule that measured best) with either cluster kernel:
            // the best unchunked kernel need not be the best chunked one.
            // Kept only if it beats the pick by 2 % in an interleaved
            // head-to-head.
            {
                std::vector<Sched> chs;
                for (int hc : {1, 2}) {
                    Sched c = pick;
                    c.horner_cluster = hc;
                    c.hchunks = 8;
                    if (chunked_ok(S, c, b)) chs.push_back(c);
                }
                if (!chs.empty()) {
                    float a = 1e30f;
                    std::vector<float> t(chs.size(), 1e30f);
                    for (int r = 0; r < 3; ++r) {
                        a = std::min(a, time_of(pick));
                        for (size_t i = 0; i < chs.size(); ++i) t[i] = std::min(t[i], time_of(chs[i]));
                    }
                    const size_t i = (size_t)(std::min_element(t.begin(), t.end()) - t.begin());
                    if (t[i] < a * 0.98f) pick = chs[i];
                }
            }
            best.emplace_back(b, pick);
        }
        check_device_error(L, st);
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // Sizes between two measured ones take the smaller one's kernels, with
    // its tensor-pass split scaled to their own size (one pass, or halves),
    // never more passes than that split.
    std::vector<Sched> table(L.cap + 1);
    for (size_t c = 1; c <= L.cap; ++c) {
        const std::pair<size_t, Sched>* s = &best[0];
        for (auto& kv : best)
            if (kv.first <= c) s = &kv;
        table[c] = s->second;
        const int whole = (int)std::min<size_t>(s->first, (size_t)L.gt_pass);
        const bool halves = s->second.tp_pass < whole;
        const size_t want = halves ? (c + 1) / 2 : c;
        table[c].tp_pass = (int)std::max<size_t>(1, std::min<size_t>(want, (size_t)L.gt_pass));
    }
    table[0] = table[1];
    return table;
}

// ipir_answer_batch on packed queries: H2D of the packed bytes, unpack on
// the device, the pipeline, then the response in the requested format.
static void answer_wire(Server* S, const uint8_t* packed, size_t count, int fmt, void* out) {
    IPB_CK(cudaSetDevice(S->device));
    Lane& L = S->lane;
    const Precomp& P = *S->pre;
    cudaStream_t st = S->stream;
    IPB_CK(cudaMemcpyAsync(L.wire_in, packed, count * S->wire_q, cudaMemcpyHostToDevice, st));
    IPB_CK(launch_query_unpack(L.wire_in, S->wire_q, S->pp.db_rows, L.qraw, S->qstride, (int)count, P.tables, st));
    run_pipeline(S, count);
    const void* src = L.resp;
    size_t bytes = count * S->resp_qstride * 8;
    if (fmt == 1) {
        IPB_CK(launch_response_pack(L.resp, S->resp_qstride, S->pp.num_cts, L.wire_out, S->wire_r, (int)count,
                                    P.tables, st));
        src = L.wire_out;
        bytes = count * S->wire_r;
    } else if (fmt == 2) {
        IPB_CK(launch_response_compress(L.resp, S->resp_qstride, S->pp.num_cts, L.codec_tmp, L.wire_out, S->wire_c,
                                        (int)count, P.tables, st));
        src = L.wire_out;
        bytes = count * S->wire_c;
    }
    check_device_error(L, st);  // nothing is written if a kernel stopped early
    IPB_CK(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, st));
    IPB_CK(cudaStreamSynchronize(st));
}

static int validate_batch(const Server* S, const ipir_query_view* qs, size_t count, const void* out) {
    if (!S || !qs || !out) return 1;
    if (count > S->max_batch) return 2;
    for (size_t i = 0; i < count; ++i) {
        const ipir_query_view& v = qs[i];
        if (!v.lwe_b_limb0 || !v.lwe_b_limb1 || !v.ksk5_b || !v.kskneg1_b || !v.rgsw) return 3;
    }
    return 0;
}

bool shard_whole_cts(const Params& global, size_t g0, size_t g1) {
    const size_t d_act = std::min(global.D, global.n_packed);
    return g0 % d_act == 0 && (g1 % d_act == 0 || g1 == global.n_packed);
}

Params shard_params(const Params& global, size_t g0, size_t g1) {
    if (g1 <= g0 || g1 > global.n_packed) throw std::invalid_argument("group shard: need 0 <= lo < hi <= n_packed");
    Params p = global;
    p.db_cols = (g1 - g0) * kN;
    p.n_packed = g1 - g0;
    if (shard_whole_cts(global, g0, g1)) {
        // whole Horner chunks: the shard's own pipeline answers its ciphertexts
        const size_t d_act = std::min(global.D, global.n_packed);
        p.D = global.D;
        p.num_cts = (p.n_packed + d_act - 1) / d_act;
    } else {
        p.D = p.n_packed;  // packs only: the Horner chains run on the owner
        p.num_cts = 1;
    }
    return p;
}

std::shared_ptr<Precomp> run_preprocess_shard(const Params& global, const uint16_t* db, size_t g0, size_t g1) {
    if (!db) throw std::invalid_argument("gpu_preprocess: null db");
    auto P = std::make_shared<Precomp>();
    P->pp = shard_params(global, g0, g1);
    IPB_CK(cudaGetDevice(&P->device));
    cudaStream_t s = nullptr;
    IPB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
        preprocess_into(*P, db, s, &global, g0);
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    return P;
}

static std::shared_ptr<Precomp> run_preprocess(const Params& pp, const uint16_t* db) {
    if (!db) throw std::invalid_argument("gpu_preprocess: null db");
    auto P = std::make_shared<Precomp>();
    P->pp = pp;
    IPB_CK(cudaGetDevice(&P->device));
    cudaStream_t s = nullptr;
    IPB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
        preprocess_into(*P, db, s);
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    return P;
}

}  // namespace ipb

// ======================================================================= C++ API
namespace inspire_b200 {

struct PreprocessState {
    std::shared_ptr<ipb::Precomp> p;
};
struct GpuServerCtx {
    ipb::Server* s;
};

static ipb::Params to_ipb(const PublicParams& pp) {
    ipb::Params p{};
    p.n_entries = pp.N_entries;
    p.w = pp.w;
    p.db_rows = pp.db_rows;
    p.db_cols = pp.db_cols;
    p.n_packed = pp.n_packed;
    p.D = pp.D;
    p.num_cts = pp.num_cts;
    std::memcpy(p.seed, pp.seed.data(), SEED_BYTES);
    return p;
}

static void check_geometry(const PublicParams& pp) {
    ipb::Params chk{};
    const char* why = nullptr;
    if (ipb::setup_geometry(pp.N_entries, pp.w, pp.db_rows, &chk, &why) != 0) throw std::invalid_argument(why);
    if (chk.db_cols != pp.db_cols || chk.n_packed != pp.n_packed || chk.D != pp.D || chk.num_cts != pp.num_cts)
        throw std::invalid_argument("PublicParams inconsistent with setup()");
}

PublicParams setup(size_t N_entries, size_t w) { return setup(N_entries, w, ipb::kDefaultDbRows); }

PublicParams setup(size_t N_entries, size_t w, size_t db_rows_override) {
    ipb::Params p{};
    const char* why = nullptr;
    if (ipb::setup_geometry(N_entries, w, db_rows_override, &p, &why) != 0) throw std::invalid_argument(why);
    PublicParams pp;
    pp.N_entries = p.n_entries;
    pp.w = p.w;
    pp.db_rows = p.db_rows;
    pp.db_cols = p.db_cols;
    pp.n_packed = p.n_packed;
    pp.D = p.D;
    pp.num_cts = p.num_cts;
    std::random_device rd;  // src/params.cpp:63-65
    std::mt19937_64 rng(rd());
    for (auto& b : pp.seed) b = (uint8_t)(rng() & 0xFF);
    return pp;
}

PreprocessData gpu_preprocess(const PublicParams& pp, const uint16_t* db) {
    check_geometry(pp);
    PreprocessData d;
    d.state = std::make_shared<PreprocessState>();
    d.state->p = ipb::run_preprocess(to_ipb(pp), db);
    return d;
}

PreprocessDevicePointers preprocess_device_pointers(const PreprocessData& precomp) {
    if (!precomp.state || !precomp.state->p) throw std::invalid_argument("preprocess_device_pointers: empty or adopted");
    const ipb::Precomp& P = *precomp.state->p;
    return PreprocessDevicePointers{P.db, P.pre_a, ipb::kGroupStrideA, P.pre_df, ipb::kGroupStrideF};
}

GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp) {
    return gpu_setup_server(pp, precomp, GpuServerConfig{});
}

GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp, const GpuServerConfig& cfg) {
    if (!precomp.state) throw std::invalid_argument("gpu_setup_server: empty PreprocessData");
    // Ownership of the device buffers moves to the context, as in the
    // reference (src/gpu_protocol.cu:856-885).
    std::shared_ptr<ipb::Precomp> p = std::move(precomp.state->p);
    ipb::DeviceRestore keep_device;
    auto* ctx = new GpuServerCtx{ipb::make_server(to_ipb(pp), std::move(p), cfg.max_batch)};
    return ctx;
}

GpuServerCaps gpu_server_caps(const GpuServerCtx* ctx) {
    GpuServerCaps c{};
    if (!ctx) return c;
    c.max_batch = ctx->s->max_batch;
    c.resident_bytes = ctx->s->resident_bytes;
    c.num_cts = ctx->s->pp.num_cts;
    size_t fr = 0, tot = 0;
    ipb::DeviceRestore keep_device;
    cudaSetDevice(ctx->s->device);
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) c.device_free_bytes = fr;
    return c;
}

void gpu_answer_batch(GpuServerCtx* ctx, const ipir_query_view* queries, size_t count, uint64_t* out) {
    if (!ctx) throw std::invalid_argument("gpu_answer_batch: null ctx");
    int rc = ipb::validate_batch(ctx->s, queries, count, out);
    if (rc == 2) throw std::invalid_argument("gpu_answer_batch: count exceeds max_batch");
    if (rc) throw std::invalid_argument("gpu_answer_batch: null argument");
    if (count == 0) return;
    ipb::DeviceRestore keep_device;
    ipb::stage_and_run(ctx->s, queries, count);
    ipb::fetch(ctx->s, count, out);
}

void gpu_answer(GpuServerCtx* ctx, const ipir_query_view& q, uint64_t* out) { gpu_answer_batch(ctx, &q, 1, out); }

void gpu_free_server(GpuServerCtx* ctx) {
    if (!ctx) return;
    ipb::DeviceRestore keep_device;
    delete ctx->s;
    delete ctx;
}

}  // namespace inspire_b200

// ======================================================================= C ABI

namespace {
template <class F>
int guarded(F&& f, int fail_code) {
    ipb::DeviceRestore keep_device;
    try {
        return f();
    } catch (const std::exception& e) {
        ipb::g_last_error = e.what();
    } catch (...) {
        ipb::g_last_error = "unknown error";
    }
    return fail_code;
}
}  // namespace

void ipb::fill_params(const ipb::Params& pp, ipir_params* o) {
    o->n_entries = pp.n_entries;
    o->entry_bytes = pp.w;
    o->db_rows = pp.db_rows;
    o->db_cols = pp.db_cols;
    o->n_packed = pp.n_packed;
    o->interp_d = pp.D;
    o->num_cts = pp.num_cts;
    o->ring_n = ipb::kN;
    o->d_eff = ipb::kDeff;
    std::memcpy(o->seed, pp.seed, 64);
}

using ipb::fill_params;

extern "C" {

const char* ipir_b200_last_error(void) { return ipb::g_last_error.c_str(); }

int ipir_b200_setup(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero, ipir_params* out) {
    if (!out) return 1;
    ipb::Params pp{};
    const char* why = nullptr;
    int rc = ipb::setup_geometry(n_entries, entry_bytes, db_rows_or_zero, &pp, &why);
    if (rc) {
        ipb::g_last_error = why ? why : "setup failed";
        return rc;
    }
    fill_params(pp, out);
    return 0;
}

ipir_server* ipir_server_create(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero, size_t max_batch,
                                const uint16_t* db, const uint8_t* crs_seed_or_null, ipir_params* out_params) {
    if (!db || !out_params || max_batch == 0) {
        ipb::g_last_error = "ipir_server_create: null argument or max_batch == 0";
        return nullptr;
    }
    ipir_server* result = nullptr;
    guarded(
        [&]() -> int {
            ipb::Params pp{};
            const char* why = nullptr;
            if (ipb::setup_geometry(n_entries, entry_bytes, db_rows_or_zero, &pp, &why) != 0)
                throw std::invalid_argument(why);
            if (crs_seed_or_null) {
                std::memcpy(pp.seed, crs_seed_or_null, 64);
            } else {
                std::random_device rd;
                std::mt19937_64 rng(rd());
                for (auto& b : pp.seed) b = (uint8_t)(rng() & 0xFF);
            }
            auto P = ipb::run_preprocess(pp, db);
            std::unique_ptr<ipb::Server> S(ipb::make_server(pp, std::move(P), max_batch));
            fill_params(pp, out_params);
            result = new ipir_server{S.release()};
            return 0;
        },
        1);
    return result;
}

void ipir_server_caps(const ipir_server* srv, ipir_caps* out) {
    if (!srv || !out) return;
    inspire_b200::GpuServerCtx ctx{srv->s};
    auto c = inspire_b200::gpu_server_caps(&ctx);
    out->max_batch = c.max_batch;
    out->resident_bytes = c.resident_bytes;
    out->device_free_bytes = c.device_free_bytes;
    out->num_cts = c.num_cts;
}

int ipir_answer_batch(ipir_server* srv, const ipir_query_view* queries, size_t count, uint64_t* out_resp) {
    if (!srv) return 1;
    int rc = ipb::validate_batch(srv->s, queries, count, out_resp);
    if (rc) return rc;
    if (count == 0) return 0;
    return guarded(
        [&]() -> int {
            ipb::stage_and_run(srv->s, queries, count);
            ipb::fetch(srv->s, count, out_resp);
            return 0;
        },
        4);
}

void ipir_server_destroy(ipir_server* srv) {
    if (!srv) return;
    ipb::DeviceRestore keep_device;
    delete srv->s;
    delete srv;
}

int ipir_b200_set_stream(ipir_server* srv, void* stream) {
    if (!srv) return 1;
    srv->s->stream = stream ? static_cast<cudaStream_t>(stream) : srv->s->own_stream;
    return 0;
}

int ipir_b200_stage_queries(ipir_server* srv, const ipir_query_view* queries, size_t count) {
    if (!srv) return 1;
    int rc = ipb::validate_batch(srv->s, queries, count, queries);
    if (rc) return rc;
    return guarded([&]() -> int { ipb::stage_queries(srv->s, queries, count); return 0; }, 4);
}

int ipir_b200_run(ipir_server* srv, size_t count) {
    if (!srv) return 1;
    if (count > srv->s->max_batch) return 2;
    if (count == 0) return 0;
    return guarded([&]() -> int { ipb::run_pipeline(srv->s, count); return 0; }, 4);
}

int ipir_b200_fetch_responses(ipir_server* srv, size_t count, uint64_t* out) {
    if (!srv || !out) return 1;
    if (count > srv->s->max_batch) return 2;
    return guarded([&]() -> int { ipb::fetch(srv->s, count, out); return 0; }, 4);
}

int ipir_b200_sync(ipir_server* srv) {
    if (!srv) return 1;
    return guarded([&]() -> int { IPB_CK(cudaStreamSynchronize(srv->s->stream)); return 0; }, 4);
}

int ipir_b200_enable_stage_timing(ipir_server* srv, int on) {
    if (!srv) return 1;
    srv->s->timing = on != 0;
    return 0;
}

int ipir_b200_stage_times(const ipir_server* srv, float* ms_out, size_t n) {
    if (!srv || !ms_out) return 1;
    for (size_t i = 0; i < n && i < 5; ++i) ms_out[i] = srv->s->stage_ms[i];
    return 0;
}

int ipir_b200_wire_sizes(const ipir_params* params, size_t* query_packed, size_t* response_packed,
                         size_t* response_compressed) {
    if (!params) return 1;
    if (query_packed) *query_packed = ipb::wire_query_bytes(params->db_rows);
    if (response_packed) *response_packed = ipb::wire_response_bytes(params->num_cts);
    if (response_compressed) *response_compressed = ipb::wire_compressed_bytes(params->num_cts);
    return 0;
}

int ipir_b200_answer_wire(ipir_server* srv, const uint8_t* packed, size_t count, int resp_format, void* out) {
    if (!srv || !packed || !out) return 1;
    if (count > srv->s->max_batch) return 2;
    if (resp_format < 0 || resp_format > 2) return 3;
    if (count == 0) return 0;
    return guarded([&]() -> int { ipb::answer_wire(srv->s, packed, count, resp_format, out); return 0; }, 4);
}

int ipir_b200_autotune(ipir_server* srv) {
    if (!srv) return 1;
    return guarded(
        [&]() -> int {
            ipb::Server* S = srv->s;
            IPB_CK(cudaSetDevice(S->device));
            S->sched = ipb::autotune(*S, S->lane, S->stream);
            S->tuned = true;
            return 0;
        },
        4);
}

int ipir_b200_get_schedule(const ipir_server* srv, size_t count, ipir_serve_schedule* out) {
    if (!srv || !out) return 1;
    if (count == 0 || count > srv->s->max_batch) return 2;
    const ipb::Sched& sc = ipb::sched_for(*srv->s, count);
    out->matvec_tc = sc.matvec_tc;
    out->tp_pass = sc.tp_pass;
    out->horner_cluster = sc.horner_cluster;
    out->tp_sms = sc.tp_sms;
    out->slice = sc.slice;
    out->hchunks = sc.hchunks;
    return 0;
}

int ipir_b200_set_schedule(ipir_server* srv, size_t count, const ipir_serve_schedule* sc) {
    if (!srv || !sc) return 1;
    ipb::Server* S = srv->s;
    if (count == 0 || count > S->max_batch) return 2;
    if (sc->matvec_tc < 0 || sc->matvec_tc > 1 || sc->horner_cluster < 0 || sc->horner_cluster > 2 ||
        sc->tp_pass < 1 || sc->tp_pass > S->lane.gt_pass || sc->tp_sms < 0 || sc->tp_sms >= S->num_sms ||
        (sc->tp_sms > 0 && !sc->matvec_tc) || (sc->slice != 0 && sc->slice != (int)ipb::kSliceQueries) ||
        sc->hchunks < 0 || sc->hchunks > ipb::kMaxHChunks) {
        ipb::g_last_error =
            "ipir_b200_set_schedule: matvec_tc 0/1, horner_cluster 0/1/2, tp_pass 1..capacity, "
            "tp_sms 0..SMs-1 (0 with the CUDA-core mat-vec), slice 0/32, hchunks 0..16";
        return 2;
    }
    S->sched[count] = ipb::Sched{sc->matvec_tc, sc->tp_pass, sc->horner_cluster, sc->tp_sms, sc->slice, sc->hchunks};
    return 0;
}

int ipir_b200_launch_count(const ipir_server* srv, unsigned long long* out) {
    if (!srv || !out) return 1;
    *out = srv->s->launches;
    return 0;
}

int ipir_b200_export_precomp(const ipir_server* srv, size_t group, uint32_t* a, uint32_t* d_plus, uint32_t* d_minus,
                             uint32_t* d_final) {
    if (!srv) return 1;
    const ipb::Server* S = srv->s;
    if (group >= S->pp.n_packed) return 2;
    return guarded(
        [&]() -> int {
            IPB_CK(cudaSetDevice(S->device));
            const ipb::Precomp& P = *S->pre;
            if (a) IPB_CK(cudaMemcpy(a, P.pre_a + group * ipb::kGroupStrideA, ipb::kGroupStrideA * 4, cudaMemcpyDeviceToHost));
            if (d_plus || d_minus) {
                ipb::DevArena tmp;
                try {
                    uint32_t* tp = tmp.alloc<uint32_t>(ipb::kGroupStrideD);
                    uint32_t* tm = tmp.alloc<uint32_t>(ipb::kGroupStrideD);
                    IPB_CK(ipb::launch_dt_export(P.pre_dt, group, S->pp.n_packed, tp, tm, 0));
                    IPB_CK(cudaDeviceSynchronize());
                    if (d_plus) IPB_CK(cudaMemcpy(d_plus, tp, ipb::kGroupStrideD * 4, cudaMemcpyDeviceToHost));
                    if (d_minus) IPB_CK(cudaMemcpy(d_minus, tm, ipb::kGroupStrideD * 4, cudaMemcpyDeviceToHost));
                } catch (...) {
                    tmp.free_all();
                    throw;
                }
                tmp.free_all();
            }
            if (d_final) IPB_CK(cudaMemcpy(d_final, P.pre_df + group * ipb::kGroupStrideF, ipb::kGroupStrideF * 4, cudaMemcpyDeviceToHost));
            return 0;
        },
        4);
}

int ipir_b200_export_db(const ipir_server* srv, size_t row0, size_t nrows, uint16_t* out) {
    if (!srv || !out) return 1;
    const ipb::Server* S = srv->s;
    if (row0 + nrows > S->pp.db_rows) return 2;
    return guarded(
        [&]() -> int {
            IPB_CK(cudaSetDevice(S->device));
            IPB_CK(cudaMemcpy(out, S->pre->db + row0 * S->pp.db_cols, nrows * S->pp.db_cols * 2, cudaMemcpyDeviceToHost));
            return 0;
        },
        4);
}

int ipir_b200_ntt(uint32_t* polys, size_t n, int limb_run, int inverse) {
    if (!polys || limb_run <= 0) return 1;
    if (n == 0) return 0;
    return guarded(
        [&]() -> int {
            ipb::DevArena A;
            try {
                ipb::DevTables* T = ipb::upload_tables(A, 0);
                uint32_t* d = A.alloc<uint32_t>(n * ipb::kN);
                IPB_CK(cudaMemcpy(d, polys, n * ipb::kN * 4, cudaMemcpyHostToDevice));
                IPB_CK(ipb::launch_ntt_batch(d, n, limb_run, inverse != 0, T, 0));
                IPB_CK(cudaMemcpy(polys, d, n * ipb::kN * 4, cudaMemcpyDeviceToHost));
            } catch (...) {
                A.free_all();
                throw;
            }
            A.free_all();
            return 0;
        },
        4);
}

int ipir_b200_decomp(const uint32_t* in, uint32_t* out, size_t n) {
    if (!in || !out) return 1;
    if (n == 0) return 0;
    return guarded(
        [&]() -> int {
            ipb::DevArena A;
            try {
                ipb::DevTables* T = ipb::upload_tables(A, 0);
                uint32_t* di = A.alloc<uint32_t>(n * 2 * ipb::kN);
                uint32_t* dout = A.alloc<uint32_t>(n * ipb::kDeff * 2 * ipb::kN);
                IPB_CK(cudaMemcpy(di, in, n * 2 * ipb::kN * 4, cudaMemcpyHostToDevice));
                IPB_CK(ipb::launch_decomp(di, dout, n, T, 0));
                IPB_CK(cudaMemcpy(out, dout, n * ipb::kDeff * 2 * ipb::kN * 4, cudaMemcpyDeviceToHost));
            } catch (...) {
                A.free_all();
                throw;
            }
            A.free_all();
            return 0;
        },
        4);
}

int ipir_b200_horner_eval(const uint64_t* rgsw, const uint64_t* cts, size_t L, uint64_t* out, int variant) {
    if (!rgsw || !cts || !out || L == 0) return 1;
    if (variant < 0 || variant > 2 || L > 4096) {
        ipb::g_last_error = "ipir_b200_horner_eval: variant 0..2, 1 <= L <= 4096";
        return 2;
    }
    return guarded(
        [&]() -> int {
            using ipb::kN;
            const size_t blk = (size_t)ipb::kDeff * 2 * kN;
            // residues as u32: a and b halves of each ciphertext, the RGSW parts
            std::vector<uint32_t> a(L * 2 * kN), b(L * 2 * kN), rg(4 * blk);
            for (size_t g = 0; g < L; ++g)
                for (size_t x = 0; x < 2 * kN; ++x) {
                    const uint64_t q = (x / kN) ? ipb::kQ1 : ipb::kQ0;
                    a[g * 2 * kN + x] = (uint32_t)(cts[g * 4 * kN + x] % q);
                    b[g * 2 * kN + x] = (uint32_t)(cts[g * 4 * kN + 2 * kN + x] % q);
                }
            for (size_t i = 0; i < 4 * blk; ++i) rg[i] = (uint32_t)(rgsw[i] % (((i / kN) & 1) ? ipb::kQ1 : ipb::kQ0));
            ipb::DevArena A;
            try {
                ipb::DevTables* T = ipb::upload_tables(A, 0);
                uint32_t* da = A.alloc<uint32_t>(a.size());
                uint32_t* db = A.alloc<uint32_t>(b.size());
                uint32_t* dr = A.alloc<uint32_t>(rg.size());
                uint64_t* dout = A.alloc<uint64_t>(4 * kN);
                int* err = A.alloc<int>(1);
                IPB_CK(cudaMemcpy(da, a.data(), a.size() * 4, cudaMemcpyHostToDevice));
                IPB_CK(cudaMemcpy(db, b.data(), b.size() * 4, cudaMemcpyHostToDevice));
                IPB_CK(cudaMemcpy(dr, rg.data(), rg.size() * 4, cudaMemcpyHostToDevice));
                IPB_CK(cudaMemset(err, 0, sizeof(int)));
                if (variant == 0)
                    IPB_CK(ipb::launch_horner(da, db, L * 2 * kN, dr, T, L, L, 1, dout, 4 * kN, 1, 0));
                else if (variant == 1)
                    IPB_CK(ipb::launch_horner_cluster(da, db, L * 2 * kN, dr, T, L, L, 1, dout, 4 * kN, 1, err, 0));
                else
                    IPB_CK(ipb::launch_horner_cluster8(da, db, L * 2 * kN, dr, T, L, L, 1, dout, 4 * kN, 1, err, 0));
                int h_err = 0;
                IPB_CK(cudaMemcpy(out, dout, 4 * kN * 8, cudaMemcpyDeviceToHost));
                IPB_CK(cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost));
                if (h_err) throw std::runtime_error("device pipeline wait timed out");
            } catch (...) {
                A.free_all();
                throw;
            }
            A.free_all();
            return 0;
        },
        4);
}

namespace {
// Scratch of ipir_b200_matvec, cached per device and grown on demand.
struct MvScratch {
    ipb::DevArena arena;
    ipb::DevTables* T = nullptr;
    int* err = nullptr;
    unsigned* tiles = nullptr;
    uint8_t* planes = nullptr;
    size_t planes_cap = 0;
    uint32_t* part = nullptr;
    size_t part_cap = 0;
};
std::mutex g_mv_mu;
MvScratch g_mv[64];
}  // namespace

int ipir_b200_matvec_ex(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries, size_t count,
                        uint32_t* out, void* stream, int sync, const ipir_matvec_opts* opts) {
    if (!db || !queries || !out) return 1;
    if (count == 0) return 0;
    ipir_matvec_opts o{};
    if (opts) o = *opts;
    const bool cores = o.path == 1;
    if (o.path != 0 && o.path != 1) {
        ipb::g_last_error = "ipir_b200_matvec_ex: path must be 0 (tensor cores) or 1 (CUDA cores)";
        return 2;
    }
    if (rows == 0 || rows % 1024 || cols == 0 || cols % (cores ? 2048 : 128) || (rows > 32768 && rows % 32768)) {
        ipb::g_last_error = "ipir_b200_matvec: rows must be a multiple of 1024 (of 32768 above 32768), "
                            "cols a multiple of 128 (2048 on the CUDA-core path)";
        return 2;
    }
    const int max_pass = cores ? 4 : 32;
    const int qpp = o.queries_per_pass ? o.queries_per_pass : max_pass;
    if (qpp < 1 || qpp > max_pass) {
        ipb::g_last_error = "ipir_b200_matvec_ex: queries_per_pass out of range";
        return 2;
    }
    if (!cores && o.kchunk_rows &&
        (o.kchunk_rows % 1024 || o.kchunk_rows > 32768 || rows % (size_t)o.kchunk_rows)) {
        ipb::g_last_error = "ipir_b200_matvec_ex: kchunk_rows must be a multiple of 1024 dividing rows, <= 32768";
        return 2;
    }
    return guarded(
        [&]() -> int {
            int dev = 0, sms = 0;
            IPB_CK(cudaGetDevice(&dev));
            if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
            IPB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            cudaStream_t s = static_cast<cudaStream_t>(stream);
            std::lock_guard<std::mutex> lk(g_mv_mu);
            MvScratch& M = g_mv[dev];
            if (!M.T) {
                M.T = ipb::upload_tables(M.arena, 0);
                M.err = M.arena.alloc<int>(1);
                M.tiles = M.arena.alloc<unsigned>(1);
                IPB_CK(cudaMemset(M.err, 0, sizeof(int)));
                IPB_CK(cudaDeviceSynchronize());  // tables visible to any stream
            }
            // exact K-chunks: tensor cores accumulate s32 over <= 32768 rows, the
            // CUDA cores stage <= 4096 rows of query words per CTA
            size_t kchunk;
            if (cores) {
                kchunk = std::min<size_t>(rows, 4096);
                while (kchunk > 1024 && (cols / 2048) * (rows / kchunk) < (size_t)(4 * sms)) kchunk /= 2;
            } else {
                kchunk = o.kchunk_rows ? (size_t)o.kchunk_rows : (size_t)ipb::matvec_tc_kchunk_rows(rows, cols, sms);
            }
            const int chunks = (int)(rows / kchunk);
            const size_t pq = (size_t)chunks * 2 * cols;  // partials of one query
            if (chunks > 1 && pq * qpp > M.part_cap) {
                M.part = M.arena.alloc<uint32_t>(pq * qpp);
                M.part_cap = pq * qpp;
            }
            if (!cores) {
                const size_t pbytes = ipb::mv_tc_planes_bytes(rows, (int)count);
                if (pbytes > M.planes_cap) {
                    M.planes = M.arena.alloc<uint8_t>(pbytes);
                    M.planes_cap = pbytes;
                }
                IPB_CK(ipb::launch_qplanes(queries, 2 * rows, rows, M.T, M.planes, (int)count, s));
            }
            for (size_t q0 = 0; q0 < count; q0 += (size_t)qpp) {
                const int n = (int)std::min<size_t>((size_t)qpp, count - q0);
                uint32_t* dst = chunks == 1 ? out + q0 * 2 * cols : M.part;
                const size_t dst_qstride = chunks == 1 ? 2 * cols : pq;
                if (cores)
                    IPB_CK(ipb::launch_matvec(db, rows, cols, chunks, queries + q0 * 2 * rows, 2 * rows, M.T, dst,
                                              dst_qstride, n, s));
                else
                    IPB_CK(ipb::launch_matvec_tc(db, rows, cols, M.planes + ipb::mv_tc_planes_offset(q0, rows), n, M.T, dst, dst_qstride,
                                                 M.err, M.tiles, sms, (int)kchunk, s));
                if (chunks > 1)
                    IPB_CK(ipb::launch_mv_chunk_reduce(M.part, pq, chunks, cols, M.T, out + q0 * 2 * cols, 2 * cols, n,
                                                       s));
            }
            if (sync) {
                int e = 0;  // read and cleared on the caller's stream, after the launches above
                IPB_CK(cudaMemcpyAsync(&e, M.err, sizeof(int), cudaMemcpyDeviceToHost, s));
                IPB_CK(cudaStreamSynchronize(s));
                if (e) {
                    IPB_CK(cudaMemsetAsync(M.err, 0, sizeof(int), s));
                    IPB_CK(cudaStreamSynchronize(s));
                    ipb::g_last_error = "ipir_b200_matvec: a kernel's pipeline wait timed out or it stopped early "
                                        "(code " + std::to_string(e) + ")";
                    return 5;
                }
            }
            return 0;
        },
        4);
}

int ipir_b200_matvec(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries, size_t count,
                     uint32_t* out, void* stream, int sync) {
    return ipir_b200_matvec_ex(db, rows, cols, queries, count, out, stream, sync, nullptr);
}

int ipir_b200_fill_db_device(uint16_t* out, size_t count, uint64_t seed, void* stream) {
    if (!out && count) return 1;
    if (count == 0) return 0;
    return guarded(
        [&]() -> int {
            IPB_CK(ipb::launch_fill_db(out, count, seed, static_cast<cudaStream_t>(stream)));
            return 0;
        },
        4);
}

int ipir_b200_synth_queries(size_t db_rows, uint64_t seed, uint64_t first_id, size_t count, uint64_t* out,
                            void* stream) {
    if (!out && count) return 1;
    if (db_rows == 0 || db_rows % ipb::kN) {
        ipb::g_last_error = "ipir_b200_synth_queries: db_rows must be a positive multiple of 2048";
        return 2;
    }
    if (count == 0) return 0;
    return guarded(
        [&]() -> int {
            IPB_CK(ipb::launch_synth_queries(out, db_rows, count, seed, first_id, static_cast<cudaStream_t>(stream)));
            return 0;
        },
        4);
}

int ipir_b200_fill_db(uint16_t* out, size_t count, uint64_t seed) {
    if (!out && count) return 1;
    // splitmix64(seed ^ k) mod 65535 at flat index k, on all host threads.
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    const size_t per = (count + nt - 1) / nt;
    for (unsigned w = 0; w < nt; ++w)
        th.emplace_back([=] {
            const size_t k0 = (size_t)w * per, k1 = std::min(count, k0 + per);
            for (size_t k = k0; k < k1; ++k) {
                uint64_t x = (seed ^ k) + 0x9e3779b97f4a7c15ULL;
                x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
                x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
                x ^= x >> 31;
                out[k] = (uint16_t)(x % 65535u);
            }
        });
    for (auto& t : th) t.join();
    return 0;
}

int ipir_b200_shake256(const uint8_t* in, size_t inlen, uint8_t* out, size_t outlen) {
    if ((!in && inlen) || (!out && outlen)) return 1;
    ipb::shake256(in, inlen, out, outlen);
    return 0;
}

int ipir_b200_expand_seed(const uint8_t* seed64, const char* domain, uint64_t index, uint32_t* out) {
    if (!seed64 || !domain || !out) return 1;
    return guarded([&]() -> int { ipb::expand_seed(seed64, domain, index, out); return 0; }, 2);
}

}  // extern "C"
