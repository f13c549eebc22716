// shard.cpp -- group sharding of one database over several GPUs.
//
// The answer's only cross-group step is the Horner chain over the packed
// ciphertexts of a ciphertext's D_act groups (HornerEval,
// src/crypto.cpp:264-279, as src/gpu_protocol.cu:1300-1334 slices it); the
// mat-vec (src/gpu_online.cu:23-175), the tensor pass
// (src/gpu_online.cu:593-779) and the per-group finalize are independent per
// group.  So a database splits into contiguous group ranges, one per GPU:
//
//   shard (one per GPU)  its column slab of the encoded DB and its groups'
//                        tensors; per batch: mat-vec over the slab, tensor
//                        pass and finalize of its groups -> the b parts of
//                        its packed ciphertexts [query][group][limb][N] u32
//   exchange             one gather of those b parts to the Horner owner
//                        (NCCL, by the caller; 2 N u32 per group and query)
//   Horner owner         the a parts of every group (copied once at set-up)
//                        and the queries' RGSW parts; runs the chains and
//                        writes the responses.
//
// Every stage computes what the single-GPU server computes on the same
// groups, so the responses are identical to ipir_answer_batch's.  The
// reference runs on one GPU only (docs/ARCHITECTURE.md:32); this split has no
// counterpart there.
#include <cstring>
#include <stdexcept>

#include "server_internal.h"

struct ipir_shard {
    ipb::Server* s;
    ipb::Params global;
    size_t g0, g1;
};
struct ipir_horner {
    ipb::Server* s;
};

namespace ipb {
namespace {

std::shared_ptr<Precomp> owner_precomp(const Params& gp, const uint32_t* a_all) {
    auto P = std::make_shared<Precomp>();
    P->pp = gp;
    IPB_CK(cudaGetDevice(&P->device));
    cudaStream_t s = nullptr;
    IPB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
        P->tables = upload_tables(P->arena, s);
        P->pre_a = P->arena.alloc<uint32_t>(gp.n_packed * kGroupStrideA);
        IPB_CK(cudaMemcpyAsync(P->pre_a, a_all, gp.n_packed * kGroupStrideA * 4, cudaMemcpyHostToDevice, s));
        IPB_CK(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    return P;
}

int check_views(const ipir_query_view* qs, size_t count, bool need_db_parts, bool need_rgsw) {
    for (size_t i = 0; i < count; ++i) {
        const ipir_query_view& v = qs[i];
        if (need_db_parts && (!v.lwe_b_limb0 || !v.lwe_b_limb1 || !v.ksk5_b || !v.kskneg1_b)) return 3;
        if (need_rgsw && !v.rgsw) return 3;
    }
    return 0;
}

template <class F>
int shard_guarded(F&& f) {
    DeviceRestore keep_device;
    try {
        return f();
    } catch (const std::exception& e) {
        set_last_error(e.what());
    } catch (...) {
        set_last_error("unknown error");
    }
    return 4;
}

}  // namespace
}  // namespace ipb

extern "C" {

ipir_shard* ipir_b200_shard_create(size_t n_entries, size_t entry_bytes, size_t db_rows_or_zero, size_t max_batch,
                                   const uint16_t* db, const uint8_t* crs_seed, size_t group_lo, size_t group_hi,
                                   ipir_params* out_params) {
    if (!db || !crs_seed || !out_params || max_batch == 0) {
        ipb::set_last_error("ipir_b200_shard_create: null argument (the CRS seed is required) or max_batch == 0");
        return nullptr;
    }
    ipir_shard* out = nullptr;
    ipb::shard_guarded([&]() -> int {
        ipb::Params gp{};
        const char* why = nullptr;
        if (ipb::setup_geometry(n_entries, entry_bytes, db_rows_or_zero, &gp, &why) != 0)
            throw std::invalid_argument(why ? why : "setup rejected the geometry");
        std::memcpy(gp.seed, crs_seed, 64);
        auto P = ipb::run_preprocess_shard(gp, db, group_lo, group_hi);
        const ipb::Params local = P->pp;
        std::unique_ptr<ipb::Server> S(ipb::make_server(local, std::move(P), max_batch));
        ipb::fill_params(gp, out_params);
        out = new ipir_shard{S.release(), gp, group_lo, group_hi};
        return 0;
    });
    return out;
}

int ipir_b200_shard_export_a(const ipir_shard* sh, uint32_t* out) {
    if (!sh || !out) return 1;
    return ipb::shard_guarded([&]() -> int {
        const ipb::Server& S = *sh->s;
        IPB_CK(cudaSetDevice(S.device));
        IPB_CK(cudaMemcpy(out, S.pre->pre_a, S.pp.n_packed * ipb::kGroupStrideA * 4, cudaMemcpyDeviceToHost));
        return 0;
    });
}

int ipir_b200_shard_pack(ipir_shard* sh, const ipir_query_view* queries, size_t count, uint32_t* out_packed_b) {
    if (!sh || !queries || !out_packed_b) return 1;
    ipb::Server* S = sh->s;
    if (count > S->max_batch) return 2;
    if (int rc = ipb::check_views(queries, count, true, false)) return rc;
    if (count == 0) return 0;
    return ipb::shard_guarded([&]() -> int {
        IPB_CK(cudaSetDevice(S->device));
        ipb::Lane& L = S->lane;
        const ipb::Sched& sc = ipb::sched_for(*S, count);
        ipb::stage_parts(*S, queries, count, 0, 4, S->stream);  // LWE vectors and KSK parts; no RGSW
        const size_t ns = ipb::slices_of(count, sc), slice = sc.slice > 0 ? (size_t)sc.slice : count;
        for (size_t k = 0; k < ns; ++k) {
            const size_t q0 = k * slice;
            S->launches += (unsigned long long)ipb::run_db_phase(*S, L, sc, q0, std::min(slice, count - q0),
                                                                 S->stream, nullptr, nullptr, 1);
        }
        ipb::check_device_error(L, S->stream);  // nothing is written if a kernel stopped early
        IPB_CK(cudaMemcpyAsync(out_packed_b, L.packed_b, count * S->pb_qstride * 4, cudaMemcpyDeviceToDevice,
                               S->stream));
        IPB_CK(cudaStreamSynchronize(S->stream));
        return 0;
    });
}

int ipir_b200_shard_answer(ipir_shard* sh, const ipir_query_view* queries, size_t count, uint64_t* out_resp) {
    if (!sh || !queries || !out_resp) return 1;
    if (!ipb::shard_whole_cts(sh->global, sh->g0, sh->g1)) {
        ipb::set_last_error("ipir_b200_shard_answer: the shard's groups do not cover whole response ciphertexts");
        return 6;
    }
    // the shard handle is a server over its own groups: the plain pipeline
    // (with its Horner chains) answers its ciphertexts
    ipir_server tmp{sh->s};
    return ipir_answer_batch(&tmp, queries, count, out_resp);
}

void ipir_b200_shard_destroy(ipir_shard* sh) {
    if (!sh) return;
    ipb::DeviceRestore keep_device;
    delete sh->s;
    delete sh;
}

ipir_horner* ipir_b200_horner_create(const ipir_params* params, const uint32_t* a_all, size_t max_batch) {
    if (!params || !a_all || max_batch == 0) {
        ipb::set_last_error("ipir_b200_horner_create: null argument or max_batch == 0");
        return nullptr;
    }
    ipir_horner* out = nullptr;
    ipb::shard_guarded([&]() -> int {
        ipb::Params gp{};
        const char* why = nullptr;
        if (ipb::setup_geometry(params->n_entries, params->entry_bytes, params->db_rows, &gp, &why) != 0)
            throw std::invalid_argument(why ? why : "setup rejected the geometry");
        if (gp.db_cols != params->db_cols || gp.n_packed != params->n_packed || gp.num_cts != params->num_cts)
            throw std::invalid_argument("ipir_b200_horner_create: params inconsistent with setup()");
        std::memcpy(gp.seed, params->seed, 64);
        std::unique_ptr<ipb::Server> S(ipb::make_server(gp, ipb::owner_precomp(gp, a_all), max_batch));
        out = new ipir_horner{S.release()};
        return 0;
    });
    return out;
}

int ipir_b200_horner_answer(ipir_horner* h, const uint32_t* packed_b, const ipir_query_view* queries, size_t count,
                            uint64_t* out_resp, void* stream) {
    if (!h || !packed_b || !queries || !out_resp) return 1;
    ipb::Server* S = h->s;
    if (count > S->max_batch) return 2;
    if (int rc = ipb::check_views(queries, count, false, true)) return rc;
    if (count == 0) return 0;
    return ipb::shard_guarded([&]() -> int {
        IPB_CK(cudaSetDevice(S->device));
        ipb::Lane& L = S->lane;
        const ipb::Sched& sc = ipb::sched_for(*S, count);
        // packed_b was produced on the caller's stream (e.g. by the gather)
        IPB_CK(cudaEventRecord(L.fork, static_cast<cudaStream_t>(stream)));
        IPB_CK(cudaStreamWaitEvent(S->stream, L.fork, 0));
        ipb::stage_parts(*S, queries, count, 4, 1, S->stream);  // RGSW parts only
        IPB_CK(launch_qprep_parts(L.qraw, S->qstride, S->pp.db_rows, S->pre->tables, L.keys, L.rgsw32, (int)count,
                                  2, S->stream));
        const size_t ns = ipb::slices_of(count, sc), slice = sc.slice > 0 ? (size_t)sc.slice : count;
        for (size_t k = 0; k < ns; ++k) {
            const size_t q0 = k * slice, n = std::min(slice, count - q0);
            ipb::enqueue_horner(*S, sc, packed_b + q0 * S->pb_qstride, L.rgsw32 + q0 * ipb::kRgswStride,
                                L.resp + q0 * S->resp_qstride, n, L.d_err, S->stream);
        }
        S->launches += 1 + ns;
        ipb::check_device_error(L, S->stream);
        IPB_CK(cudaMemcpyAsync(out_resp, L.resp, count * S->resp_qstride * 8, cudaMemcpyDeviceToHost, S->stream));
        IPB_CK(cudaStreamSynchronize(S->stream));
        return 0;
    });
}

void ipir_b200_horner_destroy(ipir_horner* h) {
    if (!h) return;
    ipb::DeviceRestore keep_device;
    delete h->s;
    delete h;
}

}  // extern "C"
