// inspire_ref_api.cpp -- the reference's C++ server API, on its own types.
//
// Defines, with the exact signatures of SoraSuegami/InsPIRe-GPU
// src/gpu_protocol.h:44-78, the functions a C++ consumer of that project
// calls:
//
//   inspire::gpu_preprocess(const PublicParams&, const uint16_t* db) -> PreprocessData
//   inspire::gpu_setup_server(pp, precomp[, GpuServerConfig])       -> GpuServerCtx*
//   inspire::gpu_server_caps(const GpuServerCtx*)                   -> GpuServerCaps
//   inspire::gpu_answer(GpuServerCtx*, const QueryMessage&)         -> std::vector<RlweCt>
//   inspire::gpu_answer_batch(GpuServerCtx*, const QueryMessage*, size_t)
//   inspire::gpu_free_server(GpuServerCtx*)
//
// so that such a consumer (its CPU client query()/extract(), its types from
// the reference's protocol.h / crypto.h / ring.h) builds unchanged and links
// against this library instead of the reference's GPU library.  It is
// compiled against the reference's own headers (the types must be the
// consumer's), so it is built only where those headers are given
// (inspire-gpu_b200/Makefile target refapi, REF=<the reference's src/>).
// The out-of-line members of those types it uses (RnsPoly's constructor and
// domain conversions) resolve from the reference CPU library the consumer
// already links.
//
// Underneath are this project's own server (include/inspire_b200.hpp): the
// queries are flattened as the reference's C ABI lays them out
// (src/capi_client.cpp:56-66: [b limb0][b limb1][ksk5][ksk-1][rgsw],
// parts [digit][limb][coeff], KSK parts in coefficient form, RGSW parts in
// NTT form) and the flat NTT-form responses are rebuilt as RlweCt.
//
// Differences from the reference, by design: errors throw
// (std::invalid_argument, std::runtime_error) where the reference calls
// exit(1); PreprocessData's per-group D_plus / D_minus pointers are null
// (those tensors live as tensor-core byte planes; ipir_b200_export_precomp
// gives them in the reference layout); its a / D_final / DB pointers are the
// device buffers, adopted by gpu_setup_server, which clears the caller's
// struct as the reference does (src/gpu_protocol.cu:856-885).
#include <cuda_runtime.h>   // the reference's gpu.cuh (included by gpu_protocol.h) names cudaStream_t

#include "gpu_protocol.h"  // the reference's declarations and types

#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <utility>

#include "inspire_b200.hpp"

namespace inspire {

struct GpuServerCtx {
    inspire_b200::GpuServerCtx* s = nullptr;
    PublicParams pp;
    size_t max_batch = 0;
    std::vector<uint64_t> flat;  // staging for one batch of flattened queries
    std::vector<uint64_t> resp;  // flat responses of one batch
};

namespace {

// Preprocess results not yet adopted, by their device DB pointer (the key a
// PreprocessData carries).
std::mutex g_mu;
std::map<const uint16_t*, inspire_b200::PreprocessData> g_pending;

inspire_b200::PublicParams to_b200(const PublicParams& pp) {
    inspire_b200::PublicParams p;
    p.N_entries = pp.N_entries;
    p.w = pp.w;
    p.db_rows = pp.db_rows;
    p.db_cols = pp.db_cols;
    p.n_packed = pp.n_packed;
    p.D = pp.D;
    p.num_cts = pp.num_cts;
    static_assert(sizeof(p.seed) == SEED_BYTES, "seed size");
    std::memcpy(p.seed.data(), pp.seed.data(), SEED_BYTES);
    return p;
}

constexpr size_t kBlk = (size_t)D_EFF * 2 * N;  // one part vector: [digit][limb][coeff]

size_t query_u64s(const PublicParams& pp) { return 2 * pp.db_rows + 6 * kBlk; }

// [digit][limb][coeff] of a part vector, converted to the wanted domain
// (a copy, through the type's own conversions, only when it is not there).
uint64_t* flatten_parts(uint64_t* dst, const std::vector<RnsPoly>& parts, bool want_ntt, const char* what) {
    if (parts.size() != (size_t)D_EFF) throw std::invalid_argument(std::string("gpu_answer: ") + what + " parts");
    for (const RnsPoly& p0 : parts) {
        const RnsPoly* p = &p0;
        RnsPoly conv;
        if (p0.is_ntt != want_ntt) {
            conv = p0;
            if (want_ntt) conv.to_ntt(); else conv.to_coeff();
            p = &conv;
        }
        for (int l = 0; l < 2; ++l) {
            if (p->limbs[l].size() != N) throw std::invalid_argument(std::string("gpu_answer: ") + what + " length");
            std::memcpy(dst, p->limbs[l].data(), N * sizeof(uint64_t));
            dst += N;
        }
    }
    return dst;
}

void flatten_query(const PublicParams& pp, const QueryMessage& q, uint64_t* dst) {
    const size_t R = pp.db_rows;
    if (q.lwe.b_limb0.size() != R || q.lwe.b_limb1.size() != R)
        throw std::invalid_argument("gpu_answer: LWE vector length differs from db_rows");
    std::memcpy(dst, q.lwe.b_limb0.data(), R * sizeof(uint64_t));
    std::memcpy(dst + R, q.lwe.b_limb1.data(), R * sizeof(uint64_t));
    uint64_t* w = dst + 2 * R;
    w = flatten_parts(w, q.ksk_5.b_parts, false, "ksk_5");
    w = flatten_parts(w, q.ksk_neg1.b_parts, false, "ksk_neg1");
    w = flatten_parts(w, q.rgsw.top.a_parts, true, "rgsw top a");
    w = flatten_parts(w, q.rgsw.top.b_parts, true, "rgsw top b");
    w = flatten_parts(w, q.rgsw.bottom.a_parts, true, "rgsw bottom a");
    flatten_parts(w, q.rgsw.bottom.b_parts, true, "rgsw bottom b");
}

ipir_query_view view_of(const PublicParams& pp, const uint64_t* flat) {
    const size_t R = pp.db_rows;
    ipir_query_view v;
    v.lwe_b_limb0 = flat;
    v.lwe_b_limb1 = flat + R;
    v.ksk5_b = flat + 2 * R;
    v.kskneg1_b = flat + 2 * R + kBlk;
    v.rgsw = flat + 2 * R + 2 * kBlk;
    return v;
}

void fill_poly(RnsPoly& p, const uint64_t* src) {
    for (int l = 0; l < 2; ++l) p.limbs[l].assign(src + (size_t)l * N, src + (size_t)(l + 1) * N);
    p.is_ntt = true;
}

// One query's flat response [ct][a|b][limb][coeff] (NTT form) as RlweCt.
std::vector<RlweCt> unflatten_response(const uint64_t* src, size_t num_cts) {
    std::vector<RlweCt> out(num_cts);
    for (size_t c = 0; c < num_cts; ++c) {
        fill_poly(out[c].a, src + c * 4 * N);
        fill_poly(out[c].b, src + c * 4 * N + 2 * N);
    }
    return out;
}

}  // namespace

PreprocessData gpu_preprocess(const PublicParams& pp, const uint16_t* db) {
    inspire_b200::PreprocessData d = inspire_b200::gpu_preprocess(to_b200(pp), db);
    const inspire_b200::PreprocessDevicePointers ptr = inspire_b200::preprocess_device_pointers(d);
    PreprocessData out;
    out.d_db_col = ptr.db;
    out.d_precomp_a.resize(pp.n_packed);
    out.d_precomp_D_final.resize(pp.n_packed);
    out.d_precomp_D_plus.assign(pp.n_packed, nullptr);
    out.d_precomp_D_minus.assign(pp.n_packed, nullptr);
    for (size_t g = 0; g < pp.n_packed; ++g) {
        out.d_precomp_a[g] = ptr.a + g * ptr.a_group_stride;
        out.d_precomp_D_final[g] = ptr.d_final + g * ptr.d_final_group_stride;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_pending[ptr.db] = std::move(d);
    return out;
}

GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp, const GpuServerConfig& cfg) {
    inspire_b200::PreprocessData d;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_pending.find(precomp.d_db_col);
        if (!precomp.d_db_col || it == g_pending.end())
            throw std::invalid_argument("gpu_setup_server: PreprocessData not from gpu_preprocess or already adopted");
        d = std::move(it->second);
        g_pending.erase(it);
    }
    inspire_b200::GpuServerConfig c;
    c.max_batch = cfg.max_batch;
    auto* ctx = new GpuServerCtx;
    try {
        ctx->s = inspire_b200::gpu_setup_server(to_b200(pp), d, c);
    } catch (...) {
        delete ctx;
        throw;
    }
    ctx->pp = pp;
    ctx->max_batch = cfg.max_batch;
    // Ownership moved to the context: clear the caller's pointers, as the
    // reference does (src/gpu_protocol.cu:856-885).
    PreprocessData& mut = const_cast<PreprocessData&>(precomp);
    mut.d_db_col = nullptr;
    mut.d_precomp_a.clear();
    mut.d_precomp_D_plus.clear();
    mut.d_precomp_D_minus.clear();
    mut.d_precomp_D_final.clear();
    return ctx;
}

GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp) {
    return gpu_setup_server(pp, precomp, GpuServerConfig{});
}

GpuServerCaps gpu_server_caps(const GpuServerCtx* ctx) {
    GpuServerCaps c{};
    if (!ctx) return c;
    const inspire_b200::GpuServerCaps b = inspire_b200::gpu_server_caps(ctx->s);
    c.max_batch = b.max_batch;
    c.resident_bytes = b.resident_bytes;
    c.device_free_bytes = b.device_free_bytes;
    c.num_cts = b.num_cts;
    return c;
}

std::vector<std::vector<RlweCt>> gpu_answer_batch(GpuServerCtx* ctx, const QueryMessage* queries, size_t count) {
    if (!ctx) throw std::invalid_argument("gpu_answer_batch: null ctx");
    if (count == 0) return {};
    if (!queries) throw std::invalid_argument("gpu_answer_batch: null queries");
    if (count > ctx->max_batch)
        throw std::invalid_argument("gpu_answer_batch: count exceeds max_batch (set GpuServerConfig.max_batch)");
    // All or nothing: every query is validated and flattened before any
    // device work; one host array, so each part side crosses in one copy.
    const size_t qn = query_u64s(ctx->pp), rn = ctx->pp.num_cts * 4 * N;
    ctx->flat.resize(count * qn);
    std::vector<ipir_query_view> views(count);
    for (size_t i = 0; i < count; ++i) {
        flatten_query(ctx->pp, queries[i], ctx->flat.data() + i * qn);
        views[i] = view_of(ctx->pp, ctx->flat.data() + i * qn);
    }
    ctx->resp.resize(count * rn);
    inspire_b200::gpu_answer_batch(ctx->s, views.data(), count, ctx->resp.data());
    std::vector<std::vector<RlweCt>> out(count);
    for (size_t i = 0; i < count; ++i) out[i] = unflatten_response(ctx->resp.data() + i * rn, ctx->pp.num_cts);
    return out;
}

std::vector<RlweCt> gpu_answer(GpuServerCtx* ctx, const QueryMessage& qry) {
    std::vector<std::vector<RlweCt>> r = gpu_answer_batch(ctx, &qry, 1);
    return std::move(r[0]);
}

void gpu_free_server(GpuServerCtx* ctx) {
    if (!ctx) return;
    inspire_b200::gpu_free_server(ctx->s);
    delete ctx;
}

}  // namespace inspire
