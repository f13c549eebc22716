// A C++ consumer of the reference's server API, written only against the
// reference's own headers (src/gpu_protocol.h, src/protocol.h) the way its
// tests/test_e2e_gpu.cu and tests/test_gpu_batch.cu drive the server:
// setup -> gpu_preprocess -> gpu_setup_server -> query() -> gpu_answer ->
// extract(), gpu_answer_batch == singles, gpu_server_caps, gpu_free_server.
// Test infrastructure: oracle/Makefile builds it twice from this one source,
// linked against this project's libinspire_b200_refapi.so and against the
// reference's own GPU library, and tests/test_gpu_ref_cpp_api.py runs both.
//
// usage: ref_consumer n_entries entry_bytes db_rows(0 = default) n_queries
// prints "ok ..." and exits 0 when every check passes.
#include <cuda_runtime.h>

#include "gpu_protocol.h"

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

using namespace inspire;

static int fail(const char* what, size_t i) {
    std::printf("FAIL %s (query %zu)\n", what, i);
    return 1;
}

static bool same_ct(const std::vector<RlweCt>& x, const std::vector<RlweCt>& y) {
    if (x.size() != y.size()) return false;
    for (size_t c = 0; c < x.size(); ++c)
        if (x[c].a.limbs != y[c].a.limbs || x[c].b.limbs != y[c].b.limbs) return false;
    return true;
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::printf("usage: %s n_entries entry_bytes db_rows n_queries\n", argv[0]);
        return 2;
    }
    const size_t n_entries = std::strtoull(argv[1], nullptr, 10), w = std::strtoull(argv[2], nullptr, 10);
    const size_t rows = std::strtoull(argv[3], nullptr, 10), nq = std::strtoull(argv[4], nullptr, 10);
    PublicParams pp = rows ? setup(n_entries, w, rows) : setup(n_entries, w);
    std::mt19937_64 rng(42);
    std::vector<uint16_t> db(pp.db_rows * pp.db_cols);
    for (auto& v : db) v = (uint16_t)(rng() % P);

    PreprocessData pre = gpu_preprocess(pp, db.data());
    GpuServerConfig cfg;
    cfg.max_batch = nq;
    GpuServerCtx* ctx = gpu_setup_server(pp, pre, cfg);
    if (pre.d_db_col != nullptr || !pre.d_precomp_a.empty()) return fail("setup did not adopt the precomp", 0);
    const GpuServerCaps caps = gpu_server_caps(ctx);
    if (caps.max_batch != nq || caps.num_cts != pp.num_cts || caps.resident_bytes == 0)
        return fail("caps", 0);

    const size_t cpe = (pp.w * 8 + P_BITS - 1) / P_BITS;
    std::vector<QueryState> st;
    std::vector<QueryMessage> qs;
    std::vector<size_t> idx;
    for (size_t i = 0; i < nq; ++i) {
        idx.push_back(i + 1 < nq ? rng() % pp.N_entries : idx[0]);  // the last repeats the first index
        auto q = query(pp, idx.back());
        st.push_back(q.first);
        qs.push_back(q.second);
    }
    std::vector<std::vector<RlweCt>> singles;
    for (size_t i = 0; i < nq; ++i) {
        singles.push_back(gpu_answer(ctx, qs[i]));
        const std::vector<uint16_t> got = extract(pp, st[i], singles[i]);
        const size_t i_star = idx[i] % pp.db_rows, col = (idx[i] / pp.db_rows) * cpe;
        if (got.size() != cpe) return fail("extract length", i);
        for (size_t c = 0; c < cpe; ++c)
            if (got[c] != db[i_star * pp.db_cols + col + c] % P) return fail("extract value", i);
    }
    const auto batch = gpu_answer_batch(ctx, qs);  // the inline vector overload
    if (batch.size() != nq) return fail("batch size", 0);
    for (size_t i = 0; i < nq; ++i)
        if (!same_ct(batch[i], singles[i])) return fail("batch != single", i);
    if (nq > 1 && same_ct(singles[0], singles[nq - 1])) return fail("repeated index, fresh keys, same ciphertext", 0);
    gpu_free_server(ctx);
    std::printf("ok %zu queries, db %zu x %zu, %zu ct(s)\n", nq, pp.db_rows, pp.db_cols, pp.num_cts);
    return 0;
}
