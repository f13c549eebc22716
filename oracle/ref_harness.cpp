// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Thin extern "C" wrappers over the reference's own CPU library (params,
// ntt, ring, crypto, protocol, capi_client), compiled from the reference's
// sources into oracle/_ref/libinspire_ref.so by oracle/Makefile.  Tests use
// it to (1) build seeded queries with the reference client, (2) extract
// responses with the reference client, and (3) pin the oracle's primitives
// against the reference's NTT, decomp, expand_seed, automorphism, ext_prod
// and horner_eval.  The product library never loads it.
#include "protocol.h"
#include "crypto.h"
#include "ring.h"
#include "ntt.h"
#include "params.h"
#include <cstring>
#include <new>
#include <random>

using namespace inspire;

namespace {
RnsPoly poly_from(const uint64_t* src, bool ntt) {
    RnsPoly p = RnsPoly::zero();
    for (size_t i = 0; i < N; i++) { p.limbs[0][i] = src[i]; p.limbs[1][i] = src[N + i]; }
    p.is_ntt = ntt;
    return p;
}
void poly_to(const RnsPoly& p, uint64_t* dst) {
    for (size_t i = 0; i < N; i++) { dst[i] = p.limbs[0][i]; dst[N + i] = p.limbs[1][i]; }
}
// [digit][limb][coeff] flatten, as capi_client.cpp:56-66 does.
uint64_t* flatten(uint64_t* dst, const std::vector<RnsPoly>& parts, bool want_ntt) {
    for (const RnsPoly& p0 : parts) {
        RnsPoly p = p0;
        if (want_ntt && !p.is_ntt) p.to_ntt();
        if (!want_ntt && p.is_ntt) p.to_coeff();
        poly_to(p, dst);
        dst += 2 * N;
    }
    return dst;
}
std::vector<RnsPoly> parts_from(const uint64_t* src, bool ntt) {
    std::vector<RnsPoly> v(D_EFF);
    for (int j = 0; j < D_EFF; j++) v[j] = poly_from(src + (size_t)j * 2 * N, ntt);
    return v;
}
RgswCt rgsw_from(const uint64_t* src) {
    const size_t blk = (size_t)D_EFF * 2 * N;
    RgswCt r;
    r.top.a_parts = parts_from(src + 0 * blk, true);
    r.top.b_parts = parts_from(src + 1 * blk, true);
    r.bottom.a_parts = parts_from(src + 2 * blk, true);
    r.bottom.b_parts = parts_from(src + 3 * blk, true);
    return r;
}
struct State { QueryState st; PublicParams pp; };
PublicParams pp_from(const uint64_t* g, const uint8_t* seed) {
    PublicParams pp;
    pp.N_entries = g[0]; pp.w = g[1]; pp.db_rows = g[2]; pp.db_cols = g[3];
    pp.n_packed = g[4]; pp.D = g[5]; pp.num_cts = g[6];
    std::memcpy(pp.seed.data(), seed, SEED_BYTES);
    return pp;
}
}  // namespace

extern "C" {

// setup() -> geometry [N_entries, w, db_rows, db_cols, n_packed, D, num_cts].
// Returns 0, or 1 when setup() throws (unsupported geometry).
int refh_setup(uint64_t n_entries, uint64_t w, uint64_t db_rows, uint64_t* out) {
    try {
        PublicParams pp = db_rows ? setup(n_entries, w, db_rows) : setup(n_entries, w);
        out[0] = pp.N_entries; out[1] = pp.w; out[2] = pp.db_rows; out[3] = pp.db_cols;
        out[4] = pp.n_packed; out[5] = pp.D; out[6] = pp.num_cts;
        return 0;
    } catch (...) {
        return 1;
    }
}

// query() of protocol.cpp:12-52 with the rng seeded (the reference draws it
// from std::random_device).  Writes the flat query of capi.h:109-112 and
// returns the client state for refh_extract.
void* refh_query(const uint64_t* geom, const uint8_t* crs_seed, uint64_t idx,
                 uint64_t rng_seed, uint64_t* out_flat) {
    try {
        PublicParams pp = pp_from(geom, crs_seed);
        std::mt19937_64 rng(rng_seed);
        size_t i_star = idx % pp.db_rows;
        size_t cpe = (pp.w * 8 + P_BITS - 1) / P_BITS;
        size_t col = (idx / pp.db_rows) * cpe;
        size_t Da = std::min(pp.D, pp.n_packed);
        size_t j_star = (col / N) % Da;
        size_t k_star = col / (N * Da);
        size_t ell_star = col % N;
        RnsPoly s = sk_gen(rng);
        RnsPoly s_ntt = s; s_ntt.to_ntt();
        Ksk k5 = ksk_gen_b(s, AUTO_GEN, pp.seed.data(), rng);
        Ksk kn1 = ksk_gen_b(s, 2 * N - 1, pp.seed.data(), rng);
        LweQuery lwe = lwe_enc_b(s, i_star, pp.db_rows, pp.seed.data(), rng);
        RnsPoly mu = RnsPoly::zero();
        size_t e = (j_star * 2 * N) / Da;
        if (e == 0) mu.set_coeff(0, 1, 1);
        else if (e < N) mu.set_coeff(e, 1, 1);
        else mu.set_coeff(e - N, Q0 - 1, Q1 - 1);
        RgswCt rg = rgsw_enc_b(s, mu, pp.seed.data(), rng);
        uint64_t* w = out_flat;
        std::memcpy(w, lwe.b_limb0.data(), pp.db_rows * 8); w += pp.db_rows;
        std::memcpy(w, lwe.b_limb1.data(), pp.db_rows * 8); w += pp.db_rows;
        w = flatten(w, k5.b_parts, false);
        w = flatten(w, kn1.b_parts, false);
        w = flatten(w, rg.top.a_parts, true);
        w = flatten(w, rg.top.b_parts, true);
        w = flatten(w, rg.bottom.a_parts, true);
        w = flatten(w, rg.bottom.b_parts, true);
        State* st = new State{QueryState{s, s_ntt, k_star, ell_star}, pp};
        return st;
    } catch (...) {
        return nullptr;
    }
}

// extract() of protocol.cpp:58-71 on a flat response [ct][a|b][limb][N].
int refh_extract(void* state, const uint64_t* resp, uint16_t* out_slots, uint64_t* n_out) {
    State* st = static_cast<State*>(state);
    if (!st) return 1;
    std::vector<RlweCt> cts(st->pp.num_cts);
    for (size_t g = 0; g < st->pp.num_cts; g++) {
        cts[g].a = poly_from(resp + g * 4 * N, true);
        cts[g].b = poly_from(resp + g * 4 * N + 2 * N, true);
    }
    std::vector<uint16_t> s = extract(st->pp, st->st, cts);
    std::memcpy(out_slots, s.data(), s.size() * 2);
    *n_out = s.size();
    return 0;
}

// rlwe_dec of response ct k* -> all N plaintext coefficients (noise checks).
int refh_decrypt(void* state, const uint64_t* resp, uint64_t* out_m) {
    State* st = static_cast<State*>(state);
    if (!st) return 1;
    RlweCt ct;
    ct.a = poly_from(resp + st->st.k_star * 4 * N, true);
    ct.b = poly_from(resp + st->st.k_star * 4 * N + 2 * N, true);
    std::vector<uint64_t> m = rlwe_dec(st->st.s_ntt, ct);
    std::memcpy(out_m, m.data(), N * 8);
    return 0;
}

// extract_compressed() of src/protocol.cpp on compressed response bytes in
// the client library's layout (src/capi_client.cpp:360-385): per ciphertext
// N x 28-bit mask values then N x 20-bit body values, MSB first.
int refh_extract_compressed(void* state, const uint8_t* in, uint16_t* out_slots, uint64_t* n_out) {
    State* st = static_cast<State*>(state);
    if (!st || !in) return 1;
    std::vector<CompressedCt> cts(st->pp.num_cts);
    uint64_t acc = 0;
    int nbits = 0;
    auto get = [&](int bits) -> uint32_t {
        while (nbits < bits) {
            acc = (acc << 8) | *in++;
            nbits += 8;
        }
        nbits -= bits;
        uint32_t v = (uint32_t)(acc >> nbits);
        acc &= (1ULL << nbits) - 1;
        return v;
    };
    for (size_t g = 0; g < st->pp.num_cts; g++) {
        cts[g].a.resize(N);
        cts[g].b.resize(N);
        for (size_t i = 0; i < N; i++) cts[g].a[i] = get(28);
        for (size_t i = 0; i < N; i++) cts[g].b[i] = get(20);
    }
    std::vector<uint16_t> s = extract_compressed(st->pp, st->st, cts);
    std::memcpy(out_slots, s.data(), s.size() * 2);
    *n_out = s.size();
    return 0;
}

void refh_state_free(void* state) { delete static_cast<State*>(state); }

void refh_ntt_forward(uint64_t* data, int limb) { ntt_forward(data, limb); }
void refh_ntt_inverse(uint64_t* data, int limb) { ntt_inverse(data, limb); }

void refh_ntt_tables(int limb, uint64_t* fwd, uint64_t* inv, uint64_t* inv_n, uint64_t* psi) {
    const NttTables& t = ntt_tables(limb);
    std::memcpy(fwd, t.fwd_twiddles.data(), N * 8);
    std::memcpy(inv, t.inv_twiddles.data(), N * 8);
    *inv_n = t.inv_n;
    *psi = t.psi;
}

// decomp(f) with f [limb][N] coefficient form -> [digit][limb][N].
void refh_decomp(const uint64_t* f, uint64_t* out) {
    std::vector<RnsPoly> d = decomp(poly_from(f, false));
    for (int j = 0; j < D_EFF; j++) poly_to(d[j], out + (size_t)j * 2 * N);
}

void refh_expand_seed(const uint8_t* seed, const char* domain, uint64_t index, uint64_t* out) {
    poly_to(expand_seed(seed, domain, index), out);
}

void refh_automorphism_ntt(const uint64_t* f_ntt, uint64_t k, uint64_t* out) {
    poly_to(automorphism_ntt(poly_from(f_ntt, true), k), out);
}

// ext_prod(rgsw, ct): rgsw [top_a|top_b|bot_a|bot_b][digit][limb][N] NTT form,
// ct [a|b][limb][N] NTT form -> out [a|b][limb][N] NTT form.
void refh_ext_prod(const uint64_t* rgsw, const uint64_t* ct, uint64_t* out) {
    RlweCt c;
    c.a = poly_from(ct, true);
    c.b = poly_from(ct + 2 * N, true);
    RlweCt r = ext_prod(rgsw_from(rgsw), c);
    poly_to(r.a, out);
    poly_to(r.b, out + 2 * N);
}

void refh_horner_eval(const uint64_t* rgsw, const uint64_t* cts, uint64_t L, uint64_t* out) {
    std::vector<RlweCt> v(L);
    for (size_t i = 0; i < L; i++) {
        v[i].a = poly_from(cts + i * 4 * N, true);
        v[i].b = poly_from(cts + i * 4 * N + 2 * N, true);
    }
    RlweCt r = horner_eval(v, rgsw_from(rgsw), L);
    poly_to(r.a, out);
    poly_to(r.b, out + 2 * N);
}

}  // extern "C"
