// host_util.cpp -- host helpers of the B200 InsPIRe server: SHAKE-256 (FIPS
// 202) for the CRS expansion, NTT tables, and setup() geometry.
#include <cstdlib>
#include "host_util.h"

#include <cstring>
#include <mutex>
#include <map>
#include <utility>
#include <stdexcept>

namespace ipb {

// ------------------------------------------------------------------ SHAKE-256
// Keccak-f[1600] sponge, rate 136 bytes, domain padding 0x1F ... 0x80
// (FIPS 202).  The reference calls OpenSSL's EVP_shake256 for the same
// function (src/ring.cpp:252-279).
namespace {
const uint64_t kRC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808AULL, 0x8000000080008000ULL,
    0x000000000000808BULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008AULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000AULL,
    0x000000008000808BULL, 0x800000000000008BULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800AULL, 0x800000008000000AULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};
// rotation offsets r[x + 5y]
const int kRot[25] = {0, 1, 62, 28, 27, 36, 44, 6, 55, 20, 3, 10, 43, 25, 39,
                      41, 45, 15, 21, 8, 18, 2, 61, 56, 14};
inline uint64_t rotl(uint64_t v, int s) { return s ? (v << s) | (v >> (64 - s)) : v; }

void keccak_f(uint64_t a[25]) {
    for (int round = 0; round < 24; ++round) {
        uint64_t c[5], d[5], b[25];
        for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; ++x) d[x] = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
        for (int i = 0; i < 25; ++i) a[i] ^= d[i % 5];
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(a[x + 5 * y], kRot[x + 5 * y]);
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= kRC[round];
    }
}
inline void xor_byte(uint64_t a[25], size_t pos, uint8_t v) { a[pos / 8] ^= (uint64_t)v << (8 * (pos % 8)); }
inline uint8_t get_byte(const uint64_t a[25], size_t pos) { return (uint8_t)(a[pos / 8] >> (8 * (pos % 8))); }
}  // namespace

void shake256(const uint8_t* in, size_t inlen, uint8_t* out, size_t outlen) {
    constexpr size_t rate = 136;
    uint64_t a[25] = {0};
    size_t pos = 0;
    for (size_t i = 0; i < inlen; ++i) {
        xor_byte(a, pos++, in[i]);
        if (pos == rate) { keccak_f(a); pos = 0; }
    }
    xor_byte(a, pos, 0x1F);
    xor_byte(a, rate - 1, 0x80);
    keccak_f(a);
    pos = 0;
    for (size_t i = 0; i < outlen; ++i) {
        if (pos == rate) { keccak_f(a); pos = 0; }
        out[i] = get_byte(a, pos++);
    }
}

// expand_seed: H(seed || domain || le64(index)) -> 2N u64 words ->
// limb0[i] = w[i] % q0, limb1[i] = w[N+i] % q1 (src/ring.cpp:252-279).
void expand_seed(const uint8_t seed[kSeedBytes], const char* domain, uint64_t index, uint32_t* out) {
    uint8_t in[kSeedBytes + 64 + 8];
    const size_t dl = std::strlen(domain);
    if (dl > 64) throw std::invalid_argument("expand_seed: domain too long");
    std::memcpy(in, seed, kSeedBytes);
    std::memcpy(in + kSeedBytes, domain, dl);
    for (int i = 0; i < 8; ++i) in[kSeedBytes + dl + i] = (uint8_t)(index >> (8 * i));
    static thread_local uint8_t raw[2 * kN * 8];
    shake256(in, kSeedBytes + dl + 8, raw, sizeof raw);
    for (size_t i = 0; i < 2 * (size_t)kN; ++i) {
        uint64_t w = 0;
        for (int b = 0; b < 8; ++b) w |= (uint64_t)raw[8 * i + b] << (8 * b);
        out[i] = (uint32_t)(i < (size_t)kN ? w % kQ0 : w % kQ1);
    }
}

// ------------------------------------------------------------------ tables
namespace {
uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = (uint64_t)((unsigned __int128)r * b % q);
        b = (uint64_t)((unsigned __int128)b * b % q);
        e >>= 1;
    }
    return r;
}
uint32_t brev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i)
        if (x & (1u << i)) r |= 1u << (bits - 1 - i);
    return r;
}
uint32_t shoup(uint32_t w, uint32_t q) { return (uint32_t)(((uint64_t)w << 32) / q); }
}  // namespace

// psi = g^((q-1)/2N) for the smallest g >= 2 with psi^N = -1 (the reference's
// deterministic choice, src/ntt.cpp:56-69); fwd[i] = psi^BR(i),
// inv[i] = fwd[i]^-1, Shoup factors floor(w 2^32 / q).
void build_tables(DevTables& T) {
    const uint32_t qs[2] = {kQ0, kQ1};
    for (int l = 0; l < 2; ++l) {
        const uint64_t q = qs[l];
        const uint64_t ex = (q - 1) / (2 * kN);
        uint64_t psi = 0;
        for (uint64_t g = 2; g < q; ++g) {
            uint64_t c = powmod(g, ex, q);
            if (powmod(c, kN, q) == q - 1) { psi = c; break; }
        }
        LimbTables& L = T.limb[l];
        L.q = (uint32_t)q;
        for (uint32_t i = 0; i < (uint32_t)kN; ++i) {
            uint32_t w = (uint32_t)powmod(psi, brev(i, kLogN), q);
            uint32_t wi = i ? (uint32_t)powmod(w, q - 2, q) : 1u;
            L.fwd[i] = make_uint2(w, shoup(w, (uint32_t)q));
            L.inv[i] = make_uint2(wi, shoup(wi, (uint32_t)q));
        }
        L.inv_n = (uint32_t)powmod(kN, q - 2, q);
        L.inv_n_p = shoup(L.inv_n, (uint32_t)q);
        L.cr = ~0ULL / q;  // = floor(2^64 / q) since q does not divide 2^64
    }
    T.crt_c[0] = (uint32_t)powmod(kQ1 % kQ0, kQ0 - 2, kQ0);
    T.crt_c[1] = (uint32_t)powmod(kQ0 % kQ1, kQ1 - 2, kQ1);
    T.crt_cp[0] = shoup(T.crt_c[0], kQ0);
    T.crt_cp[1] = shoup(T.crt_c[1], kQ1);
}

// ------------------------------------------------------------------ setup
// Mirror of src/params.cpp:23-68: coeffs_per_entry = ceil(8w/15), db_cols =
// ceil(N_entries*cpe/db_rows) rounded up to a multiple of N, n_packed =
// db_cols/N, num_cts = max(1, n_packed/D), D = 256, plus the reference's
// three geometry checks (it throws std::invalid_argument on each).
// The CRS seed is left zero here; callers fill it.
int setup_geometry(size_t n_entries, size_t w, size_t db_rows, Params* out, const char** why) {
    const char* dummy;
    if (!why) why = &dummy;
    if (!out) { *why = "null output"; return 1; }
    if (db_rows == 0) db_rows = kDefaultDbRows;
    Params pp{};
    pp.n_entries = n_entries;
    pp.w = w;
    pp.D = kDmax;
    pp.db_rows = db_rows;
    const size_t cpe = (w * 8 + kPBits - 1) / kPBits;
    if (cpe == 0) { *why = "setup: entry size must be > 0"; return 1; }
    const size_t total = n_entries * cpe;
    const size_t cols = (total + db_rows - 1) / db_rows;
    pp.db_cols = ((cols + kN - 1) / kN) * kN;
    if (pp.db_cols == 0) pp.db_cols = kN;
    pp.n_packed = pp.db_cols / kN;
    pp.num_cts = pp.n_packed / pp.D > 1 ? pp.n_packed / pp.D : 1;
    if (kN % cpe != 0) { *why = "setup: ceil(8*w/15) must divide N=2048"; return 2; }
    const size_t d_act = pp.D < pp.n_packed ? pp.D : pp.n_packed;
    if ((2 * kN) % d_act != 0) { *why = "setup: n_packed must be a power of two"; return 3; }
    if (pp.n_packed > pp.D && pp.n_packed % pp.D != 0) { *why = "setup: n_packed must be a multiple of D"; return 4; }
    // Device-side layout requirements of this server (the reference's
    // kernels assume the same: rows come in whole polys of N).
    if (db_rows % kN != 0 || (db_rows & (db_rows - 1)) != 0) {
        *why = "setup: db_rows must be a power of two and a multiple of N=2048";
        return 5;
    }
    *out = pp;
    return 0;
}

cudaError_t allow_max_dynamic_smem(const void* kernel, size_t* max_dynamic) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find({kernel, dev});
    if (it == done.end()) {
        int optin = 0;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
        cudaFuncAttributes fa{};
        if ((e = cudaFuncGetAttributes(&fa, kernel))) return e;
        const int dyn = optin - (int)fa.sharedSizeBytes;
        if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn))) return e;
        it = done.emplace(std::make_pair(kernel, dev), (size_t)dyn).first;
    }
    if (max_dynamic) *max_dynamic = it->second;
    return cudaSuccess;
}

int test_abort_after_items() {
    const char* v = std::getenv("IPB_TEST_ABORT_AFTER_ITEMS");
    const int n = v ? std::atoi(v) : 0;
    return n > 0 ? n : 0;
}

}  // namespace ipb
