/*
 * inspire_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the InsPIRe server path (preprocess + answer) of the
 * reference implementation (SoraSuegami/InsPIRe-GPU).  It is the checker the
 * CUDA server is compared against, and the timed CPU baseline of bench.py.
 * Nothing in the product library links, loads or calls this file.
 *
 * The reference has no CPU server (docs/ARCHITECTURE.md:378-380), so the
 * algorithm is restated from its GPU kernels, which define the bit-exact
 * outputs, and from its CPU primitives:
 *   NTT                      src/ntt.cpp:56-149
 *   decomp                   src/ring.cpp:205-246
 *   expand_seed (SHAKE-256)  src/ring.cpp:252-279   (OpenSSL EVP, as the reference)
 *   encode (inverse DFT)     src/gpu_preprocess.cu:931-1070
 *   CRS polys                src/gpu_protocol.cu:569-582
 *   a-side matmul            src/gpu_preprocess.cu:347-410
 *   ring_embed + perms       src/gpu_preprocess.cu:39-92, 158-194
 *   ExpandKSK_a              src/gpu_protocol.cu:364-474, src/gpu_preprocess.cu:228-270
 *   CollapseA                src/gpu_preprocess.cu:452-881
 *   mat-vec                  src/gpu_online.cu:23-41
 *   per-group pack           src/gpu_protocol.cu:1225-1283, src/gpu_online.cu:547-632
 *   perm tables              src/gpu_protocol.cu:169-215
 *   ext_prod / Horner        src/crypto.cpp:219-279, src/gpu_protocol.cu:1300-1334
 *
 * Pinning: tests/ check every primitive here against the reference's own CPU
 * code compiled from its sources (oracle/_ref, see oracle/Makefile), the
 * literal ring-embed against the NTT-based one, and the full pipeline
 * end to end through the reference's unmodified client extract().
 *
 * All arithmetic is exact: residues are canonical u64 values < q.
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <openssl/evp.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_N 2048
#define ORC_LOGN 11
#define ORC_HALF 1024
#define ORC_NSTEPS 1023
#define ORC_DGSW 3
#define ORC_DEFF 2
#define ORC_BASE_LOG 18
static const uint64_t Q[2] = {94519297ULL, 95293441ULL}; /* src/params.h:16-17 */
#define ORC_P 65535ULL                                   /* src/params.h:23 */

typedef unsigned __int128 u128;

/* ---------------------------------------------------------------- tables */
static uint64_t g_fwd[2][ORC_N], g_inv[2][ORC_N], g_inv_n[2], g_psi[2];
static uint64_t g_q1_inv_q0, g_q0_inv_q1;
static int g_init = 0;

static inline uint64_t mulmod(uint64_t a, uint64_t b, int limb) {
    /* a,b < q < 2^27 so a*b < 2^54; constant divisors per branch. */
    return limb ? (a * b) % 95293441ULL : (a * b) % 94519297ULL;
}
static inline uint64_t addmod(uint64_t a, uint64_t b, int limb) {
    uint64_t s = a + b;
    return s >= Q[limb] ? s - Q[limb] : s;
}
static inline uint64_t submod(uint64_t a, uint64_t b, int limb) {
    return a >= b ? a - b : a + Q[limb] - b;
}
static uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = (uint64_t)((u128)r * b % q);
        b = (uint64_t)((u128)b * b % q);
        e >>= 1;
    }
    return r;
}
static uint32_t brev11(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < ORC_LOGN; i++)
        if (x & (1u << i)) r |= 1u << (ORC_LOGN - 1 - i);
    return r;
}
static uint64_t modinv_u64(uint64_t a, uint64_t m) {
    int64_t old_r = (int64_t)(a % m), r = (int64_t)m, old_s = 1, s = 0;
    while (r != 0) {
        int64_t qq = old_r / r, t = r;
        r = old_r - qq * r; old_r = t;
        t = s; s = old_s - qq * s; old_s = t;
    }
    return (uint64_t)((old_s % (int64_t)m + (int64_t)m) % (int64_t)m);
}

/* Tables follow src/ntt.cpp:56-94: psi from the smallest g >= 2 whose
 * g^((q-1)/2N) has order 2N; fwd[i] = psi^BR(i); inv[i] = fwd[i]^-1. */
int orc_init(void) {
    if (g_init) return 0;
    for (int l = 0; l < 2; l++) {
        uint64_t q = Q[l], ex = (q - 1) / (2 * ORC_N);
        for (uint64_t g = 2; g < q; g++) {
            uint64_t psi = powmod(g, ex, q);
            if (powmod(psi, ORC_N, q) == q - 1) { g_psi[l] = psi; break; }
        }
        for (uint32_t i = 0; i < ORC_N; i++) g_fwd[l][i] = powmod(g_psi[l], brev11(i), q);
        g_inv[l][0] = 1;
        for (uint32_t i = 1; i < ORC_N; i++) g_inv[l][i] = powmod(g_fwd[l][i], q - 2, q);
        g_inv_n[l] = powmod(ORC_N, q - 2, q);
    }
    g_q1_inv_q0 = modinv_u64(Q[1], Q[0]);
    g_q0_inv_q1 = modinv_u64(Q[0], Q[1]);
    g_init = 1;
    return 0;
}

void orc_get_tables(uint64_t* fwd, uint64_t* inv, uint64_t* inv_n, uint64_t* psi) {
    orc_init();
    memcpy(fwd, g_fwd, sizeof g_fwd);
    memcpy(inv, g_inv, sizeof g_inv);
    inv_n[0] = g_inv_n[0]; inv_n[1] = g_inv_n[1];
    psi[0] = g_psi[0]; psi[1] = g_psi[1];
}

/* --------------------------------------------------------------- NTT */
/* Forward negacyclic CT-DIT, src/ntt.cpp:107-125. */
void orc_ntt_forward(uint64_t* a, int limb) {
    const uint64_t* w = g_fwd[limb];
    for (size_t m = 1; m < ORC_N; m <<= 1) {
        size_t t = ORC_N / (2 * m);
        for (size_t gi = 0; gi < m; gi++) {
            uint64_t tw = w[m + gi];
            uint64_t* x = a + gi * 2 * t;
            for (size_t p = 0; p < t; p++) {
                uint64_t u = x[p], v = mulmod(x[p + t], tw, limb);
                x[p] = addmod(u, v, limb);
                x[p + t] = submod(u, v, limb);
            }
        }
    }
}

/* Inverse GS, src/ntt.cpp:127-149 (N^-1 scaling included). */
void orc_ntt_inverse(uint64_t* a, int limb) {
    const uint64_t* w = g_inv[limb];
    for (size_t m = ORC_N / 2; m >= 1; m >>= 1) {
        size_t t = ORC_N / (2 * m);
        for (size_t gi = 0; gi < m; gi++) {
            uint64_t tw = w[m + gi];
            uint64_t* x = a + gi * 2 * t;
            for (size_t p = 0; p < t; p++) {
                uint64_t u = x[p], v = x[p + t];
                x[p] = addmod(u, v, limb);
                x[p + t] = mulmod(submod(u, v, limb), tw, limb);
            }
        }
        if (m == 1) break;
    }
    for (size_t i = 0; i < ORC_N; i++) a[i] = mulmod(a[i], g_inv_n[limb], limb);
}

/* ------------------------------------------------------------ decomp */
/* Approximate gadget decomposition of one coefficient, src/ring.cpp:205-246:
 * CRT lift to [0,Q), center to (-Q/2, Q/2], three signed base-2^18 digits,
 * digit 0 dropped.  Writes digits 1..2 as (mod q0, mod q1). */
static inline void decomp_coeff(uint64_t a0, uint64_t a1, uint64_t out[ORC_DEFF][2]) {
    const u128 qf = (u128)Q[0] * Q[1];
    u128 x = (u128)(((u128)a0 * g_q1_inv_q0) % Q[0]) * Q[1] +
             (u128)(((u128)a1 * g_q0_inv_q1) % Q[1]) * Q[0];
    uint64_t val = (uint64_t)(x % qf);
    int64_t r = (val <= (uint64_t)(qf / 2)) ? (int64_t)val : (int64_t)(val - (uint64_t)qf);
    const int K = 64 - ORC_BASE_LOG;
    int64_t digs[ORC_DGSW];
    for (int j = 0; j < ORC_DGSW; j++) {
        int64_t d = (int64_t)((uint64_t)r << K) >> K;
        digs[j] = d;
        r = (r - d) >> ORC_BASE_LOG;
    }
    for (int j = 0; j < ORC_DEFF; j++) {
        int64_t d = digs[j + 1];
        out[j][0] = d >= 0 ? (uint64_t)d : (uint64_t)((int64_t)Q[0] + d);
        out[j][1] = d >= 0 ? (uint64_t)d : (uint64_t)((int64_t)Q[1] + d);
    }
}

/* f: [limb][N] coefficient form -> out: [digit][limb][N] coefficient form. */
void orc_decomp(const uint64_t* f, uint64_t* out) {
    for (size_t i = 0; i < ORC_N; i++) {
        uint64_t d[ORC_DEFF][2];
        decomp_coeff(f[i], f[ORC_N + i], d);
        for (int j = 0; j < ORC_DEFF; j++) {
            out[(j * 2 + 0) * ORC_N + i] = d[j][0];
            out[(j * 2 + 1) * ORC_N + i] = d[j][1];
        }
    }
}

/* -------------------------------------------------------- expand_seed */
/* SHAKE-256(seed || domain || le64(index)) -> 2N u64 little-endian words;
 * limb0[i] = w[i] % q0, limb1[i] = w[N+i] % q1.  src/ring.cpp:252-279.
 * OpenSSL's EVP_shake256 is the reference's own dependency. */
int orc_expand_seed(const uint8_t* seed, const char* domain, uint64_t index, uint64_t* out) {
    uint8_t in[64 + 64 + 8];
    size_t dl = strlen(domain);
    if (dl > 64) return 1;
    memcpy(in, seed, 64);
    memcpy(in + 64, domain, dl);
    for (int i = 0; i < 8; i++) in[64 + dl + i] = (uint8_t)(index >> (8 * i));
    uint8_t raw[2 * ORC_N * 8];
    EVP_MD_CTX* ctx = EVP_MD_CTX_new();
    if (!ctx) return 2;
    int ok = EVP_DigestInit_ex(ctx, EVP_shake256(), NULL) &&
             EVP_DigestUpdate(ctx, in, 64 + dl + 8) &&
             EVP_DigestFinalXOF(ctx, raw, sizeof raw);
    EVP_MD_CTX_free(ctx);
    if (!ok) return 3;
    for (size_t i = 0; i < 2 * ORC_N; i++) {
        uint64_t w = 0;
        for (int b = 0; b < 8; b++) w |= (uint64_t)raw[8 * i + b] << (8 * b);
        out[i] = (i < ORC_N) ? w % Q[0] : w % Q[1];
    }
    return 0;
}

/* ------------------------------------------------------ slot permutation */
/* NTT-slot permutation of the automorphism tau_t: slot i of the result is
 * slot perm_t(i) of the source, since slot i holds the evaluation at
 * psi^(2 BR(i) + 1).  Closed form of src/gpu_preprocess.cu:158-194; the
 * brute-force table of src/gpu_protocol.cu:169-215 is the same map (pinned
 * in tests against the reference's automorphism_ntt). */
static inline uint32_t perm_t(uint32_t t, uint32_t i) {
    uint32_t e = (t * (2 * brev11(i) + 1)) & (2 * ORC_N - 1);
    return brev11((e - 1) >> 1);
}
void orc_perm_table(uint32_t t, uint32_t* out) {
    for (uint32_t i = 0; i < ORC_N; i++) out[i] = perm_t(t, i);
}
static uint32_t pow5(uint32_t e) { /* 5^e mod 2N */
    uint32_t r = 1;
    for (uint32_t k = 0; k < e; k++) r = (r * 5) & (2 * ORC_N - 1);
    return r;
}

/* -------------------------------------------------------------- encode */
/* In-place inverse DFT over Z_P[X]/(X^N+1) of each row's ct-block of D_act
 * column-polynomials, monomial twiddles, times D_act^-1 mod P.
 * src/gpu_preprocess.cu:931-1070 (bit reversal across the D axis, log2 D
 * butterfly levels, Mersenne scaling). */
void orc_encode(uint16_t* db, size_t rows, size_t cols, size_t D) {
    size_t n_packed = cols / ORC_N;
    size_t Da = D < n_packed ? D : n_packed;
    if (Da <= 1) return;
    size_t num_cts = n_packed / Da;
    int logD = 0;
    while (((size_t)1 << logD) < Da) logD++;
    uint64_t Dinv = modinv_u64(Da, ORC_P);
    const size_t twoN = 2 * ORC_N;
#pragma omp parallel
    {
        uint32_t* ev = malloc(sizeof(uint32_t) * ORC_N);
        uint32_t* tmp = malloc(sizeof(uint32_t) * ORC_N);
#pragma omp for schedule(static)
        for (size_t row = 0; row < rows; row++) {
            uint16_t* rp = db + row * cols;
            for (size_t ct = 0; ct < num_cts; ct++) {
                uint16_t* base = rp + ct * Da * ORC_N;
                for (size_t d = 0; d < Da; d++) {
                    size_t rev = 0;
                    for (int b = 0; b < logD; b++)
                        if (d & ((size_t)1 << b)) rev |= (size_t)1 << (logD - 1 - b);
                    if (d < rev)
                        for (size_t k = 0; k < ORC_N; k++) {
                            uint16_t t = base[d * ORC_N + k];
                            base[d * ORC_N + k] = base[rev * ORC_N + k];
                            base[rev * ORC_N + k] = t;
                        }
                }
                for (int level = 0; level < logD; level++) {
                    size_t sg = (size_t)2 << level, hf = sg / 2;
                    for (size_t b0 = 0; b0 < Da; b0 += sg)
                        for (size_t i = 0; i < hf; i++) {
                            size_t ex = (twoN - ((twoN * i) / sg) % twoN) % twoN;
                            uint16_t* pe = base + (b0 + i) * ORC_N;
                            uint16_t* po = base + (b0 + i + hf) * ORC_N;
                            for (size_t k = 0; k < ORC_N; k++) {
                                size_t src = k + twoN - ex;
                                if (src >= twoN) src -= twoN;
                                uint32_t t;
                                if (src < ORC_N) t = po[src];
                                else { uint32_t v = po[src - ORC_N]; t = v ? (uint32_t)ORC_P - v : 0; }
                                uint32_t e = pe[k];
                                uint32_t s = e + t; if (s >= ORC_P) s -= ORC_P;
                                uint32_t df = e + (uint32_t)ORC_P - t; if (df >= ORC_P) df -= ORC_P;
                                ev[k] = s; tmp[k] = df;
                            }
                            for (size_t k = 0; k < ORC_N; k++) { pe[k] = (uint16_t)ev[k]; po[k] = (uint16_t)tmp[k]; }
                        }
                }
                for (size_t x = 0; x < Da * ORC_N; x++)
                    base[x] = (uint16_t)(((uint64_t)base[x] * Dinv) % ORC_P);
            }
        }
        free(ev); free(tmp);
    }
}

/* ---------------------------------------------------------- preprocess */
/* Per-group precomp layout (u32, NTT form), as the reference adopts it
 * (src/protocol.h:14-17, src/gpu_protocol.cu:333-335):
 *   a       [limb][N]
 *   D_plus  [limb][step][digit][N]   (step < 1023)
 *   D_minus same
 *   D_final [limb][digit][N]                                              */
#define PRE_A (2 * ORC_N)
#define PRE_D ((size_t)2 * ORC_NSTEPS * ORC_DEFF * ORC_N)
#define PRE_F (2 * ORC_DEFF * ORC_N)

/* CRS polys a~_r = NTT(tau_{2N-1}(expand_seed("rlwe", r))), r < rows/N.
 * src/gpu_protocol.cu:569-582.  out: [r][limb][N]. */
int orc_crs_polys(const uint8_t* seed, size_t n_r, uint64_t* out) {
    orc_init();
    for (size_t r = 0; r < n_r; r++) {
        uint64_t a[2 * ORC_N];
        int rc = orc_expand_seed(seed, "rlwe", r, a);
        if (rc) return rc;
        uint64_t* o = out + r * 2 * ORC_N;
        for (int l = 0; l < 2; l++) {
            o[l * ORC_N] = a[l * ORC_N];
            for (size_t i = 1; i < ORC_N; i++) {
                uint64_t v = a[l * ORC_N + ORC_N - i];
                o[l * ORC_N + i] = v ? Q[l] - v : 0;
            }
            orc_ntt_forward(o + l * ORC_N, l);
        }
    }
    return 0;
}

/* a-side matmul for one group, src/gpu_preprocess.cu:347-410:
 *   acc_j = sum_r NTT(db[r*N + i][g*N + j], i<N) (.) a~_r ;
 *   a32[j][limb][k] = N^-1 * acc_j[limb][N-1-k].
 * out: [j][limb][N]. */
void orc_a_side(const uint16_t* db, size_t rows, size_t cols, size_t g,
                const uint64_t* crs, uint64_t* a32) {
    size_t n_r = rows / ORC_N;
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < ORC_N; j++) {
        uint64_t acc[2][ORC_N], col[ORC_N];
        memset(acc, 0, sizeof acc);
        for (size_t r = 0; r < n_r; r++)
            for (int l = 0; l < 2; l++) {
                for (size_t i = 0; i < ORC_N; i++) col[i] = db[(r * ORC_N + i) * cols + g * ORC_N + j];
                orc_ntt_forward(col, l);
                const uint64_t* ar = crs + (r * 2 + l) * ORC_N;
                for (size_t i = 0; i < ORC_N; i++)
                    acc[l][i] = addmod(acc[l][i], mulmod(col[i], ar[i], l), l);
            }
        for (int l = 0; l < 2; l++)
            for (size_t k = 0; k < ORC_N; k++)
                a32[(j * 2 + l) * ORC_N + k] = mulmod(acc[l][ORC_N - 1 - k], g_inv_n[l], l);
    }
}

/* Literal ring_embed + automorphism perms for the listed k values only,
 * src/gpu_preprocess.cu:39-92 (n^3 MAC form over the monomial table
 * mono[e] = NTT(X^e)) and :158-194.  out: [nk][dir][limb][N]. */
void orc_ring_embed_literal(const uint64_t* a32, const uint32_t* ks, size_t nk, uint64_t* out) {
    /* monomial table, src/gpu_protocol.cu:248-262 */
    uint64_t* mono = malloc(sizeof(uint64_t) * 2 * ORC_N * 2 * ORC_N);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < 2 * ORC_N; e++)
        for (int l = 0; l < 2; l++) {
            uint64_t* p = mono + (e * 2 + l) * ORC_N;
            memset(p, 0, sizeof(uint64_t) * ORC_N);
            if (e < ORC_N) p[e] = 1; else p[e - ORC_N] = Q[l] - 1;
            orc_ntt_forward(p, l);
        }
#pragma omp parallel for schedule(static) collapse(2)
    for (size_t kk = 0; kk < nk; kk++)
        for (int l = 0; l < 2; l++) {
            uint32_t k = ks[kk];
            uint32_t gpow = pow5((ORC_N - k) % ORC_N);
            uint64_t accf[ORC_N], accc[ORC_N];
            for (size_t i = 0; i < ORC_N; i++) {
                u128 sf = 0, sc = 0;
                uint32_t idx = 0;
                for (size_t j = 0; j < ORC_N; j++) {
                    uint64_t aj = a32[(j * 2 + l) * ORC_N + i];
                    uint32_t idc = (2 * ORC_N - idx) & (2 * ORC_N - 1);
                    sf += (u128)aj * mono[((size_t)idx * 2 + l) * ORC_N + i];
                    sc += (u128)aj * mono[((size_t)idc * 2 + l) * ORC_N + i];
                    idx = (idx + gpow) & (2 * ORC_N - 1);
                }
                accf[i] = (uint64_t)(sf % Q[l]);
                accc[i] = (uint64_t)(sc % Q[l]);
            }
            uint32_t tf = pow5(k), tc = (2 * ORC_N - tf) & (2 * ORC_N - 1);
            for (uint32_t i = 0; i < ORC_N; i++) {
                out[((kk * 2 + 0) * 2 + l) * ORC_N + i] = accf[perm_t(tf, i)];
                out[((kk * 2 + 1) * 2 + l) * ORC_N + i] = accc[perm_t(tc, i)];
            }
        }
    free(mono);
}

/* Same result as the literal ring_embed + perms, in O(N^2 log N):
 * acc_fwd[k][p] = A_p(zeta_p^(5^(N-k))) with A_p(z) = sum_j a32[j][p] z^j,
 * and after the slot permutation a_post_fwd[k][i] = A_{perm_{5^k}(i)}(zeta_i)
 * because 5^N = 1 mod 2N; likewise a_post_conj[k][i] = A_{perm_{-5^k}(i)}(zeta_i).
 * A_p evaluated at every zeta_m is one forward NTT of the column (a32[j][p])_j.
 * out: a_post [k][dir][limb][N] for all k < N/2. */
void orc_ring_embed_fast(const uint64_t* a32, uint64_t* a_post) {
    uint64_t* T = malloc(sizeof(uint64_t) * 2 * ORC_N * ORC_N); /* [limb][p][m] */
#pragma omp parallel for schedule(static) collapse(2)
    for (int l = 0; l < 2; l++)
        for (size_t p = 0; p < ORC_N; p++) {
            uint64_t* v = T + ((size_t)l * ORC_N + p) * ORC_N;
            for (size_t j = 0; j < ORC_N; j++) v[j] = a32[(j * 2 + l) * ORC_N + p];
            orc_ntt_forward(v, l);
        }
#pragma omp parallel for schedule(static)
    for (uint32_t k = 0; k < ORC_HALF; k++) {
        uint32_t tf = pow5(k), tc = (2 * ORC_N - tf) & (2 * ORC_N - 1);
        for (int l = 0; l < 2; l++)
            for (uint32_t i = 0; i < ORC_N; i++) {
                a_post[(((size_t)k * 2 + 0) * 2 + l) * ORC_N + i] = T[((size_t)l * ORC_N + perm_t(tf, i)) * ORC_N + i];
                a_post[(((size_t)k * 2 + 1) * 2 + l) * ORC_N + i] = T[((size_t)l * ORC_N + perm_t(tc, i)) * ORC_N + i];
            }
    }
    free(T);
}

/* ExpandKSK_a, src/gpu_protocol.cu:364-474 + src/gpu_preprocess.cu:228-270:
 *   K5[j]   = NTT(expand_seed("ksk", 5*100 + j+1))
 *   Kn1[j]  = NTT(expand_seed("ksk", (2N-1)*100 + j+1))
 *   Kplus[limb][s][j][i]  = K5[j][limb][perm_{5^s}(i)]
 *   Kminus[limb][s][j][i] = K5[j][limb][perm_{2N-5^s}(i)]
 * kplus/kminus: [limb][s][j][N]; kn1: [limb][j][N]. */
int orc_expand_ksk(const uint8_t* seed, uint64_t* kplus, uint64_t* kminus, uint64_t* kn1) {
    orc_init();
    uint64_t k5[ORC_DEFF][2 * ORC_N];
    for (int j = 0; j < ORC_DEFF; j++) {
        uint64_t t[2 * ORC_N];
        int rc = orc_expand_seed(seed, "ksk", 5 * 100 + j + 1, k5[j]);
        if (rc) return rc;
        rc = orc_expand_seed(seed, "ksk", (uint64_t)(2 * ORC_N - 1) * 100 + j + 1, t);
        if (rc) return rc;
        for (int l = 0; l < 2; l++) {
            orc_ntt_forward(k5[j] + l * ORC_N, l);
            orc_ntt_forward(t + l * ORC_N, l);
            memcpy(kn1 + ((size_t)l * ORC_DEFF + j) * ORC_N, t + l * ORC_N, sizeof(uint64_t) * ORC_N);
        }
    }
    for (uint32_t s = 0; s < ORC_NSTEPS; s++) {
        uint32_t tf = pow5(s), tc = (2 * ORC_N - tf) & (2 * ORC_N - 1);
        for (int l = 0; l < 2; l++)
            for (int j = 0; j < ORC_DEFF; j++)
                for (uint32_t i = 0; i < ORC_N; i++) {
                    size_t o = (((size_t)l * ORC_NSTEPS + s) * ORC_DEFF + j) * ORC_N + i;
                    kplus[o] = k5[j][l * ORC_N + perm_t(tf, i)];
                    kminus[o] = k5[j][l * ORC_N + perm_t(tc, i)];
                }
    }
    return 0;
}

/* Decompose state (NTT form, both limbs) into NTT-form digits and
 * accumulate sum_j dig_j (.) K_j; the collapse inner step of
 * src/gpu_preprocess.cu:511-600. dig out: [limb][digit][N]. */
static void collapse_digits(const uint64_t* state, uint64_t* dig) {
    uint64_t c[2][ORC_N];
    memcpy(c[0], state, sizeof c[0]);
    memcpy(c[1], state + ORC_N, sizeof c[1]);
    orc_ntt_inverse(c[0], 0);
    orc_ntt_inverse(c[1], 1);
    for (size_t i = 0; i < ORC_N; i++) {
        uint64_t d[ORC_DEFF][2];
        decomp_coeff(c[0][i], c[1][i], d);
        for (int j = 0; j < ORC_DEFF; j++)
            for (int l = 0; l < 2; l++) dig[((size_t)l * ORC_DEFF + j) * ORC_N + i] = d[j][l];
    }
    for (int l = 0; l < 2; l++)
        for (int j = 0; j < ORC_DEFF; j++) orc_ntt_forward(dig + ((size_t)l * ORC_DEFF + j) * ORC_N, l);
}

/* CollapseA for one group, src/gpu_preprocess.cu:452-881.
 * a_post: [k][dir][limb][N] (k < N/2).  Outputs in the precomp layout. */
void orc_collapse_group(const uint64_t* a_post, const uint64_t* kplus, const uint64_t* kminus,
                        const uint64_t* kn1, uint32_t* out_a, uint32_t* out_dp,
                        uint32_t* out_dm, uint32_t* out_df) {
    uint64_t state[2 * ORC_N], saved[2 * ORC_N], dig[2 * ORC_DEFF * ORC_N];
    for (int dir = 0; dir < 2; dir++) {
        const uint64_t* K = dir ? kminus : kplus;
        uint32_t* Dout = dir ? out_dm : out_dp;
        for (int l = 0; l < 2; l++)
            memcpy(state + l * ORC_N, a_post + (((size_t)(ORC_HALF - 1) * 2 + dir) * 2 + l) * ORC_N,
                   sizeof(uint64_t) * ORC_N);
        for (size_t s = 0; s < ORC_NSTEPS; s++) {
            size_t k = ORC_HALF - 1 - s, ks = ORC_NSTEPS - 1 - s;
            collapse_digits(state, dig);
            for (int l = 0; l < 2; l++) {
                for (int j = 0; j < ORC_DEFF; j++)
                    for (size_t i = 0; i < ORC_N; i++)
                        Dout[(((size_t)l * ORC_NSTEPS + s) * ORC_DEFF + j) * ORC_N + i] =
                            (uint32_t)dig[((size_t)l * ORC_DEFF + j) * ORC_N + i];
                const uint64_t* an = a_post + (((size_t)(k - 1) * 2 + dir) * 2 + l) * ORC_N;
                for (size_t i = 0; i < ORC_N; i++) {
                    uint64_t acc = 0;
                    for (int j = 0; j < ORC_DEFF; j++)
                        acc += dig[((size_t)l * ORC_DEFF + j) * ORC_N + i] *
                               K[(((size_t)l * ORC_NSTEPS + ks) * ORC_DEFF + j) * ORC_N + i];
                    state[l * ORC_N + i] = submod(an[i], acc % Q[l], l);
                }
            }
        }
        if (dir == 0) memcpy(saved, state, sizeof saved);
    }
    collapse_digits(state, dig);
    for (int l = 0; l < 2; l++) {
        for (int j = 0; j < ORC_DEFF; j++)
            for (size_t i = 0; i < ORC_N; i++)
                out_df[((size_t)l * ORC_DEFF + j) * ORC_N + i] = (uint32_t)dig[((size_t)l * ORC_DEFF + j) * ORC_N + i];
        for (size_t i = 0; i < ORC_N; i++) {
            uint64_t acc = 0;
            for (int j = 0; j < ORC_DEFF; j++)
                acc += dig[((size_t)l * ORC_DEFF + j) * ORC_N + i] * kn1[((size_t)l * ORC_DEFF + j) * ORC_N + i];
            out_a[l * ORC_N + i] = (uint32_t)submod(saved[l * ORC_N + i], acc % Q[l], l);
        }
    }
}

/* Full preprocess (src/gpu_protocol.cu:535-817).  db is encoded in place.
 * Precomp outputs sized n_packed * PRE_{A,D,D,F} u32.
 * group_lo/group_hi restrict the per-group work (for sampled checks). */
int orc_preprocess(const uint8_t* seed, uint16_t* db, size_t rows, size_t cols, size_t D,
                   size_t group_lo, size_t group_hi, int do_encode,
                   uint32_t* pre_a, uint32_t* pre_dp, uint32_t* pre_dm, uint32_t* pre_df) {
    orc_init();
    if (rows % ORC_N || cols % ORC_N) return 10;
    size_t n_r = rows / ORC_N;
    if (do_encode) orc_encode(db, rows, cols, D);
    uint64_t* crs = malloc(sizeof(uint64_t) * n_r * 2 * ORC_N);
    uint64_t* kp = malloc(sizeof(uint64_t) * PRE_D);
    uint64_t* km = malloc(sizeof(uint64_t) * PRE_D);
    uint64_t kn1[PRE_F];
    uint64_t* a32 = malloc(sizeof(uint64_t) * ORC_N * 2 * ORC_N);
    uint64_t* apost = malloc(sizeof(uint64_t) * ORC_HALF * 2 * 2 * ORC_N);
    int rc = orc_crs_polys(seed, n_r, crs);
    if (!rc) rc = orc_expand_ksk(seed, kp, km, kn1);
    for (size_t g = group_lo; !rc && g < group_hi; g++) {
        size_t o = g - group_lo;
        orc_a_side(db, rows, cols, g, crs, a32);
        orc_ring_embed_fast(a32, apost);
        orc_collapse_group(apost, kp, km, kn1, pre_a + o * PRE_A, pre_dp + o * PRE_D,
                           pre_dm + o * PRE_D, pre_df + o * PRE_F);
    }
    free(crs); free(kp); free(km); free(a32); free(apost);
    return rc;
}

/* ------------------------------------------------------------- answer */
/* Dual-limb mat-vec r_l[j] = sum_i db[i][j] * b_l[i] mod q_l over columns
 * [col_lo, col_hi); src/gpu_online.cu:23-41.  b: [limb][rows] (< q).
 * out: [limb][cols] (only the range is written). */
void orc_matvec(const uint16_t* db, size_t rows, size_t cols, const uint64_t* b,
                size_t col_lo, size_t col_hi, uint64_t* out) {
#pragma omp parallel for schedule(static)
    for (size_t c0 = col_lo; c0 < col_hi; c0 += 64) {
        size_t c1 = c0 + 64 < col_hi ? c0 + 64 : col_hi;
        u128 acc[2][64];
        memset(acc, 0, sizeof acc);
        for (size_t i = 0; i < rows; i++) {
            const uint16_t* rp = db + i * cols;
            uint64_t b0 = b[i], b1 = b[rows + i];
            for (size_t c = c0; c < c1; c++) {
                acc[0][c - c0] += (u128)rp[c] * b0;
                acc[1][c - c0] += (u128)rp[c] * b1;
            }
        }
        for (size_t c = c0; c < c1; c++) {
            out[c] = (uint64_t)(acc[0][c - c0] % Q[0]);
            out[cols + c] = (uint64_t)(acc[1][c - c0] % Q[1]);
        }
    }
}

/* Per-group online pack, src/gpu_protocol.cu:1225-1283:
 * b = NTT(r[g*N..]); b -= sum_s sum_j Dplus[s][j] (.) K5[j][perm_{5^(N/2-2-s)}];
 * b -= ... Dminus with perm_{2N-5^(N/2-2-s)}; b -= sum_j Dfinal[j] (.) Kn1[j].
 * r: [limb][cols]; k5/kn1: [limb][digit][N] NTT form; out_b [limb][N]. */
void orc_pack_group(const uint64_t* r, size_t cols, size_t g, const uint32_t* dp,
                    const uint32_t* dm, const uint32_t* df, const uint64_t* k5,
                    const uint64_t* kn1, uint64_t* out_b) {
    for (int l = 0; l < 2; l++) {
        uint64_t* b = out_b + l * ORC_N;
        memcpy(b, r + l * cols + g * ORC_N, sizeof(uint64_t) * ORC_N);
        orc_ntt_forward(b, l);
        for (int dir = 0; dir < 2; dir++) {
            const uint32_t* Dt = dir ? dm : dp;
            for (size_t s = 0; s < ORC_NSTEPS; s++) {
                uint32_t t = pow5(ORC_HALF - 2 - s);
                if (dir) t = (2 * ORC_N - t) & (2 * ORC_N - 1);
                for (uint32_t i = 0; i < ORC_N; i++) {
                    uint32_t pi = perm_t(t, i);
                    uint64_t acc = 0;
                    for (int j = 0; j < ORC_DEFF; j++)
                        acc += (uint64_t)Dt[(((size_t)l * ORC_NSTEPS + s) * ORC_DEFF + j) * ORC_N + i] *
                               k5[((size_t)l * ORC_DEFF + j) * ORC_N + pi];
                    b[i] = submod(b[i], acc % Q[l], l);
                }
            }
        }
        for (uint32_t i = 0; i < ORC_N; i++) {
            uint64_t acc = 0;
            for (int j = 0; j < ORC_DEFF; j++)
                acc += (uint64_t)df[((size_t)l * ORC_DEFF + j) * ORC_N + i] * kn1[((size_t)l * ORC_DEFF + j) * ORC_N + i];
            b[i] = submod(b[i], acc % Q[l], l);
        }
    }
}

/* ExtProd, src/crypto.cpp:219-257: ct (a,b) NTT form [a|b][limb][N];
 * rgsw [top_a|top_b|bot_a|bot_b][digit][limb][N] NTT form; out NTT form. */
void orc_ext_prod(const uint64_t* rgsw, const uint64_t* ct, uint64_t* out) {
    uint64_t coef[2][2 * ORC_N], dg[2][ORC_DEFF][2][ORC_N];
    for (int p = 0; p < 2; p++) {
        memcpy(coef[p], ct + p * 2 * ORC_N, sizeof coef[p]);
        orc_ntt_inverse(coef[p], 0);
        orc_ntt_inverse(coef[p] + ORC_N, 1);
        for (size_t i = 0; i < ORC_N; i++) {
            uint64_t d[ORC_DEFF][2];
            decomp_coeff(coef[p][i], coef[p][ORC_N + i], d);
            for (int j = 0; j < ORC_DEFF; j++) { dg[p][j][0][i] = d[j][0]; dg[p][j][1][i] = d[j][1]; }
        }
        for (int j = 0; j < ORC_DEFF; j++) { orc_ntt_forward(dg[p][j][0], 0); orc_ntt_forward(dg[p][j][1], 1); }
    }
    const size_t blk = (size_t)ORC_DEFF * 2 * ORC_N;
    for (int outp = 0; outp < 2; outp++)       /* 0: a, 1: b */
        for (int l = 0; l < 2; l++)
            for (size_t i = 0; i < ORC_N; i++) {
                uint64_t s = 0;
                for (int j = 0; j < ORC_DEFF; j++) {
                    /* digits of a x top row, digits of b x bottom row */
                    uint64_t top = rgsw[(0 + outp) * blk + ((size_t)j * 2 + l) * ORC_N + i];
                    uint64_t bot = rgsw[(2 + outp) * blk + ((size_t)j * 2 + l) * ORC_N + i];
                    s = addmod(s, mulmod(dg[0][j][l][i], top, l), l);
                    s = addmod(s, mulmod(dg[1][j][l][i], bot, l), l);
                }
                out[((size_t)outp * 2 + l) * ORC_N + i] = s;
            }
}

/* Full answer for one query, src/gpu_protocol.cu:1121-1339.
 * query flat (capi.h:101-112): [b0: rows][b1: rows][ksk5: blk][kskneg1: blk][rgsw: 4 blk],
 *   blk = D_EFF*2*N, ksk in coefficient form, rgsw in NTT form.
 * resp: [ct][a|b][limb][N] u64, NTT form. */
int orc_answer(const uint16_t* db_enc, size_t rows, size_t cols, size_t D,
               const uint32_t* pre_a, const uint32_t* pre_dp, const uint32_t* pre_dm,
               const uint32_t* pre_df, const uint64_t* qflat, uint64_t* resp) {
    orc_init();
    size_t G = cols / ORC_N, Da = D < G ? D : G, ncts = G / D > 1 ? G / D : 1;
    const size_t blk = (size_t)ORC_DEFF * 2 * ORC_N;
    uint64_t* b = malloc(sizeof(uint64_t) * 2 * rows);
    for (size_t i = 0; i < rows; i++) {
        b[i] = qflat[i] % Q[0];
        b[rows + i] = qflat[rows + i] % Q[1];
    }
    uint64_t* r = malloc(sizeof(uint64_t) * 2 * cols);
    orc_matvec(db_enc, rows, cols, b, 0, cols, r);
    /* keys: [digit][limb][N] coefficient form -> [limb][digit][N] NTT form */
    uint64_t k5[2 * ORC_DEFF * ORC_N], kn1[2 * ORC_DEFF * ORC_N];
    const uint64_t* kq5 = qflat + 2 * rows;
    const uint64_t* kqn = kq5 + blk;
    for (int j = 0; j < ORC_DEFF; j++)
        for (int l = 0; l < 2; l++) {
            uint64_t* d5 = k5 + ((size_t)l * ORC_DEFF + j) * ORC_N;
            uint64_t* dn = kn1 + ((size_t)l * ORC_DEFF + j) * ORC_N;
            for (size_t i = 0; i < ORC_N; i++) {
                d5[i] = kq5[((size_t)j * 2 + l) * ORC_N + i] % Q[l];
                dn[i] = kqn[((size_t)j * 2 + l) * ORC_N + i] % Q[l];
            }
            orc_ntt_forward(d5, l);
            orc_ntt_forward(dn, l);
        }
    uint64_t* rgsw = malloc(sizeof(uint64_t) * 4 * blk);
    for (size_t x = 0; x < 4 * blk; x++) rgsw[x] = qflat[2 * rows + 2 * blk + x] % Q[(x / ORC_N) & 1];
    uint64_t* packed = malloc(sizeof(uint64_t) * G * 4 * ORC_N); /* [g][a|b][limb][N] */
#pragma omp parallel for schedule(dynamic)
    for (size_t g = 0; g < G; g++) {
        uint64_t* pg = packed + g * 4 * ORC_N;
        for (size_t x = 0; x < PRE_A; x++) pg[x] = pre_a[g * PRE_A + x];
        orc_pack_group(r, cols, g, pre_dp + g * PRE_D, pre_dm + g * PRE_D, pre_df + g * PRE_F,
                       k5, kn1, pg + 2 * ORC_N);
    }
    for (size_t c = 0; c < ncts; c++) {
        size_t start = c * Da, L = (start + Da <= G ? Da : G - start);
        uint64_t acc[4 * ORC_N], nxt[4 * ORC_N];
        memcpy(acc, packed + (start + L - 1) * 4 * ORC_N, sizeof acc);
        for (long i = (long)L - 2; i >= 0; i--) {
            orc_ext_prod(rgsw, acc, nxt);
            const uint64_t* pk = packed + (start + (size_t)i) * 4 * ORC_N;
            for (size_t x = 0; x < 4 * ORC_N; x++) acc[x] = addmod(nxt[x], pk[x], (int)((x / ORC_N) & 1));
        }
        memcpy(resp + c * 4 * ORC_N, acc, sizeof acc);
    }
    free(b); free(r); free(rgsw); free(packed);
    return 0;
}

/* Horner over caller-given packed cts [L][a|b][limb][N], src/crypto.cpp:264-279. */
void orc_horner(const uint64_t* rgsw, const uint64_t* packed, size_t L, uint64_t* out) {
    uint64_t acc[4 * ORC_N], nxt[4 * ORC_N];
    memcpy(acc, packed + (L - 1) * 4 * ORC_N, sizeof acc);
    for (long i = (long)L - 2; i >= 0; i--) {
        orc_ext_prod(rgsw, acc, nxt);
        for (size_t x = 0; x < 4 * ORC_N; x++) acc[x] = addmod(nxt[x], packed[(size_t)i * 4 * ORC_N + x], (int)((x / ORC_N) & 1));
    }
    memcpy(out, acc, sizeof acc);
}

/* Deterministic DB: splitmix64(seed ^ k) mod 65535 at flat index k. */
static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
void orc_fill_db(uint16_t* db, size_t count, uint64_t seed) {
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < count; k++) db[k] = (uint16_t)(splitmix64(seed ^ k) % ORC_P);
}

/* Synthetic residues: p[k] = splitmix64(seed ^ k) mod q (q < 2^32), for
 * precomputed tensors whose values the timed CPU path does not depend on. */
void orc_fill_u32_mod(uint32_t* p, size_t count, uint64_t seed, uint32_t q) {
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < count; k++) p[k] = (uint32_t)(splitmix64(seed ^ k) % q);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
