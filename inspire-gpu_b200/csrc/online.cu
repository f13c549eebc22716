// online.cu -- per-query kernels of the B200 InsPIRe server.
//
// One answer (gpu_answer / gpu_answer_batch, reference src/gpu_protocol.cu:
// 1121-1535) runs these launches on one stream:
//   qprep     key-switching keys to NTT form, RGSW to u32 residues
//   matvec    r_l[j] = sum_i db[i][j] * b_l[i] mod q_l   (DB pass, HBM bound)
//   tensor pass (tensorpass_tc.cu): sum_{dir,s,j} D[s][j][i] * K5[j][perm_s(i)]
//   finalize  per group: NTT(r slice) - tensor partials - D_final (.) Kneg1
//   horner    one persistent CTA per response ciphertext runs the whole
//             ExtProd chain (INTT, decomp, NTT, MAC) in shared memory
// All arithmetic is exact mod q_l, so every output equals the reference's.
#include <algorithm>

#include "ipb_common.cuh"
#include "host_util.h"
#include "ipb_launch.h"

namespace ipb {

namespace {

__device__ __forceinline__ uint32_t pow5_mod2n(uint32_t e) {
    uint32_t r = 1, b = 5;
    while (e) {
        if (e & 1) r = (r * b) & (2 * kN - 1);
        b = (b * b) & (2 * kN - 1);
        e >>= 1;
    }
    return r;
}
constexpr uint32_t kInv5 = 3277;  // 5^-1 mod 2N (5 * 3277 = 4*4096 + 1)

__device__ __forceinline__ void ld8(const uint32_t* p, uint32_t (&v)[8]) {
    uint4 a = *reinterpret_cast<const uint4*>(p);
    uint4 b = *reinterpret_cast<const uint4*>(p + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void st8(uint32_t* p, const uint32_t (&v)[8]) {
    *reinterpret_cast<uint4*>(p) = make_uint4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<uint4*>(p + 4) = make_uint4(v[4], v[5], v[6], v[7]);
}

// ------------------------------------------------------------------ qprep
// grid (nq, 12): y < 8 -> one key poly NTT (key, digit, limb); y >= 8 -> a
// quarter of the RGSW u64 -> u32 reduction.  The client sends KSK b-parts in
// coefficient form and RGSW in NTT form (capi.h:47-54); the reference NTTs the
// keys on the server (src/gpu_protocol.cu:1059-1094).  Inputs are reduced
// mod q (identical to the reference on canonical inputs).
__global__ void __launch_bounds__(256) qprep_kernel(const uint64_t* __restrict__ qraw, size_t qstride,
                                                    size_t rows, const DevTables* __restrict__ T,
                                                    uint32_t* __restrict__ keys,
                                                    uint32_t* __restrict__ rgsw32, int y0) {
    __shared__ __align__(16) uint32_t sbuf[2 * kN];
    const int b = blockIdx.x, y = y0 + (int)blockIdx.y;
    const uint32_t t = threadIdx.x;
    const uint64_t* qr = qraw + (size_t)b * qstride;
    const size_t blk = (size_t)kDeff * 2 * kN;
    if (y < 8) {
        const int key = y >> 2, j = (y >> 1) & 1, l = y & 1;
        const LimbTables& L = T->limb[l];
        const uint64_t* src = qr + 2 * rows + key * blk + (size_t)(j * 2 + l) * kN;
        uint32_t r[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) r[e] = mod_u64(src[t + 256 * e], L.cr, L.q);
        ntt_fwd(r, sbuf, L.fwd, L.q, t, 0);
        uint32_t* dst = keys + (size_t)b * (4 * kDeff * kN) + (size_t)((key * 2 + l) * kDeff + j) * kN;
        st8(dst + 8 * t, r);
    } else {
        const uint64_t* src = qr + 2 * rows + 2 * blk;
        uint32_t* dst = rgsw32 + (size_t)b * 4 * blk;
        const size_t q4 = blk;  // 4*blk elements split over 4 CTAs
        for (size_t i = (size_t)(y - 8) * q4 + t; i < (size_t)(y - 7) * q4; i += 256) {
            const int l = (int)((i / kN) & 1);
            dst[i] = mod_u64(src[i], T->limb[l].cr, T->limb[l].q);
        }
    }
}

// ------------------------------------------------------------------ matvec
// Row-split dual-limb mat-vec.  CTA (x, y): columns [x*256*CPT, +256*CPT),
// rows [y*rpc, +rpc).  Each thread streams CPT u16 columns with one 16- or
// 8-byte load per row and keeps 2*BT*CPT u64 accumulators; the query words
// of the chunk are reduced mod q once into shared memory.  Products are
// < 2^43, so rpc <= 2^20 rows need no intermediate reduction.
template <int BT, int CPT>
__global__ void __launch_bounds__(256) matvec_kernel(const uint16_t* __restrict__ db, size_t rows, size_t cols,
                                                     int rpc, const uint64_t* __restrict__ qraw, size_t qstride,
                                                     const DevTables* __restrict__ T, uint32_t* __restrict__ part,
                                                     size_t part_qstride, int nq) {
    extern __shared__ __align__(16) uint32_t sb[];  // [BT][2][rpc]
    const int chunk = blockIdx.y;
    const size_t r0 = (size_t)chunk * rpc;
    for (int b = 0; b < BT; ++b) {
        const int src = b < nq ? b : 0;
        for (int l = 0; l < 2; ++l) {
            const uint64_t* qb = qraw + (size_t)src * qstride + (size_t)l * rows + r0;
            for (int i = threadIdx.x; i < rpc; i += 256)
                sb[(b * 2 + l) * rpc + i] = mod_u64(qb[i], T->limb[l].cr, T->limb[l].q);
        }
    }
    __syncthreads();
    const size_t col0 = ((size_t)blockIdx.x * 256 + threadIdx.x) * CPT;
    uint64_t acc[BT][2][CPT];
#pragma unroll
    for (int b = 0; b < BT; ++b)
#pragma unroll
        for (int c = 0; c < CPT; ++c) { acc[b][0][c] = 0; acc[b][1][c] = 0; }
    const uint16_t* p = db + r0 * cols + col0;
#pragma unroll 4
    for (int i = 0; i < rpc; ++i) {
        uint32_t w[CPT / 2];
        if (CPT == 8) {
            uint4 v = __ldcs(reinterpret_cast<const uint4*>(p + (size_t)i * cols));
            w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
        } else {
            uint2 v = __ldcs(reinterpret_cast<const uint2*>(p + (size_t)i * cols));
            w[0] = v.x; w[1] = v.y;
        }
#pragma unroll
        for (int b = 0; b < BT; ++b) {
            const uint32_t b0 = sb[(b * 2 + 0) * rpc + i];
            const uint32_t b1 = sb[(b * 2 + 1) * rpc + i];
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const uint32_t d = (c & 1) ? (w[c >> 1] >> 16) : (w[c >> 1] & 0xFFFFu);
                acc[b][0][c] += (uint64_t)d * b0;
                acc[b][1][c] += (uint64_t)d * b1;
            }
        }
    }
#pragma unroll
    for (int b = 0; b < BT; ++b) {
        if (b >= nq) break;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            uint32_t o[CPT];
#pragma unroll
            for (int c = 0; c < CPT; ++c) o[c] = mod_u64(acc[b][l][c], T->limb[l].cr, T->limb[l].q);
            uint32_t* dst = part + (size_t)b * part_qstride + ((size_t)chunk * 2 + l) * cols + col0;
            if (CPT == 8) {
                *reinterpret_cast<uint4*>(dst) = make_uint4(o[0], o[1], o[2], o[3]);
                *reinterpret_cast<uint4*>(dst + 4) = make_uint4(o[4 % CPT], o[5 % CPT], o[6 % CPT], o[7 % CPT]);
            } else {
                *reinterpret_cast<uint4*>(dst) = make_uint4(o[0], o[1], o[2], o[3]);
            }
        }
    }
}

// ------------------------------------------------------------------ finalize
// Per (group, limb, query): b = NTT(sum of the mat-vec partials of the
// group's N columns) - tensor pass - sum_j D_final[j] (.) Kneg1[j]
// (reference src/gpu_protocol.cu:1233-1274, src/gpu_online.cu:547-559).
// The tensor pass result is tp_out[l][i][q][g] (tensorpass_tc.cu).
__global__ void __launch_bounds__(256) finalize_kernel(
    const uint32_t* __restrict__ mvpart, size_t mv_qstride, int mv_chunks, size_t cols,
    const uint32_t* __restrict__ tp_out, int nq_total, int q_off, int groups, int g0,
    const uint32_t* __restrict__ df, const uint32_t* __restrict__ keys, size_t key_qstride,
    const DevTables* __restrict__ T, uint32_t* __restrict__ packed_b, size_t pb_qstride) {
    __shared__ __align__(16) uint32_t sbuf[2 * kN];
    const int g = g0 + (int)blockIdx.x, l = blockIdx.y, b = blockIdx.z;
    const uint32_t t = threadIdx.x;
    const LimbTables& L = T->limb[l];
    uint32_t r[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const size_t x = (size_t)g * kN + t + 256 * e;
        uint64_t s = 0;
        const uint32_t* mp = mvpart + (size_t)b * mv_qstride + (size_t)l * cols + x;
        for (int y = 0; y < mv_chunks; ++y) s += mp[(size_t)y * 2 * cols];
        r[e] = mod_u64(s, L.cr, L.q);
    }
    ntt_fwd(r, sbuf, L.fwd, L.q, t, 0);
    uint32_t cs[8];
#pragma unroll
    for (int e = 0; e < 8; ++e)
        cs[e] = tp_out[(((size_t)l * kN + 8 * t + e) * nq_total + q_off + b) * groups + g];
    uint32_t d0[8], d1[8], k0[8], k1[8];
    ld8(df + ((size_t)g * 2 + l) * kDeff * kN + 8 * t, d0);
    ld8(df + (((size_t)g * 2 + l) * kDeff + 1) * kN + 8 * t, d1);
    const uint32_t* kn = keys + (size_t)b * key_qstride + (size_t)((1 * 2 + l) * kDeff) * kN;  // key 1 = kskneg1
    ld8(kn + 8 * t, k0);
    ld8(kn + kN + 8 * t, k1);
    uint32_t o[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const uint32_t fin = mod_u64((uint64_t)d0[e] * k0[e] + (uint64_t)d1[e] * k1[e], L.cr, L.q);
        const uint32_t sub = add_mod(cs[e], fin, L.q);
        o[e] = sub_mod(r[e], sub, L.q);
    }
    st8(packed_b + (size_t)b * pb_qstride + ((size_t)g * 2 + l) * kN + 8 * t, o);
}

// ------------------------------------------------------------------ horner
// HornerEval (reference src/crypto.cpp:264-279, src/gpu_protocol.cu:1300-1334):
// acc = packed[start+L-1]; for i = L-2..0: acc = ExtProd(rgsw, acc) + packed[start+i].
// One CTA of four 256-thread NTT groups runs a whole chain; group (p, l)
// owns polynomial p (0 = a, 1 = b) in limb l.  Per step: inverse NTT, CRT
// exchange with the partner limb through shared memory, gadget digits,
// two forward NTTs, the RGSW multiply-accumulate (digits of a meet the top
// row, digits of b the bottom row) and a cross-group sum.  The chain never
// leaves the SM; the reference spends ~12 launches per step.
constexpr size_t kHornerSmem = 4 * kN * sizeof(uint2) + (4 * 2 * kN + 2 * 2 * kN + 2 * 2 * kN) * sizeof(uint32_t);

__global__ void __launch_bounds__(1024, 1) horner_kernel(const uint32_t* __restrict__ pre_a,
                                                         const uint32_t* __restrict__ packed_b, size_t pb_qstride,
                                                         const uint32_t* __restrict__ rgsw32,
                                                         const DevTables* __restrict__ T, size_t groups,
                                                         size_t d_act, uint64_t* __restrict__ resp,
                                                         size_t resp_qstride) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint2* tw = reinterpret_cast<uint2*>(smem);                       // [fwd0|fwd1|inv0|inv1][N]
    uint32_t* nbuf = reinterpret_cast<uint32_t*>(smem + 4 * kN * sizeof(uint2));  // [4][2][N]
    uint32_t* xcoef = nbuf + 4 * 2 * kN;                              // [p][l][N]
    uint32_t* xch = xcoef + 2 * 2 * kN;                               // [p][l][N]
    const int ct = blockIdx.x, b = blockIdx.y;
    const int gp = threadIdx.x >> 8, p = gp >> 1, l = gp & 1;
    const uint32_t t = threadIdx.x & 255;
    const int bar = 1 + gp;
    for (int i = threadIdx.x; i < kN; i += 1024) {
        tw[i] = T->limb[0].fwd[i];
        tw[kN + i] = T->limb[1].fwd[i];
        tw[2 * kN + i] = T->limb[0].inv[i];
        tw[3 * kN + i] = T->limb[1].inv[i];
    }
    __syncthreads();
    const LimbTables& L = T->limb[l];
    const uint32_t q = L.q;
    const uint2* twf = tw + l * kN;
    const uint2* twi = tw + (2 + l) * kN;
    uint32_t* mybuf = nbuf + gp * 2 * kN;
    const size_t start = (size_t)ct * d_act;
    const size_t len = (start + d_act <= groups) ? d_act : groups - start;
    const uint32_t* pbq = packed_b + (size_t)b * pb_qstride;
    auto src_of = [&](size_t i) -> const uint32_t* {
        return p ? pbq + (i * 2 + l) * kN : pre_a + (i * 2 + l) * kN;
    };
    uint32_t acc[8];
    ld8(src_of(start + len - 1) + 8 * t, acc);
    const uint32_t* rg = rgsw32 + (size_t)b * (4 * kDeff * 2 * kN);
    const uint32_t* Ra0 = rg + (size_t)(((2 * p + 0) * kDeff + 0) * 2 + l) * kN;
    const uint32_t* Ra1 = rg + (size_t)(((2 * p + 0) * kDeff + 1) * 2 + l) * kN;
    const uint32_t* Rb0 = rg + (size_t)(((2 * p + 1) * kDeff + 0) * 2 + l) * kN;
    const uint32_t* Rb1 = rg + (size_t)(((2 * p + 1) * kDeff + 1) * 2 + l) * kN;
    uint32_t* xc_me = xcoef + (p * 2 + l) * kN;
    const uint32_t* xc_ot = xcoef + (p * 2 + (1 - l)) * kN;
    uint32_t* xch_out = xch + ((1 - p) * 2 + l) * kN;
    const uint32_t* xch_in = xch + (p * 2 + l) * kN;
    for (long i = (long)len - 2; i >= 0; --i) {
        ntt_inv(acc, mybuf, twi, q, L.inv_n, L.inv_n_p, t, bar);
#pragma unroll
        for (int e = 0; e < 8; ++e) xc_me[t + 256 * e] = acc[e];
        __syncthreads();
        uint32_t d0[8], d1[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t o = xc_ot[t + 256 * e];
            int64_t s1, s2;
            decomp2(l ? o : acc[e], l ? acc[e] : o, *T, s1, s2);
            d0[e] = signed_res(s1, q);
            d1[e] = signed_res(s2, q);
        }
        ntt_fwd(d0, mybuf, twf, q, t, bar);
        ntt_fwd(d1, mybuf, twf, q, t, bar);
        uint32_t a0[8], a1[8], b0[8], b1[8];
        ld8(Ra0 + 8 * t, a0);
        ld8(Ra1 + 8 * t, a1);
        ld8(Rb0 + 8 * t, b0);
        ld8(Rb1 + 8 * t, b1);
        uint32_t own[8], oth[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t ca = mod_u64((uint64_t)d0[e] * a0[e] + (uint64_t)d1[e] * a1[e], L.cr, q);
            const uint32_t cb = mod_u64((uint64_t)d0[e] * b0[e] + (uint64_t)d1[e] * b1[e], L.cr, q);
            own[e] = p ? cb : ca;
            oth[e] = p ? ca : cb;
        }
        st8(xch_out + 8 * t, oth);
        __syncthreads();
        uint32_t o2[8], pk[8];
        ld8(xch_in + 8 * t, o2);
        ld8(src_of(start + (size_t)i) + 8 * t, pk);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[e] = add_mod(add_mod(own[e], o2[e], q), pk[e], q);
    }
    uint64_t* dst = resp + (size_t)b * resp_qstride + ((size_t)ct * 4 + p * 2 + l) * kN + 8 * t;
#pragma unroll
    for (int e = 0; e < 8; e += 2)
        *reinterpret_cast<ulonglong2*>(dst + e) = make_ulonglong2(acc[e], acc[e + 1]);
}

// ------------------------------------------------------------------ horner (cluster)
// The same chain on a cluster of four CTAs, CTA rank r = 2p + l owning
// polynomial p (0 = a, 1 = b) in limb l.  Each CTA has two NTT groups:
// group 0 holds the accumulator and runs the inverse NTT; both groups then
// decompose (CRT needs the partner limb's coefficients) and transform one
// gadget digit each; each digit is multiplied by the RGSW rows of its
// polynomial (held in registers for the whole chain), the contribution to
// the own polynomial stays local, the one to the other polynomial goes to
// that CTA, and group 0 sums.  Remote data moves with st.async into the
// receiver's shared memory and completes bytes on the receiver's mbarrier
// (partner coefficients: 8 KB per step; other-poly contributions: 16 KB per
// step), so the loop has no cluster-wide barrier.  Buffers alternate with
// the step parity; a remote write for step t is issued only after its
// receiver has finished reading the same buffer at step t - 2 (it depends on
// data the receiver sent after that read).  Every wait is bounded.
constexpr size_t kHornerClSmem =
    2 * kN * sizeof(uint2) + (2 * 2 * kN + 2 * 2 * kN + 2 * 4 * kN) * sizeof(uint32_t) + 64;

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t map_peer(const void* local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"((uint32_t)__cvta_generic_to_shared(local)), "r"(rank));
    return r;
}
// 16 bytes into a peer CTA's shared memory, completing 16 bytes on its mbarrier.
__device__ __forceinline__ void st_async4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                          uint32_t mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     addr),
                 "r"(a), "r"(b), "r"(c), "r"(d), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void hb_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(b)));
}
__device__ __forceinline__ void hb_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(b)),
                 "r"(bytes)
                 : "memory");
}
// Bounded wait on a cluster-filled mbarrier phase; false (and *err set) on timeout.
__device__ __forceinline__ bool hb_wait(uint64_t* b, uint32_t parity, int* err, int code) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(b);
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    atomicCAS(err, 0, code);
    return false;
}

__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(512, 1)
    horner_cl_kernel(const uint32_t* __restrict__ pre_a, const uint32_t* __restrict__ packed_b, size_t pb_qstride,
                     const uint32_t* __restrict__ rgsw32, const DevTables* __restrict__ T, size_t groups,
                     size_t d_act, uint64_t* __restrict__ resp, size_t resp_qstride, int* err, HornerRange hr) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint2* twf = reinterpret_cast<uint2*>(smem);
    uint2* twi = twf + kN;
    uint32_t* nbuf = reinterpret_cast<uint32_t*>(twi + kN);   // [2 groups][2][N]
    uint32_t* xc = nbuf + 2 * 2 * kN;                         // [parity][own | partner limb][N]
    uint32_t* cin = xc + 2 * 2 * kN;                          // [parity][local j0 | local j1 | peer j0 | peer j1][N]
    uint64_t* mbx = reinterpret_cast<uint64_t*>(cin + 2 * 4 * kN);  // [parity] partner coefficients
    uint64_t* mbc = mbx + 2;                                         // [parity] other-poly contributions
    __shared__ volatile int abort_flag;
    const uint32_t rank = cluster_rank();
    const int p = (int)(rank >> 1), l = (int)(rank & 1);
    const int ct = blockIdx.x >> 2, b = blockIdx.y;
    const int gp = threadIdx.x >> 8;
    const uint32_t t = threadIdx.x & 255;
    const int bar = 1 + gp;
    const LimbTables& L = T->limb[l];
    const uint32_t q = L.q;
    const uint32_t inv_n = L.inv_n, inv_n_p = L.inv_n_p;
    const CrtK ck = crt_consts(*T);
    for (int i = threadIdx.x; i < kN; i += 512) { twf[i] = L.fwd[i]; twi[i] = L.inv[i]; }
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int k = 0; k < 2; ++k) { hb_init(&mbx[k]); hb_init(&mbc[k]); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const uint32_t rank_limb = (uint32_t)((p << 1) | (1 - l));   // same poly, other limb
    const uint32_t rank_poly = (uint32_t)(((1 - p) << 1) | l);   // other poly, same limb
    const size_t start = (size_t)ct * d_act;
    const size_t len = (start + d_act <= groups) ? d_act : groups - start;
    const uint32_t* pbq = packed_b + (size_t)b * pb_qstride;
    auto src_of = [&](size_t i) -> const uint32_t* {
        return p ? pbq + (i * 2 + l) * kN : pre_a + (i * 2 + l) * kN;
    };
    // RGSW rows of this poly for digit gp: to own output (p' = p) and to the other (p' = 1 - p)
    const uint32_t* rg = rgsw32 + (size_t)b * (4 * kDeff * 2 * kN);
    uint32_t r_self[8], r_oth[8];
    ld8(rg + (size_t)(((2 * p + p) * kDeff + gp) * 2 + l) * kN + 8 * t, r_self);
    ld8(rg + (size_t)(((2 * p + (1 - p)) * kDeff + gp) * 2 + l) * kN + 8 * t, r_oth);
    // Shoup factors of the fixed RGSW values: each product below is then
    // exact with one high multiply instead of a 64-bit Barrett reduction.
    uint32_t r_self_p[8], r_oth_p[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        r_self_p[e] = (uint32_t)(((uint64_t)r_self[e] << 32) / q);
        r_oth_p[e] = (uint32_t)(((uint64_t)r_oth[e] << 32) / q);
    }
    uint32_t acc[8];
    uint32_t* const st_part = hr.state + (((size_t)b * (gridDim.x >> 2) + ct) * 4 + p * 2 + l) * kN;
    if (gp == 0) ld8((hr.i_first < 0 ? src_of(start + len - 1) : st_part) + 8 * t, acc);
    const long i_first = hr.i_first < 0 ? (long)len - 2 : (long)hr.i_first;
    cluster_sync_all();  // every CTA runs and its mbarriers are initialised before any remote access
    const uint32_t peer_x = map_peer(xc, rank_limb);       // partner's xc base
    const uint32_t peer_c = map_peer(cin, rank_poly);      // other poly CTA's cin base
    const uint32_t peer_mbx = map_peer(mbx, rank_limb);
    const uint32_t peer_mbc = map_peer(mbc, rank_poly);
    int step = 0;
    for (long i = i_first; i >= (long)hr.i_last; --i, ++step) {
        const int par = step & 1;
        const uint32_t ph = (uint32_t)(step >> 1) & 1;
        uint32_t* xown = xc + (par * 2 + 0) * kN;
        const uint32_t* xpart = xc + (par * 2 + 1) * kN;
        uint32_t* cp = cin + (size_t)par * 4 * kN;
        if (threadIdx.x == 0) {
            hb_expect(&mbx[par], kN * 4);
            hb_expect(&mbc[par], 2 * kN * 4);
        }
        uint32_t pk[8];
        if (gp == 0) {
            ld8(src_of(start + (size_t)i) + 8 * t, pk);
            ntt_inv(acc, nbuf, twi, q, inv_n, inv_n_p, t, bar);   // acc: index t + 256 e
#pragma unroll
            for (int e = 0; e < 8; ++e) xown[t + 256 * e] = acc[e];
        }
        __syncthreads();  // xown complete; abort_flag is read only here, after a block barrier,
                          // so every thread takes the same branch
        if (abort_flag) break;
        if (gp == 0) {
            // the partner's copy, sent as the contiguous block 8t..8t+7 (16-byte stores)
            const uint32_t* src = xown + 8 * t;
            const uint32_t dst = peer_x + (uint32_t)((par * 2 + 1) * kN + 8 * t) * 4;
            st_async4(dst, src[0], src[1], src[2], src[3], peer_mbx + 8 * par);
            st_async4(dst + 16, src[4], src[5], src[6], src[7], peer_mbx + 8 * par);
        }
        if (!hb_wait(&mbx[par], ph, err, 31)) abort_flag = 1;
        uint32_t d[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t own = xown[t + 256 * e], oth = xpart[t + 256 * e];
            int64_t s1, s2;
            decomp2(l ? oth : own, l ? own : oth, ck, s1, s2);
            d[e] = signed_res(gp ? s2 : s1, q);
        }
        ntt_fwd(d, nbuf + gp * 2 * kN, twf, q, t, bar);
        uint32_t es[8], eo[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            es[e] = csub(shoup_mul(d[e], r_self[e], r_self_p[e], q), q);
            eo[e] = csub(shoup_mul(d[e], r_oth[e], r_oth_p[e], q), q);
        }
        st8(cp + (size_t)gp * kN + 8 * t, es);
        const uint32_t dstc = peer_c + (uint32_t)((size_t)par * 4 * kN + (size_t)(2 + gp) * kN + 8 * t) * 4;
        st_async4(dstc, eo[0], eo[1], eo[2], eo[3], peer_mbc + 8 * par);
        st_async4(dstc + 16, eo[4], eo[5], eo[6], eo[7], peer_mbc + 8 * par);
        __syncthreads();  // local contributions complete
        if (gp == 0) {
            if (!hb_wait(&mbc[par], ph, err, 32)) abort_flag = 1;
            uint32_t v0[8], v1[8], w0[8], w1[8];
            ld8(cp + 8 * t, v0);
            ld8(cp + kN + 8 * t, v1);
            ld8(cp + 2 * kN + 8 * t, w0);
            ld8(cp + 3 * kN + 8 * t, w1);
#pragma unroll
            for (int e = 0; e < 8; ++e)
                acc[e] = add_mod(add_mod(add_mod(v0[e], v1[e], q), add_mod(w0[e], w1[e], q), q), pk[e], q);
        }
    }
    if (gp == 0 && hr.i_last == 0) {
        uint64_t* dst = resp + (size_t)b * resp_qstride + ((size_t)ct * 4 + p * 2 + l) * kN + 8 * t;
#pragma unroll
        for (int e = 0; e < 8; e += 2)
            *reinterpret_cast<ulonglong2*>(dst + e) = make_ulonglong2(acc[e], acc[e + 1]);
    } else if (gp == 0) {
        st8(st_part + 8 * t, acc);  // the chain resumes from here in the next launch
    }
    cluster_sync_all();  // no CTA leaves while a peer may still write into its shared memory
}

// ------------------------------------------------------------------ horner (8-CTA cluster)
// The chain on a cluster of eight CTAs of 256 threads, CTA rank
// r = 4p + 2l + j owning polynomial p, limb l and gadget digit j.  Both digit
// CTAs of (p, l) hold the same accumulator and run its inverse NTT; each
// sends its coefficients to the other limb's CTA of the same digit (CRT needs
// both limbs), decomposes and forward-transforms only its digit, and
// multiplies it by the RGSW rows of its polynomial.  The contribution to its
// own polynomial goes to the sibling digit CTA, the one to the other
// polynomial to both digit CTAs of that polynomial; every CTA then sums its
// own, its sibling's and the two other-polynomial contributions (modular
// sums of canonical residues: both siblings get the same accumulator).
// Remote data moves with st.async and completes on the receiver's
// transaction mbarriers (8 KB of coefficients, 24 KB of contributions per
// step); buffers alternate with the step parity, and every remote write for
// step t depends on data its receiver sent after reading the same buffer at
// step t - 2.  Half the warps per SM of the 4-CTA version, twice the SMs.
constexpr size_t kHornerCl8Smem =
    2 * kN * sizeof(uint2) + (2 * kN + 2 * 2 * kN + 2 * 4 * kN) * sizeof(uint32_t) + 64;

__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(256, 1)
    horner_cl8_kernel(const uint32_t* __restrict__ pre_a, const uint32_t* __restrict__ packed_b, size_t pb_qstride,
                      const uint32_t* __restrict__ rgsw32, const DevTables* __restrict__ T, size_t groups,
                      size_t d_act, uint64_t* __restrict__ resp, size_t resp_qstride, int* err, HornerRange hr) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint2* twf = reinterpret_cast<uint2*>(smem);
    uint2* twi = twf + kN;
    uint32_t* nbuf = reinterpret_cast<uint32_t*>(twi + kN);  // [2][N] NTT scratch
    uint32_t* xc = nbuf + 2 * kN;                            // [parity][own | partner limb][N]
    uint32_t* cin = xc + 2 * 2 * kN;                         // [parity][own | sibling | other j0 | other j1][N]
    uint64_t* mbx = reinterpret_cast<uint64_t*>(cin + 2 * 4 * kN);  // [parity] partner coefficients
    uint64_t* mbc = mbx + 2;                                         // [parity] contributions
    __shared__ volatile int abort_flag;
    const uint32_t rank = cluster_rank();
    const int p = (int)(rank >> 2), l = (int)((rank >> 1) & 1), j = (int)(rank & 1);
    const int ct = blockIdx.x >> 3, b = blockIdx.y;
    const uint32_t t = threadIdx.x;
    const LimbTables& L = T->limb[l];
    const uint32_t q = L.q;
    const uint32_t inv_n = L.inv_n, inv_n_p = L.inv_n_p;
    const CrtK ck = crt_consts(*T);
    for (int i = threadIdx.x; i < kN; i += 256) { twf[i] = L.fwd[i]; twi[i] = L.inv[i]; }
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int k = 0; k < 2; ++k) { hb_init(&mbx[k]); hb_init(&mbc[k]); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const uint32_t rank_limb = (uint32_t)((p << 2) | ((1 - l) << 1) | j);   // same poly and digit, other limb
    const uint32_t rank_sib = (uint32_t)((p << 2) | (l << 1) | (1 - j));    // same poly and limb, other digit
    const uint32_t rank_o0 = (uint32_t)(((1 - p) << 2) | (l << 1) | 0);     // other poly, same limb, digit 0
    const uint32_t rank_o1 = (uint32_t)(((1 - p) << 2) | (l << 1) | 1);     //                        digit 1
    const size_t start = (size_t)ct * d_act;
    const size_t len = (start + d_act <= groups) ? d_act : groups - start;
    const uint32_t* pbq = packed_b + (size_t)b * pb_qstride;
    auto src_of = [&](size_t i) -> const uint32_t* {
        return p ? pbq + (i * 2 + l) * kN : pre_a + (i * 2 + l) * kN;
    };
    const uint32_t* rg = rgsw32 + (size_t)b * (4 * kDeff * 2 * kN);
    uint32_t r_self[8], r_oth[8];
    ld8(rg + (size_t)(((2 * p + p) * kDeff + j) * 2 + l) * kN + 8 * t, r_self);
    ld8(rg + (size_t)(((2 * p + (1 - p)) * kDeff + j) * 2 + l) * kN + 8 * t, r_oth);
    // Shoup factors of the fixed RGSW values: each product below is then
    // exact with one high multiply instead of a 64-bit Barrett reduction.
    uint32_t r_self_p[8], r_oth_p[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        r_self_p[e] = (uint32_t)(((uint64_t)r_self[e] << 32) / q);
        r_oth_p[e] = (uint32_t)(((uint64_t)r_oth[e] << 32) / q);
    }
    uint32_t acc[8];
    uint32_t* const st_part = hr.state + (((size_t)b * (gridDim.x >> 3) + ct) * 4 + p * 2 + l) * kN;
    ld8((hr.i_first < 0 ? src_of(start + len - 1) : st_part) + 8 * t, acc);
    const long i_first = hr.i_first < 0 ? (long)len - 2 : (long)hr.i_first;
    cluster_sync_all();  // every CTA runs and its mbarriers are initialised before any remote access
    const uint32_t peer_x = map_peer(xc, rank_limb);
    const uint32_t peer_mbx = map_peer(mbx, rank_limb);
    const uint32_t sib_c = map_peer(cin, rank_sib), sib_mbc = map_peer(mbc, rank_sib);
    const uint32_t o0_c = map_peer(cin, rank_o0), o0_mbc = map_peer(mbc, rank_o0);
    const uint32_t o1_c = map_peer(cin, rank_o1), o1_mbc = map_peer(mbc, rank_o1);
    int step = 0;
    for (long i = i_first; i >= (long)hr.i_last; --i, ++step) {
        const int par = step & 1;
        const uint32_t ph = (uint32_t)(step >> 1) & 1;
        uint32_t* xown = xc + (par * 2 + 0) * kN;
        const uint32_t* xpart = xc + (par * 2 + 1) * kN;
        uint32_t* cp = cin + (size_t)par * 4 * kN;
        if (threadIdx.x == 0) {
            hb_expect(&mbx[par], kN * 4);
            hb_expect(&mbc[par], 3 * kN * 4);
        }
        uint32_t pk[8];
        ld8(src_of(start + (size_t)i) + 8 * t, pk);
        ntt_inv(acc, nbuf, twi, q, inv_n, inv_n_p, t, 0);   // acc: index t + 256 e
#pragma unroll
        for (int e = 0; e < 8; ++e) xown[t + 256 * e] = acc[e];
        __syncthreads();  // xown complete; abort_flag is read only here, after a block barrier
        if (abort_flag) break;
        {
            const uint32_t* src = xown + 8 * t;
            const uint32_t dst = peer_x + (uint32_t)((par * 2 + 1) * kN + 8 * t) * 4;
            st_async4(dst, src[0], src[1], src[2], src[3], peer_mbx + 8 * par);
            st_async4(dst + 16, src[4], src[5], src[6], src[7], peer_mbx + 8 * par);
        }
        if (!hb_wait(&mbx[par], ph, err, 33)) abort_flag = 1;
        uint32_t d[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t own = acc[e], oth = xpart[t + 256 * e];  // own: still in registers
            int64_t s1, s2;
            decomp2(l ? oth : own, l ? own : oth, ck, s1, s2);
            d[e] = signed_res(j ? s2 : s1, q);
        }
        ntt_fwd(d, nbuf, twf, q, t, 0);
        uint32_t es[8], eo[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            es[e] = csub(shoup_mul(d[e], r_self[e], r_self_p[e], q), q);
            eo[e] = csub(shoup_mul(d[e], r_oth[e], r_oth_p[e], q), q);
        }
        const uint32_t off = (uint32_t)((size_t)par * 4 * kN + 8 * t) * 4;
        st_async4(sib_c + off + kN * 4, es[0], es[1], es[2], es[3], sib_mbc + 8 * par);
        st_async4(sib_c + off + kN * 4 + 16, es[4], es[5], es[6], es[7], sib_mbc + 8 * par);
        const uint32_t off_o = off + (uint32_t)(2 + j) * kN * 4;
        st_async4(o0_c + off_o, eo[0], eo[1], eo[2], eo[3], o0_mbc + 8 * par);
        st_async4(o0_c + off_o + 16, eo[4], eo[5], eo[6], eo[7], o0_mbc + 8 * par);
        st_async4(o1_c + off_o, eo[0], eo[1], eo[2], eo[3], o1_mbc + 8 * par);
        st_async4(o1_c + off_o + 16, eo[4], eo[5], eo[6], eo[7], o1_mbc + 8 * par);
        if (!hb_wait(&mbc[par], ph, err, 34)) abort_flag = 1;
        uint32_t v1[8], w0[8], w1[8];
        ld8(cp + kN + 8 * t, v1);
        ld8(cp + 2 * kN + 8 * t, w0);
        ld8(cp + 3 * kN + 8 * t, w1);
#pragma unroll
        for (int e = 0; e < 8; ++e)
            acc[e] = add_mod(add_mod(add_mod(es[e], v1[e], q), add_mod(w0[e], w1[e], q), q), pk[e], q);
    }
    if (j == 0 && hr.i_last == 0) {
        uint64_t* dst = resp + (size_t)b * resp_qstride + ((size_t)ct * 4 + p * 2 + l) * kN + 8 * t;
#pragma unroll
        for (int e = 0; e < 8; e += 2)
            *reinterpret_cast<ulonglong2*>(dst + e) = make_ulonglong2(acc[e], acc[e + 1]);
    } else if (j == 0) {
        st8(st_part + 8 * t, acc);  // the chain resumes from here in the next launch
    }
    cluster_sync_all();  // no CTA leaves while a peer may still write into its shared memory
}

// ------------------------------------------------------------------ primitives
__global__ void __launch_bounds__(1024) ntt_batch_kernel(uint32_t* polys, size_t n, int limb_run, bool inverse,
                                                         const DevTables* __restrict__ T) {
    extern __shared__ __align__(16) uint32_t nb[];
    const int gp = threadIdx.x >> 8;
    const uint32_t t = threadIdx.x & 255;
    const size_t idx = (size_t)blockIdx.x * 4 + gp;
    if (idx >= n) return;  // whole group leaves; only group-local barriers follow
    const int l = (int)((idx / (size_t)limb_run) & 1);
    const LimbTables& L = T->limb[l];
    uint32_t* pp = polys + idx * kN;
    uint32_t r[8];
    if (!inverse) {
#pragma unroll
        for (int e = 0; e < 8; ++e) r[e] = pp[t + 256 * e];
        ntt_fwd(r, nb + gp * 2 * kN, L.fwd, L.q, t, 1 + gp);
        st8(pp + 8 * t, r);
    } else {
        ld8(pp + 8 * t, r);
        ntt_inv(r, nb + gp * 2 * kN, L.inv, L.q, L.inv_n, L.inv_n_p, t, 1 + gp);
#pragma unroll
        for (int e = 0; e < 8; ++e) pp[t + 256 * e] = r[e];
    }
}

__global__ void decomp_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n,
                              const DevTables* __restrict__ T) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * kN) return;
    const size_t i = k / kN, x = k % kN;
    int64_t s1, s2;
    decomp2(in[(i * 2) * kN + x], in[(i * 2 + 1) * kN + x], *T, s1, s2);
    uint32_t* o = out + i * kDeff * 2 * kN;
    o[(0 * 2 + 0) * kN + x] = signed_res(s1, kQ0);
    o[(0 * 2 + 1) * kN + x] = signed_res(s1, kQ1);
    o[(1 * 2 + 0) * kN + x] = signed_res(s2, kQ0);
    o[(1 * 2 + 1) * kN + x] = signed_res(s2, kQ1);
}

__global__ void __launch_bounds__(256) fill_db_kernel(uint16_t* __restrict__ out, size_t count, uint64_t seed) {
    for (size_t k = (size_t)blockIdx.x * 256 + threadIdx.x; k < count; k += (size_t)gridDim.x * 256) {
        uint64_t x = (seed ^ k) + 0x9e3779b97f4a7c15ULL;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
        x ^= x >> 31;
        out[k] = (uint16_t)(x % 65535u);
    }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// Synthetic queries for load generation: word k of query `id` (flat layout
// [b limb0: R][b limb1: R][6 blocks of [digit][limb][N]]) is
// splitmix64(splitmix64(seed ^ id * C) ^ k) mod q_l, l the limb of word k.
// Grid-stride over count * qstride words, coalesced writes.
__global__ void __launch_bounds__(256) synth_query_kernel(uint64_t* __restrict__ out, size_t rows, size_t qstride,
                                                          size_t count, uint64_t seed, uint64_t first_id) {
    const size_t total = count * qstride;
    for (size_t w = (size_t)blockIdx.x * 256 + threadIdx.x; w < total; w += (size_t)gridDim.x * 256) {
        const size_t j = w / qstride, k = w - j * qstride;
        const uint64_t h = splitmix64(seed ^ ((first_id + j) * 0xd1b54a32d192ed03ULL));
        const uint64_t x = splitmix64(h ^ k);
        const int l = k < rows ? 0 : k < 2 * rows ? 1 : (int)(((k - 2 * rows) / kN) & 1);
        out[w] = x % (l ? kQ1 : kQ0);
    }
}

}  // namespace

cudaError_t launch_synth_queries(uint64_t* out, size_t rows, size_t count, uint64_t seed, uint64_t first_id,
                                 cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const size_t qstride = 2 * rows + 6 * (size_t)kDeff * 2 * kN;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t blocks = std::min<size_t>((count * qstride + 255) / 256, (size_t)sms * 16);
    synth_query_kernel<<<(unsigned)blocks, 256, 0, s>>>(out, rows, qstride, count, seed, first_id);
    return cudaGetLastError();
}

cudaError_t launch_fill_db(uint16_t* out, size_t count, uint64_t seed, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t blocks = std::min<size_t>((count + 255) / 256, (size_t)sms * 16);
    fill_db_kernel<<<(unsigned)blocks, 256, 0, s>>>(out, count, seed);
    return cudaGetLastError();
}

// ==================================================================== wrappers
cudaError_t launch_qprep(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T,
                         uint32_t* keys, uint32_t* rgsw32, int nq, cudaStream_t s) {
    return launch_qprep_parts(qraw, qstride, rows, T, keys, rgsw32, nq, 3, s);
}

cudaError_t launch_qprep_parts(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T,
                               uint32_t* keys, uint32_t* rgsw32, int nq, int parts, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (parts < 1 || parts > 3) return cudaErrorInvalidValue;
    const int y0 = (parts & 1) ? 0 : 8, y1 = (parts & 2) ? 12 : 8;  // rows 0-7: key NTTs, 8-11: RGSW
    qprep_kernel<<<dim3(nq, y1 - y0), 256, 0, s>>>(qraw, qstride, rows, T, keys, rgsw32, y0);
    return cudaGetLastError();
}

cudaError_t launch_matvec(const uint16_t* db, size_t rows, size_t cols, int chunks, const uint64_t* qraw,
                          size_t qstride, const DevTables* T, uint32_t* part, size_t part_qstride, int nq,
                          cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (nq > 4 || chunks <= 0 || rows % (size_t)chunks) return cudaErrorInvalidValue;
    const int rpc = (int)(rows / chunks);
    if (rpc > (1 << 20)) return cudaErrorInvalidValue;
    const int bt = nq == 1 ? 1 : (nq == 2 ? 2 : 4);
    const size_t smem = (size_t)bt * 2 * rpc * sizeof(uint32_t);
    cudaError_t e;
    if (bt == 1) {
        auto k = matvec_kernel<1, 8>;
        if ((e = allow_max_smem(k))) return e;
        k<<<dim3((unsigned)(cols / 2048), chunks), 256, smem, s>>>(db, rows, cols, rpc, qraw, qstride, T, part,
                                                                   part_qstride, nq);
    } else if (bt == 2) {
        auto k = matvec_kernel<2, 4>;
        if ((e = allow_max_smem(k))) return e;
        k<<<dim3((unsigned)(cols / 1024), chunks), 256, smem, s>>>(db, rows, cols, rpc, qraw, qstride, T, part,
                                                                   part_qstride, nq);
    } else {
        auto k = matvec_kernel<4, 4>;
        if ((e = allow_max_smem(k))) return e;
        k<<<dim3((unsigned)(cols / 1024), chunks), 256, smem, s>>>(db, rows, cols, rpc, qraw, qstride, T, part,
                                                                   part_qstride, nq);
    }
    return cudaGetLastError();
}

cudaError_t launch_finalize(const uint32_t* mvpart, size_t mv_qstride, int mv_chunks, size_t cols,
                            const uint32_t* tp_out, const uint32_t* df, const uint32_t* keys, size_t key_qstride,
                            const DevTables* T, uint32_t* packed_b, size_t pb_qstride, size_t groups, int nq,
                            cudaStream_t s) {
    return launch_finalize_range(mvpart, mv_qstride, mv_chunks, cols, tp_out, nq, 0, df, keys, key_qstride, T,
                                 packed_b, pb_qstride, groups, 0, groups, nq, s);
}

cudaError_t launch_finalize_range(const uint32_t* mvpart, size_t mv_qstride, int mv_chunks, size_t cols,
                                  const uint32_t* tp_out, int tp_nq_total, int tp_q0, const uint32_t* df,
                                  const uint32_t* keys, size_t key_qstride, const DevTables* T, uint32_t* packed_b,
                                  size_t pb_qstride, size_t groups, size_t g0, size_t gn, int nq, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (gn == 0 || g0 + gn > groups || tp_q0 < 0 || tp_q0 + nq > tp_nq_total) return cudaErrorInvalidValue;
    finalize_kernel<<<dim3((unsigned)gn, 2, nq), 256, 0, s>>>(mvpart, mv_qstride, mv_chunks, cols, tp_out,
                                                              tp_nq_total, tp_q0, (int)groups, (int)g0, df, keys,
                                                              key_qstride, T, packed_b, pb_qstride);
    return cudaGetLastError();
}

cudaError_t launch_horner(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                          const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                          size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    cudaError_t e = allow_max_smem(horner_kernel);
    if (e) return e;
    horner_kernel<<<dim3((unsigned)num_cts, nq), 1024, kHornerSmem, s>>>(pre_a, packed_b, pb_qstride, rgsw32, T,
                                                                          groups, d_act, resp, resp_qstride);
    return cudaGetLastError();
}

static bool horner_range_ok(const HornerRange& hr, size_t d_act) {
    if (hr.i_first < 0 && hr.i_last == 0) return true;  // the whole chain
    return hr.state && hr.i_last >= 0 && hr.i_first < (long)d_act - 1 && (hr.i_first < 0 || hr.i_first >= hr.i_last);
}

cudaError_t launch_horner_cluster(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                                  const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                                  size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, int* err,
                                  cudaStream_t s, HornerRange hr) {
    if (nq <= 0) return cudaSuccess;
    if (!horner_range_ok(hr, d_act)) return cudaErrorInvalidValue;
    cudaError_t e = allow_max_smem(horner_cl_kernel);
    if (e) return e;
    horner_cl_kernel<<<dim3((unsigned)(4 * num_cts), nq), 512, kHornerClSmem, s>>>(pre_a, packed_b, pb_qstride,
                                                                                   rgsw32, T, groups, d_act, resp,
                                                                                   resp_qstride, err, hr);
    return cudaGetLastError();
}

cudaError_t launch_horner_cluster8(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                                   const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                                   size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, int* err,
                                   cudaStream_t s, HornerRange hr) {
    if (nq <= 0) return cudaSuccess;
    if (!horner_range_ok(hr, d_act)) return cudaErrorInvalidValue;
    cudaError_t e = allow_max_smem(horner_cl8_kernel);
    if (e) return e;
    horner_cl8_kernel<<<dim3((unsigned)(8 * num_cts), nq), 256, kHornerCl8Smem, s>>>(
        pre_a, packed_b, pb_qstride, rgsw32, T, groups, d_act, resp, resp_qstride, err, hr);
    return cudaGetLastError();
}

cudaError_t launch_ntt_batch(uint32_t* polys, size_t n, int limb_run, bool inverse, const DevTables* T,
                             cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t smem = 4 * 2 * kN * sizeof(uint32_t);
    cudaError_t e = allow_max_smem(ntt_batch_kernel);
    if (e) return e;
    ntt_batch_kernel<<<(unsigned)((n + 3) / 4), 1024, smem, s>>>(polys, n, limb_run, inverse, T);
    return cudaGetLastError();
}

cudaError_t launch_decomp(const uint32_t* in, uint32_t* out, size_t n, const DevTables* T, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    decomp_kernel<<<(unsigned)((n * kN + 255) / 256), 256, 0, s>>>(in, out, n, T);
    return cudaGetLastError();
}

}  // namespace ipb
