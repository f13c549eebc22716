// ipb_common.cuh -- constants, exact modular arithmetic and the 2048-point
// negacyclic NTT shared by every kernel of the B200 InsPIRe server.
//
// Ring Z_q[X]/(X^2048+1), q = q0*q1 with the two 27-bit NTT primes of the
// reference (src/params.h:15-18).  Residues are u32 in [0, q).
//
// NTT convention (must match the reference's CPU/GPU NTT bit for bit,
// src/ntt.cpp:107-149): Cooley-Tukey DIT forward with twiddles
// fwd[i] = psi^BR(i), Gentleman-Sande inverse with inv[i] = fwd[i]^-1 and a
// final N^-1 scale.  Output slot i holds the evaluation at psi^(2 BR(i)+1).
// Every stage here computes the same mathematical transform with Harvey
// lazy reduction and a final reduction to [0, q), so results are identical.
//
// The transform runs on one "NTT group" of 256 threads holding 8 elements
// each in registers; three shared-memory exchanges (XOR-swizzled, bank
// conflict free) move between the four register layouts
//   L1: x = t + 256 e        stages s = 10, 9, 8
//   L2: x = (t&31) + 32 e + 256 (t>>5)   s = 7, 6, 5
//   L3: x = (t&3) + 4 e + 32 (t>>2)      s = 4, 3, 2
//   L4: x = 8 t + e          stages s = 1, 0
// A forward NTT takes L1 in and leaves L4; the inverse takes L4 to L1.
// Only L1 <-> L2 moves data between warps: in L2, L3 and L4 warp w holds
// x in [256w, 256w + 256), a region the swizzle keeps in place, so those
// exchanges need a warp barrier only.  Each transform starts with a group
// barrier before its first store, which orders it after the previous
// transform's reads of the same buffer; the second buffer is only ever
// touched warp-locally.
// Several groups can share a CTA, each synchronising on its own named
// barrier (bar.sync id, 256).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ipb {

constexpr int kN = 2048;
constexpr int kLogN = 11;
constexpr int kHalf = kN / 2;
constexpr int kSteps = kHalf - 1;      // collapse steps per direction
constexpr int kDgsw = 3;               // gadget digits (src/params.h:26-29)
constexpr int kDeff = 2;               // digits kept (digit 0 dropped)
constexpr int kBaseLog = 18;
constexpr uint32_t kQ0 = 94519297u;
constexpr uint32_t kQ1 = 95293441u;
constexpr uint32_t kP = 65535u;        // plaintext modulus (Mersenne)
constexpr uint64_t kQFull = (uint64_t)kQ0 * kQ1;

// Per-limb tables, one set per device.  tw* entries are (w, floor(w 2^32/q)).
struct LimbTables {
    uint2 fwd[kN];
    uint2 inv[kN];
    uint32_t q;
    uint32_t inv_n, inv_n_p;     // N^-1 and its Shoup factor
    uint64_t cr;                 // floor(2^64 / q), exact u64 Barrett
};
struct DevTables {
    LimbTables limb[2];
    uint32_t crt_c[2], crt_cp[2];  // q1^-1 mod q0, q0^-1 mod q1 and Shoup factors
};

// ------------------------------------------------------------ arithmetic
__device__ __forceinline__ uint32_t shoup_mul(uint32_t x, uint32_t w, uint32_t wp, uint32_t q) {
    // x < 2^32, w < q: returns x*w mod q in [0, 2q).
    uint32_t t = __umulhi(x, wp);
    return x * w - t * q;
}
__device__ __forceinline__ uint32_t csub(uint32_t x, uint32_t m) {
    // x < 2m  ->  x mod m (unsigned wrap makes x-m huge when x < m).
    return min(x, x - m);
}
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) { return csub(a + b, q); }
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t q) { return csub(a + q - b, q); }
__device__ __forceinline__ uint32_t mod_u64(uint64_t x, uint64_t cr, uint32_t q) {
    // Exact for every u64: the quotient estimate is low by at most 1.
    uint64_t t = __umul64hi(x, cr);
    uint64_t r = x - t * (uint64_t)q;
    return (uint32_t)(r >= q ? r - q : r);
}
__device__ __forceinline__ uint32_t brev11(uint32_t x) { return __brev(x) >> (32 - kLogN); }

// Slot permutation of the automorphism tau_t in NTT form: result slot x is
// source slot perm(t, x) (src/gpu_preprocess.cu:158-194).  `odd` = 2 BR(x)+1.
__device__ __forceinline__ uint32_t perm_from_odd(uint32_t t, uint32_t odd) {
    uint32_t e = (t * odd) & (2 * kN - 1);
    return brev11((e - 1) >> 1);
}

// ------------------------------------------------------------ barriers
__device__ __forceinline__ void gsync(int bar) {
    if (bar == 0) __syncthreads();
    else asm volatile("bar.sync %0, 256;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ uint32_t swz(uint32_t x) { return x ^ ((x >> 3) & 0x1Cu); }

// ------------------------------------------------------------ butterflies
__device__ __forceinline__ void bf_fwd(uint32_t& u, uint32_t& v, uint2 w, uint32_t q) {
    const uint32_t q2 = 2 * q;
    uint32_t uu = csub(u, q2);                 // [0, 2q)
    uint32_t tt = shoup_mul(v, w.x, w.y, q);   // [0, 2q)
    u = uu + tt;                               // [0, 4q)
    v = uu + q2 - tt;                          // (0, 4q)
}
__device__ __forceinline__ void bf_inv(uint32_t& u, uint32_t& v, uint2 w, uint32_t q) {
    const uint32_t q2 = 2 * q;
    uint32_t s = csub(u + v, q2);              // inputs < 2q -> [0, 2q)
    uint32_t d = u + q2 - v;                   // (0, 4q)
    v = shoup_mul(d, w.x, w.y, q);             // [0, 2q)
    u = s;
}

// One stage on the register tile: e-bit k <-> x-bit (B0 + k).
template <int B0, bool FWD>
__device__ __forceinline__ void ntt_stage(uint32_t (&r)[8], const int k, const uint32_t xbase,
                                          const uint2* __restrict__ tw, uint32_t q) {
    const int s = B0 + k;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        if (e & (1 << k)) continue;
        const int e2 = e | (1 << k);
        const uint32_t x = xbase + ((uint32_t)e << B0);
        const uint2 w = tw[(1u << (10 - s)) + (x >> (s + 1))];
        if (FWD) bf_fwd(r[e], r[e2], w, q);
        else bf_inv(r[e], r[e2], w, q);
    }
}

// Layout helpers: xbase and B0 per layout id (1..4).
template <int L> __device__ __forceinline__ uint32_t lay_base(uint32_t t);
template <> __device__ __forceinline__ uint32_t lay_base<1>(uint32_t t) { return t; }
template <> __device__ __forceinline__ uint32_t lay_base<2>(uint32_t t) { return (t & 31) + 256 * (t >> 5); }
template <> __device__ __forceinline__ uint32_t lay_base<3>(uint32_t t) { return (t & 3) + 32 * (t >> 2); }
template <> __device__ __forceinline__ uint32_t lay_base<4>(uint32_t t) { return 8 * t; }
template <int L> struct LayB0;
template <> struct LayB0<1> { static constexpr int v = 8; };
template <> struct LayB0<2> { static constexpr int v = 5; };
template <> struct LayB0<3> { static constexpr int v = 2; };
template <> struct LayB0<4> { static constexpr int v = 0; };

template <int L>
__device__ __forceinline__ void lay_store(const uint32_t (&r)[8], uint32_t* s, uint32_t t) {
    if (L == 4) {
        *reinterpret_cast<uint4*>(s + swz(8 * t)) = make_uint4(r[0], r[1], r[2], r[3]);
        *reinterpret_cast<uint4*>(s + swz(8 * t + 4)) = make_uint4(r[4], r[5], r[6], r[7]);
    } else {
        const uint32_t b = lay_base<L>(t);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[swz(b + ((uint32_t)e << LayB0<L>::v))] = r[e];
    }
}
template <int L>
__device__ __forceinline__ void lay_load(uint32_t (&r)[8], const uint32_t* s, uint32_t t) {
    if (L == 4) {
        uint4 a = *reinterpret_cast<const uint4*>(s + swz(8 * t));
        uint4 b = *reinterpret_cast<const uint4*>(s + swz(8 * t + 4));
        r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
        r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
    } else {
        const uint32_t b = lay_base<L>(t);
#pragma unroll
        for (int e = 0; e < 8; ++e) r[e] = s[swz(b + ((uint32_t)e << LayB0<L>::v))];
    }
}

// Forward NTT: r in L1 (any values < 4q) -> r in L4, canonical [0, q).
// sbuf: 2*2048 u32 private to this group.  All 256 threads must call.
__device__ __forceinline__ void ntt_fwd(uint32_t (&r)[8], uint32_t* sbuf, const uint2* __restrict__ tw,
                                        uint32_t q, uint32_t t, int bar) {
    uint32_t* A = sbuf;
    uint32_t* B = sbuf + kN;
    ntt_stage<8, true>(r, 2, lay_base<1>(t), tw, q);
    ntt_stage<8, true>(r, 1, lay_base<1>(t), tw, q);
    ntt_stage<8, true>(r, 0, lay_base<1>(t), tw, q);
    gsync(bar);
    lay_store<1>(r, A, t); gsync(bar); lay_load<2>(r, A, t);
    ntt_stage<5, true>(r, 2, lay_base<2>(t), tw, q);
    ntt_stage<5, true>(r, 1, lay_base<2>(t), tw, q);
    ntt_stage<5, true>(r, 0, lay_base<2>(t), tw, q);
    lay_store<2>(r, B, t); __syncwarp(); lay_load<3>(r, B, t);
    ntt_stage<2, true>(r, 2, lay_base<3>(t), tw, q);
    ntt_stage<2, true>(r, 1, lay_base<3>(t), tw, q);
    ntt_stage<2, true>(r, 0, lay_base<3>(t), tw, q);
    lay_store<3>(r, A, t); __syncwarp(); lay_load<4>(r, A, t);
    ntt_stage<0, true>(r, 1, lay_base<4>(t), tw, q);
    ntt_stage<0, true>(r, 0, lay_base<4>(t), tw, q);
    const uint32_t q2 = 2 * q;
#pragma unroll
    for (int e = 0; e < 8; ++e) r[e] = csub(csub(r[e], q2), q);
}

// Inverse NTT incl. N^-1: r in L4 (values < 2q) -> r in L1, canonical.
__device__ __forceinline__ void ntt_inv(uint32_t (&r)[8], uint32_t* sbuf, const uint2* __restrict__ tw,
                                        uint32_t q, uint32_t inv_n, uint32_t inv_n_p, uint32_t t, int bar) {
    uint32_t* A = sbuf;
    uint32_t* B = sbuf + kN;
    ntt_stage<0, false>(r, 0, lay_base<4>(t), tw, q);
    ntt_stage<0, false>(r, 1, lay_base<4>(t), tw, q);
    gsync(bar);
    lay_store<4>(r, A, t); __syncwarp(); lay_load<3>(r, A, t);
    ntt_stage<2, false>(r, 0, lay_base<3>(t), tw, q);
    ntt_stage<2, false>(r, 1, lay_base<3>(t), tw, q);
    ntt_stage<2, false>(r, 2, lay_base<3>(t), tw, q);
    lay_store<3>(r, B, t); __syncwarp(); lay_load<2>(r, B, t);
    ntt_stage<5, false>(r, 0, lay_base<2>(t), tw, q);
    ntt_stage<5, false>(r, 1, lay_base<2>(t), tw, q);
    ntt_stage<5, false>(r, 2, lay_base<2>(t), tw, q);
    lay_store<2>(r, A, t); gsync(bar); lay_load<1>(r, A, t);
    ntt_stage<8, false>(r, 0, lay_base<1>(t), tw, q);
    ntt_stage<8, false>(r, 1, lay_base<1>(t), tw, q);
    ntt_stage<8, false>(r, 2, lay_base<1>(t), tw, q);
#pragma unroll
    for (int e = 0; e < 8; ++e) r[e] = csub(shoup_mul(r[e], inv_n, inv_n_p, q), q);
}

// ------------------------------------------------------------ gadget decomposition
// One coefficient: CRT lift of (c0 mod q0, c1 mod q1) to [0, Q), center to
// (-Q/2, Q/2], three signed base-2^18 digits, digit 0 dropped
// (src/ring.cpp:205-246).  Returns digits 1 and 2 as signed values.
// The CRT factors in registers: kernels whose loops contain asm with memory
// clobbers (mbarrier waits, st.async) would otherwise reload them from the
// table in global memory at every use.
struct CrtK {
    uint32_t c0, cp0, c1, cp1;
};
__device__ __forceinline__ CrtK crt_consts(const DevTables& T) {
    return CrtK{T.crt_c[0], T.crt_cp[0], T.crt_c[1], T.crt_cp[1]};
}
__device__ __forceinline__ void decomp2(uint32_t c0, uint32_t c1, const CrtK& k, int64_t& d1, int64_t& d2) {
    uint32_t t0 = csub(shoup_mul(c0, k.c0, k.cp0, kQ0), kQ0);
    uint32_t t1 = csub(shoup_mul(c1, k.c1, k.cp1, kQ1), kQ1);
    uint64_t v = (uint64_t)t0 * kQ1 + (uint64_t)t1 * kQ0;   // < 2Q
    if (v >= kQFull) v -= kQFull;
    int64_t r = (v <= kQFull / 2) ? (int64_t)v : (int64_t)v - (int64_t)kQFull;
    constexpr int K = 64 - kBaseLog;
    int64_t d0 = (int64_t)((uint64_t)r << K) >> K;
    r = (r - d0) >> kBaseLog;
    d1 = (int64_t)((uint64_t)r << K) >> K;
    r = (r - d1) >> kBaseLog;
    d2 = (int64_t)((uint64_t)r << K) >> K;
}
__device__ __forceinline__ void decomp2(uint32_t c0, uint32_t c1, const DevTables& T, int64_t& d1, int64_t& d2) {
    decomp2(c0, c1, crt_consts(T), d1, d2);
}
__device__ __forceinline__ uint32_t signed_res(int64_t d, uint32_t q) {
    return d >= 0 ? (uint32_t)d : (uint32_t)((int64_t)q + d);
}

}  // namespace ipb
