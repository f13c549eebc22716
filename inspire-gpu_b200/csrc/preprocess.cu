// preprocess.cu -- offline kernels of the B200 InsPIRe server.
//
// gpu_preprocess (reference src/gpu_protocol.cu:535-817) builds, per
// packing group g of N DB columns, the precomputed tensors the online
// tensor pass streams:
//   encode        in-place inverse DFT over Z_P[X]/(X^N+1) across the
//                 D_act column-polys of each row block (src/gpu_preprocess.cu:931-1070)
//   a_side        acc_j = sum_r NTT(db column j, rows r*N..) (.) crs_r
//                 (src/gpu_preprocess.cu:347-410)
//   col_ntt +     ring_embed + automorphisms (src/gpu_preprocess.cu:39-194).
//   embed_gather  The reference evaluates n^3 MACs against a 32 MB monomial
//                 table.  Since mono[e][i] = zeta_i^e, its output is
//                 a_post_fwd[k][i] = A_{perm_{5^k}(i)}(zeta_i) and
//                 a_post_conj[k][i] = A_{perm_{-5^k}(i)}(zeta_i) with
//                 A_p(z) = sum_j a32[j][p] z^j (5^N = 1 mod 2N), i.e. one
//                 forward NTT per slot p along the column index j plus a
//                 gather: N NTTs instead of N^3 MACs, exact, same residues.
//   collapse_a    CollapseA: two serial chains of 1023 steps per group
//                 (src/gpu_preprocess.cu:452-881), one CTA per (group,
//                 direction), the KSK permutations computed in registers.
//   collapse_final  CollapseOne -> D_final and the packed a.
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
constexpr uint32_t kInv5 = 3277;

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
__device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b, const LimbTables& L) {
    return mod_u64((uint64_t)a * b, L.cr, L.q);
}

// ------------------------------------------------------------------ encode
// One CTA = one row, one ct block, one set of 2^nl positions whose bits
// [l0, l0+nl) vary.  Levels l0..l0+nl-1 of the radix-2 DIT butterfly network
// run out of shared memory (double-buffered u16 polys); the first pass
// gathers its inputs in bit-reversed order from the raw upload, the last
// scales by D^-1 mod P.  Each butterfly is the reference's: t = X^ex * odd
// (negacyclic rotation), even + t and even - t with one conditional
// subtraction of P each.
__global__ void __launch_bounds__(256) encode_pass_kernel(const uint16_t* __restrict__ src, uint16_t* dst,
                                                          size_t cols, size_t d_act, int logd, int l0, int nl,
                                                          bool first, bool last, uint32_t d_inv) {
    extern __shared__ __align__(16) uint16_t eb[];  // [2][NP][N]
    const int NP = 1 << nl;
    const size_t nsets = d_act >> nl;
    const size_t row = blockIdx.x;
    const size_t ct = blockIdx.y / nsets, set = blockIdx.y % nsets;
    const size_t lowmask = ((size_t)1 << l0) - 1;
    const size_t dbase = (set & lowmask) + ((set >> l0) << (l0 + nl));
    uint16_t* A = eb;
    uint16_t* B = eb + NP * kN;
    const size_t rowoff = row * cols + ct * d_act * kN;
    for (int m = 0; m < NP; ++m) {
        const size_t d = dbase + ((size_t)m << l0);
        size_t sp = d;
        if (first) {
            sp = 0;
            for (int b = 0; b < logd; ++b)
                if (d & ((size_t)1 << b)) sp |= (size_t)1 << (logd - 1 - b);
        }
        const uint4* s4 = reinterpret_cast<const uint4*>((first ? src : dst) + rowoff + sp * kN);
        uint4* a4 = reinterpret_cast<uint4*>(A + m * kN);
        for (int k = threadIdx.x; k < kN / 8; k += blockDim.x) a4[k] = s4[k];
    }
    __syncthreads();
    for (int lv = 0; lv < nl; ++lv) {
        const int level = l0 + lv;
        const size_t half = (size_t)1 << level;
        for (int m = 0; m < NP; ++m) {
            if (m & (1 << lv)) continue;
            const int m2 = m | (1 << lv);
            const size_t d = dbase + ((size_t)m << l0);
            const size_t i = d & (half - 1);
            const uint32_t ex = (uint32_t)((2 * kN - ((2 * (size_t)kN * i) >> (level + 1)) % (2 * kN)) % (2 * kN));
            const uint16_t* ev = A + m * kN;
            const uint16_t* od = A + m2 * kN;
            uint16_t* o0 = B + m * kN;
            uint16_t* o1 = B + m2 * kN;
            for (int k = threadIdx.x; k < kN; k += blockDim.x) {
                uint32_t sidx = (uint32_t)k + 2 * kN - ex;
                if (sidx >= 2 * kN) sidx -= 2 * kN;
                uint32_t tv;
                if (sidx < (uint32_t)kN) tv = od[sidx];
                else { const uint32_t v = od[sidx - kN]; tv = v ? kP - v : 0; }
                const uint32_t e = ev[k];
                uint32_t sm = e + tv; if (sm >= kP) sm -= kP;
                uint32_t df = e + kP - tv; if (df >= kP) df -= kP;
                o0[k] = (uint16_t)sm;
                o1[k] = (uint16_t)df;
            }
        }
        __syncthreads();
        uint16_t* tmp = A; A = B; B = tmp;
    }
    for (int m = 0; m < NP; ++m) {
        const size_t d = dbase + ((size_t)m << l0);
        uint16_t* dp = dst + rowoff + d * kN;
        const uint16_t* ap = A + m * kN;
        if (last) {
            for (int k = threadIdx.x; k < kN; k += blockDim.x) dp[k] = (uint16_t)(((uint32_t)ap[k] * d_inv) % kP);
        } else {
            uint4* d4 = reinterpret_cast<uint4*>(dp);
            const uint4* a4 = reinterpret_cast<const uint4*>(ap);
            for (int k = threadIdx.x; k < kN / 8; k += blockDim.x) d4[k] = a4[k];
        }
    }
}

// ------------------------------------------------------------------ a-side
// CTA = 8 adjacent columns of group g; four NTT groups, group gp owns the
// polys (column 2gp+cc, limb l).  For every r: stage the 2048x8 u16 tile
// column-major in shared memory, forward-NTT each column, multiply by the
// CRS poly crs_r and accumulate (all in registers, L4 layout).  The output
// row p of V holds N^-1 * acc_j[N-1-p] for the tile's columns j.
constexpr size_t kASideSmem = 8 * kN * sizeof(uint16_t) + 4 * 2 * kN * sizeof(uint32_t) + 2 * kN * sizeof(uint2);

__global__ void __launch_bounds__(1024, 1) a_side_kernel(const uint16_t* __restrict__ db, size_t rows, size_t cols,
                                                         size_t g, const uint32_t* __restrict__ crs,
                                                         const DevTables* __restrict__ T, uint32_t* __restrict__ V) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint16_t* tile = reinterpret_cast<uint16_t*>(smem);                               // [8][N]
    uint32_t* nbuf = reinterpret_cast<uint32_t*>(smem + 8 * kN * sizeof(uint16_t));  // [4][2][N]
    uint2* tw = reinterpret_cast<uint2*>(nbuf + 4 * 2 * kN);                           // [2][N]
    const int tid = threadIdx.x, gp = tid >> 8;
    const uint32_t t = tid & 255;
    const size_t j0 = (size_t)blockIdx.x * 8;
    for (int i = tid; i < kN; i += 1024) { tw[i] = T->limb[0].fwd[i]; tw[kN + i] = T->limb[1].fwd[i]; }
    uint32_t acc[4][8];
#pragma unroll
    for (int pi = 0; pi < 4; ++pi)
#pragma unroll
        for (int e = 0; e < 8; ++e) acc[pi][e] = 0;
    const size_t n_r = rows / kN;
    for (size_t r = 0; r < n_r; ++r) {
        __syncthreads();
        for (int i = tid; i < kN; i += 1024) {
            const uint4 v = *reinterpret_cast<const uint4*>(db + (r * kN + i) * cols + g * kN + j0);
            tile[0 * kN + i] = (uint16_t)(v.x & 0xFFFF); tile[1 * kN + i] = (uint16_t)(v.x >> 16);
            tile[2 * kN + i] = (uint16_t)(v.y & 0xFFFF); tile[3 * kN + i] = (uint16_t)(v.y >> 16);
            tile[4 * kN + i] = (uint16_t)(v.z & 0xFFFF); tile[5 * kN + i] = (uint16_t)(v.z >> 16);
            tile[6 * kN + i] = (uint16_t)(v.w & 0xFFFF); tile[7 * kN + i] = (uint16_t)(v.w >> 16);
        }
        __syncthreads();
#pragma unroll
        for (int pi = 0; pi < 4; ++pi) {
            const int c = 2 * gp + (pi >> 1), l = pi & 1;
            const LimbTables& L = T->limb[l];
            uint32_t x[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] = tile[c * kN + t + 256 * e];
            ntt_fwd(x, nbuf + gp * 2 * kN, tw + l * kN, L.q, t, 1 + gp);
            uint32_t a[8];
            ld8(crs + (r * 2 + l) * kN + 8 * t, a);
#pragma unroll
            for (int e = 0; e < 8; ++e) acc[pi][e] = add_mod(acc[pi][e], mulmod(x[e], a[e], L), L.q);
        }
    }
    __syncthreads();
    uint32_t* stage = reinterpret_cast<uint32_t*>(smem);  // [N][8] per limb round (64 KB)
    for (int l = 0; l < 2; ++l) {
        const LimbTables& L = T->limb[l];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int c = 2 * gp + cc;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t m = 8 * t + e;
                stage[(kN - 1 - m) * 8 + c] = csub(shoup_mul(acc[cc * 2 + l][e], L.inv_n, L.inv_n_p, L.q), L.q);
            }
        }
        __syncthreads();
        for (int i = tid; i < 2 * kN; i += 1024) {
            const int p = i >> 1, h = i & 1;
            *reinterpret_cast<uint4*>(V + ((size_t)l * kN + p) * kN + j0 + 4 * h) =
                *reinterpret_cast<const uint4*>(stage + p * 8 + 4 * h);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ column NTT
__global__ void __launch_bounds__(1024) col_ntt_kernel(const uint32_t* __restrict__ V,
                                                       const DevTables* __restrict__ T, uint32_t* __restrict__ Tout) {
    extern __shared__ __align__(16) uint32_t nb[];
    const int gp = threadIdx.x >> 8;
    const uint32_t t = threadIdx.x & 255;
    const size_t p = (size_t)blockIdx.x * 4 + gp;
    const int l = blockIdx.y;
    const LimbTables& L = T->limb[l];
    const uint32_t* src = V + ((size_t)l * kN + p) * kN;
    uint32_t x[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) x[e] = src[t + 256 * e];
    ntt_fwd(x, nb + gp * 2 * kN, L.fwd, L.q, t, 1 + gp);
    st8(Tout + ((size_t)l * kN + p) * kN + 8 * t, x);
}

// a_post[k][dir][limb][i] = T[limb][perm_t(i)][i],  t = 5^k or 2N - 5^k.
__global__ void __launch_bounds__(256) embed_gather_kernel(const uint32_t* __restrict__ Tin,
                                                           uint32_t* __restrict__ a_post) {
    const int k = blockIdx.x, dir = blockIdx.y, l = blockIdx.z;
    uint32_t tk = pow5_mod2n(k);
    if (dir) tk = (2 * kN - tk) & (2 * kN - 1);
    const uint32_t* Tl = Tin + (size_t)l * kN * kN;
    uint32_t* o = a_post + (((size_t)k * 2 + dir) * 2 + l) * kN;
    for (int x = threadIdx.x; x < kN; x += 256) {
        const uint32_t pi = perm_from_odd(tk, 2 * brev11(x) + 1);
        o[x] = Tl[(size_t)pi * kN + x];
    }
}

// ------------------------------------------------------------------ CollapseA
// CTA (g, dir): two NTT groups (limb 0, limb 1) walk steps s = 0..1022,
// k = N/2-1-s: INTT the state, exchange coefficients (parity double buffer,
// one CTA barrier per step), decompose, NTT the two digits, write
// D[limb][s][digit], MAC against K5 permuted by 5^(1022-s) (or its
// conjugate) and subtract from a_post[k-1].
constexpr size_t kCollapseASmem = (2 * 2 * kN + 2 * 2 * kN + 2 * kDeff * kN) * sizeof(uint32_t);

__global__ void __launch_bounds__(512) collapse_a_kernel(const uint32_t* __restrict__ a_post, size_t ap_gstride,
                                                         const uint32_t* __restrict__ k5,
                                                         const DevTables* __restrict__ T, uint32_t* __restrict__ dp,
                                                         uint32_t* __restrict__ dm, uint32_t* __restrict__ ends) {
    extern __shared__ __align__(16) uint32_t sm[];
    uint32_t* nbuf = sm;                      // [2][2][N]
    uint32_t* xc = nbuf + 2 * 2 * kN;         // [parity][limb][N]
    uint32_t* sk = xc + 2 * 2 * kN;           // [limb][digit][N]
    const int g = blockIdx.x, dir = blockIdx.y;
    const int l = threadIdx.x >> 8;
    const uint32_t t = threadIdx.x & 255;
    const int bar = 1 + l;
    for (int i = threadIdx.x; i < 2 * kDeff * kN; i += 512) sk[i] = k5[i];
    __syncthreads();
    const LimbTables& L = T->limb[l];
    const uint32_t q = L.q;
    const uint32_t* ap = a_post + (size_t)g * ap_gstride;
    uint32_t* Dout = (dir ? dm : dp) + (size_t)g * (2 * (size_t)kSteps * kDeff * kN);
    uint32_t odd[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) odd[e] = 2 * brev11(8 * t + e) + 1;
    uint32_t st[8];
    ld8(ap + (((size_t)(kHalf - 1) * 2 + dir) * 2 + l) * kN + 8 * t, st);
    uint32_t tks = pow5_mod2n(kSteps - 1);
    const uint32_t* skl0 = sk + (l * kDeff + 0) * kN;
    const uint32_t* skl1 = sk + (l * kDeff + 1) * kN;
    for (int s = 0; s < kSteps; ++s) {
        const int k = kHalf - 1 - s;
        ntt_inv(st, nbuf + l * 2 * kN, L.inv, q, L.inv_n, L.inv_n_p, t, bar);
        uint32_t* xme = xc + ((s & 1) * 2 + l) * kN;
        const uint32_t* xot = xc + ((s & 1) * 2 + (1 - l)) * kN;
#pragma unroll
        for (int e = 0; e < 8; ++e) xme[t + 256 * e] = st[e];
        __syncthreads();
        uint32_t d0[8], d1[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t o = xot[t + 256 * e];
            int64_t s1, s2;
            decomp2(l ? o : st[e], l ? st[e] : o, *T, s1, s2);
            d0[e] = signed_res(s1, q);
            d1[e] = signed_res(s2, q);
        }
        ntt_fwd(d0, nbuf + l * 2 * kN, L.fwd, q, t, bar);
        ntt_fwd(d1, nbuf + l * 2 * kN, L.fwd, q, t, bar);
        st8(Dout + (((size_t)l * kSteps + s) * kDeff + 0) * kN + 8 * t, d0);
        st8(Dout + (((size_t)l * kSteps + s) * kDeff + 1) * kN + 8 * t, d1);
        const uint32_t tt = dir ? ((2 * kN - tks) & (2 * kN - 1)) : tks;
        uint32_t an[8];
        ld8(ap + (((size_t)(k - 1) * 2 + dir) * 2 + l) * kN + 8 * t, an);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t pi = perm_from_odd(tt, odd[e]);
            const uint32_t acc = mod_u64((uint64_t)d0[e] * skl0[pi] + (uint64_t)d1[e] * skl1[pi], L.cr, q);
            st[e] = sub_mod(an[e], acc, q);
        }
        tks = (tks * kInv5) & (2 * kN - 1);
    }
    st8(ends + (((size_t)g * 2 + dir) * 2 + l) * kN + 8 * t, st);
}

// CollapseOne: decompose the conjugate chain's end state -> D_final;
// a = (forward chain's end) - sum_j D_final[j] (.) Kneg1[j].
__global__ void __launch_bounds__(512) collapse_final_kernel(const uint32_t* __restrict__ ends,
                                                             const uint32_t* __restrict__ kn1,
                                                             const DevTables* __restrict__ T,
                                                             uint32_t* __restrict__ df, uint32_t* __restrict__ pre_a) {
    __shared__ __align__(16) uint32_t nbuf[2 * 2 * kN];
    __shared__ __align__(16) uint32_t xc[2 * kN];
    const int g = blockIdx.x;
    const int l = threadIdx.x >> 8;
    const uint32_t t = threadIdx.x & 255;
    const int bar = 1 + l;
    const LimbTables& L = T->limb[l];
    const uint32_t q = L.q;
    uint32_t st[8];
    ld8(ends + (((size_t)g * 2 + 1) * 2 + l) * kN + 8 * t, st);
    ntt_inv(st, nbuf + l * 2 * kN, L.inv, q, L.inv_n, L.inv_n_p, t, bar);
#pragma unroll
    for (int e = 0; e < 8; ++e) xc[l * kN + t + 256 * e] = st[e];
    __syncthreads();
    uint32_t d0[8], d1[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const uint32_t o = xc[(1 - l) * kN + t + 256 * e];
        int64_t s1, s2;
        decomp2(l ? o : st[e], l ? st[e] : o, *T, s1, s2);
        d0[e] = signed_res(s1, q);
        d1[e] = signed_res(s2, q);
    }
    ntt_fwd(d0, nbuf + l * 2 * kN, L.fwd, q, t, bar);
    ntt_fwd(d1, nbuf + l * 2 * kN, L.fwd, q, t, bar);
    st8(df + (((size_t)g * 2 + l) * kDeff + 0) * kN + 8 * t, d0);
    st8(df + (((size_t)g * 2 + l) * kDeff + 1) * kN + 8 * t, d1);
    uint32_t sv[8], k0[8], k1[8], o[8];
    ld8(ends + (((size_t)g * 2 + 0) * 2 + l) * kN + 8 * t, sv);
    ld8(kn1 + ((size_t)l * kDeff + 0) * kN + 8 * t, k0);
    ld8(kn1 + ((size_t)l * kDeff + 1) * kN + 8 * t, k1);
#pragma unroll
    for (int e = 0; e < 8; ++e)
        o[e] = sub_mod(sv[e], mod_u64((uint64_t)d0[e] * k0[e] + (uint64_t)d1[e] * k1[e], L.cr, q), q);
    st8(pre_a + ((size_t)g * 2 + l) * kN + 8 * t, o);
}

}  // namespace

// ==================================================================== wrappers
cudaError_t launch_encode_pass(const uint16_t* src, uint16_t* dst, size_t nrows, size_t cols, size_t d_act,
                               int logd, int l0, int nl, bool first, bool last, uint32_t d_inv, cudaStream_t s) {
    if (nrows == 0) return cudaSuccess;
    if (nl < 1 || nl > 4 || (d_act >> nl) == 0) return cudaErrorInvalidValue;
    const size_t num_cts = (cols / kN) / d_act;
    const size_t smem = (size_t)2 * (1 << nl) * kN * sizeof(uint16_t);
    cudaError_t e = allow_max_smem(encode_pass_kernel);
    if (e) return e;
    dim3 grid((unsigned)nrows, (unsigned)(num_cts * (d_act >> nl)));
    encode_pass_kernel<<<grid, 256, smem, s>>>(src, dst, cols, d_act, logd, l0, nl, first, last, d_inv);
    return cudaGetLastError();
}

cudaError_t launch_a_side(const uint16_t* db, size_t rows, size_t cols, size_t g, const uint32_t* crs,
                          const DevTables* T, uint32_t* V, cudaStream_t s) {
    cudaError_t e = allow_max_smem(a_side_kernel);
    if (e) return e;
    a_side_kernel<<<kN / 8, 1024, kASideSmem, s>>>(db, rows, cols, g, crs, T, V);
    return cudaGetLastError();
}

cudaError_t launch_col_ntt(const uint32_t* V, const DevTables* T, uint32_t* Tout, cudaStream_t s) {
    const size_t smem = 4 * 2 * kN * sizeof(uint32_t);
    cudaError_t e = allow_max_smem(col_ntt_kernel);
    if (e) return e;
    col_ntt_kernel<<<dim3(kN / 4, 2), 1024, smem, s>>>(V, T, Tout);
    return cudaGetLastError();
}

cudaError_t launch_embed_gather(const uint32_t* Tin, uint32_t* a_post, cudaStream_t s) {
    embed_gather_kernel<<<dim3(kHalf, 2, 2), 256, 0, s>>>(Tin, a_post);
    return cudaGetLastError();
}

cudaError_t launch_collapse_a(const uint32_t* a_post, size_t ap_gstride, const uint32_t* k5, const DevTables* T,
                              uint32_t* dp, uint32_t* dm, uint32_t* ends, size_t ngroups, cudaStream_t s) {
    if (ngroups == 0) return cudaSuccess;
    cudaError_t e = allow_max_smem(collapse_a_kernel);
    if (e) return e;
    collapse_a_kernel<<<dim3((unsigned)ngroups, 2), 512, kCollapseASmem, s>>>(a_post, ap_gstride, k5, T, dp, dm, ends);
    return cudaGetLastError();
}

cudaError_t launch_collapse_final(const uint32_t* ends, const uint32_t* kn1, const DevTables* T, uint32_t* df,
                                  uint32_t* pre_a, size_t ngroups, cudaStream_t s) {
    if (ngroups == 0) return cudaSuccess;
    collapse_final_kernel<<<(unsigned)ngroups, 512, 0, s>>>(ends, kn1, T, df, pre_a);
    return cudaGetLastError();
}

}  // namespace ipb
