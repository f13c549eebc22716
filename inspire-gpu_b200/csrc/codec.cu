// codec.cu -- the wire formats of the reference's client library, run on the
// server's GPU next to the answer pipeline: the 53-bit packed query
// (unpacked here), the 53-bit packed response and the modulus-switched
// compressed response (src/capi_client.cpp:156-385, src/crypto.cpp:285-313).
//
// Packed (lossless): the two 27-bit residues of a coefficient are combined
// by CRT (Garner) into one value below q0*q1 < 2^53 and written MSB first at
// 53 bits per value.  Query values: the R LWE coefficients, then the
// 6 * d_eff key / RGSW polynomials coefficient by coefficient; response
// values: the 2 * num_cts polynomials (a then b of each ciphertext).
//
// Compressed (the reference's modulus switching): per ciphertext the NTT-form
// response is taken to coefficients (inverse NTT), each coefficient lifted to
// [0, Q), Q = q0*q1, and rounded to q' = 2^28 (mask a) or 2^20 (body b) as
// floor((v * q' + floor(Q / 2)) / Q) mod q'; then N x 28 bits of a and
// N x 20 bits of b, MSB first (12288 bytes per ciphertext).
//
// Every kernel writes whole output bytes per thread: 8 values x 53 bits =
// 53 bytes, 2 x 28 bits = 7 bytes, 2 x 20 bits = 5 bytes.
#include <cstdint>

#include "host_util.h"
#include "ipb_common.cuh"
#include "ipb_launch.h"

namespace ipb {

namespace {
constexpr int kWireBits = 53;
constexpr uint64_t kQFull64 = (uint64_t)kQ0 * kQ1;

// Garner: v1 + q1 * ((v0 - v1) * q1^-1 mod q0), for canonical v0 < q0, v1 < q1.
__device__ __forceinline__ uint64_t crt_garner(uint32_t v0, uint32_t v1, const DevTables& T) {
    const uint32_t v1r = v1 >= kQ0 ? v1 - kQ0 : v1;
    const uint32_t diff = v0 >= v1r ? v0 - v1r : v0 + kQ0 - v1r;
    const uint32_t h = mod_u64((uint64_t)diff * T.crt_c[0], T.limb[0].cr, kQ0);
    return (uint64_t)v1 + (uint64_t)kQ1 * h;
}

// Query: packed bytes [q][bytes] -> flat u64 [q][2R + 6 d_eff 2 N].
__global__ void __launch_bounds__(256) query_unpack_kernel(const uint8_t* __restrict__ in, size_t in_stride,
                                                           size_t in_bytes, uint64_t* __restrict__ out,
                                                           size_t out_stride, size_t R,
                                                           const DevTables* __restrict__ T) {
    const size_t nv = R + (size_t)6 * kDeff * kN;
    const uint8_t* src = in + (size_t)blockIdx.y * in_stride;
    uint64_t* dst = out + (size_t)blockIdx.y * out_stride;
    for (size_t v = (size_t)blockIdx.x * 256 + threadIdx.x; v < nv; v += (size_t)gridDim.x * 256) {
        const size_t bit = v * kWireBits;
        const size_t b0 = bit >> 3;
        const int sh = (int)(bit & 7);
        uint64_t w = 0;  // the 8 bytes from b0, big-endian; bytes past the stream read as 0
#pragma unroll
        for (int k = 0; k < 8; ++k) w = (w << 8) | (b0 + k < in_bytes ? src[b0 + k] : 0u);
        const uint64_t val = (w >> (64 - kWireBits - sh)) & ((1ull << kWireBits) - 1);
        const uint32_t r0 = mod_u64(val, T->limb[0].cr, kQ0), r1 = mod_u64(val, T->limb[1].cr, kQ1);
        if (v < R) {
            dst[v] = r0;
            dst[R + v] = r1;
        } else {
            const size_t k = v - R, poly = k / kN, i = k % kN;
            dst[2 * R + poly * 2 * kN + i] = r0;
            dst[2 * R + poly * 2 * kN + kN + i] = r1;
        }
    }
}

// Response: flat u64 [q][polys][limb][N] (canonical residues) -> packed bytes.
__global__ void __launch_bounds__(256) response_pack_kernel(const uint64_t* __restrict__ flat, size_t flat_stride,
                                                            size_t polys, uint8_t* __restrict__ out,
                                                            size_t out_stride, const DevTables* __restrict__ T) {
    const size_t groups = polys * kN / 8;
    const uint64_t* src = flat + (size_t)blockIdx.y * flat_stride;
    uint8_t* dst = out + (size_t)blockIdx.y * out_stride;
    for (size_t g = (size_t)blockIdx.x * 256 + threadIdx.x; g < groups; g += (size_t)gridDim.x * 256) {
        uint8_t* o = dst + g * kWireBits;  // 8 values x 53 bits = 53 bytes
        uint64_t acc = 0;
        int nbits = 0;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const size_t v = g * 8 + e, j = v / kN, i = v % kN;
            const uint64_t val = crt_garner((uint32_t)src[j * 2 * kN + i], (uint32_t)src[j * 2 * kN + kN + i], *T);
            acc = (acc << kWireBits) | val;  // acc holds < 8 bits before the shift
            nbits += kWireBits;
            while (nbits >= 8) {
                nbits -= 8;
                *o++ = (uint8_t)(acc >> nbits);
            }
            acc &= (1ull << nbits) - 1;
        }
    }
}

// u64 response -> u32 copy (canonical residues) for the in-place inverse NTT.
__global__ void __launch_bounds__(256) narrow_kernel(const uint64_t* __restrict__ in, uint32_t* __restrict__ out,
                                                    size_t n) {
    for (size_t k = (size_t)blockIdx.x * 256 + threadIdx.x; k < n; k += (size_t)gridDim.x * 256)
        out[k] = (uint32_t)in[k];
}

__device__ __forceinline__ uint32_t mod_switch(uint32_t c0, uint32_t c1, const DevTables& T, int bits) {
    // lift (c0 mod q0, c1 mod q1) to [0, Q), then floor((v 2^bits + floor(Q/2)) / Q) mod 2^bits
    const uint64_t a0 = mod_u64((uint64_t)c0 * T.crt_c[0], T.limb[0].cr, kQ0);
    const uint64_t a1 = mod_u64((uint64_t)c1 * T.crt_c[1], T.limb[1].cr, kQ1);
    uint64_t v = a0 * kQ1 + a1 * kQ0;  // < 2Q
    if (v >= kQFull64) v -= kQFull64;
    const unsigned __int128 num = ((unsigned __int128)v << bits) + (kQFull64 >> 1);
    return (uint32_t)((uint64_t)(num / kQFull64) & ((1ull << bits) - 1));
}

// Coefficient-form u32 [q][ct][a|b][limb][N] -> compressed bytes [q][ct][12288].
__global__ void __launch_bounds__(256) response_compress_kernel(const uint32_t* __restrict__ coef, size_t coef_stride,
                                                                size_t num_cts, uint8_t* __restrict__ out,
                                                                size_t out_stride, const DevTables* __restrict__ T) {
    // per ciphertext: 1024 mask pairs (7 bytes each) then 1024 body pairs (5 bytes each)
    const size_t units = num_cts * kN;  // kN / 2 pairs of each kind per ciphertext
    const uint32_t* src = coef + (size_t)blockIdx.y * coef_stride;
    uint8_t* dst = out + (size_t)blockIdx.y * out_stride;
    for (size_t u = (size_t)blockIdx.x * 256 + threadIdx.x; u < units; u += (size_t)gridDim.x * 256) {
        const size_t ct = u / kN, w = u % kN;
        const bool body = w >= kN / 2;
        const size_t pair = body ? w - kN / 2 : w;
        const int bits = body ? 20 : 28;
        const uint32_t* poly = src + (ct * 2 + (body ? 1 : 0)) * 2 * kN;  // [limb][N] of a or b
        uint64_t acc = 0;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const size_t i = 2 * pair + e;
            acc = (acc << bits) | mod_switch(poly[i], poly[kN + i], *T, bits);
        }
        uint8_t* o = dst + ct * 12288 + (body ? (size_t)kN * 28 / 8 + pair * 5 : pair * 7);
        const int nbytes = body ? 5 : 7;
        for (int k = 0; k < nbytes; ++k) o[k] = (uint8_t)(acc >> (8 * (nbytes - 1 - k)));
    }
}

unsigned grid_for(size_t n) {
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 4096 ? (b ? b : 1) : 4096);
}
}  // namespace

size_t wire_query_bytes(size_t rows) { return ((rows + (size_t)6 * kDeff * kN) * kWireBits + 7) / 8; }
size_t wire_response_bytes(size_t num_cts) { return (num_cts * 2 * kN * kWireBits + 7) / 8; }
size_t wire_compressed_bytes(size_t num_cts) { return num_cts * 12288; }

cudaError_t launch_query_unpack(const uint8_t* in, size_t in_stride, size_t rows, uint64_t* out, size_t out_stride,
                                int nq, const DevTables* T, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    const size_t nv = rows + (size_t)6 * kDeff * kN;
    query_unpack_kernel<<<dim3(grid_for(nv), nq), 256, 0, s>>>(in, in_stride, wire_query_bytes(rows), out, out_stride,
                                                              rows, T);
    return cudaGetLastError();
}

cudaError_t launch_response_pack(const uint64_t* flat, size_t flat_stride, size_t num_cts, uint8_t* out,
                                 size_t out_stride, int nq, const DevTables* T, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    response_pack_kernel<<<dim3(grid_for(num_cts * 2 * kN / 8), nq), 256, 0, s>>>(flat, flat_stride, num_cts * 2,
                                                                                  out, out_stride, T);
    return cudaGetLastError();
}

cudaError_t launch_response_compress(const uint64_t* flat, size_t flat_stride, size_t num_cts, uint32_t* tmp,
                                     uint8_t* out, size_t out_stride, int nq, const DevTables* T, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    const size_t per_q = num_cts * 4 * kN;  // u32 coefficients per query in tmp
    for (int q = 0; q < nq; ++q) {
        narrow_kernel<<<grid_for(per_q), 256, 0, s>>>(flat + (size_t)q * flat_stride, tmp + (size_t)q * per_q, per_q);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
    }
    // poly index (q * num_cts + ct) * 4 + ab * 2 + limb: limb = index & 1
    cudaError_t e = launch_ntt_batch(tmp, (size_t)nq * num_cts * 4, 1, true, T, s);
    if (e) return e;
    response_compress_kernel<<<dim3(grid_for(num_cts * kN), nq), 256, 0, s>>>(tmp, per_q, num_cts, out, out_stride,
                                                                               T);
    return cudaGetLastError();
}

}  // namespace ipb
