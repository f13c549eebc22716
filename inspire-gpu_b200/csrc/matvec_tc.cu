// matvec_tc.cu -- exact database x query mat-vec on the tcgen05 tensor cores.
//
//   r_l[q][j] = sum_i db[i][j] * b_{q,l}[i]  mod q_l      (reference src/gpu_online.cu:23-175)
//
// The row-major u16 DB is read, unchanged, as a u8 matrix A'[m'][i] with
// m' = 2j + byte (lo byte at even m', hi byte at odd m'): consecutive m' are
// contiguous, i.e. an MN-major operand.  A query's two limbs are combined
// by CRT into one word B[i] < q0*q1 < 2^53 (B = b_{q,l}[i] mod q_l for both
// limbs), split into 7 bytes: B[n][i] with n = 7q + k holds byte k of query
// q's B[i] (K-major rows built by qplanes_kernel).  One
// tcgen05.mma.kind::i8 chain accumulates D[m'][n] = sum_i A'[m'][i] B[n][i]
// in s32 TMEM.  With K <= 32768 rows per chunk every D entry is
// <= 255*255*32768 < 2^31: exact.  The epilogue forms, per limb,
// sum_k (256^k mod q_l) D[m'][n_k] (< 2^61) in each of the lo and hi byte
// rows and combines them as (lo + 256 (hi mod q_l)) mod q_l: the exact
// sum_i db[i][j] b_{q,l}[i] mod q_l.  All arithmetic stays exact, so the
// result equals the reference's.  Seven planes per query instead of four
// per limb: 12.5 % fewer MMAs and query-plane bytes.
//
// CTA roles (256 threads): warp 0 issues TMA loads (DB tile 256 x 64 rows as
// two 128-byte boxes, query planes N x 64), warp 1 allocates TMEM and one
// thread issues the MMAs, warps 4..7 drain TMEM (tcgen05.ld) and write
// partial sums.  Stages are recycled through mbarriers; every wait is
// bounded and reports a timeout through *err instead of hanging.
//
// Work items (m'-tile, K-chunk) are handed out dynamically: the producer
// thread takes the next item from a per-launch atomic counter (zeroed by the
// launcher) and publishes it to the MMA thread and the epilogue through a
// ring of kRing shared slots; -1 ends the sequence.  SMs that other kernels
// hold when this one starts (the previous batch's Horner, another lane)
// simply take fewer items instead of delaying the whole pass.
#include <cuda.h>

#include "ipb_common.cuh"
#include "host_util.h"
#include "ipb_launch.h"
#include "tc_ptx.cuh"

namespace ipb {

namespace {
using namespace tc;

// DB rows per pipeline stage (bytes of K): 64, so a stage is 16 KB of DB
// plus 64 bytes of every query plane (a SWIZZLE_64B tile), 32 KB at 32
// queries, and six stages fit (three with 128-row stages).  Deeper DB
// prefetch (an L2 prefetch ahead of the ring, or a separate deeper DB ring)
// measured slower: the SMs drift apart and the DB rows lose locality.
constexpr int kKT = 64;
constexpr int kMT = 256;          // m' rows per tile (two M = 128 MMAs)
constexpr int kKChunk = 32768;    // rows per exact s32 accumulation
constexpr int kRing = 8;          // published work items in flight
constexpr int kPlanes = 7;        // CRT byte planes per query
struct TcParams {
    uint32_t* part;        // [q][chunk][limb][ld], first column of the range at part
    size_t part_qstride;
    size_t cols;           // columns in the range
    size_t ld;             // columns per (chunk, limb) row of part
    int nq;                // queries in this pass (<= 32)
    int npad;              // N = 16 ceil(7 nq / 16) (<= 224)
    uint32_t c[2][kPlanes];  // 256^k mod q_l
    int n_mtiles;
    int mt_per_range;      // > 0: the m' tiles cover ranges of this many tiles, range r starting
    int range_stride_m;    // r * range_stride_m m' rows after the first (several column ranges in one
                           // launch); 0: one contiguous range
    int n_kchunks;
    int kchunk_rows;
    int stages;
    int acc_stages;
    uint32_t tmem_cols;
    int* err;
    unsigned* tiles;       // work-item counter, zero at launch
    const DevTables* T;
    int has_qmap;          // output row of pass query q: qmap[q] (else q)
    uint8_t qmap[32];
    int abort_after;       // > 0: the MMA issuer stops after this many items and reports code 99 (a test of
                           // the abort path, IPB_TEST_ABORT_AFTER_ITEMS); 0: off
};

// First m' row (2 x column, relative to the launch's first column) of m'
// tile mt: tiles of one contiguous range, or of several equal ranges
// range_stride_m apart.
__device__ __forceinline__ int mtile_m0(const TcParams& P, int mt) {
    return P.mt_per_range ? (mt / P.mt_per_range) * P.range_stride_m + (mt % P.mt_per_range) * kMT : mt * kMT;
}

__global__ void __launch_bounds__(256, 1) mv_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                                                       const __grid_constant__ CUtensorMap map_b, TcParams P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = P.stages;
    const uint32_t a_bytes = kKT * 128;              // one 128-byte m' box x kKT rows
    const uint32_t b_bytes = (uint32_t)P.npad * kKT;
    const uint32_t stage_bytes = 2 * a_bytes + b_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * stage_bytes);
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = bars + 2 * S + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 4);
    __shared__ volatile int abort_flag;
    __shared__ volatile int item_ring[kRing];
    __shared__ uint64_t ifull[kRing], iempty[kRing];
    __shared__ uint64_t mma_done;  // the MMA issuer's final commit: all its MMAs have completed

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < S; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int a = 0; a < 2; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 128); }
        for (int r = 0; r < kRing; ++r) { mbar_init(&ifull[r], 1); mbar_init(&iempty[r], 1 + 128); }
        mbar_init(&mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(P.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int n_items = P.n_mtiles * P.n_kchunks;
    const int ktiles = P.kchunk_rows / kKT;

    if (warp == 0) {
        // ---------------- TMA producer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            unsigned issued = 0;  // stage loads issued
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                int item = -1;
                if (!abort_flag && mbar_wait_ab(&iempty[r], ((uint32_t)(it / kRing) & 1) ^ 1, P.err, 6, &abort_flag)) {
                    const unsigned t = atomicAdd(P.tiles, 1u);
                    if (t < (unsigned)n_items) item = (int)t;
                } else {
                    abort_flag = 1;
                }
                item_ring[r] = item;
                mbar_arrive(&ifull[r]);
                if (item < 0) break;
                const int mt = item % P.n_mtiles, kc = item / P.n_mtiles;
                const int m0 = mtile_m0(P, mt);
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait_ab(&empty[s], ph ^ 1, P.err, 1, &abort_flag)) { abort_flag = 1; break; }
                    uint8_t* st = smem + (size_t)s * stage_bytes;
                    mbar_expect_tx(&full[s], stage_bytes);
                    const int k0 = kc * P.kchunk_rows + kt * kKT;
                    tma_load_2d(st, &map_a, &full[s], m0, k0);
                    tma_load_2d(st + a_bytes, &map_a, &full[s], m0 + 128, k0);
                    tma_load_2d(st + 2 * a_bytes, &map_b, &full[s], k0, 0);
                    ++issued;
                    if (++s == S) { s = 0; ph ^= 1; }
                }
            }
            // Drain: every issued load has landed in shared memory before the
            // CTA exits, also when the MMA issuer stopped early (a timeout) and
            // never consumed them.  Load n went to stage n % S with phase
            // (n / S) & 1; no later load reuses a stage, so each wait is exact.
            for (unsigned i = 0; i < (unsigned)S && i < issued; ++i) {
                const unsigned n = issued - 1 - i;
                mbar_wait(&full[n % S], (n / S) & 1u, P.err, 2);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = idesc_i8(P.npad);
            int s = 0, as = 0;
            uint32_t ph = 0, aph = 0;
            bool it_mma = false;  // any MMA issued
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                if (!mbar_wait_ab(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 7, &abort_flag)) {
                    abort_flag = 1;
                    break;
                }
                const int item = item_ring[r];
                mbar_arrive(&iempty[r]);
                if (item < 0 || abort_flag) break;
                if (P.abort_after > 0 && it >= P.abort_after) {  // test hook: the designed early stop
                    atomicCAS(P.err, 0, 99);
                    abort_flag = 1;
                    break;
                }
                if (!mbar_wait_ab(&tempty[as], aph ^ 1, P.err, 3, &abort_flag)) { abort_flag = 1; break; }
                tc_fence_after();
                const uint32_t d0 = tmem_base + (uint32_t)(as * 2 * P.npad);
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait_ab(&full[s], ph, P.err, 4, &abort_flag)) { abort_flag = 1; break; }
                    tc_fence_after();
                    const uint8_t* st = smem + (size_t)s * stage_bytes;
#pragma unroll
                    for (int kk = 0; kk < kKT / 32; ++kk) {
                        // A: MN-major, rows of 128 bytes, 8-row swizzle atoms (SBO 1024 B);
                        // K advances 32 rows = 4096 bytes per MMA.
                        const uint64_t a0 = smem_desc(st + kk * 4096, 0, 1024);
                        const uint64_t a1 = smem_desc(st + a_bytes + kk * 4096, 0, 1024);
                        // B: K-major, 64-byte rows (SWIZZLE_64B), 8-row groups 512 B apart; K advances 32 bytes.
                        const uint64_t b = smem_desc_sw64(st + 2 * a_bytes + kk * 32, 512);
                        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                        mma_i8(d0, a0, b, idesc, acc);
                        mma_i8(d0 + (uint32_t)P.npad, a1, b, idesc, acc);
                    }
                    it_mma = true;
                    mma_commit(&empty[s]);
                    if (++s == S) { s = 0; ph ^= 1; }
                }
                mma_commit(&tfull[as]);
                if (++as == P.acc_stages) { as = 0; aph ^= 1; }
            }
            // Every MMA this thread issued has completed (also after an early
            // stop) before TMEM is deallocated and shared memory released.
            if (it_mma) {
                mma_commit(&mma_done);
                mbar_wait(&mma_done, 0, P.err, 9);
            }
        }
    } else if (warp >= 4) {
        // ---------------- epilogue: TMEM -> u64 dot products -> mod q
        const int wq = warp & 3;
        const uint32_t lane_base = (uint32_t)(wq * 32) << 16;
        int as = 0;
        uint32_t aph = 0;
        const uint64_t cr0 = P.T->limb[0].cr, cr1 = P.T->limb[1].cr;
        for (int it = 0;; ++it) {
            const int r = it % kRing;
            if (!mbar_wait_ab(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 8, &abort_flag)) { abort_flag = 1; break; }
            const int item = item_ring[r];
            mbar_arrive(&iempty[r]);
            if (item < 0) break;
            if (!mbar_wait_ab(&tfull[as], aph, P.err, 5, &abort_flag)) { abort_flag = 1; break; }
            tc_fence_after();
            const int mt = item % P.n_mtiles, kc = item / P.n_mtiles;
            const int m0 = mtile_m0(P, mt);
            for (int mb = 0; mb < 2; ++mb) {
                const size_t j = ((size_t)m0 + mb * 128 + wq * 32 + lane) >> 1;
                for (int q0 = 0; q0 < P.nq; q0 += 8) {
                    // queries q0..q0+7: columns 7 q0 .. 7 q0 + 55, seven 8-column
                    // loads (those at or past N are not loaded: they hold no query)
                    uint32_t t[kPlanes][8];
#pragma unroll
                    for (int c = 0; c < kPlanes; ++c) {
                        const int col = kPlanes * q0 + 8 * c;
                        if (col < P.npad) {
                            tmem_ld8_issue(tmem_base + lane_base + (uint32_t)(as * 2 * P.npad + mb * P.npad + col),
                                           t[c]);
                        } else {
#pragma unroll
                            for (int e = 0; e < 8; ++e) t[c][e] = 0;
                        }
                    }
                    uint32_t v[kPlanes * 8];
#pragma unroll
                    for (int c = 0; c < kPlanes; ++c) {
                        tmem_wait8(t[c]);  // one wait for all seven loads; the others are no-ops
#pragma unroll
                        for (int e = 0; e < 8; ++e) v[8 * c + e] = t[c][e];
                    }
                    // per limb sum_k (256^k mod q) D[row][7 q + k] (< 2^61); lane
                    // 2j+1 holds the hi DB byte's sums, lane 2j the lo byte's:
                    // result = (lo + 256 (hi mod q)) mod q
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        uint64_t a0 = 0, a1 = 0;
#pragma unroll
                        for (int k = 0; k < kPlanes; ++k) {
                            a0 += (uint64_t)P.c[0][k] * v[kPlanes * e + k];
                            a1 += (uint64_t)P.c[1][k] * v[kPlanes * e + k];
                        }
                        const uint32_t h0 = (lane & 1) ? mod_u64(a0, cr0, kQ0) : 0u;
                        const uint32_t h1 = (lane & 1) ? mod_u64(a1, cr1, kQ1) : 0u;
                        const uint32_t p0 = __shfl_down_sync(0xffffffffu, h0, 1);
                        const uint32_t p1 = __shfl_down_sync(0xffffffffu, h1, 1);
                        if ((lane & 1) == 0 && q0 + e < P.nq) {
                            const int qo = P.has_qmap ? P.qmap[q0 + e] : q0 + e;
                            uint32_t* dst = P.part + (size_t)qo * P.part_qstride + (size_t)kc * 2 * P.ld + j;
                            dst[0] = mod_u64(a0 + ((uint64_t)p0 << 8), cr0, kQ0);
                            dst[P.ld] = mod_u64(a1 + ((uint64_t)p1 << 8), cr1, kQ1);
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[as]);
            if (++as == P.acc_stages) { as = 0; aph ^= 1; }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(P.tmem_cols));
    }
}

// CRT byte planes of the queries: planes[7q + k][rows] = byte k of
// B[i] = CRT(b_0[i] mod q0, b_1[i] mod q1) < q0 q1
// (Garner: b_1 + q1 ((b_0 - b_1) q1^-1 mod q0)).
__global__ void __launch_bounds__(256) qplanes_kernel(const uint64_t* __restrict__ qraw, size_t qstride, size_t rows,
                                                      const DevTables* __restrict__ T,
                                                      uint8_t* __restrict__ planes) {
    const int q = blockIdx.y;
    const size_t i4 = ((size_t)blockIdx.x * 256 + threadIdx.x) * 4;
    if (i4 >= rows) return;
    const uint64_t* src = qraw + (size_t)q * qstride;
    uint64_t B[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const uint32_t v0 = mod_u64(src[i4 + c], T->limb[0].cr, kQ0);
        const uint32_t v1 = mod_u64(src[rows + i4 + c], T->limb[1].cr, kQ1);
        const uint32_t v1r = v1 >= kQ0 ? v1 - kQ0 : v1;
        const uint32_t diff = v0 >= v1r ? v0 - v1r : v0 + kQ0 - v1r;
        const uint32_t h = mod_u64((uint64_t)diff * T->crt_c[0], T->limb[0].cr, kQ0);
        B[c] = (uint64_t)v1 + (uint64_t)kQ1 * h;
    }
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) {
        uint32_t packed = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) packed |= (uint32_t)((B[c] >> (8 * k)) & 0xFFu) << (8 * c);
        *reinterpret_cast<uint32_t*>(planes + ((size_t)kPlanes * q + k) * rows + i4) = packed;
    }
}

// out[q][l][c] = sum over K-chunks of part[q][chunk][l][c]  mod q_l.
__global__ void __launch_bounds__(256) mv_chunk_reduce_kernel(const uint32_t* __restrict__ part, size_t part_qstride,
                                                              int chunks, size_t cols, const DevTables* __restrict__ T,
                                                              uint32_t* __restrict__ out, size_t out_qstride) {
    const int q = blockIdx.y;
    const size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x;
    if (idx >= 2 * cols) return;
    const int l = (int)(idx / cols);
    const size_t c = idx % cols;
    uint64_t s = 0;
    for (int ch = 0; ch < chunks; ++ch) s += part[(size_t)q * part_qstride + ((size_t)ch * 2 + l) * cols + c];
    out[(size_t)q * out_qstride + (size_t)l * cols + c] = mod_u64(s, T->limb[l].cr, T->limb[l].q);
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

}  // namespace

size_t mv_tc_planes_bytes(size_t rows, int max_queries) { return (size_t)kPlanes * max_queries * rows + 16 * rows; }
size_t mv_tc_planes_offset(size_t first_query, size_t rows) { return (size_t)kPlanes * first_query * rows; }

cudaError_t launch_mv_chunk_reduce(const uint32_t* part, size_t part_qstride, int chunks, size_t cols,
                                   const DevTables* T, uint32_t* out, size_t out_qstride, int nq, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    mv_chunk_reduce_kernel<<<dim3((unsigned)((2 * cols + 255) / 256), nq), 256, 0, s>>>(part, part_qstride, chunks,
                                                                                         cols, T, out, out_qstride);
    return cudaGetLastError();
}

cudaError_t launch_qplanes(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T, uint8_t* planes,
                           int nq, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (rows % 1024) return cudaErrorInvalidValue;
    qplanes_kernel<<<dim3((unsigned)(rows / 1024), nq), 256, 0, s>>>(qraw, qstride, rows, T, planes);
    return cudaGetLastError();
}

// nq <= 32 queries whose planes start at `planes` (rows bytes per plane row).
int matvec_tc_item_cols() { return kMT / 2; }

int matvec_tc_kchunk_rows(size_t rows, size_t cols, int num_sms) {
    // Rows per exact s32 accumulation: at most 32768, halved while the
    // (m'-tile, chunk) work items would leave SMs idle.
    size_t kc = rows < (size_t)kKChunk ? rows : (size_t)kKChunk;
    const size_t mtiles = (2 * cols) / kMT;
    while (mtiles * (rows / kc) < (size_t)(2 * num_sms) && kc > 1024 && kc % 2 == 0) kc /= 2;
    return (int)kc;
}

cudaError_t launch_matvec_tc(const uint16_t* db, size_t rows, size_t cols, const uint8_t* planes, int nq,
                             const DevTables* T, uint32_t* part, size_t part_qstride, int* err, unsigned* tiles,
                             int num_sms, int kchunk_rows, cudaStream_t s) {
    return launch_matvec_tc_range(db, rows, cols, 0, cols, planes, nq, T, part, part_qstride, nullptr, err, tiles,
                                  num_sms, kchunk_rows, s);
}

cudaError_t launch_matvec_tc_range(const uint16_t* db, size_t rows, size_t ld, size_t c0, size_t c1,
                                   const uint8_t* planes, int nq, const DevTables* T, uint32_t* part,
                                   size_t part_qstride, const uint8_t* qmap, int* err, unsigned* tiles, int num_sms,
                                   int kchunk_rows, cudaStream_t s) {
    if (c1 <= c0) return nq <= 0 ? cudaSuccess : cudaErrorInvalidValue;
    return launch_matvec_tc_ranges(db, rows, ld, c0, c1 - c0, 1, 0, planes, nq, T, part, part_qstride, qmap, err,
                                   tiles, num_sms, kchunk_rows, s);
}

cudaError_t launch_matvec_tc_ranges(const uint16_t* db, size_t rows, size_t ld, size_t c0, size_t cols_per_range,
                                    int n_ranges, size_t range_stride, const uint8_t* planes, int nq,
                                    const DevTables* T, uint32_t* part, size_t part_qstride, const uint8_t* qmap,
                                    int* err, unsigned* tiles, int num_sms, int kchunk_rows, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (n_ranges < 1 || cols_per_range == 0 || cols_per_range % 128 || c0 % 128 ||
        (n_ranges > 1 && (range_stride < cols_per_range || range_stride % 128)))
        return cudaErrorInvalidValue;
    // the launch's columns span [c0, c0 + cols): the ranges and the gaps between them
    const size_t cols = (size_t)(n_ranges - 1) * range_stride + cols_per_range;
    if (c0 + cols > ld) return cudaErrorInvalidValue;
    db += c0;
    part += c0;
    if (nq > 32 || rows % kKT || cols % 128 || !tiles) return cudaErrorInvalidValue;
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const int npad = ((kPlanes * nq + 15) / 16) * 16;
    const int kchunk = kchunk_rows;
    if (kchunk <= 0 || kchunk > kKChunk || kchunk % kKT || rows % (size_t)kchunk) return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    {
        cuuint64_t dims[2] = {(cuuint64_t)(2 * cols), (cuuint64_t)rows};
        cuuint64_t strides[1] = {(cuuint64_t)(2 * ld)};
        cuuint32_t box[2] = {128, (cuuint32_t)kKT};
        cuuint32_t es[2] = {1, 1};
        if (enc(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)db, dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    {
        cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)npad};
        cuuint64_t strides[1] = {(cuuint64_t)rows};
        cuuint32_t box[2] = {(cuuint32_t)kKT, (cuuint32_t)npad};
        cuuint32_t es[2] = {1, 1};
        if (enc(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)planes, dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    TcParams P{};
    P.part = part;
    P.part_qstride = part_qstride;
    P.cols = cols;
    P.ld = ld;
    P.has_qmap = qmap != nullptr;
    if (qmap)
        for (int q = 0; q < nq; ++q) P.qmap[q] = qmap[q];
    P.nq = nq;
    P.npad = npad;
    P.abort_after = test_abort_after_items();
    {
        const uint32_t qs[2] = {kQ0, kQ1};
        for (int l = 0; l < 2; ++l) {
            uint64_t c = 1;
            for (int k = 0; k < kPlanes; ++k, c = c * 256 % qs[l]) P.c[l][k] = (uint32_t)c;
        }
    }
    P.mt_per_range = n_ranges > 1 ? (int)((2 * cols_per_range) / kMT) : 0;
    P.range_stride_m = n_ranges > 1 ? (int)(2 * range_stride) : 0;
    P.n_mtiles = n_ranges > 1 ? n_ranges * P.mt_per_range : (int)((2 * cols) / kMT);
    P.kchunk_rows = kchunk;
    P.n_kchunks = (int)(rows / kchunk);
    P.acc_stages = (4 * npad <= 512) ? 2 : 1;
    uint32_t need = (uint32_t)(P.acc_stages * 2 * npad);
    uint32_t tc = 32;
    while (tc < need) tc <<= 1;
    P.tmem_cols = tc;
    P.err = err;
    P.tiles = tiles;
    P.T = T;
    const size_t stage_bytes = 2 * (size_t)kKT * 128 + (size_t)npad * kKT;
    const size_t budget = 200 * 1024;
    P.stages = (int)std::min<size_t>(8, budget / stage_bytes);
    if (P.stages < 2) return cudaErrorInvalidValue;
    const size_t smem = 1024 + (size_t)P.stages * stage_bytes + (2 * P.stages + 4) * 8 + 16;
    cudaError_t e = allow_max_smem(mv_tc_kernel);
    if (e) return e;
    const int items = P.n_mtiles * P.n_kchunks;
    const int grid = std::min(items, std::max(1, num_sms));
    if ((e = cudaMemsetAsync(tiles, 0, sizeof(unsigned), s))) return e;
    mv_tc_kernel<<<grid, 256, smem, s>>>(ma, mb, P);
    return cudaGetLastError();
}

}  // namespace ipb

// Target of the device code this library carries, read back from the loaded
// module (cudaFuncGetAttributes on the tensor-core mat-vec kernel):
// binaryVersion is 100 for sm_100a cubins.  No counterpart in the reference.
extern "C" int ipir_b200_kernel_binary_version(int* out) {
    if (!out) return 1;
    cudaFuncAttributes a{};
    cudaError_t e = cudaFuncGetAttributes(&a, ipb::mv_tc_kernel);
    if (e != cudaSuccess) {
        ipb::set_last_error(cudaGetErrorString(e));
        return 4;
    }
    *out = a.binaryVersion;
    return 0;
}


