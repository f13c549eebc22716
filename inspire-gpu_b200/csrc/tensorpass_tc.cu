// tensorpass_tc.cu -- the online tensor pass (InspiRINGOnline) as int8
// tcgen05 GEMMs.
//
// For group g, limb l and NTT slot i the reference subtracts
//   T_g[l][i] = sum_{dir, s, j} D_g[dir][l][s][j][i] * K5[l][j][perm_{t(dir,s)}(i)]
// (src/gpu_online.cu:593-714, permutations of src/gpu_protocol.cu:169-215),
// re-reading and re-permuting the query key for every group.  Index the sum
// by u = (dir*1023 + s)*2 + j < 4092 (padded to 4096).  The permuted key
//   Gq[l][i][u] = K5_q[l][j][perm_{t(dir,s)}(i)]
// does not depend on the group, so per (l, i) the pass over all groups and
// all queries of a batch is one GEMM
//   T[g][q] = sum_u D[g][u] * Gq[u],   M = groups, N = queries, K = 4096.
// Both operands are < 2^27: split each into four bytes, put D's planes in M
// (row g*4 + a) and Gq's planes in N (column q*4 + b); tcgen05.mma.kind::i8
// accumulates sum_u over bytes exactly in s32 (255^2 * 4096 < 2^31), and the
// epilogue forms sum_{a,b} (256^(a+b) mod q_l) * P[g*4+a][q*4+b] < 2^59 and
// reduces mod q_l.  Exact, so equal to the reference.
//
// Layouts (u8): Dt[l][i][g*4 + a][u] (built once at preprocess by
// dt_transpose_kernel), Gt[l][i][q*4 + b][u] with 4 nq rows per slot, no
// padding (built per pass by gen_g_kernel).  Output tp_out[l][i][q][g]
// (u32, reduced).
//
// The GEMM kernel is persistent with dynamic work items: the producer takes
// the next item from a per-launch atomic counter and publishes it to the MMA
// thread and the epilogue through a ring of shared slots (-1 ends it), so
// SMs held by other kernels at launch take fewer items.
#include <cuda.h>

#include <algorithm>

#include "ipb_common.cuh"
#include "host_util.h"
#include "ipb_launch.h"
#include "tc_ptx.cuh"

namespace ipb {

namespace {
using namespace tc;

constexpr int kUPad = 4096;       // u range, 4092 used
constexpr int kRing = 8;          // published work items in flight
constexpr int kUsed = 2 * 2 * kSteps;

__device__ __forceinline__ uint32_t pow5_mod2n(uint32_t e) {
    uint32_t r = 1, b = 5;
    while (e) {
        if (e & 1) r = (r * b) & (2 * kN - 1);
        b = (b * b) & (2 * kN - 1);
        e >>= 1;
    }
    return r;
}

// ------------------------------------------------------------------ D re-layout
// Source: one wave of groups in the reference layout [l][s][j][N] (u32) for
// each direction; destination Dt rows g*4 + a.  Tile 32 u x 32 slots.
__global__ void __launch_bounds__(256) dt_transpose_kernel(const uint32_t* __restrict__ dp,
                                                           const uint32_t* __restrict__ dm, size_t g0, size_t G,
                                                           uint8_t* __restrict__ Dt) {
    __shared__ uint32_t tile[32][33];
    const int ut = blockIdx.x, it = blockIdx.y;
    const int gw = blockIdx.z >> 1, l = blockIdx.z & 1;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const size_t gstride = (size_t)2 * kSteps * kDeff * kN;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty + 8 * k;
        const int u = ut * 32 + r;
        uint32_t v = 0;
        if (u < kUsed) {
            const int w = u >> 1, j = u & 1;
            const int dir = w >= kSteps;
            const int s = w - dir * kSteps;
            v = (dir ? dm : dp)[(size_t)gw * gstride + ((size_t)(l * kSteps + s) * kDeff + j) * kN + it * 32 + tx];
        }
        tile[r][tx] = v;
    }
    __syncthreads();
    const size_t g = g0 + gw;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int op = threadIdx.x + 256 * k;
        const int il = op >> 5, rem = op & 31;
        const int a = rem >> 3, c = rem & 7;
        uint32_t word = 0;
#pragma unroll
        for (int m = 0; m < 4; ++m) word |= ((tile[4 * c + m][il] >> (8 * a)) & 0xFFu) << (8 * m);
        const size_t row = ((size_t)(l * kN + it * 32 + il)) * 4 * G + g * 4 + a;
        *reinterpret_cast<uint32_t*>(Dt + row * kUPad + ut * 32 + 4 * c) = word;
    }
}

// Inverse of the re-layout for one group (precomp export): [l][s][j][N] u32.
__global__ void __launch_bounds__(256) dt_export_kernel(const uint8_t* __restrict__ Dt, size_t g, size_t G,
                                                        uint32_t* __restrict__ dp, uint32_t* __restrict__ dm) {
    const size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x;  // over l, i, u
    if (idx >= (size_t)2 * kN * kUsed) return;
    const int u = (int)(idx % kUsed);
    const size_t li = idx / kUsed;
    const int l = (int)(li / kN), i = (int)(li % kN);
    const uint8_t* src = Dt + (li * 4 * G + g * 4) * kUPad + u;
    const uint32_t v = (uint32_t)src[0] | ((uint32_t)src[kUPad] << 8) | ((uint32_t)src[2 * kUPad] << 16) |
                       ((uint32_t)src[3 * kUPad] << 24);
    const int w = u >> 1, j = u & 1;
    const int dir = w >= kSteps;
    const int s = w - dir * kSteps;
    (dir ? dm : dp)[((size_t)(l * kSteps + s) * kDeff + j) * kN + i] = v;
}

// ------------------------------------------------------------------ permuted keys
// Gt[l][i][q*4 + b][u] = byte b of K5_q[l][j][perm_t(i)], t = 5^(1022-s) or
// 2N - 5^(1022-s), rq = 4 nq rows per slot.  One CTA per (8 slots, query,
// limb); the query's key for the limb sits in shared memory.
__global__ void __launch_bounds__(256) gen_g_kernel(const uint32_t* __restrict__ keys, size_t key_qstride,
                                                    uint8_t* __restrict__ Gt, int rq) {
    __shared__ uint32_t k5[2][kN];
    __shared__ uint32_t tpow[kSteps];
    const int ib = blockIdx.x, q = blockIdx.y, l = blockIdx.z;
    const uint32_t* kp = keys + (size_t)q * key_qstride + (size_t)(l * kDeff) * kN;  // key 0 = ksk5, [j][N]
    for (int t = threadIdx.x; t < 2 * kN; t += 256) k5[t / kN][t % kN] = kp[t];
    for (int s = threadIdx.x; s < kSteps; s += 256) tpow[s] = pow5_mod2n(kHalf - 2 - s);
    __syncthreads();
    for (int ii = 0; ii < 8; ++ii) {
        const int i = ib * 8 + ii;
        const uint32_t odd = 2 * brev11(i) + 1;
        uint8_t* base = Gt + ((size_t)(l * kN + i) * rq + q * 4) * kUPad;
        for (int u4 = threadIdx.x; u4 < kUPad / 4; u4 += 256) {
            uint32_t v[4];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int w = 2 * u4 + h;
                if (w < 2 * kSteps) {
                    const int dir = w >= kSteps;
                    const int s = w - dir * kSteps;
                    uint32_t t = tpow[s];
                    if (dir) t = (2 * kN - t) & (2 * kN - 1);
                    const uint32_t p = perm_from_odd(t, odd);
                    v[2 * h] = k5[0][p];
                    v[2 * h + 1] = k5[1][p];
                } else {
                    v[2 * h] = v[2 * h + 1] = 0;
                }
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const uint32_t word = ((v[0] >> (8 * b)) & 0xFFu) | (((v[1] >> (8 * b)) & 0xFFu) << 8) |
                                      (((v[2] >> (8 * b)) & 0xFFu) << 16) | (((v[3] >> (8 * b)) & 0xFFu) << 24);
                *reinterpret_cast<uint32_t*>(base + (size_t)b * kUPad + 4 * u4) = word;
            }
        }
    }
}

// ------------------------------------------------------------------ GEMM
struct TpParams {
    uint32_t* out;         // tp_out[l][i][q][g]
    int nq_total;          // queries in the batch (out stride)
    int q0;                // first query of this pass
    int nq;                // queries in this pass
    int rq;                // key rows per slot in Gt (4 nq)
    int nb;                // N = key rows per item, roundup16(spi * rq)
    int G;                 // groups
    int mti;               // M tiles (128 rows) per item (4G >= 128)
    int n_mg;              // M-tile groups per (l, i)
    int spi;               // slots per item (4G < 128: several slots share one 128-row A tile)
    int rows_box;          // rows per A box
    int stages;
    int acc_stages;
    uint32_t tmem_cols;
    int* err;
    unsigned* tiles;       // work-item counter, zero at launch
    uint32_t c[2][7];      // 256^k mod q_l
    uint64_t cr[2];
    uint32_t q[2];
};

__global__ void __launch_bounds__(256, 1) tp_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                                                       const __grid_constant__ CUtensorMap map_b, TpParams P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = P.stages;
    const uint32_t a_tile = 128 * 128;
    const uint32_t a_region = (uint32_t)P.mti * a_tile;
    const uint32_t b_bytes = (uint32_t)P.nb * 128;
    const uint32_t stage_bytes = a_region + b_bytes;
    const uint32_t tx_bytes = (uint32_t)P.mti * P.rows_box * 128 + b_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * stage_bytes);
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = bars + 2 * S + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 4);
    __shared__ volatile int abort_flag;
    __shared__ volatile int item_ring[kRing];
    __shared__ uint64_t ifull[kRing], iempty[kRing];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < S; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int a = 0; a < 2; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 128); }
        for (int r = 0; r < kRing; ++r) { mbar_init(&ifull[r], 1); mbar_init(&iempty[r], 1 + 128); }
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
    const int n_items = (2 * kN / P.spi) * P.n_mg;
    constexpr int ktiles = kUPad / 128;
    const int acc_cols = P.mti * P.nb;
    const int slot_rows = 4 * P.G;  // A rows of one slot

    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                int item = -1;
                if (!abort_flag && mbar_wait(&iempty[r], ((uint32_t)(it / kRing) & 1) ^ 1, P.err, 16)) {
                    const unsigned t = atomicAdd(P.tiles, 1u);
                    if (t < (unsigned)n_items) item = (int)t;
                } else {
                    abort_flag = 1;
                }
                item_ring[r] = item;
                mbar_arrive(&ifull[r]);
                if (item < 0) break;
                const int li = (item / P.n_mg) * P.spi, mg = item % P.n_mg;
                const int rowa = li * slot_rows + mg * P.mti * 128;
                const int rowb = li * P.rq;
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait(&empty[s], ph ^ 1, P.err, 11)) { abort_flag = 1; break; }
                    uint8_t* st = smem + (size_t)s * stage_bytes;
                    mbar_expect_tx(&full[s], tx_bytes);
                    for (int mt = 0; mt < P.mti; ++mt)
                        tma_load_2d(st + mt * a_tile, &map_a, &full[s], kt * 128, rowa + mt * 128);
                    tma_load_2d(st + a_region, &map_b, &full[s], kt * 128, rowb);
                    if (++s == S) { s = 0; ph ^= 1; }
                }
            }
            for (int i = 0; i < S; ++i) {
                mbar_wait(&empty[s], ph ^ 1, P.err, 12);
                if (++s == S) { s = 0; ph ^= 1; }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // Packed slots: one M = 128 MMA over all spi slots' rows against all
            // their key rows (N = nb); the epilogue keeps the diagonal blocks
            // (slot rows x the same slot's key columns).
            const uint32_t idesc = idesc_i8_kk(P.nb);
            int s = 0, as = 0;
            uint32_t ph = 0, aph = 0;
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                if (!mbar_wait(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 17)) { abort_flag = 1; break; }
                const int item = item_ring[r];
                mbar_arrive(&iempty[r]);
                if (item < 0 || abort_flag) break;
                if (!mbar_wait(&tempty[as], aph ^ 1, P.err, 13)) { abort_flag = 1; break; }
                tc_fence_after();
                const uint32_t d0 = tmem_base + (uint32_t)(as * acc_cols);
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait(&full[s], ph, P.err, 14)) { abort_flag = 1; break; }
                    tc_fence_after();
                    const uint8_t* st = smem + (size_t)s * stage_bytes;
                    const uint8_t* bt = st + a_region;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                        if (P.spi == 1) {
                            const uint64_t b = smem_desc(bt + kk * 32, 16, 1024);
                            for (int mt = 0; mt < P.mti; ++mt)
                                mma_i8(d0 + (uint32_t)(mt * P.nb), smem_desc(st + mt * a_tile + kk * 32, 16, 1024),
                                       b, idesc, acc);
                        } else {
                            mma_i8(d0, smem_desc(st + kk * 32, 16, 1024), smem_desc(bt + kk * 32, 16, 1024), idesc,
                                   acc);
                        }
                    }
                    mma_commit(&empty[s]);
                    if (++s == S) { s = 0; ph ^= 1; }
                }
                mma_commit(&tfull[as]);
                if (++as == P.acc_stages) { as = 0; aph ^= 1; }
            }
        }
    } else if (warp >= 4) {
        const int wq = warp & 3;
        const uint32_t lane_base = (uint32_t)(wq * 32) << 16;
        int as = 0;
        uint32_t aph = 0;
        for (int it = 0;; ++it) {
            const int r = it % kRing;
            if (!mbar_wait(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 18)) { abort_flag = 1; break; }
            const int item = item_ring[r];
            mbar_arrive(&iempty[r]);
            if (item < 0) break;
            if (!mbar_wait(&tfull[as], aph, P.err, 15)) { abort_flag = 1; break; }
            tc_fence_after();
            const int li0 = (item / P.n_mg) * P.spi, mg = item % P.n_mg;
            const int l = li0 / kN;
            const uint32_t* c = P.c[l];
            // spi == 1: TMEM block mt (columns mt * nb) holds M-tile mt of the
            // slot's 4G rows.  spi > 1: lane row = sl * 4G + g*4 + a, and slot
            // sl's keys are columns sl * rq ..; the loop runs over the slots
            // this warp's 32 lanes touch (warp-uniform bounds for tcgen05.ld).
            const int row = wq * 32 + lane;
            const int nblk = P.spi > 1 ? min(P.spi - 1, (wq * 32 + 31) / slot_rows) - (wq * 32) / slot_rows + 1
                                       : P.mti;
            const int blk0 = P.spi > 1 ? (wq * 32) / slot_rows : 0;
            for (int bi = 0; bi < nblk; ++bi) {
                const int mt = blk0 + bi;
                const int li = li0 + (P.spi > 1 ? mt : 0);
                const int grow = P.spi > 1 ? row - mt * slot_rows : (mg * P.mti + mt) * 128 + row;  // g*4 + a
                const int g = grow >> 2, a = grow & 3;
                const bool valid = grow >= 0 && grow < slot_rows;
                for (int q = 0; q < P.nq; ++q) {
                    uint32_t v[4];
                    const int col = (P.spi > 1 ? mt * P.rq : mt * P.nb) + 4 * q;
                    tmem_ld4(tmem_base + lane_base + (uint32_t)(as * acc_cols + col), v);
                    uint64_t part = (uint64_t)c[a] * v[0] + (uint64_t)c[a + 1] * v[1] + (uint64_t)c[a + 2] * v[2] +
                                    (uint64_t)c[a + 3] * v[3];
                    part += __shfl_down_sync(0xffffffffu, part, 1);
                    part += __shfl_down_sync(0xffffffffu, part, 2);
                    if (a == 0 && valid)
                        P.out[((size_t)li * P.nq_total + P.q0 + q) * P.G + g] = mod_u64(part, P.cr[l], P.q[l]);
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

bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kUPad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kUPad};
    cuuint32_t box[2] = {128, box_rows};
    cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

uint32_t powmod_host(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1;
    b %= q;
    while (e) {
        if (e & 1) r = r * b % q;
        b = b * b % q;
        e >>= 1;
    }
    return (uint32_t)r;
}

}  // namespace

size_t tp_dt_bytes(size_t groups) { return (size_t)2 * kN * 4 * groups * kUPad; }
size_t tp_gt_bytes(int max_pass) { return (size_t)2 * kN * 4 * (size_t)max_pass * kUPad; }

int tp_pass_queries(size_t groups) {
    // queries per GEMM pass so that the accumulators fit TMEM (512 columns)
    const int mti = (int)std::min<size_t>(4, std::max<size_t>(1, (4 * groups + 127) / 128));
    int b = 32;
    while (b > 1 && mti * ((4 * b + 15) / 16 * 16) > 512) b /= 2;
    return b;
}

cudaError_t launch_dt_transpose(const uint32_t* dp, const uint32_t* dm, size_t g0, size_t nw, size_t G, uint8_t* Dt,
                                cudaStream_t s) {
    if (nw == 0) return cudaSuccess;
    dt_transpose_kernel<<<dim3(kUPad / 32, kN / 32, (unsigned)(nw * 2)), 256, 0, s>>>(dp, dm, g0, G, Dt);
    return cudaGetLastError();
}

cudaError_t launch_dt_export(const uint8_t* Dt, size_t g, size_t G, uint32_t* dp, uint32_t* dm, cudaStream_t s) {
    const size_t n = (size_t)2 * kN * kUsed;
    dt_export_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Dt, g, G, dp, dm);
    return cudaGetLastError();
}

cudaError_t launch_tensor_pass(const uint8_t* Dt, size_t G, const uint32_t* keys, size_t key_qstride, int nq,
                               int nq_total, int q0, uint8_t* Gt, uint32_t* tp_out, int* err, unsigned* tiles,
                               int num_sms, cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (nq > 32 || !tiles) return cudaErrorInvalidValue;
    const int rq = 4 * nq;
    gen_g_kernel<<<dim3(kN / 8, nq, 2), 256, 0, s>>>(keys, key_qstride, Gt, rq);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    TpParams P{};
    P.out = tp_out;
    P.nq_total = nq_total;
    P.q0 = q0;
    P.nq = nq;
    P.rq = rq;
    P.G = (int)G;
    const int nmt = (int)std::max<size_t>(1, (4 * G + 127) / 128);
    P.mti = std::min(nmt, 4);
    P.n_mg = nmt / P.mti;
    // Small G: pack spi slots (each 4G rows) into one 128-row A tile.  G even
    // keeps every slot start on an 8-row (1024-byte) swizzle atom; spi a power
    // of two divides kN, so a packed item never straddles the two limbs.
    auto nb_of = [&](int sp) { return ((sp * rq + 15) / 16) * 16; };
    P.spi = 1;
    if (4 * G < 128 && G % 2 == 0) {
        while (2 * P.spi * 4 * (int)G <= 128) P.spi *= 2;
        while (P.spi > 1 && (nb_of(P.spi) > 256 || 2 * nb_of(P.spi) > 512)) P.spi /= 2;
    }
    P.nb = nb_of(P.spi);
    P.rows_box = (int)std::min<size_t>(128, 4 * G * (size_t)P.spi);
    if (P.mti * P.nb > 512) return cudaErrorInvalidValue;
    P.acc_stages = (2 * P.mti * P.nb <= 512) ? 2 : 1;
    uint32_t need = (uint32_t)(P.acc_stages * P.mti * P.nb), tc = 32;
    while (tc < need) tc <<= 1;
    P.tmem_cols = tc;
    P.err = err;
    P.tiles = tiles;
    const uint32_t qs[2] = {kQ0, kQ1};
    for (int l = 0; l < 2; ++l) {
        for (int k = 0; k < 7; ++k) P.c[l][k] = powmod_host(256, k, qs[l]);
        P.cr[l] = ~0ULL / qs[l];
        P.q[l] = qs[l];
    }
    const size_t a_region = (size_t)P.mti * 128 * 128;
    const size_t stage_bytes = a_region + (size_t)P.nb * 128;
    P.stages = (int)std::min<size_t>(8, (200 * 1024) / stage_bytes);
    if (P.stages < 2) return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    if (!make_map(&ma, Dt, (uint64_t)2 * kN * 4 * G, (uint32_t)P.rows_box)) return cudaErrorInvalidValue;
    // Box rows past the last slot's keys read zeros (TMA out-of-range fill).
    if (!make_map(&mb, Gt, (uint64_t)2 * kN * rq, (uint32_t)P.nb)) return cudaErrorInvalidValue;
    const size_t smem = 1024 + (size_t)P.stages * stage_bytes + (2 * P.stages + 4) * 8 + 16;
    e = allow_max_smem(tp_tc_kernel);
    if (e) return e;
    const int items = (2 * kN / P.spi) * P.n_mg;
    if ((e = cudaMemsetAsync(tiles, 0, sizeof(unsigned), s))) return e;
    tp_tc_kernel<<<std::min(items, std::max(1, num_sms)), 256, smem, s>>>(ma, mb, P);
    return cudaGetLastError();
}

}  // namespace ipb
