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
// Layouts: Dt[l][i][g*4 + a][u] u8 (built once at preprocess by
// dt_transpose_kernel) is the A operand, loaded by TMA.  The B operand, the
// byte planes Gq[l][i][q*4 + b][u], is never stored: per pass keyt_kernel
// writes the compact key table Kt[l][j][p][q] (u32, queries innermost,
// <= 1 MB, stays in L2) and the GEMM's key warps gather from it straight
// into each stage's swizzled B tile.  Output tp_out[l][i][q][g] (u32,
// reduced).
//
// The GEMM kernel is persistent with dynamic work items: the producer takes
// the next item from a per-launch atomic counter and publishes it to the MMA
// thread, the key warps and the epilogue through a ring of shared slots
// (-1 ends it), so SMs held by other kernels at launch take fewer items.
// Warp roles (768 threads): 0 TMA producer (one thread), 1 TMEM allocation
// and MMA issue (one thread), 4..7 epilogue, 8..23 key planes in four
// groups of 128 threads, group g filling the K tiles kt = g mod 4, so four
// stages' gathers are in flight at once.  With fewer stages than groups the
// groups that fill none join the epilogue.
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
constexpr int kKeyGroups = 4;
constexpr int kKeyGroup = 128;    // threads per key group
constexpr int kKeyThreads = kKeyGroups * kKeyGroup;  // warps 8..23
constexpr int kTpThreads = 256 + kKeyThreads;
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

// ------------------------------------------------------------------ key table
// Kt[l][j][p][qq] = K5_q[l][j][p] (key 0 of query qq of the pass, NTT form)
// for qq < nq, zero for nq <= qq < W, W = 8 ceil(nq / 8): the W values of one
// position fill whole 32-byte sectors.
__global__ void __launch_bounds__(256) keyt_kernel(const uint32_t* __restrict__ keys, size_t key_qstride, int nq,
                                                   int W, uint32_t* __restrict__ Kt) {
    const size_t idx = (size_t)blockIdx.x * 256 + threadIdx.x;  // over ((l*kDeff + j)*kN + p)*W + qq
    if (idx >= (size_t)2 * kDeff * kN * W) return;
    const int qq = (int)(idx % (size_t)W);
    const size_t ljp = idx / (size_t)W;
    uint32_t v = 0;
    if (qq < nq) v = keys[(size_t)qq * key_qstride + ljp];  // keys[q][key 0][l][j][p]
    Kt[idx] = v;
}

// One 32-byte sector (8 queries' key words) in a single 256-bit load.
__device__ __forceinline__ void ld_sector(const uint32_t* p, uint32_t (&v)[8]) {
    asm volatile("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "l"(p));
}
// 32-bit store into a K-major SWIZZLE_128B tile (1024-byte aligned base):
// row r's 16-byte chunk c sits at chunk c ^ (r & 7).
__device__ __forceinline__ void st_sw128(uint8_t* tile, uint32_t row, uint32_t col, uint32_t w) {
    *reinterpret_cast<uint32_t*>(tile + row * 128 + ((((col >> 4) ^ (row & 7)) & 7) << 4) + (col & 15)) = w;
}

// One lane's row (g, a) over 4 queries' 16 accumulator columns (byte plane
// b of query k at column 4k + b): part_k = sum_b (256^(a+b) mod q) P[4k + b]
// (< 2^60, unreduced), then summed over the 4 lanes a of group g as a
// reduce-scatter, so that lane a returns query a's total.  Round 1 (xor 1)
// keeps queries a & 1 and (a & 1) + 2, round 2 (xor 2) keeps query a.
__device__ __forceinline__ uint64_t tp_reduce4(const uint32_t (&v)[16], const uint32_t* c, int a) {
    uint64_t part[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        part[k] = (uint64_t)c[a] * v[4 * k] + (uint64_t)c[a + 1] * v[4 * k + 1] + (uint64_t)c[a + 2] * v[4 * k + 2] +
                  (uint64_t)c[a + 3] * v[4 * k + 3];
    const int b0 = a & 1, b1 = (a >> 1) & 1;
    const uint64_t keep0 = b0 ? part[1] : part[0], keep1 = b0 ? part[3] : part[2];
    const uint64_t send0 = b0 ? part[0] : part[1], send1 = b0 ? part[2] : part[3];
    const uint64_t s0 = keep0 + __shfl_xor_sync(0xffffffffu, send0, 1);
    const uint64_t s1 = keep1 + __shfl_xor_sync(0xffffffffu, send1, 1);
    return (b1 ? s1 : s0) + __shfl_xor_sync(0xffffffffu, b1 ? s0 : s1, 2);
}

// ------------------------------------------------------------------ GEMM
struct TpParams {
    uint32_t* out;         // tp_out[l][i][q][g]
    int nq_total;          // queries in the batch (out stride)
    int q0;                // first query of this pass
    int nq;                // queries in this pass
    int rq;                // key rows per slot in the B tile (4 nq)
    int nb;                // N = key rows per item, roundup16(spi * rq)
    int w8;                // 8-query groups per key-table position
    const uint32_t* keyt;  // Kt[l][j][p][8 * w8], 32-byte aligned rows
    int G;                 // groups (Dt rows per slot: 4G)
    int li0;               // first (limb, slot) index l * N + i of this launch
    int n_li;              // (limb, slot) indices it covers
    int mti;               // M tiles (128 rows) per item (4G >= 128)
    int n_mg;              // M-tile groups per (l, i)
    int spi;               // slots per item (4G < 128: several slots share one 128-row A tile)
    int rows_box;          // rows per A box
    int stages;
    int acc_stages;
    uint32_t tmem_cols;
    int* err;
    unsigned* tiles;       // work-item counter, zero at launch
    int has_qmap;          // output row of pass query p: qmap[p] (else q0 + p)
    uint8_t qmap[32];
    uint32_t c[2][7];      // 256^k mod q_l
    uint64_t cr[2];
    uint32_t q[2];
    int abort_after;       // > 0: the MMA issuer stops after this many items and reports code 99 (a test of
                           // the abort path, IPB_TEST_ABORT_AFTER_ITEMS); 0: off
};

__global__ void __launch_bounds__(kTpThreads, 1) tp_tc_kernel(const __grid_constant__ CUtensorMap map_a, TpParams P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = P.stages;
    const uint32_t a_tile = 128 * 128;
    const uint32_t a_region = (uint32_t)P.mti * a_tile;
    const uint32_t b_bytes = (uint32_t)P.nb * 128;
    const uint32_t stage_bytes = a_region + b_bytes;
    const uint32_t tx_bytes = (uint32_t)P.mti * P.rows_box * 128;  // A only; B is written by the key warps
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * stage_bytes);
    uint64_t* full = bars;               // the stage's A tiles have landed (TMA bytes)
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = bars + 2 * S + 2;
    uint64_t* bfull = bars + 2 * S + 4;  // the stage's B tile is written (the key group's arrivals)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * S + 4);
    __shared__ volatile int abort_flag;
    __shared__ volatile int item_ring[kRing];
    __shared__ uint64_t ifull[kRing], iempty[kRing];
    __shared__ uint64_t mma_done;  // the MMA issuer's final commit: all its MMAs have completed
    // tw[w] for w = dir * 1023 + s: t = 5^(1022 - s), or 2N - t when dir = 1;
    // the two w of a 4-u group are one aligned 64-bit read.
    __shared__ __align__(8) uint32_t tw[2 * kSteps + 2];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = threadIdx.x; w < 2 * kSteps + 2; w += blockDim.x) {
        uint32_t t = 0;
        if (w < 2 * kSteps) {
            const int dir = w >= kSteps;
            t = pow5_mod2n(kHalf - 2 - (w - dir * kSteps));
            if (dir) t = (2 * kN - t) & (2 * kN - 1);
        }
        tw[w] = t;
    }
    if (threadIdx.x == 0) {
        abort_flag = 0;
        // full: the producer's expect_tx arrival (A bytes); bfull: the key
        // group of the stage.  Kept apart so that the producer can wait for
        // its own loads alone before the CTA exits.
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&bfull[s], kKeyGroup);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&mma_done, 1);
        // tempty: 128 epilogue threads per share (warps 4..7 and each key
        // group that fills no stages)
        const int shares = 1 + kKeyGroups - (S < kKeyGroups ? S : kKeyGroups);
        for (int a = 0; a < 2; ++a) { mbar_init(&tfull[a], 1); mbar_init(&tempty[a], 128 * shares); }
        for (int r = 0; r < kRing; ++r) { mbar_init(&ifull[r], 1); mbar_init(&iempty[r], 1 + 128 + kKeyThreads); }
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
    const int n_items = (P.n_li / P.spi) * P.n_mg;
    constexpr int ktiles = kUPad / 128;
    const int acc_cols = P.mti * P.nb;
    const int slot_rows = 4 * P.G;  // A rows of one slot

    // Epilogue (TMEM -> reduced tensor-pass values) for the rows of lane
    // quarter wq: warps 4..7 run it, and so do the warps of key groups that
    // fill no stages (fewer stages than groups), each taking every nshare-th
    // 16-column chunk, so the accumulators drain sooner when the MMA waits
    // for them (one TMEM accumulator stage at 32 queries and G >= 97).
    auto epilogue = [&](const int wq, const int share, const int nshare) {
        const uint32_t lane_base = (uint32_t)(wq * 32) << 16;
        int as = 0;
        uint32_t aph = 0;
        for (int it = 0;; ++it) {
            const int r = it % kRing;
            if (!mbar_wait_ab(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 18, &abort_flag)) { abort_flag = 1; break; }
            const int item = item_ring[r];
            mbar_arrive(&iempty[r]);
            if (item < 0) break;
            if (!mbar_wait_ab(&tfull[as], aph, P.err, 15, &abort_flag)) { abort_flag = 1; break; }
            tc_fence_after();
            const int li0 = P.li0 + (item / P.n_mg) * P.spi, mg = item % P.n_mg;
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
            const int nqc = (P.nq + 3) / 4;  // 16-column chunks per block
            for (int bi = 0; bi < nblk; ++bi) {
                const int mt = blk0 + bi;
                const int li = li0 + (P.spi > 1 ? mt : 0);
                const int grow = P.spi > 1 ? row - mt * slot_rows : (mg * P.mti + mt) * 128 + row;  // g*4 + a
                const int g = grow >> 2, a = grow & 3;
                const bool valid = grow >= 0 && grow < slot_rows;
                // four queries (16 columns) per TMEM load where the block has
                // them; the block's last columns one query at a time
                const int lim = P.spi > 1 ? P.nb : (mt + 1) * P.nb;
                for (int q = 0; q < P.nq; q += 4) {
                    if ((bi * nqc + q / 4) % nshare != share) continue;  // this warp's share of the chunks
                    const int col = (P.spi > 1 ? mt * P.rq : mt * P.nb) + 4 * q;
                    const uint32_t ta = tmem_base + lane_base + (uint32_t)(as * acc_cols + col);
                    uint32_t v[16];
                    if (col + 16 <= lim) {
                        tmem_ld16(ta, v);
                    } else {
    #pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            uint32_t t[4] = {0, 0, 0, 0};
                            if (col + 4 * k + 4 <= lim) tmem_ld4(ta + 4 * k, t);
    #pragma unroll
                            for (int e = 0; e < 4; ++e) v[4 * k + e] = t[e];
                        }
                    }
                    const uint64_t tot = tp_reduce4(v, c, a);
                    if (valid && q + a < P.nq) {
                        const int qo = P.has_qmap ? P.qmap[P.q0 + q + a] : P.q0 + q + a;
                        P.out[((size_t)li * P.nq_total + qo) * P.G + g] = mod_u64(tot, P.cr[l], P.q[l]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[as]);
            if (++as == P.acc_stages) { as = 0; aph ^= 1; }
        }
    };
    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            unsigned issued = 0;  // stage loads issued
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                int item = -1;
                if (!abort_flag && mbar_wait_ab(&iempty[r], ((uint32_t)(it / kRing) & 1) ^ 1, P.err, 16, &abort_flag)) {
                    const unsigned t = atomicAdd(P.tiles, 1u);
                    if (t < (unsigned)n_items) item = (int)t;
                } else {
                    abort_flag = 1;
                }
                item_ring[r] = item;
                mbar_arrive(&ifull[r]);
                if (item < 0) break;
                const int li = P.li0 + (item / P.n_mg) * P.spi, mg = item % P.n_mg;
                const int rowa = li * slot_rows + mg * P.mti * 128;
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait_ab(&empty[s], ph ^ 1, P.err, 11, &abort_flag)) { abort_flag = 1; break; }
                    uint8_t* st = smem + (size_t)s * stage_bytes;
                    mbar_expect_tx(&full[s], tx_bytes);
                    for (int mt = 0; mt < P.mti; ++mt)
                        tma_load_2d(st + mt * a_tile, &map_a, &full[s], kt * 128, rowa + mt * 128);
                    ++issued;
                    if (++s == S) { s = 0; ph ^= 1; }
                }
            }
            // Drain: every issued load has landed before the CTA exits, also
            // when the MMA issuer stopped early and never consumed them.  Load n
            // went to stage n % S with phase (n / S) & 1; no later load reuses
            // a stage, so each wait is exact.
            for (unsigned i = 0; i < (unsigned)S && i < issued; ++i) {
                const unsigned n = issued - 1 - i;
                mbar_wait(&full[n % S], (n / S) & 1u, P.err, 12);
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
            bool any_mma = false;
            for (int it = 0;; ++it) {
                const int r = it % kRing;
                if (!mbar_wait_ab(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 17, &abort_flag)) { abort_flag = 1; break; }
                const int item = item_ring[r];
                mbar_arrive(&iempty[r]);
                if (item < 0 || abort_flag) break;
                if (P.abort_after > 0 && it >= P.abort_after) {  // test hook: the designed early stop
                    atomicCAS(P.err, 0, 99);
                    abort_flag = 1;
                    break;
                }
                if (!mbar_wait_ab(&tempty[as], aph ^ 1, P.err, 13, &abort_flag)) { abort_flag = 1; break; }
                tc_fence_after();
                const uint32_t d0 = tmem_base + (uint32_t)(as * acc_cols);
                for (int kt = 0; kt < ktiles; ++kt) {
                    if (!mbar_wait_ab(&full[s], ph, P.err, 14, &abort_flag) || !mbar_wait_ab(&bfull[s], ph, P.err, 21, &abort_flag)) {
                        abort_flag = 1;
                        break;
                    }
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
                    any_mma = true;
                    if (++s == S) { s = 0; ph ^= 1; }
                }
                mma_commit(&tfull[as]);
                if (++as == P.acc_stages) { as = 0; aph ^= 1; }
            }
            // Every MMA this thread issued has completed (also after an early
            // stop) before TMEM is deallocated and shared memory released.
            if (any_mma) {
                mma_commit(&mma_done);
                mbar_wait(&mma_done, 0, P.err, 22);
            }
        }
    } else if (warp >= 8) {
        // ---------------- key planes: the B tile of every stage, gathered from
        // the key table.  Unit = (slot sl, 8-query group q8, 4 consecutive u
        // = steps w0, w0+1 x digits j = 0, 1): both digits of a step share the
        // permuted position, so 2 permutations and 4 sector loads; bytes are
        // regrouped into one 32-bit word per (query, byte plane) covering the
        // 4 u.  Lanes take consecutive u groups, so a warp's stores hit 32
        // distinct banks.  The stage of K tile kt of the n-th item is
        // n * ktiles + kt in the producer's sequence (slot and phase follow).
        //
        // Groups take K tiles round robin, so a group can run ahead of the MMA
        // by its stride of stages; an mbarrier parity wait tells the awaited
        // phase apart from one two phases older only if the group's stride
        // is <= the stage count.  So at most min(kKeyGroups, S) groups fill
        // stages; the others only follow the item ring.
        const int kid = (warp - 8) * 32 + lane;
        const int grp = kid / kKeyGroup, gk = kid % kKeyGroup;
        const int ngrp = S < kKeyGroups ? S : kKeyGroups;
        if (grp >= ngrp) {
            epilogue(warp & 3, 1 + grp - ngrp, 1 + kKeyGroups - ngrp);
        } else {
            const int units = P.spi * P.w8 * 32;
            const int W = 8 * P.w8;
            int base = 0;  // stages issued before this item
            for (int it = 0;; ++it, base += ktiles) {
                const int r = it % kRing;
                if (!mbar_wait_ab(&ifull[r], (uint32_t)(it / kRing) & 1, P.err, 19, &abort_flag)) { abort_flag = 1; break; }
                const int item = item_ring[r];
                mbar_arrive(&iempty[r]);
                if (item < 0) break;
                const int li0 = P.li0 + (item / P.n_mg) * P.spi;
                const int l = li0 / kN;
                const uint32_t* kl = P.keyt + (size_t)l * kDeff * kN * W;  // [j][p][W]
                for (int kt = grp; grp < ngrp && kt < ktiles; kt += ngrp) {
                    const int seq = base + kt, s = seq % S;
                    const uint32_t ph = (uint32_t)(seq / S) & 1;
                    if (!mbar_wait_ab(&empty[s], ph ^ 1, P.err, 20, &abort_flag)) { abort_flag = 1; break; }
                    uint8_t* bt = smem + (size_t)s * stage_bytes + a_region;
                    for (int unit = gk; unit < units; unit += kKeyGroup) {
                        const int u4 = unit & 31, sq = unit >> 5;
                        const int sl = sq / P.w8, q8 = sq - sl * P.w8;
                        const uint32_t odd = 2 * brev11((uint32_t)((li0 + sl) & (kN - 1))) + 1;
                        const int w0 = kt * 64 + u4 * 2;  // even: w0 and w0 + 1 both < 2046 or both not
                        uint32_t v[4][8];
                        if (w0 < 2 * kSteps) {
                            const uint2 tt = *reinterpret_cast<const uint2*>(&tw[w0]);
                            const uint32_t p0 = perm_from_odd(tt.x, odd), p1 = perm_from_odd(tt.y, odd);
                            ld_sector(kl + (size_t)p0 * W + 8 * q8, v[0]);          // w0, j = 0
                            ld_sector(kl + ((size_t)kN + p0) * W + 8 * q8, v[1]);   // w0, j = 1
                            ld_sector(kl + (size_t)p1 * W + 8 * q8, v[2]);          // w0 + 1, j = 0
                            ld_sector(kl + ((size_t)kN + p1) * W + 8 * q8, v[3]);   // w0 + 1, j = 1
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; ++e)
#pragma unroll
                                for (int c = 0; c < 8; ++c) v[e][c] = 0;
                        }
                        const uint32_t col = (uint32_t)u4 * 4;
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            const int q = q8 * 8 + c;
                            if (q >= P.nq) break;
                            const uint32_t lo01 = __byte_perm(v[0][c], v[1][c], 0x5140);
                            const uint32_t lo23 = __byte_perm(v[2][c], v[3][c], 0x5140);
                            const uint32_t hi01 = __byte_perm(v[0][c], v[1][c], 0x7362);
                            const uint32_t hi23 = __byte_perm(v[2][c], v[3][c], 0x7362);
                            const uint32_t row0 = (uint32_t)(sl * P.rq + q * 4);
                            st_sw128(bt, row0 + 0, col, __byte_perm(lo01, lo23, 0x5410));  // byte 0 of u..u+3
                            st_sw128(bt, row0 + 1, col, __byte_perm(lo01, lo23, 0x7632));  // byte 1
                            st_sw128(bt, row0 + 2, col, __byte_perm(hi01, hi23, 0x5410));  // byte 2
                            st_sw128(bt, row0 + 3, col, __byte_perm(hi01, hi23, 0x7632));  // byte 3
                        }
                    }
                    // generic-proxy stores -> visible to the tensor core's async proxy
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_arrive(&bfull[s]);
                }
            }
        }
    } else if (warp >= 4) {
        epilogue(warp & 3, 0, 1 + kKeyGroups - (S < kKeyGroups ? S : kKeyGroups));
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
size_t tp_keyt_bytes(int max_pass) { return (size_t)2 * kDeff * kN * 8 * (size_t)((max_pass + 7) / 8) * 4; }

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
                               int nq_total, int q0, uint32_t* keyt, uint32_t* tp_out, int* err, unsigned* tiles,
                               int num_sms, cudaStream_t s) {
    return launch_tensor_pass_slots(Dt, G, 0, 2 * kN, keys, key_qstride, nq, nq_total, q0, nullptr, keyt, tp_out, err,
                                    tiles, num_sms, s);
}

cudaError_t launch_tensor_pass_slots(const uint8_t* Dt, size_t G, int li0, int n_li, const uint32_t* keys,
                                     size_t key_qstride, int nq, int nq_total, int q0, const uint8_t* qmap,
                                     uint32_t* keyt, uint32_t* tp_out, int* err, unsigned* tiles, int num_sms,
                                     cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (nq > 32 || !tiles || (qmap && q0 + nq > 32)) return cudaErrorInvalidValue;
    if (n_li <= 0 || li0 < 0 || li0 + n_li > 2 * kN || li0 % 32 || n_li % 32) return cudaErrorInvalidValue;
    const int rq = 4 * nq;
    const int W = 8 * ((nq + 7) / 8);
    const size_t kt_n = (size_t)2 * kDeff * kN * W;
    keyt_kernel<<<(unsigned)((kt_n + 255) / 256), 256, 0, s>>>(keys, key_qstride, nq, W, keyt);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    TpParams P{};
    P.out = tp_out;
    P.nq_total = nq_total;
    P.q0 = q0;
    P.nq = nq;
    P.rq = rq;
    P.w8 = W / 8;
    P.keyt = keyt;
    P.G = (int)G;
    P.li0 = li0;
    P.n_li = n_li;
    P.has_qmap = qmap != nullptr;
    if (qmap)
        for (int p = 0; p < q0 + nq; ++p) P.qmap[p] = qmap[p];
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
    P.abort_after = test_abort_after_items();
    const uint32_t qs[2] = {kQ0, kQ1};
    for (int l = 0; l < 2; ++l) {
        for (int k = 0; k < 7; ++k) P.c[l][k] = powmod_host(256, k, qs[l]);
        P.cr[l] = ~0ULL / qs[l];
        P.q[l] = qs[l];
    }
    const size_t a_region = (size_t)P.mti * 128 * 128;
    const size_t stage_bytes = a_region + (size_t)P.nb * 128;
    // As many stages as the device's shared memory takes (1 KB alignment
    // slack, 256 B of barriers): at 128 groups, three up to 16 queries.
    size_t max_dyn = 0;
    e = allow_max_smem(tp_tc_kernel, &max_dyn);
    if (e) return e;
    P.stages = (int)std::min<size_t>(8, (max_dyn - 1024 - 256) / stage_bytes);
    if (P.stages < 2) return cudaErrorInvalidValue;
    CUtensorMap ma;
    if (!make_map(&ma, Dt, (uint64_t)2 * kN * 4 * G, (uint32_t)P.rows_box)) return cudaErrorInvalidValue;
    const size_t smem = 1024 + (size_t)P.stages * stage_bytes + (3 * P.stages + 4) * 8 + 16;
    const int items = (n_li / P.spi) * P.n_mg;
    if ((e = cudaMemsetAsync(tiles, 0, sizeof(unsigned), s))) return e;
    tp_tc_kernel<<<std::min(items, std::max(1, num_sms)), kTpThreads, smem, s>>>(ma, P);
    return cudaGetLastError();
}

}  // namespace ipb
