// ipb_launch.h -- host-side launch wrappers for the server's CUDA kernels.
// Every wrapper enqueues on the given stream and returns the launch status;
// none of them synchronises or allocates.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ipb {

struct DevTables;

// ---------------------------------------------------------------- online
// Flat per-query device input (u64, the capi.h flat query layout):
//   [b0: rows][b1: rows][ksk5: blk][kskneg1: blk][rgsw: 4 blk],  blk = 2*2*N.
// qprep: keys [q][key(2)][limb][digit][N] NTT form, rgsw32 [q][4][digit][limb][N].
cudaError_t launch_qprep(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T,
                         uint32_t* keys, uint32_t* rgsw32, int nq, cudaStream_t s);
// Only some of it: parts 1 = the keys, 2 = the RGSW parts, 3 = both.
cudaError_t launch_qprep_parts(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T,
                               uint32_t* keys, uint32_t* rgsw32, int nq, int parts, cudaStream_t s);

// Mat-vec row-split partials part[q][chunk][limb][cols] for nq <= 4 queries
// sharing one DB stream.  chunks must divide rows.
cudaError_t launch_matvec(const uint16_t* db, size_t rows, size_t cols, int chunks,
                          const uint64_t* qraw, size_t qstride, const DevTables* T,
                          uint32_t* part, size_t part_qstride, int nq, cudaStream_t s);

// Tensor-core mat-vec (tcgen05 kind::i8).  qplanes writes the CRT byte
// planes planes[7q + k][rows] of nq queries (byte k of CRT(b_0, b_1) < q0 q1);
// launch_matvec_tc runs nq <= 32 queries whose planes start at `planes`
// (mv_tc_planes_offset of the first query), writing
// part[q][chunk][limb][cols] with chunks = rows / kchunk_rows.  *err
// receives a nonzero code if a pipeline wait times out.
size_t mv_tc_planes_bytes(size_t rows, int max_queries);
size_t mv_tc_planes_offset(size_t first_query, size_t rows);
int matvec_tc_kchunk_rows(size_t rows, size_t cols, int num_sms);
// DB columns per mat-vec work item (one m' tile of lo and hi bytes).
int matvec_tc_item_cols();
cudaError_t launch_qplanes(const uint64_t* qraw, size_t qstride, size_t rows, const DevTables* T,
                           uint8_t* planes, int nq, cudaStream_t s);
// tiles: a device counter the launch zeroes and the kernel's CTAs draw work
// items from (one per concurrently running launch).
cudaError_t launch_matvec_tc(const uint16_t* db, size_t rows, size_t cols, const uint8_t* planes, int nq,
                             const DevTables* T, uint32_t* part, size_t part_qstride, int* err, unsigned* tiles,
                             int num_sms, int kchunk_rows, cudaStream_t s);
// The same over the DB columns [c0, c1) of a DB with ld columns per row
// (c0 a multiple of 128): writes part[q'][chunk][limb][c] for c in [c0, c1)
// of the full-width layout (ld columns per chunk and limb); q' = qmap[q]
// for pass query q when qmap (nq entries) is given, else q.
cudaError_t launch_matvec_tc_range(const uint16_t* db, size_t rows, size_t ld, size_t c0, size_t c1,
                                   const uint8_t* planes, int nq, const DevTables* T, uint32_t* part,
                                   size_t part_qstride, const uint8_t* qmap, int* err, unsigned* tiles, int num_sms,
                                   int kchunk_rows, cudaStream_t s);
// The same over n_ranges column ranges of cols_per_range columns, range r
// starting at c0 + r * range_stride, in one launch (one work-item counter,
// so the ranges share the SMs); partial sums land at their own columns.
cudaError_t launch_matvec_tc_ranges(const uint16_t* db, size_t rows, size_t ld, size_t c0, size_t cols_per_range,
                                    int n_ranges, size_t range_stride, const uint8_t* planes, int nq,
                                    const DevTables* T, uint32_t* part, size_t part_qstride, const uint8_t* qmap,
                                    int* err, unsigned* tiles, int num_sms, int kchunk_rows, cudaStream_t s);

// out[q][limb][cols] = sum over chunks of part[q][chunk][limb][cols] mod q.
cudaError_t launch_mv_chunk_reduce(const uint32_t* part, size_t part_qstride, int chunks, size_t cols,
                                   const DevTables* T, uint32_t* out, size_t out_qstride, int nq, cudaStream_t s);

// Tensor pass on tcgen05 (tensorpass_tc.cu).  Dt: re-laid-out D tensors
// [l][i][g*4 + a][4096] u8; keyt: per-pass key table scratch
// (tp_keyt_bytes); tp_out: [l][i][q][g] u32 for the nq_total queries of
// the batch.
size_t tp_dt_bytes(size_t groups);
size_t tp_keyt_bytes(int max_pass);
int tp_pass_queries(size_t groups);
cudaError_t launch_dt_transpose(const uint32_t* dp, const uint32_t* dm, size_t g0, size_t nw, size_t G, uint8_t* Dt,
                                cudaStream_t s);
cudaError_t launch_dt_export(const uint8_t* Dt, size_t g, size_t G, uint32_t* dp, uint32_t* dm, cudaStream_t s);
cudaError_t launch_tensor_pass(const uint8_t* Dt, size_t G, const uint32_t* keys, size_t key_qstride, int nq,
                               int nq_total, int q0, uint32_t* keyt, uint32_t* tp_out, int* err, unsigned* tiles,
                               int num_sms, cudaStream_t s);
// The same for the (limb, slot) indices l * N + i in [li0, li0 + n_li) only
// (multiples of 32), all groups: writes tp_out[l][i][q'][g] for those
// indices, q' = qmap[q0 + p] for pass query p when qmap (the output rows of
// queries 0 .. q0 + nq - 1 of the pass, < nq_total) is given, else q0 + p.
cudaError_t launch_tensor_pass_slots(const uint8_t* Dt, size_t G, int li0, int n_li, const uint32_t* keys,
                                     size_t key_qstride, int nq, int nq_total, int q0, const uint8_t* qmap,
                                     uint32_t* keyt, uint32_t* tp_out, int* err, unsigned* tiles, int num_sms,
                                     cudaStream_t s);

// packed_b[q][g][limb][N] = NTT(sum_y mvpart) - tp_out - Dfinal (.) Kn1.
cudaError_t launch_finalize(const uint32_t* mvpart, size_t mv_qstride, int mv_chunks, size_t cols,
                            const uint32_t* tp_out, const uint32_t* df, const uint32_t* keys, size_t key_qstride,
                            const DevTables* T, uint32_t* packed_b, size_t pb_qstride, size_t groups, int nq,
                            cudaStream_t s);
// The same for the groups [g0, g0 + gn) of nq queries whose tensor-pass
// results are queries tp_q0 .. tp_q0 + nq - 1 of a pass of tp_nq_total.
cudaError_t launch_finalize_range(const uint32_t* mvpart, size_t mv_qstride, int mv_chunks, size_t cols,
                                  const uint32_t* tp_out, int tp_nq_total, int tp_q0, const uint32_t* df,
                                  const uint32_t* keys, size_t key_qstride, const DevTables* T, uint32_t* packed_b,
                                  size_t pb_qstride, size_t groups, size_t g0, size_t gn, int nq, cudaStream_t s);

// Horner chains, one CTA per (ct, query): resp[q][ct][a|b][limb][N] u64.
cudaError_t launch_horner(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                          const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                          size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, cudaStream_t s);

// Same on a cluster of four CTAs per chain (one per polynomial and limb);
// *err receives a nonzero code if a wait for a peer's data times out.
// A sub-range of a Horner chain (one ciphertext's groups, i = d_act - 1 .. 0):
// i_first < 0 starts from the top (acc = packed[d_act - 1], then
// i = d_act - 2), else the chain resumes from acc in state and runs
// i = i_first .. i_last; i_last == 0 ends it (the response is written),
// else acc goes to state [query][ct][a|b][limb][N] u32 for the next range.
struct HornerRange {
    long i_first = -1;
    long i_last = 0;
    uint32_t* state = nullptr;
};
cudaError_t launch_horner_cluster(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                                  const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                                  size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, int* err,
                                  cudaStream_t s, HornerRange hr = HornerRange{});
// Same on a cluster of eight CTAs per chain (polynomial x limb x digit).
cudaError_t launch_horner_cluster8(const uint32_t* pre_a, const uint32_t* packed_b, size_t pb_qstride,
                                   const uint32_t* rgsw32, const DevTables* T, size_t groups, size_t d_act,
                                   size_t num_cts, uint64_t* resp, size_t resp_qstride, int nq, int* err,
                                   cudaStream_t s, HornerRange hr = HornerRange{});

// ---------------------------------------------------------------- wire codecs (codec.cu)
// Byte sizes of the client library's formats: packed query, packed
// response, compressed response (per query).
size_t wire_query_bytes(size_t rows);
size_t wire_response_bytes(size_t num_cts);
size_t wire_compressed_bytes(size_t num_cts);
// nq packed queries (in_stride bytes apart) -> flat u64 queries.
cudaError_t launch_query_unpack(const uint8_t* in, size_t in_stride, size_t rows, uint64_t* out, size_t out_stride,
                                int nq, const DevTables* T, cudaStream_t s);
// nq flat u64 responses -> packed responses (out_stride bytes apart).
cudaError_t launch_response_pack(const uint64_t* flat, size_t flat_stride, size_t num_cts, uint8_t* out,
                                 size_t out_stride, int nq, const DevTables* T, cudaStream_t s);
// nq flat u64 responses -> compressed responses; tmp: nq * num_cts * 4 * N u32.
cudaError_t launch_response_compress(const uint64_t* flat, size_t flat_stride, size_t num_cts, uint32_t* tmp,
                                     uint8_t* out, size_t out_stride, int nq, const DevTables* T, cudaStream_t s);

// ---------------------------------------------------------------- preprocess
// Encode pass over the rows [0, nrows) of a chunk: levels [l0, l0+nl) of the
// inverse DFT over Z_P[X]/(X^N+1) across each ct-block of d_act polys.
// first: source is `src` (raw, gathered in bit-reversed order) else in place.
cudaError_t launch_encode_pass(const uint16_t* src, uint16_t* dst, size_t nrows, size_t cols,
                               size_t d_act, int logd, int l0, int nl, bool first, bool last,
                               uint32_t d_inv, cudaStream_t s);

// a-side for group g: V[limb][p][j] = N^-1 * (sum_r NTT(col_j,r) (.) crs_r)[N-1-p].
cudaError_t launch_a_side(const uint16_t* db, size_t rows, size_t cols, size_t g,
                          const uint32_t* crs, const DevTables* T, uint32_t* V, cudaStream_t s);
// Column NTTs: T[limb][p][m] = NTT_j(V[limb][p][j])[m].
cudaError_t launch_col_ntt(const uint32_t* V, const DevTables* T, uint32_t* Tout, cudaStream_t s);
// a_post[k][dir][limb][i] = T[limb][perm_{+-5^k}(i)][i].
cudaError_t launch_embed_gather(const uint32_t* Tin, uint32_t* a_post, cudaStream_t s);
// CollapseA chains for groups [0, ngroups): one CTA per (group, direction).
cudaError_t launch_collapse_a(const uint32_t* a_post, size_t ap_gstride, const uint32_t* k5,
                              const DevTables* T, uint32_t* dp, uint32_t* dm, uint32_t* ends,
                              size_t ngroups, cudaStream_t s);
// Final CollapseOne per group -> D_final, a.
cudaError_t launch_collapse_final(const uint32_t* ends, const uint32_t* kn1, const DevTables* T,
                                  uint32_t* df, uint32_t* pre_a, size_t ngroups, cudaStream_t s);

// ---------------------------------------------------------------- primitives
// out[k] = splitmix64(seed ^ k) mod 65535 for k < count (the host
// ipir_b200_fill_db formula), on the device.
// Synthetic flat queries (uniform residues per limb) for ids first_id ..
// first_id + count - 1 into out[count][2 rows + 6 * 2 * 2 * N].
cudaError_t launch_synth_queries(uint64_t* out, size_t rows, size_t count, uint64_t seed, uint64_t first_id,
                                 cudaStream_t s);
cudaError_t launch_fill_db(uint16_t* out, size_t count, uint64_t seed, cudaStream_t s);
// In-place forward/inverse NTT of n polys of N u32 (< q); limb of poly i is
// (i / limb_run) & 1.
cudaError_t launch_ntt_batch(uint32_t* polys, size_t n, int limb_run, bool inverse,
                             const DevTables* T, cudaStream_t s);
// Gadget decomposition of n polys: in [i][limb][N] coeff form -> out [i][digit][limb][N].
cudaError_t launch_decomp(const uint32_t* in, uint32_t* out, size_t n, const DevTables* T,
                          cudaStream_t s);

}  // namespace ipb
