// inspire_b200.hpp -- C++ server API of the B200-native InsPIRe server.
//
// The entry points mirror the reference's server protocol, in lifecycle
// order (SoraSuegami/InsPIRe-GPU src/gpu_protocol.h:44-78):
//   setup -> gpu_preprocess -> gpu_setup_server -> gpu_answer /
//   gpu_answer_batch -> gpu_free_server,  plus gpu_server_caps.
// Queries cross as ipir_query_view (the flat layout of the reference's
// C ABI, src/capi.h:47-61) and responses as flat u64 arrays
// [query][ct][a|b][limb][coeff] in NTT form, so the reference's unchanged
// CPU client builds the queries and extracts the answers.
//
// Errors throw (std::invalid_argument for geometry, std::runtime_error for
// CUDA failures); nothing exits the process.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <memory>

#include "inspire_b200.h"

namespace inspire_b200 {

constexpr size_t N = 2048;                   // ring degree (src/params.h:15)
constexpr uint64_t Q0 = 94519297, Q1 = 95293441;
constexpr size_t D_EFF = 2;
constexpr size_t SEED_BYTES = 64;

// Field for field the reference's PublicParams (src/params.h:49-58).
struct PublicParams {
    size_t N_entries = 0;
    size_t w = 0;
    size_t db_rows = 0;
    size_t db_cols = 0;
    size_t n_packed = 0;
    size_t D = 0;
    size_t num_cts = 0;
    std::array<uint8_t, SEED_BYTES> seed{};
};

// src/params.cpp:17-68: same geometry, same rejections (throws
// std::invalid_argument); the CRS seed is drawn from std::random_device.
PublicParams setup(size_t N_entries, size_t w);
PublicParams setup(size_t N_entries, size_t w, size_t db_rows_override);

struct PreprocessState;  // device-resident encoded DB + per-group tensors

// Output of gpu_preprocess (reference src/protocol.h:12-24): owns the
// device buffers until gpu_setup_server adopts them.
struct PreprocessData {
    std::shared_ptr<PreprocessState> state;
};

// Device buffers of a preprocessed database, valid until gpu_setup_server
// adopts them (then until gpu_free_server): the encoded u16 DB (row-major
// db_rows x db_cols) and, per group g, the a part at a + g * a_group_stride
// ([limb][N] u32, NTT form) and D_final at d_final + g * d_final_group_stride
// ([limb][digit][N] u32).  D_plus / D_minus are held as tensor-core byte
// planes (ipir_b200_export_precomp returns them in the reference layout).
struct PreprocessDevicePointers {
    uint16_t* db;
    uint32_t* a;
    size_t a_group_stride;
    uint32_t* d_final;
    size_t d_final_group_stride;
};
PreprocessDevicePointers preprocess_device_pointers(const PreprocessData& precomp);

struct GpuServerConfig {  // src/gpu_protocol.h:22-24
    size_t max_batch = 16;
};
struct GpuServerCaps {    // src/gpu_protocol.h:26-33
    size_t max_batch;
    size_t resident_bytes;
    size_t device_free_bytes;
    size_t num_cts;
};
struct GpuServerCtx;

// src/gpu_protocol.h:44-78
PreprocessData gpu_preprocess(const PublicParams& pp, const uint16_t* db);
GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp);
GpuServerCtx* gpu_setup_server(const PublicParams& pp, const PreprocessData& precomp,
                               const GpuServerConfig& cfg);
GpuServerCaps gpu_server_caps(const GpuServerCtx* ctx);
// One query; out_resp: num_cts*4*N u64.
void gpu_answer(GpuServerCtx* ctx, const ipir_query_view& query, uint64_t* out_resp);
// count <= max_batch queries; out_resp: count*num_cts*4*N u64.  All or nothing.
void gpu_answer_batch(GpuServerCtx* ctx, const ipir_query_view* queries, size_t count,
                      uint64_t* out_resp);
void gpu_free_server(GpuServerCtx* ctx);

}  // namespace inspire_b200
