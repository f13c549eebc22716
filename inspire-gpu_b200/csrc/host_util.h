// host_util.h -- host helpers shared by the server's C++ and C entry points.
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "ipb_common.cuh"

namespace ipb {

constexpr size_t kSeedBytes = 64;
constexpr size_t kDefaultDbRows = 32768;  // src/params.cpp:17-21
constexpr size_t kDmax = 256;             // src/params.cpp:10
constexpr size_t kPBits = 15;

// Public parameters, field for field the reference's PublicParams
// (src/params.h:49-58).
struct Params {
    size_t n_entries;
    size_t w;
    size_t db_rows;
    size_t db_cols;
    size_t n_packed;
    size_t D;
    size_t num_cts;
    uint8_t seed[kSeedBytes];
};

void shake256(const uint8_t* in, size_t inlen, uint8_t* out, size_t outlen);
void expand_seed(const uint8_t seed[kSeedBytes], const char* domain, uint64_t index, uint32_t* out);
void build_tables(DevTables& T);
// 0 on success; otherwise an error code and *why (static string).
int setup_geometry(size_t n_entries, size_t w, size_t db_rows, Params* out, const char** why);
// Sets the calling thread's text for ipir_b200_last_error().
void set_last_error(const char* msg);
// Test hook for the tensor-core kernels' abort path: the value of
// IPB_TEST_ABORT_AFTER_ITEMS (> 0: the MMA issuer stops after that many work
// items and the launch reports a device wait failure), else 0.
int test_abort_after_items();

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum (less the kernel's static shared memory), once per kernel and
// device.  The limit is then the same for every later launch and for every
// captured graph, whatever size one launch asks for.  *max_dynamic (if
// given) receives that limit in bytes.
cudaError_t allow_max_dynamic_smem(const void* kernel, size_t* max_dynamic = nullptr);
template <class K>
inline cudaError_t allow_max_smem(K* kernel, size_t* max_dynamic = nullptr) {
    return allow_max_dynamic_smem(reinterpret_cast<const void*>(kernel), max_dynamic);
}

}  // namespace ipb
