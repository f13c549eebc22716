// matvec_noalloc.cu -- zero-allocation variant of the tensor-core mat-vec.
#include <cuda_runtime.h>

#include "host_util.h"
#include "ipb_common.cuh"
#include "ipb_launch.h"

#include <mutex>

// ===================================================================== zero-allocation entry point
// ipir_b200_matvec_noalloc: the tensor-core mat-vec for callers that cannot
// allocate device memory -- e.g. a host process whose CUDA memory is owned by
// another allocator or pool it must not bypass, or code running where a
// cudaMalloc would implicitly synchronise the device.  Its scratch (NTT
// tables, the device error word, the query byte planes) lives in the
// file-scope array below (NTT tables, error word and work-item counter, query
// byte planes), sized for at most kNoAllocMaxRows DB rows and
// kNoAllocMaxQueries queries per call; every GPU that loads this library
// holds the array until the process exits.

namespace ipb {
namespace {
constexpr size_t kNoAllocMaxRows = 32768;
constexpr size_t kNoAllocMaxQueries = 8;
constexpr size_t kNoAllocTablesOff = 0;
constexpr size_t kNoAllocErrOff = ((sizeof(DevTables) + 255) / 256) * 256;
constexpr size_t kNoAllocPlanesOff = kNoAllocErrOff + 256;
constexpr size_t kNoAllocPlanesBytes = (8 * kNoAllocMaxQueries + 16) * kNoAllocMaxRows;
constexpr size_t kNoAllocScratchBytes = kNoAllocPlanesOff + kNoAllocPlanesBytes;  // ~2.7 MB

__device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
uint8_t* g_noalloc_addr[64];  // device address of g_noalloc_scratch, per device

// Once per device, with that device current: resolve the array's device
// address (the host symbol is only a stand-in) and write the NTT tables into
// it.  No allocation.
cudaError_t noalloc_setup(int dev, uint8_t** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        static DevTables host_T;
        static std::once_flag once;
        std::call_once(once, [] { build_tables(host_T); });
        e = cudaMemcpy(static_cast<uint8_t*>(p) + kNoAllocTablesOff, &host_T, sizeof(DevTables),
                       cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}
}  // namespace
}  // namespace ipb

extern "C" int ipir_b200_matvec_noalloc(const uint16_t* db, size_t rows, size_t cols, const uint64_t* queries,
                                        size_t count, uint32_t* out, void* stream) {
    using namespace ipb;
    if (!db || !queries || !out) {
        set_last_error("ipir_b200_matvec_noalloc: null argument");
        return 1;
    }
    if (count == 0) return 0;
    if (rows == 0 || rows > kNoAllocMaxRows || rows % 1024 || count > kNoAllocMaxQueries || cols == 0 ||
        cols % 128) {
        set_last_error("ipir_b200_matvec_noalloc: needs rows a multiple of 1024 and <= 32768, count <= 8, "
                       "cols a multiple of 128 (its fixed scratch holds no more)");
        return 2;
    }
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && (dev < 0 || dev >= 64)) e = cudaErrorInvalidDevice;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint8_t* base = nullptr;
    if (e == cudaSuccess) e = noalloc_setup(dev, &base);
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return 4;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DevTables* T = reinterpret_cast<const DevTables*>(base + kNoAllocTablesOff);
    int* err = reinterpret_cast<int*>(base + kNoAllocErrOff);
    unsigned* tiles = reinterpret_cast<unsigned*>(base + kNoAllocErrOff + 128);  // same 256-byte slot
    uint8_t* planes = base + kNoAllocPlanesOff;
    e = cudaMemsetAsync(err, 0, sizeof(int), s);  // the array keeps the last call's contents
    if (e == cudaSuccess) e = launch_qplanes(queries, 2 * rows, rows, T, planes, (int)count, s);
    // rows <= 32768: one exact K-chunk, so the kernel writes the result directly.
    if (e == cudaSuccess)
        e = launch_matvec_tc(db, rows, cols, planes, (int)count, T, out, 2 * cols, err, tiles, sms, (int)rows, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return 4;
    }
    if (h_err) {
        set_last_error("ipir_b200_matvec_noalloc: device pipeline wait timed out");
        return 5;
    }
    return 0;
}
