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
struct NoAllocDevice {
    unsigned long long ctx_id;  // CUDA context the tables were written in (0: none yet)
    uint8_t* addr;              // device address of g_noalloc_scratch in that context
};
NoAllocDevice g_noalloc_dev[64];

// Unique id of the calling thread's current CUDA context (driver entry points
// through the runtime, so the library needs no -lcuda).  A device reset
// destroys the context and the module with it; a new context gets a new id,
// which makes the next call write the tables again.
cudaError_t current_context_id(unsigned long long* id) {
    typedef int (*get_current_t)(void**);
    typedef int (*get_id_t)(void*, unsigned long long*);
    static get_current_t get_current = nullptr;
    static get_id_t get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<get_current_t>(p);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<get_id_t>(p);
    });
    if (!get_current || !get_id) return cudaErrorNotSupported;
    void* ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

// Per device and context, with that device current: resolve the array's
// device address (the host symbol is only a stand-in) and write the NTT
// tables into it.  The copy is enqueued on the caller's stream and waited for
// under the lock, so neither this call's kernels (same stream) nor another
// thread's call on another stream can read the tables before they land.  No
// allocation.
cudaError_t noalloc_setup(int dev, cudaStream_t s, uint8_t** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // also makes the context current
    if (e != cudaSuccess) return e;
    unsigned long long ctx = 0;
    e = current_context_id(&ctx);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (d.ctx_id != ctx || d.addr != p) {
        static DevTables host_T;
        static std::once_flag once;
        std::call_once(once, [] { build_tables(host_T); });
        e = cudaMemcpyAsync(static_cast<uint8_t*>(p) + kNoAllocTablesOff, &host_T, sizeof(DevTables),
                            cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return e;
        d.ctx_id = ctx;
        d.addr = static_cast<uint8_t*>(p);
    }
    *out = d.addr;
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
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint8_t* base = nullptr;
    if (e == cudaSuccess) e = noalloc_setup(dev, s, &base);
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return 4;
    }
    const DevTables* T = reinterpret_cast<const DevTables*>(base + kNoAllocTablesOff);
    int* err = reinterpret_cast<int*>(base + kNoAllocErrOff);
    unsigned* tiles = reinterpret_cast<unsigned*>(base + kNoAllocErrOff + 128);  // same 256-byte slot
    uint8_t* planes = base + kNoAllocPlanesOff;
    e = cudaMemsetAsync(err, 0, sizeof(int), s);  // the array keeps the last call's contents
    if (e == cudaSuccess) e = launch_qplanes(queries, 2 * rows, rows, T, planes, (int)count, s);
    // rows <= 32768: one exact K-chunk, so the kernel writes the result directly.
    if (e == cudaSuccess)
        e = launch_matvec_tc(db, rows, cols, planes, (int)count, T, out, 2 * cols, err, tiles, sms, (int)rows, s);
    int h_err = 0;  // read back on the caller's stream: no device-wide synchronisation
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
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
