// persist.cu -- server checkpoints: a handle's resident state (the encoded
// DB, the precomputed a / D byte planes / D_final tensors and the public
// parameters) written to a file and restored into a new handle without the
// raw DB and without preprocessing.  The reference keeps this state only in
// device memory; a restart there re-runs gpu_preprocess.
//
// File layout (little-endian), 256-byte header then the sections:
//   char[8] "IPIRB200", u32 version (1), u32 header bytes (256),
//   u64 n_entries, entry_bytes, db_rows, db_cols, n_packed, interp_d, num_cts,
//   u8[64] CRS seed, u64 section bytes[4], u64 section checksums[4],
//   zero padding; sections: DB (u16 [rows][cols], encoded), a (u32
//   [group][limb][N]), D byte planes (u8 [limb][slot][g*4+byte][4096]),
//   D_final (u32 [group][limb][digit][N]).
// Checksum of a section: sum over its 8-byte words w_i of
// mix64(w_i + i * 0x9E3779B97F4A7C15) mod 2^64 (mix64: the splitmix64
// finalizer), computed on the device, so a flipped, missing or moved word
// changes it.
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "server_internal.h"

namespace ipb {

namespace {

constexpr char kMagic[8] = {'I', 'P', 'I', 'R', 'B', '2', '0', '0'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kHeaderBytes = 256;
constexpr size_t kChunk = (size_t)64 << 20;  // pinned staging per copy (two, alternating)
const char* const kSectionName[4] = {"DB", "a", "D byte planes", "D_final"};

struct Header {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    uint64_t geom[7];  // n_entries, entry_bytes, db_rows, db_cols, n_packed, interp_d, num_cts
    uint8_t seed[kSeedBytes];
    uint64_t bytes[4];
    uint64_t sums[4];
};
static_assert(sizeof(Header) <= kHeaderBytes, "checkpoint header");

struct IoError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(256) checksum_kernel(const uint64_t* __restrict__ w, size_t n,
                                                       unsigned long long* __restrict__ out) {
    uint64_t acc = 0;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256)
        acc += mix64(w[i] + i * 0x9E3779B97F4A7C15ull);
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)acc);
}

struct Sections {
    void* dev[4];
    size_t bytes[4];
};
Sections sections_of(const Precomp& P) {
    const size_t G = P.pp.n_packed;
    return Sections{{P.db, P.pre_a, P.pre_dt, P.pre_df},
                    {P.pp.db_rows * P.pp.db_cols * sizeof(uint16_t), G * kGroupStrideA * sizeof(uint32_t),
                     tp_dt_bytes(G), G * kGroupStrideF * sizeof(uint32_t)}};
}

uint64_t device_checksum(const void* d, size_t bytes, unsigned long long* scratch, int num_sms, cudaStream_t s) {
    IPB_CK(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s));
    const size_t n = bytes / 8;  // every section is a multiple of 8 bytes
    checksum_kernel<<<std::max(1, num_sms) * 8, 256, 0, s>>>(static_cast<const uint64_t*>(d), n, scratch);
    IPB_CK(cudaGetLastError());
    unsigned long long h = 0;
    IPB_CK(cudaMemcpyAsync(&h, scratch, sizeof h, cudaMemcpyDeviceToHost, s));
    IPB_CK(cudaStreamSynchronize(s));
    return h;
}

// RAII holders for the host file, a pinned staging buffer, a stream.
struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};
struct Pinned {
    void* p = nullptr;
    explicit Pinned(size_t n) { IPB_CK(cudaHostAlloc(&p, n, cudaHostAllocDefault)); }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { IPB_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
};
// Waits for the stream when it leaves scope, so that no copy into or out of
// the staging buffers (declared before it, destroyed after it) is in flight
// when an error unwinds them.
struct StreamDrain {
    cudaStream_t s;
    ~StreamDrain() { cudaStreamSynchronize(s); }
};
struct Events2 {
    cudaEvent_t e[2] = {nullptr, nullptr};
    Events2() {
        for (auto& x : e) IPB_CK(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    }
    ~Events2() {
        for (auto x : e)
            if (x) cudaEventDestroy(x);
    }
};

// n bytes between buf and the file at offset off (positional I/O).  Reads
// are split over up to 8 host threads, so the page-cache copies run in
// parallel (1 GB checkpoint: 0.29 -> 0.16 s to load; 4 GB: 1.0-1.7 ->
// 0.3-0.6 s).  Writes use one thread: parallel writers to one new file were
// slower.  write: buf -> file, else file -> buf.  False on a short transfer
// or an error.
bool file_io(int fd, void* buf, size_t n, off_t off, bool write) {
    const size_t slice = (size_t)4 << 20;
    const size_t parts = (n + slice - 1) / slice;
    const size_t nt =
        write ? 1 : std::min<size_t>(parts, std::max(1u, std::min(8u, std::thread::hardware_concurrency())));
    std::atomic<bool> ok{true};
    auto run = [&](size_t t) {
        for (size_t pi = t; pi < parts && ok; pi += nt) {
            size_t done = pi * slice;
            const size_t end = std::min(n, done + slice);
            while (done < end) {
                char* b = static_cast<char*>(buf) + done;
                const ssize_t r = write ? ::pwrite(fd, b, end - done, off + (off_t)done)
                                        : ::pread(fd, b, end - done, off + (off_t)done);
                if (r < 0 && errno == EINTR) continue;
                if (r <= 0) {
                    ok = false;
                    return;
                }
                done += (size_t)r;
            }
        }
    };
    std::vector<std::thread> th;
    for (size_t t = 1; t < nt; ++t) th.emplace_back(run, t);
    run(0);
    for (auto& x : th) x.join();
    return ok;
}

void save(const Server& S, const char* path) {
    IPB_CK(cudaSetDevice(S.device));
    const Precomp& P = *S.pre;
    const Sections sec = sections_of(P);
    Stream st;
    DevArena tmp;
    Header h{};
    try {
        unsigned long long* scratch = tmp.alloc<unsigned long long>(1);
        std::memcpy(h.magic, kMagic, 8);
        h.version = kVersion;
        h.header_bytes = kHeaderBytes;
        const Params& pp = P.pp;
        const uint64_t geom[7] = {pp.n_entries, pp.w, pp.db_rows, pp.db_cols, pp.n_packed, pp.D, pp.num_cts};
        std::memcpy(h.geom, geom, sizeof geom);
        std::memcpy(h.seed, pp.seed, kSeedBytes);
        for (int k = 0; k < 4; ++k) {
            h.bytes[k] = sec.bytes[k];
            h.sums[k] = device_checksum(sec.dev[k], sec.bytes[k], scratch, S.num_sms, st.s);
        }
        tmp.free_all();
    } catch (...) {
        tmp.free_all();
        throw;
    }
    File f;
    f.f = std::fopen(path, "wb");
    if (!f.f) throw IoError(std::string("cannot create ") + path);
    unsigned char head[kHeaderBytes] = {};
    std::memcpy(head, &h, sizeof h);
    if (std::fwrite(head, 1, kHeaderBytes, f.f) != kHeaderBytes || std::fflush(f.f) != 0)
        throw IoError("write failed (header)");
    {
        // Chunk c goes device -> staging buffer c % 2 while chunk c - 1 is
        // written from the other buffer.
        Pinned b0(kChunk), b1(kChunk);
        void* buf[2] = {b0.p, b1.p};
        Events2 ev;
        StreamDrain drain{st.s};
        const int fd = fileno(f.f);
        off_t fpos = kHeaderBytes;
        size_t c = 0, prev_n = 0;
        int prev_k = 0;
        for (int k = 0; k < 4; ++k) {
            const uint8_t* d = static_cast<const uint8_t*>(sec.dev[k]);
            for (size_t off = 0; off < sec.bytes[k]; off += kChunk, ++c) {
                const size_t n = std::min(kChunk, sec.bytes[k] - off);
                IPB_CK(cudaMemcpyAsync(buf[c & 1], d + off, n, cudaMemcpyDeviceToHost, st.s));
                IPB_CK(cudaEventRecord(ev.e[c & 1], st.s));
                if (c > 0) {
                    IPB_CK(cudaEventSynchronize(ev.e[(c - 1) & 1]));
                    if (!file_io(fd, buf[(c - 1) & 1], prev_n, fpos, true))
                        throw IoError(std::string("write failed (") + kSectionName[prev_k] + ")");
                    fpos += (off_t)prev_n;
                }
                prev_n = n;
                prev_k = k;
            }
        }
        if (c > 0) {
            IPB_CK(cudaEventSynchronize(ev.e[(c - 1) & 1]));
            if (!file_io(fd, buf[(c - 1) & 1], prev_n, fpos, true))
                throw IoError(std::string("write failed (") + kSectionName[prev_k] + ")");
        }
    }
    const int c = std::fclose(f.f);
    f.f = nullptr;
    if (c != 0) throw IoError("write failed (close)");
}

// Header and file checks, before any device work.
Params read_header(File& f, const char* path, Header& h) {
    f.f = std::fopen(path, "rb");
    if (!f.f) throw IoError(std::string("cannot open ") + path);
    unsigned char head[kHeaderBytes];
    if (std::fread(head, 1, kHeaderBytes, f.f) != kHeaderBytes) throw IoError("not a server checkpoint (short header)");
    std::memcpy(&h, head, sizeof h);
    if (std::memcmp(h.magic, kMagic, 8) != 0) throw IoError("not a server checkpoint (magic)");
    if (h.version != kVersion || h.header_bytes != kHeaderBytes)
        throw IoError("unsupported server checkpoint version");
    Params pp{};
    const char* why = nullptr;
    if (setup_geometry(h.geom[0], h.geom[1], h.geom[2], &pp, &why) != 0)
        throw IoError(std::string("checkpoint geometry rejected: ") + (why ? why : "setup"));
    if (pp.db_cols != h.geom[3] || pp.n_packed != h.geom[4] || pp.D != h.geom[5] || pp.num_cts != h.geom[6])
        throw IoError("checkpoint geometry inconsistent with setup()");
    std::memcpy(pp.seed, h.seed, kSeedBytes);
    const size_t G = pp.n_packed;
    const size_t want[4] = {pp.db_rows * pp.db_cols * sizeof(uint16_t), G * kGroupStrideA * sizeof(uint32_t),
                            tp_dt_bytes(G), G * kGroupStrideF * sizeof(uint32_t)};
    uint64_t total = kHeaderBytes;
    for (int k = 0; k < 4; ++k) {
        if (h.bytes[k] != want[k]) throw IoError(std::string("checkpoint section size wrong (") + kSectionName[k] + ")");
        total += h.bytes[k];
    }
    if (fseeko(f.f, 0, SEEK_END) != 0) throw IoError("cannot seek in checkpoint");
    const off_t size = ftello(f.f);
    if (size < 0 || (uint64_t)size != total)
        throw IoError("checkpoint truncated or oversized: " + std::to_string((long long)size) + " bytes, expected " +
                      std::to_string((unsigned long long)total));
    if (fseeko(f.f, kHeaderBytes, SEEK_SET) != 0) throw IoError("cannot seek in checkpoint");
    return pp;
}

Server* load(const char* path, size_t max_batch) {
    File f;
    Header h{};
    const Params pp = read_header(f, path, h);
    auto P = std::make_shared<Precomp>();
    P->pp = pp;
    IPB_CK(cudaGetDevice(&P->device));
    Stream st;
    alloc_precomp(*P, st.s);
    const Sections sec = sections_of(*P);
    {
        // Chunk c is read into staging buffer c % 2 while chunk c - 1
        // crosses PCIe from the other one.
        Pinned b0(kChunk), b1(kChunk);
        void* buf[2] = {b0.p, b1.p};
        Events2 ev;
        StreamDrain drain{st.s};
        const int fd = fileno(f.f);
        off_t fpos = kHeaderBytes;
        size_t c = 0;
        for (int k = 0; k < 4; ++k) {
            uint8_t* d = static_cast<uint8_t*>(sec.dev[k]);
            for (size_t off = 0; off < sec.bytes[k]; off += kChunk, ++c) {
                const size_t n = std::min(kChunk, sec.bytes[k] - off);
                if (c >= 2) IPB_CK(cudaEventSynchronize(ev.e[c & 1]));  // the copy out of this buffer is done
                if (!file_io(fd, buf[c & 1], n, fpos, false))
                    throw IoError(std::string("read failed (") + kSectionName[k] + ")");
                fpos += (off_t)n;
                IPB_CK(cudaMemcpyAsync(d + off, buf[c & 1], n, cudaMemcpyHostToDevice, st.s));
                IPB_CK(cudaEventRecord(ev.e[c & 1], st.s));
            }
        }
        IPB_CK(cudaStreamSynchronize(st.s));
    }
    int num_sms = 0;
    IPB_CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, P->device));
    DevArena tmp;
    try {
        unsigned long long* scratch = tmp.alloc<unsigned long long>(1);
        for (int k = 0; k < 4; ++k)
            if (device_checksum(sec.dev[k], sec.bytes[k], scratch, num_sms, st.s) != h.sums[k])
                throw IoError(std::string("checkpoint checksum mismatch (") + kSectionName[k] + ")");
        tmp.free_all();
    } catch (...) {
        tmp.free_all();
        throw;
    }
    return make_server(pp, std::move(P), max_batch);
}

}  // namespace
}  // namespace ipb

extern "C" {

int ipir_b200_save_server(const ipir_server* srv, const char* path) {
    if (!srv || !path) {
        ipb::set_last_error("ipir_b200_save_server: null argument");
        return 1;
    }
    ipb::DeviceRestore keep_device;  // save() switches to the handle's device
    try {
        ipb::save(*srv->s, path);
        return 0;
    } catch (const ipb::IoError& e) {
        ipb::set_last_error(e.what());
        return 5;
    } catch (const std::exception& e) {
        ipb::set_last_error(e.what());
        return 4;
    }
}

ipir_server* ipir_b200_load_server(const char* path, size_t max_batch, ipir_params* out_params) {
    if (!path || !out_params || max_batch == 0) {
        ipb::set_last_error("ipir_b200_load_server: null argument or max_batch == 0");
        return nullptr;
    }
    ipb::DeviceRestore keep_device;
    try {
        ipb::Server* S = ipb::load(path, max_batch);
        ipb::fill_params(S->pp, out_params);
        return new ipir_server{S};
    } catch (const std::exception& e) {
        ipb::set_last_error(e.what());
        return nullptr;
    }
}

}  // extern "C"
