// Failure-flag compaction that allocates no device memory.
//
// pfsf_tick_dbb turns each island's per-voxel failure flags into the
// {x, y, z, type} tuples of the failure buffer with a three-kernel
// compaction (count per chunk, scan of the counts, ordered write) whose
// per-chunk counts and offsets live in scratch the engine allocated with
// cudaMalloc.  Some callers cannot allocate: a game's physics thread that
// must not stall inside cudaMalloc / cudaFree (both can synchronise the
// whole device and blow an 8 ms tick budget), code running under a
// stream-ordered memory pool or a host allocator it does not own, or a
// caller that only borrows device buffers from another runtime.  This entry
// point runs the same compaction with its scratch in a file-scope device
// array instead, so the only memory it touches is the caller's input and
// output buffers plus that fixed array.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "compat.h"
#include "pfsf/pfsf_b200.h"

namespace {

// 4096 voxels per chunk (compat::fail_compact_blocks), so the array bounds an
// island at 16384 * 4096 = 67,108,864 voxels (the 512 x 512 x 256 grid).
constexpr int64_t kNoAllocMaxChunks = 16384;
constexpr int kMaxDevices = 64;

// counts[kNoAllocMaxChunks] followed by offsets[kNoAllocMaxChunks]: 128 KiB on
// every GPU that loads the library, held until the process exits.
static __device__ __align__(256) int32_t g_compact_scratch[2 * kNoAllocMaxChunks];

// The address is cached per device together with the CUDA context it was
// looked up in: after cudaDeviceReset (or any teardown of the primary
// context) the module is loaded again at another address, so a cached
// address is only reused while the same context is current.
struct ScratchSlot {
    CUcontext ctx;
    int32_t* addr;
};
std::mutex g_setup_mutex;
ScratchSlot g_slots[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The calling thread's current context (nullptr when none is current or the
// driver entry point is unavailable), through the runtime's driver entry
// point query, so the library needs no link against libcuda.
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<CtxGetCurrentFn>(nullptr);
        }
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of g_compact_scratch on the current device.  The host-side
// symbol is only a stand-in for the device array, so the address is looked up
// with that device current (cudaGetSymbolAddress) and cached for the context
// it was found in.
cudaError_t scratch_address(int device, int32_t** out) {
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    ScratchSlot& slot = g_slots[device];
    const CUcontext ctx = current_context();
    if (!slot.addr || !ctx || slot.ctx != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_compact_scratch);
        if (e != cudaSuccess) return e;
        slot.addr = static_cast<int32_t*>(p);
        slot.ctx = current_context();  // the lookup makes the primary context current
    }
    *out = slot.addr;
    return cudaSuccess;
}

}  // namespace

extern "C" PFSF_API pfsf_result pfsf_compact_failures_noalloc(const uint8_t* dev_fail_flags, int32_t lx, int32_t ly,
                                                              int32_t lz, pfsf_pos origin, int32_t* dev_tuples,
                                                              int32_t capacity, int32_t* dev_count, void* stream) {
    if (!dev_fail_flags || !dev_count || lx <= 0 || ly <= 0 || lz <= 0 || capacity < 0 ||
        (capacity > 0 && !dev_tuples))
        return PFSF_ERROR_INVALID_ARG;
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t chunks = pfsf_b200::compat::fail_compact_blocks(n);
    if (chunks > kNoAllocMaxChunks) {
        std::fprintf(stderr,
                     "[libpfsf] pfsf_compact_failures_noalloc: island of %lld voxels exceeds the fixed scratch "
                     "limit of %lld voxels\n",
                     (long long)n, (long long)(kNoAllocMaxChunks * 4096));
        return PFSF_ERROR_INVALID_ARG;
    }
    // An error still pending from the caller's own earlier work is not this
    // call's: report it without clearing it and launch nothing.
    if (cudaPeekAtLastError() != cudaSuccess) return PFSF_ERROR_VULKAN;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
        cudaGetLastError();
        return PFSF_ERROR_NO_DEVICE;
    }
    int32_t* scratch = nullptr;
    const cudaError_t e = scratch_address(device, &scratch);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[libpfsf] pfsf_compact_failures_noalloc: cudaGetSymbolAddress failed: %s\n",
                     cudaGetErrorString(e));
        cudaGetLastError();
        return PFSF_ERROR_VULKAN;
    }
    // Every scratch word the kernels read is written earlier in the same call
    // (counts by the count pass for every chunk in use, offsets by the scan),
    // so nothing needs clearing between calls.
    pfsf_b200::compat::fail_compact(static_cast<cudaStream_t>(stream), dev_fail_flags, lx, ly, lz, origin.x, origin.y,
                                    origin.z, scratch, scratch + kNoAllocMaxChunks, dev_count, dev_tuples, capacity);
    if (cudaGetLastError() != cudaSuccess) return PFSF_ERROR_VULKAN;
    return PFSF_OK;
}
