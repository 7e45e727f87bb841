// Batched calls over HOST arrays: the batch is cut into chunks that are copied in, computed and
// copied out on a few streams, so that the host<->device copies of one chunk overlap the kernels
// of the others.  Device scratch comes from a per-device stream-ordered memory pool that keeps
// its memory between calls, so a call allocates nothing from the driver after the first.
#pragma once
#include <functional>
#include <vector>
#include <cuda_runtime.h>

namespace agb {

/// one per-item host array of a chunked batch; a null pointer means "not used" (the kernel then
/// gets a null device pointer in its place)
struct HostIn  { const void* host; size_t itemBytes; };
struct HostOut { void* host; size_t itemBytes; };

/// the kernel launch of one chunk: items [first, first + count), device pointers of the chunk's
/// inputs and outputs (in the order given), stream to launch on
using ChunkLaunch = std::function<void(long first, long count, void* const* dIn, void* const* dOut,
    cudaStream_t stream)>;

/// Run a batch of n items over host arrays on the current device and return when the outputs
/// are in host memory.  Pinned (page-locked) host arrays give full copy/compute overlap; pageable
/// ones are staged by the driver and still overlap the kernels of the neighbouring chunks.
/// chunk = 0 picks the chunk size (n/4, at least 65536 items, at most 1 << 20).
void runChunked(long n, const std::vector<HostIn>& ins, const std::vector<HostOut>& outs,
    const ChunkLaunch& launch, long chunk = 0);

/// stream-ordered scratch of the current device from the engine's pool (kept between calls)
void* scratchAlloc(size_t bytes, cudaStream_t stream);
void scratchFree(void* ptr, cudaStream_t stream);

/// RAII holder of pool scratch, released on its stream
struct Scratch {
    void* ptr = nullptr;
    cudaStream_t stream = 0;
    Scratch(size_t bytes, cudaStream_t s) : ptr(scratchAlloc(bytes, s)), stream(s) {}
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    ~Scratch() { if(ptr) scratchFree(ptr, stream); }
};

}  // namespace agb
