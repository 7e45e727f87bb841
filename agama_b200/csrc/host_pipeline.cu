// Chunked host-array batches: copies of one chunk overlap the kernels of the others.
#include "host_pipeline.h"
#include "runtime.h"
#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>

namespace agb {

namespace {

constexpr int NUM_STREAMS = 3;
constexpr long MIN_CHUNK = 65536;
constexpr long MAX_CHUNK = 1L << 20;
constexpr size_t ALIGN = 256;

/// a set of non-blocking streams of one device, reused across calls (one caller at a time)
struct StreamSet {
    int device;
    cudaStream_t s[NUM_STREAMS];
};

std::mutex g_mutex;
std::vector<StreamSet*> g_idle;
std::map<int, cudaMemPool_t> g_pools;

StreamSet* acquireStreams(int device)
{
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        for(size_t i = 0; i < g_idle.size(); i++)
            if(g_idle[i]->device == device) {
                StreamSet* s = g_idle[i];
                g_idle.erase(g_idle.begin() + i);
                return s;
            }
    }
    StreamSet* s = new StreamSet;
    s->device = device;
    for(int k = 0; k < NUM_STREAMS; k++)
        AGB_CUDA(cudaStreamCreateWithFlags(&s->s[k], cudaStreamNonBlocking));
    return s;
}

void releaseStreams(StreamSet* s)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    g_idle.push_back(s);
}

/// the engine's own pool on a device (not the device's default pool, whose settings belong to
/// the application): memory freed back to it stays reserved for the next call
cudaMemPool_t poolFor(int device)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_pools.find(device);
    if(it != g_pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    AGB_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    AGB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    // a block freed on one stream is not handed to an allocation on another: such reuse makes
    // the allocating stream wait for the freeing one, which serialised the chunks of a host-buffer
    // call (each chunk's scratch on its own stream) instead of overlapping their kernels
    int off = 0;
    AGB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseFollowEventDependencies, &off));
    AGB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &off));
    AGB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off));
    g_pools[device] = pool;
    return pool;
}

size_t roundUp(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }

/// scratch and streams of one call; the destructor waits for the streams and returns both,
/// also when the call is left by an exception
struct Call {
    StreamSet* streams = nullptr;
    char* scratch[NUM_STREAMS] = {};
    ~Call() {
        if(!streams) return;
        for(int k = 0; k < NUM_STREAMS; k++) {
            if(scratch[k]) cudaFreeAsync(scratch[k], streams->s[k]);
            cudaStreamSynchronize(streams->s[k]);
        }
        releaseStreams(streams);
    }
};

}  // namespace

void* scratchAlloc(size_t bytes, cudaStream_t stream)
{
    int device;
    AGB_CUDA(cudaGetDevice(&device));
    void* p = nullptr;
    AGB_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, ALIGN), poolFor(device), stream));
    return p;
}

void scratchFree(void* ptr, cudaStream_t stream)
{
    if(ptr) cudaFreeAsync(ptr, stream);
}

void runChunked(long n, const std::vector<HostIn>& ins, const std::vector<HostOut>& outs,
    const ChunkLaunch& launch, long chunk)
{
    if(n <= 0) return;
    // chunk boundaries (a given chunk size, or the default below)
    std::vector<long> bounds{ 0 };
    if(chunk > 0) {
        for(long f = chunk; f < n; f += chunk) bounds.push_back(f);
    } else if(n >= 8 * MIN_CHUNK) {
        // a short first chunk (its copy in is exposed) and chunks growing so that each copy in
        // ends before the kernels of the previous chunk do; a short last chunk (its copy out is
        // exposed): fractions 0.05, 0.20, 0.35, 0.30, 0.10 of n
        const double frac[4] = { 0.05, 0.25, 0.60, 0.90 };
        for(double f : frac) bounds.push_back(static_cast<long>(f * n));
    } else {        // small batches: four chunks of at least MIN_CHUNK items
        const long c = std::min(MAX_CHUNK, std::max(MIN_CHUNK, (n + 3) / 4));
        for(long f = c; f < n; f += c) bounds.push_back(f);
    }
    bounds.push_back(n);
    for(size_t k = 0; k + 1 < bounds.size(); k++)      // no chunk above the scratch bound
        if(bounds[k + 1] - bounds[k] > MAX_CHUNK) { bounds.insert(bounds.begin() + k + 1, bounds[k] + MAX_CHUNK); }
    const long numChunks = static_cast<long>(bounds.size()) - 1;
    chunk = 0;
    for(long c = 0; c < numChunks; c++) chunk = std::max(chunk, bounds[c + 1] - bounds[c]);
    const int slots = static_cast<int>(std::min<long>(NUM_STREAMS, numChunks));
    int device;
    AGB_CUDA(cudaGetDevice(&device));
    cudaMemPool_t pool = poolFor(device);

    // per-slot scratch: every used array of one chunk, each 256-byte aligned
    std::vector<size_t> inOff(ins.size()), outOff(outs.size());
    size_t bytes = 0;
    for(size_t a = 0; a < ins.size(); a++) { inOff[a] = bytes; if(ins[a].host) bytes += roundUp(ins[a].itemBytes * chunk); }
    for(size_t a = 0; a < outs.size(); a++) { outOff[a] = bytes; if(outs[a].host) bytes += roundUp(outs[a].itemBytes * chunk); }

    Call call;
    call.streams = acquireStreams(device);
    for(int k = 0; k < slots; k++)
        AGB_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&call.scratch[k]), std::max<size_t>(bytes, ALIGN),
            pool, call.streams->s[k]));

    std::vector<void*> dIn(ins.size()), dOut(outs.size());
    auto copyOut = [&](long c) {
        const int k = static_cast<int>(c % slots);
        const long first = bounds[c], count = bounds[c + 1] - bounds[c];
        for(size_t a = 0; a < outs.size(); a++)
            if(outs[a].host)
                AGB_CUDA(cudaMemcpyAsync(static_cast<char*>(outs[a].host) + first * outs[a].itemBytes,
                    call.scratch[k] + outOff[a], count * outs[a].itemBytes, cudaMemcpyDefault, call.streams->s[k]));
    };
    // software pipeline: chunk c is copied in and launched before the copy-out of chunk c-1 is
    // issued, so that a copy-out into pageable memory (which returns only when it is done)
    // never holds back the next launch.  A slot's scratch is reused NUM_STREAMS chunks later on
    // the same stream, after its copy-out.
    for(long c = 0; c < numChunks; c++) {
        const int k = static_cast<int>(c % slots);
        const long first = bounds[c], count = bounds[c + 1] - bounds[c];
        cudaStream_t s = call.streams->s[k];
        for(size_t a = 0; a < ins.size(); a++) {
            dIn[a] = ins[a].host ? call.scratch[k] + inOff[a] : nullptr;
            if(ins[a].host)
                AGB_CUDA(cudaMemcpyAsync(dIn[a], static_cast<const char*>(ins[a].host) + first * ins[a].itemBytes,
                    count * ins[a].itemBytes, cudaMemcpyDefault, s));
        }
        for(size_t a = 0; a < outs.size(); a++)
            dOut[a] = outs[a].host ? call.scratch[k] + outOff[a] : nullptr;
        launch(first, count, dIn.data(), dOut.data(), s);
        if(c > 0) copyOut(c - 1);
    }
    copyOut(numChunks - 1);
    for(int k = 0; k < slots; k++) {
        AGB_CUDA(cudaFreeAsync(call.scratch[k], call.streams->s[k]));
        call.scratch[k] = nullptr;
    }
    for(int k = 0; k < slots; k++)
        AGB_CUDA(cudaStreamSynchronize(call.streams->s[k]));
}

}  // namespace agb
