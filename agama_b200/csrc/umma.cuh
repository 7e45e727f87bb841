// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a: tensor-memory allocation,
// shared-memory matrix descriptors, the BF16 x BF16 -> FP32 MMA, its completion barrier and
// tensor-memory loads.  Written against the PTX ISA 8.7 description of tcgen05; operands are kept
// in the canonical K-major layout without swizzle:
//
//   a 128-byte "core matrix" holds 8 rows x 8 bf16 (16 bytes per row); core matrices adjacent in K
//   are LBO bytes apart, groups of 8 rows SBO bytes apart.  Element (row r, k) of a tile whose K
//   extent is KT therefore sits at byte  (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
//   with LBO = 128 and SBO = KT / 8 * 128 (the tile is 8-row groups of KT/8 consecutive core
//   matrices).  One MMA consumes K = 16, i.e. two core matrices along K starting at the
//   descriptor's address.
#pragma once
#include <cstdint>

namespace agb {
namespace umma {

constexpr uint32_t CORE_BYTES = 128;          // one 8 x 16-byte core matrix
constexpr uint32_t LBO = 128;                 // next core matrix along K

__device__ __forceinline__ uint32_t smemAddr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/// byte offset of element (r, k) in a K-major canonical tile of K extent kt
__host__ __device__ constexpr uint32_t tileOffset(int r, int k, int kt)
{
    return static_cast<uint32_t>((r / 8) * (kt / 8) * CORE_BYTES + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2);
}

/// shared-memory matrix descriptor (no swizzle, version 1 for sm_100): start address, leading
/// (K) and stride (8-row group) byte offsets, all in 16-byte units
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

/// instruction descriptor of kind::f16 with BF16 A and B (both K-major), FP32 accumulator, M x N
__host__ __device__ constexpr uint32_t instrDescBf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

/// allocate ncols (power of two >= 32) tensor-memory columns; the address is written to *dst
/// (shared memory).  Executed by one whole warp.
__device__ __forceinline__ void tmemAlloc(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smemAddr(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

/// free the columns (the warp that allocated them)
__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync()  { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/// make generic-proxy writes to shared memory visible to the tensor cores (async proxy)
__device__ __forceinline__ void fenceSmemForAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/// D (tensor memory) = A * B^T (+ D when accumulate), one elected thread
__device__ __forceinline__ void mmaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u) : "memory");
}

/// arrive once on the shared-memory barrier when all earlier MMAs of this thread have completed
__device__ __forceinline__ void commitTo(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smemAddr(mbar)) : "memory");
}

__device__ __forceinline__ void mbarInit(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smemAddr(mbar)), "r"(count) : "memory");
}

/// wait until the barrier's phase with the given parity has completed; gives up after maxTries
/// polls (each poll may itself suspend for a while) and returns false then
__device__ __forceinline__ bool mbarWait(uint64_t* mbar, uint32_t parity, long maxTries)
{
    const uint32_t addr = smemAddr(mbar);
    for(long i = 0; i < maxTries; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if(done) return true;
    }
    return false;
}

/// 32 consecutive FP32 columns of this thread's tensor-memory lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for(int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

}  // namespace umma
}  // namespace agb
