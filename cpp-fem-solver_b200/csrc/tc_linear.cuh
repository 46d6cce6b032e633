// Tensor-core (tcgen05) dense layer of the learned IC(0) network:
//
//   Y (n x NO, FP32) = bf16(X) (n x K) W^T (W: NO x K, BF16) [+ bias]
//
// X is the FP32 node-state matrix; each 128-row tile is read once from HBM,
// rounded to BF16 (round to nearest even) and written to shared memory in the
// K-major no-swizzle canonical layout; W sits in shared memory for the whole
// kernel.  One elected thread issues K/16 tcgen05.mma (kind::f16, M = 128,
// N = NO, K = 16, FP32 accumulation in tensor memory) and commits them to an
// mbarrier; the four warps then read their 32 TMEM lanes (= rows) with
// tcgen05.ld and write Y through a swizzled shared-memory transpose, so every
// global store covers whole 128-byte lines.
//
// Persistent grid: 512 / NO CTAs per SM (one NO-column TMEM accumulator
// each, the SM's 512 columns in total); the dynamic shared-memory request is
// sized so that no more CTAs than that fit an SM, so tcgen05.alloc never has
// to wait for another CTA.  The mbarrier wait is bounded: after kMbarPolls
// unsuccessful polls every thread leaves the tile loop, the kernel records
// B2S_TIMEOUT in *err, frees its tensor memory and returns.
//
// Layout and descriptor encodings follow the PTX ISA description of the
// tcgen05 shared-memory matrix descriptor and instruction descriptor (the
// same bit fields as CUTLASS's cute::UMMA::SmemDescriptor / InstrDescriptor).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "b2s.h"

namespace b2s {
namespace tc {

constexpr int kTileRows = 128;   // M of one cta_group::1 tcgen05.mma
constexpr int kThreadsTc = 128;  // warp w owns TMEM lanes (tile rows) 32w .. 32w+31
constexpr uint32_t kMbarPolls = 1u << 20;
constexpr uint32_t kSmemPerSm = 233472;  // 228 KB of shared memory per SM

// Byte offset of element (r, k) of a K-major BF16 tile in the no-swizzle
// canonical layout: core matrices of 8 rows x 16 bytes (128 contiguous
// bytes, row after row); the K/8 core matrices of one 8-row group side by
// side (leading byte offset 128); consecutive 8-row groups K*16 bytes apart
// (stride byte offset).
template <int K>
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t r, uint32_t k)
{
    return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start address >> 4 in bits 0-13, leading
// byte offset >> 4 in bits 16-29, stride byte offset >> 4 in bits 32-45,
// descriptor version 1 in bits 46-47; base offset 0, absolute LBO mode 0,
// layout type 0 (no swizzle) in bits 61-63.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: dense, FP32 accumulator
// (bits 4-5 = 1), A and B BF16 (bits 7-9 = 1, bits 10-12 = 1), no negation,
// A and B K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

template <int K, int NO>
struct LinearShape
{
    static_assert(K % 16 == 0 && K >= 16 && K <= 256, "K: a multiple of the MMA K (16)");
    static_assert(NO >= 32 && NO <= 256 && (NO & (NO - 1)) == 0, "NO: a power of two in 32..256 (TMEM columns)");
    static constexpr uint32_t kA = kTileRows * K * 2;  // BF16 activation tile
    static constexpr uint32_t kB = NO * K * 2;         // BF16 weights
    static constexpr uint32_t kCtasPerSm = 512 / NO;
    static constexpr uint32_t kUsed = 1024 + kA + kB + 16;  // 1 KB alignment slack, mbarrier, TMEM slot
    // no more than kCtasPerSm CTAs (with their 1 KB reservation) fit one SM
    static constexpr uint32_t kFloor = kSmemPerSm / kCtasPerSm - 5120;
    static constexpr uint32_t kSmem = kUsed > kFloor ? kUsed : kFloor;
    static_assert(kCtasPerSm * (kSmem + 1024) <= kSmemPerSm, "resident CTAs must fit");
    static_assert((kCtasPerSm + 1) * (kSmem + 1024) > kSmemPerSm, "one more CTA must not fit");
    static_assert(kA >= 4 * 32 * 32 * 4, "the epilogue transpose reuses the activation tile");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kMbarPolls; ++i)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// D (TMEM) [+]= A (smem) B (smem)^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane; the wait is in the
// same statement so no use of the registers can be scheduled before it
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <int K, int NO>
__global__ void __launch_bounds__(kThreadsTc) k_linear_tc(uint32_t n, const float* __restrict__ X,
                                                         const __nv_bfloat16* __restrict__ W,
                                                         const float* __restrict__ bias, float* __restrict__ Y,
                                                         int* __restrict__ err)
{
    using S = LinearShape<K, NO>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* sA = base;
    uint8_t* sB = base + S::kA;
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + S::kA + S::kB);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t aA = smem_u32(sA), aB = smem_u32(sB), aBar = smem_u32(bar);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"((uint32_t)NO)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(aBar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: 16-byte chunks of 8 BF16 into the canonical layout
    for (int c = threadIdx.x; c < NO * K / 8; c += kThreadsTc)
    {
        const int o = c / (K / 8), kc = c % (K / 8);
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(W + (size_t)o * K + kc * 8));
        *reinterpret_cast<uint4*>(sB + kmajor_offset<K>(o, kc * 8)) = w;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    constexpr uint32_t idesc = idesc_bf16_f32(kTileRows, NO);
    constexpr uint32_t LBO = 128, SBO = K * 16;
    constexpr int F4 = kTileRows * K / 4 / kThreadsTc;  // float4 loads per thread and tile
    const uint32_t ntiles = (n + kTileRows - 1) / kTileRows;
    float* stage = reinterpret_cast<float*>(sA) + warp * 32 * 32;  // this warp's 32 x 32 transpose buffer
    uint32_t parity = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const uint32_t r0 = tile * kTileRows;
        // Activation tile.  A warp's 32 float4 cover 8 rows x 16 columns:
        // 64-byte row segments in global memory, two whole core matrices
        // (256 contiguous bytes) in shared memory.
        float4 xv[F4];
#pragma unroll
        for (int j = 0; j < F4; ++j)
        {
            const int g = warp + 4 * j;
            const uint32_t row = (g / (K / 16)) * 8 + (lane >> 2), k = (g % (K / 16)) * 16 + (lane & 3) * 4;
            xv[j] = (r0 + row < n) ? __ldg(reinterpret_cast<const float4*>(X + (size_t)(r0 + row) * K + k))
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < F4; ++j)
        {
            const int g = warp + 4 * j;
            const uint32_t row = (g / (K / 16)) * 8 + (lane >> 2), k = (g % (K / 16)) * 16 + (lane & 3) * 4;
            const __nv_bfloat162 lo = __floats2bfloat162_rn(xv[j].x, xv[j].y);
            const __nv_bfloat162 hi = __floats2bfloat162_rn(xv[j].z, xv[j].w);
            uint2 pk;
            pk.x = *reinterpret_cast<const uint32_t*>(&lo);
            pk.y = *reinterpret_cast<const uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(sA + kmajor_offset<K>(row, k)) = pk;
        }
        // generic-proxy shared-memory writes -> visible to the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0)
        {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < K / 16; ++s)
                mma_bf16(tmem, smem_desc(aA + s * 2 * LBO, LBO, SBO), smem_desc(aB + s * 2 * LBO, LBO, SBO), idesc,
                         s > 0);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(aBar)
                         : "memory");
        }
        __syncwarp();
        const bool mine = mbar_wait(aBar, parity);
        parity ^= 1u;
        ok = __syncthreads_and(mine) != 0;  // uniform: every thread leaves together
        if (!ok) break;
        tc_fence_after();
        // Epilogue: TMEM lane (32w + lane) holds tile row 32w + lane.  Each
        // 32-column slice goes through the warp's 4 KB transpose buffer
        // (float4 slots XOR-swizzled by row) and out as 4 rows x 128 bytes
        // per store instruction.
        const uint32_t wrow0 = r0 + warp * 32;
#pragma unroll 1
        for (int c0 = 0; c0 < NO; c0 += 32)
        {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                *reinterpret_cast<float4*>(stage + lane * 32 + ((q ^ (lane & 7)) * 4)) =
                    make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            __syncwarp();
            const int q = lane & 7;
            float4 b4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (bias) b4 = *reinterpret_cast<const float4*>(bias + c0 + 4 * q);
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                const int rr = i * 4 + (lane >> 3);
                float4 o = *reinterpret_cast<const float4*>(stage + rr * 32 + ((q ^ (rr & 7)) * 4));
                o.x += b4.x;
                o.y += b4.y;
                o.z += b4.z;
                o.w += b4.w;
                if (wrow0 + rr < n) *reinterpret_cast<float4*>(Y + (size_t)(wrow0 + rr) * NO + c0 + 4 * q) = o;
            }
            __syncwarp();
        }
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) atomicExch(err, (int)B2S_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)NO)
                     : "memory");
    }
}

}  // namespace tc
}  // namespace b2s
