// b2s_dot_noalloc: a dot product that allocates no device memory.
//
// Some callers cannot allocate device memory once they are running: a
// solver embedded in a host application whose device memory is owned by
// another framework's allocator (the whole budget is handed out up front), or
// an inner loop that has promised not to allocate after its set-up.  For them
// this entry point takes only device pointers and a stream -- no b2s context
// (creating one allocates) -- and keeps its reduction scratch in a fixed
// file-scope __device__ array instead of cudaMalloc'd memory.
//
// Limits and sharing:
//   - n <= B2S_DOT_NOALLOC_MAX_N (8,388,608): one partial sum per 2,048
//     elements must fit the 4,096-entry scratch; larger n returns
//     B2S_INVALID_ARG before anything is launched.
//   - The scratch is one array per device, shared by every call in the
//     process and kept until exit.  Calls that overlap on the GPU (two
//     streams, or two host threads) race on it; serialise them.
//   - The arrival counter is cleared with cudaMemsetAsync on the caller's
//     stream before every launch, so a call never depends on what the
//     previous call left in the array.
//   - The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture.  Later calls do no lookup.
#include <mutex>

#include "b2s_internal.cuh"

namespace b2s {

namespace {

constexpr uint32_t kNoAllocBlocks = 4096;     // partial sums
constexpr uint32_t kNoAllocPerThread = 8;     // elements per thread
constexpr uint32_t kNoAllocPerBlock = kThreads * kNoAllocPerThread;
static_assert((uint64_t)kNoAllocBlocks * kNoAllocPerBlock == B2S_DOT_NOALLOC_MAX_N, "limit");

// 4096 partials (32 KiB) followed by the arrival counter
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocBlocks * sizeof(double) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

__global__ void __launch_bounds__(kThreads) k_dot_noalloc(uint64_t n, const double* __restrict__ a,
                                                          const double* __restrict__ b, double* __restrict__ out,
                                                          double* partial, unsigned int* counter)
{
    double acc[1] = {0.0};
    const uint64_t base = (uint64_t)blockIdx.x * kNoAllocPerBlock + threadIdx.x;
#pragma unroll
    for (uint32_t k = 0; k < kNoAllocPerThread; ++k)
    {
        const uint64_t i = base + (uint64_t)k * kThreads;
        if (i < n) acc[0] += a[i] * b[i];
    }
    if (grid_reduce_last<1>(acc, partial, counter))
        if (threadIdx.x == 0) *out = acc[0];
}

// device address of the scratch array, looked up once per device
void* scratch_address(int device, cudaError_t* err)
{
    static std::mutex mu;
    static void* addr[64] = {nullptr};
    *err = cudaSuccess;
    if (device < 0 || device >= 64)
    {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device])
    {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (*err != cudaSuccess) return nullptr;
        addr[device] = p;
    }
    return addr[device];
}

}  // namespace

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_dot_noalloc(const double* d_a, const double* d_b, uint64_t n, double* d_out, void* stream)
{
    if (!d_out || (n && (!d_a || !d_b))) return B2S_INVALID_ARG;
    if (n > B2S_DOT_NOALLOC_MAX_N) return B2S_INVALID_ARG;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
    {
        cudaGetLastError();
        return B2S_NO_DEVICE;
    }
    cudaError_t e = cudaSuccess;
    unsigned char* scratch = static_cast<unsigned char*>(scratch_address(device, &e));
    if (!scratch)
    {
        cudaGetLastError();
        return B2S_CUDA_ERROR;
    }
    double* partial = reinterpret_cast<double*>(scratch);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + (size_t)kNoAllocBlocks * sizeof(double));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), s) != cudaSuccess)
    {
        cudaGetLastError();
        return B2S_CUDA_ERROR;
    }
    const unsigned grid = n ? (unsigned)((n + kNoAllocPerBlock - 1) / kNoAllocPerBlock) : 1u;
    k_dot_noalloc<<<grid, kThreads, 0, s>>>(n, d_a, d_b, d_out, partial, counter);
    if (cudaGetLastError() != cudaSuccess) return B2S_CUDA_ERROR;
    return B2S_OK;
}

}  // extern "C"
