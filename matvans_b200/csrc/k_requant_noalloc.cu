// mv_requant_absmax_noalloc: the absmax requantisation of mv_requant_absmax
// for callers that cannot allocate device memory.
//
// Who cannot allocate: plugins embedded in a host framework that owns the
// device allocator and forbids allocations behind its back (its pool may hold
// all free memory, so a cudaMalloc would fail or starve it), and
// latency-critical paths where the implicit device synchronisation of
// cudaMalloc/cudaFree is not acceptable.  mv_requant_absmax
// needs a caller-owned scratch word for its reduction; this variant keeps its
// scratch in a fixed array compiled into the library instead, and calls no
// allocating routine at all (not cudaMalloc, not cudaFree, no allocating
// library call, and not the library's lazily allocated status word).
//
// Scratch: g_noalloc_partials, kNoallocPartials (4096) u32 = 16 KiB, 256-byte
// aligned.  Every GPU that loads the library holds these 16 KiB until the
// process exits.  One entry per block of the first pass; a block covers
// kNoallocChunk (8192) elements, so n is limited to 4096 * 8192 = 33,554,432.
//
// Sharing: all calls on a device use the same array and it keeps the last
// call's contents.  Nothing in it has to start at zero: the first pass writes
// every entry the second pass reads.  Two calls whose kernels overlap on the
// GPU (different streams without ordering) race on the array and may produce
// wrong results; serialise them.
//
// Set-up: host code cannot pass the array's name to a kernel (it is only a
// host-side stand-in for the device symbol), so the first call on each device
// looks up the array's device address with cudaGetSymbolAddress, with that
// device current, and caches it.  That first call on a device should happen
// before any stream capture on it.
#include <algorithm>
#include <mutex>

#include "mv_device.cuh"

namespace mv {

constexpr int kNoallocPartials = 4096;
constexpr int kNoallocChunk = 8192;  // 256 threads x 32 elements
constexpr int64_t kNoallocMaxN = (int64_t)kNoallocPartials * kNoallocChunk;

static __device__ __align__(256) uint32_t g_noalloc_partials[kNoallocPartials];

__global__ void __launch_bounds__(256) noalloc_absmax_kernel(const int32_t *y, int n, uint32_t *partials) {
    const int base = blockIdx.x * kNoallocChunk;
    uint32_t local = 0;
    for (int i = base + threadIdx.x; i < min(n, base + kNoallocChunk); i += blockDim.x) {
        const int v = y[i];
        local = max(local, v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v);
    }
    for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
    __shared__ uint32_t wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = max(m, wmax[w]);
        partials[blockIdx.x] = m;
    }
}

__global__ void __launch_bounds__(256) noalloc_requant_kernel(const int32_t *y, int n, const uint32_t *partials,
                                                              int nparts, int8_t *out8, float *delta) {
    uint32_t local = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) local = max(local, partials[i]);
    for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
    __shared__ uint32_t wmax[8];
    __shared__ uint32_t total;
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = max(m, wmax[w]);
        total = m;
    }
    __syncthreads();
    // same arithmetic as requant_kernel (mv_requant_absmax)
    const float absmax = (float)(int)(float)total;
    const float d = absmax / 127.0f;
    if (blockIdx.x == 0 && threadIdx.x == 0 && delta) *delta = d;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out8[i] = (int8_t)__float2int_rn((float)y[i] / d);
}

namespace {

// Device address of g_noalloc_partials, looked up once per device.
mv_status noalloc_scratch(uint32_t **out) {
    static std::mutex mu;
    static uint32_t *addr[64] = {nullptr};
    int d = 0;
    MV_CUDA_TRY(cudaGetDevice(&d), "cudaGetDevice");
    if (d < 0 || d >= 64) return fail(MV_ERR_UNSUPPORTED, "device index %d out of range", d);
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[d]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_partials)");
        addr[d] = static_cast<uint32_t *>(p);
    }
    *out = addr[d];
    return MV_OK;
}

}  // namespace

mv_status requant_absmax_noalloc(const int32_t *y, int n, int8_t *out8, float *delta, cudaStream_t st) {
    if (!y || !out8 || n <= 0) return fail(MV_ERR_ARG, "mv_requant_absmax_noalloc: bad arguments");
    if ((int64_t)n > kNoallocMaxN)
        return fail(MV_ERR_ARG,
                    "mv_requant_absmax_noalloc: n = %d exceeds the static scratch limit of %lld elements "
                    "(use mv_requant_absmax with caller-owned scratch)",
                    n, (long long)kNoallocMaxN);
    uint32_t *partials = nullptr;
    mv_status rc = noalloc_scratch(&partials);
    if (rc) return rc;
    const int nparts = (n + kNoallocChunk - 1) / kNoallocChunk;
    noalloc_absmax_kernel<<<nparts, 256, 0, st>>>(y, n, partials);
    const int grid = std::max(1, std::min((n + 255) / 256, 4 * sm_count()));
    noalloc_requant_kernel<<<grid, 256, 0, st>>>(y, n, partials, nparts, out8, delta);
    MV_CUDA_TRY(cudaGetLastError(), "mv_requant_absmax_noalloc launch");
    return MV_OK;
}

}  // namespace mv

extern "C" mv_status mv_requant_absmax_noalloc(const int32_t *y_dev, int n, int8_t *out8_dev, float *delta_dev,
                                               void *stream) {
    return mv::requant_absmax_noalloc(y_dev, n, out8_dev, delta_dev, (cudaStream_t)stream);
}
