// Dense int8 comparator and device-wide plumbing (status word, device
// attributes).
//
// mv_dense_matvec is the uncompressed baseline the entropy-coded kernels are
// measured against: the warp-per-row dp4a matvec of
// baselines/baseline_int8/baseline_matVec_custom.cu:99-155, written for
// sm_100a: 16-byte streaming loads that bypass L1 (ld.global.nc.L1::no_allocate),
// four loads in flight per lane, x staged in shared memory, any number of
// vectors per pass sharing one read of W; from four vectors on, each warp
// takes four rows at once so that an x chunk read serves four W chunks.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "mv_device.cuh"

namespace mv {

// x chunk i of vector v: staged in shared memory, or (XG, when NV x cols does not fit) read through
// L1/L2, where every warp of the GPU reads the same few hundred KB
template <int NV, bool XG>
__device__ __forceinline__ uint4 x_chunk(const uint4 *xs, const uint4 *xg, int v, int chunks, int i, int batch) {
    if (XG) return v < batch ? __ldg(xg + (size_t)v * chunks + i) : make_uint4(0, 0, 0, 0);
    return xs[v * chunks + i];
}

template <int NV, bool XG>
__global__ void __launch_bounds__(256) dense_kernel(const int8_t *__restrict__ W, int rows, int cols,
                                                    const int8_t *__restrict__ x, int batch,
                                                    int32_t *__restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint4 *xs = reinterpret_cast<uint4 *>(smem);  // [NV][cols/16] unless XG
    const uint4 *xg = reinterpret_cast<const uint4 *>(x);
    const int chunks = cols >> 4;
    if (!XG) {
        for (int i = threadIdx.x; i < NV * chunks; i += blockDim.x) {
            const int v = i / chunks;
            xs[i] = v < batch ? xg[i] : make_uint4(0, 0, 0, 0);
        }
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int row = blockIdx.x * nw + warp; row < rows; row += gridDim.x * nw) {
        const uint4 *wr = reinterpret_cast<const uint4 *>(W + (size_t)row * cols);
        int acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0;
        int i = lane;
        for (; i + 96 < chunks; i += 128) {
            uint4 a[4];
#pragma unroll
            for (int u = 0; u < 4; u++) a[u] = ldg_nc_u4(wr + i + 32 * u);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const uint4 b = x_chunk<NV, XG>(xs, xg, v, chunks, i + 32 * u, batch);
                    acc[v] = __dp4a((int)a[u].x, (int)b.x, acc[v]);
                    acc[v] = __dp4a((int)a[u].y, (int)b.y, acc[v]);
                    acc[v] = __dp4a((int)a[u].z, (int)b.z, acc[v]);
                    acc[v] = __dp4a((int)a[u].w, (int)b.w, acc[v]);
                }
        }
        for (; i < chunks; i += 32) {
            const uint4 a = ldg_nc_u4(wr + i);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const uint4 b = x_chunk<NV, XG>(xs, xg, v, chunks, i, batch);
                acc[v] = __dp4a((int)a.x, (int)b.x, acc[v]);
                acc[v] = __dp4a((int)a.y, (int)b.y, acc[v]);
                acc[v] = __dp4a((int)a.z, (int)b.z, acc[v]);
                acc[v] = __dp4a((int)a.w, (int)b.w, acc[v]);
            }
        }
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
        if (lane == 0)
#pragma unroll
            for (int v = 0; v < NV; v++)
                if (v < batch) y[(size_t)v * rows + row] = acc[v];
    }
}

// Several vectors: a warp takes R rows at once, so that every x chunk it reads (shared memory, or the
// caches) serves R rows; each lane holds R x NV accumulators and reads R W chunks per step (R streaming
// loads in flight).  With one row per warp, 16 vectors cost 16 x-chunk reads per W chunk and the kernel was
// bound by shared memory, not by HBM.
template <int NV, int R, bool XG>
__global__ void __launch_bounds__(256) dense_kernel_rows(const int8_t *__restrict__ W, int rows, int cols,
                                                         const int8_t *__restrict__ x, int batch,
                                                         int32_t *__restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint4 *xs = reinterpret_cast<uint4 *>(smem);  // [NV][cols/16] unless XG
    const uint4 *xg = reinterpret_cast<const uint4 *>(x);
    const int chunks = cols >> 4;
    if (!XG) {
        for (int i = threadIdx.x; i < NV * chunks; i += blockDim.x) {
            const int v = i / chunks;
            xs[i] = v < batch ? xg[i] : make_uint4(0, 0, 0, 0);
        }
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r0 = (blockIdx.x * nw + warp) * R; r0 < rows; r0 += gridDim.x * nw * R) {
        int acc[R][NV];
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[r][v] = 0;
        const uint4 *wr[R];
#pragma unroll
        for (int r = 0; r < R; r++) wr[r] = reinterpret_cast<const uint4 *>(W + (size_t)min(r0 + r, rows - 1) * cols);
        for (int i = lane; i < chunks; i += 32) {
            uint4 a[R];
#pragma unroll
            for (int r = 0; r < R; r++) a[r] = ldg_nc_u4(wr[r] + i);  // rows past the end reread the last row
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const uint4 b = x_chunk<NV, XG>(xs, xg, v, chunks, i, batch);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    acc[r][v] = __dp4a((int)a[r].x, (int)b.x, acc[r][v]);
                    acc[r][v] = __dp4a((int)a[r].y, (int)b.y, acc[r][v]);
                    acc[r][v] = __dp4a((int)a[r].z, (int)b.z, acc[r][v]);
                    acc[r][v] = __dp4a((int)a[r].w, (int)b.w, acc[r][v]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int v = 0; v < NV; v++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[r][v] += __shfl_xor_sync(0xffffffffu, acc[r][v], o);
                if (lane == 0 && v < batch && r0 + r < rows) y[(size_t)v * rows + r0 + r] = acc[r][v];
            }
    }
}

namespace {

template <int NV>
mv_status launch_dense(const int8_t *W, int rows, int cols, const int8_t *x, int batch, int32_t *y,
                       cudaStream_t st) {
    const int nw = 8;
    const bool xg = (size_t)NV * cols > (size_t)max_smem_optin();
    const size_t smem = xg ? 0 : (size_t)NV * cols;
    if constexpr (NV >= 4) {
        constexpr int R = 4;
        auto kern = xg ? dense_kernel_rows<NV, R, true> : dense_kernel_rows<NV, R, false>;
        int bps = 0;
        mv_status rc = prepare_kernel((const void *)kern, smem, 32 * nw, &bps);
        if (rc) return rc;
        const int groups = (rows + R - 1) / R;
        const int grid = std::max(1, std::min((groups + nw - 1) / nw, std::max(1, bps) * sm_count()));
        kern<<<grid, 32 * nw, smem, st>>>(W, rows, cols, x, batch, y);
        MV_CUDA_TRY(cudaGetLastError(), "dense kernel launch");
        return MV_OK;
    }
    auto kern = xg ? dense_kernel<NV, true> : dense_kernel<NV, false>;
    int bps = 0;
    mv_status rc = prepare_kernel((const void *)kern, smem, 32 * nw, &bps);
    if (rc) return rc;
    const int grid = std::max(1, std::min((rows + nw - 1) / nw, std::max(1, bps) * sm_count()));
    kern<<<grid, 32 * nw, smem, st>>>(W, rows, cols, x, batch, y);
    MV_CUDA_TRY(cudaGetLastError(), "dense kernel launch");
    return MV_OK;
}

struct DevInfo {
    uint32_t *status = nullptr;
    int sms = 0;
    int smem_optin = 0;
    int smem_sm = 0;
};

std::mutex g_mu;
DevInfo g_dev[64];

DevInfo *dev_info(mv_status *st) {
    int d = 0;
    cudaError_t e = cudaGetDevice(&d);
    if (e != cudaSuccess || d < 0 || d >= 64) {
        *st = cuda_fail(e, "cudaGetDevice");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    DevInfo &di = g_dev[d];
    if (!di.sms) {
        cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, d);
        cudaDeviceGetAttribute(&di.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
        cudaDeviceGetAttribute(&di.smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, d);
    }
    *st = MV_OK;
    return &di;
}

}  // namespace

uint32_t *device_status_word(mv_status *st) {
    DevInfo *di = dev_info(st);
    if (!di) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!di->status) {
        cudaError_t e = cudaMalloc(&di->status, sizeof(uint32_t));
        if (e != cudaSuccess) {
            *st = cuda_fail(e, "cudaMalloc(status word)");
            di->status = nullptr;
            return nullptr;
        }
        e = cudaMemset(di->status, 0, sizeof(uint32_t));
        if (e != cudaSuccess) {
            *st = cuda_fail(e, "cudaMemset(status word)");
            return nullptr;
        }
    }
    return di->status;
}

static uint32_t g_wait_limit = 0;
static int g_drop_copy = 0;

uint32_t wait_spin_limit() { return g_wait_limit ? g_wait_limit : kWaitSpinLimit; }
int inject_drop_copy() { return g_drop_copy; }

int sm_count() {
    mv_status st;
    DevInfo *di = dev_info(&st);
    return di && di->sms ? di->sms : 148;
}

int max_smem_optin() {
    mv_status st;
    DevInfo *di = dev_info(&st);
    return di && di->smem_optin ? di->smem_optin : 227 * 1024;
}

int max_smem_per_sm() {
    mv_status st;
    DevInfo *di = dev_info(&st);
    return di && di->smem_sm ? di->smem_sm : 228 * 1024;
}

mv_status prepare_kernel(const void *kern, size_t smem, int threads, int *blocks_per_sm) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> smem_set;            // (kernel, device) -> bytes
    static std::map<std::tuple<const void *, int, size_t, int>, int> occ;   // -> blocks per SM
    int d = 0;
    MV_CUDA_TRY(cudaGetDevice(&d), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    int &cur = smem_set[{kern, d}];
    if ((int)smem > cur) {
        MV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "cudaFuncSetAttribute");
        cur = (int)smem;
    }
    if (blocks_per_sm) {
        auto key = std::make_tuple(kern, d, smem, threads);
        auto it = occ.find(key);
        if (it == occ.end()) {
            int n = 0;
            MV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem), "occupancy");
            it = occ.emplace(key, std::max(1, n)).first;
        }
        *blocks_per_sm = it->second;
    }
    return MV_OK;
}

mv_status dense_matvec(const int8_t *W, int rows, int cols, const int8_t *x, int batch, int32_t *y,
                       cudaStream_t st) {
    if (!W || !x || !y || rows <= 0 || cols <= 0 || batch <= 0)
        return fail(MV_ERR_ARG, "mv_dense_matvec: bad arguments");
    if (cols % 16) return fail(MV_ERR_SHAPE, "mv_dense_matvec: cols %% 16 != 0");
    if (((uintptr_t)W & 15) || ((uintptr_t)x & 15))
        return fail(MV_ERR_ARG, "mv_dense_matvec: W and x must be 16-byte aligned");
    // vectors per pass: up to 16, fewer when their x does not fit shared memory (x is then read through the
    // caches only if a single vector does not fit)
    int pass = 16;
    while (pass > 1 && (size_t)pass * cols > (size_t)max_smem_optin()) pass >>= 1;
    for (int v0 = 0; v0 < batch; v0 += pass) {
        const int nb = std::min(pass, batch - v0);
        const int8_t *xv = x + (size_t)v0 * cols;
        int32_t *yv = y + (size_t)v0 * rows;
        mv_status rc;
        if (nb == 1) rc = launch_dense<1>(W, rows, cols, xv, nb, yv, st);
        else if (nb == 2) rc = launch_dense<2>(W, rows, cols, xv, nb, yv, st);
        else if (nb <= 4) rc = launch_dense<4>(W, rows, cols, xv, nb, yv, st);
        else if (nb <= 8) rc = launch_dense<8>(W, rows, cols, xv, nb, yv, st);
        else rc = launch_dense<16>(W, rows, cols, xv, nb, yv, st);
        if (rc) return rc;
    }
    return MV_OK;
}

}  // namespace mv

extern "C" {

mv_status mv_dense_matvec(const int8_t *W_dev, int rows, int cols, const int8_t *x_dev, int batch,
                          int32_t *y_dev, void *stream) {
    return mv::dense_matvec(W_dev, rows, cols, x_dev, batch, y_dev, (cudaStream_t)stream);
}

mv_status mv_debug_inject(int what, uint32_t value) {
    if (what == MV_INJECT_WAIT_LIMIT) mv::g_wait_limit = value;
    else if (what == MV_INJECT_DROP_COPY) mv::g_drop_copy = value ? 1 : 0;
    else return mv::fail(MV_ERR_ARG, "mv_debug_inject: unknown key %d", what);
    return MV_OK;
}

mv_status mv_debug_query(int what, uint64_t *value) {
    if (!value) return mv::fail(MV_ERR_ARG, "mv_debug_query: NULL value");
    if (what != MV_QUERY_STATUS_WORD) return mv::fail(MV_ERR_ARG, "mv_debug_query: unknown key %d", what);
    int d = 0;
    MV_CUDA_TRY(cudaGetDevice(&d), "cudaGetDevice");
    if (d < 0 || d >= 64) return mv::fail(MV_ERR_ARG, "mv_debug_query: device %d out of range", d);
    std::lock_guard<std::mutex> lk(mv::g_mu);
    *value = mv::g_dev[d].status ? 1u : 0u;
    return MV_OK;
}

mv_status mv_device_status(void *stream, uint32_t *flags) {
    if (!flags) return mv::fail(MV_ERR_ARG, "mv_device_status: NULL flags");
    mv_status rc;
    uint32_t *w = mv::device_status_word(&rc);
    if (rc) return rc;
    MV_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream), "cudaStreamSynchronize");
    uint32_t v = 0;
    MV_CUDA_TRY(cudaMemcpy(&v, w, sizeof v, cudaMemcpyDeviceToHost), "read status word");
    MV_CUDA_TRY(cudaMemset(w, 0, sizeof v), "clear status word");
    *flags = v;
    return v ? mv::fail(MV_ERR_DEVICE, "device status flags 0x%x", v) : MV_OK;
}

}  // extern "C"
