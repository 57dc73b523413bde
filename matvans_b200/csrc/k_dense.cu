// Dense int8 comparator and device-wide plumbing (status word, device
// attributes).
//
// mv_dense_matvec is the uncompressed baseline the entropy-coded kernels are
// measured against: the warp-per-row dp4a matvec of
// baselines/baseline_int8/baseline_matVec_custom.cu:99-155, written for
// sm_100a: 16-byte streaming loads that bypass L1 (ld.global.nc.L1::no_allocate),
// four loads in flight per lane, x staged in shared memory, any number of
// vectors per pass sharing one read of W; from eight vectors on, each lane
// takes four rows of a column chunk, so that an x chunk read serves four rows.
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

// Reduce-scatter step over lane bit `o`: with N >= 2 sums held, each lane keeps the half of them its bit
// selects and adds its partner's copy of that half (N/2 shuffles); with one, a plain butterfly.
template <int N, int M>
__device__ __forceinline__ void scatter_step(int (&acc)[M], int o, bool bit) {
    if constexpr (N >= 2) {
#pragma unroll
        for (int j = 0; j < N / 2; j++) {
            const int send = bit ? acc[j] : acc[j + N / 2];
            const int keep = bit ? acc[j + N / 2] : acc[j];
            acc[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    } else {
        acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o);
    }
}

// Eight or more vectors: each lane takes R = 4 rows of the same 16-byte column chunk, so that an x chunk read
// from shared memory (16 bytes per vector) serves four W chunks in registers: 16 vectors cost one
// shared-memory wavefront per 4 dp4a instead of one per dp4a, and the kernel becomes bound by the dp4a
// rate (64 per SM and clock: 4.6 TB/s of W at 16 vectors), not by shared memory.  Lane l reads chunks
// l, l + 32, ... of its warp's four rows (each load instruction covers 512 contiguous bytes of one row);
// the next chunks' loads are issued before the current ones are used.  x sits in shared memory in
// slices of `slice` chunks (all of x when it fits, staged once; otherwise the CTA's 32 rows walk the
// slices, restaged per slice).  The warp's 4 x NV row sums meet in one reduce-scatter over the five lane
// bits: 62 shuffles at 16 vectors (instead of 320 for separate butterflies), two sums per lane.
template <int NV>
__global__ void __launch_bounds__(256, 2) dense_kernel_rows(const int8_t *__restrict__ W, int rows, int cols,
                                                            const int8_t *__restrict__ x, int batch,
                                                            int32_t *__restrict__ y, int slice) {
    constexpr int R = 4, M = R * NV;
    extern __shared__ __align__(16) unsigned char smem[];
    uint4 *xs = reinterpret_cast<uint4 *>(smem);  // [NV][slice]
    const uint4 *xg = reinterpret_cast<const uint4 *>(x);
    const int chunks = cols >> 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // scatter steps while two or more sums are held (up to the five lane bits); sum k = r * NV + v
    constexpr int kSteps = M >= 32 ? 5 : M >= 16 ? 4 : M >= 8 ? 3 : 2;
    constexpr int kHeld = M >> kSteps;
    const int base = (lane >> (5 - kSteps)) * kHeld;
    const bool writer = (lane & ((1 << (5 - kSteps)) - 1)) == 0;
    const bool one_slice = chunks <= slice;
    auto stage = [&](int c0, int n) {
        for (int v = 0; v < NV; v++)
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                xs[v * slice + i] = v < batch ? xg[(size_t)v * chunks + c0 + i] : make_uint4(0, 0, 0, 0);
    };
    if (one_slice) {
        stage(0, chunks);
        __syncthreads();
    }
    const int items = (rows + R * nw - 1) / (R * nw);  // 32 rows per CTA item: every warp loops alike
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int r0 = (item * nw + warp) * R;
        // chunk offsets of the four rows from the first (rows past the end reread the last row, store nothing)
        const int rb = min(r0, rows - 1);
        const uint4 *w0 = reinterpret_cast<const uint4 *>(W + (size_t)rb * cols);
        int off[R];
#pragma unroll
        for (int r = 0; r < R; r++) off[r] = (min(r0 + r, rows - 1) - rb) * chunks;
        int acc[M];
#pragma unroll
        for (int k = 0; k < M; k++) acc[k] = 0;
        for (int c0 = 0; c0 < chunks; c0 += slice) {
            const int n = min(slice, chunks - c0);
            if (!one_slice) {
                __syncthreads();  // the previous slice is consumed
                stage(c0, n);
                __syncthreads();
            }
            uint4 a[R], nx[R];
            int i = lane;
            if (i < n) {
#pragma unroll
                for (int r = 0; r < R; r++) a[r] = ldg_nc_u4(w0 + off[r] + c0 + i);
            }
            for (; i < n; i += 32) {
                if (i + 32 < n) {
#pragma unroll
                    for (int r = 0; r < R; r++) nx[r] = ldg_nc_u4(w0 + off[r] + c0 + i + 32);
                }
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const uint4 b = xs[v * slice + i];
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        int &c = acc[r * NV + v];
                        c = __dp4a((int)a[r].x, (int)b.x, c);
                        c = __dp4a((int)a[r].y, (int)b.y, c);
                        c = __dp4a((int)a[r].z, (int)b.z, c);
                        c = __dp4a((int)a[r].w, (int)b.w, c);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; r++) a[r] = nx[r];
            }
        }
        scatter_step<M, M>(acc, 16, (lane & 16) != 0);
        scatter_step<(M >= 2 ? M / 2 : 1), M>(acc, 8, (lane & 8) != 0);
        scatter_step<(M >= 4 ? M / 4 : 1), M>(acc, 4, (lane & 4) != 0);
        scatter_step<(M >= 8 ? M / 8 : 1), M>(acc, 2, (lane & 2) != 0);
        scatter_step<(M >= 16 ? M / 16 : 1), M>(acc, 1, (lane & 1) != 0);
        if (writer)
#pragma unroll
            for (int j = 0; j < kHeld; j++) {
                const int k = base + j, r = k / NV, v = k % NV;
                if (v < batch && r0 + r < rows) y[(size_t)v * rows + r0 + r] = acc[j];
            }
    }
}

namespace {

template <int NV>
mv_status launch_dense(const int8_t *W, int rows, int cols, const int8_t *x, int batch, int32_t *y,
                       cudaStream_t st) {
    const int nw = 8;
    if constexpr (NV >= 8) {
        // x slices of at most 64 KB (NV x slice x 16 bytes): two CTAs per SM.  (At 4 vectors the warp-per-row
        // kernel below measured faster: 0.55 vs 0.71 ms over 56 matrices of the 7B stack.)
        const int chunks = cols / 16, slice = std::min(chunks, 4096 / NV);
        const size_t smem = (size_t)NV * slice * 16;
        auto kern = dense_kernel_rows<NV>;
        int bps = 0;
        mv_status rc = prepare_kernel((const void *)kern, smem, 32 * nw, &bps);
        if (rc) return rc;
        const int items = (rows + 4 * nw - 1) / (4 * nw);  // four rows per warp
        const int grid = std::max(1, std::min(items, std::max(1, bps) * sm_count()));
        kern<<<grid, 32 * nw, smem, st>>>(W, rows, cols, x, batch, y, slice);
        MV_CUDA_TRY(cudaGetLastError(), "dense kernel launch");
        return MV_OK;
    }
    const bool xg = (size_t)NV * cols > (size_t)max_smem_optin();
    const size_t smem = xg ? 0 : (size_t)NV * cols;
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
    // up to 16 vectors per pass share one read of W (x that does not fit shared memory is read through L1)
    const int pass = 16;
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
