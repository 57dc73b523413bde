// Decode + int8 matvec for the reference's matvansWarpPerRow (WPR) layout on
// sm_100a.  Parity target: matvansWarpPerRow/matvansWarpPerRow-kernel.cu:46-175.
//
// One warp per row; lane l owns columns 512k + 16l .. 512k + 16l + 15 and its
// own 16-bit word stream (word k at payload[cursor + (k/8)*256 + 8l + k%8],
// create_matrices_WarpPerRow.py:405-420).  Decode step: q = head & 0xFF,
// r = ppf[q], w = min + r, head = (head >> 8) * prob(r) + (q - cdf[r]), refill
// 16 bits when head < 2^16 (kernel.cu:120-157).  B200 changes: the reference's
// per-lane 16-entry ring queue in local memory (kernel.cu:3-44) becomes one
// prefetched register word, refilled by selects (no divergent branch);
// cdf/ppf become one 256 x 32-lane conflict-free shared table of packed
// (symbol, prob, q - cdf) entries; four decoded symbols go through one dp4a
// instead of four scalar multiplies; any number of vectors share a decode.
#include <algorithm>

#include "mv_device.cuh"

namespace mv {

struct WprLaunch {
    const uint16_t *payload;
    size_t payload_size;
    const uint32_t *cursors;
    int8_t min_value;
    const uint8_t *cdf;
    int G;
    const uint8_t *ppf;
    int rows, cols;
    const int8_t *x;
    int batch;
    int32_t *y;
    const float *scales;
    float *ys;
    uint32_t *status;
};

template <int NV>
__global__ void __launch_bounds__(256) wpr_kernel(const WprLaunch L) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *lut = reinterpret_cast<uint32_t *>(smem);  // 256 * 32 words
    uint8_t *xs = reinterpret_cast<uint8_t *>(lut + 256 * 32);  // [NV][cols]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, W = blockDim.x >> 5;

    // one entry per quantile (its three table reads once), written to all 32 lane columns with a rotating
    // column index so that a warp's stores hit 32 different banks
    for (uint32_t q = threadIdx.x; q < 256; q += blockDim.x) {
        const uint32_t r = __ldg(L.ppf + q);
        uint32_t e = 0;
        if ((int)r + 1 > L.G) {
            atomicOr(L.status, MV_DEV_BAD_TABLE);
        } else {
            const uint32_t c0 = __ldg(L.cdf + r), c1 = __ldg(L.cdf + r + 1);
            const uint32_t prob = (c1 - c0) & 0xFF;
            const uint32_t bias = q - c0;  // never negative for a valid table
            if (c0 > q) atomicOr(L.status, MV_DEV_BAD_TABLE);
            e = (uint32_t)(uint8_t)(int8_t)(L.min_value + (int)r) | (prob << 8) | ((bias & 0xFFFF) << 16);
        }
#pragma unroll 8
        for (uint32_t l = 0; l < 32; l++) lut[q * 32 + ((l + q) & 31)] = e;
    }
    for (int i = threadIdx.x; i < NV * L.cols / 16; i += blockDim.x) {
        const int v = i / (L.cols / 16);
        uint4 val = make_uint4(0, 0, 0, 0);
        if (v < L.batch) val = reinterpret_cast<const uint4 *>(L.x)[i];
        reinterpret_cast<uint4 *>(xs)[i] = val;
    }
    __syncthreads();

    const uint32_t *lut_l = lut + lane;
    const int steps = L.cols / 32;
    const uint32_t size = (uint32_t)L.payload_size;  // < 0xF0000000 (checked by the launcher)
    for (int row = blockIdx.x * W + warp; row < L.rows; row += gridDim.x * W) {
        // The lane's word k sits at ix = cursor + (k / 8) * 256 + 8 * lane + k % 8: ix advances by 1 inside a
        // group of 8 words and by 249 from one group to the next.  Reads past the payload return 0 and are
        // flagged (a cursor past the payload starts the lane at its end; ix then grows by at most 249 per
        // symbol, far below 2^32 from a payload under 0xF0000000 words).  Two words are in flight ahead of
        // the state, so a fetch's latency is covered by the symbols of two refills; the refill itself is
        // selects, not a branch, because the lanes refill at different steps.
        const uint64_t ix0 = (uint64_t)__ldg(L.cursors + row) + 8u * (uint32_t)lane;
        uint32_t ix = ix0 < size ? (uint32_t)ix0 : size;
        bool ovf = (uint64_t)ix + 2u > size;
        const uint32_t w0 = ix < size ? (uint32_t)__ldg(L.payload + ix) : 0u;
        const uint32_t w1 = ix + 1u < size ? (uint32_t)__ldg(L.payload + ix + 1u) : 0u;
        uint32_t head = (w0 << 16) | w1;
        // two words in flight: nw (word k) and nw2 (word k + 1, at ix)
        ix += 2u;
        bool nw_oob = ix >= size;
        uint32_t nw = nw_oob ? 0u : (uint32_t)__ldg(L.payload + ix);
        ix += 1u;
        uint32_t j = 3;  // ix's position inside its group of 8
        bool nw2_oob = ix >= size;
        uint32_t nw2 = nw2_oob ? 0u : (uint32_t)__ldg(L.payload + ix);
        int acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0;
        for (int j0 = 0; j0 < steps; j0 += 16) {
            const int colbase = 512 * (j0 >> 4) + 16 * lane;
            uint4 xv[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) xv[v] = *reinterpret_cast<const uint4 *>(xs + (size_t)v * L.cols + colbase);
#pragma unroll
            for (int g = 0; g < 4; g++) {
                uint32_t e[4];
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    e[t] = lut_l[(head & 0xFFu) << 5];
                    head = (head >> 8) * __byte_perm(e[t], 0, 0x4441) + (e[t] >> 16);
                    const bool need = head < (1u << 16);
                    head = need ? __byte_perm(nw, head, 0x5410) : head;  // (head << 16) | nw
                    ovf |= need & nw_oob;
                    // every lane reloads nw2 each symbol, the same word again when it did not refill (an L1
                    // hit): a conditional reload measured 16% more instructions and 9% more time
                    nw = need ? nw2 : nw;
                    nw_oob = need ? nw2_oob : nw_oob;
                    ix += need ? (j == 7u ? 249u : 1u) : 0u;
                    j = (j + (need ? 1u : 0u)) & 7u;
                    nw2_oob = ix >= size;
                    nw2 = nw2_oob ? 0u : (uint32_t)__ldg(L.payload + ix);
                }
                // the four symbols (byte 0 of each entry) packed in column order
                const uint32_t wq = __byte_perm(__byte_perm(e[0], e[1], 0x0040), __byte_perm(e[2], e[3], 0x0040), 0x5410);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const uint32_t xw = g == 0 ? xv[v].x : g == 1 ? xv[v].y : g == 2 ? xv[v].z : xv[v].w;
                    acc[v] = __dp4a((int)wq, (int)xw, acc[v]);
                }
            }
        }
        // the coder ends in its initial head 1 << 16 (create_matrices_WarpPerRow.py:271,372)
        if (head != (1u << 16)) atomicOr(L.status, MV_DEV_FINAL_STATE);
        if (ovf) atomicOr(L.status, MV_DEV_STREAM_OVERRUN);
#pragma unroll
        for (int v = 0; v < NV; v++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int v = 0; v < NV; v++)
                if (v < L.batch) {
                    L.y[(size_t)v * L.rows + row] = acc[v];
                    if (L.ys) L.ys[(size_t)v * L.rows + row] = (float)acc[v] * L.scales[row];
                }
        }
    }
}

// matvansWarpPerRow.cu:51-72 + 167-172 without the host round trip.
__global__ void absmax_kernel(const int32_t *y, int n, uint32_t *m) {
    uint32_t local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = y[i];
        const uint32_t a = v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v;
        local = max(local, a);
    }
    for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
    if ((threadIdx.x & 31) == 0) atomicMax(m, local);
}

__global__ void requant_kernel(const int32_t *y, int n, const uint32_t *m, int8_t *out8, float *delta) {
    // thrust's transform_reduce there yields float(max |y|) (AbsValue returns float)
    const float absmax = (float)(int)(float)*m;
    const float d = absmax / 127.0f;
    if (blockIdx.x == 0 && threadIdx.x == 0 && delta) *delta = d;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out8[i] = (int8_t)__float2int_rn((float)y[i] / d);
}

namespace {

template <int NV>
mv_status launch_wpr(const WprLaunch &L, cudaStream_t st) {
    const int W = 8;
    const size_t smem = 256 * 32 * 4 + (size_t)NV * L.cols;
    if (smem > (size_t)max_smem_optin())
        return fail(MV_ERR_UNSUPPORTED, "WPR: %d columns x %d vectors exceed shared memory", L.cols, NV);
    auto kern = wpr_kernel<NV>;
    int bps = 0;
    mv_status rc = prepare_kernel((const void *)kern, smem, 32 * W, &bps);
    if (rc) return rc;
    const int grid = std::max(1, std::min((L.rows + W - 1) / W, std::max(1, bps) * sm_count()));
    kern<<<grid, 32 * W, smem, st>>>(L);
    MV_CUDA_TRY(cudaGetLastError(), "wpr kernel launch");
    return MV_OK;
}

}  // namespace

mv_status wpr_matvec(const uint16_t *payload, size_t payload_size, const uint32_t *cursors,
                     int8_t min_value, const uint8_t *cdf, int G, const uint8_t *ppf, int rows, int cols,
                     const int8_t *x, int batch, int32_t *y, const float *scales, float *ys,
                     cudaStream_t st) {
    if (!payload || !cursors || !cdf || !ppf || !x || !y) return fail(MV_ERR_ARG, "mv_wpr_matvec: NULL pointer");
    if (rows <= 0 || cols <= 0 || batch <= 0 || G < 1) return fail(MV_ERR_ARG, "mv_wpr_matvec: bad sizes");
    if (cols % 512) return fail(MV_ERR_SHAPE, "WPR layout needs cols %% 512 == 0 (cols=%d)", cols);
    if (((uintptr_t)payload & 15) || ((uintptr_t)x & 15))
        return fail(MV_ERR_ARG, "mv_wpr_matvec: payload and x must be 16-byte aligned");
    if (ys && !scales) return fail(MV_ERR_ARG, "mv_wpr_matvec: y_scaled needs row scales");
    if (payload_size >= 0xF0000000u) return fail(MV_ERR_UNSUPPORTED, "mv_wpr_matvec: payload of 0xF0000000 words or more");
    mv_status rc;
    WprLaunch L{};
    L.status = device_status_word(&rc);
    if (rc) return rc;
    L.payload = payload;
    L.payload_size = payload_size;
    L.cursors = cursors;
    L.min_value = min_value;
    L.cdf = cdf;
    L.G = G;
    L.ppf = ppf;
    L.rows = rows;
    L.cols = cols;
    for (int v0 = 0; v0 < batch; v0 += 16) {
        const int nb = std::min(16, batch - v0);
        WprLaunch P = L;
        P.x = x + (size_t)v0 * cols;
        P.batch = nb;
        P.y = y + (size_t)v0 * rows;
        P.scales = scales;
        P.ys = ys ? ys + (size_t)v0 * rows : nullptr;
        if (nb == 1) rc = launch_wpr<1>(P, st);
        else if (nb == 2) rc = launch_wpr<2>(P, st);
        else if (nb <= 4) rc = launch_wpr<4>(P, st);
        else if (nb <= 8) rc = launch_wpr<8>(P, st);
        else rc = launch_wpr<16>(P, st);
        if (rc) return rc;
    }
    return MV_OK;
}

mv_status requant_absmax(const int32_t *y, int n, int8_t *out8, float *delta, uint32_t *scratch,
                         cudaStream_t st) {
    if (!y || !out8 || !scratch || n <= 0) return fail(MV_ERR_ARG, "mv_requant_absmax: bad arguments");
    MV_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(uint32_t), st), "cudaMemsetAsync(absmax)");
    const int grid = std::max(1, std::min((n + 255) / 256, 4 * sm_count()));
    absmax_kernel<<<grid, 256, 0, st>>>(y, n, scratch);
    requant_kernel<<<grid, 256, 0, st>>>(y, n, scratch, out8, delta);
    MV_CUDA_TRY(cudaGetLastError(), "requant kernels launch");
    return MV_OK;
}

}  // namespace mv

extern "C" {

mv_status mv_wpr_matvec(const uint16_t *payload_dev, size_t payload_size, const uint32_t *cursors_dev,
                        int8_t min_value, const uint8_t *cdf_dev, int G, const uint8_t *ppf_dev, int rows,
                        int cols, const int8_t *x_dev, int batch, int32_t *y_dev,
                        const float *row_scales_dev, float *y_scaled_dev, void *stream) {
    return mv::wpr_matvec(payload_dev, payload_size, cursors_dev, min_value, cdf_dev, G, ppf_dev, rows, cols,
                          x_dev, batch, y_dev, row_scales_dev, y_scaled_dev, (cudaStream_t)stream);
}

mv_status mv_requant_absmax(const int32_t *y_dev, int n, int8_t *out8_dev, float *delta_dev,
                            uint32_t *absmax_scratch_dev, void *stream) {
    return mv::requant_absmax(y_dev, n, out8_dev, delta_dev, absmax_scratch_dev, (cudaStream_t)stream);
}

}  // extern "C"
