// Decode + int8 matvec for the reference's "ans-warp-rows" (AWR) layout on
// sm_100a.  Parity target: buffered/ans-warp-rows-kernel.cu:7-221.
//
// The layout makes the 32 lanes of a row share one word stream: at every quad
// step the lanes whose 64-bit state dropped below 2^32 take the next words in
// lane order (ballot + prefix popcount), from a 128-word warp-wide cache that
// holds one uint4 per lane and is read field by field (x, then y, z, w) --
// see ans-warp-rows-kernel.cu:76-139.  That consumption order is part of the
// format, so this kernel keeps one warp per row and reproduces it exactly.
// What changes on B200:
//   * the three 32-entry packed tables are expanded once per CTA into a
//     128-quantile x 32-lane shared table of 8-byte entries {p | sym << 16,
//     q - cum} at byte q*256 + l*8, so the four lookups of a quad are four
//     conflict-free loads instead of twelve warp shuffles
//     (ans-warp-rows-kernel.cu:147-189), each address is one shift and one
//     three-input logic op of the state, and q - cum arrives as a clean word;
//   * the state update forms the reference's r0 + p0 r1 + p0p1 r2 + p0p1p2 r3
//     (ans-warp-rows-kernel.cu:198-202) as (r0 + p0 r1) + (p0 p1)(r2 + p2 r3)
//     with 16x8-bit dot products: the same integer, fewer instructions;
//   * the warp cache advances lazily: a block is loaded only when a lane
//     actually consumes one of its words (the reference also reloads when the
//     cursor lands exactly on a block boundary, which can read past the row);
//   * when the stream length is known, the next block is prefetched one block
//     ahead and every load is bounds-checked;
//   * any number of vectors per pass (1..16) share one decode, x is staged
//     once per CTA, and the int32 result is exact (requantisation optional).
#include <algorithm>
#include <cstdio>

#include "mv_device.cuh"

namespace mv {

struct AwrLaunch {
    const uint4 *comp;
    size_t n_u4;  // 0 = unknown (reference shim): no prefetch, no bounds checks
    const uint32_t *offs, *ppf, *cum, *prob;
    int rows, cols;
    const int8_t *x;
    int batch;
    int32_t *y;
    const float *scales;
    float *ys;
    int8_t *out8;  // requantised output (one vector)
    float scale;
    uint32_t *status;
};

// STRIPES: the "ans-warp-stripes" layout (ans-warp-stripes-kernel.cu:21-227, encoder.py:323-391).  The
// word stream and its cache are the same, but a warp is a stripe of 32 rows: lane l is row 32u + l,
// decodes its quad j (columns 4j..4j+3) at step j and keeps its own sums (no warp reduction), and
// there is one offset per stripe.
template <int NV, bool REQUANT, bool STRIPES>
__global__ void __launch_bounds__(256) awr_kernel(const AwrLaunch L) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2 *lut = reinterpret_cast<uint2 *>(smem);        // 128 * 32 entries of 8 bytes
    uint32_t *xs = reinterpret_cast<uint32_t *>(lut + 128 * 32);  // [cols/4][NV]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, W = blockDim.x >> 5;
    const int nq = L.cols >> 2;

    // one entry per quantile (its table reads once), written to all 32 lane columns with a rotating column
    // index so that a half-warp's 8-byte stores hit distinct banks
    for (uint32_t q = threadIdx.x; q < 128; q += blockDim.x) {
        const uint32_t sh = 8 * (q & 3);
        const uint32_t sym = (__ldg(L.ppf + (q >> 2)) >> sh) & 0xFF;
        const uint32_t c = (__ldg(L.cum + (q >> 2)) >> sh) & 0xFF;
        const uint32_t p = (__ldg(L.prob + (q >> 2)) >> sh) & 0xFF;
        if (c > q || p == 0) atomicOr(L.status, MV_DEV_BAD_TABLE);
        const uint2 e = make_uint2(p | (sym << 16), (q - c) & 0xFFFFu);
#pragma unroll 8
        for (uint32_t l = 0; l < 32; l++) lut[q * 32 + ((l + q) & 31)] = e;
    }
    const bool xal = (reinterpret_cast<uintptr_t>(L.x) & 3) == 0;
    for (int i = threadIdx.x; i < nq * NV; i += blockDim.x) {
        const int c = i / NV, v = i % NV;
        uint32_t val = 0;
        if (v < L.batch) {
            const int8_t *p = L.x + (size_t)v * L.cols + 4 * c;
            if (xal) val = *reinterpret_cast<const uint32_t *>(p);
            else for (int j = 0; j < 4; j++) val |= (uint32_t)(uint8_t)p[j] << (8 * j);
        }
        xs[i] = val;
    }
    __syncthreads();

    const uint32_t lt_mask = (1u << lane) - 1u;
    const unsigned char *lut_b = reinterpret_cast<const unsigned char *>(lut);
    const uint32_t lane8 = (uint32_t)lane << 3;
    const bool bounded = L.n_u4 != 0;

    const int units = STRIPES ? L.rows / 32 : L.rows;  // warps' work units: rows or 32-row stripes
    for (int row = blockIdx.x * W + warp; row < units; row += gridDim.x * W) {
        size_t bi = __ldg(L.offs + row);  // uint4 index of the block held in `cache`
        uint4 cache = make_uint4(0, 0, 0, 0), nxt = make_uint4(0, 0, 0, 0);
        bool ovf = false;
        if (!bounded || bi + 32 <= L.n_u4) cache = L.comp[bi + lane];
        else ovf = true;
        if (bounded && bi + 64 <= L.n_u4) nxt = L.comp[bi + 32 + lane];
        unsigned long long state = ((unsigned long long)cache.w << 32) | cache.z;
        uint32_t wcc = 64;  // reference cursor into the 128-word cache
        bool lag = false;   // cursor crossed a 32-word boundary without advancing

        auto advance = [&](uint32_t leaving_gen) {
            if (leaving_gen == 3) {  // next block
                bi += 32;
                if (bounded) {
                    if (bi + 32 > L.n_u4) ovf = true;
                    cache = nxt;
                    nxt = (bi + 64 <= L.n_u4) ? L.comp[bi + 32 + lane] : make_uint4(0, 0, 0, 0);
                } else {
                    cache = L.comp[bi + lane];
                }
            } else {
                cache.x = cache.y;
                cache.y = cache.z;
                cache.z = cache.w;
            }
        };

        int acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0;

        for (int j = 0; j < nq; j += STRIPES ? 1 : 32) {
            const bool need = (state >> 32) == 0;
            const uint32_t ballot = __ballot_sync(0xffffffffu, need);
            if (ballot) {
                if (lag) {
                    advance((wcc >> 5) == 0 ? 3u : 0u);
                    lag = false;
                }
                const uint32_t off = __popc(ballot & lt_mask);
                const uint32_t num = __popc(ballot);
                const uint32_t lc = (wcc + off) & 31;
                const uint32_t gen = wcc >> 5;
                uint32_t rv = __shfl_sync(0xffffffffu, cache.x, lc);
                if (((wcc + num - 1) >> 5) != gen) {
                    advance(gen);
                    const uint32_t rv2 = __shfl_sync(0xffffffffu, cache.x, lc);
                    if (((wcc + off) >> 5) != gen) rv = rv2;
                } else if (((wcc + num) >> 5) != gen) {
                    lag = true;
                }
                if (need) state = (state << 32) | rv;
                wcc = (wcc + num) & 127;
            }
            const uint32_t lo = (uint32_t)state;
            // quantile k (bits 7k..7k+6) moved to bits 8..14, the lane's byte offset in bits 0..7
            const uint2 e0 = *reinterpret_cast<const uint2 *>(lut_b + (((lo << 8) & 0x7F00u) | lane8));
            const uint2 e1 = *reinterpret_cast<const uint2 *>(lut_b + (((lo << 1) & 0x7F00u) | lane8));
            const uint2 e2 = *reinterpret_cast<const uint2 *>(lut_b + (((lo >> 6) & 0x7F00u) | lane8));
            const uint2 e3 = *reinterpret_cast<const uint2 *>(lut_b + (((lo >> 13) & 0x7F00u) | lane8));
            const uint32_t u01 = __dp2a_lo(e1.y, e0.x, e0.y);  // r0 + p0 r1
            const uint32_t t2 = __dp2a_lo(e3.y, e2.x, e2.y);   // r2 + p2 r3
            const uint32_t p01 = __dp2a_lo(e1.x, e0.x, 0u);    // p0 p1 (+ sym1 * 0)
            const uint32_t p23 = __dp2a_lo(e3.x, e2.x, 0u);    // p2 p3
            state = (state >> 28) * (unsigned long long)(p01 * p23) + (u01 + p01 * t2);
            const uint32_t wq =
                __byte_perm(__byte_perm(e0.x, e1.x, 0x0062), __byte_perm(e2.x, e3.x, 0x0062), 0x5410);
            const uint32_t *xq = xs + (STRIPES ? j : j + lane) * NV;  // stripes: one x quad for all lanes
#pragma unroll
            for (int v = 0; v < NV; v++) acc[v] = __dp4a((int)wq, (int)xq[v], acc[v]);
        }
        if (ovf) atomicOr(L.status, MV_DEV_STREAM_OVERRUN);
        if (STRIPES) {
            const int r = row * 32 + lane;  // rows % 32 == 0
            if (REQUANT) {
                const int q = __float2int_rn((float)acc[0] * L.scale);  // ans-warp-stripes-kernel.cu:220-225
                L.out8[r] = (int8_t)max(-128, min(127, q));
            } else {
#pragma unroll
                for (int v = 0; v < NV; v++)
                    if (v < L.batch) {
                        L.y[(size_t)v * L.rows + r] = acc[v];
                        if (L.ys) L.ys[(size_t)v * L.rows + r] = (float)acc[v] * L.scales[r];
                    }
            }
            continue;
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
        }
        if (lane == 0) {
            if (REQUANT) {
                // ans-warp-rows-kernel.cu:212-220
                const int r = __float2int_rn((float)acc[0] * L.scale);
                L.out8[row] = (int8_t)max(-128, min(127, r));
            } else {
#pragma unroll
                for (int v = 0; v < NV; v++)
                    if (v < L.batch) {
                        L.y[(size_t)v * L.rows + row] = acc[v];
                        if (L.ys) L.ys[(size_t)v * L.rows + row] = (float)acc[v] * L.scales[row];
                    }
            }
        }
    }
}

namespace {

template <int NV, bool REQUANT, bool STRIPES = false>
mv_status launch_awr(const AwrLaunch &L, cudaStream_t st) {
    // stripes: few work units (rows / 32, each decoded start to end by one warp), so one-warp CTAs spread
    // them over all SMs
    const int W = STRIPES ? 1 : 8;
    const size_t smem = 128 * 32 * 8 + (size_t)(L.cols / 4) * NV * 4;
    if (smem > (size_t)max_smem_optin())
        return fail(MV_ERR_UNSUPPORTED, "AWR: %d columns x %d vectors exceed shared memory", L.cols, NV);
    auto kern = awr_kernel<NV, REQUANT, STRIPES>;
    int blocks_per_sm = 0;
    mv_status rc = prepare_kernel((const void *)kern, smem, 32 * W, &blocks_per_sm);
    if (rc) return rc;
    const int units = STRIPES ? L.rows / 32 : L.rows;
    const int want = (units + W - 1) / W;
    const int grid = std::max(1, std::min(want, std::max(1, blocks_per_sm) * sm_count()));
    kern<<<grid, 32 * W, smem, st>>>(L);
    MV_CUDA_TRY(cudaGetLastError(), "awr kernel launch");
    return MV_OK;
}

mv_status awr_common(const uint32_t *comp, size_t n_words, const uint32_t *offs, const uint32_t *ppf,
                     const uint32_t *cum, const uint32_t *prob, int rows, int cols, const int8_t *x,
                     AwrLaunch &L, bool stripes = false) {
    if (!comp || !offs || !ppf || !cum || !prob || !x) return fail(MV_ERR_ARG, "mv_awr: NULL pointer");
    if (rows <= 0 || cols <= 0) return fail(MV_ERR_ARG, "mv_awr: rows/cols must be positive");
    if (stripes) {
        if (rows % 32 || cols % 4)
            return fail(MV_ERR_SHAPE, "stripes layout needs rows %% 32 == 0 and cols %% 4 == 0 (%dx%d)", rows, cols);
    } else if (cols % 128) {
        return fail(MV_ERR_SHAPE, "AWR layout needs cols %% 128 == 0 (cols=%d)", cols);
    }
    if (((uintptr_t)comp & 15) != 0) return fail(MV_ERR_ARG, "mv_awr: compressed not 16-byte aligned");
    mv_status rc;
    L.status = device_status_word(&rc);
    if (rc) return rc;
    L.comp = reinterpret_cast<const uint4 *>(comp);
    L.n_u4 = n_words / 4;
    L.offs = offs;
    L.ppf = ppf;
    L.cum = cum;
    L.prob = prob;
    L.rows = rows;
    L.cols = cols;
    L.x = x;
    return MV_OK;
}

}  // namespace

mv_status awr_matvec(const uint32_t *comp, size_t n_words, const uint32_t *offs, const uint32_t *ppf,
                     const uint32_t *cum, const uint32_t *prob, int rows, int cols, const int8_t *x,
                     int batch, int32_t *y, const float *scales, float *ys, cudaStream_t st) {
    AwrLaunch L{};
    mv_status rc = awr_common(comp, n_words, offs, ppf, cum, prob, rows, cols, x, L);
    if (rc) return rc;
    if (!y || batch <= 0) return fail(MV_ERR_ARG, "mv_awr_matvec: bad y/batch");
    if (n_words == 0) return fail(MV_ERR_ARG, "mv_awr_matvec: n_words must be given");
    if (ys && !scales) return fail(MV_ERR_ARG, "mv_awr_matvec: y_scaled needs row scales");
    for (int v0 = 0; v0 < batch; v0 += 16) {
        const int nb = std::min(16, batch - v0);
        AwrLaunch P = L;
        P.x = x + (size_t)v0 * cols;
        P.batch = nb;
        P.y = y + (size_t)v0 * rows;
        P.scales = scales;
        P.ys = ys ? ys + (size_t)v0 * rows : nullptr;
        if (nb == 1) rc = launch_awr<1, false>(P, st);
        else if (nb == 2) rc = launch_awr<2, false>(P, st);
        else if (nb <= 4) rc = launch_awr<4, false>(P, st);
        else if (nb <= 8) rc = launch_awr<8, false>(P, st);
        else rc = launch_awr<16, false>(P, st);
        if (rc) return rc;
    }
    return MV_OK;
}

mv_status aws_matvec(const uint32_t *comp, size_t n_words, const uint32_t *offs, const uint32_t *ppf,
                     const uint32_t *cum, const uint32_t *prob, int rows, int cols, const int8_t *x,
                     int batch, int32_t *y, const float *scales, float *ys, cudaStream_t st) {
    AwrLaunch L{};
    mv_status rc = awr_common(comp, n_words, offs, ppf, cum, prob, rows, cols, x, L, true);
    if (rc) return rc;
    if (!y || batch <= 0) return fail(MV_ERR_ARG, "mv_aws_matvec: bad y/batch");
    if (n_words == 0) return fail(MV_ERR_ARG, "mv_aws_matvec: n_words must be given");
    if (ys && !scales) return fail(MV_ERR_ARG, "mv_aws_matvec: y_scaled needs row scales");
    for (int v0 = 0; v0 < batch; v0 += 16) {
        const int nb = std::min(16, batch - v0);
        AwrLaunch P = L;
        P.x = x + (size_t)v0 * cols;
        P.batch = nb;
        P.y = y + (size_t)v0 * rows;
        P.scales = scales;
        P.ys = ys ? ys + (size_t)v0 * rows : nullptr;
        if (nb == 1) rc = launch_awr<1, false, true>(P, st);
        else if (nb == 2) rc = launch_awr<2, false, true>(P, st);
        else if (nb <= 4) rc = launch_awr<4, false, true>(P, st);
        else if (nb <= 8) rc = launch_awr<8, false, true>(P, st);
        else rc = launch_awr<16, false, true>(P, st);
        if (rc) return rc;
    }
    return MV_OK;
}

mv_status aws_requant(const uint32_t *comp, size_t n_words, const uint32_t *offs, const uint32_t *ppf,
                      const uint32_t *cum, const uint32_t *prob, int rows, int cols, const int8_t *x,
                      float scale, int8_t *out8, cudaStream_t st) {
    AwrLaunch L{};
    mv_status rc = awr_common(comp, n_words, offs, ppf, cum, prob, rows, cols, x, L, true);
    if (rc) return rc;
    if (!out8) return fail(MV_ERR_ARG, "mv_aws_matvec_requant: NULL output");
    L.batch = 1;
    L.out8 = out8;
    L.scale = scale;
    return launch_awr<1, true, true>(L, st);
}

mv_status awr_requant(const uint32_t *comp, size_t n_words, const uint32_t *offs, const uint32_t *ppf,
                      const uint32_t *cum, const uint32_t *prob, int rows, int cols, const int8_t *x,
                      float scale, int8_t *out8, cudaStream_t st) {
    AwrLaunch L{};
    mv_status rc = awr_common(comp, n_words, offs, ppf, cum, prob, rows, cols, x, L);
    if (rc) return rc;
    if (!out8) return fail(MV_ERR_ARG, "mv_awr_matvec_requant: NULL output");
    L.batch = 1;
    L.out8 = out8;
    L.scale = scale;
    return launch_awr<1, true>(L, st);
}

}  // namespace mv

extern "C" {

mv_status mv_awr_matvec(const uint32_t *compressed_dev, size_t n_words, const uint32_t *warp_offsets_dev,
                        const uint32_t *ppf_dev, const uint32_t *ppf_cum_dev,
                        const uint32_t *ppf_prob_dev, int rows, int cols, const int8_t *x_dev,
                        int batch, int32_t *y_dev, const float *row_scales_dev, float *y_scaled_dev,
                        void *stream) {
    return mv::awr_matvec(compressed_dev, n_words, warp_offsets_dev, ppf_dev, ppf_cum_dev, ppf_prob_dev,
                          rows, cols, x_dev, batch, y_dev, row_scales_dev, y_scaled_dev,
                          (cudaStream_t)stream);
}

mv_status mv_awr_matvec_requant(const uint32_t *compressed_dev, size_t n_words,
                                const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                                const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev, int rows,
                                int cols, const int8_t *x_dev, float scale, int8_t *out8_dev,
                                void *stream) {
    return mv::awr_requant(compressed_dev, n_words, warp_offsets_dev, ppf_dev, ppf_cum_dev, ppf_prob_dev,
                           rows, cols, x_dev, scale, out8_dev, (cudaStream_t)stream);
}

// buffered/ans-warp-rows.cu:38-60: same arguments, same int8 output, legacy
// default stream.  The stream length is unknown here, so no bounds checks.
void mat_vec_mul_coalesced(const void *in_vector_gpu, void *out_vector_gpu, size_t in_dim, size_t out_dim,
                           float scale, const void *compressed, const uint32_t *warp_offsets,
                           const uint32_t *ppf, const uint32_t *ppf_cum, const uint32_t *ppf_prob) {
    mv_status rc = mv::awr_requant(reinterpret_cast<const uint32_t *>(compressed), 0, warp_offsets, ppf,
                                   ppf_cum, ppf_prob, (int)out_dim, (int)in_dim,
                                   reinterpret_cast<const int8_t *>(in_vector_gpu), scale,
                                   reinterpret_cast<int8_t *>(out_vector_gpu), 0);
    if (rc) std::fprintf(stderr, "mat_vec_mul_coalesced: %s\n", mv_last_error());
}

mv_status mv_aws_matvec(const uint32_t *compressed_dev, size_t n_words, const uint32_t *warp_offsets_dev,
                        const uint32_t *ppf_dev, const uint32_t *ppf_cum_dev,
                        const uint32_t *ppf_prob_dev, int rows, int cols, const int8_t *x_dev,
                        int batch, int32_t *y_dev, const float *row_scales_dev, float *y_scaled_dev,
                        void *stream) {
    return mv::aws_matvec(compressed_dev, n_words, warp_offsets_dev, ppf_dev, ppf_cum_dev, ppf_prob_dev,
                          rows, cols, x_dev, batch, y_dev, row_scales_dev, y_scaled_dev,
                          (cudaStream_t)stream);
}

mv_status mv_aws_matvec_requant(const uint32_t *compressed_dev, size_t n_words,
                                const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                                const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev, int rows,
                                int cols, const int8_t *x_dev, float scale, int8_t *out8_dev,
                                void *stream) {
    return mv::aws_requant(compressed_dev, n_words, warp_offsets_dev, ppf_dev, ppf_cum_dev, ppf_prob_dev,
                           rows, cols, x_dev, scale, out8_dev, (cudaStream_t)stream);
}

// buffered/ans-warp-stripes.cu:38-60 (the launcher of the stripes program, which has the same name as the
// rows program's; renamed here so that both live in one library): same arguments, same int8 output,
// legacy default stream, no bounds checks (the stream length is unknown).
void mat_vec_mul_coalesced_stripes(const void *in_vector_gpu, void *out_vector_gpu, size_t in_dim,
                                   size_t out_dim, float scale, const void *compressed,
                                   const uint32_t *warp_offsets, const uint32_t *ppf, const uint32_t *ppf_cum,
                                   const uint32_t *ppf_prob) {
    mv_status rc = mv::aws_requant(reinterpret_cast<const uint32_t *>(compressed), 0, warp_offsets, ppf,
                                   ppf_cum, ppf_prob, (int)out_dim, (int)in_dim,
                                   reinterpret_cast<const int8_t *>(in_vector_gpu), scale,
                                   reinterpret_cast<int8_t *>(out_vector_gpu), 0);
    if (rc) std::fprintf(stderr, "mat_vec_mul_coalesced_stripes: %s\n", mv_last_error());
}

}  // extern "C"
