// Q8-stripe decode + int8 matvec for sm_100a.
//
// Layout (built by host_q8.cpp): rows are grouped into stripes of 32, lane l
// of a warp owning row 32*stripe + l; each row is cut into segments of
// seg_quads quads (4 columns), and the (stripe, segment) pair is one block of
// 32 interleaved rANS streams (8-bit precision, four symbols per decode step,
// 64-bit state, 32-bit refill words).
//
// CTA = one stripe x W consecutive segments, one warp per segment:
//   1. lane 0 of every warp starts a 1-D bulk copy (cp.async.bulk, TMA engine)
//      of its block into its shared-memory buffer, completion on an mbarrier;
//   2. meanwhile the CTA builds the decode table: 256 quantiles x 32 lanes,
//      entry (q, l) at word q*32 + l, so lane l only ever touches bank l and the
//      four table reads per step are conflict-free even with one table per row;
//   3. x for the CTA's column range is staged as packed quads (broadcast reads);
//   4. each warp decodes its segment: refill (branch-free, one speculative
//      conflict-free shared load), 4 table reads, one 32x32->64 multiply-add for
//      the state update, one dp4a per vector;
//   5. per-row partial sums are reduced across the CTA's warps in shared
//      memory and written (or added with integer atomics, which are exact and
//      order-independent, when a row's segments span several CTAs).
#include <algorithm>
#include <cstdio>

#include "mv_device.cuh"

namespace mv {

struct Q8Launch {
    mv_q8_view m;
    const int8_t *x;       // [batch][cols]
    int batch;             // valid vectors in this pass (<= NV)
    int32_t *y;            // [*][rows], row stride ldy
    int ldy;
    int atomic;            // accumulate with atomicAdd (several CTAs per row)
    const float *scales;   // nullable
    float *ys;             // nullable, only written when !atomic
    int8_t *Wout;          // decode mode output (nullable)
    uint32_t *status;
    int buf_words;         // per-warp buffer, u32 words (multiple of 32)
    int range_quads;       // quads staged per CTA (= W * seg_quads)
    int xs_words;          // staged x words, rounded to a multiple of 4
    int tbl_stage;         // u16 table entries staged per CTA (multiple of 8)
    uint32_t spin_limit;   // barrier wait bound (iterations)
    int drop_copy;         // fault injection: do not issue the bulk copies
};

__device__ __forceinline__ uint32_t load_x_quad(const int8_t *x, int cols, int c, bool aligned) {
    const int col = 4 * c;
    if (aligned && col + 3 < cols) return *reinterpret_cast<const uint32_t *>(x + col);
    uint32_t v = 0;
    for (int j = 0; j < 4; j++)
        if (col + j < cols) v |= (uint32_t)(uint8_t)x[col + j] << (8 * j);
    return v;
}

template <int NV, bool DECODE>
__global__ void __launch_bounds__(512) q8_kernel(const Q8Launch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = blockDim.x >> 5;
    const mv_q8_view &m = L.m;

    uint32_t *lut = reinterpret_cast<uint32_t *>(smem);
    uint32_t *bufs = lut + 256 * 32;
    uint32_t *xs = bufs + W * L.buf_words;
    int *red = reinterpret_cast<int *>(xs + L.xs_words);
    uint64_t *bars = reinterpret_cast<uint64_t *>(red + (DECODE ? 0 : W * NV * 32));
    uint32_t *toff_s = reinterpret_cast<uint32_t *>(bars + W);  // [33]
    uint16_t *tsm = reinterpret_cast<uint16_t *>(toff_s + 36);  // [tbl_stage]

    const int stripe = blockIdx.x;
    const int seg = blockIdx.y * W + warp;
    const int qtot = (m.cols + 3) >> 2;
    const int qa = blockIdx.y * W * m.seg_quads;  // first quad of this CTA
    uint32_t *buf = bufs + warp * L.buf_words;

    // (1) start this warp's block copy
    uint32_t blk_rows = 0;
    if (seg < m.nseg) {
        const int b = stripe * m.nseg + seg;
        if (lane == 0) {
            const uint32_t o0 = __ldg(m.blk_off + b), o1 = __ldg(m.blk_off + b + 1);
            blk_rows = o1 - o0;
            if (o1 < o0 || o1 > m.blocks_rows || blk_rows < 2 || blk_rows > (uint32_t)m.max_blk_rows) {
                atomicOr(L.status, MV_DEV_STREAM_OVERRUN);
                blk_rows = 0;
            } else {
                mbar_init(&bars[warp], 1);
                fence_mbar_init();
                mbar_arrive_expect_tx(&bars[warp], blk_rows * 128u);
                if (!L.drop_copy) bulk_g2s(buf, m.blocks + (size_t)o0 * 32, blk_rows * 128u, &bars[warp]);
            }
        }
        blk_rows = __shfl_sync(0xffffffffu, blk_rows, 0);
    }

    // (2a) stage this stripe's tables (local: 32 consecutive row tables; global: one)
    {
        const uint32_t r0 = m.local ? (uint32_t)stripe * 32 : 0;
        const uint32_t nt = m.local ? 32 : 1;
        const uint32_t tb = __ldg(m.tbl_off + r0), te = __ldg(m.tbl_off + r0 + nt);
        const bool ok = te >= tb && te <= m.tbl_len && te - tb <= (uint32_t)L.tbl_stage;
        for (uint32_t i = threadIdx.x; i <= nt; i += blockDim.x) {
            const uint32_t o = __ldg(m.tbl_off + r0 + i);
            toff_s[i] = (ok && o >= tb && o <= te) ? o - tb : 0;
        }
        if (!ok && threadIdx.x == 0) atomicOr(L.status, MV_DEV_BAD_TABLE);
        const uint32_t n = ok ? te - tb : 0;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) tsm[i] = __ldg(m.tbl + tb + i);
    }
    // (3) stage x quads of this CTA's column range
    if (!DECODE) {
        const int nquads = min(L.range_quads, qtot - qa);
        const bool aligned = ((m.cols & 3) == 0) && ((reinterpret_cast<uintptr_t>(L.x) & 3) == 0);
        for (int i = threadIdx.x; i < L.xs_words; i += blockDim.x) {
            const int c = i / NV, v = i % NV;
            uint32_t val = 0;
            if (c < nquads && v < L.batch) val = load_x_quad(L.x + (size_t)v * m.cols, m.cols, qa + c, aligned);
            xs[i] = val;
        }
    }
    __syncthreads();

    // (2b) decode table: warp w fills quantiles [qlo, qhi) of all 32 rows from
    // the staged entries; lane = row, so every store hits the lane's own bank
    {
        const int t = m.local ? lane : 0;
        const uint32_t o0 = toff_s[t], o1 = max(toff_s[t + 1], o0);
        const int qlo = (256 * warp) / W, qhi = (256 * (warp + 1)) / W;
        uint32_t cum = 0;
        for (uint32_t k = o0; k < o1 && cum < (uint32_t)qhi; k++) {
            const uint32_t ent = tsm[k];
            const uint32_t f = ent >> 8, sym = ent & 0xFF;
            const uint32_t a = max(cum, (uint32_t)qlo), e = min(cum + f, (uint32_t)qhi);
            for (uint32_t q = a; q < e; q++) lut[q * 32 + lane] = sym | (f << 8) | ((q - cum) << 16);
            cum += f;
        }
        if (cum < (uint32_t)qhi) {  // table sums to less than 256: fill and flag
            for (uint32_t q = max(cum, (uint32_t)qlo); q < (uint32_t)qhi; q++) lut[q * 32 + lane] = 1u << 8;
            atomicOr(L.status, MV_DEV_BAD_TABLE);
        }
    }
    __syncthreads();

    int acc[NV > 0 ? NV : 1];
#pragma unroll
    for (int v = 0; v < (NV > 0 ? NV : 1); v++) acc[v] = 0;

    // (4) decode this warp's segment
    if (blk_rows) {
        if (!mbar_wait_bounded(&bars[warp], 0, L.status, L.spin_limit)) {
            mbar_wait_bounded(&bars[warp], 0, nullptr, L.spin_limit);  // let a late copy land before exit
        } else {
            uint32_t lo = buf[lane], hi = buf[32 + lane];
            uint32_t kidx = 64 + lane;
            const uint32_t kend = blk_rows * 32 + lane;
            const int q0 = seg * m.seg_quads;
            const int nq = min(m.seg_quads, qtot - q0);
            const uint32_t *lut_l = lut + lane;
            const uint32_t *xq = xs + (q0 - qa) * NV;
            const int row = stripe * 32 + lane;
            int8_t *wrow = DECODE ? L.Wout + (size_t)row * m.cols : nullptr;
            uint32_t P = 0;
#pragma unroll 2
            for (int i = 0; i < nq; i++) {
                const uint32_t w = buf[kidx];
                const bool need = (hi == 0);
                hi = need ? lo : hi;
                lo = need ? w : lo;
                kidx = need ? min(kidx + 32, kend) : kidx;
                const uint32_t e0 = lut_l[(lo & 0xFFu) << 5];
                const uint32_t e1 = lut_l[((lo >> 8) & 0xFFu) << 5];
                const uint32_t e2 = lut_l[((lo >> 16) & 0xFFu) << 5];
                const uint32_t e3 = lut_l[(lo >> 24) << 5];
                const uint32_t f0 = __byte_perm(e0, 0, 0x4441), f1 = __byte_perm(e1, 0, 0x4441);
                const uint32_t f2 = __byte_perm(e2, 0, 0x4441), f3 = __byte_perm(e3, 0, 0x4441);
                const uint32_t r0 = e0 >> 16, r1 = e1 >> 16, r2 = e2 >> 16, r3 = e3 >> 16;
                P = (f0 * f1) * (f2 * f3);
                const uint32_t ns = r0 + f0 * (r1 + f1 * (r2 + f2 * r3));
                const unsigned long long s = (unsigned long long)hi * P + ns;
                lo = (uint32_t)s;
                hi = (uint32_t)(s >> 32);
                const uint32_t wq =
                    __byte_perm(__byte_perm(e0, e1, 0x0040), __byte_perm(e2, e3, 0x0040), 0x5410);
                if (DECODE) {
                    if (row < m.rows) {
                        const int col = 4 * (q0 + i);
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            if (col + j < m.cols) wrow[col + j] = (int8_t)(wq >> (8 * j));
                    }
                } else if (NV == 1) {
                    acc[0] = __dp4a((int)wq, (int)xq[i], acc[0]);
                } else if (NV == 2) {
                    const uint2 xv = reinterpret_cast<const uint2 *>(xq)[i];
                    acc[0] = __dp4a((int)wq, (int)xv.x, acc[0]);
                    acc[1 % (NV > 0 ? NV : 1)] = __dp4a((int)wq, (int)xv.y, acc[1 % (NV > 0 ? NV : 1)]);
                } else {
#pragma unroll
                    for (int v4 = 0; v4 < NV / 4; v4++) {
                        const uint4 xv = reinterpret_cast<const uint4 *>(xq + i * NV)[v4];
                        acc[4 * v4 + 0] = __dp4a((int)wq, (int)xv.x, acc[4 * v4 + 0]);
                        acc[4 * v4 + 1] = __dp4a((int)wq, (int)xv.y, acc[4 * v4 + 1]);
                        acc[4 * v4 + 2] = __dp4a((int)wq, (int)xv.z, acc[4 * v4 + 2]);
                        acc[4 * v4 + 3] = __dp4a((int)wq, (int)xv.w, acc[4 * v4 + 3]);
                    }
                }
            }
            // the coder must end in its initial state (the last quad's probability product)
            if (nq > 0 && (hi != 0 || lo != P)) atomicOr(L.status, MV_DEV_FINAL_STATE);
        }
    }
    if (DECODE) return;

    // (5) reduce the W segment partials of each row
#pragma unroll
    for (int v = 0; v < (NV > 0 ? NV : 1); v++) red[(warp * NV + v) * 32 + lane] = acc[v];
    __syncthreads();
    for (int t = threadIdx.x; t < NV * 32; t += blockDim.x) {
        const int v = t >> 5, l = t & 31;
        int sum = 0;
        for (int w = 0; w < W; w++) sum += red[(w * NV + v) * 32 + l];
        const int row = stripe * 32 + l;
        if (row < m.rows && v < L.batch) {
            int32_t *dst = L.y + (size_t)v * L.ldy + row;
            if (L.atomic) {
                atomicAdd(dst, sum);
            } else {
                *dst = sum;
                if (L.ys) L.ys[(size_t)v * L.ldy + row] = (float)sum * L.scales[row];
            }
        }
    }
}

__global__ void scale_rows_kernel(const int32_t *y, const float *s, float *ys, int rows, int batch,
                                  int ldy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < rows * batch) {
        const int r = i % rows, v = i / rows;
        ys[(size_t)v * ldy + r] = (float)y[(size_t)v * ldy + r] * s[r];
    }
}

namespace {

int tbl_stage_entries(const mv_q8_view &m) { return (int)((m.tbl_stripe_max + 7) & ~7u); }

size_t q8_smem_bytes(const mv_q8_view &m, int W, int nv, bool decode) {
    const size_t range = (size_t)W * m.seg_quads;
    const size_t xs_words = decode ? 0 : ((range * nv + 3) & ~(size_t)3);
    return 256 * 32 * 4 + (size_t)W * (m.max_blk_rows + 1) * 32 * 4 + xs_words * 4 +
           (decode ? 0 : (size_t)W * nv * 32 * 4) + (size_t)W * 8 + 36 * 4 + (size_t)tbl_stage_entries(m) * 2;
}

template <int NV, bool DECODE>
mv_status launch_q8(const Q8Launch &base, int W, int ngroups, cudaStream_t st) {
    const mv_q8_view &m = base.m;
    Q8Launch L = base;
    L.range_quads = W * m.seg_quads;
    const int nvw = NV > 0 ? NV : 0;
    L.xs_words = DECODE ? 0 : ((L.range_quads * nvw + 3) & ~3);
    L.buf_words = (m.max_blk_rows + 1) * 32;
    L.tbl_stage = tbl_stage_entries(m);
    const size_t smem = q8_smem_bytes(m, W, nvw, DECODE);
    if (smem > (size_t)max_smem_optin())
        return fail(MV_ERR_UNSUPPORTED, "Q8 launch needs %zu B of shared memory (max %d)", smem,
                    max_smem_optin());
    auto kern = q8_kernel<NV, DECODE>;
    mv_status rc = prepare_kernel((const void *)kern, smem, 32 * W, nullptr);
    if (rc) return rc;
    const int stripes = (m.rows + 31) / 32;
    dim3 grid(stripes, ngroups), block(32 * W);
    kern<<<grid, block, smem, st>>>(L);
    MV_CUDA_TRY(cudaGetLastError(), "q8 kernel launch");
    return MV_OK;
}

mv_status check_view(const mv_q8_view *m) {
    if (!m || !m->blocks || !m->blk_off || !m->tbl || !m->tbl_off)
        return fail(MV_ERR_ARG, "mv_q8: NULL view or view pointer");
    if (m->rows <= 0 || m->cols <= 0 || m->seg_quads <= 0 || m->nseg <= 0 || m->max_blk_rows < 2)
        return fail(MV_ERR_ARG, "mv_q8: bad view dimensions");
    const int qtot = (m->cols + 3) / 4;
    if ((int64_t)m->seg_quads * m->nseg < qtot || (int64_t)m->seg_quads * (m->nseg - 1) >= qtot)
        return fail(MV_ERR_ARG, "mv_q8: nseg * seg_quads does not cover the columns");
    if (((uintptr_t)m->blocks & 15) != 0) return fail(MV_ERR_ARG, "mv_q8: blocks not 16-byte aligned");
    if (m->blocks_rows < 2 || m->tbl_len < 2) return fail(MV_ERR_ARG, "mv_q8: empty blocks or tables");
    if (m->tbl_stripe_max < 2 || m->tbl_stripe_max > 32 * 256)
        return fail(MV_ERR_ARG, "mv_q8: tbl_stripe_max out of range");
    return MV_OK;
}

// Warps (= segments) per CTA: up to 8, fewer when shared memory would not fit.
int pick_warps(const mv_q8_view &m, int nv, bool decode) {
    int W = std::max(1, std::min(m.nseg, 8));
    while (W > 1 && q8_smem_bytes(m, W, nv, decode) > (size_t)max_smem_optin()) W--;
    return W;
}

int nv_for(int nb) { return nb <= 2 ? nb : nb <= 4 ? 4 : nb <= 8 ? 8 : 16; }

}  // namespace

bool q8s_supports(const mv_q8_view *m, const int8_t *x);
mv_status q8s_matvec(const mv_q8_view *m, const int8_t *x, int batch, int32_t *y, const float *scales, float *ys,
                     const mv_q8_tuning *tuning, cudaStream_t st);

mv_status q8_matvec(const mv_q8_view *m, const int8_t *x, int batch, int32_t *y,
                    const float *scales, float *ys, cudaStream_t st) {
    mv_status rc = check_view(m);
    if (rc) return rc;
    if (!x || !y || batch <= 0) return fail(MV_ERR_ARG, "mv_q8_matvec: bad x/y/batch");
    if (ys && !scales) return fail(MV_ERR_ARG, "mv_q8_matvec: y_scaled needs row scales");
    if (q8s_supports(m, x)) return q8s_matvec(m, x, batch, y, scales, ys, nullptr, st);
    uint32_t *status = device_status_word(&rc);
    if (rc) return rc;
    for (int v0 = 0; v0 < batch; v0 += 16) {
        const int nb = std::min(16, batch - v0);
        const int W = pick_warps(*m, nv_for(nb), false);
        const int ngroups = (m->nseg + W - 1) / W;
        const bool atomic = ngroups > 1;
        Q8Launch L{};
        L.m = *m;
        L.x = x + (size_t)v0 * m->cols;
        L.batch = nb;
        L.y = y + (size_t)v0 * m->rows;
        L.ldy = m->rows;
        L.atomic = atomic;
        L.scales = scales;
        L.ys = (ys && !atomic) ? ys + (size_t)v0 * m->rows : nullptr;
        L.status = status;
        L.spin_limit = wait_spin_limit();
        L.drop_copy = inject_drop_copy();
        if (atomic)
            MV_CUDA_TRY(cudaMemsetAsync(L.y, 0, sizeof(int32_t) * (size_t)nb * m->rows, st),
                        "cudaMemsetAsync(y)");
        if (nb == 1) rc = launch_q8<1, false>(L, W, ngroups, st);
        else if (nb == 2) rc = launch_q8<2, false>(L, W, ngroups, st);
        else if (nb <= 4) rc = launch_q8<4, false>(L, W, ngroups, st);
        else if (nb <= 8) rc = launch_q8<8, false>(L, W, ngroups, st);
        else rc = launch_q8<16, false>(L, W, ngroups, st);
        if (rc) return rc;
        if (ys && atomic) {
            const int n = nb * m->rows;
            scale_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(L.y, scales, ys + (size_t)v0 * m->rows,
                                                               m->rows, nb, m->rows);
            MV_CUDA_TRY(cudaGetLastError(), "scale_rows_kernel launch");
        }
    }
    return MV_OK;
}

mv_status q8_decode(const mv_q8_view *m, int8_t *W_out, cudaStream_t st) {
    mv_status rc = check_view(m);
    if (rc) return rc;
    if (!W_out) return fail(MV_ERR_ARG, "mv_q8_decode: NULL output");
    uint32_t *status = device_status_word(&rc);
    if (rc) return rc;
    const int W = pick_warps(*m, 0, true);
    Q8Launch L{};
    L.m = *m;
    L.Wout = W_out;
    L.status = status;
    L.spin_limit = wait_spin_limit();
    L.drop_copy = inject_drop_copy();
    return launch_q8<0, true>(L, W, (m->nseg + W - 1) / W, st);
}

}  // namespace mv

extern "C" {

mv_status mv_q8_matvec(const mv_q8_view *m, const int8_t *x_dev, int batch, int32_t *y_dev,
                       const float *row_scales_dev, float *y_scaled_dev, void *stream) {
    return mv::q8_matvec(m, x_dev, batch, y_dev, row_scales_dev, y_scaled_dev, (cudaStream_t)stream);
}

mv_status mv_q8_decode(const mv_q8_view *m, int8_t *W_dev, void *stream) {
    return mv::q8_decode(m, W_dev, (cudaStream_t)stream);
}

}  // extern "C"
