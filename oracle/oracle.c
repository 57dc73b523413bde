/*
 * oracle.c -- CPU restatement of the reference's entropy-coded matvec path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the product library
 * (matvans_b200/) never links it, and only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs load it.
 *
 * What is restated, and from where (paths are within the reference project):
 *   - hash_int8_array            buffered/encoder.py:8-20 (C++ twin ans-warp-rows.cu:62-73)
 *   - AWR decode ("ans-warp-rows" layout, 7-bit quad rANS, warp-shared word
 *     stream refilled through __ballot_sync/__popc/__shfl_sync)
 *                                buffered/ans-warp-rows-kernel.cu:20-204
 *                                layout from buffered/encoder.py:394-461
 *                                tables from buffered/encoder.py:309-320, 464-470
 *   - WPR decode ("matvansWarpPerRow" layout, 8-bit rANS, per-lane u16 queues)
 *                                matvansWarpPerRow/matvansWarpPerRow-kernel.cu:46-175
 *                                layout from create_matrices_WarpPerRow.py:353-430
 *   - int8 matvec with int64 accumulation (the lossless-coding oracle for y)
 *
 * The multithreaded *_matvec_mt entry points fuse decode and dot product per
 * row and are what bench.py times as the CPU baseline.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <pthread.h>

#define ORC_OK 0
#define ORC_ERR_BOUNDS 1
#define ORC_ERR_SHAPE 2
#define ORC_ERR_MODEL 3
#define ORC_ERR_OVERFLOW 4

/* ------------------------------------------------------------------ hash */

/* FxHash-style hash of the final int8 vector: buffered/encoder.py:8-20. */
uint32_t orc_hash_int8(const int8_t *a, int64_t n)
{
    uint32_t h = 0;
    for (int64_t i = 0; i < n; i++) {
        h = (h >> 27) | (h << 5);
        h = (h ^ (uint32_t)(uint8_t)a[i]) * 0x27220A95u;
    }
    return h;
}

/* ---------------------------------------------------------- int8 matvec */

/* y[b][r] = sum_c W[r][c] * x[b][c], accumulated in int64 and checked to fit
 * int32 (the reference kernels accumulate in int32, ans-warp-rows-kernel.cu:191). */
int orc_matvec_i8(const int8_t *W, int64_t rows, int64_t cols, const int8_t *x,
                  int batch, int32_t *y)
{
    int bad = 0;
    for (int b = 0; b < batch; b++) {
        const int8_t *xb = x + (int64_t)b * cols;
        for (int64_t r = 0; r < rows; r++) {
            const int8_t *w = W + r * cols;
            int64_t acc = 0;
            for (int64_t c = 0; c < cols; c++) acc += (int64_t)w[c] * xb[c];
            if (acc > INT32_MAX || acc < INT32_MIN) bad = 1;
            y[(int64_t)b * rows + r] = (int32_t)acc;
        }
    }
    return bad ? ORC_ERR_OVERFLOW : ORC_OK;
}

/* ============================================================ AWR decode */

/* One quantile -> (symbol, left cumulative, probability) from the packed
 * tables: entry q>>2 of each u32[32] table, byte q&3 (little endian), exactly
 * as ans-warp-rows-kernel.cu:147-189 reads them through __shfl_sync. */
static inline void awr_lookup(const uint32_t *ppf, const uint32_t *cum,
                              const uint32_t *prob, uint32_t q,
                              int8_t *sym, uint32_t *c, uint32_t *p)
{
    uint32_t hi = q >> 2, sh = 8 * (q & 3);
    *sym = (int8_t)(uint8_t)(ppf[hi] >> sh);
    *c = (uint8_t)(cum[hi] >> sh);
    *p = (uint8_t)(prob[hi] >> sh);
}

typedef struct { uint32_t x, y, z, w; } orc_u4;

static inline orc_u4 awr_load_u4(const uint32_t *comp, int64_t n_words, int64_t word_idx)
{
    orc_u4 v = {0, 0, 0, 0};
    if (word_idx >= 0 && word_idx + 3 < n_words) {
        v.x = comp[word_idx];
        v.y = comp[word_idx + 1];
        v.z = comp[word_idx + 2];
        v.w = comp[word_idx + 3];
    }
    return v;
}

/* Decode one AWR row (the warp simulation of ans-warp-rows-kernel.cu:63-204).
 * `row_u4` is warp_offsets[row] (uint4 units).  Decoded symbols go to `w_out`
 * (length cols) if non-NULL; the dot products with `batch` vectors of x go to
 * `acc_out[b]` if non-NULL.  Reads past the end of `comp` (which the reference
 * kernel can issue when the warp cache reload lands exactly on a 128-word
 * boundary, ans-warp-rows-kernel.cu:103-111) return zeros; such words are
 * never consumed. */
/* stripes = 0: one AWR row (lane l holds the quad at columns 4(j+l)..+3 of step j, all lanes feed
 * acc_out[b]); stripes = 1: one "ans-warp-stripes" stripe of 32 rows (ans-warp-stripes-kernel.cu:21-227,
 * layout encoder.py:323-391): lane l is row l of the stripe and decodes its quad j (columns 4j..4j+3) at
 * step j, w_out is [32][cols] and acc_out [32][batch].  The word stream, its 128-word cache and the
 * lane-order refills are the same in both layouts. */
static int awr_row_x(const uint32_t *comp, int64_t n_words, uint32_t row_u4, int64_t cols,
                     const uint32_t *ppf, const uint32_t *cum, const uint32_t *prob,
                     int8_t *w_out, const int8_t *x, int batch, int64_t *acc_out, int stripes)
{
    int64_t cursor = (int64_t)row_u4 * 4;   /* word index of the next 128-word block */
    if (cursor + 128 > n_words) return ORC_ERR_BOUNDS;
    orc_u4 cache[32];
    uint64_t state[32];
    for (int l = 0; l < 32; l++) {
        cache[l] = awr_load_u4(comp, n_words, cursor + 4 * l);
        state[l] = ((uint64_t)cache[l].w << 32) | cache[l].z;
    }
    cursor += 128;
    uint32_t wcc = 64;
    const int64_t quads = cols / 4;
    if (acc_out) for (int b = 0; b < (stripes ? 32 * batch : batch); b++) acc_out[b] = 0;

    for (int64_t j = 0; j < quads; j += (stripes ? 1 : 32)) {
        uint32_t ballot = 0;
        for (int l = 0; l < 32; l++)
            if ((state[l] >> 32) == 0) ballot |= 1u << l;
        if (ballot) {
            uint32_t num = (uint32_t)__builtin_popcount(ballot);
            uint32_t rv[32];
            uint32_t lc[32];
            uint32_t off[32];
            for (int l = 0; l < 32; l++) {
                off[l] = (uint32_t)__builtin_popcount(ballot & ((1u << l) - 1u));
                lc[l] = (wcc + off[l]) % 32;
            }
            for (int l = 0; l < 32; l++) rv[l] = cache[lc[l]].x;
            if ((wcc + num) / 32 != wcc / 32) {
                if (wcc / 32 == 3) {
                    for (int l = 0; l < 32; l++) cache[l] = awr_load_u4(comp, n_words, cursor + 4 * l);
                    cursor += 128;
                } else {
                    for (int l = 0; l < 32; l++) {
                        cache[l].x = cache[l].y;
                        cache[l].y = cache[l].z;
                        cache[l].z = cache[l].w;
                    }
                }
                for (int l = 0; l < 32; l++)
                    if ((wcc + off[l]) / 32 != wcc / 32) rv[l] = cache[lc[l]].x;
            }
            for (int l = 0; l < 32; l++)
                if (ballot & (1u << l)) state[l] = (state[l] << 32) | rv[l];
            wcc = (wcc + num) % 128;
        }
        for (int l = 0; l < 32; l++) {
            uint64_t s = state[l];
            int8_t sym[4];
            uint32_t c[4], p[4], rem[4];
            for (int i = 0; i < 4; i++) {
                uint32_t q = (uint32_t)(s >> (7 * i)) & 0x7F;
                awr_lookup(ppf, cum, prob, q, &sym[i], &c[i], &p[i]);
                rem[i] = q - c[i];
            }
            uint32_t p01 = p[0] * p[1], p012 = p01 * p[2], p0123 = p012 * p[3];
            uint32_t ns = rem[0] + p[0] * rem[1] + p01 * rem[2] + p012 * rem[3];
            state[l] = (s >> 28) * (uint64_t)p0123 + (uint64_t)ns;
            const int64_t col = stripes ? 4 * j : 4 * (j + l);
            if (w_out) for (int i = 0; i < 4; i++) w_out[(stripes ? l * cols : 0) + col + i] = sym[i];
            if (acc_out)
                for (int b = 0; b < batch; b++) {
                    const int8_t *xb = x + (int64_t)b * cols + col;
                    acc_out[stripes ? l * batch + b : b] +=
                        (int64_t)sym[0] * xb[0] + (int64_t)sym[1] * xb[1] + (int64_t)sym[2] * xb[2] +
                        (int64_t)sym[3] * xb[3];
                }
        }
    }
    return ORC_OK;
}

static int awr_row(const uint32_t *comp, int64_t n_words, uint32_t row_u4, int64_t cols,
                   const uint32_t *ppf, const uint32_t *cum, const uint32_t *prob,
                   int8_t *w_out, const int8_t *x, int batch, int64_t *acc_out)
{
    return awr_row_x(comp, n_words, row_u4, cols, ppf, cum, prob, w_out, x, batch, acc_out, 0);
}

/* Decode a whole "ans-warp-stripes" matrix to int8 W[rows][cols] (rows % 32 == 0, cols % 4 == 0,
 * buffered/encoder.py:326-327; warp_offsets: one per stripe, in uint4 units). */
int orc_aws_decode(const uint32_t *comp, int64_t n_words, const uint32_t *warp_offsets,
                   int64_t rows, int64_t cols, const uint32_t *ppf, const uint32_t *cum,
                   const uint32_t *prob, int8_t *W)
{
    if (rows % 32 != 0 || cols % 4 != 0) return ORC_ERR_SHAPE;
    for (int64_t s = 0; s < rows / 32; s++) {
        int rc = awr_row_x(comp, n_words, warp_offsets[s], cols, ppf, cum, prob, W + s * 32 * cols,
                           NULL, 0, NULL, 1);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* Fused "ans-warp-stripes" decode + int8 dot products (single thread): x [batch][cols], y [batch][rows]. */
int orc_aws_matvec(const uint32_t *comp, int64_t n_words, const uint32_t *warp_offsets,
                   int64_t rows, int64_t cols, const uint32_t *ppf, const uint32_t *cum,
                   const uint32_t *prob, const int8_t *x, int batch, int32_t *y)
{
    if (rows % 32 != 0 || cols % 4 != 0) return ORC_ERR_SHAPE;
    if (batch < 1 || batch > 64) return ORC_ERR_SHAPE;
    int64_t acc[32 * 64];
    for (int64_t s = 0; s < rows / 32; s++) {
        int rc = awr_row_x(comp, n_words, warp_offsets[s], cols, ppf, cum, prob, NULL, x, batch, acc, 1);
        if (rc) return rc;
        for (int l = 0; l < 32; l++)
            for (int b = 0; b < batch; b++) y[(int64_t)b * rows + s * 32 + l] = (int32_t)acc[l * batch + b];
    }
    return ORC_OK;
}

/* Decode a whole AWR matrix to int8 W[rows][cols]. */
int orc_awr_decode(const uint32_t *comp, int64_t n_words, const uint32_t *warp_offsets,
                   int64_t rows, int64_t cols, const uint32_t *ppf, const uint32_t *cum,
                   const uint32_t *prob, int8_t *W)
{
    if (cols % 128 != 0) return ORC_ERR_SHAPE;   /* buffered/encoder.py:397 */
    for (int64_t r = 0; r < rows; r++) {
        int rc = awr_row(comp, n_words, warp_offsets[r], cols, ppf, cum, prob,
                         W + r * cols, NULL, 0, NULL);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* ============================================================ WPR decode */

/* Decode one WPR row (matvansWarpPerRow-kernel.cu:95-159).  Lane l's u16 word k
 * lives at payload[cursor + (k/8)*256 + l*8 + k%8] (create_matrices_WarpPerRow.py:405-420);
 * the ring queue of the reference only changes *when* words are fetched, not
 * which word each lane consumes, so the lane walk reads its words directly. */
static int wpr_row(const uint16_t *payload, int64_t payload_size, uint32_t cursor,
                   int64_t cols, int8_t min_value, const uint8_t *cdf, int G,
                   const uint8_t *ppf, int8_t *w_out, const int8_t *x, int batch,
                   int64_t *acc_out)
{
    if (acc_out) for (int b = 0; b < batch; b++) acc_out[b] = 0;
    for (int l = 0; l < 32; l++) {
        int64_t k = 0;
#define WPR_WORD(kk) ( ((int64_t)cursor + ((kk) / 8) * 256 + l * 8 + (kk) % 8) )
        int64_t i0 = WPR_WORD(0), i1 = WPR_WORD(1);
        if (i1 >= payload_size) return ORC_ERR_BOUNDS;
        uint32_t head = ((uint32_t)payload[i0] << 16) | payload[i1];
        k = 2;
        for (int64_t j = 0; j < cols / 32; j++) {
            uint32_t q = head & 0xFF;
            uint32_t r = ppf[q];
            if ((int)r + 1 > G) return ORC_ERR_MODEL;
            int8_t w = (int8_t)(min_value + (int)r);
            uint32_t prob = ((uint32_t)cdf[r + 1] - (uint32_t)cdf[r]) & 0xFF;
            head = (head >> 8) * prob + (q - cdf[r]);
            int64_t col = 512 * (j / 16) + 16 * l + j % 16;
            if (w_out) w_out[col] = w;
            if (acc_out)
                for (int b = 0; b < batch; b++) acc_out[b] += (int64_t)w * x[(int64_t)b * cols + col];
            if (head < (1u << 16)) {
                int64_t idx = WPR_WORD(k);
                if (idx >= payload_size) return ORC_ERR_BOUNDS;
                head = (head << 16) | payload[idx];
                k++;
            }
        }
#undef WPR_WORD
    }
    return ORC_OK;
}

int orc_wpr_decode(const uint16_t *payload, int64_t payload_size, const uint32_t *cursors,
                   int64_t rows, int64_t cols, int8_t min_value, const uint8_t *cdf, int G,
                   const uint8_t *ppf, int8_t *W)
{
    if (cols % 512 != 0) return ORC_ERR_SHAPE;
    for (int64_t r = 0; r < rows; r++) {
        int rc = wpr_row(payload, payload_size, cursors[r], cols, min_value, cdf, G, ppf,
                         W + r * cols, NULL, 0, NULL);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* ===================================================== threaded matvec */

typedef struct {
    int kind;  /* 0 = AWR, 1 = WPR */
    int64_t rows, cols;
    int batch;
    const int8_t *x;
    int32_t *y;
    /* AWR */
    const uint32_t *comp; int64_t n_words; const uint32_t *offsets;
    const uint32_t *ppf32, *cum32, *prob32;
    /* WPR */
    const uint16_t *payload; int64_t payload_size; const uint32_t *cursors;
    int8_t min_value; const uint8_t *cdf; int G; const uint8_t *ppf8;
    int64_t r0, r1;
    int rc;
} orc_job;

static void *orc_worker(void *arg)
{
    orc_job *jb = (orc_job *)arg;
    int64_t acc[64];
    for (int64_t r = jb->r0; r < jb->r1; r++) {
        int rc = jb->kind == 0
            ? awr_row(jb->comp, jb->n_words, jb->offsets[r], jb->cols, jb->ppf32, jb->cum32,
                      jb->prob32, NULL, jb->x, jb->batch, acc)
            : wpr_row(jb->payload, jb->payload_size, jb->cursors[r], jb->cols, jb->min_value,
                      jb->cdf, jb->G, jb->ppf8, NULL, jb->x, jb->batch, acc);
        if (rc) { jb->rc = rc; return NULL; }
        for (int b = 0; b < jb->batch; b++) jb->y[(int64_t)b * jb->rows + r] = (int32_t)acc[b];
    }
    return NULL;
}

static int orc_run(orc_job *base, int nthreads)
{
    if (base->batch < 1 || base->batch > 64) return ORC_ERR_SHAPE;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    orc_job jobs[256];
    pthread_t th[256];
    int64_t per = (base->rows + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = *base;
        jobs[t].r0 = t * per < base->rows ? t * per : base->rows;
        jobs[t].r1 = (t + 1) * per < base->rows ? (t + 1) * per : base->rows;
        jobs[t].rc = 0;
        pthread_create(&th[t], NULL, orc_worker, &jobs[t]);
    }
    int rc = 0;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        if (jobs[t].rc) rc = jobs[t].rc;
    }
    return rc;
}

/* Fused decode + int8 dot products, rows split over `nthreads` threads.
 * x is [batch][cols], y is [batch][rows]. */
int orc_awr_matvec_mt(const uint32_t *comp, int64_t n_words, const uint32_t *warp_offsets,
                      int64_t rows, int64_t cols, const uint32_t *ppf, const uint32_t *cum,
                      const uint32_t *prob, const int8_t *x, int batch, int32_t *y, int nthreads)
{
    if (cols % 128 != 0) return ORC_ERR_SHAPE;
    orc_job jb;
    memset(&jb, 0, sizeof jb);
    jb.kind = 0; jb.rows = rows; jb.cols = cols; jb.batch = batch; jb.x = x; jb.y = y;
    jb.comp = comp; jb.n_words = n_words; jb.offsets = warp_offsets;
    jb.ppf32 = ppf; jb.cum32 = cum; jb.prob32 = prob;
    return orc_run(&jb, nthreads);
}

int orc_wpr_matvec_mt(const uint16_t *payload, int64_t payload_size, const uint32_t *cursors,
                      int64_t rows, int64_t cols, int8_t min_value, const uint8_t *cdf, int G,
                      const uint8_t *ppf, const int8_t *x, int batch, int32_t *y, int nthreads)
{
    if (cols % 512 != 0) return ORC_ERR_SHAPE;
    orc_job jb;
    memset(&jb, 0, sizeof jb);
    jb.kind = 1; jb.rows = rows; jb.cols = cols; jb.batch = batch; jb.x = x; jb.y = y;
    jb.payload = payload; jb.payload_size = payload_size; jb.cursors = cursors;
    jb.min_value = min_value; jb.cdf = cdf; jb.G = G; jb.ppf8 = ppf;
    return orc_run(&jb, nthreads);
}

/* ------------------------------------------------------------ AWR encoder */

/*
 * The reference's ans-warp-rows encoder, restated so that the CPU legs of the
 * benchmark can build their inputs without the product library:
 *   fit_128bit_encoder_model           buffered/encoder.py:271-306
 *   DetachedAnsQuadCoder.encode        buffered/encoder.py:190-226
 *   compress_ans_warp_rows(matrix, 32) buffered/encoder.py:394-461
 *   decoder tables + pack_4bytes       buffered/encoder.py:309-320, 464-470
 * Output is byte-identical to the reference encoder (tests/golden/awr_cases.npz).
 * *comp_out is malloc'd (free with orc_free); offsets has `rows` entries (uint4
 * units); ppf/cum/prob are u32[32] each.
 */
static int awr_fit(const int8_t *W, int64_t n, int *min_value, uint8_t *cdf, int *ncdf)
{
    int64_t hist[256];
    memset(hist, 0, sizeof hist);
    for (int64_t i = 0; i < n; i++) hist[(uint8_t)W[i] ^ 0x80]++;
    int vals[256], nv = 0;
    for (int v = 0; v < 256; v++)
        if (hist[v]) vals[nv++] = v;
    if (nv > 128) return ORC_ERR_MODEL;  /* encoder.py:303: at most 128 values */
    /* pmf = max(1, round(float32(count) * 128 / numel)) in float32, half to even (encoder.py:278-280) */
    uint32_t pmf[256];
    const float numel = (float)n;
    uint64_t sum = 0;
    for (int i = 0; i < nv; i++) {
        volatile float t = (float)hist[vals[i]] * 128.0f;
        volatile float q = t / numel;
        uint32_t u = (uint32_t)nearbyintf(q);
        pmf[i] = u < 1 ? 1 : u;
        sum += pmf[i];
    }
    /* force the sum to 128 one unit at a time on the first maximal entry (encoder.py:281-287) */
    while (sum != 128) {
        int best = 0;
        for (int i = 1; i < nv; i++)
            if (pmf[i] > pmf[best]) best = i;
        if (sum > 128) { pmf[best]--; sum--; } else { pmf[best]++; sum++; }
    }
    /* cdf over min..max+1 with absent values given zero width (encoder.py:294-304) */
    const int minv = vals[0] - 128, maxv = vals[nv - 1] - 128;
    *min_value = minv;
    *ncdf = maxv - minv + 2;
    memset(cdf, 0, (size_t)*ncdf);
    uint32_t left = 0;
    int last = 0;
    for (int i = 0; i < nv; i++) {
        const int idx = vals[i] - 128 - minv;
        for (int k = last + 1; k < idx + 1; k++) cdf[k] = (uint8_t)left;
        last = idx;
        left += pmf[i];
    }
    cdf[*ncdf - 1] = 128;
    return ORC_OK;
}

typedef struct { uint32_t *w; int64_t n, cap; } orc_vec;

static int vec_push(orc_vec *v, uint32_t x)
{
    if (v->n == v->cap) {
        int64_t cap = v->cap ? 2 * v->cap : 1024;
        uint32_t *p = (uint32_t *)realloc(v->w, (size_t)cap * 4);
        if (!p) return ORC_ERR_OVERFLOW;
        v->w = p;
        v->cap = cap;
    }
    v->w[v->n++] = x;
    return ORC_OK;
}

int orc_awr_encode(const int8_t *W, int64_t rows, int64_t cols, uint32_t **comp_out, int64_t *n_words,
                   uint32_t *offsets, uint32_t *ppf, uint32_t *cum, uint32_t *prob)
{
    if (cols % 128 != 0 || rows <= 0) return ORC_ERR_SHAPE;
    int minv = 0, ncdf = 0;
    uint8_t cdf[260];
    int rc = awr_fit(W, rows * cols, &minv, cdf, &ncdf);
    if (rc) return rc;
    orc_vec out = {0, 0, 0}, buf = {0, 0, 0};
    uint32_t *un = NULL;
    int64_t un_cap = 0;
    uint64_t state[32];
    memset(state, 0, sizeof state);  /* the 32 coders carry their states from row to row (encoder.py:402) */
    for (int64_t r = 0; r < rows && !rc; r++) {
        if (out.n / 4 > 0xFFFFFFFFll) { rc = ORC_ERR_OVERFLOW; break; }
        offsets[r] = (uint32_t)(out.n / 4);
        buf.n = 0;
        const int8_t *row = W + r * cols;
        for (int64_t c = cols / 128 - 1; c >= 0 && !rc; c--)
            for (int l = 31; l >= 0 && !rc; l--) {
                const int8_t *qd = row + 128 * c + 4 * l;
                uint32_t lft[4], p[4];
                uint64_t total = 1;
                for (int i = 0; i < 4; i++) {
                    const int idx = qd[i] - minv;
                    lft[i] = cdf[idx];
                    p[i] = (uint32_t)cdf[idx + 1] - lft[i];
                    total *= p[i];
                }
                uint64_t s = state[l];
                if ((s >> 36) >= total) {  /* flush one word (encoder.py:208-211) */
                    rc = vec_push(&buf, (uint32_t)s);
                    s >>= 32;
                } else if (s == 0) {       /* first quad of the coder (encoder.py:212-217) */
                    s = total << 4;
                }
                uint64_t concat = 0;
                for (int i = 0; i < 4; i++) {
                    const uint64_t rem = s % p[i];
                    s /= p[i];
                    concat |= (uint64_t)(lft[i] + rem) << (7 * i);
                }
                state[l] = (s << 28) | concat;
            }
        /* per row (encoder.py:431-447): reverse, pad to 64 (mod 128), state words at 64, transpose blocks */
        const int64_t nb = buf.n;
        const int64_t pad = ((64 - nb) % 128 + 128) % 128;
        const int64_t tot = nb + pad + 64;
        if (tot > un_cap) {
            uint32_t *p = (uint32_t *)realloc(un, (size_t)tot * 4);
            if (!p) { rc = ORC_ERR_OVERFLOW; break; }
            un = p;
            un_cap = tot;
        }
        int64_t k = 0;
        for (int64_t i = 0; i < 64; i++) un[k++] = i < nb ? buf.w[nb - 1 - i] : 0u;
        for (int l = 0; l < 32; l++) un[k++] = (uint32_t)state[l];
        for (int l = 0; l < 32; l++) un[k++] = (uint32_t)(state[l] >> 32);
        for (int64_t i = 64; i < nb + pad; i++) un[k++] = i < nb ? buf.w[nb - 1 - i] : 0u;
        for (int64_t b = 0; b < tot / 128 && !rc; b++)
            for (int l = 0; l < 32 && !rc; l++)
                for (int f = 0; f < 4 && !rc; f++) rc = vec_push(&out, un[b * 128 + f * 32 + l]);
    }
    free(un);
    free(buf.w);
    if (rc) { free(out.w); return rc; }
    /* decoder tables (encoder.py:309-320), packed 4 bytes per word little-endian (:464-470) */
    uint8_t p8[128], c8[128], r8[128];
    memset(p8, 0, sizeof p8); memset(c8, 0, sizeof c8); memset(r8, 0, sizeof r8);
    for (int idx = 0; idx + 1 < ncdf; idx++)
        for (uint32_t q = cdf[idx]; q < cdf[idx + 1]; q++) {
            p8[q] = (uint8_t)(int8_t)(idx + minv);
            c8[q] = cdf[idx];
            r8[q] = (uint8_t)(cdf[idx + 1] - cdf[idx]);
        }
    for (int i = 0; i < 32; i++) {
        ppf[i] = cum[i] = prob[i] = 0;
        for (int b = 0; b < 4; b++) {
            ppf[i] |= (uint32_t)p8[4 * i + b] << (8 * b);
            cum[i] |= (uint32_t)c8[4 * i + b] << (8 * b);
            prob[i] |= (uint32_t)r8[4 * i + b] << (8 * b);
        }
    }
    *comp_out = out.w;
    *n_words = out.n;
    return ORC_OK;
}

void orc_free(void *p) { free(p); }
