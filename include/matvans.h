/*
 * matvans.h -- C ABI of the B200 entropy-coded int8 matrix-vector product.
 *
 * An int8 weight matrix is stored as interleaved rANS streams and decoded
 * inside the matvec kernel, so it never exists uncompressed in device memory.
 * Three stream layouts are supported:
 *
 *   AWR  "ans-warp-rows": the reference's safetensors layout (7-bit quad rANS,
 *        64-bit state, 32 lanes per row sharing one word stream), written by
 *        buffered/encoder.py:394-511 and decoded by
 *        buffered/ans-warp-rows-kernel.cu:7-221.
 *   WPR  "matvansWarpPerRow": the reference's .bin layout (8-bit rANS, 32-bit
 *        head, 16-bit words, one stream per lane), written by
 *        matvansWarpPerRow/create_matrices_WarpPerRow.py:353-461 and decoded by
 *        matvansWarpPerRow/matvansWarpPerRow-kernel.cu:46-175.
 *   Q8   this library's own stripe layout (8-bit quad rANS with a 64-bit state;
 *        lane = row of a 32-row stripe, rows cut into column segments; one
 *        global table or one table per row).  No reference counterpart.
 *
 * Conventions
 *   - Every function returns mv_status (0 = MV_OK); on failure
 *     mv_last_error() returns a message for the calling thread.
 *   - All pointers named *_dev are device pointers owned by the caller; the
 *     library does not allocate on the launch paths except one lazily created
 *     per-device status word (see mv_device_status).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *   - x is [batch][cols] int8 row-major; y is [batch][rows] int32.  y is
 *     exact: decoded weights times x accumulated in int32.  y_scaled, when
 *     non-NULL, is [batch][rows] float with y_scaled = (float)y * scale[row].
 *   - Launches are asynchronous; device-side stream checks (overrun, final
 *     state mismatch, wait timeout) raise bits in the per-device status word,
 *     read and cleared by mv_device_status().
 */
#ifndef MATVANS_H
#define MATVANS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mv_status;
#define MV_OK 0
#define MV_ERR_ARG 1          /* invalid argument: NULL pointer, bad size      */
#define MV_ERR_SHAPE 2        /* shape not representable in the layout         */
#define MV_ERR_FORMAT 3       /* malformed file, tensor or stream              */
#define MV_ERR_IO 4           /* file could not be read or written             */
#define MV_ERR_CUDA 5         /* a CUDA runtime call failed                    */
#define MV_ERR_DEVICE 6       /* a device-side check failed                    */
#define MV_ERR_NOMEM 7        /* host allocation failed                        */
#define MV_ERR_UNSUPPORTED 8  /* valid request this build does not implement   */

/* Device status bits (mv_device_status). */
#define MV_DEV_STREAM_OVERRUN 0x1u   /* a lane consumed more words than its stream holds */
#define MV_DEV_FINAL_STATE 0x2u      /* a coder did not end in its initial state        */
#define MV_DEV_WAIT_TIMEOUT 0x4u     /* a bounded wait on a copy or queue gave up       */
#define MV_DEV_BAD_TABLE 0x8u        /* a probability table does not sum to 2^precision */

const char *mv_version(void);
const char *mv_last_error(void);

/* Synchronises `stream`, then reads and clears the status word of the current
 * device.  *flags receives the MV_DEV_* bits raised since the last call. */
mv_status mv_device_status(void *stream, uint32_t *flags);

/* ------------------------------------------------------------------ AWR --- */

/* Replaces the host launcher mat_vec_mul_coalesced of
 * buffered/ans-warp-rows.cu:38-60 (kernel signature ans-warp-rows-kernel.cu:7-17)
 * with identical arguments and output: one int8 per row,
 * clamp(round_half_even((float)y * scale)) as in ans-warp-rows-kernel.cu:212-220.
 * Like the reference it returns nothing; errors print to stderr and are kept
 * for mv_last_error().  Launches on the legacy default stream. */
void mat_vec_mul_coalesced(const void *in_vector_gpu, void *out_vector_gpu, size_t in_dim,
                           size_t out_dim, float scale, const void *compressed,
                           const uint32_t *warp_offsets, const uint32_t *ppf,
                           const uint32_t *ppf_cum, const uint32_t *ppf_prob);

/* Exact int32 form of the same decode (the reference kernel's accumulator
 * before its fused requantisation, ans-warp-rows-kernel.cu:191-210), for
 * batch vectors.  n_words bounds every read of `compressed_dev` (u32 words,
 * 16-byte aligned).  warp_offsets are in uint4 units (buffered/encoder.py:482).
 * Requires cols % 128 == 0 (buffered/encoder.py:397). */
mv_status mv_awr_matvec(const uint32_t *compressed_dev, size_t n_words,
                        const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                        const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev, int rows,
                        int cols, const int8_t *x_dev, int batch, int32_t *y_dev,
                        const float *row_scales_dev, float *y_scaled_dev, void *stream);

/* Fused decode + dot product + requantisation to int8 for one vector, the
 * chained step of buffered/ans-warp-rows.cu:208-221: out8[r] =
 * clamp(round_half_even((float)y[r] * scale), -128, 127). */
mv_status mv_awr_matvec_requant(const uint32_t *compressed_dev, size_t n_words,
                                const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                                const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev,
                                int rows, int cols, const int8_t *x_dev, float scale,
                                int8_t *out8_dev, void *stream);

/* ------------------------------------------------------------- stripes --- */

/* The reference's "ans-warp-stripes" layout (buffered/encoder.py:323-391,
 * kernel ans-warp-stripes-kernel.cu:21-227): the AWR coder and word stream,
 * but a warp decodes a stripe of 32 rows, lane l row 32s+l, one quad per lane
 * per step; warp_offsets has one entry per stripe (uint4 units).  Exact int32
 * y for `batch` vectors.  rows % 32 == 0, cols % 4 == 0. */
mv_status mv_aws_matvec(const uint32_t *compressed_dev, size_t n_words,
                        const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                        const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev, int rows,
                        int cols, const int8_t *x_dev, int batch, int32_t *y_dev,
                        const float *row_scales_dev, float *y_scaled_dev, void *stream);

/* Fused decode + dot product + requantisation, the reference kernel's output:
 * out8[r] = clamp(round_half_even((float)y[r] * scale), -128, 127). */
mv_status mv_aws_matvec_requant(const uint32_t *compressed_dev, size_t n_words,
                                const uint32_t *warp_offsets_dev, const uint32_t *ppf_dev,
                                const uint32_t *ppf_cum_dev, const uint32_t *ppf_prob_dev,
                                int rows, int cols, const int8_t *x_dev, float scale,
                                int8_t *out8_dev, void *stream);

/* Replaces the launcher of buffered/ans-warp-stripes.cu:38-60, which has the
 * same name and arguments as the rows program's mat_vec_mul_coalesced; renamed
 * so that both layouts live in one library.  Legacy default stream; errors go
 * to stderr and mv_last_error(). */
void mat_vec_mul_coalesced_stripes(const void *in_vector_gpu, void *out_vector_gpu, size_t in_dim,
                                   size_t out_dim, float scale, const void *compressed,
                                   const uint32_t *warp_offsets, const uint32_t *ppf,
                                   const uint32_t *ppf_cum, const uint32_t *ppf_prob);

/* ------------------------------------------------------------------ WPR --- */

/* Replaces the kernel launch in CompressedMatrix::decompressAndMult,
 * matvansWarpPerRow/matvansWarpPerRow.cu:150-164 (kernel arguments of
 * matvansWarpPerRow-kernel.cu:46-50): int32 y for `batch` vectors.
 * `payload_dev` holds payload_size u16 words (16-byte aligned), `cursors_dev`
 * the per-row u16 cursors, `cdf_dev` G+1 low cdf bytes, `ppf_dev` 256 bytes.
 * Requires cols % 512 == 0 (create_matrices_WarpPerRow.py:361-366). */
mv_status mv_wpr_matvec(const uint16_t *payload_dev, size_t payload_size,
                        const uint32_t *cursors_dev, int8_t min_value, const uint8_t *cdf_dev,
                        int G, const uint8_t *ppf_dev, int rows, int cols, const int8_t *x_dev,
                        int batch, int32_t *y_dev, const float *row_scales_dev,
                        float *y_scaled_dev, void *stream);

/* The epilogue of matvansWarpPerRow.cu:51-72,167-172 fused into one kernel
 * without a host round trip: delta = max|y|/127 (fp32), out8[r] =
 * (int8)round_half_even((float)y[r] / delta), no clamp (as in the reference).
 * `absmax_scratch_dev` is one caller-owned uint32.  Writes delta to
 * *delta_dev. */
mv_status mv_requant_absmax(const int32_t *y_dev, int n, int8_t *out8_dev, float *delta_dev,
                            uint32_t *absmax_scratch_dev, void *stream);

/* Allocation-free variant of mv_requant_absmax.  No counterpart in the
 * reference.  For callers that cannot allocate device memory: plugins whose
 * host framework owns the allocator (and may hold all free memory in its
 * pool), latency-critical paths that cannot afford cudaMalloc's implicit
 * synchronisation.  Same inputs, outputs and results as mv_requant_absmax,
 * but the reduction scratch is a 16 KiB array compiled into the library
 * (held on every GPU that loads it, until exit), so it calls no allocating
 * routine.  n <= 33,554,432, else MV_ERR_ARG.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture on that device.  All calls share the array:
 * calls that overlap on the GPU race and must be serialised; no state needs
 * clearing between calls. */
mv_status mv_requant_absmax_noalloc(const int32_t *y_dev, int n, int8_t *out8_dev, float *delta_dev,
                                    void *stream);

/* ------------------------------------------------------------------- Q8 --- */

/* Device view of one Q8-stripe matrix (all pointers are device pointers).
 * Layout (built by mv_q8_encode):
 *   stripes = ceil(rows/32), nseg = ceil(ceil(cols/4) / seg_quads).
 *   Block b = stripe*nseg + seg starts at blocks + 32*blk_off[b] (128-byte
 *   units) and spans blk_off[b+1]-blk_off[b] word-rows of 32 u32: word-row 0
 *   and 1 hold the low / high halves of the 32 lanes' 64-bit coder states,
 *   word-row 2+k holds the k-th refill word of each lane (lane = row within
 *   the stripe).
 *   Table t (t = row if local, else 0) is tbl[tbl_off[t] .. tbl_off[t+1]) of
 *   u16 entries (uint8 symbol | freq << 8), sorted by symbol, freqs summing to
 *   256.  Rows past `rows` in the last stripe use table tbl_pad (local mode).
 */
typedef struct mv_q8_view {
    const uint32_t *blocks;
    const uint32_t *blk_off;  /* [stripes*nseg + 1] */
    const uint16_t *tbl;
    const uint32_t *tbl_off;  /* [ntables + 1] */
    int32_t rows, cols;
    int32_t seg_quads;        /* quads (4 columns) per lane per segment     */
    int32_t nseg;
    int32_t local;            /* 1 = one table per (padded) row, 0 = global  */
    int32_t max_blk_rows;     /* max word-rows of any block                  */
    uint32_t blocks_rows;     /* word-rows (128 bytes) readable at `blocks`  */
    uint32_t tbl_len;         /* u16 entries readable at `tbl`               */
    uint32_t tbl_stripe_max;  /* max entries of one stripe's 32 tables (local)
                                 or of the global table                      */
} mv_q8_view;

/* y = W x for any batch >= 1 (passes of up to 16 vectors share one decode). */
mv_status mv_q8_matvec(const mv_q8_view *m, const int8_t *x_dev, int batch, int32_t *y_dev,
                       const float *row_scales_dev, float *y_scaled_dev, void *stream);

/* Launch parameters of the persistent Q8 kernel (0 = library default).
 *   warps        warps per CTA (default 8; 16 for the float forward on
 *                the CUDA cores): up to 16, except 8 for the float backward
 *                and the float form on the tensor cores
 *   ilp          independent segments decoded per warp (1 or 2, default 2;
 *                1 for the float form)
 *   depth        shared-memory stream buffers per warp (1 or 2, default 1):
 *                2 keeps the next work item's bulk copies in flight
 *   ctas_per_sm  cap on resident CTAs per SM (default: occupancy limit)
 *   parts        work items per 32-row stripe (its segments split in `parts`
 *                ranges; default: whole stripes in stacks, enough parts to
 *                fill the GPU for a single matrix)
 *   engine       int8 product of 3..16 vectors: 0 = tensor cores
 *                (tcgen05.mma kind::i8, TMEM accumulators, always 16
 *                vectors wide with the missing ones zero; ilp is then 1),
 *                1 = CUDA cores (dp4a).  One or two vectors always use
 *                dp4a. */
#define MV_ENGINE_AUTO 0
#define MV_ENGINE_DP4A 1
/* Smallest integer batch that engine 0 (MV_ENGINE_AUTO) runs on the tensor
 * cores. */
#define MV_MMA_MIN_VECTORS 3
typedef struct mv_q8_tuning {
    int32_t warps, ilp, depth, ctas_per_sm, parts, engine;
} mv_q8_tuning;

/* mv_q8_matvec with explicit launch parameters (needs cols % 16 == 0,
 * seg_quads % 4 == 0 and a 16-byte aligned x; mv_q8_matvec itself falls back
 * to a non-persistent kernel otherwise). */
mv_status mv_q8_matvec_tuned(const mv_q8_view *m, const int8_t *x_dev, int batch, int32_t *y_dev,
                             const float *row_scales_dev, float *y_scaled_dev,
                             const mv_q8_tuning *tuning, void *stream);

/* One matrix of a batched launch: the matrix, its input x [batch][cols] and
 * outputs y [batch][rows] (+ optional scaled output).  ngroups, atomic and
 * item0 are filled in by mv_q8_stack_plan.  x_tiles (optional, NULL for none)
 * is device scratch of mv_q8_x_tiles_bytes(&m) bytes, 16-byte aligned: with
 * 3..16 vectors on the tensor cores, mv_q8_stack_matvec first lays x out there
 * in the MMA operand layout, and each warp then brings its x windows in with
 * asynchronous copies (four 16-byte cp.async per lane per window, completing
 * on an mbarrier) instead of loads and stores through registers. */
typedef struct mv_q8_job {
    mv_q8_view m;
    const int8_t *x;
    int32_t *y;
    const float *scales;
    float *ys;
    int32_t ngroups;
    int32_t atomic;
    uint32_t item0;
    uint32_t pad;
    int8_t *x_tiles;
} mv_q8_job;

/* Bytes of the x_tiles scratch of a job on matrix m: one 2 KB tile (16
 * vectors x 128 columns) per 32 quads of every segment. */
size_t mv_q8_x_tiles_bytes(const mv_q8_view *m);

typedef struct mv_q8_stack_info {
    uint32_t nitems;          /* work items (matrix, 32-row stripe, segment group) */
    int32_t max_blk_rows;     /* shared-memory sizing over all jobs */
    uint32_t tbl_stripe_max;
    int32_t warps, ilp, depth;
    int32_t atomic_jobs;      /* jobs whose rows span several work items (outputs zeroed, accumulated, scaled) */
} mv_q8_stack_info;

/* Plans a batched launch on the host: fills ngroups/atomic/item0 of every
 * job for the given tuning and returns the sizes the launch needs.  The
 * caller then copies `jobs` to device memory.  The plan reorders the array in
 * place, jobs with the most work per item first (stable), so that the work
 * queue ends on short items; every job keeps its own x and y, so results are
 * unaffected.  It also zeroes jobs[0].pad, the work-queue counter of the
 * launch (reset by the kernel after each launch; concurrent launches on one
 * job table race). */
mv_status mv_q8_stack_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning,
                           mv_q8_stack_info *info);

/* Every job of a (device-resident, planned) job table in ONE persistent
 * launch: CTAs walk the (matrix, stripe, segment-group) work items of all
 * matrices, so uneven shapes share the GPU without per-matrix tails.  batch
 * 1..16.  Launches the persistent decode, plus a kernel before it that zeroes
 * and one after it that scales the outputs of atomically-accumulated jobs
 * when the plan has any (info->atomic_jobs > 0); capturable in a CUDA graph
 * once the device status word exists (any earlier call creates it). */
mv_status mv_q8_stack_matvec(const mv_q8_job *jobs_dev, int njobs, const mv_q8_stack_info *info,
                             int batch, const mv_q8_tuning *tuning, void *stream);

/* Chained pipeline, the reference's end-to-end workload (buffered/ans-warp-rows.cu:208-221:
 * int32 y -> fp32 scale -> int8 -> next matrix), fused into one persistent,
 * cooperative launch.  jobs[j+1].x receives clamp(round_half_even((float)y_j[r] *
 * chain_scales[j]), -128, 127) for every row r of job j (the requantisation of
 * ans-warp-rows-kernel.cu:212-220); the last job's goes to out8 [batch][rows].
 * jobs[0].x is the input; y_j (int32) and, with scales, ys_j are written as in a stack.
 * Work items of job j+1 wait (bounded) until every item of job j is done;
 * jobs[j].pad is the device-side counter (reset by each call).  Plan with
 * mv_q8_chain_plan (checks rows_j == cols_{j+1}, whole stripes).  jobs_dev is
 * modified (the counters); concurrent calls on the same jobs_dev race. */
mv_status mv_q8_chain_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning,
                           mv_q8_stack_info *info);
mv_status mv_q8_chain_matvec(mv_q8_job *jobs_dev, int njobs, const mv_q8_stack_info *info, int batch,
                             const float *chain_scales_dev, int8_t *out8_dev,
                             const mv_q8_tuning *tuning, void *stream);

/* Float form (no reference counterpart): y[b][r] = s[r] * sum_c W[r][c] *
 * x[b][c] with x bf16 [batch][cols] (16-byte aligned), fp32 accumulation in a
 * fixed order (deterministic), fp32 y [batch][rows].  cols % 16 == 0.  Passes
 * of up to 8 vectors share one decode. */
mv_status mv_q8_matvec_bf16(const mv_q8_view *m, const uint16_t *x_dev, int batch,
                            const float *row_scales_dev, float *y_dev, const mv_q8_tuning *tuning,
                            void *stream);

/* Transposed float form, the backward of the above: dx[b][c] = sum_r W[r][c]
 * * s[r] * dy[b][r] with dy bf16 [batch][rows], fp32 dx [batch][cols]
 * (zeroed by the call).  The streams are decoded again (W is never stored);
 * the 32 rows of a stripe are summed per column inside the warp and stripes
 * are combined with fp32 atomics, so the result is reproducible to fp32
 * rounding, not bit for bit. */
mv_status mv_q8_matvec_t_bf16(const mv_q8_view *m, const uint16_t *dy_dev, int batch,
                              const float *row_scales_dev, float *dx_dev,
                              const mv_q8_tuning *tuning, void *stream);

/* Decode the whole matrix to W_dev[rows][cols] (test / debugging aid). */
mv_status mv_q8_decode(const mv_q8_view *m, int8_t *W_dev, void *stream);

/* ---------------------------------------------------------------- dense --- */

/* Dense int8 comparator: y = W x with W int8 row-major [rows][cols] in device
 * memory (the baseline of baselines/baseline_int8/baseline_matVec_custom.cu:99-155,
 * written for sm_100a).  cols % 16 == 0. */
mv_status mv_dense_matvec(const int8_t *W_dev, int rows, int cols, const int8_t *x_dev,
                          int batch, int32_t *y_dev, void *stream);

/* ------------------------------------------------------ host: encoders --- */

/* Encoders produce a blob: a set of named host arrays. */
typedef struct mv_blob mv_blob;
void mv_blob_free(mv_blob *b);
/* Looks up array `name`; *data points into the blob (valid until freed). */
mv_status mv_blob_get(const mv_blob *b, const char *name, const void **data, size_t *nbytes);
/* Scalar metadata stored in the blob (e.g. "rows", "min_value"). */
mv_status mv_blob_get_i64(const mv_blob *b, const char *name, int64_t *value);
/* Name of the i-th array (NULL past the end). */
const char *mv_blob_name(const mv_blob *b, int i);

/* Reference-compatible AWR encoder: byte-identical to
 * compress_ans_warp_rows(W, 32) of buffered/encoder.py:394-461 with the model
 * of fit_128bit_encoder_model (:271-306).  Arrays: "compressed" u32,
 * "warp_offsets" u32[rows] (uint4 units), "cdf" u8, "ppf"/"ppf_cum"/"ppf_prob"
 * u32[32] (encoder.py:309-320,464-470); scalars "min_value", "rows", "cols".
 * Fails with MV_ERR_SHAPE unless cols % 128 == 0, and MV_ERR_UNSUPPORTED for
 * more than 128 distinct values (encoder.py:303). */
mv_status mv_awr_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out);

/* Reference-compatible "ans-warp-stripes" encoder: byte-identical to
 * compress_ans_warp_stripes(W, 32) of buffered/encoder.py:323-391 (same model
 * and tables as mv_awr_encode).  Arrays as mv_awr_encode, with
 * "warp_offsets" u32[rows/32].  rows % 32 == 0, cols % 4 == 0. */
mv_status mv_aws_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out);

/* Reference-compatible WPR encoder: encode_matrix of
 * create_matrices_WarpPerRow.py:353-430 with create_entropy_model (:131-187)
 * and create_ppf (:189-208); padding words are zero.  Arrays: "payload" u16,
 * "cursors" u32[rows], "cdf" u8[G+1] (low bytes), "ppf" u8[256]; scalars
 * "min_value", "G", "rows", "cols".  cols % 512 == 0. */
mv_status mv_wpr_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out);

/* Q8-stripe encoder.  local = 1 fits one table per row, 0 one table for the
 * matrix.  seg_quads = 0 picks the segment length automatically.  Arrays:
 * "blocks" u32, "blk_off" u32, "tbl" u16, "tbl_off" u32; scalars "rows",
 * "cols", "seg_quads", "nseg", "local", "max_blk_rows", "tbl_stripe_max", "payload_bytes"
 * (blocks + tables + offsets). */
mv_status mv_q8_encode(const int8_t *W, int rows, int cols, int local, int seg_quads,
                       int nthreads, mv_blob **out);

/* --------------------------------------------------------- host: files --- */

/* Reads a safetensors file into a blob (one array per tensor; scalar
 * "<name>.ndim" and "<name>.shape<i>" entries give the shapes; dtype codes in
 * "<name>.dtype": 1 i8, 2 u8, 3 i16, 4 u16, 5 i32, 6 u32, 7 f32, 8 i64, 9 u64,
 * 10 f64).  Replaces SaneSafetensorFile (buffered/sane_safetensors.hpp:17-68). */
mv_status mv_read_safetensors(const char *path, mv_blob **out);

/* Writes the arrays of `b` as a safetensors file (shapes and dtypes from the
 * same scalar entries). */
mv_status mv_write_safetensors(const char *path, const mv_blob *b);

/* Reads a matvansWarpPerRow .bin file (create_matrices_WarpPerRow.py:440-461,
 * matvansWarpPerRow.cu:225-258).  Scalars "num_matrices", "result_hash",
 * "max_word_count", "len_v"; array "vector"; per matrix i arrays
 * "m<i>.cursors", "m<i>.cdf", "m<i>.ppf", "m<i>.payload" and scalars
 * "m<i>.rows", "m<i>.cols", "m<i>.min_value", "m<i>.G", "m<i>.payload_size". */
mv_status mv_read_wpr_bin(const char *path, mv_blob **out);

/* ------------------------------------------------------------- Q8 files --- */

/* Host arrays of one Q8 matrix (as mv_q8_encode returns them; see mv_q8_view
 * for the layout) and, optionally, its per-row fp32 scales. */
typedef struct mv_q8_host {
    const uint32_t *blocks;   size_t n_blocks;   /* u32 words, a multiple of 32 */
    const uint32_t *blk_off;  size_t n_blk_off;  /* stripes*nseg + 1            */
    const uint16_t *tbl;      size_t n_tbl;
    const uint32_t *tbl_off;  size_t n_tbl_off;  /* tables + 1                  */
    int32_t rows, cols, seg_quads, nseg, local, max_blk_rows;
    uint32_t tbl_stripe_max;
    const float *row_scales;  /* [rows] or NULL */
} mv_q8_host;

/* The chained workload stored with a file (the reference's end-to-end
 * pipeline, buffered/encoder.py:42-51), every field optional (NULL). */
typedef struct mv_q8_chain_host {
    const int8_t *initial_vector; size_t n_initial;
    const float *scales;     /* [count] requantisation scale of each step */
    const uint32_t *hashes;  /* [count] hash of each step's int8 output   */
} mv_q8_chain_host;

/* Writes `count` Q8 matrices (and the chain data, if given) as one safetensors
 * file, in the convention of the reference's files (buffered/encoder.py:473-511:
 * concatenated arrays with per-matrix start offsets; the chain tensors keep the
 * reference's names initial_vector / scales / hashes).  Tensors: q8_meta I32
 * [count, 8] (rows, cols, seg_quads, nseg, local, max_blk_rows, tbl_stripe_max,
 * has_row_scales), q8_blocks/q8_blk_off/q8_tbl/q8_tbl_off and row_scales, each
 * with a "<name>_start" U64 [count + 1].  Every matrix is checked against the
 * layout's shape rules first (MV_ERR_FORMAT). */
mv_status mv_q8_save(const char *path, const mv_q8_host *mats, int count, const mv_q8_chain_host *chain);

/* Reading: a file opened with mv_read_safetensors holds `count` matrices;
 * mv_q8_file_matrix fills `out` with pointers into the blob (valid until it is
 * freed) after the same checks, mv_q8_file_chain the chain data (NULL fields
 * when absent). */
mv_status mv_q8_file_count(const mv_blob *file, int *count);
mv_status mv_q8_file_matrix(const mv_blob *file, int index, mv_q8_host *out);
mv_status mv_q8_file_chain(const mv_blob *file, mv_q8_chain_host *out);

/* A Q8 matrix in device memory of the current device, owned by the handle
 * (these calls allocate; the launch paths never do).  mv_q8_load reads matrix
 * `index` of a file and uploads it; the view is valid until mv_q8_matrix_free. */
typedef struct mv_q8_matrix mv_q8_matrix;
mv_status mv_q8_upload(const mv_q8_host *h, mv_q8_matrix **out);
mv_status mv_q8_load(const char *path, int index, mv_q8_matrix **out);
const mv_q8_view *mv_q8_matrix_view(const mv_q8_matrix *m);
const float *mv_q8_matrix_row_scales(const mv_q8_matrix *m);  /* device pointer or NULL */
void mv_q8_matrix_free(mv_q8_matrix *m);

/* Fault injection for tests of the device-side error paths (no reference
 * counterpart).  MV_INJECT_WAIT_LIMIT sets the iteration bound of every
 * shared-memory barrier wait (0 restores the default); MV_INJECT_DROP_COPY
 * (value 1) makes Q8 launches skip their bulk copies, so their bounded waits
 * run out and raise MV_DEV_WAIT_TIMEOUT.  Process-wide, not thread-safe. */
#define MV_INJECT_WAIT_LIMIT 1
#define MV_INJECT_DROP_COPY 2
mv_status mv_debug_inject(int what, uint32_t value);

/* Test and debugging aid (no reference counterpart): MV_QUERY_STATUS_WORD sets
 * *value to 1 if the current device's status word (the library's only lazily
 * created device allocation) exists, else 0; it creates nothing. */
#define MV_QUERY_STATUS_WORD 1
mv_status mv_debug_query(int what, uint64_t *value);

/* FxHash-style hash of an int8 vector (buffered/encoder.py:8-20). */
uint32_t mv_hash_int8(const int8_t *v, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* MATVANS_H */
