// Persistent decode + int8 matvec over a list of Q8-stripe matrices
// ("jobs": one matrix with its x and y each) in one launch, for sm_100a.
//
// Work item = (job, stripe, segment group).  A group is SG = W*ILP segments
// of one stripe: warp w decodes segments g*SG + w (+ W) -- with ILP = 2 the
// two segments are independent rANS streams interleaved in one instruction
// stream, which hides the ~60-cycle latency chain of a decode step.  CTAs are
// persistent.  A stack takes its items from a work queue (one global counter,
// numbered job by job, so that consecutive items of a CTA usually share a
// global table); single matrices and chains take items c, c + G, c + 2G, ... .
// Thread 0 keeps the CTA's next two items in a small shared-memory ring, so
// that warps can copy their streams one item ahead.
//
// Per item:
//   * lane 0 of each warp moves the warp's stream blocks into shared memory
//     with 1-D bulk copies (cp.async.bulk, TMA engine, no multicast) completing
//     on an mbarrier, DEPTH steps ahead of its decode (across item boundaries);
//   * the decode table (256 quantiles x 32 lanes, conflict-free) is rebuilt
//     only when the table changes: every item for per-row tables, once per
//     job for a global table.  The table data of the next item is staged in
//     shared memory by asynchronous copies (cp.async) while the current item
//     decodes, so a rebuild does not wait for device memory.  CUDA-core
//     consumers use the wide layout, 8-byte
//     entries {f | sym << 16, r} at byte q*256 + l*8 (64 KB): one byte permute
//     of the state gives a lookup address and r needs no extraction.  The
//     tensor-core consumers, two CTAs per SM, keep the narrow layout, 4-byte
//     entries f | sym << 16 | r << 24 at word q*32 + l (32 KB);
//   * x is read through L1 with broadcast loads (all lanes of a warp read the
//     same quad), so it needs no staging;
//   * per-row partial sums are reduced across warps in shared memory and
//     stored, or added with exact integer atomics when a row spans groups.
//
// Decode step (per lane, per quad of 4 symbols; table entry e = f | sym << 16
// | r << 24 with f the symbol's frequency, r = q - cum < f <= 255):
//   refill:   if (hi == 0) { hi = lo; lo = next word } -- the lane's stream
//             position is a shared-memory byte offset that advances by one
//             128-byte word-row, clamped to the row after the block
//   lookups:  e_i = table[byte i of lo]
//   update:   u01 = r0 + f0*r1, t2 = r2 + f2*r3, f0*f1, f2*f3 (dp2a: 16-bit
//             x 8-bit dot products read f straight from the entries), t0 =
//             u01 + (f0 f1) t2, P = (f0 f1)(f2 f3), (hi:lo) = hi*P + t0 (one
//             32x32->64 IMAD)
#include <algorithm>
#include <type_traits>
#include <cstdio>

#include <cuda_bf16.h>

#include "mv_device.cuh"
#include "umma.cuh"

namespace mv {

typedef mv_q8_job Q8Job;

// Shared-memory layout of q8s_kernel (byte offsets; see q8s_layout).
constexpr uint32_t kStageOffs = 40;  // u32 per staging area: 33 relative offsets, [36] valid, [37] first entry
constexpr uint32_t kStagePad = 8;    // entries per staging area beyond tbl_stage (copies start at an even entry)
struct Q8SLayout {
    uint32_t extra, bufs, red, bars, ring, curs, sched, stage_o, rows, stage_e, total;
    uint32_t async_tables;  // 1: two staging areas, the next item's table data staged during the current item
};

__global__ void scale_rows_kernel(const int32_t *y, const float *s, float *ys, int rows, int batch, int ldy);

struct Q8SLaunch {
    Q8Job job0;            // the only job when jobs == nullptr
    const Q8Job *jobs;     // device array of njobs jobs, or nullptr
    int njobs;
    uint32_t nitems;
    int batch;           // valid vectors (<= NV)
    int x_row_words;     // unused placeholder for alignment
    uint32_t *status;
    uint32_t spin_limit;
    int drop_copy;
    int buf_words;       // per segment buffer, u32 words
    int tbl_stage;       // staged table entries
    uint32_t lut_stride; // 32 (words per quantile row of the table); a runtime value on purpose
    // chained pipeline (mv_q8_chain_matvec): job j's int8 output clamp(rn(y * chain_scales[j])) is job
    // j+1's x (the last job's goes to chain_out8); jobs[j].pad counts job j's finished work items
    const float *chain_scales;
    int8_t *chain_out8;
    // work queue of a stack (jobs[0].pad of the job table), or nullptr: static round robin
    uint32_t *queue;
    // shared-memory layout of this launch (set by the launcher; constant-bank operands in the kernel)
    Q8SLayout lay;
    uint32_t slot_bytes;  // ILP * buf_words * 4: one warp's stream slot
    uint32_t stage_len;   // entries per table staging area
};

// One work item as the CTA's scheduler hands it out (it < 0: no more items).
struct alignas(16) ItemRec {
    int32_t it, job, stripe, sb, se, pad0, pad1, pad2;
};
constexpr int kRing = 4;  // items the ring holds: the current one and up to two ahead

__device__ __forceinline__ const Q8Job &job_at(const Q8SLaunch &L, int j) { return L.jobs ? L.jobs[j] : L.job0; }

// Segment range [sb, se) of an item: its stripe's segments split into ngroups parts.
__device__ __forceinline__ void item_segs(const mv_q8_view &m, int ngroups, int group, int &sb, int &se) {
    const int spp = (m.nseg + ngroups - 1) / ngroups;
    sb = group * spp;
    se = min(m.nseg, sb + spp);
}

// Item number -> record.  Each CTA takes its items in increasing order, so the job search runs forward from
// the previous item's job (jhint): one comparison in the common case, a binary search over the rest otherwise.
__device__ __forceinline__ ItemRec make_item(const Q8SLaunch &L, uint32_t it, int &jhint) {
    ItemRec r{};
    if (it >= L.nitems) {
        r.it = -1;
        return r;
    }
    int j = 0;
    uint32_t rel = it;
    int ng = L.job0.ngroups;
    if (L.jobs) {
        j = jhint;
        if (j + 1 < L.njobs && __ldg(&L.jobs[j + 1].item0) <= it) {
            int lo = j + 1, hi = L.njobs - 1;
            while (lo < hi) {  // last job with item0 <= it
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&L.jobs[mid].item0) <= it) lo = mid;
                else hi = mid - 1;
            }
            j = lo;
        }
        jhint = j;
        rel = it - __ldg(&L.jobs[j].item0);
        ng = __ldg(&L.jobs[j].ngroups);
    }
    r.it = (int32_t)it;
    r.job = j;
    r.stripe = (int)(rel / (uint32_t)ng);
    item_segs(job_at(L, j).m, ng, (int)(rel % (uint32_t)ng), r.sb, r.se);
    return r;
}

// The CTA's k-th item number (thread 0 only).  Static: c + k G.  Queue: one atomic per item; every CTA takes
// items until one grab fails, so a launch makes exactly nitems + G grabs, and the one that makes the last of
// them (no other grab can follow it) resets the counter for the next launch.
__device__ __forceinline__ uint32_t sched_grab(const Q8SLaunch &L, uint32_t k) {
    if (!L.queue) {
        const unsigned long long v = (unsigned long long)blockIdx.x + (unsigned long long)k * gridDim.x;
        return v < L.nitems ? (uint32_t)v : L.nitems;
    }
    return atomicAdd(L.queue, 1u);
}
__device__ __forceinline__ void sched_after_grab(const Q8SLaunch &L, uint32_t v) {
    if (L.queue && v == L.nitems + gridDim.x - 1) atomicExch(L.queue, 0u);
}

// Steps of a warp in an item of n segments; step j covers segments
// sb + warp + j*W*ILP + k*W for k < ILP.
__device__ __forceinline__ int warp_steps(int n, int warp, int W, int ILP) {
    return warp < n ? (n - warp + W * ILP - 1) / (W * ILP) : 0;
}

// The next step whose stream blocks a warp copies (lane 0; kept in shared memory): ring index k of its
// item, step j of `steps`.  An item's record may be read once it is visible (written before a CTA barrier the
// warp has passed).
struct alignas(16) StepCursor {
    int k, j, steps, sb, se, stripe, job, done;
};

// Thread 0's scheduler state, kept in shared memory (off the decode loop's registers).
struct alignas(16) SchedState {
    uint32_t ngrab, pending;
    int jhint, grab_done, grab_now, pad0, pad1, pad2;
};

// Moves the cursor onto a step that exists (entering later items while they are visible); false while the
// next item is not visible yet.
__device__ __forceinline__ bool cursor_ready(StepCursor &c, const ItemRec *ring, int kvis, int warp, int W,
                                             int ILP) {
    while (!c.done && c.j >= c.steps) {
        if (c.k + 1 > kvis) return false;
        c.k++;
        const ItemRec &I = ring[c.k % kRing];
        if (I.it < 0) {
            c.done = 1;
            break;
        }
        c.j = 0;
        c.steps = warp_steps(I.se - I.sb, warp, W, ILP);
        c.sb = I.sb;
        c.se = I.se;
        c.stripe = I.stripe;
        c.job = I.job;
    }
    return !c.done;
}

// Issue the bulk copies of the cursor's step into one slot (lane 0 only).  soff is the slot's byte offset in
// shared memory.
template <int ILP>
__device__ __forceinline__ void issue_step(const Q8SLaunch &L, const StepCursor &c, int warp, int W,
                                           unsigned char *sm, uint32_t soff, uint64_t *bar, uint32_t *rows_out) {
    const mv_q8_view &m = job_at(L, c.job).m;
    const int seg0 = c.sb + warp + c.j * W * ILP;
    uint32_t total = 0;
    uint32_t o0s[ILP], rows[ILP];
#pragma unroll
    for (int k = 0; k < ILP; k++) {
        const int seg = seg0 + k * W;
        rows[k] = 0;
        o0s[k] = 0;
        if (seg < c.se) {
            const int b = c.stripe * m.nseg + seg;
            const uint32_t o0 = __ldg(m.blk_off + b), o1 = __ldg(m.blk_off + b + 1);
            const uint32_t r = o1 - o0;
            if (o1 < o0 || o1 > m.blocks_rows || r < 2 || (int)r + 1 > L.buf_words / 32) {
                atomicOr(L.status, MV_DEV_STREAM_OVERRUN);
            } else {
                rows[k] = r;
                o0s[k] = o0;
                total += r * 128u;
            }
        }
        rows_out[k] = rows[k];
    }
    mbar_arrive_expect_tx(bar, total);
    if (!L.drop_copy) {
#pragma unroll
        for (int k = 0; k < ILP; k++)
            if (rows[k])
                bulk_g2s(sm + soff + (uint32_t)k * (uint32_t)L.buf_words * 4u, m.blocks + (size_t)o0s[k] * 32,
                         rows[k] * 128u, bar);
    }
}

// x loads: plain (coherent, L1-cached) global loads rather than the read-only path.  In a chained
// launch x was written earlier by other CTAs; the acquire load and CTA barrier of chain_wait order these
// loads after those writes, which the read-only path would not guarantee.
__device__ __forceinline__ uint4 ldx_u4(const void *p) { return *reinterpret_cast<const uint4 *>(p); }
__device__ __forceinline__ uint32_t ldx_u32(const void *p) { return *reinterpret_cast<const uint32_t *>(p); }

template <int NV>
__device__ __forceinline__ void load_x(const int8_t *x, int cols, int q, uint32_t (&xv)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; v++) xv[v] = ldx_u32(reinterpret_cast<const uint32_t *>(x + (size_t)v * cols) + q);
}

// Four consecutive quads of x (16 bytes) per vector; q % 4 == 0.
template <int NV>
__device__ __forceinline__ void load_x4(const int8_t *x, int cols, int q, uint4 (&xv)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; v++) xv[v] = ldx_u4(x + (size_t)v * cols + 4 * q);
}

// The chained pipeline's epilogue of one output: job j's int8 result, the reference's fp32
// requantisation (ans-warp-rows-kernel.cu:212-220), stored as the next job's x.
__device__ __forceinline__ void chain_emit(const Q8SLaunch &L, const Q8Job &J, int j, int v, int row, int sum) {
    const int r = __float2int_rn((float)sum * __ldg(L.chain_scales + j));
    int8_t *o = j + 1 < L.njobs ? const_cast<int8_t *>(L.jobs[j + 1].x) : L.chain_out8;
    o[(size_t)v * J.m.rows + row] = (int8_t)max(-128, min(127, r));
}

template <int NV>
__device__ __forceinline__ void dot4(uint32_t w, const uint4 (&xv)[NV], int j, int (&acc)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const uint32_t xw = j == 0 ? xv[v].x : j == 1 ? xv[v].y : j == 2 ? xv[v].z : xv[v].w;
        acc[v] = __dp4a((int)w, (int)xw, acc[v]);
    }
}

// Refill of one stream.  koff is the byte offset (from the start of shared memory) of the lane's next word:
// it is read every step, and taken when the high half of the state is empty; the offset then moves one
// 128-byte word-row on, never past kend (the row after the block), so a corrupt stream rereads that row and
// fails the final-state check instead of leaving its slot.  Written as selects: the same step as an `if`
// block measured 7% slower on the 12-matrix step (197 vs 214 us).
__device__ __forceinline__ void q8_refill(uint32_t &lo, uint32_t &hi, uint32_t &koff, const uint32_t kend,
                                          const unsigned char *sm) {
    const uint32_t w = *reinterpret_cast<const uint32_t *>(sm + koff);
    const bool need = hi == 0;
    hi = need ? lo : hi;
    lo = need ? w : lo;
    koff = __viaddmin_u32(koff, need ? 128u : 0u, kend);
}

// One decode step of one stream; returns the packed four symbols.
__device__ __forceinline__ uint32_t q8_step(uint32_t &lo, uint32_t &hi, uint32_t &koff, const uint32_t kend,
                                            const unsigned char *sm, const uint32_t *lut_l, uint32_t stride,
                                            uint32_t &P) {
    q8_refill(lo, hi, koff, kend, sm);
    const uint32_t a0 = __byte_perm(lo, 0, 0x4440), a1 = __byte_perm(lo, 0, 0x4441);
    const uint32_t a2 = __byte_perm(lo, 0, 0x4442), a3 = __byte_perm(lo, 0, 0x4443);
    // stride is 32 words, passed at run time so the index math stays an IMAD
    const uint32_t e0 = lut_l[a0 * stride], e1 = lut_l[a1 * stride];
    const uint32_t e2 = lut_l[a2 * stride], e3 = lut_l[a3 * stride];
    // entry = f | sym << 16 | r << 24 (byte 1 zero, so the low half-word is exactly f)
    const uint32_t r0 = __umulhi(e0, 256u), r1 = __umulhi(e1, 256u);
    const uint32_t r2 = e2 >> 24, r3 = e3 >> 24;
    const uint32_t u01 = __dp2a_lo(r1, e0, r0);     // r0 + f0*r1
    const uint32_t t2 = __dp2a_lo(r3, e2, r2);      // r2 + f2*r3
    const uint32_t p01 = __dp2a_lo(e1, e0, 0u);     // f1*f0 + (sym1 | r1 << 8) * 0
    const uint32_t p23 = __dp2a_lo(e3, e2, 0u);     // f3*f2
    P = p01 * p23;
    const uint32_t t0 = u01 + p01 * t2;             // r0 + f0 r1 + f0 f1 (r2 + f2 r3) < P
    const unsigned long long s = (unsigned long long)hi * P + t0;
    lo = (uint32_t)s;
    hi = (uint32_t)(s >> 32);
    return __byte_perm(__byte_perm(e0, e1, 0x0062), __byte_perm(e2, e3, 0x0062), 0x5410);
}

// The same step over the wide table: 8-byte entries {f | sym << 16, r} at byte q*256 + lane*8 from the
// start of shared memory.  A quantile byte of the state lands in bits 8..15 of the address and lane*8 in
// bits 0..7, so one byte permute forms each lookup address, and r arrives as a clean word.
__device__ __forceinline__ uint32_t q8_step_wide(uint32_t &lo, uint32_t &hi, uint32_t &koff, const uint32_t kend,
                                                 const unsigned char *lut_b, uint32_t lane8, uint32_t &P) {
    q8_refill(lo, hi, koff, kend, lut_b);  // the table and the stream slots share the shared-memory base
    const uint2 e0 = *reinterpret_cast<const uint2 *>(lut_b + __byte_perm(lo, lane8, 0x5504));
    const uint2 e1 = *reinterpret_cast<const uint2 *>(lut_b + __byte_perm(lo, lane8, 0x5514));
    const uint2 e2 = *reinterpret_cast<const uint2 *>(lut_b + __byte_perm(lo, lane8, 0x5524));
    const uint2 e3 = *reinterpret_cast<const uint2 *>(lut_b + __byte_perm(lo, lane8, 0x5534));
    const uint32_t u01 = __dp2a_lo(e1.y, e0.x, e0.y);  // r0 + f0*r1
    const uint32_t t2 = __dp2a_lo(e3.y, e2.x, e2.y);   // r2 + f2*r3
    const uint32_t p01 = __dp2a_lo(e1.x, e0.x, 0u);    // f1*f0 + sym1*0
    const uint32_t p23 = __dp2a_lo(e3.x, e2.x, 0u);    // f3*f2
    P = p01 * p23;
    const uint32_t t0 = u01 + p01 * t2;                // r0 + f0 r1 + f0 f1 (r2 + f2 r3) < P
    const unsigned long long s = (unsigned long long)hi * P + t0;
    lo = (uint32_t)s;
    hi = (uint32_t)(s >> 32);
    return __byte_perm(__byte_perm(e0.x, e1.x, 0x0062), __byte_perm(e2.x, e3.x, 0x0062), 0x5410);
}

// The narrow step over 4-byte entries at a 256-byte pitch: entry (q, lane) at byte q*256 + lane*4 from the
// start of shared memory, so that one byte permute forms each address as in the wide layout (the other 128
// bytes of each 256-byte row belong to the consumer).
__device__ __forceinline__ uint32_t q8_step_n256(uint32_t &lo, uint32_t &hi, uint32_t &koff, const uint32_t kend,
                                                 const unsigned char *lut_b, uint32_t lane4, uint32_t &P) {
    q8_refill(lo, hi, koff, kend, lut_b);
    const uint32_t e0 = *reinterpret_cast<const uint32_t *>(lut_b + __byte_perm(lo, lane4, 0x5504));
    const uint32_t e1 = *reinterpret_cast<const uint32_t *>(lut_b + __byte_perm(lo, lane4, 0x5514));
    const uint32_t e2 = *reinterpret_cast<const uint32_t *>(lut_b + __byte_perm(lo, lane4, 0x5524));
    const uint32_t e3 = *reinterpret_cast<const uint32_t *>(lut_b + __byte_perm(lo, lane4, 0x5534));
    // entry = f | sym << 16 | r << 24 (byte 1 zero, so the low half-word is exactly f)
    const uint32_t r0 = __umulhi(e0, 256u), r1 = __umulhi(e1, 256u);
    const uint32_t r2 = e2 >> 24, r3 = e3 >> 24;
    const uint32_t u01 = __dp2a_lo(r1, e0, r0);     // r0 + f0*r1
    const uint32_t t2 = __dp2a_lo(r3, e2, r2);      // r2 + f2*r3
    const uint32_t p01 = __dp2a_lo(e1, e0, 0u);     // f1*f0
    const uint32_t p23 = __dp2a_lo(e3, e2, 0u);     // f3*f2
    P = p01 * p23;
    const uint32_t t0 = u01 + p01 * t2;             // r0 + f0 r1 + f0 f1 (r2 + f2 r3) < P
    const unsigned long long st = (unsigned long long)hi * P + t0;
    lo = (uint32_t)st;
    hi = (uint32_t)(st >> 32);
    return __byte_perm(__byte_perm(e0, e1, 0x0062), __byte_perm(e2, e3, 0x0062), 0x5410);
}

// One step through whichever table layout the consumer uses; sm is the start of shared memory (where the
// wide and the 256-byte-pitch narrow tables sit), lut the lane's column of the 128-byte-pitch narrow table.
template <bool kWide, bool k256 = false>
__device__ __forceinline__ uint32_t q8_step_t(uint32_t &lo, uint32_t &hi, uint32_t &koff, const uint32_t kend,
                                              const unsigned char *sm, const uint32_t *lut, uint32_t stride, int lane,
                                              uint32_t &P) {
    if constexpr (kWide)
        return q8_step_wide(lo, hi, koff, kend, sm, (uint32_t)lane << 3, P);
    else if constexpr (k256)
        return q8_step_n256(lo, hi, koff, kend, sm, (uint32_t)lane << 2, P);
    else
        return q8_step(lo, hi, koff, kend, sm, lut, stride, P);
}

// Start of a segment's stream in the slot at byte offset soff: the lane's state (word-rows 0 and 1), the
// offset of its first refill word (word-row 2) and the bound (the row after the block's `rows` rows).
struct SegStream {
    uint32_t lo, hi, koff, kend, P;
    __device__ __forceinline__ SegStream(const unsigned char *sm, uint32_t soff, uint32_t rows, int lane) {
        const uint32_t l4 = (uint32_t)lane * 4u;
        lo = *reinterpret_cast<const uint32_t *>(sm + soff + l4);
        hi = *reinterpret_cast<const uint32_t *>(sm + soff + 128u + l4);
        koff = soff + 256u + l4;
        kend = soff + rows * 128u + l4;
        P = 0;
    }
    // the encoder starts every segment from the last quad's frequency product, so the decoder ends there
    __device__ __forceinline__ bool ok() const { return hi == 0 && lo == P; }
};

// --------------------------------------------------------------- consumers
// A consumer turns decoded quads (four int8 weights of the lane's row) into
// the kernel's output.  Per item it is set up (begin_item), fed groups of four
// quads (load_group / use) and single tail quads (single), and closes the item
// (finish_item, which may synchronise the CTA).

// y = W x, int8 x, exact int32 y (+ optional fp32 s*y).
template <int NV>
struct IntCons {
    static constexpr int kNV = NV;
    static constexpr int kRedNV = NV;
    static constexpr int kRedBufs = 2;          // alternating reduction areas: one CTA barrier per item
    static constexpr bool kFinishSyncs = true;  // finish_item holds a CTA barrier
    static constexpr int kMinCtas = 1;
    static constexpr int kMaxThreads = 512;  // up to 16 warps per CTA
    static constexpr int kTmemCols = 0;
    static constexpr bool kWideLut = true;
    static constexpr bool kLut256 = false;
    static __host__ __device__ constexpr size_t extra_bytes(int) { return 0; }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int) { return 0; }
    __device__ __forceinline__ void init(const Q8SLaunch &, unsigned char *, uint32_t, int, int, int) {}
    __device__ __forceinline__ void drain(const Q8SLaunch &) {}
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane);
    const int8_t *x;
    int cols, job_idx;
    int acc[NV];
    struct Group {
        uint4 xv[NV];
    };
    __device__ __forceinline__ void begin_item(const Q8SLaunch &L, const Q8Job &J, int, int, int job) {
        x = J.x;
        cols = J.m.cols;
        job_idx = job;
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0;
    }
    __device__ __forceinline__ void load_group(Group &g, int q) const { load_x4<NV>(x, cols, q, g.xv); }
    __device__ __forceinline__ void use(const Group &g, int j, int, uint32_t wq, int) { dot4<NV>(wq, g.xv, j, acc); }
    __device__ __forceinline__ void single(int q, uint32_t wq, int) {
        uint32_t xv[NV];
        load_x<NV>(x, cols, q, xv);
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = __dp4a((int)wq, (int)xv[v], acc[v]);
    }
    // The CTA barrier here is the only one of an item without a table rebuild: `red` alternates between two
    // areas, so the next item's partial sums never meet this item's readers.  Every warp has finished its
    // decode at the barrier, so the decode table may be rebuilt right after it.
    __device__ __forceinline__ void finish_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int warp, int lane,
                                                int W, void *red_smem) {
        int *red = reinterpret_cast<int *>(red_smem);
#pragma unroll
        for (int v = 0; v < NV; v++) red[(warp * NV + v) * 32 + lane] = acc[v];
        __syncthreads();
        const mv_q8_view &m = J.m;
        for (int t = threadIdx.x; t < NV * 32; t += blockDim.x) {
            const int v = t >> 5, l = t & 31;
            int sum = 0;
            for (int w = 0; w < W; w++) sum += red[(w * NV + v) * 32 + l];
            const int row = stripe * 32 + l;
            if (row < m.rows && v < L.batch) {
                int32_t *dst = J.y + (size_t)v * m.rows + row;
                if (J.atomic) {
                    atomicAdd(dst, sum);
                } else {
                    *dst = sum;
                    if (J.ys) J.ys[(size_t)v * m.rows + row] = (float)sum * J.scales[row];
                    if (L.chain_scales) chain_emit(L, J, job_idx, v, row, sum);
                }
            }
        }
        // a chain counts the item as done (thread 0, next) only after every output of it is stored
        if (L.chain_scales) __syncthreads();
    }
};

// four int8 weights (packed) -> fp32: the bytes biased by 128 are the low
// mantissa bits of 2^23, so each conversion is one byte permute and one add
__device__ __forceinline__ void i8x4_to_f32(uint32_t wq, float (&f)[4]) {
    const uint32_t u = wq ^ 0x80808080u;
    f[0] = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7650)) - 8388736.0f;
    f[1] = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7651)) - 8388736.0f;
    f[2] = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7652)) - 8388736.0f;
    f[3] = __uint_as_float(__byte_perm(u, 0x4B000000u, 0x7653)) - 8388736.0f;
}

__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

// Y = diag(s) W X with X bf16 [NV][cols], fp32 accumulation, fp32 Y [NV][rows] (J.ys).
template <int NV>
struct FwdCons {
    static constexpr int kNV = NV;
    static constexpr int kRedNV = NV;
    static constexpr int kRedBufs = 1;
    static constexpr bool kFinishSyncs = true;
    static constexpr int kMinCtas = 1;
    static constexpr int kMaxThreads = 512;  // 16 warps: a stripe's segments over more warps (few stripes)
    static constexpr int kTmemCols = 0;
    static constexpr bool kWideLut = true;
    static constexpr bool kLut256 = false;
    static __host__ __device__ constexpr size_t extra_bytes(int) { return 0; }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int) { return 0; }
    __device__ __forceinline__ void init(const Q8SLaunch &, unsigned char *, uint32_t, int, int, int) {}
    __device__ __forceinline__ void drain(const Q8SLaunch &) {}
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane);
    const uint16_t *x;
    int cols;
    float acc[NV];
    struct Group {
        uint4 xv[NV][2];  // 16 bf16 = 4 quads
    };
    __device__ __forceinline__ void begin_item(const Q8SLaunch &, const Q8Job &J, int, int, int) {
        x = reinterpret_cast<const uint16_t *>(J.x);
        cols = J.m.cols;
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0.f;
    }
    __device__ __forceinline__ void load_group(Group &g, int q) const {
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const uint4 *p = reinterpret_cast<const uint4 *>(x + (size_t)v * cols + 4 * q);
            g.xv[v][0] = __ldg(p);
            g.xv[v][1] = __ldg(p + 1);
        }
    }
    __device__ __forceinline__ void fma4(uint32_t wq, uint32_t xa, uint32_t xb, float &a) {
        float w[4];
        i8x4_to_f32(wq, w);
        a = fmaf(w[0], bf16_lo(xa), a);
        a = fmaf(w[1], bf16_hi(xa), a);
        a = fmaf(w[2], bf16_lo(xb), a);
        a = fmaf(w[3], bf16_hi(xb), a);
    }
    __device__ __forceinline__ void use(const Group &g, int j, int, uint32_t wq, int) {
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const uint4 &h = g.xv[v][j >> 1];
            const uint32_t xa = (j & 1) ? h.z : h.x, xb = (j & 1) ? h.w : h.y;
            fma4(wq, xa, xb, acc[v]);
        }
    }
    __device__ __forceinline__ void single(int q, uint32_t wq, int) {
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const uint2 xv = __ldg(reinterpret_cast<const uint2 *>(x + (size_t)v * cols + 4 * q));
            fma4(wq, xv.x, xv.y, acc[v]);
        }
    }
    __device__ __forceinline__ void finish_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int warp, int lane,
                                                int W, void *red_smem) {
        float *red = reinterpret_cast<float *>(red_smem);
#pragma unroll
        for (int v = 0; v < NV; v++) red[(warp * NV + v) * 32 + lane] = acc[v];
        __syncthreads();
        const mv_q8_view &m = J.m;
        for (int t = threadIdx.x; t < NV * 32; t += blockDim.x) {
            const int v = t >> 5, l = t & 31;
            float sum = 0.f;
            for (int w = 0; w < W; w++) sum += red[(w * NV + v) * 32 + l];  // fixed order: deterministic
            const int row = stripe * 32 + l;
            if (row < m.rows && v < L.batch) {
                float *dst = J.ys + (size_t)v * m.rows + row;
                const float val = sum * J.scales[row];
                if (J.atomic) atomicAdd(dst, val);
                else *dst = val;
            }
        }
        __syncthreads();
    }
};

// dX = W^T (s . dY): dY bf16 [NV][rows] (J.x), dX fp32 [NV][cols] (J.ys, zeroed,
// accumulated with fp32 atomics across stripes).  The 32 lanes of a warp are
// the 32 rows of the stripe, so the four column contributions of a quad are
// summed over the lanes with a 5-step transpose-reduce (four values in, one
// column sum in each group of 8 lanes out).
template <int NV>
struct BwdCons {
    static constexpr int kNV = NV;
    static constexpr int kRedNV = NV;
    static constexpr int kRedBufs = 1;
    static constexpr bool kFinishSyncs = false;  // no barrier in finish_item: the kernel adds one per item
    static constexpr int kMinCtas = 1;
    static constexpr int kMaxThreads = 256;
    static constexpr int kTmemCols = 0;
    static constexpr bool kWideLut = false;  // its shuffle reduction already loads the shared-memory pipe
    static constexpr bool kLut256 = false;
    static __host__ __device__ constexpr size_t extra_bytes(int) { return 0; }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int) { return 0; }
    __device__ __forceinline__ void init(const Q8SLaunch &, unsigned char *, uint32_t, int, int, int) {}
    __device__ __forceinline__ void drain(const Q8SLaunch &) {}
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane);
    float g[NV];
    float *dx;
    int cols;
    // one vector: the products of a group of 4 quads (16 columns), reduced over the lanes at once
    struct Group {
        float a[NV == 1 ? 16 : 1];
        int q0;
    };
    __device__ __forceinline__ void begin_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int lane, int) {
        const int row = stripe * 32 + lane;
        const uint16_t *dy = reinterpret_cast<const uint16_t *>(J.x);
        dx = J.ys;
        cols = J.m.cols;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            float gv = 0.f;
            if (row < J.m.rows && v < L.batch)
                gv = J.scales[row] * __uint_as_float((uint32_t)__ldg(dy + (size_t)v * J.m.rows + row) << 16);
            g[v] = gv;
        }
    }
    __device__ __forceinline__ void load_group(Group &grp, int q) const { grp.q0 = q; }
    __device__ __forceinline__ void scatter(int q, uint32_t wq, int lane) {
        float w[4];
        i8x4_to_f32(wq, w);
        const bool b4 = lane & 16, b3 = lane & 8;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const float a0 = w[0] * g[v], a1 = w[1] * g[v], a2 = w[2] * g[v], a3 = w[3] * g[v];
            float k0 = b4 ? a2 : a0, k1 = b4 ? a3 : a1;
            const float s0 = b4 ? a0 : a2, s1 = b4 ? a1 : a3;
            k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
            k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
            float k = b3 ? k1 : k0;
            const float sx = b3 ? k0 : k1;
            k += __shfl_xor_sync(0xffffffffu, sx, 8);
            k += __shfl_xor_sync(0xffffffffu, k, 4);
            k += __shfl_xor_sync(0xffffffffu, k, 2);
            k += __shfl_xor_sync(0xffffffffu, k, 1);
            // column 4q + j sits in lane 8*(2*(j>>1) + (j&1)) = lanes 0, 8, 16, 24: one
            // 16-byte vector reduction from lane 0 instead of four scalar atomics
            const float c1 = __shfl_sync(0xffffffffu, k, 8), c2 = __shfl_sync(0xffffffffu, k, 16);
            const float c3 = __shfl_sync(0xffffffffu, k, 24);
            if (lane == 0) {
                float *dst = dx + (size_t)v * cols + 4 * q;
                if (4 * q + 3 < cols) {
                    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(k), "f"(c1), "f"(c2),
                                 "f"(c3)
                                 : "memory");
                } else {
                    const float c[4] = {k, c1, c2, c3};
                    for (int jj = 0; jj < 4 && 4 * q + jj < cols; jj++) atomicAdd(dst + jj, c[jj]);
                }
            }
        }
    }
    // One vector: the 16 column products of a group (columns 4 q0 .. 4 q0 + 15) meet in one reduce-scatter
    // over the lane bits 16, 8, 4, 2 (15 shuffles) and a final butterfly, after which lane l holds the sum of
    // column 4 q0 + l / 2 and the even lanes add it to dx: 16 shuffles per 4 quads instead of 9 per quad.
    __device__ __forceinline__ void flush16(Group &grp, int lane) {
        const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float send = b4 ? grp.a[j] : grp.a[j + 8], keep = b4 ? grp.a[j + 8] : grp.a[j];
            grp.a[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float send = b3 ? grp.a[j] : grp.a[j + 4], keep = b3 ? grp.a[j + 4] : grp.a[j];
            grp.a[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const float send = b2 ? grp.a[j] : grp.a[j + 2], keep = b2 ? grp.a[j + 2] : grp.a[j];
            grp.a[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        }
        {
            const float send = b1 ? grp.a[0] : grp.a[1], keep = b1 ? grp.a[1] : grp.a[0];
            grp.a[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
        }
        grp.a[0] += __shfl_xor_sync(0xffffffffu, grp.a[0], 1);
        const int col = 4 * grp.q0 + (lane >> 1);
        if (!(lane & 1) && col < cols) atomicAdd(dx + col, grp.a[0]);
    }
    __device__ __forceinline__ void use(Group &grp, int j, int q, uint32_t wq, int lane) {
        if constexpr (NV == 1) {
            float w[4];
            i8x4_to_f32(wq, w);
#pragma unroll
            for (int i = 0; i < 4; i++) grp.a[4 * j + i] = w[i] * g[0];
            if (j == 3) flush16(grp, lane);
        } else {
            scatter(q, wq, lane);
        }
    }
    __device__ __forceinline__ void single(int q, uint32_t wq, int lane) { scatter(q, wq, lane); }
    __device__ __forceinline__ void finish_item(const Q8SLaunch &, const Q8Job &, int, int, int, int, void *) {}
};

// Decode the ILP segments of one step, feeding every quad to the consumer.
template <class Cons, int ILP>
__device__ __forceinline__ void decode_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                            const uint32_t (&rows_now)[ILP], const unsigned char *sm, uint32_t soff,
                                            const uint32_t *lut_l, int lane, Cons &cons) {
    constexpr bool kW = Cons::kWideLut;
    const int qtot = (m.cols + 3) >> 2;
    const int q0A = seg0 * m.seg_quads;
    const int nqA = rows_now[0] ? min(m.seg_quads, qtot - q0A) : 0;
    SegStream A(sm, soff, rows_now[0], lane);
    int iA = 0;
    if (ILP == 2) {
        const int q0B = (seg0 + W) * m.seg_quads;
        const int nqB = rows_now[ILP - 1] ? min(m.seg_quads, qtot - q0B) : 0;
        SegStream B(sm, soff + (uint32_t)L.buf_words * 4u, rows_now[ILP - 1], lane);
        const int nboth = min(nqA, nqB) & ~3;
        for (; iA < nboth; iA += 4) {
            typename Cons::Group ga, gb;
            cons.load_group(ga, q0A + iA);
            cons.load_group(gb, q0B + iA);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t wa = q8_step_t<kW>(A.lo, A.hi, A.koff, A.kend, sm, lut_l, L.lut_stride, lane, A.P);
                const uint32_t wb = q8_step_t<kW>(B.lo, B.hi, B.koff, B.kend, sm, lut_l, L.lut_stride, lane, B.P);
                cons.use(ga, j, q0A + iA + j, wa, lane);
                cons.use(gb, j, q0B + iA + j, wb, lane);
            }
        }
        for (int j = iA; j < nqB; j++) {
            const uint32_t wb = q8_step_t<kW>(B.lo, B.hi, B.koff, B.kend, sm, lut_l, L.lut_stride, lane, B.P);
            cons.single(q0B + j, wb, lane);
        }
        if (nqB > 0 && !B.ok()) atomicOr(L.status, MV_DEV_FINAL_STATE);
    }
    for (; iA + 4 <= nqA; iA += 4) {
        typename Cons::Group ga;
        cons.load_group(ga, q0A + iA);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t wa = q8_step_t<kW>(A.lo, A.hi, A.koff, A.kend, sm, lut_l, L.lut_stride, lane, A.P);
            cons.use(ga, j, q0A + iA + j, wa, lane);
        }
    }
    for (; iA < nqA; iA++) {
        const uint32_t wa = q8_step_t<kW>(A.lo, A.hi, A.koff, A.kend, sm, lut_l, L.lut_stride, lane, A.P);
        cons.single(q0A + iA, wa, lane);
    }
    if (nqA > 0 && !A.ok()) atomicOr(L.status, MV_DEV_FINAL_STATE);
}

template <int NV>
template <int ILP>
__device__ __forceinline__ void IntCons<NV>::run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                                      const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                                      uint32_t soff, const uint32_t *lut_l, int lane) {
    decode_step<IntCons<NV>, ILP>(L, m, seg0, W, rows_now, sm, soff, lut_l, lane, *this);
}
template <int NV>
template <int ILP>
__device__ __forceinline__ void FwdCons<NV>::run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                                      const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                                      uint32_t soff, const uint32_t *lut_l, int lane) {
    decode_step<FwdCons<NV>, ILP>(L, m, seg0, W, rows_now, sm, soff, lut_l, lane, *this);
}
template <int NV>
template <int ILP>
__device__ __forceinline__ void BwdCons<NV>::run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int W,
                                                      const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                                      uint32_t soff, const uint32_t *lut_l, int lane) {
    decode_step<BwdCons<NV>, ILP>(L, m, seg0, W, rows_now, sm, soff, lut_l, lane, *this);
}

// y = W x for 8..16 int8 vectors on the tensor cores.  Every 16 decoded quads
// the 32 lanes of a warp (= the 32 rows of the stripe) hold a 32 x 64 int8
// tile of W, one row per lane: each lane writes its row straight from
// registers into its own TMEM lane (tcgen05.st, 8 quads at a time), and one
// lane issues two tcgen05.mma.kind::i8 (K = 32 each) with A = that tile in
// TMEM (M = 128: the warp's lane quarter holds its 32 rows, the other lanes
// are never written and their results never read), B = the x tile in shared
// memory (N = 16 vectors, K-major core matrices of 8 rows x 16 bytes),
// accumulating exactly in int32 in the warp's own 16 TMEM columns.  Each warp
// owns 32 TMEM columns: D [0,16) and the A tile [16,32).  One tcgen05.commit
// per 16 quads arrives on the warp's mbarrier; the A tile is rewritten only
// after the previous pair of MMAs completed (issued a whole 16-quad decode
// earlier, so the wait is normally already over).  x moves through a
// 128-column window (4 x 32 columns x 16 vectors, 2 KB per warp); the next
// window is loaded while the current one is in use.  ILP 1 only.
//
// Shared memory: the decode table takes 4-byte entries at a 256-byte pitch
// (entry (q, lane) at byte q*256 + lane*4, one byte permute per address), and
// the x tiles of warps 0..7 live in the other half of each 256-byte row: 256
// holes of 128 bytes, one core matrix each, 32 per warp (two tiles of 16).
// Core matrix c = t*16 + p*4 + n*2 + k ((n, k) of piece p of tile t) sits at
// base + c * stride: stride 256 B in the holes (LBO, K direction, 256 B; SBO,
// N direction, 512 B), 128 B for warps 8..15, whose tiles are contiguous
// behind the table (LBO 128, SBO 256).  64 KB hold table and eight warps' x
// tiles, as much as the 32 KB table with separate x tiles, so two 8-warp CTAs
// still fit an SM.  The tiles also take the cross-warp reduction.
struct MmaCons {
    static constexpr int kNV = 16;
    static constexpr int kRedNV = 0;      // reduction area: the x tiles
    static constexpr int kRedBufs = 1;
    static constexpr bool kFinishSyncs = true;
    static constexpr int kMinCtas = 1;    // with up to 16 warps: at most 128 registers per thread
    static constexpr int kMaxThreads = 512;  // 2 x 8 warps per SM (stacks) or 1 x 16 (chains)
    static constexpr int kTmemCols = 1;   // > 0: the kernel allocates TMEM
    static constexpr bool kWideLut = false;
    static constexpr bool kLut256 = true;  // 4-byte entries at a 256-byte pitch, x tiles in between
    static constexpr int kXChunks = 4;    // x tile: 4 pieces of 32 columns x 16 vectors (512 B each)
    static constexpr int kXBytes = kXChunks * 512;
    static constexpr uint32_t kHoles = kXBytes / 128;  // core matrices per tile
    // x tiles of warps 8..15 (4 KB each) at the start of the consumer region
    static __host__ __device__ constexpr size_t xr_bytes(int W) { return W > 8 ? (size_t)(W - 8) * 2 * kXBytes : 0; }
    static __host__ __device__ constexpr size_t extra_bytes(int W) {
        // those x tiles, three mbarriers per warp (MMA commits, x copies into tile 0 / 1), TMEM address slot
        // (the last 128 bytes); a multiple of 128 bytes, so the stream buffers that follow stay 16-byte
        // aligned
        return ((xr_bytes(W) + (size_t)W * 24 + 128) + 127) / 128 * 128;
    }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int) { return 0; }
    static __host__ __device__ constexpr uint32_t tmem_cols(int W) {
        return W <= 1 ? 32 : W <= 2 ? 64 : W <= 4 ? 128 : W <= 8 ? 256 : 512;
    }
    // warp w's core matrix 0 of tile 0 (byte offset from the start of shared memory) and core-matrix stride
    static __device__ __forceinline__ uint32_t tile_base(const Q8SLaunch &L, int w) {
        return w < 8 ? (uint32_t)w * (2u * kHoles) * 256u + 128u : L.lay.extra + (uint32_t)(w - 8) * 2u * kXBytes;
    }
    static __device__ __forceinline__ uint32_t tile_stride(int w) { return w < 8 ? 256u : 128u; }
    uint32_t xt, d_tmem, st_addr, ld_addr, ncommit, xcur, xcnt0, xcnt1, xb, cst;
    uint64_t b_desc0;
    uint32_t mbar, xbar;  // shared-memory addresses: the MMA barrier, the two x-window barriers (8 bytes apart)
    unsigned char *sm0;  // start of shared memory (table and holes)
    const int8_t *x;
    const int8_t *tiles;  // x laid out per (segment, window) by q8s_build_x_tiles, or null
    int cols, batch, job_idx, nwin;
    bool any;

    __device__ __forceinline__ void init(const Q8SLaunch &L, unsigned char *extra, uint32_t tmem_base, int,
                                         int lane, int W) {
        // the warp index through a shuffle from lane 0 is known warp-uniform to the compiler, so the MMA
        // operands derived from it stay in uniform registers
        const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
        sm0 = extra - L.lay.extra;  // the table (and its holes) starts shared memory
        xb = tile_base(L, warp);
        cst = tile_stride(warp);
        xt = smem_u32(sm0) + xb;  // tile 0, core matrix 0
        uint64_t *mb = reinterpret_cast<uint64_t *>(extra + xr_bytes(W)) + warp;
        uint64_t *xbp = reinterpret_cast<uint64_t *>(extra + xr_bytes(W) + (size_t)W * 8) + 2 * warp;
        if (lane == 0) {
            mbar_init(mb, 1);
            mbar_init(&xbp[0], 32);  // x windows: one arrival per lane (x_copy)
            mbar_init(&xbp[1], 32);
        }
        mbar = smem_u32(mb);
        xbar = smem_u32(xbp);
        fence_mbar_init();
        __syncwarp();
        // TMEM addresses: lane in bits [16,32), column in [0,16); a warp may touch only the 32 lanes of its
        // quarter (warp % 4) with tcgen05.ld/st, while an MMA with M = 128 addresses lanes from 0
        const uint32_t quarter = ((uint32_t)(warp & 3) * 32u) << 16;
        d_tmem = tmem_base + 32u * (uint32_t)warp;
        st_addr = d_tmem + 16u + quarter;
        ld_addr = d_tmem + quarter;
        b_desc0 = umma_smem_desc(xt, cst, 2u * cst);
        ncommit = 0;
        xcur = 1;  // the x tile of the latest window; a segment's first window goes to the other one
        xcnt0 = xcnt1 = 0;
    }
    __device__ __forceinline__ void begin_item(const Q8SLaunch &L, const Q8Job &J, int, int, int job) {
        x = J.x;
        cols = J.m.cols;
        batch = L.batch;
        any = false;
        job_idx = job;
        tiles = J.x_tiles;
        nwin = (J.m.seg_quads + 31) / 32;
    }
    // Asynchronous copies of x window w of segment seg (2 KB, contiguous in the x tiles) into tile t: lane l
    // copies the 16-byte rows l, l + 32, l + 64, l + 96 (row k = row k % 8 of core matrix k / 8, which sits in
    // its own hole) and then arrives on the tile's barrier once its copies have landed.  Every lane counts
    // the window.  The tile's previous readers (MMAs) are done.  Per-lane 16-byte copies rather than one
    // 128-byte bulk copy per core matrix: bulk copies take warp-uniform operands, so sixteen lanes each
    // issuing one compiled to a loop over the lanes that cost about 8 instructions per decode step.
    __device__ __forceinline__ void x_copy(int t, int seg, int w, int lane) {
        const int8_t *src = tiles + ((size_t)seg * nwin + w) * kXBytes;
        const uint32_t dst = xt + (uint32_t)t * kHoles * cst;
#pragma unroll
        for (uint32_t i = 0; i < kXBytes / 512; i++) {
            const uint32_t k = (uint32_t)lane + 32u * i;
            cp_async_16(dst + (k >> 3) * cst + (k & 7u) * 16u, src + (size_t)k * 16);
        }
        cp_async_mbar_arrive_noinc(xbar + 8u * (uint32_t)t);
        if (t) xcnt1++;
        else xcnt0++;
    }
    // The window's copies (generic proxy) are visible to every lane once the barrier phase completes; the
    // proxy fence orders them before the tensor core's reads of the tile (async proxy).
    __device__ __forceinline__ void x_wait(const Q8SLaunch &L, int t) {
        const uint32_t n = t ? xcnt1 : xcnt0;
        // on a timeout (flagged) wait once more, bounded, so that no copy is left in flight
        const uint32_t bar = xbar + 8u * (uint32_t)t;
        if (!mbar_wait_bounded(bar, (n - 1) & 1, L.status, L.spin_limit))
            mbar_wait_bounded(bar, (n - 1) & 1, nullptr, L.spin_limit);
        fence_proxy_async_smem();
    }
    // wait until every MMA issued so far completed (the latest commit covers all earlier MMAs)
    __device__ __forceinline__ bool wait_mma(const Q8SLaunch &L) {
        if (ncommit == 0) return true;
        return mbar_wait_bounded(mbar, (ncommit - 1) & 1, L.status, L.spin_limit);
    }
    __device__ __forceinline__ void issue(int piece, bool two) {
        tcgen05_fence_before();
        __syncwarp();
        if (elect_one()) {
            tcgen05_fence_after();
            // B descriptor start addresses are in 16-byte units: tile xcur is 16 core matrices in, piece p 4
            const uint32_t idesc = umma_idesc_i8(128, 16);
            const uint64_t bd = b_desc0 + (uint64_t)(xcur * cst + (uint32_t)piece * (cst / 4u));
            umma_i8_ts(d_tmem, d_tmem + 16u, bd, idesc, any ? 1u : 0u);
            if (two) umma_i8_ts(d_tmem, d_tmem + 24u, bd + cst / 4u, idesc, 1u);  // the next piece
            umma_commit(mbar);
        }
        __syncwarp();
        any = true;
        ncommit++;
    }
    // lane (b, h) holds 16 bytes (column half h) of vector b for each 32-column piece of a window
    __device__ __forceinline__ void load_window(uint4 (&xr)[kXChunks], const int8_t *xrow, bool xok, int colbase,
                                                int pbase, int npieces) const {
        if (xok && pbase + kXChunks <= npieces && colbase + 32 * (pbase + kXChunks - 1) < cols) {
            // a full window inside the row: plain loads, no per-piece checks
#pragma unroll
            for (int i = 0; i < kXChunks; i++) xr[i] = ldx_u4(xrow + 32 * (pbase + i));
            return;
        }
#pragma unroll
        for (int i = 0; i < kXChunks; i++) {
            const int c = pbase + i;
            xr[i] = make_uint4(0, 0, 0, 0);
            // cols % 16 == 0, so a 16-byte piece that starts inside the row ends inside it
            if (xok && c < npieces && colbase + 32 * c < cols) xr[i] = ldx_u4(xrow + 32 * c);
        }
    }
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane) {
        const int qtot = (m.cols + 3) >> 2;
        const int q0 = seg0 * m.seg_quads;
        const int nq = rows_now[0] ? min(m.seg_quads, qtot - q0) : 0;
        if (nq <= 0) return;
        const int npieces = (nq + 7) >> 3;  // 32-column pieces (8 quads each)
        const int b = lane >> 1, h = lane & 1;
        const bool xok = b < batch;
        const int colbase = 4 * q0 + 16 * h;
        const int8_t *xrow = x + (size_t)(xok ? b : 0) * cols + colbase;
        // core matrix (n, k) = (b / 8, h) of piece i is core matrix 4 i + 2 n + k of tile 0, row b % 8
        const uint32_t xdst = xt + ((uint32_t)(b >> 3) * 2u + (uint32_t)h) * cst + (uint32_t)(b & 7) * 16u;
        uint4 xr[kXChunks];
        // with x tiles: the first window goes to the tile the latest window did not use (its MMAs completed
        // before the latest window started); without: windows pass through registers into tile 0
        int xnext = xcur ^ 1u;
        if (tiles) {
            x_copy(xnext, seg0, 0, lane);
        } else {
            xcur = 0;
            load_window(xr, xrow, xok, colbase, 0, npieces);
        }
        SegStream S(sm, soff, rows_now[0], lane);
        // pieces in pairs: piece p = 2 * pair (+1); a window holds 2 pairs.  A pair of two full pieces (16
        // quads) takes the body without the tail tests; the segment's last pair may be partial.
        auto pair = [&](const int p, auto full) {
            constexpr bool kFull = decltype(full)::value;
            uint32_t w[8];
            const int qc = 8 * p;
            if (kFull || qc + 8 <= nq) {
#pragma unroll
                for (int j = 0; j < 8; j++) w[j] = q8_step_t<kWideLut, kLut256>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, L.lut_stride, lane, S.P);
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++)
                    w[j] = (qc + j < nq) ? q8_step_t<kWideLut, kLut256>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, L.lut_stride, lane, S.P) : 0u;
            }
            // the previous pair of MMAs is done with the A tile (and, at a window start, with the x tile)
            wait_mma(L);
            const int pw = p & (kXChunks - 1);  // piece within the window
            if (pw == 0 && tiles) {
                // this window's copy has landed (it was the only one in flight); the next goes to the other
                // tile, whose MMAs are done (above)
                x_wait(L, xnext);
                xcur = xnext;
                if (p + kXChunks < npieces) {
                    xnext = xcur ^ 1u;
                    x_copy(xnext, seg0, (p + kXChunks) / kXChunks, lane);
                }
            } else if (pw == 0) {
                // the whole window is stored (pieces past the segment hold zeros or stale x, and are never
                // multiplied: the MMAs of a pair read only the pieces that exist)
#pragma unroll
                for (int i = 0; i < kXChunks; i++)
                    asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" ::"r"(xdst + (uint32_t)i * 4u * cst),
                                 "r"(xr[i].x), "r"(xr[i].y), "r"(xr[i].z), "r"(xr[i].w)
                                 : "memory");
                fence_proxy_async_smem();  // the x tile is read by the tensor core (async proxy)
                if (p + kXChunks < npieces) load_window(xr, xrow, xok, colbase, p + kXChunks, npieces);
            }
            tcgen05_fence_after();
            tmem_st_32x32b_x8_nowait(st_addr, w);
            const bool two = kFull || p + 1 < npieces;
            if (two) {
                const int qc2 = qc + 8;
                if (kFull || qc2 + 8 <= nq) {
#pragma unroll
                    for (int j = 0; j < 8; j++) w[j] = q8_step_t<kWideLut, kLut256>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, L.lut_stride, lane, S.P);
                } else {
#pragma unroll
                    for (int j = 0; j < 8; j++)
                        w[j] = (qc2 + j < nq) ? q8_step_t<kWideLut, kLut256>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, L.lut_stride, lane, S.P) : 0u;
                }
                tmem_st_32x32b_x8_nowait(st_addr + 8u, w);
            }
            tmem_wait_st();
            issue(pw, two);
        };
        const int pfull = (nq >> 4) << 1;  // pieces covered by full pairs
        for (int p = 0; p < pfull; p += 2) pair(p, std::true_type{});
        if (pfull < npieces) pair(pfull, std::false_type{});
        if (!S.ok()) atomicOr(L.status, MV_DEV_FINAL_STATE);
    }
    __device__ __forceinline__ void finish_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int warp, int lane,
                                                int W, void *) {
        uint32_t r[16];
        if (any) {
            wait_mma(L);
            tcgen05_fence_after();
            tmem_ld_32x32b_x16(ld_addr, r);  // lane = stripe row, r[v] = vector v
        } else {
#pragma unroll
            for (int v = 0; v < 16; v++) r[v] = 0;
        }
        // this warp's MMAs (and x copies) are complete, so its own x tiles take its partial sums: vector v
        // of stripe row l in core matrix v of tile 0, word l
#pragma unroll
        for (int v = 0; v < 16; v++) *reinterpret_cast<int *>(sm0 + xb + (uint32_t)v * cst + 4 * lane) = (int)r[v];
        tcgen05_fence_before();
        __syncthreads();
        const mv_q8_view &m = J.m;
        const int W8 = min(W, 8);
        for (int t = threadIdx.x; t < 16 * 32; t += blockDim.x) {
            const int v = t >> 5, l = t & 31;
            int sum = 0;
            // warps 0..7: tile 0 at hole 32 w (byte 8192 w + 128), core matrix v one 256-byte row further
            const unsigned char *h = sm0 + 128u + (uint32_t)v * 256u + 4u * (uint32_t)l;
#pragma unroll
            for (int w = 0; w < 8; w++)
                if (w < W8) sum += *reinterpret_cast<const int *>(h + (uint32_t)w * 2u * kHoles * 256u);
            for (int w = 8; w < W; w++)
                sum += *reinterpret_cast<const int *>(sm0 + tile_base(L, w) + (uint32_t)v * tile_stride(w) + 4 * l);
            const int row = stripe * 32 + l;
            if (row < m.rows && v < L.batch) {
                int32_t *dst = J.y + (size_t)v * m.rows + row;
                if (J.atomic) {
                    atomicAdd(dst, sum);
                } else {
                    *dst = sum;
                    if (J.ys) J.ys[(size_t)v * m.rows + row] = (float)sum * J.scales[row];
                    if (L.chain_scales) chain_emit(L, J, job_idx, v, row, sum);
                }
            }
        }
        fence_proxy_async_smem();  // these generic accesses come before the tensor core's later reads of the tiles
        __syncthreads();  // the x tiles are written again (tables, x) by the next item
    }
    __device__ __forceinline__ void drain(const Q8SLaunch &L) {
        wait_mma(L);
        cp_async_wait_all();  // no x copy is left writing shared memory after the CTA exits
    }
};

// four int8 weights (packed) -> four bf16 (exact: |w| <= 127 needs 7 significand bits), as two bf16x2
// words in column order: lo = (w0, w1), hi = (w2, w3)
__device__ __forceinline__ void i8x4_to_bf16x4(uint32_t wq, uint32_t &lo, uint32_t &hi) {
    float f[4];
    i8x4_to_f32(wq, f);
    lo = __byte_perm(__float_as_uint(f[0]), __float_as_uint(f[1]), 0x7632);
    hi = __byte_perm(__float_as_uint(f[2]), __float_as_uint(f[3]), 0x7632);
}

// Decode one 8-quad piece of the lane's row (zeros past nq).
template <bool kWide>
__device__ __forceinline__ void decode_piece(int qc, int nq, SegStream &S, const unsigned char *sm,
                                             const uint32_t *lut_l, uint32_t stride, int lane, uint32_t (&w)[8]) {
    if (qc + 8 <= nq) {
#pragma unroll
        for (int j = 0; j < 8; j++) w[j] = q8_step_t<kWide>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, stride, lane, S.P);
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++)
            w[j] = (qc + j < nq) ? q8_step_t<kWide>(S.lo, S.hi, S.koff, S.kend, sm, lut_l, stride, lane, S.P) : 0u;
    }
}

// Float forward on the tensor cores: Y = diag(s) W X for up to 16 bf16 vectors,
// fp32 accumulation (kind::f16 MMAs, bf16 A and B: the int8 weights and the bf16
// inputs are exact in bf16, every product is exact in fp32).  Per 8 decoded
// quads each lane converts its 32 weights to bf16 and stores them into its
// TMEM lane (A, 16 columns); one lane issues two MMAs (K = 16 each) against the
// x tile (B: 16 vectors x 32 columns of bf16, K-major core matrices, 1 KB) into
// the warp's 16 fp32 D columns.  x moves through a 2-piece window (2 KB per
// warp) loaded into registers ahead of use.  The x tiles hold the cross-warp
// reduction (fixed order) at the end of a stripe and stage the decode tables.
struct FwdMma {
    static constexpr int kNV = 16;
    static constexpr int kRedNV = 0;
    static constexpr int kRedBufs = 1;
    static constexpr bool kFinishSyncs = true;
    static constexpr int kMinCtas = 2;
    static constexpr int kMaxThreads = 256;
    static constexpr int kTmemCols = 1;
    static constexpr bool kWideLut = false;
    static constexpr bool kLut256 = false;
    static constexpr int kXPieces = 2;
    static constexpr int kXBytes = kXPieces * 1024;
    static __host__ __device__ constexpr size_t extra_bytes(int W) {
        return (((size_t)W * kXBytes + (size_t)W * 8 + 128) + 127) / 128 * 128;
    }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int W) { return (size_t)W * kXBytes; }
    uint32_t xt, d_tmem, st_addr, ld_addr, ncommit;
    uint64_t b_desc0;
    uint64_t *mbar;
    float *xbase;
    const uint16_t *x;
    int cols, batch;
    bool any;

    __device__ __forceinline__ void init(const Q8SLaunch &, unsigned char *extra, uint32_t tmem_base, int, int lane,
                                         int W) {
        const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
        const uint32_t base = smem_u32(extra);
        xbase = reinterpret_cast<float *>(extra);
        xt = base + (uint32_t)warp * (uint32_t)kXBytes;
        mbar = reinterpret_cast<uint64_t *>(extra + (size_t)W * kXBytes) + warp;
        if (lane == 0) mbar_init(mbar, 1);
        fence_mbar_init();
        __syncwarp();
        const uint32_t quarter = ((uint32_t)(warp & 3) * 32u) << 16;
        d_tmem = tmem_base + 32u * (uint32_t)warp;
        st_addr = d_tmem + 16u + quarter;
        ld_addr = d_tmem + quarter;
        b_desc0 = umma_smem_desc(xt, 128u, 256u);
        ncommit = 0;
    }
    __device__ __forceinline__ void begin_item(const Q8SLaunch &L, const Q8Job &J, int, int, int) {
        x = reinterpret_cast<const uint16_t *>(J.x);
        cols = J.m.cols;
        batch = L.batch;
        any = false;
    }
    __device__ __forceinline__ bool wait_mma(const Q8SLaunch &L) {
        if (ncommit == 0) return true;
        return mbar_wait_bounded(mbar, (ncommit - 1) & 1, L.status, L.spin_limit);
    }
    // lane (b, hh) moves vector b's 8-column chunks 2*hh and 2*hh+1 of each 32-column piece of a window
    __device__ __forceinline__ void load_window(uint4 (&xr)[2 * kXPieces], const uint16_t *xrow, bool xok,
                                                int colbase, int pbase, int npieces) const {
#pragma unroll
        for (int i = 0; i < kXPieces; i++) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int p = pbase + i;
                const int off = 32 * p + 8 * j;  // columns from xrow
                xr[2 * i + j] = make_uint4(0, 0, 0, 0);
                // cols % 16 == 0: an 8-column chunk that starts inside the row ends inside it
                if (xok && p < npieces && colbase + off < cols)
                    xr[2 * i + j] = __ldg(reinterpret_cast<const uint4 *>(xrow + off));
            }
        }
    }
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane) {
        const int qtot = (m.cols + 3) >> 2;
        const int q0 = seg0 * m.seg_quads;
        const int nq = rows_now[0] ? min(m.seg_quads, qtot - q0) : 0;
        if (nq <= 0) return;
        const int npieces = (nq + 7) >> 3;
        const int b = lane >> 1, hh = lane & 1;
        const bool xok = b < batch;
        const int colbase = 4 * q0 + 16 * hh;
        const uint16_t *xrow = x + (size_t)(xok ? b : 0) * cols + colbase;
        // chunk c8 = 2 hh + j of a piece: K step c8 >> 1 (512 B), K half c8 & 1 (128 B)
        const uint32_t xdst = xt + (uint32_t)hh * 512u + (uint32_t)(b >> 3) * 256u + (uint32_t)(b & 7) * 16u;
        uint4 xr[2 * kXPieces];
        load_window(xr, xrow, xok, colbase, 0, npieces);
        SegStream S(sm, soff, rows_now[0], lane);
        for (int p = 0; p < npieces; p++) {
            uint32_t w[8];
            decode_piece<kWideLut>(8 * p, nq, S, sm, lut_l, L.lut_stride, lane, w);
            uint32_t a[16];
#pragma unroll
            for (int j = 0; j < 8; j++) i8x4_to_bf16x4(w[j], a[2 * j], a[2 * j + 1]);
            wait_mma(L);  // the previous MMAs are done with the A columns (and the x tile)
            const int pw = p & (kXPieces - 1);
            if (pw == 0) {
                const int cn = min(kXPieces, npieces - p);
#pragma unroll
                for (int i = 0; i < kXPieces; i++)
                    if (i < cn) {
#pragma unroll
                        for (int j = 0; j < 2; j++) {
                            const uint4 v = xr[2 * i + j];
                            asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" ::"r"(
                                             xdst + (uint32_t)i * 1024u + (uint32_t)j * 128u),
                                         "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                                         : "memory");
                        }
                    }
                fence_proxy_async_smem();
                if (p + kXPieces < npieces) load_window(xr, xrow, xok, colbase, p + kXPieces, npieces);
            }
            tcgen05_fence_after();
            tmem_st_32x32b_x16_nowait(st_addr, a);
            tmem_wait_st();
            tcgen05_fence_before();
            __syncwarp();
            if (elect_one()) {
                tcgen05_fence_after();
                const uint32_t idesc = umma_idesc_bf16(128, 16, 0, 0);
                const uint64_t bd = b_desc0 + (uint64_t)(pw * 64);  // 1 KB per piece, in 16-byte units
                umma_f16_ts(d_tmem, d_tmem + 16u, bd, idesc, any ? 1u : 0u);
                umma_f16_ts(d_tmem, d_tmem + 24u, bd + 32u, idesc, 1u);
                umma_commit(mbar);
            }
            __syncwarp();
            any = true;
            ncommit++;
        }
        if (!S.ok()) atomicOr(L.status, MV_DEV_FINAL_STATE);
    }
    __device__ __forceinline__ void finish_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int warp, int lane,
                                                int W, void *) {
        uint32_t r[16];
        if (any) {
            wait_mma(L);
            tcgen05_fence_after();
            tmem_ld_32x32b_x16(ld_addr, r);  // lane = stripe row, r[v] = vector v (fp32 bits)
        } else {
#pragma unroll
            for (int v = 0; v < 16; v++) r[v] = 0;
        }
        float *red = xbase + warp * (kXBytes / 4);
#pragma unroll
        for (int v = 0; v < 16; v++) red[v * 32 + lane] = __uint_as_float(r[v]);
        tcgen05_fence_before();
        __syncthreads();
        const mv_q8_view &m = J.m;
        for (int t = threadIdx.x; t < 16 * 32; t += blockDim.x) {
            const int v = t >> 5, l = t & 31;
            float sum = 0.f;
            for (int w = 0; w < W; w++) sum += xbase[w * (kXBytes / 4) + t];  // fixed order: deterministic
            const int row = stripe * 32 + l;
            if (row < m.rows && v < L.batch) {
                float *dst = J.ys + (size_t)v * m.rows + row;
                const float val = sum * J.scales[row];
                if (J.atomic) atomicAdd(dst, val);
                else *dst = val;
            }
        }
        __syncthreads();
    }
    __device__ __forceinline__ void drain(const Q8SLaunch &L) { wait_mma(L); }
};

// Float backward on the tensor cores: dX = W^T (s . dY) for up to 32 bf16
// vectors.  Per stripe the CTA builds G = s . dY for its 32 rows as a pair of
// bf16 tiles, hi = bf16(g) and lo = bf16(g - hi), so that hi + lo carries g to
// ~16 significant bits (K-major, 32 vectors x 32 rows, 4 KB, shared by the
// warps).  Per 8 decoded quads each lane converts its 32 weights to bf16 and
// writes them into the warp's W tile in shared memory (MN-major: the tile is
// B = W^T's transpose as stored, N = 32 columns, K = 32 rows); one lane issues
// four MMAs (K = 16 rows each, hi and lo) with A = G (M = 128, the start moved
// back by the warp's lane quarter so that vector v lands in TMEM lane
// 32 (warp % 4) + v; the other rows are ignored) into the warp's 32 fp32 D
// columns.  The D tile of a piece is read back while the next piece decodes
// and added to dX (fp32, zeroed by the launcher) with 16-byte vector reductions.
struct BwdMma {
    static constexpr int kNV = 32;
    static constexpr int kRedNV = 0;
    static constexpr int kRedBufs = 1;
    static constexpr bool kFinishSyncs = true;
    static constexpr int kMinCtas = 2;
    static constexpr int kMaxThreads = 256;
    static constexpr int kTmemCols = 1;
    static constexpr bool kWideLut = false;
    static constexpr bool kLut256 = false;
    static constexpr int kGBytes = 4096;  // [hi, lo][K step 0, 1] x 1 KB
    static constexpr int kWBytes = 2048;  // W tile per warp: 2 K steps x 1 KB
    static __host__ __device__ constexpr size_t extra_bytes(int W) {
        // G, W tiles, one mbarrier per warp, TMEM slot; at least the span an A operand reads (16 row groups of
        // 256 B from the last G tile), so that the ignored rows never reach past this region
        return ((std::max<size_t>((size_t)kGBytes + (size_t)W * kWBytes + (size_t)W * 8 + 128,
                                  (size_t)3 * 1024 + 16 * 256 + 128)) +
                127) /
               128 * 128;
    }
    static __host__ __device__ constexpr size_t tbl_alias_bytes(int W) { return (size_t)kGBytes + (size_t)W * kWBytes; }
    uint32_t gbase, wt, d_tmem, ld_addr, ncommit, quarter_off;
    uint64_t *mbar;
    float *dx;
    int cols, rows, batch, pend_col;
    bool pending;

    __device__ __forceinline__ void init(const Q8SLaunch &, unsigned char *extra, uint32_t tmem_base, int, int lane,
                                         int W) {
        const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
        gbase = smem_u32(extra);
        wt = gbase + (uint32_t)kGBytes + (uint32_t)warp * (uint32_t)kWBytes;
        mbar = reinterpret_cast<uint64_t *>(extra + kGBytes + (size_t)W * kWBytes) + warp;
        if (lane == 0) mbar_init(mbar, 1);
        fence_mbar_init();
        __syncwarp();
        quarter_off = (uint32_t)(warp & 3) * 1024u;  // 32 rows of A = 4 groups of 256 B
        d_tmem = tmem_base + 32u * (uint32_t)warp;
        ld_addr = d_tmem + (((uint32_t)(warp & 3) * 32u) << 16);
        ncommit = 0;
        pending = false;
    }
    __device__ __forceinline__ bool wait_mma(const Q8SLaunch &L) {
        if (ncommit == 0) return true;
        return mbar_wait_bounded(mbar, (ncommit - 1) & 1, L.status, L.spin_limit);
    }
    // CTA-wide (every warp calls it for the same item): G = s . dY of the stripe as bf16 hi/lo tiles
    __device__ __forceinline__ void begin_item(const Q8SLaunch &L, const Q8Job &J, int stripe, int, int) {
        const uint16_t *dy = reinterpret_cast<const uint16_t *>(J.x);
        dx = J.ys;
        cols = J.m.cols;
        rows = J.m.rows;
        batch = L.batch;
        pending = false;
        for (int t = threadIdx.x; t < 32 * 32; t += blockDim.x) {
            const int v = t >> 5, r = t & 31;  // vector, stripe row
            const int row = stripe * 32 + r;
            float g = 0.f;
            if (row < rows && v < batch)
                g = J.scales[row] * __uint_as_float((uint32_t)__ldg(dy + (size_t)v * rows + row) << 16);
            const __nv_bfloat16 h = __float2bfloat16_rn(g);
            const __nv_bfloat16 l = __float2bfloat16_rn(g - __bfloat162float(h));
            // K-major core matrices: vector group v/8 at 256 B, K half (r % 16) / 8 at 128 B, K step r / 16
            const uint32_t off = (uint32_t)(r >> 4) * 1024u + (uint32_t)(v >> 3) * 256u +
                                 (uint32_t)((r >> 3) & 1) * 128u + (uint32_t)(v & 7) * 16u + (uint32_t)(r & 7) * 2u;
            asm volatile("st.shared.u16 [%0], %1;" ::"r"(gbase + off), "h"(__bfloat16_as_ushort(h)) : "memory");
            asm volatile("st.shared.u16 [%0], %1;" ::"r"(gbase + 2048u + off), "h"(__bfloat16_as_ushort(l))
                         : "memory");
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
    // add the finished D tile (vectors x 32 columns at pend_col) to dX
    __device__ __forceinline__ void flush(const Q8SLaunch &L, int lane) {
        wait_mma(L);
        tcgen05_fence_after();
        uint32_t r[32];
        tmem_ld_32x32b_x32(ld_addr, r);  // lane = vector, r[j] = column pend_col + j
        if (lane < batch) {
            float *dst = dx + (size_t)lane * cols + pend_col;
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                if (pend_col + j < cols)  // cols % 16 == 0: a 4-column group inside the row stays inside
                    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst + j),
                                 "f"(__uint_as_float(r[j])), "f"(__uint_as_float(r[j + 1])),
                                 "f"(__uint_as_float(r[j + 2])), "f"(__uint_as_float(r[j + 3]))
                                 : "memory");
        }
        tcgen05_fence_before();
        pending = false;
    }
    template <int ILP>
    __device__ __forceinline__ void run_step(const Q8SLaunch &L, const mv_q8_view &m, int seg0, int,
                                             const uint32_t (&rows_now)[ILP], const unsigned char *sm,
                                             uint32_t soff, const uint32_t *lut_l, int lane) {
        const int qtot = (m.cols + 3) >> 2;
        const int q0 = seg0 * m.seg_quads;
        const int nq = rows_now[0] ? min(m.seg_quads, qtot - q0) : 0;
        if (nq <= 0) return;
        const int npieces = (nq + 7) >> 3;
        SegStream S(sm, soff, rows_now[0], lane);
        // lane = stripe row r: K step r / 16, K group (r / 8) % 2 (128 B), row r % 8 (16 B); N group g at 256 B
        const uint32_t wdst = wt + (uint32_t)(lane >> 4) * 1024u + (uint32_t)((lane >> 3) & 1) * 128u +
                              (uint32_t)(lane & 7) * 16u;
        for (int p = 0; p < npieces; p++) {
            uint32_t w[8];
            decode_piece<kWideLut>(8 * p, nq, S, sm, lut_l, L.lut_stride, lane, w);
            uint32_t a[16];
#pragma unroll
            for (int j = 0; j < 8; j++) i8x4_to_bf16x4(w[j], a[2 * j], a[2 * j + 1]);
            if (pending) flush(L, lane);  // also: the previous MMAs are done with the W tile
#pragma unroll
            for (int g = 0; g < 4; g++)
                asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" ::"r"(wdst + (uint32_t)g * 256u), "r"(a[4 * g]),
                             "r"(a[4 * g + 1]), "r"(a[4 * g + 2]), "r"(a[4 * g + 3])
                             : "memory");
            fence_proxy_async_smem();
            __syncwarp();
            if (elect_one()) {
                tcgen05_fence_after();
                const uint32_t idesc = umma_idesc_bf16(128, 32, 0, 1);
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
                    const uint64_t bd = umma_smem_desc(wt + (uint32_t)kk * 1024u, 128u, 256u);
                    const uint32_t ga = gbase + (uint32_t)kk * 1024u - quarter_off;
                    umma_f16_ss(d_tmem, umma_smem_desc(ga, 128u, 256u), bd, idesc, kk ? 1u : 0u);
                    umma_f16_ss(d_tmem, umma_smem_desc(ga + 2048u, 128u, 256u), bd, idesc, 1u);
                }
                umma_commit(mbar);
            }
            __syncwarp();
            ncommit++;
            pending = true;
            pend_col = 4 * q0 + 32 * p;
        }
        if (!S.ok()) atomicOr(L.status, MV_DEV_FINAL_STATE);
    }
    __device__ __forceinline__ void finish_item(const Q8SLaunch &L, const Q8Job &, int, int, int lane, int, void *) {
        if (pending) flush(L, lane);
        __syncthreads();  // G and the W tiles are rewritten by the next item
    }
    __device__ __forceinline__ void drain(const Q8SLaunch &L) { wait_mma(L); }
};

// Chained pipeline: wait (one thread, bounded, then the whole CTA) until every work item of job j is
// counted.  Work items are numbered in job order and each CTA takes its items in increasing order, and
// the launch is cooperative (all CTAs resident), so the items waited for are always making progress.
__device__ __forceinline__ void chain_wait(const Q8SLaunch &L, int j) {
    if (threadIdx.x == 0) {
        const uint32_t need = (j + 1 < L.njobs ? L.jobs[j + 1].item0 : L.nitems) - L.jobs[j].item0;
        const uint32_t *cnt = &L.jobs[j].pad;
        for (uint32_t it = 0;; it++) {
            uint32_t done;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(done) : "l"(cnt) : "memory");
            if (done >= need) break;
            if (it >= L.spin_limit) {
                atomicOr(L.status, MV_DEV_WAIT_TIMEOUT);
                break;
            }
            __nanosleep(64);
        }
    }
    __syncthreads();
}

__global__ void q8s_chain_reset(Q8Job *jobs, int njobs) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) jobs[j].pad = 0;
}

// Shared-memory layout of q8s_kernel (byte offsets), computed on the host and passed with the launch.
__host__ __device__ inline Q8SLayout q8s_layout(uint32_t lut_bytes, uint32_t extra_bytes, uint32_t tbl_alias, int W,
                                                int DEPTH, int ILP, int buf_words, int red_nv, int red_bufs,
                                                int tbl_stage) {
    Q8SLayout o{};
    uint32_t p = lut_bytes;
    o.extra = p;
    p += extra_bytes;
    o.bufs = p;  // [W][DEPTH][ILP][buf_words] u32 stream slots (128-byte multiples)
    p += (uint32_t)(W * DEPTH * ILP) * (uint32_t)buf_words * 4u;
    o.red = p;  // [red_bufs][W][red_nv][32] int
    p += (uint32_t)(red_bufs * W * red_nv * 32) * 4u;
    o.bars = p;  // [W][DEPTH] mbarriers
    p += (uint32_t)(W * DEPTH) * 8u;
    p = (p + 15u) & ~15u;
    o.ring = p;
    p += (uint32_t)kRing * (uint32_t)sizeof(ItemRec);
    o.curs = p;  // [W] copy cursors (lane 0 of each warp)
    p += (uint32_t)W * (uint32_t)sizeof(StepCursor);
    o.sched = p;  // scheduler state (thread 0)
    p += (uint32_t)sizeof(SchedState);
    p = (p + 15u) & ~15u;
    o.stage_o = p;  // [kStageOffs]
    p += kStageOffs * 4u;
    o.rows = p;  // [W][DEPTH][ILP] word-rows of each slot's blocks
    p += (uint32_t)(W * DEPTH * ILP) * 4u;
    p = (p + 15u) & ~15u;
    // table staging: one area of its own, staged one item ahead asynchronously (the next item's data goes in
    // only after the current item's table build and the barrier behind it, so one area serves both), or,
    // staged synchronously, one inside the consumer's region when that is free at table rebuilds and large
    // enough
    const uint32_t stage_bytes = ((uint32_t)tbl_stage + kStagePad) * 2u;
    o.async_tables = 0;
    if (tbl_alias >= stage_bytes) {
        o.stage_e = o.extra;
    } else {
        o.stage_e = p;
        o.async_tables = 1;
        p += stage_bytes;
    }
    o.total = p;
    return o;
}

// Lane 0: issue copies while the warp has free slots and its cursor is on a visible step.
template <int ILP, int DEPTH>
__device__ __forceinline__ void pump_copies(const Q8SLaunch &L, StepCursor *cp, const ItemRec *ring, int kvis,
                                            int warp, int W, uint32_t &issued, uint32_t consumed, unsigned char *sm,
                                            uint32_t my_slots, uint32_t slot_bytes, uint64_t *my_bars,
                                            uint32_t *my_rows) {
    if (issued - consumed >= (uint32_t)DEPTH) return;
    StepCursor c = *cp;
    while (issued - consumed < (uint32_t)DEPTH && cursor_ready(c, ring, kvis, warp, W, ILP)) {
        const int s = (int)(issued % DEPTH);
        issue_step<ILP>(L, c, warp, W, sm, my_slots + (uint32_t)s * slot_bytes, &my_bars[s], my_rows + s * ILP);
        issued++;
        c.j++;
    }
    *cp = c;
}

// The table data of one item staged by the whole CTA from device memory (the first item, and consumers whose
// staging area lies in their own region): offsets relative to the first entry in so[0..nt], entries from se[0].
__device__ __forceinline__ void stage_table_sync(const Q8SLaunch &L, const mv_q8_view &m, int stripe, uint32_t *so,
                                                 uint16_t *se) {
    const uint32_t r0 = m.local ? (uint32_t)stripe * 32 : 0;
    const uint32_t nt = m.local ? 32 : 1;
    const uint32_t tb = __ldg(m.tbl_off + r0), te = __ldg(m.tbl_off + r0 + nt);
    const bool ok = te >= tb && te <= m.tbl_len && te - tb <= (uint32_t)L.tbl_stage;
    for (uint32_t i = threadIdx.x; i <= nt; i += blockDim.x) {
        const uint32_t o = __ldg(m.tbl_off + r0 + i);
        so[i] = (ok && o >= tb && o <= te) ? o - tb : 0;
    }
    if (threadIdx.x == 0) {
        so[36] = ok;
        so[37] = 0;
        if (!ok) atomicOr(L.status, MV_DEV_BAD_TABLE);
    }
    const uint32_t n = ok ? te - tb : 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) se[i] = __ldg(m.tbl + tb + i);
}

// The last warp of the CTA stages the next item's table data while the current item decodes.  Phase 1: asynchronous copies
// of its nt + 1 table offsets into so[0..nt].  Phase 2 (after the warp's first decode step): they give the
// entry range, which 4-byte asynchronous copies (zero-filled past the readable end) bring in from an even entry
// on; the offsets are rewritten relative to the first entry, so[36] = valid, so[37] = where the first entry
// landed.  The copies complete before the barrier that ends the item (cp_async_wait_all).
__device__ __forceinline__ void stage_offsets_async(const mv_q8_view &mn, int stripe, int lane, uint32_t *so) {
    const uint32_t r0 = mn.local ? (uint32_t)stripe * 32u : 0u;
    const uint32_t nt = mn.local ? 32u : 1u;
    if ((uint32_t)lane <= nt) cp_async_4(so + lane, mn.tbl_off + r0 + lane, 4u);
    if (lane == 0 && nt == 32u) cp_async_4(so + 32, mn.tbl_off + r0 + 32, 4u);
    cp_async_commit();
}
__device__ __forceinline__ void stage_entries_async(const Q8SLaunch &L, const mv_q8_view &mn, int lane, uint32_t *so,
                                                    uint16_t *se) {
    cp_async_wait_all();
    __syncwarp();
    const uint32_t nt = mn.local ? 32u : 1u;
    const uint32_t o = (uint32_t)lane <= nt ? so[lane] : 0u;
    const uint32_t o32 = nt == 32u ? so[32] : 0u;
    const uint32_t tb = so[0], te = so[nt];
    __syncwarp();
    const bool ok = te >= tb && te <= mn.tbl_len && te - tb <= (uint32_t)L.tbl_stage;
    if ((uint32_t)lane <= nt) so[lane] = (ok && o >= tb && o <= te) ? o - tb : 0u;
    if (lane == 0) {
        if (nt == 32u) so[32] = (ok && o32 >= tb && o32 <= te) ? o32 - tb : 0u;
        so[36] = ok;
        so[37] = tb & 1u;
    }
    if (!ok) return;
    const uint32_t a = tb & ~1u;
    const uint32_t nch = (te - a + 1) >> 1;  // 4-byte pieces covering entries [a, te)
    if (((uintptr_t)mn.tbl & 3) == 0) {
        for (uint32_t c = lane; c < nch; c += 32) {
            const uint32_t e = a + 2 * c;
            const uint32_t avail = e < mn.tbl_len ? min(2u, mn.tbl_len - e) : 0u;
            cp_async_4(se + 2 * c, mn.tbl + e, avail * 2u);
        }
        cp_async_commit();
    } else {  // a table array that is not 4-byte aligned: plain loads
        for (uint32_t c = lane; c < nch; c += 32) {
            const uint32_t e = a + 2 * c;
            se[2 * c] = e < mn.tbl_len ? __ldg(mn.tbl + e) : (uint16_t)0;
            se[2 * c + 1] = e + 1 < mn.tbl_len ? __ldg(mn.tbl + e + 1) : (uint16_t)0;
        }
    }
}

// Decode table of one item from its staged data (so: relative offsets of the nt + 1 table bounds, tsm: the
// entries u16 symbol | freq << 8).  Warp w fills quantiles [256 w / W, 256 (w + 1) / W) of every lane column.
// Narrow entries sit at word q*kPitch + lane: kPitch 32 (128-byte rows) or 64 (256-byte rows, see MmaCons).
template <bool kWide, int kPitch = 32>
__device__ __forceinline__ void build_table(const Q8SLaunch &L, const mv_q8_view &m, uint32_t *lut,
                                            const uint32_t *so, const uint16_t *tsm, int warp, int lane, int W) {
    const int t = m.local ? lane : 0;
    const uint32_t o0 = so[t], o1 = max(so[t + 1], o0);
    const int qlo = (256 * warp) / W, qhi = (256 * (warp + 1)) / W;
    uint32_t cum = 0;
    if (kWide && !m.local) {
        // one table for every row: lane j finds the entry of quantile qlo + j (the lanes walk the symbols
        // together, without divergence) and writes it to all 32 lane columns, rotating the column so that a
        // half-warp's stores hit distinct banks
        uint2 *lut2 = reinterpret_cast<uint2 *>(lut);
        bool bad = false;
        for (uint32_t q0 = (uint32_t)qlo; q0 < (uint32_t)qhi; q0 += 32) {
            const uint32_t q = q0 + lane, qend = min(q0 + 32, (uint32_t)qhi);
            uint32_t c = 0, ent_q = 0, cum_q = 0;
            bool found = false;
            for (uint32_t k = o0; k < o1 && c < qend; k++) {
                const uint32_t ent = tsm[k], f = ent >> 8;
                if (!found && q < c + f) {  // q >= c: no earlier symbol contains q
                    ent_q = ent;
                    cum_q = c;
                    found = true;
                }
                c += f;
            }
            if (q < qend) {
                bad |= !found;
                const uint2 v = found ? make_uint2((ent_q >> 8) | ((ent_q & 0xFFu) << 16), q - cum_q)
                                      : make_uint2(1u, 0u);
#pragma unroll 8
                for (uint32_t i = 0; i < 32; i++) lut2[q * 32 + ((lane + i) & 31)] = v;
            }
        }
        if (bad) atomicOr(L.status, MV_DEV_BAD_TABLE);
        return;
    }
    uint32_t k = o0;
    if constexpr (kWide) {
        if (cum < (uint32_t)qlo) {
            // symbols that end at or before qlo: one load, shift and add each (measured: 0.8 % faster than
            // the plain loop below; the four-at-a-time walk of the narrow layouts measured 1.5 % slower here)
            uint32_t f = k < o1 ? (uint32_t)tsm[k] >> 8 : 0u;
            while (k < o1 && cum + f <= (uint32_t)qlo) {
                cum += f;
                k++;
                f = k < o1 ? (uint32_t)tsm[k] >> 8 : 0u;
            }
        }
        for (; k < o1 && cum < (uint32_t)qhi; k++) {
            const uint32_t ent = tsm[k];
            const uint32_t f = ent >> 8, sym = ent & 0xFF;
            const uint32_t a = max(cum, (uint32_t)qlo), e = min(cum + f, (uint32_t)qhi);
            for (uint32_t q = a; q < e; q++)
                reinterpret_cast<uint2 *>(lut)[q * 32 + lane] = make_uint2(f | (sym << 16), q - cum);
            cum += f;
        }
    } else {
        if (cum < (uint32_t)qlo) {
            // symbols that end at or before qlo, four at a time: the four loads are independent, so the walk
            // waits for shared memory once per four symbols instead of once per symbol (the later warps of a
            // CTA skip most of a row's list, and the CTA barrier after the build waits for them)
            while (k + 4 <= o1) {
                const uint32_t c4 = cum + ((uint32_t)tsm[k] >> 8) + ((uint32_t)tsm[k + 1] >> 8) +
                                    ((uint32_t)tsm[k + 2] >> 8) + ((uint32_t)tsm[k + 3] >> 8);
                if (c4 > (uint32_t)qlo) break;
                cum = c4;
                k += 4;
            }
            uint32_t f = k < o1 ? (uint32_t)tsm[k] >> 8 : 0u;
            while (k < o1 && cum + f <= (uint32_t)qlo) {
                cum += f;
                k++;
                f = k < o1 ? (uint32_t)tsm[k] >> 8 : 0u;
            }
        }
        // the next symbol's entry is loaded before this one's stores, off the walk's dependency chain
        uint32_t ent = k < o1 ? (uint32_t)tsm[k] : 0u;
        for (; k < o1 && cum < (uint32_t)qhi; k++) {
            const uint32_t cur = ent;
            ent = k + 1 < o1 ? (uint32_t)tsm[k + 1] : 0u;
            const uint32_t f = cur >> 8, sym = cur & 0xFF;
            const uint32_t a = max(cum, (uint32_t)qlo), e = min(cum + f, (uint32_t)qhi);
            // unrolled: measured 1 % faster for the tensor-core consumer (0.4 % slower for the wide table)
#pragma unroll 4
            for (uint32_t q = a; q < e; q++) lut[q * kPitch + lane] = f | (sym << 16) | ((q - cum) << 24);
            cum += f;
        }
    }
    if (cum < (uint32_t)qhi) {
        for (uint32_t q = max(cum, (uint32_t)qlo); q < (uint32_t)qhi; q++) {
            if constexpr (kWide)
                reinterpret_cast<uint2 *>(lut)[q * 32 + lane] = make_uint2(1u, 0u);
            else
                lut[q * kPitch + lane] = 1u;
        }
        atomicOr(L.status, MV_DEV_BAD_TABLE);
    }
}

template <class Cons, int ILP, int DEPTH>
__global__ void __launch_bounds__(Cons::kMaxThreads, Cons::kMinCtas) q8s_kernel(const Q8SLaunch L) {
    constexpr int NV = Cons::kRedNV;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = blockDim.x >> 5;

    // decode table at the start of shared memory: 256 quantiles x 32 lanes of 4 B (narrow) or 8 B (wide); the
    // rest of the layout comes with the launch (L.lay), so its offsets are constant-bank operands.
    // Asynchronous table staging: the next item's table data is staged (into the one staging area, after this
    // item's table build and its barrier) while the current item decodes.
    const bool async_tbl = L.lay.async_tables != 0;
    uint32_t *lut = reinterpret_cast<uint32_t *>(smem);
    unsigned char *extra = smem + L.lay.extra;
    ItemRec *ring = reinterpret_cast<ItemRec *>(smem + L.lay.ring);
    StepCursor *my_cur = reinterpret_cast<StepCursor *>(smem + L.lay.curs) + warp;
    SchedState *sch = reinterpret_cast<SchedState *>(smem + L.lay.sched);
    const uint32_t my_slots = L.lay.bufs + (uint32_t)(warp * DEPTH) * L.slot_bytes;  // byte offset of slot 0
    uint32_t *my_rows = reinterpret_cast<uint32_t *>(smem + L.lay.rows) + warp * DEPTH * ILP;
    uint64_t *my_bars = reinterpret_cast<uint64_t *>(smem + L.lay.bars) + warp * DEPTH;

    // tensor-memory accumulators (MMA consumers): one warp allocates, all use, it frees at the end
    uint32_t tmem_base = 0;
    if (Cons::kTmemCols) {
        uint32_t *slot = reinterpret_cast<uint32_t *>(extra + Cons::extra_bytes(W) - 128);
        if (warp == 0) tmem_alloc(slot, MmaCons::tmem_cols(W));
        tcgen05_fence_before();
        __syncthreads();
        tcgen05_fence_after();
        tmem_base = *slot;
    }
    Cons cons;
    cons.init(L, extra, tmem_base, warp, lane, W);
    if (lane == 0)
        for (int d = 0; d < DEPTH; d++) mbar_init(&my_bars[d], 1);
    fence_mbar_init();

    // scheduler (thread 0): the CTA's first two items
    if (threadIdx.x == 0) {
        SchedState st{};
        for (int k = 0; k < 2; k++) {
            ItemRec r{};
            r.it = -1;
            if (!st.grab_done) {
                const uint32_t v = sched_grab(L, st.ngrab++);
                sched_after_grab(L, v);
                r = make_item(L, v, st.jhint);
                st.grab_done = r.it < 0;
            }
            ring[k] = r;
        }
        *sch = st;
    }
    // this warp's copies run DEPTH steps ahead of its decode
    if (lane == 0) {
        StepCursor c{};
        c.k = -1;
        *my_cur = c;
    }
    __syncthreads();  // the first two ring entries, cursors and mbarrier inits are visible

    uint32_t issued = 0, consumed = 0;
    bool failed = false;  // a bounded wait ran out: no more copies or decodes (the status word has the flag)
    if (lane == 0)
        pump_copies<ILP, DEPTH>(L, my_cur, ring, 1, warp, W, issued, consumed, smem, my_slots, L.slot_bytes, my_bars,
                                my_rows);
    issued = __shfl_sync(0xffffffffu, issued, 0);  // lane 0 counts the copies; every lane tests them

    int lut_job = -1, lut_stripe = -1;
    int pf_state = 0;  // staging warp: 0 nothing to stage, 1 offsets in flight, 2 entries in flight
    const uint32_t *lut_l = Cons::kWideLut ? lut : lut + lane;  // wide steps add the lane themselves
    for (int k = 0;; k++) {
        const ItemRec I = ring[k % kRing];
        if (I.it < 0) break;
        const Q8Job &J = job_at(L, I.job);
        const mv_q8_view &m = J.m;

        // decode table, rebuilt only when it changes (uniform across the CTA).  Every warp finished the
        // previous item's decode before the CTA barrier that ended it.
        if (I.job != lut_job || (m.local && I.stripe != lut_stripe)) {
            uint32_t *so = reinterpret_cast<uint32_t *>(smem + L.lay.stage_o);
            uint16_t *se = reinterpret_cast<uint16_t *>(smem + L.lay.stage_e);
            if (!async_tbl || k == 0) {
                __syncthreads();  // the staging area may be the consumer's region
                stage_table_sync(L, m, I.stripe, so, se);
                __syncthreads();
            } else if (threadIdx.x == 0 && so[36] == 0) {
                atomicOr(L.status, MV_DEV_BAD_TABLE);
            }
            build_table<Cons::kWideLut, Cons::kLut256 ? 64 : 32>(L, m, lut, so, se + so[37], warp, lane, W);
            fence_proxy_async_smem();  // the table staging may share memory with later bulk copies
            __syncthreads();
            lut_job = I.job;
            lut_stripe = I.stripe;
        }

        // thread 0: take the CTA's item k + 2 now and record it at the end of this item (the atomic's
        // latency overlaps the decode)
        if (threadIdx.x == 0) {
            sch->grab_now = 0;
            if (!sch->grab_done) {
                sch->pending = sched_grab(L, sch->ngrab++);
                sch->grab_now = 1;
            }
        }
        // the last warp (warp 0 holds the scheduler and sums the item's rows), first phase of staging the next
        // item's table data: its offsets
        pf_state = 0;
        if (async_tbl && warp == W - 1) {
            const ItemRec &N = ring[(k + 1) % kRing];
            if (N.it >= 0) {
                const mv_q8_view &mn = job_at(L, N.job).m;
                if (N.job != I.job || (mn.local && N.stripe != I.stripe)) {
                    stage_offsets_async(mn, N.stripe, lane, reinterpret_cast<uint32_t *>(smem + L.lay.stage_o));
                    pf_state = 1;
                }
            }
        }

        if (L.chain_scales && I.job > 0) chain_wait(L, I.job - 1);
        cons.begin_item(L, J, I.stripe, lane, I.job);
        // ring[k + 1] was recorded during item k - 1 (or before the first item) and is visible now
        const int kvis = k + 1;
        if (lane == 0 && !failed)
            pump_copies<ILP, DEPTH>(L, my_cur, ring, kvis, warp, W, issued, consumed, smem, my_slots, L.slot_bytes,
                                    my_bars, my_rows);
        issued = __shfl_sync(0xffffffffu, issued, 0);
        const int steps = warp_steps(I.se - I.sb, warp, W, ILP);
        for (int j = 0; j < steps; j++) {
            const int slot = consumed % DEPTH;
            const uint32_t parity = (consumed / DEPTH) & 1;
            const bool was_issued = consumed < issued;
            uint32_t rows_now[ILP];
            bool any = false;
#pragma unroll
            for (int kk = 0; kk < ILP; kk++) {
                rows_now[kk] = my_rows[slot * ILP + kk];
                any |= rows_now[kk] != 0;
            }
            if (was_issued && any) {
                if (!failed) {
                    const bool ok =
                        __all_sync(0xffffffffu, mbar_wait_bounded(&my_bars[slot], parity, L.status, L.spin_limit));
                    if (ok) {
                        cons.template run_step<ILP>(L, m, I.sb + warp + j * W * ILP, W, rows_now, smem,
                                                    my_slots + (uint32_t)slot * L.slot_bytes, lut_l, lane);
                    } else {
                        failed = true;  // wait once more (bounded) so that no copy is left writing the slot
                        mbar_wait_bounded(&my_bars[slot], parity, nullptr, L.spin_limit);
                    }
                } else {
                    mbar_wait_bounded(&my_bars[slot], parity, nullptr, L.spin_limit);  // drain, no decode
                }
            }
            __syncwarp();
            consumed++;
            // the slot is free: refill it with the step DEPTH ahead in this warp's stream
            if (lane == 0 && !failed)
                pump_copies<ILP, DEPTH>(L, my_cur, ring, kvis, warp, W, issued, consumed, smem, my_slots,
                                        L.slot_bytes, my_bars, my_rows);
            issued = __shfl_sync(0xffffffffu, issued, 0);
            if (pf_state == 1) {  // staging warp, second phase (after its first step): the entries
                stage_entries_async(L, job_at(L, ring[(k + 1) % kRing].job).m, lane,
                                    reinterpret_cast<uint32_t *>(smem + L.lay.stage_o),
                                    reinterpret_cast<uint16_t *>(smem + L.lay.stage_e));
                pf_state = 2;
            }
        }
        if (pf_state == 1)
            stage_entries_async(L, job_at(L, ring[(k + 1) % kRing].job).m, lane,
                                reinterpret_cast<uint32_t *>(smem + L.lay.stage_o),
                                reinterpret_cast<uint16_t *>(smem + L.lay.stage_e));
        if (pf_state) cp_async_wait_all();  // visible to the CTA after the barrier that ends the item
        if (threadIdx.x == 0 && sch->grab_now) {  // record item k + 2
            SchedState st = *sch;
            sched_after_grab(L, st.pending);
            const ItemRec r = make_item(L, st.pending, st.jhint);
            st.grab_done = r.it < 0;
            *sch = st;
            ring[(k + 2) % kRing] = r;
        }

        cons.finish_item(L, J, I.stripe, warp, lane, W,
                         reinterpret_cast<int *>(smem + L.lay.red) + (Cons::kRedBufs == 2 ? (k & 1) : 0) * W * NV * 32);
        if (!Cons::kFinishSyncs) __syncthreads();
        if (L.chain_scales && threadIdx.x == 0) {
            __threadfence();  // this item's outputs are visible before it is counted
            atomicAdd(const_cast<uint32_t *>(&L.jobs[I.job].pad), 1u);
        }
    }
    // copies still in flight (only after a failed wait) land before the CTA exits
    for (; consumed < issued; consumed++)
        mbar_wait_bounded(&my_bars[consumed % DEPTH], (consumed / DEPTH) & 1, nullptr, L.spin_limit);
    if (Cons::kTmemCols) {
        cons.drain(L);
        tcgen05_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(tmem_base, MmaCons::tmem_cols(W));
    }
}

}  // namespace mv

namespace mv {

// x of every job with x_tiles, laid out per (segment, 32-quad window) in the tensor-core consumer's x tile
// layout: 2 KB per tile = 4 pieces of 32 columns; piece = 2 groups of 8 vectors (256 B); group = 2 column
// halves (128 B); half = 8 vectors x 16 bytes.  Vectors past the batch and columns past the row are zero.
__global__ void q8s_build_x_tiles(const Q8Job *jobs, int njobs, int batch) {
    for (int j = blockIdx.y; j < njobs; j += gridDim.y) {
        const Q8Job &J = jobs[j];
        if (!J.x_tiles) continue;
        const mv_q8_view &m = J.m;
        const int nwin = (m.seg_quads + 31) / 32;
        const size_t units = (size_t)m.nseg * nwin * 128;  // 16-byte units
        for (size_t u = blockIdx.x * (size_t)blockDim.x + threadIdx.x; u < units; u += (size_t)gridDim.x * blockDim.x) {
            const size_t tile = u >> 7;
            const int o = (int)(u & 127);
            const int sg = (int)(tile / nwin), w = (int)(tile % nwin);
            const int i = o >> 5, g = (o >> 4) & 1, h = (o >> 3) & 1, r = o & 7;
            const int v = 8 * g + r;
            const int col = 4 * sg * m.seg_quads + 128 * w + 32 * i + 16 * h;  // a multiple of 16
            uint4 val = make_uint4(0, 0, 0, 0);
            if (v < batch && col < m.cols) val = *reinterpret_cast<const uint4 *>(J.x + (size_t)v * m.cols + col);
            *reinterpret_cast<uint4 *>(J.x_tiles + tile * 2048 + (size_t)o * 16) = val;
        }
    }
}

__global__ void q8s_zero_atomic_y(const Q8Job *jobs, int njobs, int batch) {
    for (int j = blockIdx.y; j < njobs; j += gridDim.y) {
        const Q8Job &J = jobs[j];
        if (!J.atomic) continue;
        const size_t n = (size_t)batch * J.m.rows;
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
            J.y[i] = 0;
    }
}

__global__ void q8s_scale_atomic_y(const Q8Job *jobs, int njobs, int batch) {
    for (int j = blockIdx.y; j < njobs; j += gridDim.y) {
        const Q8Job &J = jobs[j];
        if (!J.atomic || !J.ys) continue;
        const size_t n = (size_t)batch * J.m.rows;
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
            J.ys[i] = (float)J.y[i] * J.scales[i % J.m.rows];
    }
}

namespace {

mv_status resident_ctas(const void *kern, size_t smem, int threads, int *out) {
    int d = 0, smem_sm = 0, reserved = 0;
    MV_CUDA_TRY(cudaGetDevice(&d), "cudaGetDevice");
    MV_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, d), "attribute");
    MV_CUDA_TRY(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, d), "attribute");
    cudaFuncAttributes fa{};
    MV_CUDA_TRY(cudaFuncGetAttributes(&fa, kern), "cudaFuncGetAttributes");
    const int warps = (threads + 31) / 32;
    const int regs_warp = ((std::max(1, fa.numRegs) * 32 + 255) / 256) * 256;  // allocation unit: 256 per warp
    int n = std::min(smem_sm / (int)(smem + reserved), (65536 / regs_warp) / warps);
    n = std::min(n, 64 / warps);
    *out = std::max(1, n);
    return MV_OK;
}

template <class Cons, int ILP, int DEPTH>
mv_status launch_q8s_t(const Q8SLaunch &L0, int W, int ctas_per_sm, cudaStream_t st) {
    if (32 * W > Cons::kMaxThreads)
        return fail(MV_ERR_ARG, "Q8 launch: %d warps per CTA; this engine takes at most %d", W,
                    Cons::kMaxThreads / 32);
    if (Cons::extra_bytes(W) % 16)  // the stream buffers behind the consumer region take bulk copies
        return fail(MV_ERR_UNSUPPORTED, "Q8 stack launch: consumer region of %zu B breaks 16-byte alignment",
                    Cons::extra_bytes(W));
    Q8SLaunch L = L0;
    L.lay = q8s_layout(Cons::kWideLut || Cons::kLut256 ? 256 * 256 : 256 * 32 * 4, (uint32_t)Cons::extra_bytes(W),
                       (uint32_t)Cons::tbl_alias_bytes(W), W, DEPTH, ILP, L.buf_words, Cons::kRedNV, Cons::kRedBufs,
                       L.tbl_stage);
    L.slot_bytes = (uint32_t)ILP * (uint32_t)L.buf_words * 4u;
    L.stage_len = (uint32_t)L.tbl_stage + kStagePad;
    const size_t smem = L.lay.total;
    if (smem > (size_t)max_smem_optin())
        return fail(MV_ERR_UNSUPPORTED, "Q8 stack launch needs %zu B of shared memory (max %d)", smem,
                    max_smem_optin());
    auto kern = q8s_kernel<Cons, ILP, DEPTH>;
    int bps = 0;
    mv_status rc = prepare_kernel((const void *)kern, smem, 32 * W, &bps);
    if (rc) return rc;
    if (ctas_per_sm > 0) bps = std::min(bps, ctas_per_sm);
    if (Cons::kTmemCols) {
        // resident CTAs of a tensor-memory kernel, from its resources directly: shared memory, registers,
        // threads and TMEM columns (512 per SM)
        rc = resident_ctas((const void *)kern, smem, 32 * W, &bps);
        if (rc) return rc;
        if (ctas_per_sm > 0) bps = std::min(bps, ctas_per_sm);
        bps = std::max(1, std::min<int>(bps, 512 / MmaCons::tmem_cols(W)));
    }
    if (L.chain_scales) {
        // the chained pipeline waits across CTAs: a cooperative launch guarantees that they are all resident.
        // The runtime checks the grid against its own occupancy figure (for tensor-memory kernels one CTA
        // per SM, fewer than the SM holds), and a rejected launch would also end a stream capture, so the
        // grid is taken from that figure.
        int coop = 0;
        MV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&coop, kern, 32 * W, smem), "occupancy");
        coop = std::max(1, std::min(coop, bps));
        const long long grid = std::max(1LL, std::min<long long>(L.nitems, (long long)coop * sm_count()));
        Q8SLaunch Lc = L;
        void *args[] = {&Lc};
        MV_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)grid), dim3(32 * W), args, smem, st),
                    "q8 chain cooperative launch");
        return MV_OK;
    }
    const long long grid = std::max(1LL, std::min<long long>(L.nitems, (long long)bps * sm_count()));
    kern<<<(unsigned)grid, 32 * W, smem, st>>>(L);
    MV_CUDA_TRY(cudaGetLastError(), "q8 stack kernel launch");
    return MV_OK;
}

template <class Cons>
mv_status launch_q8s_c(const Q8SLaunch &L, const mv_q8_tuning &t, cudaStream_t st) {
    if constexpr (Cons::kTmemCols != 0) {  // the MMA consumer decodes one segment per warp step
        if (t.depth == 2) return launch_q8s_t<Cons, 1, 2>(L, t.warps, t.ctas_per_sm, st);
        return launch_q8s_t<Cons, 1, 1>(L, t.warps, t.ctas_per_sm, st);
    } else {
        if (t.ilp == 2) {
            if (t.depth == 2) return launch_q8s_t<Cons, 2, 2>(L, t.warps, t.ctas_per_sm, st);
            return launch_q8s_t<Cons, 2, 1>(L, t.warps, t.ctas_per_sm, st);
        }
        if (t.depth == 2) return launch_q8s_t<Cons, 1, 2>(L, t.warps, t.ctas_per_sm, st);
        return launch_q8s_t<Cons, 1, 1>(L, t.warps, t.ctas_per_sm, st);
    }
}

// Integer batches of at least this many vectors (rounded up to 4, 8 or 16) go to the tensor-core consumer
// (engine 0), which always multiplies 16 vectors, the missing ones zero: its cost hardly depends on the batch
// (the 224-matrix stack: 3.86 ms at 8 vectors, 3.88 ms at 16), while the dp4a consumer's grows with it (4.25
// ms at 4 vectors, 2.91 ms at 1).
constexpr int kMmaMinVectors = MV_MMA_MIN_VECTORS;

mv_status launch_q8s(const Q8SLaunch &L, int nv, const mv_q8_tuning &t, cudaStream_t st) {
    if (nv >= kMmaMinVectors && t.engine == MV_ENGINE_AUTO) return launch_q8s_c<MmaCons>(L, t, st);
    switch (nv) {
        case 1: return launch_q8s_c<IntCons<1>>(L, t, st);
        case 2: return launch_q8s_c<IntCons<2>>(L, t, st);
        case 4: return launch_q8s_c<IntCons<4>>(L, t, st);
        case 8: return launch_q8s_c<IntCons<8>>(L, t, st);
        default: return launch_q8s_c<IntCons<16>>(L, t, st);
    }
}

// mode 1: float forward, mode 2: float backward (transposed); nv in {1,2,4,8}
// float form: batches of at least this many vectors go to the tensor-core consumers (engine 0)
constexpr int kFloatMmaMinBatch = 2;

// vectors per pass of the float form: the tensor-core consumers take 16 (forward) / 32 (backward)
int q8f_pass(int mode, int batch, const mv_q8_tuning &t) {
    if (t.engine == MV_ENGINE_AUTO && batch >= kFloatMmaMinBatch) return mode == 1 ? FwdMma::kNV : BwdMma::kNV;
    return 8;
}

mv_status launch_q8f(const Q8SLaunch &L, int mode, int nv, const mv_q8_tuning &t, bool mma, cudaStream_t st) {
    if (mma) return mode == 1 ? launch_q8s_c<FwdMma>(L, t, st) : launch_q8s_c<BwdMma>(L, t, st);
    if (mode == 1) {
        switch (nv) {
            case 1: return launch_q8s_c<FwdCons<1>>(L, t, st);
            case 2: return launch_q8s_c<FwdCons<2>>(L, t, st);
            case 4: return launch_q8s_c<FwdCons<4>>(L, t, st);
            default: return launch_q8s_c<FwdCons<8>>(L, t, st);
        }
    }
    switch (nv) {
        case 1: return launch_q8s_c<BwdCons<1>>(L, t, st);
        case 2: return launch_q8s_c<BwdCons<2>>(L, t, st);
        case 4: return launch_q8s_c<BwdCons<4>>(L, t, st);
        default: return launch_q8s_c<BwdCons<8>>(L, t, st);
    }
}

int nv_round(int nb) { return nb <= 2 ? nb : nb <= 4 ? 4 : nb <= 8 ? 8 : 16; }

}  // namespace

mv_status stack_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning, mv_q8_stack_info *info);

namespace {

mv_q8_tuning resolve(const mv_q8_tuning *t) {
    mv_q8_tuning r{8, 2, 1, 0, 0, MV_ENGINE_AUTO};
    if (t) {
        if (t->engine == MV_ENGINE_DP4A) r.engine = MV_ENGINE_DP4A;
        if (t->parts > 0) r.parts = t->parts;
        if (t->warps > 0) r.warps = std::min(16, t->warps);  // more than 8: the integer CUDA-core consumer only
        if (t->ilp == 1 || t->ilp == 2) r.ilp = t->ilp;
        if (t->depth == 1 || t->depth == 2) r.depth = t->depth;
        if (t->ctas_per_sm > 0) r.ctas_per_sm = t->ctas_per_sm;
    }
    return r;
}

// parts = 0: whole stripes (stacks); otherwise split each stripe's segments into `parts`
void plan_job(Q8Job &J, const mv_q8_tuning &t, uint32_t &item, int parts) {
    J.ngroups = std::max(1, std::min(parts > 0 ? parts : 1, J.m.nseg));
    J.atomic = J.ngroups > 1;
    J.item0 = item;
    J.pad = 0;  // work-queue counter (job 0 of a stack) or item counter (chains)
    item += (uint32_t)((J.m.rows + 31) / 32) * (uint32_t)J.ngroups;
}

}  // namespace

// Work items per stripe for a single matrix: enough items for ~4 per SM, but no more than it takes
// to give each of the CTA's sg = warps x ilp segment slots one segment per item (ceil, so that the
// items of a stripe are as even as its segment count allows)
int default_parts(int nseg, int sg, int stripes) {
    const int fill = (4 * sm_count() + stripes - 1) / stripes;
    const int even = (nseg + sg - 1) / sg;
    return std::max(1, std::min(fill, even));
}

// Parts per stripe for the float backward: the fewest that minimise waves of items (two CTAs per SM) times
// rounds of segments per warp within an item.  At one vector this picks 2 for 4096x11008 (49.6 us; 1, 3
// and 5 parts: 63.7, 59.6 and ~72 us) and 2 for 11008x4096 (57.5 us; 1 and 3 parts: 59.6 and 74.6 us).
int bwd_parts(int nseg, int sg, int stripes) {
    const long long slots = 2LL * sm_count();
    int best = 1;
    long long best_cost = -1;
    for (int p = 1; p <= 8 && p <= nseg; p++) {
        const long long waves = ((long long)stripes * p + slots - 1) / slots;
        const long long rounds = ((nseg + p - 1) / p + sg - 1) / sg;
        const long long cost = waves * rounds;
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = p;
        }
    }
    return best;
}

bool q8s_supports(const mv_q8_view *m, const int8_t *x) {
    return (m->cols & 15) == 0 && ((uintptr_t)x & 15) == 0 && (m->seg_quads & 3) == 0;
}

// Single matrix through the persistent kernel (one inline job).
mv_status q8s_matvec(const mv_q8_view *m, const int8_t *x, int batch, int32_t *y, const float *scales, float *ys,
                     const mv_q8_tuning *tuning, cudaStream_t st) {
    mv_status rc;
    uint32_t *status = device_status_word(&rc);
    if (rc) return rc;
    const mv_q8_tuning t = resolve(tuning);
    for (int v0 = 0; v0 < batch; v0 += 16) {
        const int nb = std::min(16, batch - v0);
        Q8SLaunch L{};
        L.job0.m = *m;
        L.job0.x = x + (size_t)v0 * m->cols;
        L.job0.y = y + (size_t)v0 * m->rows;
        L.job0.scales = scales;
        L.job0.ys = ys ? ys + (size_t)v0 * m->rows : nullptr;
        uint32_t items = 0;
        // a single matrix: split stripes so that every warp slot of the GPU gets work
        const int stripes = (m->rows + 31) / 32;
        const int sg = t.warps * t.ilp;
        int parts = t.parts > 0 ? t.parts : default_parts(m->nseg, sg, stripes);
        plan_job(L.job0, t, items, parts);
        if (L.job0.atomic) L.job0.ys = nullptr;
        L.jobs = nullptr;
        L.njobs = 1;
        L.nitems = items;
        L.batch = nb;
        L.status = status;
        L.spin_limit = wait_spin_limit();
        L.drop_copy = inject_drop_copy();
        L.buf_words = (m->max_blk_rows + 1) * 32;
        L.tbl_stage = (int)((m->tbl_stripe_max + 7) & ~7u);
        L.lut_stride = 32;
        if (L.job0.atomic)
            MV_CUDA_TRY(cudaMemsetAsync(L.job0.y, 0, sizeof(int32_t) * (size_t)nb * m->rows, st), "cudaMemsetAsync(y)");
        rc = launch_q8s(L, nv_round(nb), t, st);
        if (rc) return rc;
        if (ys && L.job0.atomic) {
            const int n = nb * m->rows;
            scale_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(L.job0.y, scales, ys + (size_t)v0 * m->rows, m->rows,
                                                               nb, m->rows);
            MV_CUDA_TRY(cudaGetLastError(), "scale_rows_kernel launch");
        }
    }
    return MV_OK;
}

// Float forward / transposed product through the persistent kernel.
mv_status q8f_run(const mv_q8_view *m, int mode, const uint16_t *in, int batch, const float *scales, float *out,
                  const mv_q8_tuning *tuning, cudaStream_t st) {
    mv_status rc;
    uint32_t *status = device_status_word(&rc);
    if (rc) return rc;
    mv_q8_tuning t = resolve(tuning);
    if (!tuning || (tuning->ilp != 1 && tuning->ilp != 2)) t.ilp = 1;  // the float form's default
    const int in_len = mode == 1 ? m->cols : m->rows;   // elements per vector in
    const int out_len = mode == 1 ? m->rows : m->cols;  // elements per vector out
    if (mode == 2) MV_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)batch * out_len, st), "memset(dx)");
    const int pass = q8f_pass(mode, batch, t);
    const bool mma = pass > 8;
    for (int v0 = 0; v0 < batch; v0 += pass) {
        const int nb = std::min(pass, batch - v0);
        Q8SLaunch L{};
        L.job0.m = *m;
        L.job0.x = reinterpret_cast<const int8_t *>(in + (size_t)v0 * in_len);
        L.job0.y = nullptr;
        L.job0.scales = scales;
        L.job0.ys = out + (size_t)v0 * out_len;
        uint32_t items = 0;
        // forward: whole stripes (deterministic sums); backward: atomics anyway, so split for parallelism
        int parts = 1;
        if (mode == 2) {
            const int stripes = (m->rows + 31) / 32, sg = t.warps * t.ilp;
            parts = t.parts > 0 ? t.parts : mma ? default_parts(m->nseg, sg, stripes) : bwd_parts(m->nseg, sg, stripes);
        }
        plan_job(L.job0, t, items, parts);
        if (mode == 1 && L.job0.atomic) return fail(MV_ERR_ARG, "float forward needs whole stripes (parts = 1)");
        L.jobs = nullptr;
        L.njobs = 1;
        L.nitems = items;
        L.batch = nb;
        L.status = status;
        L.spin_limit = wait_spin_limit();
        L.drop_copy = inject_drop_copy();
        L.buf_words = (m->max_blk_rows + 1) * 32;
        L.tbl_stage = (int)((m->tbl_stripe_max + 7) & ~7u);
        L.lut_stride = 32;
        rc = launch_q8f(L, mode, nv_round(nb), t, mma, st);
        if (rc) return rc;
    }
    return MV_OK;
}

}  // namespace mv

extern "C" {

mv_status mv_q8_matvec_bf16(const mv_q8_view *m, const uint16_t *x_dev, int batch, const float *row_scales_dev,
                            float *y_dev, const mv_q8_tuning *tuning, void *stream) {
    if (!m || !x_dev || !row_scales_dev || !y_dev || batch <= 0)
        return mv::fail(MV_ERR_ARG, "mv_q8_matvec_bf16: bad arguments");
    if ((m->cols & 15) || ((uintptr_t)x_dev & 15) || (m->seg_quads & 3))
        return mv::fail(MV_ERR_ARG, "mv_q8_matvec_bf16: needs cols %% 16 == 0, seg_quads %% 4 == 0, 16-byte aligned x");
    mv_q8_tuning t = mv::resolve(tuning);
    t.parts = 1;
    if (!tuning || (tuning->ilp != 1 && tuning->ilp != 2)) t.ilp = 1;  // the float form's default
    // the forward keeps whole stripes per item (a fixed-order reduction): with fewer stripes than SMs, the
    // CUDA-core consumer takes 16-warp CTAs so that each stripe's segments spread over more warps
    // (4096x11008, one vector: 35.0 against 43.2 us; with 344 stripes 8 warps stay faster, 43.2 against 47.3)
    if ((!tuning || tuning->warps <= 0) && mv::q8f_pass(1, batch, t) <= 8 && (m->rows + 31) / 32 < mv::sm_count())
        t.warps = 16;
    return mv::q8f_run(m, 1, x_dev, batch, row_scales_dev, y_dev, &t, (cudaStream_t)stream);
}

mv_status mv_q8_matvec_t_bf16(const mv_q8_view *m, const uint16_t *dy_dev, int batch, const float *row_scales_dev,
                              float *dx_dev, const mv_q8_tuning *tuning, void *stream) {
    if (!m || !dy_dev || !row_scales_dev || !dx_dev || batch <= 0)
        return mv::fail(MV_ERR_ARG, "mv_q8_matvec_t_bf16: bad arguments");
    if ((m->cols & 15) || (m->seg_quads & 3))
        return mv::fail(MV_ERR_ARG, "mv_q8_matvec_t_bf16: needs cols %% 16 == 0 and seg_quads %% 4 == 0");
    return mv::q8f_run(m, 2, dy_dev, batch, row_scales_dev, dx_dev, tuning, (cudaStream_t)stream);
}

mv_status mv_q8_stack_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning, mv_q8_stack_info *info) {
    if (!jobs || njobs <= 0 || !info) return mv::fail(MV_ERR_ARG, "mv_q8_stack_plan: bad arguments");
    // The work queue hands out items in job order: jobs with the most work per item (decode steps of a
    // stripe's segment group) go first, so that the last items taken, which set the end of the launch, are
    // the shortest (stable: equal jobs keep their order).  Each job carries its own x and y, so the outputs
    // do not depend on the order.
    std::stable_sort(jobs, jobs + njobs, [&](const mv_q8_job &a, const mv_q8_job &b) {
        auto work = [&](const mv_q8_job &j) {
            const int parts = std::max(1, std::min(tuning && tuning->parts > 0 ? tuning->parts : 1, std::max(1, j.m.nseg)));
            return (long long)((std::max(1, j.m.nseg) + parts - 1) / parts) * std::max(1, j.m.seg_quads);
        };
        return work(a) > work(b);
    });
    return mv::stack_plan(jobs, njobs, tuning, info);
}

}  // extern "C"

namespace mv {

mv_status stack_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning, mv_q8_stack_info *info) {
    const mv_q8_tuning t = mv::resolve(tuning);
    uint32_t item = 0;
    info->max_blk_rows = 2;
    info->tbl_stripe_max = 2;
    for (int j = 0; j < njobs; j++) {
        const mv_q8_view &m = jobs[j].m;
        if (m.rows <= 0 || m.cols <= 0 || (m.cols & 15) || m.nseg <= 0 || m.seg_quads <= 0 || (m.seg_quads & 3) ||
            ((uintptr_t)jobs[j].x & 15))
            return mv::fail(MV_ERR_ARG,
                            "mv_q8_stack_plan: job %d: needs cols %% 16 == 0, seg_quads %% 4 == 0 and a "
                            "16-byte aligned x",
                            j);
        if ((uint64_t)item + (uint64_t)((m.rows + 31) / 32) * (uint64_t)m.nseg > 0xFFFFFFFFull)
            return mv::fail(MV_ERR_SHAPE, "mv_q8_stack_plan: too many work items");
        mv::plan_job(jobs[j], t, item, t.parts);
        info->max_blk_rows = std::max(info->max_blk_rows, m.max_blk_rows);
        info->tbl_stripe_max = std::max(info->tbl_stripe_max, m.tbl_stripe_max);
    }
    info->nitems = item;
    info->atomic_jobs = 0;
    for (int j = 0; j < njobs; j++) info->atomic_jobs += jobs[j].atomic ? 1 : 0;
    info->warps = t.warps;
    info->ilp = t.ilp;
    info->depth = t.depth;
    return MV_OK;
}

}  // namespace mv

extern "C" {

size_t mv_q8_x_tiles_bytes(const mv_q8_view *m) {
    if (!m || m->nseg <= 0 || m->seg_quads <= 0) return 0;
    return (size_t)m->nseg * (size_t)((m->seg_quads + 31) / 32) * 2048;
}

mv_status mv_q8_chain_plan(mv_q8_job *jobs, int njobs, const mv_q8_tuning *tuning, mv_q8_stack_info *info) {
    if (!jobs || njobs <= 0 || !info) return mv::fail(MV_ERR_ARG, "mv_q8_chain_plan: bad arguments");
    for (int j = 0; j + 1 < njobs; j++)
        if (jobs[j].m.rows != jobs[j + 1].m.cols)
            return mv::fail(MV_ERR_SHAPE, "mv_q8_chain_plan: job %d has %d rows but job %d has %d columns", j,
                            jobs[j].m.rows, j + 1, jobs[j + 1].m.cols);
    mv_q8_tuning t = mv::resolve(tuning);
    if (t.parts > 1) return mv::fail(MV_ERR_ARG, "mv_q8_chain_plan: a chain needs whole stripes (parts <= 1)");
    t.parts = 0;
    return mv::stack_plan(jobs, njobs, &t, info);  // a chain keeps its order
}

mv_status mv_q8_chain_matvec(mv_q8_job *jobs_dev, int njobs, const mv_q8_stack_info *info, int batch,
                             const float *chain_scales_dev, int8_t *out8_dev, const mv_q8_tuning *tuning,
                             void *stream) {
    if (!jobs_dev || njobs <= 0 || !info || batch <= 0 || batch > 16 || !chain_scales_dev || !out8_dev)
        return mv::fail(MV_ERR_ARG, "mv_q8_chain_matvec: bad arguments (batch must be 1..16)");
    mv_q8_tuning t = mv::resolve(tuning);
    if (t.parts > 1) return mv::fail(MV_ERR_ARG, "mv_q8_chain_matvec: a chain needs whole stripes (parts <= 1)");
    if (t.warps != info->warps || t.ilp != info->ilp)
        return mv::fail(MV_ERR_ARG, "mv_q8_chain_matvec: tuning differs from the one the jobs were planned with");
    cudaStream_t st = (cudaStream_t)stream;
    mv_status rc;
    mv::Q8SLaunch L{};
    L.status = mv::device_status_word(&rc);
    if (rc) return rc;
    L.jobs = jobs_dev;
    L.njobs = njobs;
    L.nitems = info->nitems;
    L.batch = batch;
    L.spin_limit = mv::wait_spin_limit();
    L.drop_copy = mv::inject_drop_copy();
    L.buf_words = (info->max_blk_rows + 1) * 32;
    L.tbl_stage = (int)((info->tbl_stripe_max + 7) & ~7u);
    L.lut_stride = 32;
    L.chain_scales = chain_scales_dev;
    L.chain_out8 = out8_dev;
    mv::q8s_chain_reset<<<(njobs + 255) / 256, 256, 0, st>>>(reinterpret_cast<mv::Q8Job *>(jobs_dev), njobs);
    MV_CUDA_TRY(cudaGetLastError(), "q8s_chain_reset launch");
    return mv::launch_q8s(L, mv::nv_round(batch), t, st);
}

mv_status mv_q8_stack_matvec(const mv_q8_job *jobs_dev, int njobs, const mv_q8_stack_info *info, int batch,
                             const mv_q8_tuning *tuning, void *stream) {
    if (!jobs_dev || njobs <= 0 || !info || batch <= 0 || batch > 16)
        return mv::fail(MV_ERR_ARG, "mv_q8_stack_matvec: bad arguments (batch must be 1..16)");
    const mv_q8_tuning t = mv::resolve(tuning);
    if (t.warps != info->warps || t.ilp != info->ilp)
        return mv::fail(MV_ERR_ARG, "mv_q8_stack_matvec: tuning differs from the one the jobs were planned with");
    cudaStream_t st = (cudaStream_t)stream;
    mv_status rc;
    mv::Q8SLaunch L{};
    L.status = mv::device_status_word(&rc);
    if (rc) return rc;
    L.jobs = jobs_dev;
    L.njobs = njobs;
    L.nitems = info->nitems;
    L.batch = batch;
    L.spin_limit = mv::wait_spin_limit();
    L.drop_copy = mv::inject_drop_copy();
    L.buf_words = (info->max_blk_rows + 1) * 32;
    L.tbl_stage = (int)((info->tbl_stripe_max + 7) & ~7u);
    L.lut_stride = 32;
    // work queue: jobs_dev[0].pad, zero after planning and after every completed launch
    if (info->nitems < 0x7FFFFFFFu) L.queue = const_cast<uint32_t *>(&jobs_dev[0].pad);
    dim3 zg(64, std::min(njobs, 1024));
    if (info->atomic_jobs > 0) {
        mv::q8s_zero_atomic_y<<<zg, 256, 0, st>>>(jobs_dev, njobs, batch);
        MV_CUDA_TRY(cudaGetLastError(), "q8s_zero_atomic_y launch");
    }
    if (mv::nv_round(batch) >= mv::kMmaMinVectors && t.engine == MV_ENGINE_AUTO) {  // the tensor-core consumer reads x tiles
        mv::q8s_build_x_tiles<<<zg, 256, 0, st>>>(jobs_dev, njobs, batch);
        MV_CUDA_TRY(cudaGetLastError(), "q8s_build_x_tiles launch");
    }
    rc = mv::launch_q8s(L, mv::nv_round(batch), t, st);
    if (rc) return rc;
    if (info->atomic_jobs > 0) {
        mv::q8s_scale_atomic_y<<<zg, 256, 0, st>>>(jobs_dev, njobs, batch);
        MV_CUDA_TRY(cudaGetLastError(), "q8s_scale_atomic_y launch");
    }
    return MV_OK;
}

mv_status mv_q8_matvec_tuned(const mv_q8_view *m, const int8_t *x_dev, int batch, int32_t *y_dev,
                             const float *row_scales_dev, float *y_scaled_dev, const mv_q8_tuning *tuning,
                             void *stream) {
    if (!m || !x_dev || !y_dev || batch <= 0) return mv::fail(MV_ERR_ARG, "mv_q8_matvec_tuned: bad arguments");
    if (y_scaled_dev && !row_scales_dev) return mv::fail(MV_ERR_ARG, "mv_q8_matvec_tuned: y_scaled needs scales");
    if (!mv::q8s_supports(m, x_dev))
        return mv::fail(MV_ERR_ARG,
                        "mv_q8_matvec_tuned: needs cols %% 16 == 0, seg_quads %% 4 == 0 and 16-byte aligned x");
    return mv::q8s_matvec(m, x_dev, batch, y_dev, row_scales_dev, y_scaled_dev, tuning, (cudaStream_t)stream);
}

}  // extern "C"
