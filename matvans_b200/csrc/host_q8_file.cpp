// On-disk form of the Q8-stripe layout: a safetensors file, written and read by the same parser and writer
// as the reference's files (host_io.cpp), following the convention of buffered/encoder.py:473-511 --
// concatenated arrays of all matrices plus per-matrix start offsets, and the chain tensors under the
// reference's names:
//
//   q8_meta          I32 [count, 8]  rows, cols, seg_quads, nseg, local, max_blk_rows, tbl_stripe_max,
//                                    has_row_scales
//   q8_blocks        U32 [..]        every matrix's word-rows        q8_blocks_start   U64 [count + 1]
//   q8_blk_off       U32 [..]        block offsets (per matrix)      q8_blk_off_start  U64 [count + 1]
//   q8_tbl           U16 [..]        table entries                   q8_tbl_start      U64 [count + 1]
//   q8_tbl_off       U32 [..]        table offsets (per matrix)      q8_tbl_off_start  U64 [count + 1]
//   row_scales       F32 [..]        per-row fp32 scales (optional)  row_scales_start  U64 [count + 1]
//   initial_vector   I8  [n]         chain input (optional, encoder.py:498)
//   scales           F32 [count]     chain requantisation scale of each step (optional, encoder.py:499)
//   hashes           U32 [count]     hash of each step's int8 output (optional, encoder.py:500)
//
// Every array is validated against the layout's shape rules on read, so a truncated or inconsistent file
// is rejected on the host (MV_ERR_FORMAT) before anything reaches a kernel.
#include <cuda_runtime.h>

#include <cstdio>
#include <new>

#include "mv_internal.h"

struct mv_q8_matrix {
    mv_q8_view view{};
    void *blocks = nullptr, *blk_off = nullptr, *tbl = nullptr, *tbl_off = nullptr;
    float *row_scales = nullptr;
};

#define MV_CUDA_TRY_HOST(expr, what)                                                        \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) return mv::fail(MV_ERR_CUDA, "%s: %s", what, cudaGetErrorString(_e)); \
    } while (0)

namespace mv {
namespace {

constexpr int kMeta = 8;

template <class T>
const T *arr(const Blob &b, const char *name, size_t *n) {
    auto it = b.arrays.find(name);
    if (it == b.arrays.end()) return nullptr;
    *n = it->second.size() / sizeof(T);
    return reinterpret_cast<const T *>(it->second.data());
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Shape rules of one matrix (the ones the encoder guarantees and the kernels rely on).
mv_status check_host(const mv_q8_host &h, const char *what) {
    if (h.rows <= 0 || h.cols <= 0 || h.seg_quads <= 0 || h.nseg <= 0 || (h.local != 0 && h.local != 1))
        return fail(MV_ERR_FORMAT, "%s: bad dimensions", what);
    if (h.nseg != ceil_div(ceil_div(h.cols, 4), h.seg_quads))
        return fail(MV_ERR_FORMAT, "%s: nseg %d does not match cols %d and seg_quads %d", what, h.nseg, h.cols,
                    h.seg_quads);
    const int64_t stripes = ceil_div(h.rows, 32);
    if (!h.blk_off || (int64_t)h.n_blk_off != stripes * h.nseg + 1)
        return fail(MV_ERR_FORMAT, "%s: %zu block offsets, expected %lld", what, h.n_blk_off,
                    (long long)(stripes * h.nseg + 1));
    const int64_t ntables = h.local ? stripes * 32 : 1;
    if (!h.tbl_off || (int64_t)h.n_tbl_off != ntables + 1)
        return fail(MV_ERR_FORMAT, "%s: %zu table offsets, expected %lld", what, h.n_tbl_off,
                    (long long)(ntables + 1));
    if (!h.blocks || h.n_blocks % 32 || h.blk_off[h.n_blk_off - 1] > h.n_blocks / 32)
        return fail(MV_ERR_FORMAT, "%s: block data shorter than its offsets", what);
    for (size_t i = 0; i + 1 < h.n_blk_off; i++)
        if (h.blk_off[i + 1] < h.blk_off[i] || h.blk_off[i + 1] - h.blk_off[i] > (uint32_t)h.max_blk_rows)
            return fail(MV_ERR_FORMAT, "%s: block offsets not increasing or above max_blk_rows", what);
    if (!h.tbl || h.tbl_off[h.n_tbl_off - 1] > h.n_tbl)
        return fail(MV_ERR_FORMAT, "%s: table data shorter than its offsets", what);
    for (size_t i = 0; i + 1 < h.n_tbl_off; i++)
        if (h.tbl_off[i + 1] < h.tbl_off[i]) return fail(MV_ERR_FORMAT, "%s: table offsets not increasing", what);
    return MV_OK;
}

template <class T>
void put_cat(Blob &b, const std::string &name, int dtype, const std::vector<std::vector<T>> &parts) {
    std::vector<T> all;
    std::vector<uint64_t> start{0};
    for (const auto &p : parts) {
        all.insert(all.end(), p.begin(), p.end());
        start.push_back(all.size());
    }
    b.put(name, all);
    b.shape(name, dtype, {(int64_t)all.size()});
    b.put(name + "_start", start);
    b.shape(name + "_start", DT_U64, {(int64_t)start.size()});
}

template <class T>
mv_status dev_copy(void **dst, const T *src, size_t n, size_t pad_bytes) {
    const size_t bytes = n * sizeof(T);
    MV_CUDA_TRY_HOST(cudaMalloc(dst, bytes + pad_bytes), "cudaMalloc");
    if (pad_bytes) MV_CUDA_TRY_HOST(cudaMemset((char *)*dst + bytes, 0, pad_bytes), "cudaMemset");
    if (bytes) MV_CUDA_TRY_HOST(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
    return MV_OK;
}

}  // namespace
}  // namespace mv

extern "C" {

mv_status mv_q8_save(const char *path, const mv_q8_host *mats, int count, const mv_q8_chain_host *chain) {
    if (!path || !mats || count <= 0) return mv::fail(MV_ERR_ARG, "mv_q8_save: bad arguments");
    std::vector<std::vector<uint32_t>> blocks, blk_off, tbl_off;
    std::vector<std::vector<uint16_t>> tbl;
    std::vector<std::vector<float>> scales;
    std::vector<int32_t> meta;
    bool any_scales = false;
    for (int i = 0; i < count; i++) {
        const mv_q8_host &h = mats[i];
        char what[48];
        std::snprintf(what, sizeof what, "mv_q8_save: matrix %d", i);
        mv_status rc = mv::check_host(h, what);
        if (rc) return rc;
        blocks.emplace_back(h.blocks, h.blocks + h.n_blocks);
        blk_off.emplace_back(h.blk_off, h.blk_off + h.n_blk_off);
        tbl.emplace_back(h.tbl, h.tbl + h.n_tbl);
        tbl_off.emplace_back(h.tbl_off, h.tbl_off + h.n_tbl_off);
        scales.emplace_back(h.row_scales ? std::vector<float>(h.row_scales, h.row_scales + h.rows)
                                         : std::vector<float>());
        any_scales |= h.row_scales != nullptr;
        meta.insert(meta.end(), {h.rows, h.cols, h.seg_quads, h.nseg, h.local, h.max_blk_rows,
                                 (int32_t)h.tbl_stripe_max, h.row_scales ? 1 : 0});
    }
    mv_blob b;
    b.put("q8_meta", meta);
    b.shape("q8_meta", mv::DT_I32, {count, mv::kMeta});
    mv::put_cat(b, "q8_blocks", mv::DT_U32, blocks);
    mv::put_cat(b, "q8_blk_off", mv::DT_U32, blk_off);
    mv::put_cat(b, "q8_tbl", mv::DT_U16, tbl);
    mv::put_cat(b, "q8_tbl_off", mv::DT_U32, tbl_off);
    if (any_scales) mv::put_cat(b, "row_scales", mv::DT_F32, scales);
    if (chain) {
        if (chain->initial_vector) {
            b.put("initial_vector", std::vector<int8_t>(chain->initial_vector,
                                                       chain->initial_vector + chain->n_initial));
            b.shape("initial_vector", mv::DT_I8, {(int64_t)chain->n_initial});
        }
        if (chain->scales) {
            b.put("scales", std::vector<float>(chain->scales, chain->scales + count));
            b.shape("scales", mv::DT_F32, {count});
        }
        if (chain->hashes) {
            b.put("hashes", std::vector<uint32_t>(chain->hashes, chain->hashes + count));
            b.shape("hashes", mv::DT_U32, {count});
        }
    }
    return mv_write_safetensors(path, &b);
}

mv_status mv_q8_file_count(const mv_blob *file, int *count) {
    if (!file || !count) return mv::fail(MV_ERR_ARG, "mv_q8_file_count: NULL argument");
    size_t n = 0;
    if (!mv::arr<int32_t>(*file, "q8_meta", &n) || n % mv::kMeta || n == 0)
        return mv::fail(MV_ERR_FORMAT, "not a Q8 file: no q8_meta tensor");
    *count = (int)(n / mv::kMeta);
    return MV_OK;
}

mv_status mv_q8_file_matrix(const mv_blob *file, int index, mv_q8_host *out) {
    if (!file || !out) return mv::fail(MV_ERR_ARG, "mv_q8_file_matrix: NULL argument");
    int count = 0;
    mv_status rc = mv_q8_file_count(file, &count);
    if (rc) return rc;
    if (index < 0 || index >= count) return mv::fail(MV_ERR_ARG, "mv_q8_file_matrix: index %d of %d", index, count);
    size_t nm = 0;
    const int32_t *meta = mv::arr<int32_t>(*file, "q8_meta", &nm) + (size_t)index * mv::kMeta;
    mv_q8_host h{};
    h.rows = meta[0];
    h.cols = meta[1];
    h.seg_quads = meta[2];
    h.nseg = meta[3];
    h.local = meta[4];
    h.max_blk_rows = meta[5];
    h.tbl_stripe_max = (uint32_t)meta[6];
    // one concatenated array and its start offsets -> this matrix's part
    auto part = [&](const char *name, size_t esize, const void **p, size_t *n) -> mv_status {
        auto it = file->arrays.find(name);
        size_t ns = 0;
        const uint64_t *st = mv::arr<uint64_t>(*file, (std::string(name) + "_start").c_str(), &ns);
        if (it == file->arrays.end() || !st || ns != (size_t)count + 1)
            return mv::fail(MV_ERR_FORMAT, "Q8 file: tensor %s or its start offsets missing", name);
        const size_t total = it->second.size() / esize;
        if (st[index] > st[index + 1] || st[index + 1] > total)
            return mv::fail(MV_ERR_FORMAT, "Q8 file: start offsets of %s out of range", name);
        *p = it->second.data() + st[index] * esize;
        *n = (size_t)(st[index + 1] - st[index]);
        return MV_OK;
    };
    const void *p = nullptr;
    if ((rc = part("q8_blocks", 4, &p, &h.n_blocks))) return rc;
    h.blocks = (const uint32_t *)p;
    if ((rc = part("q8_blk_off", 4, &p, &h.n_blk_off))) return rc;
    h.blk_off = (const uint32_t *)p;
    if ((rc = part("q8_tbl", 2, &p, &h.n_tbl))) return rc;
    h.tbl = (const uint16_t *)p;
    if ((rc = part("q8_tbl_off", 4, &p, &h.n_tbl_off))) return rc;
    h.tbl_off = (const uint32_t *)p;
    h.row_scales = nullptr;
    if (meta[7]) {
        size_t n = 0;
        if ((rc = part("row_scales", 4, &p, &n))) return rc;
        if (n != (size_t)h.rows) return mv::fail(MV_ERR_FORMAT, "Q8 file: matrix %d has %zu row scales", index, n);
        h.row_scales = (const float *)p;
    }
    char what[48];
    std::snprintf(what, sizeof what, "Q8 file: matrix %d", index);
    if ((rc = mv::check_host(h, what))) return rc;
    *out = h;
    return MV_OK;
}

mv_status mv_q8_file_chain(const mv_blob *file, mv_q8_chain_host *out) {
    if (!file || !out) return mv::fail(MV_ERR_ARG, "mv_q8_file_chain: NULL argument");
    int count = 0;
    mv_status rc = mv_q8_file_count(file, &count);
    if (rc) return rc;
    mv_q8_chain_host c{};
    size_t n = 0;
    c.initial_vector = mv::arr<int8_t>(*file, "initial_vector", &n);
    c.n_initial = c.initial_vector ? n : 0;
    c.scales = mv::arr<float>(*file, "scales", &n);
    if (c.scales && n != (size_t)count) return mv::fail(MV_ERR_FORMAT, "Q8 file: %zu chain scales", n);
    c.hashes = mv::arr<uint32_t>(*file, "hashes", &n);
    if (c.hashes && n != (size_t)count) return mv::fail(MV_ERR_FORMAT, "Q8 file: %zu chain hashes", n);
    *out = c;
    return MV_OK;
}

void mv_q8_matrix_free(mv_q8_matrix *m) {
    if (!m) return;
    cudaFree(m->blocks);
    cudaFree(m->blk_off);
    cudaFree(m->tbl);
    cudaFree(m->tbl_off);
    cudaFree(m->row_scales);
    delete m;
}

mv_status mv_q8_upload(const mv_q8_host *h, mv_q8_matrix **out) {
    if (!h || !out) return mv::fail(MV_ERR_ARG, "mv_q8_upload: NULL argument");
    mv_status rc = mv::check_host(*h, "mv_q8_upload");
    if (rc) return rc;
    auto *m = new (std::nothrow) mv_q8_matrix;
    if (!m) return mv::fail(MV_ERR_NOMEM, "out of memory");
    // the stream blocks keep one readable word-row past the end; the table array a 16-byte readable tail
    if ((rc = mv::dev_copy(&m->blocks, h->blocks, h->n_blocks, 128)) ||
        (rc = mv::dev_copy(&m->blk_off, h->blk_off, h->n_blk_off, 0)) ||
        (rc = mv::dev_copy(&m->tbl, h->tbl, h->n_tbl, 16)) ||
        (rc = mv::dev_copy(&m->tbl_off, h->tbl_off, h->n_tbl_off, 0)) ||
        (h->row_scales && (rc = mv::dev_copy((void **)&m->row_scales, h->row_scales, (size_t)h->rows, 0)))) {
        mv_q8_matrix_free(m);
        return rc;
    }
    mv_q8_view &v = m->view;
    v.blocks = (const uint32_t *)m->blocks;
    v.blk_off = (const uint32_t *)m->blk_off;
    v.tbl = (const uint16_t *)m->tbl;
    v.tbl_off = (const uint32_t *)m->tbl_off;
    v.rows = h->rows;
    v.cols = h->cols;
    v.seg_quads = h->seg_quads;
    v.nseg = h->nseg;
    v.local = h->local;
    v.max_blk_rows = h->max_blk_rows;
    v.blocks_rows = (uint32_t)(h->n_blocks / 32);
    v.tbl_len = (uint32_t)h->n_tbl;
    v.tbl_stripe_max = h->tbl_stripe_max;
    *out = m;
    return MV_OK;
}

const mv_q8_view *mv_q8_matrix_view(const mv_q8_matrix *m) { return m ? &m->view : nullptr; }

const float *mv_q8_matrix_row_scales(const mv_q8_matrix *m) { return m ? m->row_scales : nullptr; }

mv_status mv_q8_load(const char *path, int index, mv_q8_matrix **out) {
    if (!path || !out) return mv::fail(MV_ERR_ARG, "mv_q8_load: NULL argument");
    mv_blob *b = nullptr;
    mv_status rc = mv_read_safetensors(path, &b);
    if (rc) return rc;
    mv_q8_host h{};
    rc = mv_q8_file_matrix(b, index, &h);
    if (!rc) rc = mv_q8_upload(&h, out);
    mv_blob_free(b);
    return rc;
}

}  // extern "C"
