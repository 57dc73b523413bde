// Reference-compatible encoders: byte-identical restatements of the
// reference's Python encoders, so that files written by this library decode
// with the reference kernels and vice versa.
//
//   AWR ("ans-warp-rows"):  buffered/encoder.py:113-268 (DetachedAnsQuadCoder),
//                           :271-306 (fit_128bit_encoder_model),
//                           :309-320 (decoder_model_from_128bit_encoder_model),
//                           :394-461 (compress_ans_warp_rows), :464-470 (pack_4bytes)
//   AWS ("ans-warp-stripes"): the same coder and model, :323-391 (compress_ans_warp_stripes)
//   WPR ("matvansWarpPerRow"): matvansWarpPerRow/create_matrices_WarpPerRow.py:
//                           :131-187 (create_entropy_model), :189-208 (create_ppf),
//                           :211-272 (AnsCoder), :353-430 (encode_matrix)
#include <algorithm>
#include <cmath>
#include <numeric>
#include <thread>

#include "mv_internal.h"

namespace mv {
namespace {

// ------------------------------------------------------------------- AWR

struct AwrModel {
    int min_value = 0;
    std::vector<uint8_t> cdf;  // max-min+2 entries, cdf.back() == 128
};

// fit_128bit_encoder_model, buffered/encoder.py:271-306.  The pmf is computed
// in float32 exactly as numpy does it: counts.astype(float32) * 128 / numel,
// rounded half to even, clamped below at 1, then the sum is forced to 128 by
// repeatedly decrementing (incrementing) the first maximal entry.
mv_status fit_awr_model(const int8_t *W, int64_t n, AwrModel &m) {
    int64_t hist[256] = {0};
    for (int64_t i = 0; i < n; i++) hist[(uint8_t)W[i] ^ 0x80]++;  // index = value + 128
    std::vector<int> values;
    std::vector<int64_t> counts;
    for (int v = 0; v < 256; v++)
        if (hist[v]) { values.push_back(v - 128); counts.push_back(hist[v]); }
    if (values.size() > 128)
        return fail(MV_ERR_UNSUPPORTED, "AWR layout holds at most 128 distinct values, got %zu",
                    values.size());
    const float numel_f = (float)n;
    std::vector<uint32_t> pmf(values.size());
    for (size_t i = 0; i < values.size(); i++) {
        volatile float c = (float)counts[i];
        volatile float t = c * 128.0f;
        volatile float q = t / numel_f;
        float r = std::nearbyintf(q);
        uint32_t u = (uint32_t)r;
        pmf[i] = std::max<uint32_t>(1u, u);
    }
    uint64_t sum = 0;
    for (auto f : pmf) sum += f;
    auto argmax = [&]() {
        size_t best = 0;
        for (size_t i = 1; i < pmf.size(); i++)
            if (pmf[i] > pmf[best]) best = i;
        return best;
    };
    if (sum > 128)
        for (uint64_t k = 0; k < sum - 128; k++) pmf[argmax()] -= 1;
    else
        for (uint64_t k = 0; k < 128 - sum; k++) pmf[argmax()] += 1;
    m.min_value = values.front();
    const int maxv = values.back();
    m.cdf.assign(maxv - m.min_value + 2, 0);
    uint32_t left = 0;
    int last = 0;
    for (size_t i = 0; i < values.size(); i++) {
        int idx = values[i] - m.min_value;
        for (int k = last + 1; k < idx + 1; k++) m.cdf[k] = (uint8_t)left;
        last = idx;
        left += pmf[i];
    }
    if (left != 128) return fail(MV_ERR_FORMAT, "AWR model does not sum to 128 (%u)", left);
    m.cdf.back() = 128;
    return MV_OK;
}

// decoder_model_from_128bit_encoder_model + pack_4bytes, encoder.py:309-320,464-470.
void awr_decoder_tables(const AwrModel &m, uint32_t ppf[32], uint32_t cum[32], uint32_t prob[32]) {
    uint8_t p8[128] = {0}, c8[128] = {0}, r8[128] = {0};
    for (size_t idx = 0; idx + 1 < m.cdf.size(); idx++) {
        uint32_t l = m.cdf[idx], r = m.cdf[idx + 1];
        for (uint32_t q = l; q < r; q++) {
            p8[q] = (uint8_t)(int8_t)(idx + m.min_value);
            c8[q] = (uint8_t)l;
            r8[q] = (uint8_t)(r - l);
        }
    }
    for (int i = 0; i < 32; i++) {
        ppf[i] = cum[i] = prob[i] = 0;
        for (int b = 0; b < 4; b++) {
            ppf[i] |= (uint32_t)p8[4 * i + b] << (8 * b);
            cum[i] |= (uint32_t)c8[4 * i + b] << (8 * b);
            prob[i] |= (uint32_t)r8[4 * i + b] << (8 * b);
        }
    }
}

// DetachedAnsQuadCoder.encode(precision=7, word=32, state=64), encoder.py:190-226.
inline void awr_encode_quad(uint64_t &state, const int8_t *quad, const AwrModel &m,
                            std::vector<uint32_t> &buf) {
    uint32_t left[4], p[4];
    uint64_t total = 1;
    for (int i = 0; i < 4; i++) {
        int idx = quad[i] - m.min_value;
        left[i] = m.cdf[idx];
        p[i] = (uint32_t)m.cdf[idx + 1] - left[i];
        total *= p[i];
    }
    if ((state >> 36) >= total) {
        buf.push_back((uint32_t)state);
        state >>= 32;
    } else if (state == 0) {
        state = total << 4;
    }
    uint64_t concat = 0;
    for (int i = 0; i < 4; i++) {
        uint64_t rem = state % p[i];
        state /= p[i];
        concat |= (uint64_t)(left[i] + rem) << (7 * i);
    }
    state = (state << 28) | concat;
}

// The word stream of one warp (an AWR row or an "ans-warp-stripes" stripe) as the decoder reads it
// (encoder.py:431-447 and :355-383, identical steps): the joint bulk of the 32 coders reversed, padded
// with zeros to a length of 64 (mod 128), the 32 low then the 32 high state words inserted at word 64,
// and every 128-word block transposed so that lane l's uint4 holds words (l, 32+l, 64+l, 96+l).
void awr_assemble(const std::vector<uint32_t> &buf, const uint64_t (&state)[32], std::vector<uint32_t> &bulk,
                  std::vector<uint32_t> &compressed) {
    bulk.assign(buf.rbegin(), buf.rend());
    int64_t pad = ((64 - (int64_t)bulk.size()) % 128 + 128) % 128;
    bulk.resize(bulk.size() + pad, 0u);
    std::vector<uint32_t> un;
    un.reserve(bulk.size() + 64);
    un.insert(un.end(), bulk.begin(), bulk.begin() + 64);
    for (int l = 0; l < 32; l++) un.push_back((uint32_t)state[l]);
    for (int l = 0; l < 32; l++) un.push_back((uint32_t)(state[l] >> 32));
    un.insert(un.end(), bulk.begin() + 64, bulk.end());
    const size_t blocks = un.size() / 128;
    for (size_t b = 0; b < blocks; b++)
        for (int l = 0; l < 32; l++)
            for (int f = 0; f < 4; f++) compressed.push_back(un[b * 128 + f * 32 + l]);
}

void awr_put_tables(const AwrModel &m, Blob &out) {
    uint32_t ppf[32], cum[32], prob[32];
    awr_decoder_tables(m, ppf, cum, prob);
    out.put("cdf", m.cdf);
    out.shape("cdf", DT_U8, {(int64_t)m.cdf.size()});
    out.put("ppf", std::vector<uint32_t>(ppf, ppf + 32));
    out.put("ppf_cum", std::vector<uint32_t>(cum, cum + 32));
    out.put("ppf_prob", std::vector<uint32_t>(prob, prob + 32));
    for (const char *n : {"ppf", "ppf_cum", "ppf_prob"}) out.shape(n, DT_U32, {32});
    out.set("min_value", m.min_value);
}

}  // namespace

// compress_ans_warp_stripes(matrix, 32), encoder.py:323-391.  Lane l of stripe s is row 32s + l; a
// stripe's quads are coded column by column from the last (lanes 31..0 within a column) into one joint
// stream, and, as in the rows layout, the 32 coders carry their states from stripe to stripe.
static mv_status aws_encode(const int8_t *W, int rows, int cols, Blob &out) {
    if (!W || rows <= 0 || cols <= 0) return fail(MV_ERR_ARG, "mv_aws_encode: bad arguments");
    if (rows % 32 || cols % 4)
        return fail(MV_ERR_SHAPE, "stripes layout needs rows %% 32 == 0 and cols %% 4 == 0 (%dx%d)", rows, cols);
    AwrModel m;
    mv_status st = fit_awr_model(W, (int64_t)rows * cols, m);
    if (st) return st;
    for (int64_t i = 0; i < (int64_t)rows * cols; i++) {
        int idx = W[i] - m.min_value;
        if (m.cdf[idx + 1] == m.cdf[idx]) return fail(MV_ERR_FORMAT, "AWR model lost a symbol");
    }
    const int stripes = rows / 32, quads = cols / 4;
    std::vector<uint32_t> compressed, offsets(stripes), buf, bulk;
    uint64_t state[32] = {0};
    for (int s = 0; s < stripes; s++) {
        if (compressed.size() / 4 > 0xFFFFFFFFull) return fail(MV_ERR_SHAPE, "stripes offsets overflow 32 bits");
        offsets[s] = (uint32_t)(compressed.size() / 4);
        buf.clear();
        for (int c = quads - 1; c >= 0; c--)
            for (int l = 31; l >= 0; l--)
                awr_encode_quad(state[l], W + ((int64_t)s * 32 + l) * cols + 4 * c, m, buf);
        awr_assemble(buf, state, bulk, compressed);
    }
    out.put("compressed", compressed);
    out.shape("compressed", DT_U32, {(int64_t)compressed.size()});
    out.put("warp_offsets", offsets);
    out.shape("warp_offsets", DT_U32, {stripes});
    awr_put_tables(m, out);
    out.set("rows", rows);
    out.set("cols", cols);
    return MV_OK;
}

// compress_ans_warp_rows(matrix, 32), encoder.py:394-461.  The 32 coders are
// created once per matrix and are NOT reset between rows (encoder.py:402), so
// each row continues from the previous row's final states; rows are therefore
// encoded in order.
static mv_status awr_encode(const int8_t *W, int rows, int cols, Blob &out) {
    if (!W || rows <= 0 || cols <= 0) return fail(MV_ERR_ARG, "mv_awr_encode: bad arguments");
    if (cols % 128) return fail(MV_ERR_SHAPE, "AWR layout needs cols %% 128 == 0 (cols=%d)", cols);
    AwrModel m;
    mv_status st = fit_awr_model(W, (int64_t)rows * cols, m);
    if (st) return st;
    for (int64_t i = 0; i < (int64_t)rows * cols; i++) {
        int idx = W[i] - m.min_value;
        if (m.cdf[idx + 1] == m.cdf[idx]) return fail(MV_ERR_FORMAT, "AWR model lost a symbol");
    }
    std::vector<uint32_t> compressed;
    std::vector<uint32_t> offsets(rows);
    uint64_t state[32] = {0};
    std::vector<uint32_t> buf, bulk;
    const int chunks = cols / 128;
    for (int r = 0; r < rows; r++) {
        if (compressed.size() / 4 > 0xFFFFFFFFull)
            return fail(MV_ERR_SHAPE, "AWR offsets overflow 32 bits");
        offsets[r] = (uint32_t)(compressed.size() / 4);
        buf.clear();
        const int8_t *row = W + (int64_t)r * cols;
        for (int c = chunks - 1; c >= 0; c--)
            for (int l = 31; l >= 0; l--) awr_encode_quad(state[l], row + 128 * c + 4 * l, m, buf);
        awr_assemble(buf, state, bulk, compressed);
    }
    out.put("compressed", compressed);
    out.shape("compressed", DT_U32, {(int64_t)compressed.size()});
    out.put("warp_offsets", offsets);
    out.shape("warp_offsets", DT_U32, {rows});
    awr_put_tables(m, out);
    out.set("rows", rows);
    out.set("cols", cols);
    return MV_OK;
}

// ------------------------------------------------------------------- WPR

namespace {

struct WprModel {
    int min_value = 0;
    int grid = 0;
    std::vector<uint16_t> cdf;  // grid + 1 entries, back() == 256
};

// create_entropy_model(data, precision=8), create_matrices_WarpPerRow.py:131-187.
// The reference sorts by count with np.argsort(counts)[::-1]; numpy's default
// argsort is not stable, so equal counts may come out in any order.  This port
// uses the stable order (ascending by count, ties by ascending value, then
// reversed), which agrees with every fixture produced by the reference.
mv_status fit_wpr_model(const int8_t *W, int64_t n, WprModel &m) {
    int64_t hist[256] = {0};
    for (int64_t i = 0; i < n; i++) hist[(uint8_t)W[i] ^ 0x80]++;
    std::vector<int> values;
    std::vector<int64_t> counts;
    for (int v = 0; v < 256; v++)
        if (hist[v]) { values.push_back(v - 128); counts.push_back(hist[v]); }
    const int precision = 8;
    m.min_value = values.front();
    const int maxv = values.back();
    if (m.min_value == maxv) {
        m.grid = 2;
        m.cdf = {0, (uint16_t)((1 << precision) - 1), (uint16_t)(1 << precision)};
        return MV_OK;
    }
    m.grid = maxv - m.min_value + 1;
    std::vector<size_t> order(values.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return counts[a] < counts[b]; });
    std::reverse(order.begin(), order.end());
    const double scale = (double)(1 << precision) / (double)n;
    std::vector<uint16_t> q(order.size());
    for (size_t i = 0; i < order.size(); i++) {
        double v = std::nearbyint((double)counts[order[i]] * scale);
        q[i] = (uint16_t)std::max(1.0, v);
    }
    int64_t excess = 0;
    for (auto f : q) excess += f;
    excess -= (1 << precision);
    if (excess > 0) {
        while (excess > 0) {
            int64_t reducible = 0;
            for (auto f : q) reducible += f > 1;
            int64_t num = std::min(excess, reducible);
            if (num <= 0) return fail(MV_ERR_FORMAT, "WPR model cannot shed excess mass");
            for (int64_t i = 0; i < num; i++) q[i] -= 1;
            excess -= num;
        }
    } else if (excess < 0) {
        if (-excess > (int64_t)q.size()) return fail(MV_ERR_FORMAT, "WPR model deficit too large");
        for (size_t i = q.size() + excess; i < q.size(); i++) q[i] += 1;
    }
    std::vector<uint16_t> padded(m.grid + 1, 0);
    for (size_t i = 0; i < order.size(); i++) padded[values[order[i]] - m.min_value + 1] = q[i];
    m.cdf.resize(m.grid + 1);
    uint16_t acc = 0;
    for (int i = 0; i <= m.grid; i++) { acc = (uint16_t)(acc + padded[i]); m.cdf[i] = acc; }
    if (m.cdf[0] != 0 || m.cdf.back() != (1 << precision))
        return fail(MV_ERR_FORMAT, "WPR model does not sum to 256");
    return MV_OK;
}

// create_ppf, create_matrices_WarpPerRow.py:189-208.
void wpr_ppf(const WprModel &m, uint8_t ppf[256]) {
    for (int p = 0; p < 256; p++) {
        ppf[p] = 0;
        for (int r = (int)m.cdf.size() - 1; r > 0; r--)
            if ((uint8_t)(m.cdf[r - 1] & 0xFF) <= p) { ppf[p] = (uint8_t)(r - 1); break; }
    }
}

}  // namespace

// encode_matrix, create_matrices_WarpPerRow.py:353-430 (for general rows x
// cols: lane j owns columns 512k + 16j .. 512k + 16j + 15).
static mv_status wpr_encode(const int8_t *W, int rows, int cols, int nthreads, Blob &out) {
    if (!W || rows <= 0 || cols <= 0) return fail(MV_ERR_ARG, "mv_wpr_encode: bad arguments");
    if (cols % 512) return fail(MV_ERR_SHAPE, "WPR layout needs cols %% 512 == 0 (cols=%d)", cols);
    WprModel m;
    mv_status st = fit_wpr_model(W, (int64_t)rows * cols, m);
    if (st) return st;
    uint8_t ppf[256];
    wpr_ppf(m, ppf);
    const int per_lane = cols / 32;
    // per (row, lane) payload in decode order: [hi, lo, words...]
    std::vector<std::vector<uint16_t>> lane_payload((size_t)rows * 32);
    auto work = [&](int r0, int r1) {
        std::vector<uint16_t> bulk;
        for (int r = r0; r < r1; r++) {
            const int8_t *row = W + (int64_t)r * cols;
            for (int l = 0; l < 32; l++) {
                uint32_t head = 1u << 16;  // AnsCoder(8, 16, compressed=[0, 1])
                bulk.clear();
                for (int j = per_lane - 1; j >= 0; j--) {
                    int col = 512 * (j / 16) + 16 * l + j % 16;
                    int s = row[col] - m.min_value;
                    uint32_t prob = (uint32_t)m.cdf[s + 1] - m.cdf[s];
                    if ((head >> 24) >= prob) {
                        while ((head >> 16) != 0) { bulk.push_back((uint16_t)head); head >>= 16; }
                    }
                    uint32_t z = head % prob + m.cdf[s];
                    head = ((head / prob) << 8) | z;
                }
                bulk.push_back((uint16_t)head);          // interrupt(): low word
                bulk.push_back((uint16_t)(head >> 16));  // then high word
                auto &dst = lane_payload[(size_t)r * 32 + l];
                dst.assign(bulk.rbegin(), bulk.rend());
            }
        }
    };
    int nt = std::max(1, std::min(nthreads_or_default(nthreads), rows));
    std::vector<std::thread> th;
    int per = (rows + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        int r0 = t * per, r1 = std::min(rows, r0 + per);
        if (r0 < r1) th.emplace_back(work, r0, r1);
    }
    for (auto &t : th) t.join();
    std::vector<uint32_t> cursors(rows);
    std::vector<uint16_t> payload;
    for (int r = 0; r < rows; r++) {
        size_t mx = 0;
        for (int l = 0; l < 32; l++) mx = std::max(mx, lane_payload[(size_t)r * 32 + l].size());
        size_t int4s = (mx + 7) / 8;
        if (payload.size() > 0xFFFFFFFFull) return fail(MV_ERR_SHAPE, "WPR cursors overflow");
        cursors[r] = (uint32_t)payload.size();
        size_t base = payload.size();
        payload.resize(base + int4s * 32 * 8, 0);
        for (int l = 0; l < 32; l++) {
            const auto &p = lane_payload[(size_t)r * 32 + l];
            for (size_t j = 0; j < p.size(); j++) payload[base + (j / 8) * 256 + l * 8 + j % 8] = p[j];
        }
    }
    std::vector<uint8_t> cdf8(m.cdf.size());
    for (size_t i = 0; i < m.cdf.size(); i++) cdf8[i] = (uint8_t)(m.cdf[i] & 0xFF);
    out.put("payload", payload);
    out.shape("payload", DT_U16, {(int64_t)payload.size()});
    out.put("cursors", cursors);
    out.shape("cursors", DT_U32, {rows});
    out.put("cdf", cdf8);
    out.shape("cdf", DT_U8, {(int64_t)cdf8.size()});
    out.put("ppf", std::vector<uint8_t>(ppf, ppf + 256));
    out.shape("ppf", DT_U8, {256});
    out.set("min_value", m.min_value);
    out.set("G", (int64_t)cdf8.size() - 1);
    out.set("rows", rows);
    out.set("cols", cols);
    return MV_OK;
}

}  // namespace mv

extern "C" {

mv_status mv_awr_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out) {
    (void)nthreads;  // rows depend on each other (shared coders); encoded in order
    if (!out) return mv::fail(MV_ERR_ARG, "mv_awr_encode: NULL out");
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "mv_awr_encode: out of memory");
    mv_status st = mv::awr_encode(W, rows, cols, *b);
    if (st) { delete b; return st; }
    *out = b;
    return MV_OK;
}

mv_status mv_aws_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out) {
    (void)nthreads;  // stripes depend on each other (shared coders); encoded in order
    if (!out) return mv::fail(MV_ERR_ARG, "mv_aws_encode: NULL out");
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "mv_aws_encode: out of memory");
    mv_status st = mv::aws_encode(W, rows, cols, *b);
    if (st) { delete b; return st; }
    *out = b;
    return MV_OK;
}

mv_status mv_wpr_encode(const int8_t *W, int rows, int cols, int nthreads, mv_blob **out) {
    if (!out) return mv::fail(MV_ERR_ARG, "mv_wpr_encode: NULL out");
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "mv_wpr_encode: out of memory");
    mv_status st = mv::wpr_encode(W, rows, cols, nthreads, *b);
    if (st) { delete b; return st; }
    *out = b;
    return MV_OK;
}

}  // extern "C"
