// Encoder for the Q8-stripe layout (this library's own layout; the kernel is
// k_q8.cu, the layout is documented on mv_q8_view in include/matvans.h).
//
// Coder: per lane, rANS with 8-bit probabilities, a 64-bit state and 32-bit
// refill words, four symbols per step (the quad coder of
// buffered/encoder.py:113-268 re-parameterised from 7-bit to 8-bit
// precision, so the four quantiles are exactly the low 32-bit word of the
// state and the update is one 32x32->64 multiply-add):
//   decode step: if (S >> 32) == 0: S = S << 32 | next_word
//                q_i = byte i of S (i = 0..3); (sym_i, f_i, c_i) = table(q_i)
//                S = (S >> 32) * prod(f_i) + (r0 + f0*(r1 + f1*(r2 + f2*r3))),
//                with r_i = q_i - c_i
//   encode step (reverse order): if E == 0: E = P (first quad)
//                elif (E >> 32) >= P: emit(E & 0xffffffff), E >>= 32
//                E = (E / P) << 32 | quantiles(E % P)
// so every decoder state after a refill lies in [2^32, 2^64) and the decoder
// of a segment ends exactly in state P of its last quad (checked on device).
#include <algorithm>
#include <cmath>
#include <thread>

#include "mv_internal.h"

namespace mv {
namespace {

struct Table {
    std::vector<uint16_t> entries;  // sym | freq << 8, sorted by sym (as uint8 of int8 value)
    uint16_t freq[256];             // by (uint8)value
    uint16_t cum[256];
    int pad_sym = 0;                // most probable symbol (int8 value)
};

// Quantise a histogram to 256 with every present symbol >= 1 and <= 255,
// minimising the cross entropy greedily from the rounded start.
void fit_table(const int64_t *counts /*[256], index = value + 128*/, Table &t) {
    std::vector<int> present;
    int64_t n = 0;
    for (int i = 0; i < 256; i++)
        if (counts[i]) { present.push_back(i); n += counts[i]; }
    std::fill(t.freq, t.freq + 256, 0);
    if (present.empty()) present.push_back(128);  // empty input: value 0
    if (present.size() == 1) {
        int s = present[0];
        int s2 = (s == 255) ? 254 : s + 1;
        t.freq[s] = 255;
        t.freq[s2] = 1;
    } else {
        std::vector<int> f(present.size());
        int64_t sum = 0;
        for (size_t i = 0; i < present.size(); i++) {
            double v = std::nearbyint((double)counts[present[i]] * 256.0 / (double)n);
            f[i] = (int)std::min(255.0, std::max(1.0, v));
            sum += f[i];
        }
        while (sum != 256) {
            size_t best = SIZE_MAX;
            double best_cost = 0;
            for (size_t i = 0; i < present.size(); i++) {
                double c = (double)counts[present[i]];
                if (sum < 256 && f[i] < 255) {
                    double gain = c * (std::log2((double)f[i] + 1) - std::log2((double)f[i]));
                    if (best == SIZE_MAX || gain > best_cost) { best = i; best_cost = gain; }
                } else if (sum > 256 && f[i] > 1) {
                    double loss = c * (std::log2((double)f[i]) - std::log2((double)f[i] - 1));
                    if (best == SIZE_MAX || loss < best_cost) { best = i; best_cost = loss; }
                }
            }
            if (best == SIZE_MAX) break;  // cannot happen: 2 <= K <= 256
            f[best] += sum < 256 ? 1 : -1;
            sum += sum < 256 ? 1 : -1;
        }
        for (size_t i = 0; i < present.size(); i++) t.freq[present[i]] = (uint16_t)f[i];
    }
    t.entries.clear();
    uint16_t acc = 0, best_f = 0;
    for (int i = 0; i < 256; i++) {
        t.cum[i] = acc;
        if (t.freq[i]) {
            // entry symbol byte = uint8 of the int8 value (i - 128)
            t.entries.push_back((uint16_t)(((uint8_t)(int8_t)(i - 128)) | (t.freq[i] << 8)));
            if (t.freq[i] > best_f) { best_f = t.freq[i]; t.pad_sym = i - 128; }
        }
        acc = (uint16_t)(acc + t.freq[i]);
    }
}

// Sort key of the kernel: entries are consumed in stored order, and the
// quantile ranges follow that order.  Store in order of the uint8 symbol byte
// so that cum[] (by value) must be recomputed in the same order.
void order_like_kernel(Table &t) {
    std::sort(t.entries.begin(), t.entries.end(),
              [](uint16_t a, uint16_t b) { return (a & 0xFF) < (b & 0xFF); });
    uint16_t acc = 0;
    for (auto e : t.entries) {
        int v = (int)(int8_t)(uint8_t)(e & 0xFF) + 128;
        t.cum[v] = acc;
        acc = (uint16_t)(acc + (e >> 8));
    }
}

struct Enc {
    const int8_t *W;
    int rows, cols, qtot, seg_quads, nseg, stripes;
    bool local;
    const std::vector<Table> *tables;  // local: stripes*32 tables, else 1
};

// Encode one lane's segment; returns words in emission order and the state.
inline void encode_lane(const Enc &e, int row, int seg, std::vector<uint32_t> &words, uint64_t &state) {
    const Table &t = (*e.tables)[e.local ? row : 0];
    const int q0 = seg * e.seg_quads, nq = std::min(e.seg_quads, e.qtot - q0);
    const bool real = row < e.rows;
    const int8_t *wr = real ? e.W + (int64_t)row * e.cols : nullptr;
    uint64_t E = 0;
    words.clear();
    for (int i = nq - 1; i >= 0; i--) {
        uint32_t f[4], c[4];
        uint64_t P = 1;
        for (int j = 0; j < 4; j++) {
            int col = 4 * (q0 + i) + j;
            int v = (real && col < e.cols) ? wr[col] : t.pad_sym;
            f[j] = t.freq[v + 128];
            c[j] = t.cum[v + 128];
            P *= f[j];
        }
        if (E == 0) {
            E = P;
        } else if ((E >> 32) >= P) {
            words.push_back((uint32_t)E);
            E >>= 32;
        }
        uint64_t x = E / P, rem = E % P;
        uint32_t quants = 0;
        for (int j = 0; j < 4; j++) {
            uint32_t r = (uint32_t)(rem % f[j]);
            rem /= f[j];
            quants |= (c[j] + r) << (8 * j);
        }
        E = (x << 32) | quants;
    }
    state = E;
}

}  // namespace

static mv_status q8_encode(const int8_t *W, int rows, int cols, int local, int seg_quads,
                           int nthreads, Blob &out) {
    if (!W || rows <= 0 || cols <= 0) return fail(MV_ERR_ARG, "mv_q8_encode: bad arguments");
    Enc e{};
    e.W = W;
    e.rows = rows;
    e.cols = cols;
    e.qtot = (cols + 3) / 4;
    e.stripes = (rows + 31) / 32;
    e.local = local != 0;
    if (seg_quads <= 0 && e.stripes >= 64 && e.qtot > 64) {
        // enough stripes to fill the GPU with whole-stripe work items: segments of 32..64 quads (a multiple
        // of 4) that the 4 or 8 warps of a CTA share most evenly (a stripe ends in a CTA barrier, so its
        // slowest warp sets its time), with a small preference for longer segments (fewer coder states)
        double best = -1.0;
        for (int sq = 64; sq >= 32; sq -= 4) {
            const int n = (e.qtot + sq - 1) / sq, last = e.qtot - (n - 1) * sq;
            double eff = 1.0;
            for (int W : {4, 8}) {
                int worst = 0;
                for (int w = 0; w < W && w < n; w++) {
                    int work = 0;
                    for (int g = w; g < n; g += W) work += (g == n - 1) ? last : sq;
                    worst = std::max(worst, work);
                }
                eff = std::min(eff, (double)e.qtot / ((double)W * worst));
            }
            const double score = eff * (1.0 - 0.1 * 16.0 / sq);
            if (score > best + 1e-9) {
                best = score;
                seg_quads = sq;
            }
        }
    } else if (seg_quads <= 0) {
        // few stripes: segments of 32..64 quads (a multiple of 4), as many as it takes to give
        // 148 SMs x 16 warps at least one (stripe, segment) each
        int64_t want = (2368 + e.stripes - 1) / e.stripes;
        int64_t lo = (e.qtot + 63) / 64, hi = std::max(1, e.qtot / 32);
        int64_t nseg = std::max(lo, std::min(want, hi));
        nseg = std::max<int64_t>(1, std::min<int64_t>(nseg, e.qtot));
        seg_quads = (int)((e.qtot + nseg - 1) / nseg);
        if (seg_quads < e.qtot) seg_quads = (seg_quads + 3) & ~3;
    }
    e.seg_quads = std::min(seg_quads, e.qtot);
    e.nseg = (e.qtot + e.seg_quads - 1) / e.seg_quads;

    // tables
    std::vector<Table> tables;
    const int nthr = nthreads_or_default(nthreads);
    auto parallel = [&](int n, auto fn) {
        int nt = std::max(1, std::min(nthr, n));
        std::vector<std::thread> th;
        int per = (n + nt - 1) / nt;
        for (int t = 0; t < nt; t++) {
            int a = t * per, b = std::min(n, a + per);
            if (a < b) th.emplace_back([=, &fn]() { for (int i = a; i < b; i++) fn(i); });
        }
        for (auto &t : th) t.join();
    };
    if (e.local) {
        tables.resize((size_t)e.stripes * 32);
        parallel(e.stripes * 32, [&](int r) {
            int64_t counts[256] = {0};
            if (r < rows) {
                const int8_t *wr = W + (int64_t)r * cols;
                for (int c = 0; c < cols; c++) counts[(uint8_t)wr[c] ^ 0x80]++;
            }
            fit_table(counts, tables[r]);
            order_like_kernel(tables[r]);
        });
    } else {
        tables.resize(1);
        std::vector<int64_t> part((size_t)nthr * 256, 0);
        parallel(nthr, [&](int t) {
            int64_t a = (int64_t)rows * t / nthr, b = (int64_t)rows * (t + 1) / nthr;
            for (int64_t r = a; r < b; r++)
                for (int c = 0; c < cols; c++) part[(size_t)t * 256 + ((uint8_t)W[r * cols + c] ^ 0x80)]++;
        });
        int64_t counts[256] = {0};
        for (int t = 0; t < nthr; t++)
            for (int i = 0; i < 256; i++) counts[i] += part[(size_t)t * 256 + i];
        fit_table(counts, tables[0]);
        order_like_kernel(tables[0]);
    }
    e.tables = &tables;

    // blocks, one vector per stripe
    std::vector<std::vector<uint32_t>> stripe_words(e.stripes);
    std::vector<std::vector<uint32_t>> stripe_rows(e.stripes);  // word-rows per block
    parallel(e.stripes, [&](int s) {
        std::vector<uint32_t> words[32];
        uint64_t state[32];
        auto &out_w = stripe_words[s];
        auto &out_r = stripe_rows[s];
        for (int g = 0; g < e.nseg; g++) {
            size_t L = 0;
            for (int l = 0; l < 32; l++) {
                encode_lane(e, s * 32 + l, g, words[l], state[l]);
                L = std::max(L, words[l].size());
            }
            size_t base = out_w.size();
            out_w.resize(base + (2 + L) * 32, 0u);
            for (int l = 0; l < 32; l++) {
                out_w[base + l] = (uint32_t)state[l];
                out_w[base + 32 + l] = (uint32_t)(state[l] >> 32);
                const auto &w = words[l];
                for (size_t k = 0; k < w.size(); k++) out_w[base + (2 + k) * 32 + l] = w[w.size() - 1 - k];
            }
            out_r.push_back((uint32_t)(2 + L));
        }
    });
    std::vector<uint32_t> blk_off;
    blk_off.reserve((size_t)e.stripes * e.nseg + 1);
    size_t total_rows = 0;
    int max_rows = 2;
    for (int s = 0; s < e.stripes; s++)
        for (uint32_t r : stripe_rows[s]) {
            if (total_rows > 0xFFFFFFFFull) return fail(MV_ERR_SHAPE, "Q8 block offsets overflow");
            blk_off.push_back((uint32_t)total_rows);
            total_rows += r;
            max_rows = std::max<int>(max_rows, (int)r);
        }
    blk_off.push_back((uint32_t)total_rows);
    std::vector<uint32_t> blocks;
    blocks.reserve(total_rows * 32 + 32);
    for (int s = 0; s < e.stripes; s++) blocks.insert(blocks.end(), stripe_words[s].begin(), stripe_words[s].end());
    blocks.resize(blocks.size() + 32, 0u);  // one slack word-row after the last block

    std::vector<uint16_t> tbl;
    std::vector<uint32_t> tbl_off;
    for (auto &t : tables) {
        tbl_off.push_back((uint32_t)tbl.size());
        tbl.insert(tbl.end(), t.entries.begin(), t.entries.end());
    }
    tbl_off.push_back((uint32_t)tbl.size());
    uint32_t stripe_max = 0;
    if (e.local) {
        for (int s = 0; s < e.stripes; s++)
            stripe_max = std::max(stripe_max, tbl_off[(size_t)s * 32 + 32] - tbl_off[(size_t)s * 32]);
    } else {
        stripe_max = tbl_off[1] - tbl_off[0];
    }

    const int64_t payload = (int64_t)total_rows * 128 + (int64_t)tbl.size() * 2 +
                            (int64_t)tbl_off.size() * 4 + (int64_t)blk_off.size() * 4;
    out.put("blocks", blocks);
    out.shape("blocks", DT_U32, {(int64_t)blocks.size()});
    out.put("blk_off", blk_off);
    out.shape("blk_off", DT_U32, {(int64_t)blk_off.size()});
    out.put("tbl", tbl);
    out.shape("tbl", DT_U16, {(int64_t)tbl.size()});
    out.put("tbl_off", tbl_off);
    out.shape("tbl_off", DT_U32, {(int64_t)tbl_off.size()});
    out.set("rows", rows);
    out.set("cols", cols);
    out.set("seg_quads", e.seg_quads);
    out.set("nseg", e.nseg);
    out.set("local", e.local ? 1 : 0);
    out.set("max_blk_rows", max_rows);
    out.set("tbl_stripe_max", stripe_max);
    out.set("payload_bytes", payload);
    out.set("stream_bytes", (int64_t)total_rows * 128);
    return MV_OK;
}

}  // namespace mv

extern "C" mv_status mv_q8_encode(const int8_t *W, int rows, int cols, int local, int seg_quads,
                                  int nthreads, mv_blob **out) {
    if (!out) return mv::fail(MV_ERR_ARG, "mv_q8_encode: NULL out");
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "mv_q8_encode: out of memory");
    mv_status st = mv::q8_encode(W, rows, cols, local, seg_quads, nthreads, *b);
    if (st) { delete b; return st; }
    *out = b;
    return MV_OK;
}
