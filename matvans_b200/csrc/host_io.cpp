// File formats of the reference, read and written by the host library.
//
//  * safetensors, as written by buffered/encoder.py:473-511 and read by
//    buffered/sane_safetensors.hpp:17-68 + safetensor_loader.cpp:9-50: an
//    8-byte little-endian header length, a JSON object {name: {"dtype",
//    "shape", "data_offsets"}}, then the raw little-endian tensor bytes.
//    A small self-contained parser replaces the vendored safetensors-cpp.
//  * the matvansWarpPerRow .bin: create_matrices_WarpPerRow.py:290-319 and
//    :440-461, read like matvansWarpPerRow.cu:100-145 and :225-258.
#include <cctype>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "mv_internal.h"

namespace mv {
namespace {

bool read_file(const char *path, std::vector<uint8_t> &out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.seekg(0, std::ios::end);
    std::streamoff n = f.tellg();
    if (n < 0) return false;
    f.seekg(0, std::ios::beg);
    out.resize((size_t)n);
    if (n) f.read(reinterpret_cast<char *>(out.data()), n);
    return (bool)f;
}

struct Json {
    const char *p, *e;
    bool ok = true;
    void ws() { while (p < e && std::isspace((unsigned char)*p)) p++; }
    bool eat(char c) {
        ws();
        if (p < e && *p == c) { p++; return true; }
        return false;
    }
    std::string str() {
        ws();
        std::string s;
        if (p >= e || *p != '"') { ok = false; return s; }
        p++;
        while (p < e && *p != '"') {
            if (*p == '\\' && p + 1 < e) { p++; }
            s.push_back(*p++);
        }
        if (p >= e) { ok = false; return s; }
        p++;
        return s;
    }
    int64_t num() {
        ws();
        int64_t v = 0;
        bool neg = false, any = false;
        if (p < e && *p == '-') { neg = true; p++; }
        while (p < e && std::isdigit((unsigned char)*p)) { v = v * 10 + (*p - '0'); p++; any = true; }
        if (!any) ok = false;
        return neg ? -v : v;
    }
    // skip any JSON value (used for __metadata__)
    void skip() {
        ws();
        if (p >= e) { ok = false; return; }
        if (*p == '"') { str(); return; }
        if (*p == '{' || *p == '[') {
            char open = *p, close = open == '{' ? '}' : ']';
            int depth = 0;
            while (p < e) {
                if (*p == '"') { str(); continue; }
                if (*p == open) depth++;
                if (*p == close) { depth--; if (depth == 0) { p++; return; } }
                p++;
            }
            ok = false;
            return;
        }
        while (p < e && *p != ',' && *p != '}' && *p != ']') p++;
    }
};

int dtype_code(const std::string &s, int *size) {
    struct D { const char *n; int code, size; };
    static const D tab[] = {{"I8", DT_I8, 1},   {"U8", DT_U8, 1},   {"I16", DT_I16, 2}, {"U16", DT_U16, 2},
                            {"I32", DT_I32, 4}, {"U32", DT_U32, 4}, {"F32", DT_F32, 4}, {"I64", DT_I64, 8},
                            {"U64", DT_U64, 8}, {"F64", DT_F64, 8}};
    for (auto &d : tab)
        if (s == d.n) { *size = d.size; return d.code; }
    return 0;
}

const char *dtype_name(int code, int *size) {
    switch (code) {
        case DT_I8: *size = 1; return "I8";
        case DT_U8: *size = 1; return "U8";
        case DT_I16: *size = 2; return "I16";
        case DT_U16: *size = 2; return "U16";
        case DT_I32: *size = 4; return "I32";
        case DT_U32: *size = 4; return "U32";
        case DT_F32: *size = 4; return "F32";
        case DT_I64: *size = 8; return "I64";
        case DT_U64: *size = 8; return "U64";
        case DT_F64: *size = 8; return "F64";
    }
    return nullptr;
}

mv_status parse_safetensors(const std::vector<uint8_t> &blob, Blob &out) {
    if (blob.size() < 8) return fail(MV_ERR_FORMAT, "safetensors: file shorter than 8 bytes");
    uint64_t n = 0;
    for (int i = 0; i < 8; i++) n |= (uint64_t)blob[i] << (8 * i);
    if (n > blob.size() - 8) return fail(MV_ERR_FORMAT, "safetensors: header length %llu exceeds file",
                                         (unsigned long long)n);
    const uint64_t base = 8 + n;
    const uint64_t data_len = blob.size() - base;
    Json j{reinterpret_cast<const char *>(blob.data() + 8), reinterpret_cast<const char *>(blob.data() + 8 + n)};
    if (!j.eat('{')) return fail(MV_ERR_FORMAT, "safetensors: header is not a JSON object");
    bool first = true;
    while (true) {
        if (j.eat('}')) break;
        if (!first && !j.eat(',')) return fail(MV_ERR_FORMAT, "safetensors: expected ','");
        first = false;
        std::string name = j.str();
        if (!j.ok || !j.eat(':')) return fail(MV_ERR_FORMAT, "safetensors: bad key");
        if (name == "__metadata__") { j.skip(); if (!j.ok) return fail(MV_ERR_FORMAT, "safetensors: bad metadata"); continue; }
        if (!j.eat('{')) return fail(MV_ERR_FORMAT, "safetensors: tensor '%s' is not an object", name.c_str());
        std::string dtype;
        std::vector<int64_t> shape;
        int64_t off0 = -1, off1 = -1;
        bool f2 = true;
        while (true) {
            if (j.eat('}')) break;
            if (!f2 && !j.eat(',')) return fail(MV_ERR_FORMAT, "safetensors: expected ',' in '%s'", name.c_str());
            f2 = false;
            std::string key = j.str();
            if (!j.ok || !j.eat(':')) return fail(MV_ERR_FORMAT, "safetensors: bad field in '%s'", name.c_str());
            if (key == "dtype") dtype = j.str();
            else if (key == "shape" || key == "data_offsets") {
                if (!j.eat('[')) return fail(MV_ERR_FORMAT, "safetensors: '%s' not a list", key.c_str());
                std::vector<int64_t> v;
                if (!j.eat(']')) {
                    do { v.push_back(j.num()); } while (j.eat(','));
                    if (!j.eat(']')) return fail(MV_ERR_FORMAT, "safetensors: unterminated list");
                }
                if (key == "shape") shape = v;
                else if (v.size() == 2) { off0 = v[0]; off1 = v[1]; }
                else return fail(MV_ERR_FORMAT, "safetensors: data_offsets of '%s'", name.c_str());
            } else {
                j.skip();
            }
            if (!j.ok) return fail(MV_ERR_FORMAT, "safetensors: malformed JSON in '%s'", name.c_str());
        }
        int esize = 0;
        int code = dtype_code(dtype, &esize);
        if (!code) return fail(MV_ERR_FORMAT, "safetensors: unsupported dtype '%s'", dtype.c_str());
        int64_t numel = 1;
        for (auto d : shape) {
            if (d < 0) return fail(MV_ERR_FORMAT, "safetensors: negative dimension in '%s'", name.c_str());
            numel *= d;
        }
        if (off0 < 0 || off1 < off0 || (uint64_t)off1 > data_len)
            return fail(MV_ERR_FORMAT, "safetensors: data_offsets of '%s' out of range", name.c_str());
        if ((off1 - off0) != numel * esize)
            return fail(MV_ERR_FORMAT, "safetensors: size of '%s' does not match its shape", name.c_str());
        out.put_bytes(name, std::vector<uint8_t>(blob.begin() + base + off0, blob.begin() + base + off1));
        out.shape(name, code, shape);
    }
    return MV_OK;
}

template <class T>
T rd(const std::vector<uint8_t> &b, size_t &off, bool &ok) {
    T v{};
    if (off + sizeof(T) > b.size()) { ok = false; return v; }
    std::memcpy(&v, b.data() + off, sizeof(T));
    off += sizeof(T);
    return v;
}

}  // namespace
}  // namespace mv

extern "C" {

mv_status mv_read_safetensors(const char *path, mv_blob **out) {
    if (!path || !out) return mv::fail(MV_ERR_ARG, "mv_read_safetensors: NULL argument");
    std::vector<uint8_t> blob;
    if (!mv::read_file(path, blob)) return mv::fail(MV_ERR_IO, "cannot read '%s'", path);
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "out of memory");
    mv_status st = mv::parse_safetensors(blob, *b);
    if (st) { delete b; return st; }
    *out = b;
    return MV_OK;
}

mv_status mv_write_safetensors(const char *path, const mv_blob *b) {
    if (!path || !b) return mv::fail(MV_ERR_ARG, "mv_write_safetensors: NULL argument");
    std::ostringstream hdr;
    hdr << "{";
    uint64_t off = 0;
    bool first = true;
    for (const auto &name : b->order) {
        auto itd = b->scalars.find(name + ".dtype");
        auto itn = b->scalars.find(name + ".ndim");
        if (itd == b->scalars.end() || itn == b->scalars.end())
            return mv::fail(MV_ERR_ARG, "mv_write_safetensors: array '%s' has no dtype/shape", name.c_str());
        int esize = 0;
        const char *dn = mv::dtype_name((int)itd->second, &esize);
        if (!dn) return mv::fail(MV_ERR_ARG, "mv_write_safetensors: bad dtype for '%s'", name.c_str());
        const auto &bytes = b->arrays.at(name);
        if (!first) hdr << ",";
        first = false;
        hdr << "\"" << name << "\":{\"dtype\":\"" << dn << "\",\"shape\":[";
        for (int64_t i = 0; i < itn->second; i++) {
            auto its = b->scalars.find(name + ".shape" + std::to_string(i));
            if (its == b->scalars.end()) return mv::fail(MV_ERR_ARG, "missing shape of '%s'", name.c_str());
            hdr << (i ? "," : "") << its->second;
        }
        hdr << "],\"data_offsets\":[" << off << "," << off + bytes.size() << "]}";
        off += bytes.size();
    }
    hdr << "}";
    std::string h = hdr.str();
    while ((8 + h.size()) % 8) h.push_back(' ');  // align the data section
    std::ofstream f(path, std::ios::binary);
    if (!f) return mv::fail(MV_ERR_IO, "cannot write '%s'", path);
    uint64_t n = h.size();
    uint8_t len[8];
    for (int i = 0; i < 8; i++) len[i] = (uint8_t)(n >> (8 * i));
    f.write(reinterpret_cast<const char *>(len), 8);
    f.write(h.data(), (std::streamsize)h.size());
    for (const auto &name : b->order) {
        const auto &bytes = b->arrays.at(name);
        f.write(reinterpret_cast<const char *>(bytes.data()), (std::streamsize)bytes.size());
    }
    if (!f) return mv::fail(MV_ERR_IO, "write to '%s' failed", path);
    return MV_OK;
}

mv_status mv_read_wpr_bin(const char *path, mv_blob **out) {
    if (!path || !out) return mv::fail(MV_ERR_ARG, "mv_read_wpr_bin: NULL argument");
    std::vector<uint8_t> blob;
    if (!mv::read_file(path, blob)) return mv::fail(MV_ERR_IO, "cannot read '%s'", path);
    auto *b = new (std::nothrow) mv_blob;
    if (!b) return mv::fail(MV_ERR_NOMEM, "out of memory");
    size_t off = 0;
    bool ok = true;
    auto bad = [&](const char *what) {
        delete b;
        return mv::fail(MV_ERR_FORMAT, "%s: truncated or malformed .bin (%s at byte %zu)", path, what, off);
    };
    uint32_t num = mv::rd<uint32_t>(blob, off, ok);
    uint32_t hash = mv::rd<uint32_t>(blob, off, ok);
    uint32_t maxwc = mv::rd<uint32_t>(blob, off, ok);
    uint32_t len_v = mv::rd<uint32_t>(blob, off, ok);
    if (!ok || off + len_v > blob.size()) return bad("header");
    b->set("num_matrices", num);
    b->set("result_hash", hash);
    b->set("max_word_count", maxwc);
    b->set("len_v", len_v);
    b->put_bytes("vector", std::vector<uint8_t>(blob.begin() + off, blob.begin() + off + len_v));
    b->shape("vector", mv::DT_I8, {len_v});
    off += len_v + (3 - (len_v + 3) % 4);
    for (uint32_t m = 0; m < num; m++) {
        const std::string p = "m" + std::to_string(m) + ".";
        uint32_t rows = mv::rd<uint32_t>(blob, off, ok);
        uint32_t cols = mv::rd<uint32_t>(blob, off, ok);
        (void)mv::rd<float>(blob, off, ok);  // grid_spacing
        if (!ok || (uint64_t)rows * 4 > blob.size() - off) return bad("matrix header");
        std::vector<uint8_t> cursors(blob.begin() + off, blob.begin() + off + (size_t)rows * 4);
        off += (size_t)rows * 4;
        uint32_t payload_size = mv::rd<uint32_t>(blob, off, ok);
        int8_t min_value = mv::rd<int8_t>(blob, off, ok);
        uint8_t G = mv::rd<uint8_t>(blob, off, ok);
        const size_t cdf_len = (size_t)G + 1;
        if (!ok || off + cdf_len > blob.size()) return bad("cdf");
        std::vector<uint8_t> cdf(blob.begin() + off, blob.begin() + off + cdf_len);
        off += cdf_len + (cdf_len % 2);
        if (off + 256 > blob.size()) return bad("ppf");
        std::vector<uint8_t> ppf(blob.begin() + off, blob.begin() + off + 256);
        off += 256;
        if ((uint64_t)payload_size * 2 > blob.size() - off) return bad("payload");
        std::vector<uint8_t> payload(blob.begin() + off, blob.begin() + off + (size_t)payload_size * 2);
        off += (size_t)payload_size * 2 + (payload_size % 2 ? 2 : 0);
        b->put_bytes(p + "cursors", std::move(cursors));
        b->shape(p + "cursors", mv::DT_U32, {rows});
        b->put_bytes(p + "cdf", std::move(cdf));
        b->shape(p + "cdf", mv::DT_U8, {(int64_t)cdf_len});
        b->put_bytes(p + "ppf", std::move(ppf));
        b->shape(p + "ppf", mv::DT_U8, {256});
        b->put_bytes(p + "payload", std::move(payload));
        b->shape(p + "payload", mv::DT_U16, {payload_size});
        b->set(p + "rows", rows);
        b->set(p + "cols", cols);
        b->set(p + "min_value", min_value);
        b->set(p + "G", G);
        b->set(p + "payload_size", payload_size);
    }
    if (off > blob.size()) return bad("end");
    *out = b;
    return MV_OK;
}

}  // extern "C"
