// Error reporting, blobs and the vector hash (host side of the C ABI).
#include <cstdio>
#include <thread>

#include "mv_internal.h"

namespace mv {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

mv_status fail(mv_status code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

const char *last_error_cstr() { return g_last_error.c_str(); }

int nthreads_or_default(int n) {
    if (n > 0) return n;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

}  // namespace mv

extern "C" {

const char *mv_version(void) { return "matvans-b200 0.1 (sm_100a)"; }

const char *mv_last_error(void) { return mv::last_error_cstr(); }

void mv_blob_free(mv_blob *b) { delete b; }

mv_status mv_blob_get(const mv_blob *b, const char *name, const void **data, size_t *nbytes) {
    if (!b || !name || !data || !nbytes) return mv::fail(MV_ERR_ARG, "mv_blob_get: NULL argument");
    auto it = b->arrays.find(name);
    if (it == b->arrays.end()) return mv::fail(MV_ERR_ARG, "mv_blob_get: no array '%s'", name);
    *data = it->second.data();
    *nbytes = it->second.size();
    return MV_OK;
}

mv_status mv_blob_get_i64(const mv_blob *b, const char *name, int64_t *value) {
    if (!b || !name || !value) return mv::fail(MV_ERR_ARG, "mv_blob_get_i64: NULL argument");
    auto it = b->scalars.find(name);
    if (it == b->scalars.end()) return mv::fail(MV_ERR_ARG, "mv_blob_get_i64: no scalar '%s'", name);
    *value = it->second;
    return MV_OK;
}

const char *mv_blob_name(const mv_blob *b, int i) {
    if (!b || i < 0 || (size_t)i >= b->order.size()) return nullptr;
    return b->order[i].c_str();
}

// FxHash-style hash: buffered/encoder.py:8-20 (C++ twin ans-warp-rows.cu:62-73).
uint32_t mv_hash_int8(const int8_t *v, size_t n) {
    uint32_t h = 0;
    for (size_t i = 0; i < n; i++) {
        h = (h >> 27) | (h << 5);
        h = (h ^ (uint32_t)(uint8_t)v[i]) * 0x27220A95u;
    }
    return h;
}

}  // extern "C"
