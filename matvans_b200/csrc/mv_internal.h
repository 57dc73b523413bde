// Internal helpers shared by the host and device translation units.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "matvans.h"

namespace mv {

// Thread-local last error (mv_last_error).
void set_error(const char *fmt, ...);
mv_status fail(mv_status code, const char *fmt, ...);

// A blob: named byte arrays plus named int64 scalars.
struct Blob {
    std::vector<std::string> order;
    std::map<std::string, std::vector<uint8_t>> arrays;
    std::map<std::string, int64_t> scalars;

    template <class T>
    void put(const std::string &name, const std::vector<T> &v) {
        std::vector<uint8_t> bytes(v.size() * sizeof(T));
        if (!v.empty()) std::memcpy(bytes.data(), v.data(), bytes.size());
        put_bytes(name, std::move(bytes));
    }
    void put_bytes(const std::string &name, std::vector<uint8_t> &&bytes) {
        if (!arrays.count(name)) order.push_back(name);
        arrays[name] = std::move(bytes);
    }
    void set(const std::string &name, int64_t v) { scalars[name] = v; }
    // shape/dtype metadata used by the safetensors writer
    void shape(const std::string &name, int dtype, std::vector<int64_t> dims) {
        set(name + ".dtype", dtype);
        set(name + ".ndim", (int64_t)dims.size());
        for (size_t i = 0; i < dims.size(); i++) set(name + ".shape" + std::to_string(i), dims[i]);
    }
};

enum DType { DT_I8 = 1, DT_U8, DT_I16, DT_U16, DT_I32, DT_U32, DT_F32, DT_I64, DT_U64, DT_F64 };

int nthreads_or_default(int n);

}  // namespace mv

struct mv_blob : mv::Blob {};
