// dq_result.hpp -- result container shared by ref_shim.cpp and oracle.cpp.
// TEST INFRASTRUCTURE ONLY (see dq_api.h).
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace dq {

struct Coo {
    std::vector<uint32_t> rows, cols;
    std::vector<double> vals;
    uint32_t nr = 0, nc = 0;
};

struct Result {
    Coo a, b;                       // H_VV (or H_eff) and H_VP
    std::vector<uint64_t> dets;     // flattened (alpha, beta) pairs
    std::vector<int32_t> offsets;   // local connections row offsets
    std::vector<double> values;     // local connections values
};

inline thread_local std::string g_err;

inline int64_t res_size(Result* r, int which) {
    switch (which) {
        case 0: return (int64_t)r->a.vals.size();
        case 1: return (int64_t)r->b.vals.size();
        case 2: return (int64_t)(r->dets.size() / 2);
        case 3: return (int64_t)r->offsets.size();
        case 4: return (int64_t)r->values.size();
    }
    return -1;
}

inline void res_coo(Result* r, int which, uint32_t* rows, uint32_t* cols,
                    double* vals, uint32_t* shape2) {
    const Coo& c = which == 0 ? r->a : r->b;
    const size_t m = c.vals.size();
    if (m) {
        std::memcpy(rows, c.rows.data(), m * sizeof(uint32_t));
        std::memcpy(cols, c.cols.data(), m * sizeof(uint32_t));
        std::memcpy(vals, c.vals.data(), m * sizeof(double));
    }
    shape2[0] = c.nr;
    shape2[1] = c.nc;
}

}  // namespace dq

#define DQ_RESULT_ACCESSORS                                                   \
    extern "C" int64_t dq_res_size(void* r, int w) {                          \
        return dq::res_size((dq::Result*)r, w);                               \
    }                                                                         \
    extern "C" void dq_res_coo(void* r, int w, uint32_t* ro, uint32_t* co,    \
                               double* va, uint32_t* sh) {                    \
        dq::res_coo((dq::Result*)r, w, ro, co, va, sh);                       \
    }                                                                         \
    extern "C" void dq_res_dets(void* r, uint64_t* out) {                     \
        auto* p = (dq::Result*)r;                                             \
        if (!p->dets.empty())                                                 \
            std::memcpy(out, p->dets.data(), p->dets.size() * 8);             \
    }                                                                         \
    extern "C" void dq_res_offsets(void* r, int32_t* out) {                   \
        auto* p = (dq::Result*)r;                                             \
        if (!p->offsets.empty())                                              \
            std::memcpy(out, p->offsets.data(), p->offsets.size() * 4);       \
    }                                                                         \
    extern "C" void dq_res_values(void* r, double* out) {                     \
        auto* p = (dq::Result*)r;                                             \
        if (!p->values.empty())                                               \
            std::memcpy(out, p->values.data(), p->values.size() * 8);         \
    }                                                                         \
    extern "C" void dq_res_free(void* r) { delete (dq::Result*)r; }           \
    extern "C" const char* dq_last_error(void) { return dq::g_err.c_str(); }
