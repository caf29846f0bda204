// common.cuh -- shared host/device utilities of libdetnqs_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "detnqs_gpu.h"

namespace dnq {

using u8 = uint8_t;
using u16 = uint16_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i64 = int64_t;

constexpr double kElemThresh = 1e-15;    // |H_ij| <= 1e-15 is dropped
constexpr double kAmpDelta = 1e-12;      // floor of |psi_i| in tau_i
constexpr u64 kEmptyKey = ~0ull;         // empty hash slot marker (alpha word)

// ---------------------------------------------------------------------------
// Errors: every C entry point converts exceptions to a status code and keeps
// the message for dnq_last_error().
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define DNQ_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t _e = (call);                                              \
        if (_e != cudaSuccess) {                                              \
            if (_e == cudaErrorMemoryAllocation) {                            \
                (void)cudaGetLastError();                                     \
                throw ::dnq::Error(DNQ_ERR_OUT_OF_MEMORY,                     \
                                   std::string("out of device memory at ") +  \
                                       #call);                                \
            }                                                                 \
            throw ::dnq::Error(DNQ_ERR_CUDA, std::string(#call) + ": " +      \
                                                 cudaGetErrorString(_e));     \
        }                                                                     \
    } while (0)

// Counts launches of this library's own kernels (every launch site is
// followed by DNQ_CHECK_LAUNCH); read with dnq_launch_count().
void count_launch();
#define DNQ_CHECK_LAUNCH()          \
    do {                            \
        ::dnq::count_launch();      \
        DNQ_CUDA(cudaGetLastError()); \
    } while (0)

#define DNQ_API_BEGIN try {
#define DNQ_API_END                                                           \
    return DNQ_OK;                                                            \
    }                                                                         \
    catch (const ::dnq::Error& e) {                                           \
        ::dnq::set_last_error(e.what());                                      \
        return e.code;                                                        \
    }                                                                         \
    catch (const std::bad_alloc&) {                                           \
        ::dnq::set_last_error("host allocation failed");                      \
        return DNQ_ERR_OUT_OF_MEMORY;                                         \
    }                                                                         \
    catch (const std::exception& e) {                                         \
        ::dnq::set_last_error(e.what());                                      \
        return DNQ_ERR_INVALID;                                               \
    }

inline void require(bool ok, int code, const std::string& msg) {
    if (!ok) throw Error(code, msg);
}

// ---------------------------------------------------------------------------
// Stream-ordered device buffers (cudaMallocAsync on the caller's stream).
// ---------------------------------------------------------------------------
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;

    DBuf() = default;
    DBuf(size_t count, cudaStream_t st) { alloc(count, st); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; s = o.s;
            o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }

    void alloc(size_t count, cudaStream_t st) {
        release();
        s = st;
        n = count;
        if (count) DNQ_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), st));
    }
    void release() noexcept {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
    T* get() const { return p; }
};

// ---------------------------------------------------------------------------
// Host/device pointer handling.  A pointer the CUDA runtime does not know is
// treated as pageable host memory.
// ---------------------------------------------------------------------------
inline bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Rejects device memory that belongs to a GPU other than `device` (managed
// memory is reachable from every GPU and passes).  Kernels of this library
// read caller buffers without peer access, so such a buffer would fault.
inline void require_on_device(const void* p, int device, const char* what) {
    if (!p) return;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    if (a.type == cudaMemoryTypeDevice && a.device != device)
        throw Error(DNQ_ERR_INVALID, std::string(what) + " is device memory of GPU " +
                                         std::to_string(a.device) + ", not of GPU " +
                                         std::to_string(device));
}

inline int current_device() {
    int d = 0;
    DNQ_CUDA(cudaGetDevice(&d));
    return d;
}

// Device view of caller data: either the caller's device pointer or a fresh
// device copy of a host buffer.  A device pointer must be memory of the
// current device.
template <class T>
struct DIn {
    const T* p = nullptr;
    DBuf<T> own;
    DIn() = default;
    DIn(const T* src, size_t count, cudaStream_t st) { set(src, count, st); }
    void set(const T* src, size_t count, cudaStream_t st) {
        if (!src || count == 0) { p = nullptr; return; }
        if (is_device_ptr(src)) {
            require_on_device(src, current_device(), "input buffer");
            p = src;
            return;
        }
        own.alloc(count, st);
        DNQ_CUDA(cudaMemcpyAsync(own.p, src, count * sizeof(T),
                                 cudaMemcpyHostToDevice, st));
        p = own.p;
    }
};

template <class T>
inline void copy_out(T* dst, const T* dsrc, size_t count, cudaStream_t st) {
    if (!dst || count == 0) return;
    DNQ_CUDA(cudaMemcpyAsync(dst, dsrc, count * sizeof(T), cudaMemcpyDefault, st));
}

// Library options (dnq_set_option).  The process-wide values are defaults:
// every handle, batch and server takes a copy when it is created and uses
// its own copy afterwards, so changing a default never reaches objects that
// exist already, and a handle's H.psi shape can be set on that handle alone.
struct Options {
    int force_walk = 0;        // V->V-only builds through the candidate walk
    long long arena_chunk = 0; // entries per warp chunk (0: default)
    long long arena_cap = 0;   // arena capacity (0: automatic)
    int partc_groupwalk = 0;   // part C short groups one at a time
    int build_f32 = 0;         // V->V builds write the FP32 copy while compacting
    int spmv_lanes = 0;        // H.psi lanes per row (0: by row length)
    int spmv_unroll = 0;       // H.psi slots per lane (0: by row length)
};
// A copy of the process-wide defaults (thread-safe).
Options default_options();
// Options for the handles the calling thread builds through dnq_build, in
// place of the defaults (a server's worker threads point it at the
// server's copy); null outside such threads.
extern thread_local const Options* g_build_opt;

inline int sm_count(int device) {
    int v = 0;
    DNQ_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    return v;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        DNQ_CUDA(cudaGetDevice(&prev));
        if (prev != dev) DNQ_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0)
            cudaSetDevice(prev);
    }
};

// N timing events, destroyed with the scope on every path (a failed check
// between their records throws); `make` false leaves them null.
template <int N>
struct Events {
    cudaEvent_t e[N] = {};
    explicit Events(bool make = true) {
        if (!make) return;
        try {
            for (auto& x : e) DNQ_CUDA(cudaEventCreate(&x));
        } catch (...) {
            release();
            throw;
        }
    }
    ~Events() { release(); }
    Events(const Events&) = delete;
    Events& operator=(const Events&) = delete;
    void release() {
        for (auto& x : e) {
            if (x) cudaEventDestroy(x);
            x = nullptr;
        }
    }
    cudaEvent_t operator[](int i) const { return e[i]; }
    cudaEvent_t* data() { return e; }
};

// ---------------------------------------------------------------------------
// Device bit helpers
// ---------------------------------------------------------------------------
__host__ __device__ inline u64 low_mask(int n) {
    return n <= 0 ? 0ull : (n >= 64 ? ~0ull : ((1ull << n) - 1ull));
}

// Number of occupied orbitals of `occ` strictly between positions x and y.
__device__ __forceinline__ int occ_between(u64 occ, int x, int y) {
    const int lo = min(x, y), hi = max(x, y);
    if (hi - lo <= 1) return 0;
    return __popcll(occ & low_mask(hi) & ~low_mask(lo + 1));
}

// Lane mask of lanes below the calling lane.
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 64-bit hash of a determinant key (murmur3 finaliser on a mixed word).
__host__ __device__ __forceinline__ u64 det_hash(u64 a, u64 b) {
    u64 x = a ^ (b * 0x9E3779B97F4A7C15ull) ^ (b >> 29);
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

}  // namespace dnq
