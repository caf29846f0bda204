// spmv.cuh -- device pieces shared by the H.psi kernels (spmv.cu, spmm.cu):
// the row accumulators (FP64 fused multiply-adds; FP32 Kahan summation),
// Dot2 for the FP64 energy sums (Ogita, Rump, Oishi, "Accurate sum and dot
// product", SIAM J. Sci. Comput. 26 (2005): TwoProduct with an fma
// residual + Knuth's TwoSum) and streaming 128-bit loads of the CSR.
#pragma once

#include "ham.cuh"

namespace dnq {
namespace {

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float z = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z));
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double z = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, z)), __dsub_rn(b, z));
}

// Accumulator of sum x_k*y_k with twice-working-precision behaviour.
template <class T>
struct Dot2 {
    T s = 0, c = 0;
    __device__ __forceinline__ void add_prod(T a, T b);
    __device__ __forceinline__ void add(T v) {
        T s2, e;
        two_sum(s, v, s2, e);
        s = s2;
        c += e;
    }
    __device__ __forceinline__ void merge(const Dot2& o) {
        T s2, e;
        two_sum(s, o.s, s2, e);
        s = s2;
        c = c + o.c + e;
    }
    __device__ __forceinline__ T value() const { return s + c; }
};

template <>
__device__ __forceinline__ void Dot2<float>::add_prod(float a, float b) {
    const float p = __fmul_rn(a, b);
    const float pe = fmaf(a, b, -p);
    float s2, e;
    two_sum(s, p, s2, e);
    s = s2;
    c = __fadd_rn(c, __fadd_rn(e, pe));
}

template <>
__device__ __forceinline__ void Dot2<double>::add_prod(double a, double b) {
    const double p = __dmul_rn(a, b);
    const double pe = fma(a, b, -p);
    double s2, e;
    two_sum(s, p, s2, e);
    s = s2;
    c = __dadd_rn(c, __dadd_rn(e, pe));
}

template <class T>
__device__ __forceinline__ Dot2<T> shfl_xor(const Dot2<T>& d, int o, unsigned mask) {
    Dot2<T> r;
    r.s = __shfl_xor_sync(mask, d.s, o);
    r.c = __shfl_xor_sync(mask, d.c, o);
    return r;
}

// Row accumulators: FP64 plain fused multiply-add, FP32 Dot2.
// reduce(G) combines the G lanes of a row group by a butterfly: at offset
// o = G/2, ..., 1 every lane merges with lane ^ o.  A merge is symmetric
// (a + b == b + a, and TwoSum's error term is exact whatever the order), so
// both lanes of a pair hold the same value after each step.  shfl(o) and
// merge(x) are the two halves of one step, for callers that exchange only
// part of their accumulators.
struct AccF64 {
    double s = 0.0;
    __device__ __forceinline__ void add_prod(double v, double x) { s = fma(v, x, s); }
    __device__ __forceinline__ void reduce(int G) {
        for (int o = G / 2; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    __device__ __forceinline__ AccF64 shfl(int o) const {
        AccF64 r;
        r.s = __shfl_xor_sync(0xffffffffu, s, o);
        return r;
    }
    __device__ __forceinline__ void merge(const AccF64& x) { s += x.s; }
    __device__ __forceinline__ double value() const { return s; }
};

// FP32 accumulator: Kahan's compensated summation of the products, each
// product entering through one fused multiply-add, y = v*x - c, with a
// single rounding (Kahan, "Further remarks on reducing truncation errors",
// CACM 8 (1965); the product needs no separate rounding).  (s, c) hold the
// sum as s - c.  Lanes merge their pairs with TwoSum: s1 + s2 = s + e
// exactly, so the merged pair is (s, (c1 + c2) - e), symmetric in its two
// arguments.
struct AccF32 {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add_prod(float v, float x) {
        const float y = fmaf(v, x, -c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ void merge(const AccF32& o) {
        float s2, e;
        two_sum(s, o.s, s2, e);
        s = s2;
        c = __fsub_rn(__fadd_rn(c, o.c), e);
    }
    __device__ __forceinline__ AccF32 shfl(int o) const {
        AccF32 r;
        r.s = __shfl_xor_sync(0xffffffffu, s, o);
        r.c = __shfl_xor_sync(0xffffffffu, c, o);
        return r;
    }
    __device__ __forceinline__ void reduce(int G) {
        for (int o = G / 2; o; o >>= 1) merge(shfl(o));
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Four consecutive values from a 16-byte aligned position, streamed past L1
// (the values are used once; L1 and L2 stay with x).
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void load4(const float* p, float (&v)[4]) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

}  // namespace
}  // namespace dnq
