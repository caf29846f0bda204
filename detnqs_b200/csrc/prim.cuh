// prim.cuh -- device-wide primitives of the build path: prefix sums, stable
// LSD radix sort of (key, payload) pairs, stream compaction, segmented
// sums and the per-row column sort of a CSR block.
//
// They replace the library sorts and scans used before, with two choices
// made for this workload:
//   * the radix sort visits only the bits a key can use: a determinant
//     word holds n_orb bits, so a (alpha, beta) key of a 13-orbital system
//     takes 4 passes of 8 bits instead of 16, and a 30-orbital one 8;
//   * the row sort keeps a block per row in shared memory (bitonic network)
//     and sends only rows longer than a block holds through the global sort.
//
// Radix sort: per pass of 8 bits, k_radix_hist counts the digits of each
// tile of 2048 keys (warp-aggregated with __match_any_sync), the digit-major
// table of counts is prefix-summed, and k_radix_scatter ranks every key
// inside its tile -- each warp walks its 256 keys in 8 rounds of 32 in input
// order, a key's rank is the count of its digit in earlier rounds plus its
// lanes before it in the round, and warps are offset per digit -- and writes
// it at (digits below + same digit in earlier tiles + rank).  Equal digits
// keep their input order, so the passes compose into a stable sort.
//
// Scan: three phases over tiles of 2048 items (tile sums, one-block scan of
// the tile sums, tile scans from their offsets).  Every phase reads its
// items before it writes, so in == out is allowed.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace dnq {
namespace prim {
// Internal linkage: every translation unit that includes this header gets
// its own instances of the kernels.
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;   // 2048
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ unsigned lt_mask() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Block-wide exclusive scan of one value per thread (256 threads); returns
// the exclusive prefix and writes the block total to *total.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T block_exclusive(T v, T* total) {
    __shared__ T warp_tot[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        T t = lane < kWarps ? warp_tot[lane] : T(0);
        T ti = t;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        if (lane < kWarps) warp_tot[lane] = ti - t;   // exclusive per warp
        if (lane == kWarps - 1) *total = ti;
    }
    __syncthreads();
    const T r = warp_tot[w] + incl - v;
    __syncthreads();
    return r;
}

template <class Tin, class Tout>
__global__ void __launch_bounds__(kThreads) k_tile_sums(const Tin* in, i64 n, Tout* sums) {
    const i64 base = (i64)blockIdx.x * kTile;
    Tout v = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 p = base + (i64)i * kThreads + threadIdx.x;
        if (p < n) v += (Tout)in[p];
    }
    __shared__ Tout tot;
    block_exclusive<Tout>(v, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block: exclusive scan of m tile sums in place, chunk by chunk.
template <class T>
__global__ void __launch_bounds__(kThreads) k_scan_sums(T* sums, i64 m) {
    __shared__ T tot;
    T carry = 0;
    for (i64 c0 = 0; c0 < m; c0 += kThreads) {
        const i64 p = c0 + threadIdx.x;
        const T v = p < m ? sums[p] : T(0);
        const T e = block_exclusive<T>(v, &tot);
        if (p < m) sums[p] = carry + e;
        carry += tot;
        __syncthreads();
    }
}

// Each thread scans kItems consecutive items of its tile.
template <class Tin, class Tout, bool Inclusive>
__global__ void __launch_bounds__(kThreads) k_scan_tiles(const Tin* in, Tout* out, i64 n,
                                                         const Tout* tile_off) {
    const i64 base = (i64)blockIdx.x * kTile + (i64)threadIdx.x * kItems;
    Tout v[kItems];
    Tout sum = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 p = base + i;
        v[i] = p < n ? (Tout)in[p] : Tout(0);
        sum += v[i];
    }
    __shared__ Tout tot;
    Tout run = tile_off[blockIdx.x] + block_exclusive<Tout>(sum, &tot);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 p = base + i;
        if (Inclusive) run += v[i];
        if (p < n) out[p] = run;
        if (!Inclusive) run += v[i];
    }
}

inline i64 tiles_of(i64 n) { return (n + kTile - 1) / kTile; }

// Temporary bytes of a scan of n items with Tout sums.
template <class Tout>
inline size_t scan_tmp_bytes(i64 n) {
    return (size_t)std::max<i64>(1, tiles_of(n)) * sizeof(Tout);
}

// out[i] = sum of in[0..i) (exclusive) or in[0..i] (inclusive).  tmp: at
// least scan_tmp_bytes<Tout>(n) bytes, or null to allocate it on s.
template <class Tin, class Tout, bool Inclusive = false>
void scan(const Tin* in, Tout* out, i64 n, cudaStream_t s, void* tmp = nullptr) {
    if (n <= 0) return;
    const i64 nt = tiles_of(n);
    DBuf<Tout> own;
    Tout* sums = static_cast<Tout*>(tmp);
    if (!sums) {
        own.alloc(nt, s);
        sums = own.p;
    }
    k_tile_sums<Tin, Tout><<<(unsigned)nt, kThreads, 0, s>>>(in, n, sums);
    DNQ_CHECK_LAUNCH();
    k_scan_sums<Tout><<<1, kThreads, 0, s>>>(sums, nt);
    DNQ_CHECK_LAUNCH();
    k_scan_tiles<Tin, Tout, Inclusive><<<(unsigned)nt, kThreads, 0, s>>>(in, out, n, sums);
    DNQ_CHECK_LAUNCH();
}

template <class Tin, class Tout>
void scan_inclusive(const Tin* in, Tout* out, i64 n, cudaStream_t s, void* tmp = nullptr) {
    scan<Tin, Tout, true>(in, out, n, s, tmp);
}

// ---------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------

// Words of a key, most significant first.
template <class K>
struct RadixKey;

template <>
struct RadixKey<u32> {
    static constexpr int W = 1;
    __device__ __forceinline__ static u64 word(const u32& k, int) { return k; }
};
template <>
struct RadixKey<u64> {
    static constexpr int W = 1;
    __device__ __forceinline__ static u64 word(const u64& k, int) { return k; }
};
// (alpha, beta) determinant keys: alpha word first.
template <>
struct RadixKey<ulonglong2> {
    static constexpr int W = 2;
    __device__ __forceinline__ static u64 word(const ulonglong2& k, int i) {
        return i == 0 ? k.x : k.y;
    }
};

template <class K>
__device__ __forceinline__ u32 digit_of(const K& k, int word, int shift) {
    return (u32)(RadixKey<K>::word(k, word) >> shift) & 0xffu;
}

template <class K>
__global__ void __launch_bounds__(kThreads) k_radix_hist(const K* keys, i64 n, int word,
                                                         int shift, u32* hist, i64 ntiles) {
    __shared__ u32 h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * kTile;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 p = base + (i64)i * kThreads + threadIdx.x;
        const bool ok = p < n;
        const u32 d = ok ? digit_of(keys[p], word, shift) : 256u;
        const unsigned m = __match_any_sync(0xffffffffu, d);
        if (ok && (m & lt_mask()) == 0) atomicAdd(&h[d], (u32)__popc(m));
    }
    __syncthreads();
    hist[(i64)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Payload pass-through: P* may be null on output (keys only); a null input
// with an output gives the input positions (P = u32).
template <class K, class P>
__global__ void __launch_bounds__(kThreads)
k_radix_scatter(const K* kin, const P* pin, K* kout, P* pout, i64 n, int word, int shift,
                const u32* offs, i64 ntiles) {
    __shared__ u32 wh[kWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kWarps * 256; t += kThreads) (&wh[0][0])[t] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * kTile + (i64)w * (kItems * 32);
    K k[kItems];
    P pl[kItems];
    u32 dg[kItems], rk[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 p = base + (i64)i * 32 + lane;
        const bool ok = p < n;
        dg[i] = 256u;
        if (ok) {
            k[i] = kin[p];
            if (pout) pl[i] = pin ? pin[p] : (P)p;
            dg[i] = digit_of(k[i], word, shift);
        }
        const unsigned m = __match_any_sync(0xffffffffu, dg[i]);
        const u32 before = ok ? wh[w][dg[i]] : 0u;
        rk[i] = before + __popc(m & lt_mask());
        __syncwarp();
        if (ok && (m & lt_mask()) == 0) wh[w][dg[i]] = before + __popc(m);
        __syncwarp();
    }
    __syncthreads();
    {   // per digit: warps' counts -> exclusive offsets
        const int d = threadIdx.x;
        u32 acc = 0;
#pragma unroll
        for (int q = 0; q < kWarps; ++q) {
            const u32 t = wh[q][d];
            wh[q][d] = acc;
            acc += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (dg[i] < 256u) {
            const u32 pos = offs[(i64)dg[i] * ntiles + blockIdx.x] + wh[w][dg[i]] + rk[i];
            kout[pos] = k[i];
            if (pout) pout[pos] = pl[i];
        }
    }
}

template <class K, class P>
__global__ void k_copy_pairs(const K* kin, const P* pin, K* kout, P* pout, i64 n) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        kout[t] = kin[t];
        if (pout) pout[t] = pin ? pin[t] : (P)t;
    }
}

// Stable sort of n (key, payload) pairs by key, ascending; n < 2^32.
// bits[i] = significant low bits of key word i (most significant word
// first; the other bits of the word must be zero, or at least equal in all
// keys).  pout == null sorts keys only; pin == null with a payload output
// gives each key's input position.  kin != kout.
template <class K, class P>
void radix_sort(const K* kin, K* kout, const P* pin, P* pout, i64 n, const int* bits,
                cudaStream_t s) {
    if (n <= 0) return;
    require(n < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "radix sort of 2^32 or more keys");
    constexpr int W = RadixKey<K>::W;
    int pw[16 * W], ps[16 * W], np = 0;
    for (int i = W - 1; i >= 0; --i)      // least significant word first
        for (int sh = 0; sh < bits[i]; sh += 8) {
            pw[np] = i;
            ps[np] = sh;
            ++np;
        }
    const unsigned grid_copy = (unsigned)std::min<i64>((n + 255) / 256, 4096);
    if (np == 0) {
        k_copy_pairs<K, P><<<grid_copy, 256, 0, s>>>(kin, pin, kout, pout, n);
        DNQ_CHECK_LAUNCH();
        return;
    }
    const i64 nt = tiles_of(n);
    DBuf<K> kt(np > 1 ? n : 0, s);
    DBuf<P> pt((np > 1 && pout) ? n : 0, s);
    DBuf<u32> hist(256 * nt, s);
    DBuf<u32> stmp(tiles_of(256 * nt), s);
    const K* ksrc = kin;
    const P* psrc = pin;
    for (int q = 0; q < np; ++q) {
        const bool to_out = ((np - 1 - q) & 1) == 0;
        K* kdst = to_out ? kout : kt.p;
        P* pdst = pout ? (to_out ? pout : pt.p) : nullptr;
        k_radix_hist<K><<<(unsigned)nt, kThreads, 0, s>>>(ksrc, n, pw[q], ps[q], hist.p, nt);
        DNQ_CHECK_LAUNCH();
        scan<u32, u32, false>(hist.p, hist.p, 256 * nt, s, stmp.p);
        k_radix_scatter<K, P><<<(unsigned)nt, kThreads, 0, s>>>(ksrc, psrc, kdst, pdst, n,
                                                                pw[q], ps[q], hist.p, nt);
        DNQ_CHECK_LAUNCH();
        ksrc = kdst;
        psrc = pdst;
    }
}

// ---------------------------------------------------------------------------
// Compaction and segmented sums
// ---------------------------------------------------------------------------

template <class F>
__global__ void k_flag_u32(const F* flag, i64 n, u32* f) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        f[t] = flag[t] != F(0) ? 1u : 0u;
}

template <class T>
__global__ void k_select_scatter(const T* in, const u32* flag, const u32* pos, i64 n, T* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        if (flag[t]) out[pos[t]] = in[t];
}

// out = the in[t] with flag[t] != 0, in order; returns their count.
template <class T, class F>
i64 select_flagged(const T* in, const F* flag, T* out, i64 n, cudaStream_t s) {
    if (n <= 0) return 0;
    DBuf<u32> f(n, s), pos(n, s);
    const unsigned g = (unsigned)std::min<i64>((n + 255) / 256, 4096);
    k_flag_u32<F><<<g, 256, 0, s>>>(flag, n, f.p);
    DNQ_CHECK_LAUNCH();
    scan<u32, u32, false>(f.p, pos.p, n, s);
    k_select_scatter<T><<<g, 256, 0, s>>>(in, f.p, pos.p, n, out);
    DNQ_CHECK_LAUNCH();
    u32 lp = 0, lf = 0;
    DNQ_CUDA(cudaMemcpyAsync(&lp, pos.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&lf, f.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    return (i64)lp + lf;
}

// out[i] = sum of v[t] over segment i = [rp[i], rp[i+1]) for integer v
// (order-free sums).  One warp per segment, lanes strided, then a butterfly;
// a segment longer than kSegWarp is listed instead (its sum set to 0) and
// summed by the whole grid in k_segment_sums_long.
constexpr i64 kSegWarp = 1 << 16;

template <class T, class Tout>
__global__ void k_segment_sums(const T* v, const i64* rp, i64 nseg, Tout* out, u32* longs,
                               u32* nlong) {
    const i64 w = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 i = w; i < nseg; i += nw) {
        const i64 b = rp[i], e = rp[i + 1];
        if (e - b > kSegWarp) {
            if (lane == 0) {
                out[i] = 0;
                longs[atomicAdd(nlong, 1u)] = (u32)i;
            }
            continue;
        }
        Tout a = 0;
        for (i64 t = b + lane; t < e; t += 32) a += (Tout)v[t];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) out[i] = a;
    }
}

template <class T, class Tout>
__global__ void k_segment_sums_long(const T* v, const i64* rp, const u32* longs,
                                    const u32* nlong, Tout* out) {
    static_assert(sizeof(Tout) == 8, "64-bit sums");
    const u32 n = *nlong;
    for (u32 q = 0; q < n; ++q) {
        const u32 i = longs[q];
        Tout a = 0;
        for (i64 t = rp[i] + blockIdx.x * (i64)blockDim.x + threadIdx.x; t < rp[i + 1];
             t += (i64)gridDim.x * blockDim.x)
            a += (Tout)v[t];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0 && a)
            atomicAdd(reinterpret_cast<unsigned long long*>(&out[i]), (unsigned long long)a);
    }
}

// out[0..nseg) = the integer sums of v over the segments of rp (64-bit out).
template <class T, class Tout>
void segment_sums(const T* v, const i64* rp, i64 nseg, Tout* out, cudaStream_t s) {
    if (nseg <= 0) return;
    DBuf<u32> longs(nseg, s), nlong(1, s);
    DNQ_CUDA(cudaMemsetAsync(nlong.p, 0, 4, s));
    const unsigned g = (unsigned)std::min<i64>((nseg * 32 + 255) / 256, 8192);
    k_segment_sums<T, Tout><<<g, 256, 0, s>>>(v, rp, nseg, out, longs.p, nlong.p);
    DNQ_CHECK_LAUNCH();
    k_segment_sums_long<T, Tout><<<1184, 256, 0, s>>>(v, rp, longs.p, nlong.p, out);
    DNQ_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Column sort of every row of a CSR block (columns of a row are distinct)
// ---------------------------------------------------------------------------

constexpr i64 kRowSortSmall = 256;     // one block of 256 threads, one entry each
constexpr i64 kRowSortMid = 4096;      // one block, 16 entries per thread
// Longer rows go through the global radix sort.

// Rows by length class: 0 = at most 1 entry (copied), 1 = small, 2 = mid,
// 3 = long.  lists: 4 x nr row ids; counts: 4.
__global__ void k_row_classes(const i64* rp, i64 nr, u32* lists, u32* counts) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nr;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 len = rp[r + 1] - rp[r];
        const int c = len <= 1 ? 0 : len <= kRowSortSmall ? 1 : len <= kRowSortMid ? 2 : 3;
        const u32 at = atomicAdd(&counts[c], 1u);
        lists[(i64)c * nr + at] = (u32)r;
    }
}

__global__ void k_row_copy(const u32* rows, const u32* cnt, const i64* rp, const u32* cin,
                           const double* vin, u32* cout, double* vout) {
    const u32 n = *cnt;
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const u32 r = rows[t];
        for (i64 k = rp[r]; k < rp[r + 1]; ++k) {
            cout[k] = cin[k];
            vout[k] = vin[k];
        }
    }
}

// One block per listed row: (column, position) pairs of the row sorted by a
// bitonic network over N = CAP slots in shared memory (padding: column
// 0xffffffff), then columns and the values they carry written in order.
template <int CAP>
__global__ void __launch_bounds__(256)
k_row_sort(const u32* rows, const u32* cnt, const i64* rp, const u32* cin, const double* vin,
           u32* cout, double* vout) {
    __shared__ u32 key[CAP];
    __shared__ u16 pos[CAP];
    const u32 n = *cnt;
    for (u32 b = blockIdx.x; b < n; b += gridDim.x) {
        const u32 r = rows[b];
        const i64 lo = rp[r];
        const int len = (int)(rp[r + 1] - lo);
        int N = 2;
        while (N < len) N <<= 1;
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            key[i] = i < len ? cin[lo + i] : 0xffffffffu;
            pos[i] = (u16)i;
        }
        __syncthreads();
        for (int k = 2; k <= N; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < N; i += blockDim.x) {
                    const int l = i ^ j;
                    if (l > i) {
                        const bool up = (i & k) == 0;
                        const u32 a = key[i], c = key[l];
                        if ((a > c) == up) {
                            key[i] = c;
                            key[l] = a;
                            const u16 t = pos[i];
                            pos[i] = pos[l];
                            pos[l] = t;
                        }
                    }
                }
                __syncthreads();
            }
        for (int i = threadIdx.x; i < len; i += blockDim.x) {
            cout[lo + i] = key[i];
            vout[lo + i] = vin[lo + pos[i]];
        }
        __syncthreads();
    }
}

// Long rows: key = (place of the row in the long list) << 32 | column.  The
// whole grid strides over each long row in turn (a row can hold millions of
// entries).
__global__ void k_long_row_keys(const u32* rows, u32 nlong, const i64* rp, const i64* base,
                                const u32* cin, u64* key, u32* src) {
    for (u32 q = 0; q < nlong; ++q) {
        const u32 r = rows[q];
        const i64 lo = rp[r], len = rp[r + 1] - lo, b = base[q];
        for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < len;
             t += (i64)gridDim.x * blockDim.x) {
            key[b + t] = ((u64)q << 32) | cin[lo + t];
            src[b + t] = (u32)(lo + t);
        }
    }
}

__global__ void k_long_row_put(const u32* rows, u32 nlong, const i64* rp, const i64* base,
                               const u64* skey, const u32* src, const double* vin, u32* cout,
                               double* vout) {
    for (u32 q = 0; q < nlong; ++q) {
        const u32 r = rows[q];
        const i64 lo = rp[r], len = rp[r + 1] - lo, b = base[q];
        for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < len;
             t += (i64)gridDim.x * blockDim.x) {
            cout[lo + t] = (u32)skey[b + t];
            vout[lo + t] = vin[src[b + t]];
        }
    }
}

__global__ void k_long_row_lens(const u32* rows, u32 nlong, const i64* rp, i64* len) {
    for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q < nlong; q += gridDim.x * blockDim.x)
        len[q] = rp[rows[q] + 1] - rp[rows[q]];
}

// cout/vout = every row of (rp, cin, vin) sorted by column.
inline void sort_row_columns(const i64* rp, i64 nr, const u32* cin, const double* vin, u32* cout,
                             double* vout, cudaStream_t s) {
    if (nr <= 0) return;
    require(nr < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "row sort of 2^32 or more rows");
    DBuf<u32> lists(4 * nr, s), counts(4, s);
    DNQ_CUDA(cudaMemsetAsync(counts.p, 0, 4 * sizeof(u32), s));
    const unsigned g = (unsigned)std::min<i64>((nr + 255) / 256, 4096);
    k_row_classes<<<g, 256, 0, s>>>(rp, nr, lists.p, counts.p);
    DNQ_CHECK_LAUNCH();
    u32 c[4];
    DNQ_CUDA(cudaMemcpyAsync(c, counts.p, sizeof(c), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    if (c[0]) {
        k_row_copy<<<(unsigned)std::min<u32>((c[0] + 255) / 256, 4096u), 256, 0, s>>>(
            lists.p, counts.p, rp, cin, vin, cout, vout);
        DNQ_CHECK_LAUNCH();
    }
    if (c[1]) {
        k_row_sort<(int)kRowSortSmall><<<(unsigned)std::min<u32>(c[1], 1u << 20), 256, 0, s>>>(
            lists.p + nr, counts.p + 1, rp, cin, vin, cout, vout);
        DNQ_CHECK_LAUNCH();
    }
    if (c[2]) {
        k_row_sort<(int)kRowSortMid><<<(unsigned)std::min<u32>(c[2], 1u << 20), 256, 0, s>>>(
            lists.p + 2 * nr, counts.p + 2, rp, cin, vin, cout, vout);
        DNQ_CHECK_LAUNCH();
    }
    if (c[3]) {
        const u32 nl = c[3];
        const u32* rows = lists.p + 3 * nr;
        DBuf<i64> len(nl + 1, s), base(nl + 1, s);
        k_long_row_lens<<<(unsigned)std::min<u32>((nl + 255) / 256, 4096u), 256, 0, s>>>(
            rows, nl, rp, len.p);
        DNQ_CHECK_LAUNCH();
        DNQ_CUDA(cudaMemsetAsync(len.p + nl, 0, sizeof(i64), s));
        scan<i64, i64, false>(len.p, base.p, nl + 1, s);
        i64 m = 0;
        DNQ_CUDA(cudaMemcpyAsync(&m, base.p + nl, sizeof(i64), cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        DBuf<u64> key(m, s), skey(m, s);
        DBuf<u32> src(m, s), ssrc(m, s);
        const unsigned gl = (unsigned)std::min<i64>((m + 255) / 256, 4096);
        k_long_row_keys<<<gl, 256, 0, s>>>(rows, nl, rp, base.p, cin, key.p, src.p);
        DNQ_CHECK_LAUNCH();
        int hb = 32;
        while (hb < 64 && ((u64)1 << (hb - 32)) < (u64)nl) ++hb;
        const int bits[1] = {hb};
        radix_sort<u64, u32>(key.p, skey.p, src.p, ssrc.p, m, bits, s);
        k_long_row_put<<<gl, 256, 0, s>>>(rows, nl, rp, base.p, skey.p, ssrc.p, vin, cout,
                                          vout);
        DNQ_CHECK_LAUNCH();
    }
}

}  // namespace
}  // namespace prim
}  // namespace dnq
