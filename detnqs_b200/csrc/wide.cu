// wide.cu -- screened build for determinants of up to 128 orbitals.
//
// The reference stores a spin string in one uint64 (det.hpp:30-36) and
// stops at 64 orbitals (integral_mo.cpp:26-28).  This file carries the same
// build -- singles and heat-bath doubles of every row of V, Slater-Condon
// elements in the reference's summation order (ham_eval.cpp:33-147), static
// or dynamic amplitude screening (build_ham.cpp:139-196), routing to V or to
// the discovered external space P in lexicographic order
// (build_ham.cpp:346-380) -- over two-word spin strings:
//
//   determinant = 4 x uint64: alpha lo, alpha hi, beta lo, beta hi
//   order       = alpha as a 128-bit integer, then beta
//
// Steps: a hash of V (32-byte keys, open addressing); warp-per-row count
// pass; exact CSR offsets; fill pass (survivors compacted with ballots in
// candidate order); per-row column sort of H_VV; 256-bit radix sort of the
// P keys, run-length unique, column relabelling; per-row sort of H_VP.  The
// result is an ordinary dnq_ham_t (words = 2), so H.psi, the proxy operator,
// downfolding and copies work on it unchanged.

#include <memory>
#include <vector>

#include "context.cuh"
#include "ham.cuh"
#include "prim.cuh"

namespace dnq {
void keep_pool(int device);

namespace {

constexpr int kWW = 8;                     // warps per block
constexpr u32 kEmpty = 0xffffffffu;

struct M2 {
    u64 lo, hi;
};

__device__ __forceinline__ bool bit(const M2& m, int i) {
    return i < 64 ? (m.lo >> i) & 1 : (m.hi >> (i - 64)) & 1;
}
__device__ __forceinline__ void flip(M2& m, int i) {
    if (i < 64) m.lo ^= 1ull << i;
    else m.hi ^= 1ull << (i - 64);
}
// bits [0, k) of a 128-bit string
__device__ __forceinline__ M2 mask_below(int k) {
    M2 r;
    r.lo = k >= 64 ? ~0ull : (k <= 0 ? 0ull : (1ull << k) - 1);
    r.hi = k >= 128 ? ~0ull : (k <= 64 ? 0ull : (1ull << (k - 64)) - 1);
    return r;
}
// occupied orbitals strictly between x and y (det_ops.cpp:85-93)
__device__ __forceinline__ int between2(const M2& m, int x, int y) {
    if (x == y) return 0;
    const int lo = min(x, y), hi = max(x, y);
    const M2 a = mask_below(hi), b = mask_below(lo + 1);
    return __popcll(m.lo & a.lo & ~b.lo) + __popcll(m.hi & a.hi & ~b.hi);
}

struct WRow {
    M2 a, b;
    int na, nb, nva, nvb, ne;
    u8 occ[256];
    u8 occa[128], occb[128], vira[128], virb[128];
};

__device__ __forceinline__ void load_wrow(WRow& R, M2 a, M2 b, int n_orb) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        R.a = a;
        R.b = b;
        int k = 0, t = 0;
        for (int o = 0; o < n_orb; ++o)
            if (bit(a, o)) { R.occa[t++] = (u8)o; R.occ[k++] = (u8)(2 * o); }
        R.na = t;
        t = 0;
        for (int o = 0; o < n_orb; ++o)
            if (bit(b, o)) { R.occb[t++] = (u8)o; R.occ[k++] = (u8)(2 * o + 1); }
        R.nb = t;
        R.ne = k;
        t = 0;
        for (int o = 0; o < n_orb; ++o)
            if (!bit(a, o)) R.vira[t++] = (u8)o;
        R.nva = t;
        t = 0;
        for (int o = 0; o < n_orb; ++o)
            if (!bit(b, o)) R.virb[t++] = (u8)o;
        R.nvb = t;
    }
    __syncwarp();
}

// ham_eval.cpp:53-86, serial per thread: one-body over alpha then beta
// occupied orbitals, then sum_{x>y} of the pair terms.
__device__ double diag2(const CtxView& C, const M2& a, const M2& b) {
    const int n = C.n;
    u8 occ[256];
    int m = 0;
    for (int o = 0; o < n; ++o)
        if (bit(a, o)) occ[m++] = (u8)(2 * o);
    for (int o = 0; o < n; ++o)
        if (bit(b, o)) occ[m++] = (u8)(2 * o + 1);
    double one = 0.0;
    for (int t = 0; t < m; ++t) {
        const int p = occ[t] >> 1;
        one += C.h1[p * n + p];
    }
    double two = 0.0;
    for (int x = 1; x < m; ++x) {
        const int P = occ[x];
        const double* dss = C.dss + (P >> 1) * n;
        const double* dos = C.dos + (P >> 1) * n;
        for (int y = 0; y < x; ++y) {
            const int Q = occ[y];
            two += ((P ^ Q) & 1) ? dos[Q >> 1] : dss[Q >> 1];
        }
    }
    return one + two;
}

// Single h -> p in spin s (ham_eval.cpp:88-115): h1 first, then the other
// occupied orbitals, alpha ascending then beta ascending.
// e + arr[occ[t]] for t = 0..cnt-1 except occ[t] == skip, added in t order;
// the loads are issued eight at a time ahead of their additions.
__device__ __forceinline__ double add_occ(double e, const double* arr, const u8* occ, int cnt,
                                          int skip) {
    int t = 0;
    for (; t + 8 <= cnt; t += 8) {
        double v[8];
        int o[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            o[q] = occ[t + q];
            v[q] = __ldg(&arr[o[q]]);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (o[q] != skip) e += v[q];
    }
    for (; t < cnt; ++t)
        if (occ[t] != skip) e += arr[occ[t]];
    return e;
}

__device__ __forceinline__ double single2(const CtxView& C, const WRow& R, int s, int h, int p) {
    const int n = C.n;
    double e = C.h1[h * n + p];
    const size_t base = ((size_t)h * n + p) * n;
    const double* ss = C.sss + base;
    const double* os = C.sos + base;
    if (s == 0) {
        e = add_occ(e, ss, R.occa, R.na, h);
        e = add_occ(e, os, R.occb, R.nb, -1);
    } else {
        e = add_occ(e, os, R.occa, R.na, -1);
        e = add_occ(e, ss, R.occb, R.nb, h);
    }
    const int perm = between2(s ? R.b : R.a, h, p);
    return (perm & 1) ? -e : e;
}

// Double i,j -> a,b (spin-orbitals, i > j, a > b) from v = <ij||ab>, with
// the phase of det_ops.cpp:101-127.
__device__ __forceinline__ double double2(const M2& ba, const M2& bb, int i, int j, int a, int b,
                                          double v) {
    const bool same = ((i ^ j) & 1) == 0;
    const double raw = (same || ((a ^ i) & 1) == 0) ? v : -v;
    int perm;
    if (same) {
        const M2& occ = (i & 1) ? bb : ba;
        const int h0 = b >> 1, h1 = a >> 1;
        const int p0 = j >> 1, p1 = i >> 1;
        perm = between2(occ, h0, p0) + between2(occ, h1, p1);
        const int A = min(h0, p0), B = max(h0, p0), Cc = min(h1, p1), D = max(h1, p1);
        if ((Cc > A && Cc < B && D > B) || (A > Cc && A < D && B > D)) ++perm;
    } else {
        const int ha = ((a & 1) == 0 ? a : b) >> 1;
        const int hb = ((a & 1) == 1 ? a : b) >> 1;
        const int pa = ((i & 1) == 0 ? i : j) >> 1;
        const int pb = ((i & 1) == 1 ? i : j) >> 1;
        perm = between2(ba, ha, pa) + between2(bb, hb, pb);
    }
    return (perm & 1) ? -raw : raw;
}

__device__ __forceinline__ i64 prefix_len(const double* v, i64 len, double cut) {
    if (cut <= 0.0 || len == 0) return len;
    const int lane = threadIdx.x & 31;
    i64 lo = 0, hi = len;
    while (hi - lo > 32) {
        const i64 step = (hi - lo + 31) / 32;
        const i64 x = lo + lane * step;
        const bool ok = x < hi && fabs(v[x]) >= cut;
        const int k = __popc(__ballot_sync(0xffffffffu, ok));
        if (k == 0) return lo;
        const i64 nlo = lo + (i64)(k - 1) * step + 1;
        const i64 nhi = min(hi, lo + (i64)k * step);
        lo = nlo;
        hi = nhi;
    }
    const i64 x = lo + lane;
    const bool ok = x < hi && fabs(v[x]) >= cut;
    return lo + __popc(__ballot_sync(0xffffffffu, ok));
}

__device__ __forceinline__ u64 mix(u64 x) {
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 29;
    return x;
}
__device__ __forceinline__ u64 hash4(const M2& a, const M2& b) {
    return mix(a.lo * 0x9E3779B97F4A7C15ull ^ mix(a.hi + 0x632BE59BD9B4E019ull) ^
               mix(b.lo * 0x94D049BB133111EBull) ^ (b.hi + 0xD6E8FEB86659FD93ull));
}
__device__ __forceinline__ bool eq4(const u64* d, const M2& a, const M2& b) {
    return d[0] == a.lo && d[1] == a.hi && d[2] == b.lo && d[3] == b.hi;
}

struct WMap {
    const u64* dets;   // 4 words per determinant
    u32* slot;         // index or kEmpty
    u64 mask;          // capacity - 1
    __device__ long long find(const M2& a, const M2& b) const {
        u64 h = hash4(a, b) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            const u32 j = slot[h];
            if (j == kEmpty) return -1;
            if (eq4(dets + 4 * (i64)j, a, b)) return j;
            h = (h + 1) & mask;
        }
        return -1;
    }
};

__global__ void k_wmap_insert(WMap M, i64 n, unsigned long long* dup) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64* d = M.dets + 4 * t;
        const M2 a{d[0], d[1]}, b{d[2], d[3]};
        u64 h = hash4(a, b) & M.mask;
        for (u64 probe = 0; probe <= M.mask; ++probe) {
            const u32 old = atomicCAS(&M.slot[h], kEmpty, (u32)t);
            if (old == kEmpty) break;
            if (eq4(M.dets + 4 * (i64)old, a, b)) {
                atomicAdd(dup, 1ull);
                break;
            }
            h = (h + 1) & M.mask;
        }
    }
}

__global__ void k_wide_check(const u64* d, i64 n, int n_orb, unsigned long long* bad) {
    const M2 keep = mask_below(n_orb);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64* x = d + 4 * t;
        if ((x[0] & ~keep.lo) | (x[1] & ~keep.hi) | (x[2] & ~keep.lo) | (x[3] & ~keep.hi))
            atomicAdd(bad, 1ull);
    }
}

__global__ void k_wide_diag(CtxView C, const u64* d, i64 n, double* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64* x = d + 4 * t;
        out[t] = diag2(C, M2{x[0], x[1]}, M2{x[2], x[3]});
    }
}

struct alignas(32) Key4 {
    u64 w[4];   // alpha lo, alpha hi, beta lo, beta hi
};

}  // namespace
namespace prim {
namespace {
// Most significant first: alpha hi, alpha lo, beta hi, beta lo.
template <>
struct RadixKey<Key4> {
    static constexpr int W = 4;
    __device__ __forceinline__ static u64 word(const Key4& k, int i) {
        return k.w[i == 0 ? 1 : i == 1 ? 0 : i == 2 ? 3 : 2];
    }
};
}  // namespace
}  // namespace prim
namespace {

struct WParams {
    CtxView C;
    WMap V;
    const u64* dets;
    i64 n;
    int n_orb;
    bool dynamic;
    double eps1;
    double cut;           // table floor (static: the cutoff itself)
    const double* psi;
    const double* diag;
    int* next_row;
    // work units: a whole row, or for rows with very many candidates one
    // segment each (segment 0 = diagonal + singles, 1 + p = occupied pair p
    // in the order x = 1.., y < x, p = x(x-1)/2 + y)
    const uint4* units;   // {row, first segment, end segment, 0}
    i64 n_units;
    u32* smask;           // per unit: survivor bits of each 32-single step
    int smask_words;      // words per unit
    u32* cnt_vv;          // per unit
    u32* cnt_vp;
    const i64* off_vv;    // per unit
    const i64* off_vp;
    u32* vv_col;
    double* vv_val;
    Key4* vp_key;
    double* vp_val;
};

constexpr u32 kAllSegments = 0xffffffffu;

__device__ __forceinline__ double row_cut(const WParams& P, int r, double& psr) {
    psr = 0.0;
    if (!P.dynamic) return P.cut;
    psr = P.psi[r];
    return fmax(P.eps1 / fmax(fabs(psr), kAmpDelta), P.cut);   // build_ham.cpp:161-186
}

// Candidates of a row: singles + the table prefix of every occupied pair
// (lane-parallel binary searches); rows above a threshold are split into
// per-pair units.
__global__ void k_wide_work(WParams P, unsigned long long* work) {
    __shared__ WRow rows[kWW];
    const int lane = threadIdx.x & 31;
    WRow& R = rows[threadIdx.x >> 5];
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    for (i64 r = gw; r < P.n; r += nw) {
        const u64* d = P.dets + 4 * r;
        load_wrow(R, M2{d[0], d[1]}, M2{d[2], d[3]}, P.n_orb);
        double psr;
        const double cut = row_cut(P, (int)r, psr);
        const int npairs = R.ne * (R.ne - 1) / 2;
        unsigned long long w = 0;
        for (int p = lane; p < npairs; p += 32) {
            int x = (int)((1.0 + sqrt(1.0 + 8.0 * p)) * 0.5);
            while (x * (x - 1) / 2 > p) --x;
            while ((x + 1) * x / 2 <= p) ++x;
            const int y = p - x * (x - 1) / 2;
            const i64 row = pair_row(R.occ[x], R.occ[y]);
            const i64 lo = __ldg(&P.C.tab.off[row]), len = __ldg(&P.C.tab.off[row + 1]) - lo;
            i64 L = 0, H = len;
            if (cut > 0.0) {
                while (L < H) {
                    const i64 mid = (L + H) >> 1;
                    if (fabs(__ldg(&P.C.tab.v[lo + mid])) >= cut) L = mid + 1; else H = mid;
                }
            } else {
                L = len;
            }
            w += (unsigned long long)L;
        }
        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (lane == 0) work[r] = w + (unsigned long long)(R.na * R.nva + R.nb * R.nvb);
        __syncwarp();
    }
}

template <bool FILL>
__global__ void __launch_bounds__(kWW * 32) k_wide_build(WParams P) {
    __shared__ WRow rows[kWW];
    const int lane = threadIdx.x & 31;
    WRow& R = rows[threadIdx.x >> 5];
    const unsigned lt = lanemask_lt();
    for (;;) {
        int ui = 0;
        if (lane == 0) ui = atomicAdd(P.next_row, 1);
        ui = __shfl_sync(0xffffffffu, ui, 0);
        if (ui >= P.n_units) break;
        const uint4 U = P.units[ui];
        const int r = (int)U.x;
        const u64* d = P.dets + 4 * (i64)r;
        load_wrow(R, M2{d[0], d[1]}, M2{d[2], d[3]}, P.n_orb);
        double psr;
        const double cut = row_cut(P, r, psr);
        const int npairs = R.ne * (R.ne - 1) / 2;
        const u32 seg_lo = U.y;
        const u32 seg_hi = U.z == kAllSegments ? (u32)npairs + 1 : U.z;
        u32 nvv = 0, nvp = 0;
        i64 wvv = FILL ? P.off_vv[ui] : 0, wvp = FILL ? P.off_vp[ui] : 0;
        // one step of 32 candidates: route, count or write in candidate order
        auto emit = [&](bool valid, const M2& ka, const M2& kb, double h) {
            int route = 0;
            long long j = -1;
            if (valid && fabs(h) > kElemThresh) {
                j = P.V.find(ka, kb);
                route = j >= 0 ? 1 : 2;
            }
            if (!FILL) {
                nvv += route == 1;
                nvp += route == 2;
                return;
            }
            const unsigned mv = __ballot_sync(0xffffffffu, route == 1);
            if (route == 1) {
                const i64 at = wvv + __popc(mv & lt);
                P.vv_col[at] = (u32)j;
                P.vv_val[at] = h;
            }
            wvv += __popc(mv);
            const unsigned mp = __ballot_sync(0xffffffffu, route == 2);
            if (route == 2) {
                const i64 at = wvp + __popc(mp & lt);
                Key4 k;
                k.w[0] = ka.lo; k.w[1] = ka.hi; k.w[2] = kb.lo; k.w[3] = kb.hi;
                P.vp_key[at] = k;
                P.vp_val[at] = h;
            }
            wvp += __popc(mp);
        };
        if (seg_lo == 0) {
            const double dg = P.diag[r];
            if (fabs(dg) > kElemThresh) {
                if (FILL && lane == 0) {
                    P.vv_col[wvv] = (u32)r;
                    P.vv_val[wvv] = dg;
                }
                if (FILL) wvv += 1;
                else if (lane == 0) nvv = 1;
            }
            // singles: alpha then beta, holes outer, particles inner.  The
            // count pass records which lanes survive screening, so the fill
            // pass evaluates only those
            const int nsa = R.na * R.nva, nst = nsa + R.nb * R.nvb;
            u32* sm = P.smask + (i64)ui * P.smask_words;
            for (int t0 = 0; t0 < nst; t0 += 32) {
                const int t = t0 + lane;
                bool valid = t < nst;
                if (FILL) valid = valid && ((sm[t0 >> 5] >> lane) & 1u);
                M2 ka = R.a, kb = R.b;
                double h = 0.0;
                if (valid) {
                    int sp, hh, pp;
                    if (t < nsa) {
                        sp = 0; hh = R.occa[t / R.nva]; pp = R.vira[t % R.nva];
                        flip(ka, hh); flip(ka, pp);
                    } else {
                        const int u = t - nsa;
                        sp = 1; hh = R.occb[u / R.nvb]; pp = R.virb[u % R.nvb];
                        flip(kb, hh); flip(kb, pp);
                    }
                    h = single2(P.C, R, sp, hh, pp);
                    if (P.dynamic && !(fabs(h * psr) >= P.eps1)) valid = false;   // :190-192
                }
                if (!FILL) {
                    const unsigned keep = __ballot_sync(0xffffffffu, valid && fabs(h) > kElemThresh);
                    if (lane == 0) sm[t0 >> 5] = keep;
                }
                emit(valid, ka, kb, h);
            }
        }
        // heat-bath doubles over occupied pairs (ham_utils.hpp:280-313)
        const int p_lo = seg_lo == 0 ? 0 : (int)seg_lo - 1;
        const int p_hi = (int)seg_hi - 1;
        int x = 1, y = 0;
        {
            int xx = (int)((1.0 + sqrt(1.0 + 8.0 * p_lo)) * 0.5);
            while (xx * (xx - 1) / 2 > p_lo) --xx;
            while ((xx + 1) * xx / 2 <= p_lo) ++xx;
            x = max(xx, 1);
            y = p_lo - x * (x - 1) / 2;
        }
        for (int p = p_lo; p < p_hi; ++p) {
            const int i = R.occ[x];
            const int jj0 = R.occ[y];
            const i64 row = pair_row(i, jj0);
            const i64 lo = __ldg(&P.C.tab.off[row]);
            const i64 len = prefix_len(P.C.tab.v + lo, __ldg(&P.C.tab.off[row + 1]) - lo, cut);
            const int ii = max(i, jj0), jj = min(i, jj0);
            for (i64 e0 = 0; e0 < len; e0 += 32) {
                const i64 e = e0 + lane;
                bool valid = e < len;
                M2 ka = R.a, kb = R.b;
                double h = 0.0;
                if (valid) {
                    const u16 ab = __ldg(&P.C.tab.ab[lo + e]);
                    const int A = ab & 0xff, B = ab >> 8;
                    const bool oA = (A >> 1) >= P.n_orb || bit((A & 1) ? R.b : R.a, A >> 1);
                    const bool oB = (B >> 1) >= P.n_orb || bit((B & 1) ? R.b : R.a, B >> 1);
                    if (oA || oB) {
                        valid = false;
                    } else {
                        M2* w[2] = {&ka, &kb};
                        flip(*w[ii & 1], ii >> 1);
                        flip(*w[jj & 1], jj >> 1);
                        flip(*w[A & 1], A >> 1);
                        flip(*w[B & 1], B >> 1);
                        h = double2(R.a, R.b, ii, jj, A, B, __ldg(&P.C.tab.v[lo + e]));
                    }
                }
                emit(valid, ka, kb, h);
            }
            if (++y == x) {
                ++x;
                y = 0;
            }
        }
        if (!FILL) {
            const u32 a = __reduce_add_sync(0xffffffffu, nvv);
            const u32 b = __reduce_add_sync(0xffffffffu, nvp);
            if (lane == 0) {
                P.cnt_vv[ui] = a;
                P.cnt_vp[ui] = b;
            }
        }
        __syncwarp();
    }
}

// Row pointers from unit offsets: row r starts at its first unit.
__global__ void k_row_starts(const i64* uoff, const u32* first_unit, i64 n, i64* rowptr) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r <= n;
         r += (i64)gridDim.x * blockDim.x)
        rowptr[r] = uoff[first_unit[r]];
}

__device__ __forceinline__ bool neq_prev(const Key4* k, i64 t) {
    return t == 0 || k[t].w[0] != k[t - 1].w[0] || k[t].w[1] != k[t - 1].w[1] ||
           k[t].w[2] != k[t - 1].w[2] || k[t].w[3] != k[t - 1].w[3];
}

__global__ void k_key4_flags(const Key4* k, i64 n, u32* flag) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        flag[t] = neq_prev(k, t) ? 1u : 0u;
}

__global__ void k_key4_scatter(const Key4* k, const u32* perm, const u32* runid, i64 n, u64* pdets,
                               u32* col) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 r = runid[t] - 1;
        if (neq_prev(k, t))
            for (int q = 0; q < 4; ++q) pdets[4 * (i64)r + q] = k[t].w[q];
        col[perm[t]] = r;
    }
}

int blocks(i64 n) {
    const i64 b = (n + 255) / 256;
    return (int)std::max<i64>(1, std::min<i64>(b, 65535));
}

template <class T>
void exscan(const T* in, i64* out, i64 n, cudaStream_t s) {
    prim::scan<T, i64, false>(in, out, n, s);
}

i64 fetch(const i64* d, cudaStream_t s) {
    i64 v = 0;
    DNQ_CUDA(cudaMemcpyAsync(&v, d, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    return v;
}

}  // namespace

void launch_wide_diag(const dnq_ctx_s* ctx, const u64* d, i64 n, double* out, cudaStream_t s) {
    if (n == 0) return;
    k_wide_diag<<<blocks(n), 256, 0, s>>>(ctx->view(), d, n, out);
    DNQ_CHECK_LAUNCH();
}

void wide_build(dnq_ctx_s* ctx, const u64* V_in, i64 n, const double* psi_in, int n_orb,
                double eps1, cudaStream_t s, dnq_ham_s* H) {
    H->device = ctx->device;
    H->stream = s;
    H->words = 2;
    H->n_v = n;
    DIn<u64> V(V_in, 4 * n, s);
    DIn<double> psi(psi_in, psi_in ? n : 0, s);
    {
        DBuf<unsigned long long> bad(1, s);
        DNQ_CUDA(cudaMemsetAsync(bad.p, 0, 8, s));
        k_wide_check<<<blocks(n), 256, 0, s>>>(V.p, n, n_orb, bad.p);
        DNQ_CHECK_LAUNCH();
        unsigned long long h = 0;
        DNQ_CUDA(cudaMemcpyAsync(&h, bad.p, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        require(h == 0, DNQ_ERR_INVALID, "determinant has orbitals >= n_orb");
    }
    // hash of V
    u64 cap = 1;
    while (cap < (u64)(2 * n)) cap <<= 1;
    DBuf<u32> slot(cap, s);
    DNQ_CUDA(cudaMemsetAsync(slot.p, 0xff, cap * 4, s));
    WMap M{V.p, slot.p, cap - 1};
    {
        DBuf<unsigned long long> dup(1, s);
        DNQ_CUDA(cudaMemsetAsync(dup.p, 0, 8, s));
        k_wmap_insert<<<blocks(n), 256, 0, s>>>(M, n, dup.p);
        DNQ_CHECK_LAUNCH();
        unsigned long long h = 0;
        DNQ_CUDA(cudaMemcpyAsync(&h, dup.p, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        require(h == 0, DNQ_ERR_DUPLICATE, "DetMap::from_ordered: duplicate determinant found");
    }
    H->diag.alloc(n, s);
    launch_wide_diag(ctx, V.p, n, H->diag.p, s);

    WParams P{};
    P.C = ctx->view();
    P.V = M;
    P.dets = V.p;
    P.n = n;
    P.n_orb = n_orb;
    P.dynamic = psi_in != nullptr;
    P.eps1 = eps1;
    P.cut = P.dynamic ? ctx->hb_thr : hb_cutoff(ctx, eps1);
    P.psi = psi.p;
    P.diag = H->diag.p;
    const int sms = sm_count(ctx->device);

    // ---- units: rows above kHeavy candidates are split per occupied pair
    constexpr unsigned long long kHeavy = 1ull << 15;
    std::vector<uint4> units;
    std::vector<u32> first(n + 1);
    {
        DBuf<unsigned long long> work(n, s);
        k_wide_work<<<sms * 16, kWW * 32, 0, s>>>(P, work.p);
        DNQ_CHECK_LAUNCH();
        std::vector<unsigned long long> hw(n);
        std::vector<u64> hd(4 * n);
        DNQ_CUDA(cudaMemcpyAsync(hw.data(), work.p, 8 * n, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaMemcpyAsync(hd.data(), V.p, 32 * n, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        units.reserve(n);
        for (i64 r = 0; r < n; ++r) {
            first[r] = (u32)units.size();
            if (hw[r] > kHeavy) {
                int ne = 0;
                for (int q = 0; q < 4; ++q) ne += __builtin_popcountll(hd[4 * r + q]);
                const u32 np = (u32)(ne * (ne - 1) / 2);
                for (u32 g = 0; g <= np; ++g) units.push_back(make_uint4((u32)r, g, g + 1, 0));
            } else {
                units.push_back(make_uint4((u32)r, 0, kAllSegments, 0));
            }
        }
        first[n] = (u32)units.size();
        int max_nst = 0;
        for (i64 r = 0; r < n; ++r) {
            int na = 0, nb = 0;
            na = __builtin_popcountll(hd[4 * r]) + __builtin_popcountll(hd[4 * r + 1]);
            nb = __builtin_popcountll(hd[4 * r + 2]) + __builtin_popcountll(hd[4 * r + 3]);
            max_nst = std::max(max_nst, na * (n_orb - na) + nb * (n_orb - nb));
        }
        P.smask_words = std::max(1, (max_nst + 31) / 32);
    }
    const i64 nu = (i64)units.size();
    DBuf<uint4> ud(nu, s);
    DBuf<u32> fd(n + 1, s);
    DNQ_CUDA(cudaMemcpyAsync(ud.p, units.data(), 16 * nu, cudaMemcpyHostToDevice, s));
    DNQ_CUDA(cudaMemcpyAsync(fd.p, first.data(), 4 * (n + 1), cudaMemcpyHostToDevice, s));
    P.units = ud.p;
    P.n_units = nu;
    DBuf<u32> smask((size_t)nu * P.smask_words, s);
    P.smask = smask.p;

    DBuf<int> next(1, s);
    DBuf<u32> cvv(nu + 1, s), cvp(nu + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cvv.p + nu, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(cvp.p + nu, 0, 4, s));
    P.next_row = next.p;
    P.cnt_vv = cvv.p;
    P.cnt_vp = cvp.p;
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wide_build<false>, kWW * 32,
                                                           0));
    const int grid = std::max(1, per_sm) * sms;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_wide_build<false><<<grid, kWW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();

    DBuf<i64> uvv(nu + 1, s), uvp(nu + 1, s);
    exscan(cvv.p, uvv.p, nu + 1, s);
    exscan(cvp.p, uvp.p, nu + 1, s);
    H->vv.nr = H->vv.nc = n;
    H->vv.rowptr.alloc(n + 1, s);
    DBuf<i64> offp(n + 1, s);
    k_row_starts<<<blocks(n + 1), 256, 0, s>>>(uvv.p, fd.p, n, H->vv.rowptr.p);
    DNQ_CHECK_LAUNCH();
    k_row_starts<<<blocks(n + 1), 256, 0, s>>>(uvp.p, fd.p, n, offp.p);
    DNQ_CHECK_LAUNCH();
    H->vv.nnz = fetch(uvv.p + nu, s);
    const i64 nvp = fetch(uvp.p + nu, s);
    require(nvp < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "H_VP has more than 2^32 entries");
    H->vv.col.alloc(H->vv.nnz, s);
    H->vv.val.alloc(H->vv.nnz, s);
    DBuf<Key4> keys(nvp, s);
    DBuf<double> vpv(nvp, s);
    P.off_vv = uvv.p;
    P.off_vp = uvp.p;
    P.vv_col = H->vv.col.p;
    P.vv_val = H->vv.val.p;
    P.vp_key = keys.p;
    P.vp_val = vpv.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_wide_build<true><<<grid, kWW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    sort_rows(H->vv, s);

    // P: 256-bit radix sort with positions, unique, relabel
    DBuf<Key4> ks(nvp, s);
    DBuf<u32> perm2(nvp, s);
    if (nvp) {
        const int hi = n_orb > 64 ? n_orb - 64 : 0, lo = n_orb > 64 ? 64 : n_orb;
        const int bits[4] = {hi, lo, hi, lo};
        prim::radix_sort<Key4, u32>(keys.p, ks.p, nullptr, perm2.p, nvp, bits, s);
    }
    keys.release();
    i64 np = 0;
    DBuf<u32> flag(nvp, s), runid(nvp, s);
    if (nvp) {
        k_key4_flags<<<blocks(nvp), 256, 0, s>>>(ks.p, nvp, flag.p);
        DNQ_CHECK_LAUNCH();
        prim::scan_inclusive<u32, u32>(flag.p, runid.p, nvp, s);
        u32 last = 0;
        DNQ_CUDA(cudaMemcpyAsync(&last, runid.p + nvp - 1, 4, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        np = last;
    }
    H->n_p = np;
    H->vp.nr = n;
    H->vp.nc = np;
    H->vp.nnz = nvp;
    H->vp.rowptr = std::move(offp);
    H->vp.val = std::move(vpv);
    H->vp.col.alloc(nvp, s);
    H->dets_p.alloc(4 * np, s);
    if (nvp) {
        k_key4_scatter<<<blocks(nvp), 256, 0, s>>>(ks.p, perm2.p, runid.p, nvp, (u64*)H->dets_p.p,
                                                   H->vp.col.p);
        DNQ_CHECK_LAUNCH();
    }
    sort_rows(H->vp, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
}

}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_wide_diag(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, double* out, void* stream) {
    DNQ_API_BEGIN
    require(ctx && (n == 0 || (dets && out)), DNQ_ERR_INVALID, "null argument");
    if (n == 0) return DNQ_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> d(dets, 4 * n, s);
    const bool dev_out = is_device_ptr(out);
    DBuf<double> tmp;
    double* o = out;
    if (!dev_out) {
        tmp.alloc(n, s);
        o = tmp.p;
    }
    launch_wide_diag(ctx, d.p, n, o, s);
    if (!dev_out) copy_out(out, o, n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_wide_build(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, const double* psi,
                   int n_orb, double eps1, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require(ctx && out && (n == 0 || dets), DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(n >= 0 && n < (int64_t)0xffffffffll, DNQ_ERR_OVERFLOW, "too many determinants");
    require(n_orb >= 1 && n_orb <= ctx->n && n_orb <= 128, DNQ_ERR_INVALID,
            "n_orb must be in [1, min(128, orbitals of the context)]");
    require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    wide_build(ctx, dets, n, psi, n_orb, eps1, s, H.get());
    *out = H.release();
    DNQ_API_END
}

}  // extern "C"
