// vvstr.cu -- V->V block of the screened Hamiltonian from string groups.
//
// When only H_VV is wanted (get_ham_vv; get_ham_conn / get_ham_conn_amp
// without the P block), every ket that can land in V is itself a member of
// V, so instead of walking all ~n_e^2 n_v^2 candidates of a row and probing
// each in a hash, the rows are matched against V directly.  V is indexed
// twice: sorted by (beta, alpha) with a hash from a beta string to its
// group, and by (alpha, beta) with a hash from an alpha string to its group.
// For a bra (a, b) the members of V connected by at most a double fall in
// three disjoint parts:
//   A  same beta string b:  alpha single or alpha-alpha double of a;
//   B  same alpha string a: beta single or beta-beta double of b;
//   C  alpha string a' = single of a, beta string a single of b:
//      the group of every single a' of a, filtered by popc(b ^ b') == 2.
// Each match gets its element exactly as HamEval::compute_elem does
// (ham_eval.cpp:88-147: same integrals, same order of operations) and is
// kept under the policy's rules; for a double |H| equals the heat-bath
// weight |<ij||ab>| bit for bit, so the table cut w >= cut is applied to
// the element.  Results are identical to the candidate walk in gen.cuh.
#include <cub/cub.cuh>
#include <cuda/std/tuple>

#include "gen.cuh"
#include "ham.cuh"

namespace dnq {

namespace {

constexpr int kWS = 8;               // warps per block
constexpr u32 kBigGroup = 2048;      // part C: search instead of scan above this

struct StrMapView {
    const ulonglong2* slots = nullptr;   // x = string (~0 empty), y = start<<32 | len
    u64 mask = 0;
    __device__ __forceinline__ bool find(u64 key, u32& start, u32& len) const {
        u64 h = det_hash(key, 0x5bd1e995ull) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            const ulonglong2 sl = __ldg(&slots[h]);
            if (sl.x == kEmptyKey) return false;
            if (sl.x == key) {
                start = (u32)(sl.y >> 32);
                len = (u32)(sl.y & 0xffffffffu);
                return true;
            }
            h = (h + 1) & mask;
        }
        return false;
    }
};

struct StrIndex {
    DBuf<u64> other;     // sorted companion string (alpha for beta groups, ...)
    DBuf<u32> idx;       // original position in V
    DBuf<ulonglong2> slots;
    u64 mask = 0;
    StrMapView view() const { return StrMapView{slots.p, mask}; }
};

struct SwapKey {
    __host__ __device__ ::cuda::std::tuple<unsigned long long&, unsigned long long&>
    operator()(ulonglong2& k) const {
        return {k.x, k.y};
    }
};

__global__ void k_keys_by(const u64* V, i64 n, int major, ulonglong2* k, u32* id) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = V[2 * t], b = V[2 * t + 1];
        k[t] = major == 0 ? make_ulonglong2(a, b) : make_ulonglong2(b, a);
        id[t] = (u32)t;
    }
}

__global__ void k_split_sorted(const ulonglong2* k, i64 n, u64* other, unsigned* head) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        other[t] = k[t].y;
        head[t] = (t == 0 || k[t].x != k[t - 1].x) ? 1u : 0u;
    }
}

// Start position of every group (gid = exclusive scan of the head flags).
__global__ void k_group_starts(const unsigned* head, const u32* gid, i64 n, u32* gstart) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        if (head[t]) gstart[gid[t]] = (u32)t;
}

// Insert one slot per group: (string, start << 32 | len).
__global__ void k_group_insert(const ulonglong2* k, const u32* gstart, i64 ngroups, i64 n,
                               ulonglong2* slots, u64 mask) {
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < ngroups;
         g += (i64)gridDim.x * blockDim.x) {
        const i64 t = gstart[g];
        const i64 e = g + 1 < ngroups ? (i64)gstart[g + 1] : n;
        const u64 key = k[t].x;
        const u64 val = ((u64)t << 32) | (u64)(e - t);
        u64 h = det_hash(key, 0x5bd1e995ull) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev = atomicCAS(
                reinterpret_cast<unsigned long long*>(&slots[h].x), kEmptyKey, key);
            if (prev == kEmptyKey) {
                slots[h].y = val;
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

int gsz(i64 n) {
    i64 b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

// major 0: groups by alpha (companion beta); major 1: groups by beta.
void build_str_index(StrIndex& X, const u64* V, i64 n, int major, cudaStream_t s) {
    DBuf<ulonglong2> k(n, s), ks(n, s);
    DBuf<u32> id(n, s);
    X.idx.alloc(n, s);
    X.other.alloc(n, s);
    k_keys_by<<<gsz(n), 256, 0, s>>>(V, n, major, k.p, id.p);
    DNQ_CHECK_LAUNCH();
    size_t tmp = 0;
    DNQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k.p, ks.p, id.p, X.idx.p, n,
                                             SwapKey{}, s));
    DBuf<u8> tb(tmp, s);
    DNQ_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, k.p, ks.p, id.p, X.idx.p, n,
                                             SwapKey{}, s));
    DBuf<unsigned> head(n, s);
    k_split_sorted<<<gsz(n), 256, 0, s>>>(ks.p, n, X.other.p, head.p);
    DNQ_CHECK_LAUNCH();
    DBuf<u32> gid(n + 1, s), gstart(n, s);
    {
        size_t t2 = 0;
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, head.p, gid.p, n, s));
        DBuf<u8> tb2(t2, s);
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(tb2.p, t2, head.p, gid.p, n, s));
    }
    u32 last_gid = 0, last_head = 0;
    DNQ_CUDA(cudaMemcpyAsync(&last_gid, gid.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&last_head, head.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    const i64 ngroups = (i64)last_gid + last_head;
    k_group_starts<<<gsz(n), 256, 0, s>>>(head.p, gid.p, n, gstart.p);
    DNQ_CHECK_LAUNCH();
    u64 cap = 1024;
    while (cap < (u64)(2 * ngroups)) cap <<= 1;
    X.mask = cap - 1;
    X.slots.alloc(cap, s);
    DNQ_CUDA(cudaMemsetAsync(X.slots.p, 0xff, cap * sizeof(ulonglong2), s));
    k_group_insert<<<gsz(ngroups), 256, 0, s>>>(ks.p, gstart.p, ngroups, n, X.slots.p, X.mask);
    DNQ_CHECK_LAUNCH();
}

__device__ __forceinline__ i64 tri2(i64 p, i64 q) {
    return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
}
__device__ __forceinline__ double eri(const double* E, int p, int q, int r, int s) {
    return __ldg(&E[tri2(tri2(p, q), tri2(r, s))]);
}

struct VVParams {
    CtxView C;
    const double* E;        // packed ERI
    const u64* V;
    i64 n;
    int n_orb;
    StrMapView amap, bmap;
    const u64* a_other;     // beta of the alpha-sorted entries
    const u32* a_idx;
    const u64* b_other;     // alpha of the beta-sorted entries
    const u32* b_idx;
    const double* diag;
    int policy;
    double eps1;
    double cut;             // doubles: keep w >= cut (and > 1e-15)
    const double* psi;
    int* next_row;
    unsigned long long* n_test;
    // single pass: rows appended to warp-private chunks of an arena
    u32* acol;
    double* aval;
    i64 cap;                          // arena capacity (entries)
    i64 chunk;                        // entries per warp chunk
    unsigned long long* cursor;       // next free arena entry
    int* overflow;                    // set when the arena is too small
    i64* row_pos;
    u32* row_len;
    u32* big;                         // rows longer than one chunk
    int* n_big;
    // two-pass fallback
    u32* cnt;
    const i64* off;
    u32* col;
    double* val;
};

constexpr i64 kChunk = 8192;   // default arena entries per warp chunk

// Warp-collective sinks of one row's entries.
struct CountOut {
    u32 c = 0;
    __device__ __forceinline__ void put(bool keep, u32, double) {
        c += __popc(__ballot_sync(0xffffffffu, keep));
    }
};

struct ExactOut {
    u32* col;
    double* val;
    i64 w;
    u32 c = 0;
    __device__ __forceinline__ void put(bool keep, u32 j, double h) {
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const i64 at = w + __popc(m & lanemask_lt());
            col[at] = j;
            val[at] = h;
        }
        w += __popc(m);
        c += __popc(m);
    }
};

// Writes into [w, end) of a chunk; past the end it only counts.
struct ChunkOut {
    u32* col;
    double* val;
    i64 w, end;
    u32 c = 0;
    bool over = false;
    __device__ __forceinline__ void put(bool keep, u32 j, double h) {
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        const int k = __popc(m);
        if (!over) {
            if (w + k > end) {
                over = true;
            } else {
                if (keep) {
                    const i64 at = w + __popc(m & lanemask_lt());
                    col[at] = j;
                    val[at] = h;
                }
                w += k;
            }
        }
        c += k;
    }
};

// Single within one spin: bra string x -> ket string y (differ in 2 bits).
__device__ __forceinline__ double str_single(const VVParams& P, u64 a, u64 b, int spin, u64 x,
                                             u64 y) {
    const u64 d = x ^ y;
    const int h = __ffsll(x & d) - 1;   // bra orbital
    const int p = __ffsll(y & d) - 1;   // ket orbital
    return single_elem(P.C, a, b, spin, h, p);
}

// Same-spin double: bra string x -> ket string y (differ in 4 bits).
__device__ __forceinline__ double str_double_same(const VVParams& P, u64 x, u64 y) {
    const u64 d = x ^ y;
    u64 pb = x & d, hk = y & d;
    const int p0 = __ffsll(pb) - 1;
    pb &= pb - 1;
    const int p1 = __ffsll(pb) - 1;
    const int h0 = __ffsll(hk) - 1;
    hk &= hk - 1;
    const int h1 = __ffsll(hk) - 1;
    // anti(p0,p1,h0,h1) = (p0 h0|p1 h1) - (p0 h1|p1 h0)   (ham_eval.cpp:124-139)
    const double raw = eri(P.E, p0, h0, p1, h1) - eri(P.E, p0, h1, p1, h0);
    int perm = occ_between(x, h0, p0) + occ_between(x, h1, p1);
    const int A = min(h0, p0), B = max(h0, p0), Cc = min(h1, p1), D = max(h1, p1);
    if ((Cc > A && Cc < B && D > B) || (A > Cc && A < D && B > D)) ++perm;
    return (perm & 1) ? -raw : raw;
}

__device__ __forceinline__ bool keep_double(double cut, double h) {
    const double w = fabs(h);
    return w > kElemThresh && w >= cut;
}

__device__ __forceinline__ bool keep_single(const VVParams& P, double psr, double h) {
    if (!(fabs(h) > kElemThresh)) return false;
    if (P.policy == DNQ_POLICY_DYNAMIC) return fabs(h * psr) >= P.eps1;
    return true;
}

// Per-warp shared state.
struct WarpShared {
    u32 start[32], len[32];
    u8 h[32], p[32];
    u8 occa[64], vira[64], occb[64], virb[64];
};

__device__ __forceinline__ void load_lists(WarpShared& S, u64 a, u64 b, u64 all) {
    if ((threadIdx.x & 31) == 0) {
        int k = 0;
        for (u64 m = a; m; m &= m - 1) S.occa[k++] = (u8)(__ffsll(m) - 1);
        k = 0;
        for (u64 m = ~a & all; m; m &= m - 1) S.vira[k++] = (u8)(__ffsll(m) - 1);
        k = 0;
        for (u64 m = b; m; m &= m - 1) S.occb[k++] = (u8)(__ffsll(m) - 1);
        k = 0;
        for (u64 m = ~b & all; m; m &= m - 1) S.virb[k++] = (u8)(__ffsll(m) - 1);
    }
    __syncwarp();
}

// All entries of row r: the diagonal first, then parts A, B and C.
template <class Out>
__device__ void vv_row(const VVParams& P, int r, u64 a, u64 b, double psr, double cut,
                       WarpShared& S, Out& out, unsigned long long& tests) {
    const int lane = threadIdx.x & 31;
    const u64 all = low_mask(P.n_orb);
    const double d = P.diag[r];
    out.put(lane == 0 && fabs(d) > kElemThresh, (u32)r, d);
    // ---- part A: same beta string
    u32 st = 0, ln = 0;
    if (lane == 0 && !P.bmap.find(b, st, ln)) ln = 0;
    st = __shfl_sync(0xffffffffu, st, 0);
    ln = __shfl_sync(0xffffffffu, ln, 0);
    tests += ln;
    for (u32 t0 = 0; t0 < ln; t0 += 32) {
        const u32 t = t0 + lane;
        bool keep = false;
        double h = 0.0;
        u32 j = 0;
        if (t < ln) {
            const u64 y = __ldg(&P.b_other[st + t]);
            const int dd = __popcll(a ^ y);
            if (dd == 2) {
                h = str_single(P, a, b, 0, a, y);
                keep = keep_single(P, psr, h);
            } else if (dd == 4) {
                h = str_double_same(P, a, y);
                keep = keep_double(cut, h);
            }
            if (keep) j = __ldg(&P.b_idx[st + t]);
        }
        out.put(keep, j, h);
    }
    // ---- part B: same alpha string
    if (lane == 0 && !P.amap.find(a, st, ln)) ln = 0;
    st = __shfl_sync(0xffffffffu, st, 0);
    ln = __shfl_sync(0xffffffffu, ln, 0);
    tests += ln;
    for (u32 t0 = 0; t0 < ln; t0 += 32) {
        const u32 t = t0 + lane;
        bool keep = false;
        double h = 0.0;
        u32 j = 0;
        if (t < ln) {
            const u64 y = __ldg(&P.a_other[st + t]);
            const int dd = __popcll(b ^ y);
            if (dd == 2) {
                h = str_single(P, a, b, 1, b, y);
                keep = keep_single(P, psr, h);
            } else if (dd == 4) {
                h = str_double_same(P, b, y);
                keep = keep_double(cut, h);
            }
            if (keep) j = __ldg(&P.a_idx[st + t]);
        }
        out.put(keep, j, h);
    }
    // ---- part C: alpha single x beta single, via the groups of the a'
    const int na = __popcll(a), nva = __popcll(~a & all);
    const int nsa = na * nva;
    const int nb = __popcll(b), nvb = __popcll(~b & all);
    for (int s0 = 0; s0 < nsa; s0 += 32) {
        const int sidx = s0 + lane;
        u32 gs = 0, gl = 0;
        int hh = 0, pp = 0;
        if (sidx < nsa) {
            hh = S.occa[sidx / nva];
            pp = S.vira[sidx % nva];
            if (!P.amap.find(a ^ (1ull << hh) ^ (1ull << pp), gs, gl)) gl = 0;
        }
        const bool big = gl > kBigGroup;
        const u32 sl = big ? 0u : gl;
        S.start[lane] = gs;
        S.len[lane] = sl;
        S.h[lane] = (u8)hh;
        S.p[lane] = (u8)pp;
        __syncwarp();
        const u32 total = __reduce_add_sync(0xffffffffu, sl);
        tests += total;
        // lane-private cursor (group l, offset o) advanced 32 members per step
        int l = 0;
        u32 o = lane;
        while (l < 32 && o >= S.len[l]) { o -= S.len[l]; ++l; }
        for (u32 t0 = 0; t0 < total; t0 += 32) {
            bool keep = false;
            double h = 0.0;
            u32 j = 0;
            if (l < 32) {
                const u32 at = S.start[l] + o;
                const u64 y = __ldg(&P.a_other[at]);
                const u64 x = b ^ y;
                if (__popcll(x) == 2) {
                    const int ha = S.h[l], pa = S.p[l];
                    const int hb = __ffsll(b & x) - 1, pb = __ffsll(y & x) - 1;
                    const double raw = eri(P.E, ha, pa, hb, pb);   // (a i|b j)
                    const int perm = occ_between(a, pa, ha) + occ_between(b, pb, hb);
                    h = (perm & 1) ? -raw : raw;
                    keep = keep_double(cut, h);
                    if (keep) j = __ldg(&P.a_idx[at]);
                }
            }
            out.put(keep, j, h);
            o += 32;
            while (l < 32 && o >= S.len[l]) { o -= S.len[l]; ++l; }
        }
        // large groups: binary-search every beta single of b instead
        unsigned bigm = __ballot_sync(0xffffffffu, big);
        while (bigm) {
            const int L = __ffs(bigm) - 1;
            bigm &= bigm - 1;
            const u32 g0 = S.start[L];
            const u32 gn = __shfl_sync(0xffffffffu, gl, L);
            const int ha = S.h[L], pa = S.p[L];
            tests += nb * nvb;
            for (int q0 = 0; q0 < nb * nvb; q0 += 32) {
                const int q = q0 + lane;
                bool keep = false;
                double h = 0.0;
                u32 j = 0;
                if (q < nb * nvb) {
                    const int hb = S.occb[q / nvb];
                    const int pb = S.virb[q % nvb];
                    const u64 y = b ^ (1ull << hb) ^ (1ull << pb);
                    u32 lo = g0, hi = g0 + gn;
                    while (lo < hi) {
                        const u32 mid = (lo + hi) >> 1;
                        if (__ldg(&P.a_other[mid]) < y) lo = mid + 1; else hi = mid;
                    }
                    if (lo < g0 + gn && __ldg(&P.a_other[lo]) == y) {
                        const double raw = eri(P.E, ha, pa, hb, pb);
                        const int perm = occ_between(a, pa, ha) + occ_between(b, pb, hb);
                        h = (perm & 1) ? -raw : raw;
                        keep = keep_double(cut, h);
                        if (keep) j = __ldg(&P.a_idx[lo]);
                    }
                }
                out.put(keep, j, h);
            }
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void row_setup(const VVParams& P, int r, u64& a, u64& b, double& psr,
                                          double& cut) {
    a = P.V[2 * (i64)r];
    b = P.V[2 * (i64)r + 1];
    psr = 0.0;
    cut = P.cut;
    if (P.policy == DNQ_POLICY_DYNAMIC) {
        psr = P.psi[r];
        cut = fmax(P.eps1 / fmax(fabs(psr), kAmpDelta), P.cut);   // build_ham.cpp:176-186
    }
}

__device__ __forceinline__ int next_row(int* ctr) {
    int r = 0;
    if ((threadIdx.x & 31) == 0) r = atomicAdd(ctr, 1);
    return __shfl_sync(0xffffffffu, r, 0);
}

__device__ __forceinline__ void add_tests(const VVParams& P, unsigned long long t) {
    if ((threadIdx.x & 31) == 0) atomicAdd(P.n_test, t);
}

// Single pass: each warp appends its rows to private chunks of the arena.
__global__ void __launch_bounds__(kWS * 32) k_vv_arena(VVParams P) {
    __shared__ WarpShared sh[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const u64 all = low_mask(P.n_orb);
    i64 cpos = 0, cend = 0;
    {   // first chunk of this warp
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(P.cursor, (unsigned long long)P.chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((i64)base + P.chunk <= P.cap) {
            cpos = (i64)base;
            cend = cpos + P.chunk;
        }
    }
    unsigned long long tests = 0;
    for (;;) {
        const int r = next_row(P.next_row);
        if (r >= P.n) break;
        if (*(volatile int*)P.overflow) continue;
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, all);
        for (int attempt = 0; attempt < 2; ++attempt) {
            ChunkOut out{P.acol, P.aval, cpos, cend};
            unsigned long long tt = 0;
            vv_row(P, r, a, b, psr, cut, S, out, tt);
            if (attempt == 0) tests += tt;
            if (!out.over) {
                if (lane == 0) {
                    P.row_pos[r] = cpos;
                    P.row_len[r] = out.c;
                }
                cpos = out.w;
                break;
            }
            if ((i64)out.c > P.chunk || attempt == 1) {   // longer than any chunk
                if (lane == 0) {
                    P.row_len[r] = out.c;
                    P.big[atomicAdd(P.n_big, 1)] = (u32)r;
                }
                break;
            }
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(P.cursor, (unsigned long long)P.chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((i64)base + P.chunk > P.cap) {
                if (lane == 0) atomicExch(P.overflow, 1);
                break;
            }
            cpos = (i64)base;
            cend = cpos + P.chunk;
        }
        __syncwarp();
    }
    add_tests(P, tests);
}

// Rows longer than a chunk: exact contiguous space, second walk.
__global__ void __launch_bounds__(kWS * 32) k_vv_big(VVParams P, int nbig) {
    __shared__ WarpShared sh[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const u64 all = low_mask(P.n_orb);
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < nbig; i += nw) {
        const int r = (int)P.big[i];
        const u32 len = P.row_len[r];
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(P.cursor, (unsigned long long)len);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((i64)base + len > P.cap) {
            if (lane == 0) atomicExch(P.overflow, 1);
            continue;
        }
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, all);
        ExactOut out{P.acol, P.aval, (i64)base};
        unsigned long long tt = 0;
        vv_row(P, r, a, b, psr, cut, S, out, tt);
        if (lane == 0) P.row_pos[r] = (i64)base;
        __syncwarp();
    }
}

// Gather the rows from the arena into a standard CSR.
__global__ void k_vv_compact(const i64* row_pos, const i64* rowptr, i64 n, const u32* acol,
                             const double* aval, u32* col, double* val) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    for (i64 r = gw; r < n; r += nw) {
        const i64 src = row_pos[r], dst = rowptr[r], len = rowptr[r + 1] - dst;
        for (i64 t = lane; t < len; t += 32) {
            col[dst + t] = acol[src + t];
            val[dst + t] = aval[src + t];
        }
    }
}

// Two-pass fallback (arena too small): count, then exact fill.
template <bool FILL>
__global__ void __launch_bounds__(kWS * 32) k_vv_twopass(VVParams P) {
    __shared__ WarpShared sh[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const u64 all = low_mask(P.n_orb);
    for (;;) {
        const int r = next_row(P.next_row);
        if (r >= P.n) break;
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, all);
        unsigned long long tt = 0;
        if (!FILL) {
            CountOut out;
            vv_row(P, r, a, b, psr, cut, S, out, tt);
            if (lane == 0) P.cnt[r] = out.c;
        } else {
            ExactOut out{P.col, P.val, P.off[r]};
            vv_row(P, r, a, b, psr, cut, S, out, tt);
        }
        __syncwarp();
    }
}

}  // namespace

void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s);

namespace {
template <class T>
void excl_scan(const T* in, i64* out, i64 n, cudaStream_t s) {
    size_t tmp = 0;
    DNQ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, s));
    DBuf<u8> tb(tmp, s);
    DNQ_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, in, out, n, s));
}
}  // namespace

// Test options: warp chunk size and arena capacity (0 = automatic).
i64 g_arena_chunk = 0;
i64 g_arena_cap = 0;

// H_VV only, from string groups.  V on the device, diag already computed.
// Rows are left in generation order (H->vv.sorted = false); copy-out
// functions sort them on demand.
void build_vv_strings(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, const double* diag, cudaStream_t s,
                      dnq_ham_s* H, double* t_ms) {
    cudaEvent_t ev[5];
    for (auto& e : ev) DNQ_CUDA(cudaEventCreate(&e));
    DNQ_CUDA(cudaEventRecord(ev[0], s));
    StrIndex A, B;
    build_str_index(A, V, n, 0, s);
    build_str_index(B, V, n, 1, s);
    VVParams P{};
    P.C = ctx->view();
    P.E = ctx->erid.p;
    P.V = V;
    P.n = n;
    P.n_orb = n_orb;
    P.amap = A.view();
    P.bmap = B.view();
    P.a_other = A.other.p;
    P.a_idx = A.idx.p;
    P.b_other = B.other.p;
    P.b_idx = B.idx.p;
    P.diag = diag;
    P.policy = policy;
    P.eps1 = eps1;
    P.cut = cut;
    P.psi = psi;
    DBuf<int> next(1, s), ovf(1, s), nbig(1, s);
    DBuf<unsigned long long> nt(1, s), cursor(1, s);
    DNQ_CUDA(cudaMemsetAsync(nt.p, 0, 8, s));
    P.next_row = next.p;
    P.n_test = nt.p;
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vv_arena, kWS * 32, 0));
    const int grid = std::max(1, per_sm) * sm_count(ctx->device);
    const i64 warps = (i64)grid * kWS;
    // arena: last build's size for this context if known, else 256 per row,
    // plus one chunk of slack per warp; capped by free memory
    size_t freeb = 0, totb = 0;
    DNQ_CUDA(cudaMemGetInfo(&freeb, &totb));
    const i64 chunk = g_arena_chunk > 0 ? g_arena_chunk : kChunk;
    i64 want = ctx->vv_nnz_hint > 0 ? (i64)(ctx->vv_nnz_hint * 1.05) : 256 * n;
    want += warps * chunk;
    const i64 maxfit = (i64)(freeb / 2 / 12);
    i64 cap = std::max<i64>(std::min(want, maxfit), chunk);
    if (g_arena_cap > 0) cap = g_arena_cap;
    DBuf<u32> acol(cap, s), rlen(n + 1, s), big(n, s);
    DBuf<double> aval(cap, s);
    DBuf<i64> rpos(n, s);
    P.acol = acol.p;
    P.aval = aval.p;
    P.cap = cap;
    P.chunk = chunk;
    P.cursor = cursor.p;
    P.overflow = ovf.p;
    P.row_pos = rpos.p;
    P.row_len = rlen.p;
    P.big = big.p;
    P.n_big = nbig.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(ovf.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(nbig.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(cursor.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(rlen.p + n, 0, 4, s));
    DNQ_CUDA(cudaEventRecord(ev[1], s));
    k_vv_arena<<<grid, kWS * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    int hb[2] = {0, 0};
    DNQ_CUDA(cudaMemcpyAsync(&hb[0], nbig.p, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&hb[1], ovf.p, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    if (hb[0] > 0 && !hb[1]) {
        k_vv_big<<<grid, kWS * 32, 0, s>>>(P, hb[0]);
        DNQ_CHECK_LAUNCH();
        DNQ_CUDA(cudaMemcpyAsync(&hb[1], ovf.p, 4, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    DNQ_CUDA(cudaEventRecord(ev[2], s));
    H->vv.nr = H->vv.nc = n;
    H->vv.rowptr.alloc(n + 1, s);
    if (!hb[1]) {
        excl_scan(rlen.p, H->vv.rowptr.p, n + 1, s);
        DNQ_CUDA(cudaMemcpyAsync(&H->vv.nnz, H->vv.rowptr.p + n, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        H->vv.col.alloc(H->vv.nnz, s);
        H->vv.val.alloc(H->vv.nnz, s);
        DNQ_CUDA(cudaEventRecord(ev[3], s));
        k_vv_compact<<<grid, kWS * 32, 0, s>>>(rpos.p, H->vv.rowptr.p, n, acol.p, aval.p,
                                               H->vv.col.p, H->vv.val.p);
        DNQ_CHECK_LAUNCH();
    } else {
        // arena too small: exact two-pass walk
        acol.release();
        aval.release();
        DBuf<u32> cnt(n + 1, s);
        DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
        P.cnt = cnt.p;
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_vv_twopass<false><<<grid, kWS * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
        excl_scan(cnt.p, H->vv.rowptr.p, n + 1, s);
        DNQ_CUDA(cudaMemcpyAsync(&H->vv.nnz, H->vv.rowptr.p + n, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        H->vv.col.alloc(H->vv.nnz, s);
        H->vv.val.alloc(H->vv.nnz, s);
        P.off = H->vv.rowptr.p;
        P.col = H->vv.col.p;
        P.val = H->vv.val.p;
        DNQ_CUDA(cudaEventRecord(ev[3], s));
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_vv_twopass<true><<<grid, kWS * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
    }
    DNQ_CUDA(cudaEventRecord(ev[4], s));
    unsigned long long tests = 0;
    DNQ_CUDA(cudaMemcpyAsync(&tests, nt.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaEventSynchronize(ev[4]));
    H->candidates = (i64)tests;
    H->vv.sorted = false;
    ctx->vv_nnz_hint = std::max<i64>(ctx->vv_nnz_hint, H->vv.nnz);
    float ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    t_ms[0] += ms;                  // string indices
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
    t_ms[1] = 0.0;                  // no count pass
    t_ms[3] = ms;                   // generation pass(es)
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[2], ev[3]));
    t_ms[2] = ms;                   // scan + allocation
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[3], ev[4]));
    t_ms[4] = ms;                   // compaction into CSR (row sort deferred)
    for (auto& e : ev) cudaEventDestroy(e);
}

}  // namespace dnq
