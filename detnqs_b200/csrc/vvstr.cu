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
// Long alpha groups in C are not scanned: each keeps a presence row (one
// bit per beta group) tested against the row's indexed beta singles.
// Each match gets its element exactly as HamEval::compute_elem does
// (ham_eval.cpp:88-147: same integrals, same order of operations) and is
// kept under the policy's rules; for a double |H| equals the heat-bath
// weight |<ij||ab>| bit for bit, so the table cut w >= cut is applied to
// the element.  Results are identical to the candidate walk in gen.cuh.
//
// The single-pass build runs in stages: k_vv_arena walks the rows and
// records their members in warp-private arena chunks (single excitations
// also in a per-warp list), k_vv_singles evaluates the singles one per
// thread, k_vv_eval turns each row's members into entries in place,
// k_vv_big / k_vv_eval_long / k_vv_compact_long handle rows longer than a
// chunk, and k_vv_compact gathers the CSR.  k_vv_twopass is the exact
// fallback when the arena runs out.

#include <algorithm>
#include <type_traits>
#include <memory>
#include <vector>

#include "gen.cuh"
#include "ham.cuh"
#include "prim.cuh"

namespace dnq {

// Part C walk over the short groups: 0 = packed across the groups of a
// round (default), 1 = one group at a time.  Both give the same entries in
// the same order.

namespace {

constexpr int kWS = 8;               // warps per block
constexpr int kBS = 512;   // beta singles of one row kept for the presence rows
constexpr u32 kBigGroup = 2048;      // part C default: search instead of scan above this

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
    DBuf<u32> other32;   // the same in 32 bits (indices of systems with n_orb <= 32)
    DBuf<u32> idx;       // original position in V
    DBuf<u32> gid;       // group number of every sorted position
    DBuf<u32> gstart;    // first sorted position of every group, then n
    i64 ngroups = 0;
    DBuf<ulonglong2> slots;
    u64 mask = 0;
    // Presence rows (alpha index only): one bit per beta group for every
    // alpha group longer than pres_min; prow[group] = its row or ~0u.
    DBuf<u32> prow;
    DBuf<uint2> pres;            // {bits, set bits in the row's earlier words}
    u32 pres_words = 0;
    u32 pres_min = 0xffffffffu;
    // Per group: the part C tests of a row whose string is the group's, when
    // it walks the groups of its singles (scanned members, groups tested by
    // presence rows, groups binary-searched, singles that are groups).
    DBuf<uint4> cost;
    DBuf<u64> ks64;          // sorted keys between the two phases of the build
    DBuf<ulonglong2> ks;
    // Per group: the group of each single excitation of its string (~0u:
    // not a string of the index), in the order of the part C walk (over the
    // occupied orbitals, then the virtual ones), nbr_stride() entries per
    // group.  Null when it would pass kNbrBytes.
    DBuf<u32> nbr;
    StrMapView view() const { return StrMapView{slots.p, mask}; }
};

__global__ void k_keys_by(const u64* V, i64 n, int major, ulonglong2* k, u32* id) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = V[2 * t], b = V[2 * t + 1];
        k[t] = major == 0 ? make_ulonglong2(a, b) : make_ulonglong2(b, a);
        id[t] = (u32)t;
    }
}

// dup (optional) is set when two sorted keys are equal: a determinant listed
// twice.
__global__ void k_split_sorted(const ulonglong2* k, i64 n, u64* other, unsigned* head, u32* dup) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        other[t] = k[t].y;
        head[t] = (t == 0 || k[t].x != k[t - 1].x) ? 1u : 0u;
        if (dup && t > 0 && k[t].x == k[t - 1].x && k[t].y == k[t - 1].y) *dup = 1u;
    }
}

// Start position of every group and n after the last; gid arrives as the
// inclusive scan of the head flags and leaves as the group number of every
// position.
__global__ void k_group_starts(const unsigned* head, u32* gid, i64 n, u32* gstart, u32* ngroups) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 g = gid[t] - 1;
        gid[t] = g;
        if (head[t]) gstart[g] = (u32)t;
        if (t == n - 1) {
            gstart[g + 1] = (u32)n;
            if (ngroups) *ngroups = g + 1;
        }
    }
}

// Group lengths by floor(log2(len - 1)) (len >= 2): the groups longer than
// 2^j are the counts of bins j and up.
__global__ void k_len_hist(const u32* gstart, const u32* ngroups, i64 nmax, u32* hist) {
    __shared__ u32 h[32];
    if (threadIdx.x < 32) h[threadIdx.x] = 0;
    __syncthreads();
    const i64 G = *ngroups;
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < G && g < nmax;
         g += (i64)gridDim.x * blockDim.x) {
        const u32 len = gstart[g + 1] - gstart[g];
        if (len >= 2) atomicAdd(&h[31 - __clz(len - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// Strings of at most 32 orbitals: one 64-bit key (group string << 32 | companion).
__global__ void k_keys_by64(const u64* V, i64 n, int major, u64* k, u32* id) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = V[2 * t], b = V[2 * t + 1];
        k[t] = major == 0 ? (a << 32) | b : (b << 32) | a;
        id[t] = (u32)t;
    }
}

__global__ void k_split_sorted64(const u64* k, i64 n, u64* other, u32* other32, unsigned* head,
                                 u32* dup) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        other[t] = k[t] & 0xffffffffull;
        other32[t] = (u32)k[t];
        head[t] = (t == 0 || (k[t] >> 32) != (k[t - 1] >> 32)) ? 1u : 0u;
        if (dup && t > 0 && k[t] == k[t - 1]) *dup = 1u;
    }
}

// Group string of sorted position t, for either key layout.
struct Key128 {
    const ulonglong2* k;
    __device__ __forceinline__ u64 operator()(i64 t) const { return k[t].x; }
};
struct Key64 {
    const u64* k;
    __device__ __forceinline__ u64 operator()(i64 t) const { return k[t] >> 32; }
};

// Insert one slot per group: (string, start << 32 | len).
template <class K>
__global__ void k_group_insert(K k, const u32* gstart, i64 ngroups, i64 n, ulonglong2* slots,
                               u64 mask) {
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < ngroups;
         g += (i64)gridDim.x * blockDim.x) {
        const i64 t = gstart[g];
        const i64 e = g + 1 < ngroups ? (i64)gstart[g + 1] : n;
        const u64 key = k(t);
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

// major 0: groups by alpha (companion beta); major 1: groups by beta.  With
// n_orb <= 32 the sort runs on 64-bit keys over 32 + n_orb bits, and the
// 32-bit companion strings of the scans come out of the same pass.
// What the host reads of an index after its first phase: the group count,
// the group lengths by floor(log2(len - 1)), and whether a determinant is
// listed twice.
struct IndexProbe {
    u32 ngroups;
    u32 dup;
    u32 hist[32];
};

// First phase of a string index (no host synchronisation): sorted keys,
// companions, group numbers and starts; the probe is filled on the device.
// The sorted keys stay in X until str_index_finish.
void str_index_begin(StrIndex& X, const u64* V, i64 n, int major, int n_orb, IndexProbe* probe,
                     cudaStream_t s) {
    const bool narrow = n_orb <= 32;
    DBuf<ulonglong2> k;
    DBuf<u64> k64;
    DBuf<u32> id(n, s);
    X.idx.alloc(n, s);
    X.other.alloc(n, s);
    DBuf<unsigned> head(n, s);
    u32* dup = major == 0 ? &probe->dup : nullptr;
    if (narrow) {
        k64.alloc(n, s);
        X.ks64.alloc(n, s);
        X.other32.alloc(n, s);
        k_keys_by64<<<gsz(n), 256, 0, s>>>(V, n, major, k64.p, id.p);
        DNQ_CHECK_LAUNCH();
        const int bits[1] = {32 + n_orb};
        prim::radix_sort<u64, u32>(k64.p, X.ks64.p, id.p, X.idx.p, n, bits, s);
        k_split_sorted64<<<gsz(n), 256, 0, s>>>(X.ks64.p, n, X.other.p, X.other32.p, head.p, dup);
        DNQ_CHECK_LAUNCH();
    } else {
        k.alloc(n, s);
        X.ks.alloc(n, s);
        k_keys_by<<<gsz(n), 256, 0, s>>>(V, n, major, k.p, id.p);
        DNQ_CHECK_LAUNCH();
        const int bits[2] = {n_orb, n_orb};
        prim::radix_sort<ulonglong2, u32>(k.p, X.ks.p, id.p, X.idx.p, n, bits, s);
        k_split_sorted<<<gsz(n), 256, 0, s>>>(X.ks.p, n, X.other.p, head.p, dup);
        DNQ_CHECK_LAUNCH();
    }
    X.gid.alloc(n, s);
    X.gstart.alloc(n + 1, s);
    prim::scan_inclusive<unsigned, u32>(head.p, X.gid.p, n, s);
    k_group_starts<<<gsz(n), 256, 0, s>>>(head.p, X.gid.p, n, X.gstart.p, &probe->ngroups);
    DNQ_CHECK_LAUNCH();
    k_len_hist<<<gsz(n), 256, 0, s>>>(X.gstart.p, &probe->ngroups, n, probe->hist);
    DNQ_CHECK_LAUNCH();
}

// Second phase, with the group count read: the string -> group hash.
void str_index_finish(StrIndex& X, i64 n, i64 ngroups, cudaStream_t s) {
    X.ngroups = ngroups;
    u64 cap = 1024;
    while (cap < (u64)(2 * ngroups)) cap <<= 1;
    X.mask = cap - 1;
    X.slots.alloc(cap, s);
    DNQ_CUDA(cudaMemsetAsync(X.slots.p, 0xff, cap * sizeof(ulonglong2), s));
    if (X.ks64.p)
        k_group_insert<<<gsz(ngroups), 256, 0, s>>>(Key64{X.ks64.p}, X.gstart.p, ngroups, n,
                                                    X.slots.p, X.mask);
    else
        k_group_insert<<<gsz(ngroups), 256, 0, s>>>(Key128{X.ks.p}, X.gstart.p, ngroups, n,
                                                    X.slots.p, X.mask);
    DNQ_CHECK_LAUNCH();
    X.ks64.release();
    X.ks.release();
}

// major 0: groups by alpha (companion beta); major 1: groups by beta.  With
// n_orb <= 32 the sort runs on 64-bit keys over 32 + n_orb bits, and the
// 32-bit companion strings of the scans come out of the same pass.
void build_str_index(StrIndex& X, const u64* V, i64 n, int major, int n_orb, cudaStream_t s) {
    if (n == 0) {   // no groups: an empty table
        X.ngroups = 0;
        X.mask = 1023;
        X.slots.alloc(1024, s);
        DNQ_CUDA(cudaMemsetAsync(X.slots.p, 0xff, 1024 * sizeof(ulonglong2), s));
        return;
    }
    DBuf<IndexProbe> probe(1, s);
    DNQ_CUDA(cudaMemsetAsync(probe.p, 0, sizeof(IndexProbe), s));
    str_index_begin(X, V, n, major, n_orb, probe.p, s);
    u32 ng = 0;
    DNQ_CUDA(cudaMemcpyAsync(&ng, &probe.p->ngroups, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    str_index_finish(X, n, ng, s);
}

__global__ void k_narrow(const u64* x, i64 n, u32* y) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        y[t] = (u32)x[t];
}

// 32-bit companion strings for scans (every string below orbital 32).
void narrow_index(StrIndex& X, i64 n, cudaStream_t s) {
    if (n == 0 || X.other32.n == (size_t)n) return;
    X.other32.alloc(n, s);
    k_narrow<<<gsz(n), 256, 0, s>>>(X.other.p, n, X.other32.p);
    DNQ_CHECK_LAUNCH();
}

constexpr u32 kPresMin = 128;                    // presence rows for alpha groups longer than this
constexpr i64 kNbrBytes = 1ll << 30;             // cap on the neighbour table of one index
// Entries per group of a neighbour table: the most single excitations a
// string of n_orb orbitals has, (n/2) (n - n/2).
__host__ __device__ __forceinline__ i64 nbr_stride(int n_orb) {
    return (i64)(n_orb / 2) * (n_orb - n_orb / 2);
}
constexpr i64 kPresBytes = 256ll << 20;          // cap on the presence rows of one index

__global__ void k_long_groups(const u32* gstart, i64 ngroups, i64 n, u32 thr, u32* flag,
                              unsigned long long* count) {
    u32 c = 0;
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < ngroups;
         g += (i64)gridDim.x * blockDim.x) {
        const i64 e = g + 1 < ngroups ? (i64)gstart[g + 1] : n;
        const u32 f = (e - (i64)gstart[g]) > (i64)thr ? 1u : 0u;
        if (flag) flag[g] = f;
        c += f;
    }
    if (count && c) atomicAdd(count, (unsigned long long)c);
}

__global__ void k_prow(const u32* flag, const u32* rank, i64 ngroups, u32* prow) {
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < ngroups;
         g += (i64)gridDim.x * blockDim.x)
        prow[g] = flag[g] ? rank[g] : 0xffffffffu;
}

// One bit per member of every long alpha group: its beta string's group.
__global__ void k_pres_fill(const u32* a_gid, const u64* a_other, const u32* prow, i64 n,
                            StrMapView bmap, const u32* b_gid, u32 words, uint2* pres) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 r = prow[a_gid[t]];
        if (r == 0xffffffffu) continue;
        u32 st = 0, ln = 0;
        if (!bmap.find(a_other[t], st, ln)) continue;   // every member's beta is indexed
        const u32 bid = b_gid[st];
        atomicOr(&pres[(i64)r * words + (bid >> 5)].x, 1u << (bid & 31));
    }
}

// .y of every word: set bits in the earlier words of its row (one warp per row).
__global__ void k_pres_rank(uint2* pres, i64 rows, u32 words) {
    const int lane = threadIdx.x & 31;
    for (i64 r = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5; r < rows;
         r += ((i64)gridDim.x * blockDim.x) >> 5) {
        uint2* w = pres + r * words;
        u32 carry = 0;
        for (u32 w0 = 0; w0 < words; w0 += 32) {
            const u32 k = w0 + lane;
            const u32 c = k < words ? (u32)__popc(w[k].x) : 0u;
            u32 incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += v;
            }
            if (k < words) w[k].y = carry + incl - c;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
}

void presence_rows(StrIndex& A, const StrIndex& B, i64 n, u32 thr, unsigned long long nl,
                   cudaStream_t s);

// Presence rows of the groups of index A over the groups of index B (alpha
// over beta, and beta over alpha for the beta-major walk).  The threshold
// starts at kPresMin and doubles until the rows fit kPresBytes.
void build_presence(StrIndex& A, const StrIndex& B, i64 n, cudaStream_t s) {
    if (n == 0 || A.ngroups == 0) return;
    const u32 words = (u32)((B.ngroups + 31) / 32);
    DBuf<unsigned long long> cnt(1, s);
    u32 thr = kPresMin;
    unsigned long long nl = 0;
    for (;;) {
        DNQ_CUDA(cudaMemsetAsync(cnt.p, 0, 8, s));
        k_long_groups<<<gsz(A.ngroups), 256, 0, s>>>(A.gstart.p, A.ngroups, n, thr, nullptr,
                                                     cnt.p);
        DNQ_CHECK_LAUNCH();
        DNQ_CUDA(cudaMemcpyAsync(&nl, cnt.p, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        if ((i64)nl * words * 8 <= kPresBytes || (i64)thr >= n) break;
        thr *= 2;
    }
    presence_rows(A, B, n, thr, nl, s);
}

// The same threshold from the group-length histogram of A (str_index_begin):
// no host synchronisation.
void build_presence_hist(StrIndex& A, const StrIndex& B, i64 n, const u32* hist,
                         cudaStream_t s) {
    if (n == 0 || A.ngroups == 0) return;
    const u32 words = (u32)((B.ngroups + 31) / 32);
    auto longer = [&](u32 t) {   // groups longer than t = 2^j: bins j and up
        unsigned long long c = 0;
        for (int b = 31 - __builtin_clz(t); b < 32; ++b) c += hist[b];
        return c;
    };
    u32 thr = kPresMin;
    unsigned long long nl = longer(thr);
    while (!((i64)nl * words * 8 <= kPresBytes || (i64)thr >= n)) {
        thr *= 2;
        nl = longer(thr);
    }
    presence_rows(A, B, n, thr, nl, s);
}

// The presence rows of the nl groups of A longer than thr.
void presence_rows(StrIndex& A, const StrIndex& B, i64 n, u32 thr, unsigned long long nl,
                   cudaStream_t s) {
    const u32 words = (u32)((B.ngroups + 31) / 32);
    if (nl == 0 || (i64)nl * words * 8 > kPresBytes) return;
    DBuf<u32> flag(A.ngroups, s), rank(A.ngroups, s);
    k_long_groups<<<gsz(A.ngroups), 256, 0, s>>>(A.gstart.p, A.ngroups, n, thr, flag.p, nullptr);
    DNQ_CHECK_LAUNCH();
    prim::scan<u32, u32, false>(flag.p, rank.p, A.ngroups, s);
    A.prow.alloc(A.ngroups, s);
    k_prow<<<gsz(A.ngroups), 256, 0, s>>>(flag.p, rank.p, A.ngroups, A.prow.p);
    DNQ_CHECK_LAUNCH();
    A.pres.alloc((size_t)nl * words, s);
    DNQ_CUDA(cudaMemsetAsync(A.pres.p, 0, (size_t)nl * words * sizeof(uint2), s));
    k_pres_fill<<<gsz(n), 256, 0, s>>>(A.gid.p, A.other.p, A.prow.p, n, B.view(), B.gid.p,
                                       words, A.pres.p);
    DNQ_CHECK_LAUNCH();
    k_pres_rank<<<gsz((i64)nl * 32), 256, 0, s>>>(A.pres.p, (i64)nl, words);
    DNQ_CHECK_LAUNCH();
    A.pres_words = words;
    A.pres_min = thr;
}

__device__ __forceinline__ i64 tri2(i64 p, i64 q) {
    return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
}
__device__ __forceinline__ double eri(const double* E, int p, int q, int r, int s) {
    return __ldg(&E[tri2(tri2(p, q), tri2(r, s))]);
}

// Part C costs of every group of index X (one warp per group): the walk of
// a row whose X string is the group's looks up the group of each single x'
// of that string and scans it, tests it through presence rows or binary-
// searches it (the same classification as part_c, with the other string's
// single count taken from the first determinant: every string of a space
// has the same electron count).  Writes the neighbour table when nbr is set.
__global__ void k_group_cost(const u64* V, const u32* idx, const u32* gstart, const u32* gid,
                             i64 ngroups, int major, int n_orb, StrMapView xmap, int has_pres,
                             u32 pres_min, u32 big_group, uint4* cost, u32* nbr) {
    __shared__ u8 lists[kWS][128];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u8* occ = lists[w];
    u8* vir = lists[w] + 64;
    const u64 all = low_mask(n_orb);
    const int ny = __popcll(V[1 - major]);
    const int nyv = ny * (n_orb - ny);
    const bool usep = has_pres && nyv <= kBS;
    for (i64 g = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5; g < ngroups;
         g += ((i64)gridDim.x * blockDim.x) >> 5) {
        const u64 x = V[2 * (i64)idx[gstart[g]] + major];
        for (int o = lane; o < n_orb; o += 32) {
            const u64 below = (1ull << o) - 1ull;
            if ((x >> o) & 1ull) occ[__popcll(x & below)] = (u8)o;
            else vir[o - __popcll(x & below)] = (u8)o;
        }
        __syncwarp();
        const int nx = __popcll(x), nvx = __popcll(~x & all), ns = nx * nvx;
        u32 scan = 0, pb = 0, bg = 0, ix = 0;
        for (int i = lane; i < ns; i += 32) {
            u32 gs = 0, gl = 0;
            const bool f = xmap.find(x ^ (1ull << occ[i / nvx]) ^ (1ull << vir[i % nvx]), gs, gl);
            if (nbr) nbr[g * nbr_stride(n_orb) + i] = f ? __ldg(&gid[gs]) : 0xffffffffu;
            if (!f) continue;
            ++ix;
            const bool pbig = usep && gl > pres_min && gl > (u32)nyv;
            if (pbig) ++pb;
            else if (gl > big_group) ++bg;
            else scan += gl;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            scan += __shfl_xor_sync(0xffffffffu, scan, o);
            pb += __shfl_xor_sync(0xffffffffu, pb, o);
            bg += __shfl_xor_sync(0xffffffffu, bg, o);
            ix += __shfl_xor_sync(0xffffffffu, ix, o);
        }
        if (lane == 0) cost[g] = make_uint4(scan, pb, bg, ix);
        __syncwarp();
    }
}

// Part C costs of every group, and its neighbour table when that fits
// kNbrBytes.
void build_group_cost(StrIndex& X, const u64* V, i64 n, int major, int n_orb, cudaStream_t s) {
    if (n == 0 || X.ngroups == 0) return;
    X.cost.alloc(X.ngroups, s);
    const i64 st = nbr_stride(n_orb);
    if (X.ngroups * st * (i64)sizeof(u32) <= kNbrBytes) X.nbr.alloc(X.ngroups * st, s);
    const i64 blocks = std::min<i64>((X.ngroups + kWS - 1) / kWS, 65535);
    k_group_cost<<<(unsigned)blocks, kWS * 32, 0, s>>>(
        V, X.idx.p, X.gstart.p, X.gid.p, X.ngroups, major, n_orb, X.view(), X.pres.p != nullptr,
        X.pres.p ? X.pres_min : 0xffffffffu, kBigGroup, X.cost.p, X.nbr.p);
    DNQ_CHECK_LAUNCH();
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
    const u32* a_other32;   // the same as u32 when n_orb <= 32 (else null)
    const u32* b_other32;
    const double* diag;
    int policy;
    double eps1;
    double cut;             // doubles: keep w >= cut (and > 1e-15)
    const double* psi;
    u32 big_group;          // part C: binary search for groups longer than this
    int c_groupwalk;        // part C: short groups one at a time instead of packed
    // part C presence rows: alpha groups longer than pres_min test the beta
    // singles of the row against one bit per beta group
    const u32* a_gid;       // group number of every alpha-sorted position
    const u32* a_prow;      // presence row of every alpha group (~0u: none)
    const u32* b_gid;       // group number of every beta-sorted position
    const uint2* pres;
    u32 pres_words;
    u32 pres_min;
    // the same for beta groups over the alpha groups (beta-major part C)
    const u32* b_prow;
    const uint2* pres_b;
    u32 pres_words_b;
    u32 pres_min_b;
    const uint4* a_cost;   // part C costs per alpha / beta group (null: alpha-major)
    const uint4* b_cost;
    // neighbour tables (group of every single of a group's string; null: hash
    // lookups) and group starts with n after the last group
    const u32* a_nbr;
    const u32* b_nbr;
    const u32* a_gstart;
    const u32* b_gstart;
};

// Where rows are written.  Single pass: rows appended to warp-private
// chunks of an arena; long rows get exact space in a second walk; the
// two-pass fallback counts, then fills at known offsets.
struct SingleOut {
    double h;
    u32 j;
    u32 keep;
};

struct Arena {
    u32* acol;
    double* aval;
    i64 cap;                          // arena capacity (entries)
    i64 chunk;                        // entries per warp chunk
    i64 restart;                      // longest row restarted in a fresh chunk
    unsigned long long* cursor;       // next free arena entry
    int* overflow;                    // set when the arena is too small
    i64* row_pos;
    u32* row_len;
    u32* big;                         // rows longer than one chunk
    u32* big_len;                     // their member counts
    int* n_big;
    int* next_row;
    const u32* order;                 // walk order of the rows (null: 0, 1, ...)
    unsigned long long* n_test;
    unsigned long long* n_hit;        // members recorded by k_vv_arena (optional)
    // single excitations recorded by k_vv_arena in warp-private slices of
    // sgl_slice entries, evaluated by k_vv_singles one per thread; past its
    // slice a warp leaves them ordinary members
    uint4* sgl;                       // (row, sorted position, kind, 0)
    SingleOut* sres;
    u32* sgl_n;                       // entries used in each warp's slice
    u32 sgl_slice;
    i64 sgl_cap;                      // warps * sgl_slice
    // arena-form output with the FP32 operator copy: k_vv_eval writes the
    // FP32 value of every entry (0 for the diagonal entry) and the FP64
    // diagonal of every row (0 where a row keeps none)
    float* val32;
    double* dg;
    u32* cnt;                         // two-pass fallback
    const i64* off;
    u32* col;
    double* val;
};

// Row sources: one system, or many systems laid end to end (block-diagonal
// global matrix; row g of system s has local row g - row_off[s] and its
// columns are offset by row_off[s]).
struct OneSys {
    VVParams P;
    __device__ __forceinline__ i64 rows() const { return P.n; }
    __device__ __forceinline__ const VVParams& at(i64 g, int& r, u32& base) const {
        r = (int)g;
        base = 0;
        return P;
    }
};

struct ManySys {
    const VVParams* sys;
    const i64* row_off;    // [n_sys + 1]
    int n_sys;
    i64 total;
    __device__ __forceinline__ i64 rows() const { return total; }
    __device__ __forceinline__ const VVParams& at(i64 g, int& r, u32& base) const {
        int lo = 0, hi = n_sys - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&row_off[mid]) <= g) lo = mid; else hi = mid - 1;
        }
        const i64 o = __ldg(&row_off[lo]);
        r = (int)(g - o);
        base = (u32)o;
        return sys[lo];
    }
};

constexpr i64 kChunk = 8192;          // default arena entries per warp chunk
constexpr i64 kChunkLarge = 16384;    // the same for single builds of at least 64 rows per
                                      // walking warp: fewer rows take the long-row kernels,
                                      // for an open-chunk reserve that is small beside them
// row_pos of a long row carries this bit: its slots hold entries and holes
// (column kHole) until k_vv_compact_long gathers them.
constexpr i64 kLongRow = 1ll << 62;
constexpr u32 kHole = 0xffffffffu;

// Warp-collective sinks of one row's entries (columns offset by `base`).
struct CountOut {
    u32 c = 0;
    u32 base = 0;
    __device__ __forceinline__ void put(bool keep, u32, double) {
        c += __popc(__ballot_sync(0xffffffffu, keep));
    }
};

struct ExactOut {
    u32* col;
    double* val;
    i64 w;
    u32 base;
    u32 c = 0;
    __device__ __forceinline__ void put(bool keep, u32 j, double h) {
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const i64 at = w + __popc(m & lanemask_lt());
            col[at] = j + base;
            val[at] = h;
        }
        w += __popc(m);
        c += __popc(m);
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

// Loads of a scan are issued kScanU steps ahead of their tests (every step
// is a dependent global load); the sink sees the kScanU steps' hits, then
// one sync, so a queue holds at most 31 + 32 kScanU members.
constexpr int kScanU = 4;
constexpr int kRing = 32 + 32 * kScanU;

constexpr int kWinW = 128;   // part C: words of group-start bits, a window of 4096 members
struct WarpShared {
    u32 off[32];               // part C: position of member m of a nonempty group is m + off
    u32 tg[32];                // part C: member tag of each nonempty group (alpha hole, particle)
    u32 first[32];             // part C: first member of each nonempty group
    uint2 sw[kWinW];           // part C: per word, bit m set where a nonempty group starts at
                               // member m, and the nonempty groups started before the word
    u8 occa[64], vira[64], occb[64], virb[64];
    u32 bs_id[kBS];            // beta group of each indexed beta single of the row
    u16 bs_hp[kBS];            // its excitation, hole | particle << 8
};

// Members awaiting evaluation in the walks that evaluate as they go.
struct HitRing {
    u32 pos[kRing], tag[kRing];
};

// Occupied and virtual orbital lists of both strings, one lane per orbital.
__device__ __forceinline__ void load_lists(WarpShared& S, u64 a, u64 b, int n_orb) {
    const int lane = threadIdx.x & 31;
    for (int o = lane; o < n_orb; o += 32) {
        const u64 below = (1ull << o) - 1ull;
        if ((a >> o) & 1ull) S.occa[__popcll(a & below)] = (u8)o;
        else S.vira[o - __popcll(a & below)] = (u8)o;
        if ((b >> o) & 1ull) S.occb[__popcll(b & below)] = (u8)o;
        else S.virb[o - __popcll(b & below)] = (u8)o;
    }
    __syncwarp();
}

// A connected member of a row is a (sorted position, tag) pair: the tag's
// low byte is its kind, and for opposite-spin doubles bits 8-15 / 16-23
// hold the alpha hole and particle.  The diagonal is a member of its own
// kind whose position is the row.  Members are found by walk_row and
// turned into elements by eval_hit, in the order found.
// kinds: same beta string, same alpha string, opposite-spin double found
// through the alpha groups (position in the alpha-sorted order, tag with the
// alpha hole and particle), diagonal, a single evaluated ahead (its position
// field is its index in the singles list), opposite-spin double found
// through the beta groups (position in the beta-sorted order, tag with the
// beta hole and particle).  kSingleBit marks a single of kind A or B as the
// walk finds it.
enum : u32 { kHitA = 0, kHitB = 1, kHitC = 2, kHitD = 3, kHitS = 4, kHitC2 = 5 };
constexpr u32 kSingleBit = 0x80;

struct Hit {
    double h;
    u32 j;
    bool keep;
};

__device__ __forceinline__ Hit eval_hit(const VVParams& P, int r, u64 a, u64 b, double psr,
                                        double cut, u32 pos, u32 tag,
                                        const SingleOut* sres = nullptr) {
    Hit e{0.0, 0u, false};
    const u32 kind = tag & 0x7f;
    if (kind == kHitS) {
        const SingleOut o = sres[pos];
        e.h = o.h;
        e.j = o.j;
        e.keep = o.keep != 0;
    } else if (kind == kHitC) {
        const u64 y = __ldg(&P.a_other[pos]);
        const u64 x = b ^ y;
        const int ha = (tag >> 8) & 0xff, pa = tag >> 16;
        const int hb = __ffsll(b & x) - 1, pb = __ffsll(y & x) - 1;
        const double raw = eri(P.E, ha, pa, hb, pb);   // (a i|b j)
        const int perm = occ_between(a, pa, ha) + occ_between(b, pb, hb);
        e.h = (perm & 1) ? -raw : raw;
        e.keep = keep_double(cut, e.h);
        if (e.keep) e.j = __ldg(&P.a_idx[pos]);
    } else if (kind == kHitC2) {
        const u64 y = __ldg(&P.b_other[pos]);   // the member's alpha string
        const u64 x = a ^ y;
        const int hb = (tag >> 8) & 0xff, pb = tag >> 16;
        const int ha = __ffsll(a & x) - 1, pa = __ffsll(y & x) - 1;
        const double raw = eri(P.E, ha, pa, hb, pb);   // (a i|b j)
        const int perm = occ_between(a, pa, ha) + occ_between(b, pb, hb);
        e.h = (perm & 1) ? -raw : raw;
        e.keep = keep_double(cut, e.h);
        if (e.keep) e.j = __ldg(&P.b_idx[pos]);
    } else if (kind == kHitD) {
        e.h = P.diag[r];
        e.keep = fabs(e.h) > kElemThresh;
        e.j = (u32)r;
    } else {
        const bool alpha = kind == kHitA;   // the alpha string moves
        const u64 y = alpha ? __ldg(&P.b_other[pos]) : __ldg(&P.a_other[pos]);
        const u64 x = alpha ? a : b;
        if (__popcll(x ^ y) == 2) {
            e.h = str_single(P, a, b, alpha ? 0 : 1, x, y);
            e.keep = keep_single(P, psr, e.h);
        } else {
            e.h = str_double_same(P, x, y);
            e.keep = keep_double(cut, e.h);
        }
        if (e.keep) e.j = alpha ? __ldg(&P.b_idx[pos]) : __ldg(&P.a_idx[pos]);
    }
    return e;
}

// Scans read the companion strings as W: u32 when every string fits in 32
// orbitals (half the bytes, one xor and popcount per test), else u64.
__device__ __forceinline__ int popc_w(u32 x) { return __popc(x); }
__device__ __forceinline__ int popc_w(u64 x) { return __popcll(x); }
template <class W> __device__ __forceinline__ const W* a_others(const VVParams& P);
template <class W> __device__ __forceinline__ const W* b_others(const VVParams& P);
template <> __device__ __forceinline__ const u64* a_others<u64>(const VVParams& P) {
    return P.a_other;
}
template <> __device__ __forceinline__ const u64* b_others<u64>(const VVParams& P) {
    return P.b_other;
}
template <> __device__ __forceinline__ const u32* a_others<u32>(const VVParams& P) {
    return P.a_other32;
}
template <> __device__ __forceinline__ const u32* b_others<u32>(const VVParams& P) {
    return P.b_other32;
}

// Part C over the short groups of one round of 32 alpha singles, packed:
// the members of all of them are numbered in group order and each step
// tests 32 consecutive members.  The nonempty groups take slots in lane
// order; a bitmap marks the member each slot starts at, with the number of
// slots started before each of its words, so a lane finds its member's slot
// as that count plus the start bits up to its own, minus one.  The bitmap
// covers windows of 32 * kWinW members.
template <class W, class Q>
__device__ __forceinline__ void part_c_packed(Q& q, WarpShared& S, const W* a_other, W b,
                                              unsigned long long& tests, u32 gs, u32 sl, int hh,
                                              int pp, u32 kind) {
    const int lane = threadIdx.x & 31;
    u32 incl = sl;   // inclusive prefix over lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    const u32 total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    const unsigned ne = __ballot_sync(0xffffffffu, sl != 0);
    if (sl != 0) {
        const int slot = __popc(ne & lanemask_lt());
        const u32 pre = incl - sl;   // first member of this lane's group
        S.off[slot] = gs - pre;
        S.tg[slot] = kind | ((u32)hh << 8) | ((u32)pp << 16);
        S.first[slot] = pre;
    }
    const int ns = __popc(ne);
    tests += total;
    for (u32 t0 = 0; t0 < total; t0 += 32 * kScanU) {
        if ((t0 & (32u * kWinW - 1u)) == 0) {   // start bits of the window from t0
            __syncwarp();
            const int nw = (int)min((total - t0 + 31u) >> 5, (u32)kWinW);
            for (int w = lane; w < nw; w += 32) S.sw[w].x = 0u;
            __syncwarp();
            const u32 f = lane < ns ? S.first[lane] : 0xffffffffu;
            if (f >= t0 && f - t0 < 32u * kWinW) atomicOr(&S.sw[(f - t0) >> 5].x, 1u << (f & 31u));
            u32 run = __popc(__ballot_sync(0xffffffffu, f < t0));
            __syncwarp();
            for (int w0 = 0; w0 < nw; w0 += 32) {   // exclusive prefix of the start counts
                const int w = w0 + lane;
                const u32 c = w < nw ? (u32)__popc(S.sw[w].x) : 0u;
                u32 ic = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u32 v = __shfl_up_sync(0xffffffffu, ic, d);
                    if (lane >= d) ic += v;
                }
                if (w < nw) S.sw[w].y = run + ic - c;
                run += __shfl_sync(0xffffffffu, ic, 31);
            }
            __syncwarp();
        }
        const int w0 = (int)((t0 >> 5) & (kWinW - 1));
        u32 at[kScanU];
        int gl[kScanU];
        W y[kScanU];
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
            const u32 m = t0 + 32 * u + lane;
            at[u] = 0;
            gl[u] = 0;
            y[u] = b;   // no hit
            if (m < total) {
                const u32 le = (2u << lane) - 1u;   // lanes up to this one
                const uint2 e = S.sw[w0 + u];
                const int l = (int)(e.y + __popc(e.x & le)) - 1;
                at[u] = m + S.off[l];
                gl[u] = l;
                y[u] = __ldg(&a_other[at[u]]);
            }
        }
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
            if (t0 + 32 * u >= total) break;
            const int l = gl[u];
            q.push(popc_w(b ^ y[u]) == 2, at[u], [&] { return S.tg[l]; });   // tag read on a hit
        }
        q.sync();
    }
    __syncwarp();
}

// Parts A and B: the members of one group [st, st + ln) whose string differs
// from x in 2 or 4 orbitals.
template <class W, class Q>
__device__ __forceinline__ void scan_same(Q& q, const W* other, W x, u32 st, u32 ln, u32 kind) {
    const int lane = threadIdx.x & 31;
    for (u32 t0 = 0; t0 < ln; t0 += 32 * kScanU) {
        W y[kScanU];
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
            const u32 t = t0 + 32 * u + lane;
            y[u] = t < ln ? __ldg(&other[st + t]) : x;
        }
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
            if (t0 + 32 * u >= ln) break;
            const int dd = popc_w(x ^ y[u]);
            q.push_ab(dd == 2 || dd == 4, st + t0 + 32 * u + lane,
                      kind | (dd == 2 ? kSingleBit : 0u));
        }
        q.sync();
    }
}

// i / d and i % d for 0 <= i < 2^12 and 1 <= d <= 64 through the correctly
// rounded reciprocal of d: the product's error (< 2^-11) is far inside the
// 1/(2d) distance of (i + 0.5) / d from an integer, so truncation gives the
// quotient exactly, for a few instructions instead of an integer division.
__device__ __forceinline__ int small_div(int i, float rcp, int d, int& r) {
    const int q = (int)(((float)i + 0.5f) * rcp);
    r = i - q * d;
    return q;
}

// Part C in one direction.  x is the string whose singles x' give the
// groups (alpha-major: x = a, the groups of the alpha index, members
// sorted by their beta strings); y is the other string, and a member is a
// hit when its string differs from y in one orbital pair.  Its tag holds
// the kind and x's hole and particle.  bm selects beta-major; the
// direction's arrays are read from P where they are used (fewer live
// registers than passing them in).  gx and gy are the groups of x and y in
// their indices (~0u: unknown); with the neighbour tables the groups of
// their singles are read from the tables, else looked up by string.
template <class W, class Q>
__device__ __forceinline__ void part_c(const VVParams& P, WarpShared& S, Q& q,
                                       unsigned long long& tests, bool bm, u64 a, u64 b, int na,
                                       int nva, int nb, int nvb, u32 gx, u32 gy) {
    const int lane = threadIdx.x & 31;
    const u64 x = bm ? b : a, y = bm ? a : b;
    const u8* occx = bm ? S.occb : S.occa;
    const u8* virx = bm ? S.virb : S.vira;
    const u8* occy = bm ? S.occa : S.occb;
    const u8* viry = bm ? S.vira : S.virb;
    const int nvx = bm ? nvb : nva, ny = bm ? na : nb, nvy = bm ? nva : nvb;
    const u32 kind = bm ? kHitC2 : kHitC;
    const W* xo = bm ? b_others<W>(P) : a_others<W>(P);
    const uint2* pres = bm ? P.pres_b : P.pres;
    const W yw = (W)y;
    const int nsx = (bm ? nb : na) * nvx;
    const int nyv = ny * nvy;
    const float rvx = __frcp_rn((float)nvx), rvy = __frcp_rn((float)nvy);
    const bool usep = pres != nullptr && nyv <= kBS;
    int nys = -1;   // indexed y singles listed in S (-1: not yet)
    // neighbour-table row of x (its first entry; ~0: none), read one round ahead
    const u32 nrow = (bm ? P.b_nbr : P.a_nbr) && gx != 0xffffffffu
                         ? gx * (u32)nbr_stride(P.n_orb) : 0xffffffffu;
    u32 gnext = nrow != 0xffffffffu && lane < nsx ? __ldg(&(bm ? P.b_nbr : P.a_nbr)[nrow + lane])
                                                  : 0xffffffffu;
    for (int s0 = 0; s0 < nsx; s0 += 32) {
        const int sidx = s0 + lane;
        const u32 gcur = gnext;
        if (nrow != 0xffffffffu && sidx + 32 < nsx)
            gnext = __ldg(&(bm ? P.b_nbr : P.a_nbr)[nrow + sidx + 32]);
        u32 gs = 0, gl = 0, gg = 0xffffffffu;
        int hh = 0, pp = 0;
        if (sidx < nsx) {
            int pi;
            hh = occx[small_div(sidx, rvx, nvx, pi)];
            pp = virx[pi];
            if (nrow != 0xffffffffu) {
                gg = gcur;
                if (gg != 0xffffffffu) {
                    const u32* gst = bm ? P.b_gstart : P.a_gstart;
                    gs = __ldg(&gst[gg]);
                    gl = __ldg(&gst[gg + 1]) - gs;
                }
            } else if (!(bm ? P.bmap : P.amap).find(x ^ (1ull << hh) ^ (1ull << pp), gs, gl)) {
                gl = 0;
            }
        }
        // presence rows for long groups (when the row's y singles fit the
        // warp's list), binary search above big_group otherwise, else a scan
        const bool pbig = usep && gl > (bm ? P.pres_min_b : P.pres_min) && gl > (u32)nyv;
        const bool big = !pbig && gl > P.big_group;
        const bool small = gl != 0 && !pbig && !big;
        const u32 prw =
            pbig ? __ldg(&(bm ? P.b_prow : P.a_prow)[gg != 0xffffffffu
                                                          ? gg
                                                          : __ldg(&(bm ? P.b_gid : P.a_gid)[gs])])
                 : 0u;
        if (!P.c_groupwalk) {
            part_c_packed(q, S, xo, yw, tests, gs, small ? gl : 0u, hh, pp, kind);
        } else {
            // one group at a time: start, length and the x excitation are
            // warp-uniform, members in order 32 per step
            unsigned m = __ballot_sync(0xffffffffu, small);
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1;
                const u32 g0 = __shfl_sync(0xffffffffu, gs, L);
                const u32 gn = __shfl_sync(0xffffffffu, gl, L);
                const u32 tag = kind | ((u32)__shfl_sync(0xffffffffu, hh, L) << 8) |
                                ((u32)__shfl_sync(0xffffffffu, pp, L) << 16);
                tests += gn;
                for (u32 t0 = 0; t0 < gn; t0 += 32 * kScanU) {
                    W w[kScanU];
#pragma unroll
                    for (int u = 0; u < kScanU; ++u) {
                        const u32 t = t0 + 32 * u + lane;
                        w[u] = t < gn ? __ldg(&xo[g0 + t]) : yw;
                    }
#pragma unroll
                    for (int u = 0; u < kScanU; ++u) {
                        if (t0 + 32 * u >= gn) break;
                        q.push(popc_w(yw ^ w[u]) == 2, g0 + t0 + 32 * u + lane, tag);
                    }
                    q.sync();
                }
            }
        }
        unsigned pm = __ballot_sync(0xffffffffu, pbig);
        if (pm && nys < 0) {   // the row's indexed y singles, once per row, in order
            nys = 0;
            for (int q0 = 0; q0 < nyv; q0 += 32) {
                const int qi = q0 + lane;
                bool f = false;
                u32 bid = 0;
                u16 e = 0;
                if (qi < nyv) {
                    int pi;
                    const int hb = occy[small_div(qi, rvy, nvy, pi)], pb = viry[pi];
                    const u32* nbt = bm ? P.a_nbr : P.b_nbr;
                    if (nbt && gy != 0xffffffffu) {
                        bid = __ldg(&nbt[(i64)gy * nbr_stride(P.n_orb) + qi]);
                        f = bid != 0xffffffffu;
                    } else {
                        u32 bst = 0, bln = 0;
                        if ((bm ? P.amap : P.bmap).find(y ^ (1ull << hb) ^ (1ull << pb), bst,
                                                        bln)) {
                            f = true;
                            bid = __ldg(&(bm ? P.a_gid : P.b_gid)[bst]);
                        }
                    }
                    if (f) e = (u16)(hb | (pb << 8));
                }
                const unsigned fm = __ballot_sync(0xffffffffu, f);
                if (f) {
                    const int at = nys + __popc(fm & lanemask_lt());
                    S.bs_id[at] = bid;
                    S.bs_hp[at] = e;
                }
                nys += __popc(fm);
            }
            __syncwarp();
        }
        while (pm) {
            // members of a long group are sorted by their y group: the member
            // with y group bid sits at the number of set bits before bid
            const int L = __ffs(pm) - 1;
            pm &= pm - 1;
            const u32 g0 = __shfl_sync(0xffffffffu, gs, L);
            const u32 tag = kind | ((u32)__shfl_sync(0xffffffffu, hh, L) << 8) |
                            ((u32)__shfl_sync(0xffffffffu, pp, L) << 16);
            const uint2* row =
                pres + (i64)__shfl_sync(0xffffffffu, prw, L) * (bm ? P.pres_words_b : P.pres_words);
            tests += nys;
            for (int q0 = 0; q0 < nys; q0 += 32 * kScanU) {
                uint2 w[kScanU];
                u32 sh[kScanU];
#pragma unroll
                for (int u = 0; u < kScanU; ++u) {
                    const int qi = q0 + 32 * u + lane;
                    w[u] = make_uint2(0u, 0u);
                    sh[u] = 0;
                    if (qi < nys) {
                        const u32 bid = S.bs_id[qi];
                        sh[u] = ~bid & 31u;   // moves the group's bit to bit 31
                        w[u] = __ldg(&row[bid >> 5]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kScanU; ++u) {
                    if (q0 + 32 * u >= nys) break;
                    const u32 lo = w[u].x << sh[u];   // the group's bit and those below
                    q.push((int)lo < 0, g0 + w[u].y + __popc(lo) - 1u, tag);
                }
                q.sync();
            }
        }
        // other large groups: binary-search every y single
        unsigned bigm = __ballot_sync(0xffffffffu, big);
        while (bigm) {
            const int L = __ffs(bigm) - 1;
            bigm &= bigm - 1;
            const u32 g0 = __shfl_sync(0xffffffffu, gs, L);
            const u32 gn = __shfl_sync(0xffffffffu, gl, L);
            const u32 tag = kind | ((u32)__shfl_sync(0xffffffffu, hh, L) << 8) |
                            ((u32)__shfl_sync(0xffffffffu, pp, L) << 16);
            tests += nyv;
            for (int q0 = 0; q0 < nyv; q0 += 32) {
                const int qi = q0 + lane;
                bool hit = false;
                u32 lo = 0;
                if (qi < nyv) {
                    int pi;
                    const int hb = occy[small_div(qi, rvy, nvy, pi)];
                    const int pb = viry[pi];
                    const u64 t = y ^ (1ull << hb) ^ (1ull << pb);
                    lo = g0;
                    u32 hi = g0 + gn;
                    while (lo < hi) {
                        const u32 mid = (lo + hi) >> 1;
                        if (__ldg(&(bm ? P.b_other : P.a_other)[mid]) < t) lo = mid + 1;
                        else hi = mid;
                    }
                    hit = lo < g0 + gn && __ldg(&(bm ? P.b_other : P.a_other)[lo]) == t;
                }
                q.push(hit, lo, tag);
                q.sync();
            }
        }
        __syncwarp();
    }
}

// Part C direction of a row from the costs of its alpha group (ca) and beta
// group (cb) and the single counts of its two strings: beta-major when that
// walk tests fewer members.
__host__ __device__ __forceinline__ bool row_bm(uint4 ca, uint4 cb, int nsa, int nsb) {
    const u64 cost_a = ca.x + (u64)ca.y * cb.w + (u64)ca.z * (u32)nsb;
    const u64 cost_b = cb.x + (u64)cb.y * ca.w + (u64)cb.z * (u32)nsa;
    return cost_b < cost_a;
}

// The members of row r = (a, b) in their fixed order: the diagonal, then
// parts A, B and C.  q.push(hit, position, tag) is warp-collective, once
// per step of 32; q.sync() follows every group of at most kScanU steps.
template <class W, class Q>
__device__ __forceinline__ void walk_row(const VVParams& P, int r, u64 a, u64 b, WarpShared& S,
                                         Q& q, unsigned long long& tests) {
    const int lane = threadIdx.x & 31;
    const W* ao = a_others<W>(P);
    const W aw = (W)a, bw = (W)b;
    const u64 all = low_mask(P.n_orb);
    q.push(lane == 0, (u32)r, kHitD);
    // groups of parts A and B, looked up by lanes 0 and 1 side by side
    u32 st = 0, ln = 0;
    if (lane == 0 && !P.bmap.find(b, st, ln)) ln = 0;
    if (lane == 1 && !P.amap.find(a, st, ln)) ln = 0;
    u32 grp = 0xffffffffu;   // lane 0: the row's beta group, lane 1: its alpha group
    if (lane < 2 && ln) grp = __ldg(&(lane == 0 ? P.b_gid : P.a_gid)[st]);
    // ---- part A (same beta string: alpha singles and doubles), then part B
    // (same alpha string: beta singles and doubles), from one call site: the
    // walk's speed depends on its code fitting the instruction cache
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {
        const u32 gst = __shfl_sync(0xffffffffu, st, part);
        const u32 gln = __shfl_sync(0xffffffffu, ln, part);
        tests += gln;
        scan_same(q, part ? ao : b_others<W>(P), part ? bw : aw, gst, gln, part ? kHitB : kHitA);
    }
    // ---- part C: alpha single x beta single.  Either direction finds the
    // same members: the groups of the row's alpha singles a' tested for a
    // beta single of b (alpha-major), or the groups of its beta singles b'
    // tested for an alpha single of a (beta-major).  The row takes the one
    // with fewer tests, from the costs precomputed per group of its two
    // strings (the same rule on every path, so a row's member order does not
    // depend on the path that builds it).
    const int na = __popcll(a), nva = __popcll(~a & all);
    const int nb = __popcll(b), nvb = __popcll(~b & all);
    bool bm = false;
    if (P.a_cost) {   // the costs of the row's two groups (found for parts A and B)
        uint4 c = make_uint4(0u, 0u, 0u, 0u);
        if (lane == 0 && ln) c = __ldg(&P.b_cost[grp]);
        if (lane == 1 && ln) c = __ldg(&P.a_cost[grp]);
        const uint4 cb = make_uint4(__shfl_sync(0xffffffffu, c.x, 0),
                                    __shfl_sync(0xffffffffu, c.y, 0),
                                    __shfl_sync(0xffffffffu, c.z, 0),
                                    __shfl_sync(0xffffffffu, c.w, 0));
        const uint4 ca = make_uint4(__shfl_sync(0xffffffffu, c.x, 1),
                                    __shfl_sync(0xffffffffu, c.y, 1),
                                    __shfl_sync(0xffffffffu, c.z, 1),
                                    __shfl_sync(0xffffffffu, c.w, 1));
        bm = row_bm(ca, cb, na * nva, nb * nvb);
    }
    // one call site for both directions: a second inlined copy of the walk
    // would not fit the instruction cache
    part_c<W>(P, S, q, tests, bm, a, b, na, nva, nb, nvb,
              __shfl_sync(0xffffffffu, grp, bm ? 0 : 1), __shfl_sync(0xffffffffu, grp, bm ? 1 : 0));
}

// A member's tag, given as a value or as a function read only on a hit.
__device__ __forceinline__ u32 tag_value(u32 t) { return t; }
template <class F>
__device__ __forceinline__ auto tag_value(const F& f) -> decltype(f()) {
    return f();
}

// Sink of walk_row that records the members only: position | tag << 32 in
// the value slots [w, end) of an arena chunk (whole 8-byte words, so no
// partial-sector writes); past the end it only counts.
struct HitOut {
    u64* mem;   // the row's first slot in the arena's value array (as u64)
    u32 room;   // slots the row may fill
    uint4* sgl = nullptr;   // this warp's singles slice (null: singles stay members)
    u32* sgn = nullptr;     // its entries used
    u32 sslice = 0;         // its size
    u32 sbase = 0;          // index of its first entry in the list
    u32 row = 0;            // global row, recorded with its singles
    u32 c = 0;              // members found; written while they fit the room
    // The row overflowed its room (c only grows, so once a step does not
    // fit, no later step writes).
    __device__ __forceinline__ bool over() const { return c > room; }
    template <class T>
    __device__ __forceinline__ void push(bool hit, u32 pos, const T& t) {
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (m == 0) return;   // most steps find nothing
        const u32 k = __popc(m);
        if (hit && c + k <= room)
            mem[c + __popc(m & lanemask_lt())] = (u64)pos | ((u64)tag_value(t) << 32);
        c += k;
    }
    // Parts A and B: a single (tag with kSingleBit) goes to the singles list
    // when there is one and it has room.
    __device__ __forceinline__ void push_ab(bool hit, u32 pos, u32 tg) {
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (m == 0) return;
        const u32 k = __popc(m);
        if (c + k <= room) {
            u64 rec = (u64)pos | ((u64)(tg & ~kSingleBit) << 32);
            const bool sg = hit && (tg & kSingleBit) && sgl;
            const unsigned sm = __ballot_sync(0xffffffffu, sg);
            if (sm) {
                const u32 idx = *sgn + __popc(sm & lanemask_lt());
                if (sg && idx < sslice) {
                    sgl[idx] = make_uint4(row, pos, tg & ~kSingleBit, 0u);
                    rec = (u64)(sbase + idx) | ((u64)kHitS << 32);
                }
                *sgn += __popc(sm);
            }
            if (hit) mem[c + __popc(m & lanemask_lt())] = rec;
        }
        c += k;
    }
    __device__ __forceinline__ void sync() {}
};

// Sink of walk_row that evaluates as it goes (the long-row and two-pass
// walks): members queue in shared memory and are evaluated 32 at a time.
template <class Out>
struct QueueEval {
    const VVParams& P;
    int r;
    u64 a, b;
    double psr, cut;
    HitRing& Q;
    Out& out;
    int n = 0, head = 0;   // queued members (warp-uniform)
    template <class T>
    __device__ __forceinline__ void push(bool hit, u32 pos, const T& t) {
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            int k = head + n + __popc(m & lanemask_lt());
            if (k >= kRing) k -= kRing;
            Q.pos[k] = pos;
            Q.tag[k] = tag_value(t) & ~kSingleBit;
        }
        n += __popc(m);
    }
    __device__ __forceinline__ void push_ab(bool hit, u32 pos, u32 t) { push(hit, pos, t); }
    __device__ __forceinline__ void eval(int cnt) {
        const int lane = threadIdx.x & 31;
        Hit e{0.0, 0u, false};
        if (lane < cnt) {
            int k = head + lane;
            if (k >= kRing) k -= kRing;
            e = eval_hit(P, r, a, b, psr, cut, Q.pos[k], Q.tag[k]);
        }
        out.put(e.keep, e.j, e.h);
        head += cnt;
        if (head >= kRing) head -= kRing;
        n -= cnt;
    }
    __device__ __forceinline__ void sync() {
        if (n >= 32) {
            __syncwarp();
            do {
                eval(32);
            } while (n >= 32);
            __syncwarp();
        }
    }
    __device__ __forceinline__ void flush() {
        sync();
        if (n) {
            __syncwarp();
            eval(n);
            __syncwarp();
        }
    }
};

// All entries of row r, evaluated in the walk.
template <class Out>
__device__ void vv_row(const VVParams& P, int r, u64 a, u64 b, double psr, double cut,
                       WarpShared& S, HitRing& ring, Out& out, unsigned long long& tests) {
    QueueEval<Out> q{P, r, a, b, psr, cut, ring, out};
    walk_row<u64>(P, r, a, b, S, q, tests);
    q.flush();
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

// Rows handed to a walking warp at a time: consecutive rows of the walk
// order share their string groups, which then stay in the SM's L1.
constexpr int kRowRun = 4;

// Word type of the scans: u32 / u64 for every row, or PerRowW to pick per
// row (batches mixing systems of at most and of more than 32 orbitals).
struct PerRowW {};
template <class W, class Q>
__device__ __forceinline__ void walk_any(const VVParams& P, int r, u64 a, u64 b, WarpShared& S,
                                         Q& q, unsigned long long& tests) {
    if constexpr (std::is_same<W, PerRowW>::value) {
        if (P.a_other32) walk_row<u32>(P, r, a, b, S, q, tests);
        else walk_row<u64>(P, r, a, b, S, q, tests);
    } else {
        walk_row<W>(P, r, a, b, S, q, tests);
    }
}

// Single pass, first half: each warp appends the members of its rows to
// private chunks of the arena (k_vv_eval turns them into entries in place).
template <class Loc, class W>
__global__ void __launch_bounds__(kWS * 32, 3) k_vv_arena(Loc L, Arena A) {
    __shared__ WarpShared sh[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const i64 nrows = L.rows();
    i64 cpos = 0, cend = 0;
    bool chunked = false;   // the first chunk is taken with the first row
    unsigned long long tests = 0, hits = 0;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint4* slice = A.sgl ? A.sgl + (i64)wid * A.sgl_slice : nullptr;
    u32 sgn = 0;
    int t = 0, t_end = 0;   // this warp's run of rows in the walk order
    for (;;) {
        if (t == t_end) {
            int base = 0;
            if (lane == 0) base = atomicAdd(A.next_row, kRowRun);
            t = __shfl_sync(0xffffffffu, base, 0);
            if (t >= nrows) break;
            t_end = (int)std::min<i64>((i64)t + kRowRun, nrows);
        }
        const int g = A.order ? (int)__ldg(&A.order[t]) : t;
        ++t;
        if (*(volatile int*)A.overflow) continue;
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, P.n_orb);
        const u32 sgn0 = sgn;   // a row that is walked again drops its singles
        if (!chunked) {   // warps that get no row take no chunk
            chunked = true;
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(A.cursor, (unsigned long long)A.chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((i64)base + A.chunk <= A.cap) {
                cpos = (i64)base;
                cend = cpos + A.chunk;
            }
        }
        // every row starts on a 4-slot boundary: the H.psi kernels split a row
        // into slots aligned to its start, so its order of accumulation is
        // then the same on every build
        cpos = std::min<i64>((cpos + 3) & ~3ll, cend);
        for (int attempt = 0; attempt < 2; ++attempt) {
            sgn = sgn0;
            HitOut out{reinterpret_cast<u64*>(A.aval) + cpos, (u32)(cend - cpos), slice, &sgn,
                       A.sgl_slice, (u32)wid * A.sgl_slice, (u32)g};
            unsigned long long tt = 0;
            walk_any<W>(P, r, a, b, S, out, tt);
            if (attempt == 0) {
                tests += tt;
                hits += out.c;
            }
            if (!out.over()) {
                if (lane == 0) {
                    A.row_pos[g] = cpos;
                    A.row_len[g] = out.c;
                }
                cpos += out.c;
                break;
            }
            // Only rows of at most `restart` entries restart in a fresh
            // chunk; longer rows take the exact second pass.  With restart =
            // chunk/4 every retired chunk is at least 3/4 full and the arena
            // never needs more than 4/3 nnz + (warps + 1) chunks (planned
            // batches); single builds restart rows up to a whole chunk and
            // fall back to the exact two-pass build if the arena runs out.
            if ((i64)out.c > A.restart || attempt == 1) {
                if (lane == 0) {
                    A.row_pos[g] = -1;   // k_vv_big places it
                    A.row_len[g] = out.c;
                    A.big[atomicAdd(A.n_big, 1)] = (u32)g;
                }
                sgn = sgn0;
                break;
            }
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(A.cursor, (unsigned long long)A.chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((i64)base + A.chunk > A.cap) {
                if (lane == 0) atomicExch(A.overflow, 1);
                break;
            }
            cpos = (i64)base;
            cend = cpos + A.chunk;
        }
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(A.n_test, tests);
        if (A.n_hit) atomicAdd(A.n_hit, hits);
        if (A.sgl) A.sgl_n[wid] = sgn < A.sgl_slice ? sgn : A.sgl_slice;
    }
}

// Single excitations recorded by the walk, one per thread: their elements
// are chains of dependent additions, which a warp per row would wait on.
template <class Loc>
__global__ void __launch_bounds__(256) k_vv_singles(Loc L, Arena A) {
    if (*(volatile int*)A.overflow) return;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < A.sgl_cap;
         i += (i64)gridDim.x * blockDim.x) {
        if ((u32)(i % A.sgl_slice) >= A.sgl_n[i / A.sgl_slice]) continue;
        const uint4 e = A.sgl[i];
        int r;
        u32 cb;
        const VVParams& P = L.at(e.x, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        const bool alpha = e.z == kHitA;   // the alpha string moves
        const u64 y = alpha ? __ldg(&P.b_other[e.y]) : __ldg(&P.a_other[e.y]);
        const double h = str_single(P, a, b, alpha ? 0 : 1, alpha ? a : b, y);
        SingleOut o;
        o.h = h;
        o.keep = keep_single(P, psr, h) ? 1u : 0u;
        o.j = alpha ? __ldg(&P.b_idx[e.y]) : __ldg(&P.a_idx[e.y]);
        A.sres[i] = o;
    }
}

// Single pass, second half: the members of every arena row become its
// entries, in place and in order (a step reads its 64 members before it
// writes, and writes only at positions below the next step's).  One warp
// per row, all lanes evaluating.
template <class Loc>
__global__ void __launch_bounds__(kWS * 32) k_vv_eval(Loc L, Arena A) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    const i64 nrows = L.rows();
    if (*(volatile int*)A.overflow) return;
    const u64* mem = reinterpret_cast<const u64*>(A.aval);
    for (i64 g = gw; g < nrows; g += nw) {
        const i64 pos = A.row_pos[g];
        if (pos < 0) continue;   // a long row
        const u32 len = A.row_len[g];
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        i64 w = pos;
        for (u32 k0 = 0; k0 < len; k0 += 64) {   // two members per lane in flight
            const u32 k1 = k0 + lane, k2 = k1 + 32;
            const u64 m1 = k1 < len ? mem[pos + k1] : 0ull;
            const u64 m2 = k2 < len ? mem[pos + k2] : 0ull;
            const u32 p1 = (u32)m1, t1 = (u32)(m1 >> 32), p2 = (u32)m2, t2 = (u32)(m2 >> 32);
            Hit e1{0.0, 0u, false}, e2{0.0, 0u, false};
            if (k1 < len) e1 = eval_hit(P, r, a, b, psr, cut, p1, t1, A.sres);
            if (k2 < len) e2 = eval_hit(P, r, a, b, psr, cut, p2, t2, A.sres);
            unsigned m = __ballot_sync(0xffffffffu, e1.keep);
            if (e1.keep) {
                const i64 at = w + __popc(m & lanemask_lt());
                A.acol[at] = e1.j + cb;
                A.aval[at] = e1.h;
                // member 0 is the diagonal (the walk records it first)
                if (A.val32) A.val32[at] = k1 == 0 ? 0.0f : (float)e1.h;
            }
            if (A.dg && k1 == 0) A.dg[g] = e1.keep ? e1.h : 0.0;
            w += __popc(m);
            m = __ballot_sync(0xffffffffu, e2.keep);
            if (e2.keep) {
                const i64 at = w + __popc(m & lanemask_lt());
                A.acol[at] = e2.j + cb;
                A.aval[at] = e2.h;
                if (A.val32) A.val32[at] = (float)e2.h;
            }
            w += __popc(m);
        }
        if (lane == 0) A.row_len[g] = (u32)(w - pos);
        __syncwarp();
    }
}

// Rows longer than a chunk: exact contiguous space and a second walk that
// records their members there (one warp per row; the walk is cheap next to
// the evaluation, which k_vv_eval_long spreads over the whole grid).  The
// count of such rows is read on the device so the launch can sit in a graph.
template <class Loc, class W>
__global__ void __launch_bounds__(kWS * 32) k_vv_big(Loc L, Arena A) {
    __shared__ WarpShared sh[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int nbig = *A.n_big;
    if (*(volatile int*)A.overflow) return;
    for (int i = gw; i < nbig; i += nw) {
        const int g = (int)A.big[i];
        const u32 len = A.row_len[g];
        unsigned long long base = 0;   // 4-slot multiples keep every start aligned
        if (lane == 0) base = atomicAdd(A.cursor, (unsigned long long)((len + 3u) & ~3u));
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((i64)base + len > A.cap) {
            if (lane == 0) atomicExch(A.overflow, 1);
            continue;
        }
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, P.n_orb);
        HitOut out{reinterpret_cast<u64*>(A.aval) + base, (u32)len};
        unsigned long long tt = 0;
        walk_any<W>(P, r, a, b, S, out, tt);
        if (lane == 0) {
            A.row_pos[g] = (i64)base | kLongRow;
            A.big_len[i] = len;
            A.row_len[g] = 0;   // entries kept, summed by k_vv_eval_long
        }
        __syncwarp();
    }
}

// The members of the long rows become entries in place, 64 per warp step
// over the whole grid; a dropped member leaves a hole.  The 64-member units
// of all long rows are dealt round-robin to the warps as one sequence (unit
// u of row i goes to warp (units before row i + u) mod warps).  Kept counts
// are summed into row_len.
template <class Loc>
__global__ void __launch_bounds__(kWS * 32) k_vv_eval_long(Loc L, Arena A) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    const int nbig = *A.n_big;
    if (*(volatile int*)A.overflow) return;
    const u64* mem = reinterpret_cast<const u64*>(A.aval);
    i64 off = 0;   // units of the rows before row i, mod nw
    for (int i = 0; i < nbig; ++i) {
        const int g = (int)A.big[i];
        const i64 len = A.big_len[i];
        const i64 units = (len + 63) / 64;
        const i64 u0 = (gw - off + nw) % nw;   // this warp's first unit of row i
        off = (off + units) % nw;
        if (u0 >= units) continue;
        const i64 pos = A.row_pos[g] & ~kLongRow;
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        u32 kept = 0;
        for (i64 k0 = u0 * 64; k0 < len; k0 += nw * 64) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const i64 k = k0 + 32 * h + lane;
                bool keep = false;
                if (k < len) {
                    const u64 m = mem[pos + k];
                    const Hit e = eval_hit(P, r, a, b, psr, cut, (u32)m, (u32)(m >> 32));
                    keep = e.keep;
                    A.acol[pos + k] = e.keep ? e.j + cb : kHole;
                    A.aval[pos + k] = e.h;
                }
                kept += __popc(__ballot_sync(0xffffffffu, keep));
            }
        }
        if (lane == 0 && kept) atomicAdd(&A.row_len[g], kept);
    }
}

// Ordered gather of the long rows (block per row): holes dropped.
__global__ void __launch_bounds__(256) k_vv_compact_long(const u32* big, const u32* big_len,
                                                         const int* n_big, const i64* row_pos,
                                                         const i64* rowptr, i64 n,
                                                         const u32* acol, const double* aval,
                                                         u32* col, double* val, i64 cap,
                                                         float* val32 = nullptr,
                                                         double* dg = nullptr) {
    __shared__ u32 wsum[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (rowptr[n] > cap) return;   // a stale plan (k_vv_compact raises the flag)
    const int nbig = *n_big;
    for (int i = blockIdx.x; i < nbig; i += gridDim.x) {
        const u32 g = big[i];
        const i64 src = row_pos[g] & ~kLongRow, dst = rowptr[g];
        const i64 len = big_len[i];
        if (val32 && threadIdx.x == 0) dg[g] = 0.0;   // set below when the row keeps it
        __syncthreads();
        i64 carry = 0;
        for (i64 t0 = 0; t0 < len; t0 += 256) {
            const i64 t = t0 + threadIdx.x;
            const u32 c = t < len ? acol[src + t] : kHole;
            const bool keep = c != kHole;
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) wsum[wid] = __popc(m);
            __syncthreads();
            u32 before = 0, total = 0;
            for (int w = 0; w < 8; ++w) {
                if (w < wid) before += wsum[w];
                total += wsum[w];
            }
            if (keep) {
                const i64 o = carry + before + __popc(m & lanemask_lt());
                const double v = aval[src + t];
                col[dst + o] = c;
                val[dst + o] = v;
                if (val32) {
                    const bool diag = o == 0 && c == g;
                    val32[dst + o] = diag ? 0.0f : (float)v;
                    if (diag) dg[g] = v;
                }
            }
            carry += total;
            __syncthreads();
        }
    }
}

// Gather the rows from the arena into a standard CSR; rows past `cap`
// entries (a stale plan) are not written and raise `*bad`.
// With val32, also the FP32 operator copy: FP32 values with the diagonal
// entry (a row's first entry when kept: the walk records it first) moved to
// dg in FP64, 0 where a row has none.
__global__ void k_vv_compact(const i64* row_pos, const i64* rowptr, i64 n, const u32* acol,
                             const double* aval, u32* col, double* val, i64 cap, int* bad,
                             float* val32 = nullptr, double* dg = nullptr) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    if (rowptr[n] > cap) {
        if (gw == 0 && lane == 0) atomicExch(bad, 1);
        return;
    }
    for (i64 r = gw; r < n; r += nw) {
        const i64 src = row_pos[r], dst = rowptr[r], len = rowptr[r + 1] - dst;
        if (src & kLongRow) continue;   // k_vv_compact_long
        if (val32 && lane == 0) dg[r] = (len > 0 && acol[src] == (u32)r) ? aval[src] : 0.0;
        for (i64 t0 = 0; t0 < len; t0 += 128) {   // four loads per lane before the stores
            u32 c[4];
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const i64 t = t0 + 32 * u + lane;
                if (t < len) {
                    c[u] = acol[src + t];
                    v[u] = aval[src + t];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const i64 t = t0 + 32 * u + lane;
                if (t < len) {
                    col[dst + t] = c[u];
                    val[dst + t] = v[u];
                    if (val32) val32[dst + t] = (t == 0 && c[u] == (u32)r) ? 0.0f : (float)v[u];
                }
            }
        }
    }
}

// Arena form: the long rows compacted in place (block per row, in order; a
// tile is read before any of it is written, and writes land below the next
// tile), with the FP32 copy and the diagonal when val32 is set.
__global__ void __launch_bounds__(256) k_vv_long_inplace(const u32* big, const u32* big_len,
                                                         const int* n_big, const i64* row_pos,
                                                         u32* acol, double* aval, float* val32,
                                                         double* dg) {
    __shared__ u32 wsum[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nbig = *n_big;
    for (int i = blockIdx.x; i < nbig; i += gridDim.x) {
        const u32 g = big[i];
        const i64 base = row_pos[g] & ~kLongRow;
        const i64 len = big_len[i];
        if (val32 && threadIdx.x == 0) dg[g] = 0.0;   // set below when the row keeps it
        __syncthreads();
        i64 carry = 0;
        for (i64 t0 = 0; t0 < len; t0 += 256) {
            const i64 t = t0 + threadIdx.x;
            const u32 c = t < len ? acol[base + t] : kHole;
            const double v = t < len ? aval[base + t] : 0.0;
            const bool keep = c != kHole;
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) wsum[wid] = __popc(m);
            __syncthreads();   // the tile is read
            u32 before = 0, total = 0;
            for (int w = 0; w < 8; ++w) {
                if (w < wid) before += wsum[w];
                total += wsum[w];
            }
            if (keep) {
                const i64 o = carry + before + __popc(m & lanemask_lt());
                acol[base + o] = c;
                aval[base + o] = v;
                if (val32) {
                    const bool diag = o == 0 && c == g;
                    val32[base + o] = diag ? 0.0f : (float)v;
                    if (diag) dg[g] = v;
                }
            }
            carry += total;
            __syncthreads();
        }
    }
}

// Arena form: start and end of every row, and the entry count.
__global__ void k_arena_rows(const i64* row_pos, const u32* row_len, i64 n, i64* start, i64* end,
                             unsigned long long* nnz) {
    unsigned long long c = 0;
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < n;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 b = row_pos[r] & ~kLongRow;
        start[r] = b;
        end[r] = b + row_len[r];
        c += row_len[r];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(nnz, c);
}

// Standard form from arena form: row r moves from [rs[r], re[r]) to
// [rp[r], rp[r + 1]), in order (warp per row).
__global__ void k_row_len(const i64* rs, const i64* re, i64 n, i64* len) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r <= n;
         r += (i64)gridDim.x * blockDim.x)
        len[r] = r < n ? re[r] - rs[r] : 0;
}

__global__ void k_gather_rows(const i64* rs, const i64* re, const i64* rp, i64 n, const u32* col,
                              const double* val, const float* val32, u32* col2, double* val2,
                              float* val32_2) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    for (i64 r = gw; r < n; r += nw) {
        const i64 src = rs[r], dst = rp[r], len = re[r] - src;
        for (i64 t = lane; t < len; t += 32) {
            col2[dst + t] = col[src + t];
            val2[dst + t] = val[src + t];
            if (val32_2) val32_2[dst + t] = val32[src + t];
        }
    }
}

// Two-pass fallback (arena too small): count, then exact fill.
template <class Loc, bool FILL>
__global__ void __launch_bounds__(kWS * 32) k_vv_twopass(Loc L, Arena A) {
    __shared__ WarpShared sh[kWS];
    __shared__ HitRing rings[kWS];
    WarpShared& S = sh[threadIdx.x >> 5];
    HitRing& R = rings[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const i64 nrows = L.rows();
    for (;;) {
        const int g = next_row(A.next_row);
        if (g >= nrows) break;
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        u64 a, b;
        double psr, cut;
        row_setup(P, r, a, b, psr, cut);
        load_lists(S, a, b, P.n_orb);
        unsigned long long tt = 0;
        if (!FILL) {
            CountOut out;
            vv_row(P, r, a, b, psr, cut, S, R, out, tt);
            if (lane == 0) A.cnt[g] = out.c;
        } else {
            ExactOut out{A.col, A.val, A.off[g], cb};
            vv_row(P, r, a, b, psr, cut, S, R, out, tt);
        }
        __syncwarp();
    }
}

}  // namespace

void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s);

namespace {
template <class T>
void excl_scan(const T* in, i64* out, i64 n, cudaStream_t s) {
    prim::scan<T, i64, false>(in, out, n, s);
}
}  // namespace

void check_orbitals(const u64* d, i64 n, int n_orb, cudaStream_t s);

// Test options: warp chunk size and arena capacity (0 = automatic).

namespace {

// Arena slots that always suffice for rows of `nnz` members in all built by
// `grid` blocks (see the restart rule of k_vv_arena).
i64 arena_bound(i64 nnz, i64 nrows, int grid, i64 chunk) {
    // members, 1/3 for the ends of retired chunks, up to 3 alignment slots
    // per row (4 with their share of the ends), the warps' open chunks
    return nnz + nnz / 3 + 1 + 4 * nrows + ((i64)grid * kWS + 1) * chunk;
}

template <class Loc>
int vv_grid(int device) {
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vv_arena<Loc, u64>,
                                                           kWS * 32, 0));
    return std::max(1, per_sm) * sm_count(device);
}

// Walk order of a single system's rows: rows walking part C alpha-major in
// the alpha-sorted order, then the beta-major ones in the beta-sorted order,
// so that a run of rows shares its groups.  Built without a host sync.
__global__ void k_row_group(const u32* idx, const u32* gid, i64 n, u32* row_gid) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        row_gid[idx[t]] = gid[t];
}

__global__ void k_row_dir(const u64* V, i64 n, int n_orb, const u32* rga, const u32* rgb,
                          const uint4* a_cost, const uint4* b_cost, u32* dir) {
    const u64 all = low_mask(n_orb);
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < n;
         g += (i64)gridDim.x * blockDim.x) {
        const u64 a = V[2 * g], b = V[2 * g + 1];
        const int nsa = __popcll(a) * __popcll(~a & all), nsb = __popcll(b) * __popcll(~b & all);
        dir[g] = row_bm(a_cost[rga[g]], b_cost[rgb[g]], nsa, nsb) ? 1u : 0u;
    }
}

// flag[t] of sorted position t: its row walks in this direction (want = 0:
// alpha-major, 1: beta-major); flag[n] = 0 so the scan ends with the count.
__global__ void k_dir_flags(const u32* idx, const u32* dir, i64 n, u32 want, u32* flag) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t <= n;
         t += (i64)gridDim.x * blockDim.x)
        flag[t] = t < n && dir[idx[t]] == want ? 1u : 0u;
}

__global__ void k_order_scatter(const u32* a_idx, const u32* fa, const u32* pa, const u32* b_idx,
                                const u32* fb, const u32* pb, i64 n, u32* order) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (fa[t]) order[pa[t]] = a_idx[t];
        if (fb[t]) order[pa[n] + pb[t]] = b_idx[t];
    }
}

void build_row_order(const StrIndex& A, const StrIndex& B, const u64* V, i64 n, int n_orb,
                     DBuf<u32>& order, cudaStream_t s) {
    if (n == 0 || !A.cost.p || !B.cost.p) return;
    DBuf<u32> rga(n, s), rgb(n, s), dir(n, s), fa(n + 1, s), fb(n + 1, s), pa(n + 1, s),
        pb(n + 1, s);
    order.alloc(n, s);
    k_row_group<<<gsz(n), 256, 0, s>>>(A.idx.p, A.gid.p, n, rga.p);
    DNQ_CHECK_LAUNCH();
    k_row_group<<<gsz(n), 256, 0, s>>>(B.idx.p, B.gid.p, n, rgb.p);
    DNQ_CHECK_LAUNCH();
    k_row_dir<<<gsz(n), 256, 0, s>>>(V, n, n_orb, rga.p, rgb.p, A.cost.p, B.cost.p, dir.p);
    DNQ_CHECK_LAUNCH();
    k_dir_flags<<<gsz(n + 1), 256, 0, s>>>(A.idx.p, dir.p, n, 0u, fa.p);
    DNQ_CHECK_LAUNCH();
    k_dir_flags<<<gsz(n + 1), 256, 0, s>>>(B.idx.p, dir.p, n, 1u, fb.p);
    DNQ_CHECK_LAUNCH();
    prim::scan<u32, u32, false>(fa.p, pa.p, n + 1, s);
    prim::scan<u32, u32, false>(fb.p, pb.p, n + 1, s);
    k_order_scatter<<<gsz(n), 256, 0, s>>>(A.idx.p, fa.p, pa.p, B.idx.p, fb.p, pb.p, n, order.p);
    DNQ_CHECK_LAUNCH();
}

// Grid of k_vv_eval: as many blocks as fit (it holds fewer registers than
// the walk, and more warps in flight hide more of its gather latency).
template <class Loc>
int eval_grid(int device) {
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vv_eval<Loc>, kWS * 32, 0));
    return std::max(1, per_sm) * sm_count(device);
}

// scan: 0 = 64-bit strings, 1 = 32-bit, 2 = chosen per row.
template <class Loc>
void launch_walk(int scan, int grid, const Loc& L, const Arena& A, cudaStream_t s) {
    if (scan == 1) k_vv_arena<Loc, u32><<<grid, kWS * 32, 0, s>>>(L, A);
    else if (scan == 2) k_vv_arena<Loc, PerRowW><<<grid, kWS * 32, 0, s>>>(L, A);
    else k_vv_arena<Loc, u64><<<grid, kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
}

template <class Loc>
void launch_big(int scan, int grid, const Loc& L, const Arena& A, cudaStream_t s) {
    if (scan == 1) k_vv_big<Loc, u32><<<grid, kWS * 32, 0, s>>>(L, A);
    else if (scan == 2) k_vv_big<Loc, PerRowW><<<grid, kWS * 32, 0, s>>>(L, A);
    else k_vv_big<Loc, u64><<<grid, kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
}

// Single-pass build of nrows rows of L into M (allocated here).  cap_hint:
// expected nnz (0 = unknown).  Falls back to the exact two-pass walk when
// the arena is too small.  With arena_out, M keeps the rows where the build
// wrote them (arena form: the arena becomes M's storage, no compaction);
// else they are compacted into a standard CSR.  With dg, the build also
// writes M.val32 (the FP32 values, diagonal entries zero) and the FP64
// diagonal into *dg; the two-pass fallback leaves both empty.  Returns the
// number of member tests.
template <class Loc>
i64 run_vv(const Loc& L, i64 nrows, i64 cap_hint, int device, cudaStream_t s, Csr& M,
           const Options& opt, double* t_gen, double* t_scan, double* t_compact,
           i64* hits_out = nullptr, int scan = 0, DBuf<double>* dg = nullptr,
           const u32* order = nullptr, bool arena_out = false) {
    Events<4> ev;
    const int grid = vv_grid<Loc>(device);
    const i64 warps = (i64)grid * kWS;
    size_t freeb = 0, totb = 0;
    DNQ_CUDA(cudaMemGetInfo(&freeb, &totb));
    // chunks of whole 4-slot groups (row starts stay aligned)
    const i64 chunk = opt.arena_chunk > 0 ? ((i64)opt.arena_chunk + 3) & ~3ll
                      : nrows >= 64 * warps             ? kChunkLarge
                                                        : kChunk;
    i64 want = cap_hint > 0 ? cap_hint + cap_hint / 8 : 512 * nrows;
    want += warps * chunk;
    const bool f32_in_build = arena_out && dg;   // k_vv_eval writes the FP32 copy
    const i64 maxfit = (i64)(freeb / 2 / (f32_in_build ? 16 : 12));
    i64 cap = std::max<i64>(std::min(want, maxfit), chunk);
    if (opt.arena_cap > 0) cap = (i64)opt.arena_cap;
    DBuf<int> next(1, s), ovf(1, s), nbig(1, s), bad(1, s);
    DBuf<unsigned long long> nt(1, s), cursor(1, s), nh(1, s);
    // singles list: ~5 per row on heat-bath spaces, in one slice per warp;
    // past its slice a warp evaluates them with their row
    const u32 slice = (u32)std::max<i64>(
        64, std::min<i64>(std::max<i64>(8 * nrows, 1024), i64(64) << 20) / warps);
    const i64 scap = (i64)slice * warps;
    DBuf<uint4> sgl(scap, s);
    DBuf<SingleOut> sres(scap, s);
    DBuf<u32> sgn(warps, s);
    DBuf<u32> acol(cap, s), rlen(nrows + 1, s), big(nrows, s), blen(nrows, s);
    DBuf<double> aval(cap, s);
    DBuf<float> av32;
    if (f32_in_build) {
        av32.alloc(cap, s);
        dg->alloc(nrows, s);
    }
    DBuf<i64> rpos(nrows, s);
    Arena A{};
    A.acol = acol.p;
    A.aval = aval.p;
    A.cap = cap;
    A.chunk = chunk;
    A.restart = chunk;
    A.cursor = cursor.p;
    A.overflow = ovf.p;
    A.row_pos = rpos.p;
    A.row_len = rlen.p;
    A.big = big.p;
    A.big_len = blen.p;
    A.n_big = nbig.p;
    A.next_row = next.p;
    A.order = order;
    A.n_test = nt.p;
    A.n_hit = nh.p;
    A.sgl = sgl.p;
    A.sres = sres.p;
    A.sgl_n = sgn.p;
    A.sgl_slice = slice;
    A.sgl_cap = scap;
    A.val32 = av32.p;
    A.dg = f32_in_build ? dg->p : nullptr;
    DNQ_CUDA(cudaMemsetAsync(nt.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(nh.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(ovf.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(nbig.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(bad.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(cursor.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(rlen.p + nrows, 0, 4, s));
    DNQ_CUDA(cudaEventRecord(ev[0], s));
    launch_walk<Loc>(scan, grid, L, A, s);
    k_vv_singles<Loc><<<grid, 256, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    k_vv_eval<Loc><<<eval_grid<Loc>(device), kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    launch_big<Loc>(scan, grid, L, A, s);
    DNQ_CHECK_LAUNCH();
    k_vv_eval_long<Loc><<<grid, kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    int hov = 0;
    unsigned long long hcur = 0;   // arena slots handed out (chunks and long rows)
    DNQ_CUDA(cudaMemcpyAsync(&hov, ovf.p, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&hcur, cursor.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_CUDA(cudaEventRecord(ev[1], s));
    M.nr = nrows;
    unsigned long long nnz_h = 0;   // arena form: read after the final sync
    DBuf<unsigned long long> nsum;
    if (!hov && arena_out) {
        DNQ_CUDA(cudaEventRecord(ev[2], s));
        k_vv_long_inplace<<<grid, 256, 0, s>>>(big.p, blen.p, nbig.p, rpos.p, acol.p, aval.p,
                                               A.val32, A.dg);
        DNQ_CHECK_LAUNCH();
        M.rowptr.alloc(nrows, s);
        M.rowend.alloc(nrows, s);
        nsum.alloc(1, s);
        DNQ_CUDA(cudaMemsetAsync(nsum.p, 0, 8, s));
        k_arena_rows<<<gsz(nrows), 256, 0, s>>>(rpos.p, rlen.p, nrows, M.rowptr.p, M.rowend.p,
                                                nsum.p);
        DNQ_CHECK_LAUNCH();
        DNQ_CUDA(cudaMemcpyAsync(&nnz_h, nsum.p, 8, cudaMemcpyDeviceToHost, s));
        // Every row lies below the cursor, which stays on a 4-slot boundary.
        // A block that left at least 3/4 of its arena unused (small systems:
        // the open-chunk reserve dominates) keeps only the handed-out prefix,
        // at the same offsets, so its H.psi reads the same slots.
        const i64 used = std::min<i64>((i64)hcur, cap);
        const i64 slot_bytes = f32_in_build ? 16 : 12;
        if (used <= cap / 4 && (cap - used) * slot_bytes >= (64ll << 20)) {
            DBuf<u32> c2(used, s);
            DBuf<double> v2(used, s);
            DNQ_CUDA(cudaMemcpyAsync(c2.p, acol.p, used * sizeof(u32), cudaMemcpyDeviceToDevice, s));
            DNQ_CUDA(cudaMemcpyAsync(v2.p, aval.p, used * sizeof(double), cudaMemcpyDeviceToDevice,
                                     s));
            acol = std::move(c2);
            aval = std::move(v2);
            if (f32_in_build) {
                DBuf<float> f2(used, s);
                DNQ_CUDA(cudaMemcpyAsync(f2.p, av32.p, used * sizeof(float),
                                         cudaMemcpyDeviceToDevice, s));
                av32 = std::move(f2);
            }
        }
        M.col = std::move(acol);
        M.val = std::move(aval);
        if (f32_in_build) M.val32 = std::move(av32);
        M.arena = true;
    } else if (!hov) {
        M.rowptr.alloc(nrows + 1, s);
        excl_scan(rlen.p, M.rowptr.p, nrows + 1, s);
        DNQ_CUDA(cudaMemcpyAsync(&M.nnz, M.rowptr.p + nrows, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        M.col.alloc(M.nnz, s);
        M.val.alloc(M.nnz, s);
        if (dg) {
            M.val32.alloc(M.nnz, s);
            dg->alloc(nrows, s);
        }
        float* v32 = dg ? M.val32.p : nullptr;
        double* dgp = dg ? dg->p : nullptr;
        DNQ_CUDA(cudaEventRecord(ev[2], s));
        k_vv_compact<<<grid, kWS * 32, 0, s>>>(rpos.p, M.rowptr.p, nrows, acol.p, aval.p, M.col.p,
                                               M.val.p, M.nnz, bad.p, v32, dgp);
        DNQ_CHECK_LAUNCH();
        k_vv_compact_long<<<grid, 256, 0, s>>>(big.p, blen.p, nbig.p, rpos.p, M.rowptr.p, nrows,
                                               acol.p, aval.p, M.col.p, M.val.p, M.nnz, v32, dgp);
        DNQ_CHECK_LAUNCH();
    } else {
        acol.release();
        aval.release();
        if (f32_in_build) {   // the two-pass fill leaves the FP32 copy to its first use
            av32.release();
            dg->release();
        }
        M.rowptr.alloc(nrows + 1, s);
        DBuf<u32> cnt(nrows + 1, s);
        DNQ_CUDA(cudaMemsetAsync(cnt.p + nrows, 0, 4, s));
        A.cnt = cnt.p;
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_vv_twopass<Loc, false><<<grid, kWS * 32, 0, s>>>(L, A);
        DNQ_CHECK_LAUNCH();
        excl_scan(cnt.p, M.rowptr.p, nrows + 1, s);
        DNQ_CUDA(cudaMemcpyAsync(&M.nnz, M.rowptr.p + nrows, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        M.col.alloc(M.nnz, s);
        M.val.alloc(M.nnz, s);
        A.off = M.rowptr.p;
        A.col = M.col.p;
        A.val = M.val.p;
        DNQ_CUDA(cudaEventRecord(ev[2], s));
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_vv_twopass<Loc, true><<<grid, kWS * 32, 0, s>>>(L, A);
        DNQ_CHECK_LAUNCH();
    }
    DNQ_CUDA(cudaEventRecord(ev[3], s));
    unsigned long long tests = 0, hits = 0;
    DNQ_CUDA(cudaMemcpyAsync(&tests, nt.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&hits, nh.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaEventSynchronize(ev[3]));
    if (M.arena) M.nnz = (i64)nnz_h;
    if (hits_out) *hits_out = hov ? std::max<i64>(M.nnz, 2 * cap) : (i64)hits;
    M.sorted = false;
    float ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    if (t_gen) *t_gen = ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
    if (t_scan) *t_scan = ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[2], ev[3]));
    if (t_compact) *t_compact = ms;
    return (i64)tests;
}

VVParams make_params(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                     double cut, const double* psi, const double* diag, const StrIndex& A,
                     const StrIndex& B, const Options& opt) {
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
    P.a_other32 = A.other32.p;
    P.b_other32 = B.other32.p;
    P.b_idx = B.idx.p;
    P.diag = diag;
    P.policy = policy;
    P.eps1 = eps1;
    P.cut = cut;
    P.psi = psi;
    P.big_group = kBigGroup;
    P.c_groupwalk = opt.partc_groupwalk;
    P.a_gid = A.gid.p;
    P.a_prow = A.prow.p;
    P.b_gid = B.gid.p;
    P.pres = A.pres.p;
    P.pres_words = A.pres_words;
    P.pres_min = A.pres.p ? A.pres_min : 0xffffffffu;
    P.b_prow = B.prow.p;
    P.pres_b = B.pres.p;
    P.pres_words_b = B.pres_words;
    P.pres_min_b = B.pres.p ? B.pres_min : 0xffffffffu;
    P.a_cost = A.cost.p;
    P.b_cost = B.cost.p;
    P.a_nbr = A.nbr.p;
    P.b_nbr = B.nbr.p;
    P.a_gstart = A.gstart.p;
    P.b_gstart = B.gstart.p;
    return P;
}

}  // namespace

// Standard form of an arena-form block: rows gathered in order into fresh
// arrays of nnz entries (the FP32 copy with them when it is ready).
void ensure_compact(Csr& m, cudaStream_t s) {
    if (!m.arena) return;
    const i64 n = m.nr;
    DBuf<i64> len(n + 1, s), rp(n + 1, s);
    k_row_len<<<gsz(n + 1), 256, 0, s>>>(m.row_start(), m.row_end(), n, len.p);
    DNQ_CHECK_LAUNCH();
    prim::scan<i64, i64, false>(len.p, rp.p, n + 1, s);
    const bool f32 = m.val32.n > 0 && m.f32_ready();
    DBuf<u32> col(m.nnz, s);
    DBuf<double> val(m.nnz, s);
    DBuf<float> v32;
    if (f32) v32.alloc(m.nnz, s);
    int dev = 0;
    DNQ_CUDA(cudaGetDevice(&dev));
    if (n > 0) {
        k_gather_rows<<<sm_count(dev) * 8, 256, 0, s>>>(m.row_start(), m.row_end(), rp.p, n,
                                                        m.col.p, m.val.p,
                                                        f32 ? m.val32.p : nullptr, col.p, val.p,
                                                        v32.p);
        DNQ_CHECK_LAUNCH();
    }
    m.rowptr = std::move(rp);
    m.rowend.release();
    m.col = std::move(col);
    m.val = std::move(val);
    if (f32) m.val32 = std::move(v32);
    else m.val32.release();
    m.arena = false;
}

void launch_check_orbitals(const u64* d, i64 n, int n_orb, unsigned long long* bad,
                           cudaStream_t s);

// H_VV only, from string groups, with dnq_build's input checks folded into
// the string indices' one host synchronisation: every orbital below n_orb,
// no determinant listed twice (equal keys side by side in the sorted alpha
// index), and the group counts and lengths of both indices, read together.
// Computes the diagonal into H->diag.  n > 0.
void build_vv_checked(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, cudaStream_t s, dnq_ham_s* H,
                      double* t_ms) {
    Events<2> tev;
    const cudaEvent_t e0 = tev[0], e1 = tev[1];
    DNQ_CUDA(cudaEventRecord(e0, s));
    DBuf<unsigned long long> bad(1, s);
    DBuf<IndexProbe> probe(2, s);
    DNQ_CUDA(cudaMemsetAsync(bad.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(probe.p, 0, 2 * sizeof(IndexProbe), s));
    launch_check_orbitals(V, n, n_orb, bad.p, s);
    StrIndex A, B;
    str_index_begin(A, V, n, 0, n_orb, probe.p, s);
    str_index_begin(B, V, n, 1, n_orb, probe.p + 1, s);
    unsigned long long hbad = 0;
    IndexProbe hp[2];
    DNQ_CUDA(cudaMemcpyAsync(&hbad, bad.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(hp, probe.p, 2 * sizeof(IndexProbe), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    require(hbad == 0, DNQ_ERR_INVALID, "determinant occupies an orbital index >= n_orb");
    require(hp[0].dup == 0, DNQ_ERR_DUPLICATE,
            "DetMap::from_ordered: duplicate determinant found");
    H->diag.alloc(n, s);
    launch_diag(ctx, V, n, H->diag.p, s);
    str_index_finish(A, n, hp[0].ngroups, s);
    str_index_finish(B, n, hp[1].ngroups, s);
    build_presence_hist(A, B, n, hp[0].hist, s);
    build_presence_hist(B, A, n, hp[1].hist, s);
    build_group_cost(A, V, n, 0, n_orb, s);
    build_group_cost(B, V, n, 1, n_orb, s);
    const bool narrow = n_orb <= 32;
    if (narrow) {
        narrow_index(A, n, s);
        narrow_index(B, n, s);
    }
    DBuf<u32> order;
    build_row_order(A, B, V, n, n_orb, order, s);
    DNQ_CUDA(cudaEventRecord(e1, s));
    OneSys L{make_params(ctx, V, n, n_orb, policy, eps1, cut, psi, H->diag.p, A, B, H->opt)};
    double tg = 0, tsc = 0, tc = 0;
    i64 hits = 0;
    H->candidates =
        run_vv(L, n, ctx->vv_nnz_hint.load(), ctx->device, s, H->vv, H->opt, &tg, &tsc, &tc,
               &hits, narrow ? 1 : 0, H->opt.build_f32 ? &H->diag_op : nullptr, order.p, true);
    H->vv.nc = n;
    const long long want = std::max<long long>(H->vv.nnz, hits);
    long long prev = ctx->vv_nnz_hint.load();
    while (prev < want && !ctx->vv_nnz_hint.compare_exchange_weak(prev, want)) {
    }
    float ms = 0;
    DNQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    t_ms[0] = ms;    // checks, string indices, diagonal
    t_ms[1] = 0.0;   // no count pass
    t_ms[3] = tg;    // generation pass(es)
    t_ms[2] = tsc;   // scan + allocation
    t_ms[4] = tc;    // arena rows (row sort deferred)
}

// H_VV only, from string groups.  V on the device, diag already computed.
// Rows are left in generation order (H->vv.sorted = false); copy-out
// functions sort them on demand.
void build_vv_strings(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, const double* diag, cudaStream_t s,
                      dnq_ham_s* H, double* t_ms) {
    Events<2> tev;
    const cudaEvent_t e0 = tev[0], e1 = tev[1];
    DNQ_CUDA(cudaEventRecord(e0, s));
    StrIndex A, B;
    build_str_index(A, V, n, 0, n_orb, s);
    build_str_index(B, V, n, 1, n_orb, s);
    build_presence(A, B, n, s);
    build_presence(B, A, n, s);
    build_group_cost(A, V, n, 0, n_orb, s);
    build_group_cost(B, V, n, 1, n_orb, s);
    const bool narrow = n_orb <= 32;
    if (narrow) {
        narrow_index(A, n, s);
        narrow_index(B, n, s);
    }
    DBuf<u32> order;
    build_row_order(A, B, V, n, n_orb, order, s);
    DNQ_CUDA(cudaEventRecord(e1, s));
    OneSys L{make_params(ctx, V, n, n_orb, policy, eps1, cut, psi, diag, A, B, H->opt)};
    double tg = 0, tsc = 0, tc = 0;
    i64 hits = 0;
    H->candidates =
        run_vv(L, n, ctx->vv_nnz_hint.load(), ctx->device, s, H->vv, H->opt, &tg, &tsc, &tc,
               &hits, narrow ? 1 : 0, H->opt.build_f32 ? &H->diag_op : nullptr, order.p, true);
    H->vv.nc = n;
    // the arena holds members before they become entries: size by the larger
    const long long want = std::max<long long>(H->vv.nnz, hits);
    long long prev = ctx->vv_nnz_hint.load();   // shared by builds on other threads
    while (prev < want && !ctx->vv_nnz_hint.compare_exchange_weak(prev, want)) {
    }
    float ms = 0;
    DNQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    t_ms[0] += ms;   // string indices
    t_ms[1] = 0.0;   // no count pass
    t_ms[3] = tg;    // generation pass(es)
    t_ms[2] = tsc;   // scan + allocation
    t_ms[4] = tc;    // compaction (row sort deferred)
}

}  // namespace dnq

// ===========================================================================
// Batched engine: many systems in one launch per phase (block-diagonal).
// ===========================================================================

namespace dnq {

void launch_f32_split(const Csr& m, float* val32, double* diag_out, cudaStream_t s);
void spmm_csr(const Csr& m, const float* val32, const double* diag32, const double* X, int ldx,
              int kx, double* Y, int ldy, int precision, int G, int U, void* scratch,
              int dev, cudaStream_t s);
size_t spmm_scratch_bytes(i64 n, int kx, int precision);
void spmv_block_g(const dnq_ham_s* h, const Csr& m, const double* x, double* y, int precision,
                  cudaStream_t s, const float* x32, const float* val32, const double* diag,
                  int G, int device, int U);
void to_f32(const double* x, i64 n, float* o, cudaStream_t s);

namespace {

// <x|H|x> of every global row, each with its own system's tables.
__global__ void k_diag_batch(ManySys L, double* out) {
    for (i64 g = blockIdx.x * (i64)blockDim.x + threadIdx.x; g < L.total;
         g += (i64)gridDim.x * blockDim.x) {
        int r;
        u32 cb;
        const VVParams& P = L.at(g, r, cb);
        out[g] = diag_elem(P.C, P.V[2 * (i64)r], P.V[2 * (i64)r + 1]);
    }
}

__device__ __forceinline__ void tsum_b(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double z = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, z)), __dsub_rn(b, z));
}

struct DDb {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add_prod(double a, double b) {
        const double p = __dmul_rn(a, b);
        const double pe = fma(a, b, -p);
        double s2, e;
        tsum_b(s, p, s2, e);
        s = s2;
        c = __dadd_rn(c, __dadd_rn(e, pe));
    }
    __device__ __forceinline__ void merge(double os, double oc) {
        double s2, e;
        tsum_b(s, os, s2, e);
        s = s2;
        c = __dadd_rn(__dadd_rn(c, oc), e);
    }
};

// One block per system: {x.y, x.x} with Dot2 and eloc = y / x.
__global__ void k_energy_sys(const i64* row_off, const double* x, const double* y, double* eloc,
                             double* e2) {
    const int sy = blockIdx.x;
    const i64 b = row_off[sy], e = row_off[sy + 1];
    DDb num, den;
    for (i64 t = b + threadIdx.x; t < e; t += blockDim.x) {
        const double xv = x[t], yv = y[t];
        num.add_prod(xv, yv);
        den.add_prod(xv, xv);
        eloc[t] = yv / xv;
    }
    for (int o = 16; o; o >>= 1) {
        num.merge(__shfl_xor_sync(0xffffffffu, num.s, o), __shfl_xor_sync(0xffffffffu, num.c, o));
        den.merge(__shfl_xor_sync(0xffffffffu, den.s, o), __shfl_xor_sync(0xffffffffu, den.c, o));
    }
    __shared__ double sh[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = num.s; sh[1][w] = num.c; sh[2][w] = den.s; sh[3][w] = den.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DDb a, c;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a.merge(sh[0][k], sh[1][k]);
            c.merge(sh[2][k], sh[3][k]);
        }
        e2[2 * sy] = a.s + a.c;
        e2[2 * sy + 1] = c.s + c.c;
    }
}

// Same sums for column j = blockIdx.y of row-major X / Y (k columns): the
// block of (system, column) runs k_energy_sys's order on that column, so
// each column's energies equal a single-column apply bit for bit.
// e2[(sy * k + j) * 2 + {0, 1}].
__global__ void k_energy_sys_multi(const i64* row_off, const double* X, const double* Y,
                                   int k, double* eloc, double* e2) {
    const int sy = blockIdx.x, j = blockIdx.y;
    const i64 b = row_off[sy], e = row_off[sy + 1];
    DDb num, den;
    for (i64 t = b + threadIdx.x; t < e; t += blockDim.x) {
        const double xv = X[t * k + j], yv = Y[t * k + j];
        num.add_prod(xv, yv);
        den.add_prod(xv, xv);
        if (eloc) eloc[t * k + j] = yv / xv;
    }
    for (int o = 16; o; o >>= 1) {
        num.merge(__shfl_xor_sync(0xffffffffu, num.s, o), __shfl_xor_sync(0xffffffffu, num.c, o));
        den.merge(__shfl_xor_sync(0xffffffffu, den.s, o), __shfl_xor_sync(0xffffffffu, den.c, o));
    }
    __shared__ double sh[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = num.s; sh[1][w] = num.c; sh[2][w] = den.s; sh[3][w] = den.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DDb a, c;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            a.merge(sh[0][q], sh[1][q]);
            c.merge(sh[2][q], sh[3][q]);
        }
        e2[((i64)sy * k + j) * 2] = a.s + a.c;
        e2[((i64)sy * k + j) * 2 + 1] = c.s + c.c;
    }
}

// After an overflow (or a total past the plan) the row pointers cannot be
// trusted: make the block empty so later kernels stay in bounds, and flag.
// Launched as ONE block, so the decision is read before any entry is zeroed;
// on the good path it returns at once.
__global__ void k_sanitize(i64* rowptr, i64 n, i64 cap, const int* overflow, int* bad) {
    __shared__ int broken;
    if (threadIdx.x == 0) broken = (*overflow != 0) || rowptr[n] > cap || rowptr[n] < 0;
    __syncthreads();
    if (!broken) return;
    if (threadIdx.x == 0) atomicExch(bad, 1);
    __syncthreads();
    for (i64 t = threadIdx.x; t <= n; t += blockDim.x) rowptr[t] = 0;
}

}  // namespace
}  // namespace dnq

struct dnq_batch_s {
    int device = 0;
    int n_sys = 0;
    dnq::Options opt = dnq::default_options();   // this batch's options
    dnq::i64 total = 0;
    std::vector<dnq_ctx_s*> ctx;
    std::vector<dnq::DBuf<dnq::u64>> V;
    std::vector<dnq::StrIndex> A, B;
    std::vector<dnq::i64> row_off_h;
    dnq::DBuf<dnq::i64> row_off;
    dnq::DBuf<dnq::VVParams> sys;
    dnq::DBuf<double> diag, x, y, eloc, e2;
    dnq::DBuf<float> x32, val32;
    dnq::DBuf<double> diag_op;
    dnq::Csr M;
    // planned arena (fixed sizes for graph replays)
    dnq::DBuf<dnq::u32> acol, rlen, big, blen;
    dnq::DBuf<uint4> sgl;
    dnq::DBuf<dnq::SingleOut> sres;
    dnq::DBuf<dnq::u32> sgn;
    dnq::u32 sgl_slice = 0;
    dnq::DBuf<double> aval;
    dnq::DBuf<dnq::i64> rpos;
    dnq::DBuf<int> next, ovf, nbig, bad;
    dnq::DBuf<unsigned long long> nt, cursor;
    dnq::DBuf<dnq::u8> scan_tmp;
    dnq::i64 cap = 0;
    dnq::i64 hits = 0;   // members of the sizing build (the arena holds members)
    int scan = 0;   // string words of the scans: 0 u64, 1 u32 (all n_orb <= 32), 2 per system
    bool planned = false;
    // tunables
    dnq::i64 chunk = dnq::kChunk;
    dnq::u32 big_group = dnq::kBigGroup;
    int spmv_group = 0;
    int spmv_unroll = 0;
    // graphs: [0] full step (build + H.psi), [1] H.psi on the resident CSR
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_prec[2] = {-1, -1};
    bool f32_ready = false;   // val32 / diag_op match the resident CSR
    // phases of the last eager step: diag, build (arena + long rows),
    // scan + compaction (+ FP32 split), H.psi + energies
    double phase_ms[4] = {0, 0, 0, 0};
    void drop_graphs() {
        for (auto& g : gexec)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
    ~dnq_batch_s() { drop_graphs(); }
};

namespace dnq {
namespace {

ManySys many(dnq_batch_s* b) {
    ManySys L;
    L.sys = b->sys.p;
    L.row_off = b->row_off.p;
    L.n_sys = b->n_sys;
    L.total = b->total;
    return L;
}

void upload_params(dnq_batch_s* b, cudaStream_t s) {
    std::vector<VVParams> hp(b->n_sys);
    DNQ_CUDA(cudaMemcpyAsync(hp.data(), b->sys.p, b->n_sys * sizeof(VVParams),
                             cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    for (auto& p : hp) p.big_group = b->big_group;
    DNQ_CUDA(cudaMemcpyAsync(b->sys.p, hp.data(), b->n_sys * sizeof(VVParams),
                             cudaMemcpyHostToDevice, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
}

// Plan: one exact build sizes the arena and the CSR; buffers then stay
// fixed so the step can be replayed from a graph.
void plan(dnq_batch_s* b, cudaStream_t s) {
    const ManySys L = many(b);
    const i64 n = b->total;
    k_diag_batch<<<sm_count(b->device) * 4, 256, 0, s>>>(L, b->diag.p);
    DNQ_CHECK_LAUNCH();
    // the sizing build fills the batch's CSR itself, so the blocks are
    // valid right after creation
    run_vv(L, n, 0, b->device, s, b->M, b->opt, nullptr, nullptr, nullptr, &b->hits, b->scan);
    b->M.nc = n;
    const i64 nnz = b->M.nnz;
    const int grid = vv_grid<ManySys>(b->device);
    b->cap = arena_bound(std::max(nnz, b->hits), n, grid, b->chunk);
    b->acol.alloc(b->cap, s);
    b->aval.alloc(b->cap, s);
    b->rlen.alloc(n + 1, s);
    b->big.alloc(n, s);
    b->blen.alloc(n, s);
    {
        const i64 warps = (i64)grid * kWS;
        b->sgl_slice = (u32)std::max<i64>(
            64, std::min<i64>(std::max<i64>(8 * n, 1024), i64(64) << 20) / warps);
        b->sgl.alloc((i64)b->sgl_slice * warps, s);
        b->sres.alloc((i64)b->sgl_slice * warps, s);
        b->sgn.alloc(warps, s);
    }
    b->rpos.alloc(n, s);
    b->next.alloc(1, s);
    b->ovf.alloc(1, s);
    b->nbig.alloc(1, s);
    b->bad.alloc(1, s);
    b->nt.alloc(1, s);
    b->cursor.alloc(1, s);
    b->val32.alloc(nnz, s);
    b->diag_op.alloc(n, s);
    b->x.alloc(n, s);
    b->y.alloc(n, s);
    b->eloc.alloc(n, s);
    b->x32.alloc(n, s);
    b->e2.alloc(2 * b->n_sys, s);
    {   // scan temporary sized once
        b->scan_tmp.alloc(prim::scan_tmp_bytes<i64>(n + 1), s);
    }
    DNQ_CUDA(cudaStreamSynchronize(s));
    b->planned = true;
}

// H.x and the per-system energies on the resident CSR (FP32: val32 and
// diag_op must already hold the split of M).
void enqueue_apply(dnq_batch_s* b, int precision, cudaStream_t s) {
    if (precision == DNQ_F32) {
        to_f32(b->x.p, b->total, b->x32.p, s);
        spmv_block_g(nullptr, b->M, b->x.p, b->y.p, DNQ_F32, s, b->x32.p, b->val32.p,
                     b->diag_op.p, b->spmv_group, b->device, b->spmv_unroll);
    } else {
        spmv_block_g(nullptr, b->M, b->x.p, b->y.p, DNQ_F64, s, nullptr, nullptr, nullptr,
                     b->spmv_group, b->device, b->spmv_unroll);
    }
    k_energy_sys<<<b->n_sys, 256, 0, s>>>(b->row_off.p, b->x.p, b->y.p, b->eloc.p, b->e2.p);
    DNQ_CHECK_LAUNCH();
}

// The step on planned buffers: diag, single-pass build (members, then their
// entries), long rows, scan, compaction, FP32 split, H.x, energies.  No
// allocation, no host sync.
void enqueue_step(dnq_batch_s* b, int precision, cudaStream_t s, cudaEvent_t* ev = nullptr) {
    auto mark = [&](int k) {
        if (ev) DNQ_CUDA(cudaEventRecord(ev[k], s));
    };
    mark(0);
    const ManySys L = many(b);
    const i64 n = b->total;
    const int grid = vv_grid<ManySys>(b->device);
    Arena A{};
    A.acol = b->acol.p;
    A.aval = b->aval.p;
    A.cap = b->cap;
    A.chunk = b->chunk;
    A.restart = b->chunk / 4;
    A.cursor = b->cursor.p;
    A.overflow = b->ovf.p;
    A.row_pos = b->rpos.p;
    A.row_len = b->rlen.p;
    A.big = b->big.p;
    A.big_len = b->blen.p;
    A.sgl = b->sgl.p;
    A.sres = b->sres.p;
    A.sgl_n = b->sgn.p;
    A.sgl_slice = b->sgl_slice;
    A.sgl_cap = (i64)b->sgl.n;
    A.n_big = b->nbig.p;
    A.next_row = b->next.p;
    A.n_test = b->nt.p;
    k_diag_batch<<<sm_count(b->device) * 4, 256, 0, s>>>(L, b->diag.p);
    DNQ_CHECK_LAUNCH();
    mark(1);
    DNQ_CUDA(cudaMemsetAsync(b->next.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(b->ovf.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(b->nbig.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(b->nt.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(b->cursor.p, 0, 8, s));
    DNQ_CUDA(cudaMemsetAsync(b->bad.p, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(b->rlen.p + n, 0, 4, s));
    launch_walk<ManySys>(b->scan, grid, L, A, s);
    k_vv_singles<ManySys><<<grid, 256, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    k_vv_eval<ManySys><<<eval_grid<ManySys>(b->device), kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    launch_big<ManySys>(b->scan, grid, L, A, s);
    k_vv_eval_long<ManySys><<<grid, kWS * 32, 0, s>>>(L, A);
    DNQ_CHECK_LAUNCH();
    mark(2);
    prim::scan<u32, i64, false>(b->rlen.p, b->M.rowptr.p, n + 1, s, b->scan_tmp.p);
    k_sanitize<<<1, 1024, 0, s>>>(b->M.rowptr.p, n, b->M.nnz, b->ovf.p, b->bad.p);
    DNQ_CHECK_LAUNCH();
    // FP32 steps write the FP32 operator copy in the same pass
    float* v32 = precision == DNQ_F32 ? b->val32.p : nullptr;
    double* dg = precision == DNQ_F32 ? b->diag_op.p : nullptr;
    k_vv_compact<<<grid, kWS * 32, 0, s>>>(b->rpos.p, b->M.rowptr.p, n, b->acol.p, b->aval.p,
                                           b->M.col.p, b->M.val.p, b->M.nnz, b->bad.p, v32, dg);
    DNQ_CHECK_LAUNCH();
    k_vv_compact_long<<<grid, 256, 0, s>>>(b->big.p, b->blen.p, b->nbig.p, b->rpos.p,
                                           b->M.rowptr.p, n, b->acol.p, b->aval.p, b->M.col.p,
                                           b->M.val.p, b->M.nnz, v32, dg);
    DNQ_CHECK_LAUNCH();
    mark(3);
    enqueue_apply(b, precision, s);
    mark(4);
}

void check_step(dnq_batch_s* b, cudaStream_t s) {
    int h[2] = {0, 0};
    DNQ_CUDA(cudaMemcpyAsync(&h[0], b->ovf.p, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&h[1], b->bad.p, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    require(!h[0] && !h[1], DNQ_ERR_OVERFLOW,
            "batched step outgrew its plan (inputs changed); destroy and recreate the batch");
}

// mode 0: full step; mode 1: H.psi only on the resident CSR.
float run_step(dnq_batch_s* b, int mode, int precision, bool graph, cudaStream_t s) {
    const bool phases = mode == 0 && !graph;
    Events<5> phe(phases);
    cudaEvent_t* ph = phe.data();
    auto enqueue = [&](cudaStream_t st) {
        if (mode == 0) enqueue_step(b, precision, st, phases ? ph : nullptr);
        else enqueue_apply(b, precision, st);
    };
    if (mode == 1 && precision == DNQ_F32 && !b->f32_ready) {
        launch_f32_split(b->M, b->val32.p, b->diag_op.p, s);   // once, outside any graph
        b->f32_ready = true;
    }
    Events<2> tev;
    const cudaEvent_t e0 = tev[0], e1 = tev[1];
    cudaGraphExec_t& ge = b->gexec[mode];
    if (graph && (ge == nullptr || b->graph_prec[mode] != precision)) {
        if (ge) {
            cudaGraphExecDestroy(ge);
            ge = nullptr;
        }
        cudaGraph_t gr;
        DNQ_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue(s);
        DNQ_CUDA(cudaStreamEndCapture(s, &gr));
        DNQ_CUDA(cudaGraphInstantiate(&ge, gr, 0));
        cudaGraphDestroy(gr);
        b->graph_prec[mode] = precision;
    }
    DNQ_CUDA(cudaEventRecord(e0, s));
    if (graph) {
        DNQ_CUDA(cudaGraphLaunch(ge, s));
    } else {
        enqueue(s);
    }
    DNQ_CUDA(cudaEventRecord(e1, s));
    DNQ_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    DNQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (phases) {
        for (int k = 0; k < 4; ++k) {
            float t = 0.f;
            DNQ_CUDA(cudaEventElapsedTime(&t, ph[k], ph[k + 1]));
            b->phase_ms[k] = t;
        }
    }
    if (mode == 0) {
        b->f32_ready = precision == DNQ_F32;
        check_step(b, s);
    }
    return ms;
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_batch_create(int n_sys, const dnq_ctx_t* ctxs, const uint64_t* const* dets,
                     const int64_t* n_dets, const int* n_orb, int policy, int use_heatbath,
                     double eps1, int device, void* stream, dnq_batch_t* out) {
    DNQ_API_BEGIN
    require(out && ctxs && dets && n_dets && n_orb, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(n_sys >= 1, DNQ_ERR_INVALID, "a batch needs at least one system");
    require(policy == DNQ_POLICY_KNOWN_SETS || policy == DNQ_POLICY_STATIC, DNQ_ERR_INVALID,
            "batched builds support the known-sets and static policies");
    DeviceGuard g(device);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<dnq_batch_s> b(new dnq_batch_s);
    b->device = device;
    if (b->opt.arena_chunk > 0) b->chunk = (dnq::i64)b->opt.arena_chunk;
    b->spmv_group = b->opt.spmv_lanes;
    b->spmv_unroll = b->opt.spmv_unroll;
    b->n_sys = n_sys;
    b->ctx.assign(ctxs, ctxs + n_sys);
    b->row_off_h.assign(n_sys + 1, 0);
    for (int k = 0; k < n_sys; ++k) {
        require(ctxs[k] && ctxs[k]->device == device, DNQ_ERR_INVALID,
                "every context must live on the batch's device");
        require_narrow(ctxs[k]);
        require(n_orb[k] >= 1 && n_orb[k] < 64 && n_orb[k] <= ctxs[k]->n, DNQ_ERR_INVALID,
                "n_orb must be in [1, min(63, orbitals of the context)]");
        require(n_dets[k] >= 1 && dets[k], DNQ_ERR_INVALID, "every system needs determinants");
        if (policy == DNQ_POLICY_STATIC && use_heatbath)
            require(ctxs[k]->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
        b->row_off_h[k + 1] = b->row_off_h[k] + n_dets[k];
    }
    b->total = b->row_off_h[n_sys];
    require(b->total < (i64)0x7fffffff, DNQ_ERR_OVERFLOW, "batch has more than 2^31 rows");
    b->diag.alloc(b->total, s);
    std::vector<VVParams> hp(n_sys);
    b->V.resize(n_sys);
    b->A.resize(n_sys);
    b->B.resize(n_sys);
    const int n_narrow = (int)std::count_if(n_orb, n_orb + n_sys, [](int o) { return o <= 32; });
    b->scan = n_narrow == n_sys ? 1 : (n_narrow > 0 ? 2 : 0);
    for (int k = 0; k < n_sys; ++k) {
        const i64 n = n_dets[k];
        b->V[k].alloc(2 * n, s);
        DNQ_CUDA(cudaMemcpyAsync(b->V[k].p, dets[k], 16 * n, cudaMemcpyDefault, s));
        check_orbitals(b->V[k].p, n, n_orb[k], s);
        DetMap dup;
        build_detmap(dup, b->V[k].p, n, true, s);   // duplicates are an error
        build_str_index(b->A[k], b->V[k].p, n, 0, n_orb[k], s);
        build_str_index(b->B[k], b->V[k].p, n, 1, n_orb[k], s);
        build_presence(b->A[k], b->B[k], n, s);
        build_presence(b->B[k], b->A[k], n, s);
        build_group_cost(b->A[k], b->V[k].p, n, 0, n_orb[k], s);
        build_group_cost(b->B[k], b->V[k].p, n, 1, n_orb[k], s);
        if (n_orb[k] <= 32) {
            narrow_index(b->A[k], n, s);
            narrow_index(b->B[k], n, s);
        }
        const double cut = (policy == DNQ_POLICY_STATIC && use_heatbath)
                               ? hb_cutoff(ctxs[k], eps1) : full_cutoff();
        hp[k] = make_params(ctxs[k], b->V[k].p, n, n_orb[k], policy, eps1, cut, nullptr,
                            b->diag.p + b->row_off_h[k], b->A[k], b->B[k], b->opt);
    }
    b->sys.alloc(n_sys, s);
    DNQ_CUDA(cudaMemcpyAsync(b->sys.p, hp.data(), n_sys * sizeof(VVParams),
                             cudaMemcpyHostToDevice, s));
    b->row_off.alloc(n_sys + 1, s);
    DNQ_CUDA(cudaMemcpyAsync(b->row_off.p, b->row_off_h.data(), (n_sys + 1) * sizeof(i64),
                             cudaMemcpyHostToDevice, s));
    plan(b.get(), s);
    *out = b.release();
    DNQ_API_END
}

int dnq_batch_destroy(dnq_batch_t b) {
    DNQ_API_BEGIN
    if (!b) return DNQ_OK;
    DeviceGuard g(b->device);
    delete b;
    DNQ_CUDA(cudaDeviceSynchronize());
    DNQ_API_END
}

int dnq_batch_info(dnq_batch_t b, int64_t* info4) {
    DNQ_API_BEGIN
    require(b && info4, DNQ_ERR_INVALID, "null argument");
    info4[0] = b->n_sys;
    info4[1] = b->total;
    info4[2] = b->M.nnz;
    info4[3] = (int64_t)(b->acol.bytes() + b->aval.bytes() + b->M.bytes() + b->val32.bytes());
    DNQ_API_END
}

int dnq_batch_set_config(dnq_batch_t b, const int64_t* cfg4) {
    DNQ_API_BEGIN
    require(b && cfg4, DNQ_ERR_INVALID, "null argument");
    require(cfg4[3] == 0 || cfg4[3] == 1 || cfg4[3] == 2 || cfg4[3] == 4, DNQ_ERR_INVALID,
            "slots per lane must be 0, 1, 2 or 4");
    require(cfg4[0] >= 64 && cfg4[0] <= (1 << 20), DNQ_ERR_INVALID, "chunk out of range");
    require(cfg4[1] >= 32, DNQ_ERR_INVALID, "group threshold out of range");
    require(cfg4[2] == 0 || cfg4[2] == 4 || cfg4[2] == 8 || cfg4[2] == 16 || cfg4[2] == 32,
            DNQ_ERR_INVALID, "lanes per row must be 0, 4, 8, 16 or 32");
    DeviceGuard g(b->device);
    const bool resize = cfg4[0] > b->chunk;
    b->chunk = cfg4[0];
    b->big_group = (u32)cfg4[1];
    b->spmv_group = (int)cfg4[2];
    b->spmv_unroll = (int)cfg4[3];
    upload_params(b, nullptr);
    if (resize) {   // larger chunks need a larger arena
        const int grid = vv_grid<ManySys>(b->device);
        b->cap = arena_bound(std::max(b->M.nnz, b->hits), b->total, grid, b->chunk);
        b->acol.alloc(b->cap, nullptr);
        b->aval.alloc(b->cap, nullptr);
        DNQ_CUDA(cudaStreamSynchronize(nullptr));
    }
    b->drop_graphs();
    DNQ_API_END
}

int dnq_batch_timings(dnq_batch_t b, double* ms4) {
    DNQ_API_BEGIN
    require(b && ms4, DNQ_ERR_INVALID, "null argument");
    for (int k = 0; k < 4; ++k) ms4[k] = b->phase_ms[k];
    DNQ_API_END
}

int dnq_batch_get_config(dnq_batch_t b, int64_t* cfg4) {
    DNQ_API_BEGIN
    require(b && cfg4, DNQ_ERR_INVALID, "null argument");
    cfg4[0] = b->chunk;
    cfg4[1] = b->big_group;
    cfg4[2] = b->spmv_group;
    cfg4[3] = b->spmv_unroll;
    DNQ_API_END
}

static int batch_run(dnq_batch_t b, int mode, const double* psi, double* eloc,
                     double* energies, int precision, int use_graph, void* stream,
                     double* step_ms) {
    DNQ_API_BEGIN
    require(b && psi, DNQ_ERR_INVALID, "null argument");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    require(s != nullptr || !use_graph, DNQ_ERR_INVALID,
            "graph replay needs an explicit (non-default) stream");
    DNQ_CUDA(cudaMemcpyAsync(b->x.p, psi, b->total * 8, cudaMemcpyDefault, s));
    const float ms = run_step(b, mode, precision, use_graph != 0, s);
    if (step_ms) *step_ms = ms;
    copy_out(eloc, b->eloc.p, b->total, s);
    copy_out(energies, b->e2.p, 2 * b->n_sys, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_batch_step(dnq_batch_t b, const double* psi, double* eloc, double* energies,
                   int precision, int use_graph, void* stream, double* step_ms) {
    return batch_run(b, 0, psi, eloc, energies, precision, use_graph, stream, step_ms);
}

int dnq_batch_apply(dnq_batch_t b, const double* psi, double* eloc, double* energies,
                    int precision, int use_graph, void* stream, double* step_ms) {
    return batch_run(b, 1, psi, eloc, energies, precision, use_graph, stream, step_ms);
}

// k amplitude sets per system in one pass over the resident CSR: X and
// eloc are total x k row-major, energies n_sys x k x 2.
int dnq_batch_apply_multi(dnq_batch_t b, const double* X, double* eloc, double* energies, int k,
                          int precision, void* stream, double* step_ms) {
    DNQ_API_BEGIN
    require(b && X, DNQ_ERR_INVALID, "null argument");
    require(k >= 1 && k <= 1024, DNQ_ERR_INVALID, "k must be in [1, 1024]");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 n = b->total;
    if (precision == DNQ_F32 && !b->f32_ready) {
        launch_f32_split(b->M, b->val32.p, b->diag_op.p, s);
        b->f32_ready = true;
    }
    DIn<double> xd(X, (size_t)n * k, s);
    DBuf<double> yd((size_t)n * k, s), e2((size_t)b->n_sys * k * 2, s);
    const bool dev_eloc = eloc && is_device_ptr(eloc);
    if (dev_eloc) require_on_device(eloc, b->device, "eloc");
    DBuf<double> ebuf;
    double* ed = nullptr;
    if (eloc) {
        if (dev_eloc) ed = eloc;
        else { ebuf.alloc((size_t)n * k, s); ed = ebuf.p; }
    }
    const int step = precision == DNQ_F32 ? 8 : 4;
    DBuf<unsigned char> scratch(spmm_scratch_bytes(n, std::min(k, step), precision), s);
    Events<2> tev;
    const cudaEvent_t e0 = tev[0], e1 = tev[1];
    DNQ_CUDA(cudaEventRecord(e0, s));
    for (int j0 = 0; j0 < k; j0 += step) {
        const int kx = std::min(step, k - j0);
        spmm_csr(b->M, b->val32.p, b->diag_op.p, xd.p + j0, k, kx, yd.p + j0, k, precision,
                 b->spmv_group, b->spmv_unroll, scratch.p, b->device, s);
    }
    k_energy_sys_multi<<<dim3((unsigned)b->n_sys, (unsigned)k), 256, 0, s>>>(
        b->row_off.p, xd.p, yd.p, k, ed, e2.p);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaEventRecord(e1, s));
    if (eloc && !dev_eloc) copy_out(eloc, ed, (size_t)n * k, s);
    copy_out(energies, e2.p, (size_t)b->n_sys * k * 2, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    DNQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (step_ms) *step_ms = ms;
    DNQ_API_END
}

// Sorted COO of one system's block, local indices (reference format).
int dnq_batch_copy_coo(dnq_batch_t b, int sys, uint32_t* rows, uint32_t* cols, double* vals,
                       int64_t* nnz) {
    DNQ_API_BEGIN
    require(b && nnz && sys >= 0 && sys < b->n_sys, DNQ_ERR_INVALID, "invalid system");
    DeviceGuard g(b->device);
    std::vector<i64> rp(b->total + 1);
    DNQ_CUDA(cudaMemcpy(rp.data(), b->M.rowptr.p, (b->total + 1) * 8, cudaMemcpyDeviceToHost));
    const i64 r0 = b->row_off_h[sys], r1 = b->row_off_h[sys + 1];
    for (i64 r = r0; r < r1; ++r)
        require(rp[r] >= 0 && rp[r] <= rp[r + 1] && rp[r + 1] <= b->M.nnz, DNQ_ERR_INVALID,
                "batch CSR row pointers are not valid");
    const i64 k0 = rp[r0], k1 = rp[r1];
    *nnz = k1 - k0;
    if (!rows && !cols && !vals) return DNQ_OK;
    std::vector<u32> c(k1 - k0);
    std::vector<double> v(k1 - k0);
    if (k1 > k0) {
        DNQ_CUDA(cudaMemcpy(c.data(), b->M.col.p + k0, (k1 - k0) * 4, cudaMemcpyDeviceToHost));
        DNQ_CUDA(cudaMemcpy(v.data(), b->M.val.p + k0, (k1 - k0) * 8, cudaMemcpyDeviceToHost));
    }
    i64 w = 0;
    for (i64 r = r0; r < r1; ++r) {   // rows are in generation order: sort each
        std::vector<std::pair<u32, double>> row;
        for (i64 k = rp[r]; k < rp[r + 1]; ++k)
            row.push_back({c[k - k0] - (u32)r0, v[k - k0]});
        std::sort(row.begin(), row.end(),
                  [](const auto& x, const auto& y) { return x.first < y.first; });
        for (auto& e : row) {
            if (rows) rows[w] = (u32)(r - r0);
            if (cols) cols[w] = e.first;
            if (vals) vals[w] = e.second;
            ++w;
        }
    }
    DNQ_API_END
}

}  // extern "C"
