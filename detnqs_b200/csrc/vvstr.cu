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

// Insert one slot per group: thread at each group head finds its end.
__global__ void k_group_insert(const ulonglong2* k, const unsigned* head, i64 n,
                               ulonglong2* slots, u64 mask) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (!head[t]) continue;
        const u64 key = k[t].x;
        i64 e = t + 1;
        while (e < n && !head[e]) ++e;
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
    u64 cap = 1024;
    while (cap < (u64)(2 * n)) cap <<= 1;
    X.mask = cap - 1;
    X.slots.alloc(cap, s);
    DNQ_CUDA(cudaMemsetAsync(X.slots.p, 0xff, cap * sizeof(ulonglong2), s));
    k_group_insert<<<gsz(n), 256, 0, s>>>(ks.p, head.p, n, X.slots.p, X.mask);
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
    u32* cnt;
    unsigned long long* n_test;
    const i64* off;
    u32* col;
    double* val;
};

template <bool FILL>
struct Emit {
    const VVParams& P;
    u32 c = 0;
    i64 w = 0;
    unsigned long long tests = 0;
    __device__ explicit Emit(const VVParams& p) : P(p) {}
    // collective over the warp
    __device__ __forceinline__ void put(bool keep, u32 j, double h) {
        if (!FILL) {
            c += keep;
            return;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const i64 at = w + __popc(m & lanemask_lt());
            P.col[at] = j;
            P.val[at] = h;
        }
        w += __popc(m);
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

__device__ __forceinline__ bool keep_double(const VVParams& P, double cut, double h) {
    const double w = fabs(h);
    return w > kElemThresh && w >= cut;
}

__device__ __forceinline__ bool keep_single(const VVParams& P, double psr, double h) {
    if (!(fabs(h) > kElemThresh)) return false;
    if (P.policy == DNQ_POLICY_DYNAMIC) return fabs(h * psr) >= P.eps1;
    return true;
}

template <bool FILL>
__global__ void __launch_bounds__(kWS * 32) k_vvstr(VVParams P) {
    __shared__ u32 s_start[kWS][32], s_len[kWS][32], s_scan[kWS][32];
    __shared__ u8 s_h[kWS][32], s_p[kWS][32];
    __shared__ u8 s_occa[kWS][64], s_vira[kWS][64], s_occb[kWS][64], s_virb[kWS][64];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 all = low_mask(P.n_orb);
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        const u64 a = P.V[2 * (i64)r], b = P.V[2 * (i64)r + 1];
        double psr = 0.0, cut = P.cut;
        if (P.policy == DNQ_POLICY_DYNAMIC) {
            psr = P.psi[r];
            cut = fmax(P.eps1 / fmax(fabs(psr), kAmpDelta), P.cut);
        }
        if (lane == 0) {
            int k = 0;
            for (u64 m = a; m; m &= m - 1) s_occa[w][k++] = (u8)(__ffsll(m) - 1);
            k = 0;
            for (u64 m = ~a & all; m; m &= m - 1) s_vira[w][k++] = (u8)(__ffsll(m) - 1);
            k = 0;
            for (u64 m = b; m; m &= m - 1) s_occb[w][k++] = (u8)(__ffsll(m) - 1);
            k = 0;
            for (u64 m = ~b & all; m; m &= m - 1) s_virb[w][k++] = (u8)(__ffsll(m) - 1);
        }
        __syncwarp();
        Emit<FILL> em(P);
        if (FILL) em.w = P.off[r];
        const double d = P.diag[r];
        const bool dk = fabs(d) > kElemThresh;
        if (FILL) {
            if (dk && lane == 0) {
                P.col[em.w] = (u32)r;
                P.val[em.w] = d;
            }
            em.w += dk;
        } else if (lane == 0) {
            em.c = dk;
        }
        // ---- part A: same beta string
        u32 st = 0, ln = 0;
        if (lane == 0) {
            if (!P.bmap.find(b, st, ln)) ln = 0;
        }
        st = __shfl_sync(0xffffffffu, st, 0);
        ln = __shfl_sync(0xffffffffu, ln, 0);
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
                    keep = keep_double(P, cut, h);
                }
                if (keep) j = __ldg(&P.b_idx[st + t]);
                ++em.tests;
            }
            em.put(keep, j, h);
        }
        // ---- part B: same alpha string
        if (lane == 0) {
            if (!P.amap.find(a, st, ln)) ln = 0;
        }
        st = __shfl_sync(0xffffffffu, st, 0);
        ln = __shfl_sync(0xffffffffu, ln, 0);
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
                    keep = keep_double(P, cut, h);
                }
                if (keep) j = __ldg(&P.a_idx[st + t]);
                ++em.tests;
            }
            em.put(keep, j, h);
        }
        // ---- part C: alpha single x beta single, via the groups of a'
        const u64 occa = a, vira = ~a & all;
        const int na = __popcll(occa), nva = __popcll(vira);
        const int nsa = na * nva;
        for (int s0 = 0; s0 < nsa; s0 += 32) {
            const int sidx = s0 + lane;
            u32 gs = 0, gl = 0;
            int hh = 0, pp = 0;
            if (sidx < nsa) {
                hh = s_occa[w][sidx / nva];
                pp = s_vira[w][sidx % nva];
                const u64 ap = a ^ (1ull << hh) ^ (1ull << pp);
                if (!P.amap.find(ap, gs, gl)) gl = 0;
            }
            const bool big = gl > kBigGroup;
            const u32 scan_len = big ? 0u : gl;
            // inclusive scan of scan_len across lanes
            u32 inc = scan_len;
            for (int o = 1; o < 32; o <<= 1) {
                const u32 y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            s_start[w][lane] = gs;
            s_len[w][lane] = scan_len;
            s_scan[w][lane] = inc;
            s_h[w][lane] = (u8)hh;
            s_p[w][lane] = (u8)pp;
            __syncwarp();
            const u32 total = __shfl_sync(0xffffffffu, inc, 31);
            for (u32 t0 = 0; t0 < total; t0 += 32) {
                const u32 t = t0 + lane;
                bool keep = false;
                double h = 0.0;
                u32 j = 0;
                if (t < total) {
                    // owner group: first l with s_scan[l] > t
                    int lo = 0, hi = 31;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (s_scan[w][mid] > t) hi = mid; else lo = mid + 1;
                    }
                    const u32 base = s_scan[w][lo] - s_len[w][lo];
                    const u32 at = s_start[w][lo] + (t - base);
                    const u64 y = __ldg(&P.a_other[at]);
                    const u64 x = b ^ y;
                    if (__popcll(x) == 2) {
                        const int ha = s_h[w][lo], pa = s_p[w][lo];
                        const int hb = __ffsll(b & x) - 1, pb = __ffsll(y & x) - 1;
                        const double raw = eri(P.E, ha, pa, hb, pb);   // (a i|b j)
                        const int perm = occ_between(a, pa, ha) + occ_between(b, pb, hb);
                        h = (perm & 1) ? -raw : raw;
                        keep = keep_double(P, cut, h);
                        if (keep) j = __ldg(&P.a_idx[at]);
                    }
                    ++em.tests;
                }
                em.put(keep, j, h);
            }
            // large groups: binary-search every beta single of b instead
            unsigned bigm = __ballot_sync(0xffffffffu, big);
            while (bigm) {
                const int l = __ffs(bigm) - 1;
                bigm &= bigm - 1;
                const u32 g0 = s_start[w][l];
                const u32 gn = __shfl_sync(0xffffffffu, gl, l);
                const int ha = s_h[w][l], pa = s_p[w][l];
                const int nb = __popcll(b), nvb = __popcll(~b & all);
                for (int q0 = 0; q0 < nb * nvb; q0 += 32) {
                    const int q = q0 + lane;
                    bool keep = false;
                    double h = 0.0;
                    u32 j = 0;
                    if (q < nb * nvb) {
                        const int hb = s_occb[w][q / nvb];
                        const int pb = s_virb[w][q % nvb];
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
                            keep = keep_double(P, cut, h);
                            if (keep) j = __ldg(&P.a_idx[lo]);
                        }
                        ++em.tests;
                    }
                    em.put(keep, j, h);
                }
            }
            __syncwarp();
        }
        if (!FILL) {
            const u32 c = __reduce_add_sync(0xffffffffu, em.c);
            unsigned long long tt = em.tests;
            for (int o = 16; o; o >>= 1) tt += __shfl_xor_sync(0xffffffffu, tt, o);
            if (lane == 0) {
                P.cnt[r] = c;
                atomicAdd(P.n_test, tt);
            }
        }
        __syncwarp();
    }
}

}  // namespace

void sort_rows(Csr& m, cudaStream_t s);
void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s);

// H_VV only, from string groups.  V on the device, diag already computed.
void build_vv_strings(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, const double* diag, cudaStream_t s,
                      dnq_ham_s* H, double* t_ms) {
    cudaEvent_t ev[6];
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
    DBuf<int> next(1, s);
    DBuf<u32> cnt(n + 1, s);
    DBuf<unsigned long long> nt(1, s);
    DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(nt.p, 0, 8, s));
    P.next_row = next.p;
    P.cnt = cnt.p;
    P.n_test = nt.p;
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vvstr<false>, kWS * 32, 0));
    const int grid = std::max(1, per_sm) * sm_count(ctx->device);
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    DNQ_CUDA(cudaEventRecord(ev[1], s));
    k_vvstr<false><<<grid, kWS * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaEventRecord(ev[2], s));
    H->vv.nr = H->vv.nc = n;
    H->vv.rowptr.alloc(n + 1, s);
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.p, H->vv.rowptr.p, n + 1, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, cnt.p, H->vv.rowptr.p, n + 1, s));
    }
    DNQ_CUDA(cudaMemcpyAsync(&H->vv.nnz, H->vv.rowptr.p + n, 8, cudaMemcpyDeviceToHost, s));
    unsigned long long tests = 0;
    DNQ_CUDA(cudaMemcpyAsync(&tests, nt.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    H->candidates = (i64)tests;
    H->vv.col.alloc(H->vv.nnz, s);
    H->vv.val.alloc(H->vv.nnz, s);
    P.off = H->vv.rowptr.p;
    P.col = H->vv.col.p;
    P.val = H->vv.val.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    DNQ_CUDA(cudaEventRecord(ev[3], s));
    k_vvstr<true><<<grid, kWS * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaEventRecord(ev[4], s));
    sort_rows(H->vv, s);
    DNQ_CUDA(cudaEventRecord(ev[5], s));
    DNQ_CUDA(cudaEventSynchronize(ev[5]));
    float ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    t_ms[0] += ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
    t_ms[1] = ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[2], ev[3]));
    t_ms[2] = ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[3], ev[4]));
    t_ms[3] = ms;
    DNQ_CUDA(cudaEventElapsedTime(&ms, ev[4], ev[5]));
    t_ms[4] = ms;
    for (auto& e : ev) cudaEventDestroy(e);
}

}  // namespace dnq
