// genp.cu -- determinant-space generators and row connectivity on the device:
//   gen_connected_dets    (det_space.cpp:167-213, bridge.cpp:265-276)
//   gen_perturbative_dets (det_space.cpp:233-255; ham_utils.cpp:546-701)
//   get_local_connections (local_conn.cpp:36-142)
//   compute_pt2           (local_conn.cpp:247-418)
//
// All use count/fill passes of one warp per bra row (exact output sizes),
// 128-bit radix sort + run-length unique for determinant sets, and hash
// lookups in the device map of V for exclusion.
#include <memory>

#include "gen.cuh"
#include "ham.cuh"
#include "prim.cuh"

namespace dnq {

void check_orbitals(const u64* d, i64 n, int n_orb, cudaStream_t s);
void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s);
double contract_energy(dnq_ctx_s* ctx, const u64* Vd, i64 n, const double* cd, int n_orb,
                       bool use_hb, double eps1, double* sigma, cudaStream_t s);

namespace {

constexpr int kW = 8;

int gsz(i64 n) {
    i64 b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

template <class T>
void scan_ex(const T* in, i64* out, i64 n, cudaStream_t s) {
    prim::scan<T, i64, false>(in, out, n, s);
}

i64 rd(const i64* d, cudaStream_t s) {
    i64 v = 0;
    DNQ_CUDA(cudaMemcpyAsync(&v, d, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    return v;
}

__device__ __forceinline__ i64 choose2(int m) { return m < 2 ? 0 : (i64)m * (m - 1) / 2; }

// k-th pair (x < y) of m items in the order x ascending, y ascending.
__device__ __forceinline__ void pair_at(i64 k, int m, int& x, int& y) {
    int a = 0;
    while (k >= m - 1 - a) { k -= m - 1 - a; ++a; }
    x = a;
    y = a + 1 + (int)k;
}

// Combinatorial singles + doubles of every bra (det_ops.hpp:123-268): no
// element values, no screening.  Emits the kets not in `excl` (optional).
struct CombParams {
    const u64* V;
    i64 n;
    int n_orb;
    DetMapView excl;
    bool has_excl;
    int* next_row;
    u32* cnt;
    const i64* off;
    ulonglong2* keys;
};

template <bool FILL>
__global__ void __launch_bounds__(kW * 32) k_comb(CombParams P) {
    __shared__ WarpRow rows[kW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        load_row(R, P.V[2 * (i64)r], P.V[2 * (i64)r + 1], P.n_orb);
        const i64 ns = (i64)R.na * R.nva + (i64)R.nb * R.nvb;
        const i64 naa = choose2(R.na) * choose2(R.nva);
        const i64 nbb = choose2(R.nb) * choose2(R.nvb);
        const i64 nab = (i64)R.na * R.nva * R.nb * R.nvb;
        const i64 tot = ns + naa + nbb + nab;
        u32 c = 0;
        i64 wpos = FILL ? P.off[r] : 0;
        for (i64 t0 = 0; t0 < tot; t0 += 32) {
            const i64 t = t0 + lane;
            bool keep = false;
            u64 ka = R.a, kb = R.b;
            if (t < tot) {
                i64 u = t;
                if (u < ns) {
                    if (u < (i64)R.na * R.nva) {
                        ka ^= (1ull << R.occa[u / R.nva]) ^ (1ull << R.vira[u % R.nva]);
                    } else {
                        u -= (i64)R.na * R.nva;
                        kb ^= (1ull << R.occb[u / R.nvb]) ^ (1ull << R.virb[u % R.nvb]);
                    }
                } else if ((u -= ns) < naa + nbb) {
                    const bool beta = u >= naa;
                    if (beta) u -= naa;
                    const int no = beta ? R.nb : R.na, nvv = beta ? R.nvb : R.nva;
                    const u8* oc = beta ? R.occb : R.occa;
                    const u8* vi = beta ? R.virb : R.vira;
                    const i64 cv = choose2(nvv);
                    int h1, h2, p1, p2;
                    pair_at(u / cv, no, h1, h2);
                    pair_at(u % cv, nvv, p1, p2);
                    const u64 flip = (1ull << oc[h1]) ^ (1ull << oc[h2]) ^ (1ull << vi[p1]) ^
                                     (1ull << vi[p2]);
                    if (beta) kb ^= flip; else ka ^= flip;
                } else {
                    u -= naa + nbb;
                    const i64 nbv = (i64)R.nb * R.nvb;
                    const i64 ia = u / nbv, ib = u % nbv;
                    ka ^= (1ull << R.occa[ia / R.nva]) ^ (1ull << R.vira[ia % R.nva]);
                    kb ^= (1ull << R.occb[ib / R.nvb]) ^ (1ull << R.virb[ib % R.nvb]);
                }
                keep = !(P.has_excl && P.excl.find(ka, kb) >= 0);
            }
            if (!FILL) {
                c += keep;
            } else {
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) P.keys[wpos + __popc(m & lanemask_lt())] = make_ulonglong2(ka, kb);
                wpos += __popc(m);
            }
        }
        if (!FILL) {
            c = __reduce_add_sync(0xffffffffu, c);
            if (lane == 0) P.cnt[r] = c;
        }
        __syncwarp();
    }
}

// Screened complement (ham_utils.cpp:590-628): singles with |h| > 1e-15
// (dynamic: also |h psi_i| >= eps1), heat-bath doubles with w >= cut and
// no element test; kets in V are dropped.
struct ScrParams {
    CtxView C;
    const u64* V;
    i64 n;
    int n_orb;
    DetMapView mapV;
    bool dynamic;
    const double* psi;
    double eps1, cut;
    int* next_row;
    u32* cnt;
    const i64* off;
    ulonglong2* keys;
};

template <bool FILL>
struct ScrSink {
    const ScrParams& P;
    double psi_row;
    u32 c = 0;
    i64 wpos = 0;
    __device__ ScrSink(const ScrParams& p, double ps) : P(p), psi_row(ps) {}
    __device__ __forceinline__ void step(const Cand& x) {
        bool keep = false;
        if (x.valid) {
            keep = true;
            if (x.single) {
                keep = fabs(x.h) > kElemThresh;
                if (keep && P.dynamic) keep = fabs(x.h * psi_row) >= P.eps1;
            }
            if (keep) keep = P.mapV.find(x.a, x.b) < 0;
        }
        if (!FILL) {
            c += keep;
            return;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) P.keys[wpos + __popc(m & lanemask_lt())] = make_ulonglong2(x.a, x.b);
        wpos += __popc(m);
    }
};

template <bool FILL>
__global__ void __launch_bounds__(kW * 32) k_screened(ScrParams P) {
    __shared__ WarpRow rows[kW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        load_row(R, P.V[2 * (i64)r], P.V[2 * (i64)r + 1], P.n_orb);
        double ps = 0.0, cut = P.cut;
        if (P.dynamic) {
            ps = P.psi[r];
            cut = fmax(P.eps1 / fmax(fabs(ps), kAmpDelta), P.cut);
        }
        ScrSink<FILL> sink(P, ps);
        if (FILL) sink.wpos = P.off[r];
        enumerate_row(P.C, R, nullptr, cut, sink);
        if (!FILL) {
            const u32 c = __reduce_add_sync(0xffffffffu, sink.c);
            if (lane == 0) P.cnt[r] = c;
        }
        __syncwarp();
    }
}

__global__ void k_flags(const ulonglong2* k, i64 n, u32* f) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        f[t] = (t == 0 || k[t].x != k[t - 1].x || k[t].y != k[t - 1].y) ? 1u : 0u;
}

__global__ void k_compact_keys(const ulonglong2* k, const u32* f, const i64* pos, i64 n,
                               unsigned long long* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        if (f[t]) {
            out[2 * pos[t]] = k[t].x;
            out[2 * pos[t] + 1] = k[t].y;
        }
}

// Sort keys, keep one of each: the sorted unique set (canonicalize,
// det_space.cpp:97-101) written to H->dets_p.
void sort_unique(DBuf<ulonglong2>& keys, i64 n, int n_orb, cudaStream_t s, dnq_ham_s* H) {
    H->n_p = 0;
    if (n == 0) return;
    DBuf<ulonglong2> sorted(n, s);
    const int bits[2] = {n_orb, n_orb};
    prim::radix_sort<ulonglong2, u32>(keys.p, sorted.p, nullptr, nullptr, n, bits, s);
    keys.release();
    DBuf<u32> f(n, s);
    DBuf<i64> pos(n + 1, s);
    k_flags<<<gsz(n), 256, 0, s>>>(sorted.p, n, f.p);
    DNQ_CHECK_LAUNCH();
    scan_ex(f.p, pos.p, n, s);
    u32 lastf = 0;
    i64 lastp = 0;
    DNQ_CUDA(cudaMemcpyAsync(&lastf, f.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&lastp, pos.p + n - 1, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    H->n_p = lastp + lastf;
    H->dets_p.alloc(2 * H->n_p, s);
    k_compact_keys<<<gsz(n), 256, 0, s>>>(sorted.p, f.p, pos.p, n, H->dets_p.p);
    DNQ_CHECK_LAUNCH();
}

int grid_of(const void* kern, int device, int block) {
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0));
    return std::max(1, per_sm) * sm_count(device);
}

// ---------------------------------------------------------------------------
// local connections
// ---------------------------------------------------------------------------
struct ConnParams {
    CtxView C;
    const u64* V;
    i64 n;
    int n_orb;
    const double* diag;
    double single_thr;
    const i64* plen;
    double cut;
    bool full_order;     // no heat-bath screening: doubles in for_each_double's order
    int* next_row;
    u32* cnt;
    const i64* off;
    ulonglong2* keys;
    double* vals;
};

template <bool FILL>
struct ConnSink {
    const ConnParams& P;
    u32 c = 0;
    i64 wpos = 0;
    __device__ explicit ConnSink(const ConnParams& p) : P(p) {}
    __device__ __forceinline__ void step(const Cand& x) {
        const bool keep = x.valid && fabs(x.h) > (x.single ? P.single_thr : kElemThresh);
        if (!FILL) {
            c += keep;
            return;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const i64 at = wpos + __popc(m & lanemask_lt());
            P.keys[at] = make_ulonglong2(x.a, x.b);
            P.vals[at] = x.h;
        }
        wpos += __popc(m);
    }
};

template <bool FILL>
__global__ void __launch_bounds__(kW * 32) k_conn(ConnParams P) {
    __shared__ WarpRow rows[kW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        const u64 a = P.V[2 * (i64)r], b = P.V[2 * (i64)r + 1];
        load_row(R, a, b, P.n_orb);
        ConnSink<FILL> sink(P);
        const double d = P.diag[r];
        const bool dk = fabs(d) > kElemThresh;     // local_conn.cpp:61-66
        if (FILL) {
            sink.wpos = P.off[r];
            if (dk) {
                if (lane == 0) {
                    P.keys[sink.wpos] = make_ulonglong2(a, b);
                    P.vals[sink.wpos] = d;
                }
                sink.wpos += 1;
            }
        } else if (dk && lane == 0) {
            sink.c = 1;
        }
        if (P.full_order) enumerate_row_full(P.C, R, sink);
        else enumerate_row(P.C, R, P.plen, P.cut, sink);
        if (!FILL) {
            const u32 c = __reduce_add_sync(0xffffffffu, sink.c);
            if (lane == 0) P.cnt[r] = c;
        }
        __syncwarp();
    }
}

__global__ void k_plen(PairTableView T, i64 nrows, double cut, i64* plen) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nrows;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 lo = T.off[r], len = T.off[r + 1] - lo;
        if (cut <= 0.0) { plen[r] = len; continue; }
        i64 L = 0, Rr = len;
        while (L < Rr) {
            const i64 mid = L + (Rr - L) / 2;
            if (fabs(T.v[lo + mid]) >= cut) L = mid + 1; else Rr = mid;
        }
        plen[r] = L;
    }
}

// ---------------------------------------------------------------------------
// EN-PT2 external part: (key, h c_i) contributions of kets outside V
// ---------------------------------------------------------------------------
struct Pt2Params {
    CtxView C;
    const u64* V;
    i64 n;
    int n_orb;
    DetMapView mapV;
    const double* coeff;
    double eps1, cut_floor;
    bool use_hb;
    const i64* plen_full;
    int* next_row;
    u32* cnt;
    const i64* off;
    ulonglong2* keys;
    double* vals;
};

template <bool FILL>
struct Pt2Sink {
    const Pt2Params& P;
    double ci;
    u32 c = 0;
    i64 wpos = 0;
    __device__ Pt2Sink(const Pt2Params& p, double cc) : P(p), ci(cc) {}
    __device__ __forceinline__ void step(const Cand& x) {
        bool keep = x.valid && fabs(x.h) > kElemThresh && fabs(x.h * ci) >= P.eps1;
        if (keep) keep = P.mapV.find(x.a, x.b) < 0;
        if (!FILL) {
            c += keep;
            return;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const i64 at = wpos + __popc(m & lanemask_lt());
            P.keys[at] = make_ulonglong2(x.a, x.b);
            P.vals[at] = x.h * ci;
        }
        wpos += __popc(m);
    }
};

template <bool FILL>
__global__ void __launch_bounds__(kW * 32) k_pt2ext(Pt2Params P) {
    __shared__ WarpRow rows[kW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        const double ci = P.coeff[r];
        if (ci * ci < 1e-15) {                    // local_conn.cpp:300
            if (!FILL && lane == 0) P.cnt[r] = 0;
            continue;
        }
        load_row(R, P.V[2 * (i64)r], P.V[2 * (i64)r + 1], P.n_orb);
        Pt2Sink<FILL> sink(P, ci);
        if (FILL) sink.wpos = P.off[r];
        if (P.use_hb) {
            const double tau = P.eps1 / fmax(fabs(ci), kAmpDelta);   // :368-372
            enumerate_row(P.C, R, nullptr, fmax(tau, P.cut_floor), sink);
        } else {
            enumerate_row(P.C, R, P.plen_full, 0.0, sink);
        }
        if (!FILL) {
            const u32 c = __reduce_add_sync(0xffffffffu, sink.c);
            if (lane == 0) P.cnt[r] = c;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void tsum2(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double z = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, z)), __dsub_rn(b, z));
}

// Per unique key: v_a = sum of its contributions (compensated), then
// v_a^2 / (e_ref - H_aa) with the reference's denominator guard.
__global__ void k_pt2_runs(CtxView C, const ulonglong2* k, const double* v, i64 n,
                           double e_ref, double* part, unsigned long long* nuniq) {
    double s = 0.0, c = 0.0;
    unsigned long long cnt = 0;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (!(t == 0 || k[t].x != k[t - 1].x || k[t].y != k[t - 1].y)) continue;
        double vs = v[t], vc = 0.0;
        for (i64 u = t + 1; u < n && k[u].x == k[t].x && k[u].y == k[t].y; ++u) {
            double s2, e;
            tsum2(vs, v[u], s2, e);
            vs = s2;
            vc += e;
        }
        const double va = vs + vc;
        const double haa = diag_elem(C, k[t].x, k[t].y);
        double den = e_ref - haa;
        if (fabs(den) < 1e-15) den = den >= 0.0 ? 1e-15 : -1e-15;
        double s2, e;
        tsum2(s, (va * va) / den, s2, e);
        s = s2;
        c += e;
        ++cnt;
    }
    for (int o = 16; o; o >>= 1) {
        const double os = __shfl_xor_sync(0xffffffffu, s, o);
        const double oc = __shfl_xor_sync(0xffffffffu, c, o);
        double s2, e;
        tsum2(s, os, s2, e);
        s = s2;
        c += oc + e;
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(nuniq, cnt);
        const i64 wid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
        part[2 * wid] = s;
        part[2 * wid + 1] = c;
    }
}

// Internal part: sum_i r_i^2 / (e_ref - h_ii), r_i = sigma_i - e_ref c_i.
__global__ void k_pt2_internal(const double* sigma, const double* coeff, const double* diag,
                               i64 n, double e_ref, double* part) {
    double s = 0.0, c = 0.0;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const double ci = coeff[t];
        if (ci * ci < 1e-15) continue;
        const double r = sigma[t] - e_ref * ci;
        double den = e_ref - diag[t];
        if (fabs(den) < 1e-15) den = den >= 0.0 ? 1e-15 : -1e-15;
        double s2, e;
        tsum2(s, (r * r) / den, s2, e);
        s = s2;
        c += e;
    }
    for (int o = 16; o; o >>= 1) {
        const double os = __shfl_xor_sync(0xffffffffu, s, o);
        const double oc = __shfl_xor_sync(0xffffffffu, c, o);
        double s2, e;
        tsum2(s, os, s2, e);
        s = s2;
        c += oc + e;
    }
    if ((threadIdx.x & 31) == 0) {
        const i64 wid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
        part[2 * wid] = s;
        part[2 * wid + 1] = c;
    }
}

double sum_parts(const DBuf<double>& part, i64 nw, cudaStream_t s) {
    std::vector<double> h(2 * nw);
    DNQ_CUDA(cudaMemcpyAsync(h.data(), part.p, 16 * nw, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    double acc = 0.0, cc = 0.0;
    for (i64 k = 0; k < nw; ++k) {
        const double y = h[2 * k] - cc;
        const double t = acc + y;
        cc = (t - acc) - y;
        acc = t;
        cc -= h[2 * k + 1];
    }
    return acc - cc;
}

}  // namespace

// Union of singles/doubles of V (optionally screened), minus V if asked.
// mode: -1 connected set (no exclusion), 0 none, 1 static, 2 dynamic.
void gen_dets(dnq_ctx_s* ctx, const u64* Vd, i64 n, int n_orb, const double* psi, int mode,
              double eps1, int device, cudaStream_t s, dnq_ham_s* H) {
    H->device = device;
    H->stream = s;
    H->n_v = n;
    if (n == 0) return;
    DetMap mapV;
    if (mode >= 0) build_detmap(mapV, Vd, n, true, s);
    DBuf<int> next(1, s);
    DBuf<u32> cnt(n + 1, s);
    DBuf<i64> off(n + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
    DBuf<ulonglong2> keys;
    if (mode <= 0) {
        CombParams P{};
        P.V = Vd;
        P.n = n;
        P.n_orb = n_orb;
        P.excl = mapV.view();
        P.has_excl = mode == 0;
        P.next_row = next.p;
        P.cnt = cnt.p;
        const int grid = grid_of((const void*)k_comb<false>, device, kW * 32);
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_comb<false><<<grid, kW * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
        scan_ex(cnt.p, off.p, n + 1, s);
        const i64 tot = rd(off.p + n, s);
        keys.alloc(tot, s);
        P.off = off.p;
        P.keys = keys.p;
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_comb<true><<<grid, kW * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
        sort_unique(keys, tot, n_orb, s, H);
    } else {
        DIn<double> ps(psi, mode == 2 ? n : 0, s);
        ScrParams P{};
        P.C = ctx->view();
        P.V = Vd;
        P.n = n;
        P.n_orb = n_orb;
        P.mapV = mapV.view();
        P.dynamic = mode == 2;
        P.psi = ps.p;
        P.eps1 = eps1;
        P.cut = mode == 2 ? ctx->hb_thr : hb_cutoff(ctx, eps1);
        P.next_row = next.p;
        P.cnt = cnt.p;
        const int grid = grid_of((const void*)k_screened<false>, device, kW * 32);
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_screened<false><<<grid, kW * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
        scan_ex(cnt.p, off.p, n + 1, s);
        const i64 tot = rd(off.p + n, s);
        keys.alloc(tot, s);
        P.off = off.p;
        P.keys = keys.p;
        DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
        k_screened<true><<<grid, kW * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
        sort_unique(keys, tot, n_orb, s, H);
    }
    DNQ_CUDA(cudaStreamSynchronize(s));
}

void local_connections(dnq_ctx_s* ctx, const u64* Vd, i64 n, int n_orb, bool use_hb,
                       double eps1, cudaStream_t s, dnq_ham_s* H) {
    H->device = ctx->device;
    H->stream = s;
    H->n_v = n;
    H->vv.nr = n;
    H->vv.rowptr.alloc(n + 1, s);
    if (n == 0) {
        DNQ_CUDA(cudaMemsetAsync(H->vv.rowptr.p, 0, 8, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        return;
    }
    DBuf<double> diag(n, s);
    launch_diag(ctx, Vd, n, diag.p, s);
    const double cut = use_hb ? hb_cutoff(ctx, eps1) : full_cutoff();
    DBuf<i64> plen(ctx->tab.n_rows, s);
    k_plen<<<gsz(ctx->tab.n_rows), 256, 0, s>>>(ctx->view().tab, ctx->tab.n_rows, cut, plen.p);
    DNQ_CHECK_LAUNCH();
    DBuf<int> next(1, s);
    DBuf<u32> cnt(n + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
    ConnParams P{};
    P.C = ctx->view();
    P.V = Vd;
    P.n = n;
    P.n_orb = n_orb;
    P.diag = diag.p;
    P.single_thr = use_hb ? std::max(eps1, kElemThresh) : kElemThresh;   // local_conn.cpp:56-58
    P.plen = plen.p;
    P.cut = cut;
    P.full_order = !use_hb;
    P.next_row = next.p;
    P.cnt = cnt.p;
    const int grid = grid_of((const void*)k_conn<false>, ctx->device, kW * 32);
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_conn<false><<<grid, kW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    scan_ex(cnt.p, H->vv.rowptr.p, n + 1, s);
    const i64 tot = rd(H->vv.rowptr.p + n, s);
    require(tot <= (i64)0x7fffffff, DNQ_ERR_OVERFLOW,
            "local connections exceed the int32 offsets of the reference format");
    H->vv.nnz = tot;
    H->n_p = tot;
    H->vv.val.alloc(tot, s);
    DBuf<ulonglong2> keys(tot, s);
    P.off = H->vv.rowptr.p;
    P.keys = keys.p;
    P.vals = H->vv.val.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_conn<true><<<grid, kW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    H->dets_p.alloc(2 * tot, s);
    if (tot)
        DNQ_CUDA(cudaMemcpyAsync(H->dets_p.p, keys.p, 16 * tot, cudaMemcpyDeviceToDevice, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
}

void pt2(dnq_ctx_s* ctx, const u64* Vd, i64 n, const double* cd, int n_orb, double e_ref,
         bool use_hb, double eps1, cudaStream_t s, double* out3) {
    // internal part: full enumeration inside V (local_conn.cpp:303-338)
    DBuf<double> sigma(n, s), diag(n, s);
    contract_energy(ctx, Vd, n, cd, n_orb, false, eps1, sigma.p, s);
    launch_diag(ctx, Vd, n, diag.p, s);
    const int nb = 4 * sm_count(ctx->device);
    DBuf<double> part(2 * (i64)nb * 8, s);
    k_pt2_internal<<<nb, 256, 0, s>>>(sigma.p, cd, diag.p, n, e_ref, part.p);
    DNQ_CHECK_LAUNCH();
    out3[0] = sum_parts(part, (i64)nb * 8, s);
    // external part (:340-415)
    DetMap mapV;
    build_detmap(mapV, Vd, n, false, s);
    DBuf<i64> plen(ctx->tab.n_rows, s);
    k_plen<<<gsz(ctx->tab.n_rows), 256, 0, s>>>(ctx->view().tab, ctx->tab.n_rows,
                                                 full_cutoff(), plen.p);
    DNQ_CHECK_LAUNCH();
    DBuf<int> next(1, s);
    DBuf<u32> cnt(n + 1, s);
    DBuf<i64> off(n + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
    Pt2Params P{};
    P.C = ctx->view();
    P.V = Vd;
    P.n = n;
    P.n_orb = n_orb;
    P.mapV = mapV.view();
    P.coeff = cd;
    P.eps1 = eps1;
    P.cut_floor = ctx->hb_thr;
    P.use_hb = use_hb;
    P.plen_full = plen.p;
    P.next_row = next.p;
    P.cnt = cnt.p;
    const int grid = grid_of((const void*)k_pt2ext<false>, ctx->device, kW * 32);
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_pt2ext<false><<<grid, kW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    scan_ex(cnt.p, off.p, n + 1, s);
    const i64 tot = rd(off.p + n, s);
    DBuf<ulonglong2> keys(tot, s), ks(tot, s);
    DBuf<double> vals(tot, s), vs(tot, s);
    P.off = off.p;
    P.keys = keys.p;
    P.vals = vals.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    k_pt2ext<true><<<grid, kW * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    out3[1] = 0.0;
    out3[2] = 0.0;
    if (tot == 0) return;
    {
        const int bits[2] = {n_orb, n_orb};
        prim::radix_sort<ulonglong2, double>(keys.p, ks.p, vals.p, vs.p, tot, bits, s);
    }
    DBuf<unsigned long long> nu(1, s);
    DNQ_CUDA(cudaMemsetAsync(nu.p, 0, 8, s));
    DBuf<double> part2(2 * (i64)nb * 8, s);
    k_pt2_runs<<<nb, 256, 0, s>>>(ctx->view(), ks.p, vs.p, tot, e_ref, part2.p, nu.p);
    DNQ_CHECK_LAUNCH();
    out3[1] = sum_parts(part2, (i64)nb * 8, s);
    unsigned long long h = 0;
    DNQ_CUDA(cudaMemcpyAsync(&h, nu.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    out3[2] = (double)h;
}

}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_gen_dets(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, int n_orb, const double* psi,
                 int mode, double eps1, int device, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(out != nullptr, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(mode >= -1 && mode <= 2, DNQ_ERR_INVALID, "invalid screen mode");
    require(n >= 0 && (n == 0 || dets), DNQ_ERR_INVALID, "null determinant array");
    require(n_orb >= 1 && n_orb <= 64, DNQ_ERR_INVALID, "n_orb must be in [1, 64]");
    if (mode >= 1) {
        require(ctx != nullptr, DNQ_ERR_INVALID, "screened modes need an integral context");
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
        require(n_orb <= ctx->n, DNQ_ERR_INVALID,
                "n_orb must be in [1, number of orbitals of the integral context]");
        if (mode == 2) require(n == 0 || psi, DNQ_ERR_INVALID, "psi_v size mismatch");
        device = ctx->device;
    }
    DeviceGuard g(device);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    DIn<u64> d(dets, 2 * n, s);
    check_orbitals(d.p, n, n_orb, s);
    gen_dets(ctx, d.p, n, n_orb, psi, mode, eps1, device, s, H.get());
    *out = H.release();
    DNQ_API_END
}

int dnq_local_connections(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, int n_orb,
                          int use_heatbath, double eps1, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx && out, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(n >= 0 && (n == 0 || dets), DNQ_ERR_INVALID, "null determinant array");
    require(n_orb >= 1 && n_orb <= ctx->n, DNQ_ERR_INVALID,
            "n_orb must be in [1, number of orbitals of the integral context]");
    if (use_heatbath)
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    DIn<u64> d(dets, 2 * n, s);
    check_orbitals(d.p, n, n_orb, s);
    local_connections(ctx, d.p, n, n_orb, use_heatbath != 0, eps1, s, H.get());
    *out = H.release();
    DNQ_API_END
}

int dnq_conn_copy(dnq_ham_t h, int32_t* offsets, uint64_t* dets, double* values, void* stream) {
    DNQ_API_BEGIN
    require(h != nullptr, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    ensure_compact(h->vv, s);
    if (offsets) {
        std::vector<i64> rp(h->n_v + 1, 0);
        if (h->vv.rowptr.p)
            DNQ_CUDA(cudaMemcpyAsync(rp.data(), h->vv.rowptr.p, (h->n_v + 1) * 8,
                                     cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> o(h->n_v + 1);
        for (i64 k = 0; k <= h->n_v; ++k) o[k] = (int32_t)rp[k];
        DNQ_CUDA(cudaMemcpyAsync(offsets, o.data(), (h->n_v + 1) * 4, cudaMemcpyDefault, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    copy_out(dets, (const uint64_t*)h->dets_p.p, 2 * h->n_p, s);
    copy_out(values, h->vv.val.p, h->vv.nnz, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_pt2(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, const double* coeffs, int n_orb,
            double e_ref, int use_heatbath, double eps1, double* out3, void* stream) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx && out3, DNQ_ERR_INVALID, "null argument");
    out3[0] = out3[1] = out3[2] = 0.0;
    require(n >= 0, DNQ_ERR_INVALID, "negative size");
    if (n == 0) return DNQ_OK;
    require(dets && coeffs, DNQ_ERR_INVALID, "null argument");
    require(n_orb >= 1 && n_orb <= ctx->n, DNQ_ERR_INVALID,
            "n_orb must be in [1, number of orbitals of the integral context]");
    if (use_heatbath)
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> d(dets, 2 * n, s);
    DIn<double> c(coeffs, n, s);
    check_orbitals(d.p, n, n_orb, s);
    pt2(ctx, d.p, n, c.p, n_orb, e_ref, use_heatbath != 0, eps1, s, out3);
    DNQ_API_END
}

}  // extern "C"
