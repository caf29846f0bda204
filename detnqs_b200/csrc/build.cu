// build.cu -- screened Hamiltonian build (replaces stream_build and its
// policies, build_ham.cpp:78-535) and element evaluation entry points.
//
// Pipeline of one dnq_build call:
//   1. V (and the optional external set) -> device hash maps; duplicates in
//      V are an error as in DetMap::from_ordered(verify_unique=true).
//   2. k_diag: one thread per determinant, reference summation order.
//   3. k_build<count>: warp per row, counts surviving V->V and V->P entries.
//   4. exclusive scans -> CSR row pointers (exact sizes, nothing guessed).
//   5. k_build<fill>: same walk, survivors compacted with __ballot_sync in
//      candidate order straight into their CSR rows.
//   6. per-row sort by column; for discovered P: radix sort of the 128-bit
//      keys, run-length unique (lexicographic (alpha, beta) order of
//      finalize_vp_deferred, build_ham.cpp:346-380) and column relabelling.

#include <cmath>
#include <memory>
#include <mutex>

#include "gen.cuh"
#include "ham.cuh"
#include "prim.cuh"

namespace dnq {

namespace {

constexpr int kWarpsPerBlock = 8;

__global__ void k_diag(CtxView C, const u64* dets, i64 n, double* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        out[t] = diag_elem(C, dets[2 * t], dets[2 * t + 1]);
}

__global__ void k_check_orbitals(const u64* dets, i64 n, int n_orb,
                                 unsigned long long* bad) {
    const u64 keep = low_mask(n_orb);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        if ((dets[2 * t] | dets[2 * t + 1]) & ~keep) atomicAdd(bad, 1ull);
}

// Prefix length of every table row for one cut (static screening).
__global__ void k_prefix_lengths(PairTableView T, i64 nrows, double cut, i64* plen) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nrows;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 lo = T.off[r], len = T.off[r + 1] - lo;
        if (cut <= 0.0) { plen[r] = len; continue; }
        i64 L = 0, R = len;
        while (L < R) {
            const i64 mid = L + (R - L) / 2;
            if (fabs(T.v[lo + mid]) >= cut) L = mid + 1; else R = mid;
        }
        plen[r] = L;
    }
}

struct BuildParams {
    CtxView C;
    DetMapView mapV, mapX;
    bool has_ext;
    int policy;
    bool want_vp;
    double eps1;
    double cut;            // static cutoff (policies 0/1)
    const i64* plen;       // prefix lengths for `cut`, or null (dynamic)
    const double* psi;
    int n_orb;
    const u64* V;
    i64 nV;
    const double* diag;
    int* next_row;
    // count pass
    u32* cnt_vv;
    u32* cnt_vp;
    unsigned long long* n_cand;
    // fill pass
    const i64* off_vv;
    const i64* off_vp;
    u32* vv_col;
    double* vv_val;
    u32* vp_col;           // known external set
    ulonglong2* vp_key;    // discovered P keys
    double* vp_val;
};

template <bool FILL>
struct BuildSink {
    const BuildParams& P;
    double psi_row;
    u32 nvv = 0, nvp = 0;
    unsigned long long ncand = 0;
    i64 wvv = 0, wvp = 0;

    __device__ BuildSink(const BuildParams& p, double psr) : P(p), psi_row(psr) {}

    __device__ __forceinline__ void step(const Cand& c) {
        int route = 0;   // 0 drop, 1 V, 2 external index, 3 P key
        long long j = -1;
        if (c.valid) {
            ++ncand;
            bool pass = fabs(c.h) > kElemThresh;
            if (pass && c.single && P.policy == DNQ_POLICY_DYNAMIC)
                pass = fabs(c.h * psi_row) >= P.eps1;   // build_ham.cpp:190-192
            if (pass) {
                j = P.mapV.find(c.a, c.b);
                if (j >= 0) route = 1;
                else if (P.policy == DNQ_POLICY_KNOWN_SETS) {
                    if (P.has_ext) {
                        j = P.mapX.find(c.a, c.b);
                        if (j >= 0) route = 2;
                    }
                } else if (P.want_vp) {
                    route = 3;
                }
            }
        }
        if (!FILL) {
            nvv += route == 1;
            nvp += route >= 2;
            return;
        }
        const unsigned lt = lanemask_lt();
        const unsigned mv = __ballot_sync(0xffffffffu, route == 1);
        if (route == 1) {
            const i64 at = wvv + __popc(mv & lt);
            P.vv_col[at] = (u32)j;
            P.vv_val[at] = c.h;
        }
        wvv += __popc(mv);
        const unsigned mp = __ballot_sync(0xffffffffu, route >= 2);
        if (route >= 2) {
            const i64 at = wvp + __popc(mp & lt);
            if (route == 2) P.vp_col[at] = (u32)j;
            else P.vp_key[at] = make_ulonglong2(c.a, c.b);
            P.vp_val[at] = c.h;
        }
        wvp += __popc(mp);
    }
};

template <bool FILL>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
k_build(BuildParams P) {
    __shared__ WarpRow rows[kWarpsPerBlock];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.nV) break;
        load_row(R, P.V[2 * (i64)r], P.V[2 * (i64)r + 1], P.n_orb);
        double psr = 0.0, cut = P.cut;
        if (P.policy == DNQ_POLICY_DYNAMIC) {
            psr = P.psi[r];
            // tau_i = eps1 / max(|psi_i|, delta)  (build_ham.cpp:176-186)
            const double amp = fmax(fabs(psr), kAmpDelta);
            cut = fmax(P.eps1 / amp, P.cut);
        }
        BuildSink<FILL> sink(P, psr);
        const double d = P.diag[r];
        const bool dkeep = fabs(d) > kElemThresh;
        if (FILL) {
            sink.wvv = P.off_vv[r];
            sink.wvp = P.off_vp[r];
            if (dkeep) {
                if (lane == 0) {
                    P.vv_col[sink.wvv] = (u32)r;
                    P.vv_val[sink.wvv] = d;
                }
                sink.wvv += 1;
            }
        } else if (dkeep && lane == 0) {
            sink.nvv = 1;
        }
        enumerate_row(P.C, R, P.policy == DNQ_POLICY_DYNAMIC ? nullptr : P.plen, cut, sink);
        if (!FILL) {
            const u32 a = __reduce_add_sync(0xffffffffu, sink.nvv);
            const u32 b = __reduce_add_sync(0xffffffffu, sink.nvp);
            unsigned long long c = sink.ncand;
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) {
                P.cnt_vv[r] = a;
                P.cnt_vp[r] = b;
                atomicAdd(P.n_cand, c);
            }
        }
        __syncwarp();
    }
}

__global__ void k_unique_flags(const ulonglong2* k, i64 n, u32* flag) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        flag[t] = (t == 0 || k[t].x != k[t - 1].x || k[t].y != k[t - 1].y) ? 1u : 0u;
}

__global__ void k_unique_scatter(const ulonglong2* k, const u32* perm, const u32* runid,
                                 i64 n, unsigned long long* pdets, u32* col) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 r = runid[t] - 1;   // inclusive scan of flags
        if (t == 0 || k[t].x != k[t - 1].x || k[t].y != k[t - 1].y) {
            pdets[2 * (i64)r] = k[t].x;
            pdets[2 * (i64)r + 1] = k[t].y;
        }
        col[perm[t]] = r;
    }
}

// (alpha, beta) <-> alpha << n_orb | beta, for n_orb <= 32.
__global__ void k_pack_keys(const ulonglong2* k, i64 n, int n_orb, u64* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        out[t] = (k[t].x << n_orb) | k[t].y;
}

__global__ void k_unpack_keys(const u64* p, i64 n, int n_orb, ulonglong2* out) {
    const u64 lo = n_orb >= 64 ? ~0ull : ((1ull << n_orb) - 1);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        out[t] = make_ulonglong2(p[t] >> n_orb, p[t] & lo);
}

// FP32 copy of every value (streaming, 2 values per thread step).
__global__ void k_vals_f32(const double2* __restrict__ v, i64 n2, float2* __restrict__ o) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n2;
         t += (i64)gridDim.x * blockDim.x) {
        const double2 x = v[t];
        o[t] = make_float2((float)x.x, (float)x.y);
    }
}

__global__ void k_val_f32_tail(const double* v, i64 n, float* o) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) o[n - 1] = (float)v[n - 1];
}

// Diagonal entry of each row (column order not assumed): moved out of the
// FP32 copy into the FP64 vector (0 when the row has none).  Warp per row.
__global__ void k_split_diag(const i64* rs, const i64* re, const u32* col, const double* val,
                             i64 nr, float* out, double* dout) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    for (i64 r = gw; r < nr; r += nw) {
        const i64 b = rs[r], e = re[r];
        double d = 0.0;
        for (i64 k0 = b; k0 < e; k0 += 32) {
            const i64 k = k0 + lane;
            const bool on = k < e && col[k] == (u32)r;
            if (on) {
                d = val[k];
                out[k] = 0.0f;
            }
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (m) {
                d = __shfl_sync(0xffffffffu, d, __ffs(m) - 1);
                break;
            }
        }
        if (dout && lane == 0) dout[r] = d;
    }
}

inline int grid_for(i64 n, int threads = 256) {
    i64 b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 65535) b = 65535;
    return (int)b;
}

template <class T>
void exclusive_scan(const T* in, i64* out, i64 n, cudaStream_t s) {
    prim::scan<T, i64, false>(in, out, n, s);
}

i64 read_i64(const i64* d, cudaStream_t s) {
    i64 v = 0;
    DNQ_CUDA(cudaMemcpyAsync(&v, d, sizeof(i64), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    return v;
}

}  // namespace

void ensure_sorted(Csr& m, cudaStream_t s) {
    if (!m.sorted) sort_rows(m, s);
}


void sort_rows(Csr& m, cudaStream_t s) {
    ensure_compact(m, s);
    m.sorted = true;
    m.val32.release();   // an FP32 copy follows the old order: rebuilt on next use
    if (m.nnz == 0 || m.nr == 0) return;
    DBuf<u32> col2(m.nnz, s);
    DBuf<double> val2(m.nnz, s);
    prim::sort_row_columns(m.rowptr.p, m.nr, m.col.p, m.val.p, col2.p, val2.p, s);
    m.col = std::move(col2);
    m.val = std::move(val2);
}

// FP32 copy + diagonal split into caller buffers (no allocation; graph-safe).
void launch_f32_split(const Csr& m, float* val32, double* diag_out, cudaStream_t s) {
    int dev = 0;
    DNQ_CUDA(cudaGetDevice(&dev));
    const int sms = sm_count(dev);
    const i64 len = m.span();   // every slot of an arena-form block (free ones too)
    if (len) {
        k_vals_f32<<<sms * 8, 256, 0, s>>>((const double2*)m.val.p, len / 2, (float2*)val32);
        DNQ_CHECK_LAUNCH();
        k_val_f32_tail<<<1, 32, 0, s>>>(m.val.p, len, val32);
        DNQ_CHECK_LAUNCH();
    }
    if (m.nr) {
        k_split_diag<<<sms * 8, 256, 0, s>>>(m.row_start(), m.row_end(), m.col.p, m.val.p, m.nr,
                                             val32, diag_out);
        DNQ_CHECK_LAUNCH();
    }
}

void make_f32(Csr& m, cudaStream_t s, DBuf<double>* diag_out) {
    m.val32.alloc(m.val.n, s);
    if (diag_out) diag_out->alloc(m.nr, s);
    if (m.nr == 0) return;
    launch_f32_split(m, m.val32.p, diag_out ? diag_out->p : nullptr, s);
}

// Validate and stage the determinants; throws on orbitals >= n_orb.
// Flags in *bad (zeroed by the caller) a determinant with an orbital >= n_orb;
// no host synchronisation.
void launch_check_orbitals(const u64* d, i64 n, int n_orb, unsigned long long* bad,
                           cudaStream_t s) {
    if (n == 0) return;
    k_check_orbitals<<<grid_for(n), 256, 0, s>>>(d, n, n_orb, bad);
    DNQ_CHECK_LAUNCH();
}

void check_orbitals(const u64* d, i64 n, int n_orb, cudaStream_t s) {
    if (n == 0) return;
    DBuf<unsigned long long> bad(1, s);
    DNQ_CUDA(cudaMemsetAsync(bad.p, 0, 8, s));
    k_check_orbitals<<<grid_for(n), 256, 0, s>>>(d, n, n_orb, bad.p);
    DNQ_CHECK_LAUNCH();
    unsigned long long h = 0;
    DNQ_CUDA(cudaMemcpyAsync(&h, bad.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    require(h == 0, DNQ_ERR_INVALID, "determinant occupies an orbital index >= n_orb");
}

void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s) {
    if (n == 0) return;
    k_diag<<<grid_for(n, 128), 128, 0, s>>>(c->view(), d, n, out);
    DNQ_CHECK_LAUNCH();
}

// CUDA events bracketing the build phases on the build stream.
struct PhaseTimer {
    Events<8> ev;
    int n = 0;
    cudaStream_t s;
    explicit PhaseTimer(cudaStream_t st) : s(st) {}
    void mark() { DNQ_CUDA(cudaEventRecord(ev[n++], s)); }
    void fill(double* out) {
        DNQ_CUDA(cudaEventSynchronize(ev[n - 1]));
        for (int k = 0; k + 1 < n; ++k) {
            float ms = 0.f;
            DNQ_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            out[k] = ms;
        }
        float tot = 0.f;
        DNQ_CUDA(cudaEventElapsedTime(&tot, ev[0], ev[n - 1]));
        out[6] = tot;
    }
};

namespace {
std::mutex g_opt_mu;
Options g_defaults;   // process-wide defaults of new handles, batches and servers
}  // namespace

Options default_options() {
    std::lock_guard<std::mutex> lk(g_opt_mu);
    return g_defaults;
}

thread_local const Options* g_build_opt = nullptr;

// Resident-table cut for a policy (see hb_cutoff / full_cutoff).
static double policy_cut(const dnq_ctx_s* c, int policy, int use_hb, double eps1) {
    if (policy == DNQ_POLICY_STATIC && use_hb) return hb_cutoff(c, eps1);
    if (policy == DNQ_POLICY_DYNAMIC) return c->hb_thr;   // floor under tau_i
    return full_cutoff();
}

void launch_wide_diag(const dnq_ctx_s* ctx, const u64* d, i64 n, double* out, cudaStream_t s);

void build_vv_strings(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, const double* diag, cudaStream_t s,
                      dnq_ham_s* H, double* t_ms);
void build_vv_checked(dnq_ctx_s* ctx, const u64* V, i64 n, int n_orb, int policy, double eps1,
                      double cut, const double* psi, cudaStream_t s, dnq_ham_s* H,
                      double* t_ms);

void build_ham(dnq_ctx_s* ctx, const u64* V_in, i64 nV, const u64* X_in, i64 nX,
               const double* psi_in, int n_orb, int policy, int use_hb, double eps1,
               bool want_vp, cudaStream_t s, dnq_ham_s* H) {
    H->device = ctx->device;
    H->stream = s;
    H->n_v = nV;
    PhaseTimer T(s);
    T.mark();
    DIn<u64> V(V_in, 2 * nV, s), X(X_in, 2 * nX, s);
    DIn<double> psi(psi_in, policy == DNQ_POLICY_DYNAMIC ? nV : 0, s);
    const bool vv_only = !want_vp && !(policy == DNQ_POLICY_KNOWN_SETS && X_in && nX > 0) &&
                         n_orb < 64 && !H->opt.force_walk;
    if (vv_only && nV > 0) {
        // V->V block only, the input checks folded into the string indices'
        // one host synchronisation (an X set the policy does not use is
        // still checked, as on every other path)
        check_orbitals(X.p, nX, n_orb, s);
        build_vv_checked(ctx, V.p, nV, n_orb, policy, eps1,
                         policy_cut(ctx, policy, use_hb, eps1), psi.p, s, H, H->t_ms);
        H->n_p = 0;
        H->t_ms[6] = H->t_ms[0] + H->t_ms[1] + H->t_ms[2] + H->t_ms[3] + H->t_ms[4];
        DNQ_CUDA(cudaStreamSynchronize(s));
        return;
    }
    check_orbitals(V.p, nV, n_orb, s);
    check_orbitals(X.p, nX, n_orb, s);
    DetMap mapV, mapX;
    build_detmap(mapV, V.p, nV, true, s);
    const bool has_ext = policy == DNQ_POLICY_KNOWN_SETS && X_in && nX > 0;
    if (has_ext) build_detmap(mapX, X.p, nX, true, s);

    H->diag.alloc(nV, s);
    launch_diag(ctx, V.p, nV, H->diag.p, s);

    if (!want_vp && !has_ext && n_orb < 64 && !H->opt.force_walk) {
        // V->V block only: match rows against V's string groups.
        T.mark();
        T.fill(H->t_ms);   // [0] maps + diagonal
        build_vv_strings(ctx, V.p, nV, n_orb, policy, eps1, policy_cut(ctx, policy, use_hb, eps1),
                         psi.p, H->diag.p, s, H, H->t_ms);
        H->n_p = 0;
        H->t_ms[6] = H->t_ms[0] + H->t_ms[1] + H->t_ms[2] + H->t_ms[3] + H->t_ms[4];
        DNQ_CUDA(cudaStreamSynchronize(s));
        return;
    }

    BuildParams P{};
    P.C = ctx->view();
    P.mapV = mapV.view();
    P.mapX = mapX.view();
    P.has_ext = has_ext;
    P.policy = policy;
    P.want_vp = want_vp;
    P.eps1 = eps1;
    P.cut = policy_cut(ctx, policy, use_hb, eps1);
    P.psi = psi.p;
    P.n_orb = n_orb;
    P.V = V.p;
    P.nV = nV;
    P.diag = H->diag.p;

    DBuf<i64> plen;
    if (policy != DNQ_POLICY_DYNAMIC) {
        plen.alloc(ctx->tab.n_rows, s);
        k_prefix_lengths<<<grid_for(ctx->tab.n_rows), 256, 0, s>>>(
            P.C.tab, ctx->tab.n_rows, P.cut, plen.p);
        DNQ_CHECK_LAUNCH();
        P.plen = plen.p;
    }
    DBuf<int> next(1, s);
    DBuf<u32> cvv(nV + 1, s), cvp(nV + 1, s);
    DBuf<unsigned long long> ncand(1, s);
    DNQ_CUDA(cudaMemsetAsync(cvv.p + nV, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(cvp.p + nV, 0, 4, s));
    DNQ_CUDA(cudaMemsetAsync(ncand.p, 0, 8, s));
    P.next_row = next.p;
    P.cnt_vv = cvv.p;
    P.cnt_vp = cvp.p;
    P.n_cand = ncand.p;

    int dev_sms = sm_count(ctx->device);
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build<false>,
                                                           kWarpsPerBlock * 32, 0));
    const int grid = std::max(1, per_sm) * dev_sms;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    T.mark();
    k_build<false><<<grid, kWarpsPerBlock * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    T.mark();

    H->vv.nr = nV;
    H->vv.nc = nV;
    H->vv.rowptr.alloc(nV + 1, s);
    exclusive_scan(cvv.p, H->vv.rowptr.p, nV + 1, s);
    DBuf<i64> offp(nV + 1, s);
    exclusive_scan(cvp.p, offp.p, nV + 1, s);
    H->vv.nnz = read_i64(H->vv.rowptr.p + nV, s);
    const i64 nvp = read_i64(offp.p + nV, s);
    DNQ_CUDA(cudaMemcpyAsync(&H->candidates, ncand.p, 8, cudaMemcpyDeviceToHost, s));

    H->vv.col.alloc(H->vv.nnz, s);
    H->vv.val.alloc(H->vv.nnz, s);
    DBuf<u32> vp_col;
    DBuf<ulonglong2> vp_key;
    DBuf<double> vp_val(nvp, s);
    if (has_ext) vp_col.alloc(nvp, s);
    else vp_key.alloc(nvp, s);
    P.off_vv = H->vv.rowptr.p;
    P.off_vp = offp.p;
    P.vv_col = H->vv.col.p;
    P.vv_val = H->vv.val.p;
    P.vp_col = vp_col.p;
    P.vp_key = vp_key.p;
    P.vp_val = vp_val.p;
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    T.mark();
    k_build<true><<<grid, kWarpsPerBlock * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    T.mark();
    sort_rows(H->vv, s);
    T.mark();

    // ---- V->P block
    const bool vp_block = has_ext || (policy != DNQ_POLICY_KNOWN_SETS && want_vp);
    if (!vp_block) {
        H->n_p = 0;
        T.mark();
        T.fill(H->t_ms);
        return;
    }
    H->vp.nr = nV;
    H->vp.nnz = nvp;
    H->vp.rowptr = std::move(offp);
    H->vp.val = std::move(vp_val);
    if (has_ext) {
        H->n_p = nX;
        H->vp.nc = nX;
        H->vp.col = std::move(vp_col);
        sort_rows(H->vp, s);
        H->dets_p.alloc(2 * nX, s);
        DNQ_CUDA(cudaMemcpyAsync(H->dets_p.p, X.p, 16 * nX, cudaMemcpyDeviceToDevice, s));
        T.mark();
        T.fill(H->t_ms);
        return;
    }
    // P discovery: sort the keys with their positions (stable), unique,
    // relabel.  The sort visits the n_orb bits of each spin string only; for
    // n_orb <= 32 both strings are packed into one word, alpha above beta,
    // which keeps the (alpha, beta) order.
    require(nvp < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "H_VP has more than 2^32 entries");
    DBuf<ulonglong2> ks(nvp, s);
    DBuf<u32> perm2(nvp, s);
    if (nvp) {
        if (2 * n_orb <= 64) {
            DBuf<u64> pk(nvp, s), pks(nvp, s);
            k_pack_keys<<<grid_for(nvp), 256, 0, s>>>(vp_key.p, nvp, n_orb, pk.p);
            DNQ_CHECK_LAUNCH();
            const int bits[1] = {2 * n_orb};
            prim::radix_sort<u64, u32>(pk.p, pks.p, nullptr, perm2.p, nvp, bits, s);
            k_unpack_keys<<<grid_for(nvp), 256, 0, s>>>(pks.p, nvp, n_orb, ks.p);
            DNQ_CHECK_LAUNCH();
        } else {
            const int bits[2] = {n_orb, n_orb};
            prim::radix_sort<ulonglong2, u32>(vp_key.p, ks.p, nullptr, perm2.p, nvp, bits, s);
        }
    }
    vp_key.release();
    DBuf<u32> flag(nvp, s), runid(nvp, s);
    i64 np = 0;
    if (nvp) {
        k_unique_flags<<<grid_for(nvp), 256, 0, s>>>(ks.p, nvp, flag.p);
        DNQ_CHECK_LAUNCH();
        prim::scan_inclusive<u32, u32>(flag.p, runid.p, nvp, s);
        u32 last = 0;
        DNQ_CUDA(cudaMemcpyAsync(&last, runid.p + nvp - 1, 4, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        np = last;
    }
    H->n_p = np;
    H->vp.nc = np;
    H->dets_p.alloc(2 * np, s);
    H->vp.col.alloc(nvp, s);
    if (nvp) {
        k_unique_scatter<<<grid_for(nvp), 256, 0, s>>>(ks.p, perm2.p, runid.p, nvp,
                                                       H->dets_p.p, H->vp.col.p);
        DNQ_CHECK_LAUNCH();
    }
    sort_rows(H->vp, s);
    T.mark();
    T.fill(H->t_ms);
}

namespace {

// compute_elem for arbitrary pairs: doubles read the packed ERIs directly
// (ham_eval.cpp:117-147) so that this path is independent of the table.
__device__ __forceinline__ double eri_mo_d(const double* eri, int p, int q, int r, int s) {
    auto tri = [](i64 x, i64 y) { return x >= y ? x * (x + 1) / 2 + y : y * (y + 1) / 2 + x; };
    return eri[tri(tri(p, q), tri(r, s))];
}

__device__ __forceinline__ double phys_d(const double* eri, int mu, int ka, int nu, int la) {
    if (((mu ^ nu) & 1) || ((ka ^ la) & 1)) return 0.0;
    return eri_mo_d(eri, mu >> 1, nu >> 1, ka >> 1, la >> 1);
}

struct ExcD {
    int degree;
    int nx[2];
    int hole[2][2], part[2][2];
    int perm;
};

__device__ ExcD analyze_d(u64 ba, u64 bb, u64 ka, u64 kb) {
    ExcD e{};
    const u64 br[2] = {ba, bb}, kt[2] = {ka, kb};
    bool bad = false;
    for (int s = 0; s < 2; ++s) {
        u64 h = kt[s] & ~br[s], p = br[s] & ~kt[s];
        const int nh = __popcll(h), np_ = __popcll(p);
        if (nh != np_) { e.nx[s] = 3; bad = true; continue; }
        e.nx[s] = nh;
        if (nh > 2) { bad = true; continue; }
        for (int k = 0; k < nh; ++k) {
            e.hole[s][k] = __ffsll(h) - 1; h &= h - 1;
            e.part[s][k] = __ffsll(p) - 1; p &= p - 1;
        }
    }
    e.degree = e.nx[0] + e.nx[1];
    if (bad || e.degree > 2) return e;
    int perm = 0;
    for (int s = 0; s < 2; ++s) {
        for (int k = 0; k < e.nx[s]; ++k) perm += occ_between(br[s], e.hole[s][k], e.part[s][k]);
        if (e.nx[s] == 2) {
            const int a = min(e.hole[s][0], e.part[s][0]), b = max(e.hole[s][0], e.part[s][0]);
            const int c = min(e.hole[s][1], e.part[s][1]), d = max(e.hole[s][1], e.part[s][1]);
            if ((c > a && c < b && d > b) || (a > c && a < d && b > d)) ++perm;
        }
    }
    e.perm = perm;
    return e;
}

__global__ void k_elems(CtxView C, const double* eri, const u64* bra, const u64* ket, i64 n,
                        double* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 ba = bra[2 * t], bb = bra[2 * t + 1], ka = ket[2 * t], kb = ket[2 * t + 1];
        const ExcD e = analyze_d(ba, bb, ka, kb);
        double v = 0.0;
        if (e.degree == 0) {
            v = diag_elem(C, ka, kb);
        } else if (e.degree == 1) {
            const int s = e.nx[0] == 1 ? 0 : 1;
            // bra orbital part[s][0] -> ket orbital hole[s][0]
            v = single_elem(C, ba, bb, s, e.part[s][0], e.hole[s][0]);
        } else if (e.degree == 2) {
            double raw;
            int s2 = e.nx[0] == 2 ? 0 : (e.nx[1] == 2 ? 1 : -1);
            if (s2 >= 0) {
                const int a = 2 * e.part[s2][0] + s2, b = 2 * e.part[s2][1] + s2;
                const int i = 2 * e.hole[s2][0] + s2, j = 2 * e.hole[s2][1] + s2;
                raw = phys_d(eri, a, b, i, j) - phys_d(eri, a, b, j, i);
            } else {
                raw = phys_d(eri, 2 * e.part[0][0], 2 * e.part[1][0] + 1, 2 * e.hole[0][0],
                             2 * e.hole[1][0] + 1);
            }
            v = (e.perm & 1) ? -raw : raw;
        }
        out[t] = v;
    }
}

__global__ void k_exc(const u64* bra, const u64* ket, i64 n, int32_t* deg, double* ph) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const ExcD e = analyze_d(bra[2 * t], bra[2 * t + 1], ket[2 * t], ket[2 * t + 1]);
        deg[t] = e.degree;
        ph[t] = e.degree > 2 ? 0.0 : ((e.perm & 1) ? -1.0 : 1.0);
    }
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_ham_diag(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, double* out, void* stream) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx != nullptr && (n == 0 || (dets && out)), DNQ_ERR_INVALID, "null argument");
    require(n >= 0, DNQ_ERR_INVALID, "negative size");
    if (n == 0) return DNQ_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> d(dets, 2 * n, s);
    check_orbitals(d.p, n, ctx->n, s);
    const bool dev_out = is_device_ptr(out);
    DBuf<double> tmp;
    double* o = out;
    if (!dev_out) {
        tmp.alloc(n, s);
        o = tmp.p;
    }
    launch_diag(ctx, d.p, n, o, s);
    if (!dev_out) copy_out(out, o, n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_elems(dnq_ctx_t ctx, const uint64_t* bra, const uint64_t* ket, int64_t n,
                  double* out, void* stream) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx != nullptr && (n == 0 || (bra && ket && out)), DNQ_ERR_INVALID, "null argument");
    if (n == 0) return DNQ_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> b(bra, 2 * n, s), k(ket, 2 * n, s);
    check_orbitals(b.p, n, ctx->n, s);
    check_orbitals(k.p, n, ctx->n, s);
    DBuf<double> tmp(n, s);
    k_elems<<<grid_for(n, 128), 128, 0, s>>>(ctx->view(), ctx->erid.p, b.p, k.p, n, tmp.p);
    DNQ_CHECK_LAUNCH();
    copy_out(out, tmp.p, n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_excitations(const uint64_t* bra, const uint64_t* ket, int64_t n, int32_t* degree,
                    double* phase, int device, void* stream) {
    DNQ_API_BEGIN
    require(n == 0 || (bra && ket && degree && phase), DNQ_ERR_INVALID, "null argument");
    if (n == 0) return DNQ_OK;
    DeviceGuard g(device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> b(bra, 2 * n, s), k(ket, 2 * n, s);
    DBuf<int32_t> d(n, s);
    DBuf<double> p(n, s);
    k_exc<<<grid_for(n), 256, 0, s>>>(b.p, k.p, n, d.p, p.p);
    DNQ_CHECK_LAUNCH();
    copy_out(degree, d.p, n, s);
    copy_out(phase, p.p, n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_build(dnq_ctx_t ctx, const uint64_t* dets_V, int64_t n_V, const uint64_t* dets_ext,
              int64_t n_ext, const double* psi, int n_orb, int policy, int use_heatbath,
              double eps1, int want_vp, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx && out, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(n_V >= 0 && n_ext >= 0, DNQ_ERR_INVALID, "negative size");
    require(policy >= 0 && policy <= 2, DNQ_ERR_INVALID, "invalid screening policy");
    require(n_orb >= 1 && n_orb <= ctx->n, DNQ_ERR_INVALID,
            "n_orb must be in [1, number of orbitals of the integral context]");
    if (policy == DNQ_POLICY_STATIC && use_heatbath)
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    if (policy == DNQ_POLICY_DYNAMIC) {
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
        require(n_V == 0 || psi, DNQ_ERR_INVALID, "size mismatch: dets_V and psi_v");
    }
    require(n_V == 0 || dets_V, DNQ_ERR_INVALID, "null determinant array");
    DeviceGuard g(ctx->device);
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    H->device = ctx->device;
    H->stream = (cudaStream_t)stream;
    if (g_build_opt) H->opt = *g_build_opt;   // a server's own options
    if (n_V > 0)
        build_ham(ctx, dets_V, n_V, dets_ext, n_ext, psi, n_orb, policy, use_heatbath, eps1,
                  want_vp != 0, (cudaStream_t)stream, H.get());
    *out = H.release();
    DNQ_API_END
}

int dnq_set_option(int option, int64_t value) {
    DNQ_API_BEGIN
    require(option >= 1 && option <= 8 && option != 6, DNQ_ERR_INVALID, "unknown option");
    require(value >= 0, DNQ_ERR_INVALID, "option value must be >= 0");
    if (option == 4)
        require(value == 0 || value == 4 || value == 8 || value == 16 || value == 32,
                DNQ_ERR_INVALID, "lanes per row must be 0, 4, 8, 16 or 32");
    if (option == 5)
        require(value == 0 || value == 1 || value == 2 || value == 4, DNQ_ERR_INVALID,
                "slots per lane must be 0, 1, 2 or 4");
    std::lock_guard<std::mutex> lk(g_opt_mu);
    Options& o = g_defaults;
    if (option == 1) o.force_walk = value != 0;
    if (option == 2) o.arena_chunk = value;
    if (option == 3) o.arena_cap = value;
    if (option == 4) o.spmv_lanes = (int)value;
    if (option == 5) o.spmv_unroll = (int)value;
    if (option == 7) o.partc_groupwalk = value != 0;
    if (option == 8) o.build_f32 = value != 0;
    DNQ_API_END
}

// The H.psi shape of one handle (DNQ_OPT_SPMV_LANES / DNQ_OPT_SPMV_UNROLL),
// leaving the defaults and other handles as they are.
int dnq_ham_set_option(dnq_ham_t h, int option, int64_t value) {
    DNQ_API_BEGIN
    require(h != nullptr, DNQ_ERR_INVALID, "null handle");
    require(option == DNQ_OPT_SPMV_LANES || option == DNQ_OPT_SPMV_UNROLL, DNQ_ERR_INVALID,
            "only the H.psi options (lanes, slots) apply to a built handle");
    if (option == DNQ_OPT_SPMV_LANES) {
        require(value == 0 || value == 4 || value == 8 || value == 16 || value == 32,
                DNQ_ERR_INVALID, "lanes per row must be 0, 4, 8, 16 or 32");
        h->opt.spmv_lanes = (int)value;
    } else {
        require(value == 0 || value == 1 || value == 2 || value == 4, DNQ_ERR_INVALID,
                "slots per lane must be 0, 1, 2 or 4");
        h->opt.spmv_unroll = (int)value;
    }
    DNQ_API_END
}

int dnq_ham_timings(dnq_ham_t h, double* ms8) {
    DNQ_API_BEGIN
    require(h && ms8, DNQ_ERR_INVALID, "null argument");
    for (int k = 0; k < 8; ++k) ms8[k] = h->t_ms[k];
    DNQ_API_END
}

int dnq_ham_destroy(dnq_ham_t h) {
    DNQ_API_BEGIN
    if (!h) return DNQ_OK;
    DeviceGuard g(h->device);
    cudaStream_t s = h->stream;
    delete h;
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_info(dnq_ham_t h, int64_t* info) {
    DNQ_API_BEGIN
    require(h && info, DNQ_ERR_INVALID, "null argument");
    info[0] = h->n_v;
    info[1] = h->vv.nnz;
    info[2] = h->n_p;
    info[3] = h->vp.nnz;
    info[4] = h->candidates;
    info[5] = (int64_t)h->bytes();
    DNQ_API_END
}

}  // extern "C"

namespace dnq {
namespace {
__global__ void k_expand_rows(const i64* rowptr, i64 nr, u32* rows) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nr;
         r += (i64)gridDim.x * blockDim.x)
        for (i64 k = rowptr[r]; k < rowptr[r + 1]; ++k) rows[k] = (u32)r;
}
}  // namespace
}  // namespace dnq

extern "C" {

int dnq_ham_copy_coo(dnq_ham_t h, int block, uint32_t* rows, uint32_t* cols, double* vals,
                     void* stream) {
    DNQ_API_BEGIN
    require(h != nullptr && (block == 0 || block == 1), DNQ_ERR_INVALID, "invalid block");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    Csr& m = block == 0 ? h->vv : h->vp;
    if (m.nnz == 0) return DNQ_OK;
    ensure_sorted(m, s);
    if (rows) {
        DBuf<u32> r(m.nnz, s);
        k_expand_rows<<<grid_for(m.nr), 256, 0, s>>>(m.rowptr.p, m.nr, r.p);
        DNQ_CHECK_LAUNCH();
        copy_out(rows, r.p, m.nnz, s);
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    copy_out(cols, m.col.p, m.nnz, s);
    copy_out(vals, m.val.p, m.nnz, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_copy_csr(dnq_ham_t h, int block, int64_t* row_ptr, uint32_t* cols, double* vals,
                     void* stream) {
    DNQ_API_BEGIN
    require(h != nullptr && (block == 0 || block == 1), DNQ_ERR_INVALID, "invalid block");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    Csr& m = block == 0 ? h->vv : h->vp;
    ensure_sorted(m, s);
    if (m.nr > 0) copy_out(row_ptr, m.rowptr.p, m.nr + 1, s);
    else if (row_ptr) {
        const int64_t z = 0;
        DNQ_CUDA(cudaMemcpyAsync(row_ptr, &z, 8, cudaMemcpyDefault, s));
    }
    copy_out(cols, m.col.p, m.nnz, s);
    copy_out(vals, m.val.p, m.nnz, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_copy_dets_p(dnq_ham_t h, uint64_t* dets, void* stream) {
    DNQ_API_BEGIN
    require(h != nullptr, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    copy_out(dets, (const uint64_t*)h->dets_p.p, 2 * (i64)h->words * h->n_p, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_p_diag(dnq_ham_t h, dnq_ctx_t ctx, double* out, void* stream) {
    DNQ_API_BEGIN
    require(h && ctx, DNQ_ERR_INVALID, "null argument");
    if (h->n_p == 0) return DNQ_OK;
    require(out != nullptr, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const bool dev_out = is_device_ptr(out);
    DBuf<double> tmp;
    double* o = out;
    if (!dev_out) {
        tmp.alloc(h->n_p, s);
        o = tmp.p;
    }
    if (h->words == 2) launch_wide_diag(ctx, (const u64*)h->dets_p.p, h->n_p, o, s);
    else launch_diag(ctx, (const u64*)h->dets_p.p, h->n_p, o, s);
    if (!dev_out) copy_out(out, o, h->n_p, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_copy_diag(dnq_ham_t h, double* diag, void* stream) {
    DNQ_API_BEGIN
    require(h != nullptr, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    copy_out(diag, h->diag.p, h->n_v, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

}  // extern "C"
