// proxy.cu -- proxy operator on T = V + P (detnqs/operator/kernel.py:87-145):
//   yv = H_VV xv + H_VP xp
//   yp = H_PV xv + diag(H_PP) xp
// H_PV is the transpose of H_VP, built once per handle on first use.

#include <memory>

#include "ham.cuh"
#include "prim.cuh"

namespace dnq {

void spmv_block(const dnq_ham_s* h, const Csr& m, const double* x, double* y,
                const double* yadd, int precision, cudaStream_t s, float* x32,
                const double* diag);
void to_f32(const double* x, i64 n, float* o, cudaStream_t s);

namespace {

// Row of every entry: one thread per entry, binary search of the row
// pointers (rows of any length, no serial walk).
__global__ void k_rows_of(const i64* rowptr, i64 nr, i64 nnz, u32* rows) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < nnz;
         k += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = nr;   // last r with rowptr[r] <= k
        while (hi - lo > 1) {
            const i64 mid = (lo + hi) >> 1;
            if (rowptr[mid] <= k) lo = mid; else hi = mid;
        }
        rows[k] = (u32)lo;
    }
}

__global__ void k_gather_t(const u32* perm, const u32* rows, const double* val, i64 n,
                           u32* tcol, double* tval) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 k = perm[t];
        tcol[t] = rows[k];
        tval[t] = val[k];
    }
}

// row pointer of the transposed block from the sorted column keys
__global__ void k_bounds(const u32* skey, i64 n, i64 ncols, i64* rowptr) {
    for (i64 c = blockIdx.x * (i64)blockDim.x + threadIdx.x; c <= ncols;
         c += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = n;
        while (lo < hi) {
            const i64 mid = (lo + hi) / 2;
            if ((i64)skey[mid] < c) lo = mid + 1; else hi = mid;
        }
        rowptr[c] = lo;
    }
}

__global__ void k_diag_mul_add(const double* d, const double* x, i64 n, double* y) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        y[t] = d[t] * x[t];
}

int gsz(i64 n) {
    i64 b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

}  // namespace

void transpose_csr(const Csr& a, Csr& t, cudaStream_t s) {
    t.nr = a.nc;
    t.nc = a.nr;
    t.nnz = a.nnz;
    t.rowptr.alloc(t.nr + 1, s);
    t.col.alloc(a.nnz, s);
    t.val.alloc(a.nnz, s);
    if (a.nnz == 0) {
        DNQ_CUDA(cudaMemsetAsync(t.rowptr.p, 0, (t.nr + 1) * sizeof(i64), s));
        return;
    }
    DBuf<u32> rows(a.nnz, s), perm2(a.nnz, s), skey(a.nnz, s);
    k_rows_of<<<gsz(a.nnz), 256, 0, s>>>(a.rowptr.p, a.nr, a.nnz, rows.p);
    DNQ_CHECK_LAUNCH();
    {   // stable by column: rows stay ascending inside each column
        int b = 1;
        while (b < 32 && ((i64)1 << b) < a.nc) ++b;
        const int bits[1] = {b};
        prim::radix_sort<u32, u32>(a.col.p, skey.p, nullptr, perm2.p, a.nnz, bits, s);
    }
    k_gather_t<<<gsz(a.nnz), 256, 0, s>>>(perm2.p, rows.p, a.val.p, a.nnz, t.col.p, t.val.p);
    DNQ_CHECK_LAUNCH();
    k_bounds<<<gsz(t.nr + 1), 256, 0, s>>>(skey.p, a.nnz, t.nr, t.rowptr.p);
    DNQ_CHECK_LAUNCH();
}

namespace {
// 0.5 (A + A^T) of a square block with column-sorted rows: one thread merges
// row r of A with row r of A^T (both sorted); absent entries count as 0.
template <bool FILL>
__global__ void k_sym_merge(const i64* arp, const u32* acol, const double* aval, const i64* trp,
                            const u32* tcol, const double* tval, i64 n, u32* cnt,
                            const i64* off, u32* ocol, double* oval) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < n;
         r += (i64)gridDim.x * blockDim.x) {
        i64 p = arp[r], pe = arp[r + 1], q = trp[r], qe = trp[r + 1];
        i64 w = FILL ? off[r] : 0;
        u32 c = 0;
        while (p < pe || q < qe) {
            u32 col;
            double x = 0.0, y = 0.0;
            if (q >= qe || (p < pe && acol[p] < tcol[q])) {
                col = acol[p];
                x = aval[p++];
            } else if (p >= pe || tcol[q] < acol[p]) {
                col = tcol[q];
                y = tval[q++];
            } else {
                col = acol[p];
                x = aval[p++];
                y = tval[q++];
            }
            if (FILL) {
                ocol[w] = col;
                oval[w] = 0.5 * (x + y);
                ++w;
            }
            ++c;
        }
        if (!FILL) cnt[r] = c;
    }
}
}  // namespace

void symmetrize_csr(Csr& a, Csr& out, cudaStream_t s) {
    ensure_sorted(a, s);
    Csr t;
    transpose_csr(a, t, s);
    const i64 n = a.nr;
    DBuf<u32> cnt(n + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cnt.p + n, 0, 4, s));
    const int grid = gsz(n);
    k_sym_merge<false><<<grid, 256, 0, s>>>(a.rowptr.p, a.col.p, a.val.p, t.rowptr.p, t.col.p,
                                            t.val.p, n, cnt.p, nullptr, nullptr, nullptr);
    DNQ_CHECK_LAUNCH();
    out.nr = out.nc = n;
    out.rowptr.alloc(n + 1, s);
    prim::scan<u32, i64, false>(cnt.p, out.rowptr.p, n + 1, s);
    DNQ_CUDA(cudaMemcpyAsync(&out.nnz, out.rowptr.p + n, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    out.col.alloc(out.nnz, s);
    out.val.alloc(out.nnz, s);
    k_sym_merge<true><<<grid, 256, 0, s>>>(a.rowptr.p, a.col.p, a.val.p, t.rowptr.p, t.col.p,
                                           t.val.p, n, nullptr, out.rowptr.p, out.col.p,
                                           out.val.p);
    DNQ_CHECK_LAUNCH();
    out.sorted = true;
    DNQ_CUDA(cudaStreamSynchronize(s));
}

}  // namespace dnq

namespace dnq {
Csr& pv_block(dnq_ham_s* h, cudaStream_t s);
void ensure_f32_all(Csr& m, cudaStream_t s);
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_ham_symmetrize(dnq_ham_t h, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require(h && out, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(h->vv.nr == h->vv.nc, DNQ_ERR_INVALID, "block is not square");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    H->device = h->device;
    H->stream = s;
    H->n_v = h->n_v;
    ensure_compact(h->vv, s);
    symmetrize_csr(h->vv, H->vv, s);
    *out = H.release();
    DNQ_API_END
}

int dnq_ham_proxy_spmv(dnq_ham_t h, const double* xv, const double* xp, const double* diag_p,
                       double* yv, double* yp, int precision, void* stream) {
    DNQ_API_BEGIN
    require(h && xv && yv, DNQ_ERR_INVALID, "null argument");
    require(h->n_p == 0 || (xp && yp && diag_p), DNQ_ERR_INVALID, "null P-space argument");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 nv = h->n_v, np = h->n_p;
    DIn<double> xvd(xv, nv, s), xpd(xp, np, s), dpd(diag_p, np, s);
    DBuf<double> yvd(nv, s), ypd(np, s), tmp(nv, s);
    if (precision == DNQ_F64) {
        spmv_block(h, h->vp, xpd.p, tmp.p, nullptr, DNQ_F64, s, nullptr, nullptr);
        spmv_block(h, h->vv, xvd.p, yvd.p, tmp.p, DNQ_F64, s, nullptr, nullptr);
        if (np) {
            Csr& pv = pv_block(h, s);
            DBuf<double> dterm(np, s);
            k_diag_mul_add<<<gsz(np), 256, 0, s>>>(dpd.p, xpd.p, np, dterm.p);
            DNQ_CHECK_LAUNCH();
            spmv_block(h, pv, xvd.p, ypd.p, dterm.p, DNQ_F64, s, nullptr, nullptr);
        }
    } else {
        // FP32 values for all three blocks; diagonal terms in FP64.
        DBuf<float> xv32(nv, s), xp32(np, s);
        to_f32(xvd.p, nv, xv32.p, s);
        to_f32(xpd.p, np, xp32.p, s);
        if (!h->vv.f32_ready() || h->diag_op.n != (size_t)h->n_v)
            make_f32(h->vv, s, &h->diag_op);
        ensure_f32_all(h->vp, s);
        spmv_block(h, h->vp, xpd.p, tmp.p, nullptr, DNQ_F32, s, xp32.p, nullptr);
        spmv_block(h, h->vv, xvd.p, yvd.p, tmp.p, DNQ_F32, s, xv32.p, h->diag_op.p);
        if (np) {
            Csr& pv = pv_block(h, s);
            ensure_f32_all(pv, s);
            DBuf<double> dterm(np, s);
            k_diag_mul_add<<<gsz(np), 256, 0, s>>>(dpd.p, xpd.p, np, dterm.p);
            DNQ_CHECK_LAUNCH();
            spmv_block(h, pv, xvd.p, ypd.p, dterm.p, DNQ_F32, s, xv32.p, nullptr);
        }
    }
    DNQ_CHECK_LAUNCH();
    copy_out(yv, yvd.p, nv, s);
    copy_out(yp, ypd.p, np, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

}  // extern "C"
