// spmv.cu -- H.psi on the device (replaces the SciPy CSR matvec of
// detnqs/operator/kernel.py:75-78 and the proxy operator of :127-139) and
// the local-energy / Rayleigh-quotient reductions.
//
// FP64 operator: y_i = sum_k H_ik x_k with FP64 values, FP64 x.
// FP32 operator: off-diagonal values and x stored in FP32; products and sums
// are kept exact to second order with TwoProduct (fmaf residual) and TwoSum
// (Knuth) per lane, the per-lane (sum, error) pairs are combined with TwoSum
// across the row group, and the FP64 diagonal term diag_i * x_i is added in
// FP64 (Ogita, Rump, Oishi, "Accurate sum and dot product", SIAM J. Sci.
// Comput. 26 (2005), Dot2).
// Reductions x.Hx and x.x use the same Dot2 scheme in FP64.
#include <cub/cub.cuh>

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

// One group of G lanes per row (G in {4, 8, 16, 32}); each lane reads 4
// consecutive entries per step with 128-bit loads (cols: one uint4; values:
// two double2 / one float4), starting from the row start rounded down to a
// multiple of 4 and masking entries outside the row, so a warp streams 128
// entries per step.  The tail of the arrays is read with scalar loads.
template <int G>
__global__ void __launch_bounds__(256)
k_spmv_f64(const i64* __restrict__ rp, const u32* __restrict__ col,
           const double* __restrict__ val, const double* __restrict__ x, i64 nr, i64 nnz,
           double* __restrict__ y, const double* __restrict__ yadd) {
    const i64 gid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const i64 ngroups = (gridDim.x * (i64)blockDim.x) / G;
    const i64 rounds = (nr + ngroups - 1) / ngroups;
    for (i64 it = 0; it < rounds; ++it) {
        const i64 r = gid + it * ngroups;
        double acc = 0.0;
        if (r < nr) {
            const i64 b = __ldg(&rp[r]), e = __ldg(&rp[r + 1]);
            for (i64 k = (b & ~3ll) + 4 * sub; k < e; k += 4 * G) {
                u32 c[4];
                double v[4];
                if (k + 3 < nnz) {
                    const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(col + k));
                    const double2 v01 = __ldg(reinterpret_cast<const double2*>(val + k));
                    const double2 v23 = __ldg(reinterpret_cast<const double2*>(val + k + 2));
                    c[0] = c4.x; c[1] = c4.y; c[2] = c4.z; c[3] = c4.w;
                    v[0] = v01.x; v[1] = v01.y; v[2] = v23.x; v[3] = v23.y;
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        c[q] = k + q < nnz ? __ldg(&col[k + q]) : 0u;
                        v[q] = k + q < nnz ? __ldg(&val[k + q]) : 0.0;
                    }
                }
                double xv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const bool in = k + q >= b && k + q < e;
                    xv[q] = in ? __ldg(&x[c[q]]) : 0.0;
                    if (!in) v[q] = 0.0;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) acc = fma(v[q], xv[q], acc);
            }
        }
#pragma unroll
        for (int o = G / 2; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (sub == 0 && r < nr) y[r] = yadd ? acc + yadd[r] : acc;
    }
}

template <int G>
__global__ void __launch_bounds__(256)
k_spmv_f32c(const i64* __restrict__ rp, const u32* __restrict__ col,
            const float* __restrict__ val, const float* __restrict__ x32,
            const double* __restrict__ diag, const double* __restrict__ x, i64 nr, i64 nnz,
            double* __restrict__ y, const double* __restrict__ yadd) {
    const i64 gid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const i64 ngroups = (gridDim.x * (i64)blockDim.x) / G;
    const i64 rounds = (nr + ngroups - 1) / ngroups;
    for (i64 it = 0; it < rounds; ++it) {
        const i64 r = gid + it * ngroups;
        Dot2<float> acc;
        if (r < nr) {
            const i64 b = __ldg(&rp[r]), e = __ldg(&rp[r + 1]);
            for (i64 k = (b & ~3ll) + 4 * sub; k < e; k += 4 * G) {
                u32 c[4];
                float v[4];
                if (k + 3 < nnz) {
                    const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(col + k));
                    const float4 v4 = __ldg(reinterpret_cast<const float4*>(val + k));
                    c[0] = c4.x; c[1] = c4.y; c[2] = c4.z; c[3] = c4.w;
                    v[0] = v4.x; v[1] = v4.y; v[2] = v4.z; v[3] = v4.w;
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        c[q] = k + q < nnz ? __ldg(&col[k + q]) : 0u;
                        v[q] = k + q < nnz ? __ldg(&val[k + q]) : 0.0f;
                    }
                }
                float xv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const bool in = k + q >= b && k + q < e;
                    xv[q] = in ? __ldg(&x32[c[q]]) : 0.0f;
                    if (!in) v[q] = 0.0f;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) acc.add_prod(v[q], xv[q]);
            }
        }
#pragma unroll
        for (int o = G / 2; o; o >>= 1) acc.merge(shfl_xor(acc, o, 0xffffffffu));
        if (sub == 0 && r < nr) {
            double v = (double)acc.s + (double)acc.c;
            if (diag) v += diag[r] * x[r];
            y[r] = yadd ? v + yadd[r] : v;
        }
    }
}

__global__ void k_to_f32_vec(const double* x, i64 n, float* o) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        o[t] = (float)x[t];
}

// Per-block Dot2 partials of x.y and x.x; eloc = y / x.
__global__ void k_energy_partials(const double* x, const double* y, i64 n, double* eloc,
                                  double* part) {
    Dot2<double> num, den;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const double xv = x[t], yv = y[t];
        num.add_prod(xv, yv);
        den.add_prod(xv, xv);
        if (eloc) eloc[t] = yv / xv;
    }
    for (int o = 16; o; o >>= 1) {
        num.merge(shfl_xor(num, o, 0xffffffffu));
        den.merge(shfl_xor(den, o, 0xffffffffu));
    }
    __shared__ double sh[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = num.s; sh[1][w] = num.c; sh[2][w] = den.s; sh[3][w] = den.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Dot2<double> a, b;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            Dot2<double> t1, t2;
            t1.s = sh[0][k]; t1.c = sh[1][k]; t2.s = sh[2][k]; t2.c = sh[3][k];
            a.merge(t1);
            b.merge(t2);
        }
        part[4 * blockIdx.x + 0] = a.s;
        part[4 * blockIdx.x + 1] = a.c;
        part[4 * blockIdx.x + 2] = b.s;
        part[4 * blockIdx.x + 3] = b.c;
    }
}

__global__ void k_energy_final(const double* part, int nb, double* out2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Dot2<double> a, b;
    for (int k = 0; k < nb; ++k) {
        Dot2<double> t1, t2;
        t1.s = part[4 * k]; t1.c = part[4 * k + 1]; t2.s = part[4 * k + 2]; t2.c = part[4 * k + 3];
        a.merge(t1);
        b.merge(t2);
    }
    out2[0] = a.value();
    out2[1] = b.value();
}

int group_for(const Csr& m) {
    const double avg = m.nr ? (double)m.nnz / (double)m.nr : 0.0;
    if (avg >= 96) return 32;
    if (avg >= 48) return 16;
    if (avg >= 24) return 8;
    return 4;
}

int spmv_grid(int device) { return sm_count(device) * 8; }

}  // namespace

// Same as spmv_block with the lanes-per-row group given (0 = automatic).
void spmv_block_g(const dnq_ham_s* h, const Csr& m, const double* x, double* y, int precision,
                  cudaStream_t s, const float* x32, const float* val32, const double* diag,
                  int G, int device) {
    if (m.nr == 0) return;
    if (G == 0) G = group_for(m);
    const int grid = spmv_grid(device), bs = 256;
    (void)h;
    if (precision == DNQ_F64 || m.nnz == 0) {
        switch (G) {
            case 32: k_spmv_f64<32><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, nullptr); break;
            case 16: k_spmv_f64<16><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, nullptr); break;
            case 8: k_spmv_f64<8><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, nullptr); break;
            default: k_spmv_f64<4><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, nullptr); break;
        }
    } else {
        switch (G) {
            case 32: k_spmv_f32c<32><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, val32, x32, diag, x, m.nr, m.nnz, y, nullptr); break;
            case 16: k_spmv_f32c<16><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, val32, x32, diag, x, m.nr, m.nnz, y, nullptr); break;
            case 8: k_spmv_f32c<8><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, val32, x32, diag, x, m.nr, m.nnz, y, nullptr); break;
            default: k_spmv_f32c<4><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, val32, x32, diag, x, m.nr, m.nnz, y, nullptr); break;
        }
    }
    DNQ_CHECK_LAUNCH();
}

// y (+)= M x for one block; x FP64 device, y FP64 device.
void spmv_block(const dnq_ham_s* h, const Csr& m, const double* x, double* y,
                const double* yadd, int precision, cudaStream_t s, float* x32,
                const double* diag) {
    if (m.nr == 0) return;
    const int G = group_for(m);
    const int grid = spmv_grid(h->device), bs = 256;
    if (precision == DNQ_F64 || m.nnz == 0) {
        switch (G) {
            case 32: k_spmv_f64<32><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, yadd); break;
            case 16: k_spmv_f64<16><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, yadd); break;
            case 8: k_spmv_f64<8><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, yadd); break;
            default: k_spmv_f64<4><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val.p, x, m.nr, m.nnz, y, yadd); break;
        }
    } else {
        switch (G) {
            case 32: k_spmv_f32c<32><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val32.p, x32, diag, x, m.nr, m.nnz, y, yadd); break;
            case 16: k_spmv_f32c<16><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val32.p, x32, diag, x, m.nr, m.nnz, y, yadd); break;
            case 8: k_spmv_f32c<8><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val32.p, x32, diag, x, m.nr, m.nnz, y, yadd); break;
            default: k_spmv_f32c<4><<<grid, bs, 0, s>>>(m.rowptr.p, m.col.p, m.val32.p, x32, diag, x, m.nr, m.nnz, y, yadd); break;
        }
    }
    DNQ_CHECK_LAUNCH();
}

void to_f32(const double* x, i64 n, float* o, cudaStream_t s) {
    if (n == 0) return;
    k_to_f32_vec<<<1184, 256, 0, s>>>(x, n, o);
    DNQ_CHECK_LAUNCH();
}

void energy_reduce(const double* x, const double* y, i64 n, double* eloc, double* out2_dev,
                   cudaStream_t s) {
    const int nb = 592;
    DBuf<double> part(4 * nb, s);
    k_energy_partials<<<nb, 256, 0, s>>>(x, y, n, eloc, part.p);
    DNQ_CHECK_LAUNCH();
    k_energy_final<<<1, 32, 0, s>>>(part.p, nb, out2_dev);
    DNQ_CHECK_LAUNCH();
}

// Same reduction with caller-provided partials (4 * nb doubles) and result
// slot: launches only, allocates nothing.
void energy_reduce_into(const double* x, const double* y, i64 n, double* eloc, double* part,
                        int nb, double* out2_dev, cudaStream_t s) {
    k_energy_partials<<<nb, 256, 0, s>>>(x, y, n, eloc, part);
    DNQ_CHECK_LAUNCH();
    k_energy_final<<<1, 32, 0, s>>>(part, nb, out2_dev);
    DNQ_CHECK_LAUNCH();
}

// Transposed copy of a CSR block (H_PV from H_VP), rows ascending inside
// each column.
void transpose_csr(const Csr& a, Csr& t, cudaStream_t s);

// H_PV (transpose of H_VP), built once per handle.
Csr& pv_block(dnq_ham_s* h, cudaStream_t s) {
    if (!h->pv_ready) {
        transpose_csr(h->vp, h->pv, s);
        h->pv_ready = true;
    }
    return h->pv;
}

namespace {
__global__ void k_all_f32(const double* v, i64 n, float* o) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        o[t] = (float)v[t];
}
}  // namespace

// FP32 copy of every value of a rectangular block (no diagonal split).
void ensure_f32_all(Csr& m, cudaStream_t s) {
    if (m.val32.n == (size_t)m.nnz && m.nnz) return;
    m.val32.alloc(m.nnz, s);
    if (m.nnz) {
        k_all_f32<<<1184, 256, 0, s>>>(m.val.p, m.nnz, m.val32.p);
        DNQ_CHECK_LAUNCH();
    }
}

// Prepare the FP32 operator buffers of the V block.
void ensure_f32(dnq_ham_s* h, cudaStream_t s) {
    if (h->vv.val32.n != (size_t)h->vv.nnz || h->diag_op.n != (size_t)h->n_v)
        make_f32(h->vv, s, &h->diag_op);
    if ((i64)h->x32.n < h->n_v) h->x32.alloc(h->n_v, s);
}

}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_ham_spmv(dnq_ham_t h, const double* x, double* y, int precision, void* stream) {
    DNQ_API_BEGIN
    require(h && x && y, DNQ_ERR_INVALID, "null argument");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 n = h->n_v;
    if (n == 0) return DNQ_OK;
    DIn<double> xd(x, n, s);
    const bool dev_out = is_device_ptr(y);
    DBuf<double> ybuf;
    double* yd = y;
    if (!dev_out) { ybuf.alloc(n, s); yd = ybuf.p; }
    if (precision == DNQ_F32) {
        ensure_f32(h, s);
        to_f32(xd.p, n, h->x32.p, s);
        spmv_block(h, h->vv, xd.p, yd, nullptr, DNQ_F32, s, h->x32.p, h->diag_op.p);
    } else {
        spmv_block(h, h->vv, xd.p, yd, nullptr, DNQ_F64, s, nullptr, nullptr);
    }
    if (!dev_out) {
        copy_out(y, yd, n, s);
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    DNQ_API_END
}

int dnq_ham_block_spmv(dnq_ham_t h, int block, const double* x, double* y, int precision,
                       void* stream) {
    DNQ_API_BEGIN
    require(h && x && y, DNQ_ERR_INVALID, "null argument");
    require(block >= 0 && block <= 2, DNQ_ERR_INVALID, "invalid block");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    if (block == 0) return dnq_ham_spmv(h, x, y, precision, stream);
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const Csr& m = block == 1 ? h->vp : pv_block(h, s);
    const i64 nin = block == 1 ? h->n_p : h->n_v;
    const i64 nout = block == 1 ? h->n_v : h->n_p;
    if (nout == 0) return DNQ_OK;
    DIn<double> xd(x, nin, s);
    const bool dev_out = is_device_ptr(y);
    DBuf<double> ybuf;
    double* yd = y;
    if (!dev_out) { ybuf.alloc(nout, s); yd = ybuf.p; }
    if (m.nnz == 0) {
        DNQ_CUDA(cudaMemsetAsync(yd, 0, nout * 8, s));
    } else if (precision == DNQ_F32) {
        Csr& mm = const_cast<Csr&>(m);
        ensure_f32_all(mm, s);
        DBuf<float> x32(nin, s);
        to_f32(xd.p, nin, x32.p, s);
        spmv_block(h, mm, xd.p, yd, nullptr, DNQ_F32, s, x32.p, nullptr);
    } else {
        spmv_block(h, m, xd.p, yd, nullptr, DNQ_F64, s, nullptr, nullptr);
    }
    if (!dev_out) copy_out(y, yd, nout, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

int dnq_ham_local_energy(dnq_ham_t h, const double* x, double* eloc, double* out2,
                         int precision, void* stream) {
    DNQ_API_BEGIN
    require(h && x && out2, DNQ_ERR_INVALID, "null argument");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 n = h->n_v;
    if (n == 0) {
        double z[2] = {0.0, 0.0};
        DNQ_CUDA(cudaMemcpyAsync(out2, z, 16, cudaMemcpyDefault, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        return DNQ_OK;
    }
    DIn<double> xd(x, n, s);
    DBuf<double> y(n, s), o2(2, s);
    if (precision == DNQ_F32) {
        ensure_f32(h, s);
        to_f32(xd.p, n, h->x32.p, s);
        spmv_block(h, h->vv, xd.p, y.p, nullptr, DNQ_F32, s, h->x32.p, h->diag_op.p);
    } else {
        spmv_block(h, h->vv, xd.p, y.p, nullptr, DNQ_F64, s, nullptr, nullptr);
    }
    const bool dev_eloc = eloc && is_device_ptr(eloc);
    DBuf<double> ebuf;
    double* ed = nullptr;
    if (eloc) {
        if (dev_eloc) ed = eloc;
        else { ebuf.alloc(n, s); ed = ebuf.p; }
    }
    energy_reduce(xd.p, y.p, n, ed, o2.p, s);
    if (eloc && !dev_eloc) copy_out(eloc, ed, n, s);
    copy_out(out2, o2.p, 2, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

}  // extern "C"
