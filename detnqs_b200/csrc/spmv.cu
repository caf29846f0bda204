// spmv.cu -- H.psi on the device (replaces the SciPy CSR matvec of
// detnqs/operator/kernel.py:75-78 and the proxy operator of :127-139) and
// the local-energy / Rayleigh-quotient reductions.
//
// FP64 operator: y_i = sum_k H_ik x_k with FP64 values, FP64 x.
// FP32 operator: off-diagonal values and x stored in FP32; each lane sums
// its products with Kahan's compensated summation, every product entering
// through one fused multiply-add (AccF32 in spmv.cuh), the per-lane
// (sum, compensation) pairs are combined with TwoSum across the row group,
// and the FP64 diagonal term diag_i * x_i is added in FP64.
// Reductions x.Hx and x.x use Dot2 in FP64 (Ogita, Rump, Oishi, "Accurate
// sum and dot product", SIAM J. Sci. Comput. 26 (2005)).

#include "ham.cuh"
#include "spmv.cuh"

namespace dnq {
namespace {

// One group of G lanes per row (G in {4, 8, 16, 32}).  Lane `sub` owns the
// 4-entry slots k = (b & ~3) + 4 sub + 4 G t, t = 0, 1, ...: it reads each
// slot with 128-bit loads (cols: one uint4; values: two double2 or one
// float4), masks entries outside [b, e), and accumulates its slots in
// ascending t; the G lane sums are then combined by a butterfly.  U slots
// are loaded before any is used, so a lane keeps U column/value loads and
// 4U gathers of x in flight; the order of accumulation does not depend on U
// (results are identical for every U).  The last entries of the arrays are
// read with scalar loads.
//   T = double: y_r = sum H_rk x_k                         (val, x)
//   T = float : y_r = Kahan sum of val32 * x32 + diag_r x_r (FP32
//               off-diagonal values, FP64 diagonal term)
template <int G, int U, class T, class Acc>
__device__ __forceinline__ Acc row_acc(const i64* __restrict__ rs, const i64* __restrict__ re,
                                       const u32* __restrict__ col, const T* __restrict__ val,
                                       const T* __restrict__ xg, i64 r, bool valid, i64 nnz,
                                       int sub) {
    Acc acc;
    if (valid) {
        const i64 b = __ldg(&rs[r]), e = __ldg(&re[r]);
        for (i64 k0 = (b & ~3ll) + 4 * sub; k0 < e; k0 += 4 * G * U) {
            u32 c[U][4];
            T v[U][4];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const i64 k = k0 + (i64)u * 4 * G;
                if (k + 3 < nnz && k < e) {
                    const uint4 c4 = __ldcs(reinterpret_cast<const uint4*>(col + k));
                    c[u][0] = c4.x; c[u][1] = c4.y; c[u][2] = c4.z; c[u][3] = c4.w;
                    load4(val + k, v[u]);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const bool ok = k < e && k + q < nnz;
                        c[u][q] = ok ? __ldg(&col[k + q]) : 0u;
                        v[u][q] = ok ? __ldg(&val[k + q]) : T(0);
                    }
                }
            }
            T xv[U][4];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const i64 kk = k0 + (i64)u * 4 * G + q;
                    const bool in = kk >= b && kk < e;
                    xv[u][q] = in ? __ldg(&xg[c[u][q]]) : T(0);
                    if (!in) v[u][q] = T(0);
                }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (k0 + (i64)u * 4 * G < e) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc.add_prod(v[u][q], xv[u][q]);
                }
        }
    }
    acc.reduce(G);
    return acc;
}

template <int G, int U, class T, class Acc>
__global__ void __launch_bounds__(256)
k_spmv(const i64* __restrict__ rs, const i64* __restrict__ re, const u32* __restrict__ col,
       const T* __restrict__ val, const T* __restrict__ xg, const double* __restrict__ diag,
       const double* __restrict__ x, i64 nr, i64 nnz, double* __restrict__ y,
       const double* __restrict__ yadd) {
    const i64 gid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const i64 ngroups = (gridDim.x * (i64)blockDim.x) / G;
    const i64 rounds = (nr + ngroups - 1) / ngroups;
    for (i64 it = 0; it < rounds; ++it) {
        const i64 r = gid + it * ngroups;
        const Acc acc = row_acc<G, U, T, Acc>(rs, re, col, val, xg, r, r < nr, nnz, sub);
        if (sub == 0 && r < nr) {
            double v = acc.value();
            if (diag) v += diag[r] * x[r];
            y[r] = yadd ? v + yadd[r] : v;
        }
    }
}

// Many independent operators in one launch: blockIdx.y selects the
// descriptor; every row is computed exactly as by k_spmv with the same
// (G, U), so a result does not depend on the other members of the group.
template <int G, int U, class T, class Acc>
__global__ void __launch_bounds__(256) k_spmv_grouped(const SpmvDesc* __restrict__ descs) {
    const SpmvDesc d = descs[blockIdx.y];
    const T* val = static_cast<const T*>(d.val);
    const T* xg = static_cast<const T*>(d.xg);
    const i64 gid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const i64 ngroups = (gridDim.x * (i64)blockDim.x) / G;
    const i64 rounds = (d.nr + ngroups - 1) / ngroups;
    for (i64 it = 0; it < rounds; ++it) {
        const i64 r = gid + it * ngroups;
        const Acc acc =
            row_acc<G, U, T, Acc>(d.rp, d.re, d.col, val, xg, r, r < d.nr, d.nnz, sub);
        if (sub == 0 && r < d.nr) {
            double v = acc.value();
            if (d.diag) v += d.diag[r] * d.x[r];
            d.y[r] = v;
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

// The partials merged by one thread in block order; the block stages them in
// shared memory first (1024 at a time), so the serial merge waits on no
// global load.
constexpr int kFinalStage = 1024;
__global__ void __launch_bounds__(256) k_energy_final(const double* part, int nb, double* out2) {
    __shared__ double st[4 * kFinalStage];
    Dot2<double> a, b;
    for (int k0 = 0; k0 < nb; k0 += kFinalStage) {
        const int m = min(kFinalStage, nb - k0);
        for (int i = threadIdx.x; i < 4 * m; i += blockDim.x) st[i] = part[4 * k0 + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < m; ++k) {
                Dot2<double> t1, t2;
                t1.s = st[4 * k]; t1.c = st[4 * k + 1]; t2.s = st[4 * k + 2]; t2.c = st[4 * k + 3];
                a.merge(t1);
                b.merge(t2);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out2[0] = a.value();
        out2[1] = b.value();
    }
}

int group_for(const Csr& m) {
    const double avg = m.nr ? (double)m.nnz / (double)m.nr : 0.0;
    if (avg >= 96) return 32;
    if (avg >= 48) return 16;
    if (avg >= 24) return 8;
    return 4;
}

// Slots in flight per lane: as many as the average row fills, at most 4.
int unroll_for(const Csr& m, int G) {
    const double avg = m.nr ? (double)m.nnz / (double)m.nr : 0.0;
    const double slots = avg / (4.0 * G);
    if (slots >= 4) return 4;
    if (slots >= 2) return 2;
    return 1;
}

template <class K>
int blocks_for(K kern, int device) {
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
    return std::max(1, per_sm) * sm_count(device);
}

template <int G, int U>
void launch_gu(const Csr& m, const double* x, double* y, const double* yadd, int precision,
               const float* x32, const float* val32, const double* diag, int device,
               cudaStream_t s) {
    if (precision == DNQ_F64 || m.nnz == 0) {
        auto kern = k_spmv<G, U, double, AccF64>;
        kern<<<blocks_for(kern, device), 256, 0, s>>>(m.row_start(), m.row_end(), m.col.p,
                                                      m.val.p, x, nullptr, x, m.nr, m.span(), y,
                                                      yadd);
    } else {
        auto kern = k_spmv<G, U, float, AccF32>;
        kern<<<blocks_for(kern, device), 256, 0, s>>>(m.row_start(), m.row_end(), m.col.p, val32,
                                                      x32, diag, x, m.nr, m.span(), y, yadd);
    }
}

template <int G>
void launch_g(int U, const Csr& m, const double* x, double* y, const double* yadd,
              int precision, const float* x32, const float* val32, const double* diag,
              int device, cudaStream_t s) {
    switch (U) {
        case 4: launch_gu<G, 4>(m, x, y, yadd, precision, x32, val32, diag, device, s); break;
        case 2: launch_gu<G, 2>(m, x, y, yadd, precision, x32, val32, diag, device, s); break;
        default: launch_gu<G, 1>(m, x, y, yadd, precision, x32, val32, diag, device, s); break;
    }
}

// G lanes per row and U slots per lane; 0 = by the average row length.
void launch_spmv(const Csr& m, const double* x, double* y, const double* yadd, int precision,
                 const float* x32, const float* val32, const double* diag, int G, int U,
                 int device, cudaStream_t s) {
    if (m.nr == 0) return;
    if (G == 0) G = group_for(m);
    if (U == 0) U = unroll_for(m, G);
    switch (G) {
        case 32: launch_g<32>(U, m, x, y, yadd, precision, x32, val32, diag, device, s); break;
        case 16: launch_g<16>(U, m, x, y, yadd, precision, x32, val32, diag, device, s); break;
        case 8: launch_g<8>(U, m, x, y, yadd, precision, x32, val32, diag, device, s); break;
        default: launch_g<4>(U, m, x, y, yadd, precision, x32, val32, diag, device, s); break;
    }
    DNQ_CHECK_LAUNCH();
}

}  // namespace

// Same as spmv_block with lanes per row G and slots per lane U given
// (0 = automatic).
void spmv_block_g(const dnq_ham_s* h, const Csr& m, const double* x, double* y, int precision,
                  cudaStream_t s, const float* x32, const float* val32, const double* diag,
                  int G, int device, int U) {
    (void)h;
    launch_spmv(m, x, y, nullptr, precision, x32, val32, diag, G, U, device, s);
}

// y (+)= M x for one block with the handle's H.psi shape; x FP64 device,
// y FP64 device.
void spmv_block(const dnq_ham_s* h, const Csr& m, const double* x, double* y,
                const double* yadd, int precision, cudaStream_t s, float* x32,
                const double* diag) {
    launch_spmv(m, x, y, yadd, precision, x32, m.val32.p, diag, h->opt.spmv_lanes,
                h->opt.spmv_unroll, h->device, s);
}

void spmv_shape(const Options& o, const Csr& m, int& G, int& U) {
    G = o.spmv_lanes ? o.spmv_lanes : group_for(m);
    U = o.spmv_unroll ? o.spmv_unroll : unroll_for(m, G);
}

namespace {
template <int G, int U>
void grouped_gu(const SpmvDesc* d, int nd, i64 max_rows, int precision, int device,
                cudaStream_t s) {
    auto launch = [&](auto kern) {
        const i64 want = (max_rows * G + 255) / 256;
        const int cap = blocks_for(kern, device);
        const dim3 grid((unsigned)std::max<i64>(1, std::min<i64>(want, cap)), (unsigned)nd);
        kern<<<grid, 256, 0, s>>>(d);
    };
    if (precision == DNQ_F64) launch(k_spmv_grouped<G, U, double, AccF64>);
    else launch(k_spmv_grouped<G, U, float, AccF32>);
}

template <int G>
void grouped_g(int U, const SpmvDesc* d, int nd, i64 max_rows, int precision, int device,
               cudaStream_t s) {
    switch (U) {
        case 4: grouped_gu<G, 4>(d, nd, max_rows, precision, device, s); break;
        case 2: grouped_gu<G, 2>(d, nd, max_rows, precision, device, s); break;
        default: grouped_gu<G, 1>(d, nd, max_rows, precision, device, s); break;
    }
}
}  // namespace

void spmv_grouped(const SpmvDesc* d_dev, int nd, i64 max_rows, int G, int U, int precision,
                  int device, cudaStream_t s) {
    if (nd <= 0) return;
    switch (G) {
        case 32: grouped_g<32>(U, d_dev, nd, max_rows, precision, device, s); break;
        case 16: grouped_g<16>(U, d_dev, nd, max_rows, precision, device, s); break;
        case 8: grouped_g<8>(U, d_dev, nd, max_rows, precision, device, s); break;
        default: grouped_g<4>(U, d_dev, nd, max_rows, precision, device, s); break;
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
    k_energy_final<<<1, 256, 0, s>>>(part.p, nb, out2_dev);
    DNQ_CHECK_LAUNCH();
}

// Same reduction with caller-provided partials (4 * nb doubles) and result
// slot: launches only, allocates nothing.
void energy_reduce_into(const double* x, const double* y, i64 n, double* eloc, double* part,
                        int nb, double* out2_dev, cudaStream_t s) {
    k_energy_partials<<<nb, 256, 0, s>>>(x, y, n, eloc, part);
    DNQ_CHECK_LAUNCH();
    k_energy_final<<<1, 256, 0, s>>>(part, nb, out2_dev);
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
    if (!h->vv.f32_ready() || h->diag_op.n != (size_t)h->n_v)
        make_f32(h->vv, s, &h->diag_op);
    if ((i64)h->x32.n < h->n_v) h->x32.alloc(h->n_v, s);
}

// FP32 V-block operator of a handle.
void spmv_vv_f32(dnq_ham_s* h, const double* x, double* y, cudaStream_t s) {
    spmv_block(h, h->vv, x, y, nullptr, DNQ_F32, s, h->x32.p, h->diag_op.p);
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
        spmv_vv_f32(h, xd.p, yd, s);
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
        spmv_vv_f32(h, xd.p, y.p, s);
    } else {
        spmv_block(h, h->vv, xd.p, y.p, nullptr, DNQ_F64, s, nullptr, nullptr);
    }
    const bool dev_eloc = eloc && is_device_ptr(eloc);
    if (dev_eloc) require_on_device(eloc, h->device, "eloc");
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
