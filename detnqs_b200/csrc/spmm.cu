// spmm.cu -- H applied to several amplitude vectors in one pass.
//
// The single-vector H.psi kernels (spmv.cu) are bound by their gathers of
// x: each stored entry fetches one x value, and the L1 serves one 32-byte
// sector per gathered value, 4 or 8 bytes of which are used.  Here k
// vectors are stored interleaved, X[c][0..k) contiguous, so the gather of
// one 32-byte sector brings the values of all of them (8 FP32 or 4 FP64
// vectors, one 256-bit load), and one pass over the CSR serves k vectors
// for about the sector cost of one.  This serves the inner loop of the
// reference's optimiser, which applies H to one psi per SciPy call
// (detnqs/operator/kernel.py:75-78), whenever several amplitude sets of the
// same determinant space are evaluated together (samples of a stochastic
// optimiser, grouped local-energy requests of the server).
//
// Each vector is accumulated in exactly the order of the single-vector
// kernel with the same lanes per row (the same slots per lane, the same
// butterfly), so every column equals dnq_ham_spmv of that vector bit for
// bit; padding columns (k below the gather width) carry zeros and are not
// written.  The energies {x_j.Hx_j, x_j.x_j} follow the single-vector
// reduction tree column by column, so they are bit-identical too.
#include <algorithm>
#include <vector>

#include "ham.cuh"
#include "spmv.cuh"

namespace dnq {

void spmv_shape(const Options& o, const Csr& m, int& G, int& U);
void ensure_f32(dnq_ham_s* h, cudaStream_t s);

namespace {

// K values of column c of an interleaved [n][K] array (K * sizeof(T) bytes
// at a K * sizeof(T)-aligned address), read through the non-coherent path.
template <int K, class T>
struct Gather;

template <>
struct Gather<8, float> {
    static __device__ __forceinline__ void get(const float* X, u32 c, float (&o)[8]) {
        asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
            : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]),
              "=f"(o[6]), "=f"(o[7])
            : "l"(X + 8 * (size_t)c));
    }
};
template <>
struct Gather<4, float> {
    static __device__ __forceinline__ void get(const float* X, u32 c, float (&o)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(X + 4 * (size_t)c));
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    }
};
template <>
struct Gather<2, float> {
    static __device__ __forceinline__ void get(const float* X, u32 c, float (&o)[2]) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(X + 2 * (size_t)c));
        o[0] = a.x; o[1] = a.y;
    }
};
template <>
struct Gather<4, double> {
    static __device__ __forceinline__ void get(const double* X, u32 c, double (&o)[4]) {
        asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
            : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
            : "l"(X + 4 * (size_t)c));
    }
};
template <>
struct Gather<2, double> {
    static __device__ __forceinline__ void get(const double* X, u32 c, double (&o)[2]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(X + 2 * (size_t)c));
        o[0] = a.x; o[1] = a.y;
    }
};

// Y[r][j] (j < kx) = sum_k H_rk X[k][j], for K interleaved columns.  The
// slot walk, masking and accumulation order are those of row_acc in
// spmv.cu, with K accumulators per lane.  Entries outside the row read the
// zero row nr of Xg (and a zero value), which adds the same +0 products as
// the single-vector kernel's masking without a branch per entry.
//   T = double: FP64 values and X (AccF64)
//   T = float : FP32 off-diagonal values and X32, Kahan sums, plus the FP64
//               diagonal term diag_r * X64[r][j] added in FP64 (AccF32)
// The G lanes of a row then combine their K sums with the single-vector
// kernel's butterfly pairs (lane ^ G/2, ..., lane ^ 1) as a reduce-scatter:
// while a lane holds more than one column, each step it keeps half of them
// (the lower half when its bit o is clear) and hands the other half to its
// partner, so a column is merged with exactly the values it meets in the
// single-vector butterfly, at a fraction of the shuffles.  Lane l ends with
// columns [j0, j0 + K / min(K, G)).
template <int G, int U, int K, class T, class Acc>
__global__ void __launch_bounds__(256)
k_spmm(const i64* __restrict__ rs, const i64* __restrict__ re, const u32* __restrict__ col,
       const T* __restrict__ val,
       const T* __restrict__ Xg, const double* __restrict__ diag, const double* __restrict__ X,
       int ldx, int kx, i64 nr, i64 nnz, double* __restrict__ Y, int ldy) {
    const i64 gid = (blockIdx.x * (i64)blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x & (G - 1);
    const i64 ngroups = (gridDim.x * (i64)blockDim.x) / G;
    const i64 rounds = (nr + ngroups - 1) / ngroups;
    const u32 zrow = (u32)nr;
    for (i64 it = 0; it < rounds; ++it) {
        const i64 r = gid + it * ngroups;
        Acc acc[K];
        if (r < nr) {
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
                            c[u][q] = ok ? __ldg(&col[k + q]) : zrow;
                            v[u][q] = ok ? __ldg(&val[k + q]) : T(0);
                        }
                    }
                }
                T xv[U][4][K];
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const i64 kk = k0 + (i64)u * 4 * G + q;
                        const bool in = kk >= b && kk < e;
                        Gather<K, T>::get(Xg, in ? c[u][q] : zrow, xv[u][q]);
                        if (!in) v[u][q] = T(0);
                    }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (k0 + (i64)u * 4 * G < e) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int j = 0; j < K; ++j) acc[j].add_prod(v[u][q], xv[u][q][j]);
                    }
            }
        }
        // reduce-scatter over the butterfly pairs
        int j0 = 0;
#pragma unroll
        for (int o = G / 2, kc = K; o; o >>= 1) {
            if (kc > 1) {
                const int h = kc / 2;
                const bool upper = (sub & o) != 0;
#pragma unroll
                for (int i = 0; i < K / 2; ++i) {
                    if (i >= h) break;
                    const Acc give = upper ? acc[i] : acc[i + h];
                    const Acc got = give.shfl(o);
                    Acc keep = upper ? acc[i + h] : acc[i];
                    keep.merge(got);
                    acc[i] = keep;
                }
                if (upper) j0 += h;
                kc = h;
            } else {
                acc[0].merge(acc[0].shfl(o));
            }
        }
        constexpr int kOwn = K > G ? K / G : 1;
        const bool writer = (K >= G) || (sub & (G / K - 1)) == 0;
        if (r < nr && writer) {
#pragma unroll
            for (int i = 0; i < kOwn; ++i) {
                const int j = j0 + i;
                if (j < kx) {
                    double y = acc[i].value();
                    if (diag) y += diag[r] * X[r * (i64)ldx + j];
                    Y[r * (i64)ldy + j] = y;
                }
            }
        }
    }
}

// Interleaved gather copy of the first kx columns of X (n x ldx, FP64):
// FP32 or FP64, zero-padded to K columns, plus a zero row n.
template <int K, class T>
__global__ void k_interleave(const double* __restrict__ X, int ldx, int kx, i64 n,
                             T* __restrict__ Xg) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < (n + 1) * K;
         t += (i64)gridDim.x * blockDim.x) {
        const i64 r = t / K;
        const int j = (int)(t - r * K);
        Xg[t] = (j < kx && r < n) ? (T)X[r * ldx + j] : T(0);
    }
}

// Energies of K columns: per block, the Dot2 partials of x_j.y_j and
// x_j.x_j with the thread / warp / block order of k_energy_partials
// (spmv.cu), so column j's sums are those of the single-vector reduction;
// eloc[r][j] = y / x.
template <int K>
__global__ void __launch_bounds__(256)
k_energy_partials_multi(const double* X, int ldx, const double* Y, int ldy, int kx, i64 n,
                        double* eloc, int lde, double* part) {
    Dot2<double> num[K], den[K];
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j >= kx) break;
            const double xv = X[t * ldx + j], yv = Y[t * ldy + j];
            num[j].add_prod(xv, yv);
            den[j].add_prod(xv, xv);
            if (eloc) eloc[t * lde + j] = yv / xv;
        }
    }
#pragma unroll
    for (int j = 0; j < K; ++j)
        for (int o = 16; o; o >>= 1) {
            num[j].merge(shfl_xor(num[j], o, 0xffffffffu));
            den[j].merge(shfl_xor(den[j], o, 0xffffffffu));
        }
    __shared__ double sh[K][4][8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            sh[j][0][w] = num[j].s; sh[j][1][w] = num[j].c;
            sh[j][2][w] = den[j].s; sh[j][3][w] = den[j].c;
        }
    }
    __syncthreads();
    if (threadIdx.x < K && (int)threadIdx.x < kx) {
        const int j = threadIdx.x;
        Dot2<double> a, b;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            Dot2<double> t1, t2;
            t1.s = sh[j][0][q]; t1.c = sh[j][1][q]; t2.s = sh[j][2][q]; t2.c = sh[j][3][q];
            a.merge(t1);
            b.merge(t2);
        }
        double* p = part + ((i64)j * gridDim.x + blockIdx.x) * 4;
        p[0] = a.s; p[1] = a.c; p[2] = b.s; p[3] = b.c;
    }
}

// Thread j < kx merges column j's partials in block order (as the single-
// vector reduction does); the block stages them in shared memory, 128 per
// column at a time, so the serial merges wait on no global load.
constexpr int kFinalChunk = 128;
__global__ void __launch_bounds__(256) k_energy_final_multi(const double* part, int nb, int kx,
                                                            double* out) {
    __shared__ double st[8][4 * kFinalChunk];
    const int j = threadIdx.x;
    Dot2<double> a, b;
    for (int q0 = 0; q0 < nb; q0 += kFinalChunk) {
        const int m = min(kFinalChunk, nb - q0);
        for (int i = threadIdx.x; i < kx * 4 * m; i += blockDim.x) {
            const int c = i / (4 * m), e = i % (4 * m);
            st[c][e] = part[((i64)c * nb + q0) * 4 + e];
        }
        __syncthreads();
        if (j < kx) {
            for (int q = 0; q < m; ++q) {
                Dot2<double> t1, t2;
                t1.s = st[j][4 * q]; t1.c = st[j][4 * q + 1];
                t2.s = st[j][4 * q + 2]; t2.c = st[j][4 * q + 3];
                a.merge(t1);
                b.merge(t2);
            }
        }
        __syncthreads();
    }
    if (j < kx) {
        out[2 * j] = a.value();
        out[2 * j + 1] = b.value();
    }
}

template <class Kern>
int blocks_of(Kern kern, int device) {
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
    return std::max(1, per_sm) * sm_count(device);
}

template <int G, int U, int K, class T, class Acc>
void launch_spmm(const Csr& m, const T* val, const T* Xg, const double* diag, const double* X,
                 int ldx, int kx, double* Y, int ldy, int device, cudaStream_t s) {
    auto kern = k_spmm<G, U, K, T, Acc>;
    kern<<<blocks_of(kern, device), 256, 0, s>>>(m.row_start(), m.row_end(), m.col.p, val, Xg,
                                                 diag, X, ldx, kx, m.nr, m.span(), Y, ldy);
    DNQ_CHECK_LAUNCH();
}

// Slots per lane in flight: the single-vector choice for 2 columns, 2 for 4
// and 8 (measured best on the 10^6-determinant matrix; 4 would not fit the
// registers of 8 columns).  Results do not depend on it.
template <int K, class T, class Acc>
void spmm_g(int G, int U, const Csr& m, const T* val, const T* Xg, const double* diag,
            const double* X, int ldx, int kx, double* Y, int ldy, int device, cudaStream_t s) {
    if (K >= 4) U = 2;
#define DNQ_SPMM_U(GG)                                                                        \
    switch (U) {                                                                              \
        case 4: launch_spmm<GG, 4, K, T, Acc>(m, val, Xg, diag, X, ldx, kx, Y, ldy, device, s); \
            break;                                                                            \
        case 2: launch_spmm<GG, 2, K, T, Acc>(m, val, Xg, diag, X, ldx, kx, Y, ldy, device, s); \
            break;                                                                            \
        default: launch_spmm<GG, 1, K, T, Acc>(m, val, Xg, diag, X, ldx, kx, Y, ldy, device, s); \
            break;                                                                            \
    }
    switch (G) {
        case 32: DNQ_SPMM_U(32) break;
        case 16: DNQ_SPMM_U(16) break;
        case 8: DNQ_SPMM_U(8) break;
        default: DNQ_SPMM_U(4) break;
    }
#undef DNQ_SPMM_U
}

constexpr int kEnergyBlocks = 592;   // the single-vector reduction's grid

}  // namespace

// Y (nr x ldy) = M X (nc x ldx) for kx <= 8 (FP32) or <= 4 (FP64) columns
// of a square CSR; X, Y device memory.  FP32 uses val32 (off-diagonal
// values) and the FP64 diagonal diag32.  G = 0 picks the lanes per row as
// the single-vector kernel does (same option, same rule), so columns match
// it bit for bit.  scratch: interleaved copy of X (spmm_scratch_bytes).
void spmm_csr(const Csr& m, const float* val32, const double* diag32, const double* X, int ldx,
              int kx, double* Y, int ldy, int precision, int G, int U, void* scratch,
              int dev, cudaStream_t s) {
    if (m.nr == 0) return;
    if (G == 0 || U == 0) {
        int g = 0, u = 0;
        spmv_shape(Options{}, m, g, u);
        if (G == 0) G = g;
        if (U == 0) U = u;
    }
    const unsigned gi = (unsigned)std::max<i64>(1, std::min<i64>(4096, (m.nr * 8 + 255) / 256));
    if (precision == DNQ_F32) {
        float* Xg = static_cast<float*>(scratch);
        const int K = kx <= 2 ? 2 : kx <= 4 ? 4 : 8;
        if (K == 2) {
            k_interleave<2, float><<<gi, 256, 0, s>>>(X, ldx, kx, m.nr, Xg);
            DNQ_CHECK_LAUNCH();
            spmm_g<2, float, AccF32>(G, U, m, val32, Xg, diag32, X, ldx, kx, Y, ldy, dev, s);
        } else if (K == 4) {
            k_interleave<4, float><<<gi, 256, 0, s>>>(X, ldx, kx, m.nr, Xg);
            DNQ_CHECK_LAUNCH();
            spmm_g<4, float, AccF32>(G, U, m, val32, Xg, diag32, X, ldx, kx, Y, ldy, dev, s);
        } else {
            k_interleave<8, float><<<gi, 256, 0, s>>>(X, ldx, kx, m.nr, Xg);
            DNQ_CHECK_LAUNCH();
            spmm_g<8, float, AccF32>(G, U, m, val32, Xg, diag32, X, ldx, kx, Y, ldy, dev, s);
        }
    } else {
        double* Xg = static_cast<double*>(scratch);
        if (kx <= 2) {
            k_interleave<2, double><<<gi, 256, 0, s>>>(X, ldx, kx, m.nr, Xg);
            DNQ_CHECK_LAUNCH();
            spmm_g<2, double, AccF64>(G, U, m, m.val.p, Xg, nullptr, X, ldx, kx, Y, ldy, dev, s);
        } else {
            k_interleave<4, double><<<gi, 256, 0, s>>>(X, ldx, kx, m.nr, Xg);
            DNQ_CHECK_LAUNCH();
            spmm_g<4, double, AccF64>(G, U, m, m.val.p, Xg, nullptr, X, ldx, kx, Y, ldy, dev, s);
        }
    }
}

// The V block of a handle (FP32: its prepared split).
void spmm_vv(dnq_ham_s* h, const double* X, int ldx, int kx, double* Y, int ldy, int precision,
             void* scratch, cudaStream_t s) {
    spmm_csr(h->vv, h->vv.val32.p, h->diag_op.p, X, ldx, kx, Y, ldy, precision,
             h->opt.spmv_lanes, h->opt.spmv_unroll, scratch, h->device, s);
}

// Bytes of the interleaved scratch for kx columns (n rows and a zero row).
size_t spmm_scratch_bytes(i64 n, int kx, int precision) {
    if (precision == DNQ_F32) return (size_t)(n + 1) * 4 * (kx <= 2 ? 2 : kx <= 4 ? 4 : 8);
    return (size_t)(n + 1) * 8 * (kx <= 2 ? 2 : 4);
}

// out[2j] = x_j.Hx_j, out[2j+1] = x_j.x_j (device), eloc[r][j] = y/x.
void energy_reduce_multi(const double* X, int ldx, const double* Y, int ldy, int kx, i64 n,
                         double* eloc, int lde, double* part, double* out_dev,
                         cudaStream_t s) {
    if (kx <= 4) {
        k_energy_partials_multi<4><<<kEnergyBlocks, 256, 0, s>>>(X, ldx, Y, ldy, kx, n, eloc,
                                                                 lde, part);
    } else {
        k_energy_partials_multi<8><<<kEnergyBlocks, 256, 0, s>>>(X, ldx, Y, ldy, kx, n, eloc,
                                                                 lde, part);
    }
    DNQ_CHECK_LAUNCH();
    k_energy_final_multi<<<1, 256, 0, s>>>(part, kEnergyBlocks, kx, out_dev);
    DNQ_CHECK_LAUNCH();
}

}  // namespace dnq

using namespace dnq;

namespace {

// Runs Y = H X for k columns in passes of at most 8 (FP32) or 4 (FP64).
void spmm_all(dnq_ham_s* h, const double* Xd, int k, double* Yd, int precision,
              cudaStream_t s) {
    const int step = precision == DNQ_F32 ? 8 : 4;
    const i64 n = h->n_v;
    if (precision == DNQ_F32) ensure_f32(h, s);
    DBuf<unsigned char> scratch(spmm_scratch_bytes(n, std::min(k, step), precision), s);
    for (int j0 = 0; j0 < k; j0 += step) {
        const int kx = std::min(step, k - j0);
        spmm_vv(h, Xd + j0, k, kx, Yd + j0, k, precision, scratch.p, s);
    }
}

}  // namespace

extern "C" {

int dnq_ham_spmv_multi(dnq_ham_t h, const double* X, double* Y, int k, int precision,
                       void* stream) {
    DNQ_API_BEGIN
    require(h && X && Y, DNQ_ERR_INVALID, "null argument");
    require(k >= 1 && k <= 1024, DNQ_ERR_INVALID, "k must be in [1, 1024]");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 n = h->n_v;
    if (n == 0) return DNQ_OK;
    DIn<double> xd(X, (size_t)n * k, s);
    const bool dev_out = is_device_ptr(Y);
    if (dev_out) require_on_device(Y, h->device, "Y");
    DBuf<double> ybuf;
    double* yd = Y;
    if (!dev_out) { ybuf.alloc((size_t)n * k, s); yd = ybuf.p; }
    spmm_all(h, xd.p, k, yd, precision, s);
    if (!dev_out) {
        copy_out(Y, yd, (size_t)n * k, s);
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    DNQ_API_END
}

int dnq_ham_local_energy_multi(dnq_ham_t h, const double* X, double* eloc, double* out,
                               int k, int precision, void* stream) {
    DNQ_API_BEGIN
    require(h && X && out, DNQ_ERR_INVALID, "null argument");
    require(k >= 1 && k <= 1024, DNQ_ERR_INVALID, "k must be in [1, 1024]");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const i64 n = h->n_v;
    if (n == 0) {
        std::vector<double> z(2 * (size_t)k, 0.0);
        DNQ_CUDA(cudaMemcpyAsync(out, z.data(), z.size() * 8, cudaMemcpyDefault, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        return DNQ_OK;
    }
    DIn<double> xd(X, (size_t)n * k, s);
    DBuf<double> yd((size_t)n * k, s);
    spmm_all(h, xd.p, k, yd.p, precision, s);
    const bool dev_eloc = eloc && is_device_ptr(eloc);
    if (dev_eloc) require_on_device(eloc, h->device, "eloc");
    DBuf<double> ebuf;
    double* ed = nullptr;
    if (eloc) {
        if (dev_eloc) ed = eloc;
        else { ebuf.alloc((size_t)n * k, s); ed = ebuf.p; }
    }
    DBuf<double> part((size_t)4 * kEnergyBlocks * std::min(k, 8), s), o((size_t)2 * k, s);
    for (int j0 = 0; j0 < k; j0 += 8) {
        const int kx = std::min(8, k - j0);
        energy_reduce_multi(xd.p + j0, k, yd.p + j0, k, kx, n, ed ? ed + j0 : nullptr, k,
                            part.p, o.p + 2 * j0, s);
    }
    if (eloc && !dev_eloc) copy_out(eloc, ed, (size_t)n * k, s);
    copy_out(out, o.p, 2 * (size_t)k, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

}  // extern "C"
