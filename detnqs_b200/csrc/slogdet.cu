// Batched sign and log|det| of small real matrices, and the gradient of
// log|det| (the reference's fused log-det kernels, csrc/ffi/logdet_cuda.cu:
// forward :187-262 by LU with partial pivoting, backward :264-331 by solving
// A^T X = I), written without cuSolverDx.
//
// One warp per matrix, grid-stride over the batch.  The matrix sits in
// shared memory, row-major with an odd row stride.  Step k of the
// right-looking LU: the lanes search rows k.. for the largest |a_rk| (the
// lowest row on ties, as LAPACK's idamax) and reduce it by shuffles; the
// rows are swapped by columns, the multipliers divided by rows, and the
// trailing block updated by columns, each lane walking its columns down the
// rows with fused multiply-adds.  A zero (or not-a-number) pivot column
// marks the matrix singular: sign 0 and log|det| -inf, gradient 0, as the
// reference reports a nonzero factorisation status.
//
// The gradient solves A Y = I from the factors (rows of I swapped as the
// factorisation swapped them, then L and U substitutions, one column of Y
// per lane) and writes cot * Y^T = cot * A^{-T}.
#include "common.cuh"

#include <cmath>

namespace dnq {

void keep_pool(int device);

namespace {

__host__ __device__ inline int lu_stride(int n) { return n | 1; }

template <class T>
__host__ __device__ inline size_t warp_bytes(int n, bool grad) {
    const size_t m = (size_t)n * lu_stride(n) * sizeof(T);
    const size_t b = grad ? 2 * m + (size_t)n * sizeof(int) : m;
    return (b + 15) & ~(size_t)15;
}

template <class T>
__device__ __forceinline__ void load_matrix(T* M, const T* A, int n, int ld, int lane) {
    for (int e = lane; e < n * n; e += 32) M[(e / n) * ld + e % n] = A[e];
}

// In-place LU with partial pivoting of the n x n matrix M (row stride ld).
// Returns false at the first pivot column without a usable value; *swaps is
// the parity of the row exchanges, piv[k] (when given) the row exchanged
// with row k.
template <class T>
__device__ bool lu_warp(T* M, int n, int ld, int lane, int* swaps, int* piv) {
    int par = 0;
    for (int k = 0; k < n; ++k) {
        T best = T(-1);
        int br = n;
        for (int r = k + lane; r < n; r += 32) {
            const T v = fabs(M[r * ld + k]);
            if (v > best) {   // rows ascend per lane: the first maximum stays
                best = v;
                br = r;
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int orow = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > best || (ov == best && orow < br)) {
                best = ov;
                br = orow;
            }
        }
        if (br >= n || !(best > T(0))) {   // warp-uniform after the reduction
            *swaps = par;
            return false;
        }
        if (piv && lane == 0) piv[k] = br;
        if (br != k) {
            par ^= 1;
            for (int c = lane; c < n; c += 32) {
                const T t = M[k * ld + c];
                M[k * ld + c] = M[br * ld + c];
                M[br * ld + c] = t;
            }
        }
        __syncwarp();
        const T p = M[k * ld + k];
        for (int r = k + 1 + lane; r < n; r += 32) M[r * ld + k] = M[r * ld + k] / p;
        __syncwarp();
        for (int c = k + 1 + lane; c < n; c += 32) {
            const T u = M[k * ld + c];
            for (int r = k + 1; r < n; ++r) M[r * ld + c] = fma(-M[r * ld + k], u, M[r * ld + c]);
        }
        __syncwarp();
    }
    *swaps = par;
    return true;
}

template <class T>
__global__ void __launch_bounds__(256) k_slogdet(const T* A, i64 B, int n, T* sign, T* logabs) {
    extern __shared__ __align__(16) unsigned char lu_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int ld = lu_stride(n);
    T* M = reinterpret_cast<T*>(lu_smem + (size_t)w * warp_bytes<T>(n, false));
    for (i64 b = blockIdx.x * (i64)wpb + w; b < B; b += (i64)gridDim.x * wpb) {
        load_matrix(M, A + b * (i64)n * n, n, ld, lane);
        __syncwarp();
        int par = 0;
        const bool ok = lu_warp(M, n, ld, lane, &par, (int*)nullptr);
        if (lane == 0) {
            double s = par ? -1.0 : 1.0, la = 0.0;
            bool good = ok;
            for (int i = 0; good && i < n; ++i) {   // as the reference: log|u_ii| summed in FP64
                const double d = (double)M[i * ld + i];
                const double ad = fabs(d);
                if (!(ad > 0.0) || !isfinite(ad)) {
                    good = false;
                    break;
                }
                la += log(ad);
                if (d < 0.0) s = -s;
            }
            sign[b] = good ? (T)s : T(0);
            logabs[b] = good ? (T)la : (T)(-INFINITY);
        }
        __syncwarp();
    }
}

template <class T>
__global__ void __launch_bounds__(256) k_slogdet_grad(const T* A, const T* cot, i64 B, int n,
                                                      T* grad) {
    extern __shared__ __align__(16) unsigned char lu_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int ld = lu_stride(n);
    unsigned char* base = lu_smem + (size_t)w * warp_bytes<T>(n, true);
    T* M = reinterpret_cast<T*>(base);
    T* Y = M + (size_t)n * ld;
    int* piv = reinterpret_cast<int*>(Y + (size_t)n * ld);
    const i64 nn = (i64)n * n;
    for (i64 b = blockIdx.x * (i64)wpb + w; b < B; b += (i64)gridDim.x * wpb) {
        load_matrix(M, A + b * nn, n, ld, lane);
        __syncwarp();
        int par = 0;
        const bool ok = lu_warp(M, n, ld, lane, &par, piv);
        T* G = grad + b * nn;
        if (!ok) {
            for (i64 e = lane; e < nn; e += 32) G[e] = T(0);
            __syncwarp();
            continue;
        }
        for (int c = lane; c < n; c += 32) {
            int pos = c;   // row of column c's one after the factorisation's swaps
            for (int k = 0; k < n; ++k) {
                if (piv[k] == pos) pos = k;
                else if (k == pos) pos = piv[k];
            }
            for (int i = 0; i < n; ++i) Y[i * ld + c] = i == pos ? T(1) : T(0);
            for (int i = 1; i < n; ++i) {   // L z = e (unit diagonal)
                T s = Y[i * ld + c];
                for (int j = 0; j < i; ++j) s = fma(-M[i * ld + j], Y[j * ld + c], s);
                Y[i * ld + c] = s;
            }
            for (int i = n - 1; i >= 0; --i) {   // U y = z
                T s = Y[i * ld + c];
                for (int j = i + 1; j < n; ++j) s = fma(-M[i * ld + j], Y[j * ld + c], s);
                Y[i * ld + c] = s / M[i * ld + i];
            }
        }
        __syncwarp();
        const T g = cot[b];
        for (i64 e = lane; e < nn; e += 32) {   // grad[i][j] = cot * (A^-1)[j][i]
            const int i = (int)(e / n), j = (int)(e % n);
            G[e] = g * Y[j * ld + i];
        }
        __syncwarp();
    }
}

// Warps per block from the shared memory each matrix needs (up to 96 KB per
// block), and the launch's dynamic shared memory.
template <class K>
void lu_launch_shape(K kernel, size_t per_warp, i64 B, int device, int& wpb, int& grid,
                     size_t& smem) {
    wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / per_warp));
    smem = per_warp * wpb;
    DNQ_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    grid = (int)std::min<i64>((B + wpb - 1) / wpb, (i64)sm_count(device) * 32);
}

template <class T>
void run_slogdet(const void* A, i64 B, int n, void* sign, void* logabs, int device,
                 cudaStream_t s) {
    DIn<T> a(static_cast<const T*>(A), (size_t)B * n * n, s);
    const bool dev_s = is_device_ptr(sign), dev_l = is_device_ptr(logabs);
    DBuf<T> ts, tl;
    T* ps = static_cast<T*>(sign);
    T* pl = static_cast<T*>(logabs);
    if (!dev_s) {
        ts.alloc(B, s);
        ps = ts.p;
    }
    if (!dev_l) {
        tl.alloc(B, s);
        pl = tl.p;
    }
    int wpb = 0, grid = 0;
    size_t smem = 0;
    lu_launch_shape(k_slogdet<T>, warp_bytes<T>(n, false), B, device, wpb, grid, smem);
    k_slogdet<T><<<grid, wpb * 32, smem, s>>>(a.p, B, n, ps, pl);
    DNQ_CHECK_LAUNCH();
    if (!dev_s) copy_out(static_cast<T*>(sign), ps, B, s);
    if (!dev_l) copy_out(static_cast<T*>(logabs), pl, B, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
}

template <class T>
void run_slogdet_grad(const void* A, const void* cot, i64 B, int n, void* grad, int device,
                      cudaStream_t s) {
    DIn<T> a(static_cast<const T*>(A), (size_t)B * n * n, s);
    DIn<T> c(static_cast<const T*>(cot), (size_t)B, s);
    const bool dev_g = is_device_ptr(grad);
    DBuf<T> tg;
    T* pg = static_cast<T*>(grad);
    if (!dev_g) {
        tg.alloc((size_t)B * n * n, s);
        pg = tg.p;
    }
    int wpb = 0, grid = 0;
    size_t smem = 0;
    lu_launch_shape(k_slogdet_grad<T>, warp_bytes<T>(n, true), B, device, wpb, grid, smem);
    k_slogdet_grad<T><<<grid, wpb * 32, smem, s>>>(a.p, c.p, B, n, pg);
    DNQ_CHECK_LAUNCH();
    if (!dev_g) copy_out(static_cast<T*>(grad), pg, (size_t)B * n * n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
}

// The reference's argument checks (logdet_cuda.cu:92-118).
void check_batch(i64 B, int n, int precision) {
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID,
            "precision must be DNQ_F64 or DNQ_F32");
    require(n >= 2 && n <= 64, DNQ_ERR_INVALID, "N must be in [2, 64]");
    require(B >= 1 && B <= (i64)0x7fffffff, DNQ_ERR_INVALID, "Batch size out of int32 range");
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_slogdet(const void* a, int64_t B, int n, int precision, void* sign, void* logabs,
                int device, void* stream) {
    DNQ_API_BEGIN
    check_batch(B, n, precision);
    require(a && sign && logabs, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(device);
    keep_pool(device);
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == DNQ_F64) run_slogdet<double>(a, B, n, sign, logabs, device, s);
    else run_slogdet<float>(a, B, n, sign, logabs, device, s);
    DNQ_API_END
}

int dnq_slogdet_grad(const void* a, const void* cot_logabs, int64_t B, int n, int precision,
                     void* grad, int device, void* stream) {
    DNQ_API_BEGIN
    check_batch(B, n, precision);
    require(a && cot_logabs && grad, DNQ_ERR_INVALID, "null argument");
    DeviceGuard g(device);
    keep_pool(device);
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == DNQ_F64) run_slogdet_grad<double>(a, cot_logabs, B, n, grad, device, s);
    else run_slogdet_grad<float>(a, cot_logabs, B, n, grad, device, s);
    DNQ_API_END
}

}  // extern "C"
