// detmap.cu -- construction of the device determinant map.
#include "detmap.cuh"
#include "prim.cuh"

namespace dnq {
namespace {

__global__ void k_map_insert(const u64* dets, i64 n, ulonglong2* keys, u32* idx,
                             u64 mask, unsigned long long* full_alpha) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        if (a == kEmptyKey) {
            atomicMin(full_alpha, (unsigned long long)t);
            continue;
        }
        u64 h = det_hash(a, b) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev = atomicCAS(
                reinterpret_cast<unsigned long long*>(&keys[h].x), kEmptyKey, a);
            if (prev == kEmptyKey) {
                keys[h].y = b;
                idx[h] = (u32)t;
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

__device__ __forceinline__ long long find_slot(const ulonglong2* keys, u64 mask, u64 a,
                                               u64 b) {
    u64 h = det_hash(a, b) & mask;
    for (u64 probe = 0; probe <= mask; ++probe) {
        const ulonglong2 k = keys[h];
        if (k.x == kEmptyKey) return -1;
        if (k.x == a && k.y == b) return (long long)h;
        h = (h + 1) & mask;
    }
    return -1;
}

// strict: count positions whose key resolves to another index.
__global__ void k_map_verify(const u64* dets, i64 n, const ulonglong2* keys,
                             const u32* idx, u64 mask, unsigned long long full_alpha,
                             unsigned long long* dup) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        if (a == kEmptyKey) {
            if ((unsigned long long)t != full_alpha) atomicAdd(dup, 1ull);
            continue;
        }
        const long long s = find_slot(keys, mask, a, b);
        if (s < 0 || idx[s] != (u32)t) atomicAdd(dup, 1ull);
    }
}

__global__ void k_map_min(const u64* dets, i64 n, const ulonglong2* keys, u32* idx,
                          u64 mask) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        if (a == kEmptyKey) continue;
        const long long s = find_slot(keys, mask, a, b);
        if (s >= 0) atomicMin(&idx[s], (u32)t);
    }
}

__global__ void k_map_first(const u64* dets, i64 n, const ulonglong2* keys,
                            const u32* idx, u64 mask, unsigned long long full_alpha,
                            u32* first) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        u32 f;
        if (a == kEmptyKey) f = ((unsigned long long)t == full_alpha);
        else {
            const long long s = find_slot(keys, mask, a, b);
            f = (s >= 0 && idx[s] == (u32)t);
        }
        first[t] = f;
    }
}

__global__ void k_map_rank(const u64* dets, i64 n, const ulonglong2* keys,
                           const u32* idx, u64 mask, unsigned long long full_alpha,
                           const u32* rank, u32* rank_out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        u32 f = (u32)t;
        if (a == kEmptyKey) f = (u32)full_alpha;
        else {
            const long long s = find_slot(keys, mask, a, b);
            if (s >= 0) f = idx[s];
        }
        rank_out[t] = rank[f];
    }
}

__global__ void k_map_relabel(const u64* dets, i64 n, const ulonglong2* keys, u32* idx,
                              u64 mask, const u32* first, const u32* rank) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (!first[t]) continue;
        const u64 a = dets[2 * t], b = dets[2 * t + 1];
        if (a == kEmptyKey) continue;
        const long long s = find_slot(keys, mask, a, b);
        if (s >= 0) idx[s] = rank[t];
    }
}

}  // namespace

void build_detmap(DetMap& m, const u64* dets, i64 n, bool strict, cudaStream_t s,
                  DBuf<u32>* rank_out) {
    require(n <= (i64)0xffffffffll, DNQ_ERR_OVERFLOW,
            "DetMap size exceeds u32 index capacity");
    u64 cap = 1024;
    while (cap < (u64)(2 * n)) cap <<= 1;
    m.n = n;
    m.mask = cap - 1;
    m.keys.alloc(cap, s);
    m.idx.alloc(cap, s);
    DNQ_CUDA(cudaMemsetAsync(m.keys.p, 0xff, cap * sizeof(ulonglong2), s));
    DBuf<unsigned long long> scal(2, s);
    const unsigned long long init[2] = {~0ull, 0ull};
    DNQ_CUDA(cudaMemcpyAsync(scal.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int threads = 256;
    const int blocks = (int)std::min<i64>((n + threads - 1) / threads + 1, 65535);
    if (n > 0) {
        k_map_insert<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask, scal.p);
        DNQ_CHECK_LAUNCH();
    }
    unsigned long long host[2];
    DNQ_CUDA(cudaMemcpyAsync(host, scal.p, sizeof(host), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    const unsigned long long full_alpha = host[0];
    m.full_alpha_idx = full_alpha == ~0ull ? -1 : (long long)full_alpha;
    if (m.full_alpha_idx >= 0) {
        u64 b;
        DNQ_CUDA(cudaMemcpyAsync(&b, dets + 2 * full_alpha + 1, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        m.full_alpha_beta = b;
    }
    if (n == 0) return;
    if (strict) {
        k_map_verify<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask,
                                                 full_alpha, scal.p + 1);
        DNQ_CHECK_LAUNCH();
        DNQ_CUDA(cudaMemcpyAsync(host, scal.p, sizeof(host), cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        require(host[1] == 0, DNQ_ERR_DUPLICATE,
                "DetMap::from_ordered: duplicate determinant found");
        if (rank_out) {
            rank_out->alloc(n, s);
            // identity ranks
            DBuf<u32> first(n, s);
            k_map_first<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask,
                                                    full_alpha, first.p);
            DNQ_CHECK_LAUNCH();
            prim::scan<u32, u32, false>(first.p, rank_out->p, n, s);
        }
        return;
    }
    k_map_min<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask);
    DNQ_CHECK_LAUNCH();
    DBuf<u32> first(n, s), rank(n, s);
    k_map_first<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask, full_alpha,
                                            first.p);
    DNQ_CHECK_LAUNCH();
    prim::scan<u32, u32, false>(first.p, rank.p, n, s);
    if (rank_out) {
        rank_out->alloc(n, s);
        k_map_rank<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask, full_alpha,
                                               rank.p, rank_out->p);
        DNQ_CHECK_LAUNCH();
    }
    k_map_relabel<<<blocks, threads, 0, s>>>(dets, n, m.keys.p, m.idx.p, m.mask, first.p,
                                              rank.p);
    DNQ_CHECK_LAUNCH();
    if (m.full_alpha_idx >= 0) {
        u32 r;
        DNQ_CUDA(cudaMemcpyAsync(&r, rank.p + m.full_alpha_idx, 4, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        m.full_alpha_idx = r;
    }
}

}  // namespace dnq
