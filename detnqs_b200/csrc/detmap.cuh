// detmap.cuh -- determinant -> index map in HBM.
//
// Replaces DetMap (det_space.cpp:23-65; std::unordered_map<Det, u32>) for
// device lookups: open addressing with linear probing over a power-of-two
// table of 16-byte keys (alpha, beta), load factor <= 1/2, and a parallel
// u32 array of indices that is read only on a hit.  A slot is claimed by a
// 64-bit CAS on its alpha word; the alpha word ~0 marks an empty slot, so a
// determinant whose alpha word is ~0 (64 occupied alpha orbitals) is held
// aside in `full_alpha_idx`.
#pragma once

#include "common.cuh"

namespace dnq {

struct DetMapView {
    const ulonglong2* keys = nullptr;
    const u32* idx = nullptr;
    u64 mask = 0;
    long long full_alpha_idx = -1;   // index of the det with alpha == ~0
    u64 full_alpha_beta = 0;

    __device__ __forceinline__ long long find(u64 a, u64 b) const {
        if (!keys) return -1;
        if (a == kEmptyKey) return (full_alpha_idx >= 0 && b == full_alpha_beta) ? full_alpha_idx : -1;
        u64 h = det_hash(a, b) & mask;
        for (u64 probe = 0; probe <= mask; ++probe) {
            const ulonglong2 k = __ldg(&keys[h]);
            if (k.x == kEmptyKey) return -1;
            if (k.x == a && k.y == b) return (long long)__ldg(&idx[h]);
            h = (h + 1) & mask;
        }
        return -1;
    }
};

struct DetMap {
    DBuf<ulonglong2> keys;
    DBuf<u32> idx;
    u64 mask = 0;
    long long full_alpha_idx = -1;
    u64 full_alpha_beta = 0;
    i64 n = 0;

    DetMapView view() const {
        DetMapView v;
        v.keys = keys.p;
        v.idx = idx.p;
        v.mask = mask;
        v.full_alpha_idx = full_alpha_idx;
        v.full_alpha_beta = full_alpha_beta;
        return v;
    }
    size_t bytes() const { return keys.bytes() + idx.bytes(); }
};

// Build the map of `dets` (device pointer, n x 2 u64).  strict = true
// throws DNQ_ERR_DUPLICATE on a repeated determinant (from_ordered with
// verify_unique = true, det_space.cpp:29-40).  With strict = false the
// first occurrence wins and `rank_out` (optional, device, length n) gets
// for every input position the index of its key in the de-duplicated
// order (det_space.cpp:41-49).
void build_detmap(DetMap& m, const u64* dets, i64 n, bool strict, cudaStream_t s,
                  DBuf<u32>* rank_out = nullptr);

}  // namespace dnq
