// Determinant batch features for the neural models (the reference's
// prepare_det_batch, csrc/src/determinant/det_batch.cpp:184-318, bound as
// detnqs.core.prepare_det_batch in csrc/bridge/bridge.cpp:347-430).
//
// One thread per determinant, grid-stride: every field is a short loop over
// set bits, so a warp keeps 32 determinants in flight.  A thread's rows are
// contiguous: it writes them four int32 (or eight mask bytes) to a store
// where the row is aligned, and the L2 merges the warp's strided stores into
// whole sectors.
// The sign is the reference's sequence: holes removed highest first,
// particles added lowest first, each flipping it by the parity of the
// occupied orbitals below (det_batch.cpp:61-98), over the set bits only.
//
// A determinant that fails a check records (index << 2 | code) with an
// atomic minimum, so the host reports the first failing determinant in
// batch order with the reference's message for its first failing check.
#include "common.cuh"

namespace dnq {

void keep_pool(int device);

namespace {

enum : int { kNeedK = 1, kNeedPhase = 2, kNeedHp = 4, kNeedPos = 8 };
enum : u64 { kBadBits = 1, kBadCount = 2, kBadHp = 3 };

// Sign of one spin's excitation from r to d (both masked).
__device__ __forceinline__ int spin_sign(u64 r, u64 d) {
    u64 h = r & ~d, p = d & ~r, o = r;
    int par = 0;
    while (h) {   // highest hole first
        const int q = 63 - __clzll((long long)h);
        par += __popcll(o & low_mask(q));
        o ^= 1ull << q;
        h ^= 1ull << q;
    }
    while (p) {   // lowest particle first
        const int q = __ffsll((long long)p) - 1;
        par += __popcll(o & low_mask(q));
        o ^= 1ull << q;
        p &= p - 1;
    }
    return (par & 1) ? -1 : 1;
}

// Consecutive int32 values of one output row: four to a 16-byte store when
// the row starts on a 16-byte boundary, one by one otherwise.
struct RowOut {
    int32_t* p;
    bool vec;
    int n = 0, b0 = 0, b1 = 0, b2 = 0;
    __device__ __forceinline__ explicit RowOut(int32_t* row)
        : p(row), vec((reinterpret_cast<uintptr_t>(row) & 15) == 0) {}
    __device__ __forceinline__ void put(int v) {
        if (!vec) {
            p[n++] = v;
            return;
        }
        const int r = n & 3;
        if (r == 3) *reinterpret_cast<int4*>(p + n - 3) = make_int4(b0, b1, b2, v);
        else if (r == 0) b0 = v;
        else if (r == 1) b1 = v;
        else b2 = v;
        ++n;
    }
    __device__ __forceinline__ void flush() {   // the last partial group
        if (!vec) return;
        const int r = n & 3, s = n - r;
        if (r > 0) p[s] = b0;
        if (r > 1) p[s + 1] = b1;
        if (r > 2) p[s + 2] = b2;
    }
};

struct BatchOut {
    int32_t* occ;
    int8_t* k;
    int8_t* phase;
    int32_t* holes;
    int32_t* parts;
    uint8_t* mask;
    int32_t* hpos;
    int32_t* ppos;
};

__global__ void __launch_bounds__(256) k_det_batch(const u64* dets, i64 B, u64 ra, u64 rb,
                                                   int n_orb, int na, int nb, int kmax,
                                                   int flags, BatchOut o,
                                                   unsigned long long* err) {
    const u64 m = low_mask(n_orb);
    const int ne = na + nb;
    ra &= m;
    rb &= m;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < B;
         i += (i64)gridDim.x * blockDim.x) {
        const u64 a = dets[2 * i], b = dets[2 * i + 1];
        u64 bad = 0;
        if ((a & ~m) || (b & ~m)) bad = kBadBits;
        else if (__popcll(a) != na || __popcll(b) != nb) bad = kBadCount;
        else if ((flags & kNeedPhase) &&
                 (__popcll(ra & ~a) != __popcll(a & ~ra) || __popcll(rb & ~b) != __popcll(b & ~rb)))
            bad = kBadHp;
        if (bad) {
            atomicMin(err, ((unsigned long long)i << 2) | bad);
            continue;
        }
        RowOut occ(o.occ + i * ne);
        for (u64 x = a; x; x &= x - 1) occ.put(__ffsll((long long)x) - 1);
        for (u64 x = b; x; x &= x - 1) occ.put(__ffsll((long long)x) - 1 + n_orb);
        occ.flush();
        const u64 ha = ra & ~a, hb = rb & ~b, pa = a & ~ra, pb = b & ~rb;
        const int kk = __popcll(ha) + __popcll(hb);
        if (flags & (kNeedK | kNeedHp)) o.k[i] = (int8_t)min(kk, 127);
        if (flags & kNeedPhase) o.phase[i] = (int8_t)(spin_sign(ra, a) * spin_sign(rb, b));
        if (!(flags & kNeedHp)) continue;
        const bool pos = flags & kNeedPos;
        const i64 row = i * kmax;
        // holes: alpha then beta (+ n_orb), each highest first; position in
        // the reference's occupied list (alpha ascending, then beta)
        {
            RowOut ho(o.holes + row), hp(pos ? o.hpos + row : o.holes + row);
            int j = 0;
            for (u64 x = ha; x && j < kmax; ++j) {
                const int q = 63 - __clzll((long long)x);
                x ^= 1ull << q;
                ho.put(q);
                if (pos) hp.put(__popcll(ra & low_mask(q)));
            }
            for (u64 x = hb; x && j < kmax; ++j) {
                const int q = 63 - __clzll((long long)x);
                x ^= 1ull << q;
                ho.put(q + n_orb);
                if (pos) hp.put(na + __popcll(rb & low_mask(q)));
            }
            for (; j < kmax; ++j) {
                ho.put(-1);
                if (pos) hp.put(-1);
            }
            ho.flush();
            if (pos) hp.flush();
        }
        // particles: alpha then beta (+ n_orb), each lowest first; position
        // in the reference's virtual list (the other spin orbitals, ascending)
        {
            RowOut po(o.parts + row), pp(pos ? o.ppos + row : o.parts + row);
            int j = 0;
            for (u64 x = pa; x && j < kmax; ++j) {
                const int q = __ffsll((long long)x) - 1;
                x &= x - 1;
                po.put(q);
                if (pos) pp.put(q - __popcll(ra & low_mask(q)));
            }
            for (u64 x = pb; x && j < kmax; ++j) {
                const int q = __ffsll((long long)x) - 1;
                x &= x - 1;
                po.put(q + n_orb);
                if (pos) pp.put(q + n_orb - na - __popcll(rb & low_mask(q)));
            }
            for (; j < kmax; ++j) {
                po.put(-1);
                if (pos) pp.put(-1);
            }
            po.flush();
            if (pos) pp.flush();
        }
        // mask: the first min(k, kmax) bytes set, eight to a store when the
        // row starts on an 8-byte boundary and holds whole words
        const int kcap = min(kk, kmax);
        uint8_t* mrow = o.mask + row;
        if ((reinterpret_cast<uintptr_t>(mrow) & 7) == 0 && (kmax & 7) == 0) {
            for (int w = 0; w < kmax; w += 8) {
                const int on = min(max(kcap - w, 0), 8);
                const u64 lo = on == 8 ? ~0ull : ((1ull << (8 * on)) - 1ull);
                *reinterpret_cast<u64*>(mrow + w) = 0x0101010101010101ull & lo;
            }
        } else {
            for (int j = 0; j < kmax; ++j) mrow[j] = j < kcap;
        }
    }
}

// Device target of one output: the caller's device buffer, or a staging
// buffer copied back to the caller's host buffer by finish().
template <class T>
struct DOut {
    T* user = nullptr;
    T* p = nullptr;
    size_t n = 0;
    DBuf<T> own;
    void set(T* dst, size_t count, cudaStream_t s) {
        user = dst;
        n = count;
        if (!dst || count == 0) return;
        if (is_device_ptr(dst)) {
            p = dst;
            return;
        }
        own.alloc(count, s);
        p = own.p;
    }
    void finish(cudaStream_t s) {
        if (own.p) copy_out(user, own.p, n, s);
    }
};

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_prepare_det_batch(const uint64_t* dets, int64_t B, const uint64_t* ref, int n_orb,
                          int n_alpha, int n_beta, int kmax, int flags, int32_t* occ,
                          int8_t* k, int8_t* phase, int32_t* holes, int32_t* parts,
                          uint8_t* hp_mask, int32_t* holes_pos, int32_t* parts_pos,
                          int device, void* stream) {
    DNQ_API_BEGIN
    // the reference's checks, in its order (det_batch.cpp:200-215, :104-124)
    require(n_orb >= 0 && n_orb <= 64, DNQ_ERR_INVALID, "n_orb out of range [0,64]");
    require(B >= 0, DNQ_ERR_INVALID, "negative size");
    require(ref != nullptr && (B == 0 || (dets && occ)), DNQ_ERR_INVALID,
            "null pointer in required outputs");
    require((flags & ~15) == 0, DNQ_ERR_INVALID, "unknown flags");
    const bool need_hp = flags & kNeedHp, need_pos = flags & kNeedPos;
    if (need_hp) flags |= kNeedK;
    require(!need_pos || need_hp, DNQ_ERR_INVALID, "need_hp_pos requires need_hp");
    require(!need_hp || kmax >= 0, DNQ_ERR_INVALID, "kmax must be non-negative");
    require(n_alpha >= 0 && n_beta >= 0, DNQ_ERR_INVALID, "electron count mismatch");
    const u64 m = low_mask(n_orb);
    const u64 ra = ref[0], rb = ref[1];
    if (need_pos)
        require(__builtin_popcountll(ra & m) == n_alpha && __builtin_popcountll(rb & m) == n_beta,
                DNQ_ERR_INVALID, "reference electron count mismatch");
    if (B == 0) return DNQ_OK;
    require(!(flags & kNeedK) || k, DNQ_ERR_INVALID, "k_out is null");
    require(!(flags & kNeedPhase) || phase, DNQ_ERR_INVALID, "phase_out is null");
    require(!need_hp || kmax == 0 || (holes && parts && hp_mask), DNQ_ERR_INVALID,
            "hp outputs are null");
    require(!need_pos || kmax == 0 || (holes_pos && parts_pos), DNQ_ERR_INVALID,
            "pos outputs are null");
    DeviceGuard g(device);
    keep_pool(device);   // the device pool keeps freed memory, as for every other entry point
    cudaStream_t s = (cudaStream_t)stream;
    const int ne = n_alpha + n_beta;
    const size_t nk = need_hp ? (size_t)B * (size_t)kmax : 0;
    DIn<u64> d(dets, 2 * (size_t)B, s);
    DOut<int32_t> o_occ, o_h, o_p, o_hp, o_pp;
    DOut<int8_t> o_k, o_ph;
    DOut<uint8_t> o_m;
    o_occ.set(occ, (size_t)B * ne, s);
    o_k.set((flags & kNeedK) ? k : nullptr, B, s);
    o_ph.set((flags & kNeedPhase) ? phase : nullptr, B, s);
    o_h.set(need_hp ? holes : nullptr, nk, s);
    o_p.set(need_hp ? parts : nullptr, nk, s);
    o_m.set(need_hp ? hp_mask : nullptr, nk, s);
    o_hp.set(need_pos ? holes_pos : nullptr, nk, s);
    o_pp.set(need_pos ? parts_pos : nullptr, nk, s);
    DBuf<unsigned long long> err(1, s);
    DNQ_CUDA(cudaMemsetAsync(err.p, 0xff, sizeof(unsigned long long), s));
    BatchOut bo{o_occ.p, o_k.p, o_ph.p, o_h.p, o_p.p, o_m.p, o_hp.p, o_pp.p};
    const int grid = (int)std::min<i64>((B + 255) / 256, (i64)sm_count(device) * 8);
    k_det_batch<<<grid, 256, 0, s>>>(d.p, B, ra, rb, n_orb, n_alpha, n_beta, kmax, flags, bo,
                                     err.p);
    DNQ_CHECK_LAUNCH();
    unsigned long long e = 0;
    DNQ_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(e), cudaMemcpyDeviceToHost, s));
    o_occ.finish(s);
    o_k.finish(s);
    o_ph.finish(s);
    o_h.finish(s);
    o_p.finish(s);
    o_m.finish(s);
    o_hp.finish(s);
    o_pp.finish(s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    if (e != ~0ull) {
        const u64 code = e & 3;
        require(code != kBadBits, DNQ_ERR_INVALID, "det bits outside n_orb range");
        require(code != kBadCount, DNQ_ERR_INVALID, "electron count mismatch");
        require(false, DNQ_ERR_INVALID, "holes != parts in spin channel");
    }
    DNQ_API_END
}

}  // extern "C"
