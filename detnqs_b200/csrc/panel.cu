// panel.cu -- column-panel layout of the FP32 operator for H.psi.
//
// The CSR H.psi gathers x[col] through L1 for every element: one 32-byte
// sector per 4-byte value, and an SM's L1 returns about one sector per
// clock, which bounds the CSR kernel (ncu: 1.0 sector per SM clock).  This
// layout moves the gathers to shared memory:
//
//   columns in panels of kPW (192 KB of FP32 x: one panel fills a CTA's
//   shared memory); a row's entries in a panel are cut into chunks of at
//   most kChunkLen, in CSR order; the chunks of a panel, ordered by length
//   (longest first), form slices of 32 chunks; a slice stores its entries
//   k-major (slot k * 32 + lane holds entry k of the slice's chunk `lane`),
//   padded to the slice's longest chunk with zero values: column offset in
//   the panel (u16) + FP32 value, 6 bytes per slot.  The chunk length bounds
//   the serial work of a lane, so rows of thousands of entries in one panel
//   do not hold a warp.
//
// One CTA per SM, persistent: panel after panel it loads x's panel into
// shared memory and its warps run their share of the panel's slices (split
// by slots), a lane summing its chunk's entries as a Dot2 (TwoProduct +
// TwoSum) pair.  The pair of each chunk is stored; a finishing kernel
// merges a row's chunk pairs in (panel, chunk) order and adds diag * x in
// FP64.  The result is the compensated FP32 operator with another order of
// accumulation (same accuracy class), and deterministic: a chunk's sum is
// one lane's, in CSR order, whichever CTA runs it.
//
// Measured on the 1e6-determinant heat-bath space it is still slower than
// the CSR kernel (1.37 ms against 1.0 ms): a row keeps ~13 entries per panel,
// so a lane's chunk is short and each warp step waits a full memory latency
// for four of them; loading sixteen ahead wasted more than it hid (2.5 ms).
// It is therefore off by default (DNQ_OPT_SPMV_PANELS).  The first layout
// (row blocks x 16k-column panels, one CTA per block) took 5.7 ms.
#include <cub/cub.cuh>

#include <vector>

#include "ham.cuh"

namespace dnq {
namespace {

constexpr i64 kPW = 49152;          // columns per panel (192 KB of FP32 x)
constexpr u32 kChunkLen = 64;       // entries of a row in a panel per chunk
constexpr int kPT = 1024;           // threads per CTA
constexpr u32 kNoRow = 0xffffffffu;

__device__ __forceinline__ void ts(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float z = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z));
}

struct Pair32 {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add_prod(float a, float b) {
        const float p = __fmul_rn(a, b);
        const float pe = fmaf(a, b, -p);
        float s2, e;
        ts(s, p, s2, e);
        s = s2;
        c = __fadd_rn(c, __fadd_rn(e, pe));
    }
    __device__ __forceinline__ void merge(float os, float oc) {
        float s2, e;
        ts(s, os, s2, e);
        s = s2;
        c = __fadd_rn(__fadd_rn(c, oc), e);
    }
};

int pg(i64 n) {
    const i64 b = (n + 255) / 256;
    return (int)std::max<i64>(1, std::min<i64>(b, 65535));
}

// ---- layout construction -------------------------------------------------

// key = panel << 32 | row of every entry (row by binary search of rowptr).
__global__ void k_pkeys(const i64* rowptr, i64 nr, const u32* col, i64 nnz, u64* key, u32* idx) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < nnz;
         k += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = nr;
        while (hi - lo > 1) {
            const i64 mid = (lo + hi) >> 1;
            if (rowptr[mid] <= k) lo = mid; else hi = mid;
        }
        key[k] = ((u64)(col[k] / (u32)kPW) << 32) | (u64)lo;
        idx[k] = (u32)k;
    }
}

__global__ void k_heads(const u64* skey, i64 n, u32* head) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        head[t] = (t == 0 || skey[t - 1] != skey[t]) ? 1u : 0u;
}

__global__ void k_iota(u32* p, i64 n) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        p[t] = (u32)t;
}

// Per (panel, row) pair: its entry count and chunk count.
__global__ void k_pairs(const u32* pstart, i64 np, i64 n, u32* pcount, u32* pnch) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < np;
         i += (i64)gridDim.x * blockDim.x) {
        const i64 b = pstart[i], e = i + 1 < np ? (i64)pstart[i + 1] : n;
        const u32 c = (u32)(e - b);
        pcount[i] = c;
        pnch[i] = (c + kChunkLen - 1) / kChunkLen;
    }
}

// Chunks of every pair, in (panel, row, chunk) order: their pair, length,
// the slicing key panel << 32 | (2^32 - 1 - length) (longest first) and the
// gathering key row << 32 | panel << 16 | chunk.
__global__ void k_chunks(const u64* skey, const u32* pstart, const u32* pcount, const i64* cpre,
                         i64 np, u32* cpair, u32* clen, u64* skey_c, u64* rkey_c) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < np;
         i += (i64)gridDim.x * blockDim.x) {
        const u64 k = skey[pstart[i]];
        const u64 panel = k >> 32, row = k & 0xffffffffull;
        const u32 cnt = pcount[i];
        for (u32 q = 0; q * kChunkLen < cnt; ++q) {
            const i64 c = cpre[i] + q;
            const u32 len = min(kChunkLen, cnt - q * kChunkLen);
            cpair[c] = (u32)i;
            clen[c] = len;
            skey_c[c] = (panel << 32) | (u64)(0xffffffffu - len);
            rkey_c[c] = (row << 32) | (panel << 16) | (u64)q;
        }
    }
}

// First sorted chunk of every panel.
__global__ void k_panel_first(const u64* skey_s, i64 m, i64 npanels, u32* first) {
    for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p <= npanels;
         p += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = m;
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if ((i64)(skey_s[mid] >> 32) < p) lo = mid + 1; else hi = mid;
        }
        first[p] = (u32)lo;
    }
}

// Sorted chunk j -> slice and lane; slice widths from their first chunk.
__global__ void k_inverse(const u32* order, i64 m, u32* inv) {
    for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < m;
         j += (i64)gridDim.x * blockDim.x)
        inv[order[j]] = (u32)j;
}

// schunk holds the chunk's place in the row-ordered list: its partial is
// written there, so a row's partials are contiguous for the merge.
__global__ void k_slices(const u32* order, const u64* skey_s, const u32* pfirst, const i64* sfirst,
                         const u32* clen, const u32* rpos, i64 m, u32* cslot, u32* swidth,
                         u32* schunk) {
    for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < m;
         j += (i64)gridDim.x * blockDim.x) {
        const u32 p = (u32)(skey_s[j] >> 32);
        const i64 rank = j - (i64)pfirst[p];
        const i64 s = sfirst[p] + rank / 32;
        const u32 lane = (u32)(rank % 32);
        const u32 c = order[j];
        cslot[c] = (u32)(s * 32 + lane);
        if (lane == 0) swidth[s] = clen[c];
        schunk[s * 32 + lane] = rpos[c];
    }
}

__global__ void k_slots(const u32* swidth, i64 ns, i64* slots) {
    for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < ns;
         s += (i64)gridDim.x * blockDim.x)
        slots[s] = (i64)swidth[s] * 32;
}

// Entry t of the (panel, row)-sorted order -> its slot.
__global__ void k_scatter(const u64* skey, const u32* perm, const u32* pair_id, const u32* pstart,
                          const i64* cpre, const u32* cslot, const i64* soff, const u32* col,
                          const float* val32, i64 n, u16* ocol, float* oval) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 i = pair_id[t] - 1;
        const i64 k = t - (i64)pstart[i];
        const u32 sl = cslot[cpre[i] + k / kChunkLen];
        const i64 dst = soff[sl / 32] + (k % kChunkLen) * 32 + (sl % 32);
        const u32 e = perm[t];
        ocol[dst] = (u16)(col[e] - (u32)((skey[t] >> 32) * (u64)kPW));
        oval[dst] = val32[e];
    }
}

// First chunk of every row in the row-sorted chunk keys.
__global__ void k_row_first(const u64* rkey_s, i64 m, i64 nr, i64* rptr) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r <= nr;
         r += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = m;
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if ((i64)(rkey_s[mid] >> 32) < r) lo = mid + 1; else hi = mid;
        }
        rptr[r] = lo;
    }
}

// Slice bounds of every CTA in every panel, by slots.
__global__ void k_split(const i64* sfirst, const i64* soff, i64 npanels, int grid, u32* split) {
    for (i64 q = blockIdx.x * (i64)blockDim.x + threadIdx.x; q < npanels * (grid + 1);
         q += (i64)gridDim.x * blockDim.x) {
        const i64 p = q / (grid + 1), c = q % (grid + 1);
        const i64 s0 = sfirst[p], s1 = sfirst[p + 1];
        if (c == grid) {
            split[q] = (u32)s1;
            continue;
        }
        const i64 target = soff[s0] + (soff[s1] - soff[s0]) * c / grid;
        i64 lo = s0, hi = s1;   // first slice starting at or after target
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if (soff[mid] < target) lo = mid + 1; else hi = mid;
        }
        split[q] = (u32)lo;
    }
}

// ---- H.psi -----------------------------------------------------------------

struct SliceView {
    i64 nr, nc, npanels;
    const u16* col;
    const float* val;
    const i64* soff;
    const u32* swidth;
    const u32* schunk;
    const u32* split;
};

// Persistent: one CTA per SM, panel after panel.
__global__ void __launch_bounds__(kPT, 1) k_spmv_slices(SliceView V, const float* __restrict__ x32,
                                                        float2* __restrict__ part) {
    extern __shared__ __align__(16) float xs[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (i64 p = 0; p < V.npanels; ++p) {
        const i64 c0 = p * kPW;
        const int ncol = (int)min(kPW, V.nc - c0);
        const float* xp = x32 + c0;   // c0 is a multiple of 4 floats (16 bytes)
        for (int t = tid; t < (ncol >> 2); t += kPT)
            reinterpret_cast<float4*>(xs)[t] = __ldg(reinterpret_cast<const float4*>(xp) + t);
        for (int t = (ncol & ~3) + tid; t < ncol; t += kPT) xs[t] = __ldg(xp + t);
        __syncthreads();
        const u32* sp = V.split + p * (gridDim.x + 1);
        const u32 s0 = sp[blockIdx.x], s1 = sp[blockIdx.x + 1];
        // the next slice's offset, width and chunk are loaded while the
        // current one is summed
        u32 s = s0 + warp;
        i64 nbase = 0;
        u32 nw = 0, nchunk = kNoRow;
        if (s < s1) {
            nbase = V.soff[s];
            nw = V.swidth[s];
            nchunk = V.schunk[(i64)s * 32 + lane];
        }
        for (; s < s1; s += kPT / 32) {
            const i64 base = nbase + lane;
            const u32 w = nw, chunk = nchunk;
            const u32 sn = s + kPT / 32;
            if (sn < s1) {
                nbase = V.soff[sn];
                nw = V.swidth[sn];
                nchunk = V.schunk[(i64)sn * 32 + lane];
            }
            Pair32 a;
            u32 k = 0;
            for (; k + 4 <= w; k += 4) {
                float v[4];
                u32 c[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    v[q] = __ldcs(V.val + base + (i64)(k + q) * 32);
                    c[q] = __ldcs(V.col + base + (i64)(k + q) * 32);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) a.add_prod(v[q], xs[c[q]]);
            }
            for (; k < w; ++k)
                a.add_prod(__ldcs(V.val + base + (i64)k * 32), xs[__ldcs(V.col + base + (i64)k * 32)]);
            if (chunk != kNoRow) part[chunk] = make_float2(a.s, a.c);
        }
        __syncthreads();   // xs free for the next panel
    }
}

// y = merge of a row's chunk pairs in (panel, chunk) order (contiguous in
// part) + diag * x (FP64).
__global__ void k_slices_finish(const float2* part, const i64* rptr, i64 nr, const double* diag,
                                const double* x, double* y) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nr;
         r += (i64)gridDim.x * blockDim.x) {
        Pair32 a;
        for (i64 j = rptr[r]; j < rptr[r + 1]; ++j) {
            const float2 q = part[j];
            a.merge(q.x, q.y);
        }
        double v = (double)a.s + (double)a.c;
        if (diag) v += diag[r] * x[r];
        y[r] = v;
    }
}

size_t panel_smem() { return (size_t)kPW * 4; }

}  // namespace

// Build the panel layout of a square block from its FP32 value copy
// (diagonal already split off).  Temporary memory: ~60 bytes per entry.
void build_panels(const Csr& M, const float* val32, Panels& P, cudaStream_t s) {
    P.nr = M.nr;
    P.nc = M.nc;
    P.nnz = M.nnz;
    const i64 npanels = std::max<i64>(1, (M.nc + kPW - 1) / kPW);
    P.npanels = npanels;
    int dev = 0;
    DNQ_CUDA(cudaGetDevice(&dev));
    P.grid = sm_count(dev);
    const i64 n = M.nnz;
    P.rptr.alloc(M.nr + 1, s);
    if (n == 0) {
        P.nslices = 0;
        P.nent = 0;
        P.nchunks = 0;
        P.col.alloc(1, s);
        P.val.alloc(1, s);
        P.soff.alloc(1, s);
        P.swidth.alloc(1, s);
        P.schunk.alloc(32, s);
        P.part.alloc(2, s);
        P.split.alloc((size_t)npanels * (P.grid + 1), s);
        DNQ_CUDA(cudaMemsetAsync(P.split.p, 0, P.split.bytes(), s));
        DNQ_CUDA(cudaMemsetAsync(P.rptr.p, 0, P.rptr.bytes(), s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        P.ready = true;
        return;
    }
    require(n < (i64)0x7fffffffll, DNQ_ERR_OVERFLOW, "panel layout: more than 2^31 entries");
    require(npanels < 65536, DNQ_ERR_OVERFLOW, "panel layout: more than 65535 panels");
    int pbits = 1;
    while (((i64)1 << pbits) < npanels + 1) ++pbits;
    // entries by (panel, row), stably: a row's entries of a panel keep their order
    DBuf<u64> key(n, s), skey(n, s);
    DBuf<u32> idx(n, s), perm(n, s);
    k_pkeys<<<pg(n), 256, 0, s>>>(M.rowptr.p, M.nr, M.col.p, n, key.p, idx.p);
    DNQ_CHECK_LAUNCH();
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, skey.p, idx.p, perm.p, n, 0,
                                                 32 + pbits, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, key.p, skey.p, idx.p, perm.p, n, 0,
                                                 32 + pbits, s));
    }
    key.release();
    idx.release();
    // (panel, row) pairs: first entry
    DBuf<u32> head(n, s), pair_id(n, s), pos(n, s), pstart(n, s);
    DBuf<i64> npair_d(1, s);
    k_heads<<<pg(n), 256, 0, s>>>(skey.p, n, head.p);
    DNQ_CHECK_LAUNCH();
    k_iota<<<pg(n), 256, 0, s>>>(pos.p, n);
    DNQ_CHECK_LAUNCH();
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, pos.p, head.p, pstart.p, npair_d.p, n, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, pos.p, head.p, pstart.p, npair_d.p, n, s));
        size_t t2 = 0;
        DNQ_CUDA(cub::DeviceScan::InclusiveSum(nullptr, t2, head.p, pair_id.p, n, s));
        DBuf<u8> tb2(t2, s);
        DNQ_CUDA(cub::DeviceScan::InclusiveSum(tb2.p, t2, head.p, pair_id.p, n, s));
    }
    pos.release();
    head.release();
    i64 np = 0;
    DNQ_CUDA(cudaMemcpyAsync(&np, npair_d.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    // chunks of every pair
    DBuf<u32> pcount(np, s), pnch(np + 1, s);
    DBuf<i64> cpre(np + 1, s);
    k_pairs<<<pg(np), 256, 0, s>>>(pstart.p, np, n, pcount.p, pnch.p);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaMemsetAsync(pnch.p + np, 0, 4, s));
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, pnch.p, cpre.p, np + 1, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, pnch.p, cpre.p, np + 1, s));
    }
    i64 mc = 0;
    DNQ_CUDA(cudaMemcpyAsync(&mc, cpre.p + np, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    P.nchunks = mc;
    DBuf<u32> cpair(mc, s), clen(mc, s), ciota(mc, s), corder(mc, s), rorder(mc, s);
    DBuf<u64> ckey(mc, s), sckey(mc, s), rkey(mc, s), srkey(mc, s);
    k_chunks<<<pg(np), 256, 0, s>>>(skey.p, pstart.p, pcount.p, cpre.p, np, cpair.p, clen.p,
                                    ckey.p, rkey.p);
    DNQ_CHECK_LAUNCH();
    k_iota<<<pg(mc), 256, 0, s>>>(ciota.p, mc);
    DNQ_CHECK_LAUNCH();
    {   // slicing order: panel, then length (longest first); row order: row, panel, chunk
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ckey.p, sckey.p, ciota.p, corder.p,
                                                 mc, 0, 32 + pbits, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, ckey.p, sckey.p, ciota.p, corder.p,
                                                 mc, 0, 32 + pbits, s));
        size_t t2 = 0;
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, rkey.p, srkey.p, ciota.p, rorder.p,
                                                 mc, 0, 64, s));
        DBuf<u8> tb2(t2, s);
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(tb2.p, t2, rkey.p, srkey.p, ciota.p, rorder.p,
                                                 mc, 0, 64, s));
    }
    DBuf<u32> pfirst(npanels + 1, s);
    k_panel_first<<<pg(npanels + 1), 256, 0, s>>>(sckey.p, mc, npanels, pfirst.p);
    DNQ_CHECK_LAUNCH();
    std::vector<u32> hfirst(npanels + 1);
    DNQ_CUDA(cudaMemcpyAsync(hfirst.data(), pfirst.p, 4 * (npanels + 1), cudaMemcpyDeviceToHost,
                             s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    std::vector<i64> hsf(npanels + 1, 0);
    for (i64 p = 0; p < npanels; ++p)
        hsf[p + 1] = hsf[p] + ((i64)hfirst[p + 1] - hfirst[p] + 31) / 32;
    const i64 ns = hsf[npanels];
    P.nslices = ns;
    DBuf<i64> sfirst(npanels + 1, s);
    DNQ_CUDA(cudaMemcpyAsync(sfirst.p, hsf.data(), 8 * (npanels + 1), cudaMemcpyHostToDevice, s));
    P.swidth.alloc(std::max<i64>(1, ns), s);
    P.schunk.alloc((size_t)std::max<i64>(1, ns) * 32, s);
    DNQ_CUDA(cudaMemsetAsync(P.schunk.p, 0xff, P.schunk.bytes(), s));
    DBuf<u32> cslot(mc, s), rpos(mc, s);
    k_inverse<<<pg(mc), 256, 0, s>>>(rorder.p, mc, rpos.p);   // chunk -> its place in row order
    DNQ_CHECK_LAUNCH();
    k_slices<<<pg(mc), 256, 0, s>>>(corder.p, sckey.p, pfirst.p, sfirst.p, clen.p, rpos.p, mc,
                                    cslot.p, P.swidth.p, P.schunk.p);
    DNQ_CHECK_LAUNCH();
    // slot offsets of the slices
    P.soff.alloc(ns + 1, s);
    {
        DBuf<i64> slots(ns + 1, s);
        DNQ_CUDA(cudaMemsetAsync(slots.p + ns, 0, 8, s));
        k_slots<<<pg(ns), 256, 0, s>>>(P.swidth.p, ns, slots.p);
        DNQ_CHECK_LAUNCH();
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, slots.p, P.soff.p, ns + 1, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, slots.p, P.soff.p, ns + 1, s));
    }
    DNQ_CUDA(cudaMemcpyAsync(&P.nent, P.soff.p + ns, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    P.col.alloc(std::max<i64>(1, P.nent), s);
    P.val.alloc(std::max<i64>(1, P.nent), s);
    DNQ_CUDA(cudaMemsetAsync(P.col.p, 0, P.col.bytes(), s));
    DNQ_CUDA(cudaMemsetAsync(P.val.p, 0, P.val.bytes(), s));
    k_scatter<<<pg(n), 256, 0, s>>>(skey.p, perm.p, pair_id.p, pstart.p, cpre.p, cslot.p,
                                    P.soff.p, M.col.p, val32, n, P.col.p, P.val.p);
    DNQ_CHECK_LAUNCH();
    // chunks of every row in (panel, chunk) order, for the finishing merge
    k_row_first<<<pg(M.nr + 1), 256, 0, s>>>(srkey.p, mc, M.nr, P.rptr.p);
    DNQ_CHECK_LAUNCH();
    P.part.alloc((size_t)std::max<i64>(1, mc) * 2, s);
    P.split.alloc((size_t)npanels * (P.grid + 1), s);
    k_split<<<pg(npanels * (P.grid + 1)), 256, 0, s>>>(sfirst.p, P.soff.p, npanels, P.grid,
                                                       P.split.p);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaStreamSynchronize(s));
    P.ready = true;
}

// y = M x with the panel layout (x32: the FP32 copy of x, nc floats).
void spmv_panels(const Panels& P, const float* x32, const double* diag, const double* x,
                 double* y, int device, cudaStream_t s) {
    (void)device;
    if (P.nr == 0) return;
    float2* part = reinterpret_cast<float2*>(P.part.p);
    if (P.nslices) {
        SliceView v{P.nr, P.nc, P.npanels, P.col.p, P.val.p, P.soff.p, P.swidth.p, P.schunk.p,
                    P.split.p};
        const size_t sm = panel_smem();
        DNQ_CUDA(cudaFuncSetAttribute(k_spmv_slices, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sm));
        k_spmv_slices<<<P.grid, kPT, sm, s>>>(v, x32, part);
        DNQ_CHECK_LAUNCH();
    }
    k_slices_finish<<<pg(P.nr), 256, 0, s>>>(part, P.rptr.p, P.nr, diag, x, y);
    DNQ_CHECK_LAUNCH();
}

}  // namespace dnq
