// panel.cu -- column-panel layout of the FP32 operator for H.psi.
//
// The CSR H.psi gathers x[col] from L2 for every element: one 32-byte
// sector per 4-byte value, which on B200 costs more than streaming the CSR
// itself (measured: 0.90 ms with gathers, 0.35 ms without, on the
// 1e6-determinant space).  This layout moves the gathers to shared memory:
//
//   rows in blocks of kRB, columns in panels of kPW;
//   entries of a block reordered panel by panel, rows ascending inside a
//   panel, the row's own order kept inside (row, panel);
//   per entry: column offset in its panel (u16) + FP32 value (6 bytes);
//   per non-empty (block, panel) "segment": panel, first entry, and the
//   kRB row lengths (u16).
//
// One CTA per row block: for each of its segments the CTA loads the x
// panel into shared memory, scans the row lengths, and its lane groups
// accumulate Dot2 (TwoProduct + TwoSum) pairs per row in shared memory,
// panel after panel; y = (s + c) + diag * x in FP64.  The result is the
// compensated FP32 operator of spmv.cu with another order of
// accumulation (same accuracy class); it is deterministic and depends on
// the matrix only.
//
// Measured on the 1e6-determinant heat-bath space it is slower than the CSR
// kernel (5.7 ms against 1.0 ms): each row contributes ~3.5 entries to each
// 64 KB panel, and the rows of a block, some with thousands of entries,
// share the block's barriers, so every segment waits for its longest row.
// It is therefore off by default (DNQ_OPT_SPMV_PANELS).
#include <cub/cub.cuh>

#include <vector>

#include "ham.cuh"

namespace dnq {
namespace {

constexpr int kPShift = 14;
constexpr int kPW = 1 << kPShift;   // columns per panel: 64 KB of FP32 x
constexpr int kRB = 2048;           // rows per block
constexpr int kPT = 512;            // threads per CTA
constexpr int kItems = kRB / kPT;   // row lengths scanned per thread

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

// ---- layout construction -------------------------------------------------

// key = ((block * npanels + panel) << rbits) | row in block; row of each
// entry by binary search of the row pointers.
__global__ void k_pkeys(const i64* rowptr, i64 nr, const u32* col, i64 nnz, i64 npanels,
                        int rbits, u64* key, u32* idx) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < nnz;
         k += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = nr;
        while (hi - lo > 1) {
            const i64 mid = (lo + hi) >> 1;
            if (rowptr[mid] <= k) lo = mid; else hi = mid;
        }
        const u64 blk = (u64)(lo / kRB), local = (u64)(lo % kRB);
        const u64 pan = col[k] >> kPShift;
        key[k] = ((blk * (u64)npanels + pan) << rbits) | local;
        idx[k] = (u32)k;
    }
}

__global__ void k_pgather(const u64* skey, const u32* perm, const u32* col, const float* val32,
                          i64 nnz, u16* ocol, float* oval, u32* seg_head, u32* row_head,
                          int rbits) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nnz;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 k = perm[t];
        ocol[t] = (u16)(col[k] & (kPW - 1));
        oval[t] = val32[k];
        const u64 kk = skey[t];
        seg_head[t] = (t == 0 || (skey[t - 1] >> rbits) != (kk >> rbits)) ? 1u : 0u;
        row_head[t] = (t == 0 || skey[t - 1] != kk) ? 1u : 0u;
    }
}

// At every segment head: its panel, block and first entry.
__global__ void k_pseg(const u64* skey, const u32* seg_head, const u32* seg_id, i64 nnz,
                       i64 npanels, int rbits, u32* seg_panel, u32* seg_block, i64* seg_base) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nnz;
         t += (i64)gridDim.x * blockDim.x) {
        if (!seg_head[t]) continue;
        const u32 s = seg_id[t] - 1;
        const u64 bp = skey[t] >> rbits;
        seg_panel[s] = (u32)(bp % (u64)npanels);
        seg_block[s] = (u32)(bp / (u64)npanels);
        seg_base[s] = t;
    }
}

// Row lengths: for each row run (head positions listed), its length goes to
// seg_len[segment * kRB + row in block].
__global__ void k_plen(const u64* skey, const u32* rpos, i64 nruns, i64 nnz, const u32* seg_id,
                       u16* seg_len) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nruns;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 b = rpos[r], e = r + 1 < nruns ? (i64)rpos[r + 1] : nnz;
        const u64 local = skey[b] & (u64)(kRB - 1);
        seg_len[(i64)(seg_id[b] - 1) * kRB + (i64)local] = (u16)(e - b);
    }
}

// First segment of every block (segments are sorted by block).
__global__ void k_pblk(const u32* seg_block, i64 nseg, i64 nblocks, i64* blk_seg) {
    for (i64 b = blockIdx.x * (i64)blockDim.x + threadIdx.x; b <= nblocks;
         b += (i64)gridDim.x * blockDim.x) {
        i64 lo = 0, hi = nseg;
        while (lo < hi) {
            const i64 mid = (lo + hi) >> 1;
            if ((i64)seg_block[mid] < b) lo = mid + 1; else hi = mid;
        }
        blk_seg[b] = lo;
    }
}

__global__ void k_piota(u32* p, i64 n) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        p[t] = (u32)t;
}

int pg(i64 n) {
    const i64 b = (n + 255) / 256;
    return (int)std::max<i64>(1, std::min<i64>(b, 65535));
}

// ---- H.psi -----------------------------------------------------------------

struct PanelView {
    i64 nr, nc, nblocks;
    const i64* blk_seg;
    const u32* seg_panel;
    const i64* seg_base;
    const u16* seg_len;
    const u16* col;
    const float* val;
};

constexpr int kPGS = 8;   // panels per task: a CTA sums one group of panels of one row block

// One CTA per (row block, group of kPGS panels): the group's segments of the
// block are summed into per-row Dot2 pairs, written as the group's partial
// (flag[task] says whether the group had any segment).
template <int G, int D, int RR>
__global__ void __launch_bounds__(kPT, 2) k_spmv_panel(PanelView P, i64 ngroups_p,
                                                    const float* __restrict__ x32,
                                                    float2* __restrict__ part,
                                                    u8* __restrict__ flag) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* xs = reinterpret_cast<float*>(smem);                         // kPW
    float2* acc = reinterpret_cast<float2*>(smem + kPW * 4);            // kRB
    u32* offs = reinterpret_cast<u32*>(smem + kPW * 4 + kRB * 8);       // kRB + 1
    using Scan = cub::BlockScan<u32, kPT>;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ i64 seg_lo, seg_hi;
    const int tid = threadIdx.x, lane = tid & 31;
    const int sub = lane & (G - 1);
    const int group = tid / G, ngroups = kPT / G;
    const i64 ntasks = P.nblocks * ngroups_p;
    for (i64 task = blockIdx.x; task < ntasks; task += gridDim.x) {
        const i64 b = task / ngroups_p, pg = task % ngroups_p;
        const i64 row0 = b * kRB;
        const int nrow = (int)min((i64)kRB, P.nr - row0);
        if (tid == 0) {   // segments of block b with panel in [pg*kPGS, (pg+1)*kPGS)
            const i64 s0 = P.blk_seg[b], s1 = P.blk_seg[b + 1];
            i64 lo = s0, hi = s1;
            while (lo < hi) {
                const i64 mid = (lo + hi) >> 1;
                if ((i64)P.seg_panel[mid] < pg * kPGS) lo = mid + 1; else hi = mid;
            }
            seg_lo = lo;
            hi = s1;
            while (lo < hi) {
                const i64 mid = (lo + hi) >> 1;
                if ((i64)P.seg_panel[mid] < (pg + 1) * kPGS) lo = mid + 1; else hi = mid;
            }
            seg_hi = lo;
        }
        for (int r = tid; r < kRB; r += kPT) acc[r] = make_float2(0.0f, 0.0f);
        __syncthreads();
        const i64 g0 = seg_lo, g1 = seg_hi;
        if (tid == 0) flag[task] = g1 > g0 ? 1 : 0;
        for (i64 sg = g0; sg < g1; ++sg) {
            const i64 c0 = (i64)P.seg_panel[sg] << kPShift;
            const int ncol = (int)min((i64)kPW, P.nc - c0);
            const float* xp = x32 + c0;
            if ((ncol & 3) == 0) {
                for (int t = tid; t < (ncol >> 2); t += kPT)
                    reinterpret_cast<float4*>(xs)[t] = __ldg(reinterpret_cast<const float4*>(xp) + t);
            } else {
                for (int t = tid; t < ncol; t += kPT) xs[t] = __ldg(xp + t);
            }
            u32 len[kItems];
            const u16* lp = P.seg_len + sg * kRB + tid * kItems;
#pragma unroll
            for (int q = 0; q < kItems; ++q) len[q] = lp[q];
            u32 ex[kItems];
            Scan(scan_tmp).ExclusiveSum(len, ex);
#pragma unroll
            for (int q = 0; q < kItems; ++q) offs[tid * kItems + q] = ex[q];
            if (tid == kPT - 1) offs[kRB] = ex[kItems - 1] + len[kItems - 1];
            __syncthreads();
            const u16* cp = P.col + P.seg_base[sg];
            const float* vp = P.val + P.seg_base[sg];
            // rows handed out in rounds of ngroups (every lane of a warp runs
            // the same rounds: the group shuffles need all lanes).  RR rounds
            // at a time, D slots per lane each, are loaded before any is
            // used, so one memory latency covers RR*D entries per lane.
            for (int r0 = 0; r0 < nrow; r0 += ngroups * RR) {
                u32 bb[RR], ee[RR];
#pragma unroll
                for (int q = 0; q < RR; ++q) {
                    const int r = r0 + q * ngroups + group;
                    const bool on = r < nrow;
                    bb[q] = on ? offs[r] : 0u;
                    ee[q] = on ? offs[r + 1] : 0u;
                }
                Pair32 a[RR];
                u32 kb[RR];
#pragma unroll
                for (int q = 0; q < RR; ++q) kb[q] = bb[q] + sub;
                bool more = true;
                while (more) {
                    float v[RR][D];
                    u32 c[RR][D];
#pragma unroll
                    for (int q = 0; q < RR; ++q)
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            const u32 k = kb[q] + (u32)(d * G);
                            const bool ok = k < ee[q];
                            v[q][d] = ok ? __ldcs(vp + k) : 0.0f;
                            c[q][d] = ok ? (u32)__ldcs(cp + k) : 0u;
                        }
                    more = false;
#pragma unroll
                    for (int q = 0; q < RR; ++q) {
#pragma unroll
                        for (int d = 0; d < D; ++d)
                            if (kb[q] + (u32)(d * G) < ee[q]) a[q].add_prod(v[q][d], xs[c[q][d]]);
                        kb[q] += (u32)(D * G);
                        more = more || kb[q] < ee[q];
                    }
                    more = __any_sync(0xffffffffu, more);
                }
#pragma unroll
                for (int q = 0; q < RR; ++q) {
                    Pair32 t = a[q];
#pragma unroll
                    for (int o = G / 2; o; o >>= 1)
                        t.merge(__shfl_xor_sync(0xffffffffu, t.s, o, G),
                                __shfl_xor_sync(0xffffffffu, t.c, o, G));
                    const int r = r0 + q * ngroups + group;
                    if (sub == 0 && r < nrow && ee[q] > bb[q]) {
                        Pair32 u;
                        u.s = acc[r].x;
                        u.c = acc[r].y;
                        u.merge(t.s, t.c);
                        acc[r] = make_float2(u.s, u.c);
                    }
                }
            }
            __syncthreads();   // xs / offs free for the next segment
        }
        if (g1 > g0)
            for (int r = tid; r < nrow; r += kPT) part[pg * P.nr + row0 + r] = acc[r];
        __syncthreads();
    }
}

// y = merge of the groups' partials in group order + diag * x (FP64).
__global__ void k_panel_finish(const float2* part, const u8* flag, i64 nr, i64 ngroups_p,
                               const double* diag, const double* x, double* y) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nr;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 b = r / kRB;
        Pair32 a;
        for (i64 pg = 0; pg < ngroups_p; ++pg)
            if (flag[b * ngroups_p + pg]) {
                const float2 p = part[pg * nr + r];
                a.merge(p.x, p.y);
            }
        double v = (double)a.s + (double)a.c;
        if (diag) v += diag[r] * x[r];
        y[r] = v;
    }
}

size_t panel_smem() { return (size_t)kPW * 4 + (size_t)kRB * 8 + (size_t)(kRB + 1) * 4; }

template <int G, int D, int RR>
void launch_panel(const PanelView& v, i64 ngroups_p, const float* x32, float2* part, u8* flag,
                  int device, cudaStream_t s) {
    auto kern = k_spmv_panel<G, D, RR>;
    const size_t sm = panel_smem();
    DNQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPT, sm));
    const i64 ntasks = v.nblocks * ngroups_p;
    const i64 grid = std::min<i64>(ntasks, (i64)std::max(1, per_sm) * sm_count(device) * 8);
    kern<<<(unsigned)std::max<i64>(1, grid), kPT, sm, s>>>(v, ngroups_p, x32, part, flag);
    DNQ_CHECK_LAUNCH();
}

}  // namespace

// Build the panel layout of a square block from its FP32 value copy
// (diagonal already split off).  Temporary memory: ~24 bytes per entry.
void build_panels(const Csr& m, const float* val32, Panels& P, cudaStream_t s) {
    P.nr = m.nr;
    P.nc = m.nc;
    P.nnz = m.nnz;
    P.nblocks = (m.nr + kRB - 1) / kRB;
    const i64 npanels = std::max<i64>(1, (m.nc + kPW - 1) >> kPShift);
    P.npanels = npanels;
    const i64 n = m.nnz;
    P.col.alloc(n, s);
    P.val.alloc(n, s);
    P.blk_seg.alloc(P.nblocks + 1, s);
    if (n == 0) {
        P.nseg = 0;
        DNQ_CUDA(cudaMemsetAsync(P.blk_seg.p, 0, (P.nblocks + 1) * 8, s));
        P.seg_panel.alloc(1, s);
        P.seg_base.alloc(1, s);
        P.seg_len.alloc(1, s);
        P.part.alloc(2 * std::max<i64>(1, m.nr), s);
        P.flag.alloc(std::max<i64>(1, P.nblocks), s);
        DNQ_CUDA(cudaMemsetAsync(P.flag.p, 0, std::max<i64>(1, P.nblocks), s));
        P.ready = true;
        return;
    }
    require(n < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "panel layout: more than 2^32 entries");
    const int rbits = 11;   // log2(kRB)
    int kbits = rbits;
    while (kbits < 64 && ((u64)1 << (kbits - rbits)) < (u64)(P.nblocks * npanels)) ++kbits;
    DBuf<u64> key(n, s), skey(n, s);
    DBuf<u32> idx(n, s), perm(n, s);
    k_pkeys<<<pg(n), 256, 0, s>>>(m.rowptr.p, m.nr, m.col.p, n, npanels, rbits, key.p, idx.p);
    DNQ_CHECK_LAUNCH();
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, skey.p, idx.p, perm.p, n, 0,
                                                 kbits, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, key.p, skey.p, idx.p, perm.p, n, 0,
                                                 kbits, s));
    }
    key.release();
    idx.release();
    DBuf<u32> seg_head(n, s), row_head(n, s), seg_id(n, s);
    k_pgather<<<pg(n), 256, 0, s>>>(skey.p, perm.p, m.col.p, val32, n, P.col.p, P.val.p,
                                    seg_head.p, row_head.p, rbits);
    DNQ_CHECK_LAUNCH();
    perm.release();
    {
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, seg_head.p, seg_id.p, n, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceScan::InclusiveSum(tb.p, tmp, seg_head.p, seg_id.p, n, s));
    }
    u32 nseg = 0;
    DNQ_CUDA(cudaMemcpyAsync(&nseg, seg_id.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    P.nseg = nseg;
    P.seg_panel.alloc(nseg, s);
    P.seg_base.alloc(nseg, s);
    P.seg_len.alloc((size_t)nseg * kRB, s);
    DNQ_CUDA(cudaMemsetAsync(P.seg_len.p, 0, (size_t)nseg * kRB * 2, s));
    DBuf<u32> seg_block(nseg, s);
    k_pseg<<<pg(n), 256, 0, s>>>(skey.p, seg_head.p, seg_id.p, n, npanels, rbits, P.seg_panel.p,
                                 seg_block.p, P.seg_base.p);
    DNQ_CHECK_LAUNCH();
    {   // row runs
        DBuf<u32> pos(n, s), rpos(n, s);
        DBuf<i64> nr(1, s);
        k_piota<<<pg(n), 256, 0, s>>>(pos.p, n);
        DNQ_CHECK_LAUNCH();
        size_t tmp = 0;
        DNQ_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, pos.p, row_head.p, rpos.p, nr.p, n, s));
        DBuf<u8> tb(tmp, s);
        DNQ_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, pos.p, row_head.p, rpos.p, nr.p, n, s));
        i64 nruns = 0;
        DNQ_CUDA(cudaMemcpyAsync(&nruns, nr.p, 8, cudaMemcpyDeviceToHost, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        k_plen<<<pg(nruns), 256, 0, s>>>(skey.p, rpos.p, nruns, n, seg_id.p, P.seg_len.p);
        DNQ_CHECK_LAUNCH();
    }
    k_pblk<<<pg(P.nblocks + 1), 256, 0, s>>>(seg_block.p, nseg, P.nblocks, P.blk_seg.p);
    DNQ_CHECK_LAUNCH();
    // lanes per row by the average entries of a (row, segment)
    const double avg = (double)n / ((double)nseg * kRB);
    P.group = avg >= 48 ? 32 : avg >= 16 ? 8 : avg >= 6 ? 4 : 1;
    {
        const i64 ngp = (npanels + kPGS - 1) / kPGS;
        P.part.alloc((size_t)ngp * m.nr * 2, s);
        P.flag.alloc((size_t)P.nblocks * ngp, s);
    }
    DNQ_CUDA(cudaStreamSynchronize(s));
    P.ready = true;
}

// y = M x with the panel layout (x32: the FP32 copy of x, nc floats).
void spmv_panels(const Panels& P, const float* x32, const double* diag, const double* x,
                 double* y, int device, cudaStream_t s) {
    if (P.nr == 0) return;
    PanelView v{P.nr, P.nc, P.nblocks, P.blk_seg.p, P.seg_panel.p, P.seg_base.p, P.seg_len.p,
                P.col.p, P.val.p};
    const i64 ngp = (P.npanels + kPGS - 1) / kPGS;
    float2* part = reinterpret_cast<float2*>(P.part.p);
    switch (P.group) {
        case 32: launch_panel<32, 4, 1>(v, ngp, x32, part, P.flag.p, device, s); break;
        case 8: launch_panel<8, 2, 2>(v, ngp, x32, part, P.flag.p, device, s); break;
        case 4: launch_panel<4, 2, 4>(v, ngp, x32, part, P.flag.p, device, s); break;
        default: launch_panel<1, 4, 4>(v, ngp, x32, part, P.flag.p, device, s); break;
    }
    k_panel_finish<<<pg(P.nr), 256, 0, s>>>(part, P.flag.p, P.nr, ngp, diag, x, y);
    DNQ_CHECK_LAUNCH();
}

}  // namespace dnq
