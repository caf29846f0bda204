// heff.cu -- downfolding H_eff = H_VV + H_VP D^-1 H_PV
// (get_ham_eff, ham_eff.cpp:35-233).
//
//   1. H_VP and H_VV canonicalised on the device (sort by (row, col), sum
//      duplicates, drop exact zeros: coo_to_csr, ham_utils.cpp:246-302);
//      H_PV = transpose (rows ascending inside each column, as coo_to_csc).
//   2. D^-1 in FP64 (sigma: d/(d^2+eps^2), linear: 1/(d+sgn(d) eps)) and
//      column screening |D^-1_k| * ||col_k||^2 < 1e-12 (ham_eff.cpp:93-106).
//   3. One warp per output row i walks the entries (k, a) of H_VP row i in
//      ascending k and scatters a*D^-1_k*H_VP[j,k] into a dense accumulator
//      over j (shared memory when it fits, else a per-warp HBM slab), with a
//      bitmap of touched columns; the k loop is sequential so every output
//      element is summed in the reference's order.  FP64 mode uses
//      unfused multiply/add like the reference build; FP32 mode reads FP32
//      H_VP values and keeps a float-float accumulator per element: each
//      product's rounding error (TwoProduct) and each sum's (TwoSum) go to
//      the error word, which is renormalised against the sum after every
//      add (FastTwoSum; Dekker 1971), so ~1e6 terms into one element stay
//      accurate to a few FP32 ulps squared.
//   4. The H_VV row is added, entries with |v| <= 1e-15 dropped
//      (csr_add, ham_utils.cpp:330-442), and the row is compacted in column
//      order from the bitmap.

#include <memory>
#include <vector>

#include "ham.cuh"
#include "prim.cuh"

namespace dnq {

void transpose_csr(const Csr& a, Csr& t, cudaStream_t s);

namespace {

constexpr int kHW = 4;   // warps per block

__global__ void k_coo_keys(const u32* r, const u32* c, i64 n, u64* key, u32* idx,
                           unsigned long long* bad, i64 nr, i64 nc) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if ((i64)r[t] >= nr || (i64)c[t] >= nc) atomicAdd(bad, 1ull);
        key[t] = ((u64)r[t] << 32) | c[t];
        idx[t] = (u32)t;
    }
}

__global__ void k_run_flags(const u64* key, i64 n, u32* flag) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        flag[t] = (t == 0 || key[t] != key[t - 1]) ? 1u : 0u;
}

// Sum each run of equal keys in input order; mark zero sums.
__global__ void k_run_sum(const u64* key, const u32* perm, const double* val, const u32* runid,
                          i64 n, double* rsum, u64* rkey) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (!(t == 0 || key[t] != key[t - 1])) continue;
        double acc = val[perm[t]];
        i64 u = t + 1;
        while (u < n && key[u] == key[t]) acc = __dadd_rn(acc, val[perm[u]]), ++u;
        rsum[runid[t] - 1] = acc;
        rkey[runid[t] - 1] = key[t];
    }
}

__global__ void k_nonzero(const double* v, i64 n, u32* f) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        f[t] = v[t] != 0.0;
}

__global__ void k_scatter_csr(const u64* rkey, const double* rsum, const u32* keep,
                              const u32* pos, i64 n, u32* col, double* val, u32* rowcnt) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        if (!keep[t]) continue;
        const u32 p = pos[t];
        col[p] = (u32)(rkey[t] & 0xffffffffu);
        val[p] = rsum[t];
        atomicAdd(&rowcnt[rkey[t] >> 32], 1u);
    }
}

__global__ void k_dinv(const double* hpp, i64 n, double e_ref, double eps, int sigma,
                       double* dinv) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < n;
         k += (i64)gridDim.x * blockDim.x) {
        const double d = __dsub_rn(e_ref, hpp[k]);
        dinv[k] = sigma ? __ddiv_rn(d, __dadd_rn(__dmul_rn(d, d), __dmul_rn(eps, eps)))
                        : __ddiv_rn(1.0, __dadd_rn(d, copysign(eps, d)));
    }
}

// ||col_k||^2 in row order (unfused, as the reference) and the skip flag.
__global__ void k_screen(const i64* rp, const double* val, i64 n, const double* dinv,
                         u8* skip) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < n;
         k += (i64)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (i64 q = rp[k]; q < rp[k + 1]; ++q) s = __dadd_rn(s, __dmul_rn(val[q], val[q]));
        skip[k] = __dmul_rn(fabs(dinv[k]), s) < 1e-12;
    }
}

// Capacity of output row i: its H_VV entries plus the sum of the H_PV
// column lengths it scatters.  Per-entry column lengths first (one thread
// per H_VP entry), then a segmented sum per row, so a row with millions of
// entries is spread over the whole GPU.
__global__ void k_cap_terms(const u32* vpcol, i64 nnz, const i64* pvrp, const u8* skip,
                            i64* len) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < nnz;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 k = vpcol[t];
        len[t] = skip[k] ? 0 : pvrp[k + 1] - pvrp[k];
    }
}

__global__ void k_cap_finish(const i64* sum, const i64* vvrp, i64 nv, i64* cap) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < nv;
         i += (i64)gridDim.x * blockDim.x) {
        const i64 c = sum[i] + (vvrp[i + 1] - vvrp[i]);
        cap[i] = c < nv ? c : nv;
    }
}

__device__ __forceinline__ void f_two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float z = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z));
}

struct HeffParams {
    i64 nv;
    const i64* vprp; const u32* vpcol; const double* vpval; const float* vpval32;
    const i64* pvrp; const u32* pvcol; const double* pvval; const float* pvval32;
    const i64* vvrp; const u32* vvcol; const double* vvval;
    const double* dinv; const u8* skip;
    const i64* capoff;
    u32* tcol; double* tval; u32* rowcnt;
    int* next_row;
    double* gacc;    // per-warp dense accumulators when not in shared memory
    u32* gbits;
    int words;       // bitmap words per warp
    // rows with very many H_VP entries: diagonal precomputed, walk limited
    // to the k's whose H_PV column holds other rows
    const int* long_id;          // per row: long-row index or -1 (null: none)
    const i64* long_off;         // per long row: range in long_j / long_v / long_v2
    const u32* long_j;           // output columns j != i of the row, ascending
    const double* long_v;        // their FP64 sums (k order)
    const float2* long_v2;       // their FP32 float-float sums
    const double* long_diag;     // FP64 diagonal sum
    const float2* long_diag2;    // FP32 float-float diagonal sum
    const u32* long_touch;       // any k of the row not screened out
};

// F32 = false: acc holds FP64 sums.  F32 = true: during the scatter acc
// holds (sum, err) float pairs, folded to FP64 before H_VV is added.
template <bool F32, bool SMEM>
__global__ void __launch_bounds__(kHW * 32) k_heff(HeffParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const i64 gw = (i64)blockIdx.x * kHW + w;
    u32* bits;
    double* acc;
    if (SMEM) {
        const size_t per = (((size_t)P.words * 4 + 15) & ~(size_t)15) + (size_t)P.nv * 8;
        unsigned char* base = smem + per * w;
        bits = (u32*)base;
        acc = (double*)(base + (((size_t)P.words * 4 + 15) & ~(size_t)15));
        for (int t = lane; t < P.words; t += 32) bits[t] = 0u;
        for (i64 t = lane; t < P.nv; t += 32) acc[t] = 0.0;
        __syncwarp();
    } else {
        bits = P.gbits + gw * P.words;
        acc = P.gacc + gw * P.nv;
    }
    float2* acc2 = reinterpret_cast<float2*>(acc);
    for (;;) {
        int i = 0;
        if (lane == 0) i = atomicAdd(P.next_row, 1);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= P.nv) break;
        // ---- scatter H_VP row i, k ascending.  Every H_PV column k of this
        // row holds row i itself, so the diagonal element receives one term
        // per k: it is kept in lane 0's registers (same order of additions).
        // The metadata of 32 k's is fetched at once by the lanes; columns
        // that hold only row i need no slab access at all.
        double dacc = 0.0;             // FP64 diagonal sum
        float dhi = 0.0f, dlo = 0.0f;  // FP32 float-float diagonal sum
        bool dtouch = false;
        const int lid = P.long_id ? P.long_id[i] : -1;
        if (lid >= 0) {   // precomputed sums of a long row (same order, same values)
            for (i64 x = P.long_off[lid] + lane; x < P.long_off[lid + 1]; x += 32) {
                const u32 j = P.long_j[x];
                atomicOr(&bits[j >> 5], 1u << (j & 31));
                if (F32) acc2[j] = P.long_v2[x];
                else acc[j] = P.long_v[x];
            }
            __syncwarp();
        }
        const i64 t_base = P.vprp[i];
        const i64 n_items = lid >= 0 ? 0 : P.vprp[i + 1] - t_base;
        for (i64 x0 = 0; x0 < n_items; x0 += 32) {
            const i64 xl = x0 + lane;
            const bool inr = xl < n_items;
            const i64 tl = inr ? t_base + xl : 0;
            u32 kl = 0;
            bool sk = true;
            double al = 0.0, sl = 0.0;
            i64 q0l = 0, q1l = 0, qdl = -1;
            if (inr) {
                kl = P.vpcol[tl];
                sk = P.skip[kl] != 0;
                sl = P.dinv[kl];
                al = F32 ? (double)P.vpval32[tl] : P.vpval[tl];
                q0l = P.pvrp[kl];
                q1l = P.pvrp[kl + 1];
                i64 lo = q0l, hi = q1l;   // position of row i in column k
                while (lo < hi) {
                    const i64 mid = (lo + hi) >> 1;
                    if (P.pvcol[mid] < (u32)i) lo = mid + 1; else hi = mid;
                }
                qdl = lo;
            }
            const double bdl = (inr && !sk) ? (F32 ? (double)P.pvval32[qdl] : P.pvval[qdl]) : 0.0;
            const int cnt = (int)min((i64)32, n_items - x0);
            for (int u = 0; u < cnt; ++u) {
                if (__shfl_sync(0xffffffffu, (int)sk, u)) continue;
                const double s = __shfl_sync(0xffffffffu, sl, u);
                const double a = __shfl_sync(0xffffffffu, al, u);
                const i64 q0 = __shfl_sync(0xffffffffu, q0l, u);
                const i64 q1 = __shfl_sync(0xffffffffu, q1l, u);
                const i64 qd = __shfl_sync(0xffffffffu, qdl, u);
                const double bd = __shfl_sync(0xffffffffu, bdl, u);
                const bool need = !(a == 0.0 || s == 0.0);
                if (!F32) {
                    const double as = __dmul_rn(a, s);
                    if (lane == 0 && lid < 0) {
                        dtouch = true;
                        if (need) dacc = __dadd_rn(dacc, __dmul_rn(as, bd));
                    }
                    if (q1 - q0 > 1) {
                        for (i64 q = q0 + lane; q < q1; q += 32) {
                            if (q == qd) continue;
                            const u32 j = P.pvcol[q];
                            atomicOr(&bits[j >> 5], 1u << (j & 31));
                            if (need) acc[j] = __dadd_rn(acc[j], __dmul_rn(as, P.pvval[q]));
                        }
                    }
                } else {
                    // a * D^-1 in FP64, carried as a float pair hi + lo (the
                    // FP64 shift keeps its precision; only stored values are
                    // FP32)
                    const double asd = __dmul_rn(a, s);
                    const float as = (float)asd;
                    const float as_lo = (float)(asd - (double)as);
                    auto add = [&](float& hi, float& lo, float b) {
                        // float-float accumulation: TwoProduct and TwoSum errors
                        // go to the error word, renormalised after each add
                        // (FastTwoSum; Dekker 1971)
                        const float p = __fmul_rn(as, b);
                        const float pe = fmaf(as, b, -p) + __fmul_rn(as_lo, b);
                        float s2, e;
                        f_two_sum(hi, p, s2, e);
                        const float c = __fadd_rn(lo, __fadd_rn(e, pe));
                        hi = __fadd_rn(s2, c);
                        lo = __fsub_rn(c, __fsub_rn(hi, s2));
                    };
                    if (lane == 0 && lid < 0) {
                        dtouch = true;
                        if (need) add(dhi, dlo, (float)bd);
                    }
                    if (q1 - q0 > 1) {
                        for (i64 q = q0 + lane; q < q1; q += 32) {
                            if (q == qd) continue;
                            const u32 j = P.pvcol[q];
                            atomicOr(&bits[j >> 5], 1u << (j & 31));
                            if (need) {
                                float2 cur = acc2[j];
                                add(cur.x, cur.y, P.pvval32[q]);
                                acc2[j] = cur;
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (lid >= 0 && lane == 0) {
            dtouch = P.long_touch[lid] != 0u;
            dacc = P.long_diag[lid];
            const float2 d2 = P.long_diag2[lid];
            dhi = d2.x;
            dlo = d2.y;
        }
        if (lane == 0 && dtouch) {
            atomicOr(&bits[i >> 5], 1u << (i & 31));
            if (F32) acc2[i] = make_float2(dhi, dlo);
            else acc[i] = dacc;
        }
        __syncwarp();
        if (F32) {   // fold (sum, err) pairs to FP64
            for (int wd = lane; wd < P.words; wd += 32)
                for (u32 m = bits[wd]; m; m &= m - 1) {
                    const u32 j = (u32)wd * 32 + (__ffs(m) - 1);
                    const float2 pr = acc2[j];
                    acc[j] = (double)pr.x + (double)pr.y;
                }
            __syncwarp();
        }
        // ---- H_VV row i: csr_add gives vv + add; untouched columns get vv
        for (i64 t = P.vvrp[i] + lane; t < P.vvrp[i + 1]; t += 32) {
            const u32 j = P.vvcol[t];
            const u32 bit = 1u << (j & 31);
            const bool was = (bits[j >> 5] & bit) != 0u;
            acc[j] = was ? __dadd_rn(P.vvval[t], acc[j]) : P.vvval[t];
            atomicOr(&bits[j >> 5], bit);
        }
        __syncwarp();
        // ---- compact in column order, keep |v| > 1e-15, clear the slab
        i64 wpos = P.capoff[i];
        u32 written = 0;
        for (int w0 = 0; w0 < P.words; w0 += 32) {
            const int wd = w0 + lane;
            const u32 word = wd < P.words ? bits[wd] : 0u;
            u32 keep = 0;
            for (u32 m = word; m; m &= m - 1) {
                const u32 j = (u32)wd * 32 + (__ffs(m) - 1);
                if (fabs(acc[j]) > 1e-15) ++keep;
            }
            u32 incl = keep;
            for (int o = 1; o < 32; o <<= 1) {
                const u32 y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const u32 total = __shfl_sync(0xffffffffu, incl, 31);
            i64 at = wpos + (incl - keep);
            for (u32 m = word; m; m &= m - 1) {
                const u32 j = (u32)wd * 32 + (__ffs(m) - 1);
                const double v = acc[j];
                if (fabs(v) > 1e-15) {
                    P.tcol[at] = j;
                    P.tval[at] = v;
                    ++at;
                }
                acc[j] = 0.0;
            }
            if (wd < P.words) bits[wd] = 0u;
            wpos += total;
            written += total;
        }
        if (lane == 0) P.rowcnt[i] = written;
        __syncwarp();
    }
}

__global__ void k_compact(const i64* capoff, const u32* tcol, const double* tval,
                          const i64* outoff, i64 nv, u32* col, double* val) {
    const int lane = threadIdx.x & 31;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = (gridDim.x * (i64)blockDim.x) >> 5;
    for (i64 i = gw; i < nv; i += nw) {
        const i64 src = capoff[i], dst = outoff[i], n = outoff[i + 1] - outoff[i];
        for (i64 t = lane; t < n; t += 32) {
            col[dst + t] = tcol[src + t];
            val[dst + t] = tval[src + t];
        }
    }
}

// Long rows.  For t in [t0, t1) of H_VP row i: the diagonal term of k =
// col[t] (H_PV[k, i] is the same stored value as H_VP[i, k], the transpose
// copies it), a flag for k's whose column holds other rows, and whether any
// k is kept.  FP64 terms are a*D^-1*a with the kernel's unfused operations.
// In FP32 mode a long row keeps its FP64 values: such a row (a reference
// determinant's, millions of entries whose terms all add to one diagonal
// element) would otherwise carry the rounding of every stored value into the
// energy (measured: 1.4e-6 Ha on 100 orbitals).  Its FP32-mode terms are the
// same FP64 products, split into (hi, lo) float pairs for the float-float
// sum.
__global__ void k_long_terms(const u32* vpcol, const double* vpval, const i64* pvrp,
                             const double* dinv, const u8* skip, i64 t0, i64 t1, bool f32,
                             double* term, float2* term2, u8* multi, u32* touch) {
    for (i64 t = t0 + blockIdx.x * (i64)blockDim.x + threadIdx.x; t < t1;
         t += (i64)gridDim.x * blockDim.x) {
        const u32 k = vpcol[t];
        const bool sk = skip[k] != 0;
        const double s = dinv[k];
        const double a = vpval[t];
        const bool need = !sk && !(a == 0.0 || s == 0.0);
        const i64 x = t - t0;
        multi[x] = (!sk && pvrp[k + 1] - pvrp[k] > 1) ? 1 : 0;
        if (!sk) atomicOr(touch, 1u);
        const double v = need ? __dmul_rn(__dmul_rn(a, s), a) : 0.0;
        if (!f32) {
            term[x] = v;
        } else {
            const float hi = (float)v;
            term2[x] = make_float2(hi, (float)(v - (double)hi));
        }
    }
}

// FP64: the terms summed in k order by one thread (the order of the
// reference's accumulation, so the result is bit-identical).  The block
// stages chunks of the terms in shared memory so the summing thread reads
// them at shared-memory latency.
constexpr int kSumChunk = 4096;
__global__ void __launch_bounds__(1024) k_long_sum64(const double* term, i64 n, double* out) {
    __shared__ double sh[kSumChunk];
    double acc = 0.0;
    for (i64 c0 = 0; c0 < n; c0 += kSumChunk) {
        const int m = (int)min((i64)kSumChunk, n - c0);
        for (int t = threadIdx.x; t < m; t += blockDim.x) sh[t] = term[c0 + t];
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (; t + 8 <= m; t += 8) {
#pragma unroll
                for (int q = 0; q < 8; ++q) acc = __dadd_rn(acc, sh[t + q]);
            }
            for (; t < m; ++t) acc = __dadd_rn(acc, sh[t]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = acc;
}

// FP32: float-float sums over a fixed tree: kSum32Blocks x 256 threads each
// sum a strided share of the terms, the block merges its threads in order,
// and k_long_merge32 merges the blocks in order.  The tree does not depend
// on the GPU, so the result is deterministic; accurate to a few FP32 ulps
// squared.
constexpr int kSum32Blocks = 256;

struct FF {
    float hi = 0.0f, lo = 0.0f;
    __device__ __forceinline__ void add(float p, float pe) {
        float s2, e;
        f_two_sum(hi, p, s2, e);
        const float c = __fadd_rn(lo, __fadd_rn(e, pe));
        hi = __fadd_rn(s2, c);
        lo = __fsub_rn(c, __fsub_rn(hi, s2));
    }
};

__global__ void __launch_bounds__(256) k_long_part32(const float2* term, i64 n, float2* part) {
    __shared__ float2 sh[256];
    FF acc;
    const i64 stride = (i64)kSum32Blocks * 256;
    for (i64 t = blockIdx.x * 256ll + threadIdx.x; t < n; t += stride) {
        const float2 v = term[t];
        acc.add(v.x, v.y);
    }
    sh[threadIdx.x] = make_float2(acc.hi, acc.lo);
    __syncthreads();
    if (threadIdx.x == 0) {
        FF b;
        for (int q = 0; q < 256; ++q) b.add(sh[q].x, sh[q].y);
        part[blockIdx.x] = make_float2(b.hi, b.lo);
    }
}

__global__ void k_long_merge32(const float2* part, float2* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        FF b;
        for (int q = 0; q < kSum32Blocks; ++q) b.add(part[q].x, part[q].y);
        *out = make_float2(b.hi, b.lo);
    }
}

// Expansion of a long row's shared columns: for each kept k (list of VP
// positions t, ascending) every H_PV entry (j != i) of column k gives one
// term; FP64 terms a*D^-1*b with the kernel's unfused operations, FP32
// terms the TwoProduct pair of the float pair of a*D^-1 (a is the long
// row's FP64 value in both modes) and the FP32 b.
__global__ void k_esc_count(const u32* list, i64 n, const u32* vpcol, const i64* pvrp, u32* cnt) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n;
         x += (i64)gridDim.x * blockDim.x) {
        const u32 k = vpcol[list[x]];
        cnt[x] = (u32)(pvrp[k + 1] - pvrp[k] - 1);
    }
}

__global__ void k_esc_fill(const u32* list, i64 n, const i64* off, u32 row, const u32* vpcol,
                           const double* vpval, const i64* pvrp,
                           const u32* pvcol, const double* pvval, const float* pvval32,
                           const double* dinv, bool f32, u32* key, double* term, float2* term2) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n;
         x += (i64)gridDim.x * blockDim.x) {
        const i64 t = list[x];
        const u32 k = vpcol[t];
        const double s = dinv[k];
        const double a = vpval[t];          // the long row's FP64 value, in both modes
        const bool need = !(a == 0.0 || s == 0.0);
        const double asd = __dmul_rn(a, s);
        const float as = (float)asd;
        const float as_lo = (float)(asd - (double)as);
        i64 w = off[x];
        for (i64 q = pvrp[k]; q < pvrp[k + 1]; ++q) {
            const u32 j = pvcol[q];
            if (j == row) continue;
            key[w] = j;
            if (!f32) {
                term[w] = need ? __dmul_rn(asd, pvval[q]) : 0.0;
            } else {
                const float b = pvval32[q];
                const float p = __fmul_rn(as, b);
                const float pe = fmaf(as, b, -p) + __fmul_rn(as_lo, b);
                term2[w] = need ? make_float2(p, pe) : make_float2(0.0f, 0.0f);
            }
            ++w;
        }
    }
}

__global__ void k_run_heads(const u32* key, i64 n, u32* flag) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        flag[t] = (t == 0 || key[t] != key[t - 1]) ? 1u : 0u;
}

// One thread per run of equal j: the run's terms (k order, by the stable
// sort) summed from 0 exactly as the kernel would sum them.
__global__ void k_run_sums(const u32* key, const u32* perm, const u32* head_pos, i64 nruns,
                           i64 n, const double* term, const float2* term2, bool f32, u32* oj,
                           double* ov, float2* ov2) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nruns;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 b = head_pos[r], e = r + 1 < nruns ? head_pos[r + 1] : n;
        oj[r] = key[b];
        if (!f32) {
            double acc = 0.0;
            for (i64 t = b; t < e; ++t) acc = __dadd_rn(acc, term[perm[t]]);
            ov[r] = acc;
        } else {
            float hi = 0.0f, lo = 0.0f;
            for (i64 t = b; t < e; ++t) {
                const float2 pp = term2[perm[t]];
                float s2, er;
                f_two_sum(hi, pp.x, s2, er);
                const float c = __fadd_rn(lo, __fadd_rn(er, pp.y));
                hi = __fadd_rn(s2, c);
                lo = __fsub_rn(c, __fsub_rn(hi, s2));
            }
            ov2[r] = make_float2(hi, lo);
        }
    }
}

__global__ void k_iota_u32(u32* p, i64 n, i64 base) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        p[t] = (u32)(base + t);
}

__global__ void k_to_f32v(const double* v, i64 n, float* o) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        o[t] = (float)v[t];
}

int gs(i64 n) {
    i64 b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 65535 ? 65535 : b));
}

template <class T>
void scan_excl(const T* in, i64* out, i64 n, cudaStream_t s) {
    prim::scan<T, i64, false>(in, out, n, s);
}

inline int bits_for(i64 n) {   // bits of the largest index below n
    int b = 1;
    while (b < 63 && ((i64)1 << b) < n) ++b;
    return b;
}

// COO (device) -> canonical CSR (sorted, duplicates summed in input order,
// exact zeros dropped).
void coo_to_csr_dev(const u32* r, const u32* c, const double* v, i64 n, i64 nr, i64 nc,
                    Csr& out, cudaStream_t s) {
    out.nr = nr;
    out.nc = nc;
    out.rowptr.alloc(nr + 1, s);
    DBuf<u32> rowcnt(nr + 1, s);
    DNQ_CUDA(cudaMemsetAsync(rowcnt.p, 0, (nr + 1) * 4, s));
    if (n == 0) {
        out.nnz = 0;
        scan_excl(rowcnt.p, out.rowptr.p, nr + 1, s);
        return;
    }
    require(n < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "COO input has more than 2^32 entries");
    DBuf<u64> key(n, s), skey(n, s), rkey(n, s);
    DBuf<u32> idx(n, s), perm(n, s), flag(n, s), runid(n, s);
    DBuf<unsigned long long> bad(1, s);
    DNQ_CUDA(cudaMemsetAsync(bad.p, 0, 8, s));
    k_coo_keys<<<gs(n), 256, 0, s>>>(r, c, n, key.p, idx.p, bad.p, nr, nc);
    DNQ_CHECK_LAUNCH();
    unsigned long long hb = 0;
    DNQ_CUDA(cudaMemcpyAsync(&hb, bad.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    require(hb == 0, DNQ_ERR_RANGE, "coo_to_csr: row index out of bounds");
    {   // (row << 32 | col): stable, so duplicates keep their input order
        const int bits[1] = {32 + bits_for(nr)};
        prim::radix_sort<u64, u32>(key.p, skey.p, idx.p, perm.p, n, bits, s);
    }
    k_run_flags<<<gs(n), 256, 0, s>>>(skey.p, n, flag.p);
    DNQ_CHECK_LAUNCH();
    prim::scan_inclusive<u32, u32>(flag.p, runid.p, n, s);
    u32 nruns = 0;
    DNQ_CUDA(cudaMemcpyAsync(&nruns, runid.p + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    DBuf<double> rsum(nruns, s);
    k_run_sum<<<gs(n), 256, 0, s>>>(skey.p, perm.p, v, runid.p, n, rsum.p, rkey.p);
    DNQ_CHECK_LAUNCH();
    DBuf<u32> keep(nruns, s);
    k_nonzero<<<gs(nruns), 256, 0, s>>>(rsum.p, nruns, keep.p);
    DNQ_CHECK_LAUNCH();
    DBuf<u32> pos32(nruns, s);
    prim::scan<u32, u32, false>(keep.p, pos32.p, (i64)nruns, s);   // n < 2^32
    u32 lastpos = 0, lastkeep = 0;
    DNQ_CUDA(cudaMemcpyAsync(&lastpos, pos32.p + nruns - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(&lastkeep, keep.p + nruns - 1, 4, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    out.nnz = (i64)lastpos + lastkeep;
    out.col.alloc(out.nnz, s);
    out.val.alloc(out.nnz, s);
    k_scatter_csr<<<gs(nruns), 256, 0, s>>>(rkey.p, rsum.p, keep.p, pos32.p, nruns, out.col.p,
                                            out.val.p, rowcnt.p);
    DNQ_CHECK_LAUNCH();
    scan_excl(rowcnt.p, out.rowptr.p, nr + 1, s);
}

}  // namespace

// Core of the downfolding on canonical CSR blocks (VV: nv x nv, VP: nv x np).
void ham_eff_csr(const Csr& VV, const Csr& VP, i64 nv, i64 np, const double* hpp, double e_ref,
                 int sigma, double eps, int precision, int device, cudaStream_t s,
                 dnq_ham_s* H) {
    H->device = device;
    H->stream = s;
    H->n_v = nv;
    Csr PV;
    transpose_csr(VP, PV, s);
    DBuf<double> dinv(np, s);
    DBuf<u8> skip(np, s);
    k_dinv<<<gs(np), 256, 0, s>>>(hpp, np, e_ref, eps, sigma, dinv.p);
    DNQ_CHECK_LAUNCH();
    k_screen<<<gs(np), 256, 0, s>>>(PV.rowptr.p, PV.val.p, np, dinv.p, skip.p);
    DNQ_CHECK_LAUNCH();
    DBuf<i64> cap(nv + 1, s), capoff(nv + 1, s);
    DNQ_CUDA(cudaMemsetAsync(cap.p + nv, 0, 8, s));
    {
        DBuf<i64> len(std::max<i64>(1, VP.nnz), s), rsum(nv, s);
        if (VP.nnz) {
            k_cap_terms<<<gs(VP.nnz), 256, 0, s>>>(VP.col.p, VP.nnz, PV.rowptr.p, skip.p, len.p);
            DNQ_CHECK_LAUNCH();
        }
        if (nv) {
            prim::segment_sums<i64, i64>(len.p, VP.rowptr.p, nv, rsum.p, s);
        }
        k_cap_finish<<<gs(nv), 256, 0, s>>>(rsum.p, VV.rowptr.p, nv, cap.p);
        DNQ_CHECK_LAUNCH();
    }
    scan_excl(cap.p, capoff.p, nv + 1, s);
    i64 captot = 0;
    DNQ_CUDA(cudaMemcpyAsync(&captot, capoff.p + nv, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));

    HeffParams P{};
    P.nv = nv;
    P.vprp = VP.rowptr.p; P.vpcol = VP.col.p; P.vpval = VP.val.p;
    P.pvrp = PV.rowptr.p; P.pvcol = PV.col.p; P.pvval = PV.val.p;
    P.vvrp = VV.rowptr.p; P.vvcol = VV.col.p; P.vvval = VV.val.p;
    P.dinv = dinv.p;
    P.skip = skip.p;
    P.capoff = capoff.p;
    DBuf<u32> tcol(captot, s), rowcnt(nv + 1, s);
    DBuf<double> tval(captot, s);
    DNQ_CUDA(cudaMemsetAsync(rowcnt.p + nv, 0, 4, s));
    P.tcol = tcol.p;
    P.tval = tval.p;
    P.rowcnt = rowcnt.p;
    DBuf<int> next(1, s);
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    P.next_row = next.p;
    P.words = (int)((nv + 31) / 32);
    DBuf<float> vp32, pv32;
    if (precision == DNQ_F32) {
        vp32.alloc(VP.nnz, s);
        pv32.alloc(PV.nnz, s);
        if (VP.nnz) k_to_f32v<<<gs(VP.nnz), 256, 0, s>>>(VP.val.p, VP.nnz, vp32.p);
        DNQ_CHECK_LAUNCH();
        if (PV.nnz) k_to_f32v<<<gs(PV.nnz), 256, 0, s>>>(PV.val.p, PV.nnz, pv32.p);
        DNQ_CHECK_LAUNCH();
        P.vpval32 = vp32.p;
        P.pvval32 = pv32.p;
    }
    // ---- rows with very many H_VP entries
    constexpr i64 kLong = 1 << 16;
    std::vector<i64> vrp(nv + 1);
    DNQ_CUDA(cudaMemcpyAsync(vrp.data(), VP.rowptr.p, (nv + 1) * 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    std::vector<i64> longs;
    for (i64 r = 0; r < nv; ++r)
        if (vrp[r + 1] - vrp[r] > kLong) longs.push_back(r);
    const int nl = (int)longs.size();
    DBuf<int> lid;
    DBuf<i64> loff;
    DBuf<u32> lj, ltouch;
    DBuf<double> ldiag, lv;
    DBuf<float2> ldiag2, lv2;
    if (nl) {
        std::vector<int> hid(nv, -1);
        for (int q = 0; q < nl; ++q) hid[longs[q]] = q;
        lid.alloc(nv, s);
        DNQ_CUDA(cudaMemcpyAsync(lid.p, hid.data(), 4 * nv, cudaMemcpyHostToDevice, s));
        ldiag.alloc(nl, s);
        ldiag2.alloc(nl, s);
        ltouch.alloc(nl, s);
        DNQ_CUDA(cudaMemsetAsync(ltouch.p, 0, 4 * nl, s));
        DNQ_CUDA(cudaMemsetAsync(ldiag.p, 0, 8 * nl, s));
        DNQ_CUDA(cudaMemsetAsync(ldiag2.p, 0, 8 * nl, s));
        std::vector<i64> hoff(nl + 1, 0);
        std::vector<DBuf<u32>> pj(nl);
        std::vector<DBuf<double>> pv(nl);
        std::vector<DBuf<float2>> pv2(nl);
        for (int q = 0; q < nl; ++q) {
            const i64 t0 = vrp[longs[q]], t1 = vrp[longs[q] + 1], m = t1 - t0;
            DBuf<double> term;
            DBuf<float2> term2;
            if (precision == DNQ_F32) term2.alloc(m, s);
            else term.alloc(m, s);
            DBuf<u8> multi(m, s);
            k_long_terms<<<gs(m), 256, 0, s>>>(VP.col.p, VP.val.p, PV.rowptr.p, dinv.p,
                                               skip.p, t0, t1, precision == DNQ_F32, term.p,
                                               term2.p, multi.p, ltouch.p + q);
            DNQ_CHECK_LAUNCH();
            if (precision == DNQ_F32) {
                DBuf<float2> part(kSum32Blocks, s);
                k_long_part32<<<kSum32Blocks, 256, 0, s>>>(term2.p, m, part.p);
                DNQ_CHECK_LAUNCH();
                k_long_merge32<<<1, 32, 0, s>>>(part.p, ldiag2.p + q);
            } else {
                k_long_sum64<<<1, 1024, 0, s>>>(term.p, m, ldiag.p + q);
            }
            DNQ_CHECK_LAUNCH();
            // kept k's whose column holds other rows, in order
            DBuf<u32> idx(m, s), sel(m, s);
            k_iota_u32<<<gs(m), 256, 0, s>>>(idx.p, m, t0);
            DNQ_CHECK_LAUNCH();
            const i64 ns = prim::select_flagged<u32, u8>(idx.p, multi.p, sel.p, m, s);
            // expand (j, term), stable sort by j, ordered sum per j
            i64 ne = 0;
            DBuf<u32> ecnt(ns + 1, s);
            DBuf<i64> eoff(ns + 1, s);
            DNQ_CUDA(cudaMemsetAsync(ecnt.p + ns, 0, 4, s));
            if (ns) {
                k_esc_count<<<gs(ns), 256, 0, s>>>(sel.p, ns, VP.col.p, PV.rowptr.p, ecnt.p);
                DNQ_CHECK_LAUNCH();
            }
            scan_excl(ecnt.p, eoff.p, ns + 1, s);
            DNQ_CUDA(cudaMemcpyAsync(&ne, eoff.p + ns, 8, cudaMemcpyDeviceToHost, s));
            DNQ_CUDA(cudaStreamSynchronize(s));
            require(ne < (i64)0xffffffffll, DNQ_ERR_OVERFLOW, "long-row expansion exceeds 2^32");
            DBuf<u32> ekey(std::max<i64>(1, ne), s), skey(std::max<i64>(1, ne), s);
            DBuf<u32> sperm(std::max<i64>(1, ne), s);
            DBuf<double> eterm;
            DBuf<float2> eterm2;
            if (precision == DNQ_F32) eterm2.alloc(std::max<i64>(1, ne), s);
            else eterm.alloc(std::max<i64>(1, ne), s);
            i64 nruns = 0;
            if (ne) {
                k_esc_fill<<<gs(ns), 256, 0, s>>>(sel.p, ns, eoff.p, (u32)longs[q], VP.col.p,
                                                  VP.val.p, PV.rowptr.p, PV.col.p,
                                                  PV.val.p, P.pvval32, dinv.p,
                                                  precision == DNQ_F32, ekey.p, eterm.p,
                                                  eterm2.p);
                DNQ_CHECK_LAUNCH();
                {   // stable by j: a run keeps its terms in k order
                    const int bits[1] = {bits_for(nv)};
                    prim::radix_sort<u32, u32>(ekey.p, skey.p, nullptr, sperm.p, ne, bits, s);
                }
                DBuf<u32> head(ne, s), hpos(ne, s);
                k_run_heads<<<gs(ne), 256, 0, s>>>(skey.p, ne, head.p);
                DNQ_CHECK_LAUNCH();
                DBuf<u32> pos(ne, s);
                k_iota_u32<<<gs(ne), 256, 0, s>>>(pos.p, ne, 0);
                DNQ_CHECK_LAUNCH();
                nruns = prim::select_flagged<u32, u32>(pos.p, head.p, hpos.p, ne, s);
                DBuf<u32> oj(nruns, s);
                DBuf<double> ov;
                DBuf<float2> ov2;
                if (precision == DNQ_F32) ov2.alloc(nruns, s);
                else ov.alloc(nruns, s);
                k_run_sums<<<gs(nruns), 256, 0, s>>>(skey.p, sperm.p, hpos.p, nruns, ne, eterm.p,
                                                     eterm2.p, precision == DNQ_F32, oj.p, ov.p,
                                                     ov2.p);
                DNQ_CHECK_LAUNCH();
                pj[q] = std::move(oj);
                pv[q] = std::move(ov);
                pv2[q] = std::move(ov2);
            }
            hoff[q + 1] = hoff[q] + nruns;
        }
        const i64 ntot = std::max<i64>(1, hoff[nl]);
        lj.alloc(ntot, s);
        if (precision == DNQ_F32) lv2.alloc(ntot, s);
        else lv.alloc(ntot, s);
        for (int q = 0; q < nl; ++q) {
            const i64 m = hoff[q + 1] - hoff[q];
            if (!m) continue;
            DNQ_CUDA(cudaMemcpyAsync(lj.p + hoff[q], pj[q].p, 4 * m, cudaMemcpyDeviceToDevice, s));
            if (precision == DNQ_F32)
                DNQ_CUDA(cudaMemcpyAsync(lv2.p + hoff[q], pv2[q].p, 8 * m,
                                         cudaMemcpyDeviceToDevice, s));
            else
                DNQ_CUDA(cudaMemcpyAsync(lv.p + hoff[q], pv[q].p, 8 * m,
                                         cudaMemcpyDeviceToDevice, s));
        }
        loff.alloc(nl + 1, s);
        DNQ_CUDA(cudaMemcpyAsync(loff.p, hoff.data(), 8 * (nl + 1), cudaMemcpyHostToDevice, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
        P.long_id = lid.p;
        P.long_off = loff.p;
        P.long_j = lj.p;
        P.long_v = lv.p;
        P.long_v2 = lv2.p;
        P.long_diag = ldiag.p;
        P.long_diag2 = ldiag2.p;
        P.long_touch = ltouch.p;
    }
    const size_t per_warp = (((size_t)P.words * 4 + 15) & ~(size_t)15) + (size_t)nv * 8;
    const bool smem = per_warp * kHW <= 200 * 1024;
    const int sms = sm_count(device);
    DBuf<double> gacc;
    DBuf<u32> gbits;
    int grid;
    if (smem) {
        const size_t sm_bytes = per_warp * kHW;
        auto kern = precision == DNQ_F32 ? k_heff<true, true> : k_heff<false, true>;
        DNQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sm_bytes));
        int per_sm = 0;
        DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kHW * 32, sm_bytes));
        grid = std::max(1, per_sm) * sms;
        kern<<<grid, kHW * 32, sm_bytes, s>>>(P);
        DNQ_CHECK_LAUNCH();
    } else {
        grid = sms * 2;
        const i64 nw = (i64)grid * kHW;
        gacc.alloc((size_t)nw * nv, s);
        gbits.alloc((size_t)nw * P.words, s);
        DNQ_CUDA(cudaMemsetAsync(gacc.p, 0, gacc.bytes(), s));
        DNQ_CUDA(cudaMemsetAsync(gbits.p, 0, gbits.bytes(), s));
        P.gacc = gacc.p;
        P.gbits = gbits.p;
        auto kern = precision == DNQ_F32 ? k_heff<true, false> : k_heff<false, false>;
        kern<<<grid, kHW * 32, 0, s>>>(P);
        DNQ_CHECK_LAUNCH();
    }
    DNQ_CHECK_LAUNCH();
    H->vv.nr = nv;
    H->vv.nc = nv;
    H->vv.rowptr.alloc(nv + 1, s);
    scan_excl(rowcnt.p, H->vv.rowptr.p, nv + 1, s);
    DNQ_CUDA(cudaMemcpyAsync(&H->vv.nnz, H->vv.rowptr.p + nv, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    H->vv.col.alloc(H->vv.nnz, s);
    H->vv.val.alloc(H->vv.nnz, s);
    k_compact<<<sms * 4, 256, 0, s>>>(capoff.p, tcol.p, tval.p, H->vv.rowptr.p, nv, H->vv.col.p,
                                      H->vv.val.p);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaStreamSynchronize(s));
}

void ham_eff(const u32* vvr, const u32* vvc, const double* vvv, i64 vvn, i64 nv,
             const u32* vpr, const u32* vpc, const double* vpv, i64 vpn, i64 np,
             const double* hpp, double e_ref, int sigma, double eps, int precision,
             int device, cudaStream_t s, dnq_ham_s* H) {
    H->device = device;
    H->stream = s;
    H->n_v = nv;
    Csr VV, VP;
    coo_to_csr_dev(vvr, vvc, vvv, vvn, nv, nv, VV, s);
    if (np == 0) {   // ham_eff.cpp:72-77: H_VV canonicalised
        H->vv = std::move(VV);
        DNQ_CUDA(cudaStreamSynchronize(s));
        return;
    }
    coo_to_csr_dev(vpr, vpc, vpv, vpn, nv, np, VP, s);
    ham_eff_csr(VV, VP, nv, np, hpp, e_ref, sigma, eps, precision, device, s, H);
}

}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_ham_eff_from(dnq_ham_t proxy, const double* h_pp, double e_ref, int reg_sigma,
                     double epsilon, int precision, void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require(proxy && out, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    require(proxy->n_p == 0 || h_pp, DNQ_ERR_INVALID, "null h_pp_diag");
    DeviceGuard g(proxy->device);
    cudaStream_t s = (cudaStream_t)stream;
    ensure_compact(proxy->vv, s);
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    if (proxy->n_p == 0 || proxy->vp.nnz == 0 && proxy->n_p == 0) {
        // empty P: H_eff is H_VV itself
        Csr copy;
        copy.nr = copy.nc = proxy->n_v;
        copy.nnz = proxy->vv.nnz;
        copy.rowptr.alloc(proxy->n_v + 1, s);
        copy.col.alloc(copy.nnz, s);
        copy.val.alloc(copy.nnz, s);
        DNQ_CUDA(cudaMemcpyAsync(copy.rowptr.p, proxy->vv.rowptr.p, (proxy->n_v + 1) * 8,
                                 cudaMemcpyDeviceToDevice, s));
        if (copy.nnz) {
            DNQ_CUDA(cudaMemcpyAsync(copy.col.p, proxy->vv.col.p, copy.nnz * 4,
                                     cudaMemcpyDeviceToDevice, s));
            DNQ_CUDA(cudaMemcpyAsync(copy.val.p, proxy->vv.val.p, copy.nnz * 8,
                                     cudaMemcpyDeviceToDevice, s));
        }
        H->device = proxy->device;
        H->stream = s;
        H->n_v = proxy->n_v;
        H->vv = std::move(copy);
        DNQ_CUDA(cudaStreamSynchronize(s));
    } else {
        DIn<double> hpp(h_pp, proxy->n_p, s);
        ham_eff_csr(proxy->vv, proxy->vp, proxy->n_v, proxy->n_p, hpp.p, e_ref, reg_sigma,
                    epsilon, precision, proxy->device, s, H.get());
    }
    *out = H.release();
    DNQ_API_END
}

int dnq_ham_eff(const uint32_t* vv_rows, const uint32_t* vv_cols, const double* vv_vals,
                int64_t vv_nnz, int64_t n_v, const uint32_t* vp_rows, const uint32_t* vp_cols,
                const double* vp_vals, int64_t vp_nnz, int64_t n_p, const double* h_pp,
                double e_ref, int reg_sigma, double epsilon, int precision, int device,
                void* stream, dnq_ham_t* out) {
    DNQ_API_BEGIN
    require(out != nullptr, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(vv_nnz >= 0 && vp_nnz >= 0 && n_v >= 0 && n_p >= 0, DNQ_ERR_INVALID, "negative size");
    require(n_v <= (int64_t)0xffffffffll && n_p <= (int64_t)0xffffffffll, DNQ_ERR_OVERFLOW,
            "dimension exceeds u32 index capacity");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    require(vv_nnz == 0 || (vv_rows && vv_cols && vv_vals), DNQ_ERR_INVALID, "null H_VV array");
    require(vp_nnz == 0 || (vp_rows && vp_cols && vp_vals), DNQ_ERR_INVALID, "null H_VP array");
    require(n_p == 0 || h_pp, DNQ_ERR_INVALID, "null h_pp_diag");
    DeviceGuard g(device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u32> vr(vv_rows, vv_nnz, s), vc(vv_cols, vv_nnz, s), pr(vp_rows, vp_nnz, s),
        pc(vp_cols, vp_nnz, s);
    DIn<double> vvv(vv_vals, vv_nnz, s), vpv(vp_vals, vp_nnz, s), hpp(h_pp, n_p, s);
    std::unique_ptr<dnq_ham_s> H(new dnq_ham_s);
    ham_eff(vr.p, vc.p, vvv.p, vv_nnz, n_v, pr.p, pc.p, vpv.p, vp_nnz, n_p, hpp.p, e_ref,
            reg_sigma, epsilon, precision, device, s, H.get());
    *out = H.release();
    DNQ_API_END
}

}  // extern "C"
