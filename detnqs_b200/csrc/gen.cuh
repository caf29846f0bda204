// gen.cuh -- warp-per-determinant enumeration of connected determinants.
//
// One warp owns one bra row.  It walks the candidates in the reference's
// order -- singles alpha then beta, holes ascending outer and particles
// ascending inner (det_ops.hpp:123-159), then heat-bath doubles over the
// occupied spin-orbital pairs (p > q in the alpha-then-beta occupied list)
// with each pair's table prefix (ham_utils.hpp:280-313) -- 32 candidates per
// step, one per lane.  Every lane forms its ket with bit operations, the
// fermionic phase with popcounts (Scemama-Giner rules, det_ops.cpp:85-196)
// and the matrix element:
//   single h->p : h1[h,p] + sum over the other occupied orbitals of the
//                 precomputed same/opposite-spin terms, in the reference's
//                 summation order (ham_eval.cpp:88-115);
//   double      : +-v from the signed pair table (no ERI reads).
// A sink object (routing, screening, output) sees each step collectively,
// so it can compact survivors with __ballot_sync in candidate order.
#pragma once

#include "context.cuh"
#include "detmap.cuh"

namespace dnq {

// Per-warp occupancy lists, in shared memory.
struct WarpRow {
    u64 a, b;                 // bra alpha / beta masks
    int na, nb, nva, nvb, ne;
    u8 occ[128];              // spin-orbitals: 2p (alpha asc) then 2p+1 (beta asc)
    u8 occa[64], occb[64], vira[64], virb[64];
};

__device__ __forceinline__ void load_row(WarpRow& R, u64 a, u64 b, int n_orb) {
    const int lane = threadIdx.x & 31;
    const u64 all = low_mask(n_orb);
    if (lane == 0) {
        R.a = a;
        R.b = b;
        int k = 0, t;
        t = 0;
        for (u64 x = a; x; x &= x - 1) { const int o = __ffsll(x) - 1; R.occa[t++] = o; R.occ[k++] = 2 * o; }
        R.na = t;
        t = 0;
        for (u64 x = b; x; x &= x - 1) { const int o = __ffsll(x) - 1; R.occb[t++] = o; R.occ[k++] = 2 * o + 1; }
        R.nb = t;
        R.ne = k;
        t = 0;
        for (u64 x = ~a & all; x; x &= x - 1) R.vira[t++] = __ffsll(x) - 1;
        R.nva = t;
        t = 0;
        for (u64 x = ~b & all; x; x &= x - 1) R.virb[t++] = __ffsll(x) - 1;
        R.nvb = t;
    }
    __syncwarp();
}

// <bra|H|bra> with the reference's order: one-body over alpha then beta
// occupied orbitals, then sum_{x>y} <occ_x occ_y||occ_x occ_y>
// (ham_eval.cpp:53-86).  Serial per thread so the rounding matches.
__device__ __forceinline__ double diag_elem(const CtxView& C, u64 a, u64 b) {
    const int n = C.n;
    u8 occ[128];
    int m = 0;
    for (u64 x = a; x; x &= x - 1) occ[m++] = (u8)(2 * (__ffsll(x) - 1));
    for (u64 x = b; x; x &= x - 1) occ[m++] = (u8)(2 * (__ffsll(x) - 1) + 1);
    double one = 0.0;
    for (int t = 0; t < m; ++t) {
        const int p = occ[t] >> 1;
        one += C.h1[p * n + p];
    }
    double two = 0.0;
    for (int x = 1; x < m; ++x) {
        const int P = occ[x];
        const double* dss = C.dss + (P >> 1) * n;
        const double* dos = C.dos + (P >> 1) * n;
        for (int y = 0; y < x; ++y) {
            const int Q = occ[y];
            two += ((P ^ Q) & 1) ? dos[Q >> 1] : dss[Q >> 1];
        }
    }
    return one + two;
}

// Single excitation h -> p in spin `s` of the bra (a, b); returns the signed
// element <bra|H|ket>.
__device__ __forceinline__ double single_elem(const CtxView& C, u64 a, u64 b, int s, int h,
                                              int p) {
    const int n = C.n;
    double e = C.h1[h * n + p];
    const size_t base = ((size_t)h * n + p) * n;
    const double* ss = C.sss + base;
    const double* os = C.sos + base;
    if (s == 0) {
        for (u64 x = a & ~(1ull << h); x; x &= x - 1) e += ss[__ffsll(x) - 1];
        for (u64 x = b; x; x &= x - 1) e += os[__ffsll(x) - 1];
    } else {
        for (u64 x = a; x; x &= x - 1) e += os[__ffsll(x) - 1];
        for (u64 x = b & ~(1ull << h); x; x &= x - 1) e += ss[__ffsll(x) - 1];
    }
    const int perm = occ_between(s ? b : a, h, p);
    return (perm & 1) ? -e : e;
}

// Double i,j -> a,b (spin-orbitals, i > j, a > b) of the bra from the
// signed table value v = <ij||ab>.
__device__ __forceinline__ double double_elem(u64 ba, u64 bb, int i, int j, int a, int b,
                                              double v) {
    const bool same = ((i ^ j) & 1) == 0;
    double raw = (same || ((a ^ i) & 1) == 0) ? v : -v;
    int perm;
    if (same) {
        const u64 occ = (i & 1) ? bb : ba;
        const int h0 = b >> 1, h1 = a >> 1;     // ket-only orbitals, ascending
        const int p0 = j >> 1, p1 = i >> 1;     // bra-only orbitals, ascending
        perm = occ_between(occ, h0, p0) + occ_between(occ, h1, p1);
        const int A = min(h0, p0), B = max(h0, p0), Cc = min(h1, p1), D = max(h1, p1);
        if ((Cc > A && Cc < B && D > B) || (A > Cc && A < D && B > D)) ++perm;
    } else {
        const int ha = ((a & 1) == 0 ? a : b) >> 1;
        const int hb = ((a & 1) == 1 ? a : b) >> 1;
        const int pa = ((i & 1) == 0 ? i : j) >> 1;
        const int pb = ((i & 1) == 1 ? i : j) >> 1;
        perm = occ_between(ba, ha, pa) + occ_between(bb, hb, pb);
    }
    return (perm & 1) ? -raw : raw;
}

// Length of the prefix of a table row whose weights are >= cut
// (HeatBathTable::RowView::with_cutoff, hb_table.hpp:131-146), found by the
// warp with 32-way probing; cut <= 0 keeps the whole row.
__device__ __forceinline__ i64 warp_prefix(const double* v, i64 len, double cut) {
    if (cut <= 0.0 || len == 0) return len;
    const int lane = threadIdx.x & 31;
    i64 lo = 0, hi = len;   // answer in [lo, hi]
    while (hi - lo > 32) {
        const i64 step = (hi - lo + 31) / 32;
        const i64 x = lo + lane * step;
        const bool ok = x < hi && fabs(v[x]) >= cut;
        const int k = __popc(__ballot_sync(0xffffffffu, ok));
        if (k == 0) return lo;
        const i64 nlo = lo + (i64)(k - 1) * step + 1;
        const i64 nhi = min(hi, lo + (i64)k * step);
        lo = nlo;
        hi = nhi;
    }
    const i64 x = lo + lane;
    const bool ok = x < hi && fabs(v[x]) >= cut;
    return lo + __popc(__ballot_sync(0xffffffffu, ok));
}

// Candidate handed to a sink (per lane).
struct Cand {
    bool valid;
    bool single;
    u64 a, b;       // ket
    double h;       // <bra|H|ket>
};

// Walk all candidates of the bra in R.  `plen` (optional) holds the prefix
// length of every table row for a cut shared by all rows; otherwise the
// prefix is searched with `cut`.  Sink::step(const Cand&) is called by all
// 32 lanes together.
// Singles of the bra in R: alpha then beta, holes ascending outer and
// particles ascending inner (det_ops.hpp:123-159, :248-253).
template <class Sink>
__device__ __forceinline__ void enumerate_singles(const CtxView& C, const WarpRow& R,
                                                  Sink& sink) {
    const int lane = threadIdx.x & 31;
    const int nsa = R.na * R.nva;
    const int nst = nsa + R.nb * R.nvb;
    for (int t0 = 0; t0 < nst; t0 += 32) {
        Cand c;
        const int t = t0 + lane;
        c.valid = t < nst;
        c.single = true;
        c.a = R.a;
        c.b = R.b;
        c.h = 0.0;
        if (c.valid) {
            int s, h, p;
            if (t < nsa) {
                s = 0;
                h = R.occa[t / R.nva];
                p = R.vira[t % R.nva];
                c.a = R.a ^ (1ull << h) ^ (1ull << p);
            } else {
                const int u = t - nsa;
                s = 1;
                h = R.occb[u / R.nvb];
                p = R.virb[u % R.nvb];
                c.b = R.b ^ (1ull << h) ^ (1ull << p);
            }
            c.h = single_elem(C, R.a, R.b, s, h, p);
        }
        sink.step(c);
    }
}

template <class Sink>
__device__ __forceinline__ void enumerate_row(const CtxView& C, const WarpRow& R,
                                              const i64* plen, double cut, Sink& sink) {
    const int lane = threadIdx.x & 31;
    enumerate_singles(C, R, sink);
    // ---- doubles
    for (int x = 1; x < R.ne; ++x) {
        const int i = R.occ[x];
        for (int y = 0; y < x; ++y) {
            const int j = R.occ[y];
            const i64 row = pair_row(i, j);
            const i64 lo = __ldg(&C.tab.off[row]);
            i64 len;
            if (plen) len = __ldg(&plen[row]);
            else len = warp_prefix(C.tab.v + lo, __ldg(&C.tab.off[row + 1]) - lo, cut);
            const int ii = max(i, j), jj = min(i, j);
            for (i64 e0 = 0; e0 < len; e0 += 32) {
                Cand c;
                const i64 e = e0 + lane;
                c.valid = e < len;
                c.single = false;
                c.a = R.a;
                c.b = R.b;
                c.h = 0.0;
                if (c.valid) {
                    const u16 ab = __ldg(&C.tab.ab[lo + e]);
                    const int A = ab & 0xff, B = ab >> 8;
                    const u64 ma = 1ull << (A >> 1), mb = 1ull << (B >> 1);
                    const bool occA = ((A & 1) ? R.b : R.a) & ma;
                    const bool occB = ((B & 1) ? R.b : R.a) & mb;
                    if (occA || occB) {
                        c.valid = false;
                    } else {
                        u64 ka = R.a, kb = R.b;
                        if (ii & 1) kb &= ~(1ull << (ii >> 1)); else ka &= ~(1ull << (ii >> 1));
                        if (jj & 1) kb &= ~(1ull << (jj >> 1)); else ka &= ~(1ull << (jj >> 1));
                        if (A & 1) kb |= ma; else ka |= ma;
                        if (B & 1) kb |= mb; else ka |= mb;
                        c.a = ka;
                        c.b = kb;
                        c.h = double_elem(R.a, R.b, ii, jj, A, B, __ldg(&C.tab.v[lo + e]));
                    }
                }
                sink.step(c);
            }
        }
    }
}

// All candidates of the bra in the order get_local_conn visits them without
// heat-bath screening (local_conn.cpp:69-91): the singles, then every double
// in det_ops::for_each_double's order -- alpha-alpha (hole pairs h1 < h2
// outer, particle pairs p1 < p2 inner; det_ops.hpp:161-187), beta-beta
// (:189-215), alpha-beta (alpha hole, alpha particle, beta hole, beta
// particle; :217-246).  A double's element comes from the ERIs through the
// same antisymmetrised value the pair table stores, so it has the same bits
// as on the table walk.
template <class Sink>
__device__ __forceinline__ void enumerate_row_full(const CtxView& C, const WarpRow& R,
                                                   Sink& sink) {
    const int lane = threadIdx.x & 31;
    enumerate_singles(C, R, sink);
    for (int s = 0; s < 2; ++s) {
        const u8* occ = s ? R.occb : R.occa;
        const u8* vir = s ? R.virb : R.vira;
        const int no = s ? R.nb : R.na, nv = s ? R.nvb : R.nva;
        if (no < 2 || nv < 2) continue;
        const int npv = nv * (nv - 1) / 2;
        for (int x1 = 0; x1 < no; ++x1)
            for (int x2 = x1 + 1; x2 < no; ++x2) {
                const int h1 = occ[x1], h2 = occ[x2];
                for (int t0 = 0; t0 < npv; t0 += 32) {
                    Cand c;
                    const int t = t0 + lane;
                    c.valid = t < npv;
                    c.single = false;
                    c.a = R.a;
                    c.b = R.b;
                    c.h = 0.0;
                    if (c.valid) {
                        int y1 = 0, rem = t;          // t-th pair y1 < y2, lexicographic
                        while (rem >= nv - 1 - y1) { rem -= nv - 1 - y1; ++y1; }
                        const int p1 = vir[y1], p2 = vir[y1 + 1 + rem];
                        const u64 m = (1ull << h1) | (1ull << h2) | (1ull << p1) | (1ull << p2);
                        if (s) c.b ^= m; else c.a ^= m;
                        const int i = 2 * h2 + s, j = 2 * h1 + s, A = 2 * p2 + s, B = 2 * p1 + s;
                        c.h = double_elem(R.a, R.b, i, j, A, B, anti_so_of(C.eri, i, j, A, B));
                    }
                    sink.step(c);
                }
            }
    }
    if (!R.na || !R.nva || !R.nb || !R.nvb) return;
    const int nsb = R.nb * R.nvb;
    for (int xa = 0; xa < R.na; ++xa)
        for (int ya = 0; ya < R.nva; ++ya) {
            const int ha = R.occa[xa], pa = R.vira[ya];
            const u64 ka = R.a ^ (1ull << ha) ^ (1ull << pa);
            for (int t0 = 0; t0 < nsb; t0 += 32) {
                Cand c;
                const int t = t0 + lane;
                c.valid = t < nsb;
                c.single = false;
                c.a = ka;
                c.b = R.b;
                c.h = 0.0;
                if (c.valid) {
                    const int hb = R.occb[t / R.nvb], pb = R.virb[t % R.nvb];
                    c.b = R.b ^ (1ull << hb) ^ (1ull << pb);
                    const int sa = 2 * ha, sb = 2 * hb + 1, ta = 2 * pa, tb = 2 * pb + 1;
                    const int i = max(sa, sb), j = min(sa, sb), A = max(ta, tb), B = min(ta, tb);
                    c.h = double_elem(R.a, R.b, i, j, A, B, anti_so_of(C.eri, i, j, A, B));
                }
                sink.step(c);
            }
        }
}

}  // namespace dnq
