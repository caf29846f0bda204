// context.cuh -- integral context resident in HBM.
//
// The reference keeps packed MO integrals (integral_mo.hpp:30-49) behind a
// spin-orbital view (integral_so.hpp:77-108) and evaluates every term of a
// matrix element on the fly.  Here the context holds, per system:
//
//   h1   [n*n]     dense one-electron integrals
//   dss  [n*n]     (pp|qq) - (pq|qp)    same-spin diagonal pair term
//   dos  [n*n]     (pp|qq)              opposite-spin diagonal pair term
//   sss  [n*n*n]   (hp|kk) - (hk|kp)    same-spin term of a single h->p
//   sos  [n*n*n]   (hp|kk)              opposite-spin term of a single h->p
//   pair table     for every occupied spin-orbital pair {i>j}: entries
//                  (a>b, v = <ij||ab>) sorted by |v| descending
//
// Each stored value is the result of the same IEEE operation the reference
// performs at run time (a table lookup or one subtraction), so sums formed
// in the reference's order reproduce its elements bit for bit.  The pair
// table stores the SIGNED antisymmetrised integral: the magnitude is the
// heat-bath weight of the reference table (hb_table.cpp:102-138) and, up to
// the fermionic phase and a sign fixed by the spins, it is also the double
// excitation matrix element (ham_eval.cpp:117-147), so doubles need no ERI
// reads at all.
#pragma once

#include <atomic>
#include <vector>

#include "common.cuh"

namespace dnq {

struct PairTableView {
    const i64* off = nullptr;  // [n_rows + 1]
    const u16* ab = nullptr;   // a | b << 8   (a > b, spin-orbital indices)
    const double* v = nullptr; // signed <ij||ab>, |v| non-increasing per row
};

struct CtxView {
    int n = 0;
    int nso = 0;
    const double* h1 = nullptr;
    const double* dss = nullptr;
    const double* dos = nullptr;
    const double* sss = nullptr;
    const double* sos = nullptr;
    const double* eri = nullptr;   // packed 8-fold (pq|rs), integral_mo.hpp:40-49
    PairTableView tab;
};

// <ij||ab> = <ij|ab> - <ij|ba> over spin-orbitals (even = alpha, odd = beta)
// from the packed ERIs, with the spin zeroing of integral_so.hpp:89-108:
// the value the pair table stores for row (i, j), entry (a, b).
__host__ __device__ __forceinline__ i64 tri_index(i64 p, i64 q) {
    return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
}
__host__ __device__ __forceinline__ double phys_so_of(const double* eri, int mu, int ka, int nu,
                                                      int la) {
    if (((mu ^ nu) & 1) || ((ka ^ la) & 1)) return 0.0;
    return eri[tri_index(tri_index(mu >> 1, nu >> 1), tri_index(ka >> 1, la >> 1))];
}
__host__ __device__ __forceinline__ double anti_so_of(const double* eri, int i, int j, int a,
                                                      int b) {
    return phys_so_of(eri, i, j, a, b) - phys_so_of(eri, i, j, b, a);
}

__host__ __device__ __forceinline__ i64 pair_row(int i, int j) {
    if (i < j) { int t = i; i = j; j = t; }
    return (i64)i * (i - 1) / 2 + j;
}

struct PairTable {
    DBuf<i64> off;
    DBuf<u16> ab;
    DBuf<double> v;
    i64 n_rows = 0;
    i64 n_entries = 0;
    double threshold = 0.0;   // entries kept: |v| >= threshold
    double tie_threshold = -1.0;   // tied weights >= this are in the reference's order
    i64 tie_rows = 0;              // rows re-ordered for ties at tie_threshold
    size_t bytes() const { return off.bytes() + ab.bytes() + v.bytes(); }
};

}  // namespace dnq

struct dnq_ctx_s {
    int device = 0;
    int n = 0;
    int nso = 0;
    double e_nuc = 0.0;
    std::vector<double> h1p, erip;   // packed host copies
    dnq::DBuf<double> h1, dss, dos, sss, sos, erid;
    dnq::PairTable tab;
    bool has_hb = false;
    double hb_thr = 0.0;
    std::atomic<long long> vv_nnz_hint{0};   // largest H_VV (entries or members) built here

    dnq::CtxView view() const {
        dnq::CtxView c;
        c.n = n;
        c.nso = nso;
        c.h1 = h1.p;
        c.dss = dss.p;
        c.dos = dos.p;
        c.sss = sss.p;
        c.sos = sos.p;
        c.eri = erid.p;
        c.tab.off = tab.off.p;
        c.tab.ab = tab.ab.p;
        c.tab.v = tab.v.p;
        return c;
    }
    int64_t bytes() const {
        return (int64_t)(h1.bytes() + dss.bytes() + dos.bytes() + sss.bytes() +
                         sos.bytes() + erid.bytes() + tab.bytes());
    }
};

namespace dnq {
// One-word entry points need spin strings that fit one uint64.
inline void require_narrow(const dnq_ctx_s* c) {
    if (c && c->n > 64)
        throw Error(DNQ_ERR_INVALID,
                    "context has more than 64 orbitals: use the two-word entry points");
}
// Smallest double strictly above 1e-15: "w > 1e-15" == "w >= kFullCut".
double full_cutoff();
// Effective heat-bath cutoff of the reference query with_cutoff(eps) on a
// table built with threshold t (hb_table.hpp:131-146).
double hb_cutoff(const dnq_ctx_s* c, double eps);
}  // namespace dnq
