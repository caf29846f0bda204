// wide.cpp -- CPU restatement of the screened build for determinants of up
// to 128 orbitals (W = 2 words per spin).  TEST INFRASTRUCTURE ONLY, like
// oracle.cpp: only tests/, smoke() and bench.py's CPU legs load it.
//
// The reference holds a spin string in one uint64 (det.hpp:30-36) and
// rejects more than 64 orbitals (integral_mo.cpp:26-28), so there is no
// reference output at 100 orbitals.  This file restates the same algorithm
// for a W-word string, W in {1, 2}:
//   excitation analysis and phase          det_ops.cpp:45-196
//   Slater-Condon elements, same order     ham_eval.cpp:33-147
//   heat-bath table and cutoff query       hb_table.cpp:39-168, hb_table.hpp:131-146
//   singles, heat-bath doubles             det_ops.hpp:123-159, ham_utils.hpp:280-313
//   static / dynamic routing and screening build_ham.cpp:139-196, :256-312
//   deferred P indexing, canonical COO     build_ham.cpp:346-380, ham_utils.cpp:41-83
// and is pinned, for n <= 64, to the reference core compiled from source
// (tests/test_oracle_wide.py): with the high words zero both W = 1 and
// W = 2 must reproduce get_ham_conn / get_ham_conn_amp bit for bit.
//
// Determinant layout: 2W uint64 per determinant, alpha words (low word
// first) then beta words.  Order: alpha as a 64W-bit integer, then beta,
// which is the reference's lexicographic (alpha, beta) order for W = 1.
#include "dq_result.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <unordered_map>
#include <vector>

namespace {

using u32 = uint32_t;
using u64 = uint64_t;

template <int W>
struct Str {
    u64 w[W];
    bool test(int i) const { return (w[i >> 6] >> (i & 63)) & 1; }
    void set(int i) { w[i >> 6] |= 1ull << (i & 63); }
    void clear(int i) { w[i >> 6] &= ~(1ull << (i & 63)); }
    int popc() const {
        int c = 0;
        for (int k = 0; k < W; ++k) c += __builtin_popcountll(w[k]);
        return c;
    }
    // set bits strictly between x and y (det_ops.cpp:85-93)
    int between(int x, int y) const {
        if (x == y) return 0;
        const int lo = std::min(x, y), hi = std::max(x, y);
        int c = 0;
        for (int i = lo + 1; i < hi; ++i) c += test(i);
        return c;
    }
    // ascending list of set bits
    int list(int* out, int base_mul, int add) const {
        int m = 0;
        for (int k = 0; k < W; ++k)
            for (u64 x = w[k]; x; x &= x - 1)
                out[m++] = base_mul * (64 * k + __builtin_ctzll(x)) + add;
        return m;
    }
};

template <int W>
struct Det {
    Str<W> a, b;
    bool operator==(const Det& o) const {
        for (int k = 0; k < W; ++k)
            if (a.w[k] != o.a.w[k] || b.w[k] != o.b.w[k]) return false;
        return true;
    }
    bool operator<(const Det& o) const {
        for (int k = W - 1; k >= 0; --k)
            if (a.w[k] != o.a.w[k]) return a.w[k] < o.a.w[k];
        for (int k = W - 1; k >= 0; --k)
            if (b.w[k] != o.b.w[k]) return b.w[k] < o.b.w[k];
        return false;
    }
};

template <int W>
struct DetHash {
    size_t operator()(const Det<W>& d) const {
        u64 x = 0x9E3779B97F4A7C15ull;
        for (int k = 0; k < W; ++k) {
            x = (x ^ d.a.w[k]) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ d.b.w[k]) * 0x94D049BB133111EBull;
        }
        return (size_t)(x ^ (x >> 31));
    }
};

inline size_t tri(size_t p, size_t q) {
    if (p < q) std::swap(p, q);
    return p * (p + 1) / 2 + q;
}

// Packed integrals (integral_mo.hpp:30-49) and the spin-orbital view
// (integral_so.hpp:77-108), for up to 128 orbitals.
struct Ints {
    int n = 0;
    double e_nuc = 0.0;
    std::vector<double> h1, h2;
    double mo1(int p, int q) const { return h1[tri(p, q)]; }
    double mo2(int p, int q, int r, int s) const { return h2[tri(tri(p, q), tri(r, s))]; }
    double phys(int mu, int ka, int nu, int la) const {
        if (((mu ^ nu) & 1) || ((ka ^ la) & 1)) return 0.0;
        return mo2(mu >> 1, nu >> 1, ka >> 1, la >> 1);
    }
    double anti(int mu, int ka, int nu, int la) const {
        return phys(mu, ka, nu, la) - phys(mu, ka, la, nu);
    }
    double so1(int mu, int nu) const {
        if ((mu ^ nu) & 1) return 0.0;
        return mo1(mu >> 1, nu >> 1);
    }
};

// Heat-bath table (hb_table.cpp:39-168); rows filled in parallel.
struct HB {
    int nso = 0;
    std::vector<size_t> off;
    std::vector<int16_t> A, B;
    std::vector<double> Wt;
    static size_t row_of(int i, int j) {
        if (i < j) std::swap(i, j);
        return (size_t)i * (i - 1) / 2 + j;
    }
    HB(const Ints& I, double thr) {
        nso = 2 * I.n;
        if (nso < 2) throw std::invalid_argument("HeatBathTable requires n_so >= 2");
        const size_t nrows = (size_t)nso * (nso - 1) / 2;
        std::vector<std::vector<std::pair<double, std::pair<int16_t, int16_t>>>> rows(nrows);
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 1; i < nso; ++i)
            for (int j = 0; j < i; ++j) {
                auto& r = rows[row_of(i, j)];
                for (int a = 1; a < nso; ++a)
                    for (int b = 0; b < a; ++b) {
                        if (a == i || a == j || b == i || b == j) continue;
                        const int si = i & 1, sj = j & 1, sa = a & 1, sb = b & 1;
                        if (!((sa == si && sb == sj) || (sa == sj && sb == si))) continue;
                        const double w = std::abs(I.anti(i, j, a, b));
                        if (w >= thr) r.push_back({w, {(int16_t)a, (int16_t)b}});
                    }
                // std::ranges::sort(row, std::greater{}, &Entry::w) of the
                // reference (hb_table.cpp:133) is libstdc++'s std::sort with
                // this comparison: the same (unstable) order of tied weights.
                std::sort(r.begin(), r.end(),
                          [](const auto& x, const auto& y) { return x.first > y.first; });
            }
        off.assign(nrows + 1, 0);
        for (size_t t = 0; t < nrows; ++t) off[t + 1] = off[t] + rows[t].size();
        A.resize(off[nrows]);
        B.resize(off[nrows]);
        Wt.resize(off[nrows]);
#pragma omp parallel for schedule(dynamic, 64)
        for (long t = 0; t < (long)nrows; ++t) {
            for (size_t k = 0; k < rows[t].size(); ++k) {
                A[off[t] + k] = rows[t][k].second.first;
                B[off[t] + k] = rows[t][k].second.second;
                Wt[off[t] + k] = rows[t][k].first;
            }
            std::vector<std::pair<double, std::pair<int16_t, int16_t>>>().swap(rows[t]);
        }
    }
    std::pair<size_t, size_t> prefix(int i, int j, double eps) const {  // hb_table.hpp:131-146
        if (i == j) return {0, 0};
        const size_t r = row_of(i, j);
        size_t lo = off[r], len = off[r + 1] - off[r];
        if (eps <= 0.0 || len == 0) return {lo, len};
        size_t L = 0, R = len;
        while (L < R) {
            const size_t mid = L + (R - L) / 2;
            if (Wt[lo + mid] >= eps) L = mid + 1; else R = mid;
        }
        return {lo, L};
    }
};

struct Ctx {
    Ints I;
    std::unique_ptr<HB> hb;
};

struct Exc {
    int degree = 0;
    double phase = 1.0;
    int nx[2] = {0, 0};
    int hole[2][2] = {{0, 0}, {0, 0}};
    int part[2][2] = {{0, 0}, {0, 0}};
};

// det_ops.cpp:45-196: holes = ket & ~bra, particles = bra & ~ket, ascending.
template <int W>
Exc analyze(const Det<W>& bra, const Det<W>& ket) {
    Exc e;
    const Str<W>* br[2] = {&bra.a, &bra.b};
    const Str<W>* kt[2] = {&ket.a, &ket.b};
    bool bad = false;
    for (int s = 0; s < 2; ++s) {
        int nh = 0, np_ = 0;
        int hs[4], ps[4];
        for (int k = 0; k < W; ++k) {
            u64 h = kt[s]->w[k] & ~br[s]->w[k], p = br[s]->w[k] & ~kt[s]->w[k];
            for (; h; h &= h - 1) {
                if (nh < 4) hs[nh] = 64 * k + __builtin_ctzll(h);
                ++nh;
            }
            for (; p; p &= p - 1) {
                if (np_ < 4) ps[np_] = 64 * k + __builtin_ctzll(p);
                ++np_;
            }
        }
        if (nh != np_) { e.nx[s] = 3; bad = true; continue; }
        e.nx[s] = nh;
        if (nh > 2) { bad = true; continue; }
        for (int t = 0; t < nh; ++t) {
            e.hole[s][t] = hs[t];
            e.part[s][t] = ps[t];
        }
    }
    e.degree = e.nx[0] + e.nx[1];
    if (bad || e.degree > 2) { e.phase = 0.0; return e; }
    int perm = 0;
    for (int s = 0; s < 2; ++s) {  // det_ops.cpp:101-127
        for (int t = 0; t < e.nx[s]; ++t) perm += br[s]->between(e.hole[s][t], e.part[s][t]);
        if (e.nx[s] == 2) {
            const int a = std::min(e.hole[s][0], e.part[s][0]);
            const int b = std::max(e.hole[s][0], e.part[s][0]);
            const int c = std::min(e.hole[s][1], e.part[s][1]);
            const int d = std::max(e.hole[s][1], e.part[s][1]);
            if ((c > a && c < b && d > b) || (a > c && a < d && b > d)) ++perm;
        }
    }
    e.phase = (perm & 1) ? -1.0 : 1.0;
    return e;
}

template <int W>
int occ_list(const Det<W>& d, int* out) {  // alpha SOs ascending, then beta
    const int m = d.a.list(out, 2, 0);
    return m + d.b.list(out + m, 2, 1);
}

template <int W>
double diag(const Ints& I, const Det<W>& d) {  // ham_eval.cpp:53-86
    int occ[256];
    const int m = occ_list(d, occ);
    double one = 0.0;
    for (int t = 0; t < m; ++t) one += I.so1(occ[t], occ[t]);
    double two = 0.0;
    for (int x = 1; x < m; ++x)
        for (int y = 0; y < x; ++y) two += I.anti(occ[x], occ[y], occ[x], occ[y]);
    return one + two;
}

template <int W>
double elem(const Ints& I, const Det<W>& bra, const Det<W>& ket) {  // ham_eval.cpp:33-147
    const Exc e = analyze(bra, ket);
    if (e.degree > 2) return 0.0;
    if (e.degree == 0) return diag(I, ket);
    if (e.degree == 1) {
        const int s = e.nx[0] == 1 ? 0 : 1;
        const int i = 2 * e.hole[s][0] + s, a = 2 * e.part[s][0] + s;
        double v = I.so1(a, i);
        int occ[256];
        const int m = occ_list(ket, occ);
        for (int t = 0; t < m; ++t)
            if (occ[t] != i) v += I.anti(a, occ[t], i, occ[t]);
        return e.phase * v;
    }
    for (int s = 0; s < 2; ++s)
        if (e.nx[s] == 2)
            return e.phase * I.anti(2 * e.part[s][0] + s, 2 * e.part[s][1] + s,
                                    2 * e.hole[s][0] + s, 2 * e.hole[s][1] + s);
    return e.phase * I.phys(2 * e.part[0][0], 2 * e.part[1][0] + 1, 2 * e.hole[0][0],
                            2 * e.hole[1][0] + 1);
}

// Singles, alpha then beta, holes ascending outer, particles inner
// (det_ops.hpp:123-159).
template <int W, class F>
void singles(const Det<W>& k, int n, F&& f) {
    for (int s = 0; s < 2; ++s) {
        const Str<W>& occ = s ? k.b : k.a;
        int hs[128], m = occ.list(hs, 1, 0);
        for (int t = 0; t < m; ++t)
            for (int p = 0; p < n; ++p) {
                if (occ.test(p)) continue;
                Det<W> ket = k;
                Str<W>& o = s ? ket.b : ket.a;
                o.clear(hs[t]);
                o.set(p);
                f(ket);
            }
    }
}

inline bool so_occ_hi(int so, int n) { return (so >> 1) >= n; }

// Heat-bath doubles (ham_utils.hpp:280-313; exc2_so ham_utils.cpp:484-506).
template <int W, class F>
void doubles_hb(const Det<W>& bra, int n, const HB& hb, double cut, F&& f) {
    int occ[256];
    const int m = occ_list(bra, occ);
    for (int p = 1; p < m; ++p)
        for (int q = 0; q < p; ++q) {
            const int i = occ[p], j = occ[q];
            auto [lo, len] = hb.prefix(i, j, cut);
            for (size_t t = lo; t < lo + len; ++t) {
                const int a = hb.A[t], b = hb.B[t];
                auto occd = [&](int so) {
                    if (so_occ_hi(so, n)) return true;
                    return ((so & 1) ? bra.b : bra.a).test(so >> 1);
                };
                if (occd(a) || occd(b)) continue;
                Det<W> ket = bra;
                Str<W>* w[2] = {&ket.a, &ket.b};
                w[i & 1]->clear(i >> 1);
                w[j & 1]->clear(j >> 1);
                w[a & 1]->set(a >> 1);
                w[b & 1]->set(b >> 1);
                f(ket);
            }
        }
}

struct Trip { u32 r, c; double v; };

void canon(std::vector<Trip>& t, dq::Coo& out) {  // ham_utils.cpp:41-83
    std::stable_sort(t.begin(), t.end(), [](const Trip& x, const Trip& y) {
        return x.r < y.r || (x.r == y.r && x.c < y.c);
    });
    out.rows.clear(); out.cols.clear(); out.vals.clear();
    for (size_t i = 0; i < t.size();) {
        double v = t[i].v;
        size_t j = i + 1;
        while (j < t.size() && t[j].r == t[i].r && t[j].c == t[i].c) v += t[j++].v;
        if (std::abs(v) > 0.0) {
            out.rows.push_back(t[i].r); out.cols.push_back(t[i].c); out.vals.push_back(v);
        }
        i = j;
    }
}

constexpr double kElemThresh = 1e-15;   // ham_utils.hpp:39
constexpr double kAmpFloor = 1e-12;     // build_ham.cpp:161-186

template <int W>
Det<W> load(const uint64_t* p) {
    Det<W> d;
    for (int k = 0; k < W; ++k) {
        d.a.w[k] = p[k];
        d.b.w[k] = p[W + k];
    }
    return d;
}

template <int W>
void store(const Det<W>& d, uint64_t* p) {
    for (int k = 0; k < W; ++k) {
        p[k] = d.a.w[k];
        p[W + k] = d.b.w[k];
    }
}

// Screened V -> {V, P} build of rows [r0, r1) of V (all of V is the row
// space for routing).  psi == nullptr: static heat-bath policy (singles
// unscreened, doubles w >= eps1); else the dynamic amplitude policy
// (singles need |h psi_i| >= eps1, doubles w >= eps1 / max(|psi_i|, 1e-12)).
template <int W>
dq::Result* build(Ctx* c, const uint64_t* Vp, int64_t n, const double* psi, int n_orb,
                  double eps1, int64_t r0, int64_t r1) {
    if (!c->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    if (n_orb > 64 * W || n_orb > c->I.n) throw std::invalid_argument("n_orb out of range");
    std::vector<Det<W>> V(n);
    std::unordered_map<Det<W>, u32, DetHash<W>> map;
    map.reserve(2 * n);
    for (int64_t i = 0; i < n; ++i) {
        V[i] = load<W>(Vp + 2 * W * i);
        if (!map.emplace(V[i], (u32)i).second)
            throw std::invalid_argument("DetMap::from_ordered: duplicate determinant found");
    }
    r0 = std::max<int64_t>(0, r0);
    r1 = std::min<int64_t>(n, r1);
    const int64_t R = std::max<int64_t>(0, r1 - r0);
    struct Keyed { u32 row; Det<W> k; double v; };
    std::vector<std::vector<Trip>> tv(R);
    std::vector<std::vector<Keyed>> tk(R);
    const Ints& I = c->I;
    const HB& hb = *c->hb;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t q = 0; q < R; ++q) {
        const u32 row = (u32)(r0 + q);
        const Det<W>& bra = V[row];
        const double hd = diag(I, bra);
        if (std::abs(hd) > kElemThresh) tv[q].push_back({row, row, hd});
        auto emit = [&](const Det<W>& ket, double h) {
            auto it = map.find(ket);
            if (it != map.end()) tv[q].push_back({row, it->second, h});
            else tk[q].push_back({row, ket, h});
        };
        singles(bra, n_orb, [&](const Det<W>& ket) {
            const double h = elem(I, bra, ket);
            if (std::abs(h) <= kElemThresh) return;
            if (psi && !(std::abs(h * psi[row]) >= eps1)) return;   // build_ham.cpp:190-192
            emit(ket, h);
        });
        const double cut = psi ? eps1 / std::max(std::abs(psi[row]), kAmpFloor) : eps1;
        doubles_hb(bra, n_orb, hb, cut, [&](const Det<W>& ket) {
            const double h = elem(I, bra, ket);
            if (std::abs(h) <= kElemThresh) return;
            emit(ket, h);
        });
    }
    std::vector<Trip> vv;
    std::vector<Keyed> vk;
    for (int64_t q = 0; q < R; ++q) {
        vv.insert(vv.end(), tv[q].begin(), tv[q].end());
        vk.insert(vk.end(), tk[q].begin(), tk[q].end());
    }
    auto* out = new dq::Result;
    canon(vv, out->a);
    out->a.nr = out->a.nc = (u32)n;
    std::vector<Det<W>> P;   // build_ham.cpp:346-380
    P.reserve(vk.size());
    for (auto& e : vk) P.push_back(e.k);
    std::sort(P.begin(), P.end());
    P.erase(std::unique(P.begin(), P.end()), P.end());
    std::vector<Trip> t;
    t.reserve(vk.size());
    for (auto& e : vk)
        t.push_back({e.row, (u32)(std::lower_bound(P.begin(), P.end(), e.k) - P.begin()), e.v});
    canon(t, out->b);
    out->b.nr = (u32)n;
    out->b.nc = (u32)P.size();
    out->dets.resize(P.size() * 2 * W);
    for (size_t i = 0; i < P.size(); ++i) store(P[i], out->dets.data() + 2 * W * i);
    return out;
}

}  // namespace

extern "C" {

void* dqw_ctx_from_arrays(int n_orb, const double* h1, const double* h2, double e_nuc) {
    try {
        if (n_orb <= 0 || n_orb > 128)
            throw std::invalid_argument("Number of orbitals must be in [1, 128]");
        auto* c = new Ctx;
        c->I.n = n_orb;
        c->I.e_nuc = e_nuc;
        const size_t n1 = (size_t)n_orb * (n_orb + 1) / 2;
        c->I.h1.assign(h1, h1 + n1);
        c->I.h2.assign(h2, h2 + n1 * (n1 + 1) / 2);
        return c;
    } catch (const std::exception& e) {
        dq::g_err = e.what();
        return nullptr;
    }
}

void dqw_ctx_free(void* c) { delete (Ctx*)c; }

int dqw_hb_prepare(void* c, double thr) {
    try {
        ((Ctx*)c)->hb = std::make_unique<HB>(((Ctx*)c)->I, thr);
        return 0;
    } catch (const std::exception& e) {
        dq::g_err = e.what();
        return 1;
    }
}

int dqw_diag(void* c, int words, const uint64_t* d, int64_t n, double* out) {
    const Ints& I = ((Ctx*)c)->I;
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i)
        out[i] = words == 1 ? diag(I, load<1>(d + 2 * i)) : diag(I, load<2>(d + 4 * i));
    return 0;
}

double dqw_elem(void* c, int words, const uint64_t* bra, const uint64_t* ket) {
    const Ints& I = ((Ctx*)c)->I;
    return words == 1 ? elem(I, load<1>(bra), load<1>(ket)) : elem(I, load<2>(bra), load<2>(ket));
}

void* dqw_build(void* c, int words, const uint64_t* V, int64_t n, const double* psi, int n_orb,
                double eps1, int64_t r0, int64_t r1) {
    try {
        if (words == 1) return build<1>((Ctx*)c, V, n, psi, n_orb, eps1, r0, r1);
        if (words == 2) return build<2>((Ctx*)c, V, n, psi, n_orb, eps1, r0, r1);
        throw std::invalid_argument("words must be 1 or 2");
    } catch (const std::exception& e) {
        dq::g_err = e.what();
        return nullptr;
    }
}

}  // extern "C"
