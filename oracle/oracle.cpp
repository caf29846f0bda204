// oracle.cpp -- CPU restatement of the DetNQS determinant-space Hamiltonian
// path, used ONLY as a checker (tests/, __graft_entry__.smoke(), and the
// cpu_baseline leg of bench.py).  It is never linked into or called by the
// product library in detnqs_b200/.
//
// Each function names the reference file:line it restates (paths relative to
// the wsmxcz/DetNQS tree).  Floating-point expressions keep the reference's
// operand order so that, compiled without FMA contraction
// (-ffp-contract=off, see oracle/Makefile), element values agree bit for bit.
//
// Parity pin: tests/test_oracle_pin.py checks this file against the
// reference core compiled from source (oracle/_ref) and against the golden
// fixtures in tests/golden/.
#include "dq_api.h"
#include "dq_result.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

using u32 = uint32_t;
using u64 = uint64_t;

// ---------------------------------------------------------------------------
// Determinant key: (alpha, beta), lexicographic order (det.hpp:30-36).
// ---------------------------------------------------------------------------
struct Key {
    u64 a, b;
    bool operator==(const Key& o) const { return a == o.a && b == o.b; }
    bool operator<(const Key& o) const { return a < o.a || (a == o.a && b < o.b); }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        u64 x = k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull);
        x ^= x >> 31;
        x *= 0xBF58476D1CE4E5B9ull;
        return (size_t)(x ^ (x >> 29));
    }
};

inline int popc(u64 x) { return __builtin_popcountll(x); }
inline int ctz(u64 x) { return __builtin_ctzll(x); }
inline u64 low_mask(int n) {  // bit_utils.hpp:114-119
    return n <= 0 ? 0 : (n >= 64 ? ~0ull : ((1ull << n) - 1));
}

// ---------------------------------------------------------------------------
// Integrals: packed keys (integral_mo.hpp:30-49), SO view with spin zeroing
// (integral_so.hpp:77-108; even SO = alpha, odd SO = beta).
// ---------------------------------------------------------------------------
inline size_t tri(size_t p, size_t q) {
    if (p < q) std::swap(p, q);
    return p * (p + 1) / 2 + q;
}

struct Ints {
    int n = 0;
    double e_nuc = 0.0;
    std::vector<double> h1, h2;

    explicit Ints(int n_) : n(n_) {
        if (n_ <= 0 || n_ > 64)
            throw std::invalid_argument("Number of orbitals must be in [1, 64]");
        size_t n1 = (size_t)n * (n + 1) / 2;
        h1.assign(n1, 0.0);
        h2.assign(n1 * (n1 + 1) / 2, 0.0);
    }
    double mo1(int p, int q) const { return h1[tri(p, q)]; }
    double mo2(int p, int q, int r, int s) const {
        return h2[tri(tri(p, q), tri(r, s))];
    }
    // <mu kappa | nu lambda> = (mu nu | kappa lambda), zero unless
    // spin(mu)=spin(nu) and spin(kappa)=spin(lambda) (integral_so.hpp:89-97).
    double phys(int mu, int ka, int nu, int la) const {
        if (((mu ^ nu) & 1) || ((ka ^ la) & 1)) return 0.0;
        return mo2(mu >> 1, nu >> 1, ka >> 1, la >> 1);
    }
    double anti(int mu, int ka, int nu, int la) const {  // integral_so.hpp:105-108
        return phys(mu, ka, nu, la) - phys(mu, ka, la, nu);
    }
    double so1(int mu, int nu) const {  // integral_so.hpp:77-83
        if ((mu ^ nu) & 1) return 0.0;
        return mo1(mu >> 1, nu >> 1);
    }
};

// FCIDUMP reader (integral_mo.cpp:48-182): the &FCI namelist is skipped,
// Fortran 'D' exponents are accepted, indices are 1-based.
void load_fcidump(Ints& I, const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("Cannot open FCIDUMP: " + path);
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty()) continue;
        const char c0 = line[0];
        if (c0 == '!' || c0 == '*' || c0 == 'C' || c0 == 'c' || c0 == '#') continue;
        if (line.find('&') != std::string::npos) continue;
        for (char& ch : line)
            if (ch == 'D' || ch == 'd') ch = 'E';
        std::istringstream is(line);
        double v;
        int p, q, r, s;
        if (!(is >> v >> p >> q >> r >> s)) continue;
        if (p == 0 && q == 0 && r == 0 && s == 0) I.e_nuc = v;
        else if (r == 0 && s == 0) I.h1[tri(p - 1, q - 1)] = v;
        else I.h2[tri(tri(p - 1, q - 1), tri(r - 1, s - 1))] = v;
    }
}

// ---------------------------------------------------------------------------
// Excitation analysis and phase (det_ops.cpp:45-196).
// holes = ket & ~bra, particles = bra & ~ket, per spin, ascending.
// ---------------------------------------------------------------------------
struct Exc {
    int degree = 0;
    double phase = 1.0;
    int nx[2] = {0, 0};         // excitations per spin
    int hole[2][2] = {{0, 0}, {0, 0}};
    int part[2][2] = {{0, 0}, {0, 0}};
};

inline int between(u64 occ, int x, int y) {  // det_ops.cpp:85-93
    if (x == y) return 0;
    int lo = std::min(x, y), hi = std::max(x, y);
    return popc(occ & low_mask(hi) & ~low_mask(lo + 1));
}

Exc analyze(Key bra, Key ket) {
    Exc e;
    const u64 br[2] = {bra.a, bra.b}, kt[2] = {ket.a, ket.b};
    int total = 0;
    bool bad = false;
    for (int s = 0; s < 2; ++s) {
        u64 h = kt[s] & ~br[s], p = br[s] & ~kt[s];
        int nh = popc(h), np_ = popc(p);
        if (nh != np_) { e.nx[s] = 3; bad = true; continue; }  // det_ops.cpp:59-62
        e.nx[s] = nh;
        if (nh > 2) { bad = true; continue; }
        for (int k = 0; k < nh; ++k) {
            e.hole[s][k] = ctz(h); h &= h - 1;
            e.part[s][k] = ctz(p); p &= p - 1;
        }
    }
    total = e.nx[0] + e.nx[1];
    e.degree = total;
    if (bad || total > 2) { e.phase = 0.0; return e; }
    int perm = 0;
    for (int s = 0; s < 2; ++s) {  // det_ops.cpp:101-127
        for (int k = 0; k < e.nx[s]; ++k)
            perm += between(br[s], e.hole[s][k], e.part[s][k]);
        if (e.nx[s] == 2) {
            int a = std::min(e.hole[s][0], e.part[s][0]);
            int b = std::max(e.hole[s][0], e.part[s][0]);
            int c = std::min(e.hole[s][1], e.part[s][1]);
            int d = std::max(e.hole[s][1], e.part[s][1]);
            if ((c > a && c < b && d > b) || (a > c && a < d && b > d)) ++perm;
        }
    }
    e.phase = (perm & 1) ? -1.0 : 1.0;
    return e;
}

// ---------------------------------------------------------------------------
// Slater-Condon elements (ham_eval.cpp:33-147).
// ---------------------------------------------------------------------------
struct Ham {
    const Ints& I;
    explicit Ham(const Ints& i) : I(i) {}

    // occupied SOs: alpha ascending (2p) then beta ascending (2p+1)
    static int occ_list(Key d, int* out) {
        int m = 0;
        for (u64 x = d.a; x; x &= x - 1) out[m++] = 2 * ctz(x);
        for (u64 x = d.b; x; x &= x - 1) out[m++] = 2 * ctz(x) + 1;
        return m;
    }

    double diag(Key d) const {  // ham_eval.cpp:53-86
        int occ[128];
        const int m = occ_list(d, occ);
        double one = 0.0;
        for (int t = 0; t < m; ++t) one += I.so1(occ[t], occ[t]);
        double two = 0.0;
        for (int x = 1; x < m; ++x)
            for (int y = 0; y < x; ++y)
                two += I.anti(occ[x], occ[y], occ[x], occ[y]);
        return one + two;
    }

    double single(const Exc& e, Key ket) const {  // ham_eval.cpp:88-115
        const int s = e.nx[0] == 1 ? 0 : 1;
        const int i = 2 * e.hole[s][0] + s;   // orbital of the ket
        const int a = 2 * e.part[s][0] + s;   // orbital of the bra
        double v = I.so1(a, i);
        for (int sp = 0; sp < 2; ++sp) {
            const u64 m = sp == 0 ? ket.a : ket.b;
            for (u64 x = m; x; x &= x - 1) {
                const int k = 2 * ctz(x) + sp;
                if (k != i) v += I.anti(a, k, i, k);
            }
        }
        return v;
    }

    double dbl(const Exc& e) const {  // ham_eval.cpp:117-147
        for (int s = 0; s < 2; ++s)
            if (e.nx[s] == 2)
                return I.anti(2 * e.part[s][0] + s, 2 * e.part[s][1] + s,
                              2 * e.hole[s][0] + s, 2 * e.hole[s][1] + s);
        return I.phys(2 * e.part[0][0], 2 * e.part[1][0] + 1,
                      2 * e.hole[0][0], 2 * e.hole[1][0] + 1);
    }

    double elem(Key bra, Key ket) const {  // ham_eval.cpp:33-51
        const Exc e = analyze(bra, ket);
        if (e.degree > 2) return 0.0;
        if (e.degree == 0) return diag(ket);
        if (e.degree == 1) return e.phase * single(e, ket);
        return e.phase * dbl(e);
    }
};

// ---------------------------------------------------------------------------
// Heat-bath table (hb_table.cpp:39-168): row {i>j} holds every virtual pair
// a>b, disjoint from {i,j}, whose spins match (s_i,s_j) in either order and
// whose weight |<ij||ab>| passes the build threshold; rows sorted by weight
// descending.  Query keeps the prefix with w >= eps (hb_table.hpp:131-146).
// ---------------------------------------------------------------------------
struct HB {
    int nso = 0;
    std::vector<size_t> off;
    std::vector<int> A, B;
    std::vector<double> W;

    static size_t row_of(int i, int j) {  // hb_table.hpp:172-175
        if (i < j) std::swap(i, j);
        return (size_t)i * (i - 1) / 2 + j;
    }

    HB(const Ints& I, double thr) {
        nso = 2 * I.n;
        if (nso < 2) throw std::invalid_argument("HeatBathTable requires n_so >= 2");
        const size_t nrows = (size_t)nso * (nso - 1) / 2;
        std::vector<std::vector<std::pair<double, std::pair<int, int>>>> rows(nrows);
        for (int i = 1; i < nso; ++i)
            for (int j = 0; j < i; ++j) {
                auto& r = rows[row_of(i, j)];
                for (int a = 1; a < nso; ++a)
                    for (int b = 0; b < a; ++b) {
                        if (a == i || a == j || b == i || b == j) continue;
                        const int si = i & 1, sj = j & 1, sa = a & 1, sb = b & 1;
                        if (!((sa == si && sb == sj) || (sa == sj && sb == si))) continue;
                        const double w = std::abs(I.anti(i, j, a, b));
                        if (w >= thr) r.push_back({w, {a, b}});
                    }
                // std::ranges::sort(row, std::greater{}, &Entry::w) of the
                // reference (hb_table.cpp:133) is libstdc++'s std::sort with
                // this comparison: the same (unstable) order of tied weights.
                std::sort(r.begin(), r.end(),
                          [](const auto& x, const auto& y) { return x.first > y.first; });
            }
        off.assign(nrows + 1, 0);
        for (size_t t = 0; t < nrows; ++t) off[t + 1] = off[t] + rows[t].size();
        A.resize(off[nrows]); B.resize(off[nrows]); W.resize(off[nrows]);
        for (size_t t = 0; t < nrows; ++t)
            for (size_t k = 0; k < rows[t].size(); ++k) {
                A[off[t] + k] = rows[t][k].second.first;
                B[off[t] + k] = rows[t][k].second.second;
                W[off[t] + k] = rows[t][k].first;
            }
    }

    // [begin, begin+len) of row {i,j} restricted to w >= eps
    std::pair<size_t, size_t> prefix(int i, int j, double eps) const {
        if (i == j) return {0, 0};
        const size_t r = row_of(i, j);
        size_t lo = off[r], len = off[r + 1] - off[r];
        if (eps <= 0.0 || len == 0) return {lo, len};
        size_t L = 0, R = len;
        while (L < R) {
            size_t mid = L + (R - L) / 2;
            if (W[lo + mid] >= eps) L = mid + 1; else R = mid;
        }
        return {lo, L};
    }
};

struct Ctx {
    Ints I;
    std::unique_ptr<HB> hb;
    explicit Ctx(int n) : I(n) {}
};

// ---------------------------------------------------------------------------
// Generators (det_ops.hpp:123-268; ham_utils.hpp:280-313)
// ---------------------------------------------------------------------------
template <class F>
void singles(Key k, int n, F&& f) {  // alpha first, then beta
    const u64 all = low_mask(n);
    for (int s = 0; s < 2; ++s) {
        const u64 occ = s ? k.b : k.a, vir = ~occ & all;
        if (!occ || !vir) continue;
        for (u64 h = occ; h; h &= h - 1)
            for (u64 p = vir; p; p &= p - 1) {
                const u64 m = occ ^ (h & -h) ^ (p & -p);
                f(s ? Key{k.a, m} : Key{m, k.b});
            }
    }
}

template <class F>
void doubles(Key k, int n, F&& f) {  // aa, bb, ab
    const u64 all = low_mask(n);
    for (int s = 0; s < 2; ++s) {
        const u64 occ = s ? k.b : k.a, vir = ~occ & all;
        if (popc(occ) < 2 || popc(vir) < 2) continue;
        for (u64 h1 = occ; h1; h1 &= h1 - 1)
            for (u64 h2 = h1 & (h1 - 1); h2; h2 &= h2 - 1)
                for (u64 p1 = vir; p1; p1 &= p1 - 1)
                    for (u64 p2 = p1 & (p1 - 1); p2; p2 &= p2 - 1) {
                        const u64 m = occ ^ (h1 & -h1) ^ (h2 & -h2) ^ (p1 & -p1) ^ (p2 & -p2);
                        f(s ? Key{k.a, m} : Key{m, k.b});
                    }
    }
    const u64 va = ~k.a & all, vb = ~k.b & all;
    if (!k.a || !va || !k.b || !vb) return;
    for (u64 ha = k.a; ha; ha &= ha - 1)
        for (u64 pa = va; pa; pa &= pa - 1) {
            const u64 na = k.a ^ (ha & -ha) ^ (pa & -pa);
            for (u64 hb = k.b; hb; hb &= hb - 1)
                for (u64 pb = vb; pb; pb &= pb - 1)
                    f(Key{na, k.b ^ (hb & -hb) ^ (pb & -pb)});
        }
}

inline bool so_occupied(Key d, int so, int n) {  // ham_utils.cpp:470-479
    const int mo = so >> 1;
    if (mo < 0 || mo >= n) return true;
    return (((so & 1) ? d.b : d.a) >> mo) & 1;
}

template <class F>
void doubles_hb(Key bra, int n, const HB& hb, double cut, F&& f) {
    int occ[128];
    const int m = Ham::occ_list(bra, occ);
    for (int p = 1; p < m; ++p)
        for (int q = 0; q < p; ++q) {
            const int i = occ[p], j = occ[q];
            auto [lo, len] = hb.prefix(i, j, cut);
            for (size_t t = lo; t < lo + len; ++t) {
                const int a = hb.A[t], b = hb.B[t];
                if (so_occupied(bra, a, n) || so_occupied(bra, b, n)) continue;
                Key ket = bra;  // exc2_so, ham_utils.cpp:484-506
                u64* w[2] = {&ket.a, &ket.b};
                *w[i & 1] &= ~(1ull << (i >> 1));
                *w[j & 1] &= ~(1ull << (j >> 1));
                *w[a & 1] |= 1ull << (a >> 1);
                *w[b & 1] |= 1ull << (b >> 1);
                f(ket);
            }
        }
}

// ---------------------------------------------------------------------------
// Index maps (det_space.cpp:23-65)
// ---------------------------------------------------------------------------
struct Map {
    std::vector<Key> keys;
    std::unordered_map<Key, u32, KeyHash> idx;
    void build(const std::vector<Key>& k, bool strict) {
        keys.clear();
        idx.clear();
        idx.reserve(k.size() * 2);
        for (const Key& x : k) {
            if (idx.count(x)) {
                if (strict)
                    throw std::invalid_argument(
                        "DetMap::from_ordered: duplicate determinant found");
                continue;
            }
            idx.emplace(x, (u32)keys.size());
            keys.push_back(x);
        }
    }
    long get(Key k) const {
        auto it = idx.find(k);
        return it == idx.end() ? -1 : (long)it->second;
    }
};

std::vector<Key> keys_of(const uint64_t* p, int64_t n) {
    std::vector<Key> v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = Key{p[2 * i], p[2 * i + 1]};
    return v;
}

void put_keys(const std::vector<Key>& k, std::vector<uint64_t>& out) {
    out.resize(k.size() * 2);
    for (size_t i = 0; i < k.size(); ++i) { out[2 * i] = k[i].a; out[2 * i + 1] = k[i].b; }
}

// ---------------------------------------------------------------------------
// COO canonicalisation: sort by (row, col), sum duplicates, drop exact zeros
// (ham_utils.cpp:41-83).
// ---------------------------------------------------------------------------
struct Trip { u32 r, c; double v; };

void canon(std::vector<Trip>& t, dq::Coo& out) {
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

// ---------------------------------------------------------------------------
// Row-streamed builder (build_ham.cpp:78-380).  One policy object decides
// the double generator, single acceptance and routing of each ket.
// ---------------------------------------------------------------------------
constexpr double kElemThresh = 1e-15;   // ham_utils.hpp:39

enum Route { R_VV, R_VPI, R_KEY, R_DROP };

struct Policy {
    int kind;                 // 0 known sets, 1 static HB, 2 dynamic amplitude
    const Map* V;
    const Map* ext;
    const HB* hb;
    bool use_hb;
    double eps1;
    const double* psi;

    Route route(Key k, long& j) const {
        j = V->get(k);
        if (j >= 0) return R_VV;
        if (kind == 0) {
            j = ext ? ext->get(k) : -1;
            return j >= 0 ? R_VPI : R_DROP;
        }
        return R_KEY;
    }
    bool accept_single(u32 row, double h) const {
        return kind != 2 || std::abs(h * psi[row]) >= eps1;  // build_ham.cpp:190-192
    }
    template <class F>
    void gen_doubles(Key bra, int n, u32 row, F&& f) const {
        if (kind == 1 && use_hb) return doubles_hb(bra, n, *hb, eps1, f);
        if (kind == 2) {
            if (!hb) return doubles(bra, n, f);
            const double amp = std::max(std::abs(psi[row]), 1e-12);  // :161-186
            return doubles_hb(bra, n, *hb, eps1 / amp, f);
        }
        return doubles(bra, n, f);
    }
};

struct Keyed { u32 row; Key k; double v; };

void stream(const std::vector<Key>& V, const Ham& H, int n, const Policy& pol,
            std::vector<Trip>& vv, std::vector<Trip>& vpi, std::vector<Keyed>& vpk) {
    const long N = (long)V.size();
    std::vector<std::vector<Trip>> tv(N), ti(N);
    std::vector<std::vector<Keyed>> tk(N);
#pragma omp parallel for schedule(dynamic, 16)
    for (long r = 0; r < N; ++r) {
        const u32 row = (u32)r;
        const Key bra = V[r];
        const double hd = H.diag(bra);
        if (std::abs(hd) > kElemThresh) tv[r].push_back({row, row, hd});
        auto emit = [&](Key ket, double h, Route rt, long j) {
            if (rt == R_VV) tv[r].push_back({row, (u32)j, h});
            else if (rt == R_VPI) ti[r].push_back({row, (u32)j, h});
            else if (rt == R_KEY) tk[r].push_back({row, ket, h});
        };
        singles(bra, n, [&](Key ket) {
            long j;
            Route rt = pol.route(ket, j);
            if (rt == R_DROP) return;
            const double h = H.elem(bra, ket);
            if (std::abs(h) <= kElemThresh) return;
            if (!pol.accept_single(row, h)) return;
            emit(ket, h, rt, j);
        });
        pol.gen_doubles(bra, n, row, [&](Key ket) {
            long j;
            Route rt = pol.route(ket, j);
            if (rt == R_DROP) return;
            const double h = H.elem(bra, ket);
            if (std::abs(h) <= kElemThresh) return;
            emit(ket, h, rt, j);
        });
    }
    for (long r = 0; r < N; ++r) {
        vv.insert(vv.end(), tv[r].begin(), tv[r].end());
        vpi.insert(vpi.end(), ti[r].begin(), ti[r].end());
        vpk.insert(vpk.end(), tk[r].begin(), tk[r].end());
    }
}

// Deferred P indexing: P = sorted unique keys, columns = rank in P
// (build_ham.cpp:346-380).
void finish_keyed(std::vector<Keyed>& k, dq::Coo& vp, std::vector<Key>& P) {
    P.clear();
    P.reserve(k.size());
    for (auto& e : k) P.push_back(e.k);
    std::sort(P.begin(), P.end());
    P.erase(std::unique(P.begin(), P.end()), P.end());
    std::vector<Trip> t;
    t.reserve(k.size());
    for (auto& e : k) {
        const u32 c = (u32)(std::lower_bound(P.begin(), P.end(), e.k) - P.begin());
        t.push_back({e.row, c, e.v});
    }
    canon(t, vp);
}

dq::Result* build_blocks(Ctx* c, const std::vector<Key>& V, int n, Policy pol,
                         const std::vector<Key>* ext) {
    Map mv, me;
    mv.build(V, true);
    pol.V = &mv;
    if (ext) { me.build(*ext, true); pol.ext = &me; }
    Ham H(c->I);
    std::vector<Trip> vv, vpi;
    std::vector<Keyed> vpk;
    stream(V, H, n, pol, vv, vpi, vpk);
    auto* r = new dq::Result;
    canon(vv, r->a);
    r->a.nr = r->a.nc = (u32)V.size();
    if (pol.kind == 0) {
        if (ext && !ext->empty()) {
            canon(vpi, r->b);
            r->b.nr = (u32)V.size();
            r->b.nc = (u32)ext->size();
            put_keys(me.keys, r->dets);
        }
    } else {
        std::vector<Key> P;
        finish_keyed(vpk, r->b, P);
        r->b.nr = (u32)V.size();
        r->b.nc = (u32)P.size();
        put_keys(P, r->dets);
    }
    return r;
}

}  // namespace

#define GUARD_BEGIN try {
#define GUARD_END(ret)                \
    }                                 \
    catch (const std::exception& e) { \
        dq::g_err = e.what();         \
        return ret;                   \
    }

extern "C" {

void* dq_ctx_from_fcidump(const char* path, int n_orb) {
    GUARD_BEGIN
    auto* c = new Ctx(n_orb);
    load_fcidump(c->I, path);
    return c;
    GUARD_END(nullptr)
}

void* dq_ctx_from_arrays(int n_orb, const double* h1, const double* h2, double e_nuc) {
    GUARD_BEGIN
    auto* c = new Ctx(n_orb);
    std::copy(h1, h1 + c->I.h1.size(), c->I.h1.begin());
    std::copy(h2, h2 + c->I.h2.size(), c->I.h2.begin());
    c->I.e_nuc = e_nuc;
    return c;
    GUARD_END(nullptr)
}

void dq_ctx_free(void* c) { delete (Ctx*)c; }
double dq_ctx_e_nuc(void* c) { return ((Ctx*)c)->I.e_nuc; }

int dq_hb_prepare(void* c, double thr) {
    GUARD_BEGIN
    ((Ctx*)c)->hb = std::make_unique<HB>(((Ctx*)c)->I, thr);
    return 0;
    GUARD_END(-1)
}

int dq_hb_clear(void* c) { ((Ctx*)c)->hb.reset(); return 0; }

int64_t dq_hb_row(void* c, int i, int j, int32_t* a, int32_t* b, double* w, int64_t cap) {
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) return -1;
    auto [lo, len] = ctx->hb->prefix(i, j, 0.0);
    for (size_t k = 0; k < len && (int64_t)k < cap; ++k) {
        a[k] = ctx->hb->A[lo + k]; b[k] = ctx->hb->B[lo + k]; w[k] = ctx->hb->W[lo + k];
    }
    return (int64_t)len;
}

int dq_analyze(const uint64_t* bra, const uint64_t* ket, int* degree, double* phase) {
    Exc e = analyze(Key{bra[0], bra[1]}, Key{ket[0], ket[1]});
    *degree = e.degree;
    *phase = e.phase;
    return 0;
}

double dq_compute_elem(void* c, const uint64_t* bra, const uint64_t* ket) {
    return Ham(((Ctx*)c)->I).elem(Key{bra[0], bra[1]}, Key{ket[0], ket[1]});
}

int dq_ham_diag(void* c, const uint64_t* d, int64_t n, double* out) {
    Ham H(((Ctx*)c)->I);
#pragma omp parallel for if (n > 256)
    for (int64_t i = 0; i < n; ++i) out[i] = H.diag(Key{d[2 * i], d[2 * i + 1]});
    return 0;
}

void* dq_get_ham_vv(void* c, const uint64_t* V, int64_t n, int n_orb) {
    GUARD_BEGIN
    auto* r = new dq::Result;
    if (n == 0) return r;
    delete r;
    Policy p{0, nullptr, nullptr, nullptr, false, 0.0, nullptr};
    return build_blocks((Ctx*)c, keys_of(V, n), n_orb, p, nullptr);
    GUARD_END(nullptr)
}

void* dq_get_ham_block(void* c, const uint64_t* V, int64_t nv, const uint64_t* P,
                       int64_t np_, int n_orb) {
    GUARD_BEGIN
    if (nv == 0) return new dq::Result;
    Policy p{0, nullptr, nullptr, nullptr, false, 0.0, nullptr};
    std::vector<Key> ext;
    if (P) ext = keys_of(P, np_);
    return build_blocks((Ctx*)c, keys_of(V, nv), n_orb, p, P ? &ext : nullptr);
    GUARD_END(nullptr)
}

void* dq_get_ham_conn(void* c, const uint64_t* V, int64_t n, int n_orb, int use_hb,
                      double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (use_hb && !ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    if (n == 0) return new dq::Result;
    Policy p{1, nullptr, nullptr, ctx->hb.get(), use_hb != 0, eps1, nullptr};
    return build_blocks(ctx, keys_of(V, n), n_orb, p, nullptr);
    GUARD_END(nullptr)
}

void* dq_get_ham_conn_amp(void* c, const uint64_t* V, int64_t n, const double* psi,
                          int n_orb, double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    if (n == 0) return new dq::Result;
    Policy p{2, nullptr, nullptr, ctx->hb.get(), true, eps1, psi};
    return build_blocks(ctx, keys_of(V, n), n_orb, p, nullptr);
    GUARD_END(nullptr)
}

void* dq_vv_hb_rows(void* c, const uint64_t* V, int64_t n, int n_orb, double eps1,
                    const int64_t* rows, int64_t n_rows) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    auto keys = keys_of(V, n);
    Map mv;
    mv.build(keys, true);
    Ham H(ctx->I);
    std::vector<std::vector<Trip>> per(n_rows);
#pragma omp parallel for schedule(dynamic)
    for (int64_t t = 0; t < n_rows; ++t) {
        const u32 row = (u32)rows[t];
        const Key bra = keys[row];
        const double hd = H.diag(bra);
        if (std::abs(hd) > kElemThresh) per[t].push_back({row, row, hd});
        auto visit = [&](Key ket) {
            long j = mv.get(ket);
            if (j < 0) return;
            const double h = H.elem(bra, ket);
            if (std::abs(h) <= kElemThresh) return;
            per[t].push_back({row, (u32)j, h});
        };
        singles(bra, n_orb, visit);
        doubles_hb(bra, n_orb, *ctx->hb, eps1, visit);
    }
    std::vector<Trip> all;
    for (auto& p : per) all.insert(all.end(), p.begin(), p.end());
    auto* r = new dq::Result;
    canon(all, r->a);
    r->a.nr = r->a.nc = (u32)n;
    return r;
    GUARD_END(nullptr)
}

// Downfolding H_eff = H_VV + H_VP D^-1 H_PV (ham_eff.cpp:35-233).
void* dq_get_ham_eff(const uint32_t* vv_r, const uint32_t* vv_c, const double* vv_v,
                     int64_t vv_nnz, uint32_t vv_nr, uint32_t vv_nc,
                     const uint32_t* vp_r, const uint32_t* vp_c, const double* vp_v,
                     int64_t vp_nnz, uint32_t vp_nr, uint32_t vp_nc,
                     const double* hpp, int64_t n_p, double e_ref, int reg_sigma,
                     double eps) {
    GUARD_BEGIN
    (void)vv_nc;
    auto* r = new dq::Result;
    std::vector<Trip> vv(vv_nnz);
    for (int64_t t = 0; t < vv_nnz; ++t) vv[t] = {vv_r[t], vv_c[t], vv_v[t]};
    if (n_p == 0) {  // ham_eff.cpp:72-77
        canon(vv, r->a);
        r->a.nr = vv_nr;
        r->a.nc = vv_nc;
        return r;
    }
    if (vp_nc != (uint32_t)n_p) throw std::invalid_argument("H_VP columns != h_pp_diag size");
    const u32 nv = vv_nr ? vv_nr : vp_nr;
    if (vp_nr != nv) throw std::invalid_argument("H_VP rows != H_VV rows");
    // CSR and CSC views of H_VP with duplicates merged (ham_utils.cpp:183-302)
    std::vector<Trip> vp(vp_nnz);
    for (int64_t t = 0; t < vp_nnz; ++t) {
        if (vp_r[t] >= nv) throw std::out_of_range("coo_to_csr: row index out of bounds");
        if (vp_c[t] >= (u32)n_p) throw std::out_of_range("coo_to_csc: column index out of bounds");
        vp[t] = {vp_r[t], vp_c[t], vp_v[t]};
    }
    dq::Coo rowm;
    canon(vp, rowm);  // row-major, unique
    const size_t m = rowm.vals.size();
    std::vector<size_t> rp(nv + 1, 0), cp(n_p + 1, 0);
    for (size_t t = 0; t < m; ++t) { rp[rowm.rows[t] + 1]++; cp[rowm.cols[t] + 1]++; }
    for (u32 i = 0; i < nv; ++i) rp[i + 1] += rp[i];
    for (int64_t k = 0; k < n_p; ++k) cp[k + 1] += cp[k];
    std::vector<u32> crow(m);
    std::vector<double> cval(m);
    {
        std::vector<size_t> fill(cp.begin(), cp.end() - 1);
        for (size_t t = 0; t < m; ++t) {  // rows ascending inside each column
            const size_t at = fill[rowm.cols[t]]++;
            crow[at] = rowm.rows[t];
            cval[at] = rowm.vals[t];
        }
    }
    std::vector<double> dinv(n_p);
    for (int64_t k = 0; k < n_p; ++k) {  // ham_eff.cpp:35-56
        const double d = e_ref - hpp[k];
        dinv[k] = reg_sigma ? d / (d * d + eps * eps) : 1.0 / (d + std::copysign(eps, d));
    }
    std::vector<char> skip(n_p, 0);
    for (int64_t k = 0; k < n_p; ++k) {  // column screening, ham_eff.cpp:93-106
        double s = 0.0;
        for (size_t t = cp[k]; t < cp[k + 1]; ++t) s += cval[t] * cval[t];
        if (std::abs(dinv[k]) * s < 1e-12) skip[k] = 1;
    }
    // Gustavson row accumulation, k ascending (ham_eff.cpp:175-221)
    std::vector<Trip> add;
    std::vector<double> acc(nv, 0.0);
    std::vector<char> hit(nv, 0);
    std::vector<u32> touched;
    for (u32 i = 0; i < nv; ++i) {
        touched.clear();
        for (size_t t = rp[i]; t < rp[i + 1]; ++t) {
            const u32 k = rowm.cols[t];
            if (skip[k]) continue;
            for (size_t q = cp[k]; q < cp[k + 1]; ++q)
                if (!hit[crow[q]]) { hit[crow[q]] = 1; touched.push_back(crow[q]); }
            const double a = rowm.vals[t];
            if (a == 0.0) continue;
            const double s = dinv[k];
            if (s == 0.0) continue;
            const double as = a * s;
            for (size_t q = cp[k]; q < cp[k + 1]; ++q) acc[crow[q]] += as * cval[q];
        }
        std::sort(touched.begin(), touched.end());
        for (u32 j : touched) { add.push_back({i, j, acc[j]}); acc[j] = 0.0; hit[j] = 0; }
    }
    // H_eff = H_VV + H_add, dropping |v| <= 1e-15 (ham_utils.cpp:330-442)
    dq::Coo vvc;
    canon(vv, vvc);
    size_t x = 0, y = 0;
    auto push = [&](u32 rr, u32 cc, double v) {
        if (std::abs(v) > kElemThresh) { r->a.rows.push_back(rr); r->a.cols.push_back(cc); r->a.vals.push_back(v); }
    };
    while (x < vvc.vals.size() || y < add.size()) {
        if (y == add.size() || (x < vvc.vals.size() &&
            (vvc.rows[x] < add[y].r || (vvc.rows[x] == add[y].r && vvc.cols[x] < add[y].c)))) {
            if (vvc.rows[x] < nv) push(vvc.rows[x], vvc.cols[x], vvc.vals[x]);
            ++x;
        } else if (x == vvc.vals.size() || add[y].r < vvc.rows[x] ||
                   (add[y].r == vvc.rows[x] && add[y].c < vvc.cols[x])) {
            push(add[y].r, add[y].c, add[y].v);
            ++y;
        } else {
            push(add[y].r, add[y].c, vvc.vals[x] + add[y].v);
            ++x; ++y;
        }
    }
    r->a.nr = r->a.nc = nv;
    return r;
    GUARD_END(nullptr)
}

// Local connectivity rows (local_conn.cpp:36-142): diagonal, singles kept
// above max(eps1, 1e-15) when heat-bath is on, doubles above 1e-15.
void* dq_local_connections(void* c, const uint64_t* d, int64_t n, int n_orb, int use_hb,
                           double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (use_hb && !ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    Ham H(ctx->I);
    auto keys = keys_of(d, n);
    const double sth = use_hb ? std::max(eps1, kElemThresh) : kElemThresh;
    std::vector<std::vector<std::pair<Key, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 32)
    for (int64_t i = 0; i < n; ++i) {
        const Key bra = keys[i];
        auto& out = rows[i];
        const double hd = H.diag(bra);
        if (std::abs(hd) > kElemThresh) out.push_back({bra, hd});
        singles(bra, n_orb, [&](Key k) {
            const double v = H.elem(bra, k);
            if (std::abs(v) > sth) out.push_back({k, v});
        });
        auto dv = [&](Key k) {
            const double v = H.elem(bra, k);
            if (std::abs(v) > kElemThresh) out.push_back({k, v});
        };
        if (use_hb) doubles_hb(bra, n_orb, *ctx->hb, eps1, dv);
        else doubles(bra, n_orb, dv);
    }
    auto* r = new dq::Result;
    r->offsets.push_back(0);
    for (auto& row : rows) {
        for (auto& [k, v] : row) { r->dets.push_back(k.a); r->dets.push_back(k.b); r->values.push_back(v); }
        r->offsets.push_back((int32_t)r->values.size());
    }
    return r;
    GUARD_END(nullptr)
}

// <Psi|H|Psi> on a fixed basis (local_conn.cpp:148-229).
int dq_variational_energy(void* c, const uint64_t* d, int64_t n, const double* co,
                          int n_orb, int use_hb, double eps1, double* out) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (n == 0) { *out = 0.0; return 0; }
    if (use_hb && !ctx->hb)
        throw std::invalid_argument("compute_variational_energy: Heat-Bath mode requires non-null hb_table");
    Ham H(ctx->I);
    auto keys = keys_of(d, n);
    Map mv;
    mv.build(keys, false);
    const double sth = use_hb ? std::max(eps1, kElemThresh) : kElemThresh;
    double e = 0.0;
#pragma omp parallel for schedule(dynamic, 32) reduction(+ : e)
    for (int64_t i = 0; i < n; ++i) {
        const Key bra = keys[i];
        const double ci = co[i];
        if (ci * ci < 1e-12) continue;
        double sig = 0.0;
        const double hd = H.diag(bra);
        if (std::abs(hd) > kElemThresh) sig += hd * ci;
        auto acc = [&](Key k, double h) {
            long j = mv.get(k);
            if (j >= 0) sig += h * co[j];
        };
        singles(bra, n_orb, [&](Key k) {
            const double v = H.elem(bra, k);
            if (std::abs(v) > sth) acc(k, v);
        });
        auto dv = [&](Key k) {
            const double v = H.elem(bra, k);
            if (std::abs(v) > kElemThresh) acc(k, v);
        };
        if (use_hb) doubles_hb(bra, n_orb, *ctx->hb, eps1, dv);
        else doubles(bra, n_orb, dv);
        e += ci * sig;
    }
    *out = e;
    return 0;
    GUARD_END(-1)
}

// EN-PT2 split into internal and external parts (local_conn.cpp:247-418).
int dq_pt2(void* c, const uint64_t* d, int64_t n, const double* co, int n_orb,
           double e_ref, int use_hb, double eps1, double* out3) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (use_hb && !ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    out3[0] = out3[1] = out3[2] = 0.0;
    if (n == 0) return 0;
    Ham H(ctx->I);
    auto keys = keys_of(d, n);
    Map mv;
    mv.build(keys, false);
    auto guard = [](double den) {
        if (std::abs(den) < 1e-15) den = den >= 0.0 ? 1e-15 : -1e-15;
        return den;
    };
    double internal = 0.0;
    std::unordered_map<Key, double, KeyHash> ext;
    for (int64_t i = 0; i < n; ++i) {
        const Key bra = keys[i];
        const double ci = co[i];
        if (ci * ci < 1e-15) continue;
        const double hii = H.diag(bra);
        double sig = hii * ci;
        auto inner = [&](Key k) {
            long j = mv.get(k);
            if (j < 0) return;
            const double h = H.elem(bra, k);
            if (std::abs(h) > kElemThresh) sig += h * co[j];
        };
        singles(bra, n_orb, inner);
        doubles(bra, n_orb, inner);
        const double res = sig - e_ref * ci;
        internal += (res * res) / guard(e_ref - hii);
        auto outer = [&](Key k) {
            if (mv.get(k) >= 0) return;
            const double h = H.elem(bra, k);
            if (std::abs(h) <= kElemThresh) return;
            if (std::abs(h * ci) < eps1) return;
            ext[k] += h * ci;
        };
        singles(bra, n_orb, outer);
        if (use_hb) {
            const double amp = std::max(std::abs(ci), 1e-12);
            doubles_hb(bra, n_orb, *ctx->hb, eps1 / amp, outer);
        } else {
            doubles(bra, n_orb, outer);
        }
    }
    double external = 0.0;
    for (auto& [k, v] : ext) external += (v * v) / guard(e_ref - H.diag(k));
    out3[0] = internal;
    out3[1] = external;
    out3[2] = (double)ext.size();
    return 0;
    GUARD_END(-1)
}

void* dq_gen_connected(const uint64_t* d, int64_t n, int n_orb) {
    GUARD_BEGIN
    std::unordered_set<Key, KeyHash> s;
    for (auto k : keys_of(d, n)) {
        singles(k, n_orb, [&](Key x) { s.insert(x); });
        doubles(k, n_orb, [&](Key x) { s.insert(x); });
    }
    std::vector<Key> v(s.begin(), s.end());
    std::sort(v.begin(), v.end());
    auto* r = new dq::Result;
    put_keys(v, r->dets);
    return r;
    GUARD_END(nullptr)
}

// P = connected(V) \ V, optionally screened (ham_utils.cpp:546-701).
void* dq_gen_perturbative(void* c, const uint64_t* V, int64_t n, int n_orb,
                          const double* psi, int mode, double eps1) {
    GUARD_BEGIN
    auto keys = keys_of(V, n);
    Map mv;
    mv.build(keys, true);
    std::unordered_set<Key, KeyHash> s;
    auto* ctx = (Ctx*)c;
    if (mode == 0) {
        for (auto k : keys) {
            auto f = [&](Key x) { if (mv.get(x) < 0) s.insert(x); };
            singles(k, n_orb, f);
            doubles(k, n_orb, f);
        }
    } else {
        if (!ctx || !ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
        Ham H(ctx->I);
        for (int64_t i = 0; i < n; ++i) {
            const Key bra = keys[i];
            singles(bra, n_orb, [&](Key k) {
                const double h = H.elem(bra, k);
                if (std::abs(h) <= kElemThresh) return;
                if (mode == 2 && std::abs(h * psi[i]) < eps1) return;
                s.insert(k);
            });
            double cut = eps1;
            if (mode == 2) cut = eps1 / std::max(std::abs(psi[i]), 1e-12);
            doubles_hb(bra, n_orb, *ctx->hb, cut, [&](Key k) { s.insert(k); });
        }
        for (auto k : keys) s.erase(k);
    }
    std::vector<Key> v(s.begin(), s.end());
    std::sort(v.begin(), v.end());
    auto* r = new dq::Result;
    put_keys(v, r->dets);
    return r;
    GUARD_END(nullptr)
}

// Determinant batch features for the neural models, restated from
// det_batch.cpp:184-318 (checks and their messages in the same order, then
// per determinant: occupied list, excitation rank, phase, hole/particle
// lists).  The phase applies the holes highest first, then the particles
// lowest first, each flipping the sign by the parity of the occupied
// orbitals below it (det_batch.cpp:61-98).
int dq_prepare_det_batch(const uint64_t* dets, int64_t B, const uint64_t* ref,
                         int n_orb, int n_alpha, int n_beta, int kmax, int flags,
                         int32_t* occ, int8_t* kout, int8_t* phase, int32_t* holes,
                         int32_t* parts, uint8_t* hp_mask, int32_t* holes_pos,
                         int32_t* parts_pos) {
    GUARD_BEGIN
    const bool need_hp = flags & 4, need_pos = flags & 8, need_phase = flags & 2;
    const bool need_k = (flags & 1) || need_hp;
    if (n_orb < 0 || n_orb > 64) throw std::invalid_argument("n_orb out of range [0,64]");
    if (!dets || !occ) throw std::invalid_argument("null pointer in required outputs");
    if (need_pos && !need_hp) throw std::invalid_argument("need_hp_pos requires need_hp");
    if (need_hp && kmax < 0) throw std::invalid_argument("kmax must be non-negative");
    const u64 m = n_orb == 64 ? ~0ull : ((1ull << n_orb) - 1);
    const u64 ra = ref[0], rb = ref[1];
    const int ne = n_alpha + n_beta;
    // position of a spin orbital in the reference's occupied list (alpha
    // ascending, then beta) or in its virtual list (the rest, ascending)
    auto below = [](u64 x, int o) { return popc(x & ((1ull << o) - 1)); };
    auto occ_pos = [&](int so) {
        return so < n_orb ? below(ra & m, so) : n_alpha + below(rb & m, so - n_orb);
    };
    auto vir_pos = [&](int so) {
        return so < n_orb ? so - below(ra & m, so) : so - n_alpha - below(rb & m, so - n_orb);
    };
    if (need_pos && (popc(ra & m) != n_alpha || popc(rb & m) != n_beta))
        throw std::invalid_argument("reference electron count mismatch");
    auto spin_phase = [](u64 r, u64 d, u64 mk) {
        r &= mk;
        d &= mk;
        u64 h = r & ~d, p = d & ~r, o = r;
        if (popc(h) != popc(p)) throw std::invalid_argument("holes != parts in spin channel");
        int par = 0;
        for (int q = 63; q >= 0; --q)
            if ((h >> q) & 1) {
                par += popc(o & ((1ull << q) - 1));
                o ^= 1ull << q;
            }
        for (int q = 0; q < 64; ++q)
            if ((p >> q) & 1) {
                par += popc(o & ((1ull << q) - 1));
                o ^= 1ull << q;
            }
        return (par & 1) ? -1 : 1;
    };
    for (int64_t i = 0; i < B; ++i) {
        const u64 a = dets[2 * i], b = dets[2 * i + 1];
        if ((a & ~m) || (b & ~m)) throw std::invalid_argument("det bits outside n_orb range");
        if (popc(a) != n_alpha || popc(b) != n_beta)
            throw std::invalid_argument("electron count mismatch");
        int32_t* orow = occ + i * ne;
        int c = 0;
        for (int o = 0; o < n_orb; ++o)
            if ((a >> o) & 1) orow[c++] = o;
        for (int o = 0; o < n_orb; ++o)
            if ((b >> o) & 1) orow[c++] = o + n_orb;
        const u64 ha = ra & ~a & m, hb = rb & ~b & m;
        const int kk = popc(ha) + popc(hb);
        if (need_k) {
            if (!kout) throw std::invalid_argument("k_out is null");
            kout[i] = (int8_t)std::min(kk, 127);
        }
        if (need_phase) {
            if (!phase) throw std::invalid_argument("phase_out is null");
            phase[i] = (int8_t)(spin_phase(ra, a, m) * spin_phase(rb, b, m));
        }
        if (!need_hp) continue;
        if (!holes || !parts || !hp_mask) throw std::invalid_argument("hp outputs are null");
        if (need_pos && (!holes_pos || !parts_pos))
            throw std::invalid_argument("pos outputs are null");
        int32_t* hrow = holes + i * kmax;
        int32_t* prow = parts + i * kmax;
        std::vector<int> hl, pl;   // holes alpha then beta, each highest first;
        for (int o = n_orb - 1; o >= 0; --o)   // particles lowest first
            if ((ha >> o) & 1) hl.push_back(o);
        for (int o = n_orb - 1; o >= 0; --o)
            if ((hb >> o) & 1) hl.push_back(o + n_orb);
        const u64 pa = a & ~ra & m, pb = b & ~rb & m;
        for (int o = 0; o < n_orb; ++o)
            if ((pa >> o) & 1) pl.push_back(o);
        for (int o = 0; o < n_orb; ++o)
            if ((pb >> o) & 1) pl.push_back(o + n_orb);
        for (int j = 0; j < kmax; ++j) {
            hrow[j] = j < (int)hl.size() ? hl[j] : -1;
            prow[j] = j < (int)pl.size() ? pl[j] : -1;
            hp_mask[i * kmax + j] = j < std::min(kk, kmax);
            if (need_pos) {
                holes_pos[i * kmax + j] = j < (int)hl.size() ? occ_pos(hl[j]) : -1;
                parts_pos[i * kmax + j] = j < (int)pl.size() ? vir_pos(pl[j]) : -1;
            }
        }
    }
    return 0;
    GUARD_END(-1)
}

}  // extern "C"

DQ_RESULT_ACCESSORS
