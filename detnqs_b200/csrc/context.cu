// context.cu -- integral context: upload, derived tables, signed pair table.
#include <atomic>
#include <cmath>
#include <memory>
#include <cstring>
#include <fstream>
#include <sstream>

#include "context.cuh"
#include "prim.cuh"
#include "refsort.cuh"

namespace dnq {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}

void set_last_error(const std::string& msg) { g_last_error = msg; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

double full_cutoff() { return std::nextafter(kElemThresh, 1.0); }

double hb_cutoff(const dnq_ctx_s* c, double eps) {
    const double t = c->hb_thr;
    if (eps <= 0.0) return t;
    return eps > t ? eps : t;
}

namespace {

__host__ __device__ __forceinline__ i64 tri(i64 p, i64 q) {
    return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
}

// (pq|rs) from the packed 8-fold array (integral_mo.hpp:40-49).
__host__ __device__ __forceinline__ double eri_mo(const double* eri, int p, int q,
                                                  int r, int s) {
    return eri[tri(tri(p, q), tri(r, s))];
}

// <mu ka | nu la> with spin zeroing (integral_so.hpp:89-97).
__host__ __device__ __forceinline__ double phys_so(const double* eri, int mu, int ka,
                                                   int nu, int la) {
    if (((mu ^ nu) & 1) || ((ka ^ la) & 1)) return 0.0;
    return eri_mo(eri, mu >> 1, nu >> 1, ka >> 1, la >> 1);
}

__host__ __device__ __forceinline__ double anti_so(const double* eri, int mu, int ka,
                                                   int nu, int la) {
    return phys_so(eri, mu, ka, nu, la) - phys_so(eri, mu, ka, la, nu);
}

// Candidate (a > b) of row (i > j): spins must match (s_i, s_j) in either
// order and {a, b} must avoid {i, j} (hb_table.cpp:107-121).
__device__ __forceinline__ bool candidate_ok(int i, int j, int a, int b) {
    if (a == i || a == j || b == i || b == j) return false;
    const int si = i & 1, sj = j & 1, sa = a & 1, sb = b & 1;
    return (sa == si && sb == sj) || (sa == sj && sb == si);
}

// Row id -> (i, j) with i > j, id = i(i-1)/2 + j.
__device__ __forceinline__ void row_pair(i64 id, int& i, int& j) {
    int ii = (int)floor((1.0 + sqrt(1.0 + 8.0 * (double)id)) * 0.5);
    while ((i64)ii * (ii - 1) / 2 > id) --ii;
    while ((i64)(ii + 1) * ii / 2 <= id) ++ii;
    i = ii;
    j = (int)(id - (i64)ii * (ii - 1) / 2);
}

__global__ void k_table_count(const double* eri, int nso, double thr, i64* counts) {
    const i64 row = blockIdx.x;
    int i, j;
    row_pair(row, i, j);
    const int ncand = nso * (nso - 1) / 2;
    int c = 0;
    for (int t = threadIdx.x; t < ncand; t += blockDim.x) {
        int a, b;
        row_pair(t, a, b);
        if (!candidate_ok(i, j, a, b)) continue;
        if (fabs(anti_so(eri, i, j, a, b)) >= thr) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ int warp_sum[32];
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += warp_sum[w];
        counts[row] = s;
    }
}

// Writes the candidates of row (i, j) with |v| >= thr in generation order
// (a ascending, then b ascending; hb_table.cpp:103-126) at keys / vals:
// key = |v| bits, val = a | b << 8 | signbit(v) << 16.  Called by a whole
// block; returns the number written.
__device__ int gen_row(const double* eri, int nso, double thr, int i, int j, u64* keys,
                       u32* vals) {
    const int ncand = nso * (nso - 1) / 2;
    __shared__ int base;
    __shared__ int wcount[32];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    for (int t0 = 0; t0 < ncand; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        bool keep = false;
        double v = 0.0;
        int a = 0, b = 0;
        if (t < ncand) {
            row_pair(t, a, b);
            if (candidate_ok(i, j, a, b)) {
                v = anti_so(eri, i, j, a, b);
                keep = fabs(v) >= thr;
            }
        }
        // block-ordered compaction: warp ballots in warp order
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wcount[threadIdx.x >> 5] = __popc(m);
        __syncthreads();
        int before = 0;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) before += wcount[w];
        const int pos = base + before + __popc(m & lanemask_lt());
        if (keep) {
            const double w = fabs(v);
            u64 bits;
            memcpy(&bits, &w, 8);
            keys[pos] = bits;
            vals[pos] = (u32)a | ((u32)b << 8) | ((signbit(v) ? 1u : 0u) << 16);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wcount[w];
            base += s;
        }
        __syncthreads();
    }
    return base;
}

__global__ void k_table_fill(const double* eri, int nso, double thr, const i64* off,
                             u64* keys, u32* vals) {
    const i64 row = blockIdx.x;
    int i, j;
    row_pair(row, i, j);
    gen_row(eri, nso, thr, i, j, keys + off[row], vals + off[row]);
}


// Rows whose entries with |v| >= thr contain equal weights are rewritten in
// the reference's order: the candidates are generated again in generation
// order into the scratch (sk, sv at the row's offset) and sorted by the
// restated std::sort.  Rows without ties are already in the unique
// descending order.  One block per table row.
__global__ void k_table_ties(const double* eri, int nso, double thr, const i64* off, u16* ab,
                             double* tv, u64* sk, u32* sv, int* n_fixed) {
    const i64 row = blockIdx.x;
    const i64 lo = off[row], len = off[row + 1] - lo;
    __shared__ i64 plen;
    if (threadIdx.x == 0) {
        i64 L = 0, R = len;
        while (L < R) {
            const i64 mid = L + (R - L) / 2;
            if (fabs(tv[lo + mid]) >= thr) L = mid + 1; else R = mid;
        }
        plen = L;
    }
    __syncthreads();
    const i64 P = plen;
    int tie = 0;
    for (i64 e = 1 + threadIdx.x; e < P; e += blockDim.x)
        tie |= fabs(tv[lo + e]) == fabs(tv[lo + e - 1]);
    if (!__syncthreads_or(tie)) return;
    int i, j;
    row_pair(row, i, j);
    const int got = gen_row(eri, nso, thr, i, j, sk + lo, sv + lo);
    if (threadIdx.x == 0) {
        if (got == P) {
            refsort::sort(refsort::Seq{sk + lo, sv + lo}, (int64_t)P);
            atomicAdd(n_fixed, 1);
        } else {
            plen = 0;     // cannot happen: same candidates, same threshold
        }
    }
    __syncthreads();
    for (i64 e = threadIdx.x; e < plen; e += blockDim.x) {
        double w;
        const u64 bits = sk[lo + e];
        memcpy(&w, &bits, 8);
        const u32 x = sv[lo + e];
        ab[lo + e] = (u16)(x & 0xffffu);
        tv[lo + e] = (x >> 16) ? -w : w;
    }
}

// Sort keys of the table: (row, ~|v| bits), one block per row.
__global__ void k_table_keys(const i64* off, const u64* k, ulonglong2* out) {
    const i64 row = blockIdx.x;
    for (i64 t = off[row] + threadIdx.x; t < off[row + 1]; t += blockDim.x)
        out[t] = make_ulonglong2((u64)row, ~k[t]);
}

__global__ void k_table_keys_back(const ulonglong2* k, i64 n, u64* out) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x)
        out[t] = ~k[t].y;
}

__global__ void k_table_unpack(const u64* keys, const u32* vals, i64 n, u16* ab,
                               double* v) {
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < n;
         t += (i64)gridDim.x * blockDim.x) {
        double w;
        const u64 bits = keys[t];
        memcpy(&w, &bits, 8);
        const u32 x = vals[t];
        ab[t] = (u16)(x & 0xffffu);
        v[t] = (x >> 16) ? -w : w;
    }
}

void build_pair_table(dnq_ctx_s* c, double thr) {
    cudaStream_t s = 0;
    PairTable& T = c->tab;
    const int nso = c->nso;
    const i64 nrows = (i64)nso * (nso - 1) / 2;
    T.n_rows = nrows;
    T.threshold = thr;
    DBuf<i64> counts(nrows + 1, s);
    DNQ_CUDA(cudaMemsetAsync(counts.p, 0, (nrows + 1) * sizeof(i64), s));
    if (nrows > 0) {
        k_table_count<<<(unsigned)nrows, 256, 0, s>>>(c->erid.p, nso, thr, counts.p);
        DNQ_CHECK_LAUNCH();
    }
    T.off.alloc(nrows + 1, s);
    prim::scan<i64, i64, false>(counts.p, T.off.p, nrows + 1, s);
    i64 total = 0;
    DNQ_CUDA(cudaMemcpyAsync(&total, T.off.p + nrows, sizeof(i64), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    T.n_entries = total;
    T.ab.alloc(total, s);
    T.v.alloc(total, s);
    if (total == 0) return;
    DBuf<u64> k0(total, s), k1(total, s);
    DBuf<u32> v0(total, s), v1(total, s);
    k_table_fill<<<(unsigned)nrows, 256, 0, s>>>(c->erid.p, nso, thr, T.off.p, k0.p, v0.p);
    DNQ_CHECK_LAUNCH();
    // Stable descending sort of each row by weight: one ascending radix sort
    // of (row, ~weight bits) over the whole table.
    {
        DBuf<ulonglong2> kk(total, s), ks(total, s);
        k_table_keys<<<(unsigned)nrows, 256, 0, s>>>(T.off.p, k0.p, kk.p);
        DNQ_CHECK_LAUNCH();
        int rb = 1;
        while (rb < 63 && ((i64)1 << rb) < nrows) ++rb;
        const int bits[2] = {rb, 64};
        prim::radix_sort<ulonglong2, u32>(kk.p, ks.p, v0.p, v1.p, total, bits, s);
        k_table_keys_back<<<1024, 256, 0, s>>>(ks.p, total, k1.p);
        DNQ_CHECK_LAUNCH();
    }
    k_table_unpack<<<1024, 256, 0, s>>>(k1.p, v1.p, total, T.ab.p, T.v.p);
    DNQ_CHECK_LAUNCH();
    // Tied weights in the reference's order; k1/v1 serve as the scratch.
    T.tie_rows = 0;
    DBuf<int> nfix(1, s);
    DNQ_CUDA(cudaMemsetAsync(nfix.p, 0, sizeof(int), s));
    k_table_ties<<<(unsigned)nrows, 256, 0, s>>>(c->erid.p, nso, thr, T.off.p, T.ab.p, T.v.p,
                                                  k1.p, v1.p, nfix.p);
    DNQ_CHECK_LAUNCH();
    int nf = 0;
    DNQ_CUDA(cudaMemcpyAsync(&nf, nfix.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    T.tie_rows = nf;
    T.tie_threshold = thr;
}

// Re-orders the tied weights of every row for a heat-bath threshold above
// the table's own (the reference's table then holds only entries >= thr,
// and its sort sees only those).
void order_ties_for(dnq_ctx_s* c, double thr) {
    PairTable& T = c->tab;
    if (T.tie_threshold == thr || T.n_entries == 0) return;
    cudaStream_t s = 0;
    DBuf<u64> sk(T.n_entries, s);
    DBuf<u32> sv(T.n_entries, s);
    DBuf<int> nfix(1, s);
    DNQ_CUDA(cudaMemsetAsync(nfix.p, 0, sizeof(int), s));
    k_table_ties<<<(unsigned)T.n_rows, 256, 0, s>>>(c->erid.p, c->nso, thr, T.off.p, T.ab.p,
                                                     T.v.p, sk.p, sv.p, nfix.p);
    DNQ_CHECK_LAUNCH();
    int nf = 0;
    DNQ_CUDA(cudaMemcpyAsync(&nf, nfix.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    T.tie_rows = nf;
    T.tie_threshold = thr;
}

void upload_tables(dnq_ctx_s* c) {
    const int n = c->n;
    const double* E = c->erip.data();
    std::vector<double> h1(n * n), dss(n * n), dos(n * n);
    std::vector<double> sss((size_t)n * n * n), sos((size_t)n * n * n);
    for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
            h1[p * n + q] = c->h1p[tri(p, q)];
            const double J = eri_mo(E, p, p, q, q);
            dos[p * n + q] = J;
            dss[p * n + q] = J - eri_mo(E, p, q, q, p);
        }
    for (int h = 0; h < n; ++h)
        for (int p = 0; p < n; ++p)
            for (int k = 0; k < n; ++k) {
                const size_t at = ((size_t)h * n + p) * n + k;
                const double J = eri_mo(E, h, p, k, k);
                sos[at] = J;
                sss[at] = J - eri_mo(E, h, k, k, p);
            }
    cudaStream_t s = 0;
    auto up = [&](DBuf<double>& d, const std::vector<double>& h) {
        d.alloc(h.size(), s);
        DNQ_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice, s));
    };
    up(c->h1, h1);
    up(c->dss, dss);
    up(c->dos, dos);
    up(c->sss, sss);
    up(c->sos, sos);
    up(c->erid, c->erip);
    DNQ_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

// Keep memory freed by cudaFreeAsync in the device's default pool instead
// of returning it to the driver at every synchronisation: repeated builds
// then reuse the same pages (process-local runtime setting).
// The device's stream-ordered pool keeps what it has mapped (no release at
// synchronisation), and an allocation never waits on another stream's work
// to reuse memory that stream freed: builds and local-energy groups run on
// separate streams, and such hidden waits chained them into each other.
void keep_pool(int device) {
    cudaMemPool_t pool;
    DNQ_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = ~0ull;
    DNQ_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    int no = 0;
    DNQ_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
}

namespace {

void init_ctx(dnq_ctx_s* c) {
    DeviceGuard g(c->device);
    keep_pool(c->device);
    upload_tables(c);
    // Table holding every entry that can yield a kept element (|v| >= 1e-15
    // covers the strict "> 1e-15" test of unscreened doubles).
    build_pair_table(c, kElemThresh);
}

// FCIDUMP reader with the reference's rules (integral_mo.cpp:48-182).
void load_fcidump(dnq_ctx_s* c, const char* path) {
    std::ifstream f(path);
    if (!f) throw Error(DNQ_ERR_IO, std::string("Cannot open FCIDUMP: ") + path);
    std::string line;
    bool in_nl = false, saw_nl = false;
    std::string nl;
    while (std::getline(f, line)) {
        if (!in_nl && (line.find("&FCI") != std::string::npos ||
                       line.find("&fci") != std::string::npos)) {
            in_nl = true;
            saw_nl = true;
        }
        if (in_nl) {
            nl += line + " ";
            if (line.find("&END") != std::string::npos ||
                line.find("&end") != std::string::npos)
                break;
        }
    }
    if (!saw_nl) throw Error(DNQ_ERR_IO, "No &FCI namelist found in FCIDUMP");
    std::string up = nl;
    for (char& ch : up) ch = (char)toupper((unsigned char)ch);
    auto pos = up.find("NORB=");
    if (pos != std::string::npos) {
        pos += 5;
        while (pos < up.size() && isspace((unsigned char)up[pos])) ++pos;
        size_t e = pos;
        while (e < up.size() && (isdigit((unsigned char)up[e]) || up[e] == '-' || up[e] == '+')) ++e;
        if (e > pos && std::stoi(up.substr(pos, e - pos)) != c->n)
            throw Error(DNQ_ERR_IO, "NORB mismatch: expected " + std::to_string(c->n) +
                                        ", got " + up.substr(pos, e - pos));
    }
    f.clear();
    f.seekg(0);
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
        if (p == 0 && q == 0 && r == 0 && s == 0) c->e_nuc = v;
        else if (r == 0 && s == 0) c->h1p[tri(p - 1, q - 1)] = v;
        else c->erip[tri(tri(p - 1, q - 1), tri(r - 1, s - 1))] = v;
    }
}

dnq_ctx_s* new_ctx(int n_orb, int device, int max_orb = 64) {
    require(n_orb >= 1 && n_orb <= max_orb, DNQ_ERR_INVALID,
            max_orb == 64 ? "Number of orbitals must be in [1, 64]"
                          : "Number of orbitals must be in [1, 128]");
    int ndev = 0;
    DNQ_CUDA(cudaGetDeviceCount(&ndev));
    require(device >= 0 && device < ndev, DNQ_ERR_INVALID, "invalid device ordinal");
    auto* c = new dnq_ctx_s;
    c->device = device;
    c->n = n_orb;
    c->nso = 2 * n_orb;
    const size_t n1 = (size_t)n_orb * (n_orb + 1) / 2;
    c->h1p.assign(n1, 0.0);
    c->erip.assign(n1 * (n1 + 1) / 2, 0.0);
    return c;
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

const char* dnq_last_error(void) { return g_last_error.c_str(); }
int dnq_version(void) { return 100; }
int64_t dnq_launch_count(void) { return g_launches.load(); }

int dnq_ctx_create(int n_orb, const double* h1e, const double* eri, double e_nuc,
                   int device, dnq_ctx_t* out) {
    DNQ_API_BEGIN
    require(out && h1e && eri, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<dnq_ctx_s> c(new_ctx(n_orb, device));
    std::memcpy(c->h1p.data(), h1e, c->h1p.size() * 8);
    std::memcpy(c->erip.data(), eri, c->erip.size() * 8);
    c->e_nuc = e_nuc;
    init_ctx(c.get());
    *out = c.release();
    DNQ_API_END
}

int dnq_ctx_create_fcidump(const char* path, int n_orb, int device, dnq_ctx_t* out) {
    DNQ_API_BEGIN
    require(out && path, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<dnq_ctx_s> c(new_ctx(n_orb, device));
    load_fcidump(c.get(), path);
    init_ctx(c.get());
    *out = c.release();
    DNQ_API_END
}

int dnq_ctx_destroy(dnq_ctx_t ctx) {
    DNQ_API_BEGIN
    if (!ctx) return DNQ_OK;
    DeviceGuard g(ctx->device);
    delete ctx;
    DNQ_CUDA(cudaDeviceSynchronize());
    DNQ_API_END
}

int dnq_ctx_e_nuc(dnq_ctx_t ctx, double* out) {
    DNQ_API_BEGIN
    require(ctx && out, DNQ_ERR_INVALID, "null argument");
    *out = ctx->e_nuc;
    DNQ_API_END
}

int dnq_ctx_device_bytes(dnq_ctx_t ctx, int64_t* out) {
    DNQ_API_BEGIN
    require(ctx && out, DNQ_ERR_INVALID, "null argument");
    *out = ctx->bytes();
    DNQ_API_END
}

int dnq_ctx_create_wide(int n_orb, const double* h1e, const double* eri, double e_nuc,
                        int device, dnq_ctx_t* out) {
    DNQ_API_BEGIN
    require(out && h1e && eri, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<dnq_ctx_s> c(new_ctx(n_orb, device, 128));
    std::memcpy(c->h1p.data(), h1e, c->h1p.size() * 8);
    std::memcpy(c->erip.data(), eri, c->erip.size() * 8);
    c->e_nuc = e_nuc;
    init_ctx(c.get());
    *out = c.release();
    DNQ_API_END
}

int dnq_hb_prepare(dnq_ctx_t ctx, double threshold) {
    DNQ_API_BEGIN
    require(ctx != nullptr, DNQ_ERR_INVALID, "null context");
    DeviceGuard g(ctx->device);
    require(ctx->nso >= 2, DNQ_ERR_INVALID, "HeatBathTable requires n_so >= 2");
    // The resident table keeps |v| >= 1e-15; a lower heat-bath threshold
    // needs the entries in between as well.
    if (threshold < ctx->tab.threshold) build_pair_table(ctx, threshold);
    else order_ties_for(ctx, threshold);
    ctx->has_hb = true;
    ctx->hb_thr = threshold;
    DNQ_API_END
}

int dnq_hb_clear(dnq_ctx_t ctx) {
    DNQ_API_BEGIN
    require(ctx != nullptr, DNQ_ERR_INVALID, "null context");
    ctx->has_hb = false;
    DNQ_API_END
}

int dnq_hb_row(dnq_ctx_t ctx, int i, int j, int32_t* a, int32_t* b, double* w,
               int64_t cap, int64_t* len) {
    DNQ_API_BEGIN
    require(ctx && len, DNQ_ERR_INVALID, "null argument");
    require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    *len = 0;
    if (i == j) return DNQ_OK;
    require(i >= 0 && j >= 0 && i < ctx->nso && j < ctx->nso, DNQ_ERR_RANGE,
            "spin-orbital index out of range");
    DeviceGuard g(ctx->device);
    const i64 r = pair_row(i, j);
    i64 se[2];
    DNQ_CUDA(cudaMemcpy(se, ctx->tab.off.p + r, 2 * sizeof(i64), cudaMemcpyDeviceToHost));
    const i64 n = se[1] - se[0];
    std::vector<u16> ab(n);
    std::vector<double> v(n);
    if (n) {
        DNQ_CUDA(cudaMemcpy(ab.data(), ctx->tab.ab.p + se[0], n * 2, cudaMemcpyDeviceToHost));
        DNQ_CUDA(cudaMemcpy(v.data(), ctx->tab.v.p + se[0], n * 8, cudaMemcpyDeviceToHost));
    }
    i64 k = 0;
    for (i64 t = 0; t < n; ++t) {
        const double wt = std::fabs(v[t]);
        if (!(wt >= ctx->hb_thr)) break;  // rows are sorted by weight
        if (k < cap) {
            if (a) a[k] = ab[t] & 0xff;
            if (b) b[k] = ab[t] >> 8;
            if (w) w[k] = wt;
        }
        ++k;
    }
    *len = k;
    DNQ_API_END
}

}  // extern "C"
