// local.cu -- matrix-free contraction sigma_i = sum_j H_ij c_j over a fixed
// basis and the variational energy E = sum_i c_i sigma_i
// (compute_variational_energy, local_conn.cpp:148-229).
//
// Same warp-per-row walk as the builder; hits in the basis are accumulated
// per lane with Dot2 (TwoProduct + TwoSum) and merged across the warp, and
// the row energies are summed with Dot2 again, so the result carries about
// twice FP64 precision before the final rounding.

#include "gen.cuh"

namespace dnq {

void check_orbitals(const u64* d, i64 n, int n_orb, cudaStream_t s);
void launch_diag(const dnq_ctx_s* c, const u64* d, i64 n, double* out, cudaStream_t s);

namespace {

constexpr int kWarps = 8;

__device__ __forceinline__ void tsum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double z = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, z)), __dsub_rn(b, z));
}

struct DD {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add_prod(double a, double b) {
        const double p = __dmul_rn(a, b);
        const double pe = fma(a, b, -p);
        double s2, e;
        tsum(s, p, s2, e);
        s = s2;
        c = __dadd_rn(c, __dadd_rn(e, pe));
    }
    __device__ __forceinline__ void merge(double os, double oc) {
        double s2, e;
        tsum(s, os, s2, e);
        s = s2;
        c = __dadd_rn(__dadd_rn(c, oc), e);
    }
};

struct ContractParams {
    CtxView C;
    DetMapView map;
    const u64* V;
    i64 n;
    const double* coeff;
    const double* diag;
    int n_orb;
    double single_thr;
    double cut;
    const i64* plen;
    int* next_row;
    double* part;     // per block (s, c)
    double* sigma;    // optional per-row sigma_i
};

struct ContractSink {
    const ContractParams& P;
    DD acc;
    __device__ explicit ContractSink(const ContractParams& p) : P(p) {}
    __device__ __forceinline__ void step(const Cand& c) {
        if (!c.valid) return;
        const double ah = fabs(c.h);
        if (!(ah > (c.single ? P.single_thr : kElemThresh))) return;
        const long long j = P.map.find(c.a, c.b);
        if (j >= 0) acc.add_prod(c.h, __ldg(&P.coeff[j]));
    }
};

__global__ void __launch_bounds__(kWarps * 32) k_contract(ContractParams P) {
    __shared__ WarpRow rows[kWarps];
    __shared__ double bs[kWarps], bc[kWarps];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpRow& R = rows[w];
    DD etot;   // meaningful in lane 0
    for (;;) {
        int r = 0;
        if (lane == 0) r = atomicAdd(P.next_row, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= P.n) break;
        const double ci = P.coeff[r];
        if (ci * ci < 1e-12) {                  // local_conn.cpp:188
            if (P.sigma && lane == 0) P.sigma[r] = 0.0;
            continue;
        }
        load_row(R, P.V[2 * (i64)r], P.V[2 * (i64)r + 1], P.n_orb);
        ContractSink sink(P);
        enumerate_row(P.C, R, P.plen, P.cut, sink);
        DD sg = sink.acc;
        for (int o = 16; o; o >>= 1) {
            const double os = __shfl_xor_sync(0xffffffffu, sg.s, o);
            const double oc = __shfl_xor_sync(0xffffffffu, sg.c, o);
            sg.merge(os, oc);
        }
        if (lane == 0) {
            const double hd = P.diag[r];
            if (fabs(hd) > kElemThresh) sg.add_prod(hd, ci);
            const double sigma = sg.s + sg.c;
            if (P.sigma) P.sigma[r] = sigma;
            etot.add_prod(ci, sg.s);
            etot.add_prod(ci, sg.c);
        }
        __syncwarp();
    }
    if (lane == 0) { bs[w] = etot.s; bc[w] = etot.c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b;
        for (int k = 0; k < kWarps; ++k) b.merge(bs[k], bc[k]);
        P.part[2 * blockIdx.x] = b.s;
        P.part[2 * blockIdx.x + 1] = b.c;
    }
}

__global__ void k_final(const double* part, int nb, double* out) {
    if (threadIdx.x || blockIdx.x) return;
    DD a;
    for (int k = 0; k < nb; ++k) a.merge(part[2 * k], part[2 * k + 1]);
    *out = a.s + a.c;
}

__global__ void k_prefix(PairTableView T, i64 nrows, double cut, i64* plen) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nrows;
         r += (i64)gridDim.x * blockDim.x) {
        const i64 lo = T.off[r], len = T.off[r + 1] - lo;
        if (cut <= 0.0) { plen[r] = len; continue; }
        i64 L = 0, R = len;
        while (L < R) {
            const i64 mid = L + (R - L) / 2;
            if (fabs(T.v[lo + mid]) >= cut) L = mid + 1; else R = mid;
        }
        plen[r] = L;
    }
}

}  // namespace

// sigma (optional) and E for a fixed basis; returns E on the host.
double contract_energy(dnq_ctx_s* ctx, const u64* Vd, i64 n, const double* cd, int n_orb,
                       bool use_hb, double eps1, double* sigma, cudaStream_t s) {
    DetMap map;
    build_detmap(map, Vd, n, false, s);
    DBuf<double> diag(n, s);
    launch_diag(ctx, Vd, n, diag.p, s);
    ContractParams P{};
    P.C = ctx->view();
    P.map = map.view();
    P.V = Vd;
    P.n = n;
    P.coeff = cd;
    P.diag = diag.p;
    P.n_orb = n_orb;
    P.single_thr = use_hb ? std::max(eps1, kElemThresh) : kElemThresh;   // :176-178
    P.cut = use_hb ? hb_cutoff(ctx, eps1) : full_cutoff();
    DBuf<i64> plen(ctx->tab.n_rows, s);
    k_prefix<<<64, 256, 0, s>>>(P.C.tab, ctx->tab.n_rows, P.cut, plen.p);
    DNQ_CHECK_LAUNCH();
    P.plen = plen.p;
    DBuf<int> next(1, s);
    DNQ_CUDA(cudaMemsetAsync(next.p, 0, 4, s));
    P.next_row = next.p;
    int per_sm = 0;
    DNQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contract, kWarps * 32, 0));
    const int grid = std::max(1, per_sm) * sm_count(ctx->device);
    DBuf<double> part(2 * grid, s), out(1, s);
    P.part = part.p;
    P.sigma = sigma;
    k_contract<<<grid, kWarps * 32, 0, s>>>(P);
    DNQ_CHECK_LAUNCH();
    k_final<<<1, 32, 0, s>>>(part.p, grid, out.p);
    DNQ_CHECK_LAUNCH();
    double e = 0.0;
    DNQ_CUDA(cudaMemcpyAsync(&e, out.p, 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaStreamSynchronize(s));
    return e;
}

}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_variational_energy(dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                           const double* coeffs, int n_orb, int use_heatbath, double eps1,
                           double* out, void* stream) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(ctx && out, DNQ_ERR_INVALID, "null argument");
    require(n >= 0, DNQ_ERR_INVALID, "negative size");
    if (n == 0) { *out = 0.0; return DNQ_OK; }
    require(dets && coeffs, DNQ_ERR_INVALID, "null argument");
    require(n_orb >= 1 && n_orb <= ctx->n, DNQ_ERR_INVALID,
            "n_orb must be in [1, number of orbitals of the integral context]");
    if (use_heatbath)
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH,
                "compute_variational_energy: Heat-Bath mode requires non-null hb_table");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    DIn<u64> d(dets, 2 * n, s);
    DIn<double> c(coeffs, n, s);
    check_orbitals(d.p, n, n_orb, s);
    *out = contract_energy(ctx, d.p, n, c.p, n_orb, use_heatbath != 0, eps1, nullptr, s);
    DNQ_API_END
}

}  // extern "C"
