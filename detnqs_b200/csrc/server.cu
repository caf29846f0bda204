// server.cu -- device-resident request loop with continuous batching.
//
// The reference rebuilds H on the host for every outer iteration and applies
// it through SciPy inside a pure_callback (detnqs/operator/kernel.py:48-84);
// each call is one request served alone.  Here a server keeps integral
// contexts, screening tables and the screened H_VV blocks resident in HBM
// between requests and serves two kinds of request:
//
//   BUILD  (system)       screened H_VV of the system's determinant set
//                         (dnq_build, V->V only) with its FP32 operator copy;
//                         optional psi -> energies as for ELOC;
//   ELOC   (system, psi)  local energies and {psi.H psi, psi.psi} on the
//                         resident H_VV (built first when absent).
//
// Threads: `slots` build workers, each with its own stream, and one
// scheduler.  The scheduler admits arrived requests in arrival order but
// lets later ones pass a request that must wait (continuous batching):
//   * an ELOC on a resident block joins the next grouped launch at once;
//   * a build is admitted when a worker is free and the HBM budget holds its
//     estimate, after evicting least-recently-used resident blocks that no
//     admitted request uses;
//   * while one grouped ELOC launch runs on the device, new ELOC requests
//     collect for the next one, and builds run beside it on their streams.
// A grouped launch = psi upload, FP32 conversion, one grouped H.psi launch
// per (precision, lanes, slots) class, one energy block per request, copies
// back.  Each request's rows are computed exactly as the standalone kernels
// compute them with the same (lanes, slots), so a result does not depend on
// what else is in its group.
//
// No device code here waits on anything; completion is observed with
// cudaEventQuery from the host.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "context.cuh"
#include "ham.cuh"

namespace dnq {
using Clock = std::chrono::steady_clock;
void keep_pool(int device);
namespace {

__device__ __forceinline__ void two_sum_d(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double z = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, z)), __dsub_rn(b, z));
}

struct Pair {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add_prod(double a, double b) {
        const double p = __dmul_rn(a, b);
        const double pe = fma(a, b, -p);
        double s2, e;
        two_sum_d(s, p, s2, e);
        s = s2;
        c = __dadd_rn(c, __dadd_rn(e, pe));
    }
    __device__ __forceinline__ void merge(double os, double oc) {
        double s2, e;
        two_sum_d(s, os, s2, e);
        s = s2;
        c = c + oc + e;
    }
};

struct EnergyDesc {
    const double* x;
    const double* y;
    double* eloc;
    float* x32;   // FP32 copy of x to fill (FP32 requests), else null
    i64 n;
};

__global__ void k_group_to_f32(const EnergyDesc* d) {
    const EnergyDesc e = d[blockIdx.y];
    if (!e.x32) return;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < e.n;
         t += (i64)gridDim.x * blockDim.x)
        e.x32[t] = (float)e.x[t];
}

// One block per request: Dot2 sums of x.y and x.x in a fixed order, and
// eloc = y / x.
__global__ void k_group_energy(const EnergyDesc* d, double* out2) {
    const EnergyDesc e = d[blockIdx.x];
    Pair num, den;
    for (i64 t = threadIdx.x; t < e.n; t += blockDim.x) {
        const double xv = e.x[t], yv = e.y[t];
        num.add_prod(xv, yv);
        den.add_prod(xv, xv);
        e.eloc[t] = yv / xv;
    }
    for (int o = 16; o; o >>= 1) {
        num.merge(__shfl_xor_sync(0xffffffffu, num.s, o), __shfl_xor_sync(0xffffffffu, num.c, o));
        den.merge(__shfl_xor_sync(0xffffffffu, den.s, o), __shfl_xor_sync(0xffffffffu, den.c, o));
    }
    __shared__ double sh[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = num.s; sh[1][w] = num.c; sh[2][w] = den.s; sh[3][w] = den.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Pair a, b;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a.merge(sh[0][k], sh[1][k]);
            b.merge(sh[2][k], sh[3][k]);
        }
        out2[2 * blockIdx.x] = a.s + a.c;
        out2[2 * blockIdx.x + 1] = b.s + b.c;
    }
}

// Pinned host buffer that only grows, at least doubling each time.  A
// replaced buffer is kept until the server closes: cudaFreeHost waits for
// the whole device, which would stall every build in flight.
template <class T>
struct Pinned {
    T* p = nullptr;
    size_t n = 0;
    std::vector<T*> retired;
    void need(size_t count) {
        if (count <= n) return;
        const size_t want = std::max<size_t>(std::max<size_t>(count, 2 * n), 1);
        T* q = nullptr;
        DNQ_CUDA(cudaHostAlloc((void**)&q, want * sizeof(T), cudaHostAllocDefault));
        if (p) retired.push_back(p);
        p = q;
        n = want;
    }
    ~Pinned() {
        if (p) cudaFreeHost(p);
        for (T* q : retired) cudaFreeHost(q);
    }
};

struct SrvSystem {
    dnq_ctx_t ctx = nullptr;
    std::vector<u64> dets;
    i64 n = 0;
    int n_orb = 0, policy = 1, use_hb = 1;
    double eps1 = 1e-6;
    dnq_ham_t H = nullptr;
    i64 bytes = 0;        // device bytes of the resident block
    i64 last_bytes = 0;   // of the last build (estimate of the next)
    unsigned long long last_use = 0;
    int pins = 0;         // admitted ELOC requests reading H
    bool busy = false;    // a build of this system is in flight
};

struct SrvReq {
    i64 id = 0;
    int kind = 0;
    int sys = 0;
    const double* psi = nullptr;
    double* eloc = nullptr;
    int precision = DNQ_F64;
    Clock::time_point t_arr, t_adm, t_done;
    double num = 0.0, den = 0.0;
    i64 nnz = 0;
    i64 reserve = 0;
    int status = DNQ_OK;
    std::string err;
    bool done = false;
    int retries = 0;
};

}  // namespace
}  // namespace dnq

struct dnq_server_s {
    int device = 0;
    dnq::Options opt = dnq::default_options();   // options of the blocks it builds
    dnq::i64 budget = 0;
    int slots = 1;
    int max_group = 64;
    std::mutex mu;
    std::condition_variable cv_sched, cv_work, cv_done;
    std::vector<std::unique_ptr<dnq::SrvSystem>> sys;
    std::unordered_map<dnq::i64, std::unique_ptr<dnq::SrvReq>> reqs;
    dnq::i64 next_id = 1;
    std::deque<dnq::i64> pending, build_q, eloc_q;
    dnq::i64 used = 0, reserved = 0, peak = 0;
    unsigned long long tick = 0;
    int free_slots = 1;
    bool stop = false;
    bool paused = false;   // hold grouped launches (requests still admitted)
    std::vector<std::thread> workers;
    std::vector<cudaStream_t> wstreams;
    std::thread sched;
    // grouped ELOC launch in flight (one at a time)
    cudaStream_t es = nullptr;
    cudaEvent_t gev = nullptr;
    bool g_busy = false;
    std::vector<dnq::i64> g_ids;
    std::vector<dnq::i64> g_off;
    dnq::DBuf<double> gx, gy, geloc, ge2;
    dnq::DBuf<float> gx32;
    dnq::DBuf<unsigned char> gdesc;
    dnq::Pinned<double> pin_in, pin_out, pin_e2;
    dnq::Pinned<unsigned char> pin_desc;
    // statistics
    long long n_done = 0, n_failed = 0, n_evict = 0, n_groups = 0, n_grouped = 0, n_builds = 0;
    double build_s = 0.0, group_s = 0.0;   // worker time in builds; launch -> done of groups
    dnq::Clock::time_point g_t0;
    int max_seen_group = 0;
};

namespace dnq {
namespace {

double secs(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

void finish(dnq_server_s* S, SrvReq* r) {
    r->done = true;
    r->t_done = Clock::now();
    if (r->status == DNQ_OK) ++S->n_done;
    else ++S->n_failed;
    S->cv_done.notify_all();
}

// Estimated device bytes of building system y: the last build's peak, or
// 32 B per entry at up to 2048 entries per row.
i64 estimate(const SrvSystem& y) {
    if (y.last_bytes > 0) return y.last_bytes + y.last_bytes / 2;
    return y.n * std::min<i64>(y.n, 2048) * 32 + y.n * 64;
}

void drop_block(dnq_server_s* S, SrvSystem& y) {
    if (!y.H) return;
    delete y.H;   // stream-ordered frees on the build stream; no host wait
    y.H = nullptr;
    S->used -= y.bytes;
    y.bytes = 0;
}

// Evict least-recently-used idle blocks (not `keep`) until `need` fits.
bool make_room(dnq_server_s* S, i64 need, const SrvSystem* keep) {
    while (S->used + S->reserved + need > S->budget) {
        SrvSystem* victim = nullptr;
        for (auto& p : S->sys) {
            SrvSystem& y = *p;
            if (&y == keep || !y.H || y.pins || y.busy) continue;
            if (!victim || y.last_use < victim->last_use) victim = &y;
        }
        if (!victim) return false;
        drop_block(S, *victim);
        ++S->n_evict;
    }
    return true;
}

void admit(dnq_server_s* S) {
    // systems with an earlier request still waiting: later requests for the
    // same system keep their order behind it
    std::vector<int> held;
    auto is_held = [&](int k) { return std::find(held.begin(), held.end(), k) != held.end(); };
    for (auto it = S->pending.begin(); it != S->pending.end();) {
        SrvReq* r = S->reqs[*it].get();
        SrvSystem& y = *S->sys[r->sys];
        if (y.busy || is_held(r->sys)) {
            if (!is_held(r->sys)) held.push_back(r->sys);
            ++it;
            continue;
        }
        const bool needs_build = r->kind == DNQ_REQ_BUILD || !y.H;
        if (!needs_build) {
            ++y.pins;
            y.last_use = ++S->tick;
            r->t_adm = Clock::now();
            S->eloc_q.push_back(r->id);
            it = S->pending.erase(it);
            continue;
        }
        if (S->free_slots == 0 || (r->kind == DNQ_REQ_BUILD && y.pins > 0)) {
            held.push_back(r->sys);
            ++it;
            continue;
        }
        const i64 need = estimate(y);
        if (need > S->budget) {
            r->status = DNQ_ERR_BUDGET;
            r->err = "request needs more device memory than the server budget";
            finish(S, r);
            it = S->pending.erase(it);
            continue;
        }
        if (!make_room(S, need, &y)) {
            held.push_back(r->sys);
            ++it;
            continue;
        }
        y.busy = true;
        r->reserve = need;
        S->reserved += need;
        r->t_adm = Clock::now();
        --S->free_slots;
        S->build_q.push_back(r->id);
        it = S->pending.erase(it);
        S->cv_work.notify_one();
    }
}

void launch_group(dnq_server_s* S) {
    const int take = std::min<int>((int)S->eloc_q.size(), S->max_group);
    S->g_ids.assign(S->eloc_q.begin(), S->eloc_q.begin() + take);
    S->eloc_q.erase(S->eloc_q.begin(), S->eloc_q.begin() + take);
    S->g_off.assign(take + 1, 0);
    i64 max_rows = 0;
    for (int k = 0; k < take; ++k) {
        const SrvReq* r = S->reqs[S->g_ids[k]].get();
        const i64 n = S->sys[r->sys]->n;
        S->g_off[k + 1] = S->g_off[k] + n;
        max_rows = std::max(max_rows, n);
    }
    const i64 R = S->g_off[take];
    cudaStream_t s = S->es;
    if ((i64)S->gx.n < R) {
        S->gx.alloc(R, s);
        S->gy.alloc(R, s);
        S->geloc.alloc(R, s);
        S->gx32.alloc(R, s);
    }
    if ((i64)S->ge2.n < 2 * take) S->ge2.alloc(2 * take, s);
    S->pin_in.need(R);
    S->pin_out.need(R);
    S->pin_e2.need(2 * take);
    for (int k = 0; k < take; ++k) {
        const SrvReq* r = S->reqs[S->g_ids[k]].get();
        std::memcpy(S->pin_in.p + S->g_off[k], r->psi, (S->g_off[k + 1] - S->g_off[k]) * 8);
    }
    DNQ_CUDA(cudaMemcpyAsync(S->gx.p, S->pin_in.p, R * 8, cudaMemcpyHostToDevice, s));
    // descriptors: energy/convert first, then H.psi sorted by class
    std::vector<EnergyDesc> ed(take);
    std::map<std::tuple<int, int, int>, std::vector<SpmvDesc>> cls;
    for (int k = 0; k < take; ++k) {
        const SrvReq* r = S->reqs[S->g_ids[k]].get();
        const dnq_ham_s* h = S->sys[r->sys]->H;
        const i64 o = S->g_off[k];
        const bool f32 = r->precision == DNQ_F32 && h->vv.nnz > 0;
        ed[k] = EnergyDesc{S->gx.p + o, S->gy.p + o, S->geloc.p + o, f32 ? S->gx32.p + o : nullptr,
                           h->n_v};
        int G = 4, U = 1;
        spmv_shape(h->opt, h->vv, G, U);
        SpmvDesc d{};
        d.rp = h->vv.row_start();
        d.re = h->vv.row_end();
        d.col = h->vv.col.p;
        d.val = f32 ? (const void*)h->vv.val32.p : (const void*)h->vv.val.p;
        d.xg = f32 ? (const void*)(S->gx32.p + o) : (const void*)(S->gx.p + o);
        d.diag = f32 ? h->diag_op.p : nullptr;
        d.x = S->gx.p + o;
        d.y = S->gy.p + o;
        d.nr = h->n_v;
        d.nnz = h->vv.span();
        cls[{f32 ? DNQ_F32 : DNQ_F64, G, U}].push_back(d);
    }
    size_t bytes = take * sizeof(EnergyDesc);
    for (auto& c : cls) bytes += c.second.size() * sizeof(SpmvDesc);
    S->pin_desc.need(bytes);
    if (S->gdesc.n < bytes) S->gdesc.alloc(bytes, s);
    unsigned char* hp = S->pin_desc.p;
    std::memcpy(hp, ed.data(), take * sizeof(EnergyDesc));
    size_t at = take * sizeof(EnergyDesc);
    std::vector<std::tuple<size_t, int, int, int, int, i64>> launches;
    for (auto& c : cls) {
        i64 mr = 0;
        for (auto& d : c.second) mr = std::max(mr, d.nr);
        std::memcpy(hp + at, c.second.data(), c.second.size() * sizeof(SpmvDesc));
        launches.emplace_back(at, (int)c.second.size(), std::get<0>(c.first), std::get<1>(c.first),
                              std::get<2>(c.first), mr);
        at += c.second.size() * sizeof(SpmvDesc);
    }
    DNQ_CUDA(cudaMemcpyAsync(S->gdesc.p, hp, bytes, cudaMemcpyHostToDevice, s));
    const EnergyDesc* ed_dev = reinterpret_cast<const EnergyDesc*>(S->gdesc.p);
    {
        const dim3 grid((unsigned)std::max<i64>(1, std::min<i64>((max_rows + 255) / 256, 256)),
                        (unsigned)take);
        k_group_to_f32<<<grid, 256, 0, s>>>(ed_dev);
        DNQ_CHECK_LAUNCH();
    }
    for (auto& L : launches) {
        const SpmvDesc* dd = reinterpret_cast<const SpmvDesc*>(S->gdesc.p + std::get<0>(L));
        spmv_grouped(dd, std::get<1>(L), std::get<5>(L), std::get<3>(L), std::get<4>(L),
                     std::get<2>(L), S->device, s);
    }
    k_group_energy<<<take, 256, 0, s>>>(ed_dev, S->ge2.p);
    DNQ_CHECK_LAUNCH();
    DNQ_CUDA(cudaMemcpyAsync(S->pin_out.p, S->geloc.p, R * 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaMemcpyAsync(S->pin_e2.p, S->ge2.p, 2 * take * 8, cudaMemcpyDeviceToHost, s));
    DNQ_CUDA(cudaEventRecord(S->gev, s));
    S->g_busy = true;
    S->g_t0 = Clock::now();
    ++S->n_groups;
    S->n_grouped += take;
    S->max_seen_group = std::max(S->max_seen_group, take);
}

void finish_group(dnq_server_s* S) {
    S->group_s += secs(S->g_t0, Clock::now());
    for (size_t k = 0; k < S->g_ids.size(); ++k) {
        SrvReq* r = S->reqs[S->g_ids[k]].get();
        SrvSystem& y = *S->sys[r->sys];
        const i64 o = S->g_off[k], n = S->g_off[k + 1] - o;
        if (r->eloc) std::memcpy(r->eloc, S->pin_out.p + o, n * 8);
        r->num = S->pin_e2.p[2 * k];
        r->den = S->pin_e2.p[2 * k + 1];
        --y.pins;
        finish(S, r);
    }
    S->g_ids.clear();
    S->g_busy = false;
}

void fail_group(dnq_server_s* S, const std::string& msg) {
    for (auto id : S->g_ids) {
        SrvReq* r = S->reqs[id].get();
        --S->sys[r->sys]->pins;
        r->status = DNQ_ERR_CUDA;
        r->err = msg;
        finish(S, r);
    }
    S->g_ids.clear();
    S->g_busy = false;
}

void scheduler(dnq_server_s* S) {
    (void)cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        if (S->g_busy) {
            const cudaError_t q = cudaEventQuery(S->gev);
            if (q == cudaSuccess) finish_group(S);
            else if (q != cudaErrorNotReady) fail_group(S, cudaGetErrorString(q));
        }
        admit(S);
        if (!S->g_busy && !S->eloc_q.empty() && !S->paused) {
            try {
                launch_group(S);
            } catch (const std::exception& e) {
                fail_group(S, e.what());
            }
        }
        if (S->g_busy) S->cv_sched.wait_for(lk, std::chrono::microseconds(20));
        else S->cv_sched.wait_for(lk, std::chrono::milliseconds(2));
    }
}

void worker(dnq_server_s* S, int slot) {
    (void)cudaSetDevice(S->device);
    cudaStream_t s = S->wstreams[slot];
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] { return S->stop || !S->build_q.empty(); });
        if (S->stop) break;
        const i64 id = S->build_q.front();
        S->build_q.pop_front();
        SrvReq* r = S->reqs[id].get();
        SrvSystem& y = *S->sys[r->sys];
        lk.unlock();
        const auto tb = Clock::now();
        dnq_ham_t H = nullptr;
        g_build_opt = &S->opt;
        int rc = dnq_build(y.ctx, y.dets.data(), y.n, nullptr, 0, nullptr, y.n_orb, y.policy,
                           y.use_hb, y.eps1, 0, s, &H);
        g_build_opt = nullptr;
        std::string err = rc == DNQ_OK ? std::string() : std::string(dnq_last_error());
        i64 bytes = 0;
        if (rc == DNQ_OK) {
            try {
                if (H->vv.nnz > 0 && (!H->vv.f32_ready() ||
                                      H->diag_op.n != (size_t)H->n_v))
                    make_f32(H->vv, s, &H->diag_op);
                DNQ_CUDA(cudaStreamSynchronize(s));
                bytes = (i64)H->bytes();
            } catch (const Error& e) {
                rc = e.code;
                err = e.what();
                delete H;
                H = nullptr;
            }
        }
        lk.lock();
        S->build_s += secs(tb, Clock::now());
        S->reserved -= r->reserve;
        r->reserve = 0;
        ++S->free_slots;
        y.busy = false;
        if (rc == DNQ_OK) {
            drop_block(S, y);   // a rebuild replaces the old block (no readers: pins == 0)
            y.H = H;
            y.bytes = bytes;
            y.last_bytes = std::max<i64>(bytes, (i64)(H->vv.nnz * 28 + y.n * 64));
            S->used += bytes;
            S->peak = std::max(S->peak, S->used + S->reserved);
            y.last_use = ++S->tick;
            r->nnz = H->vv.nnz;
            ++S->n_builds;
            if (r->kind == DNQ_REQ_ELOC || r->psi) {
                ++y.pins;
                S->eloc_q.push_back(id);
            } else {
                finish(S, r);
            }
        } else if (rc == DNQ_ERR_OUT_OF_MEMORY && r->retries < 2) {
            ++r->retries;
            y.last_bytes = std::max<i64>(y.last_bytes, estimate(y) * 2);
            S->pending.push_front(id);
        } else {
            r->status = rc;
            r->err = err;
            finish(S, r);
        }
        S->cv_sched.notify_one();
    }
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_server_create(int device, int64_t budget_bytes, int build_slots, int max_group,
                      dnq_server_t* out) {
    DNQ_API_BEGIN
    require(out, DNQ_ERR_INVALID, "null argument");
    *out = nullptr;
    require(budget_bytes > 0, DNQ_ERR_INVALID, "budget must be positive");
    require(build_slots >= 1 && build_slots <= 64, DNQ_ERR_INVALID, "build slots must be 1..64");
    require(max_group >= 1 && max_group <= 65535, DNQ_ERR_INVALID, "group size must be 1..65535");
    DeviceGuard g(device);
    auto S = std::make_unique<dnq_server_s>();
    S->device = device;
    S->budget = budget_bytes;
    S->slots = build_slots;
    S->free_slots = build_slots;
    S->max_group = max_group;
    // local-energy groups are short: give their blocks priority over the
    // long build kernels so they do not wait behind them
    int lo = 0, hi = 0;
    DNQ_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DNQ_CUDA(cudaStreamCreateWithPriority(&S->es, cudaStreamNonBlocking, hi));
    DNQ_CUDA(cudaEventCreateWithFlags(&S->gev, cudaEventDisableTiming));
    S->wstreams.resize(build_slots);
    for (auto& w : S->wstreams) DNQ_CUDA(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
    {   // own the budget up front: map it into the stream-ordered pool (kept
        // after the free) so builds never wait for the pool to grow
        keep_pool(device);
        size_t fr = 0, tot = 0;
        DNQ_CUDA(cudaMemGetInfo(&fr, &tot));
        const size_t margin = (size_t)4 << 30;
        const size_t want = std::min<size_t>((size_t)budget_bytes, fr > margin ? fr - margin : 0);
        if (want >= ((size_t)1 << 20)) {
            void* p = nullptr;
            if (cudaMallocAsync(&p, want, S->es) == cudaSuccess) {
                DNQ_CUDA(cudaFreeAsync(p, S->es));
            } else {
                (void)cudaGetLastError();
            }
            DNQ_CUDA(cudaStreamSynchronize(S->es));
        }
    }
    dnq_server_s* raw = S.get();
    for (int k = 0; k < build_slots; ++k) S->workers.emplace_back(worker, raw, k);
    S->sched = std::thread(scheduler, raw);
    *out = S.release();
    DNQ_API_END
}

int dnq_server_destroy(dnq_server_t S) {
    DNQ_API_BEGIN
    if (!S) return DNQ_OK;
    DeviceGuard g(S->device);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_sched.notify_all();
    for (auto& t : S->workers) t.join();
    S->sched.join();
    DNQ_CUDA(cudaStreamSynchronize(S->es));
    for (auto& w : S->wstreams) DNQ_CUDA(cudaStreamSynchronize(w));
    for (auto& p : S->sys) drop_block(S, *p);
    S->gx.release(); S->gy.release(); S->geloc.release(); S->ge2.release();
    S->gx32.release(); S->gdesc.release();
    for (auto& w : S->wstreams) DNQ_CUDA(cudaStreamSynchronize(w));
    DNQ_CUDA(cudaStreamSynchronize(S->es));
    for (auto& w : S->wstreams) cudaStreamDestroy(w);
    cudaStreamDestroy(S->es);
    cudaEventDestroy(S->gev);
    delete S;
    DNQ_API_END
}

int dnq_server_add_system(dnq_server_t S, dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                          int n_orb, int policy, int use_heatbath, double eps1, int* sys_id) {
    DNQ_API_BEGIN
    require_narrow(ctx);
    require(S && ctx && dets && sys_id, DNQ_ERR_INVALID, "null argument");
    require(n >= 1, DNQ_ERR_INVALID, "a system needs determinants");
    require(ctx->device == S->device, DNQ_ERR_INVALID, "context lives on another device");
    require(policy == DNQ_POLICY_KNOWN_SETS || policy == DNQ_POLICY_STATIC, DNQ_ERR_INVALID,
            "served builds support the known-sets and static policies");
    if (policy == DNQ_POLICY_STATIC && use_heatbath)
        require(ctx->has_hb, DNQ_ERR_NO_HEATBATH, "Heat-Bath table not initialized");
    auto y = std::make_unique<SrvSystem>();
    y->ctx = ctx;
    y->dets.assign(dets, dets + 2 * n);
    y->n = n;
    y->n_orb = n_orb;
    y->policy = policy;
    y->use_hb = use_heatbath;
    y->eps1 = eps1;
    std::lock_guard<std::mutex> lk(S->mu);
    *sys_id = (int)S->sys.size();
    S->sys.push_back(std::move(y));
    DNQ_API_END
}

int dnq_server_submit(dnq_server_t S, int kind, int sys_id, const double* psi, double* eloc,
                      int precision, int64_t* req_id) {
    DNQ_API_BEGIN
    require(S && req_id, DNQ_ERR_INVALID, "null argument");
    require(kind == DNQ_REQ_BUILD || kind == DNQ_REQ_ELOC, DNQ_ERR_INVALID, "unknown request kind");
    require(kind == DNQ_REQ_BUILD || psi, DNQ_ERR_INVALID, "local energies need psi");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    auto r = std::make_unique<SrvReq>();
    r->kind = kind;
    r->sys = sys_id;
    r->psi = psi;
    r->eloc = eloc;
    r->precision = precision;
    r->t_arr = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        require(sys_id >= 0 && sys_id < (int)S->sys.size(), DNQ_ERR_INVALID, "unknown system");
        r->id = S->next_id++;
        *req_id = r->id;
        S->pending.push_back(r->id);
        S->reqs[r->id] = std::move(r);
    }
    S->cv_sched.notify_one();
    DNQ_API_END
}

int dnq_server_wait(dnq_server_t S, int64_t req_id, double timeout_s, double* out4,
                    int64_t* nnz) {
    DNQ_API_BEGIN
    require(S, DNQ_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(req_id);
    require(it != S->reqs.end(), DNQ_ERR_INVALID, "unknown request");
    SrvReq* r = it->second.get();
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(std::max(0.0, timeout_s)));
    if (!S->cv_done.wait_until(lk, until, [&] { return r->done; }))
        throw Error(DNQ_ERR_TIMEOUT, "request not finished within the timeout");
    if (out4) {
        out4[0] = r->num;
        out4[1] = r->den;
        out4[2] = secs(r->t_arr, r->t_done);
        out4[3] = r->t_adm.time_since_epoch().count() ? secs(r->t_arr, r->t_adm) : 0.0;
    }
    if (nnz) *nnz = r->nnz;
    const int st = r->status;
    const std::string msg = r->err;
    S->reqs.erase(it);
    if (st != DNQ_OK) throw Error(st, msg);
    DNQ_API_END
}

int dnq_server_set_budget(dnq_server_t S, int64_t budget_bytes) {
    DNQ_API_BEGIN
    require(S, DNQ_ERR_INVALID, "null argument");
    require(budget_bytes > 0, DNQ_ERR_INVALID, "budget must be positive");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->budget = budget_bytes;
        make_room(S, 0, nullptr);   // idle blocks above the new budget go now
        S->peak = 0;   // the peak is tracked against the budget now in force
    }
    S->cv_sched.notify_one();
    DNQ_API_END
}

int dnq_server_pause(dnq_server_t S, int paused) {
    DNQ_API_BEGIN
    require(S, DNQ_ERR_INVALID, "null argument");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->paused = paused != 0;
    }
    S->cv_sched.notify_one();
    DNQ_API_END
}

int dnq_server_stats(dnq_server_t S, double* st14) {
    DNQ_API_BEGIN
    require(S && st14, DNQ_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    int resident = 0;
    for (auto& p : S->sys) resident += p->H != nullptr;
    st14[0] = (double)S->n_done;
    st14[1] = (double)S->n_failed;
    st14[2] = (double)S->n_builds;
    st14[3] = (double)S->n_groups;
    st14[4] = S->n_groups ? (double)S->n_grouped / (double)S->n_groups : 0.0;
    st14[5] = (double)S->max_seen_group;
    st14[6] = (double)S->n_evict;
    st14[7] = (double)S->used;
    st14[8] = (double)S->peak;
    st14[9] = (double)resident;
    st14[10] = (double)S->pending.size();
    st14[11] = (double)S->eloc_q.size();
    st14[12] = S->build_s;
    st14[13] = S->group_s;
    DNQ_API_END
}

}  // extern "C"
