// ref_shim.cpp -- extern "C" driver over the reference DetNQS C++ core.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
// sources (csrc/src/**.cpp of wsmxcz/DetNQS, read in place, never copied)
// into oracle/_ref/libdetnqs_ref.so by oracle/Makefile.  It calls the
// reference's public functions exactly as its nanobind bridge does
// (csrc/bridge/bridge.cpp:235-772) and converts results into dq::Result.
#include "dq_api.h"
#include "dq_result.hpp"

#include <detnqs/determinant/det.hpp>
#include <detnqs/determinant/det_batch.hpp>
#include <detnqs/determinant/det_ops.hpp>
#include <detnqs/determinant/det_space.hpp>
#include <detnqs/hamiltonian/build_ham.hpp>
#include <detnqs/hamiltonian/ham_eff.hpp>
#include <detnqs/hamiltonian/ham_eval.hpp>
#include <detnqs/hamiltonian/ham_utils.hpp>
#include <detnqs/hamiltonian/local_conn.hpp>
#include <detnqs/integral/hb_table.hpp>
#include <detnqs/integral/integral_mo.hpp>
#include <detnqs/integral/integral_so.hpp>

#include <cmath>
#include <memory>
#include <stdexcept>

using namespace detnqs;

namespace {

// Mirror of the bridge's IntCtx (bridge.cpp:108-128).
struct Ctx {
    Ctx(const std::string& path, int n) : mo(n), so(mo), ham(so) {
        mo.load_from_fcidump(path);
    }
    IntegralMO mo;
    IntegralSO so;
    HamEval ham;
    std::unique_ptr<HeatBathTable> hb;
};

std::vector<Det> to_dets(const uint64_t* p, int64_t n) {
    std::vector<Det> v;
    v.reserve(n);
    for (int64_t i = 0; i < n; ++i) v.push_back(Det{p[2 * i], p[2 * i + 1]});
    return v;
}

void put_coo(const COOMatrix& m, dq::Coo& c) {
    c.rows = m.rows;
    c.cols = m.cols;
    c.vals = m.vals;
    c.nr = m.n_rows;
    c.nc = m.n_cols;
}

void put_dets(const std::vector<Det>& d, std::vector<uint64_t>& out) {
    out.resize(d.size() * 2);
    for (size_t i = 0; i < d.size(); ++i) {
        out[2 * i] = d[i].alpha;
        out[2 * i + 1] = d[i].beta;
    }
}

dq::Result* blocks_to_result(const HamBlocks& b) {
    auto* r = new dq::Result;
    put_coo(b.H_VV, r->a);
    put_coo(b.H_VP, r->b);
    put_dets(b.map_P.all_dets(), r->dets);
    return r;
}

COOMatrix make_coo(const uint32_t* r, const uint32_t* c, const double* v,
                   int64_t nnz, uint32_t nr, uint32_t nc) {
    COOMatrix m;
    m.rows.assign(r, r + nnz);
    m.cols.assign(c, c + nnz);
    m.vals.assign(v, v + nnz);
    m.n_rows = nr;
    m.n_cols = nc;
    return m;
}

}  // namespace

#define GUARD_BEGIN try {
#define GUARD_END(ret)                 \
    }                                  \
    catch (const std::exception& e) {  \
        dq::g_err = e.what();          \
        return ret;                    \
    }

extern "C" {

void* dq_ctx_from_fcidump(const char* path, int n_orb) {
    GUARD_BEGIN
    return new Ctx(path, n_orb);
    GUARD_END(nullptr)
}

void* dq_ctx_from_arrays(int, const double*, const double*, double) {
    dq::g_err = "reference IntegralMO is loaded from FCIDUMP only";
    return nullptr;
}

void dq_ctx_free(void* c) { delete (Ctx*)c; }
double dq_ctx_e_nuc(void* c) { return ((Ctx*)c)->so.get_e_nuc(); }

int dq_hb_prepare(void* c, double thr) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    ctx->hb = std::make_unique<HeatBathTable>(ctx->so, HBBuildOptions{thr});
    ctx->hb->build();
    return 0;
    GUARD_END(-1)
}

int dq_hb_clear(void* c) {
    ((Ctx*)c)->hb.reset();
    return 0;
}

int64_t dq_hb_row(void* c, int i, int j, int32_t* a, int32_t* b, double* w,
                  int64_t cap) {
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) return -1;
    auto row = ctx->hb->row_view(i, j);
    for (size_t k = 0; k < row.len && (int64_t)k < cap; ++k) {
        a[k] = row.a[k];
        b[k] = row.b[k];
        w[k] = row.w[k];
    }
    return (int64_t)row.len;
}

int dq_analyze(const uint64_t* bra, const uint64_t* ket, int* degree,
               double* phase) {
    auto info = det_ops::analyze_excitation(Det{bra[0], bra[1]},
                                            Det{ket[0], ket[1]});
    *degree = info.degree;
    *phase = info.phase;
    return 0;
}

double dq_compute_elem(void* c, const uint64_t* bra, const uint64_t* ket) {
    return ((Ctx*)c)->ham.compute_elem(Det{bra[0], bra[1]},
                                       Det{ket[0], ket[1]});
}

int dq_ham_diag(void* c, const uint64_t* d, int64_t n, double* out) {
    GUARD_BEGIN
    auto v = get_ham_diag(to_dets(d, n), ((Ctx*)c)->ham);
    for (int64_t i = 0; i < n; ++i) out[i] = v[i];
    return 0;
    GUARD_END(-1)
}

void* dq_get_ham_vv(void* c, const uint64_t* V, int64_t n, int n_orb) {
    GUARD_BEGIN
    auto* r = new dq::Result;
    put_coo(get_ham_vv(to_dets(V, n), ((Ctx*)c)->ham, n_orb), r->a);
    return r;
    GUARD_END(nullptr)
}

void* dq_get_ham_block(void* c, const uint64_t* V, int64_t nv,
                       const uint64_t* P, int64_t np_, int n_orb) {
    GUARD_BEGIN
    auto dv = to_dets(V, nv);
    std::optional<std::span<const Det>> ps;
    std::vector<Det> dp;
    if (P) {
        dp = to_dets(P, np_);
        ps = std::span<const Det>(dp.data(), dp.size());
    }
    return blocks_to_result(get_ham_block(dv, ps, ((Ctx*)c)->ham, n_orb));
    GUARD_END(nullptr)
}

void* dq_get_ham_conn(void* c, const uint64_t* V, int64_t n, int n_orb,
                      int use_hb, double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (use_hb && !ctx->hb)
        throw std::invalid_argument("Heat-Bath table not initialized");
    return blocks_to_result(get_ham_conn(to_dets(V, n), ctx->ham, n_orb,
                                         ctx->hb.get(), eps1, use_hb != 0));
    GUARD_END(nullptr)
}

void* dq_get_ham_conn_amp(void* c, const uint64_t* V, int64_t n,
                          const double* psi, int n_orb, double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    std::vector<double> pv(psi, psi + n);
    return blocks_to_result(get_ham_conn_amp(to_dets(V, n), pv, ctx->ham,
                                             n_orb, ctx->hb.get(), eps1));
    GUARD_END(nullptr)
}

// VV-only static heat-bath rows: the routing of PolicyStaticHB
// (build_ham.cpp:118-149) applied per row exactly as stream_build does
// (build_ham.cpp:256-312), but only the V->V entries are kept so that a
// subset of rows of a large V can be timed and compared.  Built from the
// reference's public pieces: det_ops::for_each_single, for_each_double_hb,
// HamEval::compute_elem and DetMap.
void* dq_vv_hb_rows(void* c, const uint64_t* V, int64_t n, int n_orb,
                    double eps1, const int64_t* rows, int64_t n_rows) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    auto dets = to_dets(V, n);
    const DetMap map_V = DetMap::from_ordered(dets, true);
    std::vector<COOMatrix> per(n_rows);
#pragma omp parallel for schedule(dynamic)
    for (int64_t t = 0; t < n_rows; ++t) {
        const u32 row = (u32)rows[t];
        const Det& bra = dets[row];
        COOMatrix& m = per[t];
        const double hd = ctx->ham.compute_diagonal(bra);
        if (std::abs(hd) > MAT_ELEMENT_THRESH) m.push_back(row, row, hd);
        auto visit = [&](const Det& ket) {
            auto j = map_V.get_idx(ket);
            if (!j) return;
            const double h = ctx->ham.compute_elem(bra, ket);
            if (std::abs(h) <= MAT_ELEMENT_THRESH) return;
            m.push_back(row, *j, h);
        };
        det_ops::for_each_single(bra, n_orb, visit);
        for_each_double_hb(bra, n_orb, *ctx->hb, eps1, visit);
    }
    COOMatrix out;
    for (auto& m : per) {
        out.rows.insert(out.rows.end(), m.rows.begin(), m.rows.end());
        out.cols.insert(out.cols.end(), m.cols.begin(), m.cols.end());
        out.vals.insert(out.vals.end(), m.vals.begin(), m.vals.end());
    }
    (void)sort_and_merge_coo(out);
    out.n_rows = out.n_cols = (u32)n;
    auto* r = new dq::Result;
    put_coo(out, r->a);
    return r;
    GUARD_END(nullptr)
}

void* dq_get_ham_eff(const uint32_t* vv_r, const uint32_t* vv_c,
                     const double* vv_v, int64_t vv_nnz, uint32_t vv_nr,
                     uint32_t vv_nc, const uint32_t* vp_r,
                     const uint32_t* vp_c, const double* vp_v,
                     int64_t vp_nnz, uint32_t vp_nr, uint32_t vp_nc,
                     const double* h_pp, int64_t n_p, double e_ref,
                     int reg_sigma, double epsilon) {
    GUARD_BEGIN
    auto VV = make_coo(vv_r, vv_c, vv_v, vv_nnz, vv_nr, vv_nc);
    auto VP = make_coo(vp_r, vp_c, vp_v, vp_nnz, vp_nr, vp_nc);
    std::vector<double> d(h_pp, h_pp + n_p);
    HeffConfig cfg{reg_sigma ? Regularization::Sigma
                             : Regularization::LinearShift,
                   epsilon, true};
    auto* r = new dq::Result;
    put_coo(get_ham_eff(VV, VP, d, e_ref, cfg), r->a);
    return r;
    GUARD_END(nullptr)
}

void* dq_local_connections(void* c, const uint64_t* d, int64_t n, int n_orb,
                           int use_hb, double eps1) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    const HeatBathTable* hb = nullptr;
    if (use_hb) {
        if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
        hb = ctx->hb.get();
    }
    auto dets = to_dets(d, n);
    auto b = get_local_connections(dets, ctx->ham, n_orb, hb, eps1,
                                   use_hb != 0);
    auto* r = new dq::Result;
    r->offsets.assign(b.offsets.begin(), b.offsets.end());
    put_dets(b.dets, r->dets);
    r->values = b.values;
    return r;
    GUARD_END(nullptr)
}

int dq_variational_energy(void* c, const uint64_t* d, int64_t n,
                          const double* co, int n_orb, int use_hb,
                          double eps1, double* out) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    auto dets = to_dets(d, n);
    *out = compute_variational_energy(
        dets, std::span<const double>(co, n), ctx->ham, n_orb,
        use_hb ? ctx->hb.get() : nullptr, eps1, use_hb != 0);
    return 0;
    GUARD_END(-1)
}

int dq_pt2(void* c, const uint64_t* d, int64_t n, const double* co,
           int n_orb, double e_ref, int use_hb, double eps1, double* out3) {
    GUARD_BEGIN
    auto* ctx = (Ctx*)c;
    if (use_hb && !ctx->hb)
        throw std::invalid_argument("Heat-Bath table not initialized");
    auto dets = to_dets(d, n);
    auto res = compute_pt2(dets, std::span<const double>(co, n), ctx->ham,
                           n_orb, e_ref, use_hb ? ctx->hb.get() : nullptr,
                           eps1, use_hb != 0);
    out3[0] = res.e_pt2_internal;
    out3[1] = res.e_pt2_external;
    out3[2] = (double)res.n_ext;
    return 0;
    GUARD_END(-1)
}

void* dq_gen_connected(const uint64_t* d, int64_t n, int n_orb) {
    GUARD_BEGIN
    auto v = det_space::generate_connected(to_dets(d, n), n_orb);
    auto* r = new dq::Result;
    put_dets(det_space::canonicalize(std::move(v)), r->dets);
    return r;
    GUARD_END(nullptr)
}

void* dq_gen_perturbative(void* c, const uint64_t* V, int64_t n, int n_orb,
                          const double* psi, int mode, double eps1) {
    GUARD_BEGIN
    auto dets = to_dets(V, n);
    const DetMap map_V = DetMap::from_ordered(dets, true);
    auto* r = new dq::Result;
    if (mode == 0) {
        put_dets(det_space::generate_complement(dets, n_orb, map_V, true),
                 r->dets);
        return r;
    }
    auto* ctx = (Ctx*)c;
    if (!ctx->hb) throw std::invalid_argument("Heat-Bath table not initialized");
    std::span<const double> ps;
    if (mode == 2) ps = std::span<const double>(psi, n);
    put_dets(generate_complement_screened(
                 dets, n_orb, map_V, ctx->ham, ctx->hb.get(),
                 mode == 1 ? ScreenMode::Static : ScreenMode::Dynamic, ps,
                 eps1),
             r->dets);
    return r;
    GUARD_END(nullptr)
}

int dq_prepare_det_batch(const uint64_t* dets, int64_t B, const uint64_t* ref,
                         int n_orb, int n_alpha, int n_beta, int kmax, int flags,
                         int32_t* occ, int8_t* k, int8_t* phase, int32_t* holes,
                         int32_t* parts, uint8_t* hp_mask, int32_t* holes_pos,
                         int32_t* parts_pos) {
    GUARD_BEGIN
    det_batch::PrepareOptions opt;   // as bridge.cpp:363-368
    opt.kmax = kmax;
    opt.need_k = (flags & 1) || (flags & 4);
    opt.need_phase = (flags & 2) != 0;
    opt.need_hp = (flags & 4) != 0;
    opt.need_hp_pos = (flags & 8) != 0;
    det_batch::prepare_det_batch(dets, (std::size_t)B, Det{ref[0], ref[1]}, n_orb, n_alpha,
                                 n_beta, opt, occ, k, phase, holes, parts,
                                 reinterpret_cast<bool*>(hp_mask), holes_pos, parts_pos);
    return 0;
    GUARD_END(-1)
}

}  // extern "C"

DQ_RESULT_ACCESSORS
