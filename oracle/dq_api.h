/*
 * dq_api.h -- C interface shared by the two CPU checkers under oracle/.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path (detnqs_b200/) may
 * include, link or load anything from oracle/.  Two libraries implement this
 * interface:
 *
 *   oracle/_ref/libdetnqs_ref.so  -- the reference C++ core (DetNQS csrc/src)
 *                                    compiled from its own sources, driven by
 *                                    ref_shim.cpp (build recipe: oracle/Makefile)
 *   oracle/liboracle.so           -- oracle.cpp, an independent CPU
 *                                    restatement of the same algorithm
 *
 * Both are loaded by ctypes (oracle/__init__.py) and compared against each
 * other, against committed golden fixtures and against the CUDA library.
 *
 * Conventions follow the reference bridge (csrc/bridge/bridge.cpp:76-216):
 * determinants are uint64[N][2] = (alpha, beta); COO results are sorted by
 * (row, col) with u32 indices and f64 values.
 */
#ifndef DQ_API_H
#define DQ_API_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error string of the last failing call on this thread ("" if none). */
const char* dq_last_error(void);

/* ---- integral context (IntCtx, bridge.cpp:108-128) ---------------------- */
void*  dq_ctx_from_fcidump(const char* path, int n_orb);
/* Packed arrays in the reference layout (integral_mo.hpp:30-49): h1e has
 * n(n+1)/2 entries, eri has n1e(n1e+1)/2 entries.  Oracle only: the
 * reference keeps its arrays private and is fed through FCIDUMP. */
void*  dq_ctx_from_arrays(int n_orb, const double* h1e, const double* eri,
                          double e_nuc);
void   dq_ctx_free(void* ctx);
double dq_ctx_e_nuc(void* ctx);
int    dq_hb_prepare(void* ctx, double threshold);
int    dq_hb_clear(void* ctx);
/* Heat-bath row {i,j} of the table: writes up to cap entries, returns len. */
int64_t dq_hb_row(void* ctx, int i, int j, int32_t* a, int32_t* b, double* w,
                  int64_t cap);

/* ---- Slater-Condon primitives ------------------------------------------ */
int    dq_analyze(const uint64_t* bra, const uint64_t* ket, int* degree,
                  double* phase);
double dq_compute_elem(void* ctx, const uint64_t* bra, const uint64_t* ket);
int    dq_ham_diag(void* ctx, const uint64_t* dets, int64_t n, double* out);

/* ---- Hamiltonian builders (build_ham.cpp:402-535) ---------------------- */
void* dq_get_ham_vv(void* ctx, const uint64_t* V, int64_t n, int n_orb);
void* dq_get_ham_block(void* ctx, const uint64_t* V, int64_t nv,
                       const uint64_t* P, int64_t np_, int n_orb);
void* dq_get_ham_conn(void* ctx, const uint64_t* V, int64_t n, int n_orb,
                      int use_hb, double eps1);
void* dq_get_ham_conn_amp(void* ctx, const uint64_t* V, int64_t n,
                          const double* psi, int n_orb, double eps1);
/* H_VV rows of a subset of V under the static heat-bath policy
 * (build_ham.cpp:118-149 routing, VV part only). */
void* dq_vv_hb_rows(void* ctx, const uint64_t* V, int64_t n, int n_orb,
                    double eps1, const int64_t* rows, int64_t n_rows);

/* ---- downfolding (ham_eff.cpp:64-233) ----------------------------------- */
void* dq_get_ham_eff(const uint32_t* vv_r, const uint32_t* vv_c,
                     const double* vv_v, int64_t vv_nnz, uint32_t vv_nr,
                     uint32_t vv_nc,
                     const uint32_t* vp_r, const uint32_t* vp_c,
                     const double* vp_v, int64_t vp_nnz, uint32_t vp_nr,
                     uint32_t vp_nc,
                     const double* h_pp, int64_t n_p, double e_ref,
                     int reg_sigma, double epsilon);

/* ---- local connectivity / energies (local_conn.cpp) --------------------- */
void*  dq_local_connections(void* ctx, const uint64_t* dets, int64_t n,
                            int n_orb, int use_hb, double eps1);
int    dq_variational_energy(void* ctx, const uint64_t* dets, int64_t n,
                             const double* c, int n_orb, int use_hb,
                             double eps1, double* out);
int    dq_pt2(void* ctx, const uint64_t* dets, int64_t n, const double* c,
              int n_orb, double e_ref, int use_hb, double eps1, double* out3);

/* ---- determinant spaces (det_space.cpp, ham_utils.cpp:546-701) ---------- */
void* dq_gen_connected(const uint64_t* dets, int64_t n, int n_orb);
/* mode: 0 none, 1 static, 2 dynamic */
void* dq_gen_perturbative(void* ctx, const uint64_t* V, int64_t n, int n_orb,
                          const double* psi, int mode, double eps1);

/* ---- result objects ------------------------------------------------------ */
/* which: 0 = first COO (H_VV / H_eff), 1 = second COO (H_VP),
 *        2 = determinant list (det_P / connected dets),
 *        3 = offsets (local connections), 4 = values (local connections) */
int64_t dq_res_size(void* r, int which);
void    dq_res_coo(void* r, int which, uint32_t* rows, uint32_t* cols,
                   double* vals, uint32_t* shape2);
void    dq_res_dets(void* r, uint64_t* out);
void    dq_res_offsets(void* r, int32_t* out);
void    dq_res_values(void* r, double* out);
void    dq_res_free(void* r);

/* ---- determinant batch features (det_batch.hpp:38-79) -------------------
 * flags: 1 need_k, 2 need_phase, 4 need_hp, 8 need_hp_pos (the bridge's
 * prepare_det_batch, bridge.cpp:347-430, turns need_hp into need_k too).
 * occ int32[B][n_alpha + n_beta]; k, phase int8[B]; holes, parts,
 * holes_pos, parts_pos int32[B][kmax]; hp_mask uint8[B][kmax] (C++ bool).
 * Outputs not asked for may be null.  Returns 0, or -1 with
 * dq_last_error() holding the reference's message. */
int dq_prepare_det_batch(const uint64_t* dets, int64_t B, const uint64_t* ref,
                         int n_orb, int n_alpha, int n_beta, int kmax, int flags,
                         int32_t* occ, int8_t* k, int8_t* phase, int32_t* holes,
                         int32_t* parts, uint8_t* hp_mask, int32_t* holes_pos,
                         int32_t* parts_pos);

#ifdef __cplusplus
}
#endif
#endif
