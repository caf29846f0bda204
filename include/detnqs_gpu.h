/*
 * detnqs_gpu.h -- C ABI of the B200 determinant-space Hamiltonian library
 * (libdetnqs_b200.so).
 *
 * Plain pointers, sizes and status codes only.  Every input pointer may be
 * host memory or device memory of the context's GPU (the library detects
 * which and copies host buffers itself); outputs of known size are written
 * to caller pointers of either kind.  Results of data-dependent size stay in
 * HBM inside a dnq_ham_t handle and are copied out on request.
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Each entry point names the reference interface it replaces (paths inside
 * wsmxcz/DetNQS).  The reference binds those through nanobind
 * (csrc/bridge/bridge.cpp) and re-exports them from detnqs/core.py.
 *
 * Status: 0 on success, otherwise one of DNQ_ERR_*; dnq_last_error() returns
 * the message of the last failure on the calling thread.  Messages for
 * conditions the reference reports keep the reference's wording (for
 * example "Heat-Bath table not initialized", bridge.cpp:303-304).
 */
#ifndef DETNQS_GPU_H
#define DETNQS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dnq_ctx_s* dnq_ctx_t;    /* integrals + tables in HBM (IntCtx) */
typedef struct dnq_ham_s* dnq_ham_t;    /* H_VV / H_VP / P-space in HBM      */
typedef struct dnq_batch_s* dnq_batch_t;  /* many systems, one launch/phase  */
typedef struct dnq_server_s* dnq_server_t;  /* device-resident request loop   */

enum {
    DNQ_OK = 0,
    DNQ_ERR_INVALID = 1,      /* std::invalid_argument in the reference      */
    DNQ_ERR_NO_HEATBATH = 2,  /* heat-bath table required but not prepared  */
    DNQ_ERR_DUPLICATE = 3,    /* duplicate determinant in an ordered set    */
    DNQ_ERR_OUT_OF_MEMORY = 4,
    DNQ_ERR_BUDGET = 5,       /* request exceeds the context's HBM budget   */
    DNQ_ERR_OVERFLOW = 6,     /* an index would not fit in 32 bits          */
    DNQ_ERR_TIMEOUT = 7,      /* a bounded device wait gave up              */
    DNQ_ERR_CUDA = 8,
    DNQ_ERR_IO = 9,           /* FCIDUMP could not be read                  */
    DNQ_ERR_RANGE = 10        /* std::out_of_range in the reference         */
};

/* Screening policies of the row-streamed builder
 * (csrc/src/hamiltonian/build_ham.cpp:78-196). */
enum {
    DNQ_POLICY_KNOWN_SETS = 0,  /* full doubles, route to V or a given set  */
    DNQ_POLICY_STATIC = 1,      /* heat-bath doubles w >= eps1, P discovered */
    DNQ_POLICY_DYNAMIC = 2      /* tau_i = eps1/max(|psi_i|,1e-12)          */
};

/* Value storage of a built block. */
enum { DNQ_F64 = 0, DNQ_F32 = 1 };

const char* dnq_last_error(void);
int dnq_version(void);
/* Number of kernels this library has launched in the process so far
 * (its own kernels; CUB primitives it calls are not counted).  No
 * reference counterpart (instrumentation). */
int64_t dnq_launch_count(void);

/* Stable ascending order of n keys by the radix sort the build uses for
 * determinant sets (no reference counterpart; exposed so that its order can
 * be checked).  words = 1: uint64 keys; words = 2: (alpha, beta) pairs,
 * alpha first.  bits[w] = significant low bits of word w (higher bits must
 * be zero).  order[i] = input position of the i-th key in sorted order.
 * keys and order may be host or device memory. */
int dnq_sort_order(const uint64_t* keys, int64_t n, int words, const int* bits,
                   uint32_t* order, int device, void* stream);

/* ---- integral context ------------------------------------------------------
 * Replaces IntCtx(fcidump_path, num_orb) (bridge.cpp:108-128, :242-248) and
 * IntegralMO (csrc/detnqs/integral/integral_mo.hpp:58-120).  Arrays are in
 * the reference's packed layout: h1e[n(n+1)/2], eri[n1e(n1e+1)/2]. */
int dnq_ctx_create(int n_orb, const double* h1e, const double* eri,
                   double e_nuc, int device, dnq_ctx_t* out);
int dnq_ctx_create_fcidump(const char* path, int n_orb, int device,
                           dnq_ctx_t* out);
int dnq_ctx_destroy(dnq_ctx_t ctx);
int dnq_ctx_e_nuc(dnq_ctx_t ctx, double* out);      /* IntCtx.get_e_nuc   */
int dnq_ctx_device_bytes(dnq_ctx_t ctx, int64_t* out);
/* IntCtx.hb_prepare(threshold) / hb_clear() (hb_table.cpp:39-168). */
int dnq_hb_prepare(dnq_ctx_t ctx, double threshold);
int dnq_hb_clear(dnq_ctx_t ctx);
/* Row {i,j} of the heat-bath table (HeatBathTable::row_view, hb_table.hpp:
 * 155-158): writes min(len, cap) entries sorted by weight descending and
 * returns len in *len.  Weights are |<ij||ab>|. */
int dnq_hb_row(dnq_ctx_t ctx, int i, int j, int32_t* a, int32_t* b,
               double* w, int64_t cap, int64_t* len);

/* ---- Slater-Condon elements ---------------------------------------------- */
/* detnqs.core.get_ham_diag (bridge.cpp:450-457, build_ham.cpp:388-400). */
int dnq_ham_diag(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, double* out,
                 void* stream);
/* HamEval::compute_elem for n (bra, ket) pairs (ham_eval.cpp:33-51). */
int dnq_ham_elems(dnq_ctx_t ctx, const uint64_t* bra, const uint64_t* ket,
                  int64_t n, double* out, void* stream);
/* det_ops::analyze_excitation degree and phase (det_ops.cpp:159-196). */
int dnq_excitations(const uint64_t* bra, const uint64_t* ket, int64_t n,
                    int32_t* degree, double* phase, int device, void* stream);

/* ---- determinant batch features ------------------------------------------
 * detnqs.core.prepare_det_batch (bridge.cpp:347-430; det_batch.cpp:184-318,
 * det_batch.hpp:38-79): for B determinants and a reference `ref` (host
 * uint64[2]), occ int32[B][n_alpha + n_beta] (alpha orbitals ascending,
 * then beta + n_orb ascending); with DNQ_NEED_K the excitation rank
 * k int8[B] (capped at 127); with DNQ_NEED_PHASE the sign int8[B]; with
 * DNQ_NEED_HP (which implies DNQ_NEED_K) holes and parts int32[B][kmax]
 * (-1 padded) and hp_mask uint8[B][kmax]; with DNQ_NEED_HP_POS (requires
 * DNQ_NEED_HP) their positions in the reference's occupied / virtual lists.
 * Buffers may be host or device memory; outputs not asked for may be null.
 * Errors are the reference's std::invalid_argument cases (DNQ_ERR_INVALID
 * with its message), for the first failing determinant in batch order. */
enum { DNQ_NEED_K = 1, DNQ_NEED_PHASE = 2, DNQ_NEED_HP = 4, DNQ_NEED_HP_POS = 8 };

/* ---- batched log-determinant ---------------------------------------------
 * The fused log-det kernels of the reference's XLA FFI module
 * (csrc/ffi/logdet_cuda.cu:187-331, bound by detnqs/models/slogdet.py:
 * slogdet(..., use_fast_kernel=True)).  a holds B row-major n x n matrices,
 * 2 <= n <= 64, in FP64 (precision DNQ_F64) or FP32 (DNQ_F32); sign and
 * logabs (B values each) and grad (B matrices) are in the same type.
 * dnq_slogdet: sign and log|det| by LU with partial pivoting; a matrix whose
 * factorisation meets a zero pivot column gets sign 0 and log|det| -inf.
 * dnq_slogdet_grad: grad = cot_logabs[b] * A_b^{-T} (the gradient of
 * log|det|), 0 for such singular matrices.  Buffers may be host or device
 * memory.  Errors: "N must be in [2, 64]", "Batch size out of int32 range"
 * (B < 1 too), as the reference. */
int dnq_slogdet(const void* a, int64_t B, int n, int precision, void* sign,
                void* logabs, int device, void* stream);
int dnq_slogdet_grad(const void* a, const void* cot_logabs, int64_t B, int n,
                     int precision, void* grad, int device, void* stream);
int dnq_prepare_det_batch(const uint64_t* dets, int64_t B, const uint64_t* ref,
                          int n_orb, int n_alpha, int n_beta, int kmax, int flags,
                          int32_t* occ, int8_t* k, int8_t* phase, int32_t* holes,
                          int32_t* parts, uint8_t* hp_mask, int32_t* holes_pos,
                          int32_t* parts_pos, int device, void* stream);

/* ---- screened Hamiltonian build ------------------------------------------
 * One call covers the four reference builders (build_ham.cpp:402-535):
 *   get_ham_vv      : policy KNOWN_SETS, ext = NULL, want_vp = 0
 *   get_ham_block   : policy KNOWN_SETS, ext = ket set
 *   get_ham_conn    : policy STATIC (use_heatbath 0/1)
 *   get_ham_conn_amp: policy DYNAMIC, psi = amplitudes on V
 * want_vp = 0 keeps only the V->V block (the P set is not materialised).
 * Values are kept in FP64; the FP32 operator copy is made on first use. */
int dnq_build(dnq_ctx_t ctx, const uint64_t* dets_V, int64_t n_V,
              const uint64_t* dets_ext, int64_t n_ext, const double* psi,
              int n_orb, int policy, int use_heatbath, double eps1,
              int want_vp, void* stream, dnq_ham_t* out);
int dnq_ham_destroy(dnq_ham_t h);
/* Library options (no reference counterpart; used by tests to reach every
 * code path with small inputs):
 *   DNQ_OPT_FORCE_WALK  1: route V->V-only builds through the per-row
 *                          candidate walk instead of the string-group
 *                          matcher (both give identical blocks);
 *   DNQ_OPT_ARENA_CHUNK n: entries per warp chunk of the single-pass V->V
 *                          build (0 = default: 8192, and 16384 for
 *                          single builds of at least 64 rows per
 *                          walking warp);
 *   DNQ_OPT_ARENA_CAP   n: arena capacity in entries (0 = automatic); a
 *                          too-small arena falls back to an exact two-pass
 *                          build;
 *   DNQ_OPT_SPMV_LANES  n: lanes per row of H.psi, 0/4/8/16/32 (0 = by the
 *                          average row length);
 *   DNQ_OPT_SPMV_UNROLL n: 4-entry slots each lane keeps in flight, 0/1/2/4
 *                          (0 = by the average row length).  Results do
 *                          not depend on it;
 *   DNQ_OPT_PARTC_GROUPWALK n: 1 walks the short alpha-single groups of
 *                          the string-group matcher's opposite-spin doubles
 *                          one group at a time, 0 packed across the groups of
 *                          a round (default); both give identical blocks,
 *                          entry order too;
 *   DNQ_OPT_BUILD_F32   n: 1 makes V->V-only builds write the FP32 copy of
 *                          the V block and its FP64 diagonal while they
 *                          compact the rows, for handles whose first use is
 *                          an FP32 H.psi (4 bytes per entry more memory);
 *                          0 makes them on first FP32 use (default).  The
 *                          copies are the same either way. */
enum { DNQ_OPT_FORCE_WALK = 1, DNQ_OPT_ARENA_CHUNK = 2, DNQ_OPT_ARENA_CAP = 3,
       DNQ_OPT_SPMV_LANES = 4, DNQ_OPT_SPMV_UNROLL = 5, /* 6: unused */
       DNQ_OPT_PARTC_GROUPWALK = 7, DNQ_OPT_BUILD_F32 = 8 };
int dnq_set_option(int option, int64_t value);
/* The values set by dnq_set_option are process-wide defaults: every handle,
 * batch and server takes a copy when it is created and keeps using its copy,
 * so a later dnq_set_option does not reach objects that exist already.
 * dnq_ham_set_option sets the H.psi shape (DNQ_OPT_SPMV_LANES,
 * DNQ_OPT_SPMV_UNROLL) of one handle. */
int dnq_ham_set_option(dnq_ham_t h, int option, int64_t value);
/* sizes: [0] n_V, [1] nnz(H_VV), [2] n_P, [3] nnz(H_VP),
 *        [4] candidates examined, [5] device bytes held */
int dnq_ham_info(dnq_ham_t h, int64_t* info6);
/* Device time of the build phases, from CUDA events recorded on the build
 * stream (ms): [0] maps + diagonal, [1] count pass, [2] scans/allocation,
 * [3] fill pass, [4] V-row pass (V->V-only builds: long rows compacted in
 * place and row bounds; else the row sort), [5] P discovery + P-row sort, [6] total,
 * [7] unused.  No reference counterpart (instrumentation). */
int dnq_ham_timings(dnq_ham_t h, double* ms8);
/* block 0 = H_VV, 1 = H_VP; COO sorted by (row, col) as in
 * from_coo_matrix (bridge.cpp:173-196).  Any pointer may be NULL. */
int dnq_ham_copy_coo(dnq_ham_t h, int block, uint32_t* rows, uint32_t* cols,
                     double* vals, void* stream);
/* CSR view: row_ptr[n_rows+1] (int64), cols, vals (FP64). */
int dnq_ham_copy_csr(dnq_ham_t h, int block, int64_t* row_ptr, uint32_t* cols,
                     double* vals, void* stream);
int dnq_ham_copy_dets_p(dnq_ham_t h, uint64_t* dets, void* stream);
int dnq_ham_copy_diag(dnq_ham_t h, double* diag, void* stream);
/* <x|H|x> of the P determinants held by h, computed on the device
 * (get_ham_diag(det_P), hamiltonian.py:202-206). */
int dnq_ham_p_diag(dnq_ham_t h, dnq_ctx_t ctx, double* out, void* stream);

/* ---- H.psi / local energy -------------------------------------------------
 * Replaces the SciPy CSR matvec of detnqs/operator/kernel.py:75-78
 * (build_vv_operator) with y = H_VV x on the device.  precision DNQ_F64
 * computes in FP64; DNQ_F32 reads FP32 off-diagonal values and FP32 x with
 * Kahan-compensated FP32 accumulation (each product through one fused
 * multiply-add), adds the FP64 diagonal term in FP64 and writes FP64 y. */
int dnq_ham_spmv(dnq_ham_t h, const double* x, double* y, int precision,
                 void* stream);
/* Proxy operator (kernel.py:127-139):
 *   yv = H_VV xv + H_VP xp ;  yp = H_PV xv + diag_p * xp */
int dnq_ham_proxy_spmv(dnq_ham_t h, const double* xv, const double* xp,
                       const double* diag_p, double* yv, double* yp,
                       int precision, void* stream);
/* One block: 0 -> y = H_VV x, 1 -> y = H_VP x, 2 -> y = H_PV x
 * (the H_VP.dot / H_PV.dot calls of kernel.py:132-133). */
int dnq_ham_block_spmv(dnq_ham_t h, int block, const double* x, double* y,
                       int precision, void* stream);
/* Rayleigh quotient and local energies from one y = H x pass:
 * out2 = {x.Hx, x.x} (compensated FP64 sums); eloc[i] = y_i / x_i
 * (NULL to skip). */
int dnq_ham_local_energy(dnq_ham_t h, const double* x, double* eloc,
                         double* out2, int precision, void* stream);

/* H applied to k amplitude vectors at once (no reference counterpart: the
 * reference applies H to one psi per SciPy call, kernel.py:75-78).  X and Y
 * are n_V x k row-major FP64 arrays (vector j is column j), host or device
 * memory.  The vectors are gathered interleaved, 8 FP32 or 4 FP64 values
 * per 32-byte sector, so one pass over the CSR serves up to 8 (FP32) or 4
 * (FP64) vectors; larger k runs in passes.  Every column equals
 * dnq_ham_spmv of that vector bit for bit (CSR kernel, same lanes per
 * row).  1 <= k <= 1024. */
int dnq_ham_spmv_multi(dnq_ham_t h, const double* X, double* Y, int k,
                       int precision, void* stream);
/* Local energies of k vectors in one pass: out[2j] = x_j.H x_j,
 * out[2j+1] = x_j.x_j (the sums of dnq_ham_local_energy, bit for bit);
 * eloc (n_V x k row-major, may be NULL) = (H x_j)_i / x_ij. */
int dnq_ham_local_energy_multi(dnq_ham_t h, const double* X, double* eloc,
                               double* out, int k, int precision, void* stream);

/* Same result as dnq_ham_local_energy without allocating device memory.
 * No counterpart in the reference: it serves callers that may not allocate
 * on their own -- an XLA custom call (JAX FFI) that runs inside XLA's memory
 * plan, or an application that gives the library a fixed budget.  Its
 * scratch (FP32 copy of x, reduction partials) is a file-scope device array
 * of 4 MiB + 74 KiB that every GPU loading the library holds until exit, so
 * n_V is limited to 1048576 (larger handles are rejected).  x and eloc must
 * be non-overlapping device memory of the handle's GPU (eloc is required; it
 * first receives H x and then y_i / x_i).  out2 may be device memory of that
 * GPU (the call then only enqueues work on the stream) or host memory (the
 * call copies the pair back and waits for the stream).  DNQ_F32 needs the
 * handle's FP32 values to exist (one earlier FP32 call).  The first call on a
 * device sets up the scratch address with that device current: make it
 * before any stream capture; the address is cached per device ordinal and
 * does not survive cudaDeviceReset.  All calls share the scratch: calls
 * that overlap on the GPU race and must be serialised by the caller. */
int dnq_ham_local_energy_noalloc(dnq_ham_t h, const double* x, double* eloc,
                                 double* out2, int precision, void* stream);

/* ---- matrix-free contractions (csrc/src/hamiltonian/local_conn.cpp) ------ */
/* compute_variational_energy (local_conn.cpp:148-229). */
int dnq_variational_energy(dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                           const double* coeffs, int n_orb, int use_heatbath,
                           double eps1, double* out, void* stream);

/* ---- determinant-space generators ----------------------------------------
 * mode -1: gen_connected_dets (det_space.cpp:167-213 + canonicalize): all
 *          singles and doubles of dets, sorted and unique; ctx may be NULL.
 * mode  0: gen_perturbative_dets(mode="none") (det_space.cpp:233-255):
 *          the same minus dets.
 * mode  1: "static"  (ham_utils.cpp:546-701): singles with |h| > 1e-15,
 *          heat-bath doubles with w >= eps1, minus dets.
 * mode  2: "dynamic": singles also need |h psi_i| >= eps1, doubles
 *          w >= eps1 / max(|psi_i|, 1e-12).
 * The sorted result is held by *out: read its size with dnq_ham_info
 * (info[2]) and copy it with dnq_ham_copy_dets_p. */
int dnq_gen_dets(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, int n_orb,
                 const double* psi, int mode, double eps1, int device,
                 void* stream, dnq_ham_t* out);
/* get_local_connections (local_conn.cpp:96-142; bridge.cpp:635-677): per
 * row the diagonal, singles above max(eps1,1e-15) (heat-bath) or 1e-15,
 * doubles above 1e-15.  Sizes via dnq_ham_info (info[2] = total entries),
 * copy with dnq_conn_copy (offsets int32[n+1], dets, values). */
int dnq_local_connections(dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                          int n_orb, int use_heatbath, double eps1,
                          void* stream, dnq_ham_t* out);
int dnq_conn_copy(dnq_ham_t h, int32_t* offsets, uint64_t* dets,
                  double* values, void* stream);
/* compute_pt2 (local_conn.cpp:247-418): out3 = {e_pt2_internal,
 * e_pt2_external, n_ext}. */
int dnq_pt2(dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
            const double* coeffs, int n_orb, double e_ref, int use_heatbath,
            double eps1, double* out3, void* stream);

/* ---- downfolding -----------------------------------------------------------
 * get_ham_eff (ham_eff.cpp:64-233): H_eff = H_VV + H_VP D^-1 H_PV with
 * D_k = e_ref - h_pp[k]; reg_sigma 1 -> d/(d^2+eps^2), 0 -> 1/(d+sgn(d)eps).
 * Inputs are COO triplets (any order, duplicates summed).  precision
 * DNQ_F32 stores H_VP values in FP32 and accumulates each output element
 * with two-sum compensation; D^-1 stays FP64. */
/* Same downfolding from the V and P blocks of a device-resident proxy
 * build (build_effective_hamiltonian, hamiltonian.py:215-281), without
 * copying them to the host.  Returns a new handle holding H_eff. */
int dnq_ham_eff_from(dnq_ham_t proxy, const double* h_pp, double e_ref,
                     int reg_sigma, double epsilon, int precision,
                     void* stream, dnq_ham_t* out);
int dnq_ham_eff(const uint32_t* vv_rows, const uint32_t* vv_cols,
                const double* vv_vals, int64_t vv_nnz, int64_t n_v,
                const uint32_t* vp_rows, const uint32_t* vp_cols,
                const double* vp_vals, int64_t vp_nnz, int64_t n_p,
                const double* h_pp, double e_ref, int reg_sigma,
                double epsilon, int precision, int device, void* stream,
                dnq_ham_t* out);

/* 0.5 (H + H^T) of the V block as a new handle (no reference counterpart:
 * the screened blocks of the dynamic policy, and so H_eff built from them,
 * are not symmetric; eigen-solvers take this symmetric part). */
int dnq_ham_symmetrize(dnq_ham_t h, void* stream, dnq_ham_t* out);

/* ---- batched engine (no reference counterpart) ------------------------------
 * Many independent systems (each with its own integral context and V, any
 * n_orb < 64) built and contracted together: the rows of all systems form
 * one block-diagonal problem and every phase is one launch over all of
 * them.  One step = diagonal, screened V->V build (the same rules and
 * results as dnq_build with want_vp = 0), H.psi on the concatenated psi,
 * and per-system {psi.H psi, psi.psi} plus local energies.  Creation runs
 * one build to size every buffer; afterwards a step allocates nothing and
 * can be captured into a CUDA graph (use_graph = 1, explicit stream; the
 * first such call captures, later calls replay).  A step whose sizes no
 * longer match the plan fails with DNQ_ERR_OVERFLOW.
 * policy: DNQ_POLICY_KNOWN_SETS or DNQ_POLICY_STATIC. */
int dnq_batch_create(int n_sys, const dnq_ctx_t* ctxs, const uint64_t* const* dets,
                     const int64_t* n_dets, const int* n_orb, int policy,
                     int use_heatbath, double eps1, int device, void* stream,
                     dnq_batch_t* out);
int dnq_batch_destroy(dnq_batch_t b);
/* info4 = {n_sys, total rows, nnz, device bytes of the planned buffers} */
int dnq_batch_info(dnq_batch_t b, int64_t* info4);
/* cfg4 = {arena chunk entries, part-C search threshold, lanes per row of
 * H.psi (0 = by row length), 4-entry slots in flight per lane of H.psi
 * (0 = by row length)}: the tunables the autotuner chooses. */
int dnq_batch_set_config(dnq_batch_t b, const int64_t* cfg4);
int dnq_batch_get_config(dnq_batch_t b, int64_t* cfg4);
/* psi: concatenated amplitudes (host or device); eloc (total rows) and
 * energies (2 per system) may be NULL; *step_ms = device time of the step. */
int dnq_batch_step(dnq_batch_t b, const double* psi, double* eloc,
                   double* energies, int precision, int use_graph, void* stream,
                   double* step_ms);
/* H.psi and energies only, on the CSR resident from creation or the last
 * step (the inner loop between rebuilds); same arguments as
 * dnq_batch_step, its own captured graph. */
int dnq_batch_apply(dnq_batch_t b, const double* psi, double* eloc,
                    double* energies, int precision, int use_graph, void* stream,
                    double* step_ms);
/* k amplitude sets of every system in one pass over the resident CSR
 * (dnq_ham_spmv_multi on the block-diagonal batch): X and eloc are
 * total x k row-major (eloc may be NULL), energies n_sys x k x 2 =
 * {psi_j.H psi_j, psi_j.psi_j}; each column equals dnq_batch_apply of that
 * column bit for bit.  Eager (no graph); *step_ms = device time of the
 * H.psi and energy kernels. */
int dnq_batch_apply_multi(dnq_batch_t b, const double* X, double* eloc,
                          double* energies, int k, int precision, void* stream,
                          double* step_ms);
/* Device ms of the phases of the last eager (use_graph = 0) step:
 * {diagonal, build (arena + long rows), scan + compaction (+ FP32 split),
 *  H.psi + energies}. */
int dnq_batch_timings(dnq_batch_t b, double* ms4);
/* Sorted COO (local indices) of one system's block; *nnz always set. */
int dnq_batch_copy_coo(dnq_batch_t b, int sys, uint32_t* rows, uint32_t* cols,
                       double* vals, int64_t* nnz);

/* ---- serving loop (no reference counterpart) --------------------------------
 * A server keeps screened H_VV blocks resident in device memory between
 * requests and serves, for registered systems (context + determinant set):
 *   DNQ_REQ_BUILD  build the system's H_VV (dnq_build, V->V only) and its
 *                  FP32 operator copy; with psi also answers as ELOC;
 *   DNQ_REQ_ELOC   local energies of psi on the resident block (built first
 *                  when absent).
 * build_slots worker threads build on their own streams; local-energy
 * requests are grouped into one launch per (precision, H.psi shape) while the
 * previous group runs (continuous batching).  Builds are admitted while the
 * resident blocks plus the estimates of the builds in flight stay within
 * budget_bytes, evicting least-recently-used idle blocks.  A request's result
 * does not depend on the other requests served with it.
 * psi (n doubles) and eloc (n doubles, may be NULL) are host memory the caller
 * keeps valid until dnq_server_wait returns for the request.
 * Creation maps min(budget, free memory - 4 GiB) into the device's
 * stream-ordered pool, so builds do not wait for the pool to grow. */
enum { DNQ_REQ_BUILD = 0, DNQ_REQ_ELOC = 1 };
int dnq_server_create(int device, int64_t budget_bytes, int build_slots, int max_group,
                      dnq_server_t* out);
int dnq_server_destroy(dnq_server_t s);
/* Copies the determinants; the context must outlive the server. */
int dnq_server_add_system(dnq_server_t s, dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                          int n_orb, int policy, int use_heatbath, double eps1,
                          int* sys_id);
int dnq_server_submit(dnq_server_t s, int kind, int sys_id, const double* psi,
                      double* eloc, int precision, int64_t* req_id);
/* Waits up to timeout_s; DNQ_ERR_TIMEOUT leaves the request pending.  On
 * completion out4 = {psi.H psi, psi.psi, latency s (submit -> done), queue s
 * (submit -> admission)}, *nnz = nnz of the block built by this request (0
 * if none); the request's own status is returned and it is released. */
int dnq_server_wait(dnq_server_t s, int64_t req_id, double timeout_s, double* out4,
                    int64_t* nnz);
/* New admission budget: idle resident blocks above it are evicted at once
 * (least recently used first), blocks in use as soon as later builds need
 * room.  Resets the peak statistic. */
int dnq_server_set_budget(dnq_server_t s, int64_t budget_bytes);
/* paused != 0 holds grouped local-energy launches (requests are still
 * admitted and builds still run); 0 releases them. */
int dnq_server_pause(dnq_server_t s, int paused);
/* st14 = {completed, failed, builds, grouped launches, mean group size,
 *         largest group, evictions, resident bytes, peak bytes (resident +
 *         reserved), resident blocks, requests waiting for admission,
 *         requests ready for the next grouped launch, worker seconds spent
 *         in builds, seconds from launch to completion of grouped launches} */
int dnq_server_stats(dnq_server_t s, double* st14);

/* ---- two-word determinants, up to 128 orbitals (no reference counterpart:
 * the reference's Det holds one uint64 per spin, det.hpp:30-36, and its
 * IntegralMO rejects n > 64, integral_mo.cpp:26-28) ---------------------------
 * A determinant is 4 x uint64: alpha lo, alpha hi, beta lo, beta hi (bit i of
 * a spin string = orbital i); P is sorted by alpha as a 128-bit integer, then
 * beta.  Contexts with more than 64 orbitals are accepted only here; the
 * one-word entry points reject them. */
int dnq_ctx_create_wide(int n_orb, const double* h1e, const double* eri,
                        double e_nuc, int device, dnq_ctx_t* out);
/* Diagonal elements (ham_eval.cpp:53-86) of n two-word determinants. */
int dnq_wide_diag(dnq_ctx_t ctx, const uint64_t* dets, int64_t n, double* out,
                  void* stream);
/* Screened V->{V,P} build of two-word determinants: get_ham_conn with the
 * heat-bath table when psi == NULL (singles kept, doubles w >= eps1), else
 * get_ham_conn_amp (singles |h psi_i| >= eps1, doubles w >= eps1 /
 * max(|psi_i|, 1e-12)); build_ham.cpp:139-196, :256-312, :346-380.  The
 * handle holds H_VV, H_VP and P (dnq_ham_copy_dets_p copies 4 words per
 * determinant; dnq_ham_p_diag gives diag(H_PP)), so dnq_ham_spmv,
 * dnq_ham_proxy_spmv and dnq_ham_eff_from apply to it unchanged. */
int dnq_wide_build(dnq_ctx_t ctx, const uint64_t* dets, int64_t n,
                   const double* psi, int n_orb, double eps1, void* stream,
                   dnq_ham_t* out);

#ifdef __cplusplus
}
#endif
#endif /* DETNQS_GPU_H */
