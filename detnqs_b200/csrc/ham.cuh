// ham.cuh -- Hamiltonian blocks resident in HBM.
//
// CSR with int64 row pointers, u32 column indices and FP64 values (the
// reference's CSRMatrix, ham_utils.hpp:132-153).  For the FP32 operator the
// V block also keeps FP32 off-diagonal values (diagonal zeroed) beside the
// FP64 diagonal vector.
#pragma once

#include "common.cuh"

namespace dnq {

// Compressed rows.  Standard form: row r is [rowptr[r], rowptr[r + 1]) of
// col / val.  Arena form (a V->V build leaves its rows where the build
// wrote them): row r is [rowptr[r], rowend[r]), and col / val hold free
// slots between rows; ensure_compact turns it into the standard form.  The
// H.psi kernels read either through row_start() / row_end(), with span()
// (the array length) bounding their vector loads.
struct Csr {
    DBuf<i64> rowptr;
    DBuf<i64> rowend;    // arena form only
    DBuf<u32> col;
    DBuf<double> val;
    DBuf<float> val32;   // optional FP32 off-diagonal copy (ready when as long as val)
    i64 nr = 0, nc = 0, nnz = 0;
    bool sorted = true;   // columns ascending inside each row
    bool arena = false;
    const i64* row_start() const { return rowptr.p; }
    const i64* row_end() const { return arena ? rowend.p : rowptr.p + 1; }
    i64 span() const { return (i64)col.n; }
    bool f32_ready() const { return val32.n == val.n; }
    size_t bytes() const {
        return rowptr.bytes() + rowend.bytes() + col.bytes() + val.bytes() + val32.bytes();
    }
};

// Standard form of a block in arena form (no-op otherwise); drops nothing.
void ensure_compact(Csr& m, cudaStream_t s);


}  // namespace dnq

struct dnq_ham_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    dnq::i64 n_v = 0, n_p = 0;
    int words = 1;                    // uint64 words per spin string of V and P
    dnq::Csr vv, vp;
    dnq::Csr pv;                      // transpose of vp, built on first use
    bool pv_ready = false;
    dnq::DBuf<double> diag;           // H_ii of V as evaluated (Slater-Condon)
    dnq::DBuf<double> diag_op;        // diagonal entries stored in vv (0 if dropped)
    dnq::DBuf<float> x32;             // FP32 scratch for the FP32 operator
    dnq::DBuf<unsigned long long> dets_p;   // (alpha, beta) pairs
    dnq::i64 candidates = 0;
    dnq::Options opt = dnq::default_options();   // this handle's options
    // device time of the build phases (CUDA events on the build stream), ms:
    // [0] maps + diagonal, [1] count pass, [2] scans + allocation,
    // [3] fill pass, [4] V-row sort, [5] P discovery + P-row sort, [6] total
    double t_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t bytes() const {
        return vv.bytes() + vp.bytes() + pv.bytes() + diag.bytes() + diag_op.bytes() + x32.bytes() +
               dets_p.bytes();
    }
};

namespace dnq {
// Segmented sort of (col, val) pairs inside each CSR row by column.
void sort_rows(Csr& m, cudaStream_t s);
// sort_rows unless the block is already sorted.
void ensure_sorted(Csr& m, cudaStream_t s);
// One operator of a grouped H.psi launch: y = M x (+ diag .* x when diag is
// given).  val / xg are double (FP64) or float (FP32 values and x).
struct SpmvDesc {
    const i64* rp;       // row starts
    const i64* re;       // row ends
    const u32* col;
    const void* val;
    const void* xg;
    const double* diag;
    const double* x;
    double* y;
    i64 nr, nnz;         // rows; length of col / val (bounds the vector loads)
};
// Lanes per row and slots per lane the H.psi kernels use for m.
void spmv_shape(const Options& o, const Csr& m, int& G, int& U);
// One launch over nd descriptors (device array) sharing (G, U, precision).
void spmv_grouped(const SpmvDesc* d_dev, int nd, i64 max_rows, int G, int U, int precision,
                  int device, cudaStream_t s);
// FP32 off-diagonal value copy of a square block (diagonal entries zeroed)
// and, when diag_out is given, the FP64 diagonal entries (0 where absent).
void make_f32(Csr& m, cudaStream_t s, DBuf<double>* diag_out = nullptr);
}  // namespace dnq
