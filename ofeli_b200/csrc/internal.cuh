// internal.cuh -- the handle types behind the C ABI and the helpers the
// translation units share.
#pragma once

#include "common.cuh"

// Device CSR matrix.  The CSR arrays are the master copy (OFELI's SpMatrix
// layout, 0-based int32 columns on the device); a SELL-32 copy of the values
// (slices of 32 consecutive rows stored column-major, rows kept in natural
// order) is rebuilt lazily when the values change and feeds the SpMV inside
// the Krylov loops.
struct ofg_matrix {
   int64_t n = 0, nnz = 0;
   ofg::DBuf<int32_t> row_ptr, col;
   ofg::DBuf<double> val;
   uint64_t version = 1;  // bumped whenever values change

   // diagonal position of every row (OFELI's id[i]-1); -1 if absent
   ofg::DBuf<int32_t> dpos;
   bool dpos_ready = false;
   bool dpos_complete = false;

   // SELL-32 layout
   int64_t nslices = 0;
   ofg::DBuf<int32_t> sell_ptr;  // nslices+1, offsets in entries
   ofg::DBuf<int32_t> sell_col;  // padded entries point at a valid row, value 0
   ofg::DBuf<int32_t> sell_src;  // CSR index of every SELL entry, -1 for padding
   ofg::DBuf<double> sell_val;
   ofg::DBuf<float> sell_val32;
   ofg::DBuf<uint16_t> sell_valbf;  // BF16 bit patterns of the values
   // column - row of every SELL entry (0 for padding) when every offset fits
   // in 16 bits (idx16 = 1; 0 = does not fit; -1 = not built yet)
   ofg::DBuf<int16_t> sell_d16;
   int idx16 = -1;
   // slices whose 32 rows have the same 16-bit offset at every position k
   // (structured meshes in natural order): sell_uni[s] = start of the
   // slice's w offsets in sell_utab, -1 for a slice that keeps per-entry
   // offsets; uni_nnz = nonzeros in the uniform slices (built once, with the
   // 16-bit offsets)
   ofg::DBuf<int32_t> sell_uni;
   ofg::DBuf<int16_t> sell_utab;
   int64_t uni_nnz = 0, utab_len = 0;
   bool uni_ready = false;
   bool sell_ready = false;
   uint64_t sell_version = 0, sell32_version = 0, sellbf_version = 0;
   int max_row = 0;
   double avg_row = 0;

   // column-major copy of the pattern for the transposed product (built on
   // first use): column c's entries t_ptr[c] .. t_ptr[c+1], their rows in
   // ascending order and their CSR positions
   ofg::DBuf<int64_t> t_ptr;
   ofg::DBuf<int32_t> t_row, t_pos;
   bool t_ready = false;

   // element-to-CSR map of the mesh this pattern came from
   ofg_mesh* mesh = nullptr;
   ofg::DBuf<int32_t> emap;  // ne * nen * nen, -1 where a DOF is imposed
};

struct ofg_mesh {
   int dim = 2, nen = 3;
   int64_t nn = 0, ne = 0, neq = 0;
   ofg::DBuf<double> coords;  // nn * dim
   ofg::DBuf<int32_t> elem;   // ne * nen, 0-based
   ofg::DBuf<int32_t> code;   // nn
   ofg::DBuf<int32_t> dof;    // nn, 1-based equation number or 0
   // node -> element adjacency (elements in ascending order)
   ofg::DBuf<int32_t> n2e_ptr, n2e;
   // the structured rectangle's cells and line codes (rect_nx < 0 otherwise),
   // kept for the sides Mesh::put writes
   int64_t rect_nx = -1, rect_ny = -1;
   int rect_code[4] = {0, 0, 0, 0};   // cx0, cxN, cy0, cyN
};

namespace ofg {
// Strand plan of one sweep direction (see prec.cu).
struct SweepPlan {
   int64_t nstrands = 0;
   DBuf<int32_t> start;       // logical row where each strand starts, nstrands+1
   DBuf<double> strand_dot;   // per-strand partial dot products
   DBuf<int> ticket;          // [0] next strand, [1] finished strands
   // per-segment slot layout of the dependency entries: segment s of strand
   // t (t's rows in 32-row groups) owns slots seg_off[s] .. seg_off[s+1],
   // stored column-major (slot k of lane l at seg_off[s] + 32 k + l), in
   // the CSR's column order
   int64_t nseg = 0;
   int wmax = 0;              // slots of the widest segment
   DBuf<int32_t> tseg;        // first segment of each strand, nstrands+1
   DBuf<int32_t> seg_off;     // nseg+1
   DBuf<int32_t> sl_col;      // physical column, -1 for padding
   DBuf<int32_t> sl_src;      // CSR index of the value, -1 for padding
   DBuf<double> sl_val;
   // per segment: the lowest row of the previous strand that this or a
   // later segment of its strand reads from the band's shared-memory ring
   // (INT32_MAX: none); the solve sweeps publish it so that the previous
   // strand's warp never overwrites a ring slot still to be read
   DBuf<int32_t> seg_keep;
};
}  // namespace ofg

namespace ofg {
// learned.cu: frees the network buffers kept for a learned preconditioner
void learned_release(const ofg_prec* P);
}  // namespace ofg

struct ofg_prec {
   ofg_matrix* A = nullptr;
   int type = OFG_DIAG;
   ofg::DBuf<double> pivot;  // DIAG/DILU/ILU: inverse pivots; SSOR: diagonal
   uint64_t version = 0;     // matrix version the factorisation belongs to
   // forward-sweep result, kept at the "not ready" sentinel between sweeps
   ofg::DBuf<double> t;
   ofg::DBuf<int> status;    // bounded-wait failures (bit 0: timeout, bit 1: wave)
   ofg::SweepPlan fwd, bwd;
   ofg::DBuf<int32_t> tpos;  // D-ILU: transposed position of each lower entry
   ofg::DBuf<double> dot;    // (r, z) of the last backward sweep that was asked for it
   int grid = 0;             // blocks of the persistent factorisation sweep launch
   int solve_grid = 0;       // blocks of the persistent solve sweep launch
   // frozen: the solvers keep the preconditioner as it was set up even after
   // the matrix values changed (ofg_prec_freeze; refreshed by ofg_prec_update)
   bool frozen = false;
   // LEARNED: the network that predicts the factor G, and G (lower rows) and
   // G^T (upper rows) as matrices of their own; M = G^T G
   ofg_learned* net = nullptr;
   ofg_matrix* gl = nullptr;
   ofg_matrix* gu = nullptr;
   ofg::DBuf<double> partials;
   ofg::DBuf<unsigned> counter;
   ~ofg_prec()
   {
      if (type == OFG_LEARNED) ofg::learned_release(this);
      delete gl;
      delete gu;
   }
};

namespace ofg {

// matrix.cu
void ensure_dpos(ofg_matrix* A);
void ensure_sell(ofg_matrix* A);
void ensure_sell32(ofg_matrix* A);
void ensure_sell_bf16(ofg_matrix* A);
// builds the 16-bit column offsets once per pattern; true when they fit
bool ensure_sell_d16(ofg_matrix* A);
// after ensure_sell_d16 returned true
void ensure_sell_uniform(ofg_matrix* A);
void spmv_csr(const ofg_matrix* A, const double* x, double* y, bool add);
void spmv_sell(const ofg_matrix* A, const double* x, double* y, const int* skip = nullptr);
void matrix_touch(ofg_matrix* A);
void matrix_finish_pattern(ofg_matrix* A);
// a mesh with its coordinate, connectivity and code buffers allocated, and
// the rest (equation numbers from the codes, node-to-element lists) built
// once those hold the mesh (mesh.cu)
ofg_mesh* new_mesh(int dim, int64_t nn, int64_t ne);
void finish_mesh(ofg_mesh* m);
void scan_exclusive_i64(const int64_t* d_in, int64_t* d_out, int64_t n);

// prec.cu
void prec_setup(ofg_prec* P);
// true when the solvers must set the preconditioner up again before use: the
// matrix values changed since, and the preconditioner is not frozen
inline bool prec_stale(const ofg_prec* P) { return !P->frozen && P->version != P->A->version; }
// z = M^{-1} r on device buffers (r and z may alias).  With rz != nullptr
// the sweep preconditioners also leave (r, z) in *rz (device scalar).  With
// skip != nullptr every launch is a no-op while *skip != 0.
void prec_apply_device(ofg_prec* P, const double* r, double* z, double* rz = nullptr,
                       const int* skip = nullptr);
void check_status(ofg_prec* P);

// The "value not ready yet" marker of the triangular sweeps: a NaN payload
// that IEEE arithmetic never produces (results are the canonical NaN).
constexpr unsigned long long kSentinelBits = 0x7FF4DEADBEEF0001ULL;
void fill_sentinel(double* p, int64_t n);

// learned.cu: run the network on the matrix's current values and rebuild
// G / G^T; z = G^T G r in FP64 (r and z may alias; rz as above when they
// do not)
void learned_setup(ofg_prec* P);
void learned_apply(ofg_prec* P, const double* r, double* z, double* rz, const int* skip);

}  // namespace ofg
