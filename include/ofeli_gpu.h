/* ofeli_gpu.h -- C ABI of libofeli_gpu.so, the B200 (sm_100a) implementation
 * of OFELI's P1 assembly + preconditioned Krylov path.
 *
 * Every entry point takes plain pointers and sizes.  A vector argument may be
 * a host pointer (pageable or pinned) or a device pointer on the current
 * device; the library detects which and stages host data through its own
 * device buffers.  All calls are synchronous with respect to the host when
 * they return a value that depends on device work; the library runs its work
 * on one stream per device (ofg_get_stream) unless ofg_set_stream selects
 * another.
 *
 * Conventions follow OFELI (OFELI 5.3.3, paths within that project):
 *   - CSR patterns are exchanged in SpMatrix's layout: row_ptr 0-based with
 *     n+1 entries, col_ind 1-based (include/linear_algebra/SpMatrix_impl.h
 *     :108-119, 392-413).  Device storage is int32 0-based.
 *   - Preconditioner codes are OFELI's enum Preconditioner values
 *     (include/linear_algebra/Matrix.h:87-93): IDENT 0, DIAG 1, DILU 2,
 *     ILU 3, SSOR 4.  ILU is OFELI's ILUFactorize, i.e. diagonal ILU.
 *   - Krylov results are returned as OFELI does: the number of iterations
 *     when converged, minus the number of iterations when not
 *     (include/solvers/CG.h:99-157, include/solvers/GMRes.h:148-241).
 *
 * Status codes: 0 = success, negative = error (ofg_last_error() gives the
 * message of the calling thread's last failure).  Errors never leave the
 * device in a faulted state: waits inside kernels are bounded and report
 * through a status word.
 */
#ifndef OFELI_GPU_H
#define OFELI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OFG_OK 0
#define OFG_ERR_ARG (-1)        /* bad argument (null handle, size mismatch) */
#define OFG_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define OFG_ERR_PIVOT (-3)      /* zero pivot / missing diagonal (OFELIException in OFELI) */
#define OFG_ERR_JACOBIAN (-4)   /* non-positive element Jacobian (Triang3/Tetra4 throw) */
#define OFG_ERR_PATTERN (-5)    /* pattern not supported (nnz >= 2^31, row wider than limit) */
#define OFG_ERR_TIMEOUT (-6)    /* a bounded in-kernel wait ran out */
#define OFG_ERR_NOMEM (-7)
#define OFG_ERR_SIZE (-8)       /* size beyond a stated maximum */

/* OFG_LEARNED (5) has no OFELI counterpart: M = G^T G with G predicted by a
 * trained network (ofg_prec_create_learned). */
enum { OFG_IDENT = 0, OFG_DIAG = 1, OFG_DILU = 2, OFG_ILU = 3, OFG_SSOR = 4, OFG_LEARNED = 5 };

typedef struct ofg_matrix ofg_matrix;
typedef struct ofg_mesh ofg_mesh;
typedef struct ofg_prec ofg_prec;
typedef struct ofg_learned ofg_learned;
typedef struct ofg_batch ofg_batch;
typedef struct ofg_mesh_file ofg_mesh_file;

/* ---------------------------------------------------------------- runtime */
const char* ofg_last_error(void);
const char* ofg_version(void);
/* Selects the device of the calling thread and creates its stream
 * (optional: the first call on a device does the same), and loads the code
 * and the fixed scratch array of ofg_cg_diag_noalloc on that device, so
 * that its later calls take no device memory.  No counterpart in OFELI,
 * which has no device. */
int ofg_init(int device);
/* Waits for the library's work and frees its process-wide buffers (the mesh
 * reader's pinned staging buffer); handles stay valid. */
int ofg_shutdown(void);
/* Failure detection check: one device thread waits, with the bounded wait
 * of the triangular sweeps, for a value that nothing produces; the call
 * returns OFG_ERR_TIMEOUT after about two seconds and the context stays
 * usable.  No counterpart in OFELI. */
int ofg_selftest_wait(void);
/* Selects the stream used by later calls (NULL = the library's own). */
int ofg_set_stream(void* cuda_stream);
void* ofg_get_stream(void);
/* Number of kernels this library has launched in this process. */
int64_t ofg_launch_count(void);
/* CUDA-event timing of kernel families, for measurement: enabling (or
 * disabling) resets the totals; while enabled (on >= 1), every on-th launch
 * of an instrumented kernel is bracketed by events on the library stream.  Families: "spmv64", "spmv32",
 * "spmv16" (SELL SpMV in FP64 / FP32 / BF16 values, inside the solvers too),
 * "sweep" (triangular sweeps), "assembly" (row-gather assembly launches),
 * "network_gemm" (tensor-core layer products of the learned preconditioner's
 * network), "learned_apply" (the two FP32 factor products inside
 * ofg_fcg_learned).
 * *bytes = algorithmic bytes summed over the counted launches (0 when the
 * family has no bandwidth model).  Launches that found their stop flag set
 * are not counted.  No counterpart in OFELI (its Timer is wall clock). */
int ofg_profile_enable(int on);
int ofg_profile_read(const char* family, int64_t* launches, double* total_ms, double* bytes);

/* ------------------------------------------------------ sparse CSR matrix */
/* SpMatrix<real_t>(row_ptr, col_ind) -- include/linear_algebra/SpMatrix.h:94-210.
 * Values start at zero. */
int ofg_matrix_create(int64_t n, int64_t nnz, const int64_t* row_ptr, const int64_t* col_ind,
                      ofg_matrix** out);
int ofg_matrix_destroy(ofg_matrix* A);
int ofg_matrix_info(const ofg_matrix* A, int64_t* n, int64_t* nnz);
/* Pattern back in OFELI layout (getRowPtr/getColInd, SpMatrix_impl.h:816-826). */
int ofg_matrix_get_pattern(const ofg_matrix* A, int64_t* row_ptr, int64_t* col_ind);
/* SpMatrix::set values / SpMatrix::get() (SpMatrix_impl.h:983-995). */
int ofg_matrix_set_values(ofg_matrix* A, const double* a);
int ofg_matrix_get_values(const ofg_matrix* A, double* a);
/* Device pointers of the CSR arrays (int32 0-based columns, FP64 values). */
int ofg_matrix_device_arrays(const ofg_matrix* A, const int32_t** row_ptr, const int32_t** col,
                             double** values);
/* SpMatrix::clear (SpMatrix_impl.h:974-979). */
int ofg_matrix_clear(ofg_matrix* A);
/* SpMatrix::Mult / MultAdd: y = A x, y += A x (SpMatrix_impl.h:729-745). */
int ofg_spmv(const ofg_matrix* A, const double* x, double* y);
int ofg_spmv_add(const ofg_matrix* A, const double* x, double* y);
/* SpMatrix::TMult: y += A^T x, each y entry accumulating in ascending row
 * order as OFELI's loop intends (SpMatrix_impl.h:760-767; OFELI's loop reads
 * the previous entry's column, see entries.cu). */
int ofg_spmv_transpose_add(ofg_matrix* A, const double* x, double* y);
/* x_i = b_i / a_ii for every row (one division each): the explicit step of
 * TimeStepping's forward Euler scheme, b(i) /= D(i) with D the assembled
 * diagonal (src/solvers/TimeStepping.cpp:428-441).  OFG_ERR_PIVOT when a
 * row's diagonal entry is zero or absent. */
int ofg_matrix_diag_solve(ofg_matrix* A, const double* b, double* x);
/* SpMatrix::set(i,j,v) (set = 1) / add(i,j,v) (set = 0) for `count` entries,
 * 1-based indices, applied in order (SpMatrix_impl.h:785-802); a pair outside
 * the pattern stops the batch with OFG_ERR_ARG. */
int ofg_matrix_edit(ofg_matrix* A, int64_t count, const int64_t* i, const int64_t* j,
                    const double* v, int set);
/* Device-only SpMV with an explicit layout choice, for measurement:
 * kind 0 = CSR warp-segment kernel, 1 = SELL-32 kernel. */
int ofg_spmv_device(const ofg_matrix* A, int kind, const double* d_x, double* d_y);
/* Device-only SpMV with the FP32 copy of the values and FP32 vectors of
 * nslices*32 entries (the row count rounded up to a multiple of 32), for
 * measurement of the thread-to-row mappings of the SELL-32 layout:
 * kind 0 = one row per thread, 1 = four adjacent rows per thread (16-byte
 * loads), 2 = four rows from four consecutive slices per thread, 3 = two
 * adjacent rows per thread (8-byte loads).  blocks_per_sm (0 = 8) caps the
 * grid at that many 256-thread blocks per SM. */
int ofg_spmv32_device(ofg_matrix* A, int kind, int blocks_per_sm, const float* d_x, float* d_y);

/* -------------------------------------------------------------- P1 meshes */
/* Mesh(xmin,xmax,ymin,ymax,nx,ny,cx0,cxN,cy0,cyN,TRIANGLE) --
 * src/mesh/Mesh.cpp:547-676: x-major nodes, 2 triangles per cell, node code
 * from the boundary line codes; equations numbered over code-0 nodes
 * (Mesh::removeImposedDOF, include/mesh/Mesh.h:420). */
int ofg_mesh_create_rect(double xmin, double xmax, double ymin, double ymax, int64_t nx, int64_t ny,
                         int cx0, int cxN, int cy0, int cyN, ofg_mesh** out);
/* Unit cube split into M^3 cells, 6 positively oriented tetrahedra per cell
 * (Kuhn subdivision), nodes x fastest, code 1 on every face.  Replaces
 * OFELI's 3-D structured tetrahedral generator (src/mesh/Mesh.cpp:678-836),
 * which produces inverted elements. */
int ofg_mesh_create_kuhn(int64_t M, ofg_mesh** out);
/* General P1 mesh (Mesh::Add of nodes and elements, include/mesh/Mesh.h:321-325):
 * dim 2 (triangles, nen 3) or 3 (tetrahedra, nen 4); elem holds 0-based node
 * indices; a node with a non-zero code carries an imposed value and no
 * equation. */
int ofg_mesh_create(int dim, int64_t nn, const double* coords, int64_t ne, const int32_t* elem,
                    const int32_t* code, ofg_mesh** out);
int ofg_mesh_destroy(ofg_mesh* m);
int ofg_mesh_info(const ofg_mesh* m, int* dim, int64_t* nn, int64_t* ne, int64_t* neq);
int ofg_mesh_get(const ofg_mesh* m, double* coords, int32_t* elem, int32_t* code, int64_t* dof);
/* Node::setCoord for every node (coordinates only; topology unchanged). */
int ofg_mesh_set_coords(ofg_mesh* m, const double* coords);

/* NodeGraph (src/linear_algebra/GraphOfMatrix.cpp:347-375): the CSR pattern
 * of SpMatrix(mesh) built on the device, bit-identical to OFELI's sort+unique
 * result, plus the element-to-CSR scatter map used by assembly. */
int ofg_matrix_create_from_mesh(ofg_mesh* m, ofg_matrix** out);

/* Equation::build() for the stationary P1 problems (A cleared first):
 *   dim 2: Laplace2DT3::LHS (times kel when given) and BodyRHS
 *          (src/equations/laplace/Laplace2DT3.cpp:131-143);
 *   dim 3: DC3DT4::Diffusion(kel) and BodyRHS (src/equations/therm/DC3DT4.cpp
 *          :128-135, 207-211);
 * with Equation::updateBC lifting the nodal bc values of coded nodes
 * (include/equations/Equation_impl.h:160-176).  kel (ne), f (nn) and bc (nn)
 * may be NULL (k = 1, f = 0, bc = 0).  b receives the n-vector RHS. */
int ofg_assemble_p1(ofg_mesh* m, ofg_matrix* A, const double* kel, const double* f,
                    const double* bc, double* b);
/* Equa_Therm::build for DC2DT3 under backward Euler
 * (include/equations/therm/Equa_Therm.h:162-218): consistent + lumped
 * capacity (OFELI's CAPACITY and LUMPED_CAPACITY share one bit), diffusion
 * eps, convection by the nodal velocity v (2*nn, interleaved), RHS
 * (dti*eA1)*u_old plus the updateBC lift. */
int ofg_assemble_cd2d(ofg_mesh* m, ofg_matrix* A, double eps, const double* v, double dt,
                      const double* u_old, const double* bc, double* b);
/* The same under OFELI's time schemes (enum TimeScheme,
 * include/equations/Equa.h:124-137): FORWARD_EULER 1 (eMat = eA1/dt, RHS
 * (eA1/dt - eA0) u_old), BACKWARD_EULER 2 (as above), CRANK_NICOLSON 3
 * (eMat = eA1/dt + eA0/2, RHS (eA1/dt - eA0/2) u_old). */
int ofg_assemble_cd2d_scheme(ofg_mesh* m, ofg_matrix* A, double eps, const double* v, double dt,
                             int scheme, const double* u_old, const double* bc, double* b);
/* Vect::insertBC (include/linear_algebra/Vect_impl.h:1098-1130): nodal
 * vector from the equation-space solution x and bc (may be NULL). */
int ofg_insert_bc(const ofg_mesh* m, const double* x, const double* bc, double* u);

/* ------------------------------------------------------ mesh files (.m) */
/* OFELI's XML mesh format, read and written on the host (no GPU needed).
 * An ofg_mesh_file holds what Mesh::get keeps of a file: nodes (dim
 * coordinates, nb_dof codes each), elements (OFELI shape code -- LINE 2,
 * TRIANGLE 3, QUADRILATERAL 4, TETRAHEDRON 5, ... -- node indices 0-based,
 * one code each) and sides (node indices, nb_dof codes each).
 *
 * Mesh::get(file) -- src/mesh/Mesh.cpp:2639-2668 with XMLParser's mesh
 * reading (src/io/XMLParser.cpp:1174-1217, 2211-2295): coordinates rounded
 * to float as std::stof does, marks split per DOF by DOFCode
 * (src/mesh/MeshUtil.cpp:101-116), nothing read after a Material tag.
 * Converted by a team of host threads (ofg_mesh_file_set_threads). */
int ofg_mesh_file_read(const char* path, ofg_mesh_file** out);
/* Mesh::put(file) -- src/mesh/Mesh.cpp:2731-2806, byte for byte. */
int ofg_mesh_file_write(const ofg_mesh_file* f, const char* path);
/* A mesh file object from arrays (Mesh::Add of nodes, elements and sides,
 * include/mesh/Mesh.h:321-330); sides and their codes may be NULL when ns = 0. */
int ofg_mesh_file_create(int dim, int nb_dof, int64_t nn, const double* coords,
                         const int32_t* node_code, int el_shape, int el_nodes, int64_t ne,
                         const int32_t* elem, const int32_t* elem_code, int sd_shape, int sd_nodes,
                         int64_t ns, const int32_t* sides, const int32_t* side_code,
                         ofg_mesh_file** out);
/* The file view of a device mesh (one DOF per node, element code 1), e.g.
 * to put() a generated mesh; a structured rectangle gets the sides that
 * OFELI's constructor adds for negative line codes. */
int ofg_mesh_file_from_mesh(const ofg_mesh* m, ofg_mesh_file** out);
int ofg_mesh_file_info(const ofg_mesh_file* f, int* dim, int* nb_dof, int64_t* nn, int* el_shape,
                       int* el_nodes, int64_t* ne, int* sd_shape, int* sd_nodes, int64_t* ns);
/* Copies any non-NULL array out (sizes from ofg_mesh_file_info). */
int ofg_mesh_file_get(const ofg_mesh_file* f, double* coords, int32_t* node_code, int32_t* elem,
                      int32_t* elem_code, int32_t* sides, int32_t* side_code);
int ofg_mesh_file_destroy(ofg_mesh_file* f);
/* Host threads used to read and write mesh files (0 = all hardware threads). */
int ofg_mesh_file_set_threads(int n);
/* The device mesh of a P1 mesh file (triangles in 2-D, tetrahedra in 3-D,
 * nb_dof 1), as Mesh(file, true) would number it: equations on the nodes
 * with code 0 (Mesh::NumberEquations, src/mesh/Mesh.cpp:1483-1510). */
int ofg_mesh_create_from_file(const ofg_mesh_file* f, ofg_mesh** out);
/* Mesh(file, true) straight onto the device: the same mesh as
 * ofg_mesh_file_read + ofg_mesh_create_from_file (same values, same
 * rejections), with the file's bytes copied to the device once and its
 * Nodes / Elements / Sides texts tokenised and converted by kernels (rare
 * coordinate forms are converted on the host).  Keeps a pinned staging
 * buffer as large as the largest file read. */
int ofg_mesh_read(const char* path, ofg_mesh** out);

/* ------------------------------------------------------- preconditioners */
/* Prec<real_t>(A, type) -- include/solvers/Prec_impl.h:164-195: DIAG
 * inverts the diagonal, DILU/ILU run DILUFactorize (SpMatrix_impl.h:837-878),
 * SSOR keeps the diagonal.  The factorisation uses the current values of A. */
int ofg_prec_create(ofg_matrix* A, int type, ofg_prec** out);
int ofg_prec_destroy(ofg_prec* P);
/* Recompute the factorisation after the values of A changed. */
int ofg_prec_update(ofg_prec* P);
/* on != 0: the solvers keep P as it was set up even after the values of
 * its matrix changed (no refresh; ofg_prec_update still refreshes), e.g. a
 * learned factor computed once for a time-stepping scheme whose matrix is
 * the same at every step.  No counterpart in OFELI, whose Prec refactorises
 * when it is rebuilt. */
int ofg_prec_freeze(ofg_prec* P, int on);
/* Prec::solve(b, x) (Prec_impl.h:227-255). */
int ofg_prec_apply(ofg_prec* P, const double* b, double* x);
/* Prec::getPivot for all rows (inverse pivots for DIAG/DILU/ILU). */
int ofg_prec_get_pivot(const ofg_prec* P, double* pivot);

/* ----------------------------------------------------------------- Krylov */
/* CG(A, P, b, x, max_it, toler) -- include/solvers/CG.h:99-157.  x holds the
 * initial guess and receives the solution.  *result = iterations (>= 0) or
 * -iterations when max_it was reached; *res (may be NULL) = last relative
 * residual ||r||/||b||. */
int ofg_cg(ofg_prec* P, const double* b, double* x, int max_it, double toler, int* result,
           double* res);
/* ofg_cg that also records the relative residual after every iteration in
 * hist[1 .. iterations] (hist holds max_it + 1 values), the sequence OFELI
 * prints at Verbosity > 3 (CG.h:140-143). */
int ofg_cg_history(ofg_prec* P, const double* b, double* x, int max_it, double toler, int* result,
                   double* res, double* hist);
/* GMRes(A, P, b, x, m, max_it, toler) -- include/solvers/GMRes.h:148-241
 * (left preconditioned, modified Gram-Schmidt, Givens rotations). */
int ofg_gmres(ofg_prec* P, const double* b, double* x, int m, int max_it, double toler,
              int* result, double* res);
/* BiCGStab(A, P, b, x, max_it, toler) -- include/solvers/BiCGStab.h:87-161:
 * OFELI's return convention (iterations; 2 when (rr, r) vanishes; 3 when
 * omega vanishes; -(max_it+1) when the loop runs out). */
int ofg_bicgstab(ofg_prec* P, const double* b, double* x, int max_it, double toler, int* result,
                 double* res);
/* Mixed-precision solve: FP64 iterative refinement whose correction is
 * computed by Jacobi-preconditioned CG in FP32 (inner_bits 32) or with BF16
 * matrix values and FP32 vectors (inner_bits 16); inner_bits 0 picks BF16
 * values when every value of A is exactly representable in BF16 (the
 * iteration is then the FP32 one, bit for bit, with 2 bytes less per entry)
 * and FP32 values otherwise; FP64 only for b - A x,
 * x += correction and the accumulation of dot products.  No counterpart in
 * OFELI (its solvers are FP64 only).
 *   mode 0: one FP32 CG sequence; a refinement (FP64 true residual
 *           replacing the recursive one, search direction kept) happens
 *           whenever the FP32 residual fell by inner_tol since the last one
 *           or predicts convergence;
 *   mode 1: restarted refinement, each correction solved from zero to a
 *           relative inner_tol.
 * prec_type: DIAG or IDENT.  Converged when the FP64 true relative residual
 * ||b - A x|| / ||b|| <= toler.  *outer = refinement steps, *inner = total
 * inner CG iterations, *true_res = final FP64 relative residual. */
int ofg_solve_mixed(ofg_matrix* A, int prec_type, int inner_bits, int mode, const double* b,
                    double* x, int max_outer, int max_inner, double inner_tol, double toler,
                    int* outer, int* inner, double* true_res);
/* FP64 true relative residual ||b - A x|| / ||b|| on the device. */
int ofg_residual(const ofg_matrix* A, const double* b, const double* x, double* rel);

/* Jacobi-preconditioned CG (the DIAG case of ofg_cg, same arguments and
 * return convention) for callers that cannot allocate device memory while
 * running -- services that reserve their whole memory budget at start-up,
 * or host frameworks that own the allocator.  No counterpart in OFELI.
 * Everything is passed as device memory: the CSR matrix with int32 0-based
 * row_ptr (n+1) and col, FP64 values, b, and x (initial guess in, solution
 * out).  The solve allocates nothing: its scratch is one fixed device array
 * inside the library, held by every GPU that loads it until the process
 * exits.  Limit: n <= 131072 rows (larger systems are rejected with
 * OFG_ERR_SIZE).  Calls that overlap on the GPU share that array and race;
 * serialise them.  CUDA loads device code and arrays lazily, which takes
 * device memory: call ofg_init(device) for each device before the phase
 * that must not allocate (and before any stream capture); it loads this
 * solver's code and places the array.  A zero, missing or NaN diagonal
 * entry returns OFG_ERR_PIVOT with x unchanged. */
int ofg_cg_diag_noalloc(int64_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                        const double* b, double* x, int max_it, double toler, int* result,
                        double* res);

/* ------------------------------------------- learned preconditioner -----
 * No counterpart in OFELI.  A message-passing network over the matrix graph
 * (4 layers of width 64, BF16 activations and tensor-core layer products,
 * FP32 accumulation and FP32 master weights) predicts a lower-triangular G
 * on the pattern of A with a positive diagonal; the preconditioner is
 * M = G^T G (symmetric positive definite), applied as two sparse products.
 * With freshly created parameters M is Jacobi.  The parameter vector has
 * ofg_learned_num_params() floats (layout: W_in 4x64, b_in 64, W_l 4x(128x64),
 * b_l 4x64, u 64, v 64, c 1). */
int ofg_learned_create(uint64_t seed, ofg_learned** out);
int ofg_learned_destroy(ofg_learned* L);
int ofg_learned_num_params(void); /* returns the count, not a status */
/* Checkpoint: parameters, Adam moments (may be NULL) and the Adam step. */
int ofg_learned_get_params(const ofg_learned* L, float* params, float* adam_m, float* adam_v,
                           int64_t* step);
int ofg_learned_set_params(ofg_learned* L, const float* params, const float* adam_m,
                           const float* adam_v, int64_t step);
/* Training objective: 1 (default) the Kaporin number of M A,
 * (tr(MA)/n) / det(MA)^(1/n), with the trace estimated on the pairs (scale
 * invariant; its minimiser over the pattern is the factorised sparse
 * approximate inverse; the pairs' errors should be spectrally flat, e.g.
 * x* - x0 for random starting guesses x0); 0 the direct fit
 * mean_p ||M r_p - e_p||^2 / ||e_p||^2. */
int ofg_learned_set_loss(ofg_learned* L, int kind);
/* Layer products on the tensor cores (default 1) or on CUDA cores (0). */
int ofg_learned_set_tensor_cores(ofg_learned* L, int on);
/* `steps` Adam steps (learning rate lr, batches of `batch` pairs taken in
 * turn) on the selected objective.  R and E hold
 * npairs residual / error vectors of length n, pair-major (FP32).
 * loss_history (may be NULL) receives each step's batch loss (host). */
int ofg_learned_train(ofg_learned* L, ofg_matrix* A, const float* R, const float* E, int npairs,
                      int steps, int batch, float lr, float* loss_history);
/* Loss and its gradient (ofg_learned_num_params floats, may be NULL) over
 * all pairs, and the predicted factor at A's CSR positions (nnz floats,
 * lower part, may be NULL). */
int ofg_learned_grad(ofg_learned* L, ofg_matrix* A, const float* R, const float* E, int npairs,
                     double* loss, float* grads, float* factor);
/* One layer product X (rows x 128, BF16 bit patterns) times layer `layer`'s
 * weights, on the tensor cores (out_tc) and on CUDA cores (out_cc). */
int ofg_learned_gemm_check(ofg_learned* L, int layer, int64_t rows, const uint16_t* X,
                           float* out_tc, float* out_cc);
/* Preconditioner of type OFG_LEARNED for A (runs the network once; again
 * after A's values change).  Usable with ofg_cg, ofg_gmres, ofg_prec_apply;
 * the network must outlive it. */
int ofg_prec_create_learned(ofg_learned* L, ofg_matrix* A, ofg_prec** out);
/* Preconditioned CG with the learned preconditioner M = G^T G (one fixed
 * linear operator within a solve: beta = rho_k / rho_{k-1}; the name keeps
 * the "f" of the flexible Polak-Ribiere form it first had), in FP32
 * (inner_bits 32) or with BF16 matrix values (16, or 0 for BF16 only when
 * lossless, as in ofg_solve_mixed), inside FP64 iterative refinement; the
 * arguments and results are those of ofg_solve_mixed.  When the learned
 * iteration stagnates (residual not halved in 500 iterations, not finite, or
 * three refinements without a 10% gain) the solve continues with the plain
 * Jacobi iteration from the last verified x and *fell_back = 1.  Converged
 * only on the FP64 true residual. */
int ofg_fcg_learned(ofg_prec* P, int inner_bits, const double* b, double* x, int max_outer,
                    int max_inner, double inner_tol, double toler, int* outer, int* inner,
                    double* true_res, int* fell_back);

/* Flexible GMRES(m), right preconditioned, in mixed precision inside FP64
 * iterative refinement: the chosen form for nonsymmetric systems (the
 * transient convection-diffusion steps).  Replaces GMRes(A, P, b, x, m,
 * max_it, toler) (include/solvers/GMRes.h:148-241), which is FP64, left
 * preconditioned, with modified Gram-Schmidt.  Per Arnoldi step: z_j =
 * M^{-1} v_j in FP32 (P: DIAG, IDENT, or LEARNED with BF16 factor values),
 * the product A z_j in FP32 (FP32 values, or BF16 values per inner_bits as
 * in ofg_solve_mixed), classical Gram-Schmidt applied twice in FP64, Givens
 * rotations; a cycle stops when its residual estimate fell by inner_tol,
 * predicts the target, or after m steps (1 <= m <= 64).  x (initial guess
 * in, solution out) += Z y.  Converged only when the FP64 true relative
 * residual ||b - A x|| / ||b|| <= toler.  *outer = cycles, *inner = Arnoldi
 * steps, *true_res = final FP64 relative residual; with LEARNED, when two
 * cycles in a row fail to halve the residual (or it is not finite) the
 * remaining cycles use the diagonal preconditioner and *fell_back = 1. */
int ofg_fgmres_mixed(ofg_prec* P, int inner_bits, const double* b, double* x, int m,
                     int max_outer, int max_inner, double inner_tol, double toler, int* outer,
                     int* inner, double* true_res, int* fell_back);

/* ------------------------------------------------------ batched problems --
 * No counterpart in OFELI (its equivalent is a loop of build() + CG per
 * problem).  Many independent P1 problems of uneven size (one mesh each, all
 * of one dimension) are assembled and solved in one persistent launch: per
 * problem Equation::build() (k per element, f per node, Dirichlet data bc per
 * node or 0), CG with the diagonal preconditioner in FP64 to
 * ||r|| / ||b|| <= toler with the FP64 true residual checked at the end, and
 * insertBC into the nodal solution.  A block owns one problem at a time,
 * longest problems first; the launch is captured in a CUDA graph. */
/* Concatenates the meshes' data and builds every pattern; the meshes may be
 * destroyed afterwards. */
int ofg_batch_create(int nprob, ofg_mesh* const* meshes, ofg_batch** out);
int ofg_batch_destroy(ofg_batch* B);
int ofg_batch_info(const ofg_batch* B, int* nprob, int64_t* nodes, int64_t* elements,
                   int64_t* rows, int64_t* nnz);
int ofg_batch_problem_info(const ofg_batch* B, int prob, int64_t* nodes, int64_t* elements,
                           int64_t* rows, int64_t* nnz);
/* Inputs concatenated in problem order: kel per element (NULL = 1), f per
 * node (NULL = 0), bc per node (NULL = 0). */
int ofg_batch_set_inputs(ofg_batch* B, const double* kel, const double* f, const double* bc);
/* Assembles and solves every problem (one graph launch). */
int ofg_batch_solve(ofg_batch* B, int max_it, double toler);
/* Nodal solutions (concatenated), per-problem iterations (OFELI's CG
 * convention: negative when max_it ran out) and FP64 true relative residuals;
 * any argument may be NULL. */
int ofg_batch_get_results(const ofg_batch* B, double* u, int* iters, double* res);
/* Assembled values (CSR order of the problem's pattern) and RHS of one problem. */
int ofg_batch_get_matrix(const ofg_batch* B, int prob, double* values, double* rhs);
/* Autotuner: solves once to measure every problem's work (rows x
 * iterations), then times the whole batch once per launch shape (threads
 * per block x lanes per CSR row x blocks per cluster, 18 shapes;
 * ofg_batch_config_shape) and keeps the fastest; *chosen = its index,
 * times_ms (may be NULL, 18 floats) receives every shape's time.  With
 * clusters, a problem above one block's fair share of the work is solved by
 * the whole cluster. */
int ofg_batch_tune(ofg_batch* B, int max_it, double toler, int* chosen, float* times_ms);
int ofg_batch_set_config(ofg_batch* B, int config, int blocks_per_sm);
/* Inner precision: 64 (default) = CG + DIAG in FP64; 32 = CG + DIAG in FP32
 * (FP32 values, 16-bit column offsets where they fit) inside FP64 iterative
 * refinement, with the same FP64 true-residual test. */
int ofg_batch_set_precision(ofg_batch* B, int bits);
int ofg_batch_config_shape(int config, int* threads, int* lanes_per_row, int* cluster);

#ifdef __cplusplus
}
#endif
#endif /* OFELI_GPU_H */
