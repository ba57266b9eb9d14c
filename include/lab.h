/* liblinalg_b200 -- C ABI of the B200 (sm_100a) AMG-preconditioned Krylov library.
 *
 * This is the boundary the C++ API (include/linalg.h and friends, namespace
 * linalg, the same classes and free functions as the LinAlgLib reference) and
 * any foreign-language binding call.  Plain C types only: opaque handles,
 * pointers, int64 sizes, an explicit CUDA stream and an int status.
 *
 * Memory: matrices (lab_csr) and hierarchies are owned by the library and live
 * in device memory.  Vector arguments are raw pointers; unless a function says
 * otherwise they are DEVICE pointers of length m (or n) and are read/written on
 * the given stream.  A NULL stream means the legacy default stream.  Every
 * computing entry point runs on the GPU; there is no host fallback, and with no
 * usable device the library returns LAB_NO_DEVICE.
 *
 * Each declaration names the reference interface it replaces as
 * path:line inside the LinAlgLib tree.
 */
#ifndef LAB_H
#define LAB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define LAB_API __declspec(dllexport)
#else
#define LAB_API __attribute__((visibility("default")))
#endif

/* Status codes.  The reference returns iteration counts or bool and prints its
 * errors (library/src/utility.h:172-183); the C++ layer maps these back onto
 * those conventions. */
typedef enum lab_status
{
    LAB_OK            = 0,
    LAB_NOT_CONVERGED = 1, /* solver hit max_iter / max_cycle */
    LAB_BREAKDOWN     = 2, /* (p, Ap) == 0 or (z, r) == 0 in CG, or a Givens breakdown */
    LAB_NAN           = 3, /* NaN in a residual norm (iter_control.cpp:50-59) */
    LAB_BAD_ARG       = 4,
    LAB_OOM           = 5,
    LAB_TIMEOUT       = 6, /* a bounded device-side wait gave up */
    LAB_CUDA_ERROR    = 7,
    LAB_NOT_SUPPORTED = 8,
    LAB_NO_DEVICE     = 9
} lab_status;

typedef enum lab_memory
{
    LAB_MEM_HOST   = 0,
    LAB_MEM_DEVICE = 1
} lab_memory;

typedef struct lab_csr_s*     lab_csr;
typedef struct lab_hier_s*    lab_hierarchy;
typedef struct lab_precond_s* lab_precond;
typedef void*                 lab_stream; /* cudaStream_t */

/* ------------------------------------------------------------------ runtime */
LAB_API const char* lab_status_string(lab_status s);
/* Detail message of the last failing call on this thread. */
LAB_API const char* lab_last_error(void);
/* Select the device and set up the stream-ordered memory pool.  Called
 * implicitly by the first entry point that needs the device.
 * Replaces linalg::is_device_available (library/src/linalg_memory.cpp). */
LAB_API lab_status lab_init(int device);
/* Replaces linalg::synchronize (library/src/linalg_memory.cpp). */
LAB_API lab_status lab_synchronize(lab_stream s);
/* Number of kernel launches issued by this library since load (all threads). */
LAB_API int64_t lab_launch_count(void);
/* How many bounded device-side waits of the streaming row kernels ran out on the
 * current device since the library was loaded (0 in normal operation: a wait
 * that runs out ends its kernel early instead of hanging the GPU, and the rows
 * it had not reached are left unwritten).  No reference counterpart. */
LAB_API lab_status lab_wait_timeouts(int64_t* count, lab_stream s);
/* Allocate / free library device memory (stream ordered). */
LAB_API lab_status lab_malloc(void** p, size_t bytes, lab_stream s);
LAB_API lab_status lab_free(void* p, lab_stream s);
LAB_API lab_status lab_memcpy(void* dst, const void* src, size_t bytes, lab_stream s);

/* ------------------------------------------------------------------ CSR matrix */
/* Create an m x n CSR matrix with int32 indices and float64 values, copying the
 * arrays from host or device memory.  Columns must be in [0, n); the row pointer
 * must be non-decreasing with row_ptr[0] == 0 and row_ptr[m] == nnz (checked).
 * Replaces csr_matrix<double>::csr_matrix(row_ptr, col_ind, val, m, n, nnz)
 * (library/include/csr_matrix.h:113-118; library/src/csr_matrix.cpp:54-74). */
LAB_API lab_status lab_csr_create(lab_csr* A, int64_t m, int64_t n, int64_t nnz,
                                  const int32_t* row_ptr, const int32_t* col_ind,
                                  const double* val, lab_memory where, lab_stream s);
/* Allocate an uninitialised matrix (csr_matrix::resize, csr_matrix.cpp:141-151). */
LAB_API lab_status lab_csr_create_empty(lab_csr* A, int64_t m, int64_t n, int64_t nnz,
                                        lab_stream s);
LAB_API lab_status lab_csr_destroy(lab_csr A);
LAB_API lab_status lab_csr_info(lab_csr A, int64_t* m, int64_t* n, int64_t* nnz);
/* Device arrays owned by the matrix (valid until it is destroyed). */
LAB_API lab_status lab_csr_device_arrays(lab_csr A, int32_t** row_ptr, int32_t** col_ind,
                                         double** val);
/* Copy the matrix out to host or device buffers (any pointer may be NULL). */
LAB_API lab_status lab_csr_copy_to(lab_csr A, int32_t* row_ptr, int32_t* col_ind, double* val,
                                   lab_memory where, lab_stream s);
/* Deep copy (csr_matrix::copy_from, csr_matrix.cpp:153-168). */
LAB_API lab_status lab_csr_clone(lab_csr A, lab_csr* B, lab_stream s);
/* Values changed in place through lab_csr_device_arrays: the cached diagonal and
 * reduced-precision copies are released on stream s (pass the stream the matrix
 * was last used on) and the matrix takes a new identity, so solver graphs
 * captured on the old values are captured again.  Preconditioners built earlier
 * keep what they copied at build time, as the reference's build() does.  A
 * hierarchy's own level matrices are not to be changed in place (set up again).
 * The reference mutates through csr_matrix::get_row_ptr / get_col_ind / get_val
 * (csr_matrix.h:175-185) and
 * caches nothing. */
LAB_API lab_status lab_csr_values_changed(lab_csr A, lab_stream s);
/* Row pointers or column indices changed in place: lab_csr_values_changed plus
 * the SpMV plan and the triangular-solve levels (rebuilt on next use). */
LAB_API lab_status lab_csr_structure_changed(lab_csr A, lab_stream s);

/* ------------------------------------------------------------------ Matrix Market
 * Host-only file I/O (no device needed), behind csr_matrix::read_mtx / write_mtx.
 *
 * lab_mtx_read replaces csr_matrix::read_mtx (library/src/csr_matrix.cpp:523-729):
 * coordinate files with real or integer values, general or symmetric (array,
 * complex, pattern, hermitian and skew-symmetric files are refused with
 * LAB_BAD_ARG, as the reference refuses them); symmetric files are mirrored;
 * repeated entries are summed in the reference's order, so the CSR arrays are
 * bit-identical to the reference's.  Files the reference would crash on (an
 * unparsable entry, an index outside the stated size) are refused.  The three
 * arrays are allocated with malloc; release each with lab_mtx_free. */
LAB_API lab_status lab_mtx_read(const char* path, int64_t* m, int64_t* n, int64_t* nnz,
                                int32_t** row_ptr, int32_t** col_ind, double** val);
LAB_API void       lab_mtx_free(void* p);
/* Replaces csr_matrix::write_mtx (csr_matrix.cpp:731-795): the same bytes (banner,
 * comment line, sizes, one "row col value" line per entry, values "%.10f"). */
LAB_API lab_status lab_mtx_write(const char* path, int64_t m, int64_t n, int64_t nnz,
                                 const int32_t* row_ptr, const int32_t* col_ind,
                                 const double* val);

/* ------------------------------------------------------------------ SpMV */
typedef enum lab_spmv_alg
{
    LAB_SPMV_AUTO    = 0, /* chosen by lab_spmv_analysis from row statistics */
    LAB_SPMV_ROWSEQ  = 1, /* thread per row over shared-memory staged rows, fma in CSR order */
    LAB_SPMV_VECTOR  = 2, /* 2..32 lanes per row, vectorised loads, shuffle reduction */
    LAB_SPMV_MERGE   = 3, /* merge-path nnz split for skewed row lengths */
    LAB_SPMV_VECTOR_STREAM = 4, /* LAB_SPMV_VECTOR with the matrix streamed through shared
                                  memory by bulk copies (one producer warp, mbarrier
                                  stage ring) on operators of >= 8192 rows; the same
                                  per-row arithmetic, bit-identical; elsewhere as VECTOR */
    LAB_SPMV_VECTOR_HALO = 5 /* LAB_SPMV_VECTOR on a square matrix with x staged per chunk
                                of consecutive rows at the chunk's distinct columns in
                                shared memory (one list per chunk, built when first
                                forced or tuned); the same per-row arithmetic,
                                bit-identical; elsewhere as VECTOR */
} lab_spmv_alg;

/* Row-length statistics -> algorithm and launch shape, cached on the matrix.
 * Replaces csrmv_analysis (library/include/linalg_math.h:287-292). */
LAB_API lab_status lab_spmv_analysis(lab_csr A, lab_stream s);
/* Force an algorithm (LAB_SPMV_AUTO restores the analysed choice). */
LAB_API lab_status lab_spmv_set_algorithm(lab_csr A, lab_spmv_alg alg, int lanes);
LAB_API lab_status lab_spmv_get_algorithm(lab_csr A, int* alg, int* lanes);
/* Halo plan of A (built by lab_spmv_analysis for the VECTOR schedule of a square
 * matrix): chunks of *rows_per_chunk consecutive rows, *distinct staged columns
 * over all chunks, *direct_chunks chunks that read x directly; all 0 when A has
 * no halo plan.  Any output may be NULL.  No counterpart in the reference. */
LAB_API lab_status lab_spmv_halo_info(lab_csr A, int64_t* chunks, int64_t* rows_per_chunk,
                                      int64_t* distinct, int64_t* direct_chunks);
/* Autotuner: time every candidate SpMV schedule on this matrix (one thread per
 * row, and unless `exact` W = 2..32 lanes per row in the direct, streamed and halo
 * forms the matrix has) and keep the fastest; the
 * winner's time per SpMV in microseconds goes to *best_us (may be NULL).  With
 * exact != 0 only schedules that accumulate in CSR order (bit-identical to the
 * reference, host_matrix_vector.cpp:60-84) are candidates.  No counterpart in the
 * reference, which rebuilds a fixed descriptor per call (csr_matrix.cpp:307-314).
 * A solver iteration graph already captured on A is dropped and re-captured. */
LAB_API lab_status lab_spmv_autotune(lab_csr A, int exact, double* best_us, lab_stream s);
/* y = alpha*A*x + beta*y (beta == 0: y is not read).
 * Replaces csrmv_solve (library/include/linalg_math.h:304-310) and
 * csr_matrix::multiply_by_vector(_and_add) (csr_matrix.cpp:303-330). */
LAB_API lab_status lab_spmv(double alpha, lab_csr A, const double* x, double beta, double* y,
                            lab_stream s);
/* r = b - A*x.  Replaces compute_residual (library/include/linalg_math.h:144-147). */
LAB_API lab_status lab_residual(lab_csr A, const double* x, const double* b, double* r,
                                lab_stream s);
/* Multi-vector SpMM: Y[:,k] = alpha*A*X[:,k] + beta*Y[:,k], k < nrhs, column
 * major with leading dimensions ldx/ldy (no reference counterpart: batched
 * right-hand sides). */
LAB_API lab_status lab_spmm(double alpha, lab_csr A, int nrhs, const double* X, int64_t ldx,
                            double beta, double* Y, int64_t ldy, lab_stream s);

/* ------------------------------------------------------------------ BLAS-1 */
/* y = alpha*x + y.  linalg_math.h:52 (host_axpy.cpp:35-45). */
LAB_API lab_status lab_axpy(int64_t n, double alpha, const double* x, double* y, lab_stream s);
/* y = alpha*x + beta*y.  linalg_math.h:63 (host_axpy.cpp:47-69). */
LAB_API lab_status lab_axpby(int64_t n, double alpha, const double* x, double beta, double* y,
                             lab_stream s);
/* z = alpha*x + beta*y + gamma*z.  linalg_math.h:76 (host_axpy.cpp:71-82). */
LAB_API lab_status lab_axpbypgz(int64_t n, double alpha, const double* x, double beta,
                                const double* y, double gamma, double* z, lab_stream s);
/* Deterministic reductions; the result is written to *result on the host after
 * the stream is synchronised.  linalg_math.h:132, 165, 175. */
LAB_API lab_status lab_dot(int64_t n, const double* x, const double* y, double* result,
                           lab_stream s);
LAB_API lab_status lab_norm_inf(int64_t n, const double* x, double* result, lab_stream s);
LAB_API lab_status lab_norm_euclid(int64_t n, const double* x, double* result, lab_stream s);
/* x = value.  vector::fill (library/src/vector.cpp). */
LAB_API lab_status lab_fill(int64_t n, double value, double* x, lab_stream s);
/* d[i] = A(i,i) (first diagonal entry of the row, 0 if none).
 * linalg_math.h:155 (host_extract.cpp:34-52). */
LAB_API lab_status lab_diagonal(lab_csr A, double* d, lab_stream s);
/* x = rhs ./ diag.  Jacobi preconditioner solve (host_math.cpp:52-64). */
LAB_API lab_status lab_jacobi_solve(int64_t n, const double* rhs, const double* diag, double* x,
                                    lab_stream s);
/* In-place exclusive prefix sums.  linalg_primitives.h:98 (host_primitives.cpp:76-91). */
LAB_API lab_status lab_exclusive_scan_i64(int64_t n, int64_t* x, lab_stream s);
LAB_API lab_status lab_exclusive_scan_i32(int64_t n, int32_t* x, lab_stream s);
/* The int64 exclusive scan for callers that cannot allocate device memory
 * during the call (a process whose other allocator holds nearly all of the
 * device, a host thread that cannot wait on the driver's allocator, a fixed
 * memory budget after start-up): its scratch is a fixed 512 KiB array in the
 * library's device image, so it calls no cudaMalloc / cudaFree and no
 * allocating routine.  No counterpart in the reference (it has no
 * allocation-free variants).
 * Limit: n <= 134,217,728 elements; larger n returns LAB_BAD_ARG untouched.
 * The first call on each device looks up the array's device address (make
 * that first call before any stream capture).  All calls share the one array:
 * calls that overlap on the GPU (other streams, other threads) race. */
LAB_API lab_status lab_exclusive_scan_i64_noalloc(int64_t n, int64_t* x, lab_stream s);

/* Sparse triangular solve x = T^-1 b on the lower (columns < i) or upper part
 * of A, unit or stored diagonal (csrtrsv_analysis / csrtrsv_solve,
 * linalg_math.h:229-254; host_csrtrsv.cpp).  The dependency levels of A's pattern
 * are computed on first use and kept with A; b and x may be the same array. */
LAB_API lab_status lab_csrtrsv(lab_csr A, int lower, int unit_diag, const double* b, double* x,
                               lab_stream s);
/* Build (once) the dependency levels of A's pattern that the triangular solves and
 * the IC(0) / ILU(0) factorizations use; otherwise their first call builds them.
 * Replaces csrtrsv_analysis / csric0_analysis / csrilu0_analysis
 * (linalg_math.h:229-237, 469, 510). */
LAB_API lab_status lab_csrtrsv_analysis(lab_csr A, lab_stream s);
/* T = the lower (columns <= i) or upper (columns >= i) triangle of A, diagonal
 * included, a new matrix.  Replaces csr_matrix::copy_lower_triangular_from /
 * copy_upper_triangular_from (csr_matrix.h:215, 227; host_extract.cpp:54-181). */
LAB_API lab_status lab_csr_triangle(lab_csr A, int upper, lab_csr* T, lab_stream s);
/* a_ii *= scalar on the first stored diagonal entry of every row.  Replaces
 * csr_matrix::scale_diagonal_by (csr_matrix.h:254; host_scale.cpp:34-52). */
LAB_API lab_status lab_csr_scale_diagonal(lab_csr A, double scalar, lab_stream s);
/* a_ij *= 1 / a_jj (the diagonal of lab_diagonal, indexed by column, as the
 * reference computes it).  Replaces csr_matrix::scale_by_inverse_diagonal
 * (csr_matrix.h:262; csr_matrix.cpp:277-299; host_scale.cpp:54-69). */
LAB_API lab_status lab_csr_scale_by_inverse_diagonal(lab_csr A, lab_stream s);
/* The bounded wait of the triangular solves on A (the lab_csrtrsv solves and the
 * ILU / IC / Gauss-Seidel / SOR / SSOR preconditioner applications).  A row waits
 * for its dependencies by polling; after idle_rounds rounds without progress
 * (0: the default, 2^26) its warp gives up, the launch returns and the call
 * reports LAB_TIMEOUT instead of hanging.  held_row >= 0 names a row whose value
 * the solves never write, so the rows that depend on it run out of their wait:
 * a test of that path (-1: none, the normal setting).  No reference counterpart
 * (the reference's host solves are sequential loops, host_csrtrsv.cpp:36-90). */
LAB_API lab_status lab_csrtrsv_wait_control(lab_csr A, int64_t idle_rounds, int64_t held_row,
                                            lab_stream s);
/* In-place incomplete factorizations of A's values: ILU(0) (csrilu0,
 * linalg_math.h:109; host_csrilu0.cpp) and IC(0) (csric0, linalg_math.h:95;
 * host_csric0.cpp, the upper part left unchanged).  The smallest column with a
 * missing / zero pivot goes to *structural_zero / *numeric_zero (-1: none). */
LAB_API lab_status lab_csrilu0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s);
LAB_API lab_status lab_csric0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s);

/* ------------------------------------------------------------------ sparse products */
/* C = A*B (new matrix), rows sorted by column, each entry accumulated in A-row
 * then B-row order exactly as the reference host SpGEMM, so results are
 * bit-identical to it.  Replaces csrgemm_nnz + csrgemm_solve with alpha = 1,
 * beta = 0 (linalg_math.h:408-440; host_csrgemm.cpp:37-245) and
 * csr_matrix::multiply_by_matrix (csr_matrix.cpp:333-353). */
LAB_API lab_status lab_spgemm(lab_csr A, lab_csr B, lab_csr* C, lab_stream s);
/* C = alpha*A + beta*B.  Replaces csrgeam_nnz + csrgeam_solve
 * (linalg_math.h:345-372; host_csrgeam.cpp). */
LAB_API lab_status lab_spgeam(double alpha, lab_csr A, double beta, lab_csr B, lab_csr* C,
                              lab_stream s);
/* T = A^T, each row listing source rows ascending.  Replaces
 * csr_matrix::transpose (csr_matrix.cpp:437-447; host_csr2csc.cpp:30-75). */
LAB_API lab_status lab_transpose(lab_csr A, lab_csr* T, lab_stream s);

/* ------------------------------------------------------------------ AMG setup pieces */
/* conn[j] = (col != row) && |a_ij| >= eps*sqrt(|a_ii|*|a_jj|), bit-exact.
 * Replaces compute_strong_connections (amg_strength.cpp:40-52;
 * host_amg_strength.cpp:33-70).  conn: device int32[nnz]. */
LAB_API lab_status lab_strength(lab_csr A, double eps, int32_t* conn, lab_stream s);
/* RS strength -a_ij >= theta*max_{k!=i}(-a_ik) plus the strength matrix S.
 * Replaces compute_classical_strong_connections (amg_strength.cpp:57-71;
 * host_amg_strength.cpp:72-156).  conn: device int32[nnz], zeroed here. */
LAB_API lab_status lab_classical_strength(lab_csr A, double theta, int32_t* conn, lab_csr* S,
                                          lab_stream s);
/* PMIS distance-2 aggregation.  aggregates: device int64[m].  rounds (host,
 * optional) receives the number of completed rounds.  Replaces
 * compute_aggregates_using_pmis (amg_aggregation.cpp:106-215). */
LAB_API lab_status lab_pmis_aggregate(lab_csr A, const int32_t* conn, int64_t* aggregates,
                                      int* rounds, lab_stream s);
/* The same aggregation, also returning the reference's root marker array
 * (root_nodes[i] = 1 for aggregate roots, -1 otherwise, amg_aggregation.cpp:168-177).
 * root_nodes (device int64[m]) and rounds may be NULL. */
LAB_API lab_status lab_pmis_aggregate_roots(lab_csr A, const int32_t* conn, int64_t* aggregates,
                                            int64_t* root_nodes, int* rounds, lab_stream s);
/* Smoothed-aggregation prolongation (saamg.cpp:51-207), bit-exact. */
LAB_API lab_status lab_sa_prolongation(lab_csr A, const int32_t* conn, const int64_t* aggregates,
                                       double relax, lab_csr* P, lab_stream s);
/* Unsmoothed-aggregation prolongation (uaamg.cpp:49-128). */
LAB_API lab_status lab_ua_prolongation(lab_csr A, const int64_t* aggregates, lab_csr* P,
                                       lab_stream s);
/* RS C/F splitting, first and second pass (amg_aggregation.cpp:225-251;
 * host_amg_aggregation.cpp:228-519).  cf: device uint32[m]. */
LAB_API lab_status lab_cfpoints(lab_csr S, uint32_t* cf, lab_stream s);
/* Either pass alone: compute_cfpoint_first_pass (first != 0; cf is overwritten)
 * and/or compute_cfpoint_second_pass (second != 0; cf holds a first-pass result). */
LAB_API lab_status lab_cfpoints_passes(lab_csr S, uint32_t* cf, int first, int second,
                                       lab_stream s);
/* RS direct interpolation (rsamg.cpp:672-866). */
LAB_API lab_status lab_direct_interpolation(lab_csr A, lab_csr S, const uint32_t* cf,
                                            lab_csr* P, lab_stream s);

/* ------------------------------------------------------------------ hierarchy */
typedef enum lab_amg_kind
{
    LAB_AMG_SA = 0, /* saamg_setup  (library/include/iterative_solvers/amg/saamg.h:195) */
    LAB_AMG_UA = 1, /* uaamg_setup  (uaamg.h:192) */
    LAB_AMG_RS = 2  /* rsamg_setup  (rsamg.h:208) */
} lab_amg_kind;

/* Build the level hierarchy on the device (max_level capped at 20 as in
 * saamg.cpp:216).  Level 0 is a copy of A.  Replaces
 * saamg_setup / uaamg_setup / rsamg_setup. */
LAB_API lab_status lab_amg_setup(lab_amg_kind kind, lab_csr A, int max_level, lab_hierarchy* h,
                                 lab_stream s);
LAB_API lab_status lab_hierarchy_destroy(lab_hierarchy h);
/* hierarchy::total_levels (amg.h:76-99). */
LAB_API lab_status lab_hierarchy_levels(lab_hierarchy h, int* total_levels);
/* Borrowed handles to A_l (0 <= l <= total_levels) and P_l, R_l (l < total_levels);
 * any output pointer may be NULL.  hierarchy::A_cs / prolongations / restrictions. */
LAB_API lab_status lab_hierarchy_level(lab_hierarchy h, int level, lab_csr* A, lab_csr* P,
                                       lab_csr* R);
/* Setup timing of the last lab_amg_setup on this hierarchy, milliseconds. */
LAB_API lab_status lab_hierarchy_setup_ms(lab_hierarchy h, double* ms);
/* Write a built hierarchy (every A_l, P_l, R_l) to a binary file, and load one
 * back onto the device: a loaded hierarchy is bit-identical to the saved one, so
 * reruns on the same operator skip the setup.  No counterpart in the reference
 * (its hierarchy exists only in memory, amg.h:65-144); the next-row item "hierarchy
 * (de)serialisation".  A file with a bad header, a checksum mismatch or levels
 * whose shapes do not chain is rejected with LAB_BAD_ARG. */
/* lab_spmv_autotune on every level operator, prolongation and restriction; the
 * fused V-cycle passes run on the schedule chosen for their matrix.  Tune before
 * creating preconditioners on h: iteration graphs captured earlier keep their
 * schedules (their results stay correct). */
LAB_API lab_status lab_hierarchy_autotune(lab_hierarchy h, int exact, lab_stream s);
/* SpGEMM table sizing tuner: time C = A*B under every sizing of the hash row classes
 * (the symbolic tables' size against the product bound, the numeric tables' fill) and
 * keep the fastest for products of matrices of A's and B's shapes; later products of
 * such shapes (lab_spgemm, the Galerkin products of lab_amg_setup) use it.  The
 * results do not depend on the sizing (every class accumulates in the reference's
 * order).  lab_hierarchy_tune_products tunes both Galerkin products of every level of
 * a built hierarchy, so the next setup of the same operator runs tuned.  No
 * counterpart in the reference (its SpGEMM descriptors, linalg_math.h:408-440, hold
 * no tuning). */
LAB_API lab_status lab_spgemm_autotune(lab_csr A, lab_csr B, double* best_us, lab_stream s);
LAB_API lab_status lab_hierarchy_tune_products(lab_hierarchy h, lab_stream s);
/* The tuned plans (SpMV schedules from lab_spmv_autotune / lab_hierarchy_autotune,
 * SpGEMM sizings) are cached per process, keyed by the operands' shapes (rows,
 * columns, nonzeros; SpMV also by exactness): a matrix of a cached shape is not timed
 * again.  save / load keep the cache in a text file across processes (a file with a
 * bad header or entry is refused with LAB_BAD_ARG and nothing is loaded); clear empties
 * it.  Host only. */
LAB_API lab_status lab_tune_cache_save(const char* path);
LAB_API lab_status lab_tune_cache_load(const char* path);
LAB_API lab_status lab_tune_cache_clear(void);
LAB_API lab_status lab_hierarchy_save(lab_hierarchy h, const char* path, lab_stream s);
LAB_API lab_status lab_hierarchy_load(const char* path, lab_hierarchy* h, lab_stream s);

/* ------------------------------------------------------------------ cycles */
typedef enum lab_cycle
{
    LAB_CYCLE_V = 0,
    LAB_CYCLE_W = 1,
    LAB_CYCLE_F = 2
} lab_cycle; /* amg.h cycle */

typedef enum lab_smoother
{
    LAB_SMOOTH_JACOBI = 0, /* weighted Jacobi (omega = 1: the reference's jacobi.cpp:43-75) */
    LAB_SMOOTH_GS     = 1, /* multicolour Gauss-Seidel */
    LAB_SMOOTH_SGS    = 2, /* multicolour GS, forward then reverse colour order */
    LAB_SMOOTH_SOR    = 3, /* multicolour SOR, omega_sor */
    LAB_SMOOTH_SSOR   = 4
} lab_smoother; /* amg.h smoother */

typedef enum lab_coarse
{
    LAB_COARSE_DIRECT = 0, /* dense inverse (Gauss-Jordan with partial pivoting) built with
                              the preconditioner, applied as a dense matvec; a coarsest
                              level above 4096 rows falls back to LAB_COARSE_GS */
    LAB_COARSE_GS     = 1  /* the reference's 1000 (V) / 100 (W, F) lexicographic GS sweeps */
} lab_coarse;

typedef enum lab_precision
{
    LAB_PREC_FP64      = 0,
    LAB_PREC_FP32      = 1, /* hierarchy values and V-cycle arithmetic in fp32 */
    LAB_PREC_FP32_BF16 = 2  /* fp32 cycle, bf16 value storage on the two finest levels */
} lab_precision;

typedef struct lab_amg_options
{
    int    n1;        /* pre-smoothing sweeps */
    int    n2;        /* post-smoothing sweeps (n3 = n2 for W/F, amg.cpp:537) */
    int    cycle;     /* lab_cycle */
    int    smoother;  /* lab_smoother */
    double omega;     /* Jacobi weight (1.0 = reference) */
    double omega_sor; /* SOR/SSOR weight (reference 0.5, amg.cpp:133-137) */
    int    coarse;    /* lab_coarse */
    int    precision; /* lab_precision */
} lab_amg_options;

/* Defaults: V-cycle, 1+1 Jacobi with omega 1, omega_sor 0.5, direct coarse solve, fp64. */
LAB_API void lab_amg_options_default(lab_amg_options* o);

typedef struct lab_iter_control
{
    double rel_tol;   /* iter_control.h:52-78: defaults 1e-6 */
    double abs_tol;   /* 1e-6 */
    int    max_iter;  /* 1000 */
    int    max_cycle; /* 200 */
} lab_iter_control;

LAB_API void lab_iter_control_default(lab_iter_control* c);

typedef struct lab_solve_info
{
    int    iterations;       /* the reference's returned count (cg.cpp:222, amg.cpp:570) */
    int    converged;        /* iter_control::residual_converges held */
    double initial_residual; /* ||b - A x0||_inf */
    double final_residual;   /* last ||r||_inf seen by the convergence test */
    double solve_ms;         /* device time of the solve */
    int    status;           /* lab_status of the solve */
} lab_solve_info;

/* One cycle application x <- cycle(x; b) on level 0 (amg.cpp:144-513). */
LAB_API lab_status lab_amg_cycle(lab_hierarchy h, const lab_amg_options* o, const double* b,
                                 double* x, lab_stream s);
/* Stationary AMG iteration.  Replaces amg_solve (amg.h:411-418; amg.cpp:516-571). */
LAB_API lab_status lab_amg_solve(lab_hierarchy h, const lab_amg_options* o, const double* b,
                                 double* x, const lab_iter_control* c, lab_solve_info* info,
                                 lab_stream s);

/* ------------------------------------------------------------------ preconditioners */
/* AMG preconditioner: z = cycle(0; r).  The reference has no AMG preconditioner
 * class; this is the plug-in its abstract preconditioner (preconditioner.h:59-99)
 * admits.  The hierarchy must outlive the preconditioner. */
LAB_API lab_status lab_precond_create_amg(lab_hierarchy h, const lab_amg_options* o,
                                          lab_precond* M, lab_stream s);
/* jacobi_precond (preconditioner.h:101-118; preconditioner.cpp:41-78). */
LAB_API lab_status lab_precond_create_jacobi(lab_csr A, lab_precond* M, lab_stream s);
/* Triangular-solve preconditioners (preconditioner.h:172-580): ILU(0) and IC(0)
 * factor a copy of A (ilu_precond / ic_precond::build), Gauss-Seidel and SOR(omega)
 * solve with the lower part of a copy of A (gauss_seidel_precond, SOR_precond),
 * SSOR(omega) with the two triangles SSOR_precond::build makes from A.  Each
 * application runs the reference's triangular solves, bit-identical.  All need
 * 0 < omega < 2 where they take one. */
LAB_API lab_status lab_precond_create_ilu0(lab_csr A, lab_precond* M, lab_stream s);
LAB_API lab_status lab_precond_create_ic0(lab_csr A, lab_precond* M, lab_stream s);
LAB_API lab_status lab_precond_create_gauss_seidel(lab_csr A, lab_precond* M, lab_stream s);
LAB_API lab_status lab_precond_create_sor(lab_csr A, double omega, lab_precond* M, lab_stream s);
LAB_API lab_status lab_precond_create_ssor(lab_csr A, double omega, lab_precond* M, lab_stream s);
/* z = M^{-1} r.  preconditioner::solve (preconditioner.h:78). */
LAB_API lab_status lab_precond_apply(lab_precond M, const double* r, double* z, lab_stream s);
LAB_API lab_status lab_precond_destroy(lab_precond M);

/* ------------------------------------------------------------------ Krylov */
/* (P)CG with the reference's update order and stopping test (cg.cpp:136-223;
 * unpreconditioned path cg.cpp:60-134 restarts every iteration as the reference
 * does with restart_iter = -1).  b, x: device pointers; x holds the initial
 * guess.  All scalars stay on the device; the whole iteration is one CUDA graph.
 * Returns LAB_OK when converged, LAB_NOT_CONVERGED after max_iter. */
LAB_API lab_status lab_pcg_solve(lab_csr A, lab_precond M, const double* b, double* x,
                                 const lab_iter_control* c, lab_solve_info* info, lab_stream s);
/* Restarted GMRES(restart) with modified Gram-Schmidt and Givens rotations,
 * right-preconditioned by M (NULL: none).  Replaces gmres_solver
 * (gmres.h:228-346; gmres.cpp). */
LAB_API lab_status lab_gmres_solve(lab_csr A, lab_precond M, int restart, const double* b,
                                   double* x, const lab_iter_control* c, lab_solve_info* info,
                                   lab_stream s);

/* ------------------------------------------------------------------ batching
 * Many independent systems in one solve (no reference counterpart).
 *
 * lab_csr_block_diag stacks nblocks matrices into one block-diagonal matrix
 * (offsets[k] = first row of block k, host int64[nblocks + 1] written on return).
 * One AMG setup on it builds every system's hierarchy at once: strength,
 * aggregation, prolongation and Galerkin products never couple blocks. */
LAB_API lab_status lab_csr_block_diag(const lab_csr* blocks, int nblocks, lab_csr* out,
                                      int64_t* offsets, lab_stream s);
/* Batched PCG: system k owns rows [offsets[k], offsets[k+1]) of A (host
 * int64[nsys + 1]) and b / x.  Each system has its own alpha, beta, stopping
 * test (the reference's, per system) and iteration count; a converged system
 * stops updating (per-system convergence mask) while the others continue.
 * iterations / converged: host int[nsys] (may be NULL).  info summarises the
 * batch (iterations = max over systems, converged = all converged). */
LAB_API lab_status lab_batched_pcg_solve(lab_csr A, lab_precond M, int nsys,
                                         const int64_t* offsets, const double* b, double* x,
                                         const lab_iter_control* c, int* iterations,
                                         int* converged, lab_solve_info* info, lab_stream s);
/* Split nsys independent systems of the given costs (e.g. nonzeros) over nparts
 * workers, one per GPU: part[k] in [0, nparts) for each system, size-balanced by
 * the longest-processing-time greedy rule (largest first, to the least-loaded
 * worker; deterministic).  Host only, no device needed.  The workers solve their
 * systems independently (no collective on the data path); the caller gathers the
 * solutions.  No reference counterpart (the reference has no multi-GPU code). */
LAB_API lab_status lab_batch_partition(int nsys, const int64_t* cost, int nparts, int* part);
/* Block PCG for nrhs right-hand sides of one matrix: B and X are n x nrhs
 * column-major (leading dimension n).  Every column has its own scalars and
 * stopping test; the products with A use SpMM (one pass over A per block of 8
 * columns). */
LAB_API lab_status lab_multi_rhs_pcg_solve(lab_csr A, lab_precond M, int nrhs, const double* B,
                                           double* X, const lab_iter_control* c, int* iterations,
                                           int* converged, lab_solve_info* info, lab_stream s);

/* ------------------------------------------------------------------ adjoint
 * Differentiation of x = A^{-1} b for a loss L(x) (no reference counterpart:
 * LinAlgLib has no derivatives).  The forward iterates are not stored; the
 * adjoint is a second solve.
 *
 * lambda = A^{-T} g with g = dL/dx, which is dL/db.  symmetric != 0: A^T = A and
 * the solve is PCG with M (a symmetric preconditioner: the AMG cycle with equal
 * pre-/post-smoothing, or Jacobi).  symmetric == 0: A^T is formed and solved
 * with GMRES(restart 50) preconditioned by M when M was built from A^T, else
 * unpreconditioned (M = NULL). */
LAB_API lab_status lab_adjoint_solve(lab_csr A, lab_precond M, int symmetric, const double* g,
                                     double* lambda, const lab_iter_control* c,
                                     lab_solve_info* info, lab_stream s);
/* dL/dA restricted to A's sparsity pattern: grad[j] = -lambda[i] * x[col[j]] for
 * every stored entry j of row i (grad has A's nnz layout). */
LAB_API lab_status lab_adjoint_grad_A(lab_csr A, const double* lambda, const double* x,
                                      double* grad, lab_stream s);

/* Same solve, host buffers: b and x are HOST pointers, copied in and out inside
 * the call (the end-to-end form the C++ API uses for host-resident vectors). */
LAB_API lab_status lab_pcg_solve_host(lab_csr A, lab_precond M, const double* b_host,
                                      double* x_host, const lab_iter_control* c,
                                      lab_solve_info* info, lab_stream s);

#ifdef __cplusplus
}
#endif
#endif /* LAB_H */
