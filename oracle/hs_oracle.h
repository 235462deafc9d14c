/*
 * hs_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of TimThuering/Heterogeneous-Solvers' blocked SPD solve path
 * (its CPU path: init_gpu_perc=0, cpu_opt=2).  It is the checker for the CUDA
 * library, never part of it: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs load it.  Every function cites the reference
 * file:line whose arithmetic it restates (paths relative to the reference root).
 *
 * Storage convention (src/dataStructures/SymmetricMatrix.hpp:9-35): the lower
 * block triangle of an N x N symmetric matrix is cut into bsz x bsz blocks,
 * enumerated column by column; block (i,j), i >= j, has id
 *     i + nb(nb-1)/2 - (nb-j-1)(nb-j)/2,   nb = ceil(N/bsz)
 * and element (r,c) of a block sits at id*bsz*bsz + r*bsz + c (row major).
 * Diagonal blocks hold both triangles; padding rows/cols (global index >= N)
 * are zero.
 *
 * Parity: pinned against the reference's own GoogleTest golden vectors
 * (the tests/test*.cpp files and the tests/testData fixtures), extracted into
 * tests/golden/ by tests/golden/extract_reference_tests.py.
 */
#ifndef HS_ORACLE_H
#define HS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* block id of block (i,j), i >= j — SymmetricMatrix.hpp:9-35, MatrixGenerator.cpp:108-117 */
int64_t or_block_id(int64_t i, int64_t j, int64_t nb);

/* POTRF of one diagonal block — MatrixOperations.cpp:7-62 */
void or_potrf_block(double* A, int64_t N, int bsz, int blockID, int blockRow);
/* TRSM B <- B L^-T on a sub-column — MatrixMatrixOperations.cpp:109-144 */
void or_trsm_panel(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount);
/* SYRK on diagonal blocks — MatrixMatrixOperations.cpp:307-361 */
void or_syrk_diag(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount, int nb);
/* GEMM trailing update — MatrixMatrixOperations.cpp:845-906 */
void or_gemm_trailing(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount, int nb);

/* symmetric block matvec on a block sub-rectangle — MatrixVectorOperations.cpp:8-93 */
void or_symv_block(const double* A, const double* b, double* result, int bsz, int bi0, int bj0,
                   int nbi, int nbj, int nb, int reset);
/* single-block triangular solve — MatrixVectorOperations.cpp:282-335 */
void or_trsv_block(const double* A, double* b, int64_t N, int bsz, int blockRow, int blockID, int transposed);
/* block-column update b_i -= A_ij b_j — MatrixVectorOperations.cpp:337-377 */
void or_column_update(const double* A, double* b, int bsz, int blockStart, int blockCount, int blockRow,
                      int blockID, int nb, int transposed);

/* vector ops — VectorOperations.cpp:6-82 */
void or_scale_block(const double* x, double alpha, double* result, int bsz, int bi0, int nbi);
void or_add_block(const double* x, const double* y, double* result, int bsz, int bi0, int nbi);
void or_sub_block(const double* x, const double* y, double* result, int bsz, int bi0, int nbi);
void or_axpy_block(const double* x, double alpha, const double* y, double* result, int bsz, int bi0, int nbi);
/* dot product, per-chunk partial sums then a serial sum — VectorOperations.cpp:187-238 */
double or_dot_block(const double* x, const double* y, int bsz, int bi0, int nbi, int chunks);

/* right-looking blocked Cholesky driver, CPU path — Cholesky.cpp:413-493 */
void or_cholesky(double* A, int64_t N, int bsz);
/* forward + backward block substitution in place on b — TriangularSystemSolver.cpp:15-105 */
void or_triangular_solve(const double* L, double* b, int64_t N, int bsz);
/* CG driver — CG.cpp:38-163, 277-528.  Returns the iteration count. */
int64_t or_cg(const double* A, const double* b, double* x, int64_t N, int bsz, double eps, int64_t imax,
              int chunks, double* delta_new_out, double* delta_zero_out);

/* RBF kernel-matrix assembly — MatrixGenerator.cpp:134-155, generalised to
 * X (N x d, row major), per-dimension lengthscales (n_ell == 1: isotropic,
 * reference formula; n_ell == d: ARD). */
void or_rbf_assemble(double* A, const double* X, int64_t N, int d, int bsz, const double* ell, int n_ell,
                     double sf2, double sn2);
/* sliding-window inputs of the reference generator — MatrixGenerator.cpp:76-99:
 * X[i][k] = s[i+k-7] (7 leading zeros), d = 8 */
/* MatrixGenerator::generateTestKernelMatrix (MatrixGenerator.cpp:163-213) on
 * row-major inputs: K_star[j*N + i] */
void or_test_kernel_matrix(const double* X, int64_t N, const double* Xt, int64_t Nt, int d, const double* ell,
                           int n_ell, double sf2, double* K_star);
/* MatrixVectorOperations::matrixVectorGP (MatrixVectorOperations.cpp:379-395) */
void or_matrix_vector_gp(const double* A, const double* b, double* result, int64_t n, int64_t m);
void or_window_inputs(const double* series, int64_t N, double* X);

#ifdef __cplusplus
}
#endif
#endif
