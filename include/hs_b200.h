/*
 * hs_b200.h — C ABI of the B200-native blocked SPD solve path.
 *
 * Drop-in for TimThuering/Heterogeneous-Solvers' blocked SPD path for Gaussian-
 * process kernel matrices.  Every entry point below names the reference
 * interface it replaces (file:line relative to the reference's root).  The
 * reference passes a sycl::queue plus globals conf::N / conf::matrixBlockSize
 * (src/utility/Configuration.hpp:21-118); here a context carries the CUDA
 * device, stream and the problem size, and every call takes the same integer
 * block arguments, in the same order, as the reference kernel it replaces.
 *
 * Matrix storage (src/dataStructures/SymmetricMatrix.hpp:9-54): the lower
 * block triangle of an N x N symmetric matrix in nb = ceil(N/bsz) blocks per
 * side, T = nb(nb+1)/2 blocks of bsz*bsz doubles, enumerated column by column;
 * block (i,j), i >= j, has id i + nb(nb-1)/2 - (nb-j-1)(nb-j)/2; row-major
 * inside a block; diagonal blocks hold both triangles; padding is zero.
 * Vectors (src/dataStructures/RightHandSide.hpp:12-30) are nb*bsz doubles,
 * zero padded.
 *
 * Conventions: unless a parameter says "host", pointers are device pointers.
 * All work is ordered on the context's stream; hs_sync() waits for it.
 * Operator-level calls (hs_potrf_block ... hs_dot_block) launch and return.
 * No C++ exception crosses this boundary: every call returns an hs_status and
 * hs_last_error() gives the message of the calling thread's last failure.
 */
#ifndef HS_B200_H
#define HS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HS_B200_ABI_VERSION 1

typedef enum hs_status {
    HS_OK = 0,
    HS_ERR_INVALID_ARG = 1,       /* reference: std::invalid_argument / std::runtime_error */
    HS_ERR_OOM = 2,               /* reference: "Error during GPU memory allocation" (CG.cpp:231-233) */
    HS_ERR_NOT_SPD = 3,           /* reference: silent NaN (MatrixOperations.cpp:24) */
    HS_ERR_NO_CONVERGENCE = 4,    /* CG reached iMax (CG.cpp:78) */
    HS_ERR_REFINEMENT_STALLED = 5,/* mixed precision: refinement stopped improving */
    HS_ERR_CUDA = 6,
    HS_ERR_TIMEOUT = 7,           /* a bounded device-side wait gave up */
    HS_ERR_UNSUPPORTED = 8
} hs_status;

typedef struct hs_ctx_s* hs_ctx;

/* ------------------------------------------------------------------ context */
int hs_abi_version(void);
const char* hs_last_error(void);
const char* hs_status_string(hs_status s);

/* Create a context on `device`.  `stream` is the caller's cudaStream_t on which
 * every call of this context is ordered; NULL selects the CUDA default stream.
 * The context never destroys the caller's stream. */
hs_status hs_ctx_create(int device, void* stream, hs_ctx* out);
hs_status hs_ctx_destroy(hs_ctx ctx);
hs_status hs_ctx_set_stream(hs_ctx ctx, void* stream);
/* The context keeps grow-only device buffers between calls (reduction partials,
 * matvec partial sums, solver work vectors, the mixed-precision and NLML workspaces,
 * the device copies of hs_gp_solve_host);
 * this frees them all (after synchronising the stream).  They are allocated
 * again by the next call that needs them.  No reference counterpart (the
 * reference's solvers free their device copies in their destructors,
 * Cholesky.cpp:18-22). */
hs_status hs_ctx_release_buffers(hs_ctx ctx);
/* conf::N and conf::matrixBlockSize (Configuration.hpp:22, :33).  Sets nb. */
hs_status hs_ctx_set_problem(hs_ctx ctx, int64_t N, int matrixBlockSize);
hs_status hs_sync(hs_ctx ctx);
/* number of doubles of the packed matrix / of a padded vector for (N, bsz):
 * SymmetricMatrix.cpp:11-19, RightHandSide.cpp:8-15 */
int64_t hs_packed_matrix_size(int64_t N, int matrixBlockSize);
int64_t hs_padded_vector_size(int64_t N, int matrixBlockSize);

/* Instrumentation.  With profiling on, every launch of the kernels below is
 * bracketed by CUDA events on the stream it is launched on; hs_ctx_read_profile
 * synchronises, folds the finished pairs into per-kernel totals and returns
 * them (launches, summed device ms, algorithmic flops and bytes of those
 * launches).  hs_ctx_launch_count counts every kernel launched through the
 * context since its creation. */
typedef enum hs_kernel_id {
    HS_KERNEL_UPDATE = 0,    /* SYRK + GEMM trailing update (FP64) */
    HS_KERNEL_POTRF = 1,
    HS_KERNEL_TRSM = 2,
    HS_KERNEL_SYMV = 3,      /* symmetric block matvec, both phases */
    HS_KERNEL_TRSV = 4,
    HS_KERNEL_COLUPD = 5,
    HS_KERNEL_ASSEMBLE = 6,
    HS_KERNEL_VECTOR = 7,    /* vector ops, dots, CG updates */
    HS_KERNEL_ADJOINT = 8,   /* reverse-mode Cholesky block products (FP64 DMMA) */
    HS_KERNEL_GRAD = 9,      /* GP gradient contraction */
    HS_KERNEL_UPDATE_SIDE = 10, /* mixed factor: trailing-update launches on the look-ahead stream
                                   (flops are counted where the tiles are: the in-group updates
                                   here, a shared update's tiles with its first launch) */
    HS_KERNEL_COUNT = 11
} hs_kernel_id;
typedef struct hs_kernel_profile {
    int64_t launches;
    double ms;
    double flops;
    double bytes;
} hs_kernel_profile;
hs_status hs_ctx_set_profiling(hs_ctx ctx, int enable);
hs_status hs_ctx_read_profile(hs_ctx ctx, int kernel, hs_kernel_profile* out);
hs_status hs_ctx_reset_profile(hs_ctx ctx);
int64_t hs_ctx_launch_count(hs_ctx ctx);

/* Reference accumulation order.  cpu_chunks > 0 makes hs_symv_block, hs_dot_block,
 * the vector updates and hs_cg_solve follow the arithmetic of the reference's CPU
 * path exactly: one running sum per matrix row in block order
 * (MatrixVectorOperations.cpp:194-280), multiplies and adds rounded separately,
 * dot products summed in `cpu_chunks` sequential chunks and then in chunk order
 * (VectorOperations.cpp:187-238, whose chunk count is the CPU's core count).
 * CG then reproduces the reference's iterates bit for bit; it is a parity mode,
 * far slower than the default (0: fused, tree-reduced kernels). */
hs_status hs_ctx_set_reference_order(hs_ctx ctx, int cpu_chunks);

/* Mixed-precision factor (no reference counterpart): `panels` (1, 2 or 4) trailing-update
 * panel products are summed in the tensor cores' FP32 accumulator as one unit; the units
 * of an output tile are then summed with round-to-nearest FP32 adds in registers before
 * one add into the FP32 working matrix.  Fewer panels a unit is the more accurate factor:
 * at N=131072 one panel (the default) gives a 3.8x smaller log|K| error than four and 3
 * refinement steps instead of 5 for ~1 % more factor time (solve 2222 against 2257 ms);
 * hs_mixed_solve's x reaches its target either way.  hs_gp_nlml_grad_mixed always uses
 * one panel. */
hs_status hs_ctx_set_mixed_accumulation(hs_ctx ctx, int panels);

/* Mixed-precision factor (no reference counterpart): look-ahead by one panel group.
 * While at least `min_rows` rows follow the next group of 4 panels, that group's
 * diagonal blocks, panel TRSMs and in-group updates run on a high-priority stream on
 * `side_sms` SMs, beside the trailing update of the current group on the others; the
 * update's remaining tiles are then shared with a second launch on those SMs.
 * side_sms = 0 keeps the look-ahead by one diagonal block.  Defaults: 16 SMs, 24576
 * rows.  The factor is the same bit for bit either way: every block receives the same
 * products in the same order.  side_sms must be in [0, SMs / 2], min_rows >= 0. */
hs_status hs_ctx_set_mixed_lookahead(hs_ctx ctx, int side_sms, int min_rows);

/* ------------------------------------------------------------------ operators */
/* MatrixOperations::cholesky / cholesky_GPU / cholesky_optimizedGPU
 * (src/kernel/MatrixOperations.hpp:23,39,55; MatrixOperations.cpp:7-191):
 * in-place POTRF of diagonal block blockID (= block row blockRow); rows with
 * global index >= N untouched; the upper triangle becomes zero.  A non-positive
 * pivot is recorded in the context (see hs_ctx_take_info). */
hs_status hs_potrf_block(hs_ctx ctx, double* A, int blockID, int blockRow);
/* Read (and reset) the context's pivot record: *info = -1 when every POTRF since
 * the last call saw positive pivots, else the smallest failing global row.
 * Synchronises the stream. */
hs_status hs_ctx_take_info(hs_ctx ctx, int64_t* info);
/* Self-test of the failure path of every device-side wait in the library (no
 * reference counterpart): one device thread waits on a flag that nothing sets, with
 * the bounded wait the sweeps and tensor-core kernels use, for timeout_ns
 * (1e6 .. 2e9).  Returns HS_ERR_TIMEOUT when the wait ran out (the expected
 * outcome; the context stays usable), HS_OK if the flag was seen set. */
hs_status hs_selftest_bounded_wait(hs_ctx ctx, int64_t timeout_ns);

/* MatrixMatrixOperations::triangularSolve{,_optimizedGPU,_optimizedCPU}
 * (MatrixMatrixOperations.hpp:29,53,77; .cpp:5-144): B <- B L^-T for the blocks
 * at rows blockStart .. blockStart+blockCount-1 of block column blockRow. */
hs_status hs_trsm_panel(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount);

/* MatrixMatrixOperations::symmetricMatrixMatrixDiagonal{,_optimizedGPU,_optimizedCPU}
 * (MatrixMatrixOperations.hpp:98,121,145; .cpp:146-361): A_jj <- A_jj - L_jk L_jk^T,
 * lower triangle only, for diagonal blocks j in [blockStart, blockStart+blockCount). */
hs_status hs_syrk_diag(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                       int blockCountXY);

/* MatrixMatrixOperations::matrixMatrixStep{,_optimizedGPU,2,3,_optimizedCPU,2}
 * (MatrixMatrixOperations.hpp:168-290; .cpp:364-906): A_rc <- A_rc - L_rk L_ck^T
 * for blockRow < c < r, r in [blockStart, blockStart+blockCount). */
hs_status hs_gemm_trailing(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                           int blockCountXY);

/* MatrixVectorOperations::matrixVectorBlock{,_GPU,_CPU}
 * (MatrixVectorOperations.hpp:27,47,67; .cpp:8-280): result[rows of block rows
 * blockStart_i ..] (reset ? = : +=) A_sub b over the block sub-rectangle
 * [blockStart_i, +blockCount_i) x [blockStart_j, +blockCount_j) of the full
 * symmetric matrix.  Each stored block is read once and applied as A_ij and
 * A_ij^T (deterministic two-phase reduction; uses context scratch). */
hs_status hs_symv_block(hs_ctx ctx, const double* A, const double* b, double* result, int blockStart_i,
                        int blockStart_j, int blockCount_i, int blockCount_j, int blockCountXY, int reset);

/* No counterpart in the reference.  The same product as hs_symv_block, for callers
 * that cannot let the library allocate device memory (an application whose own
 * allocator already holds the free memory, or a latency-critical loop that cannot
 * afford the device-wide synchronisation of cudaMalloc/cudaFree).  Its partial sums
 * live in a fixed device array of HS_SYMV_NOALLOC_MAX_DOUBLES doubles (16 MiB) that
 * every GPU loading the library holds until the process exits; no call allocates or
 * frees anything.  A rectangle needing more than that
 * (blockCount_i * blockCount_j * matrixBlockSize doubles) is rejected with
 * HS_ERR_INVALID_ARG.  All calls on a device share the array, so calls whose
 * kernels can overlap on that device race on it: order them on one stream.  The
 * first call on each device (and the first after a reset of its context) looks up
 * the array's device address, with that device current; make that first call
 * before any stream capture starts.  Devices 0..63.  In reference-order mode
 * (hs_ctx_set_reference_order) it runs hs_symv_block's reference-order kernel,
 * which uses no scratch: the two entry points give the same bits in both modes. */
#define HS_SYMV_NOALLOC_MAX_DOUBLES (2 * 1024 * 1024)
hs_status hs_symv_block_noalloc(hs_ctx ctx, const double* A, const double* b, double* result, int blockStart_i,
                                int blockStart_j, int blockCount_i, int blockCount_j, int blockCountXY, int reset);

/* MatrixVectorOperations::triangularSolveBlockVector (MatrixVectorOperations.hpp:81;
 * .cpp:282-335): b_blockRow <- L^-1 b_blockRow (transposed: L^-T). */
hs_status hs_trsv_block(hs_ctx ctx, const double* A, double* b, int blockRow, int blockID, int transposed);

/* MatrixVectorOperations::matrixVectorColumnUpdate (MatrixVectorOperations.hpp:99;
 * .cpp:337-377): b_i -= A_{i,blockRow} b_blockRow for i in [blockStart, +blockCount)
 * (transposed: b_i -= A_{blockRow,i}^T b_blockRow). */
hs_status hs_column_update(hs_ctx ctx, const double* A, double* b, int blockStart, int blockCount, int blockRow,
                           int blockID, int blockCountXY, int transposed);

/* VectorOperations (VectorOperations.hpp:21-95; .cpp:6-185) on rows of block rows
 * [blockStart_i, blockStart_i + blockCount_i): */
hs_status hs_scale_block(hs_ctx ctx, const double* x, double alpha, double* result, int blockStart_i,
                         int blockCount_i);                                  /* scaleVectorBlock        :6   */
hs_status hs_add_block(hs_ctx ctx, const double* x, const double* y, double* result, int blockStart_i,
                       int blockCount_i);                                    /* addVectorBlock          :25  */
hs_status hs_sub_block(hs_ctx ctx, const double* x, const double* y, double* result, int blockStart_i,
                       int blockCount_i);                                    /* subVectorBlock          :45  */
hs_status hs_axpy_block(hs_ctx ctx, const double* x, double alpha, const double* y, double* result,
                        int blockStart_i, int blockCount_i);                 /* scaleAndAddVectorBlock  :64  */
/* scalarProduct + sumFinalScalarProduct (:84-185): result[0] (device) = x.y,
 * deterministic two-stage tree reduction (uses context scratch). */
hs_status hs_dot_block(hs_ctx ctx, const double* x, const double* y, double* result, int blockStart_i,
                       int blockCount_i);

/* ------------------------------------------------------------------ solvers */
/* MatrixGenerator::generateSPDMatrix (src/utility/MatrixGenerator.cpp:73-162), its
 * per-entry formula generalised from the 1-D sliding window to X (N x d, row
 * major, device): K_ij = sf2 * exp(-0.5/l^2 * |x_i - x_j|^2) + sn2 [i == j].
 * `ell` (host) holds 1 (isotropic) or d (ARD) lengthscales.  Writes all T
 * blocks, padding as zero. */
hs_status hs_rbf_assemble(hs_ctx ctx, double* A, const double* X, int d, const double* ell, int n_ell,
                          double sf2, double sn2);

/* Cholesky::solve_heterogeneous with the whole matrix on the GPU
 * (src/solver/cholesky/Cholesky.cpp:413-493): A (packed, device) is overwritten
 * by L.  *info (host, may be NULL) = -1 on success, else the global row of the
 * first non-positive pivot (then HS_ERR_NOT_SPD). */
hs_status hs_cholesky_factor(hs_ctx ctx, double* A, int64_t* info);

/* TriangularSystemSolver::solve (TriangularSystemSolver.cpp:15-105): b <- L^-T L^-1 b
 * in place (device). */
hs_status hs_cholesky_solve(hs_ctx ctx, const double* L, double* b);

/* CG::solveHeterogeneous with the whole matrix on the GPU (src/solver/cg/CG.cpp:38-163):
 * x (device) starts at zero; stop when delta_new <= epsilon^2 delta_0 or after iMax
 * iterations; true residual every 50 iterations (CG.cpp:95-101).  Outputs are host
 * pointers and may be NULL.  Returns HS_ERR_NO_CONVERGENCE when iMax is reached. */
hs_status hs_cg_solve(hs_ctx ctx, const double* A, const double* b, double* x, double epsilon, int64_t iMax,
                      int64_t* iterations, double* delta_new, double* delta_zero);

/* End-to-end GP solve through host buffers, the path of GaussianProcess::start's
 * solve (src/gaussianProcess/GaussianProcess.cpp:20-40) and main.cpp:201-249:
 * X_host (N x d), y_host (N) -> RBF assembly -> factor + solve (algorithm 0),
 * CG (algorithm 1: epsilon, iMax as in hs_cg_solve) or the mixed-precision solve
 * (no reference counterpart: algorithm 2 with 3xTF32, 3 with BF16-split, 4 with
 * FP16-split updates;
 * epsilon = backward-error target, iMax = refinement step limit;
 * report->factor_ms then covers factor and refinement) ->
 * x_host (N).  The device copies (X, the packed K, y, x) are kept by the context
 * between calls; hs_ctx_release_buffers frees them. */
typedef struct hs_solve_report {
    int64_t info;            /* factor: -1 or failing row */
    int64_t iterations;      /* CG iterations (algorithm 1) */
    double assemble_ms, factor_ms, solve_ms, total_ms;
} hs_solve_report;
hs_status hs_gp_solve_host(hs_ctx ctx, const double* X_host, const double* y_host, int d, const double* ell,
                           int n_ell, double sf2, double sn2, int algorithm, double epsilon, int64_t iMax,
                           double* x_host, hs_solve_report* report);

/* ------------------------------------------------------------------ mixed precision
 * No reference counterpart (new form).  hs_mixed_solve factors K (packed FP64,
 * device, left unchanged) in FP32 with the panel TRSM and the SYRK/GEMM trailing
 * updates on the tensor cores (tcgen05 kind::tf32, 3xTF32 split products, FP32
 * accumulation) and every diagonal-block POTRF in FP64.  HS_PRECISION_BF16X3
 * runs the trailing updates instead as BF16 split products (hi = bf16(x),
 * lo = bf16(x - hi), hi*hi + hi*lo + lo*hi on tcgen05 kind::f16, FP32
 * accumulation; ~2^-16 relative per product), the TRSM staying 3xTF32.
 * HS_PRECISION_F16X3 runs them as FP16 split products of the panel scaled by a
 * power of two s (hi = fp16(s x), lo = fp16(s x - hi): 22 significant bits, ~2^-22
 * relative per product, at the BF16 rate; s = 2^e, the largest e with
 * s sqrt(max_i K_ii) <= 2^15, is exact and is undone in the FP32 epilogue: every
 * |L_ij| <= sqrt(K_ii), so the scaled panel stays inside the FP16 range).  It then refines
 * x <- x + (L L^T)^-1 (b - K x) with FP64 residuals until the backward error
 * ||b - K x|| / (||K||_F ||x||) <= tol.  When refinement stops contracting it
 * continues with conjugate gradients preconditioned by the FP32 factor.  b and x
 * are device vectors of hs_padded_vector_size doubles.  The workspace (FP32
 * factor: half the packed matrix) is kept by the context between calls.  When
 * the low-precision factor of K meets a non-positive pivot (K too ill-conditioned
 * for it; the factorization stops at that block), a BF16- or FP16-split factor is
 * redone with 3xTF32 products (an FP16 split that met a finite negative pivot is not),
 * and then K + shift*I is factored, the shift growing from the failing pivot's size (at
 * least 1e-6 times the largest diagonal entry, 10x the previous shift, at most 0.05x), the
 * solve going straight to CG preconditioned by that factor (report->shift, report->precision_used;
 * report->logdet is then the log-determinant of the shifted matrix).  Returns HS_ERR_REFINEMENT_STALLED
 * when the target is not reached, HS_ERR_NOT_SPD when every shift fails. */
typedef enum hs_precision {
    HS_PRECISION_FP64 = 0,
    HS_PRECISION_TF32X3 = 1,
    HS_PRECISION_BF16X3 = 2,
    HS_PRECISION_F16X3 = 3
} hs_precision;
typedef struct hs_mixed_report {
    int64_t refinement_steps;
    int64_t pcg_iterations;
    int fallback_pcg;
    int factor_attempts;     /* 1 unless the low-precision factor of K broke down and was redone */
    int precision_used;      /* split products of the factor that was used (HS_PRECISION_*) */
    int reserved;
    double shift;            /* diagonal shift of the low-precision factor (0: factor of K itself) */
    double backward_error;   /* ||b - K x|| / (||K||_F ||x||) at exit */
    double initial_backward_error; /* the same for x0 = (L L^T)^-1 b, before any refinement */
    double norm_k_fro;
    double logdet;           /* log|K| = 2 sum log diag(L) from the FP64 diagonal blocks */
    double factor_ms, refine_ms, total_ms;
} hs_mixed_report;
hs_status hs_mixed_solve(hs_ctx ctx, const double* K, const double* b, double* x, int precision, double tol,
                         int max_steps, hs_mixed_report* report);

/* log|K| = 2 sum_i log L_ii of a factor from hs_cholesky_factor (packed, device);
 * *logdet is a host pointer. */
hs_status hs_cholesky_logdet(hs_ctx ctx, const double* L, double* logdet);

/* ------------------------------------------------------------------ prediction
 * MatrixGenerator::generateTestKernelMatrix (src/utility/MatrixGenerator.cpp:163-213):
 * K_star[j*N + i] = sf2 exp(-0.5/l^2 sum_k (x_ik - x*_jk)^2) for training rows
 * X (N x d, N of the context) and test rows X_test (N_test x d), row major,
 * device; `ell` (host) holds 1 or d lengthscales (ARD: each difference scaled
 * by 1/l_k).  The reference's sliding window is X[i][k] = series[i+k-7]. */
hs_status hs_gp_test_kernel_matrix(hs_ctx ctx, const double* X, const double* X_test, int64_t N_test, int d,
                                   const double* ell, int n_ell, double sf2, double* K_star);
/* MatrixVectorOperations::matrixVectorGP (src/kernel/MatrixVectorOperations.hpp:113,
 * .cpp:379-395): result[i] = sum_k A[i*n + k] b[k] for i < m (A dense m x n). */
hs_status hs_matrix_vector_gp(hs_ctx ctx, const double* A, const double* b, double* result, int64_t n, int64_t m);
/* The two calls above fused (GaussianProcess::start's prediction,
 * src/gaussianProcess/GaussianProcess.cpp:42-54): mean[j] = sum_i K_star[j][i]
 * alpha[i] with K_star recomputed on the fly and never stored.  alpha = K^-1 y
 * (N values, device), mean (N_test, device). */
hs_status hs_gp_predict(hs_ctx ctx, const double* X, const double* X_test, int64_t N_test, int d, const double* ell,
                        int n_ell, double sf2, const double* alpha, double* mean);

/* ------------------------------------------------------------------ differentiation
 * No reference counterpart (new form).  Reverse-mode blocked Cholesky: with L
 * the packed factor of A = L L^T (hs_cholesky_factor) and Abar holding, on
 * entry, the adjoint Lbar of some scalar f with respect to the lower blocks of
 * L (only the lower triangle of its diagonal blocks is read), Abar is
 * overwritten by the adjoint of f with respect to the lower entries of A
 * (entry (i,j), i >= j, of the packed storage: df = sum_{i>=j} Abar_ij dA_ij).
 * Products run on the FP64 tensor cores; matrixBlockSize 128 or 256.  L is not
 * modified.  Allocates a workspace of (nb + 132) blocks. */
hs_status hs_cholesky_adjoint(hs_ctx ctx, const double* L, double* Abar);

/* GP negative log marginal likelihood and its gradient.  X (N x d, row major)
 * and y (N) are device arrays; theta (host) = [log l_1 .. log l_n_ell, log sf2,
 * log sn2] with n_ell = 1 (isotropic) or d (ARD), K = sf2 exp(-1/2 sum_k
 * (x_ik - x_jk)^2 / l_k^2) + sn2 I (hs_rbf_assemble's matrix).
 *   *nlml = 1/2 y^T K^-1 y + 1/2 log|K| + N/2 log 2pi
 *   grad[q] = dNLML/dtheta_q = 1/2 tr((K^-1 - alpha alpha^T) dK/dtheta_q)
 * (host, n_ell + 2 values; may be NULL).  FP64 factor on the tensor cores,
 * the gradient through hs_cholesky_adjoint of sum log L_ii and an on-the-fly
 * contraction that recomputes dK/dtheta from X (nothing of size N^2 besides L
 * and its adjoint is stored; that workspace is kept by the context between
 * calls, see hs_ctx_release_buffers).  d <= 32; matrixBlockSize 128 or 256.  Returns
 * HS_ERR_NOT_SPD when K(theta) has no Cholesky factor. */
typedef struct hs_gp_report {
    double factor_ms, adjoint_ms, grad_ms, total_ms;
    double data_fit;   /* 1/2 y^T K^-1 y */
    double logdet;     /* log|K| */
} hs_gp_report;
hs_status hs_gp_nlml_grad(hs_ctx ctx, const double* X, const double* y, int d, const double* theta, int n_ell,
                          double* nlml, double* grad, hs_gp_report* report);

/* The same NLML and gradient through the mixed-precision factor (no reference
 * counterpart): the factor of hs_mixed_solve with `precision` (HS_PRECISION_*),
 * alpha = K^-1 y refined in FP64 to the backward error `tol`, log|K| from the
 * factor's FP64 diagonal blocks, and the FP64 reverse sweep run on the mixed
 * factor widened to FP64.  alpha (hence the data-fit term) has FP64 accuracy;
 * log|K| and the trace term 1/2 tr(K^-1 dK/dtheta) carry the error of the
 * low-precision factor (K~ = L~ L~^T = K + E gives log|K~| - log|K| =
 * tr(K^-1 E) - 1/2 ||K^-1/2 E K^-1/2||_F^2 + ...).  The workspace holds K, the
 * mixed factor and the adjoint: about 2.5x the packed K.  HS_ERR_NOT_SPD when the
 * factor needed a diagonal shift.  mixed_report (nullable) gets the solve's report. */
hs_status hs_gp_nlml_grad_mixed(hs_ctx ctx, const double* X, const double* y, int d, const double* theta, int n_ell,
                                int precision, double tol, double* nlml, double* grad, hs_gp_report* report,
                                hs_mixed_report* mixed_report);

#ifdef __cplusplus
}
#endif
#endif
