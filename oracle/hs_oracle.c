/*
 * hs_oracle.c — TEST INFRASTRUCTURE ONLY (see hs_oracle.h).
 *
 * Plain C + OpenMP restatement of the reference's CPU path.  Each function keeps
 * the reference's per-element accumulation order, so results do not depend on
 * the thread count (the dot product takes its chunk count explicitly, as the
 * reference's CPU dot depends on the core count, VectorOperations.cpp:187-219).
 * Loops that the reference runs as one SYCL parallel_for work-item per element
 * or row are OpenMP-parallel here; loops it runs sequentially stay sequential.
 */
#include "hs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BLK(A, id, bsz) ((A) + (size_t)(id) * (size_t)(bsz) * (size_t)(bsz))

int64_t or_block_id(int64_t i, int64_t j, int64_t nb) {
    /* SymmetricMatrix.hpp:9-35; formula as in MatrixGenerator.cpp:108-117 */
    return i + nb * (nb - 1) / 2 - (nb - j - 1) * (nb - j) / 2;
}

/* ---------------------------------------------------------------- POTRF */
void or_potrf_block(double* A, int64_t N, int bsz, int blockID, int blockRow) {
    /* MatrixOperations.cpp:7-62: one work-group of bsz work-items, local_i = row.
     * Per column k: every row reads sqrt(a_kk) before the first barrier; rows
     * below k (global row < N) divide their a_ik; after the barrier a_kk becomes
     * the root; rows < N then update their lower part right of k and zero their
     * upper part. */
    double* B = BLK(A, blockID, bsz);
    const int64_t row0 = (int64_t)blockRow * bsz;
    for (int k = 0; k < bsz; ++k) {
        const double s = sqrt(B[(size_t)k * bsz + k]);
        for (int i = k + 1; i < bsz; ++i)
            if (row0 + i < N) B[(size_t)i * bsz + k] = B[(size_t)i * bsz + k] / s;
        B[(size_t)k * bsz + k] = s;
#pragma omp parallel for schedule(static) if (bsz >= 128)
        for (int i = 0; i < bsz; ++i) {
            if (row0 + i >= N) continue;
            for (int j = k + 1; j < bsz; ++j) {
                if (i >= j) {
                    const double aik = B[(size_t)i * bsz + k];
                    const double ajk = B[(size_t)j * bsz + k];
                    B[(size_t)i * bsz + j] = B[(size_t)i * bsz + j] - aik * ajk;
                } else {
                    B[(size_t)i * bsz + j] = 0;
                }
            }
        }
    }
}

/* ---------------------------------------------------------------- TRSM */
void or_trsm_panel(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount) {
    /* MatrixMatrixOperations.cpp:109-144: one work-item per (block, row of B). */
    const double* L = BLK(A, blockID, bsz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int g = 0; g < blockCount; ++g) {
        for (int j = 0; j < bsz; ++j) {
            double* B = BLK(A, (int64_t)blockID + (blockStart - blockRow) + g, bsz);
            double* row = B + (size_t)j * bsz;
            for (int k = 0; k < bsz; ++k) {
                const double bk = row[k] / L[(size_t)k * bsz + k];
                row[k] = bk;
                for (int i = k + 1; i < bsz; ++i) row[i] = row[i] - L[(size_t)i * bsz + k] * bk;
            }
        }
    }
}

/* ---------------------------------------------------------------- SYRK */
void or_syrk_diag(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount, int nb) {
    /* MatrixMatrixOperations.cpp:307-361: lower triangle of each diagonal block,
     * value = a_ij; value -= c_ik c_jk for k ascending. */
    const int ref = (nb * (nb - 1)) / 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int g = 0; g < blockCount; ++g) {
        for (int i = 0; i < bsz; ++i) {
            const int colOff = (blockStart - blockRow) + g;
            const int diagXY = blockRow + colOff;
            const int inv = nb - (diagXY + 1);
            const int64_t idDiag = diagXY + ref - (inv * (inv + 1)) / 2;
            double* D = BLK(A, idDiag, bsz);
            const double* C = BLK(A, (int64_t)blockID + colOff, bsz);
            for (int j = 0; j <= i; ++j) {
                double v = D[(size_t)i * bsz + j];
                for (int k = 0; k < bsz; ++k) v = v - C[(size_t)i * bsz + k] * C[(size_t)j * bsz + k];
                D[(size_t)i * bsz + j] = v;
            }
        }
    }
}

/* ---------------------------------------------------------------- GEMM */
void or_gemm_trailing(double* A, int bsz, int blockID, int blockRow, int blockStart, int blockCount, int nb) {
    /* MatrixMatrixOperations.cpp:845-906 (cpu_opt=2, the reference CPU default):
     * for every block (r,c) with blockRow < c < r, r in [blockStart,
     * blockStart+blockCount): A_rc[j][i] -= sum_k L_rk[j][k] * L_ck[i][k], the
     * sum accumulated first from zero and subtracted once. */
    (void)nb;
    for (int r = blockStart; r < blockStart + blockCount; ++r) {
        const double* Brk = BLK(A, (int64_t)blockID + (r - blockRow), bsz);
#pragma omp parallel for collapse(2) schedule(static)
        for (int c = blockRow + 1; c < r; ++c) {
            for (int i = 0; i < bsz; ++i) {
                double* Arc = BLK(A, or_block_id(r, c, nb), bsz);
                const double* Cck = BLK(A, (int64_t)blockID + (c - blockRow), bsz);
                for (int j = 0; j < bsz; ++j) {
                    double v = 0;
                    for (int k = 0; k < bsz; ++k) v += Brk[(size_t)j * bsz + k] * Cck[(size_t)i * bsz + k];
                    Arc[(size_t)j * bsz + i] -= v;
                }
            }
        }
    }
}

/* ---------------------------------------------------------------- SYMV */
void or_symv_block(const double* A, const double* b, double* result, int bsz, int bi0, int bj0, int nbi, int nbj,
                   int nb, int reset) {
    /* MatrixVectorOperations.cpp:8-93: one work-item per row; a single running
     * sum over the stored blocks j <= i (row-wise) then the transposed blocks
     * j > i (column-wise). */
    const int64_t rows = (int64_t)nbi * bsz;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < rows; ++t) {
        const int64_t i = t + (int64_t)bi0 * bsz;
        const int iIn = (int)(i % bsz);
        const int bi = (int)(i / bsz);
        double v = 0;
        if (!reset) v += result[i];
        int bj = bj0;
        const int lastJ = bj0 + nbj - 1;
        for (; bj <= (bi < lastJ ? bi : lastJ); ++bj) {
            const double* row = BLK(A, or_block_id(bi, bj, nb), bsz) + (size_t)iIn * bsz;
            for (int j = 0; j < bsz; ++j) v += row[j] * b[(size_t)bj * bsz + j];
        }
        for (; bj < bj0 + nbj; ++bj) {
            const double* blk = BLK(A, or_block_id(bj, bi, nb), bsz);
            for (int j = 0; j < bsz; ++j) v += blk[(size_t)j * bsz + iIn] * b[(size_t)bj * bsz + j];
        }
        result[i] = v;
    }
}

/* ---------------------------------------------------------------- TRSV */
void or_trsv_block(const double* A, double* b, int64_t N, int bsz, int blockRow, int blockID, int transposed) {
    /* MatrixVectorOperations.cpp:282-335: column-oriented substitution; entries
     * with global index >= N are neither stored nor used for updates. */
    const double* L = BLK(A, blockID, bsz);
    double* v = b + (size_t)blockRow * bsz;
    const int64_t base = (int64_t)blockRow * bsz;
    for (int s = 0; s < bsz; ++s) {
        const int k = transposed ? bsz - (s + 1) : s;
        const double bk = v[k] / L[(size_t)k * bsz + k];
        if (base + k >= N) continue;
        v[k] = bk;
        if (!transposed) {
            for (int i = k + 1; i < bsz; ++i) v[i] = v[i] - L[(size_t)i * bsz + k] * bk;
        } else {
            for (int i = 0; i < k; ++i) v[i] = v[i] - L[(size_t)k * bsz + i] * bk;
        }
    }
}

/* ---------------------------------------------------------------- column update */
void or_column_update(const double* A, double* b, int bsz, int blockStart, int blockCount, int blockRow,
                      int blockID, int nb, int transposed) {
    /* MatrixVectorOperations.cpp:337-377: sum = sum_k a_ik b0_k (a_ki if
     * transposed), then b_i -= sum. */
    const double* b0 = b + (size_t)blockRow * bsz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int g = 0; g < blockCount; ++g) {
        for (int i = 0; i < bsz; ++i) {
            const int64_t id = !transposed ? (int64_t)blockID + (blockStart - blockRow + g)
                                           : or_block_id(blockRow, blockStart + g, nb);
            const double* M = BLK(A, id, bsz);
            double sum = 0.0;
            if (!transposed)
                for (int k = 0; k < bsz; ++k) sum += M[(size_t)i * bsz + k] * b0[k];
            else
                for (int k = 0; k < bsz; ++k) sum += M[(size_t)k * bsz + i] * b0[k];
            b[(size_t)(blockStart + g) * bsz + i] -= sum;
        }
    }
}

/* ---------------------------------------------------------------- vector ops */
/* VectorOperations.cpp:6-82 */
void or_scale_block(const double* x, double alpha, double* result, int bsz, int bi0, int nbi) {
    for (int64_t i = (int64_t)bi0 * bsz; i < (int64_t)(bi0 + nbi) * bsz; ++i) result[i] = x[i] * alpha;
}
void or_add_block(const double* x, const double* y, double* result, int bsz, int bi0, int nbi) {
    for (int64_t i = (int64_t)bi0 * bsz; i < (int64_t)(bi0 + nbi) * bsz; ++i) result[i] = x[i] + y[i];
}
void or_sub_block(const double* x, const double* y, double* result, int bsz, int bi0, int nbi) {
    for (int64_t i = (int64_t)bi0 * bsz; i < (int64_t)(bi0 + nbi) * bsz; ++i) result[i] = x[i] - y[i];
}
void or_axpy_block(const double* x, double alpha, const double* y, double* result, int bsz, int bi0, int nbi) {
    for (int64_t i = (int64_t)bi0 * bsz; i < (int64_t)(bi0 + nbi) * bsz; ++i) result[i] = x[i] + y[i] * alpha;
}

double or_dot_block(const double* x, const double* y, int bsz, int bi0, int nbi, int chunks) {
    /* VectorOperations.cpp:187-238: ceil(len/chunks) elements per chunk, each
     * chunk summed from zero, then the chunk sums added in order. */
    const int64_t len = (int64_t)nbi * bsz;
    const int64_t first = (int64_t)bi0 * bsz;
    if (chunks < 1) chunks = 1;
    const int64_t per = (len + chunks - 1) / chunks;
    double total = 0.0;
    for (int c = 0; c < chunks; ++c) {
        const int64_t s = (int64_t)c * per + first;
        const int64_t e = (s + per < first + len) ? s + per : first + len;
        double v = 0.0;
        for (int64_t i = s; i < e; ++i) v += x[i] * y[i];
        total += v;
    }
    return total;
}

/* ---------------------------------------------------------------- drivers */
void or_cholesky(double* A, int64_t N, int bsz) {
    /* Cholesky.cpp:413-493 with init_gpu_perc = 0: per block column k,
     * POTRF (:164), TRSM on rows k+1.. (:190), SYRK on diagonal blocks k+1..
     * (:213), GEMM on rows k+2.. (:233, cpu_opt = 2). */
    const int nb = (int)((N + bsz - 1) / bsz);
    const int total = nb * (nb + 1) / 2;
    for (int k = 0; k < nb; ++k) {
        const int right = nb - k;
        const int blockID = total - right * (right + 1) / 2;
        or_potrf_block(A, N, bsz, blockID, k);
        const int cnt = nb - (k + 1);
        if (cnt > 0) {
            or_trsm_panel(A, bsz, blockID, k, k + 1, cnt);
            or_syrk_diag(A, bsz, blockID, k, k + 1, cnt, nb);
        }
        if (cnt > 1) or_gemm_trailing(A, bsz, blockID, k, k + 2, cnt - 1, nb);
    }
}

void or_triangular_solve(const double* L, double* b, int64_t N, int bsz) {
    /* TriangularSystemSolver.cpp:15-105: forward sweep (:31-55) then backward
     * sweep with transposed blocks (:58-82), in place on b. */
    const int nb = (int)((N + bsz - 1) / bsz);
    const int total = nb * (nb + 1) / 2;
    for (int j = 0; j < nb; ++j) {
        const int right = nb - j;
        const int blockID = total - right * (right + 1) / 2;
        or_trsv_block(L, b, N, bsz, j, blockID, 0);
        if (j < nb - 1) or_column_update(L, b, bsz, j + 1, nb - (j + 1), j, blockID, nb, 0);
    }
    for (int j = nb - 1; j >= 0; --j) {
        const int right = nb - j;
        const int blockID = total - right * (right + 1) / 2;
        or_trsv_block(L, b, N, bsz, j, blockID, 1);
        if (j > 0) or_column_update(L, b, bsz, 0, j, j, blockID, nb, 1);
    }
}

int64_t or_cg(const double* A, const double* b, double* x, int64_t N, int bsz, double eps, int64_t imax,
              int chunks, double* delta_new_out, double* delta_zero_out) {
    /* CG.cpp:38-163 (loop), :277-340 (initCG), :342-528 (steps), CPU-only split.
     * x starts at zero (the reference's host x is value-initialised). */
    const int nb = (int)((N + bsz - 1) / bsz);
    const size_t n = (size_t)nb * bsz;
    double* r = (double*)calloc(n, sizeof(double));
    double* d = (double*)calloc(n, sizeof(double));
    double* q = (double*)calloc(n, sizeof(double));
    memset(x, 0, n * sizeof(double));

    or_symv_block(A, x, r, bsz, 0, 0, nb, nb, nb, 1);      /* r = A x        :279-286 */
    or_sub_block(b, r, r, bsz, 0, nb);                     /* r = b - r      :288-293 */
    memcpy(d, r, n * sizeof(double));                      /* d = r          :296-306 */
    double delta_new = or_dot_block(r, r, bsz, 0, nb, chunks);
    const double delta_zero = delta_new;
    const double eps2 = eps * eps;

    int64_t it = 0;
    while (it < imax && delta_new > eps2 * delta_zero) {
        or_symv_block(A, d, q, bsz, 0, 0, nb, nb, nb, 1);  /* q = A d        :356-379 */
        const double dq = or_dot_block(d, q, bsz, 0, nb, chunks);
        const double alpha = delta_new / dq;               /* :400-431 */
        or_axpy_block(x, alpha, d, x, bsz, 0, nb);         /* x = x + a d    :433-442 */
        if (it % 50 == 0) {                                /* true residual  :95-101, :444-470 */
            or_symv_block(A, x, r, bsz, 0, 0, nb, nb, nb, 1);
            or_sub_block(b, r, r, bsz, 0, nb);
        } else {
            or_axpy_block(r, -1.0 * alpha, q, r, bsz, 0, nb); /* :473-484 */
        }
        const double delta_old = delta_new;
        delta_new = or_dot_block(r, r, bsz, 0, nb, chunks);
        const double beta = delta_new / delta_old;
        or_axpy_block(r, beta, d, d, bsz, 0, nb);          /* d = r + b d    :519-528 */
        ++it;
    }
    if (delta_new_out) *delta_new_out = delta_new;
    if (delta_zero_out) *delta_zero_out = delta_zero;
    free(r);
    free(d);
    free(q);
    return it;
}

/* ---------------------------------------------------------------- assembly */
void or_rbf_assemble(double* A, const double* X, int64_t N, int d, int bsz, const double* ell, int n_ell,
                     double sf2, double sn2) {
    /* MatrixGenerator.cpp:134-155: per stored block, per in-range entry:
     * distance = sum_k (x_ik - x_jk)^2 (k ascending), K = sf2 * exp(-0.5/l^2 *
     * distance), + sn2 on the global diagonal.  The ARD form scales each
     * difference by 1/l_k first and uses exp(-0.5 * distance).  Padding entries
     * are written as zero (the reference leaves them at their zero fill). */
    const int nb = (int)((N + bsz - 1) / bsz);
    const int ref = nb * (nb - 1) / 2;
    double inv_ell[64];
    for (int k = 0; k < d && k < 64; ++k) inv_ell[k] = (n_ell == d && n_ell > 1) ? 1.0 / ell[k] : 1.0;
    const double iso_scale = -0.5 / (ell[0] * ell[0]);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int ib = 0; ib < nb; ++ib) {
        for (int jb = 0; jb < nb; ++jb) {
            if (jb > ib) continue;
            const int inv = nb - (jb + 1);
            const int64_t id = ib + ref - (inv * (inv + 1)) / 2;
            double* B = BLK(A, id, bsz);
            for (int il = 0; il < bsz; ++il) {
                for (int jl = 0; jl < bsz; ++jl) {
                    const int64_t ig = (int64_t)bsz * ib + il;
                    const int64_t jg = (int64_t)bsz * jb + jl;
                    double val = 0.0;
                    if (ig < N && jg < N) {
                        double dist = 0.0;
                        if (n_ell == d && n_ell > 1) {
                            for (int k = 0; k < d; ++k) {
                                const double t = (X[ig * d + k] - X[jg * d + k]) * inv_ell[k];
                                dist += t * t;
                            }
                            val = sf2 * exp(-0.5 * dist);
                        } else {
                            for (int k = 0; k < d; ++k) {
                                const double t = X[ig * d + k] - X[jg * d + k];
                                dist += t * t;
                            }
                            val = sf2 * exp(iso_scale * dist);
                        }
                        if (ig == jg) val += sn2;
                    }
                    B[(size_t)il * bsz + jl] = val;
                }
            }
        }
    }
}

void or_window_inputs(const double* series, int64_t N, double* X) {
    /* MatrixGenerator.cpp:76-99 and :143-147: trainingInput has 7 leading zeros
     * and element (i,k) of the window is trainingInput[i + k]. */
    for (int64_t i = 0; i < N; ++i)
        for (int k = 0; k < 8; ++k) {
            const int64_t s = i + k - 7;
            X[i * 8 + k] = s < 0 ? 0.0 : series[s];
        }
}

void or_test_kernel_matrix(const double* X, int64_t N, const double* Xt, int64_t Nt, int d, const double* ell,
                           int n_ell, double sf2, double* K_star) {
    /* MatrixGenerator.cpp:196-211: for each (test j, train i): distance =
     * sum_k (train_i,k - test_j,k)^2 with k ascending, then
     * sf2 * exp(-0.5 / l^2 * distance) stored at K_star[j * N + i]; the ARD
     * form scales each difference by 1/l_k and uses exp(-0.5 * distance). */
    const int ard = (n_ell == d && d > 1);
    const double iso_scale = -0.5 / (ell[0] * ell[0]);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < Nt; ++j) {
        for (int64_t i = 0; i < N; ++i) {
            double dist = 0.0;
            for (int k = 0; k < d; ++k) {
                const double t = ard ? (X[i * d + k] - Xt[j * d + k]) * (1.0 / ell[k]) : X[i * d + k] - Xt[j * d + k];
                dist += t * t;
            }
            K_star[j * N + i] = sf2 * exp((ard ? -0.5 : iso_scale) * dist);
        }
    }
}

void or_matrix_vector_gp(const double* A, const double* b, double* result, int64_t n, int64_t m) {
    /* MatrixVectorOperations.cpp:384-390: result[i] = sum_k A[i*n + k] b[k],
     * one running sum per row in k order */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double sum = 0.0;
        for (int64_t k = 0; k < n; ++k) sum += A[i * n + k] * b[k];
        result[i] = sum;
    }
}
