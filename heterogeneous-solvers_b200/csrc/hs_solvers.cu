// hs_solvers.cu — solver-level entry points: RBF assembly, blocked Cholesky
// factor, forward/back substitution, CG and the end-to-end host-buffer solve.
//
// Reference drivers replaced (paths relative to the reference root):
//   src/solver/cholesky/Cholesky.cpp:413-493               solve_heterogeneous
//   src/solver/cholesky/TriangularSystemSolver.cpp:15-105  solve
//   src/solver/cg/CG.cpp:38-163, 277-528                   solveHeterogeneous
//   src/utility/MatrixGenerator.cpp:73-162                 generateSPDMatrix
//   src/gaussianProcess/GaussianProcess.cpp:20-40          the GP solve
// One GPU owns every block row; the CPU/GPU split, its block copies and the
// load balancers have no counterpart here.
#include <chrono>
#include <string>

#include "hs_internal.cuh"
#include "hs_mixed.cuh"

namespace hs {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double cta_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    return s;
}

// x = x + alpha d;  r = r + q * (-alpha);  partial r.r   (CG.cpp:433-442, :473-484, :486-517)
__global__ void __launch_bounds__(kThreads) cg_update_xr(double* __restrict__ x, const double* __restrict__ d,
                                                         double* __restrict__ r, const double* __restrict__ q,
                                                         const double* __restrict__ alpha_p, int64_t n,
                                                         double* __restrict__ part) {
    __shared__ double sh[32];
    const double alpha = *alpha_p;
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = x[i] + d[i] * alpha;
        const double rv = r[i] + q[i] * (-1.0 * alpha);
        r[i] = rv;
        acc += rv * rv;
    }
    const double s = cta_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// r = b - r;  partial r.r   (CG.cpp:288-293 / :462-470 followed by :486-517)
__global__ void __launch_bounds__(kThreads) cg_residual(const double* __restrict__ b, double* __restrict__ r,
                                                        int64_t n, double* __restrict__ part) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double rv = b[i] - r[i];
        r[i] = rv;
        acc += rv * rv;
    }
    const double s = cta_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void sum_partials(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
    const double s = cta_sum(v, sh);
    if (threadIdx.x == 0) *out = s;
}

__global__ void set_i64(long long* p, long long v) { *p = v; }

int grid_for(int64_t n, int num_sms) {
    int64_t g = (n + kThreads - 1) / kThreads;
    const int64_t cap = 4LL * num_sms;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

hs_status factor_driver(hs_ctx ctx, double* A) {
    // Cholesky.cpp:446-471 with the GPU owning every block row: per block
    // column k, POTRF(k), TRSM on rows k+1.., then the SYRK on diagonal blocks
    // k+1.. and the GEMM on rows k+2...
    const int nb = ctx->nb, bsz = ctx->bsz;
    const int64_t T = total_blocks(nb);
    cudaStream_t s = ctx->stream;
    auto diag_id = [&](int k) { return (int)(T - (int64_t)(nb - k) * (nb - k + 1) / 2); };
    if ((bsz != 128 && bsz != 256) || !ctx->side_hi) {
        for (int k = 0; k < nb; ++k) {
            const int blockID = diag_id(k);
            hs_status st = launch_potrf(ctx, A, blockID, k, s);
            if (st != HS_OK) return st;
            const int cnt = nb - (k + 1);
            if (cnt > 0) {
                st = launch_trsm(ctx, A, blockID, k, k + 1, cnt, s);
                if (st != HS_OK) return st;
                st = launch_update(ctx, A, blockID, k, k + 1, cnt, k + 2, cnt - 1, s);
                if (st != HS_OK) return st;
            }
        }
        return HS_OK;
    }
    // Tensor-core form with lookahead.  The panel TRSM is a product with
    // X = L_kk^-1.  Per column k the trailing update runs in two launches: column
    // k+1 first; then, while the rest of the update runs, POTRF(k+1), X and the
    // TRSM of column k+1 run on the high-priority side stream.  Every block sees
    // the same operations in the same order as without lookahead.
    const size_t bb = (size_t)bsz * bsz;
    hs_status st = ensure_scratch(ctx, kSmallScratch + 2 * bb * sizeof(double));
    if (st != HS_OK) return st;
    double* Y = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kSmallScratch);
    double* X = Y + bb;
    auto diag = [&](int k, cudaStream_t q) -> hs_status {
        const int blockID = diag_id(k);
        hs_status s2 = launch_potrf(ctx, A, blockID, k, q);
        if (s2 != HS_OK) return s2;
        const int cnt = nb - (k + 1);
        if (cnt <= 0) return HS_OK;
        if ((s2 = launch_diag_inverse(ctx, A + (size_t)blockID * bb, Y, X, q)) != HS_OK) return s2;
        return launch_trsm_dmma(ctx, A, (int64_t)blockID + 1, cnt, X, q);
    };
    if ((st = diag(0, s)) != HS_OK) return st;
    for (int k = 0; k + 1 < nb; ++k) {
        const int blockID = diag_id(k);
        if ((st = launch_update_cols(ctx, A, blockID, k, k + 1, k + 2, s)) != HS_OK) return st;
        if (k + 2 < nb) {
            HS_CUDA(cudaEventRecord(ctx->ev_a, s));
            HS_CUDA(cudaStreamWaitEvent(ctx->side_hi, ctx->ev_a, 0));
            if ((st = diag(k + 1, ctx->side_hi)) != HS_OK) return st;
            HS_CUDA(cudaEventRecord(ctx->ev_b, ctx->side_hi));
            if ((st = launch_update_cols(ctx, A, blockID, k, k + 2, nb, s)) != HS_OK) return st;
            HS_CUDA(cudaStreamWaitEvent(s, ctx->ev_b, 0));
        } else if ((st = diag(k + 1, s)) != HS_OK) {
            return st;
        }
    }
    return HS_OK;
}

hs_status solve_driver(hs_ctx ctx, const double* L, double* b) {
    // TriangularSystemSolver.cpp:31-82
    const int nb = ctx->nb;
    const int64_t T = total_blocks(nb);
    cudaStream_t s = ctx->stream;
    if ((ctx->bsz == 128 || ctx->bsz == 256) && nb > 1) {
        // both sweeps as single cooperative launches over the FP64 factor (each row
        // reduced by one CTA in column order), with the diagonal solves as products with
        // Y_k = L_kk^-T formed for all blocks in one batched launch first; the reference's
        // 2 nb dependent launches a sweep are latency-bound
        const size_t bb = (size_t)ctx->bsz * ctx->bsz;
        const int64_t n = (int64_t)nb * ctx->bsz;
        const size_t ybytes = ((size_t)nb * bb + bb + (size_t)n) * sizeof(double);
        hs_status st = ensure_solvews(ctx, ybytes + 256 + (((size_t)nb * sizeof(unsigned) + 255) & ~size_t(255)));
        if (st != HS_OK) return st;
        double* Y = static_cast<double*>(ctx->solvews);
        double* pad = Y + (size_t)nb * bb;
        double* tmp = pad + bb;
        int* err = reinterpret_cast<int*>(static_cast<char*>(ctx->solvews) + ybytes);
        unsigned* flags = reinterpret_cast<unsigned*>(static_cast<char*>(ctx->solvews) + ybytes + 256);
        if ((st = launch_diag_inverses(ctx, L, Y, pad, s)) != HS_OK) return st;
        HS_CUDA(cudaMemsetAsync(flags, 0, (size_t)nb * sizeof(unsigned), s));
        HS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        if ((st = launch_sweep_whole_f64(ctx, L, Y, b, tmp, 1, 1u, flags, err, s)) != HS_OK) return st;
        if ((st = launch_sweep_whole_f64(ctx, L, Y, tmp, b, 0, 2u, flags, err, s)) != HS_OK) return st;
        int h_err = 0;
        HS_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        if (h_err != 0) {
            set_error("hs_cholesky_solve: a bounded wait of the triangular sweep ran out");
            return HS_ERR_TIMEOUT;
        }
        return HS_OK;
    }
    for (int j = 0; j < nb; ++j) {
        const int right = nb - j;
        const int blockID = (int)(T - (int64_t)right * (right + 1) / 2);
        hs_status st = launch_trsv(ctx, L, b, j, blockID, 0, s);
        if (st != HS_OK) return st;
        if (j < nb - 1) {
            st = launch_column_update(ctx, L, b, j + 1, nb - (j + 1), j, blockID, 0, s);
            if (st != HS_OK) return st;
        }
    }
    for (int j = nb - 1; j >= 0; --j) {
        const int right = nb - j;
        const int blockID = (int)(T - (int64_t)right * (right + 1) / 2);
        hs_status st = launch_trsv(ctx, L, b, j, blockID, 1, s);
        if (st != HS_OK) return st;
        if (j > 0) {
            st = launch_column_update(ctx, L, b, 0, j, j, blockID, 1, s);
            if (st != HS_OK) return st;
        }
    }
    return HS_OK;
}

hs_status cg_driver(hs_ctx ctx, const double* A, const double* b, double* x, double eps, int64_t imax,
                    int64_t* iters_out, double* dnew_out, double* d0_out) {
    const int nb = ctx->nb;
    const int64_t n = (int64_t)nb * ctx->bsz;
    cudaStream_t s = ctx->stream;
    const bool ref = ctx->ref_chunks > 0;
    hs_status st = ensure_work(ctx, (size_t)3 * n * sizeof(double));
    if (st != HS_OK) return st;
    // size the scratch for the matvec partials now: pointers into it stay valid below
    st = ensure_scratch(ctx, kSmallScratch + (size_t)nb * nb * ctx->bsz * sizeof(double));
    if (st != HS_OK) return st;
    double* r = static_cast<double*>(ctx->work);
    double* d = r + n;
    double* q = d + n;
    double* part = static_cast<double*>(ctx->scratch);
    double* scal = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kScalarOffset);
    double* d_dq = scal + 0;     // d.q
    double* d_delta = scal + 1;  // r.r
    double* d_alpha = scal + 2;
    volatile double* h = ctx->h_pinned;
    const int g = grid_for(n, ctx->num_sms);

    auto matvec = [&](const double* v, double* out, double* dot_with, double* dot_out) -> hs_status {
        if (!ref) return launch_symv(ctx, A, v, out, 0, 0, nb, nb, 1, dot_with, dot_out, s);
        hs_status st2 = launch_symv_refseq(ctx, A, v, out, 0, 0, nb, nb, 1, s);
        if (st2 != HS_OK || !dot_with) return st2;
        return launch_dot_refseq(ctx, dot_with, out, dot_out, 0, n, ctx->ref_chunks, s);
    };
    // r = b - r, delta = r.r
    auto residual = [&]() -> hs_status {
        if (!ref) {
            ctx->launches += 2;
            cg_residual<<<g, kThreads, 0, s>>>(b, r, n, part);
            sum_partials<<<1, kThreads, 0, s>>>(part, g, d_delta);
            HS_CHECK_LAUNCH("cg residual");
            return HS_OK;
        }
        hs_status st2 = launch_vec(ctx, 2, b, r, 0.0, r, 0, n, s);
        if (st2 != HS_OK) return st2;
        return launch_dot_refseq(ctx, r, r, d_delta, 0, n, ctx->ref_chunks, s);
    };
    auto read_scalar = [&](double* dev, int slot) -> hs_status {
        HS_CUDA(cudaMemcpyAsync((void*)(h + slot), dev, sizeof(double), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        return HS_OK;
    };

    HS_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));  // CG.cpp:217 leaves x_gpu uninitialised; x0 = 0
    // initCG (CG.cpp:277-340): r = A x; r = b - r; d = r; delta_0 = delta_new = r.r
    if ((st = matvec(x, r, nullptr, nullptr)) != HS_OK) return st;
    if ((st = residual()) != HS_OK) return st;
    HS_CUDA(cudaMemcpyAsync(d, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if ((st = read_scalar(d_delta, 1)) != HS_OK) return st;
    double delta_new = h[1];
    const double delta_zero = delta_new;
    const double eps2 = eps * eps;
    int64_t it = 0;
    while (it < imax && delta_new > eps2 * delta_zero) {
        // q = A d fused with d.q (CG.cpp:342-431)
        if ((st = matvec(d, q, d, d_dq)) != HS_OK) return st;
        if ((st = read_scalar(d_dq, 0)) != HS_OK) return st;
        const double alpha = delta_new / h[0];
        if (it % 50 == 0 || ref) {
            // x = x + alpha d (CG.cpp:433-442)
            if ((st = launch_vec(ctx, 3, x, d, alpha, x, 0, n, s)) != HS_OK) return st;
            if (it % 50 == 0) {
                // true residual r = b - A x (CG.cpp:95-101, :444-470)
                if ((st = matvec(x, r, nullptr, nullptr)) != HS_OK) return st;
                if ((st = residual()) != HS_OK) return st;
            } else {
                // r = r - alpha q (CG.cpp:473-484), delta = r.r
                if ((st = launch_vec(ctx, 3, r, q, -1.0 * alpha, r, 0, n, s)) != HS_OK) return st;
                if ((st = launch_dot_refseq(ctx, r, r, d_delta, 0, n, ctx->ref_chunks, s)) != HS_OK) return st;
            }
        } else {
            h[2] = alpha;
            HS_CUDA(cudaMemcpyAsync(d_alpha, (const void*)(h + 2), sizeof(double), cudaMemcpyHostToDevice, s));
            ctx->launches += 2;
            cg_update_xr<<<g, kThreads, 0, s>>>(x, d, r, q, d_alpha, n, part);
            sum_partials<<<1, kThreads, 0, s>>>(part, g, d_delta);
            HS_CHECK_LAUNCH("cg step");
        }
        if ((st = read_scalar(d_delta, 1)) != HS_OK) return st;
        const double delta_old = delta_new;
        delta_new = h[1];
        const double beta = delta_new / delta_old;
        // d = r + beta d (CG.cpp:519-528)
        if ((st = launch_vec(ctx, 3, r, d, beta, d, 0, n, s)) != HS_OK) return st;
        ++it;
    }
    HS_CUDA(cudaStreamSynchronize(s));
    if (iters_out) *iters_out = it;
    if (dnew_out) *dnew_out = delta_new;
    if (d0_out) *d0_out = delta_zero;
    if (it >= imax && delta_new > eps2 * delta_zero) {
        set_error("hs_cg_solve: iMax reached before the tolerance (delta_new = " + std::to_string(delta_new) +
                  ", target " + std::to_string(eps2 * delta_zero) + ")");
        return HS_ERR_NO_CONVERGENCE;
    }
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_rbf_assemble(hs_ctx ctx, double* A, const double* X, int d, const double* ell, int n_ell, double sf2,
                          double sn2) {
    hs_status st = require_ctx(ctx, "hs_rbf_assemble");
    if (st != HS_OK) return st;
    if (!A || !X || !ell) {
        set_error("hs_rbf_assemble: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    return launch_rbf_assemble(ctx, A, X, d, ell, n_ell, sf2, sn2, ctx->stream);
}

hs_status hs_cholesky_factor(hs_ctx ctx, double* A, int64_t* info) {
    hs_status st = require_ctx(ctx, "hs_cholesky_factor");
    if (st != HS_OK) return st;
    if (!A) {
        set_error("hs_cholesky_factor: null matrix");
        return HS_ERR_INVALID_ARG;
    }
    ctx->launches += 1;
    set_i64<<<1, 1, 0, ctx->stream>>>(ctx->d_info, INT64_MAX);
    st = factor_driver(ctx, A);
    if (st != HS_OK) return st;
    int64_t inf = -1;
    st = hs_ctx_take_info(ctx, &inf);
    if (st != HS_OK) return st;
    if (info) *info = inf;
    if (inf >= 0) {
        set_error("hs_cholesky_factor: matrix is not positive definite (pivot of row " + std::to_string(inf) +
                  " is not positive)");
        return HS_ERR_NOT_SPD;
    }
    return HS_OK;
}

hs_status hs_cholesky_solve(hs_ctx ctx, const double* L, double* b) {
    hs_status st = require_ctx(ctx, "hs_cholesky_solve");
    if (st != HS_OK) return st;
    if (!L || !b) {
        set_error("hs_cholesky_solve: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    return solve_driver(ctx, L, b);
}

hs_status hs_cg_solve(hs_ctx ctx, const double* A, const double* b, double* x, double epsilon, int64_t iMax,
                      int64_t* iterations, double* delta_new, double* delta_zero) {
    hs_status st = require_ctx(ctx, "hs_cg_solve");
    if (st != HS_OK) return st;
    if (!A || !b || !x) {
        set_error("hs_cg_solve: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (!(epsilon >= 0.0) || iMax < 0) {
        set_error("hs_cg_solve: epsilon must be >= 0 and iMax >= 0");
        return HS_ERR_INVALID_ARG;
    }
    return cg_driver(ctx, A, b, x, epsilon, iMax, iterations, delta_new, delta_zero);
}

hs_status hs_gp_solve_host(hs_ctx ctx, const double* X_host, const double* y_host, int d, const double* ell,
                           int n_ell, double sf2, double sn2, int algorithm, double epsilon, int64_t iMax,
                           double* x_host, hs_solve_report* report) {
    hs_status st = require_ctx(ctx, "hs_gp_solve_host");
    if (st != HS_OK) return st;
    if (!X_host || !y_host || !ell || !x_host) {
        set_error("hs_gp_solve_host: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (algorithm < 0 || algorithm > 4) {
        set_error("hs_gp_solve_host: algorithm must be 0 (cholesky), 1 (cg), 2 (mixed, 3xTF32), 3 (mixed, BF16 split) "
                  "or 4 (mixed, FP16 split)");
        return HS_ERR_INVALID_ARG;
    }
    const int64_t N = ctx->N;
    const int64_t n = (int64_t)ctx->nb * ctx->bsz;
    const size_t packed = (size_t)total_blocks(ctx->nb) * block_elems(ctx);
    cudaStream_t s = ctx->stream;
    double *Xd = nullptr, *Ad = nullptr, *bd = nullptr, *xd = nullptr;
    cudaEvent_t ev[5] = {};
    auto cleanup = [&]() {
        cudaStreamSynchronize(s);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    };
#define HS_E2E(call)                          \
    do {                                      \
        cudaError_t e_ = (call);              \
        if (e_ != cudaSuccess) {              \
            hs_status r_ = cuda_fail(e_, #call); \
            cleanup();                        \
            return r_;                        \
        }                                     \
    } while (0)
    for (auto& e : ev) HS_E2E(cudaEventCreate(&e));
    HS_E2E(cudaEventRecord(ev[0], s));
    {
        // device copies kept by the context between calls (hs_ctx_release_buffers frees them)
        const size_t xbytes = ((size_t)N * d * sizeof(double) + 255) & ~size_t(255);
        st = ensure_hostws(ctx, xbytes + (packed + 2 * (size_t)n) * sizeof(double));
        if (st != HS_OK) { cleanup(); return st; }
        Xd = static_cast<double*>(ctx->hostws);
        Ad = reinterpret_cast<double*>(static_cast<char*>(ctx->hostws) + xbytes);
        bd = Ad + packed;
        xd = bd + n;
    }
    HS_E2E(cudaMemcpyAsync(Xd, X_host, (size_t)N * d * sizeof(double), cudaMemcpyHostToDevice, s));
    HS_E2E(cudaMemsetAsync(bd, 0, n * sizeof(double), s));
    HS_E2E(cudaMemcpyAsync(bd, y_host, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s));
    st = launch_rbf_assemble(ctx, Ad, Xd, d, ell, n_ell, sf2, sn2, s);
    if (st != HS_OK) { cleanup(); return st; }
    HS_E2E(cudaEventRecord(ev[1], s));
    int64_t info = -1, iters = 0;
    if (algorithm == 0) {
        ctx->launches += 1;
        set_i64<<<1, 1, 0, s>>>(ctx->d_info, INT64_MAX);
        st = factor_driver(ctx, Ad);
        if (st != HS_OK) { cleanup(); return st; }
        HS_E2E(cudaEventRecord(ev[2], s));
        HS_E2E(cudaMemcpyAsync(xd, bd, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        st = solve_driver(ctx, Ad, xd);
        if (st != HS_OK) { cleanup(); return st; }
    } else if (algorithm == 1) {
        HS_E2E(cudaEventRecord(ev[2], s));
        st = cg_driver(ctx, Ad, bd, xd, epsilon, iMax, &iters, nullptr, nullptr);
        if (st != HS_OK && st != HS_ERR_NO_CONVERGENCE) { cleanup(); return st; }
    } else {
        // mixed precision: epsilon is the backward-error target, iMax the refinement step limit
        hs_mixed_report mr{};
        const int prec = algorithm == 4 ? HS_PRECISION_F16X3 : algorithm == 3 ? HS_PRECISION_BF16X3 : HS_PRECISION_TF32X3;
        st = mixed_solve_impl(ctx, Ad, bd, xd, prec, epsilon, (int)iMax, &mr);
        if (st != HS_OK) { cleanup(); return st; }
        iters = mr.refinement_steps + mr.pcg_iterations;
        HS_E2E(cudaEventRecord(ev[2], s));
    }
    HS_E2E(cudaEventRecord(ev[3], s));
    HS_E2E(cudaMemcpyAsync(x_host, xd, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s));
    HS_E2E(cudaEventRecord(ev[4], s));
    HS_E2E(cudaStreamSynchronize(s));
    if (algorithm == 0) {
        hs_status ist = hs_ctx_take_info(ctx, &info);
        if (ist != HS_OK) { cleanup(); return ist; }
    }
    if (report) {
        float ms = 0.f;
        report->info = info;
        report->iterations = iters;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        report->assemble_ms = ms;
        cudaEventElapsedTime(&ms, ev[1], ev[2]);
        report->factor_ms = ms;
        cudaEventElapsedTime(&ms, ev[2], ev[3]);
        report->solve_ms = ms;
        cudaEventElapsedTime(&ms, ev[0], ev[4]);
        report->total_ms = ms;
    }
    cleanup();
#undef HS_E2E
    if (algorithm == 0 && info >= 0) {
        set_error("hs_gp_solve_host: kernel matrix is not positive definite (row " + std::to_string(info) + ")");
        return HS_ERR_NOT_SPD;
    }
    return st;
}

}  // extern "C"
