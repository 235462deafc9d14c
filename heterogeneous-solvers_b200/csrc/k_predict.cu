// k_predict.cu — GP prediction: the test kernel matrix K*, the dense
// matrix-vector product of the prediction, and a fused predictive mean that
// never stores K*.
//
// Replaces MatrixGenerator::generateTestKernelMatrix
// (src/utility/MatrixGenerator.cpp:163-213: K*[j*N + i] = sf2 exp(-0.5/l^2 *
// sum_k (x_ik - x*_jk)^2), k ascending, no noise term) and
// MatrixVectorOperations::matrixVectorGP (src/kernel/MatrixVectorOperations.cpp:
// 379-395: result[i] = sum_k A[i*n + k] b[k] for i < m), the two steps of
// GaussianProcess::start's prediction (src/gaussianProcess/GaussianProcess.cpp:
// 42-54).  The inputs are row-major X (N x d) and X* (N_test x d); the
// reference's 8-sample sliding window is one instance, ARD lengthscales the
// generalisation (each difference scaled by 1/l_k, then exp(-0.5 * distance)).
#include "hs_internal.cuh"

namespace hs {
namespace {

constexpr int kMaxD = 64;
constexpr int kPredThreads = 256;

__device__ __forceinline__ double sq_dist(const double* __restrict__ a, const double* __restrict__ bT, int stride,
                                          int d, int ard, const double* __restrict__ w) {
    double dist = 0.0;
    for (int k = 0; k < d; ++k) {
        const double t = ard ? (a[k] - bT[(size_t)k * stride]) * w[k] : a[k] - bT[(size_t)k * stride];
        dist += t * t;
    }
    return dist;
}

// K*: CTA = 16 test rows x 256 training columns; X* rows and the X columns
// (transposed) staged in shared memory; each warp writes 256 contiguous bytes
// of one K* row per instruction.
__global__ void __launch_bounds__(kPredThreads) test_kernel_matrix_kernel(
    const double* __restrict__ X, int64_t N, const double* __restrict__ Xt, int64_t Nt, int d, int ard,
    const double* __restrict__ w, double scale, double sf2, double* __restrict__ Ks) {
    extern __shared__ double sm[];
    constexpr int TJ = 16, TI = 256;
    double* xt = sm;                    // [TJ][d]
    double* xT = sm + TJ * d;           // [d][TI]
    __shared__ double ws[kMaxD];
    const int64_t j0 = (int64_t)blockIdx.y * TJ, i0 = (int64_t)blockIdx.x * TI;
    for (int e = threadIdx.x; e < TJ * d; e += blockDim.x) {
        const int r = e / d, k = e % d;
        xt[e] = (j0 + r < Nt) ? Xt[(j0 + r) * d + k] : 0.0;
    }
    for (int e = threadIdx.x; e < TI * d; e += blockDim.x) {
        const int r = e / d, k = e % d;
        xT[(size_t)k * TI + r] = (i0 + r < N) ? X[(i0 + r) * d + k] : 0.0;
    }
    if (threadIdx.x < d) ws[threadIdx.x] = ard ? w[threadIdx.x] : 1.0;
    __syncthreads();
    const int il = threadIdx.x;
    const int64_t i = i0 + il;
    if (i >= N) return;
    for (int jl = 0; jl < TJ; ++jl) {
        const int64_t j = j0 + jl;
        if (j >= Nt) break;
        const double dist = sq_dist(xt + jl * d, xT + il, TI, d, ard, ws);
        __stcs(Ks + j * N + i, sf2 * exp((ard ? -0.5 : scale) * dist));
    }
}

// result[i] = sum_k A[i*n + k] b[k]: one warp per row, lanes stride the row,
// fixed-order butterfly reduction
__global__ void __launch_bounds__(kPredThreads) matvec_rows_kernel(const double* __restrict__ A,
                                                                   const double* __restrict__ b,
                                                                   double* __restrict__ result, int64_t n, int64_t m) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < m; row += warps) {
        const double* a = A + row * n;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int64_t k = lane;
        for (; k + 96 < n; k += 128) {
            s0 = fma(__ldcs(a + k), b[k], s0);
            s1 = fma(__ldcs(a + k + 32), b[k + 32], s1);
            s2 = fma(__ldcs(a + k + 64), b[k + 64], s2);
            s3 = fma(__ldcs(a + k + 96), b[k + 96], s3);
        }
        for (; k < n; k += 32) s0 = fma(__ldcs(a + k), b[k], s0);
        double s = (s0 + s1) + (s2 + s3);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) result[row] = s;
    }
}

// fused predictive mean: mean[j] = sum_i k(x*_j, x_i) alpha_i without storing
// K*.  CTA = 32 test points; 8 threads per test point, each summing a fixed
// residue class of the training points of every 256-point chunk; the 8
// partial sums are combined in a fixed order.
__global__ void __launch_bounds__(kPredThreads) predict_mean_kernel(
    const double* __restrict__ X, int64_t N, const double* __restrict__ Xt, int64_t Nt, int d, int ard,
    const double* __restrict__ w, double scale, double sf2, const double* __restrict__ alpha,
    double* __restrict__ mean) {
    extern __shared__ double sm[];
    constexpr int TJ = 32, TI = 256, PER = kPredThreads / TJ;  // 8 threads per test point
    double* xt = sm;                 // [TJ][d]
    double* xT = sm + TJ * d;        // [d][TI]
    double* al = xT + (size_t)d * TI;  // [TI]
    __shared__ double ws[kMaxD];
    __shared__ double part[TJ][PER];
    const int64_t j0 = (int64_t)blockIdx.x * TJ;
    for (int e = threadIdx.x; e < TJ * d; e += blockDim.x) {
        const int r = e / d, k = e % d;
        xt[e] = (j0 + r < Nt) ? Xt[(j0 + r) * d + k] : 0.0;
    }
    if (threadIdx.x < d) ws[threadIdx.x] = ard ? w[threadIdx.x] : 1.0;
    const int jl = threadIdx.x / PER, sub = threadIdx.x % PER;
    double acc = 0.0;
    for (int64_t i0 = 0; i0 < N; i0 += TI) {
        __syncthreads();
        for (int e = threadIdx.x; e < TI * d; e += blockDim.x) {
            const int r = e / d, k = e % d;
            xT[(size_t)k * TI + r] = (i0 + r < N) ? X[(i0 + r) * d + k] : 0.0;
        }
        for (int r = threadIdx.x; r < TI; r += blockDim.x) al[r] = (i0 + r < N) ? alpha[i0 + r] : 0.0;
        __syncthreads();
        for (int il = sub; il < TI; il += PER) {
            if (i0 + il >= N) break;
            const double dist = sq_dist(xt + jl * d, xT + il, TI, d, ard, ws);
            acc = fma(sf2 * exp((ard ? -0.5 : scale) * dist), al[il], acc);
        }
    }
    part[jl][sub] = acc;
    __syncthreads();
    if (threadIdx.x < TJ && j0 + threadIdx.x < Nt) {
        double s = 0.0;
        for (int q = 0; q < PER; ++q) s += part[threadIdx.x][q];
        mean[j0 + threadIdx.x] = s;
    }
}

struct Scales {
    int ard = 0;
    double scale = 0.0;
    double* w = nullptr;  // device, d
};

hs_status make_scales(hs_ctx ctx, int d, const double* ell, int n_ell, Scales* out) {
    HS_REQUIRE(d >= 1 && d <= kMaxD, "d must be in [1, 64]");
    HS_REQUIRE(n_ell == 1 || n_ell == d, "n_ell must be 1 or d");
    for (int k = 0; k < n_ell; ++k) HS_REQUIRE(ell[k] > 0.0, "lengthscales must be positive");
    out->ard = (n_ell == d && d > 1) ? 1 : 0;
    out->scale = -0.5 / (ell[0] * ell[0]);
    hs_status st = ensure_scratch(ctx, kSmallScratch);
    if (st != HS_OK) return st;
    double* w = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kConstOffset);
    if (out->ard) {
        double hw[kMaxD];
        for (int k = 0; k < d; ++k) hw[k] = 1.0 / ell[k];
        HS_CUDA(cudaMemcpyAsync(w, hw, d * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        HS_CUDA(cudaStreamSynchronize(ctx->stream));  // hw is a stack buffer
    }
    out->w = w;
    return HS_OK;
}

}  // namespace
}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_gp_test_kernel_matrix(hs_ctx ctx, const double* X, const double* X_test, int64_t N_test, int d,
                                   const double* ell, int n_ell, double sf2, double* K_star) {
    hs_status st = require_ctx(ctx, "hs_gp_test_kernel_matrix");
    if (st != HS_OK) return st;
    if (!X || !X_test || !ell || !K_star || N_test < 0) {
        set_error("hs_gp_test_kernel_matrix: null pointer or negative N_test");
        return HS_ERR_INVALID_ARG;
    }
    if (N_test == 0) return HS_OK;
    Scales sc;
    if ((st = make_scales(ctx, d, ell, n_ell, &sc)) != HS_OK) return st;
    const int64_t N = ctx->N;
    dim3 grid((unsigned)((N + 255) / 256), (unsigned)((N_test + 15) / 16));
    HS_REQUIRE(grid.y <= 65535, "N_test too large (at most 1048560)");
    const size_t smem = (size_t)(16 + 256) * d * sizeof(double);
    HS_CUDA(cudaFuncSetAttribute(test_kernel_matrix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    prof_begin(ctx, ctx->stream, HS_KERNEL_ASSEMBLE);
    ctx->launches += 1;
    test_kernel_matrix_kernel<<<grid, kPredThreads, smem, ctx->stream>>>(X, N, X_test, N_test, d, sc.ard, sc.w,
                                                                        sc.scale, sf2, K_star);
    HS_CHECK_LAUNCH("test_kernel_matrix");
    prof_end(ctx, ctx->stream, HS_KERNEL_ASSEMBLE, (double)N * N_test * (3.0 * d + 20.0),
             (double)N * N_test * 8.0);
    return HS_OK;
}

hs_status hs_matrix_vector_gp(hs_ctx ctx, const double* A, const double* b, double* result, int64_t n, int64_t m) {
    hs_status st = require_ctx(ctx, "hs_matrix_vector_gp");
    if (st != HS_OK) return st;
    if (!A || !b || !result || n < 0 || m < 0) {
        set_error("hs_matrix_vector_gp: null pointer or negative size");
        return HS_ERR_INVALID_ARG;
    }
    if (m == 0) return HS_OK;
    const int64_t rows_per_cta = kPredThreads / 32;
    int64_t grid = (m + rows_per_cta - 1) / rows_per_cta;
    if (grid > 16LL * ctx->num_sms) grid = 16LL * ctx->num_sms;
    prof_begin(ctx, ctx->stream, HS_KERNEL_VECTOR);
    ctx->launches += 1;
    matvec_rows_kernel<<<(unsigned)grid, kPredThreads, 0, ctx->stream>>>(A, b, result, n, m);
    HS_CHECK_LAUNCH("matrix_vector_gp");
    prof_end(ctx, ctx->stream, HS_KERNEL_VECTOR, 2.0 * n * m, 8.0 * ((double)n * m + n + m));
    return HS_OK;
}

hs_status hs_gp_predict(hs_ctx ctx, const double* X, const double* X_test, int64_t N_test, int d, const double* ell,
                        int n_ell, double sf2, const double* alpha, double* mean) {
    hs_status st = require_ctx(ctx, "hs_gp_predict");
    if (st != HS_OK) return st;
    if (!X || !X_test || !ell || !alpha || !mean || N_test < 0) {
        set_error("hs_gp_predict: null pointer or negative N_test");
        return HS_ERR_INVALID_ARG;
    }
    if (N_test == 0) return HS_OK;
    Scales sc;
    if ((st = make_scales(ctx, d, ell, n_ell, &sc)) != HS_OK) return st;
    const size_t smem = ((size_t)(32 + 256) * d + 256) * sizeof(double);
    HS_CUDA(cudaFuncSetAttribute(predict_mean_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t grid = (N_test + 31) / 32;
    HS_REQUIRE(grid < (1LL << 31), "N_test too large");
    prof_begin(ctx, ctx->stream, HS_KERNEL_VECTOR);
    ctx->launches += 1;
    predict_mean_kernel<<<(unsigned)grid, kPredThreads, smem, ctx->stream>>>(X, ctx->N, X_test, N_test, d, sc.ard,
                                                                            sc.w, sc.scale, sf2, alpha, mean);
    HS_CHECK_LAUNCH("predict_mean");
    prof_end(ctx, ctx->stream, HS_KERNEL_VECTOR, (double)ctx->N * N_test * (3.0 * d + 22.0),
             8.0 * ((double)ctx->N * (d + 1) * (double)grid + N_test * (d + 1.0)));
    return HS_OK;
}

}  // extern "C"
