// hs_mixed.cu — mixed-precision solve: 3xTF32 tensor-core factor (k_mixed.cu),
// FP64 iterative refinement to a backward-error target, and conjugate gradients
// preconditioned by the low-precision factor when refinement stalls; plus the
// log-determinant of a factor.
//
// No reference counterpart (new form).  Residuals r = b - K x use the FP64
// packed K and the FP64 matvec; the triangular solves apply the FP32 factor
// with FP64 arithmetic (FP32 off-diagonal blocks, FP64 inverses of the
// diagonal blocks), one fused launch per block column and direction.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>

#include "hs_internal.cuh"
#include "hs_mixed.cuh"

namespace hs {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double cta_sum2(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    return s;
}

// r = b - r (r holds K x on entry), partial sums of r.r and x.x
__global__ void residual2_kernel(const double* __restrict__ b, double* __restrict__ r, const double* __restrict__ x,
                                 int64_t n, double* __restrict__ part) {
    __shared__ double sh[32];
    double rr = 0.0, xx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = b[i] - r[i];
        r[i] = v;
        rr += v * v;
        xx += x[i] * x[i];
    }
    const double s1 = cta_sum2(rr, sh);
    __syncthreads();
    const double s2 = cta_sum2(xx, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s1;
        part[2 * blockIdx.x + 1] = s2;
    }
}

__global__ void sum_pairs_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    const double s1 = cta_sum2(a, sh);
    __syncthreads();
    const double s2 = cta_sum2(b, sh);
    if (threadIdx.x == 0) {
        out[0] = s1;
        out[1] = s2;
    }
}

__global__ void sum_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[32];
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += part[i];
    const double s = cta_sum2(a, sh);
    if (threadIdx.x == 0) *out = s;
}

// sum of log(diag) over the valid rows of the diagonal blocks (blocks at `ids`
// or, when ids == nullptr, nb consecutive blocks)
__global__ void logdiag_kernel(const double* __restrict__ L, int bsz, int nb, int64_t N, int consecutive,
                               double* __restrict__ out) {
    __shared__ double sh[32];
    double acc = 0.0;
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const int k = (int)(i / bsz), r = (int)(i % bsz);
        const int64_t id = consecutive ? k : block_id(k, k, nb);
        acc += log(L[id * bb + (int64_t)r * bsz + r]);
    }
    const double s = cta_sum2(acc, sh);
    if (threadIdx.x == 0) *out = 2.0 * s;
}

// largest diagonal entry over the valid rows of the packed matrix
__global__ void maxdiag_kernel(const double* __restrict__ A, int bsz, int nb, int64_t N, double* __restrict__ out) {
    __shared__ double sh[32];
    double m = 0.0;
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const int k = (int)(i / bsz), r = (int)(i % bsz);
        m = fmax(m, A[block_id(k, k, nb) * bb + (int64_t)r * bsz + r]);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
        *out = m;
    }
}

// out[i] = float(in[i]), n even
__global__ void f64_to_f32_copy_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n / 2; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = reinterpret_cast<const double2*>(in)[i];
        reinterpret_cast<float2*>(out)[i] = make_float2((float)v.x, (float)v.y);
    }
}

// x += d
__global__ void add_kernel(double* __restrict__ x, const double* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += d[i];
}

int grid_n(int64_t n, int sms) {
    int64_t g = (n + kThreads - 1) / kThreads;
    if (g > 4LL * sms) g = 4LL * sms;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

// b <- (L L^T)^-1 b with the mixed factor: FP32 off-diagonal blocks, FP64
// inverse diagonal blocks; one cooperative launch a direction.  The forward sweep
// reads b and writes L^-1 b into tmp; the backward sweep reads tmp and writes the
// result into b.
hs_status mixed_apply(hs_ctx ctx, MixedWork& w, double* b, double* tmp, cudaStream_t s) {
    hs_status st = launch_mixed_sweep_whole(ctx, w.A32, w.Y32, b, tmp, 1, ++w.epoch, w.flags, w.err + 1, s);
    if (st != HS_OK) return st;
    return launch_mixed_sweep_whole(ctx, w.A32, w.Y32, tmp, b, 0, ++w.epoch, w.flags, w.err + 1, s);
}

namespace {
struct Events {
    cudaEvent_t e[3] = {};
    ~Events() {
        for (auto& v : e)
            if (v) cudaEventDestroy(v);
    }
};
}  // namespace

hs_status mixed_solve_impl(hs_ctx ctx, const double* K, const double* b, double* x, int precision, double tol,
                           int max_steps, hs_mixed_report* out, int acc_panels) {
    if (precision != HS_PRECISION_TF32X3 && precision != HS_PRECISION_BF16X3 && precision != HS_PRECISION_F16X3) {
        set_error("hs_mixed_solve: precision must be HS_PRECISION_TF32X3, HS_PRECISION_BF16X3 or HS_PRECISION_F16X3");
        return HS_ERR_UNSUPPORTED;
    }
    if (!(tol > 0.0) || max_steps < 1) {
        set_error("hs_mixed_solve: tol must be > 0 and max_steps >= 1");
        return HS_ERR_INVALID_ARG;
    }
    cudaStream_t s = ctx->stream;
    const int nb = ctx->nb, bsz = ctx->bsz;
    const int64_t n = (int64_t)nb * bsz;
    const auto t0 = std::chrono::steady_clock::now();
    hs_mixed_report& R = *out;
    R = hs_mixed_report{};
    // workspace (kept by the context): factor + 6 vectors
    const size_t fbytes = (mixed_workspace_bytes(ctx->N, bsz) + 255) & ~size_t(255);
    hs_status st = ensure_mixed(ctx, fbytes + (size_t)6 * n * sizeof(double));
    if (st != HS_OK) return st;
    double* r = reinterpret_cast<double*>(static_cast<char*>(ctx->mixed) + fbytes);
    double* d = r + n;
    double* p = d + n;
    double* q = p + n;
    double* z = q + n;
    double* tmp = z + n;  // triangular-sweep intermediate
    MixedWork w;
    st = mixed_bind(ctx, ctx->mixed, &w);
    if (st != HS_OK) return st;
    HS_CUDA(cudaMemsetAsync(w.flags, 0, (size_t)nb * sizeof(unsigned), s));
    HS_CUDA(cudaMemsetAsync(w.err + 1, 0, sizeof(int), s));
    st = ensure_scratch(ctx, kSmallScratch + (size_t)nb * nb * bsz * sizeof(double));
    if (st != HS_OK) return st;
    double* part = static_cast<double*>(ctx->scratch);
    double* scal = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kScalarOffset) + 16;
    volatile double* h = ctx->h_pinned;
    const int g = grid_n(n, ctx->num_sms);
    Events ev;
    for (auto& e : ev.e) HS_CUDA(cudaEventCreate(&e));

    // factor (a non-positive FP64 pivot of the FP32 matrix is recorded in ctx->d_info);
    // on breakdown, factor K + shift*I with a growing shift and use it as a CG preconditioner
    double shift = 0.0;
    int prec = precision;
    HS_CUDA(cudaEventRecord(ev.e[0], s));
    // the largest diagonal entry (h[9]): the FP16 split's scale, and the unit of the shifts
    bool have_maxdiag = false;
    auto read_maxdiag = [&]() -> hs_status {
        ctx->launches += 1;
        maxdiag_kernel<<<1, 1024, 0, s>>>(K, bsz, nb, ctx->N, scal + 3);
        HS_CHECK_LAUNCH("maxdiag");
        HS_CUDA(cudaMemcpyAsync((void*)(h + 9), scal + 3, sizeof(double), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        have_maxdiag = true;
        return HS_OK;
    };
    if (prec == HS_PRECISION_F16X3 && (st = read_maxdiag()) != HS_OK) return st;
    for (int attempt = 1;; ++attempt) {
        ctx->launches += 2;
        set_i64_dev(ctx->d_info, INT64_MAX, s);
        set_i64_dev(ctx->d_info + 1, LLONG_MIN, s);
        // the first attempt's conversion to FP32 also sums ||K||_F^2
        st = mixed_factor(ctx, K, w, s, shift, prec, attempt == 1 ? part : nullptr, have_maxdiag ? h[9] + shift : 0.0,
                          acc_panels > 0 ? acc_panels : ctx->mixed_acc_panels);
        if (st != HS_OK) return st;
        HS_CUDA(cudaStreamSynchronize(s));
        if (ctx->side_hi) HS_CUDA(cudaStreamSynchronize(ctx->side_hi));
        st = mixed_check_error(ctx, w);
        if (st != HS_OK) return st;
        long long piv_bits = LLONG_MIN;
        HS_CUDA(cudaMemcpyAsync(&piv_bits, ctx->d_info + 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
        int64_t info = -1;
        st = hs_ctx_take_info(ctx, &info);  // synchronises the stream
        if (st != HS_OK) return st;
        R.factor_attempts = attempt;
        R.precision_used = prec;
        R.shift = shift;
        if (info < 0) break;
        // the failing pivot (NaN when the scaled FP16 panel overflowed: no value)
        double piv = 0.0;
        std::memcpy(&piv, &piv_bits, sizeof(piv));
        const bool have_piv = piv_bits != LLONG_MIN && std::isfinite(piv) && piv < 0.0;
        // the BF16 split (16 significant bits) is redone with 3xTF32 products, which
        // hold ~2^-21; so is a FP16 split that failed without a finite pivot (an
        // overflow of the scaled panel).  A FP16 split (~2^-22) that met a negative
        // pivot is past what any FP32 factor holds: straight to the shift.
        if (prec == HS_PRECISION_BF16X3 || (prec == HS_PRECISION_F16X3 && !have_piv)) {
            prec = HS_PRECISION_TF32X3;
            continue;
        }
        if (shift > 0.0 && shift >= 0.05 * h[9]) {
            set_error("hs_mixed_solve: the low-precision factor met a non-positive pivot at row " +
                      std::to_string(info) + " even with a diagonal shift of " + std::to_string(shift));
            return HS_ERR_NOT_SPD;
        }
        if (!have_maxdiag && (st = read_maxdiag()) != HS_OK) return st;
        // a pivot -p < 0 means the rounding of the factor moved a Schur complement by
        // more than p (the exact one is positive): the next shift covers 2 p on top of
        // the shift so far, and is at least 10x that shift (or 1e-6 x the largest
        // diagonal entry), at most 0.05x.  (30 p overshot: a weaker preconditioner cost
        // more CG iterations than the attempts it saved.)
        const double floor_shift = shift > 0.0 ? 10.0 * shift : 1e-6 * h[9];
        shift = have_piv ? std::max(floor_shift, shift + 2.0 * -piv) : floor_shift;
        shift = std::min(shift, 0.05 * h[9]);
    }
    // the sweeps read the inverse diagonal blocks in FP32 (their rounding is far below
    // the factor's own error), from the 16-bit panel area the factor no longer needs
    w.Y32 = reinterpret_cast<float*>(w.P16);
    ctx->launches += 1;
    f64_to_f32_copy_kernel<<<grid_n((int64_t)nb * bsz * bsz / 2, ctx->num_sms), kThreads, 0, s>>>(
        w.Yinv, w.Y32, (int64_t)nb * bsz * bsz);
    HS_CHECK_LAUNCH("Y32");
    {
        const int fg = mixed_fro_grid(total_blocks(nb));
        ctx->launches += 1;
        sum_kernel<<<1, kThreads, 0, s>>>(part, fg, scal);
        HS_CHECK_LAUNCH("fro2");
        HS_CUDA(cudaMemcpyAsync((void*)(h + 8), scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        R.norm_k_fro = std::sqrt(h[8]);
    }
    HS_CUDA(cudaEventRecord(ev.e[1], s));
    // log|K| from the FP64 diagonal blocks
    ctx->launches += 1;
    logdiag_kernel<<<1, 1024, 0, s>>>(w.Ld, bsz, nb, ctx->N, 1, scal + 2);
    HS_CHECK_LAUNCH("logdet");

    auto residual = [&](double* rnorm, double* xnorm) -> hs_status {
        // r = b - K x, ||r||, ||x||
        hs_status s2 = launch_symv(ctx, K, x, r, 0, 0, nb, nb, 1, nullptr, nullptr, s);
        if (s2 != HS_OK) return s2;
        ctx->launches += 2;
        residual2_kernel<<<g, kThreads, 0, s>>>(b, r, x, n, part);
        sum_pairs_kernel<<<1, kThreads, 0, s>>>(part, g, scal + 4);
        HS_CHECK_LAUNCH("residual");
        HS_CUDA(cudaMemcpyAsync((void*)(h + 10), scal + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        *rnorm = std::sqrt(h[10]);
        *xnorm = std::sqrt(h[11]);
        return HS_OK;
    };
    // x0 = M^-1 b
    HS_CUDA(cudaMemcpyAsync(x, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    st = mixed_apply(ctx, w, x, tmp, s);
    if (st != HS_OK) return st;
    double rn = 0, xn = 0, prev = INFINITY;
    bool converged = false;
    int steps = 0;
    bool r_fresh = false;  // r holds b - K x for the current x
    // a shifted factor is only a preconditioner: no refinement, straight to CG
    const int ref_steps = shift > 0.0 ? 0 : max_steps;
    for (; steps < ref_steps; ++steps) {
        st = residual(&rn, &xn);
        if (st != HS_OK) return st;
        R.backward_error = rn / (R.norm_k_fro * xn);
        if (steps == 0) R.initial_backward_error = R.backward_error;
        if (R.backward_error <= tol) {
            converged = true;
            break;
        }
        // a step that shrinks the residual by less than 8x means a poor contraction:
        // conjugate gradients with the same preconditioner converges faster from here
        if (rn > 0.125 * prev) {
            r_fresh = true;
            break;
        }
        prev = rn;
        // d = M^-1 r; x += d
        HS_CUDA(cudaMemcpyAsync(d, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        st = mixed_apply(ctx, w, d, tmp, s);
        if (st != HS_OK) return st;
        ctx->launches += 1;
        add_kernel<<<g, kThreads, 0, s>>>(x, d, n);
        HS_CHECK_LAUNCH("refine add");
    }
    R.refinement_steps = steps;
    if (!converged) {
        // conjugate gradients preconditioned by the low-precision factor, from the current x
        R.fallback_pcg = 1;
        if (!r_fresh) {
            st = residual(&rn, &xn);  // r = b - K x
            if (st != HS_OK) return st;
        }
        if (steps == 0) R.initial_backward_error = rn / (R.norm_k_fro * xn);
        HS_CUDA(cudaMemcpyAsync(z, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        st = mixed_apply(ctx, w, z, tmp, s);
        if (st != HS_OK) return st;
        HS_CUDA(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        st = launch_dot(ctx, r, z, scal + 6, 0, n, s);
        if (st != HS_OK) return st;
        HS_CUDA(cudaMemcpyAsync((void*)(h + 12), scal + 6, sizeof(double), cudaMemcpyDeviceToHost, s));
        HS_CUDA(cudaStreamSynchronize(s));
        double rho = h[12];
        const int max_pcg = 50 * max_steps + 200;
        int it = 0;
        for (; it < max_pcg; ++it) {
            st = launch_symv(ctx, K, p, q, 0, 0, nb, nb, 1, p, scal + 7, s);  // q = K p, p.q
            if (st != HS_OK) return st;
            HS_CUDA(cudaMemcpyAsync((void*)(h + 13), scal + 7, sizeof(double), cudaMemcpyDeviceToHost, s));
            HS_CUDA(cudaStreamSynchronize(s));
            const double alpha = rho / h[13];
            if ((st = launch_vec(ctx, 3, x, p, alpha, x, 0, n, s)) != HS_OK) return st;
            if ((st = launch_vec(ctx, 3, r, q, -alpha, r, 0, n, s)) != HS_OK) return st;
            const bool true_res = (it + 1) % 10 == 0;
            if (true_res) {
                st = residual(&rn, &xn);  // true residual keeps r honest
                if (st != HS_OK) return st;
            } else {
                if ((st = launch_dot(ctx, r, r, scal + 8, 0, n, s)) != HS_OK) return st;
                if ((st = launch_dot(ctx, x, x, scal + 9, 0, n, s)) != HS_OK) return st;
                HS_CUDA(cudaMemcpyAsync((void*)(h + 14), scal + 8, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
                HS_CUDA(cudaStreamSynchronize(s));
                rn = std::sqrt(h[14]);
                xn = std::sqrt(h[15]);
            }
            R.backward_error = rn / (R.norm_k_fro * xn);
            if (R.backward_error <= tol) {
                // confirm with the true residual before stopping (unless it is the true one)
                if (!true_res) {
                    st = residual(&rn, &xn);
                    if (st != HS_OK) return st;
                    R.backward_error = rn / (R.norm_k_fro * xn);
                }
                if (R.backward_error <= tol) {
                    converged = true;
                    ++it;
                    break;
                }
            }
            HS_CUDA(cudaMemcpyAsync(z, r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            if ((st = mixed_apply(ctx, w, z, tmp, s)) != HS_OK) return st;
            if ((st = launch_dot(ctx, r, z, scal + 6, 0, n, s)) != HS_OK) return st;
            HS_CUDA(cudaMemcpyAsync((void*)(h + 12), scal + 6, sizeof(double), cudaMemcpyDeviceToHost, s));
            HS_CUDA(cudaStreamSynchronize(s));
            const double rho_new = h[12];
            const double beta = rho_new / rho;
            rho = rho_new;
            if ((st = launch_vec(ctx, 3, z, p, beta, p, 0, n, s)) != HS_OK) return st;
        }
        R.pcg_iterations = it;
    }
    HS_CUDA(cudaEventRecord(ev.e[2], s));
    HS_CUDA(cudaMemcpyAsync((void*)(h + 16), scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    HS_CUDA(cudaStreamSynchronize(s));
    R.logdet = h[16];
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]);
    R.factor_ms = ms;
    cudaEventElapsedTime(&ms, ev.e[1], ev.e[2]);
    R.refine_ms = ms;
    R.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if ((st = mixed_check_error(ctx, w)) != HS_OK) return st;
    if (!converged) {
        set_error("hs_mixed_solve: backward error " + std::to_string(R.backward_error) + " above the target " +
                  std::to_string(tol) + " after refinement and preconditioned CG");
        return HS_ERR_REFINEMENT_STALLED;
    }
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_cholesky_logdet(hs_ctx ctx, const double* L, double* logdet) {
    hs_status st = require_ctx(ctx, "hs_cholesky_logdet");
    if (st != HS_OK) return st;
    if (!L || !logdet) {
        set_error("hs_cholesky_logdet: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    st = ensure_scratch(ctx, kSmallScratch);
    if (st != HS_OK) return st;
    double* out = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kScalarOffset) + 8;
    ctx->launches += 1;
    logdiag_kernel<<<1, 1024, 0, ctx->stream>>>(L, ctx->bsz, ctx->nb, ctx->N, 0, out);
    HS_CHECK_LAUNCH("logdet");
    HS_CUDA(cudaMemcpyAsync(logdet, out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    return HS_OK;
}

hs_status hs_mixed_solve(hs_ctx ctx, const double* K, const double* b, double* x, int precision, double tol,
                         int max_steps, hs_mixed_report* rep) {
    hs_status st = require_ctx(ctx, "hs_mixed_solve");
    if (st != HS_OK) return st;
    if (!K || !b || !x) {
        set_error("hs_mixed_solve: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    hs_mixed_report R{};
    st = mixed_solve_impl(ctx, K, b, x, precision, tol, max_steps, &R);
    if (rep) *rep = R;
    return st;
}

}  // extern "C"
