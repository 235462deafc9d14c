// hs_gp.cu — reverse-mode blocked Cholesky driver and the GP negative log
// marginal likelihood with its gradient (C ABI: hs_cholesky_adjoint,
// hs_gp_nlml_grad).
//
// No reference counterpart (new form).  The NLML of a GP with targets y and
// kernel matrix K(theta) = Krbf + sn2 I (the matrix of
// src/utility/MatrixGenerator.cpp:134-155 with ARD lengthscales) is
//   NLML = 1/2 y^T K^-1 y + sum_i log L_ii + N/2 log 2pi,   K = L L^T,
// and its gradient 1/2 tr((K^-1 - alpha alpha^T) dK/dtheta), alpha = K^-1 y,
// is formed from the reverse-mode Cholesky of sum_i log L_ii (k_adjoint.cu)
// and the on-the-fly contraction of k_gp.cu.
#include <cmath>
#include <string>
#include <vector>

#include "hs_gp.cuh"
#include "hs_mixed.cuh"

namespace hs {
namespace {

constexpr double kLog2Pi = 1.8378770664093454835606594728112;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// out[0] = y.alpha over n, out[1] = sum log diag(L) over the N valid rows
__global__ void nlml_terms_kernel(const double* __restrict__ y, const double* __restrict__ alpha,
                                  const double* __restrict__ L, int bsz, int nb, int64_t N, double* __restrict__ out) {
    __shared__ double sh[2][32];
    double a = 0.0, b = 0.0;
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        a += y[i] * alpha[i];
        const int k = (int)(i / bsz), r = (int)(i % bsz);
        b += log(L[block_id(k, k, nb) * bb + (int64_t)r * bsz + r]);
    }
    a = warp_sum(a);
    b = warp_sum(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sh[0][w] = a;
        sh[1][w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            s0 += sh[0][q];
            s1 += sh[1][q];
        }
        out[0] = s0;
        out[1] = s1;
    }
}

// FP64 packed copy of the mixed factor's off-diagonal FP32 blocks (diagonal blocks
// skipped); one CTA a block, grid-stride over the blocks
__global__ void offdiag_f32_to_f64_kernel(const float* __restrict__ A32, double* __restrict__ L, int nb, int bsz) {
    const int64_t bb = (int64_t)bsz * bsz;
    const int64_t T = (int64_t)nb * (nb + 1) / 2;
    for (int64_t id = blockIdx.x; id < T; id += gridDim.x) {
        int i, j;
        block_coords(id, nb, &i, &j);
        if (i == j) continue;
        const float4* src = reinterpret_cast<const float4*>(A32 + id * bb);
        double2* dst = reinterpret_cast<double2*>(L + id * bb);
        for (int64_t e = threadIdx.x; e < bb / 4; e += blockDim.x) {
            const float4 v = __ldcs(src + e);
            __stcs(dst + 2 * e, make_double2(v.x, v.y));
            __stcs(dst + 2 * e + 1, make_double2(v.z, v.w));
        }
    }
}

__global__ void copy_pad_kernel(const double* __restrict__ y, double* __restrict__ b, int64_t N, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = i < N ? y[i] : 0.0;
}

// L's diagonal blocks from the mixed factor's FP64 copies: the lower triangle of Ld_k,
// zero above
__global__ void tril_blocks_kernel(const double* __restrict__ Ld, double* __restrict__ L, int bsz, int nb) {
    const int64_t bb = (int64_t)bsz * bsz;
    const int k = blockIdx.y;
    double* Dk = L + block_id(k, k, nb) * bb;
    const double* Sk = Ld + (int64_t)k * bb;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < bb; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / bsz), j = (int)(e % bsz);
        Dk[e] = j <= i ? Sk[e] : 0.0;
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

size_t adjoint_work_bytes(int nb, int bsz) {
    const size_t bb = (size_t)bsz * bsz * sizeof(double);
    return bb * (2 * (size_t)nb + 3 + (size_t)kAdjointPartialBlocks);
}

void adjoint_bind(void* base, int nb, int bsz, AdjointWork* w) {
    const size_t bb = (size_t)bsz * bsz;
    double* p = static_cast<double*>(base);
    w->T = p;
    p += (size_t)nb * bb;
    w->Y = p;
    p += (size_t)nb * bb;
    w->W1 = p;
    p += bb;
    w->W2 = p;
    p += bb;
    w->Dp = p;
    p += bb;
    w->partial = p;
    w->partial_blocks = kAdjointPartialBlocks;
}

hs_status cholesky_adjoint_impl(hs_ctx ctx, const double* L, double* Abar, const AdjointWork& w, cudaStream_t s) {
    const int nb = ctx->nb, bsz = ctx->bsz;
    const int64_t bb = (int64_t)bsz * bsz;
    const int valid_last = (int)(ctx->N - (int64_t)(nb - 1) * bsz);
    hs_status st = launch_zero_diag_upper(ctx, Abar, s);
    if (st != HS_OK) return st;
    // Y_k = L_kk^-T for every k in one batched substitution (the last block against a
    // copy with a unit diagonal on its padding rows)
    if ((st = launch_diag_inverses(ctx, L, w.Y, w.Dp, s)) != HS_OK) return st;
    for (int k = nb - 1; k >= 0; --k) {
        const int m = nb - k - 1;
        const int64_t dk = block_id(k, k, nb);
        const double* D = L + dk * bb;
        if (k == nb - 1 && valid_last < bsz) {
            // the padded factor is diag(L, I): unit diagonal on the padding rows
            if ((st = launch_pad_unit_diag(ctx, D, w.Dp, valid_last, s)) != HS_OK) return st;
            D = w.Dp;
        }
        double* Dbar = Abar + dk * bb;
        const double* Y = w.Y + (size_t)k * bb;  // D^-T
        if (m > 0) {
            double* Pbar = Abar + (dk + 1) * bb;  // panel blocks (k+1..nb-1, k), contiguous
            const double* P = L + (dk + 1) * bb;
            // (i) Lbar_P -= (Abar + Abar^T)_trailing L_P
            ChainArgs a = chain_args(bsz);
            a.mode = CHAIN_SYMM;
            a.k = k;
            a.nb = nb;
            a.items = m;
            a.chain = nb - k;
            a.allow_split = 1;
            a.epi = EPI_ADD;
            a.alpha = -1.0;
            a.L = L;
            a.Abar = Abar;
            if ((st = launch_chain(ctx, a, w.partial, w.partial_blocks, s)) != HS_OK) return st;
            // (ii) T_r = Lbar_rk D^-1 = Lbar_rk Y^T, then Abar_P = T
            a = chain_args(bsz);
            a.items = m;
            a.chain = 1;
            a.A0 = Pbar;
            a.sAi = bb;
            a.B0 = Y;
            a.tb = 1;
            a.C0 = w.T;
            a.sCi = bb;
            if ((st = launch_chain(ctx, a, nullptr, 0, s)) != HS_OK) return st;
            HS_CUDA(cudaMemcpyAsync(Pbar, w.T, (size_t)m * bb * sizeof(double), cudaMemcpyDeviceToDevice, s));
            // (iii) Dbar -= tril(sum_r Abar_rk^T L_rk)
            a = chain_args(bsz);
            a.items = 1;
            a.chain = m;
            a.A0 = w.T;
            a.sAq = bb;
            a.ta = 1;
            a.B0 = P;
            a.sBq = bb;
            a.C0 = Dbar;
            a.epi = EPI_ADD_LOWER;
            a.alpha = -1.0;
            a.allow_split = 1;
            if ((st = launch_chain(ctx, a, w.partial, w.partial_blocks, s)) != HS_OK) return st;
        }
        // (iv) Abar_kk = tril_h(Y (H + H^T) Y^T), H = tril_h(D^T Dbar)
        ChainArgs a = chain_args(bsz);
        a.items = 1;
        a.chain = 1;
        a.A0 = D;
        a.ta = 1;
        a.B0 = Dbar;
        a.C0 = w.W1;
        if ((st = launch_chain(ctx, a, nullptr, 0, s)) != HS_OK) return st;  // W1 = D^T Dbar
        if ((st = launch_sym_tril_half(ctx, w.W1, w.W2, s)) != HS_OK) return st;  // W2 = H + H^T
        a = chain_args(bsz);
        a.items = 1;
        a.chain = 1;
        a.A0 = w.W2;
        a.B0 = Y;
        a.tb = 1;
        a.C0 = w.W1;
        if ((st = launch_chain(ctx, a, nullptr, 0, s)) != HS_OK) return st;  // W1 = W2 Y^T
        a = chain_args(bsz);
        a.items = 1;
        a.chain = 1;
        a.A0 = Y;
        a.B0 = w.W1;
        a.C0 = Dbar;
        a.epi = EPI_TRIL_HALF;
        if ((st = launch_chain(ctx, a, nullptr, 0, s)) != HS_OK) return st;  // Abar_kk
    }
    return HS_OK;
}

}  // namespace hs

using namespace hs;

extern "C" {

hs_status hs_cholesky_adjoint(hs_ctx ctx, const double* L, double* Abar) {
    hs_status st = require_ctx(ctx, "hs_cholesky_adjoint");
    if (st != HS_OK) return st;
    if (!L || !Abar) {
        set_error("hs_cholesky_adjoint: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (ctx->bsz != 128 && ctx->bsz != 256) {
        set_error("hs_cholesky_adjoint: matrixBlockSize must be 128 or 256");
        return HS_ERR_UNSUPPORTED;
    }
    DevBuf ws;
    HS_CUDA(cudaMalloc(&ws.p, adjoint_work_bytes(ctx->nb, ctx->bsz)));
    AdjointWork w;
    adjoint_bind(ws.p, ctx->nb, ctx->bsz, &w);
    st = cholesky_adjoint_impl(ctx, L, Abar, w, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (st != HS_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "hs_cholesky_adjoint");
    return HS_OK;
}

static hs_status gp_nlml_grad_impl(hs_ctx ctx, const double* X, const double* y, int d, const double* theta,
                                   int n_ell, int precision, double tol, double* nlml, double* grad,
                                   hs_gp_report* report, hs_mixed_report* mreport) {
    hs_status st = require_ctx(ctx, "hs_gp_nlml_grad");
    if (st != HS_OK) return st;
    if (!X || !y || !theta || !nlml) {
        set_error("hs_gp_nlml_grad: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (d < 1 || d > 32 || (n_ell != 1 && n_ell != d)) {
        set_error("hs_gp_nlml_grad: need 1 <= d <= 32 and n_ell = 1 or d");
        return HS_ERR_INVALID_ARG;
    }
    if (ctx->bsz != 128 && ctx->bsz != 256) {
        set_error("hs_gp_nlml_grad: matrixBlockSize must be 128 or 256");
        return HS_ERR_UNSUPPORTED;
    }
    for (int q = 0; q < n_ell + 2; ++q)
        if (!std::isfinite(theta[q])) {
            set_error("hs_gp_nlml_grad: theta must be finite");
            return HS_ERR_INVALID_ARG;
        }
    cudaStream_t s = ctx->stream;
    const int nb = ctx->nb, bsz = ctx->bsz;
    const int64_t N = ctx->N, n = (int64_t)nb * bsz;
    const size_t packed = (size_t)total_blocks(nb) * bsz * bsz;
    std::vector<double> ell(n_ell), inv_ell(d);
    for (int q = 0; q < n_ell; ++q) ell[q] = std::exp(theta[q]);
    for (int k = 0; k < d; ++k) inv_ell[k] = 1.0 / ell[n_ell == 1 ? 0 : k];
    const double sf2 = std::exp(theta[n_ell]), sn2 = std::exp(theta[n_ell + 1]);
    const int dmax = gp_grad_dmax(d);
    const int parts = 2 * ctx->num_sms;

    // workspace: L, Abar (packed), adjoint work, alpha, Xs, inv_ell, partials, results
    const size_t adj = adjoint_work_bytes(nb, bsz);
    const size_t bytes = 2 * packed * sizeof(double) + adj + (size_t)2 * n * sizeof(double) +
                         (size_t)N * d * sizeof(double) + 64 * sizeof(double) +
                         (size_t)parts * (dmax + 2) * sizeof(double) + 256 * sizeof(double);
    if ((st = ensure_gp(ctx, bytes)) != HS_OK) return st;  // kept by the context between calls
    double* L = static_cast<double*>(ctx->gpws);
    double* Abar = L + packed;
    AdjointWork w;
    adjoint_bind(Abar + packed, nb, bsz, &w);
    double* alpha = reinterpret_cast<double*>(reinterpret_cast<char*>(Abar + packed) + adj);
    double* yb = alpha + n;  // y zero-padded (right-hand side of the mixed solve)
    double* Xs = yb + n;
    double* inv_ell_d = Xs + (size_t)N * d;
    double* part = inv_ell_d + 64;
    double* res = part + (size_t)parts * (dmax + 2);

    cudaEvent_t ev[4] = {};
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() {
            for (int i = 0; i < 4; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } eg{ev};
    for (auto& e : ev) HS_CUDA(cudaEventCreate(&e));
    HS_CUDA(cudaEventRecord(ev[0], s));
    // K(theta)
    st = launch_rbf_assemble(ctx, L, X, d, ell.data(), n_ell, sf2, sn2, s);
    if (st != HS_OK) return st;
    if (precision == 0) {
        // its FP64 factor, alpha = K^-1 y
        ctx->launches += 1;
        set_i64_dev(ctx->d_info, INT64_MAX, s);
        if ((st = factor_driver(ctx, L)) != HS_OK) return st;
        HS_CUDA(cudaEventRecord(ev[1], s));
        int64_t info = -1;
        if ((st = hs_ctx_take_info(ctx, &info)) != HS_OK) return st;
        if (info >= 0) {
            set_error("hs_gp_nlml_grad: K(theta) is not positive definite (row " + std::to_string(info) + ")");
            return HS_ERR_NOT_SPD;
        }
        ctx->launches += 1;
        copy_pad_kernel<<<64, 256, 0, s>>>(y, alpha, N, n);
        HS_CHECK_LAUNCH("copy y");
        if ((st = solve_driver(ctx, L, alpha)) != HS_OK) return st;
    } else {
        // the mixed-precision factor, alpha = K^-1 y refined in FP64 against K to the
        // backward error tol; then L (FP64, packed) <- the mixed factor: off-diagonal
        // blocks widened from FP32, diagonal blocks L_kk = ((L_kk^-T)^T)^-1 from the
        // FP64 inverses the factor keeps (K is no longer needed)
        ctx->launches += 1;
        copy_pad_kernel<<<64, 256, 0, s>>>(y, yb, N, n);
        HS_CHECK_LAUNCH("copy y");
        hs_mixed_report mr{};
        // one panel an accumulation: log|K| and the trace term come from the factor itself
        st = mixed_solve_impl(ctx, L, yb, alpha, precision, tol, 30, &mr, 1);
        if (mreport) *mreport = mr;
        if (st != HS_OK) return st;
        if (mr.shift != 0.0) {
            set_error("hs_gp_nlml_grad: the mixed-precision factor of K(theta) needed a diagonal shift; its adjoint "
                      "would be that of K + shift I");
            return HS_ERR_NOT_SPD;
        }
        MixedWork mw;
        if ((st = mixed_bind(ctx, ctx->mixed, &mw)) != HS_OK) return st;
        ctx->launches += 1;
        offdiag_f32_to_f64_kernel<<<4 * ctx->num_sms, 256, 0, s>>>(mw.A32, L, nb, bsz);
        HS_CHECK_LAUNCH("widen factor");
        // the diagonal blocks: the FP64 L_kk the diagonal chains factored (lower triangle)
        ctx->launches += 1;
        tril_blocks_kernel<<<dim3(16, nb), 256, 0, s>>>(mw.Ld, L, bsz, nb);
        HS_CHECK_LAUNCH("diagonal blocks");
        HS_CUDA(cudaEventRecord(ev[1], s));
    }
    // the two NLML terms
    ctx->launches += 1;
    nlml_terms_kernel<<<1, 1024, 0, s>>>(y, alpha, L, bsz, nb, N, res);
    HS_CHECK_LAUNCH("nlml terms");
    // reverse sweep of sum_i log L_ii, then the gradient contraction
    if ((st = launch_logdet_adjoint_init(ctx, L, Abar, s)) != HS_OK) return st;
    if ((st = cholesky_adjoint_impl(ctx, L, Abar, w, s)) != HS_OK) return st;
    HS_CUDA(cudaEventRecord(ev[2], s));
    HS_CUDA(cudaMemcpyAsync(inv_ell_d, inv_ell.data(), d * sizeof(double), cudaMemcpyHostToDevice, s));
    if ((st = launch_scale_columns(ctx, X, Xs, d, inv_ell_d, s)) != HS_OK) return st;
    if ((st = launch_gp_grad(ctx, Abar, Xs, alpha, d, n_ell == d ? 1 : 0, sf2, sn2, part, parts, res + 8, s)) !=
        HS_OK)
        return st;
    HS_CUDA(cudaEventRecord(ev[3], s));
    std::vector<double> h(8 + dmax + 2);
    HS_CUDA(cudaMemcpyAsync(h.data(), res, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    HS_CUDA(cudaStreamSynchronize(s));
    *nlml = 0.5 * h[0] + h[1] + 0.5 * (double)N * kLog2Pi;
    if (grad) {
        for (int q = 0; q < n_ell; ++q) grad[q] = h[8 + q];
        grad[n_ell] = h[8 + dmax];
        grad[n_ell + 1] = h[8 + dmax + 1];
    }
    if (report) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        report->factor_ms = ms;
        cudaEventElapsedTime(&ms, ev[1], ev[2]);
        report->adjoint_ms = ms;
        cudaEventElapsedTime(&ms, ev[2], ev[3]);
        report->grad_ms = ms;
        cudaEventElapsedTime(&ms, ev[0], ev[3]);
        report->total_ms = ms;
        report->data_fit = 0.5 * h[0];
        report->logdet = 2.0 * h[1];
    }
    return HS_OK;
}

hs_status hs_gp_nlml_grad(hs_ctx ctx, const double* X, const double* y, int d, const double* theta, int n_ell,
                          double* nlml, double* grad, hs_gp_report* report) {
    return gp_nlml_grad_impl(ctx, X, y, d, theta, n_ell, 0, 0.0, nlml, grad, report, nullptr);
}

hs_status hs_gp_nlml_grad_mixed(hs_ctx ctx, const double* X, const double* y, int d, const double* theta, int n_ell,
                                int precision, double tol, double* nlml, double* grad, hs_gp_report* report,
                                hs_mixed_report* mixed_report) {
    if (precision != HS_PRECISION_TF32X3 && precision != HS_PRECISION_BF16X3 && precision != HS_PRECISION_F16X3) {
        set_error("hs_gp_nlml_grad_mixed: precision must be HS_PRECISION_TF32X3, HS_PRECISION_BF16X3 or "
                  "HS_PRECISION_F16X3");
        return HS_ERR_UNSUPPORTED;
    }
    if (!(tol > 0.0)) {
        set_error("hs_gp_nlml_grad_mixed: tol must be > 0");
        return HS_ERR_INVALID_ARG;
    }
    return gp_nlml_grad_impl(ctx, X, y, d, theta, n_ell, precision, tol, nlml, grad, report, mixed_report);
}

}  // extern "C"
