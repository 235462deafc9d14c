// k_gp.cu — the contraction of the GP marginal-likelihood gradient.
//
// No reference counterpart (new form).  With Abar the adjoint of the lower
// entries of K for sum_i log L_ii (from the reverse sweep) and alpha = K^-1 y,
// the adjoint of NLML = 1/2 y^T alpha + sum_i log L_ii + N/2 log 2pi is
// w_ij = Abar_ij - c_ij alpha_i alpha_j over stored lower entries (c = 1/2 on
// the diagonal, 1 below it), and dNLML/dtheta = sum_{i>=j} w_ij dK_ij/dtheta.
// The dK/dtheta tiles are recomputed from the inputs, never stored:
//   dK_ij/dlog l_k   = Krbf_ij (x_ik - x_jk)^2 / l_k^2
//   dK_ij/dlog sf2   = Krbf_ij,   Krbf_ij = sf2 exp(-1/2 sum_k (x_ik - x_jk)^2 / l_k^2)
//   dK_ij/dlog sn2   = sn2 [i == j]
// One CTA per stored block (grid-stride), both input panels staged in shared
// memory scaled by 1/l_k, one fixed-order reduction per component.
#include "hs_gp.cuh"

namespace hs {
namespace {

constexpr int kGradThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Xs = X / l (per column), N x d row-major
__global__ void scale_columns_kernel(const double* __restrict__ X, double* __restrict__ Xs, int64_t N, int d,
                                     const double* __restrict__ inv_ell) {
    const int64_t total = N * d;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
        Xs[e] = X[e] * inv_ell[e % d];
}

template <int DMAX>
__global__ void __launch_bounds__(kGradThreads) gp_grad_kernel(const double* __restrict__ Abar,
                                                               const double* __restrict__ Xs,
                                                               const double* __restrict__ alpha, int d, int ard,
                                                               double sf2, double sn2, int bsz, int nb, int64_t N,
                                                               int64_t T, double* __restrict__ part) {
    extern __shared__ double sm[];
    double* xr = sm;                   // [bsz][d]  rows of the row block
    double* xc = sm + (size_t)bsz * d; // [d][bsz]  rows of the column block, transposed
    constexpr int NACC = DMAX + 2;
    double acc[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) acc[q] = 0.0;
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t blk = blockIdx.x; blk < T; blk += gridDim.x) {
        int bi, bj;
        block_coords(blk, nb, &bi, &bj);
        const int64_t i0 = (int64_t)bi * bsz, j0 = (int64_t)bj * bsz;
        __syncthreads();
        for (int e = threadIdx.x; e < bsz * d; e += blockDim.x) {
            const int r = e / d, k = e % d;
            xr[e] = (i0 + r < N) ? Xs[(i0 + r) * d + k] : 0.0;
            xc[(size_t)k * bsz + r] = (j0 + r < N) ? Xs[(j0 + r) * d + k] : 0.0;
        }
        __syncthreads();
        const double* Ab = Abar + blk * bb;
        for (int64_t e = threadIdx.x; e < bb; e += blockDim.x) {
            const int i = (int)(e / bsz), j = (int)(e % bsz);
            const int64_t gi = i0 + i, gj = j0 + j;
            if (gi >= N || gj >= N || gj > gi) continue;
            double dk[DMAX];
            double dist = 0.0;
#pragma unroll
            for (int k = 0; k < DMAX; ++k) {
                if (k < d) {
                    const double t = xr[i * d + k] - xc[(size_t)k * bsz + j];
                    dk[k] = t * t;
                    dist += dk[k];
                } else {
                    dk[k] = 0.0;
                }
            }
            const double kr = sf2 * exp(-0.5 * dist);
            const double w = Ab[e] - (gi == gj ? 0.5 : 1.0) * alpha[gi] * alpha[gj];
            const double wk = w * kr;
            if (ard) {
#pragma unroll
                for (int k = 0; k < DMAX; ++k) acc[k] += wk * dk[k];
            } else {
                acc[0] += wk * dist;
            }
            acc[DMAX] += wk;
            if (gi == gj) acc[DMAX + 1] += w * sn2;
        }
    }
    // CTA reduction, fixed order
    __shared__ double red[kGradThreads / 32][NACC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < NACC; ++q) {
        const double v = warp_sum(acc[q]);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < NACC) {
        double s = 0.0;
        for (int w = 0; w < kGradThreads / 32; ++w) s += red[w][threadIdx.x];
        part[(int64_t)blockIdx.x * NACC + threadIdx.x] = s;
    }
}

template <int DMAX>
__global__ void grad_final_kernel(const double* __restrict__ part, int parts, double* __restrict__ out) {
    constexpr int NACC = DMAX + 2;
    const int q = threadIdx.x;
    if (q >= NACC) return;
    double s = 0.0;
    for (int p = 0; p < parts; ++p) s += part[(int64_t)p * NACC + q];
    out[q] = s;
}

template <int DMAX>
hs_status grad_launch(hs_ctx ctx, const double* Abar, const double* Xs, const double* alpha, int d, int ard,
                      double sf2, double sn2, double* part, int parts, double* out, cudaStream_t s) {
    const int bsz = ctx->bsz;
    const size_t smem = (size_t)2 * bsz * d * sizeof(double);
    HS_REQUIRE(smem <= 200 * 1024, "matrixBlockSize x d too large for the gradient kernel");
    HS_CUDA(cudaFuncSetAttribute(gp_grad_kernel<DMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t T = total_blocks(ctx->nb);
    prof_begin(ctx, s, HS_KERNEL_GRAD);
    ctx->launches += 2;
    gp_grad_kernel<DMAX><<<parts, kGradThreads, smem, s>>>(Abar, Xs, alpha, d, ard, sf2, sn2, bsz, ctx->nb, ctx->N,
                                                            T, part);
    grad_final_kernel<DMAX><<<1, 64, 0, s>>>(part, parts, out);
    HS_CHECK_LAUNCH("gp_grad");
    const double elems = (double)ctx->N * (ctx->N + 1) / 2.0;
    prof_end(ctx, s, HS_KERNEL_GRAD, elems * (4.0 * d + 12.0), (double)T * bsz * bsz * 8.0);
    return HS_OK;
}

}  // namespace

// out[0..DMAX) lengthscale components (out[0] only when !ard), out[DMAX] sf2,
// out[DMAX+1] sn2, where DMAX = 8, 16 or 32 is returned in the layout the
// caller reads through gp_grad_slots()
hs_status launch_gp_grad(hs_ctx ctx, const double* Abar, const double* Xs, const double* alpha, int d, int ard,
                         double sf2, double sn2, double* part, int parts, double* out, cudaStream_t s) {
    HS_REQUIRE(d >= 1 && d <= 32, "the gradient supports d <= 32 features");
    if (d <= 8) return grad_launch<8>(ctx, Abar, Xs, alpha, d, ard, sf2, sn2, part, parts, out, s);
    if (d <= 16) return grad_launch<16>(ctx, Abar, Xs, alpha, d, ard, sf2, sn2, part, parts, out, s);
    return grad_launch<32>(ctx, Abar, Xs, alpha, d, ard, sf2, sn2, part, parts, out, s);
}

hs_status launch_scale_columns(hs_ctx ctx, const double* X, double* Xs, int d, const double* inv_ell_dev,
                               cudaStream_t s) {
    ctx->launches += 1;
    scale_columns_kernel<<<4 * ctx->num_sms, 256, 0, s>>>(X, Xs, ctx->N, d, inv_ell_dev);
    HS_CHECK_LAUNCH("scale columns");
    return HS_OK;
}

}  // namespace hs
