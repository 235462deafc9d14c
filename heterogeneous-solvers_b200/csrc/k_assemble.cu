// k_assemble.cu — RBF kernel-matrix assembly into packed lower block storage.
//
// Replaces MatrixGenerator::generateSPDMatrix's per-block kernel
// (src/utility/MatrixGenerator.cpp:134-155): for every stored block and every
// in-range entry, distance = sum_k (x_ik - x_jk)^2 with k ascending,
// K = sf2 * exp(-0.5/l^2 * distance), plus sn2 on the global diagonal.  The
// reference's 1-D sliding window (x_ik = series[i+k-7]) is one instance of the
// row-major X (N x d) used here; the ARD form multiplies each difference by
// 1/l_k and uses exp(-0.5 * distance).  Padding entries are written as zero.
//
// One CTA per stored block: the block's two row panels of X are staged in
// shared memory (the column panel transposed so that consecutive threads read
// consecutive doubles), and each thread produces two horizontally adjacent
// entries that it writes with one 16-byte store, so every warp writes 512
// contiguous bytes per instruction.
#include "hs_internal.cuh"

namespace hs {
namespace {

constexpr int kMaxD = 64;

__global__ void __launch_bounds__(256) rbf_assemble_kernel(double* __restrict__ A, const double* __restrict__ X,
                                                           int64_t N, int d, int bsz, int nb, int ard,
                                                           const double* __restrict__ wsc /* device, d */,
                                                           double sf2, double sn2, double iso_scale) {
    extern __shared__ double sm[];
    double* Xi = sm;                      // bsz x d (row panel of the block row)
    double* XjT = sm + (size_t)bsz * d;   // d x bsz (column panel, transposed)
    __shared__ double w[kMaxD];
    int ib, jb;
    block_coords(blockIdx.x, nb, &ib, &jb);
    const int64_t i0 = (int64_t)ib * bsz, j0 = (int64_t)jb * bsz;
    for (int e = threadIdx.x; e < bsz * d; e += blockDim.x) {
        const int r = e / d, k = e % d;
        Xi[e] = (i0 + r < N) ? X[(i0 + r) * d + k] : 0.0;
        XjT[(size_t)k * bsz + r] = (j0 + r < N) ? X[(j0 + r) * d + k] : 0.0;
    }
    if (threadIdx.x < d) w[threadIdx.x] = ard ? wsc[threadIdx.x] : 1.0;
    __syncthreads();
    double* blk = A + (size_t)blockIdx.x * bsz * bsz;
    const int half = bsz >> 1;  // bsz even on this path
    for (int p = threadIdx.x; p < bsz * half; p += blockDim.x) {
        const int il = p / half;
        const int jl = 2 * (p % half);
        const int64_t ig = i0 + il, jg = j0 + jl;
        double v0 = 0.0, v1 = 0.0;
        if (ig < N) {
            double d0 = 0.0, d1 = 0.0;
            const double* xi = Xi + (size_t)il * d;
            if (ard) {
                for (int k = 0; k < d; ++k) {
                    const double2 xj = *reinterpret_cast<const double2*>(XjT + (size_t)k * bsz + jl);
                    const double t0 = (xi[k] - xj.x) * w[k];
                    const double t1 = (xi[k] - xj.y) * w[k];
                    d0 += t0 * t0;
                    d1 += t1 * t1;
                }
                if (jg < N) v0 = sf2 * exp(-0.5 * d0);
                if (jg + 1 < N) v1 = sf2 * exp(-0.5 * d1);
            } else {
                for (int k = 0; k < d; ++k) {
                    const double2 xj = *reinterpret_cast<const double2*>(XjT + (size_t)k * bsz + jl);
                    const double t0 = xi[k] - xj.x;
                    const double t1 = xi[k] - xj.y;
                    d0 += t0 * t0;
                    d1 += t1 * t1;
                }
                if (jg < N) v0 = sf2 * exp(iso_scale * d0);
                if (jg + 1 < N) v1 = sf2 * exp(iso_scale * d1);
            }
            if (jg < N && ig == jg) v0 += sn2;
            if (jg + 1 < N && ig == jg + 1) v1 += sn2;
        }
        __stcs(reinterpret_cast<double2*>(blk + (size_t)il * bsz + jl), make_double2(v0, v1));
    }
}

// The same entries, 4 x 4 per thread (bsz a multiple of 4 with bsz / 4 dividing
// 256): each X value read from shared memory serves four entries, which takes the
// kernel off the shared-memory bandwidth it was bound by with two entries a thread.
// Thread t takes columns 4 (t % G) .. +3 (G = bsz / 4 column groups) and rows
// 4 (t / G) + R p .. +3 in pass p (R = 4 * 256 / G rows a pass); a warp shares its
// rows (broadcast reads) and writes 32 x 32 contiguous bytes per row.  Per entry the
// distance is summed over k ascending exactly as in rbf_assemble_kernel.
__global__ void __launch_bounds__(256) rbf_assemble_tile_kernel(double* __restrict__ A,
                                                                const double* __restrict__ X, int64_t N, int d,
                                                                int bsz, int nb, int ard,
                                                                const double* __restrict__ wsc, double sf2,
                                                                double sn2, double iso_scale) {
    extern __shared__ double sm[];
    double* Xi = sm;                      // bsz x d
    double* XjT = sm + (size_t)bsz * d;   // d x bsz
    __shared__ double w[kMaxD];
    int ib, jb;
    block_coords(blockIdx.x, nb, &ib, &jb);
    const int64_t i0 = (int64_t)ib * bsz, j0 = (int64_t)jb * bsz;
    for (int e = threadIdx.x; e < bsz * d; e += blockDim.x) {
        const int r = e / d, k = e % d;
        Xi[e] = (i0 + r < N) ? X[(i0 + r) * d + k] : 0.0;
        XjT[(size_t)k * bsz + r] = (j0 + r < N) ? X[(j0 + r) * d + k] : 0.0;
    }
    if (threadIdx.x < d) w[threadIdx.x] = ard ? wsc[threadIdx.x] : 1.0;
    __syncthreads();
    double* blk = A + (size_t)blockIdx.x * bsz * bsz;
    const int G = bsz >> 2;
    const int cg = threadIdx.x % G, rg = threadIdx.x / G;
    const int rows_pass = 4 * (256 / G);
    const int jl = 4 * cg;
    for (int il0 = 4 * rg; il0 < bsz; il0 += rows_pass) {
        double acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
        for (int k = 0; k < d; ++k) {
            const double2 xa = *reinterpret_cast<const double2*>(XjT + (size_t)k * bsz + jl);
            const double2 xb = *reinterpret_cast<const double2*>(XjT + (size_t)k * bsz + jl + 2);
            const double xj[4] = {xa.x, xa.y, xb.x, xb.y};
            const double wk = w[k];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double xi = Xi[(size_t)(il0 + r) * d + k];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double t = ard ? (xi - xj[c]) * wk : xi - xj[c];
                    acc[r][c] += t * t;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int64_t ig = i0 + il0 + r;
            double v[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int64_t jg = j0 + jl + c;
                double e = 0.0;
                if (ig < N && jg < N) {
                    e = sf2 * exp(ard ? -0.5 * acc[r][c] : iso_scale * acc[r][c]);
                    if (ig == jg) e += sn2;
                }
                v[c] = e;
            }
            double* o = blk + (size_t)(il0 + r) * bsz + jl;
            __stcs(reinterpret_cast<double2*>(o), make_double2(v[0], v[1]));
            __stcs(reinterpret_cast<double2*>(o + 2), make_double2(v[2], v[3]));
        }
    }
}

// odd block sizes (tests only): one entry per thread, plain stores
__global__ void rbf_assemble_odd_kernel(double* __restrict__ A, const double* __restrict__ X, int64_t N, int d,
                                        int bsz, int nb, int ard, const double* __restrict__ wsc, double sf2,
                                        double sn2, double iso_scale) {
    int ib, jb;
    block_coords(blockIdx.x, nb, &ib, &jb);
    double* blk = A + (size_t)blockIdx.x * bsz * bsz;
    for (int e = threadIdx.x; e < bsz * bsz; e += blockDim.x) {
        const int il = e / bsz, jl = e % bsz;
        const int64_t ig = (int64_t)ib * bsz + il, jg = (int64_t)jb * bsz + jl;
        double v = 0.0;
        if (ig < N && jg < N) {
            double dist = 0.0;
            for (int k = 0; k < d; ++k) {
                const double t = ard ? (X[ig * d + k] - X[jg * d + k]) * wsc[k] : X[ig * d + k] - X[jg * d + k];
                dist += t * t;
            }
            v = sf2 * exp((ard ? -0.5 : iso_scale) * dist);
            if (ig == jg) v += sn2;
        }
        blk[e] = v;
    }
}

}  // namespace

hs_status launch_rbf_assemble(hs_ctx ctx, double* A, const double* X, int d, const double* ell_host, int n_ell,
                              double sf2, double sn2, cudaStream_t s) {
    HS_REQUIRE(d >= 1 && d <= kMaxD, "d must be in [1, 64]");
    HS_REQUIRE(n_ell == 1 || n_ell == d, "n_ell must be 1 or d");
    const int bsz = ctx->bsz, nb = ctx->nb;
    const int ard = (n_ell == d && d > 1) ? 1 : 0;
    double* wdev = nullptr;
    if (ard) {
        hs_status st = ensure_scratch(ctx, kSmallScratch);
        if (st != HS_OK) return st;
        // the small scratch area's constants slot holds the 1/l_k factors
        wdev = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kConstOffset);
        double w[kMaxD];
        for (int k = 0; k < d; ++k) {
            HS_REQUIRE(ell_host[k] > 0.0, "lengthscales must be positive");
            w[k] = 1.0 / ell_host[k];
        }
        HS_CUDA(cudaMemcpyAsync(wdev, w, d * sizeof(double), cudaMemcpyHostToDevice, s));
        // the copy reads the host stack: finish it before returning
        HS_CUDA(cudaStreamSynchronize(s));
    }
    HS_REQUIRE(ell_host[0] > 0.0, "lengthscale must be positive");
    const double iso_scale = -0.5 / (ell_host[0] * ell_host[0]);
    const int64_t T = total_blocks(nb);
    HS_REQUIRE(T < (1LL << 31), "too many blocks");
    const size_t smem = (size_t)2 * bsz * d * sizeof(double);
    prof_begin(ctx, s, HS_KERNEL_ASSEMBLE);
    ctx->launches += 1;
    if (bsz % 4 == 0 && 256 % (bsz / 4) == 0 && smem <= 200 * 1024) {
        if (smem > 48 * 1024)
            HS_CUDA(cudaFuncSetAttribute(rbf_assemble_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
        rbf_assemble_tile_kernel<<<(unsigned)T, 256, smem, s>>>(A, X, ctx->N, d, bsz, nb, ard, wdev, sf2, sn2,
                                                                iso_scale);
    } else if (bsz % 2 == 0 && smem <= 200 * 1024) {
        if (smem > 48 * 1024)
            HS_CUDA(cudaFuncSetAttribute(rbf_assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        rbf_assemble_kernel<<<(unsigned)T, 256, smem, s>>>(A, X, ctx->N, d, bsz, nb, ard, wdev, sf2, sn2, iso_scale);
    } else {
        rbf_assemble_odd_kernel<<<(unsigned)T, 256, 0, s>>>(A, X, ctx->N, d, bsz, nb, ard, wdev, sf2, sn2, iso_scale);
    }
    HS_CHECK_LAUNCH("rbf_assemble");
    prof_end(ctx, s, HS_KERNEL_ASSEMBLE, (double)T * bsz * bsz * (3.0 * d + 2.0), (double)T * bsz * bsz * 8.0);
    return HS_OK;
}

}  // namespace hs
