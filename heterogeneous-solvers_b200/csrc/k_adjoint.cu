// k_adjoint.cu — reverse-mode (adjoint) blocked Cholesky on the FP64 tensor
// cores, and the kernels of the GP marginal-likelihood gradient.
//
// No reference counterpart (new form).  The reverse sweep undoes the
// right-looking factor of src/solver/cholesky/Cholesky.cpp:446-471 block
// column by block column, k = nb-1 .. 0.  With Abar the adjoint of the lower
// entries of A (initially the adjoint Lbar of the factor), P the panel rows
// r > k of column k and D = L_kk:
//   (i)   Lbar_P -= (Abar + Abar^T)_trailing * L_P      (trailing block SYMM)
//   (ii)  Abar_P  = Lbar_P * D^-1                        (reverse of the TRSM)
//   (iii) Dbar   -= tril(sum_r Abar_rk^T L_rk)          (the TRSM's use of D)
//   (iv)  Abar_kk = tril_h(D^-T (H + H^T) D^-1),  H = tril_h(D^T Dbar)
// where tril_h keeps the lower triangle with the diagonal halved.  (iv) is
// the level-3 form of the reverse of an unblocked Cholesky (I. Murray,
// "Differentiation of the Cholesky decomposition", 2016): from A = L L^T,
// L^-1 dA L^-T = X + X^T with X = L^-1 dL lower triangular, so dL =
// L tril_h(L^-1 dA L^-T), and tr(Lbar^T dL) = tr(sym(H) L^-1 dA L^-T) with
// H = tril_h(L^T Lbar).  Every product runs on the FP64 tensor pipe
// (mma.sync m8n8k4 f64) in the chained tile kernel below.
#include <cmath>

#include "hs_gp.cuh"

namespace hs {
namespace {

// 128 x 64 output tiles, 8 warps of 32 x 32, 3-stage ring: 128 registers and 90 KB of
// shared memory, two CTAs an SM (one CTA's prologue / epilogue beside the other's MMAs)
constexpr int BM = 128, BN = 64, BK = 16, STAGES = 3;
constexpr int WM = 32, WN = 32, kWarpsN = BN / WN;
constexpr int SPAD = 20;        // row pitch (doubles) of K-contiguous operand rows
// M- / N-contiguous rows are read by lane (g, t) at row 4 kk + t, column 8 i + g: a pitch
// of 4 (mod 16) doubles puts the 16 lanes of each half-warp's 8-byte loads on 16
// different 8-byte bank pairs (a pitch of 8 mod 16 would put t and t + 2 on the same pair)
constexpr int LDTA = BM + 4;    // row pitch (doubles) of M-contiguous A rows
constexpr int LDTB = BN + 4;    // row pitch (doubles) of N-contiguous B rows
constexpr int kStageA = BM * SPAD;  // >= BK * LDTA
constexpr int kStageB = BN * SPAD;  // >= BK * LDTB
constexpr int kStage = kStageA + kStageB;
constexpr int kChainSmem = STAGES * kStage * (int)sizeof(double);  // 90 KB
static_assert(BK * LDTA <= kStageA && BK * LDTB <= kStageB, "stage layout");

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// One element of a product chain: op(A) op(B), both bsz x bsz row-major blocks.
struct Elem {
    const double* A;
    const double* B;
    int ta, tb;  // 1: the operand enters transposed
};

__device__ __forceinline__ Elem chain_elem(const ChainArgs& a, int item, int64_t q) {
    const int64_t bb = (int64_t)a.bsz * a.bsz;
    Elem e;
    if (a.mode == CHAIN_SYMM) {
        // output Lbar_rk, r = k+1+item; chain over c = k+1..r (Abar_rc L_ck) then
        // c = r..nb-1 (Abar_cr^T L_ck): the symmetric trailing adjoint times the panel
        const int k = a.k, r = k + 1 + item;
        if (q < r - k) {
            const int c = k + 1 + (int)q;
            e.A = a.Abar + block_id(r, c, a.nb) * bb;
            e.B = a.L + block_id(c, k, a.nb) * bb;
            e.ta = 0;
        } else {
            const int c = r + (int)(q - (r - k));
            e.A = a.Abar + block_id(c, r, a.nb) * bb;
            e.B = a.L + block_id(c, k, a.nb) * bb;
            e.ta = 1;
        }
        e.tb = 0;
    } else {
        // strided list: element q of item: A0 + item*sAi + q*sAq, B0 + item*sBi + q*sBq
        e.A = a.A0 + item * a.sAi + q * a.sAq;
        e.B = a.B0 + item * a.sBi + q * a.sBq;
        e.ta = a.ta;
        e.tb = a.tb;
    }
    return e;
}

// One K slab of the warp's 32 x 32 tile, for one operand orientation (TA: A staged
// M-contiguous, TB: B staged K-contiguous), as straight-line code per orientation
template <bool TA, bool TB>
__device__ __forceinline__ void slab_mma(double (&acc)[4][4][2], const double* __restrict__ As,
                                         const double* __restrict__ Bs, int wm, int wn, int g, int t) {
#pragma unroll
    for (int kk = 0; kk < BK / 4; ++kk) {
        double av[4], bv[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
            av[mi] = TA ? As[(kk * 4 + t) * LDTA + wm * WM + mi * 8 + g] : As[(wm * WM + mi * 8 + g) * SPAD + kk * 4 + t];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
            bv[ni] = TB ? Bs[(wn * WN + ni * 8 + g) * SPAD + kk * 4 + t] : Bs[(kk * 4 + t) * LDTB + wn * WN + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], av[mi], bv[ni]);
    }
}

// One CTA = one 128 x 64 tile of one output block, accumulating the chain
// elements [q0, q1) of its item; 8 warps of 32 x 32, K streamed in 16-wide
// slabs through a 3-stage cp.async ring.  Operands that enter transposed are
// staged with the M (or N) index contiguous, the others with K contiguous.
__global__ void __launch_bounds__(256, 2) chain_dmma_kernel(ChainArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int tpm = a.bsz / BM, tpn = a.bsz / BN;
    const int64_t idx = blockIdx.x;
    const int split = (int)(idx % a.splits);
    const int64_t rest = idx / a.splits;
    const int tile = (int)(rest % (tpm * tpn));
    const int item = (int)(rest / (tpm * tpn));
    const int ti = tile / tpn, tj = tile % tpn;
    const int64_t q0 = a.chain * split / a.splits, q1 = a.chain * (split + 1) / a.splits;
    // slabs per chain element: bsz / BK = 16 or 8, a power of two, so that the slab
    // index splits by shift and mask (no 64-bit division in the loop)
    const int lg = a.bsz == 256 ? 4 : 3, spb = 1 << lg;
    const int nk = (int)(q1 - q0) * spb;
    const int bsz = a.bsz;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp / kWarpsN, wn = warp % kWarpsN;
    const int g = lane >> 2, t = lane & 3;

    double acc[4][4][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;

    auto load_stage = [&](int stage, int kt) {
        const Elem e = chain_elem(a, item, q0 + (kt >> lg));
        const int kc = (kt & (spb - 1)) * BK;
        double* As = smem + stage * kStage;
        double* Bs = As + kStageA;
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {  // A: 1024 16-byte copies
            const int x = tid + 256 * qq;
            if (!e.ta) {  // A_op[m][k] = A[ti*128+m][kc+k]: rows m, K contiguous
                const int row = x >> 3, ch = x & 7;
                cp_async16(As + row * SPAD + ch * 2, e.A + (size_t)(ti * BM + row) * bsz + kc + ch * 2);
            } else {      // A_op[m][k] = A[kc+k][ti*128+m]: rows k, M contiguous
                const int row = x >> 6, ch = x & 63;
                cp_async16(As + row * LDTA + ch * 2, e.A + (size_t)(kc + row) * bsz + ti * BM + ch * 2);
            }
        }
#pragma unroll
        for (int qq = 0; qq < 2; ++qq) {  // B: 512 16-byte copies
            const int x = tid + 256 * qq;
            if (!e.tb) {  // B_op[k][n] = B[kc+k][tj*64+n]: rows k, N contiguous
                const int row = x >> 5, ch = x & 31;
                cp_async16(Bs + row * LDTB + ch * 2, e.B + (size_t)(kc + row) * bsz + tj * BN + ch * 2);
            } else {      // B_op[k][n] = B[tj*64+n][kc+k]: rows n, K contiguous
                const int row = x >> 3, ch = x & 7;
                cp_async16(Bs + row * SPAD + ch * 2, e.B + (size_t)(tj * BN + row) * bsz + kc + ch * 2);
            }
        }
    };
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0, st = 0; kt < nk; ++kt, st = st + 1 == STAGES ? 0 : st + 1) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nx = kt + STAGES - 1;
            if (nx < nk) load_stage(st == 0 ? STAGES - 1 : st - 1, nx);
            cp_async_commit();
        }
        // operand orientation of this slab's chain element (its pointers are only
        // needed by the loads): CHAIN_SYMM takes Abar_cr^T from c = r on (q >= r - k)
        const int64_t q = q0 + (kt >> lg);
        const int eta = a.mode == CHAIN_SYMM ? (q >= item + 1) : a.ta;
        const int etb = a.mode == CHAIN_SYMM ? 0 : a.tb;
        const double* As = smem + st * kStage;
        const double* Bs = As + kStageA;
        if (!eta && !etb)
            slab_mma<false, false>(acc, As, Bs, wm, wn, g, t);
        else if (eta && !etb)
            slab_mma<true, false>(acc, As, Bs, wm, wn, g, t);
        else if (!eta)
            slab_mma<false, true>(acc, As, Bs, wm, wn, g, t);
        else
            slab_mma<true, true>(acc, As, Bs, wm, wn, g, t);
    }
    cp_async_wait<0>();

    // ---- epilogue
    const int64_t bb = (int64_t)bsz * bsz;
    double* C;
    int epi = a.epi;
    if (a.splits > 1) {
        C = a.partial + ((int64_t)split * a.items + item) * bb;
        epi = EPI_STORE;
    } else if (a.mode == CHAIN_SYMM) {
        C = a.Abar + block_id(a.k + 1 + item, a.k, a.nb) * bb;
    } else {
        C = a.C0 + item * a.sCi;
    }
    const double alpha = a.alpha;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int r = ti * BM + wm * WM + mi * 8 + g;
            const int c = tj * BN + wn * WN + ni * 8 + 2 * t;
            double* p = C + (size_t)r * bsz + c;
            const double v0 = alpha * acc[mi][ni][0], v1 = alpha * acc[mi][ni][1];
            if (epi == EPI_STORE) {
                *reinterpret_cast<double2*>(p) = make_double2(v0, v1);
            } else if (epi == EPI_ADD) {
                double2 o = *reinterpret_cast<double2*>(p);
                o.x += v0;
                o.y += v1;
                *reinterpret_cast<double2*>(p) = o;
            } else if (epi == EPI_ADD_LOWER) {
                if (c <= r) p[0] += v0;
                if (c + 1 <= r) p[1] += v1;
            } else {  // EPI_TRIL_HALF: lower triangle, diagonal halved, upper zero
                p[0] = c < r ? v0 : (c == r ? 0.5 * v0 : 0.0);
                p[1] = c + 1 < r ? v1 : (c + 1 == r ? 0.5 * v1 : 0.0);
            }
        }
}

// C (+)= sum over splits of the partial blocks, in split order
__global__ void reduce_splits_kernel(const double* __restrict__ partial, int splits, int items, int64_t bb,
                                     const ChainArgs a) {
    const int item = blockIdx.y;
    double* C;
    if (a.mode == CHAIN_SYMM) C = a.Abar + block_id(a.k + 1 + item, a.k, a.nb) * bb;
    else C = a.C0 + item * a.sCi;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < bb; e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int sp = 0; sp < splits; ++sp) s += partial[((int64_t)sp * items + item) * bb + e];
        const int r = (int)(e / a.bsz), c = (int)(e % a.bsz);
        if (a.epi == EPI_STORE) C[e] = s;
        else if (a.epi == EPI_ADD) C[e] += s;
        else if (a.epi == EPI_ADD_LOWER) {
            if (c <= r) C[e] += s;
        } else {
            C[e] = c < r ? s : (c == r ? 0.5 * s : 0.0);
        }
    }
}

// ------------------------------------------------------------------ helpers
// Abar = 0 except diag(Abar_kk) = 1 / L_ii for valid rows: the adjoint of
// sum_i log L_ii with respect to L
__global__ void zero_kernel(double* __restrict__ p, int64_t total) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
        p[e] = 0.0;
}
__global__ void set_logdet_diag_kernel(const double* __restrict__ L, double* __restrict__ Abar, int bsz, int nb,
                                       int64_t N) {
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(i / bsz), r = (int)(i % bsz);
        const int64_t off = block_id(k, k, nb) * bb + (int64_t)r * bsz + r;
        Abar[off] = 1.0 / L[off];
    }
}

// Dp = D with unit diagonal on the rows >= valid (padding rows of the last
// block): the padded factor is diag(L, I), so its diagonal blocks are invertible
__global__ void pad_unit_diag_kernel(const double* __restrict__ D, double* __restrict__ Dp, int bsz, int valid) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < bsz * bsz; e += gridDim.x * blockDim.x) {
        const int i = e / bsz, j = e % bsz;
        Dp[e] = (i == j && i >= valid) ? 1.0 : D[e];
    }
}

// zero the strict upper triangles of the diagonal blocks (the adjoint of a
// lower-triangular factor has none)
__global__ void zero_diag_upper_kernel(double* __restrict__ Abar, int bsz, int nb) {
    const int64_t bb = (int64_t)bsz * bsz;
    double* D = Abar + block_id(blockIdx.y, blockIdx.y, nb) * bb;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < bsz * bsz; e += gridDim.x * blockDim.x)
        if (e % bsz > e / bsz) D[e] = 0.0;
}

__global__ void identity_kernel(double* __restrict__ Y, int bsz) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < bsz * bsz; e += gridDim.x * blockDim.x)
        Y[e] = (e / bsz == e % bsz) ? 1.0 : 0.0;
}

// M = H + H^T with H = tril_h(G): M_ij = G_ij (i > j), G_ji (i < j), G_ii (i == j)
__global__ void sym_tril_half_kernel(const double* __restrict__ G, double* __restrict__ M, int bsz) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < bsz * bsz; e += gridDim.x * blockDim.x) {
        const int i = e / bsz, j = e % bsz;
        M[e] = i >= j ? G[e] : G[(size_t)j * bsz + i];
    }
}

// Split count of a chain over `base_ctas` output tiles (`sms` = CTAs resident at once): the s that
// minimises the time model waves(base s) x ceil(chain / s) chain steps, plus the
// fixed-order reduction of the s partial blocks of each item (~0.1 chain step a
// partial tile a CTA slot), so that the last wave is not left mostly empty.
int pick_splits(int64_t base_ctas, int64_t chain, int items, int64_t partial_blocks, int sms) {
    int64_t best = 1;
    double best_cost = 1e300;
    const int64_t smax = chain < 64 ? chain : 64;
    for (int64_t s = 1; s <= smax; ++s) {
        if (s > 1 && s * items > partial_blocks) break;
        const int64_t waves = (base_ctas * s + sms - 1) / sms;
        const double cost = (double)waves * (double)((chain + s - 1) / s) +
                            (s > 1 ? 0.1 * (double)(base_ctas * s) / sms : 0.0);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = s;
        }
    }
    return (int)best;
}

bool g_chain_attr[64] = {};

hs_status chain_attrs() {
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && g_chain_attr[dev]) return HS_OK;
    HS_CUDA(cudaFuncSetAttribute(chain_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmem));
    if (dev >= 0 && dev < 64) g_chain_attr[dev] = true;
    return HS_OK;
}

}  // namespace

hs_status launch_chain(hs_ctx ctx, ChainArgs a, double* partial, int64_t partial_blocks, cudaStream_t s) {
    hs_status st = chain_attrs();
    if (st != HS_OK) return st;
    HS_REQUIRE(a.bsz == 128 || a.bsz == 256, "the tensor-core adjoint supports matrixBlockSize 128 or 256");
    if (a.items <= 0 || a.chain <= 0) return HS_OK;
    HS_REQUIRE(a.chain * (a.bsz / BK) < (1LL << 31), "product chain too long");
    const int64_t base = (int64_t)a.items * (a.bsz / BM) * (a.bsz / BN);
    a.splits = (partial && a.allow_split) ? pick_splits(base, a.chain, a.items, partial_blocks, 2 * ctx->num_sms) : 1;
    a.partial = partial;
    const int64_t grid = base * a.splits;
    HS_REQUIRE(grid < (1LL << 31), "too many tiles");
    const double n3 = (double)a.bsz * a.bsz * a.bsz;
    prof_begin(ctx, s, HS_KERNEL_ADJOINT);
    ctx->launches += 1;
    chain_dmma_kernel<<<(unsigned)grid, 256, kChainSmem, s>>>(a);
    HS_CHECK_LAUNCH("chain_dmma_kernel");
    prof_end(ctx, s, HS_KERNEL_ADJOINT, 2.0 * n3 * (double)a.chain * a.items,
             8.0 * (double)a.bsz * a.bsz * (2.0 * a.chain * a.items + 2.0 * a.items));
    if (a.splits > 1) {
        const int64_t bb = (int64_t)a.bsz * a.bsz;
        ctx->launches += 1;
        dim3 grid2((unsigned)((bb + 255) / 256 < 64 ? (bb + 255) / 256 : 64), (unsigned)a.items);
        reduce_splits_kernel<<<grid2, 256, 0, s>>>(partial, a.splits, a.items, bb, a);
        HS_CHECK_LAUNCH("reduce_splits");
    }
    return HS_OK;
}

hs_status launch_logdet_adjoint_init(hs_ctx ctx, const double* L, double* Abar, cudaStream_t s) {
    const int64_t total = total_blocks(ctx->nb) * (int64_t)ctx->bsz * ctx->bsz;
    ctx->launches += 2;
    zero_kernel<<<4 * ctx->num_sms, 256, 0, s>>>(Abar, total);
    set_logdet_diag_kernel<<<64, 256, 0, s>>>(L, Abar, ctx->bsz, ctx->nb, ctx->N);
    HS_CHECK_LAUNCH("logdet adjoint init");
    return HS_OK;
}

hs_status launch_pad_unit_diag(hs_ctx ctx, const double* D, double* Dp, int valid, cudaStream_t s) {
    ctx->launches += 1;
    pad_unit_diag_kernel<<<64, 256, 0, s>>>(D, Dp, ctx->bsz, valid);
    HS_CHECK_LAUNCH("pad diag");
    return HS_OK;
}

hs_status launch_zero_diag_upper(hs_ctx ctx, double* Abar, cudaStream_t s) {
    ctx->launches += 1;
    zero_diag_upper_kernel<<<dim3(16, ctx->nb), 256, 0, s>>>(Abar, ctx->bsz, ctx->nb);
    HS_CHECK_LAUNCH("zero diag upper");
    return HS_OK;
}

hs_status launch_identity(hs_ctx ctx, double* Y, cudaStream_t s) {
    ctx->launches += 1;
    identity_kernel<<<64, 256, 0, s>>>(Y, ctx->bsz);
    HS_CHECK_LAUNCH("identity");
    return HS_OK;
}

hs_status launch_sym_tril_half(hs_ctx ctx, const double* G, double* M, cudaStream_t s) {
    ctx->launches += 1;
    sym_tril_half_kernel<<<64, 256, 0, s>>>(G, M, ctx->bsz);
    HS_CHECK_LAUNCH("sym tril half");
    return HS_OK;
}

}  // namespace hs
