// hs_gp.cuh — internals of the reverse-mode Cholesky (k_adjoint.cu) and the
// GP marginal likelihood and gradient (k_gp.cu, hs_gp.cu).
#pragma once

#include "hs_internal.cuh"

namespace hs {

// chained tensor-core block products: one output block per item,
// C_item (op)= alpha * sum_q op(A_q) op(B_q)
enum { CHAIN_LIST = 0, CHAIN_SYMM = 1 };
enum { EPI_STORE = 0, EPI_ADD = 1, EPI_ADD_LOWER = 2, EPI_TRIL_HALF = 3 };

struct ChainArgs {
    int mode;          // CHAIN_LIST: strided operand lists; CHAIN_SYMM: reverse-sweep step (i)
    int k, nb, bsz;
    int items;         // output blocks
    int64_t chain;     // products per output block
    int splits;        // set by launch_chain
    int allow_split;   // the chain may be split across CTAs (fixed-order reduction after)
    int epi;           // EPI_*
    double alpha;
    const double* L;   // CHAIN_SYMM: factor
    double* Abar;      // CHAIN_SYMM: adjoint; outputs Lbar_rk, r = k+1+item
    const double* A0;  // CHAIN_LIST: A of (item, q) = A0 + item*sAi + q*sAq
    int64_t sAi, sAq;
    const double* B0;
    int64_t sBi, sBq;
    int ta, tb;        // CHAIN_LIST: transposed operands
    double* C0;        // CHAIN_LIST: output of item = C0 + item*sCi
    int64_t sCi;
    double* partial;   // set by launch_chain
};

inline ChainArgs chain_args(int bsz) {
    ChainArgs a{};
    a.mode = CHAIN_LIST;
    a.bsz = bsz;
    a.splits = 1;
    a.alpha = 1.0;
    a.epi = EPI_STORE;
    return a;
}

// `partial` (nullable) holds `partial_blocks` bsz x bsz blocks for split chains
hs_status launch_chain(hs_ctx ctx, ChainArgs a, double* partial, int64_t partial_blocks, cudaStream_t s);
hs_status launch_logdet_adjoint_init(hs_ctx ctx, const double* L, double* Abar, cudaStream_t s);
hs_status launch_pad_unit_diag(hs_ctx ctx, const double* D, double* Dp, int valid, cudaStream_t s);
hs_status launch_zero_diag_upper(hs_ctx ctx, double* Abar, cudaStream_t s);
hs_status launch_identity(hs_ctx ctx, double* Y, cudaStream_t s);
hs_status launch_sym_tril_half(hs_ctx ctx, const double* G, double* M, cudaStream_t s);
// B <- B L^-T for `items` contiguous bsz x bsz blocks (k_factor.cu)
hs_status launch_trsm_on(hs_ctx ctx, const double* L, int n, double* B, int items, cudaStream_t s);

// workspace of the reverse sweep
struct AdjointWork {
    double* T;        // panel temporary (nb blocks)
    double* Y;        // L_kk^-T for every diagonal block k (nb blocks)
    double* W1;
    double* W2;
    double* Dp;       // last diagonal block with unit padding diagonal
    double* partial;  // split-chain partial blocks
    int64_t partial_blocks;
};
constexpr int64_t kAdjointPartialBlocks = 512;
size_t adjoint_work_bytes(int nb, int bsz);
void adjoint_bind(void* base, int nb, int bsz, AdjointWork* w);
// Abar (packed lower blocks, holding Lbar on entry) <- adjoint of the lower
// entries of A = L L^T; L is not modified
hs_status cholesky_adjoint_impl(hs_ctx ctx, const double* L, double* Abar, const AdjointWork& w, cudaStream_t s);

// gradient of the GP NLML: sum over stored lower elements of
// (Abar_ij - c_ij alpha_i alpha_j) dK_ij/dtheta, c = 1/2 on the diagonal
inline int gp_grad_dmax(int d) { return d <= 8 ? 8 : (d <= 16 ? 16 : 32); }
hs_status launch_gp_grad(hs_ctx ctx, const double* Abar, const double* Xs, const double* alpha, int d, int ard,
                         double sf2, double sn2, double* part, int parts, double* out, cudaStream_t s);
hs_status launch_scale_columns(hs_ctx ctx, const double* X, double* Xs, int d, const double* inv_ell_dev,
                               cudaStream_t s);

// the FP64 factor / solve drivers (hs_solvers.cu)
hs_status factor_driver(hs_ctx ctx, double* A);
hs_status solve_driver(hs_ctx ctx, const double* L, double* b);

}  // namespace hs
