// hs_mixed.cuh — internals shared by the mixed-precision factor (k_mixed.cu)
// and its refinement / preconditioned-CG drivers (hs_mixed.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "hs_internal.cuh"

namespace hs {

// device workspace of one mixed-precision factorization
struct MixedWork {
    float* A32 = nullptr;   // packed FP32 copy of K; its off-diagonal blocks end as L (used by the solves)
    float* LO = nullptr;    // low parts of two panel groups (slot set p: slots p nb..), then L_kk^-1 hi / lo
    double* Ld = nullptr;   // FP64 diagonal blocks of L (nb blocks; the lower triangle is written)
    double* Yinv = nullptr; // FP64 inverse diagonal blocks, Y_k = L_kk^-T (nb blocks)
    double* S = nullptr;    // FP64 scratch block (POTRF)
    __nv_bfloat16* P16 = nullptr;  // 16-bit (BF16 or FP16) split of two panel groups: set p hi blocks 2p nb.., lo (2p+1) nb..
    int* err = nullptr;     // [0] tensor-core tile timeout, [1] triangular-sweep timeout
    unsigned long long* tile_ctr = nullptr;  // tile counters of the trailing-update launches (zeroed per factor)
    unsigned* flags = nullptr;  // per block row: epoch of the sweep that published it
    unsigned epoch = 0;         // last sweep launched (flags are cleared when it restarts at 0)
    float* Y32 = nullptr;       // FP32 copy of Yinv for the sweeps, in the P16 area once the factor is done
    CUtensorMap mA128, mL128, mL32;      // 128-byte swizzle, 32-wide K boxes of 128 / 32 rows (TRSM)
    CUtensorMap mU128, mUB, mV128, mVB;  // K boxes of 128 bytes over A32 / LO (TF32 update)
    CUtensorMap mP128, mPB;              // K boxes of 128 bytes over P16 (BF16 / FP16 update)
    CUtensorMap mC32;                    // 32x32 FP32 boxes over A32 (TMA reduce of the update's C tiles)
};

size_t mixed_workspace_bytes(int64_t N, int bsz);
hs_status mixed_bind(hs_ctx ctx, void* ws, MixedWork* w);
// shift != 0: factor K + shift*I
// fro_part (non-null): also the squared Frobenius norm of K (off-diagonal blocks twice)
// as mixed_fro_grid(blocks) CTA partials
// maxdiag: the largest diagonal entry of the matrix factored (with its shift); it sets
// the power-of-two scale of the FP16 split and is not read by the other precisions
// acc_panels: panels (1, 2 or 4, the panel group) whose trailing-update products are
// summed in the tensor cores' accumulator before one add into the FP32 matrix (fewer:
// more accurate factor, more adds)
hs_status mixed_factor(hs_ctx ctx, const double* K64, MixedWork& w, cudaStream_t s, double shift = 0.0,
                       int precision = HS_PRECISION_TF32X3, double* fro_part = nullptr, double maxdiag = 0.0,
                       int acc_panels = 4);
int mixed_fro_grid(int64_t blocks);
hs_status mixed_check_error(hs_ctx ctx, const MixedWork& w);
// b <- (L L^T)^-1 b with the mixed factor (tmp: intermediate)
hs_status mixed_apply(hs_ctx ctx, MixedWork& w, double* b, double* tmp, cudaStream_t s);
// the mixed-precision solve behind hs_mixed_solve (workspace kept by the context)
// (acc_panels <= 0: the context's setting, hs_ctx_set_mixed_accumulation)
hs_status mixed_solve_impl(hs_ctx ctx, const double* K, const double* b, double* x, int precision, double tol,
                           int max_steps, hs_mixed_report* out, int acc_panels = 0);

// TRSM of `items` bsz x bsz FP64 blocks stored contiguously at B against the
// lower triangle L (bsz x bsz): B <- B L^-T
hs_status launch_trsm_on(hs_ctx ctx, const double* L, int n, double* B, int items, cudaStream_t s);
// a whole forward / backward sweep in one cooperative launch: out = L^-1 in or
// L^-T in (block rows published through flags[] with value `epoch`; *err = 2 on a
// wait that timed out)
hs_status launch_mixed_sweep_whole(hs_ctx ctx, const float* A32, const float* Y, const double* in, double* out,
                                   int forward, unsigned epoch, unsigned* flags, int* err, cudaStream_t s);
// column update reading FP32 blocks (accumulation in FP64)
hs_status launch_column_update_f32(hs_ctx ctx, const float* A32, double* b, int blockStart, int blockCount,
                                   int blockRow, int blockID, int transposed, cudaStream_t s);

}  // namespace hs
