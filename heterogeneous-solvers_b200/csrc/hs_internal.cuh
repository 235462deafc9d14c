// hs_internal.cuh — shared internals of the B200 blocked SPD library: the
// context object, error plumbing and packed-storage index arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/hs_b200.h"

struct hs_ctx_s {
    int device = 0;
    cudaStream_t stream = nullptr;  // caller's stream; nullptr is the CUDA default stream
    int num_sms = 148;

    int64_t N = 0;   // conf::N
    int bsz = 0;     // conf::matrixBlockSize
    int nb = 0;      // blockCountXY

    // grow-only device scratch shared by the kernels that need temporaries
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // grow-only device work vectors of the solver drivers (CG r/d/q, ...)
    void* work = nullptr;
    size_t work_bytes = 0;
    // grow-only workspace of the mixed-precision factor (FP32 factor, split
    // parts, FP64 diagonal blocks, refinement vectors)
    void* mixed = nullptr;
    size_t mixed_bytes = 0;
    // grow-only workspace of the NLML + gradient (factor, adjoint, temporaries)
    void* gpws = nullptr;
    size_t gpws_bytes = 0;
    // grow-only device copies of the host-buffer GP solve (X, K, y, x)
    void* hostws = nullptr;
    size_t hostws_bytes = 0;
    // grow-only workspace of the FP64 triangular solve (inverse diagonal blocks,
    // intermediate vector, sweep flags)
    void* solvews = nullptr;
    size_t solvews_bytes = 0;

    // device words: [0] the smallest failing pivot row (INT64_MAX = none); [1] the
    // bit pattern of the most negative failing pivot of the mixed factor's FP64
    // diagonal blocks (LLONG_MIN, the pattern of -0.0 = none recorded)
    long long* d_info = nullptr;
    // pinned host staging for scalars read back by the solver drivers
    double* h_pinned = nullptr;
    // second stream + events used by the drivers for lookahead
    cudaStream_t side = nullptr;
    // high-priority stream of the FP64 factor's lookahead (its diagonal-block work
    // takes SMs ahead of the trailing update's CTAs)
    cudaStream_t side_hi = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;

    // > 0: matvec, dot and vector updates follow the reference CPU path's exact
    // accumulation order (separate multiply and add, dot products in this many
    // sequential chunks) so that CG reproduces it bit for bit
    int ref_chunks = 0;
    // mixed factor: panels (1, 2 or 4) whose trailing-update products are summed in the
    // tensor cores' accumulator before one add into the FP32 matrix
    // (hs_ctx_set_mixed_accumulation)
    int mixed_acc_panels = 1;
    // mixed factor: look-ahead by a panel group on this many SMs while at least
    // mixed_min_rows rows follow the next group (hs_ctx_set_mixed_lookahead;
    // 0 SMs: look-ahead by one diagonal block only)
    int mixed_side_sms = 16;
    int mixed_min_rows = 24576;

    // kernels launched through this context (all launch sites count)
    int64_t launches = 0;
    // optional per-kernel timing: event pairs recorded on the launching stream
    bool profiling = false;
    struct ProfRec {
        int kernel;
        cudaEvent_t start, stop;
        double flops, bytes;
    };
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    hs_kernel_profile prof_total[HS_KERNEL_COUNT] = {};
};

namespace hs {

void set_error(const std::string& msg);

hs_status cuda_fail(cudaError_t e, const char* what);

#define HS_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t hs_e_ = (call);                                     \
        if (hs_e_ != cudaSuccess) return ::hs::cuda_fail(hs_e_, #call); \
    } while (0)

#define HS_CHECK_LAUNCH(name)                                                 \
    do {                                                                      \
        cudaError_t hs_e_ = cudaGetLastError();                               \
        if (hs_e_ != cudaSuccess) return ::hs::cuda_fail(hs_e_, name);        \
    } while (0)

#define HS_REQUIRE(cond, msg)                                  \
    do {                                                       \
        if (!(cond)) {                                         \
            ::hs::set_error(std::string(__func__) + ": " + (msg)); \
            return HS_ERR_INVALID_ARG;                         \
        }                                                      \
    } while (0)

hs_status require_ctx(hs_ctx ctx, const char* fn);
void set_i64_dev(long long* p, long long v, cudaStream_t s);

// per-kernel timing around one launch (no-ops unless ctx->profiling)
void prof_begin(hs_ctx ctx, cudaStream_t s, int kernel);
void prof_end(hs_ctx ctx, cudaStream_t s, int kernel, double flops, double bytes);
// makes sure at least `bytes` of scratch are available (stream-ordered safe:
// the old buffer is released after a stream sync)
hs_status ensure_scratch(hs_ctx ctx, size_t bytes);
hs_status ensure_work(hs_ctx ctx, size_t bytes);
hs_status ensure_mixed(hs_ctx ctx, size_t bytes);
hs_status ensure_gp(hs_ctx ctx, size_t bytes);
hs_status ensure_hostws(hs_ctx ctx, size_t bytes);
hs_status ensure_solvews(hs_ctx ctx, size_t bytes);

// scratch layout: [0, 32 KB) reduction partials, [32 KB, 48 KB) solver scalars,
// [56 KB, 64 KB) small constants; matvec partial blocks start at 64 KB
constexpr size_t kSmallScratch = 64 * 1024;
constexpr size_t kScalarOffset = 32 * 1024;
constexpr size_t kConstOffset = 56 * 1024;
constexpr int kMaxPartials = 4096;

// FP64 tensor-core step: d (8 x 8, two entries a lane) += a (8 x 4, one entry) b (4 x 8,
// one entry); lane l holds a[l/4][l%4], b[l%4][l/4], d[l/4][2(l%4) .. +1]
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// --------------------------------------------------------- packed storage
// block (i,j), i >= j: id = i + nb(nb-1)/2 - (nb-j-1)(nb-j)/2
__host__ __device__ __forceinline__ int64_t block_id(int64_t i, int64_t j, int64_t nb) {
    return i + nb * (nb - 1) / 2 - (nb - j - 1) * (nb - j) / 2;
}
// first block id of block column j
__host__ __device__ __forceinline__ int64_t column_start(int64_t j, int64_t nb) {
    return j * nb - j * (j - 1) / 2;
}
__host__ __device__ __forceinline__ int64_t total_blocks(int64_t nb) { return nb * (nb + 1) / 2; }

// inverse of block_id: column j such that column_start(j) <= id < column_start(j+1)
__host__ __device__ __forceinline__ void block_coords(int64_t id, int64_t nb, int* i_out, int* j_out) {
    int lo = 0, hi = (int)nb - 1;
    while (lo < hi) {  // largest j with column_start(j) <= id
        const int mid = (lo + hi + 1) >> 1;
        if (column_start(mid, nb) <= id) lo = mid; else hi = mid - 1;
    }
    *j_out = lo;
    *i_out = (int)(lo + (id - column_start(lo, nb)));
}

// inverse triangular number: largest r with r(r+1)/2 <= t
__host__ __device__ __forceinline__ int tri_root(int64_t t) {
    int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)(r + 1) * (r + 2) / 2 <= t) ++r;
    while ((int64_t)r * (r + 1) / 2 > t) --r;
    return r;
}

inline size_t block_elems(const hs_ctx ctx) { return (size_t)ctx->bsz * (size_t)ctx->bsz; }

// ---------------------------------------------------------- kernel entry points
// (implemented in the k_*.cu files; all stream-ordered on ctx->stream unless a
// stream is passed)
hs_status launch_potrf(hs_ctx ctx, double* A, int blockID, int blockRow, cudaStream_t s);
hs_status launch_bounded_wait_selftest(hs_ctx ctx, int64_t timeout_ns);
hs_status launch_trsm(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                      cudaStream_t s);
// SYRK over diag blocks [syrkStart, syrkStart+syrkCount) and GEMM over rows
// [gemmStart, gemmStart+gemmCount) of the trailing triangle of column blockRow,
// in one launch (either count may be zero)
hs_status launch_update(hs_ctx ctx, double* A, int blockID, int blockRow, int syrkStart, int syrkCount,
                        int gemmStart, int gemmCount, cudaStream_t s);
// the same update restricted to the trailing block columns [colStart, colEnd)
// (SYRK on their diagonal blocks, GEMM below them)
hs_status launch_update_cols(hs_ctx ctx, double* A, int blockID, int blockRow, int colStart, int colEnd,
                             cudaStream_t s);
// Y_k = L_kk^-T for all nb diagonal blocks of the packed factor L (Y: nb consecutive
// blocks; pad: one block of scratch for a last block with padding rows)
hs_status launch_diag_inverses(hs_ctx ctx, const double* L, double* Y, double* pad, cudaStream_t s);
// a whole forward (L^-1 in) or backward (L^-T in) sweep over the FP64 packed factor in
// one cooperative launch, given Y_k = L_kk^-T (k_vector.cu)
hs_status launch_sweep_whole_f64(hs_ctx ctx, const double* L, const double* Y, const double* in, double* out,
                                 int forward, unsigned epoch, unsigned* flags, int* err, cudaStream_t s);
// X = L^-1 (row major) of one lower-triangular bsz x bsz block; Y is a block of scratch
hs_status launch_diag_inverse(hs_ctx ctx, const double* Lkk, double* Y, double* X, cudaStream_t s);
// B <- B X^T in place for blockCount consecutive blocks from firstBlock (bsz 128 or 256):
// the panel TRSM on the FP64 tensor pipe, given X = L_kk^-1
hs_status launch_trsm_dmma(hs_ctx ctx, double* A, int64_t firstBlock, int blockCount, const double* X,
                           cudaStream_t s);
hs_status launch_symv(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0, int nbi,
                      int nbj, int reset, double* dot_with /*nullable: also dot(result, dot_with) */,
                      double* dot_out, cudaStream_t s);
hs_status launch_trsv(hs_ctx ctx, const double* A, double* b, int blockRow, int blockID, int transposed,
                      cudaStream_t s);
hs_status launch_column_update(hs_ctx ctx, const double* A, double* b, int blockStart, int blockCount,
                               int blockRow, int blockID, int transposed, cudaStream_t s);
hs_status launch_dot(hs_ctx ctx, const double* x, const double* y, double* result, int64_t first, int64_t len,
                     cudaStream_t s);
hs_status launch_vec(hs_ctx ctx, int op, const double* x, const double* y, double alpha, double* out,
                     int64_t first, int64_t len, cudaStream_t s);
hs_status launch_symv_partials_at(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0,
                                  int nbi, int nbj, int reset, double* P, cudaStream_t s);
// reference-order forms (ctx->ref_chunks > 0)
hs_status launch_symv_refseq(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0,
                             int nbi, int nbj, int reset, cudaStream_t s);
hs_status launch_dot_refseq(hs_ctx ctx, const double* x, const double* y, double* result, int64_t first,
                            int64_t len, int chunks, cudaStream_t s);
hs_status launch_rbf_assemble(hs_ctx ctx, double* A, const double* X, int d, const double* ell_host, int n_ell,
                              double sf2, double sn2, cudaStream_t s);

}  // namespace hs
